// philox_pin.cu -- test helper (built by tests/test_gpu_philox.py): runs the
// library's Philox4x32-10 and cuRAND's on the same counters and keys.
#include <curand_kernel.h>

#include "../../mrm_b200/csrc/philox.cuh"

__global__ void pin_kernel(const unsigned int* in, unsigned int* mine, unsigned int* ref, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned int* p = in + 6 * i;
  unsigned int c[4] = {p[0], p[1], p[2], p[3]};
  mrm::philox4x32_10(c, p[4], p[5]);
  const uint4 r = curand_Philox4x32_10(make_uint4(p[0], p[1], p[2], p[3]), make_uint2(p[4], p[5]));
  for (int q = 0; q < 4; ++q) mine[4 * i + q] = c[q];
  ref[4 * i + 0] = r.x;
  ref[4 * i + 1] = r.y;
  ref[4 * i + 2] = r.z;
  ref[4 * i + 3] = r.w;
}

extern "C" int philox_pin(const unsigned int* in_host, int n, unsigned int* mine_host, unsigned int* ref_host) {
  unsigned int *in, *mine, *ref;
  if (cudaMalloc(&in, 6 * sizeof(unsigned int) * n) != cudaSuccess) return 1;
  cudaMalloc(&mine, 4 * sizeof(unsigned int) * n);
  cudaMalloc(&ref, 4 * sizeof(unsigned int) * n);
  cudaMemcpy(in, in_host, 6 * sizeof(unsigned int) * n, cudaMemcpyHostToDevice);
  pin_kernel<<<(n + 127) / 128, 128>>>(in, mine, ref, n);
  cudaMemcpy(mine_host, mine, 4 * sizeof(unsigned int) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(ref_host, ref, 4 * sizeof(unsigned int) * n, cudaMemcpyDeviceToHost);
  const int rc = cudaGetLastError() != cudaSuccess;
  cudaFree(in);
  cudaFree(mine);
  cudaFree(ref);
  return rc;
}
