// mrm_gpu.cu -- host engine and C ABI (include/mrm_gpu.h) of the B200
// grain-dynamics path.  See kernels.cuh for the per-step launch sequence.
//
// Engine: one CUDA stream, a set of runs (media realisations), one task table
// over every active run's (layer,row) blocks and spectral column groups, and
// cached CUDA graphs of K Heun steps.  The plain drop-in handle is a run in a
// private engine; the batched/served forms put many runs in one engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mrm_gpu.h"
#include "common.cuh"
#include "kernels.cuh"
#include "tensor.cuh"

using namespace mrm;

namespace {

constexpr int kBlock = 256;
constexpr int kGraphSteps = 16;
constexpr size_t kMaxSmem = 227 * 1024;

int ilog2(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}
bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

struct LayerBufs {
  int n = 0;
  bool uploaded = false;
  void *m = nullptr, *mp = nullptr, *dm = nullptr, *hf = nullptr, *hd = nullptr, *ht = nullptr, *pa = nullptr, *pb = nullptr;
  void* pv = nullptr;
  int *xidx = nullptr, *xnbr = nullptr;
  void* xcoef = nullptr;
  int *uidx = nullptr, *unbr = nullptr;
  void* ucoef = nullptr;
  int *lidx = nullptr, *lnbr = nullptr;
  void* lcoef = nullptr;
  void* xst = nullptr;   // V4<R> lattice exchange coefficients (null: CSR form)
  void* ucol = nullptr;  // R columnar interlayer coefficients (null: CSR form)
  void* lcol = nullptr;
  double hdir[3] = {0, 0, 0};
  double t_start = -1e22, t_end = 1e22, s_start = 1.0, s_end = 1.0, scale = 1.0;
  int func = 0;
  double amp = 0, fgamma = 0, phase = 0, param = 0, duty = 0, moddepth = 0, dc = 0;
  double temperature = 0.0, gamma = 1.76e7;
  int thermal = 0;
};

struct Engine;

}  // namespace

struct mrm_gpu {
  Engine* eng = nullptr;
  bool own_engine = false;
  mrm_geom g{};
  int px = 0, py = 0, lgpx = 0, lgpy = 0, nl = 0;
  LayerBufs L[MRM_MAX_LAYERS];
  void* spech = nullptr;
  void* specx = nullptr;
  void* tens = nullptr;
  bool tensor_ready = false;
  bool demag = true;
  double tensor_resid = 0.0, tensor_kept = 0.0;
  double dt = 1e-13, t_base = 0.0;
  long long step_base = 0, step = 0, step_end = 0;
  unsigned long long seed = 1;
  bool active = true;
  bool spec_valid = false;
  bool has_stats = false;
  int slot = -1;
  int row_task0 = 0, nrow_tasks = 0;
  std::string err;
};

namespace {

struct Engine {
  int prec = MRM_FP32;
  int dev = 0;
  cudaStream_t st = nullptr;
  std::vector<mrm_gpu*> runs;
  void* d_runs = nullptr;  // RunDev<R>[cap]
  int runs_cap = 0;
  Task* d_rtasks = nullptr;
  Task* d_ctasks = nullptr;
  int nrt = 0, nct = 0, rt_cap = 0, ct_cap = 0;
  size_t smem_row = 0, smem_col = 0;
  int rowcfg = 0;
  bool pref = true;  // row kernel gathers grain inputs up front (few blocks per SM)
  double* d_part = nullptr;
  int part_cap = 0;
  StatsDev* d_stats = nullptr;
  StatsDev* h_stats = nullptr;  // pinned
  int stats_cap = 0;
  void* d_tw = nullptr;  // Cx<R>[kTwN]
  bool tables_dirty = true;
  bool desc_dirty = true;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;  // (steps, with stats)
  std::string err;
  bool init_done = false;
};

size_t relem(int prec) { return prec == MRM_FP64 ? sizeof(double) : sizeof(float); }

int set_err(std::string* dst, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (dst) *dst = buf;
  return code;
}

#define CK(call)                                                                           \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      int code_ = (e_ == cudaErrorMemoryAllocation) ? MRM_ERR_NOMEM : MRM_ERR_CUDA;        \
      return set_err(errp, code_, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),  \
                     __FILE__, __LINE__);                                                  \
    }                                                                                      \
  } while (0)

int dmalloc(std::string* errp, void** p, size_t bytes) {
  CK(cudaMalloc(p, bytes ? bytes : 16));
  CK(cudaMemset(*p, 0, bytes ? bytes : 16));
  return MRM_OK;
}

void dfree(void*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}
template <typename T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

void clear_graphs(Engine* e) {
  for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
  e->graphs.clear();
}

int engine_init(Engine* e, int prec, int dev) {
  std::string* errp = &e->err;
  e->prec = prec;
  e->dev = dev;
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (dev < 0 || dev >= ndev) return set_err(errp, MRM_ERR_ARG, "device %d out of range (%d)", dev, ndev);
  CK(cudaSetDevice(dev));
  CK(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
  // twiddles e^{-2 pi i k / 4096}, computed in FP64
  std::vector<double> tw(2 * kTwN);
  for (int k = 0; k < kTwN; ++k) {
    double a = -2.0 * M_PI * (double)k / (double)kTwN;
    tw[2 * k] = std::cos(a);
    tw[2 * k + 1] = std::sin(a);
  }
  if (prec == MRM_FP64) {
    int rc = dmalloc(errp, &e->d_tw, sizeof(double) * 2 * kTwN);
    if (rc) return rc;
    CK(cudaMemcpy(e->d_tw, tw.data(), sizeof(double) * 2 * kTwN, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> twf(2 * kTwN);
    for (int k = 0; k < 2 * kTwN; ++k) twf[k] = (float)tw[k];
    int rc = dmalloc(errp, &e->d_tw, sizeof(float) * 2 * kTwN);
    if (rc) return rc;
    CK(cudaMemcpy(e->d_tw, twf.data(), sizeof(float) * 2 * kTwN, cudaMemcpyHostToDevice));
  }
  e->init_done = true;
  return MRM_OK;
}

void engine_free(Engine* e) {
  if (!e) return;
  if (e->init_done) cudaSetDevice(e->dev);
  clear_graphs(e);
  dfree(e->d_runs);
  dfree(e->d_rtasks);
  dfree(e->d_ctasks);
  dfree(e->d_part);
  dfree(e->d_stats);
  if (e->h_stats) cudaFreeHost(e->h_stats);
  e->h_stats = nullptr;
  dfree(e->d_tw);
  if (e->st) cudaStreamDestroy(e->st);
  e->st = nullptr;
}

// ---------------- FFT grid / task shapes ----------------
void fft_grid(const mrm_geom& g, int* px, int* py) {
  if (g.boundary == MRM_OPEN) {
    *px = 1 << ilog2(2 * g.nx);
    *py = 1 << ilog2(2 * g.ny);
  } else {
    *px = g.nx;
    *py = g.ny;
  }
}

int rows_per_task(const mrm_gpu* r) {
  if (r->g.nx >= kBlock) return 1;
  return std::max(1, std::min(r->g.ny, kBlock / std::max(1, r->g.nx)));
}
// columns per column task: enough sequences for one radix-16 butterfly per thread
int cols_per_task(const mrm_gpu* r) {
  int ph = r->px / 2 + 1;
  return std::max(1, std::min(ph, kBlock * 16 / (3 * r->nl * r->py)));
}
size_t cx_bytes(int prec) { return 2 * relem(prec); }
// shared memory: twiddle table of the transform length + two padded ping-pong buffers
size_t row_smem(const mrm_gpu* r, int prec) {
  return ((size_t)r->px + 2ull * rows_per_task(r) * 3 * fft_stride(r->px / 2)) * cx_bytes(prec);
}
size_t col_smem(const mrm_gpu* r, int prec) {
  size_t b = ((size_t)r->py + 2ull * cols_per_task(r) * r->nl * 3 * fft_stride(r->py)) * cx_bytes(prec);
  if (prec == MRM_FP32) {  // packed tensor slice (kernels.cuh: tens_slice_fits)
    const int reals = cols_per_task(r) * r->nl * r->nl * 9 * (r->py / 2 + 1);
    if (tens_slice_fits<float>(reals)) b += (size_t)reals * sizeof(float);
  }
  return b;
}
// row-kernel shape: grains per thread x block size
int row_config(int max_grains) {
  if (max_grains <= 256) return 0;   // GPT 1, 256 threads
  if (max_grains <= 512) return 1;   // GPT 2, 256 threads
  return 2;                          // GPT 2, 512 threads (<= 1024 grains)
}
size_t tensor_bytes(const mrm_gpu* r) {
  const size_t ph = r->px / 2 + 1, npair = (size_t)r->nl * r->nl;
  if (r->g.precision == MRM_FP64) return ph * npair * 9 * r->py * 2 * sizeof(double);
  return ph * npair * 9 * (r->py / 2 + 1) * sizeof(float);
}

int validate_geom(const mrm_geom* g, std::string* errp) {
  if (!g) return set_err(errp, MRM_ERR_ARG, "geometry is NULL");
  if (g->nx < 2 || g->ny < 2) return set_err(errp, MRM_ERR_ARG, "nx, ny must be >= 2");
  if (g->n_lay < 1 || g->n_lay > MRM_MAX_LAYERS)
    return set_err(errp, MRM_ERR_ARG, "n_lay must be in 1..%d", MRM_MAX_LAYERS);
  if (g->boundary != MRM_PERIODIC && g->boundary != MRM_OPEN)
    return set_err(errp, MRM_ERR_ARG, "boundary must be MRM_PERIODIC or MRM_OPEN");
  if (g->precision != MRM_FP32 && g->precision != MRM_FP64)
    return set_err(errp, MRM_ERR_ARG, "precision must be MRM_FP32 or MRM_FP64");
  if (!(g->dx > 0 && g->dy > 0)) return set_err(errp, MRM_ERR_ARG, "dx, dy must be > 0");
  for (int l = 0; l < g->n_lay; ++l)
    if (!(g->dz[l] > 0)) return set_err(errp, MRM_ERR_ARG, "dz[%d] must be > 0", l);
  if (g->nx > 1024)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "rows of more than 1024 grains are not supported (nx=%d)", g->nx);
  if (g->boundary == MRM_PERIODIC && (!is_pow2(g->nx) || !is_pow2(g->ny)))
    return set_err(errp, MRM_ERR_UNSUPPORTED,
                   "periodic demag needs power-of-two nx, ny on this path (got %d x %d)", g->nx, g->ny);
  int px, py;
  fft_grid(*g, &px, &py);
  if (px > kTwN || py > kTwN || px < 4 || py < 2)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "FFT grid %d x %d outside 4..%d", px, py, kTwN);
  mrm_gpu tmp;
  tmp.g = *g;
  tmp.px = px;
  tmp.py = py;
  tmp.nl = g->n_lay;
  if (row_smem(&tmp, g->precision) > kMaxSmem || col_smem(&tmp, g->precision) > kMaxSmem)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "FFT grid %d x %d x %d layers exceeds shared memory", px,
                   py, g->n_lay);
  return MRM_OK;
}

// ---------------- descriptors ----------------
template <typename R>
RunDev<R> make_desc(const mrm_gpu* r) {
  RunDev<R> d;
  std::memset(&d, 0, sizeof(d));
  d.nx = r->g.nx;
  d.ny = r->g.ny;
  d.nl = r->nl;
  d.px = r->px;
  d.py = r->py;
  d.lgpx = r->lgpx;
  d.lgpy = r->lgpy;
  d.demag = (r->demag && r->tensor_ready) ? 1 : 0;
  d.ncomp = 9;
  d.dt = r->dt;
  d.t_base = r->t_base;
  d.step_base = r->step_base;
  d.step = r->step;
  d.step_end = r->step_end;
  d.seed = r->seed;
  d.active = r->active ? 1 : 0;
  d.row_task0 = r->row_task0;
  d.nrow_tasks = r->nrow_tasks;
  d.spech = static_cast<Cx<R>*>(r->spech);
  d.specx = static_cast<Cx<R>*>(r->specx);
  d.tens = static_cast<const R*>(r->tens);
  for (int l = 0; l < r->nl; ++l) {
    const LayerBufs& b = r->L[l];
    LayerDev<R>& o = d.L[l];
    o.m = static_cast<V4<R>*>(b.m);
    o.mp = static_cast<V4<R>*>(b.mp);
    o.dm = static_cast<V4<R>*>(b.dm);
    o.hf = static_cast<V4<R>*>(b.hf);
    o.hd = static_cast<V4<R>*>(b.hd);
    o.ht = static_cast<V4<R>*>(b.ht);
    o.pa = static_cast<const V4<R>*>(b.pa);
    o.pb = static_cast<const V4<R>*>(b.pb);
    o.pv = static_cast<const V4<double>*>(b.pv);
    o.xidx = b.xidx;
    o.xnbr = b.xnbr;
    o.xcoef = static_cast<const R*>(b.xcoef);
    o.uidx = b.uidx;
    o.unbr = b.unbr;
    o.ucoef = static_cast<const R*>(b.ucoef);
    o.lidx = b.lidx;
    o.lnbr = b.lnbr;
    o.lcoef = static_cast<const R*>(b.lcoef);
    o.xst = static_cast<const V4<R>*>(b.xst);
    o.ucol = static_cast<const R*>(b.ucol);
    o.lcol = static_cast<const R*>(b.lcol);
    for (int a = 0; a < 3; ++a) o.hdir[a] = b.hdir[a];
    o.t_start = b.t_start;
    o.t_end = b.t_end;
    o.s_start = b.s_start;
    o.s_end = b.s_end;
    o.scale = b.scale;
    o.func = b.func;
    o.amp = b.amp;
    o.fgamma = b.fgamma;
    o.phase = b.phase;
    o.param = b.param;
    o.duty = b.duty;
    o.moddepth = b.moddepth;
    o.dc = b.dc;
    o.temperature = b.temperature;
    o.gamma = b.gamma;
    o.thermal = b.thermal;
    o.n = b.n;
  }
  return d;
}

size_t desc_size(int prec) { return prec == MRM_FP64 ? sizeof(RunDev<double>) : sizeof(RunDev<float>); }

int push_descs(Engine* e) {
  std::string* errp = &e->err;
  const int n = (int)e->runs.size();
  const size_t ds = desc_size(e->prec);
  if (n > e->runs_cap) {
    dfree(e->d_runs);
    int cap = std::max(n, 2 * e->runs_cap);
    int rc = dmalloc(errp, &e->d_runs, ds * cap);
    if (rc) return rc;
    e->runs_cap = cap;
    clear_graphs(e);
  }
  std::vector<unsigned char> host(ds * std::max(1, n));
  for (int i = 0; i < n; ++i) {
    e->runs[i]->slot = i;
    if (e->prec == MRM_FP64) {
      RunDev<double> d = make_desc<double>(e->runs[i]);
      std::memcpy(host.data() + i * ds, &d, ds);
    } else {
      RunDev<float> d = make_desc<float>(e->runs[i]);
      std::memcpy(host.data() + i * ds, &d, ds);
    }
  }
  if (n) CK(cudaMemcpyAsync(e->d_runs, host.data(), ds * n, cudaMemcpyHostToDevice, e->st));
  e->desc_dirty = false;
  return MRM_OK;
}

int build_tables(Engine* e) {
  std::string* errp = &e->err;
  std::vector<Task> rt, ct;
  size_t srow = 0, scol = 0;
  int maxg = 1;
  for (size_t i = 0; i < e->runs.size(); ++i) {
    mrm_gpu* r = e->runs[i];
    r->slot = (int)i;
    r->row_task0 = (int)rt.size();
    const int rpt = rows_per_task(r);
    for (int l = 0; l < r->nl; ++l)
      for (int j = 0; j < r->g.ny; j += rpt) rt.push_back(make_int4((int)i, l, j, std::min(rpt, r->g.ny - j)));
    r->nrow_tasks = (int)rt.size() - r->row_task0;
    maxg = std::max(maxg, rpt * r->g.nx);
    srow = std::max(srow, row_smem(r, e->prec));
    if (r->demag && r->tensor_ready) {
      const int cpt = cols_per_task(r), ph = r->px / 2 + 1;
      for (int k = 0; k < ph; k += cpt) ct.push_back(make_int4((int)i, k, std::min(cpt, ph - k), 0));
      scol = std::max(scol, col_smem(r, e->prec));
    }
  }
  e->nrt = (int)rt.size();
  e->nct = (int)ct.size();
  if (e->nrt > e->rt_cap) {
    dfree(e->d_rtasks);
    e->rt_cap = std::max(e->nrt, 2 * e->rt_cap);
    int rc = dmalloc(errp, (void**)&e->d_rtasks, sizeof(Task) * e->rt_cap);
    if (rc) return rc;
  }
  if (e->nct > e->ct_cap) {
    dfree(e->d_ctasks);
    e->ct_cap = std::max(e->nct, 2 * e->ct_cap);
    int rc = dmalloc(errp, (void**)&e->d_ctasks, sizeof(Task) * e->ct_cap);
    if (rc) return rc;
  }
  if (e->nrt > e->part_cap) {
    dfree(e->d_part);
    e->part_cap = std::max(e->nrt, 2 * e->part_cap);
    int rc = dmalloc(errp, (void**)&e->d_part, sizeof(double) * kNPart * e->part_cap);
    if (rc) return rc;
  }
  const int nr = (int)e->runs.size();
  if (nr > e->stats_cap) {
    dfree(e->d_stats);
    if (e->h_stats) cudaFreeHost(e->h_stats);
    e->h_stats = nullptr;
    e->stats_cap = std::max(nr, 2 * e->stats_cap);
    int rc = dmalloc(errp, (void**)&e->d_stats, sizeof(StatsDev) * e->stats_cap);
    if (rc) return rc;
    CK(cudaMallocHost((void**)&e->h_stats, sizeof(StatsDev) * e->stats_cap));
    std::memset(e->h_stats, 0, sizeof(StatsDev) * e->stats_cap);
  }
  if (e->nrt) CK(cudaMemcpyAsync(e->d_rtasks, rt.data(), sizeof(Task) * e->nrt, cudaMemcpyHostToDevice, e->st));
  if (e->nct) CK(cudaMemcpyAsync(e->d_ctasks, ct.data(), sizeof(Task) * e->nct, cudaMemcpyHostToDevice, e->st));
  e->smem_row = srow;
  e->smem_col = scol;
  e->rowcfg = row_config(maxg);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->dev);
  // enough row blocks to fill four per SM: the throughput variant wins
  e->pref = !(e->prec == MRM_FP32 && e->rowcfg <= 1 && e->nrt >= 4 * nsm);
  clear_graphs(e);
  e->tables_dirty = false;
  e->desc_dirty = true;
  return MRM_OK;
}

// The dynamic shared-memory limit is a per-function attribute shared by every
// engine in the process, so it only ever grows.
template <typename K>
int raise_smem(K* kern, size_t bytes, std::string* errp) {
  static std::map<const void*, size_t> set;
  size_t& cur = set[(const void*)kern];
  if (bytes <= cur) return MRM_OK;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  cur = bytes;
  return MRM_OK;
}

// Launch with programmatic stream serialization: the kernel may start while its
// predecessor drains; it runs its independent prologue and then waits
// (griddepcontrol.wait) for the predecessor's results.
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

template <typename R, int GPT, int BLK, bool PREF>
int set_row_attrs(size_t rs, std::string* errp) {
  int rc = 0;
  rc |= raise_smem(row_kernel<R, kInit, false, GPT, BLK, PREF>, rs, errp);
  rc |= raise_smem(row_kernel<R, kPred, false, GPT, BLK, PREF>, rs, errp);
  rc |= raise_smem(row_kernel<R, kCorr, false, GPT, BLK, PREF>, rs, errp);
  rc |= raise_smem(row_kernel<R, kCorr, true, GPT, BLK, PREF>, rs, errp);
  rc |= raise_smem(row_kernel<R, kEval, false, GPT, BLK, PREF>, rs, errp);
  return rc;
}

template <typename R>
int set_smem_attrs(Engine* e) {
  std::string* errp = &e->err;
  const size_t rs = std::max<size_t>(e->smem_row, 16), cs = std::max<size_t>(e->smem_col, 16);
  int rc = 0;
  if (e->rowcfg == 0) rc |= set_row_attrs<R, 1, 256, true>(rs, errp);
  else if (e->rowcfg == 1) rc |= set_row_attrs<R, 2, 256, true>(rs, errp);
  else rc |= set_row_attrs<R, 2, 512, true>(rs, errp);
  if constexpr (sizeof(R) == sizeof(float)) {
    if (e->rowcfg == 0) rc |= set_row_attrs<R, 1, 256, false>(rs, errp);
    else if (e->rowcfg == 1) rc |= set_row_attrs<R, 2, 256, false>(rs, errp);
  }
  rc |= raise_smem(col_kernel<R, true, kBlock>, cs, errp);
  rc |= raise_smem(col_kernel<R, false, kBlock>, cs, errp);
  return rc ? MRM_ERR_CUDA : MRM_OK;
}

template <typename R, int GPT, int BLK, bool PREF>
void launch_row_cfg(Engine* e, int stage, int istep, int flags) {
  const RunDev<R>* runs = static_cast<const RunDev<R>*>(e->d_runs);
  const Cx<R>* tw = static_cast<const Cx<R>*>(e->d_tw);
  const dim3 g(e->nrt), b(BLK);
  const size_t sm = e->smem_row;
  switch (stage) {
    case kInit:
      launch_pdl(row_kernel<R, kInit, false, GPT, BLK, PREF>, g, b, sm, e->st, runs, e->d_rtasks, tw, istep, flags, e->d_part);
      break;
    case kPred:
      launch_pdl(row_kernel<R, kPred, false, GPT, BLK, PREF>, g, b, sm, e->st, runs, e->d_rtasks, tw, istep, flags, e->d_part);
      break;
    case kCorr:
      if (flags & kFlagStats)
        launch_pdl(row_kernel<R, kCorr, true, GPT, BLK, PREF>, g, b, sm, e->st, runs, e->d_rtasks, tw, istep, flags, e->d_part);
      else
        launch_pdl(row_kernel<R, kCorr, false, GPT, BLK, PREF>, g, b, sm, e->st, runs, e->d_rtasks, tw, istep, flags, e->d_part);
      break;
    default:
      launch_pdl(row_kernel<R, kEval, false, GPT, BLK, PREF>, g, b, sm, e->st, runs, e->d_rtasks, tw, istep, flags, e->d_part);
      break;
  }
}

template <typename R>
void launch_row(Engine* e, int stage, int istep, int flags) {
  if (!e->nrt) return;
  if constexpr (sizeof(R) == sizeof(float)) {
    if (!e->pref) {
      if (e->rowcfg == 0) launch_row_cfg<R, 1, 256, false>(e, stage, istep, flags);
      else launch_row_cfg<R, 2, 256, false>(e, stage, istep, flags);
      return;
    }
  }
  if (e->rowcfg == 0) launch_row_cfg<R, 1, 256, true>(e, stage, istep, flags);
  else if (e->rowcfg == 1) launch_row_cfg<R, 2, 256, true>(e, stage, istep, flags);
  else launch_row_cfg<R, 2, 512, true>(e, stage, istep, flags);
}

template <typename R>
void launch_col(Engine* e, int istep, int flags) {
  if (!e->nct) return;
  constexpr bool packed = sizeof(R) == sizeof(float);
  launch_pdl(col_kernel<R, packed, kBlock>, dim3(e->nct), dim3(kBlock), e->smem_col, e->st,
             static_cast<const RunDev<R>*>(e->d_runs), (const Task*)e->d_ctasks,
             static_cast<const Cx<R>*>(e->d_tw), istep, flags);
}

template <typename R>
void enqueue_steps(Engine* e, int k, bool stats) {
  for (int i = 0; i < k; ++i) {
    const int last = (stats && i == k - 1) ? (kFlagStats | kFlagStoreField) : 0;
    launch_row<R>(e, kPred, i, 0);
    launch_col<R>(e, i, 0);
    launch_row<R>(e, kCorr, i, last);
    launch_col<R>(e, i, 0);
  }
  const int nr = (int)e->runs.size();
  launch_pdl(advance_kernel<R>, dim3((nr + 127) / 128), dim3(128), 0, e->st,
             static_cast<RunDev<R>*>(e->d_runs), nr, k);
  if (stats)
    launch_pdl(finalize_stats_kernel<R>, dim3(nr), dim3(256), 0, e->st,
               static_cast<const RunDev<R>*>(e->d_runs), (const Task*)e->d_rtasks,
               (const double*)e->d_part, e->d_stats, nr);
}

template <typename R>
int ensure_ready(Engine* e) {
  std::string* errp = &e->err;
  CK(cudaSetDevice(e->dev));
  if (e->tables_dirty) {
    int rc = build_tables(e);
    if (rc) return rc;
    rc = set_smem_attrs<R>(e);
    if (rc) return rc;
  }
  if (e->desc_dirty) {
    int rc = push_descs(e);
    if (rc) return rc;
  }
  // establish spec = H^(m) for runs whose state or tensor changed
  bool need = false;
  for (auto* r : e->runs)
    if (r->active && !r->spec_valid) need = true;
  if (need) {
    launch_row<R>(e, kInit, 0, kFlagForce);
    launch_col<R>(e, 0, kFlagForce);
    CK(cudaGetLastError());
    for (auto* r : e->runs)
      if (r->active) r->spec_valid = true;
  }
  return MRM_OK;
}

template <typename R>
int run_steps(Engine* e, int nsteps) {
  std::string* errp = &e->err;
  int rc = ensure_ready<R>(e);
  if (rc) return rc;
  int left = nsteps;
  while (left > 0) {
    const int k = std::min(left, kGraphSteps);
    const bool stats = (left == k);  // reductions only on the call's last step
    auto key = std::make_pair(k, stats ? 1 : 0);
    auto it = e->graphs.find(key);
    if (it == e->graphs.end()) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
      enqueue_steps<R>(e, k, stats);
      cudaError_t ce = cudaStreamEndCapture(e->st, &g);
      if (ce != cudaSuccess) return set_err(errp, MRM_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
      cudaGraphExec_t ge;
      ce = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) return set_err(errp, MRM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
      it = e->graphs.emplace(key, ge).first;
    }
    CK(cudaGraphLaunch(it->second, e->st));
    left -= k;
  }
  CK(cudaGetLastError());
  // mirror the device-side step counters
  for (auto* r : e->runs) {
    if (!r->active) continue;
    long long rem = std::max(0LL, r->step_end - r->step);
    r->step += std::min<long long>(rem, nsteps);
  }
  return MRM_OK;
}

int engine_step(Engine* e, int nsteps) {
  if (e->prec == MRM_FP64) return run_steps<double>(e, nsteps);
  return run_steps<float>(e, nsteps);
}

template <typename R>
int engine_eval(Engine* e) {
  std::string* errp = &e->err;
  int rc = ensure_ready<R>(e);
  if (rc) return rc;
  launch_row<R>(e, kEval, 0, kFlagForce | kFlagStoreField);
  CK(cudaGetLastError());
  return MRM_OK;
}

// ---------------- run buffers ----------------
int run_alloc(mrm_gpu* r) {
  std::string* errp = &r->err;
  const size_t re = relem(r->g.precision);
  const int ph = r->px / 2 + 1, pyh = r->py / 2 + 1;
  int rc = dmalloc(errp, &r->spech, (size_t)r->nl * 3 * r->g.ny * ph * 2 * re);
  if (rc) return rc;
  rc = dmalloc(errp, &r->specx, (size_t)r->nl * 3 * r->g.ny * ph * 2 * re);
  if (rc) return rc;
  (void)pyh;
  rc = dmalloc(errp, &r->tens, tensor_bytes(r));
  if (rc) return rc;
  const size_t n = (size_t)r->g.nx * r->g.ny;
  for (int l = 0; l < r->nl; ++l) {
    LayerBufs& b = r->L[l];
    b.n = (int)n;
    void** v4s[] = {&b.m, &b.mp, &b.dm, &b.hf, &b.hd, &b.ht, &b.pa, &b.pb};
    for (void** p : v4s) {
      rc = dmalloc(errp, p, n * 4 * re);
      if (rc) return rc;
    }
    rc = dmalloc(errp, &b.pv, n * 4 * sizeof(double));
    if (rc) return rc;
  }
  return MRM_OK;
}

void run_free(mrm_gpu* r) {
  dfree(r->spech);
  dfree(r->specx);
  dfree(r->tens);
  for (int l = 0; l < MRM_MAX_LAYERS; ++l) {
    LayerBufs& b = r->L[l];
    dfree(b.m); dfree(b.mp); dfree(b.dm); dfree(b.hf); dfree(b.hd); dfree(b.ht); dfree(b.pa); dfree(b.pb); dfree(b.pv);
    dfree(b.xidx); dfree(b.xnbr); dfree(b.xcoef);
    dfree(b.uidx); dfree(b.unbr); dfree(b.ucoef);
    dfree(b.lidx); dfree(b.lnbr); dfree(b.lcoef);
    dfree(b.xst); dfree(b.ucol); dfree(b.lcol);
  }
}

int64_t footprint(const mrm_geom& g) {
  int px, py;
  fft_grid(g, &px, &py);
  const size_t re = g.precision == MRM_FP64 ? 8 : 4;
  const int64_t n = (int64_t)g.nx * g.ny, nl = g.n_lay;
  const int64_t ph = px / 2 + 1, pyh = py / 2 + 1;
  int64_t b = 2 * nl * 3 * g.ny * ph * 2 * re;
  b += g.precision == MRM_FP64 ? ph * nl * nl * 9 * py * 16 : ph * nl * nl * 9 * pyh * 4;
  b += nl * n * (8 * 4 * re + 4 * 8);
  b += nl * (n + 1) * 4 + nl * n * 4 * (4 + re);  // exchange CSR (4 neighbours)
  if (nl > 1) b += 2 * nl * ((n + 1) * 4 + n * (4 + re));
  return b;
}

mrm_gpu* new_run(Engine* e, const mrm_geom* g, std::string* errp, int* rc) {
  *rc = validate_geom(g, errp);
  if (*rc) return nullptr;
  if (g->precision != e->prec) {
    *rc = set_err(errp, MRM_ERR_ARG, "run precision differs from the batch precision");
    return nullptr;
  }
  cudaSetDevice(e->dev);
  mrm_gpu* r = new mrm_gpu();
  r->eng = e;
  r->g = *g;
  r->nl = g->n_lay;
  fft_grid(*g, &r->px, &r->py);
  r->lgpx = ilog2(r->px);
  r->lgpy = ilog2(r->py);
  r->step_end = (long long)9e18;
  *rc = run_alloc(r);
  if (*rc) {
    if (errp) *errp = r->err;
    run_free(r);
    delete r;
    return nullptr;
  }
  e->runs.push_back(r);
  e->tables_dirty = true;
  e->desc_dirty = true;
  return r;
}

template <typename R>
int upload_csr(mrm_gpu* r, int n, const int32_t* index, const int32_t* grain, const double* coef,
               const double* ms_scale_nbr, int n_nbr, int** didx, int** dnbr, void** dcoef) {
  std::string* errp = &r->err;
  if (index[0] != 0) return set_err(errp, MRM_ERR_ARG, "CSR index(0) must be 0");
  for (int i = 0; i < n; ++i)
    if (index[i + 1] < index[i]) return set_err(errp, MRM_ERR_ARG, "CSR index not monotone at %d", i);
  const int nnz = index[n];
  std::vector<int> nb(std::max(nnz, 1));
  std::vector<R> cf(std::max(nnz, 1));
  for (int q = 0; q < nnz; ++q) {
    const int j = grain[q] - 1;
    if (j < 0 || j >= n_nbr) return set_err(errp, MRM_ERR_ARG, "CSR neighbour %d out of range", grain[q]);
    nb[q] = j;
    cf[q] = (R)(coef[q] * ms_scale_nbr[j]);
  }
  dfree(*didx);
  dfree(*dnbr);
  dfree(*dcoef);
  int rc = dmalloc(errp, (void**)didx, sizeof(int) * (n + 1));
  if (rc) return rc;
  rc = dmalloc(errp, (void**)dnbr, sizeof(int) * std::max(nnz, 1));
  if (rc) return rc;
  rc = dmalloc(errp, dcoef, sizeof(R) * std::max(nnz, 1));
  if (rc) return rc;
  CK(cudaMemcpy(*didx, index, sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(*dnbr, nb.data(), sizeof(int) * std::max(nnz, 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(*dcoef, cf.data(), sizeof(R) * std::max(nnz, 1), cudaMemcpyHostToDevice));
  return MRM_OK;
}

// host copies of ms_scale per layer (neighbour scaling of exchange coefficients)
struct HostLayerCache {
  std::vector<double> ms_scale;
};
std::map<const mrm_gpu*, std::vector<HostLayerCache>>& host_cache() {
  static std::map<const mrm_gpu*, std::vector<HostLayerCache>> m;
  return m;
}

template <typename R>
int upload_layer_t(mrm_gpu* r, int l, int n, const double* ms, const double* vol, const double* axis,
                   const double* hk, const double* hk_scale, const double* ms_scale,
                   const double* alpha_scale, double alpha, double gamma, double floor_ms,
                   const int32_t* g2ci, const int32_t* g2c, const int32_t* hxi, const int32_t* hxg,
                   const double* hx) {
  std::string* errp = &r->err;
  const int nx = r->g.nx, ny = r->g.ny;
  if (n != nx * ny)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "layer %d: %d grains on a %dx%d grid; this path needs one grain per cell", l, n, nx, ny);
  if (!ms || !vol || !axis || !hk || !hk_scale || !ms_scale || !alpha_scale || !g2ci || !g2c)
    return set_err(errp, MRM_ERR_ARG, "layer %d: NULL array", l);
  for (int g = 0; g < n; ++g) {
    if (g2ci[g] != g || g2ci[g + 1] != g + 1)
      return set_err(errp, MRM_ERR_UNSUPPORTED, "grain %d spans %d cells; multi-cell grains are not supported", g + 1, g2ci[g + 1] - g2ci[g]);
    const int i = g2c[2 * g] - 1, j = g2c[2 * g + 1] - 1;
    if (i != g % nx || j != g / nx)
      return set_err(errp, MRM_ERR_UNSUPPORTED, "grain %d sits at cell (%d,%d), expected (%d,%d)", g + 1, i + 1, j + 1, g % nx + 1, g / nx + 1);
  }
  const double kB = 1.380662e-16;  // field.f90:407
  const double tsig = std::sqrt(2.0 * kB * alpha / gamma);
  std::vector<R> pa(4 * n), pb(4 * n);
  std::vector<double> pv(4 * n);
  for (int g = 0; g < n; ++g) {
    pa[4 * g + 0] = (R)axis[3 * g];
    pa[4 * g + 1] = (R)axis[3 * g + 1];
    pa[4 * g + 2] = (R)axis[3 * g + 2];
    const double hks = hk_scale[g] > 0.0 ? hk_scale[g] : 0.0;  // get_uni_hk returns 0 for hk_scale <= 0
    pa[4 * g + 3] = (R)(hk[2 * g] * hks);
    pb[4 * g + 0] = (R)(ms[g] * ms_scale[g]);
    pb[4 * g + 1] = (R)(hk[2 * g + 1] * hks);
    pb[4 * g + 2] = (R)(alpha * alpha_scale[g]);
    double x = 0.0;  // field.f90:418-419 without the temperature (applied per step)
    if (ms_scale[g] > 0.0) x = alpha_scale[g] / (ms[g] * vol[g] * std::max(floor_ms, ms_scale[g]));
    pb[4 * g + 3] = (R)(std::sqrt(x) * tsig);
    pv[4 * g + 0] = vol[g];
    pv[4 * g + 1] = ms_scale[g];
    pv[4 * g + 2] = ms[g];
    pv[4 * g + 3] = 0.0;
  }
  LayerBufs& b = r->L[l];
  CK(cudaMemcpy(b.pa, pa.data(), sizeof(R) * 4 * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b.pb, pb.data(), sizeof(R) * 4 * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b.pv, pv.data(), sizeof(double) * 4 * n, cudaMemcpyHostToDevice));
  auto& hc = host_cache()[r];
  hc.resize(MRM_MAX_LAYERS);
  hc[l].ms_scale.assign(ms_scale, ms_scale + n);
  dfree(b.xst);
  if (hxi && hxg && hx) {
    int rc = upload_csr<R>(r, n, hxi, hxg, hx, ms_scale, n, &b.xidx, &b.xnbr, &b.xcoef);
    if (rc) return rc;
    // lattice form: every entry is one of the 4 periodic nearest neighbours, each
    // at most once (construct_grain.f90:1281, iwrp) -> per-grain coefficients
    bool lattice = nx >= 3 && ny >= 3;
    std::vector<R> st(lattice ? 4 * (size_t)n : 0, (R)0);
    for (int gi = 0; lattice && gi < n; ++gi) {
      const int i = gi % nx, j = gi / nx;
      const int nbrs[4] = {((j + ny - 1) % ny) * nx + i, j * nx + (i + nx - 1) % nx,
                           j * nx + (i + 1) % nx, ((j + 1) % ny) * nx + i};
      bool used[4] = {false, false, false, false};
      for (int q = hxi[gi]; q < hxi[gi + 1]; ++q) {
        const int nb = hxg[q] - 1;
        int d = -1;
        for (int k = 0; k < 4; ++k)
          if (nbrs[k] == nb && !used[k]) { d = k; break; }
        if (d < 0) { lattice = false; break; }
        used[d] = true;
        st[4 * (size_t)gi + d] = (R)(hx[q] * ms_scale[nb]);
      }
    }
    if (lattice) {
      int rc2 = dmalloc(errp, &b.xst, sizeof(R) * 4 * (size_t)n);
      if (rc2) return rc2;
      CK(cudaMemcpy(b.xst, st.data(), sizeof(R) * 4 * (size_t)n, cudaMemcpyHostToDevice));
    }
  } else {
    dfree(b.xidx); dfree(b.xnbr); dfree(b.xcoef);
  }
  b.gamma = gamma;
  b.uploaded = true;
  r->spec_valid = false;
  r->eng->desc_dirty = true;
  return MRM_OK;
}

std::vector<PairGeom> pair_geoms(const mrm_gpu* r) {
  // tensor.f90:139-200 (layer stacking from space_to_sul upwards, ks/ko = n_lay..1)
  const int nl = r->nl;
  const mrm_geom& g = r->g;
  std::vector<PairGeom> out(nl * nl);
  const bool sul_p = g.sul_mu > 1.0, head_p = g.head_mu > 1.0;
  const double mus = sul_p ? std::max(0.0, (std::max(1.0, g.sul_mu) - 1.0) / (std::max(1.0, g.sul_mu) + 1.0)) : 0.0;
  const double mush = head_p ? std::max(0.0, (std::max(1.0, g.head_mu) - 1.0) / (std::max(1.0, g.head_mu) + 1.0)) : 0.0;
  std::vector<double> hdz(nl);
  hdz[0] = g.fly_height;
  for (int k = 1; k < nl; ++k) hdz[k] = hdz[k - 1] + g.dz[k - 1] + g.il_space[k];
  for (int k = 0; k < nl; ++k) hdz[k] += 0.5 * g.dz[k];
  double zsb = g.space_to_sul;
  for (int ks = nl - 1; ks >= 0; --ks) {
    const double zst = zsb + g.dz[ks];
    double zob = g.space_to_sul;
    for (int ko = nl - 1; ko >= 0; --ko) {
      const double zot = zob + g.dz[ko];
      PairGeom& p = out[ks * nl + ko];
      p.dz_s = g.dz[ks];
      p.dz_o = g.dz[ko];
      p.rz = 0.5 * (zst - zot + zsb - zob);
      p.rz_sul = 0.5 * (-zst - zot - zsb - zob);
      p.f_sul = sul_p ? mus : 0.0;
      p.rz_head = hdz[ks] + hdz[ko];
      p.f_head = head_p ? mush : 0.0;
      p.norm = 1.0 / (g.dx * g.dy * g.dz[ko] * (double)r->px * (double)r->py);
      zob = zot + g.il_space[ko];
    }
    zsb = zst + g.il_space[ks];
  }
  return out;
}

// real-space FP64 tensor on the device (reference layout)
int tensor_real(mrm_gpu* r, double* d_n2d) {
  std::string* errp = &r->err;
  const int npair = r->nl * r->nl;
  std::vector<PairGeom> pg = pair_geoms(r);
  void* d_pg = nullptr;
  int rc = dmalloc(errp, &d_pg, sizeof(PairGeom) * npair);
  if (rc) return rc;
  CK(cudaMemcpy(d_pg, pg.data(), sizeof(PairGeom) * npair, cudaMemcpyHostToDevice));
  const int nimg = r->g.boundary == MRM_OPEN ? 0 : std::max(0, r->g.num_images);
  const long long total = (long long)npair * r->px * r->py;
  tensor_real_kernel<<<(unsigned)((total + 127) / 128), 128, 0, r->eng->st>>>(
      d_n2d, static_cast<const PairGeom*>(d_pg), npair, r->px, r->py, r->g.dx, r->g.dy, nimg);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(r->eng->st));
  dfree(d_pg);
  return MRM_OK;
}

// FP64 FFT of the real tensor and packing into the run's spectral store
int tensor_spectrum(mrm_gpu* r, const double* d_n2d) {
  std::string* errp = &r->err;
  Engine* e = r->eng;
  const int npair = r->nl * r->nl, ph = r->px / 2 + 1, pyh = r->py / 2 + 1;
  const int planes = npair * 9;
  void* d_spec = nullptr;
  int rc = dmalloc(errp, &d_spec, sizeof(double) * 2 * (size_t)planes * r->py * ph);
  if (rc) return rc;
  // FP64 twiddles (the engine's table may be FP32)
  void* d_tw64 = nullptr;
  std::vector<double> tw(2 * kTwN);
  for (int k = 0; k < kTwN; ++k) {
    double a = -2.0 * M_PI * (double)k / (double)kTwN;
    tw[2 * k] = std::cos(a);
    tw[2 * k + 1] = std::sin(a);
  }
  rc = dmalloc(errp, &d_tw64, sizeof(double) * 2 * kTwN);
  if (rc) return rc;
  CK(cudaMemcpy(d_tw64, tw.data(), sizeof(double) * 2 * kTwN, cudaMemcpyHostToDevice));
  const Cx<double>* tw64 = static_cast<const Cx<double>*>(d_tw64);
  const int M = r->px / 2;
  // two shared buffers of one padded-stride sequence each (fft.cuh)
  size_t s1 = 2 * (size_t)fft_stride(M) * sizeof(Cx<double>), s2 = 2 * (size_t)fft_stride(r->py) * sizeof(Cx<double>);
  if (raise_smem(r2c_rows_f64, s1, errp) || raise_smem(c2c_cols_f64, s2, errp)) return MRM_ERR_CUDA;
  r2c_rows_f64<<<planes * r->py, 256, s1, e->st>>>(d_n2d, static_cast<Cx<double>*>(d_spec), r->lgpx, r->py, tw64);
  CK(cudaGetLastError());
  c2c_cols_f64<<<planes * ph, 256, s2, e->st>>>(static_cast<Cx<double>*>(d_spec), r->lgpy, ph, tw64);
  CK(cudaGetLastError());
  unsigned long long* d_mx = nullptr;
  rc = dmalloc(errp, (void**)&d_mx, 2 * sizeof(unsigned long long));
  if (rc) return rc;
  if (e->prec == MRM_FP64) {
    const long long total = (long long)ph * npair * 9 * r->py;
    pack_tensor_full_kernel<<<(unsigned)((total + 255) / 256), 256, 0, e->st>>>(
        static_cast<const Cx<double>*>(d_spec), static_cast<Cx<double>*>(r->tens), npair, r->py, ph, d_mx, d_mx + 1);
  } else {
    const long long total = (long long)ph * npair * 9 * pyh;
    pack_tensor_kernel<float><<<(unsigned)((total + 255) / 256), 256, 0, e->st>>>(
        static_cast<const Cx<double>*>(d_spec), static_cast<float*>(r->tens), npair, r->py, ph, d_mx, d_mx + 1);
  }
  CK(cudaGetLastError());
  unsigned long long hm[2];
  CK(cudaMemcpyAsync(hm, d_mx, sizeof(hm), cudaMemcpyDeviceToHost, e->st));
  CK(cudaStreamSynchronize(e->st));
  double dres, dkept;
  std::memcpy(&dres, &hm[0], 8);
  std::memcpy(&dkept, &hm[1], 8);
  r->tensor_resid = dres;
  r->tensor_kept = dkept;
  dfree(d_mx);
  dfree(d_spec);
  dfree(d_tw64);
  r->tensor_ready = true;
  r->spec_valid = false;
  e->tables_dirty = true;
  e->desc_dirty = true;
  return MRM_OK;
}

thread_local std::string g_create_err;

}  // namespace

// =====================================================================
// C ABI
// =====================================================================
extern "C" {

int mrm_gpu_create(const mrm_geom* geom, int device, mrm_gpu** out) {
  if (!out) return MRM_ERR_ARG;
  *out = nullptr;
  int rc = validate_geom(geom, &g_create_err);
  if (rc) return rc;
  Engine* e = new Engine();
  rc = engine_init(e, geom->precision, device);
  if (rc) {
    g_create_err = e->err;
    engine_free(e);
    delete e;
    return rc;
  }
  mrm_gpu* r = new_run(e, geom, &g_create_err, &rc);
  if (!r) {
    engine_free(e);
    delete e;
    return rc;
  }
  r->own_engine = true;
  *out = r;
  return MRM_OK;
}

int mrm_gpu_destroy(mrm_gpu* h) {
  if (!h) return MRM_OK;
  Engine* e = h->eng;
  cudaSetDevice(e->dev);
  cudaStreamSynchronize(e->st);
  e->runs.erase(std::remove(e->runs.begin(), e->runs.end(), h), e->runs.end());
  e->tables_dirty = true;
  e->desc_dirty = true;
  host_cache().erase(h);
  run_free(h);
  const bool own = h->own_engine;
  delete h;
  if (own) {
    engine_free(e);
    delete e;
  }
  return MRM_OK;
}

const char* mrm_gpu_last_error(const mrm_gpu* h) {
  if (!h) return g_create_err.c_str();
  if (!h->err.empty()) return h->err.c_str();
  return h->eng ? h->eng->err.c_str() : "";
}

int mrm_gpu_upload_layer(mrm_gpu* h, int layer, int n_grains, const double* ms, const double* grain_vol,
                         const double* uni_axis, const double* hk, const double* hk_scale,
                         const double* ms_scale, const double* alpha_scale, double alpha, double gamma,
                         double floor_ms, const int32_t* grain2gridindex, const int32_t* grain2grid,
                         const int32_t* hxgrainindex, const int32_t* hxgrain, const double* hx) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  cudaSetDevice(h->eng->dev);
  cudaStreamSynchronize(h->eng->st);
  if (h->g.precision == MRM_FP64)
    return upload_layer_t<double>(h, layer, n_grains, ms, grain_vol, uni_axis, hk, hk_scale, ms_scale,
                                  alpha_scale, alpha, gamma, floor_ms, grain2gridindex, grain2grid,
                                  hxgrainindex, hxgrain, hx);
  return upload_layer_t<float>(h, layer, n_grains, ms, grain_vol, uni_axis, hk, hk_scale, ms_scale,
                               alpha_scale, alpha, gamma, floor_ms, grain2gridindex, grain2grid,
                               hxgrainindex, hxgrain, hx);
}

int mrm_gpu_upload_interlayer(mrm_gpu* h, int layer, int side, const int32_t* index, const int32_t* grain,
                              const double* coef) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  const int other = side == 0 ? layer - 1 : layer + 1;
  if (side < 0 || side > 1 || other < 0 || other >= h->nl)
    return set_err(&h->err, MRM_ERR_ARG, "no layer on side %d of layer %d", side, layer);
  auto& hc = host_cache()[h];
  if ((int)hc.size() <= other || hc[other].ms_scale.empty())
    return set_err(&h->err, MRM_ERR_STATE, "upload layer %d before its interlayer coupling", other);
  if (!index || !grain || !coef) return set_err(&h->err, MRM_ERR_ARG, "NULL interlayer array");
  std::string* errp = &h->err;
  cudaSetDevice(h->eng->dev);
  cudaStreamSynchronize(h->eng->st);
  LayerBufs& b = h->L[layer];
  const int n = b.n;
  int rc;
  if (h->g.precision == MRM_FP64)
    rc = side == 0 ? upload_csr<double>(h, n, index, grain, coef, hc[other].ms_scale.data(), h->L[other].n, &b.uidx, &b.unbr, &b.ucoef)
                   : upload_csr<double>(h, n, index, grain, coef, hc[other].ms_scale.data(), h->L[other].n, &b.lidx, &b.lnbr, &b.lcoef);
  else
    rc = side == 0 ? upload_csr<float>(h, n, index, grain, coef, hc[other].ms_scale.data(), h->L[other].n, &b.uidx, &b.unbr, &b.ucoef)
                   : upload_csr<float>(h, n, index, grain, coef, hc[other].ms_scale.data(), h->L[other].n, &b.lidx, &b.lnbr, &b.lcoef);
  if (rc) return rc;
  // columnar form: grain n couples to grain n of the other layer only
  void** col = side == 0 ? &b.ucol : &b.lcol;
  dfree(*col);
  bool columnar = h->L[other].n == n;
  for (int g = 0; columnar && g < n; ++g)
    columnar = (index[g + 1] - index[g] == 1) && (grain[index[g]] == g + 1);
  if (columnar) {
    const size_t re = relem(h->g.precision);
    std::vector<double> cf(n);
    for (int g = 0; g < n; ++g) cf[g] = coef[index[g]] * hc[other].ms_scale[g];
    rc = dmalloc(errp, col, re * n);
    if (rc) return rc;
    if (h->g.precision == MRM_FP64) {
      CK(cudaMemcpy(*col, cf.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> f(cf.begin(), cf.end());
      CK(cudaMemcpy(*col, f.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    }
  }
  h->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_gpu_build_tensor(mrm_gpu* h) {
  if (!h) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  CK(cudaSetDevice(h->eng->dev));
  void* d_n2d = nullptr;
  const size_t bytes = sizeof(double) * 9 * (size_t)h->nl * h->nl * h->px * h->py;
  int rc = dmalloc(errp, &d_n2d, bytes);
  if (rc) return rc;
  rc = tensor_real(h, static_cast<double*>(d_n2d));
  if (!rc) rc = tensor_spectrum(h, static_cast<const double*>(d_n2d));
  dfree(d_n2d);
  return rc;
}

int mrm_gpu_upload_tensor(mrm_gpu* h, const double* n2d, int nx_fft, int ny_fft) {
  if (!h || !n2d) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  if (nx_fft != h->px || ny_fft != h->py)
    return set_err(errp, MRM_ERR_ARG, "tensor grid %dx%d differs from the FFT grid %dx%d", nx_fft, ny_fft, h->px, h->py);
  CK(cudaSetDevice(h->eng->dev));
  void* d_n2d = nullptr;
  const size_t bytes = sizeof(double) * 9 * (size_t)h->nl * h->nl * h->px * h->py;
  int rc = dmalloc(errp, &d_n2d, bytes);
  if (rc) return rc;
  CK(cudaMemcpy(d_n2d, n2d, bytes, cudaMemcpyHostToDevice));
  rc = tensor_spectrum(h, static_cast<const double*>(d_n2d));
  dfree(d_n2d);
  return rc;
}

int mrm_gpu_download_tensor(mrm_gpu* h, double* n2d) {
  if (!h || !n2d) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  CK(cudaSetDevice(h->eng->dev));
  void* d_n2d = nullptr;
  const size_t bytes = sizeof(double) * 9 * (size_t)h->nl * h->nl * h->px * h->py;
  int rc = dmalloc(errp, &d_n2d, bytes);
  if (rc) return rc;
  rc = tensor_real(h, static_cast<double*>(d_n2d));
  if (!rc) {
    cudaError_t ce = cudaMemcpy(n2d, d_n2d, bytes, cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) rc = set_err(errp, MRM_ERR_CUDA, "download tensor: %s", cudaGetErrorString(ce));
  }
  dfree(d_n2d);
  return rc;
}

int mrm_gpu_copy_tensor(mrm_gpu* dst, const mrm_gpu* src) {
  if (!dst || !src) return MRM_ERR_ARG;
  std::string* errp = &dst->err;
  if (!src->tensor_ready) return set_err(errp, MRM_ERR_STATE, "source run has no tensor");
  if (dst->px != src->px || dst->py != src->py || dst->nl != src->nl ||
      dst->g.precision != src->g.precision || dst->eng->dev != src->eng->dev)
    return set_err(errp, MRM_ERR_ARG, "tensor geometry differs");
  for (int l = 0; l < dst->nl; ++l)
    if (dst->g.dz[l] != src->g.dz[l] || dst->g.il_space[l] != src->g.il_space[l])
      return set_err(errp, MRM_ERR_ARG, "layer stack differs");
  if (dst->g.dx != src->g.dx || dst->g.dy != src->g.dy || dst->g.boundary != src->g.boundary ||
      dst->g.num_images != src->g.num_images)
    return set_err(errp, MRM_ERR_ARG, "cell size or boundary differs");
  CK(cudaSetDevice(dst->eng->dev));
  CK(cudaStreamSynchronize(src->eng->st));
  CK(cudaMemcpyAsync(dst->tens, src->tens, tensor_bytes(dst), cudaMemcpyDeviceToDevice, dst->eng->st));
  CK(cudaStreamSynchronize(dst->eng->st));
  dst->tensor_ready = true;
  dst->tensor_resid = src->tensor_resid;
  dst->tensor_kept = src->tensor_kept;
  dst->spec_valid = false;
  dst->eng->tables_dirty = true;
  dst->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_gpu_fft_grid(const mrm_gpu* h, int* nx_fft, int* ny_fft) {
  if (!h) return MRM_ERR_ARG;
  if (nx_fft) *nx_fft = h->px;
  if (ny_fft) *ny_fft = h->py;
  return MRM_OK;
}

int mrm_gpu_tensor_residual(const mrm_gpu* h, double* resid, double* kept) {
  if (!h) return MRM_ERR_ARG;
  if (resid) *resid = h->tensor_resid;
  if (kept) *kept = h->tensor_kept;
  return MRM_OK;
}

int mrm_gpu_set_demag(mrm_gpu* h, int on) {
  if (!h) return MRM_ERR_ARG;
  h->demag = on != 0;
  h->spec_valid = false;
  h->eng->tables_dirty = true;
  h->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_gpu_set_uniform_field(mrm_gpu* h, int layer, const double hdir[3], double t_start, double t_end,
                              double s_start, double s_end, double scale) {
  if (!h || !hdir) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  if (!(t_end != t_start)) return set_err(&h->err, MRM_ERR_ARG, "t_end must differ from t_start");
  LayerBufs& b = h->L[layer];
  for (int a = 0; a < 3; ++a) b.hdir[a] = hdir[a];
  b.t_start = t_start;
  b.t_end = t_end;
  b.s_start = s_start;
  b.s_end = s_end;
  b.scale = scale;
  b.func = 0;
  if (b.s_start == b.s_end) {  // applied.f90:309-312
    b.scale *= b.s_start;
    b.s_start = 1.0;
    b.s_end = 1.0;
  }
  h->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_gpu_set_field_function(mrm_gpu* h, int layer, const double hdir[3], int func, double amp,
                               double gamma, double phase, double param, double duty,
                               double moddepth, double dc, double scale) {
  if (!h || !hdir) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  if (func < 1 || func > 5) return set_err(&h->err, MRM_ERR_ARG, "unknown time function %d", func);
  if ((func == 4 || func == 5) && !(gamma > 0 && param > 0))
    return set_err(&h->err, MRM_ERR_ARG, "STE/NEW need a period and a time constant > 0");
  LayerBufs& b = h->L[layer];
  for (int a = 0; a < 3; ++a) b.hdir[a] = hdir[a];
  b.func = func;
  b.amp = amp;
  b.fgamma = gamma;
  b.phase = phase;
  b.param = param;
  b.duty = std::max(0.0, std::min(1.0, duty));          // applied.f90:276-277
  b.moddepth = std::max(0.0, std::min(1.0, moddepth));
  b.dc = dc;
  b.scale = scale;
  h->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_gpu_set_thermal(mrm_gpu* h, int layer, int on, double temperature, uint64_t seed) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  if (temperature < 0) return set_err(&h->err, MRM_ERR_ARG, "temperature must be >= 0");
  h->L[layer].thermal = on ? 1 : 0;
  h->L[layer].temperature = temperature;
  h->seed = seed;
  h->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_gpu_set_state(mrm_gpu* h, int layer, const double* m) {
  if (!h || !m) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  if (layer < 0 || layer >= h->nl) return set_err(errp, MRM_ERR_ARG, "layer %d out of range", layer);
  if (!h->L[layer].uploaded) return set_err(errp, MRM_ERR_STATE, "upload layer %d first", layer);
  const int n = h->L[layer].n;
  CK(cudaSetDevice(h->eng->dev));
  CK(cudaStreamSynchronize(h->eng->st));
  if (h->g.precision == MRM_FP64) {
    std::vector<double> v(4 * n);
    for (int g = 0; g < n; ++g) {
      v[4 * g] = m[3 * g]; v[4 * g + 1] = m[3 * g + 1]; v[4 * g + 2] = m[3 * g + 2]; v[4 * g + 3] = 0;
    }
    CK(cudaMemcpy(h->L[layer].m, v.data(), sizeof(double) * 4 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->L[layer].mp, v.data(), sizeof(double) * 4 * n, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> v(4 * n);
    for (int g = 0; g < n; ++g) {
      v[4 * g] = (float)m[3 * g]; v[4 * g + 1] = (float)m[3 * g + 1]; v[4 * g + 2] = (float)m[3 * g + 2]; v[4 * g + 3] = 0;
    }
    CK(cudaMemcpy(h->L[layer].m, v.data(), sizeof(float) * 4 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->L[layer].mp, v.data(), sizeof(float) * 4 * n, cudaMemcpyHostToDevice));
  }
  h->spec_valid = false;
  return MRM_OK;
}

static int get_v4(mrm_gpu* h, int layer, void* src, double* out) {
  std::string* errp = &h->err;
  if (layer < 0 || layer >= h->nl) return set_err(errp, MRM_ERR_ARG, "layer %d out of range", layer);
  const int n = h->L[layer].n;
  CK(cudaSetDevice(h->eng->dev));
  CK(cudaStreamSynchronize(h->eng->st));
  if (h->g.precision == MRM_FP64) {
    std::vector<double> v(4 * n);
    CK(cudaMemcpy(v.data(), src, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost));
    for (int g = 0; g < n; ++g) { out[3 * g] = v[4 * g]; out[3 * g + 1] = v[4 * g + 1]; out[3 * g + 2] = v[4 * g + 2]; }
  } else {
    std::vector<float> v(4 * n);
    CK(cudaMemcpy(v.data(), src, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost));
    for (int g = 0; g < n; ++g) { out[3 * g] = v[4 * g]; out[3 * g + 1] = v[4 * g + 1]; out[3 * g + 2] = v[4 * g + 2]; }
  }
  return MRM_OK;
}

int mrm_gpu_get_state(mrm_gpu* h, int layer, double* m) {
  if (!h || !m) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  return get_v4(h, layer, h->L[layer].m, m);
}

int mrm_gpu_get_field(mrm_gpu* h, int layer, double* hfield) {
  if (!h || !hfield) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  return get_v4(h, layer, h->L[layer].hf, hfield);
}

int mrm_gpu_set_time(mrm_gpu* h, double t, int64_t step) {
  if (!h) return MRM_ERR_ARG;
  h->t_base = t;
  h->step_base = step;
  h->step = step;
  h->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_gpu_get_time(const mrm_gpu* h, double* t, int64_t* step) {
  if (!h) return MRM_ERR_ARG;
  if (t) *t = h->t_base + (double)(h->step - h->step_base) * h->dt;
  if (step) *step = h->step;
  return MRM_OK;
}

int mrm_gpu_eval_field(mrm_gpu* h, double t, int layer, double* hdemag) {
  if (!h) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  if (layer < 0 || layer >= h->nl) return set_err(errp, MRM_ERR_ARG, "layer %d out of range", layer);
  for (int l = 0; l < h->nl; ++l)
    if (!h->L[l].uploaded) return set_err(errp, MRM_ERR_STATE, "upload layer %d first", l);
  if (h->demag && !h->tensor_ready) return set_err(errp, MRM_ERR_STATE, "build or upload the tensor first (or disable demag)");
  Engine* e = h->eng;
  // evaluate this run alone at time t: move its time origin and park the others
  const double tb = h->t_base;
  const long long sb = h->step_base;
  h->t_base = t;
  h->step_base = h->step;
  std::vector<bool> act;
  for (auto* r : e->runs) {
    act.push_back(r->active);
    r->active = (r == h);
  }
  e->desc_dirty = true;
  int rc = e->prec == MRM_FP64 ? engine_eval<double>(e) : engine_eval<float>(e);
  for (size_t i = 0; i < e->runs.size(); ++i) e->runs[i]->active = act[i];
  h->t_base = tb;
  h->step_base = sb;
  e->desc_dirty = true;
  if (rc) {
    h->err = e->err;
    return rc;
  }
  if (hdemag) return get_v4(h, layer, h->L[layer].hd, hdemag);
  CK(cudaStreamSynchronize(e->st));
  return MRM_OK;
}

static int plain_prepare(mrm_gpu* h, int nsteps, double dt, int llg_type) {
  std::string* errp = &h->err;
  if (nsteps < 0) return set_err(errp, MRM_ERR_ARG, "nsteps must be >= 0");
  if (!(dt > 0)) return set_err(errp, MRM_ERR_ARG, "dt must be > 0");
  if (llg_type != -3) return set_err(errp, MRM_ERR_UNSUPPORTED, "llg_type %d: only Heun (-3) is on this path", llg_type);
  for (int l = 0; l < h->nl; ++l)
    if (!h->L[l].uploaded) return set_err(errp, MRM_ERR_STATE, "upload layer %d first", l);
  if (h->demag && !h->tensor_ready) return set_err(errp, MRM_ERR_STATE, "build or upload the tensor first (or disable demag)");
  Engine* e = h->eng;
  CK(cudaSetDevice(e->dev));
  if (dt != h->dt) {
    // keep t continuous across a change of dt
    h->t_base = h->t_base + (double)(h->step - h->step_base) * h->dt;
    h->step_base = h->step;
    h->dt = dt;
    e->desc_dirty = true;
  }
  if (h->step_end <= h->step + nsteps) {
    h->step_end = (long long)9e18;
    e->desc_dirty = true;
  }
  return MRM_OK;
}

int mrm_gpu_enqueue_steps(mrm_gpu* h, int nsteps, double dt, int llg_type) {
  if (!h) return MRM_ERR_ARG;
  int rc = plain_prepare(h, nsteps, dt, llg_type);
  if (rc) return rc;
  if (nsteps > 0) {
    rc = engine_step(h->eng, nsteps);
    if (rc) {
      h->err = h->eng->err;
      return rc;
    }
    h->has_stats = true;
  }
  return MRM_OK;
}

int mrm_gpu_read_stats(mrm_gpu* h, mrm_gpu_stats* out) {
  if (!h || !out) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  if (!h->has_stats) return set_err(errp, MRM_ERR_STATE, "no step has been taken");
  Engine* e = h->eng;
  CK(cudaSetDevice(e->dev));
  CK(cudaMemcpyAsync(e->h_stats + h->slot, e->d_stats + h->slot, sizeof(StatsDev), cudaMemcpyDeviceToHost, e->st));
  CK(cudaStreamSynchronize(e->st));
  static_assert(sizeof(StatsDev) == sizeof(mrm_gpu_stats), "stats layout");
  std::memcpy(out, e->h_stats + h->slot, sizeof(StatsDev));
  return MRM_OK;
}

int mrm_gpu_step(mrm_gpu* h, int nsteps, double dt, int llg_type, mrm_gpu_stats* out) {
  if (!h) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  int rc = mrm_gpu_enqueue_steps(h, nsteps, dt, llg_type);
  if (rc) return rc;
  if (out) {
    if (nsteps == 0) return set_err(errp, MRM_ERR_ARG, "stats need nsteps >= 1");
    return mrm_gpu_read_stats(h, out);
  }
  CK(cudaStreamSynchronize(h->eng->st));
  return MRM_OK;
}

int mrm_gpu_stream(const mrm_gpu* h, void** stream) {
  if (!h || !stream) return MRM_ERR_ARG;
  *stream = (void*)h->eng->st;
  return MRM_OK;
}

}  // extern "C"

template <typename R>
static int profile_t(Engine* e, int reps, double* ms_out) {
  std::string* errp = &e->err;
  int rc = ensure_ready<R>(e);
  if (rc) return rc;
  std::vector<cudaEvent_t> ev(5 * reps);
  for (auto& x : ev) CK(cudaEventCreate(&x));
  const int nr = (int)e->runs.size();
  for (int s = 0; s < reps; ++s) {
    CK(cudaEventRecord(ev[5 * s + 0], e->st));
    launch_row<R>(e, kPred, 0, 0);
    CK(cudaEventRecord(ev[5 * s + 1], e->st));
    launch_col<R>(e, 0, 0);
    CK(cudaEventRecord(ev[5 * s + 2], e->st));
    launch_row<R>(e, kCorr, 0, 0);
    CK(cudaEventRecord(ev[5 * s + 3], e->st));
    launch_col<R>(e, 0, 0);
    CK(cudaEventRecord(ev[5 * s + 4], e->st));
    advance_kernel<R><<<(nr + 127) / 128, 128, 0, e->st>>>(static_cast<RunDev<R>*>(e->d_runs), nr, 1);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(e->st));
  double acc[4] = {0, 0, 0, 0};
  for (int s = 0; s < reps; ++s)
    for (int k = 0; k < 4; ++k) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, ev[5 * s + k], ev[5 * s + k + 1]));
      acc[k] += ms;
    }
  for (auto& x : ev) cudaEventDestroy(x);
  for (int k = 0; k < 4; ++k) ms_out[k] = acc[k] / reps;
  for (auto* r : e->runs)
    if (r->active) r->step += std::min<long long>(std::max(0LL, r->step_end - r->step), reps);
  return MRM_OK;
}

extern "C" {

int mrm_gpu_profile(mrm_gpu* h, int reps, double dt, double* ms_out) {
  if (!h || !ms_out || reps < 1) return MRM_ERR_ARG;
  int rc = plain_prepare(h, reps, dt, -3);
  if (rc) return rc;
  rc = h->eng->prec == MRM_FP64 ? profile_t<double>(h->eng, reps, ms_out) : profile_t<float>(h->eng, reps, ms_out);
  if (rc) h->err = h->eng->err;
  return rc;
}

// ---------------- batch ----------------
struct mrm_batch {
  Engine eng;
};

int mrm_batch_create(int precision, int device, mrm_batch** out) {
  if (!out) return MRM_ERR_ARG;
  *out = nullptr;
  if (precision != MRM_FP32 && precision != MRM_FP64) return set_err(&g_create_err, MRM_ERR_ARG, "bad precision");
  mrm_batch* b = new mrm_batch();
  int rc = engine_init(&b->eng, precision, device);
  if (rc) {
    g_create_err = b->eng.err;
    engine_free(&b->eng);
    delete b;
    return rc;
  }
  *out = b;
  return MRM_OK;
}

int mrm_batch_destroy(mrm_batch* b) {
  if (!b) return MRM_OK;
  cudaSetDevice(b->eng.dev);
  cudaStreamSynchronize(b->eng.st);
  for (auto* r : b->eng.runs) {
    host_cache().erase(r);
    run_free(r);
    delete r;
  }
  b->eng.runs.clear();
  engine_free(&b->eng);
  delete b;
  return MRM_OK;
}

const char* mrm_batch_last_error(const mrm_batch* b) { return b ? b->eng.err.c_str() : g_create_err.c_str(); }

int mrm_batch_add(mrm_batch* b, const mrm_geom* geom, mrm_gpu** run) {
  if (!b || !run) return MRM_ERR_ARG;
  int rc = 0;
  cudaSetDevice(b->eng.dev);
  cudaStreamSynchronize(b->eng.st);
  mrm_gpu* r = new_run(&b->eng, geom, &b->eng.err, &rc);
  *run = r;
  return r ? MRM_OK : rc;
}

int mrm_batch_remove(mrm_batch* b, mrm_gpu* run) {
  if (!b || !run || run->eng != &b->eng) return MRM_ERR_ARG;
  cudaSetDevice(b->eng.dev);
  cudaStreamSynchronize(b->eng.st);
  auto& v = b->eng.runs;
  v.erase(std::remove(v.begin(), v.end(), run), v.end());
  host_cache().erase(run);
  run_free(run);
  delete run;
  b->eng.tables_dirty = true;
  b->eng.desc_dirty = true;
  return MRM_OK;
}

int mrm_batch_set_run(mrm_gpu* run, double dt, int64_t step_end, int active) {
  if (!run) return MRM_ERR_ARG;
  if (!(dt > 0)) return set_err(&run->err, MRM_ERR_ARG, "dt must be > 0");
  if (dt != run->dt) {
    run->t_base = run->t_base + (double)(run->step - run->step_base) * run->dt;
    run->step_base = run->step;
    run->dt = dt;
  }
  run->step_end = step_end;
  run->active = active != 0;
  run->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_batch_enqueue(mrm_batch* b, int nsteps, int llg_type) {
  if (!b) return MRM_ERR_ARG;
  Engine* e = &b->eng;
  std::string* errp = &e->err;
  if (llg_type != -3) return set_err(errp, MRM_ERR_UNSUPPORTED, "llg_type %d: only Heun (-3)", llg_type);
  for (auto* r : e->runs) {
    if (!r->active) continue;
    for (int l = 0; l < r->nl; ++l)
      if (!r->L[l].uploaded) return set_err(errp, MRM_ERR_STATE, "a run has layer %d not uploaded", l);
    if (r->demag && !r->tensor_ready) return set_err(errp, MRM_ERR_STATE, "a run has no tensor");
  }
  if (nsteps <= 0) return MRM_OK;
  return engine_step(e, nsteps);
}

int mrm_batch_step(mrm_batch* b, int nsteps, int llg_type) {
  int rc = mrm_batch_enqueue(b, nsteps, llg_type);
  if (rc) return rc;
  std::string* errp = &b->eng.err;
  CK(cudaStreamSynchronize(b->eng.st));
  return MRM_OK;
}

int mrm_batch_profile(mrm_batch* b, int reps, double* ms_out) {
  if (!b || !ms_out || reps < 1) return MRM_ERR_ARG;
  Engine* e = &b->eng;
  return e->prec == MRM_FP64 ? profile_t<double>(e, reps, ms_out) : profile_t<float>(e, reps, ms_out);
}

int mrm_batch_stream(const mrm_batch* b, void** stream) {
  if (!b || !stream) return MRM_ERR_ARG;
  *stream = (void*)b->eng.st;
  return MRM_OK;
}

int mrm_batch_stats(mrm_batch* b, int nruns, mrm_gpu* const* runs, mrm_gpu_stats* out) {
  if (!b || (nruns > 0 && (!runs || !out))) return MRM_ERR_ARG;
  Engine* e = &b->eng;
  std::string* errp = &e->err;
  const int nr = (int)e->runs.size();
  if (!nr) return MRM_OK;
  CK(cudaSetDevice(e->dev));
  CK(cudaMemcpyAsync(e->h_stats, e->d_stats, sizeof(StatsDev) * nr, cudaMemcpyDeviceToHost, e->st));
  CK(cudaStreamSynchronize(e->st));
  for (int i = 0; i < nruns; ++i) {
    if (!runs[i] || runs[i]->eng != e || runs[i]->slot < 0 || runs[i]->slot >= nr)
      return set_err(errp, MRM_ERR_ARG, "run %d is not in this batch", i);
    std::memcpy(&out[i], e->h_stats + runs[i]->slot, sizeof(StatsDev));
  }
  return MRM_OK;
}

}  // extern "C"

template <typename R>
static int occ_t(Engine* e, int* out2) {
  std::string* errp = &e->err;
  int a = 0, b = 0;
  if (e->rowcfg == 0 && !e->pref && sizeof(R) == sizeof(float))
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, row_kernel<R, kPred, false, 1, 256, false>, 256, e->smem_row));
  else if (e->rowcfg == 0)
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, row_kernel<R, kPred, false, 1, 256, true>, 256, e->smem_row));
  else if (e->rowcfg == 1)
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, row_kernel<R, kPred, false, 2, 256, true>, 256, e->smem_row));
  else
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, row_kernel<R, kPred, false, 2, 512, true>, 512, e->smem_row));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, col_kernel<R, sizeof(R) == 4, kBlock>, kBlock, e->smem_col));
  out2[0] = a;
  out2[1] = b;
  return MRM_OK;
}

extern "C" {

int mrm_batch_occupancy(mrm_batch* b, int* out2) {
  if (!b || !out2) return MRM_ERR_ARG;
  Engine* e = &b->eng;
  cudaSetDevice(e->dev);
  return e->prec == MRM_FP64 ? occ_t<double>(e, out2) : occ_t<float>(e, out2);
}

int64_t mrm_run_footprint(const mrm_geom* geom) {
  if (!geom) return -1;
  return footprint(*geom);
}

int mrm_device_memory(int device, int64_t* free_bytes, int64_t* total_bytes) {
  if (cudaSetDevice(device) != cudaSuccess) return MRM_ERR_CUDA;
  size_t f = 0, t = 0;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess) return MRM_ERR_CUDA;
  if (free_bytes) *free_bytes = (int64_t)f;
  if (total_bytes) *total_bytes = (int64_t)t;
  return MRM_OK;
}

}  // extern "C"

// ---------------- allocation-free demag evaluation ----------------
//
// mrm_gpu_demag_noalloc evaluates the demagnetising field of a caller's device
// magnetisation with the handle's tensor, using the same four kernels as
// mrm_gpu_eval_field (Ms*m -> forward row FFT, column FFT x tensor x inverse,
// inverse row FFT), but with every buffer of its own -- run descriptor, task
// tables, packed magnetisation, fields and both half spectra -- carved out of
// one file-scope device array instead of the handle's allocations.  The call
// itself allocates nothing (no cudaMalloc/cudaFree, no pinned host memory, no
// graph): callers running under a stream-ordered pool or a framework's
// caching allocator, or a Fortran host that must not grow device memory inside
// its time loop, can evaluate fields of trial states without an allocation.
namespace {

constexpr size_t kNoAllocBytes = 16u << 20;  // 16 MiB of scratch per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDev = 64;
struct NoAllocDev {
  unsigned char* base = nullptr;
  bool ready = false;
};
NoAllocDev g_noalloc_dev[kNoAllocMaxDev];
std::mutex g_noalloc_mu;

static_assert(sizeof(RunDev<float>) <= 4000, "run descriptor must fit in a kernel parameter block");

struct NoAllocLayout {
  size_t desc = 0, rtask = 0, ctask = 0, m = 0, hd = 0, hf = 0, specx = 0, spech = 0, total = 0;
};

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

NoAllocLayout noalloc_layout(const mrm_gpu* r, int nrt, int nct) {
  NoAllocLayout o;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += align256(bytes);
    return at;
  };
  const size_t n = (size_t)r->g.nx * r->g.ny, ph = r->px / 2 + 1;
  const size_t grains = (size_t)r->nl * n * sizeof(V4<float>);
  const size_t spec = (size_t)r->nl * 3 * r->g.ny * ph * sizeof(Cx<float>);
  o.desc = take(sizeof(RunDev<float>));
  o.rtask = take(sizeof(Task) * nrt);
  o.ctask = take(sizeof(Task) * nct);
  o.m = take(grains);
  o.hd = take(grains);
  o.hf = take(grains);
  o.specx = take(spec);
  o.spech = take(spec);
  o.total = off;
  return o;
}

// Writes the run descriptor and both task tables, and packs m (n_lay x n x 3
// floats) into the float4 layout of the row kernel.
__global__ void noalloc_pack_kernel(RunDev<float> d, RunDev<float>* __restrict__ desc,
                                    Task* __restrict__ rt, int nrt, int rpt, Task* __restrict__ ct,
                                    int nct, int cpt, const float* __restrict__ m_in,
                                    V4<float>* __restrict__ m_out, long long ntot) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *desc = d;
  if (i < nrt) {
    const int per = (d.ny + rpt - 1) / rpt;
    const int l = (int)i / per, j = ((int)i - l * per) * rpt;
    rt[i] = make_int4(0, l, j, min(rpt, d.ny - j));
  }
  if (i < nct) {
    const int k = (int)i * cpt, ph = d.px / 2 + 1;
    ct[i] = make_int4(0, k, min(cpt, ph - k), 0);
  }
  if (i < ntot) m_out[i] = V4<float>{m_in[3 * i], m_in[3 * i + 1], m_in[3 * i + 2], 0.f};
}

__global__ void noalloc_unpack_kernel(const V4<float>* __restrict__ hd, float* __restrict__ out,
                                      long long ntot) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntot) return;
  const V4<float> v = hd[i];
  out[3 * i] = v.x;
  out[3 * i + 1] = v.y;
  out[3 * i + 2] = v.z;
}

// Loads a kernel (CUDA lazy loading would otherwise load it, and allocate its
// code, at its first launch) and lets it use all opt-in shared memory.  The
// raise_smem record is lifted to the same value so that no engine lowers it.
template <typename K>
int noalloc_prepare(K* kern, int optin, std::string* errp) {
  cudaFuncAttributes fa;
  CK(cudaFuncGetAttributes(&fa, kern));
  const size_t dyn = (size_t)optin - fa.sharedSizeBytes;
  int rc = raise_smem(kern, dyn, errp);
  if (rc) return rc;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  return MRM_OK;
}

template <int GPT, int BLK>
int noalloc_prepare_rows(int optin, std::string* errp) {
  int rc = noalloc_prepare(row_kernel<float, kInit, false, GPT, BLK, true>, optin, errp);
  if (!rc) rc = noalloc_prepare(row_kernel<float, kEval, false, GPT, BLK, true>, optin, errp);
  return rc;
}

// Once per device, with that device current: the scratch address and the
// kernels' attributes.  Runs inside the first call on the device.
int noalloc_setup(int dev, std::string* errp, unsigned char** base) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocDev& s = g_noalloc_dev[dev];
  if (s.ready) {
    *base = s.base;
    return MRM_OK;
  }
  void* p = nullptr;
  CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  int optin = 0;
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  int rc = noalloc_prepare_rows<1, 256>(optin, errp);
  if (!rc) rc = noalloc_prepare_rows<2, 256>(optin, errp);
  if (!rc) rc = noalloc_prepare_rows<2, 512>(optin, errp);
  if (!rc) rc = noalloc_prepare(col_kernel<float, true, kBlock>, optin, errp);
  if (rc) return rc;
  cudaFuncAttributes fa;
  CK(cudaFuncGetAttributes(&fa, noalloc_pack_kernel));
  CK(cudaFuncGetAttributes(&fa, noalloc_unpack_kernel));
  s.base = static_cast<unsigned char*>(p);
  s.ready = true;
  *base = s.base;
  return MRM_OK;
}

// kInit follows the pack kernel with a plain launch: it reads the descriptor
// and tasks before its dependency wait, so it must not overlap their writer.
// kEval follows the column kernel with programmatic serialization, as in the
// engine.
template <int GPT, int BLK>
void noalloc_rows(int stage, int nrt, size_t smem, cudaStream_t st, const RunDev<float>* runs,
                  const Task* tasks, const Cx<float>* tw) {
  if (stage == kInit)
    row_kernel<float, kInit, false, GPT, BLK, true><<<nrt, BLK, smem, st>>>(runs, tasks, tw, 0, kFlagForce, nullptr);
  else
    launch_pdl(row_kernel<float, kEval, false, GPT, BLK, true>, dim3(nrt), dim3(BLK), smem, st, runs, tasks, tw, 0,
               kFlagForce | kFlagStoreField, (double*)nullptr);
}

void noalloc_rows_cfg(int cfg, int stage, int nrt, size_t smem, cudaStream_t st, const RunDev<float>* runs,
                      const Task* tasks, const Cx<float>* tw) {
  if (cfg == 0) noalloc_rows<1, 256>(stage, nrt, smem, st, runs, tasks, tw);
  else if (cfg == 1) noalloc_rows<2, 256>(stage, nrt, smem, st, runs, tasks, tw);
  else noalloc_rows<2, 512>(stage, nrt, smem, st, runs, tasks, tw);
}

}  // namespace

extern "C" {

int mrm_gpu_demag_noalloc(mrm_gpu* h, const float* m, float* hdemag, void* stream) {
  if (!h) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  if (!m || !hdemag) return set_err(errp, MRM_ERR_ARG, "m and hdemag must be device pointers");
  if (h->g.precision != MRM_FP32)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "the allocation-free demag evaluation takes MRM_FP32 handles");
  const int nl = h->nl, ny = h->g.ny, ph = h->px / 2 + 1;
  const int rpt = rows_per_task(h), nrt = nl * ((ny + rpt - 1) / rpt);
  const int cpt = cols_per_task(h), nct = (ph + cpt - 1) / cpt;
  const NoAllocLayout lay = noalloc_layout(h, nrt, nct);
  if (lay.total > kNoAllocBytes)
    return set_err(errp, MRM_ERR_UNSUPPORTED,
                   "%d x %d x %d grains (FFT grid %d x %d) need %zu bytes of scratch; the allocation-free "
                   "demag evaluation has %zu",
                   h->g.nx, ny, nl, h->px, h->py, lay.total, kNoAllocBytes);
  for (int l = 0; l < nl; ++l)
    if (!h->L[l].uploaded) return set_err(errp, MRM_ERR_STATE, "upload layer %d first", l);
  if (!h->tensor_ready) return set_err(errp, MRM_ERR_STATE, "build or upload the tensor first");
  Engine* e = h->eng;
  if (e->dev < 0 || e->dev >= kNoAllocMaxDev)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "device %d above the supported %d", e->dev, kNoAllocMaxDev);
  CK(cudaSetDevice(e->dev));
  unsigned char* base = nullptr;
  int rc = noalloc_setup(e->dev, errp, &base);
  if (rc) return rc;

  const long long n = (long long)h->g.nx * ny, ntot = n * nl;
  RunDev<float> d = make_desc<float>(h);
  d.active = 1;
  d.demag = 1;
  d.row_task0 = 0;
  d.nrow_tasks = nrt;
  d.specx = reinterpret_cast<Cx<float>*>(base + lay.specx);
  d.spech = reinterpret_cast<Cx<float>*>(base + lay.spech);
  V4<float>* sm = reinterpret_cast<V4<float>*>(base + lay.m);
  V4<float>* shd = reinterpret_cast<V4<float>*>(base + lay.hd);
  V4<float>* shf = reinterpret_cast<V4<float>*>(base + lay.hf);
  for (int l = 0; l < nl; ++l) {
    d.L[l].m = sm + l * n;
    d.L[l].hd = shd + l * n;
    d.L[l].hf = shf + l * n;
  }
  RunDev<float>* desc = reinterpret_cast<RunDev<float>*>(base + lay.desc);
  Task* rt = reinterpret_cast<Task*>(base + lay.rtask);
  Task* ct = reinterpret_cast<Task*>(base + lay.ctask);
  const Cx<float>* tw = static_cast<const Cx<float>*>(e->d_tw);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : e->st;
  const long long work = std::max<long long>(ntot, std::max(nrt, nct));
  const int cfg = row_config(rpt * h->g.nx);

  noalloc_pack_kernel<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(d, desc, rt, nrt, rpt, ct, nct, cpt, m, sm,
                                                                      ntot);
  noalloc_rows_cfg(cfg, kInit, nrt, row_smem(h, MRM_FP32), st, desc, rt, tw);
  launch_pdl(col_kernel<float, true, kBlock>, dim3(nct), dim3(kBlock), col_smem(h, MRM_FP32), st,
             (const RunDev<float>*)desc, (const Task*)ct, tw, 0, (int)kFlagForce);
  noalloc_rows_cfg(cfg, kEval, nrt, row_smem(h, MRM_FP32), st, desc, rt, tw);
  noalloc_unpack_kernel<<<(unsigned)((ntot + 255) / 256), 256, 0, st>>>(shd, hdemag, ntot);
  CK(cudaGetLastError());
  return MRM_OK;
}

}  // extern "C"
