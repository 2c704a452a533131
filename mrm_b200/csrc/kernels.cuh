// kernels.cuh -- fused per-step kernels of the grain-dynamics path (sm_100a).
//
// One Heun step (src/llg.f90:1195-1271, llg_type = -3) is four launches:
//   row<PRED>  : inverse row FFT of H^(m_n) -> H_demag, field assembly
//                (field.f90:197-225), Philox thermal field (field.f90:397-436),
//                Heun predictor (llg.f90:1122-1139, iter = 2), forward row FFT
//                of Ms*m* (data.f90:322-390 scatter + demag.f90:113-116)
//   col        : column FFT, tensor multiply (demag.f90:117-121), inverse
//                column FFT, all in shared memory
//   row<CORR>  : same with the corrector (iter = 1) at t+dt on m*, thermal
//                regenerated from the same counter; optional FP64 reductions
//                (llg.f90:217-237, push_llg errmx/errmx1/mmag)
//   col
// The spectrum buffer always holds H^(m) of the state it follows, so a step
// starts from it without a separate demag pass.
//
// Latency layout: every per-grain global load (state, parameters, lattice
// neighbours, columnar interlayer partner) is issued at the top of the row
// kernel, before the inverse FFT, so its latency overlaps the shared-memory
// passes; the column kernel batches its strided loads the same way.
#pragma once
#include "common.cuh"
#include "fft.cuh"
#include "philox.cuh"

namespace mrm {

enum Stage { kInit = 0, kPred = 1, kCorr = 2, kEval = 3 };
enum Flags { kFlagStats = 1, kFlagForce = 2, kFlagStoreField = 4 };

template <typename R>
MRM_D void cross3(R ax, R ay, R az, R bx, R by, R bz, R& cx, R& cy, R& cz) {
  cx = ay * bz - az * by;
  cy = az * bx - ax * bz;
  cz = ax * by - ay * bx;
}

// funct (applied.f90:328-377); Fortran mod(x,g) = x - int(x/g)*g = fmod
MRM_D double funct(int f, double t, double g, double phase, double param, double duty,
                   double moddepth) {
  if (f == 1) return sin(t * g + phase);
  if (f == 2) return cos(t * g + phase);
  if (f == 3) return exp(t * g + phase);
  if (f == 5) {  // NEW
    double x = g / param;
    const double y = exp(duty * x), w = exp(x);
    x = t + phase;
    if (x < 0.0) x = x + g * (1.0 + (double)(long long)fabs(x / g));
    x = fmod(x, g);
    if (x > duty * g) {
      x = exp((g - x) / param);
      return 1.0 - moddepth + x * (y - 1.0) * moddepth / (w - 1.0);
    }
    x = exp(-x / param);
    return 1.0 + x * (y - w) * moddepth / (w - 1.0);
  }
  if (f == 4) {  // STE: trapezoidal square wave of period g, rise time param
    double x = t + phase;
    if (x < 0.0) x = x + g * (1.0 + (double)(long long)fabs(x / g));
    x = fmod(x, g);
    if (x < 0.5 * param) return 2.0 * x / param;
    if (x < 0.5 * (g - param)) return 1.0;
    if (x < 0.5 * (g + param)) return (g - 2.0 * x) / param;
    if (x < g - 0.5 * param) return -1.0;
    return 2.0 * (x - g) / param;
  }
  return 0.0;
}

// time scale of a layer's uniform field (applied.f90:866-883; set_fld folds
// a constant ramp into `scale`, :309-312)
template <typename R>
MRM_D double ramp(const LayerDev<R>& L, double t) {
  if (L.func != 0)
    return (L.amp * funct(L.func, t, L.fgamma, L.phase, L.param, L.duty, L.moddepth) + L.dc) * L.scale;
  double u = (t - L.t_start) / (L.t_end - L.t_start);
  u = fmax(0.0, fmin(1.0, u));
  return ((L.s_end - L.s_start) * u + L.s_start) * L.scale;
}

// CSR neighbour sum  sum_j c_j m_j  (field.f90:350-363 / :326-348)
template <typename R>
MRM_D void csr_sum(const int* __restrict__ idx, const int* __restrict__ nbr,
                   const R* __restrict__ cf, const V4<R>* __restrict__ mb, int n, R& hx, R& hy,
                   R& hz) {
  const int q0 = __ldg(idx + n), q1 = __ldg(idx + n + 1);
  for (int q = q0; q < q1; ++q) {
    const int j = __ldg(nbr + q);
    const R c = __ldg(cf + q);
    const V4<R> mj = mb[j];
    hx += c * mj.x;
    hy += c * mj.y;
    hz += c * mj.z;
  }
}

// stats record slots (sums except the two maxima)
constexpr int kSlotV = 0, kSlotM = 1, kSlotM2 = 4, kSlotH = 7, kSlotWM = 10, kSlotW = 13,
              kSlotNup = 14, kSlotMaxTq = 15, kSlotMaxD2 = 16, kSlotMmag = 17, kSlotE = 18;
MRM_HD constexpr bool slot_is_max(int s) { return s == kSlotMaxTq || s == kSlotMaxD2; }

MRM_D void block_reduce_record(double* rec, double* sred /* [32][kNPart] */, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int s = 0; s < kNPart; ++s) {
    double v = rec[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double w = __shfl_xor_sync(0xffffffffu, v, o);
      v = slot_is_max(s) ? fmax(v, w) : v + w;
    }
    if (lane == 0) sred[warp * kNPart + s] = v;
  }
  __syncthreads();
  if (threadIdx.x < kNPart) {
    const int s = threadIdx.x;
    double v = sred[s];
    for (int w = 1; w < nw; ++w) v = slot_is_max(s) ? fmax(v, sred[w * kNPart + s]) : v + sred[w * kNPart + s];
    out[s] = v;
  }
}

// Per-grain inputs gathered at the top of the row kernel.
template <typename R>
struct GrainIn {
  V4<R> mf;      // state the field is evaluated on (m_n, or m* in the corrector)
  V4<R> pa, pb;  // parameters
  V4<R> cst;     // lattice exchange coefficients (j-1, i-1, i+1, j+1)
  V4<R> nb[4];   // lattice neighbours
  V4<R> dm, m0;  // corrector: predictor increment and m_n
  V4<R> vu, vl;  // columnar interlayer partners
  V4<R> ht;      // thermal field / sqrt(dt)
  R cu, cl;
};

template <int STAGE, bool STATS>
__host__ __device__ constexpr int stats_slots() { return (STAGE == kCorr && STATS) ? 32 * kNPart : 1; }

template <typename R>
__host__ __device__ constexpr int min_blocks() { return sizeof(R) == sizeof(float) ? 2 : 1; }
// PREF: gather every per-grain input into registers before the inverse FFT
// (latency-bound runs with few blocks per SM); otherwise load at use and run
// four 256-thread blocks per SM (throughput-bound batches).
template <typename R, bool PREF>
__host__ __device__ constexpr int row_min_blocks() {
  return PREF ? min_blocks<R>() : (sizeof(R) == sizeof(float) ? 4 : 2);
}

template <typename R, int STAGE, bool STATS, int GPT, int BLOCK, bool PREF>
__global__ void __launch_bounds__(BLOCK, row_min_blocks<R, PREF>()) row_kernel(const RunDev<R>* __restrict__ runs,
                                                    const Task* __restrict__ tasks,
                                                    const Cx<R>* __restrict__ tw, int istep,
                                                    int flags, double* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_launch_dependents();
  const Task tk = tasks[blockIdx.x];
  const RunDev<R>& rd = runs[tk.x];
  if (!rd.active) return;  // host-set, constant within a captured graph

  const int l = tk.y, row0 = tk.z, nrows = tk.w;
  const int nx = rd.nx, ny = rd.ny;
  const int lgpx = rd.lgpx, lgM = lgpx - 1, M = 1 << lgM, ph = M + 1;
  const int cs = fft_stride(M);  // complex stride of one sequence in shared memory
  const int nseq = nrows * 3;
  const int ngr = nrows * nx;
  const LayerDev<R>& L = rd.L[l];
  const bool demag = rd.demag != 0;
  constexpr bool stats = (STAGE == kCorr) && STATS;

  Cx<R>* tws = reinterpret_cast<Cx<R>*>(smem_raw);  // e^{-2 pi i k/px}, k < px
  Cx<R>* bufA = tws + (1 << lgpx);
  Cx<R>* bufB = bufA + nseq * cs;
  __shared__ double sred[stats_slots<STAGE, STATS>()];

  // ---------------- static inputs (not written by the previous kernel) ----------------
  if (demag) stage_twiddles(tws, tw, lgpx);
  const V4<R>* __restrict__ mfield = (STAGE == kCorr) ? L.mp : L.m;
  const LayerDev<R>* Lu = (l > 0) ? &rd.L[l - 1] : nullptr;
  const LayerDev<R>* Ll = (l + 1 < rd.nl) ? &rd.L[l + 1] : nullptr;
  const bool stencil = L.xst != nullptr;
  const bool ucol = L.ucol && Lu, lcol = L.lcol && Ll;
  const bool thermal = (STAGE == kPred || STAGE == kCorr) && L.thermal;
  const V4<R>* __restrict__ mother_u = Lu ? ((STAGE == kCorr) ? Lu->mp : Lu->m) : nullptr;
  const V4<R>* __restrict__ mother_l = Ll ? ((STAGE == kCorr) ? Ll->mp : Ll->m) : nullptr;
  // inputs that the previous kernel does not write
  auto load_static = [&](GrainIn<R>& G, int n) {
    G.pb = L.pb[n];
    if (STAGE == kInit) return;
    G.pa = L.pa[n];
    if (stencil) G.cst = L.xst[n];
    if (ucol) G.cu = L.ucol[n];
    if (lcol) G.cl = L.lcol[n];
  };
  // inputs written by the previous kernels of this step
  auto load_dynamic = [&](GrainIn<R>& G, int n, int i, int j) {
    if (STAGE == kInit) {
      G.mf = L.m[n];
      return;
    }
    G.mf = mfield[n];
    if (stencil) {
      const int jm = (j == 0 ? ny - 1 : j - 1), jp = (j == ny - 1 ? 0 : j + 1);
      const int im = (i == 0 ? nx - 1 : i - 1), ip = (i == nx - 1 ? 0 : i + 1);
      G.nb[0] = mfield[jm * nx + i];
      G.nb[1] = mfield[j * nx + im];
      G.nb[2] = mfield[j * nx + ip];
      G.nb[3] = mfield[jp * nx + i];
    }
    if (STAGE == kCorr) {
      G.dm = L.dm[n];
      G.m0 = L.m[n];
      if (thermal) G.ht = L.ht[n];
    }
    if (ucol) G.vu = mother_u[n];
    if (lcol) G.vl = mother_l[n];
  };
  GrainIn<R> g[PREF ? GPT : 1];
  if constexpr (PREF) {
#pragma unroll
    for (int q = 0; q < GPT; ++q) {
      const int idx = threadIdx.x + q * BLOCK;
      if (idx >= ngr) continue;
      const int row = idx / nx, i = idx - row * nx;
      load_static(g[q], (row0 + row) * nx + i);
    }
  }

  // predictor: Philox thermal normals (llg.f90:1083 h = H + hthm/sqrt(dt); the
  // corrector reuses them, :1262-1266), drawn for the step counter read before
  // the wait and redrawn only if the previous kernel advanced it meanwhile
  const long long step_guess = rd.step + istep;
  const R tfac = thermal ? (R)sqrt(L.temperature / rd.dt) : (R)0;
  auto draw_one = [&](GrainIn<R>& G, int n, long long st) {
    R gn[3];
    thermal_normals(rd.seed, (unsigned long long)l, (unsigned long long)st, (unsigned long long)n, gn);
    const R s = G.pb.w * tfac;
    G.ht = V4<R>{s * gn[0], s * gn[1], s * gn[2], (R)0};
  };
  auto draw = [&](long long st) {
#pragma unroll
    for (int q = 0; q < GPT; ++q) {
      const int idx = threadIdx.x + q * BLOCK;
      if (idx >= ngr) continue;
      const int row = idx / nx, i = idx - row * nx;
      draw_one(g[q], (row0 + row) * nx + i, st);
    }
  };
  if constexpr (PREF) {
    if (STAGE == kPred && thermal) draw(step_guess);
  }

  // ---------------- wait for the previous kernel's results ----------------
  pdl_wait();
  const long long step = *reinterpret_cast<const volatile long long*>(&rd.step) + istep;
  if (!(flags & kFlagForce) && step >= rd.step_end) return;
  if constexpr (PREF) {
    if (STAGE == kPred && thermal && step != step_guess) draw(step);
  }

  // ---------------- dynamic per-grain inputs ----------------
  if constexpr (PREF) {
#pragma unroll
    for (int q = 0; q < GPT; ++q) {
      const int idx = threadIdx.x + q * BLOCK;
      if (idx >= ngr) continue;
      const int row = idx / nx, i = idx - row * nx, j = row0 + row;
      load_dynamic(g[q], j * nx + i, i, j);
    }
  }

  // ---------------- inverse row transform: H^ rows -> H_demag ----------------
  Cx<R>* Z = bufA;  // after the inverse: z[n] = x[2n] + i x[2n+1] per sequence
  if (STAGE != kInit && demag) {
    __syncthreads();  // staged twiddles visible to every thread
    const int tot = nseq * M;
    for (int base = threadIdx.x; base < tot; base += 4 * BLOCK) {
      Cx<R> xk[4], xm[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int idx = base + u * BLOCK;
        if (idx < tot) {
          const int s = idx >> lgM, k = idx & (M - 1);
          const int row = s / 3, comp = s - 3 * row;
          const Cx<R>* X = rd.spech + ((size_t)(l * 3 + comp) * ny + row0 + row) * ph;
          xk[u] = X[k];
          xm[u] = X[M - k];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int idx = base + u * BLOCK;
        if (idx < tot) {
          const int s = idx >> lgM, k = idx & (M - 1);
          Cx<R> a = xk[u], b = xm[u];
          if (k == 0) { a.y = 0; b.y = 0; }  // self-conjugate bins: imaginary parts ignored (c2r)
          const Cx<R> e = cadd(a, cconj(b));
          const Cx<R> o = csub(a, cconj(b));
          const Cx<R> w = cconj(tws[k]);  // e^{+2 pi i k / px}
          bufA[s * cs + k] = cadd(e, cmul_i(cmul(o, w), (R)1));
        }
      }
    }
    __syncthreads();
    Z = block_fft_c<R, +1, 1>(bufA, bufB, lgM, nseq, tws);
  }
  Cx<R>* W = (Z == bufA) ? bufB : bufA;  // real outputs of this stage (forward input)
  const R* hdr = reinterpret_cast<const R*>(Z);
  R* outr = reinterpret_cast<R*>(W);
  const int rs = 2 * cs;  // real stride of one sequence

  // ---------------- per-grain field + integrator stage ----------------
  const double t_now = rd.t_base + (double)(step - rd.step_base) * rd.dt;
  const double t_stage = (STAGE == kCorr) ? t_now + rd.dt : t_now;
  const double sc = ramp(L, t_stage);
  const R hax = (R)(sc * L.hdir[0]), hay = (R)(sc * L.hdir[1]), haz = (R)(sc * L.hdir[2]);
  const R dt = (R)rd.dt;
  const R gamma = (R)L.gamma;
  const bool store_field = (flags & kFlagStoreField) || STAGE == kEval;

  double rec[stats ? kNPart : 1];
#pragma unroll
  for (int s = 0; s < (stats ? kNPart : 1); ++s) rec[s] = 0.0;

#pragma unroll
  for (int q = 0; q < GPT; ++q) {
    const int idx = threadIdx.x + q * BLOCK;
    if (idx >= ngr) continue;
    const int row = idx / nx, i = idx - row * nx;
    const int n = (row0 + row) * nx + i;
    GrainIn<R>& G = g[PREF ? q : 0];
    if constexpr (!PREF) {
      load_static(G, n);
      load_dynamic(G, n, i, row0 + row);
      if (STAGE == kPred && thermal) draw_one(G, n, step);
    }
    const R mse = G.pb.x;  // Ms * ms_scale
    if (STAGE == kInit) {
      outr[(row * 3 + 0) * rs + i] = mse * G.mf.x;
      outr[(row * 3 + 1) * rs + i] = mse * G.mf.y;
      outr[(row * 3 + 2) * rs + i] = mse * G.mf.z;
      continue;
    }
    const V4<R> mf = G.mf;
    R hdx = 0, hdy = 0, hdz = 0;
    if (demag) {
      hdx = hdr[(row * 3 + 0) * rs + i];
      hdy = hdr[(row * 3 + 1) * rs + i];
      hdz = hdr[(row * 3 + 2) * rs + i];
    }
    // h = h_app + h_demag + H_uni + H_ex (+ interlayer)   (field.f90:201,211-220)
    R hx = hax + hdx, hy = hay + hdy, hz = haz + hdz;
    const V4<R> pa = G.pa, pb = G.pb;
    R e_k;
    {
      // get_uni_hk (field.f90:366-375); pa.w = Hk1*hk_scale, pb.y = Hk2*hk_scale
      const R hks = mf.x * pa.x + mf.y * pa.y + mf.z * pa.z;
      const R yy = (R)1 - hks * hks;
      const R f = hks * (pa.w + pb.y * yy);
      hx += f * pa.x;
      hy += f * pa.y;
      hz += f * pa.z;
      e_k = (R)0.5 * yy * (pa.w + (R)0.5 * pb.y * yy) * mse;
    }
    R ex = 0, ey = 0, ez = 0;
    if (stencil) {
      ex = G.cst.x * G.nb[0].x + G.cst.y * G.nb[1].x + G.cst.z * G.nb[2].x + G.cst.w * G.nb[3].x;
      ey = G.cst.x * G.nb[0].y + G.cst.y * G.nb[1].y + G.cst.z * G.nb[2].y + G.cst.w * G.nb[3].y;
      ez = G.cst.x * G.nb[0].z + G.cst.y * G.nb[1].z + G.cst.z * G.nb[2].z + G.cst.w * G.nb[3].z;
    } else if (L.xidx) {
      csr_sum<R>(L.xidx, L.xnbr, L.xcoef, mfield, n, ex, ey, ez);
    }
    R vx = 0, vy = 0, vz = 0;
    if (ucol) {
      vx += G.cu * G.vu.x; vy += G.cu * G.vu.y; vz += G.cu * G.vu.z;
    } else if (L.uidx && Lu) {
      csr_sum<R>(L.uidx, L.unbr, L.ucoef, (STAGE == kCorr) ? Lu->mp : Lu->m, n, vx, vy, vz);
    }
    if (lcol) {
      vx += G.cl * G.vl.x; vy += G.cl * G.vl.y; vz += G.cl * G.vl.z;
    } else if (L.lidx && Ll) {
      csr_sum<R>(L.lidx, L.lnbr, L.lcoef, (STAGE == kCorr) ? Ll->mp : Ll->m, n, vx, vy, vz);
    }
    hx += ex + vx;
    hy += ey + vy;
    hz += ez + vz;
    if (store_field) L.hf[n] = V4<R>{hx, hy, hz, (R)0};
    if (STAGE == kEval) {
      L.hd[n] = V4<R>{hdx, hdy, hdz, (R)0};
      continue;
    }

    // thermal field / sqrt(dt) (llg.f90:1083): drawn by the predictor, reused by the corrector
    R htx = 0, hty = 0, htz = 0;
    if (thermal) {
      htx = G.ht.x;
      hty = G.ht.y;
      htz = G.ht.z;
      if (STAGE == kPred) L.ht[n] = G.ht;
    }
    const R fx = hx + htx, fy = hy + hty, fz = hz + htz;
    V4<R> mn;
    R dx = 0, dy = 0, dz = 0, tq2 = 0;
    if (mse > (R)0) {
      const R a = pb.z;  // alpha * alpha_scale
      const R s11 = -gamma * dt / ((R)1 + a * a);
      R tx, ty, tz, ux, uy, uz;
      cross3(mf.x, mf.y, mf.z, fx, fy, fz, tx, ty, tz);
      cross3(mf.x, mf.y, mf.z, tx, ty, tz, ux, uy, uz);
      dx = s11 * (tx + a * ux);
      dy = s11 * (ty + a * uy);
      dz = s11 * (tz + a * uz);
      tq2 = tx * tx + ty * ty + tz * tz;
      V4<R> m0;
      if (STAGE == kPred) {
        L.dm[n] = V4<R>{dx, dy, dz, (R)0};
        m0 = mf;
      } else {
        dx = (R)0.5 * (dx + G.dm.x);
        dy = (R)0.5 * (dy + G.dm.y);
        dz = (R)0.5 * (dz + G.dm.z);
        m0 = G.m0;
      }
      mn.x = m0.x + dx;
      mn.y = m0.y + dy;
      mn.z = m0.z + dz;
      const R y = mn.x * mn.x + mn.y * mn.y + mn.z * mn.z;
      if (y > (R)0) {
        const R r = (R)1 / sqrt(y);
        mn.x *= r;
        mn.y *= r;
        mn.z *= r;
      }
    } else {
      // ms_scale <= 0: m along the (non-thermal) field (llg.f90:1140-1148)
      const R y = sqrt(hx * hx + hy * hy + hz * hz);
      if (y > (R)0) {
        mn.x = hx / y; mn.y = hy / y; mn.z = hz / y;
      } else {
        mn = (STAGE == kCorr) ? G.m0 : mf;
      }
    }
    mn.w = (R)0;
    if (STAGE == kPred) L.mp[n] = mn;
    else L.m[n] = mn;
    outr[(row * 3 + 0) * rs + i] = mse * mn.x;
    outr[(row * 3 + 1) * rs + i] = mse * mn.y;
    outr[(row * 3 + 2) * rs + i] = mse * mn.z;

    if constexpr (stats) {
      const V4<double> pv = L.pv[n];  // {vol, ms_scale, ms, 0}
      const double v = pv.x, w = pv.z * pv.y * v;
      const double mx = mn.x, my = mn.y, mz = mn.z;
      rec[kSlotV] += v;
      rec[kSlotM + 0] += v * mx;
      rec[kSlotM + 1] += v * my;
      rec[kSlotM + 2] += v * mz;
      rec[kSlotM2 + 0] += v * mx * mx;
      rec[kSlotM2 + 1] += v * my * my;
      rec[kSlotM2 + 2] += v * mz * mz;
      rec[kSlotH + 0] += v * (double)hx;
      rec[kSlotH + 1] += v * (double)hy;
      rec[kSlotH + 2] += v * (double)hz;
      rec[kSlotWM + 0] += w * mx;
      rec[kSlotWM + 1] += w * my;
      rec[kSlotWM + 2] += w * mz;
      rec[kSlotW] += w;
      if (mx * L.hdir[0] + my * L.hdir[1] + mz * L.hdir[2] > 0.0) rec[kSlotNup] += 1.0;
      rec[kSlotMaxTq] = fmax(rec[kSlotMaxTq], (double)tq2 / (pv.z * pv.z));
      rec[kSlotMaxD2] = fmax(rec[kSlotMaxD2], (double)(dx * dx + dy * dy + dz * dz));
      rec[kSlotMmag] += sqrt(mx * mx + my * my + mz * mz) * pv.y * v;
      // energy at the evaluated state (field.f90:200, :360, :374, :339)
      const double e_d = -((double)mf.x * ((double)hdx + hax) + (double)mf.y * ((double)hdy + hay) +
                           (double)mf.z * ((double)hdz + haz)) * (double)mse;
      const double e_x = -((double)(ex + vx) * mf.x + (double)(ey + vy) * mf.y +
                           (double)(ez + vz) * mf.z) * (double)mse;
      rec[kSlotE] += (e_d + (double)e_k + e_x) * v;
    }
  }
  if constexpr (stats) {
    block_reduce_record(rec, sred, part + (size_t)blockIdx.x * kNPart);
  }
  if (STAGE == kEval || !demag) return;

  // ---------------- forward row transform of Ms*m -> spectrum rows ----------------
  const int two_m = 2 * M;
  if (nx < two_m) {
    const int pad = two_m - nx;
    for (int idx = threadIdx.x; idx < nseq * pad; idx += BLOCK) {
      const int s = idx / pad, i = nx + (idx - s * pad);
      outr[s * rs + i] = (R)0;
    }
  }
  __syncthreads();
  Cx<R>* scratch = (W == bufA) ? bufB : bufA;
  Cx<R>* Y = block_fft_c<R, -1, 1>(W, scratch, lgM, nseq, tws);
  for (int idx = threadIdx.x; idx < nseq * ph; idx += BLOCK) {
    const int s = idx / ph, k = idx - s * ph;
    const int row = s / 3, comp = s - 3 * row;
    const Cx<R> yk = Y[s * cs + (k & (M - 1))];
    const Cx<R> ymk = cconj(Y[s * cs + ((M - k) & (M - 1))]);
    const Cx<R> e = cscale(cadd(yk, ymk), (R)0.5);
    const Cx<R> o = cscale(csub(yk, ymk), (R)0.5);
    // X[k] = e - i w^k o,  w = e^{-2 pi i / px}
    const Cx<R> wo = cmul(tws[k & (two_m - 1)], o);
    rd.specx[((size_t)(l * 3 + comp) * ph + k) * ny + row0 + row] = csub(e, cmul_i(wo, (R)1));
  }
}

// Column kernel: per spectral column k, forward FFT along y of the 3*nl
// half-spectra, H^_a = sum_b N^_ab M^_b, inverse FFT, written back in place.
// PACKED: tensor stored as one real per (k, 0<=ky<=py/2) and component (the
// parity of each component restores the rest); otherwise the full complex
// tensor spectrum [k][pair][9][py] is used (FP64 runs).
// packed tensor slice of a column task staged in shared memory up to this size
constexpr int kTensSliceBytes = 48 * 1024;
template <typename R>
MRM_HD bool tens_slice_fits(int reals) { return (size_t)reals * sizeof(R) <= (size_t)kTensSliceBytes; }

template <typename R, bool PACKED, int BLOCK>
__global__ void __launch_bounds__(BLOCK, PACKED ? 3 : 1) col_kernel(const RunDev<R>* __restrict__ runs,
                                                    const Task* __restrict__ tasks,
                                                    const Cx<R>* __restrict__ tw, int istep,
                                                    int flags) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_launch_dependents();
  const Task tk = tasks[blockIdx.x];
  const RunDev<R>& rd = runs[tk.x];
  if (!rd.active || !rd.demag) return;
  const int k0 = tk.y, nc = tk.z;
  const int nl = rd.nl, ny = rd.ny, py = rd.py, lgpy = rd.lgpy;
  const int ph = (rd.px >> 1) + 1, pyh = (py >> 1) + 1;
  const int cs = fft_stride(py);
  const int nseq = nc * nl * 3;  // s = (c*nl + layer)*3 + comp
  Cx<R>* tws = reinterpret_cast<Cx<R>*>(smem_raw);  // e^{-2 pi i k/py}, k < py
  Cx<R>* A = tws + py;
  Cx<R>* B = A + nseq * cs;

  // static inputs: twiddles and this task's packed tensor slice (when it fits)
  stage_twiddles(tws, tw, lgpy);
  const int npair = nl * nl;
  const int tslice = nc * npair * 9 * pyh;  // reals
  const bool tsm = PACKED && tens_slice_fits<R>(tslice);
  R* Ts = reinterpret_cast<R*>(B + nseq * cs);
  if (tsm) {
    const R* src = rd.tens + (size_t)k0 * npair * 9 * pyh;  // columns k0.. are contiguous
    for (int q = threadIdx.x; q < tslice; q += BLOCK) Ts[q] = __ldg(src + q);
  }
  pdl_wait();
  if (!(flags & kFlagForce) && rd.step + istep >= rd.step_end) return;

  // batched, coalesced loads of the columns (column-major M^; rows >= ny are the zero padding)
  const int tot = nseq * py;
  for (int base = threadIdx.x; base < tot; base += 4 * BLOCK) {
    Cx<R> v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int idx = base + u * BLOCK;
      v[u] = Cx<R>{(R)0, (R)0};
      if (idx < tot) {
        const int j = idx & (py - 1), s = idx >> lgpy;  // s = c*nl*3 + lc
        const int c = s / (nl * 3), lc = s - c * nl * 3;
        if (j < ny) v[u] = rd.specx[((size_t)lc * ph + k0 + c) * ny + j];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int idx = base + u * BLOCK;
      if (idx < tot) A[(idx >> lgpy) * cs + (idx & (py - 1))] = v[u];
    }
  }
  __syncthreads();
  Cx<R>* F = block_fft_c<R, -1, 0>(A, B, lgpy, nseq, tws);
  Cx<R>* G = (F == A) ? B : A;

  // H^_a(k, ky) = sum_ks sum_b N^_ab(ko,ks)(k, ky) M^_b(ks)(k, ky)
  for (int idx = threadIdx.x; idx < nc * py; idx += BLOCK) {
    const int c = idx / py, ky = idx - c * py;
    for (int ko = 0; ko < nl; ++ko) {
      Cx<R> h[3] = {{0, 0}, {0, 0}, {0, 0}};
      for (int ks = 0; ks < nl; ++ks) {
        Cx<R> xm[3];
#pragma unroll
        for (int b = 0; b < 3; ++b) xm[b] = F[((c * nl + ks) * 3 + b) * cs + ky];
        if constexpr (PACKED) {
          const bool upper = ky > (py >> 1);
          const int kyh = upper ? py - ky : ky;
          const size_t off = ((size_t)c * npair + ks * nl + ko) * 9 * pyh;
          const R* Tp = tsm ? Ts + off : rd.tens + (size_t)k0 * npair * 9 * pyh + off;
          R tv[9];
#pragma unroll
          for (int cc = 0; cc < 9; ++cc) tv[cc] = Tp[cc * pyh + kyh];
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
              const int cc = 3 * a + b;
              R v = tv[cc];
              if (((kOddMask >> cc) & 1) && upper) v = -v;
              if ((kImagMask >> cc) & 1) h[a] = cadd(h[a], cmul_i(cscale(xm[b], v), (R)1));
              else h[a] = cadd(h[a], cscale(xm[b], v));
            }
        } else {
          const Cx<R>* Tc = reinterpret_cast<const Cx<R>*>(rd.tens) +
                            ((size_t)(k0 + c) * npair + ks * nl + ko) * 9 * py;
          Cx<R> tv[9];
#pragma unroll
          for (int cc = 0; cc < 9; ++cc) tv[cc] = Tc[cc * py + ky];
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) h[a] = cadd(h[a], cmul(tv[3 * a + b], xm[b]));
        }
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) G[((c * nl + ko) * 3 + a) * cs + ky] = h[a];
    }
  }
  __syncthreads();
  Cx<R>* Hs = block_fft_c<R, +1, 0>(G, F, lgpy, nseq, tws);

  const int tot2 = nseq * ny;
  for (int idx = threadIdx.x; idx < tot2; idx += BLOCK) {
    const int c = idx % nc, rest = idx / nc;
    const int j = rest % ny, lc = rest / ny;
    rd.spech[((size_t)lc * ny + j) * ph + k0 + c] = Hs[(c * nl * 3 + lc) * cs + j];
  }
}

// Advances every active run's step counter after a captured chunk of k steps.
template <typename R>
__global__ void advance_kernel(RunDev<R>* runs, int nruns, int k) {
  pdl_launch_dependents();
  pdl_wait();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  RunDev<R>& rd = runs[r];
  if (!rd.active) return;
  long long left = rd.step_end - rd.step;
  if (left < 0) left = 0;
  rd.stats_ok = left >= k ? 1 : 0;
  rd.step += (left < k) ? left : k;
}

// mrm_gpu_stats layout
struct StatsDev {
  double t;
  long long step;
  double mave[3], mvar[3], have[3];
  double errmx, errmx1, mmag, energy;
  double mave_l[kMaxLayers][3], mvar_l[kMaxLayers][3], have_l[kMaxLayers][3], mms_l[kMaxLayers][3];
  double vol_l[kMaxLayers], msvol_l[kMaxLayers];
  long long nup_l[kMaxLayers];
};

// FP64 reduction of each run's per-task stats records into StatsDev; one
// 256-thread block per run, fixed reduction order (deterministic).
template <typename R>
__global__ void __launch_bounds__(256) finalize_stats_kernel(const RunDev<R>* __restrict__ runs,
                                                             const Task* __restrict__ tasks,
                                                             const double* __restrict__ part,
                                                             StatsDev* __restrict__ out, int nruns) {
  __shared__ double sred[32 * kNPart];
  __shared__ double acc[kMaxLayers][kNPart];
  pdl_launch_dependents();
  pdl_wait();
  const int r = blockIdx.x;
  if (r >= nruns) return;
  const RunDev<R>& rd = runs[r];
  if (!rd.active || !rd.stats_ok) return;  // keep the stats of the run's last stats step
  for (int l = 0; l < rd.nl; ++l) {
    double rec[kNPart];
#pragma unroll
    for (int s = 0; s < kNPart; ++s) rec[s] = 0.0;
    for (int q = rd.row_task0 + threadIdx.x; q < rd.row_task0 + rd.nrow_tasks; q += blockDim.x) {
      if (tasks[q].y != l) continue;
      const double* p = part + (size_t)q * kNPart;
#pragma unroll
      for (int s = 0; s < kNPart; ++s) rec[s] = slot_is_max(s) ? fmax(rec[s], p[s]) : rec[s] + p[s];
    }
    block_reduce_record(rec, sred, acc[l]);
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  StatsDev& st = out[r];
  st.step = rd.step;
  st.t = rd.t_base + (double)(rd.step - rd.step_base) * rd.dt;
  double vt = 0, mt = 0, m1 = 0, mmag = 0, en = 0;
  for (int a = 0; a < 3; ++a) { st.mave[a] = 0; st.mvar[a] = 0; st.have[a] = 0; }
  for (int l = 0; l < rd.nl; ++l) vt += acc[l][kSlotV];
  for (int l = 0; l < kMaxLayers; ++l) {
    const bool on = l < rd.nl;
    const double V = on ? acc[l][kSlotV] : 0.0;
    for (int a = 0; a < 3; ++a) {
      const double mean = (on && V > 0) ? acc[l][kSlotM + a] / V : 0.0;
      st.mave_l[l][a] = mean;
      st.mvar_l[l][a] = (on && V > 0) ? acc[l][kSlotM2 + a] / V - mean * mean : 0.0;
      st.have_l[l][a] = (on && V > 0) ? acc[l][kSlotH + a] / V : 0.0;
      const double W = on ? acc[l][kSlotW] : 0.0;
      st.mms_l[l][a] = on ? acc[l][kSlotWM + a] * W / (W * W + 1e-300) : 0.0;
    }
    st.vol_l[l] = V;
    st.msvol_l[l] = on ? acc[l][kSlotW] : 0.0;
    st.nup_l[l] = on ? (long long)acc[l][kSlotNup] : 0;
    if (on && V > 0) {
      for (int a = 0; a < 3; ++a) {
        st.mave[a] += V * st.mave_l[l][a] / vt;
        st.mvar[a] += V * st.mvar_l[l][a] / vt;
        st.have[a] += V * st.have_l[l][a] / vt;
      }
      mmag += acc[l][kSlotMmag] / V;
      mt = fmax(mt, acc[l][kSlotMaxTq]);
      m1 = fmax(m1, acc[l][kSlotMaxD2]);
      en += acc[l][kSlotE];
    }
  }
  st.errmx = sqrt(mt);
  st.errmx1 = m1;
  st.mmag = mmag;
  st.energy = en;
}

}  // namespace mrm
