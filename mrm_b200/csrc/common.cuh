// common.cuh -- device types shared by the grain-dynamics kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define MRM_HD __host__ __device__ __forceinline__
#define MRM_D __device__ __forceinline__

namespace mrm {

constexpr int kMaxLayers = 8;
constexpr int kTwLog = 12;                 // FFT lengths <= 4096
constexpr int kTwN = 1 << kTwLog;
constexpr int kNPart = 20;                 // doubles per row-task stats record

template <typename R>
struct alignas(2 * sizeof(R)) Cx {
  R x, y;
};

template <typename R>
struct alignas(4 * sizeof(R)) V4 {
  R x, y, z, w;
};

template <typename R>
MRM_HD Cx<R> cmul(Cx<R> a, Cx<R> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename R>
MRM_HD Cx<R> cadd(Cx<R> a, Cx<R> b) { return {a.x + b.x, a.y + b.y}; }
template <typename R>
MRM_HD Cx<R> csub(Cx<R> a, Cx<R> b) { return {a.x - b.x, a.y - b.y}; }
template <typename R>
MRM_HD Cx<R> cconj(Cx<R> a) { return {a.x, -a.y}; }
template <typename R>
MRM_HD Cx<R> cscale(Cx<R> a, R s) { return {a.x * s, a.y * s}; }
// multiply by i*s (s = +1 or -1)
template <typename R>
MRM_HD Cx<R> cmul_i(Cx<R> a, R s) { return {-s * a.y, s * a.x}; }

// FP32 sums and differences on sm_100 as one paired add (FADD2: both lanes
// rounded as two scalar adds would be), half the issue slots of the butterflies
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
template <>
MRM_HD Cx<float> cadd<float>(Cx<float> a, Cx<float> b) {
  const float2 r = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
  return {r.x, r.y};
}
template <>
MRM_HD Cx<float> csub<float>(Cx<float> a, Cx<float> b) {
  const float2 r = __fadd2_rn(make_float2(a.x, a.y), make_float2(-b.x, -b.y));
  return {r.x, r.y};
}
#endif

// Tabulated (moving) field profile of a layer, in device memory: file_applied
// + set + interpolate (applied.f90:711-813,1471-1520,1757-1776).  Values
// v[c + 3 (i + nx j)] (Oe) at table nodes pos[i] (x), pos[nx + j] (y) (cm); the
// profile's origin sits at ox + vx (t - t0) - rx (y alike) on the grid, whose
// cell (i, j) centre is ((i + 1/2) dx, (j + 1/2) dy).
struct TabDev {
  const double* v;
  const double* pos;
  int nx, ny;
  double ox, oy, vx, vy, rx, ry, t0, dx, dy;
};

// LLB integrator of a layer (llgp%llb: push_llb, llg.f90:916-1064), in device
// memory: per grain {Tc, lambda_m = lambdaMs (spin + 1)/spin,
// 2 k_B alpha alpha_scale / (gamma Ms V) (get_thermal's variance without
// T/|m|), 0}; the layer's spin, damping alpha and floor_ms (get_thermal's
// |m| floor); the temperature is the layer's (LayerDev::temperature).  The
// grain's magnitude |m| (mag) rides in the w lane of m and mp.
// mode 1 is the MT integrator (llgp%mt: push_mt, llg.f90:735-915), mode 2 the
// Zhang integrator (llgp%zhang: push_zhang, :410-703), on the same records (Tc
// unused, lambdaMs raw), with the Brillouin equilibrium (meq_bs) and
// Garanin's tau (garanin_tau) as options.
struct LlbDev {
  const V4<double>* p;
  double spin, alpha, floor_ms;
  int mode, meq_bs, garanin_tau;
};

// Moving super-Gaussian temperature profile of a layer (HAMR: suprgaus_temp,
// set_sg / get_sg and the temperature branch of get_appl / get_applied,
// applied.f90:446-483,889-896,1778-1809, field.f90:546-560), in device
// memory: T(cell (i, j), t) = bg + s(t) dtemp fx(i) fy(j),
// fx(i) = exp(-(((i + 1/2) dx + rx - vx (t - t0) - ox) isx)^expn) (y alike,
// isx = 1/sigma_x, 0: flat), s(t) the profile's own time scale (linear ramp
// or funct, as a field's).
struct TempDev {
  double bg, dtemp, isx, isy, vx, vy, ox, oy, rx, ry, t0, dx, dy;
  int expn;
  int func;
  double t_start, t_end, s_start, s_end, scale, amp, fgamma, phase, param, duty, moddepth, dc;
};

// Temperature scaling of a layer (find_temp_scaling, temp_scaling.f90:365-433),
// in device memory: the cells' Tc; power laws (1 - T/Tc)^e of Ms and Hk
// (e < 0: none); Ms scaled by |m| instead (mag, the LLB magnitude); reduced
// tables T/Tc -> scale of Ms, alpha and Hk (table k: nt[k] nodes at
// tt + off[k], tv + off[k]; fewer than 2 nodes: none); floor_ms of the
// thermal variance.  The layer was uploaded with unit scales, which these
// replace at every field evaluation.
struct TscDev {
  const double* tc;
  const double* tt;
  const double* tv;
  int off[3], nt[3];
  double msexp, hkexp, floor_ms;
  int mag;
};

// Per-layer device view of one run.  State vectors are float4/double4
// "SoA of 4-vectors": (x,y,z,w) per grain for one 16/32-byte load (w of m and
// mp: the magnitude |m| of the LLB integrator; unused otherwise).
template <typename R>
struct LayerDev {
  V4<R>* m;         // m_n (state at step boundaries)
  V4<R>* mp;        // Heun predictor m*
  V4<R>* dm;        // predictor increment d1
  V4<R>* hf;        // last non-thermal total field (get_field output)
  V4<R>* hd;        // demag field of the last evaluation-only pass
  V4<R>* ht;        // thermal field / sqrt(dt) of the current step (predictor -> corrector)
  const V4<R>* pa;  // {kx, ky, kz, Hk1*hk_scale}
  const V4<R>* pb;  // {Ms*ms_scale, Hk2*hk_scale, alpha*alpha_scale, sigma0}
  const V4<double>* pv;  // {vol, ms_scale, ms, 0} (FP64, reductions)
  const int* xidx;  // intralayer exchange CSR (0-based), coef includes ms_scale(nbr)
  const int* xnbr;
  const R* xcoef;
  const int* uidx;  // interlayer: couples to layer-1
  const int* unbr;
  const R* ucoef;
  const int* lidx;  // interlayer: couples to layer+1
  const int* lnbr;
  const R* lcoef;
  const V4<R>* xst;  // lattice form of the intralayer exchange: coef of (j-1, i-1, i+1, j+1)
  // cubic anisotropy (null: uniaxial): per grain the crystal axes a1, a2, a3 in
  // lab coordinates as 3 records, a1's w = hk_scale * Ms (energy term)
  const V4<R>* cax;
  // grains of several cells (null cgrain: one grain per cell in grid order):
  // the cell's grain (-1: empty cell), each grain's cells (gcs[gci[g]..gci[g+1]),
  // the first one is the grain's own), the grain-averaged demag per cell
  const int* cgrain;
  const int* gci;
  const int* gcs;
  V4<R>* hdm;
  V4<R>* hapm;       // grain-averaged tabulated applied field per cell (map layers with a table)
  const R* ucol;     // columnar form of the interlayer coupling (grain n <-> grain n)
  const R* lcol;
  double hdir[3];
  double t_start, t_end, s_start, s_end, scale;
  int func;  // 0 linear ramp; 1 SIN, 2 COS, 3 EXP, 4 STE, 5 NEW, 7 ROT (applied.f90:328-396); 6 head
  double amp, fgamma, phase, param, duty, moddepth, dc;
  // moving write head (func 6): Karlqvist field of a ring head, gap hd_gap, at
  // distance hd_z above the layer's mid-plane, deep-gap field hd_hg, gap centre
  // at hd_x0 + hd_v (t - hd_t0) down-track; write polarity from bit
  // floor((t - hd_t0)/hd_tbit) mod hd_nbits of hd_bits; grain column i at (i + 1/2) hd_dx
  double hd_gap, hd_z, hd_hg, hd_v, hd_x0, hd_t0, hd_tbit, hd_dx;
  unsigned long long hd_bits;
  int hd_nbits;
  const struct TabDev* tab;  // tabulated field profile (null: the uniform hdir applies)
  const LlbDev* llb;         // LLB integrator (null: LLG)
  const TempDev* tprof;      // temperature profile (null: the uniform temperature)
  const TscDev* tsc;         // temperature scaling of Ms, alpha, Hk (null: the uploaded scales)
  double temperature;
  double gamma;
  int thermal;
  int n;
};

// Device descriptor of one run (one medium realisation).
template <typename R>
struct RunDev {
  int nx, ny, nl;
  int px, py, lgpx, lgpy;  // FFT grid (px = 2^lgpx)
  int demag;
  int ncomp;               // tensor components stored per pair (9)
  double dt;
  double t_base;           // time at step index step_base
  long long step_base;
  long long step;          // current step index (advanced by the advance kernel)
  long long step_end;      // the run advances while step < step_end
  long long step_begin;    // and idles while step < step_begin (an aligned start inside a call)
  unsigned long long seed;
  int active;
  int stats_ok;            // set by the advance kernel: the chunk's last step was executed
  int row_task0, nrow_tasks;  // range of this run's row tasks (stats partials)
  int phs, nys, pyhs;      // padded strides: spectrum row (px/2+1 -> even), spectrum column
                           // (ny -> even), packed tensor row (py/2+1 -> multiple of 4)
  int tw_row, tw_col;      // offsets of this grid's twiddle blocks in the global table (fft.cuh)
  Cx<R>* spech;            // H^ half spectra, row-major [nl][3][ny][phs] (column kernel -> row kernel)
  int lgct;                // log2 of the column-tile width T (= columns per column task)
  Cx<R>* specx;            // M^ half spectra in column tiles [nl*3][ntile][nys][T], ntile = ceil((px/2+1)/T)
                           // (row kernel -> column kernel)
  // moving demag window (gnx = 0: none): the FFT grid covers the nx x ny cells
  // from grid column wi0, row wj0 of the full gnx x gny grid of the per-grain
  // arrays; frz: the run's first stats record of the frozen grains (-1: none)
  int gnx, gny, wi0, wj0, frz;
  const R* tens;           // tensor spectrum: FP32 packed [px/2+1][nl*nl][9][pyhs] reals,
                           // FP64 full [px/2+1][nl*nl][9][py] complex
  LayerDev<R> L[kMaxLayers];
};

constexpr int kFuncHead = 6;
constexpr int kFuncRot = 7;  // the ROT time function: an in-plane field rotating at rate gamma

// Tensor component parity (c = 3*field + source): the spectrum is purely
// imaginary for xz, yz, zx, zy and odd in ky for xy, yx, yz, zy.
constexpr int kImagMask = (1 << 2) | (1 << 5) | (1 << 6) | (1 << 7);
constexpr int kOddMask = (1 << 1) | (1 << 3) | (1 << 5) | (1 << 7);

// Whether a run executes step `step` of a call: inside its budget and past its
// aligned start.
template <typename R>
MRM_HD bool step_due(const RunDev<R>& rd, long long step) {
  return step >= rd.step_begin && step < rd.step_end;
}

// row task: (run, layer, first row, number of rows); column task: (run, first column, ncols, 0)
using Task = int4;

}  // namespace mrm
