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
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mrm_gpu.h"
#include "common.cuh"
#include "kernels.cuh"
#include "launch.h"
#include "tensor.cuh"
#include "colreg.cuh"

using namespace mrm;

namespace {

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
  void* cax = nullptr;   // V4<R> x 3 per grain: cubic crystal axes (null: uniaxial)
  void* ucol = nullptr;  // R columnar interlayer coefficients (null: CSR form)
  void* lcol = nullptr;
  // grains of several cells (map layers): cell -> grain (-1 empty), grain -> cells
  // CSR, grain-averaged demag per cell; null on one-grain-per-cell layers
  int *cgrain = nullptr, *gci = nullptr, *gcs = nullptr;
  void* hdm = nullptr;
  void* hapm = nullptr;  // grain-averaged tabulated applied field per cell (map layers)
  int ng = 0;  // grains (n counts cells)
  double hdir[3] = {0, 0, 0};
  double t_start = -1e22, t_end = 1e22, s_start = 1.0, s_end = 1.0, scale = 1.0;
  int func = 0;
  double amp = 0, fgamma = 0, phase = 0, param = 0, duty = 0, moddepth = 0, dc = 0;
  double temperature = 0.0, gamma = 1.76e7, alpha = 0.1;
  int thermal = 0;
  double hd_gap = 0, hd_z = 1, hd_hg = 0, hd_v = 0, hd_x0 = 0, hd_t0 = 0, hd_tbit = 1;
  unsigned long long hd_bits = 0;
  int hd_nbits = 1;
  // tabulated field profile (null tab: none): the device TabDev, its FP64
  // values (3, nx, ny) and node positions (x then y)
  void* tab = nullptr;
  void* tb_v = nullptr;
  void* tb_pos = nullptr;
  // LLB integrator (null llb: LLG): the device LlbDev and its per-cell records
  void* llb = nullptr;
  void* llbp = nullptr;
  double floor_ms = 0.01;
  // temperature profile (null tprof: the uniform temperature): device TempDev and its host copy
  void* tprof = nullptr;
  TempDev tp{};
  // temperature scaling (null tsc: off): device TscDev, the cells' Tc, the
  // concatenated tables; host copies of the settings and reduced tables
  // (Ms, alpha, Hk, Hx)
  void* tsc = nullptr;
  void* tsc_tc = nullptr;
  void* tsc_tab = nullptr;
  bool tsc_on = false;
  double tsc_msexp = -1.0, tsc_hkexp = -1.0;
  int tsc_mag = 0;
  std::vector<double> tsc_t[4], tsc_v[4];
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
  void* xfer = nullptr;  // 3 x N doubles: host <-> device transfers of one layer's state
  void* slab = nullptr;  // one allocation holding xfer and every layer's per-grain arrays
  // tensor spectrum: runs whose tensor was copied from a run of the same
  // geometry share that run's buffer (tens_buf owns it; tens is its address),
  // so a batch of one geometry reads one tensor, which stays in L2
  void* tens = nullptr;
  std::shared_ptr<void> tens_buf;
  bool tensor_ready = false;
  bool demag = true;
  double tensor_resid = 0.0, tensor_kept = 0.0;
  double dt = 1e-13, t_base = 0.0;
  long long step_base = 0, step = 0, step_end = 0;
  long long step_begin = -(long long)9e18;  // idles while step < step_begin (mrm_batch_delay_run)
  unsigned long long seed = 1;
  bool active = true;
  bool spec_valid = false;
  bool has_stats = false;
  int slot = -1;
  int lgct = 0;  // log2 of the column-tile width (= columns per column task)
  int row_task0 = 0, nrow_tasks = 0;
  // moving demag window (wnx = 0: none; window_m, data.f90:1-65): its size, its
  // velocity and offset (window%v, window%offset), its current origin (-1: not
  // placed yet); frz: the run's first frozen-grain stats record
  int wnx = 0, wny = 0, wi0 = -1, wj0 = -1, frz = -1;
  // the grid's own FFT exceeds the path's limits: no full-grid spectra or
  // tensor; demag only through a moving window
  bool fft_big = false;
  double wvx = 0, wvy = 0, wox = 0, woy = 0;
  // the time as llg() accumulates it (t = t + dt, llg.f90:268), which places
  // the window: t_base + k dt can differ from it in the last bit, and a window
  // edge at an exact half cell would then move a step early or late
  double t_acc = 0.0;
  std::string err;
};

namespace {

struct Engine {
  int prec = MRM_FP32;
  int dev = 0;
  cudaStream_t st = nullptr;
  std::vector<mrm_gpu*> runs;
  // removed runs whose device memory is released at the next stats, step or
  // destroy (after the stream has passed their last use)
  std::vector<mrm_gpu*> retired;
  void* d_runs = nullptr;  // RunDev<R>[cap]
  int runs_cap = 0;
  Task* d_rtasks = nullptr;
  Task* d_ctasks = nullptr;
  int nrt = 0, nct = 0, rt_cap = 0, ct_cap = 0;
  Task* d_ctasks2 = nullptr;  // column tasks of the register column kernel's runs (colreg.cuh)
  int nct2 = 0, ct2_cap = 0;
  int rowv = 0, colv = 0, cpt = 0;  // row / column shapes (launch.h), columns per task (0: default)
  bool shape_forced = false;         // shapes set by the caller instead of tuned
  int force_rowv = 0, force_colv = 0, force_cpt = 0;
  bool autotune = true;
  size_t smem_row[kRowSlots] = {0, 0, 0, 0, 0, 0};  // per launch slot (launch.h row_slot)
  int stage_cap[kRowSlots] = {0, 0, 0, 0, 0, 0};
  size_t smem_col = 0;
  size_t smem_creg = 0;
  int creg_tw_cap = 0, creg_blocks = 0;  // register column kernel: twiddle room, persistent blocks
  // the corrector with reductions always runs row shape 0 over one-row tasks,
  // so that the FP64 reductions do not depend on the tuned shapes
  Task* d_stasks = nullptr;
  int nst = 0, st_cap = 0;
  size_t smem_stats[2] = {0, 0};  // reductions launch of kPred (single-stage integrator), kCorr
  int cap_stats[2] = {0, 0};
  int* d_err = nullptr;              // device error flag (tma.cuh DeviceError bits)
  bool has_window = false;           // a run with a moving demag window (general kernels)
  bool has_head = false;             // a run has a layer under the write head or a tabulated
                                     // field profile (general kernels)
  bool has_cubic = false;            // a run has a cubic-anisotropy layer (general kernels)
  bool has_llb = false;              // a run integrates with LLB / MT / Zhang (the level-2 kernels)
  bool has_tprof = false;            // a run has a temperature profile (the level-2 kernels)
  bool pred_stored = false;          // next chunk's first predictor pushes with the stored field
  bool mapped = false;               // a run has grains of several cells (grain-averaged demag)
  double* d_part = nullptr;
  int part_cap = 0;
  StatsDev* d_stats = nullptr;
  StatsDev* h_stats = nullptr;  // pinned
  int nslots = 0;               // runs in the current tables (stats slots 0 .. nslots-1)
  int stats_cap = 0;
  void* d_tw = nullptr;  // Cx<R>[tw_table_size()] (fft.cuh layout)
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

// The engine streams are non-blocking: they do not wait for work on the
// legacy default stream.  Zero-fills and uploads issued there therefore
// complete before these helpers return (a cudaMemset is asynchronous, and a
// pageable host-to-device cudaMemcpy may return before its DMA lands), so no
// later kernel on an engine stream can overtake them.
int dmalloc(std::string* errp, void** p, size_t bytes) {
  CK(cudaMalloc(p, bytes ? bytes : 16));
  CK(cudaMemset(*p, 0, bytes ? bytes : 16));
  CK(cudaStreamSynchronize(cudaStreamLegacy));
  return MRM_OK;
}

cudaError_t h2d(void* dst, const void* src, size_t bytes) {
  const cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(cudaStreamLegacy);
}

void dfree(void*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

struct CudaFreeDeleter {
  void operator()(void* p) const {
    if (p) cudaFree(p);
  }
};
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
  // twiddle table of every row / column FFT length (fft.cuh layout), in FP64
  std::vector<double> tw(2 * (size_t)tw_table_size(), 0.0);
  auto put = [&](int at, double num, double den) {
    const double a = -2.0 * M_PI * num / den;
    tw[2 * (size_t)at] = std::cos(a);
    tw[2 * (size_t)at + 1] = std::sin(a);
  };
  auto pass_tables = [&](int at, int lgn) {
    for (int lgns = 0; lgns < lgn;) {
      const int lgr = pass_lgr(lgn, lgns), R = 1 << lgr, NS = 1 << lgns;
      if (lgns > 0) {
        for (int r = 1; r < R; ++r)
          for (int k = 0; k < NS; ++k) put(at + (r - 1) * NS + k, (double)k * r, (double)NS * R);
        at += (R - 1) * NS;
      }
      lgns += lgr;
    }
  };
  for (int lg = 1; lg <= kTwLog; ++lg) {
    const int o = row_tw_off(lg), M = 1 << (lg - 1);
    for (int k = 0; k <= M; ++k) put(o + k, (double)k, (double)(2 * M));
    pass_tables(o + row_tw_post(lg), lg - 1);
    pass_tables(col_tw_off(lg), lg);
  }
  const size_t ntw = (size_t)tw_table_size();
  if (prec == MRM_FP64) {
    int rc = dmalloc(errp, &e->d_tw, sizeof(double) * 2 * ntw);
    if (rc) return rc;
    CK(h2d(e->d_tw, tw.data(), sizeof(double) * 2 * ntw));
  } else {
    std::vector<float> twf(2 * ntw);
    for (size_t k = 0; k < 2 * ntw; ++k) twf[k] = (float)tw[k];
    int rc = dmalloc(errp, &e->d_tw, sizeof(float) * 2 * ntw);
    if (rc) return rc;
    CK(h2d(e->d_tw, twf.data(), sizeof(float) * 2 * ntw));
  }
  {
    int rc = dmalloc(errp, (void**)&e->d_err, 4 * sizeof(int));  // flags, first check code, its value
    if (rc) return rc;
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
  dfree(e->d_ctasks2);
  dfree(e->d_stasks);
  dfree(e->d_part);
  dfree(e->d_stats);
  if (e->h_stats) cudaFreeHost(e->h_stats);
  e->h_stats = nullptr;
  dfree(e->d_tw);
  dfree(e->d_err);
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

// padded strides (16-byte aligned rows for the bulk copies of the kernels)
int spec_row_stride(int px) { return even_up(px / 2 + 1); }  // complex per spectrum row
int spec_col_stride(int ny) { return even_up(ny); }          // complex per spectrum column
int tens_row_stride(int py) { return (py / 2 + 1 + 3) & ~3; } // reals per packed tensor row

// default columns per column task: about 16 complex values per thread of a 256-thread block
int default_cols(const mrm_gpu* r) {
  const int ph = r->px / 2 + 1;
  return std::max(1, std::min(ph, 256 * 16 / (3 * r->nl * r->py)));
}
// columns per column task: also the width of the column tiles of the M^
// spectrum, so a power of two up to kMaxColTile
constexpr int kMaxColTile = 8;
int col_tile(int want) {
  int t = 1;
  while (2 * t <= std::min(want, kMaxColTile)) t *= 2;
  return t;
}
int cols_per_task(const Engine* e, const mrm_gpu* r) { return col_tile(e->cpt > 0 ? e->cpt : default_cols(r)); }
// shape of the register column kernel: the column shape index
int creg_v(const Engine* e) { return std::min(std::max(e->colv, 0), kCregVariants - 1); }
// cells per row and rows of the FFT source (the moving demag window, else the grid)
int fnx(const mrm_gpu* r) { return r->wnx ? r->wnx : r->g.nx; }
int fny(const mrm_gpu* r) { return r->wnx ? r->wny : r->g.ny; }
// complex values of the M^ spectrum of a run (column tiles of any width up to kMaxColTile)
size_t specx_count(const mrm_gpu* r) {
  const int ph = r->px / 2 + 1;
  return (size_t)r->nl * 3 * ((ph + kMaxColTile - 1) / kMaxColTile * kMaxColTile) * spec_col_stride(fny(r));
}
// (a windowed run's rows are segments of the grid's rows: one per task)
int rows_per_task(const mrm_gpu* r, int rpb) { return r->wnx ? 1 : std::max(1, std::min(rpb, r->g.ny)); }

// Runs whose column step is the register column kernel (colreg.cuh): FP32,
// one layer, 256..1024-point columns.  Their tensor is stored in that
// kernel's layout (tensor.cuh pack_tensor_creg_kernel).
bool creg_run(const mrm_gpu* r) {
  return r->g.precision == MRM_FP32 && r->nl == 1 && r->lgpy >= kCregMinLg && r->lgpy <= kCregMaxLg &&
         !r->fft_big;
}

size_t tensor_bytes(const mrm_gpu* r) {
  const size_t ph = r->px / 2 + 1, npair = (size_t)r->nl * r->nl;
  if (r->g.precision == MRM_FP64) return ph * npair * 9 * r->py * 2 * sizeof(double);
  if (creg_run(r)) return ph * 6 * r->py * sizeof(float);
  return ph * npair * 9 * tens_row_stride(r->py) * sizeof(float);
}

// row-kernel launch slots: kInit, kPred, kCorr, kCorr with reductions, kEval
constexpr int kSlots = kRowSlots;
constexpr int kSlotStage[kSlots] = {kInit, kPred, kCorr, kCorr, kEval, kPred};
// static shared memory of a row stage (mbarriers, reduction scratch) with margin
size_t row_static_bytes(int slot) {
  return ((slot == 3 || slot == 5) ? 32 * kNPart * sizeof(double) : sizeof(double)) + 64;
}
constexpr size_t kSmemPerSM = 228 * 1024;
constexpr size_t kSmemReserved = 1024;  // per block

// staging bytes a run needs at a stage (largest over its layers)
template <typename R>
int run_stage_bytes(const mrm_gpu* r, int stage, int rows) {
  int need = 0;
  for (int l = 0; l < r->nl; ++l) {
    const LayerBufs& b = r->L[l];
    const bool ucol = b.ucol && l > 0, lcol = b.lcol && l + 1 < r->nl;
    const RowStage p = row_stage_plan<R>(stage, fnx(r), rows, b.xst != nullptr, ucol, lcol, b.thermal != 0);
    need = std::max(need, p.bytes);
  }
  return need;
}

// Packing of short rows: an FP32 run (register row transforms, no window,
// head, field table or grain map) whose rows are shorter than the batch's
// longest takes 2^k times the shape's rows per task, as many as the FFT
// buffers sized for the longest rows hold, with at most as many grains per
// task as the longest rows' tasks: its blocks then carry about as many points
// as those of the longest rows instead of idling most of their threads.
struct RowPackCap {
  int fft = 0;     // FFT-buffer bytes of the launch (twiddles + two buffers)
  int grains = 0;  // grains of the largest unpacked task
};

template <typename R>
RowPackCap row_pack_cap(const Engine* e, int rpb) {
  RowPackCap c;
  for (auto* r : e->runs) {
    // a batch on the level-2 kernels (LLB / MT / Zhang, temperature profiles
    // or scaling) packs nothing: those kernels keep RPB rows per task
    for (int l = 0; l < r->nl; ++l)
      if (r->L[l].llb || r->L[l].tprof || r->L[l].tsc) return RowPackCap{};
    c.fft = std::max(c.fft, row_fft_smem<R>(r->lgpx, rpb));
    c.grains = std::max(c.grains, rows_per_task(r, rpb) * fnx(r));
  }
  return c;
}

bool row_packable(const mrm_gpu* r) {
  if (r->g.precision != MRM_FP32 || r->wnx || !rrow_len_ok(r->lgpx - 1)) return false;
  for (int l = 0; l < r->nl; ++l)
    if (r->L[l].tab || r->L[l].func == kFuncHead || r->L[l].cgrain) return false;
  return true;
}

template <typename R>
int rows_per_task(const mrm_gpu* r, int rpb, const RowPackCap& c) {
  int rows = rows_per_task(r, rpb);
  if (!row_packable(r)) return rows;
  while (2 * rows <= fny(r) && row_fft_smem<R>(r->lgpx, 2 * rows) <= c.fft && 2 * rows * fnx(r) <= c.grains)
    rows *= 2;
  return rows;
}

// row-kernel shared memory before the staging area: twiddles, FFT buffers and,
// for a run with a layer under the write head, the head-field table (with a
// tabulated field profile, its interpolation weights)
template <typename R>
size_t row_fixed_smem(const mrm_gpu* r, int rpb) {
  size_t b = (size_t)row_fft_smem<R>(r->lgpx, rpb), t = 0;
  for (int l = 0; l < r->nl; ++l) {
    if (r->L[l].tab) t = std::max(t, (size_t)field_table_bytes(fnx(r)));
    else if (r->L[l].func == kFuncHead) t = std::max(t, (size_t)head_table_bytes<R>(fnx(r)));
  }
  return b + t;
}

// Column-kernel shared memory for tasks of nc columns (a power of two).  The
// task's packed tensor slice is staged too where that keeps as many blocks per
// SM resident as without it (up to minb; minb = 0: never staged).
template <typename R>
size_t col_smem_of(const mrm_gpu* r, int nc, int minb) {
  const size_t b = col_fft_smem<R>(r->lgpy, ilog2(nc), r->nl * 3);
  if (sizeof(R) != sizeof(float) || minb <= 0) return b;
  const int reals = nc * r->nl * r->nl * 9 * tens_row_stride(r->py);
  if (!tens_slice_fits<R>(reals)) return b;
  const size_t with = b + (size_t)reals * sizeof(R);
  auto resident = [](size_t bytes) { return (int)(kSmemPerSM / (bytes + kSmemReserved)); };
  return resident(with) >= std::min(minb, resident(b)) ? with : b;
}

// The geometry must run with the most economical shapes (one row per row
// task, one column per column task, no staging).
// big (optional): set instead of failing when the grid's own FFT exceeds the
// path's limits (a handle that computes demag through a moving window only)
int validate_geom(const mrm_geom* g, std::string* errp, bool* big = nullptr) {
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
  if (g->boundary == MRM_PERIODIC && (!is_pow2(g->nx) || !is_pow2(g->ny)))
    return set_err(errp, MRM_ERR_UNSUPPORTED,
                   "periodic demag needs power-of-two nx, ny on this path (got %d x %d)", g->nx, g->ny);
  int px, py;
  fft_grid(*g, &px, &py);
  if (big) *big = false;
  if ((px > kTwN || py > kTwN) && big && px >= 4 && py >= 2) {
    *big = true;
    return MRM_OK;
  }
  if (px > kTwN || py > kTwN || px < 4 || py < 2)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "FFT grid %d x %d outside 4..%d", px, py, kTwN);
  mrm_gpu tmp;
  tmp.g = *g;
  tmp.px = px;
  tmp.py = py;
  tmp.lgpx = ilog2(px);
  tmp.lgpy = ilog2(py);
  tmp.nl = g->n_lay;
  const bool f64 = g->precision == MRM_FP64;
  const size_t rs = (f64 ? (size_t)row_fft_smem<double>(tmp.lgpx, 1) : (size_t)row_fft_smem<float>(tmp.lgpx, 1)) +
                    (size_t)(f64 ? head_table_bytes<double>(g->nx) : head_table_bytes<float>(g->nx));
  const size_t cs = f64 ? col_smem_of<double>(&tmp, 1, 0)
                       : creg_run(&tmp) ? (size_t)creg_smem(col_tw_count(tmp.lgpy), kCreg[1].block,
                                                            creg_stage_bytes(spec_col_stride(g->ny), 3))
                                        : col_smem_of<float>(&tmp, 1, 0);
  if (rs + row_static_bytes(3) > kMaxSmem || cs + 64 > kMaxSmem)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "FFT grid %d x %d x %d layers exceeds shared memory", px,
                   py, g->n_lay);
  return MRM_OK;
}

// ---------------- descriptors ----------------
template <typename R>
RunDev<R> make_desc(const mrm_gpu* r) {
  RunDev<R> d;
  std::memset(&d, 0, sizeof(d));
  d.nx = fnx(r);
  d.ny = fny(r);
  d.gnx = r->wnx ? r->g.nx : 0;
  d.gny = r->wnx ? r->g.ny : 0;
  d.wi0 = std::max(0, r->wi0);
  d.wj0 = std::max(0, r->wj0);
  d.frz = r->wnx ? r->frz : -1;
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
  d.step_begin = r->step_begin;
  d.seed = r->seed;
  d.active = r->active ? 1 : 0;
  d.row_task0 = r->row_task0;
  d.nrow_tasks = r->nrow_tasks;
  d.phs = spec_row_stride(r->px);
  d.nys = spec_col_stride(fny(r));
  d.lgct = r->lgct;
  d.pyhs = tens_row_stride(r->py);
  d.tw_row = row_tw_off(r->lgpx);
  d.tw_col = col_tw_off(r->lgpy);
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
    o.cax = static_cast<const V4<R>*>(b.cax);
    o.cgrain = b.cgrain;
    o.gci = b.gci;
    o.gcs = b.gcs;
    o.hdm = static_cast<V4<R>*>(b.hdm);
    o.hapm = static_cast<V4<R>*>(b.hapm);
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
    o.hd_gap = b.hd_gap;
    o.hd_z = b.hd_z;
    o.hd_hg = b.hd_hg;
    o.hd_v = b.hd_v;
    o.hd_x0 = b.hd_x0;
    o.hd_t0 = b.hd_t0;
    o.hd_tbit = b.hd_tbit;
    o.hd_dx = r->g.dx;
    o.hd_bits = b.hd_bits;
    o.hd_nbits = b.hd_nbits;
    o.tab = static_cast<const TabDev*>(b.tab);
    o.llb = static_cast<const LlbDev*>(b.llb);
    o.tprof = static_cast<const TempDev*>(b.tprof);
    o.tsc = static_cast<const TscDev*>(b.tsc);
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
  CK(cudaStreamSynchronize(e->st));  // the host buffer is released on return
  e->desc_dirty = false;
  return MRM_OK;
}

// Shared memory of every row stage and of the column kernel for the engine's
// current shapes: FFT part for the largest grid, plus grain staging up to what
// keeps the shape's intended blocks per SM resident.
template <typename R>
int plan_smem(Engine* e) {
  std::string* errp = &e->err;
  const RowVariant rv = row_variant<R>(e->rowv);
  size_t fft = 16;
  int need[kSlots] = {0, 0, 0, 0, 0, 0};
  size_t scol = 16;
  int tw_cap = 0, stage_bytes = 0;
  const RowPackCap pack = row_pack_cap<R>(e, rv.rpb);
  for (auto* r : e->runs) {
    if (r->lgpx > rv.lgmax)
      return set_err(errp, MRM_ERR_UNSUPPORTED, "row shape %d does not cover %d-column FFT grids", e->rowv, r->px);
    const int rows = rows_per_task<R>(r, rv.rpb, pack);
    fft = std::max(fft, row_fixed_smem<R>(r, rv.rpb));
    for (int q = 0; q < kSlots; ++q) need[q] = std::max(need[q], run_stage_bytes<R>(r, kSlotStage[q], rows));
    if (r->demag && r->tensor_ready) {
      if (creg_run(r)) {
        tw_cap = std::max(tw_cap, col_tw_count(r->lgpy));
        stage_bytes = std::max(stage_bytes, creg_stage_bytes(spec_col_stride(fny(r)), r->lgct));
      } else scol = std::max(scol, col_smem_of<R>(r, cols_per_task(e, r), col_variant<R>(e->colv).minb));
    }
  }
  for (int q = 0; q < kSlots; ++q) {
    const long long per_block = (long long)(kSmemPerSM / rv.minb) - (long long)kSmemReserved -
                                (long long)row_static_bytes(q) - (long long)fft;
    const long long hard = (long long)kMaxSmem - (long long)row_static_bytes(q) - (long long)fft;
    if (hard < 0) return set_err(errp, MRM_ERR_UNSUPPORTED, "row shape %d exceeds shared memory", e->rowv);
    const long long cap = std::min<long long>(need[q], std::max(0LL, std::min(per_block, hard)));
    e->stage_cap[q] = (int)(cap & ~15LL);
    e->smem_row[q] = fft + (size_t)e->stage_cap[q];
  }
  if (scol + 64 > kMaxSmem) return set_err(errp, MRM_ERR_UNSUPPORTED, "column shape exceeds shared memory");
  e->smem_col = scol;
  const size_t screg = tw_cap ? (size_t)creg_smem(tw_cap, kCreg[creg_v(e)].block, stage_bytes) : 16;
  if (screg + 64 > kMaxSmem) return set_err(errp, MRM_ERR_UNSUPPORTED, "column shape exceeds shared memory");
  e->smem_creg = screg;
  e->creg_tw_cap = tw_cap;
  CK(row_allow_smem<R>(e->rowv, e->smem_row));
  // the reductions launches (kPred of the single-stage integrator, kCorr):
  // row shape 0, one row per task
  {
    const RowVariant r0 = row_variant<R>(0);
    size_t f0 = 16;
    int n0[2] = {0, 0};
    for (auto* r : e->runs) {
      f0 = std::max(f0, row_fixed_smem<R>(r, 1));
      n0[0] = std::max(n0[0], run_stage_bytes<R>(r, kPred, 1));
      n0[1] = std::max(n0[1], run_stage_bytes<R>(r, kCorr, 1));
    }
    const long long stat = (long long)row_static_bytes(3);
    const long long per_block = (long long)(kSmemPerSM / r0.minb) - (long long)kSmemReserved - stat - (long long)f0;
    const long long hard = (long long)kMaxSmem - stat - (long long)f0;
    if (hard < 0) return set_err(errp, MRM_ERR_UNSUPPORTED, "grid exceeds shared memory");
    for (int i = 0; i < 2; ++i) {
      e->cap_stats[i] = (int)(std::min<long long>(n0[i], std::max(0LL, std::min(per_block, hard))) & ~15LL);
      e->smem_stats[i] = f0 + (size_t)e->cap_stats[i];
    }
    size_t lim[kSlots] = {0, 0, 0, e->smem_stats[1], 0, e->smem_stats[0]};
    CK(row_allow_smem<R>(0, lim));
  }
  CK(col_allow_smem<R>(e->colv, e->smem_col));
  e->creg_blocks = 0;
  if (sizeof(R) == sizeof(float) && e->creg_tw_cap) {
    CK(creg_allow_smem(creg_v(e), e->smem_creg));
    // persistent blocks: as many as stay resident
    int per_sm = 0, sms = 0;
    CK(creg_occupancy(creg_v(e), e->smem_creg, &per_sm));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->dev));
    e->creg_blocks = std::max(1, per_sm) * sms;
  }
  return MRM_OK;
}

template <typename R>
int build_tables(Engine* e) {
  std::string* errp = &e->err;
  const RowVariant rv = row_variant<R>(e->rowv);
  const RowPackCap pack = row_pack_cap<R>(e, rv.rpb);
  std::vector<Task> rt, ct, ct2, stt;
  for (size_t i = 0; i < e->runs.size(); ++i) {
    mrm_gpu* r = e->runs[i];
    r->slot = (int)i;
    const int rpt = rows_per_task<R>(r, rv.rpb, pack);
    const int ny = fny(r);
    for (int l = 0; l < r->nl; ++l)
      for (int j = 0; j < ny; j += rpt) rt.push_back(make_int4((int)i, l, j, std::min(rpt, ny - j)));
    // one-row tasks of the reductions launch; the run's partial records
    r->row_task0 = (int)stt.size();
    for (int l = 0; l < r->nl; ++l)
      for (int j = 0; j < ny; ++j) stt.push_back(make_int4((int)i, l, j, 1));
    r->nrow_tasks = (int)stt.size() - r->row_task0;
    if (r->demag && r->tensor_ready) {
      const int ph = r->px / 2 + 1;
      if (creg_run(r)) {
        // a task per block of the register column kernel: block / (py/8) columns
        const int cpt = creg_cols(r->lgpy, kCreg[creg_v(e)].block);
        r->lgct = ilog2(col_tile(cpt));
        for (int k = 0; k < ph; k += cpt) ct2.push_back(make_int4((int)i, k, std::min(cpt, ph - k), 0));
      } else {
        const int cpt = cols_per_task(e, r);
        r->lgct = ilog2(cpt);
        for (int k = 0; k < ph; k += cpt) ct.push_back(make_int4((int)i, k, std::min(cpt, ph - k), 0));
      }
    }
  }
  e->nrt = (int)rt.size();
  e->nct = (int)ct.size();
  e->nct2 = (int)ct2.size();
  e->has_head = false;
  e->has_cubic = false;
  e->has_llb = false;
  e->has_tprof = false;
  e->mapped = false;
  bool karlqvist_head = false;
  for (auto* r : e->runs)
    for (int l = 0; l < r->nl; ++l) {
      karlqvist_head = karlqvist_head || r->L[l].func == kFuncHead;
      e->has_head = e->has_head || r->L[l].func == kFuncHead || r->L[l].tab != nullptr;
      e->has_cubic = e->has_cubic || r->L[l].cax != nullptr;
      e->has_llb = e->has_llb || r->L[l].llb != nullptr;
      e->has_tprof = e->has_tprof || r->L[l].tprof != nullptr || r->L[l].tsc != nullptr;
      e->mapped = e->mapped || r->L[l].cgrain != nullptr;
    }
  if (e->mapped && karlqvist_head)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "the write head needs one grain per cell (no grain maps in the batch)");
  e->has_window = false;
  for (auto* r : e->runs) e->has_window = e->has_window || r->wnx > 0;
  if (e->has_window && (e->runs.size() > 1 || e->mapped))
    return set_err(errp, MRM_ERR_UNSUPPORTED,
                   "a moving demag window runs on a handle of its own with one grain per cell");
  e->nst = (int)stt.size();
  if (e->nst > e->st_cap) {
    dfree(e->d_stasks);
    e->st_cap = std::max(e->nst, 2 * e->st_cap);
    int rc = dmalloc(errp, (void**)&e->d_stasks, sizeof(Task) * e->st_cap);
    if (rc) return rc;
  }
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
  if (e->nct2 > e->ct2_cap) {
    dfree(e->d_ctasks2);
    e->ct2_cap = std::max(e->nct2, 2 * e->ct2_cap);
    int rc = dmalloc(errp, (void**)&e->d_ctasks2, sizeof(Task) * e->ct2_cap);
    if (rc) return rc;
  }
  // the row tasks' records, then kMaxLayers frozen-grain records per run
  const int nr = (int)e->runs.size();
  const int npart = e->nst + nr * kMaxLayers;
  for (int i = 0; i < nr; ++i) e->runs[i]->frz = e->nst + i * kMaxLayers;
  if (npart > e->part_cap) {
    dfree(e->d_part);
    e->part_cap = std::max(npart, 2 * e->part_cap);
    int rc = dmalloc(errp, (void**)&e->d_part, sizeof(double) * kNPart * e->part_cap);
    if (rc) return rc;
  }
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
  if (e->nct2) CK(cudaMemcpyAsync(e->d_ctasks2, ct2.data(), sizeof(Task) * e->nct2, cudaMemcpyHostToDevice, e->st));
  if (e->nst) CK(cudaMemcpyAsync(e->d_stasks, stt.data(), sizeof(Task) * e->nst, cudaMemcpyHostToDevice, e->st));
  CK(cudaStreamSynchronize(e->st));  // the host vectors are released on return
  int rc = plan_smem<R>(e);
  if (rc) return rc;
  clear_graphs(e);
  e->nslots = nr;
  e->tables_dirty = false;
  e->desc_dirty = true;
  return MRM_OK;
}

template <typename R>
cudaError_t launch_row_e(Engine* e, int stage, bool stats, int istep, int flags, bool pdl = true) {
  if (!e->nrt) return cudaSuccess;
  // the general kernels for the semi-implicit pushes and write heads
  const int gen = (e->has_llb || e->has_tprof) ? 2 : ((flags & kFlagBoris) || e->has_head || e->has_cubic || e->has_window);
  if (stats) {
    const int i = stage == kPred ? 0 : 1;
    RowLaunch a{e->st, e->d_runs, e->d_stasks, e->d_tw, e->d_part, e->d_err, e->nst, e->smem_stats[i],
                e->cap_stats[i], pdl, gen};
    return launch_row<R>(0, stage, true, a, istep, flags);
  }
  const int q = row_slot(stage, false);
  RowLaunch a{e->st, e->d_runs, e->d_rtasks, e->d_tw, e->d_part, e->d_err, e->nrt, e->smem_row[q],
              e->stage_cap[q], pdl, gen};
  return launch_row<R>(e->rowv, stage, false, a, istep, flags);
}

// the column step: the in-place column kernel over its runs' tasks, then the
// register column kernel over its runs' tasks (either may be absent)
template <typename R>
cudaError_t launch_col_e(Engine* e, int istep, int flags, bool pdl = true) {
  if (e->nct) {
    ColLaunch a{e->st, e->d_runs, e->d_ctasks, e->d_tw, e->d_err, e->nct, e->smem_col, pdl};
    cudaError_t ce = launch_col<R>(e->colv, a, istep, flags);
    if (ce != cudaSuccess) return ce;
  }
  if (e->nct2) {
    ColLaunch a{e->st, e->d_runs, e->d_ctasks2, e->d_tw, e->d_err, e->nct2, e->smem_creg, pdl};
    a.blocks = e->creg_blocks;
    a.tw_cap = e->creg_tw_cap;
    return launch_creg(creg_v(e), a, istep, flags);
  }
  return cudaSuccess;
}

// llg_type -3 (Heun) and -2 (semi-implicit midpoint): two field evaluations
// per step; llg_type 2 (semi-implicit): one, then the commit of the new state
template <typename R>
cudaError_t enqueue_steps(Engine* e, int k, bool stats, int llg_type, bool stored = false) {
  cudaError_t ce = cudaSuccess;
  auto acc = [&](cudaError_t x) { if (ce == cudaSuccess) ce = x; };
  // semi-implicit (2 / -2) and analytic-rotation (1 / -1) pushes: one push
  // over dt (then the commit), or the midpoint form (dt/2, then dt from m_n)
  const int f0 = (llg_type == 2 || llg_type == 1)     ? kFlagBoris | (llg_type == 1 ? kFlagRot : 0)
                 : (llg_type == -2 || llg_type == -1) ? (kFlagBoris | kFlagMid | (llg_type == -1 ? kFlagRot : 0))
                                                      : 0;
  // grains of several cells: each stage's demag comes from an evaluation stage
  // (inverse row transforms of every cell) averaged over the grains' cells
  const int f = f0 | (e->mapped ? kFlagMapped : 0);
  const int nr = (int)e->runs.size();
  auto mapped_demag = [&](int i, bool corr) {
    if (!e->mapped) return;
    acc(launch_row_e<R>(e, kEval, false, i, f0 | kFlagDemagOnly));
    int maxc = 1;
    for (auto* r : e->runs) maxc = std::max(maxc, r->g.nx * r->g.ny);
    acc(launch_kernel(gather_demag_kernel<R>, dim3((maxc + 255) / 256, nr * kMaxLayers), dim3(256), 0, e->st, false,
                      static_cast<const RunDev<R>*>(e->d_runs), nr, i, f0 | (corr ? kFlagCorrTime : 0)));
  };
  for (int i = 0; i < k; ++i) {
    const bool last = stats && i == k - 1;
    const int lf = last ? (kFlagStats | kFlagStoreField) : 0;
    if (llg_type == 2 || llg_type == 1) {
      mapped_demag(i, false);
      acc(launch_row_e<R>(e, kPred, last, i, f | lf));
      acc(launch_col_e<R>(e, i, 0));
      acc(launch_kernel(commit_kernel<R>, dim3(e->nst), dim3(256), 0, e->st, true,
                        static_cast<const RunDev<R>*>(e->d_runs), (const Task*)e->d_stasks, i, 0));
      continue;
    }
    mapped_demag(i, false);
    acc(launch_row_e<R>(e, kPred, false, i, f | ((stored && i == 0) ? kFlagStoredField : 0)));
    acc(launch_col_e<R>(e, i, 0));
    mapped_demag(i, true);
    acc(launch_row_e<R>(e, kCorr, last, i, f | lf));
    acc(launch_col_e<R>(e, i, 0));
  }
  acc(launch_kernel(advance_kernel<R>, dim3((nr + 127) / 128), dim3(128), 0, e->st, true,
                    static_cast<RunDev<R>*>(e->d_runs), nr, k));
  if (stats)
    acc(launch_kernel(finalize_stats_kernel<R>, dim3(nr), dim3(256), 0, e->st, true,
                      static_cast<const RunDev<R>*>(e->d_runs), (const Task*)e->d_stasks,
                      (const double*)e->d_part, e->d_stats, nr));
  return ce;
}

// spectrum = H^(m) for active runs whose state or tensor changed
template <typename R>
int establish_spectra(Engine* e) {
  std::string* errp = &e->err;
  bool need = false;
  for (auto* r : e->runs)
    if (r->active && !r->spec_valid) need = true;
  if (!need) return MRM_OK;
  CK(launch_row_e<R>(e, kInit, false, 0, kFlagForce));
  CK(launch_col_e<R>(e, 0, kFlagForce));
  CK(cudaGetLastError());
  for (auto* r : e->runs)
    if (r->active) r->spec_valid = true;
  return MRM_OK;
}

// ---------------- shapes: default heuristic and autotuner ----------------
template <typename R>
void default_shapes(Engine* e) {
  int maxnx = 1, maxlg = 1;
  for (auto* r : e->runs) {
    maxnx = std::max(maxnx, fnx(r));
    maxlg = std::max(maxlg, r->lgpx);
  }
  // rows per block so that a block holds about 256 grains
  const int want = std::max(1, 256 / maxnx);
  int best = 0;
  for (int v = 0; v < row_variant_count<R>(); ++v) {
    const RowVariant rv = row_variant<R>(v);
    if (rv.lgmax < maxlg || rv.block != 256) continue;
    const RowVariant bv = row_variant<R>(best);
    if (std::abs(rv.rpb - want) < std::abs(bv.rpb - want)) best = v;
  }
  e->rowv = best;
  e->colv = 0;
  e->cpt = 0;
}

// signature of a batch for the tuner's cache: precision, largest grid, layers,
// order of magnitude of the grain count
std::string shape_key(const Engine* e) {
  int lgx = 0, lgy = 0, nl = 0;
  long long grains = 0;
  for (auto* r : e->runs) {
    if (!r->active) continue;
    lgx = std::max(lgx, r->lgpx);
    lgy = std::max(lgy, r->lgpy);
    nl = std::max(nl, r->nl);
    grains += (long long)r->g.nx * r->g.ny * r->nl;
  }
  char buf[96];
  std::snprintf(buf, sizeof buf, "%d/%d/%d/%d/%d/%d", e->dev, e->prec, lgx, lgy, nl, grains > 0 ? ilog2((int)std::min<long long>(grains, 1LL << 30)) : 0);
  return buf;
}

struct Shape {
  int rowv, colv, cpt;
};
std::mutex g_tune_mu;
std::map<std::string, Shape>& tune_cache() {
  static std::map<std::string, Shape> c;
  return c;
}

// Times each column shape x columns per task, then each row shape, on the
// batch itself (one Heun step's chained launches, as the captured steps run
// them) and keeps the fastest.  The
// kernels run on the real state, which is saved before and restored after
// (m and the stored field per layer; the spectra are re-established).
template <typename R>
int autotune(Engine* e) {
  std::string* errp = &e->err;
  const std::string key = shape_key(e);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = tune_cache().find(key);
    if (it != tune_cache().end()) {
      e->rowv = it->second.rowv;
      e->colv = it->second.colv;
      e->cpt = it->second.cpt;
      return MRM_OK;
    }
  }
  default_shapes<R>(e);
  bool any = false;
  for (auto* r : e->runs) any = any || r->active;
  if (!any) return MRM_OK;
  // save the state
  std::vector<std::pair<void*, void*>> saved;  // (device buffer, copy)
  for (auto* r : e->runs)
    for (int l = 0; l < r->nl; ++l)
      for (void* p : {r->L[l].m, r->L[l].hf}) {
        void* c = nullptr;
        const size_t bytes = (size_t)r->L[l].n * sizeof(V4<R>);
        int rc = dmalloc(errp, &c, bytes);
        if (rc) return rc;
        CK(cudaMemcpyAsync(c, p, bytes, cudaMemcpyDeviceToDevice, e->st));
        saved.push_back({p, c});
      }
  cudaEvent_t ev[2];
  CK(cudaEventCreate(&ev[0]));
  CK(cudaEventCreate(&ev[1]));
  auto time_it = [&](auto&& body, int reps, float* ms) -> int {
    for (int w = 0; w < 2; ++w) CK(body());
    CK(cudaEventRecord(ev[0], e->st));
    for (int s = 0; s < reps; ++s) CK(body());
    CK(cudaEventRecord(ev[1], e->st));
    CK(cudaEventSynchronize(ev[1]));
    CK(cudaEventElapsedTime(ms, ev[0], ev[1]));
    return MRM_OK;
  };
  auto prepare = [&]() -> int {
    int rc = build_tables<R>(e);
    if (rc) return rc;
    rc = push_descs(e);
    if (rc) return rc;
    for (auto* r : e->runs) r->spec_valid = false;
    return establish_spectra<R>(e);
  };
  const int reps = 6;
  // one Heun step's four launches, chained as in the captured steps (the
  // shapes interact through the overlap of a kernel's tail with the next
  // kernel's start)
  auto heun_step = [&]() -> cudaError_t {
    cudaError_t a = launch_row_e<R>(e, kPred, false, 0, kFlagForce, true);
    cudaError_t b = launch_col_e<R>(e, 0, kFlagForce, true);
    cudaError_t c = launch_row_e<R>(e, kCorr, false, 0, kFlagForce, true);
    cudaError_t d = launch_col_e<R>(e, 0, kFlagForce, true);
    return a != cudaSuccess ? a : b != cudaSuccess ? b : c != cudaSuccess ? c : d;
  };
  // column shapes with the default row shape
  Shape best = {e->rowv, e->colv, e->cpt};
  float best_ms = 1e30f;
  // columns per task only matter for the in-place column kernel's runs
  bool any_inplace = false;
  for (auto* r : e->runs) any_inplace = any_inplace || (r->demag && r->tensor_ready && !creg_run(r));
  for (int cv = 0; cv < col_variant_count<R>(); ++cv)
    for (int nc : {1, 2, 4, 8}) {
      if (!any_inplace && nc > 1) continue;
      e->colv = cv;
      e->cpt = nc;
      e->err.clear();
      if (prepare() != MRM_OK) continue;
      float ms = 0;
      int rc = time_it(heun_step, reps, &ms);
      if (rc) return rc;
      if (ms < best_ms) {
        best_ms = ms;
        best.colv = cv;
        best.cpt = nc;
      }
    }
  e->colv = best.colv;
  e->cpt = best.cpt;
  // row shapes with the chosen column shape
  best_ms = 1e30f;
  for (int v = 0; v < row_variant_count<R>(); ++v) {
    e->rowv = v;
    e->err.clear();
    if (prepare() != MRM_OK) continue;
    float ms = 0;
    int rc = time_it(heun_step, reps, &ms);
    if (rc) return rc;
    if (ms < best_ms) {
      best_ms = ms;
      best.rowv = v;
    }
  }
  e->rowv = best.rowv;
  e->err.clear();
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  // restore the state
  for (auto& s : saved) {
    for (auto* r : e->runs)
      for (int l = 0; l < r->nl; ++l)
        if (s.first == r->L[l].m || s.first == r->L[l].hf)
          CK(cudaMemcpyAsync(s.first, s.second, (size_t)r->L[l].n * sizeof(V4<R>), cudaMemcpyDeviceToDevice, e->st));
  }
  CK(cudaStreamSynchronize(e->st));
  for (auto& s : saved) dfree(s.second);
  for (auto* r : e->runs) r->spec_valid = false;
  e->tables_dirty = true;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  tune_cache()[key] = best;
  return MRM_OK;
}

template <typename R>
int ensure_ready(Engine* e) {
  std::string* errp = &e->err;
  CK(cudaSetDevice(e->dev));
  if (e->tables_dirty) {
    if (e->shape_forced) {
      e->rowv = e->force_rowv;
      e->colv = e->force_colv;
      e->cpt = e->force_cpt;
    } else if (e->autotune) {
      // tuning needs every active run uploaded with its tensor
      bool ready = true;
      for (auto* r : e->runs)
        if (r->active && r->demag && !r->tensor_ready) ready = false;
      int rc = ready ? autotune<R>(e) : MRM_OK;
      if (!ready) default_shapes<R>(e);
      if (rc) return rc;
    } else {
      default_shapes<R>(e);
    }
    int rc = build_tables<R>(e);
    if (rc) return rc;
  }
  if (e->desc_dirty) {
    int rc = push_descs(e);
    if (rc) return rc;
  }
  return establish_spectra<R>(e);
}

template <typename R>
int run_steps(Engine* e, int nsteps, int llg_type) {
  std::string* errp = &e->err;
  // llgp%llb is one switch for all layers (push_m, llg.f90:1218); this path has
  // its Heun branch, and its formulas divide by the temperature
  for (auto* r : e->runs) {
    int nllb = 0;
    for (int l = 0; l < r->nl; ++l) nllb += r->L[l].llb != nullptr;
    if (!nllb) continue;
    if (nllb != r->nl) return set_err(errp, MRM_ERR_UNSUPPORTED, "LLB on some layers of a run but not all");
    if (llg_type != -3 && llg_type != 2 && llg_type != -2)
      return set_err(errp, MRM_ERR_UNSUPPORTED, "LLB runs with llg_type -3, 2 or -2 on this path");
    // update_do_grain refreshes the other buffer of m but not of |m|
    // (data.f90:139): a frozen grain's |m| would depend on its history
    if (r->wnx) return set_err(errp, MRM_ERR_UNSUPPORTED, "LLB with a moving demag window");
    for (int l = 0; l < r->nl; ++l)
      if (!((r->L[l].tprof ? r->L[l].tp.bg : r->L[l].temperature) > 0))
        return set_err(errp, MRM_ERR_ARG, "LLB needs a temperature > 0 (layer %d)", l);
  }
  int rc = ensure_ready<R>(e);
  if (rc) return rc;
  int left = nsteps;
  while (left > 0) {
    const int k = std::min(left, kGraphSteps);
    const bool stats = (left == k);  // reductions only on the call's last step
    const bool stored = e->pred_stored && left == nsteps;
    auto key = std::make_pair(k, (stats ? 1 : 0) + 2 * (llg_type + 3) + (stored ? 64 : 0));
    auto it = e->graphs.find(key);
    if (it == e->graphs.end()) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
      cudaError_t le = enqueue_steps<R>(e, k, stats, llg_type, stored);
      cudaError_t ce = cudaStreamEndCapture(e->st, &g);
      if (le != cudaSuccess) return set_err(errp, MRM_ERR_CUDA, "launch in capture: %s", cudaGetErrorString(le));
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
  e->pred_stored = false;
  CK(cudaGetLastError());
  // mirror the device-side step counters
  for (auto* r : e->runs) {
    if (!r->active) continue;
    long long rem = std::max(0LL, r->step_end - r->step);
    r->step += std::min<long long>(rem, nsteps);
  }
  return MRM_OK;
}

int engine_step(Engine* e, int nsteps, int llg_type) {
  if (e->prec == MRM_FP64) return run_steps<double>(e, nsteps, llg_type);
  return run_steps<float>(e, nsteps, llg_type);
}

bool llg_type_ok(int t) { return t == -3 || t == -2 || t == 2 || t == 1 || t == -1; }

template <typename R>
int engine_eval(Engine* e) {
  std::string* errp = &e->err;
  int rc = ensure_ready<R>(e);
  if (rc) return rc;
  if (e->mapped) {
    // grains of several cells: demag per cell, its grain average, then the field
    const int nr = (int)e->runs.size();
    int maxc = 1;
    for (auto* r : e->runs) maxc = std::max(maxc, r->g.nx * r->g.ny);
    CK(launch_row_e<R>(e, kEval, false, 0, kFlagForce | kFlagDemagOnly));
    CK(launch_kernel(gather_demag_kernel<R>, dim3((maxc + 255) / 256, nr * kMaxLayers), dim3(256), 0, e->st, false,
                     static_cast<const RunDev<R>*>(e->d_runs), nr, 0, 0));
    CK(launch_row_e<R>(e, kEval, false, 0, kFlagForce | kFlagStoreField | kFlagMapped));
  } else {
    CK(launch_row_e<R>(e, kEval, false, 0, kFlagForce | kFlagStoreField));
  }
  CK(cudaGetLastError());
  return MRM_OK;
}

// device-side error flag (bulk-copy waits that ran out, shapes not compiled):
// read and cleared at the host's synchronisation points
int check_device_error(Engine* e) {
  std::string* errp = &e->err;
  int v[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(v, e->d_err, sizeof(v), cudaMemcpyDeviceToHost, e->st));
  CK(cudaStreamSynchronize(e->st));
  if (v[0] == 0) return MRM_OK;
  CK(cudaMemsetAsync(e->d_err, 0, sizeof(v), e->st));
  const long long val = (long long)(unsigned)v[2] | ((long long)v[3] << 32);
  return set_err(errp, MRM_ERR_DEVICE, "device error flag 0x%x (%s; check %d, value %lld)", v[0],
                 (v[0] & kErrBarrierTimeout) ? "a bulk-copy wait ran out"
                 : (v[0] & kErrShape)        ? "kernel shape mismatch"
                                             : "self-check failed",
                 v[1], val);
}

// ---------------- state transfers ----------------
// (x, y, z) doubles of the host layout <-> the float4 / double4 grain records
// (map layers: every cell takes its grain's value, empty cells zero; a grain
// is read at its first cell)
template <typename R>
__global__ void state_in_kernel(const double* __restrict__ in, V4<R>* __restrict__ m, V4<R>* __restrict__ mp, int n,
                                const int* __restrict__ cgrain) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int g = cgrain ? cgrain[i] : i;
  // (w: |m| = 1, the magnitude the LLB integrator starts from, data.f90:202)
  const V4<R> v = g >= 0 ? V4<R>{(R)in[3 * g], (R)in[3 * g + 1], (R)in[3 * g + 2], (R)1} : V4<R>{0, 0, 0, 0};
  m[i] = v;
  mp[i] = v;
}
template <typename R>
__global__ void state_out_kernel(const V4<R>* __restrict__ src, double* __restrict__ out, int n,
                                 const int* __restrict__ gci, const int* __restrict__ gcs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const V4<R> v = src[gci ? gcs[gci[i]] : i];
  out[3 * i] = (double)v.x;
  out[3 * i + 1] = (double)v.y;
  out[3 * i + 2] = (double)v.z;
}

// the LLB magnitude |m| (w lane of m): per grain in, per grain out
template <typename R>
__global__ void mag_in_kernel(const double* __restrict__ in, V4<R>* __restrict__ m, V4<R>* __restrict__ mp, int n,
                              const int* __restrict__ cgrain) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int g = cgrain ? cgrain[i] : i;
  if (g < 0) return;
  m[i].w = (R)in[g];
  mp[i].w = (R)in[g];
}
template <typename R>
__global__ void mag_out_kernel(const V4<R>* __restrict__ src, double* __restrict__ out, int n,
                               const int* __restrict__ gci, const int* __restrict__ gcs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = (double)src[gci ? gcs[gci[i]] : i].w;
}

// ---------------- adaptive time step ----------------
// max over a layer's grains of |h + hthm * dti|^2 (get_fields, llg.f90:375-382):
// h the stored field of the last evaluation, hthm = sigma sqrt(T) N(0,1)^3 the
// thermal draw of step `step` (the one the predictor takes); the maximum goes
// to *out as the bits of a non-negative double (ordered like the values)
template <typename R>
__global__ void hmag_kernel(const RunDev<R>* __restrict__ runs, int slot, int layer, double dti, long long step,
                            unsigned long long* __restrict__ out) {
  const RunDev<R>& rd = runs[slot];
  const LayerDev<R>& L = rd.L[layer];
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  double v2 = 0.0;
  if (n < L.n) {
    const int g = L.cgrain ? L.cgrain[n] : n;  // grains only, each on its cells
    const V4<R> h = g >= 0 ? L.hf[n] : V4<R>{0, 0, 0, 0};
    double x = h.x, y = h.y, z = h.z;
    if (L.thermal && g >= 0) {
      R gn[3];
      thermal_normals(rd.seed, (unsigned long long)layer, (unsigned long long)step, (unsigned long long)g, gn);
      const double s = (double)L.pb[n].w * sqrt(L.temperature) * dti;
      x += s * (double)gn[0];
      y += s * (double)gn[1];
      z += s * (double)gn[2];
    }
    v2 = x * x + y * y + z * z;
  }
  for (int o = 16; o > 0; o >>= 1) v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(v2));
}

// ---------------- off-plane field (off_field.f90) ----------------
// Ms ms_scale m per cell of every layer (get_mag, data.f90:322-390), FP64 planes [l*3 + a][ny][nx]
template <typename R>
__global__ void mgrid_kernel(const RunDev<R>* __restrict__ runs, int slot, double* __restrict__ out) {
  const RunDev<R>& rd = runs[slot];
  const int l = blockIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const LayerDev<R>& L = rd.L[l];
  const int n = L.n;  // cells of the grid
  if (c >= n) return;
  const V4<R> m = L.m[c];
  const double f = (double)L.pb[c].x;  // 0 on empty cells
  out[((size_t)l * 3 + 0) * n + c] = f * (double)m.x;
  out[((size_t)l * 3 + 1) * n + c] = f * (double)m.y;
  out[((size_t)l * 3 + 2) * n + c] = f * (double)m.z;
}
// H^_a = sum over source layers and components of N^[ks][3a + b] M^[ks][b] (off_field.f90:70-95)
__global__ void off_mac_kernel(const Cx<double>* __restrict__ T, const Cx<double>* __restrict__ X,
                               Cx<double>* __restrict__ H, int nl, long long hplane) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= hplane) return;
  for (int a = 0; a < 3; ++a) {
    Cx<double> h{0.0, 0.0};
    for (int ks = 0; ks < nl; ++ks)
      for (int b = 0; b < 3; ++b)
        h = cadd(h, cmul(T[((long long)ks * 9 + 3 * a + b) * hplane + q], X[((long long)ks * 3 + b) * hplane + q]));
    H[(long long)a * hplane + q] = h;
  }
}

// ---------------- run buffers ----------------
// spectra and tensor of the run's FFT grid
int spectra_alloc(mrm_gpu* r) {
  std::string* errp = &r->err;
  const size_t re = relem(r->g.precision);
  int rc = dmalloc(errp, &r->spech, (size_t)r->nl * 3 * fny(r) * spec_row_stride(r->px) * 2 * re);
  if (!rc) rc = dmalloc(errp, &r->specx, specx_count(r) * 2 * re);
  return rc;
}

// the run's own tensor buffer (tensor_bytes), replacing any shared one
int tensor_alloc(mrm_gpu* r) {
  std::string* errp = &r->err;
  void* p = nullptr;
  int rc = dmalloc(errp, &p, tensor_bytes(r));
  if (rc) return rc;
  r->tens_buf = std::shared_ptr<void>(p, CudaFreeDeleter());
  r->tens = p;
  return MRM_OK;
}
void tensor_release(mrm_gpu* r) {
  r->tens_buf.reset();
  r->tens = nullptr;
}

int run_alloc(mrm_gpu* r) {
  std::string* errp = &r->err;
  const size_t re = relem(r->g.precision);
  int rc = r->fft_big ? MRM_OK : spectra_alloc(r);
  if (rc) return rc;
  // (the tensor buffer comes with the first build or upload, or is shared)
  // The transfer buffer and every layer's per-grain arrays live in one
  // zero-filled allocation (256-byte aligned pieces): a run costs one
  // allocation and one free of them instead of one per array.
  const size_t n = (size_t)r->g.nx * r->g.ny;
  auto piece = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t v4 = piece(n * 4 * re), pv = piece(n * 4 * sizeof(double)), xf = piece(n * 3 * sizeof(double));
  rc = dmalloc(errp, &r->slab, xf + (size_t)r->nl * (8 * v4 + pv));
  if (rc) return rc;
  unsigned char* at = static_cast<unsigned char*>(r->slab);
  r->xfer = at;
  at += xf;
  for (int l = 0; l < r->nl; ++l) {
    LayerBufs& b = r->L[l];
    b.n = (int)n;
    b.ng = (int)n;
    void** v4s[] = {&b.m, &b.mp, &b.dm, &b.hf, &b.hd, &b.ht, &b.pa, &b.pb};
    for (void** p : v4s) {
      *p = at;
      at += v4;
    }
    b.pv = at;
    at += pv;
  }
  return MRM_OK;
}

void run_free(mrm_gpu* r) {
  dfree(r->spech);
  dfree(r->specx);
  dfree(r->slab);  // xfer and the per-grain arrays
  r->xfer = nullptr;
  tensor_release(r);
  for (int l = 0; l < MRM_MAX_LAYERS; ++l) {
    LayerBufs& b = r->L[l];
    b.m = b.mp = b.dm = b.hf = b.hd = b.ht = b.pa = b.pb = b.pv = nullptr;
    dfree(b.xidx); dfree(b.xnbr); dfree(b.xcoef);
    dfree(b.uidx); dfree(b.unbr); dfree(b.ucoef);
    dfree(b.lidx); dfree(b.lnbr); dfree(b.lcoef);
    dfree(b.xst); dfree(b.ucol); dfree(b.lcol); dfree(b.cax);
    dfree(b.cgrain); dfree(b.gci); dfree(b.gcs); dfree(b.hdm); dfree(b.hapm);
    dfree(b.tab); dfree(b.tb_v); dfree(b.tb_pos);
    dfree(b.llb); dfree(b.llbp); dfree(b.tprof);
    dfree(b.tsc); dfree(b.tsc_tc); dfree(b.tsc_tab);
  }
}

int64_t footprint(const mrm_geom& g) {
  int px, py;
  fft_grid(g, &px, &py);
  const size_t re = g.precision == MRM_FP64 ? 8 : 4;
  const int64_t n = (int64_t)g.nx * g.ny, nl = g.n_lay;
  const int64_t ph = px / 2 + 1;
  const int64_t ph8 = (ph + kMaxColTile - 1) / kMaxColTile * kMaxColTile;  // whole column tiles
  int64_t b = nl * 3 * g.ny * spec_row_stride(px) * 2 * re + nl * 3 * ph8 * spec_col_stride(g.ny) * 2 * re;
  b += g.precision == MRM_FP64 ? ph * nl * nl * 9 * py * 16 : ph * nl * nl * 9 * tens_row_stride(py) * 4;
  b += nl * n * (8 * 4 * re + 4 * 8);
  b += n * 3 * 8;  // host transfer buffer of one layer's state
  b += nl * (n + 1) * 4 + nl * n * 4 * (4 + re);  // exchange CSR (4 neighbours)
  if (nl > 1) b += 2 * nl * ((n + 1) * 4 + n * (4 + re));
  return b;
}

mrm_gpu* new_run(Engine* e, const mrm_geom* g, std::string* errp, int* rc, bool allow_big = false) {
  bool big = false;
  *rc = validate_geom(g, errp, allow_big ? &big : nullptr);
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
  r->fft_big = big;
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
  CK(h2d(*didx, index, sizeof(int) * (n + 1)));
  CK(h2d(*dnbr, nb.data(), sizeof(int) * std::max(nnz, 1)));
  CK(h2d(*dcoef, cf.data(), sizeof(R) * std::max(nnz, 1)));
  return MRM_OK;
}

// host copies of ms_scale per layer (neighbour scaling of exchange coefficients)
struct HostLayerCache {
  std::vector<double> ms_scale, ms, hk_scale, vol, alpha_scale;  // per grain
  std::vector<int> cgrain, rep;                // map layers: cell -> grain (-1 empty), grain -> its first cell
  std::vector<double> ms_scale_cell;           // map layers: the cell's grain's ms_scale (0: empty)
};
std::map<const mrm_gpu*, std::vector<HostLayerCache>>& host_cache() {
  static std::map<const mrm_gpu*, std::vector<HostLayerCache>> m;
  return m;
}

// Frees the runs mrm_batch_remove took out of the engine: the stream has
// passed their last use (remove waited for the work then in flight, and later
// work runs on tables without them)
void release_retired(Engine* e) {
  for (auto* r : e->retired) {
    host_cache().erase(r);
    run_free(r);
    delete r;
  }
  e->retired.clear();
}

template <typename R>
int upload_layer_t(mrm_gpu* r, int l, int n, const double* ms, const double* vol, const double* axis,
                   const double* hk, const double* hk_scale, const double* ms_scale,
                   const double* alpha_scale, double alpha, double gamma, double floor_ms,
                   const int32_t* g2ci, const int32_t* g2c, const int32_t* hxi, const int32_t* hxg,
                   const double* hx) {
  std::string* errp = &r->err;
  const int nx = r->g.nx, ny = r->g.ny, nc = nx * ny;
  if (!ms || !vol || !axis || !hk || !hk_scale || !ms_scale || !alpha_scale || !g2ci || !g2c)
    return set_err(errp, MRM_ERR_ARG, "layer %d: NULL array", l);
  if (n < 1 || n > nc) return set_err(errp, MRM_ERR_ARG, "layer %d: %d grains on %d cells", l, n, nc);
  // one grain per cell in grid order (the fused path), or a grain -> cells map
  // (get_mag / get_magnetostatic, data.f90:322-390, field.f90:438-517)
  bool identity = n == nc;
  for (int g = 0; identity && g < n; ++g)
    identity = g2ci[g] == g && g2ci[g + 1] == g + 1 && g2c[2 * g] - 1 == g % nx && g2c[2 * g + 1] - 1 == g / nx;
  std::vector<int> cg, repc;
  if (!identity) {
    if (g2ci[0] != 0) return set_err(errp, MRM_ERR_ARG, "layer %d: grain2gridindex(0) must be 0", l);
    cg.assign(nc, -1);
    repc.resize(n);
    for (int g = 0; g < n; ++g) {
      if (g2ci[g + 1] <= g2ci[g]) return set_err(errp, MRM_ERR_ARG, "layer %d: grain %d has no cell", l, g + 1);
      for (int q = g2ci[g]; q < g2ci[g + 1]; ++q) {
        const int i = g2c[2 * q] - 1, j = g2c[2 * q + 1] - 1;
        if (i < 0 || i >= nx || j < 0 || j >= ny)
          return set_err(errp, MRM_ERR_ARG, "layer %d: grain %d cell (%d,%d) outside the grid", l, g + 1, i + 1, j + 1);
        const int c = j * nx + i;
        if (cg[c] >= 0) return set_err(errp, MRM_ERR_ARG, "layer %d: cell (%d,%d) in two grains", l, i + 1, j + 1);
        cg[c] = g;
        if (q == g2ci[g]) repc[g] = c;
      }
    }
  }
  // records per cell: the cell's grain's (a grain's first cell carries its
  // volume and counts it in the reductions; empty cells: Ms = 0, no dynamics)
  const double kB = 1.380662e-16;  // field.f90:407
  const double tsig = std::sqrt(2.0 * kB * alpha / gamma);
  std::vector<R> pa(4 * (size_t)nc, (R)0), pb(4 * (size_t)nc, (R)0);
  std::vector<double> pv(4 * (size_t)nc, 0.0);
  for (int c = 0; c < nc; ++c) {
    const int g = identity ? c : cg[c];
    if (g < 0) {
      pv[4 * c + 2] = 1.0;
      continue;
    }
    const bool first = identity || repc[g] == c;
    pa[4 * c + 0] = (R)axis[3 * g];
    pa[4 * c + 1] = (R)axis[3 * g + 1];
    pa[4 * c + 2] = (R)axis[3 * g + 2];
    const double hks = hk_scale[g] > 0.0 ? hk_scale[g] : 0.0;  // get_uni_hk returns 0 for hk_scale <= 0
    pa[4 * c + 3] = (R)(hk[2 * g] * hks);
    pb[4 * c + 0] = (R)(ms[g] * ms_scale[g]);
    pb[4 * c + 1] = (R)(hk[2 * g + 1] * hks);
    pb[4 * c + 2] = (R)(alpha * alpha_scale[g]);
    double x = 0.0;  // field.f90:418-419 without the temperature (applied per step)
    if (ms_scale[g] > 0.0) x = alpha_scale[g] / (ms[g] * vol[g] * std::max(floor_ms, ms_scale[g]));
    pb[4 * c + 3] = (R)(std::sqrt(x) * tsig);
    pv[4 * c + 0] = first ? vol[g] : 0.0;
    pv[4 * c + 1] = ms_scale[g];
    pv[4 * c + 2] = ms[g];
    pv[4 * c + 3] = first ? 1.0 : 0.0;
  }
  LayerBufs& b = r->L[l];
  CK(h2d(b.pa, pa.data(), sizeof(R) * 4 * nc));
  CK(h2d(b.pb, pb.data(), sizeof(R) * 4 * nc));
  CK(h2d(b.pv, pv.data(), sizeof(double) * 4 * nc));
  auto& hc = host_cache()[r];
  hc.resize(MRM_MAX_LAYERS);
  hc[l].ms_scale.assign(ms_scale, ms_scale + n);
  hc[l].ms.assign(ms, ms + n);
  hc[l].hk_scale.assign(hk_scale, hk_scale + n);
  hc[l].vol.assign(vol, vol + n);
  hc[l].alpha_scale.assign(alpha_scale, alpha_scale + n);
  hc[l].cgrain = cg;
  hc[l].rep = repc;
  hc[l].ms_scale_cell.clear();
  dfree(b.xst);
  dfree(b.cgrain); dfree(b.gci); dfree(b.gcs); dfree(b.hdm); dfree(b.hapm);
  b.ng = n;
  if (!identity) {
    hc[l].ms_scale_cell.assign(nc, 0.0);
    for (int c = 0; c < nc; ++c)
      if (cg[c] >= 0) hc[l].ms_scale_cell[c] = ms_scale[cg[c]];
    std::vector<int> cells(g2ci[n]);
    for (int q = 0; q < g2ci[n]; ++q) cells[q] = (g2c[2 * q + 1] - 1) * nx + (g2c[2 * q] - 1);
    int rc = dmalloc(errp, (void**)&b.cgrain, sizeof(int) * nc);
    if (!rc) rc = dmalloc(errp, (void**)&b.gci, sizeof(int) * (n + 1));
    if (!rc) rc = dmalloc(errp, (void**)&b.gcs, sizeof(int) * cells.size());
    if (!rc) rc = dmalloc(errp, &b.hdm, sizeof(R) * 4 * (size_t)nc);
    if (!rc) rc = dmalloc(errp, &b.hapm, sizeof(R) * 4 * (size_t)nc);
    if (rc) return rc;
    CK(h2d(b.cgrain, cg.data(), sizeof(int) * nc));
    CK(h2d(b.gci, g2ci, sizeof(int) * (n + 1)));
    CK(h2d(b.gcs, cells.data(), sizeof(int) * cells.size()));
  }
  if (!identity && hxi && hxg && hx) {
    // intralayer exchange of the grains, on every cell of each grain, with each
    // neighbour grain read at its first cell
    if (hxi[0] != 0) return set_err(errp, MRM_ERR_ARG, "CSR index(0) must be 0");
    std::vector<int> ci(nc + 1, 0), cn;
    std::vector<double> cf;
    for (int c = 0; c < nc; ++c) {
      const int g = cg[c];
      if (g >= 0)
        for (int q = hxi[g]; q < hxi[g + 1]; ++q) {
          const int j = hxg[q] - 1;
          if (j < 0 || j >= n) return set_err(errp, MRM_ERR_ARG, "CSR neighbour %d out of range", hxg[q]);
          cn.push_back(repc[j] + 1);
          cf.push_back(hx[q]);
        }
      ci[c + 1] = (int)cn.size();
    }
    int rc = upload_csr<R>(r, nc, ci.data(), cn.data(), cf.data(), hc[l].ms_scale_cell.data(), nc, &b.xidx,
                           &b.xnbr, &b.xcoef);
    if (rc) return rc;
  } else if (hxi && hxg && hx) {
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
      CK(h2d(b.xst, st.data(), sizeof(R) * 4 * (size_t)n));
    }
  } else {
    dfree(b.xidx); dfree(b.xnbr); dfree(b.xcoef);
  }
  b.gamma = gamma;
  b.alpha = alpha;
  b.floor_ms = floor_ms;
  dfree(b.llb);  // LLB records hold the old grains' parameters: set again after an upload
  dfree(b.llbp);
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
  CK(h2d(d_pg, pg.data(), sizeof(PairGeom) * npair));
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
  // a buffer shared with other runs is left to them: this run writes its own
  if (!r->tens_buf || r->tens_buf.use_count() > 1) {
    CK(cudaStreamSynchronize(e->st));
    int rc0 = tensor_alloc(r);
    if (rc0) return rc0;
  }
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
  CK(h2d(d_tw64, tw.data(), sizeof(double) * 2 * kTwN));
  const Cx<double>* tw64 = static_cast<const Cx<double>*>(d_tw64);
  const int M = r->px / 2;
  // two shared buffers of one padded-stride sequence each (fft.cuh)
  size_t s1 = 2 * (size_t)pad_stride(M) * sizeof(Cx<double>), s2 = 2 * (size_t)pad_stride(r->py) * sizeof(Cx<double>);
  CK(allow_smem((const void*)r2c_rows_f64, s1));
  CK(allow_smem((const void*)c2c_cols_f64, s2));
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
  } else if (creg_run(r)) {
    const long long total = (long long)ph * 6 * r->py;
    pack_tensor_creg_kernel<<<(unsigned)((total + 255) / 256), 256, 0, e->st>>>(
        static_cast<const Cx<double>*>(d_spec), static_cast<float*>(r->tens), r->lgpy, ph, d_mx, d_mx + 1);
  } else {
    const long long total = (long long)ph * npair * 9 * pyh;
    pack_tensor_kernel<float><<<(unsigned)((total + 255) / 256), 256, 0, e->st>>>(
        static_cast<const Cx<double>*>(d_spec), static_cast<float*>(r->tens), npair, r->py, ph,
        tens_row_stride(r->py), d_mx, d_mx + 1);
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

template <typename R>
int set_cubic_t(mrm_gpu* h, int layer, const double* cubic_axis) {
  std::string* errp = &h->err;
  LayerBufs& b = h->L[layer];
  const int n = b.n;  // cells
  const HostLayerCache& hc = host_cache()[h][layer];
  std::vector<R> v(12 * (size_t)n, (R)0);
  for (int c = 0; c < n; ++c) {
    const int g = hc.cgrain.empty() ? c : hc.cgrain[c];
    if (g < 0) continue;
    const double hs = hc.hk_scale[g] > 0.0 ? hc.hk_scale[g] : 0.0;  // get_cubic_hk returns 0 for hk_scale <= 0
    for (int i = 0; i < 3; ++i) {
      for (int k = 0; k < 3; ++k) v[12 * (size_t)c + 4 * i + k] = (R)cubic_axis[9 * (size_t)g + 3 * i + k];
      v[12 * (size_t)c + 4 * i + 3] = (R)(i == 0 ? hs * hc.ms[g] : 0.0);
    }
  }
  if (!b.cax) {
    int rc = dmalloc(errp, &b.cax, sizeof(R) * 12 * (size_t)n);
    if (rc) return rc;
  }
  CK(h2d(b.cax, v.data(), sizeof(R) * 12 * (size_t)n));
  return MRM_OK;
}

}  // namespace

// =====================================================================
// C ABI
// =====================================================================
extern "C" {

int mrm_gpu_create(const mrm_geom* geom, int device, mrm_gpu** out) {
  if (!out) return MRM_ERR_ARG;
  *out = nullptr;
  bool big = false;  // (new_run marks such a handle)
  int rc = validate_geom(geom, &g_create_err, &big);
  if (rc) return rc;
  Engine* e = new Engine();
  rc = engine_init(e, geom->precision, device);
  if (rc) {
    g_create_err = e->err;
    engine_free(e);
    delete e;
    return rc;
  }
  mrm_gpu* r = new_run(e, geom, &g_create_err, &rc, true);  // (a long track demagnetises through a window)
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
  int n = b.n;
  int rc;
  // map layers: the coupling of each grain on every one of its cells, the other
  // layer's grain read at its first cell
  std::vector<int> mi, mg;
  std::vector<double> mc;
  const double* nbr_scale = hc[other].ms_scale.data();
  int n_nbr = h->L[other].n;
  const bool mapped = !hc[layer].cgrain.empty() || !hc[other].cgrain.empty();
  if (mapped) {
    const std::vector<int>& cg = hc[layer].cgrain;
    const int ng = b.ng, ngo = h->L[other].ng;
    if (index[0] != 0) return set_err(errp, MRM_ERR_ARG, "CSR index(0) must be 0");
    mi.assign(n + 1, 0);
    for (int c = 0; c < n; ++c) {
      const int g = cg.empty() ? c : cg[c];
      if (g >= 0 && g < ng)
        for (int q = index[g]; q < index[g + 1]; ++q) {
          const int j = grain[q] - 1;
          if (j < 0 || j >= ngo) return set_err(errp, MRM_ERR_ARG, "interlayer neighbour %d out of range", grain[q]);
          mg.push_back((hc[other].cgrain.empty() ? j : hc[other].rep[j]) + 1);
          mc.push_back(coef[q]);
        }
      mi[c + 1] = (int)mg.size();
    }
    if (mg.empty()) {  // keep the arrays non-empty
      mg.push_back(1);
      mc.push_back(0.0);
    }
    index = mi.data();
    grain = mg.data();
    coef = mc.data();
    if (!hc[other].cgrain.empty()) nbr_scale = hc[other].ms_scale_cell.data();
  }
  if (h->g.precision == MRM_FP64)
    rc = side == 0 ? upload_csr<double>(h, n, index, grain, coef, nbr_scale, n_nbr, &b.uidx, &b.unbr, &b.ucoef)
                   : upload_csr<double>(h, n, index, grain, coef, nbr_scale, n_nbr, &b.lidx, &b.lnbr, &b.lcoef);
  else
    rc = side == 0 ? upload_csr<float>(h, n, index, grain, coef, nbr_scale, n_nbr, &b.uidx, &b.unbr, &b.ucoef)
                   : upload_csr<float>(h, n, index, grain, coef, nbr_scale, n_nbr, &b.lidx, &b.lnbr, &b.lcoef);
  if (rc) return rc;
  // columnar form: grain n couples to grain n of the other layer only
  void** col = side == 0 ? &b.ucol : &b.lcol;
  dfree(*col);
  bool columnar = !mapped && h->L[other].n == n;
  for (int g = 0; columnar && g < n; ++g)
    columnar = (index[g + 1] - index[g] == 1) && (grain[index[g]] == g + 1);
  if (columnar) {
    const size_t re = relem(h->g.precision);
    std::vector<double> cf(n);
    for (int g = 0; g < n; ++g) cf[g] = coef[index[g]] * hc[other].ms_scale[g];
    rc = dmalloc(errp, col, re * n);
    if (rc) return rc;
    if (h->g.precision == MRM_FP64) {
      CK(h2d(*col, cf.data(), sizeof(double) * n));
    } else {
      std::vector<float> f(cf.begin(), cf.end());
      CK(h2d(*col, f.data(), sizeof(float) * n));
    }
  }
  h->eng->desc_dirty = true;
  return MRM_OK;
}

// The stray field of all layers at an observation slab of thickness dzobs whose
// bottom is zoff above the top layer, on the nx x ny grid with the periodic
// images of the reference's off-plane tensor (off_field.f90:55-108,216-320).
int mrm_gpu_off_field(mrm_gpu* h, double zoff, double dzobs, double head_mu, double fly_height, double sul_mu,
                      double space_to_sul, int num_images, double* out) {
  if (!h || !out) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  const int nx = h->g.nx, ny = h->g.ny, nl = h->nl;
  if (!(dzobs > 0)) return set_err(errp, MRM_ERR_ARG, "dzobs must be > 0");
  if (num_images < 0) return set_err(errp, MRM_ERR_ARG, "num_images must be >= 0");
  if (!is_pow2(nx) || !is_pow2(ny) || nx < 4 || ny < 2 || nx > kTwN || ny > kTwN)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "the off-plane field needs power-of-two nx >= 4, ny >= 2 (got %d x %d)",
                   nx, ny);
  for (int l = 0; l < nl; ++l)
    if (!h->L[l].uploaded) return set_err(errp, MRM_ERR_STATE, "upload layer %d first", l);
  Engine* e = h->eng;
  CK(cudaSetDevice(e->dev));
  int rc = e->prec == MRM_FP64 ? ensure_ready<double>(e) : ensure_ready<float>(e);
  if (rc) {
    h->err = e->err;
    return rc;
  }
  // calculate_off_field_tensor (off_field.f90:216-320): source layer ks, slab above the media
  const mrm_geom& g = h->g;
  std::vector<PairGeom> pg(nl);
  const bool sul_p = sul_mu > 1.0, head_p = head_mu > 1.0;
  const double mus = sul_p ? std::max(0.0, (std::max(1.0, sul_mu) - 1.0) / (std::max(1.0, sul_mu) + 1.0)) : 0.0;
  const double mush = head_p ? std::max(0.0, (std::max(1.0, head_mu) - 1.0) / (std::max(1.0, head_mu) + 1.0)) : 0.0;
  std::vector<double> hdz(nl);
  hdz[0] = fly_height;
  for (int k = 1; k < nl; ++k) hdz[k] = hdz[k - 1] + g.dz[k - 1] + g.il_space[k];
  for (int k = 0; k < nl; ++k) hdz[k] += 0.5 * g.dz[k];
  double zob = space_to_sul + zoff;
  for (int k = 0; k < nl; ++k) zob += g.dz[k] + (k != nl - 1 ? g.il_space[k] : 0.0);
  const double zot = zob + dzobs;
  double zsb = space_to_sul;
  for (int ks = nl - 1; ks >= 0; --ks) {
    const double zst = zsb + g.dz[ks];
    PairGeom& p = pg[ks];
    p.dz_s = g.dz[ks];
    p.dz_o = dzobs;
    p.rz = 0.5 * (zst - zot + zsb - zob);
    p.rz_sul = 0.5 * (-zst - zot - zsb - zob);
    p.f_sul = mus;
    p.rz_head = hdz[ks] + fly_height - (zoff + 0.5 * dzobs);
    p.f_head = mush;
    p.norm = 1.0 / (g.dx * g.dy * dzobs * (double)nx * (double)ny);
    zsb = zst + g.il_space[ks];
  }
  const int ph = nx / 2 + 1, lgx = ilog2(nx), lgy = ilog2(ny);
  const size_t plane = (size_t)nx * ny, hplane = (size_t)ph * ny;
  void *d_pg = nullptr, *d_t = nullptr, *d_ts = nullptr, *d_m = nullptr, *d_ms = nullptr, *d_h = nullptr,
       *d_out = nullptr, *d_tw = nullptr;
  auto finish = [&](int code) {
    for (void* q : {d_pg, d_t, d_ts, d_m, d_ms, d_h, d_out, d_tw}) {
      void* qq = q;
      dfree(qq);
    }
    return code;
  };
  rc = dmalloc(errp, &d_pg, sizeof(PairGeom) * nl);
  if (!rc) rc = dmalloc(errp, &d_t, sizeof(double) * 9 * nl * plane);
  if (!rc) rc = dmalloc(errp, &d_ts, sizeof(double) * 2 * 9 * nl * hplane);
  if (!rc) rc = dmalloc(errp, &d_m, sizeof(double) * 3 * nl * plane);
  if (!rc) rc = dmalloc(errp, &d_ms, sizeof(double) * 2 * 3 * nl * hplane);
  if (!rc) rc = dmalloc(errp, &d_h, sizeof(double) * 2 * 3 * hplane);
  if (!rc) rc = dmalloc(errp, &d_out, sizeof(double) * 3 * plane);
  if (!rc) rc = dmalloc(errp, &d_tw, sizeof(double) * 2 * kTwN);
  if (rc) return finish(rc);
  std::vector<double> tw(2 * kTwN);
  for (int k = 0; k < kTwN; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)kTwN;
    tw[2 * k] = std::cos(a);
    tw[2 * k + 1] = std::sin(a);
  }
  const cudaStream_t st = e->st;
  auto ok = [&](cudaError_t c) { return c == cudaSuccess; };
  if (!ok(cudaMemcpyAsync(d_tw, tw.data(), sizeof(double) * 2 * kTwN, cudaMemcpyHostToDevice, st)) ||
      !ok(cudaMemcpyAsync(d_pg, pg.data(), sizeof(PairGeom) * nl, cudaMemcpyHostToDevice, st)))
    return finish(set_err(errp, MRM_ERR_CUDA, "off-plane field: copy"));
  const Cx<double>* tw64 = static_cast<const Cx<double>*>(d_tw);
  const long long tot = (long long)nl * plane;
  tensor_real_kernel<<<(unsigned)((tot + 127) / 128), 128, 0, st>>>(static_cast<double*>(d_t),
                                                                     static_cast<const PairGeom*>(d_pg), nl, nx, ny,
                                                                     g.dx, g.dy, num_images);
  if (e->prec == MRM_FP64)
    mgrid_kernel<double><<<dim3((unsigned)((plane + 255) / 256), nl), 256, 0, st>>>(
        static_cast<const RunDev<double>*>(e->d_runs), h->slot, static_cast<double*>(d_m));
  else
    mgrid_kernel<float><<<dim3((unsigned)((plane + 255) / 256), nl), 256, 0, st>>>(
        static_cast<const RunDev<float>*>(e->d_runs), h->slot, static_cast<double*>(d_m));
  const size_t s1 = 2 * (size_t)pad_stride(nx / 2) * sizeof(Cx<double>), s2 = 2 * (size_t)pad_stride(ny) * sizeof(Cx<double>);
  if (!ok(allow_smem((const void*)r2c_rows_f64, s1)) || !ok(allow_smem((const void*)c2c_cols_f64, s2)) ||
      !ok(allow_smem((const void*)c2c_cols_f64_inv, s2)) || !ok(allow_smem((const void*)c2r_rows_f64, s1)))
    return finish(set_err(errp, MRM_ERR_CUDA, "off-plane field: shared memory"));
  // forward transforms of the tensor and of M, the products, the inverse transform
  r2c_rows_f64<<<(unsigned)(9 * nl * ny), 256, s1, st>>>(static_cast<const double*>(d_t), static_cast<Cx<double>*>(d_ts),
                                                           lgx, ny, tw64);
  c2c_cols_f64<<<(unsigned)(9 * nl * ph), 256, s2, st>>>(static_cast<Cx<double>*>(d_ts), lgy, ph, tw64);
  r2c_rows_f64<<<(unsigned)(3 * nl * ny), 256, s1, st>>>(static_cast<const double*>(d_m), static_cast<Cx<double>*>(d_ms),
                                                           lgx, ny, tw64);
  c2c_cols_f64<<<(unsigned)(3 * nl * ph), 256, s2, st>>>(static_cast<Cx<double>*>(d_ms), lgy, ph, tw64);
  off_mac_kernel<<<(unsigned)((hplane + 255) / 256), 256, 0, st>>>(static_cast<const Cx<double>*>(d_ts),
                                                                     static_cast<const Cx<double>*>(d_ms),
                                                                     static_cast<Cx<double>*>(d_h), nl, (long long)hplane);
  c2c_cols_f64_inv<<<(unsigned)(3 * ph), 256, s2, st>>>(static_cast<Cx<double>*>(d_h), lgy, ph, tw64);
  c2r_rows_f64<<<(unsigned)(3 * ny), 256, s1, st>>>(static_cast<const Cx<double>*>(d_h), static_cast<double*>(d_out), lgx,
                                                    tw64);
  if (!ok(cudaGetLastError()) ||
      !ok(cudaMemcpyAsync(out, d_out, sizeof(double) * 3 * plane, cudaMemcpyDeviceToHost, st)) ||
      !ok(cudaStreamSynchronize(st)))
    return finish(set_err(errp, MRM_ERR_CUDA, "off-plane field: %s", cudaGetErrorString(cudaGetLastError())));
  return finish(MRM_OK);
}

static int need_fft(mrm_gpu* h);

int mrm_gpu_build_tensor(mrm_gpu* h) {
  if (!h) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  if (int rc = need_fft(h)) return rc;
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
  if (int rc = need_fft(h)) return rc;
  if (nx_fft != h->px || ny_fft != h->py)
    return set_err(errp, MRM_ERR_ARG, "tensor grid %dx%d differs from the FFT grid %dx%d", nx_fft, ny_fft, h->px, h->py);
  CK(cudaSetDevice(h->eng->dev));
  void* d_n2d = nullptr;
  const size_t bytes = sizeof(double) * 9 * (size_t)h->nl * h->nl * h->px * h->py;
  int rc = dmalloc(errp, &d_n2d, bytes);
  if (rc) return rc;
  CK(h2d(d_n2d, n2d, bytes));
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
  // the same geometry has the same tensor: share the source's buffer (it is
  // only read from now on; a later build or upload on either run writes a
  // buffer of its own).  The source's tensor must be complete; the
  // destination's own earlier buffer, if any, must be out of use before it
  // is released (a fresh run has none, and nothing in flight reads it).
  CK(cudaStreamSynchronize(src->eng->st));
  if (dst->tens_buf) CK(cudaStreamSynchronize(dst->eng->st));
  dst->tens_buf = src->tens_buf;
  dst->tens = src->tens;
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
  if (func < 1 || func > 7 || func == kFuncHead) return set_err(&h->err, MRM_ERR_ARG, "unknown time function %d", func);
  if (func == kFuncRot && std::fabs(gamma) == 1.0)
    return set_err(&h->err, MRM_ERR_UNSUPPORTED,
                   "ROT with |gamma| = 1 turns the field after the mean magnetisation of every step (llg.f90:332-360): "
                   "not on this path");
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

int mrm_gpu_set_head_field(mrm_gpu* h, int layer, double gap, double z, double hg, double velocity, double x0,
                           double t0, double bit_time, uint64_t pattern, int nbits) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  if (!(gap > 0 && z > 0 && bit_time > 0) || nbits < 1 || nbits > 64)
    return set_err(&h->err, MRM_ERR_ARG, "head field needs gap, z, bit_time > 0 and 1 <= nbits <= 64");
  LayerBufs& b = h->L[layer];
  dfree(b.tab);  // a layer has one field profile
  dfree(b.tb_v);
  dfree(b.tb_pos);
  b.func = kFuncHead;
  b.amp = 0.0;
  b.dc = 0.0;
  b.scale = 1.0;
  b.hd_gap = gap;
  b.hd_z = z;
  b.hd_hg = hg;
  b.hd_v = velocity;
  b.hd_x0 = x0;
  b.hd_t0 = t0;
  b.hd_tbit = bit_time;
  b.hd_bits = pattern;
  b.hd_nbits = nbits;
  h->eng->desc_dirty = true;
  h->eng->tables_dirty = true;  // the row kernel's shared memory grows by the head table
  return MRM_OK;
}

int mrm_gpu_set_field_table(mrm_gpu* h, int layer, int nfx, int nfy, const double* xpos, const double* ypos,
                            const double* vfld, double vel_x, double vel_y, double offset_x, double offset_y,
                            double ref_x, double ref_y, double t_origin) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  std::string* errp = &h->err;
  LayerBufs& b = h->L[layer];
  CK(cudaSetDevice(h->eng->dev));
  CK(cudaStreamSynchronize(h->eng->st));  // a step in flight may read the old table
  dfree(b.tab);
  dfree(b.tb_v);
  dfree(b.tb_pos);
  h->eng->desc_dirty = true;
  h->eng->tables_dirty = true;  // the row kernel's shared memory holds the interpolation weights
  if (nfx == 0 && nfy == 0) return MRM_OK;
  if (!xpos || !ypos || !vfld || nfx < 2 || nfy < 2)
    return set_err(errp, MRM_ERR_ARG, "a field table needs at least 2 x 2 nodes (got %d x %d)", nfx, nfy);
  for (int i = 0; i < nfx; ++i)
    if (!std::isfinite(xpos[i]) || (i && !(xpos[i] > xpos[i - 1])))
      return set_err(errp, MRM_ERR_ARG, "table x positions must be finite and ascending (node %d)", i);
  for (int j = 0; j < nfy; ++j)
    if (!std::isfinite(ypos[j]) || (j && !(ypos[j] > ypos[j - 1])))
      return set_err(errp, MRM_ERR_ARG, "table y positions must be finite and ascending (node %d)", j);
  const size_t nv = 3 * (size_t)nfx * nfy;
  std::vector<double> pos(xpos, xpos + nfx);
  pos.insert(pos.end(), ypos, ypos + nfy);
  int rc = dmalloc(errp, &b.tb_v, sizeof(double) * nv);
  if (!rc) rc = dmalloc(errp, &b.tb_pos, sizeof(double) * pos.size());
  if (!rc) rc = dmalloc(errp, &b.tab, sizeof(TabDev));
  if (rc) {
    dfree(b.tb_v);
    dfree(b.tb_pos);
    return rc;
  }
  TabDev td{};
  td.v = static_cast<const double*>(b.tb_v);
  td.pos = static_cast<const double*>(b.tb_pos);
  td.nx = nfx;
  td.ny = nfy;
  // file_applied's default offset: the centre of the grid (applied.f90:804-805)
  td.ox = offset_x < -1e200 ? h->g.dx * h->g.nx * 0.5 : offset_x;
  td.oy = offset_y < -1e200 ? h->g.dy * h->g.ny * 0.5 : offset_y;
  td.vx = vel_x;
  td.vy = vel_y;
  td.rx = ref_x;
  td.ry = ref_y;
  td.t0 = t_origin;
  td.dx = h->g.dx;
  td.dy = h->g.dy;
  CK(h2d(b.tb_v, vfld, sizeof(double) * nv));
  CK(h2d(b.tb_pos, pos.data(), sizeof(double) * pos.size()));
  CK(h2d(b.tab, &td, sizeof(TabDev)));
  if (b.func == kFuncHead) {  // back to the default time scale (1)
    b.func = 0;
    b.scale = 1.0;
    b.s_start = b.s_end = 1.0;
  }
  return MRM_OK;
}

static int set_llb_mode(mrm_gpu* h, int layer, double spin, const double* tc, const double* lambda_ms, int mode,
                        int meq_bs, int garanin_tau);

int mrm_gpu_set_llb(mrm_gpu* h, int layer, double spin, const double* tc, const double* lambda_ms) {
  return set_llb_mode(h, layer, spin, tc, lambda_ms, 0, 0, 0);
}

int mrm_gpu_set_mt(mrm_gpu* h, int layer, double spin, const double* lambda_ms, int meq_bs, int garanin_tau) {
  return set_llb_mode(h, layer, spin, lambda_ms, lambda_ms, 1, meq_bs, garanin_tau);
}

int mrm_gpu_set_zhang(mrm_gpu* h, int layer, double spin, const double* lambda_ms, int meq_bs, int garanin_tau) {
  return set_llb_mode(h, layer, spin, lambda_ms, lambda_ms, 2, meq_bs, garanin_tau);
}

static int set_llb_mode(mrm_gpu* h, int layer, double spin, const double* tc, const double* lambda_ms, int mode,
                        int meq_bs, int garanin_tau) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  std::string* errp = &h->err;
  LayerBufs& b = h->L[layer];
  if (!b.uploaded) return set_err(errp, MRM_ERR_STATE, "upload layer %d first", layer);
  CK(cudaSetDevice(h->eng->dev));
  CK(cudaStreamSynchronize(h->eng->st));
  dfree(b.llb);
  dfree(b.llbp);
  h->eng->desc_dirty = true;
  h->eng->tables_dirty = true;  // the general kernels
  if (!tc) return MRM_OK;
  if (!lambda_ms || !(spin > 0)) return set_err(errp, MRM_ERR_ARG, "LLB needs spin > 0, Tc and lambdaMs");
  const HostLayerCache& hc = host_cache()[h][layer];
  const int ng = b.ng, nc = b.n;
  if (mode == 0)
    for (int g = 0; g < ng; ++g)
      if (!(tc[g] > 0)) return set_err(errp, MRM_ERR_ARG, "LLB needs Tc > 0 (grain %d)", g);
  // per cell: Tc, lambda_m = lambdaMs (spin+1)/spin (llg.f90:931), and
  // get_thermal's 2 k_B alpha alpha_scale / (gamma Ms V) (field.f90:407,417)
  std::vector<V4<double>> rec(nc, V4<double>{1.0, 0.0, 0.0, 0.0});
  for (int c = 0; c < nc; ++c) {
    const int g = hc.cgrain.empty() ? c : hc.cgrain[c];
    if (g < 0) continue;
    const double msv = hc.ms[g] * hc.vol[g];
    rec[c].x = mode == 0 ? tc[g] : 0.0;
    // LLB: lambda_m = lambdaMs (S+1)/S; MT: lambdaMs (push_mt scales it by meq_bs)
    rec[c].y = mode == 0 ? lambda_ms[g] * (spin + 1.0) / spin : lambda_ms[g];  // (MT / Zhang: raw)
    rec[c].z = msv > 0 ? 2.0 * kBoltz * b.alpha * hc.alpha_scale[g] / (b.gamma * msv) : 0.0;
  }
  LlbDev d{};
  int rc = dmalloc(errp, &b.llbp, sizeof(V4<double>) * (size_t)nc);
  if (!rc) rc = dmalloc(errp, &b.llb, sizeof(LlbDev));
  if (rc) {
    dfree(b.llbp);
    return rc;
  }
  d.p = static_cast<const V4<double>*>(b.llbp);
  d.spin = spin;
  d.alpha = b.alpha;
  d.floor_ms = b.floor_ms;
  d.mode = mode;
  d.meq_bs = meq_bs ? 1 : 0;
  d.garanin_tau = garanin_tau ? 1 : 0;
  CK(h2d(b.llbp, rec.data(), sizeof(V4<double>) * (size_t)nc));
  CK(h2d(b.llb, &d, sizeof(LlbDev)));
  return MRM_OK;
}

static int push_temp_profile(mrm_gpu* h, LayerBufs& b) {
  std::string* errp = &h->err;
  if (!b.tprof) {
    int rc = dmalloc(errp, &b.tprof, sizeof(TempDev));
    if (rc) return rc;
  }
  CK(cudaSetDevice(h->eng->dev));
  CK(cudaStreamSynchronize(h->eng->st));
  CK(h2d(b.tprof, &b.tp, sizeof(TempDev)));
  h->eng->desc_dirty = true;
  h->eng->tables_dirty = true;  // the general kernels
  return MRM_OK;
}

int mrm_gpu_set_temp_profile(mrm_gpu* h, int layer, double background, double dtemp, double sigma_x, double sigma_y,
                             int expn, double vel_x, double vel_y, double offset_x, double offset_y, double ref_x,
                             double ref_y, double t_origin) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  std::string* errp = &h->err;
  LayerBufs& b = h->L[layer];
  if (expn < 0) {  // off
    CK(cudaSetDevice(h->eng->dev));
    CK(cudaStreamSynchronize(h->eng->st));
    dfree(b.tprof);
    h->eng->desc_dirty = true;
    h->eng->tables_dirty = true;
    return MRM_OK;
  }
  if (b.cgrain) return set_err(errp, MRM_ERR_UNSUPPORTED, "a temperature profile needs one grain per cell");
  if (expn < 1) return set_err(errp, MRM_ERR_ARG, "super-Gaussian exponent must be >= 1");
  const bool fresh = !b.tprof;
  TempDev& p = b.tp;
  if (fresh) {  // the time scale starts constant 1
    p.func = 0;
    p.t_start = -1e22;
    p.t_end = 1e22;
    p.s_start = p.s_end = 1.0;
    p.scale = 1.0;
  }
  p.bg = background;
  p.dtemp = dtemp;
  p.isx = sigma_x != 0.0 ? 1.0 / sigma_x : 0.0;  // suprgaus_temp (applied.f90:476-477)
  p.isy = sigma_y != 0.0 ? 1.0 / sigma_y : 0.0;
  p.expn = 2 * expn;
  p.vx = vel_x;
  p.vy = vel_y;
  p.ox = offset_x < -1e200 ? h->g.dx * h->g.nx * 0.5 : offset_x;  // the grid centre (:459-460)
  p.oy = offset_y < -1e200 ? h->g.dy * h->g.ny * 0.5 : offset_y;
  p.rx = ref_x;
  p.ry = ref_y;
  p.t0 = t_origin;
  p.dx = h->g.dx;
  p.dy = h->g.dy;
  return push_temp_profile(h, b);
}

// file_temp_scaling's reduction of a table as read (temp_scaling.f90:152-203):
// ordered by temperature (ties keep their order), equal temperatures merged
// pairwise from the top into the mean of their scales, an equal first pair
// and an equal last pair of scales trimmed, and temperatures whose largest
// exceeds 5 (a table in K) divided by it
static void reduce_scaling_table(int n, const double* temp, const double* scaling, std::vector<double>& t_out,
                                 std::vector<double>& v_out) {
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return temp[a] < temp[b]; });
  std::vector<double> t(n), v(n);
  for (int i = 0; i < n; ++i) {
    t[i] = temp[ord[i]];
    v[i] = scaling[ord[i]];
  }
  int merged = 0;
  for (int i = n - 1; i >= 1; --i) {
    if (t[i - 1] != t[i]) continue;
    ++merged;
    v[i - 1] = 0.5 * (v[i - 1] + v[i]);
    for (int j = i + 1; j < n; ++j) {  // the entries above move down one place (to the table's end)
      t[j - 1] = t[j];
      v[j - 1] = v[j];
    }
  }
  int m = std::max(1, n - merged);
  if (m >= 2 && v[0] == v[1]) {
    t.erase(t.begin());
    v.erase(v.begin());
    --m;
  }
  if (m > 1 && v[m - 2] == v[m - 1]) --m;
  if (t[m - 1] > 5.0) {
    const double top = t[m - 1];
    for (int i = 0; i < m; ++i) t[i] /= top;
  }
  t_out.assign(t.begin(), t.begin() + m);
  v_out.assign(v.begin(), v.begin() + m);
}

static int push_temp_scaling(mrm_gpu* h, LayerBufs& b) {
  std::string* errp = &h->err;
  CK(cudaSetDevice(h->eng->dev));
  CK(cudaStreamSynchronize(h->eng->st));
  dfree(b.tsc);
  dfree(b.tsc_tab);
  h->eng->desc_dirty = true;
  h->eng->tables_dirty = true;  // the level-2 kernels
  if (!b.tsc_on) {
    dfree(b.tsc_tc);
    return MRM_OK;
  }
  TscDev d{};
  // the tables of Ms, alpha and Hk (Hx's scales nothing in the reference)
  std::vector<double> tt, tv;
  for (int k = 0; k < 3; ++k) {
    d.off[k] = (int)tt.size();
    d.nt[k] = (int)b.tsc_t[k].size();
    tt.insert(tt.end(), b.tsc_t[k].begin(), b.tsc_t[k].end());
    tv.insert(tv.end(), b.tsc_v[k].begin(), b.tsc_v[k].end());
  }
  const size_t nt = std::max<size_t>(tt.size(), 1);
  int rc = dmalloc(errp, &b.tsc_tab, sizeof(double) * 2 * nt);
  if (!rc) rc = dmalloc(errp, &b.tsc, sizeof(TscDev));
  if (rc) return rc;
  double* tab_d = static_cast<double*>(b.tsc_tab);
  if (!tt.empty()) {
    CK(h2d(tab_d, tt.data(), sizeof(double) * tt.size()));
    CK(h2d(tab_d + nt, tv.data(), sizeof(double) * tv.size()));
  }
  d.tc = static_cast<const double*>(b.tsc_tc);
  d.tt = tab_d;
  d.tv = tab_d + nt;
  d.msexp = b.tsc_msexp;
  d.hkexp = b.tsc_hkexp;
  d.floor_ms = b.floor_ms;
  d.mag = b.tsc_mag;
  CK(h2d(b.tsc, &d, sizeof(TscDev)));
  return MRM_OK;
}

int mrm_gpu_set_temp_scaling(mrm_gpu* h, int layer, const double* tc, double msexp, double hkexp, int use_mag) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  std::string* errp = &h->err;
  LayerBufs& b = h->L[layer];
  if (!tc) {
    b.tsc_on = false;
    return push_temp_scaling(h, b);
  }
  if (!b.uploaded) return set_err(errp, MRM_ERR_STATE, "upload layer %d first", layer);
  const HostLayerCache& hc = host_cache()[h][layer];
  if (!hc.cgrain.empty()) return set_err(errp, MRM_ERR_UNSUPPORTED, "temperature scaling needs one grain per cell");
  if (h->wnx) return set_err(errp, MRM_ERR_UNSUPPORTED, "temperature scaling with a moving demag window");
  for (int g = 0; g < b.ng; ++g) {
    if (hc.ms_scale[g] != 1.0 || hc.hk_scale[g] != 1.0 || hc.alpha_scale[g] != 1.0)
      return set_err(errp, MRM_ERR_STATE, "layer %d: temperature scaling replaces the scales; upload them as 1", layer);
    if (!(tc[g] > 0)) return set_err(errp, MRM_ERR_ARG, "temperature scaling needs Tc > 0 (grain %d)", g);
  }
  CK(cudaSetDevice(h->eng->dev));
  CK(cudaStreamSynchronize(h->eng->st));
  dfree(b.tsc_tc);
  int rc = dmalloc(errp, &b.tsc_tc, sizeof(double) * (size_t)b.ng);
  if (rc) return rc;
  CK(h2d(b.tsc_tc, tc, sizeof(double) * (size_t)b.ng));
  b.tsc_on = true;
  b.tsc_msexp = msexp;
  b.tsc_hkexp = hkexp;
  b.tsc_mag = use_mag ? 1 : 0;
  return push_temp_scaling(h, b);
}

int mrm_gpu_set_temp_scaling_table(mrm_gpu* h, int layer, int which, int n, const double* temp,
                                   const double* scaling) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  if (which < 1 || which > 4) return set_err(&h->err, MRM_ERR_ARG, "table %d: 1 Ms, 2 alpha, 3 Hk, 4 Hx", which);
  if (n < 0 || (n > 0 && (!temp || !scaling))) return MRM_ERR_ARG;
  LayerBufs& b = h->L[layer];
  if (n == 0) {
    b.tsc_t[which - 1].clear();
    b.tsc_v[which - 1].clear();
  } else {
    reduce_scaling_table(n, temp, scaling, b.tsc_t[which - 1], b.tsc_v[which - 1]);
  }
  return b.tsc_on ? push_temp_scaling(h, b) : MRM_OK;
}

int mrm_gpu_get_temp_scaling_table(const mrm_gpu* h, int layer, int which, int* n, double* temp, double* scaling) {
  if (!h || !n || layer < 0 || layer >= h->nl || which < 1 || which > 4) return MRM_ERR_ARG;
  const LayerBufs& b = h->L[layer];
  const int m = (int)b.tsc_t[which - 1].size();
  if (*n < m) {
    *n = m;
    return MRM_ERR_ARG;
  }
  for (int i = 0; i < m; ++i) {
    if (temp) temp[i] = b.tsc_t[which - 1][i];
    if (scaling) scaling[i] = b.tsc_v[which - 1][i];
  }
  *n = m;
  return MRM_OK;
}

int mrm_gpu_set_temp_function(mrm_gpu* h, int layer, int func, double t_start, double t_end, double s_start,
                              double s_end, double amp, double gamma, double phase, double param, double duty,
                              double moddepth, double dc, double scale) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  LayerBufs& b = h->L[layer];
  if (!b.tprof) return set_err(&h->err, MRM_ERR_STATE, "set the temperature profile of layer %d first", layer);
  if (func < 0 || func > 5) return set_err(&h->err, MRM_ERR_ARG, "unknown time function %d", func);
  TempDev& p = b.tp;
  p.func = func;
  p.t_start = t_start;
  p.t_end = t_end;
  p.s_start = s_start;
  p.s_end = s_end;
  p.amp = amp;
  p.fgamma = gamma;
  p.phase = phase;
  p.param = param;
  p.duty = std::max(0.0, std::min(1.0, duty));
  p.moddepth = std::max(0.0, std::min(1.0, moddepth));
  p.dc = dc;
  p.scale = scale;
  return push_temp_profile(h, b);
}

int mrm_gpu_set_cubic_axes(mrm_gpu* h, int layer, const double* cubic_axis) {
  if (!h) return MRM_ERR_ARG;
  if (layer < 0 || layer >= h->nl) return set_err(&h->err, MRM_ERR_ARG, "layer %d out of range", layer);
  if (!h->L[layer].uploaded) return set_err(&h->err, MRM_ERR_STATE, "upload layer %d first", layer);
  std::string* errp = &h->err;
  CK(cudaSetDevice(h->eng->dev));
  if (!cubic_axis) {
    dfree(h->L[layer].cax);
  } else {
    int rc = h->g.precision == MRM_FP64 ? set_cubic_t<double>(h, layer, cubic_axis)
                                        : set_cubic_t<float>(h, layer, cubic_axis);
    if (rc) return rc;
  }
  h->spec_valid = false;
  h->eng->desc_dirty = true;
  h->eng->tables_dirty = true;  // the general kernels take the cubic layers
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
  const LayerBufs& b = h->L[layer];
  const int n = b.n;
  cudaStream_t st = h->eng->st;
  CK(cudaSetDevice(h->eng->dev));
  // the caller's array as it is (one record per grain), then widened on the
  // device into m and m* of every cell, in stream order after the work already queued
  CK(cudaMemcpyAsync(h->xfer, m, sizeof(double) * 3 * b.ng, cudaMemcpyHostToDevice, st));
  const unsigned blocks = (unsigned)((n + 255) / 256);
  if (h->g.precision == MRM_FP64)
    state_in_kernel<double><<<blocks, 256, 0, st>>>(static_cast<const double*>(h->xfer),
                                                     static_cast<V4<double>*>(b.m), static_cast<V4<double>*>(b.mp),
                                                     n, b.cgrain);
  else
    state_in_kernel<float><<<blocks, 256, 0, st>>>(static_cast<const double*>(h->xfer),
                                                    static_cast<V4<float>*>(b.m), static_cast<V4<float>*>(b.mp), n,
                                                    b.cgrain);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));  // the caller may reuse its array on return
  h->spec_valid = false;
  return MRM_OK;
}

static int get_v4(mrm_gpu* h, int layer, void* src, double* out) {
  std::string* errp = &h->err;
  if (layer < 0 || layer >= h->nl) return set_err(errp, MRM_ERR_ARG, "layer %d out of range", layer);
  const LayerBufs& b = h->L[layer];
  const int n = b.ng;  // grains
  cudaStream_t st = h->eng->st;
  CK(cudaSetDevice(h->eng->dev));
  const unsigned blocks = (unsigned)((n + 255) / 256);
  if (h->g.precision == MRM_FP64)
    state_out_kernel<double><<<blocks, 256, 0, st>>>(static_cast<const V4<double>*>(src),
                                                      static_cast<double*>(h->xfer), n, b.gci, b.gcs);
  else
    state_out_kernel<float><<<blocks, 256, 0, st>>>(static_cast<const V4<float>*>(src),
                                                     static_cast<double*>(h->xfer), n, b.gci, b.gcs);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, h->xfer, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MRM_OK;
}

int mrm_gpu_set_mag(mrm_gpu* h, int layer, const double* mag) {
  if (!h || !mag) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  if (layer < 0 || layer >= h->nl) return set_err(errp, MRM_ERR_ARG, "layer %d out of range", layer);
  const LayerBufs& b = h->L[layer];
  if (!b.uploaded) return set_err(errp, MRM_ERR_STATE, "upload layer %d first", layer);
  cudaStream_t st = h->eng->st;
  CK(cudaSetDevice(h->eng->dev));
  CK(cudaMemcpyAsync(h->xfer, mag, sizeof(double) * b.ng, cudaMemcpyHostToDevice, st));
  const unsigned blocks = (unsigned)((b.n + 255) / 256);
  if (h->g.precision == MRM_FP64)
    mag_in_kernel<double><<<blocks, 256, 0, st>>>(static_cast<const double*>(h->xfer), static_cast<V4<double>*>(b.m),
                                                  static_cast<V4<double>*>(b.mp), b.n, b.cgrain);
  else
    mag_in_kernel<float><<<blocks, 256, 0, st>>>(static_cast<const double*>(h->xfer), static_cast<V4<float>*>(b.m),
                                                 static_cast<V4<float>*>(b.mp), b.n, b.cgrain);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  return MRM_OK;
}

int mrm_gpu_get_mag(mrm_gpu* h, int layer, double* mag) {
  if (!h || !mag) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  if (layer < 0 || layer >= h->nl) return set_err(errp, MRM_ERR_ARG, "layer %d out of range", layer);
  const LayerBufs& b = h->L[layer];
  cudaStream_t st = h->eng->st;
  CK(cudaSetDevice(h->eng->dev));
  const unsigned blocks = (unsigned)((b.ng + 255) / 256);
  if (h->g.precision == MRM_FP64)
    mag_out_kernel<double><<<blocks, 256, 0, st>>>(static_cast<const V4<double>*>(b.m),
                                                   static_cast<double*>(h->xfer), b.ng, b.gci, b.gcs);
  else
    mag_out_kernel<float><<<blocks, 256, 0, st>>>(static_cast<const V4<float>*>(b.m), static_cast<double*>(h->xfer),
                                                  b.ng, b.gci, b.gcs);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(mag, h->xfer, sizeof(double) * b.ng, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
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
  h->t_acc = t;
  h->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_gpu_get_time(const mrm_gpu* h, double* t, int64_t* step) {
  if (!h) return MRM_ERR_ARG;
  if (t) *t = h->t_base + (double)(h->step - h->step_base) * h->dt;
  if (step) *step = h->step;
  return MRM_OK;
}

static void window_origin(const mrm_gpu* h, double t, int* i0, int* j0);
static int place_window(mrm_gpu* h, int i0, int j0);

int mrm_gpu_eval_field(mrm_gpu* h, double t, int layer, double* hdemag) {
  if (!h) return MRM_ERR_ARG;
  if (int rc = need_fft(h)) return rc;
  std::string* errp = &h->err;
  if (layer < 0 || layer >= h->nl) return set_err(errp, MRM_ERR_ARG, "layer %d out of range", layer);
  for (int l = 0; l < h->nl; ++l)
    if (!h->L[l].uploaded) return set_err(errp, MRM_ERR_STATE, "upload layer %d first", l);
  if (h->demag && !h->tensor_ready) return set_err(errp, MRM_ERR_STATE, "build or upload the tensor first (or disable demag)");
  Engine* e = h->eng;
  if (h->wnx) {  // the window where update_do_grain puts it at t
    int i0, j0;
    window_origin(h, t, &i0, &j0);
    int rc = place_window(h, i0, j0);
    if (rc) return rc;
  }
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
  if (hdemag) {
    return get_v4(h, layer, h->L[layer].hd, hdemag);
  }
  CK(cudaStreamSynchronize(e->st));
  return MRM_OK;
}

// update_do_grain (data.f90:120-135) with get_window (:52-64): the window
// origin (0-based cell offsets) at time t
static void window_origin(const mrm_gpu* h, double t, int* i0, int* j0) {
  // off = v t + offset rounded as two operations (no fused multiply-add), so
  // that a half-cell tie in nint falls the same way on every build
  volatile double vtx = h->wvx * t, vty = h->wvy * t;
  const double offx = vtx + h->wox, offy = vty + h->woy;
  const int nx = h->g.nx, ny = h->g.ny;
  *i0 = std::max(1, std::min(nx - h->wnx + 1, (int)std::lround((nx - h->wnx) * 0.5 + offx / h->g.dx))) - 1;
  *j0 = std::max(1, std::min(ny - h->wny + 1, (int)std::lround((ny - h->wny) * 0.5 + offy / h->g.dy))) - 1;
}

// Moves the window to (i0, j0): the grains now inside are the do_grain ones;
// every grain's other buffer takes its current state (data.f90:139), the
// spectrum is re-formed over the new window, and the frozen grains' stats
// records are taken (they stay fixed until the window moves again).
static int place_window(mrm_gpu* h, int i0, int j0) {
  std::string* errp = &h->err;
  Engine* e = h->eng;
  if (i0 == h->wi0 && j0 == h->wj0 && h->spec_valid) return MRM_OK;
  h->wi0 = i0;
  h->wj0 = j0;
  h->spec_valid = false;
  e->desc_dirty = true;
  int rc = e->prec == MRM_FP64 ? ensure_ready<double>(e) : ensure_ready<float>(e);
  if (rc) {
    h->err = e->err;
    return rc;
  }
  const long long n = (long long)h->g.nx * h->g.ny;
  const unsigned gx = (unsigned)std::min<long long>((n + 255) / 256, 4096);
  if (e->prec == MRM_FP64) {
    window_copy_kernel<double><<<dim3(gx, h->nl), 256, 0, e->st>>>(static_cast<const RunDev<double>*>(e->d_runs),
                                                                   h->slot);
    frozen_stats_kernel<double><<<h->nl, 256, 0, e->st>>>(static_cast<const RunDev<double>*>(e->d_runs), h->slot,
                                                          e->d_part);
  } else {
    window_copy_kernel<float><<<dim3(gx, h->nl), 256, 0, e->st>>>(static_cast<const RunDev<float>*>(e->d_runs),
                                                                  h->slot);
    frozen_stats_kernel<float><<<h->nl, 256, 0, e->st>>>(static_cast<const RunDev<float>*>(e->d_runs), h->slot,
                                                         e->d_part);
  }
  CK(cudaGetLastError());
  return MRM_OK;
}

// a grid whose own FFT exceeds the path's limits computes through a window only
static int need_fft(mrm_gpu* h) {
  if (h->fft_big && !h->wnx)
    return set_err(&h->err, MRM_ERR_UNSUPPORTED,
                   "the grid's FFT (%d x %d) exceeds the path's limits: set a moving demag window", h->px, h->py);
  return MRM_OK;
}

static int plain_prepare(mrm_gpu* h, int nsteps, double dt, int llg_type) {
  std::string* errp = &h->err;
  if (int rc = need_fft(h)) return rc;
  if (nsteps < 0) return set_err(errp, MRM_ERR_ARG, "nsteps must be >= 0");
  if (!(dt > 0)) return set_err(errp, MRM_ERR_ARG, "dt must be > 0");
  if (!llg_type_ok(llg_type))
    return set_err(errp, MRM_ERR_UNSUPPORTED,
                   "llg_type %d: this path has Heun (-3), the semi-implicit pushes (2, -2) and the "
                   "analytic rotations (1, -1)",
                   llg_type);
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
  if (nsteps > 0 && h->wnx) {
    // llg() calls update_do_grain(t) before its loop and after every step
    // (llg.f90:138,284): the steps go in runs over which the window stays put
    int left = nsteps;
    double t = h->t_acc;
    while (left > 0) {
      int i0, j0;
      window_origin(h, t, &i0, &j0);
      rc = place_window(h, i0, j0);
      if (rc) return rc;
      double tn = t + h->dt;  // the time after each further step, accumulated
      int k = 1;
      for (; k < left; ++k) {
        int a, b;
        window_origin(h, tn, &a, &b);
        if (a != i0 || b != j0) break;
        tn += h->dt;
      }
      rc = engine_step(h->eng, k, llg_type);
      if (rc) {
        h->err = h->eng->err;
        return rc;
      }
      t = tn;
      left -= k;
    }
    h->t_acc = t;
    h->has_stats = true;
    return MRM_OK;
  }
  if (nsteps > 0) {
    rc = engine_step(h->eng, nsteps, llg_type);
    if (rc) {
      h->err = h->eng->err;
      return rc;
    }
    for (int k = 0; k < nsteps; ++k) h->t_acc += h->dt;
    h->has_stats = true;
  }
  return MRM_OK;
}

int mrm_gpu_set_window(mrm_gpu* h, int nx_win, int ny_win, double vx, double vy, double offset_x, double offset_y) {
  if (!h) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  Engine* e = h->eng;
  if (!h->own_engine || e->runs.size() != 1)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "a moving demag window runs on a handle of its own, not in a batch");
  if (nx_win < 2 || ny_win < 2 || nx_win > h->g.nx || ny_win > h->g.ny)
    return set_err(errp, MRM_ERR_ARG, "window %d x %d outside 2 .. %d x %d", nx_win, ny_win, h->g.nx, h->g.ny);
  const bool none = nx_win == h->g.nx && ny_win == h->g.ny;  // update_do_grain: the whole grid (data.f90:127)
  if (none && h->fft_big)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "the grid's own FFT exceeds the path's limits: keep a window");
  mrm_geom gw = h->g;
  gw.nx = nx_win;
  gw.ny = ny_win;
  int rc = validate_geom(&gw, errp);
  if (rc) return rc;
  for (int l = 0; l < h->nl; ++l)
    if (h->L[l].cgrain) return set_err(errp, MRM_ERR_UNSUPPORTED, "a moving demag window needs one grain per cell");
  CK(cudaSetDevice(e->dev));
  CK(cudaStreamSynchronize(e->st));
  dfree(h->spech);
  dfree(h->specx);
  tensor_release(h);
  h->wnx = none ? 0 : nx_win;
  h->wny = none ? 0 : ny_win;
  h->wvx = vx;
  h->wvy = vy;
  h->wox = offset_x;
  h->woy = offset_y;
  h->wi0 = h->wj0 = -1;
  fft_grid(none ? h->g : gw, &h->px, &h->py);
  h->lgpx = ilog2(h->px);
  h->lgpy = ilog2(h->py);
  rc = spectra_alloc(h);
  if (!rc) rc = tensor_alloc(h);
  if (rc) return rc;
  h->tensor_ready = false;  // the window's tensor: build or upload it again
  h->spec_valid = false;
  e->tables_dirty = true;
  e->desc_dirty = true;
  return MRM_OK;
}

int mrm_gpu_get_window(const mrm_gpu* h, int* out4) {
  if (!h || !out4) return MRM_ERR_ARG;
  out4[0] = h->wnx ? h->wnx : h->g.nx;
  out4[1] = h->wnx ? h->wny : h->g.ny;
  out4[2] = out4[3] = 0;
  // where update_do_grain puts it at the handle's time (after the last step)
  if (h->wnx) window_origin(h, h->t_acc, &out4[2], &out4[3]);
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
  if (check_device_error(e)) {
    h->err = e->err;
    return MRM_ERR_DEVICE;
  }
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
  if (check_device_error(h->eng)) {
    h->err = h->eng->err;
    return MRM_ERR_DEVICE;
  }
  return MRM_OK;
}

// The reference's adaptive-dt loop (llg.f90:240-269 with get_fields :363-388 and
// push_m :1203-1270), driven from the host one step at a time: field at t,
// dt from the largest |h + hthm/sqrt(dt_prev)|, then the step at
// dt*max_dmdt, retried from the saved state with a smaller max_dmdt while a
// layer rotates further than max_dm.
int mrm_gpu_step_adaptive(mrm_gpu* h, int nsteps, int llg_type, double dt_frac, double dt_max,
                          const double* max_dm, double* dt, double* max_dmdt, mrm_gpu_stats* out) {
  if (!h || !max_dm || !dt || !max_dmdt) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  if (nsteps < 1) return set_err(errp, MRM_ERR_ARG, "nsteps must be >= 1");
  if (!(dt_frac > 0) || !(dt_max > 0) || !(*dt > 0) || !(*max_dmdt > 0))
    return set_err(errp, MRM_ERR_ARG, "adaptive steps need dt_frac, dt_max, dt and max_dmdt > 0");
  for (int l = 0; l < h->nl; ++l)
    if (!(max_dm[l] > 0)) return set_err(errp, MRM_ERR_ARG, "max_dm[%d] must be > 0", l);
  Engine* e = h->eng;
  if (e->runs.size() != 1)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "adaptive steps run on a handle of its own, not in a batch");
  if (h->wnx) return set_err(errp, MRM_ERR_UNSUPPORTED, "adaptive steps with a moving demag window");
  for (int l = 0; l < h->nl; ++l)
    if (h->L[l].llb) return set_err(errp, MRM_ERR_UNSUPPORTED, "adaptive steps with the LLB integrator");
  int rc = plain_prepare(h, 0, h->dt, llg_type);
  if (rc) return rc;
  const size_t re = relem(h->g.precision), n = (size_t)h->g.nx * h->g.ny;
  void* save = nullptr;
  unsigned long long* d_hm = nullptr;
  rc = dmalloc(errp, &save, (size_t)h->nl * n * 4 * re);
  if (!rc) rc = dmalloc(errp, (void**)&d_hm, sizeof(unsigned long long) * MRM_MAX_LAYERS);
  auto finish = [&](int code) {
    dfree(save);
    dfree(d_hm);
    return code;
  };
  if (rc) return finish(rc);
  mrm_gpu_stats st;
  for (int it = 0; it < nsteps; ++it) {
    const double t0 = h->t_base + (double)(h->step - h->step_base) * h->dt;
    const long long s0 = h->step;
    // get_fields: h at t, then dt from the largest |h + hthm*dti| (llg.f90:369-387)
    rc = mrm_gpu_eval_field(h, t0, 0, nullptr);
    if (rc) return finish(rc);
    const double dti = 1.0 / std::sqrt(*dt * *max_dmdt);
    unsigned long long hm[MRM_MAX_LAYERS];
    if (cudaMemsetAsync(d_hm, 0, sizeof(hm), e->st) != cudaSuccess) return finish(set_err(errp, MRM_ERR_CUDA, "memset"));
    for (int l = 0; l < h->nl; ++l) {
      const unsigned blocks = (unsigned)((n + 255) / 256);
      if (e->prec == MRM_FP64)
        hmag_kernel<double><<<blocks, 256, 0, e->st>>>(static_cast<const RunDev<double>*>(e->d_runs), h->slot, l, dti,
                                                       s0, d_hm + l);
      else
        hmag_kernel<float><<<blocks, 256, 0, e->st>>>(static_cast<const RunDev<float>*>(e->d_runs), h->slot, l, dti,
                                                      s0, d_hm + l);
    }
    if (cudaMemcpyAsync(hm, d_hm, sizeof(hm), cudaMemcpyDeviceToHost, e->st) != cudaSuccess ||
        cudaStreamSynchronize(e->st) != cudaSuccess)
      return finish(set_err(errp, MRM_ERR_CUDA, "field magnitude: %s", cudaGetErrorString(cudaGetLastError())));
    double ndt = 1e22;
    for (int l = 0; l < h->nl; ++l) {
      long long bits = (long long)hm[l];
      double hmag = 0.0;
      std::memcpy(&hmag, &bits, sizeof(hmag));
      hmag = std::sqrt(hmag);
      const LayerBufs& b = h->L[l];
      const double fact1 = (1.0 + b.alpha * b.alpha) / ((1.0 + b.alpha) * b.gamma) * dt_frac;
      ndt = std::min(ndt, std::min(dt_max, fact1 / std::max(1.0, hmag)));
    }
    *dt = ndt;
    // push_m: the step at dt*max_dmdt, retried from the saved state (llg.f90:1205-1238)
    for (int l = 0; l < h->nl; ++l)
      if (cudaMemcpyAsync(static_cast<char*>(save) + l * n * 4 * re, h->L[l].m, n * 4 * re, cudaMemcpyDeviceToDevice,
                          e->st) != cudaSuccess)
        return finish(set_err(errp, MRM_ERR_CUDA, "state copy"));
    double next = 1e22;
    for (int attempt = 0;; ++attempt) {
      if (attempt > 200) return finish(set_err(errp, MRM_ERR_DEVICE, "adaptive step: no accepted step after 200 retries"));
      const double dts = *dt * *max_dmdt;
      rc = mrm_gpu_step(h, 1, dts, llg_type, &st);
      if (rc) return finish(rc);
      bool too_far = false;
      next = 1e22;
      for (int l = 0; l < h->nl; ++l) {
        const double r = std::acos(1.0 - 0.5 * st.errmx1_l[l]) / max_dm[l];
        if (r > 1.0) {
          *max_dmdt = 0.9 * *max_dmdt / r;
          too_far = true;
          break;
        }
        next = std::min(next, r < 2.0 / 3.0 ? std::min(2.0, *max_dmdt / (r + 1e-200)) : *max_dmdt);
      }
      if (!too_far) break;
      // back to the state and time before the attempt
      for (int l = 0; l < h->nl; ++l)
        if (cudaMemcpyAsync(h->L[l].m, static_cast<char*>(save) + l * n * 4 * re, n * 4 * re,
                            cudaMemcpyDeviceToDevice, e->st) != cudaSuccess)
          return finish(set_err(errp, MRM_ERR_CUDA, "state copy"));
      h->t_base = t0;
      h->step_base = s0;
      h->step = s0;
      h->spec_valid = false;
      e->desc_dirty = true;
      e->pred_stored = true;  // the retry's predictor takes the rejected attempt's corrector field
    }
    if (next > 1e20) next = *max_dmdt;
    *dt = *dt * *max_dmdt;  // llg.f90:268
    *max_dmdt = next;
  }
  h->t_acc = h->t_base + (double)(h->step - h->step_base) * h->dt;  // (no window here)
  if (out) *out = st;
  return finish(MRM_OK);
}

int mrm_gpu_set_shape(mrm_gpu* h, int row_shape, int col_shape, int cols_per_task) {
  if (!h) return MRM_ERR_ARG;
  Engine* e = h->eng;
  const bool f64 = e->prec == MRM_FP64;
  const int nrv = f64 ? row_variant_count<double>() : row_variant_count<float>();
  const int ncv = f64 ? col_variant_count<double>() : col_variant_count<float>();
  if (row_shape < 0 || col_shape < 0) {
    e->shape_forced = false;
  } else {
    if (row_shape >= nrv || col_shape >= ncv)
      return set_err(&h->err, MRM_ERR_ARG, "shape (%d, %d) outside %d row / %d column shapes", row_shape,
                     col_shape, nrv, ncv);
    e->shape_forced = true;
    e->force_rowv = row_shape;
    e->force_colv = col_shape;
    e->force_cpt = std::max(0, cols_per_task);
  }
  e->tables_dirty = true;
  return MRM_OK;
}

int mrm_gpu_set_autotune(mrm_gpu* h, int on) {
  if (!h) return MRM_ERR_ARG;
  h->eng->autotune = on != 0;
  h->eng->tables_dirty = true;
  return MRM_OK;
}

int mrm_gpu_selftest_timeout(mrm_gpu* h) {
  if (!h) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  for (int l = 0; l < h->nl; ++l)
    if (!h->L[l].uploaded) return set_err(errp, MRM_ERR_STATE, "upload layer %d first", l);
  if (h->demag && !h->tensor_ready) return set_err(errp, MRM_ERR_STATE, "build or upload the tensor first (or disable demag)");
  Engine* e = h->eng;
  CK(cudaSetDevice(e->dev));
  int rc = check_device_error(e);  // an earlier failure is reported as such
  if (rc) {
    h->err = e->err;
    return rc;
  }
  rc = e->prec == MRM_FP64 ? ensure_ready<double>(e) : ensure_ready<float>(e);
  if (!rc) {
    cudaError_t ce = e->prec == MRM_FP64 ? launch_row_e<double>(e, kEval, false, 0, kFlagForce | kFlagProbeTimeout)
                                         : launch_row_e<float>(e, kEval, false, 0, kFlagForce | kFlagProbeTimeout);
    if (ce != cudaSuccess) rc = set_err(&e->err, MRM_ERR_CUDA, "self-test launch: %s", cudaGetErrorString(ce));
  }
  if (!rc) rc = check_device_error(e);
  if (rc) h->err = e->err;
  return rc;
}

int mrm_gpu_check_device(mrm_gpu* h) {
  if (!h) return MRM_ERR_ARG;
  int rc = check_device_error(h->eng);
  if (rc) h->err = h->eng->err;
  return rc;
}

int mrm_gpu_get_shape(const mrm_gpu* h, int* out3) {
  if (!h || !out3) return MRM_ERR_ARG;
  out3[0] = h->eng->rowv;
  out3[1] = h->eng->colv;
  out3[2] = h->eng->cpt;
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
    CK(launch_row_e<R>(e, kPred, false, 0, 0));
    CK(cudaEventRecord(ev[5 * s + 1], e->st));
    CK(launch_col_e<R>(e, 0, 0));
    CK(cudaEventRecord(ev[5 * s + 2], e->st));
    CK(launch_row_e<R>(e, kCorr, false, 0, 0));
    CK(cudaEventRecord(ev[5 * s + 3], e->st));
    CK(launch_col_e<R>(e, 0, 0));
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
  release_retired(&b->eng);
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
  // the frees wait for the next stats / step / destroy: a server removes
  // finished runs between two calls, and their frees then overlap the next
  // call instead of holding the device idle
  run->slot = -1;
  b->eng.retired.push_back(run);
  b->eng.tables_dirty = true;
  b->eng.desc_dirty = true;
  return MRM_OK;
}

int mrm_batch_adopt(mrm_batch* dst, mrm_batch* src, mrm_gpu* run) {
  if (!dst || !src || !run || run->eng != &src->eng) return MRM_ERR_ARG;
  if (dst == src) return MRM_OK;
  Engine* d = &dst->eng;
  Engine* s = &src->eng;
  std::string* errp = &d->err;
  if (d->prec != s->prec || d->dev != s->dev)
    return set_err(errp, MRM_ERR_ARG, "adopt: the batches differ in precision or device");
  CK(cudaSetDevice(d->dev));
  CK(cudaStreamSynchronize(s->st));  // the run's uploads and tensor build
  CK(cudaStreamSynchronize(d->st));  // the tables below change at the next call
  auto& v = s->runs;
  v.erase(std::remove(v.begin(), v.end(), run), v.end());
  s->tables_dirty = true;
  s->desc_dirty = true;
  run->eng = d;
  run->slot = -1;
  d->runs.push_back(run);
  d->tables_dirty = true;
  d->desc_dirty = true;
  return MRM_OK;
}

int mrm_batch_set_run(mrm_gpu* run, double dt, int64_t step_end, int active) {
  if (!run) return MRM_ERR_ARG;
  if (!(dt > 0)) return set_err(&run->err, MRM_ERR_ARG, "dt must be > 0");
  if (dt != run->dt) {
    // rebase the time at the run's next executed step (a delayed run's step
    // counter sits below it)
    const long long at = std::max(run->step, run->step_begin);
    run->t_base = run->t_base + (double)(at - run->step_base) * run->dt;
    run->step_base = at;
    run->dt = dt;
  }
  run->step_end = step_end;
  run->active = active != 0;
  run->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_batch_delay_run(mrm_gpu* run, int64_t idle_steps) {
  if (!run) return MRM_ERR_ARG;
  if (idle_steps < 0) return set_err(&run->err, MRM_ERR_ARG, "idle_steps must be >= 0");
  if (run->step < run->step_begin) return set_err(&run->err, MRM_ERR_ARG, "the run is already delayed");
  // the step counter moves back by idle_steps and the run idles until it is
  // back at its current step: state, time and thermal counters are unchanged
  run->step_begin = run->step;
  run->step -= idle_steps;
  run->eng->desc_dirty = true;
  return MRM_OK;
}

int mrm_batch_enqueue(mrm_batch* b, int nsteps, int llg_type) {
  if (!b) return MRM_ERR_ARG;
  Engine* e = &b->eng;
  std::string* errp = &e->err;
  if (!llg_type_ok(llg_type))
    return set_err(errp, MRM_ERR_UNSUPPORTED, "llg_type %d: this path has -3, -2, 2, -1 and 1", llg_type);
  for (auto* r : e->runs) {
    if (!r->active) continue;
    for (int l = 0; l < r->nl; ++l)
      if (!r->L[l].uploaded) return set_err(errp, MRM_ERR_STATE, "a run has layer %d not uploaded", l);
    if (r->demag && !r->tensor_ready) return set_err(errp, MRM_ERR_STATE, "a run has no tensor");
  }
  if (nsteps <= 0) return MRM_OK;
  return engine_step(e, nsteps, llg_type);
}

int mrm_batch_step(mrm_batch* b, int nsteps, int llg_type) {
  int rc = mrm_batch_enqueue(b, nsteps, llg_type);
  if (rc) return rc;
  std::string* errp = &b->eng.err;
  CK(cudaStreamSynchronize(b->eng.st));
  release_retired(&b->eng);
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
  // the slots of the tables the last steps ran with (runs added since then
  // have none yet)
  const int nr = e->nslots;
  CK(cudaSetDevice(e->dev));
  // removed runs: no work in flight reads them (they left the tables before
  // it was enqueued), and their frees overlap it
  release_retired(e);
  if (!nr) return MRM_OK;
  CK(cudaMemcpyAsync(e->h_stats, e->d_stats, sizeof(StatsDev) * nr, cudaMemcpyDeviceToHost, e->st));
  CK(cudaStreamSynchronize(e->st));
  if (check_device_error(e)) return MRM_ERR_DEVICE;
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
  if (!e->tables_dirty) {
    CK(row_occupancy<R>(e->rowv, kPred, e->smem_row[1], &a));
    // the column kernel of most of the batch's column tasks
    if (e->nct2 > e->nct) CK(creg_occupancy(creg_v(e), e->smem_creg, &b));
    else CK(col_occupancy<R>(e->colv, e->smem_col, &b));
  }
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

// (kernel parameter blocks hold up to 32,764 bytes from CUDA 12.1 on sm_70 and later)
static_assert(sizeof(RunDev<float>) <= 32000, "run descriptor must fit in a kernel parameter block");

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
  const size_t n = (size_t)r->g.nx * r->g.ny;
  const size_t grains = (size_t)r->nl * n * sizeof(V4<float>);
  o.desc = take(sizeof(RunDev<float>));
  o.rtask = take(sizeof(Task) * nrt);
  o.ctask = take(sizeof(Task) * nct);
  o.m = take(grains);
  o.hd = take(grains);
  o.hf = take(grains);
  o.specx = take(specx_count(r) * sizeof(Cx<float>));
  o.spech = take((size_t)r->nl * 3 * r->g.ny * spec_row_stride(r->px) * sizeof(Cx<float>));
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

// Once per device, with that device current: the scratch address, and the
// kernels of the call loaded (CUDA lazy loading would otherwise load them,
// and allocate their code, at their first launch) with their shared-memory
// limits raised to the device's maximum.  Runs inside the first call on the
// device.
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
  CK(row_load<float>(0));
  CK(col_load<float>(0));
  CK(creg_load(0));
  size_t lim[kSlots];
  for (int q = 0; q < kSlots; ++q) lim[q] = (size_t)optin - row_static_bytes(q);
  CK(row_allow_smem<float>(0, lim));
  CK(col_allow_smem<float>(0, (size_t)optin - 64));
  CK(creg_allow_smem(0, (size_t)optin - 64));
  cudaFuncAttributes fa;
  CK(cudaFuncGetAttributes(&fa, noalloc_pack_kernel));
  CK(cudaFuncGetAttributes(&fa, noalloc_unpack_kernel));
  s.base = static_cast<unsigned char*>(p);
  s.ready = true;
  *base = s.base;
  return MRM_OK;
}

}  // namespace

extern "C" {

int mrm_gpu_demag_noalloc(mrm_gpu* h, const float* m, float* hdemag, void* stream) {
  if (!h) return MRM_ERR_ARG;
  std::string* errp = &h->err;
  if (!m || !hdemag) return set_err(errp, MRM_ERR_ARG, "m and hdemag must be device pointers");
  if (h->g.precision != MRM_FP32)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "the allocation-free demag evaluation takes MRM_FP32 handles");
  if (h->wnx || h->fft_big)
    return set_err(errp, MRM_ERR_UNSUPPORTED, "the allocation-free demag evaluation has no moving window");
  for (int l = 0; l < h->nl; ++l)
    if (h->L[l].cgrain)
      return set_err(errp, MRM_ERR_UNSUPPORTED, "the allocation-free demag evaluation takes one grain per cell");
  const int nl = h->nl, ny = h->g.ny, ph = h->px / 2 + 1;
  const int rpt = 1, nrt = nl * ny;  // one row per task (row shape 0)
  const bool creg = creg_run(h);
  const int cpt = creg ? creg_cols(h->lgpy, kCreg[0].block) : col_tile(default_cols(h)), nct = (ph + cpt - 1) / cpt;
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
  d.lgct = ilog2(cpt);
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
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : e->st;
  const long long work = std::max<long long>(ntot, std::max(nrt, nct));
  // shared memory: FFT part plus grain staging where it fits
  const size_t fft = row_fixed_smem<float>(h, 1);
  auto stage_cap = [&](int stage, int slot) {
    const long long hard = (long long)kMaxSmem - (long long)row_static_bytes(slot) - (long long)fft;
    return (int)(std::min<long long>(run_stage_bytes<float>(h, stage, rpt), std::max(0LL, hard)) & ~15LL);
  };
  const int cap_init = stage_cap(kInit, 0), cap_eval = stage_cap(kEval, 4);

  noalloc_pack_kernel<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(d, desc, rt, nrt, rpt, ct, nct, cpt, m, sm,
                                                                      ntot);
  // kInit reads the descriptor and tasks before its dependency wait: a plain
  // launch, so it cannot overlap their writer; the rest chain with
  // programmatic serialization as in the engine
  bool head = false;
  for (int l = 0; l < nl; ++l) head = head || h->L[l].func == kFuncHead;
  CK(launch_row<float>(0, kInit, false,
                       RowLaunch{st, desc, rt, e->d_tw, nullptr, e->d_err, nrt, fft + cap_init, cap_init, false, head},
                       0, kFlagForce));
  if (creg) {
    ColLaunch a{st, desc, ct, e->d_tw, e->d_err, nct,
                (size_t)creg_smem(col_tw_count(h->lgpy), kCreg[0].block,
                                  creg_stage_bytes(spec_col_stride(ny), ilog2(cpt))),
                true};
    a.tw_cap = col_tw_count(h->lgpy);
    CK(launch_creg(0, a, 0, kFlagForce));
  }
  else
    CK(launch_col<float>(0, ColLaunch{st, desc, ct, e->d_tw, e->d_err, nct, col_smem_of<float>(h, cpt, col_variant<float>(0).minb), true}, 0,
                         kFlagForce));
  CK(launch_row<float>(0, kEval, false,
                       RowLaunch{st, desc, rt, e->d_tw, nullptr, e->d_err, nrt, fft + cap_eval, cap_eval, true, head},
                       0, kFlagForce | kFlagStoreField));
  noalloc_unpack_kernel<<<(unsigned)((ntot + 255) / 256), 256, 0, st>>>(shd, hdemag, ntot);
  CK(cudaGetLastError());
  return MRM_OK;
}

}  // extern "C"
