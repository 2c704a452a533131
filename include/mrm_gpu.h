/*
 * mrm_gpu.h -- C ABI of the B200 grain-dynamics path.
 *
 * Drop-in for the per-timestep body of mrm's llg() loop: push_m and the
 * get_field calls it makes (src/llg.f90:212-285, :1195-1271), i.e. the
 * stochastic LLG integrator plus the effective-field assembly
 * (src/field.f90:160-273, :326-436), the demag FFT convolution
 * (src/demag.f90:33-135, src/fftw.f90:37-93) and the magnetostatic tensor
 * (src/tensor.f90:82-216, src/tensor_element.f90:13-102,219-261).
 *
 * Conventions follow the reference's data layout (src/data.f90:91-104):
 *   - per-grain vectors are AoS (3,N) like the Fortran m(1+in:3+in,:),
 *     h(3,:), uni_axis(3,:), hk(2,:) arrays, passed as contiguous doubles;
 *   - CSR index arrays are the Fortran (0:N) arrays (N+1 cumulative counts
 *     starting at 0); neighbour / cell coordinates are 1-based as in Fortran;
 *   - the real-space tensor is Fortran n2d(nx,ny,9,n_lay,n_lay) (observation
 *     layer 4th, source layer 5th), including the 1/(dx dy dz nx ny)
 *     normalisation of tensor.f90:183;
 *   - every function returns an int status (0 = MRM_OK), mapped to the
 *     reference's logical ok_p by the Fortran shim; mrm_gpu_last_error()
 *     gives the message.  Device-side failures come back as status codes,
 *     never as traps.
 * Ownership: the caller owns every host array; the library copies on
 * upload/download and keeps no host pointer.  A handle is not thread-safe
 * (neither were the FFTW plans it replaces, src/demag.f90:256).
 */
#ifndef MRM_GPU_H
#define MRM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MRM_MAX_LAYERS 8

enum {
  MRM_OK = 0,
  MRM_ERR_ARG = 1,          /* invalid argument / size */
  MRM_ERR_CUDA = 2,         /* CUDA runtime error */
  MRM_ERR_UNSUPPORTED = 3,  /* valid reference input this path does not cover */
  MRM_ERR_STATE = 4,        /* call order (e.g. stepping before upload) */
  MRM_ERR_NOMEM = 5,        /* device memory exhausted */
  MRM_ERR_DEVICE = 6        /* kernel-reported error status */
};

enum { MRM_PERIODIC = 0, MRM_OPEN = 1 };
enum { MRM_FP32 = 0, MRM_FP64 = 1 };

/* Geometry of one medium (src/data.f90:87-89 + the demag namelist,
 * src/input.f90:221-246).  boundary MRM_PERIODIC reproduces the reference's
 * periodic tensor with num_images image pairs (tensor.f90:6,96-97);
 * MRM_OPEN zero-pads the FFT grid to the next power of two >= 2n in each
 * direction and builds the tensor on it without images. */
typedef struct mrm_geom {
  int32_t nx, ny, n_lay;
  int32_t boundary;
  int32_t num_images;
  int32_t precision; /* MRM_FP32: FP32 state/field/FFT, FP64 tensor + reductions;
                        MRM_FP64: everything FP64 */
  double dx, dy;     /* cm */
  double dz[MRM_MAX_LAYERS];
  double il_space[MRM_MAX_LAYERS];
  double space_to_sul, sul_mu, head_mu, fly_height; /* tensor.f90:9 image settings */
} mrm_geom;

/* Per-call results, FP64 (llg.f90:217-237 reductions, push_llg errmx/errmx1/mmag,
 * plot.f90:192-273 M(H) row).  Values describe the state after the last step:
 * mave/mvar/have are the volume-weighted <m>, var(m), <h> the reference's loop
 * computes at the top of its next iteration; mms_l is plot_mh's Ms*V-weighted
 * m; nup_l counts grains with m.h_dir > 0 (N+). */
typedef struct mrm_gpu_stats {
  double t;
  int64_t step;
  double mave[3], mvar[3], have[3];
  double errmx;  /* sqrt(max |m x H|^2/Ms^2) of the last stage */
  double errmx1; /* max |dm|^2 of the last stage */
  double mmag;   /* sum over layers of sum |m| ms_scale V / sum V */
  double energy; /* sum V * energy density of the last field evaluation (erg) */
  double mave_l[MRM_MAX_LAYERS][3], mvar_l[MRM_MAX_LAYERS][3];
  double have_l[MRM_MAX_LAYERS][3], mms_l[MRM_MAX_LAYERS][3];
  double vol_l[MRM_MAX_LAYERS], msvol_l[MRM_MAX_LAYERS];
  int64_t nup_l[MRM_MAX_LAYERS];
  double errmx1_l[MRM_MAX_LAYERS]; /* max |dm|^2 of the last stage per layer */
} mrm_gpu_stats;

typedef struct mrm_gpu mrm_gpu;     /* one medium realisation (a "run") */
typedef struct mrm_batch mrm_batch; /* many runs advanced by one launch sequence */

/* ---------------- plain single-run path (the drop-in) ---------------- */

/* Allocates a run on `device` (replaces start_demag/init_demag set-up,
 * src/demag.f90:184-286, and the data_m allocations). */
int mrm_gpu_create(const mrm_geom* geom, int device, mrm_gpu** out);
int mrm_gpu_destroy(mrm_gpu* h);
const char* mrm_gpu_last_error(const mrm_gpu* h);

/* Static grain data of one layer (0-based `layer`; Fortran layer k -> k-1).
 * Arrays as data_s/field_ss: ms(N), grain_vol(N), uni_axis(3,N), hk(2,N),
 * hk_scale/ms_scale/alpha_scale(N); alpha, gamma, floor_ms scalars;
 * grain2gridindex(0:N), grain2grid(2,ncell) (field.f90:22-23); intralayer
 * exchange hxgrainindex(0:N), hxgrain(nnz), hx(nnz) (field.f90:28-29), or
 * NULL for none.  One cell per grain in grid order (grains are nodes,
 * construct_grain.f90:160-189) runs the fused path; any other map (grains
 * of several cells, empty cells; each cell in at most one grain) runs the
 * grain-averaged form of get_mag / get_magnetostatic (data.f90:322-390,
 * field.f90:438-517): two more launches per stage (the cells' demag and its
 * grain average).  The state, field and demag arrays of the other calls stay
 * per grain.  A write head needs one grain per cell. */
int mrm_gpu_upload_layer(mrm_gpu* h, int layer, int n_grains, const double* ms,
                         const double* grain_vol, const double* uni_axis, const double* hk,
                         const double* hk_scale, const double* ms_scale,
                         const double* alpha_scale, double alpha, double gamma, double floor_ms,
                         const int32_t* grain2gridindex, const int32_t* grain2grid,
                         const int32_t* hxgrainindex, const int32_t* hxgrain, const double* hx);

/* Interlayer exchange CSR of `layer`: side 0 = uhx (couples to layer-1),
 * side 1 = lhx (couples to layer+1) (field.f90:211-220, :326-348). */
int mrm_gpu_upload_interlayer(mrm_gpu* h, int layer, int side, const int32_t* index,
                              const int32_t* grain, const double* coef);

/* Builds the FP64 tensor on the device (calculate_tensor + the once-per-run
 * FFT of demag.f90:259-267, in FP64) and keeps its spectrum resident. */
int mrm_gpu_build_tensor(mrm_gpu* h);
/* Uses a tensor computed by the host (calculate_tensor's n2d or mrm_N.dat)
 * for an FFT grid of nx_fft x ny_fft (must equal the handle's FFT grid). */
int mrm_gpu_upload_tensor(mrm_gpu* h, const double* n2d, int nx_fft, int ny_fft);
/* Copies the device-built real-space tensor back (for the tensor cache file). */
int mrm_gpu_download_tensor(mrm_gpu* h, double* n2d);
/* Copies the resident tensor spectrum of `src` into `dst` (same device, FFT
 * grid, layer stack and precision): runs of one geometry share a tensor
 * without rebuilding it. */
int mrm_gpu_copy_tensor(mrm_gpu* dst, const mrm_gpu* src);
/* FFT grid of the handle (nx_fft, ny_fft). */
int mrm_gpu_fft_grid(const mrm_gpu* h, int* nx_fft, int* ny_fft);
/* Diagnostic of the packed tensor spectrum: largest dropped (wrong-parity)
 * part and largest kept value, FP64. */
int mrm_gpu_tensor_residual(const mrm_gpu* h, double* resid, double* kept);
/* demag_p of the demag namelist (src/input.f90:228); default on. */
int mrm_gpu_set_demag(mrm_gpu* h, int on);

/* Uniform applied field of `layer` with a linear time ramp:
 * h_app(t) = ((s_end-s_start)*clamp((t-t_start)/(t_end-t_start),0,1)+s_start)*scale*hdir
 * (set_fld / get_appl, src/applied.f90:263-317,871-883). */
int mrm_gpu_set_uniform_field(mrm_gpu* h, int layer, const double hdir[3], double t_start,
                              double t_end, double s_start, double s_end, double scale);

/* Uniform applied field of `layer` with a time function (set_fld with func1,
 * applied.f90:263-297,328-377,866-869):
 * h_app(t) = (amp*f(t) + dc)*scale*hdir, f = 1 sin(t*gamma+phase),
 * 2 cos(t*gamma+phase), 3 exp(t*gamma+phase), 4 STE (trapezoidal square wave
 * of period gamma and rise time param), 5 NEW (exponential pulse train),
 * 7 ROT (applied.f90:378-392 with the rotation angles given, |gamma| != 1):
 * f = 1 and hdir replaced by the in-plane direction
 * (cos((2 gamma t + phase) pi), sin((2 gamma t + phase) pi), 0); hdir still
 * defines N+ in the stats.  |gamma| = 1 (a field that follows the mean
 * magnetisation step by step) returns MRM_ERR_UNSUPPORTED. */
int mrm_gpu_set_field_function(mrm_gpu* h, int layer, const double hdir[3], int func, double amp,
                               double gamma, double phase, double param, double duty,
                               double moddepth, double dc, double scale);

/* Moving write head on `layer` (applied-field form 6; the reference has no
 * analytic head and drives writes with a tabulated moving field,
 * applied.f90:711-813,1471-1520): the 2-D Karlqvist field of a ring head with
 * gap `gap` (cm) whose gap centre sits at x0 + velocity*(t - t0) down-track
 * (+x, cm), at distance z (cm) from the layer's mid-plane, deep-gap field hg
 * (Oe):
 *   h_x = P hg/pi (atan((u + gap/2)/z) - atan((u - gap/2)/z)),
 *   h_z = P hg/(2 pi) ln(((u - gap/2)^2 + z^2) / ((u + gap/2)^2 + z^2)),
 * u = (i + 1/2) dx - gap centre for grain column i; write polarity P = +1 if
 * bit floor((t - t0)/bit_time) mod nbits of `pattern` is set (bit 0 first),
 * else -1.  Replaces the layer's uniform field. */
int mrm_gpu_set_head_field(mrm_gpu* h, int layer, double gap, double z, double hg, double velocity, double x0,
                           double t0, double bit_time, uint64_t pattern, int nbits);

/* Tabulated (moving) field profile on `layer` (file_applied + the moving
 * branch of get_appl + get_applied, applied.f90:711-813,896-903,1471-1520,
 * 1757-1776, field.f90:546-560): vfld(3, nfx, nfy) in Oe (Fortran order,
 * vfld[c + 3*(i + nfx*j)]) at ascending node positions xpos(nfx), ypos(nfy)
 * (cm, nfx, nfy >= 2).  At time t the grid cell (i, j) centre
 * ((i+1/2) dx, (j+1/2) dy) sits at table position
 *   x = (i+1/2) dx - (offset_x + vel_x (t - t_origin) - ref_x)   (y alike);
 * each axis takes the interval closed by the first node above x (from the
 * second node on, at most the last) with the lower node's weight
 * clamp((x_hi - x)/(x_hi - x_lo), 0, 1) (set); the cell's field is the
 * bilinear sum scaled by the layer's time scale s(t) (the linear ramp of
 * mrm_gpu_set_uniform_field or the function of mrm_gpu_set_field_function,
 * whose direction the profile replaces), and a grain's field the average over
 * its cells.  offset_x/offset_y below -1e200 take file_applied's default, the
 * grid centre (nx dx/2, ny dy/2).  nfx = nfy = 0 removes the profile.
 * Replaces a write head on the layer. */
int mrm_gpu_set_field_table(mrm_gpu* h, int layer, int nfx, int nfy, const double* xpos, const double* ypos,
                            const double* vfld, double vel_x, double vel_y, double offset_x, double offset_y,
                            double ref_x, double ref_y, double t_origin);

/* Moving super-Gaussian temperature profile on `layer` (HAMR: suprgaus_temp
 * and ref_temp, set_sg / get_sg, applied.f90:446-483,889-896,1778-1809; the
 * grain's temperature, field.f90:546-560):
 *   T(cell i, j; t) = background + s(t) dtemp fx(i) fy(j),
 *   fx(i) = exp(-(((i + 1/2) dx + ref_x - vel_x (t - t_origin) - offset_x)/sigma_x)^(2 expn))
 * (y alike; sigma 0: flat; offsets below -1e200: the grid centre), s(t) the
 * profile's time scale (mrm_gpu_set_temp_function; default 1).  The grain's
 * temperature replaces the layer's in the thermal variance, in the LLB / MT
 * pushes and in the layer's temperature scaling (mrm_gpu_set_temp_scaling).
 * One grain per cell.  expn < 0 removes it.
 * mrm_gpu_set_temp_function: s(t) = ((s_end - s_start) clamp((t - t_start) /
 * (t_end - t_start), 0, 1) + s_start) scale (func 0) or (amp f(t) + dc) scale
 * with f as in mrm_gpu_set_field_function (func 1..5). */
int mrm_gpu_set_temp_profile(mrm_gpu* h, int layer, double background, double dtemp, double sigma_x, double sigma_y,
                             int expn, double vel_x, double vel_y, double offset_x, double offset_y, double ref_x,
                             double ref_y, double t_origin);
int mrm_gpu_set_temp_function(mrm_gpu* h, int layer, int func, double t_start, double t_end, double s_start,
                              double s_end, double amp, double gamma, double phase, double param, double duty,
                              double moddepth, double dc, double scale);

/* Temperature scaling of Ms, alpha and Hk on `layer` (set_temp_scaling and
 * find_temp_scaling, temp_scaling.f90:37-50,365-433, applied at every field
 * evaluation by get_applied, field.f90:527-595): with x = T/Tc of the grain
 * (tc[n], field%tc; T its temperature at the evaluation),
 *   ms_scale = clamp(|m|, 0, 1) (use_mag, the LLB magnitude), else
 *              clamp(1 - x, 0, 1)^msexp (msexp >= 0), else the Ms table at x;
 *   alpha_scale = the alpha table at x;  hk_scale = clamp(1 - x, 0, 1)^hkexp
 *              (hkexp >= 0), else the Hk table at x;  a scale without a rule is 1.
 * They enter as the reference's ms_scale, alpha_scale and hk_scale do: the
 * demag source, the exchange terms (the neighbours' ms_scale), anisotropy,
 * damping, the thermal variance and the reductions.  The layer must have been
 * uploaded with unit scales (the reference's, which only this scaling
 * changes), with one grain per cell and no moving window
 * (MRM_ERR_STATE / MRM_ERR_UNSUPPORTED otherwise).  tc NULL switches it off.  (No reference
 * counterpart for the C form; the Fortran host calls it where it calls
 * set_temp_scaling / init_temp_scaling.)
 * mrm_gpu_set_temp_scaling_table: table `which` (1 Ms, 2 alpha, 3 Hk, 4 Hx)
 * from n (temperature, scale) pairs as file_temp_scaling reads them
 * (temp_scaling.f90:126-239), reduced as it reduces them (ordered, equal
 * temperatures merged, equal end scales trimmed, temperatures above 5 taken
 * as K and divided by the largest); a table of one node scales nothing; n = 0
 * removes it.  The Hx table is kept but, as in the reference, scales nothing.
 * mrm_gpu_get_temp_scaling_table: the reduced table (*n: room in, nodes out). */
int mrm_gpu_set_temp_scaling(mrm_gpu* h, int layer, const double* tc, double msexp, double hkexp, int use_mag);
int mrm_gpu_set_temp_scaling_table(mrm_gpu* h, int layer, int which, int n, const double* temp,
                                   const double* scaling);
int mrm_gpu_get_temp_scaling_table(const mrm_gpu* h, int layer, int which, int* n, double* temp, double* scaling);

/* LLB integrator (llgp%llb; push_llb, llg.f90:916-1064, Heun branch
 * :1000-1047 and the |m| = 0 branch :1048-1060) on `layer`: spin S, per grain
 * Curie temperature tc (K, > 0) and lambdaMs (Oe; lambda_m = lambdaMs (S+1)/S);
 * the layer's temperature (mrm_gpu_set_thermal, > 0), damping and gamma.  Each
 * grain carries a magnitude |m| (mag, 1 after mrm_gpu_set_state) beside its
 * direction; the thermal variance divides by max(floor_ms, |m|) once |m| != 1
 * (get_thermal, field.f90:416-417); the stats' mmag is sum |m| vol over the
 * pushed grains' volume.  llgp%llb is one switch for all layers: every layer of
 * the run must have it; llg_type -3 only.  tc = NULL turns it off.  Set it after
 * the layer's upload (an upload clears it).  mrm_gpu_set_mag / _get_mag: |m|
 * per grain (layer%mag(in, :)). */
int mrm_gpu_set_llb(mrm_gpu* h, int layer, double spin, const double* tc, const double* lambda_ms);
/* MT integrator (llgp%mt: push_mt, llg.f90:735-915, dm/dt = -gamma m x H -
 * (m - m_eq)/tau + eta, with |m| per grain as for LLB): spin S, per grain
 * lambdaMs (Oe), the equilibrium from the Brillouin function B_S (meq_bs = 1,
 * the mean field lambdaMs) or the Langevin function (meq_bs = 0, lambdaMs
 * (S+1)/S), tau from Xu & Zhang (garanin_tau = 0) or Garanin (1); Heun and the
 * semi-implicit |type| = 2 branch (llg_type -3, 2, -2); the same switch, checks
 * and magnitude accessors as the LLB integrator.  lambda_ms = NULL: off. */
int mrm_gpu_set_mt(mrm_gpu* h, int layer, double spin, const double* lambda_ms, int meq_bs, int garanin_tau);
/* Zhang integrator (llgp%zhang: push_zhang, llg.f90:410-703; the thermal field
 * joins the precession with variance lambda meq/(|H| |m|)): arguments as
 * mrm_gpu_set_mt (the reference sets meq_bs = !zhang_l); Heun and the
 * |type| = 2 branch. */
int mrm_gpu_set_zhang(mrm_gpu* h, int layer, double spin, const double* lambda_ms, int meq_bs, int garanin_tau);
int mrm_gpu_set_mag(mrm_gpu* h, int layer, const double* mag);
int mrm_gpu_get_mag(mrm_gpu* h, int layer, double* mag);

/* Moving demag window (nxfft/nyfft < nx/ny; window_m and update_do_grain,
 * data.f90:1-65,120-157, get_mag / get_magnetostatic :322-390,
 * field.f90:438-517): the demag FFT covers nx_win x ny_win cells whose origin
 * follows off = v t + offset (window%v, window%offset: the CLI's field
 * VELOCITY and -REF) as
 *   i0 = clamp(nint((nx - nx_win)/2 + off_x/dx), 1, nx - nx_win + 1) - 1  (j0 alike),
 * placed before the first step and after every step.  Grains inside the
 * window (do_grain) are evaluated and pushed; the others keep their state and
 * their last field; the stats reduce every grain (a frozen grain with its last
 * field) and mmag over the grains from the window's first to its last index,
 * normalised by the pushed grains' volume, as llg() does.  The window's FFT
 * grid follows the boundary rule of mrm_geom on nx_win x ny_win; the tensor
 * must be built or uploaded again for it.  nx_win = nx and ny_win = ny: no
 * window.  One grain per cell, a handle of its own (not in a batch), fixed dt.
 * mrm_gpu_get_window: out4 = {nx_win, ny_win, i0, j0}, the origin at the
 * handle's current time (where the next step evaluates). */
int mrm_gpu_set_window(mrm_gpu* h, int nx_win, int ny_win, double vx, double vy, double offset_x, double offset_y);
int mrm_gpu_get_window(const mrm_gpu* h, int* out4);

/* Cubic magnetocrystalline anisotropy on `layer` (get_cubic_hk,
 * field.f90:377-395; set up by construct_hk_direction with k_cubic,
 * construct_grain.f90:1620-1625, which then drops the uniaxial axis):
 * cubic_axis is the reference's cubic_axis(3,3,N) (column-major: lab
 * component k of crystal axis i of grain n at cubic_axis[k + 3*i + 9*n]); the
 * layer's hk(1), hk(2) of mrm_gpu_upload_layer act as K1, K2 (Oe) and its
 * uniaxial axes are ignored.  NULL returns the layer to uniaxial anisotropy.
 * Call after mrm_gpu_upload_layer (and again after a re-upload). */
int mrm_gpu_set_cubic_axes(mrm_gpu* h, int layer, const double* cubic_axis);

/* Thermal (Brown) field of `layer` at `temperature` K (get_thermal,
 * field.f90:397-436).  The normals come from a counter-based Philox stream
 * keyed by `seed` (Philox4x64-10 for MRM_FP64 handles, Philox4x32-10 for
 * MRM_FP32; statistical, not bitwise, equivalence with the reference's
 * MT19937 stream, random.f90:231-249). */
int mrm_gpu_set_thermal(mrm_gpu* h, int layer, int on, double temperature, uint64_t seed);

/* m(3,N) of `layer` (the active half m(1+in:3+in,:)) */
int mrm_gpu_set_state(mrm_gpu* h, int layer, const double* m);
int mrm_gpu_get_state(mrm_gpu* h, int layer, double* m);
/* h(3,N): the last non-thermal total field (field.f90:201) */
int mrm_gpu_get_field(mrm_gpu* h, int layer, double* hfield);
/* time and step counter (the Philox counter) of the handle */
int mrm_gpu_set_time(mrm_gpu* h, double t, int64_t step);
int mrm_gpu_get_time(const mrm_gpu* h, double* t, int64_t* step);

/* Evaluates get_field(t) (no thermal) on the current state; h_demag(3,N) of
 * `layer` is returned if hdemag != NULL, the total field via get_field. */
int mrm_gpu_eval_field(mrm_gpu* h, double t, int layer, double* hdemag);

/* Advances nsteps fixed-dt steps of llg_type (src/llg.f90:1195-1271):
 * -3 Heun (:1122-1139, two field evaluations per step), 2 semi-implicit push
 * (:1109-1118, one field evaluation), -2 semi-implicit midpoint (predictor over
 * dt/2, field at t+dt/2 on it, push of m_n over dt).  Replaces nsteps
 * iterations of the llg() loop body for a fixed-step run (fixed_dt_p,
 * conv_torque = conv_angle = 0); other types return MRM_ERR_UNSUPPORTED.
 * `out` (may be NULL) receives the reductions of the last step. */
int mrm_gpu_step(mrm_gpu* h, int nsteps, double dt, int llg_type, mrm_gpu_stats* out);

/* Enqueues nsteps like mrm_gpu_step without waiting for them; the stats of
 * the last enqueued step are read later with mrm_gpu_read_stats (which waits). */
int mrm_gpu_enqueue_steps(mrm_gpu* h, int nsteps, double dt, int llg_type);
int mrm_gpu_read_stats(mrm_gpu* h, mrm_gpu_stats* out);
/* The cudaStream_t (as void*) the handle launches on, for event timing. */
int mrm_gpu_stream(const mrm_gpu* h, void** stream);

/* nsteps iterations of llg()'s loop with the adaptive time step (dt_frac != 0;
 * llg.f90:240-269, get_fields :363-388, push_m :1195-1271, set_llg :1452-1486):
 * each step evaluates the field at t, sets dt = min(dt_max, min over layers
 * (1+alpha^2)/((1+alpha) gamma) dt_frac / max(1, max |h + hthm/sqrt(dt*max_dmdt)|)),
 * takes the step at dt*max_dmdt and, while the first layer (in order) whose
 * rotation acos(1 - max|dm|^2/2) exceeds max_dm[layer] (radians) says so,
 * retries it from the saved state with max_dmdt *= 0.9/ratio; then
 * dt = dt*max_dmdt, the next max_dmdt follows push_m, t advances by dt.
 * *dt and *max_dmdt are llgp%dt and llgp%max_dmdt, carried from call to call
 * (start: the run's dt, 1).  Host-driven, a few synchronisations per step; a
 * handle of its own (not in a batch).  out: the stats of the last step. */
int mrm_gpu_step_adaptive(mrm_gpu* h, int nsteps, int llg_type, double dt_frac, double dt_max,
                          const double* max_dm, double* dt, double* max_dmdt, mrm_gpu_stats* out);

/* Stray field of the current state at an observation slab above the media
 * (plot_off_field / get_off_field and calculate_off_field_tensor,
 * off_field.f90:25-108,216-320; e.g. a readback plane): the slab's bottom
 * is zoff (cm) above the top of the top layer, its thickness dzobs (cm); the
 * field is averaged over the slab, on the nx x ny grid with num_images
 * periodic images in x and y (the module's periodic_x/y), a soft underlayer
 * image when sul_mu > 1 (space_to_sul below the bottom layer) and a head
 * image when head_mu > 1 (fly_height above the top layer).  out[(c*ny + j)*nx + i]
 * = H_c (Oe), c = x, y, z.  Computed in FP64 on the device (tensor, FFTs and
 * products); nx, ny powers of two. */
int mrm_gpu_off_field(mrm_gpu* h, double zoff, double dzobs, double head_mu, double fly_height, double sul_mu,
                      double space_to_sul, int num_images, double* out);

/* Kernel shapes of the engine a handle runs in (a batch run: the batch's).
 * row_shape / col_shape index the compiled row / column kernel shapes
 * (rows per block, threads, resident blocks; threads and resident blocks of
 * the column kernel) and cols_per_task > 0 fixes the spectral columns per
 * column task (rounded down to a power of two, at most 8: the width of the
 * column tiles the row kernel writes the M spectrum in); a negative shape returns to the automatic choice.  Results do
 * not depend on the shape.  Automatic: with autotuning on (the default), the
 * first step after the set of runs changes times every compiled shape on the
 * runs themselves (their state is restored) and keeps the fastest, cached per
 * grid size, layer count and grain-count magnitude; with it off, a size
 * heuristic.  mrm_gpu_get_shape: out3 = {row shape, column shape, columns per
 * task (0: default)} of the last step. */
int mrm_gpu_set_shape(mrm_gpu* h, int row_shape, int col_shape, int cols_per_task);
int mrm_gpu_set_autotune(mrm_gpu* h, int on);
int mrm_gpu_get_shape(const mrm_gpu* h, int* out3);
/* Waits for the handle's stream and reads (and clears) the device error flag
 * its kernels raise instead of trapping (bulk-copy waits that ran out, a
 * kernel shape outside its compiled range); MRM_ERR_DEVICE with the details
 * in mrm_gpu_last_error() if it was set.  The stepping calls do this at every
 * synchronisation. */
int mrm_gpu_check_device(mrm_gpu* h);
/* Device failure self-test (no counterpart in the reference: its CPU code has
 * no device waits).  Runs one field-evaluation launch of the row kernel on
 * the handle's stream in which every block's bounded wait for its grain rows
 * is made to run out (the barrier expects 16 bytes that no copy sends), so
 * each block takes the path of a bulk copy that never lands: it raises the
 * device error flag, waits once more (bounded) and returns, writing nothing.
 * Takes about two seconds; returns what the handle's next synchronisation
 * reports, MRM_ERR_DEVICE with "a bulk-copy wait ran out" in
 * mrm_gpu_last_error().  The flag is cleared on that report and the handle
 * stays usable. */
int mrm_gpu_selftest_timeout(mrm_gpu* h);
/* Advances `reps` Heun steps launching each kernel bracketed by CUDA events
 * on the handle's stream; ms_out[4] = mean ms of row(predictor), column,
 * row(corrector), column launches (the demag column launches are 0 when
 * demag is off). */
int mrm_gpu_profile(mrm_gpu* h, int reps, double dt, double* ms_out);

/* ---------------- batched / served form ---------------- */

/* A batch owns a device stream and advances all its active runs with one
 * launch sequence per Heun stage (one task table over every run's rows and
 * spectral columns), captured in CUDA graphs. */
int mrm_batch_create(int precision, int device, mrm_batch** out);
int mrm_batch_destroy(mrm_batch* b);
const char* mrm_batch_last_error(const mrm_batch* b);
/* Creates a run inside the batch (same precision/device); configure it with
 * the mrm_gpu_* upload/set functions; it is freed by mrm_batch_remove. */
int mrm_batch_add(mrm_batch* b, const mrm_geom* geom, mrm_gpu** run);
/* Takes the run out of the batch after the batch's work in flight; the run
 * handle is invalid on return.  Its device memory is released at the batch's
 * next mrm_batch_stats, mrm_batch_step or mrm_batch_destroy. */
int mrm_batch_remove(mrm_batch* b, mrm_gpu* run);
/* Moves a run of batch src into batch dst (same precision and device; no
 * reference counterpart): state, parameters, tensor and counters move with
 * it, no device copy is made.  Waits for both batches' work in flight.  A
 * server sets up arriving runs in a second batch, whose uploads and tensor
 * builds then overlap the serving batch's steps, and moves them in between
 * two calls. */
int mrm_batch_adopt(mrm_batch* dst, mrm_batch* src, mrm_gpu* run);
/* per-run time step and step budget: the run advances while step < step_end */
int mrm_batch_set_run(mrm_gpu* run, double dt, int64_t step_end, int active);
/* Aligned start (no reference counterpart): the run idles through the first
 * idle_steps steps of its next mrm_batch_step / _enqueue call, then steps on
 * from where it is (state, time and thermal counters as without the delay),
 * so that a budget of S steps ends on a call boundary of fixed length K when
 * idle_steps = K - S mod K.  step_end stays where it is: the run executes
 * the same steps, idle_steps later.  Once per run, before it starts stepping. */
int mrm_batch_delay_run(mrm_gpu* run, int64_t idle_steps);
/* Advances every active run by up to nsteps steps of llg_type (-3, 2 or -2). */
int mrm_batch_step(mrm_batch* b, int nsteps, int llg_type);
/* Stats of each listed run at its last executed step that ended an
 * mrm_batch_step / mrm_batch_enqueue call (a run whose budget ends inside a
 * call keeps the stats of its previous call: schedule calls so that budgets
 * end on call boundaries). */
int mrm_batch_stats(mrm_batch* b, int nruns, mrm_gpu* const* runs, mrm_gpu_stats* out);
/* Enqueues like mrm_batch_step without waiting (stats via mrm_batch_stats). */
int mrm_batch_enqueue(mrm_batch* b, int nsteps, int llg_type);
int mrm_batch_stream(const mrm_batch* b, void** stream);
/* Per-kernel timing of one Heun step of every active run (CUDA events on the
 * batch's stream, averaged over reps steps, which are taken):
 * ms_out[4] = predictor row, column, corrector row, column kernel. */
int mrm_batch_profile(mrm_batch* b, int reps, double* ms_out);
/* Resident blocks per SM of the row and column kernels of this batch (0 if
 * no step was taken yet): out[0] = row, out[1] = column. */
int mrm_batch_occupancy(mrm_batch* b, int* out2);
/* Device bytes a run of this geometry holds (admission by HBM footprint). */
int64_t mrm_run_footprint(const mrm_geom* geom);
/* Free / total device memory in bytes. */
int mrm_device_memory(int device, int64_t* free_bytes, int64_t* total_bytes);

/* Allocation-free demag evaluation.  No counterpart in the reference (its
 * get_demag, src/demag.f90:33-135, works on module arrays allocated in
 * init_demag); it exists for hosts that must not allocate device memory
 * while they run, e.g. under a stream-ordered pool or a caching allocator.
 *   h       an MRM_FP32 handle with every layer uploaded and a tensor built or
 *           uploaded (its tensor, parameters and twiddles are read; the one
 *           thing of the handle that is written is its device error word: a
 *           kernel of the call that fails -- a bulk-copy wait that ran out --
 *           records it there, and the handle's next synchronising call,
 *           mrm_gpu_check_device for one, reports it after the caller's
 *           stream has finished the work);
 *   m       device pointer, n_lay x n_grains x 3 floats (each layer's m(3,n));
 *   hdemag  device pointer, same shape: the demagnetising field (Oe);
 *   stream  cudaStream_t to enqueue on (NULL: the handle's stream); the call
 *           returns once the work is enqueued.
 * Scratch is one static 16 MiB device array per device; a grid whose
 * descriptor, tasks, three float4 grain arrays and two half spectra exceed it
 * returns MRM_ERR_UNSUPPORTED.  Nothing in the scratch needs to start at zero.
 * The first call on a device sets up (scratch address, kernel loading and
 * shared-memory limits) and must not be made during a stream capture.  Calls
 * whose work overlaps on the device (different streams, other threads) share
 * the scratch and race: serialise them. */
int mrm_gpu_demag_noalloc(mrm_gpu* h, const float* m, float* hdemag, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MRM_GPU_H */
