! mrm_gpu_m.f90 -- ISO_C_BINDING interface of the B200 grain-dynamics path.
!
! Binds include/mrm_gpu.h for the reference's Fortran host, in the opaque
! handle style of src/FP/fp.f90:13-36 (type(C_ptr) handle, value arguments,
! C_DOUBLE arrays by reference).  A push_m replacement (gpu_push_m below) is
! selected in llg() by a new `gpu_p` flag of the llg namelist; the Fortran
! host, namelists, CLI, grain files and checkpoints stay unchanged.
! Written for gfortran/ifort; this repository's environment has no Fortran
! compiler, so the C side of every binding is exercised from Python/ctypes.
module mrm_gpu_m
  use, intrinsic :: iso_c_binding
  implicit none
  private
  public :: mrm_geom_t, mrm_stats_t, gpu_create, gpu_destroy, gpu_upload_layer, &
            gpu_upload_interlayer, gpu_build_tensor, gpu_upload_tensor, gpu_set_uniform_field, &
            gpu_set_field_function, gpu_set_head_field, gpu_set_cubic_axes, gpu_step_adaptive, gpu_off_field, &
            gpu_set_window, gpu_set_field_table, gpu_set_llb, gpu_set_mt, gpu_set_zhang, &
            gpu_set_temp_profile, gpu_set_temp_function, gpu_set_temp_scaling, gpu_set_temp_scaling_table, &
            gpu_set_mag, gpu_get_mag, gpu_set_thermal, gpu_set_state, gpu_get_state, &
            gpu_get_field, &
            gpu_set_time, gpu_step, gpu_last_error, gpu_push_m

  integer(C_INT), parameter, public :: MRM_PERIODIC = 0, MRM_OPEN = 1, MRM_FP32 = 0, MRM_FP64 = 1
  integer, parameter :: MAXL = 8

  type, bind(C) :: mrm_geom_t
    integer(C_INT32_T) :: nx, ny, n_lay, boundary, num_images, precision
    real(C_DOUBLE) :: dx, dy, dz(MAXL), il_space(MAXL)
    real(C_DOUBLE) :: space_to_sul, sul_mu, head_mu, fly_height
  end type

  type, bind(C) :: mrm_stats_t
    real(C_DOUBLE) :: t
    integer(C_INT64_T) :: step
    real(C_DOUBLE) :: mave(3), mvar(3), have(3), errmx, errmx1, mmag, energy
    real(C_DOUBLE) :: mave_l(3, MAXL), mvar_l(3, MAXL), have_l(3, MAXL), mms_l(3, MAXL)
    real(C_DOUBLE) :: vol_l(MAXL), msvol_l(MAXL)
    integer(C_INT64_T) :: nup_l(MAXL)
    real(C_DOUBLE) :: errmx1_l(MAXL)
  end type

  interface
    integer(C_INT) function c_create(geom, device, h) bind(C, name="mrm_gpu_create")
      import :: C_INT, C_PTR, mrm_geom_t
      type(mrm_geom_t), intent(in) :: geom
      integer(C_INT), value :: device
      type(C_PTR), intent(out) :: h
    end function
    integer(C_INT) function c_destroy(h) bind(C, name="mrm_gpu_destroy")
      import :: C_INT, C_PTR
      type(C_PTR), value :: h
    end function
    type(C_PTR) function c_last_error(h) bind(C, name="mrm_gpu_last_error")
      import :: C_PTR
      type(C_PTR), value :: h
    end function
    integer(C_INT) function c_upload_layer(h, layer, n, ms, vol, axis, hk, hk_scale, ms_scale, &
        alpha_scale, alpha, gamma, floor_ms, g2ci, g2c, hxi, hxg, hx) bind(C, name="mrm_gpu_upload_layer")
      import :: C_INT, C_PTR, C_DOUBLE, C_INT32_T
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, n
      real(C_DOUBLE), intent(in) :: ms(*), vol(*), axis(*), hk(*), hk_scale(*), ms_scale(*), alpha_scale(*)
      real(C_DOUBLE), value :: alpha, gamma, floor_ms
      integer(C_INT32_T), intent(in) :: g2ci(*), g2c(*)
      type(C_PTR), value :: hxi, hxg, hx
    end function
    integer(C_INT) function c_upload_interlayer(h, layer, side, idx, grain, coef) &
        bind(C, name="mrm_gpu_upload_interlayer")
      import :: C_INT, C_PTR, C_DOUBLE, C_INT32_T
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, side
      integer(C_INT32_T), intent(in) :: idx(*), grain(*)
      real(C_DOUBLE), intent(in) :: coef(*)
    end function
    integer(C_INT) function c_build_tensor(h) bind(C, name="mrm_gpu_build_tensor")
      import :: C_INT, C_PTR
      type(C_PTR), value :: h
    end function
    integer(C_INT) function c_upload_tensor(h, n2d, nxf, nyf) bind(C, name="mrm_gpu_upload_tensor")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      real(C_DOUBLE), intent(in) :: n2d(*)
      integer(C_INT), value :: nxf, nyf
    end function
    integer(C_INT) function c_set_uniform_field(h, layer, hdir, t0, t1, s0, s1, scale) &
        bind(C, name="mrm_gpu_set_uniform_field")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer
      real(C_DOUBLE), intent(in) :: hdir(3)
      real(C_DOUBLE), value :: t0, t1, s0, s1, scale
    end function
    integer(C_INT) function c_set_field_function(h, layer, hdir, func, amp, gamma, phase, param, &
        duty, moddepth, dc, scale) bind(C, name="mrm_gpu_set_field_function")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, func
      real(C_DOUBLE), intent(in) :: hdir(3)
      real(C_DOUBLE), value :: amp, gamma, phase, param, duty, moddepth, dc, scale
    end function
    integer(C_INT) function c_set_head_field(h, layer, gap, z, hg, velocity, x0, t0, bit_time, pattern, &
        nbits) bind(C, name="mrm_gpu_set_head_field")
      import :: C_INT, C_PTR, C_DOUBLE, C_INT64_T
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, nbits
      real(C_DOUBLE), value :: gap, z, hg, velocity, x0, t0, bit_time
      integer(C_INT64_T), value :: pattern
    end function
    integer(C_INT) function c_set_cubic_axes(h, layer, cubic_axis) bind(C, name="mrm_gpu_set_cubic_axes")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer
      real(C_DOUBLE), intent(in) :: cubic_axis(3, 3, *)
    end function
    integer(C_INT) function c_set_llb(h, layer, spin, tc, lambda_ms) bind(C, name="mrm_gpu_set_llb")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer
      real(C_DOUBLE), value :: spin
      real(C_DOUBLE), intent(in) :: tc(*), lambda_ms(*)
    end function
    integer(C_INT) function c_set_mt(h, layer, spin, lambda_ms, meq_bs, garanin_tau) bind(C, name="mrm_gpu_set_mt")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, meq_bs, garanin_tau
      real(C_DOUBLE), value :: spin
      real(C_DOUBLE), intent(in) :: lambda_ms(*)
    end function
    integer(C_INT) function c_set_zhang(h, layer, spin, lambda_ms, meq_bs, garanin_tau) &
        bind(C, name="mrm_gpu_set_zhang")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, meq_bs, garanin_tau
      real(C_DOUBLE), value :: spin
      real(C_DOUBLE), intent(in) :: lambda_ms(*)
    end function
    integer(C_INT) function c_set_temp_scaling(h, layer, tc, msexp, hkexp, use_mag) &
        bind(C, name="mrm_gpu_set_temp_scaling")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, use_mag
      real(C_DOUBLE), intent(in) :: tc(*)
      real(C_DOUBLE), value :: msexp, hkexp
    end function
    integer(C_INT) function c_set_temp_scaling_table(h, layer, which, n, temp, scaling) &
        bind(C, name="mrm_gpu_set_temp_scaling_table")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, which, n
      real(C_DOUBLE), intent(in) :: temp(*), scaling(*)
    end function
    integer(C_INT) function c_set_temp_profile(h, layer, bg, dtemp, sx, sy, expn, vx, vy, ox, oy, rx, ry, t0) &
        bind(C, name="mrm_gpu_set_temp_profile")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, expn
      real(C_DOUBLE), value :: bg, dtemp, sx, sy, vx, vy, ox, oy, rx, ry, t0
    end function
    integer(C_INT) function c_set_temp_function(h, layer, func, t_start, t_end, s_start, s_end, amp, gamma, phase, &
                                                param, duty, moddepth, dc, scale) bind(C, name="mrm_gpu_set_temp_function")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, func
      real(C_DOUBLE), value :: t_start, t_end, s_start, s_end, amp, gamma, phase, param, duty, moddepth, dc, scale
    end function
    integer(C_INT) function c_set_mag(h, layer, mag) bind(C, name="mrm_gpu_set_mag")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer
      real(C_DOUBLE), intent(in) :: mag(*)
    end function
    integer(C_INT) function c_get_mag(h, layer, mag) bind(C, name="mrm_gpu_get_mag")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer
      real(C_DOUBLE), intent(out) :: mag(*)
    end function
    integer(C_INT) function c_set_window(h, nxw, nyw, vx, vy, ox, oy) bind(C, name="mrm_gpu_set_window")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: nxw, nyw
      real(C_DOUBLE), value :: vx, vy, ox, oy
    end function
    integer(C_INT) function c_set_field_table(h, layer, nfx, nfy, xpos, ypos, vfld, vx, vy, ox, oy, rx, ry, t0) &
        bind(C, name="mrm_gpu_set_field_table")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, nfx, nfy
      real(C_DOUBLE), intent(in) :: xpos(*), ypos(*), vfld(*)
      real(C_DOUBLE), value :: vx, vy, ox, oy, rx, ry, t0
    end function
    integer(C_INT) function c_off_field(h, zoff, dzobs, head_mu, fly_height, sul_mu, space_to_sul, num_images, out) &
        bind(C, name="mrm_gpu_off_field")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      real(C_DOUBLE), value :: zoff, dzobs, head_mu, fly_height, sul_mu, space_to_sul
      integer(C_INT), value :: num_images
      real(C_DOUBLE), intent(out) :: out(*)
    end function
    integer(C_INT) function c_step_adaptive(h, nsteps, llg_type, dt_frac, dt_max, max_dm, dt, max_dmdt, stats) &
        bind(C, name="mrm_gpu_step_adaptive")
      import :: C_INT, C_PTR, C_DOUBLE, mrm_stats_t
      type(C_PTR), value :: h
      integer(C_INT), value :: nsteps, llg_type
      real(C_DOUBLE), value :: dt_frac, dt_max
      real(C_DOUBLE), intent(in) :: max_dm(*)
      real(C_DOUBLE), intent(inout) :: dt, max_dmdt
      type(mrm_stats_t), intent(out) :: stats
    end function
    integer(C_INT) function c_set_thermal(h, layer, on, temperature, seed) bind(C, name="mrm_gpu_set_thermal")
      import :: C_INT, C_PTR, C_DOUBLE, C_INT64_T
      type(C_PTR), value :: h
      integer(C_INT), value :: layer, on
      real(C_DOUBLE), value :: temperature
      integer(C_INT64_T), value :: seed
    end function
    integer(C_INT) function c_set_state(h, layer, m) bind(C, name="mrm_gpu_set_state")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer
      real(C_DOUBLE), intent(in) :: m(*)
    end function
    integer(C_INT) function c_get_state(h, layer, m) bind(C, name="mrm_gpu_get_state")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer
      real(C_DOUBLE), intent(out) :: m(*)
    end function
    integer(C_INT) function c_get_field(h, layer, hf) bind(C, name="mrm_gpu_get_field")
      import :: C_INT, C_PTR, C_DOUBLE
      type(C_PTR), value :: h
      integer(C_INT), value :: layer
      real(C_DOUBLE), intent(out) :: hf(*)
    end function
    integer(C_INT) function c_set_time(h, t, step) bind(C, name="mrm_gpu_set_time")
      import :: C_INT, C_PTR, C_DOUBLE, C_INT64_T
      type(C_PTR), value :: h
      real(C_DOUBLE), value :: t
      integer(C_INT64_T), value :: step
    end function
    integer(C_INT) function c_step(h, nsteps, dt, llg_type, stats) bind(C, name="mrm_gpu_step")
      import :: C_INT, C_PTR, C_DOUBLE, mrm_stats_t
      type(C_PTR), value :: h
      integer(C_INT), value :: nsteps, llg_type
      real(C_DOUBLE), value :: dt
      type(mrm_stats_t), intent(out) :: stats
    end function
  end interface

contains

  ! status code -> the reference's logical ok_p convention (e.g. field.f90:787-837)
  logical function ok(rc)
    integer(C_INT), intent(in) :: rc
    ok = (rc == 0)
  end function

  logical function gpu_create(geom, device, h) result(ok_p)
    type(mrm_geom_t), intent(in) :: geom
    integer, intent(in) :: device
    type(C_PTR), intent(out) :: h
    ok_p = ok(c_create(geom, int(device, C_INT), h))
  end function

  logical function gpu_destroy(h) result(ok_p)
    type(C_PTR), intent(in) :: h
    ok_p = ok(c_destroy(h))
  end function

  function gpu_last_error(h) result(msg)
    type(C_PTR), intent(in) :: h
    character(len=512) :: msg
    character(kind=C_CHAR), pointer :: s(:)
    integer :: i
    msg = ' '
    call c_f_pointer(c_last_error(h), s, [512])
    do i = 1, 512
      if (s(i) == C_NULL_CHAR) exit
      msg(i:i) = s(i)
    end do
  end function

  ! one layer of data_s / field_ss (data.f90:91-104, field.f90:15-35); hx optional
  logical function gpu_upload_layer(h, layer, n, ms, vol, axis, hk, hk_scale, ms_scale, alpha_scale, &
      alpha, gamma, floor_ms, g2ci, g2c, hxi, hxg, hx) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer, n
    real(C_DOUBLE), intent(in) :: ms(:), vol(:), axis(:, :), hk(:, :), hk_scale(:), ms_scale(:), alpha_scale(:)
    real(C_DOUBLE), intent(in) :: alpha, gamma, floor_ms
    integer(C_INT32_T), intent(in) :: g2ci(0:), g2c(:, :)
    integer(C_INT32_T), intent(in), target, optional :: hxi(0:), hxg(:)
    real(C_DOUBLE), intent(in), target, optional :: hx(:)
    type(C_PTR) :: pi, pg, px
    pi = C_NULL_PTR; pg = C_NULL_PTR; px = C_NULL_PTR
    if (present(hxi)) pi = c_loc(hxi)
    if (present(hxg)) pg = c_loc(hxg)
    if (present(hx)) px = c_loc(hx)
    ok_p = ok(c_upload_layer(h, int(layer - 1, C_INT), int(n, C_INT), ms, vol, axis, hk, hk_scale, &
                            ms_scale, alpha_scale, alpha, gamma, floor_ms, g2ci, g2c, pi, pg, px))
  end function

  logical function gpu_upload_interlayer(h, layer, side, idx, grain, coef) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer, side
    integer(C_INT32_T), intent(in) :: idx(0:), grain(:)
    real(C_DOUBLE), intent(in) :: coef(:)
    ok_p = ok(c_upload_interlayer(h, int(layer - 1, C_INT), int(side, C_INT), idx, grain, coef))
  end function

  logical function gpu_build_tensor(h) result(ok_p)
    type(C_PTR), intent(in) :: h
    ok_p = ok(c_build_tensor(h))
  end function

  ! n2d(nx,ny,9,n_lay,n_lay) from calculate_tensor / mrm_N.dat (tensor.f90:82-216)
  logical function gpu_upload_tensor(h, n2d) result(ok_p)
    type(C_PTR), intent(in) :: h
    real(C_DOUBLE), intent(in) :: n2d(:, :, :, :, :)
    ok_p = ok(c_upload_tensor(h, n2d, int(size(n2d, 1), C_INT), int(size(n2d, 2), C_INT)))
  end function

  logical function gpu_set_uniform_field(h, layer, hdir, t0, t1, s0, s1, scale) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(in) :: hdir(3), t0, t1, s0, s1, scale
    ok_p = ok(c_set_uniform_field(h, int(layer - 1, C_INT), hdir, t0, t1, s0, s1, scale))
  end function

  logical function gpu_set_field_function(h, layer, hdir, func, amp, gamma, phase, param, duty, &
      moddepth, dc, scale) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer, func
    real(C_DOUBLE), intent(in) :: hdir(3), amp, gamma, phase, param, duty, moddepth, dc, scale
    ok_p = ok(c_set_field_function(h, int(layer - 1, C_INT), hdir, int(func, C_INT), amp, gamma, &
                                  phase, param, duty, moddepth, dc, scale))
  end function

  ! moving Karlqvist write head on `layer` (include/mrm_gpu.h mrm_gpu_set_head_field)
  logical function gpu_set_head_field(h, layer, gap, z, hg, velocity, x0, t0, bit_time, pattern, nbits) &
      result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer, nbits
    real(C_DOUBLE), intent(in) :: gap, z, hg, velocity, x0, t0, bit_time
    integer(C_INT64_T), intent(in) :: pattern
    ok_p = ok(c_set_head_field(h, int(layer - 1, C_INT), gap, z, hg, velocity, x0, t0, bit_time, pattern, &
                               int(nbits, C_INT)))
  end function

  ! cubic anisotropy on `layer` from field(il)%cubic_axis (include/mrm_gpu.h mrm_gpu_set_cubic_axes)
  logical function gpu_set_cubic_axes(h, layer, cubic_axis) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(in) :: cubic_axis(:, :, :)
    ok_p = ok(c_set_cubic_axes(h, int(layer - 1, C_INT), cubic_axis))
  end function

  ! llgp%llb on `layer`: layer(il)%spin, %tc(:), %lambdaMs(:) (include/mrm_gpu.h
  ! mrm_gpu_set_llb); gpu_set_mag / gpu_get_mag carry layer(il)%mag(in/3+1,:)
  logical function gpu_set_llb(h, layer, spin, tc, lambda_ms) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(in) :: spin, tc(:), lambda_ms(:)
    ok_p = ok(c_set_llb(h, int(layer - 1, C_INT), spin, tc, lambda_ms))
  end function
  ! llgp%mt on `layer` (include/mrm_gpu.h mrm_gpu_set_mt)
  logical function gpu_set_mt(h, layer, spin, lambda_ms, meq_bs, garanin_tau) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(in) :: spin, lambda_ms(:)
    logical, intent(in) :: meq_bs, garanin_tau
    ok_p = ok(c_set_mt(h, int(layer - 1, C_INT), spin, lambda_ms, merge(1_C_INT, 0_C_INT, meq_bs), &
                       merge(1_C_INT, 0_C_INT, garanin_tau)))
  end function
  ! llgp%zhang on `layer` (include/mrm_gpu.h mrm_gpu_set_zhang)
  logical function gpu_set_zhang(h, layer, spin, lambda_ms, meq_bs, garanin_tau) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(in) :: spin, lambda_ms(:)
    logical, intent(in) :: meq_bs, garanin_tau
    ok_p = ok(c_set_zhang(h, int(layer - 1, C_INT), spin, lambda_ms, merge(1_C_INT, 0_C_INT, meq_bs), &
                          merge(1_C_INT, 0_C_INT, garanin_tau)))
  end function
  ! suprgaus_temp + ref_temp of `layer` (include/mrm_gpu.h mrm_gpu_set_temp_profile):
  ! background_t, dtemp, sigma (cm, 0: flat), the exponent as suprgaus_temp takes
  ! it, fld%vel_x/y, %offset_x/y, %ref_x/y, %t_origin
  logical function gpu_set_temp_profile(h, layer, background, dtemp, sigma, expn, vel, offset, ref, t_origin) &
      result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer, expn
    real(C_DOUBLE), intent(in) :: background, dtemp, sigma(2), vel(2), offset(2), ref(2), t_origin
    ok_p = ok(c_set_temp_profile(h, int(layer - 1, C_INT), background, dtemp, sigma(1), sigma(2), int(expn, C_INT), &
                                 vel(1), vel(2), offset(1), offset(2), ref(1), ref(2), t_origin))
  end function
  ! temp_scaling(layer)%p (include/mrm_gpu.h mrm_gpu_set_temp_scaling): field(layer)%tc,
  ! %msexp, %hkexp, %use_mag_p; called where init_temp_scaling runs (grain.f90:54),
  ! after the layer's uploads with its unit scales
  logical function gpu_set_temp_scaling(h, layer, tc, msexp, hkexp, use_mag_p) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(in) :: tc(:), msexp, hkexp
    logical, intent(in) :: use_mag_p
    ok_p = ok(c_set_temp_scaling(h, int(layer - 1, C_INT), tc, msexp, hkexp, merge(1_C_INT, 0_C_INT, use_mag_p)))
  end function
  ! file_temp_scaling's table indx (1 Ms, 2 alpha, 3 Hk, 4 Hx) as read: the
  ! (temperature, scaling) pairs before the reduction, which the library applies
  logical function gpu_set_temp_scaling_table(h, layer, indx, temp, scaling) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer, indx
    real(C_DOUBLE), intent(in) :: temp(:), scaling(:)
    ok_p = ok(c_set_temp_scaling_table(h, int(layer - 1, C_INT), int(indx, C_INT), int(size(temp), C_INT), &
                                       temp, scaling))
  end function
  ! set_temp's time scale of that profile (include/mrm_gpu.h mrm_gpu_set_temp_function)
  logical function gpu_set_temp_function(h, layer, func, t_start, t_end, s_start, s_end, amp, gamma, phase, param, &
                                         duty, moddepth, dc, scale) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer, func
    real(C_DOUBLE), intent(in) :: t_start, t_end, s_start, s_end, amp, gamma, phase, param, duty, moddepth, dc, scale
    ok_p = ok(c_set_temp_function(h, int(layer - 1, C_INT), int(func, C_INT), t_start, t_end, s_start, s_end, amp, &
                                  gamma, phase, param, duty, moddepth, dc, scale))
  end function
  logical function gpu_set_mag(h, layer, mag) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(in) :: mag(:)
    ok_p = ok(c_set_mag(h, int(layer - 1, C_INT), mag))
  end function
  logical function gpu_get_mag(h, layer, mag) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(out) :: mag(:)
    ok_p = ok(c_get_mag(h, int(layer - 1, C_INT), mag))
  end function

  ! moving demag window nxfft x nyfft following window%v, window%offset
  ! (include/mrm_gpu.h mrm_gpu_set_window); build or upload its tensor afterwards
  logical function gpu_set_window(h, nxfft, nyfft, v, offset) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: nxfft, nyfft
    real(C_DOUBLE), intent(in) :: v(2), offset(2)
    ok_p = ok(c_set_window(h, int(nxfft, C_INT), int(nyfft, C_INT), v(1), v(2), offset(1), offset(2)))
  end function

  ! a file_applied field table on `layer`: vfld(3, nx, ny) at xpos(nx), ypos(ny)
  ! (include/mrm_gpu.h mrm_gpu_set_field_table)
  logical function gpu_set_field_table(h, layer, xpos, ypos, vfld, vel_x, vel_y, offset_x, offset_y, ref_x, ref_y, &
                                       t_origin) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(in) :: xpos(:), ypos(:), vfld(:, :, :)
    real(C_DOUBLE), intent(in) :: vel_x, vel_y, offset_x, offset_y, ref_x, ref_y, t_origin
    ok_p = ok(c_set_field_table(h, int(layer - 1, C_INT), int(size(xpos), C_INT), int(size(ypos), C_INT), xpos, ypos, &
                                vfld, vel_x, vel_y, offset_x, offset_y, ref_x, ref_y, t_origin))
  end function

  ! stray field of the current state on the slab zoff..zoff+dzobs (cm) above the
  ! media, as init_demag + get_off_field of off_field.f90 compute it:
  ! h(:,:,1:3) = hx, hy, hz on the nx x ny grid (include/mrm_gpu.h mrm_gpu_off_field)
  logical function gpu_off_field(h, zoff, dzobs, mu_head, fly_height, sul_mu, space_to_sul, num_images, hxyz) &
      result(ok_p)
    type(C_PTR), intent(in) :: h
    real(C_DOUBLE), intent(in) :: zoff, dzobs, mu_head, fly_height, sul_mu, space_to_sul
    integer, intent(in) :: num_images
    real(C_DOUBLE), intent(out) :: hxyz(:, :, :)
    ok_p = ok(c_off_field(h, zoff, dzobs, mu_head, fly_height, sul_mu, space_to_sul, int(num_images, C_INT), hxyz))
  end function

  ! iter steps of llg()'s adaptive loop (dt_frac /= 0): llgp%dt and llgp%max_dmdt
  ! in and out, llgl(:)%max_dm in radians (include/mrm_gpu.h mrm_gpu_step_adaptive)
  logical function gpu_step_adaptive(h, iter, llg_type, dt_frac, dt_max, max_dm, dt, max_dmdt, stats) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: iter, llg_type
    real(C_DOUBLE), intent(in) :: dt_frac, dt_max, max_dm(:)
    real(C_DOUBLE), intent(inout) :: dt, max_dmdt
    type(mrm_stats_t), intent(out) :: stats
    ok_p = ok(c_step_adaptive(h, int(iter, C_INT), int(llg_type, C_INT), dt_frac, dt_max, max_dm, dt, max_dmdt, &
                              stats))
  end function

  logical function gpu_set_thermal(h, layer, on, temperature, seed) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer, seed
    logical, intent(in) :: on
    real(C_DOUBLE), intent(in) :: temperature
    integer(C_INT) :: ion
    ion = 0
    if (on) ion = 1
    ok_p = ok(c_set_thermal(h, int(layer - 1, C_INT), ion, temperature, int(seed, C_INT64_T)))
  end function

  logical function gpu_set_state(h, layer, m) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(in) :: m(:, :)
    ok_p = ok(c_set_state(h, int(layer - 1, C_INT), m))
  end function

  logical function gpu_get_state(h, layer, m) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(out) :: m(:, :)
    ok_p = ok(c_get_state(h, int(layer - 1, C_INT), m))
  end function

  logical function gpu_get_field(h, layer, hf) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: layer
    real(C_DOUBLE), intent(out) :: hf(:, :)
    ok_p = ok(c_get_field(h, int(layer - 1, C_INT), hf))
  end function

  logical function gpu_set_time(h, t, step) result(ok_p)
    type(C_PTR), intent(in) :: h
    real(C_DOUBLE), intent(in) :: t
    integer(C_INT64_T), intent(in) :: step
    ok_p = ok(c_set_time(h, t, step))
  end function

  logical function gpu_step(h, nsteps, dt, llg_type, stats) result(ok_p)
    type(C_PTR), intent(in) :: h
    integer, intent(in) :: nsteps, llg_type
    real(C_DOUBLE), intent(in) :: dt
    type(mrm_stats_t), intent(out) :: stats
    ok_p = ok(c_step(h, int(nsteps, C_INT), dt, int(llg_type, C_INT), stats))
  end function

  ! Replacement of push_m (llg.f90:1195-1271) for a fixed-dt Heun run: the
  ! caller's llg() loop keeps its reductions, printing and stop tests; the GPU
  ! handle holds m, the spectra and the Philox counter between calls.
  logical function gpu_push_m(h, t, dt, nsteps, stats) result(ok_p)
    type(C_PTR), intent(in) :: h
    real(C_DOUBLE), intent(inout) :: t
    real(C_DOUBLE), intent(in) :: dt
    integer, intent(in) :: nsteps
    type(mrm_stats_t), intent(out) :: stats
    ok_p = gpu_step(h, nsteps, dt, -3, stats)
    if (ok_p) t = stats%t
  end function
end module mrm_gpu_m
