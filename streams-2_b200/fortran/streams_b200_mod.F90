! ISO_C_BINDING interface of the B200 backend (include/streams_b200.h).
!
! The types mirror the C structs component by component (same order, c_int / c_double), and
! every procedure takes `value` scalars and `type(c_ptr), value` arrays, the convention of the
! HIP backend's bindings (code/src/singleideal/kernels_amd.F90:1658-1677 in STREAmS-2).
! Not compiled in this repository (no Fortran compiler in the build image).
module streams_b200_mod
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: STREAMS_B200_OK = 0, STREAMS_B200_EINVAL = -1, STREAMS_B200_ECUDA = -2, &
                               STREAMS_B200_ENOMEM = -3, STREAMS_B200_ENAN = -4, STREAMS_B200_ENODEV = -6
  integer(c_int), parameter :: STREAMS_B200_MAX_CP = 12

  type, bind(c) :: streams_b200_params
    integer(c_int) :: nx, ny, nz, ng
    integer(c_int) :: ep_order, nkeep, weno_scheme, weno_version
    integer(c_int) :: flux_splitting, conservative_viscous
    real(c_double) :: sensor_threshold
    integer(c_int) :: bctags(6), force_zero_flux(6)
    integer(c_int) :: eul_imin, eul_imax, eul_jmin, eul_jmax, eul_kmin, eul_kmax
    integer(c_int) :: is_y_staggered
    integer(c_int) :: visc_model, calorically_perfect
    real(c_double) :: mu0, t0, rgas0, rho0, u0, l0
    real(c_double) :: sutherland_s, t_ref_dim, powerlaw_vtexp, prandtl
    real(c_double) :: cp0, cv0, cp_last, cv_last
    integer(c_int) :: channel_case
    real(c_double) :: theta_wall, t_wall, t_bulk_target, volchan
    integer(c_int) :: nrk
    real(c_double) :: rhork(4), gamrk(4)
    real(c_double) :: cfl
    integer(c_int) :: precision
    integer(c_int) :: bctags_nr(6)
    real(c_double) :: winf(5)
    real(c_double) :: p0
    integer(c_int) :: recyc, i_recyc, jbl_inflow
    real(c_double) :: betarecyc
    integer(c_int) :: rng_seed
    integer(c_long_long) :: rng_draws
    real(c_double) :: xshock_imp, shock_angle, tanhfacs
    real(c_double) :: winf_past_shock(5)
    ! cp(T) polynomial (calorically_perfect = 0): cp_coeff(indx_cp_l:indx_cp_r+1) at 1..
    integer(c_int) :: indx_cp_l, indx_cp_r
    real(c_double) :: cp_coeff(STREAMS_B200_MAX_CP), cv_coeff(STREAMS_B200_MAX_CP)
  end type streams_b200_params

  type, bind(c) :: streams_b200_grid
    type(c_ptr) :: x, y, z, yn
    type(c_ptr) :: dcsidx, detady, dzitdz, dcsidxs, detadys, dzitdzs
    type(c_ptr) :: coeff_deriv1
    type(c_ptr) :: ep_ord_x, ep_ord_y, ep_ord_z
    type(c_ptr) :: dcsidx2, detady2, dzitdz2
    type(c_ptr) :: coeff_deriv2
    type(c_ptr) :: wmean_inflow, yplus_inflow, eta_inflow, yplus_recyc, eta_recyc, weta_inflow
    type(c_ptr) :: map_j_inn, map_j_out
  end type streams_b200_grid

  interface
    function streams_b200_create(p, g, ctx) bind(c, name="streams_b200_create")
      import :: c_int, c_ptr, streams_b200_params, streams_b200_grid
      type(streams_b200_params), intent(in) :: p
      type(streams_b200_grid), intent(in) :: g
      type(c_ptr), intent(out) :: ctx
      integer(c_int) :: streams_b200_create
    end function
    function streams_b200_destroy(ctx) bind(c, name="streams_b200_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int) :: streams_b200_destroy
    end function
    function streams_b200_copy_from_field(ctx, w) bind(c, name="streams_b200_copy_from_field")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, w
      integer(c_int) :: streams_b200_copy_from_field
    end function
    function streams_b200_copy_to_field(ctx, w) bind(c, name="streams_b200_copy_to_field")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, w
      integer(c_int) :: streams_b200_copy_to_field
    end function
    function streams_b200_init_run(ctx) bind(c, name="streams_b200_init_run")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int) :: streams_b200_init_run
    end function
    function streams_b200_compute_dt(ctx, dt) bind(c, name="streams_b200_compute_dt")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: dt
      integer(c_int) :: streams_b200_compute_dt
    end function
    function streams_b200_rk_sync(ctx) bind(c, name="streams_b200_rk_sync")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int) :: streams_b200_rk_sync
    end function
    function streams_b200_advance(ctx, nsteps, iter_dt_recompute, icyc_start, icyc0) &
        bind(c, name="streams_b200_advance")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps, iter_dt_recompute, icyc_start, icyc0
      integer(c_int) :: streams_b200_advance
    end function
    function streams_b200_get_scalars(ctx, out) bind(c, name="streams_b200_get_scalars")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: out(7)
      integer(c_int) :: streams_b200_get_scalars
    end function
    function streams_b200_set_time(ctx, t) bind(c, name="streams_b200_set_time")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: t
      integer(c_int) :: streams_b200_set_time
    end function
    function streams_b200_compute_residual(ctx, out) bind(c, name="streams_b200_compute_residual")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: out(7)
      integer(c_int) :: streams_b200_compute_residual
    end function
    function streams_b200_count_weno(ctx, out) bind(c, name="streams_b200_count_weno")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: out(3)
      integer(c_int) :: streams_b200_count_weno
    end function
    ! running statistics (compute_stats / compute_stats_3d after a completed step)
    function streams_b200_compute_stats(ctx, itav) bind(c, name="streams_b200_compute_stats")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: itav
      integer(c_int) :: streams_b200_compute_stats
    end function
    function streams_b200_compute_stats_3d(ctx, itav) bind(c, name="streams_b200_compute_stats_3d")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: itav
      integer(c_int) :: streams_b200_compute_stats_3d
    end function
    ! which = 0: w_stat(70,nx,ny), 1: w_stat_z, 2: w_stat_3d(14,nx,ny,nz); n in doubles
    function streams_b200_get_stats(ctx, which, out, n) bind(c, name="streams_b200_get_stats")
      import :: c_int, c_ptr, c_long_long
      type(c_ptr), value :: ctx
      integer(c_int), value :: which
      type(c_ptr), value :: out
      integer(c_long_long), value :: n
      integer(c_int) :: streams_b200_get_stats
    end function
    function streams_b200_set_stats(ctx, which, in, n) bind(c, name="streams_b200_set_stats")
      import :: c_int, c_ptr, c_long_long
      type(c_ptr), value :: ctx
      integer(c_int), value :: which
      type(c_ptr), value :: in
      integer(c_long_long), value :: n
      integer(c_int) :: streams_b200_set_stats
    end function
    function streams_b200_last_error(ctx) bind(c, name="streams_b200_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr) :: streams_b200_last_error
    end function
  end interface

end module streams_b200_mod
