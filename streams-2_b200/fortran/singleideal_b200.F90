! Solver object of the B200 backend: the counterpart of equation_singleideal_gpu_object
! (code/src/singleideal/singleideal_gpu.F90 in STREAmS-2) with the same run() contract.
! The equation object (singleideal.F90) does the set-up; this object hands its arrays to the
! C ABI once and then drives the device.  Output/statistics hooks of manage_output keep using
! the equation object after copy_to_field.  Not compiled in this repository (no Fortran
! compiler in the build image).
module streams_equation_singleideal_b200_object
  use iso_c_binding
  use streams_parameters
  use streams_equation_singleideal_object
  use streams_b200_mod
  implicit none
  private
  public :: equation_singleideal_b200_object

  type :: equation_singleideal_b200_object
    type(equation_singleideal_object) :: equation_base
    type(c_ptr) :: ctx = c_null_ptr
    integer, allocatable, dimension(:) :: epx, epy, epz
    ! recycling inflow: wmean(1-i, j, 1:4), i = 1..ng, of the equation object, contiguous
    real(c_double), allocatable, dimension(:,:,:) :: wmean_inflow
    ! rank of this process and the crandom draws the set-up took (setup_draws)
    integer(c_int) :: myrank = 0
    integer(c_long_long) :: crandom_draws = 0
  contains
    procedure, pass(self) :: initialize
    procedure, pass(self) :: run
    procedure, pass(self) :: check
    procedure, pass(self) :: setup_draws
  endtype equation_singleideal_b200_object

contains

  ! crandom draws that the equation object's set-up took on this rank before the first step.
  ! initial_conditions runs on restarts too (singleideal.F90:710-712), so the count does not
  ! depend on restart_type.  The boundary layer (flow_init = 1, turbulent) draws 3 per interior
  ! cell in init_bl (singleideal.F90:3386-3392), then add_synthetic_perturbations draws the 4
  ! streak phases (:3631) and 3 per cell below the local thickness deltavec (:3663-3666).
  ! Other initialisations draw nothing that a later step depends on (no recycling inflow).
  function setup_draws(self) result(nd)
    class(equation_singleideal_b200_object), intent(in) :: self
    integer(c_long_long) :: nd
    integer :: i, j, k, ii
    nd = 0_c_long_long
    associate(eb => self%equation_base, f => self%equation_base%field)
      if (eb%flow_init /= 1 .or. eb%bl_laminar) return
      nd = 3_c_long_long * f%nx * f%ny * f%nz + 4_c_long_long
      do k = 1, f%nz
        do j = 1, f%ny
          do i = 1, f%nx
            ii = f%ncoords(1) * f%nx + i
            if (f%y(j) < eb%deltavec(ii)) nd = nd + 3_c_long_long
          enddo
        enddo
      enddo
    endassociate
  endfunction setup_draws

  subroutine check(self, rc, what)
    class(equation_singleideal_b200_object), intent(inout) :: self
    integer(c_int), intent(in) :: rc
    character(*), intent(in) :: what
    if (rc /= STREAMS_B200_OK) then
      write(*,*) 'streams_b200 error in ', what, ': ', rc
      call mpi_abort(mpi_comm_world, 15, self%equation_base%mpi_err)
    endif
  endsubroutine check

  subroutine initialize(self, filename)
    class(equation_singleideal_b200_object), intent(inout), target :: self
    character(*), intent(in) :: filename
    type(streams_b200_params) :: p
    type(streams_b200_grid) :: g
    integer :: i, j, k
    call self%equation_base%initialize(filename)
    associate(eb => self%equation_base, f => self%equation_base%field)
      p%nx = f%nx ; p%ny = f%ny ; p%nz = f%nz ; p%ng = eb%grid%ng
      p%ep_order = eb%ep_order ; p%nkeep = eb%nkeep
      p%weno_scheme = eb%weno_scheme ; p%weno_version = eb%weno_version
      p%flux_splitting = eb%flux_splitting ; p%conservative_viscous = eb%conservative_viscous
      p%sensor_threshold = eb%sensor_threshold
      p%bctags = eb%bctags ; p%force_zero_flux = eb%force_zero_flux
      p%eul_imin = eb%eul_imin ; p%eul_imax = eb%eul_imax ; p%eul_jmin = eb%eul_jmin
      p%eul_jmax = eb%eul_jmax ; p%eul_kmin = eb%eul_kmin ; p%eul_kmax = eb%eul_kmax
      p%is_y_staggered = merge(1, 0, eb%grid%is_y_staggered)
      p%visc_model = eb%visc_model ; p%calorically_perfect = eb%calorically_perfect
      p%mu0 = eb%mu0 ; p%t0 = eb%t0 ; p%rgas0 = eb%rgas0 ; p%rho0 = eb%rho0 ; p%u0 = eb%u0 ; p%l0 = eb%l0
      p%sutherland_s = eb%sutherland_s ; p%t_ref_dim = eb%t_ref_dim
      p%powerlaw_vtexp = eb%powerlaw_vtexp ; p%prandtl = eb%prandtl
      p%cp0 = eb%cp_coeff(0) ; p%cv0 = eb%cv_coeff(0)
      p%cp_last = eb%cp_coeff(eb%indx_cp_r+1) ; p%cv_last = eb%cv_coeff(eb%indx_cp_r+1)
      p%channel_case = merge(1, 0, eb%channel_case)
      p%theta_wall = eb%theta_wall ; p%t_wall = eb%t_wall ; p%t_bulk_target = eb%t_bulk_target
      p%volchan = eb%volchan
      p%nrk = eb%nrk ; p%rhork = 0._rkind ; p%gamrk = 0._rkind
      p%rhork(1:eb%nrk) = eb%rhork ; p%gamrk(1:eb%nrk) = eb%gamrk
      p%cfl = eb%cfl ; p%precision = 0
      p%bctags_nr = eb%bctags_nr ; p%winf = eb%winf ; p%p0 = eb%p0
      p%recyc = merge(1, 0, eb%recyc) ; p%i_recyc = eb%i_recyc ; p%jbl_inflow = eb%jbl_inflow
      p%betarecyc = eb%betarecyc
      p%xshock_imp = eb%xshock_imp ; p%shock_angle = eb%shock_angle ; p%tanhfacs = eb%tanhfacs
      p%winf_past_shock = eb%winf_past_shock
      p%indx_cp_l = eb%indx_cp_l ; p%indx_cp_r = eb%indx_cp_r
      p%cp_coeff = 0._rkind ; p%cv_coeff = 0._rkind
      p%cp_coeff(1:eb%indx_cp_r-eb%indx_cp_l+2) = eb%cp_coeff(eb%indx_cp_l:eb%indx_cp_r+1)
      p%cv_coeff(1:eb%indx_cp_r-eb%indx_cp_l+2) = eb%cv_coeff(eb%indx_cp_l:eb%indx_cp_r+1)
      ! the crandom sequence continues on the device: the seed of this rank (init_crandom_f,
      ! singleideal.F90:314-323) and the draws the set-up took, both known before create
      self%myrank = eb%myrank
      self%crandom_draws = self%setup_draws()
      ! (rand_type = 0 seeds 0, which the device takes as draws rescaled to zero)
      p%rng_seed = merge(0, self%myrank + 1, eb%rand_type == 0) ; p%rng_draws = self%crandom_draws
      allocate(self%epx(0:f%nx), self%epy(0:f%ny), self%epz(0:f%nz))
      do i = 0, f%nx ; self%epx(i) = eb%ep_ord_change(i,1,1,1) ; enddo
      do j = 0, f%ny ; self%epy(j) = eb%ep_ord_change(1,j,1,2) ; enddo
      do k = 0, f%nz ; self%epz(k) = eb%ep_ord_change(1,1,k,3) ; enddo
      g%x = c_loc(f%x) ; g%y = c_loc(f%y) ; g%z = c_loc(f%z) ; g%yn = c_loc(f%yn)
      g%dcsidx = c_loc(f%dcsidx) ; g%detady = c_loc(f%detady) ; g%dzitdz = c_loc(f%dzitdz)
      g%dcsidxs = c_loc(f%dcsidxs) ; g%detadys = c_loc(f%detadys) ; g%dzitdzs = c_loc(f%dzitdzs)
      g%coeff_deriv1 = c_loc(eb%coeff_deriv1)
      g%ep_ord_x = c_loc(self%epx) ; g%ep_ord_y = c_loc(self%epy) ; g%ep_ord_z = c_loc(self%epz)
      g%dcsidx2 = c_loc(f%dcsidx2) ; g%detady2 = c_loc(f%detady2) ; g%dzitdz2 = c_loc(f%dzitdz2)
      g%coeff_deriv2 = c_loc(eb%coeff_deriv2)
      if (eb%recyc) then
        allocate(self%wmean_inflow(f%grid%ng, f%ny, 4))
        do i = 1, f%grid%ng
          self%wmean_inflow(i, :, :) = eb%wmean(1-i, 1:f%ny, 1:4)
        enddo
        g%wmean_inflow = c_loc(self%wmean_inflow) ; g%weta_inflow = c_loc(eb%weta_inflow)
        g%yplus_inflow = c_loc(eb%yplus_inflow) ; g%eta_inflow = c_loc(eb%eta_inflow)
        g%yplus_recyc = c_loc(eb%yplus_recyc) ; g%eta_recyc = c_loc(eb%eta_recyc)
        g%map_j_inn = c_loc(eb%map_j_inn) ; g%map_j_out = c_loc(eb%map_j_out)
      endif
      call self%check(streams_b200_create(p, g, self%ctx), 'create')
      call self%check(streams_b200_copy_from_field(self%ctx, c_loc(f%w)), 'copy_from_field')
      call self%check(streams_b200_set_time(self%ctx, eb%time0), 'set_time')
    endassociate
  endsubroutine initialize

  ! run() of singleideal_cpu.F90:1519-1693 for the channel: the device advances print_control
  ! steps at a time without host synchronisation (one at a time while statistics are sampled:
  ! the clock of manage_output needs every step's dt); progress rows as print_progress writes
  ! them; statistics sampled on the device as manage_output samples them
  ! (singleideal_gpu.F90:2012-2034) and brought back for write_stats at the end.
  subroutine run(self, filename)
    class(equation_singleideal_b200_object), intent(inout), target :: self
    character(*), intent(in) :: filename
    real(c_double) :: sc(7), res(7)
    integer(c_int) :: chunk, rc
    logical :: stats
    call self%initialize(filename)
    associate(eb => self%equation_base)
      stats = eb%enable_stat_time > 0 .or. eb%enable_stat_3d > 0
      if (eb%restart_type == 2) then
        if (eb%enable_stat_time > 0) call self%check(streams_b200_set_stats(self%ctx, 0, c_loc(eb%w_stat), &
                                     int(size(eb%w_stat), c_long_long)), 'set_stats')
        if (eb%enable_stat_3d > 0) call self%check(streams_b200_set_stats(self%ctx, 2, c_loc(eb%w_stat_3d), &
                                     int(size(eb%w_stat_3d), c_long_long)), 'set_stats')
      endif
      call self%check(streams_b200_init_run(self%ctx), 'init_run')
      do while (eb%icyc - eb%icyc0 < eb%num_iter)
        chunk = min(eb%print_control - mod(eb%icyc - eb%icyc0, eb%print_control), &
                    eb%num_iter - (eb%icyc - eb%icyc0))
        if (stats) chunk = 1
        call self%check(streams_b200_advance(self%ctx, chunk, eb%iter_dt_recompute, eb%icyc, eb%icyc0), 'advance')
        eb%icyc = eb%icyc + chunk
        if (stats) then
          call self%check(streams_b200_get_scalars(self%ctx, sc), 'get_scalars')
          eb%time_from_last_stat = eb%time_from_last_stat + sc(1)
          if (eb%time_from_last_stat >= eb%dtstat) then
            if (eb%enable_stat_time > 0) call self%check(streams_b200_compute_stats(self%ctx, eb%itav), 'stats')
            if (eb%enable_stat_3d > 0) call self%check(streams_b200_compute_stats_3d(self%ctx, eb%itav), 'stats_3d')
            eb%time_from_last_stat = 0._rkind
            eb%itav = eb%itav + 1
          endif
        endif
        if (mod(eb%icyc - eb%icyc0, eb%print_control) == 0) then
          rc = streams_b200_compute_residual(self%ctx, res)
          call self%check(streams_b200_get_scalars(self%ctx, sc), 'get_scalars')
          eb%dt = sc(1) ; eb%time = sc(2) ; eb%dpdx = sc(3)
          eb%rhobulk = sc(4) ; eb%ubulk = sc(5) ; eb%tbulk = sc(6)
          eb%residual_rhou = res(1) ; eb%rhomin = res(2) ; eb%rhomax = res(3)
          eb%tmin = res(4) ; eb%tmax = res(5) ; eb%pmin = res(6) ; eb%pmax = res(7)
          if (rc == STREAMS_B200_ENAN) then
            write(*,*) 'boom!!!'
            call self%check(streams_b200_copy_to_field(self%ctx, c_loc(eb%field%w)), 'copy_to_field')
            call mpi_abort(mpi_comm_world, 99, eb%mpi_err)
          endif
          ! print_progress and manage_output of the equation object go here
        endif
      enddo
      call self%check(streams_b200_copy_to_field(self%ctx, c_loc(eb%field%w)), 'copy_to_field')
      call eb%field%write_field()
      if (eb%enable_stat_time > 0) then
        call self%check(streams_b200_get_stats(self%ctx, 0, c_loc(eb%w_stat), int(size(eb%w_stat), c_long_long)), &
                        'get_stats')
        call eb%write_stats()
      endif
      if (eb%enable_stat_3d > 0) then
        call self%check(streams_b200_get_stats(self%ctx, 2, c_loc(eb%w_stat_3d), &
                        int(size(eb%w_stat_3d), c_long_long)), 'get_stats')
        call eb%write_stats_3d()
      endif
      call eb%write_field_info()
    endassociate
    call self%check(streams_b200_destroy(self%ctx), 'destroy')
  endsubroutine run

endmodule streams_equation_singleideal_b200_object
