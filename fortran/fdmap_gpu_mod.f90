! fdmap_gpu_mod -- ISO_C_BINDING interfaces to the B200 time-stepping engine
! (include/fdmap_gpu.h, include/fdmap_host.h).
!
! A Fortran driver keeps its own init_domain and time loop (main.f90) and
! hands the domain to the engine once; fdmap_gpu_time_step then replaces the
! body of time_step_LS (time_step.f90:96-165) for one step.  The descriptor
! (type(fdmap_desc_t) below mirrors struct fdmap_desc field by field) holds
! plain values and c_loc() pointers to the driver's own arrays:
!   F(C%mx:C%px, C%my:C%py, nF) -> F      (no ghost layers: pass F(mx:px,my:py,:)
!                                          through a contiguous copy when the
!                                          driver keeps ghosts)
!   G%xq, G%xr, G%yq, G%yr, G%J, G%Ji -> metric pointers, same layout
!   BF%bndFL%M(:,1:5), %F0, B%bndL%n  -> fdmap_side_t of each block side
!   I%nhat, I%x, I%y, I%FR%...        -> fdmap_iface_t / fdmap_friction_t
! Every routine returns 0 or a negative FDMAP_ERR_* code; none aborts.
module fdmap_gpu_mod

  use, intrinsic :: iso_c_binding, only : c_int, c_double, c_ptr, c_char, c_long_long, c_null_ptr, c_funptr

  implicit none

  integer(c_int), parameter :: FDMAP_OK = 0, FDMAP_ERR_INVALID_ARG = -1, FDMAP_ERR_CUDA = -2, &
       FDMAP_ERR_NONFINITE = -3, FDMAP_ERR_NEWTON_NOCONV = -4, FDMAP_ERR_TIMEOUT = -5, &
       FDMAP_ERR_UNSUPPORTED = -6, FDMAP_ERR_IO = -7, FDMAP_ERR_NOMEM = -8

  ! fault fields, in checkpoint_friction order (friction.f90:528-546)
  integer(c_int), parameter :: FDMAP_OUT_FAULT = 0, FDMAP_OUT_BODY = 1

  integer(c_int), parameter :: FDMAP_FAULT_D = 0, FDMAP_FAULT_PSI = 1, FDMAP_FAULT_DPSI = 2, &
       FDMAP_FAULT_TRUP = 3, FDMAP_FAULT_V = 4, FDMAP_FAULT_O = 5, FDMAP_FAULT_S = 6, &
       FDMAP_FAULT_N = 7, FDMAP_FAULT_S0 = 8, FDMAP_FAULT_N0 = 9, FDMAP_FAULT_DS = 10, &
       FDMAP_FAULT_DN = 11, FDMAP_FAULT_DDS = 12, FDMAP_FAULT_DDN = 13, FDMAP_FAULT_W = 14, &
       FDMAP_FAULT_DW = 15, FDMAP_FAULT_NREG = 16, FDMAP_FAULT_DNREG = 17

  type, bind(C) :: fdmap_side_t
     integer(c_int) :: bc, n
     type(c_ptr) :: M, F0, normal, x, y
  end type fdmap_side_t

  type, bind(C) :: fdmap_block_t
     integer(c_int) :: mgx, pgx, mgy, pgy
     real(c_double) :: rho, cs, cp, G, M, gamma, nu
     real(c_double) :: F0(9)
     type(fdmap_side_t) :: side(4)
     integer(c_int) :: src_ok, src_i0, src_j0
     real(c_double) :: src_hx, src_hy, src_ax, src_ay
     real(c_double) :: Cdiss
     integer(c_int) :: pmlx, pmly                ! pml_list (material.f90:152-222)
     real(c_double) :: pml_n, pml_sigma, pml_kappa, pml_mx, pml_px, pml_my, pml_py
  end type fdmap_block_t

  type, bind(C) :: fdmap_friction_t
     integer(c_int) :: law, reg, rup_field
     real(c_double) :: rup_threshold, angle, xlockm, xlockp, flock, skempton
     integer(c_int) :: force
     real(c_double) :: kn_c0, kn_fd, kn_dfdx, kn_vL, kn_vR, kn_xL, kn_xR, kn_tmax
     integer(c_int) :: ld_shape
     real(c_double) :: ld_S, ld_N, ld_T, ld_R, ld_x0, ld_y0
     integer(c_int) :: tp_use
     real(c_double) :: tp_p0
     type(c_ptr) :: a, b, V0, f0, L, fw, Vw, c0, fs, fd, Dc, bsS0, bsN0
     type(c_ptr) :: V, O, S, N, S0, N0, Ds, Dn, DDs, DDn, Psi, DPsi, D, trup, W, DW, Nreg, DNreg
  end type fdmap_friction_t

  type, bind(C) :: fdmap_iface_t
     integer(c_int) :: direction, iblockm, iblockp, m, p, coupling
     type(c_ptr) :: nhat, x, y
     type(fdmap_friction_t) :: fr
  end type fdmap_iface_t

  type, bind(C) :: fdmap_source_t
     integer(c_int) :: use_singular, use_gravity, stf
     real(c_double) :: x0, y0, t_center, t_duration, Fx, Fy, Fz, Mxx, Mxy, Myy, Mzx, Mzy, gx, gy, gz
     integer(c_int) :: gauss_forcing            ! problem = 'Forcing' (source.f90:299-312)
     real(c_double) :: gauss_amp, gauss_sigma, gauss_sigmat
     type(c_ptr) :: forcing_filename            ! C string, or c_null_ptr (source.f90:409-502)
  end type fdmap_source_t

  type, bind(C) :: fdmap_desc_t
     integer(c_int) :: mode, nF, fd_method, rk_order, nx, ny, nblocks, nifaces
     type(c_ptr) :: blocks, ifaces
     integer(c_int) :: heterogeneous
     type(c_ptr) :: F, DF, x, y, xq, xr, yq, yr, J, Ji
     type(c_ptr) :: rho, cs, cp, G, M, gamma, nu
     type(fdmap_source_t) :: src
     real(c_double) :: t0, dt, CFL
     integer(c_int) :: nt
     real(c_double) :: hmin, hmax
     type(c_ptr) :: body          ! fdmap_body_t, or c_null_ptr: body arrays given by the host
     integer(c_int) :: displacement, peak  ! domain_list displacement, peak (F%displacement, F%peak)
     integer(c_int) :: energy_balance      ! domain_list energy_balance (F%energy_balance)
  end type fdmap_desc_t

  ! on-device initialisation (fdmap_desc.h: fdmap_perturb, fdmap_block_body, fdmap_body)
  type, bind(C) :: fdmap_perturb_t
     integer(c_int) :: shape
     real(c_double) :: x0, y0, Lx, Ly
     real(c_double) :: v(6)
  end type fdmap_perturb_t

  type, bind(C) :: fdmap_block_body_t
     real(c_double) :: LB(2), LT(2), RB(2), RT(2)
     real(c_double) :: F0(6)
     type(fdmap_perturb_t) :: p(5)
     real(c_double) :: Cdiss
     type(c_ptr) :: side_mat(4)
  end type fdmap_block_body_t

  type, bind(C) :: fdmap_body_t
     type(c_ptr) :: blocks
     real(c_double) :: dt_in, CFL_in, refine, tend
     integer(c_int) :: nt_in
     real(c_double) :: c
  end type fdmap_body_t

  interface

     ! ---- engine (include/fdmap_gpu.h)
     integer(c_int) function fdmap_gpu_create(d, device, init_edges, h) bind(C, name='fdmap_gpu_create')
       import :: c_int, c_ptr
       type(c_ptr), value :: d
       integer(c_int), value :: device, init_edges
       type(c_ptr), intent(out) :: h
     end function fdmap_gpu_create

     integer(c_int) function fdmap_gpu_init_edges(h, t) bind(C, name='fdmap_gpu_init_edges')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), value :: t
     end function fdmap_gpu_init_edges

     integer(c_int) function fdmap_gpu_time_step(h, t0, dt, final_step) bind(C, name='fdmap_gpu_time_step')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), value :: t0, dt
       integer(c_int), value :: final_step
     end function fdmap_gpu_time_step

     integer(c_int) function fdmap_gpu_run(h, t_start, dt, n_first, n_last, nt) bind(C, name='fdmap_gpu_run')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), value :: t_start, dt
       integer(c_int), value :: n_first, n_last, nt
     end function fdmap_gpu_run

     integer(c_int) function fdmap_gpu_synchronize(h) bind(C, name='fdmap_gpu_synchronize')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function fdmap_gpu_synchronize

     integer(c_int) function fdmap_gpu_get_fields(h, F, DF) bind(C, name='fdmap_gpu_get_fields')
       import :: c_int, c_ptr
       type(c_ptr), value :: h, F, DF
     end function fdmap_gpu_get_fields

     integer(c_int) function fdmap_gpu_set_fields(h, F, DF) bind(C, name='fdmap_gpu_set_fields')
       import :: c_int, c_ptr
       type(c_ptr), value :: h, F, DF
     end function fdmap_gpu_set_fields

     integer(c_int) function fdmap_gpu_get_fault(h, iface, field, out) bind(C, name='fdmap_gpu_get_fault')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: iface, field
       real(c_double), intent(out) :: out(*)
     end function fdmap_gpu_get_fault

     integer(c_int) function fdmap_gpu_set_fault(h, iface, field, in) bind(C, name='fdmap_gpu_set_fault')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: iface, field
       real(c_double), intent(in) :: in(*)
     end function fdmap_gpu_set_fault

     integer(c_int) function fdmap_gpu_status(h, newton_failures) bind(C, name='fdmap_gpu_status')
       import :: c_int, c_ptr, c_long_long
       type(c_ptr), value :: h
       integer(c_long_long), intent(out) :: newton_failures
     end function fdmap_gpu_status

     integer(c_int) function fdmap_gpu_newton_counts(h, counts) bind(C, name='fdmap_gpu_newton_counts')
       import :: c_int, c_ptr, c_long_long
       type(c_ptr), value :: h
       integer(c_long_long), intent(out) :: counts(2)   ! first-attempt failures, failed retries
     end function fdmap_gpu_newton_counts

     integer(c_int) function fdmap_gpu_clear_status(h) bind(C, name='fdmap_gpu_clear_status')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function fdmap_gpu_clear_status

     integer(c_int) function fdmap_gpu_set_newton_limit(h, imax) bind(C, name='fdmap_gpu_set_newton_limit')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: imax
     end function fdmap_gpu_set_newton_limit

     integer(c_int) function fdmap_gpu_test_wait_timeout(h, limit_s) bind(C, name='fdmap_gpu_test_wait_timeout')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), value :: limit_s
     end function fdmap_gpu_test_wait_timeout

     integer(c_int) function fdmap_gpu_set_tile(h, tile) bind(C, name='fdmap_gpu_set_tile')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: tile
     end function fdmap_gpu_set_tile

     integer(c_int) function fdmap_gpu_get_tile(h, tile, mw, mr) bind(C, name='fdmap_gpu_get_tile')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), intent(out) :: tile, mw, mr
     end function fdmap_gpu_get_tile

     integer(c_int) function fdmap_gpu_tune(h, dt, steps, tile, ms) bind(C, name='fdmap_gpu_tune')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), value :: dt
       integer(c_int), value :: steps
       integer(c_int), intent(out) :: tile
       real(c_double), intent(out) :: ms
     end function fdmap_gpu_tune

     ! two-stage interior passes: stages (1,2), (3,4) of a step in one pass
     ! each, bit-identical to stage by stage; on by default where the domain
     ! allows them; get_pairs returns 1 (in use), 0 or a negative code
     integer(c_int) function fdmap_gpu_set_pairs(h, enable) bind(C, name='fdmap_gpu_set_pairs')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: enable
     end function fdmap_gpu_set_pairs

     integer(c_int) function fdmap_gpu_get_pairs(h) bind(C, name='fdmap_gpu_get_pairs')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function fdmap_gpu_get_pairs

     integer(c_int) function fdmap_gpu_create_part(d, device, owned, h) bind(C, name='fdmap_gpu_create_part')
       import :: c_int, c_ptr
       type(c_ptr), value :: d
       integer(c_int), value :: device
       integer(c_int), intent(in) :: owned(*)   ! 1 for every block this GPU steps
       type(c_ptr), intent(out) :: h
     end function fdmap_gpu_create_part

     integer(c_int) function fdmap_gpu_part_buffers(h, iface, stage, send, recv, count) &
          bind(C, name='fdmap_gpu_part_buffers')
       import :: c_int, c_ptr, c_long_long
       type(c_ptr), value :: h
       integer(c_int), value :: iface
       integer(c_long_long), value :: stage
       type(c_ptr), intent(out) :: send, recv     ! device pointers
       integer(c_long_long), intent(out) :: count
     end function fdmap_gpu_part_buffers

     integer(c_int) function fdmap_gpu_set_exchange(h, fn, user) bind(C, name='fdmap_gpu_set_exchange')
       import :: c_int, c_ptr, c_funptr
       type(c_ptr), value :: h
       type(c_funptr), value :: fn     ! integer(c_int) function(user, stage, stream) bind(C)
       type(c_ptr), value :: user
     end function fdmap_gpu_set_exchange

     integer(c_int) function fdmap_gpu_group_init_edges(hs, n, t) bind(C, name='fdmap_gpu_group_init_edges')
       import :: c_int, c_ptr, c_double
       type(c_ptr), intent(in) :: hs(*)
       integer(c_int), value :: n
       real(c_double), value :: t
     end function fdmap_gpu_group_init_edges

     integer(c_int) function fdmap_gpu_group_run(hs, n, t_start, dt, n_first, n_last, nt) &
          bind(C, name='fdmap_gpu_group_run')
       import :: c_int, c_ptr, c_double
       type(c_ptr), intent(in) :: hs(*)
       integer(c_int), value :: n, n_first, n_last, nt
       real(c_double), value :: t_start, dt
     end function fdmap_gpu_group_run

     integer(c_int) function fdmap_gpu_check_finite(h, count) bind(C, name='fdmap_gpu_check_finite')
       import :: c_int, c_ptr, c_long_long
       type(c_ptr), value :: h
       integer(c_long_long), intent(out) :: count   ! returns FDMAP_ERR_NONFINITE (-3) when count > 0
     end function fdmap_gpu_check_finite

     integer(c_int) function fdmap_gpu_time_params(h, params, nt) bind(C, name='fdmap_gpu_time_params')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(out) :: params(5)   ! t0, dt, CFL, hmin, hmax
       integer(c_int), intent(out) :: nt
     end function fdmap_gpu_time_params

     integer(c_int) function fdmap_gpu_get_metric(h, which, out) bind(C, name='fdmap_gpu_get_metric')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: which              ! 0 xq, 1 xr, 2 yq, 3 yr, 4 Ji, 5 J
       real(c_double), intent(out) :: out(*)
     end function fdmap_gpu_get_metric

     integer(c_int) function fdmap_gpu_get_pml(h, which, out) bind(C, name='fdmap_gpu_get_pml')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: which              ! 0 Wx, 1 Wy
       real(c_double), intent(out) :: out(*)       ! (nx, ny, nF)
     end function fdmap_gpu_get_pml

     integer(c_int) function fdmap_gpu_set_pml(h, which, in) bind(C, name='fdmap_gpu_set_pml')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: which
       real(c_double), intent(in) :: in(*)
     end function fdmap_gpu_set_pml

     integer(c_int) function fdmap_gpu_get_displacement(h, U, DU) bind(C, name='fdmap_gpu_get_displacement')
       import :: c_int, c_ptr
       type(c_ptr), value :: h, U, DU              ! (nx, ny, nU) each, or c_null_ptr
     end function fdmap_gpu_get_displacement

     integer(c_int) function fdmap_gpu_set_displacement(h, U, DU) bind(C, name='fdmap_gpu_set_displacement')
       import :: c_int, c_ptr
       type(c_ptr), value :: h, U, DU
     end function fdmap_gpu_set_displacement

     integer(c_int) function fdmap_gpu_get_peak(h, pgv, pga) bind(C, name='fdmap_gpu_get_peak')
       import :: c_int, c_ptr
       type(c_ptr), value :: h, pgv, pga           ! (nx, ny) each, or c_null_ptr
     end function fdmap_gpu_get_peak

     integer(c_int) function fdmap_gpu_set_peak(h, pgv, pga) bind(C, name='fdmap_gpu_set_peak')
       import :: c_int, c_ptr
       type(c_ptr), value :: h, pgv, pga
     end function fdmap_gpu_set_peak

     integer(c_int) function fdmap_gpu_get_energy(h, E) bind(C, name='fdmap_gpu_get_energy')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(out) :: E(*)         ! (nblocks + 1): Ebody, then Eblock per block
     end function fdmap_gpu_get_energy

     integer(c_int) function fdmap_gpu_get_side_displacement(h, b, s, U, DU) &
          bind(C, name='fdmap_gpu_get_side_displacement')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: b, s
       type(c_ptr), value :: U, DU                 ! (n, nU) each, or c_null_ptr
     end function fdmap_gpu_get_side_displacement

     integer(c_int) function fdmap_gpu_set_side_displacement(h, b, s, U, DU) &
          bind(C, name='fdmap_gpu_set_side_displacement')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: b, s
       type(c_ptr), value :: U, DU
     end function fdmap_gpu_set_side_displacement

     integer(c_int) function fdmap_gpu_get_side_impedance(h, b, s, out) bind(C, name='fdmap_gpu_get_side_impedance')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: b, s
       real(c_double), intent(out) :: out(*)
     end function fdmap_gpu_get_side_impedance

     subroutine fdmap_gpu_destroy(h) bind(C, name='fdmap_gpu_destroy')
       import :: c_ptr
       type(c_ptr), value :: h
     end subroutine fdmap_gpu_destroy

     integer(c_int) function fdmap_gpu_set_stream(h, stream) bind(C, name='fdmap_gpu_set_stream')
       import :: c_int, c_ptr
       type(c_ptr), value :: h, stream
     end function fdmap_gpu_set_stream

     integer(c_int) function fdmap_gpu_get_fhat(h, b, s, out) bind(C, name='fdmap_gpu_get_fhat')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: b, s
       real(c_double), intent(out) :: out(*)
     end function fdmap_gpu_get_fhat

     integer(c_int) function fdmap_gpu_fault_max_noalloc(h, iface, field, out) bind(C, name='fdmap_gpu_fault_max_noalloc')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: iface, field
       real(c_double), intent(out) :: out
     end function fdmap_gpu_fault_max_noalloc

     ! ---- device-side output (write_output replacement)
     integer(c_int) function fdmap_gpu_output_add(h, name, kind, index, field, mx, px, sx, my, py, sy, &
          nmin, nmax, stride) bind(C, name='fdmap_gpu_output_add')
       import :: c_int, c_ptr, c_char, c_long_long
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: name(*)
       integer(c_int), value :: kind, index, field, mx, px, sx, my, py, sy, stride
       integer(c_long_long), value :: nmin, nmax
     end function fdmap_gpu_output_add

     integer(c_int) function fdmap_gpu_output_open(h, prefix, ring_steps) bind(C, name='fdmap_gpu_output_open')
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: prefix(*)
       integer(c_int), value :: ring_steps
     end function fdmap_gpu_output_open

     integer(c_int) function fdmap_gpu_output_flush(h) bind(C, name='fdmap_gpu_output_flush')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function fdmap_gpu_output_flush

     integer(c_int) function fdmap_gpu_output_close(h) bind(C, name='fdmap_gpu_output_close')
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function fdmap_gpu_output_close

     ! ---- batched ensemble
     integer(c_int) function fdmap_gpu_ensemble_create(descs, ninst, device, init_edges, e) &
          bind(C, name='fdmap_gpu_ensemble_create')
       import :: c_int, c_ptr
       type(c_ptr), intent(in) :: descs(*)
       integer(c_int), value :: ninst, device, init_edges
       type(c_ptr), intent(out) :: e
     end function fdmap_gpu_ensemble_create

     integer(c_int) function fdmap_gpu_ensemble_instance(e, k, h) bind(C, name='fdmap_gpu_ensemble_instance')
       import :: c_int, c_ptr
       type(c_ptr), value :: e
       integer(c_int), value :: k
       type(c_ptr), intent(out) :: h
     end function fdmap_gpu_ensemble_instance

     integer(c_int) function fdmap_gpu_ensemble_run(e, t_start, dt, n_first, n_last, nt) &
          bind(C, name='fdmap_gpu_ensemble_run')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: e
       real(c_double), value :: t_start, dt
       integer(c_int), value :: n_first, n_last, nt
     end function fdmap_gpu_ensemble_run

     integer(c_int) function fdmap_gpu_ensemble_tune(e, dt, steps, best_shape, best_ms) &
          bind(C, name='fdmap_gpu_ensemble_tune')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: e
       real(c_double), value :: dt
       integer(c_int), value :: steps
       integer(c_int), intent(out) :: best_shape(3)
       real(c_double), intent(out) :: best_ms
     end function fdmap_gpu_ensemble_tune

     subroutine fdmap_gpu_ensemble_destroy(e) bind(C, name='fdmap_gpu_ensemble_destroy')
       import :: c_ptr
       type(c_ptr), value :: e
     end subroutine fdmap_gpu_ensemble_destroy

     ! ---- forward/backward pair (misfit gradient)
     integer(c_int) function fdmap_gpu_adjoint_create(d, device, nrec, rec_i, rec_j, checkpoint_every, a) &
          bind(C, name='fdmap_gpu_adjoint_create')
       import :: c_int, c_ptr
       type(c_ptr), value :: d
       integer(c_int), value :: device, nrec, checkpoint_every
       integer(c_int), intent(in) :: rec_i(*), rec_j(*)
       type(c_ptr), intent(out) :: a
     end function fdmap_gpu_adjoint_create

     integer(c_int) function fdmap_gpu_adjoint_set_material(a, rho, G) bind(C, name='fdmap_gpu_adjoint_set_material')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: a
       real(c_double), intent(in) :: rho(*), G(*)
     end function fdmap_gpu_adjoint_set_material

     integer(c_int) function fdmap_gpu_adjoint_forward(a, t_start, dt, nt, data, traces, misfit) &
          bind(C, name='fdmap_gpu_adjoint_forward')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: a, data, traces
       real(c_double), value :: t_start, dt
       integer(c_int), value :: nt
       real(c_double), intent(out) :: misfit
     end function fdmap_gpu_adjoint_forward

     integer(c_int) function fdmap_gpu_adjoint_backward(a, grad_rho, grad_G) bind(C, name='fdmap_gpu_adjoint_backward')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: a
       real(c_double), intent(out) :: grad_rho(*), grad_G(*)
     end function fdmap_gpu_adjoint_backward

     integer(c_int) function fdmap_gpu_adjoint_time_params(a, params, nt) bind(C, name='fdmap_gpu_adjoint_time_params')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: a
       real(c_double), intent(out) :: params(5)     ! t0, dt, CFL, hmin, hmax
       integer(c_int), intent(out) :: nt
     end function fdmap_gpu_adjoint_time_params

     integer(c_int) function fdmap_gpu_adjoint_fault_size(a) bind(C, name='fdmap_gpu_adjoint_fault_size')
       import :: c_int, c_ptr
       type(c_ptr), value :: a
     end function fdmap_gpu_adjoint_fault_size

     integer(c_int) function fdmap_gpu_adjoint_set_prestress(a, S0) bind(C, name='fdmap_gpu_adjoint_set_prestress')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: a
       real(c_double), intent(in) :: S0(*)           ! fault nodes of all interfaces, in interface order
     end function fdmap_gpu_adjoint_set_prestress

     integer(c_int) function fdmap_gpu_adjoint_get_prestress(a, S0) bind(C, name='fdmap_gpu_adjoint_get_prestress')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: a
       real(c_double), intent(out) :: S0(*)
     end function fdmap_gpu_adjoint_get_prestress

     integer(c_int) function fdmap_gpu_adjoint_prestress_gradient(a, grad_S0) &
          bind(C, name='fdmap_gpu_adjoint_prestress_gradient')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: a
       real(c_double), intent(out) :: grad_S0(*)
     end function fdmap_gpu_adjoint_prestress_gradient

     integer(c_int) function fdmap_gpu_adjoint_set_store_budget(a, bytes) &
          bind(C, name='fdmap_gpu_adjoint_set_store_budget')
       import :: c_int, c_ptr, c_long_long
       type(c_ptr), value :: a
       integer(c_long_long), value :: bytes
     end function fdmap_gpu_adjoint_set_store_budget

     integer(c_long_long) function fdmap_gpu_adjoint_segment_bytes(a) &
          bind(C, name='fdmap_gpu_adjoint_segment_bytes')
       import :: c_long_long, c_ptr
       type(c_ptr), value :: a
     end function fdmap_gpu_adjoint_segment_bytes

     integer(c_int) function fdmap_gpu_adjoint_resident_segments(a) &
          bind(C, name='fdmap_gpu_adjoint_resident_segments')
       import :: c_int, c_ptr
       type(c_ptr), value :: a
     end function fdmap_gpu_adjoint_resident_segments

     subroutine fdmap_gpu_adjoint_destroy(a) bind(C, name='fdmap_gpu_adjoint_destroy')
       import :: c_ptr
       type(c_ptr), value :: a
     end subroutine fdmap_gpu_adjoint_destroy

     ! ---- host initialisation from an FDMAP input text (include/fdmap_host.h)
     integer(c_int) function fdmap_host_init(input_text, base_dir, dom) bind(C, name='fdmap_host_init')
       import :: c_int, c_ptr, c_char
       character(kind=c_char), intent(in) :: input_text(*), base_dir(*)
       type(c_ptr), intent(out) :: dom
     end function fdmap_host_init

     integer(c_int) function fdmap_host_init_ex(input_text, base_dir, flags, dom) bind(C, name='fdmap_host_init_ex')
       import :: c_int, c_ptr, c_char
       character(kind=c_char), intent(in) :: input_text(*), base_dir(*)
       integer(c_int), value :: flags               ! 1 = FDMAP_INIT_BODY_ON_DEVICE
       type(c_ptr), intent(out) :: dom
     end function fdmap_host_init_ex

     integer(c_int) function fdmap_host_set_spacing(dom, hmin, hmax) bind(C, name='fdmap_host_set_spacing')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: dom
       real(c_double), value :: hmin, hmax
     end function fdmap_host_set_spacing

     type(c_ptr) function fdmap_host_desc(dom) bind(C, name='fdmap_host_desc')
       import :: c_ptr
       type(c_ptr), value :: dom
     end function fdmap_host_desc

     subroutine fdmap_host_free(dom) bind(C, name='fdmap_host_free')
       import :: c_ptr
       type(c_ptr), value :: dom
     end subroutine fdmap_host_free

  end interface

end module fdmap_gpu_mod
