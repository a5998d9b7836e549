!
! mod_ixb.f90 -- ISO_C_BINDING interface of libixb (include/ixb.h) for the
! Ixchel2D Fortran driver.  A maintainer adds this module to
! source/CMakeLists.txt's SOURCE_FILES, links libixb.so, and replaces the
! ALGORITMO_SIMPLE body of source/main.f90:395-1217 (and the !$acc data
! region of :356-389 / :1277) by ixb_* calls: create the handle, set the
! mesh, parameters and boundary tables, upload the state, call ixb_step per
! time step, download for the writers, destroy the handle.
!
! The derived types mirror the C structs field by field (bind(C)); arrays
! keep the reference's Fortran shapes and are passed by reference.  Every
! function of ixb.h has an interface here; the batched line solves take
! device addresses (type(c_ptr), e.g. from an OpenACC host_data region).
!
module ixb
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: IXB_OK = 0, IXB_EINVAL = 1, IXB_ECUDA = 2, IXB_ENONFINITE = 3
  integer(c_int), parameter :: IXB_ETIMEOUT = 4, IXB_EBC = 5, IXB_ESTATE = 6, IXB_EIO = 7
  integer(c_int), parameter :: IXB_ENOMEM = 8
  integer(c_int), parameter :: IXB_PREC_FP64 = 0, IXB_PREC_FP32_REFINED = 1
  integer(c_int), parameter :: IXB_SOLVER_HYBRID = 0, IXB_SOLVER_EXACT = 1
  integer(c_int), parameter :: IXB_VAR_U = 0, IXB_VAR_V = 1, IXB_VAR_T = 2
  integer(c_int), parameter :: IXB_BC_OTHER = 0, IXB_BC_DIRI = 1, IXB_BC_NEUM = 2
  integer(c_int), parameter :: IXB_MESH_UNIF = 0, IXB_MESH_TUBO = 1, IXB_MESH_CENT = 2, IXB_MESH_TANH = 3
  integer(c_int), parameter :: IXB_BODY_BOX = 0, IXB_BODY_REGION = 1, IXB_BODY_TRIAN = 2, IXB_BODY_CUADR = 3
  integer(c_int), parameter :: IXB_BODY_CHIME = 4, IXB_BODY_VEL = 1, IXB_BODY_TEMP = 2

  type, bind(C) :: ixb_params
     real(c_double) :: gamma_momen, gamma_energ, Ri, Riy, dt
     real(c_double) :: rel_vel, rel_pres, rel_ener
     real(c_double) :: conv_u, conv_p, conv_t, conv_resi, conv_paso
     real(c_double) :: p_update
     integer(c_int) :: iter_ecuaci_max, iter_simple_max, solver
     integer(c_int) :: reserved(5)
  end type ixb_params

  type, bind(C) :: ixb_bc_side
     integer(c_int) :: side, ndivis
     integer(c_int) :: type(15)
     real(c_double) :: value(15)
     integer(c_int) :: index(16)
  end type ixb_bc_side

  type, bind(C) :: ixb_report
     real(c_double) :: maxbo, residuo, err_u, err_p, err_t
     integer(c_int64_t) :: n_simple, n_momen, n_pres, n_ener
     integer(c_int) :: exit_code, status
  end type ixb_report

  type, bind(C) :: ixb_nu_monitor
     integer(c_int) :: vertical, k0, k1, wall, every, reserved
     integer(c_int64_t) :: max_iters
     real(c_double) :: tol_dnu, tol_maxbo
  end type ixb_nu_monitor

  interface
     integer(c_int) function ixb_create(mi, nj, prec_mode, h) bind(C, name="ixb_create")
       import :: c_int, c_ptr
       integer(c_int), value :: mi, nj, prec_mode
       type(c_ptr) :: h
     end function ixb_create

     integer(c_int) function ixb_destroy(h) bind(C, name="ixb_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function ixb_destroy

     integer(c_int) function ixb_set_mesh(h, xu, yv, xp, yp) bind(C, name="ixb_set_mesh")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(in) :: xu(*), yv(*), xp(*), yp(*)
     end function ixb_set_mesh

     integer(c_int) function ixb_set_params(h, p) bind(C, name="ixb_set_params")
       import :: c_int, c_ptr, ixb_params
       type(c_ptr), value :: h
       type(ixb_params), intent(in) :: p
     end function ixb_set_params

     integer(c_int) function ixb_set_bc(h, var, sides) bind(C, name="ixb_set_bc")
       import :: c_int, c_ptr, ixb_bc_side
       type(c_ptr), value :: h
       integer(c_int), value :: var
       type(ixb_bc_side), intent(in) :: sides(4)
     end function ixb_set_bc

     integer(c_int) function ixb_set_sources(h, var, fcon, flin) bind(C, name="ixb_set_sources")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: var
       real(c_double), intent(in) :: fcon(*), flin(*)
     end function ixb_set_sources

     integer(c_int) function ixb_upload_state(h, u, v, p, T, u_ant, v_ant, T_ant) &
          bind(C, name="ixb_upload_state")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(in) :: u(*), v(*), p(*), T(*), u_ant(*), v_ant(*), T_ant(*)
     end function ixb_upload_state

     integer(c_int) function ixb_download_state(h, u, v, p, T, u_ant, v_ant, T_ant) &
          bind(C, name="ixb_download_state")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(out) :: u(*), v(*), p(*), T(*), u_ant(*), v_ant(*), T_ant(*)
     end function ixb_download_state

     integer(c_int) function ixb_simple_loop(h, rep) bind(C, name="ixb_simple_loop")
       import :: c_int, c_ptr, ixb_report
       type(c_ptr), value :: h
       type(ixb_report), intent(out) :: rep
     end function ixb_simple_loop

     integer(c_int) function ixb_download_state_async(h, u, v, p, T, u_ant, v_ant, T_ant) &
          bind(C, name="ixb_download_state_async")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       type(c_ptr), value :: u, v, p, T, u_ant, v_ant, T_ant  ! pinned host arrays (c_loc) or c_null_ptr
     end function ixb_download_state_async

     integer(c_int) function ixb_download_wait(h) bind(C, name="ixb_download_wait")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function ixb_download_wait

     integer(c_int) function ixb_host_alloc(bytes, p) bind(C, name="ixb_host_alloc")
       import :: c_int, c_ptr, c_size_t
       integer(c_size_t), value :: bytes
       type(c_ptr) :: p
     end function ixb_host_alloc

     integer(c_int) function ixb_host_free(p) bind(C, name="ixb_host_free")
       import :: c_int, c_ptr
       type(c_ptr), value :: p
     end function ixb_host_free

     integer(c_int) function ixb_simple_converge(h, mon, rep, nu, dnu) bind(C, name="ixb_simple_converge")
       import :: c_int, c_ptr, c_double, ixb_report, ixb_nu_monitor
       type(c_ptr), value :: h
       type(ixb_nu_monitor), intent(in) :: mon
       type(ixb_report), intent(out) :: rep
       real(c_double), intent(out) :: nu(2), dnu
     end function ixb_simple_converge

     integer(c_int) function ixb_step(h, rep) bind(C, name="ixb_step")
       import :: c_int, c_ptr, ixb_report
       type(c_ptr), value :: h
       type(ixb_report), intent(out) :: rep
     end function ixb_step

     integer(c_int) function ixb_nusselt_y(h, i0, i1, nu0, nu1) bind(C, name="ixb_nusselt_y")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: i0, i1
       real(c_double), intent(out) :: nu0, nu1
     end function ixb_nusselt_y

     integer(c_int) function ixb_read_bc_file(path, xx, mm, yy, nn, sides) bind(C, name="ixb_read_bc_file")
       import :: c_int, c_char, c_double, ixb_bc_side
       character(kind=c_char), intent(in) :: path(*)
       real(c_double), intent(in) :: xx(*), yy(*)
       integer(c_int), value :: mm, nn
       type(ixb_bc_side), intent(out) :: sides(4)
     end function ixb_read_bc_file
     integer(c_int) function ixb_simple_iterations(h, n, rep) bind(C, name="ixb_simple_iterations")
       import :: c_int, c_ptr, ixb_report
       type(c_ptr), value :: h
       integer(c_int), value :: n
       type(ixb_report), intent(out) :: rep
     end function ixb_simple_iterations

     integer(c_int) function ixb_nusselt_x(h, j0, j1, nu0, nu1) bind(C, name="ixb_nusselt_x")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: j0, j1
       real(c_double), intent(out) :: nu0, nu1
     end function ixb_nusselt_x

     integer(c_int) function ixb_body_sources(mi, nj, xp, yp, shape, prm, flags, t_value, fcon_u, flin_u, &
          fcon_v, flin_v, fcon_t, flin_t) bind(C, name="ixb_body_sources")
       import :: c_int, c_double
       integer(c_int), value :: mi, nj, shape, flags
       real(c_double), intent(in) :: xp(*), yp(*), prm(*)
       real(c_double), value :: t_value
       real(c_double), intent(inout) :: fcon_u(*), flin_u(*), fcon_v(*), flin_v(*), fcon_t(*), flin_t(*)
     end function ixb_body_sources

     integer(c_int) function ixb_staggered_mesh(mi, nj, xkind, xparam, ykind, yparam, ao, bo, xu, yv, xp, yp) &
          bind(C, name="ixb_staggered_mesh")
       import :: c_int, c_double
       integer(c_int), value :: mi, nj, xkind, ykind
       real(c_double), value :: xparam, yparam, ao, bo
       real(c_double), intent(out) :: xu(*), yv(*), xp(*), yp(*)
     end function ixb_staggered_mesh

     integer(c_int) function ixb_read_state_files(ufile, vfile, pfile, mi, nj, xu, yv, xp, yp, u, v, T, p, &
          i0, i1, iter, a) bind(C, name="ixb_read_state_files")
       import :: c_int, c_char, c_double
       character(kind=c_char), intent(in) :: ufile(*), vfile(*), pfile(*)
       integer(c_int), value :: mi, nj
       real(c_double), intent(out) :: xu(*), yv(*), xp(*), yp(*), u(*), v(*), T(*), p(*)
       integer(c_int), intent(out) :: i0, i1, iter
       real(c_double), intent(out) :: a
     end function ixb_read_state_files

     integer(c_int) function ixb_write_state_files(ufile, vfile, pfile, mi, nj, xu, yv, xp, yp, u, v, T, p, &
          i0, i1, iter, a) bind(C, name="ixb_write_state_files")
       import :: c_int, c_char, c_double
       character(kind=c_char), intent(in) :: ufile(*), vfile(*), pfile(*)
       integer(c_int), value :: mi, nj, i0, i1, iter
       real(c_double), intent(in) :: xu(*), yv(*), xp(*), yp(*), u(*), v(*), T(*), p(*)
       real(c_double), value :: a
     end function ixb_write_state_files

     integer(c_int) function ixb_batch_create(count, mi, nj, prec_mode, b) bind(C, name="ixb_batch_create")
       import :: c_int, c_ptr
       integer(c_int), value :: count, prec_mode
       integer(c_int), intent(in) :: mi(*), nj(*)
       type(c_ptr) :: b
     end function ixb_batch_create

     integer(c_int) function ixb_batch_destroy(b) bind(C, name="ixb_batch_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: b
     end function ixb_batch_destroy

     integer(c_int) function ixb_batch_instance(b, i, h) bind(C, name="ixb_batch_instance")
       import :: c_int, c_ptr
       type(c_ptr), value :: b
       integer(c_int), value :: i
       type(c_ptr) :: h
     end function ixb_batch_instance

     integer(c_int) function ixb_batch_restart(b) bind(C, name="ixb_batch_restart")
       import :: c_int, c_ptr
       type(c_ptr), value :: b
     end function ixb_batch_restart

     integer(c_int) function ixb_batch_iterate(b, max_iters, n_active) bind(C, name="ixb_batch_iterate")
       import :: c_int, c_ptr
       type(c_ptr), value :: b
       integer(c_int), value :: max_iters
       integer(c_int), intent(out) :: n_active
     end function ixb_batch_iterate

     integer(c_int) function ixb_batch_report(b, i, rep) bind(C, name="ixb_batch_report")
       import :: c_int, c_ptr, ixb_report
       type(c_ptr), value :: b
       integer(c_int), value :: i
       type(ixb_report), intent(out) :: rep
     end function ixb_batch_report
     ! ---- library, handle and diagnostics ----
     integer(c_int) function ixb_version() bind(C, name="ixb_version")
       import :: c_int
     end function ixb_version

     type(c_ptr) function ixb_strerror(status) bind(C, name="ixb_strerror")  ! a C string (c_f_pointer to read)
       import :: c_int, c_ptr
       integer(c_int), value :: status
     end function ixb_strerror

     integer(c_int) function ixb_device_count() bind(C, name="ixb_device_count")
       import :: c_int
     end function ixb_device_count

     integer(c_int) function ixb_set_stream(h, stream) bind(C, name="ixb_set_stream")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, stream          ! stream: a cudaStream_t
     end function ixb_set_stream

     integer(c_int) function ixb_download_aux(h, au, av, b_o, resu, corr_pres) bind(C, name="ixb_download_aux")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(out) :: au(*), av(*), b_o(*), resu(*), corr_pres(*)
     end function ixb_download_aux

     integer(c_int) function ixb_set_work(h, corr_pres, au, av) bind(C, name="ixb_set_work")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), intent(in) :: corr_pres(*), au(*), av(*)
     end function ixb_set_work

     integer(c_int) function ixb_roll(h) bind(C, name="ixb_roll")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function ixb_roll

     integer(c_int) function ixb_phase(h, which) bind(C, name="ixb_phase")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: which
     end function ixb_phase

     integer(c_int) function ixb_time_phases(h, reps, flush_bytes, ms) bind(C, name="ixb_time_phases")
       import :: c_int, c_ptr, c_size_t, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: reps
       integer(c_size_t), value :: flush_bytes
       real(c_double), intent(out) :: ms(*)
     end function ixb_time_phases

     ! ---- launch shapes ----
     integer(c_int) function ixb_set_sweep_shape(h, sweep, lines_per_cta, threads_per_line) &
          bind(C, name="ixb_set_sweep_shape")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: sweep, lines_per_cta, threads_per_line
     end function ixb_set_sweep_shape

     integer(c_int) function ixb_iteration_launches(h, launches) bind(C, name="ixb_iteration_launches")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), intent(out) :: launches
     end function ixb_iteration_launches

     integer(c_int) function ixb_autotune(h, reps, flush_bytes, chosen, ms) bind(C, name="ixb_autotune")
       import :: c_int, c_ptr, c_size_t, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: reps
       integer(c_size_t), value :: flush_bytes
       integer(c_int), intent(out) :: chosen(16)
       real(c_double), intent(out) :: ms(8)
     end function ixb_autotune

     integer(c_int) function ixb_batch_set_sweep_shape(b, sweep, lines_per_cta, threads_per_line) &
          bind(C, name="ixb_batch_set_sweep_shape")
       import :: c_int, c_ptr
       type(c_ptr), value :: b
       integer(c_int), value :: sweep, lines_per_cta, threads_per_line
     end function ixb_batch_set_sweep_shape

     integer(c_int) function ixb_batch_autotune(b, reps, chosen, ms) bind(C, name="ixb_batch_autotune")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: b
       integer(c_int), value :: reps
       integer(c_int), intent(out) :: chosen(16)
       real(c_double), intent(out) :: ms(8)
     end function ixb_batch_autotune

     ! ---- batched line solves on DEVICE arrays (a..x: device addresses) ----
     integer(c_int) function ixb_tridiag_f64(a, b, c, d, x, n, nsys, layout, solver, stream) &
          bind(C, name="ixb_tridiag_f64")
       import :: c_int, c_ptr
       type(c_ptr), value :: a, b, c, d, x, stream
       integer(c_int), value :: n, nsys, layout, solver
     end function ixb_tridiag_f64

     integer(c_int) function ixb_tridiag_f32(a, b, c, d, x, n, nsys, layout, solver, stream) &
          bind(C, name="ixb_tridiag_f32")
       import :: c_int, c_ptr
       type(c_ptr), value :: a, b, c, d, x, stream
       integer(c_int), value :: n, nsys, layout, solver
     end function ixb_tridiag_f32

     integer(c_int) function ixb_tridiag_f64_noalloc(a, b, c, d, x, n, nsys, layout, solver, stream) &
          bind(C, name="ixb_tridiag_f64_noalloc")
       import :: c_int, c_ptr
       type(c_ptr), value :: a, b, c, d, x, stream
       integer(c_int), value :: n, nsys, layout, solver
     end function ixb_tridiag_f64_noalloc

     integer(c_int) function ixb_tridiag_status() bind(C, name="ixb_tridiag_status")
       import :: c_int
     end function ixb_tridiag_status

     integer(c_int) function ixb_tridiag_set_first_wait_limit(polls) bind(C, name="ixb_tridiag_set_first_wait_limit")
       import :: c_int
       integer(c_int), value :: polls
     end function ixb_tridiag_set_first_wait_limit

     ! ---- energy equation with the flow held fixed, and its adjoint ----
     integer(c_int) function ixb_adjoint_simple(h, K, C, j0, j1, grad, nu0) bind(C, name="ixb_adjoint_simple")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: K, C, j0, j1
       type(c_ptr), value :: grad, nu0   ! real(c_double) arrays via c_loc (grad: nj+1 entries), or c_null_ptr
     end function ixb_adjoint_simple

     integer(c_int) function ixb_energy_iterations(h, n) bind(C, name="ixb_energy_iterations")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: n
     end function ixb_energy_iterations

     integer(c_int) function ixb_adjoint_energy(h, K, j0, j1, grad) bind(C, name="ixb_adjoint_energy")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: K, j0, j1
       real(c_double), intent(out) :: grad(*)
     end function ixb_adjoint_energy

     integer(c_int) function ixb_adjoint_energy_coupled(h, K, C, j0, j1, grad, nu0) &
          bind(C, name="ixb_adjoint_energy_coupled")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: K, C, j0, j1
       real(c_double), intent(out) :: grad(*)
       real(c_double), intent(out) :: nu0
     end function ixb_adjoint_energy_coupled

     integer(c_int) function ixb_set_bc_values(h, var, side, values) bind(C, name="ixb_set_bc_values")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: var, side
       real(c_double), intent(in) :: values(*)
     end function ixb_set_bc_values

     ! ---- host-side inputs ----
     integer(c_int) function ixb_mesh_axis(mkind, n, length, param, centre, nodes) bind(C, name="ixb_mesh_axis")
       import :: c_int, c_double
       integer(c_int), value :: mkind, n
       real(c_double), value :: length, param, centre
       real(c_double), intent(out) :: nodes(*)
     end function ixb_mesh_axis

     integer(c_int) function ixb_bc_locate(side, ndivis, x1, btype, bvalue, xx, mm, yy, nn, out) &
          bind(C, name="ixb_bc_locate")
       import :: c_int, c_double, ixb_bc_side
       integer(c_int), value :: side, ndivis, mm, nn
       real(c_double), intent(in) :: x1(*), bvalue(*), xx(*), yy(*)
       integer(c_int), intent(in) :: btype(*)
       type(ixb_bc_side), intent(out) :: out
     end function ixb_bc_locate

  end interface

end module ixb
