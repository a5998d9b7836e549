!
! ixb_driver.f90 -- PROGRAM IXCHEL2D's SIMPLE hot path on libixb, as the
! module a maintainer adds beside mod_ixb.f90 (module ixb).  Uncompiled: no
! Fortran compiler exists on this pool (gfortran, nvfortran, flang and
! lfortran were probed), so it is checked only by reading and by the
! interface test of tests/test_abi.py, which binds the same C functions.
!
! The module reads and writes the reference's own module arrays (malla,
! ec_momento, ec_energia), so source/main.f90 changes in four places only:
!
!   1. before the package loop `do ll = 1, itermax/paq_itera` (main.f90:347):
!          call ixb_arranque(IXB_PREC_FP64, dt, conv_resi, iter_ecuaci_max, &
!                            iter_simple_max)
!      (IXB_PREC_FP32_REFINED for the binary32 line solves with binary64
!      defect correction);
!   2. the `!$acc data` region that opens each package (main.f90:356-389) is
!      deleted: the library keeps the state on the device for the whole run;
!   3. inside `do kk=1,paq_itera`, the ALGORITMO_SIMPLE loop and the roll of
!      the time levels (main.f90:395-1217 and :1251-1270) become
!          call ixb_paso(maxbo, residuo)
!      and the `!$acc update self(temp(...))` before nusselt_promedio_y
!      (main.f90:1229) becomes `call ixb_temperatura()`; the messages, the
!      Nusselt record and the time update between them stay as they are;
!   4. `!$acc end data` (main.f90:1277) becomes `call ixb_estado()`, which
!      brings u, v, pres and temp back for the writers of main.f90:1278-1363;
!      after the package loop, `call ixb_cierre()` releases the handle.
!
! Every library status other than IXB_OK stops the program with the
! library's message (the reference has no status codes: its failures are
! runtime aborts).
!
module ixb_driver
  use iso_c_binding
  use ixb
  use malla, only : mi, nj, DBL, xu, yv, xp, yp
  use cond_frontera, only : tipo_cond_front
  use ec_momento, only : u, u_ant, v, v_ant, pres, Ri, Riy, gamma_momen
  use ec_momento, only : conv_u, conv_p, conv_paso, rel_pres, rel_vel
  use ec_momento, only : fuente_con_u, fuente_lin_u, fuente_con_v, fuente_lin_v
  use ec_momento, only : cond_front_ua, cond_front_ub, cond_front_uc, cond_front_ud
  use ec_momento, only : cond_front_va, cond_front_vb, cond_front_vc, cond_front_vd
  use ec_energia, only : temp, temp_ant, gamma_energ, conv_t, rel_ener
  use ec_energia, only : fuente_con_t, fuente_lin_t
  use ec_energia, only : cond_front_ta, cond_front_tb, cond_front_tc, cond_front_td
  implicit none
  private
  public :: ixb_arranque, ixb_paso, ixb_temperatura, ixb_estado, ixb_cierre

  type(c_ptr), save :: h = c_null_ptr

contains

  subroutine comprueba(st, que)
    integer(c_int), intent(in) :: st
    character(len=*), intent(in) :: que
    character(kind=c_char), pointer :: msg(:)
    integer :: n
    if (st == IXB_OK) return
    call c_f_pointer(ixb_strerror(st), msg, [64])
    n = 0
    do while (n < 64)
       if (msg(n + 1) == c_null_char) exit
       n = n + 1
    end do
    write(*,*) 'libixb: ', que, ': ', msg(1:n)
    stop 3
  end subroutine comprueba

  ! One side of a tipo_cond_front as the library's table: 'diri' and 'neum'
  ! segments keep their type and value, anything else ('desc') becomes
  ! IXB_BC_OTHER; indice_div(1..ndivis+1) is copied as it is.
  function lado(cf, side) result(s)
    type(tipo_cond_front), intent(in) :: cf
    integer, intent(in) :: side
    type(ixb_bc_side) :: s
    integer :: k
    s%side = side
    s%ndivis = cf%ndivis
    s%type = IXB_BC_OTHER
    s%value = 0.0_c_double
    s%index = 0
    do k = 1, cf%ndivis
       if (cf%tipo_condi(k) == 'diri') s%type(k) = IXB_BC_DIRI
       if (cf%tipo_condi(k) == 'neum') s%type(k) = IXB_BC_NEUM
       s%value(k) = cf%valor_cond(k)
    end do
    do k = 1, min(cf%ndivis + 1, size(cf%indice_div))
       s%index(k) = cf%indice_div(k)
    end do
  end function lado

  ! Handle, mesh, parameters (the non-dimensional values main.f90:215-244
  ! leaves in the module arrays, uniform in the reference), boundary tables,
  ! sources and the initial state: what the first `!$acc data` region copied.
  subroutine ixb_arranque(precision, dt, conv_resi, iter_ecuaci_max, iter_simple_max)
    integer(c_int), intent(in) :: precision
    real(kind=DBL), intent(in) :: dt, conv_resi
    integer, intent(in) :: iter_ecuaci_max, iter_simple_max
    type(ixb_params) :: prm
    type(ixb_bc_side) :: sides(4)
    call comprueba(ixb_create(int(mi, c_int), int(nj, c_int), precision, h), 'ixb_create')
    call comprueba(ixb_set_mesh(h, xu, yv, xp, yp), 'ixb_set_mesh')
    prm%gamma_momen = gamma_momen(1, 1)
    prm%gamma_energ = gamma_energ(1, 1)
    prm%Ri = Ri(1, 1)
    prm%Riy = Riy(1, 1)
    prm%dt = dt
    prm%rel_vel = rel_vel
    prm%rel_pres = rel_pres
    prm%rel_ener = rel_ener
    prm%conv_u = conv_u
    prm%conv_p = conv_p
    prm%conv_t = conv_t
    prm%conv_resi = conv_resi
    prm%conv_paso = conv_paso
    prm%p_update = 0.6_c_double
    prm%iter_ecuaci_max = iter_ecuaci_max
    prm%iter_simple_max = iter_simple_max
    prm%solver = IXB_SOLVER_HYBRID
    prm%reserved = 0
    call comprueba(ixb_set_params(h, prm), 'ixb_set_params')
    sides = [lado(cond_front_ua, 0), lado(cond_front_ub, 1), lado(cond_front_uc, 2), lado(cond_front_ud, 3)]
    call comprueba(ixb_set_bc(h, IXB_VAR_U, sides), 'ixb_set_bc(u)')
    sides = [lado(cond_front_va, 0), lado(cond_front_vb, 1), lado(cond_front_vc, 2), lado(cond_front_vd, 3)]
    call comprueba(ixb_set_bc(h, IXB_VAR_V, sides), 'ixb_set_bc(v)')
    sides = [lado(cond_front_ta, 0), lado(cond_front_tb, 1), lado(cond_front_tc, 2), lado(cond_front_td, 3)]
    call comprueba(ixb_set_bc(h, IXB_VAR_T, sides), 'ixb_set_bc(T)')
    call comprueba(ixb_set_sources(h, IXB_VAR_U, fuente_con_u, fuente_lin_u), 'ixb_set_sources(u)')
    call comprueba(ixb_set_sources(h, IXB_VAR_V, fuente_con_v, fuente_lin_v), 'ixb_set_sources(v)')
    call comprueba(ixb_set_sources(h, IXB_VAR_T, fuente_con_t, fuente_lin_t), 'ixb_set_sources(T)')
    call comprueba(ixb_upload_state(h, u, v, pres, temp, u_ant, v_ant, temp_ant), 'ixb_upload_state')
  end subroutine ixb_arranque

  ! One time step: the ALGORITMO_SIMPLE loop with the reference's exit tests
  ! (main.f90:395-1217), then u_ant, v_ant, temp_ant <- u, v, temp
  ! (main.f90:1251-1270), all on the device; maxbo and residuo of the last
  ! outer iteration come back for the messages of main.f90:1222-1224.
  subroutine ixb_paso(maxbo, residuo)
    real(kind=DBL), intent(out) :: maxbo, residuo
    type(ixb_report) :: rep
    call comprueba(ixb_step(h, rep), 'ixb_step')
    maxbo = rep%maxbo
    residuo = rep%residuo
  end subroutine ixb_paso

  ! temp for nusselt_promedio_y and temp_med (main.f90:1229-1241).  The
  ! interface of mod_ixb.f90 takes every array (its C function skips only
  ! NULL pointers, which an assumed-size dummy cannot pass), so the whole
  ! state comes back; the device copy stays the one that iterates.
  subroutine ixb_temperatura()
    call comprueba(ixb_download_state(h, u, v, pres, temp, u_ant, v_ant, temp_ant), 'ixb_download_state')
  end subroutine ixb_temperatura

  ! The copy-out of the `!$acc data` region (main.f90:1277): the state for
  ! the writers of main.f90:1278-1363.
  subroutine ixb_estado()
    call comprueba(ixb_download_state(h, u, v, pres, temp, u_ant, v_ant, temp_ant), 'ixb_download_state')
  end subroutine ixb_estado

  subroutine ixb_cierre()
    call comprueba(ixb_destroy(h), 'ixb_destroy')
    h = c_null_ptr
  end subroutine ixb_cierre

end module ixb_driver
