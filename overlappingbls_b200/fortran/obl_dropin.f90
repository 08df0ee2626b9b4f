!-----------------------------------------------------------------------
! obl_dropin.f90 -- the reference's own pressure-solver and projection routines, with
! their exact Fortran interfaces, running on the GPU through libobl_b200.so.
!
! Compiled INSIDE the reference tree (SBL/code), in place of its CPU versions:
!   * 109_press_stag_array.f90 is left out of the build.  This file provides its two
!     externally called routines:
!         subroutine init_coef_press()                 (called at 102_initial.f90:53)
!         subroutine press_stag_array(func, dfdx, dfdy) (called at 103_flosol.f90:168)
!     tdmaMcoef_pipelined and tdmaSolver_pipelined are only called from inside that file.
!   * In 110_project.f90 the subroutine project (lines 4-62) is deleted; readin_inflow
!     and update_fringe stay.  This file provides
!         subroutine project()                          (called at 103_flosol.f90:188)
! The call sites compile unchanged.  Link with obl_gpu.f90 and -lobl_b200.
!
! Interfaces and module inputs are those of 109_press_stag_array.f90:107-142 (func, dfdx,
! dfdy out; u, v, w, divtz from sim_param) and 110_project.f90:4-17 (no arguments; u, v, w
! updated from sim_param's dpdx, dpdy, dpdz).  Arrays are the reference's rprec
! (real(8)) module arrays, passed to the C ABI in place.
!
! One GPU holds the whole domain, so the run must have npy = npz = 1.  The GPU context is
! created by init_coef_press, which the reference calls after init_nondimensional
! (102_initial.f90:22), so lx_tot, ly_tot, lz_tot and dt are already non-dimensional and
! are passed with z_i = u_scale = 1.  Environment:
!   OBL_PRECISION = f64 (default) | mixed   -- FP64 everywhere, or FP32 with FP64 islands
!   OBL_TOP_BC    = single (default) | neumann
!       single:  the reference's npz = 1 result (top row never built, p_hat(nz-1) = 0);
!       neumann: the reference's npz >= 2 result (Neumann top row, divtz(:,:,nz) used).
!   OBL_DEVICE    = CUDA device ordinal (default 0)
! The inflow/fringe branch of project (110_project.f90:40-46) is not on the GPU path:
! project stops with a message when inflow is set.
!-----------------------------------------------------------------------
subroutine init_coef_press()
use types, only: rprec
use param, only: nxt, nyt, nzt, nynpy, nz, npy, npz, lx_tot, ly_tot, lz_tot, dt, ubc_mom
use obl_gpu, only: obl_gpu_init, OBL_PREC_F64, OBL_PREC_MIXED, OBL_TOP_SINGLE_RANK, OBL_TOP_NEUMANN
implicit none
character(len=16) :: env
integer :: prec, top, dev, ln, st
if (npy /= 1 .or. npz /= 1 .or. nynpy /= nyt .or. nz /= nzt) then
    write(*, *) 'obl_dropin: the GPU path holds the whole domain; run with npy = npz = 1'
    stop 1
end if
prec = OBL_PREC_F64
call get_environment_variable('OBL_PRECISION', env, ln, st)
if (st == 0 .and. env(1:ln) == 'mixed') prec = OBL_PREC_MIXED
top = OBL_TOP_SINGLE_RANK
call get_environment_variable('OBL_TOP_BC', env, ln, st)
if (st == 0 .and. env(1:ln) == 'neumann') top = OBL_TOP_NEUMANN
dev = 0
call get_environment_variable('OBL_DEVICE', env, ln, st)
if (st == 0 .and. ln > 0) read(env(1:ln), *) dev
call obl_gpu_init(nxt, nyt, nzt, real(lx_tot, rprec), real(ly_tot, rprec), real(lz_tot, rprec), &
                  1.0_rprec, real(dt, rprec), 1.0_rprec, prec, top, ubc_mom == 'stress free', dev)
end subroutine init_coef_press

subroutine press_stag_array(func, dfdx, dfdy)
use types, only: rprec
use param, only: ldx, nynpy, nz, nxt, theta_flag, jt, theta_init_time, lbc, g, z_i, u_scale
use sim_param, only: u, v, w, divtz
use bottombc, only: T_s
use obl_gpu, only: press_stag_array_planes_gpu
implicit none
real(kind=rprec), dimension(ldx, nynpy, 0:nz), intent(out) :: func
real(kind=rprec), dimension(ldx, nynpy, nz), intent(out) :: dfdx, dfdy
real(kind=rprec), dimension(ldx, nynpy) :: rbot
real(kind=rprec) :: T_s_mn
! bottom boundary plane; the surface-temperature term of 109_press_stag_array.f90:187-192
! is folded in here (the library applies the 1/(nxt*nyt) scaling and the transform)
rbot(:, :) = divtz(:, :, 1)
if (theta_flag .and. (jt .gt. theta_init_time) .and. (lbc .eq. 0)) then
    call calc_hor_avg3(T_s, T_s_mn)
    rbot(1:nxt, :) = divtz(1:nxt, :, 1) - g*(z_i/(u_scale**2))*(T_s(1:nxt, :) - T_s_mn)
end if
call press_stag_array_planes_gpu(func, dfdx, dfdy, u, v, w, rbot, divtz(:, :, nz))
end subroutine press_stag_array

subroutine project()
use param, only: inflow
use sim_param, only: u, v, w, dpdx, dpdy, dpdz
use obl_gpu, only: project_gpu
implicit none
if (inflow) then
    write(*, *) 'obl_dropin: the inflow/fringe branch of project is not on the GPU path'
    stop 1
end if
! interior update and the top/bottom conditions of 110_project.f90:17-61
call project_gpu(u, v, w, dpdx, dpdy, dpdz)
end subroutine project
