!-----------------------------------------------------------------------
! obl_gpu -- ISO_C_BINDING interface to libobl_b200.so (include/obl.h).
!
! Drop-in GPU versions of the reference's hot-path routines with the reference's
! own dummy-argument shapes, so that the time loop only swaps names, e.g.
!     use obl_gpu, only: ddx => ddx_gpu, ddy => ddy_gpu, &
!                        press_stag_array => press_stag_array_gpu
! Shapes follow SBL/code/004_derivatives.f90:25-26, 109_press_stag_array.f90:141-142,
! 108_01_padd.f90:83-84 with npy = npz = 1 on the GPU (nynpy = nyt, nz = nzt).
! The context is created once, in place of init_fft_plan + init_coef_press
! (102_initial.f90:34,53), by obl_gpu_init.
!
! Build: gfortran -c obl_gpu.f90 ; link with -L<dir> -lobl_b200 -lcudart (or the
! static cudart already inside libobl_b200.so).
!-----------------------------------------------------------------------
module obl_gpu
use iso_c_binding
implicit none
private
public :: obl_gpu_init, obl_gpu_finalize, ddx_gpu, ddy_gpu, ddz_uv_gpu, ddz_w_gpu, &
          divstress_uv_gpu, divstress_w_gpu, &
          zero_padding_gpu, zero_unpadding_gpu, filter_data_gpu, fftn_gpu, ifftn_gpu, &
          press_stag_array_gpu, press_stag_array_planes_gpu, dpdz_gpu, project_gpu, obl_gpu_check

integer(c_int), parameter, public :: OBL_PREC_F64 = 0, OBL_PREC_MIXED = 1, OBL_PREC_F32 = 2
integer(c_int), parameter, public :: OBL_TOP_SINGLE_RANK = 0, OBL_TOP_NEUMANN = 1

type, bind(C) :: obl_grid
    integer(c_int) :: nxt, nyt, nzt
    real(c_double) :: lx_tot, ly_tot, lz_tot, z_i, dt, u_scale
end type
type, bind(C) :: obl_options
    integer(c_int) :: precision, top_bc, ubc_stress_free
    real(c_double) :: fp64_k2_max
    integer(c_int) :: device
end type

type(c_ptr), save :: ctx = c_null_ptr
integer, save :: g_ldx = 0, g_nyt = 0, g_nz = 0

interface
    integer(c_int) function obl_ctx_create(grid, opt, out) bind(C, name="obl_ctx_create")
        import :: c_int, c_ptr, obl_grid, obl_options
        type(obl_grid), intent(in) :: grid
        type(obl_options), intent(in) :: opt
        type(c_ptr), intent(out) :: out
    end function
    integer(c_int) function obl_ctx_destroy(c) bind(C, name="obl_ctx_destroy")
        import :: c_int, c_ptr
        type(c_ptr), value :: c
    end function
    integer(c_int) function obl_last_error(c, buf, n) bind(C, name="obl_last_error")
        import :: c_int, c_ptr, c_char, c_size_t
        type(c_ptr), value :: c
        character(kind=c_char), dimension(*) :: buf
        integer(c_size_t), value :: n
    end function
    integer(c_int) function obl_ddx(c, dfdx, fun, nlev) bind(C, name="obl_ddx")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*) :: dfdx
        real(c_double), dimension(*), intent(in) :: fun
        integer(c_int), value :: nlev
    end function
    integer(c_int) function obl_ddy(c, dfdy, fun, nlev) bind(C, name="obl_ddy")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*) :: dfdy
        real(c_double), dimension(*), intent(in) :: fun
        integer(c_int), value :: nlev
    end function
    integer(c_int) function obl_ddz_uv(c, dfdz, fun) bind(C, name="obl_ddz_uv")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*) :: dfdz
        real(c_double), dimension(*), intent(in) :: fun
    end function
    integer(c_int) function obl_divstress_uv(c, divt, tx, ty, tz) bind(C, name="obl_divstress_uv")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*) :: divt
        real(c_double), dimension(*), intent(in) :: tx, ty, tz
    end function
    integer(c_int) function obl_divstress_w(c, divt, tx, ty, tz) bind(C, name="obl_divstress_w")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*) :: divt
        real(c_double), dimension(*), intent(in) :: tx, ty, tz
    end function
    integer(c_int) function obl_ddz_w(c, dfdz, fun) bind(C, name="obl_ddz_w")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*) :: dfdz
        real(c_double), dimension(*), intent(in) :: fun
    end function
    integer(c_int) function obl_zero_padding(c, var, big, nlev) bind(C, name="obl_zero_padding")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*), intent(in) :: var
        real(c_double), dimension(*) :: big
        integer(c_int), value :: nlev
    end function
    integer(c_int) function obl_zero_unpadding(c, big, var, nlev) bind(C, name="obl_zero_unpadding")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*), intent(in) :: big
        real(c_double), dimension(*) :: var
        integer(c_int), value :: nlev
    end function
    integer(c_int) function obl_filter_data(c, f, nlev) bind(C, name="obl_filter_data")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*) :: f
        integer(c_int), value :: nlev
    end function
    integer(c_int) function obl_fftn(c, fin, fout, nlev) bind(C, name="obl_fftn")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*), intent(in) :: fin
        complex(c_double), dimension(*) :: fout
        integer(c_int), value :: nlev
    end function
    integer(c_int) function obl_ifftn(c, fin, fout, nlev) bind(C, name="obl_ifftn")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        complex(c_double), dimension(*), intent(in) :: fin
        real(c_double), dimension(*) :: fout
        integer(c_int), value :: nlev
    end function
    integer(c_int) function obl_press_stag_array(c, u, v, w, dbot, dtop, p, dpdx, dpdy) &
            bind(C, name="obl_press_stag_array")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*), intent(in) :: u, v, w, dbot, dtop
        real(c_double), dimension(*) :: p, dpdx, dpdy
    end function
    integer(c_int) function obl_dpdz(c, p, dpdz) bind(C, name="obl_dpdz")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*), intent(in) :: p
        real(c_double), dimension(*) :: dpdz
    end function
    integer(c_int) function obl_project(c, u, v, w, dpdx, dpdy, dpdz) bind(C, name="obl_project")
        import :: c_int, c_ptr, c_double
        type(c_ptr), value :: c
        real(c_double), dimension(*) :: u, v, w
        real(c_double), dimension(*), intent(in) :: dpdx, dpdy, dpdz
    end function
end interface

contains

!--- replaces init_fft_plan + init_coef_press (call after init_nondimensional with the
!    DIMENSIONAL namelist values: the library non-dimensionalises them itself)
subroutine obl_gpu_init(nxt, nyt, nzt, lx_tot, ly_tot, lz_tot, z_i, dt, u_scale, &
                        precision, top_bc, stress_free, device)
    integer, intent(in) :: nxt, nyt, nzt, precision, top_bc, device
    real(c_double), intent(in) :: lx_tot, ly_tot, lz_tot, z_i, dt, u_scale
    logical, intent(in) :: stress_free
    type(obl_grid) :: g
    type(obl_options) :: o
    g = obl_grid(nxt, nyt, nzt, lx_tot, ly_tot, lz_tot, z_i, dt, u_scale)
    o%precision = precision
    o%top_bc = top_bc
    o%ubc_stress_free = merge(1, 0, stress_free)
    o%fp64_k2_max = -1.0_c_double
    o%device = device
    call obl_gpu_check(obl_ctx_create(g, o, ctx), 'obl_ctx_create')
    g_ldx = 2*(nxt/2 + 1)
    g_nyt = nyt
    g_nz = nzt
end subroutine

subroutine obl_gpu_finalize()
    integer(c_int) :: rc
    rc = obl_ctx_destroy(ctx)
    ctx = c_null_ptr
end subroutine

!--- fatal on error, as the reference stops on errors (102_initial.f90:164-168)
subroutine obl_gpu_check(rc, what)
    integer(c_int), intent(in) :: rc
    character(*), intent(in) :: what
    character(kind=c_char) :: buf(512)
    integer(c_int) :: r2
    integer :: i
    if (rc == 0) return
    buf = c_null_char
    r2 = obl_last_error(ctx, buf, int(512, c_size_t))
    write(*, '(a,a,i3,1x,512a)') what, ': status', rc, (buf(i), i = 1, 512)
    stop 1
end subroutine

subroutine ddx_gpu(dfdx, fun)                  ! 004_derivatives.f90:18-41
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(in) :: fun
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(inout) :: dfdx
    call obl_gpu_check(obl_ddx(ctx, dfdx, fun, int(g_nz + 1, c_int)), 'ddx')
end subroutine

subroutine ddy_gpu(dfdy, fun)                  ! 004_derivatives.f90:45-81
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(in) :: fun
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(inout) :: dfdy
    call obl_gpu_check(obl_ddy(ctx, dfdy, fun, int(g_nz + 1, c_int)), 'ddy')
end subroutine

subroutine ddz_uv_gpu(dfdz, fun)               ! 004_derivatives.f90:85-116
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(in) :: fun
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(inout) :: dfdz
    call obl_gpu_check(obl_ddz_uv(ctx, dfdz, fun), 'ddz_uv')
end subroutine

subroutine divstress_uv_gpu(divt, tx, ty, tz)   ! 107_divstress.f90:4-44
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(in) :: tx, ty, tz
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(out) :: divt
    call obl_gpu_check(obl_divstress_uv(ctx, divt, tx, ty, tz), 'divstress_uv')
end subroutine

subroutine divstress_w_gpu(divt, tx, ty, tz)    ! 107_divstress.f90:48-104
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(in) :: tx, ty, tz
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(out) :: divt
    call obl_gpu_check(obl_divstress_w(ctx, divt, tx, ty, tz), 'divstress_w')
end subroutine

subroutine ddz_w_gpu(dfdz, fun)                ! 004_derivatives.f90:155-183
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(in) :: fun
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(out) :: dfdz
    call obl_gpu_check(obl_ddz_w(ctx, dfdz, fun), 'ddz_w')
end subroutine

subroutine zero_padding_gpu(var, var_big)      ! 108_01_padd.f90:73-132 (one plane)
    real(c_double), dimension(g_ldx, g_nyt), intent(in) :: var
    real(c_double), dimension(3*(g_ldx - 2)/2, 3*g_nyt/2), intent(out) :: var_big
    call obl_gpu_check(obl_zero_padding(ctx, var, var_big, 1_c_int), 'zero_padding')
end subroutine

subroutine zero_unpadding_gpu(var_big, var)    ! 108_01_padd.f90:136-197 (one plane)
    real(c_double), dimension(3*(g_ldx - 2)/2, 3*g_nyt/2), intent(in) :: var_big
    real(c_double), dimension(g_ldx, g_nyt), intent(out) :: var
    call obl_gpu_check(obl_zero_unpadding(ctx, var_big, var, 1_c_int), 'zero_unpadding')
end subroutine

subroutine filter_data_gpu(f_c)                ! 006_test_filter.f90:82-105
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(inout) :: f_c
    call obl_gpu_check(obl_filter_data(ctx, f_c, int(g_nz + 1, c_int)), 'filter_data')
end subroutine

subroutine fftn_gpu(fin, fout)                 ! 203_fftn_mpi.f90:4-35 (one plane)
    real(c_double), dimension(g_ldx, g_nyt), intent(in) :: fin
    complex(c_double), dimension(g_ldx/2, g_nyt), intent(out) :: fout
    call obl_gpu_check(obl_fftn(ctx, fin, fout, 1_c_int), 'fftn')
end subroutine

subroutine ifftn_gpu(fin, fout)                ! 203_fftn_mpi.f90:39-67 (one plane)
    complex(c_double), dimension(g_ldx/2, g_nyt), intent(in) :: fin
    real(c_double), dimension(g_ldx, g_nyt), intent(out) :: fout
    call obl_gpu_check(obl_ifftn(ctx, fin, fout, 1_c_int), 'ifftn')
end subroutine

! press_stag_array reads u, v, w, divtz from module sim_param in the reference
! (109_press_stag_array.f90:135); here they are explicit arguments after the
! reference's three outputs.
subroutine press_stag_array_gpu(func, dfdx, dfdy, u, v, w, divtz)
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(out) :: func
    real(c_double), dimension(g_ldx, g_nyt, g_nz), intent(out) :: dfdx, dfdy
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(in) :: u, v, w, divtz
    call obl_gpu_check(obl_press_stag_array(ctx, u, v, w, divtz(:, :, 1), divtz(:, :, g_nz), &
                                            func, dfdx, dfdy), 'press_stag_array')
end subroutine

! The same with the two divtz boundary planes given separately, for a caller that has
! already folded the surface-temperature term of 109_press_stag_array.f90:187-192 into
! the bottom plane (obl_dropin.f90).
subroutine press_stag_array_planes_gpu(func, dfdx, dfdy, u, v, w, divtz_bot, divtz_top)
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(out) :: func
    real(c_double), dimension(g_ldx, g_nyt, g_nz), intent(out) :: dfdx, dfdy
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(in) :: u, v, w
    real(c_double), dimension(g_ldx, g_nyt), intent(in) :: divtz_bot, divtz_top
    call obl_gpu_check(obl_press_stag_array(ctx, u, v, w, divtz_bot, divtz_top, func, dfdx, dfdy), &
                       'press_stag_array')
end subroutine

subroutine dpdz_gpu(dpdz, p)                   ! 103_flosol.f90:174-175
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(in) :: p
    real(c_double), dimension(g_ldx, g_nyt, g_nz), intent(inout) :: dpdz
    call obl_gpu_check(obl_dpdz(ctx, p, dpdz), 'dpdz')
end subroutine

subroutine project_gpu(u, v, w, dpdx, dpdy, dpdz)   ! 110_project.f90:4-62
    real(c_double), dimension(g_ldx, g_nyt, 0:g_nz), intent(inout) :: u, v, w
    real(c_double), dimension(g_ldx, g_nyt, g_nz), intent(in) :: dpdx, dpdy, dpdz
    call obl_gpu_check(obl_project(ctx, u, v, w, dpdx, dpdy, dpdz), 'project')
end subroutine

end module obl_gpu
