/*
 * obl_oracle.h -- FP64 CPU restatement of the OverlappingBLs hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this library; the product path
 * (libobl_b200.so) never links or calls it.
 *
 * Parity status: PARITY UNPINNED.  The reference (Fortran 90 + MPI + FFTW 3.3.x,
 * the SBL/code Fortran sources) ships no tests, golden vectors or fixtures, and it cannot be
 * compiled here (no Fortran compiler, no MPI, no FFTW).  This restatement is
 * pinned instead against (1) analytic known-answer cases, (2) a long-double
 * naive DFT, (3) an independent numpy restatement (tests/golden/gen_golden.py)
 * and (4) the reference's own invariants (divergence-free projection, the
 * pipelined multi-rank Thomas solve equal to the sequential one).
 *
 * Array conventions follow the reference exactly (Fortran column-major):
 *   physical field  f(ldx, nyt, 0:nz)    -> f[x + ldx*(y + nyt*z)], x,y 0-based
 *   spectral plane  c(lhx, nyt)          -> c[kx + lhx*ky]  (complex double)
 *   padded plane    b(nxt2, nyt2)        -> b[x + nxt2*y]
 *   dpdx/dpdy/dpdz  (ldx, nyt, 1:nz)     -> level jz stored at slot jz-1
 * with ldx = 2*(nxt/2+1), nz = (nzt-1)/npz + 1 (SBL/code/102_initial.f90:119-141).
 * The "global" arrays used here are the single-rank (npz = 1) arrays:
 * nz = nzt, levels 0..nzt.
 */
#ifndef OBL_ORACLE_H
#define OBL_ORACLE_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_grid {
    /* inputs (dimensional, as in the namelist &domain_param / &time_param) */
    int nxt, nyt, nzt;
    double lx_tot, ly_tot, lz_tot, z_i, dt, u_scale;
    int ubc_stress_free;   /* project(): ubc_mom == 'stress free' (110_project.f90:51) */
    /* derived by orc_grid_init (102_initial.f90:119-141, 186-199) */
    int nz, lhx, lhy, ldx, ldy, nxt2, nyt2, lhx2, lhy2, ldx2, ldy2;
    double lx, ly, lz, dz, dt_nd;   /* non-dimensional (divided by z_i; dt*u_scale/z_i) */
} orc_grid;

/* ---- FFT (own mixed-radix Cooley-Tukey; unnormalised, FFTW sign convention) ---- */
/* sign = -1 forward (FFTW_FORWARD), +1 backward.  Any n >= 1. */
void orc_fft_c2c(int n, const double complex *in, double complex *out, int sign);
/* r2c: n reals -> n/2+1 complex.  c2r: n/2+1 complex -> n reals; ignores the
   imaginary parts of the DC and (even n) Nyquist bins, as FFTW's c2r does. */
void orc_fft_r2c(int n, const double *in, double complex *out);
void orc_fft_c2r(int n, const double complex *in, double *out);
/* naive O(n^2) DFT in long double, for validating the FFT */
void orc_dft_naive(int n, const double complex *in, double complex *out, int sign);

/* ---- setup ---- */
int  orc_grid_init(orc_grid *g);    /* returns 0 on success, nonzero on a bad size */
/* wavenumber tables of init_wavenumber (002_fft.f90:121-189), npy = 1:
   kx[lhx], ky[lhy], kx2d/ky2d/k2[lhx*nyt], notnyq[lhx*nyt] (1 = not Nyquist) */
void orc_wavenumbers(const orc_grid *g, double *kx, double *ky, double *kx2d,
                     double *ky2d, double *k2, int *notnyq);

/* ---- spectral derivatives (004_derivatives.f90) ----
   nlev planes starting at level 0 of f(ldx, nyt, 0:nlev-1). Only x < nxt is written. */
void orc_ddx(const orc_grid *g, double *dfdx, const double *fun, int nlev);
void orc_ddy(const orc_grid *g, double *dfdy, const double *fun, int nlev);
/* ddz_uv / ddz_w on the single-rank arrays (levels 0..nz), with the
   coordz == 0 == npz-1 branches of 004_derivatives.f90:85-116,155-183 */
void orc_ddz_uv(const orc_grid *g, double *dfdz, const double *fun);
void orc_ddz_w(const orc_grid *g, double *dfdz, const double *fun);

/* 107_divstress.f90:4-44 / 48-104, single rank: divt (ldx,nyt,0:nz) fully written */
void orc_divstress_uv(const orc_grid *g, double *divt, const double *tx, const double *ty, const double *tz);
void orc_divstress_w(const orc_grid *g, double *divt, const double *tx, const double *ty, const double *tz);

/* ---- 2D transforms of one plane (203_fftn_mpi.f90:4-67) ---- */
void orc_fftn(const orc_grid *g, const double *in, double complex *out);
void orc_ifftn(const orc_grid *g, const double complex *in, double *out);

/* ---- 3/2-rule dealiasing of one plane (108_01_padd.f90:73-197) ---- */
void orc_zero_padding(const orc_grid *g, const double *var, double *var_big);
void orc_zero_unpadding(const orc_grid *g, const double *var_big, double *var);

/* ---- Nyquist filter (006_test_filter.f90:82-105), nlev planes in place ---- */
void orc_filter_data(const orc_grid *g, double *f, int nlev);

/* ---- pressure solve (109_press_stag_array.f90) emulating npz z-ranks ----
   npz = 1  : single-rank semantics (p_hat(nz-1) forced to 0: Dirichlet top).
   npz >= 2 : pipelined multi-rank semantics (Neumann top row, divtz top plane used).
   Inputs are the global single-rank arrays u,v,w(ldx,nyt,0:nzt); divtz_bot is the
   plane divtz(:,:,1) of the bottom rank, divtz_top the plane divtz(:,:,nz) of the top
   rank (global level nzt).  Outputs: p(ldx,nyt,0:nzt) levels 0..nzt-1 written,
   dpdx/dpdy(ldx,nyt,1:nzt) levels 1..nzt-1 written.  Returns nonzero if
   (nzt-1) % npz != 0. */
int orc_press_stag_array(const orc_grid *g, int npz, const double *u,
                         const double *v, const double *w,
                         const double *divtz_bot, const double *divtz_top,
                         double *p, double *dpdx, double *dpdy);

/* flosol glue (103_flosol.f90:169-175): dpdz(jz) = (p(jz)-p(jz-1))/dz, jz=1..nz-1 */
void orc_dpdz(const orc_grid *g, const double *p, double *dpdz);

/* project() (110_project.f90:4-62) on the global arrays (bottom and top rank at once) */
void orc_project(const orc_grid *g, double *u, double *v, double *w,
                 const double *dpdx, const double *dpdy, const double *dpdz);

/* Headline step: ddx/ddy and zero_padding of u,v,w,theta on levels 0..nz, then
   press_stag_array(u,v,w) (divtz = 0), dpdz and project().  d[8] = dudx,dudy,dvdx,
   dvdy,dwdx,dwdy,dtdx,dtdy (ldx,nyt,0:nz); big[4] = u,v,w,theta padded
   (nxt2,nyt2,0:nz); p (ldx,nyt,0:nz); dp[3] = dpdx,dpdy,dpdz (ldx,nyt,1:nz);
   u,v,w updated in place. */
int orc_step(const orc_grid *g, int npz, double *u, double *v, double *w,
             const double *theta, double *const d[8], double *const big[4],
             double *p, double *const dp[3]);

/* ---- rollout problem of the adjoint (obl_oracle_adj.c) ---- */
/* Rotational convective term of convec + cross_product (108_convec.f90:11-202), single
   rank (coordz == 0 == npz-1), Stokes drift off (ust = vst = 0).  dudz, dvdz at level 1
   (set by wallstress_bottom in the reference) are taken equal to level 2; at level nz they
   are 0, the stress-free top of wallstress_top (104_wallstress.f90:249-253).
   cx, cy, cz (ldx,nyt,0:nz) are written on levels 1..nz-1, x < nxt. */
void orc_convec(const orc_grid *g, const double *u, const double *v, const double *w,
                double *cx, double *cy, double *cz);

/* P: press_stag_array with divtz = 0 in the Neumann-top (npz >= 2) mode, flosol's dpdz
   and project(), in place.  Needs (nzt-1) even. */
int orc_projection(const orc_grid *g, double *u, double *v, double *w);

/* One rollout step u1 = P(u - dt*tadv1*convec(u)), u,v,w in place. */
int orc_rollout_step(const orc_grid *g, double *u, double *v, double *w);

/* J = sum over x < nxt, all y and the levels 1..nz-1 whose uvp height (jz-0.5)*dz*z_i
   lies in (z_lo, z_hi) of ke = 0.5*(u^2 + v^2 + (0.5*(w(jz)+w(jz+1)))^2)
   (energy, 103_flosol.f90).  If lu is not NULL, lu/lv/lw receive dJ/d(u,v,w). */
double orc_ke_band(const orc_grid *g, const double *u, const double *v, const double *w,
                   double z_lo, double z_hi, double *lu, double *lv, double *lw);

/* Transposes, written as explicit transposed operators:
   orc_projection_vjp: lambda <- P^T lambda, in place;
   orc_convec_vjp: l(u,v,w) += (d convec / d(u,v,w))^T l(cx,cy,cz) at the state u,v,w;
   orc_rollout_step_vjp: lambda <- (d step / d state)^T lambda at the state u,v,w. */
int orc_projection_vjp(const orc_grid *g, double *lu, double *lv, double *lw);
void orc_convec_vjp(const orc_grid *g, const double *u, const double *v, const double *w,
                    const double *lcx, const double *lcy, const double *lcz,
                    double *lu, double *lv, double *lw);
int orc_rollout_step_vjp(const orc_grid *g, const double *u, const double *v, const double *w,
                         double *lu, double *lv, double *lw);

/* nsteps rollout steps from (u0,v0,w0) with a checkpoint of every step's state, J of
   the final state, and (when gu is not NULL) dJ/d(u0,v0,w0) by the reverse sweep.
   Returns nonzero on a bad size. */
int orc_rollout_grad(const orc_grid *g, int nsteps, const double *u0, const double *v0,
                     const double *w0, double z_lo, double z_hi, double *J,
                     double *gu, double *gv, double *gw);

/* threads used by the OpenMP loops (0 = leave the OpenMP default) */
void orc_set_threads(int n);
int  orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
