/*
 * obl_oracle_adj.c -- FP64 CPU restatement of the rollout problem of the adjoint.
 *
 * TEST INFRASTRUCTURE ONLY (see obl_oracle.h): the checker of the GPU rollout, step
 * transpose and gradient.  Nothing in the product library links or calls this file.
 *
 * The forward pieces follow the reference: the rotational convective term of convec +
 * cross_product (SBL/code/108_convec.f90:11-202, single rank, no Stokes drift), the
 * pressure projection (109_press_stag_array.f90, npz >= 2 top mode; 103_flosol.f90:174;
 * 110_project.f90) and the kinetic energy of energy (103_flosol.f90, temp_w = w at the
 * uvp node).  The rollout step u1 = P(u - dt*tadv1*convec(u)) is the explicit-Euler
 * form of the Adams-Bashforth update of 103_flosol.f90:319-389 with RHS = -convec
 * (:115) and the pressure scaling of press_stag_array (rH = u/(tadv1*dt), :166-168).
 *
 * The transposes are written here as explicit transposed operators, independent of
 * the GPU construction: the spectral symbols are conjugated (ddx^T = -ddx; for the 3/2
 * rule pad^T = (3/2)^2 unpad and unpad^T = pad/(3/2)^2), the tridiagonal system is
 * solved with the transposed bands, and every level stencil is transposed term by term.
 */
#include "obl_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

static const double TADV1 = 1.5; /* 001_param.f90:152 */

typedef struct {
    int nx, ny, ldx, nz, nx2, ny2, lhx;
    size_t pl, plb, F, FB, S;
} dims_t;

static dims_t dims(const orc_grid *g)
{
    dims_t d;
    d.nx = g->nxt;
    d.ny = g->nyt;
    d.ldx = g->ldx;
    d.nz = g->nz;
    d.nx2 = g->nxt2;
    d.ny2 = g->nyt2;
    d.lhx = g->lhx;
    d.pl = (size_t)g->ldx * g->nyt;
    d.plb = (size_t)g->nxt2 * g->nyt2;
    d.F = d.pl * (size_t)(g->nz + 1);
    d.FB = d.plb * (size_t)(g->nz + 1);
    d.S = (size_t)g->lhx * g->nyt;
    return d;
}

static double *zalloc(size_t n) { return (double *)calloc(n, sizeof(double)); }

/* x index of a flat plane offset q of a (ldx, nyt) plane */
#define XOF(q, ldx) ((int)((q) % (size_t)(ldx)))

static void pad_levels(const orc_grid *g, const double *f, double *big, int k0, int k1)
{
    dims_t d = dims(g);
#pragma omp parallel for schedule(dynamic)
    for (int k = k0; k <= k1; k++) orc_zero_padding(g, f + d.pl * k, big + d.plb * k);
}

static void unpad_levels(const orc_grid *g, const double *big, double *f, int k0, int k1)
{
    dims_t d = dims(g);
#pragma omp parallel for schedule(dynamic)
    for (int k = k0; k <= k1; k++) orc_zero_unpadding(g, big + d.plb * k, f + d.pl * k);
}

/* the six padded fields convec builds (108_convec.f90:38-76) */
typedef struct {
    double *U, *V, *W, *O1, *O2, *O3;
} bigs_t;

static void bigs_free(bigs_t *b)
{
    free(b->U);
    free(b->V);
    free(b->W);
    free(b->O1);
    free(b->O2);
    free(b->O3);
}

static void convec_fields(const orc_grid *g, const double *u, const double *v, const double *w,
                          bigs_t *b)
{
    dims_t d = dims(g);
    const int nz = d.nz, nlev = nz + 1;
    const double idz = 1.0 / g->dz;
    double *dudy = zalloc(d.F), *dvdx = zalloc(d.F), *dwdx = zalloc(d.F), *dwdy = zalloc(d.F);
    double *dudz = zalloc(d.F), *dvdz = zalloc(d.F);
    double *o1 = zalloc(d.F), *o2 = zalloc(d.F), *o3 = zalloc(d.F);
    /* 103_flosol.f90:30-37 */
    orc_ddy(g, dudy, u, nlev);
    orc_ddx(g, dvdx, v, nlev);
    orc_ddx(g, dwdx, w, nlev);
    orc_ddy(g, dwdy, w, nlev);
    for (size_t q = 0; q < d.pl; q++) {
        if (XOF(q, d.ldx) >= d.nx) continue;
        for (int k = 2; k <= nz - 1; k++) { /* ddz_uv, 004_derivatives.f90:108 */
            dudz[q + d.pl * k] = (u[q + d.pl * k] - u[q + d.pl * (k - 1)]) * idz;
            dvdz[q + d.pl * k] = (v[q + d.pl * k] - v[q + d.pl * (k - 1)]) * idz;
        }
        dudz[q + d.pl] = dudz[q + d.pl * 2]; /* wall level: taken equal to level 2 */
        dvdz[q + d.pl] = dvdz[q + d.pl * 2];
        dudz[q + d.pl * nz] = 0.0;           /* stress-free top, 104_wallstress.f90:249-253 */
        dvdz[q + d.pl * nz] = 0.0;
        for (int k = 1; k <= nz; k++) { /* 108_convec.f90:43-67 */
            size_t o = q + d.pl * k;
            if (k == 1) {
                o1[o] = 0.5 * (dwdy[o] + dwdy[o + d.pl]) - dvdz[o];
                o2[o] = dudz[o] - 0.5 * (dwdx[o] + dwdx[o + d.pl]);
            } else if (k == nz) {
                o1[o] = 0.5 * (dwdy[o] + dwdy[o - d.pl]) - dvdz[o];
                o2[o] = dudz[o] - 0.5 * (dwdx[o] + dwdx[o - d.pl]);
            } else {
                o1[o] = dwdy[o] - dvdz[o];
                o2[o] = dudz[o] - dwdx[o];
            }
            o3[o] = dvdx[o] - dudy[o];
        }
    }
    b->U = zalloc(d.FB);
    b->V = zalloc(d.FB);
    b->W = zalloc(d.FB);
    b->O1 = zalloc(d.FB);
    b->O2 = zalloc(d.FB);
    b->O3 = zalloc(d.FB);
    pad_levels(g, u, b->U, 0, nz); /* :38-42 */
    pad_levels(g, v, b->V, 0, nz);
    pad_levels(g, w, b->W, 0, nz);
    pad_levels(g, o1, b->O1, 1, nz); /* :70-74 */
    pad_levels(g, o2, b->O2, 1, nz);
    pad_levels(g, o3, b->O3, 1, nz);
    free(dudy);
    free(dvdx);
    free(dwdx);
    free(dwdy);
    free(dudz);
    free(dvdz);
    free(o1);
    free(o2);
    free(o3);
}

void orc_convec(const orc_grid *g, const double *u, const double *v, const double *w,
                double *cx, double *cy, double *cz)
{
    dims_t d = dims(g);
    const int nz = d.nz;
    bigs_t b;
    convec_fields(g, u, v, w, &b);
    double *X = zalloc(d.FB), *Y = zalloc(d.FB), *Z = zalloc(d.FB);
    const size_t P = d.plb;
    /* cross_product, coordz == 0 == npz-1, ust = vst = 0 (108_convec.f90:108-202) */
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < P; q++) {
        X[q + P] = b.V[q + P] * (-b.O3[q + P]) + 0.5 * b.W[q + 2 * P] * b.O2[q + 2 * P]; /* :123-124 */
        Y[q + P] = b.U[q + P] * b.O3[q + P] + 0.5 * b.W[q + 2 * P] * (-b.O1[q + 2 * P]); /* :153-154 */
        Z[q + P] = 0.0;                                                                 /* :180 */
        for (int k = 2; k <= nz - 1; k++) {
            size_t o = q + P * k;
            X[o] = b.V[o] * (-b.O3[o]) + 0.5 * (b.W[o + P] * b.O2[o + P] + b.W[o] * b.O2[o]); /* :145-149 */
            Y[o] = b.U[o] * b.O3[o] + 0.5 * (b.W[o + P] * (-b.O1[o + P]) + b.W[o] * (-b.O1[o])); /* :175-179 */
            Z[o] = 0.5 * ((b.U[o] + b.U[o - P]) * (-b.O2[o]) + (b.V[o] + b.V[o - P]) * b.O1[o]); /* :194-199 */
        }
    }
    unpad_levels(g, X, cx, 1, nz - 1); /* :85-89 */
    unpad_levels(g, Y, cy, 1, nz - 1);
    unpad_levels(g, Z, cz, 1, nz - 1);
    free(X);
    free(Y);
    free(Z);
    bigs_free(&b);
}

int orc_projection(const orc_grid *g, double *u, double *v, double *w)
{
    dims_t d = dims(g);
    double *zero = zalloc(d.pl), *p = zalloc(d.F);
    double *dpdx = zalloc(d.pl * d.nz), *dpdy = zalloc(d.pl * d.nz), *dpdz = zalloc(d.pl * d.nz);
    int rc = orc_press_stag_array(g, 2, u, v, w, zero, zero, p, dpdx, dpdy);
    if (!rc) {
        orc_dpdz(g, p, dpdz);
        orc_project(g, u, v, w, dpdx, dpdy, dpdz);
    }
    free(zero);
    free(p);
    free(dpdx);
    free(dpdy);
    free(dpdz);
    return rc;
}

static int size_ok(const orc_grid *g) { return g->nz >= 5 && (g->nzt - 1) % 2 == 0; }

int orc_rollout_step(const orc_grid *g, double *u, double *v, double *w)
{
    if (!size_ok(g)) return 1;
    dims_t d = dims(g);
    double *cx = zalloc(d.F), *cy = zalloc(d.F), *cz = zalloc(d.F);
    orc_convec(g, u, v, w, cx, cy, cz);
    const double f = g->dt_nd * TADV1;
    for (int k = 1; k <= d.nz - 1; k++) /* 103_flosol.f90:115, :375-383 with RHS_f = RHS */
        for (size_t q = 0; q < d.pl; q++) {
            if (XOF(q, d.ldx) >= d.nx) continue;
            size_t o = q + d.pl * k;
            u[o] -= f * cx[o];
            v[o] -= f * cy[o];
            w[o] -= f * cz[o];
        }
    free(cx);
    free(cy);
    free(cz);
    return orc_projection(g, u, v, w);
}

double orc_ke_band(const orc_grid *g, const double *u, const double *v, const double *w,
                   double z_lo, double z_hi, double *lu, double *lv, double *lw)
{
    dims_t d = dims(g);
    if (lu) {
        memset(lu, 0, sizeof(double) * d.F);
        memset(lv, 0, sizeof(double) * d.F);
        memset(lw, 0, sizeof(double) * d.F);
    }
    double J = 0.0;
    for (int k = 1; k <= d.nz - 1; k++) {
        const double z = ((double)k - 0.5) * g->dz * g->z_i; /* 012_io.f90:295 */
        if (!(z > z_lo && z < z_hi)) continue;
        double Jk = 0.0;
        for (size_t q = 0; q < d.pl; q++) {
            if (XOF(q, d.ldx) >= d.nx) continue;
            size_t o = q + d.pl * k;
            const double tw = 0.5 * (w[o] + w[o + d.pl]);
            Jk += 0.5 * (u[o] * u[o] + v[o] * v[o] + tw * tw);
            if (lu) {
                lu[o] += u[o];
                lv[o] += v[o];
                lw[o] += 0.5 * tw;
                lw[o + d.pl] += 0.5 * tw;
            }
        }
        J += Jk;
    }
    return J;
}

/* bands of init_coef_press (109_press_stag_array.f90:4-68) for the global column of
   the npz >= 2 mode: rows 1..M, M = nz-1; row 1 bottom, row M top */
static void bands(double k2, int j, int M, double dz, double *a, double *b, double *c)
{
    const double idz2 = 1.0 / (dz * dz), idz = 1.0 / dz;
    if (k2 > 0) {
        *a = j == 1 ? 0.0 : idz2;
        *c = j == M ? 0.0 : idz2;
        *b = (j == 1 || j == M) ? -(k2 + idz2) : -(k2 + 2.0 * idz2);
    } else {
        *a = j == 1 ? 0.0 : -idz;
        *b = idz;
        *c = 0.0;
    }
}

int orc_projection_vjp(const orc_grid *g, double *lu, double *lv, double *lw)
{
    if (!size_ok(g)) return 1;
    dims_t d = dims(g);
    const int nz = d.nz, M = nz - 1, lhx = d.lhx, ny = d.ny;
    const size_t S = d.S, pl = d.pl;
    const double dz = g->dz;
    const double cst = 1.0 / ((double)d.nx * (double)d.ny);
    double *kx = zalloc(lhx), *ky = zalloc(g->lhy), *kx2 = zalloc(S), *ky2 = zalloc(S), *k2 = zalloc(S);
    int *nn = (int *)calloc(S, sizeof(int));
    orc_wavenumbers(g, kx, ky, kx2, ky2, k2, nn);

    /* transpose of the stress-free copy u,v(nz-1) = u,v(nz-2) (110_project.f90:51-54) */
    if (g->ubc_stress_free)
        for (size_t q = 0; q < pl; q++) {
            lu[q + pl * (nz - 2)] += lu[q + pl * (nz - 1)];
            lu[q + pl * (nz - 1)] = 0.0;
            lv[q + pl * (nz - 2)] += lv[q + pl * (nz - 1)];
            lv[q + pl * (nz - 1)] = 0.0;
        }
    /* w(1) = 0 and w(nz) = 0 are set, not updated (110_project.f90:55-60) */
    for (size_t q = 0; q < pl; q++) {
        lw[q + pl] = 0.0;
        lw[q + pl * nz] = 0.0;
    }
    /* spectra of the updated entries: u, v at 1..nz-1 (dpdx, dpdy), w at 2..nz-1 (dpdz) */
    cplx *Lx = (cplx *)calloc(S * (nz + 1), sizeof(cplx));
    cplx *Ly = (cplx *)calloc(S * (nz + 1), sizeof(cplx));
    cplx *Lz = (cplx *)calloc(S * (nz + 2), sizeof(cplx));
    cplx *nu = (cplx *)calloc(S * (nz + 1), sizeof(cplx));
#pragma omp parallel
    {
        double *t = zalloc(pl);
#pragma omp for schedule(dynamic)
        for (int it = 0; it < 3 * (nz + 1); it++) {
            int c = it % 3, k = it / 3;
            if (k < 1 || k > nz - 1 || (c == 2 && k < 2)) continue;
            const double *s = (c == 0 ? lu : c == 1 ? lv : lw) + pl * k;
            for (size_t q = 0; q < pl; q++) t[q] = cst * s[q];
            orc_fftn(g, t, (c == 0 ? Lx : c == 1 ? Ly : Lz) + S * k);
        }
        free(t);
    }
    /* mu = G^H L (G: dpdx = i kx p, dpdy = i ky p, dpdz(j) = (p(j) - p(j-1))/dz at j =
       2..nz-1); nu = T^-T mu with the transposed bands (sub c(j-1), super a(j+1)) */
#pragma omp parallel
    {
        cplx *mu = (cplx *)malloc(sizeof(cplx) * (M + 2));
        cplx *dp = (cplx *)malloc(sizeof(cplx) * (M + 2));
        double *cp = zalloc(M + 2);
#pragma omp for schedule(static)
        for (size_t q = 0; q < S; q++) {
            if (!nn[q]) continue;
            for (int j = 1; j <= M; j++)
                mu[j] = -I * kx2[q] * Lx[q + S * j] - I * ky2[q] * Ly[q + S * j] +
                        (Lz[q + S * j] - Lz[q + S * (j + 1)]) / dz;
            for (int j = 1; j <= M; j++) {
                double a, b, c, aj1 = 0, bj1, cj1, cjm1 = 0, am, bm;
                bands(k2[q], j, M, dz, &a, &b, &c);
                if (j > 1) bands(k2[q], j - 1, M, dz, &am, &bm, &cjm1);
                if (j < M) bands(k2[q], j + 1, M, dz, &aj1, &bj1, &cj1);
                const double sub = j > 1 ? cjm1 : 0.0, sup = j < M ? aj1 : 0.0;
                const double den = b - (j > 1 ? sub * cp[j - 1] : 0.0);
                cp[j] = sup / den;
                dp[j] = (mu[j] - (j > 1 ? sub * dp[j - 1] : 0.0)) / den;
                (void)a;
                (void)c;
            }
            nu[q + S * M] = dp[M];
            for (int j = M - 1; j >= 1; j--) nu[q + S * j] = dp[j] - cp[j] * nu[q + S * (j + 1)];
        }
        free(mu);
        free(dp);
        free(cp);
    }
    /* Dv^H nu (Dv: RHS(j) = i kx Hx(j) + i ky Hy(j) + (Hz(j+1) - Hz(j))/dz for k2 > 0,
       Hz(nz) a boundary plane; RHS(j) = Hz(j) at j >= 2 for the (0,0) mode,
       109_press_stag_array.f90:203-225), inverse transforms, subtraction */
#pragma omp parallel
    {
        cplx *A = (cplx *)malloc(sizeof(cplx) * S);
        double *t = zalloc(pl);
#pragma omp for schedule(dynamic)
        for (int it = 0; it < 3 * (nz + 1); it++) {
            int c = it % 3, k = it / 3;
            if (k < 1 || k > nz - 1) continue;
            for (size_t q = 0; q < S; q++) {
                if (!nn[q]) {
                    A[q] = 0;
                    continue;
                }
                const cplx n0 = nu[q + S * k], nm = k >= 2 ? nu[q + S * (k - 1)] : 0;
                if (c == 0)
                    A[q] = -I * kx2[q] * n0;
                else if (c == 1)
                    A[q] = -I * ky2[q] * n0;
                else if (k2[q] > 0)
                    A[q] = (nm - n0) / dz;
                else
                    A[q] = k >= 2 ? n0 : 0;
            }
            orc_ifftn(g, A, t);
            double *o = (c == 0 ? lu : c == 1 ? lv : lw) + pl * k;
            for (size_t q = 0; q < pl; q++)
                if (XOF(q, d.ldx) < d.nx) o[q] -= t[q];
        }
        free(A);
        free(t);
    }
    (void)ny;
    free(Lx);
    free(Ly);
    free(Lz);
    free(nu);
    free(kx);
    free(ky);
    free(kx2);
    free(ky2);
    free(k2);
    free(nn);
    return 0;
}

void orc_convec_vjp(const orc_grid *g, const double *u, const double *v, const double *w,
                    const double *lcx, const double *lcy, const double *lcz,
                    double *lu, double *lv, double *lw)
{
    dims_t d = dims(g);
    const int nz = d.nz;
    const size_t P = d.plb, pl = d.pl;
    const double idz = 1.0 / g->dz;
    const double r = 1.5 * 1.5; /* (nxt2/nxt) * (nyt2/nyt) */
    bigs_t b;
    convec_fields(g, u, v, w, &b);
    /* unpad^T = pad / r: adjoints of the padded cross products */
    double *LX = zalloc(d.FB), *LY = zalloc(d.FB), *LZ = zalloc(d.FB);
    pad_levels(g, lcx, LX, 1, nz - 1);
    pad_levels(g, lcy, LY, 1, nz - 1);
    pad_levels(g, lcz, LZ, 2, nz - 1); /* cross_z_big(1) = 0 does not depend on the state */
    for (size_t i = 0; i < d.FB; i++) {
        LX[i] /= r;
        LY[i] /= r;
        LZ[i] /= r;
    }
    for (size_t q = 0; q < P; q++) { /* levels outside the unpadded range carry nothing */
        LX[q] = LY[q] = LZ[q] = LZ[q + P] = 0.0;
        LX[q + P * nz] = LY[q + P * nz] = LZ[q + P * nz] = 0.0;
    }
    /* transposed cross product */
    double *aU = zalloc(d.FB), *aV = zalloc(d.FB), *aW = zalloc(d.FB);
    double *a1 = zalloc(d.FB), *a2 = zalloc(d.FB), *a3 = zalloc(d.FB);
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < P; q++) {
        for (int k = 1; k <= nz - 1; k++) {
            size_t o = q + P * k;
            const double lzk = LZ[o], lzk1 = (k + 1 <= nz - 1) ? LZ[o + P] : 0.0;
            a3[o] = -b.V[o] * LX[o] + b.U[o] * LY[o];
            aU[o] = b.O3[o] * LY[o] - 0.5 * b.O2[o] * lzk - 0.5 * b.O2[o + P] * lzk1;
            aV[o] = -b.O3[o] * LX[o] + 0.5 * b.O1[o] * lzk + 0.5 * b.O1[o + P] * lzk1;
        }
        for (int k = 2; k <= nz; k++) {
            size_t o = q + P * k;
            const double sX = LX[o - P] + (k <= nz - 1 ? LX[o] : 0.0);
            const double sY = LY[o - P] + (k <= nz - 1 ? LY[o] : 0.0);
            const double lz = k <= nz - 1 ? LZ[o] : 0.0;
            aW[o] = 0.5 * b.O2[o] * sX - 0.5 * b.O1[o] * sY;
            a2[o] = 0.5 * b.W[o] * sX - 0.5 * (b.U[o] + b.U[o - P]) * lz;
            a1[o] = -0.5 * b.W[o] * sY + 0.5 * (b.V[o] + b.V[o - P]) * lz;
        }
    }
    free(LX);
    free(LY);
    free(LZ);
    bigs_free(&b);
    /* pad^T = r * unpad */
    double *sU = zalloc(d.F), *sV = zalloc(d.F), *sW = zalloc(d.F);
    double *s1 = zalloc(d.F), *s2 = zalloc(d.F), *s3 = zalloc(d.F);
    unpad_levels(g, aU, sU, 1, nz - 1);
    unpad_levels(g, aV, sV, 1, nz - 1);
    unpad_levels(g, aW, sW, 2, nz);
    unpad_levels(g, a1, s1, 2, nz);
    unpad_levels(g, a2, s2, 2, nz);
    unpad_levels(g, a3, s3, 1, nz - 1);
    free(aU);
    free(aV);
    free(aW);
    free(a1);
    free(a2);
    free(a3);
    /* transposed vorticity: adjoints of dudy, dvdx, dwdx, dwdy, dudz, dvdz */
    double *ldudy = zalloc(d.F), *ldvdx = zalloc(d.F), *ldwdx = zalloc(d.F), *ldwdy = zalloc(d.F);
    double *ldudz = zalloc(d.F), *ldvdz = zalloc(d.F);
    for (size_t q = 0; q < pl; q++) {
        if (XOF(q, d.ldx) >= d.nx) continue;
        for (int k = 1; k <= nz - 1; k++) {
            size_t o = q + pl * k;
            s1[o] *= r, s2[o] *= r, s3[o] *= r;
            sU[o] *= r, sV[o] *= r, sW[o] *= r;
            ldvdx[o] = s3[o];
            ldudy[o] = -s3[o];
        }
        s1[q + pl * nz] *= r, s2[q + pl * nz] *= r, sW[q + pl * nz] *= r;
        for (int k = 2; k <= nz - 1; k++) {
            size_t o = q + pl * k;
            ldwdy[o] += s1[o];
            ldvdz[o] = -s1[o];
            ldudz[o] = s2[o];
            ldwdx[o] -= s2[o];
        }
        /* vort1(nz) = 0.5*(dwdy(nz) + dwdy(nz-1)) - 0, vort2(nz) = 0 - 0.5*(dwdx(nz) + dwdx(nz-1)) */
        const size_t on = q + pl * nz, om = q + pl * (nz - 1);
        ldwdy[on] += 0.5 * s1[on];
        ldwdy[om] += 0.5 * s1[on];
        ldwdx[on] -= 0.5 * s2[on];
        ldwdx[om] -= 0.5 * s2[on];
    }
    /* transposed derivatives: ddx^T = -ddx, ddy^T = -ddy, level differences term by term */
    const int nlev = nz + 1;
    double *t = zalloc(d.F);
    orc_ddy(g, t, ldudy, nlev);
    for (size_t i = 0; i < d.F; i++) lu[i] -= XOF(i % pl, d.ldx) < d.nx ? t[i] : 0.0;
    orc_ddx(g, t, ldvdx, nlev);
    for (size_t i = 0; i < d.F; i++) lv[i] -= XOF(i % pl, d.ldx) < d.nx ? t[i] : 0.0;
    orc_ddx(g, t, ldwdx, nlev);
    for (size_t i = 0; i < d.F; i++) lw[i] -= XOF(i % pl, d.ldx) < d.nx ? t[i] : 0.0;
    orc_ddy(g, t, ldwdy, nlev);
    for (size_t i = 0; i < d.F; i++) lw[i] -= XOF(i % pl, d.ldx) < d.nx ? t[i] : 0.0;
    free(t);
    for (size_t q = 0; q < pl; q++) {
        if (XOF(q, d.ldx) >= d.nx) continue;
        for (int k = 2; k <= nz - 1; k++) { /* dudz(k) = (u(k) - u(k-1))/dz */
            size_t o = q + pl * k;
            lu[o] += ldudz[o] * idz;
            lu[o - pl] -= ldudz[o] * idz;
            lv[o] += ldvdz[o] * idz;
            lv[o - pl] -= ldvdz[o] * idz;
        }
        for (int k = 0; k <= nz; k++) {
            size_t o = q + pl * k;
            lu[o] += sU[o];
            lv[o] += sV[o];
            lw[o] += sW[o];
        }
    }
    free(sU);
    free(sV);
    free(sW);
    free(s1);
    free(s2);
    free(s3);
    free(ldudy);
    free(ldvdx);
    free(ldwdx);
    free(ldwdy);
    free(ldudz);
    free(ldvdz);
}

int orc_rollout_step_vjp(const orc_grid *g, const double *u, const double *v, const double *w,
                         double *lu, double *lv, double *lw)
{
    if (!size_ok(g)) return 1;
    dims_t d = dims(g);
    int rc = orc_projection_vjp(g, lu, lv, lw);
    if (rc) return rc;
    double *lcx = zalloc(d.F), *lcy = zalloc(d.F), *lcz = zalloc(d.F);
    const double f = -g->dt_nd * TADV1;
    for (int k = 1; k <= d.nz - 1; k++)
        for (size_t q = 0; q < d.pl; q++) {
            if (XOF(q, d.ldx) >= d.nx) continue;
            size_t o = q + d.pl * k;
            lcx[o] = f * lu[o];
            lcy[o] = f * lv[o];
            lcz[o] = f * lw[o];
        }
    orc_convec_vjp(g, u, v, w, lcx, lcy, lcz, lu, lv, lw);
    free(lcx);
    free(lcy);
    free(lcz);
    return 0;
}

int orc_rollout_grad(const orc_grid *g, int nsteps, const double *u0, const double *v0,
                     const double *w0, double z_lo, double z_hi, double *J,
                     double *gu, double *gv, double *gw)
{
    if (!size_ok(g) || nsteps < 0) return 1;
    dims_t d = dims(g);
    const size_t F = d.F;
    double *ck = zalloc(F * 3 * (size_t)(nsteps + 1)); /* state of every step */
    memcpy(ck, u0, sizeof(double) * F);
    memcpy(ck + F, v0, sizeof(double) * F);
    memcpy(ck + 2 * F, w0, sizeof(double) * F);
    int rc = 0;
    for (int n = 0; n < nsteps && !rc; n++) {
        double *s = ck + 3 * F * (size_t)n, *s1 = s + 3 * F;
        memcpy(s1, s, sizeof(double) * 3 * F);
        rc = orc_rollout_step(g, s1, s1 + F, s1 + 2 * F);
    }
    if (!rc) {
        double *s = ck + 3 * F * (size_t)nsteps;
        *J = orc_ke_band(g, s, s + F, s + 2 * F, z_lo, z_hi, gu, gv, gw);
        for (int n = nsteps - 1; n >= 0 && gu && !rc; n--) {
            double *sn = ck + 3 * F * (size_t)n;
            rc = orc_rollout_step_vjp(g, sn, sn + F, sn + 2 * F, gu, gv, gw);
        }
    }
    free(ck);
    return rc;
}
