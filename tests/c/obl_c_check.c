/* obl_c_check.c -- the C ABI (include/obl.h) driven from plain C with host arrays, as a C
 * or Fortran host of the reference would call it.
 *
 *   ddx, ddy        of sin(3x)cos(2y) against the closed form (004_derivatives.f90:18-81);
 *   zero_padding    of a band-limited plane against its values on the 3/2 grid
 *                   (108_01_padd.f90:73-132);
 *   press_stag_array + dpdz + project (Neumann top) on band-limited u, v, w with
 *   w = 0 at levels 1 and nz: afterwards ddx(u) + ddy(v) + ddz_w(w) vanishes at levels
 *   1..nz-1 (109_press_stag_array.f90:107-319, 110_project.f90:4-62).
 *
 * Exit status: 0 all checks passed; 1 a check failed; 2 a call failed; 3 no CUDA device.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "obl.h"

static const double PI = 3.14159265358979323846;

#define CALL(x)                                                                                  \
    do {                                                                                         \
        int rc_ = (x);                                                                           \
        if (rc_ != OBL_OK) {                                                                     \
            char m_[256];                                                                        \
            obl_last_error(ctx, m_, sizeof m_);                                                  \
            fprintf(stderr, "%s failed: %d (%s)\n", #x, rc_, m_);                              \
            return 2;                                                                            \
        }                                                                                        \
    } while (0)

static int check(const char *what, double err, double tol)
{
    printf("%-36s %.3e (tolerance %.1e)\n", what, err, tol);
    return err <= tol ? 0 : 1;
}

int main(void)
{
    const int nx = 64, ny = 48, nzt = 17;
    obl_grid g = {nx, ny, nzt, 2 * PI * 1000.0, 2 * PI * 1000.0, 1000.0, 1000.0, 0.5, 1.0};
    obl_options o = {OBL_PREC_F64, OBL_TOP_NEUMANN, 0, -1.0, 0};
    obl_ctx *ctx = NULL;
    int rc = obl_ctx_create(&g, &o, &ctx);
    if (rc == OBL_ERR_NODEV) {
        printf("no CUDA device\n");
        return 3;
    }
    if (rc != OBL_OK) {
        fprintf(stderr, "obl_ctx_create failed: %d\n", rc);
        return 2;
    }
    obl_info in;
    CALL(obl_ctx_info(ctx, &in));
    const int ldx = in.ldx, nz = in.nz, nlev = nz + 1;
    const long long nf = in.field_elems, nd = in.dfield_elems;
    const double kx0 = 2 * PI / in.lx, ky0 = 2 * PI / in.ly;
#define AT(a, x, y, z) (a)[(x) + (long long)ldx * ((y) + (long long)ny * (z))]
    double *f = calloc(nf, sizeof(double)), *d = calloc(nf, sizeof(double));
    double *u = calloc(nf, sizeof(double)), *v = calloc(nf, sizeof(double)), *w = calloc(nf, sizeof(double));
    double *p = calloc(nf, sizeof(double)), *dpdx = calloc(nd, sizeof(double)), *dpdy = calloc(nd, sizeof(double));
    double *dpdz = calloc(nd, sizeof(double)), *e1 = calloc(nf, sizeof(double)), *e2 = calloc(nf, sizeof(double));
    double *big = calloc((size_t)in.nxt2 * in.nyt2, sizeof(double));
    int bad = 0;

    /* ddx, ddy of sin(3x)cos(2y) on every level */
    for (int z = 0; z < nlev; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x)
                AT(f, x, y, z) = sin(3 * 2 * PI * x / nx) * cos(2 * 2 * PI * y / ny);
    double e = 0, m = 0;
    CALL(obl_ddx(ctx, d, f, nlev));
    for (int z = 0; z < nlev; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const double ex = 3 * kx0 * cos(3 * 2 * PI * x / nx) * cos(2 * 2 * PI * y / ny);
                e = fmax(e, fabs(AT(d, x, y, z) - ex));
                m = fmax(m, fabs(ex));
            }
    bad |= check("ddx vs closed form (max rel)", e / m, 1e-12);
    e = 0;
    m = 0;
    CALL(obl_ddy(ctx, d, f, nlev));
    for (int z = 0; z < nlev; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const double ey = -2 * ky0 * sin(3 * 2 * PI * x / nx) * sin(2 * 2 * PI * y / ny);
                e = fmax(e, fabs(AT(d, x, y, z) - ey));
                m = fmax(m, fabs(ey));
            }
    bad |= check("ddy vs closed form (max rel)", e / m, 1e-12);

    /* zero_padding of one band-limited plane */
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            f[x + (long long)ldx * y] = 1.0 + sin(2 * 2 * PI * x / nx + 0.3) * cos(3 * 2 * PI * y / ny);
    CALL(obl_zero_padding(ctx, f, big, 1));
    e = 0;
    for (int y = 0; y < in.nyt2; ++y)
        for (int x = 0; x < in.nxt2; ++x) {
            const double ex = 1.0 + sin(2 * 2 * PI * x / in.nxt2 + 0.3) * cos(3 * 2 * PI * y / in.nyt2);
            e = fmax(e, fabs(big[x + (long long)in.nxt2 * y] - ex));
        }
    bad |= check("zero_padding vs 3/2-grid values (max)", e, 1e-12);

    /* projection: band-limited u, v, w; w = 0 at levels 1 and nz */
    for (int z = 0; z < nlev; ++z) {
        const double hz = (z >= 1) ? sin(PI * (z - 1) / (nz - 1)) : 0.0;
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const double X = 2 * PI * x / nx, Y = 2 * PI * y / ny;
                AT(u, x, y, z) = sin(X) * cos(2 * Y) * (1.0 + 0.1 * z);
                AT(v, x, y, z) = cos(3 * X) * sin(Y) * (2.0 - 0.05 * z);
                AT(w, x, y, z) = sin(2 * X) * sin(3 * Y) * hz;
            }
    }
    CALL(obl_press_stag_array(ctx, u, v, w, NULL, NULL, p, dpdx, dpdy));
    CALL(obl_dpdz(ctx, p, dpdz));
    CALL(obl_project(ctx, u, v, w, dpdx, dpdy, dpdz));
    CALL(obl_ddx(ctx, e1, u, nlev));
    CALL(obl_ddy(ctx, e2, v, nlev));
    e = 0;
    m = 0;
    for (int z = 1; z <= nz - 1; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const double dwdz = (AT(w, x, y, z + 1) - AT(w, x, y, z)) / in.dz;
                e = fmax(e, fabs(AT(e1, x, y, z) + AT(e2, x, y, z) + dwdz));
                m = fmax(m, fabs(AT(e1, x, y, z)));
            }
    bad |= check("divergence after projection (max rel)", e / m, 1e-10);

    free(f); free(d); free(u); free(v); free(w); free(p); free(dpdx); free(dpdy); free(dpdz);
    free(e1); free(e2); free(big);
    CALL(obl_ctx_destroy(ctx));
    printf(bad ? "C ABI check FAILED\n" : "C ABI check passed\n");
    return bad ? 1 : 0;
}
