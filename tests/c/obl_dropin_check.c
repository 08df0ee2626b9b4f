/* obl_dropin_check.c -- the drop-in routines of overlappingbls_b200/fortran/obl_dropin.f90
 * restated in C, line for line, and driven by the slice of the reference's time loop that
 * calls them (103_flosol.f90:168-188):
 *
 *     call press_stag_array(p, dpdx, dpdy)
 *     dpdz(1:nxt, 1:nynpy, 1:nz-1) = (p(1:nxt, 1:nynpy, 1:nz-1) - p(1:nxt, 1:nynpy, 0:nz-2))/dz
 *     call project()
 *
 * As in the reference, u, v, w, divtz, p, dpdx, dpdy, dpdz and T_s are module ("global")
 * real(8) arrays in the Fortran layout, press_stag_array(func, dfdx, dfdy) reads u, v, w and
 * divtz from them, project() takes no arguments, and init_coef_press() (here: the GPU
 * context) runs after the non-dimensionalisation.  No Fortran compiler exists in this
 * image, so this C restatement is what runs; the test compares its outputs with the oracle.
 *
 *   obl_dropin_check IN OUT single|neumann
 * IN:  int32 nxt, nyt, nzt, theta_flag; float64 lx_tot, ly_tot, lz_tot, dt (non-dimensional),
 *      z_i, u_scale (dimensional, for the surface-temperature term), dz (non-dimensional,
 *      as init_parameter and init_nondimensional leave it); then u, v, w, divtz
 *      (ldx, nyt, 0:nz) and T_s (nxt, nyt).
 * OUT: p (ldx, nyt, 0:nz), dpdx, dpdy, dpdz (ldx, nyt, nz), u, v, w (ldx, nyt, 0:nz).
 * Exit status: 0 ok; 2 a call or file operation failed; 3 no CUDA device.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "obl.h"

/* ---- "module param" ---- */
static int nxt, nyt, nzt, nz, ldx, theta_flag;
static int jt = 1, theta_init_time = 0, lbc = 0;
static double lx_tot, ly_tot, lz_tot, dt, dz, z_i, u_scale;
static const double g = 9.81; /* 001_param.f90:34 */
static int top_mode;

/* ---- "module sim_param" and "module bottombc" ---- */
static double *u, *v, *w, *divtz, *p, *dpdx, *dpdy, *dpdz, *T_s;

static obl_ctx *ctx;

#define PL ((size_t)ldx * nyt)

static void die(const char *what, int rc)
{
    char m[256] = "";
    if (ctx) obl_last_error(ctx, m, sizeof m);
    fprintf(stderr, "%s: status %d %s\n", what, rc, m);
    exit(rc == OBL_ERR_NODEV ? 3 : 2);
}

/* init_coef_press (102_initial.f90:53): the GPU context, from non-dimensional values */
static void init_coef_press(void)
{
    obl_grid gr = {nxt, nyt, nzt, lx_tot, ly_tot, lz_tot, 1.0, dt, 1.0};
    obl_options o = {OBL_PREC_F64, top_mode, 0, -1.0, 0};
    int rc = obl_ctx_create(&gr, &o, &ctx);
    if (rc) die("obl_ctx_create", rc);
}

/* calc_hor_avg3 (202_parallel.f90:1041-1059) with npy = 1 */
static double calc_hor_avg3(const double *in)
{
    double s = 0;
    for (int j = 0; j < nyt; ++j)
        for (int i = 0; i < nxt; ++i) s += in[i + (size_t)nxt * j];
    return s / ((double)nxt * nyt);
}

/* press_stag_array(func, dfdx, dfdy) of obl_dropin.f90 */
static void press_stag_array(double *func, double *dfdx, double *dfdy)
{
    double *rbot = malloc(sizeof(double) * PL);
    memcpy(rbot, divtz + PL * 1, sizeof(double) * PL);
    if (theta_flag && jt > theta_init_time && lbc == 0) {
        const double T_s_mn = calc_hor_avg3(T_s);
        for (int j = 0; j < nyt; ++j)
            for (int i = 0; i < nxt; ++i)
                rbot[i + (size_t)ldx * j] = divtz[PL * 1 + i + (size_t)ldx * j] -
                                            g * (z_i / (u_scale * u_scale)) * (T_s[i + (size_t)nxt * j] - T_s_mn);
    }
    int rc = obl_press_stag_array(ctx, u, v, w, rbot, divtz + PL * nz, func, dfdx, dfdy);
    free(rbot);
    if (rc) die("press_stag_array", rc);
}

/* project() of obl_dropin.f90 */
static void project(void)
{
    int rc = obl_project(ctx, u, v, w, dpdx, dpdy, dpdz);
    if (rc) die("project", rc);
}

static void rd(FILE *f, void *a, size_t sz, size_t n)
{
    if (fread(a, sz, n, f) != n) die("read", OBL_ERR_ARG);
}

static void wr(FILE *f, const double *a, size_t n)
{
    if (fwrite(a, sizeof(double), n, f) != n) die("write", OBL_ERR_ARG);
}

int main(int argc, char **argv)
{
    if (argc != 4) {
        fprintf(stderr, "usage: %s IN OUT single|neumann\n", argv[0]);
        return 2;
    }
    top_mode = strcmp(argv[3], "neumann") == 0 ? OBL_TOP_NEUMANN : OBL_TOP_SINGLE_RANK;
    FILE *f = fopen(argv[1], "rb");
    if (!f) die("open IN", OBL_ERR_ARG);
    int hdr[4];
    double dh[7];
    rd(f, hdr, sizeof(int), 4);
    rd(f, dh, sizeof(double), 7);
    nxt = hdr[0], nyt = hdr[1], nzt = hdr[2], theta_flag = hdr[3];
    lx_tot = dh[0], ly_tot = dh[1], lz_tot = dh[2], dt = dh[3], z_i = dh[4], u_scale = dh[5];
    nz = nzt; /* npz = 1 (102_initial.f90:119) */
    ldx = 2 * (nxt / 2 + 1);
    dz = dh[6];
    const size_t nf = PL * (nz + 1), nd = PL * nz;
    u = malloc(sizeof(double) * nf), v = malloc(sizeof(double) * nf), w = malloc(sizeof(double) * nf);
    divtz = malloc(sizeof(double) * nf), p = calloc(nf, sizeof(double));
    dpdx = calloc(nd, sizeof(double)), dpdy = calloc(nd, sizeof(double)), dpdz = calloc(nd, sizeof(double));
    T_s = malloc(sizeof(double) * (size_t)nxt * nyt);
    rd(f, u, sizeof(double), nf);
    rd(f, v, sizeof(double), nf);
    rd(f, w, sizeof(double), nf);
    rd(f, divtz, sizeof(double), nf);
    rd(f, T_s, sizeof(double), (size_t)nxt * nyt);
    fclose(f);

    init_coef_press();

    /* 103_flosol.f90:168-188 */
    press_stag_array(p, dpdx, dpdy);
    for (int jz = 1; jz <= nz - 1; ++jz)
        for (int jy = 0; jy < nyt; ++jy)
            for (int jx = 0; jx < nxt; ++jx)
                dpdz[jx + (size_t)ldx * jy + PL * (jz - 1)] =
                    (p[jx + (size_t)ldx * jy + PL * jz] - p[jx + (size_t)ldx * jy + PL * (jz - 1)]) / dz;
    project();

    FILE *o = fopen(argv[2], "wb");
    if (!o) die("open OUT", OBL_ERR_ARG);
    wr(o, p, nf);
    wr(o, dpdx, nd);
    wr(o, dpdy, nd);
    wr(o, dpdz, nd);
    wr(o, u, nf);
    wr(o, v, nf);
    wr(o, w, nf);
    fclose(o);
    obl_ctx_destroy(ctx);
    free(u); free(v); free(w); free(divtz); free(p); free(dpdx); free(dpdy); free(dpdz); free(T_s);
    printf("drop-in slice done\n");
    return 0;
}
