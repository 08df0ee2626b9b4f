/*
 * obl_oracle.c -- FP64 CPU restatement of the OverlappingBLs hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker and the CPU baseline.  Nothing in the
 * product library (libobl_b200.so) links or calls this file.
 *
 * PARITY UNPINNED: the reference ships no golden vectors or tests and cannot be
 * built here (Fortran + MPI + FFTW absent).  See obl_oracle.h for what pins it.
 *
 * Every routine cites the reference file:line it restates (paths relative to the
 * reference project, SBL/code/ is canonical; BBL/SBBL carry identical copies of
 * these files).  The FFT is this file's own mixed-radix Cooley-Tukey with the
 * unnormalised FFTW sign conventions the reference relies on
 * (SBL/code/002_fft.f90:97-113).
 */
#include "obl_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

static const double PI = 3.1415926535897932384626433; /* 001_param.f90:32 */
static const double TADV1 = 1.5;                       /* 001_param.f90:152 */
static const double BOGUS = -1234567890.0;             /* 001_param.f90:40 */

/* ------------------------------------------------------------------------- */
/* threads                                                                    */
/* ------------------------------------------------------------------------- */
void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* FFT: recursive decimation-in-time mixed radix (4, 2, 3, 5, generic prime).  */
/* Twiddle table w[j] = exp(-2*pi*i*j/N) of the top-level length N is cached.  */
/* ------------------------------------------------------------------------- */
#define ORC_MAXN 8192
static cplx *g_tw[ORC_MAXN + 1];

static const cplx *twiddles(int n)
{
    cplx *t = __atomic_load_n(&g_tw[n], __ATOMIC_ACQUIRE);
    if (t) return t;
    cplx *nt = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    for (int j = 0; j < n; j++) {
        double a = -2.0 * PI * (double)j / (double)n;
        nt[j] = cos(a) + I * sin(a);
    }
    cplx *expected = NULL;
    if (!__atomic_compare_exchange_n(&g_tw[n], &expected, nt, 0, __ATOMIC_ACQ_REL,
                                     __ATOMIC_ACQUIRE)) {
        free(nt);
        return expected;
    }
    return nt;
}

static int smallest_factor(int n)
{
    if (n % 4 == 0) return 4;
    if (n % 2 == 0) return 2;
    if (n % 3 == 0) return 3;
    if (n % 5 == 0) return 5;
    for (int f = 7; f * f <= n; f += 2)
        if (n % f == 0) return f;
    return n;
}

/* out[k] = sum_j in[j*s] * W^(j*k), W = exp(sign*2*pi*i/n); tw is the table of the
   top-level length with wstep = Ntop/n. */
static void fft_rec(int n, const cplx *in, int s, cplx *out, const cplx *tw,
                    int wstep, int sign)
{
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    int R = smallest_factor(n);
    int m = n / R;
    for (int r = 0; r < R; r++)
        fft_rec(m, in + (size_t)r * s, s * R, out + (size_t)r * m, tw, wstep * R, sign);

    if (R == 2) {
        for (int k = 0; k < m; k++) {
            cplx w = tw[(size_t)k * wstep];
            if (sign > 0) w = conj(w);
            cplx a = out[k], b = out[k + m] * w;
            out[k] = a + b;
            out[k + m] = a - b;
        }
        return;
    }
    if (R == 4) {
        for (int k = 0; k < m; k++) {
            cplx w1 = tw[(size_t)k * wstep], w2 = tw[(size_t)2 * k * wstep],
                 w3 = tw[(size_t)3 * k * wstep];
            if (sign > 0) {
                w1 = conj(w1);
                w2 = conj(w2);
                w3 = conj(w3);
            }
            cplx a0 = out[k], a1 = out[k + m] * w1, a2 = out[k + 2 * m] * w2,
                 a3 = out[k + 3 * m] * w3;
            cplx t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = a1 - a3;
            /* multiply t3 by -i (forward) or +i (backward) */
            cplx t3r = (sign < 0) ? (cimag(t3) - I * creal(t3)) : (-cimag(t3) + I * creal(t3));
            out[k] = t0 + t2;
            out[k + m] = t1 + t3r;
            out[k + 2 * m] = t0 - t2;
            out[k + 3 * m] = t1 - t3r;
        }
        return;
    }
    cplx tbuf[16];
    cplx *t = (R <= 16) ? tbuf : (cplx *)malloc(sizeof(cplx) * (size_t)R);
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < R; r++) {
            cplx w = tw[(size_t)r * k * wstep];
            if (sign > 0) w = conj(w);
            t[r] = out[(size_t)r * m + k] * w;
        }
        for (int q = 0; q < R; q++) {
            cplx acc = 0;
            for (int r = 0; r < R; r++) {
                cplx w = tw[(size_t)((r * q) % R) * m * wstep];
                if (sign > 0) w = conj(w);
                acc += t[r] * w;
            }
            out[k + (size_t)q * m] = acc;
        }
    }
    if (t != tbuf) free(t);
}

void orc_fft_c2c(int n, const cplx *in, cplx *out, int sign)
{
    if (n <= 0) return;
    if (n > ORC_MAXN) { /* fall back to the naive DFT for absurd sizes */
        orc_dft_naive(n, in, out, sign);
        return;
    }
    const cplx *tw = twiddles(n);
    if (in == out) {
        cplx *tmp = (cplx *)malloc(sizeof(cplx) * (size_t)n);
        memcpy(tmp, in, sizeof(cplx) * (size_t)n);
        fft_rec(n, tmp, 1, out, tw, 1, sign);
        free(tmp);
    } else {
        fft_rec(n, in, 1, out, tw, 1, sign);
    }
}

void orc_dft_naive(int n, const cplx *in, cplx *out, int sign)
{
    const long double PIL = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < n; k++) {
        long double sr = 0, si = 0;
        for (int j = 0; j < n; j++) {
            long long jk = ((long long)j * k) % n;
            long double a = (long double)sign * 2.0L * PIL * (long double)jk / (long double)n;
            long double c = cosl(a), s = sinl(a);
            long double xr = creal(in[j]), xi = cimag(in[j]);
            sr += xr * c - xi * s;
            si += xr * s + xi * c;
        }
        out[k] = (double)sr + I * (double)si;
    }
}

/* r2c (FFTW dft_r2c_1d, unnormalised): even n via one n/2 complex FFT. */
void orc_fft_r2c(int n, const double *in, cplx *out)
{
    if (n % 2 != 0 || n < 4) {
        cplx *z = (cplx *)calloc((size_t)n * 2, sizeof(cplx));
        for (int j = 0; j < n; j++) z[j] = in[j];
        orc_fft_c2c(n, z, z + n, -1);
        for (int k = 0; k <= n / 2; k++) out[k] = z[n + k];
        free(z);
        return;
    }
    int h = n / 2;
    cplx zb[1024];
    cplx *z = (h <= 512) ? zb : (cplx *)malloc(sizeof(cplx) * (size_t)h * 2);
    cplx *Z = z + h;
    for (int m = 0; m < h; m++) z[m] = in[2 * m] + I * in[2 * m + 1];
    orc_fft_c2c(h, z, Z, -1);
    const cplx *tw = twiddles(n);
    for (int k = 0; k <= h; k++) {
        cplx zk = Z[k % h], zc = conj(Z[(h - k) % h]);
        cplx E = 0.5 * (zk + zc);
        cplx O = -0.5 * I * (zk - zc);
        out[k] = (k == h) ? (E - O) /* W^h = -1 exactly */ : (E + tw[k] * O);
    }
    if (z != zb) free(z);
}

/* c2r (FFTW dft_c2r_1d, unnormalised): imaginary parts of DC and Nyquist ignored. */
void orc_fft_c2r(int n, const cplx *in, double *out)
{
    if (n % 2 != 0 || n < 4) {
        cplx *z = (cplx *)calloc((size_t)n * 2, sizeof(cplx));
        for (int k = 0; k < n; k++) {
            if (k == 0) z[k] = creal(in[0]);
            else if (2 * k == n) z[k] = creal(in[k]);
            else if (k < n / 2 + 1) z[k] = in[k];
            else z[k] = conj(in[n - k]);
        }
        orc_fft_c2c(n, z, z + n, +1);
        for (int j = 0; j < n; j++) out[j] = creal(z[n + j]);
        free(z);
        return;
    }
    int h = n / 2;
    cplx zb[1024];
    cplx *z = (h <= 512) ? zb : (cplx *)malloc(sizeof(cplx) * (size_t)h * 2);
    cplx *Zt = z + h;
    const cplx *tw = twiddles(n);
    for (int k = 0; k < h; k++) {
        /* Hermitian extension Xh: Xh[0], Xh[h] real; Xh[k+h] = conj(Xh[h-k]) */
        cplx xk = (k == 0) ? (cplx)creal(in[0]) : in[k];
        cplx xkh = (k == 0) ? (cplx)creal(in[h]) : conj(in[h - k]);
        cplx Ee = xk + xkh;
        cplx Oo = (xk - xkh) * conj(tw[k]); /* * exp(+2 pi i k/n) */
        Zt[k] = Ee + I * Oo;
    }
    orc_fft_c2c(h, Zt, z, +1);
    for (int m = 0; m < h; m++) {
        out[2 * m] = creal(z[m]);
        out[2 * m + 1] = cimag(z[m]);
    }
    if (z != zb) free(z);
}

/* ------------------------------------------------------------------------- */
/* grid setup: init_parameter (102_initial.f90:119-141) and                    */
/* init_nondimensional (102_initial.f90:186-199)                               */
/* ------------------------------------------------------------------------- */
int orc_grid_init(orc_grid *g)
{
    if (g->nxt < 4 || g->nyt < 4 || g->nzt < 3) return 1;
    if (g->nxt % 2 || g->nyt % 2) return 1;
    g->nz = g->nzt; /* npz = 1: nz = (nzt-1)/1 + 1 */
    g->nxt2 = 3 * g->nxt / 2;
    g->nyt2 = 3 * g->nyt / 2;
    g->lhx = g->nxt / 2 + 1;
    g->lhy = g->nyt / 2 + 1;
    g->ldx = 2 * g->lhx;
    g->ldy = 2 * g->lhy;
    g->lhx2 = g->nxt2 / 2 + 1;
    g->ldx2 = 2 * g->lhx2;
    g->lhy2 = g->nyt2 / 2 + 1;
    g->ldy2 = 2 * g->lhy2;
    double dz_dim = g->lz_tot / (double)(g->nzt - 1);
    g->lx = g->lx_tot / g->z_i;
    g->ly = g->ly_tot / g->z_i;
    g->lz = g->lz_tot / g->z_i;
    g->dz = dz_dim / g->z_i;
    g->dt_nd = g->dt * g->u_scale / g->z_i;
    /* warm the twiddle cache before any parallel region */
    twiddles(g->nxt);
    twiddles(g->nyt);
    twiddles(g->nxt2);
    twiddles(g->nyt2);
    twiddles(g->nxt / 2);
    twiddles(g->nyt / 2);
    twiddles(g->nxt2 / 2);
    twiddles(g->nyt2 / 2);
    return 0;
}

/* init_wavenumber (002_fft.f90:121-167), npy = 1 so the *_mpi tables equal these. */
void orc_wavenumbers(const orc_grid *g, double *kx, double *ky, double *kx2d,
                     double *ky2d, double *k2, int *notnyq)
{
    int lhx = g->lhx, lhy = g->lhy, nyt = g->nyt, nxt = g->nxt;
    for (int i = 0; i < lhx; i++) kx[i] = (((double)i * 2.0) * PI) / g->lx; /* :131 */
    for (int i = 0; i < lhy; i++) ky[i] = (((double)i * 2.0) * PI) / g->ly; /* :132 */
    if (nxt % 2 == 0) kx[lhx - 1] = 0.0;                                   /* :135-137 */
    if (nyt % 2 == 0) ky[lhy - 1] = 0.0;                                   /* :138-140 */
    for (int j = 0; j < nyt; j++) {
        double kyv = (((double)(((j + nyt / 2) % nyt) - nyt / 2) * 2.0) * PI) / g->ly; /* :147 */
        for (int i = 0; i < lhx; i++) {
            kx2d[i + lhx * j] = kx[i]; /* :143-145 */
            ky2d[i + lhx * j] = kyv;   /* :147-153 */
            notnyq[i + lhx * j] = 1;
        }
    }
    if (nxt % 2 == 0)
        for (int j = 0; j < nyt; j++) { /* :157-160 */
            ky2d[(lhx - 1) + lhx * j] = 0.0;
            notnyq[(lhx - 1) + lhx * j] = 0;
        }
    if (nyt % 2 == 0)
        for (int i = 0; i < lhx; i++) { /* :161-165 */
            kx2d[i + lhx * (nyt / 2)] = 0.0;
            ky2d[i + lhx * (nyt / 2)] = 0.0;
            notnyq[i + lhx * (nyt / 2)] = 0;
        }
    for (int q = 0; q < lhx * nyt; q++) k2[q] = kx2d[q] * kx2d[q] + ky2d[q] * ky2d[q]; /* :167 */
}

/* ------------------------------------------------------------------------- */
/* derivatives (004_derivatives.f90)                                          */
/* ------------------------------------------------------------------------- */
void orc_ddx(const orc_grid *g, double *dfdx, const double *fun, int nlev)
{
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, lhx = g->lhx;
    double *kx = (double *)malloc(sizeof(double) * lhx);
    for (int i = 0; i < lhx; i++) kx[i] = (((double)i * 2.0) * PI) / g->lx;
    kx[lhx - 1] = 0.0;
    const double cst = 1.0 / nxt; /* :31 */
    long nrow = (long)nyt * nlev;
#pragma omp parallel
    {
        double *t = (double *)malloc(sizeof(double) * nxt);
        cplx *arr = (cplx *)malloc(sizeof(cplx) * lhx);
#pragma omp for schedule(static)
        for (long r = 0; r < nrow; r++) { /* :33-39 */
            const double *f = fun + (size_t)r * ldx;
            for (int x = 0; x < nxt; x++) t[x] = cst * f[x];
            orc_fft_r2c(nxt, t, arr);
            for (int k = 0; k < lhx; k++) arr[k] = (I * kx[k]) * arr[k]; /* :36 */
            orc_fft_c2r(nxt, arr, dfdx + (size_t)r * ldx);
        }
        free(t);
        free(arr);
    }
    free(kx);
}

void orc_ddy(const orc_grid *g, double *dfdy, const double *fun, int nlev)
{
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, lhy = g->lhy;
    double *ky = (double *)malloc(sizeof(double) * lhy);
    for (int i = 0; i < lhy; i++) ky[i] = (((double)i * 2.0) * PI) / g->ly;
    ky[lhy - 1] = 0.0;
    const double cst = 1.0 / nyt; /* :60 */
    long ncol = (long)nxt * nlev;
#pragma omp parallel
    {
        double *t = (double *)malloc(sizeof(double) * nyt);
        double *o = (double *)malloc(sizeof(double) * nyt);
        cplx *arr = (cplx *)malloc(sizeof(cplx) * lhy);
#pragma omp for schedule(static)
        for (long c = 0; c < ncol; c++) { /* :71-79, transposes are copies for npy = 1 */
            int x = (int)(c % nxt);
            long z = c / nxt;
            const double *f = fun + (size_t)z * ldx * nyt + x;
            for (int y = 0; y < nyt; y++) t[y] = cst * f[(size_t)y * ldx];
            orc_fft_r2c(nyt, t, arr);
            for (int k = 0; k < lhy; k++) arr[k] = (I * ky[k]) * arr[k]; /* :75 */
            orc_fft_c2r(nyt, arr, o);
            double *d = dfdy + (size_t)z * ldx * nyt + x;
            for (int y = 0; y < nyt; y++) d[(size_t)y * ldx] = o[y];
        }
        free(t);
        free(o);
        free(arr);
    }
    free(ky);
}

void orc_ddz_uv(const orc_grid *g, double *dfdz, const double *fun)
{
    /* single rank: coordz == 0 and coordz == npz-1 (004_derivatives.f90:85-116) */
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, nz = g->nz;
    size_t pl = (size_t)ldx * nyt;
    const double cst = 1.0 / g->dz;
    for (size_t q = 0; q < pl; q++) dfdz[q] = BOGUS; /* :100 */
    for (int z = 2; z <= nz - 1; z++)                 /* :108 */
        for (int y = 0; y < nyt; y++)
            for (int x = 0; x < nxt; x++) {
                size_t q = x + (size_t)ldx * y;
                dfdz[q + pl * z] = cst * (fun[q + pl * z] - fun[q + pl * (z - 1)]);
            }
    /* levels 1 and nz are left untouched (set by the wall stress routines) */
}

void orc_ddz_w(const orc_grid *g, double *dfdz, const double *fun)
{
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, nz = g->nz;
    size_t pl = (size_t)ldx * nyt;
    const double cst = 1.0 / g->dz;
    for (int z = 0; z <= nz - 1; z++) /* :169 */
        for (int y = 0; y < nyt; y++)
            for (int x = 0; x < nxt; x++) {
                size_t q = x + (size_t)ldx * y;
                dfdz[q + pl * z] = cst * (fun[q + pl * (z + 1)] - fun[q + pl * z]);
            }
    for (size_t q = 0; q < pl; q++) dfdz[q] = BOGUS;            /* :171-174 */
    for (size_t q = 0; q < pl; q++) dfdz[q + pl * nz] = 0.0;    /* :176-177 */
}

/* ------------------------------------------------------------------------- */
/* stress divergence (107_divstress.f90:4-104), single rank (coordz == 0 ==    */
/* npz-1): the three derivative arrays in full, then the level-by-level sum     */
/* ------------------------------------------------------------------------- */
static void divstress(const orc_grid *g, double *divt, const double *tx, const double *ty,
                      const double *tz, int w_form)
{
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, nz = g->nz;
    size_t pl = (size_t)ldx * nyt, n = pl * (size_t)(nz + 1);
    double *dx = (double *)calloc(n, sizeof(double));
    double *dy = (double *)calloc(n, sizeof(double));
    double *dz = (double *)calloc(n, sizeof(double));
    orc_ddx(g, dx, tx, nz + 1);                    /* :21, :67 */
    orc_ddy(g, dy, ty, nz + 1);                    /* :24, :71 */
    if (w_form) orc_ddz_uv(g, dz, tz);             /* :76: levels 2..nz-1 */
    else orc_ddz_w(g, dz, tz);                     /* :27: levels 0..nz-1 */
    int top = w_form ? nz : nz - 1;
    for (int z = 1; z <= top; z++)
        for (int y = 0; y < nyt; y++) {
            size_t r = (size_t)ldx * y + pl * z;
            for (int x = 0; x < nxt; x++) {
                double v = dx[r + x] + dy[r + x];
                /* uv: :36-37; w: the wall level (coordz == 0, :85) and the top level
                   (coordz == npz-1, :98) take no vertical term, :91-92 the rest */
                if (!w_form || (z >= 2 && z <= nz - 1)) v += dz[r + x];
                divt[r + x] = v;
            }
            divt[r + nxt] = 0.0;                   /* :40, :95, :99 */
            divt[r + nxt + 1] = 0.0;
        }
    for (size_t q = 0; q < pl; q++) divt[q] = BOGUS;                 /* :41, :79 */
    if (!w_form)
        for (size_t q = 0; q < pl; q++) divt[q + pl * nz] = BOGUS;   /* :42 */
    free(dx);
    free(dy);
    free(dz);
}

void orc_divstress_uv(const orc_grid *g, double *divt, const double *tx, const double *ty, const double *tz)
{
    divstress(g, divt, tx, ty, tz, 0);
}

void orc_divstress_w(const orc_grid *g, double *divt, const double *tx, const double *ty, const double *tz)
{
    divstress(g, divt, tx, ty, tz, 1);
}

/* ------------------------------------------------------------------------- */
/* 2D transforms (203_fftn_mpi.f90:4-67), npy = 1                              */
/* ------------------------------------------------------------------------- */
void orc_fftn(const orc_grid *g, const double *in, cplx *out)
{
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, lhx = g->lhx;
    cplx *hx = (cplx *)malloc(sizeof(cplx) * (size_t)lhx * nyt);
    cplx *col = (cplx *)malloc(sizeof(cplx) * (size_t)nyt * 2);
    for (int j = 0; j < nyt; j++) orc_fft_r2c(nxt, in + (size_t)j * ldx, hx + (size_t)j * lhx); /* :21-23 */
    for (int j = 0; j < nyt; j++) hx[(lhx - 1) + (size_t)lhx * j] = 0; /* :25 */
    for (int i = 0; i < lhx; i++) {                                    /* :29-31 */
        for (int j = 0; j < nyt; j++) col[j] = hx[i + (size_t)lhx * j];
        orc_fft_c2c(nyt, col, col + nyt, -1);
        for (int j = 0; j < nyt; j++) out[i + (size_t)lhx * j] = col[nyt + j];
    }
    for (int i = 0; i < lhx; i++) out[i + (size_t)lhx * (nyt / 2)] = 0; /* :33 */
    free(hx);
    free(col);
}

void orc_ifftn(const orc_grid *g, const cplx *in, double *out)
{
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, lhx = g->lhx;
    cplx *hx = (cplx *)malloc(sizeof(cplx) * (size_t)lhx * nyt);
    cplx *col = (cplx *)malloc(sizeof(cplx) * (size_t)nyt * 2);
    for (int i = 0; i < lhx; i++) { /* :57-59 */
        for (int j = 0; j < nyt; j++) col[j] = in[i + (size_t)lhx * j];
        orc_fft_c2c(nyt, col, col + nyt, +1);
        for (int j = 0; j < nyt; j++) hx[i + (size_t)lhx * j] = col[nyt + j];
    }
    for (int j = 0; j < nyt; j++) orc_fft_c2r(nxt, hx + (size_t)j * lhx, out + (size_t)j * ldx); /* :63-65 */
    free(hx);
    free(col);
}

/* ------------------------------------------------------------------------- */
/* 3/2-rule padding (108_01_padd.f90:73-197), npy = 1                          */
/* ------------------------------------------------------------------------- */
void orc_zero_padding(const orc_grid *g, const double *var, double *var_big)
{
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, nxt2 = g->nxt2, nyt2 = g->nyt2;
    int lhx = g->lhx, lhx2 = g->lhx2, lhy = g->lhy, lhy2 = g->lhy2;
    double *t = (double *)malloc(sizeof(double) * (size_t)(nxt2 > nyt2 ? nxt2 : nyt2) * 2);
    cplx *h = (cplx *)malloc(sizeof(cplx) * (size_t)(lhx2 > lhy2 ? lhx2 : lhy2) * 2);
    double *xbig = (double *)malloc(sizeof(double) * (size_t)nxt2 * nyt); /* var_x_big */
    for (int j = 0; j < nyt; j++) {
        for (int x = 0; x < nxt; x++) t[x] = var[x + (size_t)ldx * j] / nxt; /* :100 */
        orc_fft_r2c(nxt, t, h);                                              /* :102-104 */
        cplx *hb = h + lhx;
        for (int k = 0; k < lhx2; k++) hb[k] = 0; /* :97 */
        for (int k = 0; k < nxt / 2; k++) hb[k] = h[k]; /* :106-108 */
        orc_fft_c2r(nxt2, hb, xbig + (size_t)nxt2 * j); /* :110-112 */
    }
    (void)lhy;
    for (int x = 0; x < nxt2; x++) { /* :114-127, transposes are copies */
        for (int y = 0; y < nyt; y++) t[y] = xbig[x + (size_t)nxt2 * y] / nyt; /* :116 */
        orc_fft_r2c(nyt, t, h);
        cplx *hb = h + lhy2;
        for (int k = 0; k < lhy2; k++) hb[k] = 0; /* :98 */
        for (int k = 0; k < nyt / 2; k++) hb[k] = h[k]; /* :121-123 */
        orc_fft_c2r(nyt2, hb, t + nyt2);
        for (int y = 0; y < nyt2; y++) var_big[x + (size_t)nxt2 * y] = t[nyt2 + y];
    }
    free(t);
    free(h);
    free(xbig);
}

void orc_zero_unpadding(const orc_grid *g, const double *var_big, double *var)
{
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, nxt2 = g->nxt2, nyt2 = g->nyt2;
    int lhx = g->lhx, lhx2 = g->lhx2, lhy = g->lhy, lhy2 = g->lhy2;
    double *t = (double *)malloc(sizeof(double) * (size_t)(nxt2 > nyt2 ? nxt2 : nyt2) * 2);
    cplx *h = (cplx *)malloc(sizeof(cplx) * (size_t)(lhx2 > lhy2 ? lhx2 : lhy2) * 2);
    double *xs = (double *)malloc(sizeof(double) * (size_t)nxt * nyt2); /* var_x */
    for (int j = 0; j < nyt2; j++) {
        for (int x = 0; x < nxt2; x++) t[x] = var_big[x + (size_t)nxt2 * j] / nxt2; /* :161 */
        orc_fft_r2c(nxt2, t, h);                                                   /* :163-165 */
        cplx *hs = h + lhx2;
        for (int k = 0; k < nxt / 2; k++) hs[k] = h[k]; /* :167-169 */
        hs[nxt / 2] = 0;                                 /* :170 */
        (void)lhx;
        orc_fft_c2r(nxt, hs, xs + (size_t)nxt * j); /* :172-174 */
    }
    for (int x = 0; x < nxt; x++) { /* :176-192 */
        for (int y = 0; y < nyt2; y++) t[y] = xs[x + (size_t)nxt * y] / nyt2; /* :178 */
        orc_fft_r2c(nyt2, t, h);
        cplx *hs = h + lhy2;
        for (int k = 0; k < nyt / 2; k++) hs[k] = h[k]; /* :183-185 */
        hs[nyt / 2] = 0;                                 /* :186 */
        (void)lhy;
        orc_fft_c2r(nyt, hs, t + nyt2);
        for (int y = 0; y < nyt; y++) var[x + (size_t)ldx * y] = t[nyt2 + y]; /* :194 */
    }
    for (int y = 0; y < nyt; y++) /* :195 var(nxt+1:ldx,:) = var(1:2,:) */
        for (int x = nxt; x < ldx; x++) var[x + (size_t)ldx * y] = var[(x - nxt) + (size_t)ldx * y];
    free(t);
    free(h);
    free(xs);
}

/* ------------------------------------------------------------------------- */
/* filter_data (006_test_filter.f90:82-105)                                    */
/* ------------------------------------------------------------------------- */
void orc_filter_data(const orc_grid *g, double *f, int nlev)
{
    int nyt = g->nyt, ldx = g->ldx, lhx = g->lhx;
    size_t pl = (size_t)ldx * nyt;
    const double cst = 1.0 / ((double)g->nxt * (double)nyt); /* :98 */
#pragma omp parallel
    {
        cplx *tmp = (cplx *)malloc(sizeof(cplx) * (size_t)lhx * nyt);
#pragma omp for schedule(static)
        for (int z = 0; z < nlev; z++) {
            double *pz = f + pl * z;
            for (size_t q = 0; q < pl; q++) pz[q] = cst * pz[q]; /* :100 */
            orc_fftn(g, pz, tmp);                                  /* :101 */
            orc_ifftn(g, tmp, pz);                                 /* :102 */
        }
        free(tmp);
    }
}

/* ------------------------------------------------------------------------- */
/* pressure solve (109_press_stag_array.f90), emulating npz z-ranks            */
/* ------------------------------------------------------------------------- */
typedef struct {
    cplx *Hx, *Hy, *Hz;   /* (S, 0:nzl)   */
    cplx *rhs, *phat;     /* (S, 0:nzl)   (phat has one extra zero level for the */
                          /*  c(nz-1)*p_hat(nz) read on the top rank)            */
    double *ap, *bp, *cp; /* (S, 0:nzl-1) (ap/bp level 0 unused)                */
} rank_t;

int orc_press_stag_array(const orc_grid *g, int npz, const double *u,
                         const double *v, const double *w,
                         const double *divtz_bot, const double *divtz_top,
                         double *p, double *dpdx, double *dpdy)
{
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, lhx = g->lhx;
    int L = g->nzt - 1;
    if (npz < 1 || L % npz != 0 || L / npz < 2) return 1;
    int nzl = L / npz + 1;
    size_t S = (size_t)lhx * nyt;
    size_t pl = (size_t)ldx * nyt;
    double dz = g->dz, dt = g->dt_nd;
    const double cst = 1.0 / ((double)nxt * (double)nyt); /* :153 */

    double *kx = (double *)malloc(sizeof(double) * lhx);
    double *ky = (double *)malloc(sizeof(double) * g->lhy);
    double *kx2 = (double *)malloc(sizeof(double) * S);
    double *ky2 = (double *)malloc(sizeof(double) * S);
    double *k2 = (double *)malloc(sizeof(double) * S);
    int *nn = (int *)malloc(sizeof(int) * S);
    orc_wavenumbers(g, kx, ky, kx2, ky2, k2, nn);

    rank_t *R = (rank_t *)calloc((size_t)npz, sizeof(rank_t));
    for (int r = 0; r < npz; r++) {
        R[r].Hx = (cplx *)calloc(S * (nzl + 1), sizeof(cplx));
        R[r].Hy = (cplx *)calloc(S * (nzl + 1), sizeof(cplx));
        R[r].Hz = (cplx *)calloc(S * (nzl + 1), sizeof(cplx));
        R[r].rhs = (cplx *)calloc(S * (nzl + 1), sizeof(cplx));
        R[r].phat = (cplx *)calloc(S * (nzl + 1), sizeof(cplx));
        R[r].ap = (double *)calloc(S * nzl, sizeof(double));
        R[r].bp = (double *)calloc(S * nzl, sizeof(double));
        R[r].cp = (double *)calloc(S * nzl, sizeof(double));
    }

    /* (A) rH = const/tadv1*(u/dt) and fftn per level 1..nz-1 (:166-174) */
    const double sc = cst / TADV1;
    int nwork = npz * (nzl - 1);
#pragma omp parallel
    {
        double *rh = (double *)malloc(sizeof(double) * pl);
#pragma omp for schedule(dynamic)
        for (int it = 0; it < nwork * 3; it++) {
            int comp = it % 3, lw = it / 3;
            int r = lw / (nzl - 1), jz = 1 + lw % (nzl - 1);
            int G = r * (nzl - 1) + jz;
            const double *src = (comp == 0 ? u : comp == 1 ? v : w) + pl * G;
            for (size_t q = 0; q < pl; q++) rh[q] = sc * (src[q] / dt);
            cplx *dst = (comp == 0 ? R[r].Hx : comp == 1 ? R[r].Hy : R[r].Hz) + S * jz;
            orc_fftn(g, rh, dst);
        }
        free(rh);
    }
    /* (B) sendrecv H_z(1) down -> H_z(nz) of the rank below (:182-184) */
    for (int r = 0; r < npz - 1; r++) memcpy(R[r].Hz + S * nzl, R[r + 1].Hz + S * 1, S * sizeof(cplx));
    /* (C) boundary planes (:186-200); the theta/lbc==0 surface term is folded into
       divtz_bot by the caller */
    {
        double *rh = (double *)malloc(sizeof(double) * pl);
        for (size_t q = 0; q < pl; q++) rh[q] = cst * divtz_bot[q];
        orc_fftn(g, rh, R[0].Hz + 0); /* coordz == 0 */
        if (npz > 1) {                /* else if coordz == npz-1 */
            for (size_t q = 0; q < pl; q++) rh[q] = cst * divtz_top[q];
            orc_fftn(g, rh, R[npz - 1].Hz + S * nzl);
        }
        free(rh);
    }
    /* (D) RHS assembly (:203-225) */
    for (int r = 0; r < npz; r++) {
        rank_t *k = &R[r];
        int izs;
        if (r == 0) {
            for (size_t q = 0; q < S; q++) {
                if (k2[q] > 0)
                    k->rhs[q + S * 1] = I * (kx2[q] * k->Hx[q + S * 1] + ky2[q] * k->Hy[q + S * 1]) +
                                        ((k->Hz[q + S * 2] - k->Hz[q + S * 1]) + k->Hz[q]) / dz;
                k->rhs[q] = k->Hz[q];
            }
            izs = 2;
        } else {
            izs = 1;
        }
        for (int jz = izs; jz <= nzl - 1; jz++)
            for (size_t q = 0; q < S; q++) {
                if (k2[q] > 0)
                    k->rhs[q + S * jz] = I * (kx2[q] * k->Hx[q + S * jz] + ky2[q] * k->Hy[q + S * jz]) +
                                         (k->Hz[q + S * (jz + 1)] - k->Hz[q + S * jz]) / dz;
                if (k2[q] == 0 && nn[q]) k->rhs[q + S * jz] = k->Hz[q + S * jz];
            }
    }
    /* (E) init_coef_press (:4-68) + tdmaMcoef_pipelined (:72-103) */
    const double idz2 = 1.0 / (dz * dz), idz = 1.0 / dz;
    for (int r = 0; r < npz; r++) {
        rank_t *k = &R[r];
        int izs, ize;
        if (r == 0) {
            for (size_t q = 0; q < S; q++) {
                if (k2[q] > 0) {
                    k->ap[q + S] = 0;
                    k->bp[q + S] = -(k2[q] + idz2);
                    k->cp[q + S] = idz2;
                }
                if (k2[q] == 0 && nn[q]) {
                    k->ap[q + S] = 0;
                    k->bp[q + S] = idz;
                }
            }
            izs = 2;
            ize = nzl - 1;
        } else if (r == npz - 1) {
            size_t o = S * (nzl - 1);
            for (size_t q = 0; q < S; q++) {
                if (k2[q] > 0) {
                    k->ap[q + o] = idz2;
                    k->bp[q + o] = -(k2[q] + idz2);
                    k->cp[q + o] = 0;
                }
                if (k2[q] == 0 && nn[q]) {
                    k->ap[q + o] = -idz;
                    k->bp[q + o] = idz;
                }
            }
            izs = 1;
            ize = nzl - 2;
        } else {
            izs = 1;
            ize = nzl - 1;
        }
        for (int jz = izs; jz <= ize; jz++)
            for (size_t q = 0; q < S; q++) {
                size_t o = q + S * jz;
                if (k2[q] > 0) {
                    k->ap[o] = idz2;
                    k->bp[o] = -(k2[q] + 2.0 * idz2);
                    k->cp[o] = idz2;
                }
                if (k2[q] == 0 && nn[q]) {
                    k->ap[o] = -idz;
                    k->bp[o] = idz;
                }
            }
        if (r != 0) memcpy(k->cp, R[r - 1].cp + S * (nzl - 1), S * sizeof(double)); /* :84-87 */
        for (int iz = 1; iz <= nzl - 1; iz++)                                       /* :90-95 */
            for (size_t q = 0; q < S; q++)
                if (nn[q]) {
                    size_t o = q + S * iz;
                    k->bp[o] = k->bp[o] - k->ap[o] * k->cp[o - S];
                    k->cp[o] = k->cp[o] / k->bp[o];
                }
    }
    /* (F) forward sweep, pipelined across ranks (:260-277) */
    for (int r = 0; r < npz; r++) {
        rank_t *k = &R[r];
        if (r != 0) memcpy(k->rhs, R[r - 1].rhs + S * (nzl - 1), S * sizeof(cplx));
#pragma omp parallel for schedule(static)
        for (size_t q = 0; q < S; q++) {
            if (!nn[q]) continue;
            for (int iz = 1; iz <= nzl - 1; iz++) {
                size_t o = q + S * iz;
                k->rhs[o] = (k->rhs[o] - k->ap[o] * k->rhs[o - S]) / k->bp[o];
            }
        }
    }
    /* (G) backward sweep from the top rank down (:280-317) */
    for (int r = npz - 1; r >= 0; r--) {
        rank_t *k = &R[r];
        int izs, ize;
        if (r == 0) {
            izs = 1;
            ize = nzl - 2;
        } else if (r == npz - 1) {
            izs = 0;
            ize = nzl - 1;
        } else {
            izs = 0;
            ize = nzl - 2;
        }
        if (r != npz - 1)
            memcpy(k->phat + S * (nzl - 1), R[r + 1].phat, S * sizeof(cplx));
        else
            for (size_t q = 0; q < S; q++) k->phat[q + S * (nzl - 1)] = 0;
        /* p_hat(nz) (read only with c = 0 on the top rank) is the zero extra level */
#pragma omp parallel for schedule(static)
        for (size_t q = 0; q < S; q++) {
            for (int iz = ize; iz >= izs; iz--) {
                size_t o = q + S * iz;
                if (nn[q])
                    k->phat[o] = k->rhs[o] - k->cp[o] * k->phat[o + S];
                else
                    k->phat[o] = 0;
            }
            if (r == 0 && nn[q]) k->phat[q] = k->phat[q + S] - dz * k->rhs[q]; /* :313-315 */
        }
    }
    /* (H) inverse transforms (:231-238); ranks written bottom-up (overlap levels equal) */
    for (int r = 0; r < npz; r++) {
        rank_t *k = &R[r];
#pragma omp parallel
        {
            cplx *t = (cplx *)malloc(sizeof(cplx) * S);
#pragma omp for schedule(dynamic)
            for (int it = 0; it < 1 + 3 * (nzl - 1); it++) {
                if (it == 0) {
                    orc_ifftn(g, k->phat, p + pl * (size_t)(r * (nzl - 1)));
                    continue;
                }
                int jz = 1 + (it - 1) / 3, comp = (it - 1) % 3;
                int G = r * (nzl - 1) + jz;
                const cplx *ph = k->phat + S * jz;
                if (comp == 0) {
                    for (size_t q = 0; q < S; q++) t[q] = (I * kx2[q]) * ph[q];
                    orc_ifftn(g, t, dpdx + pl * (size_t)(G - 1));
                } else if (comp == 1) {
                    for (size_t q = 0; q < S; q++) t[q] = (I * ky2[q]) * ph[q];
                    orc_ifftn(g, t, dpdy + pl * (size_t)(G - 1));
                } else {
                    orc_ifftn(g, ph, p + pl * (size_t)G);
                }
            }
            free(t);
        }
    }

    for (int r = 0; r < npz; r++) {
        free(R[r].Hx);
        free(R[r].Hy);
        free(R[r].Hz);
        free(R[r].rhs);
        free(R[r].phat);
        free(R[r].ap);
        free(R[r].bp);
        free(R[r].cp);
    }
    free(R);
    free(kx);
    free(ky);
    free(kx2);
    free(ky2);
    free(k2);
    free(nn);
    return 0;
}

void orc_dpdz(const orc_grid *g, const double *p, double *dpdz)
{
    /* 103_flosol.f90:174-175 */
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, nz = g->nz;
    size_t pl = (size_t)ldx * nyt;
    for (int z = 1; z <= nz - 1; z++)
        for (int y = 0; y < nyt; y++)
            for (int x = 0; x < nxt; x++) {
                size_t q = x + (size_t)ldx * y;
                dpdz[q + pl * (z - 1)] = (p[q + pl * z] - p[q + pl * (z - 1)]) / g->dz;
            }
}

void orc_project(const orc_grid *g, double *u, double *v, double *w,
                 const double *dpdx, const double *dpdy, const double *dpdz)
{
    /* 110_project.f90:16-60; global arrays hold both the bottom (coordz == 0) and
       top (coordz == npz-1) ranks */
    int nxt = g->nxt, nyt = g->nyt, ldx = g->ldx, nz = g->nz;
    size_t pl = (size_t)ldx * nyt;
    double dt = g->dt_nd;
    for (int z = 1; z <= nz - 1; z++)
        for (int y = 0; y < nyt; y++)
            for (int x = 0; x < nxt; x++) {
                size_t q = x + (size_t)ldx * y;
                double rhs = -TADV1 * dpdx[q + pl * (z - 1)];
                u[q + pl * z] = u[q + pl * z] + dt * rhs;
                rhs = -TADV1 * dpdy[q + pl * (z - 1)];
                v[q + pl * z] = v[q + pl * z] + dt * rhs;
            }
    for (int z = 2; z <= nz - 1; z++) /* jz_min = 2 on the bottom rank */
        for (int y = 0; y < nyt; y++)
            for (int x = 0; x < nxt; x++) {
                size_t q = x + (size_t)ldx * y;
                double rhs = -TADV1 * dpdz[q + pl * (z - 1)];
                w[q + pl * z] = w[q + pl * z] + dt * rhs;
            }
    if (g->ubc_stress_free) {
        memcpy(u + pl * (nz - 1), u + pl * (nz - 2), pl * sizeof(double));
        memcpy(v + pl * (nz - 1), v + pl * (nz - 2), pl * sizeof(double));
    }
    for (size_t q = 0; q < pl; q++) w[q + pl * nz] = 0.0;
    for (size_t q = 0; q < pl; q++) w[q + pl * 1] = 0.0;
}

int orc_step(const orc_grid *g, int npz, double *u, double *v, double *w,
             const double *theta, double *const d[8], double *const big[4],
             double *p, double *const dp[3])
{
    int nlev = g->nz + 1;
    size_t pl = (size_t)g->ldx * g->nyt, plb = (size_t)g->nxt2 * g->nyt2;
    const double *f[4] = {u, v, w, theta};
    for (int c = 0; c < 4; c++) {
        orc_ddx(g, d[2 * c], f[c], nlev);
        orc_ddy(g, d[2 * c + 1], f[c], nlev);
    }
    for (int c = 0; c < 4; c++) {
#pragma omp parallel for schedule(static)
        for (int z = 0; z < nlev; z++) orc_zero_padding(g, f[c] + pl * z, big[c] + plb * z);
    }
    double *zero = (double *)calloc(pl, sizeof(double));
    int rc = orc_press_stag_array(g, npz, u, v, w, zero, zero, p, dp[0], dp[1]);
    free(zero);
    if (rc) return rc;
    orc_dpdz(g, p, dp[2]);
    orc_project(g, u, v, w, dp[0], dp[1], dp[2]);
    return 0;
}
