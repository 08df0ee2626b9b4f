// api.cu -- the C ABI of include/obl.h: context setup and every hot-path entry point.
//
// One context = one device, one stream, one grid.  It replaces the reference's
// init_parameter / init_fft_plan / init_wavenumber / init_coef_press (tables are built
// once: twiddles w_N^m in the storage precision, kx/ky wavenumbers in FP64, the FP64
// island list of the mixed mode) and owns the device work buffers.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include "common.cuh"
#include "lines.cuh"
#include "press.cuh"
#include "fused.cuh"
#include "convec.cuh"
#include "ensemble.cuh"
#include "slab.cuh"
#include "divstress.cuh"
#include "restart.cuh"

using namespace obl;

namespace {
constexpr double kPi = 3.1415926535897932384626433;   // 001_param.f90:32
constexpr double kTadv1 = 1.5;                         // 001_param.f90:152

struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
};
} // namespace

struct obl_ctx {
    int dev = 0;
    cudaStream_t stream = nullptr;
    obl_grid grid{};
    obl_options opt{};
    int nxt = 0, nyt = 0, nzt = 0, nz = 0, L = 0, lhx = 0, lhy = 0, ldx = 0, nxt2 = 0, nyt2 = 0;
    double lx = 0, ly = 0, dz = 0, dt_nd = 0;
    std::string err;
    Recorder rec;
    bool f64 = true;
    // tables
    double *d_kx = nullptr;    // kx(lhx), Nyquist 0
    double *d_ky1 = nullptr;   // ky(lhy), Nyquist 0 (1D, for ddy)
    double *d_ky2 = nullptr;   // ky_2d row (nyt), Nyquist row 0
    std::map<int, void *> tw;  // 4*n + role -> plan twiddle table in the storage precision
    // FP64 islands (mixed mode)
    int n_isl = 0;
    int *d_isl = nullptr;
    unsigned char *d_skip = nullptr;
    int *d_isl_slot = nullptr;   // column -> island index, -1 for the bulk (z-slab solve)
    int *d_ctl = nullptr;        // {work counter, error flag} of the staged solve (persistent kernel)
    // work buffers
    DevBuf spec[5];            // Hx, Hy, Hz, phat, dpdz spectrum (lhx*nyt*(nz+1) complex)
    DevBuf cscr;               // c' scratch
    DevBuf isl_c, isl_d;
    DevBuf tmp;                // pad/unpad intermediate, ifftn temporary
    DevBuf fscr;               // cluster scratch slots of the fused forward kernel
    // rollout problem of the adjoint: small (ldx,nyt,0:nz) and padded work fields, the
    // per-step state checkpoints and the objective's partial sums
    DevBuf rw_small[18];
    DevBuf rw_big[15];
    DevBuf ckpt;
    DevBuf ke;
    // z-slab solve: particular solution, spikes, modified upper band; bulk columns in the
    // storage type, FP64 island columns of the mixed mode apart
    DevBuf slab_v, slab_cp;
    IoStage io;                  // restart-file chunks (two device, two pinned host)
    DevBuf seg_iface;            // interface values of the segmented single-domain solve
    DevBuf slab_iy, slab_iv, slab_icp;
    // tuning parameters (obl_set_param)
    long long param_fused = 0;          // use the cluster-fused kernels in obl_step
    long long param_fwd_clusters = 16;  // clusters of the fused forward kernel (0 = all resident)
    long long param_fwd_csize = 8;      // CTAs per cluster
    long long param_tdma_segments = 0;  // column segments of the pressure solve (0 = by size, 1 = one sweep)
    long long param_fail_alloc = 0;     // > 0: the n-th later device allocation fails (failure-path tests)
    long long param_tdma_reg = 1;       // FP32 columns: register-segmented solve (1) or one sweep (0)
    long long param_tdma_stage = 2;     // the segmented solve fed by bulk asynchronous copies (1), by loads (0),
                                        // or (2) by copies above 128 levels (16 segments), where it is faster
    long long param_stage_timeout_test = 0;   // 1: the staged solve's waits expect bytes that never arrive
    long long param_pad_tma = 1;        // FP32 y-pad: input tiles by tensor-map copies (1) or by loads (0)
    long long param_isl_segments = 0;   // segments of each FP64 island column (0 = 16, capped at L/8; 1 = none)
    long long param_isl_concurrent = 0; // the island launches on a side stream, beside the bulk launch
                                        // (measured slower: the persistent bulk launch holds every SM)
    long long param_gform = 1;          // pressure RHS in G form: 1 with FP64 storage, 2 always, 0 never
    long long param_out_streams = 2;    // host step: device -> host copy streams (1 or 2)
    long long param_fwd_chunk = 0;      // forward pass in chunks of this many levels (0 = whole fields)
    // overlapped host step: input and output copy streams, per-field events
    cudaStream_t cin = nullptr, cout = nullptr, cout2 = nullptr;
    cudaEvent_t ev[9] = {};
    // side stream of the solve's FP64 island launches (forked from and joined to `stream`)
    cudaStream_t side = nullptr;
    cudaEvent_t side_ev[2] = {};
    std::vector<DevBuf> stage; // host-variant staging (storage type)
    std::vector<DevBuf> stage64;

    size_t es() const { return f64 ? 8 : 4; }
    long long plane() const { return (long long)ldx * nyt; }
    long long field() const { return plane() * (nz + 1); }
    long long dfield() const { return plane() * nz; }
    long long sp() const { return (long long)lhx * nyt; }
    long long big() const { return (long long)nxt2 * nyt2 * (nz + 1); }
};

// ----------------------------------------------------------------------------- helpers
namespace obl {
// readers of the index-check records of the translation units (bounds-checked build)
static std::vector<CheckReader> &check_readers()
{
    static std::vector<CheckReader> v;
    return v;
}
int check_register(CheckReader r)
{
    check_readers().push_back(r);
    return 0;
}
} // namespace obl
static int fail(obl_ctx *c, int code, const std::string &m)
{
    if (c) c->err = m;
    return code;
}
static int cuda_fail(obl_ctx *c, cudaError_t e, const char *where)
{
    return fail(c, OBL_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
// The error flag a bounded device-side wait raises (the staged pressure solve's wait for
// its copies), read once the context's work has drained; reported as OBL_ERR_TIMEOUT.
static int device_status(obl_ctx *c)
{
    if (!c->d_ctl) return OBL_OK;
    int flag = 0;
    const cudaError_t e = cudaMemcpy(&flag, c->d_ctl + 1, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(c, e, "device status");
    if (!flag) return OBL_OK;
    cudaMemset(c->d_ctl + 1, 0, sizeof(int));
    return fail(c, OBL_ERR_TIMEOUT, "a bounded wait for asynchronous copies (pressure solve or y-pad) gave up");
}
#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);                                   \
    } while (0)
#define CTX_OK()                                                                                   \
    do {                                                                                           \
        if (!ctx) return OBL_ERR_ARG;                                                              \
        cudaError_t e_ = cudaSetDevice(ctx->dev);                                                  \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, "cudaSetDevice");                         \
    } while (0)

// Every device allocation of a context goes through here.  The "fail_alloc" parameter
// (obl_set_param) or, for the allocations of obl_ctx_create, the OBL_FAIL_ALLOC
// environment variable makes the n-th allocation from then on fail as cudaMalloc would,
// so that the OBL_ERR_NOMEM paths can be tested on the host side; off (0) by default.
static cudaError_t dev_malloc(obl_ctx *ctx, void **p, size_t bytes)
{
    if (ctx && ctx->param_fail_alloc > 0 && --ctx->param_fail_alloc == 0) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}

static int ensure(obl_ctx *ctx, DevBuf &b, size_t bytes)
{
    if (b.n >= bytes) return OBL_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.n = 0;
    if (dev_malloc(ctx, &b.p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, OBL_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    b.n = bytes;
    return OBL_OK;
}

template <typename T> static const C2<T> *twt(obl_ctx *c, int n, int role)
{
    return (const C2<T> *)c->tw.at(4 * n + role);
}

static bool len_ok(int n) { return line_length_supported(n); }

// ----------------------------------------------------------------------------- typed ops
namespace {

template <typename T> struct Ops {
    obl_ctx *ctx;
    cudaStream_t s() const { return ctx->stream; }

    int chk(cudaError_t e, const char *w) { return e == cudaSuccess ? OBL_OK : cuda_fail(ctx, e, w); }

    int rows(int op, int n, const RowArgs<T> &a, const char *name)
    {
        LaunchScope ls(ctx->rec, name, s());
        return chk(launch_rows<T>(op, n, a, s()), name);
    }
    int cols(int op, bool real, int n, const ColArgs<T> &a, const char *name)
    {
        LaunchScope ls(ctx->rec, name, s());
        return chk(launch_cols<T>(op, real, n, a, s()), name);
    }

    // plan twiddle tables of the forward / backward transform of a line op of base length n
    void tables(int op, int n, const C2<T> *&f, const C2<T> *&b)
    {
        const int rf = op == OP_UNPAD ? ROLE_PADFWD : ROLE_FWD;
        const int rb = op == OP_PAD ? ROLE_PADBWD : ROLE_BWD;
        f = twt<T>(ctx, n, rf);
        b = twt<T>(ctx, n, rb);
    }
    RowArgs<T> rowargs(const void *src, long long ss, void *dst, long long ds, long long nrows, double scale,
                       int op, int n)
    {
        RowArgs<T> a{};
        a.src = src; a.dst = dst; a.src_stride = ss; a.dst_stride = ds; a.npairs = nrows / 2;
        a.scale = (T)scale; a.ktab = ctx->d_kx;
        tables(op, n, a.twF, a.twB);
        a.pad_scale = (T)1; a.pad_mode = 0;
        return a;
    }
    ColArgs<T> colargs(const void *src, long long srow, long long spl, void *dst, long long drow, long long dpl,
                       int ncols, int nlev, double scale, int op, int n)
    {
        ColArgs<T> a{};
        a.src = src; a.dst = dst; a.src_row = srow; a.dst_row = drow; a.src_plane = spl; a.dst_plane = dpl;
        a.ncols = ncols; a.nlev = nlev; a.scale = (T)scale; a.ktab = ctx->d_ky1;
        tables(op, n, a.twF, a.twB);
        a.pad_copy = 0; a.zero_nyq = 0; a.kmul = 0;
        return a;
    }

    // ---- ddx / ddy (004_derivatives.f90:18-81) ----
    int ddx(T *dfdx, const T *fun, int nlev)
    {
        auto a = rowargs(fun, ctx->ldx, dfdx, ctx->ldx, (long long)ctx->nyt * nlev, 1.0 / ctx->nxt, OP_DERIV, ctx->nxt);
        a.ktab = ctx->d_kx;
        return rows(OP_DERIV, ctx->nxt, a, "ddx_rows");
    }
    int ddy(T *dfdy, const T *fun, int nlev)
    {
        auto a = colargs(fun, ctx->ldx, ctx->plane(), dfdy, ctx->ldx, ctx->plane(), ctx->nxt, nlev,
                         1.0 / ctx->nyt, OP_DERIV, ctx->nyt);
        a.ktab = ctx->d_ky1;
        return cols(OP_DERIV, true, ctx->nyt, a, "ddy_cols");
    }

    // ---- zero_padding / zero_unpadding (108_01_padd.f90:73-197) ----
    int pad(const T *var, T *big, int nlev)
    {
        const int nx = ctx->nxt, ny = ctx->nyt, nx2 = ctx->nxt2, ny2 = ctx->nyt2;
        int rc = ensure(ctx, ctx->tmp, sizeof(T) * (size_t)nx2 * ny * nlev);
        if (rc) return rc;
        T *xb = (T *)ctx->tmp.p;  // var_x_big (nxt2, nyt, nlev)
        auto ra = rowargs(var, ctx->ldx, xb, nx2, (long long)ny * nlev, 1.0 / nx, OP_PAD, nx);
        if ((rc = rows(OP_PAD, nx, ra, "pad_rows"))) return rc;
        auto ca = colargs(xb, nx2, (long long)nx2 * ny, big, nx2, (long long)nx2 * ny2, nx2, nlev, 1.0 / ny, OP_PAD, ny);
        ca.tma = (int)ctx->param_pad_tma;
        ca.wait_err = ctx->d_ctl + 1;
        return cols(OP_PAD, true, ny, ca, "pad_cols");
    }
    // zero_padding through a caller-independent scratch plane xb (nxt2*nyt*nlev reals)
    // instead of the context's allocated buffer; used by obl_zero_padding_noalloc_dev
    int pad_with_scratch(const T *var, T *big, T *xb, int nlev)
    {
        const int nx = ctx->nxt, ny = ctx->nyt, nx2 = ctx->nxt2, ny2 = ctx->nyt2;
        auto ra = rowargs(var, ctx->ldx, xb, nx2, (long long)ny * nlev, 1.0 / nx, OP_PAD, nx);
        int rc = rows(OP_PAD, nx, ra, "pad_rows_noalloc");
        if (rc) return rc;
        auto ca = colargs(xb, nx2, (long long)nx2 * ny, big, nx2, (long long)nx2 * ny2, nx2, nlev, 1.0 / ny, OP_PAD, ny);
        return cols(OP_PAD, true, ny, ca, "pad_cols_noalloc");
    }
    int unpad(const T *big, T *var, int nlev)
    {
        const int nx = ctx->nxt, ny = ctx->nyt, nx2 = ctx->nxt2, ny2 = ctx->nyt2;
        int rc = ensure(ctx, ctx->tmp, sizeof(T) * (size_t)nx * ny2 * nlev);
        if (rc) return rc;
        T *xs = (T *)ctx->tmp.p;  // var_x (nxt, nyt2, nlev)
        auto ra = rowargs(big, nx2, xs, nx, (long long)ny2 * nlev, 1.0 / nx2, OP_UNPAD, nx);
        if ((rc = rows(OP_UNPAD, nx, ra, "unpad_rows"))) return rc;
        auto ca = colargs(xs, nx, (long long)nx * ny2, var, ctx->ldx, ctx->plane(), nx, nlev, 1.0 / ny2, OP_UNPAD, ny);
        ca.pad_copy = 1;
        return cols(OP_UNPAD, true, ny, ca, "unpad_cols");
    }

    // ---- several fields of one shape per launch (the rollout's convec and its transpose:
    // small grids whose single-field launches do not fill the GPU) ----
    int rows_multi(int op, int n, const RowArgs<T> &a, const MultiPtr<T> &m, int nf, const char *name)
    {
        LaunchScope ls(ctx->rec, name, s());
        return chk(launch_rows_multi<T>(op, n, a, m, nf, s()), name);
    }
    int cols_multi(int op, int n, const ColArgs<T> &a, const MultiPtr<T> &m, int nf, const char *name)
    {
        LaunchScope ls(ctx->rec, name, s());
        return chk(launch_cols_multi<T>(op, n, a, m, nf, s()), name);
    }
    int pad_multi(const T *const *src, T *const *big, int nf, int nlev)
    {
        const int nx = ctx->nxt, ny = ctx->nyt, nx2 = ctx->nxt2, ny2 = ctx->nyt2;
        const size_t xsz = (size_t)nx2 * ny * nlev;
        int rc = ensure(ctx, ctx->tmp, sizeof(T) * xsz * nf);
        if (rc) return rc;
        T *xb = (T *)ctx->tmp.p;
        MultiPtr<T> mr{}, mc{};
        for (int f = 0; f < nf; ++f) {
            mr.src[f] = src[f];
            mr.dst[f] = xb + f * xsz;
            mc.src[f] = xb + f * xsz;
            mc.dst[f] = big[f];
        }
        auto ra = rowargs(nullptr, ctx->ldx, nullptr, nx2, (long long)ny * nlev, 1.0 / nx, OP_PAD, nx);
        if ((rc = rows_multi(OP_PAD, nx, ra, mr, nf, "pad_rows"))) return rc;
        auto ca = colargs(nullptr, nx2, (long long)nx2 * ny, nullptr, nx2, (long long)nx2 * ny2, nx2, nlev, 1.0 / ny,
                          OP_PAD, ny);
        return cols_multi(OP_PAD, ny, ca, mc, nf, "pad_cols");
    }
    int unpad_multi(const T *const *big, T *const *var, int nf, int nlev)
    {
        const int nx = ctx->nxt, ny = ctx->nyt, nx2 = ctx->nxt2, ny2 = ctx->nyt2;
        const size_t xsz = (size_t)nx * ny2 * nlev;
        int rc = ensure(ctx, ctx->tmp, sizeof(T) * xsz * nf);
        if (rc) return rc;
        T *xs = (T *)ctx->tmp.p;
        MultiPtr<T> mr{}, mc{};
        for (int f = 0; f < nf; ++f) {
            mr.src[f] = big[f];
            mr.dst[f] = xs + f * xsz;
            mc.src[f] = xs + f * xsz;
            mc.dst[f] = var[f];
        }
        auto ra = rowargs(nullptr, nx2, nullptr, nx, (long long)ny2 * nlev, 1.0 / nx2, OP_UNPAD, nx);
        if ((rc = rows_multi(OP_UNPAD, nx, ra, mr, nf, "unpad_rows"))) return rc;
        auto ca = colargs(nullptr, nx, (long long)nx * ny2, nullptr, ctx->ldx, ctx->plane(), nx, nlev, 1.0 / ny2,
                          OP_UNPAD, ny);
        ca.pad_copy = 1;
        return cols_multi(OP_UNPAD, ny, ca, mc, nf, "unpad_cols");
    }
    int ddx_multi(T *const *out, const T *const *in, int nf, int nlev)
    {
        MultiPtr<T> m{};
        for (int f = 0; f < nf; ++f) {
            m.src[f] = in[f];
            m.dst[f] = out[f];
        }
        auto a = rowargs(nullptr, ctx->ldx, nullptr, ctx->ldx, (long long)ctx->nyt * nlev, 1.0 / ctx->nxt, OP_DERIV,
                         ctx->nxt);
        a.ktab = ctx->d_kx;
        return rows_multi(OP_DERIV, ctx->nxt, a, m, nf, "ddx_rows");
    }
    int ddy_multi(T *const *out, const T *const *in, int nf, int nlev)
    {
        MultiPtr<T> m{};
        for (int f = 0; f < nf; ++f) {
            m.src[f] = in[f];
            m.dst[f] = out[f];
        }
        auto a = colargs(nullptr, ctx->ldx, ctx->plane(), nullptr, ctx->ldx, ctx->plane(), ctx->nxt, nlev,
                         1.0 / ctx->nyt, OP_DERIV, ctx->nyt);
        a.ktab = ctx->d_ky1;
        return cols_multi(OP_DERIV, ctx->nyt, a, m, nf, "ddy_cols");
    }

    // ---- fftn / ifftn (203_fftn_mpi.f90:4-67) ----
    // real planes (ldx stride) -> complex planes (lhx stride), nlev planes
    int fftn(const T *in, C2<T> *out, int nlev, double scale)
    {
        auto ra = rowargs(in, ctx->ldx, out, ctx->lhx, (long long)ctx->nyt * nlev, scale, OP_FWD, ctx->nxt);
        int rc = rows(OP_FWD, ctx->nxt, ra, "fftn_rows");
        if (rc) return rc;
        auto ca = colargs(out, ctx->lhx, ctx->sp(), out, ctx->lhx, ctx->sp(), ctx->lhx, nlev, 1.0, OP_FWD, ctx->nyt);
        ca.zero_nyq = 1;
        return cols(OP_FWD, false, ctx->nyt, ca, "fftn_cols");
    }
    // complex planes -> real planes; tmp receives the y-inverse (may alias in when in is scratch)
    int ifftn(const C2<T> *in, C2<T> *tmp, T *out, long long out_plane_off_unused, int nlev, int kmul,
              T pad_scale = (T)1, int pad_mode = 0)
    {
        (void)out_plane_off_unused;
        auto ca = colargs(in, ctx->lhx, ctx->sp(), tmp, ctx->lhx, ctx->sp(), ctx->lhx, nlev, 1.0, OP_INV, ctx->nyt);
        ca.kmul = kmul;
        ca.ktab = kmul == 1 ? ctx->d_kx : ctx->d_ky2;
        int rc = cols(OP_INV, false, ctx->nyt, ca, "ifftn_cols");
        if (rc) return rc;
        auto ra = rowargs(tmp, ctx->lhx, out, ctx->ldx, (long long)ctx->nyt * nlev, 1.0, OP_INV, ctx->nxt);
        ra.pad_scale = pad_scale;
        ra.pad_mode = pad_mode;
        return rows(OP_INV, ctx->nxt, ra, "ifftn_rows");
    }

    int filter(T *f, int nlev)
    {
        int rc = ensure(ctx, ctx->tmp, sizeof(C2<T>) * (size_t)ctx->sp() * nlev);
        if (rc) return rc;
        C2<T> *sp = (C2<T> *)ctx->tmp.p;
        const double cst = 1.0 / ((double)ctx->nxt * ctx->nyt);   // 006_test_filter.f90:98
        if ((rc = fftn(f, sp, nlev, cst))) return rc;
        return ifftn(sp, sp, f, 0, nlev, 0, (T)cst, 1);
    }

    // ---- press_stag_array (109_press_stag_array.f90:107-240) ----
    // dpdz (optional): also return dpdz = ifftn((p_hat(z) - p_hat(z-1))/dz), the
    // spectral form of the flosol difference (103_flosol.f90:174-175), whose
    // z-difference is taken inside the solve in its own precision
    // rhs_ready: H_x, H_y, H_z at levels 1..L were already produced (by the fused
    // forward kernel); only the boundary planes H_z(0), H_z(nz) are transformed here.
    // proj: when given (with dpdz_out), the inverse is fused with project() on proj->u,v,w
    // stress_free: overrides the context's ubc_stress_free for that project() (-1: keep)
    int press(const T *u, const T *v, const T *w, const T *dbot, const T *dtop, T *p, T *dpdx, T *dpdy,
              T *dpdz_out = nullptr, bool rhs_ready = false, const obl_step_io *proj = nullptr,
              int stress_free = -1)
    {
        const long long S = ctx->sp();
        const size_t sb = sizeof(C2<T>) * (size_t)S * (ctx->nz + 1);
        int rc;
        for (int i = 0; i < (dpdz_out ? 5 : 4); ++i)
            if ((rc = ensure(ctx, ctx->spec[i], sb))) return rc;
        if ((rc = ensure(ctx, ctx->cscr, sizeof(T) * (size_t)S * ctx->L))) return rc;
        C2<T> *Hx = (C2<T> *)ctx->spec[0].p, *Hy = (C2<T> *)ctx->spec[1].p, *Hz = (C2<T> *)ctx->spec[2].p,
              *ph = (C2<T> *)ctx->spec[3].p;
        const long long pl = ctx->plane();
        const int L = ctx->L, nx = ctx->nxt, ny = ctx->nyt, lhx = ctx->lhx, ldx = ctx->ldx;
        const double cst = 1.0 / ((double)nx * ny);               // :153
        const double sc = (cst / kTadv1) * (1.0 / ctx->dt_nd);     // rH = const/tadv1*(u/dt) (:166-168)

        // x r2c of levels 1..L of u, v, w straight into the spectral buffers (one launch)
        if (!rhs_ready) {
            MultiPtr<T> m{};
            m.src[0] = u + pl; m.src[1] = v + pl; m.src[2] = w + pl;
            m.dst[0] = Hx + S; m.dst[1] = Hy + S; m.dst[2] = Hz + S;
            auto ra = rowargs(nullptr, ldx, nullptr, lhx, (long long)ny * L, sc, OP_FWD, nx);
            if ((rc = rows_multi(OP_FWD, nx, ra, m, 3, "press_fwd_rows"))) return rc;
        }
        // boundary planes H_z(0) and H_z(nz) (:186-200)
        if (dbot) {
            auto ra = rowargs(dbot, ldx, Hz, lhx, ny, cst, OP_FWD, nx);
            if ((rc = rows(OP_FWD, nx, ra, "press_fwd_rows"))) return rc;
        } else {
            CK(cudaMemsetAsync(Hz, 0, sizeof(C2<T>) * S, s()));
        }
        if (ctx->opt.top_bc == OBL_TOP_NEUMANN && dtop) {
            auto ra = rowargs(dtop, ldx, Hz + S * (L + 1), lhx, ny, cst, OP_FWD, nx);
            if ((rc = rows(OP_FWD, nx, ra, "press_fwd_rows"))) return rc;
        } else {
            CK(cudaMemsetAsync(Hz + S * (L + 1), 0, sizeof(C2<T>) * S, s()));
        }
        // y c2c (in place), y-Nyquist zeroed
        const bool gf = rhs_ready ? fwd_gform : gform(dpdz_out != nullptr);
        if (gf) {
            // H_y as it is; G = i*kx*H_x + (H_z(z+1) - H_z(z) [+ H_z(0)])/dz formed from the
            // x-spectra and transformed over H_x; H_z at level 0, and at levels 1..L only in
            // the line group of kx = 0 (the (0,0) mode's RHS, the same transform as before)
            if (!rhs_ready) {
                auto ca = colargs(Hy + S, lhx, S, Hy + S, lhx, S, lhx, L, 1.0, OP_FWD, ny);
                ca.zero_nyq = 1;
                if ((rc = cols(OP_FWD, false, ny, ca, "press_fwd_cols"))) return rc;
            }
            {
                LaunchScope ls(ctx->rec, "press_gform_cols", s());
                if ((rc = chk(launch_gform_cols<T>(ny, Hx, Hz, ctx->d_kx, S, lhx, L, ctx->dz, twt<T>(ctx, ny, ROLE_FWD),
                                                   s()),
                              "press_gform_cols")))
                    return rc;
            }
            auto ca = colargs(Hz, lhx, S, Hz, lhx, S, lhx, 1, 1.0, OP_FWD, ny);
            ca.zero_nyq = 1;
            if ((rc = cols(OP_FWD, false, ny, ca, "press_bnd_cols"))) return rc;
            auto c0 = colargs(Hz + S, lhx, S, Hz + S, lhx, S, 1, L, 1.0, OP_FWD, ny);   // column kx = 0
            c0.zero_nyq = 1;
            if ((rc = cols(OP_FWD, false, ny, c0, "press_mean_cols"))) return rc;
        } else if (!rhs_ready) {
            // H_x, H_y levels 1..L in one launch, H_z levels 0..L+1 in another
            MultiPtr<T> m{};
            m.src[0] = m.dst[0] = Hx + S;
            m.src[1] = m.dst[1] = Hy + S;
            auto ca = colargs(nullptr, lhx, S, nullptr, lhx, S, lhx, L, 1.0, OP_FWD, ny);
            ca.zero_nyq = 1;
            if ((rc = cols_multi(OP_FWD, ny, ca, m, 2, "press_fwd_cols"))) return rc;
            ca.src = ca.dst = Hz;
            ca.nlev = L + 2;
            if ((rc = cols(OP_FWD, false, ny, ca, "press_fwd_cols"))) return rc;
        } else {
            for (int zb : {0, L + 1}) {
                auto ca = colargs(Hz + S * zb, lhx, S, Hz + S * zb, lhx, S, lhx, 1, 1.0, OP_FWD, ny);
                ca.zero_nyq = 1;
                if ((rc = cols(OP_FWD, false, ny, ca, "press_bnd_cols"))) return rc;
            }
        }
        // tridiagonal solve per (kx,ky) column
        TdmaArgs<T> ta{};
        ta.Hx = Hx; ta.Hy = Hy; ta.Hz = Hz; ta.phat = ph; ta.cscr = (T *)ctx->cscr.p;
        ta.kx = ctx->d_kx; ta.ky = ctx->d_ky2; ta.skip = ctx->n_isl ? ctx->d_skip : nullptr;
        ta.S = S; ta.lhx = lhx; ta.nyt = ny; ta.L = L; ta.dz = ctx->dz;
        ta.dph = dpdz_out ? (C2<T> *)ctx->spec[4].p : nullptr;
        ta.neumann_top = ctx->opt.top_bc == OBL_TOP_NEUMANN;
        ta.gform = gf ? 1 : 0;
        const int P = solve_parts(ta.dph != nullptr);
        if (P > 1) {
            // the columns split into segments solved at once (partitioned Thomas, as across
            // z-ranks), then the reduced interface system and the back substitution
            const int seg = (L + P - 1) / P, Pn = (L + seg - 1) / seg;
            const size_t n = (size_t)S * L, ni = (size_t)(ctx->n_isl > 0 ? ctx->n_isl : 1) * L;
            if ((rc = ensure(ctx, ctx->slab_v, sizeof(T) * n)) || (rc = ensure(ctx, ctx->slab_cp, sizeof(T) * n)) ||
                (rc = ensure(ctx, ctx->slab_iy, sizeof(double2) * ni)) ||
                (rc = ensure(ctx, ctx->slab_iv, sizeof(double) * ni)) ||
                (rc = ensure(ctx, ctx->slab_icp, sizeof(double) * ni)) ||
                (rc = ensure(ctx, ctx->seg_iface, sizeof(double) * kSlabIface * (size_t)S * Pn)))
                return rc;
            SlabArgs<T> a = slab_args(0, 1);
            a.Hx = Hx; a.Hy = Hy; a.Hz = Hz; a.phat = ph; a.dph = ta.dph;
            a.iface = (double *)ctx->seg_iface.p;
            a.iface_all = a.iface;
            cudaError_t e = cudaSuccess;
            {
                LaunchScope ls(ctx->rec, "tdma_seg_solve", s());
                launch_seg_solve<T>(a, Pn, seg, s(), e);
            }
            {
                LaunchScope ls(ctx->rec, "tdma_seg_finish", s());
                launch_seg_finish<T>(a, Pn, seg, s(), e);
            }
            if (e != cudaSuccess) return cuda_fail(ctx, e, "tdma_seg");
        } else {
            cudaError_t e = cudaSuccess;
            bool done = false;
            if constexpr (std::is_same<T, float>::value) {
                if (ctx->param_tdma_reg && tdma_reg_supported(L)) {
                    // FP32 bulk columns by the register-segmented solve; FP64 islands either
                    // split into segments by the column-segmented FP64 solve (two small
                    // launches first: one thread sweeping all L levels of an island column
                    // took longer than the whole bulk), or by their sequential sweep inside
                    // the bulk launch
                    IslandArgs isl{nullptr, 0, nullptr, nullptr};
                    bool join_side = false;   // the island launches ran on the side stream
                    const int ip = isl_parts(ta);
                    if (ip > 1) {
                        const int seg = (L + ip - 1) / ip, Pn = (L + seg - 1) / seg;
                        const size_t ni = (size_t)ctx->n_isl * L;
                        if ((rc = ensure(ctx, ctx->slab_iy, sizeof(double2) * ni)) ||
                            (rc = ensure(ctx, ctx->slab_iv, sizeof(double) * ni)) ||
                            (rc = ensure(ctx, ctx->slab_icp, sizeof(double) * ni)) ||
                            (rc = ensure(ctx, ctx->seg_iface, sizeof(double) * kSlabIface * (size_t)S * Pn)))
                            return rc;
                        SlabArgs<T> sa = slab_args(0, 1);
                        sa.Hx = Hx; sa.Hy = Hy; sa.Hz = Hz; sa.phat = ph; sa.dph = ta.dph;
                        sa.v = nullptr; sa.cp = nullptr;   // bulk scratch: the island launches do not touch it
                        sa.iface = (double *)ctx->seg_iface.p;
                        sa.iface_all = sa.iface;
                        // on a side stream the island launches can run beside the bulk launch
                        // (on the SMs they hold when it starts; its units go to the others)
                        cudaStream_t is = s();
                        if (ctx->param_isl_concurrent) {
                            if (!ctx->side) {
                                CK(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
                                for (auto &ev : ctx->side_ev) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
                            }
                            CK(cudaEventRecord(ctx->side_ev[0], s()));
                            CK(cudaStreamWaitEvent(ctx->side, ctx->side_ev[0], 0));
                            is = ctx->side;
                        }
                        {
                            LaunchScope ls(ctx->rec, "tdma_isl_solve", is);
                            launch_seg_solve_isl<T>(sa, Pn, seg, is, e);
                        }
                        {
                            LaunchScope ls(ctx->rec, "tdma_isl_finish", is);
                            launch_seg_finish_isl<T>(sa, Pn, seg, is, e);
                        }
                        if (e != cudaSuccess) return cuda_fail(ctx, e, "tdma_isl");
                        if (is != s()) {
                            CK(cudaEventRecord(ctx->side_ev[1], is));
                            join_side = true;
                        }
                    } else if (ctx->n_isl) {
                        if ((rc = ensure(ctx, ctx->isl_c, sizeof(double) * (size_t)ctx->n_isl * L))) return rc;
                        if ((rc = ensure(ctx, ctx->isl_d, sizeof(double2) * (size_t)ctx->n_isl * (L + 1)))) return rc;
                        isl = IslandArgs{ctx->d_isl, ctx->n_isl, (double *)ctx->isl_c.p, (double2 *)ctx->isl_d.p};
                    }
                    const bool stage = ctx->param_tdma_stage == 1 || (ctx->param_tdma_stage == 2 && L > 128);
                    if (stage && tdma_staged_supported(ta)) {
                        LaunchScope ls(ctx->rec, "tdma_staged", s());
                        launch_tdma_staged(ta, isl, ctx->d_ctl, ctx->param_stage_timeout_test ? 16u : 0u, s(), e);
                        if (e != cudaSuccess) return cuda_fail(ctx, e, "tdma_staged");
                    } else {
                        LaunchScope ls(ctx->rec, "tdma_reg", s());
                        launch_tdma_reg<float>(ta, isl, s(), e);
                        if (e != cudaSuccess) return cuda_fail(ctx, e, "tdma_reg");
                    }
                    if (join_side) CK(cudaStreamWaitEvent(s(), ctx->side_ev[1], 0));
                    done = true;
                }
            }
            if (done) {
            } else if (ctx->n_isl) {
                // FP32 bulk and FP64 island columns in one launch
                if ((rc = ensure(ctx, ctx->isl_c, sizeof(double) * (size_t)ctx->n_isl * L))) return rc;
                if ((rc = ensure(ctx, ctx->isl_d, sizeof(double2) * (size_t)ctx->n_isl * (L + 1)))) return rc;
                IslandArgs isl{ctx->d_isl, ctx->n_isl, (double *)ctx->isl_c.p, (double2 *)ctx->isl_d.p};
                LaunchScope ls(ctx->rec, "tdma_mixed", s());
                launch_tdma_island<T>(ta, isl, s(), e);
                if (e != cudaSuccess) return cuda_fail(ctx, e, "tdma_mixed");
            } else {
                LaunchScope ls(ctx->rec, "tdma", s());
                launch_tdma<T>(ta, s(), e);
                if (e != cudaSuccess) return cuda_fail(ctx, e, "tdma");
            }
        }
        if (proj && dpdz_out) {
            // fused inverse + project: one y-inverse pass over p_hat and the dpdz spectrum,
            // one x-inverse pass over the rows that also applies project()
            PinvColArgs<T> pc{};
            pc.ph = ph; pc.dph = (const C2<T> *)ctx->spec[4].p;
            pc.Xp = Hz; pc.Xdy = Hy; pc.Xdz = (C2<T> *)ctx->spec[4].p;
            pc.S = S; pc.lhx = lhx; pc.kx = ctx->d_kx; pc.ky = ctx->d_ky2;
            pc.twB = twt<T>(ctx, ny, ROLE_BWD);
            {
                LaunchScope ls(ctx->rec, "pinv_cols", s());
                if ((rc = chk(PinvLaunch<T>::cols(ny, pc, L + 1, s()), "pinv_cols"))) return rc;
            }
            PinvRowArgs<T> pr{};
            pr.Xp = Hz; pr.kx = ctx->d_kx; pr.Xdy = Hy; pr.Xdz = (const C2<T> *)ctx->spec[4].p;
            pr.p = p; pr.dpdx = dpdx; pr.dpdy = dpdy; pr.dpdz = dpdz_out;
            pr.u = (T *)proj->u; pr.v = (T *)proj->v; pr.w = (T *)proj->w;
            pr.npairs = (long long)ny * (L + 1) / 2;
            pr.ldx = ldx; pr.ny = ny; pr.lhx = lhx;
            pr.dt_tadv1 = (T)(ctx->dt_nd * kTadv1);
            pr.twB = twt<T>(ctx, nx, ROLE_BWD);
            {
                LaunchScope ls(ctx->rec, "pinv_rows_project", s());
                if ((rc = chk(PinvLaunch<T>::rows(nx, pr, s()), "pinv_rows_project"))) return rc;
            }
            cudaError_t e = cudaSuccess;
            LaunchScope ls(ctx->rec, "project_bc", s());
            launch_project_bc<T>((T *)proj->u, (T *)proj->v, (T *)proj->w, ldx, ny, ctx->nz,
                                 stress_free < 0 ? (int)ctx->opt.ubc_stress_free : stress_free, s(), e);
            return chk(e, "project_bc");
        }
        // inverse transforms (:231-238): p at 0..L, dpdx/dpdy at 1..L; Hx/Hy/Hz are
        // free now and hold the y-inverses
        if ((rc = ifftn(ph, Hz, p, 0, L + 1, 0))) return rc;
        if ((rc = ifftn(ph + S, Hx, dpdx, 0, L, 1))) return rc;
        if ((rc = ifftn(ph + S, Hy, dpdy, 0, L, 2))) return rc;
        if (dpdz_out) {
            C2<T> *dph = (C2<T> *)ctx->spec[4].p + S;
            if ((rc = ifftn(dph, dph, dpdz_out, 0, L, 0))) return rc;
        }
        return OBL_OK;
    }

    int dpdz(const T *p, T *dp)
    {
        cudaError_t e = cudaSuccess;
        LaunchScope ls(ctx->rec, "dpdz", s());
        launch_dpdz<T>(dp, p, ctx->nxt, ctx->ldx, ctx->nyt, ctx->nz, ctx->dz, s(), e);
        return chk(e, "dpdz");
    }
    int project(T *u, T *v, T *w, const T *dpdx, const T *dpdy, const T *dpdz_)
    {
        cudaError_t e = cudaSuccess;
        LaunchScope ls(ctx->rec, "project", s());
        ctx->rec.launches += 1;   // project + boundary kernel
        launch_project<T>(u, v, w, dpdx, dpdy, dpdz_, ctx->nxt, ctx->ldx, ctx->nyt, ctx->nz, ctx->dt_nd,
                          ctx->opt.ubc_stress_free, s(), e);
        return chk(e, "project");
    }
    int ddz_uv(T *d, const T *f)
    {
        cudaError_t e = cudaSuccess;
        LaunchScope ls(ctx->rec, "ddz_uv", s());
        launch_ddz_uv<T>(d, f, ctx->nxt, ctx->ldx, ctx->nyt, ctx->nz, ctx->dz, s(), e);
        return chk(e, "ddz_uv");
    }
    int ddz_w(T *d, const T *f)
    {
        cudaError_t e = cudaSuccess;
        LaunchScope ls(ctx->rec, "ddz_w", s());
        launch_ddz_w<T>(d, f, ctx->nxt, ctx->ldx, ctx->nyt, ctx->nz, ctx->dz, s(), e);
        return chk(e, "ddz_w");
    }

    // ---- restart files (202_parallel.f90:1084-1250): levels 1..nz-1 of one field ----
    int io_reserve()
    {
        const size_t plane = (size_t)ctx->nxt * ctx->nyt, chunk = (size_t)8 << 20;   // 64 MiB of doubles
        if (ctx->param_fail_alloc > 0 && --ctx->param_fail_alloc == 0)
            return fail(ctx, OBL_ERR_NOMEM, "restart staging: allocation failed");
        return io_stage_reserve(ctx->io, chunk > plane ? chunk : plane, ctx->err);
    }
    int write_field(const T *var, int fd, long long off)
    {
        int rc = io_reserve();
        return rc ? rc : io_write_field<T>(ctx->io, s(), fd, off, var, ctx->nxt, ctx->ldx, ctx->nyt, ctx->nz, ctx->err);
    }
    int read_field(T *var, int fd, long long off)
    {
        int rc = io_reserve();
        return rc ? rc : io_read_field<T>(ctx->io, s(), fd, off, var, ctx->nxt, ctx->ldx, ctx->nyt, ctx->nz, ctx->err);
    }

    // ---- divstress_uv / divstress_w (107_divstress.f90:4-104), single-rank roles ----
    // ddx(tx) into divt's computed levels, then the ddy(ty) column pass whose stores add
    // it, the vertical difference of tz and the zero pads; BOGUS on the other levels.
    // bottom / top: the rank holds the wall / the top of the domain (coordz == 0 /
    // coordz == npz-1); a whole domain holds both
    int divstress(T *divt, const T *tx, const T *ty, const T *tz, bool w_form, bool bottom = true, bool top = true)
    {
        const int nz = ctx->nz, nlev = (w_form && top) ? nz : nz - 1;   // levels 1..nlev
        const long long pl = ctx->plane();
        auto ra = rowargs(tx + pl, ctx->ldx, divt + pl, ctx->ldx, (long long)ctx->nyt * nlev, 1.0 / ctx->nxt,
                          OP_DERIV, ctx->nxt);
        ra.ktab = ctx->d_kx;
        int rc = rows(OP_DERIV, ctx->nxt, ra, "divt_ddx_rows");
        if (rc) return rc;
        auto ca = colargs(ty + pl, ctx->ldx, pl, divt + pl, ctx->ldx, pl, ctx->nxt, nlev, 1.0 / ctx->nyt, OP_DERIV,
                          ctx->nyt);
        ca.ktab = ctx->d_ky1;
        DivEpi<T> ep{};
        ep.out = divt + pl;
        ep.tz = tz + pl;
        ep.row = ctx->ldx;
        ep.plane = pl;
        ep.ncols = ctx->nxt;
        ep.rdz = (T)(1.0 / ctx->dz);
        ep.fwd = w_form ? 0 : 1;
        ep.zlo = (w_form && bottom) ? 1 : 0;  // divstress_w: no dz(tzz) on the wall level (:81-88)
        ep.zhi = w_form ? nz - 2 : nlev - 1;  // ... nor on the top level (:97-98)
        {
            LaunchScope ls(ctx->rec, "divt_ddy_cols", s());
            if ((rc = chk(launch_cols_divt<T>(ctx->nyt, ca, ep, s()), "divt_ddy_cols"))) return rc;
        }
        cudaError_t e = cudaSuccess;
        LaunchScope ls(ctx->rec, "divt_bogus", s());
        launch_fill<T>(divt, pl, (T)-1234567890.0, s(), e);   // BOGUS, 001_param.f90:40
        if (!w_form || !top) launch_fill<T>(divt + pl * nz, pl, (T)-1234567890.0, s(), e);   // :42, :101
        return chk(e, "divt_bogus");
    }

    // ---- the fused step ----
    // cluster-fused forward pass over all (field, level) planes: ddx, ddy, zero_padding of
    // u, v, w, theta and the RHS spectra H_x, H_y, H_z of levels 1..L
    int fwd_fused(const obl_step_io *io)
    {
        const long long S = ctx->sp();
        const size_t sb = sizeof(C2<T>) * (size_t)S * (ctx->nz + 1);
        int rc;
        for (int i = 0; i < 5; ++i)
            if ((rc = ensure(ctx, ctx->spec[i], sb))) return rc;
        const int n = ctx->nxt, csize = (int)ctx->param_fwd_csize;
        int ncl = (int)ctx->param_fwd_clusters;
        const int maxc = FwdFusedLaunch<T>::max_clusters(n, csize);
        if (maxc <= 0) return fail(ctx, OBL_ERR_UNSUPPORTED, "fused forward kernel cannot be resident");
        if (ncl <= 0 || ncl > maxc) ncl = maxc;
        const int nitems = 4 * (ctx->nz + 1);
        if (ncl > nitems) ncl = nitems;
        const size_t slot = FwdFusedLaunch<T>::slot_bytes(n);
        if ((rc = ensure(ctx, ctx->fscr, slot * (size_t)ncl))) return rc;
        FwdFusedArgs<T> a{};
        for (int c = 0; c < 4; ++c) {
            a.f[c] = c == 0 ? (const T *)io->u : c == 1 ? (const T *)io->v : c == 2 ? (const T *)io->w
                                                                             : (const T *)io->theta;
            a.big[c] = (T *)io->big[c];
        }
        for (int i = 0; i < 8; ++i) a.d[i] = (T *)io->d[i];
        for (int c = 0; c < 3; ++c) a.H[c] = (C2<T> *)ctx->spec[c].p;
        a.scr = (unsigned char *)ctx->fscr.p;
        a.slot_bytes = (long long)slot;
        a.ldx = ctx->ldx;
        a.nlev = ctx->nz + 1;
        a.L = ctx->L;
        a.nfields = 4;
        a.sc_press = ((1.0 / ((double)ctx->nxt * ctx->nyt)) / kTadv1) * (1.0 / ctx->dt_nd);
        a.kx = ctx->d_kx;
        a.ky = ctx->d_ky1;
        a.twF = twt<T>(ctx, n, ROLE_FWD);
        a.twB = twt<T>(ctx, n, ROLE_BWD);
        a.twPB = twt<T>(ctx, n, ROLE_PADBWD);
        LaunchScope ls(ctx->rec, "fwd_fused", s());
        return chk(FwdFusedLaunch<T>::run(n, a, ncl, csize, s()), "fwd_fused");
    }

    // line-kernel forward pass of the step: per field one multi-output row pass (ddx,
    // x-pad, RHS x-spectrum) and the column passes (y-pad, ddy, RHS y-transform)
    int fwd_lines(const obl_step_io *io)
    {
        int rc;
        if ((rc = fwd_prepare())) return rc;
        for (int c = 0; c < 4; ++c)
            if ((rc = fwd_field(io, c))) return rc;
        return OBL_OK;
    }
    int fwd_prepare()
    {
        const size_t sb = sizeof(C2<T>) * (size_t)ctx->sp() * (ctx->nz + 1);
        int rc;
        for (int i = 0; i < 5; ++i)
            if ((rc = ensure(ctx, ctx->spec[i], sb))) return rc;
        return ensure(ctx, ctx->tmp, sizeof(T) * (size_t)ctx->nxt2 * ctx->nyt * (ctx->nz + 1));
    }
    // field c (0..3 = u, v, w, theta) of the line-kernel forward pass; its outputs d[2c],
    // d[2c+1], big[c] are final when its kernels are done
    int fwd_field(const obl_step_io *io, int c)
    {
        const int nlev = ctx->nz + 1, nx = ctx->nxt, ny = ctx->nyt, nx2 = ctx->nxt2, ny2 = ctx->nyt2;
        const long long S = ctx->sp(), pl = ctx->plane(), plb = (long long)nx2 * ny2;
        int rc;
        T *xb = (T *)ctx->tmp.p;
        const T *f[4] = {(const T *)io->u, (const T *)io->v, (const T *)io->w, (const T *)io->theta};
        const double scp = ((1.0 / ((double)nx * ny)) / kTadv1) * (1.0 / ctx->dt_nd);
        C2<T> *H = c < 3 ? (C2<T> *)ctx->spec[c].p : nullptr;
        // chunks of levels (fwd_chunk): the chunk's x-padded planes reuse the start of the
        // intermediate and the field rows are re-read by ddy while they may still be in L2
        const int ch = ctx->param_fwd_chunk > 0 ? (int)std::min<long long>(ctx->param_fwd_chunk, nlev) : nlev;
        for (int z0 = 0; z0 < nlev; z0 += ch) {
            const int nl = std::min(ch, nlev - z0);
            RowsFwd3Args<T> ra{};
            ra.src = f[c] + pl * z0; ra.dfdx = (T *)io->d[2 * c] + pl * z0; ra.xpad = xb; ra.H = H ? H + S * z0 : nullptr;
            ra.npairs = (long long)ny * nl / 2; ra.ldx = ctx->ldx; ra.ny = ny; ra.L = ctx->L; ra.z0 = z0;
            ra.sc_press = scp; ra.kx = ctx->d_kx;
            ra.twF = twt<T>(ctx, nx, ROLE_FWD); ra.twB = twt<T>(ctx, nx, ROLE_BWD);
            ra.twPB = twt<T>(ctx, nx, ROLE_PADBWD);
            {
                LaunchScope ls(ctx->rec, "rows_fwd3", s());
                if ((rc = chk(RowsFwd3Launch<T>::run(nx, ra, s()), "rows_fwd3"))) return rc;
            }
            auto ca = colargs(xb, nx2, (long long)nx2 * ny, (T *)io->big[c] + plb * z0, nx2, plb, nx2, nl,
                              1.0 / ny, OP_PAD, ny);
            ca.tma = (int)ctx->param_pad_tma;
            ca.wait_err = ctx->d_ctl + 1;
            if ((rc = cols(OP_PAD, true, ny, ca, "pad_cols"))) return rc;
            if ((rc = ddy((T *)io->d[2 * c + 1] + pl * z0, f[c] + pl * z0, nl))) return rc;
            if (H && !(fwd_gform && c != 1)) {   // G form: H_x and H_z are transformed as G in press()
                // RHS levels 1..L of this chunk
                const int a0 = std::max(z0, 1), a1 = std::min(z0 + nl - 1, ctx->L);
                if (a1 >= a0) {
                    auto cb = colargs(H + S * a0, ctx->lhx, S, H + S * a0, ctx->lhx, S, ctx->lhx, a1 - a0 + 1, 1.0,
                                      OP_FWD, ny);
                    cb.zero_nyq = 1;
                    if ((rc = cols(OP_FWD, false, ny, cb, "press_fwd_cols"))) return rc;
                }
            }
        }
        return OBL_OK;
    }

    int step(const obl_step_io *io)
    {
        const int nlev = ctx->nz + 1;
        const T *f[4] = {(const T *)io->u, (const T *)io->v, (const T *)io->w, (const T *)io->theta};
        int rc;
        // param "fused": 0 multi-output line kernels (default), 1 cluster-fused forward pass,
        // 2 the plain composition of the per-routine entry points
        if (ctx->param_fused == 0 || (ctx->param_fused == 1 && ctx->nxt == ctx->nyt)) {
            fwd_gform = ctx->param_fused == 0 && gform(true);
            if ((rc = ctx->param_fused == 0 ? fwd_lines(io) : fwd_fused(io))) return rc;
            return press(f[0], f[1], f[2], (const T *)io->divtz_bot, (const T *)io->divtz_top, (T *)io->p,
                         (T *)io->dp[0], (T *)io->dp[1], (T *)io->dp[2], true, io);
        }
        for (int c = 0; c < 4; ++c) {
            if ((rc = ddx((T *)io->d[2 * c], f[c], nlev))) return rc;
            if ((rc = ddy((T *)io->d[2 * c + 1], f[c], nlev))) return rc;
            if ((rc = pad(f[c], (T *)io->big[c], nlev))) return rc;
        }
        if ((rc = press(f[0], f[1], f[2], (const T *)io->divtz_bot, (const T *)io->divtz_top, (T *)io->p,
                        (T *)io->dp[0], (T *)io->dp[1], (T *)io->dp[2])))
            return rc;
        return project((T *)io->u, (T *)io->v, (T *)io->w, (const T *)io->dp[0], (const T *)io->dp[1],
                       (const T *)io->dp[2]);
    }

    // ---- rollout problem of the adjoint ----
    // small work fields (ldx,nyt,0:nz); in the transposed step the first ones are reused
    enum { S_DUDY, S_DVDX, S_DWDX, S_DWDY, S_O1, S_O2, S_O3, S_CX, S_CY, S_CZ, S_P, S_DPDX, S_DPDY, S_DPDZ,
           S_T1, S_T2, S_T3, S_T4, S_N };
    // padded work fields (nxt2,nyt2,0:nz)
    enum { B_U, B_V, B_W, B_O1, B_O2, B_O3, B_X, B_Y, B_Z, B_AU, B_AV, B_AW, B_A1, B_A2, B_A3, B_N };
    T *rs(int i) { return (T *)ctx->rw_small[i].p; }
    T *rb(int i) { return (T *)ctx->rw_big[i].p; }
    int rollout_bufs()
    {
        int rc;
        for (int i = 0; i < S_N; ++i)
            if ((rc = ensure(ctx, ctx->rw_small[i], sizeof(T) * (size_t)ctx->field()))) return rc;
        for (int i = 0; i < B_N; ++i)
            if ((rc = ensure(ctx, ctx->rw_big[i], sizeof(T) * (size_t)ctx->big()))) return rc;
        return OBL_OK;
    }
    BigSet<T> bigset() { return BigSet<T>{rb(B_U), rb(B_V), rb(B_W), rb(B_O1), rb(B_O2), rb(B_O3)}; }

    // ddx/ddy of u, v, w, the vorticity and the six padded fields of convec
    // (108_convec.f90:38-76, derivatives of 103_flosol.f90:30-37)
    int convec_fields(const T *u, const T *v, const T *w)
    {
        const int nlev = ctx->nz + 1;
        int rc;
        {
            const T *xin[2] = {v, w}, *yin[2] = {u, w};
            T *xout[2] = {rs(S_DVDX), rs(S_DWDX)}, *yout[2] = {rs(S_DUDY), rs(S_DWDY)};
            if ((rc = ddx_multi(xout, xin, 2, nlev)) || (rc = ddy_multi(yout, yin, 2, nlev))) return rc;
        }
        {
            cudaError_t e = cudaSuccess;
            LaunchScope ls(ctx->rec, "vort", s());
            launch_vort<T>(u, v, rs(S_DUDY), rs(S_DVDX), rs(S_DWDX), rs(S_DWDY), rs(S_O1), rs(S_O2), rs(S_O3),
                           ctx->nxt, ctx->ldx, ctx->nyt, ctx->nz, ctx->dz, s(), e);
            if ((rc = chk(e, "vort"))) return rc;
        }
        const T *src[6] = {u, v, w, rs(S_O1), rs(S_O2), rs(S_O3)};
        T *big[6] = {rb(B_U), rb(B_V), rb(B_W), rb(B_O1), rb(B_O2), rb(B_O3)};
        return pad_multi(src, big, 6, nlev);
    }

    // convec (108_convec.f90:11-99): cx, cy, cz at levels 1..nz-1
    int convec(const T *u, const T *v, const T *w, T *cx, T *cy, T *cz)
    {
        int rc;
        if ((rc = rollout_bufs()) || (rc = convec_fields(u, v, w))) return rc;
        {
            cudaError_t e = cudaSuccess;
            LaunchScope ls(ctx->rec, "cross", s());
            launch_cross<T>(bigset(), rb(B_X), rb(B_Y), rb(B_Z), ctx->nxt2, ctx->nyt2, ctx->nz, s(), e);
            if ((rc = chk(e, "cross"))) return rc;
        }
        const long long pl = ctx->plane(), plb = (long long)ctx->nxt2 * ctx->nyt2;
        const T *src[3] = {rb(B_X) + plb, rb(B_Y) + plb, rb(B_Z) + plb};
        T *dst[3] = {cx + pl, cy + pl, cz + pl};
        return unpad_multi(src, dst, 3, ctx->nz - 1);
    }

    // P: press_stag_array (divtz = 0) + dpdz + project, in place
    int projection(T *u, T *v, T *w, int stress_free)
    {
        if (int rc = rollout_bufs()) return rc;
        obl_step_io io{};
        io.u = u; io.v = v; io.w = w;
        return press(u, v, w, nullptr, nullptr, rs(S_P), rs(S_DPDX), rs(S_DPDY), rs(S_DPDZ), false, &io,
                     stress_free);
    }

    // u1 = P(u - dt*tadv1*convec(u)), in place
    int rollout_step(T *u, T *v, T *w)
    {
        int rc;
        // the work fields must exist before their addresses are taken below
        if ((rc = rollout_bufs())) return rc;
        if ((rc = convec(u, v, w, rs(S_CX), rs(S_CY), rs(S_CZ)))) return rc;
        {
            cudaError_t e = cudaSuccess;
            LaunchScope ls(ctx->rec, "update", s());
            launch_update<T>(u, v, w, rs(S_CX), rs(S_CY), rs(S_CZ), ctx->dt_nd * kTadv1, ctx->nxt, ctx->ldx,
                             ctx->nyt, ctx->nz, s(), e);
            if ((rc = chk(e, "update"))) return rc;
        }
        return projection(u, v, w, -1);
    }

    // lambda <- P^T lambda.  With the Neumann top the bands of every k^2 > 0 column are
    // symmetric and the (0,0) column's transposed integration gives back the same mean
    // removal, so P^T = (P without the stress-free copy) applied to M S^T lambda, where S^T
    // is the transposed copy and M clears w(1), w(nz), plus the one entry P does not
    // produce: the w(1) row, -dt*tadv1*p(1)/dz of that same solve.
    int projection_vjp(T *lu, T *lv, T *lw)
    {
        int rc;
        cudaError_t e = cudaSuccess;
        {
            LaunchScope ls(ctx->rec, "adj_project_bc", s());
            launch_adj_project_bc<T>(lu, lv, lw, ctx->ldx, ctx->nyt, ctx->nz, (int)ctx->opt.ubc_stress_free, s(), e);
            if ((rc = chk(e, "adj_project_bc"))) return rc;
        }
        if ((rc = projection(lu, lv, lw, 0))) return rc;
        LaunchScope ls(ctx->rec, "adj_w1", s());
        launch_adj_w1<T>(lw, rs(S_P), -(ctx->dt_nd * kTadv1) / ctx->dz, ctx->nxt, ctx->ldx, ctx->nyt, s(), e);
        return chk(e, "adj_w1");
    }

    // lambda <- (d step / d state)^T lambda at the state (u, v, w)
    int step_vjp(const T *u, const T *v, const T *w, T *lu, T *lv, T *lw)
    {
        const int nlev = ctx->nz + 1;
        int rc;
        if ((rc = rollout_bufs()) || (rc = projection_vjp(lu, lv, lw))) return rc;
        // the state's convec fields (recomputed from the checkpoint), and the padded
        // adjoints of cx, cy, cz: pad(lambda) scaled by -dt*tadv1 inside the transposed
        // cross product (unpad^T = pad/2.25 and pad^T = 2.25*unpad cancel)
        if ((rc = convec_fields(u, v, w))) return rc;
        {
            const T *lam[3] = {lu, lv, lw};
            T *big[3] = {rb(B_X), rb(B_Y), rb(B_Z)};
            if ((rc = pad_multi(lam, big, 3, nlev))) return rc;
        }
        {
            cudaError_t e = cudaSuccess;
            LaunchScope ls(ctx->rec, "cross_adj", s());
            CrossAdjOut<T> out{rb(B_AU), rb(B_AV), rb(B_AW), rb(B_A1), rb(B_A2), rb(B_A3)};
            launch_cross_adj<T>(bigset(), rb(B_X), rb(B_Y), rb(B_Z), -ctx->dt_nd * kTadv1, out, ctx->nxt2,
                                ctx->nyt2, ctx->nz, s(), e);
            if ((rc = chk(e, "cross_adj"))) return rc;
        }
        // sU, sV, sW, s1, s2, s3 (unpadded adjoints) into the first six small fields
        {
            const T *src[6] = {rb(B_AU), rb(B_AV), rb(B_AW), rb(B_A1), rb(B_A2), rb(B_A3)};
            T *dst[6] = {rs(S_DUDY), rs(S_DVDX), rs(S_DWDX), rs(S_DWDY), rs(S_O1), rs(S_O2)};
            if ((rc = unpad_multi(src, dst, 6, nlev))) return rc;
        }
        T *sU = rs(S_DUDY), *sV = rs(S_DVDX), *sW = rs(S_DWDX), *s1 = rs(S_DWDY), *s2 = rs(S_O1), *s3 = rs(S_O2);
        T *q1 = rs(S_O3), *q2 = rs(S_CX);
        {
            cudaError_t e = cudaSuccess;
            LaunchScope ls(ctx->rec, "adj_q", s());
            launch_adj_q<T>(s1, s2, q1, q2, ctx->nxt, ctx->ldx, ctx->nyt, ctx->nz, s(), e);
            if ((rc = chk(e, "adj_q"))) return rc;
        }
        // ddx^T = -ddx, ddy^T = -ddy: the signs are applied in the combine kernel
        {
            const T *xin[2] = {s3, q2}, *yin[2] = {s3, q1};
            T *xout[2] = {rs(S_T2), rs(S_T3)}, *yout[2] = {rs(S_T1), rs(S_T4)};
            if ((rc = ddx_multi(xout, xin, 2, nlev)) || (rc = ddy_multi(yout, yin, 2, nlev))) return rc;
        }
        cudaError_t e = cudaSuccess;
        LaunchScope ls(ctx->rec, "adj_combine", s());
        AdjCombineArgs<T> a{lu, lv, lw, sU, sV, sW, s1, s2, rs(S_T1), rs(S_T2), rs(S_T3), rs(S_T4)};
        launch_adj_combine<T>(a, ctx->nxt, ctx->ldx, ctx->nyt, ctx->nz, ctx->dz, s(), e);
        return chk(e, "adj_combine");
    }

    // levels 1..nz-1 whose uvp height (k-0.5)*dz*z_i (012_io.f90:295) lies in (z_lo, z_hi)
    void band(double z_lo, double z_hi, int &klo, int &khi)
    {
        klo = 1;
        khi = 0;
        bool any = false;
        for (int k = 1; k <= ctx->nz - 1; ++k) {
            const double z = ((double)k - 0.5) * ctx->dz * ctx->grid.z_i;
            if (z > z_lo && z < z_hi) {
                if (!any) klo = k;
                khi = k;
                any = true;
            }
        }
    }

    // J of energy (103_flosol.f90) over the band; seeds dJ/d(u,v,w) into lu, lv, lw if given
    int ke_band(const T *u, const T *v, const T *w, double z_lo, double z_hi, double *J, T *lu, T *lv, T *lw)
    {
        int rc;
        if ((rc = ensure(ctx, ctx->ke, sizeof(double) * (size_t)(ke_parts() + 1)))) return rc;
        int klo, khi;
        band(z_lo, z_hi, klo, khi);
        double *part = (double *)ctx->ke.p;
        {
            cudaError_t e = cudaSuccess;
            LaunchScope ls(ctx->rec, "ke_band", s());
            ctx->rec.launches += 1;   // partial sums + their fixed-order sum
            launch_ke_band<T>(u, v, w, lu, lv, lw, part, part + ke_parts(), ctx->nxt, ctx->ldx, ctx->nyt, ctx->nz,
                              klo, khi, s(), e);
            if ((rc = chk(e, "ke_band"))) return rc;
        }
        if (J) {
            CK(cudaMemcpyAsync(J, part + ke_parts(), sizeof(double), cudaMemcpyDeviceToHost, s()));
            CK(cudaStreamSynchronize(s()));
        }
        return OBL_OK;
    }

    // ---- z-slab of a domain split over P ranks (slab.cuh) ----
    // This context holds the rank's slab: levels 0..L of the rank (L = its interior levels),
    // level 0 and L+1 being the planes it shares with the ranks below and above.
    SlabArgs<T> slab_args(int rank, int P)
    {
        SlabArgs<T> a{};
        a.Hx = (const C2<T> *)ctx->spec[0].p; a.Hy = (const C2<T> *)ctx->spec[1].p; a.Hz = (const C2<T> *)ctx->spec[2].p;
        a.phat = (C2<T> *)ctx->spec[3].p; a.dph = (C2<T> *)ctx->spec[4].p;
        a.v = (T *)ctx->slab_v.p;
        a.cp = (T *)ctx->slab_cp.p;
        a.n_isl = ctx->n_isl;
        a.isl_cols = ctx->n_isl ? ctx->d_isl : nullptr;
        a.isl_slot = ctx->n_isl ? ctx->d_isl_slot : nullptr;
        a.iy = (double2 *)ctx->slab_iy.p; a.iv = (double *)ctx->slab_iv.p;
        a.icp = (double *)ctx->slab_icp.p;
        a.kx = ctx->d_kx; a.ky = ctx->d_ky2;
        a.S = ctx->sp(); a.lhx = ctx->lhx; a.nyt = ctx->nyt; a.L = ctx->L; a.dz = ctx->dz;
        a.rank = rank; a.nranks = P;
        a.own_p0 = 1;
        return a;
    }
    // Segments of the single-domain column solve: enough (kx,ky)-column segments to fill
    // the GPU (8 resident blocks of 128 threads per SM) when the columns alone do not, at
    // least 8 levels each; 1 = the sequential sweep.
    int seg_parts(long long S, int L) const
    {
        if (ctx->param_tdma_segments > 0) return (int)std::min<long long>(ctx->param_tdma_segments, L);
        if (S >= 65536) return 1;
        int dev = 0, nsm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const long long want = ((long long)nsm * 8 * 128 + S - 1) / S;
        const long long P = std::min<long long>(std::min<long long>(want, kSlabMaxRanks), L / 8);
        return P > 1 ? (int)P : 1;
    }
    // the solve's column segments for this context (with the spectral dpdz or without)
    // Segments of each FP64 island column in the mixed mode's whole-column solves (1 = the
    // island columns sweep inside the FP32 bulk launch).  The column-segmented solve serves
    // the Neumann-top step with spectral dpdz and the three-spectra RHS.
    int isl_parts(const TdmaArgs<T> &ta) const
    {
        if (!ctx->n_isl || ta.gform || !ta.dph || ctx->opt.top_bc != OBL_TOP_NEUMANN) return 1;
        const long long P = ctx->param_isl_segments > 0 ? ctx->param_isl_segments : 16;
        const long long cap = std::min<long long>(kSlabMaxRanks, ctx->L / 8);
        return (int)std::max<long long>(1, std::min<long long>(P, cap));
    }
    int solve_parts(bool dpdz) const
    {
        return (ctx->opt.top_bc == OBL_TOP_NEUMANN && dpdz) ? seg_parts(ctx->sp(), ctx->L) : 1;
    }
    // the RHS in G form: the one-sweep and register-segmented solves take it; the
    // column-segmented solve keeps the three transformed spectra.  By default only with
    // FP64 storage: the RHS is a divergence whose terms nearly cancel, and G's partial sum
    // rounded to FP32 before the transform costs the FP64 island columns their exact RHS
    // assembly (at 512^2 x 256 the mixed form's p error rose from 1.4e-7 to 8.5e-6).
    bool gform(bool dpdz) const
    {
        return (ctx->param_gform == 2 || (ctx->param_gform == 1 && ctx->f64)) && solve_parts(dpdz) == 1;
    }
    // set by the step before its line-kernel forward pass: fwd_field leaves H_x and H_z to
    // press(); the z-slab path, which transforms all three, keeps it false
    bool fwd_gform = false;
    // the rank's forward pass (ddx, ddy, zero_padding of u,v,w,theta and the RHS spectra),
    // its boundary planes, and a copy of its H_z(1) plane for the rank below
    int slab_begin(const obl_step_io *io, int rank, int P, C2<T> *plane_out)
    {
        const long long S = ctx->sp();
        const size_t L = ctx->L, n = (size_t)S * L, ni = (size_t)(ctx->n_isl > 0 ? ctx->n_isl : 1) * L;
        int rc;
        if ((rc = ensure(ctx, ctx->slab_v, sizeof(T) * n)) || (rc = ensure(ctx, ctx->slab_cp, sizeof(T) * n)) ||
            (rc = ensure(ctx, ctx->slab_iy, sizeof(double2) * ni)) || (rc = ensure(ctx, ctx->slab_iv, sizeof(double) * ni)) ||
            (rc = ensure(ctx, ctx->slab_icp, sizeof(double) * ni)))
            return rc;
        if ((rc = fwd_lines(io))) return rc;
        C2<T> *Hz = (C2<T> *)ctx->spec[2].p;
        const int ldx = ctx->ldx, ny = ctx->nyt, nx = ctx->nxt, lhx = ctx->lhx;
        const double cst = 1.0 / ((double)nx * ny);
        // H_z(0) of the bottom rank: divtz(:,:,1) (109_press_stag_array.f90:186-196)
        if (rank == 0 && io->divtz_bot) {
            auto ra = rowargs(io->divtz_bot, ldx, Hz, lhx, ny, cst, OP_FWD, nx);
            if ((rc = rows(OP_FWD, nx, ra, "press_fwd_rows"))) return rc;
        } else {
            CK(cudaMemsetAsync(Hz, 0, sizeof(C2<T>) * S, s()));
        }
        // H_z(L+1) of the top rank: divtz(:,:,nz) (:197-200); the other ranks receive it
        if (rank == P - 1 && io->divtz_top) {
            auto ra = rowargs(io->divtz_top, ldx, Hz + S * (L + 1), lhx, ny, cst, OP_FWD, nx);
            if ((rc = rows(OP_FWD, nx, ra, "press_fwd_rows"))) return rc;
        } else {
            CK(cudaMemsetAsync(Hz + S * (L + 1), 0, sizeof(C2<T>) * S, s()));
        }
        for (long long zb : {0LL, (long long)L + 1}) {
            auto ca = colargs(Hz + S * zb, lhx, S, Hz + S * zb, lhx, S, lhx, 1, 1.0, OP_FWD, ny);
            ca.zero_nyq = 1;
            if ((rc = cols(OP_FWD, false, ny, ca, "press_bnd_cols"))) return rc;
        }
        CK(cudaMemcpyAsync(plane_out, Hz + S, sizeof(C2<T>) * S, cudaMemcpyDeviceToDevice, s()));
        return OBL_OK;
    }
    int slab_solve(const C2<T> *plane_above, int rank, int P, double *iface_out)
    {
        const long long S = ctx->sp();
        if (rank < P - 1)
            CK(cudaMemcpyAsync((C2<T> *)ctx->spec[2].p + S * (ctx->L + 1), plane_above, sizeof(C2<T>) * S,
                               cudaMemcpyDeviceToDevice, s()));
        SlabArgs<T> a = slab_args(rank, P);
        a.iface = iface_out;
        cudaError_t e = cudaSuccess;
        LaunchScope ls(ctx->rec, "slab_solve", s());
        launch_slab_solve<T>(a, s(), e);
        return chk(e, "slab_solve");
    }
    int slab_finish(const obl_step_io *io, const double *iface_all, int rank, int P)
    {
        const long long S = ctx->sp();
        const int L = ctx->L, nx = ctx->nxt, ny = ctx->nyt, lhx = ctx->lhx, ldx = ctx->ldx;
        int rc;
        SlabArgs<T> a = slab_args(rank, P);
        a.iface_all = iface_all;
        {
            cudaError_t e = cudaSuccess;
            LaunchScope ls(ctx->rec, "slab_finish", s());
            launch_slab_finish<T>(a, s(), e);
            if ((rc = chk(e, "slab_finish"))) return rc;
        }
        C2<T> *Hx = (C2<T> *)ctx->spec[0].p, *Hy = (C2<T> *)ctx->spec[1].p, *Hz = (C2<T> *)ctx->spec[2].p;
        C2<T> *ph = (C2<T> *)ctx->spec[3].p, *dph = (C2<T> *)ctx->spec[4].p;
        PinvColArgs<T> pc{};
        pc.ph = ph; pc.dph = dph; pc.Xp = Hz; pc.Xdy = Hy; pc.Xdz = dph;
        pc.S = S; pc.lhx = lhx; pc.kx = ctx->d_kx; pc.ky = ctx->d_ky2; pc.twB = twt<T>(ctx, ny, ROLE_BWD);
        {
            LaunchScope ls(ctx->rec, "pinv_cols", s());
            if ((rc = chk(PinvLaunch<T>::cols(ny, pc, L + 1, s()), "pinv_cols"))) return rc;
        }
        PinvRowArgs<T> pr{};
        pr.Xp = Hz; pr.kx = ctx->d_kx; pr.Xdy = Hy; pr.Xdz = dph;
        pr.p = (T *)io->p; pr.dpdx = (T *)io->dp[0]; pr.dpdy = (T *)io->dp[1]; pr.dpdz = (T *)io->dp[2];
        pr.u = (T *)io->u; pr.v = (T *)io->v; pr.w = (T *)io->w;
        pr.npairs = (long long)ny * (L + 1) / 2;
        pr.ldx = ldx; pr.ny = ny; pr.lhx = lhx;
        pr.dt_tadv1 = (T)(ctx->dt_nd * kTadv1);
        pr.twB = twt<T>(ctx, nx, ROLE_BWD);
        pr.w_from_1 = rank > 0;   // jz_min = 2 only on the bottom rank (110_project.f90:29-33)
        {
            LaunchScope ls(ctx->rec, "pinv_rows_project", s());
            if ((rc = chk(PinvLaunch<T>::rows(nx, pr, s()), "pinv_rows_project"))) return rc;
        }
        cudaError_t e = cudaSuccess;
        LaunchScope ls(ctx->rec, "project_bc", s());
        launch_project_bc_roles<T>((T *)io->u, (T *)io->v, (T *)io->w, ldx, ny, ctx->nz, (int)ctx->opt.ubc_stress_free,
                                   rank == 0, rank == P - 1, s(), e);
        return chk(e, "project_bc");
    }

    // ---- ensemble: the arguments of this instance's units in the persistent kernel ----
    // The same arguments fwd_lines and press(rhs_ready, proj) give the line kernels, except
    // that the four x-padded intermediates (xpad4) are separate: all four fields' row units
    // run in one phase.
    int ens_inst(const obl_step_io *io, T *xpad4, EnsInst<T> &I)
    {
        const int nlev = ctx->nz + 1, nx = ctx->nxt, ny = ctx->nyt, nx2 = ctx->nxt2, ny2 = ctx->nyt2;
        const int L = ctx->L, lhx = ctx->lhx, ldx = ctx->ldx;
        const long long S = ctx->sp();
        const size_t sb = sizeof(C2<T>) * (size_t)S * (ctx->nz + 1);
        int rc;
        for (int i = 0; i < 5; ++i)
            if ((rc = ensure(ctx, ctx->spec[i], sb))) return rc;
        if ((rc = ensure(ctx, ctx->cscr, sizeof(T) * (size_t)S * L))) return rc;
        if (ctx->n_isl) {
            if ((rc = ensure(ctx, ctx->isl_c, sizeof(double) * (size_t)ctx->n_isl * L))) return rc;
            if ((rc = ensure(ctx, ctx->isl_d, sizeof(double2) * (size_t)ctx->n_isl * (L + 1)))) return rc;
        }
        C2<T> *H[3] = {(C2<T> *)ctx->spec[0].p, (C2<T> *)ctx->spec[1].p, (C2<T> *)ctx->spec[2].p};
        C2<T> *ph = (C2<T> *)ctx->spec[3].p, *dph = (C2<T> *)ctx->spec[4].p;
        const T *f[4] = {(const T *)io->u, (const T *)io->v, (const T *)io->w, (const T *)io->theta};
        const double scp = ((1.0 / ((double)nx * ny)) / kTadv1) * (1.0 / ctx->dt_nd);
        const int WB = ens_wb<T>();
        I = EnsInst<T>{};
        I.nx = nx; I.ny = ny; I.nlev = nlev; I.L = L;
        for (int c = 0; c < 4; ++c) {
            T *xb = xpad4 + (size_t)c * nx2 * ny * nlev;
            RowsFwd3Args<T> &ra = I.rows[c];
            ra.src = f[c]; ra.dfdx = (T *)io->d[2 * c]; ra.xpad = xb; ra.H = c < 3 ? H[c] : nullptr;
            ra.npairs = (long long)ny * nlev / 2; ra.ldx = ldx; ra.ny = ny; ra.L = L; ra.z0 = 0;
            ra.sc_press = scp; ra.kx = ctx->d_kx;
            ra.twF = twt<T>(ctx, nx, ROLE_FWD); ra.twB = twt<T>(ctx, nx, ROLE_BWD);
            ra.twPB = twt<T>(ctx, nx, ROLE_PADBWD);
            I.padc[c] = colargs(xb, nx2, (long long)nx2 * ny, io->big[c], nx2, (long long)nx2 * ny2, nx2, nlev,
                                1.0 / ny, OP_PAD, ny);
            I.ddyc[c] = colargs(f[c], ldx, ctx->plane(), io->d[2 * c + 1], ldx, ctx->plane(), nx, nlev, 1.0 / ny,
                                OP_DERIV, ny);
            I.ddyc[c].ktab = ctx->d_ky1;
            if (c < 3) {
                I.fwdc[c] = colargs(H[c] + S, lhx, S, H[c] + S, lhx, S, lhx, L, 1.0, OP_FWD, ny);
                I.fwdc[c].zero_nyq = 1;
            }
        }
        I.rows_units = EnsGeoHost<T>::rows_units(nx, I.rows[0].npairs);
        I.pad_nb = (nx2 / 2 + WB - 1) / WB;
        I.ddy_nb = (nx / 2 + WB - 1) / WB;
        I.fwd_nb = (lhx + WB - 1) / WB;
        I.Hz = H[2];
        I.S = S;
        TdmaArgs<T> &ta = I.tdma;
        ta.gform = 0;          // the persistent kernel transforms all three spectra
        ta.Hx = H[0]; ta.Hy = H[1]; ta.Hz = H[2]; ta.phat = ph; ta.cscr = (T *)ctx->cscr.p;
        ta.kx = ctx->d_kx; ta.ky = ctx->d_ky2; ta.skip = ctx->n_isl ? ctx->d_skip : nullptr;
        ta.S = S; ta.lhx = lhx; ta.nyt = ny; ta.L = L; ta.dz = ctx->dz; ta.dph = dph;
        ta.neumann_top = ctx->opt.top_bc == OBL_TOP_NEUMANN;
        I.isl = IslandArgs{ctx->d_isl, ctx->n_isl, (double *)ctx->isl_c.p, (double2 *)ctx->isl_d.p};
        I.isl_units = (ctx->n_isl + 255) / 256;
        I.bulk_units = (S + 255) / 256;
        PinvColArgs<T> &pc = I.pc;
        pc.ph = ph; pc.dph = dph; pc.Xp = H[2]; pc.Xdy = H[1]; pc.Xdz = dph;
        pc.S = S; pc.lhx = lhx; pc.kx = ctx->d_kx; pc.ky = ctx->d_ky2; pc.twB = twt<T>(ctx, ny, ROLE_BWD);
        I.pc_nb = (lhx + WB - 1) / WB;
        PinvRowArgs<T> &pr = I.pr;
        pr.Xp = H[2]; pr.kx = ctx->d_kx; pr.Xdy = H[1]; pr.Xdz = dph;
        pr.p = (T *)io->p; pr.dpdx = (T *)io->dp[0]; pr.dpdy = (T *)io->dp[1]; pr.dpdz = (T *)io->dp[2];
        pr.u = (T *)io->u; pr.v = (T *)io->v; pr.w = (T *)io->w;
        pr.npairs = (long long)ny * (L + 1) / 2;
        pr.ldx = ldx; pr.ny = ny; pr.lhx = lhx;
        pr.dt_tadv1 = (T)(ctx->dt_nd * kTadv1);
        pr.twB = twt<T>(ctx, nx, ROLE_BWD);
        I.pr_units = EnsGeoHost<T>::pinv_rows_units(nx, pr.npairs);
        I.u = (T *)io->u; I.v = (T *)io->v; I.w = (T *)io->w;
        I.ldx = ldx; I.nz = ctx->nz; I.stress_free = (int)ctx->opt.ubc_stress_free;
        I.count[0] = 4 * I.rows_units;
        I.count[1] = 4LL * I.pad_nb * nlev + 4LL * I.ddy_nb * nlev + 3LL * I.fwd_nb * L + 1;
        I.count[2] = I.isl_units + I.bulk_units;
        I.count[3] = (long long)I.pc_nb * (L + 1);
        I.count[4] = I.pr_units;
        I.count[5] = 1;
        return OBL_OK;
    }

    // nsteps rollout steps with a checkpoint of every step's state, J of the final state and,
    // when gu is given, the reverse sweep of step_vjp from the checkpoints (each step's convec
    // fields are recomputed from its checkpoint)
    int rollout_grad(int nsteps, const T *u0, const T *v0, const T *w0, double z_lo, double z_hi, double *J,
                     T *gu, T *gv, T *gw)
    {
        const size_t F = (size_t)ctx->field();
        int rc;
        if ((rc = ensure(ctx, ctx->ckpt, sizeof(T) * F * 3 * (size_t)(nsteps + 1)))) return rc;
        T *ck = (T *)ctx->ckpt.p;
        CK(cudaMemcpyAsync(ck, u0, sizeof(T) * F, cudaMemcpyDeviceToDevice, s()));
        CK(cudaMemcpyAsync(ck + F, v0, sizeof(T) * F, cudaMemcpyDeviceToDevice, s()));
        CK(cudaMemcpyAsync(ck + 2 * F, w0, sizeof(T) * F, cudaMemcpyDeviceToDevice, s()));
        for (int n = 0; n < nsteps; ++n) {
            T *a = ck + 3 * F * (size_t)n, *b = a + 3 * F;
            CK(cudaMemcpyAsync(b, a, sizeof(T) * 3 * F, cudaMemcpyDeviceToDevice, s()));
            if ((rc = rollout_step(b, b + F, b + 2 * F))) return rc;
        }
        T *last = ck + 3 * F * (size_t)nsteps;
        if ((rc = ke_band(last, last + F, last + 2 * F, z_lo, z_hi, J, gu, gv, gw))) return rc;
        if (!gu) return OBL_OK;
        for (int n = nsteps - 1; n >= 0; --n) {
            T *a = ck + 3 * F * (size_t)n;
            if ((rc = step_vjp(a, a + F, a + 2 * F, gu, gv, gw))) return rc;
        }
        return OBL_OK;
    }
};

// ----------------------------------------------------------------------------- host staging
// An argument of a host-variant call: host pointer, element count, and which part the
// reference routine writes (rows of nx of nrow rows at pitch ld, from row0), if any.
struct HArg {
    const void *h;
    long long n;          // elements
    bool in;              // copy host -> device before the call
    bool out;             // copy the written region back
    long long ld;         // row pitch (elements)
    long long width;      // elements written per row
    long long row0, nrows;
};

static HArg harg_in(const void *h, long long n) { return HArg{h, n, true, false, 0, 0, 0, 0}; }
// output rows: x < width of rows [row0, row0+nrows) at pitch ld
static HArg harg_out(const void *h, long long n, bool in, long long ld, long long width, long long row0,
                     long long nrows)
{
    return HArg{h, n, in, true, ld, width, row0, nrows};
}

// Runs fn(device pointers) with every argument staged on the device in the storage
// type; host arrays are double (HT = double) or float (HT = float).
template <typename HT, class F> static int host_call(obl_ctx *ctx, std::vector<HArg> args, F fn)
{
    const size_t es = ctx->es();
    if (ctx->stage.size() < args.size()) ctx->stage.resize(args.size());
    if (ctx->stage64.size() < args.size()) ctx->stage64.resize(args.size());
    std::vector<void *> dp(args.size(), nullptr);
    const bool conv = (sizeof(HT) != es);
    int rc;
    for (size_t i = 0; i < args.size(); ++i) {
        if (!args[i].h) continue;
        if ((rc = ensure(ctx, ctx->stage[i], es * args[i].n))) return rc;
        dp[i] = ctx->stage[i].p;
        if (conv && (rc = ensure(ctx, ctx->stage64[i], sizeof(HT) * args[i].n))) return rc;
    }
    cudaStream_t s = ctx->stream;
    for (size_t i = 0; i < args.size(); ++i) {
        const HArg &a = args[i];
        if (!a.h || !a.in) continue;
        void *landing = conv ? ctx->stage64[i].p : dp[i];
        CK(cudaMemcpyAsync(landing, a.h, sizeof(HT) * a.n, cudaMemcpyHostToDevice, s));
        if (conv) {
            cudaError_t e = cudaSuccess;
            LaunchScope ls(ctx->rec, "convert", s);
            if (sizeof(HT) == 8) launch_convert_d2f((float *)dp[i], (const double *)landing, a.n, s, e);
            else launch_convert_f2d((double *)dp[i], (const float *)landing, a.n, s, e);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "convert");
        }
    }
    if ((rc = fn(dp))) return rc;
    for (size_t i = 0; i < args.size(); ++i) {
        const HArg &a = args[i];
        if (!a.h || !a.out) continue;
        const void *from = dp[i];
        if (conv) {
            cudaError_t e = cudaSuccess;
            LaunchScope ls(ctx->rec, "convert", s);
            if (sizeof(HT) == 8) launch_convert_f2d((double *)ctx->stage64[i].p, (const float *)dp[i], a.n, s, e);
            else launch_convert_d2f((float *)ctx->stage64[i].p, (const double *)dp[i], a.n, s, e);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "convert");
            from = ctx->stage64[i].p;
        }
        const size_t hb = sizeof(HT);
        char *hdst = (char *)a.h + hb * a.row0 * a.ld;
        const char *dsrc = (const char *)from + hb * a.row0 * a.ld;
        if (a.width == a.ld)
            CK(cudaMemcpyAsync(hdst, dsrc, hb * a.ld * a.nrows, cudaMemcpyDeviceToHost, s));
        else
            CK(cudaMemcpy2DAsync(hdst, hb * a.ld, dsrc, hb * a.ld, hb * a.width, a.nrows, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    return device_status(ctx);
}

} // namespace

// ============================================================================= C ABI
extern "C" {

int obl_ctx_create(const obl_grid *grid, const obl_options *opt, obl_ctx **out)
{
    if (!grid || !out) return OBL_ERR_ARG;
    *out = nullptr;
    obl_options o{};
    o.precision = OBL_PREC_F64;
    o.top_bc = OBL_TOP_NEUMANN;
    o.fp64_k2_max = -1.0;
    if (opt) o = *opt;
    const obl_grid &g = *grid;
    if (o.precision < 0 || o.precision > 2 || o.top_bc < 0 || o.top_bc > 1) return OBL_ERR_ARG;
    if (g.nxt <= 0 || g.nyt <= 0 || g.nzt < 4 || !(g.lx_tot > 0) || !(g.ly_tot > 0) || !(g.lz_tot > 0) ||
        !(g.z_i > 0) || !(g.dt > 0) || !(g.u_scale > 0))
        return OBL_ERR_ARG;
    if (!len_ok(g.nxt) || !len_ok(g.nyt)) return OBL_ERR_UNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return OBL_ERR_NODEV;
    }
    if (o.device < 0 || o.device >= ndev) return OBL_ERR_ARG;

    obl_ctx *ctx = new obl_ctx();
    ctx->grid = g;
    ctx->opt = o;
    ctx->dev = o.device;
    ctx->f64 = (o.precision == OBL_PREC_F64);
    // init_parameter (102_initial.f90:119-141) with npz = npy = 1
    ctx->nxt = g.nxt;
    ctx->nyt = g.nyt;
    ctx->nzt = g.nzt;
    ctx->nz = g.nzt;
    ctx->L = g.nzt - 1;
    ctx->lhx = g.nxt / 2 + 1;
    ctx->lhy = g.nyt / 2 + 1;
    ctx->ldx = 2 * ctx->lhx;
    ctx->nxt2 = 3 * g.nxt / 2;
    ctx->nyt2 = 3 * g.nyt / 2;
    // init_nondimensional (102_initial.f90:186-199)
    ctx->lx = g.lx_tot / g.z_i;
    ctx->ly = g.ly_tot / g.z_i;
    ctx->dz = (g.lz_tot / (double)(g.nzt - 1)) / g.z_i;
    ctx->dt_nd = g.dt * g.u_scale / g.z_i;

    auto bad = [&](int code) {
        obl_ctx_destroy(ctx);
        return code;
    };
    if (const char *fa = std::getenv("OBL_FAIL_ALLOC")) ctx->param_fail_alloc = std::atoll(fa);
    if (cudaSetDevice(ctx->dev) != cudaSuccess) return bad(OBL_ERR_CUDA);

    // wavenumbers (002_fft.f90:131-165)
    std::vector<double> kx(ctx->lhx), ky1(ctx->lhy), ky2(ctx->nyt);
    for (int i = 0; i < ctx->lhx; ++i) kx[i] = (((double)i * 2.0) * kPi) / ctx->lx;
    for (int i = 0; i < ctx->lhy; ++i) ky1[i] = (((double)i * 2.0) * kPi) / ctx->ly;
    kx[ctx->lhx - 1] = 0.0;
    ky1[ctx->lhy - 1] = 0.0;
    for (int j = 0; j < ctx->nyt; ++j)
        ky2[j] = (((double)(((j + ctx->nyt / 2) % ctx->nyt) - ctx->nyt / 2) * 2.0) * kPi) / ctx->ly;
    ky2[ctx->nyt / 2] = 0.0;
    auto upload = [&](double **d, const std::vector<double> &h) {
        if (dev_malloc(ctx, (void **)d, sizeof(double) * h.size()) != cudaSuccess) return false;
        return cudaMemcpy(*d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice) == cudaSuccess;
    };
    if (!upload(&ctx->d_kx, kx) || !upload(&ctx->d_ky1, ky1) || !upload(&ctx->d_ky2, ky2)) return bad(OBL_ERR_NOMEM);
    if (dev_malloc(ctx, (void **)&ctx->d_ctl, 4 * sizeof(int)) != cudaSuccess) return bad(OBL_ERR_NOMEM);
    if (cudaMemset(ctx->d_ctl, 0, 4 * sizeof(int)) != cudaSuccess) return bad(OBL_ERR_CUDA);

    // plan twiddle tables (FP64 on the host, stored in the storage precision) for the
    // forward / backward / padded transforms of both horizontal lengths
    for (int n : {ctx->nxt, ctx->nyt})
        for (int role = 0; role < 4; ++role) {
            const int key = 4 * n + role;
            if (ctx->tw.count(key)) continue;
            const std::vector<double> h = plan_table(n, role);
            const size_t m = h.size() / 2;
            const size_t b = (ctx->f64 ? sizeof(double2) : sizeof(float2)) * (m > 0 ? m : 1);
            void *d = nullptr;
            if (dev_malloc(ctx, &d, b) != cudaSuccess) return bad(OBL_ERR_NOMEM);
            ctx->tw[key] = d;
            if (m == 0) continue;
            if (ctx->f64) {
                if (cudaMemcpy(d, h.data(), b, cudaMemcpyHostToDevice) != cudaSuccess) return bad(OBL_ERR_CUDA);
            } else {
                std::vector<float2> hf(m);
                for (size_t i = 0; i < m; ++i) hf[i] = make_float2((float)h[2 * i], (float)h[2 * i + 1]);
                if (cudaMemcpy(d, hf.data(), b, cudaMemcpyHostToDevice) != cudaSuccess) return bad(OBL_ERR_CUDA);
            }
        }

    // FP64 islands of the mixed mode: the (0,0) mean mode and every column with
    // k^2 <= fp64_k2_max (weakly diagonally dominant systems)
    if (o.precision == OBL_PREC_MIXED) {
        double k2max = o.fp64_k2_max;
        // default: columns whose condition estimate (k^2 + 4/dz^2)/k^2 exceeds ~129.  At
        // 512x512x256 that is ~3.2k columns; FP32 elimination of only the (0,0) mode in FP64
        // left a 6.6e-4 error in p, this set gives 1.5e-6 (the same as 8x more columns).
        if (k2max < 0) k2max = (4.0 / (ctx->dz * ctx->dz)) / 128.0;
        std::vector<int> cols;
        std::vector<unsigned char> skip((size_t)ctx->lhx * ctx->nyt, 0);
        for (int j = 0; j < ctx->nyt; ++j)
            for (int i = 0; i < ctx->lhx; ++i) {
                if (i == ctx->lhx - 1 || j == ctx->nyt / 2) continue;
                const double k2 = kx[i] * kx[i] + ky2[j] * ky2[j];
                if (k2 <= k2max) {
                    cols.push_back(i + ctx->lhx * j);
                    skip[(size_t)i + (size_t)ctx->lhx * j] = 1;
                }
            }
        ctx->n_isl = (int)cols.size();
        if (ctx->n_isl) {
            std::vector<int> slot(skip.size(), -1);
            for (size_t k = 0; k < cols.size(); ++k) slot[(size_t)cols[k]] = (int)k;
            if (dev_malloc(ctx, (void **)&ctx->d_isl, sizeof(int) * cols.size()) != cudaSuccess) return bad(OBL_ERR_NOMEM);
            if (dev_malloc(ctx, (void **)&ctx->d_skip, skip.size()) != cudaSuccess) return bad(OBL_ERR_NOMEM);
            if (dev_malloc(ctx, (void **)&ctx->d_isl_slot, sizeof(int) * slot.size()) != cudaSuccess)
                return bad(OBL_ERR_NOMEM);
            cudaMemcpy(ctx->d_isl, cols.data(), sizeof(int) * cols.size(), cudaMemcpyHostToDevice);
            cudaMemcpy(ctx->d_skip, skip.data(), skip.size(), cudaMemcpyHostToDevice);
            cudaMemcpy(ctx->d_isl_slot, slot.data(), sizeof(int) * slot.size(), cudaMemcpyHostToDevice);
        }
    }
    ctx->param_fail_alloc = 0;   // OBL_FAIL_ALLOC applies to the creation only
    *out = ctx;
    return OBL_OK;
}

int obl_ctx_destroy(obl_ctx *ctx)
{
    if (!ctx) return OBL_OK;
    cudaSetDevice(ctx->dev);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    else cudaDeviceSynchronize();
    cudaFree(ctx->d_kx);
    cudaFree(ctx->d_ky1);
    cudaFree(ctx->d_ky2);
    cudaFree(ctx->d_isl);
    cudaFree(ctx->d_skip);
    for (auto &kv : ctx->tw) cudaFree(kv.second);
    for (auto &b : ctx->spec) cudaFree(b.p);
    cudaFree(ctx->cscr.p);
    cudaFree(ctx->isl_c.p);
    cudaFree(ctx->isl_d.p);
    cudaFree(ctx->tmp.p);
    cudaFree(ctx->fscr.p);
    for (auto &b : ctx->rw_small) cudaFree(b.p);
    for (auto &b : ctx->rw_big) cudaFree(b.p);
    cudaFree(ctx->ckpt.p);
    cudaFree(ctx->ke.p);
    io_stage_free(ctx->io);
    cudaFree(ctx->seg_iface.p);
    cudaFree(ctx->slab_v.p);
    cudaFree(ctx->slab_cp.p);
    cudaFree(ctx->slab_iy.p);
    cudaFree(ctx->slab_iv.p);
    cudaFree(ctx->slab_icp.p);
    cudaFree(ctx->d_isl_slot);
    cudaFree(ctx->d_ctl);
    for (auto &b : ctx->stage) cudaFree(b.p);
    for (auto &b : ctx->stage64) cudaFree(b.p);
    if (ctx->cin) cudaStreamDestroy(ctx->cin);
    if (ctx->cout) cudaStreamDestroy(ctx->cout);
    if (ctx->cout2) cudaStreamDestroy(ctx->cout2);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    for (auto e : ctx->side_ev)
        if (e) cudaEventDestroy(e);
    for (auto e : ctx->ev)
        if (e) cudaEventDestroy(e);
    delete ctx;
    return OBL_OK;
}

int obl_ctx_info(const obl_ctx *ctx, obl_info *info)
{
    if (!ctx || !info) return OBL_ERR_ARG;
    info->nxt = ctx->nxt; info->nyt = ctx->nyt; info->nzt = ctx->nzt; info->nz = ctx->nz;
    info->ldx = ctx->ldx; info->lhx = ctx->lhx; info->nxt2 = ctx->nxt2; info->nyt2 = ctx->nyt2;
    info->elem_bytes = (int)ctx->es();
    info->n_fp64_columns = ctx->n_isl;
    info->dz = ctx->dz; info->dt_nd = ctx->dt_nd; info->lx = ctx->lx; info->ly = ctx->ly;
    info->field_elems = ctx->field(); info->dfield_elems = ctx->dfield(); info->big_elems = ctx->big();
    info->spec_elems = ctx->sp();
    return OBL_OK;
}

int obl_set_stream(obl_ctx *ctx, void *stream)
{
    if (!ctx) return OBL_ERR_ARG;
    ctx->stream = (cudaStream_t)stream;
    return OBL_OK;
}

int obl_synchronize(obl_ctx *ctx)
{
    CTX_OK();
    CK(cudaStreamSynchronize(ctx->stream));
    return device_status(ctx);
}

int obl_last_error(const obl_ctx *ctx, char *buf, size_t n)
{
    if (!ctx || !buf || n == 0) return OBL_ERR_ARG;
    std::strncpy(buf, ctx->err.c_str(), n - 1);
    buf[n - 1] = 0;
    return OBL_OK;
}

long long obl_launch_count(const obl_ctx *ctx) { return ctx ? ctx->rec.launches : -1; }

static long long *param_slot(obl_ctx *ctx, const char *name)
{
    if (!std::strcmp(name, "fused")) return &ctx->param_fused;
    if (!std::strcmp(name, "fwd_clusters")) return &ctx->param_fwd_clusters;
    if (!std::strcmp(name, "fwd_cluster_size")) return &ctx->param_fwd_csize;
    if (!std::strcmp(name, "tdma_segments")) return &ctx->param_tdma_segments;
    if (!std::strcmp(name, "fail_alloc")) return &ctx->param_fail_alloc;
    if (!std::strcmp(name, "tdma_reg")) return &ctx->param_tdma_reg;
    if (!std::strcmp(name, "tdma_stage")) return &ctx->param_tdma_stage;
    if (!std::strcmp(name, "stage_timeout_test")) return &ctx->param_stage_timeout_test;
    if (!std::strcmp(name, "pad_tma")) return &ctx->param_pad_tma;
    if (!std::strcmp(name, "isl_segments")) return &ctx->param_isl_segments;
    if (!std::strcmp(name, "isl_concurrent")) return &ctx->param_isl_concurrent;
    if (!std::strcmp(name, "gform")) return &ctx->param_gform;
    if (!std::strcmp(name, "out_streams")) return &ctx->param_out_streams;
    if (!std::strcmp(name, "fwd_chunk")) return &ctx->param_fwd_chunk;
    return nullptr;
}

int obl_set_param(obl_ctx *ctx, const char *name, long long value)
{
    if (!ctx || !name) return OBL_ERR_ARG;
    long long *p = param_slot(ctx, name);
    if (!p) return fail(ctx, OBL_ERR_ARG, std::string("unknown parameter ") + name);
    if (!std::strcmp(name, "fwd_cluster_size") && (value < 1 || value > 16))
        return fail(ctx, OBL_ERR_ARG, "fwd_cluster_size must be 1..16");
    if (!std::strcmp(name, "tdma_segments") && (value < 0 || value > kSlabMaxRanks))
        return fail(ctx, OBL_ERR_ARG, "tdma_segments must be 0..16");
    *p = value;
    return OBL_OK;
}

int obl_get_param(obl_ctx *ctx, const char *name, long long *value)
{
    if (!ctx || !name || !value) return OBL_ERR_ARG;
    long long *p = param_slot(ctx, name);
    if (!p) return fail(ctx, OBL_ERR_ARG, std::string("unknown parameter ") + name);
    *value = *p;
    return OBL_OK;
}

int obl_timing_enable(obl_ctx *ctx, int on)
{
    if (!ctx) return OBL_ERR_ARG;
    ctx->rec.timing = on != 0;
    return OBL_OK;
}

int obl_timing_report(obl_ctx *ctx, char *buf, size_t n)
{
    CTX_OK();
    if (!buf || n == 0) return OBL_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    std::map<std::string, std::pair<long long, double>> agg;
    for (auto &r : ctx->rec.recs) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) { cudaGetLastError(); continue; }
        auto &x = agg[r.name];
        x.first += 1;
        x.second += ms;
    }
    ctx->rec.release();
    std::string js = "{";
    bool first = true;
    for (auto &kv : agg) {
        char tmp[256];
        std::snprintf(tmp, sizeof tmp, "%s\"%s\": [%lld, %.6f]", first ? "" : ", ", kv.first.c_str(),
                      kv.second.first, kv.second.second);
        js += tmp;
        first = false;
    }
    js += "}";
    if (js.size() + 1 > n) return fail(ctx, OBL_ERR_ARG, "timing report buffer too small");
    std::memcpy(buf, js.c_str(), js.size() + 1);
    return OBL_OK;
}

} // extern "C"

namespace {
template <typename T> struct OpsT : Ops<T> { using Tt = T; };
template <class F> static int dispatchT(obl_ctx *ctx, F fn)
{
    if (ctx->f64) {
        OpsT<double> o{{ctx}};
        return fn(o);
    }
    OpsT<float> o{{ctx}};
    return fn(o);
}
} // namespace

#define DEVCALL(ctx, body)                                                                         \
    do {                                                                                           \
        if (!ctx) return OBL_ERR_ARG;                                                              \
        if (cudaSetDevice(ctx->dev) != cudaSuccess) return fail(ctx, OBL_ERR_CUDA, "cudaSetDevice"); \
        return dispatchT(ctx, [&](auto &o) -> int {                                                \
            using T = typename std::remove_reference<decltype(o)>::type::Tt;                       \
            (void)sizeof(T);                                                                       \
            body                                                                                   \
        });                                                                                        \
    } while (0)

static bool nlev_ok(const obl_ctx *c, int nlev) { return nlev > 0 && ((long long)c->nyt * nlev) % 2 == 0; }

// ---- restart files ----
namespace {
struct Fd {
    int fd = -1;
    ~Fd()
    {
        if (fd >= 0) close(fd);
    }
};
// bytes of one field in the file: the global (nxt, nyt, nzranks*(nz-1)) FP64 array
long long io_field_bytes(const obl_ctx *c, int nzranks)
{
    return (long long)c->nxt * c->nyt * (c->nz - 1) * nzranks * (long long)sizeof(double);
}
// byte offset of this rank's z-block inside a field (subarray start (nz-1)*coordz)
long long io_rank_off(const obl_ctx *c, int zrank)
{
    return (long long)c->nxt * c->nyt * (c->nz - 1) * zrank * (long long)sizeof(double);
}
bool io_ranks_ok(int zrank, int nzranks) { return nzranks >= 1 && zrank >= 0 && zrank < nzranks; }
std::string vel_tt_name(const char *path_restart, int nums)
{
    char b[32];
    std::snprintf(b, sizeof b, "vel_tt%08d.out", nums);   // 012_io.f90:524, 102_01_ic.f90:711
    return std::string(path_restart) + b;
}
template <class F> int io_call(obl_ctx *ctx, F fn)
{
    if (cudaSetDevice(ctx->dev) != cudaSuccess) return fail(ctx, OBL_ERR_CUDA, "cudaSetDevice");
    return dispatchT(ctx, [&](auto &o) -> int {
        using T = typename std::remove_reference<decltype(o)>::type::Tt;
        return fn(o, (T *)nullptr);
    });
}
int open_out(obl_ctx *ctx, const std::string &fn, Fd &f)
{
    f.fd = open(fn.c_str(), O_WRONLY | O_CREAT, 0644);   // MPI_MODE_WRONLY+MPI_MODE_CREATE: no truncation
    if (f.fd < 0) return fail(ctx, OBL_ERR_IO, "open " + fn + ": " + std::strerror(errno));
    return OBL_OK;
}
int open_in(obl_ctx *ctx, const std::string &fn, Fd &f)
{
    f.fd = open(fn.c_str(), O_RDONLY);
    if (f.fd < 0) return fail(ctx, OBL_ERR_IO, "FILE DOES NOT EXIST: " + fn);   // 202_parallel.f90:1244-1246
    return OBL_OK;
}
} // namespace

extern "C" {

int obl_ddx_dev(obl_ctx *ctx, void *dfdx, const void *fun, int nlev)
{
    if (!ctx || !dfdx || !fun || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.ddx((T *)dfdx, (const T *)fun, nlev););
}
int obl_ddy_dev(obl_ctx *ctx, void *dfdy, const void *fun, int nlev)
{
    if (!ctx || !dfdy || !fun || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.ddy((T *)dfdy, (const T *)fun, nlev););
}
int obl_ddz_uv_dev(obl_ctx *ctx, void *dfdz, const void *fun)
{
    if (!ctx || !dfdz || !fun) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.ddz_uv((T *)dfdz, (const T *)fun););
}
#if OBL_CHECK
__global__ void k_check_selftest() { ck_in(1, 1, CK_SELFTEST); }
#endif
int obl_check_selftest(void)
{
#if OBL_CHECK
    k_check_selftest<<<1, 1>>>();
    return cudaDeviceSynchronize() == cudaSuccess ? OBL_OK : OBL_ERR_CUDA;
#else
    return OBL_ERR_UNSUPPORTED;
#endif
}
int obl_check_report(long long *count, char *buf, size_t n)
{
    if (!count) return OBL_ERR_ARG;
    if (buf && n) buf[0] = 0;
#if OBL_CHECK
    if (cudaDeviceSynchronize() != cudaSuccess) return OBL_ERR_CUDA;
    unsigned long long total = 0, first = 0;
    for (CheckReader r : check_readers()) {
        CheckRecord rec{0, 0};
        r(&rec, true);
        total += rec.count;
        if (!first && rec.first) first = rec.first;
    }
    *count = (long long)total;
    if (buf && n && total)
        std::snprintf(buf, n, "check site %d, index %lld", (int)(first >> 48), (long long)(first & 0xffffffffffffULL));
#else
    *count = -1;
#endif
    return OBL_OK;
}
int obl_selftest_grid_barrier(obl_ctx *ctx, int never_released)
{
    if (!ctx) return OBL_ERR_ARG;
    if (cudaSetDevice(ctx->dev) != cudaSuccess) return fail(ctx, OBL_ERR_CUDA, "cudaSetDevice");
    std::string err;
    const int rc = ens_barrier_selftest(never_released != 0, ctx->stream, err);
    return rc ? fail(ctx, rc, err) : OBL_OK;
}
int obl_divstress_uv_dev(obl_ctx *ctx, void *divt, const void *tx, const void *ty, const void *tz)
{
    if (!ctx || !divt || !tx || !ty || !tz || ctx->nz < 2) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.divstress((T *)divt, (const T *)tx, (const T *)ty, (const T *)tz, false););
}
int obl_divstress_w_dev(obl_ctx *ctx, void *divt, const void *tx, const void *ty, const void *tz)
{
    if (!ctx || !divt || !tx || !ty || !tz || ctx->nz < 2) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.divstress((T *)divt, (const T *)tx, (const T *)ty, (const T *)tz, true););
}
int obl_divstress_uv_slab_dev(obl_ctx *ctx, void *divt, const void *tx, const void *ty, const void *tz, int rank,
                              int nranks)
{
    if (!ctx || !divt || !tx || !ty || !tz || ctx->nz < 2 || nranks < 1 || rank < 0 || rank >= nranks)
        return OBL_ERR_ARG;
    DEVCALL(ctx, return o.divstress((T *)divt, (const T *)tx, (const T *)ty, (const T *)tz, false, rank == 0,
                                    rank == nranks - 1););
}
int obl_divstress_w_slab_dev(obl_ctx *ctx, void *divt, const void *tx, const void *ty, const void *tz, int rank,
                             int nranks)
{
    if (!ctx || !divt || !tx || !ty || !tz || ctx->nz < 2 || nranks < 1 || rank < 0 || rank >= nranks)
        return OBL_ERR_ARG;
    DEVCALL(ctx, return o.divstress((T *)divt, (const T *)tx, (const T *)ty, (const T *)tz, true, rank == 0,
                                    rank == nranks - 1););
}

int obl_write_file_3d_dev(obl_ctx *ctx, const void *var, const char *fn, long long disp0, int zrank, int nzranks)
{
    if (!ctx || !var || !fn || disp0 < 0 || !io_ranks_ok(zrank, nzranks) || ctx->nz < 2) return OBL_ERR_ARG;
    Fd f;
    int rc = open_out(ctx, fn, f);
    if (rc) return rc;
    return io_call(ctx, [&](auto &o, auto *tp) -> int {
        using T = typename std::remove_pointer<decltype(tp)>::type;
        return o.write_field((const T *)var, f.fd, disp0 + io_rank_off(ctx, zrank));
    });
}
int obl_read_file_3d_dev(obl_ctx *ctx, void *var, const char *fn, long long disp0, int zrank, int nzranks)
{
    if (!ctx || !var || !fn || disp0 < 0 || !io_ranks_ok(zrank, nzranks) || ctx->nz < 2) return OBL_ERR_ARG;
    Fd f;
    int rc = open_in(ctx, fn, f);
    if (rc) return rc;
    return io_call(ctx, [&](auto &o, auto *tp) -> int {
        using T = typename std::remove_pointer<decltype(tp)>::type;
        return o.read_field((T *)var, f.fd, disp0 + io_rank_off(ctx, zrank));
    });
}
int obl_checkpoint_final_dev(obl_ctx *ctx, const char *path_restart, int nums, const void *const *fields, int zrank,
                             int nzranks)
{
    if (!ctx || !path_restart || !fields || nums < 0 || !io_ranks_ok(zrank, nzranks) || ctx->nz < 2)
        return OBL_ERR_ARG;
    // the restart directory is created when missing (012_io.f90:514-518)
    struct stat st;
    if (path_restart[0] && stat(path_restart, &st) != 0 && mkdir(path_restart, 0755) != 0 && errno != EEXIST)
        return fail(ctx, OBL_ERR_IO, std::string("mkdir ") + path_restart + ": " + std::strerror(errno));
    Fd f;
    const std::string fn = vel_tt_name(path_restart, nums);
    int rc = open_out(ctx, fn, f);
    if (rc) return rc;
    const long long disp3d = io_field_bytes(ctx, nzranks), roff = io_rank_off(ctx, zrank);
    return io_call(ctx, [&](auto &o, auto *tp) -> int {
        using T = typename std::remove_pointer<decltype(tp)>::type;
        for (int k = 0; k < OBL_VEL_TT_FIELDS; ++k) {   // 012_io.f90:526-546
            int r = o.write_field((const T *)fields[k], f.fd, k * disp3d + roff);
            if (r) return r;
        }
        return OBL_OK;
    });
}
int obl_read_flow_field_dev(obl_ctx *ctx, const char *path_restart, int nums, void *const *fields, int zrank,
                            int nzranks)
{
    if (!ctx || !path_restart || !fields || nums < 0 || !io_ranks_ok(zrank, nzranks) || ctx->nz < 2)
        return OBL_ERR_ARG;
    Fd f;
    int rc = open_in(ctx, vel_tt_name(path_restart, nums), f);
    if (rc) return rc;
    const long long disp3d = io_field_bytes(ctx, nzranks), roff = io_rank_off(ctx, zrank);
    return io_call(ctx, [&](auto &o, auto *tp) -> int {
        using T = typename std::remove_pointer<decltype(tp)>::type;
        for (int k = 0; k < OBL_VEL_TT_FIELDS; ++k) {   // 102_01_ic.f90:713-733
            if (!fields[k]) continue;
            int r = o.read_field((T *)fields[k], f.fd, k * disp3d + roff);
            if (r) return r;
        }
        return OBL_OK;
    });
}
int obl_read_total_time(const char *fn, int *nums)
{
    if (!fn || !nums) return OBL_ERR_ARG;
    FILE *fp = std::fopen(fn, "r");
    if (!fp) {   // "Restart file NOT found": the run starts from step 0 (102_01_ic.f90:699-705)
        *nums = 0;
        return OBL_OK;
    }
    long long v = 0;
    const int got = std::fscanf(fp, "%lld", &v);   // list-directed read of one integer
    std::fclose(fp);
    if (got != 1 || v < 0 || v > 2147483647LL) return OBL_ERR_IO;
    *nums = (int)v;
    return OBL_OK;
}
int obl_write_total_time(const char *fn, int nums)
{
    if (!fn || nums < 0) return OBL_ERR_ARG;
    FILE *fp = std::fopen(fn, "w");
    if (!fp) return OBL_ERR_IO;
    // list-directed write of a default integer: right-aligned in 12 columns (012_io.f90:487-489)
    const int ok = std::fprintf(fp, "%12d\n", nums) > 0;
    return (std::fclose(fp) == 0 && ok) ? OBL_OK : OBL_ERR_IO;
}

int obl_ddz_w_dev(obl_ctx *ctx, void *dfdz, const void *fun)
{
    if (!ctx || !dfdz || !fun) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.ddz_w((T *)dfdz, (const T *)fun););
}
int obl_fftn_dev(obl_ctx *ctx, const void *in, void *out, int nlev)
{
    if (!ctx || !in || !out || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.fftn((const T *)in, (C2<T> *)out, nlev, 1.0););
}
int obl_ifftn_dev(obl_ctx *ctx, const void *in, void *out, int nlev)
{
    if (!ctx || !in || !out || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    DEVCALL(ctx, {
        int rc = ensure(ctx, ctx->tmp, sizeof(C2<T>) * (size_t)ctx->sp() * nlev);
        if (rc) return rc;
        return o.ifftn((const C2<T> *)in, (C2<T> *)ctx->tmp.p, (T *)out, 0, nlev, 0);
    });
}
int obl_zero_padding_dev(obl_ctx *ctx, const void *var, void *big, int nlev)
{
    if (!ctx || !var || !big || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.pad((const T *)var, (T *)big, nlev););
}
int obl_zero_unpadding_dev(obl_ctx *ctx, const void *big, void *var, int nlev)
{
    if (!ctx || !var || !big || nlev <= 0) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.unpad((const T *)big, (T *)var, nlev););
}
int obl_filter_data_dev(obl_ctx *ctx, void *f, int nlev)
{
    if (!ctx || !f || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.filter((T *)f, nlev););
}
int obl_press_stag_array_dev(obl_ctx *ctx, const void *u, const void *v, const void *w, const void *dbot,
                             const void *dtop, void *p, void *dpdx, void *dpdy)
{
    if (!ctx || !u || !v || !w || !p || !dpdx || !dpdy) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.press((const T *)u, (const T *)v, (const T *)w, (const T *)dbot, (const T *)dtop,
                                (T *)p, (T *)dpdx, (T *)dpdy););
}
int obl_dpdz_dev(obl_ctx *ctx, const void *p, void *dpdz)
{
    if (!ctx || !p || !dpdz) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.dpdz((const T *)p, (T *)dpdz););
}
int obl_project_dev(obl_ctx *ctx, void *u, void *v, void *w, const void *dpdx, const void *dpdy,
                    const void *dpdz)
{
    if (!ctx || !u || !v || !w || !dpdx || !dpdy || !dpdz) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.project((T *)u, (T *)v, (T *)w, (const T *)dpdx, (const T *)dpdy, (const T *)dpdz););
}
static bool step_io_ok(const obl_step_io *io)
{
    if (!io || !io->u || !io->v || !io->w || !io->theta || !io->p) return false;
    for (int i = 0; i < 8; ++i)
        if (!io->d[i]) return false;
    for (int i = 0; i < 4; ++i)
        if (!io->big[i]) return false;
    for (int i = 0; i < 3; ++i)
        if (!io->dp[i]) return false;
    return true;
}
int obl_step_dev(obl_ctx *ctx, const obl_step_io *io)
{
    if (!ctx || !step_io_ok(io)) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.step(io););
}

// ---------------------------------------------------------------- host entry points
#define HOSTCALL(HT, ctx, args, body)                                                              \
    do {                                                                                           \
        if (!ctx) return OBL_ERR_ARG;                                                              \
        if (cudaSetDevice(ctx->dev) != cudaSuccess) return fail(ctx, OBL_ERR_CUDA, "cudaSetDevice"); \
        return dispatchT(ctx, [&](auto &o) -> int {                                                \
            using T = typename std::remove_reference<decltype(o)>::type::Tt;                       \
            (void)sizeof(T);                                                                       \
            return host_call<HT>(ctx, args, [&](std::vector<void *> &d) -> int { body });         \
        });                                                                                        \
    } while (0)

int obl_ddx(obl_ctx *ctx, double *dfdx, const double *fun, int nlev)
{
    if (!ctx || !dfdx || !fun || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    const long long n = ctx->plane() * nlev;
    std::vector<HArg> a{harg_in(fun, n), harg_out(dfdx, n, false, ctx->ldx, ctx->nxt, 0, (long long)ctx->nyt * nlev)};
    HOSTCALL(double, ctx, a, return o.ddx((T *)d[1], (const T *)d[0], nlev););
}
int obl_ddy(obl_ctx *ctx, double *dfdy, const double *fun, int nlev)
{
    if (!ctx || !dfdy || !fun || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    const long long n = ctx->plane() * nlev;
    std::vector<HArg> a{harg_in(fun, n), harg_out(dfdy, n, false, ctx->ldx, ctx->nxt, 0, (long long)ctx->nyt * nlev)};
    HOSTCALL(double, ctx, a, return o.ddy((T *)d[1], (const T *)d[0], nlev););
}
int obl_ddz_uv(obl_ctx *ctx, double *dfdz, const double *fun)
{
    if (!ctx || !dfdz || !fun) return OBL_ERR_ARG;
    const long long n = ctx->field(), nyt = ctx->nyt;
    // level 0 (all ldx) and levels 2..nz-1 (x < nxt): copy the device result of the
    // whole array back after staging the host output too, so untouched levels survive
    std::vector<HArg> a{harg_in(fun, n), harg_out(dfdz, n, true, ctx->ldx, ctx->ldx, 0, nyt * (ctx->nz + 1))};
    HOSTCALL(double, ctx, a, return o.ddz_uv((T *)d[1], (const T *)d[0]););
}
static int divstress_host(obl_ctx *ctx, double *divt, const double *tx, const double *ty, const double *tz,
                          bool w_form)
{
    if (!ctx || !divt || !tx || !ty || !tz || ctx->nz < 2) return OBL_ERR_ARG;
    const long long n = ctx->field(), nyt = ctx->nyt;
    std::vector<HArg> a{harg_in(tx, n), harg_in(ty, n), harg_in(tz, n),
                        harg_out(divt, n, false, ctx->ldx, ctx->ldx, 0, nyt * (ctx->nz + 1))};
    HOSTCALL(double, ctx, a,
             return o.divstress((T *)d[3], (const T *)d[0], (const T *)d[1], (const T *)d[2], w_form););
}
int obl_divstress_uv(obl_ctx *ctx, double *divt, const double *tx, const double *ty, const double *tz)
{
    return divstress_host(ctx, divt, tx, ty, tz, false);
}
int obl_divstress_w(obl_ctx *ctx, double *divt, const double *tx, const double *ty, const double *tz)
{
    return divstress_host(ctx, divt, tx, ty, tz, true);
}
int obl_ddz_w(obl_ctx *ctx, double *dfdz, const double *fun)
{
    if (!ctx || !dfdz || !fun) return OBL_ERR_ARG;
    const long long n = ctx->field(), nyt = ctx->nyt;
    std::vector<HArg> a{harg_in(fun, n), harg_out(dfdz, n, true, ctx->ldx, ctx->ldx, 0, nyt * (ctx->nz + 1))};
    HOSTCALL(double, ctx, a, return o.ddz_w((T *)d[1], (const T *)d[0]););
}
int obl_fftn(obl_ctx *ctx, const double *in, double *out, int nlev)
{
    if (!ctx || !in || !out || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    const long long ni = ctx->plane() * nlev, no = 2 * ctx->sp() * nlev;
    std::vector<HArg> a{harg_in(in, ni), harg_out(out, no, false, no, no, 0, 1)};
    HOSTCALL(double, ctx, a, return o.fftn((const T *)d[0], (C2<T> *)d[1], nlev, 1.0););
}
int obl_ifftn(obl_ctx *ctx, const double *in, double *out, int nlev)
{
    if (!ctx || !in || !out || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    const long long ni = 2 * ctx->sp() * nlev, no = ctx->plane() * nlev;
    std::vector<HArg> a{harg_in(in, ni), harg_out(out, no, false, ctx->ldx, ctx->nxt, 0, (long long)ctx->nyt * nlev)};
    HOSTCALL(double, ctx, a, {
        int rc = ensure(ctx, ctx->tmp, sizeof(C2<T>) * (size_t)ctx->sp() * nlev);
        if (rc) return rc;
        return o.ifftn((const C2<T> *)d[0], (C2<T> *)ctx->tmp.p, (T *)d[1], 0, nlev, 0);
    });
}
int obl_zero_padding(obl_ctx *ctx, const double *var, double *big, int nlev)
{
    if (!ctx || !var || !big || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    const long long ni = ctx->plane() * nlev, no = (long long)ctx->nxt2 * ctx->nyt2 * nlev;
    std::vector<HArg> a{harg_in(var, ni), harg_out(big, no, false, no, no, 0, 1)};
    HOSTCALL(double, ctx, a, return o.pad((const T *)d[0], (T *)d[1], nlev););
}
int obl_zero_unpadding(obl_ctx *ctx, const double *big, double *var, int nlev)
{
    if (!ctx || !var || !big || nlev <= 0) return OBL_ERR_ARG;
    const long long ni = (long long)ctx->nxt2 * ctx->nyt2 * nlev, no = ctx->plane() * nlev;
    std::vector<HArg> a{harg_in(big, ni), harg_out(var, no, false, no, no, 0, 1)};
    HOSTCALL(double, ctx, a, return o.unpad((const T *)d[0], (T *)d[1], nlev););
}
int obl_filter_data(obl_ctx *ctx, double *f, int nlev)
{
    if (!ctx || !f || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    const long long n = ctx->plane() * nlev;
    std::vector<HArg> a{harg_out(f, n, true, n, n, 0, 1)};
    HOSTCALL(double, ctx, a, return o.filter((T *)d[0], nlev););
}
int obl_press_stag_array(obl_ctx *ctx, const double *u, const double *v, const double *w,
                         const double *dbot, const double *dtop, double *p, double *dpdx, double *dpdy)
{
    if (!ctx || !u || !v || !w || !p || !dpdx || !dpdy) return OBL_ERR_ARG;
    const long long nf = ctx->field(), nd = ctx->dfield(), pl = ctx->plane(), ny = ctx->nyt, L = ctx->L;
    std::vector<HArg> a{harg_in(u, nf), harg_in(v, nf), harg_in(w, nf),
                        dbot ? harg_in(dbot, pl) : HArg{nullptr, 0, false, false, 0, 0, 0, 0},
                        dtop ? harg_in(dtop, pl) : HArg{nullptr, 0, false, false, 0, 0, 0, 0},
                        harg_out(p, nf, false, ctx->ldx, ctx->nxt, 0, ny * (L + 1)),
                        harg_out(dpdx, nd, false, ctx->ldx, ctx->nxt, 0, ny * L),
                        harg_out(dpdy, nd, false, ctx->ldx, ctx->nxt, 0, ny * L)};
    HOSTCALL(double, ctx, a,
             return o.press((const T *)d[0], (const T *)d[1], (const T *)d[2], (const T *)d[3], (const T *)d[4],
                            (T *)d[5], (T *)d[6], (T *)d[7]););
}
int obl_dpdz(obl_ctx *ctx, const double *p, double *dpdz)
{
    if (!ctx || !p || !dpdz) return OBL_ERR_ARG;
    const long long nf = ctx->field(), nd = ctx->dfield(), ny = ctx->nyt;
    std::vector<HArg> a{harg_in(p, nf), harg_out(dpdz, nd, false, ctx->ldx, ctx->nxt, 0, ny * ctx->L)};
    HOSTCALL(double, ctx, a, return o.dpdz((const T *)d[0], (T *)d[1]););
}
int obl_project(obl_ctx *ctx, double *u, double *v, double *w, const double *dpdx, const double *dpdy,
                const double *dpdz)
{
    if (!ctx || !u || !v || !w || !dpdx || !dpdy || !dpdz) return OBL_ERR_ARG;
    const long long nf = ctx->field(), nd = ctx->dfield();
    std::vector<HArg> a{harg_out(u, nf, true, nf, nf, 0, 1), harg_out(v, nf, true, nf, nf, 0, 1),
                        harg_out(w, nf, true, nf, nf, 0, 1), harg_in(dpdx, nd), harg_in(dpdy, nd),
                        harg_in(dpdz, nd)};
    HOSTCALL(double, ctx, a,
             return o.project((T *)d[0], (T *)d[1], (T *)d[2], (const T *)d[3], (const T *)d[4], (const T *)d[5]););
}

} // extern "C"

template <typename HT> static int step_host(obl_ctx *ctx, const obl_step_io *io)
{
    const long long nf = ctx->field(), nd = ctx->dfield(), nb = ctx->big(), pl = ctx->plane(), ny = ctx->nyt;
    const long long L = ctx->L, nlev = ctx->nz + 1;
    std::vector<HArg> a;
    a.push_back(harg_out(io->u, nf, true, nf, nf, 0, 1));
    a.push_back(harg_out(io->v, nf, true, nf, nf, 0, 1));
    a.push_back(harg_out(io->w, nf, true, nf, nf, 0, 1));
    a.push_back(harg_in(io->theta, nf));
    for (int i = 0; i < 8; ++i) a.push_back(harg_out(io->d[i], nf, false, ctx->ldx, ctx->nxt, 0, ny * nlev));
    for (int i = 0; i < 4; ++i) a.push_back(harg_out(io->big[i], nb, false, nb, nb, 0, 1));
    a.push_back(harg_out(io->p, nf, false, ctx->ldx, ctx->nxt, 0, ny * (L + 1)));
    for (int i = 0; i < 3; ++i) a.push_back(harg_out(io->dp[i], nd, false, ctx->ldx, ctx->nxt, 0, ny * L));
    a.push_back(io->divtz_bot ? harg_in(io->divtz_bot, pl) : HArg{nullptr, 0, false, false, 0, 0, 0, 0});
    a.push_back(io->divtz_top ? harg_in(io->divtz_top, pl) : HArg{nullptr, 0, false, false, 0, 0, 0, 0});
    if (cudaSetDevice(ctx->dev) != cudaSuccess) return fail(ctx, OBL_ERR_CUDA, "cudaSetDevice");
    return dispatchT(ctx, [&](auto &o) -> int {
        return host_call<HT>(ctx, a, [&](std::vector<void *> &d) -> int {
            obl_step_io dio{};
            dio.u = d[0]; dio.v = d[1]; dio.w = d[2]; dio.theta = d[3];
            for (int i = 0; i < 8; ++i) dio.d[i] = d[4 + i];
            for (int i = 0; i < 4; ++i) dio.big[i] = d[12 + i];
            dio.p = d[16];
            for (int i = 0; i < 3; ++i) dio.dp[i] = d[17 + i];
            dio.divtz_bot = d[20];
            dio.divtz_top = d[21];
            return o.step(&dio);
        });
    });
}

// The host step with its copies overlapped (line-kernel form):
//   input stream:   u, v, w, theta host -> device, one event per field;
//   compute stream: field c's forward kernels as soon as field c has landed, then the
//                   pressure solve and project();
//   output stream:  field c's ddx, ddy and padded field device -> host as soon as its
//                   kernels are done; p, dp*, u, v, w after the solve.
// The device-to-host volume (about 6 of the 7.6 GB of a 512^2 x 256 FP32 step, 13 of 15 GB
// with real(8) host arrays) dominates; it now starts after the first field instead of after
// the whole step, and the input copies run under it.  When the host type HT differs from
// the storage type T (real(8) arrays of a caller on a mixed-precision context), each input
// lands in a staging buffer of the host type and is converted on the input stream, and
// each output is converted on the output stream just before its copy.  Pinned host memory
// is needed for the copies to overlap; with pageable memory the same calls complete in
// order.  Results are the same as the staged path.
template <typename HT, typename T> static int step_host_overlapped(obl_ctx *ctx, const obl_step_io *io)
{
    constexpr bool conv = sizeof(HT) != sizeof(T);
    const long long nf = ctx->field(), nd = ctx->dfield(), nb = ctx->big(), pl = ctx->plane(), ny = ctx->nyt;
    const long long L = ctx->L, nlev = ctx->nz + 1;
    if (cudaSetDevice(ctx->dev) != cudaSuccess) return fail(ctx, OBL_ERR_CUDA, "cudaSetDevice");
    if (!ctx->cin) {
        CK(cudaStreamCreateWithFlags(&ctx->cin, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&ctx->cout, cudaStreamNonBlocking));
        for (auto &e : ctx->ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (ctx->param_out_streams > 1 && !ctx->cout2) CK(cudaStreamCreateWithFlags(&ctx->cout2, cudaStreamNonBlocking));
    // device buffers: the staging slots of the staged path (same layout)
    const long long n[22] = {nf, nf, nf, nf, nf, nf, nf, nf, nf, nf, nf, nf, nb, nb, nb, nb, nf, nd, nd, nd, pl, pl};
    const void *h[22] = {io->u, io->v, io->w, io->theta, io->d[0], io->d[1], io->d[2], io->d[3], io->d[4], io->d[5],
                         io->d[6], io->d[7], io->big[0], io->big[1], io->big[2], io->big[3], io->p, io->dp[0], io->dp[1],
                         io->dp[2], io->divtz_bot, io->divtz_top};
    if (ctx->stage.size() < 22) ctx->stage.resize(22);
    if (ctx->stage64.size() < 22) ctx->stage64.resize(22);
    void *d[22] = {}, *l[22] = {};
    int rc;
    for (int i = 0; i < 22; ++i) {
        if (!h[i]) continue;
        if ((rc = ensure(ctx, ctx->stage[i], sizeof(T) * n[i]))) return rc;
        d[i] = ctx->stage[i].p;
        if (conv) {
            if ((rc = ensure(ctx, ctx->stage64[i], sizeof(HT) * n[i]))) return rc;
            l[i] = ctx->stage64[i].p;
        } else {
            l[i] = d[i];
        }
    }
    obl_step_io dio{};
    dio.u = d[0]; dio.v = d[1]; dio.w = d[2]; dio.theta = d[3];
    for (int i = 0; i < 8; ++i) dio.d[i] = d[4 + i];
    for (int i = 0; i < 4; ++i) dio.big[i] = d[12 + i];
    dio.p = d[16];
    for (int i = 0; i < 3; ++i) dio.dp[i] = d[17 + i];
    dio.divtz_bot = d[20];
    dio.divtz_top = d[21];
    const cudaStream_t s = ctx->stream, ci = ctx->cin;
    // the outputs alternate between the copy streams (two DMA engines when there are two)
    const cudaStream_t cos[2] = {ctx->cout, ctx->param_out_streams > 1 ? ctx->cout2 : ctx->cout};
    int nout = 0;
    // host type -> storage type (or storage -> host) of n elements on stream st
    auto convert = [&](void *dst, const void *src, long long cnt, bool to_storage, cudaStream_t st) -> cudaError_t {
        cudaError_t e = cudaSuccess;
        LaunchScope ls(ctx->rec, "convert", st);
        const bool d2f = to_storage ? (sizeof(HT) == 8) : (sizeof(T) == 8);
        if (d2f) launch_convert_d2f((float *)dst, (const double *)src, cnt, st, e);
        else launch_convert_f2d((double *)dst, (const float *)src, cnt, st, e);
        return e;
    };
    auto in = [&](int i) -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(l[i], h[i], sizeof(HT) * n[i], cudaMemcpyHostToDevice, ci);
        if (e == cudaSuccess && conv) e = convert(d[i], l[i], n[i], true, ci);
        return e;
    };
    // rows [row0, row0+nrows) of pitch ld, the first width elements of each (x < nxt)
    auto out = [&](int i, long long ld, long long width, long long row0, long long nrows) -> cudaError_t {
        const cudaStream_t co = cos[(nout++) & 1];
        if (conv) {
            cudaError_t e = convert((HT *)l[i] + row0 * ld, (const T *)d[i] + row0 * ld, ld * nrows, false, co);
            if (e != cudaSuccess) return e;
        }
        char *hd = (char *)h[i] + sizeof(HT) * row0 * ld;
        const char *dd = (const char *)l[i] + sizeof(HT) * row0 * ld;
        if (width == ld) return cudaMemcpyAsync(hd, dd, sizeof(HT) * ld * nrows, cudaMemcpyDeviceToHost, co);
        return cudaMemcpy2DAsync(hd, sizeof(HT) * ld, dd, sizeof(HT) * ld, sizeof(HT) * width, nrows,
                                 cudaMemcpyDeviceToHost, co);
    };
    if (h[20]) CK(in(20));
    if (h[21]) CK(in(21));
    for (int c = 0; c < 4; ++c) {
        CK(in(c));
        CK(cudaEventRecord(ctx->ev[c], ci));
    }
    Ops<T> o{ctx};
    o.fwd_gform = o.gform(true);
    if ((rc = o.fwd_prepare())) return rc;
    for (int c = 0; c < 4; ++c) {
        CK(cudaStreamWaitEvent(s, ctx->ev[c], 0));
        if ((rc = o.fwd_field(&dio, c))) return rc;
        CK(cudaEventRecord(ctx->ev[4 + c], s));
        for (cudaStream_t co : cos) CK(cudaStreamWaitEvent(co, ctx->ev[4 + c], 0));
        CK(out(4 + 2 * c, ctx->ldx, ctx->nxt, 0, ny * nlev));
        CK(out(5 + 2 * c, ctx->ldx, ctx->nxt, 0, ny * nlev));
        CK(out(12 + c, nb, nb, 0, 1));
    }
    if ((rc = o.press((const T *)dio.u, (const T *)dio.v, (const T *)dio.w, (const T *)dio.divtz_bot,
                      (const T *)dio.divtz_top, (T *)dio.p, (T *)dio.dp[0], (T *)dio.dp[1], (T *)dio.dp[2], true, &dio)))
        return rc;
    CK(cudaEventRecord(ctx->ev[8], s));
    for (cudaStream_t co : cos) CK(cudaStreamWaitEvent(co, ctx->ev[8], 0));
    CK(out(16, ctx->ldx, ctx->nxt, 0, ny * (L + 1)));
    for (int i = 0; i < 3; ++i) CK(out(17 + i, ctx->ldx, ctx->nxt, 0, ny * L));
    for (int i = 0; i < 3; ++i) CK(out(i, nf, nf, 0, 1));
    for (cudaStream_t co : cos) CK(cudaStreamSynchronize(co));
    CK(cudaStreamSynchronize(s));
    return device_status(ctx);
}

template <typename HT> static int step_host_any(obl_ctx *ctx, const obl_step_io *io)
{
    if (ctx->param_fused == 0)
        return ctx->es() == 4 ? step_host_overlapped<HT, float>(ctx, io) : step_host_overlapped<HT, double>(ctx, io);
    return step_host<HT>(ctx, io);
}

extern "C" {

int obl_step(obl_ctx *ctx, const obl_step_io *io)
{
    if (!ctx || !step_io_ok(io)) return OBL_ERR_ARG;
    return step_host_any<double>(ctx, io);
}
int obl_step_f32(obl_ctx *ctx, const obl_step_io *io)
{
    if (!ctx || !step_io_ok(io)) return OBL_ERR_ARG;
    return step_host_any<float>(ctx, io);
}

} // extern "C"

// ============================================================================= rollout and its transpose
static int rollout_check(obl_ctx *ctx, bool transpose)
{
    if (ctx->nz < 5) return fail(ctx, OBL_ERR_UNSUPPORTED, "rollout: needs nzt >= 5");
    if (transpose && ctx->opt.top_bc != OBL_TOP_NEUMANN)
        return fail(ctx, OBL_ERR_UNSUPPORTED, "rollout transpose: only the Neumann-top pressure mode (OBL_TOP_NEUMANN)");
    return OBL_OK;
}
static const HArg kNoArg{nullptr, 0, false, false, 0, 0, 0, 0};

extern "C" {

int obl_convec_dev(obl_ctx *ctx, const void *u, const void *v, const void *w, void *cx, void *cy, void *cz)
{
    if (!ctx || !u || !v || !w || !cx || !cy || !cz) return OBL_ERR_ARG;
    if (int rc = rollout_check(ctx, false)) return rc;
    DEVCALL(ctx, return o.convec((const T *)u, (const T *)v, (const T *)w, (T *)cx, (T *)cy, (T *)cz););
}
int obl_rollout_step_dev(obl_ctx *ctx, void *u, void *v, void *w)
{
    if (!ctx || !u || !v || !w) return OBL_ERR_ARG;
    if (int rc = rollout_check(ctx, false)) return rc;
    DEVCALL(ctx, return o.rollout_step((T *)u, (T *)v, (T *)w););
}
int obl_rollout_step_vjp_dev(obl_ctx *ctx, const void *u, const void *v, const void *w, void *lu, void *lv,
                             void *lw)
{
    if (!ctx || !u || !v || !w || !lu || !lv || !lw) return OBL_ERR_ARG;
    if (int rc = rollout_check(ctx, true)) return rc;
    DEVCALL(ctx, return o.step_vjp((const T *)u, (const T *)v, (const T *)w, (T *)lu, (T *)lv, (T *)lw););
}
int obl_ke_band_dev(obl_ctx *ctx, const void *u, const void *v, const void *w, double z_lo, double z_hi,
                    double *J, void *lu, void *lv, void *lw)
{
    if (!ctx || !u || !v || !w || !J || (lu && (!lv || !lw))) return OBL_ERR_ARG;
    DEVCALL(ctx, return o.ke_band((const T *)u, (const T *)v, (const T *)w, z_lo, z_hi, J, (T *)lu, (T *)lv,
                                  (T *)lw););
}
int obl_rollout_grad_dev(obl_ctx *ctx, int nsteps, const void *u0, const void *v0, const void *w0, double z_lo,
                         double z_hi, double *J, void *gu, void *gv, void *gw)
{
    if (!ctx || nsteps < 0 || !u0 || !v0 || !w0 || !J || (gu && (!gv || !gw))) return OBL_ERR_ARG;
    if (int rc = rollout_check(ctx, gu != nullptr)) return rc;
    DEVCALL(ctx, return o.rollout_grad(nsteps, (const T *)u0, (const T *)v0, (const T *)w0, z_lo, z_hi, J,
                                       (T *)gu, (T *)gv, (T *)gw););
}

int obl_convec(obl_ctx *ctx, const double *u, const double *v, const double *w, double *cx, double *cy,
               double *cz)
{
    if (!ctx || !u || !v || !w || !cx || !cy || !cz) return OBL_ERR_ARG;
    if (int rc = rollout_check(ctx, false)) return rc;
    const long long nf = ctx->field(), ny = ctx->nyt, nl = ctx->nz - 1;
    std::vector<HArg> a{harg_in(u, nf), harg_in(v, nf), harg_in(w, nf),
                        harg_out(cx, nf, false, ctx->ldx, ctx->nxt, ny, ny * nl),
                        harg_out(cy, nf, false, ctx->ldx, ctx->nxt, ny, ny * nl),
                        harg_out(cz, nf, false, ctx->ldx, ctx->nxt, ny, ny * nl)};
    HOSTCALL(double, ctx, a,
             return o.convec((const T *)d[0], (const T *)d[1], (const T *)d[2], (T *)d[3], (T *)d[4], (T *)d[5]););
}
int obl_rollout_step(obl_ctx *ctx, double *u, double *v, double *w)
{
    if (!ctx || !u || !v || !w) return OBL_ERR_ARG;
    if (int rc = rollout_check(ctx, false)) return rc;
    const long long nf = ctx->field();
    std::vector<HArg> a{harg_out(u, nf, true, nf, nf, 0, 1), harg_out(v, nf, true, nf, nf, 0, 1),
                        harg_out(w, nf, true, nf, nf, 0, 1)};
    HOSTCALL(double, ctx, a, return o.rollout_step((T *)d[0], (T *)d[1], (T *)d[2]););
}
int obl_rollout_step_vjp(obl_ctx *ctx, const double *u, const double *v, const double *w, double *lu,
                         double *lv, double *lw)
{
    if (!ctx || !u || !v || !w || !lu || !lv || !lw) return OBL_ERR_ARG;
    if (int rc = rollout_check(ctx, true)) return rc;
    const long long nf = ctx->field();
    std::vector<HArg> a{harg_in(u, nf), harg_in(v, nf), harg_in(w, nf), harg_out(lu, nf, true, nf, nf, 0, 1),
                        harg_out(lv, nf, true, nf, nf, 0, 1), harg_out(lw, nf, true, nf, nf, 0, 1)};
    HOSTCALL(double, ctx, a,
             return o.step_vjp((const T *)d[0], (const T *)d[1], (const T *)d[2], (T *)d[3], (T *)d[4],
                               (T *)d[5]););
}
int obl_ke_band(obl_ctx *ctx, const double *u, const double *v, const double *w, double z_lo, double z_hi,
                double *J, double *lu, double *lv, double *lw)
{
    if (!ctx || !u || !v || !w || !J || (lu && (!lv || !lw))) return OBL_ERR_ARG;
    const long long nf = ctx->field();
    std::vector<HArg> a{harg_in(u, nf), harg_in(v, nf), harg_in(w, nf),
                        lu ? harg_out(lu, nf, false, nf, nf, 0, 1) : kNoArg,
                        lu ? harg_out(lv, nf, false, nf, nf, 0, 1) : kNoArg,
                        lu ? harg_out(lw, nf, false, nf, nf, 0, 1) : kNoArg};
    HOSTCALL(double, ctx, a,
             return o.ke_band((const T *)d[0], (const T *)d[1], (const T *)d[2], z_lo, z_hi, J, (T *)d[3],
                              (T *)d[4], (T *)d[5]););
}
int obl_rollout_grad(obl_ctx *ctx, int nsteps, const double *u0, const double *v0, const double *w0,
                     double z_lo, double z_hi, double *J, double *gu, double *gv, double *gw)
{
    if (!ctx || nsteps < 0 || !u0 || !v0 || !w0 || !J || (gu && (!gv || !gw))) return OBL_ERR_ARG;
    if (int rc = rollout_check(ctx, gu != nullptr)) return rc;
    const long long nf = ctx->field();
    std::vector<HArg> a{harg_in(u0, nf), harg_in(v0, nf), harg_in(w0, nf),
                        gu ? harg_out(gu, nf, false, nf, nf, 0, 1) : kNoArg,
                        gu ? harg_out(gv, nf, false, nf, nf, 0, 1) : kNoArg,
                        gu ? harg_out(gw, nf, false, nf, nf, 0, 1) : kNoArg};
    HOSTCALL(double, ctx, a,
             return o.rollout_grad(nsteps, (const T *)d[0], (const T *)d[1], (const T *)d[2], z_lo, z_hi, J,
                                   (T *)d[3], (T *)d[4], (T *)d[5]););
}

} // extern "C"

// ============================================================================= no-allocation variant
// Some callers cannot allocate device memory at call time: an application that hands all
// device memory to its own pool at start-up and forbids allocation afterwards (a time loop
// that sized its fields once), or code on a latency-critical path where cudaMalloc may
// block and cudaFree waits for the whole device.  For them zero_padding has one variant
// whose intermediate x-padded plane lives in a fixed-size static device array instead of
// a buffer that the context allocates on first use.  The array is part of the module
// image, so every GPU that loads this library holds OBL_NOALLOC_SCRATCH_BYTES until the
// process exits.
namespace {
constexpr size_t kNoAllocBytes = OBL_NOALLOC_SCRATCH_BYTES;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch, looked up once per device with that device
// current.  In host code the array's name is only a host-side stand-in, never a device
// address, so kernels receive this looked-up pointer.
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[64];

int noalloc_scratch(obl_ctx *ctx, void **out)
{
    if (ctx->dev < 0 || ctx->dev >= 64)
        return fail(ctx, OBL_ERR_ARG, "zero_padding_noalloc: device ordinal beyond the scratch table");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[ctx->dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        if (!p) return fail(ctx, OBL_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) returned NULL");
        g_noalloc_ptr[ctx->dev] = p;
    }
    *out = g_noalloc_ptr[ctx->dev];
    return OBL_OK;
}
} // namespace

extern "C" int obl_zero_padding_noalloc_dev(obl_ctx *ctx, const void *var, void *var_big, int nlev)
{
    if (!ctx || !var || !var_big || !nlev_ok(ctx, nlev)) return OBL_ERR_ARG;
    const size_t need = ctx->es() * (size_t)ctx->nxt2 * (size_t)ctx->nyt * (size_t)nlev;
    if (need > kNoAllocBytes)
        return fail(ctx, OBL_ERR_ARG,
                    "zero_padding_noalloc: " + std::to_string(nlev) + " level(s) need " + std::to_string(need) +
                        " bytes of scratch but the static scratch holds " + std::to_string(kNoAllocBytes) +
                        " bytes; pass fewer levels per call");
    // the caller's current device is put back on return
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (cudaSetDevice(ctx->dev) != cudaSuccess) return fail(ctx, OBL_ERR_CUDA, "cudaSetDevice");
    void *xb = nullptr;
    int rc = noalloc_scratch(ctx, &xb);
    if (!rc)
        rc = dispatchT(ctx, [&](auto &o) -> int {
            using T = typename std::remove_reference<decltype(o)>::type::Tt;
            return o.pad_with_scratch((const T *)var, (T *)var_big, (T *)xb, nlev);
        });
    if (prev >= 0 && prev != ctx->dev) cudaSetDevice(prev);
    return rc;
}

// ============================================================================= ensemble
// Many independent instances (each its own obl_ctx: grid, tables, work buffers) advanced
// through the step together.  Modes:
//   OBL_ENS_SEQUENTIAL  one instance after the other on the ensemble's stream;
//   OBL_ENS_CONCURRENT  every instance on its own stream, forked from and joined back
//                       to the ensemble's stream;
//   OBL_ENS_PERSISTENT  one cooperative launch of the persistent kernel over the work
//                       list of all instances (ensemble.cuh), phases separated by grid
//                       barriers;
//   OBL_ENS_PERSISTENT_SPLIT  the same work list in three cooperative launches, one per
//                       register class (rows | columns + solve | x-inverse), so that the
//                       light phases run at a higher occupancy;
//   OBL_ENS_PERSISTENT_FLOW  one cooperative launch of the dataflow form (units from one
//                       counter, each waiting only for its own instance's previous phase).
// Any mode can be captured once into a CUDA graph and replayed.
struct obl_ensemble {
    int dev = 0;
    bool f64 = false;
    cudaStream_t stream = nullptr;
    std::vector<obl_ctx *> ctx;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> ev;          // [0] fork, [1..n] joins
    int mode = OBL_ENS_PERSISTENT;
    int bps = 0;                          // persistent CTAs per SM (0: all that fit)
    bool phase_stamps = false;            // record the phase boundaries of the persistent kernel
    // persistent mode
    DevBuf xpad, inst, start, bar, flow;
    std::vector<long long> xoff;          // element offset of each instance's 4 x-padded planes
    std::vector<obl_step_io> ios;         // the buffers the uploaded work list was built for
    size_t smem[3] = {0, 0, 0};           // per launch of the persistent step
    int blocks = 0;                       // 0: launch shape not built yet
    int nblk[3] = {0, 0, 0};
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<obl_step_io> graph_ios;
    int graph_mode = -1;
    std::string err;
};

namespace {
int efail(obl_ensemble *e, int code, const std::string &m)
{
    if (e) e->err = m;
    return code;
}
#define ECK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return efail(ens, OBL_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

bool same_ios(const std::vector<obl_step_io> &a, const obl_step_io *b, int n)
{
    return (int)a.size() == n && std::memcmp(a.data(), b, sizeof(obl_step_io) * (size_t)n) == 0;
}

int ens_ctx_fail(obl_ensemble *ens, int i, int rc)
{
    return efail(ens, rc, "instance " + std::to_string(i) + ": " + ens->ctx[i]->err);
}

// builds and uploads the work list of the persistent kernel for these buffers
// the launches of the persistent step: phase ranges and CTAs per SM of each
struct EnsPart {
    int pb, pe, minb;
};
static const EnsPart kEnsAll[1] = {{0, 6, OBL_ENS_MINB}};
static const EnsPart kEnsSplit[3] = {{0, 1, 2}, {1, 4, 4}, {4, 6, 2}};

static bool ens_persistent(int mode)
{
    return mode == OBL_ENS_PERSISTENT || mode == OBL_ENS_PERSISTENT_SPLIT || mode == OBL_ENS_PERSISTENT_FLOW;
}
template <typename T> static int ens_part_bps(const EnsPart &p, size_t smem, bool flow)
{
    if (flow) return EnsFlowKernel<T, OBL_ENS_MINB>::blocks_per_sm(smem);
    if (p.pb == 0 && p.pe == 6) return EnsKernel<T, 0, 6, OBL_ENS_MINB>::blocks_per_sm(smem);
    if (p.pb == 0) return EnsKernel<T, 0, 1, 2>::blocks_per_sm(smem);
    if (p.pb == 1) return EnsKernel<T, 1, 4, 4>::blocks_per_sm(smem);
    return EnsKernel<T, 4, 6, 2>::blocks_per_sm(smem);
}
template <typename T> static cudaError_t ens_part_launch(const EnsPart &p, const EnsArgs<T> &a, int blocks, size_t smem,
                                                        cudaStream_t s, bool flow)
{
    if (flow) return EnsFlowKernel<T, OBL_ENS_MINB>::launch(a, blocks, smem, s);
    if (p.pb == 0 && p.pe == 6) return EnsKernel<T, 0, 6, OBL_ENS_MINB>::launch(a, blocks, smem, s);
    if (p.pb == 0) return EnsKernel<T, 0, 1, 2>::launch(a, blocks, smem, s);
    if (p.pb == 1) return EnsKernel<T, 1, 4, 4>::launch(a, blocks, smem, s);
    return EnsKernel<T, 4, 6, 2>::launch(a, blocks, smem, s);
}

// builds and uploads the work list of the persistent kernel for these buffers
template <typename T> int ens_prepare(obl_ensemble *ens, const obl_step_io *ios)
{
    const int n = (int)ens->ctx.size();
    if (same_ios(ens->ios, ios, n) && ens->blocks > 0) return OBL_OK;
    int rc;
    std::vector<EnsInst<T>> h(n);
    for (int i = 0; i < n; ++i) {
        if (ios[i].divtz_bot || ios[i].divtz_top)
            return efail(ens, OBL_ERR_UNSUPPORTED, "persistent ensemble: divtz planes must be NULL (zero)");
        Ops<T> o{ens->ctx[i]};
        if ((rc = o.ens_inst(&ios[i], (T *)ens->xpad.p + ens->xoff[i], h[i]))) return ens_ctx_fail(ens, i, rc);
    }
    std::vector<long long> st((size_t)kEnsPhases * (n + 1), 0);
    for (int p = 0; p < kEnsPhases; ++p)
        for (int i = 0; i < n; ++i) st[(size_t)p * (n + 1) + i + 1] = st[(size_t)p * (n + 1) + i] + h[i].count[p];
    if ((rc = ensure(ens->ctx[0], ens->inst, sizeof(EnsInst<T>) * (size_t)n))) return ens_ctx_fail(ens, 0, rc);
    if ((rc = ensure(ens->ctx[0], ens->start, sizeof(long long) * st.size()))) return ens_ctx_fail(ens, 0, rc);
    if ((rc = ensure(ens->ctx[0], ens->flow, sizeof(unsigned) * (1 + (size_t)n * kEnsPhases))))
        return ens_ctx_fail(ens, 0, rc);
    ECK(cudaMemcpyAsync(ens->inst.p, h.data(), sizeof(EnsInst<T>) * (size_t)n, cudaMemcpyHostToDevice, ens->stream));
    ECK(cudaMemcpyAsync(ens->start.p, st.data(), sizeof(long long) * st.size(), cudaMemcpyHostToDevice, ens->stream));
    ECK(cudaStreamSynchronize(ens->stream));
    int nsm = 0;
    ECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ens->dev));
    const bool split = ens->mode == OBL_ENS_PERSISTENT_SPLIT;
    const EnsPart *parts = split ? kEnsSplit : kEnsAll;
    for (int k = 0; k < (split ? 3 : 1); ++k) {
        size_t smem = 0;
        for (int i = 0; i < n; ++i)
            smem = std::max(smem, EnsGeoHost<T>::smem(ens->ctx[i]->nxt, ens->ctx[i]->nyt, parts[k].pb, parts[k].pe));
        int per = ens_part_bps<T>(parts[k], smem, ens->mode == OBL_ENS_PERSISTENT_FLOW);
        if (per <= 0) return efail(ens, OBL_ERR_UNSUPPORTED, "persistent ensemble kernel cannot be resident");
        if (ens->bps > 0 && ens->bps < per) per = ens->bps;
        ens->smem[k] = smem;
        ens->nblk[k] = per * nsm;
    }
    ens->blocks = ens->nblk[0];
    ens->ios.assign(ios, ios + n);
    return OBL_OK;
}

template <typename T> int ens_step_t(obl_ensemble *ens, const obl_step_io *ios)
{
    const int n = (int)ens->ctx.size();
    int rc;
    if (ens_persistent(ens->mode)) {
        if ((rc = ens_prepare<T>(ens, ios))) return rc;
        const bool flow = ens->mode == OBL_ENS_PERSISTENT_FLOW;
        EnsArgs<T> a{(const EnsInst<T> *)ens->inst.p, n, (const long long *)ens->start.p, (unsigned *)ens->bar.p,
                     (int *)((unsigned *)ens->bar.p + 2),
                     ens->phase_stamps && !flow ? (unsigned long long *)((unsigned *)ens->bar.p + 4) : nullptr,
                     (unsigned *)ens->flow.p};
        const bool split = ens->mode == OBL_ENS_PERSISTENT_SPLIT;
        for (int k = 0; k < (split ? 3 : 1); ++k) {
            if (flow) ECK(cudaMemsetAsync(ens->flow.p, 0, sizeof(unsigned) * (1 + (size_t)n * kEnsPhases), ens->stream));
            else ECK(cudaMemsetAsync(ens->bar.p, 0, 2 * sizeof(unsigned), ens->stream));
            LaunchScope ls(ens->ctx[0]->rec, "ensemble_persistent", ens->stream);
            ECK(ens_part_launch<T>((split ? kEnsSplit : kEnsAll)[k], a, ens->nblk[k], ens->smem[k], ens->stream, flow));
        }
        return OBL_OK;
    }
    const bool conc = ens->mode == OBL_ENS_CONCURRENT;
    if (conc) ECK(cudaEventRecord(ens->ev[0], ens->stream));
    for (int i = 0; i < n; ++i) {
        obl_ctx *c = ens->ctx[i];
        c->stream = conc ? ens->streams[i] : ens->stream;
        if (conc) ECK(cudaStreamWaitEvent(c->stream, ens->ev[0], 0));
        Ops<T> o{c};
        if ((rc = o.step(&ios[i]))) return ens_ctx_fail(ens, i, rc);
        if (conc) {
            ECK(cudaEventRecord(ens->ev[1 + i], c->stream));
            ECK(cudaStreamWaitEvent(ens->stream, ens->ev[1 + i], 0));
        }
    }
    return OBL_OK;
}

int ens_step(obl_ensemble *ens, const obl_step_io *ios)
{
    return ens->f64 ? ens_step_t<double>(ens, ios) : ens_step_t<float>(ens, ios);
}

void ens_drop_graph(obl_ensemble *ens)
{
    if (ens->exec) cudaGraphExecDestroy(ens->exec);
    if (ens->graph) cudaGraphDestroy(ens->graph);
    ens->exec = nullptr;
    ens->graph = nullptr;
    ens->graph_ios.clear();
    ens->graph_mode = -1;
}
} // namespace

extern "C" {

int obl_ensemble_create(const obl_grid *grids, int n, const obl_options *opt, obl_ensemble **out)
{
    if (!grids || n <= 0 || !out) return OBL_ERR_ARG;
    *out = nullptr;
    obl_ensemble *ens = new obl_ensemble();
    ens->dev = opt ? opt->device : 0;
    for (int i = 0; i < n; ++i) {
        obl_ctx *c = nullptr;
        int rc = obl_ctx_create(&grids[i], opt, &c);
        if (rc) {
            obl_ensemble_destroy(ens);
            return rc;
        }
        ens->ctx.push_back(c);
    }
    ens->f64 = ens->ctx[0]->f64;
    if (cudaSetDevice(ens->dev) != cudaSuccess || cudaStreamCreateWithFlags(&ens->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        obl_ensemble_destroy(ens);
        return OBL_ERR_CUDA;
    }
    ens->streams.resize(n, nullptr);
    ens->ev.resize(n + 1, nullptr);
    bool ok = true;
    for (int i = 0; i < n; ++i) {
        ok = ok && cudaStreamCreateWithFlags(&ens->streams[i], cudaStreamNonBlocking) == cudaSuccess;
        ens->ctx[i]->stream = ens->stream;
    }
    for (auto &e : ens->ev) ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
    // persistent mode: four x-padded planes per instance, barrier words
    size_t tot = 0;
    for (int i = 0; i < n && ok; ++i) {
        const obl_ctx *c = ens->ctx[i];
        ens->xoff.push_back((long long)tot);
        tot += (size_t)4 * c->nxt2 * c->nyt * (c->nz + 1);
        if (!ens_length_supported(c->nxt) || !ens_length_supported(c->nyt)) ens->mode = OBL_ENS_SEQUENTIAL;
    }
    ok = ok && ensure(ens->ctx[0], ens->xpad, ens->ctx[0]->es() * tot) == OBL_OK;
    // barrier words [0..1], error flag [2], phase stamps from [4] (8-byte aligned)
    const size_t barb = 4 * sizeof(unsigned) + (kEnsPhases + 1) * sizeof(unsigned long long);
    ok = ok && ensure(ens->ctx[0], ens->bar, barb) == OBL_OK;
    ok = ok && cudaMemset(ens->bar.p, 0, barb) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        obl_ensemble_destroy(ens);
        return OBL_ERR_NOMEM;
    }
    *out = ens;
    return OBL_OK;
}

int obl_ensemble_destroy(obl_ensemble *ens)
{
    if (!ens) return OBL_OK;
    cudaSetDevice(ens->dev);
    if (ens->stream) cudaStreamSynchronize(ens->stream);
    ens_drop_graph(ens);
    for (auto s : ens->streams)
        if (s) cudaStreamSynchronize(s), cudaStreamDestroy(s);
    for (auto e : ens->ev)
        if (e) cudaEventDestroy(e);
    for (auto c : ens->ctx) {
        c->stream = nullptr;
        obl_ctx_destroy(c);
    }
    cudaFree(ens->xpad.p);
    cudaFree(ens->inst.p);
    cudaFree(ens->start.p);
    cudaFree(ens->bar.p);
    cudaFree(ens->flow.p);
    if (ens->stream) cudaStreamDestroy(ens->stream);
    delete ens;
    return OBL_OK;
}

int obl_ensemble_size(const obl_ensemble *ens) { return ens ? (int)ens->ctx.size() : -1; }

int obl_ensemble_context(obl_ensemble *ens, int i, obl_ctx **ctx)
{
    if (!ens || !ctx || i < 0 || i >= (int)ens->ctx.size()) return OBL_ERR_ARG;
    *ctx = ens->ctx[i];
    return OBL_OK;
}

int obl_ensemble_set_mode(obl_ensemble *ens, int mode, int blocks_per_sm)
{
    if (!ens || mode < 0 || mode > OBL_ENS_PERSISTENT_FLOW || blocks_per_sm < 0) return OBL_ERR_ARG;
    if (ens_persistent(mode))
        for (auto c : ens->ctx)
            if (!ens_length_supported(c->nxt) || !ens_length_supported(c->nyt))
                return efail(ens, OBL_ERR_UNSUPPORTED, "persistent ensemble: line length " +
                                                           std::to_string(c->nxt) + "x" + std::to_string(c->nyt) +
                                                           " has no persistent-kernel instantiation");
    ens->mode = mode;
    ens->bps = blocks_per_sm;
    ens->blocks = 0;   // rebuild the launch shape on the next persistent step
    ens->ios.clear();
    for (auto c : ens->ctx) c->stream = ens->stream;
    return OBL_OK;
}

int obl_ensemble_get_mode(const obl_ensemble *ens, int *mode, int *blocks_per_sm, int *blocks)
{
    if (!ens) return OBL_ERR_ARG;
    if (mode) *mode = ens->mode;
    if (blocks_per_sm) *blocks_per_sm = ens->bps;
    if (blocks) *blocks = ens->blocks;
    return OBL_OK;
}

int obl_ensemble_step_dev(obl_ensemble *ens, const obl_step_io *ios)
{
    if (!ens || !ios) return OBL_ERR_ARG;
    for (size_t i = 0; i < ens->ctx.size(); ++i)
        if (!step_io_ok(&ios[i])) return efail(ens, OBL_ERR_ARG, "instance " + std::to_string(i) + ": missing buffer");
    if (cudaSetDevice(ens->dev) != cudaSuccess) return efail(ens, OBL_ERR_CUDA, "cudaSetDevice");
    return ens_step(ens, ios);
}

int obl_ensemble_capture_dev(obl_ensemble *ens, const obl_step_io *ios)
{
    if (!ens || !ios) return OBL_ERR_ARG;
    if (cudaSetDevice(ens->dev) != cudaSuccess) return efail(ens, OBL_ERR_CUDA, "cudaSetDevice");
    const int n = (int)ens->ctx.size();
    if (ens->exec && ens->graph_mode == ens->mode && same_ios(ens->graph_ios, ios, n)) return OBL_OK;
    ens_drop_graph(ens);
    // one uncaptured step first: every buffer is allocated and every table uploaded before
    // capture starts (nothing may allocate while a stream is being captured)
    int rc = obl_ensemble_step_dev(ens, ios);
    if (rc) return rc;
    ECK(cudaStreamSynchronize(ens->stream));
    const bool timing = ens->ctx[0]->rec.timing;
    for (auto c : ens->ctx) c->rec.timing = false;
    ECK(cudaStreamBeginCapture(ens->stream, cudaStreamCaptureModeThreadLocal));
    rc = ens_step(ens, ios);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(ens->stream, &g);
    for (auto c : ens->ctx) c->rec.timing = timing;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    ECK(ce);
    ens->graph = g;
    ECK(cudaGraphInstantiate(&ens->exec, g, 0));
    ens->graph_ios.assign(ios, ios + n);
    ens->graph_mode = ens->mode;
    return OBL_OK;
}

int obl_ensemble_replay(obl_ensemble *ens)
{
    if (!ens) return OBL_ERR_ARG;
    if (!ens->exec) return efail(ens, OBL_ERR_ARG, "no captured graph");
    if (cudaSetDevice(ens->dev) != cudaSuccess) return efail(ens, OBL_ERR_CUDA, "cudaSetDevice");
    ECK(cudaGraphLaunch(ens->exec, ens->stream));
    return OBL_OK;
}

int obl_ensemble_synchronize(obl_ensemble *ens)
{
    if (!ens) return OBL_ERR_ARG;
    if (cudaSetDevice(ens->dev) != cudaSuccess) return efail(ens, OBL_ERR_CUDA, "cudaSetDevice");
    ECK(cudaStreamSynchronize(ens->stream));
    int flag = 0;
    ECK(cudaMemcpy(&flag, (unsigned *)ens->bar.p + 2, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        cudaMemset((unsigned *)ens->bar.p + 2, 0, sizeof(int));
        return efail(ens, OBL_ERR_TIMEOUT, "persistent ensemble: a grid-barrier wait gave up");
    }
    return OBL_OK;
}

int obl_ensemble_time_dev(obl_ensemble *ens, const obl_step_io *ios, int use_graph, int warmup, int reps,
                          double *ms_per_step)
{
    if (!ens || !ios || reps <= 0 || warmup < 0 || !ms_per_step) return OBL_ERR_ARG;
    int rc;
    if (use_graph && (rc = obl_ensemble_capture_dev(ens, ios))) return rc;
    auto one = [&]() -> int { return use_graph ? obl_ensemble_replay(ens) : obl_ensemble_step_dev(ens, ios); };
    for (int i = 0; i < warmup; ++i)
        if ((rc = one())) return rc;
    if ((rc = obl_ensemble_synchronize(ens))) return rc;
    cudaEvent_t a, b;
    ECK(cudaEventCreate(&a));
    ECK(cudaEventCreate(&b));
    ECK(cudaEventRecord(a, ens->stream));
    for (int i = 0; i < reps && !rc; ++i) rc = one();
    ECK(cudaEventRecord(b, ens->stream));
    const int rs = obl_ensemble_synchronize(ens);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    if (rs) return rs;
    *ms_per_step = (double)ms / reps;
    return OBL_OK;
}

int obl_ensemble_phase_times(obl_ensemble *ens, int on, double *ms, int n)
{
    if (!ens) return OBL_ERR_ARG;
    ens->phase_stamps = on != 0;
    if (!ms) return OBL_OK;
    if (n < kEnsPhases) return efail(ens, OBL_ERR_ARG, "phase_times: need room for every phase");
    if (cudaSetDevice(ens->dev) != cudaSuccess) return efail(ens, OBL_ERR_CUDA, "cudaSetDevice");
    unsigned long long t[kEnsPhases + 1];
    ECK(cudaStreamSynchronize(ens->stream));
    ECK(cudaMemcpy(t, (unsigned *)ens->bar.p + 4, sizeof t, cudaMemcpyDeviceToHost));
    for (int i = 0; i < kEnsPhases; ++i) ms[i] = (double)(t[i + 1] - t[i]) * 1e-6;
    return OBL_OK;
}

int obl_ensemble_last_error(const obl_ensemble *ens, char *buf, size_t n)
{
    if (!ens || !buf || n == 0) return OBL_ERR_ARG;
    std::strncpy(buf, ens->err.c_str(), n - 1);
    buf[n - 1] = 0;
    return OBL_OK;
}

} // extern "C"

// ============================================================================= z-slab step
static int slab_check(obl_ctx *ctx, int rank, int nranks)
{
    if (nranks < 1 || nranks > kSlabMaxRanks || rank < 0 || rank >= nranks)
        return fail(ctx, OBL_ERR_ARG, "slab: need 0 <= rank < nranks <= " + std::to_string(kSlabMaxRanks));
    if (ctx->opt.top_bc != OBL_TOP_NEUMANN)
        return fail(ctx, OBL_ERR_UNSUPPORTED, "slab: a split domain has the npz >= 2 top (OBL_TOP_NEUMANN)");
    if (ctx->L < 2) return fail(ctx, OBL_ERR_UNSUPPORTED, "slab: needs at least 2 levels per rank");
    return OBL_OK;
}

extern "C" {

int obl_slab_sizes(obl_ctx *ctx, long long *plane_bytes, long long *iface_bytes)
{
    if (!ctx) return OBL_ERR_ARG;
    if (plane_bytes) *plane_bytes = (long long)(ctx->f64 ? sizeof(double2) : sizeof(float2)) * ctx->sp();
    if (iface_bytes) *iface_bytes = (long long)sizeof(double) * kSlabIface * ctx->sp();
    return OBL_OK;
}

int obl_slab_begin_dev(obl_ctx *ctx, const obl_step_io *io, int rank, int nranks, void *plane_out)
{
    if (!ctx || !step_io_ok(io) || !plane_out) return OBL_ERR_ARG;
    if (int rc = slab_check(ctx, rank, nranks)) return rc;
    DEVCALL(ctx, return o.slab_begin(io, rank, nranks, (C2<T> *)plane_out););
}

int obl_slab_solve_dev(obl_ctx *ctx, const void *plane_above, int rank, int nranks, void *iface_out)
{
    if (!ctx || !iface_out) return OBL_ERR_ARG;
    if (int rc = slab_check(ctx, rank, nranks)) return rc;
    if (rank < nranks - 1 && !plane_above) return fail(ctx, OBL_ERR_ARG, "slab: the plane of the rank above is missing");
    DEVCALL(ctx, return o.slab_solve((const C2<T> *)plane_above, rank, nranks, (double *)iface_out););
}

int obl_slab_finish_dev(obl_ctx *ctx, const obl_step_io *io, const void *iface_all, int rank, int nranks)
{
    if (!ctx || !step_io_ok(io) || !iface_all) return OBL_ERR_ARG;
    if (int rc = slab_check(ctx, rank, nranks)) return rc;
    DEVCALL(ctx, return o.slab_finish(io, (const double *)iface_all, rank, nranks););
}

} // extern "C"
