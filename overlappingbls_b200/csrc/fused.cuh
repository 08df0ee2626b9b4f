// fused.cuh -- cluster-fused plane kernels of the projection-plus-derivative step.
//
// The separable line kernels move every intermediate through HBM: the x-padded plane of
// zero_padding, the x spectrum of the pressure RHS, and a second read of each field for
// ddy.  Here one thread-block cluster owns one (field, level) plane at a time:
//
//   row phase    each row pair is read once and transformed once along x; from that one
//                spectrum the warp produces ddx (written out), the x-padded rows and the
//                scaled x half-spectra of the RHS (both into the cluster's scratch slot);
//   cluster.sync
//   column phase column tiles of the x-padded plane are y-padded (written out), column
//                tiles of the field give ddy (the plane was just read, so it comes from L2),
//                and column tiles of the x spectrum are y-transformed into H_x, H_y, H_z;
//   cluster.sync before the slot is reused for the next plane.
//
// The scratch slot of a cluster (x-padded plane + x spectrum, ~2.5 MB for a 512^2 FP32
// plane) is rewritten before it is read on every plane and stays in L2 while the
// cluster works on it, so only the compulsory reads and writes reach HBM: this is the
// on-GPU replacement of the pencil transposes of zero_padding and fftn_mpi
// (108_01_padd.f90:114,129; 203_fftn_mpi.f90:27).
#pragma once
#include <cooperative_groups.h>

#include "lines.cuh"

namespace obl {

namespace cg = cooperative_groups;

template <typename T> struct FwdFusedArgs {
    const T *f[4];          // u, v, w, theta: (ldx, ny, nlev)
    T *d[8];                // dudx, dudy, dvdx, dvdy, dwdx, dwdy, dtdx, dtdy
    T *big[4];              // (nx2, ny2, nlev)
    C2<T> *H[3];            // RHS spectra of u, v, w: (lhx, ny, nlev), levels 1..L written
    unsigned char *scr;     // cluster scratch slots
    long long slot_bytes;
    int ldx, nlev, L, nfields;
    double sc_press;        // const/(tadv1*dt) (109_press_stag_array.f90:166-168)
    const double *kx;       // kx(lhx) (ddx)
    const double *ky;       // ky(lhy) (ddy)
    const C2<T> *twF, *twB, *twPB;   // plans: forward N, backward N, padded backward 3N/2
};

// fused row work of one row pair: ddx, x-pad and (optionally) the scaled half spectra
template <typename T, int N>
__device__ __forceinline__ void row_fwd_fused(const T *A, const T *B, T *dA, T *dB, T *pA, T *pB, C2<T> *sA,
                                              C2<T> *sB, bool act, bool spec, double sc_press,
                                              const double *kx, const C2<T> *twF, const C2<T> *twB,
                                              const C2<T> *twPB, C2<T> *scr_line, int t)
{
    using C = C2<T>;
    using DD = LineDerived<N, OP_DERIV>;
    using DP = LineDerived<N, OP_PAD>;
    constexpr int LL = DD::LL;
    static_assert(DP::LL == LL, "deriv and pad chains must share the lane layout");
    constexpr int VD = DD::VR, VP = DP::VR;
    constexpr int RF0 = DD::RF0, RFL = DD::RFL, RPL = DP::RBL;
    constexpr int N2 = 3 * N / 2;
    LineScratch<C> sc{scr_line};
    const T scale = (T)1 / (T)N;

    T ca = 0, cb = 0;
    if (act) { ca = A[0]; cb = B[0]; }
    C v[VD > VP ? VD : VP];
    {
        using G = Geo<N, RF0, LL>;
#pragma unroll
        for (int b = 0; b < G::PER; ++b) {
            const int j = t + LL * b;
#pragma unroll
            for (int r = 0; r < RF0; ++r) {
                const int i = j + r * G::NB;
                C z = mk<T>(0, 0);
                if (act && (G::FULL || j < G::NB)) z = mk<T>((A[i] - ca) * scale, (B[i] - cb) * scale);
                v[b * RF0 + r] = z;
            }
        }
    }
    fft_regs<N, typename DD::PF, LL, true>(v, sc, twF, t);   // v = FFT((x - c)/N), layout D(RFL)

    // (1) half spectra of the RHS: FFT(sc * x) = N*sc*v + sc*c*N at DC, x-Nyquist zeroed
    if (spec) {
        using G = Geo<N, RFL, LL>;
#pragma unroll
        for (int b = 0; b < G::PER; ++b) {
            const int j = t + LL * b;
            if (G::FULL || j < G::NB)
#pragma unroll
                for (int r = 0; r < RFL; ++r) sc.st(j + r * G::NB, v[b * RFL + r]);
        }
        __syncwarp();
        const T f = (T)((double)N * sc_press);
        constexpr int H = N / 2;
        for (int k = t; k <= H; k += LL) {
            C ao = mk<T>(0, 0), bo = mk<T>(0, 0);
            if (k < H) {
                const C z = sc.ld(k), zc = cconj(sc.ld(k == 0 ? 0 : N - k));
                const C s = cadd(z, zc), d = csub(z, zc);
                ao = mk<T>((T)0.5 * f * s.x, (T)0.5 * f * s.y);
                bo = mk<T>((T)0.5 * f * d.y, (T)-0.5 * f * d.x);
                if (k == 0) {
                    ao.x += (T)(sc_press * (double)N) * ca;
                    bo.x += (T)(sc_press * (double)N) * cb;
                }
            }
            if (act) {
                sA[k] = ao;
                sB[k] = bo;
            }
        }
        __syncwarp();
    }
    // (2) x-pad to 3N/2 (108_01_padd.f90:100-112)
    {
        C w[VP];
        reg_pad<T, N, RFL, LL>(v, w, t);
        fft_regs<N2, typename DP::PB, LL, false>(w, sc, twPB, t);
        using G = Geo<N2, RPL, LL>;
        if (act) {
#pragma unroll
            for (int b = 0; b < G::PER; ++b) {
                const int j = t + LL * b;
                if (G::FULL || j < G::NB)
#pragma unroll
                    for (int r = 0; r < RPL; ++r) {
                        const int i = j + r * G::NB;
                        pA[i] = w[b * RPL + r].x + ca;
                        pB[i] = w[b * RPL + r].y + cb;
                    }
            }
        }
    }
    // (3) ddx (004_derivatives.f90:33-39)
    {
        reg_deriv<T, N, RFL, LL>(v, kx, t);
        fft_regs<N, typename DD::PB, LL, false>(v, sc, twB, t);
        using G = Geo<N, DD::RBL, LL>;
        if (act) {
#pragma unroll
            for (int b = 0; b < G::PER; ++b) {
                const int j = t + LL * b;
                if (G::FULL || j < G::NB)
#pragma unroll
                    for (int r = 0; r < DD::RBL; ++r) {
                        const int i = j + r * G::NB;
                        dA[i] = v[b * DD::RBL + r].x;
                        dB[i] = v[b * DD::RBL + r].y;
                    }
            }
        }
    }
}

template <typename T, int N> struct FwdFusedGeo {
    using C = C2<T>;
    static constexpr int N2 = 3 * N / 2, LH = N / 2 + 1;
    using DD = LineDerived<N, OP_DERIV>;
    using DP = LineDerived<N, OP_PAD>;
    static constexpr int LPW = DD::LPW;
    static constexpr int TF = DD::TF, TB = DD::TB, TPB = DP::TB;
    static constexpr size_t row_scr = sizeof(C) * (size_t)8 * LPW * scratch_len(N2);
    static constexpr size_t tile_pad = sizeof(T) * (size_t)tile_rows(N2) * ColTile<T, true, DP::LPW>::S;
    static constexpr size_t tile_der = sizeof(T) * (size_t)tile_rows(N) * ColTile<T, true, DD::LPW>::S;
    static constexpr size_t tile_cpx = sizeof(C) * (size_t)tile_rows(N) * ColTile<T, false, DD::LPW>::S;
    static constexpr size_t work = row_scr > tile_pad ? (row_scr > tile_der ? (row_scr > tile_cpx ? row_scr : tile_cpx)
                                                                             : (tile_der > tile_cpx ? tile_der : tile_cpx))
                                                      : (tile_pad > tile_der ? (tile_pad > tile_cpx ? tile_pad : tile_cpx)
                                                                             : (tile_der > tile_cpx ? tile_der : tile_cpx));
    static constexpr size_t smem = sizeof(C) * ((size_t)TF + TB + TPB) + work;
    // scratch slot: x-padded plane (N2 x N reals) + x half spectrum (LH x N complex)
    static size_t slot_bytes() { return ((sizeof(T) * (size_t)N2 * N + 255) / 256) * 256 + sizeof(C) * (size_t)LH * N; }
};

template <typename T, int N>
__global__ void __launch_bounds__(256, 2) k_fwd_fused(FwdFusedArgs<T> a)
{
    using C = C2<T>;
    using GG = FwdFusedGeo<T, N>;
    using DD = typename GG::DD;
    using DP = typename GG::DP;
    constexpr int N2 = GG::N2, LH = GG::LH, LPW = GG::LPW;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank(), csize = (int)cl.num_blocks();
    const int cid = blockIdx.x / csize, ncl = gridDim.x / csize;

    extern __shared__ __align__(16) unsigned char smraw[];
    C *twF = reinterpret_cast<C *>(smraw);
    C *twB = twF + GG::TF;
    C *twPB = twB + GG::TB;
    unsigned char *work = reinterpret_cast<unsigned char *>(twPB + GG::TPB);
    for (int i = threadIdx.x; i < GG::TF; i += blockDim.x) twF[i] = a.twF[i];
    for (int i = threadIdx.x; i < GG::TB; i += blockDim.x) twB[i] = a.twB[i];
    for (int i = threadIdx.x; i < GG::TPB; i += blockDim.x) twPB[i] = a.twPB[i];
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / DD::LL, t = lane % DD::LL;
    const long long pl = (long long)a.ldx * N, plb = (long long)N2 * N2, sp = (long long)LH * N;
    T *xpad = reinterpret_cast<T *>(a.scr + (long long)cid * a.slot_bytes);
    C *xspec = reinterpret_cast<C *>(a.scr + (long long)cid * a.slot_bytes +
                                      ((sizeof(T) * (size_t)N2 * N + 255) / 256) * 256);
    const int nitems = a.nfields * a.nlev;

    for (int item = cid; item < nitems; item += ncl) {
        const int fi = item / a.nlev, z = item - fi * a.nlev;
        const bool spec = fi < 3 && z >= 1 && z <= a.L;
        const T *fz = a.f[fi] + pl * z;
        // ---- row phase: pairs distributed over the warps of the cluster
        {
            C *scr_line = reinterpret_cast<C *>(work) + (warp * LPW + g) * scratch_len(N2);
            const int wg = rank * 8 + warp, nwg = csize * 8;
            for (int p0 = wg * LPW; p0 < N / 2; p0 += nwg * LPW) {
                const int p = p0 + g;
                const bool act = p < N / 2;
                const int y0 = 2 * (act ? p : 0);
                const T *A = fz + (long long)y0 * a.ldx;
                T *dA = a.d[2 * fi] + pl * z + (long long)y0 * a.ldx;
                T *pA = xpad + (long long)y0 * N2;
                C *sA = xspec + (long long)y0 * LH;
                row_fwd_fused<T, N>(A, A + a.ldx, dA, dA + a.ldx, pA, pA + N2, sA, sA + LH, act, spec, a.sc_press,
                                    a.kx, twF, twB, twPB, scr_line, t);
            }
        }
        cl.sync();
        // ---- column phase: y-pad tiles, ddy tiles, RHS y-transform tiles
        {
            constexpr int WP = ColTile<T, true, DP::LPW>::W, WD = ColTile<T, true, DD::LPW>::W;
            constexpr int WC = ColTile<T, false, DD::LPW>::W;
            const int np = (N2 + WP - 1) / WP, nd = (N + WD - 1) / WD, ns = spec ? (LH + WC - 1) / WC : 0;
            for (int task = rank; task < np + nd + ns; task += csize) {
                if (task < np) {
                    ColArgs<T> ca{};
                    ca.src = xpad; ca.dst = a.big[fi] + plb * z; ca.src_row = N2; ca.dst_row = N2;
                    ca.ncols = N2; ca.nlev = 1; ca.scale = (T)1 / (T)N;
                    ca.twF = twF; ca.twB = twPB;
                    col_unit<T, N, OP_PAD, true>(ca, 0, task, twF, twPB, reinterpret_cast<T *>(work));
                } else if (task < np + nd) {
                    ColArgs<T> ca{};
                    ca.src = fz; ca.dst = a.d[2 * fi + 1] + pl * z; ca.src_row = a.ldx; ca.dst_row = a.ldx;
                    ca.ncols = N; ca.nlev = 1; ca.scale = (T)1 / (T)N; ca.ktab = a.ky;
                    col_unit<T, N, OP_DERIV, true>(ca, 0, task - np, twF, twB, reinterpret_cast<T *>(work));
                } else {
                    ColArgs<T> ca{};
                    ca.src = xspec; ca.dst = a.H[fi] + sp * z; ca.src_row = LH; ca.dst_row = LH;
                    ca.ncols = LH; ca.nlev = 1; ca.scale = (T)1; ca.zero_nyq = 1;
                    col_unit<T, N, OP_FWD, false>(ca, 0, task - np - nd, twF, twB, reinterpret_cast<C *>(work));
                }
            }
        }
        cl.sync();
    }
}

// ----------------------------------------------------------------------------- multi-output rows
// One read of each row pair of a field yields ddx, the x-padded rows (zero_padding's
// first half, into the intermediate xpad) and, on levels 1..L of u, v, w, the scaled x
// half-spectra of the pressure RHS (written straight into H; the y transform then runs
// in place).  Replaces three separate row passes over the same field.
template <typename T> struct RowsFwd3Args {
    const T *src;          // field (ldx, ny, nlev)
    T *dfdx;               // (ldx, ny, nlev)
    T *xpad;               // (nx2, ny, nlev)
    C2<T> *H;              // (lhx, ny, nlev) or nullptr (theta)
    long long npairs;      // ny*nlev/2
    int ldx, ny, L;
    int z0;                // level of the first row pair (src, dfdx, H start there; a chunk of levels)
    double sc_press;
    const double *kx;
    const C2<T> *twF, *twB, *twPB;
};

// Unit u of the multi-output row pass: warp w of the CTA takes the LPW row pairs from
// (u*8 + w)*LPW.  Tables in shared memory; scr holds the 8*LPW per-line scratch lines.
// Called by k_rows_fwd3 (grid-stride over units) and by the persistent ensemble kernel.
template <typename T, int N>
__device__ __forceinline__ void rows_fwd3_unit(const RowsFwd3Args<T> &a, long long u, const C2<T> *twF,
                                               const C2<T> *twB, const C2<T> *twPB, C2<T> *scr)
{
    using C = C2<T>;
    using GG = FwdFusedGeo<T, N>;
    constexpr int N2 = GG::N2, LH = GG::LH, LPW = GG::LPW;
    constexpr int LL = GG::DD::LL;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int g = lane / LL, t = lane % LL;
    C *line = scr + (warp * LPW + g) * scratch_len(N2);
    {
        const long long base = (u * nw + warp) * LPW;
        if (base >= a.npairs) return;
        const long long p = base + g;
        const bool act = p < a.npairs;
        const long long r0 = 2 * (act ? p : base);
        // warp-uniform: the LPW pairs of a warp lie on one level (ny/2 is a multiple of LPW)
        const int zw = a.z0 + (int)((2 * base) / a.ny);
        bool spec = a.H != nullptr && zw >= 1 && zw <= a.L;
        // checked build: the pair lies in the launch's rows, on one level, and its RHS rows
        // in H's levels z0..L
        if (OBL_CHECK && !(ck_in(r0 + 1, 2 * a.npairs, CK_ROWS3_ROW) && ck_in(r0 % a.ny + 1, a.ny, CK_ROWS3_ROW)))
            return;
        if (OBL_CHECK && spec && !ck_in(r0 + 1, (long long)(a.L + 1 - a.z0) * a.ny, CK_ROWS3_SPEC)) spec = false;
        const T *A = a.src + r0 * a.ldx;
        T *dA = a.dfdx + r0 * a.ldx;
        T *pA = a.xpad + r0 * N2;
        C *sA = spec ? a.H + r0 * LH : nullptr;
        C *sB = spec ? a.H + (r0 + 1) * LH : nullptr;
        row_fwd_fused<T, N>(A, A + a.ldx, dA, dA + a.ldx, pA, pA + N2, sA, sB, act, spec, a.sc_press, a.kx,
                            twF, twB, twPB, line, t);
    }
}

template <typename T, int N>
__global__ void __launch_bounds__(256, 2) k_rows_fwd3(RowsFwd3Args<T> a)
{
    using C = C2<T>;
    using GG = FwdFusedGeo<T, N>;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *twF = reinterpret_cast<C *>(smraw);
    C *twB = twF + GG::TF;
    C *twPB = twB + GG::TB;
    C *scr = twPB + GG::TPB;
    for (int i = threadIdx.x; i < GG::TF; i += blockDim.x) twF[i] = a.twF[i];
    for (int i = threadIdx.x; i < GG::TB; i += blockDim.x) twB[i] = a.twB[i];
    for (int i = threadIdx.x; i < GG::TPB; i += blockDim.x) twPB[i] = a.twPB[i];
    __syncthreads();
    const long long per = (long long)(blockDim.x >> 5) * GG::LPW;
    for (long long u = blockIdx.x; u * per < a.npairs; u += gridDim.x) rows_fwd3_unit<T, N>(a, u, twF, twB, twPB, scr);
}

template <typename T> struct RowsFwd3Launch {
    static cudaError_t run(int n, const RowsFwd3Args<T> &a, cudaStream_t s);
};

// ----------------------------------------------------------------------------- fused inverse
// y-inverse of the pressure solution: one load of p_hat(z) gives the y-inverses of p_hat
// and i*ky*p_hat (109_press_stag_array.f90:231-238), one load of the dpdz spectrum gives
// its y-inverse; i*kx*p_hat is formed from the y-inverse of p_hat by the row pass.  Level
// 0 only needs p.  Line-minor column layout.
template <typename T> struct PinvColArgs {
    const C2<T> *ph, *dph;                // (lhx, ny, 0..L) spectra
    C2<T> *Xp, *Xdy, *Xdz;                // y-inverses of p_hat, i*ky*p_hat, dpdz spectrum
    long long S;                          // lhx*ny
    int lhx;
    const double *kx, *ky;                // kx(lhx), ky_2d row (ny)
    const C2<T> *twB;
};

// One CTA unit: line group bx of level z (twB in shared memory, buf = N*WB scratch).
template <typename T, int N, int NW = 8>
__device__ __forceinline__ void pinv_cols_unit(const PinvColArgs<T> &a, int bx, int z, const C2<T> *twB, C2<T> *buf)
{
    using C = C2<T>;
    using D = LineDerived<N, OP_INV>;
    using G = LmGeo<T, NW>;
    constexpr int WB = G::WB, LL = G::LL, VR = ColDerived<T, N, OP_INV, NW>::VR;
    constexpr int R0 = D::RB0, RL = D::RBL;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int line = lane % WB, t = lane / WB + (32 / WB) * warp;
    const int gl = bx * WB + line;
    const bool act = gl < a.lhx;
    const int glc = act ? gl : 0;
    LineMinor<C, WB> sc{buf, line};
    using G0 = Geo<N, R0, LL>;
    using GL = Geo<N, RL, LL>;
    auto load = [&](const C *src, C *v) {
#pragma unroll
        for (int b = 0; b < G0::PER; ++b) {
            const int j = t + LL * b;
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int i = j + r * G0::NB;
                v[b * R0 + r] = (act && (G0::FULL || j < G0::NB) &&
                                 ck_in((long long)i * a.lhx + glc, a.S, CK_PINV_COL_LOAD))
                                    ? __ldcg(src + a.S * z + (long long)i * a.lhx + glc)
                                    : mk<T>(0, 0);
            }
        }
    };
    auto store = [&](C *dst, const C *v) {
        if (!act) return;
#pragma unroll
        for (int b = 0; b < GL::PER; ++b) {
            const int j = t + LL * b;
            if (GL::FULL || j < GL::NB)
#pragma unroll
                for (int r = 0; r < RL; ++r)
                    if (ck_in((long long)(j + r * GL::NB) * a.lhx + gl, a.S, CK_PINV_COL_STORE))
                        dst[a.S * z + (long long)(j + r * GL::NB) * a.lhx + gl] = v[b * RL + r];
        }
    };
    C v[VR], w[VR];
    load(a.ph, v);
    // i*ky(row) and i*kx(col) multipliers act element-wise on the loaded layout
#pragma unroll
    for (int q = 0; q < VR; ++q) w[q] = v[q];
    fft_regs<N, typename D::PB, LL, false, true>(w, sc, twB, t);
    store(a.Xp, w);
    if (z == 0) return;   // uniform per block
    // i*kx p_hat needs no transform of its own: kx is constant along y, so its y-inverse
    // is i*kx times that of p_hat, applied by the x-inverse row pass when it loads Xp
#pragma unroll
    for (int b = 0; b < G0::PER; ++b) {
        const int j = t + LL * b;
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const int i = (G0::FULL || j < G0::NB) ? j + r * G0::NB : 0;
            const T kyv = (T)a.ky[i];
            const C x = v[b * R0 + r];
            w[b * R0 + r] = mk<T>(-kyv * x.y, kyv * x.x);
        }
    }
    fft_regs<N, typename D::PB, LL, false, true>(w, sc, twB, t);
    store(a.Xdy, w);
    load(a.dph, w);
    fft_regs<N, typename D::PB, LL, false, true>(w, sc, twB, t);
    store(a.Xdz, w);
}

template <typename T, int N, int NW, bool TWG = false>
__global__ void __launch_bounds__(32 * NW, TWG ? 4 : 2) k_cols_pinv(PinvColArgs<T> a)
{
    using C = C2<T>;
    using D = LineDerived<N, OP_INV>;
    extern __shared__ __align__(16) unsigned char smraw[];
    if constexpr (TWG) {   // twiddles through L1 (see col_tw_global)
        pinv_cols_unit<T, N, NW>(a, blockIdx.x, blockIdx.y, a.twB, reinterpret_cast<C *>(smraw));
    } else {
        C *twB = reinterpret_cast<C *>(smraw);
        C *buf = twB + D::TB;
        for (int i = threadIdx.x; i < D::TB; i += blockDim.x) twB[i] = a.twB[i];
        __syncthreads();
        pinv_cols_unit<T, N, NW>(a, blockIdx.x, blockIdx.y, twB, buf);
    }
}

// x-inverse of the four y-inverses and the projection (110_project.f90:16-40) in one
// pass over the rows: p at levels 0..L, dpdx/dpdy/dpdz at 1..L (slot z-1), and
// u,v (levels 1..L) and w (levels 2..L) += dt*(-tadv1*grad p).
template <typename T> struct PinvRowArgs {
    const C2<T> *Xp, *Xdy, *Xdz;          // (lhx, ny, 0..L); dpdx's is i*kx*Xp
    const double *kx;                     // kx(lhx), Nyquist entry 0
    T *p, *dpdx, *dpdy, *dpdz;            // p (ldx, ny, 0:nz); d* (ldx, ny, 1:nz)
    T *u, *v, *w;                         // updated in place (ldx, ny, 0:nz)
    long long npairs;                     // ny*(L+1)/2
    int ldx, ny, lhx;
    T dt_tadv1;                           // dt*tadv1
    const C2<T> *twB;
    int w_from_1;                         // 0: w updated from level 2 (bottom rank, jz_min = 2);
                                          // 1: from level 1 (the z-slab of a rank above it)
};

// Unit u: warp w takes work item u*8 + w (twB in shared memory, scr = 8*LPW lines).
template <typename T, int N>
__device__ __forceinline__ void pinv_rows_unit(const PinvRowArgs<T> &a, long long u, const C2<T> *twB, C2<T> *scr)
{
    using C = C2<T>;
    using D = LineDerived<N, OP_INV>;
    constexpr int LL = D::LL, LPW = D::LPW, VR = D::VR, R0 = D::RB0, RL = D::RBL;
    constexpr int SL = scratch_len(N);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int g = lane / LL, t = lane % LL;
    LineScratch<C> sc{scr + (warp * LPW + g) * SL};
    using G0 = Geo<N, R0, LL>;
    using GL = Geo<N, RL, LL>;
    const long long pl = (long long)a.ldx * a.ny;
    const long long ngroups = (a.npairs + LPW - 1) / LPW;
    // work item wi: component q = wi % 4 (0: p; 1: dpdx and u; 2: dpdy and v; 3: dpdz and w)
    // of the LPW row pairs of group wi / 4.  Independent items keep many row transforms in
    // flight per SM instead of four dependent ones per warp.
    {
        const long long wi = u * nw + warp;
        if (wi >= 4 * ngroups) return;
        const int q = (int)(wi % 4);
        const long long base = (wi / 4) * LPW;
        const long long pr = base + g;
        const bool act = pr < a.npairs;
        const long long r0 = 2 * (act ? pr : base);
        const int z = (int)((2 * base) / a.ny);            // warp-uniform level
        if (q > 0 && z == 0) return;                       // level 0 holds p only
        // checked build: the pair lies in the launch's rows and on one level
        if (OBL_CHECK && !(ck_in(r0 + 1, 2 * a.npairs, CK_PINV_ROW) && ck_in(r0 % a.ny + 1, a.ny, CK_PINV_ROW)))
            return;
        const long long off = (r0 % a.ny) * a.ldx;
        const C *X = q <= 1 ? a.Xp : q == 2 ? a.Xdy : a.Xdz;
        T *out = q == 0 ? a.p + pl * z + off : (q == 1 ? a.dpdx : q == 2 ? a.dpdy : a.dpdz) + pl * (z - 1) + off;
        T *f = (q == 1 ? a.u : q == 2 ? a.v : a.w) + pl * z + off;
        const bool proj = q == 1 || q == 2 || (q == 3 && z >= (a.w_from_1 ? 1 : 2));   // jz_min for w
        // the two rows of the field to update are read before the transform
        T fa[GL::PER * RL], fb[GL::PER * RL];
#pragma unroll
        for (int b = 0; b < GL::PER; ++b) {
            const int j = t + LL * b;
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const int i = j + r * GL::NB;
                const bool ok = proj && act && (GL::FULL || j < GL::NB);
                fa[b * RL + r] = ok ? f[i] : (T)0;
                fb[b * RL + r] = ok ? f[a.ldx + i] : (T)0;
            }
        }
        // two Hermitian half spectra (rows r0, r0+1 of X) -> Z = A + iB, Im of DC/Nyquist ignored
        C v[VR];
        {
            const C *A = X + r0 * a.lhx;
            const C *B = A + a.lhx;
#pragma unroll
            for (int b = 0; b < G0::PER; ++b) {
                const int j = t + LL * b;
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                    const int i = j + r * G0::NB;
                    C zz = mk<T>(0, 0);
                    if (act && (G0::FULL || j < G0::NB)) {
                        const bool lo = i <= N / 2;
                        const int k = lo ? i : N - i;
                        C av = __ldcg(A + k), bv = __ldcg(B + k);
                        if (k == 0 || k == N / 2) { av.y = 0; bv.y = 0; }
                        zz = lo ? mk<T>(av.x - bv.y, av.y + bv.x) : mk<T>(av.x + bv.y, bv.x - av.y);
                    }
                    v[b * R0 + r] = zz;
                }
            }
        }
        // dpdx: i*kx times the y-inverse of p_hat.  On the two Hermitian rows packed as
        // Z = A + iB that is i*k_signed*Z (k_signed = kx(k) for bins k <= N/2, -kx(N-k)
        // above), the multiplier of the x-derivative, applied after the loads
        if (q == 1) reg_deriv<T, N, R0, LL>(v, a.kx, t);
        fft_regs<N, typename D::PB, LL, false>(v, sc, twB, t);
        if (act) {
#pragma unroll
            for (int b = 0; b < GL::PER; ++b) {
                const int j = t + LL * b;
                if (GL::FULL || j < GL::NB)
#pragma unroll
                    for (int r = 0; r < RL; ++r) {
                        const int i = j + r * GL::NB;
                        const C x = v[b * RL + r];
                        out[i] = x.x;
                        out[a.ldx + i] = x.y;
                        if (proj) {   // 110_project.f90:16-40: u = u + dt*(-tadv1*dpdx)
                            f[i] = fa[b * RL + r] + (-a.dt_tadv1 * x.x);
                            f[a.ldx + i] = fb[b * RL + r] + (-a.dt_tadv1 * x.y);
                        }
                    }
            }
        }
    }
}

template <typename T, int N>
__global__ void __launch_bounds__(256, 2) k_rows_pinv(PinvRowArgs<T> a)
{
    using C = C2<T>;
    using D = LineDerived<N, OP_INV>;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *twB = reinterpret_cast<C *>(smraw);
    C *scr = twB + D::TB;
    for (int i = threadIdx.x; i < D::TB; i += blockDim.x) twB[i] = a.twB[i];
    __syncthreads();
    const long long ngroups = (a.npairs + D::LPW - 1) / D::LPW;
    const long long nunits = (4 * ngroups + (blockDim.x >> 5) - 1) / (blockDim.x >> 5);
    for (long long u = blockIdx.x; u < nunits; u += gridDim.x) pinv_rows_unit<T, N>(a, u, twB, scr);
}
template <typename T> struct PinvLaunch {
    static cudaError_t cols(int n, const PinvColArgs<T> &a, int nlev, cudaStream_t s);
    static cudaError_t rows(int n, const PinvRowArgs<T> &a, cudaStream_t s);
};

template <typename T> struct FwdFusedLaunch {
    // returns cudaErrorNotSupported for lengths without an instantiation
    static cudaError_t run(int n, const FwdFusedArgs<T> &a, int nclusters, int csize, cudaStream_t s);
    static size_t slot_bytes(int n);
    static int max_clusters(int n, int csize);
};

} // namespace obl
