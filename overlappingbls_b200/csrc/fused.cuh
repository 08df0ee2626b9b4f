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

template <typename T> struct FwdFusedLaunch {
    // returns cudaErrorNotSupported for lengths without an instantiation
    static cudaError_t run(int n, const FwdFusedArgs<T> &a, int nclusters, int csize, cudaStream_t s);
    static size_t slot_bytes(int n);
    static int max_clusters(int n, int csize);
};

} // namespace obl
