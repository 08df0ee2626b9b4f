// lines.cuh -- batched 1D spectral line operations along x (rows) and y (columns).
//
// These kernels are the building blocks of every hot-path routine:
//   rows    (x direction, contiguous):  ddx, x-pad, x-unpad, x r2c, x c2r
//   columns (y direction, strided):     ddy, y-pad, y-unpad, y c2c forward/backward
// Real lines are transformed two at a time as one complex line (z = a + i b): every
// spectral operation used here is a real-to-real linear map acting on Z[k] and Z[N-k]
// symmetrically (i*k multipliers with signed k, truncation / zero extension), so
// Re(IFFT(op(FFT(z)))) = op(a) and Im(...) = op(b), exactly what the reference's
// per-line r2c -> op -> c2r computes (004_derivatives.f90:33-39,
// 108_01_padd.f90:102-127,163-190).
//
// Rows are loaded from global memory straight into registers in the layout of the
// first FFT pass; columns are staged through a shared-memory tile (the on-GPU
// replacement of the reference's mpi_alltoall pencil transposes,
// 203_fftn_mpi.f90:71-371) whose padded column doubles as the FFT exchange scratch.
//
// Accuracy: before a real line is transformed, its first value is subtracted (exact
// by Sterbenz's lemma for fields with a large mean such as theta ~ 300 K) and the
// scale is applied after the subtraction; derivatives ignore the constant, padding
// adds it back.  FP32 FFT errors then scale with the fluctuations, not with the mean.
#pragma once
#include <cuda.h>   // CUtensorMap and its enums (the encoder is reached through the runtime)
#include <cstdint>
#include <vector>

#include "async.cuh"
#include "fft2.cuh"

namespace obl {

enum LineOp : int { OP_DERIV = 0, OP_PAD = 1, OP_UNPAD = 2, OP_FWD = 3, OP_INV = 4 };
enum PlanRole : int { ROLE_FWD = 0, ROLE_BWD = 1, ROLE_PADFWD = 2, ROLE_PADBWD = 3 };

template <typename T> struct RowArgs {
    const void *src;          // real rows (DERIV/PAD/UNPAD/FWD) or complex rows (INV)
    void *dst;                // real rows (DERIV/PAD/UNPAD/INV) or complex rows (FWD)
    long long src_stride;     // elements (of the row's type) between consecutive rows
    long long dst_stride;
    long long npairs;         // number of row pairs (rows 2p, 2p+1)
    T scale;                  // multiplies the input at load
    const double *ktab;       // DERIV: k[0..N/2] (the Nyquist entry is 0)
    const C2<T> *twF, *twB;   // plan twiddle tables of the forward / backward transforms
    T pad_scale;              // INV with pad_mode: dst pad columns *= pad_scale
    int pad_mode;
};

template <typename T> struct ColArgs {
    const void *src;
    void *dst;
    long long src_row, dst_row;      // elements between rows
    long long src_plane, dst_plane;  // elements between planes
    int ncols;                       // real columns (real ops) / complex columns
    int nlev;
    T scale;                         // multiplies the input at load
    const double *ktab;              // DERIV: k[0..N/2]; INV kmul=1: kx per column; kmul=2: ky per row
    const C2<T> *twF, *twB;
    int pad_copy;                    // UNPAD: also write columns 0,1 into ncols, ncols+1
    int zero_nyq;                    // FWD: zero the Nyquist row (203_fftn_mpi.f90:33)
    int kmul;                        // INV: 0 none, 1 multiply by i*kx(col), 2 by i*ky(row)
    int pf_ahead;                    // the unit of plane z also prefetches its input lines of
                                     // plane z + pf_ahead into L2 (0 = none)
    int tma;                         // FP32 y-pad: input tile by tensor-map copies (k_cols2_tma)
    int *wait_err;                   // set to 1 when such a copy's bounded wait gave up
};

// ----------------------------------------------------------------------------- configuration
template <int N, int OP> struct LineCfg;
template <int N> struct LineCfg<N, OP_DERIV> {
    static constexpr int NI = N, NO = N;
    using PF = FwdPlan<N>;
    using PB = BwdPlan<N>;
};
template <int N> struct LineCfg<N, OP_PAD> {
    static constexpr int NI = N, NO = 3 * N / 2;
    using PF = FwdPlan<N>;
    using PB = PadBwdPlan<N>;
};
template <int N> struct LineCfg<N, OP_UNPAD> {
    static constexpr int NI = 3 * N / 2, NO = N;
    using PF = PadFwdPlan<N>;
    using PB = BwdPlan<N>;
};
template <int N> struct LineCfg<N, OP_FWD> : LineCfg<N, OP_DERIV> {};
template <int N> struct LineCfg<N, OP_INV> : LineCfg<N, OP_DERIV> {};

template <int N, int OP> struct LineDerived {
    using Cfg = LineCfg<N, OP>;
    static constexpr int NI = Cfg::NI, NO = Cfg::NO;
    using PF = typename Cfg::PF;
    using PB = typename Cfg::PB;
    static constexpr int llf = LL_<NI, PF>::v, llb = LL_<NO, PB>::v;
    static constexpr int LL = llf < llb ? llf : llb;
    static constexpr int LPW = 32 / LL;
    static constexpr int rf = Regs<NI, LL, PF>::v, rb = Regs<NO, LL, PB>::v;
    static constexpr int VR = rf > rb ? rf : rb;
    static constexpr int NM = NI > NO ? NI : NO;
    static constexpr int TF = tw_size<NI, PF>(), TB = tw_size<NO, PB>();
    static constexpr int RFL = PlanInfo<PF>::last, RB0 = PlanInfo<PB>::first;
    static constexpr int RF0 = PlanInfo<PF>::first, RBL = PlanInfo<PB>::last;
};

// ----------------------------------------------------------------------------- register ops
// v in D(R) of length N: v *= i*k_signed (ktab[N/2] = 0 drops the Nyquist mode)
template <typename T, int N, int R, int LL>
__device__ __forceinline__ void reg_deriv(C2<T> *v, const double *ktab, int t)
{
    using G = Geo<N, R, LL>;
#pragma unroll
    for (int b = 0; b < G::PER; ++b) {
        const int j = t + LL * b;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = j + r * G::NB;
            const int kc = (G::FULL || j < G::NB) ? k : 0;
            const T kk = (kc <= N / 2) ? (T)ktab[kc] : -(T)ktab[N - kc];
            const C2<T> z = v[b * R + r];
            v[b * R + r] = mk<T>(-kk * z.y, kk * z.x);
        }
    }
}

// D(R) of length N  ->  D(3R/2) of length 3N/2, zero-extended, Nyquist bin dropped
template <typename T, int N, int R, int LL>
__device__ __forceinline__ void reg_pad(const C2<T> *v, C2<T> *w, int t)
{
    using G = Geo<N, R, LL>;
    constexpr int R2 = 3 * R / 2, H = R / 2;
#pragma unroll
    for (int b = 0; b < G::PER; ++b) {
        const int j = t + LL * b;
#pragma unroll
        for (int r2 = 0; r2 < R2; ++r2) {
            C2<T> x = mk<T>(0, 0);
            if (r2 < H) x = v[b * R + r2];
            else if (r2 >= R) x = v[b * R + (r2 - H)];
            if (r2 == R && j == 0) x = mk<T>(0, 0);   // source bin N/2 (Nyquist)
            w[b * R2 + r2] = x;
        }
    }
}

// D(3R/2) of length 3N/2  ->  D(R) of length N, truncated, new Nyquist bin zero
template <typename T, int N, int R, int LL>
__device__ __forceinline__ void reg_unpad(const C2<T> *w, C2<T> *v, int t)
{
    using G = Geo<N, R, LL>;
    constexpr int R2 = 3 * R / 2, H = R / 2;
#pragma unroll
    for (int b = 0; b < G::PER; ++b) {
        const int j = t + LL * b;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            C2<T> x = (r < H) ? w[b * R2 + r] : w[b * R2 + r + H];
            if (r == H && j == 0) x = mk<T>(0, 0);     // bin N/2
            v[b * R + r] = x;
        }
    }
}

// ----------------------------------------------------------------------------- row kernel
// copy the plan twiddle tables an op needs into shared memory (caller syncs)
template <typename T, int N, int OP>
__device__ __forceinline__ void load_tables(const C2<T> *gF, const C2<T> *gB, C2<T> *sF, C2<T> *sB)
{
    using D = LineDerived<N, OP>;
    if (OP != OP_INV)
        for (int i = threadIdx.x; i < D::TF; i += blockDim.x) sF[i] = gF[i];
    if (OP != OP_FWD)
        for (int i = threadIdx.x; i < D::TB; i += blockDim.x) sB[i] = gB[i];
}

// One warp processes the LPW row pairs base .. base+LPW-1 (pairs at or beyond a.npairs
// idle).  twF/twB: the plan twiddle tables in shared memory; scr_warp: the warp's
// scratch lines (LPW * scratch_len(NM) complex).
template <typename T, int N, int OP>
__device__ __forceinline__ void row_unit(const RowArgs<T> &a, long long base, const C2<T> *twF,
                                         const C2<T> *twB, C2<T> *scr_warp, int lane)
{
    using C = C2<T>;
    using D = LineDerived<N, OP>;
    constexpr int NI = D::NI, NO = D::NO, LL = D::LL, VR = D::VR;
    constexpr int SL = scratch_len(D::NM);
    const int g = lane / LL, t = lane % LL;
    LineScratch<C> sc{scr_warp + g * SL};
    {
        const long long pr = base + g;
        const bool act = pr < a.npairs;
        const long long r0 = 2 * (act ? pr : 0);
        C v[VR];
        T ca = 0, cb = 0;
        if constexpr (OP == OP_INV) {
            // two Hermitian half spectra A (row r0), B (row r0+1) -> Z = A + iB on all N
            // bins; Im of the DC and Nyquist bins is ignored, as in FFTW's c2r
            using G = Geo<NO, D::RB0, LL>;
            const C *A = reinterpret_cast<const C *>(a.src) + r0 * a.src_stride;
            const C *B = A + a.src_stride;
#pragma unroll
            for (int b = 0; b < G::PER; ++b) {
                const int j = t + LL * b;
#pragma unroll
                for (int r = 0; r < D::RB0; ++r) {
                    const int i = j + r * G::NB;
                    C z = mk<T>(0, 0);
                    if (act && (G::FULL || j < G::NB)) {
                        const bool lo = i <= NO / 2;
                        const int k = lo ? i : NO - i;
                        C av = A[k], bv = B[k];
                        if (k == 0 || k == NO / 2) { av.y = 0; bv.y = 0; }
                        z = lo ? mk<T>(av.x - bv.y, av.y + bv.x) : mk<T>(av.x + bv.y, bv.x - av.y);
                    }
                    v[b * D::RB0 + r] = z;
                }
            }
        } else {
            using G = Geo<NI, D::RF0, LL>;
            const T *A = reinterpret_cast<const T *>(a.src) + r0 * a.src_stride;
            const T *B = A + a.src_stride;
            if (act) { ca = A[0]; cb = B[0]; }
#pragma unroll
            for (int b = 0; b < G::PER; ++b) {
                const int j = t + LL * b;
#pragma unroll
                for (int r = 0; r < D::RF0; ++r) {
                    const int i = j + r * G::NB;
                    C z = mk<T>(0, 0);
                    if (act && (G::FULL || j < G::NB)) z = mk<T>((A[i] - ca) * a.scale, (B[i] - cb) * a.scale);
                    v[b * D::RF0 + r] = z;
                }
            }
            fft_regs<NI, typename D::PF, LL, true>(v, sc, twF, t);
        }

        if constexpr (OP == OP_FWD) {
            // split Z into the half spectra of both rows; zero the x-Nyquist
            // (203_fftn_mpi.f90:25); the subtracted constants return in the DC bins
            using G = Geo<NI, D::RFL, LL>;
#pragma unroll
            for (int b = 0; b < G::PER; ++b) {
                const int j = t + LL * b;
                if (G::FULL || j < G::NB)
#pragma unroll
                    for (int r = 0; r < D::RFL; ++r) sc.st(j + r * G::NB, v[b * D::RFL + r]);
            }
            __syncwarp();
            C *Ao = reinterpret_cast<C *>(a.dst) + r0 * a.dst_stride;
            C *Bo = Ao + a.dst_stride;
            constexpr int H = NI / 2;
            for (int k = t; k <= H; k += LL) {
                C ao = mk<T>(0, 0), bo = mk<T>(0, 0);
                if (k < H) {
                    const C z = sc.ld(k), zc = cconj(sc.ld(k == 0 ? 0 : NI - k));
                    const C s = cadd(z, zc), d = csub(z, zc);
                    ao = mk<T>((T)0.5 * s.x, (T)0.5 * s.y);
                    bo = mk<T>((T)0.5 * d.y, (T)-0.5 * d.x);
                    if (k == 0) {
                        ao.x += ca * a.scale * (T)NI;
                        bo.x += cb * a.scale * (T)NI;
                    }
                }
                if (act) {
                    Ao[k] = ao;
                    Bo[k] = bo;
                }
            }
            __syncwarp();
        } else {
            C w[VR];
            C *vb = v;
            if constexpr (OP == OP_DERIV) reg_deriv<T, N, D::RFL, LL>(v, a.ktab, t);
            if constexpr (OP == OP_PAD) { reg_pad<T, N, D::RFL, LL>(v, w, t); vb = w; }
            if constexpr (OP == OP_UNPAD) { reg_unpad<T, N, D::RB0, LL>(v, w, t); vb = w; }
            fft_regs<NO, typename D::PB, LL, false>(vb, sc, twB, t);
            using G = Geo<NO, D::RBL, LL>;
            T *A = reinterpret_cast<T *>(a.dst) + r0 * a.dst_stride;
            T *B = A + a.dst_stride;
            const T addA = (OP == OP_PAD || OP == OP_UNPAD) ? ca : (T)0;
            const T addB = (OP == OP_PAD || OP == OP_UNPAD) ? cb : (T)0;
            if (act) {
#pragma unroll
                for (int b = 0; b < G::PER; ++b) {
                    const int j = t + LL * b;
                    if (G::FULL || j < G::NB)
#pragma unroll
                        for (int r = 0; r < D::RBL; ++r) {
                            const int i = j + r * G::NB;
                            A[i] = vb[b * D::RBL + r].x + addA;
                            B[i] = vb[b * D::RBL + r].y + addB;
                        }
                }
                if (OP == OP_INV && a.pad_mode && t < 2) {
                    A[NO + t] *= a.pad_scale;
                    B[NO + t] *= a.pad_scale;
                }
            }
        }
    }
}

template <typename T, int N, int OP>
__global__ void __launch_bounds__(256) k_rows(RowArgs<T> a)
{
    using C = C2<T>;
    using D = LineDerived<N, OP>;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *twF = reinterpret_cast<C *>(smraw);
    C *twB = twF + D::TF;
    C *scr = twB + D::TB;
    load_tables<T, N, OP>(a.twF, a.twB, twF, twB);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (long long base = ((long long)blockIdx.x * nw + warp) * D::LPW; base < a.npairs;
         base += (long long)gridDim.x * nw * D::LPW)
        row_unit<T, N, OP>(a, base, twF, twB, scr + warp * D::LPW * scratch_len(D::NM), lane);
}

// ----------------------------------------------------------------------------- column kernel
template <typename T, bool REAL, int LPW> struct ColTile {
    static constexpr int LINES = 8 * LPW;                  // lines per CTA (8 warps)
    static constexpr int W = REAL ? 2 * LINES : LINES;     // tile columns (elements)
    static constexpr int S = W + 1;                        // odd row stride
};

// The whole CTA processes column tile tx of plane z: coalesced tile load, one line per
// LL lanes through forward -> op -> backward in registers (the tile column is the
// exchange scratch), coalesced store.  Contains __syncthreads(): call uniformly.
template <typename T, int N, int OP, bool REAL>
__device__ __forceinline__ void col_unit(const ColArgs<T> &a, int z, int tx, const C2<T> *twF,
                                         const C2<T> *twB,
                                         typename std::conditional<REAL, T, C2<T>>::type *tile)
{
    using C = C2<T>;
    using E = typename std::conditional<REAL, T, C>::type;
    using D = LineDerived<N, OP>;
    constexpr int NI = D::NI, NO = D::NO, LL = D::LL, LPW = D::LPW, VR = D::VR;
    using TT = ColTile<T, REAL, LPW>;
    constexpr int W = TT::W, S = TT::S;

    const int c0 = tx * W;
    const int nc = min(W, a.ncols - c0);
    const E *src = reinterpret_cast<const E *>(a.src) + (long long)z * a.src_plane + c0;
    E *dst = reinterpret_cast<E *>(a.dst) + (long long)z * a.dst_plane + c0;

    // Tile load: 256 threads, UNR independent L2-only loads (ld.global.cg) in flight per
    // thread before the shared-memory stores, so the loop is not latency-serialised.
    // L2-only loads are also what the cluster-fused kernels need for data other CTAs wrote.
    {
        constexpr int TOT = NI * W, PERT = (TOT + 255) / 256, UNR = PERT < 8 ? PERT : 8;
#pragma unroll 1
        for (int b0 = 0; b0 < PERT; b0 += UNR) {
            E buf[UNR];
#pragma unroll
            for (int u = 0; u < UNR; ++u) {
                const int idx = threadIdx.x + 256 * (b0 + u);
                const int r = idx / W, c = idx - r * W;
                E v;
                if constexpr (REAL) v = (T)0;
                else v = mk<T>(0, 0);
                if (idx < TOT && c < nc) v = __ldcg(src + (long long)r * a.src_row + c);
                buf[u] = v;
            }
#pragma unroll
            for (int u = 0; u < UNR; ++u) {
                const int idx = threadIdx.x + 256 * (b0 + u);
                const int r = idx / W, c = idx - r * W;
                if (idx < TOT) tile[sidx(r) * S + c] = buf[u];
            }
        }
    }
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / LL, t = lane % LL;
    const int l = warp * LPW + g;
    const int c = REAL ? 2 * l : l;
    const bool act = c < nc;
    const int cc = act ? c : 0;
    C v[VR];
    T cr = 0, ci = 0;

    auto body = [&](auto &acc) {
        if constexpr (OP != OP_INV) {
            using G = Geo<NI, D::RF0, LL>;
            if constexpr (REAL) {
                const C c0v = acc.ld(0);
                cr = c0v.x;
                ci = c0v.y;
            }
#pragma unroll
            for (int b = 0; b < G::PER; ++b) {
                const int j = t + LL * b;
#pragma unroll
                for (int r = 0; r < D::RF0; ++r) {
                    C x = mk<T>(0, 0);
                    if (G::FULL || j < G::NB) {
                        x = acc.ld(j + r * G::NB);
                        x.x = (x.x - cr) * a.scale;
                        x.y = (x.y - ci) * a.scale;
                    }
                    v[b * D::RF0 + r] = x;
                }
            }
            __syncwarp();
            fft_regs<NI, typename D::PF, LL, true>(v, acc, twF, t);
        }
        if constexpr (OP == OP_FWD) {
            using G = Geo<NI, D::RFL, LL>;
#pragma unroll
            for (int b = 0; b < G::PER; ++b) {
                const int j = t + LL * b;
                if (G::FULL || j < G::NB)
#pragma unroll
                    for (int r = 0; r < D::RFL; ++r) {
                        const int i = j + r * G::NB;
                        C x = v[b * D::RFL + r];
                        if (a.zero_nyq && i == NI / 2) x = mk<T>(0, 0);
                        acc.st(i, x);
                    }
            }
        } else {
            C w[VR];
            C *vb = v;
            if constexpr (OP == OP_INV) {
                using G = Geo<NO, D::RB0, LL>;
#pragma unroll
                for (int b = 0; b < G::PER; ++b) {
                    const int j = t + LL * b;
#pragma unroll
                    for (int r = 0; r < D::RB0; ++r) {
                        const int i = j + r * G::NB;
                        C x = mk<T>(0, 0);
                        if (G::FULL || j < G::NB) {
                            x = acc.ld(i);
                            if (a.kmul) {
                                const T kk = (T)(a.kmul == 1 ? a.ktab[c0 + cc] : a.ktab[i]);
                                x = mk<T>(-kk * x.y, kk * x.x);
                            }
                            x.x *= a.scale;
                            x.y *= a.scale;
                        }
                        v[b * D::RB0 + r] = x;
                    }
                }
                __syncwarp();
            }
            if constexpr (OP == OP_DERIV) reg_deriv<T, N, D::RFL, LL>(v, a.ktab, t);
            if constexpr (OP == OP_PAD) { reg_pad<T, N, D::RFL, LL>(v, w, t); vb = w; }
            if constexpr (OP == OP_UNPAD) { reg_unpad<T, N, D::RB0, LL>(v, w, t); vb = w; }
            fft_regs<NO, typename D::PB, LL, false>(vb, acc, twB, t);
            using G = Geo<NO, D::RBL, LL>;
            const T ar = (OP == OP_PAD || OP == OP_UNPAD) ? cr : (T)0;
            const T ai = (OP == OP_PAD || OP == OP_UNPAD) ? ci : (T)0;
#pragma unroll
            for (int b = 0; b < G::PER; ++b) {
                const int j = t + LL * b;
                if (G::FULL || j < G::NB)
#pragma unroll
                    for (int r = 0; r < D::RBL; ++r) {
                        C x = vb[b * D::RBL + r];
                        x.x += ar;
                        x.y += ai;
                        acc.st(j + r * G::NB, x);
                    }
            }
        }
    };
    if constexpr (REAL) {
        TilePair<T> acc{tile, S, cc, act};
        body(acc);
    } else {
        TileCol<C> acc{tile, S, cc, act};
        body(acc);
    }
    __syncthreads();

    for (int idx = threadIdx.x; idx < NO * W; idx += blockDim.x) {
        const int r = idx / W, cx = idx - r * W;
        if (cx < nc) dst[(long long)r * a.dst_row + cx] = tile[sidx(r) * S + cx];
    }
    if constexpr (OP == OP_UNPAD && REAL) {
        // var(nxt+1:ldx,:) = var(1:2,:) (108_01_padd.f90:195)
        if (a.pad_copy && c0 == 0)
            for (int r = threadIdx.x; r < NO; r += blockDim.x) {
                E *d = reinterpret_cast<E *>(a.dst) + (long long)z * a.dst_plane + (long long)r * a.dst_row;
                d[a.ncols] = tile[sidx(r) * S + 0];
                d[a.ncols + 1] = tile[sidx(r) * S + 1];
            }
    }
    __syncthreads();   // the tile may be reused by the caller's next unit
}

// ----------------------------------------------------------------------------- line-minor columns
// Column lines without a staging tile: a CTA owns WB adjacent complex lines (WB real
// column pairs, or WB complex columns) of one plane.  Lane l % WB is the line and the
// remaining lane bits and the warp index form the butterfly slot t (LL slots), so
//   * the first pass loads its operands straight from global memory: for every element
//     index the WB lanes of a line group read WB adjacent pairs (coalesced, 8/16-byte
//     vector loads), and the last pass stores the same way;
//   * the exchange scratch is line-minor (element i of line l at buf[i*WB + l]): a warp
//     always touches consecutive words, so no pass has bank conflicts;
//   * passes are separated by __syncthreads() because a line spans all warps.
template <typename T, int NW_ = 8, int WB_ = (sizeof(T) == 4 ? 8 : 4)> struct LmGeo {
    static constexpr int WB = WB_;                        // lines per CTA (WB*8-byte row segments)
    static constexpr int NW = NW_;                        // warps per CTA
    static constexpr int LL = (32 / WB) * NW;             // butterfly slots per line
};
// Warps per CTA of the standalone column kernels.  FP32 lines of 256 and more get 16
// (twice the butterfly slots per line: half the registers per lane and twice the warps per
// SM at the same shared memory), except the y-pad, which measured fastest with 8; FP64
// (4 lines per CTA, already 64 slots per line) and the persistent ensemble units use 8.
#ifndef OBL_PAD_TWG
#define OBL_PAD_TWG 1
#endif
#ifndef OBL_COLS_TWG
#define OBL_COLS_TWG 1
#endif
#ifndef OBL_PAD_NW
#define OBL_PAD_NW 8
#endif
#ifndef OBL_PAD_WB
#define OBL_PAD_WB 8
#endif
#ifndef OBL_COLS_NW
#define OBL_COLS_NW 8   // warps per CTA of the FP32 ddy / forward y-transform of long lines
#endif
#ifndef OBL_COLS_WB
#define OBL_COLS_WB 8   // lines per CTA of the same
#endif
#ifndef OBL_COL_PF
#define OBL_COL_PF 2   // y-pad column kernel: L2 prefetch distance in quarters of a residency window (0 = off)
#endif
template <typename T, int N, int OP> constexpr int col_warps()
{
    return (sizeof(T) == 4 && N >= 256) ? (OP == OP_PAD ? OBL_PAD_NW
                                                        : ((OBL_COLS_TWG && (OP == OP_DERIV || OP == OP_FWD)) ? OBL_COLS_NW : 16))
                                        : 8;
}
// Twiddles read through L1 instead of staged in shared memory, with the registers bounded
// for 4 CTAs per SM (4 independent CTAs in different phases of their load / transform /
// store cycle instead of 3, or 2 of 16 warps).  For the FP32 y-pad of long lines this
// frees the 11.5 KB of tables that kept it at 3 CTAs per SM: 23% faster.  OBL_COLS_TWG
// applies the same shape (8 warps) to ddy and the forward y-transform: 24% and 19% faster
// than 16-warp CTAs with staged tables.
template <typename T, int N, int OP> constexpr bool col_tw_global()
{
    return sizeof(T) == 4 && N >= 256 &&
           ((OP == OP_PAD && OBL_PAD_TWG) || ((OP == OP_DERIV || OP == OP_FWD) && OBL_COLS_TWG));
}
// lines per CTA of the standalone column kernels (build-time knob for the FP32 y-pad)
template <typename T, int N, int OP> constexpr int col_lines()
{
    return (sizeof(T) == 4 && N >= 256 && OP == OP_PAD)
               ? OBL_PAD_WB
               : ((sizeof(T) == 4 && N >= 256 && OBL_COLS_TWG && (OP == OP_DERIV || OP == OP_FWD)) ? OBL_COLS_WB
                                                                                                 : LmGeo<T>::WB);
}
// Minimum resident CTAs per SM the column kernels are compiled for: with twiddles through
// L1, registers are bounded so that the CTAs of 32 warps in total fit on an SM.
#ifndef OBL_COL_WARPS_SM
#define OBL_COL_WARPS_SM 32   // resident warps per SM the register bound is set for
#endif
#ifndef OBL_COLS_WARPS_SM
#define OBL_COLS_WARPS_SM OBL_COL_WARPS_SM   // the same for ddy and the y-transform alone
#endif
constexpr int col_min_blocks(int nw, bool twg, int warps_sm = OBL_COL_WARPS_SM)
{
    return twg ? (nw >= warps_sm ? 1 : warps_sm / nw) : 1;
}
template <int OP> constexpr int col_warps_sm() { return (OP == OP_DERIV || OP == OP_FWD) ? OBL_COLS_WARPS_SM : OBL_COL_WARPS_SM; }

template <typename T, int N, int OP, int NW = 8, int WB = LmGeo<T>::WB> struct ColDerived {
    using D = LineDerived<N, OP>;
    static constexpr int LL = LmGeo<T, NW, WB>::LL;
    static constexpr int rf = Regs<D::NI, LL, typename D::PF>::v, rb = Regs<D::NO, LL, typename D::PB>::v;
    static constexpr int VR = rf > rb ? rf : rb;
};

// Store hook of the column kernel's backward output: epi(z, i, line, x) may change the
// value x of row i, line `line` of plane z just before it is stored; epi.prefetch(z, i,
// line) is called for the same elements when the line is loaded, before its transforms,
// so that what the hook reads is on chip by the time it is stored.  The default does
// nothing and compiles away.
struct NoColEpi {
    template <class C> __device__ __forceinline__ void operator()(int, int, int, C &) const {}
    __device__ __forceinline__ void prefetch(int, int, int) const {}
};

// Load hook of the column kernel's input: src(z, i, line) returns element i of global line
// `line` of plane z in place of the plain load from a.src.  The default is the plain load.
struct NoColSrc {};

// One CTA unit of the line-minor column kernel: line group bx of plane z.  The plan
// tables twF/twB are already in shared memory; buf is the exchange scratch (NM*WB).
// Called by k_cols2 (one unit per CTA) and by the persistent ensemble kernel.
// tile (SMEM_IN): the unit's input already in shared memory, row i of line l at
// tile[i*WB + l] (the persistent pipelined kernel below); otherwise read from global.
template <typename T, int N, int OP, bool REAL, int NW = 8, int WB_ = LmGeo<T>::WB, class EPI = NoColEpi,
          bool SMEM_IN = false, class SRC = NoColSrc>
__device__ __forceinline__ void cols2_unit(const ColArgs<T> &a, int bx, int z, const C2<T> *twF,
                                           const C2<T> *twB, C2<T> *buf, const EPI &epi = EPI(),
                                           const C2<T> *tile = nullptr, const SRC &src = SRC())
{
    using C = C2<T>;
    using E = typename std::conditional<REAL, T, C>::type;
    using D = LineDerived<N, OP>;
    using G = LmGeo<T, NW, WB_>;
    constexpr int NI = D::NI, NO = D::NO, WB = G::WB, LL = G::LL, VR = ColDerived<T, N, OP, NW, WB_>::VR;
    (void)NI;
    (void)twF;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int line = lane % WB, t = lane / WB + (32 / WB) * warp;
    const int gl = bx * WB + line;                         // global line index
    const int nlines = REAL ? a.ncols / 2 : a.ncols;
    const bool act = gl < nlines;
    const int glc = act ? gl : 0;
    // element i of this line: a complex value (a real column pair for REAL)
    const E *srcz = reinterpret_cast<const E *>(a.src) + (long long)z * a.src_plane;
    E *dstz = reinterpret_cast<E *>(a.dst) + (long long)z * a.dst_plane;
    // the checked build tests each element's level, column and plane offset against the
    // extents the arguments give (nlev planes of src_plane / dst_plane, rows of src_row / dst_row)
    auto col_ok = [&](int i, int col, int row, long long plane, int site) {
        const int ce = REAL ? 2 * col + 1 : col;
        return ck_in(z, a.nlev, site) && ck_in(ce, row, site) && ck_in((long long)i * row + ce, plane, site);
    };
    auto gld = [&](int i) -> C {
        if constexpr (!std::is_same<SRC, NoColSrc>::value) return src(z, i, glc);
        else if constexpr (SMEM_IN) return tile[i * WB + line];
        else {
            if (OBL_CHECK && !col_ok(i, glc, a.src_row, a.src_plane, CK_COL_LOAD)) return mk<T>(0, 0);
            if constexpr (REAL) return __ldcg(reinterpret_cast<const C *>(srcz + (long long)i * a.src_row + 2 * glc));
            else return __ldcg(srcz + (long long)i * a.src_row + glc);
        }
    };
    auto gst = [&](int i, C v) {
        if (OBL_CHECK && !col_ok(i, gl, a.dst_row, a.dst_plane, CK_COL_STORE)) return;
        if constexpr (REAL) *reinterpret_cast<C *>(dstz + (long long)i * a.dst_row + 2 * gl) = v;
        else dstz[(long long)i * a.dst_row + gl] = v;
    };
    LineMinor<C, WB> sc{buf, line};
    C v[VR];
    C cref = mk<T>(0, 0);

    if constexpr (OP != OP_INV) {
        using GG = Geo<NI, D::RF0, LL>;
        if constexpr (REAL) cref = gld(0);
#pragma unroll
        for (int b = 0; b < GG::PER; ++b) {
            const int j = t + LL * b;
#pragma unroll
            for (int r = 0; r < D::RF0; ++r) {
                C x = mk<T>(0, 0);
                if (act && (GG::FULL || j < GG::NB)) {
                    x = gld(j + r * GG::NB);
                    x.x = (x.x - cref.x) * a.scale;
                    x.y = (x.y - cref.y) * a.scale;
                }
                v[b * D::RF0 + r] = x;
            }
        }
#if OBL_COL_PF
        // the CTA that processes this line group pf_ahead planes later (about one
        // residency window of CTAs) finds its input in L2
        if (!SMEM_IN && a.pf_ahead > 0 && act && z + a.pf_ahead < a.nlev) {
            const E *pz = srcz + (long long)a.pf_ahead * a.src_plane;
#pragma unroll
            for (int b = 0; b < GG::PER; ++b) {
                const int j = t + LL * b;
                if (GG::FULL || j < GG::NB)
#pragma unroll
                    for (int r = 0; r < D::RF0; ++r) {
                        const long long i = j + r * GG::NB;
                        const E *ptr = pz + i * a.src_row + (REAL ? 2 * glc : glc);
                        asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
                    }
            }
        }
#endif
        if constexpr (!std::is_same<EPI, NoColEpi>::value) {
            using GP = Geo<NO, D::RBL, LL>;
            if (act) {
#pragma unroll
                for (int b = 0; b < GP::PER; ++b) {
                    const int j = t + LL * b;
                    if (GP::FULL || j < GP::NB)
#pragma unroll
                        for (int r = 0; r < D::RBL; ++r) epi.prefetch(z, j + r * GP::NB, gl);
                }
            }
        }
        // an input tile in shared memory may be the exchange scratch itself: every thread
        // has its elements before the first pass stores into it
        if constexpr (SMEM_IN) __syncthreads();
        fft_regs<NI, typename D::PF, LL, true, true>(v, sc, twF, t);
    }
    if constexpr (OP == OP_FWD) {
        using GG = Geo<NI, D::RFL, LL>;
        if (act) {
#pragma unroll
            for (int b = 0; b < GG::PER; ++b) {
                const int j = t + LL * b;
                if (GG::FULL || j < GG::NB)
#pragma unroll
                    for (int r = 0; r < D::RFL; ++r) {
                        const int i = j + r * GG::NB;
                        C x = v[b * D::RFL + r];
                        if (a.zero_nyq && i == NI / 2) x = mk<T>(0, 0);
                        gst(i, x);
                    }
            }
        }
    } else {
        C w[VR];
        C *vb = v;
        if constexpr (OP == OP_INV) {
            using GG = Geo<NO, D::RB0, LL>;
#pragma unroll
            for (int b = 0; b < GG::PER; ++b) {
                const int j = t + LL * b;
#pragma unroll
                for (int r = 0; r < D::RB0; ++r) {
                    const int i = j + r * GG::NB;
                    C x = mk<T>(0, 0);
                    if (act && (GG::FULL || j < GG::NB)) {
                        x = gld(i);
                        if (a.kmul) {
                            const T kk = (T)(a.kmul == 1 ? a.ktab[glc] : a.ktab[i]);
                            x = mk<T>(-kk * x.y, kk * x.x);
                        }
                        x.x *= a.scale;
                        x.y *= a.scale;
                    }
                    v[b * D::RB0 + r] = x;
                }
            }
        }
        if constexpr (OP == OP_DERIV) reg_deriv<T, N, D::RFL, LL>(v, a.ktab, t);
        if constexpr (OP == OP_PAD) { reg_pad<T, N, D::RFL, LL>(v, w, t); vb = w; }
        if constexpr (OP == OP_UNPAD) { reg_unpad<T, N, D::RB0, LL>(v, w, t); vb = w; }
        fft_regs<NO, typename D::PB, LL, false, true>(vb, sc, twB, t);
        using GG = Geo<NO, D::RBL, LL>;
        const bool addc = (OP == OP_PAD || OP == OP_UNPAD);
        if (act) {
#pragma unroll
            for (int b = 0; b < GG::PER; ++b) {
                const int j = t + LL * b;
                if (GG::FULL || j < GG::NB)
#pragma unroll
                    for (int r = 0; r < D::RBL; ++r) {
                        const int i = j + r * GG::NB;
                        C x = vb[b * D::RBL + r];
                        if (addc) {
                            x.x += cref.x;
                            x.y += cref.y;
                        }
                        epi(z, i, gl, x);
                        gst(i, x);
                        if constexpr (OP == OP_UNPAD && REAL) {
                            // var(nxt+1:ldx,:) = var(1:2,:) (108_01_padd.f90:195)
                            if (a.pad_copy && gl == 0 && ck_in(a.ncols + 1, a.dst_row, CK_COL_STORE))
                                *reinterpret_cast<C *>(dstz + (long long)i * a.dst_row + a.ncols) = x;
                        }
                    }
            }
        }
    }
}

template <typename T, int N, int OP, bool REAL, int NW, int WB, bool TWG = false>
__global__ void __launch_bounds__(32 * NW, col_min_blocks(NW, TWG, col_warps_sm<OP>())) k_cols2(ColArgs<T> a)
{
    using C = C2<T>;
    using D = LineDerived<N, OP>;
    extern __shared__ __align__(16) unsigned char smraw[];
    if constexpr (TWG) {
        cols2_unit<T, N, OP, REAL, NW, WB>(a, blockIdx.x, blockIdx.y, a.twF, a.twB, reinterpret_cast<C *>(smraw));
    } else {
        C *twF = reinterpret_cast<C *>(smraw);
        C *twB = twF + D::TF;
        C *buf = twB + D::TB;
        load_tables<T, N, OP>(a.twF, a.twB, twF, twB);
        __syncthreads();
        cols2_unit<T, N, OP, REAL, NW, WB>(a, blockIdx.x, blockIdx.y, twF, twB, buf);
    }
}

// ----------------------------------------------------------------------------- pipelined columns
// Persistent form of k_cols2: each CTA walks units u = blockIdx.x, + gridDim.x, ... (line
// group u % nbx of plane u / nbx) and, while it transforms unit u, the next unit's input
// tile (NI rows x WB lines) is already on its way into shared memory with 8-byte cp.async
// copies (every address of a field row is 8-byte aligned; its 2056-byte pitch at nxt = 512
// is not the 16-byte multiple a tensor map needs).  Two tiles alternate; the exchange
// scratch is separate.  The loads of the column kernel then no longer stall its warps.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 8 : 0;   // 0: the 8 bytes are zero-filled
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::); }

template <typename T, int N, int OP, bool REAL, int NW, int WB>
__device__ __forceinline__ void cols_tile_issue(const ColArgs<T> &a, int nbx, int u, C2<T> *tile)
{
    using C = C2<T>;
    using E = typename std::conditional<REAL, T, C>::type;
    constexpr int NI = LineDerived<N, OP>::NI;
    const int bx = u % nbx, z = u / nbx;
    const int nlines = REAL ? a.ncols / 2 : a.ncols;
    const E *srcz = reinterpret_cast<const E *>(a.src) + (long long)z * a.src_plane;
    for (int idx = threadIdx.x; idx < NI * WB; idx += 32 * NW) {
        const int i = idx / WB, l = idx % WB, gl = bx * WB + l;
        const bool ok = gl < nlines;
        const E *g = srcz + (long long)i * a.src_row + (REAL ? 2 * (ok ? gl : 0) : (ok ? gl : 0));
        cp_async8(tile + idx, g, ok);
    }
}

template <typename T, int N, int OP, bool REAL, int NW, int WB>
__global__ void __launch_bounds__(32 * NW, 2) k_cols2_pipe(ColArgs<T> a, int nbx)
{
    using C = C2<T>;
    using D = LineDerived<N, OP>;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *tile0 = reinterpret_cast<C *>(smraw);
    C *tile1 = tile0 + D::NI * WB;
    C *buf = tile1 + D::NI * WB;
    const int nunits = nbx * a.nlev;
    int u = blockIdx.x;
    if (u >= nunits) return;
    cols_tile_issue<T, N, OP, REAL, NW, WB>(a, nbx, u, tile0);
    cp_async_commit();
    for (int it = 0; u < nunits; ++it, u += gridDim.x) {
        C *cur = (it & 1) ? tile1 : tile0;
        C *nxt = (it & 1) ? tile0 : tile1;
        const int un = u + gridDim.x;
        if (un < nunits) cols_tile_issue<T, N, OP, REAL, NW, WB>(a, nbx, un, nxt);
        cp_async_commit();
        cp_async_wait_prev();
        __syncthreads();
        cols2_unit<T, N, OP, REAL, NW, WB, NoColEpi, true>(a, u % nbx, u / nbx, a.twF, a.twB, buf, NoColEpi(), cur);
        __syncthreads();
    }
}

#ifndef OBL_COL_PIPE
#define OBL_COL_PIPE 0   // FP32 y-pad, ddy and y-transform of long lines: persistent prefetching form
#endif

// ----------------------------------------------------------------------------- TMA-fed y-pad
// The FP32 y-pad with its CTA's input tile (NI rows x WB real column pairs of the x-padded
// plane) brought into shared memory by tensor-map copies: one thread issues
// cp.async.bulk.tensor loads of boxes of 2*WB floats x box_rows rows (64-byte row segments,
// landing row after row: element i of line l at tile[i*WB + l], the line-minor layout of
// the exchange scratch), completing on an mbarrier, and the same thread asks L2 for the
// tile pf_ahead planes later (cp.async.bulk.prefetch.tensor).  The tile lands in the
// exchange scratch the CTA already holds, so shared memory per CTA and CTAs per SM stay
// those of k_cols2.  The tensor map covers this GPU's own x-padded planes; no multicast.
// The wait is bounded: on timeout wait_err is set (the host reports OBL_ERR_TIMEOUT), the
// CTA waits once more (bounded) for the copy, and its results are not to be used.
template <typename T, int N, int OP, bool REAL, int NW, int WB>
__global__ void __launch_bounds__(32 * NW, col_min_blocks(NW, true, col_warps_sm<OP>()))
    k_cols2_tma(ColArgs<T> a, const __grid_constant__ CUtensorMap tm, int box_rows)
{
    using C = C2<T>;
    using D = LineDerived<N, OP>;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) unsigned long long bar;
    // tensor copies write 128-byte aligned shared memory (an offset from smraw keeps the
    // pointer in the shared window for the compiler)
    C *buf = reinterpret_cast<C *>(smraw + ((128u - (smem_addr(smraw) & 127u)) & 127u));
    const unsigned sbar = smem_addr(&bar);
    const int x0 = blockIdx.x * 2 * WB, y0 = blockIdx.y * D::NI;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n\tfence.mbarrier_init.release.cluster;\n\t"
                     "fence.proxy.async.shared::cta;" ::"r"(sbar)
                     : "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sbar),
                     "r"((unsigned)(sizeof(C) * D::NI * WB))
                     : "memory");
        for (int y = 0; y < D::NI; y += box_rows)
            asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                         "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(buf + (size_t)y * WB)),
                         "l"(&tm), "r"(x0), "r"(y0 + y), "r"(sbar)
                         : "memory");
        if (a.pf_ahead > 0 && (int)blockIdx.y + a.pf_ahead < a.nlev)
            for (int y = 0; y < D::NI; y += box_rows)
                asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(&tm), "r"(x0),
                             "r"(y0 + a.pf_ahead * D::NI + y)
                             : "memory");
    }
    __syncthreads();   // the barrier is initialised before anyone waits on it
    if (!mbar_wait_bounded(sbar, 0)) {
        if (a.wait_err) atomicExch(a.wait_err, 1);
        mbar_wait_bounded(sbar, 0);   // a late copy lands before the tile is reused
    }
    cols2_unit<T, N, OP, REAL, NW, WB, NoColEpi, true>(a, blockIdx.x, blockIdx.y, a.twF, a.twB, buf, NoColEpi(), buf);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
typedef CUresult (*TensorMapEncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                         const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                         CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                         CUtensorMapFloatOOBfill);
inline TensorMapEncodeTiled tensor_map_encoder()
{
    static TensorMapEncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (TensorMapEncodeTiled)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// rows per tensor copy: NI itself up to 256 rows (the box limit), else the largest divisor
// of NI not above 256; 0 = no such split
constexpr int tma_box_rows(int ni)
{
    if (ni <= 256) return ni;
    for (int b = 256; b >= 8; --b)
        if (ni % b == 0) return b;
    return 0;
}

// ----------------------------------------------------------------------------- launchers
template <typename T, int N, int OP> inline size_t rows_smem()
{
    using D = LineDerived<N, OP>;
    return sizeof(C2<T>) * ((size_t)D::TF + D::TB + (size_t)8 * D::LPW * scratch_len(D::NM));
}
template <typename T, int N, int OP, bool REAL> inline size_t cols_smem()
{
    using D = LineDerived<N, OP>;
    using E = typename std::conditional<REAL, T, C2<T>>::type;
    using TT = ColTile<T, REAL, D::LPW>;
    return sizeof(C2<T>) * ((size_t)D::TF + D::TB) + sizeof(E) * (size_t)tile_rows(D::NM) * TT::S;
}

template <typename T, int N, int OP> cudaError_t launch_rows_t(const RowArgs<T> &a, cudaStream_t s)
{
    static int caps[kMaxDevices] = {};
    const size_t sm = rows_smem<T, N, OP>();
    auto kern = k_rows<T, N, OP>;
    const int ds = device_slot();
    int grid_cap = ds >= 0 ? caps[ds] : 0;
    if (!grid_cap) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        int dev = 0, nsm = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, sm);
        grid_cap = nsm * (per > 0 ? per : 1);
        if (ds >= 0) caps[ds] = grid_cap;
    }
    constexpr int LPW = LineDerived<N, OP>::LPW;
    const long long per_cta = 8LL * LPW;
    long long want = (a.npairs + per_cta - 1) / per_cta;
    int grid = (int)(want < grid_cap ? want : grid_cap);
    if (grid < 1) return cudaSuccess;
    kern<<<grid, 256, sm, s>>>(a);
    return cudaGetLastError();
}

template <typename T, int N, int OP, int WB = LmGeo<T>::WB> inline size_t cols2_smem()
{
    using D = LineDerived<N, OP>;
    return sizeof(C2<T>) * ((size_t)D::TF + D::TB + (size_t)D::NM * WB);
}

template <typename T, int N, int OP, bool REAL> cudaError_t launch_cols_t(const ColArgs<T> &a0, cudaStream_t s)
{
    static int residents[kMaxDevices] = {};   // CTAs of this kernel resident on the whole GPU
    constexpr int NW = col_warps<T, N, OP>(), WB = col_lines<T, N, OP>();
    constexpr bool TWG = col_tw_global<T, N, OP>();
    using D = LineDerived<N, OP>;
    const size_t sm = TWG ? sizeof(C2<T>) * (size_t)D::NM * WB : cols2_smem<T, N, OP, WB>();
    auto kern = k_cols2<T, N, OP, REAL, NW, WB, TWG>;
    const int ds = device_slot();
    int resident = ds >= 0 ? residents[ds] : 0;
    if (!resident) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        int dev = 0, nsm = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 32 * NW, sm);
        resident = nsm * (per > 0 ? per : 1);
        if (ds >= 0) residents[ds] = resident;
    }
    ColArgs<T> a = a0;
    const int nlines = REAL ? a.ncols / 2 : a.ncols;
    if constexpr (std::is_same<T, float>::value && OP == OP_PAD && REAL && TWG && tma_box_rows(D::NI) > 0) {
        // the x-padded planes as a 2-D map: ncols floats wide (pitch src_row), NI*nlev rows
        const bool fits = a.tma && a.src_plane == a.src_row * (long long)D::NI && (a.src_row * 4) % 16 == 0 &&
                          ((uintptr_t)a.src % 16) == 0 && tensor_map_encoder() != nullptr;
        if (fits) {
            constexpr int BR = tma_box_rows(D::NI);
            CUtensorMap tm;
            const cuuint64_t dims[2] = {(cuuint64_t)a.ncols, (cuuint64_t)D::NI * a.nlev};
            const cuuint64_t strides[1] = {(cuuint64_t)a.src_row * sizeof(T)};
            const cuuint32_t box[2] = {(cuuint32_t)(2 * WB), (cuuint32_t)BR};
            const cuuint32_t estr[2] = {1, 1};
            if (tensor_map_encoder()(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(a.src), dims, strides,
                                     box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return cudaErrorInvalidValue;
            static int tres[kMaxDevices] = {};
            auto tk = k_cols2_tma<T, N, OP, REAL, NW, WB>;
            const size_t tsm = sm + 128;
            int tr = ds >= 0 ? tres[ds] : 0;
            if (!tr) {
                cudaError_t e = cudaFuncSetAttribute(tk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm);
                if (e != cudaSuccess) return e;
                int dev = 0, nsm = 0, per = 0;
                cudaGetDevice(&dev);
                cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tk, 32 * NW, tsm);
                tr = nsm * (per > 0 ? per : 1);
                if (ds >= 0) tres[ds] = tr;
            }
            dim3 grid((nlines + WB - 1) / WB, a.nlev);
            if (grid.x < 1 || grid.y < 1) return cudaSuccess;
            if (OBL_COL_PF) a.pf_ahead = (int)((OBL_COL_PF * (long long)tr + 4LL * grid.x - 1) / (4LL * grid.x));
            tk<<<grid, 32 * NW, tsm, s>>>(a, tm, BR);
            return cudaGetLastError();
        }
    }
    if constexpr (OBL_COL_PIPE && TWG && OP != OP_INV) {
        static int pres[kMaxDevices] = {};
        auto pk = k_cols2_pipe<T, N, OP, REAL, NW, WB>;
        const size_t psm = sizeof(C2<T>) * ((size_t)2 * D::NI * WB + (size_t)D::NM * WB);
        int pr = ds >= 0 ? pres[ds] : 0;
        if (!pr) {
            cudaError_t e = cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm);
            if (e != cudaSuccess) return e;
            int dev = 0, nsm = 0, per = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, pk, 32 * NW, psm);
            pr = nsm * (per > 0 ? per : 1);
            if (ds >= 0) pres[ds] = pr;
        }
        const int nbx = (nlines + WB - 1) / WB;
        const long long nunits = (long long)nbx * a.nlev;
        if (nunits < 1) return cudaSuccess;
        const int grid = (int)(nunits < pr ? nunits : pr);
        pk<<<grid, 32 * NW, psm, s>>>(a, nbx);
        return cudaGetLastError();
    }
    dim3 grid((nlines + WB - 1) / WB, a.nlev);
    // y-pad only: measured 5% faster at 512x512x256; ddy and the y-transform did not gain
    if (OBL_COL_PF && OP == OP_PAD) a.pf_ahead = (int)((OBL_COL_PF * (long long)resident + 4LL * grid.x - 1) / (4LL * grid.x));
    if (grid.x < 1 || grid.y < 1) return cudaSuccess;
    kern<<<grid, 32 * NW, sm, s>>>(a);
    return cudaGetLastError();
}

// Runtime dispatch: n is the base length (the unpadded one for PAD/UNPAD).
template <typename T> cudaError_t launch_rows(int op, int n, const RowArgs<T> &a, cudaStream_t s);
template <typename T> cudaError_t launch_cols(int op, bool real, int n, const ColArgs<T> &a, cudaStream_t s);

// The same line ops on up to kMultiFields fields of one shape in one launch: field f
// reads src[f] and writes dst[f]; the args' src/dst are ignored.  Rows: OP_DERIV, OP_PAD,
// OP_UNPAD, OP_FWD; columns: the real-column OP_DERIV, OP_PAD, OP_UNPAD and the complex
// OP_FWD.  For grids whose single-field launches are too small to fill the GPU.
constexpr int kMultiFields = 6;
template <typename T> struct MultiPtr {
    const void *src[kMultiFields];
    void *dst[kMultiFields];
};
template <typename T>
cudaError_t launch_rows_multi(int op, int n, const RowArgs<T> &a, const MultiPtr<T> &m, int nf, cudaStream_t s);
template <typename T>
cudaError_t launch_cols_multi(int op, int n, const ColArgs<T> &a, const MultiPtr<T> &m, int nf, cudaStream_t s);
bool line_length_supported(int n);
// twiddle table (interleaved re,im in FP64) of the plan with the given role for base length n
std::vector<double> plan_table(int n, int role);

} // namespace obl
