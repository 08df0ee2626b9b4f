// press.cu -- batched tridiagonal pressure solve and the streaming kernels.
//
// k_tdma solves, for every horizontal wavenumber column (kx,ky), the staggered-grid
// Poisson system of press_stag_array (SBL/code/109_press_stag_array.f90): it builds
// the right-hand side from the spectra of u,v,w on the fly (:203-225), forms the
// bands of init_coef_press from k^2 on the fly (:4-63), eliminates them as
// tdmaMcoef_pipelined + the forward sweep do (:72-103, :260-277) and back-substitutes
// (:280-317).  One thread owns one column; consecutive threads own consecutive kx,
// so every level's loads and stores are coalesced along the contiguous kx index.
// On one GPU the pipelined send/recv chain across z-ranks collapses to one sequential
// sweep per column, which is the same arithmetic in the same order.
#include <cstdint>
#include <type_traits>

#include "async.cuh"
#include "common.cuh"
#include "fft.cuh"
#include "press.cuh"

namespace obl {

static constexpr double kTadv1 = 1.5;                 // 001_param.f90:152
static constexpr double kBogus = -1234567890.0;       // 001_param.f90:40

template <typename TS, typename TC, bool ISLAND, bool G = false>
__global__ void __launch_bounds__(128) k_tdma(TdmaArgs<TS> a, IslandArgs isl)
{
    tdma_column<TS, TC, ISLAND, G>(a, isl, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Mixed precision in one launch: the first nbi blocks solve the FP64 island columns (their
// long sequential FP64 sweeps start first), the remaining blocks the FP32 bulk columns,
// so the two overlap instead of running back to back.  The sweeps are latency-bound: 8
// blocks per SM (64 registers, a few FP64 spills) measured faster than 5 without spills
// (OBL_TDMA_MINB is the build-time knob).
#ifndef OBL_TDMA_MINB
#define OBL_TDMA_MINB 8
#endif
template <typename T, bool G = false>
__global__ void __launch_bounds__(128, OBL_TDMA_MINB) k_tdma_mixed(TdmaArgs<T> a, IslandArgs isl, int nbi)
{
    if ((int)blockIdx.x < nbi)
        tdma_column<T, double, true, G>(a, isl, (long long)blockIdx.x * blockDim.x + threadIdx.x);
    else
        tdma_column<T, T, false, G>(a, isl, (long long)(blockIdx.x - nbi) * blockDim.x + threadIdx.x);
}

template <typename T> void launch_tdma(const TdmaArgs<T> &a, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    IslandArgs none{nullptr, 0, nullptr, nullptr};
    const int bs = 128;
    const unsigned nb = (unsigned)((a.S + bs - 1) / bs);
    if (a.gform) k_tdma<T, T, false, true><<<nb, bs, 0, s>>>(a, none);
    else k_tdma<T, T, false><<<nb, bs, 0, s>>>(a, none);
    e = cudaGetLastError();
}

template <typename T>
void launch_tdma_island(const TdmaArgs<T> &a, const IslandArgs &isl, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    const int bs = 128;
    const int nbi = (int)((isl.n + bs - 1) / bs), nbb = (int)((a.S + bs - 1) / bs);
    if (a.gform) k_tdma_mixed<T, true><<<(unsigned)(nbi + nbb), bs, 0, s>>>(a, isl, nbi);
    else k_tdma_mixed<T><<<(unsigned)(nbi + nbb), bs, 0, s>>>(a, isl, nbi);
    e = cudaGetLastError();
}

// ----------------------------------------------------------------------------- register-segmented solve
// The FP32 bulk columns without scratch traffic.  A CTA owns 32 consecutive columns
// (lane = column, so every load and store of a level is 256 contiguous bytes) and splits
// their L rows into kRegSeg segments of Ls <= kRegLev rows, one warp per segment.  Each
// thread eliminates its segment's rows with the neighbouring segments' boundary values
// left as unknowns (the partition method: x_i = y_i + v_i x_{s-1} + w_i x_{e+1}), keeping
// the forward sweep's y', v', c' in registers; lane l of warp 0 then solves column l's
// reduced system of 2K boundary values (a 2x2-block tridiagonal chain, eliminated upward
// and substituted downward) in shared memory, and every thread back-substitutes its rows
// from registers.  HBM sees only the compulsory traffic: three RHS spectra in, p_hat and
// the dpdz spectrum out (the one-sweep solve also writes and re-reads c' and d').
// The bands, RHS and boundary rows are those of tdma_column (109_press_stag_array.f90:
// 4-63, 203-225, 280-317); the rows are the same, only the elimination order differs.
// FP64 island columns keep the sequential FP64 sweep, in the launch's first nbi blocks.
constexpr int kRegSegMax = 16;   // warps per CTA = segments per column, at most

// 1/x for the FP32 columns' recurrences: the hardware reciprocal (__fdividef, within 2 ulp)
// instead of the IEEE division sequence, which sat on the sweep's serial dependency chain;
// the FP32 columns are diagonally dominant and round at 6e-8 anyway (the weakly dominant
// ones are the FP64 islands)
#ifndef OBL_TDMA_FAST_RCP
#define OBL_TDMA_FAST_RCP 1
#endif
template <typename T> __device__ __forceinline__ T rcp_sweep(T x)
{
    if constexpr (std::is_same<T, float>::value && OBL_TDMA_FAST_RCP) return __fdividef(1.0f, x);
    else return (T)1 / x;
}
constexpr int kRegLev = 16;      // rows a segment keeps in registers (so L <= 256)

// Boundary coefficients of every segment (x_s = Ys + Vs x_{s-1} + Ws x_{e+1}, the same for
// x_e).  The reduced solve runs in place: the upward elimination (x_s^j = S_j + T_j
// x_s^{j+1}, x_e^j = P_j + Q_j x_s^{j+1}) overwrites Ys, Ws, Ye, We of row j with S, T, P, Q
// once it has read them, and the downward substitution overwrites Ys, Ye with the solved
// x_s, x_e.
template <typename T, int NSEG> struct SegShared {
    C2<T> Ys[NSEG][32], Ye[NSEG][32];
    T Vs[NSEG][32], Ve[NSEG][32], Ws[NSEG][32], We[NSEG][32];
};

// Per-lane column of a segmented unit: lane l owns column q0 + l.
template <typename T> struct SegCol {
    long long q;
    bool act, nyq, m00;
    T kx, ky, k2;
    __device__ __forceinline__ void init(const TdmaArgs<T> &a, long long q0, int lane)
    {
        q = q0 + lane;
        const bool inq = q < a.S;
        // q < S, and S (one spectral plane) fits 32 bits: one 32-bit division
        const int iy = inq ? (int)((unsigned)q / (unsigned)a.lhx) : 0, ix = inq ? (int)q - iy * a.lhx : 0;
        nyq = inq && (ix == a.lhx - 1 || iy == a.nyt / 2);
        const bool isl_col = inq && a.skip && a.skip[q];
        act = inq && !nyq && !isl_col;
        const double kxd = act ? a.kx[ix] : 0.0, kyd = act ? a.ky[iy] : 0.0;
        const double k2d = kxd * kxd + kyd * kyd;   // 002_fft.f90:167
        m00 = (k2d == 0.0);
        kx = (T)kxd;
        ky = (T)kyd;
        k2 = (T)k2d;
    }
};

// RHS of row iz from the spectra (109:203-225): i*(kx*H_x + ky*H_y) + dH_z/dz, H_z(0)
// added at iz = 1; the (0,0) mode takes H_z itself; a solved top row (npz = 1 mode) is 0.
// dH_z/dz as dH_z * (1/dz): a product instead of a division sequence per row (within 1 ulp
// of the quotient; the FP64 island columns divide in tdma_column).
// IN: a full segment away from both ends (rows 2..L-1 only), whose rows need no end cases.
template <typename T, bool IN = false>
__device__ __forceinline__ C2<T> seg_rhs(const SegCol<T> &c, int iz, int L, bool top_solved, T idz, C2<T> hx, C2<T> hy,
                                         C2<T> hzl, C2<T> hzu, C2<T> hz0)
{
    const C2<T> sxy = mk<T>(c.kx * hx.x + c.ky * hy.x, c.kx * hx.y + c.ky * hy.y);
    C2<T> dh = csub(hzu, hzl);
    if (!IN && iz == 1) dh = cadd(dh, hz0);
    C2<T> r = mk<T>(-sxy.y + dh.x * idz, sxy.x + dh.y * idz);
    if (c.m00) r = (!IN && iz == 1) ? mk<T>(0, 0) : hzl;
    if (!IN && iz == L && !top_solved) r = mk<T>(0, 0);
    return r;
}

// Forward sweep of rows s..s+ns-1 with x_{s-1} left unknown (x_i = y'_i + v'_i x_{s-1} -
// c'_i x_{i+1}), then the segment's two boundary rows in terms of x_{s-1} and x_{e+1},
// stored for the reduced solve.  Bands of 109:4-63 (the Neumann top row :33-38, npz >= 2).
// IN: a full segment of interior rows, whose bands are the same on every row.
template <typename T, int NSEG, bool IN = false>
__device__ __forceinline__ void seg_eliminate(const SegCol<T> &c, C2<T> (&y)[kRegLev], T (&cp)[kRegLev],
                                              T (&vp)[kRegLev], int s, int ns_, int L, bool top_solved, T idz,
                                              T idz2, SegShared<T, NSEG> &sh, int k, int lane)
{
    const int ns = IN ? kRegLev : ns_;
    T cprev = 0, vprev = 1;
    C2<T> yprev = mk<T>(0, 0);
    // interior bands: the (0,0) mode's dz-weighted difference rows, else the k^2 rows
    const T am_in = c.m00 ? -idz : idz2, bm_in = c.m00 ? idz : -(c.k2 + (T)2 * idz2), cm_in = c.m00 ? (T)0 : idz2;
#pragma unroll
    for (int i = 0; i < kRegLev; ++i) {
        if (i < ns) {
            const int iz = s + i;
            T am, bm, cm;
            if (IN) {
                am = am_in; bm = bm_in; cm = cm_in;
            } else if (iz == L && !top_solved) {
                am = 0; bm = 1; cm = 0;
            } else if (!c.m00) {
                const bool top = iz == L;
                am = (iz == 1) ? (T)0 : idz2;
                bm = (iz == 1 || top) ? -(c.k2 + idz2) : -(c.k2 + (T)2 * idz2);
                cm = top ? (T)0 : idz2;
            } else {
                am = (iz == 1) ? (T)0 : -idz;
                bm = idz;
                cm = 0;
            }
            const T ibp = rcp_sweep<T>(bm - am * cprev);
            cp[i] = cm * ibp;
            vp[i] = -am * vprev * ibp;
            y[i] = mk<T>((y[i].x - am * yprev.x) * ibp, (y[i].y - am * yprev.y) * ibp);
            cprev = cp[i];
            vprev = vp[i];
            yprev = y[i];
        }
    }
    C2<T> ys = y[0];
    T vs = 0, ws = 0;
#pragma unroll
    for (int i = kRegLev - 1; i >= 0; --i) {
        if (i == ns - 1) {
            ys = y[i];
            vs = vp[i];
            ws = -cp[i];
            sh.Ye[k][lane] = ys;
            sh.Ve[k][lane] = vs;
            sh.We[k][lane] = ws;
        } else if (i < ns - 1) {
            ys = mk<T>(y[i].x - cp[i] * ys.x, y[i].y - cp[i] * ys.y);
            vs = vp[i] - cp[i] * vs;
            ws = -cp[i] * ws;
        }
    }
    sh.Ys[k][lane] = ys;
    sh.Vs[k][lane] = vs;
    sh.Ws[k][lane] = ws;
}

// Lane l's reduced system of column l: 2K boundary values, a 2x2-block chain eliminated
// upward and substituted downward, in place.
template <typename T, int NSEG> __device__ __forceinline__ void seg_reduced(SegShared<T, NSEG> &sh, int K, int lane)
{
    using C = C2<T>;
    C P = mk<T>(0, 0);
    T Q = 0;
    for (int j = 0; j < K; ++j) {
        const C ys = sh.Ys[j][lane], ye = sh.Ye[j][lane];
        const T vs = sh.Vs[j][lane], ws = sh.Ws[j][lane], ve = sh.Ve[j][lane], we = sh.We[j][lane];
        const T iden = rcp_sweep<T>((T)1 - vs * Q);
        const C Sj = mk<T>((ys.x + vs * P.x) * iden, (ys.y + vs * P.y) * iden);
        const T Tj = ws * iden;
        const C Pj = mk<T>(ye.x + ve * (P.x + Q * Sj.x), ye.y + ve * (P.y + Q * Sj.y));
        const T Qj = ve * Q * Tj + we;
        sh.Ys[j][lane] = Sj;
        sh.Ws[j][lane] = Tj;
        sh.Ye[j][lane] = Pj;
        sh.We[j][lane] = Qj;
        P = Pj;
        Q = Qj;
    }
    // the top segment has no x_{e+1} (c = 0 in its last row): x_s = S, x_e = P stay in place
    C xs = sh.Ys[K - 1][lane];
    for (int j = K - 2; j >= 0; --j) {
        const T Tj = sh.Ws[j][lane], Qj = sh.We[j][lane];
        const C Sj = sh.Ys[j][lane], Pj = sh.Ye[j][lane];
        sh.Ye[j][lane] = mk<T>(Pj.x + Qj * xs.x, Pj.y + Qj * xs.y);
        xs = mk<T>(Sj.x + Tj * xs.x, Sj.y + Tj * xs.y);
        sh.Ys[j][lane] = xs;
    }
}

// Back-substitution of rows s..s+ns-1 from the neighbours' solved boundary values xl =
// x_{s-1}, xr = x_{e+1}; stores p_hat and the dpdz spectrum, and on segment 0 the Neumann
// ghost level below the wall (:313-315).
template <typename T, bool IN = false>
__device__ __forceinline__ void seg_backsub(const C2<T> (&y)[kRegLev], const T (&cp)[kRegLev], const T (&vp)[kRegLev],
                                            C2<T> xl, C2<T> xr, int s, int ns_, int k, int L, C2<T> *ph, C2<T> *dph,
                                            long long S, T dz, T rdz, C2<T> hz0)
{
    using C = C2<T>;
    const int ns = IN ? kRegLev : ns_;
    // checked build: the segment's rows lie in 1..L
    if (OBL_CHECK && !(ck_in(s - 1, L, CK_TDMA_STORE) && ck_in(s + ns - 1, L + 1, CK_TDMA_STORE))) return;
    C x = mk<T>(0, 0);
#pragma unroll
    for (int i = kRegLev - 1; i >= 0; --i) {
        if (i == ns - 1) {
            x = mk<T>(y[i].x + vp[i] * xl.x - cp[i] * xr.x, y[i].y + vp[i] * xl.y - cp[i] * xr.y);
            ph[S * (s + i)] = x;
        } else if (i < ns - 1) {
            const C xi = mk<T>(y[i].x + vp[i] * xl.x - cp[i] * x.x, y[i].y + vp[i] * xl.y - cp[i] * x.y);
            ph[S * (s + i)] = xi;
            if (dph) dph[S * (s + i + 1)] = mk<T>((x.x - xi.x) * rdz, (x.y - xi.y) * rdz);
            x = xi;
        }
    }
    if (k > 0) {
        if (dph) dph[S * s] = mk<T>((x.x - xl.x) * rdz, (x.y - xl.y) * rdz);
    } else {
        const C p0 = mk<T>(x.x - dz * hz0.x, x.y - dz * hz0.y);
        ph[0] = p0;
        if (dph) dph[S] = mk<T>((x.x - p0.x) / dz, (x.y - p0.y) / dz);
    }
}

// Nyquist columns: p_hat = 0 at every level (:303-305)
template <typename T>
__device__ __forceinline__ void seg_nyquist(C2<T> *ph, C2<T> *dph, long long S, int s, int ns, int k, int L)
{
    if (ns <= 0) return;   // idle warp
    if (OBL_CHECK && !(ck_in(s - 1, L, CK_TDMA_STORE) && ck_in(s + ns - 1, L + 1, CK_TDMA_STORE))) return;
    for (int i = 0; i < ns; ++i) {
        ph[S * (s + i)] = mk<T>(0, 0);
        if (dph) dph[S * (s + i)] = mk<T>(0, 0);
    }
    if (k == 0) ph[0] = mk<T>(0, 0);
}

// NSEG segments (warps) per column; 16 / NSEG CTAs per SM, so fewer levels run with
// smaller CTAs that overlap one another's load, solve and store phases
template <typename T, int NSEG, bool G>
__global__ void __launch_bounds__(32 * NSEG, kRegSegMax / NSEG) k_tdma_reg(TdmaArgs<T> a, IslandArgs isl, int nbi,
                                                                          int Ls, int K)
{
    using C = C2<T>;
    if ((int)blockIdx.x < nbi) {
        tdma_column<T, double, true, G>(a, isl, (long long)blockIdx.x * blockDim.x + threadIdx.x);
        return;
    }
    __shared__ SegShared<T, NSEG> sh;
    const int lane = threadIdx.x & 31, k = threadIdx.x >> 5;
    const long long S = a.S;
    const int L = a.L;
    SegCol<T> c;
    c.init(a, (long long)(blockIdx.x - nbi) * 32, lane);
    const long long q = c.q;
    const int s = 1 + k * Ls;                                   // first row of the segment
    const int ns = k < K ? min(Ls, L - s + 1) : 0;              // its rows (0: idle warp)
    const bool interior = ns == kRegLev && s > 1 && s + kRegLev - 1 < L;   // warp-uniform
    C *ph = a.phat + q;
    C *dph = a.dph ? a.dph + q : nullptr;
    if (c.nyq) seg_nyquist<T>(ph, dph, S, s, ns, k, L);

    const T dz = (T)a.dz, idz = (T)(1.0 / a.dz), idz2 = (T)(1.0 / (a.dz * a.dz));
    const bool top_solved = a.neumann_top;      // else row L is p_hat(L) = 0 (npz = 1 mode)

    C y[kRegLev];
    T cp[kRegLev], vp[kRegLev];
    C hz0 = mk<T>(0, 0);
    if (c.act && ns > 0) {
        // right-hand sides of rows s..s+ns-1.  Every load is issued without a condition
        // (levels past the segment clamp to level L+1 and are not used), so all of the
        // segment's loads are in flight together.
        hz0 = a.Hz[q];   // RHS_col(0) = H_z(0) (:209), used by segment 0
        C hx[kRegLev], hy[kRegLev];
#pragma unroll
        for (int i = 0; i < kRegLev; ++i) {
            const long long zz = min(s + i, L);
            hx[i] = __ldcs(a.Hx + q + S * zz);
            hy[i] = __ldcs(a.Hy + q + S * zz);
        }
        if constexpr (G) {
            // G + i*ky*H_y; the (0,0) mode takes H_z's own (0,0) value (q = 0)
#pragma unroll
            for (int i = 0; i < kRegLev; ++i) {
                const int iz = s + i;
                C r = mk<T>(hx[i].x - c.ky * hy[i].y, hx[i].y + c.ky * hy[i].x);
                if (c.m00) r = (iz == 1) ? mk<T>(0, 0) : a.Hz[S * min(iz, L + 1)];
                if (iz == L && !top_solved) r = mk<T>(0, 0);
                y[i] = r;
            }
        } else {
            C hz[kRegLev + 1];
#pragma unroll
            for (int i = 0; i <= kRegLev; ++i) hz[i] = __ldcs(a.Hz + q + S * min(s + i, L + 1));
            if (interior) {
#pragma unroll
                for (int i = 0; i < kRegLev; ++i)
                    y[i] = seg_rhs<T, true>(c, s + i, L, top_solved, idz, hx[i], hy[i], hz[i], hz[i + 1], hz0);
            } else {
#pragma unroll
                for (int i = 0; i < kRegLev; ++i)
                    y[i] = seg_rhs<T>(c, s + i, L, top_solved, idz, hx[i], hy[i], hz[i], hz[i + 1], hz0);
            }
        }
        if (interior) seg_eliminate<T, NSEG, true>(c, y, cp, vp, s, ns, L, top_solved, idz, idz2, sh, k, lane);
        else seg_eliminate<T, NSEG>(c, y, cp, vp, s, ns, L, top_solved, idz, idz2, sh, k, lane);
    }
    __syncthreads();
    if (k == 0 && c.act) seg_reduced<T, NSEG>(sh, K, lane);
    __syncthreads();
    if (!c.act || ns == 0) return;
    const C xl = k > 0 ? sh.Ye[k - 1][lane] : mk<T>(0, 0);
    const C xr = k < K - 1 ? sh.Ys[k + 1][lane] : mk<T>(0, 0);
    if (interior) seg_backsub<T, true>(y, cp, vp, xl, xr, s, ns, k, L, ph, dph, S, dz, (T)(1.0 / a.dz), hz0);
    else seg_backsub<T>(y, cp, vp, xl, xr, s, ns, k, L, ph, dph, S, dz, (T)(1.0 / a.dz), hz0);
}

bool tdma_reg_supported(int L) { return L >= 1 && L <= kRegSegMax * kRegLev; }

template <typename T, int NSEG>
static void launch_tdma_reg_n(const TdmaArgs<T> &a, const IslandArgs &isl, cudaStream_t s, cudaError_t &e)
{
    constexpr int bs = 32 * NSEG;
    const int Ls = (a.L + NSEG - 1) / NSEG, K = (a.L + Ls - 1) / Ls;
    const int nbi = (int)((isl.n + bs - 1) / bs), nbb = (int)((a.S + 31) / 32);
    if (a.gform) k_tdma_reg<T, NSEG, true><<<(unsigned)(nbi + nbb), bs, 0, s>>>(a, isl, nbi, Ls, K);
    else k_tdma_reg<T, NSEG, false><<<(unsigned)(nbi + nbb), bs, 0, s>>>(a, isl, nbi, Ls, K);
    e = cudaGetLastError();
}

template <typename T>
void launch_tdma_reg(const TdmaArgs<T> &a, const IslandArgs &isl, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    // the fewest segments that keep every segment within kRegLev rows
    if (a.L > 8 * kRegLev) launch_tdma_reg_n<T, 16>(a, isl, s, e);
    else if (a.L > 4 * kRegLev) launch_tdma_reg_n<T, 8>(a, isl, s, e);
    else if (a.L > 2 * kRegLev) launch_tdma_reg_n<T, 4>(a, isl, s, e);
    else launch_tdma_reg_n<T, 2>(a, isl, s, e);
}
template void launch_tdma_reg<float>(const TdmaArgs<float> &, const IslandArgs &, cudaStream_t, cudaError_t &);

// ----------------------------------------------------------------------------- staged segmented solve
// The register-segmented solve as a persistent kernel whose RHS rows arrive by bulk
// asynchronous copies.  k_tdma_reg runs one 512-thread CTA per SM at 256 levels (128
// registers a thread), so its load, eliminate, reduced-solve and store phases follow one
// another and HBM idles while the SM computes.  Here each CTA walks units taken from a
// work counter (FP64 island units first, then 32-column groups) and, as soon as a warp has
// read its segment's rows of the current group out of shared memory, it starts the copies
// of the next group's rows into the same buffer: one cp.async.bulk per level and spectrum
// (256 contiguous bytes), completing on the warp's mbarrier.  The copies of group g+1 are
// in flight while group g is eliminated, reduced, back-substituted and stored.
//
// Buffer of warp k: kStageRows rows of 32 columns, H_x and H_y at levels s..s+15 and H_z
// at s..s+16 (levels past the segment clamp to L and L+1, as in k_tdma_reg).  Copies need
// 16-byte aligned addresses and sizes: the host launches this kernel only when S is even
// and the spectra are 16-byte aligned (a group's first column is then 256-byte aligned in
// every plane and a ragged last group copies an even number of 8-byte columns).
//
// Every wait is bounded: a warp whose copies have not landed after kStageWaitNs raises the
// error flag ctl[1] (the host reports OBL_ERR_TIMEOUT) and the CTA stops after the unit,
// waiting (bounded again) for the copies it still has in flight.  extra_tx (0 in the
// product path) is added to the bytes each wait expects: bytes no copy delivers, so that a
// test can make the waits run out and check the reported status.
constexpr int kStageRows = 3 * kRegLev + 1;
template <int NSEG>
__global__ void __launch_bounds__(32 * NSEG, kRegSegMax / NSEG) k_tdma_staged(TdmaArgs<float> a, IslandArgs isl, int nbi, int Ls,
                                                              int K, int *ctl, unsigned extra_tx)
{
    using T = float;
    using C = C2<T>;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ SegShared<T, NSEG> sh;
    __shared__ __align__(8) unsigned long long sBar[NSEG];
    __shared__ int sUnit[3];   // [it & 1]: the unit after next, fetched during unit it; [2]: grab()
    __shared__ int sAbort;
    const int lane = threadIdx.x & 31, k = threadIdx.x >> 5;
    const long long S = a.S;
    const int L = a.L;
    const long long nunits = nbi + (S + 31) / 32;
    const int s = 1 + k * Ls;
    const int ns = k < K ? min(Ls, L - s + 1) : 0;
    const bool interior = ns == kRegLev && s > 1 && s + kRegLev - 1 < L;   // warp-uniform
    C *buf = reinterpret_cast<C *>(smraw) + (size_t)k * kStageRows * 32;
    const unsigned bar = smem_addr(&sBar[k]);
    const T dz = (T)a.dz, idz = (T)(1.0 / a.dz), idz2 = (T)(1.0 / (a.dz * a.dz)), rdz = idz;
    const bool top_solved = a.neumann_top;

    if (lane == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    if (threadIdx.x == 0) sAbort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n\tfence.proxy.async.shared::cta;" ::: "memory");
    auto grab = [&]() -> long long {
        __syncthreads();
        if (threadIdx.x == 0) sUnit[2] = atomicAdd(ctl, 1);
        __syncthreads();
        return sUnit[2];
    };

    // FP64 island units (the counter hands them out first): their sequential sweeps
    long long cur = grab();
    while (cur < nbi) {
        tdma_column<T, double, true, false>(a, isl, cur * blockDim.x + threadIdx.x);
        cur = grab();
    }
    if (cur >= nunits) return;
    long long nxt = grab();

    // copies of this warp's rows of group unit u into its buffer (after its reads of the
    // buffer: the proxy fence orders them before the async writes)
    auto issue = [&](long long u) {
        const long long q0 = (u - nbi) * 32;
        const unsigned rb = (unsigned)(8 * (S - q0 < 32 ? S - q0 : 32));
        // checked build: the group's columns lie in the plane (a skipped copy leaves the
        // wait to give up, which the host reports as well)
        if (OBL_CHECK && !(ck_in(q0, S, CK_TDMA_COPY) && ck_in(q0 + rb / 8 - 1, S, CK_TDMA_COPY))) return;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(rb * kStageRows + extra_tx)
                         : "memory");
        __syncwarp();
        for (int r = lane; r < kStageRows; r += 32) {
            const C *src = r < kRegLev       ? a.Hx + S * min(s + r, L)
                           : r < 2 * kRegLev ? a.Hy + S * min(s + r - kRegLev, L)
                                             : a.Hz + S * min(s + r - 2 * kRegLev, L + 1);
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             smem_addr(buf + r * 32)),
                         "l"(src + q0), "r"(rb), "r"(bar)
                         : "memory");
        }
    };

    unsigned parity = 0;
    bool pending = false;   // this warp has copies in flight
    if (ns > 0) {
        issue(cur);
        pending = true;
    }
    for (int it = 0; cur < nunits; ++it) {
        if (threadIdx.x == 0) sUnit[it & 1] = atomicAdd(ctl, 1);
        const bool nxt_bulk = nxt < nunits;   // the counter only grows: nxt > cur >= nbi
        {
            SegCol<T> c;
            c.init(a, (cur - nbi) * 32, lane);
            const long long q = c.q;
            C *ph = a.phat + q;
            C *dph = a.dph ? a.dph + q : nullptr;
            const C hz0 = (k == 0 && c.act) ? a.Hz[q] : mk<T>(0, 0);
            C y[kRegLev];
            T cp[kRegLev], vp[kRegLev];
            if (ns > 0) {
                // warp-uniform outcome; after a timeout the phase stays pending (its copies
                // may still land) and no further copies are started
                const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(bar, parity));
                if (ok) {
                    parity ^= 1;
                    pending = false;
                } else if (lane == 0) {
                    atomicExch(ctl + 1, 1);
                    sAbort = 1;
                }
                if (c.act && interior) {
#pragma unroll
                    for (int i = 0; i < kRegLev; ++i)
                        y[i] = seg_rhs<T, true>(c, s + i, L, top_solved, idz, buf[i * 32 + lane],
                                                buf[(kRegLev + i) * 32 + lane], buf[(2 * kRegLev + i) * 32 + lane],
                                                buf[(2 * kRegLev + i + 1) * 32 + lane], hz0);
                } else if (c.act) {
#pragma unroll
                    for (int i = 0; i < kRegLev; ++i)
                        y[i] = seg_rhs<T>(c, s + i, L, top_solved, idz, buf[i * 32 + lane], buf[(kRegLev + i) * 32 + lane],
                                          buf[(2 * kRegLev + i) * 32 + lane], buf[(2 * kRegLev + i + 1) * 32 + lane], hz0);
                }
                if (nxt_bulk && ok) {
                    issue(nxt);
                    pending = true;
                }
                if (c.nyq) seg_nyquist<T>(ph, dph, S, s, ns, k, L);
                if (c.act && interior) seg_eliminate<T, NSEG, true>(c, y, cp, vp, s, ns, L, top_solved, idz, idz2, sh, k, lane);
                else if (c.act) seg_eliminate<T, NSEG>(c, y, cp, vp, s, ns, L, top_solved, idz, idz2, sh, k, lane);
            }
            __syncthreads();
            if (k == 0 && c.act) seg_reduced<T, NSEG>(sh, K, lane);
            __syncthreads();
            const C xl = k > 0 ? sh.Ye[k - 1][lane] : mk<T>(0, 0);
            const C xr = k < K - 1 ? sh.Ys[k + 1][lane] : mk<T>(0, 0);
            __syncthreads();   // the next unit's boundary rows overwrite sh
            if (c.act && interior) seg_backsub<T, true>(y, cp, vp, xl, xr, s, ns, k, L, ph, dph, S, dz, rdz, hz0);
            else if (c.act && ns > 0) seg_backsub<T>(y, cp, vp, xl, xr, s, ns, k, L, ph, dph, S, dz, rdz, hz0);
        }
        cur = nxt;
        nxt = sUnit[it & 1];
        if (sAbort) break;
    }
    // copies still in flight (a stop after a timed-out wait) land before the CTA exits
    if (pending) mbar_wait_bounded(bar, parity);
}

bool tdma_staged_supported(const TdmaArgs<float> &a)
{
    const auto al = [](const void *p) { return ((uintptr_t)p % 16) == 0; };
    return tdma_reg_supported(a.L) && !a.gform && a.S % 2 == 0 && al(a.Hx) && al(a.Hy) && al(a.Hz);
}

template <int NSEG>
static void launch_tdma_staged_n(const TdmaArgs<float> &a, const IslandArgs &isl, int *ctl, unsigned extra_tx,
                                 cudaStream_t s, cudaError_t &e)
{
    constexpr int bs = 32 * NSEG;
    const size_t smem = sizeof(C2<float>) * (size_t)NSEG * kStageRows * 32;
    static int residents[kMaxDevices] = {};   // CTAs resident on the whole GPU
    const int ds = device_slot();
    int resident = ds >= 0 ? residents[ds] : 0;
    if (!resident) {
        e = cudaFuncSetAttribute(k_tdma_staged<NSEG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return;
        int dev = 0, nsm = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_tdma_staged<NSEG>, bs, smem);
        resident = nsm * (per > 0 ? per : 1);
        if (ds >= 0) residents[ds] = resident;
    }
    const int Ls = (a.L + NSEG - 1) / NSEG, K = (a.L + Ls - 1) / Ls;
    const int nbi = (int)((isl.n + bs - 1) / bs);
    const long long nunits = nbi + (a.S + 31) / 32;
    const int grid = (int)(nunits < resident ? nunits : resident);
    if (grid < 1) return;
    e = cudaMemsetAsync(ctl, 0, sizeof(int), s);   // the work counter
    if (e != cudaSuccess) return;
    k_tdma_staged<NSEG><<<grid, bs, smem, s>>>(a, isl, nbi, Ls, K, ctl, extra_tx);
    e = cudaGetLastError();
}

void launch_tdma_staged(const TdmaArgs<float> &a, const IslandArgs &isl, int *ctl, unsigned extra_tx, cudaStream_t s,
                        cudaError_t &e)
{
    if (e != cudaSuccess) return;
    if (a.L > 8 * kRegLev) launch_tdma_staged_n<16>(a, isl, ctl, extra_tx, s, e);
    else if (a.L > 4 * kRegLev) launch_tdma_staged_n<8>(a, isl, ctl, extra_tx, s, e);
    else if (a.L > 2 * kRegLev) launch_tdma_staged_n<4>(a, isl, ctl, extra_tx, s, e);
    else launch_tdma_staged_n<2>(a, isl, ctl, extra_tx, s, e);
}

// ----------------------------------------------------------------------------- streaming
// The level kernels run over (level, x-vector, y) with VW consecutive x per access (2
// when every pointer is aligned to 2 elements: ldx is even, so a row starts on a
// 2-element boundary).  blockIdx.y is the level; each thread strides over the plane,
// several vectors per thread, so a 512x512 plane is about a hundred blocks.
static inline dim3 fgrid(int ldx, int nyt, int nlev) { return dim3((ldx + 127) / 128, nyt, nlev); }

template <typename T, int VW> struct alignas(sizeof(T) * VW) Vec {
    T v[VW];
};
static constexpr int kPlaneVecsPerThread = 4;
static inline dim3 lgrid(int ldx, int nyt, int vw, int nlev)
{
    const long long n = (long long)(ldx / vw) * nyt, per = 256LL * kPlaneVecsPerThread;
    return dim3((unsigned)((n + per - 1) / per), (unsigned)nlev);
}
template <int VW, typename... P> static inline bool aligned(P... p)
{
    return ((((uintptr_t)p) % (VW * sizeof(*p)) == 0) && ...);
}

enum ZOp : int { Z_UV = 0, Z_W = 1, Z_DPDZ = 2 };

// Z_UV (004_derivatives.f90:98-113, single rank): level 0 BOGUS, levels 2..nz-1
//      cst*(fun(z) - fun(z-1)), levels 1 and nz untouched;
// Z_W (004_derivatives.f90:168-180, single rank): level 0 BOGUS, nz zero, levels 1..nz-1
//      cst*(fun(z+1) - fun(z));
// Z_DPDZ (103_flosol.f90:174-175): dpdz(jz) = (p(jz) - p(jz-1))/dz, jz = 1..nz-1, in slot jz-1.
// Level z of the grid is blockIdx.y (+1 for Z_DPDZ); x >= nxt is written only on the
// whole-plane BOGUS / zero levels.
template <typename T, int VW, int OP>
__global__ void __launch_bounds__(256) k_zdiff(T *__restrict__ out, const T *__restrict__ in, int nxt, int ldx,
                                               int nyt, int nz, T c)
{
    using V = Vec<T, VW>;
    const int hp = ldx / VW, ip = nxt / VW;
    const int npl = hp * nyt;   // vectors per plane
    const int z = blockIdx.y + (OP == Z_DPDZ ? 1 : 0);
    const V *vi = reinterpret_cast<const V *>(in);
    V *vo = reinterpret_cast<V *>(out);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npl; q += gridDim.x * blockDim.x) {
        const bool inner = q % hp < ip;
        V r;
        if (OP != Z_DPDZ && (z == 0 || (OP == Z_W && z == nz))) {
#pragma unroll
            for (int k = 0; k < VW; ++k) r.v[k] = (z == 0) ? (T)kBogus : (T)0;
            vo[(long long)npl * z + q] = r;
            continue;
        }
        if (!inner) continue;
        if (OP == Z_UV && (z < 2 || z > nz - 1)) continue;
        const int zh = (OP == Z_W) ? z + 1 : z, zl = zh - 1;
        const V a = vi[(long long)npl * zh + q], b = vi[(long long)npl * zl + q];
#pragma unroll
        for (int k = 0; k < VW; ++k) r.v[k] = (OP == Z_DPDZ) ? (a.v[k] - b.v[k]) / c : c * (a.v[k] - b.v[k]);
        vo[(long long)npl * (OP == Z_DPDZ ? z - 1 : z) + q] = r;
    }
}

template <typename T, int OP>
static void launch_zdiff(T *out, const T *in, int nxt, int ldx, int nyt, int nz, int nlev, T c, cudaStream_t s,
                         cudaError_t &e)
{
    if (e != cudaSuccess) return;
    if (aligned<2>(out, in))
        k_zdiff<T, 2, OP><<<lgrid(ldx, nyt, 2, nlev), 256, 0, s>>>(out, in, nxt, ldx, nyt, nz, c);
    else
        k_zdiff<T, 1, OP><<<lgrid(ldx, nyt, 1, nlev), 256, 0, s>>>(out, in, nxt, ldx, nyt, nz, c);
    e = cudaGetLastError();
}

template <typename T, int VW>
__global__ void __launch_bounds__(256) k_project(T *__restrict__ u, T *__restrict__ v, T *__restrict__ w,
                                                 const T *__restrict__ dpdx, const T *__restrict__ dpdy,
                                                 const T *__restrict__ dpdz, int nxt, int ldx, int nyt, T dt)
{
    // 110_project.f90:16-40 (jz_min = 2 on the bottom rank); level z = blockIdx.y + 1
    using V = Vec<T, VW>;
    const int hp = ldx / VW, ip = nxt / VW, z = blockIdx.y + 1;
    const int npl = hp * nyt;
    const T t1 = (T)kTadv1;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npl; q += gridDim.x * blockDim.x) {
        if (q % hp >= ip) continue;
        const long long o = (long long)npl * z + q, od = (long long)npl * (z - 1) + q;
        V *U = reinterpret_cast<V *>(u) + o, *Vv = reinterpret_cast<V *>(v) + o, *W = reinterpret_cast<V *>(w) + o;
        const V px = reinterpret_cast<const V *>(dpdx)[od], py = reinterpret_cast<const V *>(dpdy)[od];
        V a = *U, b = *Vv;
#pragma unroll
        for (int k = 0; k < VW; ++k) {
            T rhs = -t1 * px.v[k];
            a.v[k] = a.v[k] + dt * rhs;
            rhs = -t1 * py.v[k];
            b.v[k] = b.v[k] + dt * rhs;
        }
        *U = a;
        *Vv = b;
        if (z >= 2) {
            const V pz = reinterpret_cast<const V *>(dpdz)[od];
            V cw = *W;
#pragma unroll
            for (int k = 0; k < VW; ++k) {
                const T rhs = -t1 * pz.v[k];
                cw.v[k] = cw.v[k] + dt * rhs;
            }
            *W = cw;
        }
    }
}

template <typename T>
__global__ void k_project_bc(T *u, T *v, T *w, int ldx, int nyt, int nz, int stress_free)
{
    // 110_project.f90:50-60
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= ldx) return;
    const long long pl = (long long)ldx * nyt, o = (long long)y * ldx + x;
    if (stress_free) {
        u[o + pl * (nz - 1)] = u[o + pl * (nz - 2)];
        v[o + pl * (nz - 1)] = v[o + pl * (nz - 2)];
    }
    w[o + pl * nz] = (T)0;
    w[o + pl * 1] = (T)0;
}

template <typename T>
void launch_ddz_uv(T *dfdz, const T *fun, int nxt, int ldx, int nyt, int nz, double dz,
                   cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    launch_zdiff<T, Z_UV>(dfdz, fun, nxt, ldx, nyt, nz, nz + 1, (T)(1.0 / dz), s, e);
}
template <typename T>
void launch_ddz_w(T *dfdz, const T *fun, int nxt, int ldx, int nyt, int nz, double dz,
                  cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    launch_zdiff<T, Z_W>(dfdz, fun, nxt, ldx, nyt, nz, nz + 1, (T)(1.0 / dz), s, e);
}
template <typename T>
void launch_dpdz(T *dpdz, const T *p, int nxt, int ldx, int nyt, int nz, double dz,
                 cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    launch_zdiff<T, Z_DPDZ>(dpdz, p, nxt, ldx, nyt, nz, nz - 1, (T)dz, s, e);
}
template <typename T>
void launch_project(T *u, T *v, T *w, const T *dpdx, const T *dpdy, const T *dpdz, int nxt,
                    int ldx, int nyt, int nz, double dt, int stress_free, cudaStream_t s,
                    cudaError_t &e)
{
    if (e != cudaSuccess) return;
    if (aligned<2>(u, v, w, dpdx, dpdy, dpdz))
        k_project<T, 2><<<lgrid(ldx, nyt, 2, nz - 1), 256, 0, s>>>(u, v, w, dpdx, dpdy, dpdz, nxt, ldx, nyt, (T)dt);
    else
        k_project<T, 1><<<lgrid(ldx, nyt, 1, nz - 1), 256, 0, s>>>(u, v, w, dpdx, dpdy, dpdz, nxt, ldx, nyt, (T)dt);
    e = cudaGetLastError();
    if (e != cudaSuccess) return;
    k_project_bc<T><<<fgrid(ldx, nyt, 1), 128, 0, s>>>(u, v, w, ldx, nyt, nz, stress_free);
    e = cudaGetLastError();
}

template <typename T>
void launch_project_bc(T *u, T *v, T *w, int ldx, int nyt, int nz, int stress_free, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_project_bc<T><<<fgrid(ldx, nyt, 1), 128, 0, s>>>(u, v, w, ldx, nyt, nz, stress_free);
    e = cudaGetLastError();
}

__global__ void k_d2f(float *d, const double *s, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = (float)s[i];
}
__global__ void k_f2d(double *d, const float *s, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = (double)s[i];
}
static inline unsigned cgrid(long long n)
{
    long long g = (n + 255) / 256;
    return (unsigned)(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}
void launch_convert_d2f(float *dst, const double *src, long long n, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess || n <= 0) return;
    k_d2f<<<cgrid(n), 256, 0, s>>>(dst, src, n);
    e = cudaGetLastError();
}
void launch_convert_f2d(double *dst, const float *src, long long n, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess || n <= 0) return;
    k_f2d<<<cgrid(n), 256, 0, s>>>(dst, src, n);
    e = cudaGetLastError();
}

#define OBL_INST(T)                                                                                  \
    template void launch_tdma<T>(const TdmaArgs<T> &, cudaStream_t, cudaError_t &);                  \
    template void launch_tdma_island<T>(const TdmaArgs<T> &, const IslandArgs &, cudaStream_t,      \
                                        cudaError_t &);                                              \
    template void launch_ddz_uv<T>(T *, const T *, int, int, int, int, double, cudaStream_t,        \
                                   cudaError_t &);                                                   \
    template void launch_ddz_w<T>(T *, const T *, int, int, int, int, double, cudaStream_t,         \
                                  cudaError_t &);                                                    \
    template void launch_dpdz<T>(T *, const T *, int, int, int, int, double, cudaStream_t,          \
                                 cudaError_t &);                                                     \
    template void launch_project_bc<T>(T *, T *, T *, int, int, int, int, cudaStream_t, cudaError_t &); \
    template void launch_project<T>(T *, T *, T *, const T *, const T *, const T *, int, int, int,  \
                                    int, double, int, cudaStream_t, cudaError_t &);
OBL_INST(float)
OBL_INST(double)

} // namespace obl
