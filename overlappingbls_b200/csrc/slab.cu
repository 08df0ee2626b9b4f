// slab.cu -- partitioned Thomas solve of a z-slab (see slab.cuh).
//
// One thread per (kx,ky) column, consecutive threads on consecutive kx, so every level's
// loads and stores are coalesced along the contiguous kx index.  The bands and the
// right-hand side follow init_coef_press and press_stag_array (109_press_stag_array.f90:
// 4-68, 203-225) in the npz >= 2 form: Neumann rows at the bottom of rank 0 and at the
// top of rank P-1, and the first-order integration of the (0,0) mean mode.
#include "slab.cuh"

#include <type_traits>

namespace obl {

#ifndef OBL_SLAB_AHEAD
#define OBL_SLAB_AHEAD 2
#endif
#ifndef OBL_SLAB_BACK
#define OBL_SLAB_BACK 2
#endif
#ifndef OBL_SLAB_MINB
#define OBL_SLAB_MINB 8
#endif
// Every column of the slab is in flight at once and each thread walks its column level
// after level, so the sweeps are load-latency bound: the loads of the next kSlabAhead
// levels (kSlabBack on the downward passes) are held in register rings in their stored
// type and converted when used.  Deeper rings cost registers, and below 64 registers a
// thread the eight 4-warp blocks per SM that hide the latency no longer fit.
constexpr int kSlabAhead = OBL_SLAB_AHEAD;
constexpr int kSlabBack = OBL_SLAB_BACK;

// Where one column keeps its eliminated rows: the bulk in the storage type (y' in the
// p_hat planes 1..L, c' and v' in (S, L) scratch), an island column in FP64 (n_isl, L).
template <typename T, bool ISLAND> struct SlabRows {
    using RS = typename std::conditional<ISLAND, double, T>::type;
    C2<RS> *y;
    RS *c, *v;
    long long yo, o, st;   // y'_j at y[yo + st*j], c'_j and v'_j at [o + st*j]
    __device__ SlabRows(const SlabArgs<T> &a, long long q, long long t)
    {
        if constexpr (ISLAND) {
            y = a.iy; c = a.icp; v = a.iv; st = a.n_isl; o = t - st; yo = t - st;
        } else {
            y = a.phat; c = a.cp; v = a.v; st = a.S; o = q - st; yo = q;
        }
    }
};

// Column index of thread t, or -1 when the thread has no column of this kind.
template <typename T, bool ISLAND> __device__ __forceinline__ long long slab_col(const SlabArgs<T> &a, long long t)
{
    if constexpr (ISLAND) {
        return t < a.n_isl ? (long long)a.isl_cols[t] : -1;
    } else {
        if (t >= a.S) return -1;
        return (a.isl_slot && a.isl_slot[t] >= 0) ? -1 : t;   // solved by an island thread
    }
}

// Pass over levels L-1 .. 1 reading (c'_j, y'_j, v'_j) through the ring; f(j, c', y', v').
template <typename T, typename TC, bool ISLAND, typename F>
__device__ __forceinline__ void slab_down(const SlabRows<T, ISLAND> &R, int L, F f)
{
    using RS = typename SlabRows<T, ISLAND>::RS;
    constexpr int PF = kSlabBack;
    RS rc[PF], rv[PF];
    C2<RS> ry[PF];
    auto fill = [&](int s, int j) {
        j = j >= 1 ? j : 1;
        rc[s] = R.c[R.o + R.st * j];
        rv[s] = R.v[R.o + R.st * j];
        ry[s] = R.y[R.yo + R.st * j];
    };
#pragma unroll
    for (int s = 0; s < PF; ++s) fill(s, L - 1 - s);
    for (int base = 0; base < L - 1; base += PF) {
#pragma unroll
        for (int s = 0; s < PF; ++s) {
            const int j = L - 1 - (base + s);
            if (j < 1) break;
            const TC c = (TC)rc[s], v = (TC)rv[s];
            const C2<TC> y = mk<TC>((TC)ry[s].x, (TC)ry[s].y);
            fill(s, j - PF);
            f(j, c, y, v);
        }
    }
}

// The rank's forward elimination of one column in precision TC and its interface values.
template <typename T, typename TC, bool ISLAND>
__device__ __forceinline__ void slab_column(const SlabArgs<T> &a, long long t)
{
    using CC = C2<TC>;
    using CS = C2<T>;
    const long long q = slab_col<T, ISLAND>(a, t);
    if (q < 0) return;
    const long long S = a.S;
    const int L = a.L;
    // interface values field-major, (kSlabIface, S): each store and load is coalesced
    auto fset = [&](int k, double v) { a.iface[(long long)k * S + q] = v; };
    const int ix = (int)(q % a.lhx), iy = (int)(q / a.lhx);
    if (ix == a.lhx - 1 || iy == a.nyt / 2) {   // Nyquist columns: p_hat = 0
        for (int k = 0; k < kSlabIface; ++k) fset(k, 0.0);
        return;
    }
    const double kxd = a.kx[ix], kyd = a.ky[iy], k2d = kxd * kxd + kyd * kyd;
    const bool m00 = k2d == 0.0;
    const bool bot = a.rank == 0, topr = a.rank == a.nranks - 1;
    const TC kx = (TC)kxd, ky = (TC)kyd, k2 = (TC)k2d;
    const TC dz = (TC)a.dz, idz = (TC)(1.0 / a.dz), idz2 = (TC)(1.0 / (a.dz * a.dz));
    const SlabRows<T, ISLAND> R(a, q, t);
    using RS = typename SlabRows<T, ISLAND>::RS;
    auto raw = [&](const CS *p, int z) -> CS { return p[q + S * z]; };
    auto cv = [&](CS v) -> CC { return mk<TC>((TC)v.x, (TC)v.y); };

    // ---- forward elimination; RHS inputs through a ring (slot s: level base+s) ----
    constexpr int PF = kSlabAhead;
    const CC hz0 = cv(raw(a.Hz, 0));
    CS rx[PF], ry[PF], rz[PF];
#pragma unroll
    for (int s = 0; s < PF; ++s) {
        const int z = 1 + s;
        rx[s] = raw(a.Hx, z <= L ? z : L);
        ry[s] = raw(a.Hy, z <= L ? z : L);
        rz[s] = raw(a.Hz, z <= L + 1 ? z : L + 1);
    }
    TC cprev = 0, vp = 0, wl = 0;
    CC yp = mk<TC>(0, 0);
    for (int base = 1; base <= L; base += PF) {
#pragma unroll
        for (int s = 0; s < PF; ++s) {
            const int j = base + s;
            if (j > L) break;
            const CC hx = cv(rx[s]), hy = cv(ry[s]), hzc = cv(rz[s]);
            const CC hzn = cv(rz[(s + 1) % PF]);   // level j+1 (slot 0 was refilled at s = 0)
            {
                const int zn = j + PF;
                rx[s] = raw(a.Hx, zn <= L ? zn : L);
                ry[s] = raw(a.Hy, zn <= L ? zn : L);
                rz[s] = raw(a.Hz, zn <= L + 1 ? zn : L + 1);
            }
            const bool b1 = bot && j == 1, tl = topr && j == L;
            TC am, bm, cm;
            CC r;
            if (!m00) {
                am = b1 ? (TC)0 : idz2;
                cm = tl ? (TC)0 : idz2;
                bm = (b1 || tl) ? -(k2 + idz2) : -(k2 + (TC)2 * idz2);
                TC dx = hzn.x - hzc.x, dy = hzn.y - hzc.y;
                if (b1) {
                    dx += hz0.x;
                    dy += hz0.y;
                }
                const TC sx = kx * hx.x + ky * hy.x, sy = kx * hx.y + ky * hy.y;
                r = mk<TC>(-sy + dx / dz, sx + dy / dz);
            } else {
                am = b1 ? (TC)0 : -idz;
                bm = idz;
                cm = 0;
                r = b1 ? mk<TC>(0, 0) : hzc;
            }
            const TC asub = j == 1 ? (TC)0 : am;   // a_1 couples to the rank below
            const TC iden = (TC)1 / (bm - asub * cprev);
            const TC cpj = j == L ? (TC)0 : cm * iden;   // c_L couples to the rank above
            yp = mk<TC>((r.x - asub * yp.x) * iden, (r.y - asub * yp.y) * iden);
            vp = ((j == 1 ? am : (TC)0) - asub * vp) * iden;
            if (j == L) wl = cm * iden;
            R.c[R.o + R.st * j] = (RS)cpj;
            R.v[R.o + R.st * j] = (RS)vp;
            R.y[R.yo + R.st * j] = mk<RS>((RS)yp.x, (RS)yp.y);
            cprev = cpj;
        }
    }
    fset(2, yp.x);
    fset(3, yp.y);
    fset(5, vp);
    fset(7, wl);
    // ---- end values at row 1: y_j = y'_j - c'_j y_{j+1}, likewise v; w_j = -c'_j w_{j+1} ----
    CC yn = yp;
    TC vn = vp, wn = wl;
    slab_down<T, TC, ISLAND>(R, L, [&](int, TC c, CC y, TC v) {
        yn = mk<TC>(y.x - c * yn.x, y.y - c * yn.y);
        vn = v - c * vn;
        wn = -c * wn;
    });
    fset(0, yn.x);
    fset(1, yn.y);
    fset(4, vn);
    fset(6, wn);
}

// island blocks first (their FP64 sweeps are the longest), then the bulk columns
template <typename T>
__global__ void __launch_bounds__(128, OBL_SLAB_MINB) k_slab_solve(SlabArgs<T> a, int nbi)
{
    if ((int)blockIdx.x < nbi)
        slab_column<T, double, true>(a, (long long)blockIdx.x * blockDim.x + threadIdx.x);
    else
        slab_column<T, T, false>(a, (long long)(blockIdx.x - nbi) * blockDim.x + threadIdx.x);
}

// Back substitution of one column, the neighbours' interface unknowns known, in precision TC.
template <typename T, typename TC, bool ISLAND>
__device__ __forceinline__ void slab_rows_out(const SlabArgs<T> &a, long long q, long long t, double2 below,
                                              double2 above, double wl)
{
    using CC = C2<TC>;
    const long long S = a.S;
    const int L = a.L;
    const SlabRows<T, ISLAND> R(a, q, t);
    C2<T> *ph = a.phat + q, *dph = a.dph + q;
    const CC xb = mk<TC>((TC)below.x, (TC)below.y), xa = mk<TC>((TC)above.x, (TC)above.y);
    const TC rdz = (TC)(1.0 / a.dz);
    // row L: x_L = y'_L - v'_L x_below - w'_L x_above
    const auto yl = R.y[R.yo + R.st * L];
    const TC vl = (TC)R.v[R.o + R.st * L], w = (TC)wl;
    CC xn = mk<TC>((TC)yl.x - vl * xb.x - w * xa.x, (TC)yl.y - vl * xb.y - w * xa.y);
    ph[S * L] = mk<T>((T)xn.x, (T)xn.y);
    slab_down<T, TC, ISLAND>(R, L, [&](int j, TC c, CC y, TC v) {
        const CC x = mk<TC>(y.x - v * xb.x - c * xn.x, y.y - v * xb.y - c * xn.y);
        ph[S * j] = mk<T>((T)x.x, (T)x.y);
        dph[S * (j + 1)] = mk<T>((T)((xn.x - x.x) * rdz), (T)((xn.y - x.y) * rdz));
        xn = x;
    });
    // p_hat(0): the last unknown of the rank below, or on rank 0 the Neumann ghost
    // p_hat(1) - dz*H_z(0) (109_press_stag_array.f90:313-315)
    CC x0 = xb;
    if (a.rank == 0) {
        const C2<T> h = a.Hz[q];
        const TC dz = (TC)a.dz;
        x0 = mk<TC>(xn.x - dz * (TC)h.x, xn.y - dz * (TC)h.y);
    }
    if (a.own_p0) ph[0] = mk<T>((T)x0.x, (T)x0.y);
    dph[S] = mk<T>((T)((xn.x - x0.x) * rdz), (T)((xn.y - x0.y) * rdz));
}

// The reduced interface system and the rank's rows of one column; t as in slab_column.
template <typename T, typename TC, bool ISLAND>
__device__ __forceinline__ void slab_finish_column(const SlabArgs<T> &a, long long t)
{
    const long long q = slab_col<T, ISLAND>(a, t);
    if (q < 0) return;
    const long long S = a.S;
    const int L = a.L, P = a.nranks, r = a.rank;
    const int ix = (int)(q % a.lhx), iy = (int)(q / a.lhx);
    C2<T> *ph = a.phat + q, *dph = a.dph + q;
    if (ix == a.lhx - 1 || iy == a.nyt / 2) {
        for (int z = a.own_p0 ? 0 : 1; z <= L; ++z) ph[S * z] = mk<T>(0, 0);
        for (int z = 1; z <= L; ++z) dph[S * z] = mk<T>(0, 0);
        return;
    }
    // interface unknowns X_k = (first_k, last_k):  X_k + A_k X_{k-1} + C_k X_{k+1} = Y_k,
    // A_k = [[0, v1],[0, vm]], C_k = [[w1, 0],[wm, 0]].  Twisted elimination, in registers:
    // upward from rank 0, X_k = Z_k - G_k X_{k+1}, where G_k has only a first column (g0, g1);
    // downward from rank P-1, X_k = Z'_k - H_k X_{k-1}, where H_k has only a second column
    // (h0, h1); the two meet at this rank's own 2x2 block.
    // rank k's record of this column; the next record's loads are issued before the
    // current one is used
    auto rec = [&](int k, double *f) {
#pragma unroll
        for (int j = 0; j < kSlabIface; ++j) f[j] = a.iface_all[((long long)k * kSlabIface + j) * S + q];
    };
    double cur[kSlabIface], nxt[kSlabIface];
    double g1 = 0.0;
    double2 z1 = make_double2(0.0, 0.0);   // last_{r-1} = z1 - g1 first_r
    if (r > 0) rec(0, cur);
    for (int k = 0; k < r; ++k) {
        if (k + 1 < r) rec(k + 1, nxt);
        const double v1 = cur[4], vm = cur[5], w1 = cur[6], wm = cur[7];
        // D = I - A_k G_{k-1} = [[1 - v1 g1, 0], [-vm g1, 1]]; rhs = Y_k - A_k Z_{k-1}
        const double d00 = 1.0 - v1 * g1, d10 = -vm * g1;
        const double2 r0 = make_double2(cur[0] - v1 * z1.x, cur[1] - v1 * z1.y);
        const double2 r1 = make_double2(cur[2] - vm * z1.x, cur[3] - vm * z1.y);
        const double i00 = 1.0 / d00;
        const double2 zz0 = make_double2(r0.x * i00, r0.y * i00);
        z1 = make_double2(r1.x - d10 * zz0.x, r1.y - d10 * zz0.y);
        g1 = wm - d10 * (w1 * i00);
#pragma unroll
        for (int j = 0; j < kSlabIface; ++j) cur[j] = nxt[j];
    }
    double h0 = 0.0;
    double2 z0 = make_double2(0.0, 0.0);   // first_{r+1} = z0 - h0 last_r
    if (r < P - 1) rec(P - 1, cur);
    for (int k = P - 1; k > r; --k) {
        if (k - 1 > r) rec(k - 1, nxt);
        const double v1 = cur[4], vm = cur[5], w1 = cur[6], wm = cur[7];
        // D' = I - C_k H_{k+1} = [[1, -w1 h0], [0, 1 - wm h0]]; rhs = Y_k - C_k Z'_{k+1}
        const double d01 = -w1 * h0, d11 = 1.0 - wm * h0;
        const double2 r0 = make_double2(cur[0] - w1 * z0.x, cur[1] - w1 * z0.y);
        const double2 r1 = make_double2(cur[2] - wm * z0.x, cur[3] - wm * z0.y);
        const double i11 = 1.0 / d11;
        const double2 zz1 = make_double2(r1.x * i11, r1.y * i11);
        z0 = make_double2(r0.x - d01 * zz1.x, r0.y - d01 * zz1.y);
        h0 = v1 - d01 * (vm * i11);
#pragma unroll
        for (int j = 0; j < kSlabIface; ++j) cur[j] = nxt[j];
    }
    // the rank's own block with both neighbours substituted
    double f[kSlabIface];
    rec(r, f);
    const double v1 = f[4], vm = f[5], w1 = f[6], wm = f[7];
    const double m00 = 1.0 - v1 * g1, m01 = -w1 * h0, m10 = -vm * g1, m11 = 1.0 - wm * h0;
    const double2 c0 = make_double2(f[0] - v1 * z1.x - w1 * z0.x, f[1] - v1 * z1.y - w1 * z0.y);
    const double2 c1 = make_double2(f[2] - vm * z1.x - wm * z0.x, f[3] - vm * z1.y - wm * z0.y);
    const double idet = 1.0 / (m00 * m11 - m01 * m10);
    const double2 first = make_double2((m11 * c0.x - m01 * c1.x) * idet, (m11 * c0.y - m01 * c1.y) * idet);
    const double2 last = make_double2((m00 * c1.x - m10 * c0.x) * idet, (m00 * c1.y - m10 * c0.y) * idet);
    const double2 below = make_double2(z1.x - g1 * first.x, z1.y - g1 * first.y);
    const double2 above = make_double2(z0.x - h0 * last.x, z0.y - h0 * last.y);
    slab_rows_out<T, TC, ISLAND>(a, q, t, below, above, wm);
}

// island blocks first, then the bulk columns (one walk per warp, as in the solve)
template <typename T>
__global__ void __launch_bounds__(128, OBL_SLAB_MINB) k_slab_finish(SlabArgs<T> a, int nbi)
{
    if ((int)blockIdx.x < nbi)
        slab_finish_column<T, double, true>(a, (long long)blockIdx.x * blockDim.x + threadIdx.x);
    else
        slab_finish_column<T, T, false>(a, (long long)(blockIdx.x - nbi) * blockDim.x + threadIdx.x);
}

// Segment r of a column split on one GPU: the segment's view of the whole column's arguments.
template <typename T> __device__ __forceinline__ SlabArgs<T> seg_view(const SlabArgs<T> &a, int r, int P, int seg)
{
    SlabArgs<T> b = a;
    const long long off = (long long)r * seg * a.S, ioff = (long long)r * seg * a.n_isl;
    b.Hx = a.Hx + off;
    b.Hy = a.Hy + off;
    b.Hz = a.Hz + off;
    b.phat = a.phat + off;
    b.dph = a.dph + off;
    b.v = a.v + off;
    b.cp = a.cp + off;
    b.iy = a.iy + ioff;
    b.iv = a.iv + ioff;
    b.icp = a.icp + ioff;
    b.iface = a.iface + (long long)r * a.S * kSlabIface;
    b.iface_all = a.iface;
    b.rank = r;
    b.nranks = P;
    b.L = (a.L - r * seg) < seg ? (a.L - r * seg) : seg;
    b.own_p0 = r == 0;
    return b;
}

template <typename T>
__global__ void __launch_bounds__(128, OBL_SLAB_MINB) k_seg_solve(SlabArgs<T> a, int nbi, int seg)
{
    const SlabArgs<T> b = seg_view(a, blockIdx.y, gridDim.y, seg);
    if ((int)blockIdx.x < nbi)
        slab_column<T, double, true>(b, (long long)blockIdx.x * blockDim.x + threadIdx.x);
    else
        slab_column<T, T, false>(b, (long long)(blockIdx.x - nbi) * blockDim.x + threadIdx.x);
}

template <typename T>
__global__ void __launch_bounds__(128, OBL_SLAB_MINB) k_seg_finish(SlabArgs<T> a, int nbi, int seg)
{
    const SlabArgs<T> b = seg_view(a, blockIdx.y, gridDim.y, seg);
    if ((int)blockIdx.x < nbi)
        slab_finish_column<T, double, true>(b, (long long)blockIdx.x * blockDim.x + threadIdx.x);
    else
        slab_finish_column<T, T, false>(b, (long long)(blockIdx.x - nbi) * blockDim.x + threadIdx.x);
}

template <typename T>
__global__ void k_project_bc_roles(T *u, T *v, T *w, int ldx, int nyt, int nz, int stress_free, int bottom, int top)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= ldx) return;
    const long long pl = (long long)ldx * nyt, o = (long long)y * ldx + x;
    if (top) {
        if (stress_free) {
            u[o + pl * (nz - 1)] = u[o + pl * (nz - 2)];
            v[o + pl * (nz - 1)] = v[o + pl * (nz - 2)];
        }
        w[o + pl * nz] = (T)0;
    }
    if (bottom) w[o + pl] = (T)0;
}

template <typename T> void launch_slab_solve(const SlabArgs<T> &a, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    const int nbi = (a.n_isl + 127) / 128, nbb = (int)((a.S + 127) / 128);
    k_slab_solve<T><<<(unsigned)(nbi + nbb), 128, 0, s>>>(a, nbi);
    e = cudaGetLastError();
}
template <typename T> void launch_slab_finish(const SlabArgs<T> &a, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    if (a.nranks < 1 || a.nranks > kSlabMaxRanks) {
        e = cudaErrorInvalidValue;
        return;
    }
    const int nbi = (a.n_isl + 127) / 128, nbb = (int)((a.S + 127) / 128);
    k_slab_finish<T><<<(unsigned)(nbi + nbb), 128, 0, s>>>(a, nbi);
    e = cudaGetLastError();
}
template <typename T> void launch_seg_solve(const SlabArgs<T> &a, int P, int seg, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    const int nbi = (a.n_isl + 127) / 128, nbb = (int)((a.S + 127) / 128);
    k_seg_solve<T><<<dim3((unsigned)(nbi + nbb), (unsigned)P), 128, 0, s>>>(a, nbi, seg);
    e = cudaGetLastError();
}
template <typename T> void launch_seg_finish(const SlabArgs<T> &a, int P, int seg, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    const int nbi = (a.n_isl + 127) / 128, nbb = (int)((a.S + 127) / 128);
    k_seg_finish<T><<<dim3((unsigned)(nbi + nbb), (unsigned)P), 128, 0, s>>>(a, nbi, seg);
    e = cudaGetLastError();
}
template <typename T> void launch_seg_solve_isl(const SlabArgs<T> &a, int P, int seg, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    const int nbi = (a.n_isl + 127) / 128;   // island blocks only: every block takes the FP64 branch
    if (nbi < 1) return;
    k_seg_solve<T><<<dim3((unsigned)nbi, (unsigned)P), 128, 0, s>>>(a, nbi, seg);
    e = cudaGetLastError();
}
template <typename T> void launch_seg_finish_isl(const SlabArgs<T> &a, int P, int seg, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    const int nbi = (a.n_isl + 127) / 128;
    if (nbi < 1) return;
    k_seg_finish<T><<<dim3((unsigned)nbi, (unsigned)P), 128, 0, s>>>(a, nbi, seg);
    e = cudaGetLastError();
}
template <typename T>
void launch_project_bc_roles(T *u, T *v, T *w, int ldx, int nyt, int nz, int stress_free, int bottom, int top,
                             cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_project_bc_roles<T><<<dim3((ldx + 127) / 128, nyt), 128, 0, s>>>(u, v, w, ldx, nyt, nz, stress_free, bottom, top);
    e = cudaGetLastError();
}

#define OBL_INST(T)                                                                                      \
    template void launch_slab_solve<T>(const SlabArgs<T> &, cudaStream_t, cudaError_t &);              \
    template void launch_slab_finish<T>(const SlabArgs<T> &, cudaStream_t, cudaError_t &);             \
    template void launch_seg_solve<T>(const SlabArgs<T> &, int, int, cudaStream_t, cudaError_t &);     \
    template void launch_seg_finish<T>(const SlabArgs<T> &, int, int, cudaStream_t, cudaError_t &);    \
    template void launch_seg_solve_isl<T>(const SlabArgs<T> &, int, int, cudaStream_t, cudaError_t &); \
    template void launch_seg_finish_isl<T>(const SlabArgs<T> &, int, int, cudaStream_t, cudaError_t &); \
    template void launch_project_bc_roles<T>(T *, T *, T *, int, int, int, int, int, int, cudaStream_t,   \
                                             cudaError_t &);
OBL_INST(float)
OBL_INST(double)

} // namespace obl
