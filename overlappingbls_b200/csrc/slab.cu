// slab.cu -- partitioned Thomas solve of a z-slab (see slab.cuh).
//
// One thread per (kx,ky) column, consecutive threads on consecutive kx, so every level's
// loads and stores are coalesced along the contiguous kx index.  The bands and the
// right-hand side follow init_coef_press and press_stag_array (109_press_stag_array.f90:
// 4-68, 203-225) in the npz >= 2 form: Neumann rows at the bottom of rank 0 and at the
// top of rank P-1, and the first-order integration of the (0,0) mean mode.
#include "slab.cuh"

namespace obl {

// The rank's rows of one column in precision TC; t = the column (bulk) or island index.
template <typename T, typename TC, bool ISLAND>
__device__ __forceinline__ void slab_column(const SlabArgs<T> &a, long long t)
{
    using CC = C2<TC>;
    long long q;
    if constexpr (ISLAND) {
        if (t >= a.n_isl) return;
        q = a.isl_cols[t];
    } else {
        if (t >= a.S) return;
        q = t;
        if (a.isl_slot && a.isl_slot[q] >= 0) return;   // solved by an island thread
    }
    const long long S = a.S;
    const int L = a.L;
    double *f = a.iface + q * kSlabIface;
    const int ix = (int)(q % a.lhx), iy = (int)(q / a.lhx);
    if (ix == a.lhx - 1 || iy == a.nyt / 2) {   // Nyquist columns: p_hat = 0
        for (int k = 0; k < kSlabIface; ++k) f[k] = 0.0;
        return;
    }
    const double kxd = a.kx[ix], kyd = a.ky[iy], k2d = kxd * kxd + kyd * kyd;
    const bool m00 = k2d == 0.0;
    const bool bot = a.rank == 0, topr = a.rank == a.nranks - 1;
    const TC kx = (TC)kxd, ky = (TC)kyd, k2 = (TC)k2d;
    const TC dz = (TC)a.dz, idz = (TC)(1.0 / a.dz), idz2 = (TC)(1.0 / (a.dz * a.dz));
    auto ld = [&](const C2<T> *p, int z) -> CC {
        const C2<T> v = p[q + S * z];
        return mk<TC>((TC)v.x, (TC)v.y);
    };
    auto o = [&](int j) -> long long { return ISLAND ? t + (long long)a.n_isl * (j - 1) : q + S * (j - 1); };
    auto st = [&](int j, TC cpj, CC yj, TC vj, TC wj) {
        const long long k = o(j);
        if constexpr (ISLAND) {
            a.icp[k] = cpj; a.iy[k] = make_double2(yj.x, yj.y); a.iv[k] = vj; a.iw[k] = wj;
        } else {
            a.cp[k] = (T)cpj; a.y[k] = mk<T>((T)yj.x, (T)yj.y); a.v[k] = (T)vj; a.w[k] = (T)wj;
        }
    };
    auto ldy = [&](int j) -> CC {
        if constexpr (ISLAND) { const double2 v = a.iy[o(j)]; return mk<TC>(v.x, v.y); }
        else { const C2<T> v = a.y[o(j)]; return mk<TC>((TC)v.x, (TC)v.y); }
    };
    auto lds = [&](const T *b, const double *ib, int j) -> TC {
        if constexpr (ISLAND) return ib[o(j)];
        else return (TC)b[o(j)];
    };
    const CC hz0 = ld(a.Hz, 0);
    TC cprev = 0, vp = 0, wp = 0;
    CC yp = mk<TC>(0, 0);
    for (int j = 1; j <= L; ++j) {
        const bool b1 = bot && j == 1, tl = topr && j == L;
        TC am, bm, cm;
        CC r;
        if (!m00) {
            am = b1 ? (TC)0 : idz2;
            cm = tl ? (TC)0 : idz2;
            bm = (b1 || tl) ? -(k2 + idz2) : -(k2 + (TC)2 * idz2);
            const CC hx = ld(a.Hx, j), hy = ld(a.Hy, j), hzc = ld(a.Hz, j), hzn = ld(a.Hz, j + 1);
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
            r = b1 ? mk<TC>(0, 0) : ld(a.Hz, j);
        }
        const TC asub = j == 1 ? (TC)0 : am;   // a_1 couples to the rank below
        const TC csup = j == L ? (TC)0 : cm;   // c_L couples to the rank above
        const TC iden = (TC)1 / (bm - asub * cprev);
        const TC cpj = csup * iden;
        yp = mk<TC>((r.x - asub * yp.x) * iden, (r.y - asub * yp.y) * iden);
        vp = ((j == 1 ? am : (TC)0) - asub * vp) * iden;
        wp = ((j == L ? cm : (TC)0) - asub * wp) * iden;
        st(j, cpj, yp, vp, wp);
        cprev = cpj;
    }
    CC yn = yp;
    TC vn = vp, wn = wp;
    f[2] = yn.x;
    f[3] = yn.y;
    f[5] = vn;
    f[7] = wn;
    for (int j = L - 1; j >= 1; --j) {
        const TC c = lds(a.cp, a.icp, j);
        const CC yj = ldy(j);
        yn = mk<TC>(yj.x - c * yn.x, yj.y - c * yn.y);
        vn = lds(a.v, a.iv, j) - c * vn;
        wn = lds(a.w, a.iw, j) - c * wn;
        st(j, c, yn, vn, wn);
    }
    f[0] = yn.x;
    f[1] = yn.y;
    f[4] = vn;
    f[6] = wn;
}

// island blocks first (their FP64 sweeps are the longest), then the bulk columns
template <typename T>
__global__ void __launch_bounds__(128) k_slab_solve(SlabArgs<T> a, int nbi)
{
    if ((int)blockIdx.x < nbi)
        slab_column<T, double, true>(a, (long long)blockIdx.x * blockDim.x + threadIdx.x);
    else
        slab_column<T, T, false>(a, (long long)(blockIdx.x - nbi) * blockDim.x + threadIdx.x);
}

template <typename T>
__global__ void __launch_bounds__(128) k_slab_finish(SlabArgs<T> a)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.S) return;
    const long long S = a.S;
    const int L = a.L, P = a.nranks, r = a.rank;
    const int ix = (int)(q % a.lhx), iy = (int)(q / a.lhx);
    C2<T> *ph = a.phat + q, *dph = a.dph + q;
    if (ix == a.lhx - 1 || iy == a.nyt / 2) {
        for (int z = 0; z <= L; ++z) ph[S * z] = mk<T>(0, 0);
        for (int z = 1; z <= L; ++z) dph[S * z] = mk<T>(0, 0);
        return;
    }
    // interface unknowns X_k = (first_k, last_k):  X_k + A_k X_{k-1} + C_k X_{k+1} = Y_k,
    // A_k = [[0, v1],[0, vm]], C_k = [[w1, 0],[wm, 0]]; block Thomas over k = 0..P-1.
    // G_k = D_k^-1 C_k has a zero second column: only (g0, g1) is kept.
    double g0[kSlabMaxRanks], g1[kSlabMaxRanks];
    double2 z0[kSlabMaxRanks], z1[kSlabMaxRanks];
    for (int k = 0; k < P; ++k) {
        const double *f = a.iface_all + ((long long)k * S + q) * kSlabIface;
        const double v1 = f[4], vm = f[5], w1 = f[6], wm = f[7];
        double d00 = 1.0, d01 = 0.0, d10 = 0.0, d11 = 1.0;
        double2 r0 = make_double2(f[0], f[1]), r1 = make_double2(f[2], f[3]);
        if (k > 0) {   // D = I - A G_{k-1}, rhs = Y - A Z_{k-1}
            d00 = 1.0 - v1 * g1[k - 1];
            d10 = -vm * g1[k - 1];
            r0 = make_double2(r0.x - v1 * z1[k - 1].x, r0.y - v1 * z1[k - 1].y);
            r1 = make_double2(r1.x - vm * z1[k - 1].x, r1.y - vm * z1[k - 1].y);
        }
        const double idet = 1.0 / (d00 * d11 - d01 * d10);
        g0[k] = (d11 * w1 - d01 * wm) * idet;
        g1[k] = (-d10 * w1 + d00 * wm) * idet;
        z0[k] = make_double2((d11 * r0.x - d01 * r1.x) * idet, (d11 * r0.y - d01 * r1.y) * idet);
        z1[k] = make_double2((-d10 * r0.x + d00 * r1.x) * idet, (-d10 * r0.y + d00 * r1.y) * idet);
    }
    // back substitution: X_k = Z_k - G_k X_{k+1} (only first_{k+1} enters)
    double2 fn = make_double2(0.0, 0.0);   // first_{k+1}
    double2 below = make_double2(0.0, 0.0), above = make_double2(0.0, 0.0);
    for (int k = P - 1; k >= 0; --k) {
        const double2 fk = make_double2(z0[k].x - g0[k] * fn.x, z0[k].y - g0[k] * fn.y);
        const double2 lk = make_double2(z1[k].x - g1[k] * fn.x, z1[k].y - g1[k] * fn.y);
        if (k == r + 1) above = fk;
        if (k == r - 1) below = lk;
        fn = fk;
    }
    // the rank's rows, p_hat(0) (the last unknown of the rank below, or the Neumann ghost
    // p_hat(1) - dz*H_z(0) on rank 0, 109_press_stag_array.f90:313-315) and dpdz
    const double dz = a.dz, rdz = 1.0 / dz;
    const int slot = a.isl_slot ? a.isl_slot[q] : -1;
    double2 xprev = below;
    for (int j = 1; j <= L; ++j) {
        double2 yj;
        double vj, wj;
        if (slot >= 0) {
            const long long o = slot + (long long)a.n_isl * (j - 1);
            yj = a.iy[o];
            vj = a.iv[o];
            wj = a.iw[o];
        } else {
            const long long o = q + S * (j - 1);
            const C2<T> yv = a.y[o];
            yj = make_double2((double)yv.x, (double)yv.y);
            vj = (double)a.v[o];
            wj = (double)a.w[o];
        }
        const double2 x = make_double2(yj.x - vj * below.x - wj * above.x, yj.y - vj * below.y - wj * above.y);
        if (j == 1 && r == 0) {
            const C2<T> h = a.Hz[q];
            xprev = make_double2(x.x - dz * (double)h.x, x.y - dz * (double)h.y);
        }
        if (j == 1) ph[0] = mk<T>((T)xprev.x, (T)xprev.y);
        ph[S * j] = mk<T>((T)x.x, (T)x.y);
        dph[S * j] = mk<T>((T)((x.x - xprev.x) * rdz), (T)((x.y - xprev.y) * rdz));
        xprev = x;
    }
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
    k_slab_finish<T><<<(unsigned)((a.S + 127) / 128), 128, 0, s>>>(a);
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
    template void launch_project_bc_roles<T>(T *, T *, T *, int, int, int, int, int, int, cudaStream_t,   \
                                             cudaError_t &);
OBL_INST(float)
OBL_INST(double)

} // namespace obl
