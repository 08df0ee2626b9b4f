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
#include "common.cuh"
#include "press.cuh"

namespace obl {

static constexpr double kTadv1 = 1.5;                 // 001_param.f90:152
static constexpr double kBogus = -1234567890.0;       // 001_param.f90:40

// One column's solve; t = the thread's index among the bulk columns or in the island list.
template <typename TS, typename TC, bool ISLAND>
__device__ __forceinline__ void tdma_column(const TdmaArgs<TS> &a, const IslandArgs &isl, long long t)
{
    using CS = C2<TS>;
    using CC = C2<TC>;
    long long q;
    if constexpr (ISLAND) {
        if (t >= isl.n) return;
        q = isl.cols[t];
    } else {
        if (t >= a.S) return;
        q = t;
        if (a.skip && a.skip[q]) return;
    }
    const long long S = a.S;
    const int L = a.L;
    const int ix = (int)(q % a.lhx), iy = (int)(q / a.lhx);
    CS *ph = a.phat + q;

    // Nyquist columns: p_hat = 0 at every level (:303-305, and the caller's zero fill)
    if (ix == a.lhx - 1 || iy == a.nyt / 2) {
        for (int z = 0; z <= L; ++z) ph[S * z] = mk<TS>(0, 0);
        if (a.dph)
            for (int z = 1; z <= L; ++z) a.dph[q + S * z] = mk<TS>(0, 0);
        return;
    }
    const double kxd = a.kx[ix], kyd = a.ky[iy];
    const double k2d = kxd * kxd + kyd * kyd;   // 002_fft.f90:167
    const bool m00 = (k2d == 0.0);              // the (0,0) mean mode
    const TC kx = (TC)kxd, ky = (TC)kyd, k2 = (TC)k2d;
    const TC dz = (TC)a.dz, idz = (TC)(1.0 / a.dz), idz2 = (TC)(1.0 / (a.dz * a.dz));

    auto ld = [&](const CS *p, int z) -> CC {
        const CS v = p[q + S * z];
        return mk<TC>((TC)v.x, (TC)v.y);
    };
    auto st_d = [&](int z, CC v) {
        if constexpr (ISLAND) isl.dscr[t + (long long)isl.n * z] = make_double2(v.x, v.y);
        else ph[S * z] = v;
    };
    auto ld_d = [&](int z) -> CC {
        if constexpr (ISLAND) { const double2 v = isl.dscr[t + (long long)isl.n * z]; return mk<TC>(v.x, v.y); }
        else return ph[S * z];
    };
    auto st_c = [&](int z, TC v) {
        if constexpr (ISLAND) isl.cscr[t + (long long)isl.n * (z - 1)] = v;
        else a.cscr[q + S * (z - 1)] = v;
    };
    auto ld_c = [&](int z) -> TC {
        if constexpr (ISLAND) return isl.cscr[t + (long long)isl.n * (z - 1)];
        else return a.cscr[q + S * (z - 1)];
    };

    // ---- forward elimination ----
    // The RHS inputs of level iz+1 are loaded while level iz is eliminated (the loads are
    // independent of the recurrence; issuing them ahead hides their latency).
    const CC hz0 = ld(a.Hz, 0);     // RHS_col(0) = H_z(0) (:209)
    CC hzc = ld(a.Hz, 1);
    CC hzn = ld(a.Hz, 2);
    CC hx = ld(a.Hx, 1), hy = ld(a.Hy, 1);
    CC dprev = hz0;
    TC cprev = 0;                   // coef_cp(0) = 0 on the bottom rank
    for (int iz = 1; iz <= L; ++iz) {
        const int izn = iz < L ? iz + 1 : iz;
        const CC hx_n = ld(a.Hx, izn), hy_n = ld(a.Hy, izn), hz_n = ld(a.Hz, izn + 1);
        TC am, bm, cm;
        CC r;
        if (!m00) {
            const bool top = a.neumann_top && iz == L;
            am = (iz == 1) ? (TC)0 : idz2;
            bm = (iz == 1 || top) ? -(k2 + idz2) : -(k2 + (TC)2 * idz2);
            cm = top ? (TC)0 : idz2;
            const CC sxy = mk<TC>(kx * hx.x + ky * hy.x, kx * hx.y + ky * hy.y);
            CC dh = csub(hzn, hzc);
            if (iz == 1) dh = cadd(dh, hz0);
            r = mk<TC>(-sxy.y + dh.x / dz, sxy.x + dh.y / dz);
        } else {
            am = (iz == 1) ? (TC)0 : -idz;
            bm = idz;
            cm = 0;
            r = (iz == 1) ? mk<TC>(0, 0) : hzc;
        }
        const TC bp = bm - am * cprev;
        const TC ibp = (TC)1 / bp;
        const TC cp = cm * ibp;
        const CC d = mk<TC>((r.x - am * dprev.x) * ibp, (r.y - am * dprev.y) * ibp);
        st_c(iz, cp);
        st_d(iz, d);
        cprev = cp;
        dprev = d;
        hzc = hzn;
        hzn = hz_n;
        hx = hx_n;
        hy = hy_n;
    }
    // ---- back substitution ----
    CC pn = a.neumann_top ? dprev : mk<TC>(0, 0);   // p_hat(nz-1): solved row / forced 0
    ph[S * L] = mk<TS>((TS)pn.x, (TS)pn.y);
    C2<TS> *dph = a.dph ? a.dph + q : nullptr;
    const TC rdz = (TC)(1.0 / a.dz);
    CC dn = L > 1 ? ld_d(L - 1) : mk<TC>(0, 0);
    TC cn = L > 1 ? ld_c(L - 1) : (TC)0;
    for (int iz = L - 1; iz >= 1; --iz) {
        const CC d = dn;
        const TC cp = cn;
        if (iz > 1) {   // next level's operands ahead of this level's stores
            dn = ld_d(iz - 1);
            cn = ld_c(iz - 1);
        }
        const CC p = mk<TC>(d.x - cp * pn.x, d.y - cp * pn.y);
        if (dph) dph[S * (iz + 1)] = mk<TS>((TS)((pn.x - p.x) * rdz), (TS)((pn.y - p.y) * rdz));
        ph[S * iz] = mk<TS>((TS)p.x, (TS)p.y);
        pn = p;
    }
    // Neumann ghost level below the wall (:313-315)
    const CC p0 = mk<TC>(pn.x - dz * hz0.x, pn.y - dz * hz0.y);
    ph[0] = mk<TS>((TS)p0.x, (TS)p0.y);
    if (dph) dph[S] = mk<TS>((TS)((pn.x - p0.x) / dz), (TS)((pn.y - p0.y) / dz));
}

template <typename TS, typename TC, bool ISLAND>
__global__ void __launch_bounds__(128) k_tdma(TdmaArgs<TS> a, IslandArgs isl)
{
    tdma_column<TS, TC, ISLAND>(a, isl, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Mixed precision in one launch: the first nbi blocks solve the FP64 island columns (their
// long sequential FP64 sweeps start first), the remaining blocks the FP32 bulk columns,
// so the two overlap instead of running back to back.
template <typename T>
__global__ void __launch_bounds__(128) k_tdma_mixed(TdmaArgs<T> a, IslandArgs isl, int nbi)
{
    if ((int)blockIdx.x < nbi)
        tdma_column<T, double, true>(a, isl, (long long)blockIdx.x * blockDim.x + threadIdx.x);
    else
        tdma_column<T, T, false>(a, isl, (long long)(blockIdx.x - nbi) * blockDim.x + threadIdx.x);
}

template <typename T> void launch_tdma(const TdmaArgs<T> &a, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    IslandArgs none{nullptr, 0, nullptr, nullptr};
    const int bs = 128;
    k_tdma<T, T, false><<<(unsigned)((a.S + bs - 1) / bs), bs, 0, s>>>(a, none);
    e = cudaGetLastError();
}

template <typename T>
void launch_tdma_island(const TdmaArgs<T> &a, const IslandArgs &isl, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    const int bs = 128;
    const int nbi = (int)((isl.n + bs - 1) / bs), nbb = (int)((a.S + bs - 1) / bs);
    k_tdma_mixed<T><<<(unsigned)(nbi + nbb), bs, 0, s>>>(a, isl, nbi);
    e = cudaGetLastError();
}

// ----------------------------------------------------------------------------- streaming
// Grid convention: blockIdx.x covers x, blockIdx.y the row y, blockIdx.z the level.
static inline dim3 fgrid(int ldx, int nyt, int nlev) { return dim3((ldx + 127) / 128, nyt, nlev); }

template <typename T>
__global__ void k_ddz_uv(T *dfdz, const T *fun, int nxt, int ldx, int nyt, int nz, T cst)
{
    // 004_derivatives.f90:98-113, single rank (coordz == 0 == npz-1)
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    const long long pl = (long long)ldx * nyt, o = (long long)y * ldx + x;
    if (z == 0) {
        if (x < ldx) dfdz[o] = (T)kBogus;
    } else if (z >= 2 && z <= nz - 1 && x < nxt) {
        dfdz[o + pl * z] = cst * (fun[o + pl * z] - fun[o + pl * (z - 1)]);
    }
}

template <typename T>
__global__ void k_ddz_w(T *dfdz, const T *fun, int nxt, int ldx, int nyt, int nz, T cst)
{
    // 004_derivatives.f90:168-180, single rank
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    const long long pl = (long long)ldx * nyt, o = (long long)y * ldx + x;
    if (z == 0) {
        if (x < ldx) dfdz[o] = (T)kBogus;
    } else if (z == nz) {
        if (x < ldx) dfdz[o + pl * z] = (T)0;
    } else if (x < nxt) {
        dfdz[o + pl * z] = cst * (fun[o + pl * (z + 1)] - fun[o + pl * z]);
    }
}

template <typename T>
__global__ void k_dpdz(T *dpdz, const T *p, int nxt, int ldx, int nyt, T dz)
{
    // 103_flosol.f90:174-175: dpdz(jz) = (p(jz) - p(jz-1))/dz, jz = 1..nz-1
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z + 1;
    if (x >= nxt) return;
    const long long pl = (long long)ldx * nyt, o = (long long)y * ldx + x;
    dpdz[o + pl * (z - 1)] = (p[o + pl * z] - p[o + pl * (z - 1)]) / dz;
}

template <typename T>
__global__ void k_project(T *u, T *v, T *w, const T *dpdx, const T *dpdy, const T *dpdz,
                          int nxt, int ldx, int nyt, T dt)
{
    // 110_project.f90:16-40 (jz_min = 2 on the bottom rank)
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z + 1;
    if (x >= nxt) return;
    const long long pl = (long long)ldx * nyt, o = (long long)y * ldx + x;
    const T t1 = (T)kTadv1;
    T rhs = -t1 * dpdx[o + pl * (z - 1)];
    u[o + pl * z] = u[o + pl * z] + dt * rhs;
    rhs = -t1 * dpdy[o + pl * (z - 1)];
    v[o + pl * z] = v[o + pl * z] + dt * rhs;
    if (z >= 2) {
        rhs = -t1 * dpdz[o + pl * (z - 1)];
        w[o + pl * z] = w[o + pl * z] + dt * rhs;
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
    k_ddz_uv<T><<<fgrid(ldx, nyt, nz + 1), 128, 0, s>>>(dfdz, fun, nxt, ldx, nyt, nz, (T)(1.0 / dz));
    e = cudaGetLastError();
}
template <typename T>
void launch_ddz_w(T *dfdz, const T *fun, int nxt, int ldx, int nyt, int nz, double dz,
                  cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_ddz_w<T><<<fgrid(ldx, nyt, nz + 1), 128, 0, s>>>(dfdz, fun, nxt, ldx, nyt, nz, (T)(1.0 / dz));
    e = cudaGetLastError();
}
template <typename T>
void launch_dpdz(T *dpdz, const T *p, int nxt, int ldx, int nyt, int nz, double dz,
                 cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_dpdz<T><<<fgrid(ldx, nyt, nz - 1), 128, 0, s>>>(dpdz, p, nxt, ldx, nyt, (T)dz);
    e = cudaGetLastError();
}
template <typename T>
void launch_project(T *u, T *v, T *w, const T *dpdx, const T *dpdy, const T *dpdz, int nxt,
                    int ldx, int nyt, int nz, double dt, int stress_free, cudaStream_t s,
                    cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_project<T><<<fgrid(ldx, nyt, nz - 1), 128, 0, s>>>(u, v, w, dpdx, dpdy, dpdz, nxt, ldx, nyt, (T)dt);
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
