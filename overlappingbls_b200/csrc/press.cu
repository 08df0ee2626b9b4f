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

template <typename TS, typename TC, bool ISLAND>
__global__ void __launch_bounds__(128) k_tdma(TdmaArgs<TS> a, IslandArgs isl)
{
    tdma_column<TS, TC, ISLAND>(a, isl, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Mixed precision in one launch: the first nbi blocks solve the FP64 island columns (their
// long sequential FP64 sweeps start first), the remaining blocks the FP32 bulk columns,
// so the two overlap instead of running back to back.  The sweeps are latency-bound: 8
// blocks per SM (64 registers, a few FP64 spills) measured faster than 5 without spills
// (OBL_TDMA_MINB is the build-time knob).
#ifndef OBL_TDMA_MINB
#define OBL_TDMA_MINB 8
#endif
template <typename T>
__global__ void __launch_bounds__(128, OBL_TDMA_MINB) k_tdma_mixed(TdmaArgs<T> a, IslandArgs isl, int nbi)
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
