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
