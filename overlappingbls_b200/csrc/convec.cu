// convec.cu -- the convective term of the rollout step and its transpose (see convec.cuh).
//
// All kernels are streaming: one thread per element of a (x, y, level) grid, x fastest
// so that every warp reads and writes contiguous rows; the level neighbours k-1, k+1 of
// the staggered stencils are separate coalesced rows of the same column.
#include "convec.cuh"

namespace obl {

// Every streaming kernel covers one level per grid row (blockIdx.y) and strides over the
// level's (x, y) plane, 4 elements per thread: a 128^3 level is about 17 blocks instead of
// one block per (x-tile, y), whose scheduling cost exceeded the work.
static inline dim3 sgrid(int ld, int ny, int nlev)
{
    const long long n = (long long)ld * ny;
    return dim3((unsigned)((n + 1023) / 1024), (unsigned)nlev);
}
// one block per (x-tile of 128, y) row of a single plane, for the boundary-plane kernels
static inline dim3 rgrid(int ld, int ny) { return dim3((ld + 127) / 128, ny); }
#define OBL_PLANE_LOOP(LD, NY)                                                                     \
    for (int q_ = blockIdx.x * blockDim.x + threadIdx.x, n_ = (LD) * (NY); q_ < n_;               \
         q_ += gridDim.x * blockDim.x)

template <typename T>
__global__ void k_vort(const T *__restrict__ u, const T *__restrict__ v, const T *__restrict__ dudy,
                       const T *__restrict__ dvdx, const T *__restrict__ dwdx, const T *__restrict__ dwdy,
                       T *o1, T *o2, T *o3, int nxt, int ldx, int nyt, int nz, T idz)
{
    const int z = blockIdx.y;
    OBL_PLANE_LOOP(ldx, nyt) {
    const int x = q_ % ldx, y = q_ / ldx;
    const long long pl = (long long)ldx * nyt, o = (long long)y * ldx + x, c = o + pl * z;
    T r1 = 0, r2 = 0, r3 = 0;
    if (x < nxt && z >= 1) {
        // ddz_uv (004_derivatives.f90:108) at 2..nz-1; level 1 = level 2; level nz = 0
        auto dz_of = [&](const T *f, int k) -> T {
            if (k == nz) return (T)0;
            const int kk = k == 1 ? 2 : k;
            return (f[o + pl * kk] - f[o + pl * (kk - 1)]) * idz;
        };
        const T h = (T)0.5;
        if (z <= nz - 1) r3 = dvdx[c] - dudy[c];
        if (z == 1) {
            r1 = h * (dwdy[c] + dwdy[c + pl]) - dz_of(v, 1);
            r2 = dz_of(u, 1) - h * (dwdx[c] + dwdx[c + pl]);
        } else if (z == nz) {
            r1 = h * (dwdy[c] + dwdy[c - pl]);
            r2 = -(h * (dwdx[c] + dwdx[c - pl]));
        } else {
            r1 = dwdy[c] - dz_of(v, z);
            r2 = dz_of(u, z) - dwdx[c];
        }
    }
    o1[c] = r1;
    o2[c] = r2;
    o3[c] = r3;
    }
}

template <typename T>
__global__ void k_cross(BigSet<T> b, T *X, T *Y, T *Z, int nx2, int ny2, int nz)
{
    const int z = blockIdx.y;
    OBL_PLANE_LOOP(nx2, ny2) {
    const long long P = (long long)nx2 * ny2, c = q_ + P * z;
    const T h = (T)0.5;
    T rx = 0, ry = 0, rz = 0;
    if (z == 1) {
        rx = b.V[c] * (-b.O3[c]) + h * b.W[c + P] * b.O2[c + P];     // 108_convec.f90:123-124
        ry = b.U[c] * b.O3[c] + h * b.W[c + P] * (-b.O1[c + P]);     // :153-154
    } else if (z >= 2 && z <= nz - 1) {
        rx = b.V[c] * (-b.O3[c]) + h * (b.W[c + P] * b.O2[c + P] + b.W[c] * b.O2[c]);           // :145-149
        ry = b.U[c] * b.O3[c] + h * (b.W[c + P] * (-b.O1[c + P]) + b.W[c] * (-b.O1[c]));        // :175-179
        rz = h * ((b.U[c] + b.U[c - P]) * (-b.O2[c]) + (b.V[c] + b.V[c - P]) * b.O1[c]);        // :194-199
    }
    X[c] = rx;
    Y[c] = ry;
    Z[c] = rz;
    }
}

template <typename T>
__global__ void k_update(T *u, T *v, T *w, const T *cx, const T *cy, const T *cz, T f, int nxt, int ldx, int nyt)
{
    const int z = blockIdx.y + 1;
    OBL_PLANE_LOOP(ldx, nyt) {
    const int x = q_ % ldx;
    if (x >= nxt) continue;
    const long long c = q_ + (long long)ldx * nyt * z;
    u[c] -= f * cx[c];
    v[c] -= f * cy[c];
    w[c] -= f * cz[c];
    }
}

template <typename T>
__global__ void k_adj_project_bc(T *lu, T *lv, T *lw, int ldx, int nyt, int nz, int stress_free)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= ldx) return;
    const long long pl = (long long)ldx * nyt, o = (long long)y * ldx + x;
    if (stress_free) {
        lu[o + pl * (nz - 2)] += lu[o + pl * (nz - 1)];
        lu[o + pl * (nz - 1)] = (T)0;
        lv[o + pl * (nz - 2)] += lv[o + pl * (nz - 1)];
        lv[o + pl * (nz - 1)] = (T)0;
    }
    lw[o + pl] = (T)0;
    lw[o + pl * nz] = (T)0;
}

template <typename T>
__global__ void k_adj_w1(T *lw, const T *p, T c, int nxt, int ldx, int nyt)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= ldx) return;
    const long long pl = (long long)ldx * nyt, o = (long long)y * ldx + x + pl;
    lw[o] = x < nxt ? c * p[o] : (T)0;
}

template <typename T>
__global__ void k_cross_adj(BigSet<T> b, const T *__restrict__ LX, const T *__restrict__ LY,
                            const T *__restrict__ LZ, T f, CrossAdjOut<T> out, int nx2, int ny2, int nz)
{
    const int z = blockIdx.y;
    OBL_PLANE_LOOP(nx2, ny2) {
    const long long P = (long long)nx2 * ny2, o = q_, c = o + P * z;
    // adjoints of X, Y at levels 1..nz-1 and of Z at 2..nz-1 (cross_z_big(1) is a constant)
    auto lx = [&](int k) -> T { return (k >= 1 && k <= nz - 1) ? f * LX[o + P * k] : (T)0; };
    auto ly = [&](int k) -> T { return (k >= 1 && k <= nz - 1) ? f * LY[o + P * k] : (T)0; };
    auto lz = [&](int k) -> T { return (k >= 2 && k <= nz - 1) ? f * LZ[o + P * k] : (T)0; };
    const T h = (T)0.5;
    T aU = 0, aV = 0, aW = 0, a1 = 0, a2 = 0, a3 = 0;
    if (z >= 1 && z <= nz - 1) {
        const T lxk = lx(z), lyk = ly(z), lzk = lz(z), lzk1 = lz(z + 1);
        a3 = -b.V[c] * lxk + b.U[c] * lyk;
        aU = b.O3[c] * lyk - h * b.O2[c] * lzk - h * b.O2[c + P] * lzk1;
        aV = -b.O3[c] * lxk + h * b.O1[c] * lzk + h * b.O1[c + P] * lzk1;
    }
    if (z >= 2 && z <= nz) {
        const T sX = lx(z - 1) + lx(z), sY = ly(z - 1) + ly(z), l = lz(z);
        aW = h * b.O2[c] * sX - h * b.O1[c] * sY;
        a2 = h * b.W[c] * sX - h * (b.U[c] + b.U[c - P]) * l;
        a1 = -h * b.W[c] * sY + h * (b.V[c] + b.V[c - P]) * l;
    }
    out.U[c] = aU;
    out.V[c] = aV;
    out.W[c] = aW;
    out.O1[c] = a1;
    out.O2[c] = a2;
    out.O3[c] = a3;
    }
}

template <typename T>
__global__ void k_adj_q(const T *s1, const T *s2, T *q1, T *q2, int nxt, int ldx, int nyt, int nz)
{
    const int z = blockIdx.y;
    OBL_PLANE_LOOP(ldx, nyt) {
    const int x = q_ % ldx;
    const long long pl = (long long)ldx * nyt, o = q_, c = o + pl * z;
    T r1 = 0, r2 = 0;
    if (x < nxt) {
        if (z >= 2 && z <= nz - 1) {
            r1 = s1[c];
            r2 = s2[c];
        }
        if (z == nz - 1 || z == nz) {   // vort1(nz), vort2(nz) average dwdy, dwdx of nz-1 and nz
            r1 += (T)0.5 * s1[o + pl * nz];
            r2 += (T)0.5 * s2[o + pl * nz];
        }
    }
    q1[c] = r1;
    q2[c] = r2;
    }
}

template <typename T>
__global__ void k_adj_combine(AdjCombineArgs<T> a, int nxt, int ldx, int nyt, int nz, T idz)
{
    const int z = blockIdx.y;
    OBL_PLANE_LOOP(ldx, nyt) {
    const int x = q_ % ldx;
    if (x >= nxt) continue;
    const long long pl = (long long)ldx * nyt, c = q_ + pl * z;
    // transposed level difference of dudz(k) = (u(k) - u(k-1))/dz, k = 2..nz-1
    auto dzt = [&](const T *s) -> T {
        const T here = (z >= 2 && z <= nz - 1) ? s[c] : (T)0;
        const T above = (z + 1 >= 2 && z + 1 <= nz - 1) ? s[c + pl] : (T)0;
        return (here - above) * idz;
    };
    a.lu[c] += a.sU[c] + a.t1[c] + dzt(a.s2);
    a.lv[c] += a.sV[c] - a.t2[c] - dzt(a.s1);
    a.lw[c] += a.sW[c] + a.t3[c] - a.t4[c];
    }
}

constexpr int kKeThreads = 256;
constexpr int kKeParts = 148 * 4;
int ke_parts() { return kKeParts; }

template <typename T>
__global__ void __launch_bounds__(kKeThreads)
k_ke_band(const T *u, const T *v, const T *w, T *lu, T *lv, T *lw, double *part, int nxt, int ldx, int nyt,
          int nz, int klo, int khi)
{
    const long long pl = (long long)ldx * nyt, n = pl * (nz + 1);
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long z = i / pl;
        const int x = (int)((i - z * pl) % ldx);
        const bool in = x < nxt && z >= klo && z <= khi;             // klo >= 1, khi <= nz-1
        const bool inm = x < nxt && z - 1 >= klo && z - 1 <= khi;
        const double uu = (double)u[i], vv = (double)v[i];
        const double tw = in ? 0.5 * ((double)w[i] + (double)w[i + pl]) : 0.0;
        if (in) acc += 0.5 * (uu * uu + vv * vv + tw * tw);
        if (lu) {
            const double twm = inm ? 0.5 * ((double)w[i - pl] + (double)w[i]) : 0.0;
            lu[i] = in ? (T)uu : (T)0;
            lv[i] = in ? (T)vv : (T)0;
            lw[i] = (T)(0.5 * tw + 0.5 * twm);
        }
    }
    __shared__ double red[kKeThreads / 32];
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < kKeThreads / 32; ++k) s += red[k];
        part[blockIdx.x] = s;
    }
}

__global__ void k_sum_parts(const double *part, int n, double *out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += part[i];
        *out = s;
    }
}

template <typename T>
void launch_vort(const T *u, const T *v, const T *dudy, const T *dvdx, const T *dwdx, const T *dwdy, T *o1,
                 T *o2, T *o3, int nxt, int ldx, int nyt, int nz, double dz, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_vort<T><<<sgrid(ldx, nyt, nz + 1), 256, 0, s>>>(u, v, dudy, dvdx, dwdx, dwdy, o1, o2, o3, nxt, ldx, nyt,
                                                       nz, (T)(1.0 / dz));
    e = cudaGetLastError();
}
template <typename T>
void launch_cross(const BigSet<T> &b, T *X, T *Y, T *Z, int nx2, int ny2, int nz, cudaStream_t s,
                  cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_cross<T><<<sgrid(nx2, ny2, nz + 1), 256, 0, s>>>(b, X, Y, Z, nx2, ny2, nz);
    e = cudaGetLastError();
}
template <typename T>
void launch_update(T *u, T *v, T *w, const T *cx, const T *cy, const T *cz, double f, int nxt, int ldx,
                   int nyt, int nz, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_update<T><<<sgrid(ldx, nyt, nz - 1), 256, 0, s>>>(u, v, w, cx, cy, cz, (T)f, nxt, ldx, nyt);
    e = cudaGetLastError();
}
template <typename T>
void launch_adj_project_bc(T *lu, T *lv, T *lw, int ldx, int nyt, int nz, int stress_free, cudaStream_t s,
                           cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_adj_project_bc<T><<<rgrid(ldx, nyt), 128, 0, s>>>(lu, lv, lw, ldx, nyt, nz, stress_free);
    e = cudaGetLastError();
}
template <typename T>
void launch_adj_w1(T *lw, const T *p, double c, int nxt, int ldx, int nyt, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_adj_w1<T><<<rgrid(ldx, nyt), 128, 0, s>>>(lw, p, (T)c, nxt, ldx, nyt);
    e = cudaGetLastError();
}
template <typename T>
void launch_cross_adj(const BigSet<T> &b, const T *LX, const T *LY, const T *LZ, double f,
                      const CrossAdjOut<T> &out, int nx2, int ny2, int nz, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_cross_adj<T><<<sgrid(nx2, ny2, nz + 1), 256, 0, s>>>(b, LX, LY, LZ, (T)f, out, nx2, ny2, nz);
    e = cudaGetLastError();
}
template <typename T>
void launch_adj_q(const T *s1, const T *s2, T *q1, T *q2, int nxt, int ldx, int nyt, int nz, cudaStream_t s,
                  cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_adj_q<T><<<sgrid(ldx, nyt, nz + 1), 256, 0, s>>>(s1, s2, q1, q2, nxt, ldx, nyt, nz);
    e = cudaGetLastError();
}
template <typename T>
void launch_adj_combine(const AdjCombineArgs<T> &a, int nxt, int ldx, int nyt, int nz, double dz,
                        cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_adj_combine<T><<<sgrid(ldx, nyt, nz + 1), 256, 0, s>>>(a, nxt, ldx, nyt, nz, (T)(1.0 / dz));
    e = cudaGetLastError();
}
template <typename T>
void launch_ke_band(const T *u, const T *v, const T *w, T *lu, T *lv, T *lw, double *part, double *out,
                    int nxt, int ldx, int nyt, int nz, int klo, int khi, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess) return;
    k_ke_band<T><<<kKeParts, kKeThreads, 0, s>>>(u, v, w, lu, lv, lw, part, nxt, ldx, nyt, nz, klo, khi);
    e = cudaGetLastError();
    if (e != cudaSuccess) return;
    k_sum_parts<<<1, 32, 0, s>>>(part, kKeParts, out);
    e = cudaGetLastError();
}

#define OBL_INST(T)                                                                                      \
    template void launch_vort<T>(const T *, const T *, const T *, const T *, const T *, const T *, T *, T *,   \
                                 T *, int, int, int, int, double, cudaStream_t, cudaError_t &);          \
    template void launch_cross<T>(const BigSet<T> &, T *, T *, T *, int, int, int, cudaStream_t,          \
                                  cudaError_t &);                                                        \
    template void launch_update<T>(T *, T *, T *, const T *, const T *, const T *, double, int, int, int,  \
                                   int, cudaStream_t, cudaError_t &);                                    \
    template void launch_adj_project_bc<T>(T *, T *, T *, int, int, int, int, cudaStream_t, cudaError_t &); \
    template void launch_adj_w1<T>(T *, const T *, double, int, int, int, cudaStream_t, cudaError_t &);   \
    template void launch_cross_adj<T>(const BigSet<T> &, const T *, const T *, const T *, double,         \
                                      const CrossAdjOut<T> &, int, int, int, cudaStream_t, cudaError_t &); \
    template void launch_adj_q<T>(const T *, const T *, T *, T *, int, int, int, int, cudaStream_t,       \
                                  cudaError_t &);                                                        \
    template void launch_adj_combine<T>(const AdjCombineArgs<T> &, int, int, int, int, double,           \
                                        cudaStream_t, cudaError_t &);                                    \
    template void launch_ke_band<T>(const T *, const T *, const T *, T *, T *, T *, double *, double *,    \
                                    int, int, int, int, int, int, cudaStream_t, cudaError_t &);
OBL_INST(float)
OBL_INST(double)

} // namespace obl
