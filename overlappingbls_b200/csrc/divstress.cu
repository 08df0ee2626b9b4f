// divstress.cu -- the ddy column pass of divstress_uv / divstress_w with the sum fused into
// its stores (see divstress.cuh), for every supported line length.
#include "divstress.cuh"
#include "lines_dispatch.cuh"

namespace obl {

// k_cols2 for OP_DERIV on real columns, with the DivEpi store hook
template <typename T, int N, int NW, int WB, bool TWG>
__global__ void __launch_bounds__(32 * NW, col_min_blocks(NW, TWG, col_warps_sm<OP_DERIV>())) k_cols_divt(ColArgs<T> a, DivEpi<T> e)
{
    using C = C2<T>;
    using D = LineDerived<N, OP_DERIV>;
    extern __shared__ __align__(16) unsigned char smraw[];
    if constexpr (TWG) {
        cols2_unit<T, N, OP_DERIV, true, NW, WB, DivEpi<T>>(a, blockIdx.x, blockIdx.y, a.twF, a.twB,
                                                              reinterpret_cast<C *>(smraw), e);
    } else {
        C *twF = reinterpret_cast<C *>(smraw);
        C *twB = twF + D::TF;
        C *buf = twB + D::TB;
        load_tables<T, N, OP_DERIV>(a.twF, a.twB, twF, twB);
        __syncthreads();
        cols2_unit<T, N, OP_DERIV, true, NW, WB, DivEpi<T>>(a, blockIdx.x, blockIdx.y, twF, twB, buf, e);
    }
}

// the same CTA shape, shared memory and grid as the plain ddy pass
template <typename T, int N>
static cudaError_t launch_divt_n(const ColArgs<T> &a, const DivEpi<T> &e, cudaStream_t s)
{
    static bool inits[kMaxDevices] = {};
    constexpr int NW = col_warps<T, N, OP_DERIV>(), WB = col_lines<T, N, OP_DERIV>();
    constexpr bool TWG = col_tw_global<T, N, OP_DERIV>();
    using D = LineDerived<N, OP_DERIV>;
    const size_t sm = TWG ? sizeof(C2<T>) * (size_t)D::NM * WB : cols2_smem<T, N, OP_DERIV, WB>();
    auto kern = k_cols_divt<T, N, NW, WB, TWG>;
    const int ds = device_slot();
    if (ds < 0 || !inits[ds]) {
        cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (err != cudaSuccess) return err;
        if (ds >= 0) inits[ds] = true;
    }
    const int nlines = a.ncols / 2;
    dim3 grid((nlines + WB - 1) / WB, a.nlev);
    if (grid.x < 1 || grid.y < 1) return cudaSuccess;
    kern<<<grid, 32 * NW, sm, s>>>(a, e);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_cols_divt(int n, const ColArgs<T> &a, const DivEpi<T> &e, cudaStream_t s)
{
    switch (n) {
#define OBL_CASE(N) case N: return launch_divt_n<T, N>(a, e, s);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return cudaErrorInvalidValue;
}

template <typename T> __global__ void k_fill(T *p, long long n, T v)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

template <typename T> void launch_fill(T *p, long long n, T v, cudaStream_t s, cudaError_t &e)
{
    if (e != cudaSuccess || n <= 0) return;
    const long long want = (n + 255) / 256;
    k_fill<T><<<(unsigned)(want < 148 * 8 ? want : 148 * 8), 256, 0, s>>>(p, n, v);
    e = cudaGetLastError();
}

template cudaError_t launch_cols_divt<float>(int, const ColArgs<float> &, const DivEpi<float> &, cudaStream_t);
template cudaError_t launch_cols_divt<double>(int, const ColArgs<double> &, const DivEpi<double> &, cudaStream_t);
template void launch_fill<float>(float *, long long, float, cudaStream_t, cudaError_t &);
template void launch_fill<double>(double *, long long, double, cudaStream_t, cudaError_t &);

} // namespace obl
