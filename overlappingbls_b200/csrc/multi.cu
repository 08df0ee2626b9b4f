// multi.cu -- the row and column line kernels over several fields of one shape in one
// launch (see launch_rows_multi / launch_cols_multi in lines.cuh).  The per-line work is
// row_unit / cols2_unit unchanged; only the field of each unit is looked up first.
#include "lines_dispatch.cuh"

namespace obl {

template <typename T, int N, int OP>
__global__ void __launch_bounds__(256) k_rows_multi(RowArgs<T> a0, MultiPtr<T> m, int nf, long long npf)
{
    using C = C2<T>;
    using D = LineDerived<N, OP>;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *twF = reinterpret_cast<C *>(smraw);
    C *twB = twF + D::TF;
    C *scr = twB + D::TB;
    load_tables<T, N, OP>(a0.twF, a0.twB, twF, twB);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // npf: each field's pairs rounded up to whole warps' groups, so a group never spans fields
    for (long long base = ((long long)blockIdx.x * nw + warp) * D::LPW; base < npf * nf;
         base += (long long)gridDim.x * nw * D::LPW) {
        const int f = (int)(base / npf);
        RowArgs<T> a = a0;
        a.src = m.src[f];
        a.dst = m.dst[f];
        row_unit<T, N, OP>(a, base - f * npf, twF, twB, scr + warp * D::LPW * scratch_len(D::NM), lane);
    }
}

template <typename T, int N, int OP, bool REAL, int NW, int WB, bool TWG>
__global__ void __launch_bounds__(32 * NW, col_min_blocks(NW, TWG, col_warps_sm<OP>())) k_cols2_multi(ColArgs<T> a0, MultiPtr<T> m)
{
    using C = C2<T>;
    using D = LineDerived<N, OP>;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int f = blockIdx.y / a0.nlev, z = blockIdx.y - f * a0.nlev;
    ColArgs<T> a = a0;
    a.src = m.src[f];
    a.dst = m.dst[f];
    if constexpr (TWG) {
        cols2_unit<T, N, OP, REAL, NW, WB>(a, blockIdx.x, z, a.twF, a.twB, reinterpret_cast<C *>(smraw));
    } else {
        C *twF = reinterpret_cast<C *>(smraw);
        C *twB = twF + D::TF;
        C *buf = twB + D::TB;
        load_tables<T, N, OP>(a.twF, a.twB, twF, twB);
        __syncthreads();
        cols2_unit<T, N, OP, REAL, NW, WB>(a, blockIdx.x, z, twF, twB, buf);
    }
}

template <typename T, int N, int OP>
static cudaError_t rows_multi_t(const RowArgs<T> &a, const MultiPtr<T> &m, int nf, cudaStream_t s)
{
    static int caps[kMaxDevices] = {};
    const size_t sm = rows_smem<T, N, OP>();
    auto kern = k_rows_multi<T, N, OP>;
    const int ds = device_slot();
    int cap = ds >= 0 ? caps[ds] : 0;
    if (!cap) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        int dev = 0, nsm = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, sm);
        cap = nsm * (per > 0 ? per : 1);
        if (ds >= 0) caps[ds] = cap;
    }
    constexpr int LPW = LineDerived<N, OP>::LPW;
    const long long npf = (a.npairs + LPW - 1) / LPW * LPW;
    const long long want = (npf * nf + 8LL * LPW - 1) / (8LL * LPW);
    const int grid = (int)(want < cap ? want : cap);
    if (grid < 1) return cudaSuccess;
    kern<<<grid, 256, sm, s>>>(a, m, nf, npf);
    return cudaGetLastError();
}

template <typename T, int N, int OP, bool REAL>
static cudaError_t cols_multi_t(const ColArgs<T> &a, const MultiPtr<T> &m, int nf, cudaStream_t s)
{
    static bool inits[kMaxDevices] = {};
    constexpr int NW = col_warps<T, N, OP>(), WB = col_lines<T, N, OP>();
    constexpr bool TWG = col_tw_global<T, N, OP>();
    using D = LineDerived<N, OP>;
    const size_t sm = TWG ? sizeof(C2<T>) * (size_t)D::NM * WB : cols2_smem<T, N, OP, WB>();
    auto kern = k_cols2_multi<T, N, OP, REAL, NW, WB, TWG>;
    const int ds = device_slot();
    if (ds < 0 || !inits[ds]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        if (ds >= 0) inits[ds] = true;
    }
    ColArgs<T> b = a;
    b.pf_ahead = 0;
    const int nlines = REAL ? b.ncols / 2 : b.ncols;
    dim3 grid((nlines + WB - 1) / WB, (unsigned)(b.nlev * nf));
    if (grid.x < 1 || grid.y < 1) return cudaSuccess;
    kern<<<grid, 32 * NW, sm, s>>>(b, m);
    return cudaGetLastError();
}

template <typename T, int N>
static cudaError_t rows_multi_n(int op, const RowArgs<T> &a, const MultiPtr<T> &m, int nf, cudaStream_t s)
{
    switch (op) {
    case OP_DERIV: return rows_multi_t<T, N, OP_DERIV>(a, m, nf, s);
    case OP_PAD: return rows_multi_t<T, N, OP_PAD>(a, m, nf, s);
    case OP_UNPAD: return rows_multi_t<T, N, OP_UNPAD>(a, m, nf, s);
    case OP_FWD: return rows_multi_t<T, N, OP_FWD>(a, m, nf, s);
    }
    return cudaErrorInvalidValue;
}

template <typename T, int N>
static cudaError_t cols_multi_n(int op, const ColArgs<T> &a, const MultiPtr<T> &m, int nf, cudaStream_t s)
{
    switch (op) {
    case OP_DERIV: return cols_multi_t<T, N, OP_DERIV, true>(a, m, nf, s);
    case OP_PAD: return cols_multi_t<T, N, OP_PAD, true>(a, m, nf, s);
    case OP_UNPAD: return cols_multi_t<T, N, OP_UNPAD, true>(a, m, nf, s);
    case OP_FWD: return cols_multi_t<T, N, OP_FWD, false>(a, m, nf, s);   // complex columns
    }
    return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_rows_multi(int op, int n, const RowArgs<T> &a, const MultiPtr<T> &m, int nf, cudaStream_t s)
{
    if (nf < 1 || nf > kMultiFields) return cudaErrorInvalidValue;
    switch (n) {
#define OBL_CASE(N) case N: return rows_multi_n<T, N>(op, a, m, nf, s);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_cols_multi(int op, int n, const ColArgs<T> &a, const MultiPtr<T> &m, int nf, cudaStream_t s)
{
    if (nf < 1 || nf > kMultiFields) return cudaErrorInvalidValue;
    switch (n) {
#define OBL_CASE(N) case N: return cols_multi_n<T, N>(op, a, m, nf, s);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return cudaErrorInvalidValue;
}

template cudaError_t launch_rows_multi<float>(int, int, const RowArgs<float> &, const MultiPtr<float> &, int,
                                              cudaStream_t);
template cudaError_t launch_rows_multi<double>(int, int, const RowArgs<double> &, const MultiPtr<double> &, int,
                                               cudaStream_t);
template cudaError_t launch_cols_multi<float>(int, int, const ColArgs<float> &, const MultiPtr<float> &, int,
                                              cudaStream_t);
template cudaError_t launch_cols_multi<double>(int, int, const ColArgs<double> &, const MultiPtr<double> &, int,
                                               cudaStream_t);

} // namespace obl
