// fused.cu -- launchers and instantiations of the cluster-fused plane kernels.
#include "fused.cuh"
#include "lines_dispatch.cuh"

namespace obl {

template <typename T, int N> static cudaLaunchConfig_t fwd_cfg(int ncl, int csize, cudaStream_t s,
                                                               cudaLaunchAttribute *attr)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(ncl * csize));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = FwdFusedGeo<T, N>::smem;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

template <typename T, int N> static cudaError_t fwd_prepare(int csize)
{
    static bool inits[kMaxDevices] = {}, bigs[kMaxDevices] = {};
    auto kern = k_fwd_fused<T, N>;
    const int ds = device_slot();
    if (ds < 0 || !inits[ds]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)FwdFusedGeo<T, N>::smem);
        if (e != cudaSuccess) return e;
        if (ds >= 0) inits[ds] = true;
    }
    if (csize > 8 && (ds < 0 || !bigs[ds])) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
        if (ds >= 0) bigs[ds] = true;
    }
    return cudaSuccess;
}

template <typename T, int N>
static cudaError_t fwd_run_n(const FwdFusedArgs<T> &a, int ncl, int csize, cudaStream_t s)
{
    cudaError_t e = fwd_prepare<T, N>(csize);
    if (e != cudaSuccess) return e;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = fwd_cfg<T, N>(ncl, csize, s, attr);
    e = cudaLaunchKernelEx(&cfg, k_fwd_fused<T, N>, a);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

template <typename T, int N> static int fwd_max_clusters_n(int csize)
{
    if (fwd_prepare<T, N>(csize) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = fwd_cfg<T, N>(1, csize, nullptr, attr);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_fwd_fused<T, N>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

template <typename T>
cudaError_t FwdFusedLaunch<T>::run(int n, const FwdFusedArgs<T> &a, int ncl, int csize, cudaStream_t s)
{
    switch (n) {
#define OBL_CASE(N) case N: return fwd_run_n<T, N>(a, ncl, csize, s);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return cudaErrorNotSupported;
}

template <typename T> size_t FwdFusedLaunch<T>::slot_bytes(int n)
{
    switch (n) {
#define OBL_CASE(N) case N: return FwdFusedGeo<T, N>::slot_bytes();
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return 0;
}

template <typename T> int FwdFusedLaunch<T>::max_clusters(int n, int csize)
{
    switch (n) {
#define OBL_CASE(N) case N: return fwd_max_clusters_n<T, N>(csize);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return 0;
}

template struct FwdFusedLaunch<float>;
template struct FwdFusedLaunch<double>;

template <typename T, int N> static cudaError_t rows3_run_n(const RowsFwd3Args<T> &a, cudaStream_t s)
{
    using GG = FwdFusedGeo<T, N>;
    const size_t sm = sizeof(C2<T>) * ((size_t)GG::TF + GG::TB + GG::TPB) + GG::row_scr;
    static int caps[kMaxDevices] = {};
    auto kern = k_rows_fwd3<T, N>;
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
    const long long per_cta = 8LL * GG::LPW;
    const long long want = (a.npairs + per_cta - 1) / per_cta;
    const int grid = (int)(want < cap ? want : cap);
    if (grid < 1) return cudaSuccess;
    kern<<<grid, 256, sm, s>>>(a);
    return cudaGetLastError();
}

template <typename T> cudaError_t RowsFwd3Launch<T>::run(int n, const RowsFwd3Args<T> &a, cudaStream_t s)
{
    switch (n) {
#define OBL_CASE(N) case N: return rows3_run_n<T, N>(a, s);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return cudaErrorNotSupported;
}

template struct RowsFwd3Launch<float>;
template struct RowsFwd3Launch<double>;

template <typename T, int N> static cudaError_t pinv_cols_n(const PinvColArgs<T> &a, int nlev, cudaStream_t s)
{
    using D = LineDerived<N, OP_INV>;
    // (the 4-CTA shape of the other column kernels measured slower here: the four inverse
    // transforms of one load need more than its 64 registers)
    constexpr bool TWG = false;
    constexpr int NW = TWG ? 8 : col_warps<T, N, OP_INV>();
    const size_t sm = sizeof(C2<T>) * ((TWG ? 0 : (size_t)D::TB) + (size_t)N * LmGeo<T>::WB);
    static bool inits[kMaxDevices] = {};
    auto kern = k_cols_pinv<T, N, NW, TWG>;
    const int ds = device_slot();
    if (ds < 0 || !inits[ds]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        if (ds >= 0) inits[ds] = true;
    }
    dim3 grid((a.lhx + LmGeo<T>::WB - 1) / LmGeo<T>::WB, nlev);
    kern<<<grid, 32 * NW, sm, s>>>(a);
    return cudaGetLastError();
}

template <typename T, int N> static cudaError_t pinv_rows_n(const PinvRowArgs<T> &a, cudaStream_t s)
{
    using D = LineDerived<N, OP_INV>;
    const size_t sm = sizeof(C2<T>) * ((size_t)D::TB + (size_t)8 * D::LPW * scratch_len(N));
    static int caps[kMaxDevices] = {};
    auto kern = k_rows_pinv<T, N>;
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
    const long long items = 4 * ((a.npairs + D::LPW - 1) / D::LPW);   // (pair group, component)
    const long long want = (items + 7) / 8;
    const int grid = (int)(want < cap ? want : cap);
    if (grid < 1) return cudaSuccess;
    kern<<<grid, 256, sm, s>>>(a);
    return cudaGetLastError();
}

template <typename T> cudaError_t PinvLaunch<T>::cols(int n, const PinvColArgs<T> &a, int nlev, cudaStream_t s)
{
    switch (n) {
#define OBL_CASE(N) case N: return pinv_cols_n<T, N>(a, nlev, s);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return cudaErrorNotSupported;
}
template <typename T> cudaError_t PinvLaunch<T>::rows(int n, const PinvRowArgs<T> &a, cudaStream_t s)
{
    switch (n) {
#define OBL_CASE(N) case N: return pinv_rows_n<T, N>(a, s);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return cudaErrorNotSupported;
}
template struct PinvLaunch<float>;
template struct PinvLaunch<double>;

} // namespace obl
