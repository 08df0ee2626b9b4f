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
    static bool init = false, big = false;
    auto kern = k_fwd_fused<T, N>;
    if (!init) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)FwdFusedGeo<T, N>::smem);
        if (e != cudaSuccess) return e;
        init = true;
    }
    if (csize > 8 && !big) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
        big = true;
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

} // namespace obl
