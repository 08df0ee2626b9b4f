// ensemble.cu -- host-side geometry of the persistent ensemble kernel (ensemble.cuh);
// the kernel itself is instantiated in ensemble_all.cu and ensemble_part*.cu.
#include <algorithm>

#include "ensemble_kernel.cuh"
#include "obl.h"

namespace obl {

bool ens_length_supported(int n)
{
    switch (n) {
#define OBL_C(N) case N: return true;
        OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
    }
    return false;
}

template <typename T> int ens_wb() { return LmGeo<T>::WB; }

// ----------------------------------------------------------------------------- self-test
// One CTA through the grid barrier with its arrival counter preset: 0 releases at once;
// any other value never reaches the release count (nothing else arrives), so the bounded
// wait gives up and raises the error flag, as a lost CTA of a real launch would.
__global__ void k_barrier_selftest(unsigned *bar, int *passed)
{
    const bool ok = ens_barrier(bar, reinterpret_cast<int *>(bar + 2));
    if (threadIdx.x == 0) *passed = ok ? 1 : 0;
}

int ens_barrier_selftest(bool never_released, cudaStream_t s, std::string &err)
{
    unsigned *bar = nullptr;   // arrivals, generation, error flag, passed
    if (cudaMalloc(&bar, 4 * sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        err = "barrier self-test: allocation failed";
        return OBL_ERR_NOMEM;
    }
    const unsigned init[4] = {never_released ? 1u : 0u, 0u, 0u, 0u};
    cudaError_t e = cudaMemcpyAsync(bar, init, sizeof init, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        k_barrier_selftest<<<1, 128, 0, s>>>(bar, reinterpret_cast<int *>(bar + 3));
        e = cudaGetLastError();
    }
    unsigned out[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, bar, sizeof out, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(bar);
    if (e != cudaSuccess) {
        err = std::string("barrier self-test: ") + cudaGetErrorString(e);
        return OBL_ERR_CUDA;
    }
    if (out[2]) {
        err = "barrier self-test: the grid-barrier wait gave up";
        return OBL_ERR_TIMEOUT;
    }
    return out[3] ? OBL_OK : OBL_ERR_TIMEOUT;
}

// ----------------------------------------------------------------------------- host side
template <typename T> long long EnsGeoHost<T>::rows_units(int n, long long npairs)
{
    switch (n) {
#define OBL_C(N)                                                                                         \
    case N: {                                                                                            \
        const long long per = 8LL * FwdFusedGeo<T, N>::LPW;                                              \
        return (npairs + per - 1) / per;                                                                 \
    }
        OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
    }
    return 0;
}

template <typename T> long long EnsGeoHost<T>::pinv_rows_units(int n, long long npairs)
{
    switch (n) {
#define OBL_C(N)                                                                                         \
    case N: {                                                                                            \
        constexpr int LPW = LineDerived<N, OP_INV>::LPW;                                                 \
        const long long ngroups = (npairs + LPW - 1) / LPW;                                              \
        return (4 * ngroups + 7) / 8;                                                                    \
    }
        OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
    }
    return 0;
}

template <typename T, int N> static size_t ens_smem_rows()
{
    using GG = FwdFusedGeo<T, N>;
    return sizeof(C2<T>) * ((size_t)GG::TF + GG::TB + GG::TPB) + GG::row_scr;
}
template <typename T, int N> static size_t ens_smem_cols()
{
    size_t m = cols2_smem<T, N, OP_PAD>();
    m = std::max(m, cols2_smem<T, N, OP_DERIV>());
    m = std::max(m, cols2_smem<T, N, OP_FWD>());
    using D = LineDerived<N, OP_INV>;
    m = std::max(m, sizeof(C2<T>) * ((size_t)D::TB + (size_t)N * LmGeo<T>::WB));
    return m;
}
template <typename T, int N> static size_t ens_smem_pinv_rows()
{
    using D = LineDerived<N, OP_INV>;
    return sizeof(C2<T>) * ((size_t)D::TB + (size_t)8 * D::LPW * scratch_len(N));
}

template <typename T> size_t EnsGeoHost<T>::smem(int nx, int ny, int pb, int pe)
{
    size_t m = 0;
    const bool rows = pb <= 0 && pe > 0, mid = pb <= 3 && pe > 1, tail = pb <= 4 && pe > 4;
    switch (nx) {
#define OBL_C(N)                                                                                         \
    case N:                                                                                              \
        if (rows) m = std::max(m, ens_smem_rows<T, N>());                                                \
        if (tail) m = std::max(m, ens_smem_pinv_rows<T, N>());                                           \
        break;
        OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
    }
    switch (ny) {
#define OBL_C(N) case N: if (mid) m = std::max(m, ens_smem_cols<T, N>()); break;
        OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
    }
    return m;
}

template struct EnsGeoHost<float>;
template struct EnsGeoHost<double>;
template int ens_wb<float>();
template int ens_wb<double>();

} // namespace obl
