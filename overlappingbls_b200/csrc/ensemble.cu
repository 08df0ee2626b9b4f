// ensemble.cu -- host-side geometry of the persistent ensemble kernel (ensemble.cuh);
// the kernel itself is instantiated in ensemble_all.cu and ensemble_part*.cu.
#include <algorithm>

#include "ensemble_kernel.cuh"

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
