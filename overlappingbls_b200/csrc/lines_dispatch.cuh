// lines_dispatch.cuh -- runtime-length dispatch of the row / column kernels.
// Supported base lengths n (and their 3/2 partners): the grid sizes of the
// reference's production namelists and of the benchmark workloads.
#pragma once
#include <cmath>
#include <vector>

#include "lines.cuh"

#define OBL_FOR_EACH_N(X) \
    X(32) X(48) X(64) X(80) X(96) X(128) X(160) X(192) X(240) X(256) X(320) X(384) X(512) X(640)

namespace obl {

template <typename T, int N>
cudaError_t rows_n(int op, const RowArgs<T> &a, cudaStream_t s)
{
    switch (op) {
    case OP_DERIV: return launch_rows_t<T, N, OP_DERIV>(a, s);
    case OP_PAD: return launch_rows_t<T, N, OP_PAD>(a, s);
    case OP_UNPAD: return launch_rows_t<T, N, OP_UNPAD>(a, s);
    case OP_FWD: return launch_rows_t<T, N, OP_FWD>(a, s);
    case OP_INV: return launch_rows_t<T, N, OP_INV>(a, s);
    }
    return cudaErrorInvalidValue;
}

template <typename T, int N>
cudaError_t cols_n(int op, bool real, const ColArgs<T> &a, cudaStream_t s)
{
    if (real) {
        switch (op) {
        case OP_DERIV: return launch_cols_t<T, N, OP_DERIV, true>(a, s);
        case OP_PAD: return launch_cols_t<T, N, OP_PAD, true>(a, s);
        case OP_UNPAD: return launch_cols_t<T, N, OP_UNPAD, true>(a, s);
        }
    } else {
        switch (op) {
        case OP_FWD: return launch_cols_t<T, N, OP_FWD, false>(a, s);
        case OP_INV: return launch_cols_t<T, N, OP_INV, false>(a, s);
        }
    }
    return cudaErrorInvalidValue;
}

template <typename T> cudaError_t launch_rows(int op, int n, const RowArgs<T> &a, cudaStream_t s)
{
    switch (n) {
#define OBL_CASE(N) case N: return rows_n<T, N>(op, a, s);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return cudaErrorInvalidValue;
}

template <typename T> cudaError_t launch_cols(int op, bool real, int n, const ColArgs<T> &a, cudaStream_t s)
{
    switch (n) {
#define OBL_CASE(N) case N: return cols_n<T, N>(op, real, a, s);
        OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
    }
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------- host twiddle tables
template <class P> struct PlanVec;
template <int... Rs> struct PlanVec<RPlan<Rs...>> {
    static std::vector<int> get() { return {Rs...}; }
};

inline std::vector<double> plan_table_for(int N, const std::vector<int> &radices)
{
    const double pi = 3.14159265358979323846264338327950288;
    std::vector<double> out;
    int NS = 1;
    for (int R : radices) {
        if (NS > 1) {
            const int tws = N / (NS * R);
            for (int r = 0; r < R; ++r)
                for (int k = 0; k < NS; ++k) {
                    const long long m = (long long)r * k * tws % N;
                    const double ang = -2.0 * pi * (double)m / (double)N;
                    out.push_back(std::cos(ang));
                    out.push_back(std::sin(ang));
                }
        }
        NS *= R;
    }
    return out;
}

template <int N> std::vector<double> plan_table_n(int role)
{
    switch (role) {
    case ROLE_FWD: return plan_table_for(N, PlanVec<FwdPlan<N>>::get());
    case ROLE_BWD: return plan_table_for(N, PlanVec<BwdPlan<N>>::get());
    case ROLE_PADFWD: return plan_table_for(3 * N / 2, PlanVec<PadFwdPlan<N>>::get());
    case ROLE_PADBWD: return plan_table_for(3 * N / 2, PlanVec<PadBwdPlan<N>>::get());
    }
    return {};
}

} // namespace obl
