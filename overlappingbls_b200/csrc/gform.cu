// gform.cu -- the pressure RHS in G form: one y-transform for the x- and z-parts.
//
// The right-hand side of press_stag_array (109_press_stag_array.f90:203-225) per mode is
//     i*(kx*H_x + ky*H_y) + (H_z(z+1) - H_z(z) [+ H_z(0) at z = 1])/dz,
// with H = the 2D transform (x r2c, then y c2c) of the scaled u, v, w.  kx and the
// z-difference are constant along y, so by linearity of the y-transform
//     G = i*kx*H_x + (H_z(z+1) - H_z(z) [+ H_z(0)])/dz
// can be formed from the x-spectra before it: one y-transform of G (written over H_x)
// replaces those of H_x and H_z, and the solve forms G + i*ky*H_y.  H_z is still
// transformed at level 0 (the Neumann ghost p_hat(0) = p_hat(1) - dz*H_z(0), :313-315)
// and, at levels 1..L, in the line group of kx = 0 only: the (0,0) mode's RHS is H_z
// itself (:219-221).
#include "lines_dispatch.cuh"
#include "press.cuh"

namespace obl {

// G of level z + 1 (z = the launch's plane index); FIRST: the launch of level 1 alone,
// whose z-difference also takes H_z(0)
template <typename T, bool FIRST> struct GSrc {
    const C2<T> *Hx, *Hz;
    const double *kx;
    long long S;
    int lhx, lv0;
    T idz;
    __device__ __forceinline__ C2<T> operator()(int z, int i, int gl) const
    {
        const long long lv = lv0 + z;
        const long long q = (long long)i * lhx + gl;
        if (!ck_in(q, S, CK_GFORM_LOAD)) return mk<T>(0, 0);
        const C2<T> hx = __ldcg(Hx + S * lv + q), hzc = __ldcg(Hz + S * lv + q), hzn = __ldcg(Hz + S * (lv + 1) + q);
        C2<T> dh = csub(hzn, hzc);
        if constexpr (FIRST) dh = cadd(dh, __ldcg(Hz + q));
        const T k = (T)kx[gl];
        return mk<T>(-k * hx.y + dh.x * idz, k * hx.x + dh.y * idz);
    }
};

template <typename T, int N, int NW, int WB, bool TWG, bool FIRST>
__global__ void __launch_bounds__(32 * NW, col_min_blocks(NW, TWG, col_warps_sm<OP_FWD>())) k_cols_gform(ColArgs<T> a, GSrc<T, FIRST> g)
{
    using C = C2<T>;
    using D = LineDerived<N, OP_FWD>;
    extern __shared__ __align__(16) unsigned char smraw[];
    if constexpr (TWG) {
        cols2_unit<T, N, OP_FWD, false, NW, WB, NoColEpi, false, GSrc<T, FIRST>>(
            a, blockIdx.x, blockIdx.y, a.twF, a.twB, reinterpret_cast<C *>(smraw), NoColEpi(), nullptr, g);
    } else {
        C *twF = reinterpret_cast<C *>(smraw);
        C *buf = twF + D::TF + D::TB;
        load_tables<T, N, OP_FWD>(a.twF, a.twB, twF, twF + D::TF);
        __syncthreads();
        cols2_unit<T, N, OP_FWD, false, NW, WB, NoColEpi, false, GSrc<T, FIRST>>(a, blockIdx.x, blockIdx.y, twF,
                                                                                 twF + D::TF, buf, NoColEpi(), nullptr, g);
    }
}

// the same CTA shape and shared memory as the plain y-transform of the RHS spectra
template <typename T, int N, bool FIRST>
static cudaError_t gform_launch(const ColArgs<T> &a, const GSrc<T, FIRST> &g, cudaStream_t s)
{
    constexpr int NW = col_warps<T, N, OP_FWD>(), WB = col_lines<T, N, OP_FWD>();
    constexpr bool TWG = col_tw_global<T, N, OP_FWD>();
    using D = LineDerived<N, OP_FWD>;
    const size_t sm = TWG ? sizeof(C2<T>) * (size_t)D::NM * WB : cols2_smem<T, N, OP_FWD, WB>();
    auto kern = k_cols_gform<T, N, NW, WB, TWG, FIRST>;
    static bool inits[kMaxDevices] = {};
    const int ds = device_slot();
    if (ds < 0 || !inits[ds]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        if (ds >= 0) inits[ds] = true;
    }
    dim3 grid((a.ncols + WB - 1) / WB, a.nlev);
    if (grid.x < 1 || grid.y < 1) return cudaSuccess;
    kern<<<grid, 32 * NW, sm, s>>>(a, g);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_gform_cols(int ny, C2<T> *Hx, const C2<T> *Hz, const double *kx, long long S, int lhx, int L,
                              double dz, const C2<T> *twF, cudaStream_t s)
{
    // level 1 (with H_z(0)), then levels 2..L; G of level lv is written over H_x(lv)
    for (int part = 0; part < 2; ++part) {
        const int lv0 = part == 0 ? 1 : 2, nlev = part == 0 ? 1 : L - 1;
        if (nlev < 1) continue;
        ColArgs<T> a{};
        a.src = Hx + S * lv0;
        a.dst = Hx + S * lv0;
        a.src_row = a.dst_row = lhx;
        a.src_plane = a.dst_plane = S;
        a.ncols = lhx;
        a.nlev = nlev;
        a.scale = (T)1;
        a.twF = twF;
        a.zero_nyq = 1;   // 203_fftn_mpi.f90:33
        cudaError_t e = cudaErrorInvalidValue;
        if (part == 0) {
            GSrc<T, true> g{Hx, Hz, kx, S, lhx, lv0, (T)(1.0 / dz)};
            switch (ny) {
#define OBL_CASE(N) case N: e = gform_launch<T, N, true>(a, g, s); break;
                OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
            }
        } else {
            GSrc<T, false> g{Hx, Hz, kx, S, lhx, lv0, (T)(1.0 / dz)};
            switch (ny) {
#define OBL_CASE(N) case N: e = gform_launch<T, N, false>(a, g, s); break;
                OBL_FOR_EACH_N(OBL_CASE)
#undef OBL_CASE
            }
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template cudaError_t launch_gform_cols<float>(int, C2<float> *, const C2<float> *, const double *, long long, int, int,
                                              double, const C2<float> *, cudaStream_t);
template cudaError_t launch_gform_cols<double>(int, C2<double> *, const C2<double> *, const double *, long long, int,
                                               int, double, const C2<double> *, cudaStream_t);

} // namespace obl
