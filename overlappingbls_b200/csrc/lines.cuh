// lines.cuh -- batched 1D spectral line operations along x (rows) and y (columns).
//
// These kernels are the building blocks of every hot-path routine:
//   rows    (x direction, contiguous):  ddx, x-pad, x-unpad, x r2c, x c2r
//   columns (y direction, strided):     ddy, y-pad, y-unpad, y c2c forward/backward
// Real lines are transformed two at a time as one complex line (z = a + i b): every
// spectral operation used here is a real-to-real linear map that acts on Z[k] and
// Z[N-k] symmetrically (i*k multipliers with signed k, truncation/zero-extension),
// so Re(IFFT(op(FFT(z)))) = op(a) and Im(...) = op(b) exactly as the reference's
// per-line r2c -> op -> c2r computes them (004_derivatives.f90:33-39,
// 108_01_padd.f90:102-127,163-190).  Columns are staged through a shared-memory tile
// (the on-GPU replacement of the reference's mpi_alltoall pencil transposes,
// 203_fftn_mpi.f90:71-371) so global loads and stores stay coalesced along x.
#pragma once
#include "fft.cuh"

namespace obl {

enum LineOp : int { OP_DERIV = 0, OP_PAD = 1, OP_UNPAD = 2, OP_FWD = 3, OP_INV = 4 };

template <typename T> struct RowArgs {
    const void *src;          // real rows (DERIV/PAD/UNPAD/FWD) or complex rows (INV)
    void *dst;                // real rows (DERIV/PAD/UNPAD/INV) or complex rows (FWD)
    long long src_stride;     // elements (of the row's type) between consecutive rows
    long long dst_stride;
    long long npairs;         // number of row pairs (rows 2p, 2p+1)
    T scale;                  // multiplies the input at load
    const double *ktab;       // DERIV: k[0..N/2] (the Nyquist entry is 0)
    const C2<T> *twI, *twO;   // twiddle tables w_N^m for the input / output lengths
    T pad_scale;              // INV with pad_mode: dst pad columns *= pad_scale
    int pad_mode;
};

template <typename T> struct ColArgs {
    const void *src;
    void *dst;
    long long src_row, dst_row;      // elements between rows
    long long src_plane, dst_plane;  // elements between planes
    int ncols;                       // real columns (real ops) / complex columns
    int nlev;
    T scale;                         // multiplies the input at load
    const double *ktab;              // DERIV: k[0..N/2]; INV kmul=1: kx per column; kmul=2: ky per row
    const C2<T> *twI, *twO;
    int pad_copy;                    // UNPAD: also write columns 0,1 into ncols, ncols+1
    int zero_nyq;                    // FWD: zero the Nyquist row (203_fftn_mpi.f90:33)
    int kmul;                        // INV: 0 none, 1 multiply by i*kx(col), 2 by i*ky(row)
};

// ----------------------------------------------------------------------------- accessors
// Two adjacent real columns (c, c+1) of a real tile with row stride S, viewed as one
// complex line.
template <typename T> struct PairLine {
    T *tile; int S; int c;
    __device__ __forceinline__ C2<T> ld(int i) const { return mk<T>(tile[i * S + c], tile[i * S + c + 1]); }
    __device__ __forceinline__ void st(int i, C2<T> v) { tile[i * S + c] = v.x; tile[i * S + c + 1] = v.y; }
};
template <typename T> struct CplxLine {
    C2<T> *tile; int S; int c;
    __device__ __forceinline__ C2<T> ld(int i) const { return tile[i * S + c]; }
    __device__ __forceinline__ void st(int i, C2<T> v) { tile[i * S + c] = v; }
};

// ----------------------------------------------------------------------------- spectral ops
// z[k] *= i * ks, ks = +k (k <= N/2) or -(N-k); ktab[N/2] = 0 removes the Nyquist mode
template <typename T, int N, class Line>
__device__ __forceinline__ void op_deriv(Line &L, const double *ktab, int lane)
{
    for (int k = lane; k < N; k += 32) {
        const T kk = (k <= N / 2) ? (T)ktab[k] : -(T)ktab[N - k];
        C2<T> z = L.ld(k);
        L.st(k, mk<T>(-kk * z.y, kk * z.x));
    }
    __syncwarp();
}
// zero-extend the spectrum of length NI to NO = 3 NI / 2, dropping the Nyquist bin
template <typename T, int NI, int NO, class Line>
__device__ __forceinline__ void op_pad(Line &L, int lane)
{
    for (int m = 1 + lane; m < NI / 2; m += 32) L.st(NO - m, L.ld(NI - m));
    __syncwarp();
    for (int k = NI / 2 + lane; k <= NI; k += 32) L.st(k, mk<T>(0, 0));
    __syncwarp();
}
// truncate the spectrum of length NI = 3 NO / 2 to NO, zeroing the new Nyquist bin
template <typename T, int NI, int NO, class Line>
__device__ __forceinline__ void op_unpad(Line &L, int lane)
{
    for (int m = 1 + lane; m < NO / 2; m += 32) L.st(NO - m, L.ld(NI - m));
    __syncwarp();
    if (lane == 0) L.st(NO / 2, mk<T>(0, 0));
    __syncwarp();
}

// ----------------------------------------------------------------------------- row kernel
template <typename T, int NI, int NO, int OP>
__global__ void __launch_bounds__(256) k_rows(RowArgs<T> a)
{
    using C = C2<T>;
    constexpr int NM = NI > NO ? NI : NO;
    constexpr int LP = line_pad(NM);
    extern __shared__ __align__(16) unsigned char smraw[];
    C *twI = reinterpret_cast<C *>(smraw);
    C *twO = (NI == NO) ? twI : twI + NI;
    C *lines = twO + NO;
    for (int i = threadIdx.x; i < NI; i += blockDim.x) twI[i] = a.twI[i];
    if (NI != NO)
        for (int i = threadIdx.x; i < NO; i += blockDim.x) twO[i] = a.twO[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    SmemLine<C> L{lines + warp * LP};

    for (long long pr = (long long)blockIdx.x * nw + warp; pr < a.npairs; pr += (long long)gridDim.x * nw) {
        const long long r0 = 2 * pr;
        if constexpr (OP == OP_INV) {
            // two Hermitian half spectra A (row r0), B (row r0+1) -> Z = A + iB on all N bins;
            // Im of the DC and Nyquist bins is ignored, as in FFTW's c2r
            constexpr int H = NO / 2;
            const C *A = reinterpret_cast<const C *>(a.src) + r0 * a.src_stride;
            const C *B = A + a.src_stride;
            for (int k = lane; k <= H; k += 32) {
                C av = A[k], bv = B[k];
                if (k == 0 || k == H) { av.y = 0; bv.y = 0; }
                L.st(k, mk<T>(av.x - bv.y, av.y + bv.x));
                if (k > 0 && k < H) L.st(NO - k, mk<T>(av.x + bv.y, bv.x - av.y));
            }
        } else {
            const T *A = reinterpret_cast<const T *>(a.src) + r0 * a.src_stride;
            const T *B = A + a.src_stride;
            for (int x = lane; x < NI; x += 32) L.st(x, mk<T>(A[x] * a.scale, B[x] * a.scale));
        }
        __syncwarp();
        if constexpr (OP != OP_INV) fft_line<NI, true, C>(L, twI, lane);

        if constexpr (OP == OP_FWD) {
            // split Z into the half spectra of both rows; zero the x-Nyquist (203_fftn_mpi.f90:25)
            constexpr int H = NI / 2;
            C *Ao = reinterpret_cast<C *>(a.dst) + r0 * a.dst_stride;
            C *Bo = Ao + a.dst_stride;
            for (int k = lane; k <= H; k += 32) {
                if (k == H) {
                    Ao[k] = mk<T>(0, 0);
                    Bo[k] = mk<T>(0, 0);
                } else {
                    const C z = L.ld(k), zc = cconj(L.ld(k == 0 ? 0 : NI - k));
                    const C s = cadd(z, zc), d = csub(z, zc);
                    Ao[k] = mk<T>((T)0.5 * s.x, (T)0.5 * s.y);
                    Bo[k] = mk<T>((T)0.5 * d.y, (T)-0.5 * d.x);
                }
            }
            __syncwarp();
        } else {
            if constexpr (OP == OP_DERIV) op_deriv<T, NI>(L, a.ktab, lane);
            if constexpr (OP == OP_PAD) op_pad<T, NI, NO>(L, lane);
            if constexpr (OP == OP_UNPAD) op_unpad<T, NI, NO>(L, lane);
            fft_line<NO, false, C>(L, twO, lane);
            T *A = reinterpret_cast<T *>(a.dst) + r0 * a.dst_stride;
            T *B = A + a.dst_stride;
            for (int x = lane; x < NO; x += 32) {
                const C z = L.ld(x);
                A[x] = z.x;
                B[x] = z.y;
            }
            if (OP == OP_INV && a.pad_mode && lane < 2) {
                A[NO + lane] *= a.pad_scale;
                B[NO + lane] *= a.pad_scale;
            }
            __syncwarp();
        }
    }
}

// ----------------------------------------------------------------------------- column kernel
template <typename T, bool REAL> struct ColTile {
    // columns per tile: 128-byte row segments
    static constexpr int W = REAL ? (int)(128 / sizeof(T)) : (int)(128 / (2 * sizeof(T)));
    static constexpr int S = W + 1;   // odd row stride (in tile elements)
};

template <typename T, int NI, int NO, int OP, bool REAL>
__global__ void __launch_bounds__(256) k_cols(ColArgs<T> a)
{
    using C = C2<T>;
    using E = typename std::conditional<REAL, T, C>::type;   // tile element
    constexpr int W = ColTile<T, REAL>::W, S = ColTile<T, REAL>::S;
    constexpr int NM = NI > NO ? NI : NO;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *twI = reinterpret_cast<C *>(smraw);
    C *twO = (NI == NO) ? twI : twI + NI;
    E *tile = reinterpret_cast<E *>(twO + NO);
    (void)NM;

    const int z = blockIdx.y;
    const int c0 = blockIdx.x * W;
    const int nc = min(W, a.ncols - c0);
    const E *src = reinterpret_cast<const E *>(a.src) + (long long)z * a.src_plane + c0;
    E *dst = reinterpret_cast<E *>(a.dst) + (long long)z * a.dst_plane + c0;

    for (int i = threadIdx.x; i < NI; i += blockDim.x) twI[i] = a.twI[i];
    if (NI != NO)
        for (int i = threadIdx.x; i < NO; i += blockDim.x) twO[i] = a.twO[i];

    // coalesced tile load (rows of W elements), with the optional i*k multiplier
    for (int idx = threadIdx.x; idx < NI * W; idx += blockDim.x) {
        const int r = idx / W, c = idx - r * W;
        E v;
        if constexpr (REAL) {
            v = (c < nc) ? src[(long long)r * a.src_row + c] * a.scale : (T)0;
        } else {
            v = (c < nc) ? src[(long long)r * a.src_row + c] : mk<T>(0, 0);
            if (OP == OP_INV && a.kmul) {
                const T kk = (T)(a.kmul == 1 ? (c < nc ? a.ktab[c0 + c] : 0.0) : a.ktab[r]);
                v = mk<T>(-kk * v.y, kk * v.x);
            }
            v.x *= a.scale;
            v.y *= a.scale;
        }
        tile[r * S + c] = v;
    }
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    constexpr int NL = REAL ? W / 2 : W;
    for (int l = warp; l < NL; l += nw) {
        const int c = REAL ? 2 * l : l;
        if (c >= nc) break;
        auto run = [&](auto &L) {
            if constexpr (OP != OP_INV) fft_line<NI, true, C>(L, twI, lane);
            if constexpr (OP == OP_FWD) {
                if (a.zero_nyq && lane == 0) L.st(NI / 2, mk<T>(0, 0));
                __syncwarp();
            } else {
                if constexpr (OP == OP_DERIV) op_deriv<T, NI>(L, a.ktab, lane);
                if constexpr (OP == OP_PAD) op_pad<T, NI, NO>(L, lane);
                if constexpr (OP == OP_UNPAD) op_unpad<T, NI, NO>(L, lane);
                fft_line<NO, false, C>(L, twO, lane);
            }
        };
        if constexpr (REAL) {
            PairLine<T> L{tile, S, c};
            run(L);
        } else {
            CplxLine<T> L{tile, S, c};
            run(L);
        }
    }
    __syncthreads();

    for (int idx = threadIdx.x; idx < NO * W; idx += blockDim.x) {
        const int r = idx / W, c = idx - r * W;
        if (c < nc) dst[(long long)r * a.dst_row + c] = tile[r * S + c];
    }
    if constexpr (OP == OP_UNPAD && REAL) {
        // var(nxt+1:ldx,:) = var(1:2,:) (108_01_padd.f90:195)
        if (a.pad_copy && c0 == 0)
            for (int r = threadIdx.x; r < NO; r += blockDim.x) {
                E *d = reinterpret_cast<E *>(a.dst) + (long long)z * a.dst_plane + (long long)r * a.dst_row;
                d[a.ncols] = tile[r * S + 0];
                d[a.ncols + 1] = tile[r * S + 1];
            }
    }
}

// ----------------------------------------------------------------------------- launchers
template <typename T, int NI, int NO, int OP>
inline size_t rows_smem()
{
    constexpr int NM = NI > NO ? NI : NO;
    return sizeof(C2<T>) * ((NI == NO ? NI : NI + NO) + 8 * line_pad(NM));
}
template <typename T, int NI, int NO, int OP, bool REAL>
inline size_t cols_smem()
{
    constexpr int NM = NI > NO ? NI : NO;
    using E = typename std::conditional<REAL, T, C2<T>>::type;
    return sizeof(C2<T>) * (NI + NO) + sizeof(E) * (size_t)NM * ColTile<T, REAL>::S;
}

template <typename T, int NI, int NO, int OP>
cudaError_t launch_rows_t(const RowArgs<T> &a, cudaStream_t s)
{
    static int grid_cap = 0;
    const size_t sm = rows_smem<T, NI, NO, OP>();
    auto kern = k_rows<T, NI, NO, OP>;
    if (!grid_cap) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        int dev = 0, nsm = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, sm);
        grid_cap = nsm * (per > 0 ? per : 1);
    }
    long long want = (a.npairs + 7) / 8;
    int grid = (int)(want < grid_cap ? want : grid_cap);
    if (grid < 1) return cudaSuccess;
    kern<<<grid, 256, sm, s>>>(a);
    return cudaGetLastError();
}

template <typename T, int NI, int NO, int OP, bool REAL>
cudaError_t launch_cols_t(const ColArgs<T> &a, cudaStream_t s)
{
    static bool init = false;
    const size_t sm = cols_smem<T, NI, NO, OP, REAL>();
    auto kern = k_cols<T, NI, NO, OP, REAL>;
    if (!init) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        init = true;
    }
    constexpr int W = ColTile<T, REAL>::W;
    dim3 grid((a.ncols + W - 1) / W, a.nlev);
    if (grid.x < 1 || grid.y < 1) return cudaSuccess;
    kern<<<grid, 256, sm, s>>>(a);
    return cudaGetLastError();
}

// Runtime dispatch: n is the base length (the unpadded one for PAD/UNPAD).
template <typename T> cudaError_t launch_rows(int op, int n, const RowArgs<T> &a, cudaStream_t s);
template <typename T> cudaError_t launch_cols(int op, bool real, int n, const ColArgs<T> &a, cudaStream_t s);
bool line_length_supported(int n);

} // namespace obl
