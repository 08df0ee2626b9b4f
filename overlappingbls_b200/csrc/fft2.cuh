// fft2.cuh -- register-chained Stockham FFT for one line per LL lanes of a warp.
//
// A line of compile-time length N is spread over LL lanes (LL = 32, 16 or 8; a warp
// carries 32/LL lines in lockstep).  For a radix-R pass the butterflies are
// j = t + LL*b (t = lane within the line, b < PER = ceil(N/R / LL)); the canonical
// register layout of the pass is
//     D(R):  v[b*R + r]  holds element  j + r*(N/R)
// The first pass of a plan consumes its inputs from registers in D(R_first) (so the
// caller loads them straight from global memory or a shared tile, coalesced), every
// intermediate pass goes through a padded per-line shared-memory scratch, and the last
// pass leaves its outputs in registers in D(R_last).  A backward transform with the
// reversed plan starts from D(R_last), so forward -> spectral op -> backward needs no
// shared-memory traffic between the two transforms, and the 3/2-rule zero padding /
// truncation between lengths N and 3N/2 is a pure register remap when the padded plan
// ends with a radix 3/2 times larger (same butterfly count N/R).
//
// Inter-pass twiddles come from a per-plan table with one block per pass (NS > 1):
// block[r*NS + k] = w_N^{r*k*N/(NS*R)}, w_N = exp(-2 pi i / N), computed in FP64 on the
// host; consecutive lanes read consecutive k, so the reads are bank-conflict free.
#pragma once
#include "fft.cuh"

namespace obl {

// ----------------------------------------------------------------------------- plans
template <int... Rs> struct RPlan {};

template <class P> struct PlanInfo;
template <int R0, int... Rs> struct PlanInfo<RPlan<R0, Rs...>> {
    static constexpr int first = R0;
    static constexpr int count = 1 + sizeof...(Rs);
    static constexpr int product = R0 * PlanInfo<RPlan<Rs...>>::product;
    static constexpr int last = (sizeof...(Rs) == 0) ? R0 : PlanInfo<RPlan<Rs...>>::last;
};
template <> struct PlanInfo<RPlan<>> {
    static constexpr int first = 1, count = 0, product = 1, last = 1;
};

template <class P, class Acc = RPlan<>> struct Reverse;
template <int... A> struct Reverse<RPlan<>, RPlan<A...>> { using type = RPlan<A...>; };
template <int R0, int... Rs, int... A> struct Reverse<RPlan<R0, Rs...>, RPlan<A...>> {
    using type = typename Reverse<RPlan<Rs...>, RPlan<R0, A...>>::type;
};

// Base plans for the supported line lengths (forward direction).  The padded plan of
// length 3N/2 replaces the last radix R by 3R/2.
template <int N> struct Base;
template <> struct Base<32> { using type = RPlan<2, 4, 4>; };
template <> struct Base<48> { using type = RPlan<4, 3, 4>; };
template <> struct Base<64> { using type = RPlan<4, 4, 4>; };
template <> struct Base<96> { using type = RPlan<4, 4, 6>; };
template <> struct Base<128> { using type = RPlan<4, 4, 8>; };
template <> struct Base<192> { using type = RPlan<4, 6, 8>; };
template <> struct Base<256> { using type = RPlan<4, 8, 8>; };
template <> struct Base<384> { using type = RPlan<6, 8, 8>; };
template <> struct Base<512> { using type = RPlan<8, 8, 8>; };
// lengths with a factor 5 (FFTW plans any length, 002_fft.f90:78-117); the middle radix
// carries the 5 so that the last one stays even for its 3/2-rule partner
template <> struct Base<80> { using type = RPlan<4, 5, 4>; };
template <> struct Base<160> { using type = RPlan<4, 5, 8>; };
template <> struct Base<240> { using type = RPlan<6, 5, 8>; };
template <> struct Base<320> { using type = RPlan<8, 5, 8>; };
template <> struct Base<640> { using type = RPlan<8, 10, 8>; };

template <class P> struct PadOf;
template <int R0, int R1, int R2> struct PadOf<RPlan<R0, R1, R2>> { using type = RPlan<R0, R1, 3 * R2 / 2>; };

template <int N> using FwdPlan = typename Base<N>::type;                    // length N, forward
template <int N> using BwdPlan = typename Reverse<FwdPlan<N>>::type;       // length N, backward
template <int N> using PadFwdPlan = typename PadOf<FwdPlan<N>>::type;      // length 3N/2, forward
template <int N> using PadBwdPlan = typename Reverse<PadFwdPlan<N>>::type; // length 3N/2, backward

// number of butterflies of the smallest-count pass; lanes per line = the largest of
// 32/16/8 that keeps that pass at least half busy
template <int N, class P> struct MinNB;
template <int N, int R0> struct MinNB<N, RPlan<R0>> { static constexpr int v = N / R0; };
template <int N, int R0, int R1, int... Rs> struct MinNB<N, RPlan<R0, R1, Rs...>> {
    static constexpr int a = N / R0, b = MinNB<N, RPlan<R1, Rs...>>::v;
    static constexpr int v = a < b ? a : b;
};
template <int N, class P> struct LL_ {
    static constexpr int nb = MinNB<N, P>::v;
    static constexpr int v = nb >= 32 ? 32 : (nb >= 16 ? 16 : 8);
};

// registers per lane for a plan: max over passes of PER*R
template <int N, int LL, class P> struct Regs;
template <int N, int LL, int R0> struct Regs<N, LL, RPlan<R0>> {
    static constexpr int v = ((N / R0 + LL - 1) / LL) * R0;
};
template <int N, int LL, int R0, int R1, int... Rs> struct Regs<N, LL, RPlan<R0, R1, Rs...>> {
    static constexpr int a = ((N / R0 + LL - 1) / LL) * R0, b = Regs<N, LL, RPlan<R1, Rs...>>::v;
    static constexpr int v = a > b ? a : b;
};

// twiddle table size of a plan (entries)
template <int N, int NS, class P> struct TwSize;
template <int N, int NS> struct TwSize<N, NS, RPlan<>> { static constexpr int v = 0; };
template <int N, int NS, int R0, int... Rs> struct TwSize<N, NS, RPlan<R0, Rs...>> {
    static constexpr int v = (NS > 1 ? R0 * NS : 0) + TwSize<N, NS * R0, RPlan<Rs...>>::v;
};
template <int N, class P> constexpr int tw_size() { return TwSize<N, 1, P>::v; }

// scratch line length (complex) with one pad slot per 8 elements
// Per-line scratch with one pad element every 2^OBL_SIDX_SHIFT elements (a build-time
// tuning knob; the column tiles below keep room for the default shift of 3 or more).
#ifndef OBL_SIDX_SHIFT
#define OBL_SIDX_SHIFT 5
#endif
static_assert(OBL_SIDX_SHIFT >= 3, "tile_rows assumes at most one pad element per 8");
__host__ __device__ constexpr int scratch_len(int n) { return n + (n >> OBL_SIDX_SHIFT) + 1; }
__device__ __forceinline__ int sidx(int i) { return i + (i >> OBL_SIDX_SHIFT); }

// Scratch accessors: a padded contiguous line, a complex column of a shared tile, or
// two adjacent real columns of a shared tile read as one complex line.  Tile rows are
// padded (row i lives at physical row i + i/8) and the row stride is odd, which keeps
// the Stockham load/store patterns free of bank conflicts.
template <typename C> struct LineScratch {
    C *p;
    __device__ __forceinline__ C ld(int i) const { return p[sidx(i)]; }
    __device__ __forceinline__ void st(int i, C v) { p[sidx(i)] = v; }
};
// (`on` = false: an idle line of a partial tile; its stores are dropped)
template <typename C> struct TileCol {
    C *tile; int S; int c; bool on;
    __device__ __forceinline__ C ld(int i) const { return tile[sidx(i) * S + c]; }
    __device__ __forceinline__ void st(int i, C v)
    {
        if (on) tile[sidx(i) * S + c] = v;
    }
};
template <typename T> struct TilePair {
    T *tile; int S; int c; bool on;
    __device__ __forceinline__ C2<T> ld(int i) const
    {
        const T *p = tile + sidx(i) * S + c;
        return mk<T>(p[0], p[1]);
    }
    __device__ __forceinline__ void st(int i, C2<T> v)
    {
        if (!on) return;
        T *p = tile + sidx(i) * S + c;
        p[0] = v.x;
        p[1] = v.y;
    }
};
__host__ __device__ constexpr int tile_rows(int n) { return n + n / 8 + 1; }
// Line-minor scratch: element i of line l at p[i*WB + l].  Threads of a warp address
// consecutive lines of one or a few elements, so every access is bank-conflict free.
template <typename C, int WB> struct LineMinor {
    C *p; int l;
    __device__ __forceinline__ C ld(int i) const { return p[i * WB + l]; }
    __device__ __forceinline__ void st(int i, C v) { p[i * WB + l] = v; }
};

// ----------------------------------------------------------------------------- passes
// one radix-R pass; IN_REGS: inputs already in v (D(R)), else loaded from scratch;
// OUT_REGS: outputs stay in v (only legal for the last pass), else stored to scratch.
// BS: the lines' scratch is shared by threads of several warps (line-minor column layout),
// so passes are separated by __syncthreads() instead of __syncwarp().
template <int N, int R, int NS, int LL, bool FWD, bool IN_REGS, bool OUT_REGS, bool BS, typename C, class SC>
__device__ __forceinline__ void pass(C *v, SC &sc, const C *twb, int t)
{
    constexpr int NB = N / R;
    constexpr int PER = (NB + LL - 1) / LL;
    constexpr bool FULL = (NB % LL) == 0;
    if constexpr (!IN_REGS) {
#pragma unroll
        for (int b = 0; b < PER; ++b) {
            const int j = t + LL * b;
            if (FULL || j < NB) {
#pragma unroll
                for (int r = 0; r < R; ++r) v[b * R + r] = sc.ld(j + r * NB);
            }
        }
        if constexpr (BS) __syncthreads();
        else __syncwarp();
    }
#pragma unroll
    for (int b = 0; b < PER; ++b) {
        const int j = t + LL * b;
        if (FULL || j < NB) {
            const int k = (NS > 1) ? j % NS : 0;
            if constexpr (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    const C w = twb[r * NS + k];
                    v[b * R + r] = FWD ? cmul(v[b * R + r], w) : cmulc(v[b * R + r], w);
                }
            }
            Dft<R, FWD>::run(v + b * R);
            if constexpr (!OUT_REGS) {
                const int base = (j / NS) * NS * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) sc.st(base + r * NS, v[b * R + r]);
            }
        }
    }
    if constexpr (!OUT_REGS) {
        if constexpr (BS) __syncthreads();
        else __syncwarp();
    }
}

template <int N, int NS, int LL, bool FWD, bool FIRST, bool BS, typename C, class SC, int R0, int... Rs>
__device__ __forceinline__ void chain(C *v, SC &sc, const C *tw, int t, RPlan<R0, Rs...>)
{
    constexpr bool LAST = sizeof...(Rs) == 0;
    pass<N, R0, NS, LL, FWD, FIRST, LAST, BS>(v, sc, tw, t);
    if constexpr (!LAST) {
        constexpr int adv = (NS > 1) ? R0 * NS : 0;
        chain<N, NS * R0, LL, FWD, false, BS, C>(v, sc, tw + adv, t, RPlan<Rs...>{});
    }
}

// Transform the line held in v (layout D(first radix of P)); result in D(last radix).
// sc: scratch accessor of at least N elements; tw: the plan's twiddle table.
template <int N, class P, int LL, bool FWD, bool BS = false, typename C, class SC>
__device__ __forceinline__ void fft_regs(C *v, SC &sc, const C *tw, int t)
{
    static_assert(PlanInfo<P>::product == N, "plan does not multiply to N");
    chain<N, 1, LL, FWD, true, BS, C>(v, sc, tw, t, P{});
}

// D(R) geometry helpers
template <int N, int R, int LL> struct Geo {
    static constexpr int NB = N / R;
    static constexpr int PER = (NB + LL - 1) / LL;
    static constexpr bool FULL = (NB % LL) == 0;
};

// Host-side twiddle table of a plan (same layout as the device blocks).
template <class P> struct PlanList;
template <int... Rs> struct PlanList<RPlan<Rs...>> {
    static constexpr int n = sizeof...(Rs);
    static constexpr int r[sizeof...(Rs)] = {Rs...};
};

} // namespace obl
