// divstress.cuh -- divergence of one row of the stress tensor (107_divstress.f90:4-104).
//
//   divstress_uv: divt = ddx(tx) + ddy(ty) + ddz_w(tz) on levels 1..nz-1   (:21-37)
//   divstress_w:  divt = ddx(tx) + ddy(ty) + ddz_uv(tz) on levels 1..nz, without the
//                 vertical term on the wall level 1 and the top level nz     (:67-99)
// with the x pad columns nxt, nxt+1 zero on the computed levels (:40, :95, :99) and the
// uncomputed levels set to BOGUS (:41-42, :79), the single-rank roles (the domain holds
// the bottom and the top).
//
// Two passes over HBM: the ddx row kernel writes ddx(tx) into divt; the ddy column
// kernel's store hook then adds that value, the vertical difference of tz and writes the
// pads, so ddy(ty) and the sum never take a trip of their own.
#pragma once
#include "lines.cuh"

namespace obl {

// Store hook of the ddy column pass (see NoColEpi): plane z of the pass is level z0 + z.
template <typename T> struct DivEpi {
    T *out;             // divt at level z0 (holds ddx(tx) when the hook runs)
    const T *tz;        // tz at level z0
    long long row, plane;
    int ncols;          // nxt: the pad pair starts here
    T rdz;              // 1/dz
    int fwd;            // 1: (tz(k+1) - tz(k)) / dz (ddz_w); 0: (tz(k) - tz(k-1)) / dz (ddz_uv)
    int zlo, zhi;       // planes of the pass that take the vertical term
    __device__ __forceinline__ void operator()(int z, int i, int line, C2<T> &x) const
    {
        const long long o = (long long)z * plane + (long long)i * row + 2 * line;
        const C2<T> d = *reinterpret_cast<const C2<T> *>(out + o);
        x.x += d.x;
        x.y += d.y;
        if (z >= zlo && z <= zhi) {
            const C2<T> hi = *reinterpret_cast<const C2<T> *>(tz + o + (fwd ? plane : 0));
            const C2<T> lo = *reinterpret_cast<const C2<T> *>(tz + o - (fwd ? 0 : plane));
            x.x += rdz * (hi.x - lo.x);
            x.y += rdz * (hi.y - lo.y);
        }
        if (line == 0)
            *reinterpret_cast<C2<T> *>(out + (long long)z * plane + (long long)i * row + ncols) = mk<T>(0, 0);
    }
    // The loads above sit between stores to the same array, so they cannot be hoisted:
    // without this each would wait for HBM at store time.
    __device__ __forceinline__ void prefetch(int z, int i, int line) const
    {
        const long long o = (long long)z * plane + (long long)i * row + 2 * line;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(out + o));
        if (z >= zlo && z <= zhi) {
            asm volatile("prefetch.global.L2 [%0];" ::"l"(tz + o + (fwd ? plane : 0)));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(tz + o - (fwd ? 0 : plane)));
        }
    }
};

// ddy of the real columns of a (ldx, nyt, nlev) field with the DivEpi store hook
template <typename T>
cudaError_t launch_cols_divt(int n, const ColArgs<T> &a, const DivEpi<T> &e, cudaStream_t s);
// p[0..n) = v
template <typename T> void launch_fill(T *p, long long n, T v, cudaStream_t s, cudaError_t &e);

} // namespace obl
