// convec.cuh -- streaming kernels of the rotational convective term (108_convec.f90) and
// of its transpose, used by the rollout step u1 = P(u - dt*tadv1*convec(u)) and its
// vector-Jacobian product.
//
// Fields: small (ldx, nyt, 0:nz), padded (nxt2, nyt2, 0:nz).  Single z-rank (coordz ==
// 0 == npz-1), Stokes drift off.  dudz, dvdz at level 1 are taken equal to level 2 and
// are 0 at level nz (stress-free top, 104_wallstress.f90:249-253).
#pragma once
#include <cuda_runtime.h>

namespace obl {

// the six padded fields of convec: u, v, w, vort1, vort2, vort3 (108_convec.f90:38-76)
template <typename T> struct BigSet {
    const T *U, *V, *W, *O1, *O2, *O3;
};

// vorticity (108_convec.f90:43-68) from ddx/ddy of u, v, w and the level differences of
// u, v; o1, o2, o3 receive levels 1..nz (0 elsewhere and in the pad columns)
template <typename T>
void launch_vort(const T *u, const T *v, const T *dudy, const T *dvdx, const T *dwdx, const T *dwdy,
                 T *o1, T *o2, T *o3, int nxt, int ldx, int nyt, int nz, double dz, cudaStream_t s,
                 cudaError_t &e);

// cross_product (108_convec.f90:108-202) on the padded grid: X, Y, Z at levels 1..nz-1,
// 0 at levels 0 and nz
template <typename T>
void launch_cross(const BigSet<T> &b, T *X, T *Y, T *Z, int nx2, int ny2, int nz, cudaStream_t s,
                  cudaError_t &e);

// u,v,w(1..nz-1) -= f * (cx, cy, cz)   (x < nxt)
template <typename T>
void launch_update(T *u, T *v, T *w, const T *cx, const T *cy, const T *cz, double f, int nxt, int ldx,
                   int nyt, int nz, cudaStream_t s, cudaError_t &e);

// transpose of project()'s boundary assignments: the stress-free copy u,v(nz-1) =
// u,v(nz-2) (when stress_free) and w(1) = w(nz) = 0
template <typename T>
void launch_adj_project_bc(T *lu, T *lv, T *lw, int ldx, int nyt, int nz, int stress_free, cudaStream_t s,
                           cudaError_t &e);

// lw(1) = c * p(1) for x < nxt (the level-1 w row of the transposed projection)
template <typename T>
void launch_adj_w1(T *lw, const T *p, double c, int nxt, int ldx, int nyt, cudaStream_t s, cudaError_t &e);

// transpose of cross_product: given the padded adjoints LX, LY, LZ of X, Y, Z (scaled by
// f), the adjoints of the six padded fields
template <typename T> struct CrossAdjOut {
    T *U, *V, *W, *O1, *O2, *O3;
};
template <typename T>
void launch_cross_adj(const BigSet<T> &b, const T *LX, const T *LY, const T *LZ, double f,
                      const CrossAdjOut<T> &out, int nx2, int ny2, int nz, cudaStream_t s, cudaError_t &e);

// q1, q2: the adjoints of dwdy, dwdx (up to sign) from the unpadded vorticity adjoints
// s1, s2 (the 0.5 averages of vort1(nz), vort2(nz) included)
template <typename T>
void launch_adj_q(const T *s1, const T *s2, T *q1, T *q2, int nxt, int ldx, int nyt, int nz, cudaStream_t s,
                  cudaError_t &e);

// final accumulation of the convec transpose into lu, lv, lw (x < nxt, all levels):
//   lu += sU + t1 + dz^T(s2),  lv += sV - t2 - dz^T(s1),  lw += sW + t3 - t4
template <typename T> struct AdjCombineArgs {
    T *lu, *lv, *lw;
    const T *sU, *sV, *sW, *s1, *s2, *t1, *t2, *t3, *t4;
};
template <typename T>
void launch_adj_combine(const AdjCombineArgs<T> &a, int nxt, int ldx, int nyt, int nz, double dz,
                        cudaStream_t s, cudaError_t &e);

// J = sum over x < nxt and levels klo..khi of 0.5*(u^2 + v^2 + (0.5*(w(k)+w(k+1)))^2),
// accumulated in FP64 in a fixed order (deterministic); when lu is not null, lu, lv, lw
// receive dJ/d(u, v, w).  part holds ke_parts() doubles, out one double (device).
int ke_parts();
template <typename T>
void launch_ke_band(const T *u, const T *v, const T *w, T *lu, T *lv, T *lw, double *part, double *out,
                    int nxt, int ldx, int nyt, int nz, int klo, int khi, cudaStream_t s, cudaError_t &e);

} // namespace obl
