// press.cuh -- batched tridiagonal pressure solve and the streaming (elementwise)
// kernels of the hot path.
#pragma once
#include "fft.cuh"

namespace obl {

template <typename T> struct TdmaArgs {
    const C2<T> *Hx, *Hy, *Hz;  // spectral planes (lhx, nyt) of levels 0..nz (Hx,Hy use 1..L)
    C2<T> *phat;                // out: levels 0..L
    C2<T> *dph;                 // optional out: (p_hat(z) - p_hat(z-1))/dz at levels 1..L,
                                // formed in the solve's precision (the spectrum of dpdz)
    T *cscr;                    // bulk scratch: modified upper band c'(1..L), (S, L)
    const double *kx;           // kx(lhx), Nyquist entry 0       (002_fft.f90:131-137)
    const double *ky;           // ky_2d row (nyt), Nyquist row 0 (002_fft.f90:147,161-165)
    const unsigned char *skip;  // optional: 1 = column solved by the FP64 island kernel
    long long S;                // lhx * nyt
    int lhx, nyt, L;
    double dz;
    int neumann_top;            // OBL_TOP_NEUMANN
};

// FP64 island work list
struct IslandArgs {
    const int *cols;   // column indices q = kx + lhx*ky
    int n;
    double *cscr;      // (n, L)
    double2 *dscr;     // (n, L+1)
};

template <typename T> void launch_tdma(const TdmaArgs<T> &a, cudaStream_t s, cudaError_t &e);
template <typename T> void launch_tdma_island(const TdmaArgs<T> &a, const IslandArgs &isl,
                                              cudaStream_t s, cudaError_t &e);

// streaming kernels on (ldx, nyt, levels) fields
template <typename T> void launch_ddz_uv(T *dfdz, const T *fun, int nxt, int ldx, int nyt, int nz,
                                         double dz, cudaStream_t s, cudaError_t &e);
template <typename T> void launch_ddz_w(T *dfdz, const T *fun, int nxt, int ldx, int nyt, int nz,
                                        double dz, cudaStream_t s, cudaError_t &e);
template <typename T> void launch_dpdz(T *dpdz, const T *p, int nxt, int ldx, int nyt, int nz,
                                       double dz, cudaStream_t s, cudaError_t &e);
// only the boundary part of project (110_project.f90:50-60), after an interior update
template <typename T> void launch_project_bc(T *u, T *v, T *w, int ldx, int nyt, int nz, int stress_free,
                                             cudaStream_t s, cudaError_t &e);
template <typename T> void launch_project(T *u, T *v, T *w, const T *dpdx, const T *dpdy,
                                          const T *dpdz, int nxt, int ldx, int nyt, int nz,
                                          double dt, int stress_free, cudaStream_t s,
                                          cudaError_t &e);
void launch_convert_d2f(float *dst, const double *src, long long n, cudaStream_t s, cudaError_t &e);
void launch_convert_f2d(double *dst, const float *src, long long n, cudaStream_t s, cudaError_t &e);

} // namespace obl
