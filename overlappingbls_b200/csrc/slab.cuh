// slab.cuh -- the pressure solve of one z-slab of a domain split over P ranks.
//
// The reference splits z over npz ranks and pipelines the Thomas sweeps rank after rank
// with send/recv per y-row (109_press_stag_array.f90:244-319).  Here every rank solves its
// own rows of each (kx,ky) column at once (partitioned Thomas):
//   solve:   T_loc y = r,  T_loc v = a_s e_1,  T_loc w = c_e e_m, where T_loc is the rank's
//            block of the column's tridiagonal matrix without the two couplings a_s (to
//            the last unknown of the rank below) and c_e (to the first of the rank above),
//            so that x = y - v x_below - w x_above.  The forward elimination keeps the
//            eliminated rows (c'_j, y'_j, v'_j; w' is zero above the last row); a back
//            recurrence in registers gives the end values of y, v, w: the rank's interface
//            coefficients (y_1, y_m complex; v_1, v_m, w_1, w_m real);
//   (all ranks exchange their interface coefficients)
//   finish:  the 2P interface unknowns (first and last of every rank) solve a 2x2-block
//            tridiagonal system, redundantly on every rank; then the back substitution
//            x_j = y'_j - v'_j x_below - c'_j x_{j+1} (x_{m+1} = x_above, the last row with
//            w'_m) on the rank's rows, p_hat(0) and the spectral dpdz.
// The block systems are diagonally dominant, so the split needs no pivoting.  The rank's
// elimination runs in the storage precision for the bulk columns and in FP64 for the
// island columns of the mixed mode (as the single-domain solve does); the interface values
// and the reduced system are FP64 in every mode.
#pragma once
#include "fft.cuh"

namespace obl {

constexpr int kSlabMaxRanks = 16;
constexpr int kSlabIface = 8;   // y1.re, y1.im, ym.re, ym.im, v1, vm, w1, wm per column

template <typename T> struct SlabArgs {
    const C2<T> *Hx, *Hy, *Hz;  // local spectra: Hx, Hy levels 1..L, Hz levels 0..L+1
                                // (Hz(L+1): the first plane of the rank above, or the top plane)
    C2<T> *phat, *dph;          // out (finish): p_hat levels 0..L, spectral dpdz levels 1..L;
                                // between the kernels phat levels 1..L hold y'
    T *v, *cp;                  // bulk scratch (S, L) in the storage type: v', c'
    const int *isl_cols;        // mixed mode: the FP64 columns (k^2 small), solved in FP64 with
    const int *isl_slot;        // their own scratch (n_isl, L); isl_slot[q] = island index or -1
    int n_isl;
    double2 *iy;
    double *iv, *icp;
    double *iface;              // out (solve): (kSlabIface, S), field-major
    const double *iface_all;    // in (finish): (P, kSlabIface, S)
    const double *kx, *ky;      // kx(lhx), ky_2d row (nyt), Nyquist entries 0
    long long S;
    int lhx, nyt, L;
    double dz;
    int rank, nranks;
    int own_p0;                 // finish writes p_hat level 0 (off for the upper segments of
                                // a column split on one GPU, whose level 0 is the segment below's)
};

// The same solve on one GPU with each column split into P segments of seg levels (the last
// one shorter), solved at once: a = the whole column's arguments (L = all levels, rank 0 of
// 1), scratch (S, L) and (n_isl, L), iface (P, S, kSlabIface).  For grids with too few
// (kx,ky) columns to fill the GPU with one sequential sweep each.
template <typename T> void launch_seg_solve(const SlabArgs<T> &a, int P, int seg, cudaStream_t s, cudaError_t &e);
template <typename T> void launch_seg_finish(const SlabArgs<T> &a, int P, int seg, cudaStream_t s, cudaError_t &e);
// the same two launches over the FP64 island columns alone (the mixed mode's whole-column
// FP32 solves then leave them out): each island column's FP64 chain is split into P
// segments instead of one thread sweeping all L levels
template <typename T> void launch_seg_solve_isl(const SlabArgs<T> &a, int P, int seg, cudaStream_t s, cudaError_t &e);
template <typename T> void launch_seg_finish_isl(const SlabArgs<T> &a, int P, int seg, cudaStream_t s, cudaError_t &e);

template <typename T> void launch_slab_solve(const SlabArgs<T> &a, cudaStream_t s, cudaError_t &e);
template <typename T> void launch_slab_finish(const SlabArgs<T> &a, cudaStream_t s, cudaError_t &e);

// project()'s boundary rows by rank role: bottom rank w(1) = 0, top rank w(nz) = 0 and
// the stress-free copy (110_project.f90:50-60)
template <typename T>
void launch_project_bc_roles(T *u, T *v, T *w, int ldx, int nyt, int nz, int stress_free, int bottom, int top,
                             cudaStream_t s, cudaError_t &e);

} // namespace obl
