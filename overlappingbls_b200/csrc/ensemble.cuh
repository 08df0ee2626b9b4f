// ensemble.cuh -- one persistent launch that advances many independent instances (of
// different sizes) through the projection-plus-derivative step.
//
// The step of one instance is six dependent phases (the kernels of the line path of
// obl_step): (0) the multi-output row pass of u, v, w, theta; (1) the column passes
// (y-pad, ddy, y-transform of the RHS spectra, zeroed boundary planes); (2) the
// tridiagonal solves; (3) the y-inverse of p_hat and the dpdz spectrum; (4) the
// x-inverse fused with project(); (5) project()'s boundary rows.  The ensemble kernel
// runs phase k of every instance, then a grid barrier, then phase k+1: each phase is a
// work list of CTA-sized units over all instances, split into contiguous chunks per CTA,
// and every unit dispatches at run time on its instance's line lengths to the same
// device functions the single-instance kernels use.
#pragma once
#include <string>

#include "fused.cuh"
#include "press.cuh"

namespace obl {

constexpr int kEnsPhases = 6;

template <typename T> struct EnsInst {
    int nx, ny, nlev, L;
    // phase 0
    RowsFwd3Args<T> rows[4];
    long long rows_units;            // units per field
    // phase 1
    ColArgs<T> padc[4], ddyc[4], fwdc[3];
    int pad_nb, ddy_nb, fwd_nb;      // line groups per plane
    C2<T> *Hz;                       // H_z planes 0 and L+1 are zeroed (divtz = 0)
    long long S;
    // phase 2
    TdmaArgs<T> tdma;
    IslandArgs isl;
    long long isl_units, bulk_units; // units of 256 columns
    // phase 3
    PinvColArgs<T> pc;
    int pc_nb;
    // phase 4
    PinvRowArgs<T> pr;
    long long pr_units;
    // phase 5
    T *u, *v, *w;
    int ldx, nz, stress_free;
    long long count[kEnsPhases];     // units of this instance per phase
};

template <typename T> struct EnsArgs {
    const EnsInst<T> *inst;
    int ninst;
    const long long *start;          // (kEnsPhases, ninst+1) prefix sums of the unit counts
    unsigned *bar;                   // [0] arrivals, [1] generation
    int *err;                        // 1: a barrier wait gave up
    unsigned long long *stamps;      // optional: global-timer ns at the start and after each phase
    // dataflow form: [0] the work counter, [1 + k*kEnsPhases + ph] units of instance k's
    // phase ph completed (zeroed before each launch)
    unsigned *flow;
};

// host-side geometry of the instance kernels (per line length n; 0 if unsupported)
bool ens_length_supported(int n);
// The persistent kernel's grid barrier run by one CTA: OBL_OK when it releases,
// OBL_ERR_TIMEOUT when (never_released) its bounded wait gives up.
int ens_barrier_selftest(bool never_released, cudaStream_t s, std::string &err);
template <typename T> struct EnsGeoHost {
    static long long rows_units(int n, long long npairs);      // units of the row pass
    static long long pinv_rows_units(int n, long long npairs); // units of the x-inverse
    // dynamic shared memory of the units of phases [pb, pe)
    static size_t smem(int nx, int ny, int pb, int pe);
};
template <typename T> int ens_wb();   // lines per CTA of the line-minor column units

// The kernel over phases [PB, PE) with MINB CTAs per SM.  Instantiated: <0,6,2> (the whole
// step in one launch) and the register-class split <0,1,2> (rows), <1,4,4> (columns, solve,
// y-inverse), <4,6,2> (x-inverse + project).
#ifndef OBL_ENS_MINB
#define OBL_ENS_MINB 4   // CTAs per SM the one-launch persistent kernel's registers are bounded for
#endif
template <typename T, int PB, int PE, int MINB> struct EnsKernel {
    static cudaError_t attr(size_t smem);
    static int blocks_per_sm(size_t smem);            // CTAs of the kernel resident per SM
    static cudaError_t launch(const EnsArgs<T> &a, int blocks, size_t smem, cudaStream_t s);   // cooperative
};

// The dataflow form of the one-launch persistent kernel (OBL_ENS_PERSISTENT_FLOW): no grid
// barriers.  CTAs take units one at a time from a work counter over the whole step's
// work list (phase-major, instances in order within a phase); a unit of phase ph of
// instance k first waits until all of that instance's phase ph-1 units have completed
// (bounded, like the barrier), so instances overlap at phase boundaries instead of the
// whole grid waiting for the slowest unit of each phase.
template <typename T, int MINB> struct EnsFlowKernel {
    static cudaError_t attr(size_t smem);
    static int blocks_per_sm(size_t smem);
    static cudaError_t launch(const EnsArgs<T> &a, int blocks, size_t smem, cudaStream_t s);   // cooperative
};

} // namespace obl
