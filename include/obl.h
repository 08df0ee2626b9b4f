/*
 * obl.h -- C ABI of the B200-native OverlappingBLs hot path (libobl_b200.so).
 *
 * This is the drop-in boundary for the reference's derivative and pressure-solver
 * routines.  Each entry point names the Fortran routine it replaces (paths relative
 * to the reference project; SBL/code is canonical, BBL/SBBL carry identical copies).
 * A Fortran caller binds these through ISO_C_BINDING (overlappingbls_b200/fortran/
 * obl_gpu.f90) and keeps the reference call signatures.
 *
 * Conventions
 *   - Every function returns an int status (OBL_OK = 0); obl_last_error() gives text.
 *   - Arrays use the reference's Fortran layout (column-major, x fastest):
 *       physical field   f(ldx, nyt, 0:nz)        ldx = 2*(nxt/2+1), nz = nzt
 *       level-1-based    dpdx/dpdy/dpdz(ldx, nyt, 1:nz)   (slot jz-1 holds level jz)
 *       padded field     b(nxt2, nyt2, 0:nz)      nxt2 = 3*nxt/2
 *       spectral plane   c(lhx, nyt) complex      lhx = nxt/2+1 (interleaved re,im)
 *     One GPU holds the whole domain (npy = 1 and the z-slabs of all ranks).
 *   - Host variants take double* host arrays (Fortran real(8)); the library stages
 *     them through device buffers it owns.  Only the elements the reference routine
 *     writes are written back (e.g. x < nxt of each row), so pad columns and levels
 *     the reference leaves alone keep their host values.
 *   - *_dev variants take device pointers in the context's storage type: double for
 *     OBL_PREC_F64, float for OBL_PREC_MIXED / OBL_PREC_F32.  They are asynchronous
 *     on the context's stream.
 *   - A context is bound to one device and one stream and is not reentrant: use one
 *     context per host thread (the reference is single-threaded per MPI rank).
 */
#ifndef OBL_H
#define OBL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define OBL_OK 0
#define OBL_ERR_ARG 1         /* bad argument or shape                         */
#define OBL_ERR_CUDA 2        /* CUDA runtime error                            */
#define OBL_ERR_NOMEM 3       /* device or pinned-host allocation failed       */
#define OBL_ERR_TIMEOUT 4     /* a bounded device-side wait expired            */
#define OBL_ERR_UNSUPPORTED 5 /* grid size without a compiled FFT plan         */
#define OBL_ERR_NODEV 6       /* no CUDA device                                */
#define OBL_ERR_IO 7          /* file open, read or write failed; short file    */

/* ---- precision modes ---- */
#define OBL_PREC_F64 0   /* every kernel in FP64 (the plain FP64 GPU form)             */
#define OBL_PREC_MIXED 1 /* FP32 FFTs/dealiasing/TDMA, FP64 TDMA for (0,0) and low |k| */
#define OBL_PREC_F32 2   /* FP32 everywhere (diagnostic)                                */

/* ---- top boundary of the pressure solve (109_press_stag_array.f90:20-50,280-297) ---- */
#define OBL_TOP_SINGLE_RANK 0 /* npz = 1 semantics: p_hat(nz-1) forced to 0 (Dirichlet) */
#define OBL_TOP_NEUMANN 1     /* npz >= 2 semantics: Neumann top row, divtz top plane   */

typedef struct obl_ctx obl_ctx;

/* Grid and run constants, dimensional as in the namelist (&domain_param, &time_param,
   &flow_param); non-dimensionalised exactly as init_parameter/init_nondimensional do
   (102_initial.f90:119-141,186-199). */
typedef struct obl_grid {
    int nxt, nyt, nzt;
    double lx_tot, ly_tot, lz_tot, z_i, dt, u_scale;
} obl_grid;

typedef struct obl_options {
    int precision;        /* OBL_PREC_*                                          */
    int top_bc;           /* OBL_TOP_*                                           */
    int ubc_stress_free;  /* project(): ubc_mom == 'stress free' (110_project.f90:51) */
    double fp64_k2_max;   /* MIXED: columns with k^2 <= this are solved in FP64;
                             a negative value selects the built-in default       */
    int device;           /* CUDA device ordinal                                  */
} obl_options;

typedef struct obl_info {
    int nxt, nyt, nzt, nz, ldx, lhx, nxt2, nyt2;
    int elem_bytes;              /* storage bytes per real (8 or 4)               */
    int n_fp64_columns;          /* MIXED: (kx,ky) columns solved in FP64         */
    double dz, dt_nd, lx, ly;    /* non-dimensional                               */
    long long field_elems;       /* ldx*nyt*(nz+1)                                */
    long long dfield_elems;      /* ldx*nyt*nz                                    */
    long long big_elems;         /* nxt2*nyt2*(nz+1)                              */
    long long spec_elems;        /* lhx*nyt complex per plane                     */
} obl_info;

/* ---- context: replaces init_parameter, init_fft_plan, init_wavenumber and
        init_coef_press + tdmaMcoef_pipelined (102_initial.f90:20-53,
        002_fft.f90:78-189, 109_press_stag_array.f90:4-103) ---- */
int obl_ctx_create(const obl_grid *grid, const obl_options *opt, obl_ctx **out);
int obl_ctx_destroy(obl_ctx *ctx);
int obl_ctx_info(const obl_ctx *ctx, obl_info *info);
int obl_set_stream(obl_ctx *ctx, void *cuda_stream);  /* cudaStream_t; NULL = legacy */
int obl_synchronize(obl_ctx *ctx);
int obl_last_error(const obl_ctx *ctx, char *buf, size_t n);
/* kernels launched by this context so far */
long long obl_launch_count(const obl_ctx *ctx);
/* per-kernel CUDA-event timing: enable, then read a JSON object
   {"kernel": [launches, total_ms], ...} (synchronizes; clears the records) */
int obl_timing_enable(obl_ctx *ctx, int on);
int obl_timing_report(obl_ctx *ctx, char *buf, size_t n);
/* execution tuning (results do not depend on it beyond rounding):
     "fused"             1 = cluster-fused plane kernels in obl_step (square grids), 0 = line kernels
     "fwd_clusters"      clusters of the fused forward kernel (0 = as many as can be resident)
     "fwd_cluster_size"  CTAs per cluster (1..16; above 8 needs non-portable cluster support)
     "tdma_segments"     segments each (kx,ky) column of the pressure solve is split into
                         and solved at once (0 = chosen by size: more than one only when
                         the columns alone cannot fill the GPU; 1 = one sequential sweep;
                         up to 16; used in the Neumann-top mode with spectral dpdz)
     "tdma_reg"          FP32 storage: 1 = the register-segmented whole-column solve
                         (default), 0 = one sequential sweep per column
     "tdma_stage"        with "tdma_reg": 1 = its persistent form fed by bulk asynchronous
                         copies (needs lhx*nyt even and 16-byte aligned spectra, else the
                         load-fed form runs), 0 = the load-fed form, 2 = the copy-fed form
                         above 128 levels, where it measured faster (default)
     "isl_segments"      mixed mode, whole-column solves of the Neumann-top step: the FP64
                         island columns split into this many segments by the
                         column-segmented FP64 solve (0 = 16, capped at L/8; 1 = each island
                         column swept by one thread inside the FP32 bulk launch)
     "isl_concurrent"    1 = those island launches on a side stream beside the bulk launch
                         (default 0: measured slower)
     "gform"             the pressure RHS in G form: 1 = with FP64 storage (default),
                         2 = always, 0 = never
     "pad_tma"           FP32 y-pad (zero_padding, the step): 1 = each CTA's input tile by
                         tensor-map copies (default), 0 = by loads
     "fwd_chunk"         the step's forward pass over chunks of this many levels (0 = all)
     "out_streams"       copy streams of the host-array step's outputs (1 or 2; default 2)
     "fail_alloc"        n > 0: the n-th device allocation from now fails (tests)
     "stage_timeout_test" 1: the staged solve's waits expect bytes no copy delivers, so
                         that they give up and OBL_ERR_TIMEOUT is reported (tests) */
int obl_set_param(obl_ctx *ctx, const char *name, long long value);
int obl_get_param(obl_ctx *ctx, const char *name, long long *value);

/* ---- spectral derivatives: ddx / ddy (004_derivatives.f90:18-41, 45-81) ----
   fields (ldx, nyt, nlev) (the reference passes nlev = nz+1); x < nxt written. */
int obl_ddx(obl_ctx *ctx, double *dfdx, const double *fun, int nlev);
int obl_ddy(obl_ctx *ctx, double *dfdy, const double *fun, int nlev);
int obl_ddx_dev(obl_ctx *ctx, void *dfdx, const void *fun, int nlev);
int obl_ddy_dev(obl_ctx *ctx, void *dfdy, const void *fun, int nlev);

/* ---- vertical differences: ddz_uv / ddz_w (004_derivatives.f90:85-116, 155-183) ----
   single-rank branches: ddz_uv writes levels 0 (BOGUS) and 2..nz-1;
   ddz_w writes levels 0 (BOGUS), 1..nz-1 and nz (= 0). */
int obl_ddz_uv(obl_ctx *ctx, double *dfdz, const double *fun);
int obl_ddz_w(obl_ctx *ctx, double *dfdz, const double *fun);
int obl_ddz_uv_dev(obl_ctx *ctx, void *dfdz, const void *fun);
int obl_ddz_w_dev(obl_ctx *ctx, void *dfdz, const void *fun);

/* ---- stress divergence: divstress_uv / divstress_w (107_divstress.f90:4-44, 48-104) ----
   tx, ty, tz, divt (ldx,nyt,0:nz); single-rank roles (the domain holds the wall and the
   top).  divstress_uv: divt = ddx(tx) + ddy(ty) + ddz_w(tz) on levels 1..nz-1, BOGUS
   on levels 0 and nz.  divstress_w: divt = ddx(tx) + ddy(ty) on level 1 and nz, plus
   ddz_uv(tz) on levels 2..nz-1, BOGUS on level 0.  The x pads (nxt, nxt+1) of the
   computed levels are 0.  divt must not alias an input. */
int obl_divstress_uv(obl_ctx *ctx, double *divt, const double *tx, const double *ty, const double *tz);
int obl_divstress_w(obl_ctx *ctx, double *divt, const double *tx, const double *ty, const double *tz);
int obl_divstress_uv_dev(obl_ctx *ctx, void *divt, const void *tx, const void *ty, const void *tz);
int obl_divstress_w_dev(obl_ctx *ctx, void *divt, const void *tx, const void *ty, const void *tz);
/* The same on z-rank `rank` of `nranks` (coordz, npz), levels 0..nz of the rank with the
   ghost levels 0 and nz filled by the caller's exchange (103_flosol.f90:62-76): divstress_w
   adds ddz_uv(tz) on level 1 except on rank 0, computes level nz (without it) only on the
   top rank and leaves it BOGUS elsewhere (107_divstress.f90:81-102); divstress_uv does
   not depend on the rank. */
int obl_divstress_uv_slab_dev(obl_ctx *ctx, void *divt, const void *tx, const void *ty, const void *tz, int rank,
                              int nranks);
int obl_divstress_w_slab_dev(obl_ctx *ctx, void *divt, const void *tx, const void *ty, const void *tz, int rank,
                             int nranks);

/* ---- restart files: write_file_mpi_3d / read_file_mpi_3d (202_parallel.f90:1084-1120,
   1211-1250), checkpoint_final (012_io.f90:496-546), read_flow_field
   (102_01_ic.f90:682-734), total_time.dat (012_io.f90:485-490, 102_01_ic.f90:697-705) ----
   A field in a file is the global FP64 array (nxt, nyt, nzranks*(nz-1)) in Fortran order
   at byte offset disp0: levels 1..nz-1 of every z-rank, rank zrank's block at z offset
   zrank*(nz-1) (MPI subarray start (0, 0, (nz-1)*coordz) with npy = 1).  var is a device
   field (ldx,nyt,0:nz) in the storage type; FP32 storage widens exactly on write and
   rounds on read.  Reading leaves the pads and levels 0 and nz untouched.  Files are
   created when missing and not truncated.  A missing or short input file gives
   OBL_ERR_IO.
   vel_tt: the OBL_VEL_TT_FIELDS fields u, v, w, RHSx, RHSy, RHSz, Cs_opt2, F_LM, F_MM,
   F_QN, F_NN, one after the other, in the file path_restart + "vel_tt%08d.out" (the path
   keeps its own trailing '/'); a NULL field is written as zeros and skipped on reading.
   checkpoint_final creates the directory path_restart when it is missing.
   total_time.dat holds the step number nums as one list-directed integer; reading a
   missing file gives nums = 0 and OBL_OK, as the reference starts from step 0. */
#define OBL_VEL_TT_FIELDS 11
int obl_write_file_3d_dev(obl_ctx *ctx, const void *var, const char *fn, long long disp0, int zrank, int nzranks);
int obl_read_file_3d_dev(obl_ctx *ctx, void *var, const char *fn, long long disp0, int zrank, int nzranks);
int obl_checkpoint_final_dev(obl_ctx *ctx, const char *path_restart, int nums, const void *const *fields, int zrank,
                             int nzranks);
int obl_read_flow_field_dev(obl_ctx *ctx, const char *path_restart, int nums, void *const *fields, int zrank,
                            int nzranks);
int obl_read_total_time(const char *fn, int *nums);
int obl_write_total_time(const char *fn, int nums);

/* ---- 2D transforms fftn_mpi / ifftn_mpi (203_fftn_mpi.f90:4-35, 39-67) ----
   in (ldx, nyt, nlev) real -> out (lhx, nyt, nlev) complex, unnormalised, x- and
   y-Nyquist zeroed; ifftn: complex -> real, x < nxt written. */
int obl_fftn(obl_ctx *ctx, const double *in, double *out_cplx, int nlev);
int obl_ifftn(obl_ctx *ctx, const double *in_cplx, double *out, int nlev);
int obl_fftn_dev(obl_ctx *ctx, const void *in, void *out_cplx, int nlev);
int obl_ifftn_dev(obl_ctx *ctx, const void *in_cplx, void *out, int nlev);

/* ---- 3/2-rule dealiasing zero_padding / zero_unpadding (108_01_padd.f90:73-197) ----
   var (ldx, nyt, nlev) <-> var_big (nxt2, nyt2, nlev). */
int obl_zero_padding(obl_ctx *ctx, const double *var, double *var_big, int nlev);
int obl_zero_unpadding(obl_ctx *ctx, const double *var_big, double *var, int nlev);
int obl_zero_padding_dev(obl_ctx *ctx, const void *var, void *var_big, int nlev);
int obl_zero_unpadding_dev(obl_ctx *ctx, const void *var_big, void *var, int nlev);

/* ---- zero_padding that allocates nothing (no counterpart in the reference) ----
   For callers that cannot allocate device memory when they call: an application that
   hands all device memory to its own pool at start-up and forbids allocation afterwards
   (a time loop that sized its fields once), or code on a latency-critical path where
   cudaMalloc may block and cudaFree waits for the whole device.  Same arguments and
   result as obl_zero_padding_dev, but the intermediate x-padded plane lives in a static
   device array of OBL_NOALLOC_SCRATCH_BYTES that every GPU loading this library holds
   until the process exits; the call itself performs no cudaMalloc/cudaFree.
   - Sizes: es * nxt2 * nyt * nlev must fit in OBL_NOALLOC_SCRATCH_BYTES (es = 8 for
     OBL_PREC_F64, 4 otherwise); larger requests return OBL_ERR_ARG with an explanation
     in obl_last_error (pass fewer levels per call).
   - The first call on a device looks up the array's device address
     (cudaGetSymbolAddress) with that device current and keeps it for the process; make
     that first call before any stream capture.  A cudaDeviceReset of that device
     invalidates the kept address (and every context on the device): do not call this
     entry point again after one.
   - All calls share the one array: calls that overlap on the GPU (different streams or
     contexts without ordering) race on it, so serialise them on one stream.  Every
     element of the scratch is rewritten before it is read, so nothing needs clearing
     between calls.
   - The caller's current device is restored on return. */
#define OBL_NOALLOC_SCRATCH_BYTES (8u << 20)
int obl_zero_padding_noalloc_dev(obl_ctx *ctx, const void *var, void *var_big, int nlev);

/* ---- filter_data (006_test_filter.f90:82-105): in place on (ldx, nyt, nlev) ---- */
int obl_filter_data(obl_ctx *ctx, double *f, int nlev);
int obl_filter_data_dev(obl_ctx *ctx, void *f, int nlev);

/* ---- press_stag_array + tdmaSolver_pipelined (109_press_stag_array.f90:107-319) ----
   u,v,w (ldx,nyt,0:nz) in; divtz_bot = divtz(:,:,1), divtz_top = divtz(:,:,nz)
   planes (ldx,nyt) or NULL for zero (the theta/lbc==0 surface term of :187-192 is
   folded into divtz_bot by the caller); p (ldx,nyt,0:nz) levels 0..nz-1 written;
   dpdx, dpdy (ldx,nyt,1:nz) levels 1..nz-1 written. */
int obl_press_stag_array(obl_ctx *ctx, const double *u, const double *v, const double *w,
                         const double *divtz_bot, const double *divtz_top,
                         double *p, double *dpdx, double *dpdy);
int obl_press_stag_array_dev(obl_ctx *ctx, const void *u, const void *v, const void *w,
                             const void *divtz_bot, const void *divtz_top,
                             void *p, void *dpdx, void *dpdy);

/* ---- flosol glue (103_flosol.f90:174-175): dpdz(jz)=(p(jz)-p(jz-1))/dz, 1..nz-1 ---- */
int obl_dpdz(obl_ctx *ctx, const double *p, double *dpdz);
int obl_dpdz_dev(obl_ctx *ctx, const void *p, void *dpdz);

/* ---- project (110_project.f90:4-62): u,v,w updated in place ---- */
int obl_project(obl_ctx *ctx, double *u, double *v, double *w,
                const double *dpdx, const double *dpdy, const double *dpdz);
int obl_project_dev(obl_ctx *ctx, void *u, void *v, void *w,
                    const void *dpdx, const void *dpdy, const void *dpdz);

/* ---- fused projection-plus-derivative step ----
   The hot-path slice of one flosol time step on u,v,w,theta: ddx/ddy of
   u,v,w,theta and zero_padding of u,v,w,theta on levels 0..nz (103_flosol.f90:30-35,
   108_convec.f90:38-42, 010_scalars.f90:137-138,429-431), press_stag_array(u,v,w),
   dpdz and project (103_flosol.f90:168-188).  Pointers are host (obl_step /
   obl_step_f32) or device (obl_step_dev, storage type). */
typedef struct obl_step_io {
    void *u, *v, *w;          /* in/out (ldx,nyt,0:nz), projected in place         */
    const void *theta;        /* in (ldx,nyt,0:nz)                                  */
    void *d[8];               /* out dudx,dudy,dvdx,dvdy,dwdx,dwdy,dtdx,dtdy         */
    void *big[4];             /* out u,v,w,theta on the 3/2 grid (nxt2,nyt2,0:nz)    */
    void *p;                  /* out (ldx,nyt,0:nz)                                 */
    void *dp[3];              /* out dpdx,dpdy,dpdz (ldx,nyt,1:nz)                  */
    const void *divtz_bot;    /* optional plane (ldx,nyt), NULL = 0                 */
    const void *divtz_top;    /* optional plane (ldx,nyt), NULL = 0                 */
} obl_step_io;

int obl_step(obl_ctx *ctx, const obl_step_io *io);      /* host double*   */
int obl_step_f32(obl_ctx *ctx, const obl_step_io *io);  /* host float*    */
int obl_step_dev(obl_ctx *ctx, const obl_step_io *io);  /* device, storage type */

/* ---- convec: the rotational convective term (108_convec.f90:11-202) ----
   The padded-grid consumer of zero_padding / zero_unpadding: ddx/ddy and the level
   differences of u,v,w, the vorticity, zero_padding of u,v,w and the vorticity,
   cross_product on the 3/2 grid and zero_unpadding (single z-rank, no Stokes drift).
   The wall-model dudz, dvdz at level 1 (wallstress_bottom, 104_wallstress.f90) are
   taken equal to level 2; at level nz they are 0 (stress-free top, :249-253).
   cx, cy, cz (ldx,nyt,0:nz): levels 1..nz-1 written.  Needs nzt >= 5. */
int obl_convec(obl_ctx *ctx, const double *u, const double *v, const double *w,
               double *cx, double *cy, double *cz);
int obl_convec_dev(obl_ctx *ctx, const void *u, const void *v, const void *w,
                   void *cx, void *cy, void *cz);

/* ---- rollout step and its transpose (the adjoint) ----
   step: u1 = P(u - dt*tadv1*convec(u)) on u,v,w (ldx,nyt,0:nz) in place, where P is
   press_stag_array with divtz = 0, dpdz and project(): the explicit-Euler form of the
   Adams-Bashforth update (103_flosol.f90:115,319-389) followed by the projection
   (:168-188).  No counterpart entry point in the reference, which has no adjoint.
   step_vjp: lu,lv,lw <- (d step / d state)^T (lu,lv,lw) at the state u,v,w; the
   transposed pressure solve is the same solve (symmetric bands), the transposed 3/2
   rule is the opposite transform, the convec fields are recomputed from the state.
   Only the Neumann-top mode (OBL_TOP_NEUMANN); OBL_ERR_UNSUPPORTED otherwise. */
int obl_rollout_step(obl_ctx *ctx, double *u, double *v, double *w);
int obl_rollout_step_dev(obl_ctx *ctx, void *u, void *v, void *w);
int obl_rollout_step_vjp(obl_ctx *ctx, const double *u, const double *v, const double *w,
                         double *lu, double *lv, double *lw);
int obl_rollout_step_vjp_dev(obl_ctx *ctx, const void *u, const void *v, const void *w,
                             void *lu, void *lv, void *lw);

/* ---- kinetic-energy objective (energy, 103_flosol.f90) ----
   *J = sum over x < nxt, all y and the levels jz = 1..nz-1 whose uvp height
   (jz-0.5)*dz*z_i (012_io.f90:295, in the units of lz_tot) lies in (z_lo, z_hi) of
   0.5*(u^2 + v^2 + (0.5*(w(jz)+w(jz+1)))^2), accumulated in FP64 in a fixed order.
   lu,lv,lw: NULL, or (ldx,nyt,0:nz) outputs receiving dJ/d(u,v,w). */
int obl_ke_band(obl_ctx *ctx, const double *u, const double *v, const double *w,
                double z_lo, double z_hi, double *J, double *lu, double *lv, double *lw);
int obl_ke_band_dev(obl_ctx *ctx, const void *u, const void *v, const void *w,
                    double z_lo, double z_hi, double *J, void *lu, void *lv, void *lw);

/* ---- rollout gradient ----
   nsteps rollout steps from u0,v0,w0 with the state of every step checkpointed on the
   device, *J = ke band objective of the final state, and, when gu is not NULL, the
   reverse sweep of step_vjp (each step's convec fields recomputed from its
   checkpoint): gu,gv,gw = dJ/d(u0,v0,w0), x < nxt meaningful.  *J is a host double in
   both variants. */
int obl_rollout_grad(obl_ctx *ctx, int nsteps, const double *u0, const double *v0,
                     const double *w0, double z_lo, double z_hi, double *J,
                     double *gu, double *gv, double *gw);
int obl_rollout_grad_dev(obl_ctx *ctx, int nsteps, const void *u0, const void *v0,
                         const void *w0, double z_lo, double z_hi, double *J,
                         void *gu, void *gv, void *gw);

/* ---- ensemble: many independent instances through obl_step together ----
   No counterpart in the reference (one run = one domain).  Each instance has its own
   grid (and context: tables, work buffers); all share the options (precision, top
   mode, device).  ios[i] are device buffers in the storage type, as for obl_step_dev.
   Modes:
     OBL_ENS_SEQUENTIAL  instance after instance on the ensemble's stream;
     OBL_ENS_CONCURRENT  every instance on its own stream (fork/join);
     OBL_ENS_PERSISTENT  one cooperative launch over the work list of all instances,
                         dispatching on each unit's line lengths at run time (lengths
                         32..256; divtz planes must be NULL); every CTA takes a fixed share
                         of each phase, phases separated by grid barriers.  A barrier wait
                         that gives up is reported by obl_ensemble_synchronize as
                         OBL_ERR_TIMEOUT.
     OBL_ENS_PERSISTENT_SPLIT  the same work list in three cooperative launches, one
                         per register class (row passes at 2 CTAs/SM, column passes and
                         the solve at 4).
     OBL_ENS_PERSISTENT_FLOW  one cooperative launch without grid barriers: CTAs take
                         units from one work counter and a unit waits (bounded) only for
                         the previous phase of its own instance.  Phase times are recorded
                         by the barrier forms only.
   obl_ensemble_capture_dev records one step for the given buffers into a CUDA graph
   (after one uncaptured step that allocates every buffer); obl_ensemble_replay
   launches it.  obl_ensemble_time_dev returns the CUDA-event time per step. */
#define OBL_ENS_SEQUENTIAL 0
#define OBL_ENS_CONCURRENT 1
#define OBL_ENS_PERSISTENT 2
#define OBL_ENS_PERSISTENT_SPLIT 3
#define OBL_ENS_PERSISTENT_FLOW 4
typedef struct obl_ensemble obl_ensemble;
int obl_ensemble_create(const obl_grid *grids, int n, const obl_options *opt, obl_ensemble **out);
int obl_ensemble_destroy(obl_ensemble *ens);
int obl_ensemble_size(const obl_ensemble *ens);
int obl_ensemble_context(obl_ensemble *ens, int i, obl_ctx **ctx);
int obl_ensemble_set_mode(obl_ensemble *ens, int mode, int blocks_per_sm);
int obl_ensemble_get_mode(const obl_ensemble *ens, int *mode, int *blocks_per_sm, int *blocks);
int obl_ensemble_step_dev(obl_ensemble *ens, const obl_step_io *ios);
int obl_ensemble_capture_dev(obl_ensemble *ens, const obl_step_io *ios);
int obl_ensemble_replay(obl_ensemble *ens);
int obl_ensemble_synchronize(obl_ensemble *ens);
int obl_ensemble_time_dev(obl_ensemble *ens, const obl_step_io *ios, int use_graph, int warmup,
                          int reps, double *ms_per_step);
/* on != 0: the persistent kernel records the global timer at each phase boundary (CTA
   0); ms (n >= 6 entries, may be NULL) receives the phases of the last persistent step */
int obl_ensemble_phase_times(obl_ensemble *ens, int on, double *ms, int n);
int obl_ensemble_last_error(const obl_ensemble *ens, char *buf, size_t n);

/* Failure-path self-test (no counterpart in the reference): one CTA runs the persistent
   kernel's grid barrier on the context's stream.  never_released = 0: the barrier
   releases, OBL_OK.  never_released = 1: no other CTA ever arrives, the bounded wait gives
   up after a few seconds and OBL_ERR_TIMEOUT is returned, the context staying usable. */
int obl_selftest_grid_barrier(obl_ctx *ctx, int never_released);

/* Bounds-checked build (compiled with -DOBL_CHECK=1; no counterpart in the reference): the
   hot-path kernels test each checked global index against the extents their arguments
   give, record a failed test and skip the access instead of making it.  After the device
   has drained, *count = the failed tests since the last call (the records are then
   cleared) and buf (n > 0, may be NULL) describes the first: its check site and index.
   *count = -1 in the product build, which has no checks. */
int obl_check_report(long long *count, char *buf, size_t n);
/* Bounds-checked build: one thread fails one check (index 1 against an extent of 1, with no
   access made), so that obl_check_report then gives count 1 at site 12; the record path
   is tested without a wrong index in a kernel.  OBL_ERR_UNSUPPORTED in the product build. */
int obl_check_selftest(void);

/* ---- the step on a z-slab of a domain split over nranks ranks (one GPU each) ----
   The reference splits z over npz MPI ranks and pipelines its Thomas sweeps rank by rank
   with a send/recv per y-row (109_press_stag_array.f90:244-319, 103_flosol.f90:169-173).
   Here each rank's context holds its slab (nzt = the rank's levels + 1, lz_tot its height:
   level 0 and nz are the planes shared with the ranks below and above) and the solve is
   partitioned: every rank eliminates its own rows, the ranks exchange two kinds of small
   data through the caller's collectives, and every rank finishes its rows:
     1. obl_slab_begin_dev: the forward pass of obl_step (ddx, ddy, zero_padding, RHS
        spectra), the divtz planes (divtz_bot used on rank 0, divtz_top on rank nranks-1),
        and plane_out = this rank's H_z(1) spectrum (plane_bytes);
     2. caller: all-gather the planes; plane_above = the plane of rank+1 (ignored on the
        top rank);
     3. obl_slab_solve_dev: the rank's rows eliminated (in the storage precision, the FP64
        island columns of the mixed mode in FP64); iface_out = its interface
        coefficients (iface_bytes, FP64);
     4. caller: all-gather the interface coefficients, rank-major (nranks * iface_bytes);
     5. obl_slab_finish_dev: the reduced 2*nranks-unknown system (redundantly), the rank's
        p_hat and spectral dpdz, inverse transforms and project() with the rank's role
        (jz_min = 2 and w(1) = 0 on rank 0; w(nz) = 0 and the stress-free copy on the top).
   Levels 1..nz-1 of the outputs equal the single-domain obl_step at the same global
   levels.  Only OBL_TOP_NEUMANN (npz >= 2 semantics); nranks <= 16. */
int obl_slab_sizes(obl_ctx *ctx, long long *plane_bytes, long long *iface_bytes);
int obl_slab_begin_dev(obl_ctx *ctx, const obl_step_io *io, int rank, int nranks, void *plane_out);
int obl_slab_solve_dev(obl_ctx *ctx, const void *plane_above, int rank, int nranks, void *iface_out);
int obl_slab_finish_dev(obl_ctx *ctx, const obl_step_io *io, const void *iface_all, int rank, int nranks);

#ifdef __cplusplus
}
#endif
#endif
