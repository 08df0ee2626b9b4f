// ensemble_kernel.cuh -- device code of the persistent ensemble kernel (see ensemble.cuh).
//
// Included by the translation units that instantiate the kernel (ensemble_*.cu).  Those are
// built with -Xptxas -dlcm=cg: every global load is served by L2, so no SM reads a stale
// L1 line of data another SM wrote in an earlier phase of the same launch.  Phases are
// separated by a grid barrier whose wait is bounded: a wait that gives up sets the error
// flag and the kernel returns (the host reports OBL_ERR_TIMEOUT), so a fault in the barrier
// logic cannot hang the GPU.  The launch is cooperative, which guarantees that all CTAs are
// resident together.
#pragma once
#include "ensemble.cuh"

namespace obl {

// line lengths the ensemble kernel is instantiated for
#define OBL_ENS_FOR_EACH_N(X) X(32) X(48) X(64) X(96) X(128) X(192) X(256)

constexpr long long kEnsSpinLimit = 1LL << 24;   // ~2 s of 128 ns sleeps

// Grid barrier: arrival counter bar[0], generation bar[1].  Returns false once any CTA
// gave up waiting.
__device__ __forceinline__ bool ens_barrier(unsigned *bar, int *err)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned *gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long spins = 0;
            while (*gen == g) {
                if (++spins > kEnsSpinLimit) {
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
        if (*(volatile int *)err) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

// kinds of plan tables held in shared memory
enum { K_ROWS = 0, K_PAD, K_DDY, K_FWD, K_PINVC, K_PINVR };

template <typename T, int N>
__device__ __forceinline__ void ens_rows(const RowsFwd3Args<T> &a, long long u, C2<T> *sm, int &lk, int &ln)
{
    using GG = FwdFusedGeo<T, N>;
    C2<T> *twF = sm, *twB = twF + GG::TF, *twPB = twB + GG::TB, *scr = twPB + GG::TPB;
    if (lk != K_ROWS || ln != N) {
        __syncthreads();
        for (int i = threadIdx.x; i < GG::TF; i += blockDim.x) twF[i] = a.twF[i];
        for (int i = threadIdx.x; i < GG::TB; i += blockDim.x) twB[i] = a.twB[i];
        for (int i = threadIdx.x; i < GG::TPB; i += blockDim.x) twPB[i] = a.twPB[i];
        __syncthreads();
        lk = K_ROWS;
        ln = N;
    }
    rows_fwd3_unit<T, N>(a, u, twF, twB, twPB, scr);
}

template <typename T, int N, int OP, bool REAL>
__device__ __forceinline__ void ens_cols(const ColArgs<T> &a, int nb, long long loc, int kind, C2<T> *sm, int &lk,
                                         int &ln)
{
    using D = LineDerived<N, OP>;
    C2<T> *twF = sm, *twB = twF + D::TF, *buf = twB + D::TB;
    __syncthreads();   // the previous unit's last reads of the exchange scratch are done
    if (lk != kind || ln != N) {
        load_tables<T, N, OP>(a.twF, a.twB, twF, twB);
        __syncthreads();
        lk = kind;
        ln = N;
    }
    const int z = (int)(loc / nb), bx = (int)(loc - (long long)z * nb);
    cols2_unit<T, N, OP, REAL>(a, bx, z, twF, twB, buf);
}

template <typename T, int N>
__device__ __forceinline__ void ens_pinv_cols(const PinvColArgs<T> &a, int nb, long long loc, C2<T> *sm, int &lk,
                                              int &ln)
{
    using D = LineDerived<N, OP_INV>;
    C2<T> *twB = sm, *buf = twB + D::TB;
    __syncthreads();
    if (lk != K_PINVC || ln != N) {
        for (int i = threadIdx.x; i < D::TB; i += blockDim.x) twB[i] = a.twB[i];
        __syncthreads();
        lk = K_PINVC;
        ln = N;
    }
    const int z = (int)(loc / nb), bx = (int)(loc - (long long)z * nb);
    pinv_cols_unit<T, N>(a, bx, z, twB, buf);
}

template <typename T, int N>
__device__ __forceinline__ void ens_pinv_rows(const PinvRowArgs<T> &a, long long u, C2<T> *sm, int &lk, int &ln)
{
    using D = LineDerived<N, OP_INV>;
    C2<T> *twB = sm, *scr = twB + D::TB;
    if (lk != K_PINVR || ln != N) {
        __syncthreads();
        for (int i = threadIdx.x; i < D::TB; i += blockDim.x) twB[i] = a.twB[i];
        __syncthreads();
        lk = K_PINVR;
        ln = N;
    }
    pinv_rows_unit<T, N>(a, u, twB, scr);
}

template <typename T>
__device__ __forceinline__ void ens_unit(int ph, const EnsInst<T> &I, long long loc, C2<T> *sm, int &lk, int &ln)
{
    if (ph == 0) {   // multi-output rows: ddx, x-pad, RHS x-spectra
        const int f = (int)(loc / I.rows_units);
        const long long u = loc - (long long)f * I.rows_units;
        switch (I.nx) {
#define OBL_C(N) case N: ens_rows<T, N>(I.rows[f], u, sm, lk, ln); break;
            OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
        }
    } else if (ph == 1) {   // y-pad, ddy, y-transform of the RHS, boundary planes
        const long long np = 4LL * I.pad_nb * I.nlev, nd = 4LL * I.ddy_nb * I.nlev, nf = 3LL * I.fwd_nb * I.L;
        if (loc < np) {
            const long long per = (long long)I.pad_nb * I.nlev;
            const int f = (int)(loc / per);
            switch (I.ny) {
#define OBL_C(N) case N: ens_cols<T, N, OP_PAD, true>(I.padc[f], I.pad_nb, loc - f * per, K_PAD, sm, lk, ln); break;
                OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
            }
        } else if (loc < np + nd) {
            const long long per = (long long)I.ddy_nb * I.nlev, l = loc - np;
            const int f = (int)(l / per);
            switch (I.ny) {
#define OBL_C(N) case N: ens_cols<T, N, OP_DERIV, true>(I.ddyc[f], I.ddy_nb, l - f * per, K_DDY, sm, lk, ln); break;
                OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
            }
        } else if (loc < np + nd + nf) {
            const long long per = (long long)I.fwd_nb * I.L, l = loc - np - nd;
            const int f = (int)(l / per);
            switch (I.ny) {
#define OBL_C(N) case N: ens_cols<T, N, OP_FWD, false>(I.fwdc[f], I.fwd_nb, l - f * per, K_FWD, sm, lk, ln); break;
                OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
            }
        } else {   // H_z(0), H_z(L+1): spectra of the zero divtz planes
            C2<T> *a = I.Hz, *b = I.Hz + I.S * (I.L + 1);
            for (long long i = threadIdx.x; i < I.S; i += blockDim.x) {
                a[i] = mk<T>(0, 0);
                b[i] = mk<T>(0, 0);
            }
        }
    } else if (ph == 2) {   // tridiagonal solves: FP64 island units first, then the bulk
        if (loc < I.isl_units)
            tdma_column<T, double, true>(I.tdma, I.isl, loc * blockDim.x + threadIdx.x);
        else
            tdma_column<T, T, false>(I.tdma, I.isl, (loc - I.isl_units) * blockDim.x + threadIdx.x);
    } else if (ph == 3) {   // y-inverse of p_hat and the dpdz spectrum
        switch (I.ny) {
#define OBL_C(N) case N: ens_pinv_cols<T, N>(I.pc, I.pc_nb, loc, sm, lk, ln); break;
            OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
        }
    } else if (ph == 4) {   // x-inverse fused with project()
        switch (I.nx) {
#define OBL_C(N) case N: ens_pinv_rows<T, N>(I.pr, loc, sm, lk, ln); break;
            OBL_ENS_FOR_EACH_N(OBL_C)
#undef OBL_C
        }
    } else {   // project()'s boundary rows (110_project.f90:50-60)
        const long long pl = (long long)I.ldx * I.ny;
        for (long long o = threadIdx.x; o < pl; o += blockDim.x) {
            if (I.stress_free) {
                I.u[o + pl * (I.nz - 1)] = I.u[o + pl * (I.nz - 2)];
                I.v[o + pl * (I.nz - 1)] = I.v[o + pl * (I.nz - 2)];
            }
            I.w[o + pl * I.nz] = (T)0;
            I.w[o + pl] = (T)0;
        }
    }
}

// Phases [PB, PE) of the step; MINB CTAs per SM bound the registers (the row phases need
// ~128, the column and solve phases ~64, so the split launches run those at twice the
// occupancy).
template <typename T, int PB, int PE, int MINB>
__global__ void __launch_bounds__(256, MINB) k_ensemble(EnsArgs<T> e)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    C2<T> *sm = reinterpret_cast<C2<T> *>(smraw);
    int lk = -1, ln = -1;   // kind and line length of the tables now in shared memory
    auto stamp = [&](int i) {
        if (e.stamps && blockIdx.x == 0 && threadIdx.x == 0) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            e.stamps[i] = t;
        }
    };
    stamp(PB);
    for (int ph = PB; ph < PE; ++ph) {
        const long long *st = e.start + (long long)ph * (e.ninst + 1);
        const long long total = st[e.ninst];
        const long long chunk = (total + gridDim.x - 1) / gridDim.x;
        const long long i0 = (long long)blockIdx.x * chunk;
        const long long i1 = i0 + chunk < total ? i0 + chunk : total;
        int k = 0;
        for (long long it = i0; it < i1; ++it) {
            while (it >= st[k + 1]) ++k;
            ens_unit<T>(ph, e.inst[k], it - st[k], sm, lk, ln);
        }
        if (ph + 1 < PE && !ens_barrier(e.bar, e.err)) return;
        stamp(ph + 1);
    }
}

// Bounded wait of thread 0 until *cnt reaches need (the counter is raised by release
// reductions, read here with acquire loads); false once any CTA gave up (err), after
// raising err itself on timeout.
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ bool ens_wait_count(const unsigned *cnt, unsigned need, int *err)
{
    long long spins = 0;
    while (ld_acquire(cnt) < need) {
        if (*(volatile int *)err) return false;
        if (++spins > kEnsSpinLimit) {
            atomicExch(err, 1);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

// instances whose phase prefix sums the dataflow kernel keeps in shared memory (more are
// searched in global memory)
constexpr int kEnsFlowSmemInst = 64;

template <typename T, int MINB>
__global__ void __launch_bounds__(256, MINB) k_ensemble_flow(EnsArgs<T> e)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    C2<T> *sm = reinterpret_cast<C2<T> *>(smraw);
    __shared__ long long sSt[kEnsPhases * (kEnsFlowSmemInst + 1)];
    __shared__ long long sUnit[2];   // [it & 1]: the unit after next, taken during unit it
    __shared__ int sOk;
    // (instance, phase) pairs this CTA has seen complete, so that their later units skip the
    // check (instances past kEnsFlowSmemInst are always checked)
    __shared__ unsigned char sDone[kEnsFlowSmemInst * kEnsPhases];
    int lk = -1, ln = -1;   // kind and line length of the tables now in shared memory
    const int n1 = e.ninst + 1;
    const bool cached = e.ninst <= kEnsFlowSmemInst;
    if (cached)
        for (int i = threadIdx.x; i < kEnsPhases * n1; i += blockDim.x) sSt[i] = e.start[i];
    for (int i = threadIdx.x; i < kEnsFlowSmemInst * kEnsPhases; i += blockDim.x) sDone[i] = 0;
    const long long *st0 = cached ? sSt : e.start;
    long long total = 0;
    for (int ph = 0; ph < kEnsPhases; ++ph) total += e.start[(long long)ph * n1 + e.ninst];
    if (threadIdx.x == 0) {
        sUnit[0] = atomicAdd(e.flow, 1u);
        sUnit[1] = atomicAdd(e.flow, 1u);
    }
    __syncthreads();
    long long cur = sUnit[0], nxt = sUnit[1];
    __syncthreads();   // read before thread 0 overwrites sUnit[0]
    for (int it = 0; cur < total; ++it) {
        // the unit after next is taken while this one runs (read after the unit's last barrier)
        if (threadIdx.x == 0) sUnit[it & 1] = atomicAdd(e.flow, 1u);
        // phase (the list is phase-major) and instance (binary search of the phase's prefix sums)
        long long g = cur;
        int ph = 0;
        const long long *st = st0;
        while (g >= st[e.ninst]) {
            g -= st[e.ninst];
            ++ph;
            st += n1;
        }
        int lo = 0, hi = e.ninst - 1;   // the instance k with st[k] <= g < st[k+1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (st[mid] <= g) lo = mid;
            else hi = mid - 1;
        }
        const int k = lo;
        const EnsInst<T> &I = e.inst[k];
        unsigned *done = e.flow + 1 + (long long)k * kEnsPhases;
        if (threadIdx.x == 0) {
            const bool known = ph == 0 || (k < kEnsFlowSmemInst && sDone[k * kEnsPhases + ph - 1]);
            sOk = known ? 1 : ens_wait_count(done + ph - 1, (unsigned)I.count[ph - 1], e.err);
            if (sOk && ph > 0 && k < kEnsFlowSmemInst) sDone[k * kEnsPhases + ph - 1] = 1;
        }
        __syncthreads();
        if (!sOk) return;
        ens_unit<T>(ph, I, g - st[k], sm, lk, ln);
        __syncthreads();   // every thread's writes of the unit are issued; sOk is read
        // release: the unit's writes (ordered before by the CTA barrier) become visible to a
        // CTA that acquires the count; the reduction does not wait for them
        if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(done + ph) : "memory");
        cur = nxt;
        nxt = sUnit[it & 1];
    }
}

template <typename T, int MINB> cudaError_t EnsFlowKernel<T, MINB>::attr(size_t smem)
{
    static size_t sets[kMaxDevices] = {};
    const int ds = device_slot();
    if (ds >= 0 && smem <= sets[ds]) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_ensemble_flow<T, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && ds >= 0) sets[ds] = smem;
    return e;
}

template <typename T, int MINB> int EnsFlowKernel<T, MINB>::blocks_per_sm(size_t smem)
{
    if (attr(smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_ensemble_flow<T, MINB>, 256, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return per;
}

template <typename T, int MINB>
cudaError_t EnsFlowKernel<T, MINB>::launch(const EnsArgs<T> &a, int blocks, size_t smem, cudaStream_t s)
{
    cudaError_t e = attr(smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_ensemble_flow<T, MINB>, a);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

template <typename T, int PB, int PE, int MINB> cudaError_t EnsKernel<T, PB, PE, MINB>::attr(size_t smem)
{
    static size_t sets[kMaxDevices] = {};
    const int ds = device_slot();
    if (ds >= 0 && smem <= sets[ds]) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_ensemble<T, PB, PE, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess && ds >= 0) sets[ds] = smem;
    return e;
}

template <typename T, int PB, int PE, int MINB> int EnsKernel<T, PB, PE, MINB>::blocks_per_sm(size_t smem)
{
    if (attr(smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_ensemble<T, PB, PE, MINB>, 256, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return per;
}

template <typename T, int PB, int PE, int MINB>
cudaError_t EnsKernel<T, PB, PE, MINB>::launch(const EnsArgs<T> &a, int blocks, size_t smem, cudaStream_t s)
{
    cudaError_t e = attr(smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_ensemble<T, PB, PE, MINB>, a);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

} // namespace obl
