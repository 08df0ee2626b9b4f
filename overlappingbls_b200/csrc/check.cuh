// check.cuh -- index checks of the bounds-checked build (-DOBL_CHECK=1).
//
// In that build every checked global access of the hot-path kernels first tests its
// index against the extent of the buffer it addresses, as the kernel's arguments
// describe it.  A failed test records the check site and the offending index in this
// translation unit's record and skips the access (a load yields zero): nothing traps
// and no access leaves its buffer, so a wrong index shows up as a report, not as a
// fault.  The host reads and clears the records of all translation units through
// obl_check_report.  In the product build (OBL_CHECK = 0) the checks compile away.
#pragma once
#include <cuda_runtime.h>

#ifndef OBL_CHECK
#define OBL_CHECK 0
#endif

namespace obl {

// check sites (the first failing one is reported)
enum CheckSite : int {
    CK_COL_LOAD = 1, CK_COL_STORE, CK_ROWS3_ROW, CK_ROWS3_SPEC, CK_TDMA_STORE, CK_TDMA_COPY, CK_PINV_COL_LOAD,
    CK_PINV_COL_STORE, CK_PINV_ROW, CK_GFORM_LOAD, CK_TDMA_LOAD, CK_SELFTEST
};

struct CheckRecord {
    unsigned long long count;   // failed checks
    unsigned long long first;   // site << 48 | low 48 bits of the index, of the first one
};

// host side: every translation unit registers the reader of its record (api.cu)
typedef void (*CheckReader)(CheckRecord *, bool reset);
int check_register(CheckReader r);

#if OBL_CHECK
static __device__ CheckRecord g_check;   // one record per translation unit
static void check_read_here(CheckRecord *out, bool reset)
{
    cudaMemcpyFromSymbol(out, g_check, sizeof(CheckRecord));
    if (reset) {
        const CheckRecord z{0, 0};
        cudaMemcpyToSymbol(g_check, &z, sizeof z);
    }
}
static const int g_check_registered = check_register(check_read_here);
#endif

// true when 0 <= i < n; otherwise (checked build) the failure is recorded
__device__ __forceinline__ bool ck_in(long long i, long long n, int site)
{
#if OBL_CHECK
    if (i >= 0 && i < n) return true;
    atomicAdd(&g_check.count, 1ULL);
    atomicCAS(&g_check.first, 0ULL, ((unsigned long long)site << 48) | ((unsigned long long)i & 0xffffffffffffULL));
    return false;
#else
    (void)i; (void)n; (void)site;
    return true;
#endif
}

} // namespace obl
