// Self-checking builds (-DHSC_CHECKED): index guards that record the first
// failing check (code, value) and skip the access instead of touching memory
// out of bounds.  In normal builds HSC_IN(...) is the constant true.
#pragma once
#include <cuda_runtime.h>

namespace hsc {

#ifdef HSC_CHECKED
static __device__ long long g_hsc_fail[2];
static __device__ __noinline__ void hsc_check_fail(int code, long long v) {
    if (atomicCAS(reinterpret_cast<unsigned long long*>(&g_hsc_fail[0]), 0ull, (unsigned long long)code) == 0ull)
        g_hsc_fail[1] = v;
}
#define HSC_IN(cond, code, val) ((cond) ? true : (::hsc::hsc_check_fail((code), (long long)(val)), false))
static inline void hsc_read_fail(long long* out) {
    if (cudaMemcpyFromSymbol(out, g_hsc_fail, sizeof(long long) * 2) != cudaSuccess) { out[0] = -1; out[1] = 0; }
}
#else
#define HSC_IN(cond, code, val) true
static inline void hsc_read_fail(long long* out) { out[0] = 0; out[1] = 0; }
#endif

}  // namespace hsc
