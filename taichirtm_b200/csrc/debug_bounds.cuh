// Bounds-checking build (compile with -DRTM_BOUNDS_CHECK; the library is then
// built as librtm_b200_debug.so).  It stands in for a memory checker: every
// global access the propagation kernels make through the helpers below is
// tested against a table of the device buffers that are live for the current
// call (the plan's allocations and the caller's buffers, with their sizes).
// An access that falls outside every buffer is not performed: a load returns
// zero, a store is dropped; it is counted, and the entry point returns an
// error.  In the normal build the checks compile to nothing.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace rtm {

#ifdef RTM_BOUNDS_CHECK
constexpr int DBG_MAX_RANGES = 64;
struct DbgTable {
    unsigned long long begin[DBG_MAX_RANGES], end[DBG_MAX_RANGES];
    int n;
};
// One table per module; a module whose host code never fills it (n == 0)
// checks nothing.
__constant__ DbgTable g_dbg_table;
__device__ unsigned long long g_dbg_bad;    // accesses outside every buffer
__device__ unsigned long long g_dbg_first;  // address of the first one

__device__ __forceinline__ bool dbg_ok(const void *ptr, unsigned bytes) {
    const int n = g_dbg_table.n;
    if (n == 0) return true;
    const unsigned long long a = (unsigned long long)(uintptr_t)ptr;
    for (int k = 0; k < n; ++k)
        if (a >= g_dbg_table.begin[k] && a + bytes <= g_dbg_table.end[k]) return true;
    if (atomicAdd(&g_dbg_bad, 1ull) == 0ull) g_dbg_first = a;
    return false;
}
#define RTM_DBG_OK(ptr, bytes) ::rtm::dbg_ok((ptr), (unsigned)(bytes))

// rtm_bounds_probe: evaluate the check for one range without touching it.
__device__ int g_dbg_probe;
static __global__ void bounds_probe_kernel(const void *ptr, unsigned bytes) { g_dbg_probe = dbg_ok(ptr, bytes) ? 1 : 0; }
#else
#define RTM_DBG_OK(ptr, bytes) true
#endif

// __ldg through the check (an unchecked __ldg in the normal build).
template <typename T>
__device__ __forceinline__ T ldg_chk(const T *ptr) {
    if (!RTM_DBG_OK(ptr, sizeof(T))) return T();
    return __ldg(ptr);
}

// Plain store through the check.
template <typename T>
__device__ __forceinline__ void st_chk(T *ptr, T v) {
    if (!RTM_DBG_OK(ptr, sizeof(T))) return;
    *ptr = v;
}

}  // namespace rtm
