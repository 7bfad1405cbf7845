// Debug build of the kernels' index arithmetic (compile with -DSW_BOUNDS_CHECK;
// `python shallow-water_b200/build.py --bounds-check` makes libswcuda_bc.so).
//
// The library's device memory is registered in a table on each device: every
// DevBuf allocation (through sw_bc_register) and, for the duration of a call, the
// caller's device buffers of the entry points that take them.  The shared access
// helpers (ld4 / st4, ldv2 / stv2m, the transform intermediates and the pressure
// sweep's accessors) check that each access lies inside one registered allocation
// and is aligned for its width.  An access that fails is recorded (the count, the
// first address and width) and skipped: a load returns zeros, a store writes
// nothing, so the debug build does not itself touch memory outside the
// allocations.  Every entry point then synchronises the device and returns
// SW_ERR_CUDA with the first failing address if an access failed.
//
// Only the solver's compilation unit (sw_capi.cu) is instrumented; the
// allocation-free transform and the standalone tridiagonal solver compile without
// the checks.  The checks cost a binary search per access and the device
// synchronisation after every call: a debug build, not for timing, and not for use
// inside a caller's stream capture.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace sw {
// Registers (add != 0) or unregisters the device allocation [p, p + bytes) of the
// current device for the bounds checks; a no-op in builds without them.  Defined
// once, in sw_capi.cu, so that every compilation unit's DevBuf calls the same one.
void sw_bc_register(const void* p, size_t bytes, int add);
}  // namespace sw

#ifdef SW_BOUNDS_CHECK
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

namespace sw {
namespace bc {

constexpr int MAX_RANGES = 4096;
struct Range {
    unsigned long long lo, hi;
};
static __device__ Range g_ranges[MAX_RANGES];  // sorted by lo, disjoint
static __device__ int g_nranges;
static __device__ unsigned long long g_fault[3];  // failed accesses, first address, its width

__device__ __forceinline__ bool ok(const void* p, unsigned bytes, unsigned align) {
    const unsigned long long a = reinterpret_cast<unsigned long long>(p), e = a + bytes;
    int lo = 0, hi = g_nranges - 1, k = -1;
    while (lo <= hi) {  // last range with lo <= a
        const int mid = (lo + hi) >> 1;
        if (g_ranges[mid].lo <= a) {
            k = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    if (k >= 0 && e <= g_ranges[k].hi && (a & (unsigned long long)(align - 1)) == 0ull) return true;
    if (atomicAdd(&g_fault[0], 1ull) == 0ull) {
        g_fault[1] = a;
        g_fault[2] = bytes;
    }
    return false;
}

struct Registry {
    std::mutex mu;
    std::map<int, std::vector<Range>> by_dev;
};
inline Registry& registry() {
    static Registry r;
    return r;
}
inline void upload_locked(int dev, std::vector<Range>& v) {
    std::sort(v.begin(), v.end(), [](const Range& x, const Range& y) { return x.lo < y.lo; });
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    const int n = (int)std::min(v.size(), (size_t)MAX_RANGES);
    if (n) cudaMemcpyToSymbol(g_ranges, v.data(), sizeof(Range) * n);
    cudaMemcpyToSymbol(g_nranges, &n, sizeof(int));
    if (cur != dev) cudaSetDevice(cur);
}
inline void add(const void* p, size_t bytes) {
    if (!p || !bytes) return;
    int dev = 0;
    cudaGetDevice(&dev);
    Registry& r = registry();
    std::lock_guard<std::mutex> lk(r.mu);
    auto& v = r.by_dev[dev];
    const unsigned long long a = reinterpret_cast<unsigned long long>(p);
    v.push_back(Range{a, a + bytes});
    upload_locked(dev, v);
}
inline void remove(const void* p) {
    if (!p) return;
    const unsigned long long a = reinterpret_cast<unsigned long long>(p);
    Registry& r = registry();
    std::lock_guard<std::mutex> lk(r.mu);
    for (auto& kv : r.by_dev) {
        auto& v = kv.second;
        auto it = std::find_if(v.begin(), v.end(), [a](const Range& x) { return x.lo == a; });
        if (it != v.end()) {
            v.erase(it);
            upload_locked(kv.first, v);
            return;
        }
    }
}
// Failed accesses on the current device since the last call (and the first one's
// address and width), after the device has finished its work; clears the record.
inline unsigned long long take_fault(unsigned long long* addr, unsigned long long* bytes) {
    cudaDeviceSynchronize();
    unsigned long long f[3] = {0ull, 0ull, 0ull};
    cudaMemcpyFromSymbol(f, g_fault, sizeof(f));
    if (f[0]) {
        const unsigned long long z[3] = {0ull, 0ull, 0ull};
        cudaMemcpyToSymbol(g_fault, z, sizeof(z));
    }
    *addr = f[1];
    *bytes = f[2];
    return f[0];
}
// The caller's device buffer of one entry point, registered for that call.
struct Scoped {
    const void* p;
    Scoped(const void* p_, size_t bytes) : p(p_) { add(p_, bytes); }
    ~Scoped() {
        cudaDeviceSynchronize();
        remove(p);
    }
    Scoped(const Scoped&) = delete;
    Scoped& operator=(const Scoped&) = delete;
};

}  // namespace bc
}  // namespace sw
#define SW_BC_OK(p, bytes, align) ::sw::bc::ok((const void*)(p), (unsigned)(bytes), (unsigned)(align))
#define SW_BC_CAT2(a, b) a##b
#define SW_BC_CAT(a, b) SW_BC_CAT2(a, b)
#define SW_BC_SCOPE(p, bytes) ::sw::bc::Scoped SW_BC_CAT(sw_bc_scope_, __LINE__)((const void*)(p), (size_t)(bytes))
#else
#define SW_BC_OK(p, bytes, align) true
#define SW_BC_SCOPE(p, bytes) ((void)0)
#endif
