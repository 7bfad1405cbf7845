// Shared definitions of the shallow-water B200 library: status codes, errors,
// device buffers, physical constants and the generic launch helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sw_cuda.h"
#include "sw_fft.cuh"

namespace sw {

// NVTX range of one stage of the step (main_invert, psolve set-up, sweeps, source,
// update), shown on a profiler's timeline for host-driven steps and graph captures.
// NVTX is header-only and costs nothing when no tool is attached.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// ---- physical constants (reference src/constants.rs:8-17) -----------------
constexpr double PI = 3.14159265358979323846;
constexpr double COF = 4.0 * PI;
constexpr double CGW = 2.0 * PI;
constexpr double HBAR = 0.4;
constexpr double CDAMP = 10.0;
constexpr double NNU = 3.0;
constexpr double CSQ = CGW * CGW;
constexpr double FSQ = COF * COF;
constexpr double COFI = 1.0 / COF;
constexpr double GRAVITY = CSQ / HBAR;

constexpr int MAX_NZ = 128;

// Kernels launched by this library (process-wide), for launch accounting.
inline std::atomic<long long>& launch_counter() {
    static std::atomic<long long> c{0};
    return c;
}
inline void count_launch(long long n = 1) { launch_counter().fetch_add(n, std::memory_order_relaxed); }

// ---- errors -------------------------------------------------------------------
struct Error : std::runtime_error {
    int status;
    Error(int st, const std::string& m) : std::runtime_error(m), status(st) {}
};

#define SW_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            throw ::sw::Error(SW_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define SW_CHECK_LAUNCH() SW_CUDA(cudaGetLastError())

inline void require(bool ok, int status, const std::string& msg) {
    if (!ok) throw Error(status, msg);
}

// ---- device buffer -------------------------------------------------------------
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        release();
        p = o.p; n = o.n; o.p = nullptr; o.n = 0;
        return *this;
    }
    void alloc(size_t count) {
        release();
        if (count) SW_CUDA(cudaMalloc(&p, count * sizeof(T)));
        n = count;
        if (p) sw_bc_register(p, count * sizeof(T), 1);
    }
    void release() {
        if (p) sw_bc_register(p, 0, 0);
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
    operator T*() const { return p; }
};

// ---- generic launches ------------------------------------------------------------
// f(o, i) for o < nplanes, i < n2 (one thread per element, plane = blockIdx.y).
template <class F>
__global__ void k_planes(int n2, F f) {
    const int o = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) f(o, i);
}
template <class F>
inline void for_planes(cudaStream_t s, int nplanes, int n2, F f) {
    if (nplanes <= 0) return;
    const int threads = 256;
    int bx = (n2 + threads - 1) / threads;
    if (bx > 1024) bx = 1024;
    dim3 grid(bx, nplanes);
    k_planes<<<grid, threads, 0, s>>>(n2, f);
    SW_CHECK_LAUNCH();
    count_launch();
}

// f(o, i) for o < nplanes and i = 0, 4, 8, ... < n2 (n2 % 4 == 0): one thread per
// four consecutive elements, for bodies that move them with ld4 / st4.
template <class F>
__global__ void k_planes4(int n4, F f) {
    const int o = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x) f(o, 4 * i);
}
template <class F>
inline void for_planes4(cudaStream_t s, int nplanes, int n2, F f) {
    if (nplanes <= 0) return;
    const int threads = 256, n4 = n2 / 4;
    int bx = (n4 + threads - 1) / threads;
    if (bx > 1024) bx = 1024;
    dim3 grid(bx, nplanes);
    k_planes4<<<grid, threads, 0, s>>>(n4, f);
    SW_CHECK_LAUNCH();
    count_launch();
}
// Four consecutive elements at p (p 16-byte aligned for float, 32 for double).
__device__ __forceinline__ void ld4(const float* p, float (&v)[4]) {
    if (!SW_BC_OK(p, 16, 16)) {
        v[0] = v[1] = v[2] = v[3] = 0.f;
        return;
    }
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&v)[4]) {
    if (!SW_BC_OK(p, 32, 16)) {
        v[0] = v[1] = v[2] = v[3] = 0.0;
        return;
    }
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, const float (&v)[4]) {
    if (!SW_BC_OK(p, 16, 16)) return;
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&v)[4]) {
    if (!SW_BC_OK(p, 32, 16)) return;
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// f(c) for c < ncols: one thread per (member, horizontal point) column.
// Column bodies loop over levels; their loops are unrolled so that loads of
// later levels are in flight while earlier ones are used.
template <class F>
__global__ void k_cols(int ncols, F f) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncols; c += gridDim.x * blockDim.x) f(c);
}
template <class F>
inline void for_cols(cudaStream_t s, int ncols, F f) {
    if (ncols <= 0) return;
    const int threads = 128;
    int blocks = (ncols + threads - 1) / threads;
    k_cols<<<blocks, threads, 0, s>>>(ncols, f);
    SW_CHECK_LAUNCH();
    count_launch();
}

// Deterministic per-group reductions.  Stage 1: grid (chunks, ngroups); each
// CTA folds its share of group g with op into NV partials.  Stage 2 folds the
// chunk partials of each group in fixed order.  op: 0 = sum, 1 = max.
constexpr int RED_THREADS = 256;
constexpr int RED_CHUNKS = 16;
constexpr int RED_MAX_CHUNKS = 256;

template <int NV>
struct RedVals {
    double v[NV];
};

template <int NV, class F>
__global__ void __launch_bounds__(RED_THREADS)
k_reduce1(long long group_len, unsigned opmask, F f, double* partial) {
    const int g = blockIdx.y;
    const int ch = blockIdx.x;
    const long long per = (group_len + gridDim.x - 1) / gridDim.x;
    const long long beg = per * ch;
    const long long end = (beg + per < group_len) ? beg + per : group_len;
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) acc[v] = ((opmask >> v) & 1u) ? -INFINITY : 0.0;
    for (long long i = beg + threadIdx.x; i < end; i += blockDim.x) {
        RedVals<NV> r = f(g, i);
#pragma unroll
        for (int v = 0; v < NV; v++) acc[v] = ((opmask >> v) & 1u) ? fmax(acc[v], r.v[v]) : acc[v] + r.v[v];
    }
    __shared__ double sh[RED_THREADS];
#pragma unroll
    for (int v = 0; v < NV; v++) {
        sh[threadIdx.x] = acc[v];
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s)
                sh[threadIdx.x] = ((opmask >> v) & 1u) ? fmax(sh[threadIdx.x], sh[threadIdx.x + s])
                                                       : sh[threadIdx.x] + sh[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) partial[((size_t)g * gridDim.x + ch) * NV + v] = sh[0];
        __syncthreads();
    }
}
template <int NV>
__global__ void k_reduce2(int ngroups, int nchunks, unsigned opmask, const double* partial, double* out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ngroups * NV) return;
    const int g = t / NV, v = t % NV;
    const bool mx = (opmask >> v) & 1u;
    double a = mx ? -INFINITY : 0.0;
    for (int c = 0; c < nchunks; c++) {
        double x = partial[((size_t)g * nchunks + c) * NV + v];
        a = mx ? fmax(a, x) : a + x;
    }
    out[t] = a;
}

// Reduce ngroups groups of group_len items; f(g, i) -> RedVals<NV>; result
// out[g*NV + v] (device).  partial must hold ngroups*RED_CHUNKS*NV doubles.
// Chunks per group: enough CTAs for ~4 per SM overall, at least 1024 items each.
inline int red_chunks(int ngroups, long long group_len) {
    long long c = 592 / (ngroups > 0 ? ngroups : 1);
    const long long by_len = group_len / 1024;
    if (c > by_len) c = by_len;
    if (c > RED_MAX_CHUNKS) c = RED_MAX_CHUNKS;
    if (c < 1) c = 1;
    return (int)c;
}
template <int NV, class F>
inline void reduce_groups(cudaStream_t s, int ngroups, long long group_len, unsigned opmask, F f,
                          double* partial, double* out) {
    const int nch = red_chunks(ngroups, group_len);
    dim3 g1(nch, ngroups);
    k_reduce1<NV><<<g1, RED_THREADS, 0, s>>>(group_len, opmask, f, partial);
    SW_CHECK_LAUNCH();
    const int t = ngroups * NV;
    k_reduce2<NV><<<(t + 127) / 128, 128, 0, s>>>(ngroups, nch, opmask, partial, out);
    SW_CHECK_LAUNCH();
    count_launch(2);
}

}  // namespace sw
