// Allocation-free variant of the batched 2-D transform (sw_fft2d_noalloc).
//
// Who needs it: host programs that cannot call cudaMalloc at the point where they
// transform.  Examples are a plugin that runs inside a framework that owns all
// device memory through its own pool; code that is being recorded into a CUDA
// graph by someone else, where an allocation would invalidate the capture; and
// latency-critical loops that must not pay for allocation.  Such callers bring
// their input and output buffers; everything else this entry point needs lives in
// one fixed array compiled into the library.
//
// Limits and sharing rules:
//   * The scratch is a file-scope __device__ array of SCRATCH_BYTES
//     (16 MiB) that every GPU loading the library holds until the process exits.
//     It stores the twiddle table and the transposed intermediate of up to
//     (16 MiB - 64 KiB) / (ng*ng*8) planes at a time; larger batches are done in
//     chunks of that many planes.
//   * ng may be at most MAX_NG (1024) and must factor into 2, 3 and 5;
//     larger sizes are rejected with SW_ERR_ARG and a message.
//   * All calls share the array and leave their data in it.  Nothing in it needs to
//     start at zero (each call rewrites the twiddles and the intermediate before
//     reading them), but two calls whose work overlaps on the GPU - on different
//     streams, or from different host threads - race on it and give wrong results.
//     Serialise such calls on one stream.
//   * The first call on each device looks the array's device address up with
//     cudaGetSymbolAddress (with that device current) and caches it with the
//     device's current CUDA context; make that first call before any stream capture
//     that includes this entry point.  A call made under another context of the
//     device (after a cudaDeviceReset, say) looks the address up again.
// (compiled without the bounds checks of the debug build: only sw_capi.cu registers memory)
#undef SW_BOUNDS_CHECK
#include <cuda.h>

#include <mutex>

#include "sw_fft2d.cuh"

namespace sw {
namespace noalloc {

constexpr size_t SCRATCH_BYTES = 16u << 20;
constexpr size_t TWIDDLE_BYTES = 64u << 10;  // 4096 complex doubles
constexpr int MAX_NG = 1024;

static __device__ __align__(256) unsigned char g_scratch[SCRATCH_BYTES];

// Device address of g_scratch per device, with the context it was looked up in
// (host code cannot use the symbol itself).
static std::mutex g_mu;
static void* g_addr[64] = {nullptr};
static CUcontext g_ctx[64] = {nullptr};

// The calling thread's current CUDA context, through the driver entry point that
// the runtime hands out (no link against libcuda needed).
static CUcontext current_context() {
    using Fn = CUresult (*)(CUcontext*);
    static Fn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<Fn>(p);
    }();
    CUcontext c = nullptr;
    if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
    return c;
}

static int scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return SW_ERR_CUDA;
    if (dev < 0 || dev >= 64) return SW_ERR_ARG;
    const CUcontext ctx = current_context();
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev] || g_ctx[dev] != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || p == nullptr) return SW_ERR_CUDA;
        g_addr[dev] = p;
        g_ctx[dev] = current_context();  // the lookup may have made the primary context current
    }
    *out = g_addr[dev];
    return SW_OK;
}

// exp(-2 pi i t / n) for t < n, written into the scratch.
__global__ void k_twiddles(double2* tw, int n) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)t / (double)n, &s, &c);
        tw[t] = make_double2(c, -s);
    }
}

struct PhysLoad {  // physical plane p[iy + ng*ix]
    const double* a;
    int ng;
    __device__ __forceinline__ double operator()(int o, int iy, int ix) const {
        return a[((size_t)o * ng + ix) * ng + iy];
    }
};
struct SpecStore {  // spectral plane s[kx + ng*ky]
    double* b;
    int ng;
    __device__ __forceinline__ void operator()(int o, int kx, int ky, double v) const {
        b[((size_t)o * ng + ky) * ng + kx] = v;
    }
};
struct SpecLoad {
    const double* a;
    int ng;
    __device__ __forceinline__ double operator()(int o, int kx, int ky) const {
        return a[((size_t)o * ng + ky) * ng + kx];
    }
};
struct PhysStore {
    double* b;
    int ng;
    __device__ __forceinline__ void operator()(int o, int iy, int ix, double v) const {
        b[((size_t)o * ng + ix) * ng + iy] = v;
    }
};

static int run(int ng, int direction, int nplanes, const double* in, double* out, cudaStream_t s,
               std::string& msg) {
    if (ng < 4 || ng > MAX_NG || ng % 2 != 0) {
        msg = "sw_fft2d_noalloc: ng must be even and in [4, " + std::to_string(MAX_NG) + "]";
        return SW_ERR_ARG;
    }
    if (direction != 0 && direction != 1) {
        msg = "sw_fft2d_noalloc: direction must be 0 (ptospc) or 1 (spctop)";
        return SW_ERR_ARG;
    }
    if (nplanes < 1 || !in || !out) {
        msg = "sw_fft2d_noalloc: need nplanes >= 1 and non-null in/out";
        return SW_ERR_ARG;
    }
    FftPlan plan;
    if (build_plan(ng, plan) != SW_OK) {
        msg = "sw_fft2d_noalloc: ng must factor into 2, 3 and 5";
        return SW_ERR_FACTORISE;
    }
    // A launch error of this call must not be mixed up with an earlier error of the
    // caller's own work: report a pending one as such and leave it in place.
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        msg = std::string("sw_fft2d_noalloc: a CUDA error was pending before the call: ") +
              cudaGetErrorString(pending);
        return SW_ERR_CUDA;
    }
    void* base = nullptr;
    int st = scratch_address(&base);
    if (st != SW_OK) {
        msg = "sw_fft2d_noalloc: cudaGetSymbolAddress of the scratch array failed";
        return st;
    }
    double2* tw = reinterpret_cast<double2*>(base);
    double* mid = reinterpret_cast<double*>(static_cast<unsigned char*>(base) + TWIDDLE_BYTES);
    const size_t plane_bytes = (size_t)ng * ng * sizeof(double);
    const int cap = (int)((SCRATCH_BYTES - TWIDDLE_BYTES) / plane_bytes);
    k_twiddles<<<(ng + 255) / 256, 256, 0, s>>>(tw, ng);
    const cudaError_t le = cudaGetLastError();  // nothing was pending, so this is the launch's own
    if (le != cudaSuccess) {
        msg = std::string("sw_fft2d_noalloc: twiddle kernel launch failed: ") + cudaGetErrorString(le);
        return SW_ERR_CUDA;
    }
    const int tc = pick_tile<double>(ng);
    const double sc = 1.0 / std::sqrt((double)ng);
    for (int o0 = 0; o0 < nplanes; o0 += cap) {
        const int cnt = (nplanes - o0 < cap) ? nplanes - o0 : cap;
        const size_t off = (size_t)o0 * ng * ng;
        if (direction == 0) {
            launch_pass<double, false, true, true>(s, plan, tw, tc, sc, cnt, ng, PhysLoad{in + off, ng},
                                                   MidCP<double>{mid, ng});
            launch_pass<double, false, false, true>(s, plan, tw, tc, sc, cnt, ng, MidPC<double>{mid, ng},
                                                    SpecStore{out + off, ng});
        } else {
            launch_pass<double, true, true, false>(s, plan, tw, tc, sc, cnt, ng, SpecLoad{in + off, ng},
                                                   MidPC<double>{mid, ng});
            launch_pass<double, true, true, true>(s, plan, tw, tc, sc, cnt, ng, MidCP<double>{mid, ng},
                                                  PhysStore{out + off, ng});
        }
    }
    return SW_OK;
}

}  // namespace noalloc
}  // namespace sw

namespace sw {
void record_error(const std::string& msg);  // sets the message sw_last_error() returns
}

extern "C" {

int sw_fft2d_noalloc(int ng, int direction, int nplanes, const double* in, double* out, void* stream) {
    std::string msg;
    int st;
    try {
        st = sw::noalloc::run(ng, direction, nplanes, in, out, (cudaStream_t)stream, msg);
    } catch (const sw::Error& e) {
        msg = e.what();
        st = e.status;
    }
    if (st != SW_OK) sw::record_error(msg);
    return st;
}

}  // extern "C"
