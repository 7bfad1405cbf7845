// Batched 2-D transforms (D2FFT::ptospc / spctop, reference src/sta2dfft.rs:91-123)
// as two coalesced tile passes through an L2-resident intermediate.
//
// Layouts: physical P[iy + ng*ix], spectral S[kx + ng*ky], intermediate
// M[iy + ng*kx] (the reference's transposed work array).
//   spctop: pass A  reverse along ky for tiles of kx columns  (S -> M)
//           pass B  reverse along kx for tiles of iy columns  (M -> P)
//   ptospc: pass A  forward along ix for tiles of iy columns  (P -> M)
//           pass B  forward along iy for tiles of kx columns  (M -> S)
// User functors:
//   spctop: ld(o, kx, ky) -> T spectral input,  st(o, iy, ix, T) physical output
//   ptospc: ld(o, iy, ix) -> T physical input,  st(o, kx, ky, T) spectral output
// so products, derivatives, filters and combinations fuse into the passes.
#pragma once
#include "sw_core.cuh"

namespace sw {

template <class LD>
struct LdOff {
    LD f;
    int o0;
    __device__ __forceinline__ auto operator()(int o, int c, int p) const { return f(o0 + o, c, p); }
};
template <class ST>
struct StOff {
    ST f;
    int o0;
    template <class V>
    __device__ __forceinline__ void operator()(int o, int c, int p, V v) const { f(o0 + o, c, p, v); }
};
// intermediate addressed [pt + ng*col] (point index contiguous)
template <typename T>
struct MidPC {
    T* m;
    int ng;
    __device__ __forceinline__ T operator()(int o, int c, int p) const { return m[((size_t)o * ng + c) * ng + p]; }
    __device__ __forceinline__ void operator()(int o, int c, int p, T v) const { m[((size_t)o * ng + c) * ng + p] = v; }
};
// intermediate addressed [col + ng*pt] (column index contiguous); columns
// (c, c+1), c even, are one aligned vector access
template <typename T>
struct MidCP {
    using T2 = typename C2<T>::t;
    static constexpr bool pair_io = true;
    T* m;
    int ng;
    __device__ __forceinline__ T operator()(int o, int c, int p) const { return m[((size_t)o * ng + p) * ng + c]; }
    __device__ __forceinline__ void operator()(int o, int c, int p, T v) const { m[((size_t)o * ng + p) * ng + c] = v; }
    __device__ __forceinline__ T2 ld2(int o, int c, int p) const {
        return *reinterpret_cast<const T2*>(m + ((size_t)o * ng + p) * ng + c);
    }
    __device__ __forceinline__ void st2(int o, int c, int p, T a, T b) const {
        T2 v;
        v.x = a;
        v.y = b;
        *reinterpret_cast<T2*>(m + ((size_t)o * ng + p) * ng + c) = v;
    }
};

inline int build_plan(int n, FftPlan& plan) {
    int rem = n;
    plan.n = n;
    plan.nrad = 0;
    if (n < 2 || n > 4096) return SW_ERR_FACTORISE;
    // largest radices first: fewer shared-memory passes (n = 256 -> 16 x 16)
    const int order[6] = {16, 8, 4, 2, 3, 5};
    for (int r : order)
        while (rem % r == 0) {
            if (plan.nrad >= FFT_MAX_RAD) return SW_ERR_FACTORISE;
            if (r == 16 && n == 512 && plan.nrad == 0) break;  // 512 = 8 x 8 x 8 (fewer registers than 16 x 16 x 2)
            plan.rad[plan.nrad++] = r;
            rem /= r;
        }
    if (n == 512) {
        plan.nrad = 3;
        plan.rad[0] = plan.rad[1] = plan.rad[2] = 8;
        rem = 1;
    }
    if (rem != 1) return SW_ERR_FACTORISE;
    int Ns = 1;
    for (int s = 0; s < plan.nrad; s++) {
        FftStage& g = plan.stg[s];
        g.R = plan.rad[s];
        g.Ns = Ns;
        g.nR = n / g.R;
        g.tstride = n / (Ns * g.R);
        g.dNs = make_fastdiv((uint32_t)Ns);
        g.dnR = make_fastdiv((uint32_t)g.nR);
        Ns *= g.R;
    }
    return SW_OK;
}

// Twiddles exp(-2 pi i t/n), t < n, computed in float64 on the host.
template <typename T>
inline std::vector<typename C2<T>::t> host_twiddles(int n) {
    std::vector<typename C2<T>::t> tw(n);
    for (int t = 0; t < n; t++) {
        const double a = 2.0 * PI * (double)t / (double)n;
        tw[t].x = (T)std::cos(a);
        tw[t].y = (T)(-std::sin(a));
    }
    return tw;
}

// Columns per CTA: a power of two (>= 2), keeping the pass within ~76 KB of
// shared memory so that several CTAs share an SM.
template <typename T>
inline int pick_tile(int n) {
    const int budget = 76 * 1024 / (int)sizeof(typename C2<T>::t) - n;
    int tc = 2;
    while (tc * 2 <= 32 && (tc * 2) * padded_len(n) <= budget) tc *= 2;
    return tc;
}
inline int ilog2(int x) {
    int l = 0;
    while ((1 << (l + 1)) <= x) l++;
    return l;
}

template <typename T, bool INV, bool LCF, bool SCF, class LD, class ST>
inline void launch_pass(cudaStream_t s, const FftPlan& plan, const typename C2<T>::t* tw, int tc, T sc,
                        int nout, int ncols, LD ld, ST st) {
    if (nout <= 0) return;
    constexpr int LT128 = 5;
    const size_t smem = fft_pass_smem<T>(plan.n, tc);
    int dev = 0;
    cudaGetDevice(&dev);
    // Kernel attributes are set once per device and kernel.  The flags are atomics
    // because several host threads (one per context) may launch at once; two threads
    // that both set an attribute set the same value, which is harmless.
    // compile-time pair kernels for the common lengths when the tile matches and
    // every tile is full (the generic kernel covers the rest)
    constexpr bool pair_ok = INV ? LCF : SCF;
    if constexpr (pair_ok) {
        if (plan.n == FFT_R_N && (tc == 16 || tc == 32) && ncols % tc == 0) {
            const int np = tc / 2;
            auto kern = np == 8 ? k_fft_pass_r<T, 8, INV, LCF, SCF, LD, ST> : k_fft_pass_r<T, 16, INV, LCF, SCF, LD, ST>;
            static std::atomic<int> attr_r[64][2] = {};
            if (dev < 64 && !attr_r[dev][np == 8 ? 0 : 1].load(std::memory_order_acquire)) {
                SW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
                SW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
                attr_r[dev][np == 8 ? 0 : 1].store(1, std::memory_order_release);
            }
            dim3 grid(ncols / tc, nout);
            kern<<<grid, 16 * np, fft_pass_smem_r<T>(np), s>>>(tw, sc, ld, st);
            SW_CHECK_LAUNCH();
            count_launch();
            return;
        }
    }
    if constexpr (pair_ok) {
        // n = 128 (n = 256 tiles are all served by the register-staged pass above)
        if (plan.n == 128 && tc == (1 << LT128) && ncols % tc == 0) {
            auto kern = k_fft_pass_s<T, 128, LT128, INV, LCF, SCF, LD, ST>;
            static std::atomic<int> attr_s[64] = {};
            if (dev < 64 && !attr_s[dev].load(std::memory_order_acquire)) {
                SW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
                SW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
                attr_s[dev].store(1, std::memory_order_release);
            }
            dim3 grid(ncols / tc, nout);
            kern<<<grid, FFT_THREADS, smem, s>>>(tw, sc, ld, st);
            SW_CHECK_LAUNCH();
            count_launch();
            return;
        }
    }
    auto kern = k_fft_pass<T, 0, 0, INV, LCF, SCF, LD, ST>;
    static std::atomic<int> attr_done[64] = {};
    if (dev < 64 && !attr_done[dev].load(std::memory_order_acquire)) {
        SW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        SW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        attr_done[dev].store(1, std::memory_order_release);
    }
    dim3 grid((ncols + tc - 1) / tc, nout);
    kern<<<grid, FFT_THREADS, smem, s>>>(plan, tw, ncols, ilog2(tc), make_fastdiv((uint32_t)plan.n), sc, ld, st);
    SW_CHECK_LAUNCH();
    count_launch();
}

template <typename T>
struct Fft2d {
    using T2 = typename C2<T>::t;
    int ng = 0;
    FftPlan plan{};
    DevBuf<T2> tw;
    DevBuf<T> mid;
    T* midp = nullptr;  // the intermediate: mid, or storage lent by the owner
    int cap = 0;    // planes the intermediate holds
    int chunk = 0;  // planes per pair of pass launches (<= cap)
    int tc = 2;
    T sc = 1;

    // Default chunk: the intermediate of one launch pair stays within about 40 MB,
    // a third of the 126 MB L2, so that pass B reads what pass A wrote from L2.
    static int default_chunk(int ng, int cap) {
        const size_t plane = (size_t)ng * ng * sizeof(T);
        const int c = (int)((40u << 20) / plane);
        return c < 1 ? 1 : (c > cap ? cap : c);
    }

    // lent: storage of at least cap_planes ng*ng planes of T that the caller owns
    // and never uses while a transform of this object is queued (nullptr: allocate)
    void init(int ng_, int cap_planes, T* lent = nullptr) {
        ng = ng_;
        require(build_plan(ng, plan) == SW_OK, SW_ERR_FACTORISE, "grid size must factor into 2, 3, 5");
        auto h = host_twiddles<T>(ng);
        tw.alloc(ng);
        SW_CUDA(cudaMemcpy(tw.p, h.data(), sizeof(T2) * ng, cudaMemcpyHostToDevice));
        cap = cap_planes;
        if (lent) midp = lent;
        else {
            mid.alloc((size_t)cap * ng * ng);
            midp = mid.p;
        }
        chunk = default_chunk(ng, cap);
        // n = 256: the register-staged pass (16- or 32-column tiles, one buffer)
        tc = ng == FFT_R_N ? 2 * fft_r_np<T>() : pick_tile<T>(ng);
        sc = (T)(1.0 / std::sqrt((double)ng));
    }
    // Columns per tile of the n = 256 passes: 16 or 32 (other lengths keep their
    // fixed tile); returns the value in use.
    int set_tile(int columns) {
        if (ng == FFT_R_N && (columns == 16 || columns == 32)) tc = columns;
        return tc;
    }
    // Planes per launch pair, clamped to [1, cap]; returns the value in use.
    int set_chunk(int planes) {
        chunk = planes < 1 ? 1 : (planes > cap ? cap : planes);
        return chunk;
    }

    template <class LD, class ST>
    void spctop(cudaStream_t s, int nout, LD ld, ST st) const {
        for (int o0 = 0; o0 < nout; o0 += chunk) {
            const int cnt = (nout - o0 < chunk) ? nout - o0 : chunk;
            launch_pass<T, true, true, false>(s, plan, tw.p, tc, sc, cnt, ng, LdOff<LD>{ld, o0}, MidPC<T>{midp, ng});
            launch_pass<T, true, true, true>(s, plan, tw.p, tc, sc, cnt, ng, MidCP<T>{midp, ng}, StOff<ST>{st, o0});
        }
    }
    template <class LD, class ST>
    void ptospc(cudaStream_t s, int nout, LD ld, ST st) const {
        for (int o0 = 0; o0 < nout; o0 += chunk) {
            const int cnt = (nout - o0 < chunk) ? nout - o0 : chunk;
            launch_pass<T, false, true, true>(s, plan, tw.p, tc, sc, cnt, ng, LdOff<LD>{ld, o0}, MidCP<T>{midp, ng});
            launch_pass<T, false, false, true>(s, plan, tw.p, tc, sc, cnt, ng, MidPC<T>{midp, ng}, StOff<ST>{st, o0});
        }
    }
};

// Spectral derivative helpers (D2FFT::xderiv/yderiv, src/sta2dfft.rs:128-184):
// d/dx at Hermitian index a is dmul(a) * var[mirror(a)] along that axis.
__device__ __forceinline__ int mirror(int a, int ng) { return a == 0 ? 0 : ng - a; }
__device__ __forceinline__ double dmul(int a, int ng) {
    return (a == 0 || 2 * a == ng) ? 0.0 : ((2 * a < ng) ? -(double)a : (double)(ng - a));
}
// dmul(a) * v in v's precision.  dmul is an integer of magnitude at most ng/2, so
// the float64 product with a float value is exact and rounding it once to float
// gives the float product itself: dmul_t(a, ng, v) == (T)(dmul(a, ng) * (double)v)
// bit for bit, without the conversions and the float64 multiply.
__device__ __forceinline__ int imul(int a, int ng) { return (a == 0 || 2 * a == ng) ? 0 : ((2 * a < ng) ? -a : ng - a); }
template <typename T>
__device__ __forceinline__ T dmul_t(int a, int ng, T v) {
    return (T)imul(a, ng) * v;
}
// Parseval weight of one axis for the Hermitian packing: 1 at 0 and ng/2, else 2.
__device__ __forceinline__ double pweight(int a, int ng) { return (a == 0 || 2 * a == ng) ? 1.0 : 2.0; }

}  // namespace sw
