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
#include <cooperative_groups.h>

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
// plane-bound functors of a chunk: bind to plane o0 + o
template <class F>
__device__ __forceinline__ auto bind_ld(const LdOff<PlaneLd<F>>& f, int o) {
    return bind_ld(f.f, f.o0 + o);
}
template <class F>
__device__ __forceinline__ auto bind_st(const StOff<PlaneSt<F>>& f, int o) {
    return bind_st(f.f, f.o0 + o);
}
// intermediate addressed [pt + ng*col] (point index contiguous)
template <typename T>
struct MidPC {
    T* m;
    int ng;
    __device__ __forceinline__ T operator()(int o, int c, int p) const {
        const T* a = m + ((size_t)o * ng + c) * ng + p;
        return SW_BC_OK(a, sizeof(T), sizeof(T)) ? *a : T(0);
    }
    __device__ __forceinline__ void operator()(int o, int c, int p, T v) const {
        T* a = m + ((size_t)o * ng + c) * ng + p;
        if (SW_BC_OK(a, sizeof(T), sizeof(T))) *a = v;
    }
};
// intermediate addressed [col + ng*pt] (column index contiguous); columns
// (c, c+1), c even, are one aligned vector access
template <typename T>
struct MidCP {
    using T2 = typename C2<T>::t;
    static constexpr bool pair_io = true;
    T* m;
    int ng;
    __device__ __forceinline__ T operator()(int o, int c, int p) const {
        const T* a = m + ((size_t)o * ng + p) * ng + c;
        return SW_BC_OK(a, sizeof(T), sizeof(T)) ? *a : T(0);
    }
    __device__ __forceinline__ void operator()(int o, int c, int p, T v) const {
        T* a = m + ((size_t)o * ng + p) * ng + c;
        if (SW_BC_OK(a, sizeof(T), sizeof(T))) *a = v;
    }
    __device__ __forceinline__ T2 ld2(int o, int c, int p) const {
        const T* a = m + ((size_t)o * ng + p) * ng + c;
        if (!SW_BC_OK(a, sizeof(T2), sizeof(T2))) return T2{};
        return *reinterpret_cast<const T2*>(a);
    }
    __device__ __forceinline__ void st2(int o, int c, int p, T a, T b) const {
        T2 v;
        v.x = a;
        v.y = b;
        T* d = m + ((size_t)o * ng + p) * ng + c;
        if (SW_BC_OK(d, sizeof(T2), sizeof(T2))) *reinterpret_cast<T2*>(d) = v;
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

// ---------------------------------------------------------------------------
// Single-pass 2-D transform of n = 256 planes on thread-block clusters.
//
// A cluster of FFT2D_CL = 8 CTAs holds one plane: CTA r transforms columns
// 32 r .. 32 r + 31 along the first axis (phase 1, the first pass of the two-pass
// transform), leaving its 32 x 256 result in its own shared memory (E).  After a
// cluster barrier, CTA r reads the 32 columns of the second axis that it owns
// straight from the eight CTAs' E through distributed shared memory and
// transforms them (phase 2, the second pass).  Each plane is read from and
// written to global memory once; the transposed intermediate of the two-pass
// transform never leaves the cluster.  E shares the tile buffer: phase 1 writes it
// after its last read of the buffer (before_store), and phase 2 reuses the buffer
// only after a second cluster barrier has seen every CTA's reads of E finish
// (after_load).  Arithmetic and operation order per 1-D transform are those of the
// register-staged pass, so results equal the two-pass transform's bit for bit.
//   ptospc: phase 1 forward along ix for iy columns; E_r[kx][iy - 32 r];
//           phase 2 forward along iy for kx columns
//   spctop: phase 1 reverse along ky for kx columns; E_r[kx - 32 r][iy];
//           phase 2 reverse along kx for iy columns
// ---------------------------------------------------------------------------
constexpr int FFT2D_CL = 8;                // CTAs per cluster (portable cluster size)
constexpr int FFT2D_NP = FFT_R_N / FFT2D_CL / 2;  // column pairs per CTA (16: 256 threads)
template <typename T>
__host__ __device__ constexpr int fft2d_cl_minb() { return sizeof(T) == 8 ? 2 : 4; }
template <typename T>
inline size_t fft2d_cl_smem() {
    return sizeof(typename C2<T>::t) * ((size_t)64 + (size_t)FFT2D_NP * FFT_R_PL);
}

// E of a forward transform: [kx (256)][iy - c0 (32)]
template <typename T>
struct ClFwdStore {  // phase 1: column iy (c0 .. c0+31), mode kx
    using T2 = typename C2<T>::t;
    static constexpr bool pair_io = true;
    T* e;
    int c0;
    __device__ __forceinline__ void operator()(int, int c, int k, T v) const { e[k * 32 + (c - c0)] = v; }
    __device__ __forceinline__ void st2(int, int c, int k, T a, T b) const {
        T2 v;
        v.x = a;
        v.y = b;
        *reinterpret_cast<T2*>(e + k * 32 + (c - c0)) = v;
    }
};
template <typename T>
struct ClFwdLoad {  // phase 2: column kx, point iy, from CTA iy / 32
    using T2 = typename C2<T>::t;
    static constexpr bool pair_io = true;
    T* e;  // this CTA's E (mapped to the owner's with map_shared_rank)
    __device__ __forceinline__ T operator()(int, int c, int j) const {
        const T* src = cooperative_groups::this_cluster().map_shared_rank(e, (unsigned)(j >> 5));
        return src[c * 32 + (j & 31)];
    }
    __device__ __forceinline__ T2 ld2(int, int c, int j) const {
        const T* src = cooperative_groups::this_cluster().map_shared_rank(e, (unsigned)(j >> 5));
        T2 v;
        v.x = src[c * 32 + (j & 31)];
        v.y = src[(c + 1) * 32 + (j & 31)];
        return v;
    }
};
// E of a reverse transform: [kx - c0 (32)][iy (256)]
template <typename T>
struct ClRevStore {  // phase 1: column kx (c0 .. c0+31), point iy
    static constexpr bool pair_io = true;
    T* e;
    int c0;
    __device__ __forceinline__ void operator()(int, int c, int p, T v) const { e[(c - c0) * 256 + p] = v; }
    __device__ __forceinline__ void st2(int, int c, int p, T a, T b) const {
        e[(c - c0) * 256 + p] = a;
        e[(c + 1 - c0) * 256 + p] = b;
    }
};
template <typename T>
struct ClRevLoad {  // phase 2: column iy, point kx, from CTA kx / 32
    using T2 = typename C2<T>::t;
    static constexpr bool pair_io = true;
    T* e;
    __device__ __forceinline__ T operator()(int, int c, int p) const {
        const T* src = cooperative_groups::this_cluster().map_shared_rank(e, (unsigned)(p >> 5));
        return src[(p & 31) * 256 + c];
    }
    __device__ __forceinline__ T2 ld2(int, int c, int p) const {
        const T* src = cooperative_groups::this_cluster().map_shared_rank(e, (unsigned)(p >> 5));
        return *reinterpret_cast<const T2*>(src + (p & 31) * 256 + c);
    }
};
// Phase 1 writes E into the tile buffer it has just read: all reads first.
struct SyncBeforeStore {
    __device__ __forceinline__ void after_load() const {}
    __device__ __forceinline__ void before_store() const { __syncthreads(); }
};
// Phase 2 has read E of every CTA into registers: wait for the whole cluster
// before the tile buffer (which is E) is written again.
struct ClusterAfterLoad {
    __device__ __forceinline__ void after_load() const { cooperative_groups::this_cluster().sync(); }
    __device__ __forceinline__ void before_store() const {}
};

template <typename T, bool INV, class LD, class ST>
__global__ void __cluster_dims__(FFT2D_CL, 1, 1) __launch_bounds__(16 * FFT2D_NP, fft2d_cl_minb<T>())
k_fft2d_cluster(const typename C2<T>::t* __restrict__ twg, T sc, LD ld, ST st) {
    using T2 = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* tw = reinterpret_cast<T2*>(smem_raw);
    T2* buf = tw + 64;
    T* e = reinterpret_cast<T*>(buf);
    const int r = (int)cooperative_groups::this_cluster().block_rank();
    const int o = blockIdx.y, c0 = 32 * r;
    load_tw64(tw, twg);
    if constexpr (!INV) {
        fft_r_tile<T, FFT2D_NP, false, true, true>(tw, buf, sc, ld, ClFwdStore<T>{e, c0}, o, c0, SyncBeforeStore{});
        cooperative_groups::this_cluster().sync();
        fft_r_tile<T, FFT2D_NP, false, false, true>(tw, buf, sc, ClFwdLoad<T>{e}, st, o, c0, ClusterAfterLoad{});
    } else {
        fft_r_tile<T, FFT2D_NP, true, true, false>(tw, buf, sc, ld, ClRevStore<T>{e, c0}, o, c0, SyncBeforeStore{});
        cooperative_groups::this_cluster().sync();
        fft_r_tile<T, FFT2D_NP, true, true, true>(tw, buf, sc, ClRevLoad<T>{e}, st, o, c0, ClusterAfterLoad{});
    }
}

// nout planes of n = 256, one cluster of FFT2D_CL CTAs per plane.
template <typename T, bool INV, class LD, class ST>
inline void launch_fft2d_cluster(cudaStream_t s, const typename C2<T>::t* tw, T sc, int nout, LD ld, ST st) {
    if (nout <= 0) return;
    auto kern = k_fft2d_cluster<T, INV, LD, ST>;
    int dev = 0;
    cudaGetDevice(&dev);
    static std::atomic<int> attr[64] = {};
    if (dev < 64 && !attr[dev].load(std::memory_order_acquire)) {
        SW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fft2d_cl_smem<T>()));
        SW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        attr[dev].store(1, std::memory_order_release);
    }
    dim3 grid(FFT2D_CL, nout);
    kern<<<grid, 16 * FFT2D_NP, fft2d_cl_smem<T>(), s>>>(tw, sc, ld, st);
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
    // n = 256: one single-pass cluster launch per transform batch (k_fft2d_cluster)
    // instead of two tile passes through the intermediate
    bool single_pass = false;
    // Two-stream chunk pipeline: chunks alternate between the caller's stream and
    // s2 with two intermediates, so that one chunk's second pass overlaps the next
    // chunk's first pass and small chunks keep their intermediate in L2.
    bool overlap = false;
    cudaStream_t s2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    ~Fft2d() {
        if (s2) cudaStreamDestroy(s2);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
    }
    // On: needs the intermediate to hold two chunks (the chunk is clamped to cap/2).
    bool set_overlap(bool on) {
        if (on && !s2) {
            SW_CUDA(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
            SW_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
            SW_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        }
        overlap = on && cap >= 2;
        if (overlap && chunk > cap / 2) chunk = cap / 2;
        return overlap;
    }

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
        single_pass = false;  // measured slower than the two passes so far; opt in with set_single_pass
    }
    // Single-pass transforms on (n = 256 only); returns the setting in use.
    bool set_single_pass(bool on) {
        single_pass = on && ng == FFT_R_N;
        return single_pass;
    }
    // Columns per tile of the n = 256 passes: 16 or 32 (other lengths keep their
    // fixed tile); returns the value in use.
    int set_tile(int columns) {
        if (ng == FFT_R_N && (columns == 16 || columns == 32)) tc = columns;
        return tc;
    }
    // Planes per launch pair, clamped to [1, cap] (cap/2 with the two-stream
    // pipeline); returns the value in use.
    int set_chunk(int planes) {
        const int mx = overlap ? cap / 2 : cap;
        chunk = planes < 1 ? 1 : (planes > mx ? mx : planes);
        return chunk;
    }

    template <class LD, class ST>
    void spctop(cudaStream_t s, int nout, LD ld, ST st) const {
        if (single_pass) {
            launch_fft2d_cluster<T, true>(s, tw.p, sc, nout, ld, st);
            return;
        }
        const bool two = overlap && nout > chunk && can_fork(s);
        if (two) fork(s);
        for (int o0 = 0, k = 0; o0 < nout; o0 += chunk, k++) {
            const int cnt = (nout - o0 < chunk) ? nout - o0 : chunk;
            cudaStream_t sk = (two && (k & 1)) ? s2 : s;
            T* m = midp + ((two && (k & 1)) ? (size_t)chunk * ng * ng : 0);
            launch_pass<T, true, true, false>(sk, plan, tw.p, tc, sc, cnt, ng, LdOff<LD>{ld, o0}, MidPC<T>{m, ng});
            launch_pass<T, true, true, true>(sk, plan, tw.p, tc, sc, cnt, ng, MidCP<T>{m, ng}, StOff<ST>{st, o0});
        }
        if (two) join(s);
    }
    // s2 can take chunks of work queued on s unless s2 already belongs to another
    // stream capture than s's (it stays a member of a capture it joined until that
    // capture ends, and a conditional node's body is captured as a capture of its
    // own): then the chunks run on s alone.
    bool can_fork(cudaStream_t s) const {
        cudaStreamCaptureStatus a = cudaStreamCaptureStatusNone, b = cudaStreamCaptureStatusNone;
        unsigned long long ia = 0, ib = 0;
        SW_CUDA(cudaStreamGetCaptureInfo(s, &a, &ia));
        SW_CUDA(cudaStreamGetCaptureInfo(s2, &b, &ib));
        if (b == cudaStreamCaptureStatusNone) return true;
        return a == cudaStreamCaptureStatusActive && ia == ib;
    }
    void fork(cudaStream_t s) const {
        SW_CUDA(cudaEventRecord(ev_fork, s));
        SW_CUDA(cudaStreamWaitEvent(s2, ev_fork, 0));
    }
    void join(cudaStream_t s) const {
        SW_CUDA(cudaEventRecord(ev_join, s2));
        SW_CUDA(cudaStreamWaitEvent(s, ev_join, 0));
    }
    template <class LD, class ST>
    void ptospc(cudaStream_t s, int nout, LD ld, ST st) const {
        if (single_pass) {
            launch_fft2d_cluster<T, false>(s, tw.p, sc, nout, ld, st);
            return;
        }
        const bool two = overlap && nout > chunk && can_fork(s);
        if (two) fork(s);
        for (int o0 = 0, k = 0; o0 < nout; o0 += chunk, k++) {
            const int cnt = (nout - o0 < chunk) ? nout - o0 : chunk;
            cudaStream_t sk = (two && (k & 1)) ? s2 : s;
            T* m = midp + ((two && (k & 1)) ? (size_t)chunk * ng * ng : 0);
            launch_pass<T, false, true, true>(sk, plan, tw.p, tc, sc, cnt, ng, LdOff<LD>{ld, o0}, MidCP<T>{m, ng});
            launch_pass<T, false, false, true>(sk, plan, tw.p, tc, sc, cnt, ng, MidPC<T>{m, ng}, StOff<ST>{st, o0});
        }
        if (two) join(s);
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
// Plane-bound access to one spectral plane s ([kx + ng*ky], Hermitian-packed) at
// the kx pair (kx, kx + 1), kx even: kind 0 the values, 1 d/dx, 2 d/dy, with the
// products of dmul_t (so equal to the per-element functors' results).
template <typename T>
__device__ __forceinline__ typename C2<T>::t spec_pair(const T* s, int kind, int kx, int ky, int ng) {
    if (kind == 0) return ldv2(s + kx + ng * ky);
    if (kind == 1)
        return mk2(dmul_t(kx, ng, s[mirror(kx, ng) + ng * ky]), dmul_t(kx + 1, ng, s[mirror(kx + 1, ng) + ng * ky]));
    const auto v = ldv2(s + kx + ng * mirror(ky, ng));
    return mk2(dmul_t(ky, ng, v.x), dmul_t(ky, ng, v.y));
}
// Accessors of one plane ([col + ng*pt]) for plane-bound functors: plain values,
// plain stores, and stores of the product with a float64 operator table (the
// dealiasing filter, glap) rounded to T, as (T)(op[i] * (double)v).
template <typename T>
struct PairLd {
    const T* s;
    int ng;
    __device__ __forceinline__ typename C2<T>::t operator()(int c, int p) const { return ldv2(s + c + ng * p); }
};
template <typename T>
struct PairSt {
    T* d;
    int ng;
    __device__ __forceinline__ void operator()(int c, int p, T a, T b, int m) const { stv2m(d + c + ng * p, m, a, b); }
};
template <typename T>
struct PairStOp {
    T* d;
    const double* op;
    int ng;
    __device__ __forceinline__ void operator()(int c, int p, T a, T b, int m) const {
        const int i = c + ng * p;
        const double2 f = ldv2_ro(op + i);
        stv2m(d + i, m, (T)(f.x * (double)a), (T)(f.y * (double)b));
    }
};
// Parseval weight of one axis for the Hermitian packing: 1 at 0 and ng/2, else 2.
__device__ __forceinline__ double pweight(int a, int ng) { return (a == 0 || 2 * a == ng) ? 1.0 : 2.0; }

}  // namespace sw
