// Batched mixed-radix real FFTs in the stafft Hermitian convention, for sm_100a.
//
// Convention (reference src/stafft/mod.rs:158-452): a length-n real vector x
// maps to H with H[k] = Re F_k / sqrt(n) for 0 <= k <= n/2 and
// H[n-k] = Im F_k / sqrt(n) for 1 <= k <= (n-1)/2, where F is the
// e^{-2 pi i jk/n} DFT; the reverse transform is its exact inverse.
//
// Engine: one CTA transforms a tile of `tc` real columns of one plane.  Columns
// are paired into complex sequences z = x_{2p} + i x_{2p+1}, transformed in
// shared memory by a Stockham autosort FFT (radix 4, 2, 3, 5; natural order in
// and out, ping-pong buffers), and unpacked into Hermitian form on the way out
// (forward) or packed from it on the way in (reverse).  Global loads and stores
// go through caller functors, so products, derivatives, filters and linear
// combinations are fused into the transform passes:
//   ld(o, col, pt) -> T          value of column `col`, point `pt` of output o
//   st(o, col, pt, T value)      result for column `col`, point/mode `pt`
// LOAD_CF / STORE_CF choose whether consecutive threads walk the column index
// (true) or the point index (false), so that whichever index is contiguous in
// memory is the one the warp spans (coalesced 128-byte segments).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "sw_bc.cuh"

namespace sw {

template <typename T> struct C2;
template <> struct C2<double> { using t = double2; };
template <> struct C2<float> { using t = float2; };

constexpr int FFT_MAX_RAD = 24;
constexpr int FFT_THREADS = 256;

// Exact quotient x / d for x, d < 2^16 by multiply-high with m = ceil(2^32 / d).
struct FastDiv {
    uint32_t d, m;
};
inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f;
    f.d = d;
    f.m = (uint32_t)((((uint64_t)1 << 32) + d - 1) / d);
    return f;
}
__device__ __forceinline__ uint32_t fdiv(uint32_t x, FastDiv f) { return f.d == 1 ? x : __umulhi(x, f.m); }

struct FftStage {
    int R, Ns, nR, tstride;
    FastDiv dNs, dnR;
};

struct FftPlan {
    int n;
    int nrad;
    int rad[FFT_MAX_RAD];
    FftStage stg[FFT_MAX_RAD];
};

// Shared-memory index of element i of a sequence: one pad slot per 16 entries
// keeps the strided stores of the first radix-8/16 stage free of bank conflicts.
__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }
__host__ __device__ inline int padded_len(int n) { return n + (n >> 4) + 1; }

template <typename T2>
__device__ __forceinline__ T2 cmul(T2 a, T2 b) {
    T2 r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

// v * exp(s 2 pi i j / 16), s = -1 forward, +1 inverse; j is a compile-time constant.
template <int J, bool INV, typename T2>
__device__ __forceinline__ T2 tw16(T2 v) {
    using T = decltype(v.x);
    constexpr int j = J & 15;
    if constexpr (j == 0) return v;
    // cos and sin of 2 pi j / 16 for j = 0..15
    constexpr double C[16] = {1.0, 0.92387953251128675613, 0.70710678118654752440, 0.38268343236508977173,
                              0.0, -0.38268343236508977173, -0.70710678118654752440, -0.92387953251128675613,
                              -1.0, -0.92387953251128675613, -0.70710678118654752440, -0.38268343236508977173,
                              0.0, 0.38268343236508977173, 0.70710678118654752440, 0.92387953251128675613};
    constexpr double S[16] = {0.0, 0.38268343236508977173, 0.70710678118654752440, 0.92387953251128675613,
                              1.0, 0.92387953251128675613, 0.70710678118654752440, 0.38268343236508977173,
                              0.0, -0.38268343236508977173, -0.70710678118654752440, -0.92387953251128675613,
                              -1.0, -0.92387953251128675613, -0.70710678118654752440, -0.38268343236508977173};
    const T c = (T)C[j];
    const T sn = INV ? (T)S[j] : (T)(-S[j]);
    T2 r;
    if constexpr (j == 4) {  // multiply by s*i
        r.x = -sn * v.y; r.y = sn * v.x;
    } else if constexpr (j == 8) {
        r.x = -v.x; r.y = -v.y;
    } else if constexpr (j == 12) {
        r.x = -sn * v.y; r.y = sn * v.x;
    } else {
        r.x = v.x * c - v.y * sn;
        r.y = v.x * sn + v.y * c;
    }
    return r;
}

// In-register DFT of size R, sign -1 (forward) or +1 (INV), natural order in/out.
template <int R, bool INV, typename T2>
__device__ __forceinline__ void butterfly(T2* v) {
    using T = decltype(v[0].x);
    const T s = INV ? T(1) : T(-1);
    if constexpr (R == 2) {
        T2 a = v[0], b = v[1];
        v[0].x = a.x + b.x; v[0].y = a.y + b.y;
        v[1].x = a.x - b.x; v[1].y = a.y - b.y;
    } else if constexpr (R == 4) {
        T t0r = v[0].x + v[2].x, t0i = v[0].y + v[2].y;
        T t1r = v[0].x - v[2].x, t1i = v[0].y - v[2].y;
        T t2r = v[1].x + v[3].x, t2i = v[1].y + v[3].y;
        T t3r = v[1].x - v[3].x, t3i = v[1].y - v[3].y;
        T ur = -s * t3i, ui = s * t3r;  // (s*i) * t3
        v[0].x = t0r + t2r; v[0].y = t0i + t2i;
        v[1].x = t1r + ur;  v[1].y = t1i + ui;
        v[2].x = t0r - t2r; v[2].y = t0i - t2i;
        v[3].x = t1r - ur;  v[3].y = t1i - ui;
    } else if constexpr (R == 3) {
        const T s3 = T(0.86602540378443864676);
        T tr = v[1].x + v[2].x, ti = v[1].y + v[2].y;
        T mr = v[0].x - T(0.5) * tr, mi = v[0].y - T(0.5) * ti;
        T dr = s * s3 * (v[1].x - v[2].x), di = s * s3 * (v[1].y - v[2].y);
        v[0].x = v[0].x + tr; v[0].y = v[0].y + ti;
        v[1].x = mr - di; v[1].y = mi + dr;
        v[2].x = mr + di; v[2].y = mi - dr;
    } else if constexpr (R == 5) {
        const T c51 = T(0.30901699437494742410), c52 = T(-0.80901699437494742410);
        const T s51 = T(0.95105651629515357212), s52 = T(0.58778525229247312917);
        T a1r = v[1].x + v[4].x, a1i = v[1].y + v[4].y;
        T b1r = v[1].x - v[4].x, b1i = v[1].y - v[4].y;
        T a2r = v[2].x + v[3].x, a2i = v[2].y + v[3].y;
        T b2r = v[2].x - v[3].x, b2i = v[2].y - v[3].y;
        T p1r = v[0].x + c51 * a1r + c52 * a2r, p1i = v[0].y + c51 * a1i + c52 * a2i;
        T p2r = v[0].x + c52 * a1r + c51 * a2r, p2i = v[0].y + c52 * a1i + c51 * a2i;
        T q1r = s * (s51 * b1r + s52 * b2r), q1i = s * (s51 * b1i + s52 * b2i);
        T q2r = s * (s52 * b1r - s51 * b2r), q2i = s * (s52 * b1i - s51 * b2i);
        v[0].x = v[0].x + a1r + a2r; v[0].y = v[0].y + a1i + a2i;
        v[1].x = p1r - q1i; v[1].y = p1i + q1r;
        v[4].x = p1r + q1i; v[4].y = p1i - q1r;
        v[2].x = p2r - q2i; v[2].y = p2i + q2r;
        v[3].x = p2r + q2i; v[3].y = p2i - q2r;
    } else if constexpr (R == 8) {
        // radix-2 decimation in frequency, then two DFT-4
        T2 a[4], b[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            a[k].x = v[k].x + v[k + 4].x; a[k].y = v[k].y + v[k + 4].y;
            b[k].x = v[k].x - v[k + 4].x; b[k].y = v[k].y - v[k + 4].y;
        }
        b[1] = tw16<2, INV>(b[1]);
        b[2] = tw16<4, INV>(b[2]);
        b[3] = tw16<6, INV>(b[3]);
        butterfly<4, INV>(a);
        butterfly<4, INV>(b);
#pragma unroll
        for (int m = 0; m < 4; m++) { v[2 * m] = a[m]; v[2 * m + 1] = b[m]; }
    } else {  // R == 16: X[q + 4m] = sum_k W4^{km} W16^{kq} sum_p v[k + 4p] W4^{pq}
        T2 g[4][4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
#pragma unroll
            for (int p = 0; p < 4; p++) g[k][p] = v[k + 4 * p];
            butterfly<4, INV>(g[k]);
        }
        g[1][1] = tw16<1, INV>(g[1][1]); g[1][2] = tw16<2, INV>(g[1][2]); g[1][3] = tw16<3, INV>(g[1][3]);
        g[2][1] = tw16<2, INV>(g[2][1]); g[2][2] = tw16<4, INV>(g[2][2]); g[2][3] = tw16<6, INV>(g[2][3]);
        g[3][1] = tw16<3, INV>(g[3][1]); g[3][2] = tw16<6, INV>(g[3][2]); g[3][3] = tw16<9, INV>(g[3][3]);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            T2 h[4] = {g[0][q], g[1][q], g[2][q], g[3][q]};
            butterfly<4, INV>(h);
#pragma unroll
            for (int m = 0; m < 4; m++) v[q + 4 * m] = h[m];
        }
    }
}

// One Stockham pass of radix R over np sequences (padded, stride pl) in x -> y.
template <int R, bool INV, typename T2>
__device__ __forceinline__ void stockham_stage(const T2* __restrict__ x, T2* __restrict__ y,
                                               const T2* __restrict__ tw, const FftStage& sg, int np, int pl) {
    const int nR = sg.nR;
    for (int b = threadIdx.x; b < np * nR; b += blockDim.x) {
        const int p = (int)fdiv((uint32_t)b, sg.dnR);
        const int j = b - p * nR;
        const int jq = (int)fdiv((uint32_t)j, sg.dNs);
        const int k = j - jq * sg.Ns;
        const int base = jq * sg.Ns * R + k;
        const T2* xp = x + p * pl;
        T2* yp = y + p * pl;
        T2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = xp[pad16(j + r * nR)];
        if (sg.Ns > 1) {
            const int step = k * sg.tstride;
#pragma unroll
            for (int r = 1; r < R; r++) {
                T2 w = tw[r * step];
                if (INV) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        butterfly<R, INV>(v);
#pragma unroll
        for (int r = 0; r < R; r++) yp[pad16(base + r * sg.Ns)] = v[r];
    }
}

// Stockham pass with compile-time length, radix and stride (all index math
// reduces to shifts and masks for power-of-two lengths).
template <int R, int N, int NS, bool INV, typename T2>
__device__ __forceinline__ void stockham_stage_s(const T2* __restrict__ x, T2* __restrict__ y,
                                                 const T2* __restrict__ tw, int np, int pl) {
    constexpr int nR = N / R;
    constexpr int tstride = N / (NS * R);
    for (int b = threadIdx.x; b < np * nR; b += FFT_THREADS) {
        const int p = b / nR;
        const int j = b % nR;
        const int k = j % NS;
        const int base = (j / NS) * NS * R + k;
        const T2* xp = x + p * pl;
        T2* yp = y + p * pl;
        T2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = xp[pad16(j + r * nR)];
        if constexpr (NS > 1) {
            const int step = k * tstride;
#pragma unroll
            for (int r = 1; r < R; r++) {
                T2 w = tw[r * step];
                if (INV) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        butterfly<R, INV>(v);
#pragma unroll
        for (int r = 0; r < R; r++) yp[pad16(base + r * NS)] = v[r];
    }
}

// Compile-time plans of the specialised lengths: 256 = 16 x 16, 128 = 16 x 8.
template <int N, bool INV, typename T2>
__device__ __forceinline__ T2* smem_fft_static(T2* a, T2* b, const T2* tw, int np, int pl) {
    if constexpr (N == 256) {
        stockham_stage_s<16, 256, 1, INV>(a, b, tw, np, pl);
        __syncthreads();
        stockham_stage_s<16, 256, 16, INV>(b, a, tw, np, pl);
        __syncthreads();
        return a;
    } else {
        static_assert(N == 128, "specialised lengths: 128, 256");
        stockham_stage_s<16, 128, 1, INV>(a, b, tw, np, pl);
        __syncthreads();
        stockham_stage_s<8, 128, 16, INV>(b, a, tw, np, pl);
        __syncthreads();
        return a;
    }
}

// Full transform of np sequences; returns the buffer holding the result.
template <bool INV, typename T2>
__device__ T2* smem_fft(const FftPlan& plan, T2* a, T2* b, const T2* tw, int np, int pl) {
    for (int s = 0; s < plan.nrad; s++) {
        const FftStage& sg = plan.stg[s];
        switch (sg.R) {
            case 16: stockham_stage<16, INV>(a, b, tw, sg, np, pl); break;
            case 8: stockham_stage<8, INV>(a, b, tw, sg, np, pl); break;
            case 4: stockham_stage<4, INV>(a, b, tw, sg, np, pl); break;
            case 2: stockham_stage<2, INV>(a, b, tw, sg, np, pl); break;
            case 3: stockham_stage<3, INV>(a, b, tw, sg, np, pl); break;
            default: stockham_stage<5, INV>(a, b, tw, sg, np, pl); break;
        }
        __syncthreads();
        T2* t = a;
        a = b;
        b = t;
    }
    return a;
}

// Shared memory bytes of one pass: twiddles (n) + two tiles (tc/2 * n each).
// Functors that tag `static constexpr bool pair_io = true` provide
// ld2(o, col, pt) -> T2 and st2(o, col, pt, a, b) for the adjacent columns
// (col, col+1), col even; others get two scalar calls.
template <class F, class = void>
struct pair_io : std::false_type {};
template <class F>
struct pair_io<F, std::void_t<decltype(F::pair_io)>> : std::integral_constant<bool, F::pair_io> {};

template <typename T, class LD>
__device__ __forceinline__ void ld_pair(const LD& ld, int o, int col, int j, T& a, T& b) {
    if constexpr (pair_io<LD>::value) {
        const auto v = ld.ld2(o, col, j);
        a = v.x;
        b = v.y;
    } else {
        a = (T)ld(o, col, j);
        b = (T)ld(o, col + 1, j);
    }
}
template <typename T, class ST>
__device__ __forceinline__ void st_pair(const ST& st, int o, int col, int k, T a, T b) {
    if constexpr (pair_io<ST>::value) {
        st.st2(o, col, k, a, b);
    } else {
        st(o, col, k, a);
        st(o, col + 1, k, b);
    }
}

// Plane-bound functors.  A tile pass works on one plane o, so a functor that picks
// its source or destination by o (which field, which level, which derivative) can
// do that once per tile instead of once per element.  plane_ld(f) / plane_st(f)
// wrap a callable f(o) that returns the accessor of plane o:
//   loads:  g(col, pt) -> T2        the values of columns col and col + 1 (col even)
//   stores: g(col, pt, a, b, m)     a to column col if m & 1, b to col + 1 if m & 2
// Every pass binds its functors once per tile (bind_ld / bind_st); a functor of
// the per-element form (ld(o, col, pt), st(o, col, pt, v)) binds to itself.
template <class F>
struct PlaneLd {
    F f;
};
template <class F>
struct PlaneSt {
    F f;
};
template <class F>
inline PlaneLd<F> plane_ld(F f) {
    return PlaneLd<F>{f};
}
template <class F>
inline PlaneSt<F> plane_st(F f) {
    return PlaneSt<F>{f};
}
template <class G>
struct BoundLd {
    G g;
};
template <class G>
struct BoundSt {
    G g;
};
template <class LD>
__device__ __forceinline__ const LD& bind_ld(const LD& f, int) {
    return f;
}
template <class ST>
__device__ __forceinline__ const ST& bind_st(const ST& f, int) {
    return f;
}
template <class F>
__device__ __forceinline__ auto bind_ld(const PlaneLd<F>& f, int o) {
    return BoundLd<decltype(f.f(o))>{f.f(o)};
}
template <class F>
__device__ __forceinline__ auto bind_st(const PlaneSt<F>& f, int o) {
    return BoundSt<decltype(f.f(o))>{f.f(o)};
}
template <typename T, class G>
__device__ __forceinline__ void ld_pair(const BoundLd<G>& b, int, int col, int j, T& x, T& y) {
    const auto v = b.g(col, j);
    x = (T)v.x;
    y = (T)v.y;
}
template <typename T, class G>
__device__ __forceinline__ void st_pair(const BoundSt<G>& b, int, int col, int k, T x, T y) {
    b.g(col, k, x, y, 3);
}
// Single elements (the generic pass): a bound load reads the pair and keeps one
// value; a bound store writes one column of the pair.
template <typename T, class LD>
__device__ __forceinline__ T ld_one(const LD& ld, int o, int col, int j) {
    return (T)ld(o, col, j);
}
template <typename T, class G>
__device__ __forceinline__ T ld_one(const BoundLd<G>& b, int, int col, int j) {
    const auto v = b.g(col & ~1, j);
    return (col & 1) ? (T)v.y : (T)v.x;
}
template <typename T, class ST>
__device__ __forceinline__ void st_one(const ST& st, int o, int col, int k, T v) {
    st(o, col, k, v);
}
template <typename T, class G>
__device__ __forceinline__ void st_one(const BoundSt<G>& b, int, int col, int k, T v) {
    if (col & 1) b.g(col - 1, k, v, v, 2);
    else b.g(col, k, v, v, 1);
}
// Accessor helpers for plane-bound functors: the pair (p[0], p[1]) of an even
// index as one vector access, and a masked pair store.
template <typename T>
__device__ __forceinline__ typename C2<T>::t ldv2(const T* p) {
    if (!SW_BC_OK(p, 2 * sizeof(T), 2 * sizeof(T))) return typename C2<T>::t{};
    return *reinterpret_cast<const typename C2<T>::t*>(p);
}
template <typename T>
__device__ __forceinline__ typename C2<T>::t ldv2_ro(const T* p) {
    if (!SW_BC_OK(p, 2 * sizeof(T), 2 * sizeof(T))) return typename C2<T>::t{};
    return __ldg(reinterpret_cast<const typename C2<T>::t*>(p));
}
template <typename T>
__device__ __forceinline__ typename C2<T>::t mk2(T a, T b) {
    typename C2<T>::t v;
    v.x = a;
    v.y = b;
    return v;
}
template <typename T>
__device__ __forceinline__ void stv2m(T* p, int m, T a, T b) {
    if (m == 3) {
        if (SW_BC_OK(p, 2 * sizeof(T), 2 * sizeof(T))) *reinterpret_cast<typename C2<T>::t*>(p) = mk2(a, b);
    } else if (m == 1) {
        if (SW_BC_OK(p, sizeof(T), sizeof(T))) p[0] = a;
    } else {
        if (SW_BC_OK(p + 1, sizeof(T), sizeof(T))) p[1] = b;
    }
}

template <typename T>
inline size_t fft_pass_smem(int n, int tc) {
    return sizeof(typename C2<T>::t) * ((size_t)n + (size_t)tc * padded_len(n));
}

// Generic tile pass.  grid.x = column tiles, grid.y = output index o.
// tc (columns per tile) is a power of two, 1 << ltc.  Loads are issued in
// unrolled groups of FFT_UNROLL per thread so that many global reads are in
// flight before the tile is written to shared memory.
constexpr int FFT_UNROLL = 8;

// NS, LTCS: 0 for the general kernel (length and tile from the plan and ltc),
// otherwise a compile-time length (128 or 256) and log2 of its tile width, so
// that loop bounds and index arithmetic fold to constants.
template <typename T, int NS, int LTCS, bool INV, bool LOAD_CF, bool STORE_CF, class LD, class ST>
__global__ void __launch_bounds__(FFT_THREADS, 3)
k_fft_pass(FftPlan plan, const typename C2<T>::t* __restrict__ twg, int ncols, int ltc_rt, FastDiv dn, T sc, LD ld,
           ST st) {
    using T2 = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = NS ? NS : plan.n;
    const int ltc = NS ? LTCS : ltc_rt;
    const int tc = 1 << ltc;
    const int np = tc >> 1;
    const int pl = padded_len(n);
    T2* tw = reinterpret_cast<T2*>(smem_raw);
    T2* buf0 = tw + n;
    T2* buf1 = buf0 + (size_t)np * pl;
    const int o = blockIdx.y;
    const int c0 = blockIdx.x * tc;
    const int nthr = NS ? FFT_THREADS : (int)blockDim.x;
    const auto& ldb = bind_ld(ld, o);
    const auto& stb = bind_st(st, o);
    const int total = tc * n;

    for (int i = threadIdx.x; i < n; i += nthr) tw[i] = twg[i];
    T* rb = reinterpret_cast<T*>(buf0);
    for (int base = 0; base < total; base += nthr * FFT_UNROLL) {
        T vals[FFT_UNROLL];
#pragma unroll
        for (int u = 0; u < FFT_UNROLL; u++) {
            const int idx = base + u * nthr + threadIdx.x;
            int c, j;
            if (LOAD_CF) { c = idx & (tc - 1); j = idx >> ltc; }
            else if (NS) { j = idx % n; c = idx / n; }
            else         { j = (int)((uint32_t)idx - fdiv((uint32_t)idx, dn) * (uint32_t)n); c = (int)fdiv((uint32_t)idx, dn); }
            const int col = c0 + c;
            vals[u] = (idx < total && col < ncols) ? ld_one<T>(ldb, o, col, j) : T(0);
        }
#pragma unroll
        for (int u = 0; u < FFT_UNROLL; u++) {
            const int idx = base + u * nthr + threadIdx.x;
            if (idx < total) {
                int c, j;
                if (LOAD_CF) { c = idx & (tc - 1); j = idx >> ltc; }
                else if (NS) { c = idx / n; j = idx % n; }
                else         { c = (int)fdiv((uint32_t)idx, dn); j = idx - c * n; }
                rb[(((c >> 1) * pl + pad16(j)) << 1) + (c & 1)] = vals[u];
            }
        }
    }
    __syncthreads();
    if (INV) {
        // pack Hermitian column pairs (Ha, Hb) into Z = A + iB
        const int kh = (n - 1) / 2;
        for (int idx = threadIdx.x; idx < np * kh; idx += nthr) {
            const int p = idx / kh;
            const int k = 1 + idx - p * kh;
            T2* z = buf0 + p * pl;
            T2 lo = z[pad16(k)], hi = z[pad16(n - k)];  // lo = (Ha[k], Hb[k]), hi = (Ha[n-k], Hb[n-k])
            T2 zk, znk;
            zk.x = lo.x - hi.y;  zk.y = hi.x + lo.y;
            znk.x = lo.x + hi.y; znk.y = lo.y - hi.x;
            z[pad16(k)] = zk;
            z[pad16(n - k)] = znk;
        }
        __syncthreads();
    }
    const T2* Z;
    if constexpr (NS != 0) Z = smem_fft_static<NS, INV>(buf0, buf1, tw, np, pl);
    else Z = smem_fft<INV>(plan, buf0, buf1, tw, np, pl);
#pragma unroll 4
    for (int idx = threadIdx.x; idx < total; idx += nthr) {
        int c, k;
        if (STORE_CF) { c = idx & (tc - 1); k = idx >> ltc; }
        else if (NS)  { c = idx / n; k = idx % n; }
        else          { c = (int)fdiv((uint32_t)idx, dn); k = idx - c * n; }
        const int col = c0 + c;
        if (col >= ncols) continue;
        const T2* z = Z + (c >> 1) * pl;
        T val;
        if (!INV) {
            const T2 a = z[pad16(k)];
            const T2 b = z[pad16(k == 0 ? 0 : n - k)];
            if (2 * k <= n) val = (c & 1) ? T(0.5) * (a.y + b.y) : T(0.5) * (a.x + b.x);
            else            val = (c & 1) ? T(0.5) * (a.x - b.x) : T(0.5) * (b.y - a.y);
        } else {
            const T2 a = z[pad16(k)];
            val = (c & 1) ? a.y : a.x;
        }
        st_one<T>(stb, o, col, k, val * sc);
    }
}

// ---------------------------------------------------------------------------
// Static-length pass (n = 128 or 256, tile 1 << LTCS columns, every tile full).
// Each thread owns column PAIRS: it loads columns (2p, 2p+1) of a point together
// and writes them as one complex value, so index arithmetic, shared-memory
// traffic and the Hermitian pack/unpack are done once per pair.  The reverse
// transform packs on load: a thread takes points k and n-k of its pair and writes
// Z[k], Z[n-k] directly.  The forward transform unpacks on store the same way,
// producing modes k and n-k of both columns from two shared-memory reads.  Row
// indices are affine in the compile-time loop counter, so the functors' address
// arithmetic folds into immediate offsets.
// ---------------------------------------------------------------------------


template <typename T, int NS, int LTCS, bool INV, bool LOAD_CF, bool STORE_CF, class LD, class ST>
__global__ void __launch_bounds__(FFT_THREADS, 3)
k_fft_pass_s(const typename C2<T>::t* __restrict__ twg, T sc, LD ld_, ST st_) {
    using T2 = typename C2<T>::t;
    static_assert(NS == 128 || NS == 256, "static lengths: 128, 256");
    static_assert(!INV || LOAD_CF, "reverse passes load column-contiguous tiles");
    static_assert(INV || STORE_CF, "forward passes store column-contiguous tiles");
    constexpr int N = NS, H = N / 2, TC = 1 << LTCS, NP = TC / 2, PL = N + (N >> 4) + 1, TH = FFT_THREADS;
    constexpr int RS = TH / NP;  // rows per sweep of the pair-major mappings
    static_assert(TH % NP == 0 && H % RS == 0, "tile and block shape");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* tw = reinterpret_cast<T2*>(smem_raw);
    T2* buf0 = tw + N;
    T2* buf1 = buf0 + NP * PL;
    const int tid = threadIdx.x;
    const int o = blockIdx.y;
    const int c0 = blockIdx.x * TC;
    const auto& ld = bind_ld(ld_, o);
    const auto& st = bind_st(st_, o);
    for (int i = tid; i < N; i += TH) tw[i] = twg[i];

    if constexpr (INV) {
        // points k and n-k of pair p (k = 0 takes points 0 and n/2), packed into Z
        constexpr int U = H / RS;
        const int p = tid % NP, r0 = tid / NP, col = c0 + 2 * p;
        T a1[U], b1[U], a2[U], b2[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = r0 + RS * u;
            ld_pair<T>(ld, o, col, k, a1[u], b1[u]);
            ld_pair<T>(ld, o, col, k == 0 ? H : N - k, a2[u], b2[u]);
        }
        T2* z = buf0 + p * PL;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = r0 + RS * u;
            T2 lo, hi;
            if (k == 0) {
                lo.x = a1[u]; lo.y = b1[u];
                hi.x = a2[u]; hi.y = b2[u];
                z[pad16(0)] = lo;
                z[pad16(H)] = hi;
            } else {
                lo.x = a1[u] - b2[u]; lo.y = a2[u] + b1[u];
                hi.x = a1[u] + b2[u]; hi.y = b1[u] - a2[u];
                z[pad16(k)] = lo;
                z[pad16(N - k)] = hi;
            }
        }
    } else if constexpr (LOAD_CF) {
        constexpr int U = N / RS;
        const int p = tid % NP, r0 = tid / NP, col = c0 + 2 * p;
        T a[U], b[U];
#pragma unroll
        for (int u = 0; u < U; u++) ld_pair<T>(ld, o, col, r0 + RS * u, a[u], b[u]);
        T2* z = buf0 + p * PL;
#pragma unroll
        for (int u = 0; u < U; u++) {
            T2 v;
            v.x = a[u]; v.y = b[u];
            z[pad16(r0 + RS * u)] = v;
        }
    } else {
        // point-contiguous input: a warp reads 32 consecutive points of one column
        constexpr int PS = TH / N, U = NP / PS;
        static_assert(TH % N == 0 && NP % PS == 0, "point-major mapping");
        const int j = tid % N, pb = tid / N;
        T a[U], b[U];
#pragma unroll
        for (int u = 0; u < U; u++) ld_pair<T>(ld, o, c0 + 2 * (pb + PS * u), j, a[u], b[u]);
#pragma unroll
        for (int u = 0; u < U; u++) {
            T2 v;
            v.x = a[u]; v.y = b[u];
            buf0[(pb + PS * u) * PL + pad16(j)] = v;
        }
    }
    __syncthreads();
    const T2* Z = smem_fft_static<NS, INV>(buf0, buf1, tw, NP, PL);

    if constexpr (!INV) {
        // modes k and n-k of both columns of pair p from Z[k], Z[n-k]
        constexpr int U = H / RS;
        const int p = tid % NP, r0 = tid / NP, col = c0 + 2 * p;
        const T2* z = Z + p * PL;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = r0 + RS * u;
            if (k == 0) {
                const T2 a = z[pad16(0)], b = z[pad16(H)];
                st_pair<T>(st, o, col, 0, a.x * sc, a.y * sc);
                st_pair<T>(st, o, col, H, b.x * sc, b.y * sc);
            } else {
                const T2 a = z[pad16(k)], b = z[pad16(N - k)];
                st_pair<T>(st, o, col, k, T(0.5) * (a.x + b.x) * sc, T(0.5) * (a.y + b.y) * sc);
                st_pair<T>(st, o, col, N - k, T(0.5) * (a.y - b.y) * sc, T(0.5) * (b.x - a.x) * sc);
            }
        }
    } else if constexpr (STORE_CF) {
        constexpr int U = N / RS;
        const int p = tid % NP, r0 = tid / NP, col = c0 + 2 * p;
        const T2* z = Z + p * PL;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = r0 + RS * u;
            const T2 a = z[pad16(k)];
            st_pair<T>(st, o, col, k, a.x * sc, a.y * sc);
        }
    } else {
        constexpr int PS = TH / N, U = NP / PS;
        const int j = tid % N, pb = tid / N;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int p = pb + PS * u;
            const T2 a = Z[p * PL + pad16(j)];
            st_pair<T>(st, o, c0 + 2 * p, j, a.x * sc, a.y * sc);
        }
    }
}

// ---------------------------------------------------------------------------
// Register-staged pass for n = 256 = 16 x 16 with NP column pairs per tile
// (8 or 16): 16 NP threads, one radix-16 butterfly each per stage.  The
// butterfly next to global memory runs on registers: a forward pass loads the 16
// points j + 16 r of its pair straight into the first butterfly, and a reverse
// pass stores the 16 modes j + 16 r of its second butterfly straight to global
// memory, so one shared-memory round trip and one barrier fewer than the
// two-buffer pass.  The stage that stays in shared memory works in place (each
// thread reads and writes its own 16 slots), so one tile buffer suffices.
// ---------------------------------------------------------------------------
constexpr int FFT_R_N = 256, FFT_R_PL = 256 + 16 + 1;
// Column pairs per tile: 8 or 16, compiled for both and chosen at run time (the
// autotuner times both).  Default: 16 (256 threads, 4 CTAs per SM) for float32;
// 8 (128 threads, 4 CTAs per SM) for float64, whose 16-point butterflies need
// twice the registers (3% faster than 16 pairs at 2 CTAs per SM).
template <typename T>
__host__ __device__ constexpr int fft_r_np() { return sizeof(T) == 8 ? 8 : 16; }
// CTAs per SM the launch bounds ask for (registers per thread <= 65536 / (16 NP MINB)).
// FP64 with 8 sequences per CTA: 5 (96 registers, a few spilled) measured 2-5 %
// faster on B200 than 4 (126 registers, none spilled) and 6 (80 registers).
#ifndef SW_FFT_R_MINB_F64
#define SW_FFT_R_MINB_F64 5
#endif
template <typename T, int NP>
__host__ __device__ constexpr int fft_r_minb() {
    return NP == 8 ? (sizeof(T) == 8 ? SW_FFT_R_MINB_F64 : 8) : (sizeof(T) == 8 ? 2 : 4);
}

// Shared memory of the register-staged pass: the 64 twiddles of stage2_16x16 and
// NP padded sequences.
template <typename T>
inline size_t fft_pass_smem_r(int np) {
    return sizeof(typename C2<T>::t) * ((size_t)64 + (size_t)np * FFT_R_PL);
}

// Second radix-16 stage of 256 = 16 x 16 on the slots j + 16 r of one sequence:
// twiddles exp(-+2 pi i r j / 256), then the butterfly; natural order in and out.
// Four twiddles come from the table (r = 1, 2, 4, 8); the other eleven are
// products of at most three of them, which keeps shared-memory instructions (the
// pass's limiting pipe) down at a cost of a few roundings per twiddle.
// tw4 holds exp(-2 pi i m j / 256) for m = 1, 2, 4, 8 and j < 16 as four rows of
// 16, so that the sixteen threads of a butterfly row read consecutive entries
// (no shared-memory bank conflicts, unlike strided reads of the full table).
template <bool INV, typename T2>
__device__ __forceinline__ void stage2_16x16(T2* v, const T2* __restrict__ tw4, int j) {
    T2 w[16];
    w[1] = tw4[j];
    w[2] = tw4[16 + j];
    w[4] = tw4[32 + j];
    w[8] = tw4[48 + j];
    w[3] = cmul(w[1], w[2]);
    w[5] = cmul(w[1], w[4]);
    w[6] = cmul(w[2], w[4]);
    w[7] = cmul(w[3], w[4]);
    w[9] = cmul(w[1], w[8]);
    w[10] = cmul(w[2], w[8]);
    w[11] = cmul(w[3], w[8]);
    w[12] = cmul(w[4], w[8]);
    w[13] = cmul(w[5], w[8]);
    w[14] = cmul(w[6], w[8]);
    w[15] = cmul(w[7], w[8]);
#pragma unroll
    for (int r = 1; r < 16; r++) {
        T2 ww = w[r];
        if (INV) ww.y = -ww.y;
        v[r] = cmul(v[r], ww);
    }
    butterfly<16, INV>(v);
}

// Hooks of one register-staged tile (fft_r_tile): after_load() runs after the tile's
// global loads are in registers and before its first shared-memory write;
// before_store() runs after its last shared-memory read and before its first
// store through st.  The plain pass needs neither; the single-pass cluster
// transform (k_fft2d_cluster) uses them to share the tile buffer with the data it
// exchanges between the CTAs of a cluster.
struct NoHooks {
    __device__ __forceinline__ void after_load() const {}
    __device__ __forceinline__ void before_store() const {}
};

// Lane layout of the pair-major phases of the register-staged pass.  Thread t
// works on column pair t % NP and residue class cls(t / NP) of the 256 points
// (points j, j + 16, ..., j + 240).  The real-pair pack and unpack combine point
// k with point n - k, which lies in class 16 - j, so the classes are ordered
// 0, 8, 1, 15, 2, 14, ..., 7, 9: classes j and 16 - j sit on lanes t and t ^ NP
// of one warp (classes 0 and 8 pair with themselves) and exchange with shuffles.
__device__ __forceinline__ int fft_r_class(int g) {
    const int i = g >> 1;
    return g < 2 ? 8 * g : ((g & 1) ? 16 - i : i);
}
template <typename T2>
__device__ __forceinline__ T2 shfl_xor_c(T2 v, int m) {
    T2 r;
    r.x = __shfl_xor_sync(0xffffffffu, v.x, m);
    r.y = __shfl_xor_sync(0xffffffffu, v.y, m);
    return r;
}

// One tile of the register-staged pass: plane o, columns c0 .. c0 + 2 NP - 1, all
// 256 points; buf holds NP padded sequences, tw the 64 twiddles of stage2_16x16.
// 256 = 16 x 16: the first radix-16 stage runs on the 16 points of one residue
// class in registers, one shared-memory transpose hands each thread the 16
// first-stage outputs of one frequency class, and the second stage (twiddles and
// radix 16) leaves that thread the modes k = j + 16 r of its class.  The forward
// transform's unpack and the reverse transform's pack, which combine the complex
// values at k and n - k of a column pair, swap eight values with the partner lane
// (classes j and 16 - j) instead of going through shared memory again.
template <typename T, int NPT, bool INV, bool LOAD_CF, bool STORE_CF, class LD, class ST, class HK>
__device__ __forceinline__ void fft_r_tile(const typename C2<T>::t* __restrict__ tw, typename C2<T>::t* buf, T sc,
                                           const LD& ld_, const ST& st_, int o, int c0, const HK& hk) {
    using T2 = typename C2<T>::t;
    static_assert(!INV || LOAD_CF, "reverse passes load column-contiguous tiles");
    static_assert(INV || STORE_CF, "forward passes store column-contiguous tiles");
    constexpr int N = FFT_R_N, H = N / 2, NP = NPT, PL = FFT_R_PL;
    static_assert(NP == 8 || NP == 16, "partner classes must share a warp");
    const int tid = threadIdx.x;
    const auto& ld = bind_ld(ld_, o);
    const auto& st = bind_st(st_, o);
    // pair-major (pair index on the lanes: column-contiguous global access) with the
    // partner class order, and point-major (point index on the lanes: point-contiguous
    // global access)
    const int pl_ = tid % NP, jc = fft_r_class(tid / NP);
    const int pp = tid / 16, jp = tid % 16;
    const bool self0 = jc == 0, self8 = jc == 8;

    if constexpr (!INV) {
        const int p = LOAD_CF ? pl_ : pp, j = LOAD_CF ? jc : jp, col = c0 + 2 * p;
        T2 v[16];
#pragma unroll
        for (int r = 0; r < 16; r++) ld_pair<T>(ld, o, col, j + 16 * r, v[r].x, v[r].y);
        hk.after_load();
        butterfly<16, false>(v);  // first stage: no twiddles
        T2* y = buf + p * PL;
#pragma unroll
        for (int r = 0; r < 16; r++) y[pad16(16 * j + r)] = v[r];
        __syncthreads();
        {
            const T2* z = buf + pl_ * PL;
#pragma unroll
            for (int r = 0; r < 16; r++) v[r] = z[pad16(jc + 16 * r)];
        }
        hk.before_store();
        stage2_16x16<false>(v, tw, jc);
        // unpack: v[s] = Z[k], k = jc + 16 s < n/2 (s < 8), with Z[n - k] from the
        // partner's slot 15 - s (class 8: own slot 15 - s; class 0: own slot 16 - s,
        // and modes 0 and n/2 from slots 0 and 8)
        const int col2 = c0 + 2 * pl_;
        const T hs = T(0.5) * sc;  // (a + b) hs == (0.5 (a + b)) sc exactly: scaling by 0.5 is exact
#pragma unroll
        for (int s = 0; s < 8; s++) {
            const T2 recv = shfl_xor_c(v[15 - s], NP);
            const T2 a = v[s];
            const T2 b = self0 ? v[s == 0 ? 8 : 16 - s] : (self8 ? v[15 - s] : recv);
            const int k = jc + 16 * s;
            if (s == 0 && self0) {
                st_pair<T>(st, o, col2, 0, a.x * sc, a.y * sc);
                st_pair<T>(st, o, col2, H, b.x * sc, b.y * sc);
            } else {
                st_pair<T>(st, o, col2, k, (a.x + b.x) * hs, (a.y + b.y) * hs);
                st_pair<T>(st, o, col2, N - k, (a.y - b.y) * hs, (b.x - a.x) * hs);
            }
        }
    } else {
        // pack: points k = jc + 16 s (s < 8) and n - k of pair pl_ (k = 0 takes 0 and
        // n/2) give Z[k] (own slot s) and Z[n - k] (the partner's slot 15 - s; class
        // 8: own slot 15 - s; class 0: own slot 16 - s, or 8 for n/2)
        T2 v[16];
        {
            const int col = c0 + 2 * pl_;
            T a1[8], b1[8], a2[8], b2[8];
#pragma unroll
            for (int s = 0; s < 8; s++) {
                const int k = jc + 16 * s;
                ld_pair<T>(ld, o, col, k, a1[s], b1[s]);
                ld_pair<T>(ld, o, col, k == 0 ? H : N - k, a2[s], b2[s]);
            }
            hk.after_load();
            T2 hi0[8];
#pragma unroll
            for (int s = 0; s < 8; s++) {
                T2 lo, hi;
                if (s == 0 && self0) {
                    lo.x = a1[s]; lo.y = b1[s];
                    hi.x = a2[s]; hi.y = b2[s];
                } else {
                    lo.x = a1[s] - b2[s]; lo.y = a2[s] + b1[s];
                    hi.x = a1[s] + b2[s]; hi.y = b1[s] - a2[s];
                }
                const T2 recv = shfl_xor_c(hi, NP);
                v[s] = lo;
                v[15 - s] = self8 ? hi : recv;
                hi0[s] = hi;
            }
            if (self0) {
                v[8] = hi0[0];
#pragma unroll
                for (int s = 1; s < 8; s++) v[16 - s] = hi0[s];
            }
        }
        // first stage on class jc: slots jc + 16 r in, 16 jc + r out
        butterfly<16, true>(v);
        {
            T2* y = buf + pl_ * PL;
#pragma unroll
            for (int r = 0; r < 16; r++) y[pad16(16 * jc + r)] = v[r];
        }
        __syncthreads();
        const int p = STORE_CF ? pl_ : pp, k = STORE_CF ? jc : jp, col = c0 + 2 * p;
        const T2* z = buf + p * PL;
#pragma unroll
        for (int r = 0; r < 16; r++) v[r] = z[pad16(k + 16 * r)];
        hk.before_store();
        stage2_16x16<true>(v, tw, k);
#pragma unroll
        for (int r = 0; r < 16; r++) st_pair<T>(st, o, col, k + 16 * r, v[r].x * sc, v[r].y * sc);
    }
}

// The 64 twiddles of stage2_16x16 (exp(-2 pi i m j / 256), m = 1, 2, 4, 8, j < 16)
// from the length-256 table, into shared memory.
template <typename T2>
__device__ __forceinline__ void load_tw64(T2* tw, const T2* __restrict__ twg) {
    if (threadIdx.x < 64) tw[threadIdx.x] = twg[(1 << (threadIdx.x >> 4)) * (threadIdx.x & 15)];
}

template <typename T, int NPT, bool INV, bool LOAD_CF, bool STORE_CF, class LD, class ST>
__global__ void __launch_bounds__(16 * NPT, fft_r_minb<T, NPT>())
k_fft_pass_r(const typename C2<T>::t* __restrict__ twg, T sc, LD ld, ST st) {
    using T2 = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* tw = reinterpret_cast<T2*>(smem_raw);  // 64 entries: the rows of stage2_16x16
    T2* buf = tw + 64;
    load_tw64(tw, twg);
    fft_r_tile<T, NPT, INV, LOAD_CF, STORE_CF>(tw, buf, sc, ld, st, blockIdx.y, blockIdx.x * 2 * NPT, NoHooks{});
}

}  // namespace sw
