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

namespace sw {

template <typename T> struct C2;
template <> struct C2<double> { using t = double2; };
template <> struct C2<float> { using t = float2; };

constexpr int FFT_MAX_RAD = 24;
constexpr int FFT_THREADS = 256;

struct FftPlan {
    int n;
    int nrad;
    int rad[FFT_MAX_RAD];
};

template <typename T2>
__device__ __forceinline__ T2 cmul(T2 a, T2 b) {
    T2 r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

// In-register DFT of size R, sign -1 (forward) or +1 (INV).
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
    } else {  // R == 5
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
    }
}

// One Stockham pass of radix R over np sequences of length n held at x[p*n + j].
template <int R, bool INV, typename T2>
__device__ __forceinline__ void stockham_stage(const T2* __restrict__ x, T2* __restrict__ y,
                                               const T2* __restrict__ tw, int n, int Ns, int np) {
    const int nR = n / R;
    const int tstride = n / (Ns * R);
    for (int b = threadIdx.x; b < np * nR; b += blockDim.x) {
        const int p = b / nR;
        const int j = b - p * nR;
        const int k = j % Ns;
        const int base = (j - k) * R + k;
        const T2* xp = x + p * n;
        T2* yp = y + p * n;
        T2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = xp[j + r * nR];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                T2 w = tw[r * k * tstride];
                if (INV) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        butterfly<R, INV>(v);
#pragma unroll
        for (int r = 0; r < R; r++) yp[base + r * Ns] = v[r];
    }
}

// Full transform of np sequences; returns the buffer holding the result.
template <bool INV, typename T2>
__device__ T2* smem_fft(const FftPlan& plan, T2* a, T2* b, const T2* tw, int np) {
    int Ns = 1;
    for (int s = 0; s < plan.nrad; s++) {
        const int R = plan.rad[s];
        switch (R) {
            case 4: stockham_stage<4, INV>(a, b, tw, plan.n, Ns, np); break;
            case 2: stockham_stage<2, INV>(a, b, tw, plan.n, Ns, np); break;
            case 3: stockham_stage<3, INV>(a, b, tw, plan.n, Ns, np); break;
            default: stockham_stage<5, INV>(a, b, tw, plan.n, Ns, np); break;
        }
        __syncthreads();
        T2* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

// Shared memory bytes of one pass: twiddles (n) + two tiles (tc/2 * n each).
template <typename T>
inline size_t fft_pass_smem(int n, int tc) {
    return sizeof(typename C2<T>::t) * (size_t)n * (size_t)(1 + tc);
}

// Generic tile pass.  grid.x = column tiles, grid.y = output index o.
template <typename T, bool INV, bool LOAD_CF, bool STORE_CF, class LD, class ST>
__global__ void __launch_bounds__(FFT_THREADS)
k_fft_pass(FftPlan plan, const typename C2<T>::t* __restrict__ twg, int ncols, int tc, T sc, LD ld, ST st) {
    using T2 = typename C2<T>::t;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = plan.n;
    const int np = tc >> 1;
    T2* tw = reinterpret_cast<T2*>(smem_raw);
    T2* buf0 = tw + n;
    T2* buf1 = buf0 + (size_t)np * n;
    const int o = blockIdx.y;
    const int c0 = blockIdx.x * tc;
    const int nthr = blockDim.x;

    for (int i = threadIdx.x; i < n; i += nthr) tw[i] = twg[i];
    T* rb = reinterpret_cast<T*>(buf0);
    for (int idx = threadIdx.x; idx < tc * n; idx += nthr) {
        int c, j;
        if (LOAD_CF) { c = idx % tc; j = idx / tc; }
        else         { j = idx % n;  c = idx / n; }
        const int col = c0 + c;
        T val = (col < ncols) ? (T)ld(o, col, j) : T(0);
        rb[(((c >> 1) * n + j) << 1) + (c & 1)] = val;
    }
    __syncthreads();
    if (INV) {
        // pack Hermitian column pairs (Ha, Hb) into Z = A + iB
        const int kh = (n - 1) / 2;
        for (int idx = threadIdx.x; idx < np * kh; idx += nthr) {
            const int p = idx / kh;
            const int k = 1 + idx - p * kh;
            T2* z = buf0 + p * n;
            T2 lo = z[k], hi = z[n - k];  // lo = (Ha[k], Hb[k]), hi = (Ha[n-k], Hb[n-k])
            T2 zk, znk;
            zk.x = lo.x - hi.y;  zk.y = hi.x + lo.y;
            znk.x = lo.x + hi.y; znk.y = lo.y - hi.x;
            z[k] = zk;
            z[n - k] = znk;
        }
        __syncthreads();
    }
    const T2* Z = smem_fft<INV>(plan, buf0, buf1, tw, np);
    for (int idx = threadIdx.x; idx < tc * n; idx += nthr) {
        int c, k;
        if (STORE_CF) { c = idx % tc; k = idx / tc; }
        else          { k = idx % n;  c = idx / n; }
        const int col = c0 + c;
        if (col >= ncols) continue;
        const T2* z = Z + (c >> 1) * n;
        T val;
        if (!INV) {
            const T2 a = z[k];
            const T2 b = z[k == 0 ? 0 : n - k];
            if (2 * k <= n) val = (c & 1) ? T(0.5) * (a.y + b.y) : T(0.5) * (a.x + b.x);
            else            val = (c & 1) ? T(0.5) * (a.x - b.x) : T(0.5) * (b.y - a.y);
        } else {
            val = (c & 1) ? z[k].y : z[k].x;
        }
        st(o, col, k, val * sc);
    }
}

}  // namespace sw
