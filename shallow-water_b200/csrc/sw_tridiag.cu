// Batched tridiagonal solves (sw_tridiag_batched): the per-wavenumber vertical
// Thomas algorithm of psolve (src/nhswps/psolve.rs:285-327) as a standalone
// kernel for general coefficients, float64.
//
// nsys independent systems of n unknowns
//     a[i] x[i-1] + b[i] x[i] + c[i] x[i+1] = d[i],   i = 0 .. n-1
// (a[0] and c[n-1] are not used), stored level-major with the system index
// contiguous: element (i, s) at [s + nsys * i], the layout of the model's fields
// (one (kx, ky) column per system), so that a warp reads 32 consecutive systems
// of one level in one 256-byte transaction.
//
// One thread per system.  The forward sweep keeps the modified upper diagonal
// and right-hand side of the whole column in registers (n <= 33, the model's
// nz + 1 for nz <= 32); c and d are loaded before the recurrences, a and b as
// the elimination reaches them.  No pivoting: the systems must be safe for Gaussian
// elimination without it (e.g. diagonally dominant), as the psolve systems are.
// (compiled without the bounds checks of the debug build: only sw_capi.cu registers memory)
#undef SW_BOUNDS_CHECK
#include "sw_core.cuh"

namespace sw {
namespace tridiag {

constexpr int THREADS = 128;
constexpr int MAX_N = 33;

template <int NMAX>
__global__ void __launch_bounds__(THREADS)
k_tridiag(int n, int nsys, const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
          const double* __restrict__ d, double* __restrict__ x) {
    const int s = blockIdx.x * THREADS + threadIdx.x;
    if (s >= nsys) return;
    double cv[NMAX], dv[NMAX];
#pragma unroll
    for (int i = 0; i < NMAX; i++) {
        if (i < n) {
            const size_t p = s + (size_t)nsys * i;
            cv[i] = c[p];
            dv[i] = d[p];
        }
    }
    // forward elimination: cv <- c', dv <- d'
    {
        const double r = 1.0 / b[s];
        cv[0] *= r;
        dv[0] *= r;
    }
#pragma unroll
    for (int i = 1; i < NMAX; i++) {
        if (i < n) {
            const size_t p = s + (size_t)nsys * i;
            const double ai = a[p];
            const double r = 1.0 / (b[p] - ai * cv[i - 1]);
            cv[i] *= r;
            dv[i] = (dv[i] - ai * dv[i - 1]) * r;
        }
    }
    // back substitution
#pragma unroll
    for (int i = NMAX - 2; i >= 0; i--)
        if (i + 1 < n) dv[i] -= cv[i] * dv[i + 1];
#pragma unroll
    for (int i = 0; i < NMAX; i++)
        if (i < n) x[s + (size_t)nsys * i] = dv[i];
}

template <int NMAX>
static void launch(int n, int nsys, const double* a, const double* b, const double* c, const double* d, double* x,
                   cudaStream_t st) {
    k_tridiag<NMAX><<<(nsys + THREADS - 1) / THREADS, THREADS, 0, st>>>(n, nsys, a, b, c, d, x);
}

}  // namespace tridiag

void record_error(const std::string& msg);  // sets the message sw_last_error() returns

}  // namespace sw

extern "C" int sw_tridiag_batched(int n, int nsys, const double* a, const double* b, const double* c, const double* d,
                                  double* x, void* stream) {
    using namespace sw::tridiag;
    if (n < 1 || n > MAX_N || nsys < 1 || !a || !b || !c || !d || !x) {
        sw::record_error("sw_tridiag_batched: need 1 <= n <= " + std::to_string(MAX_N) +
                         ", nsys >= 1 and non-null arrays");
        return SW_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (n <= 8) launch<8>(n, nsys, a, b, c, d, x, st);
    else if (n <= 17) launch<17>(n, nsys, a, b, c, d, x, st);
    else launch<33>(n, nsys, a, b, c, d, x, st);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        sw::record_error(std::string("sw_tridiag_batched: launch failed: ") + cudaGetErrorString(e));
        return SW_ERR_CUDA;
    }
    sw::count_launch();
    return SW_OK;
}

extern "C" int sw_tridiag_batched_host(int n, int nsys, const double* a, const double* b, const double* c,
                                       const double* d, double* x) {
    if (n < 1 || n > sw::tridiag::MAX_N || nsys < 1 || !a || !b || !c || !d || !x)
        return sw_tridiag_batched(n, nsys, a, b, c, d, x, nullptr);  // records the argument error
    try {
        const size_t cnt = (size_t)n * nsys, bytes = cnt * sizeof(double);
        sw::DevBuf<double> buf;
        buf.alloc(5 * cnt);
        double* dv = buf.p;
        const double* src[4] = {a, b, c, d};
        for (int k = 0; k < 4; k++) SW_CUDA(cudaMemcpy(dv + k * cnt, src[k], bytes, cudaMemcpyHostToDevice));
        const int st = sw_tridiag_batched(n, nsys, dv, dv + cnt, dv + 2 * cnt, dv + 3 * cnt, dv + 4 * cnt, nullptr);
        if (st != SW_OK) return st;
        SW_CUDA(cudaMemcpy(x, dv + 4 * cnt, bytes, cudaMemcpyDeviceToHost));
        return SW_OK;
    } catch (const sw::Error& e) {
        sw::record_error(e.what());
        return e.status;
    }
}
