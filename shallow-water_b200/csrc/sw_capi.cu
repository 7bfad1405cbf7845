// extern "C" entry points of libswcuda.so (declared in include/sw_cuda.h).
#include <mutex>

#include "sw_solver.cuh"

using namespace sw;

namespace {

thread_local std::string g_last_error;

int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

template <class F>
int guarded(F&& f) {
    try {
        const int st = f();
#ifdef SW_BOUNDS_CHECK
        // debug build: wait for the call's kernels and report an access outside the
        // registered allocations (the access itself was skipped)
        if (st == SW_OK) {
            unsigned long long addr = 0, bytes = 0;
            const unsigned long long n = bc::take_fault(&addr, &bytes);
            if (n) {
                char msg[200];
                snprintf(msg, sizeof(msg), "bounds check: %llu device accesses outside the library's allocations or "
                         "misaligned, the first at 0x%llx (%llu bytes)", n, addr, bytes);
                return fail(SW_ERR_CUDA, msg);
            }
        }
#endif
        return st;
    } catch (const Error& e) {
        return fail(e.status, e.what());
    } catch (const std::bad_alloc&) {
        return fail(SW_ERR_CUDA, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(SW_ERR_ARG, e.what());
    }
}

// ---- standalone 1-D transforms on m columns of length n ------------------------------
template <typename T>
struct Plan1d {
    FftPlan plan{};
    DevBuf<typename C2<T>::t> tw;
    int tc = 2;
    T sc = 1;
};

std::mutex g_plan_mu;
std::map<std::pair<int, int>, std::shared_ptr<void>> g_plans;  // (device, n) per precision

template <typename T>
std::shared_ptr<Plan1d<T>> get_plan(int n) {
    int dev = 0;
    SW_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto key = std::make_pair(dev * 2 + (sizeof(T) == 4 ? 1 : 0), n);
    auto it = g_plans.find(key);
    if (it != g_plans.end()) return std::static_pointer_cast<Plan1d<T>>(it->second);
    auto p = std::make_shared<Plan1d<T>>();
    require(build_plan(n, p->plan) == SW_OK, SW_ERR_FACTORISE, "factorisation failed for n=" + std::to_string(n));
    auto h = host_twiddles<T>(n);
    p->tw.alloc(n);
    SW_CUDA(cudaMemcpy(p->tw.p, h.data(), sizeof(h[0]) * n, cudaMemcpyHostToDevice));
    p->tc = pick_tile<T>(n);
    p->sc = (T)(1.0 / std::sqrt((double)n));
    g_plans[key] = p;
    return p;
}

template <typename T>
struct ColIO {  // x[col + m*pt]
    T* x;
    int m;
    __device__ __forceinline__ T operator()(int, int c, int p) const { return x[c + (size_t)m * p]; }
    __device__ __forceinline__ void operator()(int, int c, int p, T v) const { x[c + (size_t)m * p] = v; }
};

template <typename T>
void fft1d_dev(int m, int n, T* x, bool inverse, cudaStream_t s) {
    auto p = get_plan<T>(n);
    ColIO<T> io{x, m};
    if (inverse) launch_pass<T, true, true, true>(s, p->plan, p->tw.p, p->tc, p->sc, 1, m, io, io);
    else launch_pass<T, false, true, true>(s, p->plan, p->tw.p, p->tc, p->sc, 1, m, io, io);
}

int check_trig(int n, const double* trig, const int factors[5]) {
    if (factors) {
        int f[5];
        int st = sw_factorisen(n, f);
        if (st) return fail(st, "factorisation failed");
        for (int i = 0; i < 5; i++)
            if (f[i] != factors[i]) return fail(SW_ERR_ARG, "factors do not match n");
    }
    (void)trig;
    return SW_OK;
}

int fft1d_host(int m, int n, double* x, const double* trig, const int factors[5], bool inverse) {
    return guarded([&] {
        require(m >= 1 && n >= 2 && x, SW_ERR_ARG, "bad forfft/revfft arguments");
        int st = check_trig(n, trig, factors);
        if (st) return st;
        const size_t cnt = (size_t)m * n;
        DevBuf<double> d(cnt);
        SW_CUDA(cudaMemcpy(d.p, x, cnt * sizeof(double), cudaMemcpyHostToDevice));
        fft1d_dev<double>(m, n, d.p, inverse, 0);
        SW_CUDA(cudaMemcpy(x, d.p, cnt * sizeof(double), cudaMemcpyDeviceToHost));
        return SW_OK;
    });
}

}  // namespace

namespace sw {
void record_error(const std::string& msg) { g_last_error = msg; }
#ifdef SW_BOUNDS_CHECK
void sw_bc_register(const void* p, size_t bytes, int add) {
    if (add) bc::add(p, bytes);
    else bc::remove(p);
}
#else
void sw_bc_register(const void*, size_t, int) {}
#endif
}  // namespace sw

// ---- the context ---------------------------------------------------------------
struct sw_ctx {
    int ng, nz, M, precision, device;
    std::unique_ptr<Solver<double>> s64;
    std::unique_ptr<Solver<float>> s32;
    DevBuf<double> hostio;  // staging for host-array operations
};

namespace {

template <class F>
int with_solver(sw_ctx* ctx, F&& f) {
    return guarded([&] {
        require(ctx != nullptr, SW_ERR_ARG, "null context");
        SW_CUDA(cudaSetDevice(ctx->device));
        if (ctx->s64) return f(*ctx->s64);
        return f(*ctx->s32);
    });
}

template <typename T>
__global__ void k_convert(const double* a, T* b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        b[i] = (T)a[i];
}
template <typename T>
__global__ void k_convert_back(const T* a, double* b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

// host -> device field copy with conversion
template <typename S>
void field_in(S& s, int field, size_t offset, const double* host, size_t n, bool sync = true) {
    if (double* d = s.field_d(field)) {
        SW_CUDA(cudaMemcpyAsync(d + offset, host, n * sizeof(double), cudaMemcpyHostToDevice, s.st));
    } else {
        auto* t = s.field_t(field);
        require(t != nullptr, SW_ERR_ARG, "bad field index");
        if constexpr (sizeof(*t) == sizeof(double)) {
            SW_CUDA(cudaMemcpyAsync(t + offset, host, n * sizeof(double), cudaMemcpyHostToDevice, s.st));
        } else {
            double* tmp = s.WD(11);
            SW_CUDA(cudaMemcpyAsync(tmp, host, n * sizeof(double), cudaMemcpyHostToDevice, s.st));
            k_convert<<<256, 256, 0, s.st>>>(tmp, t + offset, n);
            SW_CHECK_LAUNCH();
        }
    }
    if (sync) SW_CUDA(cudaStreamSynchronize(s.st));
}
template <typename S>
void field_out(S& s, int field, size_t offset, double* host, size_t n, bool sync = true) {
    if (double* d = s.field_d(field)) {
        SW_CUDA(cudaMemcpyAsync(host, d + offset, n * sizeof(double), cudaMemcpyDeviceToHost, s.st));
    } else {
        auto* t = s.field_t(field);
        require(t != nullptr, SW_ERR_ARG, "bad field index");
        if constexpr (sizeof(*t) == sizeof(double)) {
            SW_CUDA(cudaMemcpyAsync(host, t + offset, n * sizeof(double), cudaMemcpyDeviceToHost, s.st));
        } else {
            double* tmp = s.WD(11);
            k_convert_back<<<256, 256, 0, s.st>>>(t + offset, tmp, n);
            SW_CHECK_LAUNCH();
            SW_CUDA(cudaMemcpyAsync(host, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, s.st));
        }
    }
    if (sync) SW_CUDA(cudaStreamSynchronize(s.st));
}

// Copy nplanes host planes into a T work buffer (via float64 staging).
template <typename S, typename T>
void planes_in(S& s, T* dst, const double* host, size_t n) {
    double* tmp = s.WD(11);
    SW_CUDA(cudaMemcpyAsync(tmp, host, n * sizeof(double), cudaMemcpyHostToDevice, s.st));
    k_convert<<<256, 256, 0, s.st>>>(tmp, dst, n);
    SW_CHECK_LAUNCH();
}
template <typename S, typename T>
void planes_out(S& s, const T* src, double* host, size_t n) {
    double* tmp = s.WD(11);
    k_convert_back<<<256, 256, 0, s.st>>>(src, tmp, n);
    SW_CHECK_LAUNCH();
    SW_CUDA(cudaMemcpyAsync(host, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, s.st));
    SW_CUDA(cudaStreamSynchronize(s.st));
}

}  // namespace

extern "C" {

const char* sw_last_error(void) { return g_last_error.c_str(); }
int sw_version(void) { return 1; }

int sw_factorisen(int n, int factors[5]) {
    static const int fac[5] = {6, 4, 2, 3, 5};
    if (!factors) return fail(SW_ERR_ARG, "null factors");
    for (int i = 0; i < 5; i++) factors[i] = 0;
    if (n < 2) return fail(SW_ERR_FACTORISE, "Factorization failed");
    int rem = n;
    for (int i = 0; i < 5; i++)
        while (rem % fac[i] == 0) {
            factors[i]++;
            rem /= fac[i];
            if (rem == 1) return SW_OK;
        }
    return fail(SW_ERR_FACTORISE, "Factorization failed");
}

int sw_initfft(int n, int factors[5], double* trig) {
    static const int fac[5] = {6, 4, 2, 3, 5};
    int st = sw_factorisen(n, factors);
    if (st) return st;
    if (!trig) return fail(SW_ERR_ARG, "null trig");
    for (int i = 0; i < 2 * n; i++) trig[i] = 0.0;
    double ftwopin = 2.0 * PI / (double)n;
    int rem = n, m = 1;
    for (int i = 0; i < 5; i++)
        for (int e = 0; e < factors[i]; e++) {
            rem /= fac[i];
            for (int k = 1; k < fac[i]; k++)
                for (int l = 0; l < rem; l++) trig[(m++) - 1] = ftwopin * (double)(k * l);
            ftwopin *= (double)fac[i];
        }
    for (int i = 1; i < n; i++) {
        trig[i + n - 1] = -std::sin(trig[i - 1]);
        trig[i - 1] = std::cos(trig[i - 1]);
    }
    return SW_OK;
}

int sw_forfft(int m, int n, double* x, const double* trig, const int factors[5]) {
    return fft1d_host(m, n, x, trig, factors, false);
}
int sw_revfft(int m, int n, double* x, const double* trig, const int factors[5]) {
    return fft1d_host(m, n, x, trig, factors, true);
}
int sw_forfft_dev(int m, int n, void* x, int precision, void* stream) {
    return guarded([&] {
        require(m >= 1 && n >= 2 && x, SW_ERR_ARG, "bad forfft arguments");
        SW_BC_SCOPE(x, (size_t)m * n * (precision == SW_FP64 ? 8 : 4));
        if (precision == SW_FP64) fft1d_dev<double>(m, n, (double*)x, false, (cudaStream_t)stream);
        else fft1d_dev<float>(m, n, (float*)x, false, (cudaStream_t)stream);
        return SW_OK;
    });
}
int sw_revfft_dev(int m, int n, void* x, int precision, void* stream) {
    return guarded([&] {
        require(m >= 1 && n >= 2 && x, SW_ERR_ARG, "bad revfft arguments");
        SW_BC_SCOPE(x, (size_t)m * n * (precision == SW_FP64 ? 8 : 4));
        if (precision == SW_FP64) fft1d_dev<double>(m, n, (double*)x, true, (cudaStream_t)stream);
        else fft1d_dev<float>(m, n, (float*)x, true, (cudaStream_t)stream);
        return SW_OK;
    });
}

int sw_ctx_create(int ng, int nz, int nmembers, int precision, int device, sw_ctx** out) {
    return guarded([&] {
        require(out != nullptr, SW_ERR_ARG, "null output pointer");
        *out = nullptr;
        require(precision == SW_FP64 || precision == SW_MIXED || precision == SW_FP32, SW_ERR_ARG, "unknown precision");
        int ndev = 0;
        SW_CUDA(cudaGetDeviceCount(&ndev));
        require(device >= 0 && device < ndev, SW_ERR_ARG, "no such CUDA device");
        SW_CUDA(cudaSetDevice(device));
        auto* c = new sw_ctx();
        c->ng = ng; c->nz = nz; c->M = nmembers; c->precision = precision; c->device = device;
        try {
            if (precision == SW_FP32) {
                c->s32.reset(new Solver<float>(ng, nz, nmembers));
            } else {
                c->s64.reset(new Solver<double>(ng, nz, nmembers));
                if (precision == SW_MIXED) c->s64->enable_refine32();
            }
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
        return SW_OK;
    });
}

void sw_ctx_destroy(sw_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    delete ctx;
}

int sw_ctx_info(const sw_ctx* ctx, int* ng, int* nz, int* nmembers, int* precision) {
    if (!ctx) return fail(SW_ERR_ARG, "null context");
    if (ng) *ng = ctx->ng;
    if (nz) *nz = ctx->nz;
    if (nmembers) *nmembers = ctx->M;
    if (precision) *precision = ctx->precision;
    return SW_OK;
}

int sw_spectral_get(sw_ctx* ctx, const char* name, double* out, size_t n) {
    return with_solver(ctx, [&](auto& s) {
        require(name != nullptr, SW_ERR_ARG, "null name");
        std::string nm(name);
        if (nm == "kmag") {
            require(n == s.host.kmag.size() && out, SW_ERR_ARG, "bad size for kmag");
            for (size_t i = 0; i < n; i++) out[i] = s.host.kmag[i];
            return SW_OK;
        }
        if (nm == "kmax" || nm == "kmaxred") {
            require(n == 1 && out, SW_ERR_ARG, "bad size");
            out[0] = nm == "kmax" ? s.host.kmax : s.host.kmaxred;
            return SW_OK;
        }
        const auto* v = s.host.find(nm);
        require(v != nullptr, SW_ERR_ARG, "unknown operator " + nm);
        require(out && n == v->size(), SW_ERR_ARG, "bad size for " + nm);
        std::memcpy(out, v->data(), n * sizeof(double));
        return SW_OK;
    });
}

int sw_state_set(sw_ctx* ctx, int field, int member, const double* host, size_t n) {
    return with_solver(ctx, [&](auto& s) {
        require(field >= 0 && field < SW_NFIELDS && member >= 0 && member < s.M && host, SW_ERR_ARG, "bad field/member");
        require(n == (size_t)s.L * s.n2, SW_ERR_ARG, "size must be ng*ng*(nz+1)");
        field_in(s, field, (size_t)member * s.L * s.n2, host, n);
        return SW_OK;
    });
}
int sw_state_get(sw_ctx* ctx, int field, int member, double* host, size_t n) {
    return with_solver(ctx, [&](auto& s) {
        require(field >= 0 && field < SW_NFIELDS && member >= 0 && member < s.M && host, SW_ERR_ARG, "bad field/member");
        require(n == (size_t)s.L * s.n2, SW_ERR_ARG, "size must be ng*ng*(nz+1)");
        field_out(s, field, (size_t)member * s.L * s.n2, host, n);
        return SW_OK;
    });
}
int sw_state_set_all(sw_ctx* ctx, int field, const double* host, size_t n) {
    return with_solver(ctx, [&](auto& s) {
        require(field >= 0 && field < SW_NFIELDS && host && n == s.nf, SW_ERR_ARG, "bad field or size");
        field_in(s, field, 0, host, n);
        return SW_OK;
    });
}
int sw_state_get_all(sw_ctx* ctx, int field, double* host, size_t n) {
    return with_solver(ctx, [&](auto& s) {
        require(field >= 0 && field < SW_NFIELDS && host && n == s.nf, SW_ERR_ARG, "bad field or size");
        field_out(s, field, 0, host, n);
        return SW_OK;
    });
}
int sw_state_set_all_async(sw_ctx* ctx, int field, const double* host, size_t n) {
    return with_solver(ctx, [&](auto& s) {
        require(field >= 0 && field < SW_NFIELDS && host && n == s.nf, SW_ERR_ARG, "bad field or size");
        field_in(s, field, 0, host, n, false);
        return SW_OK;
    });
}
int sw_state_get_all_async(sw_ctx* ctx, int field, double* host, size_t n) {
    return with_solver(ctx, [&](auto& s) {
        require(field >= 0 && field < SW_NFIELDS && host && n == s.nf, SW_ERR_ARG, "bad field or size");
        field_out(s, field, 0, host, n, false);
        return SW_OK;
    });
}
int sw_set_time(sw_ctx* ctx, double t) {
    return with_solver(ctx, [&](auto& s) { s.t = t; return SW_OK; });
}
int sw_get_time(const sw_ctx* ctx, double* t) {
    if (!ctx || !t) return fail(SW_ERR_ARG, "null argument");
    *t = ctx->s64 ? ctx->s64->t : ctx->s32->t;
    return SW_OK;
}

}  // extern "C"

// ---- plane operations on host arrays ------------------------------------------------
namespace sw {
namespace capi {

template <typename T>
int ptospc_impl(Solver<T>& s, const double* rvar, double* svar, bool fwd) {
    require(rvar && svar, SW_ERR_ARG, "null array");
    const int ng = s.ng, n2 = s.n2;
    T *a = s.W(23), *b = s.W(22);
    planes_in(s, a, rvar, n2);
    if (fwd)
        s.fft.ptospc(s.st, 1, [=] __device__(int, int iy, int ix) -> T { return a[iy + ng * ix]; },
                     [=] __device__(int, int kx, int ky, T v) { b[kx + ng * ky] = v; });
    else
        s.fft.spctop(s.st, 1, [=] __device__(int, int kx, int ky) -> T { return a[kx + ng * ky]; },
                     [=] __device__(int, int iy, int ix, T v) { b[iy + ng * ix] = v; });
    planes_out(s, b, svar, n2);
    return SW_OK;
}

template <typename T>
int deriv_impl(Solver<T>& s, const double* var, double* der, int axis) {
    require(var && der, SW_ERR_ARG, "null array");
    const int ng = s.ng, n2 = s.n2;
    T *a = s.W(23), *b = s.W(22);
    planes_in(s, a, var, n2);
    for_planes(s.st, 1, n2, [=] __device__(int, int i) {
        const int kx = i % ng, ky = i / ng;
        b[i] = axis == 0 ? (T)(dmul(kx, ng) * (double)a[mirror(kx, ng) + ng * ky])
                         : (T)(dmul(ky, ng) * (double)a[kx + ng * mirror(ky, ng)]);
    });
    planes_out(s, b, der, n2);
    return SW_OK;
}

// jacob / divs of one plane pair (src/spectral/mod.rs:423-475)
template <typename T>
int jd_impl(Solver<T>& s, const double* aa, const double* bb, double* cs, bool jac) {
    require(aa && bb && cs, SW_ERR_ARG, "null array");
    const int ng = s.ng, n2 = s.n2;
    T *in = s.W(23), *sa = s.W(22), *d = s.W(21), *out = s.W(20);
    planes_in(s, in, aa, n2);
    planes_in(s, in + n2, bb, n2);
    s.fft.ptospc(s.st, 2, [=] __device__(int o, int iy, int ix) -> T { return in[(size_t)o * n2 + iy + ng * ix]; },
                 [=] __device__(int o, int kx, int ky, T v) { sa[(size_t)o * n2 + kx + ng * ky] = v; });
    if (jac) {
        s.fft.spctop(s.st, 4,
            [=] __device__(int o, int kx, int ky) -> T {
                const T* a = sa + (size_t)(o / 2) * n2;
                return (o & 1) ? (T)(dmul(ky, ng) * (double)a[kx + ng * mirror(ky, ng)])
                               : (T)(dmul(kx, ng) * (double)a[mirror(kx, ng) + ng * ky]);
            },
            [=] __device__(int o, int iy, int ix, T v) { d[(size_t)o * n2 + iy + ng * ix] = v; });
        s.fft.ptospc(s.st, 1,
            [=] __device__(int, int iy, int ix) -> T {
                const int i = iy + ng * ix;
                return d[i] * d[3 * (size_t)n2 + i] - d[(size_t)n2 + i] * d[2 * (size_t)n2 + i];
            },
            [=] __device__(int, int kx, int ky, T v) { out[kx + ng * ky] = v; });
    } else {
        for_planes(s.st, 1, n2, [=] __device__(int, int i) {
            const int kx = i % ng, ky = i / ng;
            out[i] = (T)(dmul(ky, ng) * (double)sa[(size_t)n2 + kx + ng * mirror(ky, ng)] +
                         dmul(kx, ng) * (double)sa[mirror(kx, ng) + ng * ky]);
        });
    }
    planes_out(s, out, cs, n2);
    return SW_OK;
}

template <typename T>
int deal_impl(Solver<T>& s, double* fp, int nplanes_req) {
    require(fp != nullptr, SW_ERR_ARG, "null array");
    const int ng = s.ng, n2 = s.n2;
    const int np = nplanes_req < 0 ? s.L : nplanes_req;
    const double* filt = s.op.filt;
    T *a = s.W(23), *b = s.W(22);
    planes_in(s, a, fp, (size_t)np * n2);
    s.fft.ptospc(s.st, np, [=] __device__(int o, int iy, int ix) -> T { return a[(size_t)o * n2 + iy + ng * ix]; },
                 [=] __device__(int o, int kx, int ky, T v) {
                     const int i = kx + ng * ky;
                     b[(size_t)o * n2 + i] = (T)(filt[i] * (double)v);
                 });
    s.fft.spctop(s.st, np, [=] __device__(int o, int kx, int ky) -> T { return b[(size_t)o * n2 + kx + ng * ky]; },
                 [=] __device__(int o, int iy, int ix, T v) { a[(size_t)o * n2 + iy + ng * ix] = v; });
    planes_out(s, a, fp, (size_t)np * n2);
    return SW_OK;
}

template <typename T>
int t3d_impl(Solver<T>& s, const double* in, double* out, int izbeg, int izend, bool fwd) {
    require(in && out && izbeg >= 0 && izend <= s.nz && izbeg <= izend, SW_ERR_ARG, "bad ptospc3d/spctop3d arguments");
    const int ng = s.ng, n2 = s.n2, np = izend - izbeg + 1;
    T *a = s.W(23), *b = s.W(22);
    planes_in(s, a, in + (size_t)izbeg * n2, (size_t)np * n2);
    if (fwd)
        s.fft.ptospc(s.st, np, [=] __device__(int o, int iy, int ix) -> T { return a[(size_t)o * n2 + iy + ng * ix]; },
                     [=] __device__(int o, int kx, int ky, T v) { b[(size_t)o * n2 + kx + ng * ky] = v; });
    else
        s.fft.spctop(s.st, np, [=] __device__(int o, int kx, int ky) -> T { return a[(size_t)o * n2 + kx + ng * ky]; },
                     [=] __device__(int o, int iy, int ix, T v) { b[(size_t)o * n2 + iy + ng * ix] = v; });
    planes_out(s, b, out + (size_t)izbeg * n2, (size_t)np * n2);
    return SW_OK;
}

template <typename T>
int fft2d_impl(Solver<T>& s, int direction, int nplanes, const void* in, void* out) {
    require(in && out && nplanes >= 1 && (direction == 0 || direction == 1), SW_ERR_ARG, "bad fft2d arguments");
    const int ng = s.ng;
    SW_BC_SCOPE(in, (size_t)nplanes * ng * ng * sizeof(T));
    SW_BC_SCOPE(out, (size_t)nplanes * ng * ng * sizeof(T));
    const T* a = (const T*)in;
    T* b = (T*)out;
    if (direction == 0)
        s.fft.ptospc(s.st, nplanes, [=] __device__(int o, int iy, int ix) -> T { return a[((size_t)o * ng + ix) * ng + iy]; },
                     [=] __device__(int o, int kx, int ky, T v) { b[((size_t)o * ng + ky) * ng + kx] = v; });
    else
        s.fft.spctop(s.st, nplanes, [=] __device__(int o, int kx, int ky) -> T { return a[((size_t)o * ng + ky) * ng + kx]; },
                     [=] __device__(int o, int iy, int ix, T v) { b[((size_t)o * ng + ix) * ng + iy] = v; });
    return SW_OK;
}


// Reduction bodies of one plane for reduce_groups: f(i) -> one value, or RedVals<2>.
template <class F>
struct PlaneSum1 {
    F f;
    __device__ RedVals<1> operator()(int, long long i) const {
        RedVals<1> r;
        r.v[0] = f((int)i);
        return r;
    }
};
template <class F>
struct PlaneSum2 {
    F f;
    __device__ RedVals<2> operator()(int, long long i) const { return f((int)i); }
};

// balinit (src/balinit.rs:21-435): the balanced 2-D initial fields of the PV strip,
// as a fixed-point iteration over one ng x ng plane, entirely on the device: the
// transforms, derivatives, products, filters and the scalar sums (deterministic
// reductions into device scalars that the following kernels read).  The host reads
// only the two relative changes per iteration for the stop test (toler 1e-9, or
// the change stops falling).  float64 only.  Returns the iteration count.
inline int balinit_impl(Solver<double>& s, const double* qin, double* qout, double* dout, double* gout) {
    const int ng = s.ng, n2 = s.n2;
    const double toler = 1.0E-9, small = 1.0E-12, dsumi = 1.0 / (double)(ng * ng);
    cudaStream_t st = s.st;
    const double *filt = s.op.filt, *opak = s.op.opak, *rlap = s.op.rlap, *helm = s.op.helm, *c2g2 = s.op.c2g2;
    DevBuf<double> B((size_t)24 * n2), S(16);
    double* const b = B.p;
    double *QQ = b, *ZZ = b + n2, *UU = b + 2 * (size_t)n2, *VV = b + 3 * (size_t)n2, *HH = b + 4 * (size_t)n2;
    double *DD = b + 5 * (size_t)n2, *GG = b + 6 * (size_t)n2, *DDP = b + 7 * (size_t)n2, *GGP = b + 8 * (size_t)n2;
    double *DSs = b + 9 * (size_t)n2, *WA = b + 10 * (size_t)n2, *WB = b + 11 * (size_t)n2;
    double *WP = b + 14 * (size_t)n2, *WQ = b + 15 * (size_t)n2;
    // 8 planes: u, v spectra (0, 1) and their derivatives (4..7) for jacob; the
    // physical products (0, 1) and their spectra (2, 3) for divs
    double* X = b + 16 * (size_t)n2;
    double* sc = S.p;  // 0 qadd, 1 qbar, 2 uio, 3 vio, 4..7 error sums
    double* part = s.red_partial.p;
    auto sum1 = [&](double* out, auto f) { reduce_groups<1>(st, 1, n2, 0u, PlaneSum1<decltype(f)>{f}, part, out); };
    auto sum2 = [&](double* out, auto f) { reduce_groups<2>(st, 1, n2, 0u, PlaneSum2<decltype(f)>{f}, part, out); };
    auto ptospc = [&](const double* src, double* dst) {
        s.fft.ptospc(st, 1, [=] __device__(int, int iy, int ix) -> double { return src[iy + ng * ix]; },
                     [=] __device__(int, int kx, int ky, double v) { dst[kx + ng * ky] = v; });
    };
    auto spctop = [&](const double* src, double* dst) {
        s.fft.spctop(st, 1, [=] __device__(int, int kx, int ky) -> double { return src[kx + ng * ky]; },
                     [=] __device__(int, int iy, int ix, double v) { dst[iy + ng * ix] = v; });
    };
    // divs(a, b) (src/spectral/mod.rs:461-475) of the physical products in X, X + n2
    auto divs = [&](double* out) {
        s.fft.ptospc(st, 2, [=] __device__(int o, int iy, int ix) -> double { return X[(size_t)o * n2 + iy + ng * ix]; },
                     [=] __device__(int o, int kx, int ky, double v) { X[(size_t)(2 + o) * n2 + kx + ng * ky] = v; });
        for_planes(st, 1, n2, [=] __device__(int, int i) {
            const int kx = i % ng, ky = i / ng;
            out[i] = dmul(ky, ng) * X[3 * (size_t)n2 + kx + ng * mirror(ky, ng)] +
                     dmul(kx, ng) * X[2 * (size_t)n2 + mirror(kx, ng) + ng * ky];
        });
    };
    // the rlap, filter and velocity block shared by the set-up and the iteration:
    // zz -> spectral, WA = rlap zz-hat, zz = filtered zz; u, v from WA (+ rlap ds)
    auto velocity = [&](bool with_ds) {
        ptospc(ZZ, WB);
        for_planes(st, 1, n2, [=] __device__(int, int i) {
            WA[i] = rlap[i] * WB[i];
            WB[i] = WB[i] * filt[i];
        });
        spctop(WB, ZZ);
        for_planes(st, 1, n2, [=] __device__(int, int i) {
            const int kx = i % ng, ky = i / ng;
            const int mx = mirror(kx, ng) + ng * ky, my = kx + ng * mirror(ky, ng);
            double u = -(dmul(ky, ng) * WA[my]), v = dmul(kx, ng) * WA[mx];  // -d/dy, d/dx of rlap zz
            if (with_ds) {
                u += dmul(kx, ng) * (rlap[mx] * DSs[mx]);
                v += dmul(ky, ng) * (rlap[my] * DSs[my]);
            }
            WP[i] = u;
            WQ[i] = v;
        });
        spctop(WP, UU);
        spctop(WQ, VV);
    };
    SW_CUDA(cudaMemcpyAsync(QQ, qin, sizeof(double) * n2, cudaMemcpyHostToDevice, st));
    SW_CUDA(cudaMemsetAsync(DD, 0, sizeof(double) * n2, st));
    SW_CUDA(cudaMemsetAsync(GG, 0, sizeof(double) * n2, st));
    SW_CUDA(cudaMemsetAsync(DDP, 0, sizeof(double) * n2, st));
    SW_CUDA(cudaMemsetAsync(GGP, 0, sizeof(double) * n2, st));
    // remove the mean of qq; hh from the inversion of f qq
    sum1(sc + 0, [=] __device__(int i) { return QQ[i]; });
    for_planes(st, 1, n2, [=] __device__(int, int i) { QQ[i] += -dsumi * sc[0]; });
    sum1(sc + 1, [=] __device__(int i) { return QQ[i]; });
    for_planes(st, 1, n2, [=] __device__(int, int i) { WP[i] = COF * QQ[i]; });
    ptospc(WP, WB);
    for_planes(st, 1, n2, [=] __device__(int, int i) { WA[i] = filt[i] * WB[i] / (opak[i] - COF * (dsumi * sc[1])); });
    spctop(WA, HH);
    sum1(sc + 0, [=] __device__(int i) { return (1.0 + HH[i]) * QQ[i]; });
    for_planes(st, 1, n2, [=] __device__(int, int i) {
        const double q = QQ[i] + (-dsumi * sc[0]);
        QQ[i] = q;
        ZZ[i] = (1.0 + HH[i]) * (COF + q) - COF;
    });
    velocity(false);
    sum1(sc + 2, [=] __device__(int i) { return HH[i] * UU[i]; });
    for_planes(st, 1, n2, [=] __device__(int, int i) { UU[i] += -sc[2] * dsumi; });
    double* hs = s.h_pinned;
    double toterrpre = 1.0 / (small * small), toterr = 0.5;
    int iters = 0;
    while (toterr > toler) {
        iters++;
        // gs = filt (div(dd u, dd v) - 2 J(u, v)); gg = spctop(gs).  J (src/spectral/
        // mod.rs:423-453): u, v to spectral, their x, y derivatives back, u_x v_y - u_y v_x
        s.fft.ptospc(st, 2, [=] __device__(int o, int iy, int ix) -> double {
                         return (o ? VV : UU)[iy + ng * ix];
                     },
                     [=] __device__(int o, int kx, int ky, double v) { X[(size_t)o * n2 + kx + ng * ky] = v; });
        s.fft.spctop(st, 4,
            [=] __device__(int o, int kx, int ky) -> double {
                const double* a = X + (size_t)(o / 2) * n2;
                return (o & 1) ? dmul(ky, ng) * a[kx + ng * mirror(ky, ng)] : dmul(kx, ng) * a[mirror(kx, ng) + ng * ky];
            },
            [=] __device__(int o, int iy, int ix, double v) { X[(size_t)(4 + o) * n2 + iy + ng * ix] = v; });
        s.fft.ptospc(st, 1,
            [=] __device__(int, int iy, int ix) -> double {
                const int i = iy + ng * ix;
                const double* d = X + 4 * (size_t)n2;
                return d[i] * d[3 * (size_t)n2 + i] - d[(size_t)n2 + i] * d[2 * (size_t)n2 + i];
            },
            [=] __device__(int, int kx, int ky, double v) { WB[kx + ng * ky] = v; });
        for_planes(st, 1, n2, [=] __device__(int, int i) {
            X[i] = DD[i] * UU[i];
            X[(size_t)n2 + i] = DD[i] * VV[i];
        });
        divs(WA);
        for_planes(st, 1, n2, [=] __device__(int, int i) { WA[i] = filt[i] * (WA[i] - 2.0 * WB[i]); });
        spctop(WA, GG);
        sum2(sc + 4, [=] __device__(int i) {
            RedVals<2> r;
            const double e = GG[i] - GGP[i];
            r.v[0] = e * e;
            r.v[1] = GGP[i] * GGP[i];
            return r;
        });
        // ds = helm (f div(zz u, zz v) - c2g2 div(hh u, hh v)); dd = spctop(ds)
        for_planes(st, 1, n2, [=] __device__(int, int i) {
            X[i] = HH[i] * UU[i];
            X[(size_t)n2 + i] = HH[i] * VV[i];
        });
        divs(WA);
        for_planes(st, 1, n2, [=] __device__(int, int i) {
            X[i] = ZZ[i] * UU[i];
            X[(size_t)n2 + i] = ZZ[i] * VV[i];
        });
        divs(WB);
        for_planes(st, 1, n2, [=] __device__(int, int i) { DSs[i] = helm[i] * (COF * WB[i] - c2g2[i] * WA[i]); });
        spctop(DSs, DD);
        sum2(sc + 6, [=] __device__(int i) {
            RedVals<2> r;
            const double e = DD[i] - DDP[i];
            r.v[0] = e * e;
            r.v[1] = DDP[i] * DDP[i];
            return r;
        });
        // hh from q and gamma; q's mean against htot; zz; u, v
        sum1(sc + 0, [=] __device__(int i) { return QQ[i] * (1.0 + HH[i]); });
        for_planes(st, 1, n2, [=] __device__(int, int i) { QQ[i] += -dsumi * sc[0]; });
        sum1(sc + 1, [=] __device__(int i) { return QQ[i]; });
        for_planes(st, 1, n2, [=] __device__(int, int i) {
            const double qbar = dsumi * sc[1];
            WP[i] = COF * (QQ[i] + HH[i] * (QQ[i] - qbar)) - GG[i];
        });
        ptospc(WP, WB);
        for_planes(st, 1, n2, [=] __device__(int, int i) { WA[i] = filt[i] * WB[i] / (opak[i] - COF * (dsumi * sc[1])); });
        spctop(WA, HH);
        sum1(sc + 0, [=] __device__(int i) { return QQ[i] * (1.0 + HH[i]); });
        for_planes(st, 1, n2, [=] __device__(int, int i) {
            const double q = QQ[i] + (-dsumi * sc[0]);
            QQ[i] = q;
            ZZ[i] = (1.0 + HH[i]) * (COF + q) - COF;
        });
        velocity(true);
        sum2(sc + 2, [=] __device__(int i) {
            RedVals<2> r;
            r.v[0] = HH[i] * UU[i];
            r.v[1] = HH[i] * VV[i];
            return r;
        });
        for_planes(st, 1, n2, [=] __device__(int, int i) {
            UU[i] += -sc[2] * dsumi;
            VV[i] += -sc[3] * dsumi;
        });
        SW_CUDA(cudaMemcpyAsync(hs, sc + 4, sizeof(double) * 4, cudaMemcpyDeviceToHost, st));
        SW_CUDA(cudaStreamSynchronize(st));
        const double ggrmserr = hs[0] / (hs[1] + small), ddrmserr = hs[2] / (hs[3] + small);
        toterr = 0.5 * (ddrmserr + ggrmserr);
        if (toterrpre <= toterr) break;
        SW_CUDA(cudaMemcpyAsync(DDP, DD, sizeof(double) * n2, cudaMemcpyDeviceToDevice, st));
        SW_CUDA(cudaMemcpyAsync(GGP, GG, sizeof(double) * n2, cudaMemcpyDeviceToDevice, st));
        toterrpre = toterr;
        require(iters < 10000, SW_ERR_PSOLVE_MAXITER, "balinit did not converge");
    }
    for_planes(st, 1, n2, [=] __device__(int, int i) { WP[i] = ZZ[i] - COF * HH[i]; });
    SW_CUDA(cudaMemcpyAsync(qout, WP, sizeof(double) * n2, cudaMemcpyDeviceToHost, st));
    SW_CUDA(cudaMemcpyAsync(dout, DD, sizeof(double) * n2, cudaMemcpyDeviceToHost, st));
    SW_CUDA(cudaMemcpyAsync(gout, GG, sizeof(double) * n2, cudaMemcpyDeviceToHost, st));
    SW_CUDA(cudaStreamSynchronize(st));
    return iters;
}

}  // namespace capi
}  // namespace sw

extern "C" {
int sw_ptospc(sw_ctx* ctx, const double* rvar, double* svar) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::ptospc_impl(s, rvar, svar, true); });
}
int sw_spctop(sw_ctx* ctx, const double* svar, double* rvar) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::ptospc_impl(s, svar, rvar, false); });
}
int sw_xderiv(sw_ctx* ctx, const double* var, double* der) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::deriv_impl(s, var, der, 0); });
}
int sw_yderiv(sw_ctx* ctx, const double* var, double* der) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::deriv_impl(s, var, der, 1); });
}
int sw_jacob(sw_ctx* ctx, const double* aa, const double* bb, double* cs) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::jd_impl(s, aa, bb, cs, true); });
}
int sw_divs(sw_ctx* ctx, const double* aa, const double* bb, double* cs) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::jd_impl(s, aa, bb, cs, false); });
}
int sw_deal2d(sw_ctx* ctx, double* fp) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::deal_impl(s, fp, 1); });
}
int sw_deal3d(sw_ctx* ctx, double* fp) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::deal_impl(s, fp, -1); });
}
int sw_ptospc3d(sw_ctx* ctx, const double* fp, double* fs, int izbeg, int izend) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::t3d_impl(s, fp, fs, izbeg, izend, true); });
}
int sw_spctop3d(sw_ctx* ctx, const double* fs, double* fp, int izbeg, int izend) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::t3d_impl(s, fs, fp, izbeg, izend, false); });
}

// spec1d (src/spectral/mod.rs:559-591): shell sums on the device, deterministic.
// balinit (src/balinit.rs:21-435) on the context's device: float64 contexts only.
int sw_balinit(sw_ctx* ctx, const double* qq_init, double* qq, double* dd, double* gg, int* iters) {
    return guarded([&] {
        require(ctx != nullptr && qq_init && qq && dd && gg, SW_ERR_ARG, "null argument");
        require(ctx->s64 != nullptr, SW_ERR_STATE, "balinit runs on SW_FP64 and SW_MIXED contexts (float64)");
        SW_CUDA(cudaSetDevice(ctx->device));
        const int n = sw::capi::balinit_impl(*ctx->s64, qq_init, qq, dd, gg);
        if (iters) *iters = n;
        return SW_OK;
    });
}

int sw_spec1d(sw_ctx* ctx, const double* ss, double* spec) {
    return with_solver(ctx, [&](auto& s) {
        require(ss && spec, SW_ERR_ARG, "null array");
        const int nb = s.host.kmax + 1;
        double* tmp = s.WD(11);
        SW_CUDA(cudaMemcpyAsync(tmp, ss, sizeof(double) * s.n2, cudaMemcpyHostToDevice, s.st));
        s.spec1d(tmp, tmp + s.n2);
        SW_CUDA(cudaMemcpyAsync(spec, tmp + s.n2, sizeof(double) * nb, cudaMemcpyDeviceToHost, s.st));
        SW_CUDA(cudaStreamSynchronize(s.st));
        return SW_OK;
    });
}
int sw_savegrid(sw_ctx* ctx, int member, double energies[3], double* spectra, int nspec, float* fields3,
                float* fields2) {
    return with_solver(ctx, [&](auto& s) {
        require(energies && spectra && fields3 && fields2 && member >= 0 && member < s.M, SW_ERR_ARG,
                "bad savegrid arguments");
        require(nspec == 3 * (s.host.kmax + 1), SW_ERR_ARG, "spectra needs 3*(kmax+1) values");
        s.savegrid(member, energies, spectra, fields3, fields2);
        return SW_OK;
    });
}

// ---- nhswps numerics -------------------------------------------------------------
int sw_main_invert(sw_ctx* ctx) {
    return with_solver(ctx, [&](auto& s) {
        s.main_invert();
        SW_CUDA(cudaStreamSynchronize(s.st));
        return SW_OK;
    });
}
int sw_vertical(sw_ctx* ctx) {
    return with_solver(ctx, [&](auto& s) {
        s.vertical();
        SW_CUDA(cudaStreamSynchronize(s.st));
        return SW_OK;
    });
}
int sw_coeffs(sw_ctx* ctx, double* sigx, double* sigy, double* cpt1, double* cpt2) {
    return with_solver(ctx, [&](auto& s) {
        s.coeffs();
        const size_t n = (size_t)s.L * s.n2;
        if (sigx) planes_out(s, s.sigx.p, sigx, n);
        if (sigy) planes_out(s, s.sigy.p, sigy, n);
        if (cpt1) planes_out(s, s.cpt1.p, cpt1, n);
        if (cpt2) planes_out(s, s.cpt2.p, cpt2, n);
        SW_CUDA(cudaStreamSynchronize(s.st));
        return SW_OK;
    });
}
int sw_cpsource(sw_ctx* ctx, double* sp0) {
    return with_solver(ctx, [&](auto& s) {
        s.cpsource();
        if (sp0) planes_out(s, s.sp0.p, sp0, (size_t)s.L * s.n2);
        SW_CUDA(cudaStreamSynchronize(s.st));
        return SW_OK;
    });
}
int sw_psolve(sw_ctx* ctx, int nitmax, int* iters, double* errp) {
    return with_solver(ctx, [&](auto& s) {
        int st = s.psolve(nitmax, iters, errp);
        SW_CUDA(cudaStreamSynchronize(s.st));
        if (st == SW_ERR_PSOLVE_DIVERGED) return fail(st, "Pressure error too large!");
        if (st == SW_ERR_PSOLVE_MAXITER) return fail(st, "Exceeded maximum number of iterations to find pressure!");
        return st;
    });
}
int sw_source(sw_ctx* ctx, double* sqs, double* sds, double* sgs) {
    return with_solver(ctx, [&](auto& s) {
        double *a = s.WD(4), *b = s.WD(5), *c = s.WD(7);
        s.source(a, b, c);
        const size_t n = (size_t)s.L * s.n2;
        if (sqs) SW_CUDA(cudaMemcpyAsync(sqs, a, n * sizeof(double), cudaMemcpyDeviceToHost, s.st));
        if (sds) SW_CUDA(cudaMemcpyAsync(sds, b, n * sizeof(double), cudaMemcpyDeviceToHost, s.st));
        if (sgs) SW_CUDA(cudaMemcpyAsync(sgs, c, n * sizeof(double), cudaMemcpyDeviceToHost, s.st));
        SW_CUDA(cudaStreamSynchronize(s.st));
        return SW_OK;
    });
}
int sw_advance(sw_ctx* ctx, int nsteps, int ggen) {
    return with_solver(ctx, [&](auto& s) {
        require(nsteps >= 0, SW_ERR_ARG, "nsteps must be >= 0");
        int st = s.advance(nsteps, ggen != 0);
        if (st == SW_ERR_PSOLVE_DIVERGED) return fail(st, "Pressure error too large!");
        if (st == SW_ERR_PSOLVE_MAXITER) return fail(st, "Exceeded maximum number of iterations to find pressure!");
        return st;
    });
}
int sw_diagnose(sw_ctx* ctx, int member, double out[4]) {
    return with_solver(ctx, [&](auto& s) {
        require(member >= 0 && member < s.M && out, SW_ERR_ARG, "bad member");
        s.diagnose_reduce();
        double raw[3];
        SW_CUDA(cudaMemcpyAsync(s.h_pinned, s.red_out.p + 3 * member, sizeof(raw), cudaMemcpyDeviceToHost, s.st));
        SW_CUDA(cudaStreamSynchronize(s.st));
        std::memcpy(raw, s.h_pinned, sizeof(raw));
        s.diag_finish(raw, out);
        return SW_OK;
    });
}
int sw_diag_history(sw_ctx* ctx, double* out, int cap, int* count) {
    return with_solver(ctx, [&](auto& s) {
        require(out && count && cap >= 0, SW_ERR_ARG, "bad arguments");
        int recorded = 0;
        SW_CUDA(cudaStreamSynchronize(s.st));
        SW_CUDA(cudaMemcpy(&recorded, s.hist_dev.p, sizeof(int), cudaMemcpyDeviceToHost));
        const int rows = std::min(std::min(recorded, s.hist_cap), cap);
        const int first = recorded - rows;
        std::vector<double> raw((size_t)s.hist_cap * s.M * 3);
        SW_CUDA(cudaMemcpy(raw.data(), s.diag_hist.p, raw.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int k = 0; k < rows; k++) {
            const double* r = raw.data() + (size_t)((first + k) % s.hist_cap) * s.M * 3;
            s.diag_finish(r, out + 4 * (size_t)k);
        }
        *count = rows;
        SW_CUDA(cudaMemset(s.hist_dev.p, 0, sizeof(int)));
        return SW_OK;
    });
}
int sw_energy(sw_ctx* ctx, int member, double out[3]) {
    return with_solver(ctx, [&](auto& s) {
        require(member >= 0 && member < s.M && out, SW_ERR_ARG, "bad member");
        s.energy(member, out);
        return SW_OK;
    });
}
int sw_last_sweeps(sw_ctx* ctx, int out[3]) {
    return with_solver(ctx, [&](auto& s) {
        require(out != nullptr, SW_ERR_ARG, "null output");
        for (int i = 0; i < 3; i++) out[i] = s.last_sweeps[i];
        return SW_OK;
    });
}
int sw_advance_async(sw_ctx* ctx, int nsteps, int ggen) {
    return with_solver(ctx, [&](auto& s) {
        require(nsteps >= 0, SW_ERR_ARG, "nsteps must be >= 0");
        if (!s.use_graphs) {  // host-driven steps synchronise per sweep anyway
            int st = s.advance(nsteps, ggen != 0);
            if (st == SW_ERR_PSOLVE_DIVERGED) return fail(st, "Pressure error too large!");
            if (st == SW_ERR_PSOLVE_MAXITER) return fail(st, "Exceeded maximum number of iterations to find pressure!");
            return st;
        }
        s.advance_enqueue(nsteps, ggen != 0);
        return SW_OK;
    });
}
int sw_sync(sw_ctx* ctx) {
    return with_solver(ctx, [&](auto& s) {
        if (s.pending) {
            int st = s.advance_finish();
            if (st == SW_ERR_PSOLVE_DIVERGED) return fail(st, "Pressure error too large!");
            if (st == SW_ERR_PSOLVE_MAXITER) return fail(st, "Exceeded maximum number of iterations to find pressure!");
            return st;
        }
        SW_CUDA(cudaStreamSynchronize(s.st));
        return SW_OK;
    });
}
int sw_field_device_ptr(sw_ctx* ctx, int field, void** ptr, int* elem_bytes) {
    return with_solver(ctx, [&](auto& s) {
        require(ptr && field >= 0 && field < SW_NFIELDS, SW_ERR_ARG, "bad field");
        if (double* d = s.field_d(field)) {
            *ptr = d;
            if (elem_bytes) *elem_bytes = 8;
        } else {
            auto* t = s.field_t(field);
            *ptr = t;
            if (elem_bytes) *elem_bytes = (int)sizeof(*t);
        }
        return SW_OK;
    });
}
int sw_stream(sw_ctx* ctx, void** stream) {
    return with_solver(ctx, [&](auto& s) {
        require(stream != nullptr, SW_ERR_ARG, "null output");
        *stream = (void*)s.st;
        return SW_OK;
    });
}
int sw_set_graphs(sw_ctx* ctx, int enable) {
    return with_solver(ctx, [&](auto& s) {
        s.use_graphs = enable != 0;
        return SW_OK;
    });
}
int sw_sweep_counts(sw_ctx* ctx, long long out[2]) {
    return with_solver(ctx, [&](auto& s) {
        require(out != nullptr, SW_ERR_ARG, "null output");
        if (s.pending) s.advance_finish();
        out[0] = s.sweeps_run[0];
        out[1] = s.sweeps_run[1];
        return SW_OK;
    });
}
int sw_set_fft_single_pass(sw_ctx* ctx, int enable, int* in_use) {
    return with_solver(ctx, [&](auto& s) {
        const bool on = s.set_fft_single_pass(enable);
        if (in_use) *in_use = on ? 1 : 0;
        return SW_OK;
    });
}
int sw_set_fft_overlap(sw_ctx* ctx, int enable, int* in_use) {
    return with_solver(ctx, [&](auto& s) {
        const bool on = s.set_fft_overlap(enable);
        if (in_use) *in_use = on ? 1 : 0;
        return SW_OK;
    });
}
int sw_set_psolve_toler(sw_ctx* ctx, double toler) {
    return with_solver(ctx, [&](auto& s) {
        s.set_refine_toler(toler);
        return SW_OK;
    });
}
int sw_set_psolve_relax(sw_ctx* ctx, double omega) {
    return with_solver(ctx, [&](auto& s) {
        s.set_psolve_relax(omega);
        return SW_OK;
    });
}
int sw_set_fft_chunk(sw_ctx* ctx, int planes, int* in_use) {
    return with_solver(ctx, [&](auto& s) {
        const int v = s.set_fft_chunk(planes);
        if (in_use) *in_use = v;
        return SW_OK;
    });
}
int sw_autotune_fft(sw_ctx* ctx, int reps, int maxc, int* tiles, int* chunks, int* overlaps, float* ms, int* ncand,
                    int* chosen_tile, int* chosen_chunk, int* chosen_overlap) {
    if (maxc < 0) return fail(SW_ERR_ARG, "maxc must be >= 0");
    return with_solver(ctx, [&](auto& s) {
        const int v = s.autotune_fft(reps, maxc, tiles, chunks, overlaps, ms, ncand, chosen_tile, chosen_overlap);
        if (chosen_chunk) *chosen_chunk = v;
        return SW_OK;
    });
}
int sw_set_fft_tile(sw_ctx* ctx, int columns, int* in_use) {
    return with_solver(ctx, [&](auto& s) {
        const int v = s.set_fft_tile(columns);
        if (in_use) *in_use = v;
        return SW_OK;
    });
}
int sw_fft2d_dev(sw_ctx* ctx, int direction, int nplanes, const void* in, void* out) {
    return with_solver(ctx, [&](auto& s) { return sw::capi::fft2d_impl(s, direction, nplanes, in, out); });
}
int sw_kernel_launches(sw_ctx* ctx, long long* count) {
    (void)ctx;
    if (!count) return fail(SW_ERR_ARG, "null output");
    *count = launch_counter().load();
    return SW_OK;
}

}  // extern "C"

// ---- ensembles of uneven grids ------------------------------------------------------
// Members with different (ng, nz): one batched context per (ng, nz) group, and one
// CUDA graph per step of the whole ensemble whose branches are the groups' steps
// (captured from the groups' streams into one graph), so that a step of every
// member is one graph launch and the groups' kernels run concurrently.
struct sw_ensemble {
    int device = 0, nmembers = 0;
    std::vector<sw_ctx*> groups;
    std::vector<std::pair<int, int>> where;  // member -> (group, index in the group)
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    bool pending = false;
    ~sw_ensemble() {
        if (master) cudaStreamSynchronize(master);
        for (auto& e : exec)
            if (e) cudaGraphExecDestroy(e);
        for (auto& j : joins)
            if (j) cudaEventDestroy(j);
        if (fork) cudaEventDestroy(fork);
        if (master) cudaStreamDestroy(master);
        for (auto* g : groups) sw_ctx_destroy(g);
    }
};

namespace {

template <class F>
int each_solver(sw_ctx* c, F&& f) {
    if (c->s64) return f(*c->s64);
    return f(*c->s32);
}

cudaGraphExec_t ensemble_graph(sw_ensemble* e, bool ggen) {
    cudaGraphExec_t& ex = e->exec[ggen ? 1 : 0];
    if (ex) return ex;
    SW_CUDA(cudaStreamBeginCapture(e->master, cudaStreamCaptureModeRelaxed));
    try {
        SW_CUDA(cudaEventRecord(e->fork, e->master));
        for (size_t g = 0; g < e->groups.size(); g++) {
            each_solver(e->groups[g], [&](auto& s) {
                SW_CUDA(cudaStreamWaitEvent(s.st, e->fork, 0));
                s.capture_step_body(ggen);
                SW_CUDA(cudaEventRecord(e->joins[g], s.st));
                return 0;
            });
            SW_CUDA(cudaStreamWaitEvent(e->master, e->joins[g], 0));
        }
    } catch (...) {
        cudaGraph_t gr = nullptr;
        cudaStreamEndCapture(e->master, &gr);
        if (gr) cudaGraphDestroy(gr);
        throw;
    }
    cudaGraph_t gr;
    SW_CUDA(cudaStreamEndCapture(e->master, &gr));
    SW_CUDA(cudaGraphInstantiate(&ex, gr, 0));
    SW_CUDA(cudaGraphDestroy(gr));
    return ex;
}

}  // namespace

extern "C" {

int sw_ensemble_create(const int* ng, const int* nz, int nmembers, int precision, int device, sw_ensemble** out) {
    return guarded([&] {
        require(out && ng && nz && nmembers >= 1, SW_ERR_ARG, "bad ensemble arguments");
        *out = nullptr;
        std::map<std::pair<int, int>, std::vector<int>> by_grid;
        for (int k = 0; k < nmembers; k++) by_grid[{ng[k], nz[k]}].push_back(k);
        std::unique_ptr<sw_ensemble> e(new sw_ensemble());
        e->device = device;
        e->nmembers = nmembers;
        e->where.resize(nmembers);
        for (auto& kv : by_grid) {
            sw_ctx* c = nullptr;
            const int st = sw_ctx_create(kv.first.first, kv.first.second, (int)kv.second.size(), precision, device, &c);
            if (st != SW_OK) return st;  // message already recorded
            const int g = (int)e->groups.size();
            e->groups.push_back(c);
            for (size_t j = 0; j < kv.second.size(); j++) e->where[kv.second[j]] = {g, (int)j};
        }
        SW_CUDA(cudaSetDevice(device));
        SW_CUDA(cudaStreamCreateWithFlags(&e->master, cudaStreamNonBlocking));
        SW_CUDA(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
        e->joins.resize(e->groups.size(), nullptr);
        for (auto& j : e->joins) SW_CUDA(cudaEventCreateWithFlags(&j, cudaEventDisableTiming));
        *out = e.release();
        return SW_OK;
    });
}

void sw_ensemble_destroy(sw_ensemble* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    delete e;
}

int sw_ensemble_info(const sw_ensemble* e, int* nmembers, int* ngroups) {
    if (!e) return fail(SW_ERR_ARG, "null ensemble");
    if (nmembers) *nmembers = e->nmembers;
    if (ngroups) *ngroups = (int)e->groups.size();
    return SW_OK;
}

int sw_ensemble_stream(sw_ensemble* e, void** stream) {
    if (!e || !stream) return fail(SW_ERR_ARG, "null argument");
    *stream = (void*)e->master;
    return SW_OK;
}

int sw_ensemble_member(sw_ensemble* e, int member, sw_ctx** ctx, int* index) {
    if (!e || !ctx || member < 0 || member >= e->nmembers) return fail(SW_ERR_ARG, "bad member");
    *ctx = e->groups[e->where[member].first];
    if (index) *index = e->where[member].second;
    return SW_OK;
}

int sw_ensemble_advance_async(sw_ensemble* e, int nsteps, int ggen) {
    return guarded([&] {
        require(e != nullptr && nsteps >= 0, SW_ERR_ARG, "bad ensemble advance arguments");
        SW_CUDA(cudaSetDevice(e->device));
        for (auto* c : e->groups)  // earlier work queued on a group's stream comes first
            each_solver(c, [&](auto& s) {
                require(s.use_graphs, SW_ERR_STATE, "ensemble steps need graphs on (sw_set_graphs)");
                SW_CUDA(cudaEventRecord(e->fork, s.st));
                SW_CUDA(cudaStreamWaitEvent(e->master, e->fork, 0));
                return 0;
            });
        for (int k = 0; k < nsteps; k++) SW_CUDA(cudaGraphLaunch(ensemble_graph(e, k == 0 ? ggen != 0 : true), e->master));
        for (auto* c : e->groups)
            each_solver(c, [&](auto& s) {
                s.note_external_steps(nsteps, ggen != 0);
                return 0;
            });
        // later calls on a group's context are ordered after these steps
        SW_CUDA(cudaEventRecord(e->fork, e->master));
        for (auto* c : e->groups)
            each_solver(c, [&](auto& s) {
                SW_CUDA(cudaStreamWaitEvent(s.st, e->fork, 0));
                return 0;
            });
        e->pending = true;
        return SW_OK;
    });
}

int sw_ensemble_sync(sw_ensemble* e) {
    return guarded([&] {
        require(e != nullptr, SW_ERR_ARG, "null ensemble");
        SW_CUDA(cudaSetDevice(e->device));
        SW_CUDA(cudaStreamSynchronize(e->master));
        int worst = SW_OK;
        for (auto* c : e->groups) {
            const int st = each_solver(c, [&](auto& s) { return s.pending ? s.advance_finish() : SW_OK; });
            if (st != SW_OK) worst = st;
        }
        e->pending = false;
        if (worst == SW_ERR_PSOLVE_DIVERGED) return fail(worst, "Pressure error too large!");
        if (worst == SW_ERR_PSOLVE_MAXITER) return fail(worst, "Exceeded maximum number of iterations to find pressure!");
        return worst;
    });
}

int sw_ensemble_advance(sw_ensemble* e, int nsteps, int ggen) {
    const int st = sw_ensemble_advance_async(e, nsteps, ggen);
    if (st != SW_OK) return st;
    return sw_ensemble_sync(e);
}

}  // extern "C"
