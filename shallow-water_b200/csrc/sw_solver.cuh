// The nhswps time-step path on the GPU: main_invert, vertical, coeffs,
// cpsource, psolve, source, advance, diagnose and the savegrid energies for an
// ensemble of M independent members of one (ng, nz) grid.
//
// Every 3-D field is stored member-major in the reference's Fortran order:
// plane q = m*(nz+1) + iz holds ng*ng values, physical p[iy + ng*ix] or spectral
// s[kx + ng*ky].  T is the precision of the transforms and of the physical
// work fields (double for SW_FP64, float for SW_MIXED); the prognostic spectral
// fields qs, ds, gs, the pressure ps, the tridiagonal solves, the residual, the
// diagnostics and the time update are float64 in both paths.
#pragma once
#include <algorithm>
#include <map>
#include <memory>

#include "sw_fft2d.cuh"
#include "sw_spectral_host.h"

namespace sw {

struct DeviceOps {
    DevBuf<double> hlap, glap, rlap, helm, c2g2, simp, rope, fope, filt, diss, opak, rdis, ap;
    DevBuf<double> htdv, etdv, weight, theta, htd1, etd1;
};

inline void upload(DevBuf<double>& d, const std::vector<double>& h) {
    d.alloc(h.size());
    SW_CUDA(cudaMemcpy(d.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
}

// Second pass of the pressure sweep's p, p_x, p_y transforms: output o of a chunk
// is (member mm, level iz, kind), o = mm * 3 nz + 3 iz + kind, and first-pass plane
// mm * 2 nz + 2 iz + (0 for p, 1 for p_y); kinds 0 and 2 read the intermediates of
// p and p_y, kind 1 reads p's with kx mirrored and the d/dx factor
// (src/sta2dfft.rs:128-155).  Columns (iy) are contiguous on both sides.
template <typename T>
struct SweepMidLoad {
    using T2 = typename C2<T>::t;
    static constexpr bool pair_io = true;
    const T* mid;
    int ng, nz;
    // f is the integer d/dx factor (or 1), so f * v in T equals the rounded
    // float64 product (as dmul_t)
    __device__ __forceinline__ const T* row(int o, int kx, T& f) const {
        const int mm = o / (3 * nz), k = o - mm * 3 * nz, iz = k / 3, kind = k - 3 * iz;
        const int plane = mm * 2 * nz + 2 * iz + (kind == 2 ? 1 : 0);
        f = kind == 1 ? (T)imul(kx, ng) : T(1);
        return mid + ((size_t)plane * ng + (kind == 1 ? mirror(kx, ng) : kx)) * ng;
    }
    __device__ __forceinline__ T operator()(int o, int c, int p) const {
        T f;
        const T* rw = row(o, p, f);
        if (!SW_BC_OK(rw + c, sizeof(T), sizeof(T))) return T(0);
        return f * rw[c];
    }
    __device__ __forceinline__ T2 ld2(int o, int c, int p) const {
        T f;
        const T* rw = row(o, p, f);
        if (!SW_BC_OK(rw + c, sizeof(T2), sizeof(T2))) return T2{};
        T2 v = *reinterpret_cast<const T2*>(rw + c);
        v.x = f * v.x;
        v.y = f * v.y;
        return v;
    }
};
template <typename T>
struct SweepPhysStore {
    using T2 = typename C2<T>::t;
    static constexpr bool pair_io = true;
    T *A, *B, *C;
    int ng, nz, L, m0;
    __device__ __forceinline__ T* dst(int o, int c, int p) const {
        const int mm = o / (3 * nz), k = o - mm * 3 * nz, iz = k / 3, kind = k - 3 * iz;
        T* base = kind == 0 ? A : kind == 1 ? B : C;
        return base + ((size_t)((m0 + mm) * L + iz) * ng + p) * ng + c;
    }
    __device__ __forceinline__ void operator()(int o, int c, int p, T v) const {
        T* d = dst(o, c, p);
        if (SW_BC_OK(d, sizeof(T), sizeof(T))) *d = v;
    }
    __device__ __forceinline__ void st2(int o, int c, int p, T a, T b) const {
        T2 v;
        v.x = a;
        v.y = b;
        T* d = dst(o, c, p);
        if (SW_BC_OK(d, sizeof(T2), sizeof(T2))) *reinterpret_cast<T2*>(d) = v;
    }
};

// Shell spectrum (spec1d, src/spectral/mod.rs:559-591) by bins of |k|: one warp
// per bin sums wt[e] * src(e) over the bin's elements e (a CSR list built once
// from kmag) in a fixed order, then a fixed shuffle tree: deterministic.
template <class SRC>
__global__ void k_spec_bins(int nbins, const int* __restrict__ off, const int* __restrict__ idx,
                            const double* __restrict__ wt, SRC src, double* __restrict__ out) {
    const int bin = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (bin >= nbins) return;
    double a = 0.0;
    for (int k = off[bin] + lane; k < off[bin + 1]; k += 32) {
        const int e = idx[k];
        a += wt[e] * src(e);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) out[bin] = a;
}

// dp/dtheta of psolve's finish (psolve.rs:371-410) for one (kx, ky) column with
// nz = NZS at compile time: the column of ps and the compact-scheme unknowns stay
// in registers (same arithmetic as the streamed loop in psolve_finish).
template <typename T, int NZS>
__global__ void __launch_bounds__(128)
k_dpdtheta(int n2, int ncols, const double* __restrict__ PS, const T* __restrict__ SP, const float* __restrict__ SPC,
           const double* __restrict__ htd1, const double* __restrict__ etd1, double hdzi, double dzi, double dz6,
           double* __restrict__ GG) {
    const int c = blockIdx.x * 128 + threadIdx.x;
    if (c >= ncols) return;
    const int m = c / n2, i = c - m * n2;
    const size_t cb = (size_t)m * (NZS + 1) * n2 + i;
    double p[NZS + 1], g[NZS + 1];
#pragma unroll
    for (int iz = 0; iz <= NZS; iz++) p[iz] = PS[cb + (size_t)iz * n2];
    const double spn = (double)SP[cb + (size_t)NZS * n2] + (SPC ? (double)SPC[cb + (size_t)NZS * n2] : 0.0);
    g[0] = 0.0;
    g[1] = (p[2] - p[0]) * hdzi * htd1[0];
#pragma unroll
    for (int iz = 2; iz < NZS; iz++) g[iz] = ((p[iz + 1] - p[iz - 1]) * hdzi - (1.0 / 6.0) * g[iz - 1]) * htd1[iz - 1];
    const double gn = dz6 * spn - p[NZS - 1] * dzi;
    g[NZS] = (gn - (1.0 / 3.0) * g[NZS - 1]) * htd1[NZS - 1];
#pragma unroll
    for (int iz = NZS - 1; iz >= 1; iz--) g[iz] = g[iz] + etd1[iz - 1] * g[iz + 1];
#pragma unroll
    for (int iz = 1; iz <= NZS; iz++) GG[cb + (size_t)iz * n2] = g[iz];
}

constexpr int UPDATE_THREADS = 128;

// Semi-implicit update of one (kx, ky) column (advance.rs:60-279; the same
// arithmetic as Solver::advance_update), LS = nz + 1 levels at compile time.  The
// summed sources of the column stay in registers across the three vertical
// passes, so each field is read once and qs, ds, gs are written once; the
// summed sds, sgs are not stored (source() recomputes them before their next use).
template <int LS, bool FIRST>
__global__ void __launch_bounds__(UPDATE_THREADS)
k_update(int n2, int ncols, double dt4, double dt4i, const double* __restrict__ diss,
         const double* __restrict__ rdis, const double* __restrict__ fope, const double* __restrict__ c2g2,
         const double* __restrict__ simp, const double* __restrict__ wgt, double* __restrict__ QS,
         double* __restrict__ DS, double* __restrict__ GS, double* __restrict__ qsi, double* __restrict__ qsm,
         const double* __restrict__ sqs, const double* __restrict__ sds, double* __restrict__ nds,
         const double* __restrict__ sgs, double* __restrict__ ngs, double* __restrict__ dsi, double* __restrict__ gsi) {
    const int c = blockIdx.x * UPDATE_THREADS + threadIdx.x;
    if (c >= ncols) return;
    const int m = c / n2, i = c - m * n2;
    const size_t cb = (size_t)m * LS * n2 + i;
    const double dis = diss[i], rd = rdis[i], fo = fope[i], cg = c2g2[i], si = simp[i];
    double sd[LS], sg[LS];
    double wka = 0.0, wkb = 0.0;
#pragma unroll
    for (int iz = 0; iz < LS; iz++) {
        const size_t p = cb + (size_t)iz * n2;
        const double sq = sqs[p];
        double qi, qm, nd, ng;
        if (FIRST) {
            const double q = QS[p], d0 = DS[p], g0 = GS[p];
            qi = q;
            qm = q + dt4 * sq;
            nd = sds[p] + dt4i * d0;
            ng = sgs[p] + dt4i * g0;
            qsi[p] = qi;
            qsm[p] = qm;
            dsi[p] = d0;
            gsi[p] = g0;
            nds[p] = nd;
            ngs[p] = ng;
        } else {
            qi = qsi[p];
            qm = qsm[p];
            nd = nds[p];
            ng = ngs[p];
        }
        QS[p] = dis * (qm + dt4 * sq) - qi;
        sd[iz] = sds[p] + nd;
        sg[iz] = sgs[p] + ng;
        const double d = sg[iz] + rd * sd[iz];
        wka += wgt[iz] * d;
        wkb += wgt[iz] * sd[iz];
    }
    wka *= fo;
    wkb *= cg;
    double wkg = 0.0;
#pragma unroll
    for (int iz = 0; iz < LS; iz++) {
        const size_t p = cb + (size_t)iz * n2;
        const double d = sg[iz] + rd * sd[iz];
        DS[p] = si * (d - wka) - dsi[p];
        const double g = wkb - FSQ * sd[iz] + rd * sg[iz];
        wkg += wgt[iz] * g;
    }
    wkg *= fo;
#pragma unroll
    for (int iz = 0; iz < LS; iz++) {
        const size_t p = cb + (size_t)iz * n2;
        const double g = wkb - FSQ * sd[iz] + rd * sg[iz];
        GS[p] = si * (g - wkg) - gsi[p];
    }
}

constexpr int THOMAS_THREADS = 128;

// Block sum of NV per-thread values into part[(m * gridDim.x + blockIdx.x) * NV + v].
template <int NV>
__device__ __forceinline__ void block_partials(const double (&v)[NV], int m, double* part) {
    __shared__ double sh[NV][THOMAS_THREADS];
#pragma unroll
    for (int k = 0; k < NV; k++) sh[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int w = THOMAS_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
#pragma unroll
            for (int k = 0; k < NV; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) part[((size_t)m * gridDim.x + blockIdx.x) * NV + k] = sh[k][0];
    }
}

// Compact fourth-order RHS and Thomas solve of one sweep (psolve.rs:285-327) for
// one (kx, ky) column per thread; member = blockIdx.y.  Writes ps and the new
// previous-iterate psa, and reduces the Parseval-weighted sums of
// (ps - psa_old)^2 and psa_old^2 per CTA into part[(m*gridDim.x + blk)*NV + {0,1}].
// NZS > 0: compile-time nz; the column is kept in registers between the forward
// elimination and the back substitution (ps is written once).
// NV = 3 (the reference sweeps of the mixed path) also writes the change of the
// sweep, D1 = ps_new - ps_old for levels 0..nz-1 in float32, and reduces the
// weighted sum of ps_new^2 into part[... + 2].
template <typename T, int NZS, int NV>
__global__ void __launch_bounds__(THOMAS_THREADS)
k_thomas(int ng, int nz_rt, int n2, const int* __restrict__ ctl, const T* __restrict__ SP,
         const double* __restrict__ htdv, const double* __restrict__ etdv, const double* __restrict__ ap,
         double* __restrict__ PS, double* __restrict__ XF, float* __restrict__ D1, float* __restrict__ Cr,
         double omega, double* __restrict__ part) {
    const int m = blockIdx.y;
    const int i = blockIdx.x * THOMAS_THREADS + threadIdx.x;
    const int nz = NZS ? NZS : nz_rt;
    const int L = nz + 1;
    double sn = 0.0, sd = 0.0, sx = 0.0;
    if (NZS && i < n2 && ctl[3 * m]) {
        const size_t cb = (size_t)m * L * n2 + i;
        const double api = ap[i];
        // every load of the column is issued before the dependent recurrences
        double sp[NZS ? NZS + 1 : 1], x[NZS ? NZS : 1], ed[NZS ? NZS : 1], old[NZS ? NZS + 1 : 1];
#pragma unroll
        for (int iz = 0; iz <= NZS; iz++) sp[iz] = (double)SP[cb + (size_t)iz * n2];
#pragma unroll
        for (int iz = 0; iz < NZS; iz++) x[iz] = htdv[i + (size_t)n2 * iz];
#pragma unroll
        for (int iz = 0; iz + 1 < NZS; iz++) ed[iz] = etdv[i + (size_t)n2 * iz];
#pragma unroll
        for (int iz = 0; iz <= NZS; iz++) old[iz] = PS[cb + (size_t)iz * n2];
        // forward elimination (x[iz] holds htdv(iz) until it is overwritten)
        x[0] = ((1.0 / 3.0) * sp[0] + (1.0 / 6.0) * sp[1]) * x[0];
#pragma unroll
        for (int iz = 1; iz < NZS; iz++) {
            const double g = (1.0 / 12.0) * (sp[iz - 1] + sp[iz + 1]) + (5.0 / 6.0) * sp[iz];
            x[iz] = (g - api * x[iz - 1]) * x[iz];
        }
#pragma unroll
        for (int iz = NZS - 2; iz >= 0; iz--) x[iz] += ed[iz] * x[iz + 1];
#pragma unroll
        for (int iz = 0; iz < NZS; iz++) {
            sn += (x[iz] - old[iz]) * (x[iz] - old[iz]);
            sd += old[iz] * old[iz];
            if (NV == 3) {
                PS[cb + (size_t)iz * n2] = x[iz];
                sx += x[iz] * x[iz];
                D1[cb + (size_t)iz * n2] = (float)(x[iz] - old[iz]);
                if (omega != 1.0) Cr[cb + (size_t)iz * n2] = (float)((omega - 1.0) * (x[iz] - old[iz]));
            } else {
                PS[cb + (size_t)iz * n2] = omega == 1.0 ? x[iz] : old[iz] + omega * (x[iz] - old[iz]);
            }
        }
        sn += old[NZS] * old[NZS];
        sd += old[NZS] * old[NZS];
        PS[cb + (size_t)NZS * n2] = 0.0;
        const int kx = i % ng, ky = i / ng;
        const double wgt = pweight(kx, ng) * pweight(ky, ng);
        sn *= wgt;
        sd *= wgt;
        sx *= wgt;
    } else if (!NZS && i < n2 && ctl[3 * m]) {
        const size_t cb = (size_t)m * L * n2 + i;
        const double api = ap[i];
        double spm = (double)SP[cb], spc = (double)SP[cb + n2];
        double x = ((1.0 / 3.0) * spm + (1.0 / 6.0) * spc) * htdv[i];
        XF[cb] = x;
#pragma unroll 4
        for (int iz = 1; iz < nz; iz++) {
            const double spp = (double)SP[cb + (size_t)(iz + 1) * n2];
            const double g = (1.0 / 12.0) * (spm + spp) + (5.0 / 6.0) * spc;
            x = (g - api * x) * htdv[i + (size_t)n2 * iz];
            XF[cb + (size_t)iz * n2] = x;
            spm = spc;
            spc = spp;
        }
        {
            const size_t p = cb + (size_t)nz * n2;
            const double old = PS[p];
            sn += old * old;
            sd += old * old;
            PS[p] = 0.0;
        }
        double xn = x;
        {
            const size_t p = cb + (size_t)(nz - 1) * n2;
            const double old = PS[p];
            sn += (xn - old) * (xn - old);
            sd += old * old;
            PS[p] = (NV == 3 || omega == 1.0) ? xn : old + omega * (xn - old);
            if (NV == 3) {
                sx += xn * xn;
                D1[p] = (float)(xn - old);
                if (omega != 1.0) Cr[p] = (float)((omega - 1.0) * (xn - old));
            }
        }
#pragma unroll 4
        for (int iz = nz - 2; iz >= 0; iz--) {
            const size_t p = cb + (size_t)iz * n2;
            const double xi = XF[p] + etdv[i + (size_t)n2 * iz] * xn;
            const double old = PS[p];
            sn += (xi - old) * (xi - old);
            sd += old * old;
            PS[p] = (NV == 3 || omega == 1.0) ? xi : old + omega * (xi - old);
            if (NV == 3) {
                sx += xi * xi;
                D1[p] = (float)(xi - old);
                if (omega != 1.0) Cr[p] = (float)((omega - 1.0) * (xi - old));
            }
            xn = xi;
        }
        const int kx = i % ng, ky = i / ng;
        const double wgt = pweight(kx, ng) * pweight(ky, ng);
        sn *= wgt;
        sd *= wgt;
        sx *= wgt;
    }
    if constexpr (NV == 3) {
        const double v[3] = {sn, sd, sx};
        block_partials<3>(v, m, part);
    } else {
        const double v[2] = {sn, sd};
        block_partials<2>(v, m, part);
    }
}

// Thomas solve of a float32 correction sweep of the mixed path: the compact RHS of
// the correction source SP32 (float32, levels 0..nz) and the solve in float64
// arithmetic give the correction c = T^-1 SP32 of the pressure against the last
// reference sweep's result (which ps holds).  The previous correction C is replaced;
// the weighted sum of (c_new - c_old)^2 goes to part[... * 3 + 0] (the numerator of
// errp; the control kernel divides by the reference sweep's sum of ps^2).
template <int NZS>
__global__ void __launch_bounds__(THOMAS_THREADS)
k_thomas_c(int ng, int nz_rt, int n2, const int* __restrict__ ctl, const float* __restrict__ SP32,
           const double* __restrict__ htdv, const double* __restrict__ etdv, const double* __restrict__ ap,
           float* __restrict__ Cr, double omega, double* __restrict__ XF, double* __restrict__ part) {
    const int m = blockIdx.y;
    const int i = blockIdx.x * THOMAS_THREADS + threadIdx.x;
    const int nz = NZS ? NZS : nz_rt;
    const int L = nz + 1;
    double sn = 0.0;
    if (NZS && i < n2 && ctl[3 * m]) {
        const size_t cb = (size_t)m * L * n2 + i;
        const double api = ap[i];
        double sp[NZS ? NZS + 1 : 1], x[NZS ? NZS : 1], ed[NZS ? NZS : 1], old[NZS ? NZS : 1];
#pragma unroll
        for (int iz = 0; iz <= NZS; iz++) sp[iz] = (double)SP32[cb + (size_t)iz * n2];
#pragma unroll
        for (int iz = 0; iz < NZS; iz++) x[iz] = htdv[i + (size_t)n2 * iz];
#pragma unroll
        for (int iz = 0; iz + 1 < NZS; iz++) ed[iz] = etdv[i + (size_t)n2 * iz];
#pragma unroll
        for (int iz = 0; iz < NZS; iz++) old[iz] = (double)Cr[cb + (size_t)iz * n2];
        x[0] = ((1.0 / 3.0) * sp[0] + (1.0 / 6.0) * sp[1]) * x[0];
#pragma unroll
        for (int iz = 1; iz < NZS; iz++) {
            const double g = (1.0 / 12.0) * (sp[iz - 1] + sp[iz + 1]) + (5.0 / 6.0) * sp[iz];
            x[iz] = (g - api * x[iz - 1]) * x[iz];
        }
#pragma unroll
        for (int iz = NZS - 2; iz >= 0; iz--) x[iz] += ed[iz] * x[iz + 1];
#pragma unroll
        for (int iz = 0; iz < NZS; iz++) {
            sn += (x[iz] - old[iz]) * (x[iz] - old[iz]);
            Cr[cb + (size_t)iz * n2] = (float)(omega == 1.0 ? x[iz] : old[iz] + omega * (x[iz] - old[iz]));
        }
        const int kx = i % ng, ky = i / ng;
        sn *= pweight(kx, ng) * pweight(ky, ng);
    } else if (!NZS && i < n2 && ctl[3 * m]) {
        const size_t cb = (size_t)m * L * n2 + i;
        const double api = ap[i];
        double spm = (double)SP32[cb], spc = (double)SP32[cb + n2];
        double x = ((1.0 / 3.0) * spm + (1.0 / 6.0) * spc) * htdv[i];
        XF[cb] = x;
#pragma unroll 4
        for (int iz = 1; iz < nz; iz++) {
            const double spp = (double)SP32[cb + (size_t)(iz + 1) * n2];
            const double g = (1.0 / 12.0) * (spm + spp) + (5.0 / 6.0) * spc;
            x = (g - api * x) * htdv[i + (size_t)n2 * iz];
            XF[cb + (size_t)iz * n2] = x;
            spm = spc;
            spc = spp;
        }
        double xn = x;
        {
            const size_t p = cb + (size_t)(nz - 1) * n2;
            const double old = (double)Cr[p];
            sn += (xn - old) * (xn - old);
            Cr[p] = (float)(omega == 1.0 ? xn : old + omega * (xn - old));
        }
#pragma unroll 4
        for (int iz = nz - 2; iz >= 0; iz--) {
            const size_t p = cb + (size_t)iz * n2;
            const double xi = XF[p] + etdv[i + (size_t)n2 * iz] * xn;
            const double old = (double)Cr[p];
            sn += (xi - old) * (xi - old);
            Cr[p] = (float)(omega == 1.0 ? xi : old + omega * (xi - old));
            xn = xi;
        }
        const int kx = i % ng, ky = i / ng;
        sn *= pweight(kx, ng) * pweight(ky, ng);
    }
    const double v[3] = {sn, 0.0, 0.0};
    block_partials<3>(v, m, part);
}

constexpr int CTRL_THREADS = 256;
constexpr int CTRL_MAX_MEMBERS = 256;

// Stop rule of one member (psolve.rs:89, 339-366).  One deliberate deviation: a
// relative change that is not finite (a NaN or an infinity anywhere in the member's
// pressure) ends the member's iteration with SW_ERR_PSOLVE_DIVERGED at any sweep.
// The reference's loop condition `while errp > toler` (psolve.rs:88) is false for a
// NaN, so there a non-finite state leaves the loop as if it had converged.
//
// Correction sweeps (kind != null, the mixed path): kind_now says whether the sweep
// just run was a float64 reference sweep (0) or a float32 correction sweep (1).  A
// reference sweep records its relative change in eref[m].  A member that goes on
// iterating asks for a new reference sweep (*want64) once its correction sweeps have
// stopped shrinking the change by 30% per sweep, or have shrunk it by 1e-6 against
// that record: the float32 rounding of a correction is relative to the distance from
// the reference point, so a nearer reference point lowers that floor.
//
// For a correction sweep the relative change is (weighted) |c_new - c_old| / |p1|,
// with |p1|^2 (the sum c of the reference sweep) kept in pnorm[m]: p1 + c_old is the
// previous iterate and |c_old| is small next to |p1|.
__device__ __forceinline__ void ctrl_member(int m, double a, double b, double c, int* ctl, double* errp,
                                                 double toler, int mixed, int nitmax, int* any, const int* kind,
                                                 int kind_now, double* eref, double* pnorm, int* want64) {
    {
        if (!ctl[3 * m]) return;
        if (kind && kind_now == 0) pnorm[m] = c;
        const double e = (kind && kind_now == 1) ? sqrt(a / (pnorm[m] + 1.0E-20)) : sqrt(a / (b + 1.0E-20));
        const double eprev = ctl[3 * m + 1] > 0 ? errp[m] : 1.0;
        const bool stagnated = mixed && e < 1.0E-4 && e > 0.7 * eprev;
        errp[m] = e;
        const int it = ctl[3 * m + 1];
        if (!isfinite(e) || (it > 0 && e > 1.0)) {
            ctl[3 * m + 2] = SW_ERR_PSOLVE_DIVERGED;
            ctl[3 * m] = 0;
            ctl[3 * m + 1] = it + 1;
            return;
        }
        ctl[3 * m + 1] = it + 1;
        if (!(e > toler) || stagnated || it + 1 >= nitmax) {
            ctl[3 * m] = 0;
            if (it + 1 >= nitmax && !(mixed && (!(e > toler) || stagnated))) ctl[3 * m + 2] = SW_ERR_PSOLVE_MAXITER;
        } else {
            atomicOr(any, 1);
            if (kind) {
                if (kind_now == 0) eref[m] = e;
                else if (e < 1.0E-6 * eref[m] || e > 0.7 * eprev) atomicOr(want64, 1);
            }
        }
    }
}

// Convergence control of one sweep (psolve.rs:89, 339-358): per member, the
// relative change errp from the CTA partials (fixed order), the divergence and
// iteration-cap statuses, and the mixed path's stop rule; then, inside a graph,
// the WHILE node's condition (any member still iterating).  Stop rule
// (psolve.rs:17, 89): float64, the reference's 1e-9 on the relative change;
// float32 transforms put a floor of ~1e-6 under that change, so the mixed path
// stops at 1e-6, or earlier once the change has stagnated (< 1e-4 and no longer
// shrinking by 30% per sweep).
// With kind set (the mixed path's correction sweeps), the kind of the next sweep is
// written to kind[0] and, inside a graph, to the conditions c64 / c32 of the two
// conditional sweep bodies.
// Partials: NV = 2 values per CTA (sn, sd), or 3 with the correction sweeps (sn,
// sd, sum of ps^2 of a reference sweep; sn alone for a correction sweep).
static __global__ void k_psolve_ctrl(int M, int nblk, int nv, const double* __restrict__ part, int* ctl, double* errp,
                                     double toler, int mixed, int nitmax, int use_cond, cudaGraphConditionalHandle cond,
                                     long long* nexec, int* kind, double* eref, double* pnorm,
                                     cudaGraphConditionalHandle c64, cudaGraphConditionalHandle c32) {
    __shared__ int any, want64;
    __shared__ double sums[3 * CTRL_MAX_MEMBERS];
    const int kind_now = kind ? kind[0] : 0;
    if (threadIdx.x == 0) {
        any = 0;
        want64 = 0;
    }
    // one warp per member: lane-strided partial sums, then a fixed shuffle tree
    // (deterministic order)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = CTRL_THREADS / 32;
    for (int m0 = 0; m0 < M; m0 += CTRL_MAX_MEMBERS) {
        const int mcount = (M - m0 < CTRL_MAX_MEMBERS) ? M - m0 : CTRL_MAX_MEMBERS;
        for (int mm = warp; mm < mcount; mm += nwarps) {
            const double* pm = part + (size_t)(m0 + mm) * nblk * nv;
            double a = 0.0, b = 0.0, c = 0.0;
#pragma unroll 8
            for (int k = lane; k < nblk; k += 32) {
                a += pm[nv * k];
                b += pm[nv * k + 1];
                if (nv == 3) c += pm[nv * k + 2];
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                a += __shfl_down_sync(0xffffffffu, a, off);
                b += __shfl_down_sync(0xffffffffu, b, off);
                c += __shfl_down_sync(0xffffffffu, c, off);
            }
            if (lane == 0) {
                sums[3 * mm] = a;
                sums[3 * mm + 1] = b;
                sums[3 * mm + 2] = c;
            }
        }
        __syncthreads();
        for (int mm = threadIdx.x; mm < mcount; mm += CTRL_THREADS)
            ctrl_member(m0 + mm, sums[3 * mm], sums[3 * mm + 1], sums[3 * mm + 2], ctl, errp, toler, mixed, nitmax,
                        &any, kind, kind_now, eref, pnorm, &want64);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int next = (kind_now == 1 && want64) ? 0 : 1;
        if (kind) kind[0] = next;
        if (use_cond) {
            nexec[kind_now] += 1;  // sweep bodies executed, per kind
            cudaGraphSetConditional(cond, any ? 1u : 0u);
            if (kind) {
                cudaGraphSetConditional(c64, (any && next == 0) ? 1u : 0u);
                cudaGraphSetConditional(c32, (any && next == 1) ? 1u : 0u);
            }
        }
    }
}

template <typename T>
struct Solver {
    int ng, nz, L, M, n2, ML;
    size_t nf;  // elements of one 3-D field for all members
    double t = 0.0;
    cudaStream_t st = nullptr;
    SpectralHost host;
    DeviceOps op;
    Fft2d<T> fft;

    // state (src/nhswps/mod.rs:87-148)
    DevBuf<T> u, v, w, z, zx, zy, r, ri, aa, zeta, pn, dpn;
    DevBuf<double> ps, qs, ds, gs;
    // persistent psolve coefficients
    DevBuf<T> sigx, sigy, cpt1, cpt2, sp0;
    // work fields
    std::vector<DevBuf<T>> wt;       // T-precision 3-D work fields
    std::vector<DevBuf<double>> wd;  // float64 3-D work fields (advance, psolve)
    DevBuf<double> plane_d;          // M*n2 float64 per-member planes (x4)
    DevBuf<T> plane_t;               // M*n2 T per-member planes (x4)
    DevBuf<double> red_partial, red_out;
    DevBuf<double> errp_d, diag_hist;
    DevBuf<int> ctrl;  // per member: active, iters, status
    double* h_pinned = nullptr;  // host staging for small readbacks
    int hist_cap = 4096;
    DevBuf<int> bin_off, bin_idx;  // elements of each |k| shell (CSR over kmag)
    DevBuf<double> bin_wt;         // 1/4 at k = 0, 1/2 on the axes, 1 elsewhere
    DevBuf<double> spec_d;         // 3 (kmax + 1) spectra
    DevBuf<float> snap;            // savegrid output staging: 6 n3 + 5 n2 floats
    // whole-step CUDA graphs (index: ggen) with device-side psolve loops
    cudaStream_t st_body = nullptr;
    cudaGraphExec_t step_exec[2] = {nullptr, nullptr};
    DevBuf<int> sweeps_dev;  // per member: sweep counts of the 3 psolve calls of the last step
    DevBuf<int> err_dev;     // sticky status of captured steps
    DevBuf<int> hist_dev;    // diagnostics rows recorded since the last read
    DevBuf<long long> sweep_exec;  // sweep bodies executed by graph launches, per kind (launch accounting)
    long long k_fixed[2] = {0, 0};  // kernels per step outside the sweep loops
    long long k_sweep = 0;          // kernels captured in one sweep loop body (both kinds)
    long long k_sweep_kind[2] = {0, 0};  // kernels a body runs when it is a reference / correction sweep
    // Mixed path: float32 correction sweeps on the float64 solver (T = double)
    bool refine32 = false;
    // Mixed path: the psolve set-up's products and filters through float32 transforms
    // (setup_w_sig_f32, setup_products<float>); the rest of the set-up stays float64.
    bool setup32 = true;
    Fft2d<float> f32;          // float32 transforms (intermediate lent by fft)
    // 11 float32 fields: 0..3 sweep planes (p, p_x, p_y, S1), 4 the correction source
    // SP32, 5..8 coefficient copies (sigx, sigy, cpt2, cpt1), 9 the last reference
    // sweep's change D1, 10 the correction C (the iterate is ps + C)
    DevBuf<float> r32;
    DevBuf<double> eref;       // per member: relative change of the last reference sweep
    DevBuf<double> pnorm;      // per member: weighted |ps|^2 after the last reference sweep
    double refine_toler = 1.0E-7;  // stop rule of the correction sweeps
    // Relaxation factor of the pressure iteration: each sweep's new iterate is
    // x + relax (G(x) - x), G one sweep (Thomas solve of the source at x).  1 (the
    // default) is the reference's iteration (psolve.rs:89-358); set_psolve_relax.
    double relax = 1.0;
    DevBuf<int> sweep_kind;    // kind of the next sweep: 0 reference (float64), 1 correction (float32)
    cudaStream_t st_if = nullptr;
    int host_kind = 0;         // host-driven loops: kind of the next sweep
    long long sweeps_run[2] = {0, 0};  // sweep launches so far: reference (float64) and correction (float32)
    float* R32(int i) { return r32.p + (size_t)i * nf; }
    int last_sweeps[3] = {0, 0, 0};

    static constexpr int NWT = 24;
    static constexpr int NWD = 12;

    Solver(int ng_, int nz_, int M_) : ng(ng_), nz(nz_), L(nz_ + 1), M(M_), n2(ng_ * ng_), ML(M_ * (nz_ + 1)) {
        require(ng >= 4 && ng % 2 == 0, SW_ERR_ARG, "ng must be even and >= 4");
        require(nz >= 2 && nz <= MAX_NZ, SW_ERR_ARG, "nz must be in [2, 128]");
        require(M >= 1, SW_ERR_ARG, "nmembers must be >= 1");
        FftPlan tmp;
        require(build_plan(ng, tmp) == SW_OK, SW_ERR_FACTORISE, "ng must factor into 2, 3 and 5");
        nf = (size_t)M * L * n2;
        SW_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        host.build(ng, nz);
        upload(op.hlap, host.hlap); upload(op.glap, host.glap); upload(op.rlap, host.rlap);
        upload(op.helm, host.helm); upload(op.c2g2, host.c2g2); upload(op.simp, host.simp);
        upload(op.rope, host.rope); upload(op.fope, host.fope); upload(op.filt, host.filt);
        upload(op.diss, host.diss); upload(op.opak, host.opak); upload(op.rdis, host.rdis);
        upload(op.ap, host.ap); upload(op.htdv, host.htdv); upload(op.etdv, host.etdv);
        upload(op.weight, host.weight); upload(op.theta, host.theta);
        upload(op.htd1, host.htd1); upload(op.etd1, host.etd1);
        fft.init(ng, 6 * ML);
        {
            const int nb = host.kmax + 1;
            std::vector<int> cnt(nb + 1, 0), off(nb + 1, 0), idx(n2);
            std::vector<double> wt_h(n2);
            for (int e = 0; e < n2; e++) cnt[host.kmag[e]]++;
            for (int k = 0; k < nb; k++) off[k + 1] = off[k] + cnt[k];
            std::vector<int> pos(off.begin(), off.end());
            for (int e = 0; e < n2; e++) idx[pos[host.kmag[e]]++] = e;
            for (int e = 0; e < n2; e++) {
                const int kx = e % ng, ky = e / ng;
                wt_h[e] = (kx == 0 && ky == 0) ? 0.25 : (kx == 0 || ky == 0) ? 0.5 : 1.0;
            }
            bin_off.alloc(nb + 1);
            bin_idx.alloc(n2);
            bin_wt.alloc(n2);
            SW_CUDA(cudaMemcpy(bin_off.p, off.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice));
            SW_CUDA(cudaMemcpy(bin_idx.p, idx.data(), sizeof(int) * n2, cudaMemcpyHostToDevice));
            upload(bin_wt, wt_h);
            spec_d.alloc((size_t)3 * nb);
        }
        for (auto* b : {&u, &v, &w, &z, &zx, &zy, &r, &ri, &aa, &zeta, &pn, &dpn, &sigx, &sigy, &cpt1, &cpt2, &sp0}) {
            b->alloc(nf);
            SW_CUDA(cudaMemset(b->p, 0, nf * sizeof(T)));
        }
        for (auto* b : {&ps, &qs, &ds, &gs}) {
            b->alloc(nf);
            SW_CUDA(cudaMemset(b->p, 0, nf * sizeof(double)));
        }
        wt.resize(NWT);
        for (auto& b : wt) b.alloc(nf);
        wd.resize(NWD);
        for (auto& b : wd) b.alloc(nf);
        plane_d.alloc((size_t)4 * M * n2);
        plane_t.alloc((size_t)4 * M * n2);
        red_partial.alloc((size_t)RED_MAX_CHUNKS * 8 * ML + 64);
        red_out.alloc((size_t)8 * ML + 64);
        errp_d.alloc((size_t)2 * M + 2);
        diag_hist.alloc((size_t)hist_cap * M * 3);
        ctrl.alloc((size_t)3 * M + 1);
        SW_CUDA(cudaMallocHost(&h_pinned, sizeof(double) * (16 * (size_t)M + 64)));
        SW_CUDA(cudaStreamCreateWithFlags(&st_body, cudaStreamNonBlocking));
        SW_CUDA(cudaStreamCreateWithFlags(&st_if, cudaStreamNonBlocking));
        sweeps_dev.alloc((size_t)3 * M);
        err_dev.alloc(1);
        hist_dev.alloc(1);
        sweep_exec.alloc(2);
        SW_CUDA(cudaMemset(sweep_exec.p, 0, 2 * sizeof(long long)));
        SW_CUDA(cudaMemset(sweeps_dev.p, 0, sizeof(int) * 3 * M));
        SW_CUDA(cudaMemset(err_dev.p, 0, sizeof(int)));
        SW_CUDA(cudaMemset(hist_dev.p, 0, sizeof(int)));
    }
    ~Solver() {
        if (st) cudaStreamSynchronize(st);
        for (auto& e : step_exec)
            if (e) cudaGraphExecDestroy(e);
        if (st_if) cudaStreamDestroy(st_if);
        if (st_body) cudaStreamDestroy(st_body);
        if (h_pinned) cudaFreeHost(h_pinned);
        if (st) cudaStreamDestroy(st);
    }

    // The mixed path on the float64 solver: pressure sweeps after the first of each
    // solve are float32 correction sweeps (sweep_correction), with float64 reference
    // sweeps wherever the control kernel asks for one.  Everything else stays float64.
    void enable_refine32() {
        if constexpr (sizeof(T) == 8) {
            if (refine32) return;
            f32.init(ng, 2 * fft.cap, reinterpret_cast<float*>(fft.midp));
            f32.set_chunk(f32.cap);
            r32.alloc((size_t)11 * nf);
            SW_CUDA(cudaMemset(r32.p, 0, sizeof(float) * 11 * nf));
            eref.alloc(M);
            SW_CUDA(cudaMemset(eref.p, 0, sizeof(double) * M));
            pnorm.alloc(M);
            SW_CUDA(cudaMemset(pnorm.p, 0, sizeof(double) * M));
            sweep_kind.alloc(1);
            SW_CUDA(cudaMemset(sweep_kind.p, 0, sizeof(int)));
            xh.alloc(9 * nf);
            SW_CUDA(cudaMemset(xh.p, 0, sizeof(double) * 9 * nf));
            xflag.alloc(9);
            SW_CUDA(cudaMemset(xflag.p, 0, 9 * sizeof(int)));
            SW_CUDA(cudaStreamSynchronize(st));
            for (auto& e : step_exec)
                if (e) {
                    SW_CUDA(cudaGraphExecDestroy(e));
                    e = nullptr;
                }
            refine32 = true;
        } else {
            require(false, SW_ERR_ARG, "correction sweeps need the float64 solver");
        }
    }

    // Mixed path: the first iterate of each pressure solve of a step is predicted
    // from the previous steps, where the reference starts from the previous solve's
    // solution.  A step solves three times, in slots j = 0 (at the step's start, the
    // ggen solve), 1 (after the predictor) and 2 (after the corrector).  At the start
    // of slot j of step n, ps holds the solution of the solve before it (slot j - 1
    // of step n, or slot 2 of step n - 1).  With D1, D2, D3 the changes between the
    // same two slots one, two and three steps earlier, the change is extrapolated
    // over the steps by a polynomial of degree 0, 1 or 2:
    //   ps + D1,   ps + 2 D1 - D2,   ps + 3 D1 - 3 D2 + D3,
    // the highest degree whose history is recorded and whose added term is smaller
    // than the one before it (|D1 - D2| <= |D1|, |D1 - 2 D2 + D3| <= |D1 - D2|).
    // H[j], G[j], K[j] (xh slots 0..2, 3..5, 6..8) hold the solution of slot j one,
    // two and three steps earlier; then K[j-1] <- G[j-1] <- H[j-1] <- the old ps.
    // The iteration and its fixed point are unchanged; a nearer first iterate needs
    // fewer sweeps.  A member whose predicted change is larger than ps itself
    // (|D1| > |ps|: a history from another run), or whose history is not yet
    // written, keeps ps.  Steps without the ggen solve clear the history.
    void extrapolate_guess(int j) {
        const int n2 = this->n2, L = this->L, ML = this->ML, M = this->M;
        const int jp = (j + 2) % 3;
        const long long nm = (long long)L * n2;
        double* PS = ps;
        double *Hj = xh.p + (size_t)j * nf, *Hp = xh.p + (size_t)jp * nf;
        double *Gj = xh.p + (size_t)(3 + j) * nf, *Gp = xh.p + (size_t)(3 + jp) * nf;
        double *Kj = xh.p + (size_t)(6 + j) * nf, *Kp = xh.p + (size_t)(6 + jp) * nf;
        int* fl = xflag.p;
        double* sums = red_out.p + (size_t)6 * ML;  // 4 M values (red_out holds 8 ML + 64)
        reduce_groups<4>(st, M, nm, 0u,
            [=] __device__(int g, long long i) {
                const size_t p = (size_t)g * nm + i;
                const double d1 = Hj[p] - Hp[p];
                const double d2 = Gj[p] - Gp[p];
                const double d3 = Kj[p] - Kp[p];
                RedVals<4> rv;
                rv.v[0] = d1 * d1;
                rv.v[1] = PS[p] * PS[p];
                rv.v[2] = (d1 - d2) * (d1 - d2);
                rv.v[3] = (d1 - 2.0 * d2 + d3) * (d1 - 2.0 * d2 + d3);
                return rv;
            }, red_partial.p, sums);
        for_planes4(st, ML, n2, [=] __device__(int q, int i) {
            const int m = q / L;
            const size_t p = (size_t)q * n2 + i;
            double c[4], hb[4], gb[4];
            ld4(PS + p, c);
            ld4(Hp + p, hb);
            ld4(Gp + p, gb);
            const double* sm = sums + 4 * m;
            const int deg = !(fl[j] && fl[jp] && sm[0] <= sm[1]) ? -1
                            : !(fl[3 + j] && fl[3 + jp] && sm[2] <= sm[0]) ? 0
                            : !(fl[6 + j] && fl[6 + jp] && sm[3] <= sm[2]) ? 1 : 2;
            if (deg >= 0) {
                double o[4], ha[4];
                ld4(Hj + p, ha);
                if (deg == 0) {
#pragma unroll
                    for (int e = 0; e < 4; e++) o[e] = c[e] + (ha[e] - hb[e]);
                } else {
                    double ga[4];
                    ld4(Gj + p, ga);
                    if (deg == 1) {
#pragma unroll
                        for (int e = 0; e < 4; e++) o[e] = c[e] + (2.0 * (ha[e] - hb[e]) - (ga[e] - gb[e]));
                    } else {
                        double ka[4], kb[4];
                        ld4(Kj + p, ka);
                        ld4(Kp + p, kb);
#pragma unroll
                        for (int e = 0; e < 4; e++)
                            o[e] = c[e] + (3.0 * (ha[e] - hb[e]) - 3.0 * (ga[e] - gb[e]) + (ka[e] - kb[e]));
                    }
                }
                st4(PS + p, o);
            }
            st4(Kp + p, gb);
            st4(Gp + p, hb);
            st4(Hp + p, c);
        });
        for_cols(st, 1, [=] __device__(int) {
            fl[6 + jp] = fl[3 + jp];
            fl[3 + jp] = fl[jp];
            fl[jp] = 1;
        });
    }
    void reset_guess_history() {
        if (xflag.p) SW_CUDA(cudaMemsetAsync(xflag.p, 0, 9 * sizeof(int), st));
    }

    // Stop rule of the correction sweeps (the mixed path); the captured step graphs
    // hold the old value, so they are dropped.
    void set_refine_toler(double toler) {
        require(refine32, SW_ERR_STATE, "the pressure tolerance is set on SW_MIXED contexts only");
        require(toler > 0.0 && toler < 1.0, SW_ERR_ARG, "tolerance must be in (0, 1)");
        SW_CUDA(cudaStreamSynchronize(st));
        for (auto& e : step_exec)
            if (e) {
                SW_CUDA(cudaGraphExecDestroy(e));
                e = nullptr;
            }
        refine_toler = toler;
    }

    // Relaxation factor of the pressure iteration (see relax).  The iteration's
    // fixed point does not depend on it; the stop rule measures the unrelaxed change
    // |G(x) - x|.  The captured step graphs hold the old value, so they are dropped.
    void set_psolve_relax(double omega) {
        require(omega > 0.0 && omega <= 1.0, SW_ERR_ARG, "relaxation factor must be in (0, 1]");
        SW_CUDA(cudaStreamSynchronize(st));
        for (auto& e : step_exec)
            if (e) {
                SW_CUDA(cudaGraphExecDestroy(e));
                e = nullptr;
            }
        relax = omega;
    }

    // Planes per 2-D transform launch pair; the captured step graphs hold the old
    // launch sequence, so they are dropped and re-captured on the next step.
    int set_fft_chunk(int planes) {
        if (planes <= 0) return fft.chunk;  // query
        if (planes == fft.chunk || (planes > fft.cap && fft.chunk == fft.cap)) return fft.chunk;
        SW_CUDA(cudaStreamSynchronize(st));
        for (auto& e : step_exec)
            if (e) {
                SW_CUDA(cudaGraphExecDestroy(e));
                e = nullptr;
            }
        const int c = fft.set_chunk(planes);
        if constexpr (sizeof(T) == 8) {
            if (refine32) f32.set_chunk(2 * c);  // the float32 engine: the same bytes per chunk
        }
        return c;
    }

    // Single-pass cluster transforms at n = 256 on or off (off by default); like the
    // chunk, the captured step graphs hold the old launches, so they are dropped.
    bool set_fft_single_pass(int enable) {
        if (enable < 0 || (enable != 0) == fft.single_pass) return fft.single_pass;
        SW_CUDA(cudaStreamSynchronize(st));
        for (auto& e : step_exec)
            if (e) {
                SW_CUDA(cudaGraphExecDestroy(e));
                e = nullptr;
            }
        if constexpr (sizeof(T) == 8) {
            if (refine32) f32.set_single_pass(enable != 0);
        }
        return fft.set_single_pass(enable != 0);
    }

    // Two-stream chunk pipeline of the batched 2-D transforms on or off (enable < 0
    // queries); like the chunk, the captured step graphs hold the old launches.
    bool set_fft_overlap(int enable) {
        if (enable < 0 || (enable != 0) == fft.overlap) return fft.overlap;
        SW_CUDA(cudaStreamSynchronize(st));
        for (auto& e : step_exec)
            if (e) {
                SW_CUDA(cudaGraphExecDestroy(e));
                e = nullptr;
            }
        const bool on = fft.set_overlap(enable != 0);
        if constexpr (sizeof(T) == 8) {
            if (refine32) {
                f32.set_overlap(on);
                f32.set_chunk(2 * fft.chunk);
            }
        }
        return on;
    }

    // Columns per tile of the n = 256 tile passes (16 or 32); like the chunk, the
    // captured step graphs hold the old launches, so they are dropped.
    int set_fft_tile(int columns) {
        if (columns <= 0 || columns == fft.tc) return fft.tc;
        SW_CUDA(cudaStreamSynchronize(st));
        for (auto& e : step_exec)
            if (e) {
                SW_CUDA(cudaGraphExecDestroy(e));
                e = nullptr;
            }
        return fft.set_tile(columns);
    }

    // Autotuner of the 2-D transform launches: times `reps` forward + inverse
    // transforms of the pressure sweep's batch (3*nz planes per member) for each
    // tile width the length has compiled kernels for (n = 256: 16 and 32 columns)
    // and each chunk (cap, cap/2, ... down to 8 planes), with CUDA events on the
    // context's stream, and keeps the fastest pair.  The batch runs on scratch
    // buffers allocated for the measurement.  Writes up to maxc (tile, chunk, ms
    // per transform pair) rows; returns the chosen chunk and sets *tile_out.
    int autotune_fft(int reps, int maxc, int* tiles, int* cand, int* ovls, float* ms, int* ncand, int* tile_out,
                     int* ovl_out) {
        if (reps < 1) reps = 1;
        const int nb = std::min(fft.cap, 3 * nz * M);
        DevBuf<T> a, b;
        a.alloc((size_t)nb * n2);
        b.alloc((size_t)nb * n2);
        SW_CUDA(cudaMemsetAsync(a.p, 0, sizeof(T) * (size_t)nb * n2, st));
        const int ng = this->ng;
        T *A = a.p, *B = b.p;
        cudaEvent_t e0, e1;
        SW_CUDA(cudaEventCreate(&e0));
        SW_CUDA(cudaEventCreate(&e1));
        std::vector<int> tcs;
        if (ng == FFT_R_N) tcs = {16, 32};
        else tcs = {fft.tc};
        int best = fft.chunk, best_tc = fft.tc, best_ovl = fft.overlap ? 1 : 0, k = 0;
        float best_ms = 1e30f;
        try {
            for (int ovl = 0; ovl < 2; ovl++) {
                set_fft_overlap(ovl);
                // chunks: the capacity halved down to 8 planes; with the pipeline, half and a
                // quarter of the capacity only.  Smaller pipelined chunks win on the plain
                // transform timed here (their intermediate stays in L2) but lose on whole
                // steps, whose fused transforms read and write more fields per plane
                // (measured at ng=256, 16 members: 51-plane chunks 2-3% slower per step
                // than 408-plane chunks, which are 3-5% faster than no pipeline).
                std::vector<int> cands;
                if (ovl) {
                    if (fft.cap / 2 >= 1) cands.push_back(fft.cap / 2);
                    if (fft.cap / 4 >= 8) cands.push_back(fft.cap / 4);
                } else {
                    for (int c = fft.cap; c >= 1; c /= 2) {
                        cands.push_back(c);
                        if (c / 2 < 8) break;
                    }
                }
                for (int tcv : tcs) {
                    set_fft_tile(tcv);
                    for (int c : cands) {
                        set_fft_chunk(c);
                        for (int r = -1; r < reps; r++) {  // r = -1: untimed warm-up
                            if (r == 0) SW_CUDA(cudaEventRecord(e0, st));
                            fft.ptospc(st, nb, [=] __device__(int o, int iy, int ix) -> T { return A[((size_t)o * ng + ix) * ng + iy]; },
                                       [=] __device__(int o, int kx, int ky, T v) { B[((size_t)o * ng + ky) * ng + kx] = v; });
                            fft.spctop(st, nb, [=] __device__(int o, int kx, int ky) -> T { return B[((size_t)o * ng + ky) * ng + kx]; },
                                       [=] __device__(int o, int iy, int ix, T v) { A[((size_t)o * ng + ix) * ng + iy] = v; });
                        }
                        SW_CUDA(cudaEventRecord(e1, st));
                        SW_CUDA(cudaEventSynchronize(e1));
                        float t = 0.f;
                        SW_CUDA(cudaEventElapsedTime(&t, e0, e1));
                        t /= (float)reps;
                        if (k < maxc) {
                            if (tiles) tiles[k] = fft.tc;
                            if (cand) cand[k] = fft.chunk;
                            if (ovls) ovls[k] = ovl;
                            if (ms) ms[k] = t;
                        }
                        k++;
                        if (t < best_ms) {
                            best_ms = t;
                            best = fft.chunk;
                            best_tc = fft.tc;
                            best_ovl = ovl;
                        }
                    }
                }
            }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ncand) *ncand = k < maxc ? k : maxc;
        const int ovl_set = set_fft_overlap(best_ovl) ? 1 : 0;
        if (ovl_out) *ovl_out = ovl_set;
        const int tc_set = set_fft_tile(best_tc);
        if (tile_out) *tile_out = tc_set;
        return set_fft_chunk(best);
    }

    T* W(int i) { return wt[i].p; }
    double* WD(int i) { return wd[i].p; }
    T* field_t(int f) {
        switch (f) {
            case SW_U: return u; case SW_V: return v; case SW_W: return w; case SW_Z: return z;
            case SW_ZX: return zx; case SW_ZY: return zy; case SW_R: return r; case SW_RI: return ri;
            case SW_AA: return aa; case SW_ZETA: return zeta; case SW_PN: return pn; case SW_DPN: return dpn;
            default: return nullptr;
        }
    }
    double* field_d(int f) {
        switch (f) {
            case SW_PS: return ps; case SW_QS: return qs; case SW_DS: return ds; case SW_GS: return gs;
            default: return nullptr;
        }
    }

    // ======================================================================
    // main_invert (src/spectral/mod.rs:305-417)
    // ======================================================================
    void main_invert() {
        NvtxRange nv("main_invert");
        const int ng = this->ng, n2 = this->n2, L = this->L, ML = this->ML;
        const double *QS = qs, *DS = ds, *GS = gs, *rope = op.rope, *rlap = op.rlap, *wgt = op.weight;
        double* wkh = plane_d.p;
        // vertical average of eta = gamma/f^2 - q/f, times rope
        for_cols(st, M * n2, [=] __device__(int c) {
            const int m = c / n2, i = c - m * n2;
            double s = 0.0;
            #pragma unroll 4
            for (int iz = 0; iz < L; iz++) {
                const size_t p = (size_t)(m * L + iz) * n2 + i;
                s += wgt[iz] * (COFI * (COFI * GS[p] - QS[p]));
            }
            wkh[c] = s * rope[i];
        });
        T *R = r, *U = u, *V = v, *ZE = zeta;
        T *SU = W(8), *SV = W(9);  // spectral u, v for psolve's set-up in this stage
        // spectral r and zeta staged in W(10), W(17) (written by P5 and source
        // before any read there): one streaming pass forms the four spectral inputs
        // of an element, then a plain transform takes them to physical space
        T *SR = W(10), *SZ = W(17);
        for_planes(st, ML, n2, [=] __device__(int q, int i) {
            const int m = q / L;
            const int kx = i % ng, ky = i / ng;
            const double* qsq = QS + (size_t)q * n2;
            const double* dsq = DS + (size_t)q * n2;
            const double* gsq = GS + (size_t)q * n2;
            const double* wk = wkh + (size_t)m * n2;
            auto wka = [&](int j) { return COFI * (COFI * gsq[j] - qsq[j]) - wk[j]; };
            auto wkb = [&](int j) { return qsq[j] + COF * wka(j); };
            const size_t p = (size_t)q * n2 + i;
            SR[p] = (T)wka(i);
            SZ[p] = (T)wkb(i);
            const int mx = mirror(kx, ng) + ng * ky, my = kx + ng * mirror(ky, ng);
            SU[p] = (T)(dmul(kx, ng) * (rlap[mx] * dsq[mx]) - dmul(ky, ng) * (rlap[my] * wkb(my)));
            SV[p] = (T)(dmul(ky, ng) * (rlap[my] * dsq[my]) + dmul(kx, ng) * (rlap[mx] * wkb(mx)));
        });
        fft.spctop(st, 4 * ML,
            plane_ld([=] __device__(int o) {
                const int which = o & 3, q = o >> 2;
                return PairLd<T>{(which == 0 ? SR : which == 1 ? SZ : which == 2 ? SU : SV) + (size_t)q * n2, ng};
            }),
            plane_st([=] __device__(int o) {
                const int which = o & 3, q = o >> 2;
                return PairSt<T>{(which == 0 ? R : which == 1 ? ZE : which == 2 ? U : V) + (size_t)q * n2, ng};
            }));
        // mean flow (uio, vio): per-plane sums of u*r and v*r
        double* sums = red_out.p;
        reduce_groups<2>(st, ML, n2, 0u,
            [=] __device__(int g, long long i) {
                const size_t p = (size_t)g * n2 + i;
                RedVals<2> rv;
                rv.v[0] = (double)U[p] * (double)R[p];
                rv.v[1] = (double)V[p] * (double)R[p];
                return rv;
            }, red_partial.p, sums);
        // (uio, vio) per member once, after the per-plane sums (not per element)
        const double dsumi = 1.0 / (double)(ng * ng);
        double* mean = sums + 2 * ML;
        for_cols(st, M, [=] __device__(int m) {
            double uio = 0.0, vio = 0.0;
            for (int iz = 0; iz < L; iz++) {
                uio -= wgt[iz] * sums[2 * (m * L + iz)] * dsumi;
                vio -= wgt[iz] * sums[2 * (m * L + iz) + 1] * dsumi;
            }
            mean[2 * m] = uio;
            mean[2 * m + 1] = vio;
        });
        for_planes4(st, ML, n2, [=] __device__(int q, int i) {
            const int m = q / L;
            const double uio = mean[2 * m], vio = mean[2 * m + 1];
            const size_t p = (size_t)q * n2 + i;
            T uv[4], vv[4];
            ld4(U + p, uv);
            ld4(V + p, vv);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                uv[e] = (T)((double)uv[e] + uio);
                vv[e] = (T)((double)vv[e] + vio);
            }
            st4(U + p, uv);
            st4(V + p, vv);
        });
    }

    // ======================================================================
    // vertical (src/nhswps/vertical.rs:8-143)
    // ======================================================================
    void vertical() {
        const int ng = this->ng, n2 = this->n2, L = this->L, nz = this->nz, M = this->M, ML = this->ML;
        const double dz2 = (HBAR / (double)nz) / 2.0;
        const double *theta = op.theta, *filt = op.filt, *DS = ds;
        T *Z = z, *R = r, *U = u, *V = v, *WW = w, *ZX = zx, *ZY = zy, *AA = aa;
        T *S1 = W(0), *SA = W(1), *SB = W(2), *RS = W(3);
        // float32 path: the derivatives are taken of the deviation z - theta, kept
        // apart from z so that its float32 rounding is relative to the deviation
        // (theta is horizontally uniform, so the derivatives are the same).
        const bool mixed = sizeof(T) == 4;
        T* zd = W(20);
        // z by trapezoidal integration of rho'_theta, then + theta
        for_cols(st, M * n2, [=] __device__(int c) {
            const int m = c / n2, i = c - m * n2;
            T* zc = Z + (size_t)m * L * n2 + i;
            const T* rc = R + (size_t)m * L * n2 + i;
            double prev = dz2 * ((double)rc[0] + (double)rc[n2]);
            zc[n2] = (T)prev;
            if (mixed) zd[(size_t)m * L * n2 + i + n2] = (T)prev;
            #pragma unroll 4
            for (int iz = 1; iz < nz; iz++) {
                prev = prev + dz2 * ((double)rc[(size_t)iz * n2] + (double)rc[(size_t)(iz + 1) * n2]);
                zc[(size_t)(iz + 1) * n2] = (T)prev;
                if (mixed) zd[(size_t)m * L * n2 + i + (size_t)(iz + 1) * n2] = (T)prev;
            }
            for (int iz = 1; iz <= nz; iz++) zc[(size_t)iz * n2] = (T)((double)zc[(size_t)iz * n2] + theta[iz]);
        });
        // z_x, z_y for iz = 1..nz
        const int Mnz = M * nz;
        const T* zsrc = mixed ? zd : Z;
        fft.ptospc(st, Mnz,
            [=] __device__(int o, int iy, int ix) -> T {
                const int m = o / nz, iz = 1 + o % nz;
                return zsrc[(size_t)(m * L + iz) * n2 + iy + ng * ix];
            },
            [=] __device__(int o, int kx, int ky, T val) {
                const int m = o / nz, iz = 1 + o % nz;
                S1[(size_t)(m * L + iz) * n2 + kx + ng * ky] = val;
            });
        fft.spctop(st, 2 * Mnz,
            [=] __device__(int o, int kx, int ky) -> T {
                const int which = o / Mnz, q = o - which * Mnz, m = q / nz, iz = 1 + q % nz;
                const T* s = S1 + (size_t)(m * L + iz) * n2;
                if (which == 0) return dmul_t(kx, ng, s[mirror(kx, ng) + ng * ky]);
                return dmul_t(ky, ng, s[kx + ng * mirror(ky, ng)]);
            },
            [=] __device__(int o, int iy, int ix, T val) {
                const int which = o / Mnz, q = o - which * Mnz, m = q / nz, iz = 1 + q % nz;
                (which == 0 ? ZX : ZY)[(size_t)(m * L + iz) * n2 + iy + ng * ix] = val;
            });
        // A = filt * (d/dx(u r) + d/dy(v r))
        fft.ptospc(st, 2 * ML,
            [=] __device__(int o, int iy, int ix) -> T {
                const int which = o / ML, q = o - which * ML;
                const size_t p = (size_t)q * n2 + iy + ng * ix;
                return (which == 0 ? U[p] : V[p]) * R[p];
            },
            [=] __device__(int o, int kx, int ky, T val) {
                const int which = o / ML, q = o - which * ML;
                (which == 0 ? SA : SB)[(size_t)q * n2 + kx + ng * ky] = val;
            });
        for_planes(st, ML, n2, [=] __device__(int q, int i) {
            const int kx = i % ng, ky = i / ng;
            const T* a = SA + (size_t)q * n2;
            const T* b = SB + (size_t)q * n2;
            const double wkb = dmul(kx, ng) * (double)a[mirror(kx, ng) + ng * ky];
            const double wkc = dmul(ky, ng) * (double)b[kx + ng * mirror(ky, ng)];
            AA[(size_t)q * n2 + i] = (T)(filt[i] * (wkb + wkc));
        });
        // rsrc = -(A + delta) in physical space
        fft.spctop(st, ML,
            [=] __device__(int q, int kx, int ky) -> T {
                const size_t p = (size_t)q * n2 + kx + ng * ky;
                return (T)((double)AA[p] + DS[p]);
            },
            [=] __device__(int q, int iy, int ix, T val) { RS[(size_t)q * n2 + iy + ng * ix] = -val; });
        // w by trapezoidal integration
        for_cols(st, M * n2, [=] __device__(int c) {
            const int m = c / n2, i = c - m * n2;
            T* wc = WW + (size_t)m * L * n2 + i;
            const T* sc = RS + (size_t)m * L * n2 + i;
            double prev = dz2 * ((double)sc[0] + (double)sc[n2]);
            wc[n2] = (T)prev;
            #pragma unroll 4
            for (int iz = 1; iz < nz; iz++) {
                prev = prev + dz2 * ((double)sc[(size_t)iz * n2] + (double)sc[(size_t)(iz + 1) * n2]);
                wc[(size_t)(iz + 1) * n2] = (T)prev;
            }
        });
        // w += deal(u z_x + v z_y), iz = 1..nz
        fft.ptospc(st, Mnz,
            [=] __device__(int o, int iy, int ix) -> T {
                const int m = o / nz, iz = 1 + o % nz;
                const size_t p = (size_t)(m * L + iz) * n2 + iy + ng * ix;
                return U[p] * ZX[p] + V[p] * ZY[p];
            },
            [=] __device__(int o, int kx, int ky, T val) {
                const int m = o / nz, iz = 1 + o % nz;
                const int i = kx + ng * ky;
                S1[(size_t)(m * L + iz) * n2 + i] = (T)(filt[i] * (double)val);
            });
        fft.spctop(st, Mnz,
            [=] __device__(int o, int kx, int ky) -> T {
                const int m = o / nz, iz = 1 + o % nz;
                return S1[(size_t)(m * L + iz) * n2 + kx + ng * ky];
            },
            [=] __device__(int o, int iy, int ix, T val) {
                const int m = o / nz, iz = 1 + o % nz;
                const size_t p = (size_t)(m * L + iz) * n2 + iy + ng * ix;
                WW[p] = WW[p] + val;
            });
    }

    // ======================================================================
    // coeffs (src/nhswps/coeffs.rs:8-101): sigx, sigy (x2), cpt1, cpt2
    // ======================================================================
    void coeffs() {
        const int ng = this->ng, n2 = this->n2, L = this->L, nz = this->nz, ML = this->ML;
        const double qdzi = (1.0 / 4.0) * (1.0 / (HBAR / (double)nz));
        const double* filt = op.filt;
        T *RI = ri, *ZX = zx, *ZY = zy, *SX = sigx, *SY = sigy, *C1 = cpt1, *C2 = cpt2;
        T *Sx = W(4), *Sy = W(5), *Sc = W(6), *D = W(7);
        fft.ptospc(st, 2 * ML,
            [=] __device__(int o, int iy, int ix) -> T {
                const int which = o / ML, q = o - which * ML;
                const size_t p = (size_t)q * n2 + iy + ng * ix;
                return RI[p] * (which == 0 ? ZX[p] : ZY[p]);
            },
            [=] __device__(int o, int kx, int ky, T val) {
                const int which = o / ML, q = o - which * ML, i = kx + ng * ky;
                (which == 0 ? Sx : Sy)[(size_t)q * n2 + i] = (T)(filt[i] * (double)val);
            });
        fft.spctop(st, 2 * ML,
            [=] __device__(int o, int kx, int ky) -> T {
                const int which = o / ML, q = o - which * ML;
                return (which == 0 ? Sx : Sy)[(size_t)q * n2 + kx + ng * ky];
            },
            [=] __device__(int o, int iy, int ix, T val) {
                const int which = o / ML, q = o - which * ML;
                (which == 0 ? SX : SY)[(size_t)q * n2 + iy + ng * ix] = val;
            });
        fft.ptospc(st, ML,
            [=] __device__(int q, int iy, int ix) -> T {
                const size_t p = (size_t)q * n2 + iy + ng * ix;
                return T(1) - RI[p] * RI[p] - SX[p] * SX[p] - SY[p] * SY[p];
            },
            [=] __device__(int q, int kx, int ky, T val) {
                const int i = kx + ng * ky;
                Sc[(size_t)q * n2 + i] = (T)(filt[i] * (double)val);
            });
        // cpt2 = deal(...) (all levels), D = div(sig) for iz >= 1
        fft.spctop(st, 2 * ML,
            [=] __device__(int o, int kx, int ky) -> T {
                const int which = o / ML, q = o - which * ML;
                if (which == 0) return Sc[(size_t)q * n2 + kx + ng * ky];
                const T* a = Sx + (size_t)q * n2;
                const T* b = Sy + (size_t)q * n2;
                return (T)(dmul(ky, ng) * (double)b[kx + ng * mirror(ky, ng)] +
                           dmul(kx, ng) * (double)a[mirror(kx, ng) + ng * ky]);
            },
            [=] __device__(int o, int iy, int ix, T val) {
                const int which = o / ML, q = o - which * ML;
                (which == 0 ? C2 : D)[(size_t)q * n2 + iy + ng * ix] = val;
            });
        for_planes(st, ML, n2, [=] __device__(int q, int i) {
            const int m = q / L, iz = q % L;
            const T* c2 = C2 + (size_t)m * L * n2 + i;
            const size_t p = (size_t)q * n2 + i;
            double val;
            if (iz == 0)
                val = qdzi * (4.0 * (double)c2[n2] - 3.0 * (double)c2[0] - (double)c2[2 * (size_t)n2]);
            else if (iz < nz)
                val = qdzi * ((double)c2[(size_t)(iz + 1) * n2] - (double)c2[(size_t)(iz - 1) * n2]) + (double)D[p];
            else
                val = qdzi * (3.0 * (double)c2[(size_t)nz * n2] + (double)c2[(size_t)(nz - 2) * n2] -
                              4.0 * (double)c2[(size_t)(nz - 1) * n2]) + (double)D[p];
            C1[p] = (T)val;
            SX[p] = SX[p] * T(2);
            SY[p] = SY[p] * T(2);
        });
    }

    // theta-derivative of a level field at level iz (cpsource.rs:46-103)
    static __device__ __forceinline__ double tderiv(const T* col, int iz, int nz, int n2, double hdzi) {
        if (iz == 0) return hdzi * (4.0 * (double)col[n2] - 3.0 * (double)col[0] - (double)col[2 * (size_t)n2]);
        if (iz == nz)
            return hdzi * (3.0 * (double)col[(size_t)nz * n2] + (double)col[(size_t)(nz - 2) * n2] -
                           4.0 * (double)col[(size_t)(nz - 1) * n2]);
        return hdzi * ((double)col[(size_t)(iz + 1) * n2] - (double)col[(size_t)(iz - 1) * n2]);
    }
    // tderiv of four consecutive columns (col 16-byte aligned for float, 32 for double)
    static __device__ __forceinline__ void tderiv4(const T* col, int iz, int nz, int n2, double hdzi, double (&d)[4]) {
        T a[4], b[4];
        if (iz == 0 || iz == nz) {
            T c[4];
            if (iz == 0) {
                ld4(col + n2, a);
                ld4(col, b);
                ld4(col + 2 * (size_t)n2, c);
#pragma unroll
                for (int e = 0; e < 4; e++) d[e] = hdzi * (4.0 * (double)a[e] - 3.0 * (double)b[e] - (double)c[e]);
            } else {
                ld4(col + (size_t)nz * n2, a);
                ld4(col + (size_t)(nz - 2) * n2, b);
                ld4(col + (size_t)(nz - 1) * n2, c);
#pragma unroll
                for (int e = 0; e < 4; e++) d[e] = hdzi * (3.0 * (double)a[e] + (double)b[e] - 4.0 * (double)c[e]);
            }
            return;
        }
        ld4(col + (size_t)(iz + 1) * n2, a);
        ld4(col + (size_t)(iz - 1) * n2, b);
#pragma unroll
        for (int e = 0; e < 4; e++) d[e] = hdzi * ((double)a[e] - (double)b[e]);
    }

    // ======================================================================
    // cpsource (src/nhswps/cpsource.rs:13-261): sp0
    // Work: W(8..10) spectral u,v,w; W(11..16) ux,uy,vx,vy,wx,wy; W(17..19)
    // spectral/physical wkp,wkq,wkr; plane_t = hsrc.
    // ======================================================================
    void cpsource() {
        const int ng = this->ng, n2 = this->n2, L = this->L, nz = this->nz, M = this->M, ML = this->ML;
        const double hdzi = (1.0 / 2.0) * (1.0 / (HBAR / (double)nz));
        const double *filt = op.filt, *glap = op.glap;
        T *Z = z, *U = u, *V = v, *WW = w, *RI = ri, *ZE = zeta, *ZX = zx, *ZY = zy, *SP0 = sp0;
        T *Su = W(8), *Sv = W(9), *Sw = W(10);
        T *UX = W(11), *UY = W(12), *VX = W(13), *VY = W(14), *WX = W(15), *WY = W(16);
        T *Pp = W(17), *Pq = W(18), *Pr = W(19);
        T* hs = plane_t.p;        // M planes: spectral then physical hsrc
        T* hsrc = plane_t.p + (size_t)M * n2;
        // float32 path: -g Lap(h) and f zeta nearly cancel (geostrophic balance), so
        // their sum is formed in float64 spectral space from qs and gs (h and zeta as
        // main_invert defines them) and only the small residual is transformed.
        const bool mixed = sizeof(T) == 4;
        T* HZ = W(21);
        if (mixed) {
            const double *QS = qs, *GS = gs, *rope = op.rope, *wgt = op.weight;
            const double dz2 = (HBAR / (double)nz) / 2.0;
            double* hspec = plane_d.p;  // per member: spectral h deviation (trapezoid of rho')
            for_cols(st, M * n2, [=] __device__(int c) {
                const int m = c / n2, i = c - m * n2;
                double w = 0.0;
                #pragma unroll 4
                for (int iz = 0; iz < L; iz++) {
                    const size_t p = (size_t)(m * L + iz) * n2 + i;
                    w += wgt[iz] * (COFI * (COFI * GS[p] - QS[p]));
                }
                w *= rope[i];
                double h = 0.0, prev = 0.0;
                #pragma unroll 4
                for (int iz = 0; iz < L; iz++) {
                    const size_t p = (size_t)(m * L + iz) * n2 + i;
                    const double wka = COFI * (COFI * GS[p] - QS[p]) - w;
                    if (iz > 0) h += dz2 * (prev + wka);
                    prev = wka;
                }
                hspec[c] = h;
                hspec[(size_t)M * n2 + c] = w;
            });
            fft.spctop(st, ML,
                [=] __device__(int q, int kx, int ky) -> T {
                    const int m = q / L, i = kx + ng * ky;
                    const size_t p = (size_t)q * n2 + i;
                    const double w = hspec[(size_t)M * n2 + (size_t)m * n2 + i];
                    const double zeta_s = QS[p] + COF * (COFI * (COFI * GS[p] - QS[p]) - w);
                    return (T)(glap[i] * hspec[(size_t)m * n2 + i] + COF * zeta_s);
                },
                [=] __device__(int q, int iy, int ix, T val) { HZ[(size_t)q * n2 + iy + ng * ix] = val; });
        }
        // hsrc = -g Lap(h) in physical space
        if (!mixed) fft.ptospc(st, M,
            [=] __device__(int m, int iy, int ix) -> T { return Z[(size_t)(m * L + nz) * n2 + iy + ng * ix]; },
            [=] __device__(int m, int kx, int ky, T val) {
                const int i = kx + ng * ky;
                hs[(size_t)m * n2 + i] = (T)((double)val * glap[i]);
            });
        if (!mixed) fft.spctop(st, M,
            [=] __device__(int m, int kx, int ky) -> T { return hs[(size_t)m * n2 + kx + ng * ky]; },
            [=] __device__(int m, int iy, int ix, T val) { hsrc[(size_t)m * n2 + iy + ng * ix] = val; });
        // horizontal derivatives of u, v, w
        fft.ptospc(st, 3 * ML,
            [=] __device__(int o, int iy, int ix) -> T {
                const int which = o / ML, q = o - which * ML;
                const size_t p = (size_t)q * n2 + iy + ng * ix;
                return which == 0 ? U[p] : which == 1 ? V[p] : WW[p];
            },
            [=] __device__(int o, int kx, int ky, T val) {
                const int which = o / ML, q = o - which * ML;
                (which == 0 ? Su : which == 1 ? Sv : Sw)[(size_t)q * n2 + kx + ng * ky] = val;
            });
        fft.spctop(st, 6 * ML,
            [=] __device__(int o, int kx, int ky) -> T {
                const int which = o / ML, q = o - which * ML;
                const T* s = (which < 2 ? Su : which < 4 ? Sv : Sw) + (size_t)q * n2;
                if ((which & 1) == 0) return dmul_t(kx, ng, s[mirror(kx, ng) + ng * ky]);
                return dmul_t(ky, ng, s[kx + ng * mirror(ky, ng)]);
            },
            [=] __device__(int o, int iy, int ix, T val) {
                const int which = o / ML, q = o - which * ML;
                T* out = which == 0 ? UX : which == 1 ? UY : which == 2 ? VX : which == 3 ? VY : which == 4 ? WX : WY;
                out[(size_t)q * n2 + iy + ng * ix] = val;
            });
        // dealiased products wkp (iz>=1), wkq (all iz), wkr (iz>=1)
        fft.ptospc(st, 3 * ML,
            [=] __device__(int o, int iy, int ix) -> T {
                const int which = o / ML, q = o - which * ML, m = q / L, iz = q % L;
                const int i = iy + ng * ix;
                const size_t p = (size_t)q * n2 + i;
                const size_t cb = (size_t)m * L * n2 + i;
                const double wt = tderiv(WW + cb, iz, nz, n2, hdzi);
                if (which == 1 && iz == 0) return (T)((double)RI[p] * wt);
                if (iz == 0) return T(0);
                const double ut = tderiv(U + cb, iz, nz, n2, hdzi);
                const double vt = tderiv(V + cb, iz, nz, n2, hdzi);
                if (which == 0) return (T)(vt * (double)ZX[p] - ut * (double)ZY[p]);
                if (which == 1) return (T)((double)UY[p] * vt - ut * (double)VY[p]);
                return (T)(ut * (double)VX[p] - (double)UX[p] * vt);
            },
            [=] __device__(int o, int kx, int ky, T val) {
                const int which = o / ML, q = o - which * ML, i = kx + ng * ky;
                (which == 0 ? Su : which == 1 ? Sv : Sw)[(size_t)q * n2 + i] = (T)(filt[i] * (double)val);
            });
        fft.spctop(st, 3 * ML,
            [=] __device__(int o, int kx, int ky) -> T {
                const int which = o / ML, q = o - which * ML;
                return (which == 0 ? Su : which == 1 ? Sv : Sw)[(size_t)q * n2 + kx + ng * ky];
            },
            [=] __device__(int o, int iy, int ix, T val) {
                const int which = o / ML, q = o - which * ML;
                (which == 0 ? Pp : which == 1 ? Pq : Pr)[(size_t)q * n2 + iy + ng * ix] = val;
            });
        // second dealiased product (iz >= 1), then sp0
        fft.ptospc(st, ML,
            [=] __device__(int q, int iy, int ix) -> T {
                const int m = q / L, iz = q % L;
                if (iz == 0) return T(0);
                const int i = iy + ng * ix;
                const size_t p = (size_t)q * n2 + i;
                const size_t cb = (size_t)m * L * n2 + i;
                const double ut = tderiv(U + cb, iz, nz, n2, hdzi);
                const double vt = tderiv(V + cb, iz, nz, n2, hdzi);
                const double wt = tderiv(WW + cb, iz, nz, n2, hdzi);
                double wkq = (double)Pq[p] * (double)ZX[p] + (double)Pr[p] * (double)ZY[p] - (double)WY[p] * vt;
                wkq += ((double)UX[p] + (double)VY[p]) * wt - (double)WX[p] * ut;
                return (T)wkq;
            },
            [=] __device__(int q, int kx, int ky, T val) {
                const int i = kx + ng * ky;
                Sw[(size_t)q * n2 + i] = (T)(filt[i] * (double)val);
            });
        fft.spctop(st, ML,
            [=] __device__(int q, int kx, int ky) -> T { return Sw[(size_t)q * n2 + kx + ng * ky]; },
            [=] __device__(int q, int iy, int ix, T val) {
                const int m = q / L, iz = q % L;
                const int i = iy + ng * ix;
                const size_t p = (size_t)q * n2 + i;
                const double ux = UX[p], uy = UY[p], vx = VX[p], vy = VY[p];
                double s;
                if (mixed) {
                    const double hz = HZ[p];  // -g Lap(h) + f zeta
                    if (iz == 0) {
                        s = hz + 2.0 * (ux * vy - uy * vx + (double)Pq[p] * (ux + vy));
                    } else {
                        const double rip = RI[p];
                        s = hz - COF * (rip * (double)Pp[p]) + 2.0 * (rip * (double)val);
                        s += 2.0 * (ux * vy - uy * vx);
                    }
                } else {
                    const double hsv = (double)hsrc[(size_t)m * n2 + i];
                    if (iz == 0) {
                        const double wkq = Pq[p];
                        s = hsv + COF * (double)ZE[p];
                        s += 2.0 * (ux * vy - uy * vx + wkq * (ux + vy));
                    } else {
                        const double rip = RI[p];
                        s = hsv + COF * ((double)ZE[p] - rip * (double)Pp[p]) + 2.0 * (rip * (double)val);
                        s += 2.0 * (ux * vy - uy * vx);
                    }
                }
                SP0[p] = (T)s;
            });
    }

    // ======================================================================
    // psolve (src/nhswps/psolve.rs:16-411)
    // Work: W(0..3) A,B,C,D physical sweep terms; W(4) sp (spectral source);
    // PS holds the previous iterate until the Thomas kernel replaces it; WD(1) is the
    // forward-elimination scratch of the streamed Thomas path and, after the loop,
    // the compact RHS for dp/dtheta.
    // ctrl: [active, iters, status] per member; errp_d: errp per member.
    // Returns member-0 status.
    // ======================================================================
    void psolve_prepare(int nitmax) {
        require(nz >= 3, SW_ERR_ARG, "psolve needs nz >= 3");
        (void)nitmax;
        if (fused_prepare) {
            psolve_prepare_fused();
            prepare_refine();
            return;
        }
        const int ng = this->ng, n2 = this->n2, ML = this->ML;
        const double* filt = op.filt;
        T *R = r, *RI = ri, *PN = pn;
        double* PS = ps;
        // ri = 1/(1+r), dealiased
        T* Sr = W(0);
        fft.ptospc(st, ML,
            [=] __device__(int q, int iy, int ix) -> T { return T(1) / (R[(size_t)q * n2 + iy + ng * ix] + T(1)); },
            [=] __device__(int q, int kx, int ky, T val) {
                const int i = kx + ng * ky;
                Sr[(size_t)q * n2 + i] = (T)(filt[i] * (double)val);
            });
        fft.spctop(st, ML,
            [=] __device__(int q, int kx, int ky) -> T { return Sr[(size_t)q * n2 + kx + ng * ky]; },
            [=] __device__(int q, int iy, int ix, T val) { RI[(size_t)q * n2 + iy + ng * ix] = val; });
        vertical();
        coeffs();
        cpsource();
        int* ctl = ctrl.p;
        // spectral pressure of the first guess, all levels: ps = ptospc(pn).  The sweep
        // reads levels 0..nz-1 only (ps(nz) = 0 in psolve.rs); the first Thomas solve
        // takes ps(nz) into the residual as the previous iterate and then zeroes it.
        fft.ptospc(st, ML,
            [=] __device__(int q, int iy, int ix) -> T { return PN[(size_t)q * n2 + iy + ng * ix]; },
            [=] __device__(int q, int kx, int ky, T val) { PS[(size_t)q * n2 + kx + ng * ky] = (double)val; });
        for_cols(st, M, [=] __device__(int m) {
            ctl[3 * m] = 1;
            ctl[3 * m + 1] = 0;
            ctl[3 * m + 2] = SW_OK;
        });
        prepare_refine();
    }

    // Mixed path: float32 copies of the sweep coefficients for the correction sweeps,
    // and the first sweep of the solve is a reference sweep.
    void prepare_refine() {
        host_kind = 0;
        if constexpr (sizeof(T) == 8) {
            if (!refine32) return;
            const int n2 = this->n2, ML = this->ML;
            const double *SX = sigx, *SY = sigy, *CC2 = cpt2, *CC1 = cpt1;
            float *X = R32(5), *Y = R32(6), *Z2 = R32(7), *Z1 = R32(8), *Cr = R32(10);
            int* kd = sweep_kind.p;
            for_planes4(st, ML, n2, [=] __device__(int q, int i) {
                const size_t p = (size_t)q * n2 + i;
                if (q == 0 && i == 0) kd[0] = 0;
                double v[4];
                float f[4] = {0.f, 0.f, 0.f, 0.f};
                st4(Cr + p, f);
                ld4(SX + p, v);
                for (int e = 0; e < 4; e++) f[e] = (float)v[e];
                st4(X + p, f);
                ld4(SY + p, v);
                for (int e = 0; e < 4; e++) f[e] = (float)v[e];
                st4(Y + p, f);
                ld4(CC2 + p, v);
                for (int e = 0; e < 4; e++) f[e] = (float)v[e];
                st4(Z2 + p, f);
                ld4(CC1 + p, v);
                for (int e = 0; e < 4; e++) f[e] = (float)v[e];
                st4(Z1 + p, f);
            });
        }
    }

    // psolve's set-up with vertical, coeffs and cpsource fused into eight large
    // batched transforms (the standalone vertical()/coeffs()/cpsource() keep the
    // reference's one-function-at-a-time order for the per-function API).  Same
    // arithmetic except that linear steps are merged: the spectral w used for
    // w_x, w_y is ptospc(w before the correction) + the correction's spectrum,
    // which equals ptospc(w after it).  ux, uy, vx, vy are left in W(11..14) for
    // source() of the same stage (u, v do not change in between).
    void psolve_prepare_fused() {
        NvtxRange nv("psolve_setup");
        const int ng = this->ng, n2 = this->n2, L = this->L, nz = this->nz, M = this->M, ML = this->ML;
        const int Mnz = M * nz;
        const bool mixed = sizeof(T) == 4;
        const double dz2 = (HBAR / (double)nz) / 2.0;
        const double *filt = op.filt, *glap = op.glap, *theta = op.theta;
        const double *DS = ds, *QS = qs, *GS = gs;
        double* PS = ps;
        T *R = r, *U = u, *V = v, *WW = w, *Z = z, *ZX = zx, *ZY = zy, *RI = ri, *AA = aa, *PN = pn;
        T *SIGX = sigx, *SIGY = sigy;
        T *Sr = W(0), *S1 = W(1), *SA = W(2), *SB = W(3), *Sx = W(17), *Sy = W(18), *D = W(7);
        T *RS = W(5), *Sd = W(6), *Su = W(8), *Sv = W(9), *Sw = W(10);
        T *UX = W(11), *UY = W(12), *VX = W(13), *VY = W(14), *WX = W(15), *WY = W(16);
        T* HZ = W(21);
        T* hs = plane_t.p;
        T* hsrc = plane_t.p + (size_t)M * n2;
        double* hspec = plane_d.p;
        // P0: z by trapezoidal integration (+ theta)
        for_cols(st, M * n2, [=] __device__(int c) {
            const int m = c / n2, i = c - m * n2;
            T* zc = Z + (size_t)m * L * n2 + i;
            const T* rc = R + (size_t)m * L * n2 + i;
            double prev = dz2 * ((double)rc[0] + (double)rc[n2]);
            zc[n2] = (T)(prev + theta[1]);
#pragma unroll 4
            for (int iz = 1; iz < nz; iz++) {
                prev = prev + dz2 * ((double)rc[(size_t)iz * n2] + (double)rc[(size_t)(iz + 1) * n2]);
                zc[(size_t)(iz + 1) * n2] = (T)(prev + theta[iz + 1]);
            }
        });
        if (mixed) {
            // The float32 path takes the spectrum of z - theta from float64 data
            // instead of transforming float32 z: main_invert sets r = spctop(rhat)
            // with rhat = cofi (cofi gs - qs) - <.>, so the trapezoid of rhat over the
            // levels is exactly the spectrum of z - theta.  Transforming float32 z
            // would put white rounding noise into z_x, z_y that the k factor of the
            // derivative amplifies.  The same loop gives the spectral h deviation
            // (the top level) and the vertical mean for cpsource's HZ term.
            const double *rope = op.rope, *wgt = op.weight;
            for_cols(st, M * n2, [=] __device__(int c) {
                const int m = c / n2, i = c - m * n2;
                double wv = 0.0;
                for (int iz = 0; iz < L; iz++) {
                    const size_t p = (size_t)(m * L + iz) * n2 + i;
                    wv += wgt[iz] * (COFI * (COFI * GS[p] - QS[p]));
                }
                wv *= rope[i];
                double h = 0.0, prev = 0.0;
                for (int iz = 0; iz < L; iz++) {
                    const size_t p = (size_t)(m * L + iz) * n2 + i;
                    const double wka = COFI * (COFI * GS[p] - QS[p]) - wv;
                    if (iz > 0) {
                        h += dz2 * (prev + wka);
                        S1[p] = (T)h;
                    }
                    prev = wka;
                }
                hspec[c] = h;
                hspec[(size_t)M * n2 + c] = wv;
            });
        }
        // P1: forward transforms of everything physical that is known now (z only on
        // the float64 path; the float32 path filled S1 above)
        // Inside advance (hints set by the step), main_invert of this stage has just
        // written the spectra of u and v to Su, Sv, and the previous pressure solve
        // of this step left its solution in ps (= ptospc(pn)), so those forward
        // transforms are skipped.
        // The first 3 ML planes are 1/(1+r), u r, v r level-major (adjacent planes
        // share r, u, v through L2).
        const bool uv_ready = hint_uv_spec, ps_ready = hint_ps_guess;
        const int o_z = 3 * ML, o_p = o_z + (mixed ? 0 : Mnz);
        const int o_u = o_p + (ps_ready ? 0 : ML), o_v = o_u + (uv_ready ? 0 : ML), o_h = o_v + (uv_ready ? 0 : ML);
        const int n1 = o_h + (mixed ? 0 : M);
        // (plane-bound functors: the field, level and product of a plane are chosen
        // once per tile; pairs of columns move as one vector access)
        fft.ptospc(st, n1,
            plane_ld([=] __device__(int o) {
                int kind = 0;  // 0 plain, 1 1/(1+r), 2 (u or v) r
                const T *s = nullptr, *rr = nullptr;
                if (o < o_z) {
                    const int q = o / 3, which = o - 3 * q;
                    rr = R + (size_t)q * n2;
                    s = (which == 1 ? U : V) + (size_t)q * n2;
                    kind = which == 0 ? 1 : 2;
                } else if (o < o_p) {
                    const int k = o - o_z, m = k / nz, iz = 1 + k % nz;
                    s = Z + (size_t)(m * L + iz) * n2;
                } else if (o < o_u) {
                    s = PN + (size_t)(o - o_p) * n2;
                } else if (o < o_v) {
                    s = U + (size_t)(o - o_u) * n2;
                } else if (o < o_h) {
                    s = V + (size_t)(o - o_v) * n2;
                } else {
                    s = Z + (size_t)((o - o_h) * L + nz) * n2;
                }
                return [=](int iy, int ix) {
                    const int pi = iy + ng * ix;
                    if (kind == 0) return ldv2(s + pi);
                    const auto r2 = ldv2(rr + pi);
                    if (kind == 1) return mk2(T(1) / (r2.x + T(1)), T(1) / (r2.y + T(1)));
                    const auto v2 = ldv2(s + pi);
                    return mk2(v2.x * r2.x, v2.y * r2.y);
                };
            }),
            plane_st([=] __device__(int o) {
                int kind = 0;  // 0 plain, 1 times a float64 operator, 2 float64 destination
                T* d = nullptr;
                double* dd = nullptr;
                const double* opd = filt;
                if (o < o_z) {
                    const int q = o / 3, which = o - 3 * q;
                    d = (which == 0 ? Sr : which == 1 ? SA : SB) + (size_t)q * n2;
                    kind = which == 0 ? 1 : 0;
                } else if (o < o_p) {
                    const int k = o - o_z, m = k / nz, iz = 1 + k % nz;
                    d = S1 + (size_t)(m * L + iz) * n2;
                } else if (o < o_u) {  // first-guess ps, all levels (see psolve_prepare)
                    dd = PS + (size_t)(o - o_p) * n2;
                    kind = 2;
                } else if (o < o_v) {
                    d = Su + (size_t)(o - o_u) * n2;
                } else if (o < o_h) {
                    d = Sv + (size_t)(o - o_v) * n2;
                } else {
                    d = hs + (size_t)(o - o_h) * n2;
                    opd = glap;
                    kind = 1;
                }
                return [=](int kx, int ky, T a, T b, int mk) {
                    const int i = kx + ng * ky;
                    if (kind == 2) {
                        stv2m(dd + i, mk, (double)a, (double)b);
                        return;
                    }
                    if (kind == 1) {
                        const double2 f = ldv2_ro(opd + i);
                        a = (T)(f.x * (double)a);
                        b = (T)(f.y * (double)b);
                    }
                    stv2m(d + i, mk, a, b);
                };
            }));
        // P2: inverse transforms: ri, z_x, z_y, rsrc (with A), u/v derivatives, hsrc or HZ
        const int q_x = ML, q_r = ML + 2 * Mnz, q_d = q_r + ML, q_h = q_d + 4 * ML;
        const int n2t = q_h + (mixed ? ML : M);
        fft.spctop(st, n2t,
            plane_ld([=] __device__(int o) {
                int kind = 0;  // 0/1/2 value, d/dx, d/dy of s; 3 rsrc (plane b); 4 HZ (plane b)
                const T* s = nullptr;
                size_t b = 0;
                if (o < q_x) {
                    s = Sr + (size_t)o * n2;
                } else if (o < q_r) {  // z_x, z_y of one level adjacent
                    const int k = o - q_x, kk = k >> 1, m = kk / nz, iz = 1 + kk % nz;
                    s = S1 + (size_t)(m * L + iz) * n2;
                    kind = 1 + (k & 1);
                } else if (o < q_d) {
                    b = (size_t)(o - q_r) * n2;
                    kind = 3;
                } else if (o < q_h) {  // u_x, u_y, v_x, v_y of one level adjacent
                    const int k = o - q_d, which = k & 3, q = k >> 2;
                    s = (which < 2 ? Su : Sv) + (size_t)q * n2;
                    kind = 1 + (which & 1);
                } else if (!mixed) {
                    s = hs + (size_t)(o - q_h) * n2;
                } else {
                    b = (size_t)(o - q_h);
                    kind = 4;
                }
                return [=](int kx, int ky) {
                    if (kind <= 2) return spec_pair(s, kind, kx, ky, ng);
                    const int i = kx + ng * ky;
                    if (kind == 3) {
                        const int myo = ng * mirror(ky, ng);
                        const double dy = dmul(ky, ng);
                        const double2 fl = ldv2_ro(filt + i);
                        const auto sb = ldv2(SB + b + kx + myo);
                        const double2 dsv = ldv2(DS + b + i);
                        const double wkb0 = dmul(kx, ng) * (double)SA[b + mirror(kx, ng) + ng * ky];
                        const double wkb1 = dmul(kx + 1, ng) * (double)SA[b + mirror(kx + 1, ng) + ng * ky];
                        const T a0 = (T)(fl.x * (wkb0 + dy * (double)sb.x));
                        const T a1 = (T)(fl.y * (wkb1 + dy * (double)sb.y));
                        stv2m(AA + b + i, 3, a0, a1);
                        return mk2((T)((double)a0 + dsv.x), (T)((double)a1 + dsv.y));
                    }
                    const int q = (int)b, m = q / L;
                    auto hz = [&](int j) {
                        const size_t p = (size_t)q * n2 + j;
                        const double wv = hspec[(size_t)M * n2 + (size_t)m * n2 + j];
                        const double zeta_s = QS[p] + COF * (COFI * (COFI * GS[p] - QS[p]) - wv);
                        return (T)(glap[j] * hspec[(size_t)m * n2 + j] + COF * zeta_s);
                    };
                    return mk2(hz(i), hz(i + 1));
                };
            }),
            plane_st([=] __device__(int o) {
                T* d;
                bool neg = false;
                if (o < q_x) {
                    d = RI + (size_t)o * n2;
                } else if (o < q_r) {
                    const int k = o - q_x, which = k & 1, kk = k >> 1, m = kk / nz, iz = 1 + kk % nz;
                    d = (which == 0 ? ZX : ZY) + (size_t)(m * L + iz) * n2;
                } else if (o < q_d) {
                    d = RS + (size_t)(o - q_r) * n2;
                    neg = true;
                } else if (o < q_h) {
                    const int k = o - q_d, which = k & 3, q = k >> 2;
                    d = (which == 0 ? UX : which == 1 ? UY : which == 2 ? VX : VY) + (size_t)q * n2;
                } else {
                    d = (mixed ? HZ : hsrc) + (size_t)(o - q_h) * n2;
                }
                return [=](int iy, int ix, T a, T b, int mk) {
                    if (neg) {
                        a = -a;
                        b = -b;
                    }
                    stv2m(d + iy + ng * ix, mk, a, b);
                };
            }));
        // P3: w by trapezoidal integration of rsrc
        for_cols(st, M * n2, [=] __device__(int c) {
            const int m = c / n2, i = c - m * n2;
            T* wc = WW + (size_t)m * L * n2 + i;
            const T* sc = RS + (size_t)m * L * n2 + i;
            double prev = dz2 * ((double)sc[0] + (double)sc[n2]);
            wc[n2] = (T)prev;
#pragma unroll 4
            for (int iz = 1; iz < nz; iz++) {
                prev = prev + dz2 * ((double)sc[(size_t)iz * n2] + (double)sc[(size_t)(iz + 1) * n2]);
                wc[(size_t)(iz + 1) * n2] = (T)prev;
            }
        });
        // P4/P5: the spectrum of w, the w correction u z_x + v z_y and ri z_x, ri z_y
        // (dealiased), then w_x, w_y, the corrected w, sigx, sigy and div(sig).  On
        // the mixed path the correction and the sig terms run through float32
        // transforms (setup_w_sig_f32).
        bool split45 = false;
        if constexpr (sizeof(T) == 8) {
            if (refine32 && setup32) {
                setup_w_sig_f32();
                split45 = true;
            }
        }
        if (!split45) {
            // P4: w, the w correction u z_x + v z_y (dealiased), ri z_x, ri z_y
            fft.ptospc(st, 2 * Mnz + 2 * ML,
                plane_ld([=] __device__(int o) {
                    int kind = 0;  // 0 w, 1 u z_x + v z_y, 2 ri z_x or ri z_y
                    size_t p0;
                    const T* zz = ZX;
                    if (o < 2 * Mnz) {
                        const int which = o / Mnz, k = o - which * Mnz, m = k / nz, iz = 1 + k % nz;
                        p0 = (size_t)(m * L + iz) * n2;
                        kind = which;
                    } else {
                        const int k = o - 2 * Mnz, which = k & 1, q = k >> 1;  // ri z_x, ri z_y of one level adjacent
                        p0 = (size_t)q * n2;
                        zz = which == 0 ? ZX : ZY;
                        kind = 2;
                    }
                    return [=](int iy, int ix) {
                        const size_t p = p0 + iy + ng * ix;
                        if (kind == 0) return ldv2(WW + p);
                        if (kind == 2) {
                            const auto r2 = ldv2(RI + p), z2 = ldv2(zz + p);
                            return mk2(r2.x * z2.x, r2.y * z2.y);
                        }
                        const auto u2 = ldv2(U + p), zx2 = ldv2(ZX + p), v2 = ldv2(V + p), zy2 = ldv2(ZY + p);
                        return mk2(u2.x * zx2.x + v2.x * zy2.x, u2.y * zx2.y + v2.y * zy2.y);
                    };
                }),
                plane_st([=] __device__(int o) {
                    T* d;
                    bool filtered = true;
                    if (o < 2 * Mnz) {
                        const int which = o / Mnz, k = o - which * Mnz, m = k / nz, iz = 1 + k % nz;
                        d = (which == 0 ? Sw : Sd) + (size_t)(m * L + iz) * n2;
                        filtered = which != 0;
                    } else {
                        const int k = o - 2 * Mnz, which = k & 1, q = k >> 1;
                        d = (which == 0 ? Sx : Sy) + (size_t)q * n2;
                    }
                    return [=](int kx, int ky, T a, T b, int mk) {
                        const int i = kx + ng * ky;
                        if (filtered) {
                            const double2 f = ldv2_ro(filt + i);
                            a = (T)(f.x * (double)a);
                            b = (T)(f.y * (double)b);
                        }
                        stv2m(d + i, mk, a, b);
                    };
                }));
            // P5: w correction, w_x, w_y, sigx, sigy, div(sig)
            fft.spctop(st, 4 * Mnz + 2 * ML,
                plane_ld([=] __device__(int o) {
                    int kind = 0;  // 0 plain s, 1/2 d/dx, d/dy of w + correction, 3 div(sig)
                    const T* s = nullptr;
                    size_t b = 0;
                    if (o < 3 * Mnz) {  // correction, w_x, w_y of one level adjacent
                        const int k = o / 3, which = o - 3 * k, m = k / nz, iz = 1 + k % nz;
                        b = (size_t)(m * L + iz) * n2;
                        s = Sd + b;
                        kind = which;
                    } else if (o < 3 * Mnz + 2 * ML) {
                        const int k = o - 3 * Mnz, which = k / ML, q = k - which * ML;
                        s = (which == 0 ? Sx : Sy) + (size_t)q * n2;
                    } else {
                        const int k = o - 3 * Mnz - 2 * ML, m = k / nz, iz = 1 + k % nz;
                        b = (size_t)(m * L + iz) * n2;
                        kind = 3;
                    }
                    return [=](int kx, int ky) {
                        if (kind == 0) return ldv2(s + kx + ng * ky);
                        if (kind == 1) {
                            const int j0 = mirror(kx, ng) + ng * ky, j1 = mirror(kx + 1, ng) + ng * ky;
                            return mk2((T)(dmul(kx, ng) * ((double)Sw[b + j0] + (double)Sd[b + j0])),
                                       (T)(dmul(kx + 1, ng) * ((double)Sw[b + j1] + (double)Sd[b + j1])));
                        }
                        const size_t my = b + kx + ng * mirror(ky, ng);
                        const double dy = dmul(ky, ng);
                        if (kind == 2) {
                            const auto w2 = ldv2(Sw + my), d2 = ldv2(Sd + my);
                            return mk2((T)(dy * ((double)w2.x + (double)d2.x)), (T)(dy * ((double)w2.y + (double)d2.y)));
                        }
                        const auto y2 = ldv2(Sy + my);
                        const double x0 = (double)Sx[b + mirror(kx, ng) + ng * ky];
                        const double x1 = (double)Sx[b + mirror(kx + 1, ng) + ng * ky];
                        return mk2((T)(dy * (double)y2.x + dmul(kx, ng) * x0), (T)(dy * (double)y2.y + dmul(kx + 1, ng) * x1));
                    };
                }),
                plane_st([=] __device__(int o) {
                    T* d;
                    bool add = false;
                    if (o < 3 * Mnz) {
                        const int k = o / 3, which = o - 3 * k, m = k / nz, iz = 1 + k % nz;
                        d = (which == 0 ? WW : which == 1 ? WX : WY) + (size_t)(m * L + iz) * n2;
                        add = which == 0;
                    } else if (o < 3 * Mnz + 2 * ML) {
                        const int k = o - 3 * Mnz, which = k / ML, q = k - which * ML;
                        d = (which == 0 ? SIGX : SIGY) + (size_t)q * n2;
                    } else {
                        const int k = o - 3 * Mnz - 2 * ML, m = k / nz, iz = 1 + k % nz;
                        d = D + (size_t)(m * L + iz) * n2;
                    }
                    return [=](int iy, int ix, T a, T b, int mk) {
                        T* dp = d + iy + ng * ix;
                        if (add) {
                            const auto w2 = ldv2(dp);
                            a = w2.x + a;
                            b = w2.y + b;
                        }
                        stv2m(dp, mk, a, b);
                    };
                }));
        }
        // P6..P10: cpt2, cpsource's dealiased products, cpt1, sp0 (setup_products);
        // on the mixed path their transforms run in float32 with float32 staging
        bool tail32 = false;
        if constexpr (sizeof(T) == 8) {
            if (refine32 && setup32) {
                float *F4 = R32(4), *F5 = R32(5), *F6 = R32(6), *F7 = R32(7), *F8 = R32(8);
                setup_products<float>(f32, F4, F5, F6, F7, F4, F5, F6, F7, F5, F6, F7, R32(3), F8, F8, F8);
                tail32 = true;
            }
        }
        if (!tail32)
            setup_products<T>(fft, W(8), W(9), W(10), W(17), W(19), W(0), W(1), W(2), W(3), W(5), W(6), W(7), W(8),
                              W(0), W(9));
        int* ctl = ctrl.p;
        for_cols(st, M, [=] __device__(int m) {
            ctl[3 * m] = 1;
            ctl[3 * m + 1] = 0;
            ctl[3 * m + 2] = SW_OK;
        });
    }

    // P6..P10 of psolve_prepare_fused (coeffs.rs:8-101, cpsource.rs:13-261): cpt2's
    // argument and cpsource's three dealiased products, staged in S planes G0..G3
    // and transformed by eng (forward with the filter into Sc, Spp, Spq, Spr, back
    // into cpt2, Pp, Pq, Pr); cpt1 = 0.5 d(cpt2)/dtheta + div(sig) (D) and sig *= 2;
    // the second dealiased product (G -> Sq2 -> Gq) and sp0.  S = T with the solver's
    // own transforms, or S = float with the float32 engine on the mixed path: these
    // products and filters are the set-up terms whose float32 rounding moves the
    // 10-step result by <= 2e-8 rel-L2 at ng=256 (an attribution with the oracle;
    // the z, u, v, w derivative transforms, h and the u r, v r terms stay float64).
    template <typename S, class E>
    void setup_products(E& eng, S* G0, S* G1, S* G2, S* G3, S* Sc, S* Spp, S* Spq, S* Spr, S* Pp, S* Pq, S* Pr,
                        const S* D, S* G, S* Sq2, S* Gq) {
        const int ng = this->ng, n2 = this->n2, L = this->L, nz = this->nz, M = this->M, ML = this->ML;
        const bool mixed = sizeof(T) == 4;
        const double hdzi = (1.0 / 2.0) * (1.0 / (HBAR / (double)nz));
        const double qdzi = (1.0 / 4.0) * (1.0 / (HBAR / (double)nz));
        const double* filt = op.filt;
        const T *U = u, *V = v, *WW = w, *ZX = zx, *ZY = zy, *RI = ri, *ZE = zeta;
        T *SIGX = sigx, *SIGY = sigy, *C1 = cpt1, *C2 = cpt2, *SP0 = sp0;
        const T *UX = W(11), *UY = W(12), *VX = W(13), *VY = W(14), *WX = W(15), *WY = W(16);
        const T* HZ = W(21);
        const T* hsrc = plane_t.p + (size_t)M * n2;
        // P6: cpt2's argument and cpsource's dealiased products.  The four values of
        // an element share the theta derivatives of u, v, w: one streaming pass forms
        // them into the staging planes, then a plain transform takes them to spectral
        // space.  (four elements per thread with 16-byte loads and stores; n2 % 4 == 0)
        for_planes4(st, ML, n2, [=] __device__(int q, int pi) {
            const int m = q / L, iz = q % L;
            const size_t p = (size_t)q * n2 + pi;
            const size_t cb = (size_t)m * L * n2 + pi;
            T ri[4], sx[4], sy[4];
            S g0[4], g1[4], g2[4], g3[4];
            ld4(RI + p, ri);
            ld4(SIGX + p, sx);
            ld4(SIGY + p, sy);
#pragma unroll
            for (int e = 0; e < 4; e++) g0[e] = (S)(T(1) - ri[e] * ri[e] - sx[e] * sx[e] - sy[e] * sy[e]);
            double wt[4];
            tderiv4(WW + cb, iz, nz, n2, hdzi, wt);
            if (iz == 0) {
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    g1[e] = S(0);
                    g2[e] = (S)(T)((double)ri[e] * wt[e]);
                    g3[e] = S(0);
                }
            } else {
                double ut[4], vt[4];
                tderiv4(U + cb, iz, nz, n2, hdzi, ut);
                tderiv4(V + cb, iz, nz, n2, hdzi, vt);
                T zx[4], zy[4], ux[4], uy[4], vx[4], vy[4];
                ld4(ZX + p, zx);
                ld4(ZY + p, zy);
                ld4(UX + p, ux);
                ld4(UY + p, uy);
                ld4(VX + p, vx);
                ld4(VY + p, vy);
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    g1[e] = (S)(T)(vt[e] * (double)zx[e] - ut[e] * (double)zy[e]);
                    g2[e] = (S)(T)((double)uy[e] * vt[e] - ut[e] * (double)vy[e]);
                    g3[e] = (S)(T)(ut[e] * (double)vx[e] - (double)ux[e] * vt[e]);
                }
            }
            st4(G0 + p, g0);
            st4(G1 + p, g1);
            st4(G2 + p, g2);
            st4(G3 + p, g3);
        });
        eng.ptospc(st, 4 * ML,
            plane_ld([=] __device__(int o) {
                const int which = o & 3, q = o >> 2;
                return PairLd<S>{(which == 0 ? G0 : which == 1 ? G1 : which == 2 ? G2 : G3) + (size_t)q * n2, ng};
            }),
            plane_st([=] __device__(int o) {
                const int which = o & 3, q = o >> 2;
                return PairStOp<S>{(which == 0 ? Sc : which == 1 ? Spp : which == 2 ? Spq : Spr) + (size_t)q * n2, filt, ng};
            }));
        // P7: cpt2 and the products back to physical space
        if constexpr (std::is_same<S, T>::value) {
            eng.spctop(st, 4 * ML,
                plane_ld([=] __device__(int o) {
                    const int which = o / ML, q = o - which * ML;
                    return PairLd<S>{(which == 0 ? Sc : which == 1 ? Spp : which == 2 ? Spq : Spr) + (size_t)q * n2, ng};
                }),
                plane_st([=] __device__(int o) {
                    const int which = o / ML, q = o - which * ML;
                    return PairSt<S>{(which == 0 ? C2 : which == 1 ? Pp : which == 2 ? Pq : Pr) + (size_t)q * n2, ng};
                }));
        } else {
            eng.spctop(st, 3 * ML,
                plane_ld([=] __device__(int o) {
                    const int which = o / ML, q = o - which * ML;
                    return PairLd<S>{(which == 0 ? Spp : which == 1 ? Spq : Spr) + (size_t)q * n2, ng};
                }),
                plane_st([=] __device__(int o) {
                    const int which = o / ML, q = o - which * ML;
                    return PairSt<S>{(which == 0 ? Pp : which == 1 ? Pq : Pr) + (size_t)q * n2, ng};
                }));
            eng.spctop(st, ML, plane_ld([=] __device__(int q) { return PairLd<S>{Sc + (size_t)q * n2, ng}; }),
                plane_st([=] __device__(int q) {
                    T* d = C2 + (size_t)q * n2;
                    return [=](int c, int pt, S a, S b, int mk) { stv2m(d + c + ng * pt, mk, (T)a, (T)b); };
                }));
        }
        // P8: cpt1 = 0.5 d(cpt2)/dtheta + div(sig); sig *= 2 (coeffs.rs:44-100)
        //     (four elements per thread; the theta derivative is tderiv's one-sided /
        //     centred form with qdzi)
        for_planes4(st, ML, n2, [=] __device__(int q, int i) {
            const int m = q / L, iz = q % L;
            const size_t p = (size_t)q * n2 + i;
            double t[4];
            tderiv4(C2 + (size_t)m * L * n2 + i, iz, nz, n2, qdzi, t);
            S dv[4];
            T c1[4], sx[4], sy[4];
            if (iz > 0) ld4(D + p, dv);
            ld4(SIGX + p, sx);
            ld4(SIGY + p, sy);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                c1[e] = (T)(iz == 0 ? t[e] : t[e] + (double)dv[e]);
                sx[e] = sx[e] * T(2);
                sy[e] = sy[e] * T(2);
            }
            st4(C1 + p, c1);
            st4(SIGX + p, sx);
            st4(SIGY + p, sy);
        });
        // P9/P10: the second dealiased product and sp0 (cpsource.rs:222-258), both
        // formed in streaming passes around plain transforms
        for_planes4(st, ML, n2, [=] __device__(int q, int pi) {
            const int m = q / L, iz = q % L;
            const size_t p = (size_t)q * n2 + pi;
            S g[4];
            if (iz == 0) {
                g[0] = g[1] = g[2] = g[3] = S(0);
                st4(G + p, g);
                return;
            }
            const size_t cb = (size_t)m * L * n2 + pi;
            double ut[4], vt[4], wt[4];
            tderiv4(U + cb, iz, nz, n2, hdzi, ut);
            tderiv4(V + cb, iz, nz, n2, hdzi, vt);
            tderiv4(WW + cb, iz, nz, n2, hdzi, wt);
            S pq[4], pr[4];
            T zx[4], zy[4], wx[4], wy[4], ux[4], vy[4];
            ld4(Pq + p, pq);
            ld4(Pr + p, pr);
            ld4(ZX + p, zx);
            ld4(ZY + p, zy);
            ld4(WX + p, wx);
            ld4(WY + p, wy);
            ld4(UX + p, ux);
            ld4(VY + p, vy);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                double wkq = (double)pq[e] * (double)zx[e] + (double)pr[e] * (double)zy[e] - (double)wy[e] * vt[e];
                wkq += ((double)ux[e] + (double)vy[e]) * wt[e] - (double)wx[e] * ut[e];
                g[e] = (S)(T)wkq;
            }
            st4(G + p, g);
        });
        eng.ptospc(st, ML, plane_ld([=] __device__(int q) { return PairLd<S>{G + (size_t)q * n2, ng}; }),
                   plane_st([=] __device__(int q) { return PairStOp<S>{Sq2 + (size_t)q * n2, filt, ng}; }));
        eng.spctop(st, ML, plane_ld([=] __device__(int q) { return PairLd<S>{Sq2 + (size_t)q * n2, ng}; }),
                   plane_st([=] __device__(int q) { return PairSt<S>{Gq + (size_t)q * n2, ng}; }));
        for_planes4(st, ML, n2, [=] __device__(int q, int pi) {
            const int m = q / L, iz = q % L;
            const size_t p = (size_t)q * n2 + pi;
            S gv[4], pqv[4], ppv[4];
            T uxv[4], uyv[4], vxv[4], vyv[4], out[4];
            ld4(Gq + p, gv);
            ld4(UX + p, uxv);
            ld4(UY + p, uyv);
            ld4(VX + p, vxv);
            ld4(VY + p, vyv);
            T hv[4], riv[4], zev[4];
            if (iz == 0) ld4(Pq + p, pqv);
            if (mixed) ld4(HZ + p, hv);
            else ld4(hsrc + (size_t)m * n2 + pi, hv);
            if (iz != 0) {
                ld4(RI + p, riv);
                ld4(Pp + p, ppv);
            }
            if (!mixed) ld4(ZE + p, zev);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const double ux = uxv[e], uy = uyv[e], vx = vxv[e], vy = vyv[e];
                double s;
                if (mixed) {
                    const double hz = hv[e];
                    if (iz == 0) {
                        s = hz + 2.0 * (ux * vy - uy * vx + (double)pqv[e] * (ux + vy));
                    } else {
                        const double rip = riv[e];
                        s = hz - COF * (rip * (double)ppv[e]) + 2.0 * (rip * (double)gv[e]);
                        s += 2.0 * (ux * vy - uy * vx);
                    }
                } else {
                    const double hsv = (double)hv[e];
                    if (iz == 0) {
                        s = hsv + COF * (double)zev[e];
                        s += 2.0 * (ux * vy - uy * vx + (double)pqv[e] * (ux + vy));
                    } else {
                        const double rip = riv[e];
                        s = hsv + COF * ((double)zev[e] - rip * (double)ppv[e]) + 2.0 * (rip * (double)gv[e]);
                        s += 2.0 * (ux * vy - uy * vx);
                    }
                }
                out[e] = (T)s;
            }
            st4(SP0 + p, out);
        });
    }

    // P4/P5 of psolve_prepare_fused on the mixed path (float64 solver with the
    // float32 engine): the spectrum of w and its x, y derivatives stay float64; the
    // w correction u z_x + v z_y, ri z_x, ri z_y (each dealiased: sigx, sigy) and
    // div(sig) go through float32 transforms (Sd, Sx, Sy, D in R32(0..3)).  The
    // products are formed in float64 and rounded once to float32 for the transform;
    // w_x, w_y take the correction's float32 spectrum into their float64 sum.
    void setup_w_sig_f32() {
        if constexpr (sizeof(T) == 8) {
            const int ng = this->ng, n2 = this->n2, L = this->L, nz = this->nz, M = this->M, ML = this->ML;
            const int Mnz = M * nz;
            const double* filt = op.filt;
            T *U = u, *V = v, *WW = w, *ZX = zx, *ZY = zy, *RI = ri, *SIGX = sigx, *SIGY = sigy;
            T *Sw = W(10), *WX = W(15), *WY = W(16);
            float *Sd = R32(0), *Sx = R32(1), *Sy = R32(2), *D = R32(3);
            // P4a (float64): w to spectral space, levels 1..nz
            fft.ptospc(st, Mnz,
                plane_ld([=] __device__(int o) {
                    const int m = o / nz, iz = 1 + o % nz;
                    return PairLd<T>{WW + (size_t)(m * L + iz) * n2, ng};
                }),
                plane_st([=] __device__(int o) {
                    const int m = o / nz, iz = 1 + o % nz;
                    return PairSt<T>{Sw + (size_t)(m * L + iz) * n2, ng};
                }));
            // P4b (float32): u z_x + v z_y (levels 1..nz), then ri z_x, ri z_y of one
            // level adjacent, all dealiased
            f32.ptospc(st, Mnz + 2 * ML,
                plane_ld([=] __device__(int o) {
                    bool corr = true;
                    size_t p0;
                    const T* zz = ZX;
                    if (o < Mnz) {
                        const int m = o / nz, iz = 1 + o % nz;
                        p0 = (size_t)(m * L + iz) * n2;
                    } else {
                        const int k = o - Mnz, q = k >> 1;
                        p0 = (size_t)q * n2;
                        zz = (k & 1) ? ZY : ZX;
                        corr = false;
                    }
                    return [=](int iy, int ix) {
                        const size_t p = p0 + iy + ng * ix;
                        if (!corr) {
                            const auto r2 = ldv2(RI + p), z2 = ldv2(zz + p);
                            return mk2(r2.x * z2.x, r2.y * z2.y);
                        }
                        const auto u2 = ldv2(U + p), zx2 = ldv2(ZX + p), v2 = ldv2(V + p), zy2 = ldv2(ZY + p);
                        return mk2(u2.x * zx2.x + v2.x * zy2.x, u2.y * zx2.y + v2.y * zy2.y);
                    };
                }),
                plane_st([=] __device__(int o) {
                    float* d;
                    if (o < Mnz) {
                        const int m = o / nz, iz = 1 + o % nz;
                        d = Sd + (size_t)(m * L + iz) * n2;
                    } else {
                        const int k = o - Mnz, q = k >> 1;
                        d = ((k & 1) ? Sy : Sx) + (size_t)q * n2;
                    }
                    return PairStOp<float>{d, filt, ng};
                }));
            // P5a (float64): w_x, w_y of one level adjacent from the spectra of w and
            // of its correction
            fft.spctop(st, 2 * Mnz,
                plane_ld([=] __device__(int o) {
                    const int k = o >> 1, which = o & 1, m = k / nz, iz = 1 + k % nz;
                    const size_t b = (size_t)(m * L + iz) * n2;
                    return [=](int kx, int ky) {
                        if (which == 0) {
                            const int j0 = mirror(kx, ng) + ng * ky, j1 = mirror(kx + 1, ng) + ng * ky;
                            return mk2(dmul(kx, ng) * ((double)Sw[b + j0] + (double)Sd[b + j0]),
                                       dmul(kx + 1, ng) * ((double)Sw[b + j1] + (double)Sd[b + j1]));
                        }
                        const size_t my = b + kx + ng * mirror(ky, ng);
                        const double dy = dmul(ky, ng);
                        const auto w2 = ldv2(Sw + my);
                        const auto d2 = ldv2(Sd + my);
                        return mk2(dy * ((double)w2.x + (double)d2.x), dy * ((double)w2.y + (double)d2.y));
                    };
                }),
                plane_st([=] __device__(int o) {
                    const int k = o >> 1, which = o & 1, m = k / nz, iz = 1 + k % nz;
                    return PairSt<T>{(which == 0 ? WX : WY) + (size_t)(m * L + iz) * n2, ng};
                }));
            // P5b (float32): the correction (added to w), sigx, sigy, div(sig)
            f32.spctop(st, 2 * Mnz + 2 * ML,
                plane_ld([=] __device__(int o) {
                    bool dv = false;
                    const float* s = nullptr;
                    size_t b = 0;
                    if (o < Mnz) {
                        const int m = o / nz, iz = 1 + o % nz;
                        s = Sd + (size_t)(m * L + iz) * n2;
                    } else if (o < Mnz + 2 * ML) {
                        const int k = o - Mnz, which = k / ML, q = k - which * ML;
                        s = (which == 0 ? Sx : Sy) + (size_t)q * n2;
                    } else {
                        const int k = o - Mnz - 2 * ML, m = k / nz, iz = 1 + k % nz;
                        b = (size_t)(m * L + iz) * n2;
                        dv = true;
                    }
                    return [=](int kx, int ky) {
                        if (!dv) return ldv2(s + kx + ng * ky);
                        const size_t my = b + kx + ng * mirror(ky, ng);
                        const double dy = dmul(ky, ng);
                        const auto y2 = ldv2(Sy + my);
                        const double x0 = (double)Sx[b + mirror(kx, ng) + ng * ky];
                        const double x1 = (double)Sx[b + mirror(kx + 1, ng) + ng * ky];
                        return mk2((float)(dy * (double)y2.x + dmul(kx, ng) * x0),
                                   (float)(dy * (double)y2.y + dmul(kx + 1, ng) * x1));
                    };
                }),
                plane_st([=] __device__(int o) {
                    int kind = 2;  // 0 add to w, 1 sig (float64 field), 2 div(sig)
                    T* dd = nullptr;
                    float* df = nullptr;
                    if (o < Mnz) {
                        const int m = o / nz, iz = 1 + o % nz;
                        dd = WW + (size_t)(m * L + iz) * n2;
                        kind = 0;
                    } else if (o < Mnz + 2 * ML) {
                        const int k = o - Mnz, which = k / ML, q = k - which * ML;
                        dd = (which == 0 ? SIGX : SIGY) + (size_t)q * n2;
                        kind = 1;
                    } else {
                        const int k = o - Mnz - 2 * ML, m = k / nz, iz = 1 + k % nz;
                        df = D + (size_t)(m * L + iz) * n2;
                    }
                    return [=](int iy, int ix, float a, float b, int mk) {
                        const int i = iy + ng * ix;
                        if (kind == 2) {
                            stv2m(df + i, mk, a, b);
                        } else if (kind == 1) {
                            stv2m(dd + i, mk, (T)a, (T)b);
                        } else {
                            const auto w2 = ldv2(dd + i);
                            stv2m(dd + i, mk, w2.x + (T)a, w2.y + (T)b);
                        }
                    };
                }));
        }
    }

    // One pressure sweep (psolve.rs:89-358) and its convergence control.  With
    // cond set, the sweep is the body of a graph WHILE node and the last kernel
    // sets the node's condition from the members still iterating.  With the
    // correction sweeps on (the mixed path), the body is two conditional nodes, a
    // float64 reference sweep and a float32 correction sweep, of which the control
    // kernel enables one for the next iteration (c64, c32); host-driven loops pass
    // the kind that the control kernel chose (host_kind).
    void psolve_sweep(int nitmax, bool use_cond, cudaGraphConditionalHandle cond, cudaGraphConditionalHandle c64 = 0,
                      cudaGraphConditionalHandle c32 = 0) {
        if (!refine32) {
            sweep_reference();
        } else if (use_cond) {
            const long long c0 = launch_counter().load();
            capture_if(c64, [&] { sweep_reference(); });
            const long long c1 = launch_counter().load();
            capture_if(c32, [&] { sweep_correction(); });
            k_sweep_kind[0] = c1 - c0 + 1;  // + the control kernel
            k_sweep_kind[1] = launch_counter().load() - c1 + 1;
        } else if (host_kind == 0) {
            sweep_reference();
        } else {
            sweep_correction();
        }
        sweep_ctrl(nitmax, use_cond, cond, c64, c32);
    }

    // Captures body() into an IF node of the graph being captured on st, enabled
    // by handle h (made in the enclosing step graph, set by the control kernel).
    template <class F>
    void capture_if(cudaGraphConditionalHandle h, F&& body) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        SW_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
        require(cs == cudaStreamCaptureStatusActive, SW_ERR_STATE, "capture_if outside a capture");
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t cn;
        SW_CUDA(cudaGraphAddNode(&cn, g, deps, nd, &cp));
        cudaGraph_t body_graph = cp.conditional.phGraph_out[0];
        SW_CUDA(cudaStreamUpdateCaptureDependencies(st, &cn, 1, cudaStreamSetCaptureDependencies));
        cudaStream_t outer = st;
        st = st_if;
        SW_CUDA(cudaStreamBeginCaptureToGraph(st, body_graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        try {
            body();
        } catch (...) {
            cudaGraph_t dummy;
            cudaStreamEndCapture(st, &dummy);
            st = outer;
            throw;
        }
        cudaGraph_t done;
        SW_CUDA(cudaStreamEndCapture(st, &done));
        st = outer;
    }

    // The total source S = S0 + S1(p) of one sweep in physical space (psolve.rs:
    // 96-240), TS-precision planes: A, B, C hold p, p_x, p_y of levels 0..nz-1; the
    // theta derivatives are formed here.  SP0 == nullptr leaves S0 out (S1 alone: the
    // correction sweeps).  S reads eight fields per element; as a streaming pass at
    // full occupancy it runs near the memory bandwidth, while inside the transform's
    // loader (sixteen pairs per thread, four CTAs per SM) the loads wait on latency.
    // Four elements per thread with 16-byte loads and stores (n2 % 4 == 0: ng is even).
    template <typename TS>
    void sweep_source(const TS* A, const TS* B, const TS* C, const TS* SP0, const TS* SIGX, const TS* SIGY,
                      const TS* C2, const TS* C1, TS* SRC) {
        const int n2 = this->n2, L = this->L, nz = this->nz, ML = this->ML;
        const double dz = HBAR / (double)nz, dz2 = dz / 2.0;
        const double dzisq = (1.0 / dz) * (1.0 / dz);
        const double hdzi = (1.0 / 2.0) * (1.0 / (HBAR / (double)nz));
        for_planes4(st, ML, n2, [=] __device__(int q, int i) {
            const int m = q / L, iz = q % L;
            const size_t p = (size_t)q * n2 + i;
            const size_t cb = (size_t)m * L * n2 + i;
            TS out[4];
            if (iz > 0 && iz < nz) {
                auto lv = [&](const TS* f, int l, TS(&v)[4]) {
                    if (l >= nz) v[0] = v[1] = v[2] = v[3] = TS(0);
                    else ld4(f + cb + (size_t)l * n2, v);
                };
                TS xp[4], xm[4], yp[4], ym[4], pp[4], pc[4], pm[4], sp0[4], sx[4], sy[4], c2[4], c1[4];
                lv(B, iz + 1, xp);
                lv(B, iz - 1, xm);
                lv(C, iz + 1, yp);
                lv(C, iz - 1, ym);
                lv(A, iz + 1, pp);
                lv(A, iz, pc);
                lv(A, iz - 1, pm);
                if (SP0) ld4(SP0 + p, sp0);
                else sp0[0] = sp0[1] = sp0[2] = sp0[3] = TS(0);
                ld4(SIGX + p, sx);
                ld4(SIGY + p, sy);
                ld4(C2 + p, c2);
                ld4(C1 + p, c1);
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const double dxt = ((double)xp[e] - (double)xm[e]) * hdzi;
                    const double dyt = ((double)yp[e] - (double)ym[e]) * hdzi;
                    const double dpdt = ((double)pp[e] - (double)pm[e]) * hdzi;
                    const double d2 = ((double)pp[e] - 2.0 * (double)pc[e] + (double)pm[e]) * dzisq;
                    double s = (double)sp0[e] + (double)sx[e] * dxt + (double)sy[e] * dyt;
                    s += (double)c2[e] * d2 + (double)c1[e] * dpdt;
                    out[e] = (TS)s;
                }
            } else {
                // boundary levels: the same stencils, four elements per 16-byte load
                // (levels at or above nz hold p = 0)
                auto lv4 = [&](const TS* f, int l, double(&v)[4]) {
                    if (l >= nz) {
                        v[0] = v[1] = v[2] = v[3] = 0.0;
                        return;
                    }
                    TS t[4];
                    ld4(f + cb + (size_t)l * n2, t);
#pragma unroll
                    for (int e = 0; e < 4; e++) v[e] = (double)t[e];
                };
                double s0[4] = {0.0, 0.0, 0.0, 0.0};
                if (SP0) {
                    TS t[4];
                    ld4(SP0 + p, t);
#pragma unroll
                    for (int e = 0; e < 4; e++) s0[e] = (double)t[e];
                }
                TS c2[4];
                ld4(C2 + p, c2);
                if (iz == 0) {
                    double P0[4], P1[4], P2[4], P3[4];
                    lv4(A, 0, P0);
                    lv4(A, 1, P1);
                    lv4(A, 2, P2);
                    lv4(A, 3, P3);
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const double d2 = (2.0 * P0[e] - 5.0 * P1[e] + 4.0 * P2[e] - P3[e]) * dzisq;
                        out[e] = (TS)(s0[e] + (double)c2[e] * d2);
                    }
                } else {
                    // extrapolation to iz = nz from nz-1, nz-2 (psolve.rs:232-238);
                    // F[j] holds level nz - j
                    double Pl[4][4], Xl[4][4], Yl[4][4];
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        lv4(A, nz - j, Pl[j]);
                        lv4(B, nz - j, Xl[j]);
                        lv4(C, nz - j, Yl[j]);
                    }
                    TS sx[4], sy[4], c1[4];
                    ld4(SIGX + p, sx);
                    ld4(SIGY + p, sy);
                    ld4(C1 + p, c1);
                    auto ext = [&](const double(&F)[4][4], int e) {
                        const double a1 = (F[0][e] - F[2][e]) * hdzi;
                        const double d1 = (F[0][e] - 2.0 * F[1][e] + F[2][e]) * dzisq;
                        const double d2 = (F[1][e] - 2.0 * F[2][e] + F[3][e]) * dzisq;
                        return a1 + dz2 * (3.0 * d1 - d2);
                    };
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const double dxt = ext(Xl, e), dyt = ext(Yl, e), dpdt = ext(Pl, e);
                        const double d1 = (Pl[0][e] - 2.0 * Pl[1][e] + Pl[2][e]) * dzisq;
                        const double d2 = (Pl[1][e] - 2.0 * Pl[2][e] + Pl[3][e]) * dzisq;
                        const double d2pdt2 = 2.0 * d1 - d2;
                        double s = s0[e] + (double)sx[e] * dxt + (double)sy[e] * dyt;
                        s += (double)c2[e] * d2pdt2 + (double)c1[e] * dpdt;
                        out[e] = (TS)s;
                    }
                }
            }
            st4(SRC + p, out);
        });
    }

    // Compact RHS and Thomas solve per (kx, ky) column (psolve.rs:285-329), with the
    // errp sums reduced per CTA.  With the correction sweeps on, the reference
    // sweep's solve also records its change D1 and |ps|^2 (NV = 3).
    void sweep_thomas(const T* SP) {
        const int ng = this->ng, n2 = this->n2, nz = this->nz, M = this->M;
        const double *htdv = op.htdv, *etdv = op.etdv, *ap = op.ap;
        double* PS = ps;
        double* XF = WD(1);
        const int* ctl = ctrl.p;
        const int nblk = (n2 + THOMAS_THREADS - 1) / THOMAS_THREADS;
        double* part = red_partial.p;
        const dim3 g(nblk, M);
        float* D1 = refine32 ? R32(9) : nullptr;
        float* Cw = refine32 ? R32(10) : nullptr;
        const double om = relax;
#define SW_THOMAS_CASE(NZV)                                                                              \
    if (refine32)                                                                                        \
        k_thomas<T, NZV, 3>                                                                              \
            <<<g, THOMAS_THREADS, 0, st>>>(ng, nz, n2, ctl, SP, htdv, etdv, ap, PS, XF, D1, Cw, om, part); \
    else                                                                                                 \
        k_thomas<T, NZV, 2>                                                                              \
            <<<g, THOMAS_THREADS, 0, st>>>(ng, nz, n2, ctl, SP, htdv, etdv, ap, PS, XF, D1, Cw, om, part);
        switch (nz) {
            case 4: SW_THOMAS_CASE(4) break;
            case 8: SW_THOMAS_CASE(8) break;
            case 16: SW_THOMAS_CASE(16) break;
            case 32: SW_THOMAS_CASE(32) break;
            default: SW_THOMAS_CASE(0) break;
        }
#undef SW_THOMAS_CASE
        SW_CHECK_LAUNCH();
        count_launch();
    }

    // The control kernel of one sweep: finishes the errp sums per member and applies
    // the stop rule (psolve.rs:89, 339-358).  Stop rule: float64, the reference's 1e-9
    // on the relative change; the correction sweeps, refine_toler; float32, 1e-6 or
    // stagnation (see ctrl_member).
    void sweep_ctrl(int nitmax, bool use_cond, cudaGraphConditionalHandle cond, cudaGraphConditionalHandle c64,
                    cudaGraphConditionalHandle c32) {
        const bool mixed = sizeof(T) == 4;
        const double toler = mixed ? 1.0E-6 : (refine32 ? refine_toler : 1.0E-9);
        const int nblk = (n2 + THOMAS_THREADS - 1) / THOMAS_THREADS;
        k_psolve_ctrl<<<1, CTRL_THREADS, 0, st>>>(M, nblk, refine32 ? 3 : 2, red_partial.p, ctrl.p, errp_d.p, toler,
                                                  mixed ? 1 : 0, nitmax, use_cond ? 1 : 0, cond, sweep_exec.p,
                                                  refine32 ? sweep_kind.p : nullptr, eref.p, pnorm.p, c64, c32);
        SW_CHECK_LAUNCH();
        count_launch();
    }

    // Correction sweeps: the iterate is ps + C.  Folds C into ps (C = 0) and, with
    // clear_sp32, clears the correction source, so that a reference sweep starts
    // from the current iterate and a finished solve leaves it in ps.
    void fold_correction(bool clear_sp32) {
        const int n2 = this->n2, ML = this->ML;
        double* PS = ps;
        float *Cr = R32(10), *SPC = R32(4);
        for_planes4(st, ML, n2, [=] __device__(int q, int i) {
            const size_t p = (size_t)q * n2 + i;
            double v[4];
            float c[4];
            ld4(PS + p, v);
            ld4(Cr + p, c);
            for (int e = 0; e < 4; e++) v[e] += (double)c[e];
            st4(PS + p, v);
            const float z[4] = {0.f, 0.f, 0.f, 0.f};
            st4(Cr + p, z);
            if (clear_sp32) st4(SPC + p, z);
        });
    }

    // A sweep in the precision of T.  (a) p, dp/dx, dp/dy to physical space for
    // levels 0..nz-1 (p(nz) = 0).  The theta derivatives of the reference
    // (psolve.rs:96-240) are linear in p, so they are formed from these in physical
    // space in (b): 3 nz transforms per member instead of the 4 nz - 1 of the derived
    // quantities.  d/dx acts on kx, which the first (reverse, along ky) pass leaves
    // alone, so p_x takes p's intermediate with the derivative applied in the second
    // pass: 2 nz first passes and 3 nz second passes per member.  (b) the total source
    // S = S0 + S1(p) in physical space, then to spectral space; (c) the Thomas solve.
    // With the correction sweeps on, this is the reference sweep: it starts from the
    // current iterate ps + C, and its solve p1 stays in ps while correction sweeps
    // run; SP keeps the spectrum of S at the reference point p_ref.
    void sweep_reference() {
        NvtxRange nv("psolve_sweep_float64");
        const int ng = this->ng, n2 = this->n2, L = this->L, nz = this->nz, M = this->M, ML = this->ML;
        double* PS = ps;
        T *A = W(0), *B = W(1), *C = W(2), *D = W(3), *SP = W(4);
        if (refine32) fold_correction(true);
        const int n2z = 2 * nz;
        // the intermediate holds all members' 2 nz first-pass planes (cap = 6 (nz + 1) M)
        const int mchunk = std::max(1, std::min(M, fft.cap / n2z));
        for (int m0 = 0; m0 < M; m0 += mchunk) {
            const int mc = std::min(mchunk, M - m0);
            launch_pass<T, true, true, false>(st, fft.plan, fft.tw.p, fft.tc, fft.sc, n2z * mc, ng,
                [=] __device__(int o, int kx, int ky) -> T {  // p, p_y of one level adjacent
                    const int mm = o / n2z, k = o - mm * n2z, iz = k >> 1, kind = k & 1;
                    const double* pc = PS + (size_t)((m0 + mm) * L + iz) * n2;
                    if (kind == 0) return (T)pc[kx + ng * ky];
                    return (T)(dmul(ky, ng) * pc[kx + ng * mirror(ky, ng)]);
                },
                MidPC<T>{fft.midp, ng});
            launch_pass<T, true, true, true>(st, fft.plan, fft.tw.p, fft.tc, fft.sc, 3 * nz * mc, ng,
                SweepMidLoad<T>{fft.midp, ng, nz}, SweepPhysStore<T>{A, B, C, ng, nz, L, m0});
        }
        sweep_source<T>(A, B, C, sp0.p, sigx.p, sigy.p, cpt2.p, cpt1.p, D);
        fft.ptospc(st, ML,
            [=] __device__(int q, int iy, int ix) -> T { return D[(size_t)q * n2 + iy + ng * ix]; },
            [=] __device__(int q, int kx, int ky, T val) { SP[(size_t)q * n2 + kx + ng * ky] = val; });
        sweep_thomas(SP);
    }

    // A float32 correction sweep of the mixed path (float64 solver only).  Apart
    // from S0 the sweep is linear in p, and so is the Thomas solve T^-1: with p_ref
    // the last reference sweep's input and p1 = T^-1 S(p_ref) its result (in ps), the
    // next iterate is p1 + c with c = T^-1 S1(d), d = p - p_ref = D1 + C the distance
    // of the current iterate p = p1 + C from p_ref.  The sweep transforms d (and its x,
    // y derivatives) in float32, forms S1(d) with float32 copies of the coefficients
    // and solves for the new C.  Its rounding is relative to |d|, which is small next
    // to |p|, so the iteration converges well below float32 rounding of p while moving
    // about half the bytes of a float64 sweep.
    void sweep_correction() {
        NvtxRange nv("psolve_sweep_float32_correction");
        if constexpr (sizeof(T) == 8) {
            const int ng = this->ng, n2 = this->n2, L = this->L, nz = this->nz, M = this->M, ML = this->ML;
            const float *D1 = R32(9), *Cr = R32(10);
            float *A = R32(0), *B = R32(1), *C = R32(2), *D = R32(3), *SPC = R32(4);
            const int n2z = 2 * nz;
            const int mchunk = std::max(1, std::min(M, f32.chunk / n2z));
            for (int m0 = 0; m0 < M; m0 += mchunk) {
                const int mc = std::min(mchunk, M - m0);
                launch_pass<float, true, true, false>(st, f32.plan, f32.tw.p, f32.tc, f32.sc, n2z * mc, ng,
                    plane_ld([=] __device__(int o) {  // d, d_y of one level adjacent
                        const int mm = o / n2z, k = o - mm * n2z, iz = k >> 1, kind = k & 1;
                        const size_t b = (size_t)((m0 + mm) * L + iz) * n2;
                        return [=](int kx, int ky) {
                            const size_t j = b + kx + ng * (kind == 0 ? ky : mirror(ky, ng));
                            const float2 a = ldv2(D1 + j), c = ldv2(Cr + j);
                            if (kind == 0) return mk2(a.x + c.x, a.y + c.y);
                            return mk2(dmul_t(ky, ng, a.x + c.x), dmul_t(ky, ng, a.y + c.y));
                        };
                    }),
                    MidPC<float>{f32.midp, ng});
                launch_pass<float, true, true, true>(st, f32.plan, f32.tw.p, f32.tc, f32.sc, 3 * nz * mc, ng,
                    SweepMidLoad<float>{f32.midp, ng, nz}, SweepPhysStore<float>{A, B, C, ng, nz, L, m0});
            }
            sweep_source<float>(A, B, C, nullptr, R32(5), R32(6), R32(7), R32(8), D);
            f32.ptospc(st, ML,
                [=] __device__(int q, int iy, int ix) -> float { return D[(size_t)q * n2 + iy + ng * ix]; },
                [=] __device__(int q, int kx, int ky, float val) { SPC[(size_t)q * n2 + kx + ng * ky] = val; });
            const double *htdv = op.htdv, *etdv = op.etdv, *ap = op.ap;
            const int* ctl = ctrl.p;
            const int nblk = (n2 + THOMAS_THREADS - 1) / THOMAS_THREADS;
            const dim3 g(nblk, M);
            float* Cw = R32(10);
            double *XF = WD(1), *part = red_partial.p;
            switch (nz) {
                case 4: k_thomas_c<4><<<g, THOMAS_THREADS, 0, st>>>(ng, nz, n2, ctl, SPC, htdv, etdv, ap, Cw, relax, XF, part); break;
                case 8: k_thomas_c<8><<<g, THOMAS_THREADS, 0, st>>>(ng, nz, n2, ctl, SPC, htdv, etdv, ap, Cw, relax, XF, part); break;
                case 16: k_thomas_c<16><<<g, THOMAS_THREADS, 0, st>>>(ng, nz, n2, ctl, SPC, htdv, etdv, ap, Cw, relax, XF, part); break;
                case 32: k_thomas_c<32><<<g, THOMAS_THREADS, 0, st>>>(ng, nz, n2, ctl, SPC, htdv, etdv, ap, Cw, relax, XF, part); break;
                default: k_thomas_c<0><<<g, THOMAS_THREADS, 0, st>>>(ng, nz, n2, ctl, SPC, htdv, etdv, ap, Cw, relax, XF, part); break;
            }
            SW_CHECK_LAUNCH();
            count_launch();
        }
    }

    // pn and dp/dtheta after convergence (psolve.rs:367-410).
    void psolve_finish() {
        NvtxRange nv("psolve_finish");
        const int ng = this->ng, n2 = this->n2, L = this->L, nz = this->nz, M = this->M, ML = this->ML;
        const double dz = HBAR / (double)nz, dzi = 1.0 / dz, dz6 = dz / 6.0;
        const double hdzi = (1.0 / 2.0) * (1.0 / (HBAR / (double)nz));
        const double *htd1 = op.htd1, *etd1 = op.etd1;
        T *PN = pn, *DPN = dpn;
        double* PS = ps;
        const T* SP = W(4);
        // correction sweeps: the iterate ps + C into ps; the last sweep's source at
        // level nz is SP + SP32 (SP32 is zero when that sweep was a reference sweep)
        if (refine32) fold_correction(false);
        const float* SPC = refine32 ? R32(4) : nullptr;
        // dp/dtheta by 4th-order compact differences (psolve.rs:371-410), levels 1..nz
        double* GG = WD(1);
        const int ncols = M * n2, nbk = (ncols + 127) / 128;
        bool done = true;
        switch (nz) {
            case 4: k_dpdtheta<T, 4><<<nbk, 128, 0, st>>>(n2, ncols, PS, SP, SPC, htd1, etd1, hdzi, dzi, dz6, GG); break;
            case 8: k_dpdtheta<T, 8><<<nbk, 128, 0, st>>>(n2, ncols, PS, SP, SPC, htd1, etd1, hdzi, dzi, dz6, GG); break;
            case 16: k_dpdtheta<T, 16><<<nbk, 128, 0, st>>>(n2, ncols, PS, SP, SPC, htd1, etd1, hdzi, dzi, dz6, GG); break;
            case 32: k_dpdtheta<T, 32><<<nbk, 128, 0, st>>>(n2, ncols, PS, SP, SPC, htd1, etd1, hdzi, dzi, dz6, GG); break;
            default: done = false;
        }
        if (done) {
            SW_CHECK_LAUNCH();
            count_launch();
        } else for_cols(st, M * n2, [=] __device__(int c) {
            const int m = c / n2, i = c - m * n2;
            const size_t cb = (size_t)m * L * n2 + i;
            auto P = [&](int iz) { return PS[cb + (size_t)iz * n2]; };
            auto G = [&](int iz) -> double& { return GG[cb + (size_t)iz * n2]; };
            // forward elimination of the compact scheme, levels 1..nz (streamed through GG)
            double gprev = (P(2) - P(0)) * hdzi * htd1[0];
            G(1) = gprev;
            #pragma unroll 4
            for (int iz = 2; iz < nz; iz++) {
                gprev = ((P(iz + 1) - P(iz - 1)) * hdzi - (1.0 / 6.0) * gprev) * htd1[iz - 1];
                G(iz) = gprev;
            }
            const double spn = (double)SP[cb + (size_t)nz * n2] + (SPC ? (double)SPC[cb + (size_t)nz * n2] : 0.0);
            double gn = dz6 * spn - P(nz - 1) * dzi;
            gn = (gn - (1.0 / 3.0) * gprev) * htd1[nz - 1];
            G(nz) = gn;
            #pragma unroll 4
            for (int iz = nz - 1; iz >= 1; iz--) {
                gn = G(iz) + etd1[iz - 1] * gn;
                G(iz) = gn;
            }
        });
        // pn = spctop(ps) for levels 0..nz-1 (pn(nz) = 0) and dpn = spctop(gg) for 1..nz, one batch
        const int Mnz = M * nz;
        fft.spctop(st, ML + Mnz,
            [=] __device__(int o, int kx, int ky) -> T {
                if (o < ML) return (T)PS[(size_t)o * n2 + kx + ng * ky];
                const int k = o - ML, m = k / nz, iz = 1 + k % nz;
                return (T)GG[(size_t)(m * L + iz) * n2 + kx + ng * ky];
            },
            [=] __device__(int o, int iy, int ix, T val) {
                if (o < ML) {
                    PN[(size_t)o * n2 + iy + ng * ix] = (o % L == nz) ? T(0) : val;
                    return;
                }
                const int k = o - ML, m = k / nz, iz = 1 + k % nz;
                DPN[(size_t)(m * L + iz) * n2 + iy + ng * ix] = val;
            });
    }

    // Host-driven psolve (psolve.rs:16-411): one stream sync per sweep.  Returns
    // the worst member status; outputs are left untouched on failure, as the
    // reference quits there.
    int psolve(int nitmax, int* iters_out, double* errp_out) {
        if (nitmax <= 0) nitmax = 100;
        psolve_prepare(nitmax);
        if (refine32 && guess_slot >= 0) extrapolate_guess(guess_slot);
        int sweeps = 0;
        int* hctl = reinterpret_cast<int*>(h_pinned);
        while (true) {
            sweeps_run[refine32 ? host_kind : 0]++;
            psolve_sweep(nitmax, false, 0);
            sweeps++;
            SW_CUDA(cudaMemcpyAsync(hctl, ctrl.p, sizeof(int) * 3 * M, cudaMemcpyDeviceToHost, st));
            if (refine32) SW_CUDA(cudaMemcpyAsync(hctl + 3 * M, sweep_kind.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            SW_CUDA(cudaStreamSynchronize(st));
            if (refine32) host_kind = hctl[3 * M];
            bool any = false;
            for (int m = 0; m < M; m++) any = any || hctl[3 * m];
            if (!any || sweeps >= nitmax) break;
        }
        const int status0 = hctl[2];
        int worst = SW_OK;
        for (int m = 0; m < M; m++)
            if (hctl[3 * m + 2] != SW_OK) worst = hctl[3 * m + 2];
        if (iters_out) *iters_out = hctl[1];
        if (errp_out) SW_CUDA(cudaMemcpy(errp_out, errp_d.p, sizeof(double), cudaMemcpyDeviceToHost));
        last_psolve_iters = hctl[1];
        if (worst != SW_OK) return worst;
        psolve_finish();
        return status0;
    }

    // psolve inside a stream capture: the sweep loop becomes a conditional WHILE
    // node, and the sweep counts and statuses are copied to device slots `slot`.
    void psolve_captured(int nitmax, int slot) {
        if (nitmax <= 0) nitmax = 100;
        psolve_prepare(nitmax);
        if (refine32 && guess_slot >= 0) extrapolate_guess(guess_slot);
        cudaStreamCaptureStatus cs;
        cudaGraph_t g;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        SW_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
        require(cs == cudaStreamCaptureStatusActive, SW_ERR_STATE, "psolve_captured outside a capture");
        cudaGraphConditionalHandle cond, c64 = 0, c32 = 0;
        SW_CUDA(cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
        if (refine32) {
            // the sweep bodies' IF conditions live in the step graph, so that every
            // launch of the step starts each solve with a reference sweep
            SW_CUDA(cudaGraphConditionalHandleCreate(&c64, g, 1, cudaGraphCondAssignDefault));
            SW_CUDA(cudaGraphConditionalHandleCreate(&c32, g, 0, cudaGraphCondAssignDefault));
        }
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cn;
        SW_CUDA(cudaGraphAddNode(&cn, g, deps, nd, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        SW_CUDA(cudaStreamUpdateCaptureDependencies(st, &cn, 1, cudaStreamSetCaptureDependencies));
        cudaStream_t outer = st;
        st = st_body;
        SW_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        const long long c0 = launch_counter().load();
        psolve_sweep(nitmax, true, cond, c64, c32);
        k_sweep = launch_counter().load() - c0;
        if (!refine32) k_sweep_kind[0] = k_sweep;
        cudaGraph_t done;
        SW_CUDA(cudaStreamEndCapture(st, &done));
        st = outer;
        const int M = this->M;
        int *ctl = ctrl.p, *sw = sweeps_dev.p, *err = err_dev.p;
        for_cols(st, M, [=] __device__(int m) {
            sw[3 * m + slot] = ctl[3 * m + 1];
            if (ctl[3 * m + 2] != SW_OK) atomicCAS(err, 0, ctl[3 * m + 2]);
        });
        psolve_finish();
    }
    int last_psolve_iters = 0;

    // ======================================================================
    // source (src/nhswps/source.rs:19-138) -> sqs, sds, sgs (float64)
    // Work: W(5..6) q, dd; W(7) F spectral; W(8..10) ff, ffx, ffy; W(11..14)
    // ux, uy, vx, vy; W(15..16) spectral u, v; W(17..22) product spectra;
    // plane_t: z derivatives at iz = 0.
    // ======================================================================
    void source(double* SQS, double* SDS, double* SGS, bool reuse_uv = false) {
        if constexpr (sizeof(T) == 8) {
            if (refine32 && setup32) {
                source_mixed(SQS, SDS, SGS, reuse_uv);
                return;
            }
        }
        NvtxRange nv("source");
        const int ng = this->ng, n2 = this->n2, L = this->L, M = this->M, ML = this->ML;
        const double *filt = op.filt, *hlap = op.hlap, *c2g2 = op.c2g2, *wgt = op.weight;
        const double *QS = qs, *DS = ds, *PSp = ps;
        T *U = u, *V = v, *RI = ri, *DPN = dpn, *Z = z, *ZX = zx, *ZY = zy, *AA = aa;
        T *Q = W(5), *DD = W(6), *F = W(7), *FF = W(8), *FX = W(9), *FY = W(10);
        T *UX = W(11), *UY = W(12), *VX = W(13), *VY = W(14), *Su = W(15), *Sv = W(16);
        T *S0 = W(17), *S1 = W(18), *S2 = W(19), *S3 = W(20), *S4 = W(21), *S5 = W(22);
        T* zs0 = plane_t.p;                       // spectral z(0)
        T* zx0 = plane_t.p + (size_t)M * n2;      // d/dx z(0)
        T* zy0 = plane_t.p + (size_t)2 * M * n2;  // d/dy z(0)
        double* wkd = plane_d.p;
        // ux, uy, vx, vy are those psolve's set-up left in W(11..14) when reuse_uv
        const int nuv = reuse_uv ? 0 : 2;
        // wkd = c2g2 * <A>
        for_cols(st, M * n2, [=] __device__(int c) {
            const int m = c / n2, i = c - m * n2;
            double s = 0.0;
            for (int iz = 0; iz < L; iz++) s += wgt[iz] * (double)AA[(size_t)(m * L + iz) * n2 + i];
            wkd[c] = s * c2g2[i];
        });
        // F = deal(ri * dpn) spectral; spectral u, v (unless reused); spectral z(0)
        const int nf1 = (1 + nuv) * ML;
        fft.ptospc(st, nf1 + M,
            plane_ld([=] __device__(int o) {
                const T *s, *s2 = nullptr;  // s2: second factor of ri * dpn
                if (o >= nf1) {
                    s = Z + (size_t)((o - nf1) * L) * n2;
                } else {
                    const int which = o / ML, q = o - which * ML;
                    s = (which == 0 ? RI : which == 1 ? U : V) + (size_t)q * n2;
                    if (which == 0) s2 = DPN + (size_t)q * n2;
                }
                return [=](int iy, int ix) {
                    const int pi = iy + ng * ix;
                    const auto a2 = ldv2(s + pi);
                    if (!s2) return a2;
                    const auto b2 = ldv2(s2 + pi);
                    return mk2(a2.x * b2.x, a2.y * b2.y);
                };
            }),
            plane_st([=] __device__(int o) {
                T* d;
                const double* opd = nullptr;
                if (o >= nf1) {
                    d = zs0 + (size_t)(o - nf1) * n2;
                } else {
                    const int which = o / ML, q = o - which * ML;
                    d = (which == 0 ? F : which == 1 ? Su : Sv) + (size_t)q * n2;
                    if (which == 0) opd = filt;
                }
                return [=](int kx, int ky, T a, T b, int mk) {
                    if (opd) PairStOp<T>{d, opd, ng}(kx, ky, a, b, mk);
                    else stv2m(d + kx + ng * ky, mk, a, b);
                };
            }));
        // q, delta, ff, ffx, ffy, (ux, uy, vx, vy), z(0) derivatives to physical space.
        // When this stage's main_invert has run, q = zeta - f r pointwise (main_invert
        // sets zeta = spctop(qs + f rhat), r = spctop(rhat)), so q is not transformed.
        const bool q_phys = hint_q_phys;
        const int q0 = q_phys ? 1 : 0;  // first transformed field
        T *ZE = zeta, *R = r;
        const int nk = 5 - q0 + 2 * nuv;  // kinds per level, level-major
        const int nf2 = nk * ML;
        fft.spctop(st, nf2 + 2 * M,
            plane_ld([=] __device__(int o) {
                int kind;  // 0/1/2 value, d/dx, d/dy of s; 3 float64 plane sd
                const T* s = nullptr;
                const double* sd = nullptr;
                if (o >= nf2) {
                    const int which = (o - nf2) / M, m = (o - nf2) % M;
                    s = zs0 + (size_t)m * n2;
                    kind = 1 + which;
                } else {
                    const int q = o / nk, which = o - nk * q + q0;
                    if (which < 2) {
                        sd = (which == 0 ? QS : DS) + (size_t)q * n2;
                        kind = 3;
                    } else {
                        const int w2 = which - 2;  // 0..2: F, F_x, F_y; 3..6: u_x, u_y, v_x, v_y
                        s = (w2 < 3 ? F : w2 < 5 ? Su : Sv) + (size_t)q * n2;
                        kind = w2 < 3 ? w2 : (w2 - 3) % 2 + 1;  // 0 value, 1 d/dx, 2 d/dy
                    }
                }
                return [=](int kx, int ky) {
                    if (kind < 3) return spec_pair(s, kind, kx, ky, ng);
                    const double2 v = ldv2(sd + kx + ng * ky);
                    return mk2((T)v.x, (T)v.y);
                };
            }),
            plane_st([=] __device__(int o) {
                T* d;
                if (o >= nf2) {
                    const int which = (o - nf2) / M, m = (o - nf2) % M;
                    d = (which == 0 ? zx0 : zy0) + (size_t)m * n2;
                } else {
                    const int q = o / nk, which = o - nk * q + q0;
                    d = (which == 0 ? Q : which == 1 ? DD : which == 2 ? FF : which == 3 ? FX : which == 4 ? FY
                         : which == 5 ? UX : which == 6 ? UY : which == 7 ? VX : VY) + (size_t)q * n2;
                }
                return PairSt<T>{d, ng};
            }));
        // products to spectral space: the six products of an element are formed in
        // one streaming pass into staging planes (W(0..4), W(7): the pressure
        // sweep's work planes and F, all consumed by now), then transformed
        T *G0 = W(0), *G1 = W(1), *G2 = W(2), *G3 = W(3), *G4 = W(4), *G5 = W(7);
        // (four elements per thread with 16-byte loads and stores; n2 % 4 == 0)
        for_planes4(st, ML, n2, [=] __device__(int q, int i) {
            const int m = q / L, iz = q % L;
            const size_t p = (size_t)q * n2 + i;
            T u[4], v[4], zx[4], zy[4], ff[4], dd[4], qv[4], bx[4], by[4], fx[4], fy[4];
            ld4(U + p, u);
            ld4(V + p, v);
            ld4(ZX + p, zx);
            ld4(ZY + p, zy);
            ld4(FF + p, ff);
            ld4(DD + p, dd);
            ld4(FX + p, fx);
            ld4(FY + p, fy);
            if (q_phys) {
                T ze[4], rr[4];
                ld4(ZE + p, ze);
                ld4(R + p, rr);
#pragma unroll
                for (int e = 0; e < 4; e++) qv[e] = (T)((double)ze[e] - COF * (double)rr[e]);
            } else {
                ld4(Q + p, qv);
            }
            if (iz == 0) {
                ld4(zx0 + (size_t)m * n2 + i, bx);
                ld4(zy0 + (size_t)m * n2 + i, by);
            } else {
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    bx[e] = zx[e];
                    by[e] = zy[e];
                }
            }
            T g0[4], g1[4], g2[4], g4[4], g5[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                g0[e] = qv[e] * u[e];
                g1[e] = qv[e] * v[e];
                g2[e] = fx[e] * by[e] - fy[e] * bx[e];
                g4[e] = ff[e] * zx[e] - dd[e] * u[e];
                g5[e] = ff[e] * zy[e] - dd[e] * v[e];
            }
            st4(G0 + p, g0);
            st4(G1 + p, g1);
            st4(G2 + p, g2);
            st4(G4 + p, g4);
            st4(G5 + p, g5);
            T ux[4], uy[4], vx[4], vy[4], g3[4];
            ld4(UX + p, ux);
            ld4(UY + p, uy);
            ld4(VX + p, vx);
            ld4(VY + p, vy);
#pragma unroll
            for (int e = 0; e < 4; e++) g3[e] = ux[e] * vy[e] - uy[e] * vx[e];
            st4(G3 + p, g3);
        });
        fft.ptospc(st, 6 * ML,  // level-major
            plane_ld([=] __device__(int o) {
                const int q = o / 6, which = o - 6 * q;
                const T* g = which == 0 ? G0 : which == 1 ? G1 : which == 2 ? G2 : which == 3 ? G3 : which == 4 ? G4 : G5;
                return PairLd<T>{g + (size_t)q * n2, ng};
            }),
            plane_st([=] __device__(int o) {
                const int q = o / 6, which = o - 6 * q;
                T* out = which == 0 ? S0 : which == 1 ? S1 : which == 2 ? S2 : which == 3 ? S3 : which == 4 ? S4 : S5;
                return PairSt<T>{out + (size_t)q * n2, ng};
            }));
        // combine in spectral space
        for_planes(st, ML, n2, [=] __device__(int q, int i) {
            const int m = q / L;
            const int kx = i % ng, ky = i / ng;
            const size_t b = (size_t)q * n2;
            const int mx = mirror(kx, ng) + ng * ky, my = kx + ng * mirror(ky, ng);
            const double wka = dmul(ky, ng) * (double)S1[b + my] + dmul(kx, ng) * (double)S0[b + mx];
            const double sq = filt[i] * ((double)S2[b + i] - wka);
            const double wkb = dmul(ky, ng) * (double)S5[b + my] + dmul(kx, ng) * (double)S4[b + mx];
            const double sd = filt[i] * (2.0 * (double)S3[b + i] + wkb - hlap[i] * PSp[b + i]);
            SQS[b + i] = sq;
            SDS[b + i] = sd;
            SGS[b + i] = COF * sq + wkd[(size_t)m * n2 + i] - FSQ * (double)AA[b + i];
        });
    }

    // source() on the mixed path (float64 solver with the float32 engine).  The same
    // terms as source(); the transforms of ff = deal(ri dpn) and its derivatives, of
    // delta to physical space, and of the products J(ff, z) and ff z_x - delta u,
    // ff z_y - delta v to spectral space run in float32 (staging in R32(0..7)): the
    // source terms whose float32 rounding moves the 10-step result by <= 3e-8 rel-L2
    // at ng=256 (an attribution with the oracle).  q u, q v, J(u, v), the spectral
    // u, v and the z(0) derivatives stay float64 (about 1e-6 each in float32).
    void source_mixed(double* SQS, double* SDS, double* SGS, bool reuse_uv) {
        if constexpr (sizeof(T) == 8) {
            NvtxRange nv("source");
            const int ng = this->ng, n2 = this->n2, L = this->L, M = this->M, ML = this->ML;
            const double *filt = op.filt, *hlap = op.hlap, *c2g2 = op.c2g2, *wgt = op.weight;
            const double *QS = qs, *DS = ds, *PSp = ps;
            T *U = u, *V = v, *RI = ri, *DPN = dpn, *Z = z, *ZX = zx, *ZY = zy, *AA = aa;
            T *Q = W(5), *UX = W(11), *UY = W(12), *VX = W(13), *VY = W(14), *Su = W(15), *Sv = W(16);
            T *S0 = W(17), *S1 = W(18), *S3 = W(20);
            T* zs0 = plane_t.p;
            T* zx0 = plane_t.p + (size_t)M * n2;
            T* zy0 = plane_t.p + (size_t)2 * M * n2;
            float *F = R32(0), *FF = R32(1), *FX = R32(2), *FY = R32(3), *DD = R32(4);
            float *G2 = R32(5), *G4 = R32(6), *G5 = R32(7);  // in place: their spectra
            double* wkd = plane_d.p;
            const int nuv = reuse_uv ? 0 : 2;
            for_cols(st, M * n2, [=] __device__(int c) {
                const int m = c / n2, i = c - m * n2;
                double s = 0.0;
                for (int iz = 0; iz < L; iz++) s += wgt[iz] * (double)AA[(size_t)(m * L + iz) * n2 + i];
                wkd[c] = s * c2g2[i];
            });
            // float64: spectral u, v (unless reused) and z(0)
            const int nf1 = nuv * ML;
            fft.ptospc(st, nf1 + M,
                plane_ld([=] __device__(int o) {
                    const T* s = o >= nf1 ? Z + (size_t)((o - nf1) * L) * n2 : (o < ML ? U : V) + (size_t)(o % ML) * n2;
                    return PairLd<T>{s, ng};
                }),
                plane_st([=] __device__(int o) {
                    T* d = o >= nf1 ? zs0 + (size_t)(o - nf1) * n2 : (o < ML ? Su : Sv) + (size_t)(o % ML) * n2;
                    return PairSt<T>{d, ng};
                }));
            // float32: F = deal(ri dpn), the product formed in float64
            f32.ptospc(st, ML,
                plane_ld([=] __device__(int q) {
                    const T *a = RI + (size_t)q * n2, *b = DPN + (size_t)q * n2;
                    return [=](int iy, int ix) {
                        const int pi = iy + ng * ix;
                        const auto a2 = ldv2(a + pi), b2 = ldv2(b + pi);
                        return mk2(a2.x * b2.x, a2.y * b2.y);
                    };
                }),
                plane_st([=] __device__(int q) { return PairStOp<float>{F + (size_t)q * n2, filt, ng}; }));
            // float64: q (unless formed pointwise), u_x, u_y, v_x, v_y (unless reused),
            // z(0)_x, z(0)_y to physical space
            const bool q_phys = hint_q_phys;
            T *ZE = zeta, *R = r;
            const int nq = q_phys ? 0 : ML, nk = 2 * nuv;
            const int nf2 = nq + nk * ML;
            fft.spctop(st, nf2 + 2 * M,
                plane_ld([=] __device__(int o) {
                    int kind = 3;  // 0/1/2 value, d/dx, d/dy of s; 3 float64 plane sd
                    const T* s = nullptr;
                    const double* sd = nullptr;
                    if (o >= nf2) {
                        const int which = (o - nf2) / M, m = (o - nf2) % M;
                        s = zs0 + (size_t)m * n2;
                        kind = 1 + which;
                    } else if (o < nq) {
                        sd = QS + (size_t)o * n2;
                    } else {
                        const int k = o - nq, q = k >> 2, w2 = k & 3;  // u_x, u_y, v_x, v_y (nk = 4)
                        s = (w2 < 2 ? Su : Sv) + (size_t)q * n2;
                        kind = 1 + (w2 & 1);
                    }
                    return [=](int kx, int ky) {
                        if (kind < 3) return spec_pair(s, kind, kx, ky, ng);
                        return ldv2(sd + kx + ng * ky);
                    };
                }),
                plane_st([=] __device__(int o) {
                    T* d;
                    if (o >= nf2) {
                        const int which = (o - nf2) / M, m = (o - nf2) % M;
                        d = (which == 0 ? zx0 : zy0) + (size_t)m * n2;
                    } else if (o < nq) {
                        d = Q + (size_t)o * n2;
                    } else {
                        const int k = o - nq, q = k >> 2, w2 = k & 3;
                        d = (w2 == 0 ? UX : w2 == 1 ? UY : w2 == 2 ? VX : VY) + (size_t)q * n2;
                    }
                    return PairSt<T>{d, ng};
                }));
            // float32: delta, ff, ff_x, ff_y to physical space (level-major)
            f32.spctop(st, 4 * ML,
                plane_ld([=] __device__(int o) {
                    const int q = o >> 2, which = o & 3;
                    const float* s = F + (size_t)q * n2;
                    const double* sd = DS + (size_t)q * n2;
                    return [=](int kx, int ky) {
                        if (which != 0) return spec_pair(s, which - 1, kx, ky, ng);
                        const double2 v = ldv2(sd + kx + ng * ky);
                        return mk2((float)v.x, (float)v.y);
                    };
                }),
                plane_st([=] __device__(int o) {
                    const int q = o >> 2, which = o & 3;
                    return PairSt<float>{(which == 0 ? DD : which == 1 ? FF : which == 2 ? FX : FY) + (size_t)q * n2, ng};
                }));
            // the six products of an element in one streaming pass: q u, q v, J(u, v)
            // into float64 staging (W(0), W(1), W(3)), J(ff, z) and the two flux
            // products into float32 staging
            T *G0 = W(0), *G1 = W(1), *G3 = W(3);
            for_planes4(st, ML, n2, [=] __device__(int q, int i) {
                const int m = q / L, iz = q % L;
                const size_t p = (size_t)q * n2 + i;
                T u[4], v[4], zx[4], zy[4], qv[4], bx[4], by[4];
                float ff[4], dd[4], fx[4], fy[4];
                ld4(U + p, u);
                ld4(V + p, v);
                ld4(ZX + p, zx);
                ld4(ZY + p, zy);
                ld4(FF + p, ff);
                ld4(DD + p, dd);
                ld4(FX + p, fx);
                ld4(FY + p, fy);
                if (q_phys) {
                    T ze[4], rr[4];
                    ld4(ZE + p, ze);
                    ld4(R + p, rr);
#pragma unroll
                    for (int e = 0; e < 4; e++) qv[e] = (T)((double)ze[e] - COF * (double)rr[e]);
                } else {
                    ld4(Q + p, qv);
                }
                if (iz == 0) {
                    ld4(zx0 + (size_t)m * n2 + i, bx);
                    ld4(zy0 + (size_t)m * n2 + i, by);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        bx[e] = zx[e];
                        by[e] = zy[e];
                    }
                }
                T g0[4], g1[4];
                float g2[4], g4[4], g5[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    g0[e] = qv[e] * u[e];
                    g1[e] = qv[e] * v[e];
                    g2[e] = (float)((double)fx[e] * by[e] - (double)fy[e] * bx[e]);
                    g4[e] = (float)((double)ff[e] * zx[e] - (double)dd[e] * u[e]);
                    g5[e] = (float)((double)ff[e] * zy[e] - (double)dd[e] * v[e]);
                }
                st4(G0 + p, g0);
                st4(G1 + p, g1);
                st4(G2 + p, g2);
                st4(G4 + p, g4);
                st4(G5 + p, g5);
                T ux[4], uy[4], vx[4], vy[4], g3[4];
                ld4(UX + p, ux);
                ld4(UY + p, uy);
                ld4(VX + p, vx);
                ld4(VY + p, vy);
#pragma unroll
                for (int e = 0; e < 4; e++) g3[e] = ux[e] * vy[e] - uy[e] * vx[e];
                st4(G3 + p, g3);
            });
            fft.ptospc(st, 3 * ML,  // level-major
                plane_ld([=] __device__(int o) {
                    const int q = o / 3, which = o - 3 * q;
                    return PairLd<T>{(which == 0 ? G0 : which == 1 ? G1 : G3) + (size_t)q * n2, ng};
                }),
                plane_st([=] __device__(int o) {
                    const int q = o / 3, which = o - 3 * q;
                    return PairSt<T>{(which == 0 ? S0 : which == 1 ? S1 : S3) + (size_t)q * n2, ng};
                }));
            f32.ptospc(st, 3 * ML,
                plane_ld([=] __device__(int o) {
                    const int q = o / 3, which = o - 3 * q;
                    return PairLd<float>{(which == 0 ? G2 : which == 1 ? G4 : G5) + (size_t)q * n2, ng};
                }),
                plane_st([=] __device__(int o) {
                    const int q = o / 3, which = o - 3 * q;
                    return PairSt<float>{(which == 0 ? G2 : which == 1 ? G4 : G5) + (size_t)q * n2, ng};
                }));
            // combine in spectral space (as source())
            const float *S2 = G2, *S4 = G4, *S5 = G5;
            for_planes(st, ML, n2, [=] __device__(int q, int i) {
                const int m = q / L;
                const int kx = i % ng, ky = i / ng;
                const size_t b = (size_t)q * n2;
                const int mx = mirror(kx, ng) + ng * ky, my = kx + ng * mirror(ky, ng);
                const double wka = dmul(ky, ng) * (double)S1[b + my] + dmul(kx, ng) * (double)S0[b + mx];
                const double sq = filt[i] * ((double)S2[b + i] - wka);
                const double wkb = dmul(ky, ng) * (double)S5[b + my] + dmul(kx, ng) * (double)S4[b + mx];
                const double sd = filt[i] * (2.0 * (double)S3[b + i] + wkb - hlap[i] * PSp[b + i]);
                SQS[b + i] = sq;
                SDS[b + i] = sd;
                SGS[b + i] = COF * sq + wkd[(size_t)m * n2 + i] - FSQ * (double)AA[b + i];
            });
        }
    }

    // Reduce the three diagnose quantities per member into red_out[0 .. 3M).
    void diagnose_reduce() {
        const int n2 = this->n2, L = this->L, nz = this->nz;
        T *U = u, *V = v, *ZE = zeta;
        reduce_groups<3>(st, M, (long long)L * n2, 0x3u,
            [=] __device__(int m, long long j) {
                const int iz = (int)(j / n2);
                const size_t p = (size_t)m * L * n2 + j;
                const double uu = (double)U[p], vv = (double)V[p], ze = (double)ZE[p];
                RedVals<3> rv;
                rv.v[0] = uu * uu + vv * vv;
                rv.v[1] = fabs(ze);
                rv.v[2] = (iz == 0 || iz == nz) ? 0.5 * ze * ze : ze * ze;
                return rv;
            }, red_partial.p, red_out.p);
    }
    // Append this step's diagnostics to the device history ring (row counter on the device).
    void diagnose_record() {
        diagnose_reduce();
        const int M3 = 3 * M, cap = hist_cap;
        double *src = red_out.p, *hist = diag_hist.p;
        int* cnt = hist_dev.p;
        for_cols(st, 1, [=] __device__(int) {
            const int row = (*cnt) % cap;
            for (int k = 0; k < M3; k++) hist[(size_t)row * M3 + k] = src[k];
            *cnt = *cnt + 1;
        });
    }
    void diag_finish(const double* raw, double* out4) const {
        const double vsumi = 1.0 / (double)(ng * ng * nz);
        const double zrms = std::sqrt(vsumi * raw[2]);
        out4[0] = (1.0 / 2.0) * zrms * zrms;
        out4[1] = zrms;
        out4[2] = raw[1];
        out4[3] = std::sqrt(raw[0]);
    }

    // energies of savegrid (src/nhswps/mod.rs:365-410)
    // Spectrum of one float64 spectral plane on the device into out (kmax + 1).
    void spec1d(const double* ss, double* out) {
        const int nb = host.kmax + 1;
        k_spec_bins<<<(nb * 32 + 255) / 256, 256, 0, st>>>(nb, bin_off.p, bin_idx.p, bin_wt.p,
            [=] __device__(int e) { return ss[e] * ss[e]; }, out);
        SW_CHECK_LAUNCH();
        count_launch();
    }

    // savegrid's data for one member (src/nhswps/mod.rs:347-663), all on the device:
    // energies (ekin, epot, etot); the level-weighted shell spectra of zeta, delta,
    // gamma times spmf (3 (kmax + 1) values); the float32 snapshots q, delta,
    // gamma (physical), r, w, p (6 n3) and the 2-D fields -w/z(nz), the vertically
    // weighted vorticity and PV, gamma and h (5 n2).  One device-to-host copy.
    void savegrid(int member, double* energies, double* spectra, float* out3, float* out2) {
        energy(member, energies);
        const int ng = this->ng, n2 = this->n2, L = this->L, nz = this->nz, nb = host.kmax + 1;
        const size_t n3 = (size_t)L * n2;
        if (!snap.p) snap.alloc(6 * n3 + 5 * (size_t)n2);
        const size_t mb = (size_t)member * n3;
        const double *QS = qs.p + mb, *DS = ds.p + mb, *GS = gs.p + mb, *wgt = op.weight;
        const T *ZE = zeta.p + mb, *R = r.p + mb, *WW = w.p + mb, *Z = z.p + mb, *PN = pn.p + mb;
        T *ZS = W(0), *GP = W(1);
        float* S = snap.p;
        double* SPEC = spec_d.p;
        // zeta to spectral space (per level)
        fft.ptospc(st, L, [=] __device__(int q, int iy, int ix) -> T { return ZE[(size_t)q * n2 + iy + ng * ix]; },
                   [=] __device__(int q, int kx, int ky, T val) { ZS[(size_t)q * n2 + kx + ng * ky] = val; });
        k_spec_bins<<<(nb * 32 + 255) / 256, 256, 0, st>>>(nb, bin_off.p, bin_idx.p, bin_wt.p,
            [=] __device__(int e) {
                double a = 0.0;
                for (int iz = 0; iz < L; iz++) {
                    const double v = ZS[(size_t)iz * n2 + e];
                    a += wgt[iz] * (v * v);
                }
                return a;
            }, SPEC);
        SW_CHECK_LAUNCH();
        count_launch();
        k_spec_bins<<<(nb * 32 + 255) / 256, 256, 0, st>>>(nb, bin_off.p, bin_idx.p, bin_wt.p,
            [=] __device__(int e) {
                double a = 0.0;
                for (int iz = 0; iz < L; iz++) {
                    const double v = DS[(size_t)iz * n2 + e];
                    a += wgt[iz] * (v * v);
                }
                return a;
            }, SPEC + nb);
        SW_CHECK_LAUNCH();
        count_launch();
        k_spec_bins<<<(nb * 32 + 255) / 256, 256, 0, st>>>(nb, bin_off.p, bin_idx.p, bin_wt.p,
            [=] __device__(int e) {
                double a = 0.0;
                for (int iz = 0; iz < L; iz++) {
                    const double v = GS[(size_t)iz * n2 + e];
                    a += wgt[iz] * (v * v);
                }
                return a;
            }, SPEC + 2 * nb);
        SW_CHECK_LAUNCH();
        count_launch();
        // q, delta, gamma to physical space (float32 snapshots; gamma also kept in T)
        fft.spctop(st, 3 * L,
            [=] __device__(int o, int kx, int ky) -> T {
                const int which = o / L, iz = o - which * L;
                return (T)(which == 0 ? QS : which == 1 ? DS : GS)[(size_t)iz * n2 + kx + ng * ky];
            },
            [=] __device__(int o, int iy, int ix, T val) {
                const size_t p = (size_t)o * n2 + iy + ng * ix;
                S[p] = (float)val;
                if (o >= 2 * L) GP[p - 2 * n3] = val;
            });
        for_planes(st, 3 * L, n2, [=] __device__(int q, int i) {
            const int which = q / L;
            const size_t p = (size_t)(q - which * L) * n2 + i;
            const T* src = which == 0 ? R : which == 1 ? WW : PN;
            S[3 * n3 + (size_t)q * n2 + i] = (float)src[p];
        });
        float* S2 = S + 6 * n3;
        for_cols(st, n2, [=] __device__(int i) {
            const double zt = (double)Z[(size_t)nz * n2 + i];
            double wz = 0.0, wg = 0.0;
            for (int iz = 0; iz < L; iz++) {
                const size_t p = (size_t)iz * n2 + i;
                const double f = 1.0 + (double)R[p];
                wz += wgt[iz] * (double)ZE[p] * f;
                wg += wgt[iz] * (double)GP[p] * f;
            }
            wz *= HBAR / zt;
            wg *= HBAR / zt;
            S2[i] = (float)(-(double)WW[(size_t)nz * n2 + i] / zt);
            S2[n2 + i] = (float)wz;
            S2[2 * (size_t)n2 + i] = (float)(HBAR * (wz + COF) / zt - COF);
            S2[3 * (size_t)n2 + i] = (float)wg;
            S2[4 * (size_t)n2 + i] = (float)((1.0 / HBAR) * zt - 1.0);
        });
        SW_CUDA(cudaMemcpyAsync(spectra, SPEC, sizeof(double) * 3 * nb, cudaMemcpyDeviceToHost, st));
        SW_CUDA(cudaMemcpyAsync(out3, S, sizeof(float) * 6 * n3, cudaMemcpyDeviceToHost, st));
        SW_CUDA(cudaMemcpyAsync(out2, S2, sizeof(float) * 5 * (size_t)n2, cudaMemcpyDeviceToHost, st));
        SW_CUDA(cudaStreamSynchronize(st));
        for (int k = 0; k < nb; k++)
            for (int j = 0; j < 3; j++) spectra[j * nb + k] *= host.spmf[k];
    }

    void energy(int member, double* out3) {
        const int n2 = this->n2, L = this->L, nz = this->nz;
        T *R = r, *U = u, *V = v, *WW = w, *Z = z;
        reduce_groups<2>(st, M, (long long)L * n2, 0u,
            [=] __device__(int m, long long j) {
                const int iz = (int)(j / n2);
                const size_t p = (size_t)m * L * n2 + j;
                const double uu = U[p], vv = V[p], ww = WW[p], rr = R[p];
                RedVals<2> rv;
                if (iz == 0) rv.v[0] = 0.5 * ((1.0 + rr) * (uu * uu + vv * vv));
                else if (iz == nz) rv.v[0] = 0.5 * ((1.0 + rr) * (uu * uu + vv * vv + ww * ww));
                else rv.v[0] = (1.0 + rr) * (uu * uu + vv * vv + ww * ww);
                if (iz == nz) {
                    const double h = (1.0 / HBAR) * (double)Z[p] - 1.0;
                    rv.v[1] = h * h;
                } else {
                    rv.v[1] = 0.0;
                }
                return rv;
            }, red_partial.p, red_out.p);
        double h[2];
        SW_CUDA(cudaMemcpyAsync(h_pinned, red_out.p + 2 * member, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
        SW_CUDA(cudaStreamSynchronize(st));
        h[0] = h_pinned[0];
        h[1] = h_pinned[1];
        const double gl = (2.0 * PI) / (double)ng, dz = HBAR / (double)nz, gvol = gl * gl * dz;
        const double ekin = h[0] * ((1.0 / 2.0) * gvol * (1.0 / HBAR));
        const double epot = (1.0 / 2.0) * (gl * gl) * CSQ * h[1];
        out3[0] = ekin;
        out3[1] = epot;
        out3[2] = ekin + epot;
    }

    // ======================================================================
    // advance (src/nhswps/advance.rs:13-279)
    // WD(2..10): qsi, qsm, sqs, sds, nds, sgs, ngs, dsi, gsi
    // ======================================================================
    void advance_update(bool first) {
        NvtxRange nv("advance_update");
        const int n2 = this->n2, L = this->L;
        const double dt = 1.0 / (double)ng, dt4 = dt / 4.0, dt4i = 1.0 / dt4;
        const double *diss = op.diss, *rdis = op.rdis, *fope = op.fope, *c2g2 = op.c2g2, *simp = op.simp,
                     *wgt = op.weight;
        double *QS = qs, *DS = ds, *GS = gs;
        double *qsi = WD(2), *qsm = WD(3), *sqs = WD(4), *sds = WD(5), *nds = WD(6), *sgs = WD(7), *ngs = WD(8),
               *dsi = WD(9), *gsi = WD(10);
        const int ncols = M * n2, nb = (ncols + UPDATE_THREADS - 1) / UPDATE_THREADS;
#define SW_UPDATE_CASE(LSV)                                                                                      \
    case LSV:                                                                                                    \
        if (first)                                                                                               \
            k_update<LSV, true><<<nb, UPDATE_THREADS, 0, st>>>(n2, ncols, dt4, dt4i, diss, rdis, fope, c2g2, simp, \
                                                               wgt, QS, DS, GS, qsi, qsm, sqs, sds, nds, sgs, ngs,  \
                                                               dsi, gsi);                                          \
        else                                                                                                     \
            k_update<LSV, false><<<nb, UPDATE_THREADS, 0, st>>>(n2, ncols, dt4, dt4i, diss, rdis, fope, c2g2,      \
                                                                simp, wgt, QS, DS, GS, qsi, qsm, sqs, sds, nds, sgs, \
                                                                ngs, dsi, gsi);                                     \
        SW_CHECK_LAUNCH();                                                                                       \
        count_launch();                                                                                          \
        return;
        switch (L) {
            SW_UPDATE_CASE(5)
            SW_UPDATE_CASE(9)
            SW_UPDATE_CASE(17)
            default: break;  // deeper columns: the streamed loop below (registers would spill)
        }
#undef SW_UPDATE_CASE
        for_cols(st, M * n2, [=] __device__(int c) {
            const int m = c / n2, i = c - m * n2;
            const size_t cb = (size_t)m * L * n2 + i;
            const double dis = diss[i], rd = rdis[i], fo = fope[i], cg = c2g2[i], si = simp[i];
            double wka = 0.0, wkb = 0.0;
            #pragma unroll 4
            for (int iz = 0; iz < L; iz++) {
                const size_t p = cb + (size_t)iz * n2;
                if (first) {
                    qsi[p] = QS[p];
                    qsm[p] = QS[p] + dt4 * sqs[p];
                    dsi[p] = DS[p];
                    gsi[p] = GS[p];
                    nds[p] = sds[p] + dt4i * dsi[p];
                    ngs[p] = sgs[p] + dt4i * gsi[p];
                }
                QS[p] = dis * (qsm[p] + dt4 * sqs[p]) - qsi[p];
                const double sd = sds[p] + nds[p];
                const double sg = sgs[p] + ngs[p];
                sds[p] = sd;
                sgs[p] = sg;
                const double d = sg + rd * sd;
                DS[p] = d;
                wka += wgt[iz] * d;
                wkb += wgt[iz] * sd;
            }
            wka *= fo;
            wkb *= cg;
            double wkg = 0.0;
            #pragma unroll 4
            for (int iz = 0; iz < L; iz++) {
                const size_t p = cb + (size_t)iz * n2;
                DS[p] = si * (DS[p] - wka) - dsi[p];
                const double g = wkb - FSQ * sds[p] + rd * sgs[p];
                GS[p] = g;
                wkg += wgt[iz] * g;
            }
            wkg *= fo;
            #pragma unroll 4
            for (int iz = 0; iz < L; iz++) {
                const size_t p = cb + (size_t)iz * n2;
                GS[p] = si * (GS[p] - wkg) - gsi[p];
            }
        });
    }

    // One step with host-driven pressure loops (one stream sync per sweep).
    int advance_direct(bool ggen) {
        NvtxRange nv("advance_step");
        int it = 0;
        double e = 0.0;
        last_sweeps[0] = last_sweeps[1] = last_sweeps[2] = 0;
        StepHints hints(*this);
        if (!ggen) reset_guess_history();
        if (ggen) {
            main_invert();
            hints.before_psolve(false, 0);
            int stt = psolve(100, &it, &e);
            last_sweeps[0] = it;
            if (stt) return stt;
        }
        diagnose_record();
        hints.before_source(ggen);
        source(WD(4), WD(5), WD(7), ggen && fused_prepare);
        advance_update(true);
        for (int k = 0; k < 2; k++) {
            main_invert();
            hints.before_psolve(ggen || k > 0, ggen ? 1 + k : -1);
            int stt = psolve(100, &it, &e);
            last_sweeps[1 + k] = it;
            if (stt) return stt;
            hints.before_source(true);
            source(WD(4), WD(5), WD(7), fused_prepare);
            advance_update(false);
        }
        t += 1.0 / (double)ng;
        last_from_graph = false;
        return SW_OK;
    }

    // Sets the reuse hints for the calls of one step and clears them when the step
    // ends (also on an error), so that the per-function entry points never see them.
    struct StepHints {
        Solver& s;
        explicit StepHints(Solver& sv) : s(sv) {}
        ~StepHints() {
            s.hint_uv_spec = s.hint_ps_guess = s.hint_q_phys = false;
            s.guess_slot = -1;
        }
        // main_invert of this stage ran; a psolve of this step already finished?
        // slot: the solve's slot in a ggen step (0, 1, 2) for the mixed path's
        // predicted first iterate, or -1
        void before_psolve(bool previous_solve_this_step, int slot = -1) {
            s.hint_uv_spec = s.fused_prepare;
            s.hint_ps_guess = s.fused_prepare && previous_solve_this_step;
            s.hint_q_phys = false;
            s.guess_slot = slot;
        }
        void before_source(bool invert_this_stage) {
            s.hint_uv_spec = s.hint_ps_guess = false;
            s.hint_q_phys = invert_this_stage;
            s.guess_slot = -1;
        }
    };

    // The work of one step as captured into a CUDA graph: the three pressure
    // solves iterate inside conditional WHILE nodes, so a step needs no host
    // round trip.
    void advance_captured(bool ggen) {
        NvtxRange nv("advance_step_capture");
        SW_CUDA(cudaMemsetAsync(sweeps_dev.p, 0, sizeof(int) * 3 * M, st));
        StepHints hints(*this);
        if (!ggen) reset_guess_history();
        if (ggen) {
            main_invert();
            hints.before_psolve(false, 0);
            psolve_captured(100, 0);
        }
        diagnose_record();
        hints.before_source(ggen);
        source(WD(4), WD(5), WD(7), ggen && fused_prepare);
        advance_update(true);
        for (int k = 0; k < 2; k++) {
            main_invert();
            hints.before_psolve(ggen || k > 0, ggen ? 1 + k : -1);
            psolve_captured(100, 1 + k);
            hints.before_source(true);
            source(WD(4), WD(5), WD(7), fused_prepare);
            advance_update(false);
        }
    }

    // The work of one step captured on st, which must be capturing already (into
    // this context's step graph or into an ensemble's combined graph).  Records the
    // kernels per step outside the sweep loops for the launch accounting.
    void capture_step_body(bool ggen) {
        const long long c0 = launch_counter().load();
        advance_captured(ggen);
        // nodes captured (nothing ran): kernels outside the sweep loops
        const long long captured = launch_counter().load() - c0;
        k_fixed[ggen ? 1 : 0] = captured - (ggen ? 3 : 2) * k_sweep;
        launch_counter().fetch_sub(captured);
    }

    // Bookkeeping of nsteps steps launched by someone else's graph on another stream
    // (an ensemble): time, pending status and launch accounting, as advance_enqueue.
    void note_external_steps(int nsteps, bool ggen_first) {
        for (int k = 0; k < nsteps; k++) {
            const bool g = k == 0 ? ggen_first : true;
            pending_fixed += k_fixed[g ? 1 : 0];
            t += 1.0 / (double)ng;
        }
        pending = true;
    }

    cudaGraphExec_t step_graph(bool ggen) {
        cudaGraphExec_t& ex = step_exec[ggen ? 1 : 0];
        if (!ex) {
            SW_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            try {
                capture_step_body(ggen);
            } catch (...) {
                cudaGraph_t g;
                cudaStreamEndCapture(st, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            cudaGraph_t g;
            SW_CUDA(cudaStreamEndCapture(st, &g));
            SW_CUDA(cudaGraphInstantiate(&ex, g, 0));
            SW_CUDA(cudaGraphDestroy(g));
        }
        return ex;
    }

    // nsteps steps as graph launches queued on the context's stream (no host
    // synchronisation); advance_finish() waits for them and checks the sticky
    // status of the pressure solves.
    void advance_enqueue(int nsteps, bool ggen_first) {
        for (int k = 0; k < nsteps; k++) {
            const bool g = k == 0 ? ggen_first : true;
            SW_CUDA(cudaGraphLaunch(step_graph(g), st));
            pending_fixed += k_fixed[g ? 1 : 0];
            t += 1.0 / (double)ng;
        }
        pending = true;
    }
    int advance_graph(int nsteps, bool ggen_first) {
        advance_enqueue(nsteps, ggen_first);
        return advance_finish();
    }
    int advance_finish() {
        const long long fixed = pending_fixed;
        pending_fixed = 0;
        pending = false;
        int* h = reinterpret_cast<int*>(h_pinned);
        long long* hx = reinterpret_cast<long long*>(h_pinned + 4);
        SW_CUDA(cudaMemcpyAsync(h, err_dev.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        SW_CUDA(cudaMemcpyAsync(h + 1, sweeps_dev.p, sizeof(int) * 3, cudaMemcpyDeviceToHost, st));
        SW_CUDA(cudaMemcpyAsync(hx, sweep_exec.p, 2 * sizeof(long long), cudaMemcpyDeviceToHost, st));
        SW_CUDA(cudaMemsetAsync(sweep_exec.p, 0, 2 * sizeof(long long), st));
        SW_CUDA(cudaStreamSynchronize(st));
        count_launch(fixed + hx[0] * k_sweep_kind[0] + hx[1] * k_sweep_kind[1]);
        sweeps_run[0] += hx[0];
        sweeps_run[1] += hx[1];
        for (int i = 0; i < 3; i++) last_sweeps[i] = h[1 + i];
        last_from_graph = true;
        if (h[0] != SW_OK) {
            SW_CUDA(cudaMemset(err_dev.p, 0, sizeof(int)));
            return h[0];
        }
        return SW_OK;
    }

    int advance(int nsteps, bool ggen_first) {
        if (use_graphs) return advance_graph(nsteps, ggen_first);
        for (int k = 0; k < nsteps; k++) {
            int stt = advance_direct(k == 0 ? ggen_first : true);
            if (stt) return stt;
        }
        return SW_OK;
    }
    bool use_graphs = true;
    // Set by the advance flows around the calls they apply to (see
    // psolve_prepare_fused and source): what earlier work of the same step left.
    bool hint_uv_spec = false;  // Su, Sv hold the spectra of u, v (main_invert ran this stage)
    bool hint_ps_guess = false; // ps holds the previous solution of this step (or, mixed path, of the last step)
    DevBuf<double> xh;          // mixed path: solutions of the last step's three solves
    DevBuf<int> xflag;          // which of them are written
    int guess_slot = -1;        // slot of the next solve in a ggen step (-1: none)
    bool hint_q_phys = false;   // zeta and r are this stage's main_invert output
    bool pending = false;        // steps queued by advance_enqueue and not yet finished
    long long pending_fixed = 0; // their kernel launches outside the sweep loops
    bool fused_prepare = true;  // psolve set-up as eight fused batched transforms
    bool last_from_graph = false;
};

}  // namespace sw
