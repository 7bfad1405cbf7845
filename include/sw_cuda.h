/*
 * sw_cuda.h -- C ABI of the B200 (sm_100a) implementation of the nhswps
 * time-step path of rse-standrewscs/shallow-water.
 *
 * Plain C: int status codes, plain pointers and sizes, no C++ or torch types.
 * All arrays are float64 in the reference's Fortran order (src/utils.rs:6-32):
 *   physical plane rvar(ny,nx) -> p[iy + ng*ix], spectral svar(nx,ny) -> s[kx + ng*ky],
 *   3-D fields add + ng*ng*iz for the nz+1 levels iz = 0..nz.
 * Host-pointer entry points copy in and out around the GPU work; the
 * `_dev` entry points take device pointers and a cudaStream_t (as void*).
 * A context is not thread-safe: use one context per host thread/stream.
 * Every entry point returns SW_OK or an error status; sw_last_error() gives the
 * message of the calling thread's last failure.
 */
#ifndef SW_CUDA_H
#define SW_CUDA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define SW_OK 0
#define SW_ERR_FACTORISE 1       /* n not of the form 2^a 3^b 5^c (stafft/mod.rs:148-149) */
#define SW_ERR_CUDA 2            /* CUDA runtime failure */
#define SW_ERR_PSOLVE_DIVERGED 3 /* pressure error > 1 after a sweep (psolve.rs:349-352) */
#define SW_ERR_PSOLVE_MAXITER 4  /* pressure iteration hit its cap (psolve.rs:360-366) */
#define SW_ERR_ARG 6             /* invalid argument or size */
#define SW_ERR_STATE 7           /* call made in the wrong state */

/* ---- precision of the hot path ---------------------------------------------- */
#define SW_FP64 0  /* everything in float64 */
/* float64 fields and most transforms; float32 where its rounding stays far below
 * 1e-5 rel-L2 after 10 steps at ng=256: (1) after each solve's float64 reference
 * sweep, the pressure sweeps are float32 correction sweeps on the distance from the
 * reference point (stop rule 1e-7, sw_set_psolve_toler), and (2) the dealiased
 * products and filters of the pressure set-up and of source go through float32
 * transforms.  Measured ~4e-7 rel-L2 on gamma against SW_FP64 after 13 steps at
 * ng=256, nz=16. */
#define SW_MIXED 1
/* float32 transforms, products and physical work fields; float64 prognostic fields,
 * tridiagonal solves, residual, diagnostics and time update; the pressure iteration
 * stops at 1e-6 or on stagnation.  Fastest, but its gravity-wave fields (delta,
 * gamma) carry ~1e-4 relative error after 10 steps at ng=256. */
#define SW_FP32 2

/* ---- fields of nhswps::State (src/nhswps/mod.rs:87-148) ------------------------ */
enum sw_field {
    SW_U = 0, SW_V, SW_W, SW_Z, SW_ZX, SW_ZY, SW_R, SW_RI, SW_AA, SW_ZETA,
    SW_PN, SW_DPN, SW_PS, SW_QS, SW_DS, SW_GS, SW_NFIELDS
};

typedef struct sw_ctx sw_ctx;

const char* sw_last_error(void);
int sw_version(void);

/* ---- stafft (src/stafft/mod.rs) ----------------------------------------------- */
/* Replaces stafft::factorisen (src/stafft/mod.rs:97-150). */
int sw_factorisen(int n, int factors[5]);
/* Replaces stafft::initfft (src/stafft/mod.rs:67-95): trig has 2n entries. */
int sw_initfft(int n, int factors[5], double* trig);
/* Replace stafft::forfft / revfft (src/stafft/mod.rs:158, 301): m transforms of
 * length n on x[i + m*j] (host memory, in place).  trig/factors are checked for
 * consistency with n when non-NULL; the GPU keeps its own twiddle tables. */
int sw_forfft(int m, int n, double* x, const double* trig, const int factors[5]);
int sw_revfft(int m, int n, double* x, const double* trig, const int factors[5]);
/* Same on device memory: precision SW_FP64 (x is double*), SW_MIXED or SW_FP32 (x is float*). */
int sw_forfft_dev(int m, int n, void* x, int precision, void* stream);
int sw_revfft_dev(int m, int n, void* x, int precision, void* stream);

/* ---- context: one ensemble of nmembers runs of the same (ng, nz) -------------- */
/* Replaces Spectral::new(ng, nz) (src/spectral/mod.rs:65-299) plus the State
 * allocation of nhswps (src/nhswps/mod.rs:190-235). */
int sw_ctx_create(int ng, int nz, int nmembers, int precision, int device, sw_ctx** out);
void sw_ctx_destroy(sw_ctx* ctx);
int sw_ctx_info(const sw_ctx* ctx, int* ng, int* nz, int* nmembers, int* precision);
/* Copy a named Spectral operator out ("hlap", "filt", "htdv", ... "kmag"); n = element count. */
int sw_spectral_get(sw_ctx* ctx, const char* name, double* out, size_t n);

/* State fields, host float64, ng*ng*(nz+1) values per member. */
int sw_state_set(sw_ctx* ctx, int field, int member, const double* host, size_t n);
int sw_state_get(sw_ctx* ctx, int field, int member, double* host, size_t n);
/* Whole-ensemble copies: host holds nmembers*ng*ng*(nz+1) values, member-major. */
int sw_state_set_all(sw_ctx* ctx, int field, const double* host, size_t n);
int sw_state_get_all(sw_ctx* ctx, int field, double* host, size_t n);
/* Same without waiting: the copies are queued on the context's stream (after any
 * queued steps) and complete at sw_sync.  host must stay valid until then and
 * should be page-locked for the copy to run asynchronously.  With several
 * contexts on their own streams, one context's copies overlap another's steps.
 * No reference counterpart. */
int sw_state_set_all_async(sw_ctx* ctx, int field, const double* host, size_t n);
int sw_state_get_all_async(sw_ctx* ctx, int field, double* host, size_t n);
int sw_set_time(sw_ctx* ctx, double t);
int sw_get_time(const sw_ctx* ctx, double* t);

/* ---- spectral operators on host arrays (member-independent) ------------------- */
/* D2FFT::ptospc / spctop (src/sta2dfft.rs:91-123): one ng*ng plane. */
int sw_ptospc(sw_ctx* ctx, const double* rvar, double* svar);
int sw_spctop(sw_ctx* ctx, const double* svar, double* rvar);
/* D2FFT::xderiv / yderiv (src/sta2dfft.rs:128-184) */
int sw_xderiv(sw_ctx* ctx, const double* var, double* der);
int sw_yderiv(sw_ctx* ctx, const double* var, double* der);
/* Spectral::jacob / divs (src/spectral/mod.rs:423-475): physical aa, bb -> spectral cs. */
int sw_jacob(sw_ctx* ctx, const double* aa, const double* bb, double* cs);
int sw_divs(sw_ctx* ctx, const double* aa, const double* bb, double* cs);
/* Spectral::deal2d (one plane) and deal3d (nz+1 planes), in place. */
int sw_deal2d(sw_ctx* ctx, double* fp);
int sw_deal3d(sw_ctx* ctx, double* fp);
/* Spectral::ptospc3d / spctop3d (src/spectral/mod.rs:479-522), levels izbeg..izend. */
int sw_ptospc3d(sw_ctx* ctx, const double* fp, double* fs, int izbeg, int izend);
int sw_spctop3d(sw_ctx* ctx, const double* fs, double* fp, int izbeg, int izend);
/* Spectral::spec1d (src/spectral/mod.rs:558-591): spec has ng+1 entries. */
int sw_spec1d(sw_ctx* ctx, const double* ss, double* spec);
/* balinit (src/balinit.rs:21-435): the balanced 2-D fields (qq, dd, gg; ng*ng each,
 * Fortran order) of the PV field qq_init, by the reference's fixed-point iteration
 * on the device.  *iters (may be NULL) gets the iteration count.  SW_FP64 and
 * SW_MIXED contexts (float64); SW_ERR_STATE on SW_FP32. */
int sw_balinit(sw_ctx* ctx, const double* qq_init, double* qq, double* dd, double* gg, int* iters);

/* ---- nhswps numerics on the context's state (all members) ----------------------- */
/* Spectral::main_invert (src/spectral/mod.rs:305-417): qs,ds,gs -> r,u,v,zeta. */
int sw_main_invert(sw_ctx* ctx);
/* vertical (src/nhswps/vertical.rs:8-143): r,u,v,ds -> z,zx,zy,aa,w. */
int sw_vertical(sw_ctx* ctx);
/* coeffs (src/nhswps/coeffs.rs:8-101); outputs of member 0 copied to host when non-NULL. */
int sw_coeffs(sw_ctx* ctx, double* sigx, double* sigy, double* cpt1, double* cpt2);
/* cpsource (src/nhswps/cpsource.rs:13-261); sp0 of member 0 to host when non-NULL. */
int sw_cpsource(sw_ctx* ctx, double* sp0);
/* psolve (src/nhswps/psolve.rs:16-411).  iters/errp (may be NULL) receive member
 * 0's sweep count and final relative change.  nitmax <= 0 selects the reference's 100. */
int sw_psolve(sw_ctx* ctx, int nitmax, int* iters, double* errp);
/* source (src/nhswps/source.rs:19-138); outputs of member 0 to host when non-NULL. */
int sw_source(sw_ctx* ctx, double* sqs, double* sds, double* sgs);
/* advance (src/nhswps/advance.rs:13-279): nsteps predictor-corrector steps.
 * ggen != 0 runs main_invert + psolve at the start of the first step (the
 * reference's State::ggen); later steps always do. */
int sw_advance(sw_ctx* ctx, int nsteps, int ggen);
/* Run each advance step as one CUDA graph whose pressure iterations are
 * conditional WHILE nodes (enable = 1, the default), or drive the iterations from
 * the host with one synchronisation per sweep (enable = 0).  Same results. */
int sw_set_graphs(sw_ctx* ctx, int enable);
/* Stop rule of the pressure iteration of an SW_MIXED context: the relative change
 * below which psolve stops (default 1e-7; SW_FP64 keeps the reference's 1e-9,
 * psolve.rs:17).  The correction sweeps converge below float32 rounding, so any
 * value down to 1e-9 is reachable.  SW_ERR_STATE on other precisions.  No reference
 * counterpart. */
int sw_set_psolve_toler(sw_ctx* ctx, double toler);
/* Relaxation factor omega in (0, 1] of the pressure iteration: each sweep's new
 * iterate is x + omega (G(x) - x), where G(x) is the Thomas solve of the source at
 * x.  The fixed point does not depend on omega; the stop rule measures the
 * unrelaxed change |G(x) - x|.  The default, 1, is the reference's iteration
 * (psolve.rs:89-358), whose sweep counts the FP64 path reproduces.  0.8 needs ~40%
 * fewer sweeps at ng=256, nz=16 (the slowest modes alternate in sign), but the fast
 * modes then contract by only 1 - omega per sweep, so at the same stop rule the
 * result lies farther from the fixed point (gamma ~10x farther at ng=256).  With
 * omega != 1 the float32/float64 sweep schedule of SW_MIXED, which is decided per
 * context, can make an ensemble member differ from its single run at ~1e-9.
 * SW_ERR_ARG outside (0, 1].  No reference counterpart. */
int sw_set_psolve_relax(sw_ctx* ctx, double omega);
/* Pressure sweeps run on the context so far (each covers all members): out[0] float64
 * sweeps (every sweep of SW_FP64 and SW_FP32, the reference sweeps of SW_MIXED),
 * out[1] float32 correction sweeps of SW_MIXED.  No reference counterpart. */
int sw_sweep_counts(sw_ctx* ctx, long long out[2]);
/* Tuning of the batched 2-D transforms: planes per pair of tile-pass launches
 * (1 .. the context's capacity, 6*(nz+1)*nmembers; planes <= 0 only queries).
 * *in_use (may be NULL) gets the value now in use.  Results do not depend on it.  No reference counterpart:
 * the reference transforms one plane at a time (src/sta2dfft.rs:91-123). */
int sw_set_fft_chunk(sw_ctx* ctx, int planes, int* in_use);
/* Batched 2-D transforms at n = 256 as one single-pass launch (enable = 1):
 * thread-block clusters of 8 CTAs each hold a plane and exchange its transposed
 * intermediate through distributed shared memory, so every plane is read and
 * written once.  enable = 0 (the default) selects the two tile passes through the
 * intermediate in global memory; enable < 0 only queries.  *in_use (may be NULL) gets the
 * setting in use (0 at other lengths).  Results are bit-identical.  No reference
 * counterpart. */
int sw_set_fft_single_pass(sw_ctx* ctx, int enable, int* in_use);
/* Two-stream chunk pipeline of the batched 2-D transforms (enable = 1): chunks
 * alternate between the context's stream and a second one with two intermediates,
 * so that one chunk's second pass overlaps the next chunk's first pass and a chunk
 * small enough keeps its intermediate in L2.  The chunk is then at most half the
 * capacity.  enable = 0 (the default) runs the chunks in order on one stream;
 * enable < 0 only queries.  *in_use (may be NULL) gets the setting.  Results are
 * bit-identical.  No reference counterpart. */
int sw_set_fft_overlap(sw_ctx* ctx, int enable, int* in_use);
/* Columns per tile of the n = 256 tile passes, 16 or 32 (other lengths have a fixed
 * tile; columns <= 0 only queries).  *in_use (may be NULL) gets the value now in
 * use.  Results do not depend on it.  No reference counterpart. */
int sw_set_fft_tile(sw_ctx* ctx, int columns, int* in_use);
/* Autotuner of the 2-D transform launches: times reps forward + inverse transforms
 * of the pressure sweep's batch (3*nz planes per member) for each tile width the
 * grid has kernels for (n = 256: 16 and 32 columns), each chunk (without the
 * two-stream pipeline: the capacity halved down to 8 planes; with it: a half and a
 * quarter of the capacity), on scratch buffers it allocates, and keeps the fastest.  Up
 * to maxc rows of (tiles[i], chunks[i], overlaps[i], ms[i] per transform pair) are
 * written when the arrays are non-NULL; *ncand gets the row count, *chosen_tile,
 * *chosen_chunk and *chosen_overlap the values now in use.  No reference
 * counterpart. */
int sw_autotune_fft(sw_ctx* ctx, int reps, int maxc, int* tiles, int* chunks, int* overlaps, float* ms, int* ncand,
                    int* chosen_tile, int* chosen_chunk, int* chosen_overlap);
/* diagnose (src/nhswps/mod.rs:666-711) of one member:
 * out = {0.5*zrms^2, zrms, zmax, umax}. */
int sw_diagnose(sw_ctx* ctx, int member, double out[4]);
/* Diagnostics recorded at the start of each advance step since the last call:
 * out holds up to cap rows of {member-0 values x4}; *count gets the row count. */
int sw_diag_history(sw_ctx* ctx, double* out, int cap, int* count);
/* Energies of savegrid (src/nhswps/mod.rs:365-410) of one member: {ekin, epot, etot}. */
int sw_energy(sw_ctx* ctx, int member, double out[3]);
/* savegrid's data for one member in one call (src/nhswps/mod.rs:347-663), computed
 * on the device: energies = {ekin, epot, etot}; spectra = the level-weighted
 * shell spectra of zeta, delta and gamma times spmf, 3 blocks of kmax+1 values
 * (nspec = 3*(kmax+1); kmax from sw_spectral_get "kmax"); fields3 = float32
 * q, delta, gamma (physical), r, w, p, 6 blocks of ng*ng*(nz+1) in Fortran order;
 * fields2 = float32 -w/z, weighted vorticity, PV, weighted gamma and h at the
 * top level, 5 blocks of ng*ng.  The caller writes the reference's text and .r4
 * records from these. */
int sw_savegrid(sw_ctx* ctx, int member, double energies[3], double* spectra, int nspec, float* fields3,
                float* fields2);
/* psolve sweep counts of the last advance step for member 0 (3 entries). */
int sw_last_sweeps(sw_ctx* ctx, int out[3]);
/* advance without waiting: queues nsteps graph-captured steps on the context's
 * stream and returns (with graphs off it runs them synchronously).  Contexts on
 * different streams then run concurrently, e.g. the groups of an ensemble with
 * uneven grid sizes.  sw_sync waits for them and returns the pressure solves'
 * status; other calls on the context are ordered after the queued steps.  No
 * reference counterpart (the reference runs one member). */
int sw_advance_async(sw_ctx* ctx, int nsteps, int ggen);
/* Synchronise the context's stream; after sw_advance_async, finish those steps
 * and return their status (as sw_advance would). */
int sw_sync(sw_ctx* ctx);

/* ---- device-resident access for benchmarking and zero-copy callers ----------------- */
/* Device pointer of a state field (all members, member-major) and its element size
 * in bytes (8 for the float64 fields; 4 for the float32 work fields of SW_FP32). */
int sw_field_device_ptr(sw_ctx* ctx, int field, void** ptr, int* elem_bytes);
/* Batched tridiagonal solves, float64: nsys independent systems of n <= 33
 * unknowns, a[i] x[i-1] + b[i] x[i] + c[i] x[i+1] = d[i] (a[0], c[n-1] unused),
 * level-major with the system index contiguous ([s + nsys*i]); no pivoting.  The
 * vertical Thomas solve of psolve (src/nhswps/psolve.rs:285-327) for general
 * coefficients; the reference has no standalone entry point.  Device arrays on
 * `stream`; the _host variant copies host arrays through device memory. */
int sw_tridiag_batched(int n, int nsys, const double* a, const double* b, const double* c, const double* d,
                       double* x, void* stream);
int sw_tridiag_batched_host(int n, int nsys, const double* a, const double* b, const double* c, const double* d,
                            double* x);
/* The context's CUDA stream (cudaStream_t as void*). */
int sw_stream(sw_ctx* ctx, void** stream);
/* Batched 2-D transforms on device memory with the context's plan: direction 0 =
 * ptospc (physical -> spectral), 1 = spctop; nplanes ng*ng planes of the context's
 * work precision (double for SW_FP64 and SW_MIXED, float for SW_FP32); in and out may alias.
 * Launches two tile passes per call (reference D2FFT::ptospc/spctop, src/sta2dfft.rs:91-123). */
int sw_fft2d_dev(sw_ctx* ctx, int direction, int nplanes, const void* in, void* out);
/* Allocation-free batched 2-D transforms (no counterpart in the reference).
 * Same transforms as sw_fft2d_dev, float64, but needing no context and calling
 * no cudaMalloc: for callers that cannot allocate device memory where they
 * transform (a plugin inside a framework that owns the device memory pool, code
 * being captured into someone else's CUDA graph, allocation-free real-time loops).
 * in/out are the caller's device buffers of nplanes ng*ng planes (may alias);
 * stream is a cudaStream_t.  Scaling as sw_fft2d_dev and D2FFT: 1/sqrt(ng) per
 * axis each way, so ptospc then spctop returns the input.  Scratch is a fixed
 * 16 MiB array inside the library, held by every GPU that loads it until exit.
 * Accepted: even ng in [4, 1024] that factors into 2, 3 and 5, direction 0 or 1,
 * nplanes >= 1 and non-NULL buffers; otherwise SW_ERR_ARG (size, direction,
 * buffers) or SW_ERR_FACTORISE (another prime factor).  A CUDA error pending from
 * the caller's earlier work is reported as SW_ERR_CUDA and left pending.  All
 * calls share the scratch array: calls overlapping on the GPU race, so serialise
 * them on one stream.  The first call on a device (and the first after the
 * device's context changes) looks the array's address up; make it before any
 * stream capture that records this call. */
int sw_fft2d_noalloc(int ng, int direction, int nplanes, const double* in, double* out, void* stream);
/* ---- ensembles of members with uneven grids ------------------------------------ */
/* nmembers members, member k of grid ng[k] x ng[k] x (nz[k]+1), all of one
 * precision on one device.  Members of one (ng, nz) share one batched context; a
 * step of the whole ensemble is ONE CUDA graph launch whose parallel branches are
 * the groups' steps, so the groups' kernels run concurrently.  The reference runs
 * one member at a time and has no counterpart. */
typedef struct sw_ensemble sw_ensemble;
int sw_ensemble_create(const int* ng, const int* nz, int nmembers, int precision, int device, sw_ensemble** out);
/* Destroys the ensemble and its group contexts. */
void sw_ensemble_destroy(sw_ensemble* e);
int sw_ensemble_info(const sw_ensemble* e, int* nmembers, int* ngroups);
/* The stream the ensemble's step graphs are launched on (cudaStream_t as void*). */
int sw_ensemble_stream(sw_ensemble* e, void** stream);
/* The context that holds member `member` and the member's index in it: fields are
 * set and read with the context's entry points (sw_state_set(ctx, field, index, ...)).
 * The context belongs to the ensemble (do not destroy it); tune it (chunk, tile,
 * tolerance) before the ensemble's first step, which captures the combined graph. */
int sw_ensemble_member(sw_ensemble* e, int member, sw_ctx** ctx, int* index);
/* nsteps steps of every member (ggen as sw_advance for the first); the _async form
 * queues them and returns, sw_ensemble_sync waits and returns the worst status. */
int sw_ensemble_advance(sw_ensemble* e, int nsteps, int ggen);
int sw_ensemble_advance_async(sw_ensemble* e, int nsteps, int ggen);
int sw_ensemble_sync(sw_ensemble* e);
/* Number of kernels the library launched on this context so far. */
int sw_kernel_launches(sw_ctx* ctx, long long* count);

#ifdef __cplusplus
}
#endif
#endif
