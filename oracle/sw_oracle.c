/*
 * CPU oracle for the nhswps time-step path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C (FP64), the algorithm of the reference
 * rse-standrewscs/shallow-water (Rust) for the hot path of `nhswps`.  It is the
 * checker the CUDA path is compared with, and the CPU baseline that
 * bench.py times.  Nothing in the product (the shallow-water_b200 package and
 * its CUDA library) links, imports or calls this code.
 *
 * Parity of this oracle is pinned against the reference's own golden vectors
 * (the .npz files in tests/golden, packed from the reference's testdata by
 * tests/golden/make_golden.py) by tests/test_oracle.py.
 *
 * Layout conventions (reference src/utils.rs:6-32): every field is Fortran
 * order.  A physical plane is rvar(ny,nx) -> p[iy + ng*ix]; a spectral plane
 * is svar(nx,ny) -> s[kx + ng*ky]; a 3-D field adds + ng*ng*iz, iz = 0..nz.
 * The pressure Thomas factors htdv/etdv are stored here the same way
 * ([kx + ng*ky + ng*ng*iz], iz < nz); the reference keeps them C-ordered.
 *
 * The 1-D transforms restate stafft's *transform* (src/stafft/mod.rs:158-452):
 * m real DFTs of length n over x[i + m*j], output in Hermitian form
 * H[k] = Re F_k / sqrt(n) (0 <= k <= n/2), H[n-k] = Im F_k / sqrt(n), with F the
 * e^{-2 pi i jk/n} DFT, and revfft its exact inverse.  The butterflies are this
 * file's own (a mixed-radix 4/2/3/5 Stockham complex FFT over pairs of real
 * vectors), so results agree with the reference to rounding, not bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- constants (reference src/constants.rs:1-17) ---------------------- */
#define ORC_PI 3.14159265358979323846
static const double COF = 4.0 * ORC_PI;
static const double CGW = 2.0 * ORC_PI;
static const double HBAR = 0.4;
static const double CDAMP = 10.0;
static const double NNU = 3.0;
#define CSQ (CGW * CGW)
#define FSQ (COF * COF)
#define COFI (1.0 / COF)
#define GRAVITY (CSQ / HBAR)

enum { F_U, F_V, F_W, F_Z, F_ZX, F_ZY, F_R, F_RI, F_AA, F_ZETA, F_PN, F_DPN,
       F_PS, F_QS, F_DS, F_GS, F_NFIELDS };

enum { ORC_OK = 0, ORC_ERR_FACTORISE = 1, ORC_ERR_PSOLVE_DIVERGED = 3,
       ORC_ERR_PSOLVE_MAXITER = 4, ORC_ERR_ARG = 6 };

static void* xmalloc(size_t n) {
    void* p = malloc(n ? n : 1);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}
static double* dzeros(size_t n) {
    double* p = (double*)xmalloc(n * sizeof(double));
    memset(p, 0, n * sizeof(double));
    return p;
}

/* ======================================================================
 * stafft: factorisation and trig table (reference src/stafft/mod.rs:67-150)
 * ====================================================================== */

/* Greedy factorisation into 6,4,2,3,5 (src/stafft/mod.rs:97-150).
 * Returns 0 on success, ORC_ERR_FACTORISE when n has another prime factor. */
int orc_factorisen(int n, int factors[5]) {
    static const int fac[5] = {6, 4, 2, 3, 5};
    int rem = n;
    for (int i = 0; i < 5; i++) factors[i] = 0;
    if (n < 2) return ORC_ERR_FACTORISE;
    for (int i = 0; i < 5; i++) {
        while (rem % fac[i] == 0) {
            factors[i]++;
            rem /= fac[i];
            if (rem == 1) return ORC_OK;
        }
    }
    return ORC_ERR_FACTORISE;
}

/* Trig table (src/stafft/mod.rs:67-95): 2n values, cos in [0,n), -sin in [n,2n). */
int orc_initfft(int n, int factors[5], double* trig) {
    static const int fac[5] = {6, 4, 2, 3, 5};
    int st = orc_factorisen(n, factors);
    if (st) return st;
    for (int i = 0; i < 2 * n; i++) trig[i] = 0.0;
    double ftwopin = 2.0 * ORC_PI / (double)n;
    int rem = n, m = 1;
    for (int i = 0; i < 5; i++) {
        for (int e = 0; e < factors[i]; e++) {
            rem /= fac[i];
            for (int k = 1; k < fac[i]; k++)
                for (int l = 0; l < rem; l++) trig[(m++) - 1] = ftwopin * (double)(k * l);
            ftwopin *= (double)fac[i];
        }
    }
    for (int i = 1; i < n; i++) {
        trig[i + n - 1] = -sin(trig[i - 1]);
        trig[i - 1] = cos(trig[i - 1]);
    }
    return ORC_OK;
}

/* ======================================================================
 * Batched complex FFT (Stockham autosort, mixed radix 4/2/3/5).
 * Data are split re/im planes with the batch index innermost:
 * z[j*nb + b], j < n.  sign = -1 forward, +1 inverse (unnormalised).
 * ====================================================================== */
typedef struct {
    int n, nrad, rad[64];
    double *wr, *wi; /* cos/sin(2 pi t / n), t < n */
} cplan;

/* Radix schedule of the plans made from now on: 0 = radix 4, 2, 3, 5 in that
 * order (the default); 1 = radix 2 in place of 4 and the order reversed (5, 3, 2).
 * The second schedule rounds differently while computing the same transform: the
 * spread between oracle runs under the two schedules is the float64 rounding floor
 * against which GPU-vs-oracle differences are judged (test infrastructure only). */
static int g_fft_order = 0;
void orc_set_fft_order(int order) { g_fft_order = order; }
int orc_get_fft_order(void) { return g_fft_order; }

static int cplan_init(cplan* p, int n) {
    int rem = n;
    p->n = n;
    p->nrad = 0;
    p->wr = p->wi = NULL;
    if (n < 1) return ORC_ERR_ARG;
    if (g_fft_order == 0) {
        while (rem % 4 == 0) { p->rad[p->nrad++] = 4; rem /= 4; }
        while (rem % 2 == 0) { p->rad[p->nrad++] = 2; rem /= 2; }
        while (rem % 3 == 0) { p->rad[p->nrad++] = 3; rem /= 3; }
        while (rem % 5 == 0) { p->rad[p->nrad++] = 5; rem /= 5; }
    } else {
        while (rem % 5 == 0) { p->rad[p->nrad++] = 5; rem /= 5; }
        while (rem % 3 == 0) { p->rad[p->nrad++] = 3; rem /= 3; }
        while (rem % 2 == 0) { p->rad[p->nrad++] = 2; rem /= 2; }
    }
    if (rem != 1) return ORC_ERR_FACTORISE;
    p->wr = (double*)xmalloc(sizeof(double) * n);
    p->wi = (double*)xmalloc(sizeof(double) * n);
    for (int t = 0; t < n; t++) {
        double a = 2.0 * ORC_PI * (double)t / (double)n;
        p->wr[t] = cos(a);
        p->wi[t] = sin(a);
    }
    return ORC_OK;
}
static void cplan_free(cplan* p) {
    free(p->wr);
    free(p->wi);
    p->wr = p->wi = NULL;
}

/* One Stockham pass of radix R: reads x (natural sub-sequences of length Ns),
 * writes y with sub-transforms of length Ns*R. */
static void stockham_pass(const cplan* p, int R, int Ns, int nb, int sign,
                          const double* xr, const double* xi, double* yr, double* yi) {
    const int n = p->n, nR = n / R, tstride = n / (Ns * R);
    const double s3 = 0.86602540378443864676; /* sin(pi/3) */
    const double c51 = 0.30901699437494742410, c52 = -0.80901699437494742410; /* cos(2pi/5), cos(4pi/5) */
    const double s51 = 0.95105651629515357212, s52 = 0.58778525229247312917;  /* sin(2pi/5), sin(4pi/5) */
    for (int j = 0; j < nR; j++) {
        const int k = j % Ns;
        const int base = (j / Ns) * Ns * R + k;
        double twr[5] = {1, 1, 1, 1, 1}, twi[5] = {0, 0, 0, 0, 0};
        for (int r = 1; r < R; r++) {
            int idx = (int)(((long)r * k * tstride) % n);
            twr[r] = p->wr[idx];
            twi[r] = sign * p->wi[idx];
        }
        const double* ar[5];
        const double* ai[5];
        double* br[5];
        double* bi[5];
        for (int r = 0; r < R; r++) {
            ar[r] = xr + (size_t)(j + r * nR) * nb;
            ai[r] = xi + (size_t)(j + r * nR) * nb;
            br[r] = yr + (size_t)(base + r * Ns) * nb;
            bi[r] = yi + (size_t)(base + r * Ns) * nb;
        }
        for (int b = 0; b < nb; b++) {
            double vr[5], vi[5];
            vr[0] = ar[0][b];
            vi[0] = ai[0][b];
            for (int r = 1; r < R; r++) {
                double a = ar[r][b], c = ai[r][b];
                vr[r] = a * twr[r] - c * twi[r];
                vi[r] = a * twi[r] + c * twr[r];
            }
            if (R == 2) {
                br[0][b] = vr[0] + vr[1]; bi[0][b] = vi[0] + vi[1];
                br[1][b] = vr[0] - vr[1]; bi[1][b] = vi[0] - vi[1];
            } else if (R == 4) {
                double t0r = vr[0] + vr[2], t0i = vi[0] + vi[2];
                double t1r = vr[0] - vr[2], t1i = vi[0] - vi[2];
                double t2r = vr[1] + vr[3], t2i = vi[1] + vi[3];
                double t3r = vr[1] - vr[3], t3i = vi[1] - vi[3];
                /* w = sign*i ; w*(t3) = sign*(-t3i + i t3r) */
                double ur = -sign * t3i, ui = sign * t3r;
                br[0][b] = t0r + t2r; bi[0][b] = t0i + t2i;
                br[1][b] = t1r + ur;  bi[1][b] = t1i + ui;
                br[2][b] = t0r - t2r; bi[2][b] = t0i - t2i;
                br[3][b] = t1r - ur;  bi[3][b] = t1i - ui;
            } else if (R == 3) {
                double tr = vr[1] + vr[2], ti = vi[1] + vi[2];
                double mr = vr[0] - 0.5 * tr, mi = vi[0] - 0.5 * ti;
                double dr = sign * s3 * (vr[1] - vr[2]), di = sign * s3 * (vi[1] - vi[2]);
                br[0][b] = vr[0] + tr; bi[0][b] = vi[0] + ti;
                br[1][b] = mr - di;    bi[1][b] = mi + dr;
                br[2][b] = mr + di;    bi[2][b] = mi - dr;
            } else { /* R == 5 */
                double a1r = vr[1] + vr[4], a1i = vi[1] + vi[4];
                double b1r = vr[1] - vr[4], b1i = vi[1] - vi[4];
                double a2r = vr[2] + vr[3], a2i = vi[2] + vi[3];
                double b2r = vr[2] - vr[3], b2i = vi[2] - vi[3];
                double p1r = vr[0] + c51 * a1r + c52 * a2r, p1i = vi[0] + c51 * a1i + c52 * a2i;
                double p2r = vr[0] + c52 * a1r + c51 * a2r, p2i = vi[0] + c52 * a1i + c51 * a2i;
                double q1r = sign * (s51 * b1r + s52 * b2r), q1i = sign * (s51 * b1i + s52 * b2i);
                double q2r = sign * (s52 * b1r - s51 * b2r), q2i = sign * (s52 * b1i - s51 * b2i);
                br[0][b] = vr[0] + a1r + a2r; bi[0][b] = vi[0] + a1i + a2i;
                br[1][b] = p1r - q1i; bi[1][b] = p1i + q1r;
                br[4][b] = p1r + q1i; bi[4][b] = p1i - q1r;
                br[2][b] = p2r - q2i; bi[2][b] = p2i + q2r;
                br[3][b] = p2r + q2i; bi[3][b] = p2i - q2r;
            }
        }
    }
}

/* Full transform; returns 0 if result is in (xr,xi), 1 if in (yr,yi). */
static int cfft_batch(const cplan* p, int nb, int sign, double* xr, double* xi, double* yr, double* yi) {
    int Ns = 1, in_x = 1;
    for (int s = 0; s < p->nrad; s++) {
        int R = p->rad[s];
        if (in_x) stockham_pass(p, R, Ns, nb, sign, xr, xi, yr, yi);
        else      stockham_pass(p, R, Ns, nb, sign, yr, yi, xr, xi);
        in_x = !in_x;
        Ns *= R;
    }
    return in_x ? 0 : 1;
}

/* m real forward transforms of length n on x[i + m*j] (in place), using a
 * prepared plan.  Restates src/stafft/mod.rs:158-293 (the transform). */
static void forfft_plan(int m, int n, double* x, const cplan* p) {
    const int mp = (m + 1) / 2;
    double* buf = (double*)xmalloc(sizeof(double) * 4 * (size_t)n * mp);
    double *zr = buf, *zi = buf + (size_t)n * mp, *yr = zi + (size_t)n * mp, *yi = yr + (size_t)n * mp;
    for (int j = 0; j < n; j++)
        for (int q = 0; q < mp; q++) {
            zr[(size_t)j * mp + q] = x[2 * q + (size_t)m * j];
            zi[(size_t)j * mp + q] = (2 * q + 1 < m) ? x[2 * q + 1 + (size_t)m * j] : 0.0;
        }
    int w = cfft_batch(p, mp, -1, zr, zi, yr, yi);
    const double* Zr = w ? yr : zr;
    const double* Zi = w ? yi : zi;
    const double sc = 1.0 / sqrt((double)n);
    for (int k = 0; k <= n / 2; k++) {
        const int kk = (n - k) % n;
        const int has_sin = (k >= 1 && k <= (n - 1) / 2);
        for (int q = 0; q < mp; q++) {
            double ar = Zr[(size_t)k * mp + q], ai = Zi[(size_t)k * mp + q];
            double cr = Zr[(size_t)kk * mp + q], ci = Zi[(size_t)kk * mp + q];
            double Ar = 0.5 * (ar + cr), Ai = 0.5 * (ai - ci);
            double Br = 0.5 * (ai + ci), Bi = 0.5 * (cr - ar);
            x[2 * q + (size_t)m * k] = Ar * sc;
            if (has_sin) x[2 * q + (size_t)m * (n - k)] = Ai * sc;
            if (2 * q + 1 < m) {
                x[2 * q + 1 + (size_t)m * k] = Br * sc;
                if (has_sin) x[2 * q + 1 + (size_t)m * (n - k)] = Bi * sc;
            }
        }
    }
    free(buf);
}

/* Inverse of forfft_plan (restates src/stafft/mod.rs:301-452). */
static void revfft_plan(int m, int n, double* x, const cplan* p) {
    const int mp = (m + 1) / 2;
    double* buf = (double*)xmalloc(sizeof(double) * 4 * (size_t)n * mp);
    double *zr = buf, *zi = buf + (size_t)n * mp, *yr = zi + (size_t)n * mp, *yi = yr + (size_t)n * mp;
    for (int k = 0; k < n; k++) {
        for (int q = 0; q < mp; q++) {
            double Ar, Ai, Br = 0.0, Bi = 0.0;
            int ca = 2 * q, cb = 2 * q + 1;
            int hasb = cb < m;
            if (k == 0 || (n % 2 == 0 && k == n / 2)) {
                Ar = x[ca + (size_t)m * k]; Ai = 0.0;
                if (hasb) { Br = x[cb + (size_t)m * k]; Bi = 0.0; }
            } else if (k <= (n - 1) / 2) {
                Ar = x[ca + (size_t)m * k]; Ai = x[ca + (size_t)m * (n - k)];
                if (hasb) { Br = x[cb + (size_t)m * k]; Bi = x[cb + (size_t)m * (n - k)]; }
            } else {
                Ar = x[ca + (size_t)m * (n - k)]; Ai = -x[ca + (size_t)m * k];
                if (hasb) { Br = x[cb + (size_t)m * (n - k)]; Bi = -x[cb + (size_t)m * k]; }
            }
            zr[(size_t)k * mp + q] = Ar - Bi;
            zi[(size_t)k * mp + q] = Ai + Br;
        }
    }
    int w = cfft_batch(p, mp, +1, zr, zi, yr, yi);
    const double* Zr = w ? yr : zr;
    const double* Zi = w ? yi : zi;
    const double sc = 1.0 / sqrt((double)n);
    for (int j = 0; j < n; j++)
        for (int q = 0; q < mp; q++) {
            x[2 * q + (size_t)m * j] = Zr[(size_t)j * mp + q] * sc;
            if (2 * q + 1 < m) x[2 * q + 1 + (size_t)m * j] = Zi[(size_t)j * mp + q] * sc;
        }
    free(buf);
}

int orc_forfft(int m, int n, double* x) {
    cplan p;
    int st = cplan_init(&p, n);
    if (st) return st;
    forfft_plan(m, n, x, &p);
    cplan_free(&p);
    return ORC_OK;
}
int orc_revfft(int m, int n, double* x) {
    cplan p;
    int st = cplan_init(&p, n);
    if (st) return st;
    revfft_plan(m, n, x, &p);
    cplan_free(&p);
    return ORC_OK;
}

/* ======================================================================
 * sta2dfft (reference src/sta2dfft.rs:37-184), square ng x ng domain 2pi.
 * ====================================================================== */
typedef struct {
    int ng;
    cplan plan;
    double* hrk; /* hrkx == hrky: (pi/lx)*k, k = 1..ng (src/sta2dfft.rs:68-83) */
} d2fft;

static int d2_init(d2fft* d, int ng) {
    d->ng = ng;
    int st = cplan_init(&d->plan, ng);
    if (st) return st;
    d->hrk = dzeros(ng);
    const double sc = ORC_PI / (2.0 * ORC_PI);
    for (int k = 1; k <= ng; k++) d->hrk[k - 1] = sc * (double)k;
    return ORC_OK;
}
static void d2_free(d2fft* d) {
    cplan_free(&d->plan);
    free(d->hrk);
}

/* ptospc (src/sta2dfft.rs:91-107): rvar(ny,nx) physical -> svar(nx,ny) spectral. */
static void d2_ptospc(const d2fft* d, const double* rvar, double* svar) {
    const int ng = d->ng;
    double* w = (double*)xmalloc(sizeof(double) * ng * ng);
    memcpy(w, rvar, sizeof(double) * ng * ng);
    forfft_plan(ng, ng, w, &d->plan);
    for (int iy = 0; iy < ng; iy++)
        for (int kx = 0; kx < ng; kx++) svar[kx + ng * iy] = w[iy + ng * kx];
    forfft_plan(ng, ng, svar, &d->plan);
    free(w);
}
/* spctop (src/sta2dfft.rs:113-123): svar(nx,ny) spectral -> rvar(ny,nx) physical. */
static void d2_spctop(const d2fft* d, const double* svar, double* rvar) {
    const int ng = d->ng;
    double* w = (double*)xmalloc(sizeof(double) * ng * ng);
    memcpy(w, svar, sizeof(double) * ng * ng);
    revfft_plan(ng, ng, w, &d->plan);
    for (int kx = 0; kx < ng; kx++)
        for (int iy = 0; iy < ng; iy++) rvar[iy + ng * kx] = w[kx + ng * iy];
    revfft_plan(ng, ng, rvar, &d->plan);
    free(w);
}
/* xderiv (src/sta2dfft.rs:128-152) */
static void d2_xderiv(const d2fft* d, const double* var, double* der) {
    const int nx = d->ng, ny = d->ng, nwx = nx / 2, nxp2 = nx + 2;
    for (int ky = 0; ky < ny; ky++) {
        der[0 + nx * ky] = 0.0;
        for (int kx = 2; kx <= nx - nwx; kx++) {
            int dkx = 2 * (kx - 1), kxc = nxp2 - kx;
            der[(kx - 1) + nx * ky] = -d->hrk[dkx - 1] * var[(kxc - 1) + nx * ky];
            der[(kxc - 1) + nx * ky] = d->hrk[dkx - 1] * var[(kx - 1) + nx * ky];
        }
    }
    if (nx % 2 == 0)
        for (int ky = 0; ky < ny; ky++) der[nwx + nx * ky] = 0.0;
}
/* yderiv (src/sta2dfft.rs:157-184) */
static void d2_yderiv(const d2fft* d, const double* var, double* der) {
    const int nx = d->ng, ny = d->ng, nwy = ny / 2, nyp2 = ny + 2;
    for (int kx = 0; kx < nx; kx++) der[kx] = 0.0;
    for (int ky = 2; ky <= ny - nwy; ky++) {
        int kyc = nyp2 - ky;
        double fac = d->hrk[2 * (ky - 1) - 1];
        for (int kx = 0; kx < nx; kx++) {
            der[kx + nx * (ky - 1)] = -fac * var[kx + nx * (kyc - 1)];
            der[kx + nx * (kyc - 1)] = fac * var[kx + nx * (ky - 1)];
        }
    }
    if (ny % 2 == 0)
        for (int kx = 0; kx < nx; kx++) der[kx + nx * nwy] = 0.0;
}

/* ======================================================================
 * Spectral (reference src/spectral/mod.rs:17-299)
 * ====================================================================== */
typedef struct {
    int ng, nz;
    d2fft d2;
    double *hlap, *glap, *rlap, *helm, *c2g2, *simp, *rope, *fope, *filt, *diss, *opak, *rdis;
    double *etdv, *htdv, *ap; /* etdv/htdv: ng*ng*nz */
    double *etd1, *htd1, *theta, *weight, *rk, *spmf, *alk;
    int* kmag;
    int kmax, kmaxred;
} orc_spectral;

void orc_spectral_free(orc_spectral* s);

orc_spectral* orc_spectral_new(int ng, int nz) {
    if (ng < 4 || nz < 2) return NULL;
    orc_spectral* s = (orc_spectral*)xmalloc(sizeof(orc_spectral));
    memset(s, 0, sizeof(*s));
    s->ng = ng;
    s->nz = nz;
    if (d2_init(&s->d2, ng)) { free(s); return NULL; }
    const size_t n2 = (size_t)ng * ng;
    const double dt = 1.0 / (double)ng, dt2 = dt * (1.0 / 2.0), dt2i = 1.0 / dt2;
    const double dz = HBAR / (double)nz, dzi = 1.0 / dz, dzisq = pow(dzi, 2.0);
    s->hlap = dzeros(n2); s->glap = dzeros(n2); s->rlap = dzeros(n2); s->helm = dzeros(n2);
    s->c2g2 = dzeros(n2); s->simp = dzeros(n2); s->rope = dzeros(n2); s->fope = dzeros(n2);
    s->filt = dzeros(n2); s->diss = dzeros(n2); s->opak = dzeros(n2); s->rdis = dzeros(n2);
    s->etdv = dzeros(n2 * nz); s->htdv = dzeros(n2 * nz); s->ap = dzeros(n2);
    s->etd1 = dzeros(nz); s->htd1 = dzeros(nz);
    s->theta = dzeros(nz + 1); s->weight = dzeros(nz + 1);
    s->rk = dzeros(ng); s->spmf = dzeros(ng + 1); s->alk = dzeros(ng);
    s->kmag = (int*)xmalloc(sizeof(int) * n2);
    double* a0 = dzeros(n2);
    double* a0b = dzeros(n2);
    double* apb = dzeros(n2);
    const double* hrkx = s->d2.hrk;

    /* wavenumbers (src/spectral/mod.rs:116-121) */
    s->rk[0] = 0.0;
    for (int k = 1; k < ng / 2; k++) {
        s->rk[k] = hrkx[2 * k - 1];
        s->rk[ng - k] = hrkx[2 * k - 1];
    }
    s->rk[ng / 2] = hrkx[ng - 1];

    /* spectrum shells (src/spectral/mod.rs:124-146) */
    const double rkmax = (double)(ng / 2);
    s->kmax = (int)ceil(rkmax * sqrt(2.0));
    for (int k = 0; k <= s->kmax && k <= ng; k++) s->spmf[k] = 0.0;
    for (int ky = 0; ky < ng; ky++)
        for (int kx = 0; kx < ng; kx++) {
            int k = (int)round(sqrt(pow(s->rk[kx], 2.0) + pow(s->rk[ky], 2.0)));
            s->kmag[kx + ng * ky] = k;
            s->spmf[k] += 1.0;
        }
    const double snorm = 4.0 * ORC_PI / (double)(ng * ng);
    s->spmf[0] = 0.0;
    for (int k = 1; k <= s->kmax; k++) {
        s->spmf[k] = snorm * (double)k / s->spmf[k];
        s->alk[k - 1] = log10((double)k);
    }
    s->kmaxred = ng / 2;

    /* operators (src/spectral/mod.rs:148-204) */
    const double anu = CDAMP * COF / pow(rkmax, 2.0 * NNU);
    const double rkfsq = pow((double)ng / 3.0, 2.0);
    for (int ky = 0; ky < ng; ky++)
        for (int kx = 0; kx < ng; kx++) {
            const size_t i = kx + (size_t)ng * ky;
            double rks = pow(s->rk[kx], 2.0) + pow(s->rk[ky], 2.0);
            s->hlap[i] = -rks;
            s->opak[i] = -(FSQ + CSQ * rks);
            s->diss[i] = anu * pow(rks, NNU);
            if (rks > rkfsq) {
                s->filt[i] = 0.0; s->glap[i] = 0.0; s->c2g2[i] = 0.0; s->rlap[i] = 0.0;
                s->helm[i] = 0.0; s->rope[i] = 0.0; s->rdis[i] = 0.0;
            } else {
                s->filt[i] = 1.0;
                s->glap[i] = GRAVITY * rks;
                s->c2g2[i] = -CSQ * rks;
                s->rlap[i] = -1.0 / (rks + 1.0E-20);
                s->helm[i] = 1.0 / s->opak[i];
                s->rope[i] = s->c2g2[i] * s->helm[i];
                s->rdis[i] = dt2i + s->diss[i];
            }
            double rrsq = pow(dt2i + s->diss[i], 2.0);
            s->fope[i] = -s->c2g2[i] / (rrsq - s->opak[i]);
            s->simp[i] = 1.0 / (rrsq + FSQ);
            s->diss[i] = 2.0 / (1.0 + dt2 * s->diss[i]);
        }
    s->rlap[0] = 0.0;

    /* theta and trapezoid weights (src/spectral/mod.rs:206-214) */
    for (int iz = 0; iz <= nz; iz++) {
        s->theta[iz] = dz * (double)iz;
        s->weight[iz] = 1.0;
    }
    s->weight[0] = 0.5;
    s->weight[nz] = 0.5;
    for (int iz = 0; iz <= nz; iz++) s->weight[iz] /= (double)nz;

    /* pressure tridiagonal factors (src/spectral/mod.rs:216-256) */
    for (int ky = 0; ky < ng; ky++)
        for (int kx = 0; kx < ng; kx++) {
            const size_t i = kx + (size_t)ng * ky;
            double rks = pow(s->rk[kx], 2.0) + pow(s->rk[ky], 2.0);
            a0[i] = -2.0 * dzisq - (5.0 / 6.0) * rks;
            a0b[i] = -dzisq - (1.0 / 3.0) * rks;
            s->ap[i] = dzisq - (1.0 / 12.0) * rks;
            apb[i] = dzisq - (1.0 / 6.0) * rks;
        }
    for (size_t i = 0; i < n2; i++) {
        s->htdv[i] = s->filt[i] / a0b[i];
        s->etdv[i] = -apb[i] * s->htdv[i];
    }
    for (int iz = 1; iz <= nz - 2; iz++)
        for (size_t i = 0; i < n2; i++) {
            s->htdv[i + n2 * iz] = s->filt[i] / (a0[i] + s->ap[i] * s->etdv[i + n2 * (iz - 1)]);
            s->etdv[i + n2 * iz] = -s->ap[i] * s->htdv[i + n2 * iz];
        }
    for (size_t i = 0; i < n2; i++)
        s->htdv[i + n2 * (nz - 1)] = s->filt[i] / (a0[i] + s->ap[i] * s->etdv[i + n2 * (nz - 2)]);

    /* compact d/dtheta factors (src/spectral/mod.rs:258-265) */
    s->htd1[0] = 1.0 / (2.0 / 3.0);
    s->etd1[0] = -(1.0 / 6.0) * s->htd1[0];
    for (int iz = 2; iz < nz; iz++) {
        s->htd1[iz - 1] = 1.0 / ((2.0 / 3.0) + (1.0 / 6.0) * s->etd1[iz - 2]);
        s->etd1[iz - 1] = -(1.0 / 6.0) * s->htd1[iz - 1];
    }
    s->htd1[nz - 1] = 1.0 / ((2.0 / 3.0) + (1.0 / 3.0) * s->etd1[nz - 2]);
    free(a0); free(a0b); free(apb);
    return s;
}

void orc_spectral_free(orc_spectral* s) {
    if (!s) return;
    d2_free(&s->d2);
    double* ps[] = {s->hlap, s->glap, s->rlap, s->helm, s->c2g2, s->simp, s->rope, s->fope, s->filt,
                    s->diss, s->opak, s->rdis, s->etdv, s->htdv, s->ap, s->etd1, s->htd1, s->theta,
                    s->weight, s->rk, s->spmf, s->alk};
    for (size_t i = 0; i < sizeof(ps) / sizeof(ps[0]); i++) free(ps[i]);
    free(s->kmag);
    free(s);
}

/* Copy one named operator out (for golden tests).  Returns element count or -1. */
long orc_spectral_get(const orc_spectral* s, const char* name, double* out) {
    const size_t n2 = (size_t)s->ng * s->ng;
    struct { const char* nm; const double* p; size_t n; } t[] = {
        {"hlap", s->hlap, n2}, {"glap", s->glap, n2}, {"rlap", s->rlap, n2}, {"helm", s->helm, n2},
        {"c2g2", s->c2g2, n2}, {"simp", s->simp, n2}, {"rope", s->rope, n2}, {"fope", s->fope, n2},
        {"filt", s->filt, n2}, {"diss", s->diss, n2}, {"opak", s->opak, n2}, {"rdis", s->rdis, n2},
        {"etdv", s->etdv, n2 * s->nz}, {"htdv", s->htdv, n2 * s->nz}, {"ap", s->ap, n2},
        {"etd1", s->etd1, (size_t)s->nz}, {"htd1", s->htd1, (size_t)s->nz},
        {"theta", s->theta, (size_t)s->nz + 1}, {"weight", s->weight, (size_t)s->nz + 1},
        {"hrkx", s->d2.hrk, (size_t)s->ng}, {"hrky", s->d2.hrk, (size_t)s->ng}, {"rk", s->rk, (size_t)s->ng},
        {"spmf", s->spmf, (size_t)s->ng + 1}, {"alk", s->alk, (size_t)s->ng}};
    for (size_t i = 0; i < sizeof(t) / sizeof(t[0]); i++)
        if (!strcmp(t[i].nm, name)) {
            if (out) memcpy(out, t[i].p, sizeof(double) * t[i].n);
            return (long)t[i].n;
        }
    if (!strcmp(name, "kmag")) {
        if (out) for (size_t i = 0; i < n2; i++) out[i] = (double)s->kmag[i];
        return (long)n2;
    }
    if (!strcmp(name, "kmax")) { if (out) out[0] = s->kmax; return 1; }
    if (!strcmp(name, "kmaxred")) { if (out) out[0] = s->kmaxred; return 1; }
    return -1;
}

/* 2-D entry points for tests */
void orc_ptospc(const orc_spectral* s, const double* rvar, double* svar) { d2_ptospc(&s->d2, rvar, svar); }
void orc_spctop(const orc_spectral* s, const double* svar, double* rvar) { d2_spctop(&s->d2, svar, rvar); }
void orc_xderiv(const orc_spectral* s, const double* var, double* der) { d2_xderiv(&s->d2, var, der); }
void orc_yderiv(const orc_spectral* s, const double* var, double* der) { d2_yderiv(&s->d2, var, der); }

#define PL(f, iz) ((f) + (size_t)ng * ng * (iz))

/* main_invert (src/spectral/mod.rs:305-417) */
void orc_main_invert(const orc_spectral* s, const double* qs, const double* ds, const double* gs,
                     double* r, double* u, double* v, double* zeta) {
    const int ng = s->ng, nz = s->nz;
    const size_t n2 = (size_t)ng * ng, n3 = n2 * (nz + 1);
    const double dsumi = 1.0 / (double)(ng * ng);
    double* es = dzeros(n3);
    double* wkh = dzeros(n2);
    double* uio_l = dzeros(nz + 1);
    double* vio_l = dzeros(nz + 1);
    for (size_t i = 0; i < n3; i++) es[i] = COFI * (COFI * gs[i] - qs[i]);
    for (int iz = 0; iz <= nz; iz++)
        for (size_t i = 0; i < n2; i++) wkh[i] += s->weight[iz] * PL(es, iz)[i];
    for (size_t i = 0; i < n2; i++) wkh[i] *= s->rope[i];
#pragma omp parallel for schedule(dynamic, 1)
    for (int iz = 0; iz <= nz; iz++) {
        double* wka = dzeros(n2); double* wkb = dzeros(n2); double* wkc = dzeros(n2);
        double* wkd = dzeros(n2); double* wke = dzeros(n2); double* wkf = dzeros(n2);
        double* wkg = dzeros(n2);
        for (size_t i = 0; i < n2; i++) {
            wka[i] = PL(es, iz)[i] - wkh[i];
            wkb[i] = PL(qs, iz)[i] + COF * wka[i];
            wkc[i] = s->rlap[i] * wkb[i];
            wkd[i] = s->rlap[i] * PL(ds, iz)[i];
        }
        d2_xderiv(&s->d2, wkd, wke);
        d2_yderiv(&s->d2, wkd, wkf);
        d2_xderiv(&s->d2, wkc, wkd);
        d2_yderiv(&s->d2, wkc, wkg);
        for (size_t i = 0; i < n2; i++) { wke[i] -= wkg[i]; wkf[i] += wkd[i]; }
        d2_spctop(&s->d2, wka, PL(r, iz));
        d2_spctop(&s->d2, wkb, PL(zeta, iz));
        d2_spctop(&s->d2, wke, PL(u, iz));
        d2_spctop(&s->d2, wkf, PL(v, iz));
        double su = 0.0, sv = 0.0;
        for (size_t i = 0; i < n2; i++) {
            su += PL(u, iz)[i] * PL(r, iz)[i];
            sv += PL(v, iz)[i] * PL(r, iz)[i];
        }
        uio_l[iz] = s->weight[iz] * su * dsumi;
        vio_l[iz] = s->weight[iz] * sv * dsumi;
        free(wka); free(wkb); free(wkc); free(wkd); free(wke); free(wkf); free(wkg);
    }
    double uio = 0.0, vio = 0.0;
    for (int iz = 0; iz <= nz; iz++) { uio -= uio_l[iz]; vio -= vio_l[iz]; }
    for (size_t i = 0; i < n3; i++) { u[i] += uio; v[i] += vio; }
    free(es); free(wkh); free(uio_l); free(vio_l);
}

/* jacob (src/spectral/mod.rs:423-453): aa, bb physical -> cs spectral */
void orc_jacob(const orc_spectral* s, const double* aa, const double* bb, double* cs) {
    const int ng = s->ng;
    const size_t n2 = (size_t)ng * ng;
    double* ax = dzeros(n2); double* ay = dzeros(n2); double* bx = dzeros(n2); double* by = dzeros(n2);
    double* wka = dzeros(n2); double* wkb = dzeros(n2);
    d2_ptospc(&s->d2, aa, wka);
    d2_xderiv(&s->d2, wka, wkb); d2_spctop(&s->d2, wkb, ax);
    d2_yderiv(&s->d2, wka, wkb); d2_spctop(&s->d2, wkb, ay);
    d2_ptospc(&s->d2, bb, wka);
    d2_xderiv(&s->d2, wka, wkb); d2_spctop(&s->d2, wkb, bx);
    d2_yderiv(&s->d2, wka, wkb); d2_spctop(&s->d2, wkb, by);
    for (size_t i = 0; i < n2; i++) wkb[i] = ax[i] * by[i] - ay[i] * bx[i];
    d2_ptospc(&s->d2, wkb, cs);
    free(ax); free(ay); free(bx); free(by); free(wka); free(wkb);
}

/* divs (src/spectral/mod.rs:457-475): aa, bb physical -> cs spectral */
void orc_divs(const orc_spectral* s, const double* aa, const double* bb, double* cs) {
    const size_t n2 = (size_t)s->ng * s->ng;
    double* wka = dzeros(n2); double* wkb = dzeros(n2);
    d2_ptospc(&s->d2, aa, wka);
    d2_xderiv(&s->d2, wka, wkb);
    d2_ptospc(&s->d2, bb, wka);
    d2_yderiv(&s->d2, wka, cs);
    for (size_t i = 0; i < n2; i++) cs[i] += wkb[i];
    free(wka); free(wkb);
}

/* ptospc3d / spctop3d (src/spectral/mod.rs:479-522) */
void orc_ptospc3d(const orc_spectral* s, const double* fp, double* fs, int izbeg, int izend) {
    const int ng = s->ng;
#pragma omp parallel for schedule(dynamic, 1)
    for (int iz = izbeg; iz <= izend; iz++) d2_ptospc(&s->d2, PL(fp, iz), PL(fs, iz));
}
void orc_spctop3d(const orc_spectral* s, const double* fs, double* fp, int izbeg, int izend) {
    const int ng = s->ng;
#pragma omp parallel for schedule(dynamic, 1)
    for (int iz = izbeg; iz <= izend; iz++) d2_spctop(&s->d2, PL(fs, iz), PL(fp, iz));
}

static void deal2d_plane(const orc_spectral* s, double* fp) {
    const size_t n2 = (size_t)s->ng * s->ng;
    double* fs = dzeros(n2);
    d2_ptospc(&s->d2, fp, fs);
    for (size_t i = 0; i < n2; i++) fs[i] *= s->filt[i];
    d2_spctop(&s->d2, fs, fp);
    free(fs);
}
/* deal3d / deal2d (src/spectral/mod.rs:526-554) */
void orc_deal3d(const orc_spectral* s, double* fp) {
    const int ng = s->ng;
#pragma omp parallel for schedule(dynamic, 1)
    for (int iz = 0; iz <= s->nz; iz++) deal2d_plane(s, PL(fp, iz));
}
void orc_deal2d(const orc_spectral* s, double* fp) { deal2d_plane(s, fp); }

/* spec1d (src/spectral/mod.rs:558-591) */
void orc_spec1d(const orc_spectral* s, const double* ss, double* spec) {
    const int ng = s->ng;
    for (int k = 0; k <= s->kmax; k++) spec[k] = 0.0;
    spec[s->kmag[0]] += (1.0 / 4.0) * pow(ss[0], 2.0);
    for (int kx = 1; kx < ng; kx++) spec[s->kmag[kx]] += (1.0 / 2.0) * pow(ss[kx], 2.0);
    for (int ky = 1; ky < ng; ky++) spec[s->kmag[ng * ky]] += (1.0 / 2.0) * pow(ss[ng * ky], 2.0);
    for (int ky = 1; ky < ng; ky++)
        for (int kx = 1; kx < ng; kx++) spec[s->kmag[kx + ng * ky]] += pow(ss[kx + ng * ky], 2.0);
}

/* ======================================================================
 * nhswps numerics (reference src/nhswps/).  Fields are passed as an
 * array of F_NFIELDS pointers in the F_* order above.
 * ====================================================================== */

/* vertical (src/nhswps/vertical.rs:8-143) */
void orc_vertical(const orc_spectral* s, double** f) {
    const int ng = s->ng, nz = s->nz;
    const size_t n2 = (size_t)ng * ng;
    const double dz2 = (HBAR / (double)nz) / 2.0;
    double *z = f[F_Z], *r = f[F_R], *u = f[F_U], *v = f[F_V], *w = f[F_W];
    double* rsrc = dzeros(n2 * (nz + 1));
    for (size_t i = 0; i < n2; i++) PL(z, 1)[i] = dz2 * (PL(r, 0)[i] + PL(r, 1)[i]);
    for (int iz = 1; iz < nz; iz++)
        for (size_t i = 0; i < n2; i++)
            PL(z, iz + 1)[i] = PL(z, iz)[i] + dz2 * (PL(r, iz)[i] + PL(r, iz + 1)[i]);
#pragma omp parallel for schedule(dynamic, 1)
    for (int iz = 1; iz <= nz; iz++) {
        double* wka = dzeros(n2); double* wkb = dzeros(n2);
        const double th = s->theta[iz];
        for (size_t i = 0; i < n2; i++) PL(z, iz)[i] += th;
        d2_ptospc(&s->d2, PL(z, iz), wka);
        d2_xderiv(&s->d2, wka, wkb);
        d2_spctop(&s->d2, wkb, PL(f[F_ZX], iz));
        d2_yderiv(&s->d2, wka, wkb);
        d2_spctop(&s->d2, wkb, PL(f[F_ZY], iz));
        free(wka); free(wkb);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int iz = 0; iz <= nz; iz++) {
        double* wkq = dzeros(n2); double* wka = dzeros(n2); double* wkb = dzeros(n2); double* wkc = dzeros(n2);
        for (size_t i = 0; i < n2; i++) wkq[i] = PL(u, iz)[i] * PL(r, iz)[i];
        d2_ptospc(&s->d2, wkq, wka);
        d2_xderiv(&s->d2, wka, wkb);
        for (size_t i = 0; i < n2; i++) wkq[i] = PL(v, iz)[i] * PL(r, iz)[i];
        d2_ptospc(&s->d2, wkq, wka);
        d2_yderiv(&s->d2, wka, wkc);
        for (size_t i = 0; i < n2; i++) {
            PL(f[F_AA], iz)[i] = s->filt[i] * (wkb[i] + wkc[i]);
            wka[i] = PL(f[F_AA], iz)[i] + PL(f[F_DS], iz)[i];
        }
        d2_spctop(&s->d2, wka, wkq);
        for (size_t i = 0; i < n2; i++) PL(rsrc, iz)[i] = -wkq[i];
        free(wkq); free(wka); free(wkb); free(wkc);
    }
    for (size_t i = 0; i < n2; i++) PL(w, 1)[i] = dz2 * (PL(rsrc, 0)[i] + PL(rsrc, 1)[i]);
    for (int iz = 1; iz < nz; iz++)
        for (size_t i = 0; i < n2; i++)
            PL(w, iz + 1)[i] = PL(w, iz)[i] + dz2 * (PL(rsrc, iz)[i] + PL(rsrc, iz + 1)[i]);
#pragma omp parallel for schedule(dynamic, 1)
    for (int iz = 1; iz <= nz; iz++) {
        double* wkq = dzeros(n2);
        for (size_t i = 0; i < n2; i++)
            wkq[i] = PL(u, iz)[i] * PL(f[F_ZX], iz)[i] + PL(v, iz)[i] * PL(f[F_ZY], iz)[i];
        deal2d_plane(s, wkq);
        for (size_t i = 0; i < n2; i++) PL(w, iz)[i] += wkq[i];
        free(wkq);
    }
    free(rsrc);
}

/* coeffs (src/nhswps/coeffs.rs:8-101) */
void orc_coeffs(const orc_spectral* s, double* const* f, double* sigx, double* sigy, double* cpt1,
                double* cpt2) {
    const int ng = s->ng, nz = s->nz;
    const size_t n2 = (size_t)ng * ng, n3 = n2 * (nz + 1);
    const double qdzi = (1.0 / 4.0) * (1.0 / (HBAR / (double)nz));
    const double *ri = f[F_RI], *zx = f[F_ZX], *zy = f[F_ZY];
    for (size_t i = 0; i < n3; i++) { sigx[i] = ri[i] * zx[i]; sigy[i] = ri[i] * zy[i]; }
    orc_deal3d(s, sigx);
    orc_deal3d(s, sigy);
    for (size_t i = 0; i < n3; i++)
        cpt2[i] = 1.0 - pow(ri[i], 2.0) - pow(sigx[i], 2.0) - pow(sigy[i], 2.0);
    orc_deal3d(s, cpt2);
#pragma omp parallel for schedule(dynamic, 1)
    for (int iz = 0; iz <= nz; iz++) {
        if (iz == 0) {
            for (size_t i = 0; i < n2; i++)
                cpt1[i] = qdzi * (4.0 * PL(cpt2, 1)[i] - 3.0 * PL(cpt2, 0)[i] - PL(cpt2, 2)[i]);
            continue;
        }
        double* wka = dzeros(n2); double* wkp = dzeros(n2);
        orc_divs(s, PL(sigx, iz), PL(sigy, iz), wka);
        d2_spctop(&s->d2, wka, wkp);
        if (iz < nz) {
            for (size_t i = 0; i < n2; i++)
                PL(cpt1, iz)[i] = qdzi * (PL(cpt2, iz + 1)[i] - PL(cpt2, iz - 1)[i]) + wkp[i];
        } else {
            for (size_t i = 0; i < n2; i++)
                PL(cpt1, nz)[i] = qdzi * (3.0 * PL(cpt2, nz)[i] + PL(cpt2, nz - 2)[i] - 4.0 * PL(cpt2, nz - 1)[i]) + wkp[i];
        }
        free(wka); free(wkp);
    }
    for (size_t i = 0; i < n3; i++) { sigx[i] *= 2.0; sigy[i] *= 2.0; }
}

/* cpsource (src/nhswps/cpsource.rs:13-261) */
void orc_cpsource(const orc_spectral* s, double* const* f, double* sp0) {
    const int ng = s->ng, nz = s->nz;
    const size_t n2 = (size_t)ng * ng, n3 = n2 * (nz + 1);
    const double hdzi = (1.0 / 2.0) * (1.0 / (HBAR / (double)nz));
    const double *u = f[F_U], *v = f[F_V], *w = f[F_W];
    double* ut = dzeros(n3); double* vt = dzeros(n3); double* wt = dzeros(n3);
    double* hsrc = dzeros(n2); double* wka0 = dzeros(n2);
    d2_ptospc(&s->d2, PL(f[F_Z], nz), wka0);
    for (size_t i = 0; i < n2; i++) wka0[i] *= s->glap[i];
    d2_spctop(&s->d2, wka0, hsrc);
    for (int iz = 0; iz <= nz; iz++) {
        const double* X[3] = {u, v, w};
        double* T[3] = {ut, vt, wt};
        for (int c = 0; c < 3; c++)
            for (size_t i = 0; i < n2; i++) {
                double val;
                if (iz == 0)
                    val = hdzi * (4.0 * PL(X[c], 1)[i] - 3.0 * PL(X[c], 0)[i] - PL(X[c], 2)[i]);
                else if (iz == nz)
                    val = hdzi * (3.0 * PL(X[c], nz)[i] + PL(X[c], nz - 2)[i] - 4.0 * PL(X[c], nz - 1)[i]);
                else
                    val = hdzi * (PL(X[c], iz + 1)[i] - PL(X[c], iz - 1)[i]);
                PL(T[c], iz)[i] = val;
            }
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int iz = 0; iz <= nz; iz++) {
        double* wka = dzeros(n2); double* wkb = dzeros(n2); double* wkp = dzeros(n2);
        double* wkq = dzeros(n2); double* wkr = dzeros(n2);
        double* ux = dzeros(n2); double* uy = dzeros(n2); double* vx = dzeros(n2); double* vy = dzeros(n2);
        double* wx = dzeros(n2); double* wy = dzeros(n2);
        const double *ri = PL(f[F_RI], iz), *zeta = PL(f[F_ZETA], iz);
        const double *zx = PL(f[F_ZX], iz), *zy = PL(f[F_ZY], iz);
        const double *utz = PL(ut, iz), *vtz = PL(vt, iz), *wtz = PL(wt, iz);
        double* out = PL(sp0, iz);
        d2_ptospc(&s->d2, PL(u, iz), wka);
        d2_xderiv(&s->d2, wka, wkb); d2_spctop(&s->d2, wkb, ux);
        d2_yderiv(&s->d2, wka, wkb); d2_spctop(&s->d2, wkb, uy);
        d2_ptospc(&s->d2, PL(v, iz), wka);
        d2_xderiv(&s->d2, wka, wkb); d2_spctop(&s->d2, wkb, vx);
        d2_yderiv(&s->d2, wka, wkb); d2_spctop(&s->d2, wkb, vy);
        if (iz == 0) {
            for (size_t i = 0; i < n2; i++) wkq[i] = ri[i] * wtz[i];
            deal2d_plane(s, wkq);
            for (size_t i = 0; i < n2; i++) {
                out[i] = hsrc[i] + COF * zeta[i];
                out[i] += 2.0 * (ux[i] * vy[i] - uy[i] * vx[i] + wkq[i] * (ux[i] + vy[i]));
            }
        } else {
            d2_ptospc(&s->d2, PL(w, iz), wka);
            d2_xderiv(&s->d2, wka, wkb); d2_spctop(&s->d2, wkb, wx);
            d2_yderiv(&s->d2, wka, wkb); d2_spctop(&s->d2, wkb, wy);
            for (size_t i = 0; i < n2; i++) wkp[i] = vtz[i] * zx[i] - utz[i] * zy[i];
            deal2d_plane(s, wkp);
            for (size_t i = 0; i < n2; i++) wkq[i] = uy[i] * vtz[i] - utz[i] * vy[i];
            deal2d_plane(s, wkq);
            for (size_t i = 0; i < n2; i++) wkr[i] = utz[i] * vx[i] - ux[i] * vtz[i];
            deal2d_plane(s, wkr);
            for (size_t i = 0; i < n2; i++) {
                wkq[i] = wkq[i] * zx[i] + wkr[i] * zy[i] - wy[i] * vtz[i];
                wkq[i] += (ux[i] + vy[i]) * wtz[i] - wx[i] * utz[i];
            }
            deal2d_plane(s, wkq);
            for (size_t i = 0; i < n2; i++) {
                out[i] = hsrc[i] + COF * (zeta[i] - ri[i] * wkp[i]) + 2.0 * (ri[i] * wkq[i]);
                out[i] += 2.0 * (ux[i] * vy[i] - uy[i] * vx[i]);
            }
        }
        free(wka); free(wkb); free(wkp); free(wkq); free(wkr);
        free(ux); free(uy); free(vx); free(vy); free(wx); free(wy);
    }
    free(ut); free(vt); free(wt); free(hsrc); free(wka0);
}

/* psolve (src/nhswps/psolve.rs:16-411).  Returns ORC_OK, or
 * ORC_ERR_PSOLVE_DIVERGED (errp > 1 after the first sweep, psolve.rs:349-352) or
 * ORC_ERR_PSOLVE_MAXITER (psolve.rs:360-366) where the reference quits.
 * nitmax <= 0 means the reference's 100. */
int orc_psolve_ex(const orc_spectral* s, double** f, int nitmax, int* iters_out, double* errp_out) {
    const int ng = s->ng, nz = s->nz;
    const size_t n2 = (size_t)ng * ng, n3 = n2 * (nz + 1);
    const double toler = 1.0E-9;
    const double dz = HBAR / (double)nz, dzi = 1.0 / dz, dz2 = dz / 2.0, dz6 = dz / 6.0;
    const double dzisq = pow(1.0 / dz, 2.0);
    const double hdzi = (1.0 / 2.0) * (1.0 / (HBAR / (double)nz));
    if (nitmax <= 0) nitmax = 100;
    if (nz < 3) return ORC_ERR_ARG;
    double *ri = f[F_RI], *r = f[F_R], *ps = f[F_PS], *pn = f[F_PN];
    double* sp0 = dzeros(n3); double* sigx = dzeros(n3); double* sigy = dzeros(n3);
    double* cpt1 = dzeros(n3); double* cpt2 = dzeros(n3);
    double* sp = dzeros(n3); double* gg = dzeros(n3);
    double* dpdt = dzeros(n2); double* d2pdt2 = dzeros(n2); double* wkq = dzeros(n2);
    double* pna = (double*)xmalloc(sizeof(double) * n3);

    for (size_t i = 0; i < n3; i++) ri[i] = 1.0 / (r[i] + 1.0);
    orc_deal3d(s, ri);
    orc_vertical(s, f);
    orc_coeffs(s, f, sigx, sigy, cpt1, cpt2);
    orc_cpsource(s, f, sp0);
    memcpy(pna, pn, sizeof(double) * n3);

    double errp = 1.0;
    int iter = 0, status = ORC_OK;
    while (errp > toler && iter < nitmax) {
        orc_ptospc3d(s, pn, ps, 0, nz - 1);
        memset(PL(ps, nz), 0, sizeof(double) * n2);
        /* lower boundary iz = 0 */
        {
            double* wkd = dzeros(n2); double* wkp = dzeros(n2);
            for (size_t i = 0; i < n2; i++)
                wkd[i] = (2.0 * PL(ps, 0)[i] - 5.0 * PL(ps, 1)[i] + 4.0 * PL(ps, 2)[i] - PL(ps, 3)[i]) * dzisq;
            d2_spctop(&s->d2, wkd, d2pdt2);
            for (size_t i = 0; i < n2; i++) wkp[i] = PL(sp0, 0)[i] + PL(cpt2, 0)[i] * d2pdt2[i];
            d2_ptospc(&s->d2, wkp, PL(sp, 0));
            free(wkd); free(wkp);
        }
        /* interior 1..nz-1 */
#pragma omp parallel for schedule(dynamic, 1)
        for (int iz = 1; iz <= nz - 1; iz++) {
            double* wka = dzeros(n2); double* wkb = dzeros(n2); double* wkc = dzeros(n2);
            double* wkd = dzeros(n2); double* wkp = dzeros(n2);
            double* d2pdxt = dzeros(n2); double* d2pdyt = dzeros(n2);
            double* dpdt_l = dzeros(n2); double* d2pdt2_l = dzeros(n2);
            for (size_t i = 0; i < n2; i++) {
                wka[i] = (PL(ps, iz + 1)[i] - PL(ps, iz - 1)[i]) * hdzi;
                wkd[i] = (PL(ps, iz + 1)[i] - 2.0 * PL(ps, iz)[i] + PL(ps, iz - 1)[i]) * dzisq;
            }
            d2_xderiv(&s->d2, wka, wkb);
            d2_yderiv(&s->d2, wka, wkc);
            d2_spctop(&s->d2, wkb, d2pdxt);
            d2_spctop(&s->d2, wkc, d2pdyt);
            for (size_t i = 0; i < n2; i++)
                wkp[i] = PL(sp0, iz)[i] + PL(sigx, iz)[i] * d2pdxt[i] + PL(sigy, iz)[i] * d2pdyt[i];
            d2_spctop(&s->d2, wka, dpdt_l);
            d2_spctop(&s->d2, wkd, d2pdt2_l);
            if (iz == nz - 1) {
                memcpy(dpdt, dpdt_l, sizeof(double) * n2);
                memcpy(d2pdt2, d2pdt2_l, sizeof(double) * n2);
            }
            if (iz == nz - 2) memcpy(wkq, d2pdt2_l, sizeof(double) * n2);
            for (size_t i = 0; i < n2; i++)
                wkp[i] += PL(cpt2, iz)[i] * d2pdt2_l[i] + PL(cpt1, iz)[i] * dpdt_l[i];
            d2_ptospc(&s->d2, wkp, PL(sp, iz));
            free(wka); free(wkb); free(wkc); free(wkd); free(wkp);
            free(d2pdxt); free(d2pdyt); free(dpdt_l); free(d2pdt2_l);
        }
        /* upper boundary iz = nz (extrapolated derivatives) */
        {
            double* wka = dzeros(n2); double* wkb = dzeros(n2); double* wkc = dzeros(n2);
            double* wkp = dzeros(n2); double* d2pdxt = dzeros(n2); double* d2pdyt = dzeros(n2);
            for (size_t i = 0; i < n2; i++) {
                dpdt[i] += dz2 * (3.0 * d2pdt2[i] - wkq[i]);
                d2pdt2[i] = 2.0 * d2pdt2[i] - wkq[i];
            }
            d2_ptospc(&s->d2, dpdt, wka);
            d2_xderiv(&s->d2, wka, wkb);
            d2_yderiv(&s->d2, wka, wkc);
            d2_spctop(&s->d2, wkb, d2pdxt);
            d2_spctop(&s->d2, wkc, d2pdyt);
            for (size_t i = 0; i < n2; i++) {
                wkp[i] = PL(sp0, nz)[i] + PL(sigx, nz)[i] * d2pdxt[i] + PL(sigy, nz)[i] * d2pdyt[i];
                wkp[i] += PL(cpt2, nz)[i] * d2pdt2[i] + PL(cpt1, nz)[i] * dpdt[i];
            }
            d2_ptospc(&s->d2, wkp, PL(sp, nz));
            free(wka); free(wkb); free(wkc); free(wkp); free(d2pdxt); free(d2pdyt);
        }
        /* compact RHS and Thomas solve per (kx,ky) (psolve.rs:285-329) */
        for (size_t i = 0; i < n2; i++) {
            PL(gg, 0)[i] = (1.0 / 3.0) * PL(sp, 0)[i] + (1.0 / 6.0) * PL(sp, 1)[i];
            for (int iz = 1; iz < nz; iz++)
                PL(gg, iz)[i] = (1.0 / 12.0) * (PL(sp, iz - 1)[i] + PL(sp, iz + 1)[i]) + (5.0 / 6.0) * PL(sp, iz)[i];
            PL(ps, 0)[i] = PL(gg, 0)[i] * s->htdv[i];
            for (int iz = 1; iz < nz; iz++)
                PL(ps, iz)[i] = (PL(gg, iz)[i] - s->ap[i] * PL(ps, iz - 1)[i]) * s->htdv[i + n2 * iz];
            for (int iz = nz - 2; iz >= 0; iz--) PL(ps, iz)[i] += s->etdv[i + n2 * iz] * PL(ps, iz + 1)[i];
            PL(ps, nz)[i] = 0.0;
        }
        orc_spctop3d(s, ps, pn, 0, nz - 1);
        memset(PL(pn, nz), 0, sizeof(double) * n2);
        double num = 0.0, den = 0.0;
        for (size_t i = 0; i < n3; i++) {
            num += pow(pn[i] - pna[i], 2.0);
            den += pow(pna[i], 2.0);
        }
        errp = sqrt(num / (den + 1.0E-20));
        if (iter > 0 && errp > 1.0) { status = ORC_ERR_PSOLVE_DIVERGED; iter++; break; }
        iter++;
        memcpy(pna, pn, sizeof(double) * n3);
    }
    /* the reference quits whenever the sweep count reached nitmax (psolve.rs:360-366) */
    if (status == ORC_OK && iter >= nitmax) status = ORC_ERR_PSOLVE_MAXITER;
    if (iters_out) *iters_out = iter;
    if (errp_out) *errp_out = errp;
    if (status == ORC_OK) {
        /* dp/dtheta by 4th-order compact differences (psolve.rs:371-410);
         * level 0 of gg keeps the last sweep's compact RHS and dpn(0) is not written. */
        for (int iz = 1; iz < nz; iz++)
            for (size_t i = 0; i < n2; i++) PL(gg, iz)[i] = (PL(ps, iz + 1)[i] - PL(ps, iz - 1)[i]) * hdzi;
        for (size_t i = 0; i < n2; i++) {
            PL(gg, nz)[i] = dz6 * PL(sp, nz)[i] - PL(ps, nz - 1)[i] * dzi;
            PL(gg, 1)[i] *= s->htd1[0];
            for (int iz = 2; iz < nz; iz++)
                PL(gg, iz)[i] = (PL(gg, iz)[i] - (1.0 / 6.0) * PL(gg, iz - 1)[i]) * s->htd1[iz - 1];
            PL(gg, nz)[i] = (PL(gg, nz)[i] - (1.0 / 3.0) * PL(gg, nz - 1)[i]) * s->htd1[nz - 1];
            for (int iz = nz - 1; iz >= 1; iz--) PL(gg, iz)[i] += s->etd1[iz - 1] * PL(gg, iz + 1)[i];
        }
        orc_spctop3d(s, gg, f[F_DPN], 1, nz);
    }
    free(sp0); free(sigx); free(sigy); free(cpt1); free(cpt2); free(sp); free(gg);
    free(dpdt); free(d2pdt2); free(wkq); free(pna);
    return status;
}
int orc_psolve(const orc_spectral* s, double** f, int* iters_out, double* errp_out) {
    return orc_psolve_ex(s, f, 100, iters_out, errp_out);
}

/* source (src/nhswps/source.rs:19-138) */
void orc_source(const orc_spectral* s, double* const* f, double* sqs, double* sds, double* sgs) {
    const int ng = s->ng, nz = s->nz;
    const size_t n2 = (size_t)ng * ng;
    double* wkd = dzeros(n2);
    for (int iz = 0; iz <= nz; iz++)
        for (size_t i = 0; i < n2; i++) wkd[i] += s->weight[iz] * PL(f[F_AA], iz)[i];
    for (size_t i = 0; i < n2; i++) wkd[i] *= s->c2g2[i];
#pragma omp parallel for schedule(dynamic, 1)
    for (int iz = 0; iz <= nz; iz++) {
        double* dd = dzeros(n2); double* ff = dzeros(n2); double* wkp = dzeros(n2); double* wkq = dzeros(n2);
        double* wka = dzeros(n2); double* wkb = dzeros(n2); double* wkc = dzeros(n2);
        const double *u = PL(f[F_U], iz), *v = PL(f[F_V], iz);
        d2_spctop(&s->d2, PL(f[F_QS], iz), wkq);
        for (size_t i = 0; i < n2; i++) { wkp[i] = wkq[i] * u[i]; wkq[i] *= v[i]; }
        orc_divs(s, wkp, wkq, wka);
        for (size_t i = 0; i < n2; i++) ff[i] = PL(f[F_RI], iz)[i] * PL(f[F_DPN], iz)[i];
        deal2d_plane(s, ff);
        orc_jacob(s, ff, PL(f[F_Z], iz), wkb);
        for (size_t i = 0; i < n2; i++) PL(sqs, iz)[i] = s->filt[i] * (wkb[i] - wka[i]);
        orc_jacob(s, u, v, wkc);
        d2_spctop(&s->d2, PL(f[F_DS], iz), dd);
        for (size_t i = 0; i < n2; i++) {
            wkp[i] = ff[i] * PL(f[F_ZX], iz)[i] - dd[i] * u[i];
            wkq[i] = ff[i] * PL(f[F_ZY], iz)[i] - dd[i] * v[i];
        }
        orc_divs(s, wkp, wkq, wkb);
        for (size_t i = 0; i < n2; i++) {
            PL(sds, iz)[i] = s->filt[i] * (2.0 * wkc[i] + wkb[i] - s->hlap[i] * PL(f[F_PS], iz)[i]);
            PL(sgs, iz)[i] = COF * PL(sqs, iz)[i] + wkd[i] - FSQ * PL(f[F_AA], iz)[i];
        }
        free(dd); free(ff); free(wkp); free(wkq); free(wka); free(wkb); free(wkc);
    }
    free(wkd);
}

/* diagnose (src/nhswps/mod.rs:666-711): out = {0.5 zrms^2, zrms, zmax, umax} */
void orc_diagnose(const orc_spectral* s, double* const* f, double* out) {
    const int ng = s->ng, nz = s->nz;
    const size_t n2 = (size_t)ng * ng, n3 = n2 * (nz + 1);
    const double *u = f[F_U], *v = f[F_V], *zeta = f[F_ZETA];
    double umax2 = NAN, zmax = NAN;
    for (size_t i = 0; i < n3; i++) {
        double a = pow(u[i], 2.0) + pow(v[i], 2.0);
        umax2 = fmax(umax2, a);
        zmax = fmax(zmax, fabs(zeta[i]));
    }
    const double vsumi = 1.0 / (double)(ng * ng * nz);
    double sum = 0.0;
    for (int i = 0; i < ng; i++)
        for (int j = 0; j < ng; j++) {
            size_t p = i + (size_t)ng * j;
            sum += (1.0 / 2.0) * pow(PL(zeta, 0)[p], 2.0);
            sum += (1.0 / 2.0) * pow(PL(zeta, nz)[p], 2.0);
            for (int k = 1; k < nz; k++) sum += pow(PL(zeta, k)[p], 2.0);
        }
    double zrms = sqrt(vsumi * sum);
    out[0] = (1.0 / 2.0) * pow(zrms, 2.0);
    out[1] = zrms;
    out[2] = zmax;
    out[3] = sqrt(umax2);
}

/* energies of savegrid (src/nhswps/mod.rs:365-410): out = {ekin, epot, etot} */
void orc_energy(const orc_spectral* s, double* const* f, double* out) {
    const int ng = s->ng, nz = s->nz;
    const size_t n2 = (size_t)ng * ng;
    const double *r = f[F_R], *u = f[F_U], *v = f[F_V], *w = f[F_W], *z = f[F_Z];
    double sum = 0.0, ekin;
    for (size_t i = 0; i < n2; i++)
        sum += (1.0 + PL(r, 0)[i]) * (pow(PL(u, 0)[i], 2.0) + pow(PL(v, 0)[i], 2.0));
    ekin = (1.0 / 2.0) * sum;
    sum = 0.0;
    for (size_t i = 0; i < n2; i++)
        sum += (1.0 + PL(r, nz)[i]) * (pow(PL(u, nz)[i], 2.0) + pow(PL(v, nz)[i], 2.0) + pow(PL(w, nz)[i], 2.0));
    ekin += (1.0 / 2.0) * sum;
    for (int iz = 1; iz < nz; iz++) {
        sum = 0.0;
        for (size_t i = 0; i < n2; i++)
            sum += (1.0 + PL(r, iz)[i]) * (pow(PL(u, iz)[i], 2.0) + pow(PL(v, iz)[i], 2.0) + pow(PL(w, iz)[i], 2.0));
        ekin += sum;
    }
    const double gl = (2.0 * ORC_PI) / (double)ng, dz = HBAR / (double)nz, gvol = gl * gl * dz;
    ekin *= (1.0 / 2.0) * gvol * (1.0 / HBAR);
    sum = 0.0;
    for (size_t i = 0; i < n2; i++) sum += pow((1.0 / HBAR) * PL(z, nz)[i] - 1.0, 2.0);
    const double epot = (1.0 / 2.0) * (gl * gl) * CSQ * sum;
    out[0] = ekin;
    out[1] = epot;
    out[2] = ekin + epot;
}

/* Semi-implicit update shared by the predictor and corrector stages
 * (src/nhswps/advance.rs:69-170 and 198-273). */
static void advance_update(const orc_spectral* s, double** f, int first, double* qsi, double* qsm,
                           double* sqs, double* sds, double* sgs, double* nds, double* ngs,
                           double* dsi, double* gsi) {
    const int ng = s->ng, nz = s->nz;
    const size_t n2 = (size_t)ng * ng, n3 = n2 * (nz + 1);
    const double dt = 1.0 / (double)ng, dt4 = dt / 4.0, dt4i = 1.0 / dt4;
    double *qs = f[F_QS], *ds = f[F_DS], *gs = f[F_GS];
    if (first) {
        memcpy(qsi, qs, sizeof(double) * n3);
        for (size_t i = 0; i < n3; i++) qsm[i] = qs[i] + dt4 * sqs[i];
    }
    for (int iz = 0; iz <= nz; iz++)
        for (size_t i = 0; i < n2; i++) {
            size_t p = i + n2 * iz;
            qs[p] = s->diss[i] * (qsm[p] + dt4 * sqs[p]) - qsi[p];
        }
    if (first) {
        memcpy(dsi, ds, sizeof(double) * n3);
        memcpy(gsi, gs, sizeof(double) * n3);
        for (size_t i = 0; i < n3; i++) {
            nds[i] = sds[i] + dt4i * dsi[i];
            ngs[i] = sgs[i] + dt4i * gsi[i];
        }
    }
    for (size_t i = 0; i < n3; i++) { sds[i] += nds[i]; sgs[i] += ngs[i]; }
    double* wka = dzeros(n2);
    double* wkb = dzeros(n2);
    for (int iz = 0; iz <= nz; iz++)
        for (size_t i = 0; i < n2; i++) {
            size_t p = i + n2 * iz;
            ds[p] = sgs[p] + s->rdis[i] * sds[p];
        }
    for (int iz = 0; iz <= nz; iz++)
        for (size_t i = 0; i < n2; i++) {
            wka[i] += s->weight[iz] * PL(ds, iz)[i];
            wkb[i] += s->weight[iz] * PL(sds, iz)[i];
        }
    for (size_t i = 0; i < n2; i++) { wka[i] *= s->fope[i]; wkb[i] *= s->c2g2[i]; }
    for (int iz = 0; iz <= nz; iz++)
        for (size_t i = 0; i < n2; i++) {
            size_t p = i + n2 * iz;
            ds[p] = s->simp[i] * (ds[p] - wka[i]) - dsi[p];
            gs[p] = wkb[i] - FSQ * sds[p] + s->rdis[i] * sgs[p];
        }
    memset(wka, 0, sizeof(double) * n2);
    for (int iz = 0; iz <= nz; iz++)
        for (size_t i = 0; i < n2; i++) wka[i] += s->weight[iz] * PL(gs, iz)[i];
    for (size_t i = 0; i < n2; i++) wka[i] *= s->fope[i];
    for (int iz = 0; iz <= nz; iz++)
        for (size_t i = 0; i < n2; i++) {
            size_t p = i + n2 * iz;
            gs[p] = s->simp[i] * (gs[p] - wka[i]) - gsi[p];
        }
    free(wka);
    free(wkb);
}

/* advance (src/nhswps/advance.rs:13-279).  diag (may be NULL) receives the
 * diagnose() values at the start of the step; *t is advanced by 1/ng.
 * psolve_iters (may be NULL) receives the sweep count of each of the 3 psolve calls
 * (index 0 unused when ggen == 0). */
int orc_advance(const orc_spectral* s, double** f, int ggen, double* t, double* diag, int* psolve_iters) {
    const int ng = s->ng, nz = s->nz;
    const size_t n3 = (size_t)ng * ng * (nz + 1);
    int st, it;
    double e;
    if (ggen) {
        orc_main_invert(s, f[F_QS], f[F_DS], f[F_GS], f[F_R], f[F_U], f[F_V], f[F_ZETA]);
        st = orc_psolve(s, f, &it, &e);
        if (psolve_iters) psolve_iters[0] = it;
        if (st) return st;
    } else if (psolve_iters) {
        psolve_iters[0] = 0;
    }
    if (diag) orc_diagnose(s, f, diag);
    double* qsi = dzeros(n3); double* qsm = dzeros(n3); double* sqs = dzeros(n3);
    double* sds = dzeros(n3); double* nds = dzeros(n3); double* sgs = dzeros(n3); double* ngs = dzeros(n3);
    double* dsi = dzeros(n3); double* gsi = dzeros(n3);
    orc_source(s, f, sqs, sds, sgs);
    advance_update(s, f, 1, qsi, qsm, sqs, sds, sgs, nds, ngs, dsi, gsi);
    st = ORC_OK;
    for (int k = 0; k < 2; k++) {
        orc_main_invert(s, f[F_QS], f[F_DS], f[F_GS], f[F_R], f[F_U], f[F_V], f[F_ZETA]);
        st = orc_psolve(s, f, &it, &e);
        if (psolve_iters) psolve_iters[1 + k] = it;
        if (st) break;
        orc_source(s, f, sqs, sds, sgs);
        advance_update(s, f, 0, qsi, qsm, sqs, sds, sgs, nds, ngs, dsi, gsi);
    }
    free(qsi); free(qsm); free(sqs); free(sds); free(nds); free(sgs); free(ngs); free(dsi); free(gsi);
    if (st) return st;
    if (t) *t += 1.0 / (double)ng;
    return ORC_OK;
}

/* ======================================================================
 * Initial-condition generators (host set-up code in the reference)
 * ====================================================================== */

/* init_pv_strip (src/vstrip.rs:8-124): qq(ng,ng) Fortran order, zero mean. */
void orc_vstrip(int ng, double strip_width, double a2, double a3, double* qq) {
    const int ngu = 16 * ng;
    const double qmax = 4.0 * ORC_PI;
    const size_t nu = (size_t)ngu;
    double* qa = dzeros(nu * nu);
    double* qod0 = dzeros(ngu / 2); double* qod1 = dzeros(ngu / 2); double* qod2 = dzeros(ngu / 2);
    double* qev0 = dzeros(ngu / 2 + 1); double* qev1 = dzeros(ngu / 2 + 1); double* qev2 = dzeros(ngu / 2 + 1);
    const double hwid = strip_width / 2.0;
    const double glu = 2.0 * ORC_PI / (double)ngu;
#define QA(j, i) qa[(size_t)(j) + nu * (size_t)(i)]
    for (int i = 0; i < ngu; i++) {
        double x = glu * (double)i - ORC_PI;
        double y1 = -hwid;
        double y2 = hwid + a2 * sin(2.0 * x) + a3 * sin(3.0 * x);
        for (int j = 0; j < ngu; j++) {
            double y = glu * (double)j - ORC_PI;
            QA(j, i) = ((y2 - y) * (y - y1) > 0.0) ? 4.0 * qmax * (y2 - y) * (y - y1) / pow(y2 - y1, 2.0) : 0.0;
        }
    }
    int ngh = ngu;
    while (ngh > ng) {
        int nguf = ngh;
        ngh /= 2;
        for (int iy = 0; iy < ngh; iy++) {
            int miy = 2 * (iy + 1);
            qod2[iy] = QA(miy - 2, nguf - 1);
            qev2[iy + 1] = QA(miy - 1, nguf - 1);
        }
        qev2[0] = QA(nguf - 1, nguf - 1);
        for (int ix = 0; ix < ngh; ix++) {
            int mix = 2 * (ix + 1), mixm1 = mix - 1;
            for (int iy = 0; iy < ngh; iy++) {
                int miy = 2 * iy;
                qod1[iy] = QA(miy, mixm1 - 1);
                qod0[iy] = QA(miy, mix - 1);
                qev1[iy + 1] = QA(miy + 1, mixm1 - 1);
                qev0[iy + 1] = QA(miy + 1, mix - 1);
            }
            qev1[0] = qev1[ngh];
            qev0[0] = qev0[ngh];
            for (int iy = 0; iy < ngh; iy++)
                QA(iy, ix) = 0.0625 * (qev0[iy + 1] + qev0[iy] + qev2[iy + 1] + qev2[iy]) +
                             0.125 * (qev1[iy + 1] + qev1[iy] + qod0[iy] + qod2[iy]) + 0.25 * qod1[iy];
            memcpy(qod2, qod0, sizeof(double) * ngh);
            memcpy(qev2 + 1, qev0 + 1, sizeof(double) * ngh);
            qev2[0] = qev0[0];
        }
    }
    double qavg = 0.0;
    for (int ix = 0; ix < ng; ix++)
        for (int iy = 0; iy < ng; iy++) qavg += QA(iy, ix);
    qavg /= (double)(ng * ng);
    for (int ix = 0; ix < ng; ix++)
        for (int iy = 0; iy < ng; iy++) qq[iy + (size_t)ng * ix] = QA(iy, ix) - qavg;
#undef QA
    free(qa); free(qod0); free(qod1); free(qod2); free(qev0); free(qev1); free(qev2);
}

static double vsum(const double* a, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += a[i];
    return s;
}

/* balinit (src/balinit.rs:21-435): 2-D balanced fields from the PV strip.
 * qq_in: vstrip output (ng*ng).  Writes qq, dd, gg (ng*ng each).
 * Returns the number of iterations taken. */
int orc_balinit(int ng, int nz, const double* qq_in, double* qq_out, double* dd_out, double* gg_out) {
    const size_t n2 = (size_t)ng * ng;
    const double toler = 1.0E-9, small = 1.0E-12, dsumi = 1.0 / (double)(ng * ng);
    orc_spectral* s = orc_spectral_new(ng, nz);
    if (!s) return -1;
    const d2fft* d = &s->d2;
    double* zz = dzeros(n2); memcpy(zz, qq_in, sizeof(double) * n2);
    double* qq = dzeros(n2); memcpy(qq, qq_in, sizeof(double) * n2);
    double *uu = dzeros(n2), *vv = dzeros(n2), *hh = dzeros(n2), *dd = dzeros(n2), *gg = dzeros(n2);
    double *wkp = dzeros(n2), *wkq = dzeros(n2), *htot = dzeros(n2), *ds = dzeros(n2), *gs = dzeros(n2);
    double *wka = dzeros(n2), *wkb = dzeros(n2), *wkc = dzeros(n2), *wkd = dzeros(n2), *wke = dzeros(n2);
    double *ddpre = dzeros(n2), *ggpre = dzeros(n2);
    double qadd, qbar, fqbar, uio, vio;
    qadd = -dsumi * vsum(qq, n2);
    for (size_t i = 0; i < n2; i++) qq[i] += qadd;
    qbar = dsumi * vsum(qq, n2);
    for (size_t i = 0; i < n2; i++) wkp[i] = COF * qq[i];
    d2_ptospc(d, wkp, wkb);
    fqbar = COF * qbar;
    for (size_t i = 0; i < n2; i++) wka[i] = s->filt[i] * wkb[i] / (s->opak[i] - fqbar);
    d2_spctop(d, wka, hh);
    for (size_t i = 0; i < n2; i++) htot[i] = 1.0 + hh[i];
    for (size_t i = 0; i < n2; i++) wkp[i] = htot[i] * qq[i];
    qadd = -dsumi * vsum(wkp, n2);
    for (size_t i = 0; i < n2; i++) qq[i] += qadd;
    for (size_t i = 0; i < n2; i++) zz[i] = htot[i] * (COF + qq[i]) - COF;
    d2_ptospc(d, zz, wkb);
    for (size_t i = 0; i < n2; i++) { wka[i] = s->rlap[i] * wkb[i]; wkb[i] *= s->filt[i]; }
    d2_spctop(d, wkb, zz);
    d2_xderiv(d, wka, wkd);
    d2_yderiv(d, wka, wkb);
    for (size_t i = 0; i < n2; i++) wkb[i] = -wkb[i];
    d2_spctop(d, wkb, uu);
    d2_spctop(d, wkd, vv);
    uio = 0.0;
    for (size_t i = 0; i < n2; i++) uio += hh[i] * uu[i];
    uio = -uio * dsumi;
    for (size_t i = 0; i < n2; i++) uu[i] += uio;

    double toterrpre = 1.0 / pow(small, 2.0), toterr = 1.0 / 2.0, ddrmserr, ggrmserr;
    int iters = 0;
    while (toterr > toler) {
        iters++;
        orc_jacob(s, uu, vv, wkb);
        for (size_t i = 0; i < n2; i++) { wkp[i] = dd[i] * uu[i]; wkq[i] = dd[i] * vv[i]; }
        orc_divs(s, wkp, wkq, wka);
        for (size_t i = 0; i < n2; i++) gs[i] = s->filt[i] * (wka[i] - 2.0 * wkb[i]);
        memcpy(wka, gs, sizeof(double) * n2);
        d2_spctop(d, wka, gg);
        {
            double a = 0.0, b = 0.0;
            for (size_t i = 0; i < n2; i++) { a += pow(gg[i] - ggpre[i], 2.0); b += pow(ggpre[i], 2.0); }
            ggrmserr = a / (b + small);
        }
        for (size_t i = 0; i < n2; i++) { wkp[i] = hh[i] * uu[i]; wkq[i] = hh[i] * vv[i]; }
        orc_divs(s, wkp, wkq, wka);
        for (size_t i = 0; i < n2; i++) { wkp[i] = zz[i] * uu[i]; wkq[i] = zz[i] * vv[i]; }
        orc_divs(s, wkp, wkq, wkb);
        for (size_t i = 0; i < n2; i++) ds[i] = s->helm[i] * (COF * wkb[i] - s->c2g2[i] * wka[i]);
        memcpy(wka, ds, sizeof(double) * n2);
        d2_spctop(d, wka, dd);
        {
            double a = 0.0, b = 0.0;
            for (size_t i = 0; i < n2; i++) { a += pow(dd[i] - ddpre[i], 2.0); b += pow(ddpre[i], 2.0); }
            ddrmserr = a / (b + small);
        }
        for (size_t i = 0; i < n2; i++) htot[i] = 1.0 + hh[i];
        qadd = 0.0;
        for (size_t i = 0; i < n2; i++) qadd += qq[i] * htot[i];
        qadd = -dsumi * qadd;
        for (size_t i = 0; i < n2; i++) qq[i] += qadd;
        qbar = dsumi * vsum(qq, n2);
        for (size_t i = 0; i < n2; i++) wkp[i] = COF * (qq[i] + hh[i] * (qq[i] - qbar)) - gg[i];
        d2_ptospc(d, wkp, wkb);
        fqbar = COF * qbar;
        for (size_t i = 0; i < n2; i++) wka[i] = s->filt[i] * wkb[i] / (s->opak[i] - fqbar);
        d2_spctop(d, wka, hh);
        for (size_t i = 0; i < n2; i++) htot[i] = 1.0 + hh[i];
        for (size_t i = 0; i < n2; i++) wkp[i] = qq[i] * htot[i];
        qadd = -dsumi * vsum(wkp, n2);
        for (size_t i = 0; i < n2; i++) qq[i] += qadd;
        for (size_t i = 0; i < n2; i++) zz[i] = htot[i] * (COF + qq[i]) - COF;
        d2_ptospc(d, zz, wkb);
        for (size_t i = 0; i < n2; i++) { wka[i] = s->rlap[i] * wkb[i]; wkb[i] *= s->filt[i]; }
        d2_spctop(d, wkb, zz);
        d2_xderiv(d, wka, wkd);
        d2_yderiv(d, wka, wkb);
        for (size_t i = 0; i < n2; i++) wke[i] = s->rlap[i] * ds[i];
        d2_xderiv(d, wke, wka);
        d2_yderiv(d, wke, wkc);
        for (size_t i = 0; i < n2; i++) { wkb[i] = wka[i] - wkb[i]; wkd[i] += wkc[i]; }
        d2_spctop(d, wkb, uu);
        d2_spctop(d, wkd, vv);
        uio = 0.0; vio = 0.0;
        for (size_t i = 0; i < n2; i++) { uio += hh[i] * uu[i]; vio += hh[i] * vv[i]; }
        uio = -uio * dsumi;
        vio = -vio * dsumi;
        for (size_t i = 0; i < n2; i++) { uu[i] += uio; vv[i] += vio; }
        toterr = (1.0 / 2.0) * (ddrmserr + ggrmserr);
        if (toterrpre <= toterr) break;
        memcpy(ddpre, dd, sizeof(double) * n2);
        memcpy(ggpre, gg, sizeof(double) * n2);
        toterrpre = toterr;
    }
    for (size_t i = 0; i < n2; i++) qq_out[i] = zz[i] - COF * hh[i];
    memcpy(dd_out, dd, sizeof(double) * n2);
    memcpy(gg_out, gg, sizeof(double) * n2);
    double* fr[] = {zz, qq, uu, vv, hh, dd, gg, wkp, wkq, htot, ds, gs, wka, wkb, wkc, wkd, wke, ddpre, ggpre};
    for (size_t i = 0; i < sizeof(fr) / sizeof(fr[0]); i++) free(fr[i]);
    orc_spectral_free(s);
    return iters;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
