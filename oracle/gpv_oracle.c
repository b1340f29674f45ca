/*
 * gpv_oracle.c -- CPU FP64 ORACLE for the subset-correlation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA library is
 * compared against; it is never linked into, loaded by, or called from the
 * product path.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg (and `bench.py --impl reference`) may load it.
 *
 * It restates, in plain C (FP64 throughout, OpenMP one subset per task), the
 * algorithm of the reference geopyv-dev crate (Rust, not buildable here: no
 * cargo/rustc in the image).  Every function cites the reference file:line
 * it follows.  Where the reference calls a third-party crate the published
 * algorithm is restated:
 *   - rustfft 6.4.1 (Cargo.lock): a complex DFT; restated as radix-2 for
 *     powers of two and Bluestein's chirp-z for every other length.  Any
 *     exact-in-FP64 DFT agrees with rustfft to ~1e-15 relative.
 *   - nalgebra 0.33.3 `try_inverse`: restated as Gauss-Jordan elimination
 *     with partial pivoting; "singular" = an exactly-zero pivot.
 *
 * Parity pin: the known-answer tests of the reference (compose golden
 * vector, norm / ZNSSD / eta hand-computed values, constant-image C, Q row
 * sums, gradient = derivative at the fractional position, clamp saturation,
 * circle mask counts) are checked against this file by tests/test_oracle_*.
 */
#define _GNU_SOURCE
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* ------------------------------------------------------------------ */
/* Shared record layouts (identical byte layout to the library's C-ABI */
/* structs gpv_subset_desc / gpv_subset_result / gpv_solve_params).    */
/* ------------------------------------------------------------------ */
typedef struct {
    double coord[2];
    double p0[12];
    int32_t order;
    int32_t radius;
} gpvo_desc;

typedef struct {
    double p[12];
    double c_zncc, c_znssd, norm;
    double eta_u, eta_v;
    double f_m, delta_f, sssig, sigma;
    int32_t iterations, converged, quality_ok, status;
    int32_t n_px, has_eta;
    int32_t texture, reserved; /* 1: fitted to the rigid-texture template */
} gpvo_result;

typedef struct {
    double max_norm;
    double tolerance;
    int32_t max_iterations;
    int32_t flags; /* bit 0: eta diagnostic; bit 2: FAGN instead of ICGN; bit 3: rigid texture */
    double s2;            /* rigid texture: blob width^2 (px^2) */
    const double *grain;  /* rigid texture: fxx, fyy, fxy maps (3 x gh x gw), or NULL */
    int64_t gh, gw;
} gpvo_params;

enum {
    ST_OK = 0,
    ST_EMPTY_MASK = 1,
    ST_FEATURELESS = 2,
    ST_SINGULAR_H = 3,
    ST_SINGULAR_WDELTA = 4,
    ST_NONFINITE = 5,
    ST_INVALID = 8
};

/* ================================================================== */
/* FFT (restatement of the complex DFT that rustfft computes)          */
/* ================================================================== */
static int is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place iterative radix-2 DIT, sign = -1 forward, +1 inverse (unnormalised). */
static void fft_pow2(cplx *a, int64_t n, int sign) {
    for (int64_t i = 1, j = 0; i < n; i++) {
        int64_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { cplx t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    for (int64_t len = 2; len <= n; len <<= 1) {
        int64_t half = len >> 1;
        for (int64_t k = 0; k < half; k++) {
            double ang = sign * 2.0 * M_PI * (double)k / (double)len;
            cplx w = cos(ang) + I * sin(ang);
            for (int64_t i = k; i < n; i += len) {
                cplx u = a[i], v = a[i + half] * w;
                a[i] = u + v;
                a[i + half] = u - v;
            }
        }
    }
}

typedef struct {
    int64_t n, m;     /* length, padded pow2 length (0 when n is pow2) */
    cplx *chirp;      /* w[j] = exp(-i*pi*j^2/n), j < n               */
    cplx *bhat;       /* FFT of the conjugate chirp, length m          */
} fft_plan;

static void plan_init(fft_plan *p, int64_t n) {
    p->n = n; p->m = 0; p->chirp = NULL; p->bhat = NULL;
    if (is_pow2(n)) return;
    int64_t m = 1;
    while (m < 2 * n - 1) m <<= 1;
    p->m = m;
    p->chirp = (cplx *)malloc(sizeof(cplx) * n);
    p->bhat = (cplx *)calloc(m, sizeof(cplx));
    for (int64_t j = 0; j < n; j++) {
        /* j^2 mod 2n keeps the argument small and exact */
        int64_t q = (j * j) % (2 * n);
        double ang = -M_PI * (double)q / (double)n;
        p->chirp[j] = cos(ang) + I * sin(ang);
    }
    p->bhat[0] = conj(p->chirp[0]);
    for (int64_t j = 1; j < n; j++) {
        p->bhat[j] = conj(p->chirp[j]);
        p->bhat[m - j] = conj(p->chirp[j]);
    }
    fft_pow2(p->bhat, m, -1);
}

static void plan_free(fft_plan *p) { free(p->chirp); free(p->bhat); }

/* Forward (sign=-1) or unnormalised inverse (sign=+1) DFT of x, in place.
 * work: m complex scratch (unused for pow2 lengths). */
static void fft_any(const fft_plan *p, cplx *x, int sign, cplx *work) {
    int64_t n = p->n;
    if (p->m == 0) { fft_pow2(x, n, sign); return; }
    int64_t m = p->m;
    /* inverse via conjugation: IDFT(x) = conj(DFT(conj(x))) */
    if (sign > 0) for (int64_t j = 0; j < n; j++) x[j] = conj(x[j]);
    for (int64_t j = 0; j < n; j++) work[j] = x[j] * p->chirp[j];
    for (int64_t j = n; j < m; j++) work[j] = 0;
    fft_pow2(work, m, -1);
    for (int64_t j = 0; j < m; j++) work[j] *= p->bhat[j];
    fft_pow2(work, m, +1);
    double s = 1.0 / (double)m;
    for (int64_t k = 0; k < n; k++) x[k] = work[k] * s * p->chirp[k];
    if (sign > 0) for (int64_t j = 0; j < n; j++) x[j] = conj(x[j]);
}

/* Exported for the FFT cross-check against numpy.fft. */
void gpvo_fft(const double *re_in, const double *im_in, int64_t n, int sign,
              double *re_out, double *im_out) {
    fft_plan p; plan_init(&p, n);
    cplx *x = (cplx *)malloc(sizeof(cplx) * n);
    cplx *w = (cplx *)malloc(sizeof(cplx) * (p.m ? p.m : 1));
    for (int64_t j = 0; j < n; j++) x[j] = re_in[j] + I * im_in[j];
    fft_any(&p, x, sign, w);
    for (int64_t j = 0; j < n; j++) { re_out[j] = creal(x[j]); im_out[j] = cimag(x[j]); }
    free(x); free(w); plan_free(&p);
}

/* ================================================================== */
/* B-spline prefilter: get_c (src/image.rs:252-327)                    */
/* ================================================================== */

/* build_kernel (src/image.rs:422-430): zero-phase quintic kernel. */
static void build_kernel(int64_t n, cplx *k) {
    static const double kk[6] = {1.0 / 120.0, 13.0 / 60.0, 11.0 / 20.0, 13.0 / 60.0, 1.0 / 120.0, 0.0};
    for (int64_t i = 0; i < n; i++) k[i] = 0;
    k[0] = kk[2]; k[1] = kk[3]; k[2] = kk[4];
    k[n - 2] = kk[0]; k[n - 1] = kk[1];
}

/* Deconvolve each of `count` contiguous lines of length n (src/image.rs:270-315). */
static void deconvolve_lines(cplx *data, int64_t count, int64_t n, int nthreads) {
    fft_plan p; plan_init(&p, n);
    cplx *kern = (cplx *)malloc(sizeof(cplx) * n);
    cplx *kw = (cplx *)malloc(sizeof(cplx) * (p.m ? p.m : 1));
    build_kernel(n, kern);
    fft_any(&p, kern, -1, kw);
    free(kw);
    double scale = 1.0 / (double)n;
#pragma omp parallel num_threads(nthreads)
    {
        cplx *work = (cplx *)malloc(sizeof(cplx) * (p.m ? p.m : 1));
#pragma omp for schedule(static)
        for (int64_t l = 0; l < count; l++) {
            cplx *row = data + l * n;
            fft_any(&p, row, -1, work);
            for (int64_t i = 0; i < n; i++) row[i] /= kern[i];
            fft_any(&p, row, +1, work);
            for (int64_t i = 0; i < n; i++) row[i] *= scale;
        }
        free(work);
    }
    free(kern);
    plan_free(&p);
}

/* get_c + pad_replicate (src/image.rs:252-327, :436-443).
 * img: (h, w) row-major; out: (h+2b, w+2b) row-major. */
void gpvo_get_c(const double *img, int64_t h, int64_t w, int64_t border, double *out, int nthreads) {
    int64_t pr = h + 2 * border, pc = w + 2 * border;
    cplx *c = (cplx *)malloc(sizeof(cplx) * pr * pc);
    for (int64_t i = 0; i < pr; i++) {
        int64_t ri = i < border ? 0 : (i - border > h - 1 ? h - 1 : i - border);
        for (int64_t j = 0; j < pc; j++) {
            int64_t ci = j < border ? 0 : (j - border > w - 1 ? w - 1 : j - border);
            c[i * pc + j] = img[ri * w + ci];
        }
    }
    deconvolve_lines(c, pr, pc, nthreads);          /* row pass */
    cplx *t = (cplx *)malloc(sizeof(cplx) * pr * pc); /* transpose (:292-297) */
    for (int64_t i = 0; i < pr; i++)
        for (int64_t j = 0; j < pc; j++) t[j * pr + i] = c[i * pc + j];
    deconvolve_lines(t, pc, pr, nthreads);          /* column pass */
    for (int64_t i = 0; i < pr; i++)                 /* real part (:324-326) */
        for (int64_t j = 0; j < pc; j++) out[i * pc + j] = creal(t[j * pr + i]);
    free(c); free(t);
}

/* ================================================================== */
/* B-spline evaluation (src/image.rs:115-230)                          */
/* ================================================================== */
static const double QM[6][6] = {
    {1.0 / 120.0, 13.0 / 60.0, 11.0 / 20.0, 13.0 / 60.0, 1.0 / 120.0, 0.0},
    {-1.0 / 24.0, -5.0 / 12.0, 0.0, 5.0 / 12.0, 1.0 / 24.0, 0.0},
    {1.0 / 12.0, 1.0 / 6.0, -1.0 / 2.0, 1.0 / 6.0, 1.0 / 12.0, 0.0},
    {-1.0 / 12.0, 1.0 / 6.0, 0.0, -1.0 / 6.0, 1.0 / 12.0, 0.0},
    {1.0 / 24.0, -1.0 / 6.0, 1.0 / 4.0, -1.0 / 6.0, 1.0 / 24.0, 0.0},
    {-1.0 / 120.0, 1.0 / 24.0, -1.0 / 12.0, 1.0 / 12.0, -1.0 / 24.0, 1.0 / 120.0},
};

/* qt_poly (src/image.rs:193-208) */
static void qt_poly(double t, double out[6]) {
    double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
    double p[6] = {1.0, t, t2, t3, t4, t4 * t};
    for (int k = 0; k < 6; k++) {
        double s = 0.0;
        for (int r = 0; r < 6; r++) s += QM[r][k] * p[r];
        out[k] = s;
    }
}

/* qt_dpoly (src/image.rs:216-230) */
static void qt_dpoly(double t, double out[6]) {
    double t2 = t * t, t3 = t2 * t;
    double p[6] = {0.0, 1.0, 2.0 * t, 3.0 * t2, 4.0 * t3, 5.0 * t2 * t2};
    for (int k = 0; k < 6; k++) {
        double s = 0.0;
        for (int r = 0; r < 6; r++) s += QM[r][k] * p[r];
        out[k] = s;
    }
}

void gpvo_qt_poly(double t, double *out) { qt_poly(t, out); }
void gpvo_qt_dpoly(double t, double *out) { qt_dpoly(t, out); }

typedef struct {
    const double *c;
    int64_t h, w, border, cw; /* image height/width, border, coefficient row length */
} spline;

/* Image::eval (src/image.rs:128-148) */
static double sp_eval(const spline *s, double x, double y) {
    double xm = (double)s->w - 1e-9, ym = (double)s->h - 1e-9;
    x = x < 0.0 ? 0.0 : (x > xm ? xm : x);
    y = y < 0.0 ? 0.0 : (y > ym ? ym : y);
    double xf = floor(x), yf = floor(y);
    double a[6], b[6];
    qt_poly(y - yf, a);
    qt_poly(x - xf, b);
    int64_t r0 = (int64_t)yf + s->border - 2, c0 = (int64_t)xf + s->border - 2;
    double val = 0.0;
    for (int r = 0; r < 6; r++) {
        const double *row = s->c + (r0 + r) * s->cw + c0;
        double acc = 0.0;
        for (int k = 0; k < 6; k++) acc += row[k] * b[k];
        val += a[r] * acc;
    }
    return val;
}

/* Image::rows + Image::eval_grad (src/image.rs:115-124, :155-178) */
static double sp_eval_grad(const spline *s, double x, double y, double *gx, double *gy) {
    double xm = (double)s->w - 1e-9, ym = (double)s->h - 1e-9;
    x = x < 0.0 ? 0.0 : (x > xm ? xm : x);
    y = y < 0.0 ? 0.0 : (y > ym ? ym : y);
    double xf = floor(x), yf = floor(y);
    double a[6], da[6], b[6], db[6];
    qt_poly(y - yf, a); qt_dpoly(y - yf, da);
    qt_poly(x - xf, b); qt_dpoly(x - xf, db);
    int64_t r0 = (int64_t)yf + s->border - 2, c0 = (int64_t)xf + s->border - 2;
    double cb[6], cq[6];
    for (int r = 0; r < 6; r++) {
        const double *row = s->c + (r0 + r) * s->cw + c0;
        double t1 = 0.0, t2 = 0.0;
        for (int k = 0; k < 6; k++) { t1 += row[k] * b[k]; t2 += row[k] * db[k]; }
        cb[r] = t1; cq[r] = t2;
    }
    double val = 0.0, vx = 0.0, vy = 0.0;
    for (int r = 0; r < 6; r++) { val += a[r] * cb[r]; vx += a[r] * cq[r]; vy += da[r] * cb[r]; }
    *gx = vx; *gy = vy;
    return val;
}

/* Batch evaluation (exported for the interpolation parity tests). */
void gpvo_eval(const double *c, int64_t h, int64_t w, int64_t border, const double *xy, int64_t n,
               double *val, double *grad) {
    spline s = {c, h, w, border, w + 2 * border};
    for (int64_t i = 0; i < n; i++) {
        if (grad) val[i] = sp_eval_grad(&s, xy[2 * i], xy[2 * i + 1], &grad[2 * i], &grad[2 * i + 1]);
        else val[i] = sp_eval(&s, xy[2 * i], xy[2 * i + 1]);
    }
}

/* ================================================================== */
/* Masks (src/masks.rs:69-109 circle, :199-263 mask_update)            */
/* ================================================================== */

/* Circle offsets, row-major scan (y outer, x inner), columns [x, y].
 * Returns n_px; coords may be NULL to count only. */
int64_t gpvo_circle(int64_t radius, double *coords) {
    int64_t n = 0, side = 2 * radius + 1;
    for (int64_t row = 0; row < side; row++)
        for (int64_t col = 0; col < side; col++) {
            int64_t x = col - radius, y = row - radius;
            double dist = sqrt((double)(x * x + y * y));
            if (dist <= (double)radius) {
                if (coords) { coords[2 * n] = (double)x; coords[2 * n + 1] = (double)y; }
                n++;
            }
        }
    return n;
}

/* mask_update for a circle template: keep, in scan order, the offsets whose
 * image pixel (trunc(centre)+offset) lies in the extracted mask window and is
 * non-zero.  The window extraction of src/masks.rs:210-247 excludes the last
 * mask row/column whenever the template reaches it (slice end clamped to
 * len-1), and that is reproduced here.  out may alias nothing; returns n. */
int64_t gpvo_mask_update(const double *coords, int64_t n_in, int64_t size, const double centre[2],
                         const uint8_t *mask, int64_t mh, int64_t mw, double *out) {
    int64_t cx = (int64_t)centre[0], cy = (int64_t)centre[1]; /* `as isize` truncates */
    int64_t ly = cy - size, uy = cy + size + 1, lx = cx - size, ux = cx + size + 1;
    if (lx < 0) lx = 0;
    if (ly < 0) ly = 0;
    if (ux >= mw) ux = mw - 1;
    if (uy >= mh) uy = mh - 1;
    int64_t n = 0;
    for (int64_t i = 0; i < n_in; i++) {
        int64_t ox = (int64_t)coords[2 * i], oy = (int64_t)coords[2 * i + 1];
        int64_t X = cx + ox, Y = cy + oy;
        if (X < lx || X >= ux || Y < ly || Y >= uy) continue;
        if (mask[Y * mw + X] == 0) continue;
        out[2 * n] = (double)ox; out[2 * n + 1] = (double)oy;
        n++;
    }
    return n;
}

/* ================================================================== */
/* Subset maths (src/subset.rs)                                        */
/* ================================================================== */
static int p_len(int order) { return order == 0 ? 2 : (order == 1 ? 6 : 12); }

/* Gauss-Jordan inverse with partial pivoting (stands in for nalgebra
 * try_inverse).  Returns 0 on an exactly-zero or non-finite pivot. */
static int invert(const double *a, int n, double *inv) {
    double m[12][24];
    for (int i = 0; i < n; i++)
        for (int j = 0; j < 2 * n; j++) m[i][j] = j < n ? a[i * n + j] : (j - n == i ? 1.0 : 0.0);
    for (int k = 0; k < n; k++) {
        int piv = k;
        double best = fabs(m[k][k]);
        for (int i = k + 1; i < n; i++)
            if (fabs(m[i][k]) > best) { best = fabs(m[i][k]); piv = i; }
        if (!(best > 0.0) || !isfinite(best)) return 0;
        if (piv != k)
            for (int j = 0; j < 2 * n; j++) { double t = m[k][j]; m[k][j] = m[piv][j]; m[piv][j] = t; }
        double d = m[k][k];
        for (int j = 0; j < 2 * n; j++) m[k][j] /= d;
        for (int i = 0; i < n; i++) {
            if (i == k) continue;
            double f = m[i][k];
            if (f == 0.0) continue;
            for (int j = 0; j < 2 * n; j++) m[i][j] -= f * m[k][j];
        }
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) inv[i * n + j] = m[i][j + n];
    return 1;
}

/* apply_warp_into (src/subset.rs:262-300) for one point */
static void warp_point(const double coord[2], const double *p, int len, double x, double y, double *ox, double *oy) {
    if (len == 2) { *ox = x + p[0]; *oy = y + p[1]; return; }
    double dx = x - coord[0], dy = y - coord[1];
    if (len <= 7) {
        *ox = x + p[0] + p[2] * dx + p[4] * dy;
        *oy = y + p[1] + p[3] * dx + p[5] * dy;
    } else {
        *ox = x + p[0] + p[2] * dx + p[4] * dy + 0.5 * p[6] * dx * dx + p[8] * dx * dy + 0.5 * p[10] * dy * dy;
        *oy = y + p[1] + p[3] * dx + p[5] * dy + 0.5 * p[7] * dx * dx + p[9] * dx * dy + 0.5 * p[11] * dy * dy;
    }
}

void gpvo_apply_warp(const double coord[2], const double *p, int len, const double *xy, int64_t n, double *out) {
    for (int64_t i = 0; i < n; i++) warp_point(coord, p, len, xy[2 * i], xy[2 * i + 1], &out[2 * i], &out[2 * i + 1]);
}

/* steepest_descent (src/subset.rs:311-343), one row */
static void sdi_row(double dx, double dy, double gx, double gy, int m, double *s) {
    s[0] = gx; s[1] = gy;
    if (m < 6) return;
    s[2] = gx * dx; s[3] = gy * dx; s[4] = gx * dy; s[5] = gy * dy;
    if (m == 12) {
        s[6] = gx * 0.5 * dx * dx; s[7] = gy * 0.5 * dx * dx;
        s[8] = gx * dx * dy; s[9] = gy * dx * dy;
        s[10] = gx * 0.5 * dy * dy; s[11] = gy * 0.5 * dy * dy;
    }
}

void gpvo_steepest_descent(const double coord[2], const double *xy, const double *grad, int64_t n, int order, double *sdi) {
    int m = p_len(order);
    for (int64_t i = 0; i < n; i++)
        sdi_row(xy[2 * i] - coord[0], xy[2 * i + 1] - coord[1], grad[2 * i], grad[2 * i + 1], m, sdi + i * m);
}

/* compose_icgn (src/subset.rs:487-611).  Returns 0 if W_delta is singular. */
static void s_terms(const double *q, double *s) {
    double u = q[0], v = q[1], ux = q[2], vx = q[3], uy = q[4], vy = q[5];
    double uxx = q[6], vxx = q[7], uxy = q[8], vxy = q[9], uyy = q[10], vyy = q[11];
    s[0] = 2.0 * ux + ux * ux + u * uxx;
    s[1] = 2.0 * u * uxy + 2.0 * (1.0 + ux) * uy;
    s[2] = uy * uy + u * uyy;
    s[3] = 2.0 * u * (1.0 + ux);
    s[4] = 2.0 * u * uy;
    s[5] = u * u;
    s[6] = 0.5 * (v * uxx + 2.0 * (1.0 + ux) * vx + u * vxx);
    s[7] = uy * vx + ux * vy + v * uxy + u * vxy + vy + ux;
    s[8] = 0.5 * (v * uyy + 2.0 * uy * (1.0 + vy) + u * vyy);
    s[9] = v + v * ux + u * vx;
    s[10] = u + v * uy + u * vy;
    s[11] = u * v;
    s[12] = vx * vx + v * vxx;
    s[13] = 2.0 * v * vxy + 2.0 * vx * (1.0 + vy);
    s[14] = 2.0 * vy + vy * vy + v * vyy;
    s[15] = 2.0 * v * vx;
    s[16] = 2.0 * v * (1.0 + vy);
    s[17] = v * v;
}

static void lifted6(const double *q, double *W) {
    double s[18];
    s_terms(q, s);
    double rows[36] = {
        1.0 + s[0], s[1], s[2], s[3], s[4], s[5],
        s[6], 1.0 + s[7], s[8], s[9], s[10], s[11],
        s[12], s[13], 1.0 + s[14], s[15], s[16], s[17],
        0.5 * q[6], q[8], 0.5 * q[10], 1.0 + q[2], q[4], q[0],
        0.5 * q[7], q[9], 0.5 * q[11], q[3], 1.0 + q[5], q[1],
        0.0, 0.0, 0.0, 0.0, 0.0, 1.0};
    memcpy(W, rows, sizeof(rows));
}

int gpvo_compose(const double *p, const double *dp, int len, double *out) {
    if (len == 2) { out[0] = p[0] - dp[0]; out[1] = p[1] - dp[1]; return 1; }
    if (len == 6) {
        double wo[9] = {1.0 + p[2], p[4], p[0], p[3], 1.0 + p[5], p[1], 0, 0, 1};
        double wd[9] = {1.0 + dp[2], dp[4], dp[0], dp[3], 1.0 + dp[5], dp[1], 0, 0, 1};
        double wi[9], wn[9];
        if (!invert(wd, 3, wi)) return 0;
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) {
                double acc = 0.0;
                for (int k = 0; k < 3; k++) acc += wo[r * 3 + k] * wi[k * 3 + c];
                wn[r * 3 + c] = acc;
            }
        out[0] = wn[0 * 3 + 2]; out[1] = wn[1 * 3 + 2];
        out[2] = wn[0] - 1.0; out[3] = wn[3]; out[4] = wn[1]; out[5] = wn[4] - 1.0;
        return 1;
    }
    double wo[36], wd[36], wi[36], wn[36];
    lifted6(p, wo);
    lifted6(dp, wd);
    if (!invert(wd, 6, wi)) return 0;
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) {
            double acc = 0.0;
            for (int k = 0; k < 6; k++) acc += wo[r * 6 + k] * wi[k * 6 + c];
            wn[r * 6 + c] = acc;
        }
    out[0] = wn[3 * 6 + 5]; out[1] = wn[4 * 6 + 5];
    out[2] = wn[3 * 6 + 3] - 1.0; out[3] = wn[4 * 6 + 3];
    out[4] = wn[3 * 6 + 4]; out[5] = wn[4 * 6 + 4] - 1.0;
    out[6] = wn[3 * 6 + 0] * 2.0; out[7] = wn[4 * 6 + 0] * 2.0;
    out[8] = wn[3 * 6 + 1]; out[9] = wn[4 * 6 + 1];
    out[10] = wn[3 * 6 + 2] * 2.0; out[11] = wn[4 * 6 + 2] * 2.0;
    return 1;
}

/* convergence_norm (src/subset.rs:622-649) */
double gpvo_norm(const double *dp, int len, double size) {
    if (len == 2) return sqrt(dp[0] * dp[0] + dp[1] * dp[1]);
    double s = dp[0] * dp[0] + dp[1] * dp[1];
    for (int k = 2; k < 6; k++) s += (dp[k] * size) * (dp[k] * size);
    if (len > 7)
        for (int k = 6; k < 12; k++) { double t = 0.5 * dp[k] * size * size; s += t * t; }
    return sqrt(s);
}

/* znssd (src/subset.rs:654-669) */
double gpvo_znssd(const double *f, const double *g, int64_t n, double f_m, double g_m, double df, double dg) {
    double acc = 0.0;
    for (int64_t i = 0; i < n; i++) { double v = (f[i] - f_m) / df - (g[i] - g_m) / dg; acc += v * v; }
    return acc;
}

/* zn_slice (src/subset.rs:698-704) */
static void zn_slice(const double *x, int64_t n, double *out) {
    double mean = 0.0;
    for (int64_t i = 0; i < n; i++) mean += x[i];
    mean /= (double)n;
    double var = 0.0;
    for (int64_t i = 0; i < n; i++) var += (x[i] - mean) * (x[i] - mean);
    var /= (double)n;
    double sd = sqrt(var > 1e-18 ? var : 1e-18);
    for (int64_t i = 0; i < n; i++) out[i] = (x[i] - mean) / sd;
}

void gpvo_zn_slice(const double *x, int64_t n, double *out) { zn_slice(x, n, out); }

/* eta_component (src/subset.rs:713-727); modes row-major (n, K). */
double gpvo_eta_component(const double *modes, int K, const double *grad_zn, const double *ec, int64_t n) {
    double *raw = (double *)malloc(sizeof(double) * n), *sc = (double *)malloc(sizeof(double) * n);
    double ss = 0.0;
    for (int k = 0; k < K; k++) {
        for (int64_t i = 0; i < n; i++) raw[i] = grad_zn[i] * modes[i * K + k];
        zn_slice(raw, n, sc);
        double pr = 0.0;
        for (int64_t i = 0; i < n; i++) pr += sc[i] * ec[i];
        pr /= (double)n;
        ss += pr * pr;
    }
    free(raw); free(sc);
    return sqrt(ss);
}

/* omitted_mode_diagnostic (src/subset.rs:748-820).  Returns 0 for an
 * unsupported order. */
int gpvo_eta(const double coord[2], int order, const double *fc, const double *grad, const double *f, double f_m,
             double df, const double *g, double g_m, double dg, int64_t n, double *eta_u, double *eta_v) {
    if (order < 0 || order > 2) return 0;
    int K = order + 2;
    double *e = (double *)malloc(sizeof(double) * n), *gx = (double *)malloc(sizeof(double) * n);
    double *gy = (double *)malloc(sizeof(double) * n), *zx = (double *)malloc(sizeof(double) * n);
    double *zy = (double *)malloc(sizeof(double) * n), *modes = (double *)malloc(sizeof(double) * n * K);
    double eb = 0.0;
    for (int64_t i = 0; i < n; i++) { e[i] = (f[i] - f_m) / df - (g[i] - g_m) / dg; eb += e[i]; }
    eb /= (double)n;
    for (int64_t i = 0; i < n; i++) { e[i] -= eb; gx[i] = grad[2 * i]; gy[i] = grad[2 * i + 1]; }
    zn_slice(gx, n, zx);
    zn_slice(gy, n, zy);
    for (int64_t i = 0; i < n; i++) {
        double xi = fc[2 * i] - coord[0], ze = fc[2 * i + 1] - coord[1];
        double *m = modes + i * K;
        if (order == 0) { m[0] = xi; m[1] = ze; }
        else if (order == 1) { m[0] = xi * xi; m[1] = xi * ze; m[2] = ze * ze; }
        else { m[0] = xi * xi * xi; m[1] = xi * xi * ze; m[2] = xi * ze * ze; m[3] = ze * ze * ze; }
    }
    *eta_u = gpvo_eta_component(modes, K, zx, e, n);
    *eta_v = gpvo_eta_component(modes, K, zy, e, n);
    free(e); free(gx); free(gy); free(zx); free(zy); free(modes);
    return 1;
}

/* ================================================================== */
/* Rigid-texture template (src/texture.rs, src/seam.rs:255-301)        */
/* ================================================================== */

/* Speckle correlation length (correlation_length, src/seam.rs:255-301):
 * the centred side x side crop (side = min(512, rows, cols), even) with its
 * mean removed, its circular autocorrelation along x and y at lags
 * 0..side/2-1 (the reference takes them from |FFT|^2; here as direct lag
 * sums), profile = mean of the two / lag 0, and the lag where it first
 * falls below 0.5, interpolated linearly.  0 ok, 1 image too small, 2 the
 * profile never falls to 0.5. */
int gpvo_correlation_length(const double *a, int64_t rows, int64_t cols, double *ell) {
    int64_t side = rows < cols ? rows : cols;
    if (side > 512) side = 512;
    side &= ~(int64_t)1;
    if (side < 16) return 1;
    const int64_t half = side / 2, cy = rows / 2, cx = cols / 2;
    double *crop = (double *)malloc(sizeof(double) * side * side);
    for (int64_t r = 0; r < side; r++)
        for (int64_t c = 0; c < side; c++) crop[r * side + c] = a[(cy - half + r) * cols + (cx - half + c)];
    double mean = 0.0;
    for (int64_t i = 0; i < side * side; i++) mean += crop[i];
    mean /= (double)(side * side);
    for (int64_t i = 0; i < side * side; i++) crop[i] -= mean;
    double *ax = (double *)malloc(sizeof(double) * half), *ay = (double *)malloc(sizeof(double) * half);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t k = 0; k < half; k++) {
        double sx = 0.0, sy = 0.0;
        for (int64_t r = 0; r < side; r++)
            for (int64_t c = 0; c < side; c++) {
                const double v = crop[r * side + c];
                sx += v * crop[r * side + (c + k) % side];
                sy += v * crop[((r + k) % side) * side + c];
            }
        ax[k] = sx;
        ay[k] = sy;
    }
    int rc = 2;
    double prev = 1.0;
    for (int64_t k = 0; k < half; k++) {
        const double prof = 0.5 * (ax[k] + ay[k]) / ax[0];
        if (prof < 0.5) {
            *ell = (double)k - 1.0 + (prev - 0.5) / (prev - prof);
            rc = 0;
            break;
        }
        prev = prof;
    }
    free(crop); free(ax); free(ay);
    return rc;
}

/* Gaussian kernel of width sigma, radius ceil(4 sigma), derivative order 0,
 * 1 or 2, as correlation weights normalised by the Gaussian's sum
 * (kernel_with, src/texture.rs:49-68).  Returns the radius. */
int gpvo_gauss_kernel(int order, double sigma, double *k) {
    const int r = (int)ceil(4.0 * sigma);
    const double s2 = sigma * sigma;
    double norm = 0.0;
    for (int i = -r; i <= r; i++) norm += exp(-(double)(i * i) / (2.0 * s2));
    for (int i = -r; i <= r; i++) {
        const double t = (double)i, gi = exp(-(double)(i * i) / (2.0 * s2));
        const double v = order == 0 ? gi : (order == 1 ? t / s2 * gi : (t * t / (s2 * s2) - 1.0 / s2) * gi);
        k[i + r] = v / norm;
    }
    return r;
}

/* Correlate rows (along x) or columns of a (rows x cols) with k (2r+1
 * taps), replicating edge pixels; a left-to-right sum of products
 * (filter_1d, src/texture.rs:70-93). */
static void filter_1d(const double *a, int64_t rows, int64_t cols, const double *k, int r, int along_rows, double *out) {
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < rows; y++)
        for (int64_t x = 0; x < cols; x++) {
            double s = 0.0;
            for (int j = 0; j <= 2 * r; j++) {
                const int64_t t = j - r;
                double v;
                if (along_rows) {
                    int64_t xx = x + t;
                    xx = xx < 0 ? 0 : (xx > cols - 1 ? cols - 1 : xx);
                    v = a[y * cols + xx];
                } else {
                    int64_t yy = y + t;
                    yy = yy < 0 ? 0 : (yy > rows - 1 ? rows - 1 : yy);
                    v = a[yy * cols + x];
                }
                s += k[j] * v;
            }
            out[y * cols + x] = s;
        }
}

/* GrainMaps::build (src/texture.rs:99-115) after the correlation length:
 * with SMOOTH = 1, fxx = cols(rows(a, k2), k0) corr, fyy = cols(rows(a, k0),
 * k2) corr, fxy = cols(rows(a, k1), k1) corr.  maps: 3 x rows x cols. */
void gpvo_grain_maps(const double *a, int64_t rows, int64_t cols, double corr, double *maps) {
    double k[3][9];
    int r = 0;
    for (int o = 0; o < 3; o++) r = gpvo_gauss_kernel(o, 1.0, k[o]);
    const int64_t np = rows * cols;
    double *h = (double *)malloc(sizeof(double) * np), *t = (double *)malloc(sizeof(double) * np);
    const int pairs[3][2] = {{2, 0}, {0, 2}, {1, 1}};  /* (row kernel, column kernel) of fxx, fyy, fxy */
    for (int m = 0; m < 3; m++) {
        filter_1d(a, rows, cols, k[pairs[m][0]], r, 1, h);
        filter_1d(h, rows, cols, k[pairs[m][1]], r, 0, t);
        for (int64_t i = 0; i < np; i++) maps[m * np + i] = t[i] * corr;
    }
    free(h); free(t);
}

/* Bilinear sample of the three maps at (x = column, y = row), clamped
 * (GrainMaps::sample, src/texture.rs:125-143). */
static void grain_sample(const double *maps, int64_t rows, int64_t cols, double x, double y, double h[3]) {
    x = x < 0.0 ? 0.0 : (x > (double)(cols - 1) ? (double)(cols - 1) : x);
    y = y < 0.0 ? 0.0 : (y > (double)(rows - 1) ? (double)(rows - 1) : y);
    int64_t x0 = (int64_t)floor(x), y0 = (int64_t)floor(y);
    if (x0 > cols - 2) x0 = cols - 2 < 0 ? 0 : cols - 2;
    if (y0 > rows - 2) y0 = rows - 2 < 0 ? 0 : rows - 2;
    const int64_t x1 = x0 + 1 < cols - 1 ? x0 + 1 : cols - 1, y1 = y0 + 1 < rows - 1 ? y0 + 1 : rows - 1;
    const double tx = x - (double)x0, ty = y - (double)y0;
    for (int m = 0; m < 3; m++) {
        const double *M = maps + m * rows * cols;
        h[m] = (1.0 - ty) * ((1.0 - tx) * M[y0 * cols + x0] + tx * M[y0 * cols + x1]) +
               ty * ((1.0 - tx) * M[y1 * cols + x0] + tx * M[y1 * cols + x1]);
    }
}

/* Green-Lagrange strain [Exx, Eyy, Exy] (src/texture.rs:200-206). */
static void green_lagrange(double ux, double vx, double uy, double vy, double e[3]) {
    e[0] = ux + 0.5 * (ux * ux + vx * vx);
    e[1] = vy + 0.5 * (uy * uy + vy * vy);
    e[2] = 0.5 * (uy + vx) + 0.5 * (ux * uy + vx * vy);
}

/* The template f + G(E(p)) with base = the subset mean, its mean and spread
 * (grain_template, src/texture.rs:213-244; rigid_template, src/subset.rs:
 * 1399-1411).  xy: (n,2) offsets of the pixels from the centre. */
static void rigid_template(const double *f, double f_m, const double *h, double s2, const double *p, int m,
                           const double *xy, int64_t n, double *t, double *t_m, double *delta_t) {
    double e[3];
    if (m <= 7) green_lagrange(p[2], p[3], p[4], p[5], e);
    for (int64_t i = 0; i < n; i++) {
        if (m > 7) {
            const double dx = xy[2 * i], dy = xy[2 * i + 1];
            green_lagrange(p[2] + p[6] * dx + p[8] * dy, p[3] + p[7] * dx + p[9] * dy, p[4] + p[8] * dx + p[10] * dy,
                           p[5] + p[9] * dx + p[11] * dy, e);
        }
        const double *hi = h + 3 * i;
        t[i] = f[i] + (-0.5 * s2 * (e[0] * hi[0] + e[1] * hi[1] + 2.0 * e[2] * hi[2]) - (e[0] + e[1]) * (f[i] - f_m));
    }
    double sum = 0.0;
    for (int64_t i = 0; i < n; i++) sum += t[i];
    *t_m = sum / (double)n;
    double ss = 0.0;
    for (int64_t i = 0; i < n; i++) ss += (t[i] - *t_m) * (t[i] - *t_m);
    *delta_t = sqrt(ss);
}

/* grain_template alone (src/texture.rs:213-244) for the template tests:
 * out = f + G(E(p)); m = 2 returns f. */
void gpvo_grain_template(const double *f, double f_m, const double *h, double s2, const double *p, int m,
                         const double *xy, int64_t n, double *out) {
    if (m == 2) {
        memcpy(out, f, sizeof(double) * n);
        return;
    }
    double t_m, dt;
    rigid_template(f, f_m, h, s2, p, m, xy, n, out, &t_m, &dt);
}

/* ================================================================== */
/* Subset::new + solve_icgn_result (src/subset.rs:836-919, 1117-1219)  */
/* ================================================================== */
typedef struct {
    int64_t n;
    double *fc;   /* (n,2) f_coords */
    double *f;    /* (n) */
    double *grad; /* (n,2) */
    double f_m, delta_f, sssig, sigma;
} subset_ref;

static int subset_new(const spline *F, const double coord[2], int64_t radius, const uint8_t *mask, int64_t mh,
                      int64_t mw, subset_ref *s) {
    memset(s, 0, sizeof(*s));
    int64_t nc = gpvo_circle(radius, NULL);
    double *coords = (double *)malloc(sizeof(double) * 2 * nc);
    gpvo_circle(radius, coords);
    int64_t n = nc;
    if (mask) {
        double *kept = (double *)malloc(sizeof(double) * 2 * nc);
        n = gpvo_mask_update(coords, nc, radius, coord, mask, mh, mw, kept);
        free(coords);
        coords = kept;
    }
    s->n = n;
    if (n == 0) { free(coords); return ST_EMPTY_MASK; }
    s->fc = (double *)malloc(sizeof(double) * 2 * n);
    s->f = (double *)malloc(sizeof(double) * n);
    s->grad = (double *)malloc(sizeof(double) * 2 * n);
    for (int64_t i = 0; i < n; i++) {
        s->fc[2 * i] = coords[2 * i] + coord[0];
        s->fc[2 * i + 1] = coords[2 * i + 1] + coord[1];
    }
    free(coords);
    for (int64_t i = 0; i < n; i++)
        s->f[i] = sp_eval_grad(F, s->fc[2 * i], s->fc[2 * i + 1], &s->grad[2 * i], &s->grad[2 * i + 1]);
    double sum = 0.0;
    for (int64_t i = 0; i < n; i++) sum += s->f[i];
    s->f_m = sum / (double)n;
    double ss = 0.0;
    for (int64_t i = 0; i < n; i++) ss += (s->f[i] - s->f_m) * (s->f[i] - s->f_m);
    s->delta_f = sqrt(ss);
    /* Subset::new rejects delta_f == 0 (src/subset.rs:888-892).  The FFT
     * prefilter leaves an exactly flat subset with delta_f ~ 1e-12 instead of
     * 0, so flatness is tested as sigma_f <= 1e-6 max(1, |f_m|) -- the same
     * test in every implementation of this library. */
    if (!(sqrt(ss / (double)n) > 1e-6 * fmax(1.0, fabs(s->f_m)))) return ST_FEATURELESS;
    double sg = 0.0;
    for (int64_t i = 0; i < n; i++) sg += 0.5 * (s->grad[2 * i] * s->grad[2 * i] + s->grad[2 * i + 1] * s->grad[2 * i + 1]);
    s->sssig = sg;
    s->sigma = sqrt(ss / (double)n);
    return ST_OK;
}

static void subset_free(subset_ref *s) { free(s->fc); free(s->f); free(s->grad); }

static void fill_failed(gpvo_result *r, const gpvo_desc *d, int len, int status) {
    memset(r, 0, sizeof(*r));
    for (int k = 0; k < len; k++) r->p[k] = d->p0[k];
    r->c_zncc = 0.0; r->c_znssd = 4.0; r->status = status;
}

/* One ICGN solve; hist (optional) receives max_iterations*3 doubles
 * (norm, zncc, znssd) per iteration. */
static void solve_one(const spline *F, const spline *G, const gpvo_desc *d, const gpvo_params *prm,
                      const uint8_t *mask, int64_t mh, int64_t mw, gpvo_result *r, double *hist) {
    int order = d->order;
    if (order < 0 || order > 2 || d->radius <= 0) { fill_failed(r, d, 12, ST_INVALID); return; }
    int m = p_len(order);
    subset_ref s;
    int st = subset_new(F, d->coord, d->radius, mask, mh, mw, &s);
    if (st != ST_OK) {
        fill_failed(r, d, m, st);
        r->n_px = (int32_t)s.n;
        r->f_m = s.f_m; r->delta_f = s.delta_f;
        subset_free(&s);
        return;
    }
    int64_t n = s.n;
    double size = sqrt((double)n);
    double *sdi = (double *)malloc(sizeof(double) * n * m);
    for (int64_t i = 0; i < n; i++)
        sdi_row(s.fc[2 * i] - d->coord[0], s.fc[2 * i + 1] - d->coord[1], s.grad[2 * i], s.grad[2 * i + 1], m, sdi + i * m);
    double H[144], Hi[144];
    for (int i = 0; i < m; i++)               /* compute_hessian (:348-364) */
        for (int j = i; j < m; j++) {
            double dot = 0.0;
            for (int64_t k = 0; k < n; k++) dot += sdi[k * m + i] * sdi[k * m + j];
            H[i * m + j] = dot; H[j * m + i] = dot;
        }
    memset(r, 0, sizeof(*r));
    r->n_px = (int32_t)n; r->f_m = s.f_m; r->delta_f = s.delta_f; r->sssig = s.sssig; r->sigma = s.sigma;
    if (!invert(H, m, Hi)) {
        fill_failed(r, d, m, ST_SINGULAR_H);
        r->n_px = (int32_t)n; r->f_m = s.f_m; r->delta_f = s.delta_f; r->sssig = s.sssig; r->sigma = s.sigma;
        free(sdi); subset_free(&s);
        return;
    }
    double p[12] = {0}, dp[12], pn[12], grad_z[12];
    for (int k = 0; k < m; k++) p[k] = d->p0[k];
    double *g = (double *)calloc(n, sizeof(double));
    int converged = 0, iters = 0, status = ST_OK;
    double last_norm = 0.0, c_zncc = 0.0, c_znssd = 4.0;
    /* rigid texture (grain_setup, src/subset.rs:1062-1097, the branch without
     * soil properties): the maps at the subset pixels, and the template
     * rebuilt from the current warp at every iteration */
    const int rigid = (prm->flags & 8) && order >= 1 && prm->grain;
    double *hmap = NULL, *tf = NULL, *off = NULL, tf_m = s.f_m, delta_tf = s.delta_f;
    const double *fv = s.f;
    if (rigid) {
        hmap = (double *)malloc(sizeof(double) * 3 * n);
        tf = (double *)malloc(sizeof(double) * n);
        off = (double *)malloc(sizeof(double) * 2 * n);
        for (int64_t i = 0; i < n; i++) {
            grain_sample(prm->grain, prm->gh, prm->gw, s.fc[2 * i], s.fc[2 * i + 1], hmap + 3 * i);
            off[2 * i] = s.fc[2 * i] - d->coord[0];
            off[2 * i + 1] = s.fc[2 * i + 1] - d->coord[1];
        }
        fv = tf;
    }
    for (int it = 1; it <= prm->max_iterations; it++) {
        if (rigid) rigid_template(s.f, s.f_m, hmap, prm->s2, p, m, off, n, tf, &tf_m, &delta_tf);
        for (int64_t i = 0; i < n; i++) {       /* apply_warp_into + eval (:1158-1161) */
            double xw, yw;
            warp_point(d->coord, p, m, s.fc[2 * i], s.fc[2 * i + 1], &xw, &yw);
            g[i] = sp_eval(G, xw, yw);
        }
        double gs = 0.0;
        for (int64_t i = 0; i < n; i++) gs += g[i];
        double g_m = gs / (double)n;
        double gss = 0.0;
        for (int64_t i = 0; i < n; i++) gss += (g[i] - g_m) * (g[i] - g_m);
        double delta_g = sqrt(gss);
        /* delta_p_and_znssd_icgn (:418-446), against the template when rigid */
        const double f_m_t = rigid ? tf_m : s.f_m, df_t = rigid ? delta_tf : s.delta_f;
        double ratio = df_t / delta_g, zacc = 0.0;
        for (int k = 0; k < m; k++) grad_z[k] = 0.0;
        for (int64_t i = 0; i < n; i++) {
            double a = fv[i] - f_m_t, b = g[i] - g_m;
            double z = a / df_t - b / delta_g;
            zacc += z * z;
            double br = a - ratio * b;
            for (int k = 0; k < m; k++) grad_z[k] += sdi[i * m + k] * br;
        }
        for (int k = 0; k < m; k++) {
            double acc = 0.0;
            for (int j = 0; j < m; j++) acc += Hi[k * m + j] * grad_z[j];
            dp[k] = -acc;
        }
        if (!gpvo_compose(p, dp, m, pn)) { status = ST_SINGULAR_WDELTA; break; }
        memcpy(p, pn, sizeof(double) * m);
        double nrm = gpvo_norm(dp, m, size);
        c_znssd = zacc;
        c_zncc = 1.0 - zacc / 2.0;
        iters = it;
        last_norm = nrm;
        if (hist) { hist[3 * (it - 1)] = nrm; hist[3 * (it - 1) + 1] = c_zncc; hist[3 * (it - 1) + 2] = zacc; }
        if (!isfinite(nrm)) { status = ST_NONFINITE; break; }
        if (nrm < prm->max_norm) { converged = 1; break; }
    }
    for (int k = 0; k < m; k++) r->p[k] = p[k];
    r->c_zncc = c_zncc; r->c_znssd = c_znssd; r->norm = last_norm;
    r->iterations = iters; r->converged = converged;
    r->quality_ok = converged && c_zncc >= prm->tolerance;
    r->status = status;
    if ((prm->flags & 1) && iters > 0 && status == ST_OK) {   /* eta (:1197-1210) */
        double gs = 0.0;
        for (int64_t i = 0; i < n; i++) gs += g[i];
        double g_m = gs / (double)n, gss = 0.0;
        for (int64_t i = 0; i < n; i++) gss += (g[i] - g_m) * (g[i] - g_m);
        gpvo_eta(d->coord, order, s.fc, s.grad, fv, rigid ? tf_m : s.f_m, rigid ? delta_tf : s.delta_f, g, g_m,
                 sqrt(gss), n, &r->eta_u, &r->eta_v);
        r->has_eta = 1;
    }
    r->texture = rigid;
    free(g); free(sdi); subset_free(&s);
    free(hmap); free(tf); free(off);
}

/* Subset::solve_fagn_result (src/subset.rs:1228-1334): per iteration the
 * target value and gradient at the warped positions, g_m and delta_g, the
 * steepest-descent images from the target gradient about the warped centre
 * coord + (u, v), H = SDI^T SDI, delta_p_fagn (:452-473), p += dp. */
static void solve_one_fagn(const spline *F, const spline *G, const gpvo_desc *d, const gpvo_params *prm,
                           const uint8_t *mask, int64_t mh, int64_t mw, gpvo_result *r, double *hist) {
    int order = d->order;
    if (order < 0 || order > 2 || d->radius <= 0) { fill_failed(r, d, 12, ST_INVALID); return; }
    int m = p_len(order);
    subset_ref s;
    int st = subset_new(F, d->coord, d->radius, mask, mh, mw, &s);
    if (st != ST_OK) {
        fill_failed(r, d, m, st);
        r->n_px = (int32_t)s.n;
        r->f_m = s.f_m; r->delta_f = s.delta_f;
        subset_free(&s);
        return;
    }
    int64_t n = s.n;
    double size = sqrt((double)n);
    double *sdi = (double *)malloc(sizeof(double) * n * m);
    double *g = (double *)calloc(n, sizeof(double));
    double *gc = (double *)malloc(sizeof(double) * 2 * n);
    double *gg = (double *)malloc(sizeof(double) * 2 * n);
    memset(r, 0, sizeof(*r));
    r->n_px = (int32_t)n; r->f_m = s.f_m; r->delta_f = s.delta_f; r->sssig = s.sssig; r->sigma = s.sigma;
    double p[12] = {0}, dp[12], grad_z[12], H[144], Hi[144];
    for (int k = 0; k < m; k++) p[k] = d->p0[k];
    int converged = 0, iters = 0, status = ST_OK;
    double last_norm = 0.0, c_zncc = 0.0, c_znssd = 4.0;
    /* rigid texture (src/subset.rs:1257-1262): the template rebuilt from the
     * current warp at every iteration, in place of f, f_m, delta_f */
    const int rigid = (prm->flags & 8) && order >= 1 && prm->grain;
    double *hmap = NULL, *tf = NULL, *off = NULL, tf_m = s.f_m, delta_tf = s.delta_f;
    const double *fv = s.f;
    if (rigid) {
        hmap = (double *)malloc(sizeof(double) * 3 * n);
        tf = (double *)malloc(sizeof(double) * n);
        off = (double *)malloc(sizeof(double) * 2 * n);
        for (int64_t i = 0; i < n; i++) {
            grain_sample(prm->grain, prm->gh, prm->gw, s.fc[2 * i], s.fc[2 * i + 1], hmap + 3 * i);
            off[2 * i] = s.fc[2 * i] - d->coord[0];
            off[2 * i + 1] = s.fc[2 * i + 1] - d->coord[1];
        }
        fv = tf;
    }
    for (int it = 1; it <= prm->max_iterations; it++) {
        if (rigid) rigid_template(s.f, s.f_m, hmap, prm->s2, p, m, off, n, tf, &tf_m, &delta_tf);
        const double f_m_t = rigid ? tf_m : s.f_m, df_t = rigid ? delta_tf : s.delta_f;
        double g_center[2] = {d->coord[0] + p[0], d->coord[1] + p[1]};
        for (int64_t i = 0; i < n; i++) {
            warp_point(d->coord, p, m, s.fc[2 * i], s.fc[2 * i + 1], &gc[2 * i], &gc[2 * i + 1]);
            g[i] = sp_eval_grad(G, gc[2 * i], gc[2 * i + 1], &gg[2 * i], &gg[2 * i + 1]);
        }
        double gs = 0.0;
        for (int64_t i = 0; i < n; i++) gs += g[i];
        double g_m = gs / (double)n, gss = 0.0;
        for (int64_t i = 0; i < n; i++) gss += (g[i] - g_m) * (g[i] - g_m);
        double delta_g = sqrt(gss);
        for (int64_t i = 0; i < n; i++)
            sdi_row(gc[2 * i] - g_center[0], gc[2 * i + 1] - g_center[1], gg[2 * i], gg[2 * i + 1], m, sdi + i * m);
        for (int a = 0; a < m; a++)
            for (int b = a; b < m; b++) {
                double dot = 0.0;
                for (int64_t k = 0; k < n; k++) dot += sdi[k * m + a] * sdi[k * m + b];
                H[a * m + b] = dot; H[b * m + a] = dot;
            }
        for (int k = 0; k < m; k++) grad_z[k] = 0.0;
        for (int k = 0; k < m; k++)
            for (int64_t i = 0; i < n; i++)
                grad_z[k] += sdi[i * m + k] * ((fv[i] - f_m_t) * (delta_g / df_t) - (g[i] - g_m));
        if (!invert(H, m, Hi)) { status = ST_SINGULAR_H; break; }  /* the reference panics */
        for (int k = 0; k < m; k++) {
            double acc = 0.0;
            for (int j = 0; j < m; j++) acc += Hi[k * m + j] * grad_z[j];
            dp[k] = acc;
        }
        for (int k = 0; k < m; k++) p[k] += dp[k];
        double nrm = gpvo_norm(dp, m, size);
        double z = gpvo_znssd(fv, g, n, f_m_t, g_m, df_t, delta_g);
        c_znssd = z;
        c_zncc = 1.0 - z / 2.0;
        iters = it;
        last_norm = nrm;
        if (hist) { hist[3 * (it - 1)] = nrm; hist[3 * (it - 1) + 1] = c_zncc; hist[3 * (it - 1) + 2] = z; }
        if (!isfinite(nrm)) { status = ST_NONFINITE; break; }
        if (nrm < prm->max_norm) { converged = 1; break; }
    }
    for (int k = 0; k < m; k++) r->p[k] = p[k];
    r->c_zncc = c_zncc; r->c_znssd = c_znssd; r->norm = last_norm;
    r->iterations = iters; r->converged = converged;
    r->quality_ok = converged && c_zncc >= prm->tolerance;
    r->status = status;
    if ((prm->flags & 1) && iters > 0 && status == ST_OK) {
        double gs = 0.0;
        for (int64_t i = 0; i < n; i++) gs += g[i];
        double g_m = gs / (double)n, gss = 0.0;
        for (int64_t i = 0; i < n; i++) gss += (g[i] - g_m) * (g[i] - g_m);
        gpvo_eta(d->coord, order, s.fc, s.grad, fv, rigid ? tf_m : s.f_m, rigid ? delta_tf : s.delta_f, g, g_m,
                 sqrt(gss), n, &r->eta_u, &r->eta_v);
        r->has_eta = 1;
    }
    r->texture = rigid;
    free(sdi); free(g); free(gc); free(gg); subset_free(&s);
    free(hmap); free(tf); free(off);
}

/* load_grayscale + gaussian_blur_5x5 (src/image.rs:450-534) on decoded RGB8
 * pixels: integer grey level, 5-tap Gaussian (sigma 1.1) horizontal then
 * vertical with BORDER_REFLECT_101 indices, FP64 left-to-right sums, rounding
 * half away from zero, clamp to 0..255.  h, w >= 3. */
static int64_t reflect101(int64_t i, int64_t n) { return i < 0 ? -i : (i >= n ? 2 * (n - 1) - i : i); }

void gpvo_ingest_rgb8(const uint8_t *rgb, int64_t h, int64_t w, uint8_t *out) {
    double raw[5], k[5], sum = 0.0;
    for (int i = 0; i < 5; i++) {
        double x = (double)i - 2.0;
        raw[i] = exp(-x * x / (2.0 * 1.1 * 1.1));
    }
    for (int i = 0; i < 5; i++) sum += raw[i];
    for (int i = 0; i < 5; i++) k[i] = raw[i] / sum;
    double *gs = (double *)malloc(sizeof(double) * h * w), *hp = (double *)malloc(sizeof(double) * h * w);
    for (int64_t i = 0; i < h * w; i++) {
        const uint8_t *p = rgb + 3 * i;
        gs[i] = (double)((2126u * p[0] + 7152u * p[1] + 722u * p[2] + 5000u) / 10000u);
    }
    for (int64_t i = 0; i < h; i++)
        for (int64_t j = 0; j < w; j++) {
            double v = 0.0;
            for (int q = 0; q < 5; q++) v += k[q] * gs[i * w + reflect101(j + q - 2, w)];
            hp[i * w + j] = v;
        }
    for (int64_t i = 0; i < h; i++)
        for (int64_t j = 0; j < w; j++) {
            double v = 0.0;
            for (int q = 0; q < 5; q++) v += k[q] * hp[reflect101(i + q - 2, h) * w + j];
            v = round(v);
            out[i * w + j] = (uint8_t)(v < 0.0 ? 0.0 : (v > 255.0 ? 255.0 : v));
        }
    free(gs); free(hp);
}

/* Batch entry: nthreads OpenMP workers, one subset per task (dynamic). */
void gpvo_solve_batch(const double *cf, const double *cg, int64_t h, int64_t w, int64_t border,
                      const gpvo_desc *desc, int64_t n, const gpvo_params *prm, const uint8_t *mask,
                      gpvo_result *out, double *history, int nthreads) {
    spline F = {cf, h, w, border, w + 2 * border};
    spline G = {cg, h, w, border, w + 2 * border};
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int64_t i = 0; i < n; i++) {
        double *hi = history ? history + i * (int64_t)prm->max_iterations * 3 : NULL;
        if (prm->flags & 4)
            solve_one_fagn(&F, &G, &desc[i], prm, mask, h, w, &out[i], hi);
        else
            solve_one(&F, &G, &desc[i], prm, mask, h, w, &out[i], hi);
    }
}

/* Reference-subset quantities only (Subset::new), for the setup parity tests. */
int gpvo_subset_setup(const double *cf, int64_t h, int64_t w, int64_t border, const double coord[2], int64_t radius,
                      const uint8_t *mask, double *f_out, double *grad_out, double *scalars /* f_m, df, sssig, sigma */,
                      int64_t *n_out) {
    spline F = {cf, h, w, border, w + 2 * border};
    subset_ref s;
    int st = subset_new(&F, coord, radius, mask, h, w, &s);
    *n_out = s.n;
    if (s.f && f_out) memcpy(f_out, s.f, sizeof(double) * s.n);
    if (s.grad && grad_out) memcpy(grad_out, s.grad, sizeof(double) * 2 * s.n);
    scalars[0] = s.f_m; scalars[1] = s.delta_f; scalars[2] = s.sssig; scalars[3] = s.sigma;
    subset_free(&s);
    return st;
}

int gpvo_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
