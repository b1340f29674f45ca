/*
 * synth.c -- seeded synthetic speckle pairs for tests and benchmarks.
 *
 * Not part of the solve path: it only manufactures inputs.  Model (this
 * project's own generator, stated here in full):
 *   - Speckle: uniform random centres over the image; blob radius r ~ U[2,4]
 *     px; blob = exp(-d^2 / r^2) (r is the 1/e half-width); blobs are added
 *     until sum(pi r^2) reaches `coverage` of the image area.  Intensity =
 *     scale * (30 + 170 * min(1, sum of blobs)).
 *   - Reference image: intensity + N(0, sigma) noise, rounded, clamped to
 *     [0, maxval].
 *   - Target image: the bi-quintic B-spline interpolant of the noise-free
 *     reference intensity (replicate border 20, circular deconvolution by
 *     the quintic kernel), sampled at the inverse-mapped position X with
 *     x = X + u(X) (fixed point, 5 passes), plus independent noise,
 *     quantised the same way.
 * Every random draw comes from a counter-based hash of (seed, stream,
 * index), so the output is independent of the thread count.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline double u01(uint64_t seed, uint64_t stream, uint64_t idx) {
    uint64_t z = mix64(seed * 0xD1B54A32D192ED03ull ^ mix64(stream * 0x8CB92BA72F3D8DD7ull + idx));
    return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static inline double gauss(uint64_t seed, uint64_t stream, uint64_t idx) {
    double a = u01(seed, stream, 2 * idx), b = u01(seed, stream, 2 * idx + 1);
    return sqrt(-2.0 * log(a)) * cos(2.0 * M_PI * b);
}

typedef struct { double x, y, r; } blob;

static int cmp_blob(const void *a, const void *b) {
    double ya = ((const blob *)a)->y, yb = ((const blob *)b)->y;
    return (ya > yb) - (ya < yb);
}

/* Noise-free speckle intensity (h, w), FP64. Returns the number of blobs. */
int64_t gpv_synth_speckle(int64_t h, int64_t w, uint64_t seed, double coverage, double scale, double *out) {
    double target = coverage * (double)h * (double)w, area = 0.0;
    int64_t cap = (int64_t)(target / (M_PI * 4.0)) + 16, n = 0;
    blob *b = (blob *)malloc(sizeof(blob) * cap);
    while (area < target) {
        if (n == cap) { cap *= 2; b = (blob *)realloc(b, sizeof(blob) * cap); }
        b[n].x = u01(seed, 1, 3 * n) * (double)w;
        b[n].y = u01(seed, 1, 3 * n + 1) * (double)h;
        b[n].r = 2.0 + 2.0 * u01(seed, 1, 3 * n + 2);
        area += M_PI * b[n].r * b[n].r;
        n++;
    }
    qsort(b, n, sizeof(blob), cmp_blob);
    const double reach = 4.0 * 4.0; /* 4 radii: exp(-16) ~ 1e-7 */
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t y = 0; y < h; y++) {
        double *row = out + y * w;
        for (int64_t x = 0; x < w; x++) row[x] = 0.0;
        /* first blob with b.y >= y - reach */
        int64_t lo = 0, hi = n;
        while (lo < hi) { int64_t mid = (lo + hi) / 2; if (b[mid].y < (double)y - reach) lo = mid + 1; else hi = mid; }
        for (int64_t k = lo; k < n && b[k].y <= (double)y + reach; k++) {
            double dy = (double)y - b[k].y, r = b[k].r, cut = 4.0 * r;
            if (fabs(dy) > cut) continue;
            int64_t x0 = (int64_t)floor(b[k].x - cut), x1 = (int64_t)ceil(b[k].x + cut);
            if (x0 < 0) x0 = 0;
            if (x1 > w - 1) x1 = w - 1;
            double inv = 1.0 / (r * r);
            for (int64_t x = x0; x <= x1; x++) {
                double dx = (double)x - b[k].x;
                row[x] += exp(-(dx * dx + dy * dy) * inv);
            }
        }
        for (int64_t x = 0; x < w; x++) row[x] = scale * (30.0 + 170.0 * (row[x] < 1.0 ? row[x] : 1.0));
    }
    free(b);
    return n;
}

/* Add N(0, sigma) noise (stream `stream`), round, clamp to [0, maxval].
 * dtype 1: uint8 out, 2: uint16 out. */
void gpv_synth_quantize(const double *in, int64_t n, double sigma, uint64_t seed, uint64_t stream, double maxval,
                        int dtype, void *out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        double v = in[i] + sigma * gauss(seed, stream, (uint64_t)i);
        v = nearbyint(v);
        v = v < 0.0 ? 0.0 : (v > maxval ? maxval : v);
        if (dtype == 1) ((uint8_t *)out)[i] = (uint8_t)v;
        else ((uint16_t *)out)[i] = (uint16_t)v;
    }
}

/* ---------------- B-spline interpolant (FP64) ---------------- */

/* Taps h[m], |m| <= M, of the periodised inverse of the quintic kernel for
 * circular length N: h[m] = (1/N) sum_j cos(2 pi j m / N) / K(2 pi j / N),
 * K(w) = 11/20 + 13/30 cos w + 1/60 cos 2w. */
static void inverse_taps(int64_t N, int M, double *h) {
    for (int m = -M; m <= M; m++) {
        double acc = 0.0;
        for (int64_t j = 0; j < N; j++) {
            double wj = 2.0 * M_PI * (double)j / (double)N;
            double K = 11.0 / 20.0 + (13.0 / 30.0) * cos(wj) + (1.0 / 60.0) * cos(2.0 * wj);
            acc += cos(wj * (double)m) / K;
        }
        h[m + M] = acc / (double)N;
    }
}

/* Circular deconvolution of lines of length N (stride `stride` between
 * elements, `lstride` between lines) in place via buffer. */
static void deconv_axis(double *a, int64_t nlines, int64_t N, int64_t stride, int64_t lstride) {
    int M = 44;
    if (2 * M + 1 > N) M = (int)((N - 1) / 2);
    double *h = (double *)malloc(sizeof(double) * (2 * M + 1));
    inverse_taps(N, M, h);
#pragma omp parallel
    {
        /* the line extended by M samples of circular wrap on each side */
        double *buf = (double *)malloc(sizeof(double) * (N + 2 * M));
#pragma omp for schedule(static)
        for (int64_t l = 0; l < nlines; l++) {
            double *line = a + l * lstride;
            for (int64_t i = -M; i < N + M; i++) buf[i + M] = line[(((i % N) + N) % N) * stride];
            for (int64_t i = 0; i < N; i++) {
                double acc = 0.0;
                for (int m = -M; m <= M; m++) acc += h[m + M] * buf[i - m + M];
                line[i * stride] = acc;
            }
        }
        free(buf);
    }
    free(h);
}

static void qt(double t, double o[6]) {
    double s = 1.0 - t;
    double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
    o[0] = s * s * s * s * s / 120.0;
    o[1] = (26.0 - 50.0 * t + 20.0 * t2 + 20.0 * t3 - 20.0 * t4 + 5.0 * t5) / 120.0;
    o[2] = (66.0 - 60.0 * t2 + 30.0 * t4 - 10.0 * t5) / 120.0;
    o[3] = (26.0 + 50.0 * t + 20.0 * t2 - 20.0 * t3 - 20.0 * t4 + 10.0 * t5) / 120.0;
    o[4] = (1.0 + 5.0 * t + 10.0 * t2 + 10.0 * t3 + 5.0 * t4 - 5.0 * t5) / 120.0;
    o[5] = t5 / 120.0;
}

typedef struct {
    double xc, yc;            /* field origin */
    double t[2];              /* translation */
    double a[4];              /* du/dx, du/dy, dv/dx, dv/dy */
    double q[6];              /* u: dx^2, dx dy, dy^2 ; v: dx^2, dx dy, dy^2 */
    double band_amp, band_y, band_w; /* u += amp * tanh((y - band_y) / band_w) */
} gpv_field;

static inline void field_eval(const gpv_field *F, double x, double y, double *u, double *v) {
    double dx = x - F->xc, dy = y - F->yc;
    *u = F->t[0] + F->a[0] * dx + F->a[1] * dy + F->q[0] * dx * dx + F->q[1] * dx * dy + F->q[2] * dy * dy;
    *v = F->t[1] + F->a[2] * dx + F->a[3] * dy + F->q[3] * dx * dx + F->q[4] * dx * dy + F->q[5] * dy * dy;
    if (F->band_w != 0.0) *u += F->band_amp * tanh((y - F->band_y) / F->band_w);
}

/* Displacement field u(x) at points (for truth values). */
void gpv_synth_field(const gpv_field *F, const double *xy, int64_t n, double *uv) {
    for (int64_t i = 0; i < n; i++) field_eval(F, xy[2 * i], xy[2 * i + 1], &uv[2 * i], &uv[2 * i + 1]);
}

/* Target intensity: S_ref(X) with x = X + u(X), for every pixel (h, w). */
void gpv_synth_warp(const double *ref, int64_t h, int64_t w, const gpv_field *F, double *out) {
    const int64_t b = 20, pr = h + 2 * b, pc = w + 2 * b;
    double *c = (double *)malloc(sizeof(double) * pr * pc);
    for (int64_t i = 0; i < pr; i++) {
        int64_t ri = i < b ? 0 : (i - b > h - 1 ? h - 1 : i - b);
        for (int64_t j = 0; j < pc; j++) {
            int64_t ci = j < b ? 0 : (j - b > w - 1 ? w - 1 : j - b);
            c[i * pc + j] = ref[ri * w + ci];
        }
    }
    deconv_axis(c, pr, pc, 1, pc);
    deconv_axis(c, pc, pr, pc, 1);
#pragma omp parallel for schedule(static)
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) {
            double X = (double)x, Y = (double)y, u, v;
            for (int it = 0; it < 5; it++) {
                field_eval(F, X, Y, &u, &v);
                X = (double)x - u;
                Y = (double)y - v;
            }
            double xx = X < 0.0 ? 0.0 : (X > (double)w - 1e-9 ? (double)w - 1e-9 : X);
            double yy = Y < 0.0 ? 0.0 : (Y > (double)h - 1e-9 ? (double)h - 1e-9 : Y);
            double xf = floor(xx), yf = floor(yy), ax[6], ay[6];
            qt(xx - xf, ax);
            qt(yy - yf, ay);
            int64_t r0 = (int64_t)yf + b - 2, c0 = (int64_t)xf + b - 2;
            double val = 0.0;
            for (int r = 0; r < 6; r++) {
                const double *row = c + (r0 + r) * pc + c0;
                double s = 0.0;
                for (int k = 0; k < 6; k++) s += row[k] * ax[k];
                val += ay[r] * s;
            }
            out[y * w + x] = val;
        }
    free(c);
}
