// icgn_common.cuh -- device pieces shared by the ICGN solve kernels.
//
// Reference: src/subset.rs (Subset::new :836-919, solve_icgn_result
// :1117-1219, apply_warp_into :262-300, steepest_descent :311-343,
// compute_hessian :348-364, compose_icgn :487-611, convergence_norm
// :622-649, omitted_mode_diagnostic :698-820) and src/masks.rs:199-263.
#pragma once
#include <cfloat>
#include <cmath>

#include "internal.h"
#include "spline.cuh"

namespace gpv {

// Arguments of every solve kernel (host-filled, passed by value).
struct KArgs {
    const float *f32, *g32;
    const double *f64, *g64;
    int64_t pitch32, pitch64;
    int h, w, border;
    const gpv_subset_desc *desc;
    const int32_t *order;
    int n;
    const short2 *offs;
    const short2 *slots;             // padded templates (rows padded to 32 lanes)
    const int32_t *tab_off, *tab_n;  // [0, R]: compact templates, [R+1, 2R+1]: slot tables
    int table_radius;
    int max_radius;
    const uint8_t *mask;
    int mh, mw;
    double max_norm, tolerance;
    int max_iter, flags;
    gpv_subset_result *out;
    double *history;
    void *scratch;
    int64_t scratch_stride;  // elements (float for mixed, double for fp64) per worker
    int *queue;
    const float *grain = nullptr;        // rigid texture: f's grain maps (3 x h x w)
    const double *grain64 = nullptr;     // the same in FP64, or null
    const double *grain_scal = nullptr;  // [mean, correlation length, s2, corr, built]
};

namespace {

constexpr int kMixedWarps = 8;  // warps per block of the mixed kernel
constexpr int kChunk = 8;       // pixels per lane between FP64 flushes
constexpr int kFp64Threads = 256;
constexpr int kFp64Warps = kFp64Threads / 32;


template <int ORDER>
struct Ord {
    static constexpr int M = ORDER == 0 ? 2 : (ORDER == 1 ? 6 : 12);  // parameters
    static constexpr int NMU = M / 2;                                 // SDI monomials per gradient axis
    static constexpr int DEG = ORDER;                                 // degree of the warp monomials
    static constexpr int NMOM = (2 * DEG + 1) * (2 * DEG + 2) / 2;    // monomials of degree <= 2*DEG
};

// SDI monomial mu (src/subset.rs:324-340): 1, dx, dy, dx^2/2, dx dy, dy^2/2
__host__ __device__ constexpr int mu_a(int mu) { return mu == 1 ? 1 : (mu == 3 ? 2 : (mu == 4 ? 1 : 0)); }
__host__ __device__ constexpr int mu_b(int mu) { return mu == 2 ? 1 : (mu == 4 ? 1 : (mu == 5 ? 2 : 0)); }
__host__ __device__ constexpr double mu_c(int mu) { return (mu == 3 || mu == 5) ? 0.5 : 1.0; }
// index of monomial dx^a dy^b among those of degree <= D, ordered by degree then b
__host__ __device__ constexpr int mom_idx(int a, int b) { return (a + b) * (a + b + 1) / 2 + b; }

template <typename T>
__device__ __forceinline__ T mu_val(int mu, T dx, T dy) {
    switch (mu) {
        case 0: return T(1);
        case 1: return dx;
        case 2: return dy;
        case 3: return T(0.5) * dx * dx;
        case 4: return dx * dy;
        default: return T(0.5) * dy * dy;
    }
}

// Flatness (Subset::new, src/subset.rs:888-892, rejects delta_f == 0): the
// prefilter's rounding leaves an exactly flat subset with delta_f ~ 1e-12 (FP64)
// or ~1e-4 (FP32) instead of 0, so a subset is featureless when
// sigma_f = delta_f / sqrt(n) <= 1e-6 max(1, |f_m|) -- in the oracle too.

// Global-mask test of LocalMask::mask_update (src/masks.rs:199-263): the
// template pixel maps to image pixel trunc(centre) + offset; the extracted
// window always stops one short of the last mask row / column.
__device__ __forceinline__ bool mask_ok(const KArgs &A, int cxi, int cyi, int ox, int oy) {
    if (!A.mask) return true;
    const int X = cxi + ox, Y = cyi + oy;
    if (X < 0 || Y < 0 || X > A.mw - 2 || Y > A.mh - 2) return false;
    return A.mask[(int64_t)Y * A.mw + X] != 0;
}

// ---------------------------------------------------------------------
// Warp composition (compose_icgn, src/subset.rs:487-611) in FP64.
// Order 2 needs only rows 3 and 4 of W_old * W_delta^-1 (the u and v rows
// that hold the 12 parameters); they are the solution Y of Y W_delta = R,
// R = rows 3, 4 of W_old.  Returns false if W_delta is singular.
// ---------------------------------------------------------------------
__device__ bool compose1(const double *p, const double *d, double *out) {
    const double a = 1.0 + d[2], b = d[4], c = d[3], e = 1.0 + d[5];
    const double det = a * e - b * c;
    if (det == 0.0 || !isfinite(det)) return false;
    const double ia = e / det, ib = -b / det, ic = -c / det, ie = a / det;
    // W_delta^-1 = [[ia, ib, -(ia du + ib dv)], [ic, ie, -(ic du + ie dv)], [0, 0, 1]]
    const double tx = -(ia * d[0] + ib * d[1]), ty = -(ic * d[0] + ie * d[1]);
    const double B00 = 1.0 + p[2], B01 = p[4], B10 = p[3], B11 = 1.0 + p[5];
    const double n00 = B00 * ia + B01 * ic, n01 = B00 * ib + B01 * ie;
    const double n10 = B10 * ia + B11 * ic, n11 = B10 * ib + B11 * ie;
    out[0] = B00 * tx + B01 * ty + p[0];
    out[1] = B10 * tx + B11 * ty + p[1];
    out[2] = n00 - 1.0;
    out[3] = n10;
    out[4] = n01;
    out[5] = n11 - 1.0;
    return true;
}

// Lifted 6x6 warp of an order-2 parameter vector on [x^2, xy, y^2, x, y, 1]
// (src/subset.rs:547-593); W is row-major 36 doubles.
__device__ __forceinline__ void lifted(const double *q, double *W) {
    const double u = q[0], v = q[1], ux = q[2], vx = q[3], uy = q[4], vy = q[5];
    const double uxx = q[6], vxx = q[7], uxy = q[8], vxy = q[9], uyy = q[10], vyy = q[11];
    W[0] = 1.0 + 2.0 * ux + ux * ux + u * uxx;
    W[1] = 2.0 * u * uxy + 2.0 * (1.0 + ux) * uy;
    W[2] = uy * uy + u * uyy;
    W[3] = 2.0 * u * (1.0 + ux);
    W[4] = 2.0 * u * uy;
    W[5] = u * u;
    W[6] = 0.5 * (v * uxx + 2.0 * (1.0 + ux) * vx + u * vxx);
    W[7] = 1.0 + uy * vx + ux * vy + v * uxy + u * vxy + vy + ux;
    W[8] = 0.5 * (v * uyy + 2.0 * uy * (1.0 + vy) + u * vyy);
    W[9] = v + v * ux + u * vx;
    W[10] = u + v * uy + u * vy;
    W[11] = u * v;
    W[12] = vx * vx + v * vxx;
    W[13] = 2.0 * v * vxy + 2.0 * vx * (1.0 + vy);
    W[14] = 1.0 + 2.0 * vy + vy * vy + v * vyy;
    W[15] = 2.0 * v * vx;
    W[16] = 2.0 * v * (1.0 + vy);
    W[17] = v * v;
    W[18] = 0.5 * uxx; W[19] = uxy; W[20] = 0.5 * uyy; W[21] = 1.0 + ux; W[22] = uy; W[23] = u;
    W[24] = 0.5 * vxx; W[25] = vxy; W[26] = 0.5 * vyy; W[27] = vx; W[28] = 1.0 + vy; W[29] = v;
    W[30] = 0.0; W[31] = 0.0; W[32] = 0.0; W[33] = 0.0; W[34] = 0.0; W[35] = 1.0;
}

// Order-2 composition by one thread; LU with partial pivoting of W_delta^T.
// ws: 96 doubles of scratch (shared or local memory).
__device__ __noinline__ bool compose2(const double *p, const double *d, double *out, double *ws) {
    double *A = ws, *X = ws + 36, *W = ws + 48;  // A = W_delta^T, X = [R^T] (6x2), W: scratch 6x6
    lifted(d, W);
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) A[i * 6 + j] = W[j * 6 + i];
    // R = rows 3, 4 of W_old: [0.5 uxx, uxy, 0.5 uyy, 1+ux, uy, u] and the v row
    X[0] = 0.5 * p[6]; X[1] = 0.5 * p[7];
    X[2] = p[8];       X[3] = p[9];
    X[4] = 0.5 * p[10]; X[5] = 0.5 * p[11];
    X[6] = 1.0 + p[2]; X[7] = p[3];
    X[8] = p[4];       X[9] = 1.0 + p[5];
    X[10] = p[0];      X[11] = p[1];
    for (int k = 0; k < 6; k++) {
        int piv = k;
        double best = fabs(A[k * 6 + k]);
        for (int i = k + 1; i < 6; i++)
            if (fabs(A[i * 6 + k]) > best) { best = fabs(A[i * 6 + k]); piv = i; }
        if (!(best > 0.0) || !isfinite(best)) return false;
        if (piv != k) {
            for (int j = 0; j < 6; j++) { double t = A[k * 6 + j]; A[k * 6 + j] = A[piv * 6 + j]; A[piv * 6 + j] = t; }
            for (int j = 0; j < 2; j++) { double t = X[k * 2 + j]; X[k * 2 + j] = X[piv * 2 + j]; X[piv * 2 + j] = t; }
        }
        const double inv = 1.0 / A[k * 6 + k];
        for (int i = k + 1; i < 6; i++) {
            const double f = A[i * 6 + k] * inv;
            if (f == 0.0) continue;
            for (int j = k; j < 6; j++) A[i * 6 + j] -= f * A[k * 6 + j];
            X[i * 2] -= f * X[k * 2];
            X[i * 2 + 1] -= f * X[k * 2 + 1];
        }
    }
    for (int k = 5; k >= 0; k--) {
        for (int j = k + 1; j < 6; j++) {
            X[k * 2] -= A[k * 6 + j] * X[j * 2];
            X[k * 2 + 1] -= A[k * 6 + j] * X[j * 2 + 1];
        }
        X[k * 2] /= A[k * 6 + k];
        X[k * 2 + 1] /= A[k * 6 + k];
    }
    // row 3 of W_new = X[:, 0], row 4 = X[:, 1]
    out[0] = X[10]; out[1] = X[11];
    out[2] = X[6] - 1.0; out[3] = X[7];
    out[4] = X[8]; out[5] = X[9] - 1.0;
    out[6] = 2.0 * X[0]; out[7] = 2.0 * X[1];
    out[8] = X[2]; out[9] = X[3];
    out[10] = 2.0 * X[4]; out[11] = 2.0 * X[5];
    return true;
}

// Order-2 composition in registers, fully unrolled: solve W_delta^T X = R^T
// by Gaussian elimination without pivoting.  The lifted warp of a
// translation is unit upper triangular, and with strain / curvature terms of
// an increment it stays close to that, so the pivots stay near 1; a zero or
// non-finite pivot reports W_delta singular.
__device__ __forceinline__ bool compose2_regs(const double *p, const double *d, double *out) {
    double W[36];
    lifted(d, W);
    double A[6][6], X[6][2];
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
        for (int j = 0; j < 6; j++) A[i][j] = W[j * 6 + i];
    X[0][0] = 0.5 * p[6]; X[0][1] = 0.5 * p[7];
    X[1][0] = p[8];       X[1][1] = p[9];
    X[2][0] = 0.5 * p[10]; X[2][1] = 0.5 * p[11];
    X[3][0] = 1.0 + p[2]; X[3][1] = p[3];
    X[4][0] = p[4];       X[4][1] = 1.0 + p[5];
    X[5][0] = p[0];       X[5][1] = p[1];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const double piv = A[k][k];
        ok = ok && (piv != 0.0) && isfinite(piv);
        const double inv = __drcp_rn(piv);  // the correctly rounded 1 / piv, without a general division
#pragma unroll
        for (int i = k + 1; i < 6; i++) {
            const double f = A[i][k] * inv;
#pragma unroll
            for (int j = k + 1; j < 6; j++) A[i][j] = fma(-f, A[k][j], A[i][j]);
            X[i][0] = fma(-f, X[k][0], X[i][0]);
            X[i][1] = fma(-f, X[k][1], X[i][1]);
        }
    }
#pragma unroll
    for (int k = 5; k >= 0; k--) {
#pragma unroll
        for (int j = k + 1; j < 6; j++) {
            X[k][0] = fma(-A[k][j], X[j][0], X[k][0]);
            X[k][1] = fma(-A[k][j], X[j][1], X[k][1]);
        }
        const double inv = __drcp_rn(A[k][k]);
        X[k][0] *= inv;
        X[k][1] *= inv;
    }
    out[0] = X[5][0]; out[1] = X[5][1];
    out[2] = X[3][0] - 1.0; out[3] = X[3][1];
    out[4] = X[4][0]; out[5] = X[4][1] - 1.0;
    out[6] = 2.0 * X[0][0]; out[7] = 2.0 * X[0][1];
    out[8] = X[1][0]; out[9] = X[1][1];
    out[10] = 2.0 * X[2][0]; out[11] = 2.0 * X[2][1];
    return ok;
}

template <int M>
__device__ double conv_norm(const double *dp, double size) {
    if (M == 2) return sqrt(dp[0] * dp[0] + dp[1] * dp[1]);
    double s = dp[0] * dp[0] + dp[1] * dp[1];
#pragma unroll
    for (int k = 2; k < 6; k++) s += (dp[k] * size) * (dp[k] * size);
    if (M == 12) {
#pragma unroll
        for (int k = 6; k < 12; k++) {
            const double t = 0.5 * dp[k] * size * size;
            s += t * t;
        }
    }
    return sqrt(s);
}

// Lane-parallel Gauss-Jordan inverse of the Jacobi-scaled SPD Hessian, in
// shared memory (lane c owns column c of the augmented [H~ | I]).
// H: M*M (in), aug: M*2M scratch, Hinv: M*M (out).  Returns false when a
// pivot is not positive (singular Hessian).  Warp-uniform result.
template <int M>
__device__ bool spd_inverse_warp(const double *H, double *aug, double *Hinv, int lane) {
    constexpr int W2 = 2 * M;
    bool ok = true;
    for (int i = 0; i < M; i++) ok = ok && (H[i * M + i] > 0.0) && isfinite(H[i * M + i]);
    if (!ok) return false;
    for (int e = lane; e < M * W2; e += 32) {
        const int i = e / W2, c = e % W2;
        aug[e] = c < M ? H[i * M + c] / sqrt(H[i * M + i] * H[c * M + c]) : (c - M == i ? 1.0 : 0.0);
    }
    __syncwarp();
    for (int k = 0; k < M; k++) {
        const double piv = aug[k * W2 + k];
        if (!(piv > 0.0) || !isfinite(piv)) return false;  // uniform (same smem value)
        const int c = lane;
        double rk = 0.0;
        if (c < W2) rk = aug[k * W2 + c] / piv;
        if (c < W2 && c != k) {
            for (int i = 0; i < M; i++)
                if (i != k) aug[i * W2 + c] = fma(-aug[i * W2 + k], rk, aug[i * W2 + c]);
        }
        __syncwarp();
        if (c < W2) aug[k * W2 + c] = rk;
        if (c == k)
            for (int i = 0; i < M; i++)
                if (i != k) aug[i * W2 + k] = 0.0;
        __syncwarp();
    }
    for (int e = lane; e < M * M; e += 32) {
        const int i = e / M, c = e % M;
        Hinv[e] = aug[i * W2 + M + c] / sqrt(H[i * M + i] * H[c * M + c]);
    }
    __syncwarp();
    return true;
}

// Assemble H (M x M) from gradient moments mom[pair][NMOM] (pair 0 = gx gx,
// 1 = gx gy, 2 = gy gy): H[j][k] = c_j c_k sum g_cj g_ck mu_j mu_k.
template <int ORDER>
__device__ void assemble_hessian(const double *mom, double *H, int lane) {
    using O = Ord<ORDER>;
    for (int e = lane; e < O::M * O::M; e += 32) {
        const int j = e / O::M, k = e % O::M;
        const int cj = j & 1, ck = k & 1, mj = j >> 1, mk = k >> 1;
        const int pair = cj + ck;  // 0 xx, 1 xy, 2 yy
        const int a = mu_a(mj) + mu_a(mk), b = mu_b(mj) + mu_b(mk);
        H[e] = mu_c(mj) * mu_c(mk) * mom[pair * O::NMOM + mom_idx(a, b)];
    }
    __syncwarp();
}

struct WarpSmem {
    double mom[3 * 15];
    double H[144];
    double Hinv[144];
    double aug[288];
    double A[12], S[12];
    double p[12], pprev[12], dp[12], grad[12];
    double red[16];   // reduced sums of the current iteration
    double misc[8];
    int flag[4];
};

__device__ __forceinline__ void write_history(const KArgs &A, int idx, int it, double nrm, double zncc, double znssd) {
    if (A.history) {
        double *h = A.history + ((int64_t)idx * A.max_iter + (it - 1)) * 3;
        h[0] = nrm;
        h[1] = zncc;
        h[2] = znssd;
    }
}

__device__ void write_failed_any(gpv_subset_result *out, int idx, const gpv_subset_desc &d, int status) {
    gpv_subset_result *o = out + idx;
#pragma unroll
    for (int k = 0; k < 12; k++) o->p[k] = d.p0[k];
    o->c_zncc = 0.0;
    o->c_znssd = 4.0;
    o->norm = o->eta_u = o->eta_v = o->f_m = o->delta_f = o->sssig = o->sigma = 0.0;
    o->iterations = o->converged = o->quality_ok = 0;
    o->status = status;
    o->n_px = 0;
    o->has_eta = 0;
    o->texture = 0;
    o->reserved = 0;
}

__device__ void write_failed(const KArgs &A, int idx, const gpv_subset_desc &d, int m, int status, int npx, double fm,
                             double df) {
    gpv_subset_result *o = A.out + idx;
#pragma unroll
    for (int k = 0; k < 12; k++) o->p[k] = k < m ? d.p0[k] : 0.0;
    o->c_zncc = 0.0;
    o->c_znssd = 4.0;
    o->norm = 0.0;
    o->eta_u = 0.0;
    o->eta_v = 0.0;
    o->f_m = fm;
    o->delta_f = df;
    o->sssig = 0.0;
    o->sigma = 0.0;
    o->iterations = 0;
    o->converged = 0;
    o->quality_ok = 0;
    o->status = status;
    o->n_px = npx;
    o->has_eta = 0;
    o->texture = 0;
    o->reserved = 0;
}

// Omitted-mode diagnostic from per-pixel (f, gx, gy, g) held by a worker;
// all sums FP64.  `reduce` is a functor summing a double over the worker.
// Returns eta_u, eta_v (src/subset.rs:698-820).
template <int ORDER, typename Reduce, typename Load>
__device__ void eta_sums(int npx, int tid, int nthr, double n, double fm, double df, double gm, double dg, Load load,
                         Reduce reduce, double &eu, double &ev) {
    constexpr int K = ORDER + 2;
    double se = 0, sx = 0, sxx = 0, sy = 0, syy = 0;
    for (int i = tid; i < npx; i += nthr) {
        double f, gx, gy, g, dx, dy;
        if (!load(i, f, gx, gy, g, dx, dy)) continue;
        const double e = (f - fm) / df - (g - gm) / dg;
        se += e;
        sx += gx; sxx += gx * gx;
        sy += gy; syy += gy * gy;
    }
    se = reduce(se); sx = reduce(sx); sxx = reduce(sxx); sy = reduce(sy); syy = reduce(syy);
    const double eb = se / n;
    const double mx = sx / n, my = sy / n;
    double vx = sxx / n - mx * mx, vy = syy / n - my * my;
    const double sdx = sqrt(vx > 1e-18 ? vx : 1e-18), sdy = sqrt(vy > 1e-18 ? vy : 1e-18);
    // one pass per (component, mode): three live accumulators
    double eta[2];
#pragma unroll 1
    for (int c = 0; c < 2; c++) {
        double ss = 0.0;
#pragma unroll 1
        for (int k = 0; k < K; k++) {
            double a1 = 0.0, a2 = 0.0, a3 = 0.0;
            for (int i = tid; i < npx; i += nthr) {
                double f, gx, gy, g, dx, dy;
                if (!load(i, f, gx, gy, g, dx, dy)) continue;
                const double e = (f - fm) / df - (g - gm) / dg;
                const double z = c == 0 ? (gx - mx) / sdx : (gy - my) / sdy;
                double md;
                if (ORDER == 0) md = k == 0 ? dx : dy;
                else if (ORDER == 1) md = k == 0 ? dx * dx : (k == 1 ? dx * dy : dy * dy);
                else md = k == 0 ? dx * dx * dx : (k == 1 ? dx * dx * dy : (k == 2 ? dx * dy * dy : dy * dy * dy));
                const double raw = z * md;
                a1 += raw;
                a2 += raw * raw;
                a3 += raw * e;
            }
            a1 = reduce(a1);
            a2 = reduce(a2);
            a3 = reduce(a3);
            const double mean = a1 / n;
            const double var = a2 / n - mean * mean;
            const double sd = sqrt(var > 1e-18 ? var : 1e-18);
            const double pr = (a3 - eb * a1) / (sd * n);
            ss += pr * pr;
        }
        eta[c] = sqrt(ss);
    }
    eu = eta[0];
    ev = eta[1];
}

}  // namespace
}  // namespace gpv
