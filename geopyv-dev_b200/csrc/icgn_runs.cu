// icgn_runs.cu -- mixed-precision ICGN with the circular template cut into
// vertical runs: one thread block per subset at a time, the subset's
// coefficient windows staged in shared memory, and every lane walking runs
// of K vertically adjacent template pixels with the 6 x 6 coefficient block
// of the current sample held in registers.
//
// Same algorithm and numerics contract as the other solve kernels --
// Subset::new + solve_icgn_result, src/subset.rs:836-919, 1117-1219 -- laid
// out for the B200's issue and shared-memory rates:
//  * Template runs.  The square around the circle (src/masks.rs:69-109) is
//    cut into bands of K rows; a band's columns dx in [-w, w] (w: the widest
//    circle row of the band) are its tasks, each task the K pixels
//    (dx, dy0 .. dy0 + K - 1) with a bit per pixel for the circle (and the
//    global mask).  The last band is moved up to end at dy = r, its rows
//    already covered above masked off.  Tasks are dealt to threads in band
//    order, so a warp's lanes hold neighbouring columns of one band.
//  * Sample loop.  Vertically adjacent template pixels land one coefficient
//    row apart after any warp of moderate strain, so a lane keeps the 6 x 6
//    coefficients of its last sample in registers and, when the next
//    sample's block is the same one moved down a row (same column, next
//    row), loads only the new row: 6 shared-memory loads per sample instead
//    of 36.  A sample whose block moved otherwise reloads all six rows (a
//    divergent branch taken by few lanes).  The taps and the row combine run
//    as sm_100 paired FP32 ops on symmetric weight pairs (b_k, b_{5-k}).
//  * Setup.  Every template pixel of an interior subset sits at an integer
//    offset from the centre, so f's value and gradient rows share one basis:
//    each run forms its K + 5 coefficient-row sums once (paired FMAs over
//    row pairs) and combines six of them per pixel.  The Hessian's gradient
//    moments are accumulated per run as powers of dy and expanded by powers
//    of the run's dx once per run.
//  * Hessian.  Factored once per subset (Cholesky of the Jacobi-scaled
//    matrix, FP64, one warp), and its inverse formed from the factor
//    (H^-1 = D L^-T L^-1 D); each iteration's increment is that inverse times
//    the gradient (FP64, 12 lanes).
//  * Sums.  The per-iteration sums (g - f_m, its square, (f - f_m)(g - f_m)
//    and the steepest-descent products) are FP32 over one run (at most K
//    samples), then FP64 per thread and across the block in a fixed order
//    (deterministic).
// Subsets whose warped square leaves the image or the staged window take a
// clamped per-sample path (the reference's edge clamp, src/image.rs:129-132),
// reading the window with clamped indices or global memory.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <utility>

#include "icgn_common.cuh"

namespace gpv {
namespace {

constexpr int kRunMaxWarps = 8;  // blocks of 64, 128 or 256 threads
constexpr int kRunMargin = 4;
constexpr int kRunLengths[2] = {4, 8};  // run lengths K with task tables

// NW: warps per block (block sums are kept per warp)
template <int NW>
struct RunSmem {
    double mom[3 * 15];
    double L[144];     // Cholesky factor of the scaled Hessian, then its inverse (row-major)
    double Hi[144];    // the Hessian, replaced by H^-1 formed from the factor
    double linv[12];   // 1 / L_jj
    double dsc[12];    // Jacobi scale 1 / sqrt(H_jj)
    double A[12], S[12];
    double p[12], pprev[12], dp[12], grad[12];
    double red[NW][16];
    double red2[NW][80];
    double aug[80];
    double tot[16];
    double misc[10];
    int flag[4];
    int item;
    int n_valid;
    int win_r0, win_c0, win_h, win_w, win_p, win_ok;
};

struct RunArgs {
    KArgs k;
    const int2 *tasks;        // task tables of this launch's run length K
    const int32_t *task_off;  // [radius]: first task of the radius
    const int32_t *task_n;    // [radius]: tasks of the radius
    const int32_t *seg;       // [start, count] of this segment in k.order
    int *queue;               // this launch's work-queue counter
    int win_cap;              // floats of dynamic shared memory for a window
    int nslot;                // record slots per block (tasks x K of the segment's largest radius, rounded)
    // one block per subset (slot_mask != nullptr): a block claims one of the
    // slots_per_sm scratch slots of the SM it starts on (a bit of
    // slot_mask[smid], n_mask words) and frees it when the subset is done
    uint32_t *slot_mask;
    int slots_per_sm, n_mask;
};

// Window row pitch: a multiple of 4 floats (16-byte rows for cp.async) that
// is not a multiple of 32, so two bands' rows read by one warp start on
// different banks.  Lanes of a warp read consecutive columns of one row.
__host__ __device__ __forceinline__ int run_pitch(int ww) {
    const int p = (ww + 3) & ~3;
    return (p & 31) ? p : p + 4;
}

// Copy coefficient rows [r0, r0+wh) x cols [c0, c0+ww) (c0, ww multiples of
// 4) into win with row pitch `pitch`; out-of-range rows / columns clamped.
// Threads [t0, NT) issue asynchronous 16-byte global-to-shared copies
// (cp.async, no registers held for the data), so all of a thread's copies
// are in flight at once; each thread waits for its own copies before it
// returns, and the caller's block barrier publishes the window.  Both
// addresses are 16-byte aligned: coefficient rows are a multiple of 32 floats
// apart, c0 and the clamped columns are multiples of 4, and the window's
// pitch is a multiple of 4 floats (run_pitch).
template <int NT>
__device__ __forceinline__ void run_stage(const float *__restrict__ C, int64_t cpitch, int ch, int r0, int c0, int wh,
                                          int ww, int pitch, float *win, int t0) {
    const int nv = ww >> 2;
    for (int idx = (int)threadIdx.x - t0; idx < wh * nv; idx += NT - t0) {
        const int rr = idx / nv, cc = (idx - rr * nv) << 2;
        int row = r0 + rr;
        row = row < 0 ? 0 : (row > ch - 1 ? ch - 1 : row);
        int col = c0 + cc;
        col = col < 0 ? 0 : (col > (int)cpitch - 4 ? (int)cpitch - 4 : col);
        const unsigned dst = (unsigned)__cvta_generic_to_shared(win + rr * pitch + cc);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(C + (int64_t)row * cpitch + col)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// A window covering pixel indices [xlo, xhi] x [ylo, yhi] (clamped to the
// image) plus the taps and kRunMargin; false if it does not fit in cap
// floats (the margin is dropped when the window with it does not fit).
__device__ __forceinline__ bool run_plan(int xlo, int xhi, int ylo, int yhi, int border, int cap, int &r0, int &c0,
                                         int &wh, int &ww, int &pitch) {
    for (int m = kRunMargin; m >= 0; m -= kRunMargin) {
        const int clo = xlo + border - 2 - m, chi = xhi + border + 3 + m;
        c0 = clo >= 0 ? (clo & ~3) : -(((-clo) + 3) & ~3);
        ww = ((chi + 1 - c0) + 3) & ~3;
        pitch = run_pitch(ww);
        r0 = ylo + border - 2 - m;
        wh = yhi + border + 3 + m + 1 - r0;
        if (pitch * wh <= cap) return true;
        if (m == 0) break;
    }
    return false;
}

template <class S>
__device__ __forceinline__ bool run_covers(const S &sm, int xlo, int xhi, int ylo, int yhi, int border) {
    if (!sm.win_ok) return false;
    return xlo + border - 2 >= sm.win_c0 && xhi + border + 3 < sm.win_c0 + sm.win_w && ylo + border - 2 >= sm.win_r0 &&
           yhi + border + 3 < sm.win_r0 + sm.win_h;
}

// Pixel extent (image pixels, clamped) of the square [-e, e]^2 of a subset
// centred at (cx, cy) under the warp p, conservatively; *inside: the extent
// with a one-pixel margin lies in the image (no sample meets the edge clamp).
template <int ORDER>
__device__ void run_extent(const double *p, double cx, double cy, int e, int w, int h, int &xlo, int &xhi, int &ylo,
                           int &yhi, bool *inside) {
    double ex = e, ey = e;
    if (ORDER >= 1) {
        ex = e * (fabs(1.0 + p[2]) + fabs(p[4]));
        ey = e * (fabs(p[3]) + fabs(1.0 + p[5]));
    }
    if (ORDER == 2) {
        const double rr = 0.5 * (double)e * e;
        ex += rr * (fabs(p[6 % 12]) + 2.0 * fabs(p[8 % 12]) + fabs(p[10 % 12]));
        ey += rr * (fabs(p[7 % 12]) + 2.0 * fabs(p[9 % 12]) + fabs(p[11 % 12]));
    }
    const double X0 = cx + p[0], Y0 = cy + p[1];
    const double a = floor(X0 - ex) - 1.0, b = floor(X0 + ex) + 1.0, c = floor(Y0 - ey) - 1.0, d = floor(Y0 + ey) + 1.0;
    if (!(isfinite(a) && isfinite(b) && isfinite(c) && isfinite(d))) {
        xlo = 0; xhi = w - 1; ylo = 0; yhi = h - 1;  // plans a window that cannot fit: global path
        *inside = false;
        return;
    }
    *inside = a >= 0.0 && b <= (double)(w - 1) && c >= 0.0 && d <= (double)(h - 1);
    xlo = (int)fmax(0.0, fmin(a, (double)(w - 1)));
    xhi = (int)fmax(0.0, fmin(b, (double)(w - 1)));
    ylo = (int)fmax(0.0, fmin(c, (double)(h - 1)));
    yhi = (int)fmax(0.0, fmin(d, (double)(h - 1)));
}

// Warp sums of K FP32 per-thread values (FP64 totals) into dst[0..K).
template <int KV, int C = 0>
__device__ __forceinline__ void run_warp_sums(const float (&a)[KV], double *dst, int lane) {
    if constexpr (C < KV) {
        constexpr int N = (KV - C) < 16 ? (KV - C) : 16;
        double v[N];
#pragma unroll
        for (int j = 0; j < N; j++) v[j] = (double)a[C + j];
        warp_sum_many<N>(v, dst + C, lane);
        run_warp_sums<KV, C + N>(a, dst, lane);
    }
}

template <int NT>
__device__ __forceinline__ double run_block_sum(double v, RunSmem<NT / 32> &sm) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const double s = warp_sum(v);
    if (lane == 0) sm.red[wid][0] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < NT / 32; w++) t += sm.red[w][0];
        sm.tot[0] = t;
    }
    __syncthreads();
    const double t = sm.tot[0];
    __syncthreads();
    return t;
}

// The Cholesky factor of the Jacobi-scaled SPD Hessian and the factor's
// inverse, by one warp in registers: D H D = L L^T with D = diag(1 /
// sqrt(H_jj)), so H^-1 = D L^-T L^-1 D.  Lane i < M builds row i of H from the gradient
// moments (H_jk = c_j c_k sum g_p g_q dx^a dy^b, the entries assemble_hessian
// gives) and keeps it in registers; the pivot and the column entries each
// step needs travel by shuffle.  Each pivot takes one reciprocal square root
// (1 / L_kk, and L_kk = pivot x that), not a square root and a division:
// the serial chain of a lone warp is what this stretch costs.  Lane c then
// solves L x = e_c for column c of L^-1 (rows of L read from Lm, M*M shared
// scratch), which then holds L^-1 (zeros above the diagonal), and lane i
// stores s_i = 1 / sqrt(H_ii) in dsc; hess_inverse_block forms H^-1 from
// them.  False (warp-uniform) when a pivot is not positive or not finite:
// a singular Hessian.
template <int ORDER>
__device__ bool hess_factor_regs(const double *mom, double *Lm, double *linv, double *dsc, int lane) {
    using O = Ord<ORDER>;
    constexpr int M = O::M;
    constexpr unsigned kAll = 0xffffffffu;
    const int li = lane < M ? lane : 0;  // lanes >= M shadow row 0; their results are never read
    const int mi = li >> 1, ci = li & 1, ai = mu_a(mi), bi = mu_b(mi);
    const double cci = mu_c(mi);
    double h[M];
#pragma unroll
    for (int k = 0; k < M; k++) {
        const int mk = k >> 1, ck = k & 1;
        h[k] = cci * mu_c(mk) * mom[(ci + ck) * O::NMOM + mom_idx(ai + mu_a(mk), bi + mu_b(mk))];
    }
    const double dii = cci * cci * mom[(2 * ci) * O::NMOM + mom_idx(2 * ai, 2 * bi)];  // h[li]
    if (__any_sync(kAll, !(dii > 0.0) || !isfinite(dii))) return false;
    const double si = rsqrt(dii);
#pragma unroll
    for (int j = 0; j < M; j++) {
        const double sj = __shfl_sync(kAll, si, j);
        h[j] *= si * sj;
    }
    // 1 / L_kk into linv (shared, M doubles) by lane k
#pragma unroll
    for (int k = 0; k < M; k++) {
        const double piv = __shfl_sync(kAll, h[k], k);
        if (!(piv > 0.0) || !isfinite(piv)) return false;  // uniform: every lane has lane k's value
        const double rk = rsqrt(piv);
        const double lkk = piv * rk;
        if (lane == k) linv[k] = rk;
        h[k] = li > k ? h[k] * rk : (li == k ? lkk : h[k]);
#pragma unroll
        for (int j = k + 1; j < M; j++) {
            const double ljk = __shfl_sync(kAll, h[k], j);
            if (li >= j) h[j] = fma(-h[k], ljk, h[j]);
        }
    }
    if (lane < M) {
#pragma unroll
        for (int j = 0; j < M; j++) Lm[lane * M + j] = j <= lane ? h[j] : 0.0;
    }
    __syncwarp();
    // column c = lane of L^-1 by forward substitution (zero above the
    // diagonal), right-looking: each x_k, once known, updates every later
    // row at once, so the dependent chain is M steps, not M (M - 1) / 2
    double x[M];
#pragma unroll
    for (int i = 0; i < M; i++) x[i] = (i == lane) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < M; k++) {
        x[k] = (k >= lane) ? x[k] * linv[k] : 0.0;
#pragma unroll
        for (int i = k + 1; i < M; i++) x[i] = fma(-Lm[i * M + k], x[k], x[i]);
    }
    __syncwarp();
    if (lane < M) {
#pragma unroll
        for (int i = 0; i < M; i++) Lm[i * M + lane] = x[i];  // Lm now holds L^-1 (lower)
    }
    if (lane < M) dsc[lane] = si;
    __syncwarp();
    return true;
}

// H^-1 = D L^-T L^-1 D from hess_factor_regs's L^-1 (Lm) and D (dsc), by
// the whole block between two barriers (no warp waits on another's serial
// work here): entry (i, j) is s_i s_j times the dot product of columns i
// and j of L^-1.
template <int M, int NT>
__device__ __forceinline__ void hess_inverse_block(const double *Lm, const double *dsc, double *Hi) {
    for (int e = threadIdx.x; e < M * M; e += NT) {
        const int i = e / M, j = e - (e / M) * M;
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < M; k++) acc = fma(Lm[k * M + i], Lm[k * M + j], acc);
        Hi[e] = dsc[i] * dsc[j] * acc;
    }
}

// The quintic basis at fraction t as symmetric pairs W[k] = (w_k, w_{5-k}),
// k = 0..2: the weights of basis() split about t = 1/2 into an even part
// e_k(v) and an odd part -u P_k(v) (u = t - 1/2, v = u^2), w_k = e_k - u P_k
// and w_{5-k} = e_k + u P_k, each one FMA (the odd part is never rounded on
// its own), in scalar FP32 ops whose polynomial coefficients are
// instruction immediates; each weight lands in its half of the pair.
__device__ __forceinline__ void basis_sym1(float t, float2 W[3]) {
    const float u = t - 0.5f;
    const float v = u * u;
    const float e0 = fmaf(fmaf(v, 1.0f / 48.0f, 1.0f / 96.0f), v, 1.0f / 3840.0f);
    const float e1 = fmaf(fmaf(v, -1.0f / 16.0f, 7.0f / 32.0f), v, 79.0f / 1280.0f);
    const float e2 = fmaf(fmaf(v, 1.0f / 24.0f, -11.0f / 48.0f), v, 841.0f / 1920.0f);
    const float q0 = fmaf(fmaf(v, 1.0f / 120.0f, 1.0f / 48.0f), v, 1.0f / 384.0f);
    const float q1 = fmaf(fmaf(v, -1.0f / 24.0f, 1.0f / 16.0f), v, 25.0f / 128.0f);
    const float q2 = fmaf(fmaf(v, 1.0f / 12.0f, -7.0f / 24.0f), v, 77.0f / 192.0f);
    W[0] = make_float2(fmaf(-u, q0, e0), fmaf(u, q0, e0));
    W[1] = make_float2(fmaf(-u, q1, e1), fmaf(u, q1, e1));
    W[2] = make_float2(fmaf(-u, q2, e2), fmaf(u, q2, e2));
}

// One coefficient row against the column weights: sum_k b_k c_k with the
// pairs (c_k, c_{5-k}) x (b_k, b_{5-k}).
__device__ __forceinline__ float row_dot(const float (&c)[6], const float2 B[3]) {
    float2 s = __fmul2_rn(make_float2(c[0], c[5]), B[0]);
    s = __ffma2_rn(make_float2(c[1], c[4]), B[1], s);
    s = __ffma2_rn(make_float2(c[2], c[3]), B[2], s);
    return s.x + s.y;
}

__device__ __forceinline__ float combine6(const float (&s)[6], const float2 A[3]) {
    float2 v = __fmul2_rn(make_float2(s[0], s[5]), A[0]);
    v = __ffma2_rn(make_float2(s[1], s[4]), A[1], v);
    v = __ffma2_rn(make_float2(s[2], s[3]), A[2], v);
    return v.x + v.y;
}

// Per-run FP32 accumulators of the iteration sums.
struct RunAcc {
    float p1, p2, pfg;
    float2 m0, m1, m2;  // sum G, sum G dy, sum G dy^2 with G = (gx, gy) (g - f_m)
};

// A Kahan-compensated FP64 sum: add() carries the rounding error of each
// addition into the next one.
struct KSum {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        const double y = x - c, t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

// One sample: rec = (df/dx, df/dy, f - s, w) with w = 1 for template
// pixels, 0 outside (the gradient pair first: one aligned register pair,
// so the steepest-descent products and sums are paired FP32 operations);
// pfg sums (f - s)(g - f_m) (corrected to f - f_m with the block totals).  KAHAN: the three ZNSSD sums (g - f_m, its square and
// the cross term) go straight into the thread's compensated FP64 sums ks
// instead of the run's FP32 partials.
template <int ORDER, bool KAHAN>
__device__ __forceinline__ void acc_sample(RunAcc &a, KSum (&ks)[3], float4 rec, float g, float fmf, float dyf) {
    const float gc = (g - fmf) * rec.w;
    if (KAHAN) {
        const double gd = (double)gc;
        ks[0].add(gd);
        ks[1].add(gd * gd);
        ks[2].add((double)rec.z * gd);
    } else {
        a.p1 += gc;
        a.p2 = fmaf(gc, gc, a.p2);
        a.pfg = fmaf(rec.z, gc, a.pfg);
    }
    const float2 gxy = __fmul2_rn(make_float2(rec.x, rec.y), make_float2(gc, gc));
    a.m0 = __fadd2_rn(a.m0, gxy);
    if (ORDER >= 1) a.m1 = __ffma2_rn(gxy, make_float2(dyf, dyf), a.m1);
    if (ORDER == 2) {
        const float d2 = dyf * dyf;
        a.m2 = __ffma2_rn(gxy, make_float2(d2, d2), a.m2);
    }
}

// The run's steepest-descent sums into the thread's totals PB[mu] (pairs
// (gx, gy) of monomial mu = 1, dx, dy, dx^2/2, dx dy, dy^2/2).
template <int ORDER>
__device__ __forceinline__ void acc_expand(const RunAcc &a, float dxf, float2 (&PB)[6]) {
    PB[0] = __fadd2_rn(PB[0], a.m0);
    if (ORDER >= 1) {
        PB[1] = __ffma2_rn(make_float2(dxf, dxf), a.m0, PB[1]);
        PB[2] = __fadd2_rn(PB[2], a.m1);
    }
    if (ORDER == 2) {
        const float h = 0.5f * dxf * dxf;
        PB[3] = __ffma2_rn(make_float2(h, h), a.m0, PB[3]);
        PB[4] = __ffma2_rn(make_float2(dxf, dxf), a.m1, PB[4]);
        PB[5] = __ffma2_rn(make_float2(0.5f, 0.5f), a.m2, PB[5]);
    }
}

__device__ __forceinline__ void unpack_task(int2 tk, int &dx, int &dy0) {
    dx = (int)(short)(tk.x & 0xffff);
    dy0 = tk.x >> 16;
}

template <int ORDER, int NT, int K, bool KAHAN>
__device__ void run_subset(const RunArgs &R, int idx, const gpv_subset_desc &d, float *base, float *win,
                           RunSmem<NT / 32> &sm) {
    const KArgs &A = R.k;
    using O = Ord<ORDER>;
    constexpr int M = O::M, NMU = O::NMU, NMOM = O::NMOM, NB = 2 * O::DEG + 1;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int r = d.radius;
    const int re = max(r, K - 1 - r);  // half side of the square the runs cover
    const int T = R.task_n[r];
    const int2 *tasks = R.tasks + R.task_off[r];
    const int NS = T * K;
    // per-pixel records (df/dx, df/dy, f - s, 1 in the template / 0 outside:
    // zero gradients outside) in slot j * T + t of run t; eta resamples; run bits
    float4 *REC = reinterpret_cast<float4 *>(base);
    float *RSG = base + 4 * R.nslot;
    int *RVM = reinterpret_cast<int *>(base + 5 * R.nslot);
    const double cx = d.coord[0], cy = d.coord[1];
    const int cxi = (int)cx, cyi = (int)cy;
    const double fxd = floor(cx), fyd = floor(cy);
    const int bx = (int)fxd, by = (int)fyd;
    const float fx = (float)(cx - fxd), fy = (float)(cy - fyd);
    const int B = A.border, ch = A.h + 2 * B;

    // ---- stage f's window ------------------------------------------------
    {
        // +-1: an FP32 fraction can round up to the next integer
        const int xlo = max(0, min(bx - re - 1, A.w - 1)), xhi = max(0, min(bx + re + 1, A.w - 1));
        const int ylo = max(0, min(by - re - 1, A.h - 1)), yhi = max(0, min(by + re + 1, A.h - 1));
        int r0, c0, wh, ww, pitch;
        const bool ok = run_plan(xlo, xhi, ylo, yhi, B, R.win_cap, r0, c0, wh, ww, pitch);
        if (ok) run_stage<NT>(A.f32, A.pitch32, ch, r0, c0, wh, ww, pitch, win, 0);
        if (tid == 0) {
            sm.win_ok = 0;  // g must be staged before the iterations
            sm.win_r0 = r0; sm.win_c0 = c0; sm.win_h = wh; sm.win_w = ww; sm.win_p = pitch;
            sm.flag[2] = ok;
        }
        __syncthreads();
    }
    const bool f_staged = sm.flag[2] != 0;
    const int fr0 = sm.win_r0, fc0 = sm.win_c0, fwh = sm.win_h, fww = sm.win_w, fP = sm.win_p;
    // interior: every run pixel sits at an integer offset from the centre
    // inside the image, so all share one fraction and one basis
    const bool interior = f_staged && bx - re >= 0 && bx + re <= A.w - 1 && by - re >= 0 && by + re <= A.h - 1;

    // ---- setup, pass 1: f and its gradient per pixel, first sums ------------
    // [count, sum (f-s), sum (f-s)^2, SSSIG, Bf_j = sum SDI_j (f-s) (M),
    //  S_j = sum SDI_j (M)] about a subset-uniform level s (the coefficient
    // under the centre: keeps the sums free of cancellation and a flat
    // subset's sums exactly zero); FP32 per thread, FP64 across the block.
    constexpr int NVA = 4 + 2 * M;
    float acc[NVA];
#pragma unroll
    for (int q = 0; q < NVA; q++) acc[q] = 0.f;
    float shift;
    if (f_staged) {
        const int wx = min(max(max(0, min(bx, A.w - 1)) + B - fc0, 0), fww - 1);
        const int wy = min(max(max(0, min(by, A.h - 1)) + B - fr0, 0), fwh - 1);
        shift = win[wy * fP + wx];
    } else {
        shift = A.f32[(int64_t)(max(0, min(by, A.h - 1)) + B) * A.pitch32 + max(0, min(bx, A.w - 1)) + B];
    }
    auto pix1 = [&](bool v, float f, float gx, float gy, int dx, int dy) {
        if (!v) return;
        const float dxf = (float)dx, dyf = (float)dy;
        const float fs = f - shift;
        acc[0] += 1.f;
        acc[1] += fs;
        acc[2] = fmaf(fs, fs, acc[2]);
        acc[3] = fmaf(0.5f * gx, gx, fmaf(0.5f * gy, gy, acc[3]));
        const float gxf = gx * fs, gyf = gy * fs;
#pragma unroll
        for (int mu = 0; mu < NMU; mu++) {
            const float mv = mu_val<float>(mu, dxf, dyf);
            acc[4 + 2 * mu] = fmaf(gxf, mv, acc[4 + 2 * mu]);
            acc[5 + 2 * mu] = fmaf(gyf, mv, acc[5 + 2 * mu]);
            acc[4 + M + 2 * mu] = fmaf(gx, mv, acc[4 + M + 2 * mu]);
            acc[5 + M + 2 * mu] = fmaf(gy, mv, acc[5 + M + 2 * mu]);
        }
    };
    {
        float a0[6], da0[6], b0[6], db0[6];
        basis(fy, a0); dbasis(fy, da0);
        basis(fx, b0); dbasis(fx, db0);
        float2 bb[6], dbb[6];  // column weights as duplicated pairs (two rows per paired FMA)
#pragma unroll
        for (int k = 0; k < 6; k++) {
            bb[k] = make_float2(b0[k], b0[k]);
            dbb[k] = make_float2(db0[k], db0[k]);
        }
        for (int t = tid; t < T; t += NT) {
            int dx, dy0;
            unpack_task(tasks[t], dx, dy0);
            uint32_t vm = (uint32_t)tasks[t].y;
            if (A.mask) {
#pragma unroll
                for (int j = 0; j < K; j++)
                    if (!mask_ok(A, cxi, cyi, dx, dy0 + j)) vm &= ~(1u << j);
            }
            RVM[t] = (int)vm;
            if (interior) {
                // coefficient-row sums (value and x-derivative weights) of the
                // run's K + 5 rows, two rows per paired FMA; then six rows per pixel
                const float *p0 = win + (by + dy0 + B - 2 - fr0) * fP + (bx + dx + B - 2 - fc0);
                float s[K + 6], q[K + 6];
#pragma unroll
                for (int m = 0; m + 1 < K + 5; m += 2) {
                    const float *r0 = p0 + m * fP, *r1 = r0 + fP;
                    float2 c = make_float2(r0[0], r1[0]);
                    float2 S2 = __fmul2_rn(c, bb[0]), D2 = __fmul2_rn(c, dbb[0]);
#pragma unroll
                    for (int k = 1; k < 6; k++) {
                        c = make_float2(r0[k], r1[k]);
                        S2 = __ffma2_rn(c, bb[k], S2);
                        D2 = __ffma2_rn(c, dbb[k], D2);
                    }
                    s[m] = S2.x; s[m + 1] = S2.y;
                    q[m] = D2.x; q[m + 1] = D2.y;
                }
                if ((K + 5) & 1) {  // the last row alone (no row past the window)
                    const float *r0 = p0 + (K + 4) * fP;
                    float sv = r0[0] * b0[0], qv = r0[0] * db0[0];
#pragma unroll
                    for (int k = 1; k < 6; k++) {
                        sv = fmaf(r0[k], b0[k], sv);
                        qv = fmaf(r0[k], db0[k], qv);
                    }
                    s[K + 4] = sv;
                    q[K + 4] = qv;
                }
#pragma unroll
                for (int j = 0; j < K; j++) {
                    float val = 0.f, vx = 0.f, vy = 0.f;
#pragma unroll
                    for (int rr = 0; rr < 6; rr++) {
                        val = fmaf(a0[rr], s[j + rr], val);
                        vx = fmaf(a0[rr], q[j + rr], vx);
                        vy = fmaf(da0[rr], s[j + rr], vy);
                    }
                    const bool v = (vm >> j) & 1u;
                    REC[j * T + t] = v ? make_float4(vx, vy, val - shift, 1.f) : make_float4(0.f, 0.f, 0.f, 0.f);
                    pix1(v, val, vx, vy, dx, dy0 + j);
                }
            } else {
                for (int j = 0; j < K; j++) {
                    const bool v = (vm >> j) & 1u;
                    int ix, iy;
                    float tx, ty;
                    split_clamped(bx, fx + (float)dx, A.w, ix, tx);
                    split_clamped(by, fy + (float)(dy0 + j), A.h, iy, ty);
                    float a[6], da[6], b[6], db[6];
                    basis(ty, a); dbasis(ty, da);
                    basis(tx, b); dbasis(tx, db);
                    float f, gx, gy;
                    if (f_staged) {
                        const int wx = min(max(ix + B - 2 - fc0, 0), fww - 6), wy = min(max(iy + B - 2 - fr0, 0), fwh - 6);
                        f = contract_grad<float>(win + wy * fP + wx, fP, a, da, b, db, gx, gy);
                    } else {
                        const float *F = A.f32 + (int64_t)(iy + B - 2) * A.pitch32 + (ix + B - 2);
                        f = contract_grad<float>(F, A.pitch32, a, da, b, db, gx, gy);
                    }
                    REC[j * T + t] = v ? make_float4(gx, gy, f - shift, 1.f) : make_float4(0.f, 0.f, 0.f, 0.f);
                    pix1(v, f, gx, gy, dx, dy0 + j);
                }
            }
        }
    }
    run_warp_sums<NVA>(acc, sm.red2[wid], lane);
    // ---- setup, pass 2: the Hessian's gradient moments ----------------------
    // sum g_p g_q dx^a dy^b (a + b <= 2 DEG) per run as powers of dy, then
    // expanded by the run's powers of dx; each thread re-reads its own records
    {
        float mom[3 * NMOM];
#pragma unroll
        for (int q = 0; q < 3 * NMOM; q++) mom[q] = 0.f;
        for (int t = tid; t < T; t += NT) {
            int dx, dy0;
            unpack_task(tasks[t], dx, dy0);
            float V[3][NB];
#pragma unroll
            for (int p = 0; p < 3; p++)
#pragma unroll
                for (int b = 0; b < NB; b++) V[p][b] = 0.f;
#pragma unroll
            for (int j = 0; j < K; j++) {
                const float4 rec = REC[j * T + t];
                const float gx = rec.x, gy = rec.y;  // zero for pixels outside the template
                const float gg[3] = {gx * gx, gx * gy, gy * gy};
                const float dyf = (float)(dy0 + j);
                float pw = 1.f;
#pragma unroll
                for (int b = 0; b < NB; b++) {
#pragma unroll
                    for (int p = 0; p < 3; p++) V[p][b] = fmaf(gg[p], pw, V[p][b]);
                    pw *= dyf;
                }
            }
            const float dxf = (float)dx;
            float xp[NB];
            xp[0] = 1.f;
#pragma unroll
            for (int a = 1; a < NB; a++) xp[a] = xp[a - 1] * dxf;
#pragma unroll
            for (int a = 0; a < NB; a++)
#pragma unroll
                for (int b = 0; a + b < NB; b++)
#pragma unroll
                    for (int p = 0; p < 3; p++)
                        mom[p * NMOM + mom_idx(a, b)] = fmaf(xp[a], V[p][b], mom[p * NMOM + mom_idx(a, b)]);
        }
        run_warp_sums<3 * NMOM>(mom, sm.red2[wid] + NVA, lane);
    }
    __syncthreads();
    constexpr int NV = NVA + 3 * NMOM;
    if (wid == 0) {
        // block sums of the warp partials, then f_m, delta_f, A_j, S_j, the
        // Hessian and its factor (warp 0) while the other warps stage g's window
        for (int q = lane; q < NV; q += 32) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < NT / 32; w++) t += sm.red2[w][q];
            sm.aug[q] = t;
        }
        __syncwarp();
        const int n = (int)(sm.aug[0] + 0.5);
        const double dn = (double)n, ms = sm.aug[1] / (n > 0 ? dn : 1.0);  // mean of f - s
        const double fm = (double)shift + ms;
        const double saa = sm.aug[2] - ms * sm.aug[1];  // sum (f - f_m)^2
        int st = GPV_OK;
        if (n == 0) st = GPV_EMPTY_MASK;
        else if (!(sqrt(fmax(saa, 0.0) / dn) > 1e-6 * fmax(1.0, fabs(fm)))) st = GPV_FEATURELESS;  // flat subset
        if (st == GPV_OK) {
            if (lane < M) {
                sm.A[lane] = sm.aug[4 + lane] - ms * sm.aug[4 + M + lane];  // sum SDI (f - f_m)
                sm.S[lane] = sm.aug[4 + M + lane];
            }
            if (lane < 3 * NMOM) sm.mom[lane] = sm.aug[NVA + lane];
            if (lane + 32 < 3 * NMOM) sm.mom[lane + 32] = sm.aug[NVA + lane + 32];
            __syncwarp();
            if (!hess_factor_regs<ORDER>(sm.mom, sm.L, sm.linv, sm.dsc, lane)) st = GPV_SINGULAR_H;
        }
        if (lane == 0) {
            sm.flag[0] = st;
            sm.misc[5] = fm;
            sm.misc[6] = saa;
            sm.misc[7] = sm.aug[3];
            sm.n_valid = n;
        }
        if (lane < M) {
            sm.p[lane] = d.p0[lane];
            sm.pprev[lane] = d.p0[lane];
        }
    } else {
        // stage g's window around the initial warp
        int xlo, xhi, ylo, yhi, r0 = 0, c0 = 0, wh = 0, ww = 0, pitch = 0;
        bool inside;
        double p0[12];
#pragma unroll
        for (int k = 0; k < 12; k++) p0[k] = d.p0[k % M];
        run_extent<ORDER>(p0, cx, cy, re, A.w, A.h, xlo, xhi, ylo, yhi, &inside);
        const bool ok = run_plan(xlo, xhi, ylo, yhi, B, R.win_cap, r0, c0, wh, ww, pitch);
        if (ok) run_stage<NT>(A.g32, A.pitch32, ch, r0, c0, wh, ww, pitch, win, 32);
        if (tid == 32) {
            sm.win_ok = ok;
            sm.win_r0 = r0; sm.win_c0 = c0; sm.win_h = wh; sm.win_w = ww; sm.win_p = pitch;
        }
    }
    __syncthreads();
    const int st0 = sm.flag[0];
    const int n = sm.n_valid;
    const double dn = (double)n;
    const double fm = sm.misc[5], saa = sm.misc[6], tot_sssig = sm.misc[7];
    const float fmf = (float)fm;
    const double df = sqrt(fmax(saa, 0.0));
    if (st0 != GPV_OK) {
        if (tid == 0) {
            write_failed(A, idx, d, M, st0, n, n ? fm : 0.0, n ? df : 0.0);
            if (st0 == GPV_SINGULAR_H) {
                A.out[idx].sssig = tot_sssig;
                A.out[idx].sigma = sqrt(saa / dn);
            }
        }
        return;
    }
    // H^-1 by every thread (warp 0 reads it only after the first iteration's barrier)
    hess_inverse_block<M, NT>(sm.L, sm.dsc, sm.Hi);

    // ---- ICGN iterations --------------------------------------------------
    const double size = sqrt(dn);
    const double inv_dn = 1.0 / dn, inv_df = 1.0 / df;
    int iters = 0, status = GPV_OK;
    bool converged = false;
    double c_zncc = 0.0, c_znssd = 4.0, last_norm = 0.0, gm_last = 0.0, dg_last = 0.0;
    for (int it = 1; it <= A.max_iter; it++) {
        // (re)stage g's window when the warped square has left it
        bool inside;
        {
            int xlo, xhi, ylo, yhi;
            run_extent<ORDER>(sm.p, cx, cy, re, A.w, A.h, xlo, xhi, ylo, yhi, &inside);
            if (!run_covers(sm, xlo, xhi, ylo, yhi, B)) {
                int r0, c0, wh, ww, pitch;
                const bool ok = run_plan(xlo, xhi, ylo, yhi, B, R.win_cap, r0, c0, wh, ww, pitch);
                __syncthreads();  // nobody still reads the old window
                if (ok) run_stage<NT>(A.g32, A.pitch32, ch, r0, c0, wh, ww, pitch, win, 0);
                if (tid == 0) {
                    sm.win_ok = ok;
                    sm.win_r0 = r0; sm.win_c0 = c0; sm.win_h = wh; sm.win_w = ww; sm.win_p = pitch;
                }
                __syncthreads();
            }
        }
        const bool staged = sm.win_ok != 0;
        const int gr0 = sm.win_r0, gc0 = sm.win_c0, gwh = sm.win_h, gww = sm.win_w, gP = sm.win_p;
        const double X0 = cx + sm.p[0], Y0 = cy + sm.p[1];
        const double bxd = floor(X0), byd = floor(Y0);
        const int wbx = (int)bxd, wby = (int)byd;
        const float ox = (float)(X0 - bxd), oy = (float)(Y0 - byd);
        float ux = 0.f, uy = 0.f, vx = 0.f, vy = 0.f, uxx = 0.f, uxy = 0.f, uyy = 0.f, vxx = 0.f, vxy = 0.f, vyy = 0.f;
        if (ORDER >= 1) { ux = (float)sm.p[2]; vx = (float)sm.p[3]; uy = (float)sm.p[4]; vy = (float)sm.p[5]; }
        if (ORDER == 2) {
            uxx = (float)(0.5 * sm.p[6 % M]); vxx = (float)(0.5 * sm.p[7 % M]); uxy = (float)sm.p[8 % M];
            vxy = (float)sm.p[9 % M]; uyy = (float)(0.5 * sm.p[10 % M]); vyy = (float)(0.5 * sm.p[11 % M]);
        }
        // window-relative origin: integer position (ix, iy) relative to (wbx,
        // wby) reads rows iy + wy0 .., columns ix + wx0 ..
        const int wy0 = wby + B - 2 - gr0, wx0 = wbx + B - 2 - gc0;
        const bool fast = staged && inside;
        // A sample's position relative to (wbx, wby) is its integer offset
        // (dx, dy) plus the small part s(dx, dy) = A2(dx) + B2(dx) dy + C2 dy^2
        // ((y, x) pairs; |s| ~ the fraction plus the deformation over the
        // subset): s is rounded in FP32 at its own small magnitude, and the
        // integer offsets join its floor exactly.
        const float2 O2 = make_float2(oy, ox), U1 = make_float2(vx, ux), U2 = make_float2(vy, uy);
        const float2 Q1 = make_float2(vxx, uxx), Q2 = make_float2(vxy, uxy), C2 = make_float2(vyy, uyy);
        double s1 = 0.0, s2 = 0.0, sfg = 0.0;
        KSum ks[3];
        float2 PB[6];
#pragma unroll
        for (int k = 0; k < 6; k++) PB[k] = make_float2(0.f, 0.f);
        for (int t = tid; t < T; t += NT) {
            int dx, dy0;
            unpack_task(tasks[t], dx, dy0);
            const float dxf = (float)dx;
            float2 A2 = O2, B2 = make_float2(0.f, 0.f);
            if (ORDER >= 1) {
                A2 = __ffma2_rn(U1, make_float2(dxf, dxf), A2);
                B2 = U2;
            }
            if (ORDER == 2) {
                A2 = __ffma2_rn(Q1, make_float2(dxf * dxf, dxf * dxf), A2);
                B2 = __ffma2_rn(Q2, make_float2(dxf, dxf), B2);
            }
            RunAcc ac;
            ac.p1 = ac.p2 = ac.pfg = 0.f;
            ac.m0 = ac.m1 = ac.m2 = make_float2(0.f, 0.f);
            if (fast) {
                // no edge clamp can apply and the window covers every tap:
                // the 6 x 6 block rolls down the run in registers
                float Rg[6][6];
                int fxp = 0, fyp = 0;
                // window position of the run's first pixel at zero small part
                const float *rbase = win + (dy0 + wy0) * gP + (dx + wx0);
                const float dy0f = (float)dy0;
#pragma unroll
                for (int j = 0; j < K; j++) {
                    const float dyf = dy0f + (float)j;  // exact: small integers
                    float2 L = A2;
                    if (ORDER >= 1) L = __ffma2_rn(B2, make_float2(dyf, dyf), L);
                    if (ORDER == 2) L = __ffma2_rn(C2, make_float2(dyf * dyf, dyf * dyf), L);
                    const float fly = floorf(L.x), flx = floorf(L.y);
                    const int iy = (int)fly, ix = (int)flx;  // floor offsets of the small part
                    const float2 tt = __fadd2_rn(L, make_float2(-fly, -flx));
                    const float *rp = rbase + (j + iy) * gP + ix;
                    if (j == 0) {
#pragma unroll
                        for (int rr = 0; rr < 6; rr++)
#pragma unroll
                            for (int k = 0; k < 6; k++) Rg[rr][k] = rp[rr * gP + k];
                    } else {
                        if (ix != fxp || iy != fyp) {  // the block did not move down one row: reload
#pragma unroll
                            for (int rr = 0; rr < 5; rr++)
#pragma unroll
                                for (int k = 0; k < 6; k++) Rg[(j + rr) % 6][k] = rp[rr * gP + k];
                        }
#pragma unroll
                        for (int k = 0; k < 6; k++) Rg[(j + 5) % 6][k] = rp[5 * gP + k];
                    }
                    fxp = ix;
                    fyp = iy;
                    float2 Aw[3], Bw[3];
                    basis_sym1(tt.x, Aw);
                    basis_sym1(tt.y, Bw);
                    float sr[6];
#pragma unroll
                    for (int rr = 0; rr < 6; rr++) sr[rr] = row_dot(Rg[(j + rr) % 6], Bw);
                    const float g = combine6(sr, Aw);
                    const int sl = j * T + t;
                    acc_sample<ORDER, KAHAN>(ac, ks, REC[sl], g, fmf, dyf);
                }
            } else {
                for (int j = 0; j < K; j++) {
                    const float dyf = (float)(dy0 + j);
                    float2 L = A2;
                    if (ORDER >= 1) L = __ffma2_rn(B2, make_float2(dyf, dyf), L);
                    if (ORDER == 2) L = __ffma2_rn(C2, make_float2(dyf * dyf, dyf * dyf), L);
                    int ix, iy;
                    float tx, ty;
                    split_clamped(wbx + dx, L.y, A.w, ix, tx);
                    split_clamped(wby + dy0 + j, L.x, A.h, iy, ty);
                    float a[6], b[6];
                    basis(ty, a);
                    basis(tx, b);
                    float g;
                    if (staged) {
                        const int wx = min(max(ix + B - 2 - gc0, 0), gww - 6), wy = min(max(iy + B - 2 - gr0, 0), gwh - 6);
                        g = contract<float>(win + wy * gP + wx, gP, a, b);
                    } else {
                        g = contract<float>(A.g32 + (int64_t)(iy + B - 2) * A.pitch32 + (ix + B - 2), A.pitch32, a, b);
                    }
                    const int sl = j * T + t;
                    acc_sample<ORDER, KAHAN>(ac, ks, REC[sl], g, fmf, dyf);
                }
            }
            if (!KAHAN) {
                s1 += (double)ac.p1;
                s2 += (double)ac.p2;
                sfg += (double)ac.pfg;
            }
            acc_expand<ORDER>(ac, dxf, PB);
        }
        // block sums: warp partials to shared memory, one barrier, then warp 0
        // adds them up and updates the warp; a second barrier publishes p
        constexpr int KR = 3 + M;
        {
            double v[KR];
            if (KAHAN) {
                s1 = ks[0].s;
                s2 = ks[1].s;
                sfg = ks[2].s;
            }
            v[0] = s1; v[1] = s2; v[2] = sfg;
#pragma unroll
            for (int j = 0; j < M / 2; j++) {
                v[3 + 2 * j] = (double)PB[j].x;
                v[4 + 2 * j] = (double)PB[j].y;
            }
            warp_sum_many<KR>(v, sm.red[wid], lane);
        }
        __syncthreads();
        if (wid == 0) {
            double tl = 0.0;
            if (lane < KR) {
#pragma unroll
                for (int w = 0; w < NT / 32; w++) tl += sm.red[w][lane];
            }
            const double t0 = __shfl_sync(0xffffffffu, tl, 0), t1 = __shfl_sync(0xffffffffu, tl, 1);
            const double t2 = __shfl_sync(0xffffffffu, tl, 2);
            const double gmt = t0 * inv_dn;
            const double dg2 = t1 - t0 * gmt;
            const double dg2p = dg2 > 0.0 ? dg2 : 0.0;
            const double dg = sqrt(dg2p);
            // sum (f - f_m)(g - g_m) = sum (f - f_m)(g - f_m) (sum (f - f_m) = 0)
            //                     = sum (f - s)(g - f_m) - (f_m - s) sum (g - f_m)
            const double sab = t2 - (fm - (double)shift) * t0;
            const double rdg = rsqrt(dg2p);  // 1 / delta_g: one reciprocal square root on the update's critical path
            const double znssd = 2.0 - 2.0 * sab * (inv_df * rdg);
            const double ratio = df * rdg;
            // lane j < M: grad_j = A_j - (df/dg)(B_j - g~_m S_j); B_j sits at lane 3 + j
            const double bj = __shfl_down_sync(0xffffffffu, tl, 3);
            const double gj = lane < M ? sm.A[lane] - ratio * (bj - gmt * sm.S[lane]) : 0.0;
            // dp = -H^-1 grad with the inverse formed from the Cholesky factor at setup
            // (12 lanes, two FMA chains each; 1.7% faster than two substitutions)
            if (lane < M) sm.grad[lane] = gj;
            __syncwarp();
            double dpj = 0.0;
            if (lane < M) {
                double a0 = 0.0, a1 = 0.0;
#pragma unroll
                for (int k = 0; k < M; k += 2) {
                    a0 = fma(sm.Hi[lane * M + k], sm.grad[k], a0);
                    if (k + 1 < M) a1 = fma(sm.Hi[lane * M + k + 1], sm.grad[k + 1], a1);
                }
                dpj = -(a0 + a1);
            }
            if (lane < M) {
                sm.dp[lane] = dpj;
                sm.pprev[lane] = sm.p[lane];
            }
            __syncwarp();
            if (lane == 0) {
                double pn[12], dpl[12], pl[12];
#pragma unroll
                for (int k = 0; k < 12; k++) {
                    dpl[k] = sm.dp[k % M];
                    pl[k] = sm.p[k % M];
                }
                bool ok = true;
                if (ORDER == 0) {
                    pn[0] = pl[0] - dpl[0];
                    pn[1] = pl[1] - dpl[1];
                } else if (ORDER == 1) {
                    ok = compose1(pl, dpl, pn);
                } else {
                    ok = compose2_regs(pl, dpl, pn);
                }
                if (ok) {
#pragma unroll
                    for (int k = 0; k < M; k++) sm.p[k] = pn[k];
                }
                sm.flag[1] = ok;
                sm.misc[1] = conv_norm<M>(dpl, size);
                sm.misc[2] = gmt;
                sm.misc[3] = dg;
                sm.misc[4] = znssd;
            }
        }
        __syncthreads();
        const double gmt = sm.misc[2], dg = sm.misc[3], znssd = sm.misc[4];
        gm_last = fm + gmt;
        dg_last = dg;
        if (!sm.flag[1]) {
            status = GPV_SINGULAR_WDELTA;  // p keeps the last valid warp
            break;
        }
        const double nrm = sm.misc[1];
        c_znssd = znssd;
        c_zncc = 1.0 - znssd / 2.0;
        iters = it;
        last_norm = nrm;
        if (tid == 0) write_history(A, idx, it, nrm, c_zncc, c_znssd);
        if (!isfinite(nrm)) { status = GPV_NONFINITE; break; }
        if (nrm < A.max_norm) { converged = true; break; }
    }

    // ---- eta diagnostic at the last sampled warp (optional) -----------------
    double eu = 0.0, ev = 0.0;
    const bool want_eta = (A.flags & GPV_SOLVE_ETA) && iters > 0 && status == GPV_OK;
    if (want_eta) {
        const double *pprev = sm.pprev;
        const double X0 = cx + pprev[0], Y0 = cy + pprev[1];
        const double bxd = floor(X0), byd = floor(Y0);
        const int wbx = (int)bxd, wby = (int)byd;
        const double ox = X0 - bxd, oy = Y0 - byd;
        for (int i = tid; i < NS; i += NT) {
            const int t = i % T, j = i / T;
            if (!((RVM[t] >> j) & 1)) continue;
            int dxi, dy0;
            unpack_task(tasks[t], dxi, dy0);
            const double dx = dxi, dy = dy0 + j;
            double lx = ox + dx, ly = oy + dy;
            if (ORDER >= 1) {
                lx += pprev[2] * dx + pprev[4] * dy;
                ly += pprev[3] * dx + pprev[5] * dy;
            }
            if (ORDER == 2) {
                lx += 0.5 * pprev[6 % M] * dx * dx + pprev[8 % M] * dx * dy + 0.5 * pprev[10 % M] * dy * dy;
                ly += 0.5 * pprev[7 % M] * dx * dx + pprev[9 % M] * dx * dy + 0.5 * pprev[11 % M] * dy * dy;
            }
            int ix, iy;
            float tx, ty;  // integer offsets added exactly, the small parts in FP32
            split_clamped(wbx + dxi, (float)(lx - dx), A.w, ix, tx);
            split_clamped(wby + dy0 + j, (float)(ly - dy), A.h, iy, ty);
            float a[6], b[6];
            basis(ty, a);
            basis(tx, b);
            RSG[i] = contract<float>(A.g32 + (int64_t)(iy + B - 2) * A.pitch32 + (ix + B - 2), A.pitch32, a, b);
        }
        __syncthreads();
        auto load = [&](int i, double &f, double &gx, double &gy, double &g, double &dx, double &dy) -> bool {
            const int t = i % T, j = i / T;
            if (!((RVM[t] >> j) & 1)) return false;
            int dxi, dy0;
            unpack_task(tasks[t], dxi, dy0);
            const float4 rec = REC[i];
            f = (double)rec.z + (double)shift;
            gx = rec.x; gy = rec.y; g = RSG[i];
            dx = dxi; dy = dy0 + j;
            return true;
        };
        auto red = [&](double v) { return run_block_sum<NT>(v, sm); };
        eta_sums<ORDER>(NS, tid, NT, dn, fm, df, gm_last, dg_last, load, red, eu, ev);
    }
    if (tid == 0) {
        gpv_subset_result *o = A.out + idx;
#pragma unroll
        for (int k = 0; k < 12; k++) o->p[k] = k < M ? sm.p[k % M] : 0.0;
        o->c_zncc = c_zncc;
        o->c_znssd = c_znssd;
        o->norm = last_norm;
        o->eta_u = eu;
        o->eta_v = ev;
        o->f_m = fm;
        o->delta_f = df;
        o->sssig = tot_sssig;
        o->sigma = sqrt(saa / dn);
        o->iterations = iters;
        o->converged = converged;
        o->quality_ok = converged && c_zncc >= A.tolerance;
        o->status = status;
        o->n_px = n;
        o->has_eta = want_eta;
        o->texture = 0;
        o->reserved = 0;
    }
}

// Claim a free scratch slot of the SM this block runs on (one block per
// subset): at most slots_per_sm blocks of a launch are resident on an SM
// and each frees its slot before it exits, so a bit is free when a block
// starts; the bounded wait only covers a block moved to another SM after a
// preemption.  -1: none claimed.
__device__ int run_claim_slot(const RunArgs &R) {
    unsigned smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    if ((int)smid >= R.n_mask) return -1;
    for (int attempt = 0; attempt < 20000; attempt++) {
        for (int j = 0; j < R.slots_per_sm; j++) {
            const unsigned bit = 1u << j;
            if (!(atomicOr(R.slot_mask + smid, bit) & bit)) return (int)smid * R.slots_per_sm + j;
        }
        __nanosleep(1000);
    }
    return -1;
}

// PER_SUBSET: one block per subset with a claimed scratch slot (subsets
// free SMs one at a time, for callers sharing the GPU); else a persistent
// grid whose blocks take subsets of their segment from the queue.
template <int ORDER, int NT, int K, bool PER_SUBSET, bool KAHAN>
__global__ void __launch_bounds__(NT, 512 / NT) icgn_runs(RunArgs R) {
    extern __shared__ float4 win4[];
    float *win = reinterpret_cast<float *>(win4);
    __shared__ RunSmem<NT / 32> sm;
    const KArgs &A = R.k;
    const int start = R.seg[0], count = R.seg[1];
    if (PER_SUBSET) {
        const int item = blockIdx.x;
        if (item >= count) return;
        if (threadIdx.x == 0) sm.item = run_claim_slot(R);
        __threadfence();
        __syncthreads();
        const int slot = sm.item;
        const int idx = A.order[start + item];
        const gpv_subset_desc d = A.desc[idx];
        if (slot < 0) {
            if (threadIdx.x == 0) write_failed(A, idx, d, 12, GPV_TIMEOUT, 0, 0.0, 0.0);
            return;
        }
        float *base = reinterpret_cast<float *>(A.scratch) + (int64_t)slot * A.scratch_stride;
        if (d.radius < 1 || d.radius > A.max_radius) {
            if (threadIdx.x == 0) write_failed(A, idx, d, 12, GPV_INVALID_SUBSET, 0, 0.0, 0.0);
        } else {
            run_subset<ORDER, NT, K, KAHAN>(R, idx, d, base, win, sm);
        }
        __threadfence();  // every scratch access of the block is done before the slot is free
        __syncthreads();
        if (threadIdx.x == 0) {
            const int own = sm.item;
            atomicAnd(R.slot_mask + own / R.slots_per_sm, ~(1u << (own % R.slots_per_sm)));
        }
        return;
    }
    float *base = reinterpret_cast<float *>(A.scratch) + (int64_t)blockIdx.x * A.scratch_stride;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) sm.item = atomicAdd(R.queue, 1);
        __syncthreads();
        const int item = sm.item;
        if (item >= count) break;
        const int idx = A.order[start + item];
        const gpv_subset_desc d = A.desc[idx];
        if (d.radius < 1 || d.radius > A.max_radius) {
            if (threadIdx.x == 0) write_failed(A, idx, d, 12, GPV_INVALID_SUBSET, 0, 0.0, 0.0);
            continue;
        }
        run_subset<ORDER, NT, K, KAHAN>(R, idx, d, base, win, sm);
    }
}

template <int NT, int K, bool PS, bool KH>
const void *run_kernel_t(int order) {
    return order == 2 ? (const void *)icgn_runs<2, NT, K, PS, KH>
                      : (order == 1 ? (const void *)icgn_runs<1, NT, K, PS, KH> : (const void *)icgn_runs<0, NT, K, PS, KH>);
}

template <int NT, int K, bool PS, bool KH>
void run_launch_t(int order, int blocks, size_t smem, cudaStream_t s, const RunArgs &R) {
    if (order == 2) icgn_runs<2, NT, K, PS, KH><<<blocks, NT, smem, s>>>(R);
    else if (order == 1) icgn_runs<1, NT, K, PS, KH><<<blocks, NT, smem, s>>>(R);
    else icgn_runs<0, NT, K, PS, KH><<<blocks, NT, smem, s>>>(R);
}

template <int NT, bool PS, bool KH>
const void *run_kernel_k(int order, int K) {
    return K == 4 ? run_kernel_t<NT, 4, PS, KH>(order) : run_kernel_t<NT, 8, PS, KH>(order);
}

template <int NT, bool PS, bool KH>
void run_launch_k(int order, int K, int blocks, size_t smem, cudaStream_t s, const RunArgs &R) {
    if (K == 4) run_launch_t<NT, 4, PS, KH>(order, blocks, smem, s, R);
    else run_launch_t<NT, 8, PS, KH>(order, blocks, smem, s, R);
}

// Instantiations: every (threads, run length, one block per subset); the
// compensated-sum form on persistent grids of 128 or 256 threads only.
template <int NT>
const void *run_kernel_nt(int order, int K, bool ps, bool kahan) {
    if constexpr (NT >= 128) {
        if (kahan) return run_kernel_k<NT, false, true>(order, K);
    }
    return ps ? run_kernel_k<NT, true, false>(order, K) : run_kernel_k<NT, false, false>(order, K);
}

template <int NT>
void run_launch_nt(int order, int K, bool ps, bool kahan, int blocks, size_t smem, cudaStream_t s, const RunArgs &R) {
    if constexpr (NT >= 128) {
        if (kahan) {
            run_launch_k<NT, false, true>(order, K, blocks, smem, s, R);
            return;
        }
    }
    if (ps) run_launch_k<NT, true, false>(order, K, blocks, smem, s, R);
    else run_launch_k<NT, false, false>(order, K, blocks, smem, s, R);
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side: run tables, sizes and launches (called by the batched launcher).
// ---------------------------------------------------------------------------

// Task tables for run lengths 4 and 8 and radii 1..max_radius: per task
// {dx (low 16 bits) | dy0 (high 16 bits), circle bits}, bands of K rows from
// dy = -r, the last band moved up to end at dy = r (its rows already in the
// band above masked off); columns [-w, w] with w the widest circle row of
// the band.
int ensure_run_tables(gpv_context *ctx, int max_radius) {
    if (max_radius <= ctx->run_table_radius) return GPV_SUCCESS;
    const int R1 = max_radius + 1;
    std::vector<int32_t> tab;  // pairs
    std::vector<int32_t> off(2 * R1, 0), cnt(2 * R1, 0);
    for (int kk = 0; kk < 2; kk++) {
        const int K = kRunLengths[kk];
        for (int r = 1; r <= max_radius; r++) {
            off[kk * R1 + r] = (int32_t)(tab.size() / 2);
            int n = 0;
            for (int b0 = -r; b0 <= r; b0 += K) {
                const int dy0 = (2 * r + 1 >= K) ? std::min(b0, r - K + 1) : -r;
                int w = -1;
                for (int j = 0; j < K; j++) {
                    const int y = dy0 + j;
                    if (y < b0 || y > r) continue;
                    // the row's exact integer half-width, then the band's widest
                    int h = (int)std::floor(std::sqrt((double)(r * r - y * y)));
                    while ((h + 1) * (h + 1) + y * y <= r * r) h++;
                    while (h > 0 && h * h + y * y > r * r) h--;
                    w = std::max(w, h);
                }
                for (int dx = -w; dx <= w; dx++) {
                    uint32_t bits = 0;
                    for (int j = 0; j < K; j++) {
                        const int y = dy0 + j;
                        if (y >= b0 && y <= r && dx * dx + y * y <= r * r) bits |= 1u << j;
                    }
                    tab.push_back((int32_t)((uint32_t)(dx & 0xffff) | ((uint32_t)dy0 << 16)));
                    tab.push_back((int32_t)bits);
                    n++;
                }
            }
            cnt[kk * R1 + r] = n;
        }
    }
    if (int rc = ctx->run_tasks.ensure(tab.size() * sizeof(int32_t))) return rc;
    if (int rc = ctx->run_off.ensure(off.size() * sizeof(int32_t))) return rc;
    if (int rc = ctx->run_n.ensure(cnt.size() * sizeof(int32_t))) return rc;
    GPV_CUDA_TRY(cudaMemcpy(ctx->run_tasks.ptr, tab.data(), tab.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    GPV_CUDA_TRY(cudaMemcpy(ctx->run_off.ptr, off.data(), off.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    GPV_CUDA_TRY(cudaMemcpy(ctx->run_n.ptr, cnt.data(), cnt.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    ctx->h_run_n = cnt;
    ctx->run_table_radius = max_radius;
    return GPV_SUCCESS;
}

int run_length_index(int K) { return K == kRunLengths[0] ? 0 : 1; }

// Window capacity (floats) of a launch for subsets up to radius rmax: the
// square of half side max(rmax, K - 1 - rmax) stretched by 6%, taps and
// margins, at a pitch of whole 32-float rows.
int run_window_cap(int rmax, int K) {
    const int e = std::max(rmax, K - 1 - rmax);
    const int rw = (int)std::ceil(1.06 * e) + 2;
    const int side = 2 * rw + 6 + 2 * kRunMargin + 4;
    return side * run_pitch(side);
}

// Record slots per block (largest radius's tasks x K, rounded to 32) and the
// scratch floats per block: a float4 record and an eta resample per slot +
// one validity word per task.
int64_t run_scratch_floats(gpv_context *ctx, int rmax, int K, int *nslot) {
    const int R1 = ctx->run_table_radius + 1;
    int T = 0;  // the most tasks of any radius up to rmax (the count is not monotone in r)
    for (int r = 1; r <= rmax; r++) T = std::max(T, (int)ctx->h_run_n[run_length_index(K) * R1 + r]);
    const int ns = (T * K + 31) / 32 * 32;
    *nslot = ns;
    return 5 * (int64_t)ns + (T + 31) / 32 * 32;
}

const void *run_kernel(int order, int nt, int K, bool per_subset, bool kahan) {
    if (nt == 64) return run_kernel_nt<64>(order, K, per_subset, kahan);
    return nt == 256 ? run_kernel_nt<256>(order, K, per_subset, kahan) : run_kernel_nt<128>(order, K, per_subset, kahan);
}

int run_launch(gpv_context *ctx, int order, int nt, int K, bool kahan, int blocks, size_t smem, cudaStream_t s,
               const KArgs &k, const int32_t *seg, int *queue, int win_cap, int nslot, uint32_t *slot_mask,
               int slots_per_sm, int n_mask) {
    RunArgs R;
    R.k = k;
    const int R1 = ctx->run_table_radius + 1, kk = run_length_index(K);
    R.tasks = static_cast<const int2 *>(ctx->run_tasks.ptr);
    R.task_off = static_cast<const int32_t *>(ctx->run_off.ptr) + kk * R1;
    R.task_n = static_cast<const int32_t *>(ctx->run_n.ptr) + kk * R1;
    R.seg = seg;
    R.queue = queue;
    R.win_cap = win_cap;
    R.nslot = nslot;
    R.slot_mask = slot_mask;
    R.slots_per_sm = slots_per_sm;
    R.n_mask = n_mask;
    const bool ps = slot_mask != nullptr;
    if (kahan && (ps || nt == 64)) {
        set_error("the compensated-sum form runs on persistent grids of 128 or 256 threads");
        return GPV_ERR_INVALID;
    }
    if (nt == 64) run_launch_nt<64>(order, K, ps, kahan, blocks, smem, s, R);
    else if (nt == 256) run_launch_nt<256>(order, K, ps, kahan, blocks, smem, s, R);
    else run_launch_nt<128>(order, K, ps, kahan, blocks, smem, s, R);
    GPV_CUDA_TRY(cudaGetLastError());
    return GPV_SUCCESS;
}

}  // namespace gpv
