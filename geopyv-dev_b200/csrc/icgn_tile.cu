// icgn_tile.cu -- mixed-precision ICGN, one thread block per subset, the
// subset's coefficient window staged in shared memory.
//
// Same algorithm and numerics as the warp-per-subset kernel (icgn.cu) --
// Subset::new + solve_icgn_result, src/subset.rs:836-919, 1117-1219 -- with
// a different execution layout:
//  * 4 warps solve one subset; pixels are dealt round-robin in the row-major
//    order of the circular template, so each warp covers 32 neighbouring
//    pixels of a template row and the 6x6 windows of its lanes overlap.
//  * The block of coefficients the subset can touch is copied once into
//    shared memory with 16-byte vector loads (f's window for the setup, g's
//    for the iterations) with a margin of kMargin px.  Every iteration checks
//    (from the warp parameters, conservatively) that the warped subset still
//    lies inside the staged block and re-stages when it does not; a subset
//    whose block exceeds the shared-memory capacity reads global memory for
//    that iteration.  Window indices are clamped, so no access can leave the
//    staged block whatever the warp.
//  * One kernel per warp order (fewer registers, smaller code); the batch is
//    partitioned by order on the device and the three kernels run on three
//    streams so each one's tail overlaps the next one's start.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <set>
#include <utility>
#include <type_traits>

#include "icgn_common.cuh"

namespace gpv {
namespace {

constexpr int kMaxTileWarps = 8;  // blocks of 128 or 256 threads
constexpr int kMargin = 4;

struct TileSmem {
    double mom[3 * 15];
    double H[144];
    double Hinv[144];
    double aug[384];  // setup sums [0, 96), Gauss-Jordan workspace [96, 384)
    double A[12], S[12];
    double p[12], pprev[12], dp[12], grad[12];
    double red[kMaxTileWarps][16];
    double redt[kMaxTileWarps][16];  // rigid texture: the template pass's warp sums (order 2), or the
                                     // fixed grain moments (redt[0..1]) and G's coefficients (redt[2]) (order 1)
    double red2[kMaxTileWarps][80];  // setup: one combined reduction
    double tot[16];
    double tt[16];  // rigid texture: the template pass's block sums
    double misc[10];
    int flag[4];
    int item;
    int n_valid;
    int win_r0, win_c0, win_h, win_w, win_ok;
};

struct TileArgs {
    KArgs k;
    const int32_t *seg;  // [start, count] of this order's segment in k.order
    int *queue;          // this kernel's work-queue counter (persistent grid)
    int win_cap;         // floats of dynamic shared memory for the window
    int layout;          // template slots: kLayoutCompact, kLayoutRows or kLayoutTiles
    // one block per subset (slot_mask != nullptr): a block claims one of the
    // slots_per_sm scratch slots of the SM it starts on (a bit of
    // slot_mask[smid], n_mask words) and frees it when the subset is done
    uint32_t *slot_mask;
    int slots_per_sm, n_mask;
};

// Template slot layouts: the compact scan order; rows padded to whole warps
// (a warp never straddles two rows); 8 x 4 tiles, one per warp, read from a
// window whose pitch is 8 mod 32 so a tile's 32 lanes hit 32 different banks.
constexpr int kLayoutCompact = 0, kLayoutRows = 1, kLayoutTiles = 2;

// Row pitch (floats) of a window `ww` columns wide in a layout.
__host__ __device__ __forceinline__ int window_pitch(int ww, int layout) {
    return layout == kLayoutTiles ? ww + ((8 - ww) % 32 + 32) % 32 : ww;
}

// Copy coefficient rows [r0, r0+wh) x cols [c0, c0+ww) (c0, ww multiples of 4)
// into win (row pitch ww).  Out-of-range rows / columns are clamped.
template <int NT>
__device__ __forceinline__ void stage(const float *__restrict__ C, int64_t pitch, int ch, int r0, int c0, int wh,
                                      int ww, float *win) {
    const int nv = ww >> 2;
    for (int idx = threadIdx.x; idx < wh * nv; idx += NT) {
        const int rr = idx / nv, cc = (idx - rr * nv) << 2;
        int row = r0 + rr;
        row = row < 0 ? 0 : (row > ch - 1 ? ch - 1 : row);
        int col = c0 + cc;
        col = col < 0 ? 0 : (col > (int)pitch - 4 ? (int)pitch - 4 : col);
        const float4 v = __ldg(reinterpret_cast<const float4 *>(C + (int64_t)row * pitch + col));
        *reinterpret_cast<float4 *>(win + rr * ww + cc) = v;
    }
}

// Same with threads [t0, NT) only (the others are busy elsewhere).
template <int NT>
__device__ __forceinline__ void stage_part(const float *__restrict__ C, int64_t pitch, int ch, int r0, int c0, int wh,
                                           int ww, float *win, int t0) {
    const int nv = ww >> 2;
    for (int idx = (int)threadIdx.x - t0; idx < wh * nv; idx += NT - t0) {
        const int rr = idx / nv, cc = (idx - rr * nv) << 2;
        int row = r0 + rr;
        row = row < 0 ? 0 : (row > ch - 1 ? ch - 1 : row);
        int col = c0 + cc;
        col = col < 0 ? 0 : (col > (int)pitch - 4 ? (int)pitch - 4 : col);
        const float4 v = __ldg(reinterpret_cast<const float4 *>(C + (int64_t)row * pitch + col));
        *reinterpret_cast<float4 *>(win + rr * ww + cc) = v;
    }
}

// Plan a window covering pixel indices [xlo, xhi] x [ylo, yhi] (already
// clamped to the image) plus kMargin; returns false if it does not fit.
__device__ __forceinline__ bool plan_window(int xlo, int xhi, int ylo, int yhi, int border, int cap, int layout,
                                            int &r0, int &c0, int &wh, int &ww) {
    for (int m = kMargin; m >= 0; m -= kMargin) {
        const int clo = xlo + border - 2 - m, chi = xhi + border + 3 + m;
        c0 = clo >= 0 ? (clo & ~3) : -(((-clo) + 3) & ~3);
        ww = window_pitch(((chi + 1 - c0) + 3) & ~3, layout);
        r0 = ylo + border - 2 - m;
        wh = yhi + border + 3 + m + 1 - r0;
        if (ww * wh <= cap) return true;
        if (m == 0) break;
    }
    return false;
}

__device__ __forceinline__ bool window_covers(const TileSmem &sm, int xlo, int xhi, int ylo, int yhi, int border) {
    if (!sm.win_ok) return false;
    return xlo + border - 2 >= sm.win_c0 && xhi + border + 3 < sm.win_c0 + sm.win_w && ylo + border - 2 >= sm.win_r0 &&
           yhi + border + 3 < sm.win_r0 + sm.win_h;
}

// Warp sums of K FP32 per-thread values (FP64 totals) into dst[0..K), in
// transposed reductions of up to 16 values.
template <int K, int C = 0>
__device__ __forceinline__ void warp_sums_chunked(const float (&a)[K], double *dst, int lane) {
    if constexpr (C < K) {
        constexpr int N = (K - C) < 16 ? (K - C) : 16;
        double v[N];
#pragma unroll
        for (int j = 0; j < N; j++) v[j] = (double)a[C + j];
        warp_sum_many<N>(v, dst + C, lane);
        warp_sums_chunked<K, C + N>(a, dst, lane);
    }
}

// Sum K per-thread values over the block into sm.tot[0..K) (FP64).
template <int NT, int K>
__device__ __forceinline__ void block_reduce(const double (&v)[K], TileSmem &sm) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const double s = warp_sum(v[k]);
        if (lane == 0) sm.red[wid][k] = s;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < NT / 32; w++) s += sm.red[w][threadIdx.x];
        sm.tot[threadIdx.x] = s;
    }
    __syncthreads();
}

template <int NT>
__device__ __forceinline__ double block_sum1(double v, TileSmem &sm) {
    const double a[1] = {v};
    block_reduce<NT, 1>(a, sm);
    return sm.tot[0];
}

// Pixel extent (in image pixels, clamped) touched by the warp p of a radius-r
// subset centred at (cx, cy), conservatively.
template <int ORDER>
__device__ void warp_extent(const double *p, double cx, double cy, int r, int w, int h, int &xlo, int &xhi, int &ylo,
                            int &yhi, bool *inside = nullptr) {
    double ex = r, ey = r;
    if (ORDER >= 1) {
        ex = r * (fabs(1.0 + p[2]) + fabs(p[4]));
        ey = r * (fabs(p[3]) + fabs(1.0 + p[5]));
    }
    if (ORDER == 2) {
        const double rr = 0.5 * (double)r * r;
        ex += rr * (fabs(p[6 % 12]) + 2.0 * fabs(p[8 % 12]) + fabs(p[10 % 12]));
        ey += rr * (fabs(p[7 % 12]) + 2.0 * fabs(p[9 % 12]) + fabs(p[11 % 12]));
    }
    const double X0 = cx + p[0], Y0 = cy + p[1];
    double a = floor(X0 - ex) - 1.0, b = floor(X0 + ex) + 1.0, c = floor(Y0 - ey) - 1.0, d = floor(Y0 + ey) + 1.0;
    if (!(isfinite(a) && isfinite(b) && isfinite(c) && isfinite(d))) {
        xlo = 0; xhi = w - 1; ylo = 0; yhi = h - 1;  // plans a window that cannot fit: global path
        if (inside) *inside = false;
        return;
    }
    // inside: the extent (with its one-pixel margin) lies in the image, so no
    // sample position meets the edge clamp
    if (inside) *inside = a >= 0.0 && b <= (double)(w - 1) && c >= 0.0 && d <= (double)(h - 1);
    xlo = (int)fmax(0.0, fmin(a, (double)(w - 1)));
    xhi = (int)fmax(0.0, fmin(b, (double)(w - 1)));
    ylo = (int)fmax(0.0, fmin(c, (double)(h - 1)));
    yhi = (int)fmax(0.0, fmin(d, (double)(h - 1)));
}

// Per-pixel record kept between the setup and the iterations: f, df/dx,
// df/dy and the template offset (dx, dy) packed as two int16 in the last
// word.  f = NaN marks a pixel removed by the global mask.
__device__ __forceinline__ float4 pack_px(float f, float gx, float gy, int dx, int dy) {
    return make_float4(f, gx, gy, __int_as_float((dx & 0xffff) | (dy << 16)));
}
__device__ __forceinline__ void unpack_off(float w, float &dx, float &dy) {
    const int v = __float_as_int(w);
    dx = (float)(int)(short)(v & 0xffff);
    dy = (float)(v >> 16);
}

// The three grain maps (fxx, fyy, fxy; rows x cols FP32) at (x = column,
// y = row), bilinear, clamped (GrainMaps::sample, src/texture.rs:125-143).
__device__ __forceinline__ void grain_sample(const float *maps, int rows, int cols, double x, double y, float h[3]) {
    x = fmin(fmax(x, 0.0), (double)(cols - 1));
    y = fmin(fmax(y, 0.0), (double)(rows - 1));
    const int x0 = min((int)floor(x), max(cols - 2, 0)), y0 = min((int)floor(y), max(rows - 2, 0));
    const int x1 = min(x0 + 1, cols - 1), y1 = min(y0 + 1, rows - 1);
    const double tx = x - (double)x0, ty = y - (double)y0;
    const int64_t np = (int64_t)rows * cols;
#pragma unroll
    for (int m = 0; m < 3; m++) {
        const float *M = maps + m * np;
        h[m] = (float)((1.0 - ty) * ((1.0 - tx) * M[(int64_t)y0 * cols + x0] + tx * M[(int64_t)y0 * cols + x1]) +
                       ty * ((1.0 - tx) * M[(int64_t)y1 * cols + x0] + tx * M[(int64_t)y1 * cols + x1]));
    }
}

// Green-Lagrange strain [Exx, Eyy, Exy] (src/texture.rs:200-206).
__device__ __forceinline__ void green_lagrange(float ux, float vx, float uy, float vy, float &e0, float &e1, float &e2) {
    e0 = ux + 0.5f * (ux * ux + vx * vx);
    e1 = vy + 0.5f * (uy * uy + vy * vy);
    e2 = 0.5f * (uy + vx) + 0.5f * (ux * uy + vx * vy);
}

// RIGID: the rigid-texture template (Texture::Rigid) when the reference image
// has measurable speckle: the maps at the subset pixels in setup (Sh: 3
// arrays of n_max), and every iteration a template pass storing the
// correction G(E(p)) per pixel (St; the template is t = f + G,
// grain_template src/texture.rs:213-244) with its warp sums, so the update
// compares g with the template (src/subset.rs:1151-1168): t - t_m in the
// cross term and the gradient, the template's spread instead of delta_f.
// The template's sums are formed as the setup's fixed FP64 sums of f - f_m
// plus per-iteration sums of the small G (sum G, sum G^2, sum (f - f_m) G,
// sum SDI_j G), so the FP32 rounding of the per-iteration pass scales with
// the strain and vanishes at zero strain, as the deformable sums do.
// Order 1 has a uniform strain, so G = c . (h0, h1, h2, f - f_m) with four
// coefficients per iteration, and those sums follow in closed form from
// fixed setup moments of the grain samples (sum h_k, h_k h_l, (f - f_m) h_k,
// SDI_j h_k): no template pass, only sum h_k (g - f_m) in the sample loop.
template <int ORDER, int NT, bool RIGID>
__device__ void tile_subset(const TileArgs &T, int idx, const gpv_subset_desc &d, float4 *S4, float *Sg, float *win,
                            TileSmem &sm, float *Sh, float *St, int64_t nmax) {
    const KArgs &A = T.k;
    using O = Ord<ORDER>;
    constexpr int M = O::M, NMU = O::NMU, NMOM = O::NMOM;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int r = d.radius;
    // compact template, rows padded to whole warps, or 8 x 4 tiles (empty slots: x = -32768)
    const int tab = T.layout * (A.table_radius + 1) + r;
    const int npx_t = A.tab_n[tab];
    const short2 *po = (T.layout != kLayoutCompact ? A.slots : A.offs) + A.tab_off[tab];
    const double cx = d.coord[0], cy = d.coord[1];
    const int cxi = (int)cx, cyi = (int)cy;
    const double fxd = floor(cx), fyd = floor(cy);
    const int bx = (int)fxd, by = (int)fyd;
    const float fx = (float)(cx - fxd), fy = (float)(cy - fyd);
    const int B = A.border, ch = A.h + 2 * B;
    const bool rigid_on = RIGID && A.grain_scal[4] != 0.0;  // uniform: maps built
    const float s2f = RIGID ? (float)A.grain_scal[2] : 0.f;
    double *const gq = &sm.redt[0][0], *const gcoef = &sm.redt[2][0];  // order-1 rigid

    // ---- stage f's window ------------------------------------------------
    {
        // +-1: an FP32 fraction can round up to the next integer
        const int xlo = max(0, min(bx - r - 1, A.w - 1)), xhi = max(0, min(bx + r + 1, A.w - 1));
        const int ylo = max(0, min(by - r - 1, A.h - 1)), yhi = max(0, min(by + r + 1, A.h - 1));
        int r0, c0, wh, ww;
        const bool ok = plan_window(xlo, xhi, ylo, yhi, B, T.win_cap, T.layout, r0, c0, wh, ww);
        if (ok) stage<NT>(A.f32, A.pitch32, ch, r0, c0, wh, ww, win);
        if (tid == 0) {
            sm.win_ok = 0;  // g must be staged before the iterations
            sm.win_r0 = r0; sm.win_c0 = c0; sm.win_h = wh; sm.win_w = ww;
            sm.flag[2] = ok;
        }
        __syncthreads();
    }
    const bool f_staged = sm.flag[2] != 0;
    const int fr0 = sm.win_r0, fc0 = sm.win_c0, fwh = sm.win_h, fww = sm.win_w;
    // interior subset: every template pixel sits at integer offsets from
    // (cx, cy) inside the image, so all share one fraction and one basis
    const bool interior = f_staged && bx - r >= 0 && bx + r <= A.w - 1 && by - r >= 0 && by + r <= A.h - 1;

    // ---- setup --------------------------------------------------------------
    // pass 1 samples f and its gradient (records) and accumulates, about a
    // subset-uniform level s (a coefficient near the centre; it keeps the
    // sums free of cancellation and a flat subset's sums exactly zero),
    //   [count, sum (f-s), sum (f-s)^2, SSSIG, Bf_j = sum SDI_j (f-s) (M), S_j = sum SDI_j (M)];
    // pass 2 (each thread re-reads its own records: no barrier) accumulates
    // the 3*NMOM gradient moments of the Hessian.  FP32 partials per thread,
    // combined across the block in FP64 by one reduction; then warp 0 forms
    // A_j = Bf_j - (f_m - s) S_j, delta_f, H and H^-1 while the other warps stage
    // g's window for the first iteration.
    constexpr int NVA = 4 + 2 * M, NV = NVA + 3 * NMOM;
    float acc[NVA];
#pragma unroll
    for (int q = 0; q < NVA; q++) acc[q] = 0.f;
    // the shift level: the coefficient under the subset centre (uniform)
    float shift = 0.f;
    if (f_staged) {
        const int wx = min(max(max(0, min(bx, A.w - 1)) + B - fc0, 0), fww - 1);
        const int wy = min(max(max(0, min(by, A.h - 1)) + B - fr0, 0), fwh - 1);
        shift = win[wy * fww + wx];
    } else {
        shift = A.f32[(int64_t)(max(0, min(by, A.h - 1)) + B) * A.pitch32 + max(0, min(bx, A.w - 1)) + B];
    }
    {
        float a0[6], da0[6], b0[6], db0[6];
        basis(fy, a0); dbasis(fy, da0);
        basis(fx, b0); dbasis(fx, db0);
        float2 bb0[6], dbb0[6];  // the column weights as duplicated pairs (paired taps)
#pragma unroll
        for (int k = 0; k < 6; k++) {
            bb0[k] = make_float2(b0[k], b0[k]);
            dbb0[k] = make_float2(db0[k], db0[k]);
        }
        for (int i = tid; i < npx_t; i += NT) {
            const short2 o = po[i];
            if (o.x == -32768 || !mask_ok(A, cxi, cyi, o.x, o.y)) {
                S4[i] = pack_px(__int_as_float(0x7fc00000), 0.f, 0.f, 0, 0);
                continue;
            }
            float gx, gy, f;
            if (interior) {
                const int wx = bx + o.x + B - 2 - fc0, wy = by + o.y + B - 2 - fr0;
                f = contract_grad_rows2(win + wy * fww + wx, fww, a0, da0, bb0, dbb0, gx, gy);
            } else {
                int ix, iy;
                float tx, ty;
                split_clamped(bx, fx + (float)o.x, A.w, ix, tx);
                split_clamped(by, fy + (float)o.y, A.h, iy, ty);
                float a[6], da[6], b[6], db[6];
                basis(ty, a); dbasis(ty, da);
                basis(tx, b); dbasis(tx, db);
                if (f_staged) {
                    const int wx = min(max(ix + B - 2 - fc0, 0), fww - 6), wy = min(max(iy + B - 2 - fr0, 0), fwh - 6);
                    f = contract_grad<float>(win + wy * fww + wx, fww, a, da, b, db, gx, gy);
                } else {
                    const float *F = A.f32 + (int64_t)(iy + B - 2) * A.pitch32 + (ix + B - 2);
                    f = contract_grad<float>(F, A.pitch32, a, da, b, db, gx, gy);
                }
            }
            S4[i] = pack_px(f, gx, gy, o.x, o.y);
            if (RIGID && rigid_on) {
                float hv[3];
                grain_sample(A.grain, A.h, A.w, cx + (double)o.x, cy + (double)o.y, hv);
                Sh[i] = hv[0];
                Sh[nmax + i] = hv[1];
                Sh[2 * nmax + i] = hv[2];
            }
            const float dx = (float)o.x, dy = (float)o.y;
            const float fs = f - shift;
            acc[0] += 1.f;
            acc[1] += fs;
            acc[2] = fmaf(fs, fs, acc[2]);
            acc[3] = fmaf(0.5f * gx, gx, fmaf(0.5f * gy, gy, acc[3]));
            const float gxf = gx * fs, gyf = gy * fs;
#pragma unroll
            for (int mu = 0; mu < NMU; mu++) {
                const float mv = mu_val<float>(mu, dx, dy);
                acc[4 + 2 * mu] = fmaf(gxf, mv, acc[4 + 2 * mu]);
                acc[5 + 2 * mu] = fmaf(gyf, mv, acc[5 + 2 * mu]);
                acc[4 + M + 2 * mu] = fmaf(gx, mv, acc[4 + M + 2 * mu]);
                acc[5 + M + 2 * mu] = fmaf(gy, mv, acc[5 + M + 2 * mu]);
            }
        }
    }
    // warp partials of pass 1 straight into red2 (frees the accumulators),
    // up to 16 values per transposed reduction
    warp_sums_chunked<NVA>(acc, sm.red2[wid], lane);
    {
        float mom[3 * NMOM];
#pragma unroll
        for (int q = 0; q < 3 * NMOM; q++) mom[q] = 0.f;
        if constexpr (ORDER == 0) {
            for (int i = tid; i < npx_t; i += NT) {
                const float4 rec = S4[i];
                if (rec.x != rec.x) continue;
                mom[0] += rec.y * rec.y;
                mom[1] += rec.y * rec.z;
                mom[2] += rec.z * rec.z;
            }
        } else {
            // the monomials in (x, y) pairs: (dx^e, dy^e) for e = 1..2 DEG,
            // (dx^2 dy, dx dy^2) and (dx^3 dy, dx dy^3); dx dy and dx^2 dy^2
            // alone; each moment takes one FMA per pixel, as a paired or a
            // plain FP32 op, in pixel order
            constexpr int E = 2 * O::DEG;
            float2 mp[3][E], m21[3], m31[3];
            float m00[3], m11[3], m22[3];
#pragma unroll
            for (int p = 0; p < 3; p++) {
#pragma unroll
                for (int e = 0; e < E; e++) mp[p][e] = make_float2(0.f, 0.f);
                m21[p] = m31[p] = make_float2(0.f, 0.f);
                m00[p] = m11[p] = m22[p] = 0.f;
            }
            for (int i = tid; i < npx_t; i += NT) {
                const float4 rec = S4[i];
                if (rec.x != rec.x) continue;
                float dx, dy;
                unpack_off(rec.w, dx, dy);
                const float gx = rec.y, gy = rec.z;
                float2 P[E];
                P[0] = make_float2(dx, dy);
#pragma unroll
                for (int e = 1; e < E; e++) P[e] = __fmul2_rn(P[e - 1], P[0]);
                const float d11 = dx * dy;
                const float gg[3] = {gx * gx, gx * gy, gy * gy};
                float2 X21, X31;
                float d22 = 0.f;
                if (ORDER == 2) {
                    const float2 sw = make_float2(dy, dx);
                    X21 = __fmul2_rn(P[1], sw);
                    X31 = __fmul2_rn(P[2], sw);
                    d22 = P[1].x * P[1].y;
                }
#pragma unroll
                for (int p = 0; p < 3; p++) {
                    const float2 G2 = make_float2(gg[p], gg[p]);
                    m00[p] += gg[p];
#pragma unroll
                    for (int e = 0; e < E; e++) mp[p][e] = __ffma2_rn(G2, P[e], mp[p][e]);
                    m11[p] = fmaf(gg[p], d11, m11[p]);
                    if (ORDER == 2) {
                        m21[p] = __ffma2_rn(G2, X21, m21[p]);
                        m31[p] = __ffma2_rn(G2, X31, m31[p]);
                        m22[p] = fmaf(gg[p], d22, m22[p]);
                    }
                }
            }
#pragma unroll
            for (int p = 0; p < 3; p++) {
                float *m = mom + p * NMOM;
                m[mom_idx(0, 0)] = m00[p];
                m[mom_idx(1, 1)] = m11[p];
#pragma unroll
                for (int e = 1; e <= E; e++) {
                    m[mom_idx(e, 0)] = mp[p][e - 1].x;
                    m[mom_idx(0, e)] = mp[p][e - 1].y;
                }
                if (ORDER == 2) {
                    m[mom_idx(2, 1)] = m21[p].x;
                    m[mom_idx(1, 2)] = m21[p].y;
                    m[mom_idx(3, 1)] = m31[p].x;
                    m[mom_idx(1, 3)] = m31[p].y;
                    m[mom_idx(2, 2)] = m22[p];
                }
            }
        }
        warp_sums_chunked<3 * NMOM>(mom, sm.red2[wid] + NVA, lane);
    }
    if (RIGID && ORDER == 1 && rigid_on) {
        // grain moments: [0,3) h_k, [3,9) h_k h_l (00 01 02 11 12 22),
        // [9,12) (f - s) h_k, [12,30) SDI_j h_k at 12 + 3 j + k
        float gm[30];
#pragma unroll
        for (int q = 0; q < 30; q++) gm[q] = 0.f;
        for (int i = tid; i < npx_t; i += NT) {
            const float4 rec = S4[i];
            if (rec.x != rec.x) continue;
            float dx, dy;
            unpack_off(rec.w, dx, dy);
            const float h[3] = {Sh[i], Sh[nmax + i], Sh[2 * nmax + i]};
            const float fs = rec.x - shift;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                gm[k] += h[k];
                gm[9 + k] = fmaf(fs, h[k], gm[9 + k]);
            }
            gm[3] = fmaf(h[0], h[0], gm[3]); gm[4] = fmaf(h[0], h[1], gm[4]); gm[5] = fmaf(h[0], h[2], gm[5]);
            gm[6] = fmaf(h[1], h[1], gm[6]); gm[7] = fmaf(h[1], h[2], gm[7]); gm[8] = fmaf(h[2], h[2], gm[8]);
#pragma unroll
            for (int mu = 0; mu < NMU; mu++) {
                const float mv = mu_val<float>(mu, dx, dy), sx = rec.y * mv, sy = rec.z * mv;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    gm[12 + 3 * (2 * mu) + k] = fmaf(sx, h[k], gm[12 + 3 * (2 * mu) + k]);
                    gm[12 + 3 * (2 * mu + 1) + k] = fmaf(sy, h[k], gm[12 + 3 * (2 * mu + 1) + k]);
                }
            }
        }
        warp_sums_chunked<30>(gm, sm.red2[wid] + NV, lane);
    }
    __syncthreads();
    if (wid == 0) {
        // sum the warp partials: aug[0..NV) (+ 30 grain moments, order-1 rigid)
        const int nv = NV + ((RIGID && ORDER == 1 && rigid_on) ? 30 : 0);
        for (int q = lane; q < nv; q += 32) {
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
            if (RIGID && ORDER == 1 && rigid_on && lane < 30)  // (f - s) h_k -> (f - f_m) h_k
                gq[lane] = (lane >= 9 && lane < 12) ? sm.aug[NV + lane] - ms * sm.aug[NV + lane - 9] : sm.aug[NV + lane];
            __syncwarp();
            assemble_hessian<ORDER>(sm.mom, sm.H, lane);
            if (!spd_inverse_warp<M>(sm.H, sm.aug + 96, sm.Hinv, lane)) st = GPV_SINGULAR_H;
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
        // meanwhile: stage g's window around the initial warp
        int xlo, xhi, ylo, yhi, r0 = 0, c0 = 0, wh = 0, ww = 0;
        double p0[12];
#pragma unroll
        for (int k = 0; k < 12; k++) p0[k] = d.p0[k % M];
        warp_extent<ORDER>(p0, cx, cy, r, A.w, A.h, xlo, xhi, ylo, yhi);
        const bool ok = plan_window(xlo, xhi, ylo, yhi, B, T.win_cap, T.layout, r0, c0, wh, ww);
        if (ok) stage_part<NT>(A.g32, A.pitch32, ch, r0, c0, wh, ww, win, 32);
        if (tid == 32) {
            sm.win_ok = ok;
            sm.win_r0 = r0; sm.win_c0 = c0; sm.win_h = wh; sm.win_w = ww;
        }
    }
    __syncthreads();
    const int st0 = sm.flag[0];
    const int n = sm.n_valid;
    const double dn = (double)n;
    const double fm = sm.misc[5], saa = sm.misc[6], tot_sssig = sm.misc[7];
    const float fmf = (float)fm;
    const double sa = 0.0;  // sum (f - f_m) is zero by construction of f_m
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

    // ---- ICGN iterations --------------------------------------------------
    const double size = sqrt(dn);
    int iters = 0, status = GPV_OK;
    bool converged = false;
    double c_zncc = 0.0, c_znssd = 4.0, last_norm = 0.0, gm_last = 0.0, dg_last = 0.0;
    for (int it = 1; it <= A.max_iter; it++) {
        // (re)stage g's window when the warped subset has left it
        bool inside;
        {
            int xlo, xhi, ylo, yhi;
            warp_extent<ORDER>(sm.p, cx, cy, r, A.w, A.h, xlo, xhi, ylo, yhi, &inside);
            if (!window_covers(sm, xlo, xhi, ylo, yhi, B)) {
                int r0, c0, wh, ww;
                const bool ok = plan_window(xlo, xhi, ylo, yhi, B, T.win_cap, T.layout, r0, c0, wh, ww);
                __syncthreads();  // nobody still reads the old window
                if (ok) stage<NT>(A.g32, A.pitch32, ch, r0, c0, wh, ww, win);
                if (tid == 0) {
                    sm.win_ok = ok;
                    sm.win_r0 = r0; sm.win_c0 = c0; sm.win_h = wh; sm.win_w = ww;
                }
                __syncthreads();
            }
        }
        const bool staged = sm.win_ok != 0;
        const int gr0 = sm.win_r0, gc0 = sm.win_c0, gwh = sm.win_h, gww = sm.win_w;
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
        // window-relative base: sample (ix, iy) reads win[(iy + B-2 - r0) * ww + (ix + B-2 - c0)]
        const int offx = B - 2 - gc0, offy = B - 2 - gr0;
        if (RIGID && rigid_on && ORDER == 2) {
            // template pass: G per pixel, sums of G, G^2, (f - f_m) G and
            // SDI_j G (their warp sums meet the iteration's reduction)
            constexpr int NT_ = 3 + M;
            float ta[NT_];
#pragma unroll
            for (int q = 0; q < NT_; q++) ta[q] = 0.f;
            float e0u = 0.f, e1u = 0.f, e2u = 0.f;
            if (ORDER == 1) green_lagrange(ux, vx, uy, vy, e0u, e1u, e2u);
            const float q6 = ORDER == 2 ? (float)sm.p[6 % M] : 0.f, q7 = ORDER == 2 ? (float)sm.p[7 % M] : 0.f;
            const float q8 = ORDER == 2 ? (float)sm.p[8 % M] : 0.f, q9 = ORDER == 2 ? (float)sm.p[9 % M] : 0.f;
            const float q10 = ORDER == 2 ? (float)sm.p[10 % M] : 0.f, q11 = ORDER == 2 ? (float)sm.p[11 % M] : 0.f;
            for (int i = tid; i < npx_t; i += NT) {
                const float4 rec = S4[i];
                if (rec.x != rec.x) continue;
                float dx, dy;
                unpack_off(rec.w, dx, dy);
                float e0 = e0u, e1 = e1u, e2 = e2u;
                if (ORDER == 2)
                    green_lagrange(ux + q6 * dx + q8 * dy, vx + q7 * dx + q9 * dy, uy + q8 * dx + q10 * dy,
                                   vy + q9 * dx + q11 * dy, e0, e1, e2);
                const float h0 = Sh[i], h1 = Sh[nmax + i], h2 = Sh[2 * nmax + i];
                const float fc = rec.x - fmf;
                const float G = -0.5f * s2f * (e0 * h0 + e1 * h1 + 2.0f * e2 * h2) - (e0 + e1) * fc;
                St[i] = G;
                ta[0] += G;
                ta[1] = fmaf(G, G, ta[1]);
                ta[2] = fmaf(fc, G, ta[2]);
                const float gxt = rec.y * G, gyt = rec.z * G;
#pragma unroll
                for (int mu = 0; mu < NMU; mu++) {
                    const float mv = mu_val<float>(mu, dx, dy);
                    ta[3 + 2 * mu] = fmaf(gxt, mv, ta[3 + 2 * mu]);
                    ta[4 + 2 * mu] = fmaf(gyt, mv, ta[4 + 2 * mu]);
                }
            }
            double tv[NT_];
#pragma unroll
            for (int q = 0; q < NT_; q++) tv[q] = (double)ta[q];
            warp_sum_many<NT_>(tv, sm.redt[wid], lane);
        }
        double s1 = 0.0, s2 = 0.0, sfg = 0.0;
        float pb[M];
#pragma unroll
        for (int j = 0; j < M; j++) pb[j] = 0.f;
        float4 rec_next = tid < npx_t ? S4[tid] : make_float4(0.f, 0.f, 0.f, 0.f);
        constexpr bool kClosed = RIGID && ORDER == 1;  // order-1 rigid: sums of h_k (g - f_m)
        double sh0 = 0.0, sh1 = 0.0, sh2 = 0.0;
        // the sample loop, specialised for subsets whose warped extent lies
        // inside the image and the staged window (no clamps per sample)
        const bool fast = staged && inside;
        const int wx0 = wbx + offx, wy0 = wby + offy;
        auto sweep = [&](auto fast_tag, auto dense_tag) {
            constexpr bool FAST = decltype(fast_tag)::value;
            constexpr bool DENSE = decltype(dense_tag)::value;  // no masked pixel: every record is valid
            // orders 1-2 without clamps: the warp and the gradient sums as
            // (x, y) pairs of paired FP32 ops (the same operations per lane)
            // (not for the closed-form first-order rigid loop, where it measured slower)
            constexpr bool kPair = FAST && (ORDER == 2 || (ORDER == 1 && !RIGID));
            // the warp's pairs in (y, x) order, as the weights take them
            const float2 U1 = make_float2(vx, ux), U2 = make_float2(vy, uy), O2 = make_float2(oy, ox);
            const float2 Q1 = make_float2(vxx, uxx), Q2 = make_float2(vxy, uxy), Q3 = make_float2(vyy, uyy);
            float2 pbp[6];
#pragma unroll
            for (int j = 0; j < 6; j++) pbp[j] = make_float2(0.f, 0.f);
            for (int base = 0; base < npx_t; base += NT * kChunk) {
                float p1 = 0.f, p2 = 0.f, pfg = 0.f, ph0 = 0.f, ph1 = 0.f, ph2 = 0.f;
#pragma unroll 2
                for (int c = 0; c < kChunk; c++) {
                    const int i = base + c * NT + tid;
                    if (i < npx_t) {
                        const float4 rec = rec_next;  // loaded one sample ahead
                        if (i + NT < npx_t) rec_next = S4[i + NT];
                        const float fv = rec.x;
                        if (DENSE || fv == fv) {
                            float dx, dy;
                            unpack_off(rec.w, dx, dy);
                            float lx, ly;
                            float dxx = 0.f, dxy = 0.f, dyy = 0.f;
                            float2 D2, E2, DXX, DXY, DYY, L;  // L = (ly, lx)
                            if (kPair) {
                                D2 = make_float2(dx, dx);
                                E2 = make_float2(dy, dy);
                                L = __fadd2_rn(__ffma2_rn(U2, E2, __ffma2_rn(U1, D2, O2)), make_float2(dy, dx));
                                if (ORDER == 2) {
                                    DXX = __fmul2_rn(D2, D2);
                                    DXY = __fmul2_rn(D2, E2);
                                    DYY = __fmul2_rn(E2, E2);
                                    L = __fadd2_rn(L, __ffma2_rn(Q1, DXX, __ffma2_rn(Q2, DXY, __fmul2_rn(Q3, DYY))));
                                }
                                lx = L.y;
                                ly = L.x;
                            } else {
                                lx = fmaf(uy, dy, fmaf(ux, dx, ox)) + dx;
                                ly = fmaf(vy, dy, fmaf(vx, dx, oy)) + dy;
                                if (ORDER == 2) {
                                    dxx = dx * dx; dxy = dx * dy; dyy = dy * dy;
                                    lx += fmaf(uxx, dxx, fmaf(uxy, dxy, uyy * dyy));
                                    ly += fmaf(vxx, dxx, fmaf(vxy, dxy, vyy * dyy));
                                }
                            }
                            float g;
                            if (FAST) {  // no edge clamp can apply and the window covers every tap
                                const float flx = floorf(lx), fly = floorf(ly);
                                float a[6], b[6];
                                if (kPair) basis_pair_yx(__fadd2_rn(L, make_float2(-fly, -flx)), a, b);
                                else basis_pair(ly - fly, lx - flx, a, b);
                                g = contract_rows2(win + ((int)fly + wy0) * gww + ((int)flx + wx0), gww, a, b);
                            } else {
                                int ix, iy;
                                float tx, ty;
                                split_clamped(wbx, lx, A.w, ix, tx);
                                split_clamped(wby, ly, A.h, iy, ty);
                                float a[6], b[6];
                                basis(ty, a);
                                basis(tx, b);
                                if (staged) {
                                    const int wx = min(max(ix + offx, 0), gww - 6), wy = min(max(iy + offy, 0), gwh - 6);
                                    g = contract<float>(win + wy * gww + wx, gww, a, b);
                                } else {
                                    g = contract<float>(A.g32 + (int64_t)(iy + B - 2) * A.pitch32 + (ix + B - 2), A.pitch32,
                                                        a, b);
                                }
                            }
                            const float gc = g - fmf;
                            if (kPair) {  // (p1, p2) += (gc * 1, gc * gc)
                                float2 q = __ffma2_rn(make_float2(gc, gc), make_float2(1.f, gc), make_float2(p1, p2));
                                p1 = q.x;
                                p2 = q.y;
                            } else {
                                p1 += gc;
                                p2 = fmaf(gc, gc, p2);
                            }
                            pfg = fmaf((RIGID && ORDER == 2 && rigid_on ? (fv - fmf) + St[i] : fv - fmf), gc, pfg);
                            if (kClosed && rigid_on) {
                                ph0 = fmaf(Sh[i], gc, ph0);
                                ph1 = fmaf(Sh[nmax + i], gc, ph1);
                                ph2 = fmaf(Sh[2 * nmax + i], gc, ph2);
                            }
                            if (kPair) {
                                const float2 G2 = __fmul2_rn(make_float2(rec.y, rec.z), make_float2(gc, gc));
                                const float2 half = make_float2(0.5f, 0.5f);
                                pbp[0] = __fadd2_rn(pbp[0], G2);
                                pbp[1] = __ffma2_rn(G2, D2, pbp[1]);
                                pbp[2] = __ffma2_rn(G2, E2, pbp[2]);
                                if (ORDER == 2) {
                                    pbp[3] = __ffma2_rn(G2, __fmul2_rn(half, DXX), pbp[3]);
                                    pbp[4] = __ffma2_rn(G2, DXY, pbp[4]);
                                    pbp[5] = __ffma2_rn(G2, __fmul2_rn(half, DYY), pbp[5]);
                                }
                                continue;
                            }
                            const float gxg = rec.y * gc, gyg = rec.z * gc;
                            pb[0] += gxg;
                            pb[1] += gyg;
                            if (ORDER >= 1) {
                                pb[2 % M] = fmaf(gxg, dx, pb[2 % M]); pb[3 % M] = fmaf(gyg, dx, pb[3 % M]);
                                pb[4 % M] = fmaf(gxg, dy, pb[4 % M]); pb[5 % M] = fmaf(gyg, dy, pb[5 % M]);
                            }
                            if (ORDER == 2) {
                                const float hxx = 0.5f * dxx, hyy = 0.5f * dyy;
                                pb[6 % M] = fmaf(gxg, hxx, pb[6 % M]); pb[7 % M] = fmaf(gyg, hxx, pb[7 % M]);
                                pb[8 % M] = fmaf(gxg, dxy, pb[8 % M]); pb[9 % M] = fmaf(gyg, dxy, pb[9 % M]);
                                pb[10 % M] = fmaf(gxg, hyy, pb[10 % M]); pb[11 % M] = fmaf(gyg, hyy, pb[11 % M]);
                            }
                        }
                    }
                }
                s1 += (double)p1;
                s2 += (double)p2;
                sfg += (double)pfg;
                if (kClosed) {
                    sh0 += (double)ph0;
                    sh1 += (double)ph1;
                    sh2 += (double)ph2;
                }
            }
            if (kPair) {
#pragma unroll
                for (int j = 0; j < M / 2; j++) {
                    pb[2 * j] = pbp[j].x;
                    pb[2 * j + 1] = pbp[j].y;
                }
            }
        };
        if (fast && n == npx_t) sweep(std::true_type{}, std::true_type{});
        else if (fast) sweep(std::true_type{}, std::false_type{});
        else sweep(std::false_type{}, std::false_type{});
        // block sums: warp partials to shared memory, one barrier, then warp 0
        // adds them up and updates the warp; a second barrier publishes p
        constexpr int KR = 3 + M + (kClosed ? 3 : 0);
        {
            double v[KR];
            v[0] = s1; v[1] = s2; v[2] = sfg;
#pragma unroll
            for (int j = 0; j < M; j++) v[3 + j] = (double)pb[j];
            if (kClosed) {
                v[(3 + M) % KR] = sh0;
                v[(4 + M) % KR] = sh1;
                v[(5 + M) % KR] = sh2;
            }
            warp_sum_many<KR>(v, sm.red[wid], lane);
        }
        __syncthreads();
        if (wid == 0) {
            if (lane < KR) {
                double t = 0.0;
#pragma unroll
                for (int w = 0; w < NT / 32; w++) t += sm.red[w][lane];
                sm.tot[lane] = t;
            }
            if (RIGID && ORDER == 2 && rigid_on && lane < 3 + M) {
                double t = 0.0;
#pragma unroll
                for (int w = 0; w < NT / 32; w++) t += sm.redt[w][lane];
                sm.tt[lane] = t;
            }
            __syncwarp();
        }
        // (all threads read tot only after the update barrier below)
        double gmt = 0.0, dg = 0.0, znssd = 0.0;
        if (wid == 0) {
            gmt = sm.tot[0] / dn;
            const double dg2 = sm.tot[1] - sm.tot[0] * gmt;
            dg = sqrt(dg2 > 0.0 ? dg2 : 0.0);
            double sab, dref = df, tmf = 0.0;
            // the template's sums sum G, G^2, (f - f_m) G, SDI_j G (tg[0..3+M))
            // and sum G (g - f_m) (tgc): the template pass's (order 2), or
            // in closed form from the fixed grain moments (order 1)
            double c0 = 0.0, c1 = 0.0, c2 = 0.0, c3 = 0.0, tg0 = 0.0, tg1 = 0.0, tg2 = 0.0, tgc = 0.0;
            if (kClosed && rigid_on) {
                double e0, e1, e2;
                const double ux = sm.p[2 % M], vx = sm.p[3 % M], uy = sm.p[4 % M], vy = sm.p[5 % M];
                e0 = ux + 0.5 * (ux * ux + vx * vx);
                e1 = vy + 0.5 * (uy * uy + vy * vy);
                e2 = 0.5 * (uy + vx) + 0.5 * (ux * uy + vx * vy);
                const double s2d = A.grain_scal[2];
                c0 = -0.5 * s2d * e0; c1 = -0.5 * s2d * e1; c2 = -s2d * e2; c3 = -(e0 + e1);
                const double *q = gq;
                tg0 = c0 * q[0] + c1 * q[1] + c2 * q[2];
                const double cfh = c0 * q[9] + c1 * q[10] + c2 * q[11];
                tg1 = c0 * c0 * q[3] + c1 * c1 * q[6] + c2 * c2 * q[8] +
                      2.0 * (c0 * c1 * q[4] + c0 * c2 * q[5] + c1 * c2 * q[7]) + 2.0 * c3 * cfh + c3 * c3 * saa;
                tg2 = cfh + c3 * saa;
                tgc = c0 * sm.tot[(3 + M) % KR] + c1 * sm.tot[(4 + M) % KR] + c2 * sm.tot[(5 + M) % KR] +
                      c3 * sm.tot[2];
            }
            if (RIGID && rigid_on) {  // the template t = f + G: t_m = f_m + tmf, spread dref
                if (ORDER == 2) {
                    tg0 = sm.tt[0];
                    tg1 = sm.tt[1];
                    tg2 = sm.tt[2];
                }
                tmf = tg0 / dn;
                const double dt2 = saa + 2.0 * tg2 + tg1 - tg0 * tmf;
                dref = sqrt(dt2 > 0.0 ? dt2 : 0.0);
                sab = sm.tot[2] + tgc - tmf * sm.tot[0];
            } else {
                sab = sm.tot[2] - gmt * sa;
            }
            znssd = 2.0 - 2.0 * sab / (dref * dg);
            const double ratio = dref / dg;
            if (lane < M) {
                double sg = 0.0;  // sum SDI_j G
                if (RIGID && rigid_on)
                    sg = ORDER == 2 ? sm.tt[3 + lane]
                                    : c0 * gq[12 + 3 * lane] + c1 * gq[13 + 3 * lane] + c2 * gq[14 + 3 * lane] +
                                          c3 * sm.A[lane];
                const double aj = (RIGID && rigid_on) ? sm.A[lane] + sg - tmf * sm.S[lane] : sm.A[lane];
                sm.grad[lane] = aj - ratio * (sm.tot[3 + lane] - gmt * sm.S[lane]);
            }
            if (lane == 0) {
                sm.misc[8] = tmf;
                sm.misc[9] = dref;
                gcoef[0] = c0;  // the order-1 template's coefficients (eta)
                gcoef[1] = c1;
                gcoef[2] = c2;
                gcoef[3] = c3;
            }
            __syncwarp();
            if (lane < M) {
                double acc = 0.0;
#pragma unroll
                for (int k = 0; k < M; k++) acc = fma(sm.Hinv[lane * M + k], sm.grad[k], acc);
                sm.dp[lane] = -acc;
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
        gmt = sm.misc[2];
        dg = sm.misc[3];
        znssd = sm.misc[4];
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
        for (int i = tid; i < npx_t; i += NT) {
            const float4 rec = S4[i];
            if (rec.x != rec.x) continue;
            float dxf, dyf;
            unpack_off(rec.w, dxf, dyf);
            const double dx = dxf, dy = dyf;
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
            float tx, ty;
            split_clamped(wbx, (float)lx, A.w, ix, tx);
            split_clamped(wby, (float)ly, A.h, iy, ty);
            float a[6], b[6];
            basis(ty, a);
            basis(tx, b);
            Sg[i] = contract<float>(A.g32 + (int64_t)(iy + B - 2) * A.pitch32 + (ix + B - 2), A.pitch32, a, b);
        }
        __syncthreads();
        auto load = [&](int i, double &f, double &gx, double &gy, double &g, double &dx, double &dy) -> bool {
            const float4 rec = S4[i];
            if (rec.x != rec.x) return false;
            float dxf, dyf;
            unpack_off(rec.w, dxf, dyf);
            f = rec.x;
            if (RIGID && rigid_on) {  // the template fitted at the last iteration
                if (ORDER == 2) f += (double)St[i];
                else f += gcoef[0] * Sh[i] + gcoef[1] * Sh[nmax + i] + gcoef[2] * Sh[2 * nmax + i] +
                          gcoef[3] * ((double)rec.x - fm);
            }
            gx = rec.y; gy = rec.z; g = Sg[i]; dx = dxf; dy = dyf;
            return true;
        };
        auto red = [&](double v) { return block_sum1<NT>(v, sm); };
        const double fm_e = (RIGID && rigid_on) ? fm + sm.misc[8] : fm, df_e = (RIGID && rigid_on) ? sm.misc[9] : df;
        eta_sums<ORDER>(npx_t, tid, NT, dn, fm_e, df_e, gm_last, dg_last, load, red, eu, ev);
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
        o->texture = (RIGID && rigid_on) ? 1 : 0;
        o->reserved = 0;
    }
}

// Claim a free scratch slot of the SM this block runs on.  At most
// slots_per_sm blocks of a launch are resident on an SM (the launch's
// occupancy), and a block frees its slot before it exits, so a bit is free
// when a block starts; the wait (bounded) only covers a block that changed
// SM after a preemption still holding its first SM's slot.  -1: none claimed.
__device__ int claim_slot(const TileArgs &T) {
    unsigned smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    if ((int)smid >= T.n_mask) return -1;
    for (int attempt = 0; attempt < 20000; attempt++) {
        for (int j = 0; j < T.slots_per_sm; j++) {
            const unsigned bit = 1u << j;
            if (!(atomicOr(T.slot_mask + smid, bit) & bit)) return (int)smid * T.slots_per_sm + j;
        }
        __nanosleep(1000);
    }
    return -1;
}

// Scratch per block: n_max float4 records + n_max floats (eta resample).
// PER_SUBSET: one block per subset with a claimed scratch slot, else a
// persistent grid taking subsets from the queue (two instantiations, so
// each holds one inlined copy of the solve).
template <int ORDER, int NT, bool PER_SUBSET, bool RIGID>
__global__ void __launch_bounds__(NT, 512 / NT) icgn_tile(TileArgs T) {
    extern __shared__ float4 win4[];
    float *win = reinterpret_cast<float *>(win4);
    __shared__ TileSmem sm;
    const KArgs &A = T.k;
    // per pixel: float4 record, eta sample (+ 3 grain samples, template value)
    const int64_t nmax = A.scratch_stride / (RIGID ? 9 : 5);
    const int start = T.seg[0], count = T.seg[1];
    if (PER_SUBSET) {
        const int item = blockIdx.x;
        if (item >= count) return;
        if (threadIdx.x == 0) sm.item = claim_slot(T);
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
            tile_subset<ORDER, NT, RIGID>(T, idx, d, reinterpret_cast<float4 *>(base), base + 4 * nmax, win, sm,
                                          base + 5 * nmax, base + 8 * nmax, nmax);
        }
        __threadfence();  // every scratch access of the block is done before the slot is free
        __syncthreads();
        if (threadIdx.x == 0) {  // the slot is re-read from shared memory (nothing else writes sm.item here)
            const int own = sm.item;
            atomicAnd(T.slot_mask + own / T.slots_per_sm, ~(1u << (own % T.slots_per_sm)));
        }
        return;
    }
    float *base = reinterpret_cast<float *>(A.scratch) + (int64_t)blockIdx.x * A.scratch_stride;
    float4 *S4 = reinterpret_cast<float4 *>(base);
    float *Sg = base + 4 * nmax;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) sm.item = atomicAdd(T.queue, 1);
        __syncthreads();
        const int item = sm.item;
        if (item >= count) break;
        const int idx = A.order[start + item];
        const gpv_subset_desc d = A.desc[idx];
        if (d.radius < 1 || d.radius > A.max_radius) {
            if (threadIdx.x == 0) write_failed(A, idx, d, 12, GPV_INVALID_SUBSET, 0, 0.0, 0.0);
            continue;
        }
        tile_subset<ORDER, NT, RIGID>(T, idx, d, S4, Sg, win, sm, base + 5 * nmax, base + 8 * nmax, nmax);
    }
}

// Split the work list into segments by (order, radius class): segment
// q = (2 - order) * kRClasses + class, the class being the first upper bound
// in kRBound that the radius does not exceed.  seg[2q], seg[2q+1] = start,
// count; order_out holds the segments back to back.  Each segment is solved
// by its own launch, with a shared-memory window and thread count sized for
// its largest radius, so small subsets in a batch with large ones keep the
// occupancy of their own size.  Subsets with an order outside {0, 1, 2} or a
// radius outside 1..max_radius are failed here.
constexpr int kRClasses = 4;
constexpr int kSegs = 3 * kRClasses;
__constant__ int kRBound[kRClasses] = {20, 32, 48, 1 << 20};
constexpr int kRBoundHost[kRClasses] = {20, 32, 48, 1 << 20};

__device__ __forceinline__ int segment_of(const gpv_subset_desc &d, int max_radius) {
    if (d.order < 0 || d.order > 2 || d.radius < 1 || d.radius > max_radius) return -1;
    int c = 0;
    while (c < kRClasses - 1 && d.radius > kRBound[c]) c++;
    return (2 - d.order) * kRClasses + c;
}

__global__ void count_orders(const gpv_subset_desc *desc, const int32_t *order_in, int n, int max_radius,
                             int32_t *cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int q = -1;
    if (i < n) q = segment_of(desc[order_in ? order_in[i] : i], max_radius);
#pragma unroll
    for (int k = 0; k < kSegs; k++) {
        const unsigned m = __ballot_sync(0xffffffffu, q == k);
        if ((threadIdx.x & 31) == 0 && m) atomicAdd(cnt + k, __popc(m));
    }
}

__global__ void scatter_orders(const gpv_subset_desc *desc, const int32_t *order_in, int n, int max_radius,
                               const int32_t *cnt, int32_t *fill, int32_t *order_out, int32_t *seg,
                               gpv_subset_result *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int idx = -1, q = -1;
    if (i < n) {
        idx = order_in ? order_in[i] : i;
        q = segment_of(desc[idx], max_radius);
    }
    int start[kSegs];
    start[0] = 0;
#pragma unroll
    for (int k = 1; k < kSegs; k++) start[k] = start[k - 1] + cnt[k - 1];
#pragma unroll
    for (int k = 0; k < kSegs; k++) {
        const unsigned m = __ballot_sync(0xffffffffu, q == k);
        if (!m) continue;
        int base = 0;
        const int leader = __ffs(m) - 1;
        if (lane == leader) base = atomicAdd(fill + k, __popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (q == k) order_out[start[k] + base + __popc(m & ((1u << lane) - 1))] = idx;
    }
    if (i < n && q < 0) {
        const gpv_subset_desc d = desc[idx];
        write_failed_any(out, idx, d, GPV_INVALID_SUBSET);
    }
    if (i == 0) {
#pragma unroll
        for (int k = 0; k < kSegs; k++) {
            seg[2 * k] = start[k];
            seg[2 * k + 1] = cnt[k];
        }
    }
}

// Instantiations: every (order, threads, per-subset) for the deformable
// template; the rigid texture (orders 1 and 2) on persistent grids only.
template <int NT, bool PS>
const void *tile_kernel_t(int order) {
    return order == 2 ? (const void *)icgn_tile<2, NT, PS, false>
                      : (order == 1 ? (const void *)icgn_tile<1, NT, PS, false> : (const void *)icgn_tile<0, NT, PS, false>);
}

template <int NT>
const void *tile_kernel_rigid(int order) {
    return order == 2 ? (const void *)icgn_tile<2, NT, false, true> : (const void *)icgn_tile<1, NT, false, true>;
}

const void *tile_kernel(int nt, bool per_subset, int order, bool rigid) {
    if (rigid) return nt == 256 ? tile_kernel_rigid<256>(order) : tile_kernel_rigid<128>(order);
    if (nt == 256) return per_subset ? tile_kernel_t<256, true>(order) : tile_kernel_t<256, false>(order);
    return per_subset ? tile_kernel_t<128, true>(order) : tile_kernel_t<128, false>(order);
}

template <int NT, bool PS>
void tile_launch_t(int order, int blocks, size_t smem, cudaStream_t s, const TileArgs &T) {
    if (order == 2) icgn_tile<2, NT, PS, false><<<blocks, NT, smem, s>>>(T);
    else if (order == 1) icgn_tile<1, NT, PS, false><<<blocks, NT, smem, s>>>(T);
    else icgn_tile<0, NT, PS, false><<<blocks, NT, smem, s>>>(T);
}

template <int NT>
void tile_launch_rigid(int order, int blocks, size_t smem, cudaStream_t s, const TileArgs &T) {
    if (order == 2) icgn_tile<2, NT, false, true><<<blocks, NT, smem, s>>>(T);
    else icgn_tile<1, NT, false, true><<<blocks, NT, smem, s>>>(T);
}

void tile_launch_one(int nt, bool per_subset, int order, bool rigid, int blocks, size_t smem, cudaStream_t s,
                     const TileArgs &T) {
    if (rigid) {
        if (nt == 256) tile_launch_rigid<256>(order, blocks, smem, s, T);
        else tile_launch_rigid<128>(order, blocks, smem, s, T);
    } else if (nt == 256) {
        if (per_subset) tile_launch_t<256, true>(order, blocks, smem, s, T);
        else tile_launch_t<256, false>(order, blocks, smem, s, T);
    } else {
        if (per_subset) tile_launch_t<128, true>(order, blocks, smem, s, T);
        else tile_launch_t<128, false>(order, blocks, smem, s, T);
    }
}

}  // namespace

bool use_run_kernel();

// Threads per block of the tiled kernel for subsets of radius r: the
// autotuned choice when one was recorded for this radius class, else a
// size rule (GPV_TILE_THREADS overrides).
int tile_threads_for(gpv_context *ctx, int max_radius);

// Raise a kernel's dynamic shared-memory limit to everything the device
// allows beside its static shared memory, once per (device, kernel).  The
// limit is a per-function attribute shared by every thread of the process:
// setting it to each launch's own size would let concurrent launches of the
// same kernel with different windows (two contexts, two host threads) undo
// each other's setting between the set and the launch.
// *max_bytes receives that limit.
static int allow_max_dynamic_smem(const void *fn, int *max_bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, int> done;
    int dev = 0;
    GPV_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    auto it = done.find({dev, fn});
    if (it != done.end()) {
        *max_bytes = it->second;
        return GPV_SUCCESS;
    }
    int optin = 0;
    GPV_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    GPV_CUDA_TRY(cudaFuncGetAttributes(&fa, fn));
    const int allowed = optin - (int)fa.sharedSizeBytes;
    GPV_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, allowed));
    done[{dev, fn}] = allowed;
    *max_bytes = allowed;
    return GPV_SUCCESS;
}

// Window capacity (floats) for subsets up to radius r: a radius-r subset
// stretched by 6%, plus margins.
static int window_cap(int r, int layout) {
    const int rw = (int)std::ceil(1.06 * r) + 2;
    const int side = 2 * rw + 6 + 2 * kMargin + 4;
    return side * window_pitch(side, layout);
}

static_assert(kTileSegs == kSegs, "segment count");

int tile_segment_of(int r, int o) {  // segment_of, on the host, for a valid subset
    int c = 0;
    while (c < kRClasses - 1 && r > kRBoundHost[c]) c++;
    return (2 - o) * kRClasses + c;
}

namespace {
__global__ void nsmid_kernel(int *out) {
    unsigned v;
    asm volatile("mov.u32 %0, %%nsmid;" : "=r"(v));
    *out = (int)v;
}
}  // namespace

int query_nsmid(int *out) {
    int *d = nullptr;
    GPV_CUDA_TRY(cudaMalloc(&d, sizeof(int)));
    nsmid_kernel<<<1, 1>>>(d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    GPV_CUDA_TRY(e);
    if (*out < 1 || *out > 4096) { set_error("unexpected SM identifier count"); return GPV_ERR_CUDA; }
    return GPV_SUCCESS;
}

// Launch one kernel per (order, radius class) segment that can hold
// subsets, spread over the context stream and its two auxiliary streams;
// kernels sharing a stream run one after the other and share its scratch.
int tile_launch(gpv_context *ctx, const KArgs &K, int64_t n, cudaStream_t s) {
    int32_t *ws = static_cast<int32_t *>(ctx->tile_ws.ptr);
    int32_t *cnt = ws, *fill = ws + 16, *seg = ws + 32, *queues = ws + 64, *order_out = ws + 96;
    GPV_CUDA_TRY(cudaMemsetAsync(ws, 0, 96 * sizeof(int32_t), s));
    const unsigned blocks = (unsigned)((n + 255) / 256);
    count_orders<<<blocks, 256, 0, s>>>(K.desc, K.order, (int)n, K.max_radius, cnt);
    scatter_orders<<<blocks, 256, 0, s>>>(K.desc, K.order, (int)n, K.max_radius, cnt, fill, order_out, seg, K.out);
    GPV_CUDA_TRY(cudaGetLastError());
    struct Plan {
        int rmax = 0, nt = 0, layout = 0, cap = 0, blocks = 0, per_sm = 0;
        bool ps = false, rigid = false;  // one block per subset; rigid-texture template
        bool runs = false;               // the run-layout kernel (icgn_runs.cu), run length run_k
        int run_k = 0, nslot = 0;
        int64_t stride = 0;
        bool live = false;
    };
    Plan plan[kSegs];
    int64_t region = 0;  // scratch floats per stream: its largest launch
    // one block per subset when the context asks for it and the host knows
    // the segment sizes (host batches); else a persistent grid
    const bool per_subset = (ctx->flags & GPV_CONTEXT_PER_SUBSET_BLOCKS) && ctx->seg_count_valid && ctx->n_smid > 0;
    for (int q = 0; q < kSegs; q++) {
        const int order = 2 - q / kRClasses, c = q % kRClasses;
        const int lo = c == 0 ? 0 : kRBoundHost[c - 1];
        Plan &P = plan[q];
        // the rigid template runs on persistent grids (orders 1 and 2)
        P.rigid = (K.flags & GPV_SOLVE_RIGID_TEXTURE) && order >= 1;
        P.ps = per_subset && !P.rigid;
        P.live = lo < K.max_radius && ((ctx->seg_mask >> q) & 1u) && (!P.ps || ctx->seg_count[q] > 0);
        if (!P.live) continue;
        P.rmax = std::min(kRBoundHost[c], K.max_radius);
        P.nt = tile_threads_for(ctx, P.rmax);
        P.layout = tile_layout_for(ctx, P.rmax);
        // persistent deformable segments run the run-layout kernel unless
        // GPV_SOLVE_KERNEL=tile asks for the tiled one
        // GPV_SOLVE_KAHAN (compensated FP64 ZNSSD sums): run-layout
        // kernel on a persistent grid
        const bool kahan = (K.flags & GPV_SOLVE_KAHAN) != 0;
        P.runs = !P.rigid && (use_run_kernel() || kahan);
        if (kahan) P.ps = false;
        if (P.runs) {
            P.run_k = run_length_for(ctx, P.rmax);
            if (int rc = ensure_run_tables(ctx, K.max_radius)) return rc;
        }
        P.cap = P.runs ? run_window_cap(P.rmax, P.run_k) : window_cap(P.rmax, P.layout);
        // 64-thread blocks exist for the run-layout kernel (not its compensated form) only
        if (P.nt == 64 && (!P.runs || kahan)) P.nt = 128;
        const void *fn = P.runs ? run_kernel(order, P.nt, P.run_k, P.ps, kahan) : tile_kernel(P.nt, P.ps, order, P.rigid);
        int max_bytes = 0;
        if (int rc = allow_max_dynamic_smem(fn, &max_bytes)) return rc;
        // a window larger than the block can hold is not staged: those
        // subsets read g's coefficients from global memory
        P.cap = std::min(P.cap, max_bytes / (int)sizeof(float) / 4 * 4);
        if (P.runs && P.nt == 64) {
            // 64-thread blocks: a window cap that lets 8 blocks share an SM
            // (16 warps, as 4 blocks of 128 threads, but 8 subsets in flight);
            // a warped window larger than the cap reads g from global memory,
            // which the autotuner weighs against 128-thread blocks
            int sm_bytes = 0, reserved = 0;
            GPV_CUDA_TRY(cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
            GPV_CUDA_TRY(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, ctx->device));
            cudaFuncAttributes fa;
            GPV_CUDA_TRY(cudaFuncGetAttributes(&fa, fn));
            const int cap8 = ((sm_bytes / 8 - reserved - (int)fa.sharedSizeBytes) / (int)sizeof(float)) & ~3;
            if (cap8 > 0) P.cap = std::min(P.cap, cap8);
        }
        const size_t smem = sizeof(float) * P.cap;
        int per_sm = 0;
        GPV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, P.nt, smem));
        if (per_sm < 1) { set_error("subset window does not fit in shared memory"); return GPV_ERR_INVALID; }
        if (per_sm > 32) per_sm = 32;  // slot claim words have 32 bits (never reached: 4 blocks of 128 threads)
        P.per_sm = per_sm;
        const int64_t nmax = (int64_t)(ctx->h_slot_n[P.rmax] + 31) / 32 * 32;
        P.stride = (P.rigid ? 9 : 5) * nmax;  // float4 record + eta sample (+ 3 grain samples, template) per pixel
        if (P.runs) P.stride = run_scratch_floats(ctx, P.rmax, P.run_k, &P.nslot);
        int64_t slots;
        if (P.ps) {
            P.blocks = (int)ctx->seg_count[q];
            slots = (int64_t)per_sm * ctx->n_smid;
        } else {
            P.blocks = per_sm * ctx->num_sms;
            slots = P.blocks;
        }
        region = std::max(region, slots * P.stride);
    }
    if (int rc = ctx->scratch.ensure((size_t)3 * region * sizeof(float))) return rc;
    GPV_CUDA_TRY(cudaEventRecord(ctx->ev[0], s));
    cudaStream_t st[3] = {s, ctx->aux[0], ctx->aux[1]};
    bool used[3] = {true, false, false};
    int next = 0;
    for (int q = 0; q < kSegs; q++) {
        const Plan &P = plan[q];
        if (!P.live) continue;
        // a persistent grid spreads its segments over three streams, so one
        // segment's tail overlaps the next one's start; per-subset blocks have
        // no long tail and stay on the caller's stream (fewer streams share
        // the device's hardware queues with other contexts' work)
        const int k = P.ps ? 0 : next;
        next = (next + 1) % 3;
        if (!used[k]) {
            GPV_CUDA_TRY(cudaStreamWaitEvent(st[k], ctx->ev[0], 0));
            used[k] = true;
        }
        TileArgs T;
        T.k = K;
        T.k.order = order_out;
        T.k.max_radius = P.rmax;
        T.win_cap = P.cap;
        T.layout = P.layout;
        T.seg = seg + 2 * q;
        T.queue = queues + q;
        T.k.scratch = static_cast<float *>(ctx->scratch.ptr) + (int64_t)k * region;
        T.k.scratch_stride = P.stride;
        T.slot_mask = P.ps ? static_cast<uint32_t *>(ctx->slot_mask.ptr) + (int64_t)k * ctx->n_smid : nullptr;
        T.slots_per_sm = P.per_sm;
        T.n_mask = ctx->n_smid;
        const size_t smem = sizeof(float) * P.cap;
        if (P.runs) {
            if (int rc = run_launch(ctx, 2 - q / kRClasses, P.nt, P.run_k, (K.flags & GPV_SOLVE_KAHAN) != 0, P.blocks,
                                    smem, st[k], T.k, T.seg, T.queue, P.cap, P.nslot, T.slot_mask, T.slots_per_sm,
                                    T.n_mask))
                return rc;
        } else {
            tile_launch_one(P.nt, P.ps, 2 - q / kRClasses, P.rigid, P.blocks, smem, st[k], T);
        }
        GPV_CUDA_TRY(cudaGetLastError());
    }
    for (int k = 1; k < 3; k++) {
        if (!used[k]) continue;
        GPV_CUDA_TRY(cudaEventRecord(ctx->ev[k], st[k]));
        GPV_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev[k], 0));
    }
    return GPV_SUCCESS;
}

// GPV_TILE_LAYOUT = compact | rows | tiles overrides; the default compact
// layout measured fastest on the second-order workload: the other two remove
// most bank conflicts but add empty slots (the autotuner may still pick them
// for a radius class).
int tile_layout_for(gpv_context *ctx, int max_radius) {
    if (const char *lay = getenv("GPV_TILE_LAYOUT"))
        return lay[0] == 'r' ? kLayoutRows : (lay[0] == 't' ? kLayoutTiles : kLayoutCompact);
    if (ctx->force_layout >= 0) return ctx->force_layout;
    const int cls = max_radius <= 20 ? 0 : (max_radius <= 40 ? 1 : 2);
    return ctx->tuned_layout[cls] >= 0 ? ctx->tuned_layout[cls] : kLayoutCompact;
}

// GPV_SOLVE_KERNEL=tile selects the tiled kernel for every segment; the
// default is the run-layout kernel for persistent deformable segments.
bool use_run_kernel() {
    const char *v = getenv("GPV_SOLVE_KERNEL");
    return !(v && v[0] == 't');
}

int run_length_for(gpv_context *ctx, int max_radius) {
    if (ctx->force_run_k) return ctx->force_run_k;
    if (const char *v = getenv("GPV_RUN_K")) return atoi(v) == 4 ? 4 : 8;
    const int cls = max_radius <= 20 ? 0 : (max_radius <= 40 ? 1 : 2);
    if (ctx->tuned_run_k[cls]) return ctx->tuned_run_k[cls];
    return 4;
}

int tile_threads_for(gpv_context *ctx, int max_radius) {
    if (ctx->force_threads) return ctx->force_threads;
    if (const char *v = getenv("GPV_TILE_THREADS")) {
        const int t = atoi(v);
        return t == 256 ? 256 : (t == 64 ? 64 : 128);
    }
    const int cls = max_radius <= 20 ? 0 : (max_radius <= 40 ? 1 : 2);
    if (ctx->tuned_threads[cls]) return ctx->tuned_threads[cls];
    return max_radius > 40 ? 256 : 128;
}

}  // namespace gpv
