// icgn.cu -- batched inverse-compositional Gauss-Newton subset solves.
//
// Reference: Subset::new (src/subset.rs:836-919) and solve_icgn_result
// (src/subset.rs:1117-1219) with apply_warp_into (:262-300),
// steepest_descent (:311-343), compute_hessian (:348-364),
// delta_p_and_znssd_icgn (:418-446), compose_icgn (:487-611),
// convergence_norm (:622-649) and omitted_mode_diagnostic (:698-820).
//
// Two kernels:
//  * icgn_mixed  -- one warp per subset, persistent (warps take subsets from
//    an atomic work queue, largest first).  Interpolation, warping and
//    residuals in FP32 on FP32 coefficients; the mean / norm sums are
//    FP32 partials over 8 pixels per lane carried in FP64, and every sum is
//    combined across lanes in FP64; the Hessian is
//    assembled in FP64 from gradient moments, Jacobi-scaled and inverted by
//    a lane-parallel Gauss-Jordan; warp composition is FP64.  The ICGN update
//    is evaluated in a single pass per iteration through the identities
//        sum (f-f_m)(g-g_m)       = sum (f-f_m) g~ - g~_m sum (f-f_m)
//        grad_j                   = A_j - (df/dg) (B_j - g~_m S_j)
//        ZNSSD                    = 2 - 2 sum(f-f_m)(g-g_m) / (df dg)
//    with g~ = g - f_m, A_j = sum SDI_ij (f_i - f_m), S_j = sum SDI_ij and
//    B_j = sum SDI_ij g~_i.
//  * icgn_fp64   -- the plain form: one thread block per subset, FP64
//    throughout on FP64 coefficients, and the reference's three sweeps per
//    iteration (g_m, then delta_g, then the fused update + ZNSSD).
#include <cstdlib>

#include "icgn_common.cuh"
#include "icgn_warp.cuh"

namespace gpv {
namespace {

__global__ void __launch_bounds__(kMixedWarps * 32, 2) icgn_mixed(KArgs A) {
    __shared__ WarpSmem smem[kMixedWarps];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t gw = (int64_t)blockIdx.x * kMixedWarps + wib;
    const int64_t nmax = A.scratch_stride / 4;
    float *S = reinterpret_cast<float *>(A.scratch) + gw * A.scratch_stride;
    WarpSmem &sm = smem[wib];
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(A.queue, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= A.n) break;
        const int idx = A.order ? A.order[item] : item;
        const gpv_subset_desc d = A.desc[idx];
        if (d.radius < 1 || d.radius > A.max_radius || d.order < 0 || d.order > 2) {
            if (lane == 0) write_failed(A, idx, d, 12, GPV_INVALID_SUBSET, 0, 0.0, 0.0);
            continue;
        }
        switch (d.order) {
            case 0: mixed_subset<0>(A, idx, d, S, nmax, sm, lane); break;
            case 1: mixed_subset<1>(A, idx, d, S, nmax, sm, lane); break;
            default: mixed_subset<2>(A, idx, d, S, nmax, sm, lane); break;
        }
        __syncwarp();
    }
}

// =====================================================================
// Plain FP64 block-per-subset solve
// =====================================================================
struct BlockSmem {
    double red[kFp64Warps][16];
    double bcast[32];
    double mom[3 * 15];
    double H[144];
    double Hinv[144];
    int flag[4];
};

// Sum K values over the block; every thread receives the totals in v.
template <int K>
__device__ void block_sum(double (&v)[K], BlockSmem &sm) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) sm.red[wid][k] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kFp64Warps; w++) s += sm.red[w][k];
        v[k] = s;
    }
}

// Block sums of K values in place, 15 at a time.
template <int K, int C = 0>
__device__ __forceinline__ void block_sums_inplace(double (&v)[K], BlockSmem &sm) {
    if constexpr (C < K) {
        constexpr int N = (K - C) < 15 ? (K - C) : 15;
        block_sum<N>(*reinterpret_cast<double(*)[N]>(&v[C]), sm);
        block_sums_inplace<K, C + N>(v, sm);
    }
}

__device__ double block_sum1(double x, BlockSmem &sm) {
    double v[1] = {x};
    block_sum<1>(v, sm);
    return v[0];
}

// Serial Gauss-Jordan with partial pivoting (one thread).
template <int M>
__device__ bool gj_inverse_serial(const double *Ain, double *Ainv) {
    double a[M][2 * M];
    for (int i = 0; i < M; i++)
        for (int j = 0; j < 2 * M; j++) a[i][j] = j < M ? Ain[i * M + j] : (j - M == i ? 1.0 : 0.0);
    for (int k = 0; k < M; k++) {
        int piv = k;
        double best = fabs(a[k][k]);
        for (int i = k + 1; i < M; i++)
            if (fabs(a[i][k]) > best) { best = fabs(a[i][k]); piv = i; }
        if (!(best > 0.0) || !isfinite(best)) return false;
        if (piv != k)
            for (int j = 0; j < 2 * M; j++) { double t = a[k][j]; a[k][j] = a[piv][j]; a[piv][j] = t; }
        const double dinv = 1.0 / a[k][k];
        for (int j = 0; j < 2 * M; j++) a[k][j] *= dinv;
        for (int i = 0; i < M; i++) {
            if (i == k) continue;
            const double f = a[i][k];
            if (f == 0.0) continue;
            for (int j = 0; j < 2 * M; j++) a[i][j] -= f * a[k][j];
        }
    }
    for (int i = 0; i < M; i++)
        for (int j = 0; j < M; j++) Ainv[i * M + j] = a[i][j + M];
    return true;
}

// The grain maps (rows x cols, FP32 or FP64) at (x = column, y = row),
// bilinear in FP64, clamped (GrainMaps::sample, src/texture.rs:125-143).
template <typename T>
__device__ __forceinline__ void grain_sample_f64(const T *maps, int rows, int cols, double x, double y, double h[3]) {
    x = fmin(fmax(x, 0.0), (double)(cols - 1));
    y = fmin(fmax(y, 0.0), (double)(rows - 1));
    const int x0 = min((int)floor(x), max(cols - 2, 0)), y0 = min((int)floor(y), max(rows - 2, 0));
    const int x1 = min(x0 + 1, cols - 1), y1 = min(y0 + 1, rows - 1);
    const double tx = x - (double)x0, ty = y - (double)y0;
    const int64_t np = (int64_t)rows * cols;
    for (int m = 0; m < 3; m++) {
        const T *Mp = maps + m * np;
        h[m] = (1.0 - ty) * ((1.0 - tx) * (double)Mp[(int64_t)y0 * cols + x0] + tx * (double)Mp[(int64_t)y0 * cols + x1]) +
               ty * ((1.0 - tx) * (double)Mp[(int64_t)y1 * cols + x0] + tx * (double)Mp[(int64_t)y1 * cols + x1]);
    }
}

// Green-Lagrange strain [Exx, Eyy, Exy] (src/texture.rs:200-206), FP64.
__device__ __forceinline__ void green_lagrange_f64(double ux, double vx, double uy, double vy, double &e0, double &e1,
                                                   double &e2) {
    e0 = ux + 0.5 * (ux * ux + vx * vx);
    e1 = vy + 0.5 * (uy * uy + vy * vy);
    e2 = 0.5 * (uy + vx) + 0.5 * (ux * uy + vx * vy);
}

template <int ORDER>
__device__ void fp64_subset(const KArgs &A, int idx, const gpv_subset_desc &d, double *S, int64_t nmax, BlockSmem &sm,
                            bool rigid_req) {
    using O = Ord<ORDER>;
    constexpr int M = O::M, NMU = O::NMU, NMOM = O::NMOM;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int r = d.radius;
    const int npx_t = A.tab_n[r];
    const short2 *po = A.offs + A.tab_off[r];
    double *Sf = S, *Sgx = S + nmax, *Sgy = S + 2 * nmax, *Sg = S + 3 * nmax;
    const double cx = d.coord[0], cy = d.coord[1];
    const int cxi = (int)cx, cyi = (int)cy;
    const double fxd = floor(cx), fyd = floor(cy);
    const int bx = (int)fxd, by = (int)fyd;
    const double fx = cx - fxd, fy = cy - fyd;
    const double *F = A.f64 + (int64_t)(A.border - 2) * A.pitch64 + (A.border - 2);
    const double *G = A.g64 + (int64_t)(A.border - 2) * A.pitch64 + (A.border - 2);

    // Subset::new: f, grad f (:877-884)
    double loc[4] = {0, 0, 0, 0};  // sum f, count, sssig
    for (int i = tid; i < npx_t; i += nthr) {
        const short2 o = po[i];
        if (!mask_ok(A, cxi, cyi, o.x, o.y)) { Sf[i] = __longlong_as_double(0x7ff8000000000000ll); continue; }
        int ix, iy;
        double tx, ty;
        split_clamped(bx, fx + (double)o.x, A.w, ix, tx);
        split_clamped(by, fy + (double)o.y, A.h, iy, ty);
        double a[6], da[6], b[6], db[6];
        basis(ty, a); dbasis(ty, da);
        basis(tx, b); dbasis(tx, db);
        double gx, gy;
        const double f = contract_grad<double>(F + (int64_t)iy * A.pitch64 + ix, A.pitch64, a, da, b, db, gx, gy);
        Sf[i] = f; Sgx[i] = gx; Sgy[i] = gy;
        loc[0] += f;
        loc[1] += 1.0;
        loc[2] += 0.5 * (gx * gx + gy * gy);
    }
    block_sum<4>(loc, sm);
    const int n = (int)loc[1];
    const double sssig = loc[2];
    if (n == 0) {
        if (tid == 0) write_failed(A, idx, d, M, GPV_EMPTY_MASK, 0, 0.0, 0.0);
        return;
    }
    const double dn = (double)n, fm = loc[0] / dn;
    double ss = 0.0;
    for (int i = tid; i < npx_t; i += nthr) {
        const double f = Sf[i];
        if (f != f) continue;
        ss += (f - fm) * (f - fm);
    }
    ss = block_sum1(ss, sm);
    const double df = sqrt(ss);
    if (!(sqrt(ss / dn) > 1e-6 * fmax(1.0, fabs(fm)))) {  // flat subset
        if (tid == 0) write_failed(A, idx, d, M, GPV_FEATURELESS, n, fm, df);
        return;
    }
    // compute_hessian (:348-364) via FP64 gradient moments
    double mom[3 * NMOM];
#pragma unroll
    for (int q = 0; q < 3 * NMOM; q++) mom[q] = 0.0;
    for (int i = tid; i < npx_t; i += nthr) {
        const double f = Sf[i];
        if (f != f) continue;
        const short2 o = po[i];
        const double gx = Sgx[i], gy = Sgy[i], dx = o.x, dy = o.y;
        double pxp[5], pyp[5];
        pxp[0] = pyp[0] = 1.0;
#pragma unroll
        for (int e = 1; e <= 2 * O::DEG; e++) { pxp[e] = pxp[e - 1] * dx; pyp[e] = pyp[e - 1] * dy; }
        const double gg[3] = {gx * gx, gx * gy, gy * gy};
#pragma unroll
        for (int dgr = 0; dgr <= 2 * O::DEG; dgr++)
#pragma unroll
            for (int bb = 0; bb <= dgr; bb++) {
                const double mono = pxp[dgr - bb] * pyp[bb];
#pragma unroll
                for (int p = 0; p < 3; p++) mom[p * NMOM + mom_idx(dgr - bb, bb)] += gg[p] * mono;
            }
    }
#pragma unroll
    for (int q = 0; q < 3 * NMOM; q++) {
        const double v = block_sum1(mom[q], sm);
        if (tid == 0) sm.mom[q] = v;
    }
    __syncthreads();
    if (tid < 32) assemble_hessian<ORDER>(sm.mom, sm.H, tid);
    __syncthreads();
    if (tid == 0) sm.flag[0] = gj_inverse_serial<M>(sm.H, sm.Hinv);
    __syncthreads();
    if (!sm.flag[0]) {
        if (tid == 0) {
            write_failed(A, idx, d, M, GPV_SINGULAR_H, n, fm, df);
            A.out[idx].sssig = sssig;
            A.out[idx].sigma = sqrt(ss / dn);
        }
        return;
    }
    const double size = sqrt(dn);
    double p[M], pprev[M];
#pragma unroll
    for (int k = 0; k < M; k++) p[k] = pprev[k] = d.p0[k];
    int iters = 0, status = GPV_OK;
    bool converged = false;
    double c_zncc = 0.0, c_znssd = 4.0, last_norm = 0.0, gm_last = 0.0, dg_last = 0.0;
    // rigid texture (src/subset.rs:1151-1168): the grain maps at the subset
    // pixels, and at every iteration the template t = f + G(E(p)) with its
    // mean and spread in place of f, f_m and delta_f (two passes, FP64)
    const bool rigid = rigid_req && ORDER >= 1 && A.grain_scal[4] != 0.0;
    double *Sh = S + 4 * nmax, *St = S + 7 * nmax;
    double tm = fm, dt = df;
    if (rigid) {
        for (int i = tid; i < npx_t; i += nthr) {
            if (Sf[i] != Sf[i]) continue;
            const short2 o = po[i];
            double hv[3];
            if (A.grain64) grain_sample_f64(A.grain64, A.h, A.w, cx + (double)o.x, cy + (double)o.y, hv);
            else grain_sample_f64(A.grain, A.h, A.w, cx + (double)o.x, cy + (double)o.y, hv);
            Sh[i] = hv[0]; Sh[nmax + i] = hv[1]; Sh[2 * nmax + i] = hv[2];
        }
    }
    const double s2g = rigid ? A.grain_scal[2] : 0.0;
    for (int it = 1; it <= A.max_iter; it++) {
        if (rigid) {
            double e0 = 0.0, e1 = 0.0, e2 = 0.0;
            if (ORDER == 1) green_lagrange_f64(p[2 % M], p[3 % M], p[4 % M], p[5 % M], e0, e1, e2);
            double st = 0.0;
            for (int i = tid; i < npx_t; i += nthr) {
                const double f = Sf[i];
                if (f != f) continue;
                if (ORDER == 2) {
                    const short2 o = po[i];
                    const double dx = o.x, dy = o.y;
                    green_lagrange_f64(p[2 % M] + p[6 % M] * dx + p[8 % M] * dy, p[3 % M] + p[7 % M] * dx + p[9 % M] * dy,
                                       p[4 % M] + p[8 % M] * dx + p[10 % M] * dy, p[5 % M] + p[9 % M] * dx + p[11 % M] * dy,
                                       e0, e1, e2);
                }
                const double t = f + (-0.5 * s2g * (e0 * Sh[i] + e1 * Sh[nmax + i] + 2.0 * e2 * Sh[2 * nmax + i]) -
                                      (e0 + e1) * (f - fm));
                St[i] = t;
                st += t;
            }
            st = block_sum1(st, sm);
            tm = st / dn;
            double stt = 0.0;
            for (int i = tid; i < npx_t; i += nthr) {
                if (Sf[i] != Sf[i]) continue;
                stt += (St[i] - tm) * (St[i] - tm);
            }
            stt = block_sum1(stt, sm);
            dt = sqrt(stt);
        }
        // apply_warp_into + eval (:1158-1161)
        double sg = 0.0;
        for (int i = tid; i < npx_t; i += nthr) {
            if (Sf[i] != Sf[i]) continue;
            const short2 o = po[i];
            const double dx = o.x, dy = o.y;
            double xw = cx + dx + p[0], yw = cy + dy + p[1];
            if (ORDER >= 1) {
                xw = (cx + dx) + p[0] + p[2] * dx + p[4] * dy;
                yw = (cy + dy) + p[1] + p[3] * dx + p[5] * dy;
            }
            if (ORDER == 2) {
                xw += 0.5 * p[6 % M] * dx * dx + p[8 % M] * dx * dy + 0.5 * p[10 % M] * dy * dy;
                yw += 0.5 * p[7 % M] * dx * dx + p[9 % M] * dx * dy + 0.5 * p[11 % M] * dy * dy;
            }
            const double xfl = floor(xw), yfl = floor(yw);
            int ix, iy;
            double tx, ty;
            split_clamped((int)xfl, xw - xfl, A.w, ix, tx);
            split_clamped((int)yfl, yw - yfl, A.h, iy, ty);
            double a[6], b[6];
            basis(ty, a);
            basis(tx, b);
            const double g = contract<double>(G + (int64_t)iy * A.pitch64 + ix, A.pitch64, a, b);
            Sg[i] = g;
            sg += g;
        }
        sg = block_sum1(sg, sm);
        const double gm = sg / dn;
        double sgg = 0.0;
        for (int i = tid; i < npx_t; i += nthr) {
            if (Sf[i] != Sf[i]) continue;
            sgg += (Sg[i] - gm) * (Sg[i] - gm);
        }
        sgg = block_sum1(sgg, sm);
        const double dg = sqrt(sgg);
        // delta_p_and_znssd_icgn (:418-446)
        const double ratio = dt / dg;
        double acc[M + 1];
#pragma unroll
        for (int k = 0; k <= M; k++) acc[k] = 0.0;
        for (int i = tid; i < npx_t; i += nthr) {
            const double f = Sf[i];
            if (f != f) continue;
            const short2 o = po[i];
            const double a = (rigid ? St[i] : f) - tm, b = Sg[i] - gm;
            const double z = a / dt - b / dg;
            acc[M] += z * z;
            const double br = a - ratio * b;
            const double gx = Sgx[i], gy = Sgy[i], dx = o.x, dy = o.y;
#pragma unroll
            for (int mu = 0; mu < NMU; mu++) {
                const double mv = mu_val<double>(mu, dx, dy);
                acc[2 * mu] += gx * mv * br;
                acc[2 * mu + 1] += gy * mv * br;
            }
        }
        block_sum<M + 1>(acc, sm);
        double dp[M];
#pragma unroll
        for (int j = 0; j < M; j++) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < M; k++) s += sm.Hinv[j * M + k] * acc[k];
            dp[j] = -s;
        }
#pragma unroll
        for (int k = 0; k < M; k++) pprev[k] = p[k];
        gm_last = gm;
        dg_last = dg;
        bool ok = true;
        if (ORDER == 0) {
            p[0] -= dp[0];
            p[1] -= dp[1];
        } else if (ORDER == 1) {
            double pn[6];
            ok = compose1(p, dp, pn);
            if (ok) {
#pragma unroll
                for (int k = 0; k < 6; k++) p[k] = pn[k];
            }
        } else {
            __syncthreads();
            if (tid == 0) {
                double pn[12];
                double ws[96];
                sm.flag[1] = compose2(p, dp, pn, ws);
                for (int k = 0; k < 12; k++) sm.bcast[k] = pn[k];
            }
            __syncthreads();
            ok = sm.flag[1] != 0;
            if (ok) {
#pragma unroll
                for (int k = 0; k < M; k++) p[k] = sm.bcast[k];
            }
        }
        if (!ok) {
#pragma unroll
            for (int k = 0; k < M; k++) p[k] = pprev[k];
            status = GPV_SINGULAR_WDELTA;
            break;
        }
        const double nrm = conv_norm<M>(dp, size);
        c_znssd = acc[M];
        c_zncc = 1.0 - acc[M] / 2.0;
        iters = it;
        last_norm = nrm;
        if (tid == 0) write_history(A, idx, it, nrm, c_zncc, c_znssd);
        if (!isfinite(nrm)) { status = GPV_NONFINITE; break; }
        if (nrm < A.max_norm) { converged = true; break; }
    }
    double eu = 0.0, ev = 0.0;
    const bool want_eta = (A.flags & GPV_SOLVE_ETA) && iters > 0 && status == GPV_OK;
    if (want_eta) {
        auto load = [&](int i, double &f, double &gx, double &gy, double &g, double &dx, double &dy) -> bool {
            f = Sf[i];
            if (f != f) return false;
            if (rigid) f = St[i];  // the template of the last iteration
            const short2 o = po[i];
            gx = Sgx[i]; gy = Sgy[i]; g = Sg[i]; dx = o.x; dy = o.y;
            return true;
        };
        auto red = [&](double v) { return block_sum1(v, sm); };
        eta_sums<ORDER>(npx_t, tid, nthr, dn, tm, dt, gm_last, dg_last, load, red, eu, ev);
    }
    if (tid == 0) {
        gpv_subset_result *o = A.out + idx;
#pragma unroll
        for (int k = 0; k < 12; k++) o->p[k] = k < M ? p[k % M] : 0.0;
        o->c_zncc = c_zncc;
        o->c_znssd = c_znssd;
        o->norm = last_norm;
        o->eta_u = eu;
        o->eta_v = ev;
        o->f_m = fm;
        o->delta_f = df;
        o->sssig = sssig;
        o->sigma = sqrt(ss / dn);
        o->iterations = iters;
        o->converged = converged;
        o->quality_ok = converged && c_zncc >= A.tolerance;
        o->status = status;
        o->n_px = n;
        o->has_eta = want_eta;
        o->texture = rigid ? 1 : 0;
        o->reserved = 0;
    }
}

// =====================================================================
// Forward additive Gauss-Newton (solve_fagn_result, src/subset.rs:1228-1334)
// =====================================================================
// One block per subset, FP64 arithmetic on FP64 coefficients when the images
// keep them, else on the FP32 coefficients.  Per iteration (:1258-1307): the
// target value and gradient at the warped positions, g_m and delta_g (two
// sweeps), the steepest-descent images from the target gradient about the
// warped centre g_center = coord + (u, v) (steepest_descent at :1281), the
// Hessian from FP64 gradient moments of those offsets, the residual
// gradient of delta_p_fagn (:452-473), p += H^-1 grad, then the norm and
// ZNSSD.  Scratch per pixel: f, df/dx, df/dy, g, dg/dx, dg/dy.
template <int ORDER, typename C>
__device__ void fagn_subset(const KArgs &A, int idx, const gpv_subset_desc &d, double *S, int64_t nmax, BlockSmem &sm,
                            const C *Fc, const C *Gc, int64_t pitch, bool rigid_req) {
    using O = Ord<ORDER>;
    constexpr int M = O::M, NMU = O::NMU, NMOM = O::NMOM;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int r = d.radius;
    const int npx_t = A.tab_n[r];
    const short2 *po = A.offs + A.tab_off[r];
    double *Sf = S, *Sgx = S + nmax, *Sgy = S + 2 * nmax, *Sg = S + 3 * nmax, *Shx = S + 4 * nmax,
           *Shy = S + 5 * nmax;
    const double cx = d.coord[0], cy = d.coord[1];
    const int cxi = (int)cx, cyi = (int)cy;
    const double fxd = floor(cx), fyd = floor(cy);
    const int bx = (int)fxd, by = (int)fyd;
    const double fx = cx - fxd, fy = cy - fyd;
    const C *F = Fc + (int64_t)(A.border - 2) * pitch + (A.border - 2);
    const C *G = Gc + (int64_t)(A.border - 2) * pitch + (A.border - 2);

    // Subset::new (:836-919)
    double loc[4] = {0, 0, 0, 0};
    for (int i = tid; i < npx_t; i += nthr) {
        const short2 o = po[i];
        if (!mask_ok(A, cxi, cyi, o.x, o.y)) { Sf[i] = __longlong_as_double(0x7ff8000000000000ll); continue; }
        int ix, iy;
        double tx, ty;
        split_clamped(bx, fx + (double)o.x, A.w, ix, tx);
        split_clamped(by, fy + (double)o.y, A.h, iy, ty);
        double a[6], da[6], b[6], db[6];
        basis(ty, a); dbasis(ty, da);
        basis(tx, b); dbasis(tx, db);
        double gx, gy;
        const double f = contract_grad<double>(F + (int64_t)iy * pitch + ix, pitch, a, da, b, db, gx, gy);
        Sf[i] = f; Sgx[i] = gx; Sgy[i] = gy;
        loc[0] += f;
        loc[1] += 1.0;
        loc[2] += 0.5 * (gx * gx + gy * gy);
    }
    block_sum<4>(loc, sm);
    const int n = (int)loc[1];
    const double sssig = loc[2];
    if (n == 0) {
        if (tid == 0) write_failed(A, idx, d, M, GPV_EMPTY_MASK, 0, 0.0, 0.0);
        return;
    }
    const double dn = (double)n, fm = loc[0] / dn;
    double ss = 0.0;
    for (int i = tid; i < npx_t; i += nthr) {
        const double f = Sf[i];
        if (f != f) continue;
        ss += (f - fm) * (f - fm);
    }
    ss = block_sum1(ss, sm);
    const double df = sqrt(ss);
    if (!(sqrt(ss / dn) > 1e-6 * fmax(1.0, fabs(fm)))) {
        if (tid == 0) write_failed(A, idx, d, M, GPV_FEATURELESS, n, fm, df);
        return;
    }
    const double size = sqrt(dn);
    double p[M];
#pragma unroll
    for (int k = 0; k < M; k++) p[k] = d.p0[k];
    int iters = 0, status = GPV_OK;
    bool converged = false;
    double c_zncc = 0.0, c_znssd = 4.0, last_norm = 0.0, gm_last = 0.0, dg_last = 0.0;
    // rigid texture (src/subset.rs:1257-1262): the grain maps at the subset
    // pixels, and at every iteration the template t = f + G(E(p)) with its
    // mean and spread in place of f, f_m and delta_f (two passes, FP64)
    const bool rigid = rigid_req && ORDER >= 1 && A.grain_scal[4] != 0.0;
    double *Sh = S + 6 * nmax, *St = S + 9 * nmax;
    double tm = fm, dt = df;
    if (rigid) {
        for (int i = tid; i < npx_t; i += nthr) {
            if (Sf[i] != Sf[i]) continue;
            const short2 o = po[i];
            double hv[3];
            if (A.grain64) grain_sample_f64(A.grain64, A.h, A.w, cx + (double)o.x, cy + (double)o.y, hv);
            else grain_sample_f64(A.grain, A.h, A.w, cx + (double)o.x, cy + (double)o.y, hv);
            Sh[i] = hv[0]; Sh[nmax + i] = hv[1]; Sh[2 * nmax + i] = hv[2];
        }
    }
    const double s2g = rigid ? A.grain_scal[2] : 0.0;
    for (int it = 1; it <= A.max_iter; it++) {
        if (rigid) {
            double e0 = 0.0, e1 = 0.0, e2 = 0.0;
            if (ORDER == 1) green_lagrange_f64(p[2 % M], p[3 % M], p[4 % M], p[5 % M], e0, e1, e2);
            double st = 0.0;
            for (int i = tid; i < npx_t; i += nthr) {
                const double f = Sf[i];
                if (f != f) continue;
                if (ORDER == 2) {
                    const short2 o = po[i];
                    const double dx = o.x, dy = o.y;
                    green_lagrange_f64(p[2 % M] + p[6 % M] * dx + p[8 % M] * dy, p[3 % M] + p[7 % M] * dx + p[9 % M] * dy,
                                       p[4 % M] + p[8 % M] * dx + p[10 % M] * dy, p[5 % M] + p[9 % M] * dx + p[11 % M] * dy,
                                       e0, e1, e2);
                }
                const double t = f + (-0.5 * s2g * (e0 * Sh[i] + e1 * Sh[nmax + i] + 2.0 * e2 * Sh[2 * nmax + i]) -
                                      (e0 + e1) * (f - fm));
                St[i] = t;
                st += t;
            }
            st = block_sum1(st, sm);
            tm = st / dn;
            double stt = 0.0;
            for (int i = tid; i < npx_t; i += nthr) {
                if (Sf[i] != Sf[i]) continue;
                stt += (St[i] - tm) * (St[i] - tm);
            }
            stt = block_sum1(stt, sm);
            dt = sqrt(stt);
        }
        // target value + gradient at the warped positions (:1265-1279)
        double sg = 0.0;
        for (int i = tid; i < npx_t; i += nthr) {
            if (Sf[i] != Sf[i]) continue;
            const short2 o = po[i];
            const double dx = o.x, dy = o.y;
            double xw = cx + dx + p[0], yw = cy + dy + p[1];
            if (ORDER >= 1) {
                xw = (cx + dx) + p[0] + p[2 % M] * dx + p[4 % M] * dy;
                yw = (cy + dy) + p[1] + p[3 % M] * dx + p[5 % M] * dy;
            }
            if (ORDER == 2) {
                xw += 0.5 * p[6 % M] * dx * dx + p[8 % M] * dx * dy + 0.5 * p[10 % M] * dy * dy;
                yw += 0.5 * p[7 % M] * dx * dx + p[9 % M] * dx * dy + 0.5 * p[11 % M] * dy * dy;
            }
            const double xfl = floor(xw), yfl = floor(yw);
            int ix, iy;
            double tx, ty;
            split_clamped((int)xfl, xw - xfl, A.w, ix, tx);
            split_clamped((int)yfl, yw - yfl, A.h, iy, ty);
            double a[6], da[6], b[6], db[6];
            basis(ty, a); dbasis(ty, da);
            basis(tx, b); dbasis(tx, db);
            double hx, hy;
            const double g = contract_grad<double>(G + (int64_t)iy * pitch + ix, pitch, a, da, b, db, hx, hy);
            Sg[i] = g; Shx[i] = hx; Shy[i] = hy;
            sg += g;
        }
        sg = block_sum1(sg, sm);
        const double gm = sg / dn;
        double sgg = 0.0;
        for (int i = tid; i < npx_t; i += nthr) {
            if (Sf[i] != Sf[i]) continue;
            sgg += (Sg[i] - gm) * (Sg[i] - gm);
        }
        sgg = block_sum1(sgg, sm);
        const double dg = sqrt(sgg);
        // Hessian moments, residual gradient and ZNSSD in one sweep
        const double gcx = cx + p[0], gcy = cy + p[1];
        const double ratio = dg / dt;
        double mom[3 * NMOM], acc[M + 1];
#pragma unroll
        for (int q = 0; q < 3 * NMOM; q++) mom[q] = 0.0;
#pragma unroll
        for (int k = 0; k <= M; k++) acc[k] = 0.0;
        for (int i = tid; i < npx_t; i += nthr) {
            const double f = Sf[i];
            if (f != f) continue;
            const short2 o = po[i];
            const double ox = o.x, oy = o.y;
            double xw = cx + ox + p[0], yw = cy + oy + p[1];
            if (ORDER >= 1) {
                xw = (cx + ox) + p[0] + p[2 % M] * ox + p[4 % M] * oy;
                yw = (cy + oy) + p[1] + p[3 % M] * ox + p[5 % M] * oy;
            }
            if (ORDER == 2) {
                xw += 0.5 * p[6 % M] * ox * ox + p[8 % M] * ox * oy + 0.5 * p[10 % M] * oy * oy;
                yw += 0.5 * p[7 % M] * ox * ox + p[9 % M] * ox * oy + 0.5 * p[11 % M] * oy * oy;
            }
            const double dx = xw - gcx, dy = yw - gcy;
            const double hx = Shx[i], hy = Shy[i], g = Sg[i];
            double pxp[5], pyp[5];
            pxp[0] = pyp[0] = 1.0;
#pragma unroll
            for (int e = 1; e <= 2 * O::DEG; e++) { pxp[e] = pxp[e - 1] * dx; pyp[e] = pyp[e - 1] * dy; }
            const double hh[3] = {hx * hx, hx * hy, hy * hy};
#pragma unroll
            for (int dgr = 0; dgr <= 2 * O::DEG; dgr++)
#pragma unroll
                for (int bb = 0; bb <= dgr; bb++) {
                    const double mono = pxp[dgr - bb] * pyp[bb];
#pragma unroll
                    for (int q = 0; q < 3; q++) mom[q * NMOM + mom_idx(dgr - bb, bb)] += hh[q] * mono;
                }
            const double a = (rigid ? St[i] : f) - tm, bq = g - gm;
            const double z = a / dt - bq / dg;
            acc[M] += z * z;
            const double res = a * ratio - bq;
#pragma unroll
            for (int mu = 0; mu < NMU; mu++) {
                const double mv = mu_val<double>(mu, dx, dy);
                acc[2 * mu] += hx * mv * res;
                acc[2 * mu + 1] += hy * mv * res;
            }
        }
        block_sum<M + 1>(acc, sm);
        // the moments in place, in block sums of up to 15 values (each
        // value's sum is the same tree as one at a time, with far fewer
        // barriers)
        block_sums_inplace<3 * NMOM>(mom, sm);
        if (tid == 0) {
#pragma unroll
            for (int q = 0; q < 3 * NMOM; q++) sm.mom[q] = mom[q];
        }
        __syncthreads();
        if (tid < 32) assemble_hessian<ORDER>(sm.mom, sm.H, tid);
        __syncthreads();
        if (tid == 0) sm.flag[0] = gj_inverse_serial<M>(sm.H, sm.Hinv);
        __syncthreads();
        gm_last = gm;
        dg_last = dg;
        if (!sm.flag[0]) {  // the reference panics ("FAGN Hessian singular")
            status = GPV_SINGULAR_H;
            break;
        }
        double dp[M];
#pragma unroll
        for (int j = 0; j < M; j++) {
            double s2 = 0.0;
#pragma unroll
            for (int k = 0; k < M; k++) s2 += sm.Hinv[j * M + k] * acc[k];
            dp[j] = s2;
        }
#pragma unroll
        for (int k = 0; k < M; k++) p[k] += dp[k];  // additive update (:1293-1296)
        const double nrm = conv_norm<M>(dp, size);
        c_znssd = acc[M];
        c_zncc = 1.0 - acc[M] / 2.0;
        iters = it;
        last_norm = nrm;
        if (tid == 0) write_history(A, idx, it, nrm, c_zncc, c_znssd);
        if (!isfinite(nrm)) { status = GPV_NONFINITE; break; }
        if (nrm < A.max_norm) { converged = true; break; }
    }
    double eu = 0.0, ev = 0.0;
    const bool want_eta = (A.flags & GPV_SOLVE_ETA) && iters > 0 && status == GPV_OK;
    if (want_eta) {  // with the last sampled target and the reference gradients (:1313-1323)
        auto load = [&](int i, double &f, double &gx, double &gy, double &g, double &dx, double &dy) -> bool {
            f = Sf[i];
            if (f != f) return false;
            if (rigid) f = St[i];  // the template of the last iteration
            const short2 o = po[i];
            gx = Sgx[i]; gy = Sgy[i]; g = Sg[i]; dx = o.x; dy = o.y;
            return true;
        };
        auto red = [&](double v) { return block_sum1(v, sm); };
        eta_sums<ORDER>(npx_t, tid, nthr, dn, tm, dt, gm_last, dg_last, load, red, eu, ev);
    }
    if (tid == 0) {
        gpv_subset_result *o = A.out + idx;
#pragma unroll
        for (int k = 0; k < 12; k++) o->p[k] = k < M ? p[k % M] : 0.0;
        o->c_zncc = c_zncc;
        o->c_znssd = c_znssd;
        o->norm = last_norm;
        o->eta_u = eu;
        o->eta_v = ev;
        o->f_m = fm;
        o->delta_f = df;
        o->sssig = sssig;
        o->sigma = sqrt(ss / dn);
        o->iterations = iters;
        o->converged = converged;
        o->quality_ok = converged && c_zncc >= A.tolerance;
        o->status = status;
        o->n_px = n;
        o->has_eta = want_eta;
        o->texture = rigid ? 1 : 0;
        o->reserved = 0;
    }
}

__global__ void __launch_bounds__(kFp64Threads) fagn_kernel(KArgs A) {
    __shared__ BlockSmem sm;
    __shared__ int item_s;
    double *S = reinterpret_cast<double *>(A.scratch) + (int64_t)blockIdx.x * A.scratch_stride;
    const bool rigid = (A.flags & GPV_SOLVE_RIGID_TEXTURE) != 0;
    // per pixel: f, f_x, f_y, g, g_x, g_y (+ 3 grain samples and the template)
    const int64_t nmax = A.scratch_stride / (rigid ? 10 : 6);
    const bool c64 = A.f64 != nullptr && A.g64 != nullptr;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item_s = atomicAdd(A.queue, 1);
        __syncthreads();
        const int item = item_s;
        if (item >= A.n) break;
        const int idx = A.order ? A.order[item] : item;
        const gpv_subset_desc d = A.desc[idx];
        if (d.radius < 1 || d.radius > A.max_radius || d.order < 0 || d.order > 2) {
            if (threadIdx.x == 0) write_failed(A, idx, d, 12, GPV_INVALID_SUBSET, 0, 0.0, 0.0);
            continue;
        }
        if (c64) {
            switch (d.order) {
                case 0: fagn_subset<0, double>(A, idx, d, S, nmax, sm, A.f64, A.g64, A.pitch64, rigid); break;
                case 1: fagn_subset<1, double>(A, idx, d, S, nmax, sm, A.f64, A.g64, A.pitch64, rigid); break;
                default: fagn_subset<2, double>(A, idx, d, S, nmax, sm, A.f64, A.g64, A.pitch64, rigid); break;
            }
        } else {
            switch (d.order) {
                case 0: fagn_subset<0, float>(A, idx, d, S, nmax, sm, A.f32, A.g32, A.pitch32, rigid); break;
                case 1: fagn_subset<1, float>(A, idx, d, S, nmax, sm, A.f32, A.g32, A.pitch32, rigid); break;
                default: fagn_subset<2, float>(A, idx, d, S, nmax, sm, A.f32, A.g32, A.pitch32, rigid); break;
            }
        }
    }
}

__global__ void __launch_bounds__(kFp64Threads) icgn_fp64(KArgs A) {
    __shared__ BlockSmem sm;
    __shared__ int item_s;
    double *S = reinterpret_cast<double *>(A.scratch) + (int64_t)blockIdx.x * A.scratch_stride;
    const bool rigid = (A.flags & GPV_SOLVE_RIGID_TEXTURE) != 0;
    // per pixel: f, f_x, f_y, g (+ 3 grain samples and the template)
    const int64_t nmax = A.scratch_stride / (rigid ? 8 : 4);
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item_s = atomicAdd(A.queue, 1);
        __syncthreads();
        const int item = item_s;
        if (item >= A.n) break;
        const int idx = A.order ? A.order[item] : item;
        const gpv_subset_desc d = A.desc[idx];
        if (d.radius < 1 || d.radius > A.max_radius || d.order < 0 || d.order > 2) {
            if (threadIdx.x == 0) write_failed(A, idx, d, 12, GPV_INVALID_SUBSET, 0, 0.0, 0.0);
            continue;
        }
        switch (d.order) {
            case 0: fp64_subset<0>(A, idx, d, S, nmax, sm, rigid); break;
            case 1: fp64_subset<1>(A, idx, d, S, nmax, sm, rigid); break;
            default: fp64_subset<2>(A, idx, d, S, nmax, sm, rigid); break;
        }
    }
}

// Point evaluation (gpv_image_eval): one thread per point.
template <typename T, typename C>
__global__ void eval_points(const C *coef, int64_t pitch, int h, int w, int border, const double *xy, int64_t n,
                            double *out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = xy[2 * i], y = xy[2 * i + 1];
    // clamp as Image::eval, then split about an exact integer base
    const double xc = fmin(fmax(x, 0.0), (double)w - 1e-9), yc = fmin(fmax(y, 0.0), (double)h - 1e-9);
    const double xf = floor(xc), yf = floor(yc);
    int ix, iy;
    T tx, ty;
    split_clamped((int)xf, (T)(xc - xf), w, ix, tx);
    split_clamped((int)yf, (T)(yc - yf), h, iy, ty);
    T a[6], da[6], b[6], db[6];
    basis(ty, a); dbasis(ty, da);
    basis(tx, b); dbasis(tx, db);
    T gx, gy;
    const C *p = coef + (int64_t)(iy + border - 2) * pitch + (ix + border - 2);
    const T v = contract_grad<T>(p, pitch, a, da, b, db, gx, gy);
    out[3 * i] = (double)v;
    out[3 * i + 1] = (double)gx;
    out[3 * i + 2] = (double)gy;
}

}  // namespace

int eval_launch(const gpv_image *img, const double *xy_dev, int64_t n, int precision, double *out_dev, cudaStream_t s) {
    if (n == 0) return GPV_SUCCESS;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (precision == GPV_PREC_FP64) {
        if (!img->c64) { set_error("FP64 evaluation needs GPV_IMAGE_KEEP_F64"); return GPV_ERR_INVALID; }
        eval_points<double, double><<<blocks, 256, 0, s>>>(img->c64, img->pitch64, (int)img->h, (int)img->w,
                                                           img->border, xy_dev, n, out_dev);
    } else {
        eval_points<float, float><<<blocks, 256, 0, s>>>(img->c32, img->pitch32, (int)img->h, (int)img->w, img->border,
                                                         xy_dev, n, out_dev);
    }
    GPV_CUDA_TRY(cudaGetLastError());
    return GPV_SUCCESS;
}

int tile_launch(gpv_context *ctx, const KArgs &K, int64_t n, cudaStream_t s);

// GPV_MIXED_KERNEL=warp selects the warp-per-subset kernel for the mixed
// precision solve (default: block per subset with a staged window).
static bool use_warp_kernel() {
    const char *v = getenv("GPV_MIXED_KERNEL");
    return v && v[0] == 'w';
}

int solve_launch(gpv_context *ctx, const SolveLaunch &L, cudaStream_t s) {
    if (L.n == 0) return GPV_SUCCESS;
    const gpv_solve_params *prm = L.prm;
    const bool fp64 = prm->precision == GPV_PREC_FP64;
    KArgs A;
    A.f32 = L.f->c32; A.g32 = L.g->c32;
    A.f64 = L.f->c64; A.g64 = L.g->c64;
    A.pitch32 = L.f->pitch32; A.pitch64 = L.f->pitch64;
    A.h = (int)L.f->h; A.w = (int)L.f->w; A.border = L.f->border;
    A.desc = L.desc; A.order = L.order; A.n = (int)L.n;
    A.offs = static_cast<const short2 *>(ctx->offs.ptr);
    A.slots = static_cast<const short2 *>(ctx->slots.ptr);
    A.table_radius = ctx->table_radius;
    A.tab_off = static_cast<const int32_t *>(ctx->tab_off.ptr);
    A.tab_n = static_cast<const int32_t *>(ctx->tab_n.ptr);
    A.max_radius = L.max_radius;
    A.mask = L.mask; A.mh = (int)L.mh; A.mw = (int)L.mw;
    A.max_norm = prm->max_norm; A.tolerance = prm->tolerance;
    A.max_iter = prm->max_iterations; A.flags = prm->flags;
    A.out = L.out; A.history = L.history;
    if (prm->flags & GPV_SOLVE_RIGID_TEXTURE) {
        if (!(prm->flags & GPV_SOLVE_FAGN) && !fp64 && use_warp_kernel()) {
            set_error("the rigid-texture template is not built into the warp-per-subset kernel");
            return GPV_ERR_INVALID;
        }
        if (!L.f->grain) {
            set_error("the rigid-texture template needs the reference image's grain maps "
                      "(GPV_IMAGE_GRAIN or gpv_image_build_grain)");
            return GPV_ERR_INVALID;
        }
        A.grain = L.f->grain;
        A.grain64 = L.f->grain64;
        A.grain_scal = L.f->grain_scal;
    }
    const int64_t npx_max = ctx->h_tab_n[L.max_radius];
    if (prm->flags & GPV_SOLVE_FAGN) {  // FP64 arithmetic in either precision mode
        if (fp64) {
            A.f64 = L.f->c64;
            A.g64 = L.g->c64;
        } else {
            A.f64 = nullptr;
            A.g64 = nullptr;
        }
        int per_sm = 0;
        GPV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fagn_kernel, kFp64Threads, 0));
        if (per_sm < 1) per_sm = 1;
        const int workers = ctx->num_sms * per_sm;
        const int64_t stride = ((prm->flags & GPV_SOLVE_RIGID_TEXTURE) ? 10 : 6) * ((npx_max + 31) / 32 * 32);
        if (int rc = ctx->scratch.ensure((size_t)workers * stride * sizeof(double))) return rc;
        if (int rc = ctx->queue.ensure(64)) return rc;
        A.scratch = ctx->scratch.ptr;
        A.scratch_stride = stride;
        A.queue = static_cast<int *>(ctx->queue.ptr);
        GPV_CUDA_TRY(cudaMemsetAsync(A.queue, 0, sizeof(int), s));
        fagn_kernel<<<workers, kFp64Threads, 0, s>>>(A);
        GPV_CUDA_TRY(cudaGetLastError());
        return GPV_SUCCESS;
    }
    if (!fp64 && !use_warp_kernel()) {
        if (int rc = ctx->tile_ws.ensure(sizeof(int32_t) * (96 + (size_t)L.n))) return rc;
        return tile_launch(ctx, A, L.n, s);
    }
    int workers, threads;
    size_t elem;
    if (fp64) {
        int per_sm = 0;
        GPV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, icgn_fp64, kFp64Threads, 0));
        if (per_sm < 1) per_sm = 1;
        workers = ctx->num_sms * per_sm;
        threads = kFp64Threads;
        elem = sizeof(double);
    } else {
        if (ctx->mixed_blocks_per_sm == 0) {
            int per_sm = 0;
            GPV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, icgn_mixed, kMixedWarps * 32, 0));
            ctx->mixed_blocks_per_sm = per_sm < 1 ? 1 : per_sm;
        }
        workers = ctx->num_sms * ctx->mixed_blocks_per_sm * kMixedWarps;  // warps
        threads = kMixedWarps * 32;
        elem = sizeof(float);
    }
    const int64_t stride = ((fp64 && (prm->flags & GPV_SOLVE_RIGID_TEXTURE)) ? 8 : 4) * ((npx_max + 31) / 32 * 32);
    const size_t need = (size_t)workers * stride * elem;
    if (int rc = ctx->scratch.ensure(need)) return rc;
    if (int rc = ctx->queue.ensure(64)) return rc;
    A.scratch = ctx->scratch.ptr;
    A.scratch_stride = stride;
    A.queue = static_cast<int *>(ctx->queue.ptr);
    GPV_CUDA_TRY(cudaMemsetAsync(A.queue, 0, sizeof(int), s));
    if (fp64) {
        icgn_fp64<<<workers, threads, 0, s>>>(A);
    } else {
        icgn_mixed<<<workers / kMixedWarps, threads, 0, s>>>(A);
    }
    GPV_CUDA_TRY(cudaGetLastError());
    return GPV_SUCCESS;
}

}  // namespace gpv
