// icgn_warp.cuh -- the warp-per-subset mixed-precision ICGN solve of one
// subset (device code shared by the kernels that run it).
//
// Reference: Subset::new + solve_icgn_result (src/subset.rs:836-919,
// 1117-1219); see icgn.cu for the numerics.
#pragma once
#include "icgn_common.cuh"

namespace gpv {
namespace {

// =====================================================================
// Mixed-precision warp-per-subset solve
// =====================================================================
template <int ORDER>
__device__ void mixed_subset(const KArgs &A, int idx, const gpv_subset_desc &d, float *S, int64_t nmax, WarpSmem &sm,
                             int lane) {
    using O = Ord<ORDER>;
    constexpr int M = O::M, NMU = O::NMU, NMOM = O::NMOM;
    const int r = d.radius;
    const int npx_t = A.tab_n[r];
    const short2 *po = A.offs + A.tab_off[r];
    float *Sf = S, *Sgx = S + nmax, *Sgy = S + 2 * nmax, *Sg = S + 3 * nmax;
    const double cx = d.coord[0], cy = d.coord[1];
    const int cxi = (int)cx, cyi = (int)cy;  // `as isize` (truncation) for the mask window
    const double fxd = floor(cx), fyd = floor(cy);
    const int bx = (int)fxd, by = (int)fyd;
    const float fx = (float)(cx - fxd), fy = (float)(cy - fyd);
    const float *F = A.f32 + (int64_t)(A.border - 2) * A.pitch32 + (A.border - 2);
    const float *G = A.g32 + (int64_t)(A.border - 2) * A.pitch32 + (A.border - 2);

    // ---- setup pass 1: f, grad f, sum f, SSSIG ------------------------------
    double sum_f = 0.0, sssig = 0.0;
    int cnt = 0;
    for (int i = lane; i < npx_t; i += 32) {
        const short2 o = po[i];
        if (!mask_ok(A, cxi, cyi, o.x, o.y)) {
            Sf[i] = __int_as_float(0x7fc00000);  // NaN marks a masked pixel
            continue;
        }
        int ix, iy;
        float tx, ty;
        split_clamped(bx, fx + (float)o.x, A.w, ix, tx);
        split_clamped(by, fy + (float)o.y, A.h, iy, ty);
        float a[6], da[6], b[6], db[6];
        basis(ty, a); dbasis(ty, da);
        basis(tx, b); dbasis(tx, db);
        float gx, gy;
        const float f = contract_grad<float>(F + (int64_t)iy * A.pitch32 + ix, A.pitch32, a, da, b, db, gx, gy);
        Sf[i] = f; Sgx[i] = gx; Sgy[i] = gy;
        sum_f += (double)f;
        sssig += 0.5 * ((double)gx * gx + (double)gy * gy);
        cnt++;
    }
    __syncwarp();
    const int n = warp_sum_int(cnt);
    sum_f = warp_sum(sum_f);
    sssig = warp_sum(sssig);
    // ---- setup pass 1b: gradient moments for the Hessian (FP32 per lane) ----
    {
        float mom[3][NMOM];
#pragma unroll
        for (int p = 0; p < 3; p++)
#pragma unroll
            for (int q = 0; q < NMOM; q++) mom[p][q] = 0.f;
        for (int i = lane; i < npx_t; i += 32) {
            if (Sf[i] != Sf[i]) continue;
            const short2 o = po[i];
            const float gx = Sgx[i], gy = Sgy[i];
            const float dx = (float)o.x, dy = (float)o.y;
            float pxp[2 * 2 + 1], pyp[2 * 2 + 1];
            pxp[0] = 1.f; pyp[0] = 1.f;
#pragma unroll
            for (int e = 1; e <= 2 * O::DEG; e++) { pxp[e] = pxp[e - 1] * dx; pyp[e] = pyp[e - 1] * dy; }
            const float gg[3] = {gx * gx, gx * gy, gy * gy};
#pragma unroll
            for (int dgr = 0; dgr <= 2 * O::DEG; dgr++)
#pragma unroll
                for (int bb = 0; bb <= dgr; bb++) {
                    const float mono = pxp[dgr - bb] * pyp[bb];
#pragma unroll
                    for (int p = 0; p < 3; p++)
                        mom[p][mom_idx(dgr - bb, bb)] = fmaf(gg[p], mono, mom[p][mom_idx(dgr - bb, bb)]);
                }
        }
#pragma unroll
        for (int p = 0; p < 3; p++)
#pragma unroll
            for (int q = 0; q < NMOM; q++) {
                const double v = warp_sum((double)mom[p][q]);
                if (lane == 0) sm.mom[p * NMOM + q] = v;
            }
    }
    if (n == 0) {
        if (lane == 0) write_failed(A, idx, d, M, GPV_EMPTY_MASK, 0, 0.0, 0.0);
        return;
    }
    const double dn = (double)n;
    const double fm = sum_f / dn;
    const float fmf = (float)fm;

    // ---- setup pass 2: delta_f, A_j, S_j ---------------------------------
    double sa = 0.0, saa = 0.0, Aj[M], Sj[M];
#pragma unroll
    for (int j = 0; j < M; j++) Aj[j] = Sj[j] = 0.0;
    for (int i = lane; i < npx_t; i += 32) {
        const float f = Sf[i];
        if (f != f) continue;
        const short2 o = po[i];
        const double a = (double)f - fm;
        const double gx = Sgx[i], gy = Sgy[i], dx = o.x, dy = o.y;
        sa += a;
        saa += a * a;
#pragma unroll
        for (int mu = 0; mu < NMU; mu++) {
            const double mv = mu_val<double>(mu, dx, dy);
            Aj[2 * mu] += gx * mv * a;
            Aj[2 * mu + 1] += gy * mv * a;
            Sj[2 * mu] += gx * mv;
            Sj[2 * mu + 1] += gy * mv;
        }
    }
    sa = warp_sum(sa);
    saa = warp_sum(saa);
#pragma unroll
    for (int j = 0; j < M; j++) {
        const double av = warp_sum(Aj[j]), sv = warp_sum(Sj[j]);
        if (lane == 0) { sm.A[j] = av; sm.S[j] = sv; }
    }
    const double df = sqrt(saa);
    if (!(sqrt(saa / dn) > 1e-6 * fmax(1.0, fabs(fm)))) {  // flat subset (see featureless_test)
        if (lane == 0) write_failed(A, idx, d, M, GPV_FEATURELESS, n, fm, df);
        return;
    }
    __syncwarp();
    assemble_hessian<ORDER>(sm.mom, sm.H, lane);
    if (!spd_inverse_warp<M>(sm.H, sm.aug, sm.Hinv, lane)) {
        if (lane == 0) {
            write_failed(A, idx, d, M, GPV_SINGULAR_H, n, fm, df);
            A.out[idx].sssig = sssig;
            A.out[idx].sigma = sqrt(saa / dn);
        }
        return;
    }

    // ---- ICGN iterations ---------------------------------------------------
    // Warp-uniform FP64 state (p, previous p, increment) lives in shared memory.
    const double size = sqrt(dn);
    if (lane < M) {
        sm.p[lane] = d.p0[lane];
        sm.pprev[lane] = d.p0[lane];
    }
    __syncwarp();
    int iters = 0, status = GPV_OK;
    bool converged = false;
    double c_zncc = 0.0, c_znssd = 4.0, last_norm = 0.0, gm_last = 0.0, dg_last = 0.0;
    for (int it = 1; it <= A.max_iter; it++) {
        // local warp coefficients (FP32) about an exact integer base
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
        // mean / norm sums: FP32 partials over kChunk pixels, FP64 across
        // chunks and lanes.  Steepest-descent sums B_j: FP32 per lane (their
        // rounding moves the increment by < 1e-9 px), FP64 across lanes.
        double s1 = 0.0, s2 = 0.0, sfg = 0.0;
        float pb[M];
#pragma unroll
        for (int j = 0; j < M; j++) pb[j] = 0.f;
        for (int base = 0; base < npx_t; base += 32 * kChunk) {
            float p1 = 0.f, p2 = 0.f, pfg = 0.f;
#pragma unroll
            for (int c = 0; c < kChunk; c++) {
                const int i = base + c * 32 + lane;
                if (i < npx_t) {
                    const float fv = Sf[i];
                    if (fv == fv) {
                        const short2 o = po[i];
                        const float dx = (float)o.x, dy = (float)o.y;
                        float lx = fmaf(uy, dy, fmaf(ux, dx, ox)) + dx;
                        float ly = fmaf(vy, dy, fmaf(vx, dx, oy)) + dy;
                        float dxx = 0.f, dxy = 0.f, dyy = 0.f;
                        if (ORDER == 2) {
                            dxx = dx * dx; dxy = dx * dy; dyy = dy * dy;
                            lx += fmaf(uxx, dxx, fmaf(uxy, dxy, uyy * dyy));
                            ly += fmaf(vxx, dxx, fmaf(vxy, dxy, vyy * dyy));
                        }
                        int ix, iy;
                        float tx, ty;
                        split_clamped(wbx, lx, A.w, ix, tx);
                        split_clamped(wby, ly, A.h, iy, ty);
                        float a[6], b[6];
                        basis(ty, a);
                        basis(tx, b);
                        const float g = contract<float>(G + (int64_t)iy * A.pitch32 + ix, A.pitch32, a, b);
                        const float gc = g - fmf;
                        p1 += gc;
                        p2 = fmaf(gc, gc, p2);
                        pfg = fmaf(fv - fmf, gc, pfg);
                        const float gxg = Sgx[i] * gc, gyg = Sgy[i] * gc;
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
        }
        // reduce; lane 0 keeps the totals in shared memory
        {
            double v;
            v = warp_sum(s1); if (lane == 0) sm.red[0] = v;
            v = warp_sum(s2); if (lane == 0) sm.red[1] = v;
            v = warp_sum(sfg); if (lane == 0) sm.red[2] = v;
#pragma unroll
            for (int j = 0; j < M; j++) {
                v = warp_sum((double)pb[j]);
                if (lane == 0) sm.red[3 + j] = v;
            }
        }
        __syncwarp();
        const double gmt = sm.red[0] / dn;               // mean of g - f_m
        const double dg2 = sm.red[1] - sm.red[0] * gmt;  // sum (g - g_m)^2
        const double dg = sqrt(dg2 > 0.0 ? dg2 : 0.0);
        const double sab = sm.red[2] - gmt * sa;         // sum (f - f_m)(g - g_m)
        const double znssd = 2.0 - 2.0 * sab / (df * dg);
        const double ratio = df / dg;
        if (lane < M) sm.grad[lane] = sm.A[lane] - ratio * (sm.red[3 + lane] - gmt * sm.S[lane]);
        __syncwarp();
        if (lane < M) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < M; k++) acc = fma(sm.Hinv[lane * M + k], sm.grad[k], acc);
            sm.dp[lane] = -acc;
            sm.pprev[lane] = sm.p[lane];
        }
        __syncwarp();
        gm_last = fm + gmt;
        dg_last = dg;
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
                ok = compose2(pl, dpl, pn, sm.aug);
            }
            if (ok) {
#pragma unroll
                for (int k = 0; k < M; k++) sm.p[k] = pn[k];
            }
            sm.flag[0] = ok;
            sm.misc[0] = conv_norm<M>(dpl, size);
        }
        __syncwarp();
        if (!sm.flag[0]) {
            status = GPV_SINGULAR_WDELTA;  // p keeps the last valid warp
            break;
        }
        const double nrm = sm.misc[0];
        c_znssd = znssd;
        c_zncc = 1.0 - znssd / 2.0;
        iters = it;
        last_norm = nrm;
        if (lane == 0) write_history(A, idx, it, nrm, c_zncc, c_znssd);
        if (!isfinite(nrm)) { status = GPV_NONFINITE; break; }
        if (nrm < A.max_norm) { converged = true; break; }
    }

    // ---- eta diagnostic at the last sampled warp (optional) ----------------
    double eu = 0.0, ev = 0.0;
    const bool want_eta = (A.flags & GPV_SOLVE_ETA) && iters > 0 && status == GPV_OK;
    if (want_eta) {
        const double *pprev = sm.pprev;
        const double X0 = cx + pprev[0], Y0 = cy + pprev[1];
        const double bxd = floor(X0), byd = floor(Y0);
        const int wbx = (int)bxd, wby = (int)byd;
        const double ox = X0 - bxd, oy = Y0 - byd;
        for (int i = lane; i < npx_t; i += 32) {
            if (Sf[i] != Sf[i]) continue;
            const short2 o = po[i];
            const double dx = o.x, dy = o.y;
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
            Sg[i] = contract<float>(G + (int64_t)iy * A.pitch32 + ix, A.pitch32, a, b);
        }
        __syncwarp();
        auto load = [&](int i, double &f, double &gx, double &gy, double &g, double &dx, double &dy) -> bool {
            const float fv = Sf[i];
            if (fv != fv) return false;
            const short2 o = po[i];
            f = fv; gx = Sgx[i]; gy = Sgy[i]; g = Sg[i]; dx = o.x; dy = o.y;
            return true;
        };
        auto red = [](double v) { return warp_sum(v); };
        eta_sums<ORDER>(npx_t, lane, 32, dn, fm, df, gm_last, dg_last, load, red, eu, ev);
    }
    if (lane == 0) {
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
        o->sssig = sssig;
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

}  // namespace
}  // namespace gpv
