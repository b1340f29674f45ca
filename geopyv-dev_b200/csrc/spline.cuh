// spline.cuh -- bi-quintic B-spline basis and evaluation on the device.
//
// The interpolant is the one of Image::eval / Image::eval_grad
// (src/image.rs:115-230): value = a(ty)^T * C_block * b(tx), with
// a, b = Q^T [1, t, ..., t^5] and the 6x6 coefficient block starting at
// C[yf + border - 2, xf + border - 2] after clamping (x, y) into
// [0, w - 1e-9] x [0, h - 1e-9].
//
// The six weights are evaluated in a symmetric split about t = 1/2
// (u = t - 1/2, v = u^2): w_k = e_k + o_k, w_{5-k} = e_k - o_k with e_k
// even quartics in u and o_k odd quintics.  The coefficients below are
// Q's columns re-expanded about t = 1/2 (exact rationals); this takes 23
// operations per axis instead of the 36 multiply-adds of Q^T [1..t^5].
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gpv {

template <typename T>
__device__ __forceinline__ void basis(T t, T w[6]) {
    const T u = t - T(0.5);
    const T v = u * u;
    const T e0 = fma(fma(v, T(1.0 / 48.0), T(1.0 / 96.0)), v, T(1.0 / 3840.0));
    const T e1 = fma(fma(v, T(-1.0 / 16.0), T(7.0 / 32.0)), v, T(79.0 / 1280.0));
    const T e2 = fma(fma(v, T(1.0 / 24.0), T(-11.0 / 48.0)), v, T(841.0 / 1920.0));
    const T o0 = -u * fma(fma(v, T(1.0 / 120.0), T(1.0 / 48.0)), v, T(1.0 / 384.0));
    const T o1 = -u * fma(fma(v, T(-1.0 / 24.0), T(1.0 / 16.0)), v, T(25.0 / 128.0));
    const T o2 = -u * fma(fma(v, T(1.0 / 12.0), T(-7.0 / 24.0)), v, T(77.0 / 192.0));
    w[0] = e0 + o0;
    w[5] = e0 - o0;
    w[1] = e1 + o1;
    w[4] = e1 - o1;
    w[2] = e2 + o2;
    w[3] = e2 - o2;
}

// basis() for two fractions at once, t = (ty, tx): a from .x, b from .y, the
// same operations per lane as basis(), issued as sm_100 paired FP32 ops.
__device__ __forceinline__ void basis_pair_yx(float2 t, float a[6], float b[6]) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    const float2 u = __fadd2_rn(t, make_float2(-0.5f, -0.5f));
    const float2 v = __fmul2_rn(u, u);
    const float2 nu = make_float2(-u.x, -u.y);
    auto poly = [&](float p2, float p1, float p0) {
        return __ffma2_rn(__ffma2_rn(v, make_float2(p2, p2), make_float2(p1, p1)), v, make_float2(p0, p0));
    };
    const float2 e0 = poly(1.0f / 48.0f, 1.0f / 96.0f, 1.0f / 3840.0f);
    const float2 e1 = poly(-1.0f / 16.0f, 7.0f / 32.0f, 79.0f / 1280.0f);
    const float2 e2 = poly(1.0f / 24.0f, -11.0f / 48.0f, 841.0f / 1920.0f);
    const float2 o0 = __fmul2_rn(nu, poly(1.0f / 120.0f, 1.0f / 48.0f, 1.0f / 384.0f));
    const float2 o1 = __fmul2_rn(nu, poly(-1.0f / 24.0f, 1.0f / 16.0f, 25.0f / 128.0f));
    const float2 o2 = __fmul2_rn(nu, poly(1.0f / 12.0f, -7.0f / 24.0f, 77.0f / 192.0f));
    const float2 w0 = __fadd2_rn(e0, o0), w5 = __fadd2_rn(e0, make_float2(-o0.x, -o0.y));
    const float2 w1 = __fadd2_rn(e1, o1), w4 = __fadd2_rn(e1, make_float2(-o1.x, -o1.y));
    const float2 w2 = __fadd2_rn(e2, o2), w3 = __fadd2_rn(e2, make_float2(-o2.x, -o2.y));
    a[0] = w0.x; a[1] = w1.x; a[2] = w2.x; a[3] = w3.x; a[4] = w4.x; a[5] = w5.x;
    b[0] = w0.y; b[1] = w1.y; b[2] = w2.y; b[3] = w3.y; b[4] = w4.y; b[5] = w5.y;
#else
    basis(t.x, a);
    basis(t.y, b);
#endif
}

__device__ __forceinline__ void basis_pair(float ty, float tx, float a[6], float b[6]) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    basis_pair_yx(make_float2(ty, tx), a, b);
#else
    basis(ty, a);
    basis(tx, b);
#endif
}

// d/dt of the weights (Image::rows uses the derivative at the fractional
// position itself, src/image.rs:210-230).
template <typename T>
__device__ __forceinline__ void dbasis(T t, T d[6]) {
    const T u = t - T(0.5);
    const T v = u * u;
    const T two_u = u + u;
    // de_k/du = 2u (q1 + 2 q2 v);  do_k/du = -(p0 + 3 p1 v + 5 p2 v^2)
    const T de0 = two_u * fma(v, T(2.0 / 48.0), T(1.0 / 96.0));
    const T de1 = two_u * fma(v, T(-2.0 / 16.0), T(7.0 / 32.0));
    const T de2 = two_u * fma(v, T(2.0 / 24.0), T(-11.0 / 48.0));
    const T do0 = -fma(fma(v, T(5.0 / 120.0), T(3.0 / 48.0)), v, T(1.0 / 384.0));
    const T do1 = -fma(fma(v, T(-5.0 / 24.0), T(3.0 / 16.0)), v, T(25.0 / 128.0));
    const T do2 = -fma(fma(v, T(5.0 / 12.0), T(-21.0 / 24.0)), v, T(77.0 / 192.0));
    d[0] = de0 + do0;
    d[5] = de0 - do0;
    d[1] = de1 + do1;
    d[4] = de1 - do1;
    d[2] = de2 + do2;
    d[3] = de2 - do2;
}

// Split a coordinate into an integer pixel index and a fraction in [0, 1]
// with the reference clamp (src/image.rs:129-132): below 0 -> (0, 0), at or
// beyond the last pixel -> (n - 1, 1 - 1e-9).  `base` is an exact integer offset
// added to the small local coordinate `loc` (keeps FP32 fractions exact).
template <typename T>
__device__ __forceinline__ void split_clamped(int base, T loc, int n, int &i, T &t) {
    const T fl = floor(loc);
    i = base + (int)fl;
    t = loc - fl;
    if (i < 0) {
        i = 0;
        t = T(0);
    } else if (i > n - 1) {
        i = n - 1;
        t = T(1) - T(1e-9);  // x clamped to n - 1e-9 (rounds to 1 in FP32)
    }
}

// Value at a clamped position; p points at C[iy + border - 2][ix + border - 2].
template <typename T, typename C>
__device__ __forceinline__ T contract(const C *__restrict__ p, int64_t pitch, const T a[6], const T b[6]) {
    T val = T(0);
#pragma unroll
    for (int r = 0; r < 6; r++) {
        const C *row = p + r * pitch;
        T s = T(row[0]) * b[0];
#pragma unroll
        for (int k = 1; k < 6; k++) s = fma(T(row[k]), b[k], s);
        val = fma(a[r], s, val);
    }
    return val;
}

// contract() for an FP32 block with rows taken in pairs: the two rows'
// partial sums share one paired FMA per tap (sm_100 FFMA2); each row sum and
// the final combine keep contract()'s operation order and rounding.
__device__ __forceinline__ float contract_rows2(const float *__restrict__ p, int pitch, const float a[6],
                                                const float b[6]) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    float2 s[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const float *r0 = p + 2 * q * pitch, *r1 = r0 + pitch;
        s[q] = __fmul2_rn(make_float2(r0[0], r1[0]), make_float2(b[0], b[0]));
#pragma unroll
        for (int k = 1; k < 6; k++) s[q] = __ffma2_rn(make_float2(r0[k], r1[k]), make_float2(b[k], b[k]), s[q]);
    }
    float val = 0.f;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        val = fmaf(a[2 * q], s[q].x, val);
        val = fmaf(a[2 * q + 1], s[q].y, val);
    }
    return val;
#else
    return contract<float>(p, pitch, a, b);
#endif
}

// Value and gradient (Image::eval_grad, src/image.rs:115-124, :155-178).
template <typename T, typename C>
__device__ __forceinline__ T contract_grad(const C *__restrict__ p, int64_t pitch, const T a[6], const T da[6],
                                           const T b[6], const T db[6], T &gx, T &gy) {
    T val = T(0), vx = T(0), vy = T(0);
#pragma unroll
    for (int r = 0; r < 6; r++) {
        const C *row = p + r * pitch;
        T s = T(0), q = T(0);
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const T c = T(row[k]);
            s = fma(c, b[k], s);
            q = fma(c, db[k], q);
        }
        val = fma(a[r], s, val);
        vx = fma(a[r], q, vx);
        vy = fma(da[r], s, vy);
    }
    gx = vx;
    gy = vy;
    return val;
}

// contract_grad() for an FP32 block with rows taken in pairs: each pair's
// value and x-derivative row sums advance by one paired FMA per tap (sm_100
// FFMA2) against the column weights given as duplicated pairs
// bb[k] = (b_k, b_k), dbb[k] = (db_k, db_k).  The row sums and the combine
// keep contract_grad()'s operation order.
__device__ __forceinline__ float contract_grad_rows2(const float *__restrict__ p, int pitch, const float a[6],
                                                     const float da[6], const float2 bb[6], const float2 dbb[6],
                                                     float &gx, float &gy) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    float val = 0.f, vx = 0.f, vy = 0.f;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const float *r0 = p + 2 * q * pitch, *r1 = r0 + pitch;
        float2 c = make_float2(r0[0], r1[0]);
        float2 s = __fmul2_rn(c, bb[0]), d = __fmul2_rn(c, dbb[0]);
#pragma unroll
        for (int k = 1; k < 6; k++) {
            c = make_float2(r0[k], r1[k]);
            s = __ffma2_rn(c, bb[k], s);
            d = __ffma2_rn(c, dbb[k], d);
        }
        val = fmaf(a[2 * q], s.x, val);
        vx = fmaf(a[2 * q], d.x, vx);
        vy = fmaf(da[2 * q], s.x, vy);
        val = fmaf(a[2 * q + 1], s.y, val);
        vx = fmaf(a[2 * q + 1], d.y, vx);
        vy = fmaf(da[2 * q + 1], s.y, vy);
    }
    gx = vx;
    gy = vy;
    return val;
#else
    float b[6], db[6];
    for (int k = 0; k < 6; k++) { b[k] = bb[k].x; db[k] = dbb[k].x; }
    return contract_grad<float>(p, pitch, a, da, b, db, gx, gy);
#endif
}

// ---- warp reductions --------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Warp sums of K <= 16 values at once, a transposed butterfly: the values
// are padded to P (4, 8 or 16); the offsets from 16 down to P add all P
// values pairwise, then each of the offsets P/2 .. 1 halves the set a lane
// keeps and sends the other half to its partner, so lane l ends with the
// total of value l mod P.  P log2(32/P) + P - 1 shuffles instead of 5 K
// (31 instead of 75 for K = 15).  Lanes l < K write their total to dst[l].
// Every total is a fixed tree over the 32 lanes (deterministic).
template <int K>
__device__ __forceinline__ void warp_sum_many(const double (&in)[K], double *dst, int lane) {
    static_assert(K >= 1 && K <= 16, "up to 16 values");
    constexpr int P = K <= 4 ? 4 : (K <= 8 ? 8 : 16);
    double v[P];
#pragma unroll
    for (int j = 0; j < P; j++) v[j] = j < K ? in[j] : 0.0;
#pragma unroll
    for (int off = 16; off >= P; off >>= 1) {
#pragma unroll
        for (int j = 0; j < P; j++) v[j] += __shfl_xor_sync(0xffffffffu, v[j], off);
    }
#pragma unroll
    for (int off = P / 2; off >= 1; off >>= 1) {
        const bool up = (lane & off) != 0;
#pragma unroll
        for (int j = 0; j < off; j++) {
            const double send = up ? v[j] : v[j + off];
            const double keep = up ? v[j + off] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
    if (lane < K) dst[lane] = v[0];
}

__device__ __forceinline__ int warp_sum_int(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace gpv
