// grain.cu -- the reference image's speckle statistics for the rigid-texture
// template (src/texture.rs): its correlation length and the three
// second-derivative maps the template's curvature term samples.
//
// * Correlation length (correlation_length, src/seam.rs:255-301): the centred
//   side x side crop (side = min(512, h, w), even) minus its mean, its
//   circular autocorrelation along x and along y at lags 0..side/2-1, the
//   profile 0.5 (ac_x + ac_y) / ac_0 and the lag where it first falls below
//   0.5, interpolated linearly.  The reference takes the two lag rows from
//   |FFT|^2; here each lag is a direct FP64 sum over the crop (one block per
//   lag and axis, a fixed reduction tree), equal to the transform's result to
//   rounding.  Then s2 = l^2 / (2 ln 2) and the smoothing correction
//   corr = ((s2/2 + 1) / (s2/2))^2 (GrainMaps::build, src/texture.rs:99-115);
//   no lag below 0.5, a crop under 16 px or a non-finite s2 leave the maps
//   unbuilt (the reference then falls back to the deformable template).
// * Maps: fxx = cols(rows(a, k2), k0), fyy = cols(rows(a, k0), k2),
//   fxy = cols(rows(a, k1), k1), each times corr, with k0..k2 the 9-tap
//   Gaussian (sigma 1) and its first and second derivatives as correlation
//   weights and replicated edges (filter_1d, :70-93).  Each output is a
//   left-to-right FP64 sum of products with explicitly rounded multiplies
//   and adds (no fused multiply-add), as the reference's loop computes it;
//   stored as FP32 for the mixed-precision solve, and in FP64 as well for an
//   image that keeps FP64 coefficients (the FP64 solve forms).  A block makes a 32 x 8
//   tile from its pixels plus a 4-pixel apron staged in shared memory.
//
// Everything runs on the image's stream with no host synchronisation: the
// length, s2, corr and the built flag stay in a small device array the maps
// kernel and the solve read.
#include <cmath>

#include "internal.h"

namespace gpv {
namespace {

constexpr int kR = 4;  // ceil(4 sigma), sigma = 1
constexpr int kTaps = 2 * kR + 1;
constexpr int kTw = 32, kTh = 8;
constexpr int kRedThreads = 256;

struct GrainTaps {
    double k[3][kTaps];  // derivative orders 0, 1, 2
};

__device__ __forceinline__ double px_at(const void *px, int dtype, int64_t i) {
    switch (dtype) {
        case GPV_U8: return (double)static_cast<const uint8_t *>(px)[i];
        case GPV_U16: return (double)static_cast<const uint16_t *>(px)[i];
        case GPV_F32: return (double)static_cast<const float *>(px)[i];
        default: return static_cast<const double *>(px)[i];
    }
}

__device__ __forceinline__ double block_sum(double v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kRedThreads / 32; w++) t += red[w];
    return t;  // valid in thread 0
}

// scal[0] = the crop's mean
__global__ void crop_mean(const void *px, int dtype, int64_t w, int64_t r0, int64_t c0, int side, double *scal) {
    __shared__ double red[kRedThreads / 32];
    double s = 0.0;
    const int64_t n = (int64_t)side * side;
    for (int64_t i = threadIdx.x; i < n; i += kRedThreads) {
        const int64_t r = i / side, c = i - r * side;
        s += px_at(px, dtype, (r0 + r) * w + c0 + c);
    }
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) scal[0] = t / (double)n;
}

// ac[axis * half + k] = sum over the crop of a(r, c) a(r, c + k) (axis 0) or
// a(r, c) a(r + k, c) (axis 1), indices modulo side, a = pixel - mean.
__global__ void crop_lags(const void *px, int dtype, int64_t w, int64_t r0, int64_t c0, int side, const double *scal,
                          double *ac) {
    __shared__ double red[kRedThreads / 32];
    const int k = blockIdx.x, axis = blockIdx.y, half = side / 2;
    const double mean = scal[0];
    double s = 0.0;
    const int64_t n = (int64_t)side * side;
    for (int64_t i = threadIdx.x; i < n; i += kRedThreads) {
        const int r = (int)(i / side), c = (int)(i - (int64_t)r * side);
        const int r2 = axis ? (r + k) % side : r, c2 = axis ? c : (c + k) % side;
        s += (px_at(px, dtype, (r0 + r) * w + c0 + c) - mean) * (px_at(px, dtype, (r0 + r2) * w + c0 + c2) - mean);
    }
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) ac[axis * half + k] = t;
}

// scal[1..4] = correlation length, s2, corr, built (1) or not (0)
__global__ void grain_finalize(const double *ac, int half, double *scal) {
    scal[1] = scal[2] = scal[3] = scal[4] = 0.0;
    const double ac0 = ac[0];
    double prev = 1.0;
    for (int k = 0; k < half; k++) {
        const double prof = 0.5 * (ac[k] + ac[half + k]) / ac0;
        if (prof < 0.5) {
            const double ell = (double)k - 1.0 + (prev - 0.5) / (prev - prof);
            const double s2 = ell * ell / (2.0 * 0.69314718055994530942);
            if (isfinite(s2) && s2 > 0.0) {
                const double q = (s2 / 2.0 + 1.0) / (s2 / 2.0);
                scal[1] = ell;
                scal[2] = s2;
                scal[3] = q * q;
                scal[4] = 1.0;
            }
            return;
        }
        prev = prof;
    }
}

__global__ void grain_maps(const void *px, int dtype, int h, int w, GrainTaps t, const double *scal, float *maps,
                           double *maps64) {
    __shared__ double a[kTh + 2 * kR][kTw + 2 * kR];
    __shared__ double rp[3][kTh + 2 * kR][kTw];  // row passes with k0, k1, k2
    if (scal[4] == 0.0) return;
    const int x0 = blockIdx.x * kTw, y0 = blockIdx.y * kTh;
    const int tid = threadIdx.y * kTw + threadIdx.x;
    for (int q = tid; q < (kTh + 2 * kR) * (kTw + 2 * kR); q += kTw * kTh) {
        const int ly = q / (kTw + 2 * kR), lx = q - ly * (kTw + 2 * kR);
        const int y = min(max(y0 + ly - kR, 0), h - 1), x = min(max(x0 + lx - kR, 0), w - 1);
        a[ly][lx] = px_at(px, dtype, (int64_t)y * w + x);
    }
    __syncthreads();
    for (int q = tid; q < (kTh + 2 * kR) * kTw; q += kTw * kTh) {
        const int ly = q / kTw, lx = q - ly * kTw;
#pragma unroll
        for (int o = 0; o < 3; o++) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < kTaps; j++) s = __dadd_rn(s, __dmul_rn(t.k[o][j], a[ly][lx + j]));
            rp[o][ly][lx] = s;
        }
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= w || y >= h) return;
    const double corr = scal[3];
    // (row kernel, column kernel): fxx (2, 0), fyy (0, 2), fxy (1, 1)
    const int rowk[3] = {2, 0, 1}, colk[3] = {0, 2, 1};
    const int64_t np = (int64_t)h * w;
#pragma unroll
    for (int m = 0; m < 3; m++) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < kTaps; j++) s = __dadd_rn(s, __dmul_rn(t.k[colk[m]][j], rp[rowk[m]][threadIdx.y + j][threadIdx.x]));
        const double v = __dmul_rn(s, corr);
        maps[m * np + (int64_t)y * w + x] = (float)v;
        if (maps64) maps64[m * np + (int64_t)y * w + x] = v;
    }
}

// The three maps at n points (x = column, y = row): bilinear in FP64 from
// the FP64 maps when the image keeps them, else the FP32 ones, clamped
// (GrainMaps::sample, src/texture.rs:125-143); out: 3 values per point.
__global__ void grain_points(const float *maps, const double *maps64, int rows, int cols, const double *xy, int64_t n,
                             double *out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = fmin(fmax(xy[2 * i], 0.0), (double)(cols - 1));
    const double y = fmin(fmax(xy[2 * i + 1], 0.0), (double)(rows - 1));
    const int x0 = min((int)floor(x), max(cols - 2, 0)), y0 = min((int)floor(y), max(rows - 2, 0));
    const int x1 = min(x0 + 1, cols - 1), y1 = min(y0 + 1, rows - 1);
    const double tx = x - (double)x0, ty = y - (double)y0;
    const int64_t np = (int64_t)rows * cols;
    for (int m = 0; m < 3; m++) {
        const int64_t a = m * np + (int64_t)y0 * cols + x0, b = m * np + (int64_t)y0 * cols + x1;
        const int64_t c = m * np + (int64_t)y1 * cols + x0, e = m * np + (int64_t)y1 * cols + x1;
        const double v00 = maps64 ? maps64[a] : (double)maps[a], v01 = maps64 ? maps64[b] : (double)maps[b];
        const double v10 = maps64 ? maps64[c] : (double)maps[c], v11 = maps64 ? maps64[e] : (double)maps[e];
        out[3 * i + m] = (1.0 - ty) * ((1.0 - tx) * v00 + tx * v01) + ty * ((1.0 - tx) * v10 + tx * v11);
    }
}

// kernel_with(order, 1.0) (src/texture.rs:49-68), on the host (libm exp).
GrainTaps grain_taps() {
    GrainTaps t;
    const double s2 = 1.0;
    double norm = 0.0;
    for (int i = -kR; i <= kR; i++) norm += std::exp(-(double)(i * i) / (2.0 * s2));
    for (int o = 0; o < 3; o++)
        for (int i = -kR; i <= kR; i++) {
            const double tt = (double)i, gi = std::exp(-(double)(i * i) / (2.0 * s2));
            const double v = o == 0 ? gi : (o == 1 ? tt / s2 * gi : (tt * tt / (s2 * s2) - 1.0 / s2) * gi);
            t.k[o][i + kR] = v / norm;
        }
    return t;
}

}  // namespace

int grain_points_launch(const gpv_image *img, const double *xy_dev, int64_t n, double *out_dev, cudaStream_t s) {
    grain_points<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(img->grain, img->grain64, (int)img->h, (int)img->w, xy_dev,
                                                              n, out_dev);
    GPV_CUDA_TRY(cudaGetLastError());
    return GPV_SUCCESS;
}

int grain_launch(gpv_image *img, const void *px_dev, int dtype, cudaStream_t s) {
    const int64_t h = img->h, w = img->w;
    int side = (int)std::min<int64_t>(512, std::min(h, w)) & ~1;
    GPV_CUDA_TRY(cudaMemsetAsync(img->grain_scal, 0, sizeof(double) * 8, s));
    if (side < 16) return GPV_SUCCESS;  // too small: no maps (deformable template)
    const int half = side / 2;
    const int64_t r0 = h / 2 - half, c0 = w / 2 - half;
    crop_mean<<<1, kRedThreads, 0, s>>>(px_dev, dtype, w, r0, c0, side, img->grain_scal);
    crop_lags<<<dim3(half, 2), kRedThreads, 0, s>>>(px_dev, dtype, w, r0, c0, side, img->grain_scal, img->grain_ac);
    grain_finalize<<<1, 1, 0, s>>>(img->grain_ac, half, img->grain_scal);
    dim3 grid((unsigned)((w + kTw - 1) / kTw), (unsigned)((h + kTh - 1) / kTh));
    grain_maps<<<grid, dim3(kTw, kTh), 0, s>>>(px_dev, dtype, (int)h, (int)w, grain_taps(), img->grain_scal, img->grain,
                                               img->grain64);
    GPV_CUDA_TRY(cudaGetLastError());
    return GPV_SUCCESS;
}

}  // namespace gpv
