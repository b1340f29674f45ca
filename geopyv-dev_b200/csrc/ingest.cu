// ingest.cu -- colour pixels to the greyscale image the prefilter reads.
//
// Image::from_file's load_grayscale (src/image.rs:450-468) and
// gaussian_blur_5x5 (:476-520) on the device: per pixel the integer grey
// level Y = (2126 R + 7152 G + 722 B + 5000) / 10000, then a 5 x 5 separable
// Gaussian (sigma = 1.1, taps normalised to sum 1) with BORDER_REFLECT_101
// indexing (reflect101, :525-534), horizontal pass first, then the vertical
// pass, each a left-to-right FP64 sum of five products, the result rounded
// half away from zero and clamped to 0..255.  Products and sums use the
// explicitly rounded intrinsics, so no multiply-add is fused and the grey
// image equals the reference's bit for bit.  The output is 8-bit greyscale,
// prefiltered into the image's coefficients by the usual path.
//
// A block produces a 32 x 8 tile: it forms the grey levels of the tile plus
// a 2-pixel apron in shared memory, the horizontal pass of the 12 rows it
// needs, then the vertical pass.
#include <cmath>
#include <string>

#include "internal.h"

namespace gpv {
namespace {

constexpr int kTw = 32, kTh = 8;

struct BlurTaps {
    double k[5];
};

__device__ __forceinline__ int reflect101(int i, int n) {  // n >= 3, -2 <= i <= n + 1
    if (i < 0) return -i;
    if (i >= n) return 2 * (n - 1) - i;
    return i;
}

__global__ void ingest_rgb8(const uint8_t *__restrict__ rgb, int h, int w, BlurTaps t, uint8_t *__restrict__ out) {
    __shared__ uint32_t grey[kTh + 4][kTw + 4];
    __shared__ double hp[kTh + 4][kTw];
    const int x0 = blockIdx.x * kTw, y0 = blockIdx.y * kTh;
    const int tid = threadIdx.y * kTw + threadIdx.x;
    for (int q = tid; q < (kTh + 4) * (kTw + 4); q += kTw * kTh) {
        const int ly = q / (kTw + 4), lx = q - ly * (kTw + 4);
        const int y = reflect101(min(max(y0 + ly - 2, -2), h + 1), h);
        const int x = reflect101(min(max(x0 + lx - 2, -2), w + 1), w);
        const uint8_t *p = rgb + 3 * ((int64_t)y * w + x);
        grey[ly][lx] = (2126u * p[0] + 7152u * p[1] + 722u * p[2] + 5000u) / 10000u;
    }
    __syncthreads();
    for (int q = tid; q < (kTh + 4) * kTw; q += kTw * kTh) {
        const int ly = q / kTw, lx = q - ly * kTw;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 5; k++) s = __dadd_rn(s, __dmul_rn(t.k[k], (double)grey[ly][lx + k]));
        hp[ly][lx] = s;
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= w || y >= h) return;
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < 5; k++) v = __dadd_rn(v, __dmul_rn(t.k[k], hp[threadIdx.y + k][threadIdx.x]));
    v = fmin(fmax(round(v), 0.0), 255.0);
    out[(int64_t)y * w + x] = (uint8_t)v;
}

// The taps exactly as the reference normalises them (host libm exp).
BlurTaps blur_taps() {
    BlurTaps t;
    double raw[5], sum = 0.0;
    for (int i = 0; i < 5; i++) {
        const double x = (double)i - 2.0;
        raw[i] = std::exp(-x * x / (2.0 * 1.1 * 1.1));
    }
    for (int i = 0; i < 5; i++) sum += raw[i];
    for (int i = 0; i < 5; i++) t.k[i] = raw[i] / sum;
    return t;
}

}  // namespace

int ingest_launch(const uint8_t *rgb_dev, int64_t h, int64_t w, uint8_t *grey_dev, cudaStream_t s) {
    if (h < 3 || w < 3 || h > INT32_MAX || w > INT32_MAX) {
        set_error("colour ingest needs an image of at least 3 x 3 pixels (the 5-tap reflected blur)");
        return GPV_ERR_INVALID;
    }
    dim3 grid((unsigned)((w + kTw - 1) / kTw), (unsigned)((h + kTh - 1) / kTh));
    ingest_rgb8<<<grid, dim3(kTw, kTh), 0, s>>>(rgb_dev, (int)h, (int)w, blur_taps(), grey_dev);
    GPV_CUDA_TRY(cudaGetLastError());
    return GPV_SUCCESS;
}

}  // namespace gpv
