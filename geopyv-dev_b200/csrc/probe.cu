// probe.cu -- throughput probes of the device this library runs on: the
// denominators of the solve kernel's rooflines, measured live instead of
// taken from a datasheet.
//
//  * FP32 FMA, scalar (FFMA) and paired (sm_100 FFMA2, two FMAs per lane per
//    instruction): independent register-only chains.  The interpolation
//    roofline takes the larger of the two.
//  * FP64 FMA (DFMA): the bound of the prefilter's FP64 passes and of the
//    solve's FP64 reductions.
//  * Shared-memory read bandwidth: conflict-free 16-byte loads from a block's
//    shared array.  The tap loads of the sample loop run on this pipe.
// Every probe launches a fixed grid of 8 blocks per SM and reports the best
// of four timed launches after one untimed one (CUDA events on the context
// stream).
#include <cmath>

#include "internal.h"

namespace gpv {
namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeChains = 8;
constexpr int kProbeIters = 4096;
constexpr int kSmemFloats = 8192;  // 32 KB per block
constexpr int kSmemIters = 2048;

__global__ void __launch_bounds__(kProbeThreads) fma_probe(float *out, float a, float b) {
    float x[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) x[c] = (float)(threadIdx.x + c);
    for (int it = 0; it < kProbeIters; it++) {
#pragma unroll
        for (int c = 0; c < kProbeChains; c++) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) s += x[c];
    if (s == 1234.5f) out[threadIdx.x] = s;  // keeps the chains live
}

// The same number of chains, each a pair: twice the FMAs per instruction.
__global__ void __launch_bounds__(kProbeThreads) fma2_probe(float *out, float a, float b) {
    float2 x[kProbeChains];
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) x[c] = make_float2((float)(threadIdx.x + c), (float)(threadIdx.x - c));
    for (int it = 0; it < kProbeIters; it++) {
#pragma unroll
        for (int c = 0; c < kProbeChains; c++) x[c] = __ffma2_rn(x[c], a2, b2);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) s += x[c].x + x[c].y;
    if (s == 1234.5f) out[threadIdx.x] = s;
}

__global__ void __launch_bounds__(kProbeThreads) dfma_probe(double *out, double a, double b) {
    double x[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) x[c] = (double)(threadIdx.x + c);
    for (int it = 0; it < kProbeIters / 4; it++) {
#pragma unroll
        for (int c = 0; c < kProbeChains; c++) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) s += x[c];
    if (s == 1234.5) out[threadIdx.x] = s;
}

// Each thread reads float4s at lane-consecutive indices, so every warp
// request touches 512 contiguous bytes (four wavefronts, no bank conflict).
// The index advances by four blocks' spans plus one float4 per step and
// wraps inside the block's array with a mask (kSmemFloats / 4 float4s, a
// power of two): the address pattern repeats only after 512 steps, so no
// load can be hoisted out of the loop.
__global__ void __launch_bounds__(kProbeThreads) lds_probe(float *out) {
    __shared__ float4 buf[kSmemFloats / 4];
    for (int i = threadIdx.x; i < kSmemFloats / 4; i += kProbeThreads)
        buf[i] = make_float4((float)i, 1.f, 2.f, 3.f);
    __syncthreads();
    constexpr int kMask = kSmemFloats / 4 - 1;
    float4 acc[4];
#pragma unroll
    for (int c = 0; c < 4; c++) acc[c] = make_float4(0.f, 0.f, 0.f, 0.f);
    int idx = threadIdx.x;
    for (int it = 0; it < kSmemIters; it++) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float4 v = buf[(idx + c * kProbeThreads) & kMask];
            acc[c].x += v.x; acc[c].y += v.y; acc[c].z += v.z; acc[c].w += v.w;
        }
        idx = (idx + 4 * kProbeThreads + 1) & kMask;
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < 4; c++) s += acc[c].x + acc[c].y + acc[c].z + acc[c].w;
    if (s == 1234.5f) out[threadIdx.x] = s;
}

// Best rate of four timed launches after one warm-up; `work` is the
// operation (or byte) count of one launch, `launch` enqueues it on s.
template <typename F>
int best_rate(cudaStream_t s, double work, F launch, double *rate) {
    cudaEvent_t e0, e1;
    GPV_CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        set_error("cudaEventCreate failed");
        return GPV_ERR_CUDA;
    }
    double best = 0.0;
    cudaError_t err = cudaSuccess;
    for (int rep = 0; rep < 5 && err == cudaSuccess; rep++) {
        cudaEventRecord(e0, s);
        launch();
        cudaEventRecord(e1, s);
        err = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms > 0.f) best = fmax(best, work / (ms * 1e-3));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    GPV_CUDA_TRY(err);
    *rate = best;
    return GPV_SUCCESS;
}

}  // namespace

int probe_peaks(gpv_context *ctx, gpv_peaks *pk) {
    const int blocks = ctx->num_sms * 8;
    void *out = nullptr;
    GPV_CUDA_TRY(cudaMalloc(&out, kProbeThreads * sizeof(double)));
    cudaStream_t s = ctx->stream;
    const double lanes = (double)blocks * kProbeThreads;
    const double fma = lanes * kProbeChains * kProbeIters;
    float *fo = static_cast<float *>(out);
    double *dout = static_cast<double *>(out);
    int rc = best_rate(s, 2.0 * fma, [&] { fma_probe<<<blocks, kProbeThreads, 0, s>>>(fo, 0.9999f, 1e-4f); },
                       &pk->fp32_scalar_tflops);
    if (!rc)
        rc = best_rate(s, 4.0 * fma, [&] { fma2_probe<<<blocks, kProbeThreads, 0, s>>>(fo, 0.9999f, 1e-4f); },
                       &pk->fp32_paired_tflops);
    if (!rc)
        rc = best_rate(s, 2.0 * fma / 4.0, [&] { dfma_probe<<<blocks, kProbeThreads, 0, s>>>(dout, 0.9999, 1e-4); },
                       &pk->fp64_tflops);
    if (!rc)
        rc = best_rate(s, lanes * kSmemIters * 4.0 * sizeof(float4),
                       [&] { lds_probe<<<blocks, kProbeThreads, 0, s>>>(fo); }, &pk->smem_gbs);
    cudaFree(out);
    if (rc) return rc;
    pk->fp32_scalar_tflops /= 1e12;
    pk->fp32_paired_tflops /= 1e12;
    pk->fp64_tflops /= 1e12;
    pk->smem_gbs /= 1e9;
    pk->sm_count = ctx->num_sms;
    pk->reserved = 0;
    return GPV_SUCCESS;
}

int probe_fp32_peak(gpv_context *ctx, double *tflops) {
    gpv_peaks pk{};
    if (int rc = probe_peaks(ctx, &pk)) return rc;
    *tflops = fmax(pk.fp32_scalar_tflops, pk.fp32_paired_tflops);
    return GPV_SUCCESS;
}

}  // namespace gpv
