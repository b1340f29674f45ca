// prefilter.cu -- bi-quintic B-spline coefficients on the device.
//
// Reference: get_c (src/image.rs:252-327).  The reference replicate-pads the
// image by `border` (pad_replicate, :436-443), then for every row and then
// every column computes IFFT(FFT(line) / FFT(kernel)) with the zero-phase
// quintic kernel [11/20, 13/60, 1/120, 0, ..., 0, 1/120, 13/60]
// (build_kernel, :422-430), keeping the real part.
//
// That is a circular convolution with the periodised inverse filter
//     h_N[m] = (1/N) sum_j cos(2 pi j m / N) / K(2 pi j / N),
//     K(w)   = 11/20 + (13/30) cos w + (1/60) cos 2w,
// whose spectrum is evaluated here in closed form once per line length N
// (the kernel's FFT in the reference).  |h_N[m]| decays as 0.4306^|m|, so
// |m| <= 44 reproduces the FFT result to FP64 rounding (1e-14 relative; see
// tests/test_prefilter_*).  An image whose coefficients are kept in FP32
// only uses |m| <= 28: the dropped taps sum to 2.7e-10 of the largest input
// per pass, below FP32 rounding.  Each pass is one kernel: a tile of 32 lines
// is staged in shared memory with its circular halo and every thread slides
// a (2 MT + 1)-tap FP64 window along 16 outputs of one line (taps are kernel
// parameters, i.e. constant-bank operands).  Row pass: pixels -> FP64
// (h, w + 2b) (rows of the border are copies of rows 0 / h-1, so only the h
// image rows are filtered); column pass: -> FP32 (and optionally FP64)
// coefficients (h + 2b, w + 2b).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"

namespace gpv {

namespace {
constexpr int kM = 44;             // taps on each side of the centre (FP64 coefficients)
constexpr int kM32 = 28;           // the same when the coefficients are kept in FP32 only
constexpr int kT = 2 * kM + 1;     // 89
constexpr int kLines = 32;         // lines per tile (one per lane)
constexpr int kGroups = 8;         // warps per block
constexpr int kQ = 16;             // outputs per thread
constexpr int kSpan = kGroups * kQ;  // 128 outputs per line per block

struct TapArg {
    double h[kT];  // h[k] multiplies x[j - mr + k]  (i.e. h_N[mr - k])
};

std::mutex g_taps_mu;
std::map<int64_t, Taps> g_taps;

template <typename P>
__device__ __forceinline__ double px_load(const P *p, int64_t i) {
    return (double)p[i];
}

// Row pass: out[r][j] = sum_k taps[k] * X[r][(j - MT + k) mod cw], X = replicate-padded row r,
// k = 0 .. 2 MT.
template <typename P, int MT>
__global__ void __launch_bounds__(kGroups * 32) rowpass_fir(const P *__restrict__ px, int64_t h, int64_t w, int64_t border,
                                                            int64_t cw, int mr, TapArg taps, double *__restrict__ out) {
    constexpr int kTaps = 2 * MT + 1, kHalo = kTaps - 1;
    extern __shared__ double tile[];  // [kLines][kSpan + kHalo + 1]
    constexpr int stride = kSpan + kHalo + 1;
    const int64_t r0 = (int64_t)blockIdx.y * kLines;
    const int64_t j0 = (int64_t)blockIdx.x * kSpan;
    for (int idx = threadIdx.x; idx < kLines * (kSpan + kHalo); idx += blockDim.x) {
        const int rr = idx / (kSpan + kHalo), s = idx % (kSpan + kHalo);
        int64_t r = r0 + rr;
        if (r > h - 1) r = h - 1;
        int64_t jj = (j0 - mr + s) % cw;
        if (jj < 0) jj += cw;
        int64_t c = jj - border;
        c = c < 0 ? 0 : (c > w - 1 ? w - 1 : c);
        tile[rr * stride + s] = px_load(px, r * w + c);
    }
    __syncthreads();
    const int rr = threadIdx.x & 31, grp = threadIdx.x >> 5;
    const double *x = tile + rr * stride + grp * kQ;
    double acc[kQ];
#pragma unroll
    for (int q = 0; q < kQ; q++) acc[q] = 0.0;
#pragma unroll
    for (int s = 0; s < kQ + kHalo; s++) {
        const double xv = x[s];
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            const int k = s - q;
            if (k >= 0 && k < kTaps) acc[q] = fma(taps.h[k], xv, acc[q]);
        }
    }
    const int64_t r = r0 + rr;
    if (r < h) {
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            const int64_t j = j0 + grp * kQ + q;
            if (j < cw) out[r * cw + j] = acc[q];
        }
    }
}

// Column pass over padded rows i: C[i][j] = sum_k taps[k] * R[(i - mr + k) mod ch][j],
// R[ii] = rowpass[clamp(ii - border, 0, h - 1)].
template <int MT>
__global__ void __launch_bounds__(kGroups * 32) colpass_fir(const double *__restrict__ rp, int64_t h, int64_t cw,
                                                            int64_t ch, int64_t border, int mr, TapArg taps,
                                                            float *__restrict__ c32, int64_t pitch32,
                                                            double *__restrict__ c64, int64_t pitch64) {
    constexpr int kTaps = 2 * MT + 1, kHalo = kTaps - 1;
    extern __shared__ double tile[];  // [kSpan + kHalo][kLines]
    const int64_t i0 = (int64_t)blockIdx.y * kSpan;
    const int64_t j0 = (int64_t)blockIdx.x * kLines;
    for (int idx = threadIdx.x; idx < (kSpan + kHalo) * kLines; idx += blockDim.x) {
        const int s = idx / kLines, c = idx % kLines;
        int64_t ii = (i0 - mr + s) % ch;
        if (ii < 0) ii += ch;
        int64_t r = ii - border;
        r = r < 0 ? 0 : (r > h - 1 ? h - 1 : r);
        int64_t j = j0 + c;
        if (j > cw - 1) j = cw - 1;
        tile[s * kLines + c] = rp[r * cw + j];
    }
    __syncthreads();
    const int c = threadIdx.x & 31, grp = threadIdx.x >> 5;
    const double *x = tile + grp * kQ * kLines + c;
    double acc[kQ];
#pragma unroll
    for (int q = 0; q < kQ; q++) acc[q] = 0.0;
#pragma unroll
    for (int s = 0; s < kQ + kHalo; s++) {
        const double xv = x[s * kLines];
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            const int k = s - q;
            if (k >= 0 && k < kTaps) acc[q] = fma(taps.h[k], xv, acc[q]);
        }
    }
    const int64_t j = j0 + c;
    if (j < cw) {
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            const int64_t i = i0 + grp * kQ + q;
            if (i < ch) {
                c32[i * pitch32 + j] = (float)acc[q];
                if (c64) c64[i * pitch64 + j] = acc[q];
            }
        }
    }
}

// Short lines (N < 89): every one of the N circulant taps, taps in global memory.
template <typename P>
__global__ void rowpass_small(const P *__restrict__ px, int64_t h, int64_t w, int64_t border, int64_t cw, int mr, int nt,
                              const double *__restrict__ taps, double *__restrict__ out) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= h * cw) return;
    const int64_t r = idx / cw, j = idx % cw;
    double acc = 0.0;
    for (int k = 0; k < nt; k++) {
        int64_t jj = (j - mr + k) % cw;
        if (jj < 0) jj += cw;
        int64_t c = jj - border;
        c = c < 0 ? 0 : (c > w - 1 ? w - 1 : c);
        acc = fma(taps[k], (double)px[r * w + c], acc);
    }
    out[idx] = acc;
}

__global__ void colpass_small(const double *__restrict__ rp, int64_t h, int64_t cw, int64_t ch, int64_t border, int mr,
                              int nt, const double *__restrict__ taps, float *__restrict__ c32, int64_t pitch32,
                              double *__restrict__ c64, int64_t pitch64) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ch * cw) return;
    const int64_t i = idx / cw, j = idx % cw;
    double acc = 0.0;
    for (int k = 0; k < nt; k++) {
        int64_t ii = (i - mr + k) % ch;
        if (ii < 0) ii += ch;
        int64_t r = ii - border;
        r = r < 0 ? 0 : (r > h - 1 ? h - 1 : r);
        acc = fma(taps[k], rp[r * cw + j], acc);
    }
    c32[i * pitch32 + j] = (float)acc;
    if (c64) c64[i * pitch64 + j] = acc;
}

// Reversed tap vector: entry k multiplies x[j - mr + k], i.e. h_N[mr - k].
void fill_taparg(const Taps &t, TapArg &a) {
    const int nt = t.ml + t.mr + 1;
    for (int k = 0; k < nt; k++) a.h[k] = t.h[t.mr - k + t.ml];
}

// The central 2 mt + 1 taps of a long line's filter (|m| <= mt), reversed.
void fill_taparg_central(const Taps &t, int mt, TapArg &a) {
    for (int k = 0; k <= 2 * mt; k++) a.h[k] = t.h[t.ml + mt - k];
}

// One FIR pass pair for lines of at least kT samples, MT taps on each side.
// Rows [r0, r0 + nr) of the image (rows are filtered independently).
template <typename P, int MT>
int launch_fir_rows(gpv_image *img, const P *px, const Taps &tr, cudaStream_t s, int64_t r0 = 0, int64_t nr = -1) {
    constexpr int kHalo = 2 * MT;
    if (nr < 0) nr = img->h - r0;
    const size_t smem_row = sizeof(double) * kLines * (kSpan + kHalo + 1);
    TapArg a;
    fill_taparg_central(tr, MT, a);
    GPV_CUDA_TRY(cudaFuncSetAttribute(rowpass_fir<P, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row));
    dim3 grid((unsigned)((img->cw + kSpan - 1) / kSpan), (unsigned)((nr + kLines - 1) / kLines));
    rowpass_fir<P, MT><<<grid, kGroups * 32, smem_row, s>>>(px + r0 * img->w, nr, img->w, img->border, img->cw, MT, a,
                                                             img->rowpass + r0 * img->cw);
    return GPV_SUCCESS;
}

template <int MT>
int launch_fir_cols(gpv_image *img, const Taps &tc, cudaStream_t s) {
    constexpr int kHalo = 2 * MT;
    const size_t smem_col = sizeof(double) * (kSpan + kHalo) * kLines;
    TapArg a;
    fill_taparg_central(tc, MT, a);
    GPV_CUDA_TRY(cudaFuncSetAttribute(colpass_fir<MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_col));
    dim3 grid((unsigned)((img->cw + kLines - 1) / kLines), (unsigned)((img->ch + kSpan - 1) / kSpan));
    colpass_fir<MT><<<grid, kGroups * 32, smem_col, s>>>(img->rowpass, img->h, img->cw, img->ch, img->border, MT, a,
                                                         img->c32, img->pitch32, img->c64, img->pitch64);
    return GPV_SUCCESS;
}

template <typename P>
int run_prefilter(gpv_image *img, const P *px, cudaStream_t s) {
    const Taps &tr = taps_for(img->cw);
    const Taps &tc = taps_for(img->ch);
    const bool f32_only = img->c64 == nullptr;  // coefficients kept in FP32 only: |m| <= kM32
    if (tr.ml + tr.mr + 1 == kT) {
        if (int rc = f32_only ? launch_fir_rows<P, kM32>(img, px, tr, s) : launch_fir_rows<P, kM>(img, px, tr, s))
            return rc;
    } else {
        const int nt = tr.ml + tr.mr + 1;
        TapArg a;
        fill_taparg(tr, a);
        double *dt = reinterpret_cast<double *>(img->rowpass) + img->h * img->cw;  // tap scratch after the row pass
        GPV_CUDA_TRY(cudaMemcpyAsync(dt, a.h, sizeof(double) * nt, cudaMemcpyHostToDevice, s));
        const int64_t total = img->h * img->cw;
        rowpass_small<P><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(px, img->h, img->w, img->border, img->cw,
                                                                          tr.mr, nt, dt, img->rowpass);
        GPV_CUDA_TRY(cudaStreamSynchronize(s));  // host tap array is reused below
    }
    GPV_CUDA_TRY(cudaGetLastError());
    if (tc.ml + tc.mr + 1 == kT) {
        if (int rc = f32_only ? launch_fir_cols<kM32>(img, tc, s) : launch_fir_cols<kM>(img, tc, s)) return rc;
    } else {
        const int nt = tc.ml + tc.mr + 1;
        TapArg a;
        fill_taparg(tc, a);
        double *dt = reinterpret_cast<double *>(img->rowpass) + img->h * img->cw + kT;
        GPV_CUDA_TRY(cudaMemcpyAsync(dt, a.h, sizeof(double) * nt, cudaMemcpyHostToDevice, s));
        const int64_t total = img->ch * img->cw;
        colpass_small<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(img->rowpass, img->h, img->cw, img->ch,
                                                                        img->border, tc.mr, nt, dt, img->c32,
                                                                        img->pitch32, img->c64, img->pitch64);
        GPV_CUDA_TRY(cudaStreamSynchronize(s));
    }
    GPV_CUDA_TRY(cudaGetLastError());
    return GPV_SUCCESS;
}

}  // namespace

const Taps &taps_for(int64_t n) {
    std::lock_guard<std::mutex> lk(g_taps_mu);
    auto it = g_taps.find(n);
    if (it != g_taps.end()) return it->second;
    Taps t;
    t.n = (int)n;
    if (n >= kT) {
        t.ml = t.mr = kM;
    } else {  // all n residues once: offsets -(n-1)/2 .. n/2
        t.ml = (int)((n - 1) / 2);
        t.mr = (int)(n / 2);
    }
    t.h.resize(t.ml + t.mr + 1);
    // spectrum of the zero-phase kernel (build_kernel) in closed form
    std::vector<double> inv(n);
    for (int64_t j = 0; j < n; j++) {
        const double wj = 2.0 * M_PI * (double)j / (double)n;
        inv[j] = 1.0 / (11.0 / 20.0 + (13.0 / 30.0) * std::cos(wj) + (1.0 / 60.0) * std::cos(2.0 * wj));
    }
    for (int m = -t.ml; m <= t.mr; m++) {
        // cos(2 pi j m / n) with the argument reduced exactly: (j*m) mod n
        double acc = 0.0;
        for (int64_t j = 0; j < n; j++) {
            int64_t q = ((j * (int64_t)m) % n + n) % n;
            acc += std::cos(2.0 * M_PI * (double)q / (double)n) * inv[j];
        }
        t.h[m + t.ml] = acc / (double)n;
    }
    return g_taps.emplace(n, std::move(t)).first->second;
}

namespace {
// Host pixels in row chunks into img->px_dev on the copy stream cs; the row
// pass of each chunk starts on s as soon as its copy has landed, so the
// copies overlap the row passes; then the column pass on s.  Lines too short
// for the FIR kernels take the whole copy, then the ordinary prefilter.
template <typename P>
int prefilter_host(gpv_image *img, const P *px_host, cudaStream_t s, cudaStream_t cs, cudaEvent_t *ev, int nev) {
    P *dst = static_cast<P *>(img->px_dev);
    const size_t row_bytes = sizeof(P) * (size_t)img->w;
    const Taps &tr = taps_for(img->cw);
    const Taps &tc = taps_for(img->ch);
    const bool fir = tr.ml + tr.mr + 1 == kT && tc.ml + tc.mr + 1 == kT;
    // rows per copy: ceil(h / (nev - 1)) rounded up to whole row tiles, so at
    // most nev - 1 chunks (events ev[1 .. nev-1]) cover the image
    const int64_t chunk = ((img->h + nev - 2) / (nev - 1) + kLines - 1) / kLines * kLines;
    // the copies wait for earlier work on s that may still read px_dev
    GPV_CUDA_TRY(cudaEventRecord(ev[0], s));
    GPV_CUDA_TRY(cudaStreamWaitEvent(cs, ev[0], 0));
    if (!fir || img->h < 2 * kLines * (nev - 1)) {
        GPV_CUDA_TRY(cudaMemcpyAsync(dst, px_host, row_bytes * (size_t)img->h, cudaMemcpyHostToDevice, cs));
        GPV_CUDA_TRY(cudaEventRecord(ev[1], cs));
        GPV_CUDA_TRY(cudaStreamWaitEvent(s, ev[1], 0));
        return run_prefilter(img, static_cast<const P *>(dst), s);
    }
    const bool f32_only = img->c64 == nullptr;
    int k = 1;
    for (int64_t r0 = 0; r0 < img->h; r0 += chunk, k++) {
        // the last event takes whatever rows remain (never an event past ev[nev - 1])
        const int64_t nr = k == nev - 1 ? img->h - r0 : std::min(chunk, img->h - r0);
        GPV_CUDA_TRY(cudaMemcpyAsync(dst + r0 * img->w, px_host + r0 * img->w, row_bytes * (size_t)nr,
                                     cudaMemcpyHostToDevice, cs));
        GPV_CUDA_TRY(cudaEventRecord(ev[k], cs));
        GPV_CUDA_TRY(cudaStreamWaitEvent(s, ev[k], 0));
        if (int rc = f32_only ? launch_fir_rows<P, kM32>(img, dst, tr, s, r0, nr)
                              : launch_fir_rows<P, kM>(img, dst, tr, s, r0, nr))
            return rc;
    }
    GPV_CUDA_TRY(cudaGetLastError());
    if (int rc = f32_only ? launch_fir_cols<kM32>(img, tc, s) : launch_fir_cols<kM>(img, tc, s)) return rc;
    GPV_CUDA_TRY(cudaGetLastError());
    return GPV_SUCCESS;
}
}  // namespace

int prefilter_from_host(gpv_image *img, const void *px_host, int dtype, cudaStream_t s, cudaStream_t cs,
                        cudaEvent_t *ev, int nev) {
    switch (dtype) {
        case GPV_U8: return prefilter_host(img, static_cast<const uint8_t *>(px_host), s, cs, ev, nev);
        case GPV_U16: return prefilter_host(img, static_cast<const uint16_t *>(px_host), s, cs, ev, nev);
        case GPV_F32: return prefilter_host(img, static_cast<const float *>(px_host), s, cs, ev, nev);
        case GPV_F64: return prefilter_host(img, static_cast<const double *>(px_host), s, cs, ev, nev);
        default: set_error("unknown pixel dtype"); return GPV_ERR_INVALID;
    }
}

int prefilter_launch(gpv_image *img, const void *px_dev, int dtype, cudaStream_t s) {
    switch (dtype) {
        case GPV_U8: return run_prefilter(img, static_cast<const uint8_t *>(px_dev), s);
        case GPV_U16: return run_prefilter(img, static_cast<const uint16_t *>(px_dev), s);
        case GPV_F32: return run_prefilter(img, static_cast<const float *>(px_dev), s);
        case GPV_F64: return run_prefilter(img, static_cast<const double *>(px_dev), s);
        default: set_error("unknown pixel dtype"); return GPV_ERR_INVALID;
    }
}

}  // namespace gpv
