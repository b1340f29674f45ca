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
// per pass, below FP32 rounding.  Both passes run in one kernel
// (prefilter_fused): every thread slides a (2 MT + 1)-tap FP64 window along
// 16 outputs of one line (taps are kernel parameters, i.e. constant-bank
// operands), first along staged pixel rows, then down a ring of FP64
// row-pass lines held in shared memory; the coefficients come out as FP32
// (and optionally FP64), (h + 2b, w + 2b).  Images with a line shorter than
// 89 samples take two simple kernels through an FP64 row-pass buffer.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"

namespace gpv {

namespace {
constexpr int kM = 44;             // taps on each side of the centre (FP64 coefficients)
constexpr int kM32 = 28;           // the same when the coefficients are kept in FP32 only
constexpr int kT = 2 * kM + 1;     // 89
constexpr int kGroups = 8;         // warps per block
constexpr int kQ = 16;             // outputs per thread

struct TapArg {
    double h[kT];  // h[k] multiplies x[j - mr + k]  (i.e. h_N[mr - k])
};

std::mutex g_taps_mu;
std::map<int64_t, Taps> g_taps;

template <typename P>
__device__ __forceinline__ double px_load(const P *p, int64_t i) {
    return (double)p[i];
}

// Both passes in one kernel.  A block owns a strip of kStrip padded columns
// [j0, j0 + kStrip) and a segment of output rows [i_beg, i_end).  It walks
// down the segment kStep rows at a time: the row pass of the next kStep
// padded rows (from pixel lines staged in shared memory) lands in a ring of
// FP64 lines that also holds the 2 MT lines before them, and the column pass
// of kStep outputs reads that ring.  The FP64 row-pass lines never leave the
// SM: DRAM sees the pixels (read once per strip; the halo columns of
// neighbouring strips come from L2) and the coefficients written.  Each
// output is the same FMA sequence, in the same order, as a separate row
// pass and column pass would give (taps k = 0 .. 2 MT, increasing).
//   row pass:    R[r][j] = sum_k tr[k] X[r][(j - MT + k) mod cw],
//                X[r][jj] = px[r][clamp(jj - border, 0, w - 1)]
//   column pass: C[i][j] = sum_k tc[k] R[clamp((i - MT + k) mod ch - border, 0, h - 1)][j]
constexpr int kStrip = 32;   // columns per block (one per lane in the column pass)
constexpr int kStep = 128;   // output rows per step (8 warps x kQ)
constexpr int kFusedThreads = kGroups * 32;
static_assert(kStep == kGroups * kQ && kStrip == 2 * kQ, "one row-pass line per two threads, one output column per lane");

// Staged pixel line pitch (elements) for kPxW pixels: lanes of a warp read 32
// different lines at one column, so the pitch in 4-byte words is odd (an odd
// number of doubles for FP64 pixels).
template <typename P, int W>
__host__ __device__ constexpr int px_pitch() {
    return sizeof(P) == 8 ? (W | 1) : (((W * (int)sizeof(P) + 3) / 4) | 1) * 4 / (int)sizeof(P);
}

template <typename P, int MT>
struct Fused {
    static constexpr int kTaps = 2 * MT + 1, kHalo = 2 * MT;
    static constexpr int kRing = kStep + kHalo;   // FP64 row-pass lines held
    static constexpr int kRingPitch = kStrip + 1;  // doubles
    static constexpr int kPxW = kStrip + kHalo;   // pixels per staged line
    static constexpr int kPxPitch = px_pitch<P, kPxW>();
    static constexpr size_t kRingBytes = sizeof(double) * kRing * kRingPitch;
    static constexpr size_t kSmem = kRingBytes + sizeof(P) * kStep * kPxPitch;
};

template <typename P, int MT>
__global__ void __launch_bounds__(kFusedThreads) prefilter_fused(const P *__restrict__ px, int64_t h, int64_t w,
                                                                int64_t border, int64_t cw, int64_t ch, int64_t i_lo,
                                                                int64_t i_hi, int64_t seg, TapArg tr, TapArg tc,
                                                                float *__restrict__ c32, int64_t pitch32,
                                                                double *__restrict__ c64, int64_t pitch64) {
    using G = Fused<P, MT>;
    extern __shared__ double smem[];
    double *ring = smem;
    P *pxs = reinterpret_cast<P *>(reinterpret_cast<unsigned char *>(smem) + G::kRingBytes);
    const int64_t j0 = (int64_t)blockIdx.x * kStrip;
    const int64_t i_beg = i_lo + (int64_t)blockIdx.y * seg;
    const int64_t i_end = i_beg + seg < i_hi ? i_beg + seg : i_hi;
    if (i_beg >= i_end) return;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

    // the strip's source columns, the same for every line: entry m of lane
    // l is staged column l + 32 m, its image column (-1 past the staged width)
    constexpr int kCols = (G::kPxW + 31) / 32;
    int csrc[kCols];
#pragma unroll
    for (int m = 0; m < kCols; m++) {
        const int sx = lane + 32 * m;
        int jj = (int)j0 - MT + sx;  // in [-MT, cw + kStrip + MT): one wrap at most (cw >= 2 MT + 1)
        jj = jj < 0 ? jj + (int)cw : (jj >= (int)cw ? jj - (int)cw : jj);
        const int c = jj - (int)border;
        csrc[m] = sx < G::kPxW ? (c < 0 ? 0 : (c > (int)w - 1 ? (int)w - 1 : c)) : -1;
    }
    // row pass of n padded rows (row0 + t) mod ch, t < n <= kStep, into ring
    // lines [dst, dst + n); the pixel lines are staged one per warp at a time
    auto produce = [&](int64_t row0, int n, int dst) {
        int base = (int)(row0 % ch);  // row0 >= -MT
        if (base < 0) base += (int)ch;
        for (int rr = wid; rr < n; rr += kGroups) {
            int ii = base + rr;
            while (ii >= (int)ch) ii -= (int)ch;
            int r = ii - (int)border;
            r = r < 0 ? 0 : (r > (int)h - 1 ? (int)h - 1 : r);
            const P *src = px + (int64_t)r * w;
            P *d = pxs + rr * G::kPxPitch + lane;
#pragma unroll
            for (int m = 0; m < kCols; m++)
                if (csrc[m] >= 0) d[32 * m] = src[csrc[m]];
        }
        __syncthreads();
        const int rr = (wid & 3) * 32 + lane, half = wid >> 2;
        if (rr < n) {
            const P *x = pxs + rr * G::kPxPitch + half * kQ;
            double acc[kQ];
#pragma unroll
            for (int q = 0; q < kQ; q++) acc[q] = 0.0;
#pragma unroll
            for (int sx = 0; sx < kQ + G::kHalo; sx++) {
                const double xv = (double)x[sx];
#pragma unroll
                for (int q = 0; q < kQ; q++) {
                    const int k = sx - q;
                    if (k >= 0 && k < G::kTaps) acc[q] = fma(tr.h[k], xv, acc[q]);
                }
            }
            double *o = ring + (dst + rr) * G::kRingPitch + half * kQ;
#pragma unroll
            for (int q = 0; q < kQ; q++) o[q] = acc[q];
        }
        __syncthreads();
    };

    // the 2 MT lines before the first output
    produce(i_beg - MT, G::kHalo, 0);
    for (int64_t done = 0; done < i_end - i_beg; done += kStep) {
        const int n = (int)(i_end - i_beg - done < kStep ? i_end - i_beg - done : kStep);
        produce(i_beg + MT + done, n, G::kHalo);
        // column pass: lane = column, warp wid = outputs [wid kQ, wid kQ + kQ) of this step
        if (wid * kQ < n) {
            const double *x = ring + (wid * kQ) * G::kRingPitch + lane;
            double acc[kQ];
#pragma unroll
            for (int q = 0; q < kQ; q++) acc[q] = 0.0;
#pragma unroll
            for (int sx = 0; sx < kQ + G::kHalo; sx++) {
                const double xv = x[sx * G::kRingPitch];
#pragma unroll
                for (int q = 0; q < kQ; q++) {
                    const int k = sx - q;
                    if (k >= 0 && k < G::kTaps) acc[q] = fma(tc.h[k], xv, acc[q]);
                }
            }
            const int64_t j = j0 + lane;
            if (j < cw) {
#pragma unroll
                for (int q = 0; q < kQ; q++) {
                    if (wid * kQ + q < n) {
                        const int64_t i = i_beg + done + wid * kQ + q;
                        c32[i * pitch32 + j] = (float)acc[q];
                        if (c64) c64[i * pitch64 + j] = acc[q];
                    }
                }
            }
        }
        if (n < kStep) break;  // the segment's last step
        __syncthreads();  // every column pass has read the ring
        // the last 2 MT lines become the first ones of the next step (n = kStep >= 2 MT: no overlap)
        for (int idx = tid; idx < G::kHalo * kStrip; idx += kFusedThreads) {
            const int rr = idx / kStrip, c = idx - rr * kStrip;
            ring[rr * G::kRingPitch + c] = ring[(kStep + rr) * G::kRingPitch + c];
        }
        __syncthreads();
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

// Blocks per SM of one fused instantiation at its shared memory (cached per
// device); also raises the kernel's dynamic shared-memory limit.
template <typename P, int MT>
int fused_blocks_per_sm(int *bps) {
    static std::mutex mu;
    static std::map<int, int> done;
    int dev = 0;
    GPV_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    auto it = done.find(dev);
    if (it == done.end()) {
        constexpr size_t smem = Fused<P, MT>::kSmem;
        GPV_CUDA_TRY(cudaFuncSetAttribute(prefilter_fused<P, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int n = 0;
        GPV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, prefilter_fused<P, MT>, kFusedThreads, smem));
        it = done.emplace(dev, n > 0 ? n : 1).first;
    }
    *bps = it->second;
    return GPV_SUCCESS;
}

// Coefficient rows [lo, hi) of an image whose lines both have at least kT
// samples, MT taps on each side.  Segments of rows split the work into about
// three waves of blocks, each segment at least 6 x 2 MT rows long (its 2 MT
// lead-in row-pass lines are the only work done twice).
template <typename P, int MT>
int launch_fused(gpv_image *img, const P *px, const Taps &tr, const Taps &tc, cudaStream_t s, int64_t lo, int64_t hi) {
    if (hi <= lo) return GPV_SUCCESS;
    int bps = 1;
    if (int rc = fused_blocks_per_sm<P, MT>(&bps)) return rc;
    TapArg ar, ac;
    fill_taparg_central(tr, MT, ar);
    fill_taparg_central(tc, MT, ac);
    const int64_t strips = (img->cw + kStrip - 1) / kStrip, rows = hi - lo;
    const int64_t target = 3LL * bps * std::max(1, img->ctx->num_sms);
    int64_t segs = std::max<int64_t>(1, (target + strips - 1) / strips);
    segs = std::min<int64_t>(segs, std::max<int64_t>(1, rows / (6 * 2 * MT)));
    const int64_t seg = (rows + segs - 1) / segs;
    segs = (rows + seg - 1) / seg;
    prefilter_fused<P, MT><<<dim3((unsigned)strips, (unsigned)segs), kFusedThreads, Fused<P, MT>::kSmem, s>>>(
        px, img->h, img->w, img->border, img->cw, img->ch, lo, hi, seg, ar, ac, img->c32, img->pitch32, img->c64,
        img->pitch64);
    GPV_CUDA_TRY(cudaGetLastError());
    return GPV_SUCCESS;
}

template <typename P>
int launch_fused_rows(gpv_image *img, const P *px, const Taps &tr, const Taps &tc, cudaStream_t s, int64_t lo,
                      int64_t hi) {
    // coefficients kept in FP32 only: |m| <= kM32
    return img->c64 == nullptr ? launch_fused<P, kM32>(img, px, tr, tc, s, lo, hi)
                               : launch_fused<P, kM>(img, px, tr, tc, s, lo, hi);
}

bool long_lines(const gpv_image *img) { return img->cw >= kT && img->ch >= kT; }

template <typename P>
int run_prefilter(gpv_image *img, const P *px, cudaStream_t s) {
    const Taps &tr = taps_for(img->cw);
    const Taps &tc = taps_for(img->ch);
    if (long_lines(img)) return launch_fused_rows(img, px, tr, tc, s, 0, img->ch);
    // a short line: every circulant tap, through the FP64 row-pass buffer
    {
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
    {
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
// Host pixels in row chunks into img->px_dev on the copy stream cs.  As each
// chunk lands, the coefficient rows whose lines all come from rows already
// landed are filtered on s, so the copies overlap the filtering; the first
// MT coefficient rows (their column taps wrap to the image's last rows) go
// after the last chunk.  Images with a short line take the whole copy, then
// the ordinary prefilter.
template <typename P>
int prefilter_host(gpv_image *img, const P *px_host, cudaStream_t s, cudaStream_t cs, cudaEvent_t *ev, int nev) {
    P *dst = static_cast<P *>(img->px_dev);
    const size_t row_bytes = sizeof(P) * (size_t)img->w;
    const Taps &tr = taps_for(img->cw);
    const Taps &tc = taps_for(img->ch);
    // rows per copy: ceil(h / (nev - 1)) rounded up to 32, so at most nev - 1
    // chunks (events ev[1 .. nev-1]) cover the image
    const int64_t chunk = ((img->h + nev - 2) / (nev - 1) + 31) / 32 * 32;
    // the copies wait for earlier work on s that may still read px_dev
    GPV_CUDA_TRY(cudaEventRecord(ev[0], s));
    GPV_CUDA_TRY(cudaStreamWaitEvent(cs, ev[0], 0));
    if (!long_lines(img) || img->h < 2 * 32 * (nev - 1)) {
        GPV_CUDA_TRY(cudaMemcpyAsync(dst, px_host, row_bytes * (size_t)img->h, cudaMemcpyHostToDevice, cs));
        GPV_CUDA_TRY(cudaEventRecord(ev[1], cs));
        GPV_CUDA_TRY(cudaStreamWaitEvent(s, ev[1], 0));
        return run_prefilter(img, static_cast<const P *>(dst), s);
    }
    const int64_t mt = img->c64 == nullptr ? kM32 : kM;
    int64_t lo = mt;  // coefficient rows [0, mt) wait for the last chunk
    int k = 1;
    for (int64_t r0 = 0; r0 < img->h; r0 += chunk, k++) {
        // the last event takes whatever rows remain (never an event past ev[nev - 1])
        const int64_t nr = k == nev - 1 ? img->h - r0 : std::min(chunk, img->h - r0);
        GPV_CUDA_TRY(cudaMemcpyAsync(dst + r0 * img->w, px_host + r0 * img->w, row_bytes * (size_t)nr,
                                     cudaMemcpyHostToDevice, cs));
        GPV_CUDA_TRY(cudaEventRecord(ev[k], cs));
        GPV_CUDA_TRY(cudaStreamWaitEvent(s, ev[k], 0));
        // coefficient row i reads image rows up to min(h - 1, i + mt - border)
        const int64_t landed = r0 + nr;
        const int64_t hi = landed >= img->h ? img->ch : std::min(img->ch, landed - mt + img->border);
        if (hi > lo) {
            if (int rc = launch_fused_rows(img, static_cast<const P *>(dst), tr, tc, s, lo, hi)) return rc;
            lo = hi;
        }
    }
    return launch_fused_rows(img, static_cast<const P *>(dst), tr, tc, s, 0, mt);
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

size_t prefilter_rowpass_bytes(int64_t h, int64_t cw, int64_t ch) {
    // the row pass plus two tap vectors of scratch, for the short-line kernels only
    return (cw >= kT && ch >= kT) ? 0 : sizeof(double) * (size_t)(h * cw + 2 * kT + 8);
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
