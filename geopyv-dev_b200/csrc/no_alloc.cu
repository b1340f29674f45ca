// no_alloc.cu -- a batched ICGN solve that allocates no device memory.
//
// Who needs it: callers that must not call cudaMalloc / cudaFree on the
// solve path -- e.g. a host process whose device memory is owned by another
// framework's pooling allocator, or a latency-sensitive loop that cannot
// afford the device-wide synchronisation an allocation implies.  They pass
// inputs and outputs they already own; every piece of working memory comes
// from one file-scope static device array (g_static_scratch below).
//
// The solve is the warp-per-subset mixed-precision kernel of icgn.cu (same
// numerics; reference Subset::new + solve_icgn_result, src/subset.rs:836-919,
// 1117-1219).  Its working memory:
//   [work-queue counter | circle templates for radii 1..kStaticMaxRadius |
//    per-warp pixel scratch for as many warps as fit]
// The templates are written once per device by the set-up; the counter is
// cleared by every call; the pixel scratch is overwritten by every subset.
//
// Limits: radius <= kStaticMaxRadius (32 px); the number of concurrently
// working warps is what fits in kStaticBytes (64 MiB; a radius-32 subset
// needs 4 x 3,232 floats per warp).  Calls that overlap on the GPU (two
// streams, or two host threads) share the one array and race: serialise them.
#include <algorithm>
#include <mutex>
#include <string>

#include "icgn_common.cuh"
#include "icgn_warp.cuh"

namespace gpv {
namespace {

constexpr int kStaticMaxRadius = 32;
constexpr size_t kStaticBytes = size_t(64) << 20;
constexpr size_t kHeaderBytes = 256;  // queue counter (and padding)

// Every GPU that loads this library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

struct StaticLayout {
    size_t tab_off, tab_n, offs, pixels;  // byte offsets into the array
    int64_t stride;                       // floats of pixel scratch per warp
    int warps;                            // warps that fit
};

constexpr int circle_count(int r) {
    int n = 0;
    for (int y = -r; y <= r; y++)
        for (int x = -r; x <= r; x++)
            if (x * x + y * y <= r * r) n++;
    return n;
}

StaticLayout static_layout() {
    StaticLayout L;
    int total = 0;
    for (int r = 1; r <= kStaticMaxRadius; r++) total += circle_count(r);
    L.tab_off = kHeaderBytes;
    L.tab_n = L.tab_off + sizeof(int32_t) * (kStaticMaxRadius + 1);
    L.offs = L.tab_n + sizeof(int32_t) * (kStaticMaxRadius + 1);
    L.pixels = (L.offs + sizeof(short2) * (size_t)total + 255) / 256 * 256;
    const int64_t npx = circle_count(kStaticMaxRadius);
    L.stride = 4 * ((npx + 31) / 32 * 32);  // f, df/dx, df/dy, g
    L.warps = (int)((kStaticBytes - L.pixels) / (sizeof(float) * (size_t)L.stride));
    L.warps -= L.warps % kMixedWarps;
    return L;
}

// Circle templates for radii 1..R in the scan order of LocalMask::circle
// (src/masks.rs:69-109), written by one block.
__global__ void static_tables(int32_t *tab_off, int32_t *tab_n, short2 *offs) {
    if (threadIdx.x != 0) return;
    int pos = 0;
    tab_off[0] = 0;
    tab_n[0] = 0;
    for (int r = 1; r <= kStaticMaxRadius; r++) {
        tab_off[r] = pos;
        for (int y = -r; y <= r; y++)
            for (int x = -r; x <= r; x++)
                if (x * x + y * y <= r * r) offs[pos++] = make_short2((short)x, (short)y);
        tab_n[r] = pos - tab_off[r];
    }
}

__global__ void __launch_bounds__(kMixedWarps * 32, 2) icgn_mixed_static(KArgs A) {
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

// Per-device set-up state: the device address of g_static_scratch.
std::mutex g_static_mu;
unsigned char *g_static_base[64] = {nullptr};

}  // namespace

// Set-up, once per device, with that device current: resolve the array's
// device address (a host-side reference to g_static_scratch is only a
// stand-in, not a device address) and write the circle templates.  It
// synchronises `s`, so the first call on a device should come before any
// stream capture.
static int static_setup(int device, cudaStream_t s, unsigned char **base) {
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (device < 0 || device >= 64) {
        set_error("device index out of range");
        return GPV_ERR_INVALID;
    }
    if (!g_static_base[device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess || !ptr) {
            set_error(std::string("cudaGetSymbolAddress(g_static_scratch): ") + cudaGetErrorString(e));
            return GPV_ERR_CUDA;
        }
        unsigned char *b = static_cast<unsigned char *>(ptr);
        const StaticLayout L = static_layout();
        static_tables<<<1, 32, 0, s>>>(reinterpret_cast<int32_t *>(b + L.tab_off), reinterpret_cast<int32_t *>(b + L.tab_n),
                                       reinterpret_cast<short2 *>(b + L.offs));
        GPV_CUDA_TRY(cudaGetLastError());
        GPV_CUDA_TRY(cudaStreamSynchronize(s));
        g_static_base[device] = b;
    }
    *base = g_static_base[device];
    return GPV_SUCCESS;
}

int solve_noalloc_launch(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc_dev,
                         int64_t n, int max_radius, const gpv_solve_params *prm, gpv_subset_result *out_dev,
                         cudaStream_t s) {
    if (max_radius < 1 || max_radius > kStaticMaxRadius) {
        set_error("gpv_solve_batch_noalloc: max_radius " + std::to_string(max_radius) +
                  " is outside 1.." + std::to_string(kStaticMaxRadius) + ", the largest subset its static scratch holds");
        return GPV_ERR_INVALID;
    }
    unsigned char *base = nullptr;
    if (int rc = static_setup(ctx->device, s, &base)) return rc;
    const StaticLayout L = static_layout();
    KArgs A;
    A.f32 = f->c32; A.g32 = g->c32;
    A.f64 = nullptr; A.g64 = nullptr;
    A.pitch32 = f->pitch32; A.pitch64 = 0;
    A.h = (int)f->h; A.w = (int)f->w; A.border = f->border;
    A.desc = desc_dev; A.order = nullptr; A.n = (int)n;
    A.offs = reinterpret_cast<const short2 *>(base + L.offs);
    A.slots = nullptr;
    A.tab_off = reinterpret_cast<const int32_t *>(base + L.tab_off);
    A.tab_n = reinterpret_cast<const int32_t *>(base + L.tab_n);
    A.table_radius = kStaticMaxRadius;
    A.max_radius = max_radius;
    A.mask = prm->mask ? prm->mask->dev : nullptr;
    A.mh = prm->mask ? (int)prm->mask->h : 0;
    A.mw = prm->mask ? (int)prm->mask->w : 0;
    A.max_norm = prm->max_norm; A.tolerance = prm->tolerance;
    A.max_iter = prm->max_iterations; A.flags = prm->flags;
    A.out = out_dev; A.history = prm->history;
    A.scratch = base + L.pixels;
    A.scratch_stride = L.stride;
    A.queue = reinterpret_cast<int *>(base);
    int per_sm = 0;
    GPV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, icgn_mixed_static, kMixedWarps * 32, 0));
    int blocks = std::max(1, per_sm) * ctx->num_sms;
    blocks = std::min(blocks, L.warps / kMixedWarps);
    // the queue counter must start at zero on every call
    GPV_CUDA_TRY(cudaMemsetAsync(A.queue, 0, sizeof(int), s));
    icgn_mixed_static<<<blocks, kMixedWarps * 32, 0, s>>>(A);
    GPV_CUDA_TRY(cudaGetLastError());
    return GPV_SUCCESS;
}

}  // namespace gpv
