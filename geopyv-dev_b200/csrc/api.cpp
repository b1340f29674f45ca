// api.cpp -- the C ABI (include/gpv.h) over the device kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "internal.h"

namespace gpv {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int DevBuf::ensure(size_t want) {
    if (want <= bytes && ptr) return GPV_SUCCESS;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    const size_t sz = want < 256 ? 256 : want;
    cudaError_t e = cudaMalloc(&ptr, sz);
    if (e != cudaSuccess) {
        ptr = nullptr;
        set_error(std::string("cudaMalloc(") + std::to_string(sz) + "): " + cudaGetErrorString(e));
        return GPV_ERR_NOMEM;
    }
    bytes = sz;
    return GPV_SUCCESS;
}

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

int HostBuf::ensure(size_t want) {
    if (want <= bytes && ptr) return GPV_SUCCESS;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
    const size_t sz = want < 4096 ? 4096 : want;
    cudaError_t e = cudaHostAlloc(&ptr, sz, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        ptr = nullptr;
        set_error(std::string("cudaHostAlloc(") + std::to_string(sz) + "): " + cudaGetErrorString(e));
        return GPV_ERR_NOMEM;
    }
    bytes = sz;
    return GPV_SUCCESS;
}

void HostBuf::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

// Layout of the pinned staging of a host batch of n subsets: descriptors,
// work order, results, each at a 256-byte boundary.
static size_t stage_off_order(int64_t n) { return (sizeof(gpv_subset_desc) * (size_t)n + 255) / 256 * 256; }
static size_t stage_off_out(int64_t n) { return stage_off_order(n) + (sizeof(int32_t) * (size_t)n + 255) / 256 * 256; }
static size_t stage_bytes(int64_t n) { return stage_off_out(n) + sizeof(gpv_subset_result) * (size_t)n; }

int image_pixels_in(gpv_image *img, const void *px_dev, int dtype, cudaStream_t s, bool staged) {
    if (int rc = prefilter_launch(img, px_dev, dtype, s)) return rc;
    img->px_current = staged;
    if (staged) img->px_dtype = dtype;
    if (img->grain) return grain_launch(img, px_dev, dtype, s);
    return GPV_SUCCESS;
}

// Whether [p, p + bytes) is page-locked host memory of one allocation (its
// two ends pinned, mapped at the same distance on the device side).
static bool host_pinned(const void *p, size_t bytes) {
    if (!p || !bytes) return false;
    cudaPointerAttributes a, b;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    if (a.type != cudaMemoryTypeHost) return false;
    const char *q = static_cast<const char *>(p) + bytes - 1;
    if (cudaPointerGetAttributes(&b, q) != cudaSuccess) { cudaGetLastError(); return false; }
    return b.type == cudaMemoryTypeHost && a.devicePointer && b.devicePointer &&
           static_cast<const char *>(b.devicePointer) - static_cast<const char *>(a.devicePointer) == (ptrdiff_t)(bytes - 1);
}

// Host -> device from pageable memory through pinned staging, in chunks, so
// that the copy of one chunk into the staging overlaps the DMA of the last.
static int upload_staged(void *dst_dev, const void *src, void *stage, size_t bytes, cudaStream_t s) {
    const size_t chunk = std::max<size_t>(size_t(2) << 20, (bytes + 7) / 8);
    for (size_t off = 0; off < bytes; off += chunk) {
        const size_t len = std::min(chunk, bytes - off);
        std::memcpy(static_cast<char *>(stage) + off, static_cast<const char *>(src) + off, len);
        GPV_CUDA_TRY(cudaMemcpyAsync(static_cast<char *>(dst_dev) + off, static_cast<char *>(stage) + off, len,
                                     cudaMemcpyHostToDevice, s));
    }
    return GPV_SUCCESS;
}

// Device -> host into pageable memory through pinned staging: at most eight
// chunks, each copied out as soon as its DMA has landed.
static int download_staged(gpv_context *ctx, void *dst, const void *src_dev, void *stage, size_t bytes, cudaStream_t s) {
    const size_t chunk = std::max<size_t>(size_t(2) << 20, (bytes + 7) / 8);
    int m = 0;
    for (size_t off = 0; off < bytes; off += chunk, m++) {
        const size_t len = std::min(chunk, bytes - off);
        GPV_CUDA_TRY(cudaMemcpyAsync(static_cast<char *>(stage) + off, static_cast<const char *>(src_dev) + off, len,
                                     cudaMemcpyDeviceToHost, s));
        GPV_CUDA_TRY(cudaEventRecord(ctx->ev_chunk[m], s));
    }
    m = 0;
    for (size_t off = 0; off < bytes; off += chunk, m++) {
        const size_t len = std::min(chunk, bytes - off);
        GPV_CUDA_TRY(cudaEventSynchronize(ctx->ev_chunk[m]));
        std::memcpy(static_cast<char *>(dst) + off, static_cast<char *>(stage) + off, len);
    }
    return GPV_SUCCESS;
}

struct short2_h {
    int16_t x, y;
};
constexpr int16_t kSlotEmpty = -32768;  // padding slot of a template row (see icgn_tile.cu)

// Circular local masks for radii 1..max_radius in the scan order of
// LocalMask::circle (src/masks.rs:69-109): rows y = -r..r, columns x = -r..r,
// kept when sqrt(x^2 + y^2) <= r (i.e. x^2 + y^2 <= r^2 for integers).
int ensure_tables(gpv_context *ctx, int max_radius) {
    if (max_radius <= ctx->table_radius) return GPV_SUCCESS;
    if (max_radius > 4000) {
        set_error("radius above 4000 is not supported");
        return GPV_ERR_INVALID;
    }
    const int R1 = max_radius + 1;
    std::vector<short2_h> offs, slots;
    std::vector<int32_t> toff(R1, 0), tn(R1, 0), soff(R1, 0), sn(R1, 0), qoff(R1, 0), qn(R1, 0), nmax(R1, 0);
    for (int r = 1; r <= max_radius; r++) {
        toff[r] = (int32_t)offs.size();
        soff[r] = (int32_t)slots.size();
        for (int y = -r; y <= r; y++) {
            int row = 0;
            for (int x = -r; x <= r; x++)
                if (x * x + y * y <= r * r) {
                    offs.push_back({(int16_t)x, (int16_t)y});
                    slots.push_back({(int16_t)x, (int16_t)y});
                    row++;
                }
            // pad the template row to whole warps: a warp never straddles two rows
            while (row % 32) {
                slots.push_back({kSlotEmpty, (int16_t)y});
                row++;
            }
        }
        tn[r] = (int32_t)offs.size() - toff[r];
        sn[r] = (int32_t)slots.size() - soff[r];
    }
    // tiles: the disk covered by 8-wide x 4-high tiles, one per warp, slots in
    // tile order (4 rows of 8); with a window pitch of 8 mod 32 the 32 lanes
    // of a tile read 32 different shared-memory banks
    for (int r = 1; r <= max_radius; r++) {
        qoff[r] = (int32_t)slots.size();
        for (int y0 = -r; y0 <= r; y0 += 4) {
            int xmin = r + 1, xmax = -r - 1;
            for (int y = y0; y < y0 + 4 && y <= r; y++)
                for (int x = -r; x <= r; x++)
                    if (x * x + y * y <= r * r) { xmin = std::min(xmin, x); xmax = std::max(xmax, x); }
            for (int x0 = xmin; x0 <= xmax; x0 += 8)
                for (int ty = 0; ty < 4; ty++)
                    for (int tx = 0; tx < 8; tx++) {
                        const int x = x0 + tx, y = y0 + ty;
                        const bool in = y <= r && x * x + y * y <= r * r;
                        slots.push_back({in ? (int16_t)x : kSlotEmpty, (int16_t)y});
                    }
        }
        qn[r] = (int32_t)slots.size() - qoff[r];
        nmax[r] = std::max(std::max(tn[r], sn[r]), qn[r]);
    }
    if (int rc = ctx->offs.ensure(offs.size() * sizeof(short2_h))) return rc;
    if (int rc = ctx->slots.ensure(slots.size() * sizeof(short2_h))) return rc;
    if (int rc = ctx->tab_off.ensure(3 * toff.size() * sizeof(int32_t))) return rc;
    if (int rc = ctx->tab_n.ensure(3 * tn.size() * sizeof(int32_t))) return rc;
    GPV_CUDA_TRY(cudaMemcpy(ctx->offs.ptr, offs.data(), offs.size() * sizeof(short2_h), cudaMemcpyHostToDevice));
    GPV_CUDA_TRY(cudaMemcpy(ctx->slots.ptr, slots.data(), slots.size() * sizeof(short2_h), cudaMemcpyHostToDevice));
    // tab_off / tab_n: compact template tables, padded-row slot tables, tile slot tables
    std::vector<int32_t> to2(toff), tn2(tn);
    to2.insert(to2.end(), soff.begin(), soff.end());
    tn2.insert(tn2.end(), sn.begin(), sn.end());
    to2.insert(to2.end(), qoff.begin(), qoff.end());
    tn2.insert(tn2.end(), qn.begin(), qn.end());
    GPV_CUDA_TRY(cudaMemcpy(ctx->tab_off.ptr, to2.data(), to2.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    GPV_CUDA_TRY(cudaMemcpy(ctx->tab_n.ptr, tn2.data(), tn2.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    ctx->h_tab_off = toff;
    ctx->h_tab_n = tn;
    ctx->h_slot_n = nmax;  // the most slots any layout uses (per-block scratch)
    ctx->table_radius = max_radius;
    return GPV_SUCCESS;
}

static size_t dtype_size(int dtype) {
    switch (dtype) {
        case GPV_U8: return 1;
        case GPV_U16: return 2;
        case GPV_F32: return 4;
        case GPV_F64: return 8;
        default: return 0;
    }
}

}  // namespace gpv

using namespace gpv;

extern "C" {

static void tune_cache_load(gpv_context *ctx);
static void context_release(gpv_context *ctx);
static int grain_alloc(gpv_image *img);

const char *gpv_version(void) { return "gpv-b200 0.1.0 (sm_100a)"; }

int gpv_abi_version(void) { return GPV_ABI_VERSION; }

size_t gpv_last_error(char *buf, size_t len) {
    const std::string &e = g_last_error;
    if (buf && len) {
        const size_t k = std::min(len - 1, e.size());
        std::memcpy(buf, e.data(), k);
        buf[k] = 0;
    }
    return e.size();
}

int gpv_context_create(int device, gpv_context **out) { return gpv_context_create_ex(device, 0, out); }

int gpv_context_create_ex(int device, uint32_t flags, gpv_context **out) {
    if (!out) { set_error("out is NULL"); return GPV_ERR_INVALID; }
    *out = nullptr;
    if (flags & ~(GPV_CONTEXT_HIGH_PRIORITY | GPV_CONTEXT_PER_SUBSET_BLOCKS)) {
        set_error("unknown context flags");
        return GPV_ERR_INVALID;
    }
    int ndev = 0;
    GPV_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) { set_error("device index out of range"); return GPV_ERR_INVALID; }
    DeviceGuard dg(device);
    auto *ctx = new gpv_context();
    ctx->device = device;
    ctx->flags = flags;
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    const int prio = (flags & GPV_CONTEXT_HIGH_PRIORITY) ? greatest : least;
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, prio);
    for (int k = 0; k < 2 && e == cudaSuccess; k++) e = cudaStreamCreateWithPriority(&ctx->aux[k], cudaStreamNonBlocking, prio);
    for (int k = 0; k < 3 && e == cudaSuccess; k++) e = cudaEventCreateWithFlags(&ctx->ev[k], cudaEventDisableTiming);
    for (int k = 0; k < 8 && e == cudaSuccess; k++) e = cudaEventCreateWithFlags(&ctx->ev_chunk[k], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        set_error(std::string("context: ") + cudaGetErrorString(e));
        context_release(ctx);
        return GPV_ERR_CUDA;
    }
    if (flags & GPV_CONTEXT_PER_SUBSET_BLOCKS) {
        // claim words of the per-subset scratch slots: one per SM identifier
        // for each of the three stream regions, zero whenever no solve runs
        int rc = query_nsmid(&ctx->n_smid);
        if (!rc) rc = ctx->slot_mask.ensure(sizeof(uint32_t) * 3 * (size_t)ctx->n_smid);
        if (!rc && cudaMemset(ctx->slot_mask.ptr, 0, sizeof(uint32_t) * 3 * (size_t)ctx->n_smid) != cudaSuccess) {
            set_error("context: clearing the slot words failed");
            rc = GPV_ERR_CUDA;
        }
        if (rc) {
            context_release(ctx);
            return rc;
        }
    }
    tune_cache_load(ctx);
    *out = ctx;
    return GPV_SUCCESS;
}

static void context_release(gpv_context *ctx) {
    if (ctx->refs.fetch_sub(1) != 1) return;
    DeviceGuard dg(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (DevBuf *b : {&ctx->offs, &ctx->slots, &ctx->tab_off, &ctx->tab_n, &ctx->scratch, &ctx->queue, &ctx->desc_dev, &ctx->out_dev,
                      &ctx->order_dev, &ctx->hist_dev, &ctx->eval_dev, &ctx->tile_ws, &ctx->slot_mask,
                      &ctx->run_tasks, &ctx->run_off, &ctx->run_n})
        b->release();
    ctx->h_stage.release();
    for (int k = 0; k < 2; k++)
        if (ctx->aux[k]) cudaStreamDestroy(ctx->aux[k]);
    for (int k = 0; k < 3; k++)
        if (ctx->ev[k]) cudaEventDestroy(ctx->ev[k]);
    for (int k = 0; k < 8; k++)
        if (ctx->ev_chunk[k]) cudaEventDestroy(ctx->ev_chunk[k]);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int gpv_context_destroy(gpv_context *ctx) {
    if (!ctx) return GPV_SUCCESS;
    context_release(ctx);
    return GPV_SUCCESS;
}

void *gpv_context_stream(gpv_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

static int image_alloc(gpv_context *ctx, int64_t h, int64_t w, int32_t border, uint32_t flags, int32_t dtype,
                       gpv_image **out) {
    if (!ctx || !out) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    *out = nullptr;
    if (h < 1 || w < 1 || border < 3) { set_error("image needs h, w >= 1 and border >= 3"); return GPV_ERR_INVALID; }
    if (h + 2 * border > (1 << 30) || w + 2 * border > (1 << 30)) { set_error("image too large"); return GPV_ERR_INVALID; }
    if (!dtype_size(dtype)) { set_error("unknown pixel dtype"); return GPV_ERR_INVALID; }
    auto *img = new gpv_image();
    img->ctx = ctx;
    ctx->refs.fetch_add(1);
    img->h = h;
    img->w = w;
    img->border = border;
    img->ch = h + 2 * border;
    img->cw = w + 2 * border;
    img->pitch32 = (img->cw + 31) / 32 * 32;
    img->pitch64 = (img->cw + 15) / 16 * 16;
    img->flags = flags;
    cudaError_t e = cudaMalloc(&img->c32, sizeof(float) * img->pitch32 * img->ch);
    if (e == cudaSuccess && (flags & GPV_IMAGE_KEEP_F64)) e = cudaMalloc(&img->c64, sizeof(double) * img->pitch64 * img->ch);
    if (const size_t rb = prefilter_rowpass_bytes(img->h, img->cw, img->ch); e == cudaSuccess && rb)
        e = cudaMalloc(&img->rowpass, rb);
    if (e == cudaSuccess && (flags & GPV_IMAGE_GRAIN) && grain_alloc(img) != GPV_SUCCESS) e = cudaErrorMemoryAllocation;
    if (e != cudaSuccess) {
        set_error(std::string("image allocation: ") + cudaGetErrorString(e));
        cudaFree(img->c32);
        cudaFree(img->c64);
        cudaFree(img->rowpass);
        delete img;
        context_release(ctx);
        return GPV_ERR_NOMEM;
    }
    *out = img;
    return GPV_SUCCESS;
}

int gpv_image_create(gpv_context *ctx, const void *px, int32_t dtype, int64_t h, int64_t w, int32_t border,
                     uint32_t flags, gpv_image **out) {
    if (!px) { set_error("px is NULL"); return GPV_ERR_INVALID; }
    if (!ctx) { set_error("ctx is NULL"); return GPV_ERR_INVALID; }
    DeviceGuard dg(ctx->device);
    int rc = image_alloc(ctx, h, w, border, flags, dtype, out);
    if (rc) return rc;
    gpv_image *img = *out;
    img->px_bytes = dtype_size(dtype) * h * w;
    cudaError_t e = cudaMalloc(&img->px_dev, img->px_bytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(img->px_dev, px, img->px_bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
        set_error(std::string("pixel upload: ") + cudaGetErrorString(e));
        gpv_image_destroy(img);
        *out = nullptr;
        return GPV_ERR_CUDA;
    }
    rc = image_pixels_in(img, img->px_dev, dtype, ctx->stream, true);
    if (rc == GPV_SUCCESS) {
        e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) { set_error(std::string("prefilter: ") + cudaGetErrorString(e)); rc = GPV_ERR_CUDA; }
    }
    if (rc) { gpv_image_destroy(img); *out = nullptr; }
    return rc;
}

int gpv_image_create_device(gpv_context *ctx, const void *px_dev, int32_t dtype, int64_t h, int64_t w, int32_t border,
                            uint32_t flags, gpv_image **out) {
    if (!px_dev || !ctx) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    DeviceGuard dg(ctx->device);
    int rc = image_alloc(ctx, h, w, border, flags, dtype, out);
    if (rc) return rc;
    rc = image_pixels_in(*out, px_dev, dtype, ctx->stream, false);
    if (rc) { gpv_image_destroy(*out); *out = nullptr; }
    return rc;
}

int gpv_image_update_device(gpv_image *img, const void *px_dev, int32_t dtype) {
    if (!img || !px_dev) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    DeviceGuard dg(img->ctx->device);
    return image_pixels_in(img, px_dev, dtype, img->ctx->stream, px_dev == img->px_dev);
}

int gpv_image_update(gpv_image *img, const void *px, int32_t dtype) {
    if (!img || !px) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    const size_t bytes = dtype_size(dtype) * img->h * img->w;
    if (!bytes) { set_error("unknown pixel dtype"); return GPV_ERR_INVALID; }
    gpv_context *ctx = img->ctx;
    DeviceGuard dg(ctx->device);
    if (bytes > img->px_bytes) {
        cudaFree(img->px_dev);
        img->px_dev = nullptr;
        img->px_bytes = 0;
        GPV_CUDA_TRY(cudaMalloc(&img->px_dev, bytes));
        img->px_bytes = bytes;
    }
    if (host_pinned(px, bytes)) {
        // pinned pixels: the upload runs in row chunks beside the row passes
        if (!img->up_stream) {
            GPV_CUDA_TRY(cudaStreamCreateWithFlags(&img->up_stream, cudaStreamNonBlocking));
            for (cudaEvent_t &e : img->up_ev) GPV_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        if (int rc = prefilter_from_host(img, px, dtype, ctx->stream, img->up_stream, img->up_ev, 5)) return rc;
        img->px_current = true;
        img->px_dtype = dtype;
        if (img->grain) {
            if (int rc = grain_launch(img, img->px_dev, dtype, ctx->stream)) return rc;
        }
    } else {
        GPV_CUDA_TRY(cudaMemcpyAsync(img->px_dev, px, bytes, cudaMemcpyHostToDevice, ctx->stream));
        if (int rc = image_pixels_in(img, img->px_dev, dtype, ctx->stream, true)) return rc;
    }
    GPV_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GPV_SUCCESS;
}

// ---- colour ingest -----------------------------------------------------------

// RGB8 at rgb_dev -> grey u8 in the image's pixel staging -> coefficients.
static int image_from_rgb_dev(gpv_image *img, const uint8_t *rgb_dev) {
    gpv_context *ctx = img->ctx;
    const size_t bytes = (size_t)img->h * (size_t)img->w;
    if (bytes > img->px_bytes) {
        cudaFree(img->px_dev);
        img->px_dev = nullptr;
        img->px_bytes = 0;
        GPV_CUDA_TRY(cudaMalloc(&img->px_dev, bytes));
        img->px_bytes = bytes;
    }
    if (int rc = ingest_launch(rgb_dev, img->h, img->w, static_cast<uint8_t *>(img->px_dev), ctx->stream)) return rc;
    return image_pixels_in(img, img->px_dev, GPV_U8, ctx->stream, true);
}

static int stage_rgb(gpv_image *img, const uint8_t *rgb) {
    gpv_context *ctx = img->ctx;
    if (!img->rgb_dev) GPV_CUDA_TRY(cudaMalloc(&img->rgb_dev, (size_t)img->h * (size_t)img->w * 3));
    GPV_CUDA_TRY(cudaMemcpyAsync(img->rgb_dev, rgb, (size_t)img->h * (size_t)img->w * 3, cudaMemcpyHostToDevice,
                                 ctx->stream));
    return GPV_SUCCESS;
}

int gpv_image_create_rgb8(gpv_context *ctx, const uint8_t *rgb, int64_t h, int64_t w, int32_t border, uint32_t flags,
                          gpv_image **out) {
    if (!rgb || !ctx || !out) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    if (h < 3 || w < 3) { set_error("colour ingest needs an image of at least 3 x 3 pixels"); return GPV_ERR_INVALID; }
    DeviceGuard dg(ctx->device);
    int rc = image_alloc(ctx, h, w, border, flags, GPV_U8, out);
    if (rc) return rc;
    gpv_image *img = *out;
    rc = stage_rgb(img, rgb);
    if (!rc) rc = image_from_rgb_dev(img, img->rgb_dev);
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) { set_error(std::string("ingest: ") + cudaGetErrorString(e)); rc = GPV_ERR_CUDA; }
    }
    if (rc) { gpv_image_destroy(img); *out = nullptr; }
    return rc;
}

int gpv_image_update_rgb8(gpv_image *img, const uint8_t *rgb) {
    if (!img || !rgb) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    if (img->h < 3 || img->w < 3) { set_error("colour ingest needs an image of at least 3 x 3 pixels"); return GPV_ERR_INVALID; }
    DeviceGuard dg(img->ctx->device);
    if (int rc = stage_rgb(img, rgb)) return rc;
    if (int rc = image_from_rgb_dev(img, img->rgb_dev)) return rc;
    GPV_CUDA_TRY(cudaStreamSynchronize(img->ctx->stream));
    return GPV_SUCCESS;
}

int gpv_image_update_rgb8_device(gpv_image *img, const uint8_t *rgb_dev) {
    if (!img || !rgb_dev) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    if (img->h < 3 || img->w < 3) { set_error("colour ingest needs an image of at least 3 x 3 pixels"); return GPV_ERR_INVALID; }
    DeviceGuard dg(img->ctx->device);
    return image_from_rgb_dev(img, rgb_dev);
}

int gpv_image_grey(const gpv_image *img, uint8_t *out) {
    if (!img || !out) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    if (!img->px_dev || img->px_bytes < (size_t)img->h * (size_t)img->w) {
        set_error("the image holds no staged pixels");
        return GPV_ERR_INVALID;
    }
    DeviceGuard dg(img->ctx->device);
    GPV_CUDA_TRY(cudaMemcpyAsync(out, img->px_dev, (size_t)img->h * (size_t)img->w, cudaMemcpyDeviceToHost,
                                 img->ctx->stream));
    GPV_CUDA_TRY(cudaStreamSynchronize(img->ctx->stream));
    return GPV_SUCCESS;
}

int gpv_image_destroy(gpv_image *img) {
    if (!img) return GPV_SUCCESS;
    DeviceGuard dg(img->ctx->device);
    cudaStreamSynchronize(img->ctx->stream);
    cudaFree(img->c32);
    cudaFree(img->c64);
    cudaFree(img->rowpass);
    cudaFree(img->px_dev);
    cudaFree(img->rgb_dev);
    cudaFree(img->grain);
    cudaFree(img->grain64);
    cudaFree(img->grain_scal);
    cudaFree(img->grain_ac);
    if (img->up_stream) {
        cudaStreamSynchronize(img->up_stream);
        cudaStreamDestroy(img->up_stream);
    }
    for (cudaEvent_t e : img->up_ev)
        if (e) cudaEventDestroy(e);
    gpv_context *ctx = img->ctx;
    delete img;
    context_release(ctx);
    return GPV_SUCCESS;
}

static int grain_alloc(gpv_image *img) {
    if (img->grain) return GPV_SUCCESS;
    cudaError_t e = cudaMalloc(&img->grain, sizeof(float) * 3 * (size_t)img->h * (size_t)img->w);
    if (e == cudaSuccess && img->c64) e = cudaMalloc(&img->grain64, sizeof(double) * 3 * (size_t)img->h * (size_t)img->w);
    if (e == cudaSuccess) e = cudaMalloc(&img->grain_scal, sizeof(double) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&img->grain_ac, sizeof(double) * 512);
    if (e != cudaSuccess) {
        cudaFree(img->grain);
        cudaFree(img->grain64);
        cudaFree(img->grain_scal);
        cudaFree(img->grain_ac);
        img->grain = nullptr;
        img->grain64 = img->grain_scal = img->grain_ac = nullptr;
        set_error(std::string("grain maps: ") + cudaGetErrorString(e));
        return GPV_ERR_NOMEM;
    }
    return GPV_SUCCESS;
}

int gpv_image_build_grain(gpv_image *img) {
    if (!img) { set_error("img is NULL"); return GPV_ERR_INVALID; }
    if (img->grain) return GPV_SUCCESS;
    if (!img->px_current) {
        set_error("the image's pixels are not staged (device pixels): create it with GPV_IMAGE_GRAIN");
        return GPV_ERR_INVALID;
    }
    DeviceGuard dg(img->ctx->device);
    if (int rc = grain_alloc(img)) return rc;
    return grain_launch(img, img->px_dev, img->px_dtype, img->ctx->stream);
}

int gpv_image_grain(gpv_image *img, double *out3, int32_t *built, float *maps) {
    if (!img) { set_error("img is NULL"); return GPV_ERR_INVALID; }
    if (!img->grain) { set_error("the image keeps no grain maps"); return GPV_ERR_INVALID; }
    DeviceGuard dg(img->ctx->device);
    double sc[8];
    GPV_CUDA_TRY(cudaMemcpyAsync(sc, img->grain_scal, sizeof sc, cudaMemcpyDeviceToHost, img->ctx->stream));
    if (maps)
        GPV_CUDA_TRY(cudaMemcpyAsync(maps, img->grain, sizeof(float) * 3 * (size_t)img->h * (size_t)img->w,
                                     cudaMemcpyDeviceToHost, img->ctx->stream));
    GPV_CUDA_TRY(cudaStreamSynchronize(img->ctx->stream));
    if (out3) { out3[0] = sc[1]; out3[1] = sc[2]; out3[2] = sc[3]; }
    if (built) *built = sc[4] != 0.0;
    return GPV_SUCCESS;
}

int gpv_image_shape(const gpv_image *img, int64_t *h, int64_t *w, int32_t *border) {
    if (!img) { set_error("img is NULL"); return GPV_ERR_INVALID; }
    if (h) *h = img->h;
    if (w) *w = img->w;
    if (border) *border = img->border;
    return GPV_SUCCESS;
}

int gpv_image_coefficients_f32(const gpv_image *img, float *out) {
    if (!img || !out) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    DeviceGuard dg(img->ctx->device);
    GPV_CUDA_TRY(cudaStreamSynchronize(img->ctx->stream));
    GPV_CUDA_TRY(cudaMemcpy2D(out, sizeof(float) * img->cw, img->c32, sizeof(float) * img->pitch32,
                              sizeof(float) * img->cw, img->ch, cudaMemcpyDeviceToHost));
    return GPV_SUCCESS;
}

int gpv_image_coefficients_f64(const gpv_image *img, double *out) {
    if (!img || !out) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    if (!img->c64) { set_error("image was created without GPV_IMAGE_KEEP_F64"); return GPV_ERR_INVALID; }
    DeviceGuard dg(img->ctx->device);
    GPV_CUDA_TRY(cudaStreamSynchronize(img->ctx->stream));
    GPV_CUDA_TRY(cudaMemcpy2D(out, sizeof(double) * img->cw, img->c64, sizeof(double) * img->pitch64,
                              sizeof(double) * img->cw, img->ch, cudaMemcpyDeviceToHost));
    return GPV_SUCCESS;
}

int gpv_image_eval(const gpv_image *img, const double *xy, int64_t n, int32_t precision, double *val, double *grad) {
    if (!img || (!xy && n) || (!val && n)) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    if (n < 0) { set_error("n < 0"); return GPV_ERR_INVALID; }
    if (n == 0) return GPV_SUCCESS;
    gpv_context *ctx = img->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    if (int rc = ctx->eval_dev.ensure(sizeof(double) * 5 * n)) return rc;
    double *dxy = static_cast<double *>(ctx->eval_dev.ptr), *dout = dxy + 2 * n;
    GPV_CUDA_TRY(cudaMemcpyAsync(dxy, xy, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, ctx->stream));
    if (int rc = eval_launch(img, dxy, n, precision, dout, ctx->stream)) return rc;
    std::vector<double> h(3 * n);
    GPV_CUDA_TRY(cudaMemcpyAsync(h.data(), dout, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, ctx->stream));
    GPV_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int64_t i = 0; i < n; i++) {
        val[i] = h[3 * i];
        if (grad) {
            grad[2 * i] = h[3 * i + 1];
            grad[2 * i + 1] = h[3 * i + 2];
        }
    }
    return GPV_SUCCESS;
}

int gpv_image_grain_sample(gpv_image *img, const double *xy, int64_t n, double *out) {
    if (!img || (n && (!xy || !out)) || n < 0) { set_error("invalid arguments"); return GPV_ERR_INVALID; }
    if (!img->grain) { set_error("the image keeps no grain maps"); return GPV_ERR_INVALID; }
    if (n == 0) return GPV_SUCCESS;
    gpv_context *ctx = img->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    if (int rc = ctx->eval_dev.ensure(sizeof(double) * 5 * n)) return rc;
    double *dxy = static_cast<double *>(ctx->eval_dev.ptr), *dout = dxy + 2 * n;
    GPV_CUDA_TRY(cudaMemcpyAsync(dxy, xy, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, ctx->stream));
    if (int rc = grain_points_launch(img, dxy, n, dout, ctx->stream)) return rc;
    GPV_CUDA_TRY(cudaMemcpyAsync(out, dout, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, ctx->stream));
    GPV_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GPV_SUCCESS;
}

int gpv_mask_create(gpv_context *ctx, const uint8_t *mask, int64_t h, int64_t w, gpv_mask **out) {
    if (!ctx || !mask || !out || h < 1 || w < 1) { set_error("invalid mask arguments"); return GPV_ERR_INVALID; }
    DeviceGuard dg(ctx->device);
    auto *m = new gpv_mask();
    m->ctx = ctx;
    ctx->refs.fetch_add(1);
    m->h = h;
    m->w = w;
    cudaError_t e = cudaMalloc(&m->dev, (size_t)h * w);
    if (e == cudaSuccess) e = cudaMemcpy(m->dev, mask, (size_t)h * w, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        set_error(std::string("mask upload: ") + cudaGetErrorString(e));
        cudaFree(m->dev);
        delete m;
        context_release(ctx);
        return GPV_ERR_CUDA;
    }
    *out = m;
    return GPV_SUCCESS;
}

int gpv_mask_destroy(gpv_mask *m) {
    if (!m) return GPV_SUCCESS;
    gpv_context *ctx = m->ctx;
    {
        DeviceGuard dg(ctx->device);
        cudaFree(m->dev);
    }
    delete m;
    context_release(ctx);
    return GPV_SUCCESS;
}

int gpv_context_reserve(gpv_context *ctx, int64_t n_subsets, int32_t max_radius, int32_t max_iterations) {
    if (!ctx || n_subsets < 0 || max_radius < 1) { set_error("invalid reserve arguments"); return GPV_ERR_INVALID; }
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    if (int rc = ensure_tables(ctx, max_radius)) return rc;
    const int64_t npx = ctx->h_tab_n[max_radius];
    const int64_t stride = 4 * ((npx + 31) / 32 * 32);
    // enough for either kernel: 8 B per element, one slot per resident warp
    const size_t need = (size_t)ctx->num_sms * 64 * stride * sizeof(double);
    if (int rc = ctx->scratch.ensure(need)) return rc;
    if (int rc = ctx->queue.ensure(64)) return rc;
    if (int rc = ctx->desc_dev.ensure(sizeof(gpv_subset_desc) * (size_t)n_subsets)) return rc;
    if (int rc = ctx->out_dev.ensure(sizeof(gpv_subset_result) * (size_t)n_subsets)) return rc;
    if (int rc = ctx->order_dev.ensure(sizeof(int32_t) * (size_t)n_subsets)) return rc;
    if (int rc = ctx->tile_ws.ensure(sizeof(int32_t) * (96 + (size_t)n_subsets))) return rc;
    if (int rc = ctx->h_stage.ensure(stage_bytes(n_subsets))) return rc;
    (void)max_iterations;
    return GPV_SUCCESS;
}

static int check_pair(const gpv_image *f, const gpv_image *g, const gpv_solve_params *prm) {
    if (!f || !g || !prm) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    if (f->h != g->h || f->w != g->w || f->border != g->border) {
        set_error("reference and target images must have the same shape and border");
        return GPV_ERR_INVALID;
    }
    if (f->ctx != g->ctx) { set_error("images belong to different contexts"); return GPV_ERR_INVALID; }
    if (prm->max_iterations < 0) { set_error("max_iterations < 0"); return GPV_ERR_INVALID; }
    if (prm->precision != GPV_PREC_MIXED && prm->precision != GPV_PREC_FP64) {
        set_error("unknown precision");
        return GPV_ERR_INVALID;
    }
    if (prm->precision == GPV_PREC_FP64 && (!f->c64 || !g->c64)) {
        set_error("GPV_PREC_FP64 needs images created with GPV_IMAGE_KEEP_F64");
        return GPV_ERR_INVALID;
    }
    if (!(prm->max_norm >= 0.0)) { set_error("max_norm must be >= 0"); return GPV_ERR_INVALID; }
    return GPV_SUCCESS;
}

int gpv_solve_batch(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc, int64_t n,
                    const gpv_solve_params *prm, gpv_subset_result *out) {
    if (!ctx) { set_error("ctx is NULL"); return GPV_ERR_INVALID; }
    if (int rc = check_pair(f, g, prm)) return rc;
    if (n < 0 || (n > 0 && (!desc || !out))) { set_error("invalid batch arrays"); return GPV_ERR_INVALID; }
    if (n > INT32_MAX) { set_error("batch too large"); return GPV_ERR_INVALID; }
    if (n == 0) return GPV_SUCCESS;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    // the work order, and descriptors / results not already in pinned memory,
    // pass through pinned staging (copies from pageable memory go through the
    // driver's own staging, which can wait behind other streams' work)
    if (int rc = ctx->h_stage.ensure(stage_bytes(n))) return rc;
    char *stage = static_cast<char *>(ctx->h_stage.ptr);
    int32_t *order = reinterpret_cast<int32_t *>(stage + stage_off_order(n));
    const size_t desc_bytes = sizeof(gpv_subset_desc) * (size_t)n, out_bytes = sizeof(gpv_subset_result) * (size_t)n;
    const bool desc_pinned = host_pinned(desc, desc_bytes), out_pinned = host_pinned(out, out_bytes);
    if (int rc = ctx->desc_dev.ensure(desc_bytes)) return rc;
    if (int rc = ctx->out_dev.ensure(out_bytes)) return rc;
    if (int rc = ctx->order_dev.ensure(sizeof(int32_t) * n)) return rc;
    double *hist_dev = nullptr;
    const size_t hist_bytes = sizeof(double) * 3 * (size_t)n * (size_t)(prm->max_iterations > 0 ? prm->max_iterations : 1);
    if (prm->history) {
        if (int rc = ctx->hist_dev.ensure(hist_bytes)) return rc;
        hist_dev = static_cast<double *>(ctx->hist_dev.ptr);
        GPV_CUDA_TRY(cudaMemsetAsync(hist_dev, 0, hist_bytes, ctx->stream));
    }
    // the descriptors travel while the host builds the work order
    if (desc_pinned) {
        GPV_CUDA_TRY(cudaMemcpyAsync(ctx->desc_dev.ptr, desc, desc_bytes, cudaMemcpyHostToDevice, ctx->stream));
    } else if (int rc = upload_staged(ctx->desc_dev.ptr, desc, stage, desc_bytes, ctx->stream)) {
        return rc;
    }
    // largest subsets first (longest-processing-time order for the work
    // queue): a counting sort on key = 3 * radius + order, larger radius
    // first, order 2 before 1 before 0 (invalid subsets in bucket 0).  One
    // pass builds the histogram and finds the largest radius; the segment
    // sizes of the tiled launch come from the histogram.
    constexpr int kMaxR = 4000;
    constexpr int nk = 3 * (kMaxR + 1);
    static_assert(nk <= 65536, "work-order keys are 16-bit");
    std::vector<int64_t> start(nk + 1, 0);
    auto key = [](const gpv_subset_desc &d) -> int {
        const int r = d.radius, o = d.order;
        if (r < 1 || r > kMaxR || o < 0 || o > 2) return 0;
        return nk - 1 - (3 * r + o);
    };
    // the descriptors are read once: keys kept compact for the scatter
    ctx->h_keys.resize((size_t)n);
    uint16_t *keys = ctx->h_keys.data();
    int max_r = 1;
    for (int64_t i = 0; i < n; i++) {
        const gpv_subset_desc &d = desc[i];
        const int k = key(d);
        keys[i] = (uint16_t)k;
        start[k + 1]++;
        if (d.radius > max_r && d.radius <= kMaxR) max_r = d.radius;
    }
    const bool one_key = start[keys[0] + 1] == n;  // every subset in one bucket: the order is 0..n-1
    if (int rc = ensure_tables(ctx, max_r)) return rc;
    uint32_t seg_mask = 0;
    for (int q = 0; q < kTileSegs; q++) ctx->seg_count[q] = 0;
    for (int r = 1; r <= max_r; r++)
        for (int o = 0; o <= 2; o++) {
            const int64_t c = start[nk - 1 - (3 * r + o) + 1];
            if (!c) continue;
            const int q = tile_segment_of(r, o);
            ctx->seg_count[q] += c;
            seg_mask |= 1u << q;
        }
    if (one_key) {
        for (int64_t i = 0; i < n; i++) order[i] = (int32_t)i;
    } else {
        for (int k = 0; k < nk; k++) start[k + 1] += start[k];
        for (int64_t i = 0; i < n; i++) order[start[keys[i]]++] = (int32_t)i;
    }
    GPV_CUDA_TRY(cudaMemcpyAsync(ctx->order_dev.ptr, order, sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->stream));
    SolveLaunch L;
    L.f = f;
    L.g = g;
    L.desc = static_cast<const gpv_subset_desc *>(ctx->desc_dev.ptr);
    L.order = static_cast<const int32_t *>(ctx->order_dev.ptr);
    L.n = n;
    L.prm = prm;
    L.mask = prm->mask ? prm->mask->dev : nullptr;
    L.mh = prm->mask ? prm->mask->h : 0;
    L.mw = prm->mask ? prm->mask->w : 0;
    L.out = static_cast<gpv_subset_result *>(ctx->out_dev.ptr);
    L.history = hist_dev;
    L.max_radius = max_r;
    // launch only the segments this batch holds, each sized by its count
    ctx->seg_mask = seg_mask;
    ctx->seg_count_valid = true;
    const int rc_launch = solve_launch(ctx, L, ctx->stream);
    ctx->seg_mask = 0xFFFFFFFFu;
    ctx->seg_count_valid = false;
    if (rc_launch) return rc_launch;
    if (out_pinned) {
        GPV_CUDA_TRY(cudaMemcpyAsync(out, ctx->out_dev.ptr, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    } else if (int rc = download_staged(ctx, out, ctx->out_dev.ptr, stage + stage_off_out(n), out_bytes, ctx->stream)) {
        return rc;
    }
    if (prm->history) {
        GPV_CUDA_TRY(cudaMemcpyAsync(prm->history, hist_dev, hist_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    }
    GPV_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GPV_SUCCESS;
}

int gpv_solve_batch_device(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc_dev,
                           const int32_t *work_order_dev, int64_t n, const gpv_solve_params *prm,
                           gpv_subset_result *out_dev, void *stream) {
    if (!ctx) { set_error("ctx is NULL"); return GPV_ERR_INVALID; }
    if (int rc = check_pair(f, g, prm)) return rc;
    if (n < 0 || (n > 0 && (!desc_dev || !out_dev))) { set_error("invalid batch arrays"); return GPV_ERR_INVALID; }
    if (n > INT32_MAX) { set_error("batch too large"); return GPV_ERR_INVALID; }
    if (n == 0) return GPV_SUCCESS;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    if (ctx->table_radius < 1) {
        set_error("call gpv_context_reserve first (it fixes the largest radius the device path accepts)");
        return GPV_ERR_INVALID;
    }
    SolveLaunch L;
    L.f = f;
    L.g = g;
    L.desc = desc_dev;
    L.order = work_order_dev;
    L.n = n;
    L.prm = prm;
    L.mask = prm->mask ? prm->mask->dev : nullptr;
    L.mh = prm->mask ? prm->mask->h : 0;
    L.mw = prm->mask ? prm->mask->w : 0;
    L.out = out_dev;
    L.history = prm->history;
    L.max_radius = ctx->table_radius;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    return solve_launch(ctx, L, s);
}

}  // extern "C"

// Addresses of the context workspace a captured solve reads and writes.
struct WorkspaceAddrs {
    const void *p[11];
    bool operator==(const WorkspaceAddrs &o) const { return std::memcmp(p, o.p, sizeof p) == 0; }
};
static WorkspaceAddrs workspace_addrs(const gpv_context *ctx) {
    return WorkspaceAddrs{{ctx->scratch.ptr, ctx->queue.ptr, ctx->tile_ws.ptr, ctx->offs.ptr, ctx->slots.ptr,
                           ctx->tab_off.ptr, ctx->tab_n.ptr, ctx->slot_mask.ptr, ctx->run_tasks.ptr, ctx->run_off.ptr,
                           ctx->run_n.ptr}};
}

struct gpv_batch_graph {
    gpv_context *ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    WorkspaceAddrs ws{};
};

extern "C" {

int gpv_batch_graph_create(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc_dev,
                           const int32_t *work_order_dev, int64_t n, const gpv_solve_params *prm,
                           gpv_subset_result *out_dev, gpv_batch_graph **out) {
    if (!out) { set_error("out is NULL"); return GPV_ERR_INVALID; }
    *out = nullptr;
    if (prm && prm->history) { set_error("a batch graph keeps no iteration history"); return GPV_ERR_INVALID; }
    if (n < 1) { set_error("a batch graph needs at least one subset"); return GPV_ERR_INVALID; }
    // the eager run checks the arguments and sizes the workspace
    if (int rc = gpv_solve_batch_device(ctx, f, g, desc_dev, work_order_dev, n, prm, out_dev, nullptr)) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    GPV_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    SolveLaunch L;
    L.f = f;
    L.g = g;
    L.desc = desc_dev;
    L.order = work_order_dev;
    L.n = n;
    L.prm = prm;
    L.mask = prm->mask ? prm->mask->dev : nullptr;
    L.mh = prm->mask ? prm->mask->h : 0;
    L.mw = prm->mask ? prm->mask->w : 0;
    L.out = out_dev;
    L.history = nullptr;
    L.max_radius = ctx->table_radius;
    auto *bg = new gpv_batch_graph();
    bg->ctx = ctx;
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        delete bg;
        set_error(std::string("stream capture: ") + cudaGetErrorString(e));
        return GPV_ERR_CUDA;
    }
    const int rc = solve_launch(ctx, L, st);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(st, &graph);
    if (rc || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        delete bg;
        if (!rc) set_error(std::string("stream capture: ") + cudaGetErrorString(e));
        return rc ? rc : GPV_ERR_CUDA;
    }
    bg->graph = graph;
    e = cudaGraphInstantiate(&bg->exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        delete bg;
        set_error(std::string("graph instantiate: ") + cudaGetErrorString(e));
        return GPV_ERR_CUDA;
    }
    bg->ws = workspace_addrs(ctx);
    ctx->refs.fetch_add(1);  // the graph uses the context's workspace
    *out = bg;
    return GPV_SUCCESS;
}

int gpv_batch_graph_launch(gpv_batch_graph *bg, void *stream) {
    if (!bg) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    gpv_context *ctx = bg->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!(workspace_addrs(ctx) == bg->ws)) {
        set_error("the context's workspace moved since the graph was captured (reserve first, or recreate the graph)");
        return GPV_ERR_INVALID;
    }
    DeviceGuard dg(ctx->device);
    GPV_CUDA_TRY(cudaGraphLaunch(bg->exec, stream ? static_cast<cudaStream_t>(stream) : ctx->stream));
    return GPV_SUCCESS;
}

int gpv_batch_graph_destroy(gpv_batch_graph *bg) {
    if (!bg) return GPV_SUCCESS;
    gpv_context *ctx = bg->ctx;
    {
        DeviceGuard dg(ctx->device);
        if (bg->exec) cudaGraphExecDestroy(bg->exec);
        if (bg->graph) cudaGraphDestroy(bg->graph);
    }
    delete bg;
    context_release(ctx);
    return GPV_SUCCESS;
}

static int check_pair(const gpv_image *f, const gpv_image *g, const gpv_solve_params *prm);

int gpv_solve_batch_noalloc(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc_dev,
                            int64_t n, int32_t max_radius, const gpv_solve_params *prm, gpv_subset_result *out_dev,
                            void *stream) {
    if (!ctx) { set_error("ctx is NULL"); return GPV_ERR_INVALID; }
    if (int rc = check_pair(f, g, prm)) return rc;
    if (prm->precision != GPV_PREC_MIXED || (prm->flags & (GPV_SOLVE_FAGN | GPV_SOLVE_RIGID_TEXTURE))) {
        set_error("gpv_solve_batch_noalloc runs the mixed-precision ICGN solve with the deformable template only");
        return GPV_ERR_INVALID;
    }
    if (n < 0 || (n > 0 && (!desc_dev || !out_dev)) || n > INT32_MAX) { set_error("invalid batch arrays"); return GPV_ERR_INVALID; }
    if (n == 0) return GPV_SUCCESS;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    return solve_noalloc_launch(ctx, f, g, desc_dev, n, max_radius, prm, out_dev, s);
}

// ---- mesh driver ----------------------------------------------------------

struct GpuMeshSolver {
    gpv_context *ctx;
    const gpv_image *f, *g;
    gpv_solve_params prm;
};

static int gpu_mesh_solver(void *user, const gpv_subset_desc *desc, int64_t n, double tolerance,
                           gpv_subset_result *out) {
    auto *S = static_cast<GpuMeshSolver *>(user);
    gpv_solve_params q = S->prm;
    q.tolerance = tolerance;
    return gpv_solve_batch(S->ctx, S->f, S->g, desc, n, &q, out);
}

int gpv_mesh_drive(const double *nodes, int64_t n_nodes, const int64_t *elements, int64_t n_elements,
                   int32_t nodes_per_element, const gpv_mesh_params *params, gpv_batch_solver_fn solver,
                   void *solver_user, gpv_subset_result *out, int32_t *rounds, gpv_mesh_stats *stats) {
    return gpv::mesh_drive(nodes, n_nodes, elements, n_elements, nodes_per_element, params, solver, solver_user, out,
                           rounds, stats);
}

int gpv_mesh_solve(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const double *nodes, int64_t n_nodes,
                   const int64_t *elements, int64_t n_elements, int32_t nodes_per_element,
                   const gpv_mesh_params *params, gpv_subset_result *out, int32_t *rounds, gpv_mesh_stats *stats) {
    if (!ctx || !params) { set_error("ctx or params is NULL"); return GPV_ERR_INVALID; }
    GpuMeshSolver S;
    S.ctx = ctx; S.f = f; S.g = g;
    std::memset(&S.prm, 0, sizeof(S.prm));
    S.prm.max_norm = params->max_norm;
    S.prm.tolerance = params->tolerance;
    S.prm.max_iterations = params->max_iterations;
    S.prm.precision = params->precision;
    S.prm.mask = params->mask;
    S.prm.flags = (params->method == 1 ? GPV_SOLVE_FAGN : 0u) | (params->texture == 1 ? GPV_SOLVE_RIGID_TEXTURE : 0u);
    if (int rc = check_pair(f, g, &S.prm)) return rc;
    return gpv::mesh_drive(nodes, n_nodes, elements, n_elements, nodes_per_element, params, gpu_mesh_solver, &S, out,
                           rounds, stats);
}

static int radius_class(int r) { return r <= 20 ? 0 : (r <= 40 ? 1 : 2); }

extern "C++" {
namespace gpv {
bool use_run_kernel();  // icgn_tile.cu
}
}

static void tune_cache_load(gpv_context *ctx) {
    const char *path = getenv("GPV_TUNE_CACHE");
    if (!path) return;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) return;
    FILE *fh = fopen(path, "r");
    if (!fh) return;
    char line[512];
    while (fgets(line, sizeof line, fh)) {
        char name[256];
        int cls = -1, nt = 0, layout = -1, runk = 0;
        const int got = sscanf(line, "%255[^|]|%d|%d|%d|%d", name, &cls, &nt, &layout, &runk);
        if (got >= 3 && cls >= 0 && cls < 3 && strcmp(name, prop.name) == 0 && (nt == 64 || nt == 128 || nt == 256)) {
            ctx->tuned_threads[cls] = nt;  // later lines win
            ctx->tuned_layout[cls] = (got >= 4 && layout >= 0 && layout <= 2) ? layout : -1;
            ctx->tuned_run_k[cls] = (got == 5 && (runk == 4 || runk == 8)) ? runk : 0;
        }
    }
    fclose(fh);
}

int gpv_autotune(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc, int64_t n,
                 const gpv_solve_params *prm, int32_t sample_per_class, int32_t *threads_out) {
    if (!ctx || !desc || n <= 0 || sample_per_class < 1) { set_error("invalid autotune arguments"); return GPV_ERR_INVALID; }
    if (int rc = check_pair(f, g, prm)) return rc;
    std::vector<std::vector<gpv_subset_desc>> cls(3);
    for (int64_t i = 0; i < n; i++) {
        const int r = desc[i].radius;
        if (r < 1 || r > 4000 || desc[i].order < 0 || desc[i].order > 2) continue;
        cls[radius_class(r)].push_back(desc[i]);
    }
    gpv_solve_params p = *prm;
    p.precision = GPV_PREC_MIXED;
    p.history = nullptr;
    p.flags &= ~(GPV_SOLVE_ETA | GPV_SOLVE_FAGN | GPV_SOLVE_RIGID_TEXTURE);  // the tuned kernel is the mixed ICGN one
    // candidates: threads per block x run length (run-layout kernel), or
    // threads per block x template layout (compact, 8 x 4 tiles) when the
    // tiled kernel is selected
    const bool runs = use_run_kernel();
    static const int cand_runs[6][2] = {{128, 8}, {256, 8}, {128, 4}, {256, 4}, {64, 4}, {64, 8}};
    static const int cand_tile[4][2] = {{128, 0}, {256, 0}, {128, 2}, {256, 2}};
    const int(*cand)[2] = runs ? cand_runs : cand_tile;
    const int ncand = runs ? 6 : 4;
    for (int c = 0; c < 3; c++) {
        if (threads_out) threads_out[c] = 0;
        if (cls[c].empty()) continue;
        // an even sample of the class
        std::vector<gpv_subset_desc> smp;
        const size_t k = std::min<size_t>(cls[c].size(), (size_t)sample_per_class);
        for (size_t j = 0; j < k; j++) smp.push_back(cls[c][j * cls[c].size() / k]);
        std::vector<gpv_subset_result> out(smp.size());
        double best = 1e300;
        int best_nt = 128, best_layout = 0, best_k = 0;
        for (int ci = 0; ci < ncand; ci++) {
            const int *cd = cand[ci];
            const int t = cd[0];
            ctx->force_threads = t;
            ctx->force_layout = runs ? -1 : cd[1];
            ctx->force_run_k = runs ? cd[1] : 0;
            double ms_best = 1e300;
            for (int rep = 0; rep < 3; rep++) {
                cudaEvent_t e0, e1;
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                cudaEventRecord(e0, ctx->stream);
                int rc = gpv_solve_batch(ctx, f, g, smp.data(), (int64_t)smp.size(), &p, out.data());
                cudaEventRecord(e1, ctx->stream);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                if (rc) { ctx->force_threads = 0; ctx->force_layout = -1; ctx->force_run_k = 0; return rc; }
                if (rep > 0) ms_best = std::min(ms_best, (double)ms);
            }
            if (ms_best < best) {
                best = ms_best;
                best_nt = t;
                best_layout = runs ? -1 : cd[1];
                best_k = runs ? cd[1] : 0;
            }
        }
        ctx->force_threads = 0;
        ctx->force_layout = -1;
        ctx->force_run_k = 0;
        ctx->tuned_threads[c] = best_nt;
        ctx->tuned_layout[c] = best_layout;
        ctx->tuned_run_k[c] = best_k;
        if (threads_out) threads_out[c] = best_nt;
        if (const char *path = getenv("GPV_TUNE_CACHE")) {
            cudaDeviceProp prop;
            if (cudaGetDeviceProperties(&prop, ctx->device) == cudaSuccess) {
                if (FILE *fh = fopen(path, "a")) {
                    fprintf(fh, "%s|%d|%d|%d|%d\n", prop.name, c, best_nt, best_layout, best_k);
                    fclose(fh);
                }
            }
        }
    }
    return GPV_SUCCESS;
}

int gpv_context_tuning(gpv_context *ctx, int32_t *threads, int32_t *layouts) {
    if (!ctx) { set_error("ctx is NULL"); return GPV_ERR_INVALID; }
    std::lock_guard<std::mutex> lk(ctx->mu);
    for (int c = 0; c < 3; c++) {
        if (threads) threads[c] = ctx->tuned_threads[c];
        if (layouts) layouts[c] = ctx->tuned_layout[c];
    }
    return GPV_SUCCESS;
}

int gpv_context_tuning_get(gpv_context *ctx, gpv_tuning *out) {
    if (!ctx || !out) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    std::lock_guard<std::mutex> lk(ctx->mu);
    for (int c = 0; c < 3; c++) {
        out[c].threads = ctx->tuned_threads[c];
        out[c].layout = ctx->tuned_layout[c];
        out[c].run_length = ctx->tuned_run_k[c];
        out[c].subsets_per_block = 0;
        out[c].staging = 0;
        out[c].reserved = 0;
    }
    return GPV_SUCCESS;
}

int gpv_probe_fp32_peak(gpv_context *ctx, double *tflops) {
    if (!ctx || !tflops) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    return probe_fp32_peak(ctx, tflops);
}

int gpv_probe_peaks(gpv_context *ctx, gpv_peaks *out) {
    if (!ctx || !out) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    return probe_peaks(ctx, out);
}

}  // extern "C"
