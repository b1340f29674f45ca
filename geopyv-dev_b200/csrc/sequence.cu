// sequence.cu -- frame-to-frame subset tracking with device-resident seeds.
//
// The per-frame work of a sequence (src/sequence.rs:624-968): a new target
// image is prefiltered (a1 again, :693-694, :914) and every subset is solved
// against the fixed reference with its initial warp taken from its own
// previous solution.  Here that work never leaves the device: the frame's
// pixels go to a staging buffer owned by the tracker, the target image is
// re-prefiltered in place, a kernel copies each subset's last converged warp
// into its descriptor, and the batched solve writes the frame's results.
// From the second frame on, those three steps are one CUDA graph, replayed
// once per frame; only the pixel upload and the optional result download
// sit outside it.
#include <algorithm>
#include <cstring>
#include <string>

#include "internal.h"

namespace gpv {
namespace {

// Seed every subset from its previous solution when that solve converged
// (status OK and converged); a failed subset keeps its last good warp.
__global__ void seed_from_previous(gpv_subset_desc *desc, const gpv_subset_result *prev, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const gpv_subset_result &r = prev[i];
    if (r.status != GPV_OK || !r.converged) return;
#pragma unroll
    for (int k = 0; k < 12; k++) desc[i].p0[k] = r.p[k];
}

}  // namespace
}  // namespace gpv

struct gpv_sequence {
    gpv_context *ctx = nullptr;
    const gpv_image *f = nullptr;
    gpv_image *g = nullptr;
    gpv_subset_desc *desc_dev = nullptr;
    gpv_subset_result *out_dev = nullptr;
    void *px_dev = nullptr;
    size_t px_bytes = 0;
    int32_t dtype = 0;
    int64_t n = 0;
    int max_radius = 0;
    gpv_solve_params prm{};
    uint32_t flags = 0;
    int64_t frames = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

using namespace gpv;

namespace {

// One frame's device work on ctx->stream: re-prefilter, seed, solve.
int frame_work(gpv_sequence *s, bool seed) {
    gpv_context *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    if (int rc = image_pixels_in(s->g, s->px_dev, s->dtype, st, false)) return rc;
    if (seed) {
        seed_from_previous<<<(unsigned)((s->n + 255) / 256), 256, 0, st>>>(s->desc_dev, s->out_dev, (int)s->n);
        GPV_CUDA_TRY(cudaGetLastError());
    }
    SolveLaunch L;
    L.f = s->f;
    L.g = s->g;
    L.desc = s->desc_dev;
    L.order = nullptr;
    L.n = s->n;
    L.prm = &s->prm;
    L.mask = s->prm.mask ? s->prm.mask->dev : nullptr;
    L.mh = s->prm.mask ? s->prm.mask->h : 0;
    L.mw = s->prm.mask ? s->prm.mask->w : 0;
    L.out = s->out_dev;
    L.history = nullptr;
    L.max_radius = s->max_radius;  // within the context's tables (reserved at creation)
    return solve_launch(ctx, L, st);
}

void release(gpv_sequence *s) {
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    cudaFree(s->desc_dev);
    cudaFree(s->out_dev);
    cudaFree(s->px_dev);
}

}  // namespace

extern "C" {

int gpv_sequence_create(gpv_context *ctx, const gpv_image *f, gpv_image *g, const gpv_subset_desc *desc, int64_t n,
                        const gpv_solve_params *params, int32_t dtype, uint32_t flags, gpv_sequence **out) {
    if (!ctx || !f || !g || !desc || !params || !out || n < 1 || n > INT32_MAX) {
        set_error("invalid sequence arguments");
        return GPV_ERR_INVALID;
    }
    *out = nullptr;
    if (f->ctx != ctx || g->ctx != ctx || f->h != g->h || f->w != g->w || f->border != g->border) {
        set_error("reference and target images must share the context, shape and border");
        return GPV_ERR_INVALID;
    }
    if (params->history) {
        set_error("a sequence keeps no iteration history");
        return GPV_ERR_INVALID;
    }
    if (params->precision == GPV_PREC_FP64 && (!f->c64 || !g->c64)) {
        set_error("GPV_PREC_FP64 needs images created with GPV_IMAGE_KEEP_F64");
        return GPV_ERR_INVALID;
    }
    const size_t esz = dtype == GPV_U8 ? 1 : dtype == GPV_U16 ? 2 : dtype == GPV_F32 ? 4 : dtype == GPV_F64 ? 8 : 0;
    if (!esz) {
        set_error("unknown pixel dtype");
        return GPV_ERR_INVALID;
    }
    int max_r = 0;
    for (int64_t i = 0; i < n; i++) max_r = std::max(max_r, (int)desc[i].radius);
    if (max_r < 1) {
        set_error("subset radii must be >= 1");
        return GPV_ERR_INVALID;
    }
    if (int rc = gpv_context_reserve(ctx, n, max_r, params->max_iterations)) return rc;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    auto *s = new gpv_sequence();
    s->ctx = ctx;
    s->f = f;
    s->g = g;
    s->n = n;
    s->max_radius = max_r;
    s->prm = *params;
    s->flags = flags;
    s->dtype = dtype;
    s->px_bytes = esz * (size_t)g->h * (size_t)g->w;
    cudaError_t e = cudaMalloc(&s->desc_dev, sizeof(gpv_subset_desc) * n);
    if (e == cudaSuccess) e = cudaMalloc(&s->out_dev, sizeof(gpv_subset_result) * n);
    if (e == cudaSuccess) e = cudaMalloc(&s->px_dev, s->px_bytes);
    if (e == cudaSuccess) e = cudaMemcpy(s->desc_dev, desc, sizeof(gpv_subset_desc) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(s->out_dev, 0, sizeof(gpv_subset_result) * n);
    if (e != cudaSuccess) {
        set_error(std::string("sequence allocation: ") + cudaGetErrorString(e));
        release(s);
        delete s;
        return GPV_ERR_NOMEM;
    }
    ctx->refs.fetch_add(1);
    *out = s;
    return GPV_SUCCESS;
}

int gpv_sequence_frame(gpv_sequence *s, const void *px, int32_t px_on_device, gpv_subset_result *out) {
    if (!s || !px) {
        set_error("NULL argument");
        return GPV_ERR_INVALID;
    }
    gpv_context *ctx = s->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    DeviceGuard dg(ctx->device);
    cudaStream_t st = ctx->stream;
    GPV_CUDA_TRY(cudaMemcpyAsync(s->px_dev, px, s->px_bytes,
                                 px_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    const bool seed = s->frames > 0;
    // the graph needs the large-image prefilter (no host synchronisation)
    const bool graph_ok = !(s->flags & GPV_SEQUENCE_NO_GRAPH) && s->g->cw >= 89 && s->g->ch >= 89;
    if (!seed || !graph_ok) {
        if (int rc = frame_work(s, seed)) return rc;
    } else {
        if (!s->exec) {
            GPV_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            const int rc = frame_work(s, true);
            cudaGraph_t graph = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(st, &graph);
            if (rc) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            GPV_CUDA_TRY(ce);
            s->graph = graph;
            GPV_CUDA_TRY(cudaGraphInstantiate(&s->exec, s->graph, 0));
        }
        GPV_CUDA_TRY(cudaGraphLaunch(s->exec, st));
    }
    s->frames++;
    if (out) {
        GPV_CUDA_TRY(cudaMemcpyAsync(out, s->out_dev, sizeof(gpv_subset_result) * s->n, cudaMemcpyDeviceToHost, st));
        GPV_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return GPV_SUCCESS;
}

gpv_subset_result *gpv_sequence_results_device(gpv_sequence *s) { return s ? s->out_dev : nullptr; }

int64_t gpv_sequence_frames(const gpv_sequence *s) { return s ? s->frames : -1; }

int gpv_sequence_destroy(gpv_sequence *s) {
    if (!s) return GPV_SUCCESS;
    gpv_context *ctx = s->ctx;
    {
        DeviceGuard dg(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        release(s);
    }
    delete s;
    gpv_context_destroy(ctx);  // drops the tracker's reference
    return GPV_SUCCESS;
}

}  // extern "C"
