// internal.h -- host-side objects behind the C ABI (include/gpv.h).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gpv.h"

namespace gpv {

void set_error(const std::string &msg);

#define GPV_CUDA_TRY(expr)                                                                       \
    do {                                                                                         \
        cudaError_t _e = (expr);                                                                 \
        if (_e != cudaSuccess) {                                                                 \
            ::gpv::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));                \
            return GPV_ERR_CUDA;                                                                 \
        }                                                                                        \
    } while (0)

// Taps of the periodised inverse quintic filter for one circular length.
// c[n] = sum_{m=-ml}^{mr} h[m + ml] * x[(n - m) mod N].
struct Taps {
    int n = 0, ml = 0, mr = 0;
    std::vector<double> h;
};
const Taps &taps_for(int64_t n);  // cached, thread-safe

// Device buffer that only grows.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t want);
    void release();
};

// Pinned (page-locked) host memory, grown on demand.  Copies between the
// device and pageable memory go through the driver's own staging and can
// wait behind other streams' work; from pinned memory they are plain DMA on
// the caller's stream.
struct HostBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t want);
    void release();
};

// Makes `dev` current for a scope and restores the caller's device.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace gpv

struct gpv_context {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    // circular mask offset tables, radii 1..table_radius (short2 per pixel)
    int table_radius = 0;
    gpv::DevBuf offs;     // short2, compact circle templates
    gpv::DevBuf slots;    // short2, templates with rows padded to 32 (x = -32768: empty)
    gpv::DevBuf tab_off;  // int32 [table_radius + 1]
    gpv::DevBuf tab_n;    // int32 [table_radius + 1]
    std::vector<int32_t> h_tab_off, h_tab_n, h_slot_n;
    std::vector<uint16_t> h_keys;  // work-order keys of a host batch (one pass over its descriptors)
    // solve workspace
    gpv::DevBuf scratch;   // per-warp / per-block pixel arrays
    gpv::DevBuf queue;     // work-queue counters
    gpv::DevBuf desc_dev;  // staging for the host API
    gpv::DevBuf out_dev;
    gpv::DevBuf order_dev;
    gpv::DevBuf hist_dev;
    gpv::DevBuf eval_dev;
    gpv::DevBuf tile_ws;               // order partition + per-kernel queues
    cudaStream_t aux[2] = {nullptr, nullptr};  // extra streams for the per-order kernels
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    int mixed_blocks_per_sm = 0;
    int tuned_threads[3] = {0, 0, 0};  // autotuned threads per block by radius class
    int force_threads = 0;             // set while the autotuner times a candidate
    int tuned_layout[3] = {-1, -1, -1};  // autotuned template layout by radius class (-1: compact)
    int force_layout = -1;               // set while the autotuner times a candidate
    uint32_t seg_mask = 0xFFFFFFFFu;   // tiled-solve segments a host batch holds (all when unknown)
    int64_t seg_count[12] = {};        // subsets per segment of that batch (valid with seg_count_valid)
    bool seg_count_valid = false;
    uint32_t flags = 0;                // GPV_CONTEXT_*
    int n_smid = 0;                    // SM identifiers of the device (per-subset blocks)
    gpv::DevBuf slot_mask;             // per stream region, per SM: claimed scratch slots
    // run tables of the run-layout solve (icgn_runs.cu): lengths 4 and 8, radii 1..run_table_radius
    int run_table_radius = 0;
    gpv::DevBuf run_tasks;             // int2 per task: dx | dy0 << 16, circle bits
    gpv::DevBuf run_off, run_n;        // int32 [2][run_table_radius + 1]
    std::vector<int32_t> h_run_n;
    int tuned_run_k[3] = {0, 0, 0};    // autotuned run length by radius class (0: default)
    int force_run_k = 0;               // set while the autotuner times a candidate
    gpv::HostBuf h_stage;              // pinned staging of host batches: desc | work order | results
    cudaEvent_t ev_chunk[8] = {};      // chunked result downloads through h_stage
    // owner reference + one per image / mask created on it: the context is
    // freed when gpv_context_destroy and every dependant's destroy have run,
    // in whatever order they come
    std::atomic<int> refs{1};
};

struct gpv_image {
    gpv_context *ctx = nullptr;
    int64_t h = 0, w = 0, ch = 0, cw = 0;
    int32_t border = 0;
    int64_t pitch32 = 0, pitch64 = 0;  // elements per coefficient row
    float *c32 = nullptr;
    double *c64 = nullptr;
    double *rowpass = nullptr;  // FP64 row-pass intermediate (h, cw): images with a line under 89 samples only
    void *px_dev = nullptr;     // staging for host pixels
    size_t px_bytes = 0;
    uint8_t *rgb_dev = nullptr;  // staging for colour pixels (h * w * 3)
    uint32_t flags = 0;
    int32_t px_dtype = -1;     // pixel type of px_dev
    bool px_current = false;   // px_dev holds the pixels behind the coefficients
    // rigid-texture speckle statistics (grain.cu): fxx, fyy, fxy maps (3 h w
    // FP32) and [mean, correlation length, s2, corr, built] on the device
    float *grain = nullptr;
    double *grain64 = nullptr;  // the same maps in FP64 (images that keep FP64 coefficients)
    double *grain_scal = nullptr;
    double *grain_ac = nullptr;  // autocorrelation lag sums (2 x 256)
    // chunked uploads of pinned host pixels (created on first use)
    cudaStream_t up_stream = nullptr;
    cudaEvent_t up_ev[5] = {};
};

struct gpv_mask {
    gpv_context *ctx = nullptr;
    int64_t h = 0, w = 0;
    uint8_t *dev = nullptr;
};

namespace gpv {
// prefilter.cu
int prefilter_launch(gpv_image *img, const void *px_dev, int dtype, cudaStream_t s);
// the FP64 row-pass buffer an image of this padded size needs (bytes; 0: none)
size_t prefilter_rowpass_bytes(int64_t h, int64_t cw, int64_t ch);
// host pixels (pinned) -> img->px_dev in row chunks on cs, each chunk's row
// pass on s once it has landed, then the column pass on s; ev: nev >= 2 events
int prefilter_from_host(gpv_image *img, const void *px_host, int dtype, cudaStream_t s, cudaStream_t cs,
                        cudaEvent_t *ev, int nev);
// New pixels into an image: prefilter, and the grain maps when it keeps them.
// staged: px_dev is the image's own staging (it then holds the pixels).
int image_pixels_in(gpv_image *img, const void *px_dev, int dtype, cudaStream_t s, bool staged);
// grain.cu: correlation length, s2, corr and the three maps of img from its pixels
int grain_launch(gpv_image *img, const void *px_dev, int dtype, cudaStream_t s);
// the maps at n device points (x, y) -> 3 values per point
int grain_points_launch(const gpv_image *img, const double *xy_dev, int64_t n, double *out_dev, cudaStream_t s);
// icgn.cu
struct SolveLaunch {
    const gpv_image *f, *g;
    const gpv_subset_desc *desc;  // device
    const int32_t *order;         // device or null
    int64_t n;
    const gpv_solve_params *prm;
    const uint8_t *mask;
    int64_t mh, mw;
    gpv_subset_result *out;  // device
    double *history;         // device or null
    int max_radius;
};
int solve_launch(gpv_context *ctx, const SolveLaunch &L, cudaStream_t s);
int eval_launch(const gpv_image *img, const double *xy_dev, int64_t n, int precision, double *out_dev,
                cudaStream_t s);
int ensure_tables(gpv_context *ctx, int max_radius);
int probe_fp32_peak(gpv_context *ctx, double *tflops);
int probe_peaks(gpv_context *ctx, gpv_peaks *out);  // probe.cu
int mesh_drive(const double *nodes, int64_t n_nodes, const int64_t *elements, int64_t n_elements,
               int32_t nodes_per_element, const gpv_mesh_params *mp, gpv_batch_solver_fn solver, void *solver_user,
               gpv_subset_result *out, int32_t *rounds, gpv_mesh_stats *stats);
// Colour ingest (load_grayscale + gaussian_blur_5x5): RGB8 (h, w, 3) -> u8 grey.
int ingest_launch(const uint8_t *rgb_dev, int64_t h, int64_t w, uint8_t *grey_dev, cudaStream_t s);
// Threads per block / template layout (0 compact, 1 padded rows, 2 tiles) of
// the tiled solve for subsets up to max_radius: GPV_TILE_THREADS /
// GPV_TILE_LAYOUT, else a candidate being timed, else the tuned choice.
int tile_threads_for(gpv_context *ctx, int max_radius);
int tile_layout_for(gpv_context *ctx, int max_radius);
// The (order, radius class) segment of the tiled solve that holds a valid
// subset of radius r and warp order o (0 <= q < kTileSegs); a host batch's
// per-segment counts let the launcher skip empty segments and size
// one-block-per-subset grids.
constexpr int kTileSegs = 12;
int tile_segment_of(int r, int o);
// Number of SM identifiers (%nsmid) of the current device.
int query_nsmid(int *out);
// icgn_runs.cu: the run-layout solve kernel (one block per subset at a
// time, runs of K template pixels per lane)
int ensure_run_tables(gpv_context *ctx, int max_radius);
int run_window_cap(int rmax, int K);
int64_t run_scratch_floats(gpv_context *ctx, int rmax, int K, int *nslot);
const void *run_kernel(int order, int nt, int K, bool per_subset, bool kahan);
struct KArgs;
int run_launch(gpv_context *ctx, int order, int nt, int K, bool kahan, int blocks, size_t smem, cudaStream_t s,
               const KArgs &k, const int32_t *seg, int *queue, int win_cap, int nslot, uint32_t *slot_mask,
               int slots_per_sm, int n_mask);
// Run length of the run-layout kernel for subsets up to max_radius
// (GPV_RUN_K, else a candidate being timed, else the tuned choice, else 4).
int run_length_for(gpv_context *ctx, int max_radius);
int solve_noalloc_launch(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc_dev,
                         int64_t n, int max_radius, const gpv_solve_params *prm, gpv_subset_result *out_dev,
                         cudaStream_t s);
}  // namespace gpv
