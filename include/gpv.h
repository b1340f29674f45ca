/*
 * gpv.h -- C ABI of libgpv_b200, the B200 (sm_100a) subset-correlation
 * library: bi-quintic B-spline prefilter + batched ICGN subset solves.
 *
 * Each entry point replaces a call of the reference geopyv-dev crate (Rust)
 * on its hot path; the replaced interface is cited beside it (paths within
 * the geopyv-dev repository).  Plain C types only; every pointer is a host
 * pointer unless its name ends in `_dev`.  No entry point aborts: failures
 * return a negative gpv_err and leave a message for gpv_last_error().
 * Per-subset failures are reported in gpv_subset_result.status, never as
 * an API error (the reference returns Err / panics per subset instead).
 */
#ifndef GPV_H
#define GPV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPV_ABI_VERSION 1

/* ---- API return codes -------------------------------------------------- */
typedef enum {
    GPV_SUCCESS = 0,
    GPV_ERR_INVALID = -1,   /* bad argument (src/error.rs:5-40 InvalidInput) */
    GPV_ERR_CUDA = -2,      /* CUDA runtime error                            */
    GPV_ERR_NOMEM = -3,     /* device allocation failed / admission refused  */
    GPV_ERR_CANCELLED = -4, /* src/error.rs Cancelled (progress observer)    */
    GPV_ERR_TIMEOUT = -5,   /* bounded wait expired                          */
    GPV_ERR_NOT_FOUND = -6  /* unknown request id                            */
} gpv_err;

/* ---- per-subset status (gpv_subset_result.status) ---------------------- */
typedef enum {
    GPV_OK = 0,
    GPV_EMPTY_MASK = 1,       /* src/subset.rs:853-856  Err(InvalidInput)   */
    GPV_FEATURELESS = 2,      /* src/subset.rs:888-892  Err(InvalidInput)   */
    GPV_SINGULAR_H = 3,       /* src/subset.rs:1143     panic               */
    GPV_SINGULAR_WDELTA = 4,  /* src/subset.rs:520,595  panic               */
    GPV_NONFINITE = 5,        /* increment or norm not finite               */
    GPV_TIMEOUT = 6,
    GPV_CANCELLED = 7,
    GPV_INVALID_SUBSET = 8    /* order not in {0,1,2} or radius < 1         */
} gpv_status;

/* ---- pixel types ------------------------------------------------------- */
typedef enum { GPV_U8 = 1, GPV_U16 = 2, GPV_F32 = 3, GPV_F64 = 4 } gpv_dtype;

/* ---- precision of the solve -------------------------------------------- */
typedef enum {
    GPV_PREC_MIXED = 0, /* FP32 interpolation/warp/residual, FP64 reductions,
                           Hessian solve and warp composition; one thread block
                           per subset at a time                               */
    GPV_PREC_FP64 = 1   /* FP64 throughout, one subset per thread block      */
} gpv_precision;

/* gpv_solve_params.flags */
#define GPV_SOLVE_ETA 1u     /* omitted-mode diagnostic (src/subset.rs:748-820) */
#define GPV_SOLVE_HISTORY 2u /* per-iteration (norm, zncc, znssd) history       */
#define GPV_SOLVE_FAGN 4u    /* forward additive Gauss-Newton instead of ICGN
                                (solve_fagn_result, src/subset.rs:1228-1334);
                                FP64 arithmetic in either precision mode, on the
                                FP64 coefficients when precision is FP64     */
#define GPV_SOLVE_KAHAN 16u  /* mixed precision: accumulate the ZNSSD sums
                                (g - g_m, its square, the cross term with
                                f - f_m) per sample in Kahan-compensated FP64
                                instead of FP32 over each run of template
                                pixels (no counterpart in the reference: its
                                sums are plain FP64, src/subset.rs:418-446) */
#define GPV_SOLVE_RIGID_TEXTURE 8u /* Texture::Rigid (src/texture.rs,
                                src/subset.rs:1062-1097, 1151-1168): fit g to the
                                template f + G(E(p)) rebuilt every iteration
                                from the reference image's grain maps (f needs
                                them: GPV_IMAGE_GRAIN or gpv_image_build_grain);
                                orders 1 and 2; ICGN in both precisions and
                                FAGN (an image with FP64 coefficients keeps
                                the maps in FP64 too).  An
                                image without measurable speckle keeps the
                                deformable template (result texture = 0), as the
                                reference falls back.  The branch for known
                                soil grains (soil properties) is not part of
                                this library. */

/* gpv_image_create flags */
#define GPV_IMAGE_KEEP_F64 1u /* also keep FP64 coefficients (needed by GPV_PREC_FP64) */
#define GPV_IMAGE_GRAIN 2u    /* also keep the rigid-texture grain maps, rebuilt with every new set of pixels */

typedef struct gpv_context gpv_context;
typedef struct gpv_image gpv_image;
typedef struct gpv_mask gpv_mask;
typedef struct gpv_server gpv_server;
typedef struct gpv_sequence gpv_sequence;

/* One subset to solve (src/subset.rs:836-843 Subset::new arguments +
 * src/subset.rs:992-999 p_0).  Layout fixed: 120 bytes. */
typedef struct {
    double coord[2];  /* centre [x = column, y = row]                         */
    double p0[12];    /* initial warp; first 2/6/12 used (p_0 resize, :1134-1136) */
    int32_t order;    /* 0, 1 or 2 (src/subset.rs:16-20)                       */
    int32_t radius;   /* circular local mask radius (src/masks.rs:69-109)      */
} gpv_subset_desc;

/* Solver settings (src/subset.rs:992-999; python/src/py_subset.rs:217
 * defaults max_norm=1e-3, max_iterations=50, tolerance=0.75). */
typedef struct {
    double max_norm;
    double tolerance;
    int32_t max_iterations;
    int32_t flags;      /* GPV_SOLVE_* */
    int32_t precision;  /* gpv_precision */
    int32_t reserved;
    const gpv_mask *mask; /* global mask (src/masks.rs:199-263) or NULL */
    double *history;      /* host, n * max_iterations * 3 doubles, or NULL */
} gpv_solve_params;

/* SolveResult fields (src/subset.rs:145-191) + Subset scalars.  200 bytes.
 * texture: 1 when the solve fitted the rigid-texture template
 * (SolveResult::texture = Texture::Rigid), else 0. */
typedef struct {
    double p[12];
    double c_zncc, c_znssd, norm;
    double eta_u, eta_v;
    double f_m, delta_f, sssig, sigma;
    int32_t iterations, converged, quality_ok, status;
    int32_t n_px, has_eta;
    int32_t texture, reserved;
} gpv_subset_result;

/* ---- library ----------------------------------------------------------- */
const char *gpv_version(void);
int gpv_abi_version(void);
/* Copies the calling thread's last error message; returns its length. */
size_t gpv_last_error(char *buf, size_t len);

/* ---- context: one device, one stream, reusable workspace ---------------- */
int gpv_context_create(int device, gpv_context **out);
/* Context options (no counterpart in the reference):
 * GPV_CONTEXT_HIGH_PRIORITY: the context's streams run at the device's
 *   greatest stream priority, so its kernels' blocks are dispatched before
 *   pending blocks of ordinary streams as SMs free up;
 * GPV_CONTEXT_PER_SUBSET_BLOCKS: host-batch solves (gpv_solve_batch and the
 *   callers built on it) launch one thread block per subset instead of a
 *   persistent grid, so SMs free up at subset granularity while a large
 *   batch runs and other streams' work gets them; results are the same
 *   bytes as the persistent form. */
#define GPV_CONTEXT_HIGH_PRIORITY 1u
#define GPV_CONTEXT_PER_SUBSET_BLOCKS 2u
int gpv_context_create_ex(int device, uint32_t flags, gpv_context **out);
/* The context's resources are freed once gpv_context_destroy and the destroy
 * of every image and mask created on it have all run, in any order. */
int gpv_context_destroy(gpv_context *ctx);
/* The context's CUDA stream, as a cudaStream_t cast to void*. */
void *gpv_context_stream(gpv_context *ctx);
/* Pre-size the solve workspace so that later solves of up to n_subsets
 * subsets of radius <= max_radius allocate nothing (graph-capturable). */
int gpv_context_reserve(gpv_context *ctx, int64_t n_subsets, int32_t max_radius, int32_t max_iterations);

/* ---- image: device-resident coefficients --------------------------------
 * Replaces Image::from_array(image_gs, border) -> get_c
 * (src/image.rs:83-86, :252-327; python/src/py_image.rs:42-64).
 * px: host pixels (h, w) row-major of `dtype`; border >= 3 (default 20). */
int gpv_image_create(gpv_context *ctx, const void *px, int32_t dtype, int64_t h, int64_t w, int32_t border,
                     uint32_t flags, gpv_image **out);
/* Same, pixels already on the device (async on the context stream). */
int gpv_image_create_device(gpv_context *ctx, const void *px_dev, int32_t dtype, int64_t h, int64_t w,
                            int32_t border, uint32_t flags, gpv_image **out);
/* Re-prefilter new pixels of the same shape into an existing image
 * (sequence frames: src/sequence.rs:693-694,914), no allocation. */
int gpv_image_update_device(gpv_image *img, const void *px_dev, int32_t dtype);
/* Same from host pixels (copied through the image's staging buffer; fast
 * when px is page-locked).  Synchronous. */
int gpv_image_update(gpv_image *img, const void *px, int32_t dtype);
int gpv_image_destroy(gpv_image *img);
/* Rigid texture (GrainMaps::build, src/texture.rs:99-115, with the speckle
 * correlation length of src/seam.rs:255-301): builds the grain maps of an
 * image from its staged pixels (an image created or last updated from host
 * or colour pixels; device pixels need GPV_IMAGE_GRAIN at creation) and keeps
 * them up to date with later updates.  Asynchronous on the context stream. */
int gpv_image_build_grain(gpv_image *img);
/* The grain statistics (synchronises the context stream): out3 = correlation
 * length, s2, smoothing correction; *built = 0 when the image has no
 * measurable speckle; maps (host, 3 x h x w FP32: fxx, fyy, fxy) or NULL. */
int gpv_image_grain(gpv_image *img, double *out3, int32_t *built, float *maps);
/* The maps at n points (host xy, x = column, y = row): fxx, fyy, fxy per
 * point into out (host, 3n), bilinear and clamped as the solves sample them
 * (GrainMaps::sample, src/texture.rs:125-143).  Synchronous. */
int gpv_image_grain_sample(gpv_image *img, const double *xy, int64_t n, double *out);
int gpv_image_shape(const gpv_image *img, int64_t *h, int64_t *w, int32_t *border);
/* Download coefficients C (h+2b, w+2b) row-major: FP32 always, FP64 if kept. */
int gpv_image_coefficients_f32(const gpv_image *img, float *out);
int gpv_image_coefficients_f64(const gpv_image *img, double *out);
/* Value (+ gradient) of the spline at n points (x, y) -- Image::eval /
 * Image::eval_grad (src/image.rs:115-178), evaluated on the device in the
 * given precision.  grad may be NULL. */
int gpv_image_eval(const gpv_image *img, const double *xy, int64_t n, int32_t precision, double *val,
                   double *grad);

/* ---- colour ingest: Image::from_file's pre-processing --------------------
 * load_grayscale + gaussian_blur_5x5 (src/image.rs:450-534) on the device,
 * for decoded 8-bit RGB pixels (h, w, 3) row-major (file decoding itself is
 * not part of this library): the integer grey level
 * (2126 R + 7152 G + 722 B + 5000) / 10000, a 5 x 5 Gaussian blur
 * (sigma 1.1, BORDER_REFLECT_101), rounding and clamping to 0..255 -- bit for
 * bit the reference's grey image -- then the prefilter.  h, w >= 3. */
int gpv_image_create_rgb8(gpv_context *ctx, const uint8_t *rgb, int64_t h, int64_t w, int32_t border, uint32_t flags,
                          gpv_image **out);
int gpv_image_update_rgb8(gpv_image *img, const uint8_t *rgb);
/* Same from device pixels, asynchronous on the context stream. */
int gpv_image_update_rgb8_device(gpv_image *img, const uint8_t *rgb_dev);
/* The 8-bit greyscale pixels an RGB8 image was built from (h * w bytes). */
int gpv_image_grey(const gpv_image *img, uint8_t *out);

/* ---- global mask: LocalMask::mask_update (src/masks.rs:199-263) --------- */
int gpv_mask_create(gpv_context *ctx, const uint8_t *mask, int64_t h, int64_t w, gpv_mask **out);
int gpv_mask_destroy(gpv_mask *m);

/* ---- batched subset solve ----------------------------------------------
 * Replaces, per subset, Subset::new + Subset::solve_icgn_result
 * (src/subset.rs:836-919, :1117-1219) as called from
 * Mesh::solve_one_with_tolerance (src/mesh.rs:1025-1040) and
 * PySubset::solve_icgn (python/src/py_subset.rs:217-237).
 * Host arrays in and out; synchronous. */
int gpv_solve_batch(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc,
                    int64_t n, const gpv_solve_params *params, gpv_subset_result *out);
/* Device arrays in and out, asynchronous on `stream` (a cudaStream_t, or
 * NULL for the context stream).  work_order_dev (optional, int32[n]) is the
 * order in which subsets are taken from the work queue (largest first is
 * best); history (params->history) must then be a device pointer or NULL.
 * Allocates nothing once gpv_context_reserve covers the call. */
int gpv_solve_batch_device(gpv_context *ctx, const gpv_image *f, const gpv_image *g,
                           const gpv_subset_desc *desc_dev, const int32_t *work_order_dev, int64_t n,
                           const gpv_solve_params *params, gpv_subset_result *out_dev, void *stream);

/* ---- one device batch as a CUDA graph (no counterpart in the reference) --
 * Captures one gpv_solve_batch_device call (same arguments; runs it once
 * eagerly first, which sizes the context's workspace) as a CUDA graph:
 * the order partition and one persistent kernel per (order, radius class)
 * segment on the context's three streams.  A launch replays it on the
 * current contents of the images, descriptors and work order (same buffers:
 * update them in place), on `stream` (a cudaStream_t, or NULL for the
 * context stream), asynchronously.  The graph holds the context's workspace
 * addresses: a launch after another call on the context has moved them
 * (a larger batch or radius; reserve first) returns GPV_ERR_INVALID, and it
 * must not overlap other work of the same context.  History is not
 * supported. */
typedef struct gpv_batch_graph gpv_batch_graph;
int gpv_batch_graph_create(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc_dev,
                           const int32_t *work_order_dev, int64_t n, const gpv_solve_params *params,
                           gpv_subset_result *out_dev, gpv_batch_graph **out);
int gpv_batch_graph_launch(gpv_batch_graph *bg, void *stream);
int gpv_batch_graph_destroy(gpv_batch_graph *bg);

/* ---- batched subset solve without device allocation ---------------------
 * No counterpart in the reference: an extra entry point for callers that may
 * not allocate device memory on the solve path (their device memory belongs
 * to another framework's pool, or an allocation's implicit device-wide
 * synchronisation is not acceptable in their loop).  Same arguments and
 * results as gpv_solve_batch_device (mixed precision, device arrays, async
 * on `stream`), but all working memory comes from one static device array of
 * 64 MiB that every GPU loading this library holds until exit: subsets up to
 * radius 32 only (max_radius > 32 is rejected with GPV_ERR_INVALID; subsets
 * above max_radius get GPV_INVALID_SUBSET), no work-order array.  The first
 * call on a device performs a one-time set-up that synchronises `stream`, so
 * make it before any stream capture.  Calls share the array: calls that
 * overlap on the GPU race, so serialise them.  Allocates nothing. */
int gpv_solve_batch_noalloc(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc_dev,
                            int64_t n, int32_t max_radius, const gpv_solve_params *params,
                            gpv_subset_result *out_dev, void *stream);

/* ---- sequence: frame-to-frame tracking with device-resident seeds -------
 * The per-frame work of Sequence::solve (src/sequence.rs:624-968) for a
 * fixed set of subsets: each frame's target is re-prefiltered in place
 * (a1 again, :693-694, :914) and every subset is solved against the fixed
 * reference f with its initial warp taken from its own last converged
 * solution (desc p0 on the first frame).  Seeds and results stay on the
 * device; from the second frame on, the frame's device work (prefilter,
 * seeding, solve) is one CUDA graph replayed per frame, unless
 * GPV_SEQUENCE_NO_GRAPH is given or the image is narrower than 89 px.
 * f and g must outlive the sequence; g's coefficients are overwritten by
 * every frame. */
#define GPV_SEQUENCE_NO_GRAPH 1u
int gpv_sequence_create(gpv_context *ctx, const gpv_image *f, gpv_image *g, const gpv_subset_desc *desc, int64_t n,
                        const gpv_solve_params *params, int32_t dtype, uint32_t flags, gpv_sequence **out);
/* One frame: px (h x w of the sequence's dtype) on the host, or on the
 * device when px_on_device != 0.  out (host, n results) may be NULL: the
 * frame then stays asynchronous on the context stream and its results are
 * at gpv_sequence_results_device() until the next frame. */
int gpv_sequence_frame(gpv_sequence *s, const void *px, int32_t px_on_device, gpv_subset_result *out);
gpv_subset_result *gpv_sequence_results_device(gpv_sequence *s);
int64_t gpv_sequence_frames(const gpv_sequence *s);
int gpv_sequence_destroy(gpv_sequence *s);

/* ---- mesh driver: reliability-guided propagation -------------------------
 * Replaces the propagation stage of Mesh::solve_impl (src/mesh.rs:628-764):
 * the seed node (find_seed_node :1682-1690, the forced seed warp and the seed
 * tolerance, :667-677), then either the serial RG cascade
 * (Preconditioning::Rg, :683-705, solve_neighbours_from :1112-1154) or the
 * epsilon-band layer-RG rounds (Preconditioning::LayerRg, :706-764) whose
 * graph colours (expand_parallel :1169-1252, greedy_graph_colour :1884-1903)
 * are solved as one batch each.  Per node: the two attempts of solve_node
 * (:1068-1106) -- the preconditioned warp of precondition_warp
 * (:2130-2233), then the zero warp for the nodes that missed quality_ok --
 * folded in ascending node order by store_result (:2385-2402).  The
 * corrections stage (:766-790), element strains and the quality gate's
 * error (:792-799) stay with the caller; gpv_mesh_stats.n_bad is the count
 * that gate tests.  Every node's result (or, for a node the propagation
 * never reaches, a zeroed result with status GPV_INVALID_SUBSET and round
 * -1) is written to out[i]; rounds[i] (optional) is the batch round that
 * solved node i: nodes of one round never share an element. */

/* Progress observer (src/progress.rs:17-38): called after every stored
 * node; a nonzero return cancels the solve with GPV_ERR_CANCELLED. */
typedef int (*gpv_progress_fn)(void *user, int64_t done, int64_t total);

/* Batch solver used by gpv_mesh_drive: solve n subsets at `tolerance`
 * (the seed node uses the seed tolerance); returns a gpv_err. */
typedef int (*gpv_batch_solver_fn)(void *user, const gpv_subset_desc *desc, int64_t n, double tolerance,
                                   gpv_subset_result *out);

/* SolveConfig + SeedConfig + LayerRgConfig (src/mesh.rs:222-262, :339-356;
 * python/src/py_mesh.rs:215-225 defaults in brackets).  208 bytes. */
typedef struct {
    double seed_coord[2];
    double seed_warp[12];     /* first 6 * subset_order used          [0]    */
    double seed_tolerance;    /*                                      [0.9]  */
    double max_norm;          /*                                      [1e-5] */
    double tolerance;         /*                                      [0.75] */
    double root_rel_eps;      /* layer-RG epsilon band                [0.02] */
    int32_t max_iterations;   /*                                      [50]   */
    int32_t subset_order;     /* 1 or 2 (mesh p_len = 6 * order, :636)       */
    int32_t radius;           /* circular local mask radius                  */
    int32_t precision;        /* gpv_precision (gpv_mesh_solve only)          */
    int32_t layer_rg;         /* 0 = "RG", 1 = "layer-RG"             [0]    */
    int32_t batch_factor;     /* layer-RG roots per round / worker    [4]    */
    int32_t max_workers;      /* the worker count rounds are sized by (the
                                 reference's rayon pool size), >= 1          */
    int32_t method;           /* 0 = ICGN, 1 = FAGN (SolveMethod, :284-288)  */
    int32_t texture;          /* 0 = deformable, 1 = rigid (Texture, :317-330;
                                 gpv_mesh_solve: GPV_SOLVE_RIGID_TEXTURE)    */
    int32_t reserved;
    const gpv_mask *mask;     /* global mask or NULL (gpv_mesh_solve only)   */
    gpv_progress_fn progress; /* or NULL */
    void *progress_user;
} gpv_mesh_params;

typedef struct {
    int64_t n_bad;       /* nodes without quality_ok (unreached included)   */
    int64_t n_unreached; /* nodes the propagation never reached              */
    int64_t batches;     /* solver calls                                     */
    int64_t solves;      /* subset solves, zero-warp retries included        */
    int64_t retries;     /* zero-warp second attempts                        */
    int64_t rounds;      /* fold rounds                                      */
    int64_t seed_node;
} gpv_mesh_stats;

/* The mesh driver on this library's GPU batch solve (gpv_solve_batch on
 * ctx with params->precision / mask / max_norm / max_iterations).
 * nodes: n_nodes x 2 (x, y); elements: n_elements x nodes_per_element
 * (3 or 6) node indices.  Synchronous; host arrays. */
int gpv_mesh_solve(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const double *nodes, int64_t n_nodes,
                   const int64_t *elements, int64_t n_elements, int32_t nodes_per_element,
                   const gpv_mesh_params *params, gpv_subset_result *out, int32_t *rounds, gpv_mesh_stats *stats);
/* The same driver over any batch solver (no device work of its own). */
int gpv_mesh_drive(const double *nodes, int64_t n_nodes, const int64_t *elements, int64_t n_elements,
                   int32_t nodes_per_element, const gpv_mesh_params *params, gpv_batch_solver_fn solver,
                   void *solver_user, gpv_subset_result *out, int32_t *rounds, gpv_mesh_stats *stats);

/* ---- serving: a request loop (no single counterpart in the reference) ----
 * Requests -- an image pair, subsets, solver settings -- are submitted from
 * any host thread and served by `workers` worker threads, each with its own
 * context (CUDA stream and solve workspace) on `device`, so several requests
 * are on the GPU at once.  Admission is by device-memory footprint against
 * `hbm_budget` bytes (0 = 80% of the memory free at creation): requests start
 * in arrival order when they fit; a request that does not fit is overtaken
 * by later ones that do (at most 8 times); one larger than the whole budget
 * runs alone.  With a priority lane (priority_workers > 0) small requests
 * and large ones are served by separate workers, the small ones on
 * high-priority streams.  A session (nonzero `session`) is served by one worker, in
 * order, and keeps its reference coefficients and its last results on that
 * worker: GPV_REQUEST_REUSE_REFERENCE skips the reference upload and
 * prefilter (f_px may then be NULL), GPV_REQUEST_SEED_FROM_PREVIOUS starts
 * every subset from its last converged warp (same subset count), as a
 * sequence's frame loop does (src/sequence.rs:624-968).  Host buffers
 * (pixels, desc, out) must stay valid until gpv_server_wait returns; desc is
 * copied at submit. */
#define GPV_REQUEST_REUSE_REFERENCE 1u
#define GPV_REQUEST_SEED_FROM_PREVIOUS 2u

typedef struct {
    const void *f_px;   /* reference pixels, host, h x w of dtype (or NULL, see above) */
    const void *g_px;   /* target pixels, host                                     */
    int32_t dtype;      /* gpv_dtype                                               */
    int32_t border;     /* >= 3 (20 as Image::from_array's default)                */
    int64_t h, w;
    const gpv_subset_desc *desc;
    int64_t n;
    gpv_solve_params params;  /* mixed precision; no mask, no history           */
    uint64_t session;         /* 0 = none                                        */
    uint32_t flags;           /* GPV_REQUEST_*                                   */
    uint32_t reserved;
    gpv_subset_result *out;   /* host, n results, written before completion     */
} gpv_request;

/* Executes one request on worker `worker` (desc is the server's copy,
 * already seeded); returns a gpv_err.  NULL = the GPU solve of this library
 * (a stand-in lets the request loop itself be exercised without a GPU). */
typedef int (*gpv_request_executor_fn)(void *user, int32_t worker, const gpv_request *req, gpv_subset_desc *desc,
                                       gpv_subset_result *out);

typedef struct {
    size_t hbm_budget;   /* bytes; 0 = 80% of free device memory */
    int32_t workers;     /* 1..64 */
    int32_t device;
    gpv_request_executor_fn executor;  /* NULL = GPU */
    void *executor_user;
    int64_t reserve_subsets;  /* size each worker's workspace for this many subsets */
    int32_t reserve_radius;   /* of up to this radius (0, 0 = grow on demand)       */
    /* Priority lane (0 = off): workers 0..priority_workers-1 run on
     * high-priority streams and take the requests of at most
     * priority_subsets subsets; the other workers take the larger ones, and
     * every worker solves with one thread block per subset, so a small
     * request's blocks get SMs as soon as subsets of the large ones finish
     * instead of after their whole batch.  Session requests stay on their
     * session's worker whatever their size. */
    int32_t priority_workers;
    int64_t priority_subsets;
} gpv_server_config;

typedef struct {
    int64_t submitted, completed, failed, queued, in_flight, subsets;
    double p50_ms, p99_ms, mean_ms, max_ms;  /* submit -> results in host memory */
    double mean_queue_ms, mean_service_ms;   /* submit -> start, start -> done */
    double subsets_per_s;                    /* completed subsets / (last done - first submit) */
    size_t bytes_in_flight, peak_bytes, hbm_budget;
} gpv_server_stats;

int gpv_server_create(const gpv_server_config *cfg, gpv_server **out);
int gpv_server_submit(gpv_server *s, const gpv_request *req, uint64_t *id);
/* Creates (or grows) every worker's cached image pair for requests of shape
 * h x w, `border` and pixel type `dtype`, waiting up to timeout_ms per
 * worker, so that serving such requests allocates no device memory (an
 * allocation or free on the request path can stall every stream of the
 * device).  Not counted in the statistics. */
int gpv_server_prepare(gpv_server *s, int64_t h, int64_t w, int32_t border, int32_t dtype, int32_t timeout_ms);
/* Waits up to timeout_ms for request `id`: GPV_ERR_TIMEOUT if unfinished,
 * GPV_ERR_NOT_FOUND for an unknown or already collected id; otherwise
 * GPV_SUCCESS with the request's own gpv_err in *req_status. */
int gpv_server_wait(gpv_server *s, uint64_t id, int32_t timeout_ms, int32_t *req_status, double *latency_ms);
int gpv_server_get_stats(gpv_server *s, gpv_server_stats *out);
int gpv_server_reset_stats(gpv_server *s);
/* Serves what is queued, then stops the workers and frees every resource. */
int gpv_server_destroy(gpv_server *s);

/* ---- autotuning (no counterpart in the reference) ------------------------
 * Times the candidate launch shapes of the mixed-precision kernel (threads
 * per subset block: 64, 128 or 256; template pixels per run of the
 * run-layout kernel: 4 or 8 -- or, with GPV_SOLVE_KERNEL=tile, 128 or 256
 * threads and the tiled kernel's
 * template layout: compact scan order or 8 x 4 tiles) on a sample of up to
 * sample_per_class subsets of each radius class
 * (r <= 20, 21..40, > 40) present in desc, keeps the fastest per class in the
 * context, and returns the thread choices in threads_out[3] (0 = class
 * absent).  If the environment variable GPV_TUNE_CACHE names a file, the
 * choices are appended to it keyed by device name, and gpv_context_create
 * reads them back. */
int gpv_autotune(gpv_context *ctx, const gpv_image *f, const gpv_image *g, const gpv_subset_desc *desc, int64_t n,
                 const gpv_solve_params *params, int32_t sample_per_class, int32_t *threads_out);
/* The context's tuned choices per radius class: threads (0 = none) and
 * layout (-1 = none, 0 compact, 1 padded rows, 2 tiles); either may be NULL. */
int gpv_context_tuning(gpv_context *ctx, int32_t *threads, int32_t *layouts);

/* Every tuned launch dimension of one radius class (no counterpart in the
 * reference).  0 / -1 = not tuned (the default applies). */
typedef struct {
    int32_t threads;            /* threads per block: 64, 128 or 256                    */
    int32_t layout;             /* tiled kernel's template layout (-1, 0, 1, 2)         */
    int32_t run_length;         /* run-layout kernel: template pixels per run, 4 or 8   */
    int32_t subsets_per_block;  /* subsets a block solves side by side (1 or 2)         */
    int32_t staging;            /* coefficient-window buffers per subset (1 or 2)       */
    int32_t reserved;
} gpv_tuning;

/* The context's tuning for radius classes r <= 20, 21-40, > 40 (out[3]). */
int gpv_context_tuning_get(gpv_context *ctx, gpv_tuning *out);

/* ---- calibration (no counterpart in the reference) ----------------------
 * Measured FP32 FMA throughput of this device (TFLOP/s, 2 FLOP per FMA) from
 * a register-only FMA kernel: the denominator of the interpolation roofline. */
int gpv_probe_fp32_peak(gpv_context *ctx, double *tflops);

/* Measured throughputs of this device (no reference counterpart: the
 * denominators of the solve's rooflines).  FP32 FMA as scalar FFMA chains
 * and as sm_100 paired FFMA2 chains (gpv_probe_fp32_peak reports the larger),
 * FP64 DFMA, and shared-memory read bandwidth over all SMs (conflict-free
 * 16-byte loads).  TFLOP/s count 2 FLOP per FMA. */
typedef struct {
    double fp32_scalar_tflops;
    double fp32_paired_tflops;
    double fp64_tflops;
    double smem_gbs;
    int32_t sm_count;
    int32_t reserved;
} gpv_peaks;

int gpv_probe_peaks(gpv_context *ctx, gpv_peaks *out);

#ifdef __cplusplus
}
#endif
#endif /* GPV_H */
