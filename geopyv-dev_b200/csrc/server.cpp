// server.cpp -- request loop for subset-correlation requests.
//
// Requests (an image pair, a set of subsets, solver settings) arrive from any
// host thread and are served by a pool of workers, each owning one library
// context (its own CUDA stream and solve workspace) on the same GPU, so that
// several requests are in flight on the device at once and a small request
// never waits for a large one to finish.  Admission is by device-memory
// footprint: a request starts only when its estimated footprint fits in the
// budget next to the requests already running (taken in arrival order, a
// request that does not fit is overtaken by later ones that do, for at most
// kMaxBypass admissions; one that exceeds the whole budget runs alone).
// Sessions keep a reference image's coefficients and the last results
// resident on their worker: later requests of the session can skip the
// reference upload and prefilter and seed every subset from its previous
// converged warp, as the frame loop of a sequence does (src/sequence.rs:
// 624-968).  With a priority lane, the first priority_workers workers own
// high-priority contexts and serve only requests of up to priority_subsets
// subsets, the others serve the larger ones, and all of them solve with one
// thread block per subset: a large batch then holds each SM slot for one
// subset at a time, and the block scheduler hands freed slots to the
// pending blocks of the high-priority streams first.  Every wait in this
// file is bounded.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "internal.h"

namespace gpv {
namespace {

using Clock = std::chrono::steady_clock;
constexpr int kMaxBypass = 8;

struct Request {
    uint64_t id = 0;
    gpv_request r{};
    std::vector<gpv_subset_desc> desc;  // copied at submit; seeded at start
    size_t footprint = 0;
    int worker = -1;  // session affinity, -1 = any
    int bypassed = 0;
    bool prepare = false;  // gpv_server_prepare: create the worker's image pair for (h, w, border, dtype)
    Clock::time_point t_submit, t_start, t_done;
    bool done = false;
    int status = GPV_SUCCESS;
    std::string error;
};

struct Session {
    gpv_image *f = nullptr;  // resident reference coefficients
    int64_t h = 0, w = 0;
    int32_t border = 0;
    std::vector<gpv_subset_result> last;  // last results (host)
};

struct Worker {
    int index = 0;
    gpv_context *ctx = nullptr;
    // reusable image pairs keyed by (h, w, border)
    std::map<std::tuple<int64_t, int64_t, int32_t>, std::pair<gpv_image *, gpv_image *>> images;
    std::unordered_map<uint64_t, Session> sessions;
    std::thread th;
};

size_t estimate_footprint(const gpv_request &r) {
    const size_t ch = (size_t)(r.h + 2 * r.border), cw = (size_t)(r.w + 2 * r.border);
    const size_t pitch = (cw + 31) / 32 * 32;
    const size_t esz = r.dtype == GPV_U8 ? 1 : r.dtype == GPV_U16 ? 2 : r.dtype == GPV_F32 ? 4 : 8;
    const size_t coef = 2 * sizeof(float) * pitch * ch;             // f and g coefficients
    const size_t rowpass = 2 * prefilter_rowpass_bytes(r.h, (int64_t)cw, (int64_t)ch);  // short-line images only
    const size_t pixels = 2 * esz * (size_t)r.h * (size_t)r.w;       // staged pixels
    const size_t subsets = (size_t)r.n * (sizeof(gpv_subset_desc) + sizeof(gpv_subset_result) + 4);
    return coef + rowpass + pixels + subsets;
}

}  // namespace
}  // namespace gpv

using namespace gpv;

struct gpv_server {
    gpv_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> reqs;
    std::vector<std::unique_ptr<Worker>> workers;
    uint64_t next_id = 1;
    bool stopping = false;
    size_t bytes_in_flight = 0, peak_bytes = 0;
    int64_t submitted = 0, completed = 0, failed = 0, in_flight = 0, subsets_done = 0;
    std::vector<double> latencies_ms;
    double queue_ms_sum = 0.0, service_ms_sum = 0.0;
    Clock::time_point t_first, t_last;
    bool any_done = false;
};

namespace {

int default_execute(gpv_server *S, Worker &W, Request &q, gpv_subset_result *out) {
    const gpv_request &r = q.r;
    gpv_context *ctx = W.ctx;
    Session *sess = nullptr;
    if (r.session) sess = &W.sessions[r.session];
    // target (and, unless resident, reference) images
    auto key = std::make_tuple(r.h, r.w, r.border);
    auto &pair = W.images[key];
    if (!pair.second) {
        if (int rc = gpv_image_create(ctx, r.g_px, r.dtype, r.h, r.w, r.border, 0, &pair.second)) return rc;
    } else if (int rc = gpv_image_update(pair.second, r.g_px, r.dtype)) {
        return rc;
    }
    gpv_image *F = nullptr;
    const bool reuse = (r.flags & GPV_REQUEST_REUSE_REFERENCE) && sess && sess->f && sess->h == r.h &&
                       sess->w == r.w && sess->border == r.border;
    if (reuse) {
        F = sess->f;
    } else if (sess) {
        if (!r.f_px) { set_error("request without reference pixels and no resident reference"); return GPV_ERR_INVALID; }
        if (sess->f && (sess->h != r.h || sess->w != r.w || sess->border != r.border)) {
            gpv_image_destroy(sess->f);
            sess->f = nullptr;
        }
        if (!sess->f) {
            if (int rc = gpv_image_create(ctx, r.f_px, r.dtype, r.h, r.w, r.border, 0, &sess->f)) return rc;
        } else if (int rc = gpv_image_update(sess->f, r.f_px, r.dtype)) {
            return rc;
        }
        sess->h = r.h;
        sess->w = r.w;
        sess->border = r.border;
        F = sess->f;
    } else {
        if (!r.f_px) { set_error("request without reference pixels"); return GPV_ERR_INVALID; }
        if (!pair.first) {
            if (int rc = gpv_image_create(ctx, r.f_px, r.dtype, r.h, r.w, r.border, 0, &pair.first)) return rc;
        } else if (int rc = gpv_image_update(pair.first, r.f_px, r.dtype)) {
            return rc;
        }
        F = pair.first;
    }
    // the rigid texture reads the reference's grain maps: built on the first
    // such request (an allocation), then kept up to date with every upload
    if ((r.params.flags & GPV_SOLVE_RIGID_TEXTURE) && !F->grain)
        if (int rc = gpv_image_build_grain(F)) return rc;
    // seeds from the session's previous converged warps
    if (sess && (r.flags & GPV_REQUEST_SEED_FROM_PREVIOUS) && (int64_t)sess->last.size() == r.n) {
        for (int64_t i = 0; i < r.n; i++) {
            const gpv_subset_result &p = sess->last[i];
            if (p.status == GPV_OK && p.converged) std::memcpy(q.desc[i].p0, p.p, sizeof(p.p));
        }
    }
    if (int rc = gpv_solve_batch(ctx, F, pair.second, q.desc.data(), r.n, &r.params, out)) return rc;
    if (sess) sess->last.assign(out, out + r.n);
    (void)S;
    return GPV_SUCCESS;
}

// Whether worker W may take request c: its session's worker only; with a
// priority lane, small requests go to the priority workers and large ones
// to the others.
bool eligible(const gpv_server *S, const Worker *W, const Request &c) {
    if (c.worker >= 0) return c.worker == W->index;
    if (S->cfg.priority_workers <= 0) return true;
    const bool small = c.r.n <= S->cfg.priority_subsets;
    return (W->index < S->cfg.priority_workers) == small;
}

// Create (or grow) the worker's cached image pair for the request's shape
// and pixel type, so that requests of that shape allocate nothing.
int prepare_images(Worker &W, const gpv_request &r) {
    const size_t esz = r.dtype == GPV_U8 ? 1 : r.dtype == GPV_U16 ? 2 : r.dtype == GPV_F32 ? 4 : 8;
    std::vector<uint8_t> zeros(esz * (size_t)r.h * (size_t)r.w, 0);
    auto &pair = W.images[std::make_tuple(r.h, r.w, r.border)];
    for (gpv_image **img : {&pair.first, &pair.second}) {
        if (!*img) {
            if (int rc = gpv_image_create(W.ctx, zeros.data(), r.dtype, r.h, r.w, r.border, 0, img)) return rc;
        } else if (int rc = gpv_image_update(*img, zeros.data(), r.dtype)) {
            return rc;
        }
    }
    GPV_CUDA_TRY(cudaStreamSynchronize(W.ctx->stream));
    return GPV_SUCCESS;
}

void worker_loop(gpv_server *S, Worker *W) {
    for (;;) {
        std::shared_ptr<Request> q;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            for (;;) {
                if (S->stopping && S->queue.empty()) return;
                // first request in arrival order that is ours and fits
                auto pick = S->queue.end();
                for (auto it = S->queue.begin(); it != S->queue.end(); ++it) {
                    Request &c = **it;
                    if (!eligible(S, W, c)) continue;
                    const bool fits = S->bytes_in_flight + c.footprint <= S->cfg.hbm_budget ||
                                      S->bytes_in_flight == 0;
                    if (fits) {
                        pick = it;
                        break;
                    }
                    if (c.bypassed >= kMaxBypass) break;  // no more overtaking this one
                }
                if (pick != S->queue.end()) {
                    for (auto it = S->queue.begin(); it != pick; ++it)
                        if (eligible(S, W, **it)) (*it)->bypassed++;
                    q = *pick;
                    S->queue.erase(pick);
                    S->bytes_in_flight += q->footprint;
                    S->peak_bytes = std::max(S->peak_bytes, S->bytes_in_flight);
                    S->in_flight++;
                    break;
                }
                S->cv_work.wait_for(lk, std::chrono::milliseconds(50));
            }
        }
        q->t_start = Clock::now();
        std::vector<gpv_subset_result> tmp;
        gpv_subset_result *out = q->r.out;
        if (!out) {
            tmp.resize(q->r.n);
            out = tmp.data();
        }
        int rc;
        std::string err;
        if (q->prepare) {
            rc = S->cfg.executor ? GPV_SUCCESS : prepare_images(*W, q->r);
        } else if (S->cfg.executor) {
            rc = S->cfg.executor(S->cfg.executor_user, W->index, &q->r, q->desc.data(), out);
        } else {
            rc = default_execute(S, *W, *q, out);
        }
        if (rc) {
            char buf[512];
            gpv_last_error(buf, sizeof buf);
            err = buf;
        }
        {
            std::lock_guard<std::mutex> lk(S->mu);
            q->t_done = Clock::now();
            q->status = rc;
            q->error = err;
            q->done = true;
            S->bytes_in_flight -= q->footprint;
            S->in_flight--;
            if (q->prepare) {
                // not a served request: no statistics
            } else if (rc) {
                S->failed++;
            } else {
                S->completed++;
                S->subsets_done += q->r.n;
                S->latencies_ms.push_back(std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count());
                S->queue_ms_sum += std::chrono::duration<double, std::milli>(q->t_start - q->t_submit).count();
                S->service_ms_sum += std::chrono::duration<double, std::milli>(q->t_done - q->t_start).count();
                if (!S->any_done) S->t_first = q->t_submit;
                S->any_done = true;
                S->t_last = q->t_done;
            }
        }
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

void release_worker(Worker &W) {
    for (auto &kv : W.sessions)
        if (kv.second.f) gpv_image_destroy(kv.second.f);
    for (auto &kv : W.images) {
        if (kv.second.first) gpv_image_destroy(kv.second.first);
        if (kv.second.second) gpv_image_destroy(kv.second.second);
    }
    W.sessions.clear();
    W.images.clear();
    if (W.ctx) gpv_context_destroy(W.ctx);
    W.ctx = nullptr;
}

}  // namespace

extern "C" {

int gpv_server_create(const gpv_server_config *cfg, gpv_server **out) {
    if (!cfg || !out || cfg->workers < 1 || cfg->workers > 64) {
        set_error("invalid server configuration (1..64 workers)");
        return GPV_ERR_INVALID;
    }
    if (cfg->priority_workers < 0 || (cfg->priority_workers > 0 && cfg->priority_workers >= cfg->workers) ||
        (cfg->priority_workers > 0 && cfg->priority_subsets < 1)) {
        set_error("a priority lane needs 1..workers-1 priority workers and priority_subsets >= 1");
        return GPV_ERR_INVALID;
    }
    *out = nullptr;
    auto *S = new gpv_server();
    S->cfg = *cfg;
    if (S->cfg.hbm_budget == 0) {
        size_t free_b = 0, total_b = 0;
        if (!cfg->executor && cudaSetDevice(cfg->device) == cudaSuccess && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
            S->cfg.hbm_budget = free_b / 10 * 8;  // 80% of what is free now
        else
            S->cfg.hbm_budget = (size_t)1 << 34;
    }
    for (int k = 0; k < cfg->workers; k++) {
        auto W = std::make_unique<Worker>();
        W->index = k;
        if (!cfg->executor) {
            uint32_t flags = 0;
            if (cfg->priority_workers > 0)
                flags = GPV_CONTEXT_PER_SUBSET_BLOCKS | (k < cfg->priority_workers ? GPV_CONTEXT_HIGH_PRIORITY : 0u);
            int rc = gpv_context_create_ex(cfg->device, flags, &W->ctx);
            // sized once here, the workspace never grows (nor frees) while serving
            if (!rc && cfg->reserve_subsets > 0 && cfg->reserve_radius > 0)
                rc = gpv_context_reserve(W->ctx, cfg->reserve_subsets, cfg->reserve_radius, 50);
            if (rc) {
                S->workers.push_back(std::move(W));
                for (auto &w : S->workers) release_worker(*w);
                delete S;
                return rc;
            }
        }
        S->workers.push_back(std::move(W));
    }
    for (auto &W : S->workers) W->th = std::thread(worker_loop, S, W.get());
    *out = S;
    return GPV_SUCCESS;
}

int gpv_server_submit(gpv_server *S, const gpv_request *r, uint64_t *id) {
    if (!S || !r || !id) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    if (r->n < 1 || !r->desc || !r->g_px || r->h < 1 || r->w < 1 || r->border < 3) {
        set_error("request needs subsets, target pixels, a positive shape and border >= 3");
        return GPV_ERR_INVALID;
    }
    if (r->dtype != GPV_U8 && r->dtype != GPV_U16 && r->dtype != GPV_F32 && r->dtype != GPV_F64) {
        set_error("unknown pixel dtype");
        return GPV_ERR_INVALID;
    }
    if (r->params.history || r->params.mask || r->params.precision != GPV_PREC_MIXED) {
        set_error("served requests use the mixed-precision solve without history or global mask");
        return GPV_ERR_INVALID;
    }
    if (!r->session && (r->flags & (GPV_REQUEST_REUSE_REFERENCE | GPV_REQUEST_SEED_FROM_PREVIOUS))) {
        set_error("reference reuse and seeding need a session");
        return GPV_ERR_INVALID;
    }
    auto q = std::make_shared<Request>();
    q->r = *r;
    q->desc.assign(r->desc, r->desc + r->n);
    q->r.desc = nullptr;  // the copy above is used
    q->footprint = estimate_footprint(*r);
    q->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping) { set_error("server is shutting down"); return GPV_ERR_INVALID; }
        q->id = S->next_id++;
        q->worker = r->session ? (int)(r->session % (uint64_t)S->workers.size()) : -1;
        S->reqs[q->id] = q;
        S->queue.push_back(q);
        S->submitted++;
        *id = q->id;
    }
    S->cv_work.notify_all();
    return GPV_SUCCESS;
}

int gpv_server_prepare(gpv_server *S, int64_t h, int64_t w, int32_t border, int32_t dtype, int32_t timeout_ms) {
    if (!S) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    if (h < 1 || w < 1 || border < 3) { set_error("prepare needs a positive shape and border >= 3"); return GPV_ERR_INVALID; }
    if (dtype != GPV_U8 && dtype != GPV_U16 && dtype != GPV_F32 && dtype != GPV_F64) {
        set_error("unknown pixel dtype");
        return GPV_ERR_INVALID;
    }
    std::vector<uint64_t> ids;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping) { set_error("server is shutting down"); return GPV_ERR_INVALID; }
        for (size_t k = 0; k < S->workers.size(); k++) {
            auto q = std::make_shared<Request>();
            q->prepare = true;
            q->r.h = h;
            q->r.w = w;
            q->r.border = border;
            q->r.dtype = dtype;
            q->worker = (int)k;
            q->t_submit = Clock::now();
            q->id = S->next_id++;
            S->reqs[q->id] = q;
            S->queue.push_back(q);
            ids.push_back(q->id);
        }
    }
    S->cv_work.notify_all();
    int first_rc = GPV_SUCCESS;
    std::string first_err;
    for (uint64_t id : ids) {
        int32_t st = 0;
        int rc = gpv_server_wait(S, id, timeout_ms, &st, nullptr);
        if (!rc && st) rc = st;
        if (rc && !first_rc) {
            first_rc = rc;
            char buf[512];
            gpv_last_error(buf, sizeof buf);
            first_err = buf;
        }
    }
    if (first_rc) set_error(first_err);
    return first_rc;
}

int gpv_server_wait(gpv_server *S, uint64_t id, int32_t timeout_ms, int32_t *req_status, double *latency_ms) {
    if (!S) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) { set_error("unknown request id"); return GPV_ERR_NOT_FOUND; }
    auto q = it->second;
    const auto deadline = Clock::now() + std::chrono::milliseconds(std::max(0, timeout_ms));
    while (!q->done) {
        if (S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !q->done) {
            set_error("request not finished within the timeout");
            return GPV_ERR_TIMEOUT;
        }
    }
    if (req_status) *req_status = q->status;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count();
    S->reqs.erase(id);  // results are in the caller's buffer; the id is spent
    if (q->status) set_error(q->error);
    return GPV_SUCCESS;
}

int gpv_server_get_stats(gpv_server *S, gpv_server_stats *st) {
    if (!S || !st) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    std::lock_guard<std::mutex> lk(S->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = S->submitted;
    st->completed = S->completed;
    st->failed = S->failed;
    st->queued = (int64_t)S->queue.size();
    st->in_flight = S->in_flight;
    st->subsets = S->subsets_done;
    st->bytes_in_flight = S->bytes_in_flight;
    st->peak_bytes = S->peak_bytes;
    st->hbm_budget = S->cfg.hbm_budget;
    if (!S->latencies_ms.empty()) {
        std::vector<double> v = S->latencies_ms;
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) {
            const double x = p * (double)(v.size() - 1);
            const size_t i = (size_t)x;
            const double f = x - (double)i;
            return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
        };
        st->p50_ms = pct(0.50);
        st->p99_ms = pct(0.99);
        st->max_ms = v.back();
        double s = 0.0;
        for (double x : v) s += x;
        st->mean_ms = s / (double)v.size();
        st->mean_queue_ms = S->queue_ms_sum / (double)v.size();
        st->mean_service_ms = S->service_ms_sum / (double)v.size();
        const double span = std::chrono::duration<double>(S->t_last - S->t_first).count();
        st->subsets_per_s = span > 0 ? (double)S->subsets_done / span : 0.0;
    }
    return GPV_SUCCESS;
}

int gpv_server_reset_stats(gpv_server *S) {
    if (!S) { set_error("NULL argument"); return GPV_ERR_INVALID; }
    std::lock_guard<std::mutex> lk(S->mu);
    S->latencies_ms.clear();
    S->queue_ms_sum = S->service_ms_sum = 0.0;
    S->completed = S->failed = S->subsets_done = 0;
    S->submitted = (int64_t)S->queue.size() + S->in_flight;
    S->peak_bytes = S->bytes_in_flight;
    S->any_done = false;
    return GPV_SUCCESS;
}

int gpv_server_destroy(gpv_server *S) {
    if (!S) return GPV_SUCCESS;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv_work.notify_all();
    for (auto &W : S->workers)
        if (W->th.joinable()) W->th.join();
    for (auto &W : S->workers) release_worker(*W);
    delete S;
    return GPV_SUCCESS;
}

}  // extern "C"
