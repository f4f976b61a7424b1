// Serving loop: many independent solve+Grad requests on one GPU.
//
// Requests (problem, densities, load) are queued by tosp_server_submit.  A
// dispatcher admits them in arrival order whenever a slot is free and the
// request's device memory fits the HBM budget (continuous admission: a request
// that arrives while others run starts as soon as a slot and memory free up).
// Each slot is a worker thread driving a solve handle on its own CUDA stream,
// so the kernels of concurrent requests overlap on the device; every handle
// replays its CG iteration as a captured CUDA graph.  Handles are cached per
// problem shape and reused by later requests of the same shape (hierarchy
// buffers, captured graph), and evicted when another shape needs the memory.
#include <algorithm>
#include <cmath>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "tosp_internal.h"
#include "trace.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    // problem (deep copy)
    tosp_problem pb{};
    std::vector<int64_t> freedofs, fixed_dens, free_dens_g;
    tosp_mg_params mg{};
    int32_t precision = TOSP_PREC_MIXED;
    std::vector<double> xfil, f;
    std::vector<double> u0;        // warm start (FP64 re-run after a stalled mixed solve)
    int fallbacks = 0;
    // results
    std::vector<double> u, g;
    tosp_request_stats st{};
    int state = TOSP_REQ_QUEUED;
    int status = TOSP_OK;
    std::string err;
    Clock::time_point t_submit, t_start;
    int64_t est_bytes = 0;
    std::string key;
    // in flight
    tosp_handle *h = nullptr;
    std::vector<double> x;         // iterate on the free dofs (host)
    bool solve_failed = false;     // setup or an iteration failed: no final update
};

struct CachedHandle {
    tosp_handle *h = nullptr;
    std::string key;
    int64_t bytes = 0;
    bool busy = false;
    Clock::time_point last_used;
};

std::string shape_key(const Request &r) {
    // everything that fixes a handle's buffers and hierarchy
    std::string k;
    auto add = [&](const void *p, size_t n) { k.append(static_cast<const char *>(p), n); };
    add(&r.pb.nelx, sizeof(int32_t) * 3);
    add(&r.pb.el, sizeof(double) * 7);
    add(&r.pb.mr_n, sizeof(int32_t) * 2);
    add(&r.pb.rmin, sizeof(double));
    // field by field: the struct's padding bytes are not part of the key
    const tosp_mg_params &m = r.mg;
    for (int32_t v : {m.ngrids, m.cycle, m.smoother, m.smoothiter1, m.smoothiter2, m.maxiterMG, m.nmaxchol,
                      m.flexible, m.maxstall, m.warp_stencil_max, m.small_cycle_max, m.cg_product})
        add(&v, sizeof(v));
    for (double v : {m.omega, m.tolMG, m.replace_drop}) add(&v, sizeof(v));
    add(&r.precision, sizeof(r.precision));
    uint64_t hsh = 1469598103934665603ull;
    auto mix = [&](const std::vector<int64_t> &v) {
        for (int64_t x : v) {
            hsh ^= (uint64_t)x;
            hsh *= 1099511628211ull;
        }
        hsh ^= v.size();
        hsh *= 1099511628211ull;
    };
    mix(r.freedofs);
    mix(r.fixed_dens);
    mix(r.free_dens_g);
    add(&hsh, sizeof(hsh));
    return k;
}

// Multigrid parameters of a served request: as submitted, except that only
// mixed-precision requests keep mg.cg_product (the tensor-core CG product
// with residual replacement; the batch runner replaces residuals per member
// after each tick).  A request with mg.small_cycle_max > 0 runs its small
// levels as the persistent cycle, which the batch runner launches once per
// visit for all same-shape requests.
tosp_mg_params serving_mg(const tosp_mg_params &mg, int precision) {
    tosp_mg_params m = mg;
    if (precision != TOSP_PREC_MIXED) m.cg_product = 0;
    return m;
}

int64_t estimate_bytes(const Request &r) {
    const int64_t nx = r.pb.nelx + 1, ny = r.pb.nely + 1, nz = r.pb.nelz + 1;
    const int64_t ndof = 3 * nx * ny * nz;
    const int64_t nel = (int64_t)r.pb.nelx * r.pb.nely * r.pb.nelz;
    const int64_t nsub = nel * r.pb.mr_n * r.pb.mr_n * r.pb.mr_n;
    const int64_t tsz = r.precision == TOSP_PREC_FP64 ? 8 : 4;
    int64_t b = ndof * (8 * 10 + 4 * tsz + 1) + nsub * 50 + nel * 2;
    b += (nel / 8 + 1) * 576 * 8 * 8 / 7;                  // Galerkin element matrices, all levels
    b += (ndof / 3 / 8 + 1) * 243 * tsz * 8 / 7;           // coarse stencils
    b += (ndof / 8 + 1) * tsz * 4 * 8 / 7;                 // coarse cycle vectors
    b += 64ll << 20;                                       // dense coarsest, scratch, slack
    return b;
}

}  // namespace

// One batch: requests of one shape in flight, stepped together by their own
// runner thread (batches of different shapes do not wait for each other).
struct Batch {
    std::vector<std::shared_ptr<Request>> mem;
    cudaStream_t stream = nullptr;      // the batched small-level launches
    cudaEvent_t ev_small = nullptr;
    std::vector<cudaEvent_t> ev_mem;
    tosp::BatchPlan plan;
    bool dirty = true, unbatched = false;
    std::deque<std::shared_ptr<Request>> join_q;   // first iteration done: joins at the next tick
    std::thread th;                                  // this batch's runner
};

constexpr int BATCH_ENT_CAP = 3 * 64;

struct tosp_server {
    int device = 0;
    int max_slots = 1;
    int64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_dispatch, cv_done, cv_runner;
    std::deque<std::shared_ptr<Request>> queue;     // submitted, not admitted
    std::map<int64_t, std::shared_ptr<Request>> reqs;
    std::vector<CachedHandle> cache;
    std::map<std::string, int64_t> measured;        // device bytes of a created handle, per shape key
    int64_t used_bytes = 0;
    int active = 0;                                 // admitted and not finished
    int64_t next_id = 1;
    bool stopping = false;
    std::vector<std::thread> workers;
    std::map<std::string, std::unique_ptr<Batch>> batches;   // per batch key
    std::deque<std::shared_ptr<Request>> finish_q;  // solve ended: Grad and results
    std::atomic<int64_t> completed{0};
    std::atomic<int64_t> ticks{0}, batched_iterations{0}, max_batch{0};
};

namespace {

int64_t footprint(tosp_server *s, const Request &r) {
    auto it = s->measured.find(r.key);
    return it != s->measured.end() ? it->second : r.est_bytes;
}

// Acquire a handle for the request (called with the lock held).  Returns
// nullptr if the memory budget does not allow it now.  Admission counts a
// shape's measured footprint once one of its handles exists.
CachedHandle *acquire_locked(tosp_server *s, Request &r) {
    for (auto &c : s->cache)
        if (!c.busy && c.key == r.key) {
            c.busy = true;
            return &c;
        }
    const int64_t need = footprint(s, r);
    // need a new handle: evict idle handles of other shapes until it fits
    while (s->used_bytes + need > s->budget) {
        auto victim = s->cache.end();
        for (auto it = s->cache.begin(); it != s->cache.end(); ++it)
            if (!it->busy && it->h && (victim == s->cache.end() || it->last_used < victim->last_used)) victim = it;
        if (victim == s->cache.end()) return nullptr;
        tosp_destroy(victim->h);
        s->used_bytes -= victim->bytes;
        s->cache.erase(victim);
    }
    CachedHandle c;
    c.key = r.key;
    c.busy = true;
    c.bytes = need;            // replaced by the measured size after creation
    s->used_bytes += c.bytes;
    s->cache.push_back(c);
    return &s->cache.back();
}

tosp_handle *create_handle(const Request &r, std::string &err) {
    tosp_problem pb = r.pb;
    pb.freedofs = r.freedofs.data();
    pb.fixed_dens = r.fixed_dens.empty() ? nullptr : r.fixed_dens.data();
    pb.free_dens_g = r.free_dens_g.empty() ? nullptr : r.free_dens_g.data();
    tosp_handle *h = nullptr;
    if (tosp_create(&pb, &r.mg, r.precision, &h) != TOSP_OK) {
        err = tosp_last_error(nullptr);
        return nullptr;
    }
    return h;
}

// Bind a newly created handle to its cache slot (or drop the slot when the
// creation failed); record the shape's measured footprint.  Lock held.
void bind_handle_locked(tosp_server *s, const std::string &key, tosp_handle *h) {
    for (auto it = s->cache.begin(); it != s->cache.end(); ++it) {
        if (!(it->busy && it->key == key && it->h == nullptr)) continue;
        if (!h) {
            s->used_bytes -= it->bytes;
            s->cache.erase(it);
            return;
        }
        it->h = h;
        int32_t ng;
        int64_t nc, nb;
        if (tosp_info(h, &ng, &nc, &nb) == TOSP_OK) {
            s->used_bytes += nb - it->bytes;
            it->bytes = nb;
            s->measured[key] = nb;
        }
        return;
    }
}

void release_handle_locked(tosp_server *s, tosp_handle *h) {
    for (auto &c : s->cache)
        if (c.h == h) {
            c.busy = false;
            c.last_used = Clock::now();
            return;
        }
}

void batch_main(tosp_server *s, Batch *b);

// Setup and the first CG iteration of an admitted request (worker thread).
void start_request(tosp_server *s, const std::shared_ptr<Request> &r) {
    tosp::TraceRange trace_("serving request start");
    r->t_start = Clock::now();
    tosp_handle *h = r->h;
    int rc = tosp_setup_gmg(h, r->xfil.data(), (int64_t)r->xfil.size());
    r->x.assign(r->freedofs.size(), 0.0);
    if (r->u0.size() == r->x.size()) r->x = r->u0;
    if (rc == TOSP_OK) rc = tosp::solve_start(h, r->x.data(), r->f.data());
    std::lock_guard<std::mutex> lk(s->mu);
    if (rc != TOSP_OK) {
        r->status = rc;
        r->err = tosp_last_error(h);
        r->solve_failed = true;
        s->finish_q.push_back(r);
        s->cv_dispatch.notify_all();
    } else if (tosp::solve_state(h).done) {
        s->finish_q.push_back(r);
        s->cv_dispatch.notify_all();
    } else {
        std::unique_ptr<Batch> &bp = s->batches[tosp::batch_key(h)];
        if (!bp) {
            bp.reset(new Batch());
            bp->th = std::thread(batch_main, s, bp.get());
        }
        bp->join_q.push_back(r);
        s->cv_runner.notify_all();
    }
}

// Final update, u to the host, Grad, statistics (worker thread).
void finish_request(tosp_server *s, Request &r) {
    tosp::TraceRange trace_("serving request finish");
    tosp_handle *h = r.h;
    int32_t it = 0;
    double rr = 0;
    int rc = r.status;
    if (!r.solve_failed) {
        rc = tosp::solve_stop(h, r.x.data(), &it, &rr);
        if (rc < 0) r.err = tosp_last_error(h);
    }
    if (rc == TOSP_OK || rc == TOSP_NOT_CONVERGED) {
        const int64_t ndof = 3ll * (r.pb.nelx + 1) * (r.pb.nely + 1) * (r.pb.nelz + 1);
        std::vector<double> ufull(ndof, 0.0);
        for (size_t i = 0; i < r.x.size(); ++i) ufull[r.freedofs[i] - 1] = r.x[i];
        r.g.assign(r.xfil.size(), 0.0);
        const int rg = tosp_grad(h, ufull.data(), ndof, r.g.data(), nullptr, (int64_t)r.g.size());
        if (rg != TOSP_OK) {
            rc = rg;
            r.err = tosp_last_error(h);
        }
    }
    r.u = r.x;
    const auto t1 = Clock::now();
    r.status = rc;
    r.st.it = it;
    r.st.relres = rr;
    r.st.ms_run = std::chrono::duration<double, std::milli>(t1 - r.t_start).count();
    r.st.ms_latency = std::chrono::duration<double, std::milli>(t1 - r.t_submit).count();
    r.st.ms_queue = r.st.ms_latency - r.st.ms_run;
    r.st.precision = r.precision;
    if (tosp::metrics_on()) {
        char buf[320];
        std::snprintf(buf, sizeof buf,
                      "{\"event\": \"request\", \"id\": %lld, \"mesh\": [%d, %d, %d], \"mr_n\": %d, "
                      "\"precision\": %d, \"it\": %d, \"relres\": %.6e, \"ms_latency\": %.3f, "
                      "\"ms_queue\": %.3f, \"ms_run\": %.3f, \"status\": %d}",
                      (long long)r.id, r.pb.nelx, r.pb.nely, r.pb.nelz, r.pb.mr_n, r.precision, it, rr,
                      r.st.ms_latency, r.st.ms_queue, r.st.ms_run, rc);
        tosp::metrics_line(buf);
    }
    (void)s;
}

void worker_main(tosp_server *s) {
    cudaSetDevice(s->device);
    for (;;) {
        std::shared_ptr<Request> r;
        bool finishing = false;
        CachedHandle *c = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (!s->finish_q.empty()) {
                    r = s->finish_q.front();
                    s->finish_q.pop_front();
                    finishing = true;
                    break;
                }
                if (s->stopping && s->queue.empty() && s->active == 0) return;
                // FIFO admission: the head waits until a slot and memory are free
                if (!s->stopping && !s->queue.empty() && s->active < s->max_slots) {
                    c = acquire_locked(s, *s->queue.front());
                    if (c) {
                        r = s->queue.front();
                        s->queue.pop_front();
                        r->state = TOSP_REQ_RUNNING;
                        s->active++;
                        break;
                    }
                }
                s->cv_dispatch.wait(lk);
            }
        }
        if (!finishing) {
            tosp_handle *h = c->h;
            const std::string key = c->key;
            if (!h) {
                std::string err;
                h = create_handle(*r, err);
                std::lock_guard<std::mutex> lk(s->mu);
                bind_handle_locked(s, key, h);
                if (!h) {
                    r->status = TOSP_ERR_CUDA;
                    r->err = err;
                    r->state = TOSP_REQ_FAILED;
                    s->active--;
                    s->completed++;
                    s->cv_done.notify_all();
                    s->cv_dispatch.notify_all();
                    continue;
                }
            }
            r->h = h;
            start_request(s, r);
            continue;
        }
        // a breakdown leaves the handle's iterate unusable for a warm start
        finish_request(s, *r);
        if (r->status == TOSP_ERR_BREAKDOWN) r->u.clear();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            release_handle_locked(s, r->h);
            r->h = nullptr;
            const bool stalled = r->status == TOSP_NOT_CONVERGED || r->status == TOSP_ERR_BREAKDOWN;
            if (stalled && r->precision == TOSP_PREC_MIXED && r->fallbacks == 0) {
                // re-run once in FP64 (front of the queue), warm-started from
                // the mixed iterate when it is finite
                r->fallbacks = 1;
                r->precision = TOSP_PREC_FP64;
                r->mg.maxstall = 0;
                r->mg.cg_product = 0;
                r->u0.clear();
                bool finite = !r->u.empty();
                for (double v : r->u) finite = finite && std::isfinite(v);
                if (finite) r->u0 = r->u;
                r->key = shape_key(*r);
                r->est_bytes = estimate_bytes(*r);
                r->state = TOSP_REQ_QUEUED;
                r->status = TOSP_OK;
                r->solve_failed = false;
                r->err.clear();
                s->queue.push_front(r);
            } else {
                r->state = r->status < 0 ? TOSP_REQ_FAILED : TOSP_REQ_DONE;
            }
            s->active--;
            s->completed++;
        }
        s->cv_done.notify_all();
        s->cv_dispatch.notify_all();
    }
}


// Tables of the batched small-level launch for the current members.
void batch_rebuild(Batch &b) {
    b.dirty = false;
    b.unbatched = false;
    b.plan.mem.clear();
    for (auto &r : b.mem) b.plan.mem.push_back(r->h);
    while (b.ev_mem.size() < b.mem.size()) {
        cudaEvent_t e = nullptr;
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        b.ev_mem.push_back(e);
    }
    std::string err;
    if ((int)b.mem.size() * 3 > BATCH_ENT_CAP || tosp::batch_prepare(b.plan, b.stream, err) != TOSP_OK)
        b.unbatched = true;   // members then step one by one
}

// A batch's runner: every tick queues one CG iteration of every member,
// waits, and does each member's loop bookkeeping; members that are done go to
// the workers, new ones join before the next tick.
void batch_main(tosp_server *s, Batch *b) {
    cudaSetDevice(s->device);
    cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&b->ev_small, cudaEventDisableTiming);
    cudaMalloc(&b->plan.d_ent, sizeof(tosp::SmallBatchEntry) * BATCH_ENT_CAP);
    cudaMalloc(&b->plan.d_bar, sizeof(tosp::GridBarrier));
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_runner.wait(lk, [&] {
                return !b->mem.empty() || !b->join_q.empty() || (s->stopping && s->active == 0);
            });
            if (b->mem.empty() && b->join_q.empty()) break;   // stopping, nothing in flight
            for (auto &r : b->join_q) b->mem.push_back(r);
            if (!b->join_q.empty()) b->dirty = true;
            b->join_q.clear();
        }
        if (b->dirty) batch_rebuild(*b);
        tosp::TraceRange trace_("serving batch tick");
        if (!b->unbatched) {
            std::string err;
            if (tosp::batch_tick(b->plan, b->stream, b->ev_mem.data(), b->ev_small, err) != TOSP_OK) {
                // nothing of a failed tick is trusted: members fail
                for (auto &r : b->mem) {
                    r->solve_failed = true;
                    r->status = TOSP_ERR_CUDA;
                    r->err = "batched iteration: " + err;
                }
            }
            for (auto &r : b->mem) cudaStreamSynchronize(tosp::handle_stream(r->h));
            cudaStreamSynchronize(b->stream);
            // a batched small-level launch whose bounded barrier wait ran out
            // leaves its members' iterates unusable: they fail
            tosp::GridBarrier gb{};
            bool timed_out = false;
            if (b->plan.blocks > 0 && cudaMemcpy(&gb, b->plan.d_bar, sizeof gb, cudaMemcpyDeviceToHost) == cudaSuccess &&
                gb.err) {
                timed_out = true;
                cudaMemset(b->plan.d_bar, 0, sizeof gb);
            }
            for (auto &r : b->mem) {
                if (r->solve_failed) continue;
                if (timed_out) {
                    r->solve_failed = true;
                    r->status = TOSP_ERR_TIMEOUT;
                    r->err = "batched small-level cycle: grid barrier wait timed out";
                } else if (tosp::solve_step_account(r->h) != TOSP_OK) {
                    r->solve_failed = true;
                    r->status = TOSP_ERR_CUDA;
                    r->err = tosp_last_error(r->h);
                }
            }
            s->batched_iterations += (int64_t)b->mem.size();
            if ((int64_t)b->mem.size() > s->max_batch) s->max_batch = (int64_t)b->mem.size();
        } else {
            // one member at a time on its own stream (its own graphs)
            for (auto &r : b->mem)
                if (tosp::solve_step(r->h) != TOSP_OK) r->solve_failed = true;
        }
        std::vector<std::shared_ptr<Request>> done;
        for (size_t i = 0; i < b->mem.size();) {
            auto &r = b->mem[i];
            if (r->solve_failed || tosp::solve_state(r->h).done) {
                if (r->solve_failed && r->status == TOSP_OK) {
                    r->status = TOSP_ERR_CUDA;
                    r->err = tosp_last_error(r->h);
                }
                done.push_back(r);
                b->mem.erase(b->mem.begin() + i);
                b->dirty = true;
            } else {
                ++i;
            }
        }
        s->ticks++;
        if (!done.empty()) {
            std::lock_guard<std::mutex> lk(s->mu);
            for (auto &r : done) s->finish_q.push_back(r);
            s->cv_dispatch.notify_all();
        }
    }
    for (auto &e : b->ev_mem)
        if (e) cudaEventDestroy(e);
    if (b->ev_small) cudaEventDestroy(b->ev_small);
    if (b->plan.d_ent) cudaFree(b->plan.d_ent);
    if (b->plan.d_bar) cudaFree(b->plan.d_bar);
    if (b->stream) cudaStreamDestroy(b->stream);
}

}  // namespace

extern "C" {

int tosp_server_create(int32_t max_slots, int64_t hbm_budget_bytes, tosp_server **out) {
    if (!out || max_slots < 1 || max_slots > 64 || hbm_budget_bytes <= 0) return TOSP_ERR_BAD_ARG;
    auto *s = new (std::nothrow) tosp_server();
    if (!s) return TOSP_ERR_OOM;
    cudaGetDevice(&s->device);
    s->max_slots = max_slots;
    s->budget = hbm_budget_bytes;
    // workers set requests up and finish them; each shape's batch has its own
    // runner thread, started with the first request of that shape
    const int nworkers = max_slots;
    for (int i = 0; i < nworkers; ++i) s->workers.emplace_back(worker_main, s);
    *out = s;
    return TOSP_OK;
}

int tosp_server_prepare(tosp_server *s, const tosp_problem *pb, const tosp_mg_params *mg, int32_t precision,
                        int32_t count) {
    if (!s || !pb || !mg || !pb->freedofs || count < 0) return TOSP_ERR_BAD_ARG;
    Request r;
    r.pb = *pb;
    r.freedofs.assign(pb->freedofs, pb->freedofs + pb->nfree);
    if (pb->fixed_dens && pb->nfixed_dens > 0) r.fixed_dens.assign(pb->fixed_dens, pb->fixed_dens + pb->nfixed_dens);
    if (pb->free_dens_g && pb->nfree_dens_g > 0)
        r.free_dens_g.assign(pb->free_dens_g, pb->free_dens_g + pb->nfree_dens_g);
    r.pb.freedofs = nullptr;
    r.pb.fixed_dens = nullptr;
    r.pb.free_dens_g = nullptr;
    r.mg = serving_mg(*mg, precision);
    r.precision = precision;
    r.key = shape_key(r);
    r.est_bytes = estimate_bytes(r);
    cudaSetDevice(s->device);
    for (int k = 0; k < count; ++k) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            int have = 0;
            for (auto &c : s->cache) have += c.key == r.key;
            if (have > k) continue;          // enough handles of this shape exist
            if (s->used_bytes + footprint(s, r) > s->budget) return TOSP_ERR_OOM;
            CachedHandle c;
            c.key = r.key;
            c.busy = true;
            c.bytes = footprint(s, r);
            s->used_bytes += c.bytes;
            s->cache.push_back(c);
        }
        std::string err;
        tosp_handle *h = create_handle(r, err);
        std::lock_guard<std::mutex> lk(s->mu);
        bind_handle_locked(s, r.key, h);
        if (!h) return TOSP_ERR_CUDA;
        release_handle_locked(s, h);
    }
    return TOSP_OK;
}

int tosp_server_submit(tosp_server *s, const tosp_problem *pb, const tosp_mg_params *mg, int32_t precision,
                       const double *xfil, int64_t ndens, const double *f, int64_t nfree, int64_t *request_id) {
    if (!s || !pb || !mg || !xfil || !f || !request_id || !pb->freedofs || pb->nfree != nfree) return TOSP_ERR_BAD_ARG;
    const int64_t nel = (int64_t)pb->nelx * pb->nely * pb->nelz;
    if (pb->mr_n < 1 || pb->mr_n > 3 || ndens != nel * pb->mr_n * pb->mr_n * pb->mr_n) return TOSP_ERR_BAD_ARG;
    auto r = std::make_shared<Request>();
    r->pb = *pb;
    r->freedofs.assign(pb->freedofs, pb->freedofs + pb->nfree);
    if (pb->fixed_dens && pb->nfixed_dens > 0)
        r->fixed_dens.assign(pb->fixed_dens, pb->fixed_dens + pb->nfixed_dens);
    if (pb->free_dens_g && pb->nfree_dens_g > 0)
        r->free_dens_g.assign(pb->free_dens_g, pb->free_dens_g + pb->nfree_dens_g);
    r->pb.freedofs = nullptr;
    r->pb.fixed_dens = nullptr;
    r->pb.free_dens_g = nullptr;
    r->mg = serving_mg(*mg, precision);
    r->precision = precision;
    r->xfil.assign(xfil, xfil + ndens);
    r->f.assign(f, f + nfree);
    r->key = shape_key(*r);
    r->est_bytes = estimate_bytes(*r);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (footprint(s, *r) > s->budget) return TOSP_ERR_OOM;    // can never be admitted
        r->id = s->next_id++;
        s->reqs[r->id] = r;
        s->queue.push_back(r);
        *request_id = r->id;
    }
    s->cv_dispatch.notify_all();
    return TOSP_OK;
}

int tosp_server_poll(tosp_server *s, int64_t id, int32_t *state) {
    if (!s || !state) return TOSP_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return TOSP_ERR_BAD_ARG;
    *state = it->second->state;
    return TOSP_OK;
}

int tosp_server_wait(tosp_server *s, int64_t id, double timeout_s) {
    if (!s) return TOSP_ERR_BAD_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return TOSP_ERR_BAD_ARG;
    auto r = it->second;
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
        return r->state == TOSP_REQ_DONE || r->state == TOSP_REQ_FAILED || r->state == TOSP_REQ_CANCELLED;
    });
    return ok ? TOSP_OK : TOSP_ERR_TIMEOUT;
}

int tosp_server_result(tosp_server *s, int64_t id, double *u, int64_t nfree, double *fgrad, int64_t ndens,
                       tosp_request_stats *st) {
    if (!s) return TOSP_ERR_BAD_ARG;
    std::shared_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) return TOSP_ERR_BAD_ARG;
        r = it->second;
        if (r->state == TOSP_REQ_QUEUED || r->state == TOSP_REQ_RUNNING) return TOSP_ERR_STATE;
        if (r->state == TOSP_REQ_CANCELLED) return TOSP_ERR_CANCELLED;
    }
    if (st) *st = r->st;
    if (r->status < 0) return r->status;
    if (u) {
        if (nfree != (int64_t)r->u.size()) return TOSP_ERR_BAD_ARG;
        std::memcpy(u, r->u.data(), sizeof(double) * r->u.size());
    }
    if (fgrad) {
        if (ndens != (int64_t)r->g.size()) return TOSP_ERR_BAD_ARG;
        std::memcpy(fgrad, r->g.data(), sizeof(double) * r->g.size());
    }
    return r->status;
}

int tosp_server_cancel(tosp_server *s, int64_t id) {
    if (!s) return TOSP_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return TOSP_ERR_BAD_ARG;
    auto r = it->second;
    if (r->state != TOSP_REQ_QUEUED) return TOSP_ERR_STATE;   // running requests finish
    s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), r), s->queue.end());
    r->state = TOSP_REQ_CANCELLED;
    s->cv_done.notify_all();
    s->cv_dispatch.notify_all();
    return TOSP_OK;
}

int tosp_server_release(tosp_server *s, int64_t id) {
    if (!s) return TOSP_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return TOSP_ERR_BAD_ARG;
    if (it->second->state == TOSP_REQ_QUEUED || it->second->state == TOSP_REQ_RUNNING) return TOSP_ERR_STATE;
    s->reqs.erase(it);
    return TOSP_OK;
}

int tosp_server_info(tosp_server *s, int32_t *active, int32_t *queued, int64_t *used_bytes, int64_t *cached_handles) {
    if (!s) return TOSP_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (active) *active = s->active;
    if (queued) *queued = (int32_t)s->queue.size();
    if (used_bytes) *used_bytes = s->used_bytes;
    if (cached_handles) *cached_handles = (int64_t)s->cache.size();
    return TOSP_OK;
}

int tosp_server_counters(tosp_server *s, int64_t *ticks, int64_t *batched_iterations, int64_t *max_batch) {
    if (!s) return TOSP_ERR_BAD_ARG;
    if (ticks) *ticks = s->ticks.load();
    if (batched_iterations) *batched_iterations = s->batched_iterations.load();
    if (max_batch) *max_batch = s->max_batch.load();
    return TOSP_OK;
}

int tosp_server_destroy(tosp_server *s) {
    if (!s) return TOSP_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        for (auto &r : s->queue) r->state = TOSP_REQ_CANCELLED;
        s->queue.clear();
    }
    s->cv_dispatch.notify_all();
    s->cv_runner.notify_all();
    for (auto &t : s->workers) t.join();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->cv_runner.notify_all();
    }
    for (auto &kv : s->batches)
        if (kv.second->th.joinable()) kv.second->th.join();
    for (auto &c : s->cache)
        if (c.h) tosp_destroy(c.h);
    delete s;
    return TOSP_OK;
}

}  // extern "C"
