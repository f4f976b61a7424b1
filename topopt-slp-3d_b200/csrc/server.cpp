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
    Clock::time_point t_submit;
    int64_t est_bytes = 0;
    std::string key;
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
    add(&r.mg, sizeof(r.mg));
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

struct tosp_server {
    int device = 0;
    int max_slots = 1;
    int64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_dispatch, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::map<int64_t, std::shared_ptr<Request>> reqs;
    std::vector<CachedHandle> cache;
    int64_t used_bytes = 0;
    int active = 0;
    int64_t next_id = 1;
    bool stopping = false;
    std::vector<std::thread> workers;
    std::deque<std::shared_ptr<Request>> ready;   // admitted, waiting for a worker
    std::atomic<int64_t> completed{0};
};

namespace {

// Acquire a handle for the request (called with the lock held).  Returns
// nullptr if the memory budget does not allow it now.
CachedHandle *acquire_locked(tosp_server *s, Request &r) {
    for (auto &c : s->cache)
        if (!c.busy && c.key == r.key) {
            c.busy = true;
            return &c;
        }
    // need a new handle: evict idle handles of other shapes until it fits
    while (s->used_bytes + r.est_bytes > s->budget) {
        auto victim = s->cache.end();
        for (auto it = s->cache.begin(); it != s->cache.end(); ++it)
            if (!it->busy && (victim == s->cache.end() || it->last_used < victim->last_used)) victim = it;
        if (victim == s->cache.end()) return nullptr;
        tosp_destroy(victim->h);
        s->used_bytes -= victim->bytes;
        s->cache.erase(victim);
    }
    CachedHandle c;
    c.key = r.key;
    c.busy = true;
    c.bytes = r.est_bytes;     // replaced by the measured size after creation
    s->used_bytes += c.bytes;
    s->cache.push_back(c);
    return &s->cache.back();
}

void run_request(tosp_server *s, Request &r, tosp_handle *h) {
    const auto t0 = Clock::now();
    int rc = tosp_setup_gmg(h, r.xfil.data(), (int64_t)r.xfil.size());
    std::vector<double> x(r.freedofs.size(), 0.0);
    if (r.u0.size() == x.size()) x = r.u0;
    int32_t it = 0;
    double rr = 0;
    if (rc == TOSP_OK) rc = tosp_solve_mg(h, x.data(), r.f.data(), (int64_t)x.size(), &it, &rr);
    if (rc == TOSP_OK || rc == TOSP_NOT_CONVERGED) {
        const int64_t ndof = 3ll * (r.pb.nelx + 1) * (r.pb.nely + 1) * (r.pb.nelz + 1);
        std::vector<double> ufull(ndof, 0.0);
        for (size_t i = 0; i < x.size(); ++i) ufull[r.freedofs[i] - 1] = x[i];
        r.g.assign(r.xfil.size(), 0.0);
        const int rg = tosp_grad(h, ufull.data(), ndof, r.g.data(), nullptr, (int64_t)r.g.size());
        if (rg != TOSP_OK) rc = rg;
        r.u = std::move(x);
    }
    tosp_solve_stats st;
    tosp_last_stats(h, &st);
    const auto t1 = Clock::now();
    r.status = rc;
    if (rc < 0) r.err = tosp_last_error(h);
    r.st.it = it;
    r.st.relres = rr;
    r.st.ms_run = std::chrono::duration<double, std::milli>(t1 - t0).count();
    r.st.ms_latency = std::chrono::duration<double, std::milli>(t1 - r.t_submit).count();
    r.st.ms_queue = r.st.ms_latency - r.st.ms_run;
    r.st.precision = r.precision;
    (void)s;
}

void worker_main(tosp_server *s) {
    cudaSetDevice(s->device);
    for (;;) {
        std::shared_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_dispatch.wait(lk, [&] { return s->stopping || !s->queue.empty(); });
            if (s->stopping && s->queue.empty()) return;
            // FIFO admission: the head waits until a slot and memory are free
            CachedHandle *c = nullptr;
            for (;;) {
                if (s->stopping && s->queue.empty()) return;
                if (!s->queue.empty()) {
                    c = acquire_locked(s, *s->queue.front());
                    if (c) break;
                }
                s->cv_dispatch.wait(lk);
            }
            r = s->queue.front();
            s->queue.pop_front();
            r->state = TOSP_REQ_RUNNING;
            s->active++;
            // create the handle outside the lock if needed
            tosp_handle *h = c->h;
            std::string key = c->key;
            lk.unlock();
            int rc = TOSP_OK;
            if (!h) {
                tosp_problem pb = r->pb;
                pb.freedofs = r->freedofs.data();
                pb.fixed_dens = r->fixed_dens.empty() ? nullptr : r->fixed_dens.data();
                pb.free_dens_g = r->free_dens_g.empty() ? nullptr : r->free_dens_g.data();
                rc = tosp_create(&pb, &r->mg, r->precision, &h);
                if (rc != TOSP_OK) {
                    r->err = tosp_last_error(nullptr);
                    h = nullptr;
                }
            }
            if (h) {
                // a breakdown leaves the handle's iterate unusable for a warm start
                run_request(s, *r, h);
                if (r->status == TOSP_ERR_BREAKDOWN) r->u.clear();
            } else {
                r->status = rc;
            }
            lk.lock();
            for (auto it = s->cache.begin(); it != s->cache.end(); ++it) {
                if (it->busy && it->key == key && (it->h == h || it->h == nullptr)) {
                    if (!h) {
                        s->used_bytes -= it->bytes;
                        s->cache.erase(it);
                    } else {
                        if (!it->h) {
                            it->h = h;
                            int32_t ng;
                            int64_t nc, nb;
                            if (tosp_info(h, &ng, &nc, &nb) == TOSP_OK) {
                                s->used_bytes += nb - it->bytes;
                                it->bytes = nb;
                            }
                        }
                        it->busy = false;
                        it->last_used = Clock::now();
                    }
                    break;
                }
            }
            const bool stalled = r->status == TOSP_NOT_CONVERGED || r->status == TOSP_ERR_BREAKDOWN;
            if (stalled && r->precision == TOSP_PREC_MIXED && r->fallbacks == 0) {
                // re-run once in FP64 (front of the queue), warm-started from
                // the mixed iterate when it is finite
                r->fallbacks = 1;
                r->precision = TOSP_PREC_FP64;
                r->mg.maxstall = 0;
                r->u0.clear();
                bool finite = !r->u.empty();
                for (double v : r->u) finite = finite && std::isfinite(v);
                if (finite) r->u0 = r->u;
                r->key = shape_key(*r);
                r->est_bytes = estimate_bytes(*r);
                r->state = TOSP_REQ_QUEUED;
                r->status = TOSP_OK;
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

}  // namespace

extern "C" {

int tosp_server_create(int32_t max_slots, int64_t hbm_budget_bytes, tosp_server **out) {
    if (!out || max_slots < 1 || max_slots > 64 || hbm_budget_bytes <= 0) return TOSP_ERR_BAD_ARG;
    auto *s = new (std::nothrow) tosp_server();
    if (!s) return TOSP_ERR_OOM;
    cudaGetDevice(&s->device);
    s->max_slots = max_slots;
    s->budget = hbm_budget_bytes;
    for (int i = 0; i < max_slots; ++i) s->workers.emplace_back(worker_main, s);
    *out = s;
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
    r->mg = *mg;
    r->precision = precision;
    r->xfil.assign(xfil, xfil + ndens);
    r->f.assign(f, f + nfree);
    r->key = shape_key(*r);
    r->est_bytes = estimate_bytes(*r);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (r->est_bytes > s->budget) return TOSP_ERR_OOM;    // can never be admitted
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

int tosp_server_destroy(tosp_server *s) {
    if (!s) return TOSP_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        for (auto &r : s->queue) r->state = TOSP_REQ_CANCELLED;
        s->queue.clear();
    }
    s->cv_dispatch.notify_all();
    for (auto &t : s->workers) t.join();
    for (auto &c : s->cache)
        if (c.h) tosp_destroy(c.h);
    delete s;
    return TOSP_OK;
}

}  // extern "C"
