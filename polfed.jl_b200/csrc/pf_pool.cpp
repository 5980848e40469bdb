// pf_pool.cpp -- batched and served POLFED solves on one device.
//
// A pool owns W worker threads, each with its own pf_handle (stream, cuBLAS,
// cuSOLVER, workspaces).  Requests wait in one FIFO queue; a free worker takes
// the head as soon as its estimated device footprint fits in the pool's HBM
// budget (continuous batching: requests that arrive while others run start as
// workers and memory free up).  Each request runs exactly pf_solve on a view
// of its operator bound to the worker's handle, so a result does not depend on
// what else is in flight.  Solver workspaces are stream-ordered allocations
// from the device pool, so concurrent solves never synchronise the device.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "pf_internal.h"
#include "pf_solver.h"

namespace pf {

using Clock = std::chrono::steady_clock;

struct PoolRequest {
    int64_t id = 0;
    // the request's own view of the caller's operator (taken at submit; it
    // shares the device tables and the tuned step widths of that moment), so
    // the caller may destroy its operator as soon as the call returns
    std::unique_ptr<pf_op, void (*)(pf_op *)> own{nullptr, destroy_op};
    pf_op *op = nullptr;
    pf_params params{};
    int s = 1, nev = 1;
    std::vector<double> x0_copy;        // serving path: owned copy of x0
    const double *x0 = nullptr;         // what the solve reads
    int x0_mem = PF_MEM_HOST;
    double *vecs_out = nullptr;
    int vecs_mem = PF_MEM_HOST;
    double *vals_out = nullptr;         // batch path: caller's arrays
    pf_report *rep_out = nullptr;
    int *nconv_out = nullptr;
    std::vector<double> vals;           // serving path: results kept until fetch
    pf_report rep{};
    int nconv = 0;
    int state = PF_REQ_QUEUED;
    int status = PF_OK;
    std::string error;
    double footprint = 0.0;
    double cost = 0.0;                  // expected solve work (admission order)
    bool cancelled = false, batch = false, urgent = false, started = false;
    Clock::time_point t_submit, t_start, t_done;
};

}  // namespace pf

struct pf_pool {
    int device = 0;
    std::vector<pf_handle *> handles;   // one per worker, default stream priority
    std::vector<pf_handle *> urgent;    // one per worker, the device's highest stream priority
    int64_t priority_dim = 65536;       // requests with D <= this run on the urgent handles
    int admission = PF_ADMIT_FIFO;
    double max_wait = 30.0;             // PF_ADMIT_SHORTEST: seconds after which a request goes in arrival order
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<pf::PoolRequest>> queue;
    std::unordered_map<int64_t, std::shared_ptr<pf::PoolRequest>> requests;
    double budget = 0.0, in_use = 0.0, peak = 0.0;
    int64_t next_id = 1, submitted = 0, completed = 0, failed = 0, rejected = 0, running = 0, eigenpairs = 0;
    std::vector<double> latencies;
    double busy = 0.0;
    pf::Clock::time_point busy_since, t_created;
    bool stop = false;
    int waiters = 0;                    // threads blocked in fetch / solve_batch (destroy waits for them)
    pf_engine *engine = nullptr;        // batches the Clenshaw steps of every solve in flight
    bool batching = false;              // requests hand their filters to the engine
};

namespace pf {

// Device memory a handle may still grow after creation (library workspaces,
// its auxiliary handle); the default HBM budget keeps this much per handle free.
constexpr size_t kHandleReserveBytes = size_t(96) << 20;

static bool finished(int state) {
    return state == PF_REQ_DONE || state == PF_REQ_FAILED || state == PF_REQ_REJECTED;
}

double solve_footprint(const pf_op *op, const pf_params *p, int s, int nev) {
    const double D = (double)op->dim;
    const int64_t md0 = (int64_t)std::ceil((20.427 * s + 1.696 * nev) * p->overestimate_iters);
    const double maxdim = (double)((md0 + s - 1) / s * s);
    const double ext = (p->has_Emin && p->has_Emax) ? 0.0 : (double)(p->extrema_maxdim > 0 ? p->extrema_maxdim : 1000);
    const double w = p->precision == PF_PREC_FP64 ? 8.0 : 4.0;
    double bytes = 8.0 * D * std::max(ext + 3.0, maxdim + 3.0 * s);  // Krylov basis + Lanczos blocks
    bytes += 4.0 * D * s * w + 2.0 * 8.0 * D * s;                     // filter blocks, x0 copies
    bytes += 2.0 * D * 64 * w;                                        // KPM probe blocks
    bytes += 2.0 * 8.0 * D * nev;                                     // Ritz vectors and H psi
    bytes += 3.0 * 8.0 * maxdim * maxdim + (64 << 20);                // projected matrix, its eigenvectors, slack
    return bytes;
}

// Expected work of a solve: the filter order grows like D / nev, a step costs
// D * s, and the Krylov budget is (20.427 s + 1.696 nev) columns
// (PolfedDefaults.jl:61-62), so work ~ D^2 (20.427 s + 1.696 nev) / nev.
static double expected_cost(const pf_op *op, int s, int nev) {
    const double D = (double)op->dim;
    return D * D * (20.427 * s + 1.696 * nev) / std::max(nev, 1);
}

// Index in the queue of the request to start now, or -1.  A request larger
// than the whole budget still runs alone.  FIFO: the head only.  SHORTEST:
// cancelled entries and requests that waited max_wait seconds first, in
// arrival order (nothing overtakes an aged request), otherwise the fitting
// request of least expected cost (earliest among equals).
static long pick_request(pf_pool *pool) {
    auto fits = [&](const std::shared_ptr<PoolRequest> &r) {
        return pool->in_use + r->footprint <= pool->budget || pool->running == 0;
    };
    if (pool->queue.empty()) return -1;
    if (pool->admission == PF_ADMIT_FIFO) {
        const auto &head = pool->queue.front();
        return (head->cancelled || fits(head)) ? 0 : -1;
    }
    const auto now = Clock::now();
    for (size_t i = 0; i < pool->queue.size(); ++i) {
        const auto &r = pool->queue[i];
        if (r->cancelled) return (long)i;
        if (std::chrono::duration<double>(now - r->t_submit).count() >= pool->max_wait) return fits(r) ? (long)i : -1;
    }
    long best = -1;
    for (size_t i = 0; i < pool->queue.size(); ++i) {
        const auto &r = pool->queue[i];
        if (fits(r) && (best < 0 || r->cost < pool->queue[(size_t)best]->cost)) best = (long)i;
    }
    return best;
}

static void pool_worker(pf_pool *pool, int w) {
    cudaSetDevice(pool->device);
    while (true) {
        std::shared_ptr<PoolRequest> req;
        {
            std::unique_lock<std::mutex> lock(pool->mu);
            long pick = -1;
            pool->cv_work.wait(lock, [&] {
                if (pool->stop) return true;
                pick = pick_request(pool);
                return pick >= 0;
            });
            if (pool->stop) return;   // pool_destroy has already failed every queued request
            if (pick < 0 || pool->queue.empty()) continue;
            req = pool->queue[(size_t)pick];
            pool->queue.erase(pool->queue.begin() + pick);
            if (req->cancelled) {
                pool->requests.erase(req->id);
                pool->cv_work.notify_all();
                continue;
            }
            req->urgent = req->op->dim <= pool->priority_dim;
            req->started = true;
            req->t_start = Clock::now();
            pool->in_use += req->footprint;
            pool->peak = std::max(pool->peak, pool->in_use);
            if (pool->running++ == 0) pool->busy_since = Clock::now();
            req->state = PF_REQ_RUNNING;
        }
        // small solves on the high-priority stream: their short launches are
        // dispatched ahead of queued launches of larger solves (same results)
        pf_handle *h = req->urgent ? pool->urgent[w] : pool->handles[w];
        {
            std::lock_guard<std::mutex> lock(pool->mu);
            h->engine = pool->batching ? pool->engine : nullptr;
        }
        int status = PF_OK;
        bool infeasible = false;
        std::string err;
        pf_op *view = nullptr;
        try {
            view = bind_op(req->op, h);
            double *vals = req->batch ? req->vals_out : req->vals.data();
            solve(view, &req->params, req->s, req->nev, req->x0, req->x0_mem, vals, req->vecs_out, req->vecs_mem,
                  &req->rep, &req->nconv);
        } catch (const Error &e) {
            status = e.code;
            err = e.what();
            infeasible = e.infeasible;
        } catch (const std::exception &e) {
            status = PF_ERR_CUDA;
            err = e.what();
        }
        destroy_op(view);
        {
            std::lock_guard<std::mutex> lock(pool->mu);
            pool->in_use -= req->footprint;
            if (--pool->running == 0)
                pool->busy += std::chrono::duration<double>(Clock::now() - pool->busy_since).count();
            req->t_done = Clock::now();
            req->status = status;
            req->error = err;
            // an infeasible request (fewer than nev states within reach of its
            // target, the reference's bisection error) is rejected, not failed
            req->state = status == PF_OK ? PF_REQ_DONE : (infeasible ? PF_REQ_REJECTED : PF_REQ_FAILED);
            if (status == PF_OK) {
                ++pool->completed;
                pool->eigenpairs += req->nconv;
                pool->latencies.push_back(std::chrono::duration<double>(req->t_done - req->t_submit).count());
                if (req->batch) {
                    if (req->rep_out) *req->rep_out = req->rep;
                    if (req->nconv_out) *req->nconv_out = req->nconv;
                }
            } else if (infeasible) {
                ++pool->rejected;
            } else {
                ++pool->failed;
            }
            if (req->cancelled) pool->requests.erase(req->id);
        }
        pool->cv_done.notify_all();
        pool->cv_work.notify_all();
    }
}

pf_pool *pool_create(int device, int workers, double budget) {
    PF_CHECK(workers >= 1 && workers <= 64, PF_ERR_INVALID, "a pool needs 1..64 workers");
    PF_CUDA(cudaSetDevice(device));
    pf_pool *pool = new pf_pool();
    pool->device = device;
    pool->t_created = Clock::now();
    try {
        int least = 0, greatest = 0;
        PF_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        for (int w = 0; w < workers; ++w) {
            pf_handle *h = nullptr;
            if (pf_handle_create(device, &h) != PF_OK) throw Error(PF_ERR_CUDA, pf_last_error());
            pool->handles.push_back(h);
            const int saved = t_new_handle_priority;
            t_new_handle_priority = greatest;
            const int st = pf_handle_create(device, &h);
            t_new_handle_priority = saved;
            if (st != PF_OK) throw Error(PF_ERR_CUDA, pf_last_error());
            pool->urgent.push_back(h);
        }
        if (budget <= 0) {
            // read after the handles exist; each of the 2 W handles later grows
            // library workspaces and an auxiliary handle of its own, so keep a
            // reserve for those out of the budget
            size_t fr = 0, tot = 0;
            PF_CUDA(cudaMemGetInfo(&fr, &tot));
            const double reserve = 2.0 * workers * double(kHandleReserveBytes);
            budget = std::max(0.0, 0.9 * ((double)fr - reserve));
        }
        pool->budget = budget;
        pool->engine = engine_create(device);
        for (int w = 0; w < workers; ++w) pool->threads.emplace_back(pool_worker, pool, w);
    } catch (...) {
        {
            std::lock_guard<std::mutex> lock(pool->mu);
            pool->stop = true;
        }
        pool->cv_work.notify_all();
        for (auto &t : pool->threads) t.join();
        for (auto h : pool->handles) pf_handle_destroy(h);
        for (auto h : pool->urgent) pf_handle_destroy(h);
        engine_destroy(pool->engine);
        delete pool;
        throw;
    }
    return pool;
}

void pool_shutdown(pf_pool *pool) {
    if (!pool) return;
    {
        // queued requests never run: they fail with "pool destroyed", and
        // threads waiting for them in fetch / solve_batch are woken
        std::lock_guard<std::mutex> lock(pool->mu);
        if (pool->stop) return;
        for (auto &r : pool->queue) {
            r->state = PF_REQ_FAILED;
            r->status = PF_ERR_INVALID;
            r->error = "pool destroyed before the request started";
            r->t_done = Clock::now();
            ++pool->failed;
        }
        pool->queue.clear();
        pool->stop = true;
    }
    pool->cv_work.notify_all();
    pool->cv_done.notify_all();
    for (auto &t : pool->threads) t.join();   // running requests finish
    pool->threads.clear();
}

void pool_destroy(pf_pool *pool) {
    if (!pool) return;
    pool_shutdown(pool);
    {
        // no thread may still be inside fetch / wait / solve_batch when the pool goes
        std::unique_lock<std::mutex> lock(pool->mu);
        pool->cv_done.notify_all();
        pool->cv_done.wait(lock, [&] { return pool->waiters == 0; });
    }
    engine_destroy(pool->engine);
    for (auto h : pool->handles) pf_handle_destroy(h);
    for (auto h : pool->urgent) pf_handle_destroy(h);
    delete pool;
}

void pool_set_batching(pf_pool *pool, int on) {
    PF_CHECK(pool, PF_ERR_INVALID, "null pool");
    std::lock_guard<std::mutex> lock(pool->mu);
    pool->batching = on != 0;
}

void pool_set_admission(pf_pool *pool, int policy, double max_wait) {
    PF_CHECK(pool && (policy == PF_ADMIT_FIFO || policy == PF_ADMIT_SHORTEST) && max_wait >= 0, PF_ERR_INVALID,
             "invalid admission policy");
    {
        std::lock_guard<std::mutex> lock(pool->mu);
        pool->admission = policy;
        pool->max_wait = max_wait;
    }
    pool->cv_work.notify_all();
}

void pool_set_priority_dim(pf_pool *pool, int64_t dim) {
    PF_CHECK(pool && dim >= 0, PF_ERR_INVALID, "invalid argument");
    std::lock_guard<std::mutex> lock(pool->mu);
    pool->priority_dim = dim;
}

cudaStream_t pool_stream(pf_pool *pool, int worker) {
    const int W = (int)pool->handles.size();
    PF_CHECK(worker >= 0 && worker < 2 * W, PF_ERR_INVALID, "no such worker stream");
    return worker < W ? pool->handles[worker]->stream : pool->urgent[worker - W]->stream;
}

static std::shared_ptr<PoolRequest> make_request(pf_pool *pool, pf_op *op, const pf_params *p, int s, int nev) {
    PF_CHECK(op && p, PF_ERR_INVALID, "null argument");
    PF_CHECK(op->h && op->h->device == pool->device, PF_ERR_INVALID, "operator and pool are on different devices");
    PF_CHECK(s >= 1 && nev >= 1, PF_ERR_INVALID, "s and nev must be positive");
    auto r = std::make_shared<PoolRequest>();
    r->own.reset(bind_op(op, op->h));
    r->op = r->own.get();
    r->params = *p;
    r->s = s;
    r->nev = nev;
    r->footprint = solve_footprint(op, p, s, nev);
    r->cost = expected_cost(op, s, nev);
    r->t_submit = Clock::now();
    return r;
}

static void enqueue(pf_pool *pool, const std::shared_ptr<PoolRequest> &r) {
    {
        std::lock_guard<std::mutex> lock(pool->mu);
        PF_CHECK(!pool->stop, PF_ERR_INVALID, "pool is shutting down");
        r->id = pool->next_id++;
        pool->requests[r->id] = r;
        pool->queue.push_back(r);
        ++pool->submitted;
    }
    pool->cv_work.notify_all();
}

int64_t pool_submit(pf_pool *pool, pf_op *op, const pf_params *p, int s, int nev, const double *x0,
                    double *vecs_out, int vecs_mem) {
    PF_CHECK(pool && x0, PF_ERR_INVALID, "null argument");
    auto r = make_request(pool, op, p, s, nev);
    PF_CHECK(!p->probes, PF_ERR_INVALID, "served requests draw their KPM probes from params.seed");
    r->x0_copy.assign(x0, x0 + (size_t)op->dim * s);
    r->x0 = r->x0_copy.data();
    r->x0_mem = PF_MEM_HOST;
    r->vals.assign(nev, 0.0);
    r->vecs_out = vecs_out;
    r->vecs_mem = vecs_mem;
    enqueue(pool, r);
    return r->id;
}

int pool_solve_batch(pf_pool *pool, int n, pf_op *const *ops, const pf_params *const *params, const int *s,
                     const int *nev, const double *const *x0, int x0_mem, double *const *vals, double *const *vecs,
                     int vecs_mem, pf_report *reports, int *nconv, std::string &first_error) {
    PF_CHECK(pool && n >= 0 && (n == 0 || (ops && params && s && nev && x0 && vals && nconv)), PF_ERR_INVALID,
             "null argument");
    std::vector<std::shared_ptr<PoolRequest>> reqs;
    for (int i = 0; i < n; ++i) {
        auto r = make_request(pool, ops[i], params[i], s[i], nev[i]);
        r->batch = true;
        r->x0 = x0[i];
        r->x0_mem = x0_mem;
        r->vals_out = vals[i];
        r->vecs_out = vecs ? vecs[i] : nullptr;
        r->vecs_mem = vecs_mem;
        r->rep_out = reports ? reports + i : nullptr;
        r->nconv_out = nconv + i;
        reqs.push_back(r);
    }
    for (auto &r : reqs) enqueue(pool, r);
    int status = PF_OK;
    std::unique_lock<std::mutex> lock(pool->mu);
    ++pool->waiters;
    for (auto &r : reqs) {
        pool->cv_done.wait(lock, [&] { return finished(r->state); });
        if (r->status != PF_OK && status == PF_OK) {
            status = r->status;
            first_error = r->error;
        }
        pool->requests.erase(r->id);
    }
    --pool->waiters;
    pool->cv_done.notify_all();
    return status;
}

int pool_poll(pf_pool *pool, int64_t id) {
    std::lock_guard<std::mutex> lock(pool->mu);
    auto it = pool->requests.find(id);
    PF_CHECK(it != pool->requests.end(), PF_ERR_INVALID, "unknown request");
    return it->second->state;
}

int pool_fetch(pf_pool *pool, int64_t id, double timeout_s, double *vals, pf_report *rep, int *nconv,
               std::string &error) {
    std::unique_lock<std::mutex> lock(pool->mu);
    auto it = pool->requests.find(id);
    PF_CHECK(it != pool->requests.end(), PF_ERR_INVALID, "unknown request");
    auto r = it->second;
    PF_CHECK(!r->batch, PF_ERR_INVALID, "batch requests are collected by pf_pool_solve_batch");
    PF_CHECK(!r->cancelled, PF_ERR_INVALID, "request was cancelled");
    auto done = [&] { return finished(r->state); };
    ++pool->waiters;
    bool ok = true;
    if (timeout_s < 0) pool->cv_done.wait(lock, done);
    else ok = pool->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), done);
    --pool->waiters;
    pool->cv_done.notify_all();
    if (!ok) throw Error(PF_ERR_NUMERIC, "request not finished within the timeout");
    pool->requests.erase(id);
    if (r->status != PF_OK) {
        error = r->error;
        if (nconv) *nconv = -r->state;
        return r->status;
    }
    if (vals) std::copy(r->vals.begin(), r->vals.begin() + r->nconv, vals);
    if (rep) *rep = r->rep;
    if (nconv) *nconv = r->nconv;
    return PF_OK;
}

void pool_cancel(pf_pool *pool, int64_t id) {
    std::lock_guard<std::mutex> lock(pool->mu);
    auto it = pool->requests.find(id);
    PF_CHECK(it != pool->requests.end(), PF_ERR_INVALID, "unknown request");
    auto r = it->second;
    r->cancelled = true;
    if (r->state == PF_REQ_QUEUED) {
        pool->queue.erase(std::remove(pool->queue.begin(), pool->queue.end(), r), pool->queue.end());
        pool->requests.erase(it);
    } else if (r->state != PF_REQ_RUNNING) {
        pool->requests.erase(it);
    }
    pool->cv_work.notify_all();
}

int pool_wait(pf_pool *pool, int64_t id, double timeout_s) {
    std::unique_lock<std::mutex> lock(pool->mu);
    auto it = pool->requests.find(id);
    PF_CHECK(it != pool->requests.end(), PF_ERR_INVALID, "unknown request");
    auto r = it->second;
    PF_CHECK(!r->cancelled, PF_ERR_INVALID, "request was cancelled");
    auto done = [&] { return finished(r->state); };
    ++pool->waiters;
    if (timeout_s < 0) pool->cv_done.wait(lock, done);
    else pool->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), done);
    --pool->waiters;
    pool->cv_done.notify_all();
    return r->state;
}

void pool_request_times(pf_pool *pool, int64_t id, double *times) {
    std::lock_guard<std::mutex> lock(pool->mu);
    auto it = pool->requests.find(id);
    PF_CHECK(it != pool->requests.end(), PF_ERR_INVALID, "unknown request");
    const auto &r = it->second;
    auto since = [&](Clock::time_point t) { return std::chrono::duration<double>(t - pool->t_created).count(); };
    times[0] = since(r->t_submit);
    times[1] = r->started ? since(r->t_start) : -1.0;
    times[2] = finished(r->state) ? since(r->t_done) : -1.0;
}

void pool_stats(pf_pool *pool, pf_pool_stats *st) {
    std::lock_guard<std::mutex> lock(pool->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = pool->submitted;
    st->completed = pool->completed;
    st->failed = pool->failed;
    st->rejected = pool->rejected;
    if (pool->engine)
        engine_stats(pool->engine, &st->filter_launches, &st->filter_seconds, &st->filter_bytes,
                     &st->filter_instance_steps);
    st->queued = (int64_t)pool->queue.size();
    st->running = pool->running;
    st->eigenpairs = pool->eigenpairs;
    st->bytes_budget = pool->budget;
    st->bytes_in_use = pool->in_use;
    st->bytes_peak = pool->peak;
    st->busy_seconds =
        pool->busy + (pool->running > 0 ? std::chrono::duration<double>(Clock::now() - pool->busy_since).count() : 0.0);
    std::vector<double> l = pool->latencies;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) {
            const double pos = q * (l.size() - 1);
            const size_t i = (size_t)pos;
            const double f = pos - i;
            return i + 1 < l.size() ? l[i] * (1 - f) + l[i + 1] * f : l[i];
        };
        st->p50_latency = pct(0.50);
        st->p99_latency = pct(0.99);
        double m = 0;
        for (double v : l) m += v;
        st->mean_latency = m / l.size();
    }
}

}  // namespace pf
