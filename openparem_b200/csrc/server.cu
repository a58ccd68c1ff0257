// Serving loop: solve requests (a problem, a frequency list, solver options)
// from many callers run on one GPU with continuous admission.
//
// The reference solves one project per process (OpenParEM3D.cpp:494-555 loops
// over the frequency plan of a single mesh); this loop has no counterpart
// there.  It keeps each problem's operators resident on the device between
// requests and runs up to `slots` requests at once, each on its own slot
// context (own CUDA stream and pinned scratch), so their kernels overlap on
// the GPU.  A queued request is admitted when a slot is free and its device
// footprint (request_bytes_estimate) fits in what the running requests leave
// of the budget; a request is always admitted when nothing runs, so one that
// is larger than the budget still completes.  Admission scans the queue in
// arrival order and takes the first request that fits (a later small request
// may overtake a waiting large one); requests on the same problem never run
// at the same time.  Results do not depend on what else runs: every kernel of
// a request reads only that request's data, and all reductions are
// deterministic.  A request can be cancelled: dropped if still queued, or
// stopped at its next Krylov step through the problem's cancel flag, which
// the FP64 and batched solvers poll between steps.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"

using namespace opem;

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t id = 0;
    opem_problem prob = nullptr;
    std::vector<double> freqs;
    opem_solver_opts opts{};
    double bytes = -1;  // admitted footprint (estimated when the request is first considered)
    bool done = false;
    int status = OPEM_OK;
    std::string error;
    std::vector<double> S;
    std::vector<opem_solve_stats> stats;
    double t_submit = 0, t_start = 0, t_end = 0;
};

}  // namespace

struct opem_server_s {
    int device = 0;
    int nslots = 1;
    double budget = 0;
    double in_use = 0;
    int running = 0;
    int64_t next_id = 1, completed = 0;
    double epoch = 0;
    std::vector<std::unique_ptr<opem_context_s>> slot_ctx;
    std::deque<std::shared_ptr<Request>> queue;
    std::map<int64_t, std::shared_ptr<Request>> table;
    std::set<opem_problem> busy;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    std::vector<std::thread> workers;
};

namespace {

// first queued request that may start now (caller holds the lock).  The
// footprint is estimated here, while no request runs on the problem, so the
// estimate never reads a problem that a worker is assembling.
std::deque<std::shared_ptr<Request>>::iterator pick(opem_server_s* S) {
    for (auto it = S->queue.begin(); it != S->queue.end(); ++it) {
        Request& r = **it;
        if (S->busy.count(r.prob)) continue;
        if (r.bytes < 0) r.bytes = request_bytes_estimate(r.prob->p, (int)r.freqs.size(), r.opts);
        if (S->running == 0 || S->in_use + r.bytes <= S->budget) return it;
    }
    return S->queue.end();
}

void run_request(Request& rq, opem_context_s* slot) {
    Problem& P = rq.prob->p;
    Context* owner = P.ctx;
    const int64_t cap = P.ws_cap;
    P.ctx = &slot->c;   // the request runs on the slot's stream
    P.ws_cap = (int64_t)rq.bytes;
    const int N0 = std::max(1, P.nsports());
    int rc = OPEM_OK;
    if (!P.assembled) rc = opem_problem_assemble(rq.prob);
    if (rc == OPEM_OK) {
        const int N = std::max(1, P.nsports());
        rq.S.assign((size_t)2 * N * N * rq.freqs.size(), 0.0);
        rq.stats.assign(rq.freqs.size(), opem_solve_stats{});
        rc = opem_solve_sweep(rq.prob, (int)rq.freqs.size(), rq.freqs.data(), &rq.opts, rq.S.data(), rq.stats.data());
    } else {
        rq.S.assign((size_t)2 * N0 * N0 * rq.freqs.size(), 0.0);
        rq.stats.assign(rq.freqs.size(), opem_solve_stats{});
    }
    if (rc != OPEM_OK) rq.error = slot->c.last_error;
    rq.status = rc;
    P.ctx = owner;
    P.ws_cap = cap;
}

void worker(opem_server_s* S, int slot) {
    cudaSetDevice(S->device);
    for (;;) {
        std::shared_ptr<Request> rq;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stop || pick(S) != S->queue.end(); });
            if (S->stop) return;
            auto it = pick(S);
            rq = *it;
            S->queue.erase(it);
            S->busy.insert(rq->prob);
            rq->prob->p.cancel.store(0);   // under the lock: a cancel from now on is seen
            S->in_use += rq->bytes;
            ++S->running;
            rq->t_start = now_s();
        }
        run_request(*rq, S->slot_ctx[slot].get());
        {
            std::lock_guard<std::mutex> lk(S->mu);
            rq->t_end = now_s();
            rq->done = true;
            S->busy.erase(rq->prob);
            S->in_use -= rq->bytes;
            --S->running;
            ++S->completed;
        }
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

}  // namespace

extern "C" {

int opem_server_create(int device, int slots, int64_t hbm_budget_bytes, opem_server* out) {
    if (!out || slots < 1 || slots > 64) return OPEM_ERR_ARG;
    *out = nullptr;
    auto S = std::make_unique<opem_server_s>();
    S->device = device;
    S->nslots = slots;
    S->epoch = now_s();
    for (int k = 0; k < slots; ++k) {
        opem_context c = nullptr;
        int rc = opem_context_create(device, &c);
        if (rc != OPEM_OK) {
            for (auto& sc : S->slot_ctx) opem_context_destroy(sc.release());
            return rc;
        }
        S->slot_ctx.emplace_back(c);
    }
    if (hbm_budget_bytes > 0) {
        S->budget = (double)hbm_budget_bytes;
    } else {
        size_t freeb = 0, totb = 0;
        cudaSetDevice(device);
        if (cudaMemGetInfo(&freeb, &totb) != cudaSuccess) {
            for (auto& sc : S->slot_ctx) opem_context_destroy(sc.release());
            return OPEM_ERR_CUDA;
        }
        S->budget = 0.9 * (double)freeb;
    }
    opem_server_s* raw = S.release();
    for (int k = 0; k < slots; ++k) raw->workers.emplace_back(worker, raw, k);
    *out = raw;
    return OPEM_OK;
}

int opem_server_destroy(opem_server srv) {
    if (!srv) return OPEM_ERR_ARG;
    {
        std::unique_lock<std::mutex> lk(srv->mu);
        // queued requests are dropped; running ones finish first
        for (auto& q : srv->queue) {
            q->done = true;
            q->status = OPEM_ERR_STATE;
            q->error = "server destroyed before the request started";
        }
        srv->queue.clear();
        srv->cv_done.wait(lk, [&] { return srv->running == 0; });
        srv->stop = true;
    }
    srv->cv_work.notify_all();
    for (auto& t : srv->workers) t.join();
    for (auto& sc : srv->slot_ctx) opem_context_destroy(sc.release());
    delete srv;
    return OPEM_OK;
}

int opem_server_submit(opem_server srv, opem_problem prob, int nfreq, const double* freqs,
                       const opem_solver_opts* opts, int64_t* request_id) {
    if (!srv || !prob || nfreq <= 0 || !freqs || !opts || !request_id) return OPEM_ERR_ARG;
    if (prob->p.ctx->device != srv->device) return OPEM_ERR_ARG;
    for (int f = 0; f < nfreq; ++f)
        if (!(freqs[f] > 0)) return OPEM_ERR_ARG;
    auto rq = std::make_shared<Request>();
    rq->prob = prob;
    rq->freqs.assign(freqs, freqs + nfreq);
    rq->opts = *opts;
    rq->t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        if (srv->stop) return OPEM_ERR_STATE;
        rq->id = srv->next_id++;
        srv->queue.push_back(rq);
        srv->table[rq->id] = rq;
        *request_id = rq->id;
    }
    srv->cv_work.notify_all();
    return OPEM_OK;
}

int opem_server_wait(opem_server srv, int64_t request_id, double timeout_s, double* S_out, opem_solve_stats* stats,
                     double* times_out) {
    if (!srv) return OPEM_ERR_ARG;
    std::shared_ptr<Request> rq;
    {
        std::unique_lock<std::mutex> lk(srv->mu);
        auto it = srv->table.find(request_id);
        if (it == srv->table.end()) return OPEM_ERR_ARG;
        rq = it->second;
        auto ready = [&] { return rq->done; };
        if (timeout_s < 0) {
            srv->cv_done.wait(lk, ready);
        } else if (!srv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
            return OPEM_ERR_TIMEOUT;   // still queued or running; wait again later
        }
        srv->table.erase(request_id);
    }
    if (S_out && !rq->S.empty()) std::memcpy(S_out, rq->S.data(), rq->S.size() * sizeof(double));
    if (stats)
        for (size_t f = 0; f < rq->stats.size(); ++f) stats[f] = rq->stats[f];
    if (times_out) {
        times_out[0] = rq->t_submit - srv->epoch;
        times_out[1] = rq->t_start - srv->epoch;
        times_out[2] = rq->t_end - srv->epoch;
    }
    return rq->status;
}

int opem_server_cancel(opem_server srv, int64_t request_id) {
    if (!srv) return OPEM_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        auto it = srv->table.find(request_id);
        if (it == srv->table.end()) return OPEM_ERR_ARG;
        std::shared_ptr<Request> rq = it->second;
        if (rq->done) return OPEM_OK;
        auto q = std::find(srv->queue.begin(), srv->queue.end(), rq);
        if (q == srv->queue.end()) {   // running: the solver stops at its next Krylov step
            rq->prob->p.cancel.store(1);
            return OPEM_OK;
        }
        srv->queue.erase(q);
        rq->done = true;
        rq->status = OPEM_ERR_CANCELLED;
        rq->error = "cancelled before it started";
        rq->t_start = rq->t_end = now_s();
    }
    srv->cv_done.notify_all();
    return OPEM_OK;
}

int opem_server_info(opem_server srv, int64_t* info, int ninfo) {
    if (!srv || !info) return OPEM_ERR_ARG;
    std::lock_guard<std::mutex> lk(srv->mu);
    const int64_t v[6] = {(int64_t)srv->queue.size(), srv->running, srv->completed, (int64_t)srv->in_use,
                          (int64_t)srv->budget, srv->nslots};
    for (int i = 0; i < ninfo && i < 6; ++i) info[i] = v[i];
    return OPEM_OK;
}

}  // extern "C"
