// Continuous-batching solve server over the mixed-precision engine.
//
// Client threads queue requests (gauge, kappa, sources, accuracy); one server
// thread owns the GPU work.  Every loop it
//   1. admits queued requests in arrival order while their solve memory fits
//      the budget and the engine has free slots on their lattice,
//   2. runs one chunk of CG iterations for every admitted solve (one launch per
//      phase for all of them),
//   3. retires requests whose solves all finished and hands their solutions to
//      the waiting clients.
// Solves that arrive while others are on the GPU join at the next chunk; the
// engine's batch-invariant reductions make every result independent of the mix.
//
// Locks: the context lock (GPU work) is always taken before the server lock
// (queues); a thread holding the server lock never waits for the context lock.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include "engine_host.h"

namespace hw {

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { REQ_QUEUED, REQ_RUNNING, REQ_DONE };

struct Request {
    uint64_t id = 0;
    int gauge_id = 0;
    double kappa = 0, tol = 0;
    int maxiters = 0;
    int nrhs = 0;
    std::vector<std::vector<double>> src;  // EVEN sites, checkerboard order, 24 doubles each
    std::vector<std::vector<double>> sol;  // same layout, filled on completion
    std::vector<int> slots;
    size_t bytes = 0;
    ReqState state = REQ_QUEUED;
    bool cancel = false;
    hw_request_result res{};
    Clock::time_point t_submit, t_admit;
};

struct GaugeEntry {
    const hw_gauge *gauge = nullptr;
    int dims[4] = {0, 0, 0, 0};
    long V = 0, Vh = 0;
};

// copy the EVEN sites of a canonical (lexicographic) host spinor into
// checkerboard order (even lexicographic sites in increasing order), or back
void gather_even(const GaugeEntry &G, const double *lex, double *cb) {
    size_t n = 0;
    for (int t = 0; t < G.dims[3]; t++)
        for (int z = 0; z < G.dims[2]; z++)
            for (int y = 0; y < G.dims[1]; y++) {
                const long row = (long)G.dims[0] * (y + (long)G.dims[1] * (z + (long)G.dims[2] * t));
                for (int x = (y + z + t) & 1; x < G.dims[0]; x += 2) {
                    std::memcpy(cb + n, lex + (row + x) * 24, 24 * sizeof(double));
                    n += 24;
                }
            }
}
void scatter_even(const GaugeEntry &G, const double *cb, double *lex) {
    std::memset(lex, 0, (size_t)G.V * 24 * sizeof(double));
    size_t n = 0;
    for (int t = 0; t < G.dims[3]; t++)
        for (int z = 0; z < G.dims[2]; z++)
            for (int y = 0; y < G.dims[1]; y++) {
                const long row = (long)G.dims[0] * (y + (long)G.dims[1] * (z + (long)G.dims[2] * t));
                for (int x = (y + z + t) & 1; x < G.dims[0]; x += 2) {
                    std::memcpy(lex + (row + x) * 24, cb + n, 24 * sizeof(double));
                    n += 24;
                }
            }
}

}  // namespace
}  // namespace hw

struct hw_server {
    hw_context *ctx = nullptr;
    std::unique_ptr<hw::Engine> eng;
    hw_server_config cfg{};
    std::vector<hw::GaugeEntry> gauges;
    std::mutex mu;  // guards everything below
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<hw::Request>> queue;
    std::vector<std::shared_ptr<hw::Request>> running;
    std::map<uint64_t, std::shared_ptr<hw::Request>> all;
    std::vector<double> latencies;
    uint64_t next_id = 1;
    hw_server_stats stats{};
    size_t bytes_in_use = 0;
    bool stop = false;
    std::thread worker;
    std::string worker_error;
    hw::DevBuf stage;  // checkerboard AoS staging for one half field
    uint64_t layout_launches = 0;  // AoS <-> SoA kernels of admit / retire
};

namespace hw {
namespace {

// queue -> engine slots (context lock and server lock held)
int admit_waiting(hw_server *S) {
    Engine &E = *S->eng;
    while (!S->queue.empty()) {
        std::shared_ptr<Request> q = S->queue.front();
        if (q->cancel) {
            S->queue.pop_front();
            q->state = REQ_DONE;
            q->res.status = HW_ERR_CANCELLED;
            q->res.nrhs = q->nrhs;
            S->stats.cancelled++;
            S->cv_done.notify_all();
            continue;
        }
        const GaugeEntry &G = S->gauges[q->gauge_id];
        int l;
        int rc = E.lattice_index(G.gauge, &l);
        if (rc != HW_OK) return rc;
        if (E.free_slots_on(l) < q->nrhs) break;  // wait for slots on this lattice (keeps arrival order)
        const size_t need = (size_t)q->nrhs * E.slot_bytes(l);
        if (S->bytes_in_use + need > S->cfg.hbm_budget_bytes) break;  // wait for memory
        S->queue.pop_front();
        q->bytes = need;
        S->bytes_in_use += need;
        q->t_admit = Clock::now();
        hw_context *ctx = S->ctx;
        const int stride = E.lattice(l).stride;
        for (int k = 0; k < q->nrhs; k++) {
            int slot;
            if ((rc = E.admit(l, q->kappa, nullptr, nullptr, q->tol, q->maxiters, S->cfg.delta, ENG_MODE_SOLVE,
                              &slot)) != HW_OK)
                return rc;
            q->slots.push_back(slot);
            // source: host (checkerboard AoS) -> staging -> slot-owned b; x = 0
            HW_CUDA(cudaMemcpyAsync(S->stage.ptr, q->src[k].data(), q->src[k].size() * sizeof(double),
                                    cudaMemcpyHostToDevice, ctx->stream));
            launch_aos_to_soa((int)G.Vh, S->stage.as<double>(), HalfF64{E.own_b(slot), stride}, ctx->stream);
            S->layout_launches++;
            HW_CUDA(cudaMemsetAsync(E.own_x(slot), 0, (size_t)12 * stride * sizeof(double2), ctx->stream));
        }
        q->src.clear();
        q->src.shrink_to_fit();
        q->state = REQ_RUNNING;
        S->running.push_back(q);
    }
    return HW_OK;
}

// finished requests -> host solutions (context lock and server lock held)
int retire_finished(hw_server *S) {
    Engine &E = *S->eng;
    hw_context *ctx = S->ctx;
    for (size_t n = 0; n < S->running.size();) {
        std::shared_ptr<Request> q = S->running[n];
        bool all_done = true;
        for (int slot : q->slots)
            if (E.state(slot).status == ENG_RUNNING) all_done = false;
        if (!all_done && !q->cancel) {
            n++;
            continue;
        }
        const GaugeEntry &G = S->gauges[q->gauge_id];
        int status = HW_OK;
        q->res.nrhs = q->nrhs;
        if (q->cancel) {
            status = HW_ERR_CANCELLED;
            S->stats.cancelled++;
        } else {
            q->sol.resize(q->nrhs);
            for (int k = 0; k < q->nrhs; k++) {
                const int slot = q->slots[k];
                const EngState &s = E.state(slot);
                q->res.iterations = std::max(q->res.iterations, s.iter);
                q->res.reliable_updates = std::max(q->res.reliable_updates, s.n_ru);
                const double tr = s.b2 > 0 ? std::sqrt(s.s2 / s.b2) : 0.0;
                q->res.true_residual = std::max(q->res.true_residual, tr);
                if (s.status == ENG_BREAKDOWN)
                    status = HW_ERR_BREAKDOWN;
                else if (s.status != ENG_CONVERGED && status == HW_OK)
                    status = HW_ERR_NOT_CONVERGED;
                q->sol[k].resize((size_t)G.Vh * 24);
                const int l = E.slot_lattice(slot);
                launch_soa_to_aos((int)G.Vh, HalfF64{E.own_x(slot), E.lattice(l).stride}, S->stage.as<double>(),
                                  ctx->stream);
                S->layout_launches++;
                HW_CUDA(cudaMemcpyAsync(q->sol[k].data(), S->stage.ptr, q->sol[k].size() * sizeof(double),
                                        cudaMemcpyDeviceToHost, ctx->stream));
                HW_CUDA(cudaStreamSynchronize(ctx->stream));
            }
            S->stats.completed++;
            S->stats.solves_completed += q->nrhs;
        }
        for (int slot : q->slots) E.release(slot);
        S->bytes_in_use -= q->bytes;
        q->res.status = status;
        q->res.latency_seconds = std::chrono::duration<double>(Clock::now() - q->t_submit).count();
        q->res.queue_seconds = std::chrono::duration<double>(q->t_admit - q->t_submit).count();
        if (status == HW_OK) S->latencies.push_back(q->res.latency_seconds);
        q->state = REQ_DONE;
        S->running.erase(S->running.begin() + n);
        S->cv_done.notify_all();
    }
    E.prune_lattices();
    return HW_OK;
}

void fail_all(hw_server *S, int rc) {
    S->worker_error = hw_last_error();
    for (auto &q : S->running) {
        for (int slot : q->slots) S->eng->release(slot);
        q->res.status = rc;
        q->state = REQ_DONE;
    }
    S->running.clear();
    for (auto &q : S->queue) {
        q->res.status = rc;
        q->state = REQ_DONE;
    }
    S->queue.clear();
    S->bytes_in_use = 0;
    S->cv_done.notify_all();
}

void server_loop(hw_server *S) {
    cudaSetDevice(S->ctx->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty() || !S->running.empty(); });
            if (S->stop) return;
        }
        std::lock_guard<std::recursive_mutex> glk(S->ctx->mu);
        std::unique_lock<std::mutex> lk(S->mu);
        if (S->stop) return;
        int rc = admit_waiting(S);
        if (rc == HW_OK && !S->running.empty()) {
            rc = S->eng->launch_chunk(S->cfg.chunk_iters);
            if (rc == HW_OK) {
                // clients can submit and wait while the chunk runs on the device
                lk.unlock();
                rc = S->eng->read_states();
                lk.lock();
                // every chunk graph runs one begin kernel, then 11 kernels per loop body
                S->stats.chunks++;
                S->stats.kernel_launches = S->layout_launches + S->stats.chunks + 11 * S->eng->bodies_total();
            }
        }
        if (rc == HW_OK) rc = retire_finished(S);
        if (rc != HW_OK) fail_all(S, rc);
    }
}

}  // namespace
}  // namespace hw

using namespace hw;

extern "C" {

int hw_server_create(hw_context *ctx, const hw_server_config *config, hw_server **out) {
    HW_CHECK_ARG(ctx && out, "null argument");
    *out = nullptr;
    hw_server_config cfg{};
    cfg.precision = HW_PREC_F16;
    if (config) cfg = *config;
    HW_CHECK_ARG(cfg.precision == HW_PREC_F16 || cfg.precision == HW_PREC_F32, "server precision must be F16 or F32");
    if (cfg.delta <= 0) cfg.delta = cfg.precision == HW_PREC_F16 ? 0.005 : 1e-5;
    if (cfg.chunk_iters <= 0) cfg.chunk_iters = 8;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    if (cfg.hbm_budget_bytes == 0) {
        size_t free_b = 0, total_b = 0;
        HW_CUDA(cudaMemGetInfo(&free_b, &total_b));
        cfg.hbm_budget_bytes = (size_t)(0.8 * (double)free_b);
    }
    std::unique_ptr<hw_server> S(new hw_server());
    S->ctx = ctx;
    S->cfg = cfg;
    S->eng.reset(new Engine(ctx, cfg.precision == HW_PREC_F16 ? LOW_F16 : LOW_F32));
    int rc = S->eng->init();
    if (rc != HW_OK) return rc;
    S->stats.bytes_budget = cfg.hbm_budget_bytes;
    hw_server *raw = S.get();
    S->worker = std::thread([raw] { server_loop(raw); });
    *out = S.release();
    return HW_OK;
}

int hw_server_destroy(hw_server *S) {
    if (!S) return HW_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    if (S->worker.joinable()) S->worker.join();
    {
        std::lock_guard<std::recursive_mutex> glk(S->ctx->mu);
        S->eng.reset();
        S->stage.release();
    }
    delete S;
    return HW_OK;
}

int hw_server_add_gauge(hw_server *S, const hw_gauge *gauge, int *gauge_id) {
    HW_CHECK_ARG(S && gauge && gauge_id, "null argument");
    HW_CHECK_ARG(gauge->lat->ctx == S->ctx, "gauge belongs to another context");
    GaugeEntry G;
    G.gauge = gauge;
    for (int d = 0; d < 4; d++) G.dims[d] = gauge->lat->dims[d];
    G.V = gauge->lat->V;
    G.Vh = gauge->lat->Vh;
    std::lock_guard<std::recursive_mutex> glk(S->ctx->mu);
    std::lock_guard<std::mutex> lk(S->mu);
    const size_t need = (size_t)G.Vh * 24 * sizeof(double);
    if (S->stage.bytes < need) {
        HW_CUDA(cudaStreamSynchronize(S->ctx->stream));
        int rc = S->stage.alloc(need);
        if (rc != HW_OK) return rc;
    }
    int rc = ensure_low_links(gauge, S->eng->low(), false);
    if (rc != HW_OK) return rc;
    tune_hop(gauge->lat, gauge);
    S->gauges.push_back(G);
    *gauge_id = (int)S->gauges.size() - 1;
    return HW_OK;
}

int hw_server_submit(hw_server *S, int gauge_id, double kappa, int nrhs, const double *const *sources,
                     double accuracy, int maxiters, uint64_t *request_id) {
    HW_CHECK_ARG(S && sources && request_id, "null argument");
    HW_CHECK_ARG(nrhs >= 1 && nrhs <= kEngMaxRhs, "nrhs must be 1..%d", kEngMaxRhs);
    HW_CHECK_ARG(accuracy > 0 && maxiters > 0, "bad accuracy or maxiters");
    for (int k = 0; k < nrhs; k++) HW_CHECK_ARG(sources[k], "source %d is null", k);
    GaugeEntry G;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        HW_CHECK_ARG(gauge_id >= 0 && gauge_id < (int)S->gauges.size(), "unknown gauge id %d", gauge_id);
        if (!S->worker_error.empty()) {
            set_error("server failed: %s", S->worker_error.c_str());
            return HW_ERR_CUDA;
        }
        G = S->gauges[gauge_id];
    }
    std::shared_ptr<Request> q(new Request());
    q->gauge_id = gauge_id;
    q->kappa = kappa;
    q->tol = accuracy;
    q->maxiters = maxiters;
    q->nrhs = nrhs;
    q->t_submit = Clock::now();
    q->src.resize(nrhs);
    for (int k = 0; k < nrhs; k++) {
        q->src[k].resize((size_t)G.Vh * 24);
        gather_even(G, sources[k], q->src[k].data());
    }
    std::lock_guard<std::mutex> lk(S->mu);
    q->id = S->next_id++;
    S->stats.submitted++;
    S->all[q->id] = q;
    *request_id = q->id;
    // a request that can never fit the budget is rejected now
    const size_t need = (size_t)nrhs * S->eng->slot_bytes_for_stride(padded_stride(G.Vh));
    if (need > S->cfg.hbm_budget_bytes) {
        q->src.clear();
        q->state = REQ_DONE;
        q->res.status = HW_ERR_REJECTED;
        q->res.nrhs = nrhs;
        S->stats.rejected++;
        return HW_OK;
    }
    S->queue.push_back(q);
    S->cv_work.notify_all();
    return HW_OK;
}

int hw_server_wait(hw_server *S, uint64_t request_id, double *const *solutions, double timeout_seconds,
                   hw_request_result *result) {
    HW_CHECK_ARG(S, "null argument");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(request_id);
    HW_CHECK_ARG(it != S->all.end(), "unknown request id %llu", (unsigned long long)request_id);
    std::shared_ptr<Request> q = it->second;
    auto done = [&] { return q->state == REQ_DONE; };
    if (timeout_seconds < 0)
        S->cv_done.wait(lk, done);
    else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_seconds), done)) {
        set_error("request %llu still running", (unsigned long long)request_id);
        return HW_ERR_TIMEOUT;
    }
    if (result) *result = q->res;
    S->all.erase(request_id);
    const GaugeEntry G = S->gauges[q->gauge_id];
    lk.unlock();
    if (solutions && !q->sol.empty())
        for (int k = 0; k < q->nrhs; k++)
            if (solutions[k]) scatter_even(G, q->sol[k].data(), solutions[k]);
    return q->res.status == HW_ERR_CANCELLED || q->res.status == HW_ERR_REJECTED ? q->res.status : HW_OK;
}

int hw_server_cancel(hw_server *S, uint64_t request_id) {
    HW_CHECK_ARG(S, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->all.find(request_id);
    HW_CHECK_ARG(it != S->all.end(), "unknown request id %llu", (unsigned long long)request_id);
    it->second->cancel = true;
    S->cv_work.notify_all();
    return HW_OK;
}

int hw_server_stats_get(hw_server *S, hw_server_stats *out) {
    HW_CHECK_ARG(S && out, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    hw_server_stats st = S->stats;
    st.running = S->running.size();
    st.queued = S->queue.size();
    st.bytes_in_use = S->bytes_in_use;
    st.bytes_budget = S->cfg.hbm_budget_bytes;
    std::vector<double> l = S->latencies;
    std::sort(l.begin(), l.end());
    st.latency_p50_seconds = l.empty() ? 0.0 : l[l.size() / 2];
    st.latency_p99_seconds = l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(0.99 * l.size()))];
    *out = st;
    return HW_OK;
}

}  // extern "C"
