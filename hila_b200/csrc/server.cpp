// Continuous-batching solve server over the mixed-precision engine.
//
// Client threads queue requests (gauge, kappa, sources, accuracy); one server
// thread owns the GPU work.  Every loop it
//   1. admits queued requests in arrival order per lattice (a request waiting
//      for slots on its lattice holds back later requests for that lattice
//      only) while their solve memory fits the budget,
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

// where a request's sources come from and its solutions go
enum ReqMode {
    REQ_HOST_LEX,  // host arrays in lexicographic site order (EVEN sites gathered at submit)
    REQ_HOST_EO,   // host arrays in even-first site order: the EVEN half is one contiguous block
    REQ_FIELDS     // device fields: the engine reads b and writes x in place
};

// page-locked host memory (cudaHostAlloc or cudaHostRegister): copied by DMA directly
bool host_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Recycled page-locked host buffers, so source and solution copies run
// asynchronously at full PCIe rate (page-locking memory per request would
// cost more than the copy).
class PinnedPool {
  public:
    void set_keep_bytes(size_t b) { keep_bytes_ = b; }
    ~PinnedPool() {
        for (auto &e : free_) cudaFreeHost(e.second);
    }
    // an idle buffer of n doubles, or null (never allocates)
    double *try_get(size_t n) {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = free_.find(n);
        if (it == free_.end()) return nullptr;
        double *p = it->second;
        free_.erase(it);
        held_ -= n;
        return p;
    }
    double *get(size_t n) {
        if (double *p = try_get(n)) return p;
        void *p = nullptr;
        if (cudaHostAlloc(&p, n * sizeof(double), cudaHostAllocDefault) != cudaSuccess) return nullptr;
        return static_cast<double *>(p);
    }
    void put(double *p, size_t n) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(mu_);
        if ((held_ + n) * sizeof(double) > keep_bytes_) {
            cudaFreeHost(p);
            return;
        }
        free_.emplace(n, p);
        held_ += n;
    }

  private:
    size_t keep_bytes_ = size_t(16) << 30;  // idle buffers kept for reuse (hw_server_config.host_pool_bytes)
    std::mutex mu_;
    std::multimap<size_t, double *> free_;
    size_t held_ = 0;  // doubles in free_
};

struct Request {
    uint64_t id = 0;
    int gauge_id = 0;
    double kappa = 0, tol = 0;
    int maxiters = 0;
    int nrhs = 0;
    PinnedPool *pool = nullptr;
    size_t n = 0;  // doubles per source / solution (EVEN sites x 24)
    // sources, EVEN sites in checkerboard order, in pinned buffers of the pool (each
    // later receives its solution); pageable only if page-locking fails
    std::vector<double *> pin;
    std::vector<std::unique_ptr<double[]>> src;
    std::vector<double *> sol;  // pinned, same layout, filled on completion
    int mode = REQ_HOST_LEX;
    // REQ_HOST_EO: the caller's page-locked sources (read by DMA; null: staged in pin) and
    // solution arrays (written by DMA when page-locked, else copied from sol at wait)
    std::vector<const double *> src_direct;
    std::vector<double *> user_sol;
    std::vector<char> sol_direct;
    // REQ_FIELDS: EVEN halves of the caller's device fields (Wilson or staggered)
    std::vector<double2 *> fb, fx;
    int fermion = FERM_WILSON;
    uint64_t admit_chunk = 0, retire_chunk = 0;  // server chunks launched before admission / retirement
    // entries of its lattice's staging ring holding sources copied to the device while
    // the request waited for slots (host modes); empty: not staged
    std::vector<int> stage;
    const double *source(int k) const {
        if (!src_direct.empty() && src_direct[k]) return src_direct[k];
        return pin[k] ? pin[k] : src[k].get();
    }
    std::vector<int> slots;
    size_t bytes = 0;
    ReqState state = REQ_QUEUED;
    bool cancel = false;
    hw_request_result res{};
    Clock::time_point t_submit, t_admit;
    void release_sources() {  // pinned sources stay until they become solutions
        src.clear();
        src.shrink_to_fit();
    }
    void release_solutions() {
        for (double *p : sol) pool->put(p, n);
        sol.clear();
        for (double *p : pin) pool->put(p, n);
        pin.clear();
    }
    ~Request() {
        release_sources();
        release_solutions();
    }
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
    hw::PinnedPool pool;  // outlives every request (declared before them)
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
    uint64_t layout_launches = 0;  // AoS <-> SoA kernels of admit / retire
    // Host -> device copies and layout conversions of admitted solves run on in_stream,
    // those of retired solves on out_stream, ordered against the engine's stream by
    // events, so they overlap the chunks of the other solves and each other (the two
    // copy directions use separate copy engines).  A retired solution is converted into
    // its slot's staging buffer before it is copied out, so the slot can take a new
    // source as soon as that conversion (conv_event) is done.
    cudaStream_t in_stream = nullptr, out_stream = nullptr;
    cudaEvent_t conv_event = nullptr;
    bool conv_recorded = false;
    // Sources of queued requests are copied to the device ahead of their admission, into
    // a staging ring per gauge field (kEngMaxRhs source buffers, allocated the first time
    // a request of that gauge field waits, kept until the server is destroyed), so the
    // copies overlap the chunks of earlier requests.  An entry is free again as soon as
    // the admission has enqueued its conversion: later copies into it follow on in_stream.
    struct StageRing {
        std::vector<std::unique_ptr<hw::DevBuf>> buf;
        std::vector<int> free_list;
    };
    std::map<int, StageRing> rings;  // by gauge id
    size_t ring_bytes = 0;           // device memory the rings hold (a ring is made only if it fits the budget)
    void release_stage(hw::Request &q) {
        if (q.stage.empty()) return;
        StageRing &R = rings[q.gauge_id];
        for (int e : q.stage) R.free_list.push_back(e);
        q.stage.clear();
    }
    bool take_stage(hw::Request &q) {
        auto it = rings.find(q.gauge_id);
        if (it == rings.end()) {
            const size_t bytes = q.n * sizeof(double), total = bytes * hw::kEngMaxRhs;
            if (bytes_in_use + ring_bytes + total > cfg.hbm_budget_bytes) return false;
            StageRing R;
            for (int e = 0; e < hw::kEngMaxRhs; e++) {
                R.buf.emplace_back(new hw::DevBuf());
                if (R.buf[e]->alloc(bytes) != HW_OK) {
                    hw::clear_error();
                    return false;  // the DevBufs free what was allocated
                }
                R.free_list.push_back(hw::kEngMaxRhs - 1 - e);
            }
            ring_bytes += total;
            it = rings.emplace(q.gauge_id, std::move(R)).first;
        }
        StageRing &R = it->second;
        if ((int)R.free_list.size() < q.nrhs) return false;
        for (int k = 0; k < q.nrhs; k++) {
            q.stage.push_back(R.free_list.back());
            R.free_list.pop_back();
        }
        return true;
    }
    const void *stage_ptr(const hw::Request &q, int k) { return rings[q.gauge_id].buf[q.stage[k]]->ptr; }
    std::vector<cudaEvent_t> free_events;
    struct Round {
        cudaEvent_t done;                                // solutions of `reqs` are on the host
        std::vector<std::shared_ptr<hw::Request>> reqs;
    };
    std::deque<Round> retiring;
    cudaEvent_t event() {
        if (!free_events.empty()) {
            cudaEvent_t e = free_events.back();
            free_events.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        return e;
    }
};

namespace hw {
namespace {

// queue -> engine slots (context lock and server lock held).  Arrival order is
// kept per lattice: a request without enough free slots on its lattice holds
// back the later requests for that lattice, not those for other lattices.  A
// request that does not fit the memory budget stops admission (the budget is
// shared by all lattices).
int admit_waiting(hw_server *S) {
    Engine &E = *S->eng;
    std::vector<int> blocked;  // lattices with a waiting request ahead in the queue
    bool admitted = false;
    for (auto it = S->queue.begin(); it != S->queue.end();) {
        std::shared_ptr<Request> q = *it;
        if (q->cancel) {
            it = S->queue.erase(it);
            S->release_stage(*q);  // later copies into its entries follow its own on in_stream
            q->state = REQ_DONE;
            q->res.status = HW_ERR_CANCELLED;
            q->res.nrhs = q->nrhs;
            S->stats.cancelled++;
            S->cv_done.notify_all();
            continue;
        }
        const GaugeEntry &G = S->gauges[q->gauge_id];
        int l;
        int rc = E.lattice_index(G.gauge, &l, q->fermion);
        if (rc != HW_OK) return rc;
        if (std::find(blocked.begin(), blocked.end(), l) != blocked.end()) {
            ++it;
            continue;
        }
        if (E.free_slots_on(l) < q->nrhs) {
            blocked.push_back(l);
            ++it;
            continue;
        }
        const size_t need = (size_t)q->nrhs * E.slot_bytes(l);
        if (S->bytes_in_use + need > S->cfg.hbm_budget_bytes) break;
        it = S->queue.erase(it);
        // running from here on, so a failure below (fail_all) releases its slots and
        // completes it instead of leaving its waiter behind
        q->state = REQ_RUNNING;
        S->running.push_back(q);
        q->bytes = need;
        S->bytes_in_use += need;
        q->t_admit = Clock::now();
        const int stride = E.lattice(l).stride;
        q->admit_chunk = S->stats.chunks;
        for (int k = 0; k < q->nrhs; k++) {
            int slot;
            if (q->mode == REQ_FIELDS) {
                // the engine reads b and accumulates x in the caller's fields (x: initial guess);
                // FP64 staggered solves: a reliable update only confirms convergence (delta 0)
                const double delta = q->fermion != FERM_STAGGERED ? S->cfg.delta
                                     : S->cfg.staggered_precision == HW_PREC_F16 ? 0.05
                                                                                 : 0.0;
                if ((rc = E.admit(l, q->kappa, q->fb[k], q->fx[k], q->tol, q->maxiters, delta, ENG_MODE_SOLVE,
                                  &slot)) != HW_OK)
                    return rc;
                q->slots.push_back(slot);
                continue;
            }
            if ((rc = E.admit(l, q->kappa, nullptr, nullptr, q->tol, q->maxiters, S->cfg.delta, ENG_MODE_SOLVE,
                              &slot)) != HW_OK)
                return rc;
            q->slots.push_back(slot);
            // source: host (checkerboard AoS) -> the slot's x buffer as staging -> SoA b;
            // then x = 0, on the copy stream (the pageable source is staged by the
            // driver before the call returns, so it can be freed right after)
            if (S->conv_recorded) {  // the slot's x may still be read by a retire conversion
                HW_CUDA(cudaStreamWaitEvent(S->in_stream, S->conv_event, 0));
                S->conv_recorded = false;
            }
            const double *stage;
            if (!q->stage.empty()) {  // copied ahead while the request waited
                stage = static_cast<const double *>(S->stage_ptr(*q, k));
            } else {
                double *st = reinterpret_cast<double *>(E.own_x(slot));
                HW_CUDA(cudaMemcpyAsync(st, q->source(k), q->n * sizeof(double), cudaMemcpyHostToDevice,
                                        S->in_stream));
                stage = st;
            }
            launch_aos_to_soa((int)G.Vh, stage, HalfF64{E.own_b(slot), stride}, S->in_stream);
            S->layout_launches++;
            HW_CUDA(cudaMemsetAsync(E.own_x(slot), 0, (size_t)12 * stride * sizeof(double2), S->in_stream));
        }
        S->release_stage(*q);  // its conversions are enqueued: the entries can take new copies
        q->release_sources();
        admitted = true;
    }
    if (admitted) {  // the next chunk starts after the new sources are in place
        cudaEvent_t e = S->event();
        HW_CUDA(cudaEventRecord(e, S->in_stream));
        HW_CUDA(cudaStreamWaitEvent(S->ctx->stream, e, 0));
        S->free_events.push_back(e);
    }
    // copy the sources of the requests still queued (in arrival order) to the device now,
    // behind the admissions above on the same stream, while the admitted solves run
    for (const std::shared_ptr<Request> &q : S->queue) {
        if (q->cancel || q->mode == REQ_FIELDS || !q->stage.empty()) continue;
        if (!S->take_stage(*q)) continue;  // its ring is full: the next request may use another
        for (int k = 0; k < q->nrhs; k++)
            HW_CUDA(cudaMemcpyAsync(const_cast<void *>(S->stage_ptr(*q, k)), q->source(k), q->n * sizeof(double),
                                    cudaMemcpyHostToDevice, S->in_stream));
    }
    return HW_OK;
}

// finished requests -> host solutions (context lock and server lock held).
// After the engine's stream is done with them, each solution is converted to
// checkerboard AoS in the slot's b buffer (no longer needed) and copied to a
// pinned host buffer on the copy stream, overlapping the next chunk; the
// round's requests complete when its event does (finish_rounds).
int retire_finished(hw_server *S) {
    Engine &E = *S->eng;
    hw_context *ctx = S->ctx;
    std::vector<std::shared_ptr<Request>> done;
    struct Copy {
        double *dst;
        const double *src;
        size_t bytes;
    };
    std::vector<Copy> copies;
    bool ordered = false;
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
            if (!ordered) {
                cudaEvent_t e = S->event();
                HW_CUDA(cudaEventRecord(e, ctx->stream));
                HW_CUDA(cudaStreamWaitEvent(S->out_stream, e, 0));
                S->free_events.push_back(e);
                ordered = true;
            }
            q->sol.assign(q->nrhs, nullptr);
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
                if (q->mode == REQ_FIELDS) continue;  // the solution is in the caller's field
                // the caller's page-locked solution array, or the pinned source buffer (its
                // copy to the device finished earlier on this stream), receives the solution
                double *dst;
                if (q->mode == REQ_HOST_EO && q->sol_direct[k]) {
                    dst = q->user_sol[k];
                } else {
                    q->sol[k] = q->pin[k] ? q->pin[k] : S->pool.get(q->n);
                    q->pin[k] = nullptr;
                    if (!q->sol[k]) {
                        set_error("page-locked host allocation of %zu bytes failed", q->n * sizeof(double));
                        return HW_ERR_OOM;
                    }
                    dst = q->sol[k];
                }
                const int l = E.slot_lattice(slot);
                double *stage = reinterpret_cast<double *>(E.own_xfer(slot));
                launch_soa_to_aos((int)G.Vh, HalfF64{E.own_x(slot), E.lattice(l).stride}, stage, S->out_stream);
                S->layout_launches++;
                copies.push_back({dst, stage, q->n * sizeof(double)});
            }
            S->stats.completed++;
            S->stats.solves_completed += q->nrhs;
        }
        q->retire_chunk = S->stats.chunks;
        q->res.admit_chunk = q->admit_chunk;
        q->res.retire_chunk = q->retire_chunk;
        // a slot's buffers are reused only by copy-stream work queued after these copies
        for (int slot : q->slots) E.release(slot);
        S->bytes_in_use -= q->bytes;
        q->res.status = status;
        done.push_back(q);
        S->running.erase(S->running.begin() + n);
    }
    if (!copies.empty()) {
        // the slots' x buffers are free for new sources once these conversions are done;
        // the copies to the host follow on the same stream
        HW_CUDA(cudaEventRecord(S->conv_event, S->out_stream));
        S->conv_recorded = true;
        for (const Copy &c : copies)
            HW_CUDA(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, S->out_stream));
    }
    if (!done.empty()) {
        hw_server::Round r;
        r.done = S->event();
        HW_CUDA(cudaEventRecord(r.done, S->out_stream));
        r.reqs = std::move(done);
        S->retiring.push_back(std::move(r));
    }
    E.prune_lattices();
    return HW_OK;
}

// Complete the retiring rounds whose copies have finished (server lock held);
// with block, wait for the oldest one first.
int finish_rounds(hw_server *S, bool block) {
    while (!S->retiring.empty()) {
        hw_server::Round &r = S->retiring.front();
        if (block) {
            HW_CUDA(cudaEventSynchronize(r.done));
            block = false;
        } else {
            const cudaError_t e = cudaEventQuery(r.done);
            if (e == cudaErrorNotReady) break;
            HW_CUDA(e);
        }
        const Clock::time_point now = Clock::now();
        for (auto &q : r.reqs) {
            q->res.latency_seconds = std::chrono::duration<double>(now - q->t_submit).count();
            q->res.queue_seconds = std::chrono::duration<double>(q->t_admit - q->t_submit).count();
            if (q->res.status == HW_OK) S->latencies.push_back(q->res.latency_seconds);
            q->state = REQ_DONE;
        }
        S->free_events.push_back(r.done);
        S->retiring.pop_front();
        S->cv_done.notify_all();
    }
    return HW_OK;
}

void fail_all(hw_server *S, int rc) {
    S->worker_error = hw_last_error();
    for (auto &q : S->running) {
        for (int slot : q->slots) S->eng->release(slot);
        S->release_stage(*q);
        q->release_solutions();  // possibly not copied: nothing is handed out
        q->res.status = rc;
        q->state = REQ_DONE;
    }
    S->running.clear();
    for (auto &r : S->retiring) {
        for (auto &q : r.reqs) {
            q->release_solutions();
            q->res.status = rc;
            q->state = REQ_DONE;
        }
        S->free_events.push_back(r.done);
    }
    S->retiring.clear();
    for (auto &q : S->queue) {
        S->release_stage(*q);
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
            S->cv_work.wait(lk, [&] {
                return S->stop || !S->queue.empty() || !S->running.empty() || !S->retiring.empty();
            });
            if (S->stop) return;
        }
        std::lock_guard<std::recursive_mutex> glk(S->ctx->mu);
        std::unique_lock<std::mutex> lk(S->mu);
        if (S->stop) return;
        auto since = [](Clock::time_point t) { return std::chrono::duration<double>(Clock::now() - t).count(); };
        Clock::time_point t0 = Clock::now();
        int rc = admit_waiting(S);
        double dt = since(t0);
        S->stats.seconds_admit += dt;
        S->stats.max_admit_seconds = std::max(S->stats.max_admit_seconds, dt);
        if (rc == HW_OK && !S->running.empty()) {
            t0 = Clock::now();
            rc = S->eng->launch_chunk(S->cfg.chunk_iters);
            S->stats.max_launch_seconds = std::max(S->stats.max_launch_seconds, since(t0));
            if (rc == HW_OK) {
                // clients can submit and wait while the chunk runs on the device
                lk.unlock();
                rc = S->eng->read_states();
                lk.lock();
                // every chunk graph runs one begin kernel, then 11 kernels per loop body
                S->stats.chunks++;
                S->stats.kernel_launches = S->layout_launches + S->stats.chunks + 11 * S->eng->bodies_total();
            }
            S->stats.seconds_run += since(t0);
        }
        t0 = Clock::now();
        if (rc == HW_OK) rc = retire_finished(S);
        // with nothing left on the engine, wait for the oldest copies instead of spinning
        if (rc == HW_OK) rc = finish_rounds(S, S->running.empty() && S->queue.empty());
        dt = since(t0);
        S->stats.seconds_retire += dt;
        S->stats.max_retire_seconds = std::max(S->stats.max_retire_seconds, dt);
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
    HW_CHECK_ARG(cfg.staggered_precision == HW_PREC_F64 ||
                     (cfg.staggered_precision == HW_PREC_F16 && cfg.precision == HW_PREC_F16),
                 "staggered precision must be F64, or F16 on an F16 server");
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
    HW_CUDA(cudaStreamCreateWithFlags(&S->in_stream, cudaStreamNonBlocking));
    HW_CUDA(cudaStreamCreateWithFlags(&S->out_stream, cudaStreamNonBlocking));
    HW_CUDA(cudaEventCreateWithFlags(&S->conv_event, cudaEventDisableTiming));
    if (cfg.host_pool_bytes) S->pool.set_keep_bytes(cfg.host_pool_bytes);
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
        cudaSetDevice(S->ctx->device);
        for (cudaStream_t st : {S->in_stream, S->out_stream})
            if (st) cudaStreamSynchronize(st);
        S->rings.clear();  // the staging rings (streams synchronised above)
        S->eng.reset();
        for (auto &r : S->retiring) S->free_events.push_back(r.done);
        S->retiring.clear();
        for (cudaEvent_t e : S->free_events) cudaEventDestroy(e);
        S->free_events.clear();
        for (cudaStream_t st : {S->in_stream, S->out_stream})
            if (st) cudaStreamDestroy(st);
        if (S->conv_event) cudaEventDestroy(S->conv_event);
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
    int rc = ensure_low_links(gauge, S->eng->low(), S->eng->full18());
    if (rc != HW_OK) return rc;
    tune_hop(gauge->lat, gauge);
    S->gauges.push_back(G);
    *gauge_id = (int)S->gauges.size() - 1;
    // slots sized for the largest lattice when every slot fits in half the budget: a slot
    // then takes any lattice without allocating (allocation stalls the device mid-stream)
    int max_stride = 0;
    for (const GaugeEntry &e : S->gauges) max_stride = std::max(max_stride, padded_stride(e.Vh));
    const size_t all_slots = (size_t)kEngMaxProb * S->eng->slot_bytes_for_stride(max_stride);
    S->eng->set_min_stride(all_slots <= S->cfg.hbm_budget_bytes / 2 ? max_stride : 0);
    return HW_OK;
}

}  // extern "C"

namespace hw {
namespace {

// checks shared by every submit form; G receives the gauge's lattice
int submit_check(hw_server *S, int gauge_id, int nrhs, double accuracy, int maxiters, GaugeEntry *G) {
    HW_CHECK_ARG(nrhs >= 1 && nrhs <= kEngMaxRhs, "nrhs must be 1..%d", kEngMaxRhs);
    HW_CHECK_ARG(accuracy > 0 && maxiters > 0, "bad accuracy or maxiters");
    std::lock_guard<std::mutex> lk(S->mu);
    HW_CHECK_ARG(gauge_id >= 0 && gauge_id < (int)S->gauges.size(), "unknown gauge id %d", gauge_id);
    if (!S->worker_error.empty()) {
        set_error("server failed: %s", S->worker_error.c_str());
        return HW_ERR_CUDA;
    }
    *G = S->gauges[gauge_id];
    return HW_OK;
}

std::shared_ptr<Request> new_request(hw_server *S, const GaugeEntry &G, int gauge_id, double kappa, int nrhs,
                                      double accuracy, int maxiters, int mode) {
    std::shared_ptr<Request> q(new Request());
    q->gauge_id = gauge_id;
    q->kappa = kappa;
    q->tol = accuracy;
    q->maxiters = maxiters;
    q->nrhs = nrhs;
    q->mode = mode;
    q->t_submit = Clock::now();
    q->pool = &S->pool;
    q->n = (size_t)G.Vh * 24;
    q->pin.assign(nrhs, nullptr);
    q->src.resize(nrhs);
    return q;
}

// queue a request (or reject one that can never fit the memory budget)
int enqueue_request(hw_server *S, const GaugeEntry &G, std::shared_ptr<Request> q, uint64_t *request_id) {
    std::lock_guard<std::mutex> lk(S->mu);
    q->id = S->next_id++;
    S->stats.submitted++;
    S->all[q->id] = q;
    *request_id = q->id;
    const size_t need = (size_t)q->nrhs * S->eng->slot_bytes_for_stride(padded_stride(G.Vh));
    if (need > S->cfg.hbm_budget_bytes) {
        q->release_sources();
        q->state = REQ_DONE;
        q->res.status = HW_ERR_REJECTED;
        q->res.nrhs = q->nrhs;
        S->stats.rejected++;
        return HW_OK;
    }
    S->queue.push_back(q);
    S->cv_work.notify_all();
    return HW_OK;
}

}  // namespace
}  // namespace hw

extern "C" {

int hw_server_submit(hw_server *S, int gauge_id, double kappa, int nrhs, const double *const *sources,
                     double accuracy, int maxiters, uint64_t *request_id) {
    HW_CHECK_ARG(S && sources && request_id, "null argument");
    GaugeEntry G;
    int rc = submit_check(S, gauge_id, nrhs, accuracy, maxiters, &G);
    if (rc != HW_OK) return rc;
    for (int k = 0; k < nrhs; k++) HW_CHECK_ARG(sources[k], "source %d is null", k);
    std::shared_ptr<Request> q = new_request(S, G, gauge_id, kappa, nrhs, accuracy, maxiters, REQ_HOST_LEX);
    for (int k = 0; k < nrhs; k++) {
        double *dst = q->pin[k] = S->pool.get(q->n);
        if (!dst) {
            q->src[k].reset(new double[q->n]);
            dst = q->src[k].get();
        }
        gather_even(G, sources[k], dst);
    }
    return enqueue_request(S, G, q, request_id);
}

int hw_server_submit_eo(hw_server *S, int gauge_id, double kappa, int nrhs, const double *const *sources,
                        double *const *solutions, double accuracy, int maxiters, uint64_t *request_id) {
    HW_CHECK_ARG(S && sources && request_id, "null argument");
    GaugeEntry G;
    int rc = submit_check(S, gauge_id, nrhs, accuracy, maxiters, &G);
    if (rc != HW_OK) return rc;
    for (int k = 0; k < nrhs; k++) HW_CHECK_ARG(sources[k], "source %d is null", k);
    std::shared_ptr<Request> q = new_request(S, G, gauge_id, kappa, nrhs, accuracy, maxiters, REQ_HOST_EO);
    q->src_direct.assign(nrhs, nullptr);
    q->user_sol.assign(nrhs, nullptr);
    if (solutions) q->user_sol.assign(solutions, solutions + nrhs);
    q->sol_direct.assign(nrhs, 0);
    for (int k = 0; k < nrhs; k++) {
        q->sol_direct[k] = q->user_sol[k] && host_pinned(q->user_sol[k]) ? 1 : 0;
        if (host_pinned(sources[k])) {
            q->src_direct[k] = sources[k];  // read by DMA at admission
            // the page-locked buffer that receives the solution is taken here, on the
            // caller's thread, not by the server thread at retirement
            if (!q->sol_direct[k]) q->pin[k] = S->pool.get(q->n);
            continue;
        }
        // pageable: one contiguous copy of the EVEN half into a page-locked buffer
        double *dst = q->pin[k] = S->pool.get(q->n);
        if (!dst) {
            q->src[k].reset(new double[q->n]);
            dst = q->src[k].get();
        }
        std::memcpy(dst, sources[k], q->n * sizeof(double));
    }
    return enqueue_request(S, G, q, request_id);
}

int hw_server_submit_fields(hw_server *S, int gauge_id, double kappa, int nrhs, const hw_field *const *sources,
                            hw_field *const *solutions, double accuracy, int maxiters, uint64_t *request_id) {
    HW_CHECK_ARG(S && sources && solutions && request_id, "null argument");
    GaugeEntry G;
    int rc = submit_check(S, gauge_id, nrhs, accuracy, maxiters, &G);
    if (rc != HW_OK) return rc;
    std::shared_ptr<Request> q = new_request(S, G, gauge_id, kappa, nrhs, accuracy, maxiters, REQ_FIELDS);
    for (int k = 0; k < nrhs; k++) {
        HW_CHECK_ARG(sources[k] && solutions[k], "source or solution field %d is null", k);
        HW_CHECK_ARG(sources[k]->lat == G.gauge->lat && solutions[k]->lat == G.gauge->lat,
                     "field %d belongs to another lattice than the gauge field", k);
        HW_CHECK_ARG(sources[k] != solutions[k], "source and solution %d are the same field", k);
        q->fb.push_back(const_cast<double2 *>(sources[k]->half[0].buf.as<double2>()));
        q->fx.push_back(solutions[k]->half[0].buf.as<double2>());
    }
    return enqueue_request(S, G, q, request_id);
}

int hw_server_submit_staggered(hw_server *S, int gauge_id, double mass, int nrhs, const hw_stag_field *const *sources,
                               hw_stag_field *const *solutions, double accuracy, int maxiters, uint64_t *request_id) {
    HW_CHECK_ARG(S && sources && solutions && request_id, "null argument");
    HW_CHECK_ARG(std::isfinite(mass) && mass != 0.0, "mass must be finite and nonzero");
    GaugeEntry G;
    int rc = submit_check(S, gauge_id, nrhs, accuracy, maxiters, &G);
    if (rc != HW_OK) return rc;
    std::shared_ptr<Request> q = new_request(S, G, gauge_id, mass, nrhs, accuracy, maxiters, REQ_FIELDS);
    q->fermion = FERM_STAGGERED;
    for (int k = 0; k < nrhs; k++) {
        HW_CHECK_ARG(sources[k] && solutions[k], "source or solution field %d is null", k);
        HW_CHECK_ARG(sources[k]->lat == G.gauge->lat && solutions[k]->lat == G.gauge->lat,
                     "field %d belongs to another lattice than the gauge field", k);
        HW_CHECK_ARG(sources[k] != solutions[k], "source and solution %d are the same field", k);
        q->fb.push_back(const_cast<double2 *>(sources[k]->half[0].as<double2>()));
        q->fx.push_back(solutions[k]->half[0].as<double2>());
    }
    return enqueue_request(S, G, q, request_id);
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
    if (q->mode == REQ_HOST_EO && !q->sol.empty()) {
        // solutions not written by DMA at retirement (pageable arrays, or arrays given only
        // here): the EVEN half, in even-first order
        for (int k = 0; k < q->nrhs; k++) {
            double *dst = q->user_sol[k] ? q->user_sol[k] : (solutions ? solutions[k] : nullptr);
            if (!q->sol_direct[k] && q->sol[k] && dst) std::memcpy(dst, q->sol[k], q->n * sizeof(double));
        }
    } else if (q->mode == REQ_HOST_LEX && solutions && !q->sol.empty()) {
        for (int k = 0; k < q->nrhs; k++)
            if (solutions[k]) scatter_even(G, q->sol[k], solutions[k]);
    }
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
