// Mixed-precision and batched solves on the engine (engine.h):
//   * hw_cg_solve / hw_wilson_evenodd_solve with precision FP32 or FP16
//   * hw_batch_solve: many right-hand sides on many lattices in the same launches
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "engine_host.h"

namespace hw {

namespace {

int low_of(int precision) { return precision == HW_PREC_F16 ? LOW_F16 : LOW_F32; }

void fill_result(const EngState &s, double seconds, int chunks, hw_cg_result *R) {
    std::memset(R, 0, sizeof(*R));
    R->iterations = s.iter;
    R->reliable_updates = s.n_ru;
    R->restarts = 0;
    R->rr_relative = s.b2 > 0 ? s.rr / s.b2 : 0.0;
    R->true_residual = s.b2 > 0 ? std::sqrt(s.s2 / s.b2) : 0.0;
    R->seconds = seconds;
    // every loop body launches 10 phase kernels and one control kernel; the
    // first body of a slot is its initial residual (no inner iteration)
    R->kernel_launches = chunks + 11 * (s.iter + 1);
    if (s.status == ENG_CONVERGED)
        R->status = HW_OK;
    else if (s.status == ENG_BREAKDOWN)
        R->status = HW_ERR_BREAKDOWN;
    else
        R->status = HW_ERR_NOT_CONVERGED;
}

}  // namespace

// hw_cg_solve / hw_wilson_evenodd_solve with precision != FP64.  mode 0: normal
// system M^dag M x = src (reference CG semantics), 1: M x = src.
int mixed_solve(const hw_gauge *G, double kappa, const hw_field *src, hw_field *x, int mode, const hw_cg_params &P,
                hw_cg_result *R) {
    hw_context *ctx = G->lat->ctx;
    Engine *E;
    int rc;
    if ((rc = get_engine(ctx, low_of(P.precision), &E)) != HW_OK) return rc;
    int l;
    if ((rc = E->lattice_index(G, &l)) != HW_OK) return rc;
    int slot;
    const int emode = mode == 1 ? ENG_MODE_SOLVE : ENG_MODE_NORMAL;
    if ((rc = E->admit(l, kappa, src->half[0].buf.as<double2>(), x->half[0].buf.as<double2>(), P.accuracy,
                       P.maxiters, P.delta, emode, &slot, 1.0 + P.hasenbusch_mh)) != HW_OK)
        return rc;
    HW_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    int chunks = 0;
    const int max_chunks = P.maxiters / 64 + 16;  // every slot stops by maxiters; this bounds the host loop too
    for (;;) {
        if ((rc = E->launch_chunk(64)) != HW_OK) break;
        chunks++;
        if ((rc = E->read_states()) != HW_OK) break;
        if (E->state(slot).status != ENG_RUNNING) break;
        if (chunks > max_chunks) {
            set_error("mixed-precision solve did not finish within %d chunks", max_chunks);
            rc = HW_ERR_TIMEOUT;
            break;
        }
    }
    if (rc != HW_OK) {
        E->release(slot);
        return rc;
    }
    HW_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    HW_CUDA(cudaEventSynchronize(ctx->ev1));
    float ms = 0;
    HW_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    hw_cg_result tmp;
    fill_result(E->state(slot), ms * 1e-3, chunks, R ? R : &tmp);
    const int status = R ? R->status : tmp.status;
    E->release(slot);
    E->prune_lattices();
    HW_CUDA(cudaMemsetAsync(x->half[1].buf.ptr, 0, x->half[1].buf.bytes, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return status;
}

// Admit requests 0..n-1 in order as slots free up, run chunks of iterations for all
// admitted slots, and collect each result as its slot finishes.  lattice_of(k, &l) finds
// (or adds) request k's lattice entry, admit(k, l, &slot) starts it, finished(k) clears
// what the solve leaves behind (enqueued before the slot is released).  Context lock held.
int drive_batch(hw_context *ctx, Engine *E, int n, long max_chunks, hw_cg_result *results,
                const std::function<int(int, int *)> &lattice_of, const std::function<int(int, int, int *)> &admit,
                const std::function<cudaError_t(int)> &finished) {
    std::vector<int> slot_of(n, -1), done(n, 0);
    int next = 0, finished_n = 0, chunks = 0, rc;
    // on an error, give back the slots still held by this batch
    auto fail = [&](int code) {
        for (int k = 0; k < next; k++)
            if (!done[k] && slot_of[k] >= 0) E->release(slot_of[k]);
        E->prune_lattices();
        return code;
    };
    const auto t0 = std::chrono::steady_clock::now();
    while (finished_n < n) {
        // admit as many waiting requests as there are free slots (in order)
        while (next < n) {
            int l;
            if ((rc = lattice_of(next, &l)) != HW_OK) return fail(rc);
            if (E->free_slots_on(l) <= 0) break;
            int slot;
            if ((rc = admit(next, l, &slot)) != HW_OK) return fail(rc);
            slot_of[next] = slot;
            next++;
        }
        if ((rc = E->launch_chunk(16)) != HW_OK) return fail(rc);
        chunks++;
        if ((rc = E->read_states()) != HW_OK) return fail(rc);
        const double now = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        for (int k = 0; k < next; k++) {
            if (done[k]) continue;
            const EngState &s = E->state(slot_of[k]);
            if (s.status == ENG_RUNNING) continue;
            fill_result(s, now, chunks, &results[k]);
            HW_CUDA(finished(k));
            E->release(slot_of[k]);
            done[k] = 1;
            finished_n++;
        }
        E->prune_lattices();
        if (chunks > max_chunks) {
            set_error("batch solve did not finish within %ld chunks", max_chunks);
            return fail(HW_ERR_TIMEOUT);
        }
        if (next == 0 && n > 0) {
            set_error("batch solve could not admit any request");
            return HW_ERR_INVALID;
        }
    }
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    int status = HW_OK;
    for (int k = 0; k < n; k++)
        if (results[k].status != HW_OK) status = results[k].status;
    return status;
}

}  // namespace hw

using namespace hw;

extern "C" {

int hw_batch_solve(hw_context *ctx, int precision, double delta, const hw_solve_request *reqs, int n,
                   hw_cg_result *results) {
    HW_CHECK_ARG(ctx && reqs && results && n >= 0, "null argument");
    HW_CHECK_ARG(precision == HW_PREC_F32 || precision == HW_PREC_F16, "batched solves run in mixed precision");
    if (delta <= 0) delta = 0.1;
    for (int k = 0; k < n; k++) {
        const hw_solve_request &q = reqs[k];
        HW_CHECK_ARG(q.gauge && q.b && q.x, "request %d: null gauge or field", k);
        HW_CHECK_ARG(q.gauge->lat->ctx == ctx, "request %d: gauge belongs to another context", k);
        HW_CHECK_ARG(q.b->lat == q.gauge->lat && q.x->lat == q.gauge->lat, "request %d: lattice mismatch", k);
        HW_CHECK_ARG(q.b != q.x, "request %d: b and x must differ", k);
        HW_CHECK_ARG(q.accuracy > 0 && q.maxiters > 0, "request %d: bad accuracy or maxiters", k);
        HW_CHECK_ARG(std::isfinite(q.hasenbusch_mh) && q.hasenbusch_mh > -1.0, "request %d: bad hasenbusch_mh", k);
    }
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    Engine *E;
    int rc;
    if ((rc = get_engine(ctx, precision == HW_PREC_F16 ? LOW_F16 : LOW_F32, &E)) != HW_OK) return rc;
    for (int k = 0; k < n; k++) tune_hop(reqs[k].gauge->lat, reqs[k].gauge);
    long max_chunks = 16;
    for (int k = 0; k < n; k++) max_chunks += reqs[k].maxiters / 16 + 2;
    return drive_batch(
        ctx, E, n, max_chunks, results,
        [&](int k, int *l) { return E->lattice_index(reqs[k].gauge, l); },
        [&](int k, int l, int *slot) {
            const hw_solve_request &q = reqs[k];
            return E->admit(l, q.kappa, q.b->half[0].buf.as<double2>(), q.x->half[0].buf.as<double2>(), q.accuracy,
                            q.maxiters, delta, ENG_MODE_SOLVE, slot, 1.0 + q.hasenbusch_mh);
        },
        [&](int k) { return cudaMemsetAsync(reqs[k].x->half[1].buf.ptr, 0, reqs[k].x->half[1].buf.bytes, ctx->stream); });
}

int hw_staggered_batch_solve(hw_context *ctx, const hw_stag_solve_request *reqs, int n, hw_cg_result *results) {
    HW_CHECK_ARG(ctx && reqs && results && n >= 0, "null argument");
    for (int k = 0; k < n; k++) {
        const hw_stag_solve_request &q = reqs[k];
        HW_CHECK_ARG(q.gauge && q.in && q.out, "request %d: null gauge or field", k);
        HW_CHECK_ARG(q.gauge->lat->ctx == ctx, "request %d: gauge belongs to another context", k);
        HW_CHECK_ARG(q.in->lat == q.gauge->lat && q.out->lat == q.gauge->lat, "request %d: lattice mismatch", k);
        HW_CHECK_ARG(q.in != q.out, "request %d: in and out must differ", k);
        HW_CHECK_ARG(q.accuracy > 0 && q.maxiters > 0, "request %d: bad accuracy or maxiters", k);
        HW_CHECK_ARG(std::isfinite(q.mass) && q.mass != 0.0, "request %d: mass must be finite and nonzero", k);
        HW_CHECK_ARG(q.precision == HW_PREC_F64 || q.precision == HW_PREC_F16,
                     "request %d: staggered precision must be HW_PREC_F64 or HW_PREC_F16", k);
    }
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    // staggered slots run their own phases in the engine that also serves FP16 Wilson solves
    Engine *E;
    int rc;
    if ((rc = get_engine(ctx, LOW_F16, &E)) != HW_OK) return rc;
    long max_chunks = 16;
    for (int k = 0; k < n; k++) max_chunks += reqs[k].maxiters / 16 + 2;
    return drive_batch(
        ctx, E, n, max_chunks, results,
        [&](int k, int *l) { return E->lattice_index(reqs[k].gauge, l, FERM_STAGGERED); },
        [&](int k, int l, int *slot) {
            const hw_stag_solve_request &q = reqs[k];
            // FP64 throughout: a reliable update only confirms convergence (delta 0); FP16
            // inner iterations: a reliable update when |r| fell by delta
            // (default 0.05: measured fastest for staggered FP16, whose iterations lose more
            // to FP16 rounding than the Wilson ones at 0.005)
            const double delta = q.precision == HW_PREC_F16 ? (q.delta > 0 ? q.delta : 0.05) : 0.0;
            return E->admit(l, q.mass, q.in->half[0].as<double2>(), q.out->half[0].as<double2>(), q.accuracy,
                            q.maxiters, delta, q.normal ? ENG_MODE_NORMAL : ENG_MODE_SOLVE, slot);
        },
        [&](int k) { return cudaMemsetAsync(reqs[k].out->half[1].ptr, 0, reqs[k].out->half[1].bytes, ctx->stream); });
}

int hw_engine_profile_enable(hw_context *ctx, int enable) {
    HW_CHECK_ARG(ctx, "ctx is null");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    if (enable && !ctx->engine_profile)
        for (Engine *e : ctx->engines)
            if (e) e->reset_profile();
    ctx->engine_profile = enable != 0;
    return HW_OK;
}

int hw_engine_profile_get(hw_context *ctx, int precision, hw_engine_profile *out) {
    HW_CHECK_ARG(ctx && out, "null argument");
    HW_CHECK_ARG(precision == HW_PREC_F32 || precision == HW_PREC_F16, "precision must be HW_PREC_F32 or HW_PREC_F16");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    std::memset(out, 0, sizeof(*out));
    static_assert(HW_ENGINE_PHASES == kEngPhases, "phase count");
    static_assert(HW_ENGINE_WORK_KINDS == kEngWorkKinds, "work kinds");
    if (Engine *e = ctx->engines[low_of(precision)]) e->profile(out->launches, out->ms, &out->work[0][0]);
    return HW_OK;
}

int hw_engine_tuning_get(hw_context *ctx, int precision, hw_engine_tuning *out, int max, int *n) {
    HW_CHECK_ARG(ctx && n && (out || max <= 0), "null argument");
    HW_CHECK_ARG(precision == HW_PREC_F32 || precision == HW_PREC_F16, "precision must be HW_PREC_F32 or HW_PREC_F16");
    static_assert(HW_TUNE_MAX_SHAPES == kTuneMaxShapes, "tuner shapes");
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    *n = 0;
    Engine *e = ctx->engines[low_of(precision)];
    if (!e) return HW_OK;
    const TuneShape *shapes = nullptr;
    const int ns = e->tune_shapes(&shapes);
    if (ns <= 0) return HW_OK;
    for (const auto &kv : e->tuning()) {
        if (*n >= max) break;
        hw_engine_tuning &t = out[(*n)++];
        std::memset(&t, 0, sizeof(t));
        t.work_class = kv.first;
        t.nshapes = ns;
        for (int c = 0; c < ns; c++) {
            t.variant[c] = shapes[c].variant;
            t.dynamic_order[c] = shapes[c].dyn;
            t.ms_per_iteration[c] = kv.second.samples[c] ? kv.second.ms[c] : 0.0;
            t.samples[c] = kv.second.samples[c];
        }
        t.chosen = kv.second.chosen;
    }
    return HW_OK;
}

}  // extern "C"
