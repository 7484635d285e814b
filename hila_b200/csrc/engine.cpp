// Host side of the batched mixed-precision CG engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "engine_host.h"

namespace hw {

int ensure_low_links(const hw_gauge *G, int low, bool full18) {
    hw_lattice *lat = G->lat;
    hw_context *ctx = lat->ctx;
    const size_t st = lat->stride;
    int rc;
    const double2 *l64 = G->f64.as<double2>();
    const int planes = G->U().planes;
    if (low == LOW_F32 && full18) {
        if (!G->f32a.ptr) {
            if ((rc = G->f32a.alloc(32 * st * sizeof(float4))) != HW_OK) return rc;
            if ((rc = G->f32b.alloc(8 * st * sizeof(float2))) != HW_OK) return rc;
            eng_convert_links(lat->g, l64, planes, lat->stride, nullptr, nullptr, nullptr, G->f32a.as<float4>(),
                              G->f32b.as<float2>(), nullptr, nullptr, ctx->stream);
        }
    } else if (low == LOW_F32) {
        if (!G->f32.ptr) {
            if ((rc = G->f32.alloc(24 * st * sizeof(float4))) != HW_OK) return rc;
            eng_convert_links(lat->g, l64, planes, lat->stride, G->f32.as<float4>(), nullptr, nullptr, nullptr,
                              nullptr, nullptr, nullptr, ctx->stream);
        }
    } else if (full18) {
        if (!G->f16x.ptr) {
            if ((rc = G->f16x.alloc(16 * st * sizeof(uint4))) != HW_OK) return rc;
            if ((rc = G->f16z.alloc(8 * st * sizeof(unsigned))) != HW_OK) return rc;
            eng_convert_links(lat->g, l64, planes, lat->stride, nullptr, nullptr, nullptr, nullptr, nullptr,
                              G->f16x.as<uint4>(), G->f16z.as<unsigned>(), ctx->stream);
        }
    } else if (!G->f16a.ptr) {
        if ((rc = G->f16a.alloc(8 * st * sizeof(uint4))) != HW_OK) return rc;
        if ((rc = G->f16b.alloc(8 * st * sizeof(uint2))) != HW_OK) return rc;
        eng_convert_links(lat->g, l64, planes, lat->stride, nullptr, G->f16a.as<uint4>(), G->f16b.as<uint2>(),
                          nullptr, nullptr, nullptr, nullptr, ctx->stream);
    }
    HW_CUDA(cudaGetLastError());
    return HW_OK;
}

Engine::~Engine() {
    if (ctx_) {
        cudaSetDevice(ctx_->device);
        cudaStreamSynchronize(ctx_->stream);
    }
    if (chunk_exec_) cudaGraphExecDestroy(chunk_exec_);
    if (pinned_states_) cudaFreeHost(pinned_states_);
    if (pinned_ctl_) cudaFreeHost(pinned_ctl_);
    if (pinned_work_) cudaFreeHost(pinned_work_);
    for (cudaEvent_t e : prof_ev_)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : tune_ev_)
        if (e) cudaEventDestroy(e);
}

int Engine::init() {
    if (ready_) return HW_OK;
    int rc;
    if ((rc = d_tables_.alloc(sizeof(EngTables))) != HW_OK) return rc;
    if ((rc = d_states_.alloc(sizeof(EngState) * kEngMaxProb)) != HW_OK) return rc;
    if ((rc = d_tickets_.alloc(sizeof(unsigned) * kEngMaxLat)) != HW_OK) return rc;
    if ((rc = d_ctl_.alloc(sizeof(int) * 8)) != HW_OK) return rc;
    if ((rc = d_work_.alloc(sizeof(unsigned long long) * kEngPhases * kEngWorkKinds)) != HW_OK) return rc;
    if ((rc = d_sched_.alloc(sizeof(int) * kEngPhases)) != HW_OK) return rc;
    HW_CUDA(cudaMemsetAsync(d_sched_.ptr, 0, d_sched_.bytes, ctx_->stream));
    HW_CUDA(cudaMemsetAsync(d_tickets_.ptr, 0, d_tickets_.bytes, ctx_->stream));
    HW_CUDA(cudaMemsetAsync(d_ctl_.ptr, 0, d_ctl_.bytes, ctx_->stream));
    HW_CUDA(cudaMemsetAsync(d_work_.ptr, 0, d_work_.bytes, ctx_->stream));
    HW_CUDA(cudaMallocHost(&pinned_states_, sizeof(EngState) * kEngMaxProb));
    HW_CUDA(cudaMallocHost(&pinned_ctl_, sizeof(int) * 8));
    HW_CUDA(cudaMallocHost(&pinned_work_, d_work_.bytes));
    std::memset(pinned_work_, 0, d_work_.bytes);
    std::memset(&tables_, 0, sizeof(tables_));
    // dynamic tile order of the inner phases until launch_chunk picks the chunk's shape
    tables_.dyn = 1;
    for (int j = 0; j < kEngMaxProb; j++) {
        std::memset(&host_states_[j], 0, sizeof(EngState));
        host_states_[j].status = ENG_IDLE;
    }
    HW_CUDA(cudaMemcpyAsync(d_states_.ptr, host_states_, sizeof(host_states_), cudaMemcpyHostToDevice, ctx_->stream));
    // inner links: FP16 engines read all 18 reals (no third-row rebuild in the hop,
    // measured fastest), FP32 engines the 12-real links (fewest bytes);
    // HW_ENGINE_LINKS=12 / 18 overrides.  The tensor-core variant needs 18-real FP16 links.
    full18_ = low_ == LOW_F16;
    if (const char *env = std::getenv("HW_ENGINE_LINKS")) full18_ = std::atoi(env) == 18;
    if (const char *env = std::getenv("HW_ENGINE_VARIANT"))
        if (std::atoi(env) == 4 && low_ == LOW_F16) full18_ = true;
    grid_ = eng_grid_size(low_, default_variant(), full18_ ? 1 : 0, 1);
    // HW_USE_GRAPH=0 runs the iterations from a host loop instead of the captured
    // WHILE graph (profilers see the individual kernel launches)
    if (const char *env = std::getenv("HW_USE_GRAPH")) use_graph_ = std::atoi(env) != 0;
    if ((rc = ensure_partials()) != HW_OK) return rc;
    ready_ = true;
    return HW_OK;
}

int Engine::ensure_partials() {
    size_t need = std::max<size_t>(tables_.max_tiles, 1);
    if (d_partials_.ptr && partial_tiles_ >= need) return HW_OK;
    size_t cap = std::max<size_t>(need, 1024);
    HW_CUDA(cudaStreamSynchronize(ctx_->stream));
    int rc = d_partials_.alloc(sizeof(double) * 2 * kEngMaxProb * cap);
    if (rc != HW_OK) return rc;
    partial_tiles_ = cap;
    if (chunk_exec_) {  // pointer changed: rebuild the graph
        cudaGraphExecDestroy(chunk_exec_);
        chunk_exec_ = nullptr;
    }
    return HW_OK;
}

int Engine::lattice_index(const hw_gauge *G, int *idx, int fermion) {
    HW_CHECK_ARG(fermion == FERM_WILSON || fermion == FERM_STAGGERED, "unknown fermion kind %d", fermion);
    for (int l = 0; l < tables_.nlat; l++)
        if (gauges_[l] == G && tables_.lat[l].fermion == fermion) {
            *idx = l;
            return HW_OK;
        }
    HW_CHECK_ARG(tables_.nlat < kEngMaxLat, "engine holds %d lattices already", kEngMaxLat);
    int rc;
    // staggered solves run in FP64 and need no low-precision links
    if (fermion == FERM_WILSON && (rc = ensure_low_links(G, low_, full18_)) != HW_OK) return rc;
    hw_lattice *lat = G->lat;
    const int l = tables_.nlat;
    EngLattice &L = tables_.lat[l];
    std::memset(&L, 0, sizeof(L));
    L.fermion = fermion;
    L.g = lat->g;
    L.stride = lat->stride;
    L.ntiles = (int)((lat->Vh + kEngTile - 1) / kEngTile);
    L.tile0 = tables_.ntiles;
    L.nprob = 0;
    L.l64 = G->f64.as<double2>();
    L.l64_planes = G->U().planes;
    L.l32 = G->f32.as<float4>();
    L.l16a = G->f16a.as<uint4>();
    L.l16b = G->f16b.as<uint2>();
    L.l32a = G->f32a.as<float4>();
    L.l32b = G->f32b.as<float2>();
    L.l16x = G->f16x.as<uint4>();
    L.l16z = G->f16z.as<unsigned>();
    tables_.ntiles += L.ntiles;
    tables_.max_tiles = std::max(tables_.max_tiles, L.ntiles);
    tables_.nlat = l + 1;
    gauges_.push_back(G);
    tables_dirty_ = true;
    if ((rc = ensure_partials()) != HW_OK) return rc;
    *idx = l;
    return HW_OK;
}

int Engine::prune_lattices() {
    // keep lattices that still have used slots; renumber them and their slots
    std::vector<int> keep;
    for (int l = 0; l < tables_.nlat; l++) {
        bool used = false;
        for (int j = 0; j < kEngMaxProb; j++)
            if (slots_[j].used && slots_[j].lat == l) used = true;
        if (used) keep.push_back(l);
    }
    if ((int)keep.size() == tables_.nlat) return HW_OK;
    EngTables nt;
    std::memset(&nt, 0, sizeof(nt));
    nt.dyn = tables_.dyn;
    std::vector<const hw_gauge *> ng;
    std::vector<int> remap(tables_.nlat, -1);
    for (int l : keep) {
        const int k = nt.nlat++;
        remap[l] = k;
        nt.lat[k] = tables_.lat[l];
        nt.lat[k].tile0 = nt.ntiles;
        nt.ntiles += nt.lat[k].ntiles;
        nt.max_tiles = std::max(nt.max_tiles, nt.lat[k].ntiles);
        ng.push_back(gauges_[l]);
    }
    std::memcpy(nt.prob, tables_.prob, sizeof(nt.prob));
    for (int j = 0; j < kEngMaxProb; j++) {
        if (slots_[j].lat >= 0) slots_[j].lat = remap[slots_[j].lat];
        if (!slots_[j].used) slots_[j].lat = -1;
        nt.prob[j].lat = slots_[j].lat;
    }
    tables_ = nt;
    gauges_ = ng;
    tables_dirty_ = true;
    return HW_OK;
}

int Engine::free_slots_on(int lat) const {
    int used = 0, free_total = 0;
    for (int j = 0; j < kEngMaxProb; j++) {
        if (slots_[j].used) {
            if (slots_[j].lat == lat) used++;
        } else {
            free_total++;
        }
    }
    return std::min(kEngMaxRhs - used, free_total);
}

size_t Engine::slot_bytes_for_stride(int stride) const {
    const size_t st = stride;
    const size_t low_site = low_ == LOW_F16 ? (48 + 4) : 96;
    // p, r, Dp, t (low) + y (FP32) + s, t64 (FP64) + owned x, b and solution staging (FP64)
    return st * (4 * low_site + 96 + 2 * 192) + st * 3 * 192;
}

size_t Engine::slot_bytes(int lat) const { return slot_bytes_for_stride(tables_.lat[lat].stride); }

size_t Engine::buffer_bytes(const SlotBuffers &B) {
    size_t n = 0;
    for (const DevBuf *d : {&B.p, &B.r, &B.Dp, &B.t, &B.pn, &B.rn, &B.Dpn, &B.tn, &B.y, &B.s, &B.t64, &B.x_own,
                            &B.b_own, &B.xfer})
        n += d->bytes;
    return n;
}

void Engine::park_buffers(std::unique_ptr<SlotBuffers> B) {
    const size_t n = buffer_bytes(*B);
    if (idle_bytes_ + n > kIdleCapBytes) return;  // freed here (the DevBufs release themselves)
    idle_bytes_ += n;
    idle_bufs_.emplace(B->stride, std::move(B));
}

void Engine::free_idle() {
    if (idle_bufs_.empty()) return;
    cudaStreamSynchronize(ctx_->stream);
    idle_bufs_.clear();
    idle_bytes_ = 0;
}

int Engine::ensure_slot_buffers(int slot, int stride) {
    std::unique_ptr<SlotBuffers> &cur = bufs_[slot];
    if (cur && cur->stride >= stride && cur->p.ptr) return HW_OK;
    if (cur && cur->p.ptr) park_buffers(std::move(cur));
    // the smallest idle set that is large enough
    auto it = idle_bufs_.lower_bound(stride);
    if (it != idle_bufs_.end()) {
        idle_bytes_ -= buffer_bytes(*it->second);
        cur = std::move(it->second);
        idle_bufs_.erase(it);
        return HW_OK;
    }
    if (stride < min_stride_) stride = min_stride_;
    int rc = alloc_slot_buffers(cur, stride);
    if (rc == HW_ERR_OOM && !idle_bufs_.empty()) {  // give the idle sets back and try once more
        clear_error();
        free_idle();
        rc = alloc_slot_buffers(cur, stride);
    }
    if (rc != HW_OK) cur.reset();  // no half-made set stays with the slot
    return rc;
}

int Engine::alloc_slot_buffers(std::unique_ptr<SlotBuffers> &cur, int stride) {
    cur.reset(new SlotBuffers());
    SlotBuffers &B = *cur;
    const size_t st = stride;
    int rc;
    if (low_ == LOW_F16) {
        for (DevBuf *d : {&B.p, &B.r, &B.Dp, &B.t})
            if ((rc = d->alloc(3 * st * sizeof(uint4))) != HW_OK) return rc;
        for (DevBuf *d : {&B.pn, &B.rn, &B.Dpn, &B.tn})
            if ((rc = d->alloc(st * sizeof(float))) != HW_OK) return rc;
    } else {
        for (DevBuf *d : {&B.p, &B.r, &B.Dp, &B.t})
            if ((rc = d->alloc(6 * st * sizeof(float4))) != HW_OK) return rc;
        for (DevBuf *d : {&B.pn, &B.rn, &B.Dpn, &B.tn}) d->release();
    }
    if ((rc = B.y.alloc(6 * st * sizeof(float4))) != HW_OK) return rc;
    if ((rc = B.s.alloc(12 * st * sizeof(double2))) != HW_OK) return rc;
    if ((rc = B.t64.alloc(12 * st * sizeof(double2))) != HW_OK) return rc;
    B.stride = stride;
    return HW_OK;
}

int Engine::ensure_own(int slot) {
    SlotBuffers &B = *bufs_[slot];
    const size_t bytes = 12 * (size_t)B.stride * sizeof(double2);
    int rc;
    if (!B.x_own.ptr || B.x_own.bytes < bytes)
        if ((rc = B.x_own.alloc(bytes)) != HW_OK) return rc;
    if (!B.b_own.ptr || B.b_own.bytes < bytes)
        if ((rc = B.b_own.alloc(bytes)) != HW_OK) return rc;
    if (!B.xfer.ptr || B.xfer.bytes < bytes)
        if ((rc = B.xfer.alloc(bytes)) != HW_OK) return rc;
    return HW_OK;
}

int Engine::admit(int lat, double kappa, double2 *b, double2 *x, double tol, int maxiter, double delta, int mode,
                  int *slot_out, double diag) {
    HW_CHECK_ARG(lat >= 0 && lat < tables_.nlat, "bad lattice index");
    EngLattice &L = tables_.lat[lat];
    HW_CHECK_ARG(L.nprob < kEngMaxRhs, "lattice holds %d solves already", kEngMaxRhs);
    // a free slot whose buffers fit the lattice with the least to spare, else the first free one
    int slot = -1, fit = -1;
    for (int j = 0; j < kEngMaxProb; j++) {
        if (slots_[j].used) continue;
        if (slot < 0) slot = j;
        const SlotBuffers *B = bufs_[j].get();
        if (B && B->p.ptr && B->stride >= L.stride && (fit < 0 || B->stride < bufs_[fit]->stride)) fit = j;
    }
    if (fit >= 0) slot = fit;
    HW_CHECK_ARG(slot >= 0, "no free solve slot (%d in use)", kEngMaxProb);
    int rc;
    // a staggered solve with a reliable-update factor runs its inner iterations in FP16
    // (engine_stag.cuh), which reads the 18-real FP16 links
    const bool stag_low = L.fermion == FERM_STAGGERED && delta > 0.0;
    if (stag_low) {
        HW_CHECK_ARG(low_ == LOW_F16 && full18_, "low-precision staggered solves need the FP16 engine with 18-real links");
        if ((rc = ensure_low_links(gauges_[lat], low_, full18_)) != HW_OK) return rc;
        L.l16x = gauges_[lat]->f16x.as<uint4>();
        L.l16z = gauges_[lat]->f16z.as<unsigned>();
    }
    if ((rc = ensure_slot_buffers(slot, L.stride)) != HW_OK) return rc;
    SlotBuffers &B = *bufs_[slot];
    if (!b || !x) {
        if ((rc = ensure_own(slot)) != HW_OK) return rc;
        if (!b) b = B.b_own.as<double2>();
        if (!x) x = B.x_own.as<double2>();
    }
    EngProblem &P = tables_.prob[slot];
    std::memset(&P, 0, sizeof(P));
    P.lat = lat;
    P.mode = mode;
    P.stag_low = stag_low ? 1 : 0;
    P.kappa = kappa;
    P.diag = diag;
    P.p = B.p.ptr;
    P.r = B.r.ptr;
    P.Dp = B.Dp.ptr;
    P.t = B.t.ptr;
    P.pn = B.pn.as<float>();
    P.rn = B.rn.as<float>();
    P.Dpn = B.Dpn.as<float>();
    P.tn = B.tn.as<float>();
    P.y = B.y.as<float4>();
    P.x = x;
    P.b = b;
    P.s = B.s.as<double2>();
    P.t64 = B.t64.as<double2>();
    L.prob[L.nprob++] = slot;
    slots_[slot].used = true;
    slots_[slot].lat = lat;
    tables_dirty_ = true;

    EngState &S = host_states_[slot];
    std::memset(&S, 0, sizeof(S));
    S.status = ENG_RUNNING;
    S.mode = mode;
    S.fermion = stag_low ? FERM_STAGGERED_LOW : L.fermion;
    S.ru = 1;
    S.init = 1;
    S.tol2 = tol * tol;
    S.delta2 = delta * delta;
    S.maxiter = maxiter;
    S.ratio2 = 1.0;
    HW_CUDA(cudaMemsetAsync(B.y.ptr, 0, B.y.bytes, ctx_->stream));
    HW_CUDA(cudaMemcpyAsync(d_states_.as<EngState>() + slot, &S, sizeof(S), cudaMemcpyHostToDevice, ctx_->stream));
    // a pending reliable update computes the first residual from x
    static const int one = 1;
    HW_CUDA(cudaMemcpyAsync(d_ctl_.as<int>() + 2, &one, sizeof(int), cudaMemcpyHostToDevice, ctx_->stream));
    *slot_out = slot;
    return HW_OK;
}

void Engine::release(int slot) {
    if (slot < 0 || slot >= kEngMaxProb || !slots_[slot].used) return;
    const int l = slots_[slot].lat;
    EngLattice &L = tables_.lat[l];
    int k = 0;
    for (int q = 0; q < L.nprob; q++)
        if (L.prob[q] != slot) L.prob[k++] = L.prob[q];
    L.nprob = k;
    slots_[slot].used = false;
    host_states_[slot].status = ENG_IDLE;
    host_states_[slot].ru = 0;
    cudaMemcpyAsync(d_states_.as<EngState>() + slot, &host_states_[slot], sizeof(EngState), cudaMemcpyHostToDevice,
                    ctx_->stream);
    tables_dirty_ = true;
}

int Engine::nslots_used() const {
    int n = 0;
    for (int j = 0; j < kEngMaxProb; j++) n += slots_[j].used;
    return n;
}

int Engine::upload_tables() {
    if (!tables_dirty_) return HW_OK;
    HW_CUDA(cudaMemcpyAsync(d_tables_.ptr, &tables_, sizeof(tables_), cudaMemcpyHostToDevice, ctx_->stream));
    tables_dirty_ = false;
    return HW_OK;
}

void Engine::set_ptrs() {
    ptrs_.T = d_tables_.as<EngTables>();
    ptrs_.S = d_states_.as<EngState>();
    ptrs_.partials = d_partials_.as<double>();
    ptrs_.tickets = d_tickets_.as<unsigned>();
    ptrs_.ctl = d_ctl_.as<int>();
    ptrs_.work = d_work_.as<unsigned long long>();
    ptrs_.sched = d_sched_.as<int>();
}

int Engine::build_graph() {
    set_ptrs();
    cudaStream_t s = ctx_->stream;
    cudaGraph_t g = nullptr;
    HW_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    HW_CUDA(cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
    // chunk begin
    HW_CUDA(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    eng_enqueue_chunk_begin(ptrs_, s);
    cudaGraph_t tmp = nullptr;
    HW_CUDA(cudaStreamEndCapture(s, &tmp));
    size_t n = 0;
    HW_CUDA(cudaGraphGetNodes(g, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    HW_CUDA(cudaGraphGetNodes(g, nodes.data(), &n));
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = cond;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t wnode;
    HW_CUDA(cudaGraphAddNode(&wnode, g, nodes.data(), nodes.size(), &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    HW_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    eng_enqueue_iteration(low_, ptrs_, grid_, s);
    eng_enqueue_control(ptrs_, kEngMaxProb, 0, cond, 1, s);
    HW_CUDA(cudaStreamEndCapture(s, &tmp));
    cudaError_t e = cudaGraphInstantiate(&chunk_exec_, g, 0);
    cudaGraphDestroy(g);
    HW_CUDA(e);
    return HW_OK;
}

int Engine::configure() {
    int mask = 0, fermions = 0;
    for (int l = 0; l < tables_.nlat; l++) {
        mask |= tables_.lat[l].l64_planes == 9 ? 1 : 2;
        fermions |= 1 << tables_.lat[l].fermion;
    }
    if (mask == 0) mask = 1;
    if (fermions == 0) fermions = 1;
    int variant = want_variant_ ? want_variant_ : default_variant();
    if (const char *env = std::getenv("HW_ENGINE_VARIANT")) variant = std::atoi(env);
    // launch shapes (engine.cu): 2 for both precisions, 4 and 7 for FP16 only; the
    // tensor-core variant 4 reads the 18-real FP16 links, which exist only with full18_
    const bool known =
        variant == 2 || (low_ == LOW_F16 && (variant == 7 || (variant == 4 && full18_)));
    if (!known) variant = default_variant();
    if (variant != grid_.variant || mask != grid_.planes_mask || fermions != grid_.fermions) {
        grid_ = eng_grid_size(low_, variant, full18_ ? 1 : 0, mask);
        grid_.fermions = fermions;  // the phases the iteration launches (engine.cu)
        if (chunk_exec_) {
            HW_CUDA(cudaStreamSynchronize(ctx_->stream));
            cudaGraphExecDestroy(chunk_exec_);
            chunk_exec_ = nullptr;
        }
    }
    return HW_OK;
}

// HW_ENGINE_TUNE=0 turns the tuner off; a shape or tile order forced by HW_ENGINE_VARIANT
// or HW_ENGINE_SCHED is not tuned (read at every chunk)
int Engine::tune_shapes(const TuneShape **shapes) const {
    static const TuneShape f16[] = {{7, 1}, {2, 1}, {7, 0}, {2, 0}};
    static const TuneShape f32[] = {{2, 1}, {2, 0}};
    if (const char *env = std::getenv("HW_ENGINE_TUNE"))
        if (std::atoi(env) == 0) return 0;
    if (std::getenv("HW_ENGINE_VARIANT") || std::getenv("HW_ENGINE_SCHED")) return 0;
    *shapes = low_ == LOW_F16 ? f16 : f32;
    return low_ == LOW_F16 ? 4 : 2;
}

int Engine::work_class() const {
    unsigned long long units = 0;
    for (int j = 0; j < kEngMaxProb; j++) {
        if (!slots_[j].used || host_states_[j].status != ENG_RUNNING) continue;
        const EngLattice &L = tables_.lat[slots_[j].lat];
        if (L.fermion == FERM_WILSON) units += (unsigned long long)L.ntiles;
    }
    return tune_work_class(units);
}

int Engine::launch_chunk(int iters) {
    int rc;
    // the chunk's shape: forced by the environment, the tuner's for this work class (a
    // candidate still being timed, or the fastest), or the default
    const TuneShape *shapes = nullptr;
    const int nshapes = tune_shapes(&shapes);
    int cls = 0, shape = -1, dyn = 1;
    want_variant_ = 0;
    if (const char *env = std::getenv("HW_ENGINE_SCHED")) dyn = std::atoi(env) != 0;
    if (nshapes > 1 && (cls = work_class()) >= kTuneMinClass) {
        bool timed = false;
        shape = tune_pick(tune_[cls], &timed);
        want_variant_ = shapes[shape].variant;
        dyn = shapes[shape].dyn;
        if (!timed || ctx_->engine_profile) cls = 0;  // decided, or profiling: no timing
    } else {
        cls = 0;
    }
    if (tables_.dyn != dyn) {
        tables_.dyn = dyn;
        tables_dirty_ = true;
    }
    if ((rc = configure()) != HW_OK) return rc;
    if ((rc = ensure_partials()) != HW_OK) return rc;
    if (cls > 0) {
        if ((rc = upload_tables()) != HW_OK) return rc;
        tune_pending_.cls = cls;
        tune_pending_.shape = shape;
        return launch_chunk_timed(iters);
    }
    if (use_graph_ && !chunk_exec_ && (rc = build_graph()) != HW_OK) return rc;
    if ((rc = upload_tables()) != HW_OK) return rc;
    if (ctx_->engine_profile) return launch_chunk_profiled(iters);
    if (!use_graph_) {
        set_ptrs();
        eng_enqueue_chunk_begin(ptrs_, ctx_->stream);
        for (int k = 0; k < iters; k++) {
            eng_enqueue_iteration(low_, ptrs_, grid_, ctx_->stream);
            eng_enqueue_control(ptrs_, kEngMaxProb, iters, 0, 0, ctx_->stream);
        }
        HW_CUDA(cudaGetLastError());
        return HW_OK;
    }
    // pageable source: the value is staged before the call returns
    HW_CUDA(cudaMemcpyAsync(d_ctl_.as<int>() + 3, &iters, sizeof(int), cudaMemcpyHostToDevice, ctx_->stream));
    HW_CUDA(cudaGraphLaunch(chunk_exec_, ctx_->stream));
    return HW_OK;
}

// A chunk of the tuner: the iterations from the host (no graph) with events around the
// phases of the first kTuneMaxIters; read_states turns them into a sample.
int Engine::launch_chunk_timed(int iters) {
    if (tune_ev_.empty()) {
        tune_ev_.assign((size_t)kTuneMaxIters * (kEngPhases + 1), nullptr);
        for (cudaEvent_t &e : tune_ev_) HW_CUDA(cudaEventCreate(&e));
    }
    int running = 0;
    for (int j = 0; j < kEngMaxProb; j++) running += slots_[j].used && host_states_[j].status == ENG_RUNNING;
    tune_pending_.running = running;
    tune_pending_.iters = iters < kTuneMaxIters ? iters : kTuneMaxIters;
    set_ptrs();
    eng_enqueue_chunk_begin(ptrs_, ctx_->stream);
    for (int k = 0; k < iters; k++) {
        const cudaEvent_t *ev = k < tune_pending_.iters ? &tune_ev_[(size_t)k * (kEngPhases + 1)] : nullptr;
        eng_enqueue_iteration(low_, ptrs_, grid_, ctx_->stream, ev);
        eng_enqueue_control(ptrs_, kEngMaxProb, iters, 0, 0, ctx_->stream);
    }
    HW_CUDA(cudaGetLastError());
    return HW_OK;
}

// After the synchronisation of read_states: a timed chunk in which every solve ran all
// its iterations (none finished, so no iteration was partly idle) gives a sample.
void Engine::tune_collect() {
    const int cls = tune_pending_.cls, shape = tune_pending_.shape, n = tune_pending_.iters;
    tune_pending_.cls = -1;
    if (cls <= 0 || n <= 0) return;
    int running = 0;
    for (int j = 0; j < kEngMaxProb; j++) running += slots_[j].used && host_states_[j].status == ENG_RUNNING;
    const TuneShape *shapes = nullptr;
    const int ns = tune_shapes(&shapes);
    if (ns <= 0) return;
    TuneEntry &e = tune_[cls];
    if (running != tune_pending_.running) {  // a solve finished inside the chunk
        tune_record(e, shape, ns, false, 0.0);
        return;
    }
    std::vector<double> it(n);
    for (int k = 0; k < n; k++) {
        const cudaEvent_t *ev = &tune_ev_[(size_t)k * (kEngPhases + 1)];
        float a = 0.f, b = 0.f;
        if (cudaEventElapsedTime(&a, ev[0], ev[PH_R1]) != cudaSuccess ||
            cudaEventElapsedTime(&b, ev[PH_P5], ev[kEngPhases]) != cudaSuccess) {
            cudaGetLastError();
            tune_record(e, shape, ns, false, 0.0);
            return;
        }
        it[k] = (double)a + (double)b;
    }
    std::sort(it.begin(), it.end());
    tune_record(e, shape, ns, true, it[n / 2]);
}

// Host-loop chunk with events around every phase; synchronises after each
// iteration to attribute its phase times.  A phase launch counts when its work
// units (engine.h) grew: launches that found no active slot are left out.
int Engine::launch_chunk_profiled(int iters) {
    for (cudaEvent_t &e : prof_ev_)
        if (!e) HW_CUDA(cudaEventCreate(&e));
    set_ptrs();
    eng_enqueue_chunk_begin(ptrs_, ctx_->stream);
    // the counters as they are now (launches outside profiling also count)
    HW_CUDA(cudaMemcpyAsync(pinned_work_, d_work_.ptr, d_work_.bytes, cudaMemcpyDeviceToHost, ctx_->stream));
    HW_CUDA(cudaStreamSynchronize(ctx_->stream));
    for (int k = 0; k < iters; k++) {
        int running = 0;
        for (int j = 0; j < kEngMaxProb; j++)
            if (slots_[j].used) running += host_states_[j].status == ENG_RUNNING;
        if (running == 0) break;
        std::memcpy(work_seen_, pinned_work_, sizeof(work_seen_));
        eng_enqueue_iteration(low_, ptrs_, grid_, ctx_->stream, prof_ev_);
        eng_enqueue_control(ptrs_, kEngMaxProb, iters, 0, 0, ctx_->stream);
        int rc;
        if ((rc = read_states()) != HW_OK) return rc;
        for (int ph = 0; ph < kEngPhases; ph++) {
            bool did = false;
            for (int w = 0; w < kEngWorkKinds; w++) {
                const int q = ph * kEngWorkKinds + w;
                did |= pinned_work_[q] != work_seen_[q];
            }
            if (!did) continue;
            float ms = 0.f;
            HW_CUDA(cudaEventElapsedTime(&ms, prof_ev_[ph], prof_ev_[ph + 1]));
            prof_ms_[ph] += ms;
            prof_n_[ph] += 1;
            for (int w = 0; w < kEngWorkKinds; w++) {
                const int q = ph * kEngWorkKinds + w;
                prof_work_[q] += pinned_work_[q] - work_seen_[q];
            }
        }
    }
    HW_CUDA(cudaGetLastError());
    return HW_OK;
}

void Engine::reset_profile() {
    for (int ph = 0; ph < kEngPhases; ph++) {
        prof_n_[ph] = 0;
        prof_ms_[ph] = 0.0;
    }
    std::memset(prof_work_, 0, sizeof(prof_work_));
}

void Engine::profile(int *launches, double *ms, unsigned long long *work) const {
    for (int ph = 0; ph < kEngPhases; ph++) {
        launches[ph] = (int)prof_n_[ph];
        ms[ph] = prof_ms_[ph];
    }
    std::memcpy(work, prof_work_, sizeof(prof_work_));
}

int Engine::read_states() {
    HW_CUDA(cudaMemcpyAsync(pinned_states_, d_states_.ptr, sizeof(EngState) * kEngMaxProb, cudaMemcpyDeviceToHost,
                            ctx_->stream));
    HW_CUDA(cudaMemcpyAsync(pinned_ctl_, d_ctl_.ptr, sizeof(int) * 8, cudaMemcpyDeviceToHost, ctx_->stream));
    HW_CUDA(cudaMemcpyAsync(pinned_work_, d_work_.ptr, d_work_.bytes, cudaMemcpyDeviceToHost, ctx_->stream));
    HW_CUDA(cudaStreamSynchronize(ctx_->stream));
    HW_CUDA(cudaGetLastError());
    bodies_total_ = reinterpret_cast<const unsigned long long *>(pinned_ctl_ + 6)[0];
    for (int j = 0; j < kEngMaxProb; j++)
        if (slots_[j].used) host_states_[j] = pinned_states_[j];
    tune_collect();
    return HW_OK;
}

int get_engine(hw_context *ctx, int low, Engine **eng) {
    HW_CHECK_ARG(low == LOW_F32 || low == LOW_F16, "engine precision must be FP32 or FP16");
    if (!ctx->engines[low]) {
        Engine *e = new Engine(ctx, low);
        int rc = e->init();
        if (rc != HW_OK) {
            delete e;
            return rc;
        }
        ctx->engines[low] = e;
    }
    *eng = ctx->engines[low];
    return HW_OK;
}

void destroy_engines(hw_context *ctx) {
    for (int k = 0; k < 3; k++) {
        delete ctx->engines[k];
        ctx->engines[k] = nullptr;
    }
}

}  // namespace hw
