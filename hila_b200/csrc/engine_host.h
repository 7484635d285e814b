// Host side of the batched mixed-precision CG engine (kernels in engine.cu).
#pragma once

#include <map>
#include <memory>
#include <vector>

#include "engine.h"
#include "engine_tune.h"
#include "hw_internal.h"

namespace hw {

// Device buffers of one solve slot, sized for a lattice stride.
struct SlotBuffers {
    DevBuf p, r, Dp, t, pn, rn, Dpn, tn, y, s, t64;
    DevBuf x_own, b_own;  // FP64 EVEN halves for slots that own their source / solution
    DevBuf xfer;          // layout staging of an owned solution on its way to the host
    int stride = 0;
};

struct SlotInfo {
    bool used = false;
    int lat = -1;
};

// Online choice of the inner phases' launch shape: the candidates (engine_tune.h) are
// timed on real iterations of the running batch (median over a chunk of the device time
// of P1..P4 and P5, which the shape changes; the reliable-update phases do not depend on
// it) and the fastest is kept per work class.

class Engine {
  public:
    Engine(hw_context *ctx, int low) : ctx_(ctx), low_(low) {}
    ~Engine();
    int init();
    int low() const { return low_; }
    bool full18() const { return full18_; }  // inner phases read 18-real links

    // index of the lattice entry of `gauge` for a fermion (EngFermion) in this engine,
    // adding it if needed
    int lattice_index(const hw_gauge *gauge, int *idx, int fermion = FERM_WILSON);
    // drop lattices with no used slot (compacts the tile list)
    int prune_lattices();
    int free_slots_on(int lat) const;

    // Start a solve in a free slot.  b, x: FP64 EVEN halves (stride of the
    // lattice); null means slot-owned buffers (filled with upload_b / read with x_ptr).
    // diag = 1 + m_h solves with the Hasenbusch operator M + m_h (1: M itself).
    int admit(int lat, double kappa, double2 *b, double2 *x, double tol, int maxiter, double delta, int mode,
              int *slot, double diag = 1.0);
    double2 *own_b(int slot) { return bufs_[slot]->b_own.as<double2>(); }
    double2 *own_x(int slot) { return bufs_[slot]->x_own.as<double2>(); }
    double2 *own_xfer(int slot) { return bufs_[slot]->xfer.as<double2>(); }
    int ensure_own(int slot);
    // stream-ordered: run up to `iters` iterations of every running slot
    // (stops early when none runs)
    int launch_chunk(int iters);
    // copy the slot states to the host mirror (synchronises the stream)
    int read_states();
    // loop bodies (10 phase kernels + 1 control kernel each) run since init, as of the last read_states
    unsigned long long bodies_total() const { return bodies_total_; }
    // per-phase device time and work units (engine.h, kEngWorkKinds) of the launches
    // that did work, while the context's engine profiling is on (iterations then run
    // from a synchronising host loop)
    void reset_profile();
    void profile(int *launches, double *ms, unsigned long long *work) const;
    const EngState &state(int slot) const { return host_states_[slot]; }
    void release(int slot);
    int nslots_used() const;
    size_t slot_bytes(int lat) const;
    // device bytes of one solve slot (including slot-owned b and x) for a lattice stride
    size_t slot_bytes_for_stride(int stride) const;
    int slot_lattice(int slot) const { return slots_[slot].lat; }
    // Size every slot's buffers for at least this stride when they are first made, so a slot
    // can later take any lattice up to it without allocating (0: each lattice's own stride)
    void set_min_stride(int stride) { min_stride_ = stride; }
    const EngLattice &lattice(int l) const { return tables_.lat[l]; }
    int nlat() const { return tables_.nlat; }
    const hw_gauge *gauge(int l) const { return gauges_[l]; }
    int upload_tables();
    // launch-shape candidates of this engine (empty when a shape is forced by the
    // environment or tuning is off) and the tuner's entries by work class
    int tune_shapes(const TuneShape **shapes) const;
    const std::map<int, TuneEntry> &tuning() const { return tune_; }
    // work class of the running Wilson solves: bit length of the sum over them of
    // their lattice's tiles (0: none)
    int work_class() const;

  private:
    int ensure_slot_buffers(int slot, int stride);
    int build_graph();
    void set_ptrs();
    int configure();
    int ensure_partials();

    hw_context *ctx_;
    int low_;
    bool ready_ = false;
    EngTables tables_{};
    std::vector<const hw_gauge *> gauges_;
    SlotInfo slots_[kEngMaxProb];
    std::unique_ptr<SlotBuffers> bufs_[kEngMaxProb];
    // Slot buffers set aside by a slot that took a lattice of another size, by stride.  A
    // slot whose buffers are too small swaps them for idle ones before anything is
    // allocated: cudaMalloc and cudaFree synchronise the device, and a server admitting
    // requests of many lattice sizes stalled on them.  Idle buffers beyond the cap are freed.
    std::multimap<int, std::unique_ptr<SlotBuffers>> idle_bufs_;
    size_t idle_bytes_ = 0;
    int min_stride_ = 0;
    void free_idle();
    int alloc_slot_buffers(std::unique_ptr<SlotBuffers> &cur, int stride);
    static constexpr size_t kIdleCapBytes = size_t(16) << 30;
    static size_t buffer_bytes(const SlotBuffers &B);
    void park_buffers(std::unique_ptr<SlotBuffers> B);
    EngState host_states_[kEngMaxProb];
    EngState *pinned_states_ = nullptr;
    int *pinned_ctl_ = nullptr;
    unsigned long long *pinned_work_ = nullptr;  // kEngPhases x kEngWorkKinds, as of the last read_states
    unsigned long long work_seen_[kEngPhases * kEngWorkKinds] = {};
    unsigned long long prof_work_[kEngPhases * kEngWorkKinds] = {};
    unsigned long long bodies_total_ = 0;
    cudaEvent_t prof_ev_[kEngPhases + 1] = {};
    long prof_n_[kEngPhases] = {};
    double prof_ms_[kEngPhases] = {};
    int launch_chunk_profiled(int iters);
    int launch_chunk_timed(int iters);
    void tune_collect();
    int want_variant_ = 0;  // the tuner's shape for the next chunks (0: the default)
    std::map<int, TuneEntry> tune_;
    std::vector<cudaEvent_t> tune_ev_;  // kTuneMaxIters x (kEngPhases + 1)
    struct {
        int cls = -1, shape = -1, iters = 0, running = 0;
    } tune_pending_;
    DevBuf d_tables_, d_states_, d_partials_, d_tickets_, d_ctl_, d_work_, d_sched_;
    size_t partial_tiles_ = 0;
    EngGrid grid_{};
    EngPtrs ptrs_{};
    cudaGraphExec_t chunk_exec_ = nullptr;
    bool tables_dirty_ = true;
    bool use_graph_ = true;
    bool full18_ = false;
    // launch shape of the inner phases (engine.cu) when the tuner has none: FP16 packed
    // two-solve P1 / P3 (fastest measured at 32^4); FP32 one solve per thread
    int default_variant() const { return low_ == LOW_F16 ? 7 : 2; }
};

// per-context engine for a low precision (LOW_F32 / LOW_F16), created on first use
int get_engine(hw_context *ctx, int low, Engine **eng);
// make the FP32 / FP16 link copies of a gauge field
int ensure_low_links(const hw_gauge *G, int low, bool full18);

}  // namespace hw
