// Batched mixed-precision CG engine: device tables shared by engine.cu and engine.cpp.
//
// An engine holds up to kEngMaxLat lattices (each with its gauge field) and up
// to kEngMaxProb solve slots.  Every phase of a CG iteration is ONE launch of a
// persistent-style grid that walks the tiles (kEngTile sites) of all lattices,
// and inside each tile every active slot on that lattice, so links loaded for
// the first right-hand side are re-read from L1/L2 by the others.  The slot
// states live in device memory; the kernels read the tables through a pointer,
// so the same captured CUDA graph serves every batch composition.
//
// Inner iteration (low precision: FP32, or FP16 with a per-site scale; links
// 12 reals; accumulation in FP32; dot products in FP64):
//   P1  t  = H^{oe}_+ p
//   P2  Dp = p - kappa^2 H^{eo}_+ t           |Dp|^2 -> alpha
//   P3  t  = H^{oe}_- Dp
//   P4  DDp = Dp - kappa^2 H^{eo}_- t; r -= alpha DDp; y += alpha p (FP32)
//                                              |r|^2 -> beta, reliable-update decision
// Reliable update (FP64, only slots that asked for it):
//   R1  x += y; y = 0                          (FP64 solution accumulation)
//   R2  t64 = H^{oe}_+ x
//   R3  solve mode:  s = b - (x - kappa^2 H t64)   |s|^2, |b|^2; s kept in FP32 (in y)
//       normal mode: s = x - kappa^2 H t64         (= M x, FP64)
//   R4  normal mode: t64 = H^{oe}_- s
//   R4L solve mode:  t = H^{oe}_- s               (FP32, in the t64 buffer; low-precision links)
//   R5  normal mode: r = b - (s - kappa^2 H^dag t64) (= b - M^dag M x), |b|^2
//   R5L solve mode:  r = s - kappa^2 H^dag t       (= M^dag (b - M x), FP32); y cleared
//       r_low = r, |r|^2 -> true residual, convergence, beta
//   P5  p = r + beta p   (p = r on a slot's first iteration)
#pragma once

#include "kernels.h"

namespace hw {

constexpr int kEngTile = 128;      // sites per tile = threads per block of the engine kernels
constexpr int kEngMaxLat = 32;     // lattices per engine
constexpr int kEngMaxProb = 64;    // solve slots per engine
constexpr int kEngMaxRhs = 16;     // slots per lattice

enum EngStatus : int { ENG_RUNNING = 0, ENG_CONVERGED = 1, ENG_MAXITER = 2, ENG_BREAKDOWN = 3, ENG_IDLE = 4 };
// fermion of a lattice entry (and of its slots).  Staggered solves (staggered.h) run the
// same phase sequence and state machine in FP64 on colour-vector fields (engine_stag.cuh):
//   P1 t = (1/m) D^{oe}_+ p   P2 Dp = m p + D^{eo}_+ t, |Dp|^2   P3 t = (1/m) D^{oe}_- Dp
//   P4 r -= alpha (m Dp + D^{eo}_- t), x += alpha p (FP64), |r|^2
//   R1 flags a nonzero initial x; R2, R3 s = b - M x; R4(L), R5(L) r = M^dag s; P5 p = r + beta p
// with D_s = 0.5 s hop (staggered.h:48-68) and the slot's kappa holding the mass m.
// A slot with stag_low set runs P1..P5 in FP32 arithmetic on FP16 fields with a per-site
// norm and FP16 links, P4 accumulating alpha p in the FP32 y, R1 x += y, and the reliable
// update in FP64 (t64 holds the odd FP64 half, R5(L) stores r in FP16).
// (a slot's EngState.fermion is FERM_STAGGERED_LOW for a staggered solve with FP16 inner
// iterations; lattice entries are FERM_WILSON or FERM_STAGGERED)
enum EngFermion : int { FERM_WILSON = 0, FERM_STAGGERED = 1, FERM_STAGGERED_LOW = 2 };
enum EngMode : int { ENG_MODE_SOLVE = 0, ENG_MODE_NORMAL = 1 };

struct EngLattice {
    Geom g;
    int stride;       // padded sites per parity of every field of this lattice
    int tile0;        // first global tile
    int ntiles;       // tiles of one parity
    int nprob;        // slots on this lattice
    int fermion;      // EngFermion of the lattice entry (one gauge field may have one of each)
    int prob[kEngMaxRhs];
    // links: FP64 (18 or 12 reals) for the reliable updates, low precision for the inner solve
    const double2 *l64;
    int l64_planes;
    const float4 *l32;   // FP32, 12 reals: 3 float4 planes per (parity, dir)
    const uint4 *l16a;   // FP16, 12 reals: 8 halves ...
    const uint2 *l16b;   // ... + 4 halves per link
    const float4 *l32a;  // FP32, 18 reals: 4 float4 planes ...
    const float2 *l32b;  // ... + 1 float2 plane per (parity, dir)
    const uint4 *l16x;     // FP16, 18 reals: elements 0..7 in 2 uint4 planes ...
    const unsigned *l16z;  // ... + element 8 in 1 plane per (parity, dir)
};

struct EngProblem {
    int lat;
    int mode;
    int stag_low;  // staggered slot with FP16 inner iterations (FP64 reliable updates); 0: FP64 throughout
    int pad;
    double kappa;
    double diag;  // 1 + m_h: the Hasenbusch operator M + m_h (Hasenbusch.h:16-52); 1 for M
    // low precision (EVEN: p, r, Dp; ODD: t); FP16 fields carry a norm plane
    void *p, *r, *Dp, *t;
    float *pn, *rn, *Dpn, *tn;
    float4 *y;  // FP32 solution increment since the last reliable update (6 float4 planes)
    // FP64 (EVEN: x, b, s; ODD: t64)
    double2 *x, *b, *s, *t64;
};

struct EngState {
    double rr;       // |r|^2 (iterated, or true after a reliable update)
    double rr_old;   // |r|^2 of the previous iteration (beta after a reliable update)
    double pAp;
    double alpha, beta;
    double rmax2;    // largest |r|^2 since the last reliable update
    double b2;       // |b|^2 of the system being solved
    double s2;       // |b - M x|^2 (solve mode) at the last reliable update
    double ratio2;   // s2 / rr at the last reliable update: estimates |b - M x| from |r|
    double tol2;     // accuracy^2
    double delta2;   // reliable-update factor^2
    double seconds;  // unused by the device; host bookkeeping
    int iter, maxiter;
    int status;      // EngStatus
    int ru;          // 1: reliable update pending
    int init;        // 1: first reliable update (r from x), p = r afterwards
    int n_ru;
    int mode;        // EngMode of the slot (copy of its problem's, read by the phase selection)
    int xnz;         // 1: the initial x has a nonzero component (set by R1 of the first update)
    int fermion;     // EngFermion of the slot's lattice (read by the phase selection)
};

struct EngTables {
    int nlat;
    int ntiles;  // total tiles over all lattices
    int max_tiles;  // partial-sum stride: largest ntiles of any lattice
    int dyn;     // 1: the inner phases' blocks take tiles from a counter (balances lattices whose
                 // tiles carry different numbers of active slots); 0: tile = block + k * grid
    EngLattice lat[kEngMaxLat];
    EngProblem prob[kEngMaxProb];
};

// device pointers the engine kernels take
struct EngPtrs {
    const EngTables *T;
    EngState *S;
    double *partials;     // kEngMaxProb * 2 * max_tiles
    unsigned *tickets;    // one per lattice
    int *ctl;             // [0] iterations run in this chunk, [1] running slots,
                          // [2] reliable updates requested in this iteration,
                          // [3] iteration limit of a chunk (control kernel with chunk <= 0)
    unsigned long long *work;  // kEngPhases x kEngWorkKinds cumulative work units (below)
    int *sched;           // kEngPhases tile counters of the inner phases' dynamic tile order
                          // (zeroed at the start of a chunk and by every iteration's control kernel)
};

// Work units counted by every phase launch (cumulative, per phase), from which the
// algorithmic bytes of the launches that did work follow:
//   [0] sites x slots that ran the phase's main form
//   [1] sites x slots of its alternate form: R1 normal-system slots (y also cleared),
//       R3 solve-mode slots of a first update from x = 0 (no hop), P5 first iterations
//       (p = r, p not read)
//   [2] sites whose links were read (once per site and launch, shared by the slots)
//   [3] R3: sites x slots of the normal system (s = M x in FP64)
constexpr int kEngWorkKinds = 4;

struct EngGrid {
    int low;  // blocks of the low-precision phases (all SMs x resident blocks)
    int f64;  // blocks of the FP64 reliable-update phases
    int pk;   // blocks of the packed two-solve phases of the hybrid shapes (engine.cu)
    int variant;  // launch shape of the low-precision phases (engine.cu)
    int full18;   // 1: inner phases read 18-real links (FP32 or FP16); 0: the 12-real links of the precision
    int planes_mask;  // FP64 link formats present: bit 0 = 18 reals, bit 1 = 12 reals
    int fermions;     // lattice kinds present: bit 0 Wilson, bit 1 staggered (phases launched)
};

// in launch order; R4 / R5 serve slots of the normal system (FP64), R4L / R5L those of
// M x = b (FP32: r = M^dag s only feeds the low-precision iteration, and s = b - M x,
// on which convergence is decided, is formed and measured in FP64)
enum EngPhase : int {
    PH_P1 = 0, PH_P2, PH_P3, PH_P4, PH_R1, PH_R2, PH_R3, PH_R4, PH_R4L, PH_R5, PH_R5L, PH_P5
};
constexpr int kEngPhases = 12;
__host__ __device__ constexpr bool eng_ru_phase(int ph) { return ph >= PH_R1 && ph <= PH_R5L; }

// low-precision format of one engine (template parameter of the inner phases)
enum EngLow : int { LOW_F32 = 1, LOW_F16 = 2 };

// Enqueue one CG iteration (all phases) on stream s.  With ev (kEngPhases + 1
// events) ev[k] is recorded before phase k and ev[kEngPhases] after the last.
void eng_enqueue_iteration(int low, const EngPtrs &P, const EngGrid &G, cudaStream_t s,
                           const cudaEvent_t *ev = nullptr);
// While-loop control: counts running slots, stops after `chunk` iterations or when none runs.
void eng_enqueue_control(const EngPtrs &P, int nprob, int chunk, cudaGraphConditionalHandle h, int use_cond,
                         cudaStream_t s);
void eng_enqueue_chunk_begin(const EngPtrs &P, cudaStream_t s);
// Convert FP64 link planes to the 12-real FP32 / FP16 planes of the inner solve.
void eng_convert_links(const Geom &g, const double2 *l64, int planes, int stride, float4 *l32, uint4 *l16a,
                       uint2 *l16b, float4 *l32a, float2 *l32b, uint4 *l16x, unsigned *l16z, cudaStream_t s);
// launch configuration of the engine kernels on the current device
EngGrid eng_grid_size(int low, int variant, int full18, int planes_mask);

}  // namespace hw
