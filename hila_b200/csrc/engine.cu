// Kernels of the batched mixed-precision CG engine (phase list in engine.h).
//
// All phases share one grid of kEngTile-thread blocks that strides over the
// tiles of every lattice; inside a tile the block walks the lattice's active
// slots.  Dot products are reduced per (slot, tile) with a fixed tree and
// summed per slot in tile order by the last block to finish the lattice, so a
// slot's arithmetic does not depend on which other slots share the launch:
// a solve gives bitwise the same result alone and inside any batch.
#include <cuda_fp16.h>

#include <mutex>
#include <type_traits>

#include "engine.h"
#include "pair.cuh"
#include "reduce.cuh"
#include "staggered_math.cuh"
#include "storage.cuh"

namespace hw {

namespace {

template <int LOW>
struct Low;

template <>
struct Low<LOW_F32> {
    using Sp = SpinorF32;
    using Lk = LinksF32x12;
    static __device__ __forceinline__ Sp sp(void *p, float *, int stride) {
        return Sp{static_cast<float4 *>(p), stride};
    }
    static __device__ __forceinline__ Lk lk(const EngLattice &L) { return Lk{L.l32, L.stride}; }
};

template <>
struct Low<LOW_F16> {
    using Sp = SpinorF16;
    using Lk = LinksF16x12;
    static __device__ __forceinline__ Sp sp(void *p, float *n, int stride) {
        return Sp{static_cast<uint4 *>(p), n, stride};
    }
    static __device__ __forceinline__ Lk lk(const EngLattice &L) { return Lk{L.l16a, L.l16b, L.stride}; }
};

// links of the inner phases: the precision's own 12-real format, or all 18 reals
// in the precision (no third-row rebuild)
template <int LOW, bool FULL18>
struct InnerLinks {
    using Lk = typename Low<LOW>::Lk;
    static __device__ __forceinline__ Lk lk(const EngLattice &L) { return Low<LOW>::lk(L); }
};
template <>
struct InnerLinks<LOW_F32, true> {
    using Lk = LinksF32x18;
    static __device__ __forceinline__ Lk lk(const EngLattice &L) { return Lk{L.l32a, L.l32b, L.stride}; }
};
template <>
struct InnerLinks<LOW_F16, true> {
    using Lk = LinksF16x18;
    static __device__ __forceinline__ Lk lk(const EngLattice &L) { return Lk{L.l16x, L.l16z, L.stride}; }
};

__device__ __forceinline__ int find_lattice(const EngTables *T, int tile) {
    int l = 0;
    const int n = T->nlat;
    for (int k = 1; k < n; k++)
        if (tile >= T->lat[k].tile0) l = k;
    return l;
}

// Which slots take part in a phase.  States only change in the finishers,
// which run after every tile of the lattice is done, so all blocks agree.
template <int PHASE, int FERM = FERM_WILSON>
__device__ __forceinline__ bool active(const EngState &s) {
    // the other fermion's kernels serve this slot; the FP64 staggered kernels also run the
    // reliable update of the staggered slots with FP16 inner iterations
    const bool mine = s.fermion == FERM ||
                      (FERM == FERM_STAGGERED && s.fermion == FERM_STAGGERED_LOW && eng_ru_phase(PHASE));
    if (!mine) return false;
    // the first update of a solve from x = 0: H x is zero, R2 has nothing to do
    if (PHASE == PH_R2) return s.ru != 0 && !(s.init && !s.xnz);
    if (PHASE == PH_R4 || PHASE == PH_R5) return s.ru != 0 && s.mode == ENG_MODE_NORMAL;
    if (PHASE == PH_R4L || PHASE == PH_R5L) return s.ru != 0 && s.mode == ENG_MODE_SOLVE;
    if (eng_ru_phase(PHASE)) return s.ru != 0;
    return s.status == ENG_RUNNING && s.ru == 0;
}

__device__ __forceinline__ Cx<double> ldc(const double2 *p, int stride, int c, int i) {
    double2 v = p[(size_t)c * stride + i];
    return {v.x, v.y};
}
__device__ __forceinline__ void stc(double2 *p, int stride, int c, int i, Cx<double> v) {
    p[(size_t)c * stride + i] = make_double2(v.re, v.im);
}

static_assert(kEngMaxRhs <= 32, "one warp lane per slot of a lattice");

// Work units of a phase launch (engine.h, kEngWorkKinds).  Called once per lattice and
// launch (by the block that meets the lattice's first tile), with every site of the
// lattice counted: all tiles of a lattice see the same active slots.
__device__ __forceinline__ void count_work(const EngPtrs &P, int phase, int kind, unsigned long long units) {
    if (units) atomicAdd(P.work + phase * kEngWorkKinds + kind, units);
}

// Active slots of every lattice for one phase launch, built once per block: slot
// states change only in the finishers, and a lattice's finisher runs after all of
// its work items, so the table stays valid for every item the block still meets.
struct ActiveTable {
    int slot[kEngMaxLat][kEngMaxRhs];  // slot[l][a]: the a-th active slot of lattice l
    int n[kEngMaxLat];
};

template <int PHASE, int FERM = FERM_WILSON>
__device__ __forceinline__ void build_active(const EngPtrs &P, ActiveTable &A) {
    const EngTables *T = P.T;
    for (int l = threadIdx.x; l < T->nlat; l += blockDim.x) {
        const EngLattice &La = T->lat[l];
        int na = 0;
        for (int q = 0; q < La.nprob; q++) {
            const int j = La.prob[q];
            if (active<PHASE, FERM>(P.S[j])) A.slot[l][na++] = j;
        }
        A.n[l] = na;
    }
    __syncthreads();
}

// ------------------------------------------------------------------ epilogues

// Low-precision phases P1..P4.  acc = (H in)(i) in FP32.
template <int PHASE, int LOW>
__device__ __forceinline__ void epi_low(const EngProblem &pr, const EngState &st, int stride, int i,
                                        Spinor<float> &acc, double *red) {
    using L = Low<LOW>;
    // d p as an uncontracted product: with d = 1 the sums round exactly as p - k^2 acc
    const float dg = (float)pr.diag;
    auto ds = [dg](Cx<float> v) -> Cx<float> { return {__fmul_rn(dg, v.re), __fmul_rn(dg, v.im)}; };
    if (PHASE == PH_P1 || PHASE == PH_P3) {
        L::sp(pr.t, pr.tn, stride).store(i, acc);
    } else if (PHASE == PH_R4L) {
        SpinorF32{reinterpret_cast<float4 *>(pr.t64), stride}.store(i, acc);  // FP32 in the FP64 t buffer
    } else if (PHASE == PH_R5L) {
        // r = d s - k^2 H^dag t with s in FP32 in y (reliable update of M x = b); |r|^2;
        // y is cleared again for the solution increments that follow
        const float k2 = (float)(pr.kappa * pr.kappa);
        Spinor<float> sv;
        SpinorF32 ys{pr.y, stride};
        ys.load_cached(i, sv);
        double n2 = 0;
#pragma unroll
        for (int c = 0; c < 12; c++) {
            Cx<float> v = ds(sv.s[c / 3][c % 3]) - k2 * acc.s[c / 3][c % 3];
            acc.s[c / 3][c % 3] = v;
            n2 += (double)norm2(v);
        }
        L::sp(pr.r, pr.rn, stride).store(i, acc);
        Spinor<float> zero;
#pragma unroll
        for (int c = 0; c < 12; c++) zero.s[c / 3][c % 3] = {0.f, 0.f};
        ys.store(i, zero);
        red[0] = n2;
    } else if (PHASE == PH_P2) {
        const float k2 = (float)(pr.kappa * pr.kappa);
        Spinor<float> p;
        L::sp(pr.p, pr.pn, stride).load_cached(i, p);
        double n2 = 0;
#pragma unroll
        for (int c = 0; c < 12; c++) {
            Cx<float> v = ds(p.s[c / 3][c % 3]) - k2 * acc.s[c / 3][c % 3];
            acc.s[c / 3][c % 3] = v;
            n2 += (double)norm2(v);
        }
        L::sp(pr.Dp, pr.Dpn, stride).store(i, acc);
        red[0] = n2;
    } else if (PHASE == PH_P4) {
        const float k2 = (float)(pr.kappa * pr.kappa);
        const float alpha = (float)st.alpha;
        Spinor<float> d, r;
        L::sp(pr.Dp, pr.Dpn, stride).load_cached(i, d);
        L::sp(pr.r, pr.rn, stride).load_cached(i, r);
        double n2 = 0;
#pragma unroll
        for (int c = 0; c < 12; c++) {
            Cx<float> ddp = ds(d.s[c / 3][c % 3]) - k2 * acc.s[c / 3][c % 3];
            Cx<float> rv = r.s[c / 3][c % 3] - alpha * ddp;
            r.s[c / 3][c % 3] = rv;
            n2 += (double)norm2(rv);
        }
        L::sp(pr.r, pr.rn, stride).store(i, r);
        // y += alpha p in FP32
        Spinor<float> p, y;
        L::sp(pr.p, pr.pn, stride).load_cached(i, p);
        SpinorF32 ys{pr.y, stride};
        ys.load_cached(i, y);
#pragma unroll
        for (int c = 0; c < 12; c++) y.s[c / 3][c % 3] = y.s[c / 3][c % 3] + alpha * p.s[c / 3][c % 3];
        ys.store(i, y);
        red[0] = n2;
    }
}

// FP64 reliable-update phases R2..R5.  acc = (H in)(i) in FP64.  The problem's
// pointers are copied to locals first: stores through them could otherwise alias
// the table and force reloads.
template <int PHASE, int LOW>
__device__ __forceinline__ void epi_f64(const EngProblem &pr, int stride, int i, Spinor<double> &acc,
                                        double *red) {
    const double k2 = pr.kappa * pr.kappa;
    const bool solve = pr.mode == ENG_MODE_SOLVE;
    const double dg = pr.diag;
    auto ds = [dg](Cx<double> v) -> Cx<double> { return {__dmul_rn(dg, v.re), __dmul_rn(dg, v.im)}; };
    if (PHASE == PH_R2 || PHASE == PH_R4) {
        SpinorF64{pr.t64, stride}.store(i, acc);
    } else if (PHASE == PH_R3) {
        const double2 *__restrict__ x = pr.x;
        const double2 *__restrict__ b = pr.b;
        double2 *__restrict__ sp = pr.s;
        double n2 = 0, d2 = 0;
        if (solve) {
            Spinor<float> sl;
#pragma unroll
            for (int c = 0; c < 12; c++) {
                const Cx<double> mx = ds(ldc(x, stride, c, i)) - k2 * acc.s[c / 3][c % 3];
                const Cx<double> bv = ldc(b, stride, c, i);
                const Cx<double> sv = bv - mx;
                // s itself is only read by the FP64 R4 / R5 of the normal system; solve mode
                // continues from its low-precision copy
                sl.s[c / 3][c % 3] = {(float)sv.re, (float)sv.im};
                n2 += norm2(sv);
                d2 += norm2(bv);
            }
            SpinorF32{pr.y, stride}.store(i, sl);  // input of R4L / R5L (y was cleared by R1)
        } else {
#pragma unroll
            for (int c = 0; c < 12; c++) stc(sp, stride, c, i, ds(ldc(x, stride, c, i)) - k2 * acc.s[c / 3][c % 3]);
        }
        red[0] = n2;
        red[1] = d2;
    } else if (PHASE == PH_R5) {
        const double2 *__restrict__ sv = pr.s;
        const double2 *__restrict__ b = pr.b;
        double n2 = 0, d2 = 0;
        Spinor<float> rl;
        if (solve) {
#pragma unroll
            for (int c = 0; c < 12; c++) {
                const Cx<double> v = ds(ldc(sv, stride, c, i)) - k2 * acc.s[c / 3][c % 3];
                n2 += norm2(v);
                rl.s[c / 3][c % 3] = {(float)v.re, (float)v.im};
            }
        } else {
#pragma unroll
            for (int c = 0; c < 12; c++) {
                const Cx<double> bv = ldc(b, stride, c, i);
                const Cx<double> v = bv - (ds(ldc(sv, stride, c, i)) - k2 * acc.s[c / 3][c % 3]);
                d2 += norm2(bv);
                n2 += norm2(v);
                rl.s[c / 3][c % 3] = {(float)v.re, (float)v.im};
            }
        }
        Low<LOW>::sp(pr.r, pr.rn, stride).store(i, rl);
        red[0] = n2;
        red[1] = d2;
    }
}

// ------------------------------------------------------------------ finishers

template <int PHASE>
__device__ void finish(EngState &s, const EngProblem &pr, const double *tot, int *ctl) {
    if (PHASE == PH_P2) {
        s.pAp = tot[0];
        if (!(tot[0] > 0.0) || !isfinite(tot[0])) {
            s.status = ENG_BREAKDOWN;
            s.alpha = 0.0;
        } else {
            s.alpha = s.rr / tot[0];
        }
    } else if (PHASE == PH_P4) {
        const double rr = tot[0];
        s.iter += 1;
        if (!isfinite(rr)) {
            s.status = ENG_BREAKDOWN;
            return;
        }
        s.rr_old = s.rr;
        s.rr = rr;
        s.beta = rr / s.rr_old;
        if (rr > s.rmax2) s.rmax2 = rr;
        // reliable update: residual fell by delta, or it looks converged, or the iterations ran out
        const bool drop = rr < s.delta2 * s.rmax2;
        const bool conv = pr.mode == ENG_MODE_SOLVE ? (s.ratio2 * rr <= s.tol2 * s.b2) : (rr <= s.tol2 * s.b2);
        if (drop || conv || s.iter >= s.maxiter) {
            s.ru = 1;
            atomicAdd(ctl + 2, 1);
        }
    } else if (PHASE == PH_R3) {
        if (pr.mode == ENG_MODE_SOLVE) {
            s.s2 = tot[0];
            s.b2 = tot[1];
        }
    } else if (PHASE == PH_R5 || PHASE == PH_R5L) {
        const double r2 = tot[0];
        if (PHASE == PH_R5 && pr.mode == ENG_MODE_NORMAL) {
            s.b2 = tot[1];
            s.s2 = r2;
        }
        s.ru = 0;
        s.n_ru += 1;
        if (!isfinite(r2) || !isfinite(s.s2) || !isfinite(s.b2)) {
            s.status = ENG_BREAKDOWN;
            return;
        }
        if (s.b2 == 0.0 || s.s2 <= s.tol2 * s.b2) {
            s.status = ENG_CONVERGED;
            return;
        }
        if (s.iter >= s.maxiter) {
            s.status = ENG_MAXITER;
            return;
        }
        if (s.init) {
            s.rr_old = r2;
            s.beta = 0.0;
        } else {
            s.beta = r2 / s.rr_old;
        }
        s.rr = r2;
        s.rmax2 = r2;
        s.ratio2 = r2 > 0.0 ? s.s2 / r2 : 1.0;
    }
}

// ------------------------------------------------------------------ hop phases

// Arrival of one work item of lattice l (a tile, or a (tile, slot) pair: the
// lattice expects `expected` of them); the last arrival sums every active
// slot's partials in tile order and runs the finisher.
template <int PHASE, int NRED, int FERM = FERM_WILSON>
__device__ __forceinline__ void arrive_and_finish(const EngPtrs &P, const EngLattice &La, int l, double *smem,
                                                  bool &last, int expected) {
    const EngTables *T = P.T;
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned t = atomicAdd(P.tickets + l, 1u);
        last = (t == (unsigned)expected - 1u);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        const int nt = La.ntiles;
        const int max_tiles = T->max_tiles;
        for (int q = 0; q < La.nprob; q++) {
            const int j = La.prob[q];
            if (!active<PHASE, FERM>(P.S[j])) continue;
            double tot[2] = {0.0, 0.0};
#pragma unroll
            for (int k = 0; k < NRED; k++) {
                const double *pp = P.partials + ((size_t)j * 2 + k) * max_tiles;
                double s = 0.0;
                for (int t2 = threadIdx.x; t2 < nt; t2 += kEngTile) s += __ldcg(pp + t2);
                tot[k] = block_sum<kEngTile>(s, smem);
            }
            if (threadIdx.x == 0) finish<PHASE>(P.S[j], T->prob[j], tot, P.ctl);
            __syncthreads();
        }
        if (threadIdx.x == 0) P.tickets[l] = 0u;
    }
    __syncthreads();
}

#include "engine_mma.cuh"
#include "engine_stag.cuh"

// Inner phases P1..P4 in low precision.  Each thread owns one site and up to
// NR right-hand sides at a time, so links, their third rows and the neighbour
// indices are shared by the NR solves.  PK (with NR = 2 and FP16 input): the two
// solves run in the two lanes of packed FP32 instructions (pair.cuh).
template <int PHASE, int LOW, int NR, int MINB, bool FULL18, bool PK = false>
__global__ void __launch_bounds__(kEngTile, MINB) k_eng_low(EngPtrs P) {
    constexpr int SIGN = (PHASE == PH_P1 || PHASE == PH_P2) ? 1 : -1;
    constexpr int OUTPAR = (PHASE == PH_P1 || PHASE == PH_P3 || PHASE == PH_R4L) ? 1 : 0;
    constexpr int NRED = (PHASE == PH_P2 || PHASE == PH_P4 || PHASE == PH_R5L) ? 1 : 0;
    using L = Low<LOW>;
    if (eng_ru_phase(PHASE) && *(volatile int *)(P.ctl + 2) == 0) return;  // no reliable update pending
    // 18-real FP16 links: a site's eight links are copied into shared memory once per
    // tile and read from there by each of its right-hand sides.  Not in P4 and R5L,
    // whose epilogues need the resident blocks the 36 KB would cost (measured slower).
    constexpr bool STAGE = LOW == LOW_F16 && FULL18 && PHASE != PH_P4 && PHASE != PH_R5L;
    __shared__ double smem[kEngTile / 32];
    __shared__ bool last;
    __shared__ int s_act[kEngMaxRhs];
    __shared__ int s_na;
    __shared__ uint4 s_lx[STAGE ? 16 * kEngTile : 1];
    __shared__ unsigned s_lz[STAGE ? 8 * kEngTile : 1];
    __shared__ int s_tile;
    __shared__ double s_red[NRED > 0 ? kEngMaxRhs : 1][kEngTile / 32];
    const EngTables *T = P.T;
    const int ntiles = T->ntiles;
    const int max_tiles = T->max_tiles;
    const bool dyn = T->dyn != 0;
    // the next tile: block + k * grid, or the next value of the phase's counter; the
    // partial sums are per (slot, tile), so the tile order does not change any result
    auto next_tile = [&](int cur) {
        if (!dyn) return cur + (int)gridDim.x;
        if (threadIdx.x == 0) s_tile = atomicAdd(P.sched + PHASE, 1);
        __syncthreads();
        return s_tile;
    };
    for (int tile = dyn ? next_tile(0) : (int)blockIdx.x; tile < ntiles; tile = next_tile(tile)) {
        const int l = find_lattice(T, tile);
        const EngLattice &La = T->lat[l];
        const Geom g = La.g;
        const int stride = La.stride;
        const int lt = tile - La.tile0;
        const int i = lt * kEngTile + threadIdx.x;
        const bool valid = i < g.Vh;
        if (threadIdx.x < 32) {
            // the lattice's active slots in list order: one lane per slot, one ballot
            const int q = threadIdx.x;
            int j = 0;
            bool on = false;
            if (q < La.nprob) {
                j = La.prob[q];
                on = active<PHASE>(P.S[j]);
            }
            const unsigned m = __ballot_sync(0xffffffffu, on);
            if (on) s_act[__popc(m & ((1u << q) - 1u))] = j;
            if (q == 0) s_na = __popc(m);
        }
        __syncthreads();
        const int na = s_na;
        if (lt == 0 && threadIdx.x == 0 && na > 0) {
            count_work(P, PHASE, 0, (unsigned long long)na * g.Vh);
            count_work(P, PHASE, 2, g.Vh);
        }
        SiteNbrs nb;
        if (valid && na > 0) nb = site_neighbours(g, i, OUTPAR);
        const LinksF16x18Smem<kEngTile> US{s_lx, s_lz, OUTPAR};
        if constexpr (STAGE) {
            if (valid && na > 0) {
                US.stage(InnerLinks<LOW, FULL18>::lk(La), nb, i);
                cp_async_wait_all();
            }
        }
        for (int g0 = 0; g0 < na; g0 += NR) {
            const int cnt = min(NR, na - g0);
            // the reliable update of M x = b reads FP32 fields: s (in y) and t (in t64)
            constexpr bool ru32 = PHASE == PH_R4L || PHASE == PH_R5L;
            using InSp = typename std::conditional<ru32, SpinorF32, typename L::Sp>::type;
            InSp in[NR];
#pragma unroll
            for (int r = 0; r < NR; r++) {
                const EngProblem &pr = T->prob[s_act[g0 + min(r, cnt - 1)]];
                if constexpr (ru32) {
                    in[r] = SpinorF32{PHASE == PH_R4L ? pr.y : reinterpret_cast<float4 *>(pr.t64), stride};
                } else {
                    void *ip = (PHASE == PH_P1) ? pr.p : (PHASE == PH_P3 ? pr.Dp : pr.t);
                    float *inn = (PHASE == PH_P1) ? pr.pn : (PHASE == PH_P3 ? pr.Dpn : pr.tn);
                    in[r] = L::sp(ip, inn, stride);
                }
            }
            Spinor<float> acc[NR];
#pragma unroll
            for (int r = 0; r < NR; r++)
#pragma unroll
                for (int c = 0; c < 12; c++) acc[r].s[c / 3][c % 3] = {0.f, 0.f};
            if (valid) {
                using Lk = typename std::conditional<STAGE, LinksF16x18Smem<kEngTile>,
                                                     typename InnerLinks<LOW, FULL18>::Lk>::type;
                const Lk U = [&]() -> Lk {
                    if constexpr (STAGE)
                        return US;
                    else
                        return InnerLinks<LOW, FULL18>::lk(La);
                }();
                if constexpr (PK && NR == 2 && std::is_same<InSp, SpinorF16>::value) {
                    // a lone last solve fills both lanes (in[1] repeats in[0]); lane y is dropped
                    Spinor2 a2;
#pragma unroll
                    for (int c = 0; c < 12; c++) a2.s[c / 3][c % 3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
                    hop_dir_pair<0, SIGN>(nb, OUTPAR, i, in[0], in[1], U, a2);
                    hop_dir_pair<1, SIGN>(nb, OUTPAR, i, in[0], in[1], U, a2);
                    hop_dir_pair<2, SIGN>(nb, OUTPAR, i, in[0], in[1], U, a2);
                    hop_dir_pair<3, SIGN>(nb, OUTPAR, i, in[0], in[1], U, a2);
#pragma unroll
                    for (int c = 0; c < 12; c++) {
                        acc[0].s[c / 3][c % 3] = {a2.s[c / 3][c % 3].re.x, a2.s[c / 3][c % 3].im.x};
                        acc[NR - 1].s[c / 3][c % 3] = {a2.s[c / 3][c % 3].re.y, a2.s[c / 3][c % 3].im.y};
                    }
                } else {
                    hop_dir_multi<0, SIGN>(nb, OUTPAR, i, in, cnt, U, acc);
                    hop_dir_multi<1, SIGN>(nb, OUTPAR, i, in, cnt, U, acc);
                    hop_dir_multi<2, SIGN>(nb, OUTPAR, i, in, cnt, U, acc);
                    hop_dir_multi<3, SIGN>(nb, OUTPAR, i, in, cnt, U, acc);
                }
            }
#pragma unroll
            for (int r = 0; r < NR; r++) {
                if (r < cnt) {
                    const int j = s_act[g0 + r];
                    double red[2] = {0.0, 0.0};
                    if (valid) epi_low<PHASE, LOW>(T->prob[j], P.S[j], stride, i, acc[r], red);
                    // each warp keeps its sum in shared memory; the slots' sums are formed
                    // once per tile below, in block_sum's order (one barrier per tile
                    // instead of two per slot)
                    if constexpr (NRED > 0) {
                        const double v = warp_sum(red[0]);
                        if ((threadIdx.x & 31) == 0) s_red[g0 + r][threadIdx.x >> 5] = v;
                    }
                }
            }
        }
        if constexpr (NRED > 0) {
            __syncthreads();
            if (threadIdx.x < na) {
                double sum = 0;
#pragma unroll
                for (int w = 0; w < kEngTile / 32; w++) sum += s_red[threadIdx.x][w];
                P.partials[((size_t)s_act[threadIdx.x] * 2) * max_tiles + lt] = sum;
                __threadfence();  // visible before the lattice's ticket is taken
            }
        }
        __syncthreads();  // s_act is rewritten by the next tile
        if constexpr (NRED > 0) arrive_and_finish<PHASE, NRED>(P, La, l, smem, last, La.ntiles);
    }
}

// FP64 reliable-update phases R2..R5 for lattices whose FP64 links have PLANES
// planes per (parity, dir); a second launch serves the other format if present.
// Work items are (tile, a) pairs, a the position of a slot in the lattice's list
// of slots with a pending reliable update, so each block iteration is one
// independent hop over 128 sites (no loop over slots inside a block) and the
// lattice's last arrival (tiles x active slots of them) runs the finisher.
// Items of one tile are consecutive, so its links are re-read from L2.
template <int PHASE, int LOW, int PLANES>
__global__ void __launch_bounds__(kEngTile, 3) k_eng_f64(EngPtrs P) {
    constexpr int SIGN = (PHASE == PH_R2 || PHASE == PH_R3) ? 1 : -1;
    constexpr int OUTPAR = (PHASE == PH_R2 || PHASE == PH_R4) ? 1 : 0;
    constexpr int NRED = (PHASE == PH_R3 || PHASE == PH_R5) ? 2 : 0;
    using Lk = typename std::conditional<PLANES == 9, LinksF64x18, LinksF64x12>::type;
    __shared__ double smem[kEngTile / 32];
    __shared__ bool last;
    __shared__ ActiveTable act;
    if (*(volatile int *)(P.ctl + 2) == 0) return;  // no reliable update pending
    const EngTables *T = P.T;
    const int nitems = T->ntiles * kEngMaxRhs;
    const int max_tiles = T->max_tiles;
    build_active<PHASE>(P, act);
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int tile = item / kEngMaxRhs, a = item % kEngMaxRhs;
        const int l = find_lattice(T, tile);
        const EngLattice &La = T->lat[l];
        const int na = act.n[l];
        // the a-th slot with a pending update
        if (La.l64_planes != PLANES || a >= na) continue;
        const int j = act.slot[l][a];
        const Geom g = La.g;
        const int stride = La.stride;
        const int lt = tile - La.tile0;
        const int i = lt * kEngTile + threadIdx.x;
        const EngProblem &pr = T->prob[j];
        if (lt == 0 && threadIdx.x == 0) {
            // R3 of a first update from x = 0 runs no hop (below); the links are read
            // once per site when some slot of the lattice runs its hop
            const bool nohop = PHASE == PH_R3 && P.S[j].init && !P.S[j].xnz;
            const int kind = (PHASE == PH_R3 && pr.mode == ENG_MODE_NORMAL) ? 3 : (nohop ? 1 : 0);
            count_work(P, PHASE, kind, (unsigned long long)g.Vh);
            if (a == 0) {
                bool hop = false;
                for (int q = 0; q < na; q++) {
                    const EngState &sq = P.S[act.slot[l][q]];
                    hop |= !(PHASE == PH_R3 && sq.init && !sq.xnz);
                }
                if (hop) count_work(P, PHASE, 2, (unsigned long long)g.Vh);
            }
        }
        double red[2] = {0.0, 0.0};
        if (i < g.Vh) {
            const SiteNbrs nb = site_neighbours(g, i, OUTPAR);
            const Lk U{La.l64, stride};
            const double2 *in = (PHASE == PH_R2) ? pr.x : (PHASE == PH_R4 ? pr.s : pr.t64);
            const SpinorF64 sin{const_cast<double2 *>(in), stride};
            Spinor<double> acc;
#pragma unroll
            for (int c = 0; c < 12; c++) acc.s[c / 3][c % 3] = {0.0, 0.0};
            // R3 of a first update from x = 0: R2 was skipped and H t64 = 0, so s = b with
            // the same bits the hop of zeros would give (b - (+-0) = b)
            const bool zero_in = PHASE == PH_R3 && P.S[j].init && !P.S[j].xnz;
            if (!zero_in) {
                hop_dir_lean<0, SIGN>(nb, OUTPAR, i, sin, U, acc);
                hop_dir_lean<1, SIGN>(nb, OUTPAR, i, sin, U, acc);
                hop_dir_lean<2, SIGN>(nb, OUTPAR, i, sin, U, acc);
                hop_dir_lean<3, SIGN>(nb, OUTPAR, i, sin, U, acc);
            }
            epi_f64<PHASE, LOW>(pr, stride, i, acc, red);
        }
        if constexpr (NRED > 0) {
            // the item's sums with one barrier: warp sums in shared memory, added by thread 0
            // in warp order (block_sum's order, the same bits)
            __shared__ double s_w[NRED][kEngTile / 32];
#pragma unroll
            for (int k = 0; k < NRED; k++) {
                const double v = warp_sum(red[k]);
                if ((threadIdx.x & 31) == 0) s_w[k][threadIdx.x >> 5] = v;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
#pragma unroll
                for (int k = 0; k < NRED; k++) {
                    double sum = 0;
#pragma unroll
                    for (int w = 0; w < kEngTile / 32; w++) sum += s_w[k][w];
                    P.partials[((size_t)j * 2 + k) * max_tiles + lt] = sum;
                }
            }
            arrive_and_finish<PHASE, NRED>(P, La, l, smem, last, La.ntiles * na);
        }
    }
}

// ------------------------------------------------------------------ vector phases

// R1: x += y; y = 0 for the normal system (slots with a pending reliable update)
// P5: p = r + beta p, or p = r on a slot's first iteration (running slots)
template <int PHASE, int LOW>
__global__ void __launch_bounds__(kEngTile) k_eng_vec(EngPtrs P) {
    using L = Low<LOW>;
    if (PHASE == PH_R1 && *(volatile int *)(P.ctl + 2) == 0) return;
    const EngTables *T = P.T;
    const int ntiles = T->ntiles;
    // static tile order: the vector phases are short and bound by DRAM, and the barriers of a
    // dynamic order measured slower here (P5 0.176 -> 0.197 ms at 32^4, 12 sources)
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int l = find_lattice(T, tile);
        const EngLattice &La = T->lat[l];
        const int stride = La.stride;
        const int i = (tile - La.tile0) * kEngTile + threadIdx.x;
        if (i >= La.g.Vh) continue;
        for (int q = 0; q < La.nprob; q++) {
            const int j = La.prob[q];
            const EngState &s = P.S[j];
            if (!active<PHASE>(s)) continue;
            const EngProblem &pr = T->prob[j];
            if (i == 0) {
                const bool alt = PHASE == PH_R1 ? pr.mode == ENG_MODE_NORMAL : s.init != 0;
                count_work(P, PHASE, alt ? 1 : 0, (unsigned long long)La.g.Vh);
            }
            if (PHASE == PH_R1) {
                SpinorF32 ys{pr.y, stride};
                Spinor<float> y;
                ys.load_cached(i, y);
                bool nz = false;
#pragma unroll
                for (int c = 0; c < 12; c++) {
                    Cx<double> xv = ldc(pr.x, stride, c, i);
                    nz |= xv.re != 0.0 || xv.im != 0.0;
                    xv.re += (double)y.s[c / 3][c % 3].re;
                    xv.im += (double)y.s[c / 3][c % 3].im;
                    stc(pr.x, stride, c, i, xv);
                    y.s[c / 3][c % 3] = {0.f, 0.f};
                }
                // first update: record whether the initial x is nonzero anywhere (one atomic
                // per warp at most; the flag is read by R2 and R3 after this launch)
                if (s.init) {
                    const unsigned am = __activemask();
                    if (__any_sync(am, nz) && (threadIdx.x & 31) == __ffs(am) - 1 && !*(volatile int *)&P.S[j].xnz)
                        atomicOr(&P.S[j].xnz, 1);
                }
                // M x = b: R3 overwrites y with s and R5L clears it, so only the normal system clears here
                if (pr.mode == ENG_MODE_NORMAL) ys.store(i, y);
            } else {
                Spinor<float> r, p;
                L::sp(pr.r, pr.rn, stride).load_cached(i, r);
                if (s.init) {
                    L::sp(pr.p, pr.pn, stride).store(i, r);
                } else {
                    const float beta = (float)s.beta;
                    L::sp(pr.p, pr.pn, stride).load_cached(i, p);
#pragma unroll
                    for (int c = 0; c < 12; c++) p.s[c / 3][c % 3] = r.s[c / 3][c % 3] + beta * p.s[c / 3][c % 3];
                    L::sp(pr.p, pr.pn, stride).store(i, p);
                }
            }
        }
    }
}

// One block: end of an iteration.  Clears the first-iteration flags, counts
// running slots, and keeps the chunk's WHILE loop going while some slot runs
// and fewer than `chunk` iterations ran.  No waiting: the loop is bounded by
// `chunk` and by every slot's maxiter.
__global__ void k_eng_control(EngPtrs P, int nprob, int chunk, cudaGraphConditionalHandle h, int use_cond) {
    __shared__ int running;
    if (threadIdx.x == 0) running = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < nprob; j += blockDim.x) {
        EngState &s = P.S[j];
        if (s.status == ENG_RUNNING && s.ru == 0 && s.init) s.init = 0;
        if (s.status == ENG_RUNNING) atomicAdd(&running, 1);
    }
    __syncthreads();
    if (threadIdx.x < kEngPhases) P.sched[threadIdx.x] = 0;  // the next iteration's tile counters
    if (threadIdx.x == 0) {
        if (chunk <= 0) chunk = P.ctl[3];
        const int it = P.ctl[0] + 1;
        P.ctl[0] = it;
        P.ctl[1] = running;
        P.ctl[2] = 0;  // pending reliable updates were served this iteration
        reinterpret_cast<unsigned long long *>(P.ctl + 6)[0] += 1;  // loop bodies since init
        if (use_cond) cudaGraphSetConditional(h, (running > 0 && it < chunk) ? 1u : 0u);
    }
}

__global__ void k_eng_chunk_begin(EngPtrs P) {
    P.ctl[0] = 0;
    for (int k = 0; k < kEngPhases; k++) P.sched[k] = 0;
}

// FP64 link planes (first six elements = rows 0 and 1) -> FP32 / FP16 12-real planes
__global__ void k_eng_links(Geom g, const double2 *l64, int planes, int stride, float4 *l32, uint4 *l16a,
                            uint2 *l16b, float4 *l32a, float2 *l32b, uint4 *l16x, unsigned *l16z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int pd = blockIdx.y;  // parity*4 + dir
    if (i >= g.Vh) return;
    if (l16x) {
        // all 18 reals; a 12-real FP64 source gets its third row rebuilt in FP64 first
        Su3<double> u;
        for (int k = 0; k < 9; k++) {
            if (k < planes) {
                double2 v = l64[((size_t)pd * planes + k) * stride + i];
                u.e[k / 3][k % 3] = {v.x, v.y};
            }
        }
        if (planes == 6) reconstruct_row2(u);
        __half2 h[9];
#pragma unroll
        for (int k = 0; k < 9; k++) h[k] = __floats2half2_rn((float)u.e[k / 3][k % 3].re, (float)u.e[k / 3][k % 3].im);
        l16x[(size_t)(2 * pd) * stride + i] = *reinterpret_cast<const uint4 *>(&h[0]);
        l16x[(size_t)(2 * pd + 1) * stride + i] = *reinterpret_cast<const uint4 *>(&h[4]);
        l16z[(size_t)pd * stride + i] = *reinterpret_cast<const unsigned *>(&h[8]);
    }
    if (l32a) {
        Su3<double> u;
        for (int k = 0; k < 9; k++) {
            if (k < planes) {
                double2 v = l64[((size_t)pd * planes + k) * stride + i];
                u.e[k / 3][k % 3] = {v.x, v.y};
            }
        }
        if (planes == 6) reconstruct_row2(u);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int e0 = 2 * k, e1 = 2 * k + 1;
            l32a[((size_t)pd * 4 + k) * stride + i] =
                make_float4((float)u.e[e0 / 3][e0 % 3].re, (float)u.e[e0 / 3][e0 % 3].im,
                            (float)u.e[e1 / 3][e1 % 3].re, (float)u.e[e1 / 3][e1 % 3].im);
        }
        l32b[(size_t)pd * stride + i] = make_float2((float)u.e[2][2].re, (float)u.e[2][2].im);
    }
    float e[12];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        double2 v = l64[((size_t)pd * planes + k) * stride + i];
        e[2 * k] = (float)v.x;
        e[2 * k + 1] = (float)v.y;
    }
    if (l32) {
#pragma unroll
        for (int k = 0; k < 3; k++)
            l32[((size_t)pd * 3 + k) * stride + i] = make_float4(e[4 * k], e[4 * k + 1], e[4 * k + 2], e[4 * k + 3]);
    }
    if (l16a) {
        uint4 a;
        uint2 b;
        __half2 *ha = reinterpret_cast<__half2 *>(&a);
        __half2 *hb = reinterpret_cast<__half2 *>(&b);
#pragma unroll
        for (int k = 0; k < 4; k++) ha[k] = __floats2half2_rn(e[2 * k], e[2 * k + 1]);
#pragma unroll
        for (int k = 0; k < 2; k++) hb[k] = __floats2half2_rn(e[8 + 2 * k], e[9 + 2 * k]);
        l16a[(size_t)pd * stride + i] = a;
        l16b[(size_t)pd * stride + i] = b;
    }
}

template <int PHASE, int LOW>
void launch_f64(const EngPtrs &P, const EngGrid &G, cudaStream_t s) {
    if (G.planes_mask & 1) k_eng_f64<PHASE, LOW, 9><<<G.f64, kEngTile, 0, s>>>(P);
    if (G.planes_mask & 2) k_eng_f64<PHASE, LOW, 6><<<G.f64, kEngTile, 0, s>>>(P);
}

// profiling marks: ev (when not null) holds kEngPhases + 1 events, ev[k] recorded before phase k
inline void mark(const cudaEvent_t *ev, int k, cudaStream_t s) {
    if (ev) cudaEventRecord(ev[k], s);
}

// R1..R5L and P5 (phases 4..11), shared by every launch shape of the inner phases;
// LowRU launches R4L / R5L in the inner phases' shape
template <int LOW, class LowRU>
void enqueue_reliable_update(const EngPtrs &P, const EngGrid &G, cudaStream_t s, const cudaEvent_t *ev) {
    k_eng_vec<PH_R1, LOW><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, PH_R2, s);
    launch_f64<PH_R2, LOW>(P, G, s);
    mark(ev, PH_R3, s);
    launch_f64<PH_R3, LOW>(P, G, s);
    mark(ev, PH_R4, s);
    launch_f64<PH_R4, LOW>(P, G, s);
    mark(ev, PH_R4L, s);
    LowRU::template launch<PH_R4L>(P, G, s);
    mark(ev, PH_R5, s);
    launch_f64<PH_R5, LOW>(P, G, s);
    mark(ev, PH_R5L, s);
    LowRU::template launch<PH_R5L>(P, G, s);
    mark(ev, PH_P5, s);
    k_eng_vec<PH_P5, LOW><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, kEngPhases, s);
}

template <int LOW, int NR, int MINB, bool FULL18, bool PK = false>
struct LowShape {
    template <int PHASE>
    static void launch(const EngPtrs &P, const EngGrid &G, cudaStream_t s) {
        k_eng_low<PHASE, LOW, NR, MINB, FULL18, PK><<<G.low, kEngTile, 0, s>>>(P);
    }
};

template <int LOW, int NR, int MINB, bool FULL18, bool PK = false>
void enqueue_iteration_t(const EngPtrs &P, const EngGrid &G, cudaStream_t s, const cudaEvent_t *ev) {
    mark(ev, 0, s);
    k_eng_low<PH_P1, LOW, NR, MINB, FULL18, PK><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, 1, s);
    k_eng_low<PH_P2, LOW, NR, MINB, FULL18, PK><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, 2, s);
    k_eng_low<PH_P3, LOW, NR, MINB, FULL18, PK><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, 3, s);
    k_eng_low<PH_P4, LOW, NR, MINB, FULL18, PK><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, 4, s);
    enqueue_reliable_update<LOW, LowShape<LOW, NR, MINB, FULL18, PK>>(P, G, s, ev);
}

// P1 and P3 with two solves per thread in packed FP32 (MINB_PK blocks per SM, G.pk
// blocks), P2, P4 and the reliable update in the shape of variant 2 (G.low blocks)
template <int LOW, int MINB_PK, bool FULL18>
void enqueue_iteration_hybrid(const EngPtrs &P, const EngGrid &G, cudaStream_t s, const cudaEvent_t *ev) {
    mark(ev, 0, s);
    k_eng_low<PH_P1, LOW, 2, MINB_PK, FULL18, true><<<G.pk, kEngTile, 0, s>>>(P);
    mark(ev, 1, s);
    k_eng_low<PH_P2, LOW, 1, 6, FULL18><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, 2, s);
    k_eng_low<PH_P3, LOW, 2, MINB_PK, FULL18, true><<<G.pk, kEngTile, 0, s>>>(P);
    mark(ev, 3, s);
    k_eng_low<PH_P4, LOW, 1, 6, FULL18><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, 4, s);
    enqueue_reliable_update<LOW, LowShape<LOW, 1, 6, FULL18>>(P, G, s, ev);
}

constexpr int kMmaMinBlocks = 4;

// FP16 inner phases on the tensor cores (engine_mma.cuh), the rest as usual
void enqueue_iteration_mma(const EngPtrs &P, const EngGrid &G, cudaStream_t s, const cudaEvent_t *ev) {
    mark(ev, 0, s);
    k_eng_mma<PH_P1, kMmaMinBlocks><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, 1, s);
    k_eng_mma<PH_P2, kMmaMinBlocks><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, 2, s);
    k_eng_mma<PH_P3, kMmaMinBlocks><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, 3, s);
    k_eng_mma<PH_P4, kMmaMinBlocks><<<G.low, kEngTile, 0, s>>>(P);
    mark(ev, 4, s);
    enqueue_reliable_update<LOW_F16, LowShape<LOW_F16, 1, 6, true>>(P, G, s, ev);
}

// Launch shapes of the low-precision phases (EngGrid::variant):
//   2: one right-hand side per thread, <= 85 registers (6 blocks of 128 per SM); the FP32 default
//   4: FP16 only: the hop as tensor-core products over groups of sources (engine_mma.cuh)
//   7: FP16 only, the default: P1, P3 with two right-hand sides per thread in the lanes of
//      packed FP32 instructions (pair.cuh), <= 168 registers (3 blocks); P2, P4 and the
//      reliable update as variant 2
// 2 and 7 round every operation alike (same bits); the engine's tuner picks between them
// by timing (engine.cpp).  4 sums its products in another order.
// (one right-hand side per thread at 4 or 5 blocks per SM, two per thread sharing the links
// without packing, packed P1..P4, packed P1..P3, and P1/P3 streaming their neighbour data
// through a cp.async ring in shared memory were measured slower or no faster and removed)
template <int LOW, bool FULL18>
void enqueue_iteration_v(const EngPtrs &P, const EngGrid &G, cudaStream_t s, const cudaEvent_t *ev) {
    if constexpr (LOW == LOW_F16) {
        if (G.variant == 4) {
            enqueue_iteration_mma(P, G, s, ev);
            return;
        }
        if (G.variant == 7) {
            enqueue_iteration_hybrid<LOW, 3, FULL18>(P, G, s, ev);
            return;
        }
    }
    enqueue_iteration_t<LOW, 1, 6, FULL18>(P, G, s, ev);
}

template <int LOW>
void enqueue_iteration_nr(const EngPtrs &P, const EngGrid &G, cudaStream_t s, const cudaEvent_t *ev) {
    if (G.full18)
        enqueue_iteration_v<LOW, true>(P, G, s, ev);
    else
        enqueue_iteration_v<LOW, false>(P, G, s, ev);
}

}  // namespace

void eng_enqueue_iteration(int low, const EngPtrs &P, const EngGrid &G, cudaStream_t s, const cudaEvent_t *ev) {
    if (G.fermions & 1) {
        if (low == LOW_F16)
            enqueue_iteration_nr<LOW_F16>(P, G, s, ev);
        else
            enqueue_iteration_nr<LOW_F32>(P, G, s, ev);
    }
    // staggered phases after the Wilson ones (outside the profiling events)
    if (G.fermions & 2) enqueue_stag_iteration(P, G, s);
}

void eng_enqueue_control(const EngPtrs &P, int nprob, int chunk, cudaGraphConditionalHandle h, int use_cond,
                         cudaStream_t s) {
    k_eng_control<<<1, 64, 0, s>>>(P, nprob, chunk, h, use_cond);
}

void eng_enqueue_chunk_begin(const EngPtrs &P, cudaStream_t s) { k_eng_chunk_begin<<<1, 1, 0, s>>>(P); }

void eng_convert_links(const Geom &g, const double2 *l64, int planes, int stride, float4 *l32, uint4 *l16a,
                       uint2 *l16b, float4 *l32a, float2 *l32b, uint4 *l16x, unsigned *l16z, cudaStream_t s) {
    dim3 grid((g.Vh + 255) / 256, 8);
    k_eng_links<<<grid, 256, 0, s>>>(g, l64, planes, stride, l32, l16a, l16b, l32a, l32b, l16x, l16z);
}

template <int LOW, int NR, int MINB, bool PK = false, int PHASE = PH_P4>
int occupancy_low() {
    int lo = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&lo, k_eng_low<PHASE, LOW, NR, MINB, true, PK>, kEngTile, 0);
    return lo < 1 ? 1 : lo;
}

template <int LOW>
int occupancy_variant(int v) {
    if (LOW == LOW_F16 && v == 4) {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_eng_mma<PH_P4, kMmaMinBlocks>, kEngTile, 0);
        return n < 1 ? 1 : n;
    }
    return occupancy_low<LOW, 1, 6>();
}

EngGrid eng_grid_size(int low, int variant, int full18, int planes_mask) {
    int dev = 0, sms = 148, lo = 1, hi = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    lo = low == LOW_F16 ? occupancy_variant<LOW_F16>(variant) : occupancy_variant<LOW_F32>(variant);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&hi, k_eng_f64<PH_R5, LOW_F32, 9>, kEngTile, 0);
    EngGrid G;
    G.low = sms * lo;
    G.pk = G.low;
    if (variant == 7 && low == LOW_F16) G.pk = sms * occupancy_low<LOW_F16, 2, 3, true, PH_P1>();
    G.f64 = sms * (hi < 1 ? 1 : hi);
    G.fermions = 1;
    G.variant = variant;
    G.full18 = full18;
    G.planes_mask = planes_mask;
    return G;
}

}  // namespace hw
