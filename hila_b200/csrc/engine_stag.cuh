// Staggered fermions on the solver engine (engine.h lists the phases).  Included by
// engine.cu inside its anonymous namespace, after the finishers: the staggered slots
// share the Wilson slots' tables, states, finishers, per-(slot, tile) reductions and
// chunk graphs, so staggered and Wilson solves run in the same batches and through the
// same server, and a solve is bitwise the same alone and in any batch.
//
// The operator is dirac_staggered_evenodd (staggered.h:193-279) as the reference codes
// it: M_s in = m in_e + D^{eo}_s (1/m) D^{oe}_s in_e with D_s = 0.5 s hop, M^dag = M_{-s}.
// Everything runs in FP64 (the colour vector is small, the phases are bound by memory
// and latency); the low-precision buffers of a slot hold FP64 half lattices here (3
// double2 planes: 48 bytes per site, the size of a Wilson FP16 buffer).  Work items are
// (tile, active slot) pairs as in the Wilson FP64 phases.  The site algebra comes from
// staggered_math.cuh, which engine.cu includes at file scope.
#pragma once

// An FP16 colour-vector half lattice of a low-precision staggered slot: the three
// colours as (re, im) half pairs in the first uint4 plane of the slot's buffer (the
// fourth word unused) and a per-site scale, the largest |component| of the site.
struct HalfStag16 {
    uint4 *p;
    float *n;
    __device__ __forceinline__ static void unpack(uint4 v, float s, Cx<float> w[3]) {
        const __half2 *h = reinterpret_cast<const __half2 *>(&v);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float2 f = __half22float2(h[c]);
            w[c] = {f.x * s, f.y * s};
        }
    }
    __device__ __forceinline__ void ld(int i, Cx<float> w[3]) const { unpack(__ldg(p + i), __ldg(n + i), w); }
    // plain (coherent) load, for arrays the same kernel also writes
    __device__ __forceinline__ void ldp(int i, Cx<float> w[3]) const { unpack(p[i], n[i], w); }
    __device__ __forceinline__ void st(int i, const Cx<float> w[3]) const {
        float m = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) m = fmaxf(m, fmaxf(fabsf(w[c].re), fabsf(w[c].im)));
        const float inv = m > 0.f ? 1.0f / m : 0.f;
        n[i] = m;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        __half2 *h = reinterpret_cast<__half2 *>(&v);
#pragma unroll
        for (int c = 0; c < 3; c++) h[c] = __floats2half2_rn(w[c].re * inv, w[c].im * inv);
        p[i] = v;
    }
};

// The FP32 solution increment y of a low-precision staggered slot: colour c of site i at
// y[c * stride + i] (the slot's y buffer viewed as float2 planes).
struct HalfStagY {
    float2 *p;
    int stride;
    __device__ __forceinline__ Cx<float> ld(int c, int i) const {
        const float2 v = p[(size_t)c * stride + i];
        return {v.x, v.y};
    }
    __device__ __forceinline__ void st(int c, int i, Cx<float> v) const {
        p[(size_t)c * stride + i] = make_float2(v.re, v.im);
    }
};

// stag_hop_site in FP32 from FP16 fields and 18-real FP16 links (from memory, or the
// tile's copy in shared memory); n: the neighbours of site i of output parity par
template <class Lk>
__device__ __forceinline__ void stag_hop_site_low(const Geom &g, const Lk &U, const SiteNbrs &n, int par, int i,
                                                  const HalfStag16 &v, Cx<float> acc[3]) {
    int c[4];
    site_coords(g, i, par, c);
#pragma unroll
    for (int a = 0; a < 3; a++) acc[a] = {0.f, 0.f};
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const float eta = (float)stag_eta(c, d);
        const float sf = (d == 3 && n.tfwd_wrap) ? -eta : eta;
        const float sb = (d == 3 && n.tbwd_wrap) ? -eta : eta;
        Su3<float> u;
        Cx<float> w[3];
        U.load(par, d, i, u);
        v.ld(n.fwd[d], w);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const Cx<float> t = cmul(u.e[a][0], w[0]) + cmul(u.e[a][1], w[1]) + cmul(u.e[a][2], w[2]);
            acc[a] = acc[a] + sf * t;
        }
        U.load(1 - par, d, n.bwd[d], u);
        v.ld(n.bwd[d], w);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const Cx<float> t = cmul(conj(u.e[0][a]), w[0]) + cmul(conj(u.e[1][a]), w[1]) + cmul(conj(u.e[2][a]), w[2]);
            acc[a] = acc[a] - sb * t;
        }
    }
}

// P1..P5 of a low-precision staggered slot at site i (FP32 arithmetic, FP16 fields);
// red[0] receives the phase's |.|^2 contribution
template <int PHASE, class Lk>
__device__ __forceinline__ void stag_low_site(const EngLattice &La, const EngProblem &pr, const EngState &st,
                                              const Lk &U, const SiteNbrs &nb, int i, double *red) {
    constexpr int SIGN = (PHASE == PH_P1 || PHASE == PH_P2) ? 1 : -1;
    constexpr int OUTPAR = (PHASE == PH_P1 || PHASE == PH_P3) ? 1 : 0;
    const int stride = La.stride;
    const float m = (float)pr.kappa;  // the mass
    const HalfStag16 p{static_cast<uint4 *>(pr.p), pr.pn}, r{static_cast<uint4 *>(pr.r), pr.rn};
    const HalfStag16 Dp{static_cast<uint4 *>(pr.Dp), pr.Dpn}, t{static_cast<uint4 *>(pr.t), pr.tn};
    if constexpr (PHASE == PH_P5) {
        Cx<float> rv[3], pv[3];
        r.ld(i, rv);
        if (!st.init) {
            const float beta = (float)st.beta;
            p.ldp(i, pv);
#pragma unroll
            for (int c = 0; c < 3; c++) rv[c] = rv[c] + beta * pv[c];
        }
        p.st(i, rv);
    } else {
        const HalfStag16 in = PHASE == PH_P1 ? p : PHASE == PH_P3 ? Dp : t;
        Cx<float> acc[3], h[3];
        stag_hop_site_low(La.g, U, nb, OUTPAR, i, in, acc);
#pragma unroll
        for (int c = 0; c < 3; c++) h[c] = (0.5f * SIGN) * acc[c];
        if constexpr (OUTPAR == 1) {  // P1, P3: t = (1/m) D in
            const float im = 1.0f / m;
#pragma unroll
            for (int c = 0; c < 3; c++) h[c] = im * h[c];
            t.st(i, h);
        } else if constexpr (PHASE == PH_P2) {  // Dp = m p + D t
            Cx<float> pv[3];
            p.ld(i, pv);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                h[c] = m * pv[c] + h[c];
                red[0] += (double)norm2(h[c]);
            }
            Dp.st(i, h);
        } else {  // P4: r -= alpha (m Dp + D t), y += alpha p
            const float alpha = (float)st.alpha;
            Cx<float> dv[3], rv[3], pv[3];
            Dp.ld(i, dv);
            r.ldp(i, rv);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                rv[c] = rv[c] - alpha * (m * dv[c] + h[c]);
                red[0] += (double)norm2(rv[c]);
            }
            r.st(i, rv);
            p.ld(i, pv);
            const HalfStagY y{reinterpret_cast<float2 *>(pr.y), stride};
#pragma unroll
            for (int c = 0; c < 3; c++) y.st(c, i, y.ld(c, i) + alpha * pv[c]);
        }
    }
}

// P1..P5 of the staggered slots with FP16 inner iterations, in the shape of the Wilson
// inner phases: a block walks tiles (block + k x grid); per tile, the sites' eight FP16
// links are copied into shared memory once and read from there by every such slot of the
// lattice, and each slot's partial sum is formed once per tile in block_sum's order.
template <int PHASE>
__global__ void __launch_bounds__(kEngTile, 4) k_stag_low(EngPtrs P) {
    constexpr int OUTPAR = (PHASE == PH_P1 || PHASE == PH_P3) ? 1 : 0;
    constexpr int NRED = (PHASE == PH_P2 || PHASE == PH_P4) ? 1 : 0;
    constexpr bool HOP = PHASE != PH_P5;
    __shared__ double smem[kEngTile / 32];
    __shared__ bool last;
    __shared__ int s_act[kEngMaxRhs];
    __shared__ int s_na;
    __shared__ uint4 s_lx[HOP ? 16 * kEngTile : 1];
    __shared__ unsigned s_lz[HOP ? 8 * kEngTile : 1];
    __shared__ double s_red[NRED > 0 ? kEngMaxRhs : 1][kEngTile / 32];
    const EngTables *T = P.T;
    const int ntiles = T->ntiles;
    const int max_tiles = T->max_tiles;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int l = find_lattice(T, tile);
        const EngLattice &La = T->lat[l];
        if (La.fermion != FERM_STAGGERED) continue;
        const int lt = tile - La.tile0;
        const int i = lt * kEngTile + threadIdx.x;
        const bool valid = i < La.g.Vh;
        if (threadIdx.x < 32) {
            const int q = threadIdx.x;
            int j = 0;
            bool on = false;
            if (q < La.nprob) {
                j = La.prob[q];
                on = active<PHASE, FERM_STAGGERED_LOW>(P.S[j]);
            }
            const unsigned m = __ballot_sync(0xffffffffu, on);
            if (on) s_act[__popc(m & ((1u << q) - 1u))] = j;
            if (q == 0) s_na = __popc(m);
        }
        __syncthreads();
        const int na = s_na;
        // every tile of a lattice sees the same active slots: a lattice without any is left
        // alone (no arrival, its ticket untouched)
        if (na == 0) {
            __syncthreads();
            continue;
        }
        const LinksF16x18Smem<kEngTile> US{s_lx, s_lz, OUTPAR};
        SiteNbrs nb;
        if constexpr (HOP) {
            if (valid) {
                nb = site_neighbours(La.g, i, OUTPAR);
                US.stage(LinksF16x18{La.l16x, La.l16z, La.stride}, nb, i);
                cp_async_wait_all();
            }
        }
        for (int a = 0; a < na; a++) {
            const int j = s_act[a];
            double red[1] = {0.0};
            if (valid) stag_low_site<PHASE>(La, T->prob[j], P.S[j], US, nb, i, red);
            if constexpr (NRED > 0) {
                const double v = warp_sum(red[0]);
                if ((threadIdx.x & 31) == 0) s_red[a][threadIdx.x >> 5] = v;
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
        __syncthreads();  // s_act and the staged links are rewritten by the next tile
        if constexpr (NRED > 0) arrive_and_finish<PHASE, NRED, FERM_STAGGERED_LOW>(P, La, l, smem, last, La.ntiles);
    }
}

template <int PHASE>
__global__ void __launch_bounds__(kEngTile, 3) k_stag_eng(EngPtrs P) {
    constexpr int SIGN = (PHASE == PH_P1 || PHASE == PH_P2 || PHASE == PH_R2 || PHASE == PH_R3) ? 1 : -1;
    constexpr int OUTPAR =
        (PHASE == PH_P1 || PHASE == PH_P3 || PHASE == PH_R2 || PHASE == PH_R4 || PHASE == PH_R4L) ? 1 : 0;
    constexpr int NRED = (PHASE == PH_P2 || PHASE == PH_P4 || PHASE == PH_R5L) ? 1
                         : (PHASE == PH_R3 || PHASE == PH_R5)                   ? 2
                                                                                : 0;
    constexpr bool HOP = PHASE != PH_R1 && PHASE != PH_P5;
    __shared__ double smem[kEngTile / 32];
    __shared__ bool last;
    __shared__ ActiveTable act;
    if (eng_ru_phase(PHASE) && *(volatile int *)(P.ctl + 2) == 0) return;  // no reliable update pending
    const EngTables *T = P.T;
    const int nitems = T->ntiles * kEngMaxRhs;
    const int max_tiles = T->max_tiles;
    build_active<PHASE, FERM_STAGGERED>(P, act);
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int tile = item / kEngMaxRhs, a = item % kEngMaxRhs;
        const int l = find_lattice(T, tile);
        const EngLattice &La = T->lat[l];
        const int na = act.n[l];
        if (La.fermion != FERM_STAGGERED || a >= na) continue;
        const int j = act.slot[l][a];
        const Geom g = La.g;
        const int stride = La.stride;
        const int lt = tile - La.tile0;
        const int i = lt * kEngTile + threadIdx.x;
        const EngProblem &pr = T->prob[j];
        const EngState &st = P.S[j];
        const double m = pr.kappa;  // the mass of a staggered solve
        const bool low = pr.stag_low != 0;
        const HalfStag x{pr.x, stride}, b{pr.b, stride}, sv{pr.s, stride};
        const HalfStag p{static_cast<double2 *>(pr.p), stride}, r{static_cast<double2 *>(pr.r), stride};
        const HalfStag Dp{static_cast<double2 *>(pr.Dp), stride};
        // the odd FP64 half of the reliable update: t itself, or t64 beside the FP16 t
        const HalfStag t{low ? pr.t64 : static_cast<double2 *>(pr.t), stride};
        double red[2] = {0.0, 0.0};
        if (i < g.Vh) {
            if constexpr (PHASE == PH_R1) {
                // first update: record whether the initial x is nonzero anywhere (read by R2, R3)
                bool nz = false;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const Cx<double> v = x.ld(c, i);
                    nz |= v.re != 0.0 || v.im != 0.0;
                }
                const unsigned am = __activemask();
                if (st.init && __any_sync(am, nz) && (threadIdx.x & 31) == __ffs(am) - 1 &&
                    !*(volatile int *)&P.S[j].xnz)
                    atomicOr(&P.S[j].xnz, 1);
                if (low) {  // x += y, y = 0
                    const HalfStagY y{reinterpret_cast<float2 *>(pr.y), stride};
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const Cx<float> yv = y.ld(c, i);
                        const Cx<double> xv = x.ldp(c, i);
                        x.st(c, i, {xv.re + (double)yv.re, xv.im + (double)yv.im});
                        y.st(c, i, {0.f, 0.f});
                    }
                }
            } else if constexpr (PHASE == PH_P5) {
                const double beta = st.beta;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const Cx<double> rv = r.ld(c, i);
                    p.st(c, i, st.init ? rv : rv + beta * p.ldp(c, i));
                }
            } else {
                static_assert(HOP, "hop phases");
                const HalfStag in = PHASE == PH_P1 ? p : PHASE == PH_P3 ? Dp : PHASE == PH_R2 ? x
                                                     : (PHASE == PH_R4 || PHASE == PH_R4L) ? sv
                                                                                          : t;
                // R3 of a first update from x = 0: R2 did not run and the hop of zeros is zero
                const bool zero_in = PHASE == PH_R3 && st.init && !st.xnz;
                Cx<double> acc[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
                if (!zero_in) {
                    if (La.l64_planes == 9)
                        stag_hop_site(g, LinksF64x18{La.l64, stride}, OUTPAR, i, in, acc);
                    else
                        stag_hop_site(g, LinksF64x12{La.l64, stride}, OUTPAR, i, in, acc);
                }
                Cx<double> h[3];
#pragma unroll
                for (int c = 0; c < 3; c++) h[c] = (0.5 * SIGN) * acc[c];
                if constexpr (OUTPAR == 1) {  // P1, P3, R2, R4, R4L: t = (1/m) D in
                    const double im = 1.0 / m;
#pragma unroll
                    for (int c = 0; c < 3; c++) t.st(c, i, im * h[c]);
                } else if constexpr (PHASE == PH_P2) {  // Dp = m p + D t
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const Cx<double> v = m * p.ld(c, i) + h[c];
                        Dp.st(c, i, v);
                        red[0] += norm2(v);
                    }
                } else if constexpr (PHASE == PH_P4) {  // r -= alpha (m Dp + D t), x += alpha p
                    const double alpha = st.alpha;
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const Cx<double> ddp = m * Dp.ld(c, i) + h[c];
                        const Cx<double> rv = r.ldp(c, i) - alpha * ddp;
                        r.st(c, i, rv);
                        x.st(c, i, x.ldp(c, i) + alpha * p.ld(c, i));
                        red[0] += norm2(rv);
                    }
                } else if constexpr (PHASE == PH_R3) {  // s = b - M x (solve) or s = M x (normal)
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const Cx<double> mx = m * x.ld(c, i) + h[c];
                        if (pr.mode == ENG_MODE_SOLVE) {
                            const Cx<double> bv = b.ld(c, i);
                            const Cx<double> v = bv - mx;
                            sv.st(c, i, v);
                            red[0] += norm2(v);
                            red[1] += norm2(bv);
                        } else {
                            sv.st(c, i, mx);
                        }
                    }
                } else if constexpr (PHASE == PH_R5L || PHASE == PH_R5) {
                    // R5L: r = M^dag s; R5: r = b - M^dag M x (normal system); FP16 r for a
                    // low-precision slot
                    Cx<float> rl[3];
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        Cx<double> v = m * sv.ld(c, i) + h[c];
                        if (PHASE == PH_R5) {
                            const Cx<double> bv = b.ld(c, i);
                            v = bv - v;
                            red[1] += norm2(bv);
                        }
                        red[0] += norm2(v);
                        if (low)
                            rl[c] = {(float)v.re, (float)v.im};
                        else
                            r.st(c, i, v);
                    }
                    if (low) HalfStag16{static_cast<uint4 *>(pr.r), pr.rn}.st(i, rl);
                }
            }
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
            arrive_and_finish<PHASE, NRED, FERM_STAGGERED>(P, La, l, smem, last, La.ntiles * na);
        }
    }
}

// one iteration of the staggered slots (the reliable-update phases return at once unless
// some slot asked for one)
void enqueue_stag_iteration(const EngPtrs &P, const EngGrid &G, cudaStream_t s) {
    // FP64 and FP16 slots of a phase are disjoint; each kernel finishes its own
    k_stag_eng<PH_P1><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_low<PH_P1><<<G.low, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_P2><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_low<PH_P2><<<G.low, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_P3><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_low<PH_P3><<<G.low, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_P4><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_low<PH_P4><<<G.low, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R1><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R2><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R3><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R4><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R4L><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R5><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R5L><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_P5><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_low<PH_P5><<<G.low, kEngTile, 0, s>>>(P);
}
