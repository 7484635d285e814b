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
        const HalfStag x{pr.x, stride}, b{pr.b, stride}, sv{pr.s, stride};
        const HalfStag p{static_cast<double2 *>(pr.p), stride}, r{static_cast<double2 *>(pr.r), stride};
        const HalfStag Dp{static_cast<double2 *>(pr.Dp), stride}, t{static_cast<double2 *>(pr.t), stride};
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
                } else if constexpr (PHASE == PH_R5L) {  // r = M^dag s
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const Cx<double> v = m * sv.ld(c, i) + h[c];
                        r.st(c, i, v);
                        red[0] += norm2(v);
                    }
                } else if constexpr (PHASE == PH_R5) {  // r = b - M^dag M x
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const Cx<double> bv = b.ld(c, i);
                        const Cx<double> v = bv - (m * sv.ld(c, i) + h[c]);
                        r.st(c, i, v);
                        red[0] += norm2(v);
                        red[1] += norm2(bv);
                    }
                }
            }
        }
        if constexpr (NRED > 0) {
#pragma unroll
            for (int k = 0; k < NRED; k++) {
                const double sum = block_sum<kEngTile>(red[k], smem);
                if (threadIdx.x == 0) P.partials[((size_t)j * 2 + k) * max_tiles + lt] = sum;
            }
            arrive_and_finish<PHASE, NRED, FERM_STAGGERED>(P, La, l, smem, last, La.ntiles * na);
        }
    }
}

// one iteration of the staggered slots (the reliable-update phases return at once unless
// some slot asked for one)
void enqueue_stag_iteration(const EngPtrs &P, const EngGrid &G, cudaStream_t s) {
    k_stag_eng<PH_P1><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_P2><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_P3><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_P4><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R1><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R2><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R3><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R4><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R4L><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R5><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_R5L><<<G.f64, kEngTile, 0, s>>>(P);
    k_stag_eng<PH_P5><<<G.f64, kEngTile, 0, s>>>(P);
}
