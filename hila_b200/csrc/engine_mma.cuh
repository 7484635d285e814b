// Tensor-core hopping term of the FP16 engine phases P1..P4 (included by
// engine.cu inside its anonymous namespace, after the epilogues and finishers).
//
// For one output site x and a group of RG right-hand sides, the hop
// (H_s psi)(x) = sum_mu E_{mu,s}(U_mu(x) P_{mu,s} psi(x+mu))
//              + E_{mu,-s}(U_mu(x-mu)^dag P_{mu,-s} psi(x-mu))
// (wilson.h:15-50 with the backward term at x-mu, projection and expansion
// tables of wilson_vector.h:439-567) is, per direction mu, one small real
// matrix product accumulated over mu:
//
//   C[m][n] += sum_k A[m][k] B[k][n]
//   m = 4 r + 2 ul + sigma   r: source within the group; ul = 0: upper spins
//                            (the projection itself), ul = 1: lower spins (the
//                            expansion's phase-permuted copy); sigma: spin in the pair
//   k = 8 b + 2 c' + ri      b = 0: forward (x+mu), 1: backward (x-mu);
//                            c' colour (c' = 3 is zero padding); ri: re / im
//   n = 2 c + ri_out         output colour and re / im (n = 6, 7 padding)
//
// The lower-spin rows use E's phase permutation before the colour product,
// which commutes with it (the phase is a complex scalar).  A row r is scaled by
// the neighbour's FP16 norm over the largest of the 8 neighbour norms of
// (x, r), so |A| <= 2 in FP16; C is multiplied back by that largest norm.  B is
// U_mu(x) or U_mu(x-mu)^dag in real form, from the 18-real FP16 link copy.
// One mma.sync.m16n8k16 (FP16 operands, FP32 accumulation) applies a link
// pair to four sources at once.
//
// Work split: each warp owns 32 consecutive sites of the block's tile.  For a
// group of RG sources (4 or 8) it takes SG = 32 / RG sites at a time; lane
// (s, r) = (lane / RG, lane % RG) stages the eight projected neighbours of
// (site s, source r) into shared memory, one direction per round so every lane
// runs the same projection, then the warp runs the MMAs site by site, writes C
// back through shared memory and lane (s, r) applies the phase epilogue of
// (site s, source r) exactly as the scalar kernels do.  Dot products are summed
// per source over the warp's sites in site order and over the warps in warp
// order: the arithmetic of a source does not depend on the other sources in
// the batch, so results stay bitwise the same alone and in any mix.

// shared-memory A buffer of one warp: 4 row blocks (one per 2 ul + sigma), 32
// rows each (one per staging lane) of 3 16-byte units (forward 8 halves,
// backward 8 halves, padding); a row block spans 98 units.  Rows 3 units apart
// and blocks 98 = 2 (mod 8) units apart keep both the staging stores and the
// ldmatrix row reads free of bank conflicts.
constexpr int kMmaBlockUnits = 98;
constexpr int kMmaABytes = 4 * kMmaBlockUnits * 16;

// Stage one neighbour spinor of this lane's (site, source) for direction
// (MU, B): load the FP16 spinor, project, scale by f2, and store the four A
// rows (upper, lower spin pairs) at byte offset B * 16 of this lane's rows.
template <int MU, int S, int B>
__device__ __forceinline__ void mma_stage(const uint4 *in, int stride, int site, bool live, unsigned f2,
                                          char *arow) {
    using T = ProjTable<MU, S>;
    unsigned w[12];
    if (live) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const uint4 v = __ldg(in + (size_t)k * stride + site);
            w[4 * k] = v.x;
            w[4 * k + 1] = v.y;
            w[4 * k + 2] = v.z;
            w[4 * k + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 12; k++) w[k] = 0u;
    }
    unsigned h[2][3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        h[0][c] = h2_mul(h2_add(w[c], h2_phase<T::ph0>(w[3 * T::pa0 + c])), f2);
        h[1][c] = h2_mul(h2_add(w[3 + c], h2_phase<T::ph1>(w[3 * T::pa1 + c])), f2);
    }
    uint4 *row = reinterpret_cast<uint4 *>(arow + B * 16);
    constexpr int bstride = kMmaBlockUnits;  // in uint4 units
    row[0 * bstride] = make_uint4(h[0][0], h[0][1], h[0][2], 0u);
    row[1 * bstride] = make_uint4(h[1][0], h[1][1], h[1][2], 0u);
    row[2 * bstride] = make_uint4(h2_phase<T::ps0>(h[T::q0][0]), h2_phase<T::ps0>(h[T::q0][1]),
                                  h2_phase<T::ps0>(h[T::q0][2]), 0u);
    row[3 * bstride] = make_uint4(h2_phase<T::ps1>(h[T::q1][0]), h2_phase<T::ps1>(h[T::q1][1]),
                                  h2_phase<T::ps1>(h[T::q1][2]), 0u);
}

// element e (row * 3 + col) of the FP16 18-real link of plane pd at site i, as half2 bits
__device__ __forceinline__ unsigned link_elem(const unsigned *lkx, const unsigned *lkz, int stride, int pd, int e,
                                              int i) {
    if (e == 8) return __ldg(lkz + (size_t)pd * stride + i);
    return __ldg(lkx + ((size_t)(2 * pd + (e >> 2)) * stride + i) * 4 + (e & 3));
}

__device__ __forceinline__ void ldsm_x4(unsigned addr, unsigned (&a)[4]) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                 : "r"(addr));
}

__device__ __forceinline__ void mma_16816(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// per-warp shared state of the tensor-core phases
struct MmaWarpSmem {
    alignas(16) char a[kMmaABytes];
    alignas(16) float2 c[32][12];  // C of each (site, source) pair of a site group
    double n2[32];                 // per-pair dot-product terms
    double acc[kEngMaxRhs];        // per-source sums over the warp's sites
};

// One group of RG sources (positions rg .. rg + nused - 1 of the active list)
// over the warp's 32 sites.
template <int PHASE, int RG>
__device__ __forceinline__ void mma_group(const EngPtrs &P, const EngLattice &La, const int *s_act, int rg,
                                          int nused, int site0, MmaWarpSmem &W) {
    constexpr int SIGN = (PHASE == PH_P1 || PHASE == PH_P2) ? 1 : -1;
    constexpr int OUTPAR = (PHASE == PH_P1 || PHASE == PH_P3) ? 1 : 0;
    constexpr int NRED = (PHASE == PH_P2 || PHASE == PH_P4) ? 1 : 0;
    constexpr int SG = 32 / RG;  // sites per site group
    constexpr int MT = RG / 4;   // m tiles per site
    using L = Low<LOW_F16>;
    const EngTables *T = P.T;
    const int lane = threadIdx.x & 31;
    const Geom g = La.g;
    const int stride = La.stride;
    const unsigned *lkx = reinterpret_cast<const unsigned *>(La.l16x);  // 4 words per site and plane
    const unsigned *lkz = La.l16z;
    // this lane as a staging / epilogue lane: (site s, source r)
    const int s_me = lane / RG, r_me = lane % RG;
    const bool src_live = r_me < nused;
    const int j_me = src_live ? s_act[rg + r_me] : s_act[rg];
    const EngProblem &pr_me = T->prob[j_me];
    const uint4 *in = static_cast<const uint4 *>(
        (PHASE == PH_P1) ? pr_me.p : (PHASE == PH_P3 ? pr_me.Dp : pr_me.t));
    const float *innorm = (PHASE == PH_P1) ? pr_me.pn : (PHASE == PH_P3 ? pr_me.Dpn : pr_me.tn);
    // this lane as an MMA lane: fragment row group gq, thread-in-group tq
    const int gq = lane >> 2, tq = lane & 3;
    const bool b_live = gq < 6 && tq < 3;
    const int bc = gq >> 1, brio = gq & 1;
    // ldmatrix row of this lane inside an m tile: m = (lane & 7) | (lane & 8)
    const int lm = (lane & 7) | (lane & 8);
    const unsigned a_base = (unsigned)__cvta_generic_to_shared(W.a);
    const unsigned a_lane = a_base + (unsigned)((((lm & 3) * kMmaBlockUnits) + (lm >> 2) * 3 + (lane >> 4)) * 16);
    char *const arow = W.a + lane * 48;

    for (int sg = 0; sg < 32; sg += SG) {
        const int i_me = site0 + sg + s_me;
        const bool valid_me = i_me < g.Vh;
        const bool live = valid_me && src_live;
        SiteNbrs nb;
        if (valid_me) nb = site_neighbours(g, i_me, OUTPAR);
        // neighbour norms and the scale of this (site, source)
        float nrm[8];
#pragma unroll
        for (int mu = 0; mu < 4; mu++) {
            nrm[2 * mu] = live ? __ldg(innorm + nb.fwd[mu]) : 0.f;
            nrm[2 * mu + 1] = live ? __ldg(innorm + nb.bwd[mu]) : 0.f;
        }
        float smax = 0.f;
#pragma unroll
        for (int d = 0; d < 8; d++) smax = fmaxf(smax, nrm[d]);
        const float inv = smax > 0.f ? 1.0f / smax : 0.f;
        float cacc[SG][MT][4];
#pragma unroll
        for (int s = 0; s < SG; s++)
#pragma unroll
            for (int i = 0; i < MT; i++)
#pragma unroll
                for (int e = 0; e < 4; e++) cacc[s][i][e] = 0.f;

#pragma unroll
        for (int mu = 0; mu < 4; mu++) {
            float ff = nrm[2 * mu] * inv, fb = nrm[2 * mu + 1] * inv;
            if (mu == 3 && valid_me && nb.tfwd_wrap) ff = -ff;
            if (mu == 3 && valid_me && nb.tbwd_wrap) fb = -fb;
            const int sf = valid_me ? nb.fwd[mu] : 0, sb = valid_me ? nb.bwd[mu] : 0;
            __half2 hf = __float2half2_rn(ff), hb = __float2half2_rn(fb);
            if (mu == 0) {
                mma_stage<0, SIGN, 0>(in, stride, sf, live, *reinterpret_cast<unsigned *>(&hf), arow);
                mma_stage<0, -SIGN, 1>(in, stride, sb, live, *reinterpret_cast<unsigned *>(&hb), arow);
            } else if (mu == 1) {
                mma_stage<1, SIGN, 0>(in, stride, sf, live, *reinterpret_cast<unsigned *>(&hf), arow);
                mma_stage<1, -SIGN, 1>(in, stride, sb, live, *reinterpret_cast<unsigned *>(&hb), arow);
            } else if (mu == 2) {
                mma_stage<2, SIGN, 0>(in, stride, sf, live, *reinterpret_cast<unsigned *>(&hf), arow);
                mma_stage<2, -SIGN, 1>(in, stride, sb, live, *reinterpret_cast<unsigned *>(&hb), arow);
            } else {
                mma_stage<3, SIGN, 0>(in, stride, sf, live, *reinterpret_cast<unsigned *>(&hf), arow);
                mma_stage<3, -SIGN, 1>(in, stride, sb, live, *reinterpret_cast<unsigned *>(&hb), arow);
            }
            __syncwarp();
#pragma unroll
            for (int s = 0; s < SG; s++) {
                const int i_s = site0 + sg + s;
                const int nbb = __shfl_sync(0xffffffffu, sb, s * RG);
                unsigned b0 = 0u, b1 = 0u;
                if (b_live && i_s < g.Vh) {
                    const unsigned uf = link_elem(lkx, lkz, stride, OUTPAR * 4 + mu, bc * 3 + tq, i_s);
                    const unsigned ub = link_elem(lkx, lkz, stride, (1 - OUTPAR) * 4 + mu, tq * 3 + bc, nbb);
                    // forward U[c][c']: (re, -im) | (im, re); backward conj(V[c'][c]): (re, im) | (-im, re)
                    b0 = brio ? h2_swap(uf) : (uf ^ 0x80000000u);
                    b1 = brio ? (h2_swap(ub) ^ 0x00008000u) : ub;
                }
#pragma unroll
                for (int i = 0; i < MT; i++) {
                    unsigned a[4];
                    ldsm_x4(a_lane + (unsigned)((s * RG + 4 * i) * 48), a);
                    mma_16816(cacc[s][i], a, b0, b1);
                }
            }
            __syncwarp();
        }
        // C -> shared memory as (pair, spin * 3 + colour) complex
        if (tq < 3) {
#pragma unroll
            for (int s = 0; s < SG; s++)
#pragma unroll
                for (int i = 0; i < MT; i++) {
                    const int r0 = 4 * i + (gq >> 2), q = gq & 3;
                    W.c[s * RG + r0][q * 3 + tq] = make_float2(cacc[s][i][0], cacc[s][i][1]);
                    W.c[s * RG + r0 + 2][q * 3 + tq] = make_float2(cacc[s][i][2], cacc[s][i][3]);
                }
        }
        __syncwarp();
        // epilogue of (site s_me, source r_me)
        double red[2] = {0.0, 0.0};
        if (live) {
            Spinor<float> acc;
            const float4 *cv = reinterpret_cast<const float4 *>(W.c[lane]);
#pragma unroll
            for (int k = 0; k < 6; k++) {
                const float4 v = cv[k];
                acc.s[(2 * k) / 3][(2 * k) % 3] = {v.x * smax, v.y * smax};
                acc.s[(2 * k + 1) / 3][(2 * k + 1) % 3] = {v.z * smax, v.w * smax};
            }
            epi_low<PHASE, LOW_F16>(pr_me, P.S[j_me], stride, i_me, acc, red);
        }
        if constexpr (NRED > 0) {
            W.n2[lane] = red[0];
            __syncwarp();
            if (lane < nused) {
                double a = W.acc[rg + lane];
#pragma unroll
                for (int s = 0; s < SG; s++) a += W.n2[s * RG + lane];
                W.acc[rg + lane] = a;
            }
        }
        __syncwarp();
    }
}

template <int PHASE, int MINB>
__global__ void __launch_bounds__(kEngTile, MINB) k_eng_mma(EngPtrs P) {
    constexpr int NRED = (PHASE == PH_P2 || PHASE == PH_P4) ? 1 : 0;
    constexpr int NW = kEngTile / 32;
    __shared__ MmaWarpSmem wsm[NW];
    __shared__ double smem[kEngTile / 32];
    __shared__ bool last;
    __shared__ int s_act[kEngMaxRhs];
    __shared__ int s_na;
    const EngTables *T = P.T;
    const int ntiles = T->ntiles;
    const int max_tiles = T->max_tiles;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    MmaWarpSmem &W = wsm[warp];
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int l = find_lattice(T, tile);
        const EngLattice &La = T->lat[l];
        const int lt = tile - La.tile0;
        if (threadIdx.x == 0) {
            int na = 0;
            for (int q = 0; q < La.nprob; q++) {
                const int j = La.prob[q];
                if (active<PHASE>(P.S[j])) s_act[na++] = j;
            }
            s_na = na;
        }
        if (lane < kEngMaxRhs) W.acc[lane] = 0.0;
        __syncthreads();
        const int na = s_na;
        if (lt == 0 && threadIdx.x == 0 && na > 0) {
            count_work(P, PHASE, 0, (unsigned long long)na * La.g.Vh);
            count_work(P, PHASE, 2, La.g.Vh);
        }
        const int site0 = lt * kEngTile + warp * 32;
        for (int rg = 0; rg < na;) {
            const int left = na - rg;
            if (left > 4) {
                mma_group<PHASE, 8>(P, La, s_act, rg, left < 8 ? left : 8, site0, W);
                rg += 8;
            } else {
                mma_group<PHASE, 4>(P, La, s_act, rg, left, site0, W);
                rg += 4;
            }
        }
        __syncthreads();
        if constexpr (NRED > 0) {
            if (threadIdx.x < na) {
                double a = 0.0;
#pragma unroll
                for (int w = 0; w < NW; w++) a += wsm[w].acc[threadIdx.x];
                P.partials[((size_t)s_act[threadIdx.x] * 2) * max_tiles + lt] = a;
                __threadfence();
            }
            __syncthreads();  // every partial written before thread 0 takes the ticket
            arrive_and_finish<PHASE, NRED>(P, La, l, smem, last, La.ntiles);
        } else {
            __syncthreads();  // s_act and the warp buffers are rewritten by the next tile
        }
    }
}
