// HBM storage formats for spinor and gauge fields, and their device accessors.
//
// All fields are stored per parity ("half-lattice arrays") in a
// structure-of-arrays layout over checkerboard sites, so that a warp reading
// one component for 32 consecutive sites issues one fully coalesced 512-byte
// (FP64) or 256-byte request:
//
//   FP64 spinor   12 x double2 planes           component c at p[c*stride + i]
//   FP32 spinor    6 x float4 planes            components 2k,2k+1 at p[k*stride + i]
//   FP16 spinor    3 x uint4 planes + float     components 4k..4k+3 (8 halves) at
//                  norm plane                   p[k*stride + i], scaled by norm[i]
//
//   FP64 links, 18 reals: 9 double2 planes per (parity, dir)
//   FP64 links, 12 reals: 6 double2 planes (rows 0,1; row 2 rebuilt)
//   FP32 links, 12 reals: 3 float4 planes
//   FP16 links, 12 reals: 1 uint4 plane (elements 0..3) + 1 uint2 plane (4,5)
//
// Plane index for links: ((parity*4 + dir)*planes + k)*stride + i.
// `stride` is the padded number of sites per parity (a multiple of 64).
#pragma once

#include "wilson_math.cuh"

namespace hw {

enum Prec : int { PREC_F64 = 0, PREC_F32 = 1, PREC_F16 = 2 };

// ------------------------------------------------------------------ spinors

// ------------------------------------------------------------------ FP16 projection
// Half-spinor projection on packed FP16 complex values (re in the low half, im
// in the high half).

__device__ __forceinline__ unsigned h2_swap(unsigned x) { return __byte_perm(x, 0, 0x1032); }

// x * phase, phase code 0: 1, 1: i, 2: -1, 3: -i; (re, im) in the low / high half
template <int PH>
__device__ __forceinline__ unsigned h2_phase(unsigned x) {
    if constexpr (PH == 0)
        return x;
    else if constexpr (PH == 1)
        return h2_swap(x) ^ 0x00008000u;  // i (re, im) = (-im, re)
    else if constexpr (PH == 2)
        return x ^ 0x80008000u;
    else
        return h2_swap(x) ^ 0x80000000u;  // -i (re, im) = (im, -re)
}

__device__ __forceinline__ unsigned h2_add(unsigned a, unsigned b) {
    unsigned r;
    asm("add.rn.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ unsigned h2_mul(unsigned a, unsigned b) {
    unsigned r;
    asm("mul.rn.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}

// Projection P_{mu,s} (h0 = w0 + ph0 w_pa0, h1 = w1 + ph1 w_pa1) and the lower
// spins of E_{mu,s} (spin 2 = ps0 h_q0, spin 3 = ps1 h_q1), wilson_vector.h:439-567.
template <int MU, int S>
struct ProjTable {
    static constexpr int pa0 = (MU == 0 || MU == 1) ? 3 : 2;
    static constexpr int pa1 = (MU == 0 || MU == 1) ? 2 : 3;
    static constexpr int ph0 = MU == 0 ? (S > 0 ? 1 : 3) : MU == 1 ? (S > 0 ? 2 : 0) : MU == 2 ? (S > 0 ? 1 : 3)
                                                                                                : (S > 0 ? 0 : 2);
    static constexpr int ph1 = MU == 0 ? (S > 0 ? 1 : 3) : MU == 1 ? (S > 0 ? 0 : 2) : MU == 2 ? (S > 0 ? 3 : 1)
                                                                                                : (S > 0 ? 0 : 2);
    static constexpr int q0 = (MU == 0 || MU == 1) ? 1 : 0;
    static constexpr int q1 = (MU == 0 || MU == 1) ? 0 : 1;
    static constexpr int ps0 = MU == 0 ? (S > 0 ? 3 : 1) : MU == 1 ? (S > 0 ? 0 : 2) : MU == 2 ? (S > 0 ? 3 : 1)
                                                                                                : (S > 0 ? 0 : 2);
    static constexpr int ps1 = MU == 0 ? (S > 0 ? 3 : 1) : MU == 1 ? (S > 0 ? 2 : 0) : MU == 2 ? (S > 0 ? 1 : 3)
                                                                                                : (S > 0 ? 0 : 2);
};

struct SpinorF64 {
    using R = double;
    double2 *p;
    int stride;
    __device__ __forceinline__ void load(int i, Spinor<double> &w) const {
#pragma unroll
        for (int c = 0; c < 12; c++) {
            double2 v = __ldg(p + (size_t)c * stride + i);
            w.s[c / 3][c % 3] = {v.x, v.y};
        }
    }
    __device__ __forceinline__ void load_cached(int i, Spinor<double> &w) const {
#pragma unroll
        for (int c = 0; c < 12; c++) {
            double2 v = p[(size_t)c * stride + i];
            w.s[c / 3][c % 3] = {v.x, v.y};
        }
    }
    template <int MU, int S>
    __device__ __forceinline__ void load_proj(int i, Cx<double> h0[3], Cx<double> h1[3], double &sc) const {
        Spinor<double> w;
        load_raw(i, w, sc);
        project<MU, S>(w, h0, h1);
    }
    __device__ __forceinline__ void load_raw(int i, Spinor<double> &w, double &sc) const {
        sc = 1.0;
        load(i, w);
    }
    __device__ __forceinline__ void store(int i, const Spinor<double> &w) const {
#pragma unroll
        for (int c = 0; c < 12; c++) p[(size_t)c * stride + i] = make_double2(w.s[c / 3][c % 3].re, w.s[c / 3][c % 3].im);
    }
};

struct SpinorF32 {
    using R = float;
    float4 *p;
    int stride;
    __device__ __forceinline__ void load(int i, Spinor<float> &w) const {
#pragma unroll
        for (int k = 0; k < 6; k++) {
            float4 v = __ldg(p + (size_t)k * stride + i);
            int c0 = 2 * k, c1 = 2 * k + 1;
            w.s[c0 / 3][c0 % 3] = {v.x, v.y};
            w.s[c1 / 3][c1 % 3] = {v.z, v.w};
        }
    }
    __device__ __forceinline__ void load_cached(int i, Spinor<float> &w) const { load(i, w); }
    __device__ __forceinline__ void load_raw(int i, Spinor<float> &w, float &sc) const {
        sc = 1.0f;
        load(i, w);
    }
    template <int MU, int S>
    __device__ __forceinline__ void load_proj(int i, Cx<float> h0[3], Cx<float> h1[3], float &sc) const {
        Spinor<float> w;
        load_raw(i, w, sc);
        project<MU, S>(w, h0, h1);
    }
    __device__ __forceinline__ void store(int i, const Spinor<float> &w) const {
#pragma unroll
        for (int k = 0; k < 6; k++) {
            int c0 = 2 * k, c1 = 2 * k + 1;
            p[(size_t)k * stride + i] = make_float4(w.s[c0 / 3][c0 % 3].re, w.s[c0 / 3][c0 % 3].im,
                                                    w.s[c1 / 3][c1 % 3].re, w.s[c1 / 3][c1 % 3].im);
        }
    }
};

// FP16 storage with a per-site scale: the 24 reals of a site are divided by
// their largest magnitude (stored in norm[i]) before rounding to half, so
// every stored value lies in [-1, 1].
struct SpinorF16 {
    using R = float;
    uint4 *p;
    float *norm;
    int stride;
    static __device__ __forceinline__ void unpack(const uint4 (&v)[3], float nrm, Spinor<float> &w) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const __half2 *h = reinterpret_cast<const __half2 *>(&v[k]);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float2 f = __half22float2(h[q]);
                int c = 4 * k + q;
                w.s[c / 3][c % 3] = {f.x * nrm, f.y * nrm};
            }
        }
    }
    __device__ __forceinline__ void load(int i, Spinor<float> &w) const {
        const uint4 v[3] = {__ldg(p + i), __ldg(p + (size_t)stride + i), __ldg(p + (size_t)2 * stride + i)};
        unpack(v, __ldg(norm + i), w);
    }
    __device__ __forceinline__ void load_cached(int i, Spinor<float> &w) const { load(i, w); }

    // unscaled values; the caller multiplies by *sc (the site norm)
    __device__ __forceinline__ void load_raw(int i, Spinor<float> &w, float &sc) const {
        sc = __ldg(norm + i);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            uint4 v = __ldg(p + (size_t)k * stride + i);
            const __half2 *h = reinterpret_cast<const __half2 *>(&v);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float2 f = __half22float2(h[q]);
                int c = 4 * k + q;
                w.s[c / 3][c % 3] = {f.x, f.y};
            }
        }
    }
    // P_{MU,S} of the unscaled site values in FP32; the caller multiplies by *sc.
    // (Summing in FP16 instead saved 5% of the hop's time but cost the 32^4 solve
    // one more iteration and one more reliable update.)
    template <int MU, int S>
    __device__ __forceinline__ void load_proj(int i, Cx<float> h0[3], Cx<float> h1[3], float &sc) const {
        Spinor<float> w;
        load_raw(i, w, sc);
        project<MU, S>(w, h0, h1);
    }
    __device__ __forceinline__ void store(int i, const Spinor<float> &w) const {
        float m = 0.f;
#pragma unroll
        for (int c = 0; c < 12; c++) m = fmaxf(m, fmaxf(fabsf(w.s[c / 3][c % 3].re), fabsf(w.s[c / 3][c % 3].im)));
        float inv = m > 0.f ? 1.0f / m : 0.f;
        norm[i] = m;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            uint4 v;
            __half2 *h = reinterpret_cast<__half2 *>(&v);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                int c = 4 * k + q;
                h[q] = __floats2half2_rn(w.s[c / 3][c % 3].re * inv, w.s[c / 3][c % 3].im * inv);
            }
            p[(size_t)k * stride + i] = v;
        }
    }
};

// ------------------------------------------------------------------ links

struct LinksF64x18 {
    using R = double;
    static constexpr int planes = 9;
    const double2 *p;
    int stride;
    __device__ __forceinline__ void load(int par, int dir, int i, Su3<double> &u) const {
        const double2 *b = p + (size_t)((par * 4 + dir) * 9) * stride + i;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            double2 v = __ldg(b + (size_t)k * stride);
            u.e[k / 3][k % 3] = {v.x, v.y};
        }
    }
};

struct LinksF64x12 {
    using R = double;
    static constexpr int planes = 6;
    const double2 *p;
    int stride;
    __device__ __forceinline__ void load(int par, int dir, int i, Su3<double> &u) const {
        const double2 *b = p + (size_t)((par * 4 + dir) * 6) * stride + i;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            double2 v = __ldg(b + (size_t)k * stride);
            u.e[k / 3][k % 3] = {v.x, v.y};
        }
        reconstruct_row2(u);
    }
};

struct LinksF32x12 {
    using R = float;
    static constexpr int planes = 3;
    const float4 *p;
    int stride;
    __device__ __forceinline__ void load(int par, int dir, int i, Su3<float> &u) const {
        const float4 *b = p + (size_t)((par * 4 + dir) * 3) * stride + i;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float4 v = __ldg(b + (size_t)k * stride);
            int e0 = 2 * k, e1 = 2 * k + 1;
            u.e[e0 / 3][e0 % 3] = {v.x, v.y};
            u.e[e1 / 3][e1 % 3] = {v.z, v.w};
        }
        reconstruct_row2(u);
    }
};

// FP32, all 18 reals: 4 float4 planes (elements 0..7) + 1 float2 plane (element 8)
// per (parity, dir).  No third-row rebuild: used where the same links serve many
// right-hand sides from cache and instructions, not bytes, bound the kernel.
struct LinksF32x18 {
    using R = float;
    const float4 *a;
    const float2 *b;
    int stride;
    __device__ __forceinline__ void load(int par, int dir, int i, Su3<float> &u) const {
        const float4 *pa = a + (size_t)((par * 4 + dir) * 4) * stride + i;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float4 v = __ldg(pa + (size_t)k * stride);
            int e0 = 2 * k, e1 = 2 * k + 1;
            u.e[e0 / 3][e0 % 3] = {v.x, v.y};
            u.e[e1 / 3][e1 % 3] = {v.z, v.w};
        }
        float2 w = __ldg(b + (size_t)(par * 4 + dir) * stride + i);
        u.e[2][2] = {w.x, w.y};
    }
};

// Link entries of an SU(3) matrix lie in [-1, 1]; FP16 stores them unscaled.
struct LinksF16x12 {
    using R = float;
    const uint4 *p;   // elements 0..3 of rows 0,1 (per (parity, dir) plane)
    const uint2 *q;   // elements 4..5
    int stride;
    __device__ __forceinline__ void load(int par, int dir, int i, Su3<float> &u) const {
        size_t o = (size_t)(par * 4 + dir) * stride + i;
        uint4 a = __ldg(p + o);
        uint2 b = __ldg(q + o);
        const __half2 *ha = reinterpret_cast<const __half2 *>(&a);
        const __half2 *hb = reinterpret_cast<const __half2 *>(&b);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float2 f = __half22float2(ha[k]);
            u.e[k / 3][k % 3] = {f.x, f.y};
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            float2 f = __half22float2(hb[k]);
            u.e[(k + 4) / 3][(k + 4) % 3] = {f.x, f.y};
        }
        reconstruct_row2(u);
    }
};

// All 18 reals in FP16: elements 0..7 in two uint4 planes, element 8 in one
// 32-bit plane per (parity, dir).  No third-row rebuild in the hop.
struct LinksF16x18 {
    using R = float;
    const uint4 *p;      // 2 planes per (parity, dir)
    const unsigned *q;   // 1 plane per (parity, dir)
    int stride;
    static __device__ __forceinline__ void unpack(const uint4 (&a)[2], unsigned b, Su3<float> &u) {
        const __half2 *ha = reinterpret_cast<const __half2 *>(a);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            float2 f = __half22float2(ha[k]);
            u.e[k / 3][k % 3] = {f.x, f.y};
        }
        float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&b));
        u.e[2][2] = {f.x, f.y};
    }
    __device__ __forceinline__ void load(int par, int dir, int i, Su3<float> &u) const {
        const int pd = par * 4 + dir;
        uint4 a[2];
        a[0] = __ldg(p + (size_t)(2 * pd) * stride + i);
        a[1] = __ldg(p + (size_t)(2 * pd + 1) * stride + i);
        unpack(a, __ldg(q + (size_t)pd * stride + i), u);
    }
};

// cp.async (per-thread asynchronous global -> shared copies; a thread that reads
// only what it copied itself needs cp_async_wait_all and no block barrier)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The eight links of the hop at one output site (forward U_mu(x) in slots 0..3,
// backward U_mu(x - mu) in slots 4..7) of 18-real FP16 links, copied once into
// shared memory and read from there by every right-hand side of the site.
// Slot k of thread t: x[(2k + w) * BLOCK + t] (w = 0, 1), z[k * BLOCK + t].
template <int BLOCK>
struct LinksF16x18Smem {
    using R = float;
    uint4 *x;
    unsigned *z;
    int outpar;  // parity of the output site: par == outpar selects the forward slots
    __device__ __forceinline__ void stage(const LinksF16x18 &U, const SiteNbrs &n, int i) const {
        const int t = threadIdx.x;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int dir = k & 3;
            const int pd = (k < 4 ? outpar : 1 - outpar) * 4 + dir;
            const int idx = k < 4 ? i : n.bwd[dir];
            cp_async16(x + (2 * k) * BLOCK + t, U.p + (size_t)(2 * pd) * U.stride + idx);
            cp_async16(x + (2 * k + 1) * BLOCK + t, U.p + (size_t)(2 * pd + 1) * U.stride + idx);
            cp_async4(z + k * BLOCK + t, U.q + (size_t)pd * U.stride + idx);
        }
    }
    __device__ __forceinline__ void load(int par, int dir, int, Su3<float> &u) const {
        const int k = (par == outpar ? 0 : 4) + dir;
        const int t = threadIdx.x;
        const uint4 a[2] = {x[(2 * k) * BLOCK + t], x[(2 * k + 1) * BLOCK + t]};
        LinksF16x18::unpack(a, z[k * BLOCK + t], u);
    }
};

// ------------------------------------------------------------------ hopping term
//
// acc = (H_s in)(x) for checkerboard site i of parity par (the output parity);
// `in` holds the opposite parity.  Forward term uses U_mu(x) (parity par),
// backward term U_mu(x-mu) (opposite parity, at the neighbour's index).

template <int MU, int SIGN, class SpIn, class Lk, typename R>
__device__ __forceinline__ void hop_dir(const SiteNbrs &n, int par, int i, const SpIn &in, const Lk &U,
                                        Spinor<R> &acc) {
    Cx<R> h0[3], h1[3], v0[3], v1[3];
    Su3<R> u;
    {
        Spinor<R> w;
        in.load(n.fwd[MU], w);
        project<MU, SIGN>(w, h0, h1);
        if (MU == 3) {
            const R sg = n.tfwd_wrap ? R(-1) : R(1);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                h0[k] = sg * h0[k];
                h1[k] = sg * h1[k];
            }
        }
        U.load(par, MU, i, u);
        su3_mul(u, h0, v0);
        su3_mul(u, h1, v1);
        expand_add<MU, SIGN>(acc, v0, v1);
    }
    {
        Spinor<R> w;
        in.load(n.bwd[MU], w);
        project<MU, -SIGN>(w, h0, h1);
        if (MU == 3) {
            const R sg = n.tbwd_wrap ? R(-1) : R(1);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                h0[k] = sg * h0[k];
                h1[k] = sg * h1[k];
            }
        }
        U.load(1 - par, MU, n.bwd[MU], u);
        su3_adj_mul(u, h0, v0);
        su3_adj_mul(u, h1, v1);
        expand_add<MU, -SIGN>(acc, v0, v1);
    }
}

// Hopping term for NR right-hand sides that share the links: every link is
// loaded (and its third row rebuilt) once for all of them.  in[r] is read at
// the neighbour sites; cnt <= NR of them are live.
template <int MU, int SIGN, int NR, class SpIn, class Lk, typename R>
__device__ __forceinline__ void hop_dir_multi(const SiteNbrs &n, int par, int i, const SpIn (&in)[NR], int cnt,
                                              const Lk &U, Spinor<R> (&acc)[NR]) {
    Cx<R> h0[3], h1[3], v0[3], v1[3];
    Su3<R> u;
    // one colour-multiplied half spinor live at a time (expand_add_scaled_half)
    U.load(par, MU, i, u);
#pragma unroll
    for (int r = 0; r < NR; r++) {
        if (r < cnt) {
            R sc;
            in[r].template load_proj<MU, SIGN>(n.fwd[MU], h0, h1, sc);
            if (MU == 3 && n.tfwd_wrap) sc = -sc;
            su3_mul(u, h0, v0);
            expand_add_scaled_half<MU, SIGN, 0>(acc[r], v0, sc);
            su3_mul(u, h1, v1);
            expand_add_scaled_half<MU, SIGN, 1>(acc[r], v1, sc);
        }
    }
    U.load(1 - par, MU, n.bwd[MU], u);
#pragma unroll
    for (int r = 0; r < NR; r++) {
        if (r < cnt) {
            R sc;
            in[r].template load_proj<MU, -SIGN>(n.bwd[MU], h0, h1, sc);
            if (MU == 3 && n.tbwd_wrap) sc = -sc;
            su3_adj_mul(u, h0, v0);
            expand_add_scaled_half<MU, -SIGN, 0>(acc[r], v0, sc);
            su3_adj_mul(u, h1, v1);
            expand_add_scaled_half<MU, -SIGN, 1>(acc[r], v1, sc);
        }
    }
}

// hop_dir with one colour-multiplied half spinor live at a time (expand_add_half):
// the same arithmetic in the same order, fewer registers
template <int MU, int SIGN, class SpIn, class Lk, typename R>
__device__ __forceinline__ void hop_dir_lean(const SiteNbrs &n, int par, int i, const SpIn &in, const Lk &U,
                                             Spinor<R> &acc) {
#pragma unroll
    for (int b = 0; b < 2; b++) {
        Cx<R> h0[3], h1[3], v[3];
        {
            Spinor<R> w;
            in.load(b == 0 ? n.fwd[MU] : n.bwd[MU], w);
            if (b == 0)
                project<MU, SIGN>(w, h0, h1);
            else
                project<MU, -SIGN>(w, h0, h1);
            if (MU == 3) {
                const R sg = (b == 0 ? n.tfwd_wrap : n.tbwd_wrap) ? R(-1) : R(1);
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    h0[k] = sg * h0[k];
                    h1[k] = sg * h1[k];
                }
            }
        }
        Su3<R> u;
        if (b == 0) {
            U.load(par, MU, i, u);
            su3_mul(u, h0, v);
            expand_add_half<MU, SIGN, 0>(acc, v);
            su3_mul(u, h1, v);
            expand_add_half<MU, SIGN, 1>(acc, v);
        } else {
            U.load(1 - par, MU, n.bwd[MU], u);
            su3_adj_mul(u, h0, v);
            expand_add_half<MU, -SIGN, 0>(acc, v);
            su3_adj_mul(u, h1, v);
            expand_add_half<MU, -SIGN, 1>(acc, v);
        }
    }
}

template <int SIGN, class SpIn, class Lk, typename R>
__device__ __forceinline__ void hop_site(const Geom &g, int par, int i, const SpIn &in, const Lk &U,
                                         Spinor<R> &acc) {
#pragma unroll
    for (int c = 0; c < 12; c++) acc.s[c / 3][c % 3] = {R(0), R(0)};
    SiteNbrs n = site_neighbours(g, i, par);
    hop_dir_lean<0, SIGN>(n, par, i, in, U, acc);
    hop_dir_lean<1, SIGN>(n, par, i, in, U, acc);
    hop_dir_lean<2, SIGN>(n, par, i, in, U, acc);
    hop_dir_lean<3, SIGN>(n, par, i, in, U, acc);
}

}  // namespace hw
