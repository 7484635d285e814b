// Hopping term for two right-hand sides at once in packed FP32 (sm_100a FFMA2,
// FADD2, FMUL2: one instruction does the same operation on the two lanes of a
// float2).  Lane x carries one solve and lane y another; every lane rounds as
// the scalar fmaf / __fadd_rn / __fmul_rn of its own values, so a solve's result
// does not depend on which solve shares the thread with it.
//
// The algebra is that of hop_dir_multi (storage.cuh): P_{mu,s} of the FP16
// neighbour values in FP32, the link (or its adjoint) times both half spinors,
// and E_{mu,s} scaled by the site norm into the accumulator.  A complex number of
// the pair is stored as two float2 (real parts, imaginary parts), so no lane ever
// has to be swapped: multiplication by i only exchanges which float2 is used.
#pragma once

#include <cuda_fp16.h>

#include "storage.cuh"

namespace hw {

struct Cx2 {
    float2 re, im;  // (solve A, solve B)
};

struct Spinor2 {
    Cx2 s[4][3];
};

__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
// a - b: the product b * (-1) is exact, so the single rounding is that of a - b
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// a + i b and a - i b
__device__ __forceinline__ Cx2 add_i2(Cx2 a, Cx2 b) { return {sub2(a.re, b.im), add2(a.im, b.re)}; }
__device__ __forceinline__ Cx2 sub_i2(Cx2 a, Cx2 b) { return {add2(a.re, b.im), sub2(a.im, b.re)}; }
__device__ __forceinline__ Cx2 add_c2(Cx2 a, Cx2 b) { return {add2(a.re, b.re), add2(a.im, b.im)}; }
__device__ __forceinline__ Cx2 sub_c2(Cx2 a, Cx2 b) { return {sub2(a.re, b.re), sub2(a.im, b.im)}; }

// acc + s v and acc + s (i v) with s a pair of scales
__device__ __forceinline__ Cx2 axpy2(Cx2 a, float2 s, Cx2 v) { return {fma2(s, v.re, a.re), fma2(s, v.im, a.im)}; }
// ns = -s
__device__ __forceinline__ Cx2 axpy_i2(Cx2 a, float2 s, float2 ns, Cx2 v) {
    return {fma2(ns, v.im, a.re), fma2(s, v.re, a.im)};
}

// One site of an FP16 spinor as stored: 12 (re, im) half pairs and the site norm.
struct RawF16 {
    __half2 h[12];
    float sc;
};

__device__ __forceinline__ void load_raw16(const SpinorF16 &s, int i, RawF16 &w) {
    w.sc = __ldg(s.norm + i);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const uint4 v = __ldg(s.p + (size_t)k * s.stride + i);
        w.h[4 * k + 0] = *reinterpret_cast<const __half2 *>(&v.x);
        w.h[4 * k + 1] = *reinterpret_cast<const __half2 *>(&v.y);
        w.h[4 * k + 2] = *reinterpret_cast<const __half2 *>(&v.z);
        w.h[4 * k + 3] = *reinterpret_cast<const __half2 *>(&v.w);
    }
}

// component c = 3*spin + colour of solves A and B, unscaled, in FP32
__device__ __forceinline__ Cx2 comp2(const RawF16 &a, const RawF16 &b, int c) {
    const float2 fa = __half22float2(a.h[c]), fb = __half22float2(b.h[c]);
    return {make_float2(fa.x, fb.x), make_float2(fa.y, fb.y)};
}

// colour k of h = P_{dir,sign} w for both solves (project(), wilson_math.cuh)
template <int DIR, int SIGN>
__device__ __forceinline__ void project2(const RawF16 &a, const RawF16 &b, int k, Cx2 &h0, Cx2 &h1) {
    const Cx2 w0 = comp2(a, b, k), w1 = comp2(a, b, 3 + k), w2 = comp2(a, b, 6 + k), w3 = comp2(a, b, 9 + k);
    if (DIR == 0) {  // w0 + s i w3, w1 + s i w2
        h0 = SIGN > 0 ? add_i2(w0, w3) : sub_i2(w0, w3);
        h1 = SIGN > 0 ? add_i2(w1, w2) : sub_i2(w1, w2);
    } else if (DIR == 1) {  // w0 - s w3, w1 + s w2
        h0 = SIGN > 0 ? sub_c2(w0, w3) : add_c2(w0, w3);
        h1 = SIGN > 0 ? add_c2(w1, w2) : sub_c2(w1, w2);
    } else if (DIR == 2) {  // w0 + s i w2, w1 - s i w3
        h0 = SIGN > 0 ? add_i2(w0, w2) : sub_i2(w0, w2);
        h1 = SIGN > 0 ? sub_i2(w1, w3) : add_i2(w1, w3);
    } else {  // w0 + s w2, w1 + s w3
        h0 = SIGN > 0 ? add_c2(w0, w2) : sub_c2(w0, w2);
        h1 = SIGN > 0 ? add_c2(w1, w3) : sub_c2(w1, w3);
    }
}

// acc += sc E_{dir,sign}(v0, v1) for colour k (expand_add_scaled, wilson_math.cuh);
// sp = sign * sc, nsp = -sp
template <int DIR, int SIGN>
__device__ __forceinline__ void expand2(Spinor2 &acc, int k, const Cx2 &v0, const Cx2 &v1, float2 sc, float2 sp,
                                        float2 nsp) {
    acc.s[0][k] = axpy2(acc.s[0][k], sc, v0);
    acc.s[1][k] = axpy2(acc.s[1][k], sc, v1);
    if (DIR == 0) {  // r2 = -s i h1, r3 = -s i h0
        acc.s[2][k] = axpy_i2(acc.s[2][k], nsp, sp, v1);
        acc.s[3][k] = axpy_i2(acc.s[3][k], nsp, sp, v0);
    } else if (DIR == 1) {  // r2 = s h1, r3 = -s h0
        acc.s[2][k] = axpy2(acc.s[2][k], sp, v1);
        acc.s[3][k] = axpy2(acc.s[3][k], nsp, v0);
    } else if (DIR == 2) {  // r2 = -s i h0, r3 = s i h1
        acc.s[2][k] = axpy_i2(acc.s[2][k], nsp, sp, v0);
        acc.s[3][k] = axpy_i2(acc.s[3][k], sp, nsp, v1);
    } else {  // r2 = s h0, r3 = s h1
        acc.s[2][k] = axpy2(acc.s[2][k], sp, v0);
        acc.s[3][k] = axpy2(acc.s[3][k], sp, v1);
    }
}

// One term of the hop: neighbour site j of both solves, link u (ADJ: its adjoint),
// flip = antiperiodic sign.  Each link element is widened to a pair once and used
// for both half spinors; a colour row of U h is expanded as soon as it is done.
template <int MU, int S, bool ADJ>
__device__ __forceinline__ void hop_term2(const Su3<float> &u, const RawF16 &a, const RawF16 &b, bool flip,
                                          Spinor2 &acc) {
    Cx2 h0[3], h1[3];
#pragma unroll
    for (int k = 0; k < 3; k++) project2<MU, S>(a, b, k, h0[k], h1[k]);
    // the product's minus sign sits on the half spinor: -im (U h) or -re (U^dag h)
    float2 n0[3], n1[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        n0[k] = neg2(ADJ ? h0[k].re : h0[k].im);
        n1[k] = neg2(ADJ ? h1[k].re : h1[k].im);
    }
    const float2 sc = flip ? make_float2(-a.sc, -b.sc) : make_float2(a.sc, b.sc);
    const float2 sp = S > 0 ? sc : neg2(sc);
    const float2 nsp = neg2(sp);
#pragma unroll
    for (int r = 0; r < 3; r++) {
        Cx2 v0, v1;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const Cx<float> e = ADJ ? u.e[c][r] : u.e[r][c];
            const float2 er = bc2(e.re), ei = bc2(e.im);
            if (!ADJ) {  // v += e h
                v0.re = c == 0 ? mul2(er, h0[c].re) : fma2(er, h0[c].re, v0.re);
                v0.im = c == 0 ? mul2(er, h0[c].im) : fma2(er, h0[c].im, v0.im);
                v1.re = c == 0 ? mul2(er, h1[c].re) : fma2(er, h1[c].re, v1.re);
                v1.im = c == 0 ? mul2(er, h1[c].im) : fma2(er, h1[c].im, v1.im);
                v0.re = fma2(ei, n0[c], v0.re);
                v0.im = fma2(ei, h0[c].re, v0.im);
                v1.re = fma2(ei, n1[c], v1.re);
                v1.im = fma2(ei, h1[c].re, v1.im);
            } else {  // v += conj(e) h
                v0.re = c == 0 ? mul2(er, h0[c].re) : fma2(er, h0[c].re, v0.re);
                v0.im = c == 0 ? mul2(er, h0[c].im) : fma2(er, h0[c].im, v0.im);
                v1.re = c == 0 ? mul2(er, h1[c].re) : fma2(er, h1[c].re, v1.re);
                v1.im = c == 0 ? mul2(er, h1[c].im) : fma2(er, h1[c].im, v1.im);
                v0.re = fma2(ei, h0[c].im, v0.re);
                v0.im = fma2(ei, n0[c], v0.im);
                v1.re = fma2(ei, h1[c].im, v1.re);
                v1.im = fma2(ei, n1[c], v1.im);
            }
        }
        expand2<MU, S>(acc, r, v0, v1, sc, sp, nsp);
    }
}

// Both terms of direction MU for solves A (ia) and B (ib) at checkerboard site i
// of parity par (hop_dir_multi with two right-hand sides).
template <int MU, int SIGN, class Lk>
__device__ __forceinline__ void hop_dir_pair(const SiteNbrs &n, int par, int i, const SpinorF16 &ia,
                                             const SpinorF16 &ib, const Lk &U, Spinor2 &acc) {
    {
        RawF16 a, b;
        load_raw16(ia, n.fwd[MU], a);
        load_raw16(ib, n.fwd[MU], b);
        Su3<float> u;
        U.load(par, MU, i, u);
        hop_term2<MU, SIGN, false>(u, a, b, MU == 3 && n.tfwd_wrap, acc);
    }
    {
        RawF16 a, b;
        load_raw16(ia, n.bwd[MU], a);
        load_raw16(ib, n.bwd[MU], b);
        Su3<float> u;
        U.load(1 - par, MU, n.bwd[MU], u);
        hop_term2<MU, -SIGN, true>(u, a, b, MU == 3 && n.tbwd_wrap, acc);
    }
}

}  // namespace hw
