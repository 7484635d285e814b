// Device-side site algebra for the Wilson even-odd operator on sm_100a.
//
// Complex arithmetic, SU(3) x colour-vector products, the half-spinor
// projection P_{mu,s} and expansion E_{mu,s} of HILA's
// libraries/datatypes/wilson_vector.h:439-567 (gamma basis :311-347), and the
// even-odd site index arithmetic of libraries/plumbing/lattice.cpp:171-184.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace hw {

// ----------------------------------------------------------------- complex

template <typename R>
struct Cx {
    R re, im;
};

template <typename R>
__device__ __forceinline__ Cx<R> cx(R a, R b) {
    return Cx<R>{a, b};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator+(Cx<R> a, Cx<R> b) {
    return {a.re + b.re, a.im + b.im};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator-(Cx<R> a, Cx<R> b) {
    return {a.re - b.re, a.im - b.im};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator-(Cx<R> a) {
    return {-a.re, -a.im};
}
template <typename R>
__device__ __forceinline__ Cx<R> operator*(R s, Cx<R> a) {
    return {s * a.re, s * a.im};
}
// i * a
template <typename R>
__device__ __forceinline__ Cx<R> mul_i(Cx<R> a) {
    return {-a.im, a.re};
}
// a product rounded on its own (never contracted into a following add)
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
// a * b: the products by a.re rounded, then the a.im terms fused.  The order is fixed
// (and is the one of the packed two-solve hop), so every launch shape rounds alike.
template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {
    return {fma(-a.im, b.im, mul_rn(a.re, b.re)), fma(a.im, b.re, mul_rn(a.re, b.im))};
}
// acc + a * b
template <typename R>
__device__ __forceinline__ Cx<R> cmadd(Cx<R> acc, Cx<R> a, Cx<R> b) {
    acc.re = fma(a.re, b.re, acc.re);
    acc.re = fma(-a.im, b.im, acc.re);
    acc.im = fma(a.re, b.im, acc.im);
    acc.im = fma(a.im, b.re, acc.im);
    return acc;
}
// acc + conj(a) * b
template <typename R>
__device__ __forceinline__ Cx<R> cjmadd(Cx<R> acc, Cx<R> a, Cx<R> b) {
    acc.re = fma(a.re, b.re, acc.re);
    acc.re = fma(a.im, b.im, acc.re);
    acc.im = fma(a.re, b.im, acc.im);
    acc.im = fma(-a.im, b.re, acc.im);
    return acc;
}
template <typename R>
__device__ __forceinline__ Cx<R> conj(Cx<R> a) {
    return {a.re, -a.im};
}
template <typename R>
__device__ __forceinline__ R norm2(Cx<R> a) {
    return a.re * a.re + a.im * a.im;
}

// ----------------------------------------------------------------- SU(3)

// 3x3 complex colour matrix, row-major.  Links may be stored with only their
// first two rows; the third row of a special unitary matrix is
// conj(row0 x row1).
template <typename R>
struct Su3 {
    Cx<R> e[3][3];
};

template <typename R>
__device__ __forceinline__ void reconstruct_row2(Su3<R> &u) {
    // c_k = conj(a_i b_j - a_j b_i), (i,j,k) cyclic
    const Cx<R> *a = u.e[0];
    const Cx<R> *b = u.e[1];
    u.e[2][0] = conj(cmul(a[1], b[2]) - cmul(a[2], b[1]));
    u.e[2][1] = conj(cmul(a[2], b[0]) - cmul(a[0], b[2]));
    u.e[2][2] = conj(cmul(a[0], b[1]) - cmul(a[1], b[0]));
}

// v = U h  (colour vector)
template <typename R>
__device__ __forceinline__ void su3_mul(const Su3<R> &u, const Cx<R> h[3], Cx<R> v[3]) {
#pragma unroll
    for (int i = 0; i < 3; i++) {
        Cx<R> a = cmul(u.e[i][0], h[0]);
        a = cmadd(a, u.e[i][1], h[1]);
        a = cmadd(a, u.e[i][2], h[2]);
        v[i] = a;
    }
}
// v = U^dagger h
template <typename R>
__device__ __forceinline__ void su3_adj_mul(const Su3<R> &u, const Cx<R> h[3], Cx<R> v[3]) {
#pragma unroll
    for (int i = 0; i < 3; i++) {
        Cx<R> a = {fma(u.e[0][i].im, h[0].im, mul_rn(u.e[0][i].re, h[0].re)),
                   fma(-u.e[0][i].im, h[0].re, mul_rn(u.e[0][i].re, h[0].im))};
        a = cjmadd(a, u.e[1][i], h[1]);
        a = cjmadd(a, u.e[2][i], h[2]);
        v[i] = a;
    }
}

// ----------------------------------------------------------------- spinors
//
// A Wilson spinor is 4 spins x 3 colours; component index c = 3*spin + colour.

template <typename R>
struct Spinor {
    Cx<R> s[4][3];
};

// Half spinor h = P_{dir,sign} w, wilson_vector.h:439-491.
template <int DIR, int SIGN, typename R>
__device__ __forceinline__ void project(const Spinor<R> &w, Cx<R> h0[3], Cx<R> h1[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (DIR == 0) {  // x: w0 + s i w3, w1 + s i w2
            if (SIGN > 0) {
                h0[k] = w.s[0][k] + mul_i(w.s[3][k]);
                h1[k] = w.s[1][k] + mul_i(w.s[2][k]);
            } else {
                h0[k] = w.s[0][k] - mul_i(w.s[3][k]);
                h1[k] = w.s[1][k] - mul_i(w.s[2][k]);
            }
        } else if (DIR == 1) {  // y: w0 - s w3, w1 + s w2
            if (SIGN > 0) {
                h0[k] = w.s[0][k] - w.s[3][k];
                h1[k] = w.s[1][k] + w.s[2][k];
            } else {
                h0[k] = w.s[0][k] + w.s[3][k];
                h1[k] = w.s[1][k] - w.s[2][k];
            }
        } else if (DIR == 2) {  // z: w0 + s i w2, w1 - s i w3
            if (SIGN > 0) {
                h0[k] = w.s[0][k] + mul_i(w.s[2][k]);
                h1[k] = w.s[1][k] - mul_i(w.s[3][k]);
            } else {
                h0[k] = w.s[0][k] - mul_i(w.s[2][k]);
                h1[k] = w.s[1][k] + mul_i(w.s[3][k]);
            }
        } else {  // t: w0 + s w2, w1 + s w3
            if (SIGN > 0) {
                h0[k] = w.s[0][k] + w.s[2][k];
                h1[k] = w.s[1][k] + w.s[3][k];
            } else {
                h0[k] = w.s[0][k] - w.s[2][k];
                h1[k] = w.s[1][k] - w.s[3][k];
            }
        }
    }
}

// acc += E_{dir,sign}(h) = (1 + sign gamma_dir) w, wilson_vector.h:493-567.
template <int DIR, int SIGN, typename R>
__device__ __forceinline__ void expand_add(Spinor<R> &acc, const Cx<R> h0[3], const Cx<R> h1[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        acc.s[0][k] = acc.s[0][k] + h0[k];
        acc.s[1][k] = acc.s[1][k] + h1[k];
        if (DIR == 0) {  // r2 = -s i h1, r3 = -s i h0
            if (SIGN > 0) {
                acc.s[2][k] = acc.s[2][k] - mul_i(h1[k]);
                acc.s[3][k] = acc.s[3][k] - mul_i(h0[k]);
            } else {
                acc.s[2][k] = acc.s[2][k] + mul_i(h1[k]);
                acc.s[3][k] = acc.s[3][k] + mul_i(h0[k]);
            }
        } else if (DIR == 1) {  // r2 = s h1, r3 = -s h0
            if (SIGN > 0) {
                acc.s[2][k] = acc.s[2][k] + h1[k];
                acc.s[3][k] = acc.s[3][k] - h0[k];
            } else {
                acc.s[2][k] = acc.s[2][k] - h1[k];
                acc.s[3][k] = acc.s[3][k] + h0[k];
            }
        } else if (DIR == 2) {  // r2 = -s i h0, r3 = s i h1
            if (SIGN > 0) {
                acc.s[2][k] = acc.s[2][k] - mul_i(h0[k]);
                acc.s[3][k] = acc.s[3][k] + mul_i(h1[k]);
            } else {
                acc.s[2][k] = acc.s[2][k] + mul_i(h0[k]);
                acc.s[3][k] = acc.s[3][k] - mul_i(h1[k]);
            }
        } else {  // r2 = s h0, r3 = s h1
            if (SIGN > 0) {
                acc.s[2][k] = acc.s[2][k] + h0[k];
                acc.s[3][k] = acc.s[3][k] + h1[k];
            } else {
                acc.s[2][k] = acc.s[2][k] - h0[k];
                acc.s[3][k] = acc.s[3][k] - h1[k];
            }
        }
    }
}

// The contributions of one projected component to E_{dir,sign}: Q = 0 adds h0
// (spin 0 and the lower spin built from h0), Q = 1 adds h1.  expand_add<DIR,
// SIGN>(acc, h0, h1) equals expand_add_half<DIR, SIGN, 0>(acc, h0) followed by
// expand_add_half<DIR, SIGN, 1>(acc, h1), element by element (each element of
// acc receives one term), so a hop can hold one of h0, h1 at a time.
template <int DIR, int SIGN, int Q, typename R>
__device__ __forceinline__ void expand_add_half(Spinor<R> &acc, const Cx<R> h[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        acc.s[Q][k] = acc.s[Q][k] + h[k];
        if (DIR == 0) {  // r2 = -s i h1, r3 = -s i h0
            Cx<R> &lo = acc.s[Q == 0 ? 3 : 2][k];
            lo = SIGN > 0 ? lo - mul_i(h[k]) : lo + mul_i(h[k]);
        } else if (DIR == 1) {  // r2 = s h1, r3 = -s h0
            if (Q == 0)
                acc.s[3][k] = SIGN > 0 ? acc.s[3][k] - h[k] : acc.s[3][k] + h[k];
            else
                acc.s[2][k] = SIGN > 0 ? acc.s[2][k] + h[k] : acc.s[2][k] - h[k];
        } else if (DIR == 2) {  // r2 = -s i h0, r3 = s i h1
            if (Q == 0)
                acc.s[2][k] = SIGN > 0 ? acc.s[2][k] - mul_i(h[k]) : acc.s[2][k] + mul_i(h[k]);
            else
                acc.s[3][k] = SIGN > 0 ? acc.s[3][k] + mul_i(h[k]) : acc.s[3][k] - mul_i(h[k]);
        } else {  // r2 = s h0, r3 = s h1
            Cx<R> &lo = acc.s[Q == 0 ? 2 : 3][k];
            lo = SIGN > 0 ? lo + h[k] : lo - h[k];
        }
    }
}

// a + s v and a + s (i v), component-wise FMAs
template <typename R>
__device__ __forceinline__ Cx<R> axpy(Cx<R> a, R s, Cx<R> v) {
    return {fma(s, v.re, a.re), fma(s, v.im, a.im)};
}
template <typename R>
__device__ __forceinline__ Cx<R> axpy_i(Cx<R> a, R s, Cx<R> v) {
    return {fma(-s, v.im, a.re), fma(s, v.re, a.im)};
}

// acc += sc * E_{dir,sign}(h): expand_add with a scale folded into the FMAs
// (the per-site norm of FP16 storage and the antiperiodic sign cost nothing).
template <int DIR, int SIGN, typename R>
__device__ __forceinline__ void expand_add_scaled(Spinor<R> &acc, const Cx<R> h0[3], const Cx<R> h1[3], R sc) {
    const R sp = SIGN > 0 ? sc : -sc;  // sign * sc
#pragma unroll
    for (int k = 0; k < 3; k++) {
        acc.s[0][k] = axpy(acc.s[0][k], sc, h0[k]);
        acc.s[1][k] = axpy(acc.s[1][k], sc, h1[k]);
        if (DIR == 0) {  // r2 = -s i h1, r3 = -s i h0
            acc.s[2][k] = axpy_i(acc.s[2][k], -sp, h1[k]);
            acc.s[3][k] = axpy_i(acc.s[3][k], -sp, h0[k]);
        } else if (DIR == 1) {  // r2 = s h1, r3 = -s h0
            acc.s[2][k] = axpy(acc.s[2][k], sp, h1[k]);
            acc.s[3][k] = axpy(acc.s[3][k], -sp, h0[k]);
        } else if (DIR == 2) {  // r2 = -s i h0, r3 = s i h1
            acc.s[2][k] = axpy_i(acc.s[2][k], -sp, h0[k]);
            acc.s[3][k] = axpy_i(acc.s[3][k], sp, h1[k]);
        } else {  // r2 = s h0, r3 = s h1
            acc.s[2][k] = axpy(acc.s[2][k], sp, h0[k]);
            acc.s[3][k] = axpy(acc.s[3][k], sp, h1[k]);
        }
    }
}

// expand_add_scaled for one projected component (Q = 0: h0, Q = 1: h1); the pair
// for Q = 0 and 1 equals expand_add_scaled element by element
template <int DIR, int SIGN, int Q, typename R>
__device__ __forceinline__ void expand_add_scaled_half(Spinor<R> &acc, const Cx<R> h[3], R sc) {
    const R sp = SIGN > 0 ? sc : -sc;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        acc.s[Q][k] = axpy(acc.s[Q][k], sc, h[k]);
        if (DIR == 0) {  // r2 = -s i h1, r3 = -s i h0
            acc.s[Q == 0 ? 3 : 2][k] = axpy_i(acc.s[Q == 0 ? 3 : 2][k], -sp, h[k]);
        } else if (DIR == 1) {  // r2 = s h1, r3 = -s h0
            if (Q == 0)
                acc.s[3][k] = axpy(acc.s[3][k], -sp, h[k]);
            else
                acc.s[2][k] = axpy(acc.s[2][k], sp, h[k]);
        } else if (DIR == 2) {  // r2 = -s i h0, r3 = s i h1
            if (Q == 0)
                acc.s[2][k] = axpy_i(acc.s[2][k], -sp, h[k]);
            else
                acc.s[3][k] = axpy_i(acc.s[3][k], sp, h[k]);
        } else {  // r2 = s h0, r3 = s h1
            acc.s[Q == 0 ? 2 : 3][k] = axpy(acc.s[Q == 0 ? 2 : 3][k], sp, h[k]);
        }
    }
}

// ----------------------------------------------------------------- geometry
//
// Even-odd layout: a site with lexicographic index
// lex = x + Lx*(y + Ly*(z + Lz*t)) and parity (x+y+z+t)&1 lives at
// checkerboard index lex/2 inside the half-lattice array of its parity
// (lattice.cpp:171-184 with even sites first).  Lx must be even.

// Exact unsigned division by a divisor fixed at set-up: q = umulhi64(n, m) with
// m = ceil(2^64 / d) equals floor(n / d) for all n, d < 2^32 (the rounding error
// n * (m d - 2^64) / 2^64 < n d / 2^64 < 1 cannot reach the next multiple).
// m = 0 encodes d = 1.
struct FastDiv {
    unsigned long long m;
    unsigned d;
    __host__ __device__ void init(unsigned div) {
        d = div;
        m = (div <= 1) ? 0ull : (~0ull / div) + 1ull;
    }
    __device__ __forceinline__ unsigned div(unsigned n) const {
        return m ? (unsigned)__umul64hi((unsigned long long)n, m) : n;
    }
};

struct Geom {
    int L[4];       // Lx, Ly, Lz, Lt
    int lxh;        // Lx / 2
    int Vh;         // sites per parity
    int sy, sz, st; // checkerboard strides of y, z, t: lxh, lxh*Ly, lxh*Ly*Lz
    int tap;        // 1: fermion values crossing the t boundary are negated
    int hop_variant;  // launch shape of the FP64 hop kernels (host-side choice, see dslash_f64.cu)
    FastDiv dx, dy, dz;  // division by lxh, Ly, Lz
};

// fill a Geom for dims (all even) and the fermion boundary condition in t
inline void geom_setup(Geom &g, const int dims[4], int tap) {
    for (int d = 0; d < 4; d++) g.L[d] = dims[d];
    g.lxh = dims[0] / 2;
    g.Vh = (int)((long)dims[0] * dims[1] * dims[2] * dims[3] / 2);
    g.sy = g.lxh;
    g.sz = g.lxh * dims[1];
    g.st = g.lxh * dims[1] * dims[2];
    g.tap = tap ? 1 : 0;
    g.hop_variant = 0;
    g.dx.init((unsigned)g.lxh);
    g.dy.init((unsigned)dims[1]);
    g.dz.init((unsigned)dims[2]);
}

struct SiteNbrs {
    int fwd[4], bwd[4];  // checkerboard index of x+mu, x-mu (opposite parity)
    bool tfwd_wrap, tbwd_wrap;
};

// coordinates (x, y, z, t) of checkerboard site i of parity par
__device__ __forceinline__ void site_coords(const Geom &g, int i, int par, int c[4]) {
    const int q1 = (int)g.dx.div((unsigned)i);
    const int xh = i - q1 * g.lxh;
    const int q2 = (int)g.dy.div((unsigned)q1);
    c[1] = q1 - q2 * g.L[1];
    c[3] = (int)g.dz.div((unsigned)q2);
    c[2] = q2 - c[3] * g.L[2];
    c[0] = 2 * xh + ((c[1] + c[2] + c[3] + par) & 1);
}

// neighbours of checkerboard site i of parity par
__device__ __forceinline__ SiteNbrs site_neighbours(const Geom &g, int i, int par) {
    SiteNbrs n;
    const int q1 = (int)g.dx.div((unsigned)i);
    const int xh = i - q1 * g.lxh;
    const int q2 = (int)g.dy.div((unsigned)q1);
    const int y = q1 - q2 * g.L[1];
    const int t = (int)g.dz.div((unsigned)q2);
    const int z = q2 - t * g.L[2];
    const int x = 2 * xh + ((y + z + t + par) & 1);
    int base = i - xh;
    int xp = (x + 1 == g.L[0]) ? 0 : x + 1;
    int xm = (x == 0) ? g.L[0] - 1 : x - 1;
    n.fwd[0] = base + (xp >> 1);
    n.bwd[0] = base + (xm >> 1);
    n.fwd[1] = (y + 1 == g.L[1]) ? i - (g.L[1] - 1) * g.sy : i + g.sy;
    n.bwd[1] = (y == 0) ? i + (g.L[1] - 1) * g.sy : i - g.sy;
    n.fwd[2] = (z + 1 == g.L[2]) ? i - (g.L[2] - 1) * g.sz : i + g.sz;
    n.bwd[2] = (z == 0) ? i + (g.L[2] - 1) * g.sz : i - g.sz;
    n.tfwd_wrap = (t + 1 == g.L[3]);
    n.tbwd_wrap = (t == 0);
    n.fwd[3] = n.tfwd_wrap ? i - (g.L[3] - 1) * g.st : i + g.st;
    n.bwd[3] = n.tbwd_wrap ? i + (g.L[3] - 1) * g.st : i - g.st;
    n.tfwd_wrap = n.tfwd_wrap && g.tap;
    n.tbwd_wrap = n.tbwd_wrap && g.tap;
    return n;
}

}  // namespace hw
