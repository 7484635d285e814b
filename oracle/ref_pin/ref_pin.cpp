// Pin library: the reference's own site algebra and input generators, compiled with g++.
//
// Test infrastructure only (golden vectors for tests/golden/); nothing in the product
// links it.  It builds only where the reference sources are present: the Makefile next
// to this file cuts the code it needs out of the reference, verbatim (extract.py lists
// the ranges and why they cannot be included whole), and compiles it here together with
// the reference headers that still compile as they are, in the reference's own HILAPP
// configuration (plumbing/defs.h with HILAPP defined needs no MPI, CUDA or FFTW):
//   datatypes/cmplx.h, datatypes/matrix.h  Complex, Vector, SU(3) products, exp()
//                                          (matrix.h:3289-3309)
//   datatypes/sun_matrix.h                 Algebra::gaussian_random / expand_scaled
//                                          (:480-560), reunitarize (:137-196)
//   wilson_vector.h (cut)                  gamma matrices (:307-371), HalfWilsonVector
//                                          projection and expand() (:425-739)
//   random.cpp (cut)                       mt19937_64 + 9000 warm-up draws, Box-Muller
// This file adds only what is not reference arithmetic: a plain container for the four
// spin components of a Wilson vector (the class at wilson_vector.h:56-245 no longer
// compiles), conversions from and to the canonical host layouts, the site loops and the
// antiperiodic sign of values gathered across the time boundary.  The hop follows
// wilson.h:15-95 with its intended backward term (gather of the U^dagger-multiplied
// projection from x - mu; wilson.h:47 gathers it from x + mu) and the even-odd operator
// wilson.h:272-289.
//
// Host layouts: spinor double[V][4][3][2], links double[4][V][3][3][2], lexicographic
// site index x + Lx (y + Ly (z + Lz t)) (lattice.cpp:559-565).
#include "plumbing/defs.h"
#include "datatypes/cmplx.h"
#include "datatypes/matrix.h"
#include "datatypes/sun_matrix.h"
#include "plumbing/coordinates.h"

#include <cstdint>
#include <cstring>
#include <random>

namespace hila {
// random.cpp:47-55 shuffles the seed by MPI rank; on one rank it is left as given
uint64_t shuffle_rng_seed(uint64_t seed) { return seed; }
}  // namespace hila

#include "random_parts.inc"

// the four spin components of a Wilson vector, each a colour vector
template <int N, typename T>
struct WilsonVector {
    Vector<N, Complex<T>> c[4];
};

#include "wilson_vector_parts.inc"

namespace {

using WV = WilsonVector<3, double>;
using HWV = HalfWilsonVector<3, double>;
using SU3 = SU<3, double>;

WV load_wv(const double *p) {
    WV w;
    for (int s = 0; s < 4; s++)
        for (int c = 0; c < 3; c++) w.c[s].e(c) = Complex<double>(p[2 * (3 * s + c)], p[2 * (3 * s + c) + 1]);
    return w;
}
void store_wv(const WV &w, double *p) {
    for (int s = 0; s < 4; s++)
        for (int c = 0; c < 3; c++) {
            p[2 * (3 * s + c)] = w.c[s].e(c).re;
            p[2 * (3 * s + c) + 1] = w.c[s].e(c).im;
        }
}
SU3 load_su3(const double *p) {
    SU3 u;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) u.e(i, j) = Complex<double>(p[2 * (3 * i + j)], p[2 * (3 * i + j) + 1]);
    return u;
}
void store_su3(const SU3 &u, double *p) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            p[2 * (3 * i + j)] = u.e(i, j).re;
            p[2 * (3 * i + j) + 1] = u.e(i, j).im;
        }
}

struct Lat {
    int L[4];
    long V;
    explicit Lat(const int *d) {
        V = 1;
        for (int k = 0; k < 4; k++) {
            L[k] = d[k];
            V *= d[k];
        }
    }
    void coords(long i, int x[4]) const {
        for (int k = 0; k < 4; k++) {
            x[k] = (int)(i % L[k]);
            i /= L[k];
        }
    }
    long index(const int x[4]) const { return x[0] + (long)L[0] * (x[1] + (long)L[1] * (x[2] + (long)L[2] * x[3])); }
    int parity(long i) const {
        int x[4];
        coords(i, x);
        return (x[0] + x[1] + x[2] + x[3]) & 1;
    }
    // neighbour of site i in direction mu, step +1 / -1; *wrapped_t: the step crossed the time boundary
    long step(long i, int mu, int s, bool *wrapped_t) const {
        int x[4];
        coords(i, x);
        int v = x[mu] + s;
        *wrapped_t = false;
        if (v < 0 || v >= L[mu]) {
            v = (v + L[mu]) % L[mu];
            *wrapped_t = mu == 3;
        }
        x[mu] = v;
        return index(x);
    }
};

const Direction kDir[4] = {e_x, e_y, e_z, e_t};

HWV negated(const HWV &h) { return -h; }

// U h on each colour vector of a half Wilson vector (the product in wilson.h:30,46)
HWV mul(const SU3 &u, const HWV &h) {
    HWV r;
    for (int k = 0; k < Gammadim / 2; k++) r.c[k] = u * h.c[k];
    return r;
}

// v_out[X] (on parity par) = (set ? 0 : v_out[X]) - kappa sum_mu [ (U_mu(X) P_{mu,s} v_in(X+mu)).expand(mu, s)
//                                                + (U_mu(X-mu)^dag P_{mu,-s} v_in(X-mu)).expand(mu, -s) ]
void hop(const Lat &lat, bool antiperiodic, const double *U, double kappa, const double *in, double *out, int par,
         int sign, bool set) {
    for (long i = 0; i < lat.V; i++) {
        if (lat.parity(i) != par) continue;
        WV acc = set ? WV{} : load_wv(out + 24 * i);
        if (set)
            for (int s = 0; s < 4; s++) acc.c[s] = 0;
        for (int m = 0; m < 4; m++) {
            const Direction dir = kDir[m];
            bool wf, wb;
            const long jf = lat.step(i, m, +1, &wf), jb = lat.step(i, m, -1, &wb);
            // vtemp[dir][X + dir]: the projection at the forward neighbour (wilson.h:33-36)
            HWV hf(load_wv(in + 24 * jf), dir, sign);
            if (wf && antiperiodic) hf = negated(hf);
            // vtemp[-dir][X - dir]: U^dag times the projection at the backward neighbour (wilson.h:29-32)
            HWV hb = mul(load_su3(U + 18 * (m * lat.V + jb)).adjoint(), HWV(load_wv(in + 24 * jb), dir, -sign));
            if (wb && antiperiodic) hb = negated(hb);
            const SU3 kU = kappa * load_su3(U + 18 * (m * lat.V + i));
            const WV ef = mul(kU, hf).expand(dir, sign);
            const WV eb = (kappa * hb).expand(dir, -sign);
            for (int s = 0; s < 4; s++) acc.c[s] = acc.c[s] - ef.c[s] - eb.c[s];
        }
        store_wv(acc, out + 24 * i);
    }
}

}  // namespace

extern "C" {

// n Gaussian numbers of hila::gaussrand() after initialize_host_rng(seed); n even, so the
// pair cache of gaussrand() is empty again afterwards
int rp_gaussrand(uint64_t seed, int n, double *out) {
    if (n < 0 || n % 2) return -1;
    hila::initialize_host_rng(seed);
    for (int k = 0; k < n; k++) out[k] = hila::gaussrand();
    return 0;
}

// links U = reunitarize(exp(eps A)), A from Algebra<SU<3>>::gaussian_random() (width sqrt 2)
// and expand_scaled(eps); drawn direction-major, then lexicographic site
int rp_gen_links(const int dims[4], double eps, uint64_t seed, double *U) {
    const Lat lat(dims);
    hila::initialize_host_rng(seed);
    for (int m = 0; m < 4; m++)
        for (long i = 0; i < lat.V; i++) {
            Algebra<SU3> a;
            a.gaussian_random();
            SU3 u = exp(a.expand_scaled(eps));
            u.reunitarize();
            store_su3(u, U + 18 * (m * lat.V + i));
        }
    return 0;
}

// Gaussian spinor: every complex entry from Complex::gaussian_random() on the sites whose
// parity is in parity_mask (1 EVEN, 2 ODD, 3 ALL), zero elsewhere; sites in lexicographic order
int rp_gen_spinor(const int dims[4], uint64_t seed, int parity_mask, double *out) {
    const Lat lat(dims);
    hila::initialize_host_rng(seed);
    for (long i = 0; i < lat.V; i++) {
        WV w;
        for (int s = 0; s < 4; s++) w.c[s] = 0;
        if (parity_mask & (lat.parity(i) ? 2 : 1))
            for (int s = 0; s < 4; s++)
                for (int c = 0; c < 3; c++) w.c[s].e(c).gaussian_random();
        store_wv(w, out + 24 * i);
    }
    return 0;
}

// HalfWilsonVector(w, dir, sign): h = 2 spin components x 3 colours (complex)
int rp_project(const double *w, int dir, int sign, double *h) {
    const HWV r(load_wv(w), kDir[dir], sign);
    for (int k = 0; k < 2; k++)
        for (int c = 0; c < 3; c++) {
            h[2 * (3 * k + c)] = r.c[k].e(c).re;
            h[2 * (3 * k + c) + 1] = r.c[k].e(c).im;
        }
    return 0;
}

// HalfWilsonVector::expand(dir, sign)
int rp_expand(const double *h, int dir, int sign, double *w) {
    HWV r;
    for (int k = 0; k < 2; k++)
        for (int c = 0; c < 3; c++) r.c[k].e(c) = Complex<double>(h[2 * (3 * k + c)], h[2 * (3 * k + c) + 1]);
    store_wv(r.expand(kDir[dir], sign), w);
    return 0;
}

// gamma_g * w for g = 0, 1, 2, 3, 5
int rp_gamma(int g, const double *w, double *out) {
    GammaMatrix gm;
    switch (g) {
    case 0: gm = gamma0; break;
    case 1: gm = gamma1; break;
    case 2: gm = gamma2; break;
    case 3: gm = gamma3; break;
    case 5: gm = gamma5; break;
    default: return -1;
    }
    store_wv(gm * load_wv(w), out);
    return 0;
}

// Dirac_Wilson_hop(_set) on the sites of parity par (0 EVEN, 1 ODD)
int rp_hop(const int dims[4], int antiperiodic, const double *U, double kappa, const double *in, double *out,
           int par, int sign, int set) {
    hop(Lat(dims), antiperiodic != 0, U, kappa, in, out, par, sign, set != 0);
    return 0;
}

// Dirac_Wilson_evenodd::apply (sign 1) / dagger (sign -1), wilson.h:272-289:
// out_e = in_e - kappa^2 H^{eo} H^{oe} in_e (diag = identity), out_o = 0
int rp_eo_apply(const int dims[4], int antiperiodic, const double *U, double kappa, const double *in, double *out,
                int sign) {
    const Lat lat(dims);
    for (long i = 0; i < lat.V; i++)
        if (lat.parity(i) == 0) std::memcpy(out + 24 * i, in + 24 * i, 24 * sizeof(double));
    hop(lat, antiperiodic != 0, U, kappa, in, out, 1, sign, true);
    hop(lat, antiperiodic != 0, U, -kappa, out, out, 0, sign, false);
    for (long i = 0; i < lat.V; i++)
        if (lat.parity(i) == 1) std::memset(out + 24 * i, 0, 24 * sizeof(double));
    return 0;
}

}  // extern "C"
