// Seeded synthetic gauge and spinor fields on the host.
//
// Restates HILA's input generators so that benches and servers can build the
// workloads without any external data:
//   * host RNG: std::mt19937_64 seeded with `seed`, 9000 warm-up draws,
//     uniform doubles in [0,1) (plumbing/random.cpp:60-70)
//   * Box-Muller pair, variance 1 (random.cpp:187-199); a complex Gaussian
//     takes re = r sin(phi), im = r cos(phi) (datatypes/cmplx.h:344-349)
//   * su(3) algebra element from 8 coefficients of width sqrt(2)
//     (datatypes/sun_matrix.h:548-551) expanded to an anti-Hermitian
//     traceless matrix A (sun_matrix.h:480-510)
//   * U = exp(eps A) by the order-20 Horner Taylor series of
//     datatypes/matrix.h:3289-3309, then reunitarize = Gram-Schmidt rows +
//     determinant phase (sun_matrix.h:137-196)
// The coefficients are drawn sequentially (direction-major, then
// lexicographic site) and the matrix work runs in parallel, so the result does
// not depend on the thread count.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/hila_b200.h"

namespace {

using C = std::complex<double>;

struct M3 {
    C a[9];
    C &operator()(int i, int j) { return a[3 * i + j]; }
    C operator()(int i, int j) const { return a[3 * i + j]; }
};

M3 mul(const M3 &x, const M3 &y) {
    M3 z;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) z(i, j) = x(i, 0) * y(0, j) + x(i, 1) * y(1, j) + x(i, 2) * y(2, j);
    return z;
}

class Rng {
  public:
    explicit Rng(uint64_t seed) : gen_(seed) { gen_.discard(9000); }
    double uniform() { return dist_(gen_); }
    // returns r*sin(phi), second = r*cos(phi)
    double gauss_pair(double &second) {
        const double phi = 2.0 * M_PI * uniform();
        double u;
        do {
            u = 1.0 - uniform();
        } while (u == 0.0);
        const double r = std::sqrt(-2.0 * std::log(u));
        second = r * std::cos(phi);
        return r * std::sin(phi);
    }

  private:
    std::mt19937_64 gen_;
    std::uniform_real_distribution<double> dist_{0.0, 1.0};
};

M3 su3_from_coefficients(const double *c, double eps) {
    M3 A;
    for (auto &v : A.a) v = 0.0;
    // diagonal generators diag(i,-i,0)/2 and diag(i,i,-2i)/(2 sqrt 3)
    const double r1 = c[0] * 0.5;
    const double r2 = c[1] * std::sqrt(1.0 / 12.0);
    A(0, 0) = C(0.0, eps * (r1 + r2));
    A(1, 1) = C(0.0, eps * (-r1 + r2));
    A(2, 2) = C(0.0, eps * (-2.0 * r2));
    // off-diagonal pairs (0,1), (0,2), (1,2): A_ij = (c_k + i c_{k+1})/2, A_ji = -conj(A_ij)
    const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int q = 0; q < 3; q++) {
        const C v(eps * 0.5 * c[2 + 2 * q], eps * 0.5 * c[3 + 2 * q]);
        A(pairs[q][0], pairs[q][1]) = v;
        A(pairs[q][1], pairs[q][0]) = -std::conj(v);
    }
    // exp(A) = 1 + A(1 + A/2(1 + A/3(...))) to order 20
    M3 R = A;
    for (int k = 20; k > 1; k--) {
        for (auto &v : R.a) v *= 1.0 / k;
        for (int i = 0; i < 3; i++) R(i, i) += 1.0;
        R = mul(R, A);
    }
    for (int i = 0; i < 3; i++) R(i, i) += 1.0;
    // unitarise rows, then remove the determinant phase
    for (int r = 0; r < 3; r++) {
        double n2 = 0;
        for (int i = 0; i < 3; i++) n2 += std::norm(R(r, i));
        const double inv = 1.0 / std::sqrt(n2);
        for (int i = 0; i < 3; i++) R(r, i) *= inv;
        for (int j = r + 1; j < 3; j++) {
            C d = 0;
            for (int i = 0; i < 3; i++) d += std::conj(R(r, i)) * R(j, i);
            for (int i = 0; i < 3; i++) R(j, i) -= d * R(r, i);
        }
    }
    const C det = R(0, 0) * (R(1, 1) * R(2, 2) - R(1, 2) * R(2, 1)) - R(0, 1) * (R(1, 0) * R(2, 2) - R(1, 2) * R(2, 0)) +
                  R(0, 2) * (R(1, 0) * R(2, 1) - R(1, 1) * R(2, 0));
    const double th = std::arg(det) / 3.0;
    const C ph(std::cos(-th), std::sin(-th));
    for (auto &v : R.a) v *= ph;
    return R;
}

bool valid_dims(const int *dims, long *V) {
    if (!dims) return false;
    long v = 1;
    for (int d = 0; d < 4; d++) {
        if (dims[d] < 2 || dims[d] % 2) return false;
        v *= dims[d];
    }
    *V = v;
    return true;
}

}  // namespace

extern "C" {

int hw_generate_links(const int dims[4], double eps, uint64_t seed, double *links) {
    long V;
    if (!valid_dims(dims, &V) || !links) return HW_ERR_INVALID;
    Rng rng(seed);
    const long nl = 4 * V;
    std::vector<double> coef((size_t)nl * 8);
    const double width = std::sqrt(2.0);
    for (size_t n = 0; n < coef.size(); n += 2) {
        double second;
        coef[n] = rng.gauss_pair(second) * width;
        coef[n + 1] = second * width;
    }
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nl; l++) {
        const M3 U = su3_from_coefficients(&coef[(size_t)l * 8], eps);
        double *o = links + (size_t)l * 18;
        for (int e = 0; e < 9; e++) {
            o[2 * e] = U.a[e].real();
            o[2 * e + 1] = U.a[e].imag();
        }
    }
    return HW_OK;
}

int hw_generate_spinor(const int dims[4], uint64_t seed, int parity_mask, double *spinor) {
    long V;
    if (!valid_dims(dims, &V) || !spinor || parity_mask < 0 || parity_mask > 3) return HW_ERR_INVALID;
    Rng rng(seed);
    for (long i = 0; i < V; i++) {
        long r = i;
        int par = 0;
        for (int d = 0; d < 4; d++) {
            par += (int)(r % dims[d]);
            r /= dims[d];
        }
        double *o = spinor + (size_t)i * 24;
        if (!(parity_mask & ((par & 1) ? 2 : 1))) {
            std::memset(o, 0, 24 * sizeof(double));
            continue;
        }
        for (int c = 0; c < 12; c++) {
            double second;
            o[2 * c] = rng.gauss_pair(second);
            o[2 * c + 1] = second;
        }
    }
    return HW_OK;
}

}  // extern "C"
