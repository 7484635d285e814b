// The Dirac_Wilson_evenodd block of the reference's test
// (applications/test_cases/test_CG.cpp:215-288) written against the C++ facade,
// on random SU(3) links instead of unit links.  Exit code 0 = all asserts hold.
#include <cmath>
#include <cstdio>
#include <random>

#include "hila_b200/wilson.hpp"

using namespace hila_b200;

static std::complex<double> dot_even(Lattice &L, Field<WilsonVector> &a, Field<WilsonVector> &b) {
    std::complex<double> s = 0;
    const auto &d = L.size();
    for (int t = 0; t < d[3]; t++)
        for (int z = 0; z < d[2]; z++)
            for (int y = 0; y < d[1]; y++)
                for (int x = 0; x < d[0]; x++) {
                    if ((x + y + z + t) & 1) continue;
                    int64_t i = L.index(x, y, z, t);
                    const WilsonVector &u = a.at(i), &v = b.at(i);
                    for (int sp = 0; sp < 4; sp++)
                        for (int c = 0; c < 3; c++) s += std::conj(u.c[sp][c]) * v.c[sp][c];
                }
    return s;
}

static void gaussian_even(Lattice &L, Field<WilsonVector> &f, std::mt19937_64 &rng) {
    std::normal_distribution<double> n(0.0, 1.0);
    const auto &d = L.size();
    for (int64_t i = 0; i < L.volume(); i++) {
        int64_t r = i;
        int par = 0;
        for (int k = 0; k < 4; k++) {
            par += (int)(r % d[k]);
            r /= d[k];
        }
        WilsonVector &w = f[i];
        for (int sp = 0; sp < 4; sp++)
            for (int c = 0; c < 3; c++) w.c[sp][c] = (par & 1) ? 0.0 : std::complex<double>(n(rng), n(rng));
    }
}

#define CHECK(cond, msg)                                      \
    do {                                                      \
        if (!(cond)) {                                        \
            std::fprintf(stderr, "FAILED: %s\n", msg);        \
            return 1;                                         \
        }                                                     \
    } while (0)

int main() {
    Lattice L({16, 8, 8, 8});
    GaugeField U(L);
    U.random(0.3, 2);
    using dirac = Dirac_Wilson_evenodd<SU<3, double>>;
    dirac D(0.12, U);
    Field<WilsonVector> a(L), b(L), Db(L), Ddaggera(L), DdaggerDb(L);
    std::mt19937_64 rng(2);
    gaussian_even(L, a, rng);
    gaussian_even(L, b, rng);

    D.apply(b, Db);
    D.dagger(a, Ddaggera);
    std::complex<double> diff = dot_even(L, a, Db) - dot_even(L, Ddaggera, b);
    CHECK(diff.real() * diff.real() < 1e-16 && diff.imag() * diff.imag() < 1e-16, "test Dirac_Wilson_evenodd");

    // D (DdgD)^-1 Ddg = 1
    CG<dirac> inverse(D);
    b.zero();
    gaussian_even(L, a, rng);
    D.dagger(a, Ddaggera);
    inverse.apply(Ddaggera, b);
    D.apply(b, Db);
    double d2 = 0;
    for (int64_t i = 0; i < L.volume(); i++)
        for (int sp = 0; sp < 4; sp++)
            for (int c = 0; c < 3; c++) d2 += std::norm(a.at(i).c[sp][c] - Db.at(i).c[sp][c]);
    std::printf("D inv Dg %g (iterations %d)\n", d2, inverse.last_iterations());
    CHECK(d2 * d2 < 1e-16, "test D (DdgD)^-1 Ddg");

    // (DdgD)^-1 DdgD = 1
    gaussian_even(L, b, rng);
    D.apply(b, Db);
    D.dagger(Db, DdaggerDb);
    a.zero();
    inverse.apply(DdaggerDb, a);
    d2 = 0;
    for (int64_t i = 0; i < L.volume(); i++)
        for (int sp = 0; sp < 4; sp++)
            for (int c = 0; c < 3; c++) d2 += std::norm(a.at(i).c[sp][c] - b.at(i).c[sp][c]);
    CHECK(d2 * d2 < 1e-16, "test (DdgD)^-1 DdgD");

    // the same in mixed precision (FP16 inner solve, FP64 reliable updates)
    CG<dirac> mixed(D, 1e-12);
    mixed.set_precision(HW_PREC_F16);
    a.zero();
    mixed.apply(DdaggerDb, a);
    CHECK(mixed.last_status() == HW_OK, "mixed-precision CG converged");
    std::printf("facade test passed\n");
    return 0;
}
