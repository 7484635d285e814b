// The operator blocks of the reference's test program (applications/test_cases/
// test_CG.cpp:127-353) written against the C++ facade the way a HILA application
// writes them: Field<SU<3,double>> U[NDIM], fields with their boundary condition set
// per field, Dirac_Wilson, dirac_staggered_evenodd, Dirac_Wilson_evenodd and
// Hasenbusch_operator with CG<Op>, and MRE_guess.  The links are random SU(3)
// (hw_generate_links, eps 0.3) instead of the reference's unit links, and the
// tolerances are the reference's.  Exit code 0 = every assertion holds.
#include <cmath>
#include <cstdio>
#include <random>

#include "hila_b200/wilson.hpp"

using namespace hila_b200;

#define CHECK(cond, msg)                                  \
    do {                                                  \
        if (!(cond)) {                                    \
            std::fprintf(stderr, "FAILED: %s\n", msg);    \
            return 1;                                     \
        }                                                 \
    } while (0)

static std::mt19937_64 rng(2);

static int parity_of(const Lattice &L, int64_t i) {
    const auto &d = L.size();
    int par = 0;
    for (int k = 0; k < 4; k++) {
        par += (int)(i % d[k]);
        i /= d[k];
    }
    return par & 1;
}

// onsites(par) { f[X].gaussian_random(); }   (par: 0 EVEN, 1 ODD, 2 ALL)
template <typename V>
static void gaussian(Field<V> &f, int par) {
    std::normal_distribution<double> n(0.0, 1.0);
    Lattice &L = f.lattice();
    for (int64_t i = 0; i < L.volume(); i++) {
        if (par != 2 && parity_of(L, i) != par) continue;
        V &v = f[i];
        std::complex<double> *c = reinterpret_cast<std::complex<double> *>(&v);
        for (size_t k = 0; k < sizeof(V) / sizeof(std::complex<double>); k++) c[k] = {n(rng), n(rng)};
    }
}

// sum over par of a[X].dot(b[X]) (conj(a) b)
template <typename V>
static std::complex<double> dot(const Field<V> &a, const Field<V> &b, int par) {
    Lattice &L = a.lattice();
    std::complex<double> s = 0;
    for (int64_t i = 0; i < L.volume(); i++) {
        if (par != 2 && parity_of(L, i) != par) continue;
        const std::complex<double> *x = reinterpret_cast<const std::complex<double> *>(&a.at(i));
        const std::complex<double> *y = reinterpret_cast<const std::complex<double> *>(&b.at(i));
        for (size_t k = 0; k < sizeof(V) / sizeof(std::complex<double>); k++) s += std::conj(x[k]) * y[k];
    }
    return s;
}

// sum over par of squarenorm(a[X] - b[X])
template <typename V>
static double diff2(const Field<V> &a, const Field<V> &b, int par) {
    Lattice &L = a.lattice();
    double s = 0;
    for (int64_t i = 0; i < L.volume(); i++) {
        if (par != 2 && parity_of(L, i) != par) continue;
        const std::complex<double> *x = reinterpret_cast<const std::complex<double> *>(&a.at(i));
        const std::complex<double> *y = reinterpret_cast<const std::complex<double> *>(&b.at(i));
        for (size_t k = 0; k < sizeof(V) / sizeof(std::complex<double>); k++) s += std::norm(x[k] - y[k]);
    }
    return s;
}

int main() {
    Lattice lattice({16, 8, 8, 8}, 0, false);  // fields periodic unless set otherwise, as in HILA
    Field<SU<3, double>> U[4];
    {
        std::vector<SU<3, double>> links((size_t)4 * lattice.volume());
        check(hw_generate_links(lattice.size().data(), 0.3, 2, reinterpret_cast<double *>(links.data())));
        for (int d = 0; d < 4; d++)
            for (int64_t i = 0; i < lattice.volume(); i++) U[d][i] = links[(size_t)d * lattice.volume() + i];
    }
    const int E = 0, ALLS = 2;

    // Dirac_Wilson (test_CG.cpp:127-182)
    {
        using dirac = Dirac_Wilson<SU<3, double>>;
        dirac D(0.05, U);
        Field<WilsonVector> a, b, Db, Ddaggera, DdaggerDb;
        a.set_boundary_condition(e_t, bc::ANTIPERIODIC);
        b.copy_boundary_condition(a);
        Db.copy_boundary_condition(a);
        Ddaggera.copy_boundary_condition(a);
        DdaggerDb.copy_boundary_condition(a);
        gaussian(a, ALLS);
        gaussian(b, ALLS);
        D.apply(b, Db);
        D.dagger(a, Ddaggera);
        std::complex<double> d = dot(a, Db, ALLS) - dot(Ddaggera, b, ALLS);
        CHECK(d.real() * d.real() < 1e-16 && d.imag() * d.imag() < 1e-16, "test Dirac_Wilson");
        CG<dirac> inverse(D);
        b.zero();
        gaussian(a, ALLS);
        inverse.apply(a, b);
        // D^dag (D b): test_CG.cpp:160-162 applies dagger first, which equals this only for
        // its unit links (the free operator is normal); CG<Op> solves D^dag D b = a
        D.apply(b, Db);
        D.dagger(Db, DdaggerDb);
        double r = diff2(a, DdaggerDb, ALLS);
        CHECK(r * r < 1e-8, "test DdgD (DdgD)^-1");
        b.zero();
        gaussian(a, ALLS);
        D.dagger(a, Ddaggera);
        inverse.apply(Ddaggera, b);
        D.apply(b, Db);
        r = diff2(a, Db, ALLS);
        CHECK(r * r < 1e-8, "test D (DdgD)^-1 Ddg");
        std::printf("Dirac_Wilson ok (%d iterations)\n", inverse.last_iterations());
    }

    // dirac_staggered_evenodd (test_CG.cpp:184-212)
    {
        dirac_staggered_evenodd D(5.0, U);
        Field<SU_vector<3, double>> a, b, Db, Ddaggera, DdaggerDb;
        gaussian(a, ALLS);
        gaussian(b, ALLS);
        D.apply(b, Db);
        D.dagger(a, Ddaggera);
        std::complex<double> d = dot(a, Db, E) - dot(Ddaggera, b, E);
        CHECK(d.real() * d.real() < 1e-16 && d.imag() * d.imag() < 1e-16, "test dirac_staggered_evenodd");
        CG<dirac_staggered_evenodd> inverse(D);
        b.zero();
        inverse.apply(Ddaggera, b);
        D.apply(b, Db);
        const double r = diff2(a, Db, E);
        CHECK(r * r < 1e-8, "test CG");
        std::printf("dirac_staggered_evenodd ok (%d iterations)\n", inverse.last_iterations());
    }

    // Dirac_Wilson_evenodd (test_CG.cpp:214-288)
    {
        using dirac = Dirac_Wilson_evenodd<SU<3, double>>;
        dirac D(0.12, U);
        Field<WilsonVector> a, b, Db, Ddaggera, DdaggerDb;
        for (Field<WilsonVector> *f : {&a, &b, &Db, &Ddaggera, &DdaggerDb})
            f->set_boundary_condition(e_t, bc::ANTIPERIODIC);
        a.zero(ODD);
        b.zero(ODD);
        gaussian(a, E);
        gaussian(b, E);
        D.apply(b, Db);
        D.dagger(a, Ddaggera);
        std::complex<double> d = dot(a, Db, E) - dot(Ddaggera, b, E);
        CHECK(d.real() * d.real() < 1e-16 && d.imag() * d.imag() < 1e-16, "test Dirac_Wilson_evenodd");
        CG<dirac> inverse(D);
        a.zero();
        b.zero();
        gaussian(a, E);
        D.dagger(a, Ddaggera);
        inverse.apply(Ddaggera, b);
        D.apply(b, Db);
        double r = diff2(a, Db, E);
        std::printf("D inv Dg %g\n", r);
        CHECK(r * r < 1e-16, "test D (DdgD)^-1 Ddg");
        gaussian(a, E);
        b.zero();
        inverse.apply(a, b);
        D.apply(b, Db);
        D.dagger(Db, DdaggerDb);
        r = diff2(a, DdaggerDb, E);
        CHECK(r * r < 1e-16, "test DdgD (DdgD)^-1");
        gaussian(b, E);
        D.apply(b, Db);
        D.dagger(Db, DdaggerDb);
        a.zero();
        inverse.apply(DdaggerDb, a);
        r = diff2(a, b, E);
        CHECK(r * r < 1e-16, "test (DdgD)^-1 DdgD");
        // MRE_guess from two earlier solutions, then CG from the guess
        Field<WilsonVector> x1, x2, guess;
        for (Field<WilsonVector> *f : {&x1, &x2, &guess}) f->set_boundary_condition(e_t, bc::ANTIPERIODIC);
        inverse.apply(a, x1);
        inverse.apply(DdaggerDb, x2);
        MRE_guess(guess, a, D, {&x1, &x2});
        CG<dirac> from_guess(D);
        from_guess.apply(a, guess);
        CHECK(from_guess.last_status() == HW_OK && from_guess.last_iterations() < inverse.last_iterations(),
              "MRE_guess: CG from the guess takes fewer iterations");
        std::printf("Dirac_Wilson_evenodd ok\n");
    }

    // Hasenbusch_operator (test_CG.cpp:290-353)
    {
        using dirac_base = Dirac_Wilson_evenodd<SU<3, double>>;
        dirac_base Dbase(0.1, U);
        using dirac = Hasenbusch_operator<dirac_base>;
        dirac D(Dbase, 0.1);
        Field<WilsonVector> a, b, Db, Ddaggera, DdaggerDb;
        a.zero(ODD);
        b.zero(ODD);
        gaussian(a, E);
        gaussian(b, E);
        D.apply(b, Db);
        D.dagger(a, Ddaggera);
        std::complex<double> d = dot(a, Db, E) - dot(Ddaggera, b, E);
        CHECK(d.real() * d.real() < 1e-16 && d.imag() * d.imag() < 1e-16, "test Hasenbusch_operator");
        CG<dirac> inverse(D);
        b.zero();
        inverse.apply(Ddaggera, b);
        D.apply(b, Db);
        double r = diff2(a, Db, E);
        CHECK(r * r < 1e-16, "test CG");
        gaussian(a, E);
        b.zero();
        inverse.apply(a, b);
        D.apply(b, Db);
        D.dagger(Db, DdaggerDb);
        r = diff2(a, DdaggerDb, E);
        CHECK(r * r < 1e-16, "test DdgD (DdgD)^-1");
        gaussian(b, E);
        D.apply(b, Db);
        D.dagger(Db, DdaggerDb);
        a.zero();
        inverse.apply(DdaggerDb, a);
        r = diff2(a, b, E);
        CHECK(r * r < 1e-16, "test (DdgD)^-1 DdgD");
        std::printf("Hasenbusch_operator ok\n");
    }
    std::printf("reference blocks passed\n");
    return 0;
}
