// hila_b200/wilson.hpp — header-only C++ facade with HILA's class names and call
// signatures over the C ABI in ../hila_b200.h.
//
//   reference                                             here
//   lattice.setup(size)                                   hila_b200::Lattice L(size)  (the current lattice)
//   Field<SU<3,double>> U[NDIM]                           same, or hila_b200::GaugeField
//   Field<Wilson_vector<3,double>>                        same (Field<WilsonVector>)
//   Field<SU_vector<3,double>>                            same (staggered fields)
//   f.set_boundary_condition(e_t, hila::bc::ANTIPERIODIC) same (bc::ANTIPERIODIC; t direction)
//   Dirac_Wilson_evenodd<SU<3,double>> D(kappa, U)        same (libraries/dirac/wilson.h:234-312)
//   Dirac_Wilson<SU<3,double>> D(kappa, U)                same (wilson.h:146-201)
//   Hasenbusch_operator<Op> D(Dbase, mh)                  same (dirac/Hasenbusch.h:14-52)
//   dirac_staggered_evenodd D(mass, U)                    same (dirac/staggered.h:193-279)
//       D.apply(in, out) / D.dagger(in, out)              same
//   CG<decltype(D)> inv(D[, acc[, maxiters]])             same (conjugate_gradient.h:33-40)
//       inv.apply(in, out)                                same (conjugate_gradient.h:46-104)
//   MRE_guess(psi, chi, D, old_chi_inv)                   same (hmc/MRE_guess.h:9-88)
//
// Fields keep a host copy in HILA's canonical lexicographic layout (x fastest,
// [spin][colour] per site) for element access and mirror it to the device on
// demand; operators run on the device copies only.  Writing through a non-const
// operator[] marks the host copy changed; reads through at() or a const Field leave
// the device copy as it is.  The fermion boundary condition belongs to the field, as
// in HILA: a field lives on the device lattice of its condition in t (periodic or
// antiperiodic), and an operator uses the gauge field of its input's condition.
// Errors throw hila_b200::error (the reference asserts); CG keeps `void apply(...)`
// and exposes last_status(), last_iterations() and last_true_residual().
#pragma once

#include <array>
#include <complex>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../hila_b200.h"

namespace hila_b200 {

struct error : std::runtime_error {
    int code;
    error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != HW_OK) throw error(rc, std::string("hila_b200: ") + hw_last_error());
}

enum class Parity : int { even = HW_EVEN, odd = HW_ODD, all = HW_ALL };
constexpr Parity EVEN = Parity::even, ODD = Parity::odd, ALL = Parity::all;

// coordinates.h: e_x .. e_t
enum Direction : int { e_x = 0, e_y = 1, e_z = 2, e_t = 3 };

// hila::bc
namespace bc {
enum BoundaryCondition : int { PERIODIC = 0, ANTIPERIODIC = 1 };
}

// One lattice on one GPU (lattice.setup(size) + the device context).  The most
// recently constructed lattice is the current one, which fields constructed without
// a lattice use (HILA's global `lattice`).  Fields start with the t boundary
// condition given here.
class Lattice {
  public:
    Lattice(std::array<int, 4> dims, int device = 0, bool t_antiperiodic = true)
        : dims_(dims), default_ap_(t_antiperiodic) {
        check(hw_context_create(device, &ctx_));
        volume_ = (int64_t)dims[0] * dims[1] * dims[2] * dims[3];
        try {
            handle(default_ap_);
        } catch (...) {
            hw_context_destroy(ctx_);
            throw;
        }
        current() = this;
    }
    ~Lattice() {
        for (hw_lattice *l : lat_)
            if (l) hw_lattice_destroy(l);
        hw_context_destroy(ctx_);
        if (current() == this) current() = nullptr;
    }
    Lattice(const Lattice &) = delete;
    Lattice &operator=(const Lattice &) = delete;
    int64_t volume() const { return volume_; }
    const std::array<int, 4> &size() const { return dims_; }
    // the device lattice of fermion fields with this t boundary condition
    hw_lattice *handle(bool antiperiodic) {
        hw_lattice *&l = lat_[antiperiodic ? 1 : 0];
        if (!l) check(hw_lattice_create(ctx_, dims_.data(), antiperiodic ? 1 : 0, &l));
        return l;
    }
    hw_lattice *handle() { return handle(default_ap_); }
    bool default_antiperiodic() const { return default_ap_; }
    hw_context *context() const { return ctx_; }
    int64_t index(int x, int y, int z, int t) const {
        return x + (int64_t)dims_[0] * (y + (int64_t)dims_[1] * (z + (int64_t)dims_[2] * t));
    }
    static Lattice *&current() {
        static Lattice *cur = nullptr;
        return cur;
    }

  private:
    std::array<int, 4> dims_;
    bool default_ap_;
    hw_context *ctx_ = nullptr;
    hw_lattice *lat_[2] = {nullptr, nullptr};
    int64_t volume_ = 0;
};

inline Lattice &current_lattice() {
    if (!Lattice::current()) throw error(HW_ERR_INVALID, "hila_b200: no lattice has been set up");
    return *Lattice::current();
}

template <int N, typename T>
struct SU {
    std::complex<T> e[N][N];
};

template <int N, typename T>
struct WilsonVector_t {
    std::complex<T> c[4][N];  // [spin][colour]
};
using WilsonVector = WilsonVector_t<3, double>;
template <int N, typename T>
using Wilson_vector = WilsonVector_t<N, T>;

template <int N, typename T>
struct SU_vector {
    std::complex<T> c[N];  // colour
};

// device calls of the two fermion field kinds
template <typename V>
struct FieldOps;
template <>
struct FieldOps<WilsonVector> {
    using handle_type = hw_field;
    static constexpr int reals = 24;
    static int create(hw_lattice *l, hw_field **f) { return hw_field_create(l, f); }
    static int destroy(hw_field *f) { return hw_field_destroy(f); }
    static int upload(hw_field *f, const double *h) { return hw_field_upload(f, h, HW_ALL); }
    static int download(const hw_field *f, double *h) { return hw_field_download(f, h, HW_ALL); }
};
template <>
struct FieldOps<SU_vector<3, double>> {
    using handle_type = hw_stag_field;
    static constexpr int reals = 6;
    static int create(hw_lattice *l, hw_stag_field **f) { return hw_stag_field_create(l, f); }
    static int destroy(hw_stag_field *f) { return hw_stag_field_destroy(f); }
    static int upload(hw_stag_field *f, const double *h) { return hw_stag_field_upload(f, h, HW_ALL); }
    static int download(const hw_stag_field *f, double *h) { return hw_stag_field_download(f, h, HW_ALL); }
};

// Field<V> for the fermion vector types: host mirror + device field.
template <typename V>
class Field {
    using Ops = FieldOps<V>;
    using H = typename Ops::handle_type;

  public:
    Field() : Field(current_lattice()) {}
    explicit Field(Lattice &lat) : lat_(&lat), ap_(lat.default_antiperiodic()), host_((size_t)lat.volume()) {
        check(Ops::create(lat.handle(ap_), &f_));
    }
    ~Field() { Ops::destroy(f_); }
    Field(const Field &) = delete;
    Field &operator=(const Field &) = delete;

    // element access: writing through it marks the host copy changed
    V &operator[](int64_t i) {
        pull();
        dirty_host_ = true;
        return host_[i];
    }
    // reads leave the device copy as it is
    const V &operator[](int64_t i) const { return at(i); }
    const V &at(int64_t i) const {
        pull();
        return host_[i];
    }
    // f[par] = 0
    void zero(Parity p = ALL) {
        pull();
        const auto &d = lat_->size();
        for (int64_t i = 0; i < lat_->volume(); i++) {
            int64_t r = i;
            int par = 0;
            for (int k = 0; k < 4; k++) {
                par += (int)(r % d[k]);
                r /= d[k];
            }
            const bool odd = par & 1;
            if (p == ALL || (p == ODD) == odd) host_[i] = V{};
        }
        dirty_host_ = true;
    }
    // HILA's fermion boundary condition; the kernels implement it in the t direction
    void set_boundary_condition(Direction d, bc::BoundaryCondition b) {
        if (d != e_t) {
            if (b != bc::PERIODIC) throw error(HW_ERR_INVALID, "hila_b200: antiperiodic only in the t direction");
            return;
        }
        const bool ap = b == bc::ANTIPERIODIC;
        if (ap == ap_) return;
        pull();
        H *nf = nullptr;
        check(Ops::create(lat_->handle(ap), &nf));
        Ops::destroy(f_);
        f_ = nf;
        ap_ = ap;
        dirty_host_ = true;  // the new device field receives the values at the next push
    }
    template <typename W>
    void copy_boundary_condition(const Field<W> &o) {
        set_boundary_condition(e_t, o.antiperiodic() ? bc::ANTIPERIODIC : bc::PERIODIC);
    }
    bool antiperiodic() const { return ap_; }
    // host edits to the device (called by the operators)
    void push() const {
        if (dirty_host_) check(Ops::upload(f_, data()));
        dirty_host_ = false;
    }
    // device values into the host mirror
    void pull() const {
        if (stale_host_) check(Ops::download(f_, const_cast<double *>(data())));
        stale_host_ = false;
    }
    void mark_device_changed() { stale_host_ = true; }
    H *handle() const { return f_; }
    const double *data() const { return reinterpret_cast<const double *>(host_.data()); }
    Lattice &lattice() const { return *lat_; }

  private:
    Lattice *lat_;
    bool ap_;
    H *f_ = nullptr;
    mutable std::vector<V> host_;
    mutable bool dirty_host_ = true;
    mutable bool stale_host_ = false;
};

// Field<SU<3,double>>: one direction of a gauge field, host resident (the operators
// upload the four directions together when one of them changed).
template <>
class Field<SU<3, double>> {
  public:
    Field() : Field(current_lattice()) {}
    explicit Field(Lattice &lat) : lat_(&lat), host_((size_t)lat.volume()) {}
    SU<3, double> &operator[](int64_t i) {
        ++version_;
        return host_[i];
    }
    const SU<3, double> &operator[](int64_t i) const { return host_[i]; }
    // U[d][ALL] = 1
    void unit() {
        ++version_;
        for (auto &u : host_)
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) u.e[i][j] = (i == j) ? 1.0 : 0.0;
    }
    uint64_t version() const { return version_; }
    const SU<3, double> *data() const { return host_.data(); }
    SU<3, double> *data_for_write() {
        ++version_;
        return host_.data();
    }
    Lattice &lattice() const { return *lat_; }

  private:
    Lattice *lat_;
    std::vector<SU<3, double>> host_;
    uint64_t version_ = 1;
};

// The four directions of Field<SU<3,double>> U[NDIM] held as device gauge fields (one
// per fermion boundary condition, built on first use).
class GaugeField {
  public:
    GaugeField(Lattice &lat, int link_format = HW_LINKS_18)
        : lat_(&lat), links_((size_t)4 * lat.volume()), fmt_(link_format) {}
    ~GaugeField() { invalidate(); }
    GaugeField(const GaugeField &) = delete;
    GaugeField &operator=(const GaugeField &) = delete;
    SU<3, double> &link(int dir, int64_t site) {
        invalidate();
        return links_[(size_t)dir * lat_->volume() + site];
    }
    // seeded links exp(i eps H), see hw_generate_links
    void random(double eps, uint64_t seed) {
        invalidate();
        check(hw_generate_links(lat_->size().data(), eps, seed, reinterpret_cast<double *>(links_.data())));
    }
    void unit() {
        invalidate();
        for (auto &u : links_)
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) u.e[i][j] = (i == j) ? 1.0 : 0.0;
    }
    // the links of Field<SU<3,double>> U[4]
    void assign(const Field<SU<3, double>> (&U)[4]) {
        invalidate();
        const int64_t V = lat_->volume();
        for (int d = 0; d < 4; d++)
            for (int64_t i = 0; i < V; i++) links_[(size_t)d * V + i] = U[d][i];
    }
    // GaugeField::config_write / config_read (gaugefield.h:196-271), HILA's binary format
    void config_write(const std::string &filename) const {
        check(hw_gauge_config_write(filename.c_str(), lat_->size().data(),
                                    reinterpret_cast<const double *>(links_.data())));
    }
    void config_read(const std::string &filename) {
        invalidate();
        check(hw_gauge_config_read(filename.c_str(), lat_->size().data(), reinterpret_cast<double *>(links_.data())));
    }
    // the device gauge field on the lattice of fermion fields with this t boundary condition
    hw_gauge *handle(bool antiperiodic) {
        hw_gauge *&g = g_[antiperiodic ? 1 : 0];
        if (!g)
            check(hw_gauge_create(lat_->handle(antiperiodic), reinterpret_cast<const double *>(links_.data()), fmt_,
                                  &g));
        return g;
    }
    hw_gauge *handle() { return handle(lat_->default_antiperiodic()); }
    Lattice &lattice() { return *lat_; }

  private:
    void invalidate() {
        for (hw_gauge *&g : g_) {
            if (g) hw_gauge_destroy(g);
            g = nullptr;
        }
    }
    Lattice *lat_;
    std::vector<SU<3, double>> links_;
    int fmt_;
    hw_gauge *g_[2] = {nullptr, nullptr};
};

// An operator's gauge field: a GaugeField, or Field<SU<3,double>> U[4] that the operator
// keeps a reference to (as the reference does, wilson.h:237) and uploads when changed.
class GaugeRef {
  public:
    explicit GaugeRef(GaugeField &g) : g_(&g) {}
    explicit GaugeRef(Field<SU<3, double>> (&U)[4]) : U_(U) {}
    GaugeRef(const GaugeRef &o) : g_(o.g_), U_(o.U_) {}
    hw_gauge *handle(bool antiperiodic) {
        if (g_) return g_->handle(antiperiodic);
        uint64_t v = 0;
        for (int d = 0; d < 4; d++) v += U_[d].version();
        if (!own_ || v != version_) {
            own_.reset(new GaugeField(U_[0].lattice()));
            own_->assign(*reinterpret_cast<Field<SU<3, double>>(*)[4]>(U_));
            version_ = v;
        }
        return own_->handle(antiperiodic);
    }
    Lattice &lattice() { return g_ ? g_->lattice() : U_[0].lattice(); }

  private:
    GaugeField *g_ = nullptr;
    Field<SU<3, double>> *U_ = nullptr;
    std::shared_ptr<GaugeField> own_;
    uint64_t version_ = 0;
};

// the boundary conditions of an operator's fields must agree
template <typename V>
inline bool same_bc(const Field<V> &in, const Field<V> &out) {
    if (in.antiperiodic() != out.antiperiodic())
        throw error(HW_ERR_INVALID, "hila_b200: input and output fields have different boundary conditions");
    return in.antiperiodic();
}

constexpr int CG_DEFAULT_MAXITERS = 10000;
constexpr double CG_DEFAULT_ACCURACY = 1e-12;

// Dirac_Wilson_evenodd<SU<3,double>> (libraries/dirac/wilson.h:234-312)
template <typename matrix>
class Dirac_Wilson_evenodd {
  public:
    using vector_type = WilsonVector;
    using matrix_type = matrix;
    static constexpr int N = 3;
    double kappa;
    Parity par = EVEN;

    Dirac_Wilson_evenodd(double k, GaugeField &U) : kappa(k), U_(U) {}
    Dirac_Wilson_evenodd(double k, Field<SU<3, double>> (&U)[4]) : kappa(k), U_(U) {}
    Dirac_Wilson_evenodd(Dirac_Wilson_evenodd &d) : kappa(d.kappa), U_(d.U_) {}

    void apply(const Field<vector_type> &in, Field<vector_type> &out) { run(in, out, 1); }
    void dagger(const Field<vector_type> &in, Field<vector_type> &out) { run(in, out, -1); }
    // force(chi, psi, force, sign), wilson.h:293-311: force[dir][site] = dS/dU_dir(site)
    // of S = Re(chi^dag M_s psi), lexicographic sites
    void force(const Field<vector_type> &chi, const Field<vector_type> &psi, std::vector<SU<3, double>> (&force)[4],
               int sign) {
        const bool ap = same_bc(chi, psi);
        chi.push();
        psi.push();
        const int64_t V = U_.lattice().volume();
        std::vector<SU<3, double>> all((size_t)(4 * V));
        check(hw_wilson_evenodd_force(U_.handle(ap), kappa, chi.handle(), psi.handle(), sign,
                                      reinterpret_cast<double *>(all.data())));
        for (int d = 0; d < 4; d++) force[d].assign(all.begin() + d * V, all.begin() + (d + 1) * V);
    }
    // CG<Op>::apply for this operator: M^dag M out = in on EVEN
    int solve(const Field<vector_type> &in, Field<vector_type> &out, hw_cg_params p, hw_cg_result *r) {
        const bool ap = same_bc(in, out);
        in.push();
        out.push();
        int rc = hw_cg_solve(U_.handle(ap), kappa, in.handle(), out.handle(), &p, r);
        out.mark_device_changed();
        return rc;
    }
    hw_gauge *gauge_handle(bool ap) { return U_.handle(ap); }

  private:
    void run(const Field<vector_type> &in, Field<vector_type> &out, int sign) {
        const bool ap = same_bc(in, out);
        in.push();
        out.push();
        check(sign > 0 ? hw_wilson_evenodd_apply(U_.handle(ap), kappa, in.handle(), out.handle())
                       : hw_wilson_evenodd_dagger(U_.handle(ap), kappa, in.handle(), out.handle()));
        out.mark_device_changed();
    }
    GaugeRef U_;
};

// Dirac_Wilson<SU<3,double>> (wilson.h:146-201): D_s = 1 - kappa H_s on ALL sites
template <typename matrix>
class Dirac_Wilson {
  public:
    using vector_type = WilsonVector;
    using matrix_type = matrix;
    double kappa;
    Parity par = ALL;

    Dirac_Wilson(double k, GaugeField &U) : kappa(k), U_(U) {}
    Dirac_Wilson(double k, Field<SU<3, double>> (&U)[4]) : kappa(k), U_(U) {}
    Dirac_Wilson(Dirac_Wilson &d) : kappa(d.kappa), U_(d.U_) {}

    void apply(const Field<vector_type> &in, Field<vector_type> &out) { run(in, out, 1); }
    void dagger(const Field<vector_type> &in, Field<vector_type> &out) { run(in, out, -1); }
    // CG<Dirac_Wilson>::apply: M^dag M out = in on ALL sites (FP64)
    int solve(const Field<vector_type> &in, Field<vector_type> &out, hw_cg_params p, hw_cg_result *r) {
        const bool ap = same_bc(in, out);
        in.push();
        out.push();
        p.precision = HW_PREC_F64;
        int rc = hw_wilson_cg_solve(U_.handle(ap), kappa, in.handle(), out.handle(), &p, r);
        out.mark_device_changed();
        return rc;
    }

  private:
    void run(const Field<vector_type> &in, Field<vector_type> &out, int sign) {
        const bool ap = same_bc(in, out);
        in.push();
        out.push();
        check(hw_wilson_apply(U_.handle(ap), kappa, sign, in.handle(), out.handle()));
        out.mark_device_changed();
    }
    GaugeRef U_;
};

// Hasenbusch_operator<Dirac_Wilson_evenodd<...>> (dirac/Hasenbusch.h:14-52): M + m_h on EVEN
template <typename Dirac_type>
class Hasenbusch_operator {
  public:
    using vector_type = typename Dirac_type::vector_type;
    Dirac_type D;
    Parity par;
    double h_parameter;

    Hasenbusch_operator(Dirac_type &d, double hasenbusch_parameter)
        : D(d), par(d.par), h_parameter(hasenbusch_parameter) {}
    Hasenbusch_operator(Hasenbusch_operator &h) : D(h.D), par(h.par), h_parameter(h.h_parameter) {}

    void apply(const Field<vector_type> &in, Field<vector_type> &out) { run(in, out, 1); }
    void dagger(const Field<vector_type> &in, Field<vector_type> &out) { run(in, out, -1); }
    int solve(const Field<vector_type> &in, Field<vector_type> &out, hw_cg_params p, hw_cg_result *r) {
        p.hasenbusch_mh = h_parameter;
        return D.solve(in, out, p, r);
    }

  private:
    void run(const Field<vector_type> &in, Field<vector_type> &out, int sign) {
        const bool ap = same_bc(in, out);
        in.push();
        out.push();
        hw_gauge *g = D.gauge_handle(ap);
        check(sign > 0 ? hw_hasenbusch_evenodd_apply(g, D.kappa, h_parameter, in.handle(), out.handle())
                       : hw_hasenbusch_evenodd_dagger(g, D.kappa, h_parameter, in.handle(), out.handle()));
        out.mark_device_changed();
    }
};

// dirac_staggered_evenodd (dirac/staggered.h:193-279) on Field<SU_vector<3,double>>
class dirac_staggered_evenodd {
  public:
    using vector_type = SU_vector<3, double>;
    double mass;
    Parity par = EVEN;

    dirac_staggered_evenodd(double m, GaugeField &U) : mass(m), U_(U) {}
    dirac_staggered_evenodd(double m, Field<SU<3, double>> (&U)[4]) : mass(m), U_(U) {}
    dirac_staggered_evenodd(dirac_staggered_evenodd &d) : mass(d.mass), U_(d.U_) {}

    void apply(const Field<vector_type> &in, Field<vector_type> &out) { run(in, out, 1); }
    void dagger(const Field<vector_type> &in, Field<vector_type> &out) { run(in, out, -1); }
    int solve(const Field<vector_type> &in, Field<vector_type> &out, hw_cg_params p, hw_cg_result *r) {
        const bool ap = same_bc(in, out);
        in.push();
        out.push();
        p.precision = HW_PREC_F64;
        int rc = hw_staggered_cg_solve(U_.handle(ap), mass, in.handle(), out.handle(), &p, r);
        out.mark_device_changed();
        return rc;
    }

  private:
    void run(const Field<vector_type> &in, Field<vector_type> &out, int sign) {
        const bool ap = same_bc(in, out);
        in.push();
        out.push();
        check(sign > 0 ? hw_staggered_evenodd_apply(U_.handle(ap), mass, in.handle(), out.handle())
                       : hw_staggered_evenodd_dagger(U_.handle(ap), mass, in.handle(), out.handle()));
        out.mark_device_changed();
    }
    GaugeRef U_;
};

// CG<Op> (libraries/dirac/conjugate_gradient.h:18-104): apply(in, out) solves
// (M^dag M) out = in on the operator's parity; out holds the initial guess.
template <typename Op>
class CG {
  public:
    using vector_type = typename Op::vector_type;
    CG(Op &op) : M_(op) {}
    CG(Op &op, double accuracy) : M_(op), accuracy_(accuracy) {}
    CG(Op &op, double accuracy, int maxiters) : M_(op), accuracy_(accuracy), maxiters_(maxiters) {}

    // Wilson even-odd operators: mixed precision (HW_PREC_F32 / HW_PREC_F16 inner solve
    // with FP64 reliable updates); the other operators solve in FP64
    void set_precision(int precision) { precision_ = precision; }

    void apply(const Field<vector_type> &in, Field<vector_type> &out) {
        hw_cg_params p;
        hw_cg_params_default(&p);
        p.accuracy = accuracy_;
        p.maxiters = maxiters_;
        p.precision = precision_;
        const int rc = M_.solve(in, out, p, &last_);
        if (rc != HW_OK && rc != HW_ERR_NOT_CONVERGED && rc != HW_ERR_BREAKDOWN) check(rc);
    }
    int last_status() const { return last_.status; }
    int last_iterations() const { return last_.iterations; }
    double last_true_residual() const { return last_.true_residual; }
    double last_relative_residue() const { return last_.rr_relative; }

  private:
    Op &M_;
    double accuracy_ = CG_DEFAULT_ACCURACY;
    int maxiters_ = CG_DEFAULT_MAXITERS;
    int precision_ = HW_PREC_F64;
    hw_cg_result last_{};
};

// MRE_guess(psi, chi, D, old_chi_inv) (hmc/MRE_guess.h:9-88): initial guess psi for
// CG<Op> on (M^dag M) psi = chi from earlier solutions, for Dirac_Wilson_evenodd and
// its Hasenbusch_operator (hw_mre_guess).  The earlier solutions are passed by pointer
// (the reference takes a vector of Field copies; these fields are not copyable).
template <typename matrix>
void MRE_guess(Field<WilsonVector> &psi, Field<WilsonVector> &chi, Dirac_Wilson_evenodd<matrix> &D,
               std::vector<Field<WilsonVector> *> old_chi_inv, double mh = 0.0) {
    const bool ap = same_bc(psi, chi);
    std::vector<const hw_field *> h;
    for (Field<WilsonVector> *f : old_chi_inv) {
        f->push();
        h.push_back(f->handle());
    }
    chi.push();
    psi.push();
    check(hw_mre_guess(D.gauge_handle(ap), D.kappa, mh, h.data(), (int)h.size(), chi.handle(), psi.handle()));
    psi.mark_device_changed();
}

template <typename Dirac_type>
void MRE_guess(Field<WilsonVector> &psi, Field<WilsonVector> &chi, Hasenbusch_operator<Dirac_type> &H,
               std::vector<Field<WilsonVector> *> old_chi_inv) {
    MRE_guess(psi, chi, H.D, old_chi_inv, H.h_parameter);
}

}  // namespace hila_b200
