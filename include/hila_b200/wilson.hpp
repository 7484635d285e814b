// hila_b200/wilson.hpp — header-only C++ facade with HILA's class names and call
// signatures over the C ABI in ../hila_b200.h.
//
//   reference                                             here
//   Field<SU<3,double>> U[NDIM]                           hila_b200::GaugeField (or Field<SU<3,double>> U[4])
//   Field<Wilson_vector<3,double>>                        hila_b200::Field<WilsonVector>
//   Dirac_Wilson_evenodd<SU<3,double>> D(kappa, U)        hila_b200::Dirac_Wilson_evenodd<SU<3,double>>
//       D.apply(in, out) / D.dagger(in, out)              same (libraries/dirac/wilson.h:272-289)
//   CG<decltype(D)> inv(D[, acc[, maxiters]])             hila_b200::CG<...>  (conjugate_gradient.h:33-40)
//       inv.apply(in, out)                                same (conjugate_gradient.h:46-104)
//
// Fields keep a host copy in HILA's canonical lexicographic layout (x fastest,
// [spin][colour] per site) for element access and mirror it to the device on
// demand; operators run on the device copies only.  Errors throw
// hila_b200::error (the reference asserts); CG keeps `void apply(...)` and exposes
// last_status(), last_iterations() and last_true_residual().
#pragma once

#include <array>
#include <complex>
#include <cstdint>
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

// One lattice on one GPU (lattice.setup(size) + the device context).
class Lattice {
  public:
    Lattice(std::array<int, 4> dims, int device = 0, bool t_antiperiodic = true) : dims_(dims) {
        check(hw_context_create(device, &ctx_));
        int rc = hw_lattice_create(ctx_, dims.data(), t_antiperiodic ? 1 : 0, &lat_);
        if (rc != HW_OK) {
            hw_context_destroy(ctx_);
            check(rc);
        }
        volume_ = (int64_t)dims[0] * dims[1] * dims[2] * dims[3];
    }
    ~Lattice() {
        hw_lattice_destroy(lat_);
        hw_context_destroy(ctx_);
    }
    Lattice(const Lattice &) = delete;
    Lattice &operator=(const Lattice &) = delete;
    int64_t volume() const { return volume_; }
    const std::array<int, 4> &size() const { return dims_; }
    hw_lattice *handle() const { return lat_; }
    hw_context *context() const { return ctx_; }
    int64_t index(int x, int y, int z, int t) const {
        return x + (int64_t)dims_[0] * (y + (int64_t)dims_[1] * (z + (int64_t)dims_[2] * t));
    }

  private:
    std::array<int, 4> dims_;
    hw_context *ctx_ = nullptr;
    hw_lattice *lat_ = nullptr;
    int64_t volume_ = 0;
};

template <int N, typename T>
struct SU {
    std::complex<T> e[N][N];
};

template <int N, typename T>
struct WilsonVector_t {
    std::complex<T> c[4][N];  // [spin][colour]
};
using WilsonVector = WilsonVector_t<3, double>;

template <typename T>
class Field;

// Field<Wilson_vector<3,double>>: host mirror + device field.
template <>
class Field<WilsonVector> {
  public:
    explicit Field(Lattice &lat) : lat_(&lat), host_((size_t)lat.volume()) {
        check(hw_field_create(lat.handle(), &f_));
    }
    ~Field() { hw_field_destroy(f_); }
    Field(const Field &) = delete;
    Field &operator=(const Field &) = delete;

    WilsonVector &operator[](int64_t i) {
        dirty_host_ = true;
        pull();
        return host_[i];
    }
    const WilsonVector &at(int64_t i) {
        pull();
        return host_[i];
    }
    // f[ALL] = 0, f[ODD] = 0, ...
    void zero(Parity p = ALL) {
        push();
        check(hw_field_zero(f_, (int)p));
        stale_host_ = true;
    }
    // push host edits to the device (called by the operators)
    void push() {
        if (dirty_host_) check(hw_field_upload(f_, data(), HW_ALL));
        dirty_host_ = false;
    }
    // fetch the device values into the host mirror
    void pull() {
        if (stale_host_) check(hw_field_download(f_, data(), HW_ALL));
        stale_host_ = false;
    }
    void mark_device_changed() { stale_host_ = true; }
    hw_field *handle() { return f_; }
    double *data() { return reinterpret_cast<double *>(host_.data()); }
    Lattice &lattice() { return *lat_; }

  private:
    Lattice *lat_;
    hw_field *f_ = nullptr;
    std::vector<WilsonVector> host_;
    bool dirty_host_ = true;
    bool stale_host_ = false;
};

// Field<SU<3,double>> U[NDIM] held as one device gauge field.
class GaugeField {
  public:
    GaugeField(Lattice &lat, int link_format = HW_LINKS_18) : lat_(&lat), links_((size_t)4 * lat.volume()), fmt_(link_format) {}
    ~GaugeField() { hw_gauge_destroy(g_); }
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
    // GaugeField::config_write / config_read (gaugefield.h:196-271), HILA's binary format
    void config_write(const std::string &filename) const {
        check(hw_gauge_config_write(filename.c_str(), lat_->size().data(),
                                    reinterpret_cast<const double *>(links_.data())));
    }
    void config_read(const std::string &filename) {
        invalidate();
        check(hw_gauge_config_read(filename.c_str(), lat_->size().data(), reinterpret_cast<double *>(links_.data())));
    }
    hw_gauge *handle() {
        if (!g_) check(hw_gauge_create(lat_->handle(), reinterpret_cast<const double *>(links_.data()), fmt_, &g_));
        return g_;
    }
    Lattice &lattice() { return *lat_; }

  private:
    void invalidate() {
        if (g_) hw_gauge_destroy(g_);
        g_ = nullptr;
    }
    Lattice *lat_;
    std::vector<SU<3, double>> links_;
    int fmt_;
    hw_gauge *g_ = nullptr;
};

// Dirac_Wilson_evenodd<SU<3,double>> (libraries/dirac/wilson.h:234-312)
template <typename matrix>
class Dirac_Wilson_evenodd {
  public:
    using vector_type = WilsonVector;
    using matrix_type = matrix;
    static constexpr int N = 3;
    double kappa;
    Parity par = EVEN;

    Dirac_Wilson_evenodd(double k, GaugeField &U) : kappa(k), U_(&U) {}
    Dirac_Wilson_evenodd(Dirac_Wilson_evenodd &d) : kappa(d.kappa), U_(d.U_) {}

    void apply(Field<vector_type> &in, Field<vector_type> &out) {
        in.push();
        out.push();
        check(hw_wilson_evenodd_apply(U_->handle(), kappa, in.handle(), out.handle()));
        out.mark_device_changed();
    }
    void dagger(Field<vector_type> &in, Field<vector_type> &out) {
        in.push();
        out.push();
        check(hw_wilson_evenodd_dagger(U_->handle(), kappa, in.handle(), out.handle()));
        out.mark_device_changed();
    }
    // force(chi, psi, force, sign), wilson.h:293-311: force[dir][site] = dS/dU_dir(site)
    // of S = Re(chi^dag M_s psi), lexicographic sites
    void force(Field<vector_type> &chi, Field<vector_type> &psi, std::vector<SU<3, double>> (&force)[4], int sign) {
        chi.push();
        psi.push();
        const int64_t V = U_->lattice().volume();
        std::vector<SU<3, double>> all((size_t)(4 * V));
        check(hw_wilson_evenodd_force(U_->handle(), kappa, chi.handle(), psi.handle(), sign,
                                      reinterpret_cast<double *>(all.data())));
        for (int d = 0; d < 4; d++) force[d].assign(all.begin() + d * V, all.begin() + (d + 1) * V);
    }
    GaugeField &gauge() { return *U_; }

  private:
    GaugeField *U_;
};

constexpr int CG_DEFAULT_MAXITERS = 10000;
constexpr double CG_DEFAULT_ACCURACY = 1e-12;

// CG<Op> (libraries/dirac/conjugate_gradient.h:18-104): apply(in, out) solves
// (M^dag M) out = in on the operator's parity; out holds the initial guess.
template <typename Op>
class CG {
  public:
    using vector_type = typename Op::vector_type;
    CG(Op &op) : M_(op) {}
    CG(Op &op, double accuracy) : M_(op), accuracy_(accuracy) {}
    CG(Op &op, double accuracy, int maxiters) : M_(op), accuracy_(accuracy), maxiters_(maxiters) {}

    // mixed precision (HW_PREC_F32 / HW_PREC_F16 inner solve with FP64 reliable updates)
    void set_precision(int precision) { precision_ = precision; }

    void apply(Field<vector_type> &in, Field<vector_type> &out) {
        in.push();
        out.push();
        hw_cg_params p;
        hw_cg_params_default(&p);
        p.accuracy = accuracy_;
        p.maxiters = maxiters_;
        p.precision = precision_;
        int rc = hw_cg_solve(M_.gauge().handle(), M_.kappa, in.handle(), out.handle(), &p, &last_);
        out.mark_device_changed();
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

}  // namespace hila_b200
