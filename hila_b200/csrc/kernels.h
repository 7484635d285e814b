// Host-side launch interface of the CUDA kernels (no CUDA types beyond
// streams and graph handles).  Implemented in dslash_f64.cu and layout.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "wilson_math.cuh"

namespace hw {

constexpr int kHopBlock = 128;
constexpr int kHopMinBlock = 128;  // smallest block of any hop launch shape (sizes reduction buffers)
constexpr int kHopVariants = 3;

// Device-resident scalars of one FP64 conjugate-gradient solve
// (conjugate_gradient.h:55-57 keeps the same quantities on the host).
struct CgState {
    double rr;         // |r|^2 of the current residual
    double pAp;        // |M p|^2
    double alpha, beta;
    double target_rr;  // stop when |r|^2 < target_rr
    double src_norm2;  // |in|^2 over EVEN
    double res_num2;   // last explicit residual check: |b - A x|^2
    double res_den2;   //                                |b|^2
    int iter, maxiter;
    int status;        // CG_RUNNING / CG_CONVERGED / CG_MAXITER / CG_BREAKDOWN
    int do_pupdate;    // set by the CG update, consumed by the p update of the same iteration
};
enum : int { CG_RUNNING = 0, CG_CONVERGED = 1, CG_MAXITER = 2, CG_BREAKDOWN = 3 };

// Work buffers for one grid reduction: partial sums and the arrival ticket.
struct RedBuf {
    double *partials;  // >= 4 * max blocks
    unsigned *ticket;  // one counter, zero between uses
};

// FP64 spinor half-lattice: 12 double2 planes
struct HalfF64 {
    double2 *p;
    int stride;
};

// link_planes: 9 (18 reals) or 6 (12 reals, third row rebuilt)
struct GaugeF64 {
    const double2 *p;
    int stride;
    int planes;
};

// ---- FP64 hopping-term launches. `out` has parity par, `in` the opposite.
// out = a * H_s in
void launch_hop_scale(const Geom &g, const GaugeF64 &U, int par, int sign, HalfF64 in, HalfF64 out, double a,
                      const CgState *st, cudaStream_t s);
// The x-type term of the epilogues below carries a factor d (1 + m_h for the
// Hasenbusch operator M + m_h, Hasenbusch.h:16-52; 1 for M itself).
// out = d x + b * H_s in; with red != null also |out|^2 -> st->pAp and alpha = rr/pAp.
// zero (optional): a half-lattice field on out's sites (the other parity of out) that
// the same launch clears, site i by the thread of output site i.
void launch_hop_xpay(const Geom &g, const GaugeF64 &U, int par, int sign, HalfF64 in, HalfF64 x, HalfF64 out,
                     double b, CgState *st, const RedBuf *red, cudaStream_t s, double d = 1.0,
                     double2 *zero = nullptr);
// CG update fused into the last hop of M^dagger M p:
//   DDp = d Dp + b * H_s t;  r -= alpha DDp;  x += alpha p;  |r|^2 -> st (beta, status)
void launch_hop_cg_update(const Geom &g, const GaugeF64 &U, int par, int sign, HalfF64 t, HalfF64 Dp,
                          HalfF64 r, HalfF64 x, HalfF64 p, double b, CgState *st, const RedBuf &red,
                          cudaStream_t s, double d = 1.0);
// explicit residual: res = src - (d x + b * H_s t); |res|^2 -> st->res_num2, |src|^2 -> st->res_den2
void launch_hop_residual(const Geom &g, const GaugeF64 &U, int par, int sign, HalfF64 t, HalfF64 x,
                         HalfF64 src, HalfF64 res, double b, CgState *st, const RedBuf &red, cudaStream_t s,
                         double d = 1.0);

// ---- FP64 vector kernels over one half lattice
// CG start: r = src - Ax (Ax may be null: x = 0), p = r; sets rr, src_norm2, target_rr, status
void launch_cg_init(int Vh, HalfF64 src, HalfF64 Ax, HalfF64 r, HalfF64 p, double acc2, int maxiter,
                    CgState *st, const RedBuf &red, cudaStream_t s);
// p = r + beta p  (beta from st)
void launch_cg_pupdate(int Vh, HalfF64 r, HalfF64 p, const CgState *st, cudaStream_t s);
// end of a loop-body iteration: clears do_pupdate, enforces maxiter and (use_cond)
// keeps the graph while loop going while st->status == CG_RUNNING
void launch_loop_control(CgState *st, cudaGraphConditionalHandle cond, int use_cond, cudaStream_t s);
// y = a * x
void launch_scale(int Vh, HalfF64 x, HalfF64 y, double a, cudaStream_t s);

// ---- layout conversion (host canonical lexicographic AoS <-> device even-odd SoA)
void launch_spinor_lex_to_eo(const Geom &g, const double *lex, int par, HalfF64 out, cudaStream_t s);
void launch_spinor_eo_to_lex(const Geom &g, HalfF64 in, int par, double *lex, cudaStream_t s);
// checkerboard-ordered AoS [n][12] complex <-> the SoA planes of one half lattice
void launch_aos_to_soa(int n, const double *aos, HalfF64 out, cudaStream_t s);
void launch_soa_to_aos(int n, HalfF64 in, double *aos, cudaStream_t s);
// one direction of links [V][3][3] complex (lexicographic) -> the planes of (par, dir)
void launch_links_lex_to_eo(const Geom &g, const double *lex_dir, double2 *dst, int nplanes, int stride, int par,
                            cudaStream_t s);

}  // namespace hw
