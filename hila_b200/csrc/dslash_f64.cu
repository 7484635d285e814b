// FP64 even-odd Wilson hopping-term kernels with fused epilogues, and the
// FP64 vector kernels of the conjugate gradient.
//
// One thread per output site over the SoA even-odd layout (storage.cuh).  The
// hopping term follows libraries/dirac/wilson.h:15-95 (with the intended
// backward gather vtemp[-dir][X-dir]); instead of the reference's eight
// projection kernels, eight temporary half-spinor fields and four accumulate
// kernels per hop, each output site gathers its eight neighbours, projects,
// multiplies by the link and expands in registers, and the epilogue fuses
// whatever the caller does next (scaling, the diagonal term of the even-odd
// operator, the CG axpy updates and their dot products).
#include <mutex>

#include "kernels.h"
#include "reduce.cuh"
#include "storage.cuh"

namespace hw {

namespace {

__host__ __device__ __forceinline__ SpinorF64 sp(HalfF64 h) { return SpinorF64{h.p, h.stride}; }

// Epilogue operands read at the output site (not at neighbours) are copied into
// shared memory with cp.async when the thread starts, so their HBM reads overlap
// the hop instead of following it.  An epilogue with NPRE > 0 names them in
// pre(k) and reads them from stg (component c of operand k at stg.p[(k*12 + c)
// * BLOCK + threadIdx.x]; `stg.stride` = BLOCK, index ix = threadIdx.x).
// (cp_async16 and cp_async_wait_all: storage.cuh)
// operand k of a staged epilogue as a field over the block's threads
__device__ __forceinline__ SpinorF64 staged(double2 *stage, int block, int k) {
    return SpinorF64{stage + (size_t)k * 12 * block, block};
}

// out = a * H in
struct EpiScale {
    static constexpr int NRED = 0;
    static constexpr int NPRE = 0;
    SpinorF64 out;
    double a;
    const CgState *st;
    __device__ bool skip() const { return st && st->status != CG_RUNNING; }
    __device__ void operator()(int i, Spinor<double> &acc, double *) const {
#pragma unroll
        for (int c = 0; c < 12; c++) acc.s[c / 3][c % 3] = a * acc.s[c / 3][c % 3];
        out.store(i, acc);
    }
};

// Component c (0..11) of a half-lattice FP64 field at site i
__device__ __forceinline__ Cx<double> load_c(const SpinorF64 &f, int c, int i) {
    double2 v = f.p[(size_t)c * f.stride + i];
    return {v.x, v.y};
}
__device__ __forceinline__ void store_c(const SpinorF64 &f, int c, int i, Cx<double> v) {
    f.p[(size_t)c * f.stride + i] = make_double2(v.re, v.im);
}

// d x as an uncontracted product: with d = 1 the sums below round exactly as x + b H in
__device__ __forceinline__ Cx<double> dscale(double d, Cx<double> v) { return {__dmul_rn(d, v.re), __dmul_rn(d, v.im)}; }

// out = d x + b * H in ; optionally pAp = |out|^2 and alpha = rr / pAp.  d = 1 + m_h
// gives the Hasenbusch operator M + m_h (Hasenbusch.h:16-52), d = 1 the plain one.
template <bool RED>
struct EpiXpay {
    static constexpr int NRED = RED ? 1 : 0;
    static constexpr int NPRE = 1;  // x
    SpinorF64 x, out;
    double b;
    CgState *st;
    double d;
    double2 *zero;  // optional: cleared at site i (stride of out)
    __device__ SpinorF64 pre(int) const { return x; }
    __device__ bool skip() const { return st && st->status != CG_RUNNING; }
    __device__ void operator()(int i, Spinor<double> &acc, double *red, double2 *stage, int block) const {
        const SpinorF64 xs = staged(stage, block, 0);
        const int ix = threadIdx.x;
        double n2 = 0;
#pragma unroll
        for (int c = 0; c < 12; c++) {
            Cx<double> v = dscale(d, load_c(xs, c, ix)) + b * acc.s[c / 3][c % 3];
            store_c(out, c, i, v);
            n2 += norm2(v);
        }
        if (zero)
#pragma unroll
            for (int c = 0; c < 12; c++) zero[(size_t)c * out.stride + i] = make_double2(0.0, 0.0);
        if (RED) red[0] = n2;
    }
    __device__ void operator()(const double *tot) {
        st->pAp = tot[0];
        if (!(tot[0] > 0.0) || !isfinite(tot[0])) {
            st->status = CG_BREAKDOWN;
            st->alpha = 0.0;
        } else {
            st->alpha = st->rr / tot[0];
        }
    }
};

// CG step fused into the second hop of M^dagger (conjugate_gradient.h:77-95):
// DDp = d Dp + b H t ; x += alpha p ; r -= alpha DDp ; rrnew = |r|^2
struct EpiCgUpdate {
    static constexpr int NRED = 1;
    static constexpr int NPRE = 2;  // Dp, r
    SpinorF64 Dp, r, x, p;
    double b;
    CgState *st;
    double d;
    __device__ SpinorF64 pre(int k) const { return k == 0 ? Dp : r; }
    __device__ bool skip() const { return st->status != CG_RUNNING; }
    __device__ void operator()(int i, Spinor<double> &acc, double *red, double2 *stage, int block) const {
        const SpinorF64 ds = staged(stage, block, 0), rs = staged(stage, block, 1);
        const int ix = threadIdx.x;
        const double alpha = st->alpha;
        double n2 = 0;
#pragma unroll
        for (int c = 0; c < 12; c++) {
            Cx<double> ddp = dscale(d, load_c(ds, c, ix)) + b * acc.s[c / 3][c % 3];
            Cx<double> rv = load_c(rs, c, ix) - alpha * ddp;
            store_c(r, c, i, rv);
            store_c(x, c, i, load_c(x, c, i) + alpha * load_c(p, c, i));
            n2 += norm2(rv);
        }
        red[0] = n2;
    }
    __device__ void operator()(const double *tot) {
        const double rrnew = tot[0];
        st->iter += 1;
        if (!isfinite(rrnew)) {
            st->status = CG_BREAKDOWN;
        } else {
            st->beta = rrnew / st->rr;
            st->rr = rrnew;
            if (rrnew < st->target_rr)
                st->status = CG_CONVERGED;
            else if (st->iter >= st->maxiter)
                st->status = CG_MAXITER;
        }
        st->do_pupdate = st->status != CG_BREAKDOWN;
    }
};

// res = src - (d x + b H t) ; |res|^2, |src|^2
struct EpiResidual {
    static constexpr int NRED = 2;
    static constexpr int NPRE = 2;  // x, src
    SpinorF64 x, src, res;
    double b;
    CgState *st;
    double d;
    __device__ SpinorF64 pre(int k) const { return k == 0 ? x : src; }
    __device__ bool skip() const { return false; }
    __device__ void operator()(int i, Spinor<double> &acc, double *red, double2 *stage, int block) const {
        const SpinorF64 xs = staged(stage, block, 0), ss = staged(stage, block, 1);
        const int ix = threadIdx.x;
        double n2 = 0, d2 = 0;
#pragma unroll
        for (int c = 0; c < 12; c++) {
            Cx<double> sv = load_c(ss, c, ix);
            Cx<double> v = sv - (dscale(d, load_c(xs, c, ix)) + b * acc.s[c / 3][c % 3]);
            if (res.p) store_c(res, c, i, v);
            n2 += norm2(v);
            d2 += norm2(sv);
        }
        red[0] = n2;
        red[1] = d2;
    }
    __device__ void operator()(const double *tot) {
        st->res_num2 = tot[0];
        st->res_den2 = tot[1];
    }
};

template <int SIGN, int BLOCK, int MINB, class Lk, class Epi>
__global__ void __launch_bounds__(BLOCK, MINB) k_hop(Geom g, Lk U, int par, SpinorF64 in, Epi epi, RedBuf red) {
    extern __shared__ double2 stage[];  // Epi::NPRE x 12 x BLOCK
    if (epi.skip()) return;
    const int i = blockIdx.x * BLOCK + threadIdx.x;
    double v[Epi::NRED > 0 ? Epi::NRED : 1];
#pragma unroll
    for (int k = 0; k < (Epi::NRED > 0 ? Epi::NRED : 1); k++) v[k] = 0.0;
    if (i < g.Vh) {
        if constexpr (Epi::NPRE > 0) {
#pragma unroll
            for (int k = 0; k < Epi::NPRE; k++) {
                const SpinorF64 f = epi.pre(k);
#pragma unroll
                for (int c = 0; c < 12; c++)
                    cp_async16(stage + ((size_t)k * 12 + c) * BLOCK + threadIdx.x, f.p + (size_t)c * f.stride + i);
            }
        }
        Spinor<double> acc;
        hop_site<SIGN>(g, par, i, in, U, acc);
        if constexpr (Epi::NPRE > 0) {
            cp_async_wait_all();  // this thread's own copies: no block barrier needed
            epi(i, acc, v, stage, BLOCK);
        } else {
            epi(i, acc, v);
        }
    }
    if constexpr (Epi::NRED > 0) grid_reduce<Epi::NRED, BLOCK>(v, red.partials, red.ticket, epi);
}

// shared memory of the staged epilogue operands.  Near the 48 KB default the kernel is
// opted in to more, once per instantiation and device (the attribute belongs to the
// device that is current when it is set; contexts on several GPUs share one process).
// If the opt-in fails the launch itself reports the error.
template <int SIGN, int BLOCK, int MINB, class Lk, class Epi>
size_t hop_smem() {
    constexpr size_t bytes = (size_t)Epi::NPRE * 12 * BLOCK * sizeof(double2);
    if constexpr (bytes > 32 * 1024) {
        static std::mutex mu;
        static unsigned long long done = 0;  // bit d: set on device d
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) {
            std::lock_guard<std::mutex> lk(mu);
            if (!((done >> dev) & 1ull) &&
                cudaFuncSetAttribute(k_hop<SIGN, BLOCK, MINB, Lk, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bytes) == cudaSuccess)
                done |= 1ull << dev;
        }
    }
    return bytes;
}

template <int BLOCK, int MINB, class Lk, class Epi>
void launch_variant(const Geom &g, const Lk &L, int par, int sign, SpinorF64 sin, const Epi &epi, RedBuf rb,
                    cudaStream_t s) {
    dim3 grid((g.Vh + BLOCK - 1) / BLOCK);
    if (sign > 0)
        k_hop<1, BLOCK, MINB><<<grid, BLOCK, hop_smem<1, BLOCK, MINB, Lk, Epi>(), s>>>(g, L, par, sin, epi, rb);
    else
        k_hop<-1, BLOCK, MINB><<<grid, BLOCK, hop_smem<-1, BLOCK, MINB, Lk, Epi>(), s>>>(g, L, par, sin, epi, rb);
}

// Launch shapes the autotuner chooses from (HopVariant in kernels.h):
//   0: 128 threads, registers unconstrained   1: 128 threads, <= 128 registers (4 blocks/SM)
//   2: 256 threads, <= 128 registers
// (128 threads at <= 102 registers spills about 600 bytes per thread and measured 0.63 of
// HBM peak against 0.80-0.83 for these.)
template <class Lk, class Epi>
void launch_shape(const Geom &g, const Lk &L, int par, int sign, SpinorF64 sin, const Epi &epi, RedBuf rb,
                  cudaStream_t s) {
    switch (g.hop_variant) {
    case 1:
        launch_variant<128, 4>(g, L, par, sign, sin, epi, rb, s);
        break;
    case 2:
        launch_variant<256, 2>(g, L, par, sign, sin, epi, rb, s);
        break;
    default:
        launch_variant<128, 1>(g, L, par, sign, sin, epi, rb, s);
        break;
    }
}

template <class Epi>
void dispatch_hop(const Geom &g, const GaugeF64 &U, int par, int sign, HalfF64 in, const Epi &epi, const RedBuf *red,
                  cudaStream_t s) {
    RedBuf rb = red ? *red : RedBuf{nullptr, nullptr};
    SpinorF64 sin{in.p, in.stride};
    if (U.planes == 9)
        launch_shape(g, LinksF64x18{U.p, U.stride}, par, sign, sin, epi, rb, s);
    else
        launch_shape(g, LinksF64x12{U.p, U.stride}, par, sign, sin, epi, rb, s);
}

// ------------------------------------------------------------------ vectors

constexpr int kVecBlock = 256;

struct FinCgInit {
    CgState *st;
    double acc2;
    int maxiter;
    __device__ void operator()(const double *tot) {
        st->rr = tot[0];
        st->src_norm2 = tot[1];
        st->target_rr = acc2 * tot[1];
        st->iter = 0;
        st->maxiter = maxiter;
        st->alpha = st->beta = 0.0;
        st->do_pupdate = 0;
        if (!isfinite(tot[0]) || !isfinite(tot[1]))
            st->status = CG_BREAKDOWN;
        else if (tot[1] == 0.0 || tot[0] < st->target_rr)
            st->status = CG_CONVERGED;
        else
            st->status = CG_RUNNING;
    }
};

__global__ void __launch_bounds__(kVecBlock) k_cg_init(int Vh, SpinorF64 src, SpinorF64 Ax, int have_ax, SpinorF64 r,
                                                       SpinorF64 p, FinCgInit fin, RedBuf red) {
    const int i = blockIdx.x * kVecBlock + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < Vh) {
        Spinor<double> b, a;
        src.load_cached(i, b);
        if (have_ax) Ax.load_cached(i, a);
#pragma unroll
        for (int c = 0; c < 12; c++) {
            const int s = c / 3, k = c % 3;
            v[1] += norm2(b.s[s][k]);
            if (have_ax) b.s[s][k] = b.s[s][k] - a.s[s][k];
            v[0] += norm2(b.s[s][k]);
        }
        r.store(i, b);
        p.store(i, b);
    }
    grid_reduce<2, kVecBlock>(v, red.partials, red.ticket, fin);
}

__global__ void __launch_bounds__(kVecBlock) k_cg_pupdate(int Vh, SpinorF64 r, SpinorF64 p, const CgState *st) {
    if (!st->do_pupdate) return;
    const int i = blockIdx.x * kVecBlock + threadIdx.x;
    if (i >= Vh) return;
    const double beta = st->beta;
#pragma unroll
    for (int c = 0; c < 12; c++) {
        double2 rv = r.p[(size_t)c * r.stride + i];
        double2 pv = p.p[(size_t)c * p.stride + i];
        p.p[(size_t)c * p.stride + i] = make_double2(fma(beta, pv.x, rv.x), fma(beta, pv.y, rv.y));
    }
}

// Last node of every CG loop-body iteration: keeps the graph's while loop
// going only while the solve is running.  It always runs, so the loop ends
// even when every other body kernel returned early; the iteration counter is
// bounded by maxiter, so the loop is bounded.
__global__ void k_loop_control(CgState *st, cudaGraphConditionalHandle cond, int use_cond) {
    st->do_pupdate = 0;
    if (st->status == CG_RUNNING && st->iter >= st->maxiter) st->status = CG_MAXITER;
    if (use_cond) cudaGraphSetConditional(cond, st->status == CG_RUNNING ? 1u : 0u);
}

__global__ void __launch_bounds__(kVecBlock) k_scale(int Vh, SpinorF64 x, SpinorF64 y, double a) {
    const int i = blockIdx.x * kVecBlock + threadIdx.x;
    if (i >= Vh) return;
#pragma unroll
    for (int c = 0; c < 12; c++) {
        double2 v = x.p[(size_t)c * x.stride + i];
        y.p[(size_t)c * y.stride + i] = make_double2(a * v.x, a * v.y);
    }
}

// ------------------------------------------------------------------ layout

// lexicographic AoS [V][4][3] complex -> even-odd SoA half lattice of parity par
__global__ void k_spinor_lex_to_eo(Geom g, const double2 *lex, int par, SpinorF64 out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.Vh) return;
    const int xh = i % g.lxh;
    int r = i / g.lxh;
    const int y = r % g.L[1];
    r /= g.L[1];
    const int z = r % g.L[2];
    const int t = r / g.L[2];
    const int x = 2 * xh + ((y + z + t + par) & 1);
    const size_t lexi = x + (size_t)g.L[0] * (y + (size_t)g.L[1] * (z + (size_t)g.L[2] * t));
#pragma unroll
    for (int c = 0; c < 12; c++) out.p[(size_t)c * out.stride + i] = lex[lexi * 12 + c];
}

__global__ void k_spinor_eo_to_lex(Geom g, SpinorF64 in, int par, double2 *lex) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.Vh) return;
    const int xh = i % g.lxh;
    int r = i / g.lxh;
    const int y = r % g.L[1];
    r /= g.L[1];
    const int z = r % g.L[2];
    const int t = r / g.L[2];
    const int x = 2 * xh + ((y + z + t + par) & 1);
    const size_t lexi = x + (size_t)g.L[0] * (y + (size_t)g.L[1] * (z + (size_t)g.L[2] * t));
#pragma unroll
    for (int c = 0; c < 12; c++) lex[lexi * 12 + c] = in.p[(size_t)c * in.stride + i];
}

// links of one direction, [V][3][3] complex lexicographic -> the `nplanes`
// planes of (par, dir): dst[k*stride + i]
__global__ void k_links_lex_to_eo(Geom g, const double2 *lex_dir, double2 *dst, int nplanes, int stride, int par) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.Vh) return;
    const int xh = i % g.lxh;
    int r = i / g.lxh;
    const int y = r % g.L[1];
    r /= g.L[1];
    const int z = r % g.L[2];
    const int t = r / g.L[2];
    const int x = 2 * xh + ((y + z + t + par) & 1);
    const size_t lexi = x + (size_t)g.L[0] * (y + (size_t)g.L[1] * (z + (size_t)g.L[2] * t));
    const double2 *src = lex_dir + lexi * 9;
    for (int k = 0; k < nplanes; k++) dst[(size_t)k * stride + i] = src[k];
}

// checkerboard-ordered AoS [Vh][12] complex <-> SoA planes of one parity
__global__ void k_aos_to_soa(int n, const double2 *aos, SpinorF64 out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < 12; c++) out.p[(size_t)c * out.stride + i] = aos[(size_t)i * 12 + c];
}
__global__ void k_soa_to_aos(int n, SpinorF64 in, double2 *aos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int c = 0; c < 12; c++) aos[(size_t)i * 12 + c] = in.p[(size_t)c * in.stride + i];
}

}  // namespace

void launch_aos_to_soa(int n, const double *aos, HalfF64 out, cudaStream_t s) {
    k_aos_to_soa<<<(n + 255) / 256, 256, 0, s>>>(n, reinterpret_cast<const double2 *>(aos), sp(out));
}
void launch_soa_to_aos(int n, HalfF64 in, double *aos, cudaStream_t s) {
    k_soa_to_aos<<<(n + 255) / 256, 256, 0, s>>>(n, sp(in), reinterpret_cast<double2 *>(aos));
}

// ------------------------------------------------------------------ launchers

void launch_hop_scale(const Geom &g, const GaugeF64 &U, int par, int sign, HalfF64 in, HalfF64 out, double a,
                      const CgState *st, cudaStream_t s) {
    EpiScale e{sp(out), a, st};
    dispatch_hop(g, U, par, sign, in, e, nullptr, s);
}

void launch_hop_xpay(const Geom &g, const GaugeF64 &U, int par, int sign, HalfF64 in, HalfF64 x, HalfF64 out,
                     double b, CgState *st, const RedBuf *red, cudaStream_t s, double d, double2 *zero) {
    if (red) {
        EpiXpay<true> e{sp(x), sp(out), b, st, d, zero};
        dispatch_hop(g, U, par, sign, in, e, red, s);
    } else {
        EpiXpay<false> e{sp(x), sp(out), b, st, d, zero};
        dispatch_hop(g, U, par, sign, in, e, nullptr, s);
    }
}

void launch_hop_cg_update(const Geom &g, const GaugeF64 &U, int par, int sign, HalfF64 t, HalfF64 Dp, HalfF64 r,
                          HalfF64 x, HalfF64 p, double b, CgState *st, const RedBuf &red,
                          cudaStream_t s, double d) {
    EpiCgUpdate e{sp(Dp), sp(r), sp(x), sp(p), b, st, d};
    dispatch_hop(g, U, par, sign, t, e, &red, s);
}

void launch_hop_residual(const Geom &g, const GaugeF64 &U, int par, int sign, HalfF64 t, HalfF64 x, HalfF64 src,
                         HalfF64 res, double b, CgState *st, const RedBuf &red, cudaStream_t s, double d) {
    EpiResidual e{sp(x), sp(src), sp(res), b, st, d};
    dispatch_hop(g, U, par, sign, t, e, &red, s);
}

void launch_cg_init(int Vh, HalfF64 src, HalfF64 Ax, HalfF64 r, HalfF64 p, double acc2, int maxiter, CgState *st,
                    const RedBuf &red, cudaStream_t s) {
    FinCgInit fin{st, acc2, maxiter};
    k_cg_init<<<(Vh + kVecBlock - 1) / kVecBlock, kVecBlock, 0, s>>>(Vh, sp(src), sp(Ax), Ax.p != nullptr, sp(r),
                                                                      sp(p), fin, red);
}

void launch_cg_pupdate(int Vh, HalfF64 r, HalfF64 p, const CgState *st, cudaStream_t s) {
    k_cg_pupdate<<<(Vh + kVecBlock - 1) / kVecBlock, kVecBlock, 0, s>>>(Vh, sp(r), sp(p), st);
}

void launch_loop_control(CgState *st, cudaGraphConditionalHandle cond, int use_cond, cudaStream_t s) {
    k_loop_control<<<1, 1, 0, s>>>(st, cond, use_cond);
}

void launch_scale(int Vh, HalfF64 x, HalfF64 y, double a, cudaStream_t s) {
    k_scale<<<(Vh + kVecBlock - 1) / kVecBlock, kVecBlock, 0, s>>>(Vh, sp(x), sp(y), a);
}

void launch_spinor_lex_to_eo(const Geom &g, const double *lex, int par, HalfF64 out, cudaStream_t s) {
    k_spinor_lex_to_eo<<<(g.Vh + 255) / 256, 256, 0, s>>>(g, reinterpret_cast<const double2 *>(lex), par, sp(out));
}

void launch_spinor_eo_to_lex(const Geom &g, HalfF64 in, int par, double *lex, cudaStream_t s) {
    k_spinor_eo_to_lex<<<(g.Vh + 255) / 256, 256, 0, s>>>(g, sp(in), par, reinterpret_cast<double2 *>(lex));
}

void launch_links_lex_to_eo(const Geom &g, const double *lex_dir, double2 *dst, int nplanes, int stride, int par,
                            cudaStream_t s) {
    k_links_lex_to_eo<<<(g.Vh + 255) / 256, 256, 0, s>>>(g, reinterpret_cast<const double2 *>(lex_dir), dst, nplanes,
                                                        stride, par);
}

}  // namespace hw
