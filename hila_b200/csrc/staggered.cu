// Staggered fermions (libraries/dirac/staggered.h): colour-vector fields, the
// even-odd operator, its force, and CG on its normal equations, all in FP64.
//
//   eta_d(x)  = ((sum_{d' < d} x_d') % 2) * 2 - 1      (staggered.h:14-28 as coded; its
//                                                       comment states the opposite sign)
//   hop_s v(x) = 0.5 s sum_d eta_d(x) [U_d(x) v(x+d) - U_d(x-d)^dag v(x-d)]   (:48-68)
//   M_s in    : out_o = (1/m) hop_s in_e ;  out_e = m in_e + hop_s out_o       (:224-242)
// with the fermion boundary sign on values gathered across the t boundary.
// out_o keeps (1/m) D_oe in_e, as the reference leaves it.  Fields are two
// half lattices of 3 double2 planes (stride = the lattice's padded parity size).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "hw_internal.h"
#include "reduce.cuh"
#include "staggered_math.cuh"
#include "storage.cuh"


namespace hw {
namespace {

constexpr int kStagBlock = 128;
constexpr int kStagVecBlock = 256;
constexpr int kStagMaxBlocks = 1024;

HalfStag half_of(const hw_stag_field *f, int p) {
    return HalfStag{f->half[p].as<double2>(), f->lat->stride};
}

// out = a * 0.5 SIGN acc  (x null)   or   out = m x + 0.5 SIGN acc
template <int SIGN, class Lk>
__global__ void __launch_bounds__(kStagBlock) k_stag_hop(Geom g, Lk U, int par, HalfStag in, HalfStag x, double m,
                                                          double a, HalfStag out) {
    const int i = blockIdx.x * kStagBlock + threadIdx.x;
    if (i >= g.Vh) return;
    Cx<double> acc[3];
    stag_hop_site(g, U, par, i, in, acc);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const Cx<double> h = (0.5 * SIGN) * acc[k];
        out.st(k, i, x.p ? m * x.ld(k, i) + h : a * h);
    }
}

template <class Lk>
void stag_hop(const Geom &g, const Lk &U, int par, int sign, HalfStag in, HalfStag x, double m, double a,
              HalfStag out, cudaStream_t s) {
    const int blocks = (int)((g.Vh + kStagBlock - 1) / kStagBlock);
    if (sign > 0)
        k_stag_hop<1><<<blocks, kStagBlock, 0, s>>>(g, U, par, in, x, m, a, out);
    else
        k_stag_hop<-1><<<blocks, kStagBlock, 0, s>>>(g, U, par, in, x, m, a, out);
}

// hop over both link formats
void stag_hop_any(const hw_gauge *G, int par, int sign, HalfStag in, HalfStag x, double m, double a, HalfStag out,
                  cudaStream_t s) {
    const GaugeF64 U = G->U();
    const Geom &g = G->lat->g;
    if (U.planes == 9)
        stag_hop(g, LinksF64x18{U.p, U.stride}, par, sign, in, x, m, a, out, s);
    else
        stag_hop(g, LinksF64x12{U.p, U.stride}, par, sign, in, x, m, a, out, s);
}

// M_s: out_o = (1/m) hop in_e ; out_e = m in_e + hop out_o
void stag_eo_apply(const hw_gauge *G, double mass, HalfStag in_e, HalfStag out_e, HalfStag out_o, int sign,
                   cudaStream_t s) {
    stag_hop_any(G, 1, sign, in_e, HalfStag{nullptr, 0}, 0.0, 1.0 / mass, out_o, s);
    stag_hop_any(G, 0, sign, out_o, in_e, mass, 0.0, out_e, s);
}

// ---- layout: host lexicographic [V][3] complex <-> half lattices
__global__ void k_stag_layout(Geom g, int par, double2 *lex, HalfStag f, int to_eo) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.Vh) return;
    int c[4];
    site_coords(g, i, par, c);
    const size_t s = c[0] + (size_t)g.L[0] * (c[1] + (size_t)g.L[1] * (c[2] + (size_t)g.L[2] * c[3]));
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (to_eo)
            f.p[(size_t)k * f.stride + i] = lex[s * 3 + k];
        else
            lex[s * 3 + k] = f.p[(size_t)k * f.stride + i];
    }
}

// ---- vector operations on EVEN halves (deterministic partial sums, summed on the host in order)
__global__ void __launch_bounds__(kStagVecBlock) k_stag_dot(int Vh, HalfStag a, HalfStag b, double *partials) {
    __shared__ double smem[kStagVecBlock / 32];
    double s = 0.0;
    for (int i = blockIdx.x * kStagVecBlock + threadIdx.x; i < Vh; i += gridDim.x * kStagVecBlock)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double2 u = a.p[(size_t)k * a.stride + i], v = b.p[(size_t)k * b.stride + i];
            s += u.x * v.x + u.y * v.y;
        }
    const double t = block_sum<kStagVecBlock>(s, smem);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// y = a x + b y (x may alias nothing; b = 1 gives axpy)
__global__ void __launch_bounds__(kStagVecBlock) k_stag_axpby(int Vh, double a, HalfStag x, double b, HalfStag y) {
    for (int i = blockIdx.x * kStagVecBlock + threadIdx.x; i < Vh; i += gridDim.x * kStagVecBlock)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double2 u = x.p[(size_t)k * x.stride + i];
            double2 &v = y.p[(size_t)k * y.stride + i];
            v = make_double2(a * u.x + b * v.x, a * u.y + b * v.y);
        }
}

struct StagVec {
    hw_context *ctx;
    int Vh, blocks;
    DevBuf partials;
    std::vector<double> host;
    int init(hw_lattice *lat) {
        ctx = lat->ctx;
        Vh = (int)lat->Vh;
        blocks = (int)std::min<long>((lat->Vh + kStagVecBlock - 1) / kStagVecBlock, kStagMaxBlocks);
        host.resize(blocks);
        return partials.alloc(sizeof(double) * blocks);
    }
    // Re <a, b> over EVEN
    int dot(HalfStag a, HalfStag b, double *out) {
        k_stag_dot<<<blocks, kStagVecBlock, 0, ctx->stream>>>(Vh, a, b, partials.as<double>());
        HW_CUDA(cudaGetLastError());
        HW_CUDA(cudaMemcpyAsync(host.data(), partials.ptr, sizeof(double) * blocks, cudaMemcpyDeviceToHost,
                                ctx->stream));
        HW_CUDA(cudaStreamSynchronize(ctx->stream));
        double s = 0.0;
        for (int k = 0; k < blocks; k++) s += host[k];
        *out = s;
        return HW_OK;
    }
    int axpby(double a, HalfStag x, double b, HalfStag y) {
        k_stag_axpby<<<blocks, kStagVecBlock, 0, ctx->stream>>>(Vh, a, x, b, y);
        HW_CUDA(cudaGetLastError());
        return HW_OK;
    }
};

// ---- force (staggered.h:70-86, 246-265); t1 = (1/m) hop_{-s} chi, t2 = (1/m) hop_s psi on ODD
//   x even: F_d = -s/2 eta_d t1(x+d) (x) psi(x) + s/2 eta_d t2(x+d) (x) chi(x)
//   x odd:  F_d =  s/2 eta_d psi(x+d) (x) t1(x) - s/2 eta_d chi(x+d) (x) t2(x)
// (eta_d(x+d) = eta_d(x): it depends on the coordinates below d only)
template <int SIGN>
__global__ void __launch_bounds__(kStagBlock) k_stag_force(Geom g, HalfStag chi, HalfStag psi, HalfStag t1,
                                                            HalfStag t2, long V, double2 *out) {
    const int par = blockIdx.y;
    const int i = blockIdx.x * kStagBlock + threadIdx.x;
    if (i >= g.Vh) return;
    const SiteNbrs n = site_neighbours(g, i, par);
    int c[4];
    site_coords(g, i, par, c);
    const long lex = c[0] + (long)g.L[0] * (c[1] + (long)g.L[1] * (c[2] + (long)g.L[2] * c[3]));
    const HalfStag &A1 = par == 0 ? t1 : psi, &B1 = par == 0 ? psi : t1;
    const HalfStag &A2 = par == 0 ? t2 : chi, &B2 = par == 0 ? chi : t2;
    const double f1 = par == 0 ? -0.5 * SIGN : 0.5 * SIGN, f2 = -f1;
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const int y = n.fwd[d];
        const double e = (d == 3 && n.tfwd_wrap) ? -stag_eta(c, d) : stag_eta(c, d);
        double2 *o = out + ((size_t)d * V + lex) * 9;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const Cx<double> a1 = A1.ld(a, y), a2 = A2.ld(a, y);
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const Cx<double> v = (f1 * e) * cmul(a1, conj(B1.ld(b, i))) + (f2 * e) * cmul(a2, conj(B2.ld(b, i)));
                o[a * 3 + b] = make_double2(v.re, v.im);
            }
        }
    }
}

}  // namespace
}  // namespace hw

using namespace hw;

namespace {

int check_stag_op(const hw_gauge *G, const hw_stag_field *a, const hw_stag_field *b, double mass) {
    HW_CHECK_ARG(G && a && b, "null argument");
    HW_CHECK_ARG(a->lat == G->lat && b->lat == G->lat, "fields and gauge live on different lattices");
    HW_CHECK_ARG(std::isfinite(mass) && mass != 0.0, "mass must be finite and non-zero");
    return HW_OK;
}

int stag_apply(const hw_gauge *G, double mass, const hw_stag_field *in, hw_stag_field *out, int sign) {
    int rc = check_stag_op(G, in, out, mass);
    if (rc != HW_OK) return rc;
    HW_CHECK_ARG(in != out, "in and out must be different fields");
    hw_context *ctx = G->lat->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    stag_eo_apply(G, mass, half_of(in, 0), half_of(out, 0), half_of(out, 1), sign, ctx->stream);
    HW_CUDA(cudaGetLastError());
    return HW_OK;
}

}  // namespace

extern "C" {

int hw_stag_field_create(hw_lattice *lat, hw_stag_field **out) {
    HW_CHECK_ARG(lat && out, "null argument");
    *out = nullptr;
    std::lock_guard<std::recursive_mutex> lk(lat->ctx->mu);
    HW_CUDA(cudaSetDevice(lat->ctx->device));
    std::unique_ptr<hw_stag_field> f(new hw_stag_field());
    f->lat = lat;
    for (int p = 0; p < 2; p++) {
        int rc = f->half[p].alloc((size_t)3 * lat->stride * sizeof(double2));
        if (rc != HW_OK) return rc;
        HW_CUDA(cudaMemsetAsync(f->half[p].ptr, 0, f->half[p].bytes, lat->ctx->stream));
    }
    HW_CUDA(cudaStreamSynchronize(lat->ctx->stream));
    *out = f.release();
    return HW_OK;
}

int hw_stag_field_destroy(hw_stag_field *f) {
    if (!f) return HW_OK;
    {
        std::lock_guard<std::recursive_mutex> lk(f->lat->ctx->mu);
        cudaSetDevice(f->lat->ctx->device);
        for (auto &h : f->half) h.release();
    }
    delete f;
    return HW_OK;
}

int hw_stag_field_upload(hw_stag_field *f, const double *host, int parity) {
    HW_CHECK_ARG(f && host, "null argument");
    HW_CHECK_ARG(parity >= 1 && parity <= 3, "parity must be HW_EVEN, HW_ODD or HW_ALL");
    hw_lattice *lat = f->lat;
    hw_context *ctx = lat->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    const size_t bytes = (size_t)lat->V * 6 * sizeof(double);
    int rc;
    if ((rc = ensure_stage(ctx, bytes)) != HW_OK) return rc;
    HW_CUDA(cudaMemcpyAsync(ctx->stage.ptr, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    for (int p = 0; p < 2; p++)
        if (parity & (1 << p))
            k_stag_layout<<<(unsigned)((lat->Vh + 255) / 256), 256, 0, ctx->stream>>>(
                lat->g, p, ctx->stage.as<double2>(), half_of(f, p), 1);
    HW_CUDA(cudaGetLastError());
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return HW_OK;
}

int hw_stag_field_download(const hw_stag_field *f, double *host, int parity) {
    HW_CHECK_ARG(f && host, "null argument");
    HW_CHECK_ARG(parity >= 1 && parity <= 3, "parity must be HW_EVEN, HW_ODD or HW_ALL");
    hw_lattice *lat = f->lat;
    hw_context *ctx = lat->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    const size_t bytes = (size_t)lat->V * 6 * sizeof(double);
    int rc;
    if ((rc = ensure_stage(ctx, bytes)) != HW_OK) return rc;
    // sites of the other parity come back as zero
    HW_CUDA(cudaMemsetAsync(ctx->stage.ptr, 0, bytes, ctx->stream));
    for (int p = 0; p < 2; p++)
        if (parity & (1 << p))
            k_stag_layout<<<(unsigned)((lat->Vh + 255) / 256), 256, 0, ctx->stream>>>(
                lat->g, p, ctx->stage.as<double2>(), half_of(f, p), 0);
    HW_CUDA(cudaGetLastError());
    HW_CUDA(cudaMemcpyAsync(host, ctx->stage.ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return HW_OK;
}

int hw_stag_field_zero(hw_stag_field *f, int parity) {
    HW_CHECK_ARG(f, "null argument");
    HW_CHECK_ARG(parity >= 1 && parity <= 3, "parity must be HW_EVEN, HW_ODD or HW_ALL");
    hw_context *ctx = f->lat->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    for (int p = 0; p < 2; p++)
        if (parity & (1 << p)) HW_CUDA(cudaMemsetAsync(f->half[p].ptr, 0, f->half[p].bytes, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return HW_OK;
}

int hw_staggered_evenodd_apply(const hw_gauge *gauge, double mass, const hw_stag_field *in, hw_stag_field *out) {
    return stag_apply(gauge, mass, in, out, +1);
}

int hw_staggered_evenodd_dagger(const hw_gauge *gauge, double mass, const hw_stag_field *in, hw_stag_field *out) {
    return stag_apply(gauge, mass, in, out, -1);
}

int hw_staggered_evenodd_force(const hw_gauge *gauge, double mass, const hw_stag_field *chi, const hw_stag_field *psi,
                               int sign, double *force) {
    int rc = check_stag_op(gauge, chi, psi, mass);
    if (rc != HW_OK) return rc;
    HW_CHECK_ARG(force, "null argument");
    HW_CHECK_ARG(sign == 1 || sign == -1, "sign must be +1 or -1");
    hw_lattice *lat = gauge->lat;
    hw_context *ctx = lat->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    const int stride = lat->stride;
    DevBuf t1, t2, out;
    if ((rc = t1.alloc((size_t)3 * stride * sizeof(double2))) != HW_OK) return rc;
    if ((rc = t2.alloc((size_t)3 * stride * sizeof(double2))) != HW_OK) return rc;
    if ((rc = out.alloc((size_t)36 * lat->V * sizeof(double2))) != HW_OK) return rc;
    const HalfStag h1{t1.as<double2>(), stride}, h2{t2.as<double2>(), stride}, none{nullptr, 0};
    stag_hop_any(gauge, 1, -sign, half_of(chi, 0), none, 0.0, 1.0 / mass, h1, ctx->stream);
    stag_hop_any(gauge, 1, sign, half_of(psi, 0), none, 0.0, 1.0 / mass, h2, ctx->stream);
    dim3 grid((unsigned)((lat->Vh + kStagBlock - 1) / kStagBlock), 2);
    if (sign > 0)
        k_stag_force<1><<<grid, kStagBlock, 0, ctx->stream>>>(lat->g, half_of(chi, 0), half_of(psi, 0), h1, h2,
                                                              lat->V, out.as<double2>());
    else
        k_stag_force<-1><<<grid, kStagBlock, 0, ctx->stream>>>(lat->g, half_of(chi, 0), half_of(psi, 0), h1, h2,
                                                               lat->V, out.as<double2>());
    HW_CUDA(cudaGetLastError());
    HW_CUDA(cudaMemcpyAsync(force, out.ptr, out.bytes, cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return HW_OK;
}

// CG<dirac_staggered_evenodd>::apply (conjugate_gradient.h:46-104): M^dag M out = in
// on EVEN, out the initial guess; stops when |r|^2 < accuracy^2 |in|^2 (with
// true_residual set, also on the recomputed |in - M^dag M out|).  FP64, host loop.
int hw_staggered_cg_solve(const hw_gauge *gauge, double mass, const hw_stag_field *in, hw_stag_field *out,
                          const hw_cg_params *params, hw_cg_result *result) {
    int rc = check_stag_op(gauge, in, out, mass);
    if (rc != HW_OK) return rc;
    HW_CHECK_ARG(in != out, "in and out must be different fields");
    hw_cg_params P;
    hw_cg_params_default(&P);
    if (params) P = *params;
    HW_CHECK_ARG(P.accuracy > 0 && P.maxiters > 0, "bad accuracy or maxiters");
    HW_CHECK_ARG(P.precision == HW_PREC_F64, "staggered solves run in FP64");
    hw_lattice *lat = gauge->lat;
    hw_context *ctx = lat->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    const int stride = lat->stride;
    const size_t hb = (size_t)3 * stride * sizeof(double2);
    DevBuf br, bp, bAp, be, bo;
    for (DevBuf *d : {&br, &bp, &bAp, &be, &bo})
        if ((rc = d->alloc(hb)) != HW_OK) return rc;
    const HalfStag r{br.as<double2>(), stride}, p{bp.as<double2>(), stride}, Ap{bAp.as<double2>(), stride};
    const HalfStag te{be.as<double2>(), stride}, to{bo.as<double2>(), stride};
    const HalfStag b = half_of(in, 0), x = half_of(out, 0);
    StagVec V;
    if ((rc = V.init(lat)) != HW_OK) return rc;
    cudaStream_t s = ctx->stream;
    auto A = [&](HalfStag v, HalfStag w) {  // w = M^dag M v
        stag_eo_apply(gauge, mass, v, te, to, +1, s);
        stag_eo_apply(gauge, mass, te, w, to, -1, s);
    };
    HW_CUDA(cudaEventRecord(ctx->ev0, s));
    // r = b - A x ; p = r
    A(x, Ap);
    HW_CUDA(cudaMemcpyAsync(r.p, b.p, hb, cudaMemcpyDeviceToDevice, s));
    if ((rc = V.axpby(-1.0, Ap, 1.0, r)) != HW_OK) return rc;
    HW_CUDA(cudaMemcpyAsync(p.p, r.p, hb, cudaMemcpyDeviceToDevice, s));
    double bb, rr;
    if ((rc = V.dot(b, b, &bb)) != HW_OK) return rc;
    if ((rc = V.dot(r, r, &rr)) != HW_OK) return rc;
    const double target = P.accuracy * P.accuracy * bb;
    int it = 0, status = HW_OK;
    long launches = 4 + 2;
    while (rr >= target && bb > 0) {
        if (it >= P.maxiters) {
            status = HW_ERR_NOT_CONVERGED;
            break;
        }
        A(p, Ap);
        double pAp;
        if ((rc = V.dot(p, Ap, &pAp)) != HW_OK) return rc;
        if (!(pAp > 0.0) || !std::isfinite(pAp)) {
            status = HW_ERR_BREAKDOWN;
            break;
        }
        const double alpha = rr / pAp;
        if ((rc = V.axpby(alpha, p, 1.0, x)) != HW_OK) return rc;
        if ((rc = V.axpby(-alpha, Ap, 1.0, r)) != HW_OK) return rc;
        double rr_new;
        if ((rc = V.dot(r, r, &rr_new)) != HW_OK) return rc;
        const double beta = rr_new / rr;
        rr = rr_new;
        if ((rc = V.axpby(1.0, r, beta, p)) != HW_OK) return rc;
        it++;
        launches += 4 + 5;
    }
    // explicit residual |b - A x| / |b| in FP64
    A(x, Ap);
    HW_CUDA(cudaMemcpyAsync(r.p, b.p, hb, cudaMemcpyDeviceToDevice, s));
    if ((rc = V.axpby(-1.0, Ap, 1.0, r)) != HW_OK) return rc;
    double res2;
    if ((rc = V.dot(r, r, &res2)) != HW_OK) return rc;
    HW_CUDA(cudaMemsetAsync(out->half[1].ptr, 0, out->half[1].bytes, s));
    HW_CUDA(cudaEventRecord(ctx->ev1, s));
    HW_CUDA(cudaEventSynchronize(ctx->ev1));
    const double true_res = bb > 0 ? std::sqrt(res2 / bb) : 0.0;
    if (status == HW_OK && P.true_residual && true_res > P.accuracy) status = HW_ERR_NOT_CONVERGED;
    if (result) {
        std::memset(result, 0, sizeof(*result));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        result->status = status;
        result->iterations = it;
        result->rr_relative = bb > 0 ? rr / bb : 0.0;
        result->true_residual = true_res;
        result->seconds = ms * 1e-3;
        result->kernel_launches = (int)(launches + 6);
    }
    return status;
}

}  // extern "C"
