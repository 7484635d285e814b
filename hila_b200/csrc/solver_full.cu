// CG<Dirac_Wilson>::apply (libraries/dirac/conjugate_gradient.h:46-104 on the
// unpreconditioned operator of wilson.h:146-201): M^dag M out = in on ALL sites, FP64.
//
// The unpreconditioned operator is the reference's test operator (test_CG.cpp:127-182),
// not the production path, so this solver is a plain host loop over device kernels:
// the operator (two fused hop launches per application), and dot products and axpys
// over whole fields.  A field's two halves are contiguous plane arrays whose padding
// sites are never written, so the vector kernels run over the flat arrays.  Partial
// sums are added on the host in block order: the result does not depend on scheduling.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "hw_internal.h"
#include "reduce.cuh"

namespace hw {
namespace {

constexpr int kFlatBlock = 256;
constexpr int kFlatMaxBlocks = 1024;

// partials[block] = sum Re conj(a) b over the block's elements of both halves
__global__ void __launch_bounds__(kFlatBlock) k_flat_dot(long n, const double2 *a0, const double2 *b0,
                                                         const double2 *a1, const double2 *b1, double *partials) {
    __shared__ double smem[kFlatBlock / 32];
    double s = 0.0;
    for (long k = blockIdx.x * (long)kFlatBlock + threadIdx.x; k < n; k += (long)gridDim.x * kFlatBlock) {
        const double2 x0 = a0[k], y0 = b0[k], x1 = a1[k], y1 = b1[k];
        s += x0.x * y0.x + x0.y * y0.y + x1.x * y1.x + x1.y * y1.y;
    }
    const double t = block_sum<kFlatBlock>(s, smem);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// y = a x + b y over both halves
__global__ void __launch_bounds__(kFlatBlock) k_flat_axpby(long n, double a, const double2 *x0, const double2 *x1,
                                                           double b, double2 *y0, double2 *y1) {
    for (long k = blockIdx.x * (long)kFlatBlock + threadIdx.x; k < n; k += (long)gridDim.x * kFlatBlock) {
        const double2 u0 = x0[k], u1 = x1[k];
        double2 v0 = y0[k], v1 = y1[k];
        v0.x = a * u0.x + b * v0.x;
        v0.y = a * u0.y + b * v0.y;
        v1.x = a * u1.x + b * v1.x;
        v1.y = a * u1.y + b * v1.y;
        y0[k] = v0;
        y1[k] = v1;
    }
}

struct Full {  // the two halves of a Wilson field
    double2 *h[2];
};

class FullVec {
  public:
    int init(hw_lattice *lat) {
        ctx_ = lat->ctx;
        n_ = (long)12 * lat->stride;
        blocks_ = (int)std::min<long>((n_ + kFlatBlock - 1) / kFlatBlock, kFlatMaxBlocks);
        host_.resize(blocks_);
        return partials_.alloc(sizeof(double) * blocks_);
    }
    int dot(Full a, Full b, double *out) {
        k_flat_dot<<<blocks_, kFlatBlock, 0, ctx_->stream>>>(n_, a.h[0], b.h[0], a.h[1], b.h[1],
                                                              partials_.as<double>());
        HW_CUDA(cudaGetLastError());
        HW_CUDA(cudaMemcpyAsync(host_.data(), partials_.ptr, sizeof(double) * blocks_, cudaMemcpyDeviceToHost,
                                ctx_->stream));
        HW_CUDA(cudaStreamSynchronize(ctx_->stream));
        double s = 0.0;
        for (int k = 0; k < blocks_; k++) s += host_[k];
        *out = s;
        return HW_OK;
    }
    int axpby(double a, Full x, double b, Full y) {
        k_flat_axpby<<<blocks_, kFlatBlock, 0, ctx_->stream>>>(n_, a, x.h[0], x.h[1], b, y.h[0], y.h[1]);
        HW_CUDA(cudaGetLastError());
        return HW_OK;
    }
    int copy(Full src, Full dst) {
        for (int p = 0; p < 2; p++)
            HW_CUDA(cudaMemcpyAsync(dst.h[p], src.h[p], n_ * sizeof(double2), cudaMemcpyDeviceToDevice,
                                    ctx_->stream));
        return HW_OK;
    }

  private:
    hw_context *ctx_ = nullptr;
    long n_ = 0;
    int blocks_ = 1;
    DevBuf partials_;
    std::vector<double> host_;
};

Full full_of(const hw_field *f) { return Full{{f->half[0].buf.as<double2>(), f->half[1].buf.as<double2>()}}; }

}  // namespace
}  // namespace hw

using namespace hw;

extern "C" int hw_wilson_cg_solve(const hw_gauge *gauge, double kappa, const hw_field *in, hw_field *out,
                                  const hw_cg_params *params, hw_cg_result *result) {
    HW_CHECK_ARG(gauge && in && out, "null argument");
    HW_CHECK_ARG(in->lat == gauge->lat && out->lat == gauge->lat, "fields and gauge belong to different lattices");
    HW_CHECK_ARG(in != out, "in and out must be different fields");
    hw_cg_params P;
    hw_cg_params_default(&P);
    if (params) P = *params;
    HW_CHECK_ARG(P.accuracy > 0 && P.maxiters > 0, "bad accuracy or maxiters");
    HW_CHECK_ARG(P.precision == HW_PREC_F64, "the unpreconditioned solve runs in FP64");
    hw_lattice *lat = gauge->lat;
    hw_context *ctx = lat->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    int rc;
    // workspace fields r, p, A p and the intermediate M v
    hw_field *ws[4] = {nullptr, nullptr, nullptr, nullptr};
    auto release = [&]() {
        for (hw_field *f : ws) hw_field_destroy(f);
    };
    for (hw_field *&f : ws)
        if ((rc = hw_field_create(lat, &f)) != HW_OK) {
            release();
            return rc;
        }
    FullVec V;
    if ((rc = V.init(lat)) != HW_OK) {
        release();
        return rc;
    }
    const Full b = full_of(in), x = full_of(out), r = full_of(ws[0]), p = full_of(ws[1]), Ap = full_of(ws[2]);
    auto A = [&](const hw_field *v, hw_field *w) {  // w = M^dag M v
        int e = hw_wilson_apply(gauge, kappa, 1, v, ws[3]);
        return e != HW_OK ? e : hw_wilson_apply(gauge, kappa, -1, ws[3], w);
    };
    auto body = [&](hw_cg_result *R) -> int {
        cudaStream_t s = ctx->stream;
        HW_CUDA(cudaEventRecord(ctx->ev0, s));
        int e;
        // r = b - A x ; p = r   (conjugate_gradient.h:57-63)
        if ((e = A(out, ws[2])) != HW_OK) return e;
        if ((e = V.copy(b, r)) != HW_OK || (e = V.axpby(-1.0, Ap, 1.0, r)) != HW_OK || (e = V.copy(r, p)) != HW_OK)
            return e;
        double bb, rr;
        if ((e = V.dot(b, b, &bb)) != HW_OK || (e = V.dot(r, r, &rr)) != HW_OK) return e;
        const double target = P.accuracy * P.accuracy * bb;
        int it = 0, status = HW_OK;
        while (rr >= target && bb > 0) {
            if (it >= P.maxiters) {
                status = HW_ERR_NOT_CONVERGED;
                break;
            }
            if ((e = A(ws[1], ws[2])) != HW_OK) return e;
            double pAp;
            if ((e = V.dot(p, Ap, &pAp)) != HW_OK) return e;
            if (!(pAp > 0.0) || !std::isfinite(pAp)) {
                status = HW_ERR_BREAKDOWN;
                break;
            }
            const double alpha = rr / pAp;
            if ((e = V.axpby(alpha, p, 1.0, x)) != HW_OK || (e = V.axpby(-alpha, Ap, 1.0, r)) != HW_OK) return e;
            double rr_new;
            if ((e = V.dot(r, r, &rr_new)) != HW_OK) return e;
            const double beta = rr_new / rr;
            rr = rr_new;
            if ((e = V.axpby(1.0, r, beta, p)) != HW_OK) return e;
            it++;
        }
        // explicit residual |b - A x| / |b| in FP64
        if ((e = A(out, ws[2])) != HW_OK) return e;
        if ((e = V.copy(b, r)) != HW_OK || (e = V.axpby(-1.0, Ap, 1.0, r)) != HW_OK) return e;
        double res2;
        if ((e = V.dot(r, r, &res2)) != HW_OK) return e;
        HW_CUDA(cudaEventRecord(ctx->ev1, s));
        HW_CUDA(cudaEventSynchronize(ctx->ev1));
        const double true_res = bb > 0 ? std::sqrt(res2 / bb) : 0.0;
        if (status == HW_OK && P.true_residual && true_res > P.accuracy) status = HW_ERR_NOT_CONVERGED;
        std::memset(R, 0, sizeof(*R));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        R->status = status;
        R->iterations = it;
        R->rr_relative = bb > 0 ? rr / bb : 0.0;
        R->true_residual = true_res;
        R->seconds = ms * 1e-3;
        return status;
    };
    hw_cg_result tmp;
    rc = body(result ? result : &tmp);
    release();
    return rc;
}
