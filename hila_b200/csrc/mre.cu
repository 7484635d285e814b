// Initial guess for a solve from earlier solutions (MRE_guess, MRE_guess.h:9-88):
// the minimal-residual combination psi = sum_i c_i b_i of an orthogonalised basis
// b_i of the old solutions, with the real coefficients c solving the projected
// system  Re<b_j, A b_i> c_i = Re<b_j, chi>,  A = (M + m_h)^dag (M + m_h) (the
// normal operator of the solver; m_h = 0 for M itself).  Dots over EVEN sites,
// real part (WilsonVector::rdot), as in the reference.
//
// Differences from the reference text, which as written does not build this
// combination: its Gram-Schmidt step divides the overlap by |b_i|^2 instead of
// |b_j|^2 (MRE_guess.h:21-29), and its last loop assigns psi = b_i + v_i b_i
// for every i instead of accumulating psi += v_i b_i (MRE_guess.h:83-87).  Here
// both follow the method the function's comment names; the small system is
// solved by the reference's Gauss-Jordan elimination, including dropping a
// direction whose pivot is below 1e-16 (MRE_guess.h:55-80).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "hw_internal.h"
#include "reduce.cuh"

namespace hw {
namespace {

constexpr int kMreBlock = 256;
constexpr int kMreMaxBlocks = 1024;

// per-block partial of Re sum_i conj(a_i) b_i over EVEN sites (fixed grid-stride and tree order)
__global__ void __launch_bounds__(kMreBlock) k_rdot(int Vh, HalfF64 a, HalfF64 b, double *partials) {
    __shared__ double smem[kMreBlock / 32];
    double s = 0.0;
    for (int i = blockIdx.x * kMreBlock + threadIdx.x; i < Vh; i += gridDim.x * kMreBlock)
#pragma unroll
        for (int c = 0; c < 12; c++) {
            const double2 u = a.p[(size_t)c * a.stride + i], v = b.p[(size_t)c * b.stride + i];
            s += u.x * v.x + u.y * v.y;
        }
    const double t = block_sum<kMreBlock>(s, smem);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// y += a x over EVEN sites
__global__ void __launch_bounds__(kMreBlock) k_axpy(int Vh, double a, HalfF64 x, HalfF64 y) {
    for (int i = blockIdx.x * kMreBlock + threadIdx.x; i < Vh; i += gridDim.x * kMreBlock)
#pragma unroll
        for (int c = 0; c < 12; c++) {
            const double2 u = x.p[(size_t)c * x.stride + i];
            double2 &v = y.p[(size_t)c * y.stride + i];
            v = make_double2(v.x + a * u.x, v.y + a * u.y);
        }
}

struct Mre {
    hw_context *ctx;
    int Vh;
    int blocks;
    DevBuf partials;
    std::vector<double> host;

    int rdot(HalfF64 a, HalfF64 b, double *out) {
        k_rdot<<<blocks, kMreBlock, 0, ctx->stream>>>(Vh, a, b, partials.as<double>());
        HW_CUDA(cudaGetLastError());
        HW_CUDA(cudaMemcpyAsync(host.data(), partials.ptr, sizeof(double) * blocks, cudaMemcpyDeviceToHost,
                                ctx->stream));
        HW_CUDA(cudaStreamSynchronize(ctx->stream));
        double s = 0.0;
        for (int k = 0; k < blocks; k++) s += host[k];
        *out = s;
        return HW_OK;
    }
    int axpy(double a, HalfF64 x, HalfF64 y) {
        k_axpy<<<blocks, kMreBlock, 0, ctx->stream>>>(Vh, a, x, y);
        HW_CUDA(cudaGetLastError());
        return HW_OK;
    }
};

}  // namespace
}  // namespace hw

using namespace hw;

extern "C" int hw_mre_guess(const hw_gauge *gauge, double kappa, double mh, const hw_field *const *old, int n,
                            const hw_field *chi, hw_field *psi) {
    HW_CHECK_ARG(gauge && chi && psi && (n == 0 || old), "null argument");
    HW_CHECK_ARG(n >= 0 && n <= 64, "n must be 0..64");
    HW_CHECK_ARG(std::isfinite(mh), "mh must be finite");
    hw_lattice *lat = gauge->lat;
    HW_CHECK_ARG(chi->lat == lat && psi->lat == lat, "fields and gauge live on different lattices");
    for (int i = 0; i < n; i++) HW_CHECK_ARG(old[i] && old[i]->lat == lat, "old solution %d: null or other lattice", i);
    hw_context *ctx = lat->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    int rc;
    if ((rc = ensure_workspace(lat)) != HW_OK) return rc;
    if ((rc = tune_hop(lat, gauge)) != HW_OK) return rc;
    const int stride = lat->stride;
    const size_t half_bytes = (size_t)12 * stride * sizeof(double2);
    Mre m;
    m.ctx = ctx;
    m.Vh = (int)lat->Vh;
    m.blocks = (int)std::min<long>((lat->Vh + kMreBlock - 1) / kMreBlock, kMreMaxBlocks);
    m.host.resize(m.blocks);
    if ((rc = m.partials.alloc(sizeof(double) * m.blocks)) != HW_OK) return rc;
    std::vector<DevBuf> basis(n);
    DevBuf t1, t2;
    if ((rc = t1.alloc(half_bytes)) != HW_OK) return rc;
    if ((rc = t2.alloc(half_bytes)) != HW_OK) return rc;
    auto h = [stride](const DevBuf &b) { return HalfF64{b.as<double2>(), stride}; };
    // orthogonalised basis: b_i = old_i - sum_{j<i} (Re<b_j, b_i> / |b_j|^2) b_j
    std::vector<double> bb(n, 0.0);
    for (int i = 0; i < n; i++) {
        if ((rc = basis[i].alloc(half_bytes)) != HW_OK) return rc;
        HW_CUDA(cudaMemcpyAsync(basis[i].ptr, old[i]->half[0].buf.ptr, half_bytes, cudaMemcpyDeviceToDevice,
                                ctx->stream));
        for (int j = 0; j < i; j++) {
            if (!(bb[j] > 1e-300)) continue;
            double ov;
            if ((rc = m.rdot(h(basis[j]), h(basis[i]), &ov)) != HW_OK) return rc;
            if ((rc = m.axpy(-ov / bb[j], h(basis[j]), h(basis[i]))) != HW_OK) return rc;
        }
        if ((rc = m.rdot(h(basis[i]), h(basis[i]), &bb[i])) != HW_OK) return rc;
    }
    // projected system  M[j][i] = Re<b_j, A b_i>,  v[i] = Re<b_i, chi>
    const double d = 1.0 + mh;
    std::vector<double> Mm((size_t)n * n), v(n);
    for (int i = 0; i < n; i++) {
        eo_apply_half(gauge, kappa, h(basis[i]), h(t1), +1, d);
        eo_apply_half(gauge, kappa, h(t1), h(t2), -1, d);
        for (int j = 0; j < n; j++)
            if ((rc = m.rdot(h(basis[j]), h(t2), &Mm[(size_t)j * n + i])) != HW_OK) return rc;
        if ((rc = m.rdot(h(basis[i]), chi->half[0].h(), &v[i])) != HW_OK) return rc;
    }
    // Gauss-Jordan elimination (MRE_guess.h:55-80)
    for (int i = 0; i < n; i++) {
        double *Mi = &Mm[(size_t)i * n];
        if (Mi[i] * Mi[i] > 1e-32) {
            const double inv = 1.0 / Mi[i];
            for (int j = 0; j < n; j++) Mi[j] *= inv;
            v[i] *= inv;
            for (int k = 0; k < n; k++)
                if (k != i) {
                    double *Mk = &Mm[(size_t)k * n];
                    const double wgt = Mk[i];
                    for (int j = 0; j < n; j++) Mk[j] -= wgt * Mi[j];
                    v[k] -= wgt * v[i];
                }
        } else {
            v[i] = 0.0;
            for (int j = 0; j < n; j++) Mm[(size_t)j * n + i] = 0.0;
        }
    }
    // psi = sum_i v_i b_i on EVEN, 0 on ODD
    HW_CUDA(cudaMemsetAsync(psi->half[0].buf.ptr, 0, psi->half[0].buf.bytes, ctx->stream));
    HW_CUDA(cudaMemsetAsync(psi->half[1].buf.ptr, 0, psi->half[1].buf.bytes, ctx->stream));
    for (int i = 0; i < n; i++)
        if (std::isfinite(v[i]) && v[i] != 0.0)
            if ((rc = m.axpy(v[i], h(basis[i]), psi->half[0].h())) != HW_OK) return rc;
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return HW_OK;
}
