// Wilson fermion force of the even-odd operator (Dirac_Wilson_evenodd::force,
// wilson.h:293-311, with Dirac_Wilson_calc_force, wilson.h:110-137).
//
// With s the operator sign, t1 = -kappa H^{oe}_{-s} chi and t2 = -kappa H^{oe}_s psi
// (both ODD; hop_set with the diagonal inverse a no-op), the derivative of
// Re(chi^dag M_s psi) with respect to U_dir(X) is, for every positive dir,
//   X even:  F = kappa sg [ (1 - s g_dir) t1(X+dir) (x) psi(X) + (1 + s g_dir) t2(X+dir) (x) chi(X) ]
//   X odd:   F = kappa sg [ (1 + s g_dir) psi(X+dir) (x) t1(X) + (1 - s g_dir) chi(X+dir) (x) t2(X) ]
// where (a (x) b)_ij = sum_spin a_i conj(b_j) (matrix.h:1437-1448 summed over
// spin, wilson_vector.h:229-233), (1 +- s g_dir) v = E_{dir,+-s} P_{dir,+-s} v,
// and sg = -1 when X+dir crosses the antiperiodic t boundary.  One thread per
// site of both parities; the 4 x 9 complex entries of the site are written in
// the canonical lexicographic layout F[4][V][3][3].
#include <cuda_runtime.h>

#include "hw_internal.h"
#include "storage.cuh"

namespace hw {
namespace {

constexpr int kForceBlock = 128;

__device__ __forceinline__ void force_outer(const Spinor<double> &v, const Spinor<double> &b, Cx<double> f[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<double> acc = {0.0, 0.0};
#pragma unroll
            for (int sp = 0; sp < 4; sp++) acc = acc + cmul(v.s[sp][i], conj(b.s[sp][j]));
            f[i][j] = acc;
        }
}

// (1 + S g_DIR) w
template <int DIR, int S>
__device__ __forceinline__ Spinor<double> spin_proj(const Spinor<double> &w) {
    Cx<double> h0[3], h1[3];
    project<DIR, S>(w, h0, h1);
    Spinor<double> r;
#pragma unroll
    for (int c = 0; c < 12; c++) r.s[c / 3][c % 3] = {0.0, 0.0};
    expand_add<DIR, S>(r, h0, h1);
    return r;
}

// one direction: F = kappa sg [ (1 + S1 g) A(X+dir) (x) B(X) + (1 + S2 g) C(X+dir) (x) D(X) ]
template <int DIR, int S1, int S2>
__device__ __forceinline__ void force_dir(const SiteNbrs &nb, const SpinorF64 &A, const Spinor<double> &b,
                                          const SpinorF64 &C, const Spinor<double> &d, double kappa, long V,
                                          long lex, double2 *out) {
    const int y = nb.fwd[DIR];
    const double k = (DIR == 3 && nb.tfwd_wrap) ? -kappa : kappa;
    Spinor<double> a, c;
    A.load(y, a);
    C.load(y, c);
    Cx<double> f1[3][3], f2[3][3];
    force_outer(spin_proj<DIR, S1>(a), b, f1);
    force_outer(spin_proj<DIR, S2>(c), d, f2);
    double2 *o = out + ((size_t)DIR * V + lex) * 9;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const Cx<double> v = k * f1[i][j] + k * f2[i][j];
            o[i * 3 + j] = make_double2(v.re, v.im);
        }
}

template <int SIGN>
__global__ void __launch_bounds__(kForceBlock) k_eo_force(Geom g, SpinorF64 chi, SpinorF64 psi, SpinorF64 t1,
                                                         SpinorF64 t2, double kappa, long V, double2 *out) {
    const int par = blockIdx.y;  // 0 EVEN, 1 ODD
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.Vh; i += gridDim.x * blockDim.x) {
        const SiteNbrs nb = site_neighbours(g, i, par);
        // lexicographic index: i = xh + lxh * q1 with q1 = y + Ly (z + Lz t), x = 2 xh + parity offset
        const int q1 = (int)g.dx.div((unsigned)i);
        const int xh = i - q1 * g.lxh;
        const int q2 = (int)g.dy.div((unsigned)q1);
        const int y = q1 - q2 * g.L[1];
        const int t = (int)g.dz.div((unsigned)q2);
        const int z = q2 - t * g.L[2];
        const long lex = 2 * xh + ((y + z + t + par) & 1) + (long)g.L[0] * q1;
        Spinor<double> b, d;
        if (par == 0) {
            psi.load(i, b);
            chi.load(i, d);
            force_dir<0, -SIGN, SIGN>(nb, t1, b, t2, d, kappa, V, lex, out);
            force_dir<1, -SIGN, SIGN>(nb, t1, b, t2, d, kappa, V, lex, out);
            force_dir<2, -SIGN, SIGN>(nb, t1, b, t2, d, kappa, V, lex, out);
            force_dir<3, -SIGN, SIGN>(nb, t1, b, t2, d, kappa, V, lex, out);
        } else {
            t1.load(i, b);
            t2.load(i, d);
            force_dir<0, SIGN, -SIGN>(nb, psi, b, chi, d, kappa, V, lex, out);
            force_dir<1, SIGN, -SIGN>(nb, psi, b, chi, d, kappa, V, lex, out);
            force_dir<2, SIGN, -SIGN>(nb, psi, b, chi, d, kappa, V, lex, out);
            force_dir<3, SIGN, -SIGN>(nb, psi, b, chi, d, kappa, V, lex, out);
        }
    }
}

}  // namespace
}  // namespace hw

using namespace hw;

extern "C" int hw_wilson_evenodd_force(const hw_gauge *gauge, double kappa, const hw_field *chi, const hw_field *psi,
                                       int sign, double *force) {
    HW_CHECK_ARG(gauge && chi && psi && force, "null argument");
    HW_CHECK_ARG(sign == 1 || sign == -1, "sign must be +1 or -1");
    hw_lattice *lat = gauge->lat;
    HW_CHECK_ARG(chi->lat == lat && psi->lat == lat, "fields and gauge live on different lattices");
    hw_context *ctx = lat->ctx;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    HW_CUDA(cudaSetDevice(ctx->device));
    int rc;
    if ((rc = tune_hop(lat, gauge)) != HW_OK) return rc;
    const int stride = lat->stride;
    DevBuf t1, t2, out;
    if ((rc = t1.alloc((size_t)12 * stride * sizeof(double2))) != HW_OK) return rc;
    if ((rc = t2.alloc((size_t)12 * stride * sizeof(double2))) != HW_OK) return rc;
    if ((rc = out.alloc((size_t)36 * lat->V * sizeof(double2))) != HW_OK) return rc;
    const HalfF64 h1{t1.as<double2>(), stride}, h2{t2.as<double2>(), stride};
    // t1 = -kappa H^{oe}_{-s} chi, t2 = -kappa H^{oe}_s psi (wilson.h:298-307)
    launch_hop_scale(lat->g, gauge->U(), 1, -sign, chi->half[0].h(), h1, -kappa, nullptr, ctx->stream);
    launch_hop_scale(lat->g, gauge->U(), 1, sign, psi->half[0].h(), h2, -kappa, nullptr, ctx->stream);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long want = (lat->Vh + kForceBlock - 1) / kForceBlock;
    dim3 grid((unsigned)std::min<long>(want, 8L * sms), 2);
    const SpinorF64 c{chi->half[0].buf.as<double2>(), stride}, p{psi->half[0].buf.as<double2>(), stride};
    const SpinorF64 s1{h1.p, stride}, s2{h2.p, stride};
    if (sign > 0)
        k_eo_force<1><<<grid, kForceBlock, 0, ctx->stream>>>(lat->g, c, p, s1, s2, kappa, lat->V, out.as<double2>());
    else
        k_eo_force<-1><<<grid, kForceBlock, 0, ctx->stream>>>(lat->g, c, p, s1, s2, kappa, lat->V, out.as<double2>());
    HW_CUDA(cudaGetLastError());
    HW_CUDA(cudaMemcpyAsync(force, out.ptr, out.bytes, cudaMemcpyDeviceToHost, ctx->stream));
    HW_CUDA(cudaStreamSynchronize(ctx->stream));
    return HW_OK;
}
