// Device site algebra of staggered fermions (libraries/dirac/staggered.h), shared by
// the standalone operator kernels (staggered.cu) and the batched solver engine.
//
//   eta_d(x)  = ((sum_{d' < d} x_d') % 2) * 2 - 1      (staggered.h:14-28 as coded; its
//                                                       comment states the opposite sign)
//   hop v(x)  = sum_d eta_d(x) [U_d(x) v(x+d) - U_d(x-d)^dag v(x-d)]   (:48-68, without
//               the factor 0.5 s the callers apply)
// with the fermion boundary sign on values gathered across the t boundary.  A half
// lattice of a colour-vector field is 3 double2 planes (stride = padded parity size).
#pragma once

#include "storage.cuh"

namespace hw {

struct HalfStag {
    double2 *p;
    int stride;
    __device__ __forceinline__ Cx<double> ld(int c, int i) const {
        const double2 v = __ldg(p + (size_t)c * stride + i);
        return {v.x, v.y};
    }
    // plain (coherent) load, for arrays the same kernel also writes
    __device__ __forceinline__ Cx<double> ldp(int c, int i) const {
        const double2 v = p[(size_t)c * stride + i];
        return {v.x, v.y};
    }
    __device__ __forceinline__ void st(int c, int i, Cx<double> v) const {
        p[(size_t)c * stride + i] = make_double2(v.re, v.im);
    }
};

__device__ __forceinline__ double stag_eta(const int c[4], int d) {
    int s = 0;
    for (int k = 0; k < d; k++) s += c[k];
    return (s & 1) ? 1.0 : -1.0;
}

// acc = sum_d eta_d(x) [U_d(x) v(x+d) - U_d(x-d)^dag v(x-d)] at checkerboard site i of parity par
template <class Lk>
__device__ __forceinline__ void stag_hop_site(const Geom &g, const Lk &U, int par, int i, const HalfStag &v,
                                              Cx<double> acc[3]) {
    const SiteNbrs n = site_neighbours(g, i, par);
    int c[4];
    site_coords(g, i, par, c);
#pragma unroll
    for (int a = 0; a < 3; a++) acc[a] = {0.0, 0.0};
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const double eta = stag_eta(c, d);
        const double sf = (d == 3 && n.tfwd_wrap) ? -eta : eta;
        const double sb = (d == 3 && n.tbwd_wrap) ? -eta : eta;
        Su3<double> u;
        U.load(par, d, i, u);
        Cx<double> w[3];
#pragma unroll
        for (int b = 0; b < 3; b++) w[b] = v.ld(b, n.fwd[d]);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            Cx<double> t = cmul(u.e[a][0], w[0]) + cmul(u.e[a][1], w[1]) + cmul(u.e[a][2], w[2]);
            acc[a] = acc[a] + sf * t;
        }
        U.load(1 - par, d, n.bwd[d], u);
#pragma unroll
        for (int b = 0; b < 3; b++) w[b] = v.ld(b, n.bwd[d]);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            Cx<double> t = cmul(conj(u.e[0][a]), w[0]) + cmul(conj(u.e[1][a]), w[1]) + cmul(conj(u.e[2][a]), w[2]);
            acc[a] = acc[a] - sb * t;
        }
    }
}

}  // namespace hw
