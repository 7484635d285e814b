"""Generate the reference golden fixtures in this folder from the reference's own code.

    python tests/golden/make_ref_golden.py

Builds oracle/_ref/libref_pin.so from the reference sources (oracle/ref_pin/Makefile:
the reference headers compiled with g++, plus code cut verbatim out of wilson_vector.h
and random.cpp) and writes ref_wilson.npz.  For two lattices, 4^4 and 2x4x4x6:
  links    reunitarize(exp(eps A)), A from Algebra<SU<3>>::gaussian_random, eps 0.3, seed 1
           (sun_matrix.h, matrix.h:3289-3309, random.cpp)
  source   Complex::gaussian_random on EVEN sites, seed 2; `full` on all sites, seed 3
  apply / dagger  Dirac_Wilson_evenodd (wilson.h:272-289) at kappa 0.12, t antiperiodic and
           periodic, every site product through HalfWilsonVector / expand / SU(3) x vector
  hop      Dirac_Wilson_hop_set on EVEN (sign +1) and ODD (sign -1) of `full`
and, independent of the lattice: 64 numbers of hila::gaussrand() after seed 5, and for four
Gaussian Wilson vectors the projections and expansions of all (direction, sign) pairs and the
products with gamma 0, 1, 2, 3, 5.  The fixtures are committed; the GPU box has no reference.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.ref_pin import pin  # noqa: E402

LATTICES = [(4, 4, 4, 4), (2, 4, 4, 6)]
KAPPA, EPS = 0.12, 0.3


def main():
    pin.build()
    out = {"kappa": np.array(KAPPA), "eps": np.array(EPS), "gaussrand_seed5": pin.gaussrand(5, 64)}
    for n, dims in enumerate(LATTICES):
        U = pin.gen_links(dims, EPS, 1)
        src = pin.gen_spinor(dims, 2, 1)
        full = pin.gen_spinor(dims, 3, 3)
        out[f"dims{n}"] = np.array(dims)
        out[f"links{n}"] = U
        out[f"source{n}"] = src
        out[f"full{n}"] = full
        for ap in (True, False):
            tag = "ap" if ap else "per"
            out[f"apply_{tag}{n}"] = pin.eo_apply(dims, U, KAPPA, src, 1, ap)
            out[f"dagger_{tag}{n}"] = pin.eo_apply(dims, U, KAPPA, src, -1, ap)
        out[f"hop_even_plus{n}"] = pin.hop(dims, U, KAPPA, full, 0, 1)
        out[f"hop_odd_minus{n}"] = pin.hop(dims, U, KAPPA, full, 1, -1)
    w = pin.gen_spinor((2, 2, 2, 2), 4, 3)[:4]
    out["site_w"] = w
    out["site_proj"] = np.array([[[pin.project(w[k], d, s) for s in (1, -1)] for d in range(4)] for k in range(4)])
    out["site_expand"] = np.array([[[pin.expand(pin.project(w[k], d, s), d, s) for s in (1, -1)] for d in range(4)]
                                   for k in range(4)])
    out["site_gamma"] = np.array([[pin.gamma(g, w[k]) for g in (0, 1, 2, 3, 5)] for k in range(4)])
    np.savez_compressed(os.path.join(HERE, "ref_wilson.npz"), **out)


if __name__ == "__main__":
    main()
