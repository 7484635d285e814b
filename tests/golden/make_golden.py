"""Generate the golden fixtures in this folder from the CPU oracle.

    python tests/golden/make_golden.py

wilson_4x4x4x4.npz holds, for a 4^4 lattice (t antiperiodic), seeded links
(eps = 0.3, seed 1) and an EVEN Gaussian source (seed 2): the even-odd apply
and dagger at kappa = 0.12, Dirac_Wilson_hop_set on both parities, and the
CG<Dirac_Wilson_evenodd> solution of M^dag M x = source (accuracy 1e-12).
The oracle it comes from is pinned by the reference's identity tests and an
independent numpy restatement (tests/test_oracle.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as o  # noqa: E402


def main():
    dims = (4, 4, 4, 4)
    kappa = 0.12
    U = o.gen_links(dims, 0.3, 1)
    src = o.gen_spinor(dims, 2, o.EVEN)
    full = o.gen_spinor(dims, 3, o.ALL)
    hop_e = np.zeros_like(full)
    o.hop(dims, U, kappa, full, hop_e, o.EVEN, 1, True)
    hop_o = np.zeros_like(full)
    o.hop(dims, U, kappa, full, hop_o, o.ODD, -1, True)
    x, it, rr = o.cg(dims, U, kappa, src)
    np.savez_compressed(
        os.path.join(HERE, "wilson_4x4x4x4.npz"),
        dims=np.array(dims), kappa=np.array(kappa), links=U, source=src, full=full,
        apply=o.eo_apply(dims, U, kappa, src, 1), dagger=o.eo_apply(dims, U, kappa, src, -1),
        hop_even_plus=hop_e, hop_odd_minus=hop_o, cg_solution=x, cg_iterations=np.array(it),
    )


if __name__ == "__main__":
    main()
