"""The oracle against the committed golden fixtures (tests/golden/make_golden.py)."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_reproduces_golden(oracle):
    g = np.load(os.path.join(HERE, "golden", "wilson_4x4x4x4.npz"))
    dims = tuple(int(d) for d in g["dims"])
    kappa = float(g["kappa"])
    U = oracle.gen_links(dims, 0.3, 1)
    assert np.abs(U - g["links"]).max() < 1e-15
    src = np.ascontiguousarray(g["source"])
    assert np.array_equal(oracle.gen_spinor(dims, 2, oracle.EVEN), src)
    Ug = np.ascontiguousarray(g["links"])
    assert np.abs(oracle.eo_apply(dims, Ug, kappa, src, 1) - g["apply"]).max() < 1e-13
    assert np.abs(oracle.eo_apply(dims, Ug, kappa, src, -1) - g["dagger"]).max() < 1e-13
    full = np.ascontiguousarray(g["full"])
    h = np.zeros_like(full)
    oracle.hop(dims, Ug, kappa, full, h, oracle.EVEN, 1, True)
    assert np.abs(h - g["hop_even_plus"]).max() < 1e-13
    x, it, rr = oracle.cg(dims, Ug, kappa, src)
    assert abs(it - int(g["cg_iterations"])) <= 1
    assert np.abs(x - g["cg_solution"]).max() < 1e-10
