"""The oracle and the host generators against golden vectors made by the reference's own code.

tests/golden/ref_wilson.npz comes from oracle/_ref/libref_pin.so, which compiles the
reference's site algebra and generators with g++ (oracle/ref_pin/: the reference headers
cmplx.h, matrix.h, sun_matrix.h as they are, plus wilson_vector.h's gamma matrices,
HalfWilsonVector projection and expand(), and random.cpp's generator cut out verbatim);
tests/golden/make_ref_golden.py regenerates it.  Checked here, on the CPU:
  * the oracle's projection, expansion and gamma tables, site by site, exactly;
  * the oracle's even-odd operator (apply, dagger; t antiperiodic and periodic) and
    hopping term against the reference-built ones: <= 1e-13 relative per site;
  * the oracle's and the library's input generators against the reference's: spinors
    and the Gaussian stream bit for bit, links to 1e-15.
The GPU operator is checked against the same fixtures in tests/test_gpu_parity.py.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_wilson.npz")
SITE_TOL = 1e-13


@pytest.fixture(scope="module")
def ref():
    return dict(np.load(FIX))


def lattices(ref):
    n = 0
    while f"dims{n}" in ref:
        yield n, tuple(int(v) for v in ref[f"dims{n}"])
        n += 1


def rel_site_err(a, b):
    a, b = a.reshape(-1, 24), b.reshape(-1, 24)
    num = np.linalg.norm(a - b, axis=1)
    den = np.linalg.norm(b, axis=1)
    return np.where(den > 0, num / np.maximum(den, 1e-300), num).max()


def test_site_algebra_tables(oracle, ref):
    w = ref["site_w"]
    for k in range(len(w)):
        for d in range(4):
            for si, s in enumerate((1, -1)):
                h = oracle.project(w[k], d, s)
                assert np.array_equal(h, ref["site_proj"][k, d, si]), (k, d, s)
                assert np.array_equal(oracle.expand(h, d, s), ref["site_expand"][k, d, si]), (k, d, s)
        for gi, g in enumerate((0, 1, 2, 3, 5)):
            assert np.array_equal(oracle.gamma(g, w[k]), ref["site_gamma"][k, gi]), (k, g)


def test_operator_against_reference(oracle, ref):
    kappa = float(ref["kappa"])
    for n, dims in lattices(ref):
        U, src, full = ref[f"links{n}"], ref[f"source{n}"], ref[f"full{n}"]
        for ap, tag in ((True, "ap"), (False, "per")):
            for sign, name in ((1, "apply"), (-1, "dagger")):
                got = oracle.eo_apply(dims, U, kappa, src, sign, ap)
                assert rel_site_err(got, ref[f"{name}_{tag}{n}"]) <= SITE_TOL, (dims, name, tag)
        for par, sign, name in ((oracle.EVEN, 1, "hop_even_plus"), (oracle.ODD, -1, "hop_odd_minus")):
            out = np.zeros_like(full)
            oracle.hop(dims, U, kappa, full, out, par, sign, True)
            mask = oracle.parity_mask(dims) == (0 if par == oracle.EVEN else 1)
            assert rel_site_err(out[mask], ref[f"{name}{n}"][mask]) <= SITE_TOL, (dims, name)


def test_generators_against_reference(oracle, hw, ref):
    eps = float(ref["eps"])
    for n, dims in lattices(ref):
        U = ref[f"links{n}"]
        assert np.abs(oracle.gen_links(dims, eps, 1) - U).max() <= 1e-15
        assert np.abs(hw.generate_links(dims, eps, 1) - U).max() <= 1e-15
        assert np.array_equal(oracle.gen_spinor(dims, 2, oracle.EVEN), ref[f"source{n}"])
        assert np.array_equal(hw.generate_spinor(dims, 2, hw.EVEN), ref[f"source{n}"])
        assert np.array_equal(oracle.gen_spinor(dims, 3, oracle.ALL), ref[f"full{n}"])


def test_gaussian_stream(oracle, ref):
    """hila::gaussrand() after seed 5: the spinor generator draws the same Box-Muller pairs
    (re = first, im = second), so a one-site, all-parity spinor of seed 5 repeats the stream."""
    g = ref["gaussrand_seed5"]
    s = oracle.gen_spinor((2, 2, 2, 2), 5, oracle.ALL).reshape(-1)
    assert np.array_equal(s[:64], g)


def test_fixture_regenerates():
    """Where the pin library has been built (it needs the reference sources), it reproduces
    the committed fixture bit for bit."""
    from oracle.ref_pin import pin
    if not pin.available():
        pytest.skip("pin library not built here (reference sources absent)")
    r = dict(np.load(FIX))
    assert np.array_equal(pin.gaussrand(5, 64), r["gaussrand_seed5"])
    for n, dims in lattices(r):
        U = pin.gen_links(dims, float(r["eps"]), 1)
        assert np.array_equal(U, r[f"links{n}"])
        assert np.array_equal(pin.eo_apply(dims, U, float(r["kappa"]), r[f"source{n}"], 1, True), r[f"apply_ap{n}"])
