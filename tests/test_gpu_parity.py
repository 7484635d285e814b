"""GPU parity of the FP64 operators and CG against the CPU oracle.

Tolerances (FP64): per-site relative error ||gpu - oracle|| / ||oracle|| <= 1e-13
for the operators; every solve's true residual |b - M x| / |b|, recomputed by
the oracle in FP64, <= 1e-10.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SITE_TOL = 1e-13


def rel_site_err(a, b):
    a = a.reshape(-1, 24)
    b = b.reshape(-1, 24)
    num = np.linalg.norm(a - b, axis=1)
    den = np.linalg.norm(b, axis=1)
    return np.where(den > 1e-300, num / np.maximum(den, 1e-300), num).max()


def setup(hw, ctx, oracle, dims, eps=0.3, seed=1, link_format=18, antiperiodic=True):
    U = oracle.gen_links(dims, eps, seed)
    lat = hw.Lattice(ctx, dims, antiperiodic)
    G = hw.GaugeField(lat, U, link_format)
    return U, lat, G


DIMS = [(4, 4, 4, 4), (2, 4, 6, 8), (8, 8, 8, 8), (6, 2, 4, 10), (16, 8, 8, 8)]


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("link_format", [18, 12])
def test_evenodd_apply_dagger(hw, ctx, oracle, dims, link_format):
    U, lat, G = setup(hw, ctx, oracle, dims, seed=3, link_format=link_format)
    psi = oracle.gen_spinor(dims, 4, oracle.EVEN)
    fin, fout = hw.Field(lat, psi), hw.Field(lat)
    D = hw.Dirac_Wilson_evenodd(0.12, G)
    for sign, fn in ((1, D.apply), (-1, D.dagger)):
        fn(fin, fout)
        gpu = fout.download()
        ref = oracle.eo_apply(dims, U, 0.12, psi, sign)
        assert rel_site_err(gpu, ref) <= SITE_TOL
        assert np.all(gpu.reshape(-1, 24)[np.linalg.norm(ref.reshape(-1, 24), axis=1) == 0] == 0)


@pytest.mark.parametrize("link_format", [18, 12])
def test_evenodd_against_reference_fixture(hw, ctx, link_format):
    """The GPU operator against the reference-built golden vectors of tests/golden/ref_wilson.npz
    (the reference's HalfWilsonVector / expand / SU(3) arithmetic and its generators, compiled
    with g++; tests/golden/make_ref_golden.py): apply and dagger, t antiperiodic and periodic,
    and Dirac_Wilson_hop_set on both parities, <= 1e-13 relative per site."""
    import os
    ref = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_wilson.npz")))
    kappa = float(ref["kappa"])
    n = 0
    while f"dims{n}" in ref:
        dims = tuple(int(v) for v in ref[f"dims{n}"])
        U = ref[f"links{n}"]
        for ap, tag in ((True, "ap"), (False, "per")):
            lat = hw.Lattice(ctx, dims, ap)
            G = hw.GaugeField(lat, U, link_format)
            D = hw.Dirac_Wilson_evenodd(kappa, G)
            fin, fout = hw.Field(lat, ref[f"source{n}"]), hw.Field(lat)
            for fn, name in ((D.apply, "apply"), (D.dagger, "dagger")):
                fn(fin, fout)
                assert rel_site_err(fout.download(), ref[f"{name}_{tag}{n}"]) <= SITE_TOL, (dims, name, tag)
            if ap:
                ff = hw.Field(lat, ref[f"full{n}"])
                for par, sign, name in ((hw.EVEN, 1, "hop_even_plus"), (hw.ODD, -1, "hop_odd_minus")):
                    fh = hw.Field(lat)
                    D.hop(ff, fh, par, sign, True)
                    got = fh.download(par)
                    mask = np.zeros(got.shape[0], bool)
                    want = ref[f"{name}{n}"]
                    mask[np.linalg.norm(want.reshape(-1, 24), axis=1) > 0] = True
                    assert rel_site_err(got[mask], want[mask]) <= SITE_TOL, (dims, name)
                    fh.close()
                ff.close()
            for h in (fin, fout, G, lat):
                h.close()
        n += 1


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (2, 6, 4, 8)])
@pytest.mark.parametrize("antiperiodic", [True, False])
def test_hop_and_unpreconditioned(hw, ctx, oracle, dims, antiperiodic):
    U, lat, G = setup(hw, ctx, oracle, dims, seed=5, antiperiodic=antiperiodic)
    psi = oracle.gen_spinor(dims, 6, oracle.ALL)
    prev = oracle.gen_spinor(dims, 7, oracle.ALL)
    fin = hw.Field(lat, psi)
    D = hw.Dirac_Wilson_evenodd(0.11, G)
    for par in (oracle.EVEN, oracle.ODD):
        for sign in (1, -1):
            for set_ in (True, False):
                fout = hw.Field(lat, prev)
                D.hop(fin, fout, par, sign, set_)
                ref = prev.copy()
                oracle.hop(dims, U, 0.11, psi, ref, par, sign, set_, antiperiodic)
                assert rel_site_err(fout.download(), ref) <= SITE_TOL
    W = hw.Dirac_Wilson(0.05, G)
    fout = hw.Field(lat)
    for sign, fn in ((1, W.apply), (-1, W.dagger)):
        fn(fin, fout)
        ref = oracle.wilson_apply(dims, U, 0.05, psi, sign, antiperiodic)
        assert rel_site_err(fout.download(), ref) <= SITE_TOL


def test_dslash_32_4(hw, ctx, oracle):
    """The dslash bench size: 32^4, eps = 0.3, apply and dagger within 1e-13 per site."""
    dims = (32, 32, 32, 32)
    for link_format in (18, 12):
        U, lat, G = setup(hw, ctx, oracle, dims, seed=100, link_format=link_format)
        psi = oracle.gen_spinor(dims, 101, oracle.EVEN)
        fin, fout = hw.Field(lat, psi), hw.Field(lat)
        D = hw.Dirac_Wilson_evenodd(0.124, G)
        for sign, fn in ((1, D.apply), (-1, D.dagger)):
            fn(fin, fout)
            ref = oracle.eo_apply(dims, U, 0.124, psi, sign)
            assert rel_site_err(fout.download(), ref) <= SITE_TOL


def test_adjointness_linearity_gpu(hw, ctx, oracle):
    dims = (16, 16, 16, 16)
    U, lat, G = setup(hw, ctx, oracle, dims, seed=9)
    a = oracle.gen_spinor(dims, 10, oracle.EVEN)
    b = oracle.gen_spinor(dims, 11, oracle.EVEN)
    D = hw.Dirac_Wilson_evenodd(0.124, G)
    fa, fb, o1, o2 = hw.Field(lat, a), hw.Field(lat, b), hw.Field(lat), hw.Field(lat)
    D.apply(fb, o1)
    D.dagger(fa, o2)
    Mb, Mda = o1.download(), o2.download()
    d = oracle.dot(dims, a, Mb, oracle.EVEN) - oracle.dot(dims, Mda, b, oracle.EVEN)
    scale = np.sqrt(oracle.squarenorm(dims, a) * oracle.squarenorm(dims, b))
    assert abs(d) / scale < 1e-14
    # linearity: M(2a + b) = 2 Ma + Mb
    fc = hw.Field(lat, 2 * a + b)
    D.apply(fc, o2)
    D.apply(fa, o1)
    Ma = o1.download()
    lhs = o2.download()
    assert rel_site_err(lhs, 2 * Ma + Mb) < 1e-13


# ---------------------------------------------------------------- solver

def test_cg_reference_semantics(hw, ctx, oracle):
    """CG<Dirac_Wilson_evenodd>::apply on the 8^4 workload vs the oracle's CG."""
    dims = (8, 8, 8, 8)
    U, lat, G = setup(hw, ctx, oracle, dims, seed=1)
    src = oracle.gen_spinor(dims, 2, oracle.EVEN)
    D = hw.Dirac_Wilson_evenodd(0.12, G)
    for use_graph in (True, False):
        fin, fout = hw.Field(lat, src), hw.Field(lat)
        res = hw.CG(D, use_graph=use_graph).apply(fin, fout)
        assert res.converged
        x = fout.download()
        xo, it_o, rr_o = oracle.cg(dims, U, 0.12, src)
        assert abs(res.iterations - it_o) <= 1
        assert res.rr_relative < 1e-24
        assert oracle.true_residual_normal(dims, U, 0.12, src, x) < 1e-10
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-9


@pytest.mark.parametrize("dims,kappa", [((8, 8, 8, 8), 0.12), ((4, 4, 4, 4), 0.124), ((2, 4, 6, 8), 0.115)])
def test_solve_true_residual(hw, ctx, oracle, dims, kappa):
    U, lat, G = setup(hw, ctx, oracle, dims, seed=21)
    b = oracle.gen_spinor(dims, 22, oracle.EVEN)
    D = hw.Dirac_Wilson_evenodd(kappa, G)
    fb, fx = hw.Field(lat, b), hw.Field(lat)
    res = D.solve(fb, fx, accuracy=1e-10)
    assert res.converged, res
    x = fx.download()
    tr = oracle.true_residual(dims, U, kappa, b, x)
    assert tr <= 1e-10
    assert abs(tr - res.true_residual) <= 1e-3 * tr + 1e-14
    # host-array entry point gives the same solution
    xh = np.zeros_like(b)
    res2 = D.solve_host(b, xh, accuracy=1e-10)
    assert res2.converged and res2.iterations == res.iterations
    assert np.array_equal(xh, x)


def test_solve_edge_cases(hw, ctx, oracle):
    dims = (4, 4, 4, 4)
    U, lat, G = setup(hw, ctx, oracle, dims, seed=31)
    D = hw.Dirac_Wilson_evenodd(0.12, G)
    # zero source: converged immediately with x = 0
    fb, fx = hw.Field(lat), hw.Field(lat)
    res = D.solve(fb, fx)
    assert res.converged and res.iterations == 0
    assert not fx.download().any()
    # maxiters = 1 reports not converged
    b = oracle.gen_spinor(dims, 32, oracle.EVEN)
    fb.upload(b)
    res = D.solve(fb, fx, accuracy=1e-10, maxiters=1)
    assert res.status == hw.HW_ERR_NOT_CONVERGED and res.iterations == 1
    # non-finite source reports breakdown, context stays usable
    bad = b.copy()
    bad[0, 0, 0, 0] = np.nan
    fb.upload(bad)
    fx.zero()
    res = D.solve(fb, fx)
    assert res.status == hw.HW_ERR_BREAKDOWN
    fb.upload(b)
    fx.zero()
    assert D.solve(fb, fx).converged


def test_golden_fixtures_gpu(hw, ctx, oracle):
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "wilson_4x4x4x4.npz")
    g = np.load(path)
    dims = tuple(int(d) for d in g["dims"])
    lat = hw.Lattice(ctx, dims, True)
    G = hw.GaugeField(lat, np.ascontiguousarray(g["links"]))
    D = hw.Dirac_Wilson_evenodd(float(g["kappa"]), G)
    fin, fout = hw.Field(lat, np.ascontiguousarray(g["source"])), hw.Field(lat)
    D.apply(fin, fout)
    assert rel_site_err(fout.download(), g["apply"]) <= SITE_TOL
    D.dagger(fin, fout)
    assert rel_site_err(fout.download(), g["dagger"]) <= SITE_TOL


@pytest.mark.parametrize("antiperiodic", [True, False])
def test_unpreconditioned_cg(hw, ctx, oracle, antiperiodic):
    """CG<Dirac_Wilson>::apply (hw_wilson_cg_solve): M^dag M x = b on ALL sites, judged by the
    oracle's FP64 residual |b - M^dag M x| / |b| with M the unpreconditioned operator."""
    dims = (4, 4, 4, 8)
    U, lat, G = setup(hw, ctx, oracle, dims, seed=41, antiperiodic=antiperiodic)
    b = oracle.gen_spinor(dims, 42, oracle.ALL)
    D = hw.Dirac_Wilson(0.11, G)
    fb, fx = hw.Field(lat, b), hw.Field(lat)
    r = D.cg(fb, fx, accuracy=1e-11, true_residual=True)
    assert r.converged, r
    x = fx.download()
    mx = oracle.wilson_apply(dims, U, 0.11, x, 1, antiperiodic)
    mmx = oracle.wilson_apply(dims, U, 0.11, mx, -1, antiperiodic)
    res = np.linalg.norm(mmx - b) / np.linalg.norm(b)
    assert res <= 1e-10 and abs(res - r.true_residual) <= 1e-3 * res + 1e-15
