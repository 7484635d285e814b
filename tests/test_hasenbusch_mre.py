"""Hasenbusch operator M + m_h (Hasenbusch.h:16-52) and the MRE initial guess
(MRE_guess.h:9-88), against the oracle."""
import numpy as np
import pytest

DIMS = (4, 4, 4, 6)
KAPPA = 0.12


def _A(oracle, dims, U, mh, v):
    w = oracle.hasenbusch_eo_apply(dims, U, KAPPA, mh, v, +1)
    return oracle.hasenbusch_eo_apply(dims, U, KAPPA, mh, w, -1)


@pytest.mark.parametrize("mh", [0.0, 0.3])
def test_oracle_hasenbusch_adjoint(oracle, mh):
    U = oracle.gen_links(DIMS, 0.3, 61)
    a = oracle.gen_spinor(DIMS, 62, oracle.EVEN)
    b = oracle.gen_spinor(DIMS, 63, oracle.EVEN)
    lhs = oracle.dot(DIMS, a, oracle.hasenbusch_eo_apply(DIMS, U, KAPPA, mh, b, +1), oracle.EVEN)
    rhs = oracle.dot(DIMS, oracle.hasenbusch_eo_apply(DIMS, U, KAPPA, mh, a, -1), b, oracle.EVEN)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    # M + m_h differs from M by m_h on EVEN only
    d = oracle.hasenbusch_eo_apply(DIMS, U, KAPPA, mh, b, +1) - oracle.eo_apply(DIMS, U, KAPPA, b, +1)
    assert np.allclose(d, mh * b, rtol=0, atol=1e-14)


@pytest.mark.parametrize("mh", [0.0, 0.25])
def test_oracle_mre_exact_in_span(oracle, mh):
    """chi = A x with x in the span of the old solutions: the guess is x."""
    U = oracle.gen_links(DIMS, 0.3, 64)
    old = [oracle.gen_spinor(DIMS, 70 + k, oracle.EVEN) for k in range(4)]
    coef = np.array([0.7, -1.3, 0.2, 2.1])
    x = sum(c * o for c, o in zip(coef, old))
    chi = _A(oracle, DIMS, U, mh, x)
    g = oracle.mre_guess(DIMS, U, KAPPA, mh, old, chi)
    assert np.linalg.norm(g - x) <= 1e-10 * np.linalg.norm(x)
    assert not np.any(oracle.mre_guess(DIMS, U, KAPPA, mh, [], chi))


def test_oracle_mre_linearly_dependent(oracle):
    """A repeated old solution drops out (zero direction after Gram-Schmidt)."""
    U = oracle.gen_links(DIMS, 0.3, 65)
    o1 = oracle.gen_spinor(DIMS, 80, oracle.EVEN)
    o2 = oracle.gen_spinor(DIMS, 81, oracle.EVEN)
    chi = _A(oracle, DIMS, U, 0.0, 0.5 * o1 - o2)
    g = oracle.mre_guess(DIMS, U, KAPPA, 0.0, [o1, o2, o1.copy()], chi)
    assert np.linalg.norm(g - (0.5 * o1 - o2)) <= 1e-10 * np.linalg.norm(o1)


@pytest.mark.gpu
@pytest.mark.parametrize("sign", [1, -1])
def test_gpu_hasenbusch_apply(hw, ctx, oracle, sign):
    dims, mh = (8, 8, 8, 8), 0.35
    U = oracle.gen_links(dims, 0.3, 66)
    inp = oracle.gen_spinor(dims, 67, oracle.EVEN)
    ref = oracle.hasenbusch_eo_apply(dims, U, KAPPA, mh, inp, sign)
    lat = hw.Lattice(ctx, dims, True)
    G = hw.GaugeField(lat, U, 12)
    H = hw.Hasenbusch_operator(hw.Dirac_Wilson_evenodd(KAPPA, G), mh)
    fi, fo = hw.Field(lat, inp), hw.Field(lat)
    (H.apply if sign > 0 else H.dagger)(fi, fo)
    got = fo.download()
    err = np.linalg.norm((got - ref).reshape(-1, 24), axis=1)
    assert (err <= 1e-13 * np.maximum(np.linalg.norm(ref.reshape(-1, 24), axis=1), 1e-300)).all()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32", "f16"])
def test_gpu_hasenbusch_solve(hw, ctx, oracle, precision):
    dims, mh = (8, 8, 8, 8), 0.2
    U = oracle.gen_links(dims, 0.3, 68)
    b = oracle.gen_spinor(dims, 69, oracle.EVEN)
    lat = hw.Lattice(ctx, dims, True)
    G = hw.GaugeField(lat, U, 18)
    H = hw.Hasenbusch_operator(hw.Dirac_Wilson_evenodd(KAPPA, G), mh)
    fb, fx = hw.Field(lat, b), hw.Field(lat)
    r = H.solve(fb, fx, accuracy=1e-10, precision=precision, delta=0.005 if precision == "f16" else 1e-5)
    assert r.converged
    x = fx.download()
    res = b - oracle.hasenbusch_eo_apply(dims, U, KAPPA, mh, x, +1)
    assert np.linalg.norm(res) <= 1e-10 * np.linalg.norm(b)
    # the batched path solves the same system
    fx2 = hw.Field(lat)
    [rb] = hw.batch_solve(ctx, [(H, fb, fx2, 1e-10)], precision="f16", delta=0.005)
    assert rb.converged
    res2 = b - oracle.hasenbusch_eo_apply(dims, U, KAPPA, mh, fx2.download(), +1)
    assert np.linalg.norm(res2) <= 1e-10 * np.linalg.norm(b)


@pytest.mark.gpu
@pytest.mark.parametrize("mh", [0.0, 0.2])
def test_gpu_mre_guess(hw, ctx, oracle, mh):
    dims = (8, 8, 8, 8)
    U = oracle.gen_links(dims, 0.3, 90)
    lat = hw.Lattice(ctx, dims, True)
    G = hw.GaugeField(lat, U, 12)
    D = hw.Dirac_Wilson_evenodd(KAPPA, G)
    op = hw.Hasenbusch_operator(D, mh) if mh else D
    old_h = [oracle.gen_spinor(dims, 91 + k, oracle.EVEN) for k in range(5)]
    chi_h = oracle.gen_spinor(dims, 99, oracle.EVEN)
    ref = oracle.mre_guess(dims, U, KAPPA, mh, old_h, chi_h)
    old = [hw.Field(lat, o) for o in old_h]
    chi, psi = hw.Field(lat, chi_h), hw.Field(lat)
    hw.mre_guess(op, old, chi, psi)
    got = psi.download()
    assert np.linalg.norm(got - ref) <= 1e-10 * np.linalg.norm(ref)
    # exact when the solution lies in the span
    x = 0.3 * old_h[0] - 1.1 * old_h[3]
    chi2 = hw.Field(lat, _A(oracle, dims, U, mh, x))
    hw.mre_guess(op, old, chi2, psi)
    assert np.linalg.norm(psi.download() - x) <= 1e-9 * np.linalg.norm(x)


@pytest.mark.gpu
def test_gpu_mre_guess_saves_iterations(hw, ctx, oracle):
    """Earlier solutions of nearby sources: CG from the MRE guess needs fewer iterations."""
    dims = (8, 8, 8, 8)
    U = oracle.gen_links(dims, 0.3, 100)
    lat = hw.Lattice(ctx, dims, True)
    G = hw.GaugeField(lat, U, 12)
    D = hw.Dirac_Wilson_evenodd(KAPPA, G)
    cg = hw.CG(D, accuracy=1e-10)
    srcs = [oracle.gen_spinor(dims, 101 + k, oracle.EVEN) for k in range(3)]
    old = []
    for s_ in srcs:
        x = hw.Field(lat)
        cg.apply(hw.Field(lat, s_), x)
        old.append(x)
    new = srcs[1] + 0.01 * oracle.gen_spinor(dims, 120, oracle.EVEN)
    chi = hw.Field(lat, new)
    cold, warm = hw.Field(lat), hw.Field(lat)
    r0 = cg.apply(chi, cold)
    hw.mre_guess(D, old, chi, warm)
    r1 = cg.apply(chi, warm)
    assert r1.converged and r0.converged
    assert r1.iterations < r0.iterations
