"""CPU tests that pin the oracle.

The reference ships no golden vectors for the Wilson path; its own tests
(applications/test_cases/test_CG.cpp) pin it by identities.  These tests run
the same identities on random SU(3) links (the reference uses unit links),
plus: agreement with an independent numpy restatement written from the gamma
matrices, the analytic free-field plane-wave spectrum, gamma5-hermiticity, and
a dense-matrix solve.
"""
import numpy as np
import pytest

import np_wilson as nw


def rel_site_err(a, b):
    a = a.reshape(-1, 24)
    b = b.reshape(-1, 24)
    num = np.linalg.norm(a - b, axis=1)
    den = np.linalg.norm(b, axis=1)
    return np.where(den > 1e-300, num / np.maximum(den, 1e-300), num).max()


# ---------------------------------------------------------------- test_CG.cpp:10-42

def test_gamma_identities(oracle):
    """gamma5^2 = 1, gamma_d^2 = 1, projector norms, (U h).expand == U (1 +- gamma) w."""
    rng = np.random.default_rng(1)
    U = oracle.gen_links((2, 2, 2, 2), 0.7, 3)[0, 0]
    for trial in range(5):
        w1 = rng.standard_normal((4, 3, 2))
        w2 = w1 - oracle.gamma(4, oracle.gamma(4, w1))
        assert (w2 ** 2).sum() < 1e-28
        for d in range(4):
            gd = [1, 2, 3, 0][d]  # gamma_matrix[] = {gamma1, gamma2, gamma3, gamma0}
            w2 = w1 - oracle.gamma(gd, oracle.gamma(gd, w1))
            assert (w2 ** 2).sum() < 1e-24
            for sign in (1, -1):
                w2 = w1 + sign * oracle.gamma(gd, w1)
                h1 = oracle.project(w1, d, sign)
                diff = (w2 ** 2).sum() - 2 * (h1 ** 2).sum()
                assert diff * diff < 1e-20
                Uc = U[..., 0] + 1j * U[..., 1]
                w2c = w2[..., 0] + 1j * w2[..., 1]
                Uh = oracle.mul_half(U, h1)
                w3 = oracle.expand(Uh, d, sign)
                w3c = w3[..., 0] + 1j * w3[..., 1]
                ref = np.einsum("ij,sj->si", Uc, w2c)
                assert np.abs(w3c - ref).max() < 1e-13


# ---------------------------------------------------------------- independent restatement

@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (2, 4, 6, 4), (6, 2, 4, 8)])
@pytest.mark.parametrize("antiperiodic", [True, False])
def test_hop_matches_numpy_restatement(oracle, dims, antiperiodic):
    U = oracle.gen_links(dims, 0.3, 5)
    psi = oracle.gen_spinor(dims, 7, oracle.ALL)
    Ug, pg = nw.links_to_grid(U, dims), nw.to_grid(psi, dims)
    for sign in (1, -1):
        out = np.zeros_like(psi)
        oracle.hop(dims, U, 1.0, psi, out, oracle.ALL, sign, True, antiperiodic)
        ref = nw.from_grid(-nw.hop(Ug, pg, sign, antiperiodic))
        assert rel_site_err(out, ref) < 1e-13


def test_eo_apply_matches_numpy_restatement(oracle):
    dims = (4, 4, 2, 6)
    U = oracle.gen_links(dims, 0.3, 11)
    pe = oracle.gen_spinor(dims, 12, oracle.EVEN)
    for sign in (1, -1):
        a = oracle.eo_apply(dims, U, 0.12, pe, sign)
        b = nw.from_grid(nw.eo_apply(nw.links_to_grid(U, dims), nw.to_grid(pe, dims), 0.12, sign, dims))
        assert rel_site_err(a, b) < 1e-13


# ---------------------------------------------------------------- analytic free field

@pytest.mark.parametrize("sign", [1, -1])
def test_free_field_plane_wave(oracle, sign):
    """U = 1: H_s e^{ipx} u = sum_mu [2 cos p_mu + 2 i s gamma_mu sin p_mu] e^{ipx} u,
    with antiperiodic t momenta p_t = (2n+1) pi / Lt."""
    dims = (4, 6, 4, 8)
    U = oracle.unit_links(dims)
    Lx, Ly, Lz, Lt = dims
    n = (1, 2, 3, 1)
    p = [2 * np.pi * n[0] / Lx, 2 * np.pi * n[1] / Ly, 2 * np.pi * n[2] / Lz, (2 * n[3] + 1) * np.pi / Lt]
    rng = np.random.default_rng(4)
    u = rng.standard_normal((4, 3)) + 1j * rng.standard_normal((4, 3))
    t, z, y, x = np.meshgrid(np.arange(Lt), np.arange(Lz), np.arange(Ly), np.arange(Lx), indexing="ij")
    phase = np.exp(1j * (p[0] * x + p[1] * y + p[2] * z + p[3] * t))
    psig = phase[..., None, None] * u
    psi = nw.from_grid(psig)
    out = np.zeros_like(psi)
    oracle.hop(dims, U, -1.0, psi, out, oracle.ALL, sign, True, True)  # out = +H psi
    K = sum(2 * np.cos(p[mu]) * np.eye(4) + 2j * sign * np.sin(p[mu]) * nw.GAMMA[nw.DIR_GAMMA[mu]]
            for mu in range(4))
    ref = nw.from_grid(phase[..., None, None] * np.einsum("st,tc->sc", K, u))
    assert np.abs(out - ref).max() < 1e-12


# ---------------------------------------------------------------- test_CG.cpp:145-154, 236-245

@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (8, 4, 4, 6)])
def test_adjointness_random_links(oracle, dims):
    U = oracle.gen_links(dims, 0.3, 21)
    a = oracle.gen_spinor(dims, 22, oracle.EVEN)
    b = oracle.gen_spinor(dims, 23, oracle.EVEN)
    Db = oracle.eo_apply(dims, U, 0.12, b, 1)
    Dda = oracle.eo_apply(dims, U, 0.12, a, -1)
    d = oracle.dot(dims, a, Db, oracle.EVEN) - oracle.dot(dims, Dda, b, oracle.EVEN)
    scale = np.sqrt(oracle.squarenorm(dims, a) * oracle.squarenorm(dims, b))
    assert abs(d.real) / scale < 1e-15 and abs(d.imag) / scale < 1e-15
    # unpreconditioned Dirac_Wilson (test_CG.cpp:145-154), kappa 0.05
    a = oracle.gen_spinor(dims, 24)
    b = oracle.gen_spinor(dims, 25)
    d = oracle.dot(dims, a, oracle.wilson_apply(dims, U, 0.05, b, 1)) - \
        oracle.dot(dims, oracle.wilson_apply(dims, U, 0.05, a, -1), b)
    scale = np.sqrt(oracle.squarenorm(dims, a) * oracle.squarenorm(dims, b))
    assert abs(d) / scale < 1e-15


def test_gamma5_hermiticity(oracle):
    dims = (4, 4, 4, 4)
    U = oracle.gen_links(dims, 0.3, 31)
    psi = oracle.gen_spinor(dims, 32)
    g5 = np.ones((1, 4, 1, 1))
    g5[0, 2:] = -1
    for sign in (1, -1):
        lhs = g5 * oracle.wilson_apply(dims, U, 0.1, np.ascontiguousarray(g5 * psi), sign)
        rhs = oracle.wilson_apply(dims, U, 0.1, psi, -sign)
        assert rel_site_err(lhs, rhs) < 1e-13
        pe = oracle.gen_spinor(dims, 33, oracle.EVEN)
        lhs = g5 * oracle.eo_apply(dims, U, 0.12, np.ascontiguousarray(g5 * pe), sign)
        rhs = oracle.eo_apply(dims, U, 0.12, pe, -sign)
        assert rel_site_err(lhs, rhs) < 1e-13


# ---------------------------------------------------------------- test_CG.cpp:247-287

def test_cg_identities(oracle):
    dims = (4, 4, 4, 8)
    U = oracle.gen_links(dims, 0.3, 41)
    kappa = 0.12
    a = oracle.gen_spinor(dims, 42, oracle.EVEN)
    # D (D^dag D)^-1 D^dag a = a
    Dda = oracle.eo_apply(dims, U, kappa, a, -1)
    b, it, rr = oracle.cg(dims, U, kappa, Dda)
    Db = oracle.eo_apply(dims, U, kappa, b, 1)
    diff = oracle.squarenorm(dims, a - Db, oracle.EVEN)
    assert diff * diff < 1e-16 and it > 0
    # D^dag D (D^dag D)^-1 a = a
    b, it, rr = oracle.cg(dims, U, kappa, a)
    DDb = oracle.eo_apply(dims, U, kappa, oracle.eo_apply(dims, U, kappa, b, 1), -1)
    diff = oracle.squarenorm(dims, a - DDb, oracle.EVEN)
    assert diff * diff < 1e-16
    assert rr < 1e-24
    # (D^dag D)^-1 D^dag D b = b
    b = oracle.gen_spinor(dims, 43, oracle.EVEN)
    DDb = oracle.eo_apply(dims, U, kappa, oracle.eo_apply(dims, U, kappa, b, 1), -1)
    x, it, rr = oracle.cg(dims, U, kappa, DDb)
    diff = oracle.squarenorm(dims, x - b, oracle.EVEN)
    assert diff * diff < 1e-16


def test_dense_solve_crosscheck(oracle):
    """Build M as a dense matrix on a tiny lattice and solve M x = b by LU."""
    dims = (2, 2, 4, 4)
    U = oracle.gen_links(dims, 0.5, 51)
    kappa = 0.12
    V = int(np.prod(dims))
    par = np.array([sum((i // np.prod(dims[:d])) % dims[d] for d in range(4)) % 2 for i in range(V)])
    even = np.where(par == 0)[0]
    n = len(even) * 12
    Mdense = np.zeros((n, n), complex)
    for k in range(n):
        e = np.zeros((V, 4, 3, 2))
        site, comp = even[k // 12], k % 12
        e[site, comp // 3, comp % 3, 0] = 1.0
        col = oracle.eo_apply(dims, U, kappa, e, 1)
        c = col[..., 0] + 1j * col[..., 1]
        Mdense[:, k] = c.reshape(V, 12)[even].reshape(-1)
    b = oracle.gen_spinor(dims, 52, oracle.EVEN)
    bc = (b[..., 0] + 1j * b[..., 1]).reshape(V, 12)[even].reshape(-1)
    xd = np.linalg.solve(Mdense, bc)
    Mdb = oracle.eo_apply(dims, U, kappa, b, -1)
    x, it, rr = oracle.cg(dims, U, kappa, Mdb, acc=1e-14)
    xc = (x[..., 0] + 1j * x[..., 1]).reshape(V, 12)[even].reshape(-1)
    assert np.linalg.norm(xc - xd) / np.linalg.norm(xd) < 1e-11
    assert oracle.true_residual(dims, U, kappa, b, x) < 1e-12


def test_reference_structured_matches(oracle):
    dims = (4, 4, 4, 6)
    U = oracle.gen_links(dims, 0.3, 61)
    pe = oracle.gen_spinor(dims, 62, oracle.EVEN)
    R = oracle.RefStructured(dims)
    for sign in (1, -1):
        out = np.zeros_like(pe)
        R.eo_apply(U, 0.12, pe, out, sign)
        ref = oracle.eo_apply(dims, U, 0.12, pe, sign)
        assert rel_site_err(out, ref) < 1e-13
    R.close()


def test_links_are_special_unitary(oracle):
    U = oracle.gen_links((4, 4, 4, 4), 0.3, 71)
    Uc = oracle.to_complex_links(U)
    eye = np.einsum("dvij,dvkj->dvik", Uc, Uc.conj())
    assert np.abs(eye - np.eye(3)).max() < 1e-14
    assert np.abs(np.linalg.det(Uc) - 1).max() < 1e-14
    # eps = 0.3: <Re tr U>/3 = 1 - eps^2 <tr H^2>/6 + ... with <tr H^2> = 8
    assert abs(np.trace(Uc, axis1=2, axis2=3).real.mean() / 3 - 0.886) < 0.01
