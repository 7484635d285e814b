"""Wilson fermion force (Dirac_Wilson_evenodd::force, wilson.h:293-311).

The oracle is pinned by the finite-difference check of the reference's own
test (test_forces.cpp:15-100): for a link U_dir(c) -> (1 + i eps T) U_dir(c),
d/d eps Re(chi^dag M_s psi) equals Re Tr(P(U F) i T), where F is the force and
P the traceless anti-Hermitian projection that gauge_field.h:249-256 applies
before adding U F to the momentum.  The GPU force is compared with the oracle.
"""
import numpy as np
import pytest

DIMS = (4, 4, 4, 6)
KAPPA = 0.12


def _c(a):
    return a[..., 0] + 1j * a[..., 1]


def _r(z):
    return np.stack([z.real, z.imag], axis=-1)


def project_antihermitean(m):
    a = 0.5 * (m - m.conj().T)
    return a - np.trace(a) / 3.0 * np.eye(3)


def gell_mann():
    l = np.zeros((8, 3, 3), complex)
    l[0][0, 1] = l[0][1, 0] = 1
    l[1][0, 1], l[1][1, 0] = -1j, 1j
    l[2][0, 0], l[2][1, 1] = 1, -1
    l[3][0, 2] = l[3][2, 0] = 1
    l[4][0, 2], l[4][2, 0] = -1j, 1j
    l[5][1, 2] = l[5][2, 1] = 1
    l[6][1, 2], l[6][2, 1] = -1j, 1j
    l[7] = np.diag([1, 1, -2]) / np.sqrt(3)
    return l / 2  # Hermitian, traceless, Tr(T_a T_b) = delta_ab / 2


def action(oracle, U, chi, psi, sign):
    return oracle.dot(DIMS, chi, oracle.eo_apply(DIMS, U, KAPPA, psi, sign), oracle.EVEN).real


@pytest.mark.parametrize("sign", [1, -1])
def test_oracle_force_finite_difference(oracle, sign):
    U = oracle.gen_links(DIMS, 0.3, 41)
    chi = oracle.gen_spinor(DIMS, 42, oracle.EVEN)
    psi = oracle.gen_spinor(DIMS, 43, oracle.EVEN)
    F = _c(oracle.eo_force(DIMS, U, KAPPA, chi, psi, sign))
    T = gell_mann()
    eps = 1e-5
    rng = np.random.default_rng(7)
    V = oracle.volume(DIMS)
    checked = 0
    for _ in range(6):
        d, site, a = int(rng.integers(4)), int(rng.integers(V)), int(rng.integers(8))
        u0 = _c(U[d, site]).copy()
        f2 = np.trace(project_antihermitean(u0 @ F[d, site]) @ (1j * T[a])).real
        s = []
        for e in (eps, -eps):
            Up = U.copy()
            Up[d, site] = _r((np.eye(3) + 1j * e * T[a]) @ u0)
            s.append(action(oracle, Up, chi, psi, sign))
        f1 = (s[0] - s[1]) / (2 * eps)
        assert abs(f1 - f2) <= 1e-6 * max(1.0, abs(f1)), (d, site, a, f1, f2)
        checked += 1
    assert checked == 6


def test_oracle_force_parities(oracle):
    """Every link gets a force: the even-site and the odd-site terms are both non-zero."""
    U = oracle.gen_links(DIMS, 0.3, 44)
    chi = oracle.gen_spinor(DIMS, 45, oracle.EVEN)
    psi = oracle.gen_spinor(DIMS, 46, oracle.EVEN)
    F = _c(oracle.eo_force(DIMS, U, KAPPA, chi, psi, 1))
    n = np.abs(F).reshape(4, -1, 9).sum(axis=2)
    assert (n > 0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("dims,lf", [((4, 4, 4, 6), 18), ((8, 8, 8, 8), 12), ((6, 4, 4, 10), 18)])
@pytest.mark.parametrize("sign", [1, -1])
def test_gpu_force_matches_oracle(hw, ctx, oracle, dims, lf, sign):
    U = oracle.gen_links(dims, 0.3, 51)
    chi_h = oracle.gen_spinor(dims, 52, oracle.EVEN)
    psi_h = oracle.gen_spinor(dims, 53, oracle.EVEN)
    ref = oracle.eo_force(dims, U, KAPPA, chi_h, psi_h, sign)
    lat = hw.Lattice(ctx, dims, True)
    G = hw.GaugeField(lat, U, lf)
    chi, psi = hw.Field(lat, chi_h), hw.Field(lat, psi_h)
    D = hw.Dirac_Wilson_evenodd(KAPPA, G)
    got = D.force(chi, psi, sign)
    assert got.shape == ref.shape
    err = np.linalg.norm((got - ref).reshape(4, -1, 18), axis=2)
    scale = np.linalg.norm(ref.reshape(4, -1, 18), axis=2)
    assert (err <= 1e-13 * np.maximum(scale, 1e-300)).all(), float((err / np.maximum(scale, 1e-300)).max())
