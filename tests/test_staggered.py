"""Staggered even-odd operator (staggered.h), its force and CG, against the oracle.

The oracle is pinned by the reference's identities: M^dag is the adjoint of M,
for this operator M^dag = M on EVEN (D is anti-Hermitian, so the two signs of
D_eo D_oe agree), and the force passes the finite-difference check of
test_forces.cpp:15-100 (staggered cases at :265-277).  As written the operator
is m - (1/m) D_oe^dag D_oe (the Schur complement of m + D would carry the other
sign), so it is Hermitian but positive only at large mass."""
import numpy as np
import pytest

DIMS = (4, 4, 4, 6)
MASS = 0.2


def _c(a):
    return a[..., 0] + 1j * a[..., 1]


def _even(oracle, dims):
    return oracle.parity_mask(dims) == 0


def test_oracle_staggered_identities(oracle):
    U = oracle.gen_links(DIMS, 0.3, 201)
    a = oracle.gen_colour_vector(DIMS, 202, oracle.EVEN)
    b = oracle.gen_colour_vector(DIMS, 203, oracle.EVEN)
    ev = _even(oracle, DIMS)
    Mb = oracle.staggered_eo_apply(DIMS, U, MASS, b, 1)
    Mda = oracle.staggered_eo_apply(DIMS, U, MASS, a, -1)
    lhs = np.vdot(_c(a)[ev], _c(Mb)[ev])
    rhs = np.vdot(_c(Mda)[ev], _c(b)[ev])
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    Mdb = oracle.staggered_eo_apply(DIMS, U, MASS, b, -1)
    assert np.array_equal(Mb[ev], Mdb[ev])
    assert np.allclose(Mb[~ev], -Mdb[~ev], rtol=0, atol=1e-14)  # the ODD intermediate flips sign
    # Hermitian: <b, M b> is real
    assert abs(np.vdot(_c(b)[ev], _c(Mb)[ev]).imag) <= 1e-12 * abs(np.vdot(_c(b)[ev], _c(Mb)[ev]))


def _pah(m):
    a = 0.5 * (m - m.conj().T)
    return a - np.trace(a) / 3.0 * np.eye(3)


@pytest.mark.parametrize("sign", [1, -1])
def test_oracle_staggered_force_finite_difference(oracle, sign):
    from tests.test_force import gell_mann
    U = oracle.gen_links(DIMS, 0.3, 211)
    chi = oracle.gen_colour_vector(DIMS, 212, oracle.EVEN)
    psi = oracle.gen_colour_vector(DIMS, 213, oracle.EVEN)
    ev = _even(oracle, DIMS)
    F = _c(oracle.staggered_eo_force(DIMS, U, MASS, chi, psi, sign))
    T = gell_mann()
    rng = np.random.default_rng(9)
    eps = 1e-5

    def S(Uc):
        return np.vdot(_c(chi)[ev], _c(oracle.staggered_eo_apply(DIMS, Uc, MASS, psi, sign))[ev]).real

    for _ in range(6):
        d, site, a = int(rng.integers(4)), int(rng.integers(oracle.volume(DIMS))), int(rng.integers(8))
        u0 = _c(U[d, site]).copy()
        f2 = np.trace(_pah(u0 @ F[d, site]) @ (1j * T[a])).real
        s = []
        for e in (eps, -eps):
            Up = U.copy()
            m = (np.eye(3) + 1j * e * T[a]) @ u0
            Up[d, site] = np.stack([m.real, m.imag], axis=-1)
            s.append(S(Up))
        f1 = (s[0] - s[1]) / (2 * eps)
        assert abs(f1 - f2) <= 1e-6 * max(1.0, abs(f1)), (d, site, a, f1, f2)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,lf", [((4, 4, 4, 6), 18), ((8, 8, 8, 8), 12), ((6, 4, 4, 10), 12)])
@pytest.mark.parametrize("sign", [1, -1])
def test_gpu_staggered_apply(hw, ctx, oracle, dims, lf, sign):
    U = oracle.gen_links(dims, 0.3, 221)
    inp = oracle.gen_colour_vector(dims, 222, oracle.EVEN)
    ref = oracle.staggered_eo_apply(dims, U, MASS, inp, sign)
    lat = hw.Lattice(ctx, dims, True)
    G = hw.GaugeField(lat, U, lf)
    D = hw.dirac_staggered_evenodd(MASS, G)
    fi, fo = hw.StaggeredField(lat, inp), hw.StaggeredField(lat)
    (D.apply if sign > 0 else D.dagger)(fi, fo)
    got = fo.download()
    err = np.linalg.norm((got - ref).reshape(-1, 6), axis=1)
    assert (err <= 1e-13 * np.maximum(np.linalg.norm(ref.reshape(-1, 6), axis=1), 1e-300)).all()


@pytest.mark.gpu
@pytest.mark.parametrize("sign", [1, -1])
def test_gpu_staggered_force(hw, ctx, oracle, sign):
    dims = (8, 8, 8, 8)
    U = oracle.gen_links(dims, 0.3, 231)
    chi_h = oracle.gen_colour_vector(dims, 232, oracle.EVEN)
    psi_h = oracle.gen_colour_vector(dims, 233, oracle.EVEN)
    ref = oracle.staggered_eo_force(dims, U, MASS, chi_h, psi_h, sign)
    lat = hw.Lattice(ctx, dims, True)
    D = hw.dirac_staggered_evenodd(MASS, hw.GaugeField(lat, U, 18))
    got = D.force(hw.StaggeredField(lat, chi_h), hw.StaggeredField(lat, psi_h), sign)
    err = np.linalg.norm((got - ref).reshape(4, -1, 18), axis=2)
    scale = np.linalg.norm(ref.reshape(4, -1, 18), axis=2)
    assert (err <= 1e-13 * np.maximum(scale, 1e-300)).all()


@pytest.mark.gpu
def test_gpu_staggered_cg(hw, ctx, oracle):
    """CG on M^dag M at the reference's test mass (test_forces.cpp:265): the operator as
    the reference writes it is m - (1/m) D_oe^dag D_oe, positive only for m^2 above the
    largest eigenvalue of D_oe^dag D_oe, so a small mass leaves it indefinite and CG on
    its square does not reach 1e-10."""
    dims, mass = (8, 8, 8, 8), 5.0
    U = oracle.gen_links(dims, 0.3, 241)
    b = oracle.gen_colour_vector(dims, 242, oracle.EVEN)
    lat = hw.Lattice(ctx, dims, True)
    D = hw.dirac_staggered_evenodd(mass, hw.GaugeField(lat, U, 12))
    fb, fx = hw.StaggeredField(lat, b), hw.StaggeredField(lat)
    r = D.cg(fb, fx, accuracy=1e-10, true_residual=True)
    assert r.converged and r.iterations > 0
    x = fx.download()
    Mx = oracle.staggered_eo_apply(dims, U, mass, x, 1)
    Mx[~_even(oracle, dims)] = 0.0
    MMx = oracle.staggered_eo_apply(dims, U, mass, Mx, -1)
    ev = _even(oracle, dims)
    assert np.linalg.norm((b - MMx)[ev]) <= 1e-10 * np.linalg.norm(b[ev])
    assert not np.any(x[~ev])
