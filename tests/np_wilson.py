"""Independent numpy restatement of the Wilson hopping term (test helper).

Written from the gamma-matrix definitions rather than the half-spinor
projection tables the C++ oracle uses, so that agreement between the two
checks the projection/expansion tables themselves:

    (H_s psi)(x) = sum_mu (1 + s gamma_mu) U_mu(x) psi(x+mu)
                        + (1 - s gamma_mu) U_mu(x-mu)^dagger psi(x-mu)

Gamma matrices as HILA defines them (libraries/datatypes/wilson_vector.h:311-347),
direction map x->gamma1, y->gamma2, z->gamma3, t->gamma0 (wilson_vector.h:23).
Fermion values that cross the t boundary are negated when antiperiodic
(libraries/plumbing/field_comm.h:28-41).
"""
from __future__ import annotations

import numpy as np

I = 1j
GAMMA = {
    0: np.array([[0, 0, 1, 0], [0, 0, 0, 1], [1, 0, 0, 0], [0, 1, 0, 0]], complex),
    1: np.array([[0, 0, 0, I], [0, 0, I, 0], [0, -I, 0, 0], [-I, 0, 0, 0]], complex),
    2: np.array([[0, 0, 0, -1], [0, 0, 1, 0], [0, 1, 0, 0], [-1, 0, 0, 0]], complex),
    3: np.array([[0, 0, I, 0], [0, 0, 0, -I], [-I, 0, 0, 0], [0, I, 0, 0]], complex),
    5: np.diag([1, 1, -1, -1]).astype(complex),
}
DIR_GAMMA = [1, 2, 3, 0]  # x, y, z, t
AXIS = [3, 2, 1, 0]  # numpy axis of (t, z, y, x) grids for directions x, y, z, t


def to_grid(psi: np.ndarray, dims) -> np.ndarray:
    """(V,4,3,2) float64 lexicographic -> (Lt,Lz,Ly,Lx,4,3) complex."""
    Lx, Ly, Lz, Lt = dims
    c = psi.reshape(-1, 4, 3, 2)
    c = c[..., 0] + 1j * c[..., 1]
    return c.reshape(Lt, Lz, Ly, Lx, 4, 3)


def from_grid(g: np.ndarray) -> np.ndarray:
    out = np.empty(g.shape + (2,), np.float64)
    out[..., 0] = g.real
    out[..., 1] = g.imag
    return out.reshape(-1, 4, 3, 2)


def links_to_grid(U: np.ndarray, dims) -> np.ndarray:
    Lx, Ly, Lz, Lt = dims
    c = U.reshape(4, -1, 3, 3, 2)
    c = c[..., 0] + 1j * c[..., 1]
    return c.reshape(4, Lt, Lz, Ly, Lx, 3, 3)


def shift(f: np.ndarray, mu: int, step: int, antiperiodic: bool) -> np.ndarray:
    """f(x + step*mu) with the fermion t-boundary sign."""
    ax = AXIS[mu]
    g = np.roll(f, -step, axis=ax)
    if mu == 3 and antiperiodic:
        idx = [slice(None)] * g.ndim
        idx[ax] = -1 if step > 0 else 0
        g[tuple(idx)] *= -1
    return g


def hop(Ug: np.ndarray, psig: np.ndarray, sign: int, antiperiodic: bool = True) -> np.ndarray:
    out = np.zeros_like(psig)
    one = np.eye(4)
    for mu in range(4):
        gm = GAMMA[DIR_GAMMA[mu]]
        pf = one + sign * gm
        pb = one - sign * gm
        fwd = shift(psig, mu, +1, antiperiodic)
        Ufwd = np.einsum("...ij,...sj->...si", Ug[mu], fwd)
        out += np.einsum("st,...tc->...sc", pf, Ufwd)
        Um = shift(Ug[mu], mu, -1, False)  # U_mu(x - mu), links periodic
        bwd = shift(psig, mu, -1, antiperiodic)
        Ubwd = np.einsum("...ji,...sj->...si", Um.conj(), bwd)
        out += np.einsum("st,...tc->...sc", pb, Ubwd)
    return out


def parity_mask(dims) -> np.ndarray:
    Lx, Ly, Lz, Lt = dims
    t, z, y, x = np.meshgrid(np.arange(Lt), np.arange(Lz), np.arange(Ly), np.arange(Lx), indexing="ij")
    return ((x + y + z + t) % 2).astype(np.int64)


def eo_apply(Ug, psig, kappa, sign, dims, antiperiodic=True):
    """M_s psi_e = psi_e - kappa^2 H^{eo} H^{oe} psi_e on EVEN; zero on ODD."""
    par = parity_mask(dims)
    even = (par == 0)[..., None, None]
    pe = np.where(even, psig, 0)
    t = hop(Ug, pe, sign, antiperiodic)
    t = np.where(even, 0, t)
    out = pe - kappa * kappa * hop(Ug, t, sign, antiperiodic)
    return np.where(even, out, 0)
