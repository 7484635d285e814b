"""ctypes front end of the CPU oracle (``liboracle.so``) — TEST INFRASTRUCTURE ONLY.

The oracle restates HILA's Wilson even-odd operator and CG on the host (see
``wilson_oracle.cpp`` for the reference file:line each function follows).  The
test suite, the smoke check and the CPU-baseline leg of the bench use it as the
checker; nothing in the product library imports it.

Array conventions (numpy, float64):
  * spinor field: shape (V, 4, 3, 2) or any shape with V*24 doubles,
    lexicographic sites x + Lx*(y + Ly*(z + Lz*t)), [spin][colour][re,im]
  * gauge field:  shape (4, V, 3, 3, 2), row-major colour matrices
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

EVEN, ODD, ALL = 1, 2, 3

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "wilson_oracle.cpp"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        v = None
        sig = {
            "or_gen_links": (v, [_ip, ctypes.c_double, ctypes.c_uint64, _dp]),
            "or_unit_links": (v, [_ip, _dp]),
            "or_gen_spinor": (v, [_ip, ctypes.c_uint64, ctypes.c_int, _dp]),
            "or_gamma": (v, [ctypes.c_int, _dp, _dp]),
            "or_project": (v, [_dp, ctypes.c_int, ctypes.c_int, _dp]),
            "or_expand": (v, [_dp, ctypes.c_int, ctypes.c_int, _dp]),
            "or_mul_half": (v, [_dp, _dp, _dp]),
            "or_wilson_hop": (v, [_ip, ctypes.c_int, _dp, ctypes.c_double, _dp, _dp,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int]),
            "or_wilson_apply": (v, [_ip, ctypes.c_int, _dp, ctypes.c_double, _dp, _dp, ctypes.c_int]),
            "or_wilson_eo_apply": (v, [_ip, ctypes.c_int, _dp, ctypes.c_double, _dp, _dp, ctypes.c_int]),
            "or_wilson_eo_force": (v, [_ip, ctypes.c_int, _dp, ctypes.c_double, _dp, _dp, ctypes.c_int, _dp]),
            "or_staggered_hop": (v, [_ip, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int]),
            "or_staggered_eo_apply": (v, [_ip, ctypes.c_int, _dp, ctypes.c_double, _dp, _dp, ctypes.c_int]),
            "or_staggered_eo_force": (v, [_ip, ctypes.c_int, _dp, ctypes.c_double, _dp, _dp, ctypes.c_int, _dp]),
            "or_dot": (v, [_ip, _dp, _dp, ctypes.c_int, _dp, _dp]),
            "or_squarenorm": (ctypes.c_double, [_ip, _dp, ctypes.c_int]),
            "or_cg": (ctypes.c_int, [_ip, ctypes.c_int, _dp, ctypes.c_double, _dp, _dp,
                                     ctypes.c_double, ctypes.c_int, _dp]),
            "or_true_residual": (ctypes.c_double, [_ip, ctypes.c_int, _dp, ctypes.c_double, _dp, _dp,
                                                   ctypes.c_int]),
            "or_true_residual_normal": (ctypes.c_double, [_ip, ctypes.c_int, _dp, ctypes.c_double,
                                                          _dp, _dp]),
            "or_ref_create": (ctypes.c_void_p, [_ip, ctypes.c_int]),
            "or_ref_destroy": (v, [ctypes.c_void_p]),
            "or_ref_eo_apply": (v, [ctypes.c_void_p, _dp, ctypes.c_double, _dp, _dp, ctypes.c_int]),
            "or_ref_cg": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_double, _dp, _dp,
                                         ctypes.c_double, ctypes.c_int, _dp]),
            "or_num_threads": (ctypes.c_int, []),
            "or_set_num_threads": (v, [ctypes.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def _dims(dims):
    return (ctypes.c_int * 4)(*[int(d) for d in dims])


def volume(dims) -> int:
    return int(np.prod(dims))


def gen_links(dims, eps: float, seed: int) -> np.ndarray:
    U = np.empty((4, volume(dims), 3, 3, 2), np.float64)
    lib().or_gen_links(_dims(dims), eps, seed, _d(U))
    return U


def unit_links(dims) -> np.ndarray:
    U = np.empty((4, volume(dims), 3, 3, 2), np.float64)
    lib().or_unit_links(_dims(dims), _d(U))
    return U


def gen_spinor(dims, seed: int, parity: int = ALL) -> np.ndarray:
    psi = np.empty((volume(dims), 4, 3, 2), np.float64)
    lib().or_gen_spinor(_dims(dims), seed, parity, _d(psi))
    return psi


def hop(dims, U, kappa, inp, out, par, sign, set_=True, antiperiodic=True):
    lib().or_wilson_hop(_dims(dims), int(antiperiodic), _d(U), kappa, _d(inp), _d(out), par, sign,
                        int(set_))
    return out


def wilson_apply(dims, U, kappa, inp, sign=1, antiperiodic=True):
    out = np.empty_like(inp)
    lib().or_wilson_apply(_dims(dims), int(antiperiodic), _d(U), kappa, _d(inp), _d(out), sign)
    return out


def eo_apply(dims, U, kappa, inp, sign=1, antiperiodic=True):
    out = np.zeros_like(inp)
    lib().or_wilson_eo_apply(_dims(dims), int(antiperiodic), _d(U), kappa, _d(inp), _d(out), sign)
    return out


def dot(dims, a, b, par=ALL) -> complex:
    re, im = ctypes.c_double(), ctypes.c_double()
    lib().or_dot(_dims(dims), _d(a), _d(b), par, ctypes.byref(re), ctypes.byref(im))
    return complex(re.value, im.value)


def squarenorm(dims, a, par=ALL) -> float:
    return lib().or_squarenorm(_dims(dims), _d(a), par)


def cg(dims, U, kappa, inp, out=None, acc=1e-12, maxiters=10000, antiperiodic=True):
    """CG<Dirac_Wilson_evenodd>::apply(in, out): solves M^dag M out = in on EVEN."""
    if out is None:
        out = np.zeros_like(inp)
    rr = ctypes.c_double()
    it = lib().or_cg(_dims(dims), int(antiperiodic), _d(U), kappa, _d(inp), _d(out), acc, maxiters,
                     ctypes.byref(rr))
    return out, it, rr.value


def eo_force(dims, U, kappa, chi, psi, sign=1, antiperiodic=True) -> np.ndarray:
    """Dirac_Wilson_evenodd::force (wilson.h:293-311): d Re(chi^dag M_s psi) / d links,
    as [4][V][3][3] complex (shape (4, V, 3, 3, 2))."""
    chi = np.ascontiguousarray(chi, np.float64)
    psi = np.ascontiguousarray(psi, np.float64)
    out = np.zeros((4, volume(dims), 3, 3, 2))
    lib().or_wilson_eo_force(_dims(dims), int(antiperiodic), _d(U), kappa, _d(chi), _d(psi), sign, _d(out))
    return out


def hasenbusch_eo_apply(dims, U, kappa, mh, inp, sign=1, antiperiodic=True):
    """Hasenbusch_operator::apply / dagger (Hasenbusch.h:39-47): (M_s + m_h) inp on EVEN."""
    out = eo_apply(dims, U, kappa, inp, sign, antiperiodic)
    even = parity_mask(dims) == 0
    out[even] += mh * inp[even]
    return out


def parity_mask(dims) -> np.ndarray:
    """(x + y + z + t) mod 2 per lexicographic site."""
    x, y, z, t = np.meshgrid(*[np.arange(d) for d in dims], indexing="ij")
    return ((x + y + z + t) % 2).transpose(3, 2, 1, 0).reshape(-1)


def mre_guess(dims, U, kappa, mh, old, chi, antiperiodic=True) -> np.ndarray:
    """MRE_guess (MRE_guess.h:9-88) with the intended Gram-Schmidt (overlap over |b_j|^2)
    and accumulation psi = sum_i v_i b_i; real inner products over EVEN (rdot)."""
    even = parity_mask(dims) == 0

    def rdot(a, b):
        return float(np.sum(a[even] * b[even]))

    def A(v):
        w = hasenbusch_eo_apply(dims, U, kappa, mh, v, +1, antiperiodic)
        return hasenbusch_eo_apply(dims, U, kappa, mh, w, -1, antiperiodic)

    n = len(old)
    basis = []
    for i in range(n):
        b = np.array(old[i], np.float64, copy=True)
        b[~even] = 0.0
        for bj in basis:
            nj = rdot(bj, bj)
            if nj > 1e-300:
                b -= rdot(bj, b) / nj * bj
        basis.append(b)
    M = np.zeros((n, n))
    v = np.zeros(n)
    for i in range(n):
        Ab = A(basis[i])
        for j in range(n):
            M[j, i] = rdot(basis[j], Ab)
        v[i] = rdot(basis[i], chi)
    for i in range(n):  # Gauss-Jordan as MRE_guess.h:55-80
        if M[i, i] * M[i, i] > 1e-32:
            inv = 1.0 / M[i, i]
            M[i, :] *= inv
            v[i] *= inv
            for k in range(n):
                if k != i:
                    w = M[k, i]
                    M[k, :] -= w * M[i, :]
                    v[k] -= w * v[i]
        else:
            v[i] = 0.0
            M[:, i] = 0.0
    psi = np.zeros_like(np.asarray(chi, np.float64))
    for i in range(n):
        if np.isfinite(v[i]) and v[i] != 0.0:
            psi += v[i] * basis[i]
    return psi


def staggered_eo_apply(dims, U, mass, inp, sign=1, antiperiodic=True) -> np.ndarray:
    """dirac_staggered_evenodd::apply / dagger (staggered.h:224-242) on colour-vector fields
    (V, 3, 2); out[ODD] keeps (1/m) D_oe in as the reference leaves it."""
    inp = np.ascontiguousarray(inp, np.float64)
    out = np.zeros_like(inp)
    lib().or_staggered_eo_apply(_dims(dims), int(antiperiodic), _d(U), mass, _d(inp), _d(out), sign)
    return out


def staggered_eo_force(dims, U, mass, chi, psi, sign=1, antiperiodic=True) -> np.ndarray:
    """dirac_staggered_evenodd::force (staggered.h:246-265), shape (4, V, 3, 3, 2)."""
    chi = np.ascontiguousarray(chi, np.float64)
    psi = np.ascontiguousarray(psi, np.float64)
    out = np.zeros((4, volume(dims), 3, 3, 2))
    lib().or_staggered_eo_force(_dims(dims), int(antiperiodic), _d(U), mass, _d(chi), _d(psi), sign, _d(out))
    return out


def gen_colour_vector(dims, seed: int, parity: int = ALL) -> np.ndarray:
    """Gaussian colour-vector field (V, 3, 2), zero outside `parity` (tests only)."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((volume(dims), 3, 2))
    if parity != ALL:
        v[parity_mask(dims) != (0 if parity == EVEN else 1)] = 0.0
    return v


def true_residual(dims, U, kappa, b, x, sign=1, antiperiodic=True) -> float:
    return lib().or_true_residual(_dims(dims), int(antiperiodic), _d(U), kappa, _d(b), _d(x), sign)


def true_residual_normal(dims, U, kappa, b, x, antiperiodic=True) -> float:
    return lib().or_true_residual_normal(_dims(dims), int(antiperiodic), _d(U), kappa, _d(b), _d(x))


def gamma(g: int, w: np.ndarray) -> np.ndarray:
    w = np.ascontiguousarray(w, np.float64)
    out = np.empty_like(w)
    lib().or_gamma(g, _d(w), _d(out))
    return out


def project(w, dir_, sign):
    w = np.ascontiguousarray(w, np.float64)
    h = np.empty((2, 3, 2), np.float64)
    lib().or_project(_d(w), dir_, sign, _d(h))
    return h


def expand(h, dir_, sign):
    h = np.ascontiguousarray(h, np.float64)
    w = np.empty((4, 3, 2), np.float64)
    lib().or_expand(_d(h), dir_, sign, _d(w))
    return w


def mul_half(U, h):
    U = np.ascontiguousarray(U, np.float64)
    h = np.ascontiguousarray(h, np.float64)
    out = np.empty((2, 3, 2), np.float64)
    lib().or_mul_half(_d(U), _d(h), _d(out))
    return out


class RefStructured:
    """The operator in the reference's loop structure (timed CPU baseline)."""

    def __init__(self, dims, antiperiodic=True):
        self.dims = tuple(dims)
        self.ws = lib().or_ref_create(_dims(dims), int(antiperiodic))

    def eo_apply(self, U, kappa, inp, out, sign=1):
        lib().or_ref_eo_apply(self.ws, _d(U), kappa, _d(inp), _d(out), sign)
        return out

    def cg(self, U, kappa, inp, out, acc, maxiters):
        rr = ctypes.c_double()
        it = lib().or_ref_cg(self.ws, _d(U), kappa, _d(inp), _d(out), acc, maxiters, ctypes.byref(rr))
        return it, rr.value

    def close(self):
        if self.ws:
            lib().or_ref_destroy(self.ws)
            self.ws = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def num_threads() -> int:
    return lib().or_num_threads()


def set_num_threads(n: int) -> None:
    lib().or_set_num_threads(n)


def to_complex_spinor(a: np.ndarray) -> np.ndarray:
    """(V,4,3,2) float64 -> (V,4,3) complex128 view-copy."""
    a = a.reshape(-1, 4, 3, 2)
    return a[..., 0] + 1j * a[..., 1]


def to_complex_links(U: np.ndarray) -> np.ndarray:
    U = U.reshape(4, -1, 3, 3, 2)
    return U[..., 0] + 1j * U[..., 1]
