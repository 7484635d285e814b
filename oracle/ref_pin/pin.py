"""ctypes wrapper of the pin library (oracle/_ref/libref_pin.so, built by oracle/ref_pin/Makefile
from the reference's own sources).  Test infrastructure: used to generate the reference
golden fixtures in tests/golden/ and, where the library has been built, to check that they
can be regenerated."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(os.path.dirname(HERE), "_ref", "libref_pin.so")
REFERENCE = os.environ.get("HILA_REFERENCE", "/root/reference")

_lib = None


def reference_present() -> bool:
    return os.path.isfile(os.path.join(REFERENCE, "libraries", "datatypes", "wilson_vector.h"))


def build() -> str:
    """Build the pin library (needs the reference sources)."""
    if not reference_present():
        raise FileNotFoundError(f"reference sources not found under {REFERENCE}")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE}"], check=True)
    return LIB


def available() -> bool:
    return os.path.isfile(LIB)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB)
        vp, i, d, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_uint64
        sig = {"rp_gaussrand": [u64, i, vp], "rp_gen_links": [vp, d, u64, vp], "rp_gen_spinor": [vp, u64, i, vp],
               "rp_project": [vp, i, i, vp], "rp_expand": [vp, i, i, vp], "rp_gamma": [i, vp, vp],
               "rp_hop": [vp, i, vp, d, vp, vp, i, i, i], "rp_eo_apply": [vp, i, vp, d, vp, vp, i]}
        for name, args in sig.items():
            f = getattr(_lib, name)
            f.argtypes, f.restype = args, i
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


def _dims(dims):
    return (ctypes.c_int * 4)(*dims)


def _ok(rc):
    if rc != 0:
        raise ValueError(f"pin library call failed ({rc})")


def gaussrand(seed: int, n: int) -> np.ndarray:
    out = np.empty(n)
    _ok(lib().rp_gaussrand(seed, n, _p(out)))
    return out


def gen_links(dims, eps: float, seed: int) -> np.ndarray:
    U = np.empty((4, int(np.prod(dims)), 3, 3, 2))
    _ok(lib().rp_gen_links(_dims(dims), eps, seed, _p(U)))
    return U


def gen_spinor(dims, seed: int, parity_mask: int) -> np.ndarray:
    s = np.empty((int(np.prod(dims)), 4, 3, 2))
    _ok(lib().rp_gen_spinor(_dims(dims), seed, parity_mask, _p(s)))
    return s


def project(w, dir_: int, sign: int) -> np.ndarray:
    h = np.empty((2, 3, 2))
    _ok(lib().rp_project(_p(np.ascontiguousarray(w, np.float64)), dir_, sign, _p(h)))
    return h


def expand(h, dir_: int, sign: int) -> np.ndarray:
    w = np.empty((4, 3, 2))
    _ok(lib().rp_expand(_p(np.ascontiguousarray(h, np.float64)), dir_, sign, _p(w)))
    return w


def gamma(g: int, w) -> np.ndarray:
    out = np.empty((4, 3, 2))
    _ok(lib().rp_gamma(g, _p(np.ascontiguousarray(w, np.float64)), _p(out)))
    return out


def hop(dims, U, kappa: float, inp, par: int, sign: int, antiperiodic: bool = True) -> np.ndarray:
    out = np.zeros_like(inp)
    _ok(lib().rp_hop(_dims(dims), int(antiperiodic), _p(U), kappa, _p(inp), _p(out), par, sign, 1))
    return out


def eo_apply(dims, U, kappa: float, inp, sign: int, antiperiodic: bool = True) -> np.ndarray:
    out = np.zeros_like(inp)
    _ok(lib().rp_eo_apply(_dims(dims), int(antiperiodic), _p(U), kappa, _p(inp), _p(out), sign))
    return out
