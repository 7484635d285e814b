"""hila_b200 — B200-native Wilson-fermion solve path with HILA's interface.

Python mirror of the reference's operator/solver API over the C ABI in
``include/hila_b200.h`` (``libhila_b200.so``, built by ``hila_b200.build``):

    =====================================  ===========================================
    reference (C++)                        here
    =====================================  ===========================================
    lattice.setup(size)                    Lattice(ctx, dims, antiperiodic=True)
    Field<SU<3,double>> U[NDIM]            GaugeField(lattice, links)
    Field<Wilson_vector<3,double>>         Field(lattice)
    Dirac_Wilson_evenodd<SU<3>> D(k, U)    Dirac_Wilson_evenodd(kappa, gauge)
    D.apply(in, out) / D.dagger(in, out)   same
    Dirac_Wilson<SU<3>> D(k, U)            Dirac_Wilson(kappa, gauge)
    CG<Op> inv(D[, acc[, maxiters]])       CG(D, accuracy=1e-12, maxiters=10000)
    inv.apply(in, out)                     same; returns a CGResult
    =====================================  ===========================================

(libraries/dirac/wilson.h:146-312, libraries/dirac/conjugate_gradient.h:18-104.)

There is no CPU fallback: every operator call runs the CUDA kernels, and the
module raises ImportError when the library has not been built.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhila_b200.so")

HW_OK = 0
HW_ERR_INVALID = -1
HW_ERR_OOM = -2
HW_ERR_CUDA = -3
HW_ERR_NOT_CONVERGED = -4
HW_ERR_BREAKDOWN = -5
HW_ERR_TIMEOUT = -6
HW_ERR_REJECTED = -7
HW_ERR_CANCELLED = -8
HW_ERR_NO_DEVICE = -9

EVEN, ODD, ALL = 1, 2, 3
PREC_F64, PREC_F32, PREC_F16 = 0, 1, 2
PRECISIONS = {"f64": PREC_F64, "f32": PREC_F32, "f16": PREC_F16}

_STATUS_NAMES = {
    HW_OK: "ok", HW_ERR_INVALID: "invalid argument", HW_ERR_OOM: "out of device memory",
    HW_ERR_CUDA: "CUDA error", HW_ERR_NOT_CONVERGED: "not converged", HW_ERR_BREAKDOWN: "CG breakdown",
    HW_ERR_TIMEOUT: "device wait timed out", HW_ERR_REJECTED: "rejected", HW_ERR_CANCELLED: "cancelled",
    HW_ERR_NO_DEVICE: "no CUDA device",
}


class HilaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class _CgParams(ctypes.Structure):
    _fields_ = [("accuracy", ctypes.c_double), ("maxiters", ctypes.c_int), ("precision", ctypes.c_int),
                ("delta", ctypes.c_double), ("true_residual", ctypes.c_int), ("use_graph", ctypes.c_int),
                ("hasenbusch_mh", ctypes.c_double)]


class _CgResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iterations", ctypes.c_int), ("reliable_updates", ctypes.c_int),
                ("restarts", ctypes.c_int), ("rr_relative", ctypes.c_double), ("true_residual", ctypes.c_double),
                ("seconds", ctypes.c_double), ("kernel_launches", ctypes.c_int)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("delta", ctypes.c_double), ("hbm_budget_bytes", ctypes.c_size_t),
                ("chunk_iters", ctypes.c_int), ("host_pool_bytes", ctypes.c_size_t),
                ("staggered_precision", ctypes.c_int)]


class _RequestResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("nrhs", ctypes.c_int), ("iterations", ctypes.c_int),
                ("reliable_updates", ctypes.c_int), ("true_residual", ctypes.c_double),
                ("latency_seconds", ctypes.c_double), ("queue_seconds", ctypes.c_double),
                ("admit_chunk", ctypes.c_uint64), ("retire_chunk", ctypes.c_uint64)]


class _EngineProfile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int * 12), ("ms", ctypes.c_double * 12),
                ("work", (ctypes.c_uint64 * 4) * 12)]


class _EngineTuning(ctypes.Structure):
    _fields_ = [("work_class", ctypes.c_int), ("nshapes", ctypes.c_int), ("variant", ctypes.c_int * 4),
                ("dynamic_order", ctypes.c_int * 4), ("ms_per_iteration", ctypes.c_double * 4),
                ("samples", ctypes.c_int * 4), ("chosen", ctypes.c_int)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("cancelled", ctypes.c_uint64), ("running", ctypes.c_uint64), ("queued", ctypes.c_uint64),
                ("bytes_in_use", ctypes.c_size_t), ("bytes_budget", ctypes.c_size_t),
                ("latency_p50_seconds", ctypes.c_double), ("latency_p99_seconds", ctypes.c_double),
                ("solves_completed", ctypes.c_uint64), ("chunks", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64), ("seconds_admit", ctypes.c_double),
                ("seconds_run", ctypes.c_double), ("seconds_retire", ctypes.c_double),
                ("max_admit_seconds", ctypes.c_double), ("max_launch_seconds", ctypes.c_double),
                ("max_retire_seconds", ctypes.c_double)]


class _SolveRequest(ctypes.Structure):
    _fields_ = [("gauge", ctypes.c_void_p), ("kappa", ctypes.c_double), ("b", ctypes.c_void_p),
                ("x", ctypes.c_void_p), ("accuracy", ctypes.c_double), ("maxiters", ctypes.c_int),
                ("hasenbusch_mh", ctypes.c_double)]


class _StagSolveRequest(ctypes.Structure):
    _fields_ = [("gauge", ctypes.c_void_p), ("mass", ctypes.c_double), ("inp", ctypes.c_void_p),
                ("out", ctypes.c_void_p), ("accuracy", ctypes.c_double), ("maxiters", ctypes.c_int),
                ("normal", ctypes.c_int), ("precision", ctypes.c_int), ("delta", ctypes.c_double)]


_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_SIGNATURES = {
    "hw_api_version": (ctypes.c_int, []),
    "hw_last_error": (ctypes.c_char_p, []),
    "hw_device_count": (ctypes.c_int, [_ip]),
    "hw_context_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "hw_context_destroy": (ctypes.c_int, [_vp]),
    "hw_context_synchronize": (ctypes.c_int, [_vp]),
    "hw_context_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "hw_engine_profile_enable": (ctypes.c_int, [_vp, ctypes.c_int]),
    "hw_engine_profile_get": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "hw_engine_tuning_get": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "hw_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(_vp)]),
    "hw_host_free": (ctypes.c_int, [_vp]),
    "hw_lattice_create": (ctypes.c_int, [_vp, _ip, ctypes.c_int, ctypes.POINTER(_vp)]),
    "hw_lattice_destroy": (ctypes.c_int, [_vp]),
    "hw_lattice_volume": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "hw_gauge_create": (ctypes.c_int, [_vp, _dp, ctypes.c_int, ctypes.POINTER(_vp)]),
    "hw_gauge_destroy": (ctypes.c_int, [_vp]),
    "hw_field_create": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "hw_field_destroy": (ctypes.c_int, [_vp]),
    "hw_field_upload": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    "hw_field_upload_eo": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    "hw_field_download_eo": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    "hw_field_download": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    "hw_field_zero": (ctypes.c_int, [_vp, ctypes.c_int]),
    "hw_wilson_evenodd_apply": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp]),
    "hw_wilson_evenodd_dagger": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp]),
    "hw_wilson_evenodd_force": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp, ctypes.c_int, _dp]),
    "hw_hasenbusch_evenodd_apply": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _vp, _vp]),
    "hw_hasenbusch_evenodd_dagger": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _vp, _vp]),
    "hw_mre_guess": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.POINTER(_vp), ctypes.c_int, _vp,
                                    _vp]),
    "hw_stag_field_create": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "hw_stag_field_destroy": (ctypes.c_int, [_vp]),
    "hw_stag_field_upload": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    "hw_stag_field_download": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
    "hw_stag_field_zero": (ctypes.c_int, [_vp, ctypes.c_int]),
    "hw_staggered_evenodd_apply": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp]),
    "hw_staggered_evenodd_dagger": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp]),
    "hw_staggered_evenodd_force": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp, ctypes.c_int, _dp]),
    "hw_staggered_cg_solve": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp, _vp, _vp]),
    "hw_staggered_batch_solve": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp]),
    "hw_server_submit_staggered": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                  ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.c_double,
                                                  ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]),
    "hw_gauge_config_dims": (ctypes.c_int, [ctypes.c_char_p, _ip]),
    "hw_gauge_config_write": (ctypes.c_int, [ctypes.c_char_p, _ip, _dp]),
    "hw_gauge_config_read": (ctypes.c_int, [ctypes.c_char_p, _ip, _dp]),
    "hw_wilson_apply": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int, _vp, _vp]),
    "hw_wilson_cg_solve": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp, _vp, _vp]),
    "hw_wilson_hop": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "hw_cg_params_default": (None, [ctypes.POINTER(_CgParams)]),
    "hw_cg_solve": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp, ctypes.POINTER(_CgParams),
                                   ctypes.POINTER(_CgResult)]),
    "hw_wilson_evenodd_solve": (ctypes.c_int, [_vp, ctypes.c_double, _vp, _vp, ctypes.POINTER(_CgParams),
                                               ctypes.POINTER(_CgResult)]),
    "hw_wilson_evenodd_solve_host": (ctypes.c_int, [_vp, ctypes.c_double, _dp, _dp, ctypes.POINTER(_CgParams),
                                                    ctypes.POINTER(_CgResult)]),
    "hw_wilson_evenodd_apply_noalloc": (ctypes.c_int, [_ip, ctypes.c_int, ctypes.c_double, ctypes.c_int, _vp,
                                                       ctypes.c_int, _vp, _vp, ctypes.c_int, _vp]),
    "hw_batch_solve": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.POINTER(_SolveRequest),
                                      ctypes.c_int, ctypes.POINTER(_CgResult)]),
    "hw_server_create": (ctypes.c_int, [_vp, ctypes.POINTER(_ServerConfig), ctypes.POINTER(_vp)]),
    "hw_server_destroy": (ctypes.c_int, [_vp]),
    "hw_server_add_gauge": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_int)]),
    "hw_server_submit": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(_dp),
                                        ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]),
    "hw_server_wait": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.POINTER(_dp), ctypes.c_double,
                                      ctypes.POINTER(_RequestResult)]),
    "hw_server_submit_eo": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(_dp),
                                           ctypes.POINTER(_dp), ctypes.c_double, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_uint64)]),
    "hw_server_submit_fields": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                               ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.c_double,
                                               ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]),
    "hw_server_cancel": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "hw_server_stats_get": (ctypes.c_int, [_vp, ctypes.POINTER(_ServerStats)]),
    "hw_generate_links": (ctypes.c_int, [_ip, ctypes.c_double, ctypes.c_uint64, _dp]),
    "hw_generate_spinor": (ctypes.c_int, [_ip, ctypes.c_uint64, ctypes.c_int, _dp]),
}

_lib = None


API_VERSION = 2  # HW_API_VERSION of include/hila_b200.h whose structs this binding mirrors


def load_library() -> ctypes.CDLL:
    """Load libhila_b200.so; raises ImportError if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m hila_b200.build` "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        if L.hw_api_version() != API_VERSION:
            raise ImportError(f"{LIB_PATH} has API version {L.hw_api_version()}, this binding expects "
                              f"{API_VERSION}: rebuild it with `python -m hila_b200.build`")
        _lib = L
    return _lib


def lib() -> ctypes.CDLL:
    return load_library()


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def _check(rc: int) -> int:
    if rc != HW_OK:
        raise HilaError(rc, lib().hw_last_error().decode(errors="replace"))
    return rc


def _dims(dims):
    return (ctypes.c_int * 4)(*[int(d) for d in dims])


def _dptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_dp)


def device_count() -> int:
    n = ctypes.c_int(0)
    rc = lib().hw_device_count(ctypes.byref(n))
    return n.value if rc == HW_OK else 0


# ------------------------------------------------------------------ inputs

def generate_links(dims, eps: float, seed: int) -> np.ndarray:
    """Seeded SU(3) links U = exp(i eps H), shape (4, V, 3, 3, 2) float64."""
    V = int(np.prod(dims))
    U = np.empty((4, V, 3, 3, 2), np.float64)
    _check(lib().hw_generate_links(_dims(dims), float(eps), int(seed), _dptr(U)))
    return U


def generate_spinor(dims, seed: int, parity: int = ALL) -> np.ndarray:
    """Seeded Gaussian Wilson spinor field, shape (V, 4, 3, 2) float64."""
    V = int(np.prod(dims))
    psi = np.empty((V, 4, 3, 2), np.float64)
    _check(lib().hw_generate_spinor(_dims(dims), int(seed), int(parity), _dptr(psi)))
    return psi


def eo_order(dims) -> np.ndarray:
    """Lexicographic site index of each position of HILA's even-first site order
    (lattice.cpp:171-184): EVEN sites in increasing lexicographic order, then ODD.
    `lex_array[eo_order(dims)]` is the array in even-first order."""
    Lx, Ly, Lz, Lt = dims
    lex = np.arange(Lx * Ly * Lz * Lt)
    par = (lex % Lx + (lex // Lx) % Ly + (lex // (Lx * Ly)) % Lz + lex // (Lx * Ly * Lz)) % 2
    return np.concatenate([lex[par == 0], lex[par == 1]])


class PinnedArray:
    """A float64 numpy array in page-locked host memory (hw_host_alloc)."""

    def __init__(self, shape):
        n = int(np.prod(shape))
        self._ptr = _vp()
        _check(lib().hw_host_alloc(n * 8, ctypes.byref(self._ptr)))
        buf = (ctypes.c_double * n).from_address(self._ptr.value)
        self.array = np.frombuffer(buf, np.float64).reshape(shape)

    def free(self):
        if self._ptr:
            lib().hw_host_free(self._ptr)
            self._ptr = _vp()
            self.array = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ------------------------------------------------------------------ handles

def _close_children(children):
    for ref in reversed(children):
        obj = ref()
        if obj is not None:
            obj.close()


class Context:
    """One GPU (stream, reduction buffers, graph caches).

    Handles made on a context (lattices, gauge and spinor fields, servers)
    register here; close() releases them first, newest first, so no handle can
    reach the C context after it is gone."""

    def __init__(self, device: int = 0):
        self.handle = _vp()
        _check(lib().hw_context_create(int(device), ctypes.byref(self.handle)))
        self.device = device
        self._children = []

    def _adopt(self, obj):
        import weakref
        self._children.append(weakref.ref(obj))

    def synchronize(self):
        _check(lib().hw_context_synchronize(self.handle))

    ENGINE_PHASES = ("P1", "P2", "P3", "P4", "R1", "R2", "R3", "R4", "R4L", "R5", "R5L", "P5")

    def engine_profile(self, enable: bool) -> None:
        """Per-phase event timing of the batched engines (hw_engine_profile_enable)."""
        _check(lib().hw_engine_profile_enable(self.handle, int(bool(enable))))

    def engine_profile_get(self, precision: str = "f16") -> dict:
        """{phase: (launches with work, summed ms, work units)} of one engine (hw_engine_profile_get).

        The work units are the four counters of ``hw_engine_profile.work`` (sites x solves of
        the main form, of the alternate form, sites whose links were read, R3 of the normal
        system); multiplied by the bytes of each unit they give the algorithmic bytes."""
        out = _EngineProfile()
        _check(lib().hw_engine_profile_get(self.handle, PRECISIONS[precision], ctypes.byref(out)))
        return {name: (out.launches[k], out.ms[k], tuple(int(v) for v in out.work[k]))
                for k, name in enumerate(self.ENGINE_PHASES)}

    def engine_tuning(self, precision: str = "f16") -> list:
        """The launch-shape tuner's entries of one engine (hw_engine_tuning_get), by work class:
        [{"work_class", "shapes": [(variant, dynamic_order, ms_per_iteration, samples)],
        "chosen": index or None}]."""
        out = (_EngineTuning * 64)()
        n = ctypes.c_int(0)
        _check(lib().hw_engine_tuning_get(self.handle, PRECISIONS[precision], out, 64, ctypes.byref(n)))
        res = []
        for t in out[:n.value]:
            shapes = [(t.variant[c], t.dynamic_order[c], t.ms_per_iteration[c], t.samples[c])
                      for c in range(t.nshapes)]
            res.append({"work_class": t.work_class, "shapes": shapes,
                        "chosen": t.chosen if t.chosen >= 0 else None})
        return res

    def stream(self) -> int:
        """The library's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        s = _vp()
        _check(lib().hw_context_stream(self.handle, ctypes.byref(s)))
        return s.value or 0

    def close(self):
        if self.handle:
            _close_children(self._children)
            self._children = []
            lib().hw_context_destroy(self.handle)
            self.handle = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Lattice:
    """lattice.setup(dims) (plumbing/lattice.cpp:37-104); t antiperiodic for fermions.
    close() first releases the gauge and spinor fields made on it."""

    def __init__(self, ctx: Context, dims, antiperiodic: bool = True):
        self.ctx = ctx
        self.dims = tuple(int(d) for d in dims)
        self.volume = int(np.prod(self.dims))
        self.handle = _vp()
        _check(lib().hw_lattice_create(ctx.handle, _dims(self.dims), int(bool(antiperiodic)),
                                       ctypes.byref(self.handle)))
        self._children = []
        ctx._adopt(self)

    def _adopt(self, obj):
        import weakref
        self._children.append(weakref.ref(obj))
        self.ctx._adopt(obj)

    def close(self):
        if self.handle:
            _close_children(self._children)
            self._children = []
            lib().hw_lattice_destroy(self.handle)
            self.handle = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GaugeField:
    """Field<SU<3,double>> U[NDIM] uploaded once to the device."""

    def __init__(self, lattice: Lattice, links: np.ndarray, link_format: int = 18):
        links = np.ascontiguousarray(links, np.float64)
        if links.size != 4 * lattice.volume * 18:
            raise ValueError("links must hold 4*V*18 doubles")
        self.lattice = lattice
        self.link_format = link_format
        self.handle = _vp()
        _check(lib().hw_gauge_create(lattice.handle, _dptr(links), int(link_format), ctypes.byref(self.handle)))
        lattice._adopt(self)

    def close(self):
        if self.handle:
            lib().hw_gauge_destroy(self.handle)
            self.handle = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Field:
    """Field<Wilson_vector<3,double>>: a device-resident FP64 spinor field."""

    def __init__(self, lattice: Lattice, data: np.ndarray | None = None, parity: int = ALL):
        self.lattice = lattice
        self.handle = _vp()
        _check(lib().hw_field_create(lattice.handle, ctypes.byref(self.handle)))
        lattice._adopt(self)
        if data is not None:
            self.upload(data, parity)

    def upload(self, data: np.ndarray, parity: int = ALL):
        data = np.ascontiguousarray(data, np.float64)
        if data.size != self.lattice.volume * 24:
            raise ValueError("spinor arrays hold V*24 doubles")
        _check(lib().hw_field_upload(self.handle, _dptr(data), int(parity)))

    def download(self, parity: int = ALL, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.zeros((self.lattice.volume, 4, 3, 2), np.float64)
        _check(lib().hw_field_download(self.handle, _dptr(out), int(parity)))
        return out

    def upload_eo(self, data: np.ndarray, parity: int = ALL):
        """hw_field_upload_eo: `data` in even-first site order ((V,4,3,2), EVEN sites first);
        only the sites of `parity` are copied (for EVEN a (V/2,4,3,2) array suffices)."""
        need = self.lattice.volume * (12 if parity == EVEN else 24)
        if data.dtype != np.float64 or not data.flags.c_contiguous or data.size < need:
            raise ValueError("spinor arrays hold V*24 contiguous doubles (V*12 for the EVEN half)")
        _check(lib().hw_field_upload_eo(self.handle, _dptr(data), int(parity)))

    def download_eo(self, parity: int = ALL, out: np.ndarray | None = None) -> np.ndarray:
        """hw_field_download_eo: the sites of `parity` into `out` in even-first site order; the
        other parity of `out` is left as it is."""
        if out is None:
            out = np.zeros((self.lattice.volume, 4, 3, 2), np.float64)
        need = self.lattice.volume * (12 if parity == EVEN else 24)
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size < need:
            raise ValueError("spinor arrays hold V*24 contiguous doubles (V*12 for the EVEN half)")
        _check(lib().hw_field_download_eo(self.handle, _dptr(out), int(parity)))
        return out

    def zero(self, parity: int = ALL):
        _check(lib().hw_field_zero(self.handle, int(parity)))

    def close(self):
        if self.handle:
            lib().hw_field_destroy(self.handle)
            self.handle = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ operators

class Dirac_Wilson_evenodd:
    """Dirac_Wilson_evenodd<SU<3,double>> (wilson.h:234-312): M = 1 - kappa^2 H^{eo} H^{oe} on EVEN."""

    par = EVEN

    def __init__(self, kappa: float, gauge: GaugeField):
        self.kappa = float(kappa)
        self.gauge = gauge

    def apply(self, inp: Field, out: Field):
        _check(lib().hw_wilson_evenodd_apply(self.gauge.handle, self.kappa, inp.handle, out.handle))

    def dagger(self, inp: Field, out: Field):
        _check(lib().hw_wilson_evenodd_dagger(self.gauge.handle, self.kappa, inp.handle, out.handle))

    def force(self, chi: Field, psi: Field, sign: int = 1) -> np.ndarray:
        """d Re(chi^dag M_s psi) / d links (wilson.h:293-311), shape (4, V, 3, 3, 2)."""
        out = np.zeros((4, self.gauge.lattice.volume, 3, 3, 2), np.float64)
        _check(lib().hw_wilson_evenodd_force(self.gauge.handle, self.kappa, chi.handle, psi.handle, int(sign),
                                             _dptr(out)))
        return out

    def hop(self, inp: Field, out: Field, parity: int, sign: int, set_: bool = True):
        """Dirac_Wilson_hop_set (set_) / Dirac_Wilson_hop with this operator's kappa."""
        _check(lib().hw_wilson_hop(self.gauge.handle, self.kappa, inp.handle, out.handle, int(parity), int(sign),
                                   int(bool(set_))))

    def solve(self, b: Field, x: Field, accuracy: float = 1e-10, maxiters: int = 10000, precision: str = "f64",
              delta: float = 0.1, use_graph: bool = True) -> "CGResult":
        """M x = b by CG on M^dag M with source M^dag b until |b - M x|/|b| <= accuracy."""
        p = _params(accuracy, maxiters, precision, delta, True, use_graph)
        r = _CgResult()
        rc = lib().hw_wilson_evenodd_solve(self.gauge.handle, self.kappa, b.handle, x.handle, ctypes.byref(p),
                                           ctypes.byref(r))
        if rc not in (HW_OK, HW_ERR_NOT_CONVERGED, HW_ERR_BREAKDOWN):
            _check(rc)
        return CGResult.from_c(r)

    def solve_host(self, b: np.ndarray, x: np.ndarray, accuracy: float = 1e-10, maxiters: int = 10000,
                   precision: str = "f64", delta: float = 0.1) -> "CGResult":
        """Host arrays in and out (copies included in the call)."""
        p = _params(accuracy, maxiters, precision, delta, True, True)
        r = _CgResult()
        rc = lib().hw_wilson_evenodd_solve_host(self.gauge.handle, self.kappa, _dptr(b), _dptr(x), ctypes.byref(p),
                                                ctypes.byref(r))
        if rc not in (HW_OK, HW_ERR_NOT_CONVERGED, HW_ERR_BREAKDOWN):
            _check(rc)
        return CGResult.from_c(r)


class StaggeredField:
    """Field<SU_vector<3,double>> for staggered fermions; host arrays (V, 3, 2)."""

    def __init__(self, lattice: Lattice, data: np.ndarray | None = None, parity: int = ALL):
        self.lattice = lattice
        self.handle = _vp()
        _check(lib().hw_stag_field_create(lattice.handle, ctypes.byref(self.handle)))
        lattice._adopt(self)
        if data is not None:
            self.upload(data, parity)

    def upload(self, data: np.ndarray, parity: int = ALL):
        data = np.ascontiguousarray(data, np.float64)
        if data.size != self.lattice.volume * 6:
            raise ValueError("staggered arrays hold V*6 doubles")
        _check(lib().hw_stag_field_upload(self.handle, _dptr(data), int(parity)))

    def download(self, parity: int = ALL) -> np.ndarray:
        out = np.zeros((self.lattice.volume, 3, 2), np.float64)
        _check(lib().hw_stag_field_download(self.handle, _dptr(out), int(parity)))
        return out

    def zero(self, parity: int = ALL):
        _check(lib().hw_stag_field_zero(self.handle, int(parity)))

    def close(self):
        if self.handle:
            lib().hw_stag_field_destroy(self.handle)
            self.handle = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class dirac_staggered_evenodd:
    """dirac_staggered_evenodd<SU<3,double>> (staggered.h:174-265) on EVEN."""

    par = EVEN

    def __init__(self, mass: float, gauge: GaugeField):
        self.mass = float(mass)
        self.gauge = gauge

    def apply(self, inp: StaggeredField, out: StaggeredField):
        _check(lib().hw_staggered_evenodd_apply(self.gauge.handle, self.mass, inp.handle, out.handle))

    def dagger(self, inp: StaggeredField, out: StaggeredField):
        _check(lib().hw_staggered_evenodd_dagger(self.gauge.handle, self.mass, inp.handle, out.handle))

    def force(self, chi: StaggeredField, psi: StaggeredField, sign: int = 1) -> np.ndarray:
        out = np.zeros((4, self.gauge.lattice.volume, 3, 3, 2), np.float64)
        _check(lib().hw_staggered_evenodd_force(self.gauge.handle, self.mass, chi.handle, psi.handle, int(sign),
                                                _dptr(out)))
        return out

    def cg(self, inp: StaggeredField, out: StaggeredField, accuracy: float = 1e-12, maxiters: int = 10000,
           true_residual: bool = False) -> "CGResult":
        """CG<dirac_staggered_evenodd>::apply: M^dag M out = inp, out the initial guess."""
        p = _params(accuracy, maxiters, "f64", 0.1, true_residual, False)
        r = _CgResult()
        rc = lib().hw_staggered_cg_solve(self.gauge.handle, self.mass, inp.handle, out.handle, ctypes.byref(p),
                                         ctypes.byref(r))
        if rc not in (HW_OK, HW_ERR_NOT_CONVERGED, HW_ERR_BREAKDOWN):
            _check(rc)
        return CGResult.from_c(r)


class Hasenbusch_operator:
    """Hasenbusch_operator<Dirac_Wilson_evenodd> (Hasenbusch.h:16-52): M + m_h on EVEN."""

    def __init__(self, D: "Dirac_Wilson_evenodd", h_parameter: float):
        self.D = D
        self.h_parameter = float(h_parameter)
        self.par = D.par

    def apply(self, inp: Field, out: Field):
        _check(lib().hw_hasenbusch_evenodd_apply(self.D.gauge.handle, self.D.kappa, self.h_parameter, inp.handle,
                                                 out.handle))

    def dagger(self, inp: Field, out: Field):
        _check(lib().hw_hasenbusch_evenodd_dagger(self.D.gauge.handle, self.D.kappa, self.h_parameter, inp.handle,
                                                  out.handle))

    def force(self, chi: Field, psi: Field, sign: int = 1) -> np.ndarray:
        """The operator's force (Hasenbusch.h:49-52): m_h does not depend on the links."""
        return self.D.force(chi, psi, sign)

    def solve(self, b: Field, x: Field, accuracy: float = 1e-10, maxiters: int = 10000, precision: str = "f64",
              delta: float = 0.1, use_graph: bool = True) -> "CGResult":
        """(M + m_h) x = b by CG on the normal equations."""
        p = _params(accuracy, maxiters, precision, delta, True, use_graph, self.h_parameter)
        r = _CgResult()
        rc = lib().hw_wilson_evenodd_solve(self.D.gauge.handle, self.D.kappa, b.handle, x.handle, ctypes.byref(p),
                                           ctypes.byref(r))
        if rc not in (HW_OK, HW_ERR_NOT_CONVERGED, HW_ERR_BREAKDOWN):
            _check(rc)
        return CGResult.from_c(r)


def mre_guess(op, old, chi: Field, psi: Field) -> None:
    """MRE_guess (MRE_guess.h:9-88): psi = initial guess for op^dag op psi = chi from the
    earlier solutions `old` (list of Field); op is Dirac_Wilson_evenodd or Hasenbusch_operator."""
    D, mh = (op.D, op.h_parameter) if isinstance(op, Hasenbusch_operator) else (op, 0.0)
    arr = (_vp * max(len(old), 1))(*[f.handle for f in old])
    _check(lib().hw_mre_guess(D.gauge.handle, D.kappa, mh, arr, len(old), chi.handle, psi.handle))


class Dirac_Wilson:
    """Dirac_Wilson<SU<3,double>> (wilson.h:146-201): D = 1 - kappa H over ALL sites."""

    par = ALL

    def __init__(self, kappa: float, gauge: GaugeField):
        self.kappa = float(kappa)
        self.gauge = gauge

    def apply(self, inp: Field, out: Field):
        _check(lib().hw_wilson_apply(self.gauge.handle, self.kappa, 1, inp.handle, out.handle))

    def dagger(self, inp: Field, out: Field):
        _check(lib().hw_wilson_apply(self.gauge.handle, self.kappa, -1, inp.handle, out.handle))

    def cg(self, inp: Field, out: Field, accuracy: float = 1e-12, maxiters: int = 10000,
           true_residual: bool = False) -> "CGResult":
        """CG<Dirac_Wilson>::apply (hw_wilson_cg_solve): M^dag M out = inp on ALL sites, FP64."""
        p = _params(accuracy, maxiters, "f64", 0.1, true_residual, False)
        r = _CgResult()
        rc = lib().hw_wilson_cg_solve(self.gauge.handle, self.kappa, inp.handle, out.handle, ctypes.byref(p),
                                      ctypes.byref(r))
        if rc not in (HW_OK, HW_ERR_NOT_CONVERGED, HW_ERR_BREAKDOWN):
            _check(rc)
        return CGResult.from_c(r)


@dataclass
class CGResult:
    status: int
    iterations: int
    reliable_updates: int
    restarts: int
    rr_relative: float
    true_residual: float
    seconds: float
    kernel_launches: int = 0

    @property
    def converged(self) -> bool:
        return self.status == HW_OK

    @classmethod
    def from_c(cls, r: _CgResult) -> "CGResult":
        return cls(r.status, r.iterations, r.reliable_updates, r.restarts, r.rr_relative, r.true_residual,
                   r.seconds, r.kernel_launches)


def _params(accuracy, maxiters, precision, delta, true_residual, use_graph, mh=0.0) -> _CgParams:
    p = _CgParams()
    lib().hw_cg_params_default(ctypes.byref(p))
    p.hasenbusch_mh = float(mh)
    p.accuracy = float(accuracy)
    p.maxiters = int(maxiters)
    p.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    p.delta = float(delta)
    p.true_residual = int(bool(true_residual))
    p.use_graph = int(bool(use_graph))
    return p


class CG:
    """CG<Op> (conjugate_gradient.h:18-104): apply(in, out) solves (M^dag M) out = in.

    Defaults follow the reference: accuracy 1e-12, maxiters 10000, stopping
    when |r|^2 < accuracy^2 |in|^2.  ``true_residual=True`` instead continues
    until the recomputed FP64 residual |in - M^dag M out| / |in| <= accuracy.
    """

    def __init__(self, op: Dirac_Wilson_evenodd, accuracy: float = 1e-12, maxiters: int = 10000,
                 precision: str = "f64", true_residual: bool = False, delta: float = 0.1, use_graph: bool = True):
        if not isinstance(op, Dirac_Wilson_evenodd):
            raise TypeError("CG runs on Dirac_Wilson_evenodd")
        self.M = op
        self.accuracy = float(accuracy)
        self.maxiters = int(maxiters)
        self.precision = precision
        self.true_residual = true_residual
        self.delta = delta
        self.use_graph = use_graph
        self.last = None

    def apply(self, inp: Field, out: Field) -> CGResult:
        p = _params(self.accuracy, self.maxiters, self.precision, self.delta, self.true_residual, self.use_graph)
        r = _CgResult()
        rc = lib().hw_cg_solve(self.M.gauge.handle, self.M.kappa, inp.handle, out.handle, ctypes.byref(p),
                               ctypes.byref(r))
        if rc not in (HW_OK, HW_ERR_NOT_CONVERGED, HW_ERR_BREAKDOWN):
            _check(rc)
        self.last = CGResult.from_c(r)
        return self.last


def batch_solve(ctx: Context, requests, precision: str = "f16", delta: float = 0.1) -> list:
    """Solve many M x = b at once: requests are (op, b_field, x_field[, accuracy[, maxiters]]);
    op is a Dirac_Wilson_evenodd or a Hasenbusch_operator ((M + m_h) x = b).

    All right-hand sides on all lattices advance together, one kernel launch
    per CG phase (hw_batch_solve); returns one CGResult per request.
    """
    n = len(requests)
    arr = (_SolveRequest * max(n, 1))()
    for k, req in enumerate(requests):
        op, b, x = req[0], req[1], req[2]
        acc = req[3] if len(req) > 3 else 1e-10
        mi = req[4] if len(req) > 4 else 10000
        D, mh = (op.D, op.h_parameter) if isinstance(op, Hasenbusch_operator) else (op, 0.0)
        arr[k] = _SolveRequest(D.gauge.handle.value, D.kappa, b.handle.value, x.handle.value, float(acc), int(mi),
                               float(mh))
    res = (_CgResult * max(n, 1))()
    rc = lib().hw_batch_solve(ctx.handle, PRECISIONS[precision], float(delta), arr, n, res)
    if rc not in (HW_OK, HW_ERR_NOT_CONVERGED, HW_ERR_BREAKDOWN):
        _check(rc)
    return [CGResult.from_c(res[k]) for k in range(n)]


def staggered_batch_solve(ctx: Context, requests, precision: str = "f64", delta: float = 0.0) -> list:
    """Many staggered solves at once on the batched engine (hw_staggered_batch_solve):
    requests are (dirac_staggered_evenodd, in_field, out_field[, accuracy[, maxiters[, normal]]]);
    normal=False solves M out = in, normal=True M^dag M out = in (CG<Op>::apply).
    precision "f64" runs FP64 throughout, "f16" the inner iterations on FP16 fields with
    FP64 reliable updates (delta <= 0: 0.05)."""
    if precision not in ("f64", "f16"):
        raise ValueError("staggered precision is 'f64' or 'f16'")
    n = len(requests)
    arr = (_StagSolveRequest * max(n, 1))()
    for k, req in enumerate(requests):
        op, b, x = req[0], req[1], req[2]
        acc = req[3] if len(req) > 3 else 1e-10
        mi = req[4] if len(req) > 4 else 10000
        normal = req[5] if len(req) > 5 else False
        arr[k] = _StagSolveRequest(op.gauge.handle.value, op.mass, b.handle.value, x.handle.value, float(acc),
                                   int(mi), int(bool(normal)), PRECISIONS[precision], float(delta))
    res = (_CgResult * max(n, 1))()
    rc = lib().hw_staggered_batch_solve(ctx.handle, arr, n, res)
    if rc not in (HW_OK, HW_ERR_NOT_CONVERGED, HW_ERR_BREAKDOWN):
        _check(rc)
    return [CGResult.from_c(res[k]) for k in range(n)]


def wilson_evenodd_apply_noalloc(dims, kappa: float, sign: int, links_ptr: int, in_ptr: int, out_ptr: int,
                                 stride: int, link_format: int = 18, antiperiodic: bool = True,
                                 stream: int = 0) -> None:
    """hw_wilson_evenodd_apply_noalloc on raw device pointers (even-odd layout).

    Allocates no device memory: for callers that cannot allocate.  At most
    32768 sites per parity; stream-ordered on `stream`.
    """
    _check(lib().hw_wilson_evenodd_apply_noalloc(_dims(dims), int(bool(antiperiodic)), float(kappa), int(sign),
                                                 _vp(links_ptr), int(link_format), _vp(in_ptr), _vp(out_ptr),
                                                 int(stride), _vp(stream)))


@dataclass
class RequestResult:
    status: int
    nrhs: int
    iterations: int
    reliable_updates: int
    true_residual: float
    latency_seconds: float
    queue_seconds: float
    admit_chunk: int = 0
    retire_chunk: int = 0

    @property
    def converged(self) -> bool:
        return self.status == HW_OK


# ------------------------------------------------------------------ configuration files

def config_dims(path: str) -> tuple:
    """Lattice size recorded in a HILA gauge configuration file (hw_gauge_config_dims)."""
    d = (ctypes.c_int * 4)()
    _check(lib().hw_gauge_config_dims(os.fsencode(path), d))
    return tuple(d)


def config_write(path: str, dims, links: np.ndarray) -> None:
    """GaugeField::config_write (gaugefield.h:196-217): links (4, V, 3, 3, 2) to a file."""
    links = np.ascontiguousarray(links, np.float64)
    dims = tuple(int(v) for v in dims)
    if links.size != 4 * int(np.prod(dims)) * 18:
        raise ValueError("links must hold 4*V*18 doubles")
    _check(lib().hw_gauge_config_write(os.fsencode(path), (ctypes.c_int * 4)(*dims), _dptr(links)))


def config_read(path: str, dims=None) -> np.ndarray:
    """GaugeField::config_read (gaugefield.h:219-271): links (4, V, 3, 3, 2) for a lattice of
    size dims (default: the file's); a smaller file is replicated periodically."""
    dims = tuple(int(v) for v in (dims if dims is not None else config_dims(path)))
    out = np.zeros((4, int(np.prod(dims)), 3, 3, 2), np.float64)
    _check(lib().hw_gauge_config_read(os.fsencode(path), (ctypes.c_int * 4)(*dims), _dptr(out)))
    return out


class Server:
    """Continuous-batching solve server (hw_server_*).

    Submit requests from any thread; gauge fields stay on the device; requests
    that arrive while others run join at the next chunk; every result is
    bitwise the same alone and in any mix."""

    def __init__(self, ctx: Context, precision: str = "f16", delta: float = 0.0, hbm_budget_bytes: int = 0,
                 chunk_iters: int = 8, host_pool_bytes: int = 0, staggered_precision: str = "f64"):
        cfg = _ServerConfig(PRECISIONS[precision], float(delta), int(hbm_budget_bytes), int(chunk_iters),
                            int(host_pool_bytes), PRECISIONS[staggered_precision])
        self.ctx = ctx
        self.handle = _vp()
        _check(lib().hw_server_create(ctx.handle, ctypes.byref(cfg), ctypes.byref(self.handle)))
        ctx._adopt(self)

    def add_gauge(self, gauge: GaugeField) -> int:
        gid = ctypes.c_int()
        _check(lib().hw_server_add_gauge(self.handle, gauge.handle, ctypes.byref(gid)))
        return gid.value

    def submit(self, gauge_id: int, kappa: float, sources, accuracy: float = 1e-10, maxiters: int = 10000) -> int:
        srcs = [np.ascontiguousarray(s_, np.float64) for s_ in sources]
        arr = (_dp * len(srcs))(*[_dptr(s_) for s_ in srcs])
        rid = ctypes.c_uint64()
        _check(lib().hw_server_submit(self.handle, int(gauge_id), float(kappa), len(srcs), arr, float(accuracy),
                                      int(maxiters), ctypes.byref(rid)))
        return rid.value

    def submit_eo(self, gauge_id: int, kappa: float, sources, solutions, accuracy: float = 1e-10,
                  maxiters: int = 10000) -> int:
        """hw_server_submit_eo: host arrays in even-first site order ((V,4,3,2), EVEN sites first;
        only the EVEN half is used, so (V/2,4,3,2) arrays suffice).  Page-locked arrays
        (PinnedArray) are copied by DMA directly; keep every array alive and untouched until
        wait() returns, which also fills pageable solutions.  solutions=None: the solutions
        stay in the server's buffers (wait(copy=True) returns them in even-first order)."""
        for a in list(sources) + list(solutions or []):
            assert a.dtype == np.float64 and a.flags.c_contiguous
        src = (_dp * len(sources))(*[_dptr(a) for a in sources])
        sol = (_dp * len(solutions))(*[_dptr(a) for a in solutions]) if solutions else None
        rid = ctypes.c_uint64()
        _check(lib().hw_server_submit_eo(self.handle, int(gauge_id), float(kappa), len(sources), src, sol,
                                         float(accuracy), int(maxiters), ctypes.byref(rid)))
        return rid.value

    def submit_fields(self, gauge_id: int, kappa: float, sources, solutions, accuracy: float = 1e-10,
                      maxiters: int = 10000) -> int:
        """hw_server_submit_fields: device Fields; the solution fields hold the initial guess."""
        src = (_vp * len(sources))(*[f.handle for f in sources])
        sol = (_vp * len(solutions))(*[f.handle for f in solutions])
        rid = ctypes.c_uint64()
        _check(lib().hw_server_submit_fields(self.handle, int(gauge_id), float(kappa), len(sources), src, sol,
                                             float(accuracy), int(maxiters), ctypes.byref(rid)))
        return rid.value

    def submit_staggered(self, gauge_id: int, mass: float, sources, solutions, accuracy: float = 1e-10,
                         maxiters: int = 10000) -> int:
        """hw_server_submit_staggered: staggered M x = b on device StaggeredFields, in place."""
        src = (_vp * len(sources))(*[f.handle for f in sources])
        sol = (_vp * len(solutions))(*[f.handle for f in solutions])
        rid = ctypes.c_uint64()
        _check(lib().hw_server_submit_staggered(self.handle, int(gauge_id), float(mass), len(sources), src, sol,
                                                float(accuracy), int(maxiters), ctypes.byref(rid)))
        return rid.value

    def wait(self, request_id: int, nrhs: int, volume: int, timeout: float = -1.0, copy: bool = True):
        """Returns (solutions, RequestResult); solutions is a list of (V,4,3,2)
        arrays, or None with copy=False."""
        sols, arr = None, None
        if copy:
            sols = [np.zeros((volume, 4, 3, 2), np.float64) for _ in range(nrhs)]
            arr = (_dp * nrhs)(*[_dptr(s_) for s_ in sols])
        r = _RequestResult()
        rc = lib().hw_server_wait(self.handle, ctypes.c_uint64(request_id), arr, float(timeout), ctypes.byref(r))
        if rc not in (HW_OK, HW_ERR_CANCELLED, HW_ERR_REJECTED):
            _check(rc)
        return sols, RequestResult(r.status, r.nrhs, r.iterations, r.reliable_updates, r.true_residual,
                                   r.latency_seconds, r.queue_seconds, r.admit_chunk, r.retire_chunk)

    def poll(self, request_id: int, nrhs: int, volume: int, copy: bool = False):
        """wait() that returns None at once while the request is still running."""
        try:
            return self.wait(request_id, nrhs, volume, timeout=0.0, copy=copy)
        except HilaError as e:
            if e.code == HW_ERR_TIMEOUT:
                return None
            raise

    def cancel(self, request_id: int) -> None:
        _check(lib().hw_server_cancel(self.handle, ctypes.c_uint64(request_id)))

    def stats(self) -> dict:
        st = _ServerStats()
        _check(lib().hw_server_stats_get(self.handle, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in _ServerStats._fields_}

    def close(self):
        if self.handle:
            lib().hw_server_destroy(self.handle)
            self.handle = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
