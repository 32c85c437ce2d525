"""ctypes binding of the engine's C ABI (include/elegant_b200.h).

The library is loaded from the package directory.  There is no CPU fallback:
if the library or a CUDA device is missing, calls raise ``EngineError``.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libelegant_b200.so")

B2E_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "unsupported lattice",
    -3: "CUDA error",
    -4: "device out of memory",
    -5: "call out of order",
    -6: "device wait timed out",
    -7: "device fault flag",
}

CSR_PAGE_HEADER = 12  # B2E_CSR_PAGE_HEADER
# element type codes (include/elegant_b200.h)
DRIF, EDRIFT, KQUAD, KSEXT, CSBEND, RFCA, MAXAMP, MARK, CHARGE, CSRCSBEND, CSRDRIFT, MALIGN, WATCH = range(1, 14)
MAX_PARAMS = 40
RING_VARIANTS = 17

EXPORTED = [
    "b2e_create", "b2e_destroy", "b2e_last_error", "b2e_version", "b2e_load_lattice",
    "b2e_upload_particles", "b2e_track", "b2e_download", "b2e_track_host", "b2e_track_device",
    "b2e_load_ensemble", "b2e_ensemble_history", "b2e_csr_wakes", "b2e_stream",
    "b2e_kernel_launches", "b2e_ring_tuning", "b2e_history_passes", "b2e_csr_bend_static",
]


class Element(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("reserved", ctypes.c_int32), ("name", ctypes.c_char * 32),
                ("p", ctypes.c_double * MAX_PARAMS)]


class RunOptions(ctypes.Structure):
    _fields_ = [("p_central", ctypes.c_double), ("n_passes", ctypes.c_int32), ("default_order", ctypes.c_int32),
                ("coord_limit", ctypes.c_double), ("slope_limit", ctypes.c_double),
                ("passes_per_launch", ctypes.c_int32), ("ring_variant", ctypes.c_int32),
                ("record_history", ctypes.c_int32), ("compact_every", ctypes.c_int32),
                ("sr_gaussian_limit", ctypes.c_double), ("isr_seed", ctypes.c_uint64),
                ("record_tbt", ctypes.c_int32), ("fiducial_particles", ctypes.c_int32)]


class Override(ctypes.Structure):
    _fields_ = [("element", ctypes.c_int32), ("slot", ctypes.c_int32), ("values", ctypes.POINTER(ctypes.c_double))]


# int (*)(void *user, int32_t op, void *dev_buf, int64_t count, void *stream)
REDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64,
                             ctypes.c_void_p)


class EngineError(RuntimeError):
    """A C-ABI call returned a nonzero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {message}")
        self.code = code


_lib = None


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load the engine library (built by ``elegant_b200.build``)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise EngineError(-5, f"{p} is missing; run `python -m elegant_b200.build`")
    lib = ctypes.CDLL(p)
    vp, c_int, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
    dpp = ctypes.POINTER(ctypes.c_void_p)
    sig = {
        "b2e_create": (c_int, [ctypes.POINTER(vp), c_int]),
        "b2e_destroy": (c_int, [vp]),
        "b2e_last_error": (ctypes.c_char_p, [vp]),
        "b2e_version": (c_int, []),
        "b2e_load_lattice": (c_int, [vp, ctypes.POINTER(Element), ctypes.c_int32, ctypes.POINTER(RunOptions)]),
        "b2e_upload_particles": (c_int, [vp, dpp, vp, i64]),
        "b2e_track": (c_int, [vp, ctypes.POINTER(ctypes.c_double)]),
        "b2e_download": (c_int, [vp, dpp, vp, vp, vp, ctypes.POINTER(i64)]),
        "b2e_track_host": (c_int, [vp, dpp, vp, i64, vp, vp, ctypes.POINTER(i64), ctypes.POINTER(ctypes.c_double)]),
        "b2e_track_device": (c_int, [vp, dpp, vp, i64, vp, vp, ctypes.POINTER(ctypes.c_double)]),
        "b2e_load_ensemble": (c_int, [vp, ctypes.c_int32, vp, ctypes.POINTER(Override), ctypes.c_int32]),
        "b2e_ensemble_history": (c_int, [vp, vp, vp, vp, vp, vp]),
        "b2e_csr_wakes": (c_int, [vp, vp, i64, ctypes.POINTER(i64)]),
        "b2e_set_csr_pages": (c_int, [vp, ctypes.c_int32]),
        "b2e_set_csr_timing": (c_int, [vp, ctypes.c_int32]),
        "b2e_csr_timing": (c_int, [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(i64), ctypes.POINTER(i64)]),
        "b2e_csr_pages": (c_int, [vp, vp, i64, ctypes.POINTER(i64)]),
        "b2e_stream": (vp, [vp]),
        "b2e_kernel_launches": (i64, [vp]),
        "b2e_history_passes": (i64, [vp]),
        "b2e_set_csr_reducer": (c_int, [vp, vp, vp]),
        "b2e_set_csr_surrogate": (c_int, [vp, vp, ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_int32]),
        "b2e_csr_surrogate_stats": (c_int, [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), vp, i64,
                                            ctypes.POINTER(i64)]),
        "b2e_tbt": (c_int, [vp, vp, i64, ctypes.POINTER(i64)]),
        "b2e_set_watch": (c_int, [vp, i64]),
        "b2e_watch_records": (c_int, [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(i64), vp, vp,
                                      ctypes.c_int32]),
        "b2e_watch_data": (c_int, [vp, ctypes.c_int32, vp]),
        "b2e_tbt_tunes": (c_int, [vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp, vp]),
        "b2e_naff": (c_int, [vp, i64, ctypes.c_int32, vp, vp, vp, vp]),
        "b2e_element_defaults": (c_int, [ctypes.c_int32, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    bind_extra(lib)
    if path is None:
        _lib = lib
    return lib


def pointer_array(ptrs) -> ctypes.Array:
    arr = (ctypes.c_void_p * len(ptrs))()
    for i, p in enumerate(ptrs):
        arr[i] = p
    return arr


def bind_extra(lib: ctypes.CDLL) -> None:
    """Signatures of the instrumentation entry points."""
    lib.b2e_ring_tuning.restype = ctypes.c_int
    lib.b2e_ring_tuning.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_float)]
