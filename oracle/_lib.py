"""ctypes binding of ``libfss_oracle.so`` (test infrastructure only; see ``oracle/__init__``)."""
from __future__ import annotations

import contextlib
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# "f64": the overlap sums in double, as the reference's numba path (the oracle proper);
# "f32": the same code with the sums in float, the reference's Triton precision (a control)
_SO = {"f64": os.path.join(_HERE, "libfss_oracle.so"),
       "f32": os.path.join(_HERE, "libfss_oracle_f32.so")}
_LIBS: dict = {}
_PRECISION = ["f64"]

MODE_SHAPE, MODE_ESP, MODE_PHARM, MODE_COMBO, MODE_COLOR_COMBO = 0, 1, 2, 3, 4

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p


def build(force: bool = False) -> str:
    """Compile the oracle (both precisions) with its Makefile (gcc, no GPU needed)."""
    src = os.path.join(_HERE, "fss_oracle.c")
    if force or any(not os.path.exists(p) or os.path.getmtime(p) < os.path.getmtime(src)
                    for p in _SO.values()):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO["f64"]


@contextlib.contextmanager
def precision(p: str):
    """Run the oracle calls inside the block with the overlap sums in ``p`` ("f64" or
    "f32")."""
    if p not in _SO:
        raise ValueError("precision must be 'f64' or 'f32'")
    _PRECISION.append(p)
    try:
        yield
    finally:
        _PRECISION.pop()


def lib(which: str = None):
    which = which or _PRECISION[-1]
    L = _LIBS.get(which)
    if L is None:
        if not os.path.exists(_SO[which]):
            build()
        L = ctypes.CDLL(_SO[which])
        L.fsso_overlap_grad.argtypes = [ctypes.c_int] * 3 + [_vp] * 6 + [_vp, _vp] + [
            ctypes.c_double, ctypes.c_double, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int]
        L.fsso_overlap_grad.restype = None
        L.fsso_pharm_grad.argtypes = [ctypes.c_int] * 3 + [_vp] * 10 + [_vp] * 3 + [
            ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int]
        L.fsso_pharm_grad.restype = None
        L.fsso_fine_loop_flat.argtypes = (
            [ctypes.c_int] * 4 + [_vp] * 6 + [ctypes.c_int] * 2 + [_vp] * 11 +
            [ctypes.c_double] * 3 + [_vp] * 4 + [ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                                  ctypes.c_double] + [_vp] * 3 +
            [ctypes.c_int] * 3)
        L.fsso_fine_loop_flat.restype = ctypes.c_int
        L.fsso_esp_compare.argtypes = [ctypes.c_int] * 3 + [_vp] * 7 + [ctypes.c_double] * 3 + [_vp]
        L.fsso_esp_compare.restype = None
        L.fsso_esp_combo_loop.argtypes = (
            [ctypes.c_int] * 3 + [_vp] * 4 + [ctypes.c_int] * 2 + [_vp] * 8 +
            [ctypes.c_int] * 2 + [_vp] * 6 + [ctypes.c_double] * 5 + [ctypes.c_int, _vp, _vp, _vp,
                                                                       ctypes.c_int, ctypes.c_float,
                                                                       _vp, _vp, _vp, ctypes.c_int])
        L.fsso_esp_combo_loop.restype = None
        L.fsso_max_threads.restype = ctypes.c_int
        _LIBS[which] = L
    return L


def ptr(a):
    """Raw data pointer of a C-contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data


def max_threads() -> int:
    return int(lib().fsso_max_threads())
