"""ctypes binding of libfss_cuda.so (the C ABI declared in include/fss_cuda.h).

The library is the only compute path of this package: there is no CPU fallback.  Loading
fails loudly when the shared object is missing and cannot be built, and every call checks
that its tensors live on a CUDA device.
"""
from __future__ import annotations

import ctypes
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
# FSS_LIB selects another build of the same ABI (e.g. one compiled with other tuning macros)
LIB_PATH = os.environ.get("FSS_LIB") or os.path.join(_HERE, "libfss_cuda.so")

FSS_OK, FSS_ERR_INVALID, FSS_ERR_CUDA, FSS_ERR_NOMEM, FSS_ERR_UNSUPPORTED, FSS_ERR_TIMEOUT = range(6)
MODE_SHAPE, MODE_ESP, MODE_PHARM, MODE_SHAPE_PHARM, MODE_SHAPE_COLOR, MODE_ESP_COMBO = range(6)

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_f32 = ctypes.c_float


class AlignDesc(ctypes.Structure):
    """Mirror of ``fss_align_desc`` (include/fss_cuda.h)."""
    _fields_ = [
        ("mode", _i32), ("n_pairs", _i32), ("n_starts", _i32), ("steps", _i32),
        ("pair_ref", _vp), ("pair_fit", _vp), ("order", _vp),
        ("ref_pts", _vp), ("ref_off", _vp), ("fit_pts", _vp), ("fit_off", _vp),
        ("ref_self", _vp), ("fit_self", _vp),
        ("ref_anc", _vp), ("ref_vec", _vp), ("ref_ph_off", _vp),
        ("fit_anc", _vp), ("fit_vec", _vp), ("fit_ph_off", _vp),
        ("ref_self_ph", _vp), ("fit_self_ph", _vp),
        ("seed_q", _vp), ("seed_t", _vp),
        ("alpha", _f32), ("inv_lam", _f32), ("color_weight", _f32), ("lr", _f32),
        ("row_score", _vp), ("row_q", _vp), ("row_t", _vp),
        ("out_score", _vp), ("out_q", _vp), ("out_t", _vp),
        ("max_ref_points", _i32), ("max_fit_points", _i32),
        ("max_ref_features", _i32), ("max_fit_features", _i32),
        ("lanes_per_pose", _i32), ("chunks", _i32), ("cta_per_sm", _i32),
        ("accumulate", _i32), ("kernel_variant", _i32), ("pharm_extended", _i32),
        ("similarity", _i32), ("tversky_sigma", _f32),
        ("ref_atoms", _vp), ("ref_radii", _vp), ("ref_atom_off", _vp),
        ("fit_atoms", _vp), ("fit_radii", _vp), ("fit_atom_off", _vp),
        ("ref_surf", _vp), ("ref_surf_off", _vp), ("fit_surf", _vp), ("fit_surf_off", _vp),
        ("max_ref_atoms", _i32), ("max_fit_atoms", _i32), ("max_ref_surf", _i32),
        ("max_fit_surf", _i32), ("esp_inv_lam", _f32), ("coulomb", _f32),
        ("probe_radius", _f32), ("esp_weight", _f32), ("esp_stride", _i32),
        ("scratch", _vp), ("fit_f16", _i32),
    ]


_SIGS = {
    "fss_abi_version": ([], ctypes.c_int),
    "fss_last_error": ([], ctypes.c_char_p),
    "fss_max_points": ([], ctypes.c_int),
    "fss_overlap_grad": ([_vp] * 8 + [_i32] * 3 + [_f32, _f32, _i32] + [_vp] * 4, ctypes.c_int),
    "fss_pharm_grad": ([_vp] * 10 + [_i32] * 5 + [_vp] * 4, ctypes.c_int),
    "fss_tanimoto_adam_step": ([_vp] * 13 + [_i32, _f32, _vp], ctypes.c_int),
    "fss_self_overlap": ([_vp, _vp, _i32, _i32, _f32, _i32, _f32, _i32, _vp, _vp], ctypes.c_int),
    "fss_pharm_self_overlap": ([_vp, _vp, _vp, _i32, _i32, _i32, _i32, _i32, _vp, _vp],
                               ctypes.c_int),
    "fss_seeds": ([_vp] * 6 + [_i32, _i32, _vp, _i32, _i32, _vp, _vp, _vp], ctypes.c_int),
    "fss_align": ([ctypes.POINTER(AlignDesc), _vp], ctypes.c_int),
    "fss_align_static": ([ctypes.POINTER(AlignDesc), _vp], ctypes.c_int),
    "fss_pick_best": ([_vp] * 3 + [_i32, _i32] + [_vp] * 4, ctypes.c_int),
    "fss_score_fwd": ([_vp] * 6 + [_i32, _i32, _i32, _f32, _i32, _f32, _vp, _vp, _vp],
                      ctypes.c_int),
    "fss_score_bwd": ([_vp] * 6 + [_i32, _i32, _i32, _f32, _i32, _f32] + [_vp] * 5,
                      ctypes.c_int),
    "fss_score_fwd_dense": ([_vp, _vp, _i32, _vp, _vp, _i32, _vp, _vp, _i32, _f32, _i32, _f32,
                             _vp, _vp, _vp], ctypes.c_int),
    "fss_score_bwd_dense": ([_vp, _vp, _i32, _vp, _vp, _i32, _vp, _vp, _i32, _f32, _i32, _f32]
                            + [_vp] * 7, ctypes.c_int),
    "fss_score_fwd_moments_dense": ([_vp, _vp, _i32, _vp, _vp, _i32, _vp, _vp, _i32, _f32,
                                     _i32, _f32] + [_vp] * 5, ctypes.c_int),
    "fss_score_bwd_moments_dense": ([_vp, _vp, _i32, _i32, _i32, _f32, _i32, _f32]
                                    + [_vp] * 8 + [_i32, _vp], ctypes.c_int),
    "fss_probe_peak": ([_i32, _i32, _i32, _vp, ctypes.POINTER(ctypes.c_longlong), _vp],
                       ctypes.c_int),
}

EXPORTED = tuple(_SIGS)

_LIB = None
_LOCK = threading.Lock()


def load(build_if_missing: bool = True):
    """Load (building first if needed) and type the shared library."""
    global _LIB
    if _LIB is not None:   # loaded: no lock on the per-call path
        return _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        if build_if_missing and not os.environ.get("FSS_LIB"):
            from . import build as _build
            if _build.needs_build():
                try:
                    _build.build()
                except Exception as exc:  # pragma: no cover - depends on the toolchain
                    if not os.path.exists(LIB_PATH):
                        raise RuntimeError(
                            f"libfss_cuda.so is missing and could not be built: {exc}") from exc
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libfss_cuda.so not found at {LIB_PATH}; run "
                               "`python -m fast_shepherd_score_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (argt, rest) in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = argt
            fn.restype = rest
        if lib.fss_abi_version() != 3:
            raise RuntimeError("libfss_cuda.so ABI version mismatch; rebuild the library")
        _LIB = lib
        return lib


_STATUS_EXC = {FSS_ERR_INVALID: ValueError, FSS_ERR_NOMEM: MemoryError,
               FSS_ERR_UNSUPPORTED: ValueError}


def raise_status(rc: int, msg: str) -> None:
    """Raise the Python exception of an fss_status code: FSS_ERR_INVALID / UNSUPPORTED ->
    ValueError, FSS_ERR_NOMEM -> MemoryError (callers halve a batch on it), else
    RuntimeError."""
    raise _STATUS_EXC.get(rc, RuntimeError)(msg)


def check(rc: int, what: str = "") -> None:
    """Raise the Python exception matching an fss_status code returned by the library."""
    if rc == FSS_OK:
        return
    msg = load().fss_last_error().decode(errors="replace")
    raise_status(rc, f"{what}: {msg}" if what else msg)


def ptr(t, dtype=None, name="tensor"):
    """Device pointer of a contiguous CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (this backend has no CPU path)")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t.data_ptr() if t.numel() else None


_RAW_STREAM = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def stream_ptr(device=None):
    """The current torch stream of `device` as a cudaStream_t.  Read as a raw handle when torch
    offers it (no Stream object per call: the eager autograd path makes four such calls a
    step), else through torch.cuda.current_stream."""
    if _RAW_STREAM is not None:
        idx = None
        if device is not None:
            idx = (device if isinstance(device, torch.device) else torch.device(device)).index
        return _RAW_STREAM(torch.cuda.current_device() if idx is None else idx)
    return torch.cuda.current_stream(device).cuda_stream
