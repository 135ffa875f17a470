"""Kernel-level API of the CUDA backend (torch tensors in, torch tensors out).

Functions keep the names, argument meaning and return values of the reference's kernel
dispatch layer (shepherd_score/accel/kernels/dispatch.py and the Triton modules it routes
to), so code written against ``shepherd_score.accel.kernels`` can call these directly:

* :func:`overlap_score_grad_se3_batch`      (shape_triton.py:191-249)
* :func:`overlap_score_grad_esp_se3_batch`  (esp_triton.py:174-262)
* :func:`pharm_grad_dq_se3_batch`           (pharm_triton.py:403-467)
* :func:`pharm_color_score_grad_se3_batch`  (pharm_triton.py:254-293)
* :func:`_batch_self_overlap`, :func:`_batch_self_overlap_esp` (shape_triton.py:436, esp_triton.py:393)

plus the packed-layout kernels the fused driver uses (:func:`self_overlap`, :func:`seeds`,
:func:`align_packed`).  Every call runs on the current torch stream of the tensors' device.
"""
from __future__ import annotations

import math
from functools import lru_cache
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_ptr
from .layout import CloudSet, PharmSet

_f32, _i32 = torch.float32, torch.int32


def _c(t, dtype):
    return t.to(dtype).contiguous()


def _counts(x, K, pad, device):
    if x is None:
        return torch.full((K,), pad, dtype=_i32, device=device)
    return torch.as_tensor(x, device=device).to(_i32).contiguous()


def overlap_score_grad_se3_batch(A, B, q, t, *, alpha: float = 0.81, N_real=None, M_real=None,
                                 NEED_GRAD: bool = True, **_tuning):
    """Shape overlap V and dV/dq, dV/dt per pose. A (K,N_pad,3), B (K,M_pad,3), q (K,4), t (K,3)."""
    return _overlap(A, B, None, None, q, t, alpha, 0.0, N_real, M_real, NEED_GRAD)


def overlap_score_grad_esp_se3_batch(A, B, charges_A, charges_B, q, t, *, alpha: float = 0.81,
                                     lam: float = 0.3, N_real=None, M_real=None,
                                     NEED_GRAD: bool = True, **_tuning):
    """ESP-weighted overlap: the shape kernel times exp(-(c_i - c_j)^2 / lam) per term."""
    return _overlap(A, B, charges_A, charges_B, q, t, alpha, 1.0 / float(lam), N_real, M_real,
                    NEED_GRAD)


def _overlap(A, B, CA, CB, q, t, alpha, inv_lam, N_real, M_real, need_grad):
    K, N_pad, _ = A.shape
    M_pad = B.shape[1]
    dev = A.device
    A, B, q, t = _c(A, _f32), _c(B, _f32), _c(q, _f32), _c(t, _f32)
    CA = None if CA is None else _c(CA, _f32)
    CB = None if CB is None else _c(CB, _f32)
    Nr, Mr = _counts(N_real, K, N_pad, dev), _counts(M_real, K, M_pad, dev)
    V = torch.empty(K, dtype=_f32, device=dev)
    dQ = torch.zeros(K, 4, dtype=_f32, device=dev)
    dT = torch.zeros(K, 3, dtype=_f32, device=dev)
    L = _lib.load()
    check(L.fss_overlap_grad(ptr(A, _f32, "A"), ptr(B, _f32, "B"), ptr(CA, _f32, "charges_A"),
                             ptr(CB, _f32, "charges_B"), ptr(q, _f32, "q"), ptr(t, _f32, "t"),
                             ptr(Nr, _i32), ptr(Mr, _i32), K, N_pad, M_pad, float(alpha),
                             float(inv_lam), int(bool(need_grad)), ptr(V), ptr(dQ), ptr(dT),
                             stream_ptr(dev)), "overlap_score_grad_se3_batch")
    return V, dQ, dT


def pharm_grad_dq_se3_batch(q, t, ref_types, fit_types, ref_anchors, fit_anchors, ref_vectors,
                            fit_vectors, alphas=None, Ks=None, cats=None, *, N_real=None,
                            M_real=None, NEED_GRAD: bool = True, **_tuning):
    """Directional typed pharmacophore overlap and dO/dq, dO/dt (q assumed unit).

    The lookup tables are the reference's fixed per-type constants and are built into the
    kernel; ``alphas``/``Ks``/``cats`` are accepted for signature compatibility.
    """
    return _pharm(ref_anchors, fit_anchors, ref_vectors, fit_vectors, ref_types, fit_types, q,
                  t, N_real, M_real, True, NEED_GRAD)


def pharm_color_score_grad_se3_batch(A, B, q, t, ref_types, fit_types, alphas=None, Ks=None,
                                     cats=None, *, N_real=None, M_real=None,
                                     NEED_GRAD: bool = True, **_tuning):
    """Directionless (colour) typed overlap and dO/dq, dO/dt."""
    return _pharm(A, B, None, None, ref_types, fit_types, q, t, N_real, M_real, False,
                  NEED_GRAD)


def _pharm(A, B, RV, FV, At, Bt, q, t, N_real, M_real, directional, need_grad):
    K, N_pad, _ = A.shape
    M_pad = B.shape[1]
    dev = A.device
    A, B, q, t = _c(A, _f32), _c(B, _f32), _c(q, _f32), _c(t, _f32)
    RV = None if RV is None else _c(RV, _f32)
    FV = None if FV is None else _c(FV, _f32)
    At, Bt = _c(At, _i32), _c(Bt, _i32)
    Nr, Mr = _counts(N_real, K, N_pad, dev), _counts(M_real, K, M_pad, dev)
    O = torch.empty(K, dtype=_f32, device=dev)
    dQ = torch.zeros(K, 4, dtype=_f32, device=dev)
    dT = torch.zeros(K, 3, dtype=_f32, device=dev)
    L = _lib.load()
    check(L.fss_pharm_grad(ptr(A, _f32), ptr(B, _f32), ptr(RV, _f32), ptr(FV, _f32),
                           ptr(At, _i32), ptr(Bt, _i32), ptr(q, _f32), ptr(t, _f32),
                           ptr(Nr, _i32), ptr(Mr, _i32), K, N_pad, M_pad, int(directional),
                           int(bool(need_grad)), ptr(O), ptr(dQ), ptr(dT), stream_ptr(dev)),
          "pharm_grad_dq_se3_batch")
    return O, dQ, dT


def _identity(K, dev):
    q = torch.zeros(K, 4, dtype=_f32, device=dev)
    q[:, 0] = 1.0
    return q, torch.zeros(K, 3, dtype=_f32, device=dev)


@torch.no_grad()
def _batch_self_overlap(P_pad, N_real, alpha: float = 0.81):
    """V_PP at the identity pose for a padded batch (shape_triton.py:436-448)."""
    q, t = _identity(P_pad.shape[0], P_pad.device)
    return overlap_score_grad_se3_batch(P_pad, P_pad, q, t, alpha=alpha, N_real=N_real,
                                        M_real=N_real, NEED_GRAD=False)[0]


@torch.no_grad()
def _batch_self_overlap_esp(P_pad, charges, N_real, alpha: float = 0.81, lam: float = 0.3):
    """ESP self overlap at the identity pose (esp_triton.py:393-425)."""
    q, t = _identity(P_pad.shape[0], P_pad.device)
    return overlap_score_grad_esp_se3_batch(P_pad, P_pad, charges, charges, q, t, alpha=alpha,
                                            lam=lam, N_real=N_real, M_real=N_real,
                                            NEED_GRAD=False)[0]


def tanimoto_adam_step(V, dQ, dT, U, q, t, mq, vq, mt, vt, best, bq, bt, lr):
    """One Tanimoto + best-tracking + tangent-projected Adam step over K rows, in place
    (accel/drivers/shape.py:114-130 + shape_triton.py:383-406)."""
    L = _lib.load()
    K = q.shape[0]
    check(L.fss_tanimoto_adam_step(ptr(V, _f32), ptr(dQ, _f32), ptr(dT, _f32), ptr(U, _f32),
                                   ptr(q, _f32), ptr(t, _f32), ptr(mq, _f32), ptr(vq, _f32),
                                   ptr(mt, _f32), ptr(vt, _f32), ptr(best, _f32), ptr(bq, _f32),
                                   ptr(bt, _f32), K, float(lr), stream_ptr(q.device)),
          "tanimoto_adam_step")


# ------------------------------------------------------------------------------------------
# Packed layout kernels
# ------------------------------------------------------------------------------------------
def points(t: torch.Tensor, name: str = "points"):
    """(device pointer, float16 flag) of packed (n, 4) points: float32, or float16 for a
    library kept in float16 (the kernels widen it in their staging loads)."""
    if isinstance(t, torch.Tensor) and t.dtype == torch.float16:
        return ptr(t, torch.float16, name), 1
    return ptr(t, _f32, name), 0


def self_overlap(cs: CloudSet, alpha: float, esp: bool = False, lam: Optional[float] = None):
    """Per-molecule self overlap of a packed cloud set (shape, or ESP with lam)."""
    out = torch.empty(cs.n_mol, dtype=_f32, device=cs.device)
    inv_lam = 1.0 / float(lam) if esp else 0.0
    pts, f16 = points(cs.pts, "cloud points")
    check(_lib.load().fss_self_overlap(pts, ptr(cs.off, _i32), cs.n_mol, cs.max_points,
                                       float(alpha), int(esp), inv_lam, f16, ptr(out),
                                       stream_ptr(cs.device)), "self_overlap")
    return out


def pharm_self_overlap(ps: PharmSet, directional: bool = True, extended: int = 0):
    """Self overlap per molecule; ``extended`` 0 (cosine weights), 1 (extended points and
    anchors) or 2 (extended points only), as batch_pharm_self_overlap
    (accel/drivers/pharm_overlap.py:413)."""
    out = torch.empty(ps.n_mol, dtype=_f32, device=ps.anc.device)
    anc, f16 = points(ps.anc, "pharmacophore anchors")
    vec, vf16 = points(ps.vec, "pharmacophore vectors")
    if vf16 != f16:
        raise ValueError("pharmacophore anchors and vectors must share one dtype")
    check(_lib.load().fss_pharm_self_overlap(anc, vec, ptr(ps.off, _i32), ps.n_mol,
                                             ps.max_points, int(directional), int(extended), f16,
                                             ptr(out), stream_ptr(ps.anc.device)),
          "pharm_self_overlap")
    return out


@lru_cache(maxsize=64)
def _fibo_host(n: int) -> np.ndarray:
    """Fibonacci-sphere quaternions (+x rotated onto each golden-spiral point), float32.

    The reference builds these in float32 torch (alignment/_torch.py:173-195 with
    generate_point_cloud.py:234-261); this is the same construction in numpy.
    """
    if n <= 0:
        return np.zeros((0, 4), np.float32)
    offset = 2.0 / n
    inc = np.pi * (3.0 - np.sqrt(5.0))
    i = np.arange(n)
    y = ((i * offset) - 1) + (offset / 2)
    r = np.sqrt(1 - np.square(y))
    phi = np.mod(i + 1, n) * inc
    fibo = np.column_stack((np.cos(phi) * r, y, np.sin(phi) * r)).astype(np.float32)
    unit = np.tile(np.array([1.0, 0.0, 0.0], np.float32), (n, 1))
    ang = np.arccos(np.clip((unit * fibo).sum(1), -1.0, 1.0)).astype(np.float32)[:, None]
    same = np.isclose(unit, fibo).sum(1) == 3
    axes = np.zeros((n, 3), np.float32)
    axes[:, 0] = 1.0
    cr = np.cross(unit, fibo).astype(np.float32)
    axes[~same] = cr[~same]
    axes = (axes / np.maximum(np.linalg.norm(axes, axis=1, keepdims=True), 1e-12)).astype(np.float32)
    half = ang / np.float32(2.0)
    return np.concatenate([np.cos(half), axes * np.sin(half)], 1).astype(np.float32)


_FIBO_DEV: dict = {}


def _fibo_device(n: int, dev) -> torch.Tensor:
    """The Fibonacci quaternions on `dev`, copied once per (device, n): a fresh pageable copy
    per call would synchronise the stream with the work already queued on it."""
    dev = torch.device(dev)
    key = (dev.type, dev.index, n)
    t = _FIBO_DEV.get(key)
    if t is None:
        t = torch.from_numpy(_fibo_host(n)).to(dev)
        _FIBO_DEV[key] = t
    return t


def seeds(ref: CloudSet, fit: CloudSet, pair_ref, pair_fit, num_seeds: int):
    """(P,S,4) quaternions and (P,S,3) translations: batched_seeds_torch (_common.py:281-441)."""
    dev = ref.device
    P = int(pair_ref.shape[0])
    S = 1 if num_seeds == 1 else max(int(num_seeds), 5)
    if S > 64:
        raise ValueError("num_seeds above 64 is not supported by the seed kernel")
    n_struct = min(max(S - 5, 0), 6)
    n_fibo = max(S - 5 - n_struct, 0)
    fibo = _fibo_device(n_fibo, dev) if n_fibo else None
    sq = torch.empty(P, S, 4, dtype=_f32, device=dev)
    st = torch.empty(P, S, 3, dtype=_f32, device=dev)
    fit_pts, fit_f16 = points(fit.pts, "fit points")
    check(_lib.load().fss_seeds(ptr(ref.pts, _f32, "ref points"), ptr(ref.off, _i32), fit_pts,
                                ptr(fit.off, _i32), ptr(pair_ref, _i32), ptr(pair_fit, _i32), P,
                                S, ptr(fibo, _f32), n_fibo, fit_f16, ptr(sq), ptr(st),
                                stream_ptr(dev)),
          "seeds")
    return sq, st
