"""Differentiable Tanimoto scores with a hand-written CUDA adjoint.

The reference computes d(score)/d(coordinates, charges) with torch autograd through
``cdist``/``exp`` (score/gaussian_overlap.py:62-117 ``get_overlap``,
score/electrostatic_scoring.py:55-120 ``get_overlap_esp``), materialising N x M distance
matrices.  Here the forward pass (``fss_score_fwd``) and its adjoint (``fss_score_bwd``) are
single kernels over packed clouds; :class:`PackedTanimoto` wraps them as a
``torch.autograd.Function`` whose inputs are the packed float4 point tensors (x, y, z,
charge), so gradients reach the caller's coordinate and charge tensors through the ordinary
torch ops that pack them.

* :func:`tanimoto_packed` -- P pairs of molecules in two packed sets (the general form; a
  fixed target shared by many queries is one molecule of the ref set).
* :func:`get_overlap`, :func:`get_overlap_esp` -- the reference's signatures for one pair
  ((N,3) vs (M,3)) or a matched batch ((B,N,3) vs (B,M,3)); :class:`DenseTanimoto` runs them
  on the padded tensors directly, with no packing and gradients written straight into the
  input shapes: ``fss_score_fwd_moments_dense`` (value, plus per-point adjoint moments of the
  sides that need a gradient, in one pass) and the elementwise ``fss_score_bwd_moments_dense``;
  clouds too large for its shared-memory staging take ``fss_score_fwd_dense`` /
  ``fss_score_bwd_dense``.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_ptr

LAM_SCALING = (1e4 / (4 * 55.263 * math.pi)) ** 2
_f32, _i32 = torch.float32, torch.int32


class PackedTanimoto(torch.autograd.Function):
    """score_p = V_AB / (V_AA + V_BB - V_AB) for P pairs of packed clouds."""

    @staticmethod
    def forward(ctx, ref_pts, fit_pts, ref_off, fit_off, pair_ref, pair_fit, max_ref, max_fit,
                alpha, esp, inv_lam):
        dev = ref_pts.device
        P = int(pair_ref.shape[0])
        ref_pts, fit_pts = ref_pts.contiguous(), fit_pts.contiguous()
        score = torch.empty(P, dtype=_f32, device=dev)
        ov = torch.empty(P, 3, dtype=_f32, device=dev)
        check(_lib.load().fss_score_fwd(ptr(ref_pts, _f32), ptr(ref_off, _i32), ptr(fit_pts, _f32),
                                        ptr(fit_off, _i32), ptr(pair_ref, _i32),
                                        ptr(pair_fit, _i32), P, int(max_ref), int(max_fit),
                                        float(alpha), int(esp), float(inv_lam), ptr(score),
                                        ptr(ov), stream_ptr(dev)), "score_fwd")
        ctx.save_for_backward(ref_pts, fit_pts, ref_off, fit_off, pair_ref, pair_fit, ov)
        ctx.cfg = (int(max_ref), int(max_fit), float(alpha), int(esp), float(inv_lam))
        ctx.mark_non_differentiable(ov)
        return score, ov

    @staticmethod
    def backward(ctx, g_score, g_ov):
        ref_pts, fit_pts, ref_off, fit_off, pair_ref, pair_fit, ov = ctx.saved_tensors
        max_ref, max_fit, alpha, esp, inv_lam = ctx.cfg
        need_r, need_f = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (need_r or need_f):
            return (None,) * 11
        gr = torch.zeros_like(ref_pts) if need_r else None
        gf = torch.zeros_like(fit_pts) if need_f else None
        g = g_score.to(_f32).contiguous()
        check(_lib.load().fss_score_bwd(ptr(ref_pts, _f32), ptr(ref_off, _i32), ptr(fit_pts, _f32),
                                        ptr(fit_off, _i32), ptr(pair_ref, _i32),
                                        ptr(pair_fit, _i32), int(pair_ref.shape[0]), max_ref,
                                        max_fit, alpha, esp, inv_lam, ptr(ov), ptr(g), ptr(gr),
                                        ptr(gf), stream_ptr(ref_pts.device)), "score_bwd")
        return gr, gf, None, None, None, None, None, None, None, None, None


def tanimoto_packed(ref_pts, ref_off, fit_pts, fit_off, pair_ref, pair_fit, *, alpha=0.81,
                    lam=None, max_ref=None, max_fit=None, return_overlaps=False):
    """Differentiable Tanimoto for pairs of packed clouds.

    ``ref_pts``/``fit_pts`` (n, 4) float32 CUDA tensors (x, y, z, charge), ``*_off`` int32
    prefix offsets, ``pair_*`` int32 molecule indices.  ``lam`` (kernel lambda) switches the
    ESP weighting on.  Gradients flow to ``ref_pts`` and ``fit_pts`` (w = d/d charge).
    """
    if max_ref is None:
        max_ref = int((ref_off[1:] - ref_off[:-1]).max()) if ref_off.numel() > 1 else 0
    if max_fit is None:
        max_fit = int((fit_off[1:] - fit_off[:-1]).max()) if fit_off.numel() > 1 else 0
    esp = lam is not None
    score, ov = PackedTanimoto.apply(ref_pts, fit_pts, ref_off.to(_i32).contiguous(),
                                     fit_off.to(_i32).contiguous(),
                                     pair_ref.to(_i32).contiguous(), pair_fit.to(_i32).contiguous(),
                                     max_ref, max_fit, alpha, esp,
                                     1.0 / float(lam) if esp else 0.0)
    return (score, ov) if return_overlaps else score


# per device: one int32 arange and one zeros tensor, grown to the largest batch seen; a pair
# index is a prefix view of one of them, so changing batch sizes allocate nothing new
_IDX_CACHE: dict = {}
_IDX_OLD: list = []


def _pair_index(B, n_mol, device):
    """int32 molecule index of each pair: identity, or 0 for a broadcast molecule (a view of
    a per-device cached tensor)."""
    key = (str(device), n_mol == B)
    t = _IDX_CACHE.get(key)
    if t is None or t.numel() < B:
        if t is not None:
            # a captured CUDA graph may hold the old tensor's address: keep it alive (the
            # sizes grow geometrically, so all of them together stay below twice the last)
            _IDX_OLD.append(t)
        n = max(B, 2 * (t.numel() if t is not None else 0))
        t = (torch.arange(n, dtype=_i32, device=device) if n_mol == B
             else torch.zeros(n, dtype=_i32, device=device))
        _IDX_CACHE[key] = t
    return t[:B]


def _f32c(t):
    """float32 contiguous view or copy (no dispatcher round trip when already so)."""
    return t if t.dtype is _f32 and t.is_contiguous() else t.to(_f32).contiguous()


class DenseTanimoto(torch.autograd.Function):
    """score_b = V_AB / (V_AA + V_BB - V_AB) for padded (B, N, 3) / (B, M, 3) batches (either
    side may be a single molecule broadcast over the batch); optional (B, N) charges.

    With grad mode on, the forward also writes the adjoint moments of every side that needs a
    gradient (``fss_score_fwd_moments_dense``), so the backward is one elementwise launch and
    the Gaussians are evaluated once per step; a side nobody differentiates (e.g. a shared
    target) gets no moments and no adjoint at all.  Clouds too large for the moments kernel's
    shared-memory staging (about 4700 points together) keep the inputs and take the two-pass
    adjoint (``fss_score_fwd_dense`` + ``fss_score_bwd_dense``)."""

    @staticmethod
    def forward(ctx, x1, x2, q1, q2, alpha, inv_lam, grad_on):
        esp = q1 is not None
        B = max(x1.shape[0], x2.shape[0])
        dev = x1.device
        x1, x2 = _f32c(x1), _f32c(x2)
        q1 = _f32c(q1) if esp else None
        q2 = _f32c(q2) if esp else None
        pr, pf = _pair_index(B, x1.shape[0], dev), _pair_index(B, x2.shape[0], dev)
        score = torch.empty(B, dtype=_f32, device=dev)
        ov = torch.empty(B, 3, dtype=_f32, device=dev)
        need = ctx.needs_input_grad
        side1 = bool(grad_on and (need[0] or (esp and need[2])))
        side2 = bool(grad_on and (need[1] or (esp and need[3])))
        lib = _lib.load()
        args = (ptr(x1), ptr(q1), x1.shape[1], ptr(x2), ptr(q2), x2.shape[1], ptr(pr, _i32),
                ptr(pf, _i32), B, float(alpha), int(esp), float(inv_lam), ptr(score), ptr(ov))
        m1 = torch.empty(B, x1.shape[1], 8, dtype=_f32, device=dev) if side1 else None
        m2 = torch.empty(B, x2.shape[1], 8, dtype=_f32, device=dev) if side2 else None
        # factored kernel (value only when neither side needs moments)
        rc = lib.fss_score_fwd_moments_dense(*args, ptr(m1), ptr(m2), stream_ptr(dev))
        two_pass = rc == _lib.FSS_ERR_UNSUPPORTED
        if two_pass:   # clouds too large to stage: direct kernel, two-pass adjoint below
            m1 = m2 = None
            check(lib.fss_score_fwd_dense(*args, stream_ptr(dev)), "score_fwd_dense")
        else:
            check(rc, "score_fwd_moments_dense")
        two_pass = two_pass and (side1 or side2)
        keep = (x1, x2, q1, q2) if two_pass else (None, None, None, None)
        ctx.save_for_backward(pr, pf, ov, m1, m2, *keep)
        ctx.cfg = (float(alpha), esp, float(inv_lam), x1.shape, x2.shape, dev, side1, side2)
        return score

    @staticmethod
    def backward(ctx, g_score):
        pr, pf, ov, m1, m2, x1, x2, q1, q2 = ctx.saved_tensors
        alpha, esp, inv_lam, shape1, shape2, dev, side1, side2 = ctx.cfg
        need = ctx.needs_input_grad
        if not (side1 or side2):
            return None, None, None, None, None, None, None
        B = int(pr.shape[0])
        moments = m1 is not None or m2 is not None
        # the moments backward stores the rows of a side with one molecule per pair; a
        # broadcast molecule (and the two-pass adjoint) accumulates into zeroed buffers
        own1, own2 = moments and shape1[0] == B, moments and shape2[0] == B

        def buf(shape, own):
            return (torch.empty if own else torch.zeros)(shape, dtype=_f32, device=dev)

        g1 = buf(shape1, own1) if side1 else None
        g2 = buf(shape2, own2) if side2 else None
        gq1 = buf(shape1[:2], own1) if esp and side1 else None
        gq2 = buf(shape2[:2], own2) if esp and side2 else None
        g = g_score.to(_f32).contiguous()
        lib = _lib.load()
        if moments:
            check(lib.fss_score_bwd_moments_dense(
                ptr(pr, _i32), ptr(pf, _i32), B, shape1[1], shape2[1], alpha, int(esp),
                inv_lam, ptr(ov), ptr(g), ptr(m1), ptr(m2), ptr(g1), ptr(gq1), ptr(g2),
                ptr(gq2), int(own1) | (int(own2) << 1), stream_ptr(dev)),
                "score_bwd_moments_dense")
        else:
            check(lib.fss_score_bwd_dense(
                ptr(x1), ptr(q1), shape1[1], ptr(x2), ptr(q2), shape2[1], ptr(pr, _i32),
                ptr(pf, _i32), int(pr.shape[0]), alpha, int(esp), inv_lam, ptr(ov), ptr(g),
                ptr(g1), ptr(gq1), ptr(g2), ptr(gq2), stream_ptr(dev)), "score_bwd_dense")
        return (g1 if need[0] else None, g2 if need[1] else None,
                gq1 if esp and need[2] else None, gq2 if esp and need[3] else None,
                None, None, None)


def _batched(c1, c2, q1=None, q2=None):
    single = c1.dim() == 2 and c2.dim() == 2
    if c1.dim() == 2:
        c1 = c1.unsqueeze(0)
        q1 = None if q1 is None else q1.reshape(1, -1)
    if c2.dim() == 2:
        c2 = c2.unsqueeze(0)
        q2 = None if q2 is None else q2.reshape(1, -1)
    B = max(c1.shape[0], c2.shape[0])
    return c1, c2, q1, q2, B, single


def _score(c1, c2, q1, q2, alpha, lam):
    c1, c2, q1, q2, B, single = _batched(c1, c2, q1, q2)
    if not (c1.is_cuda and c2.is_cuda):
        raise ValueError("fast_shepherd_score_b200 scores CUDA tensors only")
    if c1.shape[0] not in (1, B) or c2.shape[0] not in (1, B):
        raise ValueError("batch sizes must match or be 1")
    s = DenseTanimoto.apply(c1, c2, q1, q2, alpha, 1.0 / float(lam) if lam is not None else 0.0,
                            torch.is_grad_enabled())
    s = s.to(c1.dtype) if c1.dtype != _f32 else s
    return s[0] if single else s


def get_overlap(centers_1, centers_2, alpha: float = 0.81):
    """Shape Tanimoto (gaussian_overlap.py:73), differentiable in both clouds.

    (N,3) vs (M,3) -> scalar; (B,N,3) vs (B,M,3), or a single cloud against a batch -> (B,).
    """
    return _score(centers_1, centers_2, None, None, alpha, None)


def get_overlap_esp(centers_1, centers_2, charges_1, charges_2, alpha: float = 0.81,
                    lam: float = 0.3 * LAM_SCALING):
    """ESP-weighted Tanimoto (electrostatic_scoring.py:69), differentiable in coordinates and
    charges; ``lam`` as the reference's (surface default 0.3 * LAM_SCALING)."""
    return _score(centers_1, centers_2, charges_1, charges_2, alpha, lam)
