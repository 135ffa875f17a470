"""Alignment drivers of the CUDA backend.

:func:`align_packed` is the core: one fused persistent kernel runs every (pair, start)
pose through all Adam steps (``fss_align``).  The ``coarse_fine_*_align_many`` functions
keep the signatures and return values of the reference drivers and route to it:

* :func:`coarse_fine_align_many`          (shepherd_score/accel/drivers/shape.py:155-313)
* :func:`coarse_fine_esp_align_many`      (accel/drivers/esp.py:139-367)
* :func:`coarse_fine_pharm_align_many`    (accel/drivers/pharm.py:123-517)
* :func:`coarse_fine_vol_color_align_many`(accel/drivers/vol_color.py:199-518)
* :func:`coarse_fine_vol_pharm_align_many` -- shape + *directional* pharmacophore with one
  shared pose (the combination the reference offers only per pair,
  alignment/_torch.py:1376 ``optimize_vol_color_overlay(directionless=False)``).

Early stop: the fused kernel always runs the full ``steps_fine`` (the reference's early
stop is batch-global, which makes a pair's result depend on the other pairs of its
batch; running every step can only raise a pose's running-max best score).  The
``early_stop_*`` arguments are accepted for signature compatibility.

Two more drivers exist for comparison and for callers that want per-step control:
:class:`GraphedFineLoop` (per-step kernels captured in one CUDA graph and replayed, the
reference's ``_graphed.py`` structure) and :func:`align_one_pair_per_launch` (the plain
form: one overlap launch + one Adam launch per pair per step).
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np
import torch

from . import _lib, autotune, kernels, legacy_seeds, memory
from ._lib import AlignDesc, check, ptr, stream_ptr
from .layout import CloudSet, PharmSet, cost_order_device

_f32, _i32 = torch.float32, torch.int32
# Tversky weights of the reference (accel/drivers/pharm.py:40)
TVERSKY_SIGMA = {"tversky": 0.95, "tversky_ref": 1.0, "tversky_fit": 0.05}
LAM_SCALING = (1e4 / (4 * 55.263 * math.pi)) ** 2   # score/constants.py:16-17

MODE_IDS = {"shape": _lib.MODE_SHAPE, "esp": _lib.MODE_ESP, "pharm": _lib.MODE_PHARM,
            "shape_pharm": _lib.MODE_SHAPE_PHARM, "shape_color": _lib.MODE_SHAPE_COLOR,
            "esp_combo": _lib.MODE_ESP_COMBO}
COULOMB_SCALING = 1e4 / (4 * 55.263 * math.pi)   # score/constants.py:16

_SCRATCH: dict = {}
LAST_TILE: dict = {}   # tiling of the most recent fused launch (for reports)


def _scratch(device, stream=None) -> torch.Tensor:
    """The 2-int32 scratch (persistent-grid work counter + status word) of launches on
    (device, stream), defaulting to the device's current stream.

    The launch resets the counter on its own stream before the kernel starts, so launches on
    one stream are ordered and can share one buffer; two launches that may run at the same
    time (different streams, e.g. a server's stream and the caller's) must not, or both
    kernels would take work items from the same counter.  Hence one buffer per stream."""
    device = torch.device(device)
    if stream is None:
        stream = torch.cuda.current_stream(device)
    key = (device.index, int(stream.cuda_stream))
    s = _SCRATCH.get(key)
    if s is None:
        s = torch.zeros(2, dtype=_i32, device=device)
        _SCRATCH[key] = s
    return s


class AlignResult(tuple):
    """(score (P,), q (P,4), t (P,3)) plus optional per-row results in ``.rows``."""
    rows: Optional[tuple] = None


def align_packed(mode: str, *, pair_ref, pair_fit, seed_q, seed_t, steps: int, lr: float,
                 ref: Optional[CloudSet] = None, fit: Optional[CloudSet] = None,
                 ref_ph: Optional[PharmSet] = None, fit_ph: Optional[PharmSet] = None,
                 alpha: float = 0.81, lam: Optional[float] = None, color_weight: float = 0.5,
                 ref_self=None, fit_self=None, ref_self_ph=None, fit_self_ph=None,
                 order=None, lanes_per_pose: int = 0, chunks: int = 0, cta_per_sm: int = 0,
                 accumulate: int = 0, kernel_variant: int = 0, similarity: str = "tanimoto",
                 pharm_extended: int = 0, ref_atoms: Optional[CloudSet] = None,
                 fit_atoms: Optional[CloudSet] = None, ref_radii=None, fit_radii=None,
                 ref_surf: Optional[CloudSet] = None, fit_surf: Optional[CloudSet] = None,
                 probe_radius: float = 1.0, esp_weight: float = 0.5, esp_stride: int = 1,
                 rows=None, out=None, scratch=None,
                 check_status: bool = True, validate: bool = True):
    """Run the fused alignment kernel over packed clouds.

    ``mode`` in {"shape", "esp", "pharm", "shape_pharm", "shape_color"}.  ``seed_q``/``seed_t``
    are (P,S,4)/(P,S,3).  Returns (score, q, t) per pair; ``rows`` (if given, a tuple of
    (P*S,), (P*S,4), (P*S,3) tensors) receives every start's best score and pose.
    Self overlaps default to the kernels' own (:func:`kernels.self_overlap`).
    ``accumulate`` picks where the shape/ESP sums run: 0 automatic (autotuned), 1 FP32 lanes,
    2 tensor-core value/gradient sums, 3 tensor-core exponents (2 and 3: modes "shape" and
    "esp", 32 lanes per pose).  ``kernel_variant`` picks the
    FP32-lane loop's code variant: 0 automatic, 1 base, 2 wide register tile, 3 one-CTA/SM
    register budget (2 and 3 for "shape" and "esp").  Mode "pharm" only: ``similarity`` in
    ("tanimoto", "tversky", "tversky_ref", "tversky_fit") and ``pharm_extended`` 0 (cosine
    weights), 1 (extended points and anchors), 2 (extended points only).
    Mode "esp_combo" (vol_and_surf_esp): ``ref``/``fit`` are the shape centres; ``ref_atoms`` /
    ``fit_atoms`` the atoms with hydrogens (w = partial charge) with per-point ``*_radii``,
    ``ref_surf``/``fit_surf`` the surface points (w = ESP at the point); ``lam`` is the raw
    ShaEP weight (LAM_SCALING applied here), ``esp_stride`` the combo-score tracking stride.
    ``validate=False`` skips the pair-index range check (a device read-back) for callers that
    validated their indices on the host; ``check_status=False`` skips reading the kernel's
    status word (both keep the launch free of host synchronisation).
    ``scratch`` (2 int32: work counter, status word) defaults to one buffer per (device,
    current stream); a caller passing its own must not share it between launches that can
    overlap on the GPU.
    """
    m = MODE_IDS[mode]
    shape = m != _lib.MODE_PHARM
    pharm = m in (_lib.MODE_PHARM, _lib.MODE_SHAPE_PHARM, _lib.MODE_SHAPE_COLOR)
    directional = m in (_lib.MODE_PHARM, _lib.MODE_SHAPE_PHARM)
    dev = seed_q.device
    P, S = int(seed_q.shape[0]), int(seed_q.shape[1])
    if shape and (ref is None or fit is None):
        raise ValueError(f"mode {mode!r} needs ref and fit clouds")
    if pharm and (ref_ph is None or fit_ph is None):
        raise ValueError(f"mode {mode!r} needs ref and fit pharmacophores")
    if m == _lib.MODE_ESP and lam is None:
        raise ValueError("esp mode needs lam")
    combo = m == _lib.MODE_ESP_COMBO
    if combo:
        if any(x is None for x in (ref_atoms, fit_atoms, ref_radii, fit_radii, ref_surf,
                                   fit_surf)):
            raise ValueError("esp_combo needs atoms, radii and surfaces for both sides")
        if (ref_atoms.n_mol != ref.n_mol or ref_surf.n_mol != ref.n_mol or
                fit_atoms.n_mol != fit.n_mol or fit_surf.n_mol != fit.n_mol):
            raise ValueError("esp_combo sets must describe the same molecules")
        if ref_radii.numel() != ref_atoms.pts.shape[0] or fit_radii.numel() != fit_atoms.pts.shape[0]:
            raise ValueError("one radius per atom")
        lam = 0.001 if lam is None else float(lam)
        if not lam > 0:
            raise ValueError("lam must be > 0")
    similarity = similarity.lower()
    if similarity != "tanimoto" and similarity not in TVERSKY_SIGMA:
        raise ValueError("similarity must be one of ('tanimoto','tversky','tversky_ref',"
                         "'tversky_fit')")
    if (similarity != "tanimoto" or pharm_extended) and m != _lib.MODE_PHARM:
        raise ValueError("Tversky similarity and extended points apply to mode 'pharm' only")
    if pharm_extended not in (0, 1, 2):
        raise ValueError("pharm_extended must be 0, 1 or 2")
    pair_ref = torch.as_tensor(pair_ref, device=dev).to(_i32).contiguous()
    pair_fit = torch.as_tensor(pair_fit, device=dev).to(_i32).contiguous()
    seed_q = seed_q.to(_f32).contiguous()
    seed_t = seed_t.to(_f32).contiguous()
    if pair_ref.shape != (P,) or pair_fit.shape != (P,) or tuple(seed_t.shape) != (P, S, 3) \
            or tuple(seed_q.shape) != (P, S, 4):
        raise ValueError("pair_ref/pair_fit must be (P,), seeds (P,S,4) and (P,S,3)")
    n_ref = ref.n_mol if shape else ref_ph.n_mol
    n_fit = fit.n_mol if shape else fit_ph.n_mol
    if shape and pharm and (ref_ph.n_mol != n_ref or fit_ph.n_mol != n_fit):
        raise ValueError("shape and pharmacophore sets must describe the same molecules")
    if P and validate:
        # one device-to-host read for the four bounds
        rmin, fmin, rmax, fmax = torch.stack([pair_ref.min(), pair_fit.min(), pair_ref.max(),
                                              pair_fit.max()]).tolist()
        if min(rmin, fmin) < 0 or rmax >= n_ref or fmax >= n_fit:
            raise ValueError("pair index outside the molecule tables")
    if shape:
        esp_self = m == _lib.MODE_ESP
        if ref_self is None:
            ref_self = kernels.self_overlap(ref, alpha, esp_self, lam if esp_self else None)
        if fit_self is None:
            fit_self = kernels.self_overlap(fit, alpha, esp_self, lam if esp_self else None)
    if pharm:
        if m == _lib.MODE_PHARM:
            if ref_self is None:
                ref_self = kernels.pharm_self_overlap(ref_ph, directional, pharm_extended)
            if fit_self is None:
                fit_self = kernels.pharm_self_overlap(fit_ph, directional, pharm_extended)
        else:
            if ref_self_ph is None:
                ref_self_ph = kernels.pharm_self_overlap(ref_ph, directional)
            if fit_self_ph is None:
                fit_self_ph = kernels.pharm_self_overlap(fit_ph, directional)
    if order is None and P > 1:
        cr, cf = (ref, fit) if shape else (ref_ph, fit_ph)
        order = cost_order_device(cr.off, cf.off, pair_ref, pair_fit)
    tuned = (lanes_per_pose == 0 and chunks == 0 and cta_per_sm == 0 and accumulate == 0
             and kernel_variant == 0 and autotune.enabled() and P >= 64 and steps > 0)
    if tuned:
        extra = (dict(ref_atoms=ref_atoms, fit_atoms=fit_atoms, ref_radii=ref_radii,
                      fit_radii=fit_radii, ref_surf=ref_surf, fit_surf=fit_surf,
                      probe_radius=probe_radius, esp_weight=esp_weight, esp_stride=esp_stride)
                 if combo else dict(similarity=similarity, pharm_extended=pharm_extended))
        tile = _tuned_tile(mode, shape, ref, fit, ref_ph, fit_ph, pair_ref, pair_fit, seed_q,
                           seed_t, steps, lr, alpha, lam, color_weight, ref_self, fit_self,
                           ref_self_ph, fit_self_ph, extra)
        lanes_per_pose, chunks, cta_per_sm = (tile["lanes_per_pose"], tile["chunks"],
                                              tile["cta_per_sm"])
        accumulate = tile.get("accumulate", 0)
        kernel_variant = tile.get("kernel_variant", 0)
    if rows is None:
        rows = (memory.empty(P * S, _f32, dev), memory.empty((P * S, 4), _f32, dev),
                memory.empty((P * S, 3), _f32, dev))
    if out is None:
        out = (memory.empty(P, _f32, dev), memory.empty((P, 4), _f32, dev),
               memory.empty((P, 3), _f32, dev))
    scratch = _scratch(dev) if scratch is None else scratch
    LAST_TILE.clear()
    LAST_TILE.update(lanes_per_pose=int(lanes_per_pose), chunks=int(chunks),
                     cta_per_sm=int(cta_per_sm), accumulate=int(accumulate),
                     kernel_variant=int(kernel_variant),
                     autotuned=tuned)
    d = AlignDesc()
    d.mode, d.n_pairs, d.n_starts, d.steps = m, P, S, int(steps)
    d.pair_ref, d.pair_fit = ptr(pair_ref, _i32), ptr(pair_fit, _i32)
    d.order = ptr(order, _i32) if order is not None else None
    # the fit (library) side may be kept in float16; the kernel widens it while staging
    halves = set()
    if shape:
        d.ref_pts, d.ref_off = ptr(ref.pts, _f32, "ref points"), ptr(ref.off, _i32)
        d.fit_pts, h = kernels.points(fit.pts, "fit points")
        halves.add(h)
        d.fit_off = ptr(fit.off, _i32)
        d.max_ref_points, d.max_fit_points = ref.max_points, fit.max_points
    if pharm:
        d.ref_anc, d.ref_ph_off = ptr(ref_ph.anc, _f32, "ref anchors"), ptr(ref_ph.off, _i32)
        d.fit_anc, h = kernels.points(fit_ph.anc, "fit anchors")
        halves.add(h)
        d.fit_ph_off = ptr(fit_ph.off, _i32)
        if directional:
            d.ref_vec = ptr(ref_ph.vec, _f32, "ref vectors")
            d.fit_vec, h = kernels.points(fit_ph.vec, "fit vectors")
            halves.add(h)
        d.max_ref_features, d.max_fit_features = ref_ph.max_points, fit_ph.max_points
        d.ref_self_ph = ptr(ref_self_ph, _f32) if ref_self_ph is not None else None
        d.fit_self_ph = ptr(fit_self_ph, _f32) if fit_self_ph is not None else None
    d.ref_self, d.fit_self = ptr(ref_self, _f32), ptr(fit_self, _f32)
    d.seed_q, d.seed_t = ptr(seed_q, _f32), ptr(seed_t, _f32)
    d.alpha = float(alpha)
    d.inv_lam = 1.0 / float(lam) if (m == _lib.MODE_ESP) else 0.0
    d.color_weight = float(color_weight)
    d.lr = float(lr)
    d.row_score, d.row_q, d.row_t = (ptr(rows[0], _f32), ptr(rows[1], _f32), ptr(rows[2], _f32))
    d.out_score, d.out_q, d.out_t = (ptr(out[0], _f32), ptr(out[1], _f32), ptr(out[2], _f32))
    d.lanes_per_pose, d.chunks, d.cta_per_sm = int(lanes_per_pose), int(chunks), int(cta_per_sm)
    d.accumulate = int(accumulate)
    d.kernel_variant = int(kernel_variant)
    d.pharm_extended = int(pharm_extended)
    if combo:
        rr = ref_radii.to(_f32).contiguous()
        fr = fit_radii.to(_f32).contiguous()
        d.ref_atoms, d.ref_radii, d.ref_atom_off = (ptr(ref_atoms.pts, _f32), ptr(rr, _f32),
                                                    ptr(ref_atoms.off, _i32))
        d.fit_atoms, d.fit_radii, d.fit_atom_off = (ptr(fit_atoms.pts, _f32), ptr(fr, _f32),
                                                    ptr(fit_atoms.off, _i32))
        d.ref_surf, d.ref_surf_off = ptr(ref_surf.pts, _f32), ptr(ref_surf.off, _i32)
        d.fit_surf, d.fit_surf_off = ptr(fit_surf.pts, _f32), ptr(fit_surf.off, _i32)
        d.max_ref_atoms, d.max_fit_atoms = ref_atoms.max_points, fit_atoms.max_points
        d.max_ref_surf, d.max_fit_surf = ref_surf.max_points, fit_surf.max_points
        d.esp_inv_lam = 1.0 / (LAM_SCALING * lam)
        d.coulomb = COULOMB_SCALING
        d.probe_radius = float(probe_radius)
        d.esp_weight = float(esp_weight)
        d.esp_stride = int(esp_stride)
    if similarity != "tanimoto":
        d.similarity, d.tversky_sigma = 1, TVERSKY_SIGMA[similarity]
    if len(halves) > 1:
        raise ValueError("the fit clouds and pharmacophores must share one dtype")
    d.fit_f16 = halves.pop() if halves else 0
    d.scratch = ptr(scratch, _i32)
    check(_lib.load().fss_align(d, stream_ptr(dev)), f"align[{mode}]")
    if check_status:
        status = int(scratch[1].item())
        if status:
            raise RuntimeError(f"align[{mode}]: a pair exceeded the staged extents (status {status})")
    res = AlignResult(out)
    res.rows = rows
    return res


def _tuned_tile(mode, shape, ref, fit, ref_ph, fit_ph, pair_ref, pair_fit, seed_q, seed_t,
                steps, lr, alpha, lam, color_weight, ref_self, fit_self, ref_self_ph,
                fit_self_ph, extra=None):
    """The autotuned tile for this launch's shape bucket (tuned on first sight)."""
    cs_r, cs_f = (ref, fit) if shape else (ref_ph, fit_ph)
    S = int(seed_q.shape[1])
    P = int(seed_q.shape[0])
    key = autotune.shape_key(seed_q.device, mode, cs_r.max_points, cs_f.max_points,
                             float(np.mean(cs_f.counts)) if len(cs_f.counts) else 0.0, S, P,
                             int(steps))
    rec = autotune.lookup(key)
    if rec is not None:
        return rec
    pr = pair_ref.cpu().numpy()
    pf = pair_fit.cpu().numpy()
    cost = cs_r.counts[pr].astype(np.int64) * cs_f.counts[pf].astype(np.int64)
    # enough pairs for many waves of CTAs, so the sample is throughput- not latency-bound and
    # its load balance resembles the full launch's: 16 pairs per SM, or half the batch (up to
    # 64 per SM) so tiles with long work items (1-2 lanes per pose) are not ranked by a tail
    sms = torch.cuda.get_device_properties(seed_q.device).multi_processor_count
    k = min(P, max(16 * sms, min(P // 2, 64 * sms)))
    sel = torch.from_numpy(autotune.sample_pairs(cost, k)).to(seed_q.device)
    sub = dict(ref=ref, fit=fit, ref_ph=ref_ph, fit_ph=fit_ph, pair_ref=pair_ref[sel],
               pair_fit=pair_fit[sel], seed_q=seed_q[sel], seed_t=seed_t[sel],
               steps=min(int(steps), 10), lr=lr, alpha=alpha, lam=lam,
               color_weight=color_weight, ref_self=ref_self, fit_self=fit_self,
               ref_self_ph=ref_self_ph, fit_self_ph=fit_self_ph, check_status=False,
               scratch=torch.zeros(2, dtype=_i32, device=seed_q.device))
    sub.update(extra or {})

    def run(**tile):
        align_packed(mode, **sub, **tile)

    # A sample that is the whole batch is tuned at the real step count: the candidate launch
    # is then the launch itself, and per-launch costs (staging, the last wave) weigh in it as
    # they will.  A partial sample is lengthened until a run of the library's default tile
    # takes >= 10 ms (capped at the real step count), so launch jitter does not rank it.
    cands = autotune.candidates(mode, cs_f.max_points, S)
    if k >= P:
        sub["steps"] = int(steps)
    else:
        ms = autotune.time_once(run, accumulate=1)   # an explicit tile: no recursive tuning
        if ms < 10.0 and sub["steps"] < steps:
            sub["steps"] = int(min(steps, math.ceil(sub["steps"] * 10.0 / max(ms, 1e-3))))
    return autotune.tune(run, key, cands, repeats=3)


# ------------------------------------------------------------------------------------------
# Reference-signature drivers (padded batches in, per-pair best out)
# ------------------------------------------------------------------------------------------
def _self_pairs(K, dev):
    idx = torch.arange(K, dtype=_i32, device=dev)
    return idx, idx


def _default_counts(x, K, pad, dev):
    if x is None:
        return torch.full((K,), pad, dtype=torch.int64, device=dev)
    return torch.as_tensor(x, device=dev).to(torch.int64)


TILE_KEYS = ("lanes_per_pose", "chunks", "cta_per_sm", "accumulate", "kernel_variant")


def coarse_tile(tile: dict) -> dict:
    """Extra arguments of the one-step coarse-scoring launch: the library's built-in tile
    unless the caller chose one (tuning a one-step launch costs far more than the launch)."""
    return {} if any(tile.get(k) for k in TILE_KEYS) else {"accumulate": 1}


def _trans_seeds(run, g_ref: CloudSet, g_fit: CloudSet, trans_centers, trans_centers_real,
                 per_trans: int, topk: int, shift=None):
    """Start poses of the translation-seeded path (the reference's trans_centers branch,
    drivers/esp.py:228-262 and its twins): the legacy grid of every pair
    (:mod:`legacy_seeds`), each pose scored once by the fused kernel (``run(seeds, 1)`` returns
    the per-row scores of a one-step launch, i.e. the seed poses' own scores), and the top-k
    poses per pair as (K,topk,4), (K,topk,3) seeds for the fine run."""
    K = trans_centers.shape[0]
    dev = trans_centers.device
    n = _default_counts(trans_centers_real, K, trans_centers.shape[1], dev)
    centres = CloudSet.from_padded(trans_centers.to(_f32), n)
    pr, pf = _self_pairs(K, dev)
    gq, gt, G = legacy_seeds.grid_packed(g_ref, g_fit, centres, pr, pf, per_trans, shift)
    return legacy_seeds.select(run((gq, gt), 1), gq, gt, G, topk)


def coarse_fine_align_many(A_batch, B_batch, VAA, VBB, *, alpha: float = 0.81,
                           num_seeds: int = 50, steps_fine: int = 100, lr: float = 0.075,
                           N_real=None, M_real=None, early_stop_patience: int = 2,
                           early_stop_tol: float = 1e-5, seeds: Optional[tuple] = None,
                           prune_after: int = 0, prune_keep: int = 0, **tile):
    """Batched shape alignment (vol / surf); returns (score (B,), q (B,4), t (B,3))."""
    K, npad, _ = A_batch.shape
    dev = A_batch.device
    N_real = _default_counts(N_real, K, npad, dev)
    M_real = _default_counts(M_real, K, B_batch.shape[1], dev)
    ref = CloudSet.from_padded(A_batch, N_real)
    fit = CloudSet.from_padded(B_batch, M_real)
    pr, pf = _self_pairs(K, dev)
    if seeds is None:
        seeds = kernels.seeds(ref, fit, pr, pf, num_seeds)
    return align_packed("shape", ref=ref, fit=fit, pair_ref=pr, pair_fit=pf, seed_q=seeds[0],
                        seed_t=seeds[1], steps=steps_fine, lr=lr, alpha=alpha,
                        ref_self=VAA.to(_f32).contiguous(), fit_self=VBB.to(_f32).contiguous(),
                        **tile)


def coarse_fine_esp_align_many(A_batch, B_batch, CA_batch, CB_batch, VAA, VBB, *,
                               alpha: float = 0.81, lam: float = 0.3, num_seeds: int = 50,
                               trans_centers=None, trans_centers_real=None,
                               num_repeats_per_trans: int = 10, topk: int = 30,
                               steps_fine: int = 100, lr: float = 0.075, N_real=None,
                               M_real=None, early_stop_patience: int = 5,
                               early_stop_tol: float = 1e-5, seeds: Optional[tuple] = None,
                               **tile):
    """Batched ESP alignment; ``lam`` is the kernel lambda (LAM_SCALING*lam for surfaces).

    ``trans_centers`` (K,P,3) with ``trans_centers_real`` selects the translation-seeded
    starts (trans_init=True): the legacy grid of 5 + num_repeats_per_trans * P poses per pair,
    scored once, its ``topk`` best refined."""
    K, npad, _ = A_batch.shape
    dev = A_batch.device
    N_real = _default_counts(N_real, K, npad, dev)
    M_real = _default_counts(M_real, K, B_batch.shape[1], dev)
    ref = CloudSet.from_padded(A_batch, N_real, CA_batch)
    fit = CloudSet.from_padded(B_batch, M_real, CB_batch)
    pr, pf = _self_pairs(K, dev)
    VAA, VBB = VAA.to(_f32).contiguous(), VBB.to(_f32).contiguous()

    def run(sd, steps, **extra):
        return align_packed("esp", ref=ref, fit=fit, pair_ref=pr, pair_fit=pf, seed_q=sd[0],
                            seed_t=sd[1], steps=steps, lr=lr, alpha=alpha, lam=lam,
                            ref_self=VAA, fit_self=VBB, **tile, **extra)

    if trans_centers is not None:
        coarse = lambda sd, st: run(sd, st, **coarse_tile(tile)).rows[0]
        seeds = _trans_seeds(coarse, ref, fit, trans_centers,
                             trans_centers_real, num_repeats_per_trans, topk)
    elif seeds is None:
        seeds = kernels.seeds(ref, fit, pr, pf, num_seeds)
    return run(seeds, steps_fine)


def _centroids(X, n):
    K, npad, _ = X.shape
    mask = (torch.arange(npad, device=X.device)[None] < n[:, None]).to(X.dtype)
    return (X * mask.unsqueeze(-1)).sum(1) / n.clamp(min=1).to(X.dtype).unsqueeze(-1)


def _quat_rot(q):
    q = torch.nn.functional.normalize(q, dim=-1)
    w, x, y, z = q.unbind(-1)
    return torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                        2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                        2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
                       -1).reshape(q.shape[:-1] + (3, 3))


def extended_code(extended_points: bool, only_extended: bool) -> int:
    """fss_align_desc.pharm_extended for the reference's flags (only_extended matters only
    with extended_points, analytical_gradients/_torch.py:288-297)."""
    return 0 if not extended_points else (2 if only_extended else 1)


def coarse_fine_pharm_align_many(anchors_1, anchors_2, vectors_1, vectors_2, types_1, types_2,
                                 VAA=None, VBB=None, *, similarity: str = "tanimoto",
                                 extended_points: bool = False, only_extended: bool = False,
                                 num_seeds: int = 50, trans_centers=None,
                                 trans_centers_real=None, num_repeats_per_trans: int = 10,
                                 topk: int = 30, steps_fine: int = 100, lr: float = 0.075,
                                 N_real=None, M_real=None, early_stop_patience: int = 5,
                                 early_stop_tol: float = 1e-5, seeds: Optional[tuple] = None,
                                 **tile):
    """Batched directional pharmacophore alignment (Tanimoto or Tversky, optionally with
    extended points).

    Clouds are centred on their own centroids first and the translation folded back at the
    end, as the reference does (pharm.py:205-225, :509-517).  ``seeds`` (if given) are for
    the centred clouds.  VAA/VBB are recomputed by the kernel with the same extended-point
    convention as the cross overlap, as in the reference (pharm.py:732-748).
    """
    K, npad, _ = anchors_1.shape
    dev = anchors_1.device
    N_real = _default_counts(N_real, K, npad, dev)
    M_real = _default_counts(M_real, K, anchors_2.shape[1], dev)
    a1 = anchors_1.to(_f32)
    a2 = anchors_2.to(_f32)
    c_ref = _centroids(a1, N_real)
    c_fit = _centroids(a2, M_real)
    a1c = a1 - c_ref[:, None, :]
    a2c = a2 - c_fit[:, None, :]
    ref_ph = PharmSet.from_padded(a1c, types_1, vectors_1, N_real)
    fit_ph = PharmSet.from_padded(a2c, types_2, vectors_2, M_real)
    pr, pf = _self_pairs(K, dev)

    def run(sd, steps, **extra):
        return align_packed("pharm", ref_ph=ref_ph, fit_ph=fit_ph, pair_ref=pr, pair_fit=pf,
                            seed_q=sd[0], seed_t=sd[1], steps=steps, lr=lr,
                            similarity=similarity,
                            pharm_extended=extended_code(extended_points, only_extended),
                            **tile, **extra)

    if trans_centers is not None:
        # centres are points of the original reference frame: shift them with the anchors
        coarse = lambda sd, st: run(sd, st, **coarse_tile(tile)).rows[0]
        seeds = _trans_seeds(coarse, CloudSet.from_padded(a1c, N_real),
                             CloudSet.from_padded(a2c, M_real), trans_centers.to(_f32),
                             trans_centers_real, num_repeats_per_trans, topk, shift=c_ref)
    elif seeds is None:
        seeds = kernels.seeds(CloudSet.from_padded(a1c, N_real),
                              CloudSet.from_padded(a2c, M_real), pr, pf, num_seeds)
    sc, q, t = run(seeds, steps_fine)
    R = _quat_rot(q)
    t = t - torch.einsum('bij,bj->bi', R, c_fit) + c_ref
    return sc, q, t


def coarse_fine_esp_combo_align_many(centers_w_H_1, centers_w_H_2, centers_1, centers_2,
                                     points_1, points_2, partial_charges_1, partial_charges_2,
                                     point_charges_1, point_charges_2, radii_1, radii_2,
                                     VAA=None, VBB=None, *, alpha: float, lam: float = 0.001,
                                     probe_radius: float = 1.0, esp_weight: float = 0.5,
                                     num_seeds: int = 50, trans_centers=None,
                                     trans_centers_real=None, num_repeats_per_trans: int = 10,
                                     topk: int = 30, steps_fine: int = 100, lr: float = 0.075,
                                     N_real_centers=None, M_real_centers=None,
                                     N_real_atoms_w_H_1=None, M_real_atoms_w_H_2=None,
                                     N_real_surf_1=None, M_real_surf_2=None,
                                     early_stop_patience: int = 5, early_stop_tol: float = 1e-5,
                                     seeds: Optional[tuple] = None, esp_stride: int = 1,
                                     **tile):
    """vol_and_surf_esp alignment with the reference signature (esp_combo.py:334-595).

    The pose follows the volumetric shape gradient of the centres, scaled by (1 - esp_weight);
    the tracked score is esp_weight * ShaEP ESP similarity (surface points of each molecule
    against the other's atoms with hydrogens) + (1 - esp_weight) * shape Tanimoto.
    ``esp_stride`` = 1 scores every step as the reference's CUDA-graph loop does; 5 matches its
    eager loop.  VAA/VBB (shape self overlaps) are recomputed when not given.
    """
    K = centers_1.shape[0]
    dev = centers_1.device
    cnt = lambda n, x: _default_counts(n, K, x.shape[1], dev)
    NC, MC = cnt(N_real_centers, centers_1), cnt(M_real_centers, centers_2)
    NA, MA = cnt(N_real_atoms_w_H_1, centers_w_H_1), cnt(M_real_atoms_w_H_2, centers_w_H_2)
    NS, MS = cnt(N_real_surf_1, points_1), cnt(M_real_surf_2, points_2)
    ref = CloudSet.from_padded(centers_1.to(_f32), NC)
    fit = CloudSet.from_padded(centers_2.to(_f32), MC)
    ra = CloudSet.from_padded(centers_w_H_1.to(_f32), NA, partial_charges_1)
    fa = CloudSet.from_padded(centers_w_H_2.to(_f32), MA, partial_charges_2)
    rrad = _packed_values(radii_1, NA)
    frad = _packed_values(radii_2, MA)
    rs = CloudSet.from_padded(points_1.to(_f32), NS, point_charges_1)
    fs = CloudSet.from_padded(points_2.to(_f32), MS, point_charges_2)
    pr, pf = _self_pairs(K, dev)

    def run(sd, steps, **extra):
        return align_packed("esp_combo", ref=ref, fit=fit, pair_ref=pr, pair_fit=pf,
                            seed_q=sd[0], seed_t=sd[1], steps=steps, lr=lr, alpha=alpha,
                            lam=lam, ref_self=VAA, fit_self=VBB, ref_atoms=ra, fit_atoms=fa,
                            ref_radii=rrad, fit_radii=frad, ref_surf=rs, fit_surf=fs,
                            probe_radius=probe_radius, esp_weight=esp_weight,
                            esp_stride=esp_stride, **tile, **extra)

    if trans_centers is not None:
        # the legacy grid is built from the surface clouds (esp_combo.py:409-412)
        coarse = lambda sd, st: run(sd, st, **coarse_tile(tile)).rows[0]
        seeds = _trans_seeds(coarse, rs, fs, trans_centers,
                             trans_centers_real, num_repeats_per_trans, topk)
    elif seeds is None:
        seeds = kernels.seeds(ref, fit, pr, pf, num_seeds)
    return run(seeds, steps_fine)


def _packed_values(X, n_real):
    """(K, N_pad) per-point values -> the packed order of CloudSet.from_padded."""
    K, npad = X.shape
    n = torch.as_tensor(n_real, device=X.device).to(torch.int64).clamp(0, npad)
    mask = torch.arange(npad, device=X.device)[None, :] < n[:, None]
    return X.to(_f32)[mask].contiguous()


def coarse_fine_vol_color_align_many(centers_1, centers_2, ptype_1, ptype_2, anchors_1,
                                     anchors_2, VAA, VBB, *, alpha: float = 0.81,
                                     color_weight: float = 0.5, num_seeds: int = 50,
                                     trans_centers=None, trans_centers_real=None,
                                     num_repeats_per_trans: int = 10, topk: int = 30,
                                     steps_fine: int = 100, lr: float = 0.075,
                                     N_real_centers=None, M_real_centers=None,
                                     N_real_pharm=None, M_real_pharm=None,
                                     early_stop_patience: int = 2, early_stop_tol: float = 1e-5,
                                     seeds: Optional[tuple] = None, vectors_1=None,
                                     vectors_2=None, directional: bool = False, **tile):
    """Shape + pharmacophore alignment with the joint gradient of the two Tanimotos.

    ``directional=False`` is the reference vol_color mode (directionless colour);
    ``directional=True`` weights same-type pairs by the vector cosine (needs vectors).
    """
    K = centers_1.shape[0]
    dev = centers_1.device
    Nc = _default_counts(N_real_centers, K, centers_1.shape[1], dev)
    Mc = _default_counts(M_real_centers, K, centers_2.shape[1], dev)
    Np = _default_counts(N_real_pharm, K, anchors_1.shape[1], dev)
    Mp = _default_counts(M_real_pharm, K, anchors_2.shape[1], dev)
    ref = CloudSet.from_padded(centers_1, Nc)
    fit = CloudSet.from_padded(centers_2, Mc)
    ref_ph = PharmSet.from_padded(anchors_1, ptype_1, vectors_1 if directional else None, Np)
    fit_ph = PharmSet.from_padded(anchors_2, ptype_2, vectors_2 if directional else None, Mp)
    pr, pf = _self_pairs(K, dev)
    VAA, VBB = VAA.to(_f32).contiguous(), VBB.to(_f32).contiguous()

    def run(sd, steps, **extra):
        return align_packed("shape_pharm" if directional else "shape_color", ref=ref, fit=fit,
                            ref_ph=ref_ph, fit_ph=fit_ph, pair_ref=pr, pair_fit=pf,
                            seed_q=sd[0], seed_t=sd[1], steps=steps, lr=lr, alpha=alpha,
                            color_weight=color_weight, ref_self=VAA, fit_self=VBB, **tile,
                            **extra)

    if trans_centers is not None:
        coarse = lambda sd, st: run(sd, st, **coarse_tile(tile)).rows[0]
        seeds = _trans_seeds(coarse, ref, fit, trans_centers,
                             trans_centers_real, num_repeats_per_trans, topk)
    elif seeds is None:
        seeds = kernels.seeds(ref, fit, pr, pf, num_seeds)
    return run(seeds, steps_fine)


def coarse_fine_vol_pharm_align_many(centers_1, centers_2, ptype_1, ptype_2, anchors_1,
                                     anchors_2, vectors_1, vectors_2, VAA, VBB, **kw):
    """Shape + directional pharmacophore combined alignment (cosine-weighted typed overlap)."""
    return coarse_fine_vol_color_align_many(centers_1, centers_2, ptype_1, ptype_2, anchors_1,
                                            anchors_2, VAA, VBB, vectors_1=vectors_1,
                                            vectors_2=vectors_2, directional=True, **kw)


# ------------------------------------------------------------------------------------------
# Step-by-step drivers (comparison forms)
# ------------------------------------------------------------------------------------------
class GraphedFineLoop:
    """Per-step shape/ESP fine loop captured once in a CUDA graph and replayed ``steps``
    times (the structure of the reference's accel/drivers/_graphed.py): every step launches
    the single-evaluation overlap kernel over all pose rows and the Tanimoto/Adam kernel.
    Rows are the reference's padded per-start expansion (K = pairs x starts)."""

    def __init__(self, A_k, B_k, N_k, M_k, U, q_seed, t_seed, *, alpha, lr, CA_k=None,
                 CB_k=None, lam=None):
        self.A, self.B = A_k.contiguous(), B_k.contiguous()
        self.CA = None if CA_k is None else CA_k.contiguous()
        self.CB = None if CB_k is None else CB_k.contiguous()
        self.N, self.M = N_k.to(_i32).contiguous(), M_k.to(_i32).contiguous()
        self.U = U.to(_f32).contiguous()
        self.qs, self.ts = q_seed.contiguous(), t_seed.contiguous()
        self.alpha, self.lr, self.lam = float(alpha), float(lr), lam
        K = self.qs.shape[0]
        dev = self.qs.device
        f = lambda *s: torch.empty(*s, dtype=_f32, device=dev)
        self.q, self.t = f(K, 4), f(K, 3)
        self.mq, self.vq, self.mt, self.vt = f(K, 4), f(K, 4), f(K, 3), f(K, 3)
        self.best, self.bq, self.bt = f(K), f(K, 4), f(K, 3)
        self.V, self.dQ, self.dT = f(K), f(K, 4), f(K, 3)
        self.graph = None

    def _reset(self):
        self.q.copy_(self.qs); self.t.copy_(self.ts)
        for b in (self.mq, self.vq, self.mt, self.vt):
            b.zero_()
        self.best.fill_(-float("inf")); self.bq.copy_(self.qs); self.bt.copy_(self.ts)

    def _step(self):
        L = _lib.load()
        K, npad, _ = self.A.shape
        st = stream_ptr(self.A.device)
        inv_lam = 0.0 if self.CA is None else 1.0 / float(self.lam)
        check(L.fss_overlap_grad(ptr(self.A), ptr(self.B), ptr(self.CA), ptr(self.CB),
                                 ptr(self.q), ptr(self.t), ptr(self.N), ptr(self.M), K, npad,
                                 self.B.shape[1], self.alpha, inv_lam, 1, ptr(self.V),
                                 ptr(self.dQ), ptr(self.dT), st), "graph step overlap")
        check(L.fss_tanimoto_adam_step(ptr(self.V), ptr(self.dQ), ptr(self.dT), ptr(self.U),
                                       ptr(self.q), ptr(self.t), ptr(self.mq), ptr(self.vq),
                                       ptr(self.mt), ptr(self.vt), ptr(self.best), ptr(self.bq),
                                       ptr(self.bt), K, self.lr, st), "graph step adam")

    def capture(self):
        self._reset()
        s = torch.cuda.Stream(self.A.device)
        s.wait_stream(torch.cuda.current_stream(self.A.device))
        with torch.cuda.stream(s):
            self._step()  # warm-up (sets the kernels' shared-memory attributes)
        torch.cuda.current_stream(self.A.device).wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._step()
        return self

    def run(self, steps: int):
        if self.graph is None:
            self.capture()
        self._reset()
        for _ in range(int(steps)):
            self.graph.replay()
        return self.best, self.bq, self.bt


def align_one_pair_per_launch(A, B, n, m, U, q_seed, t_seed, *, steps, alpha, lr, CA=None,
                              CB=None, lam=None):
    """The plain comparator: one pair at a time, two launches per Adam step (overlap over
    the pair's S start rows, then the Tanimoto/Adam kernel).  A (N,3), B (M,3) of ONE pair,
    q_seed (S,4), t_seed (S,3); returns that pair's per-start best score and pose."""
    S = q_seed.shape[0]
    dev = q_seed.device
    A_k = A.to(_f32).expand(S, -1, -1).contiguous()
    B_k = B.to(_f32).expand(S, -1, -1).contiguous()
    CA_k = None if CA is None else CA.to(_f32).expand(S, -1).contiguous()
    CB_k = None if CB is None else CB.to(_f32).expand(S, -1).contiguous()
    N_k = torch.full((S,), int(n), dtype=_i32, device=dev)
    M_k = torch.full((S,), int(m), dtype=_i32, device=dev)
    U_k = torch.full((S,), float(U), dtype=_f32, device=dev)
    loop = GraphedFineLoop(A_k, B_k, N_k, M_k, U_k, q_seed, t_seed, alpha=alpha, lr=lr,
                           CA_k=CA_k, CB_k=CB_k, lam=lam)
    loop._reset()
    for _ in range(int(steps)):
        loop._step()
    return loop.best, loop.bq, loop.bt
