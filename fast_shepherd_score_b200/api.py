"""Array-level public API: align batches of molecule clouds given as host arrays.

This is the call a user makes when the molecules are plain arrays rather than
``MoleculePair`` objects (the object-level drop-in is :mod:`fast_shepherd_score_b200.batch`).
Inputs are copied host->device once (pinned, asynchronous), every pair is aligned by the
fused kernel, and scores / poses / 4x4 transforms come back as numpy arrays.

Modes and their reference counterparts (shepherd_score.accel.batch.aligners):

=============  ==========================================  ====================
mode           channels                                    reference aligner
=============  ==========================================  ====================
vol / surf     Gaussian shape                              _align_batch_vol/_surf
vol_esp        shape x exp(-(dq)^2/lam), raw lam           _align_batch_vol_esp
surf_esp       shape x exp(-(dq)^2/lam), lam*LAM_SCALING   _align_batch_surf_esp
pharm          directional typed pharmacophores            _align_batch_pharm
vol_color      (1-w) shape + w directionless colour        _align_batch_vol_color
vol_pharm      (1-w) shape + w directional pharmacophore   (per-pair only in the reference)
=============  ==========================================  ====================
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import align as al
from . import kernels as K
from . import legacy_seeds, memory
from .layout import CloudSet, PharmSet, _offsets

LAM_SCALING = al.LAM_SCALING
# rows (pairs x grid poses) of one coarse-scoring launch of the translation-seeded path
TRANS_GRID_ROWS = 1 << 22

SHAPE_MODES = ("vol", "surf", "vol_esp", "surf_esp")
PHARM_MODES = ("pharm",)
COMBO_MODES = ("vol_color", "vol_pharm")
ESP_COMBO_MODES = ("vol_and_surf_esp",)
MODES = SHAPE_MODES + PHARM_MODES + COMBO_MODES + ESP_COMBO_MODES


@dataclass
class AlignOutput:
    scores: np.ndarray        # (P,) best Tanimoto (or combined) score
    q: np.ndarray             # (P, 4) best quaternion (w, x, y, z)
    t: np.ndarray             # (P, 3) best translation
    rows: Optional[tuple] = None  # per-start (score, q, t) as device tensors when requested

    @property
    def transforms(self) -> np.ndarray:
        """(P, 4, 4) SE(3) matrices, aligned = fit @ R^T + t (quaternions_to_SE3_batch,
        shepherd_score/alignment/utils/se3.py:16-30)."""
        return se3_from_qt(self.q, self.t)


def se3_from_qt(q: np.ndarray, t: np.ndarray) -> np.ndarray:
    q = np.asarray(q, np.float32)
    r, i, j, k = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.stack([1 - 2 * (j * j + k * k), 2 * (i * j - k * r), 2 * (i * k + j * r),
                  2 * (i * j + k * r), 1 - 2 * (i * i + k * k), 2 * (j * k - i * r),
                  2 * (i * k - j * r), 2 * (j * k + i * r), 1 - 2 * (i * i + j * j)],
                 1).reshape(-1, 3, 3)
    T = np.tile(np.eye(4, dtype=np.float32), (len(q), 1, 1))
    T[:, :3, :3] = R
    T[:, :3, 3] = t
    return T


class HostBatch:
    """Packed host-side input of one alignment batch (pinned for asynchronous H2D).

    ``pts`` (total, 4) float32 = x, y, z, charge; ``counts`` per molecule.  Pharmacophores:
    ``anc`` (total, 4) with the int32 type in w's bits, ``vec`` (total, 4).
    """

    def __init__(self, pts=None, counts=None, anc=None, vec=None, ph_counts=None, pin=True):
        def pinned(a):
            if a is None:
                return None
            t = torch.from_numpy(np.ascontiguousarray(a, np.float32))
            return t.pin_memory() if (pin and torch.cuda.is_available()) else t
        self.pts, self.anc, self.vec = pinned(pts), pinned(anc), pinned(vec)
        self.counts = None if counts is None else np.asarray(counts, np.int64)
        self.ph_counts = None if ph_counts is None else np.asarray(ph_counts, np.int64)

    @staticmethod
    def from_lists(points: Sequence = None, charges: Sequence = None, pharm_types=None,
                   pharm_anchors=None, pharm_vectors=None, pin=True) -> "HostBatch":
        pts = counts = anc = vec = phc = None
        if points is not None:
            counts = np.array([len(p) for p in points], np.int64)
            pts = np.zeros((int(counts.sum()), 4), np.float32)
            if len(pts):
                pts[:, :3] = np.concatenate([np.asarray(p, np.float32).reshape(-1, 3)
                                             for p in points])
                if charges is not None:
                    pts[:, 3] = np.concatenate([np.asarray(c, np.float32).reshape(-1)
                                                for c in charges])
        if pharm_anchors is not None:
            phc = np.array([len(a) for a in pharm_anchors], np.int64)
            anc = np.zeros((int(phc.sum()), 4), np.float32)
            vec = np.zeros((int(phc.sum()), 4), np.float32)
            if len(anc):
                anc[:, :3] = np.concatenate([np.asarray(a, np.float32).reshape(-1, 3)
                                             for a in pharm_anchors])
                ty = np.concatenate([np.asarray(t).reshape(-1) for t in pharm_types])
                ty = np.where((ty < 0) | (ty > 8), 8, ty).astype(np.int32)
                anc[:, 3] = ty.view(np.float32)
                if pharm_vectors is not None:
                    vec[:, :3] = np.concatenate([np.asarray(v, np.float32).reshape(-1, 3)
                                                 for v in pharm_vectors])
        return HostBatch(pts, counts, anc, vec, phc, pin)

    @property
    def nbytes(self) -> int:
        n = 0
        for a in (self.pts, self.anc, self.vec):
            if a is not None:
                n += a.numel() * 4
        for c in (self.counts, self.ph_counts):
            if c is not None:
                n += (len(c) + 1) * 4
        return n

    def to_device(self, device):
        cs = ps = None
        if self.pts is not None:
            off = torch.from_numpy(_offsets(self.counts))
            cs = CloudSet(self.pts.to(device, non_blocking=True),
                          off.to(device, non_blocking=True), self.counts,
                          int(self.counts.max()) if len(self.counts) else 0)
        if self.anc is not None:
            off = torch.from_numpy(_offsets(self.ph_counts))
            ps = PharmSet(self.anc.to(device, non_blocking=True),
                          self.vec.to(device, non_blocking=True),
                          off.to(device, non_blocking=True), self.ph_counts,
                          int(self.ph_counts.max()) if len(self.ph_counts) else 0)
        return cs, ps


def _kernel_lam(mode, lam):
    if mode == "surf_esp":
        return LAM_SCALING * float(lam)
    return float(lam)


def align_host(mode: str, ref: HostBatch, fit: HostBatch, *, pair_ref=None, pair_fit=None,
               alpha: float = 0.81, lam: float = 0.3, color_weight: float = 0.5,
               num_seeds: int = 50, steps: int = 200, lr: float = 0.1, device="cuda",
               return_rows: bool = False, **tile) -> AlignOutput:
    """Align pairs of host-resident clouds; results come back on the host.

    By default pair i is (ref molecule i, fit molecule i); ``pair_ref``/``pair_fit`` index
    arbitrary pairs (e.g. one query against a library).  For ``surf_esp`` ``lam`` is the
    user-facing weight (scaled by LAM_SCALING, aligners.py:383); for ``vol_esp`` it is raw.
    """
    if mode not in MODES:
        raise ValueError(f"unknown mode {mode!r}; valid: {list(MODES)}")
    device = torch.device(device)
    rc, rp = ref.to_device(device)
    fc, fp = fit.to_device(device)
    n_ref = len(ref.counts if ref.counts is not None else ref.ph_counts)
    n_fit = len(fit.counts if fit.counts is not None else fit.ph_counts)
    if pair_ref is None:
        if n_ref != n_fit:
            raise ValueError("ref and fit batches differ in size; pass pair_ref/pair_fit")
        pr = pf = torch.arange(n_ref, dtype=torch.int32)
    else:
        pr = torch.as_tensor(np.asarray(pair_ref), dtype=torch.int32)
        pf = torch.as_tensor(np.asarray(pair_fit), dtype=torch.int32)
    pr = pr.pin_memory().to(device, non_blocking=True) if torch.cuda.is_available() else pr
    pf = pf.pin_memory().to(device, non_blocking=True) if torch.cuda.is_available() else pf
    res = align_device(mode, rc, fc, rp, fp, pr, pf, alpha=alpha, lam=lam,
                       color_weight=color_weight, num_seeds=num_seeds, steps=steps, lr=lr,
                       **tile)
    sc, q, t = res
    out = torch.cat([sc[:, None], q, t], 1).to("cpu", non_blocking=False).numpy()
    return AlignOutput(out[:, 0].copy(), out[:, 1:5].copy(), out[:, 5:8].copy(),
                       res.rows if return_rows else None)


def align_device(mode, ref: Optional[CloudSet], fit: Optional[CloudSet],
                 ref_ph: Optional[PharmSet], fit_ph: Optional[PharmSet], pair_ref, pair_fit,
                 *, num_seeds=50, seeds=None, trans_centres: Optional[CloudSet] = None,
                 num_repeats_per_trans: int = 10, topk: int = 30,
                 max_chunk_pairs: Optional[int] = None, **kw):
    """Device-resident form of :func:`align_host` (all tensors already on the GPU).
    ``similarity`` / ``extended_points`` / ``only_extended`` apply to mode "pharm".

    The pairs run in memory-bounded chunks (:mod:`fast_shepherd_score_b200.memory`): a chunk
    holds at most 0.7 x the free device memory (or ``max_chunk_pairs`` pairs) and halves on
    an out-of-memory error.  Pairs are independent, so the results equal one call's.
    Everything else is :func:`_align_device_once`."""
    P = int(pair_ref.shape[0])
    if seeds is not None:
        starts, grid = int(seeds[0].shape[1]), 0
    elif trans_centres is not None:
        starts = topk
        grid = 5 + num_repeats_per_trans * int(trans_centres.max_points)
    else:
        starts, grid = int(num_seeds), 0

    def process(a, k):
        sd = None if seeds is None else (seeds[0][a:a + k], seeds[1][a:a + k])
        return _align_device_once(mode, ref, fit, ref_ph, fit_ph, pair_ref[a:a + k],
                                  pair_fit[a:a + k], num_seeds=num_seeds, seeds=sd,
                                  trans_centres=trans_centres,
                                  num_repeats_per_trans=num_repeats_per_trans, topk=topk, **kw)

    return memory.run_chunked(P, memory.align_bytes_per_pair(starts, grid), process,
                              pair_ref.device, max_chunk=max_chunk_pairs)


def _align_device_once(mode, ref: Optional[CloudSet], fit: Optional[CloudSet],
                       ref_ph: Optional[PharmSet], fit_ph: Optional[PharmSet], pair_ref,
                       pair_fit, *, alpha=0.81, lam=0.3, color_weight=0.5, num_seeds=50,
                       steps=200, lr=0.1, seeds=None, ref_self=None, fit_self=None,
                       ref_self_ph=None, fit_self_ph=None, similarity="tanimoto",
                       extended_points=False, only_extended=False,
                       trans_centres: Optional[CloudSet] = None,
                       num_repeats_per_trans: int = 10, topk: int = 30, **tile):
    """One call of :func:`align_device` without chunking.

    ``trans_centres`` (a CloudSet indexed like the reference molecules) selects the
    translation-seeded starts of the reference's ``trans_init=True``: per pair the legacy grid
    (identity, 4 principal-axis poses, ``num_repeats_per_trans`` Fibonacci rotations per
    centre) built from the clouds the reference seeds from (the surfaces for
    vol_and_surf_esp, the centred anchors for pharm, else the aligned clouds), every pose
    scored by a one-step launch, and the ``topk`` best refined for ``steps``."""
    if mode != "pharm" and (similarity != "tanimoto" or extended_points or only_extended):
        raise ValueError("similarity and extended points apply to mode 'pharm' only")
    if trans_centres is not None:
        if seeds is not None:
            raise ValueError("seeds and trans_centres are exclusive")
        kw = dict(alpha=alpha, lam=lam, color_weight=color_weight, lr=lr, ref_self=ref_self,
                  fit_self=fit_self, ref_self_ph=ref_self_ph, fit_self_ph=fit_self_ph,
                  similarity=similarity, extended_points=extended_points,
                  only_extended=only_extended, **tile)
        shift = None
        if mode == "pharm":
            rph, shift = _centred_pharm(ref_ph)
            g_ref, g_fit = _as_cloud(rph), _as_cloud(_centred_pharm(fit_ph)[0])
        elif mode in ESP_COMBO_MODES:
            g_ref, g_fit = tile["ref_surf"], tile["fit_surf"]
        else:
            g_ref, g_fit = ref, fit
        kw.update(al.coarse_tile(tile))
        # the grid holds 5 + 10 x centres poses per pair: score it in pair chunks of at most
        # TRANS_GRID_ROWS rows, so a library shard's grid never has to exist at once
        P = int(pair_ref.shape[0])
        g_max = 5 + num_repeats_per_trans * int(trans_centres.max_points)
        step = max(1, TRANS_GRID_ROWS // max(g_max, 1))
        sel_q, sel_t = [], []
        for a in range(0, P, step):
            pr, pf = pair_ref[a:a + step], pair_fit[a:a + step]
            gq, gt, G = legacy_seeds.grid_packed(g_ref, g_fit, trans_centres, pr, pf,
                                                 num_repeats_per_trans, shift)
            coarse = _align_device_once(mode, ref, fit, ref_ph, fit_ph, pr, pf, steps=1,
                                        seeds=(gq, gt), **kw)
            q_, t_ = legacy_seeds.select(coarse.rows[0], gq, gt, G, topk)
            sel_q.append(q_)
            sel_t.append(t_)
        seeds = (torch.cat(sel_q), torch.cat(sel_t)) if sel_q else None
        if seeds is None:
            seeds = (torch.zeros(0, topk, 4, device=pair_ref.device),
                     torch.zeros(0, topk, 3, device=pair_ref.device))
    if mode in ESP_COMBO_MODES:
        # shape centres steer the pose; tile holds the ESP-comparison sets and parameters
        if seeds is None:
            seeds = K.seeds(ref, fit, pair_ref, pair_fit, num_seeds)
        return al.align_packed("esp_combo", ref=ref, fit=fit, pair_ref=pair_ref,
                               pair_fit=pair_fit, seed_q=seeds[0], seed_t=seeds[1],
                               steps=steps, lr=lr, alpha=alpha, lam=lam, ref_self=ref_self,
                               fit_self=fit_self, **tile)
    if mode in SHAPE_MODES:
        esp = mode in ("vol_esp", "surf_esp")
        kl = _kernel_lam(mode, lam) if esp else None
        if seeds is None:
            seeds = K.seeds(ref, fit, pair_ref, pair_fit, num_seeds)
        return al.align_packed("esp" if esp else "shape", ref=ref, fit=fit, pair_ref=pair_ref,
                               pair_fit=pair_fit, seed_q=seeds[0], seed_t=seeds[1],
                               steps=steps, lr=lr, alpha=alpha, lam=kl, ref_self=ref_self,
                               fit_self=fit_self, **tile)
    if mode == "pharm":
        # the reference optimises each pair on per-cloud centred pharmacophores and folds
        # the centroids back into the translation (pharm.py:205-225, :509-517)
        rph, c_ref = _centred_pharm(ref_ph)
        fph, c_fit = _centred_pharm(fit_ph)
        if seeds is None:
            seeds = K.seeds(_as_cloud(rph), _as_cloud(fph), pair_ref, pair_fit, num_seeds)
        res = al.align_packed("pharm", ref_ph=rph, fit_ph=fph, pair_ref=pair_ref,
                              pair_fit=pair_fit, seed_q=seeds[0], seed_t=seeds[1],
                              steps=steps, lr=lr, ref_self=ref_self, fit_self=fit_self,
                              similarity=similarity,
                              pharm_extended=al.extended_code(extended_points, only_extended),
                              **tile)
        sc, q, t = res
        cr = c_ref[pair_ref.long()]
        cf = c_fit[pair_fit.long()]
        t = t - torch.einsum("bij,bj->bi", al._quat_rot(q), cf) + cr
        rows = res.rows
        out = al.AlignResult((sc, q, t))
        out.rows = rows
        return out
    if seeds is None:
        seeds = K.seeds(ref, fit, pair_ref, pair_fit, num_seeds)
    return al.align_packed("shape_color" if mode == "vol_color" else "shape_pharm", ref=ref,
                           fit=fit, ref_ph=ref_ph, fit_ph=fit_ph, pair_ref=pair_ref,
                           pair_fit=pair_fit, seed_q=seeds[0], seed_t=seeds[1], steps=steps,
                           lr=lr, alpha=alpha, color_weight=color_weight, ref_self=ref_self,
                           fit_self=fit_self, ref_self_ph=ref_self_ph, fit_self_ph=fit_self_ph,
                           **tile)


def _centred_pharm(ps: PharmSet):
    """The set with every molecule's anchors centred on its own centroid (types kept).  The
    centroid is a padded per-molecule sum (the reference's masked sum, pharm.py:215-219), so
    it is deterministic (an atomic scatter-add would make the last bits run-dependent)."""
    if ps.anc.dtype != torch.float32:
        raise ValueError("mode 'pharm' re-centres its anchors: it needs float32 sets")
    dev = ps.anc.device
    n = torch.as_tensor(ps.counts, device=dev)
    mol = torch.repeat_interleave(torch.arange(len(ps.counts), device=dev), n)
    xyz = ps.anc[:, :3]
    L = max(int(ps.max_points), 1)
    ar = torch.arange(L, device=dev)[None, :]
    off = torch.cumsum(n, 0) - n
    mask = ar < n[:, None]
    rows = torch.where(mask, off[:, None] + ar, torch.zeros_like(ar))
    pts = xyz[rows] if xyz.shape[0] else torch.zeros(len(ps.counts), L, 3, device=dev)
    c = torch.where(mask[..., None], pts, torch.zeros_like(pts)).sum(1)
    c = c / n.clamp(min=1).to(xyz.dtype)[:, None]
    anc = ps.anc.clone()
    anc[:, :3] = xyz - c[mol]
    return PharmSet(anc, ps.vec, ps.off, ps.counts, ps.max_points), c


def _as_cloud(ps: PharmSet) -> CloudSet:
    """Anchor positions of a pharmacophore set as a plain point cloud (for seeding)."""
    pts = torch.zeros_like(ps.anc)
    pts[:, :3] = ps.anc[:, :3]
    return CloudSet(pts, ps.off, ps.counts, ps.max_points)
