"""Per-mode batch aligners on duck-typed MoleculePair objects (the reference's seam).

Each ``_align_batch_<mode>(pairs, **kw)`` keeps the contract of the reference function of the
same name in shepherd_score/accel/batch/aligners.py: it reads the pairs' cached tensors
(``_ref_xyz_t``/``_fit_xyz_t``, ``_*_surf_t``, ``_*_surf_esp_t``, ``_*_pharm_{types,ancs,vecs}_t``),
building a missing one from ``p.ref_molec`` / ``p.fit_molec`` arrays as the reference's
``_batch_upload`` does (aligners.py:45-94), aligns every pair, and writes
``p.transform_<mode>`` (a float32 (4,4) CPU tensor, aligned = fit @ R^T + t) and
``p.sim_aligned_<mode>`` (a float) in place.

Differences from the reference's bucketed path: no padding buckets (clouds are packed), one
fused kernel launch per call, and ``num_repeats`` / ``lr`` are honoured for every mode (the
reference's vol/surf path fixes them, aligners.py:151,180).  A batch whose pairs all share the
same reference tensor (one query against many fits, as the screen builds it) stages that
reference once.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from . import api
from .layout import CloudSet, PharmSet
from .modes import MODE_ATTRS, seeds_for

_f32 = torch.float32


def _device_of(pairs) -> torch.device:
    dev = getattr(pairs[0], "device", None)
    dev = torch.device(dev) if dev is not None else torch.device("cuda")
    if dev.type != "cuda":
        raise ValueError("backend='cuda' needs the pairs on a CUDA device (this backend has "
                         "no CPU path); use backend='numba' of shepherd_score for CPU")
    return dev


def _ensure(pairs, attr, src, dtype, device):
    """p.<attr> as a tensor on `device`, built from p.ref_molec/fit_molec.<src> (an attribute
    name, or a callable of the molecule) if absent."""
    side = "ref_molec" if attr.startswith("_ref_") else "fit_molec"
    out = []
    for p in pairs:
        t = getattr(p, attr, None)
        if t is None:
            mol = getattr(p, side, None)
            if mol is None:
                arr = None
            elif callable(src):
                arr = src(mol)
            else:
                arr = getattr(mol, src, None)
            if arr is None:
                raise ValueError(f"pair is missing {attr} and {side}.{src}")
            t = torch.as_tensor(np.asarray(arr), dtype=dtype)
            setattr(p, attr, t)
        if t.device != device:
            t = t.to(device, non_blocking=True)
            setattr(p, attr, t)
        out.append(t)
    return out


def _shared(tensors) -> bool:
    return len(tensors) > 1 and all(t is tensors[0] for t in tensors)


def _cloud_set(tensors, charges=None, device=None, dedup=None) -> tuple:
    """Pack per-pair clouds; returns (CloudSet, marker) where the marker is not None when
    every pair shares molecule 0 (one staged reference for a query-vs-library batch)."""
    if dedup is None:
        dedup = _shared(tensors)
    if dedup:
        tensors = tensors[:1]
        charges = charges[:1] if charges is not None else None
        idx = torch.zeros(0, dtype=torch.int32)
    else:
        idx = None
    counts = [int(t.shape[0]) for t in tensors]
    pts = torch.zeros(sum(counts), 4, dtype=_f32, device=device)
    if counts and sum(counts):
        pts[:, :3] = torch.cat([t.reshape(-1, 3).to(_f32) for t in tensors])
        if charges is not None:
            pts[:, 3] = torch.cat([c.reshape(-1).to(_f32) for c in charges])
    off = torch.zeros(len(counts) + 1, dtype=torch.int32)
    off[1:] = torch.cumsum(torch.tensor(counts, dtype=torch.int64), 0).to(torch.int32)
    cs = CloudSet(pts, off.to(device), np.array(counts, np.int64), max(counts) if counts else 0)
    return cs, idx


def _pharm_set(types, ancs, vecs, device, dedup=None) -> tuple:
    if dedup is None:
        dedup = _shared(ancs)
    if dedup:
        types, ancs, vecs = types[:1], ancs[:1], (vecs[:1] if vecs is not None else None)
        idx = torch.zeros(0, dtype=torch.int32)
    else:
        idx = None
    counts = [int(a.shape[0]) for a in ancs]
    n = sum(counts)
    anc = torch.zeros(n, 4, dtype=_f32, device=device)
    vec = torch.zeros(n, 4, dtype=_f32, device=device)
    if n:
        anc[:, :3] = torch.cat([a.reshape(-1, 3).to(_f32) for a in ancs])
        ty = torch.cat([t.reshape(-1).to(torch.int64) for t in types])
        ty = torch.where((ty < 0) | (ty > 8), torch.full_like(ty, 8), ty).to(torch.int32)
        anc[:, 3] = ty.view(torch.float32)
        if vecs is not None:
            vec[:, :3] = torch.cat([v.reshape(-1, 3).to(_f32) for v in vecs])
    off = torch.zeros(len(counts) + 1, dtype=torch.int32)
    off[1:] = torch.cumsum(torch.tensor(counts, dtype=torch.int64), 0).to(torch.int32)
    return PharmSet(anc, vec, off.to(device), np.array(counts, np.int64),
                    max(counts) if counts else 0), idx


def _pairs_index(n, ref_idx, fit_idx, device):
    r = torch.zeros(n, dtype=torch.int32) if ref_idx is not None else torch.arange(n, dtype=torch.int32)
    f = torch.zeros(n, dtype=torch.int32) if fit_idx is not None else torch.arange(n, dtype=torch.int32)
    return r.to(device), f.to(device)


def _write(pairs, mode, out):
    sc, q, t = out
    host = torch.cat([sc[:, None], q, t], 1).cpu()
    T = torch.from_numpy(api.se3_from_qt(host[:, 1:5].numpy(), host[:, 5:8].numpy()))
    tf_attr, sc_attr = MODE_ATTRS[mode]
    scores = host[:, 0].tolist()
    for p, s, S in zip(pairs, scores, T):
        setattr(p, tf_attr, S)
        setattr(p, sc_attr, float(s))
    return np.asarray(scores, dtype=float)


def _align(pairs, mode, ref, fit, ref_ph, fit_ph, r_idx, f_idx, **kw):
    dev = (ref.pts.device if ref is not None else ref_ph.anc.device)
    pr, pf = _pairs_index(len(pairs), r_idx, f_idx, dev)
    out = api.align_device(mode, ref, fit, ref_ph, fit_ph, pr, pf, **kw)
    return _write(pairs, mode, out)


def _trans_kw(pairs, trans_init, attr, src, dev, r_idx, num_repeats_per_trans=10, topk=30):
    """Keyword arguments of the translation-seeded starts (trans_init=True): the reference
    molecules' translation centres (p.<attr>, built from ref_molec.<src> if absent) packed like
    the reference clouds (shared when the reference is)."""
    if not trans_init:
        return {}
    t = _ensure(pairs, attr, src, _f32, dev)
    centres, _ = _cloud_set(t, device=dev, dedup=r_idx is not None)
    return dict(trans_centres=centres, num_repeats_per_trans=num_repeats_per_trans, topk=topk)


def _align_batch_vol(pairs, *, alpha: float = 0.81, steps_fine: int = 100,
                     num_repeats: Optional[int] = None, lr: float = 0.075):
    """Volumetric (heavy-atom) shape alignment; writes transform_vol_noH / sim_aligned_vol_noH."""
    if not pairs:
        return
    dev = _device_of(pairs)
    ref, ri = _cloud_set(_ensure(pairs, "_ref_xyz_t", "atom_pos", _f32, dev), device=dev)
    fit, fi = _cloud_set(_ensure(pairs, "_fit_xyz_t", "atom_pos", _f32, dev), device=dev)
    return _align(pairs, "vol", ref, fit, None, None, ri, fi, alpha=alpha, steps=steps_fine,
                  lr=lr, num_seeds=num_repeats or seeds_for("vol"))


def _align_batch_surf(pairs, *, alpha: float = 0.81, steps_fine: int = 100,
                      num_repeats: Optional[int] = None, lr: float = 0.075):
    """Surface-point shape alignment; writes transform_surf / sim_aligned_surf."""
    if not pairs:
        return
    dev = _device_of(pairs)
    ref, ri = _cloud_set(_ensure(pairs, "_ref_surf_t", "surf_pos", _f32, dev), device=dev)
    fit, fi = _cloud_set(_ensure(pairs, "_fit_surf_t", "surf_pos", _f32, dev), device=dev)
    return _align(pairs, "surf", ref, fit, None, None, ri, fi, alpha=alpha, steps=steps_fine,
                  lr=lr, num_seeds=num_repeats or seeds_for("surf"))


def _align_batch_surf_esp(pairs, *, alpha: float, lam: float, trans_init: bool = False,
                          num_repeats: int = 50, num_repeats_per_trans: int = 10,
                          topk: int = 30, steps_fine: int = 100, lr: float = 0.075):
    """Surface ESP alignment (lam scaled by LAM_SCALING, aligners.py:383); writes
    transform_surf_esp / sim_aligned_surf_esp."""
    if not pairs:
        return
    dev = _device_of(pairs)
    pts_r = _ensure(pairs, "_ref_surf_t", "surf_pos", _f32, dev)
    pts_f = _ensure(pairs, "_fit_surf_t", "surf_pos", _f32, dev)
    esp_r = _ensure(pairs, "_ref_surf_esp_t", "surf_esp", _f32, dev)
    esp_f = _ensure(pairs, "_fit_surf_esp_t", "surf_esp", _f32, dev)
    ref, ri = _cloud_set(pts_r, esp_r, device=dev)
    fit, fi = _cloud_set(pts_f, esp_f, device=dev)
    # trans_init: translation centres are the reference atoms (aligners.py:408-412)
    tk = _trans_kw(pairs, trans_init, "_ref_xyz_t", "atom_pos", dev, ri, num_repeats_per_trans,
                   topk)
    return _align(pairs, "surf_esp", ref, fit, None, None, ri, fi, alpha=alpha, lam=lam,
                  steps=steps_fine, lr=lr, num_seeds=num_repeats or seeds_for("surf_esp"), **tk)


_align_batch_esp = _align_batch_surf_esp


def _align_batch_vol_esp(pairs, *, lam: float, alpha: float = 0.81, trans_init: bool = False,
                         num_repeats: int = 50, num_repeats_per_trans: int = 10,
                         topk: int = 30, steps_fine: int = 100, lr: float = 0.075):
    """Heavy-atom charge-weighted alignment (raw lam, aligners.py:642); writes
    transform_vol_esp_noH / sim_aligned_vol_esp_noH.  Uses ``_*_xyz_noH_t`` /
    ``_*_xyz_esp_t`` when present, else atom positions and partial charges."""
    if not pairs:
        return
    dev = _device_of(pairs)
    for side in ("ref", "fit"):
        for p in pairs:
            if getattr(p, f"_{side}_xyz_noH_t", None) is None and \
                    getattr(p, f"_{side}_xyz_t", None) is not None:
                setattr(p, f"_{side}_xyz_noH_t", getattr(p, f"_{side}_xyz_t"))
    pts_r = _ensure(pairs, "_ref_xyz_noH_t", "atom_pos", _f32, dev)
    pts_f = _ensure(pairs, "_fit_xyz_noH_t", "atom_pos", _f32, dev)
    ch_r = _ensure(pairs, "_ref_xyz_esp_t", "partial_charges", _f32, dev)
    ch_f = _ensure(pairs, "_fit_xyz_esp_t", "partial_charges", _f32, dev)
    ref, ri = _cloud_set(pts_r, ch_r, device=dev)
    fit, fi = _cloud_set(pts_f, ch_f, device=dev)
    tk = _trans_kw(pairs, trans_init, "_ref_xyz_t", "atom_pos", dev, ri, num_repeats_per_trans,
                   topk)
    return _align(pairs, "vol_esp", ref, fit, None, None, ri, fi, alpha=alpha, lam=lam,
                  steps=steps_fine, lr=lr, num_seeds=num_repeats or seeds_for("vol_esp"), **tk)


def _conformer_positions(mol):
    """All-atom (with hydrogens) positions of a molecule's RDKit conformer."""
    rd = getattr(mol, "mol", None)
    return None if rd is None else rd.GetConformer().GetPositions()


def _align_batch_vol_and_surf_esp(pairs, *, alpha: float, lam: float = 0.001,
                                  probe_radius: float = 1.0, esp_weight: float = 0.5,
                                  trans_init: bool = False, num_repeats: int = 50,
                                  num_repeats_per_trans: int = 10, topk: int = 30,
                                  steps_fine: int = 100, lr: float = 0.075,
                                  esp_stride: int = 1):
    """ShaEP-style combo (aligners.py:651-864): shape centres (heavy atoms when alpha is 0.81,
    else surface points) steer the pose; the score adds the surface ESP comparison against the
    other molecule's atoms with hydrogens.  Writes transform_vol_and_surf_esp /
    sim_aligned_vol_and_surf_esp."""
    if not pairs:
        return
    dev = _device_of(pairs)
    sets = {}
    for side in ("ref", "fit"):
        surf = _ensure(pairs, f"_{side}_surf_t", "surf_pos", _f32, dev)
        esp = _ensure(pairs, f"_{side}_surf_esp_t", "surf_esp", _f32, dev)
        wh = _ensure(pairs, f"_{side}_centers_w_H_t", _conformer_positions, _f32, dev)
        q = _ensure(pairs, f"_{side}_partial_t", "partial_charges", _f32, dev)
        rad = _ensure(pairs, f"_{side}_radii_t", "radii", _f32, dev)
        cent = (_ensure(pairs, f"_{side}_xyz_t", "atom_pos", _f32, dev) if alpha == 0.81
                else surf)
        dd = _shared(surf) and _shared(wh) and _shared(cent)
        centres, idx = _cloud_set(cent, device=dev, dedup=dd)
        atoms, _ = _cloud_set(wh, q, device=dev, dedup=dd)
        surfs, _ = _cloud_set(surf, esp, device=dev, dedup=dd)
        radii = torch.cat([r.reshape(-1).to(_f32) for r in (rad[:1] if dd else rad)]).to(dev)
        sets[side] = (centres, idx, atoms, radii, surfs)
    (ref, ri, ra, rr, rs), (fit, fi, fa, fr, fs) = sets["ref"], sets["fit"]
    # trans_init: centres are the reference atoms (aligners.py:712-727, :816-822)
    tk = _trans_kw(pairs, trans_init, "_ref_xyz_t", "atom_pos", dev, ri, num_repeats_per_trans,
                   topk)
    return _align(pairs, "vol_and_surf_esp", ref, fit, None, None, ri, fi, alpha=alpha, lam=lam,
                  steps=steps_fine, lr=lr,
                  num_seeds=num_repeats or seeds_for("vol_and_surf_esp"),
                  ref_atoms=ra, fit_atoms=fa, ref_radii=rr, fit_radii=fr, ref_surf=rs,
                  fit_surf=fs, probe_radius=probe_radius, esp_weight=esp_weight,
                  esp_stride=esp_stride, **tk)


_align_batch_esp_combo = _align_batch_vol_and_surf_esp


def _pharm_inputs(pairs, dev, with_vectors=True):
    tr = _ensure(pairs, "_ref_pharm_types_t", "pharm_types", torch.int64, dev)
    tf = _ensure(pairs, "_fit_pharm_types_t", "pharm_types", torch.int64, dev)
    ar = _ensure(pairs, "_ref_pharm_ancs_t", "pharm_ancs", _f32, dev)
    af = _ensure(pairs, "_fit_pharm_ancs_t", "pharm_ancs", _f32, dev)
    vr = _ensure(pairs, "_ref_pharm_vecs_t", "pharm_vecs", _f32, dev) if with_vectors else None
    vf = _ensure(pairs, "_fit_pharm_vecs_t", "pharm_vecs", _f32, dev) if with_vectors else None
    rp, ri = _pharm_set(tr, ar, vr, dev)
    fp, fi = _pharm_set(tf, af, vf, dev)
    return rp, fp, ri, fi


def _align_batch_pharm(pairs, *, similarity: str = "tanimoto", extended_points: bool = False,
                       only_extended: bool = False, trans_init: bool = False,
                       num_repeats: Optional[int] = None, topk: int = 30,
                       steps_fine: int = 100, lr: float = 0.075):
    """Directional pharmacophore alignment; writes transform_pharm / sim_aligned_pharm."""
    if not pairs:
        return
    dev = _device_of(pairs)
    rp, fp, ri, fi = _pharm_inputs(pairs, dev)
    # trans_init: centres are the reference anchors (aligners.py:932, :966-967)
    tk = _trans_kw(pairs, trans_init, "_ref_pharm_ancs_t", "pharm_ancs", dev, ri, 10, topk)
    return _align(pairs, "pharm", None, None, rp, fp, ri, fi, steps=steps_fine, lr=lr,
                  num_seeds=num_repeats or seeds_for("pharm"), similarity=similarity,
                  extended_points=extended_points, only_extended=only_extended, **tk)


def _align_batch_vol_color(pairs, *, alpha: float = 0.81, color_weight: float = 0.5,
                           trans_init: bool = False, num_repeats: int = 50,
                           num_repeats_per_trans: int = 10, topk: int = 30,
                           steps_fine: int = 100, lr: float = 0.075):
    """Atom shape + directionless colour; writes transform_vol_color / sim_aligned_vol_color."""
    return _combo(pairs, "vol_color", alpha, color_weight, trans_init, num_repeats, steps_fine,
                  lr, num_repeats_per_trans, topk)


def _align_batch_vol_pharm(pairs, *, alpha: float = 0.81, color_weight: float = 0.5,
                           trans_init: bool = False, num_repeats: int = 50,
                           num_repeats_per_trans: int = 10, topk: int = 30,
                           steps_fine: int = 100, lr: float = 0.075, **_):
    """Atom shape + directional (cosine-weighted) pharmacophores with one shared pose;
    writes transform_vol_pharm / sim_aligned_vol_pharm."""
    return _combo(pairs, "vol_pharm", alpha, color_weight, trans_init, num_repeats, steps_fine,
                  lr, num_repeats_per_trans, topk)


def _combo(pairs, mode, alpha, color_weight, trans_init, num_repeats, steps_fine, lr,
           num_repeats_per_trans=10, topk=30):
    if not pairs:
        return
    dev = _device_of(pairs)
    xr = _ensure(pairs, "_ref_xyz_t", "atom_pos", _f32, dev)
    xf = _ensure(pairs, "_fit_xyz_t", "atom_pos", _f32, dev)
    vec = mode == "vol_pharm"
    tr = _ensure(pairs, "_ref_pharm_types_t", "pharm_types", torch.int64, dev)
    tf = _ensure(pairs, "_fit_pharm_types_t", "pharm_types", torch.int64, dev)
    ar = _ensure(pairs, "_ref_pharm_ancs_t", "pharm_ancs", _f32, dev)
    af = _ensure(pairs, "_fit_pharm_ancs_t", "pharm_ancs", _f32, dev)
    vr = _ensure(pairs, "_ref_pharm_vecs_t", "pharm_vecs", _f32, dev) if vec else None
    vf = _ensure(pairs, "_fit_pharm_vecs_t", "pharm_vecs", _f32, dev) if vec else None
    # one molecule table per side: dedup only when atoms AND pharmacophores are shared
    dr = _shared(xr) and _shared(ar)
    df = _shared(xf) and _shared(af)
    ref, ri = _cloud_set(xr, device=dev, dedup=dr)
    fit, fi = _cloud_set(xf, device=dev, dedup=df)
    rp, _ = _pharm_set(tr, ar, vr, dev, dedup=dr)
    fp, _ = _pharm_set(tf, af, vf, dev, dedup=df)
    # trans_init: centres are the reference atoms (aligners.py:1064, :1109-1113)
    tk = _trans_kw(pairs, trans_init, "_ref_xyz_t", "atom_pos", dev, ri, num_repeats_per_trans,
                   topk)
    return _align(pairs, mode, ref, fit, rp, fp, ri, fi, alpha=alpha, color_weight=color_weight,
                  steps=steps_fine, lr=lr, num_seeds=num_repeats or seeds_for(mode), **tk)
