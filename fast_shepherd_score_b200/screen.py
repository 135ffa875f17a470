"""Screening front-end: ``screen()`` / ``screen_many()`` over a sharded profile store.

Mirrors shepherd_score/screen.py for the CUDA path: the library is a ``ProfileStore``
(:mod:`fast_shepherd_score_b200.store`, the reference's on-disk format; a store object of
shepherd_score itself is accepted too), ``screen_many`` (:1038) streams every shard once for
a whole query panel, ``screen`` (:1141) is the one-query wrapper, ``Hit`` (:75) is
``(score, id, transform)``.

Each shard is uploaded once (float16 coordinates expand to float32 on the device) and kept
as packed device clouds; every query is one reference molecule staged once per work item,
aligned against all of the shard's molecules by one fused kernel launch.  Top-K survivors
are selected on the device, so only K transforms are built per shard and query.
"""
from __future__ import annotations

import heapq
import os
from collections import namedtuple
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import api, library
from .layout import CloudSet, PharmSet, _offsets
from .modes import canonical, seeds_for, steps_for
from .store import ProfileStore  # noqa: F401  (re-exported: the screening entry points take it)

Hit = namedtuple("Hit", ["score", "id", "transform"])

_SURF_ALPHA_MODES = {"surf", "surf_esp"}
_SCREEN_MODES = ("vol", "vol_esp", "surf", "surf_esp", "vol_and_surf_esp", "pharm", "vol_color",
                 "vol_pharm")


def ALPHA(num_points):
    """Surface Gaussian width for a point count: quadratic interpolation of the reference's
    calibration table (score/constants.py:9-13)."""
    from scipy.interpolate import interp1d
    f = interp1d(np.array([50, 100, 150, 200, 300, 400]),
                 np.array([0.6011, 0.8668, 1.022, 1.118, 1.216, 1.258]), "quadratic")
    return float(f(num_points))


# -----------------------------------------------------------------------------------------
# Device-side shard expansion
# -----------------------------------------------------------------------------------------
def _dev(a, device, dtype=torch.float32):
    """Upload an array in its stored dtype, then convert on the device (radii only)."""
    return library.upload(a, device).to(dtype)


# the fit sets the fused kernel reads directly keep a float16 store's dtype on the device (the
# kernels widen it while staging); the pharmacophore mode re-centres its anchors and the
# ShaEP combo mode has no float16 form, so those two widen on upload
_KEEP_HALF = ("vol", "vol_esp", "surf", "surf_esp", "vol_color", "vol_pharm")


def shard_to_device(arrs: dict, mode: str, device, alpha: float = 0.81, widen: bool = False):
    """(fit CloudSet or None, fit PharmSet or None, extra kwargs) of one shard for `mode`;
    vol_and_surf_esp adds the atoms with hydrogens, their radii and the surfaces.  Columns
    of a float16 store stay float16 for the modes in ``_KEEP_HALF`` unless ``widen``."""
    widen = widen or mode not in _KEEP_HALF
    csr, dense = library.cloud_from_csr, library.cloud_from_dense
    if mode == "vol_and_surf_esp":
        # shape centres: heavy atoms at alpha 0.81, else the surface (aligners.py:795-803)
        surf = dense(arrs["surf_pos"], device, arrs["surf_esp"], widen=True)
        cs = (csr(arrs["atom_pos"], arrs["atom_off"], device, widen=True) if alpha == 0.81
              else dense(arrs["surf_pos"], device, widen=True))
        atoms = csr(arrs["cwh"], arrs["all_off"], device, arrs["charges"], widen=True)
        return cs, None, dict(fit_atoms=atoms, fit_radii=_dev(arrs["radii"], device),
                              fit_surf=surf)
    if mode in ("vol", "vol_color", "vol_pharm"):
        cs = csr(arrs["atom_pos"], arrs["atom_off"], device, widen=widen)
    elif mode == "vol_esp":
        cs = csr(arrs["atom_pos"], arrs["atom_off"], device, arrs["charges"], widen=widen)
    elif mode == "surf":
        cs = dense(arrs["surf_pos"], device, widen=widen)
    elif mode == "surf_esp":
        cs = dense(arrs["surf_pos"], device, arrs["surf_esp"], widen=widen)
    else:
        cs = None
    ps = None
    if mode in ("pharm", "vol_color", "vol_pharm"):
        ps = library.pharm_from_csr(arrs["pharm_types"], arrs["pharm_ancs"], arrs["pharm_vecs"],
                                    arrs["pharm_off"], device,
                                    with_vectors=(mode != "vol_color"), widen=widen)
    return cs, ps, {}


def query_to_device(q, mode: str, device, alpha: float = 0.81):
    """One query molecule (attributes atom_pos / surf_pos / surf_esp / partial_charges /
    pharm_types / pharm_ancs / pharm_vecs, and centers_w_H / radii for vol_and_surf_esp) as a
    one-molecule (CloudSet, PharmSet, extra kwargs)."""
    g = lambda name: getattr(q, name, None) if not isinstance(q, dict) else q.get(name)
    if mode == "vol_and_surf_esp":
        cwh = g("centers_w_H")
        if cwh is None and g("mol") is not None:
            cwh = g("mol").GetConformer().GetPositions()
        cs = CloudSet.from_arrays([g("atom_pos") if alpha == 0.81 else g("surf_pos")],
                                  device=device)
        atoms = CloudSet.from_arrays([np.asarray(cwh, np.float32)], [g("partial_charges")],
                                     device=device)
        surf = CloudSet.from_arrays([g("surf_pos")], [g("surf_esp")], device=device)
        radii = torch.as_tensor(np.asarray(g("radii"), np.float32), device=device)
        return cs, None, dict(ref_atoms=atoms, ref_radii=radii, ref_surf=surf)
    cs = ps = None
    if mode in ("vol", "vol_color", "vol_pharm"):
        cs = CloudSet.from_arrays([g("atom_pos")], device=device)
    elif mode == "vol_esp":
        cs = CloudSet.from_arrays([g("atom_pos")], [g("partial_charges")], device=device)
    elif mode == "surf":
        cs = CloudSet.from_arrays([g("surf_pos")], device=device)
    elif mode == "surf_esp":
        cs = CloudSet.from_arrays([g("surf_pos")], [g("surf_esp")], device=device)
    if mode in ("pharm", "vol_color", "vol_pharm"):
        ps = PharmSet.from_arrays([g("pharm_types")], [g("pharm_ancs")],
                                  None if mode == "vol_color" else [g("pharm_vecs")],
                                  device=device)
    return cs, ps, {}


def _query_centres(q, mode: str, device) -> CloudSet:
    """The query's translation centres for trans_init: its heavy atoms, or its pharmacophore
    anchors in mode pharm (the reference's aligners take them from the reference molecule)."""
    g = lambda name: getattr(q, name, None) if not isinstance(q, dict) else q.get(name)
    pts = g("pharm_ancs") if mode == "pharm" else g("atom_pos")
    if pts is None:
        raise ValueError("trans_init needs the query's "
                         + ("pharm_ancs" if mode == "pharm" else "atom_pos"))
    return CloudSet.from_arrays([np.asarray(pts, np.float32)], device=device)


def _centred_query(q):
    """A copy of the query with every coordinate array shifted by its atom COM."""
    get = (lambda n: q.get(n)) if isinstance(q, dict) else (lambda n: getattr(q, n, None))
    c = np.asarray(get("atom_pos"), np.float32).mean(0)
    out = {}
    cwh = get("centers_w_H")
    if cwh is None and get("mol") is not None:
        cwh = get("mol").GetConformer().GetPositions()
    out["centers_w_H"] = None if cwh is None else np.asarray(cwh, np.float32) - c
    for n in ("atom_pos", "surf_pos", "pharm_ancs"):
        v = get(n)
        out[n] = None if v is None else np.asarray(v, np.float32) - c
    for n in ("surf_esp", "partial_charges", "pharm_types", "pharm_vecs", "radii"):
        out[n] = get(n)
    return out


class _TopK:
    """Bounded max-list keyed on score (screen.py:898-935)."""

    def __init__(self, k):
        self.k, self.heap, self._c = k, [], 0

    def push(self, score, id_, transform):
        self._c += 1
        item = (score, self._c, id_, transform)
        if len(self.heap) < self.k:
            heapq.heappush(self.heap, item)
        elif score > self.heap[0][0]:
            heapq.heapreplace(self.heap, item)

    def threshold(self):
        return self.heap[0][0] if len(self.heap) >= self.k else -np.inf

    def sorted(self):
        return [Hit(score=s, id=i, transform=t)
                for (s, _, i, t) in sorted(self.heap, key=lambda x: x[0], reverse=True)]


def _batch_kwargs(mode, ak, alpha):
    steps = ak.get("max_num_steps", steps_for(mode))
    lr = ak.get("lr", 0.075 if mode in ("vol", "surf") else 0.1)
    kw = dict(steps=steps, lr=lr, num_seeds=ak.get("num_repeats", seeds_for(mode)))
    if mode in ("vol", "surf", "vol_esp", "surf_esp", "vol_color", "vol_pharm"):
        kw["alpha"] = alpha
    if mode == "surf_esp":
        kw["lam"] = ak.get("lam", 0.3)
    if mode == "vol_esp":
        kw["lam"] = ak["lam"]
    if mode in ("vol_color", "vol_pharm"):
        kw["color_weight"] = ak.get("color_weight", 0.5)
    if mode == "vol_and_surf_esp":
        kw.update(alpha=alpha, lam=ak.get("lam", 0.001),
                  probe_radius=ak.get("probe_radius", 1.0),
                  esp_weight=ak.get("esp_weight", 0.5), esp_stride=ak.get("esp_stride", 1))
    # an explicit kernel tile (lanes_per_pose, chunks, ...) passes through to the launch
    from .align import TILE_KEYS
    kw.update({k: int(ak[k]) for k in TILE_KEYS if ak.get(k)})
    return kw


def _screen_shards(qs, store: ProfileStore, mode: str, shards, kw: dict, ak: dict, alpha,
                   top_k: int, center: bool, device, so=None, progress: bool = False):
    """Align the (already centred) queries ``qs`` against the store shards yielded by
    ``shards`` on ``device``; returns one _TopK per query.  ``so``: per-query full score
    arrays to fill (or None)."""
    so = so or [None] * len(qs)
    heaps = [_TopK(top_k) for _ in qs]
    qdev = [query_to_device(q, mode, device, alpha) for q in qs]
    # trans_init: the legacy translation-seeded starts with the query's atoms (anchors for
    # pharm) as translation centres, as the reference's per-pair screening path aligns
    # MoleculePair(query, library molecule) (screen.py:1006-1008); vol and surf ignore it there
    trans = bool(ak.get("trans_init")) and mode not in ("vol", "surf")
    tks = [dict(trans_centres=_query_centres(q, mode, device),
                num_repeats_per_trans=int(ak.get("num_repeats_per_trans", 10)),
                topk=int(ak.get("topk", 30))) if trans else {} for q in qs]
    done = 0
    for si in shards:
        sh, arrs = store.read_shard(si)
        if center and not store.pre_centered:
            arrs = _center_shard(arrs, mode)
        # the translation-seeded grid reads the fit clouds on the host side: float32 there
        fit, fit_ph, fit_x = shard_to_device(arrs, mode, device, alpha, widen=trans)
        K = int(sh["n"])
        pr = torch.zeros(K, dtype=torch.int32, device=device)
        pf = torch.arange(K, dtype=torch.int32, device=device)
        ids = arrs["ids"]
        for qi, (rc, rp, ref_x) in enumerate(qdev):
            sc, q, t = api.align_device(mode, rc, fit, rp, fit_ph, pr, pf, **kw, **ref_x,
                                        **fit_x, **tks[qi])
            if so[qi] is not None:
                so[qi][sh["start"]:sh["start"] + K] = sc.cpu().numpy()
            k = min(top_k, K)
            top_s, top_i = torch.topk(sc, k)
            keep = top_s > heaps[qi].threshold()
            top_s, top_i = top_s[keep], top_i[keep]
            T = api.se3_from_qt(q[top_i].cpu().numpy(), t[top_i].cpu().numpy())
            for s_, i, tf in zip(top_s.cpu().tolist(), top_i.cpu().tolist(), T):
                heaps[qi].push(float(s_), _id_to_py(ids[i]), tf)
        done += K
        if progress:
            print(f"[screen] {done}/{len(store)} library molecules aligned x {len(qs)} queries",
                  flush=True)
    return heaps


def _screen_worker(rank, store_path, qs, mode, kw, ak, alpha, top_k, center, shard_q, out_q):
    """One GPU of a multi-GPU screen: pulls shard indices off ``shard_q`` until a None
    sentinel, aligns them on cuda:rank and sends its per-query top-K lists to ``out_q``."""
    try:
        torch.cuda.set_device(rank)
        store = ProfileStore.open(store_path)

        def shards():
            while True:
                idx = shard_q.get()
                if idx is None:
                    return
                yield idx
        heaps = _screen_shards(qs, store, mode, shards(), kw, ak, alpha, top_k, center,
                               torch.device("cuda", rank))
        torch.cuda.synchronize()
        out_q.put((rank, [h.heap for h in heaps]))
    except Exception:                                   # relayed to the parent
        import traceback
        out_q.put((rank, "__ERR__", traceback.format_exc()))


def _screen_multi_gpu(qs, store: ProfileStore, mode, ndev, kw, ak, alpha, top_k, center):
    """Process-per-GPU screen (the structure of the reference's _screen_many_multigpu,
    screen.py:1237-1297): ``ndev`` spawned workers stream disjoint shards from one queue, each
    keeps its own top-K per query, and the parent merges them."""
    import torch.multiprocessing as mp
    ndev = max(1, min(int(ndev), torch.cuda.device_count()))
    ctx = mp.get_context("spawn")
    shard_q, out_q = ctx.Queue(), ctx.Queue()
    for idx in range(store.num_shards):
        shard_q.put(idx)
    for _ in range(ndev):
        shard_q.put(None)                               # one sentinel per worker
    procs = [ctx.Process(target=_screen_worker,
                         args=(r, store.path, qs, mode, kw, ak, alpha, top_k, center, shard_q,
                               out_q)) for r in range(ndev)]
    for p in procs:
        p.start()
    results, errs = {}, []
    for _ in range(ndev):
        msg = out_q.get()
        if len(msg) == 3 and msg[1] == "__ERR__":
            errs.append((msg[0], msg[2]))
        else:
            results[msg[0]] = msg[1]
    for p in procs:
        p.join()
    if errs:
        raise RuntimeError("multi-GPU screen failed on ranks " + str([r for r, _ in errs]) +
                           ":\n" + "\n".join(f"[rank {r}]\n{tb}" for r, tb in errs))
    heaps = [_TopK(top_k) for _ in qs]
    for rank in sorted(results):
        for qi, items in enumerate(results[rank]):
            for score, _, id_, tf in items:
                heaps[qi].push(score, id_, tf)
    return heaps


def screen_many(queries: Sequence, store: ProfileStore, mode: str = "surf_esp", *,
                backend: Optional[str] = None, do_center: Optional[bool] = None,
                top_k: int = 1000, ndev: Optional[int] = None, scores_out=None,
                alpha: Optional[float] = None, progress: bool = False, device=None,
                **align_kwargs) -> List[List[Hit]]:
    """Screen a panel of queries against ``store``; one streaming pass over its shards.

    ``ndev`` > 1 spreads the shards over that many GPUs (at most the visible ones), one
    spawned process per GPU pulling shards from a shared queue; the per-GPU top-K lists are
    merged on the host.  ``scores_out`` needs the single-process path (ndev 1 or None), as in
    the reference (screen.py:1114-1124)."""
    if backend not in (None, "cuda"):
        raise ValueError(f"backend {backend!r} is provided by shepherd_score; this package "
                         "implements backend='cuda'")
    multi = bool(ndev and ndev > 1)
    if multi and scores_out is not None:
        raise ValueError("scores_out is not supported with ndev>1 (each GPU returns only its "
                         "per-query top-K)")
    mode = canonical(mode)
    if mode not in _SCREEN_MODES:
        raise ValueError(f"unknown mode {mode!r}; valid: {list(_SCREEN_MODES)}")
    if not store.supports(mode):
        raise ValueError(f"store at {store.path!r} was built for modes {store.modes} and does "
                         f"not support {mode!r}")
    if align_kwargs.get("no_H") is False:
        raise ValueError("screen() aligns heavy atoms only; no_H=False is not supported")
    if mode == "vol_esp" and "lam" not in align_kwargs:
        raise ValueError("vol_esp requires an explicit lam=...")
    if alpha is None:
        # vol_and_surf_esp takes alpha explicitly in the reference; 0.81 selects the heavy-atom
        # shape centres
        alpha = ALPHA(store.num_surf_points) if mode in _SURF_ALPHA_MODES else 0.81
    center = (not store.pre_centered) if do_center is None else bool(do_center)
    qs = [_centred_query(q) if (store.pre_centered or center) else q for q in queries]
    kw = _batch_kwargs(mode, align_kwargs, alpha)
    if multi:
        qs = [_plain_query(q) for q in qs]
        heaps = _screen_multi_gpu(qs, store, mode, ndev, kw, dict(align_kwargs), alpha, top_k,
                                  center)
        return [h.sorted() for h in heaps]
    device = torch.device(device or "cuda")
    so = None
    if scores_out is not None:
        so = [scores_out] if isinstance(scores_out, np.ndarray) and len(qs) == 1 else list(scores_out)
    heaps = _screen_shards(qs, store, mode, range(store.num_shards), kw, align_kwargs, alpha,
                           top_k, center, device, so, progress)
    return [h.sorted() for h in heaps]


def _plain_query(q):
    """The query as a dict of numpy arrays (picklable for the spawned GPU workers)."""
    if isinstance(q, dict):
        return {k: (None if v is None else np.asarray(v)) for k, v in q.items()}
    names = ("atom_pos", "surf_pos", "surf_esp", "partial_charges", "pharm_types",
             "pharm_ancs", "pharm_vecs", "radii", "centers_w_H")
    out = {n: getattr(q, n, None) for n in names}
    if out["centers_w_H"] is None and getattr(q, "mol", None) is not None:
        out["centers_w_H"] = q.mol.GetConformer().GetPositions()
    return {k: (None if v is None else np.asarray(v)) for k, v in out.items()}


def screen(query, store: ProfileStore, mode: str = "surf_esp", **kw) -> List[Hit]:
    """Stream ``store`` past one query and return its ``top_k`` hits (screen.py:1141)."""
    return screen_many([query], store, mode, **kw)[0]


def _center_shard(arrs, mode):
    """Centre every molecule of a non-pre-centred shard on its atom COM."""
    arrs = dict(arrs)
    off = arrs["atom_off"]
    pos = arrs["atom_pos"].astype(np.float32)
    n = np.diff(off)
    mol = np.repeat(np.arange(len(n)), n)
    c = np.zeros((len(n), 3), np.float32)
    np.add.at(c, mol, pos)
    c /= np.maximum(n, 1)[:, None]
    arrs["atom_pos"] = pos - c[mol]
    if "surf_pos" in arrs:
        arrs["surf_pos"] = arrs["surf_pos"].astype(np.float32) - c[:, None, :]
    if "pharm_ancs" in arrs:
        pn = np.diff(arrs["pharm_off"])
        arrs["pharm_ancs"] = arrs["pharm_ancs"].astype(np.float32) - c[np.repeat(np.arange(len(pn)), pn)]
    if "cwh" in arrs:
        an = np.diff(arrs["all_off"])
        arrs["cwh"] = arrs["cwh"].astype(np.float32) - c[np.repeat(np.arange(len(an)), an)]
    return arrs


def _id_to_py(x):
    return x.item() if hasattr(x, "item") else x
