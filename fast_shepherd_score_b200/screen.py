"""Screening front-end: ``screen()`` / ``screen_many()`` over a sharded profile store.

Mirrors shepherd_score/screen.py for the CUDA path: ``ProfileStore`` (:317-606) reads and
writes the reference's on-disk format (``manifest.json`` with ``version`` 1 and a shard list,
``shard_NNNNN.npz`` holding concatenated arrays with CSR offsets, float16 or float32),
``screen_many`` (:1038) streams every shard once for a whole query panel, ``screen`` (:1141)
is the one-query wrapper, ``Hit`` (:75) is ``(score, id, transform)``.

Each shard is uploaded once (float16 coordinates expand to float32 on the device) and kept
as packed device clouds; every query is one reference molecule staged once per work item,
aligned against all of the shard's molecules by one fused kernel launch.  Top-K survivors
are selected on the device, so only K transforms are built per shard and query.
"""
from __future__ import annotations

import heapq
import json
import os
import re
from collections import namedtuple
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import api
from .layout import CloudSet, PharmSet, _offsets
from .modes import CANONICAL_MODES, canonical, seeds_for, steps_for

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


def _schema_from_modes(modes) -> dict:
    """Which arrays a store keeps for its modes (screen.py:203-216)."""
    modes = {canonical(m) for m in modes}
    unknown = modes - set(CANONICAL_MODES)
    if unknown:
        raise ValueError(f"unknown modes {sorted(unknown)}; valid: {list(CANONICAL_MODES)}")
    return dict(surf=bool({"surf", "surf_esp", "vol_and_surf_esp"} & modes),
                surf_esp=bool({"surf_esp", "vol_and_surf_esp"} & modes),
                charges=bool({"vol_esp", "vol_and_surf_esp"} & modes),
                with_H="vol_and_surf_esp" in modes, radii="vol_and_surf_esp" in modes,
                centers_w_H="vol_and_surf_esp" in modes,
                pharm=bool({"pharm", "vol_color", "vol_pharm"} & modes))


def _supports(schema, mode) -> bool:
    """screen.py:219-236 (plus vol_pharm, which needs the pharmacophore arrays)."""
    mode = canonical(mode)
    if mode == "vol":
        return True
    if mode == "vol_esp":
        return schema["charges"]
    if mode == "surf":
        return schema["surf"]
    if mode == "surf_esp":
        return schema["surf"] and schema["surf_esp"]
    if mode in ("pharm", "vol_color", "vol_pharm"):
        return schema["pharm"]
    if mode == "vol_and_surf_esp":
        return (schema["surf"] and schema["surf_esp"] and schema["centers_w_H"]
                and schema["radii"] and schema["charges"] and schema["with_H"])
    return False


class ProfileStore:
    """Sharded on-disk molecule profiles (the reference's format, VERSION 1)."""
    MANIFEST = "manifest.json"
    VERSION = 1

    def __init__(self, path, manifest, rw):
        self.path, self.manifest, self._rw = path, manifest, rw
        self._buf: list = []
        self._n = int(manifest.get("n_total", 0))
        self._shard_id = len(manifest.get("shards", []))

    # ---- writer -----------------------------------------------------------------------
    @classmethod
    def create(cls, path, *, num_surf_points: int, modes: Sequence[str], dtype: str = "float16",
               shard_size: int = 100_000, pre_centered: bool = True,
               overwrite: bool = False) -> "ProfileStore":
        if dtype not in ("float16", "float32"):
            raise ValueError("dtype must be 'float16' or 'float32'")
        schema = _schema_from_modes(modes)
        os.makedirs(path, exist_ok=True)
        mpath = os.path.join(path, cls.MANIFEST)
        if os.path.exists(mpath) and not overwrite:
            raise FileExistsError(f"{mpath} already exists; pass overwrite=True to replace it")
        if overwrite:
            for f in os.listdir(path):
                if f == cls.MANIFEST or re.fullmatch(r"shard_\d{5}\.npz", f):
                    os.remove(os.path.join(path, f))
        manifest = dict(version=cls.VERSION, num_surf_points=int(num_surf_points),
                        modes=list(modes), schema=schema, dtype=dtype,
                        shard_size=int(shard_size), pre_centered=bool(pre_centered), n_total=0,
                        shards=[])
        st = cls(path, manifest, "w")
        st._write_manifest()
        return st

    def add_arrays(self, *, atom_pos, surf_pos=None, surf_esp=None, partial_charges=None,
                   pharm_types=None, pharm_ancs=None, pharm_vecs=None, centers_w_H=None,
                   radii=None, nonH_atoms_idx=None, id=None) -> None:
        """Buffer one molecule given as arrays (centred on its atom COM when the store is
        pre-centred, as the reference's writer does).  Stores with hydrogens
        (vol_and_surf_esp) take ``partial_charges``, ``radii`` and ``centers_w_H`` for all
        atoms and ``nonH_atoms_idx`` (default: the first len(atom_pos) atoms are the heavy
        ones)."""
        if self._rw != "w":
            raise RuntimeError("store is open for reading")
        rec = dict(atom_pos=np.asarray(atom_pos, np.float32), surf_pos=surf_pos,
                   surf_esp=surf_esp, partial_charges=partial_charges, pharm_types=pharm_types,
                   pharm_ancs=pharm_ancs, pharm_vecs=pharm_vecs, centers_w_H=centers_w_H,
                   radii=radii, nonH=nonH_atoms_idx,
                   id=self._n + len(self._buf) if id is None else id)
        if self.manifest["schema"]["with_H"]:
            if centers_w_H is None or radii is None or partial_charges is None:
                raise ValueError("a store with hydrogens needs centers_w_H, radii and "
                                 "partial_charges for every atom")
            if rec["nonH"] is None:
                rec["nonH"] = np.arange(len(rec["atom_pos"]), dtype=np.int64)
        if self.manifest["pre_centered"]:
            c = rec["atom_pos"].mean(0)
            rec["atom_pos"] = rec["atom_pos"] - c
            if surf_pos is not None:
                rec["surf_pos"] = np.asarray(surf_pos, np.float32) - c
            if pharm_ancs is not None:
                rec["pharm_ancs"] = np.asarray(pharm_ancs, np.float32) - c
            if centers_w_H is not None:
                rec["centers_w_H"] = np.asarray(centers_w_H, np.float32) - c
        self._buf.append(rec)
        if len(self._buf) >= self.manifest["shard_size"]:
            self._flush()

    def close(self):
        if self._rw == "w":
            self._flush()
            self._write_manifest()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _write_manifest(self):
        with open(os.path.join(self.path, self.MANIFEST), "w") as fh:
            json.dump(self.manifest, fh, indent=2)

    def _flush(self):
        if not self._buf:
            return
        sch = self.manifest["schema"]
        dt = np.float16 if self.manifest["dtype"] == "float16" else np.float32
        recs = self._buf
        off = lambda L: np.concatenate([[0], np.cumsum(L)]).astype(np.int64)
        out = {"ids": np.array([r["id"] for r in recs])}
        out["atom_off"] = off([len(r["atom_pos"]) for r in recs])
        out["atom_pos"] = np.concatenate([r["atom_pos"] for r in recs]).astype(dt)
        if sch["surf"]:
            out["surf_pos"] = np.stack([r["surf_pos"] for r in recs]).astype(dt)
        if sch["surf_esp"]:
            out["surf_esp"] = np.stack([r["surf_esp"] for r in recs]).astype(dt)
        if sch["charges"] and sch["with_H"]:
            # layout of the reference's writer (screen.py:470-481): all-atom arrays with their
            # own offsets, heavy-atom indices into them
            out["all_off"] = off([len(r["partial_charges"]) for r in recs])
            out["charges"] = np.concatenate([r["partial_charges"] for r in recs]).astype(dt)
            out["nonH"] = np.concatenate([r["nonH"] for r in recs]).astype(np.int64)
            if sch["radii"]:
                out["radii"] = np.concatenate([r["radii"] for r in recs]).astype(dt)
            if sch["centers_w_H"]:
                out["cwh"] = np.concatenate([r["centers_w_H"] for r in recs]).astype(dt)
        elif sch["charges"]:
            out["charges"] = np.concatenate([r["partial_charges"] for r in recs]).astype(dt)
        if sch["pharm"]:
            out["pharm_off"] = off([len(r["pharm_types"]) for r in recs])
            out["pharm_types"] = np.concatenate([r["pharm_types"] for r in recs]).astype(np.int32)
            out["pharm_ancs"] = np.concatenate([r["pharm_ancs"] for r in recs]).astype(dt)
            out["pharm_vecs"] = np.concatenate([r["pharm_vecs"] for r in recs]).astype(dt)
        name = f"shard_{self._shard_id:05d}.npz"
        np.savez(os.path.join(self.path, name), **out)
        self.manifest["shards"].append(dict(name=name, n=len(recs), start=self._n))
        self._n += len(recs)
        self.manifest["n_total"] = self._n
        self._buf = []
        self._shard_id += 1
        self._write_manifest()

    # ---- reader -----------------------------------------------------------------------
    @classmethod
    def open(cls, path) -> "ProfileStore":
        with open(os.path.join(path, cls.MANIFEST)) as fh:
            manifest = json.load(fh)
        if manifest.get("version") != cls.VERSION:
            raise ValueError(f"ProfileStore at {path!r} has on-disk format version "
                             f"{manifest.get('version')!r}; this reader reads {cls.VERSION}")
        return cls(path, manifest, "r")

    def __len__(self):
        return int(self.manifest["n_total"])

    @property
    def num_surf_points(self) -> int:
        return int(self.manifest["num_surf_points"])

    @property
    def modes(self) -> tuple:
        return tuple(self.manifest["modes"])

    @property
    def pre_centered(self) -> bool:
        return bool(self.manifest["pre_centered"])

    @property
    def num_shards(self) -> int:
        return len(self.manifest["shards"])

    def supports(self, mode) -> bool:
        return _supports(self.manifest["schema"], mode)

    def read_shard(self, idx: int):
        sh = self.manifest["shards"][idx]
        with np.load(os.path.join(self.path, sh["name"])) as data:
            return sh, {k: data[k] for k in data.files}


# -----------------------------------------------------------------------------------------
# Device-side shard expansion
# -----------------------------------------------------------------------------------------
def _dev(a, device, dtype=torch.float32):
    """Upload an array in its stored dtype (float16 halves the copy), widen on the device."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    if torch.cuda.is_available():
        t = t.pin_memory()
    return t.to(device, non_blocking=True).to(dtype)


def _cloud_from_csr(pos, off, device, w=None) -> CloudSet:
    off = np.asarray(off, np.int64)
    n = np.diff(off)
    pts = torch.zeros(int(off[-1]), 4, device=device)
    pts[:, :3] = _dev(pos, device)
    if w is not None:
        pts[:, 3] = _dev(w, device)
    return CloudSet(pts, torch.from_numpy(off.astype(np.int32)).to(device), n,
                    int(n.max()) if len(n) else 0)


def _cloud_from_dense(pos, device, w=None) -> CloudSet:
    K, S, _ = pos.shape
    pts = torch.zeros(K * S, 4, device=device)
    pts[:, :3] = _dev(pos.reshape(-1, 3), device)
    if w is not None:
        pts[:, 3] = _dev(w.reshape(-1), device)
    counts = np.full(K, S, np.int64)
    return CloudSet(pts, torch.from_numpy(_offsets(counts)).to(device), counts, S)


def _pharm_from_csr(types, ancs, vecs, off, device, with_vectors=True) -> PharmSet:
    off = np.asarray(off, np.int64)
    n = np.diff(off)
    total = int(off[-1])
    anc = torch.zeros(total, 4, device=device)
    anc[:, :3] = _dev(ancs, device)
    ty = np.asarray(types).astype(np.int64)
    ty = np.where((ty < 0) | (ty > 8), 8, ty).astype(np.int32)
    anc[:, 3] = torch.from_numpy(ty).to(device).view(torch.float32)
    vec = torch.zeros(total, 4, device=device)
    if with_vectors and vecs is not None:
        vec[:, :3] = _dev(vecs, device)
    return PharmSet(anc, vec, torch.from_numpy(off.astype(np.int32)).to(device), n,
                    int(n.max()) if len(n) else 0)


def shard_to_device(arrs: dict, mode: str, device, alpha: float = 0.81):
    """(fit CloudSet or None, fit PharmSet or None, extra kwargs) of one shard for `mode`;
    vol_and_surf_esp adds the atoms with hydrogens, their radii and the surfaces."""
    if mode == "vol_and_surf_esp":
        # shape centres: heavy atoms at alpha 0.81, else the surface (aligners.py:795-803)
        surf = _cloud_from_dense(arrs["surf_pos"], device, arrs["surf_esp"])
        cs = (_cloud_from_csr(arrs["atom_pos"], arrs["atom_off"], device) if alpha == 0.81
              else _cloud_from_dense(arrs["surf_pos"], device))
        atoms = _cloud_from_csr(arrs["cwh"], arrs["all_off"], device, arrs["charges"])
        return cs, None, dict(fit_atoms=atoms, fit_radii=_dev(arrs["radii"], device),
                              fit_surf=surf)
    if mode in ("vol", "vol_color", "vol_pharm"):
        cs = _cloud_from_csr(arrs["atom_pos"], arrs["atom_off"], device)
    elif mode == "vol_esp":
        cs = _cloud_from_csr(arrs["atom_pos"], arrs["atom_off"], device, arrs["charges"])
    elif mode == "surf":
        cs = _cloud_from_dense(arrs["surf_pos"], device)
    elif mode == "surf_esp":
        cs = _cloud_from_dense(arrs["surf_pos"], device, arrs["surf_esp"])
    else:
        cs = None
    ps = None
    if mode in ("pharm", "vol_color", "vol_pharm"):
        ps = _pharm_from_csr(arrs["pharm_types"], arrs["pharm_ancs"], arrs["pharm_vecs"],
                             arrs["pharm_off"], device, with_vectors=(mode != "vol_color"))
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
        fit, fit_ph, fit_x = shard_to_device(arrs, mode, device, alpha)
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
