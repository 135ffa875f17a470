"""Screening libraries on the device, built from ProfileStore columns in their stored dtype.

A float16 store stays float16 in HBM: its coordinates are copied host -> device as they are
(half the bytes of float32) and packed into 8-byte (x, y, z, w) points, which the alignment,
seed and self-overlap kernels widen to float32 in their staging loads.  Packing writes the
float16 values into place without arithmetic, so a float16 library scores exactly as the
same values widened to float32 would.  A float32 store packs as float32.

* :func:`cloud_from_csr` / :func:`cloud_from_dense` / :func:`pharm_from_csr` -- one shard's
  ragged or fixed-size columns as a packed ``CloudSet`` / ``PharmSet``;
* :class:`Library` -- every shard of a store uploaded once into one device arena (the
  resident library of :class:`fast_shepherd_score_b200.server.ScreenServer`).

Pharmacophore anchors carry their type in w: as int32 bits in float32 sets, as an exact
float16 value (0..8) in float16 sets.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from .layout import DUMMY_TYPE, N_PHARM_TYPES, CloudSet, PharmSet, _offsets

_HALF = torch.float16


def _set_dtype(stored, widen: bool) -> torch.dtype:
    return _HALF if (not widen and np.dtype(stored) == np.float16) else torch.float32


def upload(a, device) -> torch.Tensor:
    """Host array -> device tensor in its own dtype (pinned, asynchronous)."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    if torch.cuda.is_available() and torch.device(device).type == "cuda":
        t = t.pin_memory()
    return t.to(device, non_blocking=True)


def _fill(dst: torch.Tensor, src, device):
    """dst <- src (dst's dtype; a float16 -> float16 copy moves bits, no arithmetic)."""
    dst.copy_(upload(src, device))


def cloud_from_csr(pos, off, device, w=None, widen: bool = False) -> CloudSet:
    """Ragged (sum n_i, 3) points with int offsets (+ optional per-point values) as a packed
    set; float16 columns stay float16 unless ``widen``."""
    off = np.asarray(off, np.int64)
    n = np.diff(off)
    pts = torch.zeros(int(off[-1]), 4, dtype=_set_dtype(np.asarray(pos).dtype, widen),
                      device=device)
    _fill(pts[:, :3], np.asarray(pos).reshape(-1, 3), device)
    if w is not None:
        _fill(pts[:, 3], np.asarray(w).reshape(-1), device)
    return CloudSet(pts, upload(off.astype(np.int32), device), n, int(n.max()) if len(n) else 0)


def cloud_from_dense(pos, device, w=None, widen: bool = False) -> CloudSet:
    """Fixed-size (K, S, 3) points (surfaces) as a packed set of K molecules of S points."""
    K, S, _ = pos.shape
    pts = torch.zeros(K * S, 4, dtype=_set_dtype(pos.dtype, widen), device=device)
    _fill(pts[:, :3], pos.reshape(-1, 3), device)
    if w is not None:
        _fill(pts[:, 3], np.asarray(w).reshape(-1), device)
    counts = np.full(K, S, np.int64)
    return CloudSet(pts, upload(_offsets(counts), device), counts, S)


def _types(types) -> np.ndarray:
    ty = np.asarray(types).astype(np.int64)
    return np.where((ty < 0) | (ty >= N_PHARM_TYPES), DUMMY_TYPE, ty).astype(np.int32)


def pharm_from_csr(types, ancs, vecs, off, device, with_vectors: bool = True,
                   widen: bool = False) -> PharmSet:
    """Ragged pharmacophores (types, anchors, vectors) as a packed set."""
    off = np.asarray(off, np.int64)
    n = np.diff(off)
    total = int(off[-1])
    dt = _set_dtype(np.asarray(ancs).dtype, widen)
    anc = torch.zeros(total, 4, dtype=dt, device=device)
    _fill(anc[:, :3], np.asarray(ancs).reshape(-1, 3), device)
    ty = _types(types)
    if dt == _HALF:
        anc[:, 3] = upload(ty, device).to(_HALF)         # 0..8: exact in float16
    else:
        anc[:, 3] = upload(ty, device).view(torch.float32)
    vec = torch.zeros(total, 4, dtype=dt, device=device)
    if with_vectors and vecs is not None:
        _fill(vec[:, :3], np.asarray(vecs).reshape(-1, 3), device)
    return PharmSet(anc, vec, upload(off.astype(np.int32), device), n,
                    int(n.max()) if len(n) else 0)


@dataclass
class Library:
    """A whole store resident on one device: heavy-atom clouds and (if stored)
    pharmacophores in one arena each, plus the molecules' store ids."""
    atoms: CloudSet
    pharm: Optional[PharmSet]
    ids: np.ndarray
    dtype: torch.dtype

    @property
    def n_mol(self) -> int:
        return self.atoms.n_mol

    @property
    def nbytes(self) -> int:
        n = self.atoms.pts.nbytes + self.atoms.off.nbytes
        if self.pharm is not None:
            n += self.pharm.anc.nbytes + self.pharm.vec.nbytes + self.pharm.off.nbytes
        return n

    @classmethod
    def from_store(cls, store, device=None, *, pharm: Optional[bool] = None,
                   vectors: bool = True, widen: bool = False) -> "Library":
        """Upload every shard of ``store`` (a ProfileStore, shepherd_score's or this
        package's, or a path) once.  ``pharm`` (default: when the store keeps them) adds
        the pharmacophores, ``vectors=False`` leaves their vectors zero (colour mode).
        float16 stores stay float16 on the device unless ``widen``."""
        from .store import ProfileStore
        if isinstance(store, str):
            store = ProfileStore.open(store)
        device = torch.device(device or "cuda")
        if pharm is None:
            pharm = bool(store.schema.get("pharm")) if hasattr(store, "schema") else \
                bool(store.manifest["schema"].get("pharm"))
        # pass 1: offset tables only, for the arena sizes
        atom_n, ph_n = [], []
        for i in range(store.num_shards):
            _, cols = store.read_shard(i, ["atom_off", "pharm_off"]) if _selective(store) \
                else store.read_shard(i)
            atom_n.append(np.diff(np.asarray(cols["atom_off"], np.int64)))
            if pharm:
                ph_n.append(np.diff(np.asarray(cols["pharm_off"], np.int64)))
        counts = np.concatenate(atom_n) if atom_n else np.zeros(0, np.int64)
        stored = np.float16 if store.manifest["dtype"] == "float16" else np.float32
        dt = _set_dtype(stored, widen)
        pts = torch.zeros(int(counts.sum()), 4, dtype=dt, device=device)
        ph_counts = np.concatenate(ph_n) if ph_n else np.zeros(0, np.int64)
        anc = torch.zeros(int(ph_counts.sum()), 4, dtype=dt, device=device) if pharm else None
        vec = torch.zeros_like(anc) if pharm else None
        ids = []
        a0 = p0 = 0
        # pass 2: fill the arena shard by shard (one shard's host arrays at a time)
        for i in range(store.num_shards):
            _, cols = store.read_shard(i)
            ids.append(np.asarray(cols["ids"]))
            pos = np.asarray(cols["atom_pos"]).reshape(-1, 3)
            _fill(pts[a0:a0 + len(pos), :3], pos, device)
            a0 += len(pos)
            if pharm:
                ancs = np.asarray(cols["pharm_ancs"]).reshape(-1, 3)
                k = len(ancs)
                _fill(anc[p0:p0 + k, :3], ancs, device)
                ty = upload(_types(cols["pharm_types"]), device)
                anc[p0:p0 + k, 3] = ty.to(_HALF) if dt == _HALF else ty.view(torch.float32)
                if vectors:
                    _fill(vec[p0:p0 + k, :3], np.asarray(cols["pharm_vecs"]).reshape(-1, 3),
                          device)
                p0 += k
        atoms = CloudSet(pts, upload(_offsets(counts), device), counts,
                         int(counts.max()) if len(counts) else 0)
        ph = (PharmSet(anc, vec, upload(_offsets(ph_counts), device), ph_counts,
                       int(ph_counts.max()) if len(ph_counts) else 0) if pharm else None)
        return cls(atoms, ph, np.concatenate(ids) if ids else np.zeros(0, np.int64), dt)


def _selective(store) -> bool:
    """True for stores whose read_shard takes a column list (this package's)."""
    import inspect
    try:
        return "columns" in inspect.signature(store.read_shard).parameters
    except (TypeError, ValueError):
        return False
