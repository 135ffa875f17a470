"""Packed device layouts of ragged molecule clouds.

A *cloud set* stores many molecules' points back to back as float4 (x, y, z, w) with an
int32 prefix-offset table, so a fused kernel reads molecule ``m`` as
``pts[off[m]:off[m+1]]`` with 16-byte coalesced loads and no padding.  ``w`` carries the
per-point charge (ESP) or 0.  A *pharmacophore set* stores anchors as float4 with the
int32 type in ``w``'s bit pattern, and direction vectors as float4 (x, y, z, 0).

These replace the reference's padded (K, N_pad, 3) batches (accel/batch/_pad.py
``_scatter_fill``) and its per-start expansion of the clouds (accel/drivers/shape.py:218-219):
each molecule is stored once, however many pairs or starts use it.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

N_PHARM_TYPES = 9
DUMMY_TYPE = 8


def _offsets(counts) -> np.ndarray:
    off = np.zeros(len(counts) + 1, np.int64)
    np.cumsum(np.asarray(counts, np.int64), out=off[1:])
    if off[-1] >= 2 ** 31:
        raise ValueError("cloud set exceeds 2^31 points; split it")
    return off.astype(np.int32)


@dataclass
class CloudSet:
    """Molecules' points packed as float4 on one device."""
    pts: torch.Tensor          # (total, 4) float32
    off: torch.Tensor          # (n_mol + 1,) int32
    counts: np.ndarray         # host copy of the per-molecule counts
    max_points: int

    @property
    def n_mol(self) -> int:
        return len(self.counts)

    @property
    def device(self):
        return self.pts.device

    @staticmethod
    def from_arrays(points: Sequence, charges: Optional[Sequence] = None, device="cuda",
                    non_blocking: bool = False) -> "CloudSet":
        """Pack a list of (n_i, 3) arrays/tensors (and optional (n_i,) charges)."""
        counts = np.array([len(p) for p in points], np.int64)
        total = int(counts.sum())
        host = np.zeros((total, 4), np.float32)
        if total:
            host[:, :3] = np.concatenate([np.asarray(_np(p), np.float32).reshape(-1, 3)
                                          for p in points])
            if charges is not None:
                host[:, 3] = np.concatenate([np.asarray(_np(c), np.float32).reshape(-1)
                                             for c in charges])
        return CloudSet.from_host(host, counts, device, non_blocking)

    @staticmethod
    def from_host(host: np.ndarray, counts, device="cuda", non_blocking=False) -> "CloudSet":
        counts = np.asarray(counts, np.int64)
        off = _offsets(counts)
        pin = non_blocking and torch.cuda.is_available()
        pts = torch.from_numpy(np.ascontiguousarray(host, np.float32))
        offt = torch.from_numpy(off)
        if pin:
            pts, offt = pts.pin_memory(), offt.pin_memory()
        return CloudSet(pts.to(device, non_blocking=non_blocking),
                        offt.to(device, non_blocking=non_blocking), counts,
                        int(counts.max()) if len(counts) else 0)

    @staticmethod
    def from_padded(X: torch.Tensor, n_real, C: Optional[torch.Tensor] = None) -> "CloudSet":
        """Pack a padded (K, N_pad, 3) batch with real counts, on X's device."""
        K, npad, _ = X.shape
        n = torch.as_tensor(n_real, device=X.device).to(torch.int64).clamp(0, npad)
        mask = torch.arange(npad, device=X.device)[None, :] < n[:, None]
        w = (C.to(X.dtype) if C is not None else torch.zeros(K, npad, device=X.device,
                                                               dtype=X.dtype))
        pts = torch.cat([X, w.unsqueeze(-1)], dim=-1)[mask].to(torch.float32).contiguous()
        counts = n.cpu().numpy()
        off = torch.from_numpy(_offsets(counts)).to(X.device)
        return CloudSet(pts, off, counts, int(counts.max()) if K else 0)


@dataclass
class PharmSet:
    """Pharmacophores packed as float4 anchors (type in w's bits) + float4 vectors."""
    anc: torch.Tensor          # (total, 4) float32, w = int32 type bits
    vec: torch.Tensor          # (total, 4) float32
    off: torch.Tensor          # (n_mol + 1,) int32
    counts: np.ndarray
    max_points: int

    @property
    def n_mol(self) -> int:
        return len(self.counts)

    @staticmethod
    def from_arrays(types: Sequence, anchors: Sequence, vectors: Optional[Sequence] = None,
                    device="cuda", non_blocking: bool = False) -> "PharmSet":
        counts = np.array([len(a) for a in anchors], np.int64)
        total = int(counts.sum())
        anc = np.zeros((total, 4), np.float32)
        vec = np.zeros((total, 4), np.float32)
        if total:
            anc[:, :3] = np.concatenate([np.asarray(_np(a), np.float32).reshape(-1, 3)
                                         for a in anchors])
            ty = np.concatenate([np.asarray(_np(t)).reshape(-1) for t in types]).astype(np.int64)
            if ty.size != total:
                raise ValueError("pharmacophore types and anchors differ in length")
            ty = np.where((ty < 0) | (ty >= N_PHARM_TYPES), DUMMY_TYPE, ty).astype(np.int32)
            anc[:, 3] = ty.view(np.float32)
            if vectors is not None:
                vec[:, :3] = np.concatenate([np.asarray(_np(v), np.float32).reshape(-1, 3)
                                             for v in vectors])
        off = _offsets(counts)
        mk = lambda a: torch.from_numpy(a).to(device, non_blocking=non_blocking)
        return PharmSet(mk(anc), mk(vec), mk(off), counts, int(counts.max()) if len(counts) else 0)

    @staticmethod
    def from_padded(A: torch.Tensor, T: torch.Tensor, V: Optional[torch.Tensor], n_real
                    ) -> "PharmSet":
        K, npad, _ = A.shape
        n = torch.as_tensor(n_real, device=A.device).to(torch.int64).clamp(0, npad)
        mask = torch.arange(npad, device=A.device)[None, :] < n[:, None]
        ty = T.to(torch.int64)
        ty = torch.where((ty < 0) | (ty >= N_PHARM_TYPES), torch.full_like(ty, DUMMY_TYPE), ty)
        tyf = ty.to(torch.int32).view(torch.float32)
        anc = torch.cat([A.to(torch.float32), tyf.unsqueeze(-1)], -1)[mask].contiguous()
        if V is None:
            vec = torch.zeros_like(anc)
        else:
            vec = torch.cat([V.to(torch.float32), torch.zeros(K, npad, 1, device=A.device)],
                            -1)[mask].contiguous()
        counts = n.cpu().numpy()
        off = torch.from_numpy(_offsets(counts)).to(A.device)
        return PharmSet(anc, vec, off, counts, int(counts.max()) if K else 0)


def _np(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return x


def cost_order_device(ref_off: torch.Tensor, fit_off: torch.Tensor, pair_ref: torch.Tensor,
                      pair_fit: torch.Tensor) -> torch.Tensor:
    """cost_order computed where the pairs live (no device-to-host copy, no stream sync): the
    per-molecule counts come from the packed sets' offsets."""
    n_ref = (ref_off[1:] - ref_off[:-1]).to(torch.int64)
    n_fit = (fit_off[1:] - fit_off[:-1]).to(torch.int64)
    cost = n_ref[pair_ref.long()] * n_fit[pair_fit.long()]
    return torch.argsort(-cost, stable=True).to(torch.int32)
