"""Continuous-batching screening server over a device-resident library.

A request is one query molecule scored against a set of library molecules (1k-100k) and
answered with its top-K hits.  The library (packed clouds + pharmacophores + per-molecule
self overlaps) is uploaded once and stays in HBM.  A scheduler thread keeps the GPU fed:

* **admission** -- pending requests are cut into slices (consecutive library ranges) and
  admitted FIFO while the launch's pair budget and the in-flight HBM budget (seeds, rows and
  results of every launch not yet retired) allow; a request that does not fit waits for
  earlier launches to retire;
* **continuous batching** -- one fused-kernel launch carries slices of many requests (each
  request's query is one molecule of the launch's query set); requests that arrive while
  launches run join the next launch, and up to ``max_in_flight`` launches are queued on the
  stream so the device never idles between them;
* **retirement** -- when a launch's completion event fires, its per-pair results (already
  copied to pinned host memory) are merged into each request's running top-K; the last
  slice resolves the request's future and records its latency.

Every pair is computed independently with a fixed tiling, so a request's result is the same
alone and in any mix (tests/test_gpu_server.py).  Reference counterpart: the streaming loop
of shepherd_score/screen.py:962-1035, which re-buckets per query and has no admission,
overlap or latency accounting.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import math
import threading
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from . import align as al
from . import api
from . import kernels as K
from .layout import CloudSet, PharmSet, _offsets


# ----------------------------------------------------------------------------------------
# Host-side planning (no device state; unit-tested on CPU)
# ----------------------------------------------------------------------------------------
@dataclass(eq=False)   # identity semantics: requests are hashed and removed by identity
class Request:
    rid: int
    query: dict
    lib_idx: np.ndarray            # int32 library molecule indices to score
    top_k: int
    arrival: float
    future: Optional[cf.Future] = None
    next: int = 0                  # first library position not yet scheduled
    remaining: int = 0             # pairs not yet retired
    best_s: np.ndarray = None
    best_i: np.ndarray = None
    best_q: np.ndarray = None
    best_t: np.ndarray = None
    finished: Optional[float] = None

    def __post_init__(self):
        self.remaining = len(self.lib_idx)


@dataclass
class Slice:
    req: Request
    start: int
    stop: int

    @property
    def n(self) -> int:
        return self.stop - self.start


class Planner:
    """Cuts pending requests into slices for the next launch under two budgets."""

    def __init__(self, max_pairs_per_launch: int, hbm_budget_bytes: int, bytes_per_pair: int,
                 slice_pairs: int = 8192):
        self.max_pairs = int(max_pairs_per_launch)
        self.budget = int(hbm_budget_bytes)
        self.bpp = int(bytes_per_pair)
        self.slice_pairs = int(slice_pairs)
        self.in_flight_bytes = 0

    def plan(self, pending: "collections.deque[Request]") -> List[Slice]:
        out, pairs = [], 0
        for req in pending:                      # FIFO; earlier requests first
            while req.next < len(req.lib_idx) and pairs < self.max_pairs:
                n = min(self.slice_pairs, len(req.lib_idx) - req.next, self.max_pairs - pairs)
                need = n * self.bpp
                if self.in_flight_bytes + pairs * self.bpp + need > self.budget:
                    return out                   # HBM budget exhausted: wait for retirement
                out.append(Slice(req, req.next, req.next + n))
                req.next += n
                pairs += n
            if pairs >= self.max_pairs:
                break
        return out

    def admit(self, slices: List[Slice]) -> int:
        b = sum(s.n for s in slices) * self.bpp
        self.in_flight_bytes += b
        return b

    def retire(self, nbytes: int):
        self.in_flight_bytes -= nbytes


def merge_topk(req: Request, scores, idx, q, t):
    """Fold one slice's results into the request's running top-K (host, numpy)."""
    if req.best_s is None:
        s, i, qq, tt = scores, idx, q, t
    else:
        s = np.concatenate([req.best_s, scores])
        i = np.concatenate([req.best_i, idx])
        qq = np.concatenate([req.best_q, q])
        tt = np.concatenate([req.best_t, t])
    k = min(req.top_k, len(s))
    sel = np.argpartition(-s, k - 1)[:k] if len(s) > k else np.arange(len(s))
    req.best_s, req.best_i, req.best_q, req.best_t = s[sel], i[sel], qq[sel], tt[sel]


def finalize(req: Request, ids=None):
    order = np.lexsort((req.best_i, -req.best_s))   # score desc, library index asc
    T = api.se3_from_qt(req.best_q[order], req.best_t[order])
    from .screen import Hit
    lib = req.best_i[order]
    return [Hit(score=float(s), id=int(ids[j]) if ids is not None else int(j), transform=tf)
            for s, j, tf in zip(req.best_s[order], lib, T)]


def percentile(xs, p):
    if not xs:
        return float("nan")
    return float(np.percentile(np.asarray(xs), p))


# ----------------------------------------------------------------------------------------
# Device side
# ----------------------------------------------------------------------------------------
@dataclass
class _Launch:
    slices: List[Slice]
    host: torch.Tensor            # pinned (P, 8): score, q, t
    event: torch.cuda.Event
    nbytes: int
    keep: list = field(default_factory=list)   # device tensors alive until retirement


class ScreenServer:
    """Serve screening requests against a device-resident library.

    ``library`` = (CloudSet atoms, PharmSet pharmacophores) on ``device`` (e.g. from
    :func:`fast_shepherd_score_b200.synthetic.library_on_device` or loaded from a
    ``ProfileStore``).  ``mode`` is "vol_pharm" (shape + directional pharmacophores, the
    default), "vol_color" or "vol".
    """

    def __init__(self, library, *, mode: str = "vol_pharm", starts: int = 20, steps: int = 100,
                 lr: float = 0.1, alpha: float = 0.81, color_weight: float = 0.5,
                 max_pairs_per_launch: int = 65536, hbm_budget_bytes: Optional[int] = None,
                 lanes_per_pose: int = 8, max_in_flight: int = 2, slice_pairs: int = 8192,
                 ids=None, device=None, tile: Optional[dict] = None):
        self.atoms, self.pharm = library
        self.dev = torch.device(device or self.atoms.pts.device)
        self.mode = mode
        self.S, self.steps, self.lr = int(starts), int(steps), float(lr)
        self.alpha, self.w = float(alpha), float(color_weight)
        self.lpp = int(lanes_per_pose)
        # the remaining tile fields (chunks, cta_per_sm, kernel_variant), fixed for the server's
        # life so a request's result does not depend on its launch-mates
        self.tile = {k: int(v) for k, v in (tile or {}).items()
                     if k in ("chunks", "cta_per_sm", "kernel_variant")}
        self.ids = ids
        self.max_in_flight = int(max_in_flight)
        directional = mode == "vol_pharm"
        with torch.cuda.device(self.dev):
            self.lib_self = K.self_overlap(self.atoms, self.alpha)
            self.lib_self_ph = (K.pharm_self_overlap(self.pharm, directional)
                                if mode != "vol" else None)
        # bytes per in-flight pair: seeds (7 floats/start), rows (8 floats/start), results,
        # pair indices
        bpp = self.S * (7 + 8) * 4 + 8 * 4 + 8
        if hbm_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.dev)
            hbm_budget_bytes = int(0.25 * free)
        self.planner = Planner(max_pairs_per_launch, hbm_budget_bytes, bpp, slice_pairs)
        self.pending: "collections.deque[Request]" = collections.deque()
        self.in_flight: "collections.deque[_Launch]" = collections.deque()
        self.latencies: List[float] = []
        self.completed = 0
        self.pairs_done = 0
        self.max_queue = 0
        self._rid = 0
        self._cv = threading.Condition()
        self._stop = False
        self._err: Optional[BaseException] = None
        self.stream = torch.cuda.Stream(self.dev)
        self._thread = threading.Thread(target=self._run, name="fss-screen-server", daemon=True)
        self._thread.start()

    # ---- client side -------------------------------------------------------------------
    def submit(self, query: dict, lib_idx=None, top_k: int = 100) -> cf.Future:
        """Queue one query against ``lib_idx`` (default: the whole library)."""
        if lib_idx is None:
            lib_idx = np.arange(self.atoms.n_mol, dtype=np.int32)
        lib_idx = np.asarray(lib_idx, dtype=np.int32)
        if len(lib_idx) == 0:
            raise ValueError("empty request")
        if lib_idx.min() < 0 or lib_idx.max() >= self.atoms.n_mol:
            raise ValueError("library index out of range")
        fut: cf.Future = cf.Future()
        with self._cv:
            if self._err is not None:
                raise RuntimeError("screen server stopped after an error") from self._err
            req = Request(self._rid, query, lib_idx, int(top_k), time.perf_counter(), fut)
            self._rid += 1
            self.pending.append(req)
            self.max_queue = max(self.max_queue, len(self.pending))
            self._cv.notify()
        return fut

    def stats(self) -> dict:
        with self._cv:
            lat = list(self.latencies)
            return {"completed": self.completed, "pairs_done": self.pairs_done,
                    "p50_ms": percentile(lat, 50) * 1e3, "p99_ms": percentile(lat, 99) * 1e3,
                    "queue_depth": len(self.pending), "max_queue_depth": self.max_queue,
                    "in_flight_bytes": self.planner.in_flight_bytes}

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify()
        self._thread.join()
        if self._err is not None:
            raise RuntimeError("screen server failed") from self._err

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- scheduler thread --------------------------------------------------------------
    def _run(self):
        try:
            torch.cuda.set_device(self.dev)
            with torch.cuda.stream(self.stream):
                while True:
                    with self._cv:
                        while (not self._stop and not self.in_flight
                               and not any(r.next < len(r.lib_idx) for r in self.pending)):
                            self._cv.wait(0.05)
                        if self._stop and not self.in_flight and not self.pending:
                            return
                        slices = []
                        if len(self.in_flight) < self.max_in_flight:
                            slices = self.planner.plan(self.pending)
                            if slices:
                                nbytes = self.planner.admit(slices)
                    if slices:
                        self.in_flight.append(self._launch(slices, nbytes))
                        continue                 # keep the queue of launches full
                    if self.in_flight:
                        self.in_flight[0].event.synchronize()
                        self._retire(self.in_flight.popleft())
        except BaseException as exc:             # surface errors to every waiter
            with self._cv:
                self._err = exc
                for r in self.pending:
                    if r.future is not None and not r.future.done():
                        r.future.set_exception(exc)

    def _launch(self, slices: List[Slice], nbytes: int) -> _Launch:
        dev = self.dev
        reqs = list(dict.fromkeys(s.req for s in slices))   # unique, in order
        qpos = {r.rid: k for k, r in enumerate(reqs)}
        qa = [r.query["atom_pos"] for r in reqs]
        qset = CloudSet.from_arrays(qa, device=dev, non_blocking=True)
        qph = None
        if self.mode != "vol":
            qph = PharmSet.from_arrays([r.query["pharm_types"] for r in reqs],
                                       [r.query["pharm_ancs"] for r in reqs],
                                       [r.query.get("pharm_vecs") for r in reqs]
                                       if self.mode == "vol_pharm" else None,
                                       device=dev, non_blocking=True)
        pr = np.concatenate([np.full(s.n, qpos[s.req.rid], np.int32) for s in slices])
        pf = np.concatenate([s.req.lib_idx[s.start:s.stop] for s in slices])
        P = len(pr)
        cost = qset.counts[pr].astype(np.int64) * self.atoms.counts[pf].astype(np.int64)
        order = np.argsort(-cost, kind="stable").astype(np.int32)
        pin = lambda a: torch.from_numpy(a).pin_memory().to(dev, non_blocking=True)
        pr_d, pf_d, ord_d = pin(pr), pin(pf), pin(order)
        q_self = K.self_overlap(qset, self.alpha)
        q_self_ph = (K.pharm_self_overlap(qph, self.mode == "vol_pharm")
                     if self.mode != "vol" else None)
        sq, st = K.seeds(qset, self.atoms, pr_d, pf_d, self.S)
        amode = {"vol": "shape", "vol_color": "shape_color", "vol_pharm": "shape_pharm"}[self.mode]
        res = al.align_packed(amode, ref=qset, fit=self.atoms,
                              ref_ph=qph, fit_ph=self.pharm if self.mode != "vol" else None,
                              pair_ref=pr_d, pair_fit=pf_d, seed_q=sq, seed_t=st,
                              steps=self.steps, lr=self.lr, alpha=self.alpha,
                              color_weight=self.w, ref_self=q_self, fit_self=self.lib_self,
                              ref_self_ph=q_self_ph, fit_self_ph=self.lib_self_ph, order=ord_d,
                              lanes_per_pose=self.lpp, check_status=False, validate=False,
                              **self.tile)
        sc, q, t = res
        host = torch.empty(P, 8, dtype=torch.float32, pin_memory=True)
        host.copy_(torch.cat([sc[:, None], q, t], 1), non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        return _Launch(slices, host, ev, nbytes, keep=[res, sq, st, pr_d, pf_d, ord_d, qset, qph])

    def _retire(self, L: _Launch):
        h = L.host.numpy()
        off = 0
        now = time.perf_counter()
        with self._cv:
            for s in L.slices:
                blk = h[off:off + s.n]
                merge_topk(s.req, blk[:, 0], s.req.lib_idx[s.start:s.stop], blk[:, 1:5],
                           blk[:, 5:8])
                s.req.remaining -= s.n
                off += s.n
                self.pairs_done += s.n
                if s.req.remaining == 0:
                    s.req.finished = now
                    self.latencies.append(now - s.req.arrival)
                    self.completed += 1
                    self.pending.remove(s.req)
                    if s.req.future is not None:
                        s.req.future.set_result(finalize(s.req, self.ids))
            self.planner.retire(L.nbytes)


def shard_ranges(n: int, world: int):
    """Contiguous library ranges for ``world`` ranks (one process per GPU); the per-rank
    top-K lists are merged by score on the host."""
    edges = np.linspace(0, n, world + 1).astype(np.int64)
    return [(int(edges[i]), int(edges[i + 1])) for i in range(world)]


def merge_hits(lists, top_k: int):
    """Merge per-rank hit lists (each sorted by score) into the global top-K."""
    allh = [h for lst in lists for h in lst]
    allh.sort(key=lambda h: (-h.score, h.id))
    return allh[:top_k]
