"""Continuous-batching screening server over a device-resident library.

A request is one query molecule scored against a set of library molecules (1k-100k) and
answered with its top-K hits.  The library (packed clouds + pharmacophores + per-molecule
self overlaps) is uploaded once and stays in HBM (:meth:`ScreenServer.from_store` loads a
ProfileStore; a float16 store stays float16 on the device and the kernels widen it while
staging).  A scheduler thread keeps the GPU fed:

* **admission** -- pending requests are cut into slices (consecutive ranges of their library
  indices) and admitted while the launch's pair budget and the in-flight HBM budget (seeds,
  rows and results of every launch not yet retired) allow; a request that does not fit waits
  for earlier launches to retire.  The order is shortest-remaining-first with ageing (a
  request's unscheduled pairs divided by 1 + its waiting time / ``aging_s``), so a small
  request does not queue behind a large one's slices, and a large one is not starved;
  ``policy="fifo"`` admits in arrival order;
* **continuous batching** -- one fused-kernel launch carries slices of many requests (each
  request's query is one molecule of the launch's query set); requests that arrive while
  launches run join the next launch, and up to ``max_in_flight`` launches are queued on the
  stream so the device never idles between them;
* **retirement** -- when a launch's completion event fires, its per-pair results (already
  copied to pinned host memory) are merged into each request's running top-K; the last
  slice resolves the request's future and records its latency (by request size);
* **cancellation and deadlines** -- ``future.cancel()`` (or :meth:`ScreenServer.cancel`) and a
  per-request ``timeout`` end a request early: its unscheduled slices are never admitted, the
  slices already in flight are dropped when their launch retires (which returns their HBM
  budget), and the future is never resolved with hits (cancelled, or ``TimeoutError``).

The scheduling logic (:class:`ServeLoop`) is host-only and drives an *engine* with two calls,
``launch(slices)`` and ``wait(handle) -> (P, 8) array`` (score, q, t per pair); the CUDA engine
is :class:`_CudaEngine`, tests substitute a host one.  Every pair is computed independently
with a fixed tiling, so a request's result is the same alone and in any mix
(tests/test_gpu_server.py).  Reference counterpart: the streaming loop of
shepherd_score/screen.py:962-1035, which re-buckets per query and has no admission, overlap,
cancellation or latency accounting.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import math
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np
import torch

from . import align as al
from . import api
from . import kernels as K
from .layout import CloudSet, PharmSet


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
    deadline: Optional[float] = None   # absolute time (the server's clock); None: no limit
    next: int = 0                  # first library position not yet scheduled
    remaining: int = 0             # pairs not yet retired
    best_s: np.ndarray = None
    best_i: np.ndarray = None
    best_q: np.ndarray = None
    best_t: np.ndarray = None
    finished: Optional[float] = None
    dead: bool = False             # cancelled or past its deadline: nothing more is scheduled

    def __post_init__(self):
        self.remaining = len(self.lib_idx)

    @property
    def unscheduled(self) -> int:
        return len(self.lib_idx) - self.next


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
                 slice_pairs: int = 8192, policy: str = "srpt", aging_s: float = 0.25):
        if policy not in ("srpt", "fifo"):
            raise ValueError("policy must be 'srpt' or 'fifo'")
        self.max_pairs = int(max_pairs_per_launch)
        self.budget = int(hbm_budget_bytes)
        self.bpp = int(bytes_per_pair)
        self.slice_pairs = int(slice_pairs)
        self.policy = policy
        self.aging_s = float(aging_s)
        self.in_flight_bytes = 0

    def order(self, pending, now: float = 0.0) -> List[Request]:
        """Live requests with unscheduled pairs, in admission order."""
        live = [r for r in pending if not r.dead and r.unscheduled > 0]
        if self.policy == "fifo":
            return live
        age = lambda r: max(0.0, now - r.arrival)
        return sorted(live, key=lambda r: (r.unscheduled / (1.0 + age(r) / self.aging_s),
                                           r.arrival, r.rid))

    def plan(self, pending, now: float = 0.0) -> List[Slice]:
        out, pairs = [], 0
        for req in self.order(pending, now):
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


def _py(x):
    return x.item() if isinstance(x, np.generic) else x


def finalize(req: Request, ids=None):
    """The request's hits: score descending, then library index ascending."""
    order = np.lexsort((req.best_i, -req.best_s))
    T = api.se3_from_qt(req.best_q[order], req.best_t[order])
    from .screen import Hit
    lib = req.best_i[order]
    return [Hit(score=float(s), id=_py(ids[j]) if ids is not None else int(j), transform=tf)
            for s, j, tf in zip(req.best_s[order], lib, T)]


def percentile(xs, p):
    if not xs:
        return float("nan")
    return float(np.percentile(np.asarray(xs), p))


def latency_by_decade(records) -> dict:
    """{"1e3-1e4": {"requests", "p50_ms", "p99_ms"}, ...} from (pairs, seconds) records."""
    out = {}
    for lo in range(0, 9):
        sel = [t for n, t in records if 10 ** lo <= n < 10 ** (lo + 1)]
        if sel:
            out[f"1e{lo}-1e{lo + 1}"] = {"requests": len(sel),
                                         "p50_ms": round(percentile(sel, 50) * 1e3, 2),
                                         "p99_ms": round(percentile(sel, 99) * 1e3, 2)}
    return out


def slowdown(records, capacity_pairs_per_s: float) -> dict:
    """Latency over the request's own service time at full capacity (pairs / capacity), from
    (pairs, seconds) records: {"p50", "p99", "by_request_size": {decade: {"p50", "p99"}}}.
    Unlike raw latency it does not grow with the request's size, so it shows how much waiting
    the admission order adds for small and large requests alike (1 = served alone at full
    speed)."""
    if not records or not capacity_pairs_per_s > 0:
        return {}
    sd = [(n, t * capacity_pairs_per_s / max(n, 1)) for n, t in records]
    out = {"p50": round(percentile([x for _, x in sd], 50), 2),
           "p99": round(percentile([x for _, x in sd], 99), 2), "by_request_size": {}}
    for lo in range(0, 9):
        sel = [x for n, x in sd if 10 ** lo <= n < 10 ** (lo + 1)]
        if sel:
            out["by_request_size"][f"1e{lo}-1e{lo + 1}"] = {
                "p50": round(percentile(sel, 50), 2), "p99": round(percentile(sel, 99), 2)}
    return out


class ServeLoop:
    """The scheduler: admission, continuous batching, retirement, cancellation and deadlines,
    over an engine with ``launch(slices) -> handle`` and ``wait(handle) -> (P, 8) results``
    (one row per pair of the launch's slices, in slice order: score, q (4), t (3))."""

    def __init__(self, engine, n_lib: int, planner: Planner, *, max_in_flight: int = 2,
                 ids=None, clock: Callable[[], float] = time.perf_counter,
                 name: str = "fss-screen-server"):
        self.engine = engine
        self.n_lib = int(n_lib)
        self.planner = planner
        self.max_in_flight = int(max_in_flight)
        self.ids = ids
        self.clock = clock
        self.pending: "collections.deque[Request]" = collections.deque()
        self.in_flight: "collections.deque" = collections.deque()
        self.latencies: List[float] = []
        self.size_latency: List[tuple] = []
        self.completed = self.cancelled = self.expired = 0
        self.pairs_done = 0
        self.max_queue = 0
        self._rid = 0
        self._cv = threading.Condition()
        self._stop = False
        self._err: Optional[BaseException] = None
        self._thread = threading.Thread(target=self._run, name=name, daemon=True)
        self._thread.start()

    # ---- client side -------------------------------------------------------------------
    def submit(self, query: dict, lib_idx=None, top_k: int = 100,
               timeout: Optional[float] = None) -> cf.Future:
        """Queue one query against ``lib_idx`` (default: the whole library).  ``timeout``
        (seconds from now) is the request's deadline: past it the future fails with
        ``TimeoutError`` and its remaining work is dropped."""
        if lib_idx is None:
            lib_idx = np.arange(self.n_lib, dtype=np.int32)
        lib_idx = np.asarray(lib_idx, dtype=np.int32)
        if len(lib_idx) == 0:
            raise ValueError("empty request")
        if lib_idx.min() < 0 or lib_idx.max() >= self.n_lib:
            raise ValueError("library index out of range")
        if top_k < 1:
            raise ValueError("top_k must be >= 1")
        fut: cf.Future = cf.Future()
        with self._cv:
            if self._err is not None:
                raise RuntimeError("screen server stopped after an error") from self._err
            if self._stop:
                raise RuntimeError("screen server is closed")
            now = self.clock()
            req = Request(self._rid, self._prepare(query), lib_idx, int(top_k), now, fut,
                          None if timeout is None else now + float(timeout))
            self._rid += 1
            self.pending.append(req)
            self.max_queue = max(self.max_queue, len(self.pending))
            self._cv.notify()
        return fut

    def _prepare(self, query):
        return query

    def cancel(self, fut: cf.Future) -> bool:
        """Cancel a request that has not resolved; True when it is cancelled."""
        ok = fut.cancel()
        with self._cv:
            self._cv.notify()
        return ok

    def stats(self) -> dict:
        with self._cv:
            lat = list(self.latencies)
            return {"completed": self.completed, "cancelled": self.cancelled,
                    "expired": self.expired, "pairs_done": self.pairs_done,
                    "p50_ms": percentile(lat, 50) * 1e3, "p99_ms": percentile(lat, 99) * 1e3,
                    "by_request_size": latency_by_decade(self.size_latency),
                    "queue_depth": len(self.pending), "max_queue_depth": self.max_queue,
                    "in_flight_bytes": self.planner.in_flight_bytes,
                    "in_flight_launches": len(self.in_flight)}

    def close(self):
        """Finish every admitted and pending request, then stop the scheduler."""
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
    def _reap(self, now: float):
        """Drop cancelled and expired requests from the queue (under the lock)."""
        for r in list(self.pending):
            if r.dead:
                continue
            if r.future is not None and r.future.cancelled():
                r.dead = True
                self.cancelled += 1
            elif r.deadline is not None and now > r.deadline:
                r.dead = True
                self.expired += 1
                if r.future is not None and not r.future.done():
                    r.future.set_exception(TimeoutError(
                        f"request {r.rid} passed its deadline with {r.remaining} of "
                        f"{len(r.lib_idx)} pairs unscored"))
            if r.dead:
                self.pending.remove(r)

    def _has_work(self) -> bool:
        return any(not r.dead and r.unscheduled > 0 for r in self.pending)

    def _run(self):
        try:
            self._enter_thread()
            while True:
                with self._cv:
                    while (not self._stop and not self.in_flight and not self._has_work()):
                        self._cv.wait(0.05)
                        self._reap(self.clock())
                    self._reap(self.clock())
                    if self._stop and not self.in_flight and not self.pending:
                        return
                    slices, nbytes = [], 0
                    if len(self.in_flight) < self.max_in_flight:
                        slices = self.planner.plan(self.pending, self.clock())
                        if slices:
                            nbytes = self.planner.admit(slices)
                if slices:
                    self.in_flight.append((slices, nbytes, self.engine.launch(slices)))
                    continue                     # keep the queue of launches full
                if self.in_flight:
                    slices, nbytes, handle = self.in_flight[0]
                    res = self.engine.wait(handle)
                    self.in_flight.popleft()
                    self._retire(slices, nbytes, res)
        except BaseException as exc:             # surface errors to every waiter
            with self._cv:
                self._err = exc
                for r in self.pending:
                    if r.future is not None and not r.future.done():
                        r.future.set_exception(exc)

    def _enter_thread(self):
        pass

    def _retire(self, slices: List[Slice], nbytes: int, h: np.ndarray):
        off = 0
        now = self.clock()
        with self._cv:
            self._reap(now)
            for s in slices:
                blk = h[off:off + s.n]
                off += s.n
                if s.req.dead:                   # cancelled / expired: results dropped
                    continue
                merge_topk(s.req, blk[:, 0], s.req.lib_idx[s.start:s.stop], blk[:, 1:5],
                           blk[:, 5:8])
                s.req.remaining -= s.n
                self.pairs_done += s.n
                if s.req.remaining == 0:
                    s.req.finished = now
                    self.latencies.append(now - s.req.arrival)
                    self.size_latency.append((len(s.req.lib_idx), now - s.req.arrival))
                    self.completed += 1
                    self.pending.remove(s.req)
                    if s.req.future is not None and not s.req.future.done():
                        s.req.future.set_result(finalize(s.req, self.ids))
            self.planner.retire(nbytes)


# ----------------------------------------------------------------------------------------
# Device side
# ----------------------------------------------------------------------------------------
@dataclass
class _Launch:
    host: torch.Tensor            # pinned (P, 8): score, q, t
    event: torch.cuda.Event
    keep: list = field(default_factory=list)   # device tensors alive until retirement


class _CudaEngine:
    """One fused launch per admitted slice set, on the server's stream."""

    def __init__(self, atoms: CloudSet, pharm: Optional[PharmSet], mode: str, S: int,
                 steps: int, lr: float, alpha: float, w: float, lpp: int, tile: dict, dev):
        self.atoms, self.pharm, self.mode = atoms, pharm, mode
        self.S, self.steps, self.lr, self.alpha, self.w = S, steps, lr, alpha, w
        self.lpp, self.tile, self.dev = lpp, tile, dev
        directional = mode == "vol_pharm"
        with torch.cuda.device(dev):
            self.lib_self = K.self_overlap(atoms, alpha)
            self.lib_self_ph = (K.pharm_self_overlap(pharm, directional)
                                if mode != "vol" else None)
        self.stream = torch.cuda.Stream(dev)

    def launch(self, slices: List[Slice]) -> _Launch:
        dev = self.dev
        with torch.cuda.stream(self.stream):
            reqs = list(dict.fromkeys(s.req for s in slices))   # unique, in order
            qpos = {r.rid: k for k, r in enumerate(reqs)}
            qset = CloudSet.from_arrays([r.query["atom_pos"] for r in reqs], device=dev,
                                        non_blocking=True)
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
            amode = {"vol": "shape", "vol_color": "shape_color",
                     "vol_pharm": "shape_pharm"}[self.mode]
            res = al.align_packed(amode, ref=qset, fit=self.atoms,
                                  ref_ph=qph, fit_ph=self.pharm if self.mode != "vol" else None,
                                  pair_ref=pr_d, pair_fit=pf_d, seed_q=sq, seed_t=st,
                                  steps=self.steps, lr=self.lr, alpha=self.alpha,
                                  color_weight=self.w, ref_self=q_self, fit_self=self.lib_self,
                                  ref_self_ph=q_self_ph, fit_self_ph=self.lib_self_ph,
                                  order=ord_d, lanes_per_pose=self.lpp, check_status=False,
                                  validate=False, **self.tile)
            sc, q, t = res
            host = torch.empty(P, 8, dtype=torch.float32, pin_memory=True)
            host.copy_(torch.cat([sc[:, None], q, t], 1), non_blocking=True)
            ev = torch.cuda.Event()
            ev.record()
        return _Launch(host, ev, keep=[res, sq, st, pr_d, pf_d, ord_d, qset, qph])

    def wait(self, L: _Launch) -> np.ndarray:
        L.event.synchronize()
        return L.host.numpy()


class ScreenServer(ServeLoop):
    """Serve screening requests against a device-resident library.

    ``library`` = (CloudSet atoms, PharmSet pharmacophores) on ``device`` (e.g. from
    :func:`fast_shepherd_score_b200.synthetic.library_on_device`), or use :meth:`from_store`.
    ``mode`` is "vol_pharm" (shape + directional pharmacophores, the default), "vol_color" or
    "vol".  Queries are dicts of arrays (``atom_pos``, ``pharm_types`` / ``pharm_ancs`` /
    ``pharm_vecs``); ``center_queries`` shifts each to its atom centroid first (for a
    pre-centred library).
    """

    def __init__(self, library, *, mode: str = "vol_pharm", starts: int = 20, steps: int = 100,
                 lr: float = 0.1, alpha: float = 0.81, color_weight: float = 0.5,
                 max_pairs_per_launch: int = 8192, hbm_budget_bytes: Optional[int] = None,
                 lanes_per_pose: int = 8, max_in_flight: int = 2, slice_pairs: int = 8192,
                 ids=None, device=None, tile: Optional[dict] = None, policy: str = "srpt",
                 aging_s: float = 0.25, center_queries: bool = False):
        if mode not in ("vol", "vol_color", "vol_pharm"):
            raise ValueError("mode must be 'vol', 'vol_color' or 'vol_pharm'")
        self.atoms, self.pharm = library
        self.dev = torch.device(device or self.atoms.pts.device)
        self.mode = mode
        self.S = int(starts)
        self.center_queries = bool(center_queries)
        # the tile (lanes per pose, start blocks, CTAs per SM, code variant) is fixed for the
        # server's life, so a request's result does not depend on its launch-mates
        tile = {k: int(v) for k, v in (tile or {}).items()
                if k in ("chunks", "cta_per_sm", "kernel_variant")}
        self.engine = _CudaEngine(self.atoms, self.pharm, mode, self.S, int(steps), float(lr),
                                  float(alpha), float(color_weight), int(lanes_per_pose), tile,
                                  self.dev)
        self.stream = self.engine.stream
        # bytes per in-flight pair: seeds (7 floats/start), rows (8 floats/start), results,
        # pair indices
        bpp = self.S * (7 + 8) * 4 + 8 * 4 + 8
        if hbm_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.dev)
            hbm_budget_bytes = int(0.25 * free)
        planner = Planner(max_pairs_per_launch, hbm_budget_bytes, bpp, slice_pairs, policy,
                          aging_s)
        super().__init__(self.engine, self.atoms.n_mol, planner, max_in_flight=max_in_flight,
                         ids=ids)

    @classmethod
    def from_store(cls, store, device=None, *, mode: str = "vol_pharm", widen: bool = False,
                   **kw) -> "ScreenServer":
        """A server over every molecule of a ProfileStore (this package's or shepherd_score's
        object, or a path), uploaded once in the store's dtype (``widen`` converts a float16
        store to float32 on upload instead).  Hits carry the store's ids; queries are centred
        on their atoms when the store is pre-centred, as screen() does."""
        from .library import Library
        from .store import ProfileStore
        if isinstance(store, str):
            store = ProfileStore.open(store)
        if not store.supports(mode):
            raise ValueError(f"store at {store.path!r} does not support mode {mode!r}")
        lib = Library.from_store(store, device, pharm=mode != "vol",
                                 vectors=mode == "vol_pharm", widen=widen)
        kw.setdefault("center_queries", bool(store.pre_centered))
        srv = cls((lib.atoms, lib.pharm), mode=mode, ids=lib.ids, device=device, **kw)
        srv.library = lib
        return srv

    def _prepare(self, query):
        if self.center_queries:
            from .screen import _centred_query
            return _centred_query(query)
        return query

    def _enter_thread(self):
        torch.cuda.set_device(self.dev)


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
