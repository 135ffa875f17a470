"""Screening server over a library sharded across GPUs (one process per GPU).

Every rank keeps one contiguous range of the library resident (``server.shard_ranges``) and
runs its own continuous-batching server over it.  Rank 0 is the front end: a request
(query + library indices) submitted there is broadcast to every rank, each rank scores the
indices that fall in its range, and the per-rank top-K lists come back to rank 0, which merges
them (``server.merge_hits``) and resolves the request's future.  The reference's counterpart is
its process-per-GPU screen (shepherd_score/screen.py:1202-1297, accel/multi_gpu.py:92-221),
which re-reads the store per call and exchanges results through multiprocessing queues.

The exchange is a control plane of small host objects (queries, index lists, top-K lists:
kilobytes per request), so it runs over a gloo process group on the host, never over NCCL,
and no device memory crosses GPUs.  All ranks run the same tick loop -- one broadcast of the
new messages from rank 0, then one gather of the finished local results to rank 0 -- so every
rank takes the same collective steps in the same order, including on shutdown and on errors
(an error in a rank's local server is reported for the affected requests, not raised out of
the loop).
"""
from __future__ import annotations

import concurrent.futures as cf
import threading
import time
from typing import Dict, List, Optional

import numpy as np
import torch.distributed as dist

from .server import merge_hits


class ShardedScreenServer:
    """``local`` is this rank's server over library positions [lo, hi) (indices local to the
    shard, hits carrying global ids); ``group`` a gloo process group spanning the ranks
    (default: a new gloo group over the default group's ranks)."""

    def __init__(self, local, lo: int, hi: int, n_lib: int, *, group=None,
                 tick_s: float = 0.002):
        self.local = local
        self.lo, self.hi, self.n_lib = int(lo), int(hi), int(n_lib)
        self.group = group if group is not None else dist.new_group(backend="gloo")
        self.rank = dist.get_rank(self.group)
        self.world = dist.get_world_size(self.group)
        self.tick_s = float(tick_s)
        self._lock = threading.Lock()
        self._outbox: List[tuple] = []            # rank 0: messages for the next broadcast
        self._futures: Dict[int, cf.Future] = {}  # rank 0: rid -> the caller's future
        self._topk: Dict[int, int] = {}
        self._parts: Dict[int, Dict[int, list]] = {}   # rank 0: rid -> rank -> hits
        self._local: Dict[int, cf.Future] = {}    # every rank: rid -> local future
        self._rid = 0
        self._stop = False
        self.ticks = 0
        self.error: Optional[BaseException] = None
        self._thread = threading.Thread(target=self._loop, name="fss-sharded-screen",
                                        daemon=True)
        self._thread.start()

    # ---- front end (rank 0) ------------------------------------------------------------
    def submit(self, query: dict, lib_idx=None, top_k: int = 100,
               timeout: Optional[float] = None) -> cf.Future:
        if self.rank != 0:
            raise RuntimeError("requests are submitted on rank 0")
        if lib_idx is None:
            lib_idx = np.arange(self.n_lib, dtype=np.int32)
        lib_idx = np.asarray(lib_idx, np.int64)
        if len(lib_idx) == 0 or lib_idx.min() < 0 or lib_idx.max() >= self.n_lib:
            raise ValueError("library indices must be a non-empty subset of the library")
        fut: cf.Future = cf.Future()
        with self._lock:
            if self._stop:
                raise RuntimeError("sharded server is closed")
            rid = self._rid
            self._rid += 1
            self._futures[rid] = fut
            self._topk[rid] = int(top_k)
            self._parts[rid] = {}
            self._outbox.append(("submit", rid, query, lib_idx, int(top_k), timeout))
        return fut

    def cancel(self, fut: cf.Future) -> bool:
        with self._lock:
            rid = next((r for r, f in self._futures.items() if f is fut), None)
            ok = fut.cancel()
            if ok and rid is not None:
                self._outbox.append(("cancel", rid))
        return ok

    def close(self):
        """Rank 0: finish the outstanding requests, then stop every rank's loop.  Other
        ranks: wait until rank 0 has stopped the loop."""
        if self.rank == 0:
            with self._lock:
                self._stop = True
        self._thread.join()
        self.local.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- every rank ---------------------------------------------------------------------
    def _apply(self, msg):
        kind = msg[0]
        if kind == "submit":
            _, rid, query, lib_idx, top_k, timeout = msg
            mine = lib_idx[(lib_idx >= self.lo) & (lib_idx < self.hi)] - self.lo
            if len(mine) == 0:
                done: cf.Future = cf.Future()
                done.set_result([])
                self._local[rid] = done
                return
            try:
                self._local[rid] = self.local.submit(query, mine.astype(np.int32), top_k,
                                                     timeout=timeout)
            except Exception as exc:             # reported to rank 0 for this request only
                failed: cf.Future = cf.Future()
                failed.set_exception(exc)
                self._local[rid] = failed
        elif kind == "cancel":
            fut = self._local.get(msg[1])
            if fut is not None:
                self.local.cancel(fut)

    def _finished(self) -> list:
        out = []
        for rid, fut in list(self._local.items()):
            if not fut.done():
                continue
            del self._local[rid]
            if fut.cancelled():
                out.append((rid, "cancelled", None))
            elif isinstance(fut.exception(), TimeoutError):
                out.append((rid, "timeout", str(fut.exception())))
            elif fut.exception() is not None:
                out.append((rid, "error", repr(fut.exception())))
            else:
                out.append((rid, "ok", [tuple(h) for h in fut.result()]))
        return out

    def _merge(self, gathered):
        from .screen import Hit
        for rank, done in enumerate(gathered):
            for rid, status, payload in done:
                fut = self._futures.get(rid)
                if fut is None:
                    continue
                if status != "ok":
                    if not fut.done():
                        if status == "error":
                            fut.set_exception(RuntimeError(f"rank {rank}: {payload}"))
                        elif status == "timeout":
                            fut.set_exception(TimeoutError(f"rank {rank}: {payload}"))
                        else:
                            fut.cancel()
                    self._parts[rid][rank] = []
                else:
                    self._parts[rid][rank] = [Hit(*h) for h in payload]
                if len(self._parts[rid]) == self.world:
                    if not fut.done():
                        fut.set_result(merge_hits(list(self._parts[rid].values()),
                                                  self._topk[rid]))
                    del self._futures[rid], self._parts[rid], self._topk[rid]

    def _loop(self):
        try:
            self._ticks()
        except Exception as exc:                 # a collective failed: a peer is gone
            self.error = exc
            with self._lock:
                self._stop = True
                for fut in self._futures.values():
                    if not fut.done():
                        fut.set_exception(RuntimeError(f"sharded server stopped: {exc!r}"))

    def _ticks(self):
        while True:
            msgs = [None]
            if self.rank == 0:
                with self._lock:
                    batch, self._outbox = self._outbox, []
                    stop = self._stop and not batch and not self._futures
                msgs = [(batch, stop)]
            dist.broadcast_object_list(msgs, src=0, group=self.group)
            batch, stop = msgs[0]
            for m in batch:
                self._apply(m)
            done = self._finished()
            gathered = [None] * self.world if self.rank == 0 else None
            dist.gather_object(done, gathered, dst=0, group=self.group)
            self.ticks += 1
            if self.rank == 0:
                with self._lock:
                    self._merge(gathered)
            if stop:
                return
            if not batch and not done:
                time.sleep(self.tick_s)
