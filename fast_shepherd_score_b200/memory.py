"""Memory-bounded sub-batching of independent pairs, with halving on out-of-memory.

Pairs are independent (each result is its own maximum over starts, and a pair's result does
not depend on the other pairs of its launch), so splitting a batch into chunks and
concatenating the results is exactly equivalent to one call; it only bounds the device memory
a call holds at once.  This is the role of the reference's ``_subbatched_align``
(shepherd_score/accel/batch/_pad.py:24-97).  Here the per-pair footprint is not measured but
known: the host layer allocates every buffer of a launch itself (the CUDA library allocates
nothing), so :func:`align_bytes_per_pair` counts them.  A chunk is sized to ``SAFETY`` x (free
device memory + torch's reusable cache); an out-of-memory error on a chunk halves it and
retries, down to one pair.

Every buffer of the alignment path is requested through :func:`empty`, which consults an
optional allocation hook first.  The hook exists for fault injection (tests make it refuse
large requests as a device allocator would, with ``FSS_ERR_NOMEM`` mapped to ``MemoryError``)
and for callers that want a hard cap.
"""
from __future__ import annotations

import threading
from typing import Callable, Optional, Sequence

import torch

SAFETY = 0.7
# bytes per pose row of a fused launch: best score (4) + pose (16 + 12), and the seeds (28)
ROW_BYTES = 4 + 16 + 12
SEED_BYTES = 16 + 12
# per pair: index pair (8), cost order (4 + sort scratch 16), outputs (32), self overlaps (8)
PAIR_BYTES = 8 + 20 + 32 + 8

_HOOK: Optional[Callable[[int, torch.device], int]] = None
_LOCK = threading.Lock()
LAST_CHUNKS: list = []   # chunk sizes of the most recent chunked call (for reports and tests)


def set_alloc_hook(hook: Optional[Callable[[int, torch.device], int]]) -> None:
    """Install ``hook(nbytes, device) -> fss status`` (0 = go ahead); a non-zero status is
    raised as the library's exception for it (``FSS_ERR_NOMEM`` -> ``MemoryError``).  None
    removes it."""
    global _HOOK
    with _LOCK:
        _HOOK = hook


def empty(shape, dtype=torch.float32, device=None) -> torch.Tensor:
    """``torch.empty`` for the alignment path's buffers, through the allocation hook."""
    hook = _HOOK
    if hook is not None:
        n = 1
        for s in (shape if isinstance(shape, (tuple, list)) else (shape,)):
            n *= int(s)
        rc = hook(n * torch.empty((), dtype=dtype).element_size(), torch.device(device))
        if rc:
            from . import _lib
            _lib.raise_status(rc, f"allocation of {tuple(shape) if isinstance(shape, (tuple, list)) else (shape,)}")
    return torch.empty(shape, dtype=dtype, device=device)


def align_bytes_per_pair(starts: int, grid_poses: int = 0) -> int:
    """Device bytes one pair holds during an alignment call with ``starts`` starts (plus a
    translation-seeded grid of ``grid_poses`` scored poses, if any)."""
    return PAIR_BYTES + starts * (ROW_BYTES + SEED_BYTES) + grid_poses * (ROW_BYTES + SEED_BYTES)


def budget_bytes(device, need: int = 0) -> int:
    """``SAFETY`` x (free device memory + memory torch holds but does not use).  When
    ``SAFETY`` x the free memory alone already covers ``need`` bytes, that is returned without
    reading torch's allocator statistics (a few hundred microseconds a call)."""
    device = torch.device(device)
    free, _ = torch.cuda.mem_get_info(device)
    if need and SAFETY * free >= need:
        return int(SAFETY * free)
    reusable = torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)
    return int(SAFETY * (free + max(0, reusable)))


def is_oom(exc: BaseException) -> bool:
    if isinstance(exc, (MemoryError, torch.cuda.OutOfMemoryError)):
        return True
    return isinstance(exc, RuntimeError) and "out of memory" in str(exc).lower()


def run_chunked(n: int, per_item_bytes: int, process: Callable[[int, int], Sequence],
                device, *, budget: Optional[int] = None, max_chunk: Optional[int] = None):
    """Run ``process(start, count)`` over ``n`` independent items in chunks that fit the
    memory budget and concatenate its per-item results along dim 0.

    ``process`` returns a sequence of tensors whose first dimension is ``count`` (``None``
    entries stay ``None``); a chunked call returns the concatenation, a single chunk returns
    ``process(0, n)`` as it is.  An out-of-memory error halves the chunk and retries it; one
    item that does not fit re-raises."""
    LAST_CHUNKS.clear()
    if n <= 0:
        return process(0, n)
    if budget is None:
        budget = (budget_bytes(device, n * per_item_bytes) if torch.device(device).type == "cuda"
                  else 1 << 62)
    chunk = max(1, min(n, int(budget // max(1, per_item_bytes))))
    if max_chunk:
        chunk = max(1, min(chunk, int(max_chunk)))
    parts = []
    start = 0
    while start < n:
        k = min(chunk, n - start)
        try:
            res = process(start, k)
        except BaseException as exc:  # noqa: B036 - re-raised unless it is an OOM
            if not is_oom(exc) or k <= 1:
                raise
            if torch.device(device).type == "cuda":
                torch.cuda.empty_cache()
            chunk = max(1, k // 2)
            continue
        LAST_CHUNKS.append(k)
        parts.append(res)
        start += k
    if len(parts) == 1:
        return parts[0]
    return _concat(parts)


def _concat(parts):
    first = parts[0]
    out = []
    for i in range(len(first)):
        col = [p[i] for p in parts]
        out.append(None if any(c is None for c in col) else torch.cat(col))
    rows = [getattr(p, "rows", None) for p in parts]
    res = type(first)(out) if isinstance(first, tuple) and type(first) is not tuple else tuple(out)
    if hasattr(first, "rows"):
        res.rows = (None if any(r is None for r in rows)
                    else tuple(torch.cat([r[j] for r in rows]) for j in range(len(rows[0]))))
    return res
