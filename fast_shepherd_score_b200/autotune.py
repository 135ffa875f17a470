"""Autotuner for the fused alignment kernel's tiling.

Tunables of one launch (``fss_align_desc``):
  lanes_per_pose  1, 2, 4, 8, 16 or 32 lanes cooperate on one pose (so 32/lanes starts per
                  warp; 1 and 2 are tried for small molecules: no per-step lane reduction,
                  but few warps unless the batch is large)
  chunks          start blocks per pair (a CTA owns one pair and n_starts/chunks starts)
  cta_per_sm      persistent CTAs per SM (1 or 2; 2 hides latency, 1 leaves more L1)
  accumulate      1 = value/gradient sums on the FP32 lanes, 2 = sums on the tensor cores,
                  3 = pairwise exponents on the tensor cores (2 and 3: shape/ESP modes,
                  32 lanes per pose)
  kernel_variant  code variant of the FP32-lane loop (shape/ESP modes): 1 base, 2 wide
                  register tile, 3 one-CTA/SM register budget, 4 base tile unrolled 4x,
                  5 eight-point register tile (small molecules)

For a new problem shape the tuner times each candidate on a sample of the batch's pairs
(the costliest and a spread of the rest) for a few Adam steps, with CUDA events, and keeps
the fastest.  Results are cached per (device, mode, size buckets, starts, pair bucket, step-count
class) in memory and in a JSON file (``$FSS_AUTOTUNE_CACHE`` or ``~/.cache/fast_shepherd_score_b200/autotune.json``).
Set ``FSS_AUTOTUNE=0`` to disable tuning (the library's built-in default is then used).
"""
from __future__ import annotations

import json
import math
import os
import threading
from typing import Optional

import numpy as np
import torch

_LOCK = threading.Lock()
_MEM: dict = {}
_LOADED = False
LANES = (1, 2, 4, 8, 16, 32)


def _cache_path() -> str:
    p = os.environ.get("FSS_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "fast_shepherd_score_b200",
                        "autotune.json")


def _load():
    global _LOADED
    if _LOADED:
        return
    _LOADED = True
    try:
        with open(_cache_path()) as f:
            _MEM.update(json.load(f))
    except Exception:
        pass


def _save():
    try:
        path = _cache_path()
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(_MEM, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except Exception:
        pass


def enabled() -> bool:
    return os.environ.get("FSS_AUTOTUNE", "1") != "0"


def _bucket(x: int) -> int:
    return 0 if x <= 0 else 1 << int(math.ceil(math.log2(max(int(x), 1))))


def steps_class(steps: int) -> int:
    """0: one step (a scoring pass), 1: up to 16 steps (launch- and tail-dominated), 2: longer
    runs (throughput-dominated).  A tile tuned for a few steps is a poor choice for 200."""
    return 0 if steps <= 1 else 1 if steps <= 16 else 2


_NAMES: dict = {}


def _device_name(device) -> str:
    """The device's name (queried once per device: every launch builds a key)."""
    idx = torch.device(device).index
    idx = torch.cuda.current_device() if idx is None else idx
    name = _NAMES.get(idx)
    if name is None:
        name = _NAMES[idx] = torch.cuda.get_device_name(idx).replace(" ", "_")
    return name


def shape_key(device, mode: str, max_ref: int, max_fit: int, mean_fit: float, n_starts: int,
              n_pairs: int, steps: int = 200) -> str:
    name = _device_name(device)
    return (f"{name}|{mode}|r{_bucket(max_ref)}|f{_bucket(max_fit)}|m{_bucket(int(mean_fit))}"
            f"|s{n_starts}|p{_bucket(n_pairs)}|t{steps_class(steps)}")


def candidates(mode: str, max_fit: int, n_starts: int, tensor_cores: bool = None):
    """The tiles the tuner times.  The tensor-core options (``accumulate`` 2 and 3) are timed
    only when ``tensor_cores`` is true (default: ``$FSS_AUTOTUNE_TC=1``): on B200 they were
    measured slower than the FP32 lanes on every workload, so the default sweep leaves them
    out (they stay selectable explicitly)."""
    if tensor_cores is None:
        tensor_cores = os.environ.get("FSS_AUTOTUNE_TC", "0") == "1"
    out = []
    # variant 5 (8 fit points per lane) only where it saves a pass over the reference cloud:
    # fit clouds of at most 8 x 8 lanes' points
    variants = ((1, 2, 3, 4, 5) if mode in ("shape", "esp") and max_fit <= 64 else
                (1, 2, 3, 4) if mode in ("shape", "esp") else
                (1, 3) if mode == "esp_combo" else (0,))
    for lpp in LANES:
        if mode != "pharm" and lpp > 4 and lpp // 2 >= max(max_fit, 1):
            continue  # more lanes than fit points: idle lanes
        if lpp < 4 and max_fit >= 64:
            continue  # a pose per 1-2 lanes pays off only for small molecules in large batches
        if mode == "pharm" and lpp > 8:
            continue
        for var in variants:
            for cps in (0, 2, 1):   # 0 = as many CTAs per SM as fit
                out.append({"lanes_per_pose": lpp, "chunks": 0, "cta_per_sm": cps,
                            "kernel_variant": var})
            # smaller CTAs (twice the default start blocks): less waiting at the per-item barrier
            base = _auto_chunks(lpp, n_starts)
            if 2 * base <= n_starts:
                out.append({"lanes_per_pose": lpp, "chunks": 2 * base, "cta_per_sm": 0,
                            "kernel_variant": var})
            # start blocks that fill whole warps (no lanes shadow an idle start except in a
            # pair's last block), in CTAs of 1, 2 or 4 warps: CTAs whose warps spread evenly
            # over the SM's four schedulers.  A 5-warp CTA puts two warps on one scheduler,
            # and its other warps then wait ~24 % of the time at the per-item barrier
            # (measured on 200-400 point surfaces).
            for warps in ((1, 2, 4) if max_fit < 64 else (2, 4)):
                ppc = warps * (32 // lpp)
                ch = -(-n_starts // ppc)
                if ch not in (base, 2 * base) and ch <= n_starts:
                    out.append({"lanes_per_pose": lpp, "chunks": ch, "cta_per_sm": 0,
                                "kernel_variant": var})
    if tensor_cores and mode in ("shape", "esp") and max_fit >= 16:
        base = _auto_chunks(32, n_starts)
        ch4 = -(-n_starts // 4)     # one pose per warp: CTAs of 4 warps
        for acc in (2, 3):
            for ch, cps in ((0, 0), (0, 1), (2 * base, 0), (ch4, 0)):
                if ch <= n_starts:
                    out.append({"lanes_per_pose": 32, "chunks": ch, "cta_per_sm": cps,
                                "accumulate": acc})
    return out


def _auto_chunks(lpp: int, n_starts: int, max_threads: int = 320) -> int:
    """The library's default start-block count for a lanes-per-pose choice: the fewest idle
    pose slots with CTAs of at most max_threads threads (fss_align.cu auto_tile)."""
    best_c, best_w = 1, 1 << 30
    for c in range(1, n_starts + 1):
        ppc = -(-n_starts // c)
        if ppc > max_threads // lpp:
            continue
        warps = -(-ppc * lpp // 32)
        waste = warps * 32 // lpp * c - n_starts
        if waste < best_w:
            best_c, best_w = c, waste
        if waste == 0:
            break
    return best_c


def lookup(key: str) -> Optional[dict]:
    with _LOCK:
        _load()
        return _MEM.get(key)


def time_once(run, **tile) -> float:
    """Milliseconds of one warm ``run(**tile)`` (CUDA events on the current stream)."""
    run(**tile)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    run(**tile)
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1)


def _time(run, c, repeats):
    ms = []
    for _ in range(repeats):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        run(**c)
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return ms


def _tag(c) -> str:
    acc = c.get("accumulate", 0)
    tag = "tc" if acc == 2 else "tce" if acc == 3 else f"v{c.get('kernel_variant', 0)}:"
    return f"{tag}{c['lanes_per_pose']}x{c['cta_per_sm']}c{c['chunks']}"


def tune(run, key: str, cands, repeats: int = 2, finalists: int = 4,
         final_repeats: int = 5) -> dict:
    """Time ``run(**tile)`` for each candidate tile (best of ``repeats``), re-time the
    ``finalists`` fastest ``final_repeats`` more times each, in turns, and cache and return
    the one with the lowest median of those runs."""
    timings = {}
    first = []
    for c in cands:
        try:
            run(**c)  # warm (shared-memory attribute, first-launch costs)
            t = min(_time(run, c, repeats))
        except (ValueError, RuntimeError):
            continue
        timings[_tag(c)] = round(t, 4)
        first.append((t, len(first), c))
    first.sort(key=lambda x: (x[0], x[1]))
    best, best_ms = None, float("inf")
    if first:
        top = [c for _, _, c in first[:finalists]]
        runs = {i: [] for i in range(len(top))}
        for _ in range(final_repeats):      # in turns: slow drifts hit every finalist alike
            for i, c in enumerate(top):
                runs[i].extend(_time(run, c, 1))
        for i, c in enumerate(top):
            t = float(np.median(runs[i]))
            timings["final:" + _tag(c)] = round(t, 4)
            if t < best_ms:
                best, best_ms = c, t
    if best is None:
        best = {"lanes_per_pose": 0, "chunks": 0, "cta_per_sm": 0}
    rec = dict(best)
    rec["ms"] = round(best_ms, 4) if best_ms < float("inf") else None
    rec["timings"] = timings
    with _LOCK:
        _load()
        _MEM[key] = rec
        _save()
    return rec


def sample_pairs(cost: np.ndarray, k: int) -> np.ndarray:
    """Indices of a representative sample: the costliest pairs and an even spread."""
    order = np.argsort(-cost, kind="stable")
    if len(order) <= k:
        return order
    head = order[: k // 4]
    rest = order[k // 4:]
    spread = rest[np.linspace(0, len(rest) - 1, k - len(head)).astype(np.int64)]
    return np.concatenate([head, spread])
