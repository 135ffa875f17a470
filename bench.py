"""Benchmark of the fused alignment path (one JSON line on rank 0).

Workload (default): the ragged ESP surface batch -- 4096 pairs of surface clouds with
200-400 points each (5 A sphere + N(0, 0.3) jitter, charges N(0, 0.1)), surf_esp scoring
(alpha 0.81, lam 0.3 -> lam * LAM_SCALING), 50 starts x 200 Adam steps, lr 0.1.  Seeded
synthetic data; no dataset.  A *step* is one pass of the hot path over the whole batch:
self overlaps, seeds, the fused alignment kernel and the per-pair pick.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]
                  [--workload surf_esp|vol|vol_pharm] [--pairs P]

value      aligned pairs/s with the inputs resident in HBM (device-timed, CUDA events),
           L2 flushed between timed steps (a 256 MB write, outside the timed windows)
e2e        the same through the host-array public API (fast_shepherd_score_b200.api.align_host)
           with pinned host inputs: H2D of the packed clouds + compute + D2H of the results
roofline   achieved pair-terms/s of the fused kernel against the MUFU ex2 roof measured on
           this GPU by the probe kernel (1 ex2 per pair-term)
cpu_baseline  the CPU oracle (C restatement of the reference's numba path, all host
           threads) on a bounded sample of the same workload
--impl reference  times only that CPU implementation (rank 0; other ranks exit 0)
Multi-GPU: one process per GPU (torchrun), each rank aligns its own batch (weak scaling),
time = max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
import warnings

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "surf_esp": dict(mode="surf_esp", pairs=4096, lo=200, hi=400, starts=50, steps=200,
                     lr=0.1, alpha=0.81, lam=0.3,
                     desc="ragged ESP surface batch: 4096 pairs, 200-400 pts, surf_esp, "
                          "50 starts x 200 Adam steps"),
    "vol": dict(mode="vol", pairs=256, lo=15, hi=50, starts=50, steps=200, lr=0.1, alpha=0.81,
                lam=0.0, desc="plain shape alignment: 256 pairs, 15-50 atoms, vol, "
                              "50 starts x 200 Adam steps"),
    "vol_pharm": dict(mode="vol_pharm", pairs=16384, lo=15, hi=60, starts=50, steps=200,
                      lr=0.1, alpha=0.81, lam=0.0,
                      desc="combined shape+pharmacophore: 16384 pairs, 15-60 atoms + 3-20 "
                           "features, 50 starts x 200 Adam steps"),
    "score_grad": dict(mode="score_grad", pairs=1024, lo=60, hi=300, starts=1, steps=1,
                       lr=0.0, alpha=0.81, lam=0.3,
                       desc="differentiable scoring: 1024 queries of 60 atoms + 300 surface "
                            "points (charges N(0, 0.1^2)) vs 4 fixed targets; vol Tanimoto "
                            "(alpha 0.81) + surface ESP Tanimoto (alpha 1.216) and their "
                            "coordinate/charge gradients"),
    "vol_and_surf_esp": dict(mode="vol_and_surf_esp", pairs=4096, lo=10, hi=25, starts=8,
                             steps=60, lr=0.1, alpha=0.81, lam=0.001,
                             desc="ShaEP combo: 4096 pairs, 10-25 heavy atoms (+H), 100-200 "
                                  "surface points with ESP, 8 starts x 60 Adam steps, combo "
                                  "score every step"),
}


# The headline metric (the 50-start x 200-step alignment workloads); both arms of the bench
# print this exact string for it, so their lines are directly comparable.
HEADLINE_METRIC = ("aligned pairs/s (50 starts\u00d7200 steps) batched vs plain; p50/p99 screen "
                   "latency")


def metric_of(wl):
    """The metric string of a workload, identical in the CUDA and the reference arm."""
    if wl["mode"] == "score_grad":
        return ("scored queries/s (vol + surface-ESP Tanimoto with coordinate and charge "
                "gradients)")
    if wl["starts"] == 50 and wl["steps"] == 200:
        return HEADLINE_METRIC
    return f"aligned pairs/s ({wl['mode']}: {wl['starts']} starts x {wl['steps']} Adam steps)"


def dist_env():
    """(world size, rank, local rank) of this process (torchrun's environment)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def e2e_count(warm_ms: float) -> int:
    """Timed end-to-end calls after the warm-up: at least 3, and for short calls enough to
    span about a second (at most 21), so that host jitter on a shared machine does not decide
    a millisecond-scale median."""
    return max(3, min(21, int(1000.0 / max(warm_ms, 1e-3))))


def make_inputs(wl, n_pairs, seed):
    from fast_shepherd_score_b200 import synthetic as syn
    from fast_shepherd_score_b200.api import HostBatch
    if wl["mode"] == "vol_and_surf_esp":
        refs, fits = syn.esp_combo_pairs(n_pairs, seed=seed, heavy_lo=wl["lo"], heavy_hi=wl["hi"])
        return None, None, (refs, fits)
    if wl["mode"] == "surf_esp":
        refs, fits = syn.esp_surface_pairs(n_pairs, seed=seed, lo=wl["lo"], hi=wl["hi"])
        ref = HostBatch.from_lists([p for p, _ in refs], [c for _, c in refs])
        fit = HostBatch.from_lists([p for p, _ in fits], [c for _, c in fits])
        raw = (refs, fits)
    elif wl["mode"] == "vol":
        refs, fits = syn.shape_pairs(n_pairs, seed=seed, lo=wl["lo"], hi=wl["hi"])
        ref, fit = HostBatch.from_lists(refs), HostBatch.from_lists(fits)
        raw = (refs, fits)
    else:
        refs, fits = syn.shape_pharm_pairs(n_pairs, seed=seed, atom_lo=wl["lo"], atom_hi=wl["hi"])
        mk = lambda ms: HostBatch.from_lists([m["atom_pos"] for m in ms], None,
                                             [m["pharm_types"] for m in ms],
                                             [m["pharm_ancs"] for m in ms],
                                             [m["pharm_vecs"] for m in ms])
        ref, fit = mk(refs), mk(fits)
        raw = (refs, fits)
    return ref, fit, raw


def algorithmic_terms(wl, ref, fit):
    """Pair-terms of one step: starts x steps x sum over pairs of N*M (real, unpadded)."""
    per = (ref.counts.astype(np.int64) * fit.counts.astype(np.int64)).sum()
    if wl["mode"] == "vol_pharm":
        per += (ref.ph_counts.astype(np.int64) * fit.ph_counts.astype(np.int64)).sum()
    return int(per) * wl["starts"] * wl["steps"]


class ClockSampler:
    """nvidia-smi clock / throttle sampling in the background during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace('.', '').isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace('.', '').isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9
                          for i, v in enumerate(r[5:9]) if v.strip().lower() == "active"})
        load = sorted(sm)[len(sm) // 4:] if sm else []   # drop idle-ish samples at the edges
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(sm)}


def measure_peak(dev):
    """MUFU ex2 and FP32 FMA throughput of this GPU (ops/s) from the probe kernel."""
    import ctypes
    import torch
    from fast_shepherd_score_b200 import _lib
    L = _lib.load()
    out = torch.zeros(1 << 16, device=dev)
    res = {}
    for which, name in ((0, "ex2"), (1, "ffma")):
        ops = ctypes.c_longlong(0)
        iters = 4096 if which == 0 else 16384
        st = _lib.stream_ptr(dev)
        _lib.check(L.fss_probe_peak(which, 256, 8, _lib.ptr(out), ctypes.byref(ops), st))
        torch.cuda.synchronize(dev)
        best = 0.0
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.check(L.fss_probe_peak(which, iters, 8, _lib.ptr(out), ctypes.byref(ops), st))
            e1.record()
            torch.cuda.synchronize(dev)
            best = max(best, ops.value / (e0.elapsed_time(e1) * 1e-3))
        res[name] = best
    return res


def flush_l2(buf):
    buf.add_(1.0)   # 256 MB read+write: evicts the 126 MB L2


# DRAM bytes (read + write) per pair of one fused-kernel launch, from an ncu capture of the
# same workload at 256 pairs (dram__bytes_read.sum + dram__bytes_write.sum = 3.318 MB + 0 B),
# scaled by pairs; the kernel's traffic grows with the pairs it processes.
DRAM_BYTES_PER_PAIR = {"surf_esp": (3.318272e6 + 0.0) / 256}


def hbm_peak_gbs():
    """HBM copy bandwidth to compare the fused kernel's DRAM traffic with: the driver-measured
    figure when the repository carries one, else the pool's earlier measurement (6650 GB/s)."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        v = d.get("hbm_gbs")
        if isinstance(v, dict):
            v = v.get("burst", v.get("value"))
        return float(v), "measured"
    except Exception:
        return 6650.0, "fallback"


def hbm_side(traffic_bytes, kernel_ms):
    """The HBM view of a launch that is not HBM-bound: achieved DRAM GB/s and its fraction."""
    if traffic_bytes is None:
        return None
    peak, src = hbm_peak_gbs()
    gbs = traffic_bytes / (kernel_ms * 1e-3) / 1e9
    return {"achieved": round(gbs, 2), "peak": peak, "unit": "GB/s",
            "frac": round(gbs / peak, 6), "peak_source": src}


def run_cuda(args, wl):
    import torch
    import torch.distributed as dist
    from fast_shepherd_score_b200 import _lib, api, kernels as K
    from fast_shepherd_score_b200 import align as al
    from fast_shepherd_score_b200.layout import cost_order_device

    world, rank, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n_pairs = args.pairs or wl["pairs"]
    ref_h, fit_h, raw = make_inputs(wl, n_pairs, seed=1 + rank)
    mode = wl["mode"]
    terms = algorithmic_terms(wl, ref_h, fit_h)

    # ---- device-resident step ---------------------------------------------------------
    rc, rp = ref_h.to_device(dev)
    fc, fp = fit_h.to_device(dev)
    idx = torch.arange(n_pairs, dtype=torch.int32, device=dev)
    cs_r, cs_f = (rc, fc) if rc is not None else (rp, fp)
    order = cost_order_device(cs_r.off, cs_f.off, idx, idx)
    esp = mode == "surf_esp"
    kl = api._kernel_lam(mode, wl["lam"]) if esp else None
    P, S = n_pairs, wl["starts"]
    rows = (torch.empty(P * S, device=dev), torch.empty(P * S, 4, device=dev),
            torch.empty(P * S, 3, device=dev))
    outb = (torch.empty(P, device=dev), torch.empty(P, 4, device=dev), torch.empty(P, 3, device=dev))
    align_ms = []
    tile = {}
    if args.tile:   # fixed tiling (no autotuning): lanes_per_pose,chunks,cta_per_sm,accumulate
        v = [int(x) for x in args.tile.split(",")]
        tile = dict(zip(("lanes_per_pose", "chunks", "cta_per_sm", "accumulate",
                             "kernel_variant"), v))

    def step(record_kernel=False):
        if mode == "vol_pharm":
            rs = K.self_overlap(rc, wl["alpha"]); fs = K.self_overlap(fc, wl["alpha"])
            rsp = K.pharm_self_overlap(rp, True); fsp = K.pharm_self_overlap(fp, True)
        else:
            rs = K.self_overlap(rc, wl["alpha"], esp, kl); fs = K.self_overlap(fc, wl["alpha"], esp, kl)
            rsp = fsp = None
        sq, st = K.seeds(rc, fc, idx, idx, S)
        if record_kernel:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
        amode = {"surf_esp": "esp", "vol": "shape", "vol_pharm": "shape_pharm"}[mode]
        al.align_packed(amode, ref=rc, fit=fc, ref_ph=rp, fit_ph=fp, pair_ref=idx, pair_fit=idx,
                        seed_q=sq, seed_t=st, steps=wl["steps"], lr=wl["lr"], alpha=wl["alpha"],
                        lam=kl, ref_self=rs, fit_self=fs, ref_self_ph=rsp, fit_self_ph=fsp,
                        order=order, rows=rows, out=outb, check_status=False, validate=False,
                        **tile)
        if record_kernel:
            e1.record()
            align_ms.append((e0, e1))
        return outb

    launches_per_step = 5 if mode != "vol_pharm" else 7
    l2 = torch.empty(64 << 20, device=dev)   # 256 MB
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local).start()
    times = []
    for _ in range(args.steps):
        flush_l2(l2)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step(record_kernel=True)
        e1.record()
        times.append((e0, e1))
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in times)
    kern_ms = [a.elapsed_time(b) for a, b in align_ms]
    t_max = torch.tensor([total_ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms_per_step = float(t_max.item()) / args.steps
    value = n_pairs * world / (ms_per_step * 1e-3)
    status = int(al._scratch(dev)[1].item())
    if status:
        raise RuntimeError(f"kernel status flags {status}")

    # ---- end to end through the host-array API ----------------------------------------
    h2d = ref_h.nbytes + fit_h.nbytes + 2 * 4 * n_pairs
    d2h = n_pairs * 8 * 4

    def e2e_call():
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        res = api.align_host(mode, ref_h, fit_h, alpha=wl["alpha"], lam=wl["lam"],
                             num_seeds=S, steps=wl["steps"], lr=wl["lr"], device=dev)
        return res, (time.perf_counter() - t0) * 1e3

    e2e_ms = []
    if args.e2e:
        out, warm_ms = e2e_call()   # warm-up
        for _ in range(e2e_count(warm_ms)):
            out, ms = e2e_call()
            e2e_ms.append(ms)
    e2e_t = torch.tensor([statistics.median(e2e_ms) if e2e_ms else float("nan")], device=dev,
                         dtype=torch.float64)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = n_pairs * world / (float(e2e_t.item()) * 1e-3)
    if e2e_ms:
        assert np.all(np.isfinite(out.scores))

    if rank != 0:
        return None

    # ---- roofline ---------------------------------------------------------------------
    peak = measure_peak(dev)
    kavg = statistics.mean(kern_ms)
    achieved = terms / (kavg * 1e-3)
    # FP32 operations per pair-term of the fused kernel (factored exponent): shape 7, ESP 8
    per_term_fp32 = {"surf_esp": 8, "vol": 7, "vol_pharm": 7}[mode]
    roof = min(peak["ex2"], peak["ffma"] / per_term_fp32)

    line = {
        "metric": metric_of(wl),
        "value": round(value, 2), "unit": "aligned pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["desc"], "mode": mode, "pairs_per_gpu": n_pairs,
                   "starts": S, "adam_steps": wl["steps"], "lr": wl["lr"],
                   "alpha": wl["alpha"], "lam": wl["lam"],
                   "l2": "flushed between timed steps (256 MB write outside timed windows)",
                   "parallelism": f"dp{world} (independent pair shards, no collective)",
                   "tile": dict(al.LAST_TILE)},
        "e2e": {"value": round(e2e_value, 2), "unit": "aligned pairs/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "api": "fast_shepherd_score_b200.api.align_host (pinned host arrays)"},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "mufu", "achieved": round(achieved / 1e9, 1),
                     "peak": round(roof / 1e9, 1), "unit": "Gterm/s",
                     "frac": round(achieved / roof, 4),
                     "traffic": (round(DRAM_BYTES_PER_PAIR[mode] * n_pairs)
                                 if mode in DRAM_BYTES_PER_PAIR else None),
                     "traffic_source": "bytes per launch: ncu dram__bytes_read+write of the "
                                       "256-pair case, scaled by pairs",
                     "peak_source": "measured by fss_probe_peak on this GPU: "
                                    f"ex2 {peak['ex2'] / 1e9:.0f} G/s, ffma "
                                    f"{peak['ffma'] / 1e9:.0f} G/s /{per_term_fp32} per term",
                     "terms_per_launch": terms, "kernel_ms": round(kavg, 3),
                     "hbm": hbm_side(DRAM_BYTES_PER_PAIR[mode] * n_pairs
                                     if mode in DRAM_BYTES_PER_PAIR else None, kavg)},
        "clocks": clk,
    }
    if args.cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(wl, raw, budget_s=args.cpu_seconds)
    if args.comparators and world == 1:
        line["comparators"] = comparators(wl, raw, dev)
        plain = (line["comparators"] or {}).get("plain_one_pair_per_launch")
        if plain:
            line["comparators"]["batched_over_plain"] = round(value / plain["value"], 1)
    if args.server and world == 1:
        line["server"] = server_bench(dev, duration=args.server_seconds,
                                      launch_pairs=args.server_launch_pairs,
                                      policy=args.server_policy)
    return line


def _pad(clouds, fill=0.0, dtype=np.float32):
    n = np.array([len(c) for c in clouds])
    out = np.full((len(clouds), max(int(n.max()), 1)) + np.asarray(clouds[0]).shape[1:], fill,
                  dtype)
    for i, c in enumerate(clouds):
        out[i, :len(c)] = c
    return out, n


def cpu_align_sample(wl, raw, k, nthreads=None):
    """Run the oracle on the first k pairs; returns (seconds, pairs)."""
    from oracle import align as oa
    refs, fits = raw
    t0 = time.perf_counter()
    if wl["mode"] == "vol_and_surf_esp":
        pads = []
        for key in ("centers", "atoms", "charges", "radii", "surf", "surf_esp"):
            for ms in (refs, fits):
                pads.append(_pad([m[key] for m in ms[:k]]))
        (C1, CN), (C2, CM), (A1, AN), (A2, AM), (Q1, _), (Q2, _), (R1, _), (R2, _), \
            (S1, SN), (S2, SM), (P1, _), (P2, _) = pads
        oa.align_esp_combo(C1, C2, CN, CM, A1, A2, Q1, Q2, R1, R2, AN, AM, S1, S2, P1, P2, SN, SM,
                           alpha=wl["alpha"], lam=wl["lam"], num_seeds=wl["starts"],
                           steps=wl["steps"], lr=wl["lr"], stride=1, nthreads=nthreads)
    elif wl["mode"] == "surf_esp":
        A, N = _pad([p for p, _ in refs[:k]]); B, M = _pad([p for p, _ in fits[:k]])
        CA, _ = _pad([c for _, c in refs[:k]]); CB, _ = _pad([c for _, c in fits[:k]])
        oa.align_esp(A, B, CA, CB, N, M, alpha=wl["alpha"], lam=oa.LAM_SCALING * wl["lam"],
                     num_seeds=wl["starts"], steps=wl["steps"], lr=wl["lr"], nthreads=nthreads)
    elif wl["mode"] == "vol":
        A, N = _pad(refs[:k]); B, M = _pad(fits[:k])
        oa.align_shape(A, B, N, M, alpha=wl["alpha"], num_seeds=wl["starts"], steps=wl["steps"],
                       lr=wl["lr"], nthreads=nthreads)
    else:
        g = lambda ms, key: [m[key] for m in ms[:k]]
        A, N = _pad(g(refs, "atom_pos")); B, M = _pad(g(fits, "atom_pos"))
        PA, PN = _pad(g(refs, "pharm_ancs")); PB, PM = _pad(g(fits, "pharm_ancs"))
        RV, _ = _pad(g(refs, "pharm_vecs")); FV, _ = _pad(g(fits, "pharm_vecs"))
        At, _ = _pad(g(refs, "pharm_types"), 8, np.int64); Bt, _ = _pad(g(fits, "pharm_types"), 8, np.int64)
        oa.align_combo(A, B, N, M, PA, PB, RV, FV, At, Bt, PN, PM, alpha=wl["alpha"], w=0.5,
                       num_seeds=wl["starts"], steps=wl["steps"], lr=wl["lr"], nthreads=nthreads)
    return time.perf_counter() - t0, k


def cpu_baseline(wl, raw, budget_s=15.0):
    """The CPU oracle on a bounded sample of the workload, all host threads."""
    from oracle import _lib as ol
    ol.build()
    cores = ol.max_threads()
    dt, k = cpu_align_sample(wl, raw, max(1, min(cores, 8)))
    per_pair = dt / k
    k2 = int(max(k, min(len(raw[0]), budget_s / max(per_pair, 1e-6))))
    k2 = max(cores, (k2 // cores) * cores) if k2 >= cores else k2
    k2 = min(k2, len(raw[0]))
    dt, k2 = cpu_align_sample(wl, raw, k2)
    return {"value": round(k2 / dt, 3), "unit": "aligned pairs/s", "cores": cores,
            "kind": "port",
            "sample": f"first {k2} pairs of the same workload ({dt:.1f} s, all {cores} host "
                      "threads, C oracle restating the reference numba fine loop)"}


def comparators(wl, raw, dev, n_plain=16, n_graph=256):
    """Plain one-pair-per-launch and per-step CUDA-graph forms on subsets (pairs/s)."""
    import torch
    from fast_shepherd_score_b200 import align as al, kernels as K
    from fast_shepherd_score_b200.api import _kernel_lam
    if wl["mode"] not in ("surf_esp", "vol"):
        return None
    refs, fits = raw
    esp = wl["mode"] == "surf_esp"
    S, steps = wl["starts"], wl["steps"]
    kl = _kernel_lam(wl["mode"], wl["lam"]) if esp else None
    def padded(k):
        if esp:
            A, N = _pad([p for p, _ in refs[:k]]); B, M = _pad([p for p, _ in fits[:k]])
            CA, _ = _pad([c for _, c in refs[:k]]); CB, _ = _pad([c for _, c in fits[:k]])
        else:
            A, N = _pad(refs[:k]); B, M = _pad(fits[:k]); CA = CB = None
        t = lambda a: None if a is None else torch.as_tensor(a, device=dev)
        return t(A), t(B), t(CA), t(CB), t(N), t(M)
    out = {}
    # plain: one pair at a time, two launches per Adam step
    A, B, CA, CB, N, M = padded(n_plain)
    VAA = (K._batch_self_overlap_esp(A, CA, N, wl["alpha"], kl) if esp
           else K._batch_self_overlap(A, N, wl["alpha"]))
    VBB = (K._batch_self_overlap_esp(B, CB, M, wl["alpha"], kl) if esp
           else K._batch_self_overlap(B, M, wl["alpha"]))
    from fast_shepherd_score_b200.layout import CloudSet
    idx = torch.arange(n_plain, dtype=torch.int32, device=dev)
    sq, st = K.seeds(CloudSet.from_padded(A, N, CA), CloudSet.from_padded(B, M, CB), idx, idx, S)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for i in range(n_plain):
        n, m = int(N[i]), int(M[i])
        al.align_one_pair_per_launch(A[i, :n], B[i, :m], n, m, float(VAA[i] + VBB[i]), sq[i],
                                     st[i], steps=steps, alpha=wl["alpha"], lr=wl["lr"],
                                     CA=None if CA is None else CA[i, :n],
                                     CB=None if CB is None else CB[i, :m], lam=kl)
    torch.cuda.synchronize(dev)
    dt = time.perf_counter() - t0
    out["plain_one_pair_per_launch"] = {"value": round(n_plain / dt, 3), "unit": "aligned pairs/s",
                                        "pairs": n_plain, "launches_per_pair": 2 * steps}
    # per-step CUDA graph over a batch (reference _graphed.py structure)
    A, B, CA, CB, N, M = padded(n_graph)
    idx = torch.arange(n_graph, dtype=torch.int32, device=dev)
    sq, st = K.seeds(CloudSet.from_padded(A, N, CA), CloudSet.from_padded(B, M, CB), idx, idx, S)
    VAA = (K._batch_self_overlap_esp(A, CA, N, wl["alpha"], kl) if esp
           else K._batch_self_overlap(A, N, wl["alpha"]))
    VBB = (K._batch_self_overlap_esp(B, CB, M, wl["alpha"], kl) if esp
           else K._batch_self_overlap(B, M, wl["alpha"]))
    rep = lambda x: None if x is None else x.repeat_interleave(S, 0)
    loop = al.GraphedFineLoop(rep(A), rep(B), rep(N), rep(M), rep(VAA + VBB), sq.reshape(-1, 4),
                              st.reshape(-1, 3), alpha=wl["alpha"], lr=wl["lr"], CA_k=rep(CA),
                              CB_k=rep(CB), lam=kl).capture()
    loop.run(2)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    loop.run(steps)
    e1.record()
    torch.cuda.synchronize(dev)
    dt = e0.elapsed_time(e1) * 1e-3
    out["graph_per_step"] = {"value": round(n_graph / dt, 2), "unit": "aligned pairs/s",
                             "pairs": n_graph, "launches_per_step": 2}
    return out


def server_bench(dev, duration=20.0, n_lib=1_000_000, load=0.6, seed=7, launch_pairs=8192,
                 policy="srpt"):
    """Screening server under a Poisson request stream (bounded run, rank 0).

    1M-molecule device-resident library (15-60 atoms + 3-20 pharmacophores), shape +
    directional pharmacophore scoring, 20 starts x 100 Adam steps, request sizes log-uniform
    in [1e3, 1e5] library molecules, offered load = `load` x the measured capacity; at most
    ``launch_pairs`` pairs per fused launch, admission ``policy`` ("srpt" or "fifo")."""
    import torch
    from fast_shepherd_score_b200 import align as al, kernels as K, synthetic as syn
    from fast_shepherd_score_b200.server import ScreenServer, latency_by_decade, slowdown
    t0 = time.perf_counter()
    atoms, ph = syn.library_on_device(n_lib, seed, dev)
    torch.cuda.synchronize(dev)
    gen_s = time.perf_counter() - t0
    rng = np.random.default_rng(seed)
    pool = []
    for i in rng.choice(n_lib, 64, replace=False):
        a0, a1 = int(atoms.off[i]), int(atoms.off[i + 1])
        p0, p1 = int(ph.off[i]), int(ph.off[i + 1])
        anc = ph.anc[p0:p1].cpu()
        pool.append({"atom_pos": atoms.pts[a0:a1, :3].cpu().numpy(),
                     "pharm_types": anc[:, 3].contiguous().view(torch.int32).numpy(),
                     "pharm_ancs": anc[:, :3].numpy(), "pharm_vecs": ph.vec[p0:p1, :3].cpu().numpy()})
    # tile choice for this library (autotuned once on a representative launch)
    from fast_shepherd_score_b200.layout import CloudSet, PharmSet
    q0 = pool[0]
    qset = CloudSet.from_arrays([q0["atom_pos"]], device=dev)
    qph = PharmSet.from_arrays([q0["pharm_types"]], [q0["pharm_ancs"]], [q0["pharm_vecs"]], device=dev)
    P = 65536
    pr = torch.zeros(P, dtype=torch.int32, device=dev)
    pf = torch.as_tensor(rng.choice(n_lib, P, replace=False).astype(np.int32), device=dev)
    sq, st = K.seeds(qset, atoms, pr, pf, 20)
    al.align_packed("shape_pharm", ref=qset, fit=atoms, ref_ph=qph, fit_ph=ph, pair_ref=pr,
                    pair_fit=pf, seed_q=sq, seed_t=st, steps=100, lr=0.1)
    lpp = al.LAST_TILE.get("lanes_per_pose") or 8
    tile = {k: al.LAST_TILE[k] for k in ("chunks", "cta_per_sm", "kernel_variant")
            if k in al.LAST_TILE}
    # library bytes a pair reads from HBM: the molecule's packed atoms + pharmacophores
    mol_bytes = (atoms.pts.nbytes + ph.anc.nbytes + ph.vec.nbytes) / n_lib
    with ScreenServer((atoms, ph), mode="vol_pharm", starts=20, steps=100, lanes_per_pose=lpp,
                      max_pairs_per_launch=launch_pairs, tile=tile, policy=policy) as srv:
        # capacity: after one warm-up request (first launches load kernels and grow the
        # pinned-buffer cache), two large requests in flight together
        srv.submit(pool[1], rng.choice(n_lib, 65536, replace=False), top_k=100).result()
        t1 = time.perf_counter()
        big = [srv.submit(pool[k], rng.choice(n_lib, 131072, replace=False), top_k=100)
               for k in (0, 2)]
        for f in big:
            f.result()
        cap = 2 * 131072 / (time.perf_counter() - t1)
        n_probe = 65536 + 2 * 131072
        mean_req = (1e5 - 1e3) / math.log(1e5 / 1e3)
        rate = load * cap / mean_req
        futs = []
        t_start = time.perf_counter()
        nxt = t_start
        while nxt - t_start < duration:
            now = time.perf_counter()
            if now < nxt:
                time.sleep(nxt - now)
            n = int(round(math.exp(rng.uniform(math.log(1e3), math.log(1e5)))))
            futs.append(srv.submit(pool[int(rng.integers(len(pool)))],
                                   rng.choice(n_lib, n, replace=False), top_k=100))
            nxt += rng.exponential(1.0 / rate)
        for f in futs:
            f.result()
        wall = time.perf_counter() - t_start
        lat = np.array(srv.latencies[3:]) * 1e3      # drop the warm-up and capacity probes
        by_size = latency_by_decade(srv.size_latency[3:])
        slow = slowdown(srv.size_latency[3:], cap)
        st = srv.stats()
    return {"library": n_lib, "mode": "vol_pharm (shape + directional pharmacophore)",
            "starts": 20, "adam_steps": 100, "request_pairs": "log-uniform [1e3, 1e5]",
            "capacity_pairs_per_s": round(cap, 1),
            "offered_load": {"requests_per_s": round(rate, 3), "fraction_of_capacity": load},
            "requests": int(len(lat)), "duration_s": round(wall, 2),
            "pairs_per_s": round((st["pairs_done"] - n_probe) / wall, 1),
            "p50_ms": round(float(np.percentile(lat, 50)), 2),
            "p99_ms": round(float(np.percentile(lat, 99)), 2),
            "by_request_size": by_size, "slowdown": slow,
            "policy": policy, "max_pairs_per_launch": launch_pairs,
            "max_queue_depth": st["max_queue_depth"], "tile": dict(tile, lanes_per_pose=lpp),
            "library_bytes_per_molecule": round(mol_bytes, 1),
            "library_hbm_gbs_at_capacity": round(cap * mol_bytes / 1e9, 3),
            "library_build_s": round(gen_s, 1)}


def _score_grad_inputs(nq, seed, n_atoms=60, n_surf=300, nt=4):
    from fast_shepherd_score_b200 import synthetic as syn
    rng = np.random.default_rng(seed)
    atoms = syn.ball_clouds(rng, [n_atoms] * (nq + nt))
    surf = syn.sphere_clouds(rng, [n_surf] * (nq + nt))
    A = np.stack(atoms).astype(np.float32)
    S = np.stack([p for p, _ in surf]).astype(np.float32)
    Q = np.stack([c for _, c in surf]).astype(np.float32)
    tgt = np.arange(nq) % nt
    return A, S, Q, tgt


def run_score_grad(args, wl):
    """Differentiable scoring: one step = forward (vol + surface ESP Tanimoto of every query
    against its target) and backward (d score / d coordinates and charges) through
    fast_shepherd_score_b200.autograd.  Work units: pair-terms of the forward and the adjoint
    (each one MUFU ex2)."""
    import torch
    import torch.distributed as dist
    from fast_shepherd_score_b200 import autograd as AG
    world, rank, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    nq = args.pairs or wl["pairs"]
    A, S, Q, tgt = _score_grad_inputs(nq, 1 + rank)
    terms = int(2 * nq * (A.shape[1] ** 2 + S.shape[1] ** 2))
    surf_alpha, lam = 1.216, wl["lam"] * AG.LAM_SCALING

    def step(qa, qs, qc, ta, ts, tc):
        qa.grad = qs.grad = qc.grad = None
        vol = AG.get_overlap(ta, qa, alpha=wl["alpha"])
        esp = AG.get_overlap_esp(ts, qs, tc, qc, alpha=surf_alpha, lam=lam)
        (vol.sum() + esp.sum()).backward()
        return vol, esp

    Ad, Sd, Qd = (torch.from_numpy(x).to(dev) for x in (A, S, Q))
    ti = torch.from_numpy(tgt).to(dev)
    ta, ts, tc = Ad[nq:][ti], Sd[nq:][ti], Qd[nq:][ti]
    qa, qs, qc = (x[:nq].clone().requires_grad_(True) for x in (Ad, Sd, Qd))
    l2 = torch.empty(64 << 20, device=dev)
    # the same step captured once as a CUDA graph (fixed shapes and buffers, the way a loop
    # over fixed-size batches runs it): every replay launches the same 4 kernels on the same
    # inputs, without the per-call Python/autograd host work of the eager form
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    # the leaves live on the default stream; their gradient accumulation on the capture
    # stream is ordered by the capture itself
    warnings.filterwarnings("ignore", message="The AccumulateGrad node's stream")
    with torch.cuda.stream(side):
        for _ in range(max(3, args.warmup)):
            step(qa, qs, qc, ta, ts, tc)
    torch.cuda.current_stream(dev).wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        static_out = step(qa, qs, qc, ta, ts, tc)
    static_out += (qa.grad, qs.grad, qc.grad)   # the graph's outputs stay referenced

    def timed(run):
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        times = []
        for _ in range(args.steps):
            flush_l2(l2)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run()
            e1.record()
            times.append((e0, e1))
        torch.cuda.synchronize(dev)
        t = torch.tensor([sum(a.elapsed_time(b) for a, b in times)], device=dev,
                         dtype=torch.float64)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()) / args.steps

    clocks = ClockSampler(local).start()   # spans both timed loops (each is short)
    eager_ms = timed(lambda: step(qa, qs, qc, ta, ts, tc))
    ms_per_step = timed(graph.replay)
    clk = clocks.stop()
    value = nq * world / (ms_per_step * 1e-3)

    # end to end: pinned host queries -> device -> scores + gradients back on the host
    hq = [torch.from_numpy(x[:nq]).pin_memory() for x in (A, S, Q)]
    # pinned result buffers: scores and the three gradients come back asynchronously
    ho = [torch.empty(nq).pin_memory(), torch.empty(nq).pin_memory()] + \
        [torch.empty_like(x).pin_memory() for x in hq]
    e2e_ms = []
    # a step is ~1 ms end to end: the median of 20 (after one warm-up) steadies the host jitter
    for i in range(21 if args.e2e else 0):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        a, s_, c = (x.to(dev, non_blocking=True).requires_grad_(True) for x in hq)
        vol, esp = step(a, s_, c, ta, ts, tc)
        for h, d in zip(ho, (vol.detach(), esp.detach(), a.grad, s_.grad, c.grad)):
            h.copy_(d, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        t1 = time.perf_counter()
        if i:
            e2e_ms.append((t1 - t0) * 1e3)
    e2e_t = torch.tensor([statistics.median(e2e_ms) if e2e_ms else float("nan")], device=dev,
                         dtype=torch.float64)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    if rank != 0:
        return None
    peak = measure_peak(dev)
    achieved = terms / (ms_per_step * 1e-3)
    h2d = sum(x.nbytes for x in hq)
    d2h = nq * 4 * 2 + h2d
    line = {
        "metric": metric_of(wl),
        "value": round(value, 2), "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": wl["desc"], "mode": "score_grad", "queries_per_gpu": nq,
                   "l2": "flushed between timed steps (256 MB write outside timed windows)",
                   "parallelism": f"dp{world} (independent query shards, no collective)",
                   "timing": "value: the fwd + backward step captured once as a CUDA graph "
                             "and replayed (same kernels and inputs every step); eager: the "
                             "same step through eager torch autograd; e2e: eager"},
        "eager": {"value": round(nq * world / (eager_ms * 1e-3), 2), "unit": "queries/s",
                  "ms_per_step": round(eager_ms, 3)},
        "e2e": {"value": round(nq * world / (float(e2e_t.item()) * 1e-3), 2), "unit": "queries/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "api": "fast_shepherd_score_b200.autograd.get_overlap / get_overlap_esp"},
        "gpu_launches": 4 * args.steps,
        "roofline": {"bound": "mufu", "achieved": round(achieved / 1e9, 1),
                     "peak": round(peak["ex2"] / 1e9, 1), "unit": "Gterm/s",
                     "frac": round(achieved / peak["ex2"], 4), "traffic": None,
                     "peak_source": "measured ex2 rate; step time includes the loss sums and "
                                    "the gradient buffers' zeroing",
                     "terms_per_step": terms},
        "clocks": clk,
    }
    if args.cpu_baseline and world == 1:
        from oracle import scores as osc
        k, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < min(args.cpu_seconds, 10.0) and k < nq:
            i = nq + int(tgt[k])
            osc.shape_tanimoto_grad(A[i], A[k], wl["alpha"])
            osc.esp_tanimoto_grad(S[i], S[k], Q[i], Q[k], surf_alpha, lam)
            k += 1
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(k / dt, 3), "unit": "queries/s", "cores": 1,
                                "kind": "port",
                                "sample": f"{k} queries (fp64 numpy restatement of the "
                                          "reference's torch scoring and its gradients, one "
                                          "thread)"}
    return line


def run_esp_combo(args, wl):
    """vol_and_surf_esp: device-resident step (self overlaps + seeds + fused kernel + pick) and
    an end-to-end leg from pinned host arrays (H2D of every cloud, align, D2H of the results).
    Work units: shape terms S*T*N_c*M_c plus ESP-comparison pairs S*T*(N_s*M_a + M_s*N_a)
    (each one MUFU rsqrt or ex2)."""
    import torch
    import torch.distributed as dist
    from fast_shepherd_score_b200 import align as al, kernels as K
    from fast_shepherd_score_b200.layout import CloudSet
    world, rank, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n_pairs = args.pairs or wl["pairs"]
    _, _, raw = make_inputs(wl, n_pairs, seed=1 + rank)
    refs, fits = raw
    S, T = wl["starts"], wl["steps"]
    cnt = lambda ms, k: np.array([len(m[k]) for m in ms], np.int64)
    terms = int(S * T * ((cnt(refs, "centers") * cnt(fits, "centers")).sum() +
                         (cnt(refs, "surf") * cnt(fits, "atoms")).sum() +
                         (cnt(fits, "surf") * cnt(refs, "atoms")).sum()))

    def sets(ms):
        g = lambda k: [m[k] for m in ms]
        c = CloudSet.from_arrays(g("centers"), device=dev)
        a = CloudSet.from_arrays(g("atoms"), g("charges"), device=dev)
        r = torch.from_numpy(np.concatenate(g("radii")).astype(np.float32)).to(dev)
        sf = CloudSet.from_arrays(g("surf"), g("surf_esp"), device=dev)
        return c, a, r, sf

    def host_sets(ms):
        """One side's four sets packed into pinned host memory (before any timed region)."""
        g = lambda k: [m[k] for m in ms]

        def packed(pts, vals=None):
            cs = CloudSet.from_arrays(pts, vals, device="cpu")
            return cs.pts.pin_memory(), cs.off.pin_memory(), cs.counts, cs.max_points
        radii = torch.from_numpy(np.concatenate(g("radii")).astype(np.float32)).pin_memory()
        return (packed(g("centers")), packed(g("atoms"), g("charges")), radii,
                packed(g("surf"), g("surf_esp")))

    def to_dev(h):
        """H2D of one side's pinned sets (asynchronous copies on the current stream)."""
        mk = lambda p, o, c, m: CloudSet(p.to(dev, non_blocking=True),
                                         o.to(dev, non_blocking=True), c, m)
        c, a, r, sf = h
        return mk(*c), mk(*a), r.to(dev, non_blocking=True), mk(*sf)

    rc, ra, rr, rs = sets(refs)
    fc, fa, fr, fs = sets(fits)
    host_r, host_f = (host_sets(refs), host_sets(fits)) if args.e2e else (None, None)
    idx = torch.arange(n_pairs, dtype=torch.int32, device=dev)
    tile = {}
    if args.tile:
        v = [int(x) for x in args.tile.split(",")]
        tile = dict(zip(("lanes_per_pose", "chunks", "cta_per_sm", "accumulate",
                             "kernel_variant"), v))
    kern = []

    def step(c1, c2, a1, a2, r1, r2, s1, s2, record=False):
        vs = K.self_overlap(c1, wl["alpha"]); vf = K.self_overlap(c2, wl["alpha"])
        sq, st = K.seeds(c1, c2, idx, idx, S)
        if record:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
        out = al.align_packed("esp_combo", ref=c1, fit=c2, pair_ref=idx, pair_fit=idx,
                              seed_q=sq, seed_t=st, steps=T, lr=wl["lr"], alpha=wl["alpha"],
                              lam=wl["lam"], ref_self=vs, fit_self=vf, ref_atoms=a1,
                              fit_atoms=a2, ref_radii=r1, fit_radii=r2, ref_surf=s1,
                              fit_surf=s2, esp_stride=1, check_status=False, validate=False,
                              **tile)
        if record:
            e1.record()
            kern.append((e0, e1))
        return out

    args_dev = (rc, fc, ra, fa, rr, fr, rs, fs)
    l2 = torch.empty(64 << 20, device=dev)
    for _ in range(args.warmup):
        step(*args_dev)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local).start()
    times = []
    for _ in range(args.steps):
        flush_l2(l2)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step(*args_dev, record=True)
        e1.record()
        times.append((e0, e1))
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    t_max = torch.tensor([sum(a.elapsed_time(b) for a, b in times)], device=dev,
                         dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms_per_step = float(t_max.item()) / args.steps
    value = n_pairs * world / (ms_per_step * 1e-3)

    # end to end: pinned host arrays -> device sets -> align -> scores/poses on the host
    e2e_ms, h2d = [], 0

    def e2e_call():
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        r4 = to_dev(host_r)
        f4 = to_dev(host_f)
        sc, q, t = step(r4[0], f4[0], r4[1], f4[1], r4[2], f4[2], r4[3], f4[3])
        torch.cat([sc[:, None], q, t], 1).cpu()
        ms = (time.perf_counter() - t0) * 1e3
        nb = sum(x.pts.nbytes + x.off.nbytes
                 for x in (r4[0], r4[1], r4[3], f4[0], f4[1], f4[3])) + \
            r4[2].nbytes + f4[2].nbytes
        return nb, ms

    if args.e2e:
        h2d, warm_ms = e2e_call()   # warm-up
        for _ in range(e2e_count(warm_ms)):
            h2d, ms = e2e_call()
            e2e_ms.append(ms)
    e2e_t = torch.tensor([statistics.median(e2e_ms) if e2e_ms else float("nan")], device=dev,
                         dtype=torch.float64)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    if rank != 0:
        return None
    peak = measure_peak(dev)
    kavg = statistics.mean(a.elapsed_time(b) for a, b in kern)
    achieved = terms / (kavg * 1e-3)
    line = {
        "metric": metric_of(wl),
        "value": round(value, 2), "unit": "aligned pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["desc"], "mode": wl["mode"], "pairs_per_gpu": n_pairs,
                   "starts": S, "adam_steps": T, "lr": wl["lr"], "alpha": wl["alpha"],
                   "lam": wl["lam"], "esp_stride": 1,
                   "l2": "flushed between timed steps (256 MB write outside timed windows)",
                   "parallelism": f"dp{world} (independent pair shards, no collective)",
                   "tile": dict(al.LAST_TILE)},
        "e2e": {"value": round(n_pairs * world / (float(e2e_t.item()) * 1e-3), 2),
                "unit": "aligned pairs/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": n_pairs * 8 * 4,
                "api": "fast_shepherd_score_b200.align.align_packed from pinned host arrays"},
        "gpu_launches": 5 * args.steps,
        "roofline": {"bound": "mufu", "achieved": round(achieved / 1e9, 1),
                     "peak": round(peak["ex2"] / 1e9, 1), "unit": "Gterm/s",
                     "frac": round(achieved / peak["ex2"], 4), "traffic": None,
                     "peak_source": "measured ex2 rate (one MUFU op per shape term and per "
                                    "ESP-comparison pair)",
                     "terms_per_launch": terms, "kernel_ms": round(kavg, 3)},
        "clocks": clk,
    }
    if args.cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(wl, raw, budget_s=args.cpu_seconds)
    return line


def _reference_score_grad(args, wl, world):
    """CPU arm of the differentiable-scoring workload: the fp64 numpy restatement of the
    reference's torch scores and gradients, one thread, bounded sample per step."""
    from fast_shepherd_score_b200.autograd import LAM_SCALING
    from oracle import scores as osc
    nq = args.pairs or wl["pairs"]
    A, S, Q, tgt = _score_grad_inputs(nq, 1)
    budget = max(0.5, args.cpu_seconds / max(1, args.steps + args.warmup))
    rates = []
    for it in range(args.warmup + args.steps):
        k, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget and k < nq:
            i = nq + int(tgt[k])
            osc.shape_tanimoto_grad(A[i], A[k], wl["alpha"])
            osc.esp_tanimoto_grad(S[i], S[k], Q[i], Q[k], 1.216, wl["lam"] * LAM_SCALING)
            k += 1
        if it >= args.warmup:
            rates.append(k / (time.perf_counter() - t0))
    value = statistics.median(rates)
    line = {"impl": "reference", "metric": metric_of(wl),
            "value": round(value, 3), "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * nq / value, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": wl["desc"], "mode": "score_grad"},
            "cpu_baseline": {"value": round(value, 3), "unit": "queries/s", "cores": 1,
                             "kind": "port", "sample": f"{budget:.1f} s of queries per step"},
            "e2e": {"value": round(value, 3), "unit": "queries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    return line


def run_reference(args, wl):
    """The CPU implementation of the path (oracle port of the reference numba path)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    if wl["mode"] == "score_grad":
        return _reference_score_grad(args, wl, world)
    from oracle import _lib as ol
    ol.build()
    cores = ol.max_threads()
    n_pairs = args.pairs or wl["pairs"]
    _, _, raw = make_inputs(wl, n_pairs, seed=1)
    # calibrate a sample so that warm-up + steps stay within a few minutes
    dt, k = cpu_align_sample(wl, raw, max(1, min(cores, 8)))
    per_pair = dt / k
    k = int(max(1, min(n_pairs, args.cpu_seconds / max(per_pair, 1e-6))))
    for _ in range(args.warmup if per_pair * k * args.warmup < 60 else 0):
        cpu_align_sample(wl, raw, max(1, min(k, cores)))
    times = []
    for _ in range(args.steps):
        dt, kk = cpu_align_sample(wl, raw, k)
        times.append(dt)
    ms = statistics.median(times) * 1e3
    value = k / (ms * 1e-3)
    line = {"impl": "reference",
            "metric": metric_of(wl),
            "value": round(value, 3), "unit": "aligned pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": wl["desc"], "mode": wl["mode"], "sample_pairs_per_step": k},
            "cpu_baseline": {"value": round(value, 3), "unit": "aligned pairs/s", "cores": cores,
                             "kind": "port",
                             "sample": f"{k} pairs of the workload per step on all {cores} "
                                       "host threads (C oracle restating the reference numba "
                                       "fine loop; the reference itself is Python and is not "
                                       "present on the GPU box)"},
            "e2e": {"value": round(value, 3), "unit": "aligned pairs/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


# The other workloads, measured in the same run and reported under the line's "configs" key
# (one GPU only): each with its own value, kernel time, algorithmic work and roofline fraction.
CONFIG_WORKLOADS = ("vol", "vol_pharm", "score_grad", "vol_and_surf_esp")


def run_workload(args, wl):
    if wl["mode"] == "vol_and_surf_esp":
        return run_esp_combo(args, wl)
    if wl["mode"] == "score_grad":
        return run_score_grad(args, wl)
    return run_cuda(args, wl)


def other_configs(args, headline):
    """Short runs of the other workloads (warm-up 3, at most 5 timed steps, no CPU legs)."""
    sub = argparse.Namespace(**vars(args))
    sub.steps, sub.warmup = max(3, min(args.steps, 5)), 3
    sub.pairs, sub.tile = 0, ""
    sub.cpu_baseline = sub.comparators = sub.server = False
    out = {}
    for name in CONFIG_WORKLOADS:
        if name == headline:
            continue
        line = run_workload(sub, WORKLOADS[name])
        roof = line["roofline"]
        rec = {"workload": line["config"]["workload"], "metric": line["metric"],
               "value": line["value"], "unit": line["unit"], "steps": sub.steps,
               "warmup": sub.warmup, "ms_per_step": line["ms_per_step"],
               "e2e": line["e2e"]["value"],
               "kernel_ms": roof.get("kernel_ms"),
               "terms_per_launch": roof.get("terms_per_launch", roof.get("terms_per_step")),
               "roofline": {k: roof[k] for k in ("achieved", "peak", "unit", "frac")},
               "clocks": {k: line["clocks"].get(k) for k in ("sm_mhz", "reasons")}}
        if "tile" in line["config"]:
            rec["tile"] = line["config"]["tile"]
        if "eager" in line:
            rec["eager"] = line["eager"]["value"]
        out[name] = rec
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--workload", default="surf_esp", choices=list(WORKLOADS))
    ap.add_argument("--pairs", type=int, default=0, help="override pairs per GPU")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-comparators", dest="comparators", action="store_false")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false",
                    help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-server", dest="server", action="store_false",
                    help="skip the screening-server leg (Poisson stream, p50/p99)")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="skip the short runs of the other workloads (the 'configs' key)")
    ap.add_argument("--server-seconds", type=float, default=20.0)
    ap.add_argument("--server-launch-pairs", type=int, default=8192,
                    help="largest fused launch of the screening server (pairs)")
    ap.add_argument("--server-policy", default="srpt", choices=["srpt", "fifo"])
    ap.add_argument("--tile", default="", help="fixed tiling instead of the autotuner: "
                    "lanes_per_pose,chunks,cta_per_sm,accumulate[,kernel_variant] (e.g. 32,0,0,2 or "
                    "16,7,0,0,4)")
    ap.add_argument("--server-only", action="store_true",
                    help="run only the screening-server leg on one GPU and print its JSON "
                         "(library-streaming profiles)")
    args = ap.parse_args(argv)
    wl = WORKLOADS[args.workload]
    if args.server_only:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"server": server_bench(dev, duration=args.server_seconds,
                                                 launch_pairs=args.server_launch_pairs,
                                                 policy=args.server_policy)}), flush=True)
        return None
    if args.impl == "reference":
        line = run_reference(args, wl)
        if line is not None:
            print(json.dumps(line), flush=True)
        return line
    world, rank, local = dist_env()
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        # this rank's GPU before the process group exists, so NCCL binds its communicator
        # (and every barrier) to it
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    try:
        line = run_workload(args, wl)
        if line is not None and args.configs and world == 1:
            line["configs"] = other_configs(args, args.workload)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
    return line


if __name__ == "__main__":
    main()
