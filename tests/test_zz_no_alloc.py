"""The allocation-free alignment entry point (fss_align_static) against fss_align.

fss_align_static exists for callers that cannot allocate device memory where they align
(for example a host runtime that passes only input and output buffers, or code inside
another framework's memory pool): its scratch is a library-owned static device array.
These tests call it through the C ABI and check it against fss_align on the same inputs,
with the same tiling (so the kernels do identical arithmetic): twice in a row (the second
call reuses the array the first left behind), then a different, smaller problem (rows the
first call left beyond it must not leak in), a pair larger than the declared extents (its
score comes back NaN and the optional status word reports it), the ESP mode, and the
rejection of a batch larger than the array.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-6   # same kernel, same tile: results agree to rounding of identical arithmetic


def _problem(dev, n=24, seed=77, starts=12, esp=False):
    from fast_shepherd_score_b200 import align as al
    from fast_shepherd_score_b200 import kernels as K
    from fast_shepherd_score_b200 import synthetic as syn
    from fast_shepherd_score_b200.layout import CloudSet
    if esp:
        refs, fits = syn.esp_surface_pairs(n, seed=seed, lo=40, hi=90)
        ref = CloudSet.from_arrays([p for p, _ in refs], [c for _, c in refs], device=dev)
        fit = CloudSet.from_arrays([p for p, _ in fits], [c for _, c in fits], device=dev)
        lam = al.LAM_SCALING * 0.3
        rs, fs = K.self_overlap(ref, 0.81, True, lam), K.self_overlap(fit, 0.81, True, lam)
    else:
        refs, fits = syn.shape_pairs(n, seed=seed)
        ref = CloudSet.from_arrays(refs, device=dev)
        fit = CloudSet.from_arrays(fits, device=dev)
        lam = None
        rs, fs = K.self_overlap(ref, 0.81), K.self_overlap(fit, 0.81)
    idx = torch.arange(n, dtype=torch.int32, device=dev)
    sq, st = K.seeds(ref, fit, idx, idx, starts)
    return dict(ref=ref, fit=fit, idx=idx, sq=sq, st=st, rs=rs, fs=fs, lam=lam)


def _want(pb):
    from fast_shepherd_score_b200 import align as al
    return al.align_packed("esp" if pb["lam"] else "shape", ref=pb["ref"], fit=pb["fit"],
                           pair_ref=pb["idx"], pair_fit=pb["idx"], seed_q=pb["sq"],
                           seed_t=pb["st"], steps=40, lr=0.1, alpha=0.81, lam=pb["lam"],
                           ref_self=pb["rs"], fit_self=pb["fs"], lanes_per_pose=8, chunks=1)


def _static_call(pb, dev, n_pairs=None, max_fit=None, status=None):
    from fast_shepherd_score_b200 import _lib
    from fast_shepherd_score_b200._lib import ptr
    ref, fit, idx = pb["ref"], pb["fit"], pb["idx"]
    P = int(idx.shape[0]) if n_pairs is None else n_pairs
    out = (torch.full((P,), -1.0, device=dev), torch.zeros(P, 4, device=dev),
           torch.zeros(P, 3, device=dev))
    d = _lib.AlignDesc()
    d.mode = _lib.MODE_ESP if pb["lam"] else _lib.MODE_SHAPE
    d.n_pairs, d.n_starts, d.steps = P, int(pb["sq"].shape[1]), 40
    d.pair_ref = d.pair_fit = ptr(idx)
    d.ref_pts, d.ref_off, d.fit_pts, d.fit_off = ptr(ref.pts), ptr(ref.off), ptr(fit.pts), ptr(fit.off)
    d.ref_self, d.fit_self = ptr(pb["rs"]), ptr(pb["fs"])
    d.seed_q, d.seed_t = ptr(pb["sq"]), ptr(pb["st"])
    d.alpha, d.lr = 0.81, 0.1
    d.inv_lam = 1.0 / pb["lam"] if pb["lam"] else 0.0
    d.out_score, d.out_q, d.out_t = ptr(out[0]), ptr(out[1]), ptr(out[2])
    d.max_ref_points = ref.max_points
    d.max_fit_points = fit.max_points if max_fit is None else max_fit
    d.lanes_per_pose, d.chunks, d.cta_per_sm = 8, 1, 0
    d.scratch = ptr(status) if status is not None else None
    rc = _lib.load().fss_align_static(ctypes.byref(d), _lib.stream_ptr(dev))
    return rc, out


def _close(got, want, rows=None):
    for g, w in zip(got, want):
        g, w = g.cpu().numpy(), w.cpu().numpy()
        if rows is not None:
            g, w = g[rows], w[rows]
        np.testing.assert_allclose(g, w, rtol=0, atol=TOL)


def test_static_scratch_matches_fss_align_twice(cuda):
    pb = _problem(cuda)
    want = _want(pb)
    for _ in range(2):
        rc, got = _static_call(pb, cuda)
        assert rc == 0
        torch.cuda.synchronize(cuda)
        _close(got, want)
        assert torch.all(got[0] > 0)


def test_static_scratch_second_problem_and_esp(cuda):
    """A larger problem, then a smaller different one, then an ESP problem: each call's
    results equal fss_align's, whatever the array held before."""
    for pb in (_problem(cuda, n=40, seed=5, starts=16), _problem(cuda, n=9, seed=6, starts=7),
               _problem(cuda, n=16, seed=8, starts=10, esp=True)):
        want = _want(pb)
        rc, got = _static_call(pb, cuda)
        assert rc == 0
        torch.cuda.synchronize(cuda)
        _close(got, want)


def test_static_scratch_oversized_pair_is_nan_and_flagged(cuda):
    """A pair whose fit cloud exceeds the declared max_fit_points is skipped: its score is
    NaN (not a stale row of an earlier call), the others are fss_align's, and the status
    word reports it; a normal call clears the word."""
    pb = _problem(cuda, n=20, seed=11, starts=8)
    want = _want(pb)
    counts = pb["fit"].counts
    big = int(np.argmax(counts))
    limit = int(counts[big]) - 1
    over = counts > limit
    status = torch.full((1,), -1, dtype=torch.int32, device=cuda)
    rc, got = _static_call(pb, cuda, max_fit=limit, status=status)
    assert rc == 0
    torch.cuda.synchronize(cuda)
    sc = got[0].cpu().numpy()
    assert np.all(np.isnan(sc[over])) and np.all(np.isfinite(sc[~over]))
    _close(got, want, rows=~over)
    assert int(status.item()) == 1
    rc, got = _static_call(pb, cuda, status=status)
    assert rc == 0
    torch.cuda.synchronize(cuda)
    assert int(status.item()) == 0
    _close(got, want)


def test_static_scratch_rejects_oversized_batch(cuda):
    from fast_shepherd_score_b200 import _lib
    pb = _problem(cuda)
    big = 131072 // int(pb["sq"].shape[1]) + 1       # n_pairs * n_starts just above the limit
    rc, _ = _static_call(pb, cuda, n_pairs=big)
    assert rc == _lib.FSS_ERR_UNSUPPORTED
    assert b"FSS_STATIC_MAX_ROWS" in _lib.load().fss_last_error()
