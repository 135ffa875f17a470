"""The allocation-free alignment entry point (fss_align_static) against fss_align.

fss_align_static exists for callers that cannot allocate device memory where they align
(for example a host runtime that passes only input and output buffers, or code inside
another framework's memory pool): its scratch is a library-owned static device array.
This test calls it through the C ABI twice in a row -- the second call reuses the array
the first call left behind -- and checks both results against fss_align on the same
inputs, with the same tiling (so the kernels do identical arithmetic), plus the rejection
of a batch larger than the array.  It lives in its own file named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-6   # same kernel, same tile: results agree to rounding of identical arithmetic


def _problem(dev):
    from fast_shepherd_score_b200 import kernels as K
    from fast_shepherd_score_b200 import synthetic as syn
    from fast_shepherd_score_b200.layout import CloudSet
    refs, fits = syn.shape_pairs(24, seed=77)
    ref = CloudSet.from_arrays(refs, device=dev)
    fit = CloudSet.from_arrays(fits, device=dev)
    idx = torch.arange(24, dtype=torch.int32, device=dev)
    sq, st = K.seeds(ref, fit, idx, idx, 12)
    return ref, fit, idx, sq, st, K.self_overlap(ref, 0.81), K.self_overlap(fit, 0.81)


def _static_call(ref, fit, idx, sq, st, rs, fs, dev, n_pairs=None):
    from fast_shepherd_score_b200 import _lib
    from fast_shepherd_score_b200._lib import ptr
    P = int(idx.shape[0]) if n_pairs is None else n_pairs
    out = (torch.full((P,), -1.0, device=dev), torch.zeros(P, 4, device=dev),
           torch.zeros(P, 3, device=dev))
    d = _lib.AlignDesc()
    d.mode, d.n_pairs, d.n_starts, d.steps = _lib.MODE_SHAPE, P, int(sq.shape[1]), 40
    d.pair_ref = d.pair_fit = ptr(idx)
    d.ref_pts, d.ref_off, d.fit_pts, d.fit_off = ptr(ref.pts), ptr(ref.off), ptr(fit.pts), ptr(fit.off)
    d.ref_self, d.fit_self = ptr(rs), ptr(fs)
    d.seed_q, d.seed_t = ptr(sq), ptr(st)
    d.alpha, d.lr = 0.81, 0.1
    d.out_score, d.out_q, d.out_t = ptr(out[0]), ptr(out[1]), ptr(out[2])
    d.max_ref_points, d.max_fit_points = ref.max_points, fit.max_points
    d.lanes_per_pose, d.chunks, d.cta_per_sm = 8, 1, 0
    rc = _lib.load().fss_align_static(ctypes.byref(d), _lib.stream_ptr(dev))
    return rc, out


def test_static_scratch_matches_fss_align_twice(cuda):
    from fast_shepherd_score_b200 import align as al
    ref, fit, idx, sq, st, rs, fs = _problem(cuda)
    want = al.align_packed("shape", ref=ref, fit=fit, pair_ref=idx, pair_fit=idx, seed_q=sq,
                           seed_t=st, steps=40, lr=0.1, alpha=0.81, ref_self=rs, fit_self=fs,
                           lanes_per_pose=8, chunks=1)
    for _ in range(2):
        rc, got = _static_call(ref, fit, idx, sq, st, rs, fs, cuda)
        assert rc == 0
        torch.cuda.synchronize(cuda)
        for g, w in zip(got, want):
            np.testing.assert_allclose(g.cpu().numpy(), w.cpu().numpy(), rtol=0, atol=TOL)
        assert torch.all(got[0] > 0)


def test_static_scratch_rejects_oversized_batch(cuda):
    from fast_shepherd_score_b200 import _lib
    ref, fit, idx, sq, st, rs, fs = _problem(cuda)
    big = 131072 // int(sq.shape[1]) + 1       # n_pairs * n_starts just above the limit
    rc, _ = _static_call(ref, fit, idx, sq, st, rs, fs, cuda, n_pairs=big)
    assert rc == _lib.FSS_ERR_UNSUPPORTED
    assert b"FSS_STATIC_MAX_ROWS" in _lib.load().fss_last_error()
