"""The tensor-core paths (accumulate=2: value/gradient sums as mma tf32 hi/lo products;
accumulate=3: pairwise exponents as 3-pass tf32 mma; one warp per pose) against the reference
fixtures, the oracle and the FP32-lane path.

Step 1 scores are the seeds' own Tanimoto values, so they compare at fp32 rounding
(rtol 2e-5); later steps compare by best score (Adam amplifies rounding chaotically once a
pose has converged, as in test_gpu_align)."""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import align as al
from fast_shepherd_score_b200 import kernels as K
from fast_shepherd_score_b200 import synthetic as syn
from fast_shepherd_score_b200.layout import CloudSet

from test_gpu_align import _t, assert_parity

pytestmark = pytest.mark.gpu
ACCS = pytest.mark.parametrize("acc", [2, 3])
LAM_SURF = 0.3 * (1e4 / (4 * 55.263 * np.pi)) ** 2


def _golden_sets(g, cuda, tag):
    ref = CloudSet.from_padded(_t(g[f"{tag}_A"], cuda), _t(g[f"{tag}_N"], cuda),
                               _t(g[f"{tag}_CA"], cuda) if tag == "esp" else None)
    fit = CloudSet.from_padded(_t(g[f"{tag}_B"], cuda), _t(g[f"{tag}_M"], cuda),
                               _t(g[f"{tag}_CB"], cuda) if tag == "esp" else None)
    return ref, fit


@ACCS
def test_shape_tensor_sums_track_oracle_stepwise(golden, cuda, acc):
    from oracle import align as oa
    g = golden["align"]
    qs, ts = g["shape_seeds_q"], g["shape_seeds_t"]
    A, B, N, M = g["shape_A"], g["shape_B"], g["shape_N"], g["shape_M"]
    ref, fit = _golden_sets(g, cuda, "shape")
    idx = torch.arange(len(N), dtype=torch.int32, device=cuda)
    for steps in (1, 3):
        res = al.align_packed("shape", ref=ref, fit=fit, pair_ref=idx, pair_fit=idx,
                              seed_q=_t(qs, cuda), seed_t=_t(ts, cuda), steps=steps, lr=0.1,
                              accumulate=acc)
        rows = res.rows[0].cpu().numpy()
        _, _, _, (best, _, _) = oa.align_shape(A, B, N, M, alpha=0.81, steps=steps, lr=0.1,
                                               seeds=(qs, ts), return_rows=True)
        tol = dict(rtol=2e-5, atol=1e-6) if steps == 1 else dict(rtol=0, atol=5e-5)
        np.testing.assert_allclose(rows, best, **tol)


@ACCS
def test_shape_tensor_sums_match_reference(golden, cuda, acc):
    g = golden["align"]
    ref, fit = _golden_sets(g, cuda, "shape")
    idx = torch.arange(len(g["shape_N"]), dtype=torch.int32, device=cuda)
    res = al.align_packed("shape", ref=ref, fit=fit, pair_ref=idx, pair_fit=idx,
                          seed_q=_t(g["shape_seeds_q"], cuda),
                          seed_t=_t(g["shape_seeds_t"], cuda), steps=80, lr=0.1,
                          accumulate=acc)
    sc = res[0].cpu().numpy()
    assert_parity(sc, g["shape_score"])
    assert (sc[:2] > 0.99).all()


@ACCS
def test_esp_tensor_sums_match_reference(golden, cuda, acc):
    g = golden["align"]
    ref, fit = _golden_sets(g, cuda, "esp")
    idx = torch.arange(len(g["esp_N"]), dtype=torch.int32, device=cuda)
    res = al.align_packed("esp", ref=ref, fit=fit, pair_ref=idx, pair_fit=idx,
                          seed_q=_t(g["esp_seeds_q"], cuda), seed_t=_t(g["esp_seeds_t"], cuda),
                          steps=60, lr=0.1, lam=float(g["esp_lam"]), accumulate=acc)
    sc = res[0].cpu().numpy()
    assert_parity(sc, g["esp_score"])
    assert sc[0] > 0.99


def _surface_sets(cuda, n_pairs, seed):
    refs, fits = syn.esp_surface_pairs(n_pairs, seed=seed)
    ref = CloudSet.from_arrays([p for p, _ in refs], [c for _, c in refs], device=cuda)
    fit = CloudSet.from_arrays([p for p, _ in fits], [c for _, c in fits], device=cuda)
    return ref, fit


@ACCS
def test_surface_esp_first_step_matches_fp32_path(cuda, acc):
    """200-400 point surfaces with charges (the surf_esp workload's shapes): every start's
    step-1 score agrees with the FP32 path to fp32 rounding, then best scores agree."""
    ref, fit = _surface_sets(cuda, 24, seed=11)
    idx = torch.arange(24, dtype=torch.int32, device=cuda)
    sq, st = K.seeds(ref, fit, idx, idx, 50)
    kw = dict(ref=ref, fit=fit, pair_ref=idx, pair_fit=idx, seed_q=sq, seed_t=st, lr=0.1,
              lam=LAM_SURF)
    a = al.align_packed("esp", steps=1, accumulate=1, **kw).rows[0].cpu().numpy()
    b = al.align_packed("esp", steps=1, accumulate=acc, **kw).rows[0].cpu().numpy()
    np.testing.assert_allclose(b, a, rtol=2e-5, atol=1e-6)
    a = al.align_packed("esp", steps=40, accumulate=1, **kw)[0].cpu().numpy()
    b = al.align_packed("esp", steps=40, accumulate=acc, **kw)[0].cpu().numpy()
    assert_parity(b, a, worst=2e-3)


@ACCS
def test_far_poses_use_the_unfactored_exponent(cuda, acc):
    """Seeds 20 A away push k|b'|^2 past the factoring limit; the unfactored branch must give
    the same (tiny) step-1 scores as the FP32 path."""
    ref, fit = _surface_sets(cuda, 4, seed=12)
    idx = torch.arange(4, dtype=torch.int32, device=cuda)
    sq, st = K.seeds(ref, fit, idx, idx, 10)
    st = st + torch.tensor([20.0, 0.0, 0.0], device=cuda)
    kw = dict(ref=ref, fit=fit, pair_ref=idx, pair_fit=idx, seed_q=sq, seed_t=st, lr=0.1,
              steps=1)
    a = al.align_packed("shape", accumulate=1, **kw).rows[0].cpu().numpy()
    b = al.align_packed("shape", accumulate=acc, **kw).rows[0].cpu().numpy()
    assert np.all(np.isfinite(b))
    np.testing.assert_allclose(b, a, rtol=1e-4, atol=1e-9)


@ACCS
def test_tensor_sums_edge_sizes(cuda, acc):
    """Empty clouds, single points and every remainder of the 32-row pass / 8-point block."""
    rng = np.random.default_rng(7)
    sizes = [(1, 1), (0, 5), (5, 0), (7, 31), (8, 32), (9, 33), (33, 17), (64, 65), (1, 40),
             (16, 15), (17, 16)]
    refs = [rng.standard_normal((n, 3)).astype(np.float32) * 2 for n, _ in sizes]
    fits = [rng.standard_normal((m, 3)).astype(np.float32) * 2 for _, m in sizes]
    ref = CloudSet.from_arrays(refs, device=cuda)
    fit = CloudSet.from_arrays(fits, device=cuda)
    idx = torch.arange(len(sizes), dtype=torch.int32, device=cuda)
    sq, st = K.seeds(ref, fit, idx, idx, 10)
    kw = dict(ref=ref, fit=fit, pair_ref=idx, pair_fit=idx, seed_q=sq, seed_t=st, lr=0.1)
    a = al.align_packed("shape", steps=1, accumulate=1, **kw).rows[0].cpu().numpy()
    b = al.align_packed("shape", steps=1, accumulate=acc, **kw).rows[0].cpu().numpy()
    np.testing.assert_allclose(b, a, rtol=2e-5, atol=1e-6)
    sc = al.align_packed("shape", steps=20, accumulate=acc, **kw)[0].cpu().numpy()
    assert np.all(np.isfinite(sc)) and np.all((sc >= 0) & (sc <= 1.0 + 1e-5))
    assert sc[1] == 0 and sc[2] == 0


@ACCS
def test_tensor_sums_reject_other_modes(cuda, acc):
    ref, fit = _surface_sets(cuda, 2, seed=3)
    idx = torch.arange(2, dtype=torch.int32, device=cuda)
    sq, st = K.seeds(ref, fit, idx, idx, 4)
    with pytest.raises((ValueError, RuntimeError)):
        al.align_packed("shape", ref=ref, fit=fit, pair_ref=idx, pair_fit=idx, seed_q=sq,
                        seed_t=st, steps=1, lr=0.1, accumulate=acc, lanes_per_pose=8)
