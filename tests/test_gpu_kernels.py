"""GPU parity of the single-evaluation kernels, self overlaps and seeds against the golden
fixtures (reference outputs) and the oracle.  Tolerances: overlap values 1e-5 relative,
gradients 1e-4 relative to the row's largest component (fp32 kernel vs fp64 reference)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _t(a, dev, dtype=None):
    t = torch.as_tensor(np.ascontiguousarray(a), device=dev)
    return t if dtype is None else t.to(dtype)


def _rel_rows(got, ref):
    scale = np.abs(ref).max(1, keepdims=True) + 1e-6
    return np.max(np.abs(got - ref) / scale)


def test_shape_overlap_grad_matches_reference(golden, cuda):
    from fast_shepherd_score_b200 import kernels as K
    g = golden["kernels"]
    V, dQ, dT = K.overlap_score_grad_se3_batch(_t(g["A"], cuda), _t(g["B"], cuda),
                                               _t(g["q"], cuda), _t(g["t"], cuda), alpha=0.81,
                                               N_real=_t(g["N"], cuda), M_real=_t(g["M"], cuda))
    V, dQ, dT = V.cpu().numpy(), dQ.cpu().numpy(), dT.cpu().numpy()
    big = g["shape_V"] > 1e-3
    np.testing.assert_allclose(V[big], g["shape_V"][big], rtol=1e-5)
    np.testing.assert_allclose(V[~big], g["shape_V"][~big], atol=1e-7)
    assert _rel_rows(dQ[big], g["shape_dQ"][big]) < 1e-4
    assert _rel_rows(dT[big], g["shape_dT"][big]) < 1e-4


@pytest.mark.parametrize("tag", ["esp_surf", "esp_raw"])
def test_esp_overlap_grad_matches_reference(golden, cuda, tag):
    from fast_shepherd_score_b200 import kernels as K
    g = golden["kernels"]
    V, dQ, dT = K.overlap_score_grad_esp_se3_batch(
        _t(g["A"], cuda), _t(g["B"], cuda), _t(g["CA"], cuda), _t(g["CB"], cuda),
        _t(g["q"], cuda), _t(g["t"], cuda), alpha=0.81, lam=float(g[f"{tag}_lam"]),
        N_real=_t(g["N"], cuda), M_real=_t(g["M"], cuda))
    V, dQ, dT = V.cpu().numpy(), dQ.cpu().numpy(), dT.cpu().numpy()
    ref = g[f"{tag}_V"]
    big = ref > 1e-3
    np.testing.assert_allclose(V[big], ref[big], rtol=1e-5)
    assert _rel_rows(dQ[big], g[f"{tag}_dQ"][big]) < 1e-4
    assert _rel_rows(dT[big], g[f"{tag}_dT"][big]) < 1e-4


@pytest.mark.parametrize("directional", [True, False])
def test_pharm_grad_matches_reference(golden, cuda, directional):
    from fast_shepherd_score_b200 import kernels as K
    g = golden["kernels"]
    args = [_t(g[k], cuda) for k in ("pq", "pt", "PAt", "PBt", "PA", "PB", "PRV", "PFV")]
    if directional:
        O, dQ, dT = K.pharm_grad_dq_se3_batch(*args, N_real=_t(g["PN"], cuda),
                                              M_real=_t(g["PM"], cuda))
        tag = "pharm"
    else:
        q, t, At, Bt, A, B = args[:6]
        O, dQ, dT = K.pharm_color_score_grad_se3_batch(A, B, q, t, At, Bt,
                                                       N_real=_t(g["PN"], cuda),
                                                       M_real=_t(g["PM"], cuda))
        tag = "color"
    O, dQ, dT = O.cpu().numpy(), dQ.cpu().numpy(), dT.cpu().numpy()
    ref = g[f"{tag}_O"]
    np.testing.assert_allclose(O, ref, rtol=1e-5, atol=1e-7)
    big = ref > 1e-3
    assert _rel_rows(dQ[big], g[f"{tag}_dQ"][big]) < 1e-4
    assert _rel_rows(dT[big], g[f"{tag}_dT"][big]) < 1e-4


def test_type_masks_are_exact(cuda):
    """A fit feature only ever overlaps reference features of the identical type: shuffling
    the reference types so that no type matches gives exactly zero overlap and gradient."""
    from fast_shepherd_score_b200 import kernels as K
    rng = np.random.default_rng(3)
    A = rng.standard_normal((4, 10, 3)).astype(np.float32)
    V = rng.standard_normal((4, 10, 3)).astype(np.float32)
    At = np.tile(np.arange(10) % 4, (4, 1))              # types 0..3
    Bt = np.tile(4 + np.arange(10) % 4, (4, 1))          # types 4..7
    q = np.tile([1.0, 0, 0, 0], (4, 1)).astype(np.float32)
    t = np.zeros((4, 3), np.float32)
    O, dQ, dT = K.pharm_grad_dq_se3_batch(_t(q, cuda), _t(t, cuda), _t(At, cuda), _t(Bt, cuda),
                                          _t(A, cuda), _t(A, cuda), _t(V, cuda), _t(V, cuda))
    assert torch.all(O == 0) and torch.all(dQ == 0) and torch.all(dT == 0)
    # dummy type (8) and out-of-table types are skipped entirely
    Bt2 = np.full((4, 10), 8)
    O, _, _ = K.pharm_grad_dq_se3_batch(_t(q, cuda), _t(t, cuda), _t(Bt2, cuda), _t(Bt2, cuda),
                                        _t(A, cuda), _t(A, cuda), _t(V, cuda), _t(V, cuda))
    assert torch.all(O == 0)


def test_self_overlap_packed_matches_reference(golden, cuda):
    from fast_shepherd_score_b200 import kernels as K
    from fast_shepherd_score_b200.layout import CloudSet
    g = golden["kernels"]
    cs = CloudSet.from_padded(_t(g["A"], cuda), _t(g["N"], cuda))
    np.testing.assert_allclose(K.self_overlap(cs, 0.81).cpu().numpy(), g["self_shape_A"],
                               rtol=1e-5)
    cs = CloudSet.from_padded(_t(g["A"], cuda), _t(g["N"], cuda), _t(g["CA"], cuda))
    np.testing.assert_allclose(K.self_overlap(cs, 0.81, esp=True, lam=0.3).cpu().numpy(),
                               g["self_esp_A"], rtol=1e-5)
    # padded-batch wrappers agree with the packed kernel
    v = K._batch_self_overlap(_t(g["A"], cuda), _t(g["N"], cuda), 0.81).cpu().numpy()
    np.testing.assert_allclose(v, g["self_shape_A"], rtol=1e-5)


@pytest.mark.parametrize("ns", [1, 3, 8, 10, 16, 32, 50])
def test_seeds_match_reference(golden, cuda, ns):
    from fast_shepherd_score_b200 import kernels as K
    from fast_shepherd_score_b200.layout import CloudSet
    s = golden["seeds"]
    ref = CloudSet.from_padded(_t(s["A"], cuda), _t(s["N"], cuda))
    fit = CloudSet.from_padded(_t(s["B"], cuda), _t(s["M"], cuda))
    idx = torch.arange(len(s["N"]), dtype=torch.int32, device=cuda)
    q, t = K.seeds(ref, fit, idx, idx, ns)
    np.testing.assert_allclose(q.cpu().numpy(), s[f"q_{ns}"], atol=2e-5)
    np.testing.assert_allclose(t.cpu().numpy(), s[f"t_{ns}"], atol=5e-5)


def _tail_np(V, dQ, dT, U, q, t, mq, vq, mt, vt, best, bq, bt, lr):
    """Numpy statement of the reference tail (accel/kernels/cpu_fused.py:54-108): float32
    state, Tanimoto scale, pre-update best, tangent-projected Adam, renormalisation."""
    f = np.float32
    denom = U - V
    denom = np.where(denom == 0, f(1e-12), denom)
    score = V / denom
    scale = U / (denom * denom)
    better = score > best
    best = np.where(better, score, best)
    bq = np.where(better[:, None], q, bq)
    bt = np.where(better[:, None], t, bt)
    gq = -scale[:, None] * dQ
    gt = -scale[:, None] * dT
    d = gq - q * (gq * q).sum(1, keepdims=True)
    mq = f(0.9) * mq + f(0.1) * d
    vq = f(0.999) * vq + f(1 - f(0.999)) * d * d
    q = q - f(lr) * mq / np.sqrt(vq + f(1e-8))
    mt = f(0.9) * mt + f(0.1) * gt
    vt = f(0.999) * vt + f(1 - f(0.999)) * gt * gt
    t = t - f(lr) * mt / np.sqrt(vt + f(1e-8))
    q = q / np.maximum(np.sqrt((q * q).sum(1, keepdims=True)), f(1e-12))
    return q, t, mq, vq, mt, vt, best, bq, bt


def test_tanimoto_adam_step_matches_reference_tail(cuda):
    """Three optimiser steps on the GPU equal the reference tail applied to the same kernel
    outputs (float32 arithmetic both sides)."""
    from fast_shepherd_score_b200 import kernels as K
    rng = np.random.default_rng(7)
    A = rng.standard_normal((6, 20, 3)).astype(np.float32) * 2
    B = rng.standard_normal((6, 18, 3)).astype(np.float32) * 2
    q = rng.standard_normal((6, 4)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    t = (0.3 * rng.standard_normal((6, 3))).astype(np.float32)
    f = lambda a: _t(a, cuda, torch.float32).contiguous()
    U = (K._batch_self_overlap(f(A), None) + K._batch_self_overlap(f(B), None)).contiguous()
    qd, td = f(q), f(t)
    z4, z3 = torch.zeros(6, 4, device=cuda), torch.zeros(6, 3, device=cuda)
    mq, vq, mt, vt = z4.clone(), z4.clone(), z3.clone(), z3.clone()
    bs = torch.full((6,), -float("inf"), device=cuda)
    bqd, btd = qd.clone(), td.clone()
    st = [q.copy(), t.copy(), np.zeros((6, 4), np.float32), np.zeros((6, 4), np.float32),
          np.zeros((6, 3), np.float32), np.zeros((6, 3), np.float32),
          np.full(6, -np.inf, np.float32), q.copy(), t.copy()]
    for _ in range(3):
        V, dQ, dT = K.overlap_score_grad_se3_batch(f(A), f(B), qd, td, alpha=0.81)
        h = [x.cpu().numpy() for x in (V, dQ, dT, U)]
        st = list(_tail_np(*h, *st, 0.1))
        K.tanimoto_adam_step(V, dQ, dT, U, qd, td, mq, vq, mt, vt, bs, bqd, btd, 0.1)
        # Adam's m/sqrt(v+eps) turns a 1-ulp gradient difference on a near-zero component
        # into ~1e-6 in q; wrong constants or signs would show up at 1e-2
        np.testing.assert_allclose(qd.cpu().numpy(), st[0], atol=2e-5)
        np.testing.assert_allclose(td.cpu().numpy(), st[1], atol=2e-5)
        np.testing.assert_allclose(bs.cpu().numpy(), st[6], rtol=1e-6)
        np.testing.assert_allclose(bqd.cpu().numpy(), st[7], atol=2e-5)
