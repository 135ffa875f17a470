"""GPU: differentiable Tanimoto scores (hand-written adjoint behind torch.autograd.Function).

Checked against (a) the reference's own torch-autograd gradients (golden fixtures, fp64),
(b) fp64 central finite differences of the fp64 scoring oracle (h = 1e-4), and (c) exact
invariances at the configuration-4 size (1024 queries of 60 atoms + 300 surface points).
Tolerance: scores 1e-5 relative; gradients 1e-4 relative (vector norm) and elementwise
1e-4 of the largest component."""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import autograd as AG
from fast_shepherd_score_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _close_grad(got, want):
    got, want = np.asarray(got, np.float64), np.asarray(want, np.float64)
    scale = np.abs(want).max() + 1e-12
    assert np.linalg.norm(got - want) <= 1e-4 * np.linalg.norm(want) + 1e-9, \
        np.linalg.norm(got - want) / np.linalg.norm(want)
    assert np.max(np.abs(got - want)) <= 1e-4 * scale


def _leaf(a, dev):
    return torch.tensor(np.asarray(a), dtype=torch.float32, device=dev, requires_grad=True)


def test_shape_matches_reference_autograd(golden, cuda):
    s = golden["scores"]
    x1, x2 = _leaf(s["c_ref"], cuda), _leaf(s["c_fit"], cuda)
    v = AG.get_overlap(x1, x2, alpha=0.81)
    v.backward()
    np.testing.assert_allclose(v.item(), s["vol_score"], rtol=1e-5)
    _close_grad(x1.grad.cpu().numpy(), s["vol_grad_ref"])
    _close_grad(x2.grad.cpu().numpy(), s["vol_grad_fit"])


@pytest.mark.parametrize("tag", ["esp_surf", "esp_raw"])
def test_esp_matches_reference_autograd(golden, cuda, tag):
    s = golden["scores"]
    p1, p2 = _leaf(s["s_ref"], cuda), _leaf(s["s_fit"], cuda)
    q1, q2 = _leaf(s["q_ref"], cuda), _leaf(s["q_fit"], cuda)
    v = AG.get_overlap_esp(p1, p2, q1, q2, alpha=1.216, lam=float(s[f"{tag}_lam"]))
    v.backward()
    np.testing.assert_allclose(v.item(), s[f"{tag}_score"], rtol=1e-5)
    _close_grad(p1.grad.cpu().numpy(), s[f"{tag}_grad_ref"])
    _close_grad(p2.grad.cpu().numpy(), s[f"{tag}_grad_fit"])
    _close_grad(q1.grad.cpu().numpy(), s[f"{tag}_gradq_ref"])
    _close_grad(q2.grad.cpu().numpy(), s[f"{tag}_gradq_fit"])


def test_against_fp64_finite_differences(cuda):
    from oracle import scores as osc
    rng = np.random.default_rng(2)
    x = syn.ball_clouds(rng, [12])[0].astype(np.float64)
    y = (syn.ball_clouds(rng, [10])[0] + 0.5).astype(np.float64)
    cx = 0.3 * rng.standard_normal(12)
    cy = 0.3 * rng.standard_normal(10)
    lam = 0.3
    f = lambda X, Y, CX, CY: osc.esp_tanimoto(X, Y, CX, CY, 0.81, lam)
    h = 1e-4
    fd_x = np.zeros_like(x)
    for i in range(x.shape[0]):
        for d in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, d] += h; xm[i, d] -= h
            fd_x[i, d] = (f(xp, y, cx, cy) - f(xm, y, cx, cy)) / (2 * h)
    fd_cy = np.zeros_like(cy)
    for j in range(cy.shape[0]):
        cp, cm = cy.copy(), cy.copy()
        cp[j] += h; cm[j] -= h
        fd_cy[j] = (f(x, y, cx, cp) - f(x, y, cx, cm)) / (2 * h)
    X, Y, CX, CY = (_leaf(a, cuda) for a in (x, y, cx, cy))
    v = AG.get_overlap_esp(X, Y, CX, CY, alpha=0.81, lam=lam)
    v.backward()
    np.testing.assert_allclose(v.item(), f(x, y, cx, cy), rtol=1e-5)
    _close_grad(X.grad.cpu().numpy(), fd_x)
    _close_grad(CY.grad.cpu().numpy(), fd_cy)


def test_config4_size_invariances_and_oracle_sample(cuda):
    """1024 queries (60 atoms + 300 surface points, charges N(0, 0.1)) against 4 fixed
    targets that need no gradient: finite gradients everywhere, and a sample of pairs matches
    the fp64 analytic gradients and scores (the rigid-motion invariances at this size are
    checked with both sides differentiable in the next test)."""
    from oracle import scores as osc
    rng = np.random.default_rng(4)
    nq, nt = 1024, 4
    atoms = syn.ball_clouds(rng, [60] * (nq + nt))
    surf = syn.sphere_clouds(rng, [300] * (nq + nt))
    A = torch.tensor(np.stack(atoms), device=cuda)
    S = torch.tensor(np.stack([p for p, _ in surf]), device=cuda)
    Q = torch.tensor(np.stack([c for _, c in surf]), device=cuda)
    qa = A[:nq].clone().requires_grad_(True)
    qs = S[:nq].clone().requires_grad_(True)
    qc = Q[:nq].clone().requires_grad_(True)
    tgt = torch.arange(nq, device=cuda) % nt
    ta, ts, tc = A[nq:][tgt], S[nq:][tgt], Q[nq:][tgt]
    vol = AG.get_overlap(ta, qa, alpha=0.81)
    esp = AG.get_overlap_esp(ts, qs, tc, qc, alpha=1.216)
    (vol.sum() + esp.sum()).backward()
    assert vol.shape == (nq,) and esp.shape == (nq,)
    assert torch.isfinite(qa.grad).all() and torch.isfinite(qs.grad).all()
    for k in range(0, nq, 128):
        i = int(tgt[k])
        gx, gy = osc.shape_tanimoto_grad(atoms[nq + i], atoms[k], 0.81)
        _close_grad(qa.grad[k].cpu().numpy(), gy)
        gx, gy, gcx, gcy = osc.esp_tanimoto_grad(surf[nq + i][0], surf[k][0], surf[nq + i][1],
                                                 surf[k][1], 1.216, 0.3 * AG.LAM_SCALING)
        _close_grad(qs.grad[k].cpu().numpy(), gy)
        _close_grad(qc.grad[k].cpu().numpy(), gcy)
        assert abs(vol[k].item() - osc.shape_tanimoto(atoms[nq + i], atoms[k], 0.81)) < 1e-5


def test_shared_target_accumulates(cuda):
    """A target used by several pairs receives the sum of the pairs' gradients."""
    rng = np.random.default_rng(6)
    t = syn.ball_clouds(rng, [20])[0]
    qs = syn.ball_clouds(rng, [15, 18, 22])
    T = _leaf(t, cuda)
    tot = sum(AG.get_overlap(T, _leaf(q, cuda)) for q in qs)
    tot.backward()
    g_sum = T.grad.clone()
    T2 = _leaf(t, cuda)
    from fast_shepherd_score_b200.layout import CloudSet
    ref = CloudSet.from_arrays([t], device=cuda)
    fit = CloudSet.from_arrays(qs, device=cuda)
    rp = ref.pts.clone().requires_grad_(True)
    s = AG.tanimoto_packed(rp, ref.off, fit.pts, fit.off,
                           torch.zeros(3, dtype=torch.int32, device=cuda),
                           torch.arange(3, dtype=torch.int32, device=cuda))
    s.sum().backward()
    torch.testing.assert_close(rp.grad[:, :3], g_sum, rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("query_side", [0, 1])
@pytest.mark.parametrize("esp", [False, True])
def test_one_sided_backward_matches_two_sided(cuda, esp, query_side):
    """Only the side that requires grad gets adjoint moments; its gradient is the one the
    two-sided backward gives (same moments, same expressions), the other side's .grad stays
    None, and the scores agree to the last bits (summation order may differ)."""
    rng = np.random.default_rng(8)
    surf = syn.sphere_clouds(rng, [41] * 7)
    X = torch.tensor(np.stack([p for p, _ in surf]), device=cuda)
    C = torch.tensor(np.stack([c for _, c in surf]), device=cuda)
    t, tc = X[6:7].expand(6, -1, -1), C[6:7].expand(6, -1)

    def run(grad_target):
        q, qc = X[:6].clone().requires_grad_(True), C[:6].clone().requires_grad_(True)
        tt, ttc = t.clone().requires_grad_(grad_target), tc.clone().requires_grad_(grad_target)
        a, b, ca, cb = (q, tt, qc, ttc) if query_side == 0 else (tt, q, ttc, qc)
        s = (AG.get_overlap_esp(a, b, ca, cb, alpha=1.216, lam=0.3) if esp
             else AG.get_overlap(a, b, alpha=1.216))
        s.sum().backward()
        return s.detach(), q.grad, qc.grad, tt.grad

    s1, g1, gc1, gt1 = run(False)
    s2, g2, gc2, gt2 = run(True)
    assert gt1 is None and gt2 is not None
    torch.testing.assert_close(s1, s2, rtol=5e-6, atol=0)
    torch.testing.assert_close(g1, g2, rtol=2e-5, atol=1e-7)
    if esp:
        torch.testing.assert_close(gc1, gc2, rtol=2e-5, atol=1e-7)
    with torch.no_grad():
        s0 = (AG.get_overlap_esp(X[:6], t, C[:6], tc, alpha=1.216, lam=0.3) if esp
              else AG.get_overlap(X[:6], t, alpha=1.216))
    torch.testing.assert_close(s0, s1, rtol=5e-6, atol=0)


@pytest.mark.parametrize("esp", [0, 1])
def test_moment_backward_matches_two_pass_backward(cuda, esp):
    """fss_score_fwd_moments_dense + fss_score_bwd_moments_dense against fss_score_fwd_dense
    + fss_score_bwd_dense on the same batch (odd cloud sizes, a broadcast target, whose
    gradient accumulates over the pairs, while the per-pair side is stored over NaN-filled
    buffers): overlaps and gradients of both sides to fp32 rounding (the moments kernel evaluates the exponent
    with pre-scaled charges and packed f32x2 arithmetic, so the last bits differ)."""
    from fast_shepherd_score_b200 import _lib
    from fast_shepherd_score_b200._lib import ptr, stream_ptr
    rng = np.random.default_rng(9)
    B, N, M = 5, 37, 50
    x1 = torch.tensor(np.stack(syn.ball_clouds(rng, [N] * B)), device=cuda)
    x2 = torch.tensor(syn.ball_clouds(rng, [M])[0][None], device=cuda)
    q1 = torch.tensor(0.1 * rng.standard_normal((B, N)), dtype=torch.float32, device=cuda)
    q2 = torch.tensor(0.1 * rng.standard_normal((1, M)), dtype=torch.float32, device=cuda)
    pr = torch.arange(B, dtype=torch.int32, device=cuda)
    pf = torch.zeros(B, dtype=torch.int32, device=cuda)
    gs = torch.linspace(0.5, 1.5, B, device=cuda)
    lib, st = _lib.load(), stream_ptr(cuda)
    inv_lam = 1.0 / 0.3 if esp else 0.0
    qa, qb = (ptr(q1), ptr(q2)) if esp else (None, None)

    def fresh():
        return (torch.zeros_like(x1), torch.zeros_like(q1), torch.zeros_like(x2),
                torch.zeros_like(q2))

    sa, ova = torch.empty(B, device=cuda), torch.empty(B, 3, device=cuda)
    assert lib.fss_score_fwd_dense(ptr(x1), qa, N, ptr(x2), qb, M, ptr(pr), ptr(pf), B, 0.81,
                                   esp, inv_lam, ptr(sa), ptr(ova), st) == 0
    ga = fresh()
    assert lib.fss_score_bwd_dense(ptr(x1), qa, N, ptr(x2), qb, M, ptr(pr), ptr(pf), B, 0.81,
                                   esp, inv_lam, ptr(ova), ptr(gs), *(ptr(t) for t in ga),
                                   st) == 0
    sb, ovb = torch.empty(B, device=cuda), torch.empty(B, 3, device=cuda)
    m1, m2 = torch.empty(B, N, 8, device=cuda), torch.empty(B, M, 8, device=cuda)
    assert lib.fss_score_fwd_moments_dense(ptr(x1), qa, N, ptr(x2), qb, M, ptr(pr), ptr(pf), B,
                                           0.81, esp, inv_lam, ptr(sb), ptr(ovb), ptr(m1),
                                           ptr(m2), st) == 0
    gb = fresh()
    gb[0].fill_(float("nan"))   # the ref side (one molecule per pair) is stored, not added
    if esp:                     # (no charge gradients are written without ESP)
        gb[1].fill_(float("nan"))
    assert lib.fss_score_bwd_moments_dense(ptr(pr), ptr(pf), B, N, M, 0.81, esp, inv_lam,
                                           ptr(ova), ptr(gs), ptr(m1), ptr(m2),
                                           *(ptr(t) for t in gb), 1, st) == 0
    torch.cuda.synchronize(cuda)
    torch.testing.assert_close(ovb, ova, rtol=5e-6, atol=0)
    torch.testing.assert_close(sb, sa, rtol=5e-6, atol=0)
    for a, b in zip(ga, gb):
        scale = a.abs().max().item()
        torch.testing.assert_close(b, a, rtol=1e-5, atol=1e-6 * scale)


def test_graph_captured_step_matches_eager(cuda):
    """Forward + backward through get_overlap_esp captured as one CUDA graph: a replay on new
    query values gives the eager scores and gradients (the launches use the capture stream
    and allocate only from the graph's pool)."""
    rng = np.random.default_rng(10)
    surf = syn.sphere_clouds(rng, [33] * 9)
    X = torch.tensor(np.stack([p for p, _ in surf]), device=cuda)
    C = torch.tensor(np.stack([c for _, c in surf]), device=cuda)
    t, tc = X[8:9].expand(4, -1, -1).contiguous(), C[8:9].expand(4, -1).contiguous()
    q = X[:4].clone().requires_grad_(True)
    qc = C[:4].clone().requires_grad_(True)

    def step():
        q.grad = qc.grad = None
        s = AG.get_overlap_esp(t, q, tc, qc, alpha=1.216, lam=0.3)
        s.sum().backward()
        return s

    side = torch.cuda.Stream(cuda)
    side.wait_stream(torch.cuda.current_stream(cuda))
    with torch.cuda.stream(side):
        for _ in range(3):
            step()
    torch.cuda.current_stream(cuda).wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        s_static = step()
    gq, gqc = q.grad, qc.grad
    with torch.no_grad():
        q.copy_(X[4:8])
        qc.copy_(C[4:8])
    g.replay()
    torch.cuda.synchronize(cuda)
    got = (s_static.clone(), gq.clone(), gqc.clone())
    s_eager = step()
    torch.testing.assert_close(got[0], s_eager.detach(), rtol=0, atol=0)
    torch.testing.assert_close(got[1], q.grad, rtol=0, atol=0)
    torch.testing.assert_close(got[2], qc.grad, rtol=0, atol=0)


@pytest.mark.parametrize("n", [700, 2500])
def test_large_clouds_both_adjoint_paths(cuda, n):
    """700-point clouds take the moments kernel with several rows per thread; 2500 + 2500
    points exceed its shared-memory staging (48 bytes a point) and take the two-pass adjoint.
    Both match the fp64 oracle: score 1e-5 relative, gradients 1e-4."""
    from oracle import scores as osc
    rng = np.random.default_rng(11)
    (x, cx), (y, cy) = syn.sphere_clouds(rng, [n, n])
    y = y + 0.3
    lam = 0.3 * AG.LAM_SCALING
    X, Y, CX, CY = (_leaf(a, cuda) for a in (x, y, cx, cy))
    v = AG.get_overlap_esp(X, Y, CX, CY, alpha=1.216, lam=lam)
    v.backward()
    np.testing.assert_allclose(v.item(), osc.esp_tanimoto(x, y, cx, cy, 1.216, lam), rtol=1e-5)
    gx, gy, gcx, gcy = osc.esp_tanimoto_grad(x, y, cx, cy, 1.216, lam)
    _close_grad(X.grad.cpu().numpy(), gx)
    _close_grad(Y.grad.cpu().numpy(), gy)
    _close_grad(CX.grad.cpu().numpy(), gcx)
    _close_grad(CY.grad.cpu().numpy(), gcy)


def test_moments_guard_rows_mixed_with_factored_rows(cuda):
    """Surfaces of radius ~10.5 A: with alpha 1.216 the factored exponent's row factor passes
    its 2^96 bound near that radius, so warps mix rows in the factored and the direct form.
    Scores and both sides' gradients still match the fp64 oracle (1e-5 / 1e-4)."""
    from oracle import scores as osc
    rng = np.random.default_rng(12)

    def surface(n):
        u = rng.standard_normal((n, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        return 10.5 * u + 0.8 * rng.standard_normal((n, 3)), 0.1 * rng.standard_normal(n)

    (x, cx), (y, cy) = surface(320), surface(280)
    y = y + np.array([0.4, -0.3, 0.2])
    lam = 0.3 * AG.LAM_SCALING
    w = -1.216 / 2 * np.log2(np.e) * np.sum((x - x.mean(0)) ** 2, axis=1)
    assert (w < -96).any() and (w > -96).any()   # both forms occur
    X, Y, CX, CY = (_leaf(a, cuda) for a in (x, y, cx, cy))
    v = AG.get_overlap_esp(X, Y, CX, CY, alpha=1.216, lam=lam)
    v.backward()
    np.testing.assert_allclose(v.item(), osc.esp_tanimoto(x, y, cx, cy, 1.216, lam), rtol=1e-5)
    gx, gy, gcx, gcy = osc.esp_tanimoto_grad(x, y, cx, cy, 1.216, lam)
    _close_grad(X.grad.cpu().numpy(), gx)
    _close_grad(Y.grad.cpu().numpy(), gy)
    _close_grad(CX.grad.cpu().numpy(), gcx)
    _close_grad(CY.grad.cpu().numpy(), gcy)


@pytest.mark.parametrize("n", [300, 2500])
def test_no_grad_scores_match_oracle(cuda, n):
    """Under torch.no_grad the dense forward is the factored value-only kernel (300 points) or,
    past its shared-memory staging, the direct kernel (2500 + 2500 points); both give the fp64
    oracle's vol and ESP Tanimoto scores to 1e-5."""
    from oracle import scores as osc
    rng = np.random.default_rng(13)
    surf = syn.sphere_clouds(rng, [n] * 4)
    X = torch.tensor(np.stack([p for p, _ in surf[:2]]), device=cuda)
    Y = torch.tensor(np.stack([p for p, _ in surf[2:]]) + 0.3, device=cuda)
    CX = torch.tensor(np.stack([c for _, c in surf[:2]]), device=cuda)
    CY = torch.tensor(np.stack([c for _, c in surf[2:]]), device=cuda)
    lam = 0.3 * AG.LAM_SCALING
    with torch.no_grad():
        e = AG.get_overlap_esp(X, Y, CX, CY, alpha=1.216, lam=lam).cpu().numpy()
        v = AG.get_overlap(X, Y, alpha=0.81).cpu().numpy()
    for b in range(2):
        x, y = X[b].cpu().numpy().astype(np.float64), Y[b].cpu().numpy().astype(np.float64)
        cx, cy = CX[b].cpu().numpy(), CY[b].cpu().numpy()
        np.testing.assert_allclose(e[b], osc.esp_tanimoto(x, y, cx, cy, 1.216, lam), rtol=1e-5)
        np.testing.assert_allclose(v[b], osc.shape_tanimoto(x, y, 0.81), rtol=1e-5)


def test_config4_size_rigid_motion_invariance(cuda):
    """1024 pairs (60 atoms + 300 charged surface points a side), both sides differentiable:
    a rigid motion of both clouds leaves each score unchanged, so per pair the coordinate
    gradients sum to zero over both clouds (translation) and so do x cross g (rotation), to
    1e-4 of the pair's total gradient magnitude (times its extent for the torque)."""
    rng = np.random.default_rng(14)
    nq = 1024
    atoms = syn.ball_clouds(rng, [60] * (2 * nq))
    surf = syn.sphere_clouds(rng, [300] * (2 * nq))
    A = torch.tensor(np.stack(atoms), device=cuda)
    S = torch.tensor(np.stack([p for p, _ in surf]), device=cuda)
    Q = torch.tensor(np.stack([c for _, c in surf]), device=cuda)
    ta, qa = A[:nq].clone().requires_grad_(True), (A[nq:] + 0.5).requires_grad_(True)
    ts, qs = S[:nq].clone().requires_grad_(True), (S[nq:] + 0.5).requires_grad_(True)
    tc, qc = Q[:nq].clone().requires_grad_(True), Q[nq:].clone().requires_grad_(True)
    vol = AG.get_overlap(ta, qa, alpha=0.81)
    esp = AG.get_overlap_esp(ts, qs, tc, qc, alpha=1.216)
    (vol.sum() + esp.sum()).backward()
    for (x1, x2) in ((ta, qa), (ts, qs)):
        g = torch.cat([x1.grad, x2.grad], 1).double()          # (nq, n1 + n2, 3)
        x = torch.cat([x1.detach(), x2.detach()], 1).double()
        mag = g.norm(dim=2).sum(1)
        force = g.sum(1).norm(dim=1)
        torque = torch.cross(x, g, dim=2).sum(1).norm(dim=1)
        ext = x.norm(dim=2).max(1).values
        assert (force <= 1e-4 * mag).all(), (force / mag).max().item()
        assert (torque <= 1e-4 * mag * ext).all(), (torque / (mag * ext)).max().item()


@pytest.mark.parametrize("both", [False, True])
def test_strong_charge_term_matches_oracle(cuda, both):
    """Raw lambda 0.3 (the vol_esp convention) with charges N(0, 0.5^2): the charge factor
    exp(-(c_i - c_j)^2 / lambda) varies strongly, so the factored charge coefficients and the
    charge moments carry real weight.  4 pairs of 150-point clouds, one or both sides
    differentiable, against the fp64 oracle (1e-5 / 1e-4)."""
    from oracle import scores as osc
    rng = np.random.default_rng(15)
    xs = syn.ball_clouds(rng, [150] * 8)
    cs = [0.5 * rng.standard_normal(150) for _ in range(8)]
    X = torch.tensor(np.stack(xs[:4]), device=cuda).requires_grad_(both)
    Y = torch.tensor(np.stack(xs[4:]) + 0.4, device=cuda).requires_grad_(True)
    CX = torch.tensor(np.stack(cs[:4]), dtype=torch.float32, device=cuda).requires_grad_(both)
    CY = torch.tensor(np.stack(cs[4:]), dtype=torch.float32, device=cuda).requires_grad_(True)
    s = AG.get_overlap_esp(X, Y, CX, CY, alpha=0.81, lam=0.3)
    s.sum().backward()
    for b in range(4):
        x, y = X[b].detach().cpu().numpy().astype(np.float64), Y[b].detach().cpu().numpy().astype(np.float64)
        cx, cy = CX[b].detach().cpu().numpy().astype(np.float64), CY[b].detach().cpu().numpy().astype(np.float64)
        np.testing.assert_allclose(s[b].item(), osc.esp_tanimoto(x, y, cx, cy, 0.81, 0.3), rtol=1e-5)
        gx, gy, gcx, gcy = osc.esp_tanimoto_grad(x, y, cx, cy, 0.81, 0.3)
        _close_grad(Y.grad[b].cpu().numpy(), gy)
        _close_grad(CY.grad[b].cpu().numpy(), gcy)
        if both:
            _close_grad(X.grad[b].cpu().numpy(), gx)
            _close_grad(CX.grad[b].cpu().numpy(), gcx)
