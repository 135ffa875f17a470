"""Translation-seeded starts (trans_init=True) without a GPU: the host-side legacy grid against
the reference's own grids (tests/golden/trans_init.npz), the top-k selection, and the
oracle's coarse grid + top-k + fine path against the reference's alignments."""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import legacy_seeds as L
from fast_shepherd_score_b200.kernels import _fibo_host
from fast_shepherd_score_b200.layout import CloudSet

TAGS = ("esp", "pharm", "color", "combo")


def _centred(x):
    """Cloud minus its centroid as the reference's pharmacophore driver computes it
    (float32 torch sum / count)."""
    t = torch.as_tensor(np.ascontiguousarray(x))
    return (t - t.sum(0) / float(len(x))).numpy()


def grid_inputs(g, tag, i):
    """(ref, fit, centres) real points the reference builds pair i's legacy grid from."""
    if tag == "esp":
        n, m, c = g["esp_N"][i], g["esp_M"][i], g["esp_TN"][i]
        return g["esp_A"][i, :n], g["esp_B"][i, :m], g["esp_TC"][i, :c]
    if tag == "pharm":
        n, m = g["pharm_N"][i], g["pharm_M"][i]
        a = _centred(g["pharm_A"][i, :n])
        return a, _centred(g["pharm_B"][i, :m]), a
    if tag == "color":
        n, m = g["color_N"][i], g["color_M"][i]
        return g["color_A"][i, :n], g["color_B"][i, :m], g["color_A"][i, :n]
    n, m, c = g["combo_SN1"][i], g["combo_SN2"][i], g["combo_CN1"][i]
    return g["combo_S1"][i, :n], g["combo_S2"][i, :m], g["combo_C1"][i, :c]


@pytest.mark.parametrize("tag", TAGS)
def test_legacy_grid_matches_reference(golden, tag):
    """Identity, the 4 principal-axis poses (LAPACK eigenvector signs included) and the
    Fibonacci rotations per centre agree with the reference's grid to float32 rounding.  The
    inertia sums run in another order than the reference's numpy calls; for clouds of a
    handful of anchors, whose inertia moments lie close together, that moves an axis by up
    to ~1e-5, hence the quaternion tolerance."""
    g = golden["trans_init"]
    for i in range(len(g[f"{tag}_G"])):
        ref, fit, ctr = grid_inputs(g, tag, i)
        q, t = L.pair_grid(ref, fit, ctr, 10)
        G = int(g[f"{tag}_G"][i])
        assert q.shape == (G, 4) and t.shape == (G, 3)
        np.testing.assert_allclose(q.numpy(), g[f"{tag}_GQ"][i, :G], atol=1e-5)
        np.testing.assert_allclose(t.numpy(), g[f"{tag}_GT"][i, :G], atol=4e-6)


def test_45_rotation_grid(golden):
    """num_repeats_per_trans=45 uses the reference's precomputed 45-rotation table; the
    Fibonacci construction reproduces it."""
    g = golden["trans_init"]
    np.testing.assert_allclose(_fibo_host(45), g["fibo45"], atol=2e-7)
    ref, fit, ctr = grid_inputs(g, "esp", 1)
    q, t = L.pair_grid(ref, fit, ctr[:2], 45)
    np.testing.assert_allclose(q.numpy(), g["g45_q"], atol=1e-6)
    np.testing.assert_allclose(t.numpy(), g["g45_t"], atol=4e-6)


def test_grid_packed_pads_and_shifts():
    """Packed clouds give the per-pair grids; rows past G repeat pose 0; centre_shift moves
    each reference molecule's centres."""
    rng = np.random.default_rng(3)
    refs = [rng.standard_normal((n, 3)).astype(np.float32) * 2 for n in (6, 9)]
    fits = [rng.standard_normal((n, 3)).astype(np.float32) * 2 for n in (7, 5)]
    ctrs = [r[:k] for r, k in zip(refs, (2, 4))]
    cs = lambda xs: CloudSet.from_arrays(xs, device="cpu")
    pr = torch.tensor([1, 0, 1], dtype=torch.int32)
    pf = torch.tensor([0, 1, 1], dtype=torch.int32)
    shift = torch.tensor([[0.5, 0, 0], [0, -1.0, 0]])
    q, t, G = L.grid_packed(cs(refs), cs(fits), cs(ctrs), pr, pf, 3, shift)
    assert list(G) == [5 + 3 * 4, 5 + 3 * 2, 5 + 3 * 4] and q.shape == (3, 17, 4)
    for k, (i, j) in enumerate(zip(pr.tolist(), pf.tolist())):
        qq, tt = L.pair_grid(refs[i], fits[j], ctrs[i] - shift[i].numpy(), 3)
        np.testing.assert_array_equal(q[k, :G[k]].numpy(), qq.numpy())
        np.testing.assert_array_equal(t[k, :G[k]].numpy(), tt.numpy())
        assert torch.equal(q[k, G[k]:], qq[0].expand(17 - G[k], 4))


def test_select_excludes_padding_and_checks_topk():
    q = torch.arange(2 * 6 * 4, dtype=torch.float32).reshape(2, 6, 4)
    t = torch.arange(2 * 6 * 3, dtype=torch.float32).reshape(2, 6, 3)
    sc = torch.tensor([[0.1, 0.5, 0.3, 0.9, 0.9, 0.9], [0.2, 0.1, 0.4, 0.3, 0.0, 0.05]])
    sq, st = L.select(sc.reshape(-1), q, t, np.array([3, 6]), 2)
    assert torch.equal(sq[0], q[0, [1, 2]]) and torch.equal(st[0], t[0, [1, 2]])
    assert torch.equal(sq[1], q[1, [2, 3]])
    with pytest.raises(ValueError):
        L.select(sc.reshape(-1), q, t, np.array([3, 6]), 4)


def oracle_call(g, tag):
    """(oracle driver, positional args, keyword args) of the reference call in the fixture."""
    from oracle import align as oa
    if tag == "esp":
        return oa.align_esp, tuple(g[f"esp_{k}"] for k in ("A", "B", "CA", "CB", "N", "M")), \
            dict(alpha=0.81, lam=float(g["esp_lam"]))
    if tag == "pharm":
        return oa.align_pharm, tuple(g[f"pharm_{k}"] for k in
                                     ("A", "B", "RV", "FV", "At", "Bt", "N", "M")), {}
    if tag == "color":
        return oa.align_combo, (g["color_A"], g["color_B"], g["color_N"], g["color_M"],
                                g["pharm_A"], g["pharm_B"], None, None, g["color_At"],
                                g["color_Bt"], g["pharm_N"], g["pharm_M"]), \
            dict(alpha=0.81, w=0.5, directional=False)
    keys = ("C1", "C2", "CN1", "CN2", "A1", "A2", "Q1", "Q2", "R1", "R2", "AN1", "AN2", "S1",
            "S2", "PE1", "PE2", "SN1", "SN2")
    return oa.align_esp_combo, tuple(g["combo_" + k] for k in keys), \
        dict(alpha=0.81, lam=0.001, probe_radius=1.0, esp_weight=0.5, stride=5)


@pytest.mark.parametrize("tag", TAGS)
def test_oracle_trans_path_matches_reference(golden, tag):
    """The oracle's coarse grid + top-k 30 + 30 fine steps from the reference's grid give the
    reference's best scores (the oracle's alignment tolerance, 2e-3)."""
    from oracle import align as oa
    g = golden["trans_init"]
    fn, args, kw = oracle_call(g, tag)
    sc, _, _ = oa.align_trans(fn, args, g[f"{tag}_GQ"], g[f"{tag}_GT"], g[f"{tag}_G"], topk=30,
                              steps=30, lr=0.1, **kw)
    np.testing.assert_allclose(sc, g[f"{tag}_score"], atol=2e-3)


def test_degenerate_clouds_give_finite_grids():
    """One-point and collinear clouds (equal or antiparallel principal axes; the reference's
    axis-angle step divides 0 by 0 there) still give unit quaternions and finite
    translations, and an empty batch gives empty grids."""
    one = np.ones((1, 3), np.float32)
    line = np.stack([np.linspace(-2, 2, 5)] * 3, 1).astype(np.float32)
    for ref, fit in ((one, one * 0), (line, line[::-1] * 1.5), (line, one)):
        q, t = L.pair_grid(ref, fit, ref[:2], 10)
        assert torch.isfinite(q).all() and torch.isfinite(t).all()
        np.testing.assert_allclose(q.norm(dim=1).numpy(), 1.0, atol=1e-6)
    q, t, G = L.grid_padded(torch.zeros(0, 4, 3), [], torch.zeros(0, 5, 3), [],
                            torch.zeros(0, 2, 3), [], 10)
    assert q.shape == (0, 5, 4) and t.shape == (0, 5, 3) and len(G) == 0
