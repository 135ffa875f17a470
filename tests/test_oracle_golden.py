"""The CPU oracle reproduces the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the reference numba path and torch scoring)."""
import numpy as np
import pytest

from oracle import align as oa
from oracle import scores as osc
from oracle.seeds import batched_seeds


def _rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-6))


def test_shape_kernel(golden):
    g = golden["kernels"]
    V, dQ, dT = oa.overlap_grad(g["A"], g["B"], g["q"], g["t"], g["N"], g["M"], alpha=0.81)
    assert _rel(V, g["shape_V"]) < 1e-6
    scale = np.abs(g["shape_dQ"]).max(1, keepdims=True) + 1e-6
    assert np.max(np.abs(dQ - g["shape_dQ"]) / scale) < 1e-5
    scale = np.abs(g["shape_dT"]).max(1, keepdims=True) + 1e-6
    assert np.max(np.abs(dT - g["shape_dT"]) / scale) < 1e-5


@pytest.mark.parametrize("tag", ["esp_surf", "esp_raw"])
def test_esp_kernel(golden, tag):
    g = golden["kernels"]
    V, dQ, dT = oa.overlap_grad(g["A"], g["B"], g["q"], g["t"], g["N"], g["M"], alpha=0.81,
                                CA=g["CA"], CB=g["CB"], lam=float(g[f"{tag}_lam"]))
    assert _rel(V, g[f"{tag}_V"]) < 1e-6
    scale = np.abs(g[f"{tag}_dQ"]).max(1, keepdims=True) + 1e-6
    assert np.max(np.abs(dQ - g[f"{tag}_dQ"]) / scale) < 1e-5


def test_self_overlaps(golden):
    g = golden["kernels"]
    np.testing.assert_allclose(oa.self_overlap(g["A"], g["N"]), g["self_shape_A"], rtol=1e-6)
    np.testing.assert_allclose(oa.self_overlap(g["A"], g["N"], C=g["CA"], lam=0.3),
                               g["self_esp_A"], rtol=1e-6)


@pytest.mark.parametrize("directionless", [False, True])
def test_pharm_kernels(golden, directionless):
    g = golden["kernels"]
    tag = "color" if directionless else "pharm"
    O, dQ, dT = oa.pharm_grad(g["PA"], g["PB"], None if directionless else g["PRV"],
                              None if directionless else g["PFV"], g["PAt"], g["PBt"], g["pq"],
                              g["pt"], g["PN"], g["PM"], directionless=directionless)
    np.testing.assert_allclose(O, g[f"{tag}_O"], rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(dQ, g[f"{tag}_dQ"], rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(dT, g[f"{tag}_dT"], rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("ns", [1, 3, 8, 10, 16, 32, 50])
def test_seeds(golden, ns):
    s = golden["seeds"]
    q, t = batched_seeds(s["A"], s["B"], s["N"], s["M"], ns)
    np.testing.assert_allclose(q, s[f"q_{ns}"], atol=2e-6)
    np.testing.assert_allclose(t, s[f"t_{ns}"], atol=2e-6)


def test_align_shape_matches_reference_exactly(golden):
    g = golden["align"]
    sc, q, t = oa.align_shape(g["shape_A"], g["shape_B"], g["shape_N"], g["shape_M"], alpha=0.81,
                              steps=80, lr=0.1, seeds=(g["shape_seeds_q"], g["shape_seeds_t"]))
    np.testing.assert_allclose(sc, g["shape_score"], atol=1e-6)
    assert sc[0] > 0.99 and sc[1] > 0.99          # rotated self copies


def test_align_esp(golden):
    g = golden["align"]
    sc, q, t = oa.align_esp(g["esp_A"], g["esp_B"], g["esp_CA"], g["esp_CB"], g["esp_N"],
                            g["esp_M"], alpha=0.81, lam=float(g["esp_lam"]), num_seeds=10,
                            steps=60, lr=0.1)
    np.testing.assert_allclose(sc, g["esp_score"], atol=1e-4)
    assert sc[0] > 0.99


def test_align_pharm(golden):
    # Adam amplifies 1e-7 seed differences chaotically; best scores stay within 1e-3 here
    # (pairs not yet converged at 60 steps) and self-copies reach 1.
    g = golden["align"]
    sc, q, t = oa.align_pharm(g["pharm_A"], g["pharm_B"], g["pharm_RV"], g["pharm_FV"],
                              g["pharm_At"], g["pharm_Bt"], g["pharm_N"], g["pharm_M"],
                              num_seeds=16, steps=60, lr=0.1)
    np.testing.assert_allclose(sc, g["pharm_score"], atol=1e-3)
    assert sc[0] > 0.99


def test_align_vol_color(golden):
    g = golden["align"]
    sc, q, t = oa.align_combo(g["color_A"], g["color_B"], g["color_N"], g["color_M"],
                              g["pharm_A"], g["pharm_B"], None, None, g["color_At"],
                              g["color_Bt"], g["pharm_N"], g["pharm_M"], alpha=0.81, w=0.5,
                              directional=False, num_seeds=16, steps=60, lr=0.1)
    np.testing.assert_allclose(sc, g["color_score"], atol=1e-4)
    assert sc[0] > 0.99


def test_fp64_scores(golden):
    s = golden["scores"]
    v = osc.shape_tanimoto(s["c_ref"], s["c_fit"], 0.81)
    np.testing.assert_allclose(v, s["vol_score"], rtol=1e-12)
    for tag in ("esp_surf", "esp_raw"):
        v = osc.esp_tanimoto(s["s_ref"], s["s_fit"], s["q_ref"], s["q_fit"], 1.216,
                             float(s[f"{tag}_lam"]))
        np.testing.assert_allclose(v, s[f"{tag}_score"], rtol=1e-12)
    for dl in (0, 1):
        v = osc.pharm_tanimoto(s["pt_ref"], s["pt_fit"], s["pa_ref"], s["pa_fit"], s["pv_ref"],
                               s["pv_fit"], directionless=bool(dl))
        np.testing.assert_allclose(v, s[f"pharm_score_dl{dl}"], rtol=1e-10)
        v = osc.combo_score(s["c_ref"], s["c_fit"], s["pt_ref"], s["pt_fit"], s["pa_ref"],
                            s["pa_fit"], s["pv_ref"], s["pv_fit"], alpha=0.81, w=0.5,
                            directionless=bool(dl))
        np.testing.assert_allclose(v, s[f"combo_score_dl{dl}"], rtol=1e-10)


def test_fp64_coordinate_gradients(golden):
    s = golden["scores"]
    gr, gf = osc.shape_tanimoto_grad(s["c_ref"], s["c_fit"], 0.81)
    np.testing.assert_allclose(gr, s["vol_grad_ref"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(gf, s["vol_grad_fit"], rtol=1e-9, atol=1e-12)
    for tag in ("esp_surf", "esp_raw"):
        gr, gf, gqr, gqf = osc.esp_tanimoto_grad(s["s_ref"], s["s_fit"], s["q_ref"], s["q_fit"],
                                                 1.216, float(s[f"{tag}_lam"]))
        np.testing.assert_allclose(gr, s[f"{tag}_grad_ref"], rtol=1e-8, atol=1e-12)
        np.testing.assert_allclose(gf, s[f"{tag}_grad_fit"], rtol=1e-8, atol=1e-12)
        np.testing.assert_allclose(gqr, s[f"{tag}_gradq_ref"], rtol=1e-8, atol=1e-12)
        np.testing.assert_allclose(gqf, s[f"{tag}_gradq_fit"], rtol=1e-8, atol=1e-12)


@pytest.mark.parametrize("ext", [1, 2])
def test_pharm_extended_points_kernel(golden, ext):
    """Extended-point overlap (the typed overlap of the batched fine loop, extended_points /
    only_extended): value, dO/dt and the tangential part of dO/dq (the reference normalises q
    inside its transform, so its autograd dO/dq is tangent to the unit sphere)."""
    g = golden["pharm_ext"]
    O, dQ, dT = oa.pharm_grad(g["sp_A"], g["sp_B"], g["sp_RV"], g["sp_FV"], g["sp_At"],
                              g["sp_Bt"], g["sp_q"], g["sp_t"], ext=ext)
    q = g["sp_q"].astype(np.float64)
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    dQ = dQ - q * (dQ * q).sum(1, keepdims=True)
    # q is fp32 (|q| = 1 to 1e-7) and the reference normalises it; the oracle does not
    np.testing.assert_allclose(O, g[f"sp{ext}_O"], rtol=5e-6, atol=1e-9)
    np.testing.assert_allclose(dT, g[f"sp{ext}_dT"], rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(dQ, g[f"sp{ext}_dQ"], rtol=1e-5, atol=1e-6)
    assert np.all(O > 0)


@pytest.mark.parametrize("tag,ext", [("tv", 0), ("ext", 1), ("onlyref", 2)])
def test_pharm_extended_self_overlaps(golden, tag, ext):
    g = golden["pharm_ext"]
    ca, A = oa.center_anchors(g["al_A"], g["al_N"])
    cb, B = oa.center_anchors(g["al_B"], g["al_M"])
    va = oa.pharm_self_overlap(A, g["al_RV"], g["al_At"], g["al_N"], ext=ext)
    vb = oa.pharm_self_overlap(B, g["al_FV"], g["al_Bt"], g["al_M"], ext=ext)
    np.testing.assert_allclose(va, g[f"{tag}_VAA"], rtol=1e-5)
    np.testing.assert_allclose(vb, g[f"{tag}_VBB"], rtol=1e-5)


@pytest.mark.parametrize("tag,sim,ext,only", [("tv", "tversky", False, False),
                                              ("tvfit", "tversky_fit", False, False),
                                              ("ext", "tanimoto", True, False),
                                              ("onlyref", "tversky_ref", True, True)])
def test_align_pharm_tversky_and_extended(golden, tag, sim, ext, only):
    """Tversky tails and extended points in the pharmacophore fine loop: best scores match
    the reference's eager loop (the self copy reaches 1; Adam trajectories of two fp
    implementations separate chaotically, so the rest compare by best score)."""
    g = golden["pharm_ext"]
    sc, q, t = oa.align_pharm(g["al_A"], g["al_B"], g["al_RV"], g["al_FV"], g["al_At"],
                              g["al_Bt"], g["al_N"], g["al_M"], num_seeds=16, steps=40, lr=0.1,
                              similarity=sim, extended_points=ext, only_extended=only)
    ref = g[f"{tag}_score"]
    assert sc[0] > 0.99 and ref[0] > 0.99
    np.testing.assert_allclose(sc, ref, atol=2e-3)


def test_esp_comparison(golden):
    """ShaEP ESP comparison (esp_comparison_batch): masked Gaussian of the ESP difference."""
    g = golden["esp_combo"]
    S = oa.esp_compare(g["cmp_P"], g["cmp_PE"], g["cmp_A"], g["cmp_Q"], g["cmp_R"], g["cmp_N"],
                       g["cmp_M"], lam=0.001, probe_radius=1.0)
    np.testing.assert_allclose(S, g["cmp_S"], rtol=1e-6)
    assert np.all(S > 0) and np.all(S < g["cmp_N"])     # some points blocked, some kept


def _combo_args(g):
    return [g["al_" + k] for k in ("C1", "C2", "CN1", "CN2", "A1", "A2", "Q1", "Q2", "R1", "R2",
                                   "AN1", "AN2", "S1", "S2", "PE1", "PE2", "SN1", "SN2")]


def test_align_esp_combo(golden):
    """vol_and_surf_esp fine loop (shape-steered pose, combo score tracked every 5th step and
    on the last, as the reference's eager loop): best scores within 1e-4 of the reference's."""
    g = golden["esp_combo"]
    sc, q, t = oa.align_esp_combo(*_combo_args(g), alpha=0.81, lam=0.001, probe_radius=1.0,
                                  esp_weight=0.5, num_seeds=8, steps=30, lr=0.1, stride=5)
    np.testing.assert_allclose(sc, g["al_score"], atol=1e-4)
    assert sc[0] > 0.9
