"""Tversky similarity and extended pharmacophore points on the CUDA path, against the
reference's fixtures (tests/golden/pharm_ext.npz) and the oracle.

Extended points follow the typed overlap the reference's batched fine loop differentiates
(acceptor/donor extended, halogen cosine-weighted); Tversky scores are min(O/D, 1) with
D = sigma V_AA + (1 - sigma) V_BB."""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import align as al
from fast_shepherd_score_b200 import kernels as K
from fast_shepherd_score_b200.layout import CloudSet, PharmSet

from test_gpu_align import _t

pytestmark = pytest.mark.gpu
CASES = [("tv", "tversky", False, False), ("tvfit", "tversky_fit", False, False),
         ("ext", "tanimoto", True, False), ("onlyref", "tversky_ref", True, True)]


def _sets(g, cuda, centre=True):
    from oracle import align as oa
    A, B = g["al_A"], g["al_B"]
    if centre:
        _, A = oa.center_anchors(A, g["al_N"])
        _, B = oa.center_anchors(B, g["al_M"])
    ref = PharmSet.from_padded(_t(A, cuda), _t(g["al_At"], cuda), _t(g["al_RV"], cuda),
                               _t(g["al_N"], cuda))
    fit = PharmSet.from_padded(_t(B, cuda), _t(g["al_Bt"], cuda), _t(g["al_FV"], cuda),
                               _t(g["al_M"], cuda))
    return ref, fit, A, B


@pytest.mark.parametrize("tag,ext", [("tv", 0), ("ext", 1), ("onlyref", 2)])
def test_extended_self_overlaps_match_reference(golden, cuda, tag, ext):
    g = golden["pharm_ext"]
    ref, fit, _, _ = _sets(g, cuda, centre=False)
    np.testing.assert_allclose(K.pharm_self_overlap(ref, True, ext).cpu().numpy(),
                               g[f"{tag}_VAA"], rtol=1e-5)
    np.testing.assert_allclose(K.pharm_self_overlap(fit, True, ext).cpu().numpy(),
                               g[f"{tag}_VBB"], rtol=1e-5)


@pytest.mark.parametrize("tag,sim,ext,only", CASES)
def test_pharm_variants_track_oracle_stepwise(golden, cuda, tag, sim, ext, only):
    """Every start's step-1 score equals the oracle's to fp32 rounding; after 3 steps the
    trajectories still agree to 5e-5."""
    from oracle import align as oa
    g = golden["pharm_ext"]
    ref, fit, A, B = _sets(g, cuda)
    idx = torch.arange(len(g["al_N"]), dtype=torch.int32, device=cuda)
    sq, st = K.seeds(CloudSet.from_padded(_t(A, cuda), _t(g["al_N"], cuda)),
                     CloudSet.from_padded(_t(B, cuda), _t(g["al_M"], cuda)), idx, idx, 16)
    seeds = (sq.cpu().numpy(), st.cpu().numpy())
    code = al.extended_code(ext, only)
    for steps in (1, 3):
        res = al.align_packed("pharm", ref_ph=ref, fit_ph=fit, pair_ref=idx, pair_fit=idx,
                              seed_q=sq, seed_t=st, steps=steps, lr=0.1, similarity=sim,
                              pharm_extended=code)
        rows = res.rows[0].cpu().numpy()
        *_, (best, _, _) = oa.align_pharm(g["al_A"], g["al_B"], g["al_RV"], g["al_FV"],
                                          g["al_At"], g["al_Bt"], g["al_N"], g["al_M"],
                                          seeds=seeds, steps=steps, lr=0.1, similarity=sim,
                                          extended_points=ext, only_extended=only,
                                          return_rows=True)
        tol = dict(rtol=2e-5, atol=1e-6) if steps == 1 else dict(rtol=0, atol=5e-5)
        np.testing.assert_allclose(rows, best, **tol)


@pytest.mark.parametrize("tag,sim,ext,only", CASES)
def test_pharm_variants_match_reference(golden, cuda, tag, sim, ext, only):
    """Batched alignment with the reference's driver signature: best scores within the
    oracle's own tolerance of the reference (2e-3; the self copy reaches 1), and the pose
    reproduces the score in the original frames."""
    g = golden["pharm_ext"]
    args = [_t(g[k], cuda) for k in ("al_A", "al_B", "al_RV", "al_FV", "al_At", "al_Bt")]
    sc, q, t = al.coarse_fine_pharm_align_many(
        *args, similarity=sim, extended_points=ext, only_extended=only, num_seeds=16,
        steps_fine=40, lr=0.1, N_real=_t(g["al_N"], cuda), M_real=_t(g["al_M"], cuda))
    sc = sc.cpu().numpy()
    assert sc[0] > 0.99
    np.testing.assert_allclose(sc, g[f"{tag}_score"], atol=2e-3)
    # the returned pose reproduces the score in the original frames
    from oracle import align as oa
    R = al._quat_rot(q).cpu().numpy()
    tt = t.cpu().numpy()
    Bw = np.einsum("bij,bnj->bni", R, g["al_B"]) + tt[:, None, :]
    Vw = np.einsum("bij,bnj->bni", R, g["al_FV"])
    qi = np.zeros((len(sc), 4), np.float32)
    qi[:, 0] = 1
    O, _, _ = oa.pharm_grad(g["al_A"], Bw, g["al_RV"], Vw, g["al_At"], g["al_Bt"], qi,
                            np.zeros((len(sc), 3), np.float32), g["al_N"], g["al_M"],
                            ext=al.extended_code(ext, only), need_grad=False)
    VAA, VBB = g[f"{tag}_VAA"].astype(np.float64), g[f"{tag}_VBB"].astype(np.float64)
    if sim == "tanimoto":
        s = O / (VAA + VBB - O)
    else:
        sg = al.TVERSKY_SIGMA[sim]
        s = np.minimum(O / (sg * VAA + (1 - sg) * VBB), 1.0)
    np.testing.assert_allclose(s, sc, atol=2e-4)


def test_tversky_rejected_outside_pharm(cuda):
    ref = CloudSet.from_arrays([np.zeros((3, 3), np.float32)], device=cuda)
    idx = torch.zeros(1, dtype=torch.int32, device=cuda)
    sq = torch.tensor([[[1.0, 0, 0, 0]]], device=cuda)
    st = torch.zeros(1, 1, 3, device=cuda)
    with pytest.raises(ValueError):
        al.align_packed("shape", ref=ref, fit=ref, pair_ref=idx, pair_fit=idx, seed_q=sq,
                        seed_t=st, steps=1, lr=0.1, similarity="tversky")


def test_interleaved_and_out_of_range_types_track_oracle(cuda):
    """The fused kernel stages the reference features grouped by type and visits only a fit
    feature's own type; features whose types are interleaved, repeated or out of the 9-entry
    table (read as Dummy) give the oracle's rows after 1 and 3 steps, in the pharmacophore
    and the shape + pharmacophore modes."""
    from oracle import align as oa
    from fast_shepherd_score_b200 import synthetic as syn
    rng = np.random.default_rng(17)
    refs, fits = syn.shape_pharm_pairs(12, seed=17)
    pool = np.array([-1, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 12])
    for m in refs + fits:
        m["pharm_types"] = rng.choice(pool, size=len(m["pharm_types"])).astype(np.int64)
    g = lambda ms, k: [m[k] for m in ms]

    def pad(xs, fill=0.0, dtype=np.float32):
        n = np.array([len(x) for x in xs])
        out = np.full((len(xs), int(n.max())) + np.asarray(xs[0]).shape[1:], fill, dtype)
        for i, x in enumerate(xs):
            out[i, :len(x)] = x
        return out, n

    table = lambda t: np.where((t < 0) | (t > 8), 8, t)   # out of the table reads as Dummy
    A, N = pad(g(refs, "pharm_ancs")); B, M = pad(g(fits, "pharm_ancs"))
    RV, _ = pad(g(refs, "pharm_vecs")); FV, _ = pad(g(fits, "pharm_vecs"))
    At, _ = pad([table(t) for t in g(refs, "pharm_types")], 8, np.int64)
    Bt, _ = pad([table(t) for t in g(fits, "pharm_types")], 8, np.int64)
    mk = lambda ms: PharmSet.from_arrays(g(ms, "pharm_types"), g(ms, "pharm_ancs"),
                                         g(ms, "pharm_vecs"), device=cuda)
    ref_ph, fit_ph = mk(refs), mk(fits)
    idx = torch.arange(12, dtype=torch.int32, device=cuda)
    # pharmacophore mode: seeds of the centred anchors, as the driver takes them
    _, Ac = oa.center_anchors(A, N)
    _, Bc = oa.center_anchors(B, M)
    sq, st = K.seeds(CloudSet.from_padded(_t(Ac, cuda), _t(N, cuda)),
                     CloudSet.from_padded(_t(Bc, cuda), _t(M, cuda)), idx, idx, 12)
    seeds = (sq.cpu().numpy(), st.cpu().numpy())
    # the raw types (out-of-table ones included) go to the device; the set reads them as Dummy
    rawt = lambda ms: pad(g(ms, "pharm_types"), 8, np.int64)[0]
    rph = PharmSet.from_padded(_t(Ac, cuda), _t(rawt(refs), cuda), _t(RV, cuda), _t(N, cuda))
    fph = PharmSet.from_padded(_t(Bc, cuda), _t(rawt(fits), cuda), _t(FV, cuda), _t(M, cuda))
    for steps in (1, 3):
        tol = dict(rtol=2e-5, atol=1e-6) if steps == 1 else dict(rtol=0, atol=5e-5)
        *_, (best, _, _) = oa.align_pharm(A, B, RV, FV, At, Bt, N, M, seeds=seeds, steps=steps,
                                          lr=0.1, return_rows=True)
        res = al.align_packed("pharm", ref_ph=rph, fit_ph=fph, pair_ref=idx, pair_fit=idx,
                              seed_q=sq, seed_t=st, steps=steps, lr=0.1)
        np.testing.assert_allclose(res.rows[0].cpu().numpy(), best, **tol)
    # shape + pharmacophore (the clouds' own frames, seeds on the atoms)
    X, XN = pad(g(refs, "atom_pos")); Y, YM = pad(g(fits, "atom_pos"))
    ref = CloudSet.from_arrays(g(refs, "atom_pos"), device=cuda)
    fit = CloudSet.from_arrays(g(fits, "atom_pos"), device=cuda)
    sq, st = K.seeds(ref, fit, idx, idx, 12)
    seeds = (sq.cpu().numpy(), st.cpu().numpy())
    for steps in (1, 3):
        tol = dict(rtol=2e-5, atol=1e-6) if steps == 1 else dict(rtol=0, atol=5e-5)
        *_, (best, _, _) = oa.align_combo(X, Y, XN, YM, A, B, RV, FV, At, Bt, N, M, alpha=0.81,
                                          w=0.5, directional=True, steps=steps, lr=0.1,
                                          seeds=seeds, return_rows=True)
        res = al.align_packed("shape_pharm", ref=ref, fit=fit, ref_ph=ref_ph, fit_ph=fit_ph,
                              pair_ref=idx, pair_fit=idx, seed_q=sq, seed_t=st, steps=steps,
                              lr=0.1, alpha=0.81, color_weight=0.5)
        np.testing.assert_allclose(res.rows[0].cpu().numpy(), best, **tol)
