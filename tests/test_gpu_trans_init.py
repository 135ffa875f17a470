"""Translation-seeded starts (trans_init=True) on the CUDA path against the reference's
fixtures (tests/golden/trans_init.npz) and the oracle: the one-step scores of the legacy grid
poses, the full coarse grid + top-k + fine alignments of the four drivers, and the object API."""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import align as al
from fast_shepherd_score_b200 import kernels as K
from fast_shepherd_score_b200.batch import MoleculePairBatch
from fast_shepherd_score_b200.layout import CloudSet

from test_gpu_align import _t, assert_parity

pytestmark = pytest.mark.gpu
COMBO_KEYS = ("A1", "A2", "C1", "C2", "S1", "S2", "Q1", "Q2", "PE1", "PE2", "R1", "R2")


def _run(g, tag, cuda, **kw):
    """The CUDA driver of `tag` with the fixture's translation centres, 30 fine steps."""
    x = lambda k: _t(g[k], cuda)
    common = dict(num_repeats_per_trans=10, topk=30, steps_fine=30, lr=0.1, **kw)
    if tag == "esp":
        ref = CloudSet.from_padded(x("esp_A"), x("esp_N"), x("esp_CA"))
        fit = CloudSet.from_padded(x("esp_B"), x("esp_M"), x("esp_CB"))
        lam = float(g["esp_lam"])
        VAA = K.self_overlap(ref, 0.81, True, lam)
        VBB = K.self_overlap(fit, 0.81, True, lam)
        return al.coarse_fine_esp_align_many(
            x("esp_A"), x("esp_B"), x("esp_CA"), x("esp_CB"), VAA, VBB, alpha=0.81, lam=lam,
            trans_centers=x("esp_TC"), trans_centers_real=x("esp_TN"), N_real=x("esp_N"),
            M_real=x("esp_M"), **common)
    if tag == "pharm":
        args = [x(f"pharm_{k}") for k in ("A", "B", "RV", "FV", "At", "Bt")]
        return al.coarse_fine_pharm_align_many(
            *args, trans_centers=x("pharm_A"), trans_centers_real=x("pharm_N"),
            N_real=x("pharm_N"), M_real=x("pharm_M"), **common)
    if tag == "color":
        VAA = K.self_overlap(CloudSet.from_padded(x("color_A"), x("color_N")), 0.81)
        VBB = K.self_overlap(CloudSet.from_padded(x("color_B"), x("color_M")), 0.81)
        return al.coarse_fine_vol_color_align_many(
            x("color_A"), x("color_B"), x("color_At"), x("color_Bt"), x("pharm_A"),
            x("pharm_B"), VAA, VBB, alpha=0.81, color_weight=0.5, trans_centers=x("color_A"),
            trans_centers_real=x("color_N"), N_real_centers=x("color_N"),
            M_real_centers=x("color_M"), N_real_pharm=x("pharm_N"), M_real_pharm=x("pharm_M"),
            **common)
    return al.coarse_fine_esp_combo_align_many(
        *[x("combo_" + k) for k in COMBO_KEYS], alpha=0.81, lam=0.001, probe_radius=1.0,
        esp_weight=0.5, trans_centers=x("combo_C1"), trans_centers_real=x("combo_CN1"),
        N_real_centers=x("combo_CN1"), M_real_centers=x("combo_CN2"),
        N_real_atoms_w_H_1=x("combo_AN1"), M_real_atoms_w_H_2=x("combo_AN2"),
        N_real_surf_1=x("combo_SN1"), M_real_surf_2=x("combo_SN2"), esp_stride=5, **common)


@pytest.mark.parametrize("tag", ["esp", "pharm", "color", "combo"])
def test_trans_init_matches_reference(golden, cuda, tag):
    """Ragged grids of one batch (5 + 10 x centres poses per pair, padded and masked), scored
    once, top 30 refined for 30 steps: best scores at the reference's (pair 0 of surf_esp is a
    rotated copy and reaches 1)."""
    g = golden["trans_init"]
    sc = _run(g, tag, cuda)[0].cpu().numpy()
    assert_parity(sc, g[f"{tag}_score"])
    if tag == "esp":
        assert sc[0] > 0.99


def test_grid_poses_scored_like_the_oracle(golden, cuda):
    """A one-step launch over the reference's legacy grid records each pose's own score:
    every row within fp32 rounding of the oracle's."""
    from oracle import align as oa
    g = golden["trans_init"]
    x = lambda k: _t(g[k], cuda)
    ref = CloudSet.from_padded(x("esp_A"), x("esp_N"), x("esp_CA"))
    fit = CloudSet.from_padded(x("esp_B"), x("esp_M"), x("esp_CB"))
    idx = torch.arange(len(g["esp_N"]), dtype=torch.int32, device=cuda)
    lam = float(g["esp_lam"])
    res = al.align_packed("esp", ref=ref, fit=fit, pair_ref=idx, pair_fit=idx,
                          seed_q=x("esp_GQ"), seed_t=x("esp_GT"), steps=1, lr=0.1, lam=lam)
    *_, (best, _, _) = oa.align_esp(*[g[f"esp_{k}"] for k in ("A", "B", "CA", "CB", "N", "M")],
                                    alpha=0.81, lam=lam, seeds=(g["esp_GQ"], g["esp_GT"]),
                                    steps=1, return_rows=True)
    np.testing.assert_allclose(res.rows[0].cpu().numpy(), best, rtol=2e-5, atol=1e-6)


class _Molec:
    def __init__(self, atoms, surf, esp):
        self.atom_pos, self.surf_pos, self.surf_esp = atoms, surf, esp


class _Pair:
    def __init__(self, r, f):
        self.ref_molec, self.fit_molec = r, f
        self.device = torch.device("cuda:0")


def test_object_api_trans_init(golden, cuda):
    """align_with_surf_esp(trans_init=True) uses the reference atoms as translation centres and
    gives the driver's result; vol/surf accept and ignore the flag as the reference's fast
    path does."""
    g = golden["trans_init"]
    K = len(g["esp_N"])
    mols = []
    for i in range(K):
        n, m, c = g["esp_N"][i], g["esp_M"][i], g["esp_TN"][i]
        r = _Molec(g["esp_TC"][i, :c], g["esp_A"][i, :n], g["esp_CA"][i, :n])
        f = _Molec(g["esp_TC"][i, :c] + 1.0, g["esp_B"][i, :m], g["esp_CB"][i, :m])
        mols.append((r, f))
    pairs = [_Pair(r, f) for r, f in mols]
    lam = float(g["esp_lam"]) / al.LAM_SCALING
    sc, _ = MoleculePairBatch(pairs).align_with_surf_esp(alpha=0.81, lam=lam, trans_init=True,
                                                         max_num_steps=30, backend="cuda")
    assert all(hasattr(p, "transform_surf_esp") for p in pairs)
    ref_sc = _run(g, "esp", cuda)[0].cpu().numpy()
    np.testing.assert_allclose(sc, ref_sc, atol=1e-5)
    sv, _ = MoleculePairBatch(pairs).align_with_vol(trans_init=True, max_num_steps=5,
                                                    backend="cuda")
    assert np.all(np.isfinite(sv))


def test_screen_trans_init_matches_driver(tmp_path, cuda):
    """screen(trans_init=True) takes the query's atoms as translation centres and gives the
    driver's translation-seeded scores for every library molecule (float32 store, no
    centring, one shard boundary inside the library).  The top-k of the coarse grid is
    sensitive to rounding among near-equal poses, so both sides see the same coordinates."""
    from fast_shepherd_score_b200.screen import ProfileStore, screen
    from test_store import _mols
    mols = _mols(9, seed=4)
    path = str(tmp_path / "lib")
    with ProfileStore.create(path, num_surf_points=64, modes=["surf_esp"], dtype="float32",
                             shard_size=5, pre_centered=False) as st:
        for m in mols:
            st.add_arrays(**m)
    store = ProfileStore.open(path)
    q = mols[0]
    out = np.zeros(len(mols), np.float32)
    screen(q, store, "surf_esp", do_center=False, alpha=0.81, top_k=3, scores_out=out,
           trans_init=True, max_num_steps=20, lr=0.1)
    pad = lambda xs: torch.nn.utils.rnn.pad_sequence([torch.as_tensor(x) for x in xs],
                                                      batch_first=True).to(cuda)
    n = lambda xs: torch.tensor([len(x) for x in xs], device=cuda)
    A = pad([q["surf_pos"]] * len(mols))
    B = pad([m["surf_pos"] for m in mols])
    CA = pad([q["surf_esp"]] * len(mols))
    CB = pad([m["surf_esp"] for m in mols])
    lam = 0.3 * al.LAM_SCALING
    VAA = K.self_overlap(CloudSet.from_padded(A, n([q["surf_pos"]] * len(mols)), CA), 0.81,
                         True, lam)
    VBB = K.self_overlap(CloudSet.from_padded(B, n([m["surf_pos"] for m in mols]), CB), 0.81,
                         True, lam)
    sc, _, _ = al.coarse_fine_esp_align_many(
        A, B, CA, CB, VAA, VBB, alpha=0.81, lam=lam, trans_centers=pad([q["atom_pos"]] * len(mols)),
        steps_fine=20, lr=0.1, N_real=n([q["surf_pos"]] * len(mols)),
        M_real=n([m["surf_pos"] for m in mols]))
    np.testing.assert_allclose(out, sc.cpu().numpy(), atol=1e-5)
    assert out[0] > 0.99


@pytest.mark.parametrize("mode", ["pharm", "vol_color"])
def test_object_api_trans_init_pharm_modes(cuda, mode):
    """align_with_pharm / align_with_vol_color(trans_init=True): the reference's centres
    (anchors for pharm, atoms for vol_color) and the drivers' translation-seeded results."""
    from test_gpu_api import _mols, _pairs
    refs, fits = _mols(6, 21), _mols(6, 22)
    pairs = _pairs(refs, fits, cuda)
    b = MoleculePairBatch(pairs)
    pad = lambda xs, dt=None: torch.nn.utils.rnn.pad_sequence(
        [torch.as_tensor(np.asarray(x)) for x in xs], batch_first=True).to(cuda)
    n = lambda xs: torch.tensor([len(x) for x in xs], device=cuda)
    g = lambda ms, k: [m[k] for m in ms]
    kw = dict(num_repeats_per_trans=10, topk=30, steps_fine=20, lr=0.1)
    if mode == "pharm":
        sc = b.align_with_pharm(trans_init=True, max_num_steps=20, backend="cuda")[0]
        ref, _, _ = al.coarse_fine_pharm_align_many(
            pad(g(refs, "pharm_ancs")), pad(g(fits, "pharm_ancs")), pad(g(refs, "pharm_vecs")),
            pad(g(fits, "pharm_vecs")), pad(g(refs, "pharm_types")), pad(g(fits, "pharm_types")),
            trans_centers=pad(g(refs, "pharm_ancs")), trans_centers_real=n(g(refs, "pharm_ancs")),
            N_real=n(g(refs, "pharm_ancs")), M_real=n(g(fits, "pharm_ancs")), **kw)
    else:
        sc = b.align_with_vol_color(trans_init=True, max_num_steps=20, backend="cuda")[0]
        A, B = pad(g(refs, "atom_pos")), pad(g(fits, "atom_pos"))
        NA, NB = n(g(refs, "atom_pos")), n(g(fits, "atom_pos"))
        VAA = K.self_overlap(CloudSet.from_padded(A, NA), 0.81)
        VBB = K.self_overlap(CloudSet.from_padded(B, NB), 0.81)
        tp = lambda ms: pad([np.asarray(t, np.int64) for t in g(ms, "pharm_types")])
        ref, _, _ = al.coarse_fine_vol_color_align_many(
            A, B, tp(refs), tp(fits), pad(g(refs, "pharm_ancs")), pad(g(fits, "pharm_ancs")),
            VAA, VBB, alpha=0.81, color_weight=0.5, trans_centers=A, trans_centers_real=NA,
            N_real_centers=NA, M_real_centers=NB, N_real_pharm=n(g(refs, "pharm_ancs")),
            M_real_pharm=n(g(fits, "pharm_ancs")), **kw)
    np.testing.assert_allclose(np.asarray(sc, np.float32), ref.cpu().numpy(), atol=1e-5)
