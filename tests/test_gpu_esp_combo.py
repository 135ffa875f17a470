"""vol_and_surf_esp (ShaEP-style combo) on the CUDA path against the reference fixtures
(tests/golden/esp_combo.npz) and the oracle.

The pose follows the shape gradient of the centres; the tracked score is
w * ESP similarity + (1 - w) * shape Tanimoto.  Step-1 scores (the seeds' own combo scores)
compare at fp32 rounding of the ESP sums (rtol 5e-5: rsqrt-based 1/d and fp32 sums against
the fp64 oracle); longer runs compare by best score."""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import align as al
from fast_shepherd_score_b200 import kernels as K
from fast_shepherd_score_b200 import synthetic as syn
from fast_shepherd_score_b200.batch import MoleculePairBatch
from fast_shepherd_score_b200.layout import CloudSet

from test_gpu_align import _t, assert_parity

pytestmark = pytest.mark.gpu
KEYS = ("C1", "C2", "CN1", "CN2", "A1", "A2", "Q1", "Q2", "R1", "R2", "AN1", "AN2", "S1", "S2",
        "PE1", "PE2", "SN1", "SN2")


def _args(g, cuda):
    a = {k: _t(g["al_" + k], cuda) for k in KEYS}
    return (a["A1"], a["A2"], a["C1"], a["C2"], a["S1"], a["S2"], a["Q1"], a["Q2"], a["PE1"],
            a["PE2"], a["R1"], a["R2"]), dict(
        N_real_centers=a["CN1"], M_real_centers=a["CN2"], N_real_atoms_w_H_1=a["AN1"],
        M_real_atoms_w_H_2=a["AN2"], N_real_surf_1=a["SN1"], M_real_surf_2=a["SN2"])


def test_combo_rows_track_oracle_stepwise(golden, cuda):
    from oracle import align as oa
    g = golden["esp_combo"]
    pos, cnt = _args(g, cuda)
    idx = torch.arange(len(g["al_CN1"]), dtype=torch.int32, device=cuda)
    sq, st = K.seeds(CloudSet.from_padded(pos[2], cnt["N_real_centers"]),
                     CloudSet.from_padded(pos[3], cnt["M_real_centers"]), idx, idx, 8)
    seeds = (sq.cpu().numpy(), st.cpu().numpy())
    for steps, tol in ((1, dict(rtol=5e-5, atol=1e-6)), (3, dict(rtol=0, atol=1e-4))):
        res = al.coarse_fine_esp_combo_align_many(*pos, alpha=0.81, lam=0.001, probe_radius=1.0,
                                                  esp_weight=0.5, steps_fine=steps, lr=0.1,
                                                  seeds=(sq, st), esp_stride=1, **cnt)
        rows = res.rows[0].cpu().numpy()
        *_, (best, _, _) = oa.align_esp_combo(*[g["al_" + k] for k in KEYS], steps=steps,
                                              lr=0.1, stride=1, seeds=seeds, return_rows=True)
        np.testing.assert_allclose(rows, best, **tol)


def test_combo_alignment_matches_reference(golden, cuda):
    """The reference's eager loop scores every 5th step; with the same stride the best scores
    match its fixtures (self copy first)."""
    g = golden["esp_combo"]
    pos, cnt = _args(g, cuda)
    sc, q, t = al.coarse_fine_esp_combo_align_many(*pos, alpha=0.81, lam=0.001,
                                                   probe_radius=1.0, esp_weight=0.5,
                                                   num_seeds=8, steps_fine=30, lr=0.1,
                                                   esp_stride=5, **cnt)
    sc = sc.cpu().numpy()
    assert_parity(sc, g["al_score"])
    assert sc[0] > 0.9


def test_dense_scoring_never_loses(golden, cuda):
    """Scoring every step visits a superset of the strided poses on the same trajectory."""
    g = golden["esp_combo"]
    pos, cnt = _args(g, cuda)
    kw = dict(alpha=0.81, lam=0.001, probe_radius=1.0, esp_weight=0.5, num_seeds=8,
              steps_fine=30, lr=0.1, **cnt)
    dense = al.coarse_fine_esp_combo_align_many(*pos, esp_stride=1, **kw)[0].cpu().numpy()
    sparse = al.coarse_fine_esp_combo_align_many(*pos, esp_stride=5, **kw)[0].cpu().numpy()
    assert np.all(dense >= sparse - 1e-6)


class _Conf:
    def __init__(self, x):
        self._x = x

    def GetPositions(self):
        return self._x


class _Mol:
    def __init__(self, x):
        self._c = _Conf(x)

    def GetConformer(self):
        return self._c


class _Molec:
    def __init__(self, m):
        self.atom_pos = m["centers"]
        self.surf_pos = m["surf"]
        self.surf_esp = m["surf_esp"]
        self.partial_charges = m["charges"]
        self.radii = m["radii"]
        self.mol = _Mol(m["atoms"].astype(np.float64))


class _Pair:
    def __init__(self, r, f):
        self.ref_molec, self.fit_molec = _Molec(r), _Molec(f)
        self.device = torch.device("cuda:0")


def test_object_api_matches_driver(cuda):
    """MoleculePairBatch.align_with_vol_and_surf_esp writes the reference's attributes and
    gives the driver's scores on the same molecules (and its legacy alias works)."""
    refs, fits = syn.esp_combo_pairs(6, seed=41)
    pairs = [_Pair(r, f) for r, f in zip(refs, fits)]
    scores, _ = MoleculePairBatch(pairs).align_with_vol_and_surf_esp(alpha=0.81, backend="cuda")
    assert all(hasattr(p, "transform_vol_and_surf_esp") for p in pairs)
    assert np.allclose([p.sim_aligned_vol_and_surf_esp for p in pairs], scores)
    assert np.all((scores > 0) & (scores <= 1))
    pad = lambda xs: torch.nn.utils.rnn.pad_sequence([torch.as_tensor(x) for x in xs],
                                                      batch_first=True).to(cuda)
    n = lambda xs: torch.tensor([len(x) for x in xs], device=cuda)
    get = lambda ms, k: [m[k] for m in ms]
    sc, _, _ = al.coarse_fine_esp_combo_align_many(
        pad(get(refs, "atoms")), pad(get(fits, "atoms")), pad(get(refs, "centers")),
        pad(get(fits, "centers")), pad(get(refs, "surf")), pad(get(fits, "surf")),
        pad(get(refs, "charges")), pad(get(fits, "charges")), pad(get(refs, "surf_esp")),
        pad(get(fits, "surf_esp")), pad(get(refs, "radii")), pad(get(fits, "radii")),
        alpha=0.81, lam=0.001, num_seeds=8, steps_fine=60, lr=0.1,
        N_real_centers=n(get(refs, "centers")), M_real_centers=n(get(fits, "centers")),
        N_real_atoms_w_H_1=n(get(refs, "atoms")), M_real_atoms_w_H_2=n(get(fits, "atoms")),
        N_real_surf_1=n(get(refs, "surf")), M_real_surf_2=n(get(fits, "surf")))
    np.testing.assert_allclose(scores, sc.cpu().numpy(), atol=1e-6)
    s2, _ = MoleculePairBatch(pairs).align_with_esp_combo(alpha=0.81, backend="cuda")
    np.testing.assert_allclose(s2, scores, atol=1e-6)


def test_screen_matches_driver(tmp_path, cuda):
    """screen() over a vol_and_surf_esp ProfileStore returns the driver's scores for every
    library molecule (same seeds, steps and tile; float32 store, no centring)."""
    from test_store import _combo_store
    from fast_shepherd_score_b200.screen import screen
    rng = np.random.default_rng(8)
    mols = syn.esp_combo_molecules(12, rng, surf_lo=120, surf_hi=120)
    st = _combo_store(str(tmp_path / "c.fss"), mols, shard_size=5)
    q = dict(atom_pos=mols[0]["centers"], surf_pos=mols[0]["surf"],
             surf_esp=mols[0]["surf_esp"], partial_charges=mols[0]["charges"],
             radii=mols[0]["radii"], centers_w_H=mols[0]["atoms"])
    out = np.zeros(len(mols), np.float32)
    hits = screen(q, st, mode="vol_and_surf_esp", do_center=False, top_k=5, scores_out=out,
                  num_repeats=8, max_num_steps=30, lr=0.1)
    assert len(hits) == 5 and hits[0].id == 0 and hits[0].score > 0.9
    pad = lambda xs: torch.nn.utils.rnn.pad_sequence([torch.as_tensor(x) for x in xs],
                                                      batch_first=True).to(cuda)
    n = lambda xs: torch.tensor([len(x) for x in xs], device=cuda)
    get = lambda k: [m[k] for m in mols]
    rep = lambda k: [mols[0][k]] * len(mols)
    sc, _, _ = al.coarse_fine_esp_combo_align_many(
        pad(rep("atoms")), pad(get("atoms")), pad(rep("centers")), pad(get("centers")),
        pad(rep("surf")), pad(get("surf")), pad(rep("charges")), pad(get("charges")),
        pad(rep("surf_esp")), pad(get("surf_esp")), pad(rep("radii")), pad(get("radii")),
        alpha=0.81, lam=0.001, num_seeds=8, steps_fine=30, lr=0.1,
        N_real_centers=n(rep("centers")), M_real_centers=n(get("centers")),
        N_real_atoms_w_H_1=n(rep("atoms")), M_real_atoms_w_H_2=n(get("atoms")),
        N_real_surf_1=n(rep("surf")), M_real_surf_2=n(get("surf")))
    np.testing.assert_allclose(out, sc.cpu().numpy(), atol=1e-5)
