"""GPU: the object-level drop-in (MoleculePairBatch / per-mode aligners) and screen().

Fake pairs carry only what the reference's aligners read (the pattern of the reference's
tests/test_cpu_pool.py ``_Pair`` and screen.py ``_FastPair``).  Every returned transform is
checked to reproduce the returned score with the fp64 scoring oracle."""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import synthetic as syn
from fast_shepherd_score_b200.batch import MoleculePairBatch

pytestmark = pytest.mark.gpu


class _Mol:
    def __init__(self, d):
        self.__dict__.update(d)


class _Pair:
    def __init__(self, ref, fit, device):
        self.ref_molec, self.fit_molec, self.device = _Mol(ref), _Mol(fit), device


def _mols(n, seed, surf=100):
    rng = np.random.default_rng(seed)
    ms = syn.shape_pharm_molecules(n, rng, atom_lo=15, atom_hi=40)
    for m, (p, c) in zip(ms, syn.sphere_clouds(rng, [surf] * n)):
        m["surf_pos"], m["surf_esp"] = p + m["atom_pos"].mean(0), c
        m["partial_charges"] = (0.3 * rng.standard_normal(len(m["atom_pos"]))).astype(np.float32)
    return ms


def _moved(m, rng):
    R = syn.random_rotation(rng).astype(np.float32)
    s = rng.standard_normal(3).astype(np.float32)
    out = dict(m)
    for k in ("atom_pos", "surf_pos", "pharm_ancs"):
        out[k] = (m[k] @ R.T + s).astype(np.float32)
    out["pharm_vecs"] = (m["pharm_vecs"] @ R.T).astype(np.float32)
    return out


def _apply(T, X):
    T = np.asarray(T, np.float64)
    return np.asarray(X, np.float64) @ T[:3, :3].T + T[:3, 3]


@pytest.fixture(scope="module")
def pairs_data():
    rng = np.random.default_rng(11)
    refs = _mols(8, 1)
    fits = _mols(8, 2)
    fits[0] = _moved(refs[0], rng)
    return refs, fits


def _pairs(refs, fits, dev):
    return [_Pair(r, f, dev) for r, f in zip(refs, fits)]


def test_align_with_vol_and_surf(pairs_data, cuda):
    from oracle import scores as osc
    refs, fits = pairs_data
    ps = _pairs(refs, fits, cuda)
    sc, al = MoleculePairBatch(ps).align_with_vol(num_repeats=20, max_num_steps=100,
                                                  return_aligned=True, backend="cuda")
    assert sc[0] > 0.99
    for p, s, r, a in zip(ps, sc, refs, al):
        assert p.sim_aligned_vol_noH == pytest.approx(s)
        assert abs(osc.shape_tanimoto(r["atom_pos"], a, 0.81) - s) < 2e-4
    sc, al = MoleculePairBatch(ps).align_with_surf(alpha=0.9, num_repeats=10, max_num_steps=60,
                                                   return_aligned=True)
    assert sc[0] > 0.98
    for s, r, a in zip(sc, refs, al):
        assert abs(osc.shape_tanimoto(r["surf_pos"], a, 0.9) - s) < 2e-4


def test_align_with_esp_modes(pairs_data, cuda):
    from oracle import scores as osc
    from fast_shepherd_score_b200.api import LAM_SCALING
    refs, fits = pairs_data
    ps = _pairs(refs, fits, cuda)
    sc, al = MoleculePairBatch(ps).align_with_surf_esp(alpha=0.9, lam=0.3, num_repeats=10,
                                                       max_num_steps=60, return_aligned=True)
    assert sc[0] > 0.98
    for p, s, r, f, a in zip(ps, sc, refs, fits, al):
        v = osc.esp_tanimoto(r["surf_pos"], a, r["surf_esp"], f["surf_esp"], 0.9, 0.3 * LAM_SCALING)
        assert abs(v - s) < 2e-4
    sc, al = MoleculePairBatch(ps).align_with_vol_esp(lam=0.3, num_repeats=10, max_num_steps=60,
                                                      return_aligned=True)
    for s, r, f, a in zip(sc, refs, fits, al):
        v = osc.esp_tanimoto(r["atom_pos"], a, r["partial_charges"], f["partial_charges"], 0.81, 0.3)
        assert abs(v - s) < 2e-4


def test_align_with_pharm_and_combos(pairs_data, cuda):
    from oracle import scores as osc
    refs, fits = pairs_data
    ps = _pairs(refs, fits, cuda)
    sc, ancs, vecs = MoleculePairBatch(ps).align_with_pharm(num_repeats=16, max_num_steps=80,
                                                            return_aligned=True)
    assert sc[0] > 0.99
    for s, r, f, a, v in zip(sc, refs, fits, ancs, vecs):
        t = osc.pharm_tanimoto(r["pharm_types"], f["pharm_types"], r["pharm_ancs"], a,
                               r["pharm_vecs"], v)
        assert abs(t - s) < 2e-4
    for mode, dl in (("vol_color", True), ("vol_pharm", False)):
        sc, al = getattr(MoleculePairBatch(ps), f"align_with_{mode}")(
            num_repeats=16, max_num_steps=80, return_aligned=True)
        assert sc[0] > 0.99
        for p, s, r, f, a in zip(ps, sc, refs, fits, al):
            T = getattr(p, f"transform_{mode}")
            fa = _apply(T, f["pharm_ancs"])
            fv = np.asarray(f["pharm_vecs"], np.float64) @ np.asarray(T, np.float64)[:3, :3].T
            v = osc.combo_score(r["atom_pos"], a, r["pharm_types"], f["pharm_types"],
                                r["pharm_ancs"], fa, r["pharm_vecs"], fv, directionless=dl)
            assert abs(v - s) < 2e-4, (mode, v, s)


def test_shared_reference_is_staged_once_with_identical_results(pairs_data, cuda):
    from fast_shepherd_score_b200 import aligners as A
    refs, fits = pairs_data
    q = torch.as_tensor(refs[0]["atom_pos"], device=cuda)
    shared = _pairs([refs[0]] * 8, fits, cuda)
    for p in shared:
        p._ref_xyz_t = q                      # one tensor object: the screen's query reuse
    copies = _pairs([refs[0]] * 8, fits, cuda)
    a = A._align_batch_vol(shared, steps_fine=40, num_repeats=10)
    b = A._align_batch_vol(copies, steps_fine=40, num_repeats=10)
    np.testing.assert_array_equal(a, b)


def test_backend_names(pairs_data, cuda):
    refs, fits = pairs_data
    b = MoleculePairBatch(_pairs(refs[:2], fits[:2], cuda))
    with pytest.raises(ValueError, match="shepherd_score"):
        b.align_with_vol(backend="numba")
    with pytest.raises(ValueError, match="unknown backend"):
        b.align_with_vol(backend="bogus")


@pytest.mark.parametrize("dtype", ["float32", "float16"])
def test_screen_finds_the_moved_copy(tmp_path, cuda, dtype):
    from fast_shepherd_score_b200.screen import ProfileStore, screen
    rng = np.random.default_rng(5)
    lib = _mols(60, 9)
    query = lib[17]
    lib[42] = _moved(query, rng)              # a rigidly moved copy of the query
    path = str(tmp_path / "lib")
    with ProfileStore.create(path, num_surf_points=100, modes=["surf_esp", "pharm"],
                             dtype=dtype, shard_size=25) as st:
        for m in lib:
            st.add_arrays(**m)
    store = ProfileStore.open(path)
    out = np.zeros(len(store))
    hits = screen(query, store, "surf_esp", top_k=5, num_repeats=10, max_num_steps=60,
                  scores_out=out)
    assert len(hits) == 5 and hits[0].score >= hits[-1].score
    assert {hits[0].id, hits[1].id} == {17, 42}
    assert hits[0].score > 0.97
    assert np.isclose(out.max(), hits[0].score)
    hits = screen(query, store, "pharm", top_k=3, num_repeats=16, max_num_steps=60)
    assert {hits[0].id, hits[1].id} == {17, 42} and hits[1].score > 0.97
