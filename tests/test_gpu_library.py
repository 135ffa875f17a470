"""GPU: float16 libraries widened inside the kernels, and the server fed from a ProfileStore.

* A float16 ProfileStore loaded into HBM as float16 (8-byte points) and aligned with the
  kernels' in-staging widening gives bit-identical scores and poses to the same store widened
  to float32 by a torch cast before the launch -- for shape + directional pharmacophores,
  colour, shape only, and the seed and self-overlap kernels that read the library too.
* ``ScreenServer.from_store`` over a float16 store answers a request with the same top-K as
  ``screen()`` streaming that store (same tile, so the same arithmetic).
"""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import align as al
from fast_shepherd_score_b200 import kernels as K
from fast_shepherd_score_b200 import synthetic as syn
from fast_shepherd_score_b200.library import Library
from fast_shepherd_score_b200.screen import screen
from fast_shepherd_score_b200.server import ScreenServer
from fast_shepherd_score_b200.store import ProfileStore

pytestmark = pytest.mark.gpu
N_LIB = 700


@pytest.fixture(scope="module")
def store16(tmp_path_factory):
    rng = np.random.default_rng(17)
    mols = syn.shape_pharm_molecules(N_LIB, rng)
    path = str(tmp_path_factory.mktemp("lib") / "lib16")
    with ProfileStore.create(path, num_surf_points=64, modes=["vol_color", "pharm"],
                             dtype="float16", shard_size=256, pre_centered=True) as st:
        for i, m in enumerate(mols):
            st.add_arrays(id=1000 + i, **m)
    return ProfileStore.open(path), mols


def _query(mols, i):
    m = mols[i]
    return {k: m[k] for k in ("atom_pos", "pharm_types", "pharm_ancs", "pharm_vecs")}


@pytest.mark.parametrize("mode", ["shape_pharm", "shape_color", "shape"])
def test_f16_library_matches_f32_widened(store16, cuda, mode):
    store, mols = store16
    vectors = mode == "shape_pharm"
    lib16 = Library.from_store(store, cuda, vectors=vectors)
    lib32 = Library.from_store(store, cuda, vectors=vectors, widen=True)
    assert lib16.atoms.pts.dtype == torch.float16 and lib32.atoms.pts.dtype == torch.float32
    assert lib16.nbytes < 0.6 * lib32.nbytes
    assert torch.equal(lib16.atoms.pts.float(), lib32.atoms.pts)
    q = _query(mols, 3)
    from fast_shepherd_score_b200.layout import CloudSet, PharmSet
    qa = CloudSet.from_arrays([q["atom_pos"] - q["atom_pos"].mean(0)], device=cuda)
    qp = PharmSet.from_arrays([q["pharm_types"]], [q["pharm_ancs"] - q["atom_pos"].mean(0)],
                              [q["pharm_vecs"]] if vectors else None, device=cuda)
    pr = torch.zeros(N_LIB, dtype=torch.int32, device=cuda)
    pf = torch.arange(N_LIB, dtype=torch.int32, device=cuda)
    out = []
    for lib in (lib16, lib32):
        sq, st = K.seeds(qa, lib.atoms, pr, pf, 10)
        fs = K.self_overlap(lib.atoms, 0.81)
        fsp = K.pharm_self_overlap(lib.pharm, vectors) if mode != "shape" else None
        res = al.align_packed(mode, ref=qa, fit=lib.atoms, ref_ph=qp if mode != "shape" else None,
                              fit_ph=lib.pharm if mode != "shape" else None, pair_ref=pr,
                              pair_fit=pf, seed_q=sq, seed_t=st, steps=25, lr=0.1,
                              fit_self=fs, fit_self_ph=fsp, lanes_per_pose=4, chunks=1)
        out.append((sq, st, fs, fsp) + tuple(res))
    for a, b in zip(*out):
        if a is not None:
            assert torch.equal(a, b)


def test_server_from_f16_store_matches_screen(store16, cuda):
    store, mols = store16
    q = _query(mols, 42)
    kw = dict(num_repeats=8, max_num_steps=30, lanes_per_pose=8)
    want = screen(q, store, "vol_pharm", top_k=25, **kw)
    with ScreenServer.from_store(store, cuda, mode="vol_pharm", starts=8, steps=30,
                                 lanes_per_pose=8, max_pairs_per_launch=300,
                                 slice_pairs=128) as srv:
        assert srv.library.dtype == torch.float16
        got = srv.submit(q, top_k=25).result(timeout=300)
        part = srv.submit(q, np.arange(100, 400), top_k=5).result(timeout=300)
    key = lambda hits: sorted((-h.score, h.id) for h in hits)
    assert key(got) == key(want)
    assert got[0].id == 1042 and got[0].score > 0.999
    sub = sorted((h for h in want if 1100 <= h.id < 1400), key=lambda h: (-h.score, h.id))
    assert [h.id for h in part][:len(sub[:5])] == [h.id for h in sub[:5]]
