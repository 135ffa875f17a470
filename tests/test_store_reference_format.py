"""ProfileStore format compatibility with shepherd_score's own store (CPU only).

The same molecules written by this package's writer and by the reference's writer
(shepherd_score/screen.py:317-606) give the same manifest and byte-identical shard arrays, for
both on-disk dtypes, with and without pre-centring, for a heavy-atom store (surfaces, ESP,
heavy charges, pharmacophores) and a store with hydrogens (vol_and_surf_esp); and each side
reads the other's store.  Skipped when the reference source tree is absent.
"""
import json
import os

import numpy as np
import pytest

from fast_shepherd_score_b200 import synthetic as syn
from fast_shepherd_score_b200.store import ProfileStore
from tests.reference_import import import_reference

REF = import_reference()
pytestmark = pytest.mark.skipif(REF is None, reason="reference source tree not present")


def _heavy_mols(n, seed=0, n_surf=64):
    rng = np.random.default_rng(seed)
    mols = syn.shape_pharm_molecules(n, rng)
    surf = syn.sphere_clouds(rng, [n_surf] * n)
    for m, (p, c) in zip(mols, surf):
        m["surf_pos"], m["surf_esp"] = p + rng.standard_normal(3).astype(np.float32), c
        m["atom_pos"] = m["atom_pos"] + rng.standard_normal(3).astype(np.float32)
        m["partial_charges"] = (0.2 * rng.standard_normal(len(m["atom_pos"]))).astype(np.float32)
    return mols


def _h_mols(n, seed=1):
    rng = np.random.default_rng(seed)
    out = []
    for m in syn.esp_combo_molecules(n, rng, surf_lo=80, surf_hi=80):
        # the heavy atoms are the first rows of the all-atom list
        out.append(dict(atom_pos=m["centers"], surf_pos=m["surf"], surf_esp=m["surf_esp"],
                        partial_charges=m["charges"], radii=m["radii"], centers_w_H=m["atoms"],
                        nonH_atoms_idx=np.arange(len(m["centers"]))))
    return out


def _write_both(tmp_path, mols, modes, dtype, pre, shard_size=7, n_surf=64):
    _, _, ref_screen = REF
    a, b = str(tmp_path / "ours"), str(tmp_path / "theirs")
    with ProfileStore.create(a, num_surf_points=n_surf, modes=modes, dtype=dtype,
                             shard_size=shard_size, pre_centered=pre) as st:
        for m in mols:
            st.add_arrays(**m)
    with ref_screen.ProfileStore.create(b, num_surf_points=n_surf, modes=modes, dtype=dtype,
                                        shard_size=shard_size, pre_centered=pre) as st:
        for m in mols:
            st.add_profile(ref_screen.MoleculeProfile(**m))
    return a, b


def _same_store(a, b):
    ma = json.load(open(os.path.join(a, "manifest.json")))
    mb = json.load(open(os.path.join(b, "manifest.json")))
    assert ma == mb
    for sh in ma["shards"]:
        with np.load(os.path.join(a, sh["name"])) as x, np.load(os.path.join(b, sh["name"])) as y:
            assert sorted(x.files) == sorted(y.files)
            for k in x.files:
                assert x[k].dtype == y[k].dtype, k
                np.testing.assert_array_equal(x[k], y[k], err_msg=k)


@pytest.mark.parametrize("dtype", ["float16", "float32"])
@pytest.mark.parametrize("pre", [True, False])
def test_heavy_store_same_bytes_as_reference(tmp_path, dtype, pre):
    mols = _heavy_mols(17)
    a, b = _write_both(tmp_path, mols, ["surf_esp", "vol_esp", "pharm"], dtype, pre)
    _same_store(a, b)


@pytest.mark.parametrize("pre", [True, False])
def test_store_with_hydrogens_same_bytes_as_reference(tmp_path, pre):
    mols = _h_mols(9)
    a, b = _write_both(tmp_path, mols, ["vol_and_surf_esp"], "float32", pre, shard_size=4,
                       n_surf=80)
    _same_store(a, b)


def test_heavy_centres_column(tmp_path):
    """A molecule whose heavy Gaussian centres are not its atom_pos rows (the all-atom list
    is not heavy-first) makes both writers add heavy_off / xyz_noH, identically."""
    mols = _h_mols(6, seed=2)
    for m in mols[:2]:
        m["nonH_atoms_idx"] = m["nonH_atoms_idx"][::-1].copy()
    a, b = _write_both(tmp_path, mols, ["vol_and_surf_esp", "vol_esp"], "float16", True,
                       shard_size=4, n_surf=80)
    _same_store(a, b)
    with np.load(os.path.join(a, "shard_00000.npz")) as x:
        assert "xyz_noH" in x.files and "heavy_off" in x.files
    with np.load(os.path.join(a, "shard_00001.npz")) as x:
        assert "xyz_noH" not in x.files


def test_each_side_reads_the_other(tmp_path):
    _, _, ref_screen = REF
    mols = _heavy_mols(11, seed=4)
    a, b = _write_both(tmp_path, mols, ["surf_esp", "vol_esp", "pharm"], "float16", True,
                       shard_size=5)
    for ours_path, theirs_path in ((a, b), (b, a)):
        ours = ProfileStore.open(theirs_path)
        theirs = ref_screen.ProfileStore.open(ours_path)
        assert len(ours) == len(theirs) == 11 and ours.num_shards == theirs.num_shards == 3
        for mode in ("vol", "surf_esp", "vol_esp", "pharm", "vol_and_surf_esp", "surf"):
            assert ours.supports(mode) == theirs.supports(mode), mode
        got = [p for shard in ours.iter_shards() for p in shard]
        want = [p for shard in theirs.iter_shards() for p in shard]
        for g, w in zip(got, want):
            assert g.id == w.id
            for attr in ("atom_pos", "surf_pos", "surf_esp", "partial_charges", "pharm_types",
                         "pharm_ancs", "pharm_vecs"):
                np.testing.assert_array_equal(np.asarray(getattr(g, attr), np.float32),
                                              np.asarray(getattr(w, attr), np.float32), attr)
