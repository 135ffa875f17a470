"""ProfileStore format (CPU): round trip, fp16 loss bound, manifest guards, mode support."""
import json
import os

import numpy as np
import pytest

from fast_shepherd_score_b200 import synthetic as syn
from fast_shepherd_score_b200.screen import ProfileStore, _center_shard, _centred_query


def _mols(n, seed=0):
    rng = np.random.default_rng(seed)
    mols = syn.shape_pharm_molecules(n, rng)
    surf = syn.sphere_clouds(rng, [64] * n)
    for m, (p, c) in zip(mols, surf):
        m["surf_pos"], m["surf_esp"] = p, c
        m["partial_charges"] = (0.2 * rng.standard_normal(len(m["atom_pos"]))).astype(np.float32)
    return mols


@pytest.mark.parametrize("dtype", ["float32", "float16"])
def test_round_trip(tmp_path, dtype):
    mols = _mols(23)
    path = str(tmp_path / "lib.fss")
    with ProfileStore.create(path, num_surf_points=64, modes=["surf_esp", "vol_esp", "pharm"],
                             dtype=dtype, shard_size=10, pre_centered=False) as st:
        for m in mols:
            st.add_arrays(**m)
    st = ProfileStore.open(path)
    assert len(st) == 23 and st.num_shards == 3
    assert st.supports("surf_esp") and st.supports("pharm") and st.supports("vol_esp")
    assert st.supports("vol") and not ProfileStore.open(path).supports("vol_and_surf_esp")
    tol = 0 if dtype == "float32" else 1e-2
    k = 0
    for s in range(st.num_shards):
        sh, a = st.read_shard(s)
        assert sh["start"] == k
        for i in range(sh["n"]):
            m = mols[k + i]
            a0, a1 = a["atom_off"][i], a["atom_off"][i + 1]
            np.testing.assert_allclose(a["atom_pos"][a0:a1], m["atom_pos"], atol=tol)
            np.testing.assert_allclose(a["surf_pos"][i], m["surf_pos"], atol=tol)
            np.testing.assert_allclose(a["charges"][a0:a1], m["partial_charges"], atol=tol)
            p0, p1 = a["pharm_off"][i], a["pharm_off"][i + 1]
            np.testing.assert_array_equal(a["pharm_types"][p0:p1], m["pharm_types"])
        k += sh["n"]


def test_version_guard(tmp_path):
    path = str(tmp_path / "s")
    ProfileStore.create(path, num_surf_points=64, modes=["vol"]).close()
    man = json.load(open(os.path.join(path, "manifest.json")))
    man["version"] = 2
    json.dump(man, open(os.path.join(path, "manifest.json"), "w"))
    with pytest.raises(ValueError, match="version"):
        ProfileStore.open(path)
    with pytest.raises(FileExistsError):
        ProfileStore.create(path, num_surf_points=64, modes=["vol"])


def test_pre_centred_store_and_query(tmp_path):
    mols = _mols(5, seed=3)
    path = str(tmp_path / "c")
    with ProfileStore.create(path, num_surf_points=64, modes=["surf", "pharm"],
                             dtype="float32", pre_centered=True) as st:
        for m in mols:
            st.add_arrays(**m)
    sh, a = ProfileStore.open(path).read_shard(0)
    for i in range(5):
        a0, a1 = a["atom_off"][i], a["atom_off"][i + 1]
        np.testing.assert_allclose(a["atom_pos"][a0:a1].mean(0), 0, atol=1e-5)
    q = _centred_query(mols[0])
    np.testing.assert_allclose(q["atom_pos"].mean(0), 0, atol=1e-5)
    np.testing.assert_allclose(q["surf_pos"] - q["atom_pos"][0],
                               mols[0]["surf_pos"] - mols[0]["atom_pos"][0], atol=1e-5)
    # centring an uncentred shard on the fly gives the same arrays as a pre-centred store
    path2 = str(tmp_path / "u")
    with ProfileStore.create(path2, num_surf_points=64, modes=["surf", "pharm"],
                             dtype="float32", pre_centered=False) as st:
        for m in mols:
            st.add_arrays(**m)
    _, b = ProfileStore.open(path2).read_shard(0)
    b = _center_shard(b, "surf")
    np.testing.assert_allclose(b["atom_pos"], a["atom_pos"], atol=1e-5)
    np.testing.assert_allclose(b["surf_pos"], a["surf_pos"], atol=1e-5)
    np.testing.assert_allclose(b["pharm_ancs"], a["pharm_ancs"], atol=1e-5)


def _combo_store(path, mols, dtype="float32", pre_centered=False, shard_size=7):
    with ProfileStore.create(path, num_surf_points=len(mols[0]["surf"]),
                             modes=["vol_and_surf_esp"], dtype=dtype, shard_size=shard_size,
                             pre_centered=pre_centered) as st:
        for m in mols:
            st.add_arrays(atom_pos=m["centers"], surf_pos=m["surf"], surf_esp=m["surf_esp"],
                          partial_charges=m["charges"], radii=m["radii"],
                          centers_w_H=m["atoms"])
    return ProfileStore.open(path)


def test_with_hydrogens_store_round_trip(tmp_path):
    """vol_and_surf_esp stores keep all-atom charges, radii and positions with their own
    offsets and the heavy-atom index (the reference writer's layout)."""
    rng = np.random.default_rng(3)
    mols = syn.esp_combo_molecules(16, rng, surf_lo=80, surf_hi=80)
    st = _combo_store(str(tmp_path / "combo.fss"), mols)
    assert st.supports("vol_and_surf_esp") and st.supports("surf_esp") and st.supports("vol")
    assert not st.supports("pharm")
    k = 0
    for s in range(st.num_shards):
        sh, a = st.read_shard(s)
        for i in range(sh["n"]):
            m = mols[k + i]
            a0, a1 = a["all_off"][i], a["all_off"][i + 1]
            np.testing.assert_array_equal(a["cwh"][a0:a1], m["atoms"])
            np.testing.assert_array_equal(a["charges"][a0:a1], m["charges"])
            np.testing.assert_array_equal(a["radii"][a0:a1], m["radii"])
            h0, h1 = a["atom_off"][i], a["atom_off"][i + 1]
            np.testing.assert_array_equal(a["atom_pos"][h0:h1], m["centers"])
            np.testing.assert_array_equal(a["surf_esp"][i], m["surf_esp"])
        k += sh["n"]
    with pytest.raises(ValueError):
        with ProfileStore.create(str(tmp_path / "bad.fss"), num_surf_points=80,
                                 modes=["vol_and_surf_esp"]) as bad:
            bad.add_arrays(atom_pos=mols[0]["centers"], surf_pos=mols[0]["surf"],
                           surf_esp=mols[0]["surf_esp"])
