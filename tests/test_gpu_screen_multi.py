"""screen(ndev>1): the process-per-GPU path (spawned workers pulling shards from one queue,
per-GPU top-K lists merged on the host) returns the single-process hits.  On a box with one
visible GPU, ndev is clamped to one worker, which still runs the whole spawn / queue / merge
path."""
import numpy as np
import pytest

from test_gpu_api import _mols, _moved

pytestmark = pytest.mark.gpu


def test_multi_gpu_screen_matches_single_process(tmp_path, cuda):
    from fast_shepherd_score_b200.screen import ProfileStore, screen_many
    rng = np.random.default_rng(6)
    lib = _mols(40, 12)
    queries = [lib[3], lib[27]]
    lib[11] = _moved(lib[3], rng)
    path = str(tmp_path / "lib")
    with ProfileStore.create(path, num_surf_points=100, modes=["surf_esp", "pharm"],
                             dtype="float32", shard_size=7) as st:
        for m in lib:
            st.add_arrays(**m)
    store = ProfileStore.open(path)
    kw = dict(top_k=6, num_repeats=10, max_num_steps=30)
    for mode in ("surf_esp", "pharm"):
        one = screen_many(queries, store, mode, **kw)
        many = screen_many(queries, store, mode, ndev=2, **kw)
        for a, b in zip(one, many):
            # same hits with the same scores and poses (equal scores may list in either order)
            da = {h.id: h for h in a}
            db = {h.id: h for h in b}
            assert set(da) == set(db)
            for i in da:
                assert abs(da[i].score - db[i].score) <= 1e-6
                np.testing.assert_allclose(da[i].transform, db[i].transform, atol=1e-5)
    assert {h.id for h in one[0][:2]} == {3, 11}
    with pytest.raises(ValueError):
        screen_many(queries, store, "surf_esp", ndev=2, scores_out=[np.zeros(40)] * 2, **kw)
