"""GPU: the continuous-batching screening server.  A request's hits are identical alone and
when it shares launches with other requests (every pair is computed independently with a
fixed tiling), and equal to scoring the same pairs directly through the array API."""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import api, synthetic as syn
from fast_shepherd_score_b200.server import ScreenServer

pytestmark = pytest.mark.gpu

KW = dict(mode="vol_pharm", starts=8, steps=30, max_pairs_per_launch=3000, slice_pairs=700,
          lanes_per_pose=8)


def _query(lib, i):
    atoms, ph = lib
    a0, a1 = int(atoms.off[i]), int(atoms.off[i + 1])
    p0, p1 = int(ph.off[i]), int(ph.off[i + 1])
    anc = ph.anc[p0:p1].cpu()
    return {"atom_pos": atoms.pts[a0:a1, :3].cpu().numpy(),
            "pharm_types": anc[:, 3].contiguous().view(torch.int32).numpy(),
            "pharm_ancs": anc[:, :3].numpy(), "pharm_vecs": ph.vec[p0:p1, :3].cpu().numpy()}


@pytest.fixture(scope="module")
def lib(cuda):
    return syn.library_on_device(2500, seed=3, device=cuda)


def test_alone_equals_in_the_mix(lib, cuda):
    q = _query(lib, 11)
    idx = np.arange(100, 1900, dtype=np.int32)
    with ScreenServer(lib, **KW) as srv:
        alone = srv.submit(q, idx, top_k=20).result(timeout=300)
    rng = np.random.default_rng(0)
    with ScreenServer(lib, **KW) as srv:
        futs = []
        for j in range(6):
            n = int(rng.integers(300, 2400))
            futs.append(srv.submit(_query(lib, 40 + j), rng.choice(2500, n, replace=False),
                                   top_k=10))
            if j == 2:
                mixed_f = srv.submit(q, idx, top_k=20)
        mixed = mixed_f.result(timeout=300)
        others = [f.result(timeout=300) for f in futs]
        st = srv.stats()
    assert [(h.id, h.score) for h in alone] == [(h.id, h.score) for h in mixed]
    assert all(len(o) == 10 for o in others)
    assert st["completed"] == 7 and st["p99_ms"] >= st["p50_ms"] > 0
    assert st["in_flight_bytes"] == 0


def test_server_matches_direct_alignment(lib, cuda):
    atoms, ph = lib
    q = _query(lib, 5)
    idx = np.arange(0, 1200, dtype=np.int32)
    with ScreenServer(lib, **KW) as srv:
        hits = srv.submit(q, idx, top_k=1200).result(timeout=300)
    ref = api.HostBatch.from_lists([q["atom_pos"]], None, [q["pharm_types"]], [q["pharm_ancs"]],
                                   [q["pharm_vecs"]])
    rc, rp = ref.to_device(cuda)
    out = api.align_device("vol_pharm", rc, atoms, rp, ph,
                           torch.zeros(len(idx), dtype=torch.int32, device=cuda),
                           torch.as_tensor(idx, device=cuda), num_seeds=8, steps=30, lr=0.1,
                           lanes_per_pose=8)
    direct = out[0].cpu().numpy()
    got = np.zeros(len(idx))
    for h in hits:
        got[h.id] = h.score
    np.testing.assert_array_equal(got, direct)
    assert hits[0].id == 5 and hits[0].score > 0.999        # the query itself is in the library
