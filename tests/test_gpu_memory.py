"""Memory-bounded alignment on the GPU: chunked and OOM-halved calls give exactly the
results of one call (pairs are independent; a fixed tile makes the arithmetic identical).
The out-of-memory condition is injected on the host through the allocation hook (the
library's FSS_ERR_NOMEM status for row buffers above a cap); no device allocation fails."""
import pytest
import torch

from fast_shepherd_score_b200 import _lib, api, memory
from fast_shepherd_score_b200 import synthetic as syn

pytestmark = pytest.mark.gpu
TILE = dict(lanes_per_pose=8, chunks=1)


@pytest.fixture(autouse=True)
def no_hook():
    yield
    memory.set_alloc_hook(None)


def _batch(cuda, n=300):
    refs, fits = syn.shape_pairs(n, seed=9)
    rc, _ = api.HostBatch.from_lists(refs).to_device(cuda)
    fc, _ = api.HostBatch.from_lists(fits).to_device(cuda)
    idx = torch.arange(n, dtype=torch.int32, device=cuda)
    return rc, fc, idx


def _same(a, b):
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    for x, y in zip(a.rows, b.rows):
        assert torch.equal(x, y)


def test_oom_halving_matches_one_call(cuda):
    rc, fc, idx = _batch(cuda)
    kw = dict(num_seeds=20, steps=30, lr=0.1, **TILE)
    one = api.align_device("vol", rc, fc, None, None, idx, idx, **kw)
    assert memory.LAST_CHUNKS == [300]
    cap = 64 * 20 * 16            # the (pairs x starts, 4) pose rows of 64 pairs
    memory.set_alloc_hook(lambda nbytes, dev: _lib.FSS_ERR_NOMEM if nbytes > cap else 0)
    got = api.align_device("vol", rc, fc, None, None, idx, idx, **kw)
    assert memory.LAST_CHUNKS == [37] * 8 + [4]      # 300 -> 150 -> 75 -> 37 refused / fits
    _same(got, one)


def test_pair_cap_matches_one_call(cuda):
    rc, fc, idx = _batch(cuda, 250)
    kw = dict(num_seeds=10, steps=20, lr=0.1, **TILE)
    one = api.align_device("vol", rc, fc, None, None, idx, idx, **kw)
    got = api.align_device("vol", rc, fc, None, None, idx, idx, max_chunk_pairs=100, **kw)
    assert memory.LAST_CHUNKS == [100, 100, 50]
    _same(got, one)
