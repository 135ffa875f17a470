"""Memory-bounded sub-batching and the out-of-memory halving path (host side, CPU only).

Allocation failures are injected through the alignment path's allocation hook, which
returns the library's FSS_ERR_NOMEM status for requests above a cap, as a device allocator
that ran out would; it is raised as MemoryError and the driver halves the chunk.  No GPU is
involved: the "launch" is a host function whose per-item results do not depend on the chunk.
"""
import numpy as np
import pytest
import torch

from fast_shepherd_score_b200 import _lib, memory


@pytest.fixture(autouse=True)
def no_hook():
    yield
    memory.set_alloc_hook(None)


def _fake_launch(values, item_bytes=64):
    """process(start, count): allocates its buffers through memory.empty, then computes a
    per-item result that depends only on the item (as a pair's alignment does)."""
    calls = []

    def process(a, k):
        calls.append((a, k))
        buf = memory.empty((k, item_bytes // 4), torch.float32, "cpu")
        buf.zero_()
        x = values[a:a + k]
        return (x * 2.0, x.unsqueeze(1).repeat(1, 4), None)
    return process, calls


def test_budget_sets_the_chunk():
    vals = torch.arange(100, dtype=torch.float32)
    process, calls = _fake_launch(vals)
    out = memory.run_chunked(100, 64, process, "cpu", budget=64 * 30)
    assert memory.LAST_CHUNKS == [30, 30, 30, 10]
    torch.testing.assert_close(out[0], vals * 2)
    assert out[2] is None and out[1].shape == (100, 4)


def test_nomem_halves_and_matches_one_call():
    vals = torch.randn(1000)
    want = _fake_launch(vals)[0](0, 1000)
    cap = 64 * 150      # refuse any single request above 150 items
    memory.set_alloc_hook(lambda nbytes, dev: _lib.FSS_ERR_NOMEM if nbytes > cap else 0)
    process, calls = _fake_launch(vals)
    got = memory.run_chunked(1000, 64, process, "cpu", budget=1 << 40)
    # 1000 refused, 500 refused, 250 refused, then chunks of 125
    assert [k for _, k in calls[:4]] == [1000, 500, 250, 125]
    assert memory.LAST_CHUNKS == [125] * 8
    for g, w in zip(got, want):
        if w is None:
            assert g is None
        else:
            assert torch.equal(g, w)


def test_nomem_on_a_single_item_is_raised():
    memory.set_alloc_hook(lambda nbytes, dev: _lib.FSS_ERR_NOMEM)
    process, _ = _fake_launch(torch.zeros(5))
    with pytest.raises(MemoryError):
        memory.run_chunked(5, 64, process, "cpu", budget=1 << 40)


def test_other_errors_are_not_retried():
    def process(a, k):
        raise ValueError("bad input")
    with pytest.raises(ValueError):
        memory.run_chunked(10, 64, process, "cpu")
    assert memory.LAST_CHUNKS == []


def test_status_mapping():
    with pytest.raises(MemoryError):
        _lib.raise_status(_lib.FSS_ERR_NOMEM, "x")
    with pytest.raises(ValueError):
        _lib.raise_status(_lib.FSS_ERR_INVALID, "x")
    with pytest.raises(RuntimeError):
        _lib.raise_status(_lib.FSS_ERR_CUDA, "x")


def test_bytes_per_pair_counts_rows_and_seeds():
    assert memory.align_bytes_per_pair(50) == memory.PAIR_BYTES + 50 * 60
    assert memory.align_bytes_per_pair(30, 605) == memory.PAIR_BYTES + 635 * 60


def test_budget_reads_allocator_statistics_only_when_needed(monkeypatch):
    """budget_bytes(device, need): free memory alone decides when it covers the call; the
    memory torch caches but does not use is added only when it does not (fakes for the CUDA
    queries, no GPU)."""
    stats = []
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (1000, 4000))
    monkeypatch.setattr(torch.cuda, "memory_reserved", lambda dev=None: stats.append(1) or 900)
    monkeypatch.setattr(torch.cuda, "memory_allocated", lambda dev=None: 100)
    assert memory.budget_bytes("cuda:0", need=500) == int(memory.SAFETY * 1000)
    assert not stats
    assert memory.budget_bytes("cuda:0", need=5000) == int(memory.SAFETY * (1000 + 800))
    assert stats
    stats.clear()
    assert memory.budget_bytes("cuda:0") == int(memory.SAFETY * 1800)   # no need given
    assert stats
