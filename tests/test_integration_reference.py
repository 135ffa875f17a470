"""The ``backend="cuda"`` shim on the reference's own MoleculePairBatch and screen (CPU only).

``fast_shepherd_score_b200.integration.install()`` patches shepherd_score's dispatch
(container/_batch.py:100, :127-151, :1320-1360; screen.py:1038, :1141).  These tests import the
reference from its source tree (``$FSS_REFERENCE`` or a ``reference`` checkout beside this
repository; skipped when neither exists), apply the shim and check, with the aligners replaced
by recorders so no GPU is needed:

* ``backend="cuda"`` reaches this package's ``_align_batch_<mode>`` with the keyword arguments
  the reference passes, and each real aligner of this package accepts exactly those arguments;
* the reference's own ``_triton_align`` then reads the in-place results back;
* ``"triton"`` and ``"numba"`` still reach the reference's aligners, unknown names still raise;
* the pharmacophore branch and ``screen()`` route the same way;
* ``uninstall()`` restores the reference's routing.
"""
import inspect
import types

import numpy as np
import pytest
import torch

from tests.reference_import import import_reference

REF = import_reference()
pytestmark = pytest.mark.skipif(REF is None, reason="reference source tree not present")

MODE_CALLS = {
    # mode: (align_with_* kwargs, score attribute, transform attribute)
    "vol": (dict(), "sim_aligned_vol_noH", "transform_vol_noH"),
    "vol_esp": (dict(lam=0.1), "sim_aligned_vol_esp_noH", "transform_vol_esp_noH"),
    "surf": (dict(alpha=1.216), "sim_aligned_surf", "transform_surf"),
    "surf_esp": (dict(alpha=1.216, lam=0.3), "sim_aligned_surf_esp", "transform_surf_esp"),
    "vol_and_surf_esp": (dict(alpha=0.81), "sim_aligned_vol_and_surf_esp",
                         "transform_vol_and_surf_esp"),
    "vol_color": (dict(), "sim_aligned_vol_color", "transform_vol_color"),
}


def _pairs(n, device="cpu"):
    return [types.SimpleNamespace(device=torch.device(device), idx=i) for i in range(n)]


class Recorder:
    """Stands in for an aligner: records its call and writes results in place."""

    def __init__(self, score_attr, tf_attr, name):
        self.calls = []
        self.score_attr, self.tf_attr = score_attr, tf_attr
        self.__name__ = name

    def __call__(self, pairs, **kw):
        self.calls.append(kw)
        for p in pairs:
            setattr(p, self.score_attr, 0.5 + 0.01 * p.idx)
            setattr(p, self.tf_attr, torch.eye(4))


@pytest.fixture
def shim(monkeypatch):
    from fast_shepherd_score_b200 import integration
    integration.install()
    moved = []
    monkeypatch.setattr(integration, "_to_cuda", lambda pairs: moved.append(len(pairs)))
    yield integration, moved
    integration.uninstall()


@pytest.mark.parametrize("mode", list(MODE_CALLS))
def test_cuda_routes_to_this_package(shim, monkeypatch, mode):
    from fast_shepherd_score_b200 import aligners
    integration, moved = shim
    batch_mod, core_mod, _ = REF
    kw, s_attr, t_attr = MODE_CALLS[mode]
    name = "_align_batch_" + mode
    real = getattr(aligners, name)
    mine = Recorder(s_attr, t_attr, name)
    theirs = Recorder(s_attr, t_attr, name)
    monkeypatch.setattr(aligners, name, mine)
    monkeypatch.setattr(core_mod.MoleculePair, name, staticmethod(theirs))
    pairs = _pairs(3)
    scores, aligned = getattr(batch_mod.MoleculePairBatch(pairs), "align_with_" + mode)(
        backend="cuda", **kw)
    assert len(mine.calls) == 1 and not theirs.calls
    assert moved == [3]
    np.testing.assert_allclose(scores, [0.5, 0.51, 0.52])
    assert aligned == [None] * 3
    # the real aligner of this package accepts exactly what the reference passed
    inspect.signature(real).bind(pairs, **mine.calls[0])


@pytest.mark.parametrize("backend", ["triton", "gpu"])
def test_triton_names_still_reach_the_reference(shim, monkeypatch, backend):
    from fast_shepherd_score_b200 import aligners
    batch_mod, core_mod, _ = REF
    mine = Recorder("sim_aligned_vol_noH", "transform_vol_noH", "_align_batch_vol")
    theirs = Recorder("sim_aligned_vol_noH", "transform_vol_noH", "_align_batch_vol")
    monkeypatch.setattr(aligners, "_align_batch_vol", mine)
    monkeypatch.setattr(core_mod.MoleculePair, "_align_batch_vol", staticmethod(theirs))
    batch_mod.MoleculePairBatch(_pairs(2)).align_with_vol(backend=backend)
    assert len(theirs.calls) == 1 and not mine.calls


def test_numba_still_reaches_the_reference(shim, monkeypatch):
    pytest.importorskip("numba")
    from fast_shepherd_score_b200 import aligners
    batch_mod, core_mod, _ = REF
    mine = Recorder("sim_aligned_surf", "transform_surf", "_align_batch_surf")
    theirs = Recorder("sim_aligned_surf", "transform_surf", "_align_batch_surf")
    monkeypatch.setattr(aligners, "_align_batch_surf", mine)
    monkeypatch.setattr(core_mod.MoleculePair, "_align_batch_surf", staticmethod(theirs))
    pairs = _pairs(2, "cuda")   # a device object only; the numba path moves pairs to the CPU
    batch_mod.MoleculePairBatch(pairs).align_with_surf(alpha=1.216, backend="numba")
    assert len(theirs.calls) == 1 and not mine.calls
    assert all(p.device.type == "cpu" for p in pairs)


def test_unknown_backend_still_raises(shim):
    batch_mod, _, _ = REF
    with pytest.raises(ValueError):
        batch_mod.MoleculePairBatch(_pairs(1)).align_with_vol(backend="tpu")
    with pytest.raises(ValueError):
        batch_mod.MoleculePairBatch(_pairs(1)).align_with_pharm(backend="tpu")


def test_pharm_branch(shim, monkeypatch):
    from fast_shepherd_score_b200 import aligners
    batch_mod, core_mod, _ = REF
    real = aligners._align_batch_pharm
    mine = Recorder("sim_aligned_pharm", "transform_pharm", "_align_batch_pharm")
    theirs = Recorder("sim_aligned_pharm", "transform_pharm", "_align_batch_pharm")
    monkeypatch.setattr(aligners, "_align_batch_pharm", mine)
    monkeypatch.setattr(core_mod.MoleculePair, "_align_batch_pharm", staticmethod(theirs))
    pairs = _pairs(2)
    scores, anchors, vectors = batch_mod.MoleculePairBatch(pairs).align_with_pharm(
        backend="cuda", similarity="tversky", extended_points=True)
    assert len(mine.calls) == 1 and not theirs.calls
    assert mine.calls[0]["similarity"] == "tversky" and mine.calls[0]["extended_points"]
    np.testing.assert_allclose(scores, [0.5, 0.51])
    assert anchors == [None, None] and vectors == [None, None]
    inspect.signature(real).bind(pairs, **mine.calls[0])
    batch_mod.MoleculePairBatch(_pairs(2)).align_with_pharm(backend="triton")
    assert len(theirs.calls) == 1 and len(mine.calls) == 1


def test_screen_routes(shim, monkeypatch):
    from fast_shepherd_score_b200 import screen as cuda_screen
    _, _, screen_mod = REF
    calls = []

    def fake_screen_many(queries, store, mode, **kw):
        calls.append((len(queries), mode, kw))
        return [[(0.9, 7, np.eye(4, dtype=np.float32))] for _ in queries]

    monkeypatch.setattr(cuda_screen, "screen_many", fake_screen_many)
    hits = screen_mod.screen(object(), object(), "vol", backend="cuda", top_k=5)
    assert calls == [(1, "vol", dict(backend="cuda", top_k=5))]
    assert isinstance(hits[0], screen_mod.Hit) and hits[0].id == 7
    panel = screen_mod.screen_many([object(), object()], object(), "pharm", backend="cuda")
    assert len(panel) == 2 and panel[1][0].score == 0.9
    # another backend reaches the reference's own screen (which rejects a non-store)
    with pytest.raises(Exception):
        screen_mod.screen(object(), object(), "vol", backend="numba")
    assert len(calls) == 2


def test_uninstall_restores_the_reference(monkeypatch):
    from fast_shepherd_score_b200 import integration
    batch_mod, _, screen_mod = REF
    cls = batch_mod.MoleculePairBatch
    before = (cls._TRITON_BACKENDS, cls.__dict__["_run_fast_or_fallthrough"],
              cls.__dict__["align_with_pharm"], screen_mod.screen, screen_mod.screen_many)
    with integration.cuda_backend():
        assert "cuda" not in cls._TRITON_BACKENDS and cls._CUDA_BACKENDS == ("cuda",)
        assert cls.__dict__["_run_fast_or_fallthrough"] is not before[1]
    after = (cls._TRITON_BACKENDS, cls.__dict__["_run_fast_or_fallthrough"],
             cls.__dict__["align_with_pharm"], screen_mod.screen, screen_mod.screen_many)
    assert after == before
    assert "cuda" in cls._TRITON_BACKENDS and not hasattr(cls, "_CUDA_BACKENDS")
