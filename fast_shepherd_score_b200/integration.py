"""Plug this package into shepherd_score as its ``backend="cuda"``.

shepherd_score routes every batched alignment of ``MoleculePairBatch`` through
``_run_fast_or_fallthrough`` (shepherd_score/container/_batch.py:127-151) and, for
pharmacophores, through its own branch of ``align_with_pharm`` (:1320-1360); there ``"cuda"``
is an alias of the Triton path (:100).  :func:`install` changes exactly that routing, on the
reference's own classes and modules:

* ``MoleculePairBatch._TRITON_BACKENDS`` loses ``"cuda"`` and ``_CUDA_BACKENDS = ("cuda",)``
  is added beside it;
* ``_run_fast_or_fallthrough`` sends ``"cuda"`` to this package's ``_align_batch_<mode>``
  (:mod:`fast_shepherd_score_b200.aligners`: the same function names, keyword arguments and
  in-place results as shepherd_score/accel/batch/aligners.py) through the reference's own
  ``_triton_align``, which then collects the scores and builds ``aligned_list`` as it does
  for Triton;
* ``align_with_pharm`` sends ``"cuda"`` to this package's pharmacophore aligner and returns
  the reference's ``(scores, aligned_anchors, aligned_vectors)`` tuple;
* ``shepherd_score.screen.screen`` / ``screen_many`` send ``backend="cuda"`` to
  :mod:`fast_shepherd_score_b200.screen`, which reads the same ``ProfileStore`` (the
  reference's store object is accepted as it is) and returns the reference's ``Hit`` tuples.

Every other backend name (``"triton"``, ``"gpu"``, ``"numba"``, ``"cpu"``, ``"jax"``, and
``None``, which shepherd_score resolves to triton or numba) reaches the reference's code
unchanged, and unknown names still raise its ``ValueError``.  Pairs that live on the CPU are
moved to the current CUDA device for ``"cuda"``, as the reference moves them to the CPU for
``"numba"`` (``_prepare_numba``, _batch.py:107-125).  :func:`uninstall` restores the
originals; :func:`cuda_backend` is the context-manager form.  Nothing here runs on import.
"""
from __future__ import annotations

import contextlib
import functools
import importlib
from typing import Optional

CUDA_BACKENDS = ("cuda",)

# installed state: the reference objects that were replaced, to put back on uninstall
_SAVED: dict = {}


def _reference():
    """(container._batch module, screen module) of the importable shepherd_score."""
    batch_mod = importlib.import_module("shepherd_score.container._batch")
    screen_mod = importlib.import_module("shepherd_score.screen")
    return batch_mod, screen_mod


def is_installed() -> bool:
    return bool(_SAVED)


def _cuda_aligner(align_fn):
    """This package's aligner of the same name as the reference's ``align_fn``.  The
    reference binds its legacy names (``_align_batch_esp``, ``_align_batch_esp_combo``) to
    the canonical functions, so ``__name__`` is always the canonical one."""
    from . import aligners
    name = getattr(align_fn, "__name__", "")
    fn = getattr(aligners, name, None) if name.startswith("_align_batch_") else None
    if fn is None:
        raise ValueError(f"backend='cuda' has no aligner for {name or align_fn!r}")
    return fn


def _to_cuda(pairs):
    """Point every pair at a CUDA device (their cached tensors move on first use)."""
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("backend='cuda' needs a CUDA device (this backend has no CPU path); "
                           "use backend='numba' for the CPU")
    dev = torch.device("cuda", torch.cuda.current_device())
    for p in pairs:
        d = getattr(p, "device", None)
        if d is None or torch.device(d).type != "cuda":
            p.device = dev


def install() -> None:
    """Route ``backend="cuda"`` of the importable shepherd_score to this package."""
    if _SAVED:
        return
    batch_mod, screen_mod = _reference()
    cls = batch_mod.MoleculePairBatch
    saved = dict(cls=cls, screen_mod=screen_mod, triton=cls.__dict__["_TRITON_BACKENDS"],
                 had_cuda_attr="_CUDA_BACKENDS" in cls.__dict__,
                 cuda_attr=cls.__dict__.get("_CUDA_BACKENDS"),
                 run=cls.__dict__["_run_fast_or_fallthrough"],
                 pharm=cls.__dict__["align_with_pharm"],
                 screen=screen_mod.screen, screen_many=screen_mod.screen_many)
    resolve = batch_mod._resolve_backend
    orig_run, orig_pharm = saved["run"], saved["pharm"]

    @functools.wraps(orig_run)
    def _run_fast_or_fallthrough(self, backend, align_fn, align_kwargs, score_attr,
                                 transform_attr, fit_attr, return_aligned, *,
                                 num_workers: int = 1, precheck=None):
        if resolve(backend) in type(self)._CUDA_BACKENDS:
            fn = _cuda_aligner(align_fn)
            _to_cuda(self.pairs)
            if precheck is not None:
                precheck()
            # num_workers shards CPU pairs over a process pool in the reference; one fused
            # launch covers the whole batch here
            return True, self._triton_align(fn, align_kwargs, score_attr, transform_attr,
                                            fit_attr, return_aligned, num_workers=1)
        return orig_run(self, backend, align_fn, align_kwargs, score_attr, transform_attr,
                        fit_attr, return_aligned, num_workers=num_workers, precheck=precheck)

    @functools.wraps(orig_pharm)
    def align_with_pharm(self, similarity: str = "tanimoto", extended_points: bool = False,
                         only_extended: bool = False, num_repeats: int = None,
                         trans_init: bool = False, lr: float = 0.1,
                         max_num_steps: int = None, num_workers: int = 1,
                         use_shmap: bool = True, num_buckets: int = 1, verbose: bool = False,
                         backend: Optional[str] = None, return_aligned: bool = False):
        if resolve(backend) in type(self)._CUDA_BACKENDS:
            from .batch import MoleculePairBatch as CudaBatch
            _to_cuda(self.pairs)
            return CudaBatch(self.pairs).align_with_pharm(
                similarity=similarity, extended_points=extended_points,
                only_extended=only_extended, num_repeats=num_repeats, trans_init=trans_init,
                lr=lr, max_num_steps=max_num_steps, verbose=verbose, backend="cuda",
                return_aligned=return_aligned)
        return orig_pharm(self, similarity=similarity, extended_points=extended_points,
                          only_extended=only_extended, num_repeats=num_repeats,
                          trans_init=trans_init, lr=lr, max_num_steps=max_num_steps,
                          num_workers=num_workers, use_shmap=use_shmap,
                          num_buckets=num_buckets, verbose=verbose, backend=backend,
                          return_aligned=return_aligned)

    orig_screen_many = saved["screen_many"]

    @functools.wraps(orig_screen_many)
    def screen_many(queries, store, mode: str = "surf_esp", *, backend: Optional[str] = None,
                    **kw):
        if backend in CUDA_BACKENDS:
            from . import screen as cuda_screen
            hit = screen_mod.Hit
            out = cuda_screen.screen_many(queries, store, mode, backend="cuda", **kw)
            return [[hit(*h) for h in hits] for hits in out]
        return orig_screen_many(queries, store, mode, backend=backend, **kw)

    @functools.wraps(saved["screen"])
    def screen(query, store, mode: str = "surf_esp", *, backend: Optional[str] = None, **kw):
        if backend in CUDA_BACKENDS:
            return screen_many([query], store, mode, backend=backend, **kw)[0]
        return saved["screen"](query, store, mode, backend=backend, **kw)

    cls._TRITON_BACKENDS = tuple(b for b in saved["triton"] if b not in CUDA_BACKENDS)
    cls._CUDA_BACKENDS = CUDA_BACKENDS
    cls._run_fast_or_fallthrough = _run_fast_or_fallthrough
    cls.align_with_pharm = align_with_pharm
    screen_mod.screen_many = screen_many
    screen_mod.screen = screen
    _SAVED.update(saved)


def uninstall() -> None:
    """Put the reference's original routing back."""
    if not _SAVED:
        return
    cls, screen_mod = _SAVED["cls"], _SAVED["screen_mod"]
    cls._TRITON_BACKENDS = _SAVED["triton"]
    if _SAVED["had_cuda_attr"]:
        cls._CUDA_BACKENDS = _SAVED["cuda_attr"]
    else:
        del cls._CUDA_BACKENDS
    cls._run_fast_or_fallthrough = _SAVED["run"]
    cls.align_with_pharm = _SAVED["pharm"]
    screen_mod.screen = _SAVED["screen"]
    screen_mod.screen_many = _SAVED["screen_many"]
    _SAVED.clear()


@contextlib.contextmanager
def cuda_backend():
    """``with cuda_backend(): ...`` -- :func:`install` for the duration of the block (a no-op
    when already installed, so nesting keeps the outer installation)."""
    was = is_installed()
    install()
    try:
        yield
    finally:
        if not was:
            uninstall()
