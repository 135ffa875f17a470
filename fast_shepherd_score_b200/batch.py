"""``MoleculePairBatch`` with ``backend="cuda"`` -- the object-level drop-in.

Mirrors shepherd_score/container/_batch.py's ``MoleculePairBatch.align_with_*`` signatures
(:274, :496, :745, :881, :1104, :1238) for the modes on the CUDA path.  Every method routes to
the per-mode aligner of :mod:`fast_shepherd_score_b200.aligners`, writes the results onto the
pairs under the reference's attribute names, and returns ``(scores, aligned_list)``
(``(scores, aligned_anchors, aligned_vectors)`` for pharm, as ``_batch.py:1339``).

Backend names: ``None`` and ``"cuda"`` run here.  The reference's other backends
(``"triton"``, ``"gpu"``, ``"numba"``, ``"cpu"``, ``"jax"``) belong to shepherd_score itself
and raise ``ValueError`` here, as unknown names do in the reference (``_batch.py:149-150``).
Arguments that only steer those backends (``num_workers``, ``use_shmap``, ``num_buckets``,
``use_jax``, ``use_analytical``) are accepted and ignored.
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np
import torch

from . import aligners as A
from .modes import MODE_ATTRS, seeds_for, steps_for

_CUDA_BACKENDS = ("cuda",)
_REFERENCE_BACKENDS = ("triton", "gpu", "numba", "cpu", "jax")


def _resolve(backend):
    if backend is None or backend in _CUDA_BACKENDS:
        return "cuda"
    if backend in _REFERENCE_BACKENDS:
        raise ValueError(f"backend {backend!r} is provided by shepherd_score; "
                         "fast_shepherd_score_b200 implements backend='cuda'")
    raise ValueError(f"unknown backend {backend!r}; use 'cuda'")


class MoleculePairBatch:
    """A batch of MoleculePair-like objects (anything carrying the cached ``_*_t`` tensors
    or ``ref_molec``/``fit_molec`` arrays and a ``device``)."""

    def __init__(self, pairs: List):
        self.pairs = pairs

    # -------------------------------------------------------------------------------------
    def _finish(self, mode, scores, fit_attr, return_aligned, verbose):
        if verbose:
            for i, s in enumerate(scores):
                print(f"pair {i}: {s:.4f}")
        if not return_aligned:
            return np.asarray(scores, dtype=float), [None] * len(self.pairs)
        tf_attr = MODE_ATTRS[mode][0]
        aligned = []
        for p in self.pairs:
            X = getattr(p, fit_attr).to(torch.float32).cpu()
            T = torch.as_tensor(getattr(p, tf_attr), dtype=torch.float32)
            aligned.append((X @ T[:3, :3].T + T[:3, 3]).numpy())
        return np.asarray(scores, dtype=float), aligned

    @staticmethod
    def _steps(mode, max_num_steps):
        return steps_for(mode) if max_num_steps is None else int(max_num_steps)

    @staticmethod
    def _seeds(mode, num_repeats):
        return seeds_for(mode) if num_repeats is None else int(num_repeats)

    # -------------------------------------------------------------------------------------
    def align_with_vol(self, no_H: bool = True, num_repeats: int = None, trans_init: bool = False,
                       lr: float = 0.1, max_num_steps: int = None, num_workers: int = 1,
                       use_shmap: bool = True, num_buckets: int = 1, verbose: bool = False,
                       backend: Optional[str] = None, alpha: float = 0.81,
                       return_aligned: bool = False) -> Tuple[np.ndarray, list]:
        _resolve(backend)
        if not no_H:
            raise ValueError("backend='cuda' aligns heavy atoms (no_H=True)")
        # trans_init is not forwarded to the vol fast path by the reference either
        # (container/_batch.py:362-368): batched seeds are used
        sc = A._align_batch_vol(self.pairs, alpha=alpha, steps_fine=self._steps("vol", max_num_steps),
                                num_repeats=self._seeds("vol", num_repeats), lr=lr)
        return self._finish("vol", sc, "_fit_xyz_t", return_aligned, verbose)

    def align_with_vol_esp(self, lam: float = 0.1, no_H: bool = True, num_repeats: int = None,
                           trans_init: bool = False, lr: float = 0.1, max_num_steps: int = None,
                           num_workers: int = 1, use_shmap: bool = True, num_buckets: int = 1,
                           verbose: bool = False, backend: Optional[str] = None,
                           alpha: float = 0.81, return_aligned: bool = False):
        _resolve(backend)
        if not no_H:
            raise ValueError("backend='cuda' aligns heavy atoms (no_H=True)")
        sc = A._align_batch_vol_esp(self.pairs, lam=lam, alpha=alpha, trans_init=trans_init,
                                    num_repeats=self._seeds("vol_esp", num_repeats),
                                    steps_fine=self._steps("vol_esp", max_num_steps), lr=lr)
        return self._finish("vol_esp", sc, "_fit_xyz_noH_t", return_aligned, verbose)

    def align_with_surf(self, alpha: float, num_repeats: int = None, trans_init: bool = False,
                        lr: float = 0.1, max_num_steps: int = None, use_jax: bool = True,
                        use_analytical: bool = True, num_workers: int = 1,
                        use_shmap: bool = False, verbose: bool = False,
                        backend: Optional[str] = None, return_aligned: bool = False):
        _resolve(backend)
        # as for vol, the reference's surf fast path ignores trans_init (_batch.py:813-818)
        sc = A._align_batch_surf(self.pairs, alpha=alpha,
                                 steps_fine=self._steps("surf", max_num_steps),
                                 num_repeats=self._seeds("surf", num_repeats), lr=lr)
        return self._finish("surf", sc, "_fit_surf_t", return_aligned, verbose)

    def align_with_surf_esp(self, alpha: float, lam: float = 0.3, num_repeats: int = None,
                            trans_init: bool = False, lr: float = 0.1,
                            max_num_steps: int = None, use_jax: bool = True,
                            use_analytical: bool = True, num_workers: int = 1,
                            use_shmap: bool = False, verbose: bool = False,
                            backend: Optional[str] = None, return_aligned: bool = False):
        _resolve(backend)
        sc = A._align_batch_surf_esp(self.pairs, alpha=alpha, lam=lam, trans_init=trans_init,
                                     num_repeats=self._seeds("surf_esp", num_repeats),
                                     steps_fine=self._steps("surf_esp", max_num_steps), lr=lr)
        return self._finish("surf_esp", sc, "_fit_surf_t", return_aligned, verbose)

    align_with_esp = align_with_surf_esp   # legacy name (accel/_modes.py LEGACY_MODE_ALIASES)

    def align_with_vol_and_surf_esp(self, alpha: float, lam: float = 0.001,
                                    probe_radius: float = 1.0, esp_weight: float = 0.5,
                                    num_repeats: int = None, trans_init: bool = False,
                                    lr: float = 0.1, max_num_steps: int = None,
                                    verbose: bool = False, backend: Optional[str] = None,
                                    return_aligned: bool = False, esp_stride: int = 1):
        """ShaEP-style combo (_batch.py:1030): the shape centres steer the pose, the score adds
        the surface ESP comparison.  ``esp_stride`` (this backend's knob) tracks the combo
        score every step by default, as the reference's CUDA-graph loop; 5 matches its eager
        loop."""
        _resolve(backend)
        sc = A._align_batch_vol_and_surf_esp(
            self.pairs, alpha=alpha, lam=lam, probe_radius=probe_radius, esp_weight=esp_weight,
            trans_init=trans_init, num_repeats=self._seeds("vol_and_surf_esp", num_repeats),
            steps_fine=self._steps("vol_and_surf_esp", max_num_steps), lr=lr,
            esp_stride=esp_stride)
        return self._finish("vol_and_surf_esp", sc, "_fit_surf_t", return_aligned, verbose)

    align_with_esp_combo = align_with_vol_and_surf_esp   # legacy name

    def align_with_vol_color(self, color_weight: float = 0.5, alpha: float = 0.81,
                             num_repeats: int = None, trans_init: bool = False, lr: float = 0.1,
                             max_num_steps: int = None, verbose: bool = False,
                             backend: Optional[str] = None, return_aligned: bool = False):
        _resolve(backend)
        sc = A._align_batch_vol_color(self.pairs, alpha=alpha, color_weight=color_weight,
                                      trans_init=trans_init,
                                      num_repeats=self._seeds("vol_color", num_repeats),
                                      steps_fine=self._steps("vol_color", max_num_steps), lr=lr)
        return self._finish("vol_color", sc, "_fit_xyz_t", return_aligned, verbose)

    def align_with_vol_pharm(self, color_weight: float = 0.5, alpha: float = 0.81,
                             num_repeats: int = None, trans_init: bool = False, lr: float = 0.1,
                             max_num_steps: int = None, verbose: bool = False,
                             backend: Optional[str] = None, return_aligned: bool = False):
        """Shape + directional pharmacophores with one shared pose (cosine-weighted typed
        overlap, the directional counterpart of vol_color)."""
        _resolve(backend)
        sc = A._align_batch_vol_pharm(self.pairs, alpha=alpha, color_weight=color_weight,
                                      trans_init=trans_init,
                                      num_repeats=self._seeds("vol_pharm", num_repeats),
                                      steps_fine=self._steps("vol_pharm", max_num_steps), lr=lr)
        return self._finish("vol_pharm", sc, "_fit_xyz_t", return_aligned, verbose)

    def align_with_pharm(self, similarity: str = 'tanimoto', extended_points: bool = False,
                         only_extended: bool = False, num_repeats: int = None,
                         trans_init: bool = False, lr: float = 0.1, max_num_steps: int = None,
                         num_workers: int = 1, use_shmap: bool = True, num_buckets: int = 1,
                         verbose: bool = False, backend: Optional[str] = None,
                         return_aligned: bool = False):
        _resolve(backend)
        A._align_batch_pharm(self.pairs, similarity=similarity,
                             extended_points=extended_points, only_extended=only_extended,
                             trans_init=trans_init, num_repeats=self._seeds("pharm", num_repeats),
                             steps_fine=self._steps("pharm", max_num_steps), lr=lr)
        # read back from the pairs, as the reference does (_batch.py:1335): the aligner's
        # contract is the in-place result
        scores = np.array([float(p.sim_aligned_pharm) for p in self.pairs], dtype=float)
        if not return_aligned:
            return scores, [None] * len(self.pairs), [None] * len(self.pairs)
        ancs, vecs = [], []
        for p in self.pairs:
            T = torch.as_tensor(p.transform_pharm, dtype=torch.float32)
            a = p._fit_pharm_ancs_t.to(torch.float32).cpu()
            v = p._fit_pharm_vecs_t.to(torch.float32).cpu()
            ancs.append((a @ T[:3, :3].T + T[:3, 3]).numpy())
            vecs.append((v @ T[:3, :3].T).numpy())
        return scores, ancs, vecs
