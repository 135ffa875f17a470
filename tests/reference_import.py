"""Import the reference package (shepherd_score) from its source tree for CPU-side tests.

The tree is found through ``$FSS_REFERENCE`` or, failing that, a ``reference`` checkout next to
this repository.  shepherd_score imports RDKit and Open3D at module level (featurisation,
visualisation), which the code paths under test never call; they are replaced by permissive
import-only stand-ins, so ``import shepherd_score.container`` succeeds without them.  Nothing
here runs reference computations that need those packages.
"""
from __future__ import annotations

import importlib.abc
import importlib.machinery
import os
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STUBBED = ("rdkit", "open3d")


def reference_root():
    """The reference source tree, or None when it is not present on this machine."""
    for cand in (os.environ.get("FSS_REFERENCE"), os.path.join(os.path.dirname(ROOT), "reference")):
        if cand and os.path.isfile(os.path.join(cand, "shepherd_score", "__init__.py")):
            return os.path.abspath(cand)
    return None


class _AnyMeta(type):
    """Class attribute access yields another permissive class (``Chem.rdchem.Mol`` etc.)."""

    def __getattr__(cls, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _AnyMeta(name, (_Any,), {})


class _Any(metaclass=_AnyMeta):
    def __init__(self, *a, **k):
        pass

    def __call__(self, *a, **k):
        return _Any()

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _Any()


class _StubModule(types.ModuleType):
    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        value = _AnyMeta(name, (_Any,), {})
        setattr(self, name, value)
        return value


class _StubFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, name, path, target=None):
        if name.split(".")[0] in STUBBED:
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        mod = _StubModule(spec.name)
        mod.__path__ = []
        return mod

    def exec_module(self, module):
        pass


_FINDER = _StubFinder()


def import_reference():
    """Put the reference tree on sys.path (with the stand-ins) and return its
    ``(container._batch, container._core, screen)`` modules; None when the tree is absent."""
    root = reference_root()
    if root is None:
        return None
    for name in STUBBED:
        try:   # a real installation wins over the stand-in
            __import__(name)
        except ImportError:
            if _FINDER not in sys.meta_path:
                sys.meta_path.insert(0, _FINDER)
    if root not in sys.path:
        sys.path.insert(0, root)
    import importlib
    return (importlib.import_module("shepherd_score.container._batch"),
            importlib.import_module("shepherd_score.container._core"),
            importlib.import_module("shepherd_score.screen"))
