"""The C-ABI library loads (no GPU needed) and exports every function include/fss_cuda.h
declares; the ctypes descriptor matches the C struct layout."""
import ctypes
import os
import re

from fast_shepherd_score_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "fss_cuda.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fss_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = _declared()
    assert "fss_align" in names and len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTED)


def test_abi_version_and_limits():
    lib = _lib.load()
    assert lib.fss_abi_version() == 3
    assert lib.fss_max_points() >= 1024


def test_descriptor_layout_matches_header():
    # 4 int32, 19 pointers, 4 floats, 6 pointers, 7 int32, 1 pointer with natural alignment
    fields = [f for f, _ in _lib.AlignDesc._fields_]
    txt = open(os.path.join(ROOT, "include", "fss_cuda.h")).read()
    body = txt[txt.index("typedef struct fss_align_desc"):txt.index("} fss_align_desc;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    decl = re.findall(r"(?:const\s+)?(?:int32_t|float)\s*\*?\s*([^;]+);", body)
    hdr = [n.strip().lstrip("*").strip() for d in decl for n in d.split(",")]
    hdr = [h.lstrip("*").strip() for h in hdr]
    assert hdr == fields
    assert ctypes.sizeof(_lib.AlignDesc) % 8 == 0


def test_invalid_arguments_raise_without_gpu():
    lib = _lib.load()
    # argument validation happens before any CUDA call
    rc = lib.fss_pick_best(None, None, None, -1, 1, None, None, None, None)
    assert rc == _lib.FSS_ERR_INVALID
    assert b"fss_pick_best" in lib.fss_last_error()
    rc = lib.fss_seeds(None, None, None, None, None, None, 4, 3, None, 0, 0, None, None, None)
    assert rc == _lib.FSS_ERR_INVALID
