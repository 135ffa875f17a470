"""Build libfss_cuda.so in-tree with nvcc for sm_100a (no GPU needed to build).

    python -m fast_shepherd_score_b200.build [--verbose]

The library statically links the CUDA runtime so it only needs the NVIDIA driver at run
time; the host language binding (``fast_shepherd_score_b200._lib``) loads it with ctypes.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libfss_cuda.so")
SOURCES = ["fss_capi.cu", "fss_align.cu", "fss_align_shape.cu", "fss_align_esp.cu",
           "fss_align_pharm.cu", "fss_align_combo.cu", "fss_eval.cu", "fss_seeds.cu", "fss_score.cu", "fss_probe.cu",
           "fss_static.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; set NVCC or put the CUDA toolkit on PATH")


def sources():
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "fss_cuda.h"))
    return deps


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in sources())


def build(force: bool = False, verbose: bool = False, out: str = None, defines=()) -> str:
    """Compile every source and link ``out`` (default: the package's libfss_cuda.so).
    ``defines`` (e.g. ``["FSS_JB2=3"]``) set the kernels' compile-time tuning macros."""
    target = os.path.abspath(out) if out else LIB
    if not force and target == LIB and not needs_build():
        return LIB
    objdir = (os.path.join(HERE, "_build") if target == LIB else
              os.path.join(os.path.dirname(target), "_build_" + os.path.basename(target)))
    os.makedirs(objdir, exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-cudart", "static",
                    "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if verbose:
        flags += ["-Xptxas", "-v"]
    flags += [f"-D{d}" for d in defines]
    objs = [os.path.join(objdir, src.replace(".cu", ".o")) for src in SOURCES]

    def compile_one(src_obj):
        src, obj = src_obj
        subprocess.run([nvcc(), "-c", os.path.join(CSRC, src), "-o", obj] + flags, check=True)

    # translation units are independent: compile them in parallel
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        list(ex.map(compile_one, zip(SOURCES, objs)))
    tmp = target + ".tmp"
    subprocess.run([nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-cudart", "static"], check=True)
    os.replace(tmp, target)
    return target


if __name__ == "__main__":
    build(force=True, verbose="--verbose" in sys.argv)
    print(LIB)
