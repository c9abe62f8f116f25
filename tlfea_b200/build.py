"""Build recipes for the sm_100a library and the CPU oracle.

``build_library()`` compiles every CUDA source in ``tlfea_b200/csrc`` into the
in-tree shared library ``tlfea_b200/libtlfea_b200.so`` (nvcc cross-compiles for
sm_100a without a GPU).  ``build_oracle()`` compiles the CPU restatement in
``oracle/`` (test infrastructure) into ``oracle/liborc.so`` and a portable
``oracle/liborc_generic.so``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libtlfea_b200.so"
ORACLE = ROOT / "oracle"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O3", "-shared"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: Path, sources) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(Path(s).stat().st_mtime <= t for s in sources)


def library_sources():
    srcs = sorted(CSRC.glob("*.cu"))
    deps = srcs + sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))
    return srcs, deps


def build_library(force: bool = False, verbose: bool = False, extra=None) -> Path:
    """One nvcc per source (in parallel, objects under tlfea_b200/_build/), then one link."""
    srcs, deps = library_sources()
    if not force and _newer(LIB, deps):
        return LIB
    obj_dir = PKG / "_build"
    obj_dir.mkdir(exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]

    def compile_one(src: Path) -> Path:
        obj = obj_dir / (src.stem + ".o")
        cmd = [nvcc(), *ARCH, *compile_flags, *(extra or []), "-c", "-o", str(obj), str(src)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=str(ROOT))
        return obj

    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(compile_one, srcs))
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB), *map(str, objs)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=str(ROOT))
    return LIB


def build_oracle(force: bool = False) -> Path:
    src = ORACLE / "tlfea_oracle.c"
    deps = [src, ORACLE / "tlfea_oracle.h"]
    outs = {
        ORACLE / "liborc.so": ["-O3", "-march=x86-64-v3"],
        ORACLE / "liborc_generic.so": ["-O3"],
    }
    for out, flags in outs.items():
        if not force and _newer(out, deps):
            continue
        cmd = ["gcc", *flags, "-std=c99", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(out),
               str(src), "-lm"]
        subprocess.run(cmd, check=True, cwd=str(ROOT))
    return ORACLE / "liborc.so"


def build_all(force: bool = False) -> None:
    build_oracle(force=force)
    build_library(force=force)


if __name__ == "__main__":
    import sys

    build_all(force="--force" in sys.argv)
    print(LIB)
