"""Recipe: the reference's own CUDA build, as a parity harness (test infrastructure).

Compiles the reference's unchanged element and solver sources

    src/elements/FEAT10Data.cu   src/elements/FEAT4Data.cu
    src/solvers/LinearStaticSolver.cu
    src/solvers/SyncedNesterov.cu   src/solvers/SyncedAdamW.cu   src/solvers/SyncedAdamWNocoop.cu

for sm_100a, where they lie in the reference checkout, against the project-written
stand-ins for its two absent dependencies (``oracle/refshim/Eigen/Dense`` for the Eigen
subset it uses, ``oracle/refshim/MoPhiEssentials.h`` for the un-vendored MoPhiEssentials
submodule), together with ``oracle/ref_harness.cu`` (a C ABI over the reference's classes).
The flags are the reference's own (CMakeLists.txt:5-28: C++17, ``-Xcompiler -fPIC
--expt-relaxed-constexpr``, no fast-math) with the architecture set to sm_100a. It links
cuSPARSE and cuBLAS as the reference does.

Output: ``oracle/_ref/libtlfea_ref.so`` (git-ignored; it travels with the working tree).
Nothing is copied from the reference into this repository.

Usage: ``python oracle/build_ref.py [--reference DIR] [--force]``; DIR defaults to the
``TLFEA_REFERENCE`` environment variable, else /root/reference (where this project's build
container mounts the reference checkout).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "_ref"
LIB = OUT_DIR / "libtlfea_ref.so"
SHIM = HERE / "refshim"
HARNESS = HERE / "ref_harness.cu"

REF_SOURCES = [
    "src/elements/FEAT10Data.cu",
    "src/elements/FEAT4Data.cu",
    "src/solvers/LinearStaticSolver.cu",
    "src/solvers/SyncedNesterov.cu",
    "src/solvers/SyncedAdamW.cu",
    "src/solvers/SyncedAdamWNocoop.cu",
]
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC", "-lineinfo"]


def default_reference() -> Path:
    return Path(os.environ.get("TLFEA_REFERENCE", "/root/reference"))


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _up_to_date(ref: Path) -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    deps = [ref / s for s in REF_SOURCES] + [HARNESS, *SHIM.rglob("*")]
    return all(p.stat().st_mtime <= t for p in deps if p.is_file())


def build(reference: Path | None = None, force: bool = False, jobs: int = 7) -> Path | None:
    """Builds oracle/_ref/libtlfea_ref.so; returns None when the reference checkout is absent."""
    ref = Path(reference) if reference is not None else default_reference()
    if not (ref / REF_SOURCES[0]).exists():
        return None
    if not force and _up_to_date(ref):
        return LIB
    OUT_DIR.mkdir(exist_ok=True)
    obj_dir = OUT_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    inc = ["-I", str(SHIM), "-I", str(ref / "src")]
    units = [(ref / s, obj_dir / (Path(s).stem + ".o")) for s in REF_SOURCES] + [(HARNESS, obj_dir / "harness.o")]

    def compile_one(unit):
        src, obj = unit
        subprocess.run([nvcc, *FLAGS, *inc, "-c", str(src), "-o", str(obj)], check=True)
        return obj

    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(compile_one, units))
    cuda_lib = Path(nvcc).resolve().parent.parent / "lib64"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC", "-o",
                    str(LIB), *map(str, objs), f"-L{cuda_lib}", "-lcusparse", "-lcublas",
                    "-Xlinker", f"-rpath,{cuda_lib}"], check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", type=Path, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    out = build(a.reference, a.force)
    print(out if out else "reference checkout not found: nothing built")
