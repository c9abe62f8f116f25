"""Regenerate the mesh fixtures from the reference's data files.

Usage: ``python tests/golden/make_golden.py REFERENCE_DIR`` (the reference
checkout); the tests only read the .npz files this writes.

* cube_t10.npz: data/meshes/T10/cube.1.node/.ele (TetGen, 27 nodes, 6 TET10),
  read with the reference's T10 index remap (cpu_utils.cc:596-737).
* beam_t10.npz: data/meshes/T10/beam.vtu (81 nodes, 24 TET10).
"""
import argparse
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
from tlfea_b200 import mesh as M  # noqa: E402


def main():
    ap = argparse.ArgumentParser(description="mesh fixtures from the reference's data files")
    ap.add_argument("reference", type=Path, help="the reference checkout (holds data/meshes/)")
    REF = ap.parse_args().reference
    x, y, z, conn = M.read_tetgen_t10(REF / "data/meshes/T10/cube.1.node", REF / "data/meshes/T10/cube.1.ele")
    np.savez(HERE / "cube_t10.npz", x=x, y=y, z=z, conn=conn)
    x, y, z, conn, ct = M.read_vtu(REF / "data/meshes/T10/beam.vtu")
    np.savez(HERE / "beam_t10.npz", x=x, y=y, z=z, conn=conn)
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    main()
