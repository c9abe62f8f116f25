"""Build and run the C++ test driver tests/cpp/beam_linear_static.cpp (the
reference's linear-static example flow through include/tlfea/tlfea.hpp)."""
from __future__ import annotations

import struct
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def build(out_dir: Path) -> Path:
    exe = out_dir / "beam_linear_static"
    libdir = ROOT / "tlfea_b200"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "beam_linear_static.cpp"), "-L", str(libdir), "-ltlfea_b200",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True, capture_output=True, text=True)
    return exe


def write_input(path: Path, x, y, z, conn, fixed, f):
    conn_cm = np.ascontiguousarray(np.asarray(conn, np.int32).T).ravel()
    with open(path, "wb") as fh:
        fh.write(struct.pack("iii", len(x), conn.shape[0], len(fixed)))
        for a in (x, y, z):
            fh.write(np.asarray(a, np.float64).tobytes())
        fh.write(conn_cm.tobytes())
        fh.write(np.asarray(fixed, np.int32).tobytes())
        fh.write(np.asarray(f, np.float64).tobytes())


def read_output(path: Path, n_nodes: int):
    b = path.read_bytes()
    it = struct.unpack_from("i", b, 0)[0]
    res = struct.unpack_from("d", b, 4)[0]
    u = np.frombuffer(b, np.float64, 3 * n_nodes, 12)
    return it, res, u
