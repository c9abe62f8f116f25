"""Inputs of the reference-run fixtures (shared by the generator and the tests).

Each case fixes a mesh, a material, boundary conditions and seeded perturbations; the
generator (``make_ref_fixtures.py``) feeds them to the reference's own CUDA build and the
tests feed the same inputs to this library and to the oracle.

Cases (sizes from the benchmark configurations):

* ``cube_t10`` -- the reference's own TetGen cube (data/meshes/T10/cube.1.*, 27 nodes,
  6 TET10) with the parameters of examples/test_feat10_nesterov.cc:28-30,78-104
  (E = 7e8, nu = 0.33, rho = 2700; z = 0 clamped; 1000 N on DOF 3*6+0).
* ``cfg1_t10`` / ``cfg1_t4`` -- the 1.0 x 0.1 x 0.1 m cantilever, 10x2x2 cells
  (240 elements), E = 1e7, nu = 0.3, rho = 1000, x = 0 clamped, 100 N in -z over the
  x = 1 face.
* ``cfg4_t10`` / ``cfg4_t4`` -- the same beam with 40x8x8 cells (15,360 elements).
* ``cfg2_t10`` / ``cfg2_t4`` -- 200x20x20 cells (480,000 elements; 674,081 TET10 nodes,
  88,641 TET4 nodes), tip load magnitude U[10, 1000] N in -z from seed 0.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from tlfea_b200 import mesh as M

HERE = Path(__file__).resolve().parent

# SyncedNesterovParams with zero tolerances: both sides run 2 x 40 inner iterations per step.
NESTEROV_FIXED = (1.0e-8, 1e14, 0.0, 0.0, 2, 40, 1.0e-3)
# examples/test_feat10_nesterov.cc:189
NESTEROV_REF = (1.0e-8, 1e14, 1.0e-6, 1.0e-6, 5, 300, 1.0e-3)
# examples/test_feat10_adamw.cc:189
ADAMW_REF = (2e-4, 0.9, 0.999, 1e-8, 1e-4, 0.995, 1e-1, 1e-6, 1e14, 5, 500, 1e-3, 10, 0.0)
# AdamW without early exit and with eps = 1: with eps = 1e-8 the normalised step turns
# rounding-level gradients of unloaded DOFs into full steps, so two summation orders
# (or two runs of the reference's atomics) do not agree; with eps = 1 the map is smooth.
ADAMW_FIXED = (2e-4, 0.9, 0.999, 1.0, 1e-4, 0.995, 0.0, 0.0, 1e4, 2, 60, 1e-3, 10, 0.0)

SMALL = ("cube_t10", "cfg1_t10", "cfg1_t4")
MID = ("cfg4_t10", "cfg4_t4")
LARGE = ("cfg2_t10", "cfg2_t4")
ALL = SMALL + MID + LARGE


def fixture_path(name: str) -> Path:
    return HERE / f"ref_{name}.npz"


def case(name: str) -> dict:
    """Mesh, material, boundary conditions of a case (no GPU, no reference needed)."""
    if name == "cube_t10":
        fx = np.load(HERE / "cube_t10.npz")
        x, y, z, conn = fx["x"], fx["y"], fx["z"], fx["conn"]
        fixed = np.nonzero(np.abs(z) < 1e-8)[0].astype(np.int32)
        f = np.zeros(3 * len(x))
        f[3 * 6 + 0] = 1000.0
        E_mod, nu, rho, scale = 7e8, 0.33, 2700.0, 1e-3
    else:
        cfg, tet = name.split("_")
        order = 10 if tet == "t10" else 4
        cells = {"cfg1": (10, 2, 2), "cfg4": (40, 8, 8), "cfg2": (200, 20, 20)}[cfg]
        x, y, z, conn = M.box_mesh(*cells, order)
        load = 100.0
        if cfg == "cfg2":
            load = float(np.random.default_rng(0).uniform(10.0, 1000.0))
        fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -load))
        E_mod, nu, rho, scale = 1e7, 0.3, 1000.0, 1e-4
    return dict(x=x, y=y, z=z, conn=np.ascontiguousarray(conn, np.int32), fixed=fixed, f=f, E=E_mod, nu=nu,
                rho=rho, scale=scale)


def perturbed(c: dict, seed: int = 1):
    """Seeded Gaussian perturbation of the positions (scale relative to the mesh size)."""
    r = np.random.default_rng(seed)
    n = len(c["x"])
    return tuple(c[k] + c["scale"] * r.standard_normal(n) for k in ("x", "y", "z"))


def generic_load(c: dict):
    """The configuration-1 cantilever with a load that is not aligned with an axis."""
    fixed, f, _ = M.cantilever_loads(c["x"], c["y"], c["z"], (30.0, -50.0, -100.0))
    return fixed, f


def projections(n: int, k: int = 16, seed: int = 7) -> np.ndarray:
    """k seeded Gaussian directions of length n (size-independent checks of long vectors)."""
    return np.random.default_rng(seed).standard_normal((k, n))


def sample_index(n: int, k: int = 2048, seed: int = 11) -> np.ndarray:
    return np.sort(np.random.default_rng(seed).choice(n, size=min(k, n), replace=False))


def summary(v: np.ndarray) -> dict:
    """Norm, projections and a sample of a long vector."""
    v = np.asarray(v, np.float64)
    return {"norm": np.linalg.norm(v), "proj": projections(len(v)) @ v, "sample": v[sample_index(len(v))]}
