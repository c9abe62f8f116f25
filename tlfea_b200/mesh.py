"""Mesh utilities on either side of the hot path.

* ``box_mesh``: structured box of nx*ny*nz hex cells, each Kuhn-split into 6
  positively oriented tetrahedra (TET10 midnodes on the half-spacing grid).
  The synthetic beams of the benchmark configurations are built with it.
* ``read_tetgen_t10``: TetGen ``.node`` / ``.ele`` reader with the reference's
  T10 index remap (cpu_utils.cc:596-737).
* ``read_vtu``: ASCII VTU reader for VTK_QUADRATIC_TETRA (24) and VTK_TETRA
  (10) cells (the format of the reference's data/meshes files).
* ``write_vtk``: legacy ASCII VTK writer (WriteOutputVTK, FEAT10Data.cu:759-794).

Connectivity is returned row-major (E, NPE) int32; node coordinates as three
float64 arrays.
"""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np

_PERMS = [(0, 1, 2), (1, 2, 0), (2, 0, 1), (0, 2, 1), (2, 1, 0), (1, 0, 2)]  # first three even
_EDGES = [(0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3)]


def box_counts(nx: int, ny: int, nz: int, order: int = 10):
    m = 2 if order == 10 else 1
    return (m * nx + 1) * (m * ny + 1) * (m * nz + 1), 6 * nx * ny * nz


def box_mesh(nx: int, ny: int, nz: int, order: int = 10, lx: float = 1.0, ly: float = 0.1, lz: float = 0.1):
    """Kuhn-split box.  Node id = (ix*NY + iy)*NZ + iz on the (half-)grid, x slowest.
    Element e = ((cx*ny + cy)*nz + cz)*6 + k; tets k>=3 (odd permutations) have
    vertices 1 and 2 swapped so every detJ is positive."""
    if order not in (4, 10):
        raise ValueError("order must be 4 or 10")
    m = 2 if order == 10 else 1
    NX, NY, NZ = m * nx + 1, m * ny + 1, m * nz + 1
    ix, iy, iz = np.meshgrid(np.arange(NX), np.arange(NY), np.arange(NZ), indexing="ij")
    x = (lx * ix.ravel().astype(np.float64) / float(m * nx))
    y = (ly * iy.ravel().astype(np.float64) / float(m * ny))
    z = (lz * iz.ravel().astype(np.float64) / float(m * nz))
    cx, cy, cz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    base = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1)  # (C, 3)
    C = base.shape[0]
    verts = np.zeros((C, 6, 4, 3), dtype=np.int64)
    for k, perm in enumerate(_PERMS):
        p = base.copy()
        verts[:, k, 0] = p
        for s in range(3):
            p = p.copy()
            p[:, perm[s]] += 1
            verts[:, k, s + 1] = p
        if k >= 3:
            verts[:, k, [1, 2]] = verts[:, k, [2, 1]]
    hv = verts * m
    if order == 10:
        mids = np.stack([(hv[:, :, a] + hv[:, :, b]) // 2 for a, b in _EDGES], axis=2)
        hv = np.concatenate([hv, mids], axis=2)
    ids = (hv[..., 0] * NY + hv[..., 1]) * NZ + hv[..., 2]
    conn = ids.reshape(C * 6, order).astype(np.int32)
    return x, y, z, np.ascontiguousarray(conn)


def remap_tetgen_t10(tg: np.ndarray) -> np.ndarray:
    """TetGen [v0..v3,(3-4),(1-4),(1-2),(2-3),(2-4),(1-3)] -> reference order (cpu_utils.cc:596-611)."""
    return tg[..., [0, 1, 2, 3, 6, 7, 9, 5, 8, 4]]


def read_tetgen_t10(node_file, ele_file):
    """FEAT10_read_nodes / FEAT10_read_elements (cpu_utils.cc:613-737): 0- or
    1-based ids detected from the minimum id."""
    lines = [l.split() for l in Path(node_file).read_text().splitlines() if l.strip() and not l.startswith("#")]
    n, dim = int(lines[0][0]), int(lines[0][1])
    if dim != 3:
        raise ValueError("only 3D nodes are supported")
    rows = [(int(r[0]), float(r[1]), float(r[2]), float(r[3])) for r in lines[1:1 + n]]
    min_id = min(r[0] for r in rows)
    off = 0 if min_id == 0 else 1
    xyz = np.zeros((n, 3))
    for r in rows:
        xyz[r[0] - off] = r[1:]
    lines = [l.split() for l in Path(ele_file).read_text().splitlines() if l.strip() and not l.startswith("#")]
    ne, npe = int(lines[0][0]), int(lines[0][1])
    if npe != 10:
        raise ValueError("only T10 elements (10 nodes) are supported")
    erows = [[int(v) for v in r[:11]] for r in lines[1:1 + ne]]
    min_e = min(r[0] for r in erows)
    min_n = min(min(r[1:]) for r in erows)
    conn = np.zeros((ne, 10), dtype=np.int32)
    for r in erows:
        tg = np.array(r[1:], dtype=np.int32) - (0 if min_n == 0 else 1)
        conn[r[0] - (0 if min_e == 0 else 1)] = remap_tetgen_t10(tg)
    return xyz[:, 0].copy(), xyz[:, 1].copy(), xyz[:, 2].copy(), conn


def _data_array(text: str, name_pat: str):
    m = re.search(r"<DataArray[^>]*" + name_pat + r"[^>]*>(.*?)</DataArray>", text, re.S)
    if not m:
        raise ValueError(f"DataArray {name_pat} not found")
    # values come before any nested element (e.g. <InformationKey>)
    return np.array(m.group(1).split("<", 1)[0].split(), dtype=np.float64)


def read_vtu(path):
    """ASCII VTU: returns x, y, z, conn, cell_type for the first tet cell type present."""
    text = Path(path).read_text()
    pts = _data_array(text, r'Name="Points"').reshape(-1, 3)
    cells = re.search(r"<Cells>(.*?)</Cells>", text, re.S).group(1)
    conn_flat = _data_array(cells, r'Name="connectivity"').astype(np.int64)
    offs = _data_array(cells, r'Name="offsets"').astype(np.int64)
    types = _data_array(cells, r'Name="types"').astype(np.int64)
    starts = np.concatenate([[0], offs[:-1]])
    for ct, npe in ((24, 10), (10, 4)):
        sel = np.nonzero(types == ct)[0]
        if sel.size:
            conn = np.stack([conn_flat[starts[s]:starts[s] + npe] for s in sel]).astype(np.int32)
            return pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy(), conn, ct
    raise ValueError("no TET10 or TET4 cells")


def write_vtk(path, x, y, z, conn):
    """Legacy ASCII VTK (FEAT10Data.cu:759-794 layout; type 24 for T10, 10 for T4)."""
    npe = conn.shape[1]
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 3.0\n%s mesh output\nASCII\nDATASET UNSTRUCTURED_GRID\n"
                % ("T10" if npe == 10 else "T4"))
        f.write(f"POINTS {len(x)} float\n")
        for i in range(len(x)):
            f.write(f"{x[i]:g} {y[i]:g} {z[i]:g}\n")
        f.write(f"CELLS {conn.shape[0]} {conn.shape[0] * (npe + 1)}\n")
        for row in conn:
            f.write(f"{npe} " + " ".join(str(int(v)) for v in row) + " \n")
        f.write(f"CELL_TYPES {conn.shape[0]}\n")
        f.write(("24\n" if npe == 10 else "10\n") * conn.shape[0])


def cantilever_loads(x, y, z, total_force=(0.0, 0.0, -100.0), tol_frac=1e-9):
    """Fixed nodes at x = min(x) and the external force split equally over the
    x = max(x) face nodes (the clamped-tip-loaded cantilever of the benchmark configurations)."""
    L = x.max() - x.min()
    tol = max(tol_frac * L, 1e-12)
    fixed = np.nonzero(np.abs(x - x.min()) < tol)[0].astype(np.int32)
    tip = np.nonzero(np.abs(x - x.max()) < tol)[0]
    f = np.zeros(3 * len(x))
    for d in range(3):
        f[3 * tip + d] = total_force[d] / len(tip)
    return fixed, f, tip


def random_beam(seed: int, nx_range=(8, 64), ny_range=(2, 8), h=0.01, E_range=(1e6, 1e9), nu_range=(0.2, 0.45),
                load_range=(1.0, 500.0), order: int = 10):
    """One seeded cantilever of the uneven batch: nx ~ U{nx_range}, ny = nz ~
    U{ny_range}, cross-section ny*h x ny*h, length 10*ny*h (cell length
    10*ny*h/nx), E log-uniform, nu uniform, tip force with direction uniform on
    the unit sphere and uniform magnitude, split over the free-end nodes;
    the x = 0 face is clamped.  Returns a dict."""
    r = np.random.default_rng(seed)
    nx = int(r.integers(nx_range[0], nx_range[1] + 1))
    ny = int(r.integers(ny_range[0], ny_range[1] + 1))
    E = float(np.exp(r.uniform(np.log(E_range[0]), np.log(E_range[1]))))
    nu = float(r.uniform(*nu_range))
    d = r.standard_normal(3)
    d /= np.linalg.norm(d)
    mag = float(r.uniform(*load_range))
    w = ny * h
    x, y, z, conn = box_mesh(nx, ny, ny, order, 10.0 * w, w, w)
    fixed, f, tip = cantilever_loads(x, y, z, tuple(mag * d))
    return {"x": x, "y": y, "z": z, "conn": conn, "fixed": fixed, "f": f, "E": E, "nu": nu, "nx": nx, "ny": ny,
            "direction": d, "magnitude": mag}
