"""GPU parity of LinearStaticSolver: stiffness (BCs applied) vs the oracle,
CG iterates vs the oracle CG, solution vs a direct solve, positions x += u."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import tlfea_b200 as T
from oracle import oracle as O
from tlfea_b200 import mesh as M

from .helpers import box, lame, make_element, rel

pytestmark = pytest.mark.gpu
LAM, MU = lame()


def _problem(order, nx=10, ny=2, nz=2, load=(0.0, 0.0, -100.0)):
    x, y, z, conn = box(nx, ny, nz, order)
    fixed, f, tip = M.cantilever_loads(x, y, z, load)
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    return el, (x, y, z, conn, fixed, f)


def _oracle_system(x, y, z, conn, fixed, f):
    g, dj = O.dndu_pre(x, y, z, conn)
    off, cols, vals = O.stiffness(x, y, z, conn, g, dj, LAM, MU)
    kv, fb = O.apply_bcs(off, cols, vals, f, fixed)
    return off, cols, kv, fb


@pytest.mark.parametrize("order", [10, 4])
def test_stiffness_and_cg_match_oracle(order):
    el, (x, y, z, conn, fixed, f) = _problem(order)
    s = T.LinearStaticSolver(el, 1e-10, 50000)
    s.Solve()
    off, cols, kv, fb = _oracle_system(x, y, z, conn, fixed, f)
    o2, c2, v2 = s.RetrieveStiffnessCSRToCPU()
    assert np.array_equal(o2, off) and np.array_equal(c2, cols)
    assert rel(v2, kv) < 1e-12
    u_ref, it_ref, res_ref, rc = O.cg(off, cols, kv, fb, 1e-10, 50000)
    assert rc == 0
    it, res = s.GetLastIterCount(), s.GetLastResidual()
    assert res < 1e-10
    # unpreconditioned CG iteration counts move with rounding (exact parity at a
    # fixed count is test_cg_fixed_iteration_count_parity); TET10's matrix-free product
    # rounds differently from an assembled SpMV and moves them further
    assert abs(it - it_ref) <= max(10, (0.10 if order == 10 else 0.05) * it_ref)
    x2, y2, z2 = el.RetrievePositionToCPU()
    u = np.stack([x2 - x, y2 - y, z2 - z], 1).ravel()
    K = sp.csr_matrix((kv, cols, off)).tocsc()
    u_dir = spla.spsolve(K, fb)
    assert rel(u, u_dir) < 1e-7
    assert rel(u, u_ref) < 1e-7
    el.Destroy()


def test_cg_fixed_iteration_count_parity():
    """At a fixed iteration count the CG iterates agree to rounding."""
    el, (x, y, z, conn, fixed, f) = _problem(10)
    s = T.LinearStaticSolver(el, 0.0, 25)  # tol 0: run exactly 25 iterations
    s.Solve()
    off, cols, kv, fb = _oracle_system(x, y, z, conn, fixed, f)
    u_ref, it_ref, res_ref, _ = O.cg(off, cols, kv, fb, 0.0, 25)
    assert s.GetLastIterCount() == it_ref == 25
    assert abs(s.GetLastResidual() - res_ref) < 1e-9 * max(res_ref, 1e-300)
    x2, y2, z2 = el.RetrievePositionToCPU()
    u = np.stack([x2 - x, y2 - y, z2 - z], 1).ravel()
    assert rel(u, u_ref) < 1e-10
    el.Destroy()


def test_zero_load_and_zero_iterations():
    el, (x, y, z, conn, fixed, f) = _problem(10, load=(0.0, 0.0, 0.0))
    s = T.LinearStaticSolver(el, 1e-10, 100)
    s.Solve()
    assert s.GetLastIterCount() == 0 and s.GetLastResidual() == 0.0
    x2, _, _ = el.RetrievePositionToCPU()
    assert np.array_equal(x2, x)
    el.Destroy()


def test_beam_fixture_tip_deflection():
    """beam.vtu (24 TET10, 10x1x1): clamp x=0, load the x=10 face; tip deflection
    within 30% of Euler-Bernoulli PL^3/(3EI) (the reference's only physics check,
    examples/beam_linear_static.cc:219-234; a coarse mesh is stiffer)."""
    from pathlib import Path

    fx = np.load(Path(__file__).parent / "golden" / "beam_t10.npz")
    x, y, z, conn = fx["x"], fx["y"], fx["z"], fx["conn"]
    E_mod, P = 2e9, -1000.0
    fixed, f, tip = M.cantilever_loads(x, y, z, (0.0, 0.0, P))
    el = make_element(x, y, z, conn, E_mod=E_mod, fixed=fixed, f_ext=f)
    s = T.LinearStaticSolver(el, 1e-10, 50000)
    s.Solve()
    _, _, z2 = el.RetrievePositionToCPU()
    delta = abs((z2 - z)[tip].min())
    L, b, h = 10.0, 1.0, 1.0
    delta_eb = abs(P) * L ** 3 / (3 * E_mod * b * h ** 3 / 12)
    assert 0.3 < delta / delta_eb < 1.3
    el.Destroy()


def test_cpp_class_driver_solves_like_the_python_path(tmp_path):
    """The reference's linear-static example flow through the C++ classes
    (include/tlfea/tlfea.hpp): same displacement as a direct solve of the
    oracle's system."""
    import subprocess

    from . import cpp_driver as D

    x, y, z, conn = box(10, 2, 2, 10)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -100.0))
    exe = D.build(tmp_path)
    D.write_input(tmp_path / "in.bin", x, y, z, conn, fixed, f)
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    it, res, u = D.read_output(tmp_path / "out.bin", len(x))
    assert it > 0 and res < 1e-10
    off, cols, kv, fb = _oracle_system(x, y, z, conn, fixed, f)
    u_dir = spla.spsolve(sp.csr_matrix((kv, cols, off)).tocsc(), fb)
    assert rel(u, u_dir) < 1e-7


def _numpy_pcg(K, f, fixed_dofs, iters):
    """Block-Jacobi PCG restated in numpy (3x3 node diagonal blocks of K)."""
    n = K.shape[0]
    Kd = K.toarray() if n <= 6000 else None
    D = np.zeros((n // 3, 3, 3))
    for i in range(n // 3):
        D[i] = np.linalg.inv(Kd[3 * i:3 * i + 3, 3 * i:3 * i + 3])
    prec = lambda r: np.einsum("nij,nj->ni", D, r.reshape(-1, 3)).ravel()
    u = np.zeros(n)
    r = f.copy()
    z = prec(r)
    p = z.copy()
    rz = r @ z
    for _ in range(iters):
        q = K @ p
        a = rz / (p @ q)
        u += a * p
        r -= a * q
        z = prec(r)
        rzn = r @ z
        p = z + (rzn / rz) * p
        rz = rzn
    return u


def test_block_jacobi_pcg_matches_numpy_and_needs_fewer_iterations():
    el, (x, y, z, conn, fixed, f) = _problem(10)
    s = T.LinearStaticSolver(el, 1e-10, 50000)
    s.Solve()
    it_cg = s.GetLastIterCount()
    el.ResetPositions()
    s.SetPreconditioner("block_jacobi")
    s.Solve()
    it_pcg, res = s.GetLastIterCount(), s.GetLastResidual()
    assert res < 1e-10 and it_pcg < it_cg
    x2, y2, z2 = el.RetrievePositionToCPU()
    u = np.stack([x2 - x, y2 - y, z2 - z], 1).ravel()
    off, cols, kv, fb = _oracle_system(x, y, z, conn, fixed, f)
    K = sp.csr_matrix((kv, cols, off))
    assert rel(u, spla.spsolve(K.tocsc(), fb)) < 1e-7
    # fixed iteration count: the iterate matches a numpy restatement
    el.ResetPositions()
    s2 = T.LinearStaticSolver(el, 0.0, 20)
    s2.SetPreconditioner("block_jacobi")
    s2.Solve()
    x3, y3, z3 = el.RetrievePositionToCPU()
    u20 = np.stack([x3 - x, y3 - y, z3 - z], 1).ravel()
    assert rel(u20, _numpy_pcg(K, fb, None, 20)) < 1e-9
    el.Destroy()


@pytest.mark.parametrize("order", [10])  # the matrix-free operator is TET10's (TET4 keeps the assembled K)
def test_matrix_free_operator_matches_the_assembled_stiffness(order):
    """The default matrix-free K p (the SVK tangent applied element by element in every
    CG iteration) against the assembled K of the reference: K x for random x with fixed
    components (their columns dropped, their rows identity), at deformed positions (so
    the tangent's geometric terms are exercised), the CG solution and iteration count, and
    the stiffness retrieved after a matrix-free solve."""
    import torch

    x, y, z, conn = box(12, 3, 2, order)
    fixed, f, _ = M.cantilever_loads(x, y, z, (20.0, -30.0, -100.0))
    out = {}
    for mode in ("assembled", "matrix-free"):
        el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
        r = np.random.default_rng(5)
        xs = [v + 1e-4 * r.standard_normal(v.shape) for v in (x, y, z)]  # deformed, K still positive definite
        el.UpdatePositions(*xs)
        s = T.LinearStaticSolver(el, 1e-10, 50000)
        s.SetOperator(mode)
        s.Solve()
        u = np.stack(el.RetrievePositionToCPU()) - np.stack(xs)
        xv = torch.tensor(r.standard_normal(3 * len(x)), dtype=torch.float64, device="cuda")
        yv = torch.empty_like(xv)
        torch.cuda.synchronize()
        s.Apply(xv.data_ptr(), yv.data_ptr())
        torch.cuda.synchronize()
        Kx = yv.cpu().numpy()
        off, cols, vals = s.RetrieveStiffnessCSRToCPU()
        out[mode] = (u, s.GetLastIterCount(), s.GetLastResidual(), Kx, vals, xv.cpu().numpy())
        del s
        el.Destroy()
    ua, ia, ra, Ka, va, xa = out["assembled"]
    um, im, rm, Km, vm, xm = out["matrix-free"]
    assert np.array_equal(xa, xm)
    assert rel(Km, Ka) < 1e-12
    assert np.array_equal(va, vm)  # K assembled on demand at the matrix-free solve's positions
    assert rm < 1e-10 and abs(im - ia) <= max(2, 0.10 * ia), (im, ia)
    assert rel(um, ua) < 1e-8
