"""GPU parity of the element path (CUDA via the C ABI vs the CPU oracle).

Tolerances: FP64 mode rel 1e-10, FP32 force mode rel 1e-5 (norm-wise, against
the FP64 oracle); integer patterns bit-exact."""
import numpy as np
import pytest

import tlfea_b200 as T
from oracle import oracle as O

from .helpers import RHO, box, lame, make_element, perturb, rel

pytestmark = pytest.mark.gpu
LAM, MU = lame()
TOL64, TOL32 = 1e-10, 1e-5


def _setup(order, nx=10, ny=2, nz=2, seed=0, scale=2e-3):
    x, y, z, conn = box(nx, ny, nz, order)
    el = make_element(x, y, z, conn)
    xp, yp, zp = perturb(x, y, z, scale, seed)
    return el, (x, y, z, conn), (xp, yp, zp)


@pytest.mark.parametrize("order", [10, 4])
def test_dndu_and_detj_match_oracle(order):
    el, (x, y, z, conn), _ = _setup(order)
    g, dj = O.dndu_pre(x, y, z, conn)
    G = O.grad_to_array(g, conn.shape[0], order)
    assert rel(el.RetrieveDnDuPreToCPU(), G) < 1e-14
    nqp = 5 if order == 10 else 1
    assert rel(el.RetrieveDetJToCPU(), dj.reshape(-1, nqp)) < 1e-14
    assert np.array_equal(el.RetrieveConnectivityToCPU(), conn)
    el.Destroy()


@pytest.mark.parametrize("order", [10, 4])
def test_mass_csr_matches_oracle(order):
    el, (x, y, z, conn), _ = _setup(order)
    g, dj = O.dndu_pre(x, y, z, conn)
    off, cols, vals = O.mass(conn, dj, len(x), RHO)
    o2, c2, v2 = el.RetrieveMassCSRToCPU()
    assert np.array_equal(o2, off) and np.array_equal(c2, cols)
    assert rel(v2, vals) < 1e-13
    el.Destroy()


@pytest.mark.parametrize("order", [10, 4])
def test_calc_p_and_calc_internal_force(order):
    el, (x, y, z, conn), xs = _setup(order)
    g, dj = O.dndu_pre(x, y, z, conn)
    el.UpdatePositions(*xs)
    el.CalcP()
    _, P = O.calc_p(*xs, conn, g, LAM, MU)
    nqp = 5 if order == 10 else 1
    P_ref = P.reshape(-1, nqp, 3, 3).transpose(0, 1, 3, 2)
    assert rel(el.RetrievePFromFToCPU(), P_ref) < TOL64
    el.CalcInternalForce()
    f_ref = O.internal_force_from_p(conn, g, dj, P, len(x))
    assert rel(el.RetrieveInternalForceToCPU(), f_ref) < TOL64
    # the reference does not clear f_int: a second call doubles it
    el.CalcInternalForce()
    assert rel(el.RetrieveInternalForceToCPU(), 2 * f_ref) < TOL64
    el.Destroy()


@pytest.mark.parametrize("order", [10, 4])
@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_fused_internal_force(order, prec, tol):
    el, (x, y, z, conn), xs = _setup(order, 12, 3, 3, seed=3)
    g, dj = O.dndu_pre(x, y, z, conn)
    el.UpdatePositions(*xs)
    el.SetForcePrecision(prec)
    el.ComputeInternalForce()
    f = el.RetrieveInternalForceToCPU()
    f_ref = O.force(*xs, conn, g, dj, LAM, MU)
    assert rel(f, f_ref) < tol
    # deterministic: a second evaluation is bitwise identical
    el.ComputeInternalForce()
    assert np.array_equal(el.RetrieveInternalForceToCPU(), f)
    el.Destroy()


@pytest.mark.parametrize("order", [10, 4])
def test_fused_force_with_kelvin_voigt_damping(order):
    x, y, z, conn = box(8, 2, 2, order)
    el = make_element(x, y, z, conn, eta=2.0e3, lamd=5.0e2)
    xs = perturb(x, y, z, 1e-3, 5)
    el.UpdatePositions(*xs)
    v = np.random.default_rng(9).standard_normal(3 * len(x)) * 0.1
    import torch

    dv = torch.tensor(v, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    el.ComputeInternalForce(dv.data_ptr())
    g, dj = O.dndu_pre(x, y, z, conn)
    f_ref = O.force(*xs, conn, g, dj, LAM, MU, 2.0e3, 5.0e2, v)
    assert rel(el.RetrieveInternalForceToCPU(), f_ref) < TOL64
    el.Destroy()


@pytest.mark.parametrize("kernel", ["compact", "direct", "pipeline"])
@pytest.mark.parametrize("order", [10, 4])
@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_force_kernel_variants_match_oracle(kernel, order, prec, tol):
    """Every launch variant of the fused force kernel -- the compact geometry
    stream (J^-1 per QP) among them -- against the oracle, with and without
    Kelvin-Voigt damping, and bitwise repeatable."""
    import torch

    x, y, z, conn = box(9, 3, 2, order)
    el = make_element(x, y, z, conn, eta=2.0e3, lamd=5.0e2)
    el.SetLaunchConfig(kernel)
    el.SetForcePrecision(prec)
    xs = perturb(x, y, z, 2e-3, 6)
    el.UpdatePositions(*xs)
    g, dj = O.dndu_pre(x, y, z, conn)
    el.ComputeInternalForce()
    f = el.RetrieveInternalForceToCPU()
    assert rel(f, O.force(*xs, conn, g, dj, LAM, MU)) < tol
    el.ComputeInternalForce()
    assert np.array_equal(el.RetrieveInternalForceToCPU(), f)
    v = np.random.default_rng(2).standard_normal(3 * len(x)) * 0.1
    dv = torch.tensor(v, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    el.ComputeInternalForce(dv.data_ptr())
    f_ref = O.force(*xs, conn, g, dj, LAM, MU, 2.0e3, 5.0e2, v)
    assert rel(el.RetrieveInternalForceToCPU(), f_ref) < tol
    el.Destroy()


def test_compact_kernel_large_mesh_rigid_motion():
    """200x20x20 TET10 on the compact stream: a rigid rotation gives zero force,
    and the FP32 and FP64 forces agree with the gradient-stream kernel."""
    x, y, z, conn = box(200, 20, 20, 10)
    el = make_element(x, y, z, conn, mass=False)
    el.SetLaunchConfig("compact")
    th = 0.4
    R = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    el.UpdatePositions(*(R @ np.stack([x, y, z]) + 0.5))
    el.ComputeInternalForce()
    f_rigid = el.RetrieveInternalForceToCPU()
    xs = perturb(x, y, z, 1e-4, 4)
    el.UpdatePositions(*xs)
    out = {}
    for k in ("compact", "tma"):
        el.SetLaunchConfig(k)
        for prec in ("fp64", "fp32"):
            el.SetForcePrecision(prec)
            el.ComputeInternalForce()
            out[k, prec] = el.RetrieveInternalForceToCPU()
    assert np.abs(f_rigid).max() < 1e-8 * np.abs(out["compact", "fp64"]).max()
    assert rel(out["compact", "fp64"], out["tma", "fp64"]) < 1e-12
    assert rel(out["compact", "fp32"], out["tma", "fp64"]) < TOL32
    el.Destroy()


def test_cube_fixture_matches_oracle():
    from pathlib import Path

    fx = np.load(Path(__file__).parent / "golden" / "cube_t10.npz")
    x, y, z, conn = fx["x"], fx["y"], fx["z"], fx["conn"]
    el = make_element(x, y, z, conn)
    g, dj = O.dndu_pre(x, y, z, conn)
    assert rel(el.RetrieveDetJToCPU(), dj.reshape(-1, 5)) < 1e-14
    xs = perturb(x, y, z, 1e-2, 11)
    el.UpdatePositions(*xs)
    el.ComputeInternalForce()
    assert rel(el.RetrieveInternalForceToCPU(), O.force(*xs, conn, g, dj, LAM, MU)) < TOL64
    el.Destroy()


@pytest.mark.parametrize("order", [10, 4])
def test_large_mesh_properties(order):
    """The 200x20x20 cantilever (480,000 TET10 elements): rigid motion gives zero force,
    FP32 vs FP64 agree, and every node gets written."""
    x, y, z, conn = box(200, 20, 20, order)
    el = make_element(x, y, z, conn, mass=False)
    th = 0.4
    R = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    Xr = R @ np.stack([x, y, z]) + 0.5
    el.UpdatePositions(*Xr)
    el.ComputeInternalForce()
    f = el.RetrieveInternalForceToCPU()
    xs = perturb(x, y, z, 1e-4, 4)
    el.UpdatePositions(*xs)
    el.ComputeInternalForce()
    f64 = el.RetrieveInternalForceToCPU()
    assert np.abs(f).max() < 1e-8 * np.abs(f64).max()
    el.SetForcePrecision("fp32")
    el.ComputeInternalForce()
    f32 = el.RetrieveInternalForceToCPU()
    assert rel(f32, f64) < TOL32
    el.Destroy()


def test_errors_are_reported():
    x, y, z, conn = box(2, 1, 1, 10)
    el = T.GPU_FEAT10_Data(conn.shape[0], len(x))
    el.Initialize()
    with pytest.raises(T.TLFEAError):
        el.SetDensity(1.0)  # before Setup
    with pytest.raises(T.TLFEAError):
        el.SetExternalForce(np.zeros(5))  # size mismatch
    el.Destroy()


def test_gravity_body_force_is_mass_row_sums_times_g():
    """AddGravity adds (sum_j M_ij) g to f_ext; the total equals rho V g."""
    x, y, z, conn = box(10, 2, 2, 10)
    f0 = np.random.default_rng(4).standard_normal(3 * len(x))
    el = make_element(x, y, z, conn, f_ext=f0)
    g = (0.0, -2.0, -9.81)
    el.AddGravity(*g)
    f = el.RetrieveExternalForceToCPU()
    _, dj = O.dndu_pre(x, y, z, conn)
    off, cols, vals = O.mass(conn, dj, len(x), RHO)
    rows = np.add.reduceat(vals, off[:-1])
    ref = f0 + np.outer(rows, g).ravel()
    assert rel(f, ref) < 1e-13
    total = (f - f0).reshape(-1, 3).sum(0)
    assert np.allclose(total, RHO * 1.0 * 0.1 * 0.1 * np.array(g), rtol=1e-12, atol=1e-12)
    el.Destroy()
