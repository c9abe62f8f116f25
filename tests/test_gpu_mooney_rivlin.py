"""Mooney-Rivlin (SetMooneyRivlin, MooneyRivlin.cuh:46-104) on the GPU against
the oracle: the fused internal force (FP64 rel 1e-10, FP32 rel 1e-5) with and
without Kelvin-Voigt damping, CalcP / CalcInternalForce, the allocation-free
entry point, a fixed-count Nesterov trajectory, and the Mooney-Rivlin tangent
of LinearStaticSolver."""
import ctypes as C

import numpy as np
import pytest

import tlfea_b200 as T
from oracle import oracle as O
from tlfea_b200 import _capi
from tlfea_b200 import mesh as M

from .helpers import E_MOD, NU, RHO, box, make_element, perturb, rel

pytestmark = pytest.mark.gpu

MR = (2.0e6, 5.0e5, 5.0e7)  # mu10, mu01, kappa
TOL64, TOL32 = 1e-10, 1e-5


def _element(order, nx=9, ny=3, nz=2, eta=0.0, lamd=0.0, **kw):
    x, y, z, conn = box(nx, ny, nz, order)
    el = make_element(x, y, z, conn, eta=eta, lamd=lamd, **kw)
    el.SetMooneyRivlin(*MR)
    return el, (x, y, z, conn)


@pytest.mark.parametrize("order", [10, 4])
@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_mooney_rivlin_force_matches_oracle(order, prec, tol):
    import torch

    el, (x, y, z, conn) = _element(order, eta=2.0e3, lamd=5.0e2)
    el.SetForcePrecision(prec)
    xs = perturb(x, y, z, 3e-3, 8)
    el.UpdatePositions(*xs)
    g, dj = O.dndu_pre(x, y, z, conn)
    v = np.random.default_rng(4).standard_normal(3 * len(x)) * 0.1
    dv = torch.tensor(v, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    el.ComputeInternalForce()
    f = el.RetrieveInternalForceToCPU()
    el.ComputeInternalForce(dv.data_ptr())
    f_damp = el.RetrieveInternalForceToCPU()
    with O.mooney_rivlin(*MR):
        f_ref = O.force(*xs, conn, g, dj, 0.0, 0.0)
        f_damp_ref = O.force(*xs, conn, g, dj, 0.0, 0.0, 2.0e3, 5.0e2, v)
    assert rel(f, f_ref) < tol
    assert rel(f_damp, f_damp_ref) < tol
    # not the SVK force
    lam = (E_MOD * NU) / ((1 + NU) * (1 - 2 * NU))
    assert rel(O.force(*xs, conn, g, dj, lam, E_MOD / (2 * (1 + NU))), f_ref) > 1e-3
    el.Destroy()


@pytest.mark.parametrize("order", [10, 4])
def test_mooney_rivlin_calc_p_noalloc_and_rigid_motion(order):
    import torch

    el, (x, y, z, conn) = _element(order)
    g, dj = O.dndu_pre(x, y, z, conn)
    xs = perturb(x, y, z, 2e-3, 3)
    el.UpdatePositions(*xs)
    el.CalcP()
    with O.mooney_rivlin(*MR):
        _, P = O.calc_p(*xs, conn, g, 0.0, 0.0)
        f_ref = O.force(*xs, conn, g, dj, 0.0, 0.0)
    nqp = 5 if order == 10 else 1
    assert rel(el.RetrievePFromFToCPU(), P.reshape(-1, nqp, 3, 3).transpose(0, 1, 3, 2)) < TOL64
    el.CalcInternalForce()
    assert rel(el.RetrieveInternalForceToCPU(), f_ref) < TOL64
    out = torch.zeros(3 * len(x), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _capi.call("tlfea_element_compute_internal_force_noalloc", el._handle(), None, C.c_void_p(out.data_ptr()))
    assert rel(out.cpu().numpy(), f_ref) < TOL64
    th = 0.6
    R = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    el.UpdatePositions(*(R @ np.stack([x, y, z]) + 0.2))
    el.ComputeInternalForce()
    assert np.abs(el.RetrieveInternalForceToCPU()).max() < 1e-8 * np.abs(f_ref).max()
    el.Destroy()


def test_mooney_rivlin_nesterov_fixed_iterations():
    """Zero inner tolerance: the GPU Nesterov trajectory with the Mooney-Rivlin
    law against the oracle's (same iteration counts)."""
    params = (1.0e-8, 1e14, 0.0, 0.0, 2, 40, 1.0e-3)
    x, y, z, conn = box(10, 2, 2, 10)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -100.0))
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    el.SetMooneyRivlin(*MR)
    s = T.SyncedNesterovSolver(el, el.get_n_constraint())
    s.Setup()
    s.SetParameters(T.SyncedNesterovParams(*params))
    with O.mooney_rivlin(*MR):
        m = O.OracleModel(x, y, z, conn, E_MOD, NU, RHO, fixed, f)
        m.set_parameters()
        for _ in range(2):
            s.Solve()
            st = m.nesterov_solve(*params)
            assert s.GetStats()["inner_iters_total"] == st["inner_iters_total"] == 80
    xg = el.RetrievePositionToCPU()
    du = np.stack([xg[0] - x, xg[1] - y, xg[2] - z])
    assert rel(du, np.stack([m.x - x, m.y - y, m.z - z])) < 1e-8
    el.Destroy()


@pytest.mark.parametrize("order", [10, 4])
def test_mooney_rivlin_stiffness_and_linear_static_solve(order):
    """LinearStaticSolver on a Mooney-Rivlin element: the tangent assembled at
    deformed positions against the oracle's, and the solve against a direct one."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    x, y, z, conn = box(8, 2, 2, order)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -100.0))
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    el.SetMooneyRivlin(*MR)
    xs = perturb(x, y, z, 1e-3, 21)
    el.UpdatePositions(*xs)
    s = T.LinearStaticSolver(el, 1e-11, 50000)
    s.Solve()
    g, dj = O.dndu_pre(x, y, z, conn)
    with O.mooney_rivlin(*MR):
        off, cols, vals = O.stiffness(*xs, conn, g, dj, 0.0, 0.0)
    kv, fb = O.apply_bcs(off, cols, vals, f, fixed)
    o2, c2, v2 = s.RetrieveStiffnessCSRToCPU()
    assert np.array_equal(o2, off) and np.array_equal(c2, cols)
    assert rel(v2, kv) < 1e-12
    el.Destroy()
    # at the reference configuration (stress free, K positive definite) the CG
    # solve matches a direct solve of the oracle's system
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    el.SetMooneyRivlin(*MR)
    s = T.LinearStaticSolver(el, 1e-11, 50000)
    s.Solve()
    assert s.GetLastResidual() < 1e-11
    with O.mooney_rivlin(*MR):
        off, cols, vals = O.stiffness(x, y, z, conn, g, dj, 0.0, 0.0)
    kv, fb = O.apply_bcs(off, cols, vals, f, fixed)
    x2, y2, z2 = el.RetrievePositionToCPU()
    u = np.stack([x2 - x, y2 - y, z2 - z], 1).ravel()
    u_dir = spla.spsolve(sp.csr_matrix((kv, cols, off)).tocsc(), fb)
    assert rel(u, u_dir) < 1e-7
    el.Destroy()
