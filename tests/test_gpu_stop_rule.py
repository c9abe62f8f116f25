"""The relative-residual stop rule of the first-order solvers:
||(f_int - f_ext)_free|| / ||f_ext|| < tol, evaluated in FP64 at the positions
of the last force evaluation, which the solve keeps.  The reported residual is
checked against the oracle's static residual at the GPU's final positions."""
import ctypes as C

import numpy as np
import pytest

import tlfea_b200 as T
from oracle import oracle as O
from tlfea_b200 import _capi
from tlfea_b200 import mesh as M

from .helpers import E_MOD, NU, RHO, box, make_element

pytestmark = pytest.mark.gpu

NESTEROV = (1.0e-8, 1e14, 1.0e-6, 1.0e-6, 5, 300, 1.0e-3)  # test_feat10_nesterov.cc:189


def _cfg1():
    x, y, z, conn = box(10, 2, 2, 10)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -100.0))
    return x, y, z, conn, fixed, f


def _oracle_residual(x, y, z, conn, fixed, f, xs):
    om = O.OracleModel(x, y, z, conn, E_MOD, NU, RHO, fixed, f)
    om.x[:], om.y[:], om.z[:] = xs
    return om.static_residual()


def test_rule_fires_at_the_first_evaluation_when_loose():
    x, y, z, conn, fixed, f = _cfg1()
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    s = T.SyncedNesterovSolver(el, el.get_n_constraint())
    s.Setup()
    s.SetParameters(T.SyncedNesterovParams(*NESTEROV))
    s.SetRelativeResidualStop(2.0)
    s.Solve()
    st = s.GetStats()
    assert st["stop_rule_met"] == 1 and st["inner_iters_total"] == 1 and st["outer_iters"] == 1
    # first evaluation at the reference positions: f_int = 0 up to the rounding of
    # F = (dX/dxi) J^-1 = I (E ~ 1e7 times 1e-16), so ||f_free|| / ||f|| = 1 to ~1e-11
    assert st["rel_residual"] == pytest.approx(1.0, rel=1e-10)
    xs = el.RetrievePositionToCPU()
    assert all(np.array_equal(a, b) for a, b in zip(xs, (x, y, z)))
    el.Destroy()


def _step_hessian_lmax(x, y, z, conn, fixed, dt, rho_alm, iters=300):
    """Largest eigenvalue of the inner problem's Hessian M/dt + dt K (+ dt^2 rho on
    fixed DOFs), by power iteration on the oracle's matrices."""
    import scipy.sparse as sp

    from .helpers import lame

    lam, mu = lame()
    g, dj = O.dndu_pre(x, y, z, conn)
    off, cols, vals = O.stiffness(x, y, z, conn, g, dj, lam, mu)
    K = sp.csr_matrix((vals, cols, off))
    moff, mcol, mval = O.mass(conn, dj, len(x), RHO)
    Mn = sp.csr_matrix((mval, mcol, moff))
    M = sp.kron(Mn, sp.identity(3)).tocsr()
    d = np.zeros(3 * len(x))
    for n in fixed:
        d[3 * n:3 * n + 3] = dt * dt * rho_alm
    H = M / dt + dt * K + sp.diags(d)
    v = np.random.default_rng(0).standard_normal(H.shape[0])
    for _ in range(iters):
        v = H @ v
        v /= np.linalg.norm(v)
    return float(v @ (H @ v))


def test_rule_ends_a_quasi_static_solve_at_a_checked_residual():
    """dt = 1 makes each inner problem nearly static; alpha from the largest
    eigenvalue of its Hessian.  The rule ends the solve once the static residual
    is below 0.5, and the reported value is the oracle's at the final positions."""
    x, y, z, conn, fixed, f = _cfg1()
    dt, rho_alm = 1.0, 1e6
    alpha = 0.9 / _step_hessian_lmax(x, y, z, conn, fixed, dt, rho_alm)
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    s = T.SyncedNesterovSolver(el, el.get_n_constraint())
    s.Setup()
    s.SetParameters(T.SyncedNesterovParams(alpha, rho_alm, 0.0, 1e-300, 1, 20000, dt))
    s.SetRelativeResidualStop(0.5)
    s.Solve()
    st = s.GetStats()
    assert st["stop_rule_met"] == 1, st
    assert 1 < st["inner_iters_total"] < 20000
    assert st["rel_residual"] < 0.5
    xs = el.RetrievePositionToCPU()
    r_orc = _oracle_residual(x, y, z, conn, fixed, f, xs)
    assert abs(r_orc - st["rel_residual"]) <= 1e-9 * r_orc
    # with the rule off the same solve runs to its iteration cap
    s.SetRelativeResidualStop(0.0)
    s.SetParameters(T.SyncedNesterovParams(alpha, rho_alm, 0.0, 1e-300, 1, 50, dt))
    s.Solve()
    st2 = s.GetStats()
    assert st2["stop_rule_met"] == 0 and st2["inner_iters_total"] == 50
    el.Destroy()


def test_rule_is_rejected_for_the_linear_static_solver():
    x, y, z, conn, fixed, f = _cfg1()
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    s = T.LinearStaticSolver(el, 1e-10, 100)
    with pytest.raises(T.TLFEAError):
        _capi.call("tlfea_solver_set_stop_rule", s._h, C.c_double(1e-6))
    del s
    el.Destroy()
