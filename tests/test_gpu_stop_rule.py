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
    # first evaluation at the reference positions: f_int = 0, residual = ||f_free|| / ||f|| = 1
    assert st["rel_residual"] == pytest.approx(1.0, rel=1e-14)
    xs = el.RetrievePositionToCPU()
    assert all(np.array_equal(a, b) for a, b in zip(xs, (x, y, z)))
    el.Destroy()


def test_rule_ends_a_time_stepping_run_at_a_checked_residual():
    x, y, z, conn, fixed, f = _cfg1()
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    s = T.SyncedNesterovSolver(el, el.get_n_constraint())
    s.Setup()
    s.SetParameters(T.SyncedNesterovParams(*NESTEROV))
    s.SetRelativeResidualStop(0.9)
    met = False
    for _ in range(400):
        s.Solve()
        st = s.GetStats()
        if st["stop_rule_met"]:
            met = True
            break
        assert st["rel_residual"] >= 0.9
    assert met, "the static residual never dropped below 0.9"
    assert st["rel_residual"] < 0.9
    xs = el.RetrievePositionToCPU()
    r_orc = _oracle_residual(x, y, z, conn, fixed, f, xs)
    assert abs(r_orc - st["rel_residual"]) <= 1e-9 * r_orc
    # turning the rule off restores the reference's stopping
    s.SetRelativeResidualStop(0.0)
    s.Solve()
    assert s.GetStats()["stop_rule_met"] == 0
    el.Destroy()


def test_rule_is_rejected_for_the_linear_static_solver():
    x, y, z, conn, fixed, f = _cfg1()
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    s = T.LinearStaticSolver(el, 1e-10, 100)
    with pytest.raises(T.TLFEAError):
        _capi.call("tlfea_solver_set_stop_rule", s._h, C.c_double(1e-6))
    del s
    el.Destroy()
