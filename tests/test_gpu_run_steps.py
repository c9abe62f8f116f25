"""RunSteps: n calls of Solve() in one graph launch, with the load computed on
the device as f_base + (amp * sin(omega * t_k + phase)) * f_var.  It must give,
bit for bit, what the reference's host loop of SetExternalForce + Solve gives
(examples/beam_simulation.cc:275-283), and the oracle's trajectory for the same
loop at a fixed iteration count."""
import math

import numpy as np
import pytest

import tlfea_b200 as T
from oracle import oracle as O
from tlfea_b200 import mesh as M

from .helpers import E_MOD, NU, RHO, box, make_element, rel

pytestmark = pytest.mark.gpu

NESTEROV = (1.0e-8, 1e14, 1.0e-6, 1.0e-6, 5, 300, 1.0e-3)  # test_feat10_nesterov.cc:189
ADAMW = (2e-4, 0.9, 0.999, 1e-8, 1e-4, 0.995, 1e-1, 1e-6, 1e14, 5, 500, 1e-3, 10, 0.0)  # test_feat10_adamw.cc:189


def _case():
    x, y, z, conn = box(10, 2, 2, 10)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -100.0))
    fvar = np.zeros_like(f)
    tip = np.nonzero(np.abs(x - x.max()) < 1e-9)[0]
    fvar.reshape(-1, 3)[tip, 1] = 40.0 / len(tip)  # a sideways tip load that oscillates
    return x, y, z, conn, fixed, f, fvar


def _solver(kind, prec="fp64", params=None):
    x, y, z, conn, fixed, f, fvar = _case()
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    if prec != "fp64":
        el.SetForcePrecision(prec)
    cls = T.SyncedNesterovSolver if kind == "nesterov" else T.SyncedAdamWSolver
    s = cls(el, el.get_n_constraint())
    s.Setup()
    if kind == "nesterov":
        s.SetParameters(T.SyncedNesterovParams(*(params or NESTEROV)))
    else:
        s.SetParameters(T.SyncedAdamWParams(*(params or ADAMW)))
    return el, s, f, fvar


def _scale(k, t0, dt, amp, omega, phase):
    return amp * math.sin(omega * (t0 + (k + 1) * dt) + phase)


@pytest.mark.parametrize("kind,prec", [("nesterov", "fp64"), ("nesterov", "fp32"), ("adamw", "fp64")])
def test_run_steps_constant_load_equals_the_solve_loop(kind, prec):
    n = 4
    el_a, s_a, _, _ = _solver(kind, prec)
    its_a = []
    for _ in range(n):
        s_a.Solve()
        its_a.append(s_a.GetStats()["inner_iters_total"])
    el_b, s_b, _, _ = _solver(kind, prec)
    its_b = s_b.RunSteps(n)
    assert list(its_b) == its_a
    for a, b in zip(el_a.RetrievePositionToCPU(), el_b.RetrievePositionToCPU()):
        assert np.array_equal(a, b)
    for a, b in zip(s_a.GetVelocity(), s_b.GetVelocity()):
        assert np.array_equal(a, b)
    sa, sb = s_a.GetStats(), s_b.GetStats()
    for key in ("outer_iters", "inner_iters_total", "last_inner_iters", "status", "last_norm_g"):
        assert sa[key] == sb[key], key
    el_a.Destroy()
    el_b.Destroy()


@pytest.mark.parametrize("kind", ["nesterov", "adamw"])
def test_run_steps_time_varying_load_equals_the_host_loop(kind):
    n, t0, amp, omega, phase = 5, 0.25, 1.5, 300.0, 0.4
    el_a, s_a, f0, fvar = _solver(kind)
    dt = NESTEROV[6] if kind == "nesterov" else ADAMW[11]
    its_a = []
    for k in range(n):
        a = _scale(k, t0, dt, amp, omega, phase)
        el_a.SetExternalForce(f0 + a * fvar)
        s_a.Solve()
        its_a.append(s_a.GetStats()["inner_iters_total"])
    el_b, s_b, _, _ = _solver(kind)
    its_b = s_b.RunSteps(n, fvar, amp=amp, omega=omega, phase=phase, t0=t0)
    assert list(its_b) == its_a
    xa, xb = el_a.RetrievePositionToCPU(), el_b.RetrievePositionToCPU()
    for a, b in zip(xa, xb):
        assert np.array_equal(a, b)
    # the load moved the beam sideways: the y displacement is not the constant-load one
    x0, y0, z0, *_ = _case()
    assert np.abs(xb[1] - y0).max() > 0
    el_a.Destroy()
    el_b.Destroy()


def test_run_steps_tracks_the_oracle_trajectory():
    """Fixed iteration counts (zero inner tolerance): the GPU trajectory under the
    device-computed load against the oracle's host loop."""
    params = (1.0e-8, 1e14, 0.0, 0.0, 2, 40, 1.0e-3)
    n, amp, omega, phase = 3, 2.0, 500.0, 0.0
    el, s, f0, fvar = _solver("nesterov", params=params)
    its = s.RunSteps(n, fvar, amp=amp, omega=omega, phase=phase)
    assert list(its) == [80] * n
    x, y, z, conn, fixed, f, _ = _case()
    m = O.OracleModel(x, y, z, conn, E_MOD, NU, RHO, fixed, f)
    m.set_parameters()
    for k in range(n):
        m.f_ext = f0 + _scale(k, 0.0, params[6], amp, omega, phase) * fvar
        m.nesterov_solve(*params)
    xg = el.RetrievePositionToCPU()
    du = np.stack([xg[0] - x, xg[1] - y, xg[2] - z])
    du_ref = np.stack([m.x - x, m.y - y, m.z - z])
    # positions agree to ~1e-16 (the fixed-count Nesterov tests); the tip
    # displacement here is ~1e-7, so the relative tolerance on it is 1e-8
    assert rel(du, du_ref) < 1e-8
    el.Destroy()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_run_steps_tet4_with_damping_and_stop_rule(prec):
    """TET4, Kelvin-Voigt damping, FP32 or FP64 forces and the relative-residual
    stop rule: the graph of steps equals the host loop bitwise."""
    x, y, z, conn = box(10, 2, 2, 4)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -100.0))
    fvar = np.zeros_like(f)
    fvar.reshape(-1, 3)[np.nonzero(np.abs(x - x.max()) < 1e-9)[0], 1] = 10.0

    def make():
        el = make_element(x, y, z, conn, fixed=fixed, f_ext=f, eta=50.0, lamd=10.0)
        if prec != "fp64":
            el.SetForcePrecision(prec)
        s = T.SyncedNesterovSolver(el, el.get_n_constraint())
        s.Setup()
        s.SetParameters(T.SyncedNesterovParams(*NESTEROV))
        s.SetRelativeResidualStop(1e-3)
        return el, s

    n, amp, omega = 4, 2.0, 100.0
    el_a, s_a = make()
    its_a, rel_a = [], []
    for k in range(n):
        el_a.SetExternalForce(f + _scale(k, 0.0, NESTEROV[6], amp, omega, 0.0) * fvar)
        s_a.Solve()
        st = s_a.GetStats()
        its_a.append(st["inner_iters_total"])
        rel_a.append(st["rel_residual"])
    el_b, s_b = make()
    its_b = s_b.RunSteps(n, fvar, amp=amp, omega=omega)
    assert list(its_b) == its_a
    assert s_b.GetStats()["rel_residual"] == rel_a[-1]
    for a, b in zip(el_a.RetrievePositionToCPU(), el_b.RetrievePositionToCPU()):
        assert np.array_equal(a, b)
    el_a.Destroy()
    el_b.Destroy()


def test_run_steps_refuses_bad_input():
    el, s, _, _ = _solver("nesterov")
    with pytest.raises(Exception):
        s.RunSteps(0)
    el.Destroy()
    x, y, z, conn, fixed, f, _ = _case()
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    ls = T.LinearStaticSolver(el, 1e-8, 100)
    from tlfea_b200 import _capi

    rc = _capi.lib().tlfea_solver_run_steps(ls._h, 2, 0.0, None, 1.0, 0.0, 0.0, None)
    assert rc != 0
    el.Destroy()
