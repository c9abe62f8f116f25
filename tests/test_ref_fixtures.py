"""The oracle against fixtures produced by the reference's own CUDA build.

``tests/golden/ref_*.npz`` were written on a B200 by ``tests/golden/make_ref_fixtures.py``
from the reference's unchanged element and solver sources (compiled by
``oracle/build_ref.py``).  These CPU tests feed the same inputs (``ref_cases.py``) to the
oracle and compare, which pins the oracle to the reference itself; the GPU tests in
``test_gpu_ref_fixtures.py`` compare the CUDA path with the same fixtures.

Tolerances: the reference sums element contributions with atomicAdd in an unspecified
order and its CG dots come from cuBLAS, so FP64 arrays agree to rounding (rel 1e-12 for
element arrays, 1e-10 for the 25-iteration CG iterate); integer patterns are bit-exact.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
import ref_cases as RC  # noqa: E402

from .helpers import rel  # noqa: E402

ORACLE_CASES = RC.SMALL + RC.MID


def load(name):
    p = RC.fixture_path(name)
    if not p.exists():
        pytest.skip(f"{p.name} not generated")
    return dict(np.load(p))


def lame(c):
    E, nu = c["E"], c["nu"]
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


def oracle_element(name):
    c = RC.case(name)
    g, dj = O.dndu_pre(c["x"], c["y"], c["z"], c["conn"])
    return c, g, dj


@pytest.mark.parametrize("name", ORACLE_CASES + RC.LARGE)
def test_oracle_force_matches_reference(name):
    fx = load(name)
    c, g, dj = oracle_element(name)
    lam, mu = lame(c)
    xp, yp, zp = RC.perturbed(c)
    f = O.force(xp, yp, zp, c["conn"], g, dj, lam, mu)
    if name in RC.LARGE:
        s = RC.summary(f)
        assert abs(s["norm"] - fx["f_int_norm"][0]) <= 1e-12 * s["norm"]
        assert rel(s["proj"], fx["f_int_proj"]) < 1e-11
        assert rel(s["sample"], fx["f_int_sample"]) < 1e-12
    else:
        assert rel(f, fx["f_int"]) < 1e-12
    if "P" in fx:
        _, P = O.calc_p(xp, yp, zp, c["conn"], g, lam, mu)
        assert rel(P, fx["P"]) < 1e-13


@pytest.mark.parametrize("name", RC.SMALL)
def test_oracle_geometry_and_mass_match_reference(name):
    fx = load(name)
    c, g, dj = oracle_element(name)
    assert rel(g, fx["grad"]) < 1e-13
    assert rel(dj, fx["detj"]) < 1e-14
    off, cols, vals = O.mass(c["conn"], dj, len(c["x"]), c["rho"])
    assert np.array_equal(off, fx["mass_off"]) and np.array_equal(cols, fx["mass_col"])
    assert rel(vals, fx["mass_val"]) < 1e-13


@pytest.mark.parametrize("name", RC.MID)
def test_oracle_mass_row_sums_match_reference(name):
    fx = load(name)
    c, g, dj = oracle_element(name)
    off, cols, vals = O.mass(c["conn"], dj, len(c["x"]), c["rho"])
    assert len(vals) == int(fx["mass_nnz"][0])
    assert rel(np.add.reduceat(vals, off[:-1]), fx["mass_rowsum"]) < 1e-13
    assert abs(dj.sum() - fx["detj_sum"][0]) <= 1e-12 * abs(dj.sum())


@pytest.mark.parametrize("name", RC.SMALL)
def test_reference_constraint_arrays(name):
    """c = x(fixed) - x_jac(fixed) (FEAT10DataFunc.cuh:470-481) and the unit J / J^T CSR
    (FEAT10Data.cu:420-562): the reference's arrays against their definition."""
    fx = load(name)
    c = RC.case(name)
    xp, yp, zp = RC.perturbed(c)
    fixed = c["fixed"]
    cref = np.stack([xp[fixed] - c["x"][fixed], yp[fixed] - c["y"][fixed], zp[fixed] - c["z"][fixed]], 1).ravel()
    assert rel(fx["constraint"], cref) < 1e-15
    nc = 3 * len(fixed)
    dofs = (3 * fixed[:, None] + np.arange(3)[None, :]).ravel()
    assert np.array_equal(fx["j_off"], np.arange(nc + 1))
    assert np.array_equal(fx["j_col"], dofs) and np.all(fx["j_val"] == 1.0)
    rows = np.zeros(3 * len(c["x"]), np.int32)
    rows[dofs] = 1
    assert np.array_equal(fx["jt_off"], np.concatenate([[0], np.cumsum(rows)]))
    order = np.argsort(dofs, kind="stable")
    assert np.array_equal(fx["jt_col"], np.arange(nc)[order]) and np.all(fx["jt_val"] == 1.0)


@pytest.mark.parametrize("name", RC.SMALL + RC.MID)
def test_oracle_linear_static_matches_reference(name):
    fx = load(name)
    c, g, dj = oracle_element(name)
    lam, mu = lame(c)
    off, cols, vals = O.stiffness(c["x"], c["y"], c["z"], c["conn"], g, dj, lam, mu)
    kv, fb = O.apply_bcs(off, cols, vals, c["f"], c["fixed"])
    if "K_val" in fx:
        assert np.array_equal(off, fx["K_off"]) and np.array_equal(cols, fx["K_col"])
        assert rel(kv, fx["K_val"]) < 1e-12
    u25, it25, _, _ = O.cg(off, cols, kv, fb, 1e-10, 25)
    assert it25 == int(fx["cg25_iters"][0]) == 25
    assert rel(u25, fx["u_cg25"]) < 1e-10
    u, it, res, _ = O.cg(off, cols, kv, fb, 1e-10, 200000)
    it_ref = int(fx["cg_iters"][0])
    assert abs(it - it_ref) <= max(2, 0.01 * it_ref), (it, it_ref)
    assert rel(u, fx["u_cg"]) < 1e-7


def _oracle_run(c, kind, params, steps, fixed, f, eta=0.0, lamd=0.0):
    m = O.OracleModel(c["x"], c["y"], c["z"], c["conn"], c["E"], c["nu"], c["rho"], fixed, f, eta, lamd)
    m.set_parameters()
    pos = []
    for _ in range(steps):
        if kind == "nesterov":
            m.nesterov_solve(*params)
        elif kind == "adamw":
            m.adamw_solve(*params)
        else:
            m.adamw_nocoop_solve(*params)
        pos.append(np.stack([m.x, m.y, m.z]))
    return np.stack(pos), m.v_guess[:3 * len(c["x"])]


def first_order_runs(name):
    """(tag, kind, params, steps, load, position tolerance, velocity tolerance) of the
    fixture's solver trajectories.  Fixed-count runs compare tightly; the reference
    examples' parameters stop on |d||g||| < 1e-6 and |d||v||| < 1e-6 tests whose outcome
    can flip between two summation orders, so those compare the trajectory loosely.
    Multipliers move by rho*dt*c with rho = 1e14, amplifying one ulp of a position to
    ~1e-5 in lambda, so velocities compare looser than positions."""
    runs = [("nes_fixed", "nesterov", RC.NESTEROV_FIXED, 3, None, 1e-11, 1e-8)]
    if name == "cube_t10":
        runs += [("nes_ref", "nesterov", RC.NESTEROV_REF, 5, None, 1e-8, None),
                 ("adamw_ref", "adamw", RC.ADAMW_REF, 3, None, 1e-7, None),
                 ("nocoop_ref", "nocoop", RC.ADAMW_REF, 3, None, 1e-7, None)]
    else:
        runs += [("adamw_fixed", "adamw", RC.ADAMW_FIXED, 2, "generic", 1e-9, 1e-7),
                 ("nocoop_fixed", "nocoop", RC.ADAMW_FIXED, 2, "generic", 1e-9, 1e-7)]
        if name == "cfg1_t10":
            runs.append(("nes_damped", "nesterov", RC.NESTEROV_FIXED, 2, "damped", 1e-11, 1e-8))
    return runs


@pytest.mark.parametrize("name", RC.SMALL)
def test_oracle_first_order_solvers_match_reference(name):
    fx = load(name)
    c = RC.case(name)
    for tag, kind, params, steps, load_kind, tol_x, tol_v in first_order_runs(name):
        fixed, f, eta, lamd = c["fixed"], c["f"], 0.0, 0.0
        if load_kind == "generic":
            fixed, f = RC.generic_load(c)
        elif load_kind == "damped":
            lamd = 0.1
        pos, v = _oracle_run(c, kind, params, steps, fixed, f, eta, lamd)
        X0 = np.stack([c["x"], c["y"], c["z"]])
        ref = fx[f"{tag}_pos"]
        for k in range(steps):
            assert rel(pos[k] - X0, ref[k] - X0) < tol_x, (tag, k, rel(pos[k] - X0, ref[k] - X0))
        if tol_v is not None:
            assert rel(v, fx[f"{tag}_v"]) < tol_v, (tag, rel(v, fx[f"{tag}_v"]))
