"""The oracle against fixtures produced by the reference's own CUDA build.

``tests/golden/ref_*.npz`` were written on a B200 by ``tests/golden/make_ref_fixtures.py``
from the reference's unchanged element and solver sources (compiled by
``oracle/build_ref.py``).  These CPU tests feed the same inputs (``ref_cases.py``) to the
oracle and compare, which pins the oracle to the reference itself; the GPU tests in
``test_gpu_ref_fixtures.py`` compare the CUDA path with the same fixtures.

Tolerances: the reference sums element contributions with atomicAdd in an unspecified
order and its CG dots come from cuBLAS, so FP64 arrays agree to rounding: rel 1e-12 for
forces, mass and stiffness, 1e-11 for P (at small strain P = lambda tr(E) F + mu (F F^T F - F)
cancels, amplifying rounding by |F| / |F - I|); integer patterns are bit-exact.  Iterative
results are compared against a bar calibrated on the case itself: max(1e-10, 3 s), where s is
how far the oracle's own result moves when its input is perturbed by 1e-15 (relative).  Where
the iteration amplifies rounding -- the cube's stiffness with unit rows for its clamped DOFs
beside entries of 1e8 (condition number 3.6e9, so its 25-iteration CG iterate is chaotic),
multipliers with rho = 1e14, AdamW with eps = 1e-8 -- s is far above 1e-10 and no two
summation orders can agree closer; elsewhere the bar is the 1e-10 of the parity contract.
Converged CG runs agree in their solution and in their iteration count within 5% (CG's count
to a tight tolerance moves with rounding over thousands of iterations).
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
        assert rel(P, fx["P"]) < 1e-11


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
    assert rel(u25, fx["u_cg25"]) < cg25_bar(off, cols, kv, fb)
    u, it, res, _ = O.cg(off, cols, kv, fb, 1e-10, 200000)
    it_ref = int(fx["cg_iters"][0])
    assert abs(it - it_ref) <= cg_iteration_bar(it_ref), (it, it_ref)
    assert rel(u, fx["u_cg"]) < 1e-7


def cg25_bar(off, cols, kv, fb, iters=25):
    """max(1e-10, 3 s): s = the largest change of the oracle's `iters`-iteration CG iterate
    when the stiffness values are perturbed by 1e-15 (relative; three seeds)."""
    u, *_ = O.cg(off, cols, kv, fb, 0.0, iters)
    s = 0.0
    for seed in (3, 4, 5):
        kp = kv * (1.0 + 1e-15 * np.random.default_rng(seed).standard_normal(kv.size))
        up, *_ = O.cg(off, cols, kp, fb, 0.0, iters)
        s = max(s, rel(up, u))
    return max(1e-10, 3.0 * s)


def cg_iteration_bar(it_ref):
    return max(2, 0.05 * it_ref)


def _oracle_run(c, kind, params, steps, fixed, f, eta=0.0, lamd=0.0, pert=0.0, seed=1):
    """The oracle's displacements after each step (relative to the reference positions it
    was given, which `pert` perturbs) and its final velocity guess."""
    x = c["x"] if pert == 0.0 else c["x"] * (1.0 + pert * np.random.default_rng(seed).standard_normal(len(c["x"])))
    m = O.OracleModel(x, c["y"], c["z"], c["conn"], c["E"], c["nu"], c["rho"], fixed, f, eta, lamd)
    m.set_parameters()
    X0 = np.stack([x, c["y"], c["z"]])
    disp = []
    for _ in range(steps):
        if kind == "nesterov":
            m.nesterov_solve(*params)
        elif kind == "adamw":
            m.adamw_solve(*params)
        else:
            m.adamw_nocoop_solve(*params)
        disp.append(np.stack([m.x, m.y, m.z]) - X0)
    return np.stack(disp), m.v_guess[:3 * len(c["x"])]


def first_order_runs(name):
    """(tag, kind, params, steps, load) of the fixture's solver trajectories: fixed
    iteration counts (zero tolerances), and on the cube the reference examples' own
    parameters."""
    runs = [("nes_fixed", "nesterov", RC.NESTEROV_FIXED, 3, None)]
    if name == "cube_t10":
        runs += [("nes_ref", "nesterov", RC.NESTEROV_REF, 5, None),
                 ("adamw_ref", "adamw", RC.ADAMW_REF, 3, None),
                 ("nocoop_ref", "nocoop", RC.ADAMW_REF, 3, None)]
    else:
        runs += [("adamw_fixed", "adamw", RC.ADAMW_FIXED, 2, "generic"),
                 ("nocoop_fixed", "nocoop", RC.ADAMW_FIXED, 2, "generic")]
        if name == "cfg1_t10":
            runs.append(("nes_damped", "nesterov", RC.NESTEROV_FIXED, 2, "damped"))
    return runs


def run_inputs(c, load_kind):
    fixed, f, lamd = c["fixed"], c["f"], 0.0
    if load_kind == "generic":
        fixed, f = RC.generic_load(c)
    elif load_kind == "damped":
        lamd = 0.1  # examples/beam_simulation.cc:203
    return fixed, f, lamd


def first_order_bars(c, kind, params, steps, fixed, f, lamd):
    """(position bar, velocity bar): max(1e-10, 3 s) with s the largest change of the
    oracle's trajectory (displacements over the steps, each from the reference positions
    that run started from) when the reference positions are perturbed by 1e-15 (relative;
    two seeds)."""
    p0, v0 = _oracle_run(c, kind, params, steps, fixed, f, 0.0, lamd)
    sx = sv = 0.0
    for seed in (1, 2):
        p1, v1 = _oracle_run(c, kind, params, steps, fixed, f, 0.0, lamd, pert=1e-15, seed=seed)
        sx = max(sx, max(rel(p1[k], p0[k]) for k in range(steps)))
        sv = max(sv, rel(v1, v0))
    return max(1e-10, 3.0 * sx), max(1e-10, 3.0 * sv)


@pytest.mark.parametrize("name", RC.SMALL)
def test_oracle_first_order_solvers_match_reference(name):
    fx = load(name)
    c = RC.case(name)
    for tag, kind, params, steps, load_kind in first_order_runs(name):
        fixed, f, lamd = run_inputs(c, load_kind)
        disp, v = _oracle_run(c, kind, params, steps, fixed, f, 0.0, lamd)
        bx, bv = first_order_bars(c, kind, params, steps, fixed, f, lamd)
        X0 = np.stack([c["x"], c["y"], c["z"]])
        ref = fx[f"{tag}_pos"]
        for k in range(steps):
            assert rel(disp[k], ref[k] - X0) < bx, (tag, k, rel(disp[k], ref[k] - X0), bx)
        assert rel(v, fx[f"{tag}_v"]) < bv, (tag, rel(v, fx[f"{tag}_v"]), bv)
