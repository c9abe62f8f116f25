"""Batched time-stepping sequences (tlfea_dynbatch_*, BatchedDynamics): B sequences on
one mesh, each implicit step solved by the SyncedNesterov iteration, against the
oracle's SyncedNesterov restatement run sequence by sequence.

With zero tolerances both run the same number of iterations (max_outer x max_inner per
step), so each sequence's trajectory compares within a bar calibrated on the case:
max(1e-10, 3 s), s being how far the oracle's own displacements move when its reference
positions are perturbed by 1e-15 (relative).  The multipliers (rho = 1e14) amplify rounding
to s ~ 3e-9 on these meshes; the oracle and the reference's own CUDA build differ by
1.2e-9 on the same kind of run.  With the stop rule on, the residual each sequence reports is checked against one
recomputed from the oracle's mass matrix and internal force at its final state."""
import numpy as np
import pytest

import tlfea_b200 as T
from oracle import oracle as O
from tlfea_b200 import mesh as M

from .helpers import box, make_element, rel

pytestmark = pytest.mark.gpu

RHO = 1000.0
FIXED = (1.0e-8, 1e14, 0.0, 0.0, 2, 40, 1.0e-3)


def _mesh(cells=(10, 2, 2), order=10, load=(0.0, 0.0, -100.0)):
    x, y, z, conn = box(*cells, order)
    fixed, f, tip = M.cantilever_loads(x, y, z, load)
    return x, y, z, conn, fixed, f, tip


def _oracle_steps(x, y, z, conn, E, nu, fixed, loads, params, lamd=0.0, pert=0.0, seed=1):
    """The oracle's displacements (from the reference positions it was given) and velocity
    guess after each SyncedNesterov step, one external force per step."""
    xp = x if pert == 0.0 else x * (1.0 + pert * np.random.default_rng(seed).standard_normal(len(x)))
    m = O.OracleModel(xp, y, z, conn, E, nu, RHO, fixed, loads[0], 0.0, lamd)
    m.set_parameters()
    X0 = np.stack([xp, y, z])
    disp, vel = [], []
    for fk in loads:
        m.f_ext[:] = fk
        m.nesterov_solve(*params)
        disp.append(np.stack([m.x, m.y, m.z]) - X0)
        vel.append(m.v_guess[:3 * len(x)].copy())
    return disp, vel


def _oracle_with_bar(x, y, z, conn, E, nu, fixed, loads, params, lamd=0.0):
    """(displacements, velocities, displacement bar, velocity bar): each bar is
    max(1e-10, 3 s) over two perturbation seeds, s the largest relative change of a step's
    displacement (or velocity)."""
    d0, v0 = _oracle_steps(x, y, z, conn, E, nu, fixed, loads, params, lamd)
    sx = sv = 0.0
    for seed in (1, 2):
        d1, v1 = _oracle_steps(x, y, z, conn, E, nu, fixed, loads, params, lamd, 1e-15, seed)
        sx = max(sx, max(rel(a, b) for a, b in zip(d1, d0)))
        sv = max(sv, max(rel(a, b) for a, b in zip(v1, v0)))
    return d0, v0, max(1e-10, 3.0 * sx), max(1e-10, 3.0 * sv)


def _batch(x, y, z, conn, fixed, f, E, nu, params, rel_tol=0.0, lamd=0.0):
    el = make_element(x, y, z, conn, E_mod=float(E[0]), nu=float(nu[0]), rho=RHO, fixed=fixed, f_ext=f, lamd=lamd)
    b = T.BatchedDynamics(el, len(E))
    b.SetMaterial(E, nu)
    b.SetParameters(T.SyncedNesterovParams(*params), rel_tol)
    return el, b


@pytest.mark.parametrize("lamd", [0.0, 0.1])
def test_fixed_iterations_match_the_oracle_per_sequence(lamd):
    x, y, z, conn, fixed, f, _ = _mesh()
    E = np.array([1e7, 3e6, 2.5e7])
    nu = np.array([0.3, 0.25, 0.4])
    el, b = _batch(x, y, z, conn, fixed, f, E, nu, FIXED, lamd=lamd)
    refs = [_oracle_with_bar(x, y, z, conn, E[s], nu[s], fixed, [f, f], FIXED, lamd) for s in range(len(E))]
    X0 = np.stack([x, y, z])
    for step in range(2):
        it, res, conv = b.Step(T.BatchedDynamics.WARM_PREVIOUS)
        assert list(it) == [80, 80, 80] and not conv.any()
        for s, (disp, vel, bx, bv) in enumerate(refs):
            e = rel(np.stack(b.RetrievePositions(s)) - X0, disp[step])
            assert e < bx, (step, s, e, bx)
            e = rel(b.RetrieveVelocity(s), vel[step])
            assert e < bv, (step, s, e, bv)
    b.Destroy()
    el.Destroy()


def test_time_varying_load_matches_the_oracle():
    """f_ext(t_k) = f_base + amp sin(omega t_k + phase) f_var, evaluated on the device at
    t_k = k dt, against the same load set on the oracle step by step (TET4 mesh)."""
    x, y, z, conn, fixed, f0, tip = _mesh(order=4)
    f_var = np.zeros(3 * len(x))
    f_var[3 * tip + 2] = -50.0 / len(tip)
    E, nu = np.array([1e7, 5e6]), np.array([0.3, 0.35])
    el, b = _batch(x, y, z, conn, fixed, f0, E, nu, FIXED)
    amp, omega, phase = 1.0, 2 * np.pi * 5.0, 0.3
    b.SetLoad(f_var, amp, omega, phase)
    loads = [f0 + (amp * np.sin(omega * (k * FIXED[6]) + phase)) * f_var for k in range(1, 4)]
    refs = [_oracle_with_bar(x, y, z, conn, E[s], nu[s], fixed, loads, FIXED) for s in range(2)]
    X0 = np.stack([x, y, z])
    for k in range(3):
        b.Step(0)
        for s, (disp, _, bar, _) in enumerate(refs):
            e = rel(np.stack(b.RetrievePositions(s)) - X0, disp[k])
            assert e < bar, (k, s, e, bar)
    b.Destroy()
    el.Destroy()


def _hessian_lmax(x, y, z, conn, fixed, E, nu, dt, rho_alm, iters=200):
    """Largest eigenvalue of the step's Hessian M/dt + dt K (+ dt^2 rho on fixed DOFs)."""
    import scipy.sparse as sp

    m = O.OracleModel(x, y, z, conn, E, nu, RHO, fixed, np.zeros(3 * len(x)))
    off, cols, vals = O.stiffness(x, y, z, conn, m.grad, m.detJ, m.lam, m.mu)
    K = sp.csr_matrix((vals, cols, off))
    Mf = sp.kron(sp.csr_matrix((m.m_val, m.m_col, m.m_off)), sp.identity(3)).tocsr()
    d = np.zeros(3 * len(x))
    for n in fixed:
        d[3 * n:3 * n + 3] = dt * dt * rho_alm
    H = Mf / dt + dt * K + sp.diags(d)
    v = np.random.default_rng(0).standard_normal(H.shape[0])
    for _ in range(iters):
        v = H @ v
        v /= np.linalg.norm(v)
    return float(v @ (H @ v))


def _step_residual(x, y, z, conn, fixed, f, E, nu, xs, v, v_prev, dt):
    """||g_free|| / ||f_ext|| of a step from the oracle's pieces: g = M (v - v_prev) / dt +
    f_int(x) - f_ext (the constraint term is zero on free DOFs)."""
    import scipy.sparse as sp

    m = O.OracleModel(x, y, z, conn, E, nu, RHO, fixed, f)
    fi = O.force(*xs, conn, m.grad, m.detJ, m.lam, m.mu)
    Mn = sp.csr_matrix((m.m_val, m.m_col, m.m_off))
    g = (Mn @ (v - v_prev).reshape(-1, 3)).ravel() / dt + fi - f
    free = np.ones(len(x), bool)
    free[fixed] = False
    return np.linalg.norm(g.reshape(-1, 3)[free]) / np.linalg.norm(f)


def test_stop_rule_ends_each_sequence_at_a_checked_residual():
    x, y, z, conn, fixed, f, _ = _mesh()
    E, nu = np.array([1e7, 2e6]), np.array([0.3, 0.3])
    dt, rho_alm = 1e-3, 1e8
    alphas = [0.9 / _hessian_lmax(x, y, z, conn, fixed, E[s], nu[s], dt, rho_alm) for s in range(2)]
    params = (alphas[0], rho_alm, 0.0, 1e-300, 1, 20000, dt)
    el, b = _batch(x, y, z, conn, fixed, f, E, nu, params, rel_tol=1e-6)
    b.SetStepSizes(alphas)
    vprev = [np.zeros(3 * len(x)) for _ in E]
    for step in range(2):
        it, res, conv = b.Step(T.BatchedDynamics.WARM_LINEAR if step else 0)
        assert conv.all() and (res < 1e-6).all() and (it < 20000).all(), (it, res, conv)
        for s in range(len(E)):
            xs = b.RetrievePositions(s)
            vs = b.RetrieveVelocity(s)
            r = _step_residual(x, y, z, conn, fixed, f, E[s], nu[s], xs, vs, vprev[s], dt)
            assert abs(r - res[s]) <= 1e-6 * r + 1e-13, (r, res[s])
            vprev[s] = vs
    # a given warm start: the converged first-step velocities end a fresh first step at its
    # first residual evaluation
    import torch

    b.Reset()
    b.Step(0)
    v1 = np.concatenate([b.RetrieveVelocity(s) for s in range(len(E))])
    guess = torch.tensor(v1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    b.Reset()
    it, res, conv = b.Step(T.BatchedDynamics.WARM_GIVEN, guess.data_ptr())
    assert conv.all() and list(it) == [1] * len(E), (it, res)
    b.Destroy()
    el.Destroy()


def test_learned_step_predictor_reduces_iterations():
    """What the trained network gains (configuration-5 style, small mesh): a StepPredictor
    trained on the solver's own steps of other sequences warm-starts each step; to the same
    residual tolerance it needs fewer Nesterov iterations than the reference's start (the
    previous velocity), and its residuals are checked by the same stop rule."""
    import torch
    from tlfea_b200 import warmstart as W

    x, y, z, conn, fixed, _, tip = _mesh(cells=(10, 2, 2))
    N = len(x)
    el = make_element(x, y, z, conn, E_mod=1e7, nu=0.3, rho=RHO, fixed=fixed, f_ext=np.zeros(3 * N))
    el.AddGravity(0.0, 0.0, -9.81)
    f_var = np.zeros(3 * N)
    f_var[3 * tip + 2] = -50.0 / len(tip)
    omega, dt, rho_alm = 2 * np.pi * 5.0, 1e-3, 1e8
    r = np.random.default_rng(3)
    E = np.exp(r.uniform(np.log(5e6), np.log(2e7), 8))
    nu = r.uniform(0.25, 0.35, 8)
    alphas = np.array([0.9 / (_hessian_lmax(x, y, z, conn, fixed, E[s], nu[s], dt, rho_alm, 100)) for s in range(8)])
    params = T.SyncedNesterovParams(float(alphas.min()), rho_alm, 0.0, 1e-6, 3, 20000, dt)
    X0 = torch.as_tensor(np.stack([x, y, z], 1).reshape(-1), device="cuda")

    def make(seqs):
        b = T.BatchedDynamics(el, len(seqs))
        b.SetMaterial(E[seqs], nu[seqs])
        b.SetParameters(params, 1e-6)
        b.SetStepSizes(alphas[seqs])
        b.SetLoad(f_var, 1.0, omega, 0.0)
        return b

    def state(b, B):
        p = b.DevicePtrs()
        v = W.device_view(p["v"], (B, 3 * N))
        vh = W.device_view(p["v_hist"], (B, 3 * N))
        u = torch.stack([W.device_view(p[k], (B, N)) for k in ("x", "y", "z")], 2).reshape(B, 3 * N) - X0
        return v, vh, u

    def lf(n):
        return np.array([[np.sin(omega * (n - 1 + j) * dt) for j in range(3)]])

    tr, ev, steps = np.arange(4, 8), np.arange(4), 12
    bt = make(tr)
    V = torch.empty(4, steps, 3 * N, dtype=torch.float64, device="cuda")
    U = torch.empty_like(V)
    for k in range(steps):
        bt.Step(T.BatchedDynamics.WARM_LINEAR)
        v, _, u = state(bt, 4)
        V[:, k], U[:, k] = v, u
    bt.Destroy()
    sp = W.StepPredictor(k_in=8, k_out=16, hidden=(128, 128), max_batch=128, seed=0, E_range=(5e6, 2e7),
                         nu_range=(0.25, 0.35))
    mats = sp.material_features(E, nu)
    sp.fit(V, U, np.concatenate([lf(n) for n in range(1, steps + 1)]), mats[tr], epochs=300, batch=32)
    b = make(ev)
    totals = {}
    for name in ("previous", "learned"):
        b.Reset()
        tot = 0
        for n in range(1, 7):
            if name == "previous":
                it, res, conv = b.Step(T.BatchedDynamics.WARM_PREVIOUS)
            elif n == 1:
                it, res, conv = b.Step(T.BatchedDynamics.WARM_LINEAR)
            else:
                v, vh, u = state(b, 4)
                g = sp.predict(v, vh, u, np.repeat(lf(n - 1), 4, 0), mats[ev])
                it, res, conv = b.Step(T.BatchedDynamics.WARM_GIVEN, int(g.data_ptr()))
            assert conv.all() and (res < 1e-6).all()
            tot += int(it.sum())
        totals[name] = tot
    assert totals["learned"] < totals["previous"], totals
    b.Destroy()
    sp.destroy()
    el.Destroy()


def test_momentum_restart_converges_in_fewer_iterations_to_a_checked_residual():
    """With the gradient restart test (g . (v_next - v_k) > 0 starts the beta sequence
    afresh) each step reaches the stop rule in fewer inner iterations than the
    reference's schedule, and the residual it reports is the one recomputed from the
    oracle's pieces at its final state."""
    x, y, z, conn, fixed, f, _ = _mesh()
    E, nu = np.array([2e7, 3e6]), np.array([0.3, 0.3])
    dt, rho_alm = 1e-3, 1e8
    alphas = [0.9 / _hessian_lmax(x, y, z, conn, fixed, E[s], nu[s], dt, rho_alm) for s in range(2)]
    params = (alphas[0], rho_alm, 0.0, 1e-300, 1, 40000, dt)
    its = {}
    for restart in (False, True):
        el, b = _batch(x, y, z, conn, fixed, f, E, nu, params, rel_tol=1e-6)
        b.SetStepSizes(alphas)
        b.SetRestart(restart)
        vprev = [np.zeros(3 * len(x)) for _ in E]
        its[restart] = []
        for step in range(2):
            it, res, conv = b.Step(T.BatchedDynamics.WARM_LINEAR if step else 0)
            assert conv.all() and (res < 1e-6).all(), (restart, it, res)
            its[restart].append(it.copy())
            for s in range(len(E)):
                xs = b.RetrievePositions(s)
                vs = b.RetrieveVelocity(s)
                r = _step_residual(x, y, z, conn, fixed, f, E[s], nu[s], xs, vs, vprev[s], dt)
                assert abs(r - res[s]) <= 1e-6 * r + 1e-13, (r, res[s])
                vprev[s] = vs
        b.Destroy()
        el.Destroy()
    # a CPU run of the same iteration: about 6,800 inner iterations per step without the
    # restart, about 600 with it (E = 2e7)
    assert np.sum(its[True]) < 0.3 * np.sum(its[False]), its
