"""GPU parity of the batched linear-static solve: the matrix-free K_bc x of
every instance against the oracle's assembled stiffness with BCs applied, the
CG solution against the oracle CG and a direct solve, warm starts, edge cases,
FP32 element work, the autotuner and graph replays."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import tlfea_b200 as T
from oracle import oracle as O
from tlfea_b200 import mesh as M

from .helpers import lame, rel

pytestmark = pytest.mark.gpu

SMALL = dict(nx_range=(3, 7), ny_range=(2, 3))


def _instances(n, order=10, seed0=100, **kw):
    return [M.random_beam(seed0 + i, order=order, **{**SMALL, **kw}) for i in range(n)]


def _batch(insts, order=10):
    b = T.BatchedLinearStaticSolver([(d["x"], d["y"], d["z"], d["conn"]) for d in insts],
                                    T.TYPE_T10 if order == 10 else T.TYPE_T4)
    b.SetMaterial([d["E"] for d in insts], [d["nu"] for d in insts])
    b.SetNodalFixed([d["fixed"] for d in insts])
    b.SetExternalForce([d["f"] for d in insts])
    return b


def _oracle_kbc(d):
    lam, mu = lame(d["E"], d["nu"])
    g, dj = O.dndu_pre(d["x"], d["y"], d["z"], d["conn"])
    off, cols, vals = O.stiffness(d["x"], d["y"], d["z"], d["conn"], g, dj, lam, mu)
    kv, fb = O.apply_bcs(off, cols, vals, d["f"], d["fixed"])
    return off, cols, kv, fb


@pytest.mark.parametrize("order", [10, 4])
def test_batch_apply_matches_oracle(order):
    import torch

    insts = _instances(4, order)
    b = _batch(insts, order)
    r = np.random.default_rng(0)
    xs = [r.standard_normal(3 * len(d["x"])) for d in insts]
    xd = torch.tensor(np.concatenate(xs), dtype=torch.float64, device="cuda")
    yd = torch.empty_like(xd)
    b.Apply(xd.data_ptr(), yd.data_ptr())
    y = yd.cpu().numpy()
    o = 0
    for d, xv in zip(insts, xs):
        off, cols, kv, _ = _oracle_kbc(d)
        y_ref = O.spmv(off, cols, kv, xv)
        assert rel(y[o:o + xv.size], y_ref) < 1e-12
        o += xv.size
    b.Destroy()


def test_batch_solve_matches_oracle_and_direct():
    insts = _instances(5)
    b = _batch(insts)
    b.Solve(1e-10, 20000)
    it, res, st = b.GetResults()
    us = b.RetrieveDisplacement()
    assert np.all(st == 0) and np.all(res < 1e-10)
    for k, d in enumerate(insts):
        off, cols, kv, fb = _oracle_kbc(d)
        u_dir = spla.spsolve(sp.csr_matrix((kv, cols, off)).tocsc(), fb)
        assert rel(us[k], u_dir) < 1e-7
        u_ref, it_ref, res_ref, rc = O.cg(off, cols, kv, fb, 1e-10, 20000)
        assert rc == 0
        # same stop rule as the reference CG for a cold start; at 1e-10 the count of
        # an unpreconditioned CG moves with rounding (exact parity at a fixed count below)
        assert abs(int(it[k]) - it_ref) <= max(10, 0.15 * it_ref)
        assert rel(us[k], u_ref) < 1e-7
    b.Destroy()


def test_batch_cg_fixed_iteration_count_parity():
    """After exactly 30 iterations every instance's iterate matches the oracle CG's."""
    insts = _instances(4)
    b = _batch(insts)
    b.Solve(1e-300, 30)
    it, res, st = b.GetResults()
    assert np.all(it == 30) and np.all(st == 2)
    us = b.RetrieveDisplacement()
    for k, d in enumerate(insts):
        off, cols, kv, fb = _oracle_kbc(d)
        u_ref, it_ref, res_ref, rc = O.cg(off, cols, kv, fb, 0.0, 30)
        assert it_ref == 30
        assert rel(us[k], u_ref) < 1e-9
        assert abs(res[k] - res_ref) <= 1e-6 * res_ref
    b.Destroy()


def test_batch_uneven_sizes_and_t4():
    insts = _instances(6, order=4, nx_range=(2, 12), ny_range=(1, 4))
    b = _batch(insts, order=4)
    b.Solve(1e-9, 20000)
    it, res, st = b.GetResults()
    us = b.RetrieveDisplacement()
    assert np.all(st == 0)
    for k, d in enumerate(insts):
        off, cols, kv, fb = _oracle_kbc(d)
        u_dir = spla.spsolve(sp.csr_matrix((kv, cols, off)).tocsc(), fb)
        assert rel(us[k], u_dir) < 1e-6
    b.Destroy()


def test_batch_warm_start():
    insts = _instances(3)
    b = _batch(insts)
    b.Solve(1e-8, 20000)
    it_cold, _, _ = b.GetResults()
    u = b.RetrieveDisplacement(split=False)
    b.SetInitialGuess(u)  # the solution itself: converged before the first iteration
    b.Solve(1e-8, 20000)
    it_exact, res, st = b.GetResults()
    assert np.all(st == 0) and np.all(it_exact <= 1)
    b.SetInitialGuess(u * (1.0 + 1e-4))  # a close guess: fewer iterations than cold
    b.Solve(1e-8, 20000)
    it_close, res, st = b.GetResults()
    assert np.all(st == 0) and np.all(it_close < it_cold)
    u2 = b.RetrieveDisplacement(split=False)
    assert rel(u2, u) < 1e-6
    b.SetInitialGuess(None)
    b.Solve(1e-8, 20000)
    assert np.array_equal(b.GetResults()[0], it_cold)
    b.Destroy()


def test_batch_edge_cases():
    insts = _instances(4)
    insts[1]["f"] = np.zeros_like(insts[1]["f"])          # no load
    insts[2]["fixed"] = np.arange(len(insts[2]["x"]))      # every node fixed
    b = _batch(insts)
    b.Solve(1e-10, 20000)
    it, res, st = b.GetResults()
    us = b.RetrieveDisplacement()
    assert it[1] == 0 and st[1] == 0 and np.all(us[1] == 0.0)
    assert it[2] == 0 and st[2] == 0 and np.all(us[2] == 0.0)
    assert st[0] == 0 and st[3] == 0 and it[0] > 0
    b.Solve(1e-10, 3)  # iteration cap
    it, res, st = b.GetResults()
    assert st[0] == 2 and it[0] == 3 and st[1] == 0
    b.Destroy()


def test_batch_fp32_elements_with_fp64_refinement():
    """FP32 element work, FP64 verdict: iterative refinement (FP64 residual,
    FP32-element CG on the correction) until the true ||f - K u|| / ||f|| with
    the FP64 operator is below tol; the answer matches the FP64 solve and the
    reported residual is the FP64 one."""
    import torch

    insts = _instances(4)
    b = _batch(insts)
    b.Solve(1e-10, 20000)
    u64 = b.RetrieveDisplacement(split=False)
    it64 = b.GetResults()[0]
    b.SetPrecision("fp32")
    b.Solve(1e-8, 20000)
    it, res, st = b.GetResults()
    assert np.all(st == 0) and np.all(res < 1e-8) and np.all(it > 0)
    u32 = b.RetrieveDisplacement(split=False)
    assert rel(u32, u64) < 1e-7
    # the reported residual is the FP64 one: recompute it with the FP64 operator
    b.SetPrecision("fp64")
    ud = torch.tensor(u32, device="cuda")
    ku = torch.empty_like(ud)
    torch.cuda.synchronize()
    b.Apply(ud.data_ptr(), ku.data_ptr())
    ku = ku.cpu().numpy()
    o = 0
    for k, d in enumerate(insts):
        n3 = 3 * len(d["x"])
        f = d["f"].copy()
        r = f - ku[o:o + n3]
        for arr in (r, f):
            arr.reshape(-1, 3)[d["fixed"]] = 0.0
        assert abs(np.linalg.norm(r) / np.linalg.norm(f) - res[k]) <= 1e-6 * res[k] + 1e-15
        o += n3
    b.Destroy()


def test_batch_autotune_and_replay_determinism():
    insts = _instances(8)
    b = _batch(insts)
    b.SetMode("persistent")
    cfg = b.Autotune(4)
    assert cfg["blocks_per_sm"] >= 1 and cfg["chunk_nodes"] in (128, 256, 512, 1024)
    L = b.GetLaunch()
    assert L["blocks_per_sm"] == cfg["blocks_per_sm"] and L["grid"] > 0
    b.SetMode("phased")  # per-phase launches tune the chunk size only
    cfg = b.Autotune(4)
    assert cfg["blocks_per_sm"] == 0 and cfg["chunk_nodes"] in (128, 256, 512, 1024)
    b.Solve(1e-9, 20000)
    u1 = b.RetrieveDisplacement(split=False)
    r1 = b.GetResults()
    b.Solve(1e-9, 20000)  # graph replay
    u2 = b.RetrieveDisplacement(split=False)
    r2 = b.GetResults()
    assert np.array_equal(u1, u2) and np.array_equal(r1[0], r2[0])
    b.SetLaunch(1, 128)  # a different launch shape: same answer to rounding
    b.Solve(1e-9, 20000)
    u3 = b.RetrieveDisplacement(split=False)
    assert rel(u3, u1) < 1e-7
    b.Destroy()


@pytest.mark.parametrize("shared", [False, True])
def test_phased_and_persistent_launches_agree_bitwise(shared):
    """The per-phase kernels (default) and the persistent cooperative launch run the
    same phase code with the same fixed summation orders: bitwise the same solution,
    iteration counts and residuals, cold and warm, and the same FP32-refined answer."""
    if shared:
        d0 = M.random_beam(5, order=10, **SMALL)
        r = np.random.default_rng(4)
        n = 11
        b = T.BatchedLinearStaticSolver([(d0["x"], d0["y"], d0["z"], d0["conn"])] * n, T.TYPE_T10, shared=True)
        b.SetMaterial(np.exp(r.uniform(np.log(1e6), np.log(1e9), n)), r.uniform(0.2, 0.45, n))
        b.SetNodalFixed([d0["fixed"]] * n)
        b.SetExternalForce([d0["f"] * s for s in r.uniform(0.5, 2.0, n)])
    else:
        b = _batch(_instances(9))
    out = {}
    for mode in ("persistent", "phased"):
        b.SetMode(mode)
        b.SetInitialGuess(None)
        b.Solve(1e-9, 20000)
        u = b.RetrieveDisplacement(split=False)
        res = b.GetResults()
        b.SetInitialGuess(0.9 * u)
        b.Solve(1e-9, 20000)
        uw = b.RetrieveDisplacement(split=False)
        resw = b.GetResults()
        b.SetInitialGuess(None)
        b.SetPrecision("fp32")
        b.Solve(1e-8, 20000)
        u32 = b.RetrieveDisplacement(split=False)
        b.SetPrecision("fp64")
        b.Solve(1e-12, 7)  # the iteration cap ends every instance with status 2
        capped = b.GetResults()
        out[mode] = (u, res, uw, resw, u32, capped)
    a, c = out["persistent"], out["phased"]
    assert np.all(a[1][2] == 0) and np.all(a[3][2] == 0)
    assert np.all(c[5][0] == 7) and np.all(c[5][2] == 2)
    for x, y in zip(a, c):
        if isinstance(x, tuple):
            for xx, yy in zip(x, y):
                assert np.array_equal(xx, yy)
        else:
            assert np.array_equal(x, y)
    b.Destroy()


@pytest.mark.parametrize("order", [10, 4])
def test_shared_mesh_batch_matches_the_general_batch(order):
    """One mesh, many materials / loads / fixed sets: the shared-mesh batch (one
    tiling for all instances) gives the general batch's products and solutions."""
    import torch

    d0 = M.random_beam(7, order=order, **SMALL)
    n = 5
    r = np.random.default_rng(3)
    E = np.exp(r.uniform(np.log(1e6), np.log(1e9), n))
    nu = r.uniform(0.2, 0.45, n)
    loads = [d0["f"] * s for s in r.uniform(0.5, 2.0, n)]
    fixed = [d0["fixed"]] * (n - 1) + [np.concatenate([d0["fixed"], [len(d0["x"]) - 1]])]
    mesh = (d0["x"], d0["y"], d0["z"], d0["conn"])
    T_ = T.TYPE_T10 if order == 10 else T.TYPE_T4
    bs = T.BatchedLinearStaticSolver([mesh] * n, T_, shared=True)
    bg = T.BatchedLinearStaticSolver([mesh] * n, T_)
    for b in (bs, bg):
        b.SetMaterial(E, nu)
        b.SetNodalFixed(fixed)
        b.SetExternalForce(loads)
    assert bs.GetCounts()["nodes"] == bg.GetCounts()["nodes"]
    xv = torch.tensor(r.standard_normal(3 * bs.n_nodes), device="cuda")
    ys, yg = torch.empty_like(xv), torch.empty_like(xv)
    torch.cuda.synchronize()
    bs.Apply(xv.data_ptr(), ys.data_ptr())
    bg.Apply(xv.data_ptr(), yg.data_ptr())
    assert rel(ys.cpu().numpy(), yg.cpu().numpy()) < 1e-12
    for b in (bs, bg):
        b.Solve(1e-9, 20000)
    us, ug = bs.RetrieveDisplacement(split=False), bg.RetrieveDisplacement(split=False)
    its, itg = bs.GetResults()[0], bg.GetResults()[0]
    assert rel(us, ug) < 1e-7 and np.all(np.abs(its - itg) <= np.maximum(5, 0.05 * itg))
    for k in range(n):  # each instance against the oracle's assembled system
        d = dict(d0, E=E[k], nu=nu[k], f=loads[k], fixed=fixed[k])
        off, cols, kv, fb = _oracle_kbc(d)
        u_dir = spla.spsolve(sp.csr_matrix((kv, cols, off)).tocsc(), fb)
        assert rel(us[3 * k * len(d0["x"]):3 * (k + 1) * len(d0["x"])], u_dir) < 1e-6
    bs.Destroy()
    bg.Destroy()


def test_shared_mesh_single_instance_and_fp32_refinement():
    """A shared-mesh batch of one instance, and a shared-mesh batch in FP32
    element work with FP64 refinement, against the general batch."""
    d0 = M.random_beam(11, order=10, **SMALL)
    mesh = (d0["x"], d0["y"], d0["z"], d0["conn"])
    for n in (1, 9):
        r = np.random.default_rng(n)
        E = np.exp(r.uniform(np.log(1e6), np.log(1e9), n))
        nu = r.uniform(0.2, 0.45, n)
        loads = [d0["f"] * s for s in r.uniform(0.5, 2.0, n)]
        bs = T.BatchedLinearStaticSolver([mesh] * n, T.TYPE_T10, shared=True)
        bg = T.BatchedLinearStaticSolver([mesh] * n, T.TYPE_T10)
        for b in (bs, bg):
            b.SetMaterial(E, nu)
            b.SetNodalFixed([d0["fixed"]] * n)
            b.SetExternalForce(loads)
        bg.Solve(1e-10, 20000)
        ug = bg.RetrieveDisplacement(split=False)
        bs.Solve(1e-10, 20000)
        assert np.all(bs.GetResults()[2] == 0)
        assert rel(bs.RetrieveDisplacement(split=False), ug) < 1e-7
        bs.SetPrecision("fp32")
        bs.Solve(1e-8, 20000)
        it, res, st = bs.GetResults()
        assert np.all(st == 0) and np.all(res < 1e-8)
        assert rel(bs.RetrieveDisplacement(split=False), ug) < 1e-6
        bs.Destroy()
        bg.Destroy()


def test_configuration3_batch_sample_matches_oracle_inside_the_full_launch():
    """The benchmark's 512 seeded uneven cantilevers (nx ~ U{8..64}, ny = nz ~ U{2..8})
    in one launch, stopped after exactly 25 CG iterations; 8 instances spread over the
    batch (the largest among them) against the oracle CG at the same count."""
    insts = [M.random_beam(s) for s in range(512)]
    b = _batch(insts)
    b.Solve(1e-300, 25)
    it, res, st = b.GetResults()
    assert np.all(it == 25)
    us = b.RetrieveDisplacement()
    sizes = np.array([len(d["x"]) for d in insts])
    picks = sorted(set(np.linspace(0, 511, 7).astype(int).tolist() + [int(np.argmax(sizes))]))
    for k in picks:
        d = insts[k]
        off, cols, kv, fb = _oracle_kbc(d)
        u_ref, it_ref, res_ref, rc = O.cg(off, cols, kv, fb, 0.0, 25)
        assert it_ref == 25
        assert rel(us[k], u_ref) < 1e-9, (k, rel(us[k], u_ref))
    b.Destroy()
