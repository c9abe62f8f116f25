#!/usr/bin/env python
"""Benchmark: solves/s at relative residual 1e-6 on one B200; element-force GB/s.

Workload (configuration 2, TET10, the metric's single-GPU configuration; the
learned-vs-plain comparison runs on configuration 4's fixed mesh and is reported
under "learned"): 1.0 x 0.1 x 0.1 m cantilever,
200 x 20 x 20 hex cells Kuhn-split into 480,000 TET10 elements / 674,081 nodes
(2,022,243 DOF); SVK E = 1e7 Pa, nu = 0.3, rho = 1000; nodes at x = 0 clamped;
a seeded total load (magnitude U[10, 1000] N, seed 0) in -z split over the
x = 1 face.  A step is one LinearStaticSolver::Solve() from the reference
configuration: stiffness assembly at the current positions, Dirichlet
elimination, unpreconditioned FP64 CG to ||r||/||f|| < 1e-6, position update.

The JSON line carries
  value     solves/s with all inputs resident in HBM (CUDA events on the
            element's stream, max over ranks; --gpus N runs N replicas);
  e2e       the same through the public API with host buffers: per step the
            external force and reference positions go host->device and the
            solved positions come back;
  roofline  the dominant kernel of the step (the CG's matrix-free K p: gather,
            k_mf_geo, combine);
  elem_force  the fused element-force kernel (FP32 and FP64) in GB/s of the
            algorithmic bytes E*(4*NPE + QP*NPE*3*s + QP*s) + N*6*s;
  gpu_reference the reference's own CUDA build (its unchanged sources compiled
            for sm_100a, oracle/build_ref.py) on the same workload and GPU: its
            LinearStaticSolver::Solve() and its CalcP + CalcInternalForce;
  cpu_baseline the CPU oracle (C + OpenMP) on a bounded sample of the workload,
            plus one complete CPU solve of the configuration-4 beam.
--impl reference times the reference's own CUDA build on this workload (the
reference has no CPU implementation of the path); where that build is absent it
falls back to the CPU oracle port.
Inputs are larger than L2 (the matrix-free product's streams: 0.53 GB; K: 1.35 GB;
the force kernels' gradient streams: 0.29 / 0.58 GB).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CFG = dict(nx=200, ny=20, nz=20, order=10, lx=1.0, ly=0.1, lz=0.1, E=1e7, nu=0.3, rho=1000.0, tol=1e-6, seed=0)
METRIC = "solves/s at rel. residual 1e-6 (learned vs plain, 1 B200); elem-force GB/s"
WORKLOAD = ("configuration 2: cantilever 200x20x20 TET10, plain linear static CG to 1e-6 (the metric's single-GPU "
            "configuration; learned vs plain on configuration 4 under 'learned')")
# CG iterations of this workload's solve (7071 to reach 1e-6 on a B200); the bounded
# CPU sample of the fallback reference arm is scaled to one solve with it.
CG_ITERS_CFG2 = 7071
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) per launch from ncu captures:
# the SpMV on the 120x16x16 beam moved 1.026 x its algorithmic bytes (the 200x20x20 K is
# too large for a multi-pass capture; traffic scales with the blocks streamed); on the
# 160x16x16 beam the gradient-stream force kernel moved 1.118 (FP32) / 1.073 (FP64) x its
# algorithmic bytes and the matrix-free product 1.073 x (the tile tables come on top;
# both scale with the elements), so the 200x20x20 traffic is those ratios x its bytes.
SPMV_TRAFFIC_RATIO = 1.026
FORCE_TRAFFIC_RATIO = {"fp32": 1.118, "fp64": 1.073}
MF_TRAFFIC_RATIO = 1.121


def progress(msg):
    """One progress line on stderr (the JSON result goes to stdout)."""
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_magnitude(seed):
    return float(np.random.default_rng(seed).uniform(10.0, 1000.0))


def build_mesh(cfg):
    from tlfea_b200 import mesh as M

    x, y, z, conn = M.box_mesh(cfg["nx"], cfg["ny"], cfg["nz"], cfg["order"], cfg["lx"], cfg["ly"], cfg["lz"])
    fixed, f, tip = M.cantilever_loads(x, y, z, (0.0, 0.0, -load_magnitude(cfg["seed"])))
    return x, y, z, conn, fixed, f


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device_index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(dist, seconds, device):
    """The slowest rank's time; every rank calls this in the same order (replicas
    only: this is the one collective of the benchmark)."""
    if not dist:
        return seconds
    import torch

    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, seconds):
    """Units of all ranks divided by the slowest rank's time."""
    return world * units_per_rank / seconds


def elem_force_bytes(E, N, npe, nqp, s):
    return E * (4 * npe + nqp * npe * 3 * s + nqp * s) + N * 6 * s


def elem_force_bytes_compact(E, N, npe, nqp, s):
    """The compact geometry stream: J^-1 (9 values) and dV per QP instead of the
    3 * NPE gradients."""
    return E * (4 * npe + nqp * 10 * s) + N * 6 * s


def mf_apply_bytes(E, N, npe, nqp):
    """Algorithmic bytes of one matrix-free K p: per element and QP the FP64 compact
    geometry (J^-1, dV) and the solve's tangent stream (F, S): 25 values; local
    connectivity and incidence (4 B per node slot); per node p read and q written (FP64)."""
    return E * (4 * npe + nqp * 25 * 8) + N * 3 * 8 * 2


def mf_apply_flops(E, nqp):
    """FP64 operations of one matrix-free K p, counted from the kernel's arithmetic per
    element and QP: dp/dxi (57), dF = (dp/dxi) J^-1 (27 FMA), symmetric dE (42), dS (12),
    dP = dF S + F dS scaled by dV (63), Q = dP J^-T (27 FMA), the nodal scatter (84);
    an FMA counts 2."""
    per_qp_ops = 57 + 27 + 42 + 12 + 63 + 27 + 84
    return E * nqp * per_qp_ops * 2


def spmv_bytes(N, nnzb):
    """Bytes one block SpMV must move: every 3x3 node block (72 B values +
    4 B column), the row offsets, p read and q written once."""
    return nnzb * (9 * 8 + 4) + (N + 1) * 4 + 3 * N * 8 * 2


def spmv_bytes_full_csr(N, nnzb):
    """The same product on the reference's full 3N x 3N FP64 CSR (8 B value +
    4 B column per entry, 3N+1 offsets, p and q)."""
    return 9 * nnzb * 12 + (3 * N + 1) * 4 + 3 * N * 8 * 2


def time_stream(torch, stream_ptr, fn, reps):
    st = torch.cuda.ExternalStream(stream_ptr)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def _lame(cfg):
    return cfg["E"] * cfg["nu"] / ((1 + cfg["nu"]) * (1 - 2 * cfg["nu"])), cfg["E"] / (2 * (1 + cfg["nu"]))


def cpu_sample(x, y, z, conn, fixed, f, cfg, iters_per_solve, iters_source, threads=0, cg_iters=50):
    """The oracle (C + OpenMP) on the host cores, on a bounded sample of the
    workload: the full stiffness assembly with Dirichlet BCs and `cg_iters` CG
    iterations are timed; one solve is assembly + `iters_per_solve` iterations,
    the count this workload's CG takes (from `iters_source`).  The gradient
    precompute (set-up) is not counted.  Reported as a modelled figure."""
    from oracle import oracle as O

    if threads:
        O.set_threads(threads)
    lam, mu = _lame(cfg)
    g, dj = O.dndu_pre(x, y, z, conn)
    t0 = time.perf_counter()
    off, cols, vals = O.stiffness(x, y, z, conn, g, dj, lam, mu)
    kv, fb = O.apply_bcs(off, cols, vals, f, fixed)
    t_asm = time.perf_counter() - t0
    del g
    t0 = time.perf_counter()
    u, it, res, rc = O.cg(off, cols, kv, fb, 0.0, cg_iters)
    t_cg = (time.perf_counter() - t0) / max(it, 1)
    per_solve = t_asm + iters_per_solve * t_cg
    return {"value": 1.0 / per_solve, "unit": "solves/s", "cores": O.get_threads(), "kind": "port",
            "modelled": True,
            "sample": (f"oracle (C, OpenMP) on this workload: stiffness assembly + BCs ({t_asm:.2f} s) and {it} CG "
                       f"iterations ({t_cg * 1e3:.1f} ms each) timed; one solve = assembly + {iters_per_solve} "
                       f"iterations ({iters_source})"),
            "timed": {"assembly_s": round(t_asm, 3), "cg_iterations": it, "cg_iteration_ms": round(t_cg * 1e3, 3)}}


def cpu_full_solve(threads=0, cells=(40, 8, 8)):
    """One complete CPU solve by the oracle, every stage timed: the
    configuration-4 beam (40x8x8 TET10, 70,227 DOF; E = 1e7, nu = 0.3, 100 N in
    -z over the tip face) -- gradients, stiffness assembly, BCs and CG to 1e-6."""
    from oracle import oracle as O
    from tlfea_b200 import mesh as M

    if threads:
        O.set_threads(threads)
    x, y, z, conn = M.box_mesh(*cells, 10)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -100.0))
    lam, mu = _lame(CFG)
    t0 = time.perf_counter()
    g, dj = O.dndu_pre(x, y, z, conn)
    off, cols, vals = O.stiffness(x, y, z, conn, g, dj, lam, mu)
    kv, fb = O.apply_bcs(off, cols, vals, f, fixed)
    u, it, res, rc = O.cg(off, cols, kv, fb, 1e-6, 1000000)
    dt = time.perf_counter() - t0
    return {"workload": f"configuration 4 beam {cells[0]}x{cells[1]}x{cells[2]} TET10 ({3 * len(x)} DOF), linear "
                        f"static CG to 1e-6, one complete solve", "value": round(1.0 / dt, 4), "unit": "solves/s",
            "seconds": round(dt, 3), "cg_iterations": it, "final_rel_residual": res, "cores": O.get_threads(),
            "kind": "port"}


def gpu_reference_leg(cfg, x, y, z, conn, fixed, f, steps, warmup, force_reps=5):
    """The reference's own CUDA build (oracle/_ref/libtlfea_ref.so: its unchanged
    sources for sm_100a) on the same workload and GPU.  A step resets the positions
    (UpdatePositions, host -> device) and runs LinearStaticSolver::Solve()
    (LinearStaticSolver.cu:590-603: assembly with atomics into its full 3N x 3N CSR,
    BCs, cuSPARSE/cuBLAS CG with host-synchronised dots, position update); host wall
    time, the reference's calls being synchronous.  Its CalcP + CalcInternalForce
    (FEAT10Data.cu:287-323) is timed on a fresh element and reported in GB/s of the
    same FP64 algorithmic bytes as this library's force kernel."""
    from oracle import ref_lib as R

    el = R.RefElement(x, y, z, conn, cfg["E"], cfg["nu"], cfg["rho"], fixed, f, with_mass=False)
    ls = R.RefLinearStatic(el, cfg["tol"], 1000000)

    def step():
        el.update_positions(x, y, z)
        return ls.solve()

    it = res = None
    for _ in range(warmup):
        it, res, _ = step()
    t0 = time.perf_counter()
    for _ in range(steps):
        it, res, _ = step()
    per = (time.perf_counter() - t0) / steps
    ls.destroy()
    el.destroy()
    el = R.RefElement(x, y, z, conn, cfg["E"], cfg["nu"], cfg["rho"], fixed, f, with_mass=False)
    r = np.random.default_rng(1)
    el.update_positions(*(v + 1e-4 * r.standard_normal(v.shape) for v in (x, y, z)))
    ms_f = el.time_force(force_reps)
    el.destroy()
    E, N = conn.shape[0], len(x)
    b = elem_force_bytes(E, N, conn.shape[1], 5 if conn.shape[1] == 10 else 1, 8)
    return {"value": round(1.0 / per, 4), "unit": "solves/s", "ms_per_step": round(per * 1e3, 2), "steps": steps,
            "cg_iters_per_solve": it, "final_rel_residual": res,
            "elem_force_fp64": {"ms": round(ms_f, 4), "achieved_gbs": round(b / (ms_f / 1e3) / 1e9, 1),
                                "algorithmic_bytes": int(b), "path": "CalcP + CalcInternalForce"},
            "build": "reference sources unchanged, nvcc -gencode arch=compute_100a,code=sm_100a -O3 (oracle/build_ref.py)"}


def run_reference(args):
    """--impl reference: the reference's own implementation of the path on this box.
    The reference's path is CUDA code (it has no CPU implementation), so this times
    its own CUDA build on the GPU; without that build, the CPU oracle port."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = dict(CFG)
    x, y, z, conn, fixed, f = build_mesh(cfg)
    from oracle import ref_lib as R

    out = {"impl": "reference", "metric": METRIC, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic",
           "config": {"workload": WORKLOAD, "elements": int(conn.shape[0]), "nodes": int(len(x)),
                      "parallelism": "single process (rank 0)"}}
    if R.available():
        g = gpu_reference_leg(cfg, x, y, z, conn, fixed, f, args.steps, max(1, args.warmup))
        v = g["value"]
        out.update(value=v, ms_per_step=g["ms_per_step"], gpu_reference=g)
        out["cpu_baseline"] = {"value": v, "unit": "solves/s", "cores": 0, "kind": "reference",
                               "sample": ("the reference's own CUDA build on one B200 (the reference has no CPU "
                                          f"implementation of this path): {args.steps} complete solves timed"),
                               "device": "B200"}
    else:
        vals = []
        for i in range(args.warmup + args.steps):
            s = cpu_sample(x, y, z, conn, fixed, f, cfg, CG_ITERS_CFG2, "this workload's CG on a B200")
            if i >= args.warmup:
                vals.append(s["value"])
        v = float(np.median(vals))
        s["value"] = v
        out.update(value=v, ms_per_step=1e3 / v, cpu_baseline=s)
    out["e2e"] = {"value": out["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(out))


def setup_element(T, cfg, x, y, z, conn, fixed, f):
    el = T.GPU_FEAT10_Data(conn.shape[0], len(x))
    el.Initialize()
    el.SetNodalFixed(fixed)
    el.SetExternalForce(f)
    el.Setup(*T.Quadrature.t10(), x, y, z, conn)
    el.SetDensity(cfg["rho"])
    el.SetDamping(0.0, 0.0)
    el.SetSVK(cfg["E"], cfg["nu"])
    el.CalcDnDuPre()
    return el


def kernels_only(args):
    """A small profiling case per --kernels-only value: on the --mesh beam the fused
    element force (force: 2 x FP32 then 2 x FP64), the CG operator (spmv: a 5-iteration
    solve, then 3 applies), the benchmark solve capped at --cg-iters iterations (cg), or
    SyncedNesterov in per-phase launches (nesterov); the batched CG (batch: shared mesh,
    batch-uneven: uneven instances), the persistent first-order solver (steps), the
    warm-start network's training step (mlp) or its BF16 product alone (gemm,
    --gemm-size cubed)."""
    import torch
    import tlfea_b200 as T

    torch.cuda.set_device(0)
    if args.kernels_only == "steps":
        # the persistent first-order solver: 2 AdamW steps of the configuration-5 sequence
        class _A:
            dyn_steps = 2
        print(json.dumps({"kernels_only": "steps", "dynamics": dynamics_leg(_A, T)["value"]}))
        return
    if args.kernels_only == "batch":
        # the batched CG: 64 load / material cases on the 40x8x8 TET10 beam, 10 iterations
        from tlfea_b200 import warmstart as W

        fm = W.FixedMeshCases(40, 8, 8, batch=64)
        if args.batch_mode != "auto":
            fm.solver.SetMode(args.batch_mode)
        fm.solve(W.sample_cases(64, seed=5), tol=1e-12, max_iter=10)
        torch.cuda.synchronize()
        print(json.dumps({"kernels_only": "batch", "cases": 64, "iterations": 10}))
        fm.destroy()
        return
    if args.kernels_only == "mlp":
        # the warm-start network's training step: 6-256-256-256-64, a batch of 512, 20 steps
        net = T.WarmStartMLP((6, 256, 256, 256, 64), max_batch=512, seed=0)
        g = torch.Generator(device="cuda").manual_seed(0)
        xb = torch.randn(512, 6, device="cuda", generator=g)
        tb = torch.randn(512, 64, device="cuda", generator=g)
        torch.cuda.synchronize()
        for _ in range(20):
            net.TrainStep(xb.data_ptr(), tb.data_ptr(), 512)
        torch.cuda.synchronize()
        print(json.dumps({"kernels_only": "mlp", "dims": [6, 256, 256, 256, 64], "batch": 512, "steps": 20}))
        net.Destroy()
        return
    if args.kernels_only == "nesterov":
        # SyncedNesterov on the --mesh beam in per-phase launches: one warm-up solve,
        # then 2 outer x 10 inner iterations at zero tolerances (FP64 element forces)
        cfg = dict(CFG)
        cfg["nx"], cfg["ny"], cfg["nz"] = (int(v) for v in (args.mesh or "200x20x20").split("x"))
        x, y, z, conn, fixed, f = build_mesh(cfg)
        el = setup_element(T, cfg, x, y, z, conn, fixed, f)
        el.CalcMassMatrix()
        el.CalcConstraintData()
        el.ConvertToCSR_ConstraintJacT()
        s = T.SyncedNesterovSolver(el, el.get_n_constraint())
        s.Setup()
        s.SetMode("phased")
        for _ in range(2):
            s.SetParameters(T.SyncedNesterovParams(1.0e-8, 1e14, 0.0, 0.0, 2, 10, 1.0e-3))
            el.ResetPositions()
            s.Solve()
        torch.cuda.synchronize()
        print(json.dumps({"kernels_only": "nesterov", "elements": int(conn.shape[0]), "nodes": int(len(x)),
                          "inner_iters": s.GetStats()["inner_iters_total"]}))
        return
    if args.kernels_only == "gemm":
        # the MLP's tcgen05 product on its own at a size that fills the GPU:
        # D[8192 x 8192] = A[8192 x 8192] B^T, BF16 operands, FP32 accumulation and output
        n = args.gemm_size
        g = torch.Generator(device="cuda").manual_seed(0)
        A = torch.randn(n, n, device="cuda", generator=g).to(torch.bfloat16)
        B = torch.randn(n, n, device="cuda", generator=g).to(torch.bfloat16)
        D = torch.empty(n, n, device="cuda")
        st = torch.cuda.current_stream()
        flag = torch.zeros(1, dtype=torch.int32, device="cuda")

        def launch():
            T.gemm_bf16_async(n, n, n, A.data_ptr(), n, B.data_ptr(), n, 0, D.data_ptr(), n, flag.data_ptr(),
                              st.cuda_stream)

        for _ in range(3):
            launch()
        # operands (2 x 128 MB at the default size) exceed L2, so back-to-back launches stream them
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(args.steps):
            launch()
        e1.record(st)
        torch.cuda.synchronize()
        if int(flag.item()) != 0:
            raise RuntimeError("gemm: a bounded wait in the kernel ran out")
        ref = (A[:256].float() @ B[:256].float().T)
        err = float((D[:256, :256] - ref).abs().max() / ref.abs().max())
        t = e0.elapsed_time(e1) * 1e-3 / args.steps
        tf = 2.0 * n ** 3 / t / 1e12
        pk = ROOT / "MEASURED_PEAKS.json"
        peak = float(json.loads(pk.read_text())["bf16_tflops"]) if pk.exists() else 1590.0
        print(json.dumps({"kernels_only": "gemm", "M": n, "N": n, "K": n, "ms": t * 1e3, "tflops": tf,
                          "peak_tflops": peak, "frac": tf / peak if peak else None, "max_rel_err_256": err}))
        return
    if args.kernels_only == "batch-uneven":
        # the batched CG of the uneven batch (general tiling): the first 64 seeded
        # cantilevers of the 512-instance batch, 10 iterations
        from tlfea_b200 import mesh as M

        insts = [M.random_beam(s) for s in range(64)]
        b = T.BatchedLinearStaticSolver([(d["x"], d["y"], d["z"], d["conn"]) for d in insts], T.TYPE_T10)
        b.SetMaterial([d["E"] for d in insts], [d["nu"] for d in insts])
        b.SetNodalFixed([d["fixed"] for d in insts])
        b.SetExternalForce(np.concatenate([d["f"] for d in insts]))
        b.Solve(1e-12, 10)
        torch.cuda.synchronize()
        print(json.dumps({"kernels_only": "batch-uneven", "cases": 64, "iterations": 10,
                          "nodes": b.GetCounts()["nodes"]}))
        b.Destroy()
        return
    cfg = dict(CFG)
    x, y, z, conn, fixed, f = build_mesh(cfg)
    el = setup_element(T, cfg, x, y, z, conn, fixed, f)
    r = np.random.default_rng(1)
    el.UpdatePositions(*(v + 1e-4 * r.standard_normal(v.shape) for v in (x, y, z)))
    if args.kernels_only == "force":
        # gradient-stream kernel, then the compact-geometry kernel
        for kern in ("tma", "compact"):
            el.SetLaunchConfig(kern)
            for prec in ("fp32", "fp32", "fp64", "fp64"):
                el.SetForcePrecision(prec)
                el.ComputeInternalForce()
    elif args.kernels_only == "cg":
        # the benchmark's solve capped at --cg-iters iterations: the per-iteration
        # launch mix of the full solve in a launch list short enough to capture
        el.ResetPositions()
        s = T.LinearStaticSolver(el, cfg["tol"], args.cg_iters)
        s.Solve()
        del s
    else:
        s = T.LinearStaticSolver(el, cfg["tol"], 5)
        s.SetOperator(args.operator)
        s.Solve()
        xin = torch.randn(3 * len(x), dtype=torch.float64, device="cuda")
        yout = torch.empty_like(xin)
        torch.cuda.synchronize()
        for _ in range(3):
            s.Apply(xin.data_ptr(), yout.data_ptr())
        del s
    torch.cuda.synchronize()
    print(json.dumps({"kernels_only": args.kernels_only, "elements": int(conn.shape[0]), "nodes": int(len(x))}))
    el.Destroy()


def _plain_solve_time(T, x, y, z, conn, fixed, f, E, nu, tol, el=None):
    """One cold-start LinearStaticSolver solve through the reference-named API;
    returns (seconds, iterations, element) -- set-up (gradients) is not timed."""
    import torch

    if el is None:
        el = T.GPU_FEAT10_Data(conn.shape[0], len(x))
        el.Initialize()
        el.SetNodalFixed(fixed)
        el.Setup(*T.Quadrature.t10(), x, y, z, conn)
        el.SetDensity(1000.0)
        el.SetDamping(0.0, 0.0)
        el.CalcDnDuPre()
    el.SetSVK(E, nu)
    el.SetExternalForce(f)
    el.ResetPositions()
    s = T.LinearStaticSolver(el, tol, 1000000)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.Solve()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    it = s.GetLastIterCount()
    del s
    return dt, it, el


def batched_leg(args, T):
    """Uneven batch: 512 seeded cantilevers (nx ~ U{8..64}, ny = nz ~ U{2..8},
    h = 0.01 m, length 10 ny h; E log-uniform 1e6..1e9, nu U[0.2, 0.45]; tip
    load direction on the sphere, magnitude U[1, 500] N) solved to 1e-6 by the batched
    CG (one kernel per phase, chunks of iterations replayed as CUDA graphs), against
    single-instance plain solves; the one-launch persistent mode timed beside it."""
    import torch
    from tlfea_b200 import mesh as M

    n = args.batch_size
    insts = [M.random_beam(s) for s in range(n)]
    b = T.BatchedLinearStaticSolver([(d["x"], d["y"], d["z"], d["conn"]) for d in insts], T.TYPE_T10)
    b.SetMaterial([d["E"] for d in insts], [d["nu"] for d in insts])
    b.SetNodalFixed([d["fixed"] for d in insts])
    f_all = np.concatenate([d["f"] for d in insts])
    b.SetExternalForce(f_all)
    b.SetPrecision(args.batch_precision)
    tune = b.Autotune(4)
    counts = b.GetCounts()
    st = b.GetStream()

    def step():
        b.Solve(1e-6, 200000)

    for _ in range(max(1, args.warmup // 3)):
        step()
    it, res, status = b.GetResults()
    reps = max(1, args.steps // 2)
    ms = time_stream(torch, st, step, reps)
    # end to end: loads host -> device, solve, displacements device -> host
    f_pin = torch.from_numpy(f_all).pin_memory()
    u_host = torch.empty(3 * b.n_nodes, dtype=torch.float64).pin_memory()
    t0 = time.perf_counter()
    for _ in range(reps):
        b.SetExternalForce(f_pin.numpy())
        step()
        u_host.numpy()[:] = b.RetrieveDisplacement(split=False)
    t_e2e = (time.perf_counter() - t0) / reps
    launch = b.GetLaunch()
    u_main = b.RetrieveDisplacement(split=False)
    # the same solve as one persistent cooperative launch, for comparison
    b.SetMode("persistent")
    pt = b.Autotune(4)
    b.SetLaunch(pt["blocks_per_sm"], launch["chunk_nodes"])  # the same chunks: the same sums
    step()
    ms_pers = time_stream(torch, st, step, 1)
    same_pers = bool(np.array_equal(b.RetrieveDisplacement(split=False), u_main))
    b.SetMode("phased")
    b.SetLaunch(0, launch["chunk_nodes"])
    # the same batch with the other element precision, for comparison
    other = "fp64" if args.batch_precision == "fp32" else "fp32"
    b.SetPrecision(other)
    step()
    ms_other = time_stream(torch, st, step, 1)
    it_o, res_o, st_o = b.GetResults()
    u_other = b.RetrieveDisplacement(split=False)
    b.Destroy()
    u64, u32 = (u_main, u_other) if other == "fp32" else (u_other, u_main)
    disp_err = float(np.linalg.norm(u32 - u64) / np.linalg.norm(u64))
    # plain path: one instance at a time, cold start (a seeded sample of the batch)
    k = min(args.plain_sample, n)
    tot, its = 0.0, []
    for d in insts[:k]:
        dt, itp, el = _plain_solve_time(T, d["x"], d["y"], d["z"], d["conn"], d["fixed"], d["f"], d["E"], d["nu"],
                                        1e-6)
        el.Destroy()
        tot += dt
        its.append(itp)
    plain = k / tot
    value = n / (ms / 1e3)
    # roofline of the batched CG: per iteration an instance streams its compact geometry
    # (J^-1 and dV per element and QP, FP64) and makes ~14 passes over 3N-vectors (the
    # matrix-free K p reads p and writes q; p.Kp, u/r update with r.r, p update); summed
    # over the iterations each instance ran, over the batch's time
    hbm, _ = peaks()
    per_iter = np.array([d["conn"].shape[0] * 5 * 10 * 8 + 3 * len(d["x"]) * 8 * 14 for d in insts], np.float64)
    moved = float(np.sum(per_iter * np.asarray(it, np.float64)))
    ach = moved / (ms / 1e3) / 1e9
    roof = {"kernel": "k_bcg_* (whole solve)", "bound": "hbm", "achieved": round(ach, 1), "peak": hbm,
            "unit": "GB/s", "frac": round(ach / hbm, 4), "algorithmic_bytes": int(moved),
            "model": "per instance and iteration: E*5*10*8 (J^-1 + dV stream) + 3N*8*14 (vector passes)"}
    return {"workload": f"{n} uneven TET10 cantilevers, linear static CG to 1e-6 (per-phase kernels, graph chunks)",
            "roofline": roof,
            "elements": counts["elements"], "nodes": counts["nodes"], "dof": 3 * counts["nodes"],
            "precision": args.batch_precision, "value": round(value, 2), "unit": "solves/s",
            "ms_per_batch": round(ms, 3), "iters_mean": float(np.mean(it)), "iters_max": int(np.max(it)),
            "converged": int(np.sum(status == 0)), "max_rel_residual": float(np.max(res)),
            "e2e": {"value": round(n / t_e2e, 2), "unit": "solves/s", "h2d_bytes_per_step": int(f_all.nbytes),
                    "d2h_bytes_per_step": int(8 * 3 * counts["nodes"])},
            "launch": launch, "autotune": tune,
            "persistent_launch": {"ms_per_batch": round(ms_pers, 3), "value": round(n / (ms_pers / 1e3), 2),
                                  "bitwise_same_displacement": same_pers},
            "other_precision": {"precision": other, "value": round(n / (ms_other / 1e3), 2),
                                "ms_per_batch": round(ms_other, 3), "iters_mean": float(np.mean(it_o)),
                                "converged": int(np.sum(st_o == 0)), "max_rel_residual": float(np.max(res_o)),
                                "fp32_displacement_rel_error_vs_fp64": disp_err},
            "plain_sequential": {"value": round(plain, 2), "unit": "solves/s", "sample": k,
                                 "iters_mean": float(np.mean(its)),
                                 "path": "LinearStaticSolver per instance (assembled K, CG graph), cold start"},
            "speedup_vs_plain": round(value / plain, 2)}


def dynamics_leg(args, T):
    """Configuration 5, one sequence: 100x10x10 TET10 cantilever (60,000 elements),
    SVK E = 1e7, nu = 0.3, rho = 1000, clamped at x = 0; gravity 9.81 m/s^2 in -z
    (consistent-mass row sums) plus a 50 sin(2 pi 5 t) N tip load in -z; SyncedAdamW
    with dt = 1e-3 and the damping and parameters of the reference's dynamics example
    (beam_simulation.cc:203, 226).  `--dyn-steps` implicit steps run as one CUDA graph
    with the load computed on the device (RunSteps), against the reference's host
    loop of SetExternalForce + Solve (beam_simulation.cc:275-283; same answer)."""
    import torch
    from tlfea_b200 import mesh as M

    x, y, z, conn = M.box_mesh(100, 10, 10, 10, 1.0, 0.1, 0.1)
    fixed, f_tip, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -50.0))
    params = T.SyncedAdamWParams(2e-4, 0.9, 0.999, 1e-8, 1e-4, 0.995, 1e-1, 1e-6, 1e14, 5, 300, 1e-3, 10, 0.0)
    omega = 2 * np.pi * 5.0
    n = args.dyn_steps

    def make():
        el = T.GPU_FEAT10_Data(conn.shape[0], len(x))
        el.Initialize()
        el.SetNodalFixed(fixed)
        el.SetExternalForce(np.zeros(3 * len(x)))
        el.Setup(*T.Quadrature.t10(), x, y, z, conn)
        el.SetDensity(1000.0)
        el.SetDamping(0.0, 0.1)
        el.SetSVK(1e7, 0.3)
        el.CalcDnDuPre()
        el.CalcMassMatrix()
        el.CalcConstraintData()
        el.ConvertToCSR_ConstraintJacT()
        el.AddGravity(0.0, 0.0, -9.81)
        s = T.SyncedAdamWSolver(el, el.get_n_constraint())
        s.Setup()
        s.SetParameters(params)
        return el, s

    el, s = make()
    s.RunSteps(1)  # warm-up: first launch, graph build
    el.Destroy()
    el, s = make()
    f_grav = el.RetrieveExternalForceToCPU()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    its = s.RunSteps(n, f_tip, amp=1.0, omega=omega, phase=0.0, t0=0.0)
    t_graph = time.perf_counter() - t0
    x_graph = np.stack(el.RetrievePositionToCPU())
    el.Destroy()
    el, s = make()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    its_h = []
    for k in range(n):
        el.SetExternalForce(f_grav + np.sin(omega * ((k + 1) * 1.0e-3)) * f_tip)
        s.Solve()
        its_h.append(s.GetStats()["inner_iters_total"])
    t_host = time.perf_counter() - t0
    x_host = np.stack(el.RetrievePositionToCPU())
    tip_z = float((x_graph[2] - z).min())
    el.Destroy()
    return {"workload": f"configuration 5 (one sequence): 100x10x10 TET10, gravity + 50 sin(2 pi 5 t) N tip load, "
                        f"SyncedAdamW dt 1e-3, {n} steps", "elements": int(conn.shape[0]), "nodes": int(len(x)),
            "value": round(n / t_graph, 3), "unit": "steps/s", "inner_iters_per_step": float(np.mean(its)),
            "host_loop": {"value": round(n / t_host, 3), "unit": "steps/s",
                          "inner_iters_per_step": float(np.mean(its_h))},
            "graph_vs_host_loop_max_abs_position_diff": float(np.abs(x_graph - x_host).max()),
            "tip_deflection_min_z": tip_z}


def config2_more_legs(args, T, cfg):
    """Configuration 2's other legs.
    * SyncedNesterov on the 200x20x20 TET10 mesh (2,022,243 DOF), one implicit step with
      the parameters of the reference's Nesterov example (test_feat10_nesterov.cc:189:
      alpha 1e-8, rho 1e14, tolerances 1e-6, 5 x 300 iterations, dt 1e-3) from the
      reference configuration under the seeded tip load, FP64 and FP32 element forces.
      Reported per inner iteration (the unit of the method's work).  The reference's own
      Nesterov kernel is not timed: at this size it clamps its grid to the co-resident
      blocks and never updates the DOFs beyond it (SyncedNesterov.cu:391-397).
    * The TET4 variant: the same beam with corner nodes only (201x21x21 = 88,641 nodes,
      480,000 TET4 elements), linear static CG to 1e-6, beside the reference's own CUDA
      build on the same GPU."""
    import torch
    from tlfea_b200 import mesh as M

    out = {}
    x, y, z, conn, fixed, f = build_mesh(cfg)
    el = setup_element(T, cfg, x, y, z, conn, fixed, f)
    el.CalcMassMatrix()
    el.CalcConstraintData()
    el.ConvertToCSR_ConstraintJacT()
    nes = {}
    for prec in ("fp64", "fp32"):
        el.SetForcePrecision(prec)
        s = T.SyncedNesterovSolver(el, el.get_n_constraint())
        s.Setup()
        s.SetParameters(T.SyncedNesterovParams(1.0e-8, 1e14, 1.0e-6, 1.0e-6, 5, 300, 1.0e-3))
        el.ResetPositions()
        s.Solve()  # warm-up (first launch)
        s.SetParameters(T.SyncedNesterovParams(1.0e-8, 1e14, 1.0e-6, 1.0e-6, 5, 300, 1.0e-3))
        el.ResetPositions()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.Solve()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        st = s.GetStats()
        it = max(1, st["inner_iters_total"])
        nes[prec] = {"step_s": round(dt, 4), "inner_iters": st["inner_iters_total"], "outer_iters": st["outer_iters"],
                     "ms_per_inner_iteration": round(1e3 * dt / it, 4),
                     "inner_iterations_per_s": round(it / dt, 1), "kernel_ms": round(st["kernel_ms"], 3)}
        # the cost of one inner iteration: 60 iterations at zero tolerances (2 outer x 30
        # inner), in both launch modes
        fixed_it = {}
        for mode in ("phased", "persistent"):
            s.SetMode(mode)
            s.SetParameters(T.SyncedNesterovParams(1.0e-8, 1e14, 0.0, 0.0, 2, 30, 1.0e-3))
            el.ResetPositions()
            s.Solve()
            s.SetParameters(T.SyncedNesterovParams(1.0e-8, 1e14, 0.0, 0.0, 2, 30, 1.0e-3))
            el.ResetPositions()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.Solve()
            torch.cuda.synchronize()
            dtf = time.perf_counter() - t0
            stf = s.GetStats()
            itf = max(1, stf["inner_iters_total"])
            fixed_it[mode] = {"inner_iters": itf, "ms_per_inner_iteration": round(1e3 * dtf / itf, 4),
                              "gpu_ms_per_inner_iteration": round(stf["kernel_ms"] / itf, 4)}
        s.SetMode("auto")
        nes[prec]["fixed_60_iterations"] = fixed_it
        del s
    el.SetForcePrecision("fp64")
    el.Destroy()
    out["nesterov_200x20x20_t10"] = {
        "workload": "SyncedNesterov, one implicit step from rest, the reference example's parameters",
        **nes, "reference": "not timed: its cooperative kernel leaves DOFs beyond the co-resident grid un-updated"}
    # TET4 CG
    c4 = dict(cfg, order=4)
    x4, y4, z4, conn4 = M.box_mesh(c4["nx"], c4["ny"], c4["nz"], 4, c4["lx"], c4["ly"], c4["lz"])
    fixed4, f4, _ = M.cantilever_loads(x4, y4, z4, (0.0, 0.0, -load_magnitude(c4["seed"])))
    el = T.GPU_FEAT4_Data(conn4.shape[0], len(x4))
    el.Initialize()
    el.SetNodalFixed(fixed4)
    el.SetExternalForce(f4)
    el.Setup(*T.Quadrature.t4(), x4, y4, z4, conn4)
    el.SetDensity(c4["rho"])
    el.SetDamping(0.0, 0.0)
    el.SetSVK(c4["E"], c4["nu"])
    el.CalcDnDuPre()
    solver = T.LinearStaticSolver(el, c4["tol"], 1000000)
    stream = el.GetStream()

    def step():
        el.ResetPositions()
        solver.Solve()

    for _ in range(2):
        step()
    ms = time_stream(torch, stream, step, max(1, args.steps))
    t4 = {"value": round(1e3 / ms, 3), "unit": "solves/s", "ms_per_step": round(ms, 3),
          "cg_iters_per_solve": solver.GetLastIterCount(), "final_rel_residual": solver.GetLastResidual(),
          "elements": int(conn4.shape[0]), "nodes": int(len(x4))}
    for _ in range(3):
        el.ComputeInternalForce()
    ms_f = time_stream(torch, stream, el.ComputeInternalForce, args.kernel_reps)
    b = elem_force_bytes(conn4.shape[0], len(x4), 4, 1, 8)
    hbm, _ = peaks()
    t4["elem_force_fp64"] = {"ms": round(ms_f, 4), "achieved_gbs": round(b / (ms_f / 1e3) / 1e9, 1),
                             "frac": round(b / (ms_f / 1e3) / 1e9 / hbm, 4), "algorithmic_bytes": int(b)}
    del solver
    el.Destroy()
    from oracle import ref_lib as R

    if R.available() and not args.no_gpu_ref:
        g = gpu_reference_leg(c4, x4, y4, z4, conn4, fixed4, f4, steps=2, warmup=1)
        t4["gpu_reference"] = {k: g[k] for k in ("value", "ms_per_step", "cg_iters_per_solve", "elem_force_fp64")}
        t4["speedup_vs_reference"] = round(t4["value"] / g["value"], 3)
    out["cg_200x20x20_t4"] = t4
    return out


def config5_leg(args, T):
    """Configuration 5: 64 sequences on the 100x10x10 TET10 cantilever (60,000 elements,
    88,641 nodes; SVK, rho = 1000, seeded E log-uniform in [3e6, 3e7] Pa and nu in
    [0.25, 0.4]), clamped at x = 0, gravity 9.81 m/s^2 (consistent-mass row sums) plus a
    50 sin(2 pi 5 t) N tip load in -z, implicit steps dt = 1e-3 each solved by the
    SyncedNesterov iteration (with the gradient momentum restart) to ||g_free|| / ||f_ext||
    < 1e-6, all 64 sequences batched in the same kernels (BatchedDynamics).  Warm starts of
    each step compared from rest over the same steps: a cold start (v = 0), the previous
    velocity (the reference's behaviour), linear extrapolation, and the learned step
    predictor (an MLP correction of the linear extrapolation, trained on the solver's own
    steps of 16 other seeded sequences).
    Step size per sequence: 0.9 / lambda_max of the step Hessian M/dt + dt K_s
    (+ dt^2 rho on fixed DOFs), lambda_max by a batched power iteration with this
    library's K x and mass matrix."""
    import torch
    from tlfea_b200 import mesh as M
    from tlfea_b200 import warmstart as W

    dt, rho_alm, tol, omega = 1e-3, 1e8, 1e-6, 2 * np.pi * 5.0
    n_eval, n_train = args.dyn_batch, 16
    steps_eval, steps_train = args.dyn_eval_steps, args.dyn_train_steps
    x, y, z, conn = M.box_mesh(100, 10, 10, 10, 1.0, 0.1, 0.1)
    fixed, f_tip, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -50.0))
    N, dof = len(x), 3 * len(x)
    r = np.random.default_rng(5)
    E_all = np.exp(r.uniform(np.log(3e6), np.log(3e7), n_eval + n_train))
    nu_all = r.uniform(0.25, 0.4, n_eval + n_train)
    el = T.GPU_FEAT10_Data(conn.shape[0], N)
    el.Initialize()
    el.SetNodalFixed(fixed)
    el.SetExternalForce(np.zeros(dof))
    el.Setup(*T.Quadrature.t10(), x, y, z, conn)
    el.SetDensity(1000.0)
    el.SetDamping(0.0, 0.0)
    el.SetSVK(1e7, 0.3)
    el.CalcDnDuPre()
    el.CalcMassMatrix()
    el.CalcConstraintData()
    el.ConvertToCSR_ConstraintJacT()
    el.AddGravity(0.0, 0.0, -9.81)

    # lambda_max of M/dt + dt K_s over the free DOFs, every sequence at once
    t0 = time.perf_counter()
    moff, mcol, mval = el.RetrieveMassCSRToCPU()
    Mn = torch.sparse_csr_tensor(torch.as_tensor(moff, dtype=torch.int64), torch.as_tensor(mcol, dtype=torch.int64),
                                 torch.as_tensor(mval), size=(N, N)).to("cuda")
    nb = n_eval + n_train
    kb = T.BatchedLinearStaticSolver([(x, y, z, conn)] * nb, T.TYPE_T10, shared=True)
    kb.SetMaterial(E_all, nu_all)
    kb.SetNodalFixed([fixed] * nb)
    free = torch.ones(N, 3, dtype=torch.float64, device="cuda")
    free[torch.as_tensor(fixed, device="cuda")] = 0.0
    free = free.reshape(-1)
    X = torch.randn(nb, dof, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    Y = torch.empty_like(X)
    lmax = None
    for _ in range(60):
        X *= free
        X /= X.norm(dim=1, keepdim=True)
        torch.cuda.synchronize()
        kb.Apply(int(X.data_ptr()), int(Y.data_ptr()))
        MX = (Mn @ X.reshape(nb, N, 3).permute(1, 0, 2).reshape(N, nb * 3)).reshape(N, nb, 3).permute(1, 0, 2)
        HX = (MX.reshape(nb, dof) / dt + dt * Y) * free
        lmax = (HX * X).sum(1)
        X = HX
    kb.Destroy()
    alpha_all = 0.9 / (lmax.cpu().numpy() + dt * dt * rho_alm)
    t_alpha = time.perf_counter() - t0
    progress(f"config5: step sizes {alpha_all.min():.3e}..{alpha_all.max():.3e} in {t_alpha:.1f} s")

    params = T.SyncedNesterovParams(float(alpha_all.min()), rho_alm, 0.0, 1e-6, 3, 20000, dt)

    def make(seqs):
        b = T.BatchedDynamics(el, len(seqs))
        b.SetMaterial(E_all[seqs], nu_all[seqs])
        b.SetParameters(params, tol)
        b.SetStepSizes(alpha_all[seqs])
        f_var = np.zeros(dof)
        f_var[:] = f_tip
        b.SetLoad(f_var, 1.0, omega, 0.0)
        b.SetChunk(16)
        # the reference's beta schedule alone converges sublinearly on these steps
        # (condition number ~7.5e3 at E = 1e7): restart the momentum on g . dv > 0
        b.SetRestart(True)
        return b

    def load_factors(n):  # (sin at t_(n-1), t_n, t_(n+1)), t_k = k dt
        return np.array([[np.sin(omega * (n - 1 + j) * dt) for j in range(3)]])

    X0 = torch.as_tensor(np.stack([x, y, z], 1).reshape(-1), device="cuda")

    def state(b, B):
        p = b.DevicePtrs()
        v = W.device_view(p["v"], (B, dof))
        vh = W.device_view(p["v_hist"], (B, dof))
        xs = [W.device_view(p[k], (B, N)) for k in ("x", "y", "z")]
        u = torch.stack(xs, 2).reshape(B, dof) - X0
        return v, vh, u

    # training data: the solver's own steps (linear extrapolation) on 16 other sequences
    t0 = time.perf_counter()
    tr = np.arange(n_eval, n_eval + n_train)
    bt = make(tr)
    V = torch.empty(n_train, steps_train, dof, dtype=torch.float64, device="cuda")
    U = torch.empty_like(V)
    it_train = []
    for k in range(steps_train):
        it, res, conv = bt.Step(T.BatchedDynamics.WARM_LINEAR)
        it_train.append(it)
        progress(f"config5: training step {k + 1}: inner iterations mean {np.mean(it):.0f} max {np.max(it)}, "
                 f"converged {np.mean(conv):.2f}, {time.perf_counter() - t0:.1f} s")
        v, _, u = state(bt, n_train)
        V[:, k] = v
        U[:, k] = u
    bt.Destroy()
    loads_tr = np.concatenate([load_factors(n) for n in range(1, steps_train + 1)])
    sp = W.StepPredictor(k_in=16, k_out=32, hidden=(256, 256), max_batch=128, seed=0, E_range=(3e6, 3e7),
                         nu_range=(0.25, 0.4))
    mats = sp.material_features(E_all, nu_all)
    # samples: steps 1..T-1 of each training sequence; a batch is a multiple of 16 rows
    n_samples = n_train * (steps_train - 1)
    hist = sp.fit(V, U, loads_tr, mats[tr], epochs=args.dyn_epochs, batch=min(128, n_samples // 16 * 16))
    del V, U
    t_train = time.perf_counter() - t0

    # evaluation: the 64 sequences from rest, the same steps with each warm start
    ev = np.arange(n_eval)
    b = make(ev)
    out = {}
    zero = torch.zeros(n_eval, dof, dtype=torch.float64, device="cuda")
    for name in ("cold", "previous", "linear", "learned"):
        b.Reset()
        torch.cuda.synchronize()
        its, conv_all, t_guess = [], [], 0.0
        t0 = time.perf_counter()
        for n in range(1, steps_eval + 1):
            if name == "cold":
                torch.cuda.synchronize()
                it, res, conv = b.Step(T.BatchedDynamics.WARM_GIVEN, int(zero.data_ptr()))
            elif name == "previous":
                it, res, conv = b.Step(T.BatchedDynamics.WARM_PREVIOUS)
            elif name == "linear" or n == 1:
                it, res, conv = b.Step(T.BatchedDynamics.WARM_LINEAR)
            else:
                tg = time.perf_counter()
                v, vh, u = state(b, n_eval)
                g = sp.predict(v, vh, u, np.repeat(load_factors(n - 1), n_eval, 0), mats[ev])
                t_guess += time.perf_counter() - tg
                it, res, conv = b.Step(T.BatchedDynamics.WARM_GIVEN, int(g.data_ptr()))
            its.append(it)
            conv_all.append(conv)
            progress(f"config5: {name} step {n}: inner iterations mean {np.mean(it):.0f} max {np.max(it)}, "
                     f"converged {np.mean(conv):.2f}, {time.perf_counter() - t0:.1f} s")
        torch.cuda.synchronize()
        dt_run = time.perf_counter() - t0
        its = np.array(its)
        out[name] = {"steps_per_s": round(steps_eval / dt_run, 3),
                     "sequence_steps_per_s": round(n_eval * steps_eval / dt_run, 2),
                     "inner_iters_mean": float(its.mean()), "inner_iters_per_step": its.mean(1).round(1).tolist(),
                     "converged_fraction": float(np.mean(conv_all)), "seconds": round(dt_run, 3),
                     "guess_seconds": round(t_guess, 3)}
    b.Destroy()
    sp.destroy()
    el.Destroy()
    base = out["previous"]["inner_iters_mean"]
    cold = out["cold"]["inner_iters_mean"]
    return {"workload": f"configuration 5: {n_eval} sequences, 100x10x10 TET10 (60,000 elements, 88,641 nodes), "
                        f"gravity + 50 sin(2 pi 5 t) N tip load, dt 1e-3, SyncedNesterov (momentum restart) per "
                        f"step to rel. residual {tol:g}, steps 1..{steps_eval} from rest with each warm start",
            "value": out["learned"]["sequence_steps_per_s"], "unit": "sequence-steps/s",
            "warm_starts": out,
            "iteration_ratio_cold_over_learned": round(cold / out["learned"]["inner_iters_mean"], 3),
            "iteration_ratio_previous_over_linear": round(base / out["linear"]["inner_iters_mean"], 3),
            "iteration_ratio_previous_over_learned": round(base / out["learned"]["inner_iters_mean"], 3),
            "iteration_ratio_linear_over_learned": round(out["linear"]["inner_iters_mean"] /
                                                         out["learned"]["inner_iters_mean"], 3),
            "training": {"sequences": n_train, "steps": steps_train, "samples": n_train * (steps_train - 1),
                         "epochs": args.dyn_epochs, "final_loss": float(hist[-1]), "seconds": round(t_train, 2),
                         "train_inner_iters_mean": float(np.mean(it_train))},
            "step_size": {"alpha_min": float(alpha_all.min()), "alpha_max": float(alpha_all.max()),
                          "power_iteration_s": round(t_alpha, 2), "rho": rho_alm}}


def learned_leg(args, T):
    """Learned warm start on the fixed 40 x 8 x 8 TET10 cantilever (1.0 x 0.1 x
    0.1 m): 4096 solver-generated training cases (E log-uniform 1e6..1e8, nu
    U[0.2, 0.45], load direction on the sphere, magnitude U[1, 200] N), PCA to
    64 modes, a 6-256-256-256-64 GELU MLP trained on the GPU; 512 held-out
    cases solved warm and cold (batched) and cold one at a time (plain)."""
    import torch
    from tlfea_b200 import warmstart as W

    t_setup = time.perf_counter()
    fm = W.FixedMeshCases(40, 8, 8, 1.0, 0.1, 0.1, batch=512)
    fm.solver.SetPrecision(args.batch_precision)
    t_setup = time.perf_counter() - t_setup
    train = W.sample_cases(args.train_cases, seed=1)
    t0 = time.perf_counter()
    us, its = [], []
    for b0 in range(0, len(train), 512):
        u, it, res, stt = fm.solve(train[b0:b0 + 512], tol=1e-6)
        us.append(u)
        its.append(it)
    t_gen = time.perf_counter() - t0
    u_train = np.concatenate(us)
    ws = W.LearnedWarmStart(hidden=(256, 256, 256), k=64, max_batch=512, seed=0)
    t0 = time.perf_counter()
    hist = ws.fit(train, u_train, epochs=args.epochs, batch=512, lr=1e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    test = W.sample_cases(512, seed=12345)
    st = fm.solver.GetStream()
    # the held-out loads and materials are resident before each timed region
    fm._load(test)
    held = {}

    def cold():
        fm.solver.SetInitialGuess(None)
        fm.solver.Solve(1e-6, 200000)

    def warm():
        # network inference + PCA reconstruction (complete when predict returns),
        # then the warm-started batched solve
        held["guess"] = g = ws.predict(test)
        fm.solver.SetInitialGuess(int(g.data_ptr()))
        fm.solver.Solve(1e-6, 200000)

    cold()
    it_c, res_c, st_c = fm.solver.GetResults()
    u_c = fm.solver.RetrieveDisplacement(split=False).reshape(512, -1)
    warm()
    it_w, res_w, st_w = fm.solver.GetResults()
    g = held["guess"].cpu().numpy()
    guess_err = np.linalg.norm(g - u_c, axis=1) / np.linalg.norm(u_c, axis=1)
    # starting residual of the guess, ||f - K u0||_free / ||f|| (a cold start's is 1)
    kg = torch.empty_like(held["guess"])
    torch.cuda.synchronize()
    fm.solver.Apply(int(held["guess"].data_ptr()), int(kg.data_ptr()))
    F = fm.loads(test)
    r0 = F - kg.cpu().numpy()
    r0.reshape(512, -1, 3)[:, fm.fixed, :] = 0.0
    guess_res = np.linalg.norm(r0, axis=1) / np.linalg.norm(F, axis=1)
    # the Galerkin solution in the same learned basis (no network), for comparison
    gws = W.GalerkinWarmStart(ws.pca, fm)
    fm._load(test)

    def galerkin():
        held["gal"] = g2 = gws.predict(test)
        fm.solver.SetInitialGuess(int(g2.data_ptr()))
        fm.solver.Solve(1e-6, 200000)

    galerkin()
    it_g, res_g, st_g = fm.solver.GetResults()
    gal_err = np.linalg.norm(held["gal"].cpu().numpy() - u_c, axis=1) / np.linalg.norm(u_c, axis=1)
    reps = max(1, args.steps // 2)
    ms_cold = time_stream(torch, st, cold, reps)
    ms_warm = time_stream(torch, st, warm, reps)
    ms_gal = time_stream(torch, st, galerkin, reps)
    # plain: one case at a time through LinearStaticSolver, cold start
    k = min(args.plain_sample, 512)
    F = fm.loads(test[:k])
    tot, itp_all, el = 0.0, [], None
    for i in range(k):
        dt, itp, el = _plain_solve_time(T, fm.x, fm.y, fm.z, fm.conn, fm.fixed, F[i], test[i, 0], test[i, 1], 1e-6, el)
        tot += dt
        itp_all.append(itp)
    el.Destroy()
    plain = k / tot
    learned = 512 / (ms_warm / 1e3)
    ws.destroy()
    fm.destroy()
    return {"workload": "learned warm start, 40x8x8 TET10 cantilever (15,360 elements, 70,227 DOF), "
                        "512 held-out cases to 1e-6",
            "precision": args.batch_precision,
            "value": round(learned, 2), "unit": "solves/s",
            "learned_batched": {"value": round(learned, 2), "ms_per_batch": round(ms_warm, 3),
                                "iters_mean": float(np.mean(it_w)), "iters_max": int(np.max(it_w)),
                                "converged": int(np.sum(st_w == 0)), "max_rel_residual": float(np.max(res_w))},
            "cold_batched": {"value": round(512 / (ms_cold / 1e3), 2), "ms_per_batch": round(ms_cold, 3),
                             "iters_mean": float(np.mean(it_c)), "iters_max": int(np.max(it_c))},
            "plain_sequential": {"value": round(plain, 2), "sample": k, "iters_mean": float(np.mean(itp_all)),
                                 "path": "LinearStaticSolver per case (assembled K, CG graph), cold start"},
            "galerkin_batched": {"value": round(512 / (ms_gal / 1e3), 2), "ms_per_batch": round(ms_gal, 3),
                                 "iters_mean": float(np.mean(it_g)), "iters_max": int(np.max(it_g)),
                                 "converged": int(np.sum(st_g == 0)), "guess_rel_error_median": float(np.median(gal_err)),
                                 "speedup_vs_plain": round(512 / (ms_gal / 1e3) / plain, 2),
                                 "path": "Galerkin solution in the learned PCA basis (no network) as the warm start"},
            "speedup_learned_vs_plain": round(learned / plain, 2),
            "speedup_learned_vs_cold_batched": round(ms_cold / ms_warm, 2),
            "guess_rel_error_median": float(np.median(guess_err)),
            "guess_rel_residual_median": float(np.median(guess_res)),
            "training": {"cases": int(len(train)), "gen_s": round(t_gen, 2), "train_s": round(t_train, 2),
                         "epochs": args.epochs, "final_loss": float(hist[-1]), "pca_energy": ws.pca.energy
                         if hasattr(ws.pca, "energy") else None, "setup_s": round(t_setup, 2),
                         "train_iters_mean": float(np.mean(np.concatenate(its)))}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tlfea", choices=["tlfea", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-gpu-ref", action="store_true", help="skip the reference's own CUDA build leg")
    ap.add_argument("--kernel-reps", type=int, default=20)
    ap.add_argument("--operator", default="auto", choices=["auto", "assembled", "matrix-free"],
                    help="K operator of --kernels-only spmv")
    ap.add_argument("--batch-mode", default="auto", choices=["auto", "phased", "persistent"],
                    help="launch mode of --kernels-only batch")
    ap.add_argument("--gemm-size", type=int, default=8192, help="M = N = K of --kernels-only gemm")
    ap.add_argument("--cg-iters", type=int, default=120, help="iteration cap of --kernels-only cg")
    ap.add_argument("--kernels-only", choices=["force", "spmv", "cg", "batch", "batch-uneven", "steps", "mlp", "gemm", "nesterov"], default=None,
                    help="profiling case: set up, then launch only the named kernel a few times")
    ap.add_argument("--mesh", default=None, help="cells NXxNYxNZ (default 200x20x20)")
    ap.add_argument("--no-batch", action="store_true", help="skip the uneven-batch leg")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start leg")
    ap.add_argument("--no-dynamics", action="store_true", help="skip the time-stepping leg")
    ap.add_argument("--dyn-steps", type=int, default=50, help="implicit steps of the time-stepping leg")
    ap.add_argument("--no-config5", action="store_true", help="skip the configuration-5 batched sequences leg")
    ap.add_argument("--no-config2-more", action="store_true",
                    help="skip configuration 2's Nesterov and TET4 legs")
    ap.add_argument("--dyn-batch", type=int, default=64, help="sequences of the configuration-5 leg")
    ap.add_argument("--dyn-eval-steps", type=int, default=3, help="steps per warm start in the configuration-5 leg")
    ap.add_argument("--dyn-train-steps", type=int, default=8, help="training steps of the step predictor")
    ap.add_argument("--dyn-epochs", type=int, default=400, help="training epochs of the step predictor")
    ap.add_argument("--batch-size", type=int, default=512)
    ap.add_argument("--batch-precision", default="fp64", choices=["fp64", "fp32"],
                    help="element work of the batched solves (the CG and its stop test stay FP64)")
    ap.add_argument("--plain-sample", type=int, default=48, help="single-instance solves timed for the plain path")
    ap.add_argument("--train-cases", type=int, default=4096)
    ap.add_argument("--epochs", type=int, default=1500)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.mesh:
        CFG["nx"], CFG["ny"], CFG["nz"] = (int(v) for v in args.mesh.lower().split("x"))
    if args.kernels_only:
        return kernels_only(args)

    import torch
    import tlfea_b200 as T

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    cfg = dict(CFG)
    x, y, z, conn, fixed, f = build_mesh(cfg)
    N, E = len(x), conn.shape[0]
    el = setup_element(T, cfg, x, y, z, conn, fixed, f)
    el.CalcMassMatrix()
    solver = T.LinearStaticSolver(el, cfg["tol"], 1000000)
    stream = el.GetStream()

    def step():
        el.ResetPositions()
        solver.Solve()

    for _ in range(args.warmup):
        step()
    iters = solver.GetLastIterCount()
    resid = solver.GetLastResidual()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = T.launch_count()
    with ClockSampler(local) as clk:
        ms = time_stream(torch, stream, step, args.steps)
    launches = T.launch_count() - l0
    t_total = max_over_ranks(dist, ms * args.steps / 1e3, "cuda")
    value = whole_job_rate(world, args.steps, t_total)

    # opt-in block-Jacobi preconditioned CG on the same workload (not the headline:
    # the reference's method is the unpreconditioned CG above)
    solver.SetPreconditioner("block_jacobi")
    step()
    pcg_iters = solver.GetLastIterCount()
    ms_pcg = time_stream(torch, stream, step, max(1, args.steps // 2))
    pcg = {"value": round(1e3 / ms_pcg, 4), "unit": "solves/s", "ms_per_step": round(ms_pcg, 3),
           "cg_iters_per_solve": pcg_iters, "final_rel_residual": solver.GetLastResidual(),
           "preconditioner": "block Jacobi (3x3 node diagonal blocks)"}
    hbm, peak_kind = peaks()
    xin = torch.randn(3 * N, dtype=torch.float64, device="cuda")
    yout = torch.empty_like(xin)
    torch.cuda.synchronize()
    # the assembled K of the last (preconditioned) solve: its SpMV, and the plain CG on it
    el.SetBlocking(False)
    for _ in range(3):
        solver.Apply(xin.data_ptr(), yout.data_ptr())
    ms_spmv = time_stream(torch, stream, lambda: solver.Apply(xin.data_ptr(), yout.data_ptr()), args.kernel_reps)
    el.SetBlocking(True)
    solver.SetPreconditioner("none")
    off_m, cols_m, _ = el.RetrieveMassCSRToCPU()
    nnzb = len(cols_m)
    b_spmv = spmv_bytes(N, nnzb)
    ach_s = b_spmv / (ms_spmv / 1e3) / 1e9
    solver.SetOperator("assembled")
    step()
    ms_asm = time_stream(torch, stream, step, 1)
    asm_iters = solver.GetLastIterCount()
    solver.SetOperator("auto")
    assembled = {"value": round(1e3 / ms_asm, 4), "unit": "solves/s", "ms_per_step": round(ms_asm, 3),
                 "cg_iters_per_solve": asm_iters,
                 "spmv": {"kernel": "k_cg_spmv_dot", "bound": "hbm", "achieved": round(ach_s, 1), "peak": hbm,
                          "unit": "GB/s", "frac": round(ach_s / hbm, 4), "algorithmic_bytes": int(b_spmv),
                          "format": "row-planar 3x3 node blocks", "ms": round(ms_spmv, 4),
                          "traffic": int(SPMV_TRAFFIC_RATIO * b_spmv)},
                 "path": "the reference's operator: K assembled (3x3 node blocks) once per solve, SpMV per iteration"}

    # e2e through the public API with host buffers
    def e2e_step():
        el.SetExternalForce(f)
        el.UpdatePositions(x, y, z)
        solver.Solve()
        return el.RetrievePositionToCPU()

    e2e_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    t_e2e = max_over_ranks(dist, time.perf_counter() - t0, "cuda")
    e2e = {"value": whole_job_rate(world, args.steps, t_e2e), "unit": "solves/s", "h2d_bytes_per_step": 6 * N * 8,
           "d2h_bytes_per_step": 3 * N * 8}

    # dominant kernel: the matrix-free K p of the CG (tile kernel + shared-node combine
    # with p.q), timed back to back on the element stream at the last solve's positions
    el.SetBlocking(False)
    for _ in range(3):
        solver.Apply(xin.data_ptr(), yout.data_ptr())
    ms_mf = time_stream(torch, stream, lambda: solver.Apply(xin.data_ptr(), yout.data_ptr()), args.kernel_reps)
    b_mf = mf_apply_bytes(E, N, 10, 5)
    ach = b_mf / (ms_mf / 1e3) / 1e9
    roofline = {"kernel": "k_mf_gather + k_mf_geo + k_mf_combine_dot", "bound": "hbm", "achieved": round(ach, 1), "peak": hbm,
                "unit": "GB/s", "frac": round(ach / hbm, 4), "peak_kind": peak_kind, "algorithmic_bytes": int(b_mf),
                "format": "matrix-free SVK tangent: per QP J^-1, dV and the solve's F, S (FP64), p per tile",
                "ms": round(ms_mf, 4), "traffic": int(MF_TRAFFIC_RATIO * b_mf),
                "fp64_tflops": round(mf_apply_flops(E, 5) / (ms_mf / 1e3) / 1e12, 2)}
    # fused element force, FP32 and FP64
    ef = {}
    f_by_prec = {}
    for prec, s in (("fp32", 4), ("fp64", 8)):
        el.SetForcePrecision(prec)
        for _ in range(3):
            el.ComputeInternalForce()
        ms_f = time_stream(torch, stream, el.ComputeInternalForce, args.kernel_reps)
        f_by_prec[prec] = el.RetrieveInternalForceToCPU()
        b = elem_force_bytes(E, N, 10, 5, s)
        a = b / (ms_f / 1e3) / 1e9
        ef[prec] = {"kernel": "k_tile_force+k_combine", "bound": "hbm", "achieved": round(a, 1), "peak": hbm,
                    "unit": "GB/s", "frac": round(a / hbm, 4), "algorithmic_bytes": int(b), "ms": round(ms_f, 4),
                    "traffic": int(FORCE_TRAFFIC_RATIO[prec] * b)}
    # FP32 force error against the FP64 force at the same (deformed) positions
    ef["fp32"]["rel_error_vs_fp64"] = float(np.linalg.norm(f_by_prec["fp32"] - f_by_prec["fp64"]) /
                                            np.linalg.norm(f_by_prec["fp64"]))
    # the same contract with the persistent producer/consumer pipeline kernel
    el.SetLaunchConfig("pipeline")
    for prec, s in (("fp32", 4), ("fp64", 8)):
        el.SetForcePrecision(prec)
        for _ in range(3):
            el.ComputeInternalForce()
        ms_f = time_stream(torch, stream, el.ComputeInternalForce, args.kernel_reps)
        b = elem_force_bytes(E, N, 10, 5, s)
        a = b / (ms_f / 1e3) / 1e9
        ef["pipeline_" + prec] = {"kernel": "k_force_pipe+k_combine", "bound": "hbm", "achieved": round(a, 1),
                                  "peak": hbm, "unit": "GB/s", "frac": round(a / hbm, 4), "algorithmic_bytes": int(b),
                                  "ms": round(ms_f, 4)}
    # the same forces from the compact geometry stream (J^-1 and dV per QP)
    el.SetLaunchConfig("compact")
    for prec, s in (("fp32", 4), ("fp64", 8)):
        el.SetForcePrecision(prec)
        for _ in range(3):
            el.ComputeInternalForce()
        ms_f = time_stream(torch, stream, el.ComputeInternalForce, args.kernel_reps)
        b = elem_force_bytes_compact(E, N, 10, 5, s)
        a = b / (ms_f / 1e3) / 1e9
        ef["compact_" + prec] = {"kernel": "k_tile_force_geo+k_combine", "achieved": round(a, 1), "peak": hbm,
                                 "unit": "GB/s", "frac": round(a / hbm, 4), "algorithmic_bytes": int(b),
                                 "ms": round(ms_f, 4),
                                 "speedup_vs_gradient_stream": round(ef[prec]["ms"] / ms_f, 3)}
    el.SetLaunchConfig("tma")
    # the same evaluations with the tile-ordered node record rebuilt every time (as after
    # every change of positions): once a caller holds the positions' device pointer the
    # element can no longer tell, and refreshes before each evaluation
    el.GetX12DevicePtr()
    for prec in ("fp32", "fp64"):
        el.SetForcePrecision(prec)
        for _ in range(3):
            el.ComputeInternalForce()
        ef[prec]["ms_with_record_refresh"] = round(time_stream(torch, stream, el.ComputeInternalForce,
                                                               args.kernel_reps), 4)
    el.SetForcePrecision("fp64")
    el.SetBlocking(True)

    out = {"metric": METRIC, "value": round(value, 4), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(t_total * 1e3 / args.steps, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": WORKLOAD, "elements": E, "nodes": N,
                      "dof": 3 * N, "cg_iters_per_solve": iters, "final_rel_residual": resid,
                      "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (K 1.35 GB)"},
           "e2e": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in e2e.items()},
           "roofline": roofline, "elem_force": ef, "gpu_launches": int(launches), "clocks": clk.summary(),
           "pcg": pcg, "assembled_operator": assembled}
    el.Destroy()
    if not args.no_config2_more:
        out["config2_more"] = config2_more_legs(args, T, cfg)
    if not args.no_batch:
        out["batched"] = batched_leg(args, T)
    if not args.no_learned:
        out["learned"] = learned_leg(args, T)
    if not args.no_dynamics:
        out["dynamics"] = dynamics_leg(args, T)
    if not args.no_config5:
        out["config5"] = config5_leg(args, T)
    if rank == 0 and world == 1 and not args.no_gpu_ref:
        from oracle import ref_lib as R

        if R.available():
            g = gpu_reference_leg(cfg, x, y, z, conn, fixed, f, steps=2, warmup=1)
            g["speedup_value_vs_reference"] = round(out["value"] / g["value"], 3)
            g["speedup_e2e_vs_reference"] = round(out["e2e"]["value"] / g["value"], 3)
            g["speedup_elem_force_fp64"] = round(g["elem_force_fp64"]["ms"] / ef["fp64"]["ms"], 3)
            out["gpu_reference"] = g
    if rank == 0 and world == 1 and not args.no_cpu:
        src = f"this library's CG on this workload in this run ({iters} iterations)"
        out["cpu_baseline"] = cpu_sample(x, y, z, conn, fixed, f, cfg, iters, src)
        out["cpu_baseline"]["full_solve"] = cpu_full_solve()
    if rank == 0:
        print(json.dumps(out))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
