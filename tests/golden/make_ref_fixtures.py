"""Generate the reference-run fixtures ``tests/golden/ref_*.npz`` on a CUDA GPU.

Runs the reference's own CUDA build (``oracle/_ref/libtlfea_ref.so``, built from the
reference's unchanged sources by ``oracle/build_ref.py``) on the cases of ``ref_cases.py``
and stores what it returns:

* every case: ``CalcP`` + ``CalcInternalForce`` on a fresh ``Setup`` at seeded perturbed
  positions (FEAT10Data.cu:287-323), ``LinearStaticSolver::Solve`` stopped after 25 CG
  iterations (max_iter = 25) and run to its tolerance (LinearStaticSolver.cu:590-603),
  with the iteration counts and residuals;
* small cases (cube, configuration 1): the reference gradients and detJ
  (FEAT10Data.cu:92-198, FEAT4Data.cu:98-195), the mass CSR (FEAT10Data.cu:341-417), P,
  the constraint vector and the J / J^T CSR (FEAT10Data.cu:420-562, FEAT10DataFunc.cuh:
  470-481), the stiffness CSR with Dirichlet rows and columns applied, and trajectories of
  SyncedNesterov (SyncedNesterov.cu:97-414), SyncedAdamW and SyncedAdamWNocoop at fixed
  iteration counts and with the reference examples' parameters;
* mid cases (configuration 4): full force and displacement vectors, mass row sums;
* large cases (configuration 2): norms, 16 seeded projections and a 2048-entry sample of
  each long vector (``ref_cases.summary``).

The reference's Nesterov kernel leaves DOFs beyond its co-residency-limited grid untouched
(SyncedNesterov.cu:391-397) and its cooperative AdamW refuses such sizes, so the first-order
solvers run only on the small cases.

Usage (on a GPU box): ``python tests/golden/make_ref_fixtures.py --out DIR [--cases a,b]``.
Also writes ``DIR/ref_timings.json`` with the reference's wall times per call.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

import ref_cases as RC  # noqa: E402
from oracle import ref_lib as R  # noqa: E402


def _el(c, x=None, y=None, z=None, fixed=None, f=None, **kw):
    return R.RefElement(c["x"] if x is None else x, c["y"] if y is None else y, c["z"] if z is None else z,
                        c["conn"], c["E"], c["nu"], c["rho"], c["fixed"] if fixed is None else fixed,
                        c["f"] if f is None else f, **kw)


def run_case(name: str, timings: dict) -> dict:
    c = RC.case(name)
    small, large = name in RC.SMALL, name in RC.LARGE
    out: dict = {}
    t = {}
    # element arrays and the force at a perturbed state (fresh Setup: CalcInternalForce accumulates)
    el = _el(c, with_mass=not large)
    if small:
        g, dj = el.grad()
        out["grad"], out["detj"] = g, dj
        out["mass_off"], out["mass_col"], out["mass_val"] = el.mass()
    elif not large:
        _, dj = el.grad()
        off, _, val = el.mass()
        out["detj_sum"] = np.array([dj.sum()])
        out["mass_rowsum"] = np.add.reduceat(val, off[:-1]) if len(val) else np.zeros(len(off) - 1)
        out["mass_nnz"] = np.array([len(val)])
    xp, yp, zp = RC.perturbed(c)
    el.update_positions(xp, yp, zp)
    P = el.calc_p(want=small)
    f_int = el.calc_internal_force()
    if small:
        out["P"] = P
        out["constraint"] = el.constraint()
        (jo, jc, jv), (to, tc, tv) = el.constraint_csr()
        out.update(j_off=jo, j_col=jc, j_val=jv, jt_off=to, jt_col=tc, jt_val=tv)
    if large:
        s = RC.summary(f_int)
        out.update(f_int_norm=np.array([s["norm"]]), f_int_proj=s["proj"], f_int_sample=s["sample"])
        t["force_ms"] = el.time_force(5)
    else:
        out["f_int"] = f_int
        t["force_ms"] = el.time_force(20)
    el.destroy()

    # linear static: 25 CG iterations, then the full solve
    tol = 1e-6 if large else 1e-10
    for tag, max_iter in (("cg25", 25), ("cg", 200000)):
        el = _el(c, with_mass=False)
        ls = R.RefLinearStatic(el, tol, max_iter)
        it, res, ms = ls.solve()
        x, y, z = el.positions()
        u = np.stack([x - c["x"], y - c["y"], z - c["z"]], 1).ravel()
        out[f"{tag}_iters"], out[f"{tag}_res"] = np.array([it]), np.array([res])
        t[f"{tag}_ms"], t[f"{tag}_iters"] = ms, it
        if large:
            s = RC.summary(u)
            out.update({f"u_{tag}_norm": np.array([s["norm"]]), f"u_{tag}_proj": s["proj"],
                        f"u_{tag}_sample": s["sample"]})
        else:
            out[f"u_{tag}"] = u
        if small and tag == "cg":
            out["K_off"], out["K_col"], out["K_val"] = ls.stiffness()
        ls.destroy()
        el.destroy()

    if small:
        runs = [("nes_fixed", "nesterov", RC.NESTEROV_FIXED, 3, None)]
        if name == "cube_t10":
            runs += [("nes_ref", "nesterov", RC.NESTEROV_REF, 5, None),
                     ("adamw_ref", "adamw", RC.ADAMW_REF, 3, None),
                     ("nocoop_ref", "nocoop", RC.ADAMW_REF, 3, None)]
        else:
            gen = RC.generic_load(c)
            runs += [("adamw_fixed", "adamw", RC.ADAMW_FIXED, 2, gen),
                     ("nocoop_fixed", "nocoop", RC.ADAMW_FIXED, 2, gen)]
            if name == "cfg1_t10":
                runs.append(("nes_damped", "nesterov", RC.NESTEROV_FIXED, 2, "damped"))
        for tag, kind, params, steps, load in runs:
            kw = {}
            fixed, f = c["fixed"], c["f"]
            if load == "damped":
                kw = dict(eta=0.0, lamd=0.1)  # examples/beam_simulation.cc:203
            elif load is not None:
                fixed, f = load
            el = _el(c, fixed=fixed, f=f, **kw)
            if kind == "nesterov":
                s = R.RefNesterov(el, *params)
            else:
                s = R.RefAdamW(el, params, nocoop=(kind == "nocoop"))
            pos = []
            ms = 0.0
            for _ in range(steps):
                ms += s.steps(1)
                x, y, z = el.positions()
                pos.append(np.stack([x, y, z]))
            out[f"{tag}_pos"] = np.stack(pos)
            out[f"{tag}_v"] = s.velocity()
            t[f"{tag}_ms"] = ms
            s.destroy()
            el.destroy()
    timings[name] = t
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, required=True)
    ap.add_argument("--cases", default=",".join(RC.ALL))
    a = ap.parse_args()
    a.out.mkdir(parents=True, exist_ok=True)
    timings: dict = {}
    for name in a.cases.split(","):
        t0 = time.time()
        out = run_case(name, timings)
        np.savez_compressed(a.out / f"ref_{name}.npz", **out)
        print(f"{name}: {len(out)} arrays, {time.time() - t0:.1f} s", flush=True)
    (a.out / "ref_timings.json").write_text(json.dumps(timings, indent=1))


if __name__ == "__main__":
    main()
