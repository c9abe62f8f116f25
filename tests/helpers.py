"""Shared set-up for the parity tests: the same seeded mesh and loads go to the
CUDA path (through the C ABI, via the reference-named classes) and to the
CPU oracle."""
from __future__ import annotations

import numpy as np

import tlfea_b200 as T
from tlfea_b200 import mesh as M
from tlfea_b200 import quadrature as Q

E_MOD, NU, RHO = 1e7, 0.3, 1000.0


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def box(nx, ny, nz, order=10, lx=1.0, ly=0.1, lz=0.1):
    return M.box_mesh(nx, ny, nz, order, lx, ly, lz)


def perturb(x, y, z, scale=1e-3, seed=0):
    r = np.random.default_rng(seed)
    return (x + scale * r.standard_normal(x.shape), y + scale * r.standard_normal(y.shape),
            z + scale * r.standard_normal(z.shape))


def make_element(x, y, z, conn, E_mod=E_MOD, nu=NU, rho=RHO, fixed=None, f_ext=None, eta=0.0, lamd=0.0,
                 precompute=True, mass=True):
    """Reference call order of examples/test_feat10_nesterov.cc:52-161."""
    npe = conn.shape[1]
    cls = T.GPU_FEAT10_Data if npe == 10 else T.GPU_FEAT4_Data
    el = cls(conn.shape[0], len(x))
    el.Initialize()
    if fixed is not None:
        el.SetNodalFixed(fixed)
    if f_ext is not None:
        el.SetExternalForce(f_ext)
    q = Q.t10() if npe == 10 else Q.t4()
    el.Setup(*q, x, y, z, conn)
    el.SetDensity(rho)
    el.SetDamping(eta, lamd)
    el.SetSVK(E_mod, nu)
    if precompute:
        el.CalcDnDuPre()
    if mass:
        el.CalcMassMatrix()
    if fixed is not None:
        el.CalcConstraintData()
        el.ConvertToCSR_ConstraintJacT()
    return el


def lame(E_mod=E_MOD, nu=NU):
    return (E_mod * nu) / ((1 + nu) * (1 - 2 * nu)), E_mod / (2 * (1 + nu))
