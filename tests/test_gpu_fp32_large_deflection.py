"""FP32 force mode at large displacements.

The configuration-2 cantilever (200x20x20 cells, seeded tip load U[10, 1000] N) is
solved with the linear-static CG; at the solved positions the tip has moved by metres,
so the displacement is large compared with its variation across an element.  The FP32
force there (every force kernel) must match the FP64 oracle force at the same positions
to rel 1e-5, the FP32 tolerance of the parity contract, and the FP64 force to rel 1e-10.
"""
import numpy as np
import pytest

from oracle import oracle as O
import tlfea_b200 as T
from tlfea_b200 import mesh as M

from .helpers import E_MOD, NU, box, lame, make_element, rel

pytestmark = pytest.mark.gpu
TOL32, TOL64 = 1e-5, 1e-10


@pytest.mark.parametrize("order", [10, 4])
def test_fp32_force_at_solved_configuration2_deflection(order):
    x, y, z, conn = box(200, 20, 20, order)
    load = float(np.random.default_rng(0).uniform(10.0, 1000.0))
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -load))
    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f, mass=False)
    s = T.LinearStaticSolver(el, 1e-6, 100000)
    s.Solve()
    assert s.GetLastResidual() < 1e-6
    xs = el.RetrievePositionToCPU()
    tip = np.abs(xs[2] - z).max()
    assert tip > 0.1, tip  # the regime under test: displacements far above the element size
    lam, mu = lame(E_MOD, NU)
    g, dj = O.dndu_pre(x, y, z, conn)
    f_ref = O.force(*xs, conn, g, dj, lam, mu)
    del g
    el.ComputeInternalForce()
    assert rel(el.RetrieveInternalForceToCPU(), f_ref) < TOL64
    el.SetForcePrecision("fp32")
    for kernel in ("tma", "compact", "pipeline"):
        el.SetLaunchConfig(kernel)
        el.ComputeInternalForce()
        err = rel(el.RetrieveInternalForceToCPU(), f_ref)
        assert err < TOL32, (kernel, err)
    del s
    el.Destroy()
