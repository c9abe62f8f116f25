"""GPU parity at the headline size against the oracle: configuration 2's cantilever
(200x20x20 TET10 cells: 480,000 elements, 674,081 nodes, 2,022,243 DOF).

* K with the BCs applied, assembled on demand after a matrix-free solve, against the
  oracle's K (LinearStaticSolver.cu:196-306) -- the same sparsity, values to rounding;
* the matrix-free product K x (the CG's operator at this size) against the oracle's K x;
* the CG iterate after 25 iterations (tolerance 0), with the matrix-free operator and with
  the assembled one, against the oracle's CG (LinearStaticSolver.cu:469-565).

Bars: measured on the oracle, a 1e-14 relative perturbation of every K entry moves the
25-iteration iterate by 7e-14 (1e-13: 7e-13), so the iterate bars (1e-10 assembled,
1e-9 matrix-free, whose element-by-element sums round differently from a CSR row)
leave orders of magnitude of margin while still catching any wrong term."""
import numpy as np
import pytest
import scipy.sparse as sp

import tlfea_b200 as T
from oracle import oracle as O
from tlfea_b200 import mesh as M

from .helpers import box, lame, make_element, rel

pytestmark = pytest.mark.gpu
LAM, MU = lame()


def test_config2_stiffness_product_and_cg_iterates_match_oracle():
    import torch

    x, y, z, conn = box(200, 20, 20, 10)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -100.0))
    g, dj = O.dndu_pre(x, y, z, conn)
    off, cols, vals = O.stiffness(x, y, z, conn, g, dj, LAM, MU)
    kv, fb = O.apply_bcs(off, cols, vals, f, fixed)
    del vals, g, dj
    u_ref, it_ref, _, _ = O.cg(off, cols, kv, fb, 0.0, 25)
    assert it_ref == 25

    el = make_element(x, y, z, conn, fixed=fixed, f_ext=f)
    s = T.LinearStaticSolver(el, 0.0, 25)  # tolerance 0: exactly 25 iterations
    s.Solve()  # matrix-free: the default at 480,000 TET10 elements
    assert s.GetLastIterCount() == 25
    u_mf = (np.stack(el.RetrievePositionToCPU()) - np.stack([x, y, z])).T.ravel()
    assert rel(u_mf, u_ref) < 1e-9

    # the product at the solve's positions against the oracle's K
    n = 3 * len(x)
    xv = torch.tensor(np.random.default_rng(2).standard_normal(n), dtype=torch.float64, device="cuda")
    yv = torch.empty_like(xv)
    torch.cuda.synchronize()
    s.Apply(xv.data_ptr(), yv.data_ptr())
    torch.cuda.synchronize()
    K = sp.csr_matrix((kv, cols, off), shape=(n, n), copy=False)
    assert rel(yv.cpu().numpy(), K @ xv.cpu().numpy()) < 1e-12

    # K assembled on demand at the solve's positions
    o2, c2, v2 = s.RetrieveStiffnessCSRToCPU()
    assert np.array_equal(o2, off) and np.array_equal(c2, cols)
    assert rel(v2, kv) < 1e-12
    del o2, c2, v2

    # the reference's assembled operator, from the reference configuration again
    el.ResetPositions()
    s.SetOperator("assembled")
    s.Solve()
    assert s.GetLastIterCount() == 25
    u_as = (np.stack(el.RetrievePositionToCPU()) - np.stack([x, y, z])).T.ravel()
    assert rel(u_as, u_ref) < 1e-10
    del s
    el.Destroy()
