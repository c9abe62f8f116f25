"""The allocation-free internal-force entry point
(tlfea_element_compute_internal_force_noalloc) against the regular one.

It serves callers that may not allocate device memory once running (a host
that owns all GPU memory through its own pool, or a time-critical loop that
cannot afford an allocation's device-wide synchronisation): its scratch lives
in a static device array, and the caller provides the output buffer.  The test
calls it through the C ABI twice in a row (the array keeps the previous
call's contents) and compares each result with the regular entry point's at the
FP64 parity tolerance.  It runs last so a stop-at-first-failure run has run
every other test first, and it works alone in a fresh process too."""
import ctypes as C

import numpy as np
import pytest

from tlfea_b200 import _capi

from .helpers import box, make_element, perturb, rel

pytestmark = pytest.mark.gpu
TOL64 = 1e-10


@pytest.mark.parametrize("order", [10, 4])
def test_noalloc_force_matches_regular_entry_point(order):
    import torch

    x, y, z, conn = box(24, 4, 4, order)
    el = make_element(x, y, z, conn, mass=False)
    out = torch.full((3 * len(x),), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for call, seed in enumerate((7, 8)):
        el.UpdatePositions(*perturb(x, y, z, 1e-3, seed))
        el.ComputeInternalForce()
        f_ref = el.RetrieveInternalForceToCPU()
        _capi.call("tlfea_element_compute_internal_force_noalloc", el._handle(), None, C.c_void_p(out.data_ptr()))
        torch.cuda.synchronize()
        f = out.cpu().numpy()
        assert np.isfinite(f).all(), f"call {call}"
        assert rel(f, f_ref) < TOL64, f"call {call}"
    el.Destroy()


def test_noalloc_refuses_fp32_force_mode():
    import torch

    from tlfea_b200 import TLFEAError

    x, y, z, conn = box(4, 2, 2, 10)
    el = make_element(x, y, z, conn, mass=False)
    el.SetForcePrecision("fp32")
    out = torch.zeros(3 * len(x), dtype=torch.float64, device="cuda")
    with pytest.raises(TLFEAError):
        _capi.call("tlfea_element_compute_internal_force_noalloc", el._handle(), None, C.c_void_p(out.data_ptr()))
    el.Destroy()
