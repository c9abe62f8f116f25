"""CPU tests of the host side: the C-ABI library loads and exports every
symbol include/*.h declares (no compute calls without a GPU), the Python
mirror of the reference API behaves like the reference on the host, and the
mesh readers parse the reference's fixtures."""
import re
from pathlib import Path

import numpy as np
import pytest

import tlfea_b200 as T
from tlfea_b200 import _capi
from tlfea_b200 import mesh as M

ROOT = Path(__file__).resolve().parent.parent


def _declared_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        syms |= set(re.findall(r"\b(tlfea_[a-z0-9_]+)\s*\(", h.read_text()))
    return syms


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    syms = _declared_symbols()
    assert len(syms) > 40
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_the_header():
    assert _declared_symbols() <= set(_capi.exported_symbols())


def test_no_device_is_reported_not_crashed():
    import ctypes as C

    lib = _capi.lib()
    h = C.c_void_p()
    st = lib.tlfea_element_create(_capi.TYPE_T10, 10, 10, C.byref(h))
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        assert st == _capi.OK
        lib.tlfea_element_destroy(h)
    else:
        assert st == _capi.NO_CUDA_DEVICE
        assert "CUDA" in _capi.last_error()


def test_invalid_arguments_rejected_without_device():
    import ctypes as C

    lib = _capi.lib()
    h = C.c_void_p()
    assert lib.tlfea_element_create(7, 10, 10, C.byref(h)) == _capi.INVALID_ARG
    assert lib.tlfea_element_create(_capi.TYPE_T4, 0, 10, C.byref(h)) == _capi.INVALID_ARG
    assert lib.tlfea_element_destroy(None) == _capi.INVALID_ARG
    assert lib.tlfea_solver_solve(None) == _capi.INVALID_ARG


def test_feasolver_registry_semantics():
    fea = T.FEASolver()
    a, b = object(), object()
    fea.AddElement("e", a)
    with pytest.raises(ValueError):
        fea.AddElement("e", b)
    with pytest.raises(ValueError):
        fea.AddElement("x", None)
    with pytest.raises(KeyError):
        fea.GetElement("nope")
    assert fea.GetElement("e") is a and fea.GetNumElements() == 1
    fea.AddSolver("s", b)
    with pytest.raises(ValueError):
        fea.AddSolver("s", a)
    with pytest.raises(KeyError):
        fea.GetSolver("t")
    assert fea.GetSolver("s") is b and fea.GetNumSolvers() == 1


def test_params_are_layout_compatible():
    import ctypes as C

    p = T.SyncedNesterovParams(1e-8, 1e14, 1e-6, 1e-6, 5, 300, 1e-3)
    c = _capi.NesterovParams(*(p.alpha, p.rho, p.inner_tol, p.outer_tol, p.max_outer, p.max_inner, p.time_step))
    assert C.sizeof(c) == 8 * 4 + 4 * 2 + 8
    a = T.SyncedAdamWParams(2e-4, 0.9, 0.999, 1e-8, 1e-4, 0.995, 1e-1, 1e-6, 1e14, 5, 300, 1e-3, 10, 0.0)
    ca = _capi.AdamWParams(*(getattr(a, f) for f, _ in _capi.AdamWParams._fields_))
    assert ca.convergence_check_interval == 10 and ca.inner_rtol == 0.0


def test_mesh_fixtures_parse():
    g = ROOT / "tests" / "golden"
    cube = np.load(g / "cube_t10.npz")
    assert cube["conn"].shape == (6, 10) and len(cube["x"]) == 27
    beam = np.load(g / "beam_t10.npz")
    assert beam["conn"].shape == (24, 10) and len(beam["x"]) == 81
    # every element uses distinct nodes
    for c in (cube["conn"], beam["conn"]):
        assert all(len(set(r)) == 10 for r in c)


def test_vtk_writer_roundtrip(tmp_path):
    x, y, z, conn = M.box_mesh(2, 1, 1, 10)
    p = tmp_path / "m.vtk"
    M.write_vtk(p, x, y, z, conn)
    txt = p.read_text().splitlines()
    assert txt[0] == "# vtk DataFile Version 3.0"
    assert f"POINTS {len(x)} float" in txt
    assert f"CELLS {conn.shape[0]} {conn.shape[0] * 11}" in txt
    assert txt[-1] == "24"


def test_cantilever_loads_sum():
    x, y, z, conn = M.box_mesh(10, 2, 2, 10)
    fixed, f, tip = M.cantilever_loads(x, y, z, (0.0, 0.0, -100.0))
    assert len(fixed) == 25 and len(tip) == 25
    assert f.reshape(-1, 3)[:, 2].sum() == pytest.approx(-100.0)


def test_random_beam_instances_follow_the_batch_distribution():
    """The seeded uneven-batch generator: sizes, material and load ranges,
    clamped x = 0 face and a tip load of the drawn magnitude."""
    from tlfea_b200 import mesh as M

    seen_nx, seen_ny = set(), set()
    for s in range(64):
        d = M.random_beam(s)
        assert 8 <= d["nx"] <= 64 and 2 <= d["ny"] <= 8
        seen_nx.add(d["nx"])
        seen_ny.add(d["ny"])
        assert 1e6 <= d["E"] <= 1e9 and 0.2 <= d["nu"] <= 0.45
        assert abs(np.linalg.norm(d["direction"]) - 1.0) < 1e-12
        ftot = d["f"].reshape(-1, 3).sum(0)
        assert np.allclose(ftot, d["magnitude"] * d["direction"], rtol=1e-12, atol=1e-12)
        nn, ne = M.box_counts(d["nx"], d["ny"], d["ny"])
        assert len(d["x"]) == nn and d["conn"].shape == (ne, 10)
        assert np.all(d["x"][d["fixed"]] == 0.0)
        assert abs(d["x"].max() - 10 * d["ny"] * 0.01) < 1e-12
        assert M.random_beam(s)["E"] == d["E"]  # seeded
    assert len(seen_nx) > 10 and len(seen_ny) > 3


def test_cpp_class_shim_builds_links_and_reports_no_device(tmp_path):
    """The C++ classes of include/tlfea/tlfea.hpp compile (-Wall -Wextra), link
    against the library and, without a GPU, end cleanly with the no-device code."""
    from . import cpp_driver as D

    exe = D.build(tmp_path)
    x, y, z, conn = M.box_mesh(4, 1, 1, 10)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -1.0))
    D.write_input(tmp_path / "in.bin", x, y, z, conn, fixed, f)
    import subprocess

    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True,
                       text=True, env={"CUDA_VISIBLE_DEVICES": ""})
    assert r.returncode == 3, r.stderr


def test_bench_byte_and_flop_models_match_the_documented_configuration2_figures():
    """The roofline's algorithmic bytes per unit (bench.py) at configuration 2
    (480,000 TET10 elements, 674,081 nodes): the matrix-free product's 531.6 MB, the
    fused force's 333.0 MB (FP32) / 646.8 MB (FP64), the compact stream's 131.4 MB /
    243.6 MB."""
    import bench as B

    E, N = 480000, 674081
    assert B.mf_apply_bytes(E, N, 10, 5) == 531555888
    assert B.elem_force_bytes(E, N, 10, 5, 4) == 332977944
    assert B.elem_force_bytes(E, N, 10, 5, 8) == 646755888
    assert B.elem_force_bytes_compact(E, N, 10, 5, 4) == 131377944
    assert B.elem_force_bytes_compact(E, N, 10, 5, 8) == 243555888
    # the FP64 operation count behind the roofline's fp64_tflops: 312 per element and QP
    assert B.mf_apply_flops(E, 5) == E * 5 * 312 * 2


def test_warm_start_cases_and_features_span_their_ranges():
    """The learned warm start's case sampler (E log-uniform, nu uniform, unit load
    direction, uniform magnitude) and its network features (each in [-1, 1])."""
    from tlfea_b200 import warmstart as W

    c = W.sample_cases(4096, seed=3)
    assert c.shape == (4096, 6)
    r = W.CaseRanges()
    assert r.E[0] <= c[:, 0].min() and c[:, 0].max() <= r.E[1]
    assert r.nu[0] <= c[:, 1].min() and c[:, 1].max() <= r.nu[1]
    assert np.allclose(np.linalg.norm(c[:, 2:5], axis=1), 1.0)
    assert r.magnitude[0] <= c[:, 5].min() and c[:, 5].max() <= r.magnitude[1]
    # log-uniform E: about half the cases below the geometric mean of the range
    assert abs(np.mean(c[:, 0] < np.sqrt(r.E[0] * r.E[1])) - 0.5) < 0.05
    f = W.features(c)
    assert f.dtype == np.float32 and f.shape == (4096, 6)
    assert f.min() >= -1.0 - 1e-6 and f.max() <= 1.0 + 1e-6
    assert np.array_equal(W.sample_cases(16, seed=3), W.sample_cases(16, seed=3))
