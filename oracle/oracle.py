"""numpy binding of the CPU oracle (oracle/tlfea_oracle.c) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker / reported CPU baseline.  Layouts are the
reference's device layouts (see tlfea_oracle.h).  Parity status: pinned to fixtures
written by the reference's own CUDA build (tests/golden/ref_*.npz, checked by
tests/test_ref_fixtures.py) and by analytic known-answer tests (tests/test_oracle.py).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_lib = None

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def _cpu_has_avx2() -> bool:
    try:
        flags = Path("/proc/cpuinfo").read_text()
        return " avx2" in flags and " fma" in flags
    except OSError:
        return False


def lib():
    global _lib
    if _lib is None:
        cand = HERE / ("liborc.so" if _cpu_has_avx2() else "liborc_generic.so")
        if not cand.exists():
            raise ImportError(f"{cand} missing: build the oracle (python -m tlfea_b200.build)")
        _lib = C.CDLL(str(cand))
        L = _lib
        L.orc_node_pattern.restype = C.c_longlong
        L.orc_dof_pattern.restype = C.c_longlong
        L.orc_static_residual.restype = C.c_double
        L.orc_cg.restype = C.c_int
    return _lib


def d(a):
    return a.ctypes.data_as(_D) if a is not None else None


def i(a):
    return a.ctypes.data_as(_I) if a is not None else None


def f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


class mooney_rivlin:
    """Context: the oracle's stress routines use the Mooney-Rivlin law
    (MooneyRivlin.cuh:46-104) instead of SVK while it is active."""

    def __init__(self, mu10: float, mu01: float, kappa: float):
        self.prm = (float(mu10), float(mu01), float(kappa))

    def __enter__(self):
        lib().orc_set_material(1, C.c_double(self.prm[0]), C.c_double(self.prm[1]), C.c_double(self.prm[2]))
        return self

    def __exit__(self, *exc):
        lib().orc_set_material(0, C.c_double(0.0), C.c_double(0.0), C.c_double(0.0))
        return False


def colmajor(conn):
    """(E, NPE) -> reference layout conn[e + a*E]."""
    return i32(np.asarray(conn).T.ravel())


def box_mesh(nx, ny, nz, order=10, lx=1.0, ly=0.1, lz=0.1):
    nn, ne = C.c_int(), C.c_int()
    assert lib().orc_box_counts(nx, ny, nz, order, C.byref(nn), C.byref(ne)) == 0
    x, y, z = (np.zeros(nn.value) for _ in range(3))
    conn = np.zeros(ne.value * order, np.int32)
    lib().orc_box_mesh(nx, ny, nz, order, C.c_double(lx), C.c_double(ly), C.c_double(lz), d(x), d(y), d(z), i(conn))
    return x, y, z, conn.reshape(order, ne.value).T.copy()


def quadrature(npe):
    n = 5 if npe == 10 else 1
    q = [np.zeros(n) for _ in range(4)]
    (lib().orc_quadrature_t10 if npe == 10 else lib().orc_quadrature_t4)(*[d(a) for a in q])
    return q


def dndu_pre(x, y, z, conn):
    E, npe = conn.shape
    nqp = 5 if npe == 10 else 1
    cm = colmajor(conn)
    grad = np.zeros(E * nqp * npe * 3)
    detJ = np.zeros(E * nqp)
    x, y, z = f64(x), f64(y), f64(z)
    if npe == 10:
        qx, qy, qz, _ = quadrature(10)
        lib().orc_dndu_pre_t10(E, d(x), d(y), d(z), i(cm), d(qx), d(qy), d(qz), d(grad), d(detJ))
    else:
        lib().orc_dndu_pre_t4(E, d(x), d(y), d(z), i(cm), d(grad), d(detJ))
    return grad, detJ


def grad_to_array(grad, E, npe):
    """reference flat layout -> (E, QP, NPE, 3)."""
    nqp = 5 if npe == 10 else 1
    return grad.reshape(E, nqp, 3, npe).transpose(0, 1, 3, 2)


def calc_p(x, y, z, conn, grad, lam, mu, eta=0.0, lamd=0.0, v=None):
    E, npe = conn.shape
    nqp = 5 if npe == 10 else 1
    F = np.zeros(E * nqp * 9)
    P = np.zeros(E * nqp * 9)
    lib().orc_calc_p(npe, nqp, E, d(f64(x)), d(f64(y)), d(f64(z)), i(colmajor(conn)), d(grad), C.c_double(lam),
                     C.c_double(mu), C.c_double(eta), C.c_double(lamd), d(f64(v)) if v is not None else None, d(F),
                     d(P), None, None)
    return F, P


def internal_force_from_p(conn, grad, detJ, P, N, f_init=None):
    E, npe = conn.shape
    nqp = 5 if npe == 10 else 1
    qw = quadrature(npe)[3]
    f = f64(f_init).copy() if f_init is not None else np.zeros(3 * N)
    lib().orc_internal_force(npe, nqp, E, N, i(colmajor(conn)), d(grad), d(detJ), d(qw), d(f64(P)), d(f))
    return f


def force(x, y, z, conn, grad, detJ, lam, mu, eta=0.0, lamd=0.0, v=None):
    E, npe = conn.shape
    nqp = 5 if npe == 10 else 1
    N = len(x)
    qw = quadrature(npe)[3]
    f = np.zeros(3 * N)
    lib().orc_force(npe, nqp, E, N, d(f64(x)), d(f64(y)), d(f64(z)), i(colmajor(conn)), d(grad), d(detJ), d(qw),
                    C.c_double(lam), C.c_double(mu), C.c_double(eta), C.c_double(lamd),
                    d(f64(v)) if v is not None else None, d(f))
    return f


def node_pattern(conn, N):
    E, npe = conn.shape
    cm = colmajor(conn)
    nnz = lib().orc_node_pattern(npe, E, N, i(cm), None, None)
    off = np.zeros(N + 1, np.int32)
    cols = np.zeros(max(nnz, 1), np.int32)
    lib().orc_node_pattern(npe, E, N, i(cm), i(off), i(cols))
    return off, cols[:nnz]


def mass(conn, detJ, N, rho):
    E, npe = conn.shape
    nqp = 5 if npe == 10 else 1
    off, cols = node_pattern(conn, N)
    qx, qy, qz, qw = quadrature(npe)
    vals = np.zeros(max(len(cols), 1))
    lib().orc_mass_values(npe, nqp, E, N, i(colmajor(conn)), d(detJ), d(qx), d(qy), d(qz), d(qw), C.c_double(rho),
                          i(off), i(cols), d(vals))
    return off, cols, vals[:len(cols)]


def dof_pattern(noff, ncol, N):
    nnz = lib().orc_dof_pattern(N, i(noff), i(ncol), None, None)
    off = np.zeros(3 * N + 1, np.int32)
    cols = np.zeros(max(nnz, 1), np.int32)
    lib().orc_dof_pattern(N, i(noff), i(ncol), i(off), i(cols))
    return off, cols[:nnz]


def stiffness(x, y, z, conn, grad, detJ, lam, mu, eta=0.0, lamd=0.0, h=1.0):
    E, npe = conn.shape
    nqp = 5 if npe == 10 else 1
    N = len(x)
    noff, ncol = node_pattern(conn, N)
    off, cols = dof_pattern(noff, ncol, N)
    vals = np.zeros(max(len(cols), 1))
    qw = quadrature(npe)[3]
    lib().orc_stiffness_assemble(npe, nqp, E, N, d(f64(x)), d(f64(y)), d(f64(z)), i(colmajor(conn)), d(grad), d(detJ),
                                 d(qw), C.c_double(lam), C.c_double(mu), C.c_double(eta), C.c_double(lamd),
                                 C.c_double(h), i(off), i(cols), d(vals))
    return off, cols, vals[:len(cols)]


def apply_bcs(off, cols, vals, f, fixed):
    vals = f64(vals).copy()
    f = f64(f).copy()
    fx = i32(fixed)
    lib().orc_apply_bcs(len(off) - 1, len(fx), i(fx), i(off), i(cols), d(vals), d(f))
    return vals, f


def cg(off, cols, vals, f, tol, max_iter):
    n = len(off) - 1
    u = np.zeros(n)
    it, res = C.c_int(), C.c_double()
    rc = lib().orc_cg(n, i(off), i(cols), d(f64(vals)), d(f64(f)), d(u), C.c_double(tol), int(max_iter),
                      C.byref(it), C.byref(res))
    return u, it.value, res.value, rc


def spmv(off, cols, vals, xv):
    n = len(off) - 1
    y = np.zeros(n)
    lib().orc_spmv(n, i(off), i(cols), d(f64(vals)), d(f64(xv)), d(y))
    return y


# ------------------------------------------------------------------ solvers

class Problem(C.Structure):
    _fields_ = [("npe", C.c_int), ("nqp", C.c_int), ("E", C.c_int), ("N", C.c_int), ("conn", _I), ("grad", _D),
                ("detJ", _D), ("qw", _D), ("lambda_", C.c_double), ("mu", C.c_double), ("eta_d", C.c_double),
                ("lambda_d", C.c_double), ("m_off", _I), ("m_col", _I), ("m_val", _D), ("n_fixed", C.c_int),
                ("fixed", _I), ("x", _D), ("y", _D), ("z", _D), ("xj", _D), ("yj", _D), ("zj", _D), ("f_ext", _D)]


class NesterovParams(C.Structure):
    _fields_ = [("alpha", C.c_double), ("rho", C.c_double), ("inner_tol", C.c_double), ("outer_tol", C.c_double),
                ("max_outer", C.c_int), ("max_inner", C.c_int), ("time_step", C.c_double)]


class AdamWParams(C.Structure):
    _fields_ = [("lr", C.c_double), ("beta1", C.c_double), ("beta2", C.c_double), ("eps", C.c_double),
                ("weight_decay", C.c_double), ("lr_decay", C.c_double), ("inner_tol", C.c_double),
                ("outer_tol", C.c_double), ("rho", C.c_double), ("max_outer", C.c_int), ("max_inner", C.c_int),
                ("time_step", C.c_double), ("convergence_check_interval", C.c_int), ("inner_rtol", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("outer_iters", C.c_int), ("inner_iters_total", C.c_int), ("last_inner_iters", C.c_int),
                ("last_norm_g", C.c_double)]


class OracleModel:
    """Element + solver state for the Nesterov / AdamW restatements (the
    fields GPU_FEAT10_Data and the synced solvers hold)."""

    def __init__(self, x, y, z, conn, E_mod, nu, rho, fixed, f_ext, eta=0.0, lamd=0.0):
        self.conn = i32(conn)
        E, npe = self.conn.shape
        self.npe, self.nqp, self.E, self.N = npe, (5 if npe == 10 else 1), E, len(x)
        self.x, self.y, self.z = f64(x).copy(), f64(y).copy(), f64(z).copy()
        self.xj, self.yj, self.zj = self.x.copy(), self.y.copy(), self.z.copy()
        self.mu = E_mod / (2 * (1 + nu))
        self.lam = (E_mod * nu) / ((1 + nu) * (1 - 2 * nu))
        self.eta, self.lamd = eta, lamd
        self.grad, self.detJ = dndu_pre(self.x, self.y, self.z, self.conn)
        self.m_off, self.m_col, self.m_val = mass(self.conn, self.detJ, self.N, rho)
        self.fixed = i32(fixed)
        self.f_ext = f64(f_ext).copy()
        self.qw = quadrature(npe)[3]
        self.cm = colmajor(self.conn)
        n3, nc = 3 * self.N, 3 * len(self.fixed)
        self.v_guess, self.v_prev, self.lam_mult = np.zeros(n3), np.zeros(n3), np.zeros(max(nc, 1))

    def problem(self):
        p = Problem()
        p.npe, p.nqp, p.E, p.N = self.npe, self.nqp, self.E, self.N
        p.conn, p.grad, p.detJ, p.qw = i(self.cm), d(self.grad), d(self.detJ), d(self.qw)
        p.lambda_, p.mu, p.eta_d, p.lambda_d = self.lam, self.mu, self.eta, self.lamd
        p.m_off, p.m_col, p.m_val = i(self.m_off), i(self.m_col), d(self.m_val)
        p.n_fixed, p.fixed = len(self.fixed), i(self.fixed)
        p.x, p.y, p.z = d(self.x), d(self.y), d(self.z)
        p.xj, p.yj, p.zj = d(self.xj), d(self.yj), d(self.zj)
        p.f_ext = d(self.f_ext)
        return p

    def set_parameters(self):
        self.v_guess[:] = 0
        self.v_prev[:] = 0
        self.lam_mult[:] = 0

    def nesterov_solve(self, alpha, rho, inner_tol, outer_tol, max_outer, max_inner, time_step):
        prm = NesterovParams(alpha, rho, inner_tol, outer_tol, max_outer, max_inner, time_step)
        st = Stats()
        p = self.problem()
        lib().orc_nesterov_solve(C.byref(p), C.byref(prm), d(self.v_guess), d(self.v_prev), d(self.lam_mult),
                                 C.byref(st))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def _adamw(self, fn, params):
        prm = AdamWParams(*params)
        st = Stats()
        p = self.problem()
        fn(C.byref(p), C.byref(prm), d(self.v_guess), d(self.v_prev), d(self.lam_mult), C.byref(st))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def adamw_solve(self, *params):
        return self._adamw(lib().orc_adamw_solve, params)

    def adamw_nocoop_solve(self, *params):
        return self._adamw(lib().orc_adamw_nocoop_solve, params)

    def static_residual(self):
        p = self.problem()
        return lib().orc_static_residual(C.byref(p))
