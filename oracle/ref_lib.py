"""ctypes binding of ``oracle/_ref/libtlfea_ref.so`` (test infrastructure).

The library is the reference's own CUDA build (its unchanged element and solver sources
compiled for sm_100a by ``oracle/build_ref.py``) with the C ABI of ``oracle/ref_harness.cu``.
It is used to generate the golden fixtures under ``tests/golden/`` on a GPU and to time the
reference's CUDA path beside this library's; the product never loads it.

``RefElement`` / ``RefLinearStatic`` / ``RefNesterov`` / ``RefAdamW`` follow the reference's
classes and call order (examples/test_feat10_nesterov.cc:52-199).  Every call raises
``RuntimeError`` when the reference reported a CUDA failure or a MOPHI_ERROR misuse.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libtlfea_ref.so"
_lib = None

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with oracle/build_ref.py")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        L.ref_element_create.restype = vp
        L.ref_element_create.argtypes = [C.c_int, C.c_int, C.c_int, _D, _D, _D, _I, _I, C.c_int, _D, C.c_double,
                                         C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                                         C.c_double, C.c_double, C.c_int]
        for name, args in {
            "ref_element_destroy": [vp],
            "ref_element_grad": [vp, _D, _D],
            "ref_element_mass_nnz": [vp],
            "ref_element_mass": [vp, _I, _I, _D],
            "ref_element_update_positions": [vp, _D, _D, _D],
            "ref_element_calc_p": [vp, _D],
            "ref_element_calc_internal_force": [vp, _D],
            "ref_element_positions": [vp, _D, _D, _D],
            "ref_element_constraint": [vp, _D],
            "ref_element_constraint_csr": [vp, _I, _I, _D, _I, _I, _D],
            "ref_linear_static_solve": [vp, _I, _D, _D],
            "ref_linear_static_k": [vp, _I, _I, _D],
            "ref_solver_steps": [vp, C.c_int, _D],
            "ref_solver_velocity": [vp, _D],
            "ref_solver_destroy": [vp],
            "ref_last_error": [C.c_char_p, C.c_int],
        }.items():
            getattr(L, name).restype = C.c_int
            getattr(L, name).argtypes = args
        L.ref_element_time_force.restype = C.c_double
        L.ref_element_time_force.argtypes = [vp, C.c_int]
        L.ref_linear_static_create.restype = vp
        L.ref_linear_static_create.argtypes = [vp, C.c_double, C.c_int]
        L.ref_nesterov_create.restype = vp
        L.ref_nesterov_create.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                          C.c_double]
        L.ref_adamw_create.restype = vp
        L.ref_adamw_create.argtypes = [vp, C.c_int] + [C.c_double] * 9 + [C.c_int, C.c_int, C.c_double, C.c_int,
                                                                        C.c_double]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_D) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_I) if a is not None else None


def _check(rc, what):
    if rc != 0:
        buf = C.create_string_buffer(256)
        lib().ref_last_error(buf, 256)
        raise RuntimeError(f"reference {what} failed (status {rc}) {buf.value.decode(errors='replace')}")


class RefElement:
    """GPU_FEAT10_Data / GPU_FEAT4_Data of the reference, set up as its examples do."""

    def __init__(self, x, y, z, conn, E_mod, nu, rho, fixed=None, f_ext=None, eta=0.0, lamd=0.0, mooney=None,
                 with_mass=True):
        self.x = np.ascontiguousarray(x, np.float64)
        self.y = np.ascontiguousarray(y, np.float64)
        self.z = np.ascontiguousarray(z, np.float64)
        self.conn = np.ascontiguousarray(conn, np.int32)
        self.E, self.npe = self.conn.shape
        self.N = len(self.x)
        self.nqp = 5 if self.npe == 10 else 1
        fx = None if fixed is None else np.ascontiguousarray(fixed, np.int32)
        fe = None if f_ext is None else np.ascontiguousarray(f_ext, np.float64)
        self.n_fixed = 0 if fx is None else len(fx)
        mat, m10, m01, kap = (0, 0.0, 0.0, 0.0) if mooney is None else (1, *mooney)
        self.h = lib().ref_element_create(self.npe, self.E, self.N, _d(self.x), _d(self.y), _d(self.z),
                                          _i(self.conn), _i(fx), self.n_fixed, _d(fe), E_mod, nu, rho, eta, lamd,
                                          mat, m10, m01, kap, int(with_mass))
        if not self.h:
            _check(2, "element set-up")

    def grad(self):
        g = np.empty(self.E * self.nqp * self.npe * 3)
        dj = np.empty(self.E * self.nqp)
        _check(lib().ref_element_grad(self.h, _d(g), _d(dj)), "grad")
        return g, dj

    def mass(self):
        nnz = lib().ref_element_mass_nnz(self.h)
        off = np.empty(self.N + 1, np.int32)
        col = np.empty(nnz, np.int32)
        val = np.empty(nnz)
        _check(lib().ref_element_mass(self.h, _i(off), _i(col), _d(val)), "mass")
        return off, col, val

    def update_positions(self, x, y, z):
        a, b, c = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
        _check(lib().ref_element_update_positions(self.h, _d(a), _d(b), _d(c)), "UpdatePositions")

    def calc_p(self, want=True):
        P = np.empty(self.E * self.nqp * 9) if want else None
        _check(lib().ref_element_calc_p(self.h, _d(P)), "CalcP")
        return P

    def calc_internal_force(self):
        f = np.empty(3 * self.N)
        _check(lib().ref_element_calc_internal_force(self.h, _d(f)), "CalcInternalForce")
        return f

    def positions(self):
        x, y, z = np.empty(self.N), np.empty(self.N), np.empty(self.N)
        _check(lib().ref_element_positions(self.h, _d(x), _d(y), _d(z)), "positions")
        return x, y, z

    def constraint(self):
        c = np.empty(3 * self.n_fixed)
        _check(lib().ref_element_constraint(self.h, _d(c)), "constraint")
        return c

    def constraint_csr(self):
        nc = 3 * self.n_fixed
        jo, jc, jv = np.empty(nc + 1, np.int32), np.empty(nc, np.int32), np.empty(nc)
        to, tc, tv = np.empty(3 * self.N + 1, np.int32), np.empty(nc, np.int32), np.empty(nc)
        _check(lib().ref_element_constraint_csr(self.h, _i(jo), _i(jc), _d(jv), _i(to), _i(tc), _d(tv)), "J CSR")
        return (jo, jc, jv), (to, tc, tv)

    def time_force(self, reps):
        ms = lib().ref_element_time_force(self.h, reps)
        if ms < 0:
            _check(2, "force timing")
        return ms

    def destroy(self):
        if self.h:
            lib().ref_element_destroy(self.h)
            self.h = None


class _RefSolver:
    def __init__(self, h, el):
        if not h:
            _check(2, "solver set-up")
        self.h, self.el = h, el

    def destroy(self):
        if self.h:
            lib().ref_solver_destroy(self.h)
            self.h = None


class RefLinearStatic(_RefSolver):
    def __init__(self, el: RefElement, tol=1e-10, max_iter=10000):
        super().__init__(lib().ref_linear_static_create(el.h, tol, max_iter), el)

    def solve(self):
        it, res, ms = C.c_int(0), C.c_double(0), C.c_double(0)
        _check(lib().ref_linear_static_solve(self.h, C.byref(it), C.byref(res), C.byref(ms)), "Solve")
        return it.value, res.value, ms.value

    def stiffness(self):
        nnz = lib().ref_linear_static_k(self.h, None, None, None)
        off = np.empty(3 * self.el.N + 1, np.int32)
        col, val = np.empty(nnz, np.int32), np.empty(nnz)
        _check(lib().ref_linear_static_k(self.h, _i(off), _i(col), _d(val)), "K")
        return off, col, val


class _RefFirstOrder(_RefSolver):
    def steps(self, n):
        ms = C.c_double(0)
        _check(lib().ref_solver_steps(self.h, n, C.byref(ms)), "Solve steps")
        return ms.value

    def velocity(self):
        v = np.empty(3 * self.el.N)
        _check(lib().ref_solver_velocity(self.h, _d(v)), "velocity")
        return v


class RefNesterov(_RefFirstOrder):
    """SyncedNesterovParams{alpha, rho, inner_tol, outer_tol, max_outer, max_inner, time_step}."""

    def __init__(self, el: RefElement, *params):
        a, rho, it, ot, mo, mi, dt = params
        super().__init__(lib().ref_nesterov_create(el.h, a, rho, it, ot, int(mo), int(mi), dt), el)


class RefAdamW(_RefFirstOrder):
    """SyncedAdamWParams field for field; nocoop selects SyncedAdamWNocoopSolver."""

    def __init__(self, el: RefElement, params, nocoop=False):
        lr, b1, b2, eps, wd, lrd, it, ot, rho, mo, mi, dt, ci, rt = params
        super().__init__(lib().ref_adamw_create(el.h, int(nocoop), lr, b1, b2, eps, wd, lrd, it, ot, rho, int(mo),
                                                int(mi), dt, int(ci), rt), el)
