"""Python mirror of the reference's class API over the C ABI.

Names, argument meaning and call order follow the reference (Ruochun/TLFEA):
``GPU_FEAT10_Data`` / ``GPU_FEAT4_Data`` (src/elements/FEAT10Data.cuh,
FEAT4Data.cuh), ``SyncedNesterovSolver`` (src/solvers/SyncedNesterov.cuh),
``SyncedAdamWSolver`` (SyncedAdamW.cuh), ``SyncedAdamWNocoopSolver``
(SyncedAdamWNocoop.cuh), ``LinearStaticSolver`` (LinearStaticSolver.cuh) and
``FEASolver`` (src/FEASolver.h).  Eigen vectors and matrices become numpy
arrays; ``MatrixXi`` connectivity is an (E, NPE) int array; per-QP matrix
lists become (E, QP, ...) arrays.  Errors the reference reports with
MOPHI_ERROR raise ``TLFEAError``; FEASolver raises ValueError / KeyError where
the reference throws std::invalid_argument / std::out_of_range.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, astuple

import numpy as np

from . import _capi as capi
from ._capi import TLFEAError
from . import quadrature as Quadrature

# ElementType (ElementBase.h:22)
TYPE_3243, TYPE_3443, TYPE_T10, TYPE_T4 = 0, 1, 2, 3
# MaterialModel (MaterialModel.cuh:16-19)
MATERIAL_MODEL_SVK, MATERIAL_MODEL_MOONEY_RIVLIN = 0, 1


def _f64(a, n=None, name="array"):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
    if n is not None and a.size != n:
        raise TLFEAError(capi.SIZE_MISMATCH, name, f"expected {n} values, got {a.size}")
    return a


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


class ElementBase:
    """ElementBase (ElementBase.h:24-48)."""

    type: int = -1

    def get_n_beam(self) -> int:
        return self.n_elem

    def get_n_coef(self) -> int:
        return self.n_coef


class _TetData(ElementBase):
    NPE = 10
    NQP = 5
    TYPE = TYPE_T10

    def __init__(self, num_elements: int, num_nodes: int):
        self.n_elem = int(num_elements)
        self.n_coef = int(num_nodes)
        self.n_constraint = 0
        self.type = self.TYPE
        self._h = None
        self.d_data = None

    # -- lifecycle ---------------------------------------------------------
    def Initialize(self):
        h = C.c_void_p()
        capi.call("tlfea_element_create", self.TYPE, self.n_elem, self.n_coef, C.byref(h))
        self._h = h
        self.d_data = h

    def _handle(self):
        if self._h is None:
            raise TLFEAError(capi.NOT_SETUP, type(self).__name__, "Initialize() has not been called")
        return self._h

    def Destroy(self):
        if self._h is not None:
            capi.call("tlfea_element_destroy", self._h)
            self._h = None
            self.d_data = None

    def Setup(self, q_x, q_y, q_z, q_w, h_x12, h_y12, h_z12, element_connectivity):
        conn = np.asarray(element_connectivity, dtype=np.int32)
        if conn.shape != (self.n_elem, self.NPE):
            raise TLFEAError(capi.SIZE_MISMATCH, "Setup", f"connectivity must be ({self.n_elem}, {self.NPE})")
        conn_cm = np.ascontiguousarray(conn.T).ravel()
        qs = [_f64(q, self.NQP, "quadrature") for q in (q_x, q_y, q_z, q_w)]
        xs = [_f64(v, self.n_coef, "positions") for v in (h_x12, h_y12, h_z12)]
        capi.call("tlfea_element_setup", self._handle(), *[capi.dptr(q) for q in qs], self.NQP,
                  *[capi.dptr(v) for v in xs], capi.iptr(conn_cm))

    # -- material / loads ----------------------------------------------------
    def SetDensity(self, rho0: float):
        capi.call("tlfea_element_set_density", self._handle(), float(rho0))

    def SetDamping(self, eta_damp: float, lambda_damp: float):
        capi.call("tlfea_element_set_damping", self._handle(), float(eta_damp), float(lambda_damp))

    def SetSVK(self, E: float | None = None, nu: float | None = None):
        if E is None:
            capi.call("tlfea_element_set_svk_default", self._handle())
        else:
            capi.call("tlfea_element_set_svk", self._handle(), float(E), float(nu))

    def SetMooneyRivlin(self, mu10: float, mu01: float, kappa: float):
        capi.call("tlfea_element_set_mooney_rivlin", self._handle(), float(mu10), float(mu01), float(kappa))

    def SetExternalForce(self, h_f_ext):
        f = _f64(h_f_ext)
        capi.call("tlfea_element_set_external_force", self._handle(), capi.dptr(f), int(f.size))

    def AddGravity(self, gx: float, gy: float, gz: float):
        """New: f_ext += M g (consistent-mass row sums); after CalcMassMatrix."""
        capi.call("tlfea_element_add_gravity", self._handle(), float(gx), float(gy), float(gz))

    def SetNodalFixed(self, fixed_nodes):
        a = _i32(fixed_nodes)
        capi.call("tlfea_element_set_nodal_fixed", self._handle(), capi.iptr(a), int(a.size))
        self.n_constraint = 3 * int(a.size)

    def UpdateNodalFixed(self, fixed_nodes):
        a = _i32(fixed_nodes)
        capi.call("tlfea_element_update_nodal_fixed", self._handle(), capi.iptr(a), int(a.size))
        self.n_constraint = 3 * int(a.size)

    def UpdatePositions(self, h_x12, h_y12, h_z12):
        xs = [_f64(v) for v in (h_x12, h_y12, h_z12)]
        capi.call("tlfea_element_update_positions", self._handle(), *[capi.dptr(v) for v in xs], int(xs[0].size))

    def UpdateConstraintTargets(self, h_x12, h_y12, h_z12):
        xs = [_f64(v) for v in (h_x12, h_y12, h_z12)]
        capi.call("tlfea_element_update_constraint_targets", self._handle(), *[capi.dptr(v) for v in xs],
                  int(xs[0].size))

    # -- computation -----------------------------------------------------------
    def CalcDnDuPre(self):
        capi.call("tlfea_element_calc_dndu_pre", self._handle())

    def CalcMassMatrix(self):
        capi.call("tlfea_element_calc_mass_matrix", self._handle())

    def BuildMassCSRPattern(self):
        """The pattern is built by CalcMassMatrix (kept for API compatibility)."""

    def CalcP(self):
        capi.call("tlfea_element_calc_p", self._handle())

    def CalcInternalForce(self):
        capi.call("tlfea_element_calc_internal_force", self._handle())

    def CalcConstraintData(self):
        capi.call("tlfea_element_calc_constraint_data", self._handle())

    def ConvertToCSR_ConstraintJacT(self):
        capi.call("tlfea_element_build_constraint_jact_csr", self._handle())

    def ConvertToCSR_ConstraintJac(self):
        capi.call("tlfea_element_build_constraint_jac_csr", self._handle())

    BuildConstraintJacobianTransposeCSR = ConvertToCSR_ConstraintJacT
    BuildConstraintJacobianCSR = ConvertToCSR_ConstraintJac

    def ComputeInternalForce(self, d_v: int | None = None):
        """New fused hot path: f_int = internal force at the current positions
        (one pass, deterministic scatter).  d_v: optional device pointer to 3N
        interleaved velocities for the Kelvin-Voigt term."""
        capi.call("tlfea_element_compute_internal_force", self._handle(), C.c_void_p(d_v) if d_v else None)

    def SetForcePrecision(self, precision: str):
        p = {"fp64": capi.PRECISION_FP64, "fp32": capi.PRECISION_FP32}[precision]
        capi.call("tlfea_element_set_force_precision", self._handle(), p)

    FORCE_KERNELS = {"tma": 0, "direct": 1, "pipeline": 2, "compact": 3}

    def SetLaunchConfig(self, force_kernel="tma", grid_limit: int = 0):
        """New: the fused force kernel -- "tma" (gradient stream, bulk-copy double
        buffered), "direct", "pipeline" (persistent producer/consumer) or
        "compact" (J^-1 stream, gradients formed in registers)."""
        k = self.FORCE_KERNELS[force_kernel] if isinstance(force_kernel, str) else int(force_kernel)
        capi.call("tlfea_element_set_launch_config", self._handle(), k, int(grid_limit))

    # -- retrieval ---------------------------------------------------------------
    def RetrieveMassCSRToCPU(self):
        nnz = C.c_longlong()
        capi.call("tlfea_element_get_mass_nnz", self._handle(), C.byref(nnz))
        off = np.zeros(self.n_coef + 1, np.int32)
        cols = np.zeros(max(nnz.value, 1), np.int32)
        vals = np.zeros(max(nnz.value, 1), np.float64)
        capi.call("tlfea_element_retrieve_mass_csr", self._handle(), capi.iptr(off), capi.iptr(cols), capi.dptr(vals))
        return off, cols[:nnz.value], vals[:nnz.value]

    def RetrieveInternalForceToCPU(self):
        f = np.zeros(3 * self.n_coef)
        capi.call("tlfea_element_retrieve_internal_force", self._handle(), capi.dptr(f), f.size)
        return f

    def RetrieveExternalForceToCPU(self):
        f = np.zeros(3 * self.n_coef)
        capi.call("tlfea_element_retrieve_external_force", self._handle(), capi.dptr(f), f.size)
        return f

    def RetrievePositionToCPU(self):
        x, y, z = (np.zeros(self.n_coef) for _ in range(3))
        capi.call("tlfea_element_retrieve_positions", self._handle(), capi.dptr(x), capi.dptr(y), capi.dptr(z),
                  self.n_coef)
        return x, y, z

    def RetrievePFromFToCPU(self):
        """(E, QP, 3, 3) with P[e, q, i, j]."""
        P = np.zeros(self.n_elem * self.NQP * 9)
        capi.call("tlfea_element_retrieve_p", self._handle(), capi.dptr(P), P.size)
        return P.reshape(self.n_elem, self.NQP, 3, 3).transpose(0, 1, 3, 2).copy()

    def RetrieveDnDuPreToCPU(self):
        """(E, QP, NPE, 3) with grad_N[e, q, a, j] = dN_a/dx_j."""
        g = np.zeros(self.n_elem * self.NQP * self.NPE * 3)
        capi.call("tlfea_element_retrieve_dndu_pre", self._handle(), capi.dptr(g), g.size)
        return g.reshape(self.n_elem, self.NQP, 3, self.NPE).transpose(0, 1, 3, 2).copy()

    def RetrieveDetJToCPU(self):
        d = np.zeros(self.n_elem * self.NQP)
        capi.call("tlfea_element_retrieve_detj", self._handle(), capi.dptr(d), d.size)
        return d.reshape(self.n_elem, self.NQP)

    def RetrieveConnectivityToCPU(self):
        c = np.zeros(self.n_elem * self.NPE, np.int32)
        capi.call("tlfea_element_retrieve_connectivity", self._handle(), capi.iptr(c), c.size)
        return c.reshape(self.NPE, self.n_elem).T.copy()

    def RetrieveConstraintDataToCPU(self):
        c = np.zeros(self.n_constraint)
        if self.n_constraint:
            capi.call("tlfea_element_retrieve_constraint", self._handle(), capi.dptr(c), c.size)
        return c

    def RetrieveConstraintJacobianCSRToCPU(self, transpose: bool = False):
        """New: (offsets, columns, values) of J (or J^T) as built by
        ConvertToCSR_ConstraintJac(T) (FEAT10Data.cu:420-562)."""
        rows = 3 * self.n_coef if transpose else self.n_constraint
        off = np.zeros(rows + 1, np.int32)
        cols = np.zeros(max(self.n_constraint, 1), np.int32)
        vals = np.zeros(max(self.n_constraint, 1))
        capi.call("tlfea_element_retrieve_constraint_jac_csr", self._handle(), int(transpose), capi.iptr(off),
                  capi.iptr(cols), capi.dptr(vals))
        return off, cols[:self.n_constraint], vals[:self.n_constraint]

    def WriteOutputVTK(self, filename: str):
        capi.call("tlfea_element_write_vtk", self._handle(), str(filename).encode())

    def _ptr(self, k):
        """Device pointer k of (x, y, z, f_ext, f_int); only that one is requested (taking a
        position pointer makes the element rebuild its derived position records before
        every force evaluation, since the caller may write the positions directly)."""
        p = C.c_void_p()
        args = [None] * 5
        args[k] = C.byref(p)
        capi.call("tlfea_element_device_ptrs", self._handle(), *args)
        return p.value

    def GetX12DevicePtr(self):
        return self._ptr(0)

    def GetY12DevicePtr(self):
        return self._ptr(1)

    def GetZ12DevicePtr(self):
        return self._ptr(2)

    def GetExternalForceDevicePtr(self):
        return self._ptr(3)

    def GetInternalForceDevicePtr(self):
        return self._ptr(4)

    def SetBlocking(self, blocking: bool):
        """New: False makes compute calls return after enqueueing on GetStream()."""
        capi.call("tlfea_element_set_blocking", self._handle(), 1 if blocking else 0)

    def ResetPositions(self):
        """New: positions = the reference configuration of the last CalcDnDuPre (device copy)."""
        capi.call("tlfea_element_reset_positions", self._handle())

    def GetStream(self) -> int:
        s = C.c_void_p()
        capi.call("tlfea_element_get_stream", self._handle(), C.byref(s))
        return s.value or 0

    def get_n_elem(self):
        return self.n_elem

    def get_n_constraint(self):
        return self.n_constraint

    def __del__(self):
        try:
            self.Destroy()
        except Exception:
            pass


class GPU_FEAT10_Data(_TetData):
    """GPU_FEAT10_Data (FEAT10Data.cuh:22-810): 10-node tetrahedra, 5-point rule."""
    NPE, NQP, TYPE = 10, 5, TYPE_T10


class GPU_FEAT4_Data(_TetData):
    """GPU_FEAT4_Data (FEAT4Data.cuh:22-): 4-node tetrahedra, centroid rule."""
    NPE, NQP, TYPE = 4, 1, TYPE_T4


# ------------------------------------------------------------------- solvers

class SolverBase:
    """SolverBase (SolverBase.h:18-25)."""

    def Solve(self):
        raise NotImplementedError

    def SetParameters(self, params):
        raise NotImplementedError


@dataclass
class SyncedNesterovParams:
    """SyncedNesterovParams (SyncedNesterov.cuh:31-35), positional like the C++ brace init."""
    alpha: float
    rho: float
    inner_tol: float
    outer_tol: float
    max_outer: int
    max_inner: int
    time_step: float


@dataclass
class SyncedAdamWParams:
    """SyncedAdamWParams (SyncedAdamW.cuh:32-39)."""
    lr: float
    beta1: float
    beta2: float
    eps: float
    weight_decay: float
    lr_decay: float
    inner_tol: float
    outer_tol: float
    rho: float
    max_outer: int
    max_inner: int
    time_step: float
    convergence_check_interval: int
    inner_rtol: float = 0.0


SyncedAdamWNocoopParams = SyncedAdamWParams


class _FirstOrder(SolverBase):
    _CREATE = ""

    def __init__(self, data: _TetData, n_constraints: int):
        self.data = data
        self.n_coef = data.n_coef
        self.n_constraints = int(n_constraints)
        h = C.c_void_p()
        capi.call(self._CREATE, data._handle(), self.n_constraints, C.byref(h))
        self._h = h

    def Setup(self):
        capi.call("tlfea_solver_setup", self._h)

    def Solve(self):
        capi.call("tlfea_solver_solve", self._h)

    def GetVelocity(self):
        vg, vp = np.zeros(3 * self.n_coef), np.zeros(3 * self.n_coef)
        capi.call("tlfea_solver_get_velocity", self._h, capi.dptr(vg), capi.dptr(vp), vg.size)
        return vg, vp

    def SetVelocityGuess(self, v_guess, v_prev=None):
        vg = _f64(v_guess, 3 * self.n_coef)
        vp = _f64(v_prev, 3 * self.n_coef) if v_prev is not None else None
        capi.call("tlfea_solver_set_velocity", self._h, capi.dptr(vg), capi.dptr(vp) if vp is not None else None,
                  vg.size)

    def GetMultipliers(self):
        lam = np.zeros(self.n_constraints)
        if self.n_constraints:
            capi.call("tlfea_solver_get_multipliers", self._h, capi.dptr(lam), lam.size)
        return lam

    def GetStats(self) -> dict:
        st = capi.SolveStats()
        capi.call("tlfea_solver_get_stats", self._h, C.byref(st))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def SetRelativeResidualStop(self, rel_tol: float):
        """New: end Solve() once ||(f_int - f_ext)_free|| / ||f_ext|| < rel_tol
        (FP64, evaluated every inner iteration); 0 turns the rule off."""
        capi.call("tlfea_solver_set_stop_rule", self._h, float(rel_tol))

    def SetMode(self, mode: str = "auto"):
        """New: "phased" -- one kernel per phase, the loop state on the device, chunks of
        iterations replayed as CUDA graphs -- or "persistent" (the whole Solve() in one
        cooperative launch); "auto" (the default) takes the per-phase launches from
        200,000 nodes."""
        capi.call("tlfea_solver_set_mode", self._h, {"auto": 0, "persistent": 1, "phased": 2}[mode])

    def RunSteps(self, n_steps: int, f_var=None, amp: float = 1.0, omega: float = 0.0, phase: float = 0.0,
                 t0: float = 0.0):
        """New: n_steps calls of Solve() in one launch (one CUDA graph), the loop
        of examples/beam_simulation.cc:275-283.  With f_var, step k runs with
        f_ext = f_base + (amp * sin(omega * t_k + phase)) * f_var, where f_base is
        the external force set before the call and t_k = t0 + (k + 1) * time_step.
        Returns each step's total inner iterations."""
        n = int(n_steps)
        its = np.zeros(max(n, 1), dtype=np.int32)
        fv = _f64(f_var, 3 * self.n_coef) if f_var is not None else None
        capi.call("tlfea_solver_run_steps", self._h, n, float(t0), capi.dptr(fv) if fv is not None else None,
                  float(amp), float(omega), float(phase), capi.iptr(its))
        return its

    def __del__(self):
        try:
            if getattr(self, "_h", None) is not None:
                capi.call("tlfea_solver_destroy", self._h)
                self._h = None
        except Exception:
            pass


class SyncedNesterovSolver(_FirstOrder):
    """SyncedNesterovSolver (SyncedNesterov.cuh:39-322)."""
    _CREATE = "tlfea_nesterov_create"

    def SetParameters(self, params: SyncedNesterovParams):
        p = capi.NesterovParams(*astuple(params))
        capi.call("tlfea_solver_set_parameters", self._h, C.cast(C.byref(p), C.c_void_p))


class SyncedAdamWSolver(_FirstOrder):
    """SyncedAdamWSolver (SyncedAdamW.cuh:43-)."""
    _CREATE = "tlfea_adamw_create"

    def SetParameters(self, params: SyncedAdamWParams):
        p = capi.AdamWParams(*astuple(params))
        capi.call("tlfea_solver_set_parameters", self._h, C.cast(C.byref(p), C.c_void_p))


class SyncedAdamWNocoopSolver(SyncedAdamWSolver):
    """SyncedAdamWNocoopSolver (SyncedAdamWNocoop.cuh:25-)."""
    _CREATE = "tlfea_adamw_nocoop_create"


class LinearStaticSolver(SolverBase):
    """LinearStaticSolver<T>(data, tol, max_iter) (LinearStaticSolver.cuh:44-117)."""

    def __init__(self, data: _TetData, tol: float = 1e-10, max_iter: int = 10000):
        self.data = data
        h = C.c_void_p()
        capi.call("tlfea_linear_static_create", data._handle(), float(tol), int(max_iter), C.byref(h))
        self._h = h

    def Solve(self):
        capi.call("tlfea_solver_solve", self._h)

    def SetParameters(self, params=None):
        """No-op: parameters are set through the constructor."""

    def SetPreconditioner(self, kind: str = "none"):
        """New, opt-in: "block_jacobi" (3x3 node diagonal blocks) or "none" (the
        reference's unpreconditioned CG, the default)."""
        capi.call("tlfea_linear_static_set_preconditioner", self._h, {"none": 0, "block_jacobi": 1}[kind])

    def SetOperator(self, mode: str = "auto"):
        """New: "matrix-free" (TET10, SVK, no damping, no preconditioner), "assembled"
        (the reference's assembled K), or "auto" (the default: matrix-free from 100,000
        elements where it applies)."""
        capi.call("tlfea_linear_static_set_operator", self._h, {"auto": 0, "assembled": 1, "matrix-free": 2}[mode])

    def _last(self):
        it, res = C.c_int(), C.c_double()
        capi.call("tlfea_linear_static_last", self._h, C.byref(it), C.byref(res))
        return it.value, res.value

    def GetLastIterCount(self) -> int:
        return self._last()[0]

    def GetLastResidual(self) -> float:
        return self._last()[1]

    def Apply(self, d_x: int, d_y: int):
        """New: y = K x on device pointers (3N doubles each), the CG's SpMV kernel."""
        capi.call("tlfea_linear_static_apply", self._h, C.c_void_p(d_x), C.c_void_p(d_y))

    def RetrieveStiffnessCSRToCPU(self):
        """K (BCs applied) as 3N x 3N CSR (new; the reference keeps K private)."""
        nnz = C.c_longlong()
        capi.call("tlfea_linear_static_retrieve_k", self._h, C.byref(nnz), None, None, None)
        off = np.zeros(3 * self.data.n_coef + 1, np.int32)
        cols = np.zeros(max(nnz.value, 1), np.int32)
        vals = np.zeros(max(nnz.value, 1))
        capi.call("tlfea_linear_static_retrieve_k", self._h, C.byref(nnz), capi.iptr(off), capi.iptr(cols),
                  capi.dptr(vals))
        return off, cols[:nnz.value], vals[:nnz.value]

    def __del__(self):
        try:
            if getattr(self, "_h", None) is not None:
                capi.call("tlfea_solver_destroy", self._h)
                self._h = None
        except Exception:
            pass


LinearStaticSolverT10 = LinearStaticSolver
LinearStaticSolverT4 = LinearStaticSolver


class BatchedLinearStaticSolver:
    """New, no reference counterpart: many independent meshes solved by one
    persistent, graph-captured launch.

    Per instance the iteration is LinearStaticSolver's CG
    (LinearStaticSolver.cu:469-565) on the linear stiffness at the reference
    configuration, applied matrix-free; fixed DOFs are eliminated as
    apply_bcs_kernel does.  Stop rule: ||r|| / ||f_free|| < tol in FP64.

    meshes: list of (x, y, z, conn) with conn an (E_i, NPE) array of
    instance-local node ids.  Device pointers passed in must hold finished
    data: the library orders its own work on its own stream (GetStream) and
    does not wait for other streams.
    """

    def __init__(self, meshes, element_type: int = TYPE_T10, shared: bool = False):
        """shared=True: every entry of `meshes` is the same mesh (one tiling and
        gradient stream serve all instances; only material, fixed nodes and loads
        differ).  Pass the mesh once and the count: meshes=[mesh] * n."""
        if shared:
            self._init_shared(meshes[0], len(meshes), element_type)
            return
        if element_type not in (TYPE_T10, TYPE_T4):
            raise TLFEAError(capi.INVALID_ARG, "BatchedLinearStaticSolver", "element type must be TYPE_T10 or TYPE_T4")
        npe = 10 if element_type == TYPE_T10 else 4
        q = Quadrature.t10() if element_type == TYPE_T10 else Quadrature.t4()
        self.n_inst = len(meshes)
        nn = [len(m[0]) for m in meshes]
        ne = [np.asarray(m[3]).shape[0] for m in meshes]
        self.node_off = np.zeros(self.n_inst + 1, np.int32)
        self.elem_off = np.zeros(self.n_inst + 1, np.int32)
        self.node_off[1:] = np.cumsum(nn)
        self.elem_off[1:] = np.cumsum(ne)
        x = _f64(np.concatenate([m[0] for m in meshes]))
        y = _f64(np.concatenate([m[1] for m in meshes]))
        z = _f64(np.concatenate([m[2] for m in meshes]))
        conn = _i32(np.concatenate([np.asarray(m[3], dtype=np.int32).reshape(-1, npe) for m in meshes]))
        qx, qy, qz, qw = (_f64(a) for a in q)
        h = C.c_void_p()
        capi.call("tlfea_batch_create", int(element_type), self.n_inst, capi.iptr(self.node_off),
                  capi.iptr(self.elem_off), capi.dptr(qx), capi.dptr(qy), capi.dptr(qz), capi.dptr(qw), len(qw),
                  capi.dptr(x), capi.dptr(y), capi.dptr(z), capi.iptr(conn), C.byref(h))
        self._h = h
        self.n_nodes = int(self.node_off[-1])

    def _init_shared(self, mesh, n, element_type):
        if element_type not in (TYPE_T10, TYPE_T4):
            raise TLFEAError(capi.INVALID_ARG, "BatchedLinearStaticSolver", "element type must be TYPE_T10 or TYPE_T4")
        npe = 10 if element_type == TYPE_T10 else 4
        q = Quadrature.t10() if element_type == TYPE_T10 else Quadrature.t4()
        x, y, z, conn = _f64(mesh[0]), _f64(mesh[1]), _f64(mesh[2]), np.asarray(mesh[3], dtype=np.int32)
        nn, ne = len(x), conn.shape[0]
        self.n_inst = int(n)
        self.node_off = (np.arange(self.n_inst + 1) * nn).astype(np.int32)
        self.elem_off = (np.arange(self.n_inst + 1) * ne).astype(np.int32)
        qx, qy, qz, qw = (_f64(a) for a in q)
        c = _i32(conn.reshape(-1, npe))
        h = C.c_void_p()
        capi.call("tlfea_batch_create_shared", int(element_type), self.n_inst, nn, ne, capi.dptr(qx), capi.dptr(qy),
                  capi.dptr(qz), capi.dptr(qw), len(qw), capi.dptr(x), capi.dptr(y), capi.dptr(z), capi.iptr(c),
                  C.byref(h))
        self._h = h
        self.n_nodes = int(self.node_off[-1])

    def GetCounts(self) -> dict:
        a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        capi.call("tlfea_batch_get_counts", self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        return {"instances": a.value, "elements": b.value, "nodes": c.value, "tiles": d.value}

    def GetStream(self) -> int:
        s = C.c_void_p()
        capi.call("tlfea_batch_get_stream", self._h, C.byref(s))
        return s.value or 0

    def SetMaterial(self, E, nu):
        capi.call("tlfea_batch_set_material", self._h, capi.dptr(_f64(E, self.n_inst, "E")),
                  capi.dptr(_f64(nu, self.n_inst, "nu")))

    def SetNodalFixed(self, fixed_per_instance):
        """Fixed nodes, one array of instance-local ids per instance."""
        g = [np.asarray(f, dtype=np.int64) + int(self.node_off[i]) for i, f in enumerate(fixed_per_instance)]
        allf = _i32(np.concatenate(g) if g else np.zeros(0))
        capi.call("tlfea_batch_set_fixed", self._h, capi.iptr(allf) if allf.size else None, int(allf.size))

    def SetExternalForce(self, f):
        """f: concatenated 3 * n_nodes array, a list of per-instance arrays, or a device pointer (int)."""
        if isinstance(f, int):
            capi.call("tlfea_batch_set_external_force", self._h, C.c_void_p(f), 3 * self.n_nodes, 1)
            return
        if isinstance(f, (list, tuple)):
            f = np.concatenate([np.asarray(v, dtype=np.float64).ravel() for v in f])
        a = _f64(f, 3 * self.n_nodes, "f_ext")
        capi.call("tlfea_batch_set_external_force", self._h, a.ctypes.data_as(C.c_void_p), a.size, 0)

    def SetInitialGuess(self, u0=None):
        """Warm start (concatenated 3 * n_nodes, or a device pointer); None = cold start."""
        if u0 is None:
            capi.call("tlfea_batch_set_initial_guess", self._h, None, 0, 0)
        elif isinstance(u0, int):
            capi.call("tlfea_batch_set_initial_guess", self._h, C.c_void_p(u0), 3 * self.n_nodes, 1)
        else:
            a = _f64(u0, 3 * self.n_nodes, "u0")
            capi.call("tlfea_batch_set_initial_guess", self._h, a.ctypes.data_as(C.c_void_p), a.size, 0)

    def SetPrecision(self, precision: str):
        p = {"fp64": capi.PRECISION_FP64, "fp32": capi.PRECISION_FP32}[precision.lower()]
        capi.call("tlfea_batch_set_precision", self._h, p)

    def SetLaunch(self, blocks_per_sm: int = 0, chunk_nodes: int = 0):
        capi.call("tlfea_batch_set_launch", self._h, int(blocks_per_sm), int(chunk_nodes))

    MODES = {"phased": 0, "persistent": 1}

    def SetMode(self, mode: str = "phased"):
        """New: "phased" (default) -- one kernel per CG phase, chunks of iterations
        replayed as CUDA graphs -- or "persistent" (one cooperative launch)."""
        capi.call("tlfea_batch_set_mode", self._h, self.MODES[mode])

    def GetLaunch(self) -> dict:
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        capi.call("tlfea_batch_get_launch", self._h, C.byref(a), C.byref(b), C.byref(c))
        return {"blocks_per_sm": a.value, "chunk_nodes": b.value, "grid": c.value}

    def Autotune(self, trial_iters: int = 8) -> dict:
        a, b, ms = C.c_int(), C.c_int(), C.c_float()
        capi.call("tlfea_batch_autotune", self._h, int(trial_iters), C.byref(a), C.byref(b), C.byref(ms))
        return {"blocks_per_sm": a.value, "chunk_nodes": b.value, "trial_ms": ms.value}

    def Solve(self, tol: float = 1e-6, max_iter: int = 100000):
        capi.call("tlfea_batch_solve", self._h, float(tol), int(max_iter))

    def GetResults(self):
        """(iterations, ||r||/||f_free||, status) per instance; status 0 converged,
        1 non-positive p.Kp, 2 max_iter reached."""
        it = np.zeros(self.n_inst, np.int32)
        rel = np.zeros(self.n_inst)
        st = np.zeros(self.n_inst, np.int32)
        capi.call("tlfea_batch_get_results", self._h, capi.iptr(it), capi.dptr(rel), capi.iptr(st))
        return it, rel, st

    def RetrieveDisplacement(self, split: bool = True):
        u = np.zeros(3 * self.n_nodes)
        capi.call("tlfea_batch_retrieve_displacement", self._h, capi.dptr(u), u.size)
        if not split:
            return u
        return [u[3 * self.node_off[i]:3 * self.node_off[i + 1]] for i in range(self.n_inst)]

    def DevicePtrs(self) -> dict:
        u, f, u0 = C.c_void_p(), C.c_void_p(), C.c_void_p()
        capi.call("tlfea_batch_device_ptrs", self._h, C.byref(u), C.byref(f), C.byref(u0))
        return {"u": u.value, "f_ext": f.value, "u0": u0.value}

    def Apply(self, d_x: int, d_y: int):
        """y = K_bc x over the whole batch (device pointers, 3 * n_nodes doubles)."""
        capi.call("tlfea_batch_apply", self._h, C.c_void_p(d_x), C.c_void_p(d_y))

    def Destroy(self):
        if getattr(self, "_h", None) is not None:
            capi.call("tlfea_batch_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.Destroy()
        except Exception:
            pass


# -------------------------------------------------------------------- manager

class BatchedDynamics:
    """New: B sequences of implicit time steps on one mesh, each step solved by the
    SyncedNesterov iteration (SyncedNesterov.cu:97-360) in the same kernels for all
    sequences (tlfea_dynbatch_* in include/tlfea_b200.h).  `mesh` is a set-up element
    (Setup, CalcDnDuPre, CalcMassMatrix, fixed nodes, density, damping, external force
    such as gravity); each sequence has its own E and nu."""

    WARM_PREVIOUS, WARM_LINEAR, WARM_GIVEN = 0, 1, 2

    def __init__(self, mesh: _TetData, n_seq: int):
        self.mesh = mesh
        self.n_seq = int(n_seq)
        self.N = mesh.n_coef
        h = C.c_void_p()
        capi.call("tlfea_dynbatch_create", mesh._handle(), self.n_seq, C.byref(h))
        self._h = h

    def SetMaterial(self, E, nu):
        E = _f64(E, self.n_seq, "E")
        nu = _f64(nu, self.n_seq, "nu")
        capi.call("tlfea_dynbatch_set_material", self._h, capi.dptr(E), capi.dptr(nu))

    def SetParameters(self, params: SyncedNesterovParams, rel_tol: float = 0.0):
        p = capi.NesterovParams(*astuple(params))
        capi.call("tlfea_dynbatch_set_parameters", self._h, C.cast(C.byref(p), C.c_void_p), float(rel_tol))

    def SetStepSizes(self, alpha):
        a = _f64(alpha, self.n_seq, "alpha")
        capi.call("tlfea_dynbatch_set_step_sizes", self._h, capi.dptr(a))

    def SetLoad(self, f_var=None, amp: float = 0.0, omega: float = 0.0, phase: float = 0.0):
        fv = None if f_var is None else _f64(f_var, 3 * self.N, "f_var")
        capi.call("tlfea_dynbatch_set_load", self._h, capi.dptr(fv) if fv is not None else None, 3 * self.N,
                  float(amp), float(omega), float(phase))

    def SetChunk(self, chunk: int):
        capi.call("tlfea_dynbatch_set_chunk", self._h, int(chunk))

    def SetRestart(self, on: bool = True):
        """New: momentum restart of the inner Nesterov loop when g . (v_next - v_k) > 0
        (off by default: the reference's iteration)."""
        capi.call("tlfea_dynbatch_set_restart", self._h, 1 if on else 0)

    def Reset(self):
        capi.call("tlfea_dynbatch_reset", self._h)

    def Step(self, warm_start: int = 0, d_v_guess: int | None = None):
        """One step of every sequence; returns (iterations, relative residual, converged) per sequence."""
        it = np.zeros(self.n_seq, np.int32)
        rel = np.zeros(self.n_seq)
        conv = np.zeros(self.n_seq, np.int32)
        capi.call("tlfea_dynbatch_step", self._h, int(warm_start),
                  C.c_void_p(d_v_guess) if d_v_guess is not None else None, capi.iptr(it), capi.dptr(rel),
                  capi.iptr(conv))
        return it, rel, conv

    def DevicePtrs(self) -> dict:
        ptrs = [C.c_void_p() for _ in range(5)]
        capi.call("tlfea_dynbatch_device_ptrs", self._h, *[C.byref(p) for p in ptrs])
        return dict(zip(("x", "y", "z", "v", "v_hist"), (p.value for p in ptrs)))

    def RetrievePositions(self, seq: int):
        x, y, z = (np.zeros(self.N) for _ in range(3))
        capi.call("tlfea_dynbatch_retrieve_positions", self._h, int(seq), capi.dptr(x), capi.dptr(y), capi.dptr(z))
        return x, y, z

    def RetrieveVelocity(self, seq: int):
        v = np.zeros(3 * self.N)
        capi.call("tlfea_dynbatch_retrieve_velocity", self._h, int(seq), capi.dptr(v))
        return v

    def Destroy(self):
        if getattr(self, "_h", None):
            capi.call("tlfea_dynbatch_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.Destroy()
        except Exception:
            pass


class FEASolver:
    """FEASolver (FEASolver.h:35-138): name -> non-owning element / solver registry."""

    def __init__(self):
        self._elements: dict = {}
        self._solvers: dict = {}

    def AddElement(self, name: str, element):
        if element is None:
            raise ValueError("FEASolver::AddElement: element pointer is null")
        if name in self._elements:
            raise ValueError(f"FEASolver::AddElement: element '{name}' already registered")
        self._elements[name] = element

    def GetElement(self, name: str):
        if name not in self._elements:
            raise KeyError(f"FEASolver::GetElement: element '{name}' not found")
        return self._elements[name]

    def GetNumElements(self) -> int:
        return len(self._elements)

    def AddSolver(self, name: str, solver):
        if solver is None:
            raise ValueError("FEASolver::AddSolver: solver pointer is null")
        if name in self._solvers:
            raise ValueError(f"FEASolver::AddSolver: solver '{name}' already registered")
        self._solvers[name] = solver

    def GetSolver(self, name: str):
        if name not in self._solvers:
            raise KeyError(f"FEASolver::GetSolver: solver '{name}' not found")
        return self._solvers[name]

    def GetNumSolvers(self) -> int:
        return len(self._solvers)


class WarmStartMLP:
    """New, no reference counterpart: the warm-start network, trained and
    evaluated by this library's tcgen05 kernels (BF16 operands, FP32
    accumulation, FP32 master weights, AdamW, mean-squared-error loss).

    dims: layer widths, e.g. (6, 256, 256, 256, 64); GELU between layers.
    Tensors passed as ints are device pointers (FP32, row-major); the kernels
    run on the network's own stream (GetStream), so producers of those tensors
    either run on that stream or finish first.
    """

    def __init__(self, dims, max_batch: int = 512, seed: int = 0):
        self.dims = [int(d) for d in dims]
        d = np.asarray(self.dims, np.int32)
        h = C.c_void_p()
        capi.call("tlfea_mlp_create", len(self.dims) - 1, capi.iptr(d), int(max_batch), int(seed), C.byref(h))
        self._h = h
        self.max_batch = int(max_batch)
        n = C.c_longlong()
        capi.call("tlfea_mlp_param_count", self._h, C.byref(n))
        self.n_params = n.value

    def GetStream(self) -> int:
        s = C.c_void_p()
        capi.call("tlfea_mlp_get_stream", self._h, C.byref(s))
        return s.value or 0

    def SetParams(self, flat):
        a = np.ascontiguousarray(np.asarray(flat, dtype=np.float32).ravel())
        capi.call("tlfea_mlp_set_params", self._h, capi.fptr(a), a.size)

    def GetParams(self) -> np.ndarray:
        a = np.zeros(self.n_params, np.float32)
        capi.call("tlfea_mlp_get_params", self._h, capi.fptr(a), a.size)
        return a

    def GetGrads(self) -> np.ndarray:
        a = np.zeros(self.n_params, np.float32)
        capi.call("tlfea_mlp_get_grads", self._h, capi.fptr(a), a.size)
        return a

    def Forward(self, d_x: int, batch: int, d_y: int):
        capi.call("tlfea_mlp_forward", self._h, C.c_void_p(d_x), int(batch), C.c_void_p(d_y))

    def LossGrad(self, d_x: int, d_t: int, batch: int) -> float:
        loss = C.c_float()
        capi.call("tlfea_mlp_loss_grad", self._h, C.c_void_p(d_x), C.c_void_p(d_t), int(batch), C.byref(loss))
        return loss.value

    def AdamWStep(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        capi.call("tlfea_mlp_adamw_step", self._h, lr, beta1, beta2, eps, weight_decay)

    def TrainStep(self, d_x: int, d_t: int, batch: int, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8,
                  weight_decay=0.0, want_loss=False):
        loss = C.c_float()
        capi.call("tlfea_mlp_train_step", self._h, C.c_void_p(d_x), C.c_void_p(d_t), int(batch), lr, beta1, beta2,
                  eps, weight_decay, C.byref(loss) if want_loss else None)
        return loss.value if want_loss else None

    def Sync(self):
        capi.call("tlfea_mlp_sync", self._h)

    def Destroy(self):
        if getattr(self, "_h", None) is not None:
            capi.call("tlfea_mlp_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.Destroy()
        except Exception:
            pass


def gemm_bf16(M, N, K, d_a, lda, d_b, ldb, d_bias, d_d, ldd, stream=0):
    """The MLP's tcgen05 product on its own: D = A B^T (+ bias), BF16 in, FP32 out."""
    capi.call("tlfea_mlp_gemm_bf16", int(M), int(N), int(K), C.c_void_p(d_a), int(lda), C.c_void_p(d_b), int(ldb),
              C.c_void_p(d_bias) if d_bias else None, C.c_void_p(d_d), int(ldd), C.c_void_p(stream))


def gemm_bf16_async(M, N, K, d_a, lda, d_b, ldb, d_bias, d_d, ldd, d_err, stream=0):
    """gemm_bf16 only enqueued on `stream`; *d_err (device int32, zeroed by the
    caller) turns non-zero if a bounded wait in the kernel ran out."""
    capi.call("tlfea_mlp_gemm_bf16_async", int(M), int(N), int(K), C.c_void_p(d_a), int(lda), C.c_void_p(d_b),
              int(ldb), C.c_void_p(d_bias) if d_bias else None, C.c_void_p(d_d), int(ldd), C.c_void_p(d_err),
              C.c_void_p(stream))
