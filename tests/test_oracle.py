"""CPU tests of the oracle itself (no GPU): analytic known-answer tests that pin
the restatement, plus the mesh utilities it is checked against.  The reference
ships no golden vectors (see oracle/tlfea_oracle.h), so these are the pins."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import oracle as O
from tlfea_b200 import mesh as M
from tlfea_b200 import quadrature as Q

from .helpers import lame, rel

LAM, MU = lame()


@pytest.mark.parametrize("order", [10, 4])
def test_box_mesh_counts_match_configs(order):
    # the benchmark meshes: cells -> (nodes, elements); 10x2x2 T10 is 525 / 240.
    for (nx, ny, nz) in [(10, 2, 2), (40, 8, 8), (100, 10, 10)]:
        nn, ne = M.box_counts(nx, ny, nz, order)
        x, y, z, conn = O.box_mesh(nx, ny, nz, order)
        assert (len(x), conn.shape[0]) == (nn, ne)
    assert M.box_counts(10, 2, 2, 10) == (525, 240)
    assert M.box_counts(200, 20, 20, 10) == (674081, 480000)
    assert M.box_counts(200, 20, 20, 4) == (88641, 480000)
    assert M.box_counts(40, 8, 8, 10) == (23409, 15360)


@pytest.mark.parametrize("order", [10, 4])
def test_python_and_c_mesh_generators_agree(order):
    a = O.box_mesh(7, 3, 2, order, 0.7, 0.3, 0.2)
    b = M.box_mesh(7, 3, 2, order, 0.7, 0.3, 0.2)
    for u, v in zip(a[:3], b[:3]):
        assert np.array_equal(u, v)
    assert np.array_equal(a[3], b[3])


def test_quadrature_tables():
    qx, qy, qz, qw = O.quadrature(10)
    assert np.array_equal(qx, Q.tet5pt_x) and np.array_equal(qy, Q.tet5pt_y) and np.array_equal(qz, Q.tet5pt_z)
    assert np.array_equal(qw, Q.tet5pt_weights)
    assert qw.sum() == pytest.approx(1.0 / 6.0, rel=1e-15)
    # Keast 5-point is exact for cubics on the unit tet: int x^3 = 1/120, int xyz = 1/720
    assert np.dot(qw, qx ** 3) == pytest.approx(1 / 120, rel=1e-13)
    assert np.dot(qw, qx * qy * qz) == pytest.approx(1 / 720, rel=1e-13)


@pytest.mark.parametrize("order", [10, 4])
def test_positive_jacobians_and_volume(order):
    x, y, z, conn = O.box_mesh(10, 2, 2, order)
    g, dj = O.dndu_pre(x, y, z, conn)
    assert (dj > 0).all()
    nqp = 5 if order == 10 else 1
    assert (dj.reshape(-1, nqp) * O.quadrature(order)[3]).sum() == pytest.approx(0.01, rel=1e-13)
    # sum_a X_a (x) grad N_a = I at every QP
    G = O.grad_to_array(g, conn.shape[0], order)
    X = np.stack([x, y, z], 1)[conn]  # (E, NPE, 3)
    F = np.einsum("eai,eqaj->eqij", X, G)
    assert np.abs(F - np.eye(3)).max() < 1e-12


@pytest.mark.parametrize("order", [10, 4])
def test_rigid_motion_gives_zero_stress(order):
    x, y, z, conn = O.box_mesh(10, 2, 2, order)
    g, dj = O.dndu_pre(x, y, z, conn)
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    Xr = R @ np.stack([x, y, z]) + np.array([[0.3], [-0.2], [1.0]])
    f = O.force(*Xr, conn, g, dj, LAM, MU)
    assert np.abs(f).max() < 1e-9 * MU * 1e-2


@pytest.mark.parametrize("order", [10, 4])
def test_kelvin_voigt_damping_known_answers(order):
    """Known answers for the oracle's Kelvin-Voigt term (FEAT10DataFunc.cuh:130-231):
    a rigid spin v = w x (x - c) of a deformed body has zero rate of strain, so
    the damped force equals the undamped one; under a homogeneous deformation
    x = A X moving with v = B X, the viscous stress at every QP is
    P_vis = A (2 eta Ed + lambda_d tr(Ed) I), Ed = (B^T A + A^T B) / 2."""
    eta, lamd = 3.0e3, 7.0e2
    x, y, z, conn = O.box_mesh(4, 2, 2, order, 0.4, 0.2, 0.2)
    g, dj = O.dndu_pre(x, y, z, conn)
    xs = np.stack([x, y, z]) + 2e-3 * np.random.default_rng(3).standard_normal((3, len(x)))
    w = np.array([0.3, -1.1, 0.7])
    v = np.cross(w, (xs - xs.mean(1, keepdims=True)).T).ravel()
    f0 = O.force(*xs, conn, g, dj, LAM, MU)
    fd = O.force(*xs, conn, g, dj, LAM, MU, eta, lamd, v)
    assert rel(fd, f0) < 1e-10
    A = np.array([[1.02, 0.01, 0.0], [0.0, 0.99, 0.02], [0.01, 0.0, 1.01]])
    B = np.array([[0.3, -0.1, 0.2], [0.05, -0.2, 0.1], [0.0, 0.15, 0.25]])
    X = np.stack([x, y, z])
    F, P = O.calc_p(*(A @ X), conn, g, LAM, MU)
    _, Pd = O.calc_p(*(A @ X), conn, g, LAM, MU, eta, lamd, (B @ X).T.ravel())
    Ed = 0.5 * (B.T @ A + A.T @ B)
    Pv = A @ (2 * eta * Ed + lamd * np.trace(Ed) * np.eye(3))
    dP = (Pd - P).reshape(-1, 3, 3).transpose(0, 2, 1)
    assert rel(dP, np.broadcast_to(Pv, dP.shape)) < 1e-10


@pytest.mark.parametrize("order", [10, 4])
def test_homogeneous_deformation_patch(order):
    x, y, z, conn = O.box_mesh(6, 3, 3, order, 0.6, 0.3, 0.3)
    g, dj = O.dndu_pre(x, y, z, conn)
    A = np.array([[1.01, 0.002, 0.0], [0.0, 0.995, 0.003], [0.001, 0.0, 1.002]])
    Xa = A @ np.stack([x, y, z])
    F, P = O.calc_p(*Xa, conn, g, LAM, MU)
    F = F.reshape(-1, 3, 3).transpose(0, 2, 1)
    assert np.abs(F - A).max() < 1e-12
    E = 0.5 * (A.T @ A - np.eye(3))
    P_ref = A @ (LAM * np.trace(E) * np.eye(3) + 2 * MU * E)
    P = P.reshape(-1, 3, 3).transpose(0, 2, 1)
    assert rel(P, np.broadcast_to(P_ref, P.shape)) < 1e-11
    f = O.force(*Xa, conn, g, dj, LAM, MU).reshape(-1, 3)
    tol = 1e-12
    interior = ~(np.isclose(x, x.min(), atol=tol) | np.isclose(x, x.max(), atol=tol) | np.isclose(y, y.min(), atol=tol)
                 | np.isclose(y, y.max(), atol=tol) | np.isclose(z, z.min(), atol=tol) | np.isclose(z, z.max(), atol=tol))
    assert interior.any()
    assert np.abs(f[interior]).max() < 1e-9 * np.abs(f).max()


def _mr_energy(F, mu10, mu01, kappa):
    """Mooney-Rivlin strain energy mu10 (I1bar - 3) + mu01 (I2bar - 3) + kappa/2 (J - 1)^2,
    whose derivative dW/dF is the first Piola stress of MooneyRivlin.cuh:46-104."""
    C = F.T @ F
    I1 = np.trace(C)
    I2 = 0.5 * (I1 ** 2 - np.trace(C @ C))
    J = np.linalg.det(F)
    return mu10 * (J ** (-2 / 3) * I1 - 3) + mu01 * (J ** (-4 / 3) * I2 - 3) + 0.5 * kappa * (J - 1) ** 2


@pytest.mark.parametrize("order", [10, 4])
def test_mooney_rivlin_stress_is_the_energy_derivative(order):
    """Known answer for the Mooney-Rivlin oracle: under a homogeneous deformation
    x = A X the stress at every QP is dW/dF at A (central differences), a rigid
    rotation gives zero force, and interior nodes are in equilibrium."""
    mu10, mu01, kappa = 2.0e5, 5.0e4, 1.0e7
    x, y, z, conn = O.box_mesh(4, 2, 2, order, 0.4, 0.2, 0.2)
    g, dj = O.dndu_pre(x, y, z, conn)
    A = np.array([[1.04, 0.02, -0.01], [0.01, 0.97, 0.03], [0.02, -0.01, 1.01]])
    with O.mooney_rivlin(mu10, mu01, kappa):
        F, P = O.calc_p(*(A @ np.stack([x, y, z])), conn, g, 0.0, 0.0)
        th = 0.5
        R = np.array([[np.cos(th), -np.sin(th), 0.0], [np.sin(th), np.cos(th), 0.0], [0.0, 0.0, 1.0]])
        f_rigid = O.force(*(R @ np.stack([x, y, z]) + 0.3), conn, g, dj, 0.0, 0.0)
        f_hom = O.force(*(A @ np.stack([x, y, z])), conn, g, dj, 0.0, 0.0).reshape(-1, 3)
    P = P.reshape(-1, 3, 3).transpose(0, 2, 1)
    h = 1e-6
    dW = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            Ap, Am = A.copy(), A.copy()
            Ap[i, j] += h
            Am[i, j] -= h
            dW[i, j] = (_mr_energy(Ap, mu10, mu01, kappa) - _mr_energy(Am, mu10, mu01, kappa)) / (2 * h)
    assert rel(P, np.broadcast_to(dW, P.shape)) < 1e-7
    assert np.abs(f_rigid).max() < 1e-9 * np.abs(f_hom).max()
    tol = 1e-12
    interior = ~(np.isclose(x, x.min(), atol=tol) | np.isclose(x, x.max(), atol=tol) | np.isclose(y, y.min(), atol=tol)
                 | np.isclose(y, y.max(), atol=tol) | np.isclose(z, z.min(), atol=tol) | np.isclose(z, z.max(), atol=tol))
    if interior.any():
        assert np.abs(f_hom[interior]).max() < 1e-9 * np.abs(f_hom).max()


@pytest.mark.parametrize("order", [10, 4])
def test_internal_force_from_p_matches_fused(order):
    x, y, z, conn = O.box_mesh(5, 2, 2, order, 0.5, 0.2, 0.2)
    g, dj = O.dndu_pre(x, y, z, conn)
    r = np.random.default_rng(1)
    xs = [v + 1e-3 * r.standard_normal(v.shape) for v in (x, y, z)]
    _, P = O.calc_p(*xs, conn, g, LAM, MU)
    f1 = O.internal_force_from_p(conn, g, dj, P, len(x))
    f2 = O.force(*xs, conn, g, dj, LAM, MU)
    assert rel(f1, f2) < 1e-13
    # CalcInternalForce accumulates (FEAT10Data.cu:318-323 does not clear f_int)
    f3 = O.internal_force_from_p(conn, g, dj, P, len(x), f_init=f1)
    assert rel(f3, 2 * f1) < 1e-14


@pytest.mark.parametrize("order", [10, 4])
def test_mass_total_and_symmetry(order):
    x, y, z, conn = O.box_mesh(10, 2, 2, order)
    g, dj = O.dndu_pre(x, y, z, conn)
    off, cols, vals = O.mass(conn, dj, len(x), 1000.0)
    Mm = sp.csr_matrix((vals, cols, off))
    assert vals.sum() == pytest.approx(1000.0 * 0.01, rel=1e-12)
    assert abs(Mm - Mm.T).max() < 1e-15


@pytest.mark.parametrize("order", [10, 4])
def test_elementwise_mass_product_equals_assembled(order):
    """The first-order solvers apply M (v - v_prev) element by element: per QP,
    w(q) = sum_b N_b(q) w_b and f_a += rho N_a(q) dV w(q), with the corner
    L_i (2 L_i - 1) and edge 4 L_i L_j shape functions at the barycentric QPs.
    That product equals the oracle's assembled consistent mass times w."""
    x, y, z, conn = O.box_mesh(4, 2, 2, order, 0.4, 0.2, 0.2)
    N, E = len(x), conn.shape[0]
    g, dj = O.dndu_pre(x, y, z, conn)
    rho = 1000.0
    off, cols, vals = O.mass(conn, dj, N, rho)
    w = np.random.default_rng(7).standard_normal((N, 3))
    ref = sp.csr_matrix((vals, cols, off)) @ w
    qx, qy, qz, qw = O.quadrature(conn.shape[1])
    nqp = len(qw)
    L = np.stack([1.0 - qx - qy - qz, qx, qy, qz], 1)  # (nqp, 4)
    if order == 10:
        edges = [(0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3)]
        Nq = np.concatenate([L * (2.0 * L - 1.0), np.stack([4.0 * L[:, i] * L[:, j] for i, j in edges], 1)], 1)
    else:
        Nq = L
    dV = dj.reshape(E, nqp) * qw[None, :]
    we = w[conn]                                        # (E, NPE, 3)
    wq = np.einsum("qb,ebd->eqd", Nq, we)               # w at the QPs
    fe = rho * np.einsum("qa,eq,eqd->ead", Nq, dV, wq)  # element contributions
    out = np.zeros((N, 3))
    np.add.at(out, conn.ravel(), fe.reshape(-1, 3))
    assert rel(out, ref) < 1e-13


@pytest.mark.parametrize("order", [10, 4])
def test_stiffness_is_consistent_tangent(order):
    x, y, z, conn = O.box_mesh(4, 2, 2, order, 0.4, 0.2, 0.2)
    g, dj = O.dndu_pre(x, y, z, conn)
    r = np.random.default_rng(2)
    xs = [v + 2e-3 * r.standard_normal(v.shape) for v in (x, y, z)]
    off, cols, vals = O.stiffness(*xs, conn, g, dj, LAM, MU)
    K = sp.csr_matrix((vals, cols, off))
    # rigid translation in the null space; symmetric; K = d f_int / d x (central differences)
    du = 1e-7 * r.standard_normal(3 * len(x))
    X = np.stack(xs, 1).ravel()
    fp = O.force(*(X + du).reshape(-1, 3).T, conn, g, dj, LAM, MU)
    fm = O.force(*(X - du).reshape(-1, 3).T, conn, g, dj, LAM, MU)
    assert rel((fp - fm) / 2, K @ du) < 1e-6
    assert abs(K - K.T).max() < 1e-8 * abs(K).max()


@pytest.mark.parametrize("order", [10, 4])
def test_mooney_rivlin_stiffness_is_consistent_tangent(order):
    """The oracle's Mooney-Rivlin stiffness is d f_int / d x of its Mooney-Rivlin force."""
    x, y, z, conn = O.box_mesh(4, 2, 2, order, 0.4, 0.2, 0.2)
    g, dj = O.dndu_pre(x, y, z, conn)
    r = np.random.default_rng(5)
    xs = [v + 3e-3 * r.standard_normal(v.shape) for v in (x, y, z)]
    du = 1e-7 * r.standard_normal(3 * len(x))
    X = np.stack(xs, 1).ravel()
    with O.mooney_rivlin(2.0e6, 5.0e5, 5.0e7):
        off, cols, vals = O.stiffness(*xs, conn, g, dj, 0.0, 0.0)
        fp = O.force(*(X + du).reshape(-1, 3).T, conn, g, dj, 0.0, 0.0)
        fm = O.force(*(X - du).reshape(-1, 3).T, conn, g, dj, 0.0, 0.0)
    K = sp.csr_matrix((vals, cols, off))
    assert rel((fp - fm) / 2, K @ du) < 1e-6
    assert abs(K - K.T).max() < 1e-8 * abs(K).max()


def test_cg_matches_direct_solve():
    x, y, z, conn = O.box_mesh(10, 2, 2, 10)
    g, dj = O.dndu_pre(x, y, z, conn)
    off, cols, vals = O.stiffness(x, y, z, conn, g, dj, LAM, MU)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -100.0))
    kv, fb = O.apply_bcs(off, cols, vals, f, fixed)
    u, it, res, rc = O.cg(off, cols, kv, fb, 1e-12, 20000)
    assert rc == 0 and res < 1e-12 and it > 0
    K = sp.csr_matrix((kv, cols, off)).tocsc()
    u_ref = spla.spsolve(K, fb)
    assert rel(u, u_ref) < 1e-9


def test_tetgen_remap_is_a_permutation():
    tg = np.arange(10, dtype=np.int32)
    st = M.remap_tetgen_t10(tg)
    assert sorted(st.tolist()) == list(range(10))
    assert st.tolist() == [0, 1, 2, 3, 6, 7, 9, 5, 8, 4]


def test_nesterov_oracle_at_rest_stays_at_rest():
    x, y, z, conn = O.box_mesh(4, 1, 1, 10, 0.4, 0.1, 0.1)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, 0.0))
    m = O.OracleModel(x, y, z, conn, 1e7, 0.3, 1000.0, fixed, f)
    m.set_parameters()
    st = m.nesterov_solve(1e-8, 1e14, 1e-6, 1e-6, 2, 20, 1e-3)
    # only the rounding of f_int(X) ~ 1e-16 * stiffness drives it
    assert np.abs(m.v_guess).max() < 1e-12
    assert np.abs(m.x - x).max() < 1e-14
    assert st["outer_iters"] >= 1


def test_adamw_oracles_reduce_residual():
    x, y, z, conn = O.box_mesh(4, 1, 1, 10, 0.4, 0.1, 0.1)
    fixed, f, _ = M.cantilever_loads(x, y, z, (0.0, 0.0, -1.0))
    for fn in ("adamw_solve", "adamw_nocoop_solve"):
        m = O.OracleModel(x, y, z, conn, 1e7, 0.3, 1000.0, fixed, f)
        m.set_parameters()
        st = getattr(m, fn)(2e-4, 0.9, 0.999, 1e-8, 1e-4, 0.9995, 1e-6, 1e-6, 1e14, 3, 200, 1e-3, 5, 1e-3)
        assert st["inner_iters_total"] > 0
        assert np.isfinite(m.x).all()
