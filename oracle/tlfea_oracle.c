/*
 * tlfea_oracle.c -- CPU restatement of the TLFEA hot path (TEST INFRASTRUCTURE).
 *
 * Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg, as the checker.  Plain FP64 C99 + OpenMP.  Each routine follows the
 * reference step cited in tlfea_oracle.h and keeps the reference's operation
 * order where it is sequential (norms, per-QP sums, per-element sums).  The
 * reference scatters element forces and stiffness blocks with atomicAdd in an
 * unspecified order; here they are added in element order (deterministic).
 *
 * Parity: pinned to fixtures written by the reference's own CUDA build
 * (tests/golden/ref_*.npz, checked by tests/test_ref_fixtures.py) and by analytic
 * known-answer tests in tests/.
 */
#include "tlfea_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 0;

void orc_set_threads(int n) {
    g_threads = n;
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* ===================================================================== meshes */

int orc_box_counts(int nx, int ny, int nz, int order, int* n_nodes, int* n_elems) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || (order != 10 && order != 4)) return 1;
    int m = (order == 10) ? 2 : 1;
    *n_nodes = (m * nx + 1) * (m * ny + 1) * (m * nz + 1);
    *n_elems = 6 * nx * ny * nz;
    return 0;
}

/* Kuhn split: tet k walks v000 -> +e_a -> +e_a+e_b -> v111 along permutation
 * (a,b,c) of the axes.  Odd permutations have negative volume; their vertices
 * 1 and 2 are swapped (the reference never takes |detJ|). */
int orc_box_mesh(int nx, int ny, int nz, int order, double lx, double ly, double lz, double* x, double* y,
                 double* z, int* conn) {
    int NN, NE;
    if (orc_box_counts(nx, ny, nz, order, &NN, &NE)) return 1;
    const int m = (order == 10) ? 2 : 1;
    const int NX = m * nx + 1, NY = m * ny + 1, NZ = m * nz + 1;
    for (int ix = 0; ix < NX; ++ix)
        for (int iy = 0; iy < NY; ++iy)
            for (int iz = 0; iz < NZ; ++iz) {
                int id = (ix * NY + iy) * NZ + iz;
                x[id] = lx * (double)ix / (double)(m * nx);
                y[id] = ly * (double)iy / (double)(m * ny);
                z[id] = lz * (double)iz / (double)(m * nz);
            }
    static const int perms[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
    static const int edges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
    const int npe = order;
    int e = 0;
    for (int cx = 0; cx < nx; ++cx)
        for (int cy = 0; cy < ny; ++cy)
            for (int cz = 0; cz < nz; ++cz)
                for (int k = 0; k < 6; ++k) {
                    int g[4][3];
                    int p[3] = {cx, cy, cz};
                    g[0][0] = p[0]; g[0][1] = p[1]; g[0][2] = p[2];
                    for (int s = 1; s < 4; ++s) {
                        p[perms[k][s - 1]] += 1;
                        g[s][0] = p[0]; g[s][1] = p[1]; g[s][2] = p[2];
                    }
                    if (k >= 3) { /* odd permutation: swap vertices 1 and 2 */
                        for (int d = 0; d < 3; ++d) {
                            int t = g[1][d]; g[1][d] = g[2][d]; g[2][d] = t;
                        }
                    }
                    int hv[10][3];
                    for (int a = 0; a < 4; ++a)
                        for (int d = 0; d < 3; ++d) hv[a][d] = m * g[a][d];
                    if (order == 10)
                        for (int s = 0; s < 6; ++s)
                            for (int d = 0; d < 3; ++d)
                                hv[4 + s][d] = (hv[edges[s][0]][d] + hv[edges[s][1]][d]) / 2;
                    for (int a = 0; a < npe; ++a) conn[e + a * NE] = (hv[a][0] * NY + hv[a][1]) * NZ + hv[a][2];
                    ++e;
                }
    return 0;
}

/* quadrature_utils.h:134-164 (tet5pt_bary columns 1..3, weights) and :176-179. */
void orc_quadrature_t10(double* qx, double* qy, double* qz, double* qw) {
    const double a = 0.25, b = 0.5, c = 1.0 / 6.0;
    /* rows of tet5pt_bary are (L1..L4); x, y, z are its columns 1, 2, 3 */
    const double bx[5] = {a, c, b, c, c};
    const double by[5] = {a, c, c, b, c};
    const double bz[5] = {a, c, c, c, b};
    const double w[5] = {-4.0 / 5.0, 9.0 / 20.0, 9.0 / 20.0, 9.0 / 20.0, 9.0 / 20.0};
    for (int q = 0; q < 5; ++q) {
        qx[q] = bx[q];
        qy[q] = by[q];
        qz[q] = bz[q];
        qw[q] = w[q] * (1.0 / 6.0);
    }
}

void orc_quadrature_t4(double* qx, double* qy, double* qz, double* qw) {
    qx[0] = 0.25;
    qy[0] = 0.25;
    qz[0] = 0.25;
    qw[0] = 1.0 / 6.0;
}

void orc_remap_tetgen_t10(const int* tg, int* st) {
    static const int map[10] = {0, 1, 2, 3, 6, 7, 9, 5, 8, 4};
    for (int i = 0; i < 10; ++i) st[i] = tg[map[i]];
}

/* ============================================================== precompute */

/* solve_3x3_system (FEAT10DataFunc.cuh:32-84): partial pivoting, |pivot|<1e-14 -> 0. */
static void solve3(const double A[3][3], const double b[3], double xo[3]) {
    double aug[3][4];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) aug[i][j] = A[i][j];
        aug[i][3] = b[i];
    }
    for (int k = 0; k < 3; ++k) {
        int pr = k;
        double mv = fabs(aug[k][k]);
        for (int i = k + 1; i < 3; ++i)
            if (fabs(aug[i][k]) > mv) {
                mv = fabs(aug[i][k]);
                pr = i;
            }
        if (pr != k)
            for (int j = 0; j < 4; ++j) {
                double t = aug[k][j];
                aug[k][j] = aug[pr][j];
                aug[pr][j] = t;
            }
        if (fabs(aug[k][k]) < 1e-14) {
            xo[0] = xo[1] = xo[2] = 0.0;
            return;
        }
        for (int i = k + 1; i < 3; ++i) {
            double f = aug[i][k] / aug[k][k];
            for (int j = k; j < 4; ++j) aug[i][j] -= f * aug[k][j];
        }
    }
    xo[2] = aug[2][3] / aug[2][2];
    xo[1] = (aug[1][3] - aug[1][2] * xo[2]) / aug[1][1];
    xo[0] = (aug[0][3] - aug[0][2] * xo[2] - aug[0][1] * xo[1]) / aug[0][0];
}

static double det3(const double J[3][3]) {
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

void orc_dndu_pre_t10(int E, const double* x, const double* y, const double* z, const int* conn,
                      const double* qx, const double* qy, const double* qz, double* grad, double* detJ) {
    static const int edges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
    static const double dL[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
#pragma omp parallel for schedule(static)
    for (int e = 0; e < E; ++e) {
        for (int q = 0; q < 5; ++q) {
            double xi = qx[q], eta = qy[q], zeta = qz[q];
            double L[4] = {1.0 - xi - eta - zeta, xi, eta, zeta};
            double dN[10][3];
            for (int i = 0; i < 4; ++i) {
                double f = 4.0 * L[i] - 1.0;
                for (int j = 0; j < 3; ++j) dN[i][j] = f * dL[i][j];
            }
            for (int k = 0; k < 6; ++k) {
                int i = edges[k][0], j = edges[k][1];
                for (int d = 0; d < 3; ++d) dN[k + 4][d] = 4.0 * (L[i] * dL[j][d] + L[j] * dL[i][d]);
            }
            double X[10][3];
            for (int a = 0; a < 10; ++a) {
                int n = conn[e + a * E];
                X[a][0] = x[n];
                X[a][1] = y[n];
                X[a][2] = z[n];
            }
            double J[3][3] = {{0}};
            for (int a = 0; a < 10; ++a)
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) J[i][j] += X[a][i] * dN[a][j];
            double dj = det3(J);
            detJ[e * 5 + q] = dj;
            double JT[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) JT[i][j] = J[j][i];
            double* gq = grad + (size_t)(e * 5 + q) * 30;
            for (int a = 0; a < 10; ++a) {
                double g[3];
                solve3(JT, dN[a], g);
                gq[a + 0] = g[0];
                gq[a + 10] = g[1];
                gq[a + 20] = g[2];
            }
        }
    }
}

void orc_dndu_pre_t4(int E, const double* x, const double* y, const double* z, const int* conn, double* grad,
                     double* detJ) {
    static const double dN[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
#pragma omp parallel for schedule(static)
    for (int e = 0; e < E; ++e) {
        double X[4][3];
        for (int a = 0; a < 4; ++a) {
            int n = conn[e + a * E];
            X[a][0] = x[n];
            X[a][1] = y[n];
            X[a][2] = z[n];
        }
        double J[3][3] = {{0}};
        for (int a = 0; a < 4; ++a)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) J[i][j] += X[a][i] * dN[a][j];
        detJ[e] = det3(J);
        double JT[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) JT[i][j] = J[j][i];
        double dT = det3(JT);
        double inv = (dT != 0.0) ? 1.0 / dT : 0.0;
        double Ji[3][3];
        Ji[0][0] = (JT[1][1] * JT[2][2] - JT[1][2] * JT[2][1]) * inv;
        Ji[0][1] = -(JT[0][1] * JT[2][2] - JT[0][2] * JT[2][1]) * inv;
        Ji[0][2] = (JT[0][1] * JT[1][2] - JT[0][2] * JT[1][1]) * inv;
        Ji[1][0] = -(JT[1][0] * JT[2][2] - JT[1][2] * JT[2][0]) * inv;
        Ji[1][1] = (JT[0][0] * JT[2][2] - JT[0][2] * JT[2][0]) * inv;
        Ji[1][2] = -(JT[0][0] * JT[1][2] - JT[0][2] * JT[1][0]) * inv;
        Ji[2][0] = (JT[1][0] * JT[2][1] - JT[1][1] * JT[2][0]) * inv;
        Ji[2][1] = -(JT[0][0] * JT[2][1] - JT[0][1] * JT[2][0]) * inv;
        Ji[2][2] = (JT[0][0] * JT[1][1] - JT[0][1] * JT[1][0]) * inv;
        double* gq = grad + (size_t)e * 12;
        for (int a = 0; a < 4; ++a)
            for (int i = 0; i < 3; ++i) {
                double s = 0.0;
                for (int j = 0; j < 3; ++j) s += Ji[i][j] * dN[a][j];
                gq[a + 4 * i] = s;
            }
    }
}

/* ======================================================== stress and force */

/* Material of the stress routines: 0 = SVK (lambda, mu passed per call), 1 =
 * Mooney-Rivlin with these parameters (FEAT10Data.cuh material_model switch). */
static int g_material = 0;
static double g_mu10 = 0.0, g_mu01 = 0.0, g_kappa = 0.0;

void orc_set_material(int model, double mu10, double mu01, double kappa) {
    g_material = model;
    g_mu10 = mu10;
    g_mu01 = mu01;
    g_kappa = kappa;
}

/* Mooney-Rivlin first Piola stress (mr_compute_P, MooneyRivlin.cuh:46-104):
 * C = F^T F, I1 = tr C, I2 = (I1^2 - tr C^2) / 2, J = det F, F^-T by cofactors
 * with |J| clamped to 1e-12 for the inverse, and
 * P = 2 mu10 J^-2/3 (F - I1/3 F^-T) + 2 mu01 J^-4/3 (I1 F - F C - 2 I2/3 F^-T)
 *   + kappa (J - 1) J F^-T. */
static void mr_p(const double F[3][3], double mu10, double mu01, double kappa, double P[3][3]) {
    double C[3][3] = {{0}}, C2[3][3] = {{0}}, FC[3][3] = {{0}}, FiT[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) C[i][j] += F[k][i] * F[k][j];
    const double I1 = C[0][0] + C[1][1] + C[2][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) C2[i][j] += C[i][k] * C[k][j];
    const double I2 = 0.5 * (I1 * I1 - (C2[0][0] + C2[1][1] + C2[2][2]));
    const double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                     F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                     F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
    double dj = J;
    if (fabs(dj) < 1e-12) dj = (dj >= 0.0) ? 1e-12 : -1e-12;
    const double id = 1.0 / dj;
    FiT[0][0] = (F[1][1] * F[2][2] - F[1][2] * F[2][1]) * id;
    FiT[0][1] = (F[1][2] * F[2][0] - F[1][0] * F[2][2]) * id;
    FiT[0][2] = (F[1][0] * F[2][1] - F[1][1] * F[2][0]) * id;
    FiT[1][0] = (F[0][2] * F[2][1] - F[0][1] * F[2][2]) * id;
    FiT[1][1] = (F[0][0] * F[2][2] - F[0][2] * F[2][0]) * id;
    FiT[1][2] = (F[0][1] * F[2][0] - F[0][0] * F[2][1]) * id;
    FiT[2][0] = (F[0][1] * F[1][2] - F[0][2] * F[1][1]) * id;
    FiT[2][1] = (F[0][2] * F[1][0] - F[0][0] * F[1][2]) * id;
    FiT[2][2] = (F[0][0] * F[1][1] - F[0][1] * F[1][0]) * id;
    const double j13 = cbrt(J);
    const double jm23 = 1.0 / (j13 * j13), jm43 = jm23 * jm23;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) FC[i][j] += F[i][k] * C[k][j];
    const double t1 = 2.0 * mu10 * jm23, t2 = 2.0 * mu01 * jm43, t3 = kappa * (J - 1.0) * J;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            P[i][j] = t1 * (F[i][j] - (I1 / 3.0) * FiT[i][j]) +
                      t2 * (I1 * F[i][j] - FC[i][j] - (2.0 * I2 / 3.0) * FiT[i][j]) + t3 * FiT[i][j];
}

/* Mooney-Rivlin consistent tangent A_ijkl = dP_ij / dF_kl (mr_compute_tangent_tensor,
 * MooneyRivlin.cuh:106-221: the exact derivative of mr_p, term by term) contracted
 * with the gradient of node a: B[i][k][l] = sum_j A_ijkl ga[j], so that the
 * (a, b) stiffness block is K[i][k] = sum_l B[i][k][l] gb[l] dV. */
static void mr_tangent_a(const double F[3][3], double mu10, double mu01, double kappa, const double ga[3],
                         double B[3][3][3]) {
    double C[3][3] = {{0}}, C2[3][3] = {{0}}, FC[3][3] = {{0}}, FFT[3][3] = {{0}}, FiT[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) {
                C[i][j] += F[k][i] * F[k][j];
                FFT[i][j] += F[i][k] * F[j][k];
            }
    const double I1 = C[0][0] + C[1][1] + C[2][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) C2[i][j] += C[i][k] * C[k][j];
    const double I2 = 0.5 * (I1 * I1 - (C2[0][0] + C2[1][1] + C2[2][2]));
    const double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                     F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                     F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
    double dj = J;
    if (fabs(dj) < 1e-12) dj = (dj >= 0.0) ? 1e-12 : -1e-12;
    const double id = 1.0 / dj;
    FiT[0][0] = (F[1][1] * F[2][2] - F[1][2] * F[2][1]) * id;
    FiT[0][1] = (F[1][2] * F[2][0] - F[1][0] * F[2][2]) * id;
    FiT[0][2] = (F[1][0] * F[2][1] - F[1][1] * F[2][0]) * id;
    FiT[1][0] = (F[0][2] * F[2][1] - F[0][1] * F[2][2]) * id;
    FiT[1][1] = (F[0][0] * F[2][2] - F[0][2] * F[2][0]) * id;
    FiT[1][2] = (F[0][1] * F[2][0] - F[0][0] * F[2][1]) * id;
    FiT[2][0] = (F[0][1] * F[1][2] - F[0][2] * F[1][1]) * id;
    FiT[2][1] = (F[0][2] * F[1][0] - F[0][0] * F[1][2]) * id;
    FiT[2][2] = (F[0][0] * F[1][1] - F[0][1] * F[1][0]) * id;
    const double j13 = cbrt(J);
    const double jm23 = 1.0 / (j13 * j13), jm43 = jm23 * jm23;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) FC[i][j] += F[i][k] * C[k][j];
    const double t1 = 2.0 * mu10 * jm23, t2 = 2.0 * mu01 * jm43, t3 = kappa * (J - 1.0) * J;
    double T1[3][3], T2[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T1[i][j] = F[i][j] - (I1 / 3.0) * FiT[i][j];
            T2[i][j] = I1 * F[i][j] - FC[i][j] - (2.0 * I2 / 3.0) * FiT[i][j];
        }
    const double dt3c = kappa * (2.0 * J - 1.0) * J;
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) {
                double s = 0.0;
                for (int j = 0; j < 3; ++j) {
                    const double dik = (i == k) ? 1.0 : 0.0, djl = (j == l) ? 1.0 : 0.0;
                    const double dFiT = -FiT[i][l] * FiT[k][j];
                    const double dT1 = dik * djl - (2.0 / 3.0) * F[k][l] * FiT[i][j] + (I1 / 3.0) * FiT[i][l] * FiT[k][j];
                    const double dT2 = 2.0 * F[k][l] * F[i][j] + I1 * dik * djl -
                                       (dik * C[l][j] + F[i][l] * F[k][j] + djl * FFT[i][k]) -
                                       (4.0 / 3.0) * (I1 * F[k][l] - FC[k][l]) * FiT[i][j] +
                                       (2.0 * I2 / 3.0) * FiT[i][l] * FiT[k][j];
                    const double A = (-2.0 / 3.0) * t1 * FiT[k][l] * T1[i][j] + t1 * dT1 +
                                     (-4.0 / 3.0) * t2 * FiT[k][l] * T2[i][j] + t2 * dT2 +
                                     dt3c * FiT[k][l] * FiT[i][j] + t3 * dFiT;
                    s += A * ga[j];
                }
                B[i][k][l] = s;
            }
}

/* compute_p for one (e,q): F, SVK P (SVK.cuh:17-39 via the trFtF/FFtF path) or
 * the Mooney-Rivlin P (FEAT10DataFunc.cuh:273-278), plus the optional
 * Kelvin-Voigt term (FEAT10DataFunc.cuh:130-231). */
static void qp_stress(int npe, const double X[][3], const double* gq, double lambda, double mu, double eta,
                      double lamd, const double V[][3], double F[3][3], double P[3][3], double Fd[3][3],
                      double Pv[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) F[i][j] = 0.0;
    for (int a = 0; a < npe; ++a)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) F[i][j] += X[a][i] * gq[a + npe * j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            Fd[i][j] = 0.0;
            Pv[i][j] = 0.0;
        }
    if (V && (eta != 0.0 || lamd != 0.0)) {
        for (int a = 0; a < npe; ++a)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) Fd[i][j] += V[a][i] * gq[a + npe * j];
        double A[3][3] = {{0}}, B[3][3] = {{0}}, Ed[3][3], S[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) A[i][j] += Fd[k][i] * F[k][j];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) B[i][j] += F[k][i] * Fd[k][j];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Ed[i][j] = 0.5 * (A[i][j] + B[i][j]);
        double tr = Ed[0][0] + Ed[1][1] + Ed[2][2];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) S[i][j] = 2.0 * eta * Ed[i][j] + lamd * tr * (i == j ? 1.0 : 0.0);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) Pv[i][j] += F[i][k] * S[k][j];
    }
    double FtF[3][3] = {{0}}, FFt[3][3] = {{0}}, FFtF[3][3] = {{0}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) FtF[i][j] += F[k][i] * F[k][j];
    double tr = FtF[0][0] + FtF[1][1] + FtF[2][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) FFt[i][j] += F[i][k] * F[j][k];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) FFtF[i][j] += FFt[i][k] * F[k][j];
    if (g_material == 1) {
        double Pm[3][3];
        mr_p(F, g_mu10, g_mu01, g_kappa, Pm);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) P[i][j] = Pm[i][j] + Pv[i][j];
        return;
    }
    double lf = lambda * (0.5 * tr - 1.5);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) P[i][j] = lf * F[i][j] + mu * (FFtF[i][j] - F[i][j]) + Pv[i][j];
}

static void gather_elem(int npe, int E, int e, const int* conn, const double* x, const double* y, const double* z,
                        double X[][3]) {
    for (int a = 0; a < npe; ++a) {
        int n = conn[e + a * E];
        X[a][0] = x[n];
        X[a][1] = y[n];
        X[a][2] = z[n];
    }
}

static void gather_vel(int npe, int E, int e, const int* conn, const double* v, double V[][3]) {
    for (int a = 0; a < npe; ++a) {
        int n = conn[e + a * E];
        V[a][0] = v[3 * n + 0];
        V[a][1] = v[3 * n + 1];
        V[a][2] = v[3 * n + 2];
    }
}

void orc_calc_p(int npe, int nqp, int E, const double* x, const double* y, const double* z, const int* conn,
                const double* grad, double lambda, double mu, double eta_d, double lambda_d, const double* v,
                double* Fo, double* Po, double* Fdo, double* Pvo) {
#pragma omp parallel for schedule(static)
    for (int e = 0; e < E; ++e) {
        double X[10][3], V[10][3];
        gather_elem(npe, E, e, conn, x, y, z, X);
        if (v) gather_vel(npe, E, e, conn, v, V);
        for (int q = 0; q < nqp; ++q) {
            double F[3][3], P[3][3], Fd[3][3], Pv[3][3];
            qp_stress(npe, (const double(*)[3])X, grad + (size_t)(e * nqp + q) * npe * 3, lambda, mu, eta_d,
                      lambda_d, v ? (const double(*)[3])V : NULL, F, P, Fd, Pv);
            size_t o = (size_t)(e * nqp + q) * 9;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    if (Fo) Fo[o + i + 3 * j] = F[i][j];
                    if (Po) Po[o + i + 3 * j] = P[i][j];
                    if (Fdo) Fdo[o + i + 3 * j] = Fd[i][j];
                    if (Pvo) Pvo[o + i + 3 * j] = Pv[i][j];
                }
        }
    }
}

/* Element nodal forces from P: fe[a][i] = sum_q (sum_j P_ij g_aj) * detJ*w_q. */
static void elem_force_from_p(int npe, int nqp, const double* Pe /* nqp*9, ref layout */, const double* ge,
                              const double* dj, const double* qw, double fe[][3]) {
    for (int a = 0; a < npe; ++a) {
        double fn[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < nqp; ++q) {
            const double* P = Pe + q * 9;
            const double* g = ge + (size_t)q * npe * 3;
            double dV = dj[q] * qw[q];
            for (int i = 0; i < 3; ++i) {
                double fc = 0.0;
                for (int j = 0; j < 3; ++j) fc += P[i + 3 * j] * g[a + npe * j];
                fn[i] += fc * dV;
            }
        }
        fe[a][0] = fn[0];
        fe[a][1] = fn[1];
        fe[a][2] = fn[2];
    }
}

void orc_internal_force(int npe, int nqp, int E, int N, const int* conn, const double* grad, const double* detJ,
                        const double* qw, const double* P, double* f_int) {
    (void)N;
    double* fe = (double*)malloc(sizeof(double) * (size_t)E * npe * 3);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < E; ++e)
        elem_force_from_p(npe, nqp, P + (size_t)e * nqp * 9, grad + (size_t)e * nqp * npe * 3, detJ + (size_t)e * nqp,
                          qw, (double(*)[3])(fe + (size_t)e * npe * 3));
    for (int e = 0; e < E; ++e)
        for (int a = 0; a < npe; ++a) {
            int n = conn[e + a * E];
            for (int i = 0; i < 3; ++i) f_int[3 * n + i] += fe[((size_t)e * npe + a) * 3 + i];
        }
    free(fe);
}

void orc_force(int npe, int nqp, int E, int N, const double* x, const double* y, const double* z, const int* conn,
               const double* grad, const double* detJ, const double* qw, double lambda, double mu, double eta_d,
               double lambda_d, const double* v, double* f_int) {
    double* fe = (double*)malloc(sizeof(double) * (size_t)E * npe * 3);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < E; ++e) {
        double X[10][3], V[10][3], Pe[5 * 9];
        gather_elem(npe, E, e, conn, x, y, z, X);
        if (v) gather_vel(npe, E, e, conn, v, V);
        for (int q = 0; q < nqp; ++q) {
            double F[3][3], P[3][3], Fd[3][3], Pv[3][3];
            qp_stress(npe, (const double(*)[3])X, grad + (size_t)(e * nqp + q) * npe * 3, lambda, mu, eta_d,
                      lambda_d, v ? (const double(*)[3])V : NULL, F, P, Fd, Pv);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) Pe[q * 9 + i + 3 * j] = P[i][j];
        }
        elem_force_from_p(npe, nqp, Pe, grad + (size_t)e * nqp * npe * 3, detJ + (size_t)e * nqp, qw,
                          (double(*)[3])(fe + (size_t)e * npe * 3));
    }
    memset(f_int, 0, sizeof(double) * 3 * (size_t)N);
    for (int e = 0; e < E; ++e)
        for (int a = 0; a < npe; ++a) {
            int n = conn[e + a * E];
            for (int i = 0; i < 3; ++i) f_int[3 * n + i] += fe[((size_t)e * npe + a) * 3 + i];
        }
    free(fe);
}

/* ============================================================== CSR patterns */

static int cmp_int(const void* a, const void* b) {
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* node -> element incidence (cpu_utils.cc:97-109 semantics, CSR form). */
static void build_incidence(int npe, int E, int N, const int* conn, int** off_out, int** ent_out) {
    int* off = (int*)calloc((size_t)N + 1, sizeof(int));
    for (int e = 0; e < E; ++e)
        for (int a = 0; a < npe; ++a) off[conn[e + a * E] + 1]++;
    for (int i = 0; i < N; ++i) off[i + 1] += off[i];
    int* pos = (int*)malloc(sizeof(int) * (size_t)N);
    memcpy(pos, off, sizeof(int) * (size_t)N);
    int* ent = (int*)malloc(sizeof(int) * (size_t)E * npe);
    for (int e = 0; e < E; ++e)
        for (int a = 0; a < npe; ++a) ent[pos[conn[e + a * E]]++] = e;
    free(pos);
    *off_out = off;
    *ent_out = ent;
}

static int row_unique(int npe, int E, const int* conn, const int* ioff, const int* ient, int i, int* buf) {
    int m = 0;
    for (int k = ioff[i]; k < ioff[i + 1]; ++k) {
        int e = ient[k];
        for (int b = 0; b < npe; ++b) buf[m++] = conn[e + b * E];
    }
    qsort(buf, (size_t)m, sizeof(int), cmp_int);
    int u = 0;
    for (int k = 0; k < m; ++k)
        if (u == 0 || buf[k] != buf[u - 1]) buf[u++] = buf[k];
    return u;
}

long long orc_node_pattern(int npe, int E, int N, const int* conn, int* offsets, int* cols) {
    int *ioff, *ient;
    build_incidence(npe, E, N, conn, &ioff, &ient);
    int maxinc = 0;
    for (int i = 0; i < N; ++i)
        if (ioff[i + 1] - ioff[i] > maxinc) maxinc = ioff[i + 1] - ioff[i];
    int* cnt = (int*)malloc(sizeof(int) * (size_t)N);
#pragma omp parallel
    {
        int* buf = (int*)malloc(sizeof(int) * (size_t)(maxinc * npe + 1));
#pragma omp for schedule(dynamic, 1024)
        for (int i = 0; i < N; ++i) cnt[i] = row_unique(npe, E, conn, ioff, ient, i, buf);
        free(buf);
    }
    long long nnz = 0;
    for (int i = 0; i < N; ++i) nnz += cnt[i];
    if (offsets) {
        long long s = 0;
        for (int i = 0; i < N; ++i) {
            offsets[i] = (int)s;
            s += cnt[i];
        }
        offsets[N] = (int)s;
    }
    if (cols && offsets) {
#pragma omp parallel
        {
            int* buf = (int*)malloc(sizeof(int) * (size_t)(maxinc * npe + 1));
#pragma omp for schedule(dynamic, 1024)
            for (int i = 0; i < N; ++i) {
                int u = row_unique(npe, E, conn, ioff, ient, i, buf);
                memcpy(cols + offsets[i], buf, sizeof(int) * (size_t)u);
            }
            free(buf);
        }
    }
    free(cnt);
    free(ioff);
    free(ient);
    return nnz;
}

static int find_col(const int* cols, int b, int e, int target) {
    int l = b, r = e - 1;
    while (l <= r) {
        int m = l + ((r - l) >> 1);
        if (cols[m] == target) return m;
        if (cols[m] < target)
            l = m + 1;
        else
            r = m - 1;
    }
    return -1;
}

static void shape_values(int npe, double xi, double eta, double zeta, double* N) {
    double L[4] = {1.0 - xi - eta - zeta, xi, eta, zeta};
    if (npe == 4) {
        for (int k = 0; k < 4; ++k) N[k] = L[k];
        return;
    }
    static const int edges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
    for (int k = 0; k < 4; ++k) N[k] = L[k] * (2.0 * L[k] - 1.0);
    for (int k = 0; k < 6; ++k) N[k + 4] = 4.0 * L[edges[k][0]] * L[edges[k][1]];
}

void orc_mass_values(int npe, int nqp, int E, int N, const int* conn, const double* detJ, const double* qx,
                     const double* qy, const double* qz, const double* qw, double rho, const int* offsets,
                     const int* cols, double* vals) {
    memset(vals, 0, sizeof(double) * (size_t)offsets[N]);
    double Nq[5][10];
    for (int q = 0; q < nqp; ++q) shape_values(npe, qx[q], qy[q], qz[q], Nq[q]);
    for (int e = 0; e < E; ++e)
        for (int i = 0; i < npe; ++i) {
            int ig = conn[e + i * E];
            for (int j = 0; j < npe; ++j) {
                int jg = conn[e + j * E];
                double m = 0.0;
                for (int q = 0; q < nqp; ++q) m += rho * Nq[q][i] * Nq[q][j] * detJ[e * nqp + q] * qw[q];
                int p = find_col(cols, offsets[ig], offsets[ig + 1], jg);
                if (p >= 0) vals[p] += m;
            }
        }
}

long long orc_dof_pattern(int N, const int* noff, const int* ncol, int* offsets, int* cols) {
    long long nnz = 9LL * (long long)noff[N];
    if (offsets) {
        long long s = 0;
        for (int i = 0; i < N; ++i) {
            int len = 3 * (noff[i + 1] - noff[i]);
            for (int d = 0; d < 3; ++d) {
                offsets[3 * i + d] = (int)s;
                s += len;
            }
        }
        offsets[3 * N] = (int)s;
    }
    if (cols && offsets) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < N; ++i)
            for (int d = 0; d < 3; ++d) {
                int o = offsets[3 * i + d];
                for (int k = noff[i]; k < noff[i + 1]; ++k)
                    for (int e = 0; e < 3; ++e) cols[o++] = 3 * ncol[k] + e;
            }
    }
    return nnz;
}

/* ================================================================ stiffness */

/* Row-parallel: node row i gathers, for each incident (element, slot a) in
 * element order, the blocks (a, b) of that element's tangent.  Each K entry is
 * owned by one row, so the OpenMP loop needs no atomics. */
void orc_stiffness_assemble(int npe, int nqp, int E, int N, const double* x, const double* y, const double* z,
                            const int* conn, const double* grad, const double* detJ, const double* qw, double lambda,
                            double mu, double eta_d, double lambda_d, double h, const int* offsets, const int* cols,
                            double* vals) {
    int* ioff = (int*)calloc((size_t)N + 1, sizeof(int));
    for (int e = 0; e < E; ++e)
        for (int a = 0; a < npe; ++a) ioff[conn[e + a * E] + 1]++;
    for (int i = 0; i < N; ++i) ioff[i + 1] += ioff[i];
    int* pos = (int*)malloc(sizeof(int) * (size_t)N);
    memcpy(pos, ioff, sizeof(int) * (size_t)N);
    int* ie = (int*)malloc(sizeof(int) * (size_t)E * npe);
    int* ia = (int*)malloc(sizeof(int) * (size_t)E * npe);
    for (int e = 0; e < E; ++e)
        for (int a = 0; a < npe; ++a) {
            int n = conn[e + a * E];
            ie[pos[n]] = e;
            ia[pos[n]] = a;
            pos[n]++;
        }
    free(pos);
    const int visc = (eta_d != 0.0 || lambda_d != 0.0);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < N; ++i) {
        for (int k = ioff[i]; k < ioff[i + 1]; ++k) {
            const int e = ie[k], a = ia[k];
            double X[10][3];
            gather_elem(npe, E, e, conn, x, y, z, X);
            for (int q = 0; q < nqp; ++q) {
                const double* gq = grad + (size_t)(e * nqp + q) * npe * 3;
                double g[10][3];
                for (int b = 0; b < npe; ++b)
                    for (int j = 0; j < 3; ++j) g[b][j] = gq[b + npe * j];
                double F[3][3] = {{0}};
                for (int b = 0; b < npe; ++b)
                    for (int r = 0; r < 3; ++r)
                        for (int j = 0; j < 3; ++j) F[r][j] += X[b][r] * g[b][j];
                double C[3][3] = {{0}}, FFT[3][3] = {{0}};
                for (int r = 0; r < 3; ++r)
                    for (int j = 0; j < 3; ++j)
                        for (int m = 0; m < 3; ++m) C[r][j] += F[m][r] * F[m][j];
                double trE = 0.5 * ((C[0][0] + C[1][1] + C[2][2]) - 3.0);
                for (int r = 0; r < 3; ++r)
                    for (int j = 0; j < 3; ++j)
                        for (int m = 0; m < 3; ++m) FFT[r][j] += F[r][m] * F[j][m];
                double Fh[10][3];
                for (int b = 0; b < npe; ++b)
                    for (int r = 0; r < 3; ++r) {
                        Fh[b][r] = 0.0;
                        for (int c = 0; c < 3; ++c) Fh[b][r] += F[r][c] * g[b][c];
                    }
                const double dV = detJ[e * nqp + q] * qw[q];
                double Bmr[3][3][3];
                if (g_material == 1) mr_tangent_a(F, g_mu10, g_mu01, g_kappa, g[a], Bmr);
                for (int b = 0; b < npe; ++b) {
                    const int nb = conn[e + b * E];
                    /* svk_compute_tangent_block(Fh_a, Fh_b, ...) (SVK.cuh:41-67) */
                    const double hij = g[b][0] * g[a][0] + g[b][1] * g[a][1] + g[b][2] * g[a][2];
                    const double fdf = Fh[b][0] * Fh[a][0] + Fh[b][1] * Fh[a][1] + Fh[b][2] * Fh[a][2];
                    const double hd = g[a][0] * g[b][0] + g[a][1] * g[b][1] + g[a][2] * g[b][2];
                    for (int d = 0; d < 3; ++d) {
                        const int row = 3 * i + d;
                        for (int ee = 0; ee < 3; ++ee) {
                            const int p = find_col(cols, offsets[row], offsets[row + 1], 3 * nb + ee);
                            if (p < 0) continue;
                            const double delta = (d == ee) ? 1.0 : 0.0;
                            if (g_material == 1) {
                                /* the Mooney-Rivlin block, FEAT10DataFunc.cuh:607-640 */
                                const double kb = Bmr[d][ee][0] * g[b][0] + Bmr[d][ee][1] * g[b][1] +
                                                  Bmr[d][ee][2] * g[b][2];
                                vals[p] += h * (kb * dV);
                            } else {
                                const double A = lambda * Fh[a][d] * Fh[b][ee];
                                const double B = lambda * trE * hij * delta;
                                const double C1 = mu * fdf * delta;
                                const double D = mu * Fh[b][d] * Fh[a][ee];
                                const double Et = mu * hij * FFT[d][ee];
                                const double Ft = -mu * hij * delta;
                                vals[p] += h * ((A + B + C1 + D + Et + Ft) * dV);
                            }
                            /* Kelvin-Voigt block, FEAT10DataFunc.cuh:686-768 (not scaled by h) */
                            if (visc)
                                vals[p] += (eta_d * (Fh[b][d] * Fh[a][ee]) + eta_d * FFT[d][ee] * hd +
                                            lambda_d * (Fh[a][d] * Fh[b][ee])) *
                                           dV;
                        }
                    }
                }
            }
        }
    }
    free(ioff);
    free(ie);
    free(ia);
}

void orc_apply_bcs(int n_dof, int n_fixed, const int* fixed, const int* offsets, const int* cols, double* vals,
                   double* f) {
    char* isf = (char*)calloc((size_t)n_dof, 1);
    for (int k = 0; k < n_fixed; ++k)
        for (int d = 0; d < 3; ++d) isf[3 * fixed[k] + d] = 1;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n_dof; ++r) {
        if (isf[r]) {
            for (int k = offsets[r]; k < offsets[r + 1]; ++k) vals[k] = (cols[k] == r) ? 1.0 : 0.0;
            f[r] = 0.0;
        } else {
            for (int k = offsets[r]; k < offsets[r + 1]; ++k)
                if (isf[cols[k]]) vals[k] = 0.0;
        }
    }
    free(isf);
}

/* ======================================================================= CG */

void orc_spmv(int n, const int* offsets, const int* cols, const double* vals, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; ++r) {
        double s = 0.0;
        for (int k = offsets[r]; k < offsets[r + 1]; ++k) s += vals[k] * x[cols[k]];
        y[r] = s;
    }
}

/* Dot product with a fixed blocked summation order (independent of threads). */
#define ORC_DOT_BLOCK 4096
static double dot(int n, const double* a, const double* b) {
    int nb = (n + ORC_DOT_BLOCK - 1) / ORC_DOT_BLOCK;
    double* part = (double*)malloc(sizeof(double) * (size_t)(nb > 0 ? nb : 1));
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nb; ++k) {
        double s = 0.0;
        int lo = k * ORC_DOT_BLOCK, hi = lo + ORC_DOT_BLOCK < n ? lo + ORC_DOT_BLOCK : n;
        for (int i = lo; i < hi; ++i) s += a[i] * b[i];
        part[k] = s;
    }
    double s = 0.0;
    for (int k = 0; k < nb; ++k) s += part[k];
    free(part);
    return s;
}

int orc_cg(int n, const int* offsets, const int* cols, const double* vals, const double* f, double* u, double tol,
           int max_iter, int* iters, double* rel_res) {
    double* r = (double*)malloc(sizeof(double) * (size_t)n);
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    double* Kp = (double*)malloc(sizeof(double) * (size_t)n);
    int ret = 0;
    memset(u, 0, sizeof(double) * (size_t)n);
    memcpy(r, f, sizeof(double) * (size_t)n);
    memcpy(p, f, sizeof(double) * (size_t)n);
    double rr0 = dot(n, r, r);
    if (rr0 == 0.0) {
        *iters = 0;
        *rel_res = 0.0;
        goto done;
    }
    double rr = rr0;
    *iters = max_iter;
    *rel_res = 1.0;
    for (int it = 0; it < max_iter; ++it) {
        orc_spmv(n, offsets, cols, vals, p, Kp);
        double pKp = dot(n, p, Kp);
        if (pKp <= 0.0) {
            ret = 1;
            break;
        }
        double alpha = rr / pKp;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            u[i] += alpha * p[i];
            r[i] -= alpha * Kp[i];
        }
        double rrn = dot(n, r, r);
        double rel = sqrt(rrn / rr0);
        if (rel < tol) {
            *iters = it + 1;
            *rel_res = rel;
            break;
        }
        double beta = rrn / rr;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
        rr = rrn;
        if (it == max_iter - 1) {
            *iters = max_iter;
            *rel_res = rel;
        }
    }
done:
    free(r);
    free(p);
    free(Kp);
    return ret;
}

/* ================================================================= solvers */

void orc_constraint(const orc_problem* pb, double* c) {
    for (int k = 0; k < pb->n_fixed; ++k) {
        int n = pb->fixed[k];
        c[3 * k + 0] = pb->x[n] - pb->xj[n];
        c[3 * k + 1] = pb->y[n] - pb->yj[n];
        c[3 * k + 2] = pb->z[n] - pb->zj[n];
    }
}

void orc_grad_L(const orc_problem* pb, const double* f_int, const double* c, const double* lam, const double* vg,
                const double* vp, double dt, double rho, double* g) {
    const int N = pb->N;
    const double inv_dt = 1.0 / dt;
    /* J^T rows: constraint k acts on DOF 3*fixed[k/3] + k%3 (FEAT10Data.cu:510-562). */
    int nc = 3 * pb->n_fixed;
    int* cnt = (int*)calloc((size_t)3 * N + 1, sizeof(int));
    for (int k = 0; k < nc; ++k) cnt[3 * pb->fixed[k / 3] + k % 3 + 1]++;
    for (int i = 0; i < 3 * N; ++i) cnt[i + 1] += cnt[i];
    int* pos = (int*)malloc(sizeof(int) * (size_t)3 * N + 1);
    memcpy(pos, cnt, sizeof(int) * (size_t)3 * N);
    int* ent = (int*)malloc(sizeof(int) * (size_t)(nc > 0 ? nc : 1));
    for (int k = 0; k < nc; ++k) ent[pos[3 * pb->fixed[k / 3] + k % 3]++] = k;
#pragma omp parallel for schedule(static)
    for (int t = 0; t < 3 * N; ++t) {
        int ni = t / 3, di = t % 3;
        double res = 0.0;
        for (int k = pb->m_off[ni]; k < pb->m_off[ni + 1]; ++k) {
            int tj = pb->m_col[k] * 3 + di;
            double vd = vg[tj] - vp[tj];
            res += pb->m_val[k] * vd * inv_dt;
        }
        res -= (-f_int[t]);
        res -= pb->f_ext[t];
        for (int k = cnt[t]; k < cnt[t + 1]; ++k) {
            int ci = ent[k];
            res += dt * 1.0 * (lam[ci] + rho * c[ci]);
        }
        g[t] = res;
    }
    free(cnt);
    free(pos);
    free(ent);
}

static void solver_force(const orc_problem* pb, const double* v, double* f_int) {
    orc_force(pb->npe, pb->nqp, pb->E, pb->N, pb->x, pb->y, pb->z, pb->conn, pb->grad, pb->detJ, pb->qw, pb->lambda,
              pb->mu, pb->eta_d, pb->lambda_d, v, f_int);
}

static void set_positions(const orc_problem* pb, const double* xp, const double* yp, const double* zp,
                          const double* v, double dt) {
    for (int i = 0; i < pb->N; ++i) {
        pb->x[i] = xp[i] + dt * v[3 * i + 0];
        pb->y[i] = yp[i] + dt * v[3 * i + 1];
        pb->z[i] = zp[i] + dt * v[3 * i + 2];
    }
}

/* positions after an outer iteration: x_prev + v*dt (operand order as SyncedNesterov.cu:300-307) */
static void set_positions_vdt(const orc_problem* pb, const double* xp, const double* yp, const double* zp,
                              const double* v, double dt) {
    for (int i = 0; i < pb->N; ++i) {
        pb->x[i] = xp[i] + v[3 * i + 0] * dt;
        pb->y[i] = yp[i] + v[3 * i + 1] * dt;
        pb->z[i] = zp[i] + v[3 * i + 2] * dt;
    }
}

static double seq_norm(int n, const double* a) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += a[i] * a[i];
    return sqrt(s);
}

void orc_nesterov_solve(const orc_problem* pb, const orc_nesterov_params* prm, double* vg, double* vp, double* lam,
                        orc_solve_stats* st) {
    const int N = pb->N, n = 3 * N, nc = 3 * pb->n_fixed;
    const double dt = prm->time_step;
    double* xp = (double*)malloc(sizeof(double) * N);
    double* yp = (double*)malloc(sizeof(double) * N);
    double* zp = (double*)malloc(sizeof(double) * N);
    double* vk = (double*)malloc(sizeof(double) * n);
    double* vkm1 = (double*)malloc(sizeof(double) * n);
    double* vnext = (double*)malloc(sizeof(double) * n);
    double* ybuf = (double*)malloc(sizeof(double) * n);
    double* g = (double*)malloc(sizeof(double) * n);
    double* fi = (double*)malloc(sizeof(double) * n);
    double* c = (double*)malloc(sizeof(double) * (nc > 0 ? nc : 1));
    memcpy(xp, pb->x, sizeof(double) * N);
    memcpy(yp, pb->y, sizeof(double) * N);
    memcpy(zp, pb->z, sizeof(double) * N);
    memset(c, 0, sizeof(double) * (nc > 0 ? nc : 1));
    int outer_flag = 0;
    if (st) memset(st, 0, sizeof(*st));
    for (int outer = 0; outer < prm->max_outer; ++outer) {
        if (outer_flag) continue;
        if (st) st->outer_iters++;
        double t = 1.0, t_next = 1.0;
        double prev_norm_g = 0.0, norm_g = 0.0;
        int inner_flag = 0, inner_count = 0;
        for (int i = 0; i < n; ++i) {
            vk[i] = vg[i];
            vkm1[i] = vg[i];
        }
        for (int inner = 0; inner < prm->max_inner; ++inner) {
            if (inner_flag) continue;
            inner_count++;
            t_next = 0.5 * (1.0 + sqrt(1.0 + 4.0 * t * t));
            double beta = (t - 1.0) / t_next;
            for (int i = 0; i < n; ++i) {
                ybuf[i] = vk[i] + beta * (vk[i] - vkm1[i]);
                vg[i] = ybuf[i];
            }
            set_positions(pb, xp, yp, zp, vg, dt);
            solver_force(pb, vg, fi);
            orc_constraint(pb, c);
            orc_grad_L(pb, fi, c, lam, vg, vp, dt, prm->rho, g);
            norm_g = seq_norm(n, g);
            if (inner > 0 && fabs(norm_g - prev_norm_g) < prm->inner_tol) inner_flag = 1;
            for (int i = 0; i < n; ++i) vnext[i] = ybuf[i] - prm->alpha * g[i];
            double nvn = seq_norm(n, vnext), nvk = seq_norm(n, vk);
            if (inner > 0 && fabs(nvn - nvk) < prm->inner_tol) inner_flag = 1;
            for (int i = 0; i < n; ++i) {
                vkm1[i] = vk[i];
                vk[i] = vnext[i];
                vg[i] = vnext[i];
            }
            t = t_next;
            prev_norm_g = norm_g;
        }
        if (st) {
            st->inner_iters_total += inner_count;
            st->last_inner_iters = inner_count;
            st->last_norm_g = norm_g;
        }
        memcpy(vp, vg, sizeof(double) * n);
        set_positions_vdt(pb, xp, yp, zp, vg, dt);
        orc_constraint(pb, c);
        for (int i = 0; i < nc; ++i) lam[i] += prm->rho * dt * c[i];
        double nrm = seq_norm(nc, c);
        if (fabs(nrm) < prm->outer_tol) outer_flag = 1;
    }
    set_positions_vdt(pb, xp, yp, zp, vg, dt);
    free(xp); free(yp); free(zp); free(vk); free(vkm1); free(vnext); free(ybuf); free(g); free(fi); free(c);
}

void orc_adamw_solve(const orc_problem* pb, const orc_adamw_params* prm, double* vg, double* vp, double* lam,
                     orc_solve_stats* st) {
    const int N = pb->N, n = 3 * N, nc = 3 * pb->n_fixed;
    const double dt = prm->time_step;
    double* xp = (double*)malloc(sizeof(double) * N);
    double* yp = (double*)malloc(sizeof(double) * N);
    double* zp = (double*)malloc(sizeof(double) * N);
    double* m = (double*)malloc(sizeof(double) * n);
    double* v = (double*)malloc(sizeof(double) * n);
    double* g = (double*)malloc(sizeof(double) * n);
    double* fi = (double*)malloc(sizeof(double) * n);
    double* c = (double*)malloc(sizeof(double) * (nc > 0 ? nc : 1));
    memcpy(xp, pb->x, sizeof(double) * N);
    memcpy(yp, pb->y, sizeof(double) * N);
    memcpy(zp, pb->z, sizeof(double) * N);
    memset(c, 0, sizeof(double) * (nc > 0 ? nc : 1));
    int outer_flag = 0;
    int k_check = prm->convergence_check_interval;
    if (st) memset(st, 0, sizeof(*st));
    for (int outer = 0; outer < prm->max_outer; ++outer) {
        if (outer_flag) continue;
        if (st) st->outer_iters++;
        double lr = prm->lr, t = 1.0;
        double norm_g = 0.0, norm_g0 = -1.0;
        int inner_flag = 0, inner_count = 0;
        for (int i = 0; i < n; ++i) {
            m[i] = 0.0;
            v[i] = 0.0;
            g[i] = 0.0;
        }
        for (int inner = 0; inner < prm->max_inner; ++inner) {
            if (inner_flag) continue;
            inner_count++;
            /* SyncedAdamW.cu:156-171: every thread advances lr and t identically. */
            lr = lr * prm->lr_decay;
            t += 1;
            const double b1t = 1 - pow(prm->beta1, t), b2t = 1 - pow(prm->beta2, t);
            for (int i = 0; i < n; ++i) {
                double gi = g[i];
                m[i] = prm->beta1 * m[i] + (1 - prm->beta1) * gi;
                v[i] = prm->beta2 * v[i] + (1 - prm->beta2) * gi * gi;
                double mh = m[i] / b1t;
                double vh = v[i] / b2t;
                vg[i] = vg[i] - lr * (mh / (sqrt(vh) + prm->eps) + prm->weight_decay * vg[i]);
            }
            set_positions(pb, xp, yp, zp, vg, dt);
            solver_force(pb, vg, fi);
            orc_constraint(pb, c);
            orc_grad_L(pb, fi, c, lam, vg, vp, dt, prm->rho, g);
            if (k_check > 0 && inner % k_check == 0) {
                norm_g = seq_norm(n, g);
                if (norm_g0 < 0.0) norm_g0 = norm_g;
                double nv = seq_norm(n, vg);
                double tol_abs = prm->inner_tol * (1.0 + nv);
                double tol_rel = (prm->inner_rtol > 0.0 && norm_g0 > 0.0) ? (prm->inner_rtol * norm_g0) : 0.0;
                if (norm_g <= tol_abs || (tol_rel > 0.0 && norm_g <= tol_rel)) inner_flag = 1;
            }
        }
        if (st) {
            st->inner_iters_total += inner_count;
            st->last_inner_iters = inner_count;
            st->last_norm_g = norm_g;
        }
        memcpy(vp, vg, sizeof(double) * n);
        set_positions_vdt(pb, xp, yp, zp, vg, dt);
        orc_constraint(pb, c);
        for (int i = 0; i < nc; ++i) lam[i] += prm->rho * dt * c[i];
        double nrm = seq_norm(nc, c);
        if (nrm < prm->outer_tol) outer_flag = 1;
    }
    set_positions_vdt(pb, xp, yp, zp, vg, dt);
    free(xp); free(yp); free(zp); free(m); free(v); free(g); free(fi); free(c);
}

void orc_adamw_nocoop_solve(const orc_problem* pb, const orc_adamw_params* prm, double* vg, double* vp, double* lam,
                            orc_solve_stats* st) {
    const int N = pb->N, n = 3 * N, nc = 3 * pb->n_fixed;
    const double dt = prm->time_step;
    double* xp = (double*)malloc(sizeof(double) * N);
    double* yp = (double*)malloc(sizeof(double) * N);
    double* zp = (double*)malloc(sizeof(double) * N);
    double* m = (double*)malloc(sizeof(double) * n);
    double* v = (double*)malloc(sizeof(double) * n);
    double* g = (double*)malloc(sizeof(double) * n);
    double* fi = (double*)malloc(sizeof(double) * n);
    double* c = (double*)malloc(sizeof(double) * (nc > 0 ? nc : 1));
    memcpy(xp, pb->x, sizeof(double) * N);
    memcpy(yp, pb->y, sizeof(double) * N);
    memcpy(zp, pb->z, sizeof(double) * N);
    memset(c, 0, sizeof(double) * (nc > 0 ? nc : 1));
    int k_check = prm->convergence_check_interval <= 0 ? 1 : prm->convergence_check_interval;
    int eff_outer = (nc == 0) ? 1 : prm->max_outer; /* SyncedAdamWNocoop.cu:298-301 */
    int outer_flag = 0;
    if (st) memset(st, 0, sizeof(*st));
    for (int outer = 0; outer < eff_outer; ++outer) {
        if (outer_flag) break;
        if (st) st->outer_iters++;
        for (int i = 0; i < n; ++i) {
            g[i] = 0.0;
            m[i] = 0.0;
            v[i] = 0.0;
        }
        int inner_flag = 0, inner_count = 0;
        double norm_g0 = -1.0, norm_g = 0.0;
        for (int inner = 0; inner < prm->max_inner; ++inner) {
            if (inner_flag) break;
            inner_count++;
            double lr_cur = prm->lr * pow(prm->lr_decay, inner + 1);
            double tc = (double)(inner + 2);
            double i1 = 1.0 / (1.0 - pow(prm->beta1, tc));
            double i2 = 1.0 / (1.0 - pow(prm->beta2, tc));
            for (int i = 0; i < n; ++i) {
                double gi = g[i];
                double mt = prm->beta1 * m[i] + (1.0 - prm->beta1) * gi;
                double vt = prm->beta2 * v[i] + (1.0 - prm->beta2) * gi * gi;
                double mh = mt * i1, vh = vt * i2;
                double yv = vg[i] - lr_cur * (mh / (sqrt(vh) + prm->eps) + prm->weight_decay * vg[i]);
                m[i] = mt;
                v[i] = vt;
                vg[i] = yv;
            }
            set_positions(pb, xp, yp, zp, vg, dt);
            solver_force(pb, vg, fi);
            if (nc > 0) orc_constraint(pb, c);
            orc_grad_L(pb, fi, c, lam, vg, vp, dt, prm->rho, g);
            if (inner % k_check == 0) {
                norm_g = seq_norm(n, g);
                double nv = seq_norm(n, vg);
                if (norm_g0 < 0.0) norm_g0 = norm_g;
                double tol_abs = prm->inner_tol * (1.0 + nv);
                double tol_rel = (prm->inner_rtol > 0.0 && norm_g0 > 0.0) ? (prm->inner_rtol * norm_g0) : 0.0;
                if (norm_g <= tol_abs || (tol_rel > 0.0 && norm_g <= tol_rel)) inner_flag = 1;
            }
        }
        if (st) {
            st->inner_iters_total += inner_count;
            st->last_inner_iters = inner_count;
            st->last_norm_g = norm_g;
        }
        memcpy(vp, vg, sizeof(double) * n);
        /* adamw_update_positions_from_prev_kernel: x_prev + dt*v (SyncedAdamWNocoop.cu:178-186). */
        set_positions(pb, xp, yp, zp, vg, dt);
        if (nc > 0) {
            orc_constraint(pb, c);
            for (int i = 0; i < nc; ++i) lam[i] += prm->rho * dt * c[i];
            double nrm = seq_norm(nc, c);
            if (nrm < prm->outer_tol && inner_flag) outer_flag = 1;
        }
    }
    set_positions(pb, xp, yp, zp, vg, dt);
    free(xp); free(yp); free(zp); free(m); free(v); free(g); free(fi); free(c);
}

double orc_static_residual(const orc_problem* pb) {
    const int N = pb->N, n = 3 * N;
    double* fi = (double*)malloc(sizeof(double) * n);
    char* isf = (char*)calloc((size_t)N, 1);
    for (int k = 0; k < pb->n_fixed; ++k) isf[pb->fixed[k]] = 1;
    solver_force(pb, NULL, fi);
    double rr = 0.0, ff = 0.0;
    for (int i = 0; i < n; ++i) {
        ff += pb->f_ext[i] * pb->f_ext[i];
        if (!isf[i / 3]) {
            double r = fi[i] - pb->f_ext[i];
            rr += r * r;
        }
    }
    free(fi);
    free(isf);
    return ff > 0.0 ? sqrt(rr / ff) : sqrt(rr);
}
