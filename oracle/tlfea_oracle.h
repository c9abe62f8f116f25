/*
 * tlfea_oracle.h -- CPU restatement of the TLFEA hot path (TEST INFRASTRUCTURE).
 *
 * This library is the parity checker for the CUDA path in tlfea_b200/.  Only
 * the test suite, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it; the product path never calls it and has no CPU fallback.
 *
 * Every routine restates, in plain FP64 C, one step of the reference
 * (Ruochun/TLFEA) and cites the file:line it follows.  Array layouts are the
 * reference's device layouts so results compare element by element:
 *   conn(e,a)          conn[e + a*E]                     (FEAT10Data.cuh:41-43, column-major Eigen)
 *   grad_N(e,q)(a,j)   grad[(e*QP+q)*NPE*3 + a + NPE*j]  (FEAT10Data.cuh:45-51)
 *   F,P(e,q)(i,j)      F[(e*QP+q)*9 + i + 3*j]           (FEAT10Data.cuh:113-127)
 *   detJ(e,q)          detJ[e*QP+q]
 *   nodal vectors      SoA x/y/z (length N); forces/velocities interleaved [3*node+d]
 *
 * Parity status: pinned to the reference's own CUDA build.  The reference ships no
 * golden vectors for this path, and its own build system needs Eigen3 and the
 * un-vendored MoPhiEssentials submodule; oracle/build_ref.py compiles its unchanged
 * element and solver sources for sm_100a against project-written stand-ins for those
 * two headers (oracle/refshim), and tests/golden/make_ref_fixtures.py ran that build
 * on a B200 to write tests/golden/ref_*.npz (geometry, mass, forces, P, stiffness,
 * CG, SyncedNesterov / SyncedAdamW trajectories, constraint arrays).
 * tests/test_ref_fixtures.py checks this restatement against those fixtures; the
 * analytic known-answer tests (rigid motion, patch tests, mass = rho*V, stiffness
 * rigid modes and symmetry, CG vs a direct solve) stay beside them.
 */
#ifndef TLFEA_ORACLE_H
#define TLFEA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- meshes */

/* Structured box mesh: nx*ny*nz hex cells, each Kuhn-split into 6 tets with
 * positive orientation.  order = 10 (TET10, nodes on the half-spacing grid)
 * or 4 (TET4, corner grid).  Node index = (ix*NY + iy)*NZ + iz (x slowest).
 * Returns 0 on success.  conn is column-major (E x NPE). */
int orc_box_counts(int nx, int ny, int nz, int order, int* n_nodes, int* n_elems);
int orc_box_mesh(int nx, int ny, int nz, int order, double lx, double ly, double lz,
                 double* x, double* y, double* z, int* conn);

/* Keast 5-point rule and the TET4 centroid rule (quadrature_utils.h:125-179). */
void orc_quadrature_t10(double* qx, double* qy, double* qz, double* qw);
void orc_quadrature_t4(double* qx, double* qy, double* qz, double* qw);

/* TetGen T10 element order -> reference order (cpu_utils.cc:596-611). */
void orc_remap_tetgen_t10(const int* tetgen10, int* standard10);

/* ------------------------------------------------------ element precompute */

/* a2: dn_du_pre_kernel + solve_3x3_system (FEAT10Data.cu:92-198,
 *     FEAT10DataFunc.cuh:32-84). */
void orc_dndu_pre_t10(int E, const double* x, const double* y, const double* z, const int* conn,
                      const double* qx, const double* qy, const double* qz, double* grad, double* detJ);
/* a3: dn_du_pre_feat4_kernel (FEAT4Data.cu:98-195). */
void orc_dndu_pre_t4(int E, const double* x, const double* y, const double* z, const int* conn,
                     double* grad, double* detJ);

/* a4: compute_p (FEAT10DataFunc.cuh:86-291, FEAT4DataFunc.cuh:33-222) with the
 * SVK law (SVK.cuh:17-39).  v may be NULL (no viscous term, as CalcP does).
 * Outputs may be NULL when not wanted. */
void orc_calc_p(int npe, int nqp, int E, const double* x, const double* y, const double* z, const int* conn,
                const double* grad, double lambda, double mu, double eta_d, double lambda_d, const double* v,
                double* F, double* P, double* Fdot, double* Pvis);

/* a5: compute_internal_force (FEAT10DataFunc.cuh:404-460): f_int += sum_q
 * P(e,q) grad_N_a detJ w_q, ACCUMULATING into f_int (3N) like CalcInternalForce. */
void orc_internal_force(int npe, int nqp, int E, int N, const int* conn, const double* grad,
                        const double* detJ, const double* qw, const double* P, double* f_int);

/* a4+a5 fused, used by the solvers: f_int = internal force at (x, v). */
void orc_force(int npe, int nqp, int E, int N, const double* x, const double* y, const double* z,
               const int* conn, const double* grad, const double* detJ, const double* qw,
               double lambda, double mu, double eta_d, double lambda_d, const double* v, double* f_int);

/* ------------------------------------------------------------ CSR patterns */

/* a7 / a13: node-level pattern (sorted unique (i,j) over element node pairs,
 * FEAT10Data.cu:361-417).  Call with cols=NULL to get nnz only. */
long long orc_node_pattern(int npe, int E, int N, const int* conn, int* offsets, int* cols);

/* a7: mass values (FEAT10Data.cu:200-271, FEAT4Data.cu:197-243). vals zeroed first. */
void orc_mass_values(int npe, int nqp, int E, int N, const int* conn, const double* detJ, const double* qx,
                     const double* qy, const double* qz, const double* qw, double rho, const int* offsets,
                     const int* cols, double* vals);

/* a13: DOF-level pattern: row 3i+d has columns 3j+e for j in node row i
 * (LinearStaticSolver.cu:196-244, 361-416).  cols=NULL -> nnz only. */
long long orc_dof_pattern(int N, const int* node_offsets, const int* node_cols, int* offsets, int* cols);

/* a14: K += h*K_elem (+ viscous C_elem) at the current x
 * (compute_hessian_assemble_csr, FEAT10DataFunc.cuh:512-768; SVK.cuh:41-67).
 * vals is NOT zeroed (AssembleLinearStiffness zeroes it first).  Row-parallel:
 * each node row sums its incident elements' blocks in element order. */
void orc_stiffness_assemble(int npe, int nqp, int E, int N, const double* x, const double* y, const double* z,
                            const int* conn, const double* grad, const double* detJ, const double* qw,
                            double lambda, double mu, double eta_d, double lambda_d, double h,
                            const int* offsets, const int* cols, double* vals);

/* a15: Dirichlet row/column elimination (LinearStaticSolver.cu:268-306). */
void orc_apply_bcs(int n_dof, int n_fixed, const int* fixed_nodes, const int* offsets, const int* cols,
                   double* vals, double* f);

/* a16: unpreconditioned CG (LinearStaticSolver.cu:469-565).  Returns 0, or 1
 * when p.Kp <= 0 aborted the loop. */
int orc_cg(int n, const int* offsets, const int* cols, const double* vals, const double* f, double* u,
           double tol, int max_iter, int* iters, double* rel_res);

/* CSR y = A x (row order, sequential per row). */
void orc_spmv(int n, const int* offsets, const int* cols, const double* vals, const double* x, double* y);

/* ------------------------------------------------------------ the solvers */

/* State shared by the Nesterov / AdamW restatements (the fields of
 * GPU_FEAT10_Data / GPU_FEAT4_Data that the solvers touch). */
typedef struct {
    int npe, nqp, E, N;
    const int* conn;
    const double* grad;
    const double* detJ;
    const double* qw;
    double lambda, mu, eta_d, lambda_d;
    const int* m_off; /* node-level mass CSR */
    const int* m_col;
    const double* m_val;
    int n_fixed;
    const int* fixed;
    double* x; /* current positions, updated in place */
    double* y;
    double* z;
    const double* xj; /* constraint targets (x12_jac) */
    const double* yj;
    const double* zj;
    const double* f_ext;
} orc_problem;

/* Same field order and types as SyncedNesterovParams (SyncedNesterov.cuh:31-35). */
typedef struct {
    double alpha, rho, inner_tol, outer_tol;
    int max_outer, max_inner;
    double time_step;
} orc_nesterov_params;

/* Same field order and types as SyncedAdamWParams (SyncedAdamW.cuh:32-39). */
typedef struct {
    double lr, beta1, beta2, eps, weight_decay, lr_decay;
    double inner_tol, outer_tol, rho;
    int max_outer, max_inner;
    double time_step;
    int convergence_check_interval;
    double inner_rtol;
} orc_adamw_params;

/* Per-call diagnostics (not in the reference; filled by the restatements). */
typedef struct {
    int outer_iters;
    int inner_iters_total;
    int last_inner_iters;
    double last_norm_g;
} orc_solve_stats;

/* a9: solver_grad_L (SyncedNesterov.cu:32-95) for all 3N DOFs.  c and lam have
 * 3*n_fixed entries; f_int must hold the internal force at the current x. */
void orc_grad_L(const orc_problem* pb, const double* f_int, const double* c, const double* lam,
                const double* v_guess, const double* v_prev, double dt, double rho, double* g);

/* a8: c = x(fixed) - x_jac(fixed) (FEAT10DataFunc.cuh:470-481). */
void orc_constraint(const orc_problem* pb, double* c);

/* a10: one SyncedNesterovSolver::Solve() (SyncedNesterov.cu:97-360). */
void orc_nesterov_solve(const orc_problem* pb, const orc_nesterov_params* prm, double* v_guess, double* v_prev,
                        double* lam, orc_solve_stats* st);

/* a11: one SyncedAdamWSolver::Solve() (SyncedAdamW.cu:99-344). */
void orc_adamw_solve(const orc_problem* pb, const orc_adamw_params* prm, double* v_guess, double* v_prev,
                     double* lam, orc_solve_stats* st);

/* a12: one SyncedAdamWNocoopSolver::Solve() (SyncedAdamWNocoop.cu:255-458). */
void orc_adamw_nocoop_solve(const orc_problem* pb, const orc_adamw_params* prm, double* v_guess, double* v_prev,
                            double* lam, orc_solve_stats* st);

/* a19(i): relative static residual ||(f_int - f_ext)_free|| / ||f_ext|| at the
 * current positions (fixed nodes' DOFs excluded). */
double orc_static_residual(const orc_problem* pb);

/* Threads used by the OpenMP loops (0 = library default). */
void orc_set_threads(int n);
/* Material of the stress routines: 0 = SVK (default), 1 = Mooney-Rivlin(mu10, mu01, kappa). */
void orc_set_material(int model, double mu10, double mu01, double kappa);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
