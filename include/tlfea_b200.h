/*
 * tlfea_b200.h -- C ABI of the B200 (sm_100a) TLFEA hot path.
 *
 * Plain pointers, sizes and int status codes: no C++ types, no exceptions.
 * Each entry point replaces one method of the reference's class API
 * (Ruochun/TLFEA, paths relative to its src/); the C++ classes in
 * include/tlfea/ and the Python classes in tlfea_b200/ forward to these.
 *
 * Conventions
 *   - Host arrays are FP64 (Real = double, types.h:19) and int32.
 *   - Connectivity is column-major E x NPE (Eigen MatrixXi::data(),
 *     FEAT10Data.cuh:41-43): conn[e + a*E].
 *   - Nodal vectors are SoA x/y/z (length N); forces and velocities are
 *     interleaved [3*node + d] (FEAT10Data.cuh:147-177).
 *   - Every call is synchronous with respect to the host unless noted, like
 *     the reference (cudaDeviceSynchronize after each launch).  Work runs on
 *     the handle's stream (default: the legacy default stream).
 *   - A handle is not thread-safe (the reference is single-threaded, device 0;
 *     here the device current at create time is used for the handle's life).
 */
#ifndef TLFEA_B200_H
#define TLFEA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (the reference logs with MOPHI_ERROR and returns,
 * FEAT10Data.cuh:426-429; here the condition is returned instead). */
enum {
    TLFEA_OK = 0,
    TLFEA_INVALID_ARG = 1,
    TLFEA_NOT_SETUP = 2,
    TLFEA_SIZE_MISMATCH = 3,
    TLFEA_CUDA_ERROR = 4,
    TLFEA_NO_CONVERGENCE = 5,
    TLFEA_BUDGET_EXCEEDED = 6,
    TLFEA_NONFINITE = 7,
    TLFEA_UNSUPPORTED = 8,
    TLFEA_ALREADY_SETUP = 9,
    TLFEA_NO_CUDA_DEVICE = 10
};

/* ElementType values of ElementBase.h:22 (TYPE_3243, TYPE_3443, TYPE_T10, TYPE_T4). */
enum { TLFEA_TYPE_T10 = 2, TLFEA_TYPE_T4 = 3 };

/* MaterialModel values of MaterialModel.cuh:16-19. */
enum { TLFEA_MATERIAL_SVK = 0, TLFEA_MATERIAL_MOONEY_RIVLIN = 1 };

/* Force precision of the fused element kernel (new, no reference counterpart). */
enum { TLFEA_PRECISION_FP64 = 0, TLFEA_PRECISION_FP32 = 1 };

typedef struct tlfea_element_s* tlfea_element;
typedef struct tlfea_solver_s* tlfea_solver;

/* Same field order and types as SyncedNesterovParams (SyncedNesterov.cuh:31-35). */
typedef struct {
    double alpha, rho, inner_tol, outer_tol;
    int max_outer, max_inner;
    double time_step;
} tlfea_nesterov_params;

/* Same field order and types as SyncedAdamWParams (SyncedAdamW.cuh:32-39);
 * SyncedAdamWNocoopParams is the same struct (SyncedAdamWNocoop.cuh:23). */
typedef struct {
    double lr, beta1, beta2, eps, weight_decay, lr_decay;
    double inner_tol, outer_tol, rho;
    int max_outer, max_inner;
    double time_step;
    int convergence_check_interval;
    double inner_rtol;
} tlfea_adamw_params;

/* Diagnostics of the last Solve() (new). */
typedef struct {
    int outer_iters;       /* outer (augmented-Lagrangian) iterations run */
    int inner_iters_total; /* inner iterations summed over outer iterations */
    int last_inner_iters;  /* inner iterations of the last outer iteration */
    int status;            /* TLFEA_OK, TLFEA_NONFINITE, TLFEA_BUDGET_EXCEEDED */
    double last_norm_g;    /* ||g|| at the last evaluated inner iteration */
    double kernel_ms;      /* device time of the solve (CUDA events) */
    double rel_residual;   /* ||(f_int - f_ext)_free|| / ||f_ext|| at the last inner iteration (stop rule on) */
    int stop_rule_met;     /* 1 if the relative-residual stop rule ended the solve */
} tlfea_solve_stats;

/* ------------------------------------------------------------- library */

/* Text of the last error on this thread ("" if none). */
const char* tlfea_last_error(void);
/* Kernels launched by this library since load (graph launches count their nodes). */
long long tlfea_launch_count(void);
/* Library version string. */
const char* tlfea_version(void);

/* ------------------------------------------------------------- elements */

/* GPU_FEAT10_Data(E, N) + Initialize()  (FEAT10Data.cuh:354-416);
 * GPU_FEAT4_Data(E, N) + Initialize()   (FEAT4Data.cuh). type = TLFEA_TYPE_T10/T4. */
int tlfea_element_create(int type, int n_elem, int n_nodes, tlfea_element* out);
/* Destroy()  (FEAT10Data.cuh:659-723): frees every device buffer and the handle. */
int tlfea_element_destroy(tlfea_element h);
/* Sets / gets the CUDA stream (cudaStream_t) used by this element and the
 * solvers built on it.  By default each element owns a non-blocking stream
 * (CUDA graphs cannot be captured on the legacy default stream). */
int tlfea_element_set_stream(tlfea_element h, void* stream);
int tlfea_element_get_stream(tlfea_element h, void** stream);
/* blocking = 1 (default, the reference's behaviour): every compute call
 * synchronises the stream before returning.  blocking = 0: compute calls
 * (compute/calc force, calc_p, reset_positions, linear_static_apply) return
 * after enqueueing; the caller synchronises the stream. */
int tlfea_element_set_blocking(tlfea_element h, int blocking);
/* x12 = reference positions captured by the last CalcDnDuPre (device copy). */
int tlfea_element_reset_positions(tlfea_element h);
int tlfea_element_get_counts(tlfea_element h, int* n_elem, int* n_nodes, int* n_constraint);

/* Setup(qx, qy, qz, qw, x, y, z, conn)  (FEAT10Data.cuh:418-503).  n_qp must
 * be 5 (T10) or 1 (T4).  Positions are copied to x12 and to the constraint
 * targets x12_jac; material scalars reset to zero, SVK selected. */
int tlfea_element_setup(tlfea_element h, const double* qx, const double* qy, const double* qz, const double* qw,
                        int n_qp, const double* x, const double* y, const double* z, const int* conn_colmajor);
/* SetDensity (:508-514), SetDamping (:521-528), SetSVK() (:533-547),
 * SetSVK(E, nu) (:553-569), SetMooneyRivlin (:576-587). */
int tlfea_element_set_density(tlfea_element h, double rho0);
int tlfea_element_set_damping(tlfea_element h, double eta_damp, double lambda_damp);
int tlfea_element_set_svk_default(tlfea_element h);
int tlfea_element_set_svk(tlfea_element h, double E, double nu);
/* Stores the Mooney-Rivlin parameters and selects the model (SetMooneyRivlin,
 * FEAT10Data.cuh:576-587).  The internal force (every entry point; on the
 * compact-geometry kernel), CalcP / CalcInternalForce and the first-order
 * solvers then use the Mooney-Rivlin stress of MooneyRivlin.cuh:46-104 (in FP64,
 * also in FP32 force mode), and LinearStaticSolver its consistent tangent
 * (MooneyRivlin.cuh:106-221). */
int tlfea_element_set_mooney_rivlin(tlfea_element h, double mu10, double mu01, double kappa);
/* SetExternalForce (:589-597); n must be 3*N. */
int tlfea_element_set_external_force(tlfea_element h, const double* f_ext, int n);
/* New (no reference counterpart): adds the gravity body force of a uniform
 * acceleration (gx, gy, gz) to f_ext, f_i += (sum_j M_ij) g with the consistent
 * mass of CalcMassMatrix (required first).  SetExternalForce replaces f_ext. */
int tlfea_element_add_gravity(tlfea_element h, double gx, double gy, double gz);
/* SetNodalFixed (FEAT10Data.cu:650-672) / UpdateNodalFixed (:674-752). */
int tlfea_element_set_nodal_fixed(tlfea_element h, const int* fixed_nodes, int n_fixed);
int tlfea_element_update_nodal_fixed(tlfea_element h, const int* fixed_nodes, int n_fixed);
/* UpdatePositions (FEAT10Data.cuh:628-640), UpdateConstraintTargets (:642-654). */
int tlfea_element_update_positions(tlfea_element h, const double* x, const double* y, const double* z, int n);
int tlfea_element_update_constraint_targets(tlfea_element h, const double* x, const double* y, const double* z,
                                            int n);

/* CalcDnDuPre  (FEAT10Data.cu:277-285; FEAT4Data.cu): reference gradients and
 * signed detJ at every QP, stored in the tiled layout the force kernel streams. */
int tlfea_element_calc_dndu_pre(tlfea_element h);
/* CalcMassMatrix + BuildMassCSRPattern (FEAT10Data.cu:341-417): node-level
 * consistent mass CSR, deterministic (no atomics). */
int tlfea_element_calc_mass_matrix(tlfea_element h);
/* CalcP (FEAT10Data.cu:300-305): P at every QP from the current positions,
 * no viscous term, stored for RetrievePFromFToCPU and CalcInternalForce. */
int tlfea_element_calc_p(tlfea_element h);
/* CalcInternalForce (FEAT10Data.cu:318-323): f_int += forces of the stored P.
 * Like the reference it does not clear f_int first. */
int tlfea_element_calc_internal_force(tlfea_element h);
/* CalcConstraintData (FEAT10Data.cu:325-339). */
int tlfea_element_calc_constraint_data(tlfea_element h);
/* ConvertToCSR_ConstraintJacT (FEAT10Data.cu:510-562) and
 * ConvertToCSR_ConstraintJac (:465-505). */
int tlfea_element_build_constraint_jact_csr(tlfea_element h);
int tlfea_element_build_constraint_jac_csr(tlfea_element h);

/* NEW fused hot path: f_int = internal force at the current positions (and
 * velocities v, interleaved 3N device pointer, or NULL for none), in one
 * pass over the element stream with a deterministic, atomic-free scatter.
 * This is compute_p + clear_internal_force + compute_internal_force of the
 * solver loops (SyncedNesterov.cu:180-207).  v may be NULL. */
int tlfea_element_compute_internal_force(tlfea_element h, const double* d_v);
/* Force precision for tlfea_element_compute_internal_force and the solvers. */
int tlfea_element_set_force_precision(tlfea_element h, int precision);
/* Launch configuration of the fused force kernel (new; the autotuner's knob):
 * force_kernel 0 = one tile per block with bulk-copy double-buffered QP
 * slices of the gradient stream (default), 1 = one tile per block with direct
 * loads, 2 = persistent producer/consumer pipeline, 3 = as 0 on the compact
 * geometry stream (J^-1 and dV per QP, gradients formed in registers);
 * grid_limit caps the persistent grid (0 = all resident blocks). */
int tlfea_element_set_launch_config(tlfea_element h, int force_kernel, int grid_limit);

/* Allocation-free internal force.  No counterpart in the reference.
 *
 * For callers that may not allocate device memory once they are running:
 * hosts whose GPU memory comes from their own pool and forbid cudaMalloc /
 * cudaFree after start-up, or time-critical loops where an allocation's
 * implicit device-wide synchronisation would stall their other streams.
 *
 * d_f_out (3N doubles, interleaved, caller-allocated) = the FP64 internal force
 * at the current positions; d_v as in tlfea_element_compute_internal_force.
 * The same kernels as that entry point, but their scratch (partial sums of
 * nodes shared between element tiles) lives in one static device array of
 * 2^20 doubles (8 MiB) that every GPU loading the library holds until exit.
 * Meshes needing more (3 per shared-node slot, about 7.3 per TET10 element:
 * roughly above 140k TET10 elements) are rejected with TLFEA_SIZE_MISMATCH.
 * It computes in FP64 only: an element in FP32 force mode is refused with
 * TLFEA_UNSUPPORTED.  The looked-up address is kept for the process; after a
 * cudaDeviceReset of that device it is stale, so do not call this entry point
 * again on a device that has been reset.  Nothing is allocated: no
 * cudaMalloc, cudaFree or allocating library call.  The first call on a
 * device looks up the array's device address; make that call before any
 * stream capture.  All calls share the array and it keeps the last call's
 * contents; calls that overlap on the GPU race. */
int tlfea_element_compute_internal_force_noalloc(tlfea_element h, const double* d_v, double* d_f_out);

/* Retrieve*ToCPU (FEAT10Data.cu:564-649, 753-757).  Sizes are in elements of
 * the output array and must match exactly. */
int tlfea_element_get_mass_nnz(tlfea_element h, long long* nnz);
int tlfea_element_retrieve_mass_csr(tlfea_element h, int* offsets, int* columns, double* values);
int tlfea_element_retrieve_internal_force(tlfea_element h, double* f, int n);
int tlfea_element_retrieve_external_force(tlfea_element h, double* f, int n);
int tlfea_element_retrieve_positions(tlfea_element h, double* x, double* y, double* z, int n);
int tlfea_element_retrieve_p(tlfea_element h, double* P, long long n);        /* E*QP*9 */
int tlfea_element_retrieve_dndu_pre(tlfea_element h, double* g, long long n); /* E*QP*NPE*3 */
int tlfea_element_retrieve_detj(tlfea_element h, double* detJ, long long n);  /* E*QP */
int tlfea_element_retrieve_connectivity(tlfea_element h, int* conn_colmajor, long long n);
int tlfea_element_retrieve_constraint(tlfea_element h, double* c, int n);
/* The constraint Jacobian CSR built by ConvertToCSR_ConstraintJac (which = 0: J,
 * n_constraint rows) or ConvertToCSR_ConstraintJacT (which = 1: J^T, 3N rows);
 * n_constraint unit entries each.  The reference keeps these arrays private and
 * reads them through device accessors (FEAT10Data.cuh:262-286); this is the
 * host-side view a caller needs to check them.  offsets has rows + 1 entries,
 * columns and values n_constraint; TLFEA_NOT_SETUP if that CSR was not built. */
int tlfea_element_retrieve_constraint_jac_csr(tlfea_element h, int which, int* offsets, int* columns,
                                              double* values);
/* WriteOutputVTK (FEAT10Data.cu:759-794): legacy ASCII VTK of the current mesh. */
int tlfea_element_write_vtk(tlfea_element h, const char* filename);
/* Get{X,Y,Z}12DevicePtr, GetExternalForceDevicePtr (FEAT10Data.cuh:599-621).  Pass NULL
 * for pointers not wanted.  Once a position pointer has been handed out, the caller may
 * write the positions at any time, so the element rebuilds the records it derives from
 * them (the tile-ordered node values, FP32 mode's displacements) before every force
 * evaluation from then on. */
int tlfea_element_device_ptrs(tlfea_element h, double** x, double** y, double** z, double** f_ext, double** f_int);

/* ------------------------------------------------------------- solvers */

/* SyncedNesterovSolver(ElementBase*, n_constraints) (SyncedNesterov.cuh:39-110). */
int tlfea_nesterov_create(tlfea_element e, int n_constraints, tlfea_solver* out);
/* SyncedAdamWSolver (SyncedAdamW.cuh:43-) and SyncedAdamWNocoopSolver
 * (SyncedAdamWNocoop.cuh:25-). */
int tlfea_adamw_create(tlfea_element e, int n_constraints, tlfea_solver* out);
int tlfea_adamw_nocoop_create(tlfea_element e, int n_constraints, tlfea_solver* out);
/* LinearStaticSolver<T>(data, tol, max_iter) (LinearStaticSolver.cuh:56). */
int tlfea_linear_static_create(tlfea_element e, double tol, int max_iter, tlfea_solver* out);
/* ~Solver. */
int tlfea_solver_destroy(tlfea_solver s);
/* Setup() (SyncedNesterov.cuh:157-179): zeroes every solver vector. */
int tlfea_solver_setup(tlfea_solver s);
/* SetParameters(void*) (SyncedNesterov.cuh:139-155, SyncedAdamW.cuh:159-184):
 * copies the struct and zeroes v_guess, v_prev and the multipliers.  params
 * points at tlfea_nesterov_params or tlfea_adamw_params as the solver needs;
 * a no-op for the linear static solver (LinearStaticSolver.cuh:65). */
int tlfea_solver_set_parameters(tlfea_solver s, const void* params);
/* Solve() (SyncedNesterov.cuh:266-268, SyncedAdamW.cuh, LinearStaticSolver.cu:590-603). */
int tlfea_solver_solve(tlfea_solver s);
/* New (no reference counterpart, opt-in): preconditioner of the linear static
 * CG.  kind 0 = none (default, the reference's unpreconditioned CG); 1 = block
 * Jacobi on the 3x3 node diagonal blocks of K (BCs applied).  The stop test
 * stays sqrt(r.r / r0.r0) < tol. */
int tlfea_linear_static_set_preconditioner(tlfea_solver s, int kind);
/* How the CG applies K (new).  2 = matrix-free where it applies (TET10, SVK, no
 * damping, no preconditioner; elsewhere the assembled K): K p element by element in each
 * iteration from the tangent at the solve's positions (F and S of every QP formed once per
 * solve, 15 doubles per element and QP), never assembled (K is assembled on demand, at the
 * positions of the last solve, for tlfea_linear_static_retrieve_k); 1 = the assembled K of
 * the reference (3x3 node blocks); 0 (default) = matrix-free where it applies from 100,000
 * elements, assembled otherwise.  Both are the same operator: the solutions and iteration
 * counts agree to rounding. */
int tlfea_linear_static_set_operator(tlfea_solver s, int mode);
/* GetLastIterCount / GetLastResidual (LinearStaticSolver.cuh:68-72). */
int tlfea_linear_static_last(tlfea_solver s, int* iters, double* rel_residual);
/* Retrieve the LinearStaticSolver stiffness (BCs applied) as 3N x 3N CSR
 * (new; the reference keeps K private).  Call with NULL arrays for nnz. */
int tlfea_linear_static_retrieve_k(tlfea_solver s, long long* nnz, int* offsets, int* columns, double* values);
/* d_y = K d_x with the stiffness of the last Solve() (device pointers, 3N
 * each); the CG loop's operator (matrix-free or the SpMV kernel; new). */
int tlfea_linear_static_apply(tlfea_solver s, const double* d_x, double* d_y);
/* Velocity state of the first-order solvers (v_guess, v_prev: 3N; lambda: n_c). */
int tlfea_solver_get_velocity(tlfea_solver s, double* v_guess, double* v_prev, int n);
int tlfea_solver_set_velocity(tlfea_solver s, const double* v_guess, const double* v_prev, int n);
int tlfea_solver_get_multipliers(tlfea_solver s, double* lam, int n);
int tlfea_solver_get_stats(tlfea_solver s, tlfea_solve_stats* st);
/* New (no reference counterpart): relative-residual stop rule of the Nesterov /
 * AdamW solvers.  With rel_tol > 0 every inner iteration also evaluates
 * ||(f_int - f_ext)_free|| / ||f_ext|| in FP64 (free = not a fixed node) at the
 * positions the internal force was computed at, and the solve ends -- keeping
 * those positions -- once it is below rel_tol.  0 turns it off (default). */
int tlfea_solver_set_stop_rule(tlfea_solver s, double rel_tol);
/* New: launch mode of the Nesterov / AdamW solvers.  2 = one kernel per phase
 * (velocity guess, forces, gradient, update, outer update) with the loop state on the
 * device, chunks of iterations replayed as CUDA graphs until the solve ends; 1 = the
 * whole Solve() in one persistent cooperative launch; 0 (default) = per-phase from
 * 200,000 nodes, persistent below.  The iterations are the same; with fixed iteration
 * counts so are the trajectories, bit for bit. */
int tlfea_solver_set_mode(tlfea_solver s, int mode);

/* New, no reference counterpart: n_steps implicit steps of a first-order solver
 * in one call -- the loop a reference driver writes around SetExternalForce +
 * Solve (examples/beam_simulation.cc:275-283, examples/test_feat10_nesterov.cc:
 * 197-199) -- launched as one CUDA graph with
 * the load computed on the device.  Step k (0-based) ends at
 * t_k = t0 + (k + 1) * time_step and runs with
 *     f_ext = f_base + (amp * sin(omega * t_k + phase)) * f_var
 * (f_base = the external force set before the call, f_var a host array of
 * 3 * n_nodes doubles; products and sums rounded separately, no fused
 * multiply-add).  f_var NULL keeps f_ext constant.  inner_iters (NULL or n_steps
 * ints) receives each step's total inner iterations; the solve statistics are
 * those of the last step, with status the last non-zero step status.  After
 * the call f_ext holds the last step's load.  The linear static solver is
 * refused (TLFEA_INVALID_ARG). */
int tlfea_solver_run_steps(tlfea_solver s, int n_steps, double t0, const double* f_var, double amp,
                           double omega, double phase, int* inner_iters);

/* ------------------------------------------------- batched linear static
 * New, no reference counterpart: many independent meshes solved by one
 * persistent cooperative launch (captured in a CUDA graph).  Per instance the
 * iteration is LinearStaticSolver's CG (LinearStaticSolver.cu:469-565) on the
 * linear stiffness at the reference configuration (the tangent of
 * compute_hessian_assemble_csr, FEAT10DataFunc.cuh:512-684, at F = I),
 * applied matrix-free, with fixed DOFs eliminated as apply_bcs_kernel does
 * (LinearStaticSolver.cu:284-306).  Stop rule ||r|| / ||f_free|| < tol (FP64).
 *
 * Instances are concatenated: instance i owns nodes [node_off[i], node_off[i+1])
 * and elements [elem_off[i], elem_off[i+1]); conn is row-major
 * [elem_off[n_inst]][npe] with node ids local to the instance; x, y, z hold the
 * concatenated reference positions; the quadrature is Setup()'s. */
typedef struct tlfea_batch_s* tlfea_batch;
int tlfea_batch_create(int type, int n_inst, const int* node_off, const int* elem_off, const double* qx,
                       const double* qy, const double* qz, const double* qw, int n_qp, const double* x,
                       const double* y, const double* z, const int* conn, tlfea_batch* out);
/* Shared-mesh batch: n_inst instances of ONE mesh (n_nodes nodes, n_elem
 * elements, conn row-major [n_elem][npe]) that differ only in material, fixed
 * nodes and loads.  The mesh's tiling and gradients are stored once; node
 * vectors are concatenated instance by instance (instance i owns nodes
 * [i*n_nodes, (i+1)*n_nodes)).  Every other batch call works unchanged. */
int tlfea_batch_create_shared(int type, int n_inst, int n_nodes, int n_elem, const double* qx, const double* qy,
                              const double* qz, const double* qw, int n_qp, const double* x, const double* y,
                              const double* z, const int* conn, tlfea_batch* out);
int tlfea_batch_destroy(tlfea_batch b);
int tlfea_batch_get_counts(tlfea_batch b, int* n_inst, int* n_elem, int* n_nodes, int* n_tiles);
int tlfea_batch_get_stream(tlfea_batch b, void** stream);
/* Per-instance Young's modulus and Poisson ratio (Lame parameters as SetSVK). */
int tlfea_batch_set_material(tlfea_batch b, const double* E, const double* nu);
/* Fixed nodes (concatenated numbering); nodes that no element touches are always fixed. */
int tlfea_batch_set_fixed(tlfea_batch b, const int* nodes, int n);
/* External force, 3 * n_nodes interleaved; on_device selects a device pointer. */
int tlfea_batch_set_external_force(tlfea_batch b, const double* f, long long n, int on_device);
/* Warm start u0 (3 * n_nodes; NULL = cold start u0 = 0). */
int tlfea_batch_set_initial_guess(tlfea_batch b, const double* u0, long long n, int on_device);
/* TLFEA_PRECISION_FP64 (default) or FP32 element work.  With FP32 the solve is
 * iterative refinement: the true residual r = f - K u (free DOFs) is evaluated
 * with the FP64 operator, the correction K d = r is solved by the CG with FP32
 * element work (vectors, dots and its stop test FP64) to the relative tolerance
 * max(tol, min(0.1, max(1e-4, sqrt(tol) / 2))), u += d, and again until every
 * instance's FP64 residual ||r|| / ||f_free|| is below tol (at most 8 passes).
 * The residual and status reported are the FP64 ones, the iterations the sum
 * over passes.  FP32 solves are not graph-captured. */
int tlfea_batch_set_precision(tlfea_batch b, int precision);
/* Launch mode: 0 (default) = one kernel per CG phase (element tiles, p.q, update,
 * direction) at the occupancy each allows, chunks of iterations replayed as CUDA
 * graphs until every instance is done; 1 = the whole solve in one persistent
 * cooperative launch with grid barriers between the phases. */
int tlfea_batch_set_mode(tlfea_batch b, int mode);
/* Launch shape: resident blocks per SM of the persistent kernel (mode 1; 0 =
 * occupancy maximum) and nodes per reduction chunk (0 = keep). */
int tlfea_batch_set_launch(tlfea_batch b, int blocks_per_sm, int chunk_nodes);
int tlfea_batch_get_launch(tlfea_batch b, int* blocks_per_sm, int* chunk_nodes, int* grid);
/* Times trial_iters CG iterations per candidate and keeps the fastest: chunk sizes
 * (mode 0; best_blocks_per_sm = 0), or (blocks per SM, chunk size) pairs (mode 1).
 * Overwrites the solution vectors. */
int tlfea_batch_autotune(tlfea_batch b, int trial_iters, int* best_blocks_per_sm, int* best_chunk, float* best_ms);
/* Solves every instance; per-instance iterations, ||r||/||f_free|| and status
 * (0 converged, 1 non-positive p.Kp, 2 max_iter reached). */
int tlfea_batch_solve(tlfea_batch b, double tol, int max_iter);
int tlfea_batch_get_results(tlfea_batch b, int* iters, double* rel_residual, int* status);
int tlfea_batch_retrieve_displacement(tlfea_batch b, double* u, long long n);
int tlfea_batch_device_ptrs(tlfea_batch b, double** u, double** f_ext, double** u0);
/* d_y = K_bc d_x over the whole batch (device pointers, 3 * n_nodes). */
int tlfea_batch_apply(tlfea_batch b, const double* d_x, double* d_y);

/* ------------------------------------------------------ warm-start MLP
 * New, no reference counterpart: dims[0] -> dims[1] -> ... -> dims[n_layers]
 * with GELU between layers, BF16 operands and FP32 accumulation on the
 * tcgen05 tensor cores, FP32 master weights, AdamW, mean-squared-error loss.
 * Hidden and output widths are multiples of 16; max_batch a multiple of 128.
 * Flat parameter layout: per layer W [dims[l+1] x dims[l]] row-major, then b.
 * Tensor arguments named d_* are device pointers (FP32, row-major). */
typedef struct tlfea_mlp_s* tlfea_mlp;
int tlfea_mlp_create(int n_layers, const int* dims, int max_batch, unsigned long long seed, tlfea_mlp* out);
int tlfea_mlp_destroy(tlfea_mlp m);
int tlfea_mlp_get_stream(tlfea_mlp m, void** stream);
int tlfea_mlp_param_count(tlfea_mlp m, long long* n);
int tlfea_mlp_set_params(tlfea_mlp m, const float* params, long long n);
int tlfea_mlp_get_params(tlfea_mlp m, float* params, long long n);
int tlfea_mlp_get_grads(tlfea_mlp m, float* grads, long long n);
int tlfea_mlp_forward(tlfea_mlp m, const float* d_x, int batch, float* d_y);
int tlfea_mlp_loss_grad(tlfea_mlp m, const float* d_x, const float* d_target, int batch, float* loss);
int tlfea_mlp_adamw_step(tlfea_mlp m, float lr, float beta1, float beta2, float eps, float weight_decay);
int tlfea_mlp_train_step(tlfea_mlp m, const float* d_x, const float* d_target, int batch, float lr, float beta1,
                         float beta2, float eps, float weight_decay, float* loss);
int tlfea_mlp_sync(tlfea_mlp m);
/* ------------------------------------------- batched time-stepping sequences
 *
 * New, no reference counterpart in this form: B sequences of implicit time steps on
 * one mesh, each step solved by SyncedNesterov's iteration (SyncedNesterov.cu:97-360:
 * the outer augmented-Lagrangian loop around the inner Nesterov loop, with the
 * inertia M (v - v_prev) / dt), all sequences in the same kernels.  The mesh element
 * (Setup, CalcDnDuPre, CalcMassMatrix, SetNodalFixed, SVK, density, damping and its
 * external force -- e.g. gravity via add_gravity -- already set) is shared; each
 * sequence has its own E, nu, step size and state, starting at rest in the reference
 * configuration.  A sequence's inner loop ends when ||g_free|| / ||f_ext|| < rel_tol
 * (g: the step's gradient, inertia + internal - external force + constraint terms;
 * free = not fixed) or after max_inner iterations (rel_tol = 0: always max_inner, the
 * reference's iteration with zero inner tolerance); its outer loop ends when the rule
 * was met or ||c|| < outer_tol, or after max_outer iterations. */
typedef struct tlfea_dynbatch_s* tlfea_dynbatch;
int tlfea_dynbatch_create(tlfea_element mesh, int n_seq, tlfea_dynbatch* out);
int tlfea_dynbatch_destroy(tlfea_dynbatch b);
/* Per-sequence E and nu (n_seq each); mu and lambda as SetSVK(E, nu) (FEAT10Data.cuh:553-569). */
int tlfea_dynbatch_set_material(tlfea_dynbatch b, const double* E, const double* nu);
/* SyncedNesterovParams (inner_tol unused: the stop rule above ends the inner loop). */
int tlfea_dynbatch_set_parameters(tlfea_dynbatch b, const tlfea_nesterov_params* p, double rel_tol);
/* Per-sequence step sizes alpha (n_seq, each > 0), after set_parameters (which gives
 * every sequence p->alpha). */
int tlfea_dynbatch_set_step_sizes(tlfea_dynbatch b, const double* alpha);
/* Time-varying load: f_ext(t) = f_base + amp * sin(omega * t + phase) * f_var at the end
 * time t = k dt of step k, computed on the device; f_base = the element's f_ext when the
 * batch was created.  f_var: host, n = 3N (NULL: zero). */
int tlfea_dynbatch_set_load(tlfea_dynbatch b, const double* f_var, int n, double amp, double omega, double phase);
/* Inner iterations per CUDA-graph replay (default 8). */
int tlfea_dynbatch_set_chunk(tlfea_dynbatch b, int chunk);
/* Momentum restart of the inner Nesterov loop (new; 0 = off, the reference's
 * iteration, the default): a sequence whose step works against its momentum,
 * g . (v_next - v_k) > 0, starts the beta sequence afresh at its next look-ahead (the
 * gradient restart test of O'Donoghue and Candes, 2015).  Without a restart the
 * reference's beta schedule converges sublinearly on a well-conditioned but stiff
 * step Hessian; with it, linearly at about sqrt(condition number) iterations per
 * e-fold of the residual. */
int tlfea_dynbatch_set_restart(tlfea_dynbatch b, int on);
/* Every sequence back to rest in the reference configuration, t = 0. */
int tlfea_dynbatch_reset(tlfea_dynbatch b);
/* One implicit step of every sequence.  warm_start: 0 = the previous step's velocity
 * (the reference's behaviour), 1 = linear extrapolation 2 v_n - v_(n-1), 2 = d_v_guess
 * (device, n_seq x 3N interleaved).  iters, rel, converged: host arrays of n_seq (or
 * NULL): inner iterations of the step, the last relative residual, 1 if the stop rule
 * ended it. */
int tlfea_dynbatch_step(tlfea_dynbatch b, int warm_start, const double* d_v_guess, int* iters, double* rel,
                        int* converged);
/* Device pointers of the state: positions (n_seq x N per component), the velocity
 * (n_seq x 3N) and the previous step's velocity. */
int tlfea_dynbatch_device_ptrs(tlfea_dynbatch b, double** x, double** y, double** z, double** v, double** v_hist);
int tlfea_dynbatch_retrieve_positions(tlfea_dynbatch b, int seq, double* x, double* y, double* z);
int tlfea_dynbatch_retrieve_velocity(tlfea_dynbatch b, int seq, double* v);

/* The MLP's tensor-core product on its own: d_d[M x N] (FP32, leading dim ldd)
 * = d_a[M x K] (BF16, lda) * d_b[N x K]^T (BF16, ldb) + d_bias[N] (or NULL).
 * N and K multiples of 16, lda and ldb multiples of 8 and >= K, operands
 * 16-byte aligned.  Synchronises the stream and reports a product that did not
 * complete as TLFEA_CUDA_ERROR. */
int tlfea_mlp_gemm_bf16(int M, int N, int K, const void* d_a, int lda, const void* d_b, int ldb, const float* d_bias,
                        float* d_d, int ldd, void* stream);

/* The same product, only enqueued on the stream (no host synchronisation):
 * *d_err (a device int the caller zeroes) becomes non-zero if a bounded wait
 * inside the kernel ran out. */
int tlfea_mlp_gemm_bf16_async(int M, int N, int K, const void* d_a, int lda, const void* d_b, int ldb,
                              const float* d_bias, float* d_d, int ldd, int* d_err, void* stream);

#ifdef __cplusplus
}
#endif
#endif
