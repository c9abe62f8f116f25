// solver.cuh -- solver state shared by the first-order (Nesterov / AdamW) and the
// linear static (CG) solvers.
#pragma once

#include <vector>

#include "element.cuh"

namespace tlfea {

enum SolverKind { KIND_NESTEROV = 0, KIND_ADAMW = 1, KIND_ADAMW_NOCOOP = 2, KIND_LINEAR_STATIC = 3 };

// Device-resident scalars of the CG loop (read and written only by kernels
// between host synchronisations).
struct CgCtl {
    unsigned int ticket;  // last-block-done counter, reset by the last block
    int done;             // 1 once converged, broken down or out of iterations
    int iters;            // completed iterations
    int status;           // 0 ok, 1 p.Kp <= 0, 2 max_iter reached
    double rr0, rr, alpha, beta, rel;  // preconditioned: rr holds r.z, rres the true r.r
    double pq;
    double rres;
};

// Load of step k of a multi-step run: f_ext = f_base + amp * sin(omega * t_k + phase) * f_var,
// t_k = t0 + (k + 1) * dt (the time at the end of step k).
struct StepLoad {
    const double* f_base;
    const double* f_var;
    double t0, amp, omega, phase;
};

}  // namespace tlfea

struct tlfea_solver_s {
    int kind = tlfea::KIND_NESTEROV;
    tlfea_element_s* el = nullptr;
    int n_constraints = 0;
    int device = 0;

    // first-order state (3N / n_c), FP64
    double *v_guess = nullptr, *v_prev = nullptr, *v_k = nullptr, *v_km1 = nullptr;
    double *g = nullptr, *lam = nullptr, *m = nullptr, *va = nullptr;
    double *xp = nullptr, *yp = nullptr, *zp = nullptr;
    double* red = nullptr;   // per-block partial sums (6 arrays of max_blocks)
    double rel_tol = 0.0;    // relative-residual stop rule (0 = off)
    unsigned char* node_fixed = nullptr;  // N, for the stop rule's free-DOF norm
    int max_blocks = 0;
    int* dstat = nullptr;    // device diagnostics (tlfea_solve_stats fields)
    int fo_mode = 0;         // 0 = by size (per-phase from FO_PHASED_MIN_NODES), 1 = persistent, 2 = per-phase
    void* fo_ctl = nullptr;  // per-phase mode: the device-side loop state
    cudaGraphExec_t fo_graph[2] = {nullptr, nullptr};  // per-phase mode: chunks of 8 and 32 slots
    std::vector<unsigned char> fo_graph_key;             // what the captured chunks bake in
    tlfea_nesterov_params np{};
    tlfea_adamw_params ap{};
    bool params_set = false;
    tlfea_solve_stats stats{};

    // linear static
    double tol = 1e-10;
    int max_iter = 10000;
    int last_iters = 0;
    double last_res = 0.0;
    double* K = nullptr;  // 3x3 blocks on the node pattern, 9 doubles per block
    double *u = nullptr, *f = nullptr, *r = nullptr, *p = nullptr, *q = nullptr;
    unsigned char* is_fixed = nullptr;  // 3N
    tlfea::CgCtl* ctl = nullptr;
    tlfea::CgCtl* ctl_apply = nullptr;  // scratch control block of linear_static_apply
    double* cg_part = nullptr;  // per-block partials (2 arrays of cg_blocks)
    int precond = 0;            // 0 none (the reference's CG), 1 block Jacobi (3x3 node diagonal blocks)
    double* dinv = nullptr;     // block Jacobi: inverse diagonal blocks, 9 per node
    double* z = nullptr;        // block Jacobi: z = D^-1 r
    int cg_graph_precond = -1;  // preconditioner the captured graph was built for
    int cg_graph_mf = -1;       // operator the captured graph was built for (1 = matrix-free)
    int op_mode = 0;            // 0: by size (matrix-free from MF_MIN_ELEMENTS), 1: assembled, 2: matrix-free
    bool mf_last = false;       // the last solve ran matrix-free: K is assembled on demand
    double* mf_part = nullptr;  // matrix-free p.q partials: one per tile, then one per combine block
    double* mf_prec = nullptr;     // p in the node record's tile order (3 per padded slot)
    uint16_t* mf_pfix = nullptr;   // fixed-DOF flags per padded slot
    double* mf_tan = nullptr;      // F and S per element QP at the last solve's positions
    double *xk = nullptr, *yk = nullptr, *zk = nullptr;  // positions of the last matrix-free solve
    int cg_blocks = 0;
    cudaGraphExec_t cg_graph = nullptr;
    int cg_graph_iters = 0;
    bool k_built = false;
};
