// solver_api.cu -- C ABI of the solvers (include/tlfea_b200.h).
#include <algorithm>
#include <cstring>

#include "solver.cuh"

namespace tlfea {
int first_order_alloc(tlfea_solver_s* s);
void first_order_free(tlfea_solver_s* s);
int first_order_solve(tlfea_solver_s* s);
int first_order_steps(tlfea_solver_s* s, int steps, const StepLoad* load, int* inner_iters);
int linear_static_solve(tlfea_solver_s* s);
int linear_static_retrieve_k(tlfea_solver_s* s, long long* nnz, int* offsets, int* columns, double* values);
int linear_static_apply(tlfea_solver_s* s, const double* d_x, double* d_y);
void linear_static_free(tlfea_solver_s* s);

static int zero_first_order(tlfea_solver_s* s, bool all) {
    tlfea_element_s* el = s->el;
    const size_t n3 = 3 * (size_t)el->N, N = el->N;
    cudaStream_t st = el->stream;
    TLFEA_CUDA(cudaMemsetAsync(s->v_guess, 0, n3 * sizeof(double), st));
    TLFEA_CUDA(cudaMemsetAsync(s->v_prev, 0, n3 * sizeof(double), st));
    TLFEA_CUDA(cudaMemsetAsync(s->lam, 0, std::max(s->n_constraints, 1) * sizeof(double), st));
    if (all) {
        TLFEA_CUDA(cudaMemsetAsync(s->v_k, 0, n3 * sizeof(double), st));
        TLFEA_CUDA(cudaMemsetAsync(s->v_km1, 0, n3 * sizeof(double), st));
        TLFEA_CUDA(cudaMemsetAsync(s->g, 0, n3 * sizeof(double), st));
        TLFEA_CUDA(cudaMemsetAsync(s->m, 0, n3 * sizeof(double), st));
        TLFEA_CUDA(cudaMemsetAsync(s->va, 0, n3 * sizeof(double), st));
        TLFEA_CUDA(cudaMemsetAsync(s->xp, 0, N * sizeof(double), st));
        TLFEA_CUDA(cudaMemsetAsync(s->yp, 0, N * sizeof(double), st));
        TLFEA_CUDA(cudaMemsetAsync(s->zp, 0, N * sizeof(double), st));
    }
    TLFEA_CUDA(cudaStreamSynchronize(st));
    return TLFEA_OK;
}

static int create_first_order(tlfea_element e, int n_constraints, int kind, tlfea_solver* out) {
    if (!e || !out || n_constraints < 0) return TLFEA_INVALID_ARG;
    *out = nullptr;
    TLFEA_CUDA(cudaSetDevice(e->device));
    tlfea_solver_s* s = new tlfea_solver_s();
    s->kind = kind;
    s->el = e;
    s->device = e->device;
    s->n_constraints = n_constraints;
    int st = first_order_alloc(s);
    if (st == TLFEA_OK) st = zero_first_order(s, true);
    if (st) {
        first_order_free(s);
        delete s;
        return st;
    }
    *out = s;
    return TLFEA_OK;
}

}  // namespace tlfea

using namespace tlfea;

extern "C" {

int tlfea_nesterov_create(tlfea_element e, int n_constraints, tlfea_solver* out) {
    return create_first_order(e, n_constraints, KIND_NESTEROV, out);
}

int tlfea_adamw_create(tlfea_element e, int n_constraints, tlfea_solver* out) {
    return create_first_order(e, n_constraints, KIND_ADAMW, out);
}

int tlfea_adamw_nocoop_create(tlfea_element e, int n_constraints, tlfea_solver* out) {
    return create_first_order(e, n_constraints, KIND_ADAMW_NOCOOP, out);
}

int tlfea_linear_static_create(tlfea_element e, double tol, int max_iter, tlfea_solver* out) {
    if (!e || !out) return TLFEA_INVALID_ARG;
    *out = nullptr;
    tlfea_solver_s* s = new tlfea_solver_s();
    s->kind = KIND_LINEAR_STATIC;
    s->el = e;
    s->device = e->device;
    s->tol = tol;
    s->max_iter = max_iter;
    *out = s;
    return TLFEA_OK;
}

int tlfea_solver_destroy(tlfea_solver s) {
    if (!s) return TLFEA_INVALID_ARG;
    TLFEA_CUDA(cudaSetDevice(s->device));
    if (s->kind == KIND_LINEAR_STATIC)
        linear_static_free(s);
    else
        first_order_free(s);
    delete s;
    return TLFEA_OK;
}

int tlfea_solver_setup(tlfea_solver s) {
    if (!s) return TLFEA_INVALID_ARG;
    TLFEA_CUDA(cudaSetDevice(s->device));
    if (s->kind == KIND_LINEAR_STATIC) return TLFEA_OK;
    return zero_first_order(s, true);
}

int tlfea_solver_set_parameters(tlfea_solver s, const void* params) {
    if (!s) return TLFEA_INVALID_ARG;
    TLFEA_CUDA(cudaSetDevice(s->device));
    if (s->kind == KIND_LINEAR_STATIC) return TLFEA_OK;
    if (!params) return TLFEA_INVALID_ARG;
    if (s->kind == KIND_NESTEROV)
        memcpy(&s->np, params, sizeof(tlfea_nesterov_params));
    else
        memcpy(&s->ap, params, sizeof(tlfea_adamw_params));
    s->params_set = true;
    return zero_first_order(s, false);
}

int tlfea_solver_solve(tlfea_solver s) {
    if (!s) return TLFEA_INVALID_ARG;
    TLFEA_CUDA(cudaSetDevice(s->device));
    if (s->kind == KIND_LINEAR_STATIC) return linear_static_solve(s);
    return first_order_solve(s);
}

int tlfea_solver_run_steps(tlfea_solver s, int n_steps, double t0, const double* f_var, double amp,
                           double omega, double phase, int* inner_iters) {
    if (!s || n_steps < 1) return TLFEA_INVALID_ARG;
    if (s->kind == KIND_LINEAR_STATIC) {
        set_error("run_steps: the linear static solver has no time steps");
        return TLFEA_INVALID_ARG;
    }
    TLFEA_CUDA(cudaSetDevice(s->device));
    if (!s->el->is_setup) {
        set_error("element must be set up first");
        return TLFEA_NOT_SETUP;
    }
    if (!f_var) return first_order_steps(s, n_steps, nullptr, inner_iters);
    tlfea_element_s* el = s->el;
    const size_t n3 = 3 * (size_t)el->N;
    double *base = nullptr, *var = nullptr;
    if (dalloc(&base, n3) || dalloc(&var, n3)) {
        dfree(base);
        dfree(var);
        return TLFEA_CUDA_ERROR;
    }
    int st = TLFEA_OK;
    if (cudaMemcpyAsync(base, el->f_ext, n3 * sizeof(double), cudaMemcpyDeviceToDevice, el->stream) != cudaSuccess ||
        cudaMemcpyAsync(var, f_var, n3 * sizeof(double), cudaMemcpyHostToDevice, el->stream) != cudaSuccess) {
        set_error("run_steps: load upload failed");
        st = TLFEA_CUDA_ERROR;
    }
    if (!st) {
        StepLoad L{base, var, t0, amp, omega, phase};
        st = first_order_steps(s, n_steps, &L, inner_iters);
    }
    cudaStreamSynchronize(el->stream);
    dfree(base);
    dfree(var);
    return st;
}

int tlfea_linear_static_last(tlfea_solver s, int* iters, double* rel_residual) {
    if (!s || s->kind != KIND_LINEAR_STATIC) return TLFEA_INVALID_ARG;
    if (iters) *iters = s->last_iters;
    if (rel_residual) *rel_residual = s->last_res;
    return TLFEA_OK;
}

int tlfea_linear_static_retrieve_k(tlfea_solver s, long long* nnz, int* offsets, int* columns, double* values) {
    if (!s || s->kind != KIND_LINEAR_STATIC) return TLFEA_INVALID_ARG;
    TLFEA_CUDA(cudaSetDevice(s->device));
    return linear_static_retrieve_k(s, nnz, offsets, columns, values);
}

int tlfea_linear_static_set_preconditioner(tlfea_solver s, int kind) {
    if (!s || s->kind != KIND_LINEAR_STATIC || (kind != 0 && kind != 1)) return TLFEA_INVALID_ARG;
    s->precond = kind;
    return TLFEA_OK;
}

int tlfea_linear_static_set_operator(tlfea_solver s, int mode) {
    if (!s || s->kind != KIND_LINEAR_STATIC || mode < 0 || mode > 2) return TLFEA_INVALID_ARG;
    s->op_mode = mode;
    return TLFEA_OK;
}

int tlfea_linear_static_apply(tlfea_solver s, const double* d_x, double* d_y) {
    if (!s || s->kind != KIND_LINEAR_STATIC || !d_x || !d_y) return TLFEA_INVALID_ARG;
    TLFEA_CUDA(cudaSetDevice(s->device));
    return linear_static_apply(s, d_x, d_y);
}

int tlfea_solver_get_velocity(tlfea_solver s, double* v_guess, double* v_prev, int n) {
    if (!s || s->kind == KIND_LINEAR_STATIC) return TLFEA_INVALID_ARG;
    if (n != 3 * s->el->N) return TLFEA_SIZE_MISMATCH;
    TLFEA_CUDA(cudaSetDevice(s->device));
    TLFEA_CUDA(cudaStreamSynchronize(s->el->stream));
    if (v_guess) TLFEA_CUDA(cudaMemcpy(v_guess, s->v_guess, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (v_prev) TLFEA_CUDA(cudaMemcpy(v_prev, s->v_prev, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return TLFEA_OK;
}

int tlfea_solver_set_velocity(tlfea_solver s, const double* v_guess, const double* v_prev, int n) {
    if (!s || s->kind == KIND_LINEAR_STATIC) return TLFEA_INVALID_ARG;
    if (n != 3 * s->el->N) return TLFEA_SIZE_MISMATCH;
    TLFEA_CUDA(cudaSetDevice(s->device));
    TLFEA_CUDA(cudaStreamSynchronize(s->el->stream));
    cudaStream_t st = s->el->stream;
    if (v_guess) TLFEA_CUDA(cudaMemcpyAsync(s->v_guess, v_guess, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    if (v_prev) TLFEA_CUDA(cudaMemcpyAsync(s->v_prev, v_prev, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    TLFEA_CUDA(cudaStreamSynchronize(st));
    return TLFEA_OK;
}

int tlfea_solver_get_multipliers(tlfea_solver s, double* lam, int n) {
    if (!s || s->kind == KIND_LINEAR_STATIC || !lam) return TLFEA_INVALID_ARG;
    if (n != s->n_constraints) return TLFEA_SIZE_MISMATCH;
    if (n == 0) return TLFEA_OK;
    TLFEA_CUDA(cudaSetDevice(s->device));
    TLFEA_CUDA(cudaStreamSynchronize(s->el->stream));
    TLFEA_CUDA(cudaMemcpy(lam, s->lam, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return TLFEA_OK;
}

int tlfea_solver_get_stats(tlfea_solver s, tlfea_solve_stats* st) {
    if (!s || !st) return TLFEA_INVALID_ARG;
    *st = s->stats;
    return TLFEA_OK;
}

int tlfea_solver_set_stop_rule(tlfea_solver s, double rel_tol) {
    if (!s || !(rel_tol >= 0.0)) return TLFEA_INVALID_ARG;
    if (s->kind == tlfea::KIND_LINEAR_STATIC) {
        tlfea::set_error("the stop rule applies to the Nesterov / AdamW solvers (CG has its own tolerance)");
        return TLFEA_UNSUPPORTED;
    }
    s->rel_tol = rel_tol;
    return TLFEA_OK;
}

int tlfea_solver_set_mode(tlfea_solver s, int mode) {
    if (!s || mode < 0 || mode > 2) return TLFEA_INVALID_ARG;
    if (s->kind == tlfea::KIND_LINEAR_STATIC) {
        tlfea::set_error("the launch mode applies to the Nesterov / AdamW solvers");
        return TLFEA_UNSUPPORTED;
    }
    s->fo_mode = mode;
    return TLFEA_OK;
}

}  // extern "C"
