// Parity harness over the reference's own CUDA build (test infrastructure only).
//
// This translation unit is compiled together with the reference's unchanged sources
// (src/elements/FEAT10Data.cu, FEAT4Data.cu, src/solvers/LinearStaticSolver.cu,
// SyncedNesterov.cu, SyncedAdamW.cu, SyncedAdamWNocoop.cu) and the project-written shim
// headers in oracle/refshim/ into oracle/_ref/libtlfea_ref.so (recipe: oracle/build_ref.py).
// It exposes a plain C ABI so that the fixture generator and the GPU-reference timing can
// drive the reference's classes in the order its example drivers use
// (examples/test_feat10_nesterov.cc:52-199, examples/beam_linear_static.cc:120-194).
// The product library never loads it.
//
// Fields the reference keeps private (the constraint vector, J / J^T CSR, the stiffness CSR
// of LinearStaticSolver, solver velocities) are read through access re-labelled in this
// translation unit only; the class layouts are the reference's.
#include <cooperative_groups.h>
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusparse.h>
#include <thrust/device_ptr.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include <Eigen/Dense>
#include <MoPhiEssentials.h>

#define private public
#define protected public
#include "elements/FEAT10Data.cuh"
#include "elements/FEAT4Data.cuh"
#include "solvers/LinearStaticSolver.cuh"
#include "solvers/SyncedAdamW.cuh"
#include "solvers/SyncedAdamWNocoop.cuh"
#include "solvers/SyncedNesterov.cuh"
#undef private
#undef protected

using namespace tlfea;

// The first-order solvers' constructors name the ANCF elements' precompute for ANCF element
// types (SyncedNesterov.cuh:42-54); the ANCF sources are not part of this harness (FEAT10 /
// TET4 only), so these stand-ins only report misuse if an ANCF element ever reached them.
void tlfea::GPU_ANCF3243_Data::CalcDsDuPre() {
    MOPHI_ERROR("ANCF3243 elements are not built into the reference harness");
}
void tlfea::GPU_ANCF3443_Data::CalcDsDuPre() {
    MOPHI_ERROR("ANCF3443 elements are not built into the reference harness");
}

namespace {

struct RefElement {
    int npe = 0, n_elem = 0, n_node = 0, n_fixed = 0;
    GPU_FEAT10_Data* t10 = nullptr;
    GPU_FEAT4_Data* t4 = nullptr;
    ElementBase* base() const { return t10 ? static_cast<ElementBase*>(t10) : static_cast<ElementBase*>(t4); }
};

struct RefSolver {
    int kind = 0;  // 0 linear static, 1 Nesterov, 2 AdamW, 3 AdamW no-coop
    RefElement* el = nullptr;
    LinearStaticSolver<GPU_FEAT10_Data>* ls10 = nullptr;
    LinearStaticSolver<GPU_FEAT4_Data>* ls4 = nullptr;
    SyncedNesterovSolver* nes = nullptr;
    SyncedAdamWSolver* adw = nullptr;
    SyncedAdamWNocoopSolver* adn = nullptr;
    SyncedNesterovParams np{};
    SyncedAdamWParams ap{};
};

// Status of the last call: the first CUDA failure or MOPHI_ERROR report seen by the shim.
int take_status() {
    mophi::ShimStatus& s = mophi::shim_status();
    cudaError_t pending = cudaGetLastError();
    int rc = 0;
    if (s.cuda_error != 0)
        rc = 2;
    else if (pending != cudaSuccess)
        rc = 2;
    else if (s.n_errors != 0)
        rc = 1;
    s.cuda_error = 0;
    s.n_errors = 0;
    return rc;
}

VectorXR vec(const double* p, int n) {
    VectorXR v(n);
    for (int i = 0; i < n; ++i)
        v(i) = p[i];
    return v;
}

template <typename D>
void copy_csr(int* d_off, int* d_col, double* d_val, int rows, int nnz, int* off, int* col, double* val) {
    if (off)
        cudaMemcpy(off, d_off, sizeof(int) * (rows + 1), cudaMemcpyDeviceToHost);
    if (col)
        cudaMemcpy(col, d_col, sizeof(int) * nnz, cudaMemcpyDeviceToHost);
    if (val)
        cudaMemcpy(val, d_val, sizeof(double) * nnz, cudaMemcpyDeviceToHost);
}

template <typename E>
void setup_element(E* el, int npe, int n_elem, int n_node, const double* x, const double* y, const double* z,
                   const int* conn, const int* fixed, int n_fixed, const double* f_ext, double E_mod, double nu,
                   double rho, double eta, double lamd, int material, double mu10, double mu01, double kappa,
                   int with_mass) {
    el->Initialize();
    if (n_fixed > 0) {
        VectorXi fx(n_fixed);
        for (int i = 0; i < n_fixed; ++i)
            fx(i) = fixed[i];
        el->SetNodalFixed(fx);
    }
    if (f_ext)
        el->SetExternalForce(vec(f_ext, 3 * n_node));
    MatrixXi c(n_elem, npe);
    for (int e = 0; e < n_elem; ++e)
        for (int a = 0; a < npe; ++a)
            c(e, a) = conn[static_cast<size_t>(e) * npe + a];
    if (npe == 10)
        el->Setup(Quadrature::tet5pt_x, Quadrature::tet5pt_y, Quadrature::tet5pt_z, Quadrature::tet5pt_weights,
                  vec(x, n_node), vec(y, n_node), vec(z, n_node), c);
    else
        el->Setup(Quadrature::tet1pt_x, Quadrature::tet1pt_y, Quadrature::tet1pt_z, Quadrature::tet1pt_weights,
                  vec(x, n_node), vec(y, n_node), vec(z, n_node), c);
    el->SetDensity(rho);
    el->SetDamping(eta, lamd);
    if (material == 1)
        el->SetMooneyRivlin(mu10, mu01, kappa);
    else
        el->SetSVK(E_mod, nu);
    el->CalcDnDuPre();
    if (with_mass)
        el->CalcMassMatrix();
    if (n_fixed > 0) {
        el->CalcConstraintData();
        el->ConvertToCSR_ConstraintJacT();
        el->ConvertToCSR_ConstraintJac();
    }
}

// The reference's element constructors leave most scalar members and device pointers
// uninitialised (FEAT10Data.cuh:353-356); start them from zero so unset flags read false.
template <typename E>
E* zeroed_new(int n_elem, int n_node) {
    void* mem = ::operator new(sizeof(E));
    std::memset(mem, 0, sizeof(E));
    return new (mem) E(n_elem, n_node);
}

template <typename Fn>
auto with_element(RefElement* r, Fn&& fn) {
    if (r->t10)
        return fn(r->t10);
    return fn(r->t4);
}

}  // namespace

extern "C" {

// Creates and sets up a TET10 (npe = 10) or TET4 (npe = 4) element object of the reference
// in the call order of examples/test_feat10_nesterov.cc:52-161. conn is row-major
// (n_elem x npe); fixed / f_ext may be null. Returns null on failure.
void* ref_element_create(int npe, int n_elem, int n_node, const double* x, const double* y, const double* z,
                         const int* conn, const int* fixed, int n_fixed, const double* f_ext, double E_mod,
                         double nu, double rho, double eta, double lamd, int material, double mu10, double mu01,
                         double kappa, int with_mass) {
    take_status();
    auto* r = new RefElement();
    r->npe = npe;
    r->n_elem = n_elem;
    r->n_node = n_node;
    r->n_fixed = n_fixed;
    if (npe == 10) {
        r->t10 = zeroed_new<GPU_FEAT10_Data>(n_elem, n_node);
        setup_element(r->t10, npe, n_elem, n_node, x, y, z, conn, fixed, n_fixed, f_ext, E_mod, nu, rho, eta, lamd,
                      material, mu10, mu01, kappa, with_mass);
    } else if (npe == 4) {
        r->t4 = zeroed_new<GPU_FEAT4_Data>(n_elem, n_node);
        setup_element(r->t4, npe, n_elem, n_node, x, y, z, conn, fixed, n_fixed, f_ext, E_mod, nu, rho, eta, lamd,
                      material, mu10, mu01, kappa, with_mass);
    } else {
        delete r;
        return nullptr;
    }
    if (take_status() != 0) {
        with_element(r, [](auto* e) {
            e->Destroy();
            delete e;
            return 0;
        });
        delete r;
        return nullptr;
    }
    return r;
}

int ref_element_destroy(void* h) {
    auto* r = static_cast<RefElement*>(h);
    if (!r)
        return 0;
    with_element(r, [](auto* e) {
        e->Destroy();
        delete e;
        return 0;
    });
    delete r;
    return take_status();
}

// Reference gradients d_grad_N_ref ((e*QP+q)*NPE*3 + a + NPE*j) and detJ (e*QP+q).
int ref_element_grad(void* h, double* grad, double* detj) {
    auto* r = static_cast<RefElement*>(h);
    return with_element(r, [&](auto* e) {
        const int nqp = r->npe == 10 ? 5 : 1;
        const size_t ng = static_cast<size_t>(r->n_elem) * nqp * r->npe * 3;
        if (grad)
            cudaMemcpy(grad, e->d_grad_N_ref, ng * sizeof(double), cudaMemcpyDeviceToHost);
        if (detj)
            cudaMemcpy(detj, e->d_detJ_ref, sizeof(double) * r->n_elem * nqp, cudaMemcpyDeviceToHost);
        return take_status();
    });
}

int ref_element_mass_nnz(void* h) {
    auto* r = static_cast<RefElement*>(h);
    return with_element(r, [&](auto* e) {
        int nnz = 0;
        if (e->is_csr_setup)
            cudaMemcpy(&nnz, e->d_nnz, sizeof(int), cudaMemcpyDeviceToHost);
        return take_status() ? -1 : nnz;
    });
}

// RetrieveMassCSRToCPU (FEAT10Data.cu:634-657).
int ref_element_mass(void* h, int* off, int* col, double* val) {
    auto* r = static_cast<RefElement*>(h);
    return with_element(r, [&](auto* e) {
        std::vector<int> o, c;
        std::vector<Real> v;
        e->RetrieveMassCSRToCPU(o, c, v);
        std::copy(o.begin(), o.end(), off);
        std::copy(c.begin(), c.end(), col);
        std::copy(v.begin(), v.end(), val);
        return take_status();
    });
}

int ref_element_update_positions(void* h, const double* x, const double* y, const double* z) {
    auto* r = static_cast<RefElement*>(h);
    return with_element(r, [&](auto* e) {
        e->UpdatePositions(vec(x, r->n_node), vec(y, r->n_node), vec(z, r->n_node));
        return take_status();
    });
}

// CalcP (no viscous term: FEAT10Data.cu:287-305); P in the reference layout (e*QP+q)*9 + i + 3j.
int ref_element_calc_p(void* h, double* P) {
    auto* r = static_cast<RefElement*>(h);
    return with_element(r, [&](auto* e) {
        e->CalcP();
        if (P) {
            const int nqp = r->npe == 10 ? 5 : 1;
            cudaMemcpy(P, e->d_P, sizeof(double) * 9 * r->n_elem * nqp, cudaMemcpyDeviceToHost);
        }
        return take_status();
    });
}

// CalcInternalForce: adds onto f_int, which only Setup zeroes (FEAT10Data.cu:307-323).
int ref_element_calc_internal_force(void* h, double* f) {
    auto* r = static_cast<RefElement*>(h);
    return with_element(r, [&](auto* e) {
        e->CalcInternalForce();
        if (f) {
            VectorXR fi;
            e->RetrieveInternalForceToCPU(fi);
            std::copy(fi.data(), fi.data() + 3 * r->n_node, f);
        }
        return take_status();
    });
}

int ref_element_positions(void* h, double* x, double* y, double* z) {
    auto* r = static_cast<RefElement*>(h);
    return with_element(r, [&](auto* e) {
        VectorXR a, b, c;
        e->RetrievePositionToCPU(a, b, c);
        std::copy(a.data(), a.data() + r->n_node, x);
        std::copy(b.data(), b.data() + r->n_node, y);
        std::copy(c.data(), c.data() + r->n_node, z);
        return take_status();
    });
}

// Constraint vector c (compute_constraint_data, FEAT10DataFunc.cuh:470-481) after CalcConstraintData.
int ref_element_constraint(void* h, double* c) {
    auto* r = static_cast<RefElement*>(h);
    return with_element(r, [&](auto* e) {
        e->CalcConstraintData();
        if (e->n_constraint > 0)
            cudaMemcpy(c, e->d_constraint, sizeof(double) * e->n_constraint, cudaMemcpyDeviceToHost);
        return take_status();
    });
}

// J (n_constraint rows) and J^T (3N rows) CSR (FEAT10Data.cu:420-562); n_constraint nonzeros each.
int ref_element_constraint_csr(void* h, int* j_off, int* j_col, double* j_val, int* jt_off, int* jt_col,
                               double* jt_val) {
    auto* r = static_cast<RefElement*>(h);
    return with_element(r, [&](auto* e) {
        const int nc = e->n_constraint;
        if (nc > 0) {
            copy_csr<double>(e->d_j_csr_offsets, e->d_j_csr_columns, e->d_j_csr_values, nc, nc, j_off, j_col, j_val);
            copy_csr<double>(e->d_cj_csr_offsets, e->d_cj_csr_columns, e->d_cj_csr_values, 3 * r->n_node, nc, jt_off,
                             jt_col, jt_val);
        }
        return take_status();
    });
}

// Mean wall time (ms) of CalcP + CalcInternalForce over reps calls, after one warm-up call;
// each reference call ends in cudaDeviceSynchronize, so host time is device time plus launch.
double ref_element_time_force(void* h, int reps) {
    auto* r = static_cast<RefElement*>(h);
    return with_element(r, [&](auto* e) {
        e->CalcP();
        e->CalcInternalForce();
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        for (int i = 0; i < reps; ++i) {
            e->CalcP();
            e->CalcInternalForce();
        }
        cudaDeviceSynchronize();
        auto t1 = std::chrono::steady_clock::now();
        if (take_status() != 0)
            return -1.0;
        return std::chrono::duration<double, std::milli>(t1 - t0).count() / reps;
    });
}

// LinearStaticSolver<T>(data, tol, max_iter) (LinearStaticSolver.cuh:56).
void* ref_linear_static_create(void* h, double tol, int max_iter) {
    auto* r = static_cast<RefElement*>(h);
    auto* s = new RefSolver();
    s->kind = 0;
    s->el = r;
    if (r->t10)
        s->ls10 = new LinearStaticSolver<GPU_FEAT10_Data>(r->t10, tol, max_iter);
    else
        s->ls4 = new LinearStaticSolver<GPU_FEAT4_Data>(r->t4, tol, max_iter);
    if (take_status() != 0) {
        delete s->ls10;
        delete s->ls4;
        delete s;
        return nullptr;
    }
    return s;
}

// Solve() (LinearStaticSolver.cu:590-603); ms = host wall time of the call.
int ref_linear_static_solve(void* sh, int* iters, double* residual, double* ms) {
    auto* s = static_cast<RefSolver*>(sh);
    auto t0 = std::chrono::steady_clock::now();
    if (s->ls10)
        s->ls10->Solve();
    else
        s->ls4->Solve();
    cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    if (ms)
        *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (iters)
        *iters = s->ls10 ? s->ls10->GetLastIterCount() : s->ls4->GetLastIterCount();
    if (residual)
        *residual = s->ls10 ? s->ls10->GetLastResidual() : s->ls4->GetLastResidual();
    return take_status();
}

// Stiffness CSR after Solve (K with the Dirichlet rows/columns applied, 3N rows). nnz only if
// off == null.
int ref_linear_static_k(void* sh, int* off, int* col, double* val) {
    auto* s = static_cast<RefSolver*>(sh);
    auto get = [&](auto* ls) {
        if (!off)
            return ls->K_nnz_;
        copy_csr<double>(ls->d_K_offsets_, ls->d_K_columns_, ls->d_K_values_, ls->n_dof_, ls->K_nnz_, off, col, val);
        return take_status();
    };
    return s->ls10 ? get(s->ls10) : get(s->ls4);
}

// SyncedNesterovSolver(data, n_constraints), Setup, SetParameters
// (examples/test_feat10_nesterov.cc:189-194).
void* ref_nesterov_create(void* h, double alpha, double rho, double inner_tol, double outer_tol, int max_outer,
                          int max_inner, double dt) {
    auto* r = static_cast<RefElement*>(h);
    auto* s = new RefSolver();
    s->kind = 1;
    s->el = r;
    s->np = SyncedNesterovParams{alpha, rho, inner_tol, outer_tol, max_outer, max_inner, dt};
    ElementBase* b = r->base();
    s->nes = new SyncedNesterovSolver(b, r->n_fixed * 3);
    s->nes->Setup();
    s->nes->SetParameters(&s->np);
    if (take_status() != 0) {
        delete s->nes;
        delete s;
        return nullptr;
    }
    return s;
}

// SyncedAdamWSolver (nocoop = 0) or SyncedAdamWNocoopSolver (nocoop = 1) with SyncedAdamWParams
// field for field (SyncedAdamW.cuh:32-39).
void* ref_adamw_create(void* h, int nocoop, double lr, double beta1, double beta2, double eps, double weight_decay,
                       double lr_decay, double inner_tol, double outer_tol, double rho, int max_outer, int max_inner,
                       double dt, int check_interval, double inner_rtol) {
    auto* r = static_cast<RefElement*>(h);
    auto* s = new RefSolver();
    s->kind = nocoop ? 3 : 2;
    s->el = r;
    s->ap = SyncedAdamWParams{lr,  beta1,     beta2,     eps, weight_decay,   lr_decay,  inner_tol,
                              outer_tol, rho, max_outer, max_inner, dt, check_interval, inner_rtol};
    ElementBase* b = r->base();
    if (nocoop) {
        s->adn = new SyncedAdamWNocoopSolver(b, r->n_fixed * 3);
        s->adn->Setup();
        s->adn->SetParameters(&s->ap);
    } else {
        s->adw = new SyncedAdamWSolver(b, r->n_fixed * 3);
        s->adw->Setup();
        s->adw->SetParameters(&s->ap);
    }
    if (take_status() != 0) {
        delete s->adn;
        delete s->adw;
        delete s;
        return nullptr;
    }
    return s;
}

// n_steps calls of Solve() (one implicit step each); ms = host wall time of all of them.
int ref_solver_steps(void* sh, int n_steps, double* ms) {
    auto* s = static_cast<RefSolver*>(sh);
    auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < n_steps; ++k) {
        if (s->nes)
            s->nes->Solve();
        else if (s->adw)
            s->adw->Solve();
        else if (s->adn)
            s->adn->Solve();
        if (mophi::shim_status().cuda_error != 0 || mophi::shim_status().n_errors != 0)
            break;
    }
    cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    if (ms)
        *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return take_status();
}

// The solver's current velocity iterate v_guess (3N, interleaved).
int ref_solver_velocity(void* sh, double* v) {
    auto* s = static_cast<RefSolver*>(sh);
    const int n = 3 * s->el->n_node;
    const double* d = s->nes ? s->nes->d_v_guess_ : (s->adw ? s->adw->d_v_guess_ : s->adn->d_v_guess_);
    cudaMemcpy(v, d, sizeof(double) * n, cudaMemcpyDeviceToHost);
    return take_status();
}

int ref_solver_destroy(void* sh) {
    auto* s = static_cast<RefSolver*>(sh);
    if (!s)
        return 0;
    delete s->ls10;
    delete s->ls4;
    delete s->nes;
    delete s->adw;
    delete s->adn;
    delete s;
    return take_status();
}

// Where the first CUDA failure of the shim was recorded (empty if none).
int ref_last_error(char* buf, int n) {
    std::snprintf(buf, n, "%s", mophi::shim_status().where);
    return mophi::shim_status().cuda_error;
}

}  // extern "C"
