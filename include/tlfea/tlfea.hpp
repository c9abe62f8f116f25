// tlfea/tlfea.hpp -- header-only C++ classes with the reference's names and
// methods (src/FEASolver.h, src/elements/FEAT10Data.cuh, FEAT4Data.cuh,
// src/solvers/SyncedNesterov.cuh, SyncedAdamW.cuh, SyncedAdamWNocoop.cuh,
// LinearStaticSolver.cuh), each method forwarding to one call of the C ABI in
// tlfea_b200.h.  Eigen vectors become std::vector<double> (x, y, z SoA; forces
// interleaved [3*node + d]); MatrixXi connectivity is an E x NPE column-major
// std::vector<int> (MatrixXi::data() order).  A failing call logs the library's
// message to stderr and returns, as the reference's MOPHI_ERROR does;
// FEASolver throws std::invalid_argument / std::out_of_range like the reference.
// Link with -ltlfea_b200 (tlfea_b200/libtlfea_b200.so).
#pragma once

#include <algorithm>
#include <cstdio>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../tlfea_b200.h"

namespace tlfea_cxx {

using Real = double;
using VectorXR = std::vector<Real>;

enum ElementType { TYPE_3243 = 0, TYPE_3443 = 1, TYPE_T10 = 2, TYPE_T4 = 3 };

// Logs a non-OK status with the library's message; returns true on success.
inline bool check(int status, const char* what) {
    if (status == TLFEA_OK) return true;
    std::fprintf(stderr, "tlfea_b200: %s failed (status %d): %s\n", what, status, tlfea_last_error());
    return false;
}

// ElementBase (ElementBase.h:24-48)
class ElementBase {
  public:
    virtual ~ElementBase() = default;
    ElementType type = TYPE_T10;
    int n_elem = 0, n_coef = 0, n_constraint = 0;
    int get_n_beam() const { return n_elem; }
    int get_n_coef() const { return n_coef; }
    int get_n_constraint() const { return n_constraint; }
    virtual void CalcMassMatrix() = 0;
    virtual void CalcInternalForce() = 0;
    virtual void CalcConstraintData() = 0;
    virtual void CalcP() = 0;
    virtual void RetrieveInternalForceToCPU(VectorXR& f) = 0;
    tlfea_element handle() const { return h_; }

  protected:
    tlfea_element h_ = nullptr;
};

// GPU_FEAT10_Data / GPU_FEAT4_Data (FEAT10Data.cuh:291-731; FEAT4Data.cuh)
template <int NPE, ElementType TYPE>
class GPU_TetData : public ElementBase {
  public:
    GPU_TetData(int num_elements, int num_nodes) {
        type = TYPE;
        n_elem = num_elements;
        n_coef = num_nodes;
    }
    void Initialize() { check(tlfea_element_create(TYPE, n_elem, n_coef, &h_), "Initialize"); }
    void Destroy() {
        if (h_) tlfea_element_destroy(h_);
        h_ = nullptr;
    }
    void Setup(const VectorXR& qx, const VectorXR& qy, const VectorXR& qz, const VectorXR& qw, const VectorXR& x,
               const VectorXR& y, const VectorXR& z, const std::vector<int>& conn_colmajor) {
        check(tlfea_element_setup(h_, qx.data(), qy.data(), qz.data(), qw.data(), (int)qx.size(), x.data(), y.data(),
                                  z.data(), conn_colmajor.data()),
              "Setup");
    }
    void SetDensity(Real rho0) { check(tlfea_element_set_density(h_, rho0), "SetDensity"); }
    void SetDamping(Real eta, Real lambda) { check(tlfea_element_set_damping(h_, eta, lambda), "SetDamping"); }
    void SetSVK() { check(tlfea_element_set_svk_default(h_), "SetSVK"); }
    void SetSVK(Real E, Real nu) { check(tlfea_element_set_svk(h_, E, nu), "SetSVK"); }
    void SetMooneyRivlin(Real mu10, Real mu01, Real kappa) {
        check(tlfea_element_set_mooney_rivlin(h_, mu10, mu01, kappa), "SetMooneyRivlin");
    }
    void SetExternalForce(const VectorXR& f) {
        check(tlfea_element_set_external_force(h_, f.data(), (int)f.size()), "SetExternalForce");
    }
    // new: f_ext += M g (consistent-mass row sums); after CalcMassMatrix
    void AddGravity(Real gx, Real gy, Real gz) { check(tlfea_element_add_gravity(h_, gx, gy, gz), "AddGravity"); }
    void SetNodalFixed(const std::vector<int>& nodes) {
        if (check(tlfea_element_set_nodal_fixed(h_, nodes.data(), (int)nodes.size()), "SetNodalFixed"))
            n_constraint = 3 * (int)nodes.size();
    }
    void UpdateNodalFixed(const std::vector<int>& nodes) {
        if (check(tlfea_element_update_nodal_fixed(h_, nodes.data(), (int)nodes.size()), "UpdateNodalFixed"))
            n_constraint = 3 * (int)nodes.size();
    }
    void UpdatePositions(const VectorXR& x, const VectorXR& y, const VectorXR& z) {
        check(tlfea_element_update_positions(h_, x.data(), y.data(), z.data(), (int)x.size()), "UpdatePositions");
    }
    void UpdateConstraintTargets(const VectorXR& x, const VectorXR& y, const VectorXR& z) {
        check(tlfea_element_update_constraint_targets(h_, x.data(), y.data(), z.data(), (int)x.size()),
              "UpdateConstraintTargets");
    }
    void CalcDnDuPre() { check(tlfea_element_calc_dndu_pre(h_), "CalcDnDuPre"); }
    void CalcMassMatrix() override { check(tlfea_element_calc_mass_matrix(h_), "CalcMassMatrix"); }
    void CalcP() override { check(tlfea_element_calc_p(h_), "CalcP"); }
    void CalcInternalForce() override { check(tlfea_element_calc_internal_force(h_), "CalcInternalForce"); }
    void CalcConstraintData() override { check(tlfea_element_calc_constraint_data(h_), "CalcConstraintData"); }
    void ConvertToCSR_ConstraintJacT() {
        check(tlfea_element_build_constraint_jact_csr(h_), "ConvertToCSR_ConstraintJacT");
    }
    void ConvertToCSR_ConstraintJac() { check(tlfea_element_build_constraint_jac_csr(h_), "ConvertToCSR_ConstraintJac"); }
    // new: the fused internal force (one pass, deterministic)
    void ComputeInternalForce(const double* d_v = nullptr) {
        check(tlfea_element_compute_internal_force(h_, d_v), "ComputeInternalForce");
    }
    void RetrieveInternalForceToCPU(VectorXR& f) override {
        f.assign(3 * (size_t)n_coef, 0.0);
        check(tlfea_element_retrieve_internal_force(h_, f.data(), (int)f.size()), "RetrieveInternalForceToCPU");
    }
    void RetrieveExternalForceToCPU(VectorXR& f) {
        f.assign(3 * (size_t)n_coef, 0.0);
        check(tlfea_element_retrieve_external_force(h_, f.data(), (int)f.size()), "RetrieveExternalForceToCPU");
    }
    void RetrievePositionToCPU(VectorXR& x, VectorXR& y, VectorXR& z) {
        x.assign(n_coef, 0.0);
        y.assign(n_coef, 0.0);
        z.assign(n_coef, 0.0);
        check(tlfea_element_retrieve_positions(h_, x.data(), y.data(), z.data(), n_coef), "RetrievePositionToCPU");
    }
    // mass CSR (offsets N+1, columns, values)
    void RetrieveMassCSRToCPU(std::vector<int>& off, std::vector<int>& col, VectorXR& val) {
        long long nnz = 0;
        if (!check(tlfea_element_get_mass_nnz(h_, &nnz), "RetrieveMassCSRToCPU")) return;
        off.assign((size_t)n_coef + 1, 0);
        col.assign((size_t)nnz, 0);
        val.assign((size_t)nnz, 0.0);
        check(tlfea_element_retrieve_mass_csr(h_, off.data(), col.data(), val.data()), "RetrieveMassCSRToCPU");
    }
    void WriteOutputVTK(const std::string& file) { check(tlfea_element_write_vtk(h_, file.c_str()), "WriteOutputVTK"); }
};

using GPU_FEAT10_Data = GPU_TetData<10, TYPE_T10>;
using GPU_FEAT4_Data = GPU_TetData<4, TYPE_T4>;

// SolverBase (FEASolver.h:22-28)
class SolverBase {
  public:
    virtual ~SolverBase() {
        if (s_) tlfea_solver_destroy(s_);
    }
    virtual void Solve() { check(tlfea_solver_solve(s_), "Solve"); }
    virtual void SetParameters(void* params) { check(tlfea_solver_set_parameters(s_, params), "SetParameters"); }
    void Setup() { check(tlfea_solver_setup(s_), "Setup"); }
    tlfea_solve_stats GetStats() const {
        tlfea_solve_stats st{};
        tlfea_solver_get_stats(s_, &st);
        return st;
    }
    // new: ||(f_int - f_ext)_free|| / ||f_ext|| < rel_tol ends a solve (0 = off)
    void SetRelativeResidualStop(double rel_tol) { check(tlfea_solver_set_stop_rule(s_, rel_tol), "SetStopRule"); }
    // new: n_steps Solve() calls in one graph launch, load f_base + amp sin(omega t_k + phase) f_var
    // (f_var empty = constant load); returns each step's total inner iterations
    std::vector<int> RunSteps(int n_steps, const VectorXR& f_var = {}, double amp = 1.0, double omega = 0.0,
                              double phase = 0.0, double t0 = 0.0) {
        std::vector<int> its((size_t)std::max(n_steps, 1), 0);
        check(tlfea_solver_run_steps(s_, n_steps, t0, f_var.empty() ? nullptr : f_var.data(), amp, omega, phase,
                                     its.data()),
              "RunSteps");
        return its;
    }

  protected:
    tlfea_solver s_ = nullptr;
};

using SyncedNesterovParams = tlfea_nesterov_params;
using SyncedAdamWParams = tlfea_adamw_params;
using SyncedAdamWNocoopParams = tlfea_adamw_params;

class SyncedNesterovSolver : public SolverBase {
  public:
    SyncedNesterovSolver(ElementBase* data, int n_constraints) {
        check(tlfea_nesterov_create(data->handle(), n_constraints, &s_), "SyncedNesterovSolver");
    }
};

class SyncedAdamWSolver : public SolverBase {
  public:
    SyncedAdamWSolver(ElementBase* data, int n_constraints) {
        check(tlfea_adamw_create(data->handle(), n_constraints, &s_), "SyncedAdamWSolver");
    }
};

class SyncedAdamWNocoopSolver : public SolverBase {
  public:
    SyncedAdamWNocoopSolver(ElementBase* data, int n_constraints) {
        check(tlfea_adamw_nocoop_create(data->handle(), n_constraints, &s_), "SyncedAdamWNocoopSolver");
    }
};

// LinearStaticSolver<T> (LinearStaticSolver.cuh:44-117)
template <typename T>
class LinearStaticSolver : public SolverBase {
  public:
    LinearStaticSolver(T* data, Real tol = 1e-10, int max_iter = 10000) {
        check(tlfea_linear_static_create(data->handle(), tol, max_iter, &s_), "LinearStaticSolver");
    }
    void SetParameters(void*) override {}
    // new, opt-in: 1 = block Jacobi on the 3x3 node diagonal blocks, 0 = none (default)
    void SetPreconditioner(int kind) {
        check(tlfea_linear_static_set_preconditioner(s_, kind), "SetPreconditioner");
    }
    int GetLastIterCount() const {
        int it = 0;
        double r = 0.0;
        tlfea_linear_static_last(s_, &it, &r);
        return it;
    }
    Real GetLastResidual() const {
        int it = 0;
        double r = 0.0;
        tlfea_linear_static_last(s_, &it, &r);
        return r;
    }
};

// FEASolver (FEASolver.h:35-138): a name -> non-owning pointer registry.
class FEASolver {
  public:
    void AddElement(const std::string& name, ElementBase* e) {
        if (!e) throw std::invalid_argument("FEASolver::AddElement: element pointer is null");
        if (elements_.count(name)) throw std::invalid_argument("FEASolver::AddElement: element '" + name + "' exists");
        elements_[name] = e;
    }
    void AddSolver(const std::string& name, SolverBase* s) {
        if (!s) throw std::invalid_argument("FEASolver::AddSolver: solver pointer is null");
        if (solvers_.count(name)) throw std::invalid_argument("FEASolver::AddSolver: solver '" + name + "' exists");
        solvers_[name] = s;
    }
    ElementBase* GetElement(const std::string& name) {
        auto it = elements_.find(name);
        if (it == elements_.end()) throw std::out_of_range("FEASolver::GetElement: no element '" + name + "'");
        return it->second;
    }
    SolverBase* GetSolver(const std::string& name) {
        auto it = solvers_.find(name);
        if (it == solvers_.end()) throw std::out_of_range("FEASolver::GetSolver: no solver '" + name + "'");
        return it->second;
    }
    int GetNumElements() const { return (int)elements_.size(); }
    int GetNumSolvers() const { return (int)solvers_.size(); }

  private:
    std::map<std::string, ElementBase*> elements_;
    std::map<std::string, SolverBase*> solvers_;
};

}  // namespace tlfea_cxx
