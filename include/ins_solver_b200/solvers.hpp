// C++ classes with the names and call signatures that INS-Solver's time-step code
// uses for its pressure and viscous solves, implemented over the C ABI of
// sipg_b200.h. A solver built from them is a drop-in for:
//   LinearSolver and its subclasses  PETScPMultigrid, PETScJacobiSolver,
//     PETScBlockJacobiSolver, PETScInvMassSolver (configured at
//     src/solvers/3d/ins_solver_base.cpp:149-184, :1522-1536; solve at
//     ins_solver.cpp:345, mp_ins_solver.cpp:632, :852);
//   the matrix classes PoissonMatrixFreeDiag3D, FactorPoissonMatrixFreeDiag3D,
//     MMPoissonMatrixFree3D, FactorMMPoissonMatrixFreeDiag3D / BlockDiag3D,
//     PoissonCoarseMatrix3D / FactorPoissonCoarseMatrix3D (ins_solver.cpp:91-139,
//     mp_ins_solver.cpp:85-89);
//   Matrix3Vec, FactorViscousMatrix3D, ViscousMatrix3D and ViscousSolver3D
//     (include/slip_matrix/3d/*.h);
//   initial_guess_extrapolation / add_to_pr_history (ins_solver_base.cpp:1374-1388);
//   the element-local velocity projection of INSSolverBase3D/2D::project_velocity
//     with div_div = 1 (ins_solver_base.cpp:1052-1124, 2D :894-955).
//
// The reference passes OP2 op_dats; here an op_dat is represented by a view of
// its host array (Dat: `dim` values per set element, element-major, which is the
// layout of an op_dat in OP2's CPU builds). Failures the reference reports with
// dg_abort throw ins_solver_b200::SolverError; solve() returns false when the solver did not
// converge, as in the reference.
#pragma once

#include <algorithm>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../sipg_b200.h"

namespace ins_solver_b200 {

struct SolverError : std::runtime_error {
  int status;
  SolverError(int st, const std::string& what) : std::runtime_error(what), status(st) {}
};

inline void check(int st, const char* what) {
  if (st != SIPG_OK) throw SolverError(st, std::string(what) + ": " + sipg_last_error());
}

// View of an op_dat's host array.
struct Dat {
  double* data = nullptr;
  int set_size = 0;
  int dim = 0;
  size_t size() const { return (size_t)set_size * dim; }
};
struct IntDat {
  int* data = nullptr;
  int set_size = 0;
  int dim = 1;
};

// Resident mesh (DGMesh3D / DGMesh2D): vertices and element-to-vertex lists.
class DGMesh {
 public:
  DGMesh(int dim, int num_vertices, const double* coords, int num_cells, const int* cell2vertices) {
    check(sipg_mesh_create(dim, num_vertices, coords, num_cells, cell2vertices, &m_), "mesh");
    check(sipg_mesh_sizes(m_, &cells_, &faces_, &bfaces_), "mesh sizes");
    dim_ = dim;
  }
  ~DGMesh() { sipg_mesh_destroy(m_); }
  DGMesh(const DGMesh&) = delete;
  DGMesh& operator=(const DGMesh&) = delete;
  sipg_mesh* handle() const { return m_; }
  int dim() const { return dim_; }
  int num_cells() const { return cells_; }
  int num_bfaces() const { return bfaces_; }

 private:
  sipg_mesh* m_ = nullptr;
  int dim_ = 0, cells_ = 0, faces_ = 0, bfaces_ = 0;
};
class DGMesh3D : public DGMesh {
 public:
  DGMesh3D(int nv, const double* coords, int k, const int* c2v) : DGMesh(3, nv, coords, k, c2v) {}
};
class DGMesh2D : public DGMesh {
 public:
  DGMesh2D(int nv, const double* coords, int k, const int* c2v) : DGMesh(2, nv, coords, k, c2v) {}
};

// ---- scalar operators (PoissonMatrix family)
class PoissonMatrix {
 public:
  virtual ~PoissonMatrix() { sipg_op_destroy(op_); }
  PoissonMatrix(const PoissonMatrix&) = delete;
  PoissonMatrix& operator=(const PoissonMatrix&) = delete;
  // 0 Dirichlet, 1 Neumann per boundary face (problem_specific_3d.h:31-32)
  virtual void set_bc_types(IntDat bc_types) {
    check(sipg_op_set_bc_types(op_, bc_types.data), "set_bc_types");
    ++version_;
  }
  // y = A x on host arrays (mult of the matrix-free classes)
  void mult(Dat in, Dat out) {
    check(sipg_op_apply_host(op_, in.data, out.data), "mult");
  }
  // rhs += lifted boundary data (apply_bc)
  void apply_bc(Dat rhs, Dat bc) { check(sipg_op_apply_bc_host(op_, bc.data, rhs.data), "apply_bc"); }
  sipg_op* handle() const { return op_; }
  unsigned version() const { return version_; }
  DGMesh* mesh() const { return mesh_; }

 protected:
  PoissonMatrix(DGMesh* m, int order, int ncomp = 1) : mesh_(m) {
    check(sipg_op_create(m->handle(), order, ncomp, &op_), "operator");
  }
  sipg_op* op_ = nullptr;
  DGMesh* mesh_ = nullptr;
  unsigned version_ = 0;
};

class PoissonMatrixFreeDiag3D : public PoissonMatrix {
 public:
  explicit PoissonMatrixFreeDiag3D(DGMesh* m, int order = 3) : PoissonMatrix(m, order) {}
};
class PoissonMatrixFreeDiag2D : public PoissonMatrixFreeDiag3D {
 public:
  explicit PoissonMatrixFreeDiag2D(DGMesh* m, int order = 3) : PoissonMatrixFreeDiag3D(m, order) {}
};

// -div(f grad u) with a nodal factor f (mp_ins_solver.cpp:515-521: f = 1/rho)
class FactorPoissonMatrixFreeDiag3D : public PoissonMatrixFreeDiag3D {
 public:
  explicit FactorPoissonMatrixFreeDiag3D(DGMesh* m, int order = 3) : PoissonMatrixFreeDiag3D(m, order) {}
  void set_factor(Dat f) {
    check(sipg_op_set_factor(op_, f.data), "set_factor");
    ++version_;
  }
};
using FactorPoissonMatrixFreeDiag2D = FactorPoissonMatrixFreeDiag3D;

// Helmholtz c M + K with a scalar c (MMPoissonMatrixFree3D::set_factor / get_factor)
class MMPoissonMatrixFree3D : public PoissonMatrix {
 public:
  explicit MMPoissonMatrixFree3D(DGMesh* m, int order = 3) : PoissonMatrix(m, order) {}
  void set_factor(double c) {
    check(sipg_op_set_mm(op_, SIPG_MM_SCALAR, c, nullptr), "set_factor");
    c_ = c;
    ++version_;
  }
  double get_factor() const { return c_; }

 private:
  double c_ = 0.0;
};

// Helmholtz with nodal factors: mm_factor M + K_f
class FactorMMPoissonMatrixFreeDiag3D : public FactorPoissonMatrixFreeDiag3D {
 public:
  explicit FactorMMPoissonMatrixFreeDiag3D(DGMesh* m, int order = 3) : FactorPoissonMatrixFreeDiag3D(m, order) {}
  void set_mm_factor(Dat mm) {
    check(sipg_op_set_mm(op_, SIPG_MM_NODAL, 0.0, mm.data), "set_mm_factor");
    ++version_;
  }
  // the diagonal / block diagonal are computed by the solver's set-up
  void calc_mat_partial() {}
};
using FactorMMPoissonMatrixFreeBlockDiag3D = FactorMMPoissonMatrixFreeDiag3D;

// The p-multigrid derives its coarse levels from the fine operator; the coarse
// matrix objects of the reference keep their interface and carry no data.
class PoissonCoarseMatrix {
 public:
  virtual ~PoissonCoarseMatrix() = default;
  virtual void set_bc_types(IntDat) {}
};
class PoissonCoarseMatrix3D : public PoissonCoarseMatrix {
 public:
  explicit PoissonCoarseMatrix3D(DGMesh*) {}
};
class FactorPoissonCoarseMatrix3D : public PoissonCoarseMatrix3D {
 public:
  explicit FactorPoissonCoarseMatrix3D(DGMesh* m) : PoissonCoarseMatrix3D(m) {}
  void set_factor(Dat) {}
};

// ---- LinearSolver family
class LinearSolver {
 public:
  enum Solvers { PETSC_AMG, PETSC_JACOBI, PETSC_BLOCK_JACOBI, PETSC_INV_MASS, PETSC_PMULTIGRID };
  virtual ~LinearSolver() {
    if (s_) sipg_solver_destroy(s_);
  }
  LinearSolver(const LinearSolver&) = delete;
  LinearSolver& operator=(const LinearSolver&) = delete;
  virtual void set_matrix(PoissonMatrix* m) {
    if (m != matrix_ && s_) {
      sipg_solver_destroy(s_);
      s_ = nullptr;
    }
    matrix_ = m;
  }
  void set_bcs(Dat bcs) { bcs_ = bcs; }
  void set_nullspace(bool ns) {
    opts_.nullspace = ns ? 1 : 0;
    rebuild_ = true;
  }
  void set_tol_and_iter(double rtol, double atol, int max_iter) {
    opts_.rel_tol = rtol;
    opts_.abs_tol = atol;
    opts_.max_iter = max_iter;
    rebuild_ = true;
  }
  virtual void init() {}
  // Solve A ans = rhs (+ lifted boundary data); ans holds the initial guess.
  virtual bool solve(Dat rhs, Dat ans) {
    if (!matrix_) throw SolverError(SIPG_INVALID_ARG, "solve: no matrix");
    ensure();
    std::vector<double> b(rhs.data, rhs.data + rhs.size());
    if (bcs_.data) check(sipg_op_apply_bc_host(matrix_->handle(), bcs_.data, b.data()), "apply_bc");
    int st = sipg_solver_solve_host(s_, b.data(), ans.data, &info_);
    if (st != SIPG_OK && st != SIPG_NOT_CONVERGED && st != SIPG_BREAKDOWN) check(st, "solve");
    return st == SIPG_OK;
  }
  const sipg_solve_info& last_info() const { return info_; }
  sipg_solver_opts& options() {
    rebuild_ = true;
    return opts_;
  }

 protected:
  explicit LinearSolver(int kind) : kind_(kind) { check(sipg_solver_default_opts(kind, &opts_), "options"); }
  void ensure() {
    if (s_ && rebuild_) {
      sipg_solver_destroy(s_);
      s_ = nullptr;
    }
    if (!s_) {
      check(sipg_solver_create(matrix_->handle(), kind_, &opts_, &s_), "solver");
      seen_ = matrix_->version();
      rebuild_ = false;
      return;
    }
    if (seen_ != matrix_->version()) {  // coefficients changed since the last set-up
      check(sipg_solver_setup(s_), "setup");
      seen_ = matrix_->version();
    }
  }
  int kind_;
  sipg_solver_opts opts_{};
  sipg_solver* s_ = nullptr;
  PoissonMatrix* matrix_ = nullptr;
  Dat bcs_{};
  sipg_solve_info info_{};
  unsigned seen_ = 0;
  bool rebuild_ = false;
};

class PETScPMultigrid : public LinearSolver {
 public:
  explicit PETScPMultigrid(DGMesh*) : LinearSolver(SIPG_SOLVER_PMULTIGRID) {}
  void set_coarse_matrix(PoissonCoarseMatrix*) {}
  // SIPG_FP32: the V-cycle in FP32 on the tensor cores, outer CG in FP64 (default SIPG_FP64)
  void set_precision(int precision) {
    opts_.precision = precision;
    rebuild_ = true;
  }
};
class PETScJacobiSolver : public LinearSolver {
 public:
  explicit PETScJacobiSolver(DGMesh*) : LinearSolver(SIPG_SOLVER_JACOBI) {}
};
class PETScBlockJacobiSolver : public LinearSolver {
 public:
  explicit PETScBlockJacobiSolver(DGMesh*) : LinearSolver(SIPG_SOLVER_BLOCK_JACOBI) {}
};
class PETScInvMassSolver : public LinearSolver {
 public:
  explicit PETScInvMassSolver(DGMesh*) : LinearSolver(SIPG_SOLVER_INV_MASS) {}
  void setFactor(double f) {
    opts_.inv_mass_factor = f;
    rebuild_ = true;
  }
};

// ---- three-component viscous operators (include/slip_matrix/3d/matrix_3_vec.h)
class Matrix3Vec {
 public:
  virtual ~Matrix3Vec() { sipg_op_destroy(op_); }
  Matrix3Vec(const Matrix3Vec&) = delete;
  Matrix3Vec& operator=(const Matrix3Vec&) = delete;
  // 0 Dirichlet, 1 Neumann, 2 slip per boundary face and component
  virtual void set_bc_types(IntDat u, IntDat v, IntDat w) {
    const int kb = u.set_size;
    std::vector<int> t(3 * (size_t)kb);
    for (int i = 0; i < kb; ++i) {
      t[i] = u.data[i];
      t[kb + i] = v.data[i];
      t[2 * kb + i] = w.data[i];
    }
    check(sipg_op_set_bc_types(op_, t.data()), "set_bc_types");
    ++version_;
  }
  virtual void apply_bc(Dat u_rhs, Dat v_rhs, Dat w_rhs, Dat u_bc, Dat v_bc, Dat w_bc) {
    std::vector<double> rhs = pack(u_rhs, v_rhs, w_rhs), bc = pack(u_bc, v_bc, w_bc);
    check(sipg_op_apply_bc_host(op_, bc.data(), rhs.data()), "apply_bc");
    unpack(rhs, u_rhs, v_rhs, w_rhs);
  }
  virtual void mult(Dat u_in, Dat v_in, Dat w_in, Dat u_out, Dat v_out, Dat w_out) {
    std::vector<double> x = pack(u_in, v_in, w_in), y(x.size());
    check(sipg_op_apply_host(op_, x.data(), y.data()), "mult");
    unpack(y, u_out, v_out, w_out);
  }
  sipg_op* handle() const { return op_; }
  unsigned version() const { return version_; }

  static std::vector<double> pack(Dat u, Dat v, Dat w) {
    std::vector<double> p;
    p.reserve(3 * u.size());
    p.insert(p.end(), u.data, u.data + u.size());
    p.insert(p.end(), v.data, v.data + v.size());
    p.insert(p.end(), w.data, w.data + w.size());
    return p;
  }
  static void unpack(const std::vector<double>& p, Dat u, Dat v, Dat w) {
    const size_t n = u.size();
    std::copy(p.begin(), p.begin() + n, u.data);
    std::copy(p.begin() + n, p.begin() + 2 * n, v.data);
    std::copy(p.begin() + 2 * n, p.begin() + 3 * n, w.data);
  }

 protected:
  Matrix3Vec(DGMesh* m, int order) { check(sipg_op_create(m->handle(), order, m->dim(), &op_), "operator"); }
  sipg_op* op_ = nullptr;
  unsigned version_ = 0;
};

// c M + K on (u, v, w) with slip coupling, scalar c (viscous_matrix.h)
class ViscousMatrix3D : public Matrix3Vec {
 public:
  explicit ViscousMatrix3D(DGMesh* m, int order = 3) : Matrix3Vec(m, order) {}
  void set_factor(double c) {
    check(sipg_op_set_mm(op_, SIPG_MM_SCALAR, c, nullptr), "set_factor");
    c_ = c;
    ++version_;
  }
  double get_factor() const { return c_; }

 private:
  double c_ = 0.0;
};

// mm_factor M + K_f on (u, v, w) (factor_viscous_matrix.h)
class FactorViscousMatrix3D : public Matrix3Vec {
 public:
  explicit FactorViscousMatrix3D(DGMesh* m, bool = false, bool = false, int order = 3) : Matrix3Vec(m, order) {}
  void set_factor(Dat f) {
    check(sipg_op_set_factor(op_, f.data), "set_factor");
    ++version_;
  }
  void set_mm_factor(Dat mm) {
    check(sipg_op_set_mm(op_, SIPG_MM_NODAL, 0.0, mm.data), "set_mm_factor");
    ++version_;
  }
  void calc_diag() {}
  void calc_inv_block_diag() {}
};

class ViscousSolver3D {
 public:
  enum Preconditioners { NONE, INV_MASS, FACTOR_INV_MASS, RECP_FACTOR_DAT_INV_MASS, JACOBI, BLOCK_JACOBI };
  explicit ViscousSolver3D(DGMesh*) {}
  virtual ~ViscousSolver3D() {
    if (s_) sipg_solver_destroy(s_);
  }
  ViscousSolver3D(const ViscousSolver3D&) = delete;
  ViscousSolver3D& operator=(const ViscousSolver3D&) = delete;
  virtual void set_matrix(Matrix3Vec* m) {
    if (m != matrix_) drop();
    matrix_ = m;
  }
  void set_bcs(Dat u_bcs, Dat v_bcs, Dat w_bcs) {
    u_bc_ = u_bcs;
    v_bc_ = v_bcs;
    w_bc_ = w_bcs;
  }
  void set_nullspace(bool ns) {
    nullspace_ = ns;
    drop();
  }
  virtual void set_tol_and_iter(double rtol, double atol, int maxiter) {
    rtol_ = rtol;
    atol_ = atol;
    max_iter_ = maxiter;
    drop();
  }
  virtual void set_preconditioner(Preconditioners p) {
    pre_ = p;
    drop();
  }
  void set_inv_mass_factor(double f) {
    inv_mass_factor_ = f;
    drop();
  }
  // solve (viscous_solver.cpp:63-86): lift the boundary data, then (P)CG with the
  // reference's absolute stopping test (abs_tol; rel_tol is kept as given)
  virtual bool solve(Dat u_rhs, Dat v_rhs, Dat w_rhs, Dat u_ans, Dat v_ans, Dat w_ans) {
    if (!matrix_) throw SolverError(SIPG_INVALID_ARG, "solve: no matrix");
    if (u_bc_.data) matrix_->apply_bc(u_rhs, v_rhs, w_rhs, u_bc_, v_bc_, w_bc_);
    ensure();
    std::vector<double> b = Matrix3Vec::pack(u_rhs, v_rhs, w_rhs), x = Matrix3Vec::pack(u_ans, v_ans, w_ans);
    int st = sipg_solver_solve_host(s_, b.data(), x.data(), &info_);
    if (st != SIPG_OK && st != SIPG_NOT_CONVERGED && st != SIPG_BREAKDOWN) check(st, "solve");
    Matrix3Vec::unpack(x, u_ans, v_ans, w_ans);
    return st == SIPG_OK;
  }
  const sipg_solve_info& last_info() const { return info_; }

 private:
  void drop() {
    if (s_) sipg_solver_destroy(s_);
    s_ = nullptr;
  }
  int kind() const {
    switch (pre_) {
      case NONE: return SIPG_SOLVER_CG;
      case JACOBI: return SIPG_SOLVER_JACOBI;
      case BLOCK_JACOBI: return SIPG_SOLVER_BLOCK_JACOBI;
      default: return SIPG_SOLVER_INV_MASS;
    }
  }
  void ensure() {
    if (s_ && seen_ != matrix_->version()) {
      check(sipg_solver_setup(s_), "setup");
      seen_ = matrix_->version();
    }
    if (s_) return;
    sipg_solver_opts o;
    check(sipg_solver_default_opts(kind(), &o), "options");
    o.rel_tol = rtol_;
    o.abs_tol = atol_;
    o.max_iter = max_iter_;
    o.nullspace = nullspace_ ? 1 : 0;
    o.inv_mass_factor = inv_mass_factor_;
    check(sipg_solver_create(matrix_->handle(), kind(), &o, &s_), "solver");
    seen_ = matrix_->version();
  }
  Matrix3Vec* matrix_ = nullptr;
  sipg_solver* s_ = nullptr;
  Dat u_bc_{}, v_bc_{}, w_bc_{};
  bool nullspace_ = false;
  double rtol_ = 1e-8, atol_ = 1e-9, inv_mass_factor_ = 1.0;
  int max_iter_ = 5000;
  Preconditioners pre_ = FACTOR_INV_MASS;
  sipg_solve_info info_{};
  unsigned seen_ = 0;
};

// ---- initial guess from the pressure history (add_to_pr_history /
// initial_guess_extrapolation of the reference; history size as its
// EXTRAPOLATE_HISTORY_SIZE, here a constructor argument)
class PressureHistory {
 public:
  explicit PressureHistory(size_t max_size = 3) : max_(max_size) {}
  void add(double t, Dat pr) {
    hist_.emplace_back(t, std::vector<double>(pr.data, pr.data + pr.size()));
    while (hist_.size() > max_) hist_.erase(hist_.begin());
  }
  // pr <- extrapolation to time t (unchanged while the history is empty)
  void initial_guess_extrapolation(Dat pr, double t) const {
    if (hist_.empty()) return;
    std::vector<double> times;
    std::vector<const double*> ptr;
    for (auto& h : hist_) {
      times.push_back(h.first);
      ptr.push_back(h.second.data());
    }
    check(sipg_extrapolate_initial_guess_host((int)hist_.size(), times.data(), ptr.data(), t, pr.size(), pr.data),
          "initial_guess_extrapolation");
  }
  size_t size() const { return hist_.size(); }

 private:
  size_t max_;
  std::vector<std::pair<double, std::vector<double>>> hist_;
};

// Element-local velocity projection of the pressure step: the body of
// INSSolverBase3D::project_velocity / INSSolverBase2D::project_velocity with
// div_div = 1 (src/solvers/3d/ins_solver_base.cpp:1052-1124; 2D
// src/solvers/2d/ins_solver_base.cpp:894-955): velTT = the per-element CG
// projection of velT - dt * grad p with the penalty factor the reference uses
// (dt in 3D, dt * 1e3 in 2D). The reference's velocity and gradient components
// are separate op_dats; they are passed here as dim Dats each. project()
// returns the number of converged cells (the reference's num_converge; the
// 2D solver aborts when it is not num_cells, src/solvers/2d/ins_solver_base.cpp:946-949)
// and, if asked, the mean iteration count (num_iter / num_cells).
class VelocityProjection {
 public:
  VelocityProjection(DGMesh* mesh, int order) : mesh_(mesh), order_(order) {}
  int project(double dt, const Dat* dpd, const Dat* velT, Dat* velTT, double* mean_iters = nullptr) {
    const int dim = mesh_->dim();
    const size_t n = velT[0].size();
    in_dp_.resize(dim * n);
    in_v_.resize(dim * n);
    out_.resize(dim * n);
    for (int c = 0; c < dim; ++c) {
      std::copy(dpd[c].data, dpd[c].data + n, in_dp_.begin() + c * n);
      std::copy(velT[c].data, velT[c].data + n, in_v_.begin() + c * n);
    }
    double st[3] = {0, 0, 0};
    const double factor = dim == 3 ? dt : dt * 1e3;
    check(sipg_project_velocity_host(mesh_->handle(), order_, dt, factor, in_dp_.data(), in_v_.data(),
                                     out_.data(), st),
          "project_velocity");
    for (int c = 0; c < dim; ++c) std::copy(out_.begin() + c * n, out_.begin() + (c + 1) * n, velTT[c].data);
    if (mean_iters) *mean_iters = st[0] > 0 ? st[2] / st[0] : 0.0;
    return (int)st[1];
  }
  // Right-hand side of the pressure solve (INSSolver3D::pressure,
  // src/solvers/3d/ins_solver.cpp:313-322): rhs = J M (-div_c(velT) / dt +
  // LIFT (b0 dPdN + b1 dPdN_old)), dPdN_old updated in place; dPdN / dPdN_old
  // are the cells x (dim + 1) * Nfp face dats (data == nullptr: zero, not written).
  void pressure_rhs(double dt, double b0, double b1, const Dat* velT, Dat dPdN, Dat dPdN_old, Dat rhs) {
    const int dim = mesh_->dim();
    const size_t n = velT[0].size();
    in_v_.resize(dim * n);
    for (int c = 0; c < dim; ++c) std::copy(velT[c].data, velT[c].data + n, in_v_.begin() + c * n);
    check(sipg_pressure_rhs_host(mesh_->handle(), order_, dt, b0, b1, in_v_.data(), dPdN.data, dPdN_old.data,
                                 rhs.data),
          "pressure_rhs");
  }
  // The pressure step from the pressure itself: grad_with_central_flux(pr),
  // update_pressure_gradient (/ rho; rho.data == nullptr for the single-phase
  // solver) and project_velocity (src/solvers/3d/mp_ins_solver.cpp:653-659,
  // ins_solver.cpp:361-363) in one call.
  int project_from_pressure(double dt, Dat pr, Dat rho, const Dat* velT, Dat* velTT, double* mean_iters = nullptr) {
    const int dim = mesh_->dim();
    const size_t n = velT[0].size();
    in_v_.resize(dim * n);
    out_.resize(dim * n);
    for (int c = 0; c < dim; ++c) std::copy(velT[c].data, velT[c].data + n, in_v_.begin() + c * n);
    double st[3] = {0, 0, 0};
    const double factor = dim == 3 ? dt : dt * 1e3;
    check(sipg_pressure_projection_host(mesh_->handle(), order_, dt, factor, pr.data, rho.data, in_v_.data(),
                                        out_.data(), st),
          "pressure_projection");
    for (int c = 0; c < dim; ++c) std::copy(out_.begin() + c * n, out_.begin() + (c + 1) * n, velTT[c].data);
    if (mean_iters) *mean_iters = st[0] > 0 ? st[2] / st[0] : 0.0;
    return (int)st[1];
  }

 private:
  DGMesh* mesh_;
  int order_;
  std::vector<double> in_dp_, in_v_, out_;
};

}  // namespace ins_solver_b200
