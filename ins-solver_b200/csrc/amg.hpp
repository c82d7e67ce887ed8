// Algebraic multigrid for the lowest-order level of the p-multigrid hierarchy.
//
// The reference solves its p=1 coarse problem with PETSc's algebraic multigrid
// (`coarse_solver = petsc`, `[petsc-amg]`, examples/3d/oscillating_droplet/config.ini:24-31,52-64;
// PETScPMultigrid is unvendored). Here the p=1 DG level is smoothed like the
// others and its residual is restricted to piecewise constants (p=0). The
// Galerkin projection of the SIPG operator onto element-wise constants keeps only
// the penalty term (gradients of constants vanish and D_r 1 = 0), so the p=0
// operator is a weighted graph Laplacian on the element dual graph:
//   A0[e][k] = -sJ_f tau_f          for the interior face f shared by e and k,
//   A0[e][e] = sum_f sJ_f tau_f  +  2 sJ_f tau_f over Dirichlet faces of e.
// Below p=0 a smoothed-aggregation hierarchy (greedy strength-based aggregation,
// Jacobi-smoothed prolongator, Galerkin coarse operators) is built on the host and
// applied on the device; the coarsest level is solved with a dense inverse.
#pragma once
#include <cstdint>
#include <vector>

namespace sipg {

struct Csr {
  int rows = 0, cols = 0;
  std::vector<int> ptr, idx;
  std::vector<double> val;
  size_t nnz() const { return val.size(); }
};

struct AmgLevel {
  Csr A;       // level operator
  Csr P, R;    // prolongation to the finer level (fine x coarse) and R = P^T
};

struct AmgHierarchy {
  Csr Pdg, Rdg;                   // DG p=1 unknowns x level-0 unknowns, and its transpose
  std::vector<AmgLevel> levels;   // levels[0].A is the coarse-space operator; P/R of level l map l <-> l+1
  std::vector<double> coarse_inv; // dense inverse of the coarsest operator (n x n, row-major)
  std::vector<double> coarse_dense;  // without the host inverse: the coarsest operator, dense (shifted when singular)
  bool singular = false;
  int coarse_n = 0;
};

// p=0 Galerkin operator of the SIPG penalty term. sJ, tau: K x Nf per element
// face; nbr: K x Nf (neighbour or -(bface+1)); bc_dirichlet[b] != 0 marks
// Dirichlet boundary faces.
Csr p0_operator(int K, int Nf, const double* sJ, const double* tau, const int* nbr,
                const std::vector<uint8_t>& bc_dirichlet);

// Continuous piecewise-linear coarse space. For u, v continuous the SIPG form
// keeps only its volume term and its Dirichlet boundary terms (interior jumps
// vanish), so the Galerkin operator P^T A P is assembled from element volume
// blocks J sum_d Dx_d^T M F Dx_d and Dirichlet face blocks
// sJ (tau MF - MF F Dn - Dn^T MF F) of the p=1 apply (F the nodal factor, Dn the
// normal derivative; the p=1 nodes are the vertices). Pdg maps vertex values to
// the p=1 DG nodes (injection).
// ref1: order-1 reference element; geof K x ngeof; e2v K x (dim+1);
// factor1 K x Np1 (null: 1); tau1, sJ K x Nf; nbr K x Nf; mm: mode/scalar/nodal K x Np1.
struct RefElement;
// Sparsity of the continuous P1 operator of a mesh and, per element entry (e, i, j),
// its position in the CSR values (built once per mesh, reused by every assembly).
struct P1Plan {
  int Nv = 0;
  std::vector<int> ptr, idx, slot;
};
P1Plan p1c_plan(int K, int Nv, int Np, const int* e2v);
void p1c_operator(const RefElement& ref1, int K, int Nv, const double* geof, const int* e2v,
                  const double* factor1, const double* tau1, const double* sJ, const double* nx,
                  const double* ny, const double* nz, const int* nbr,
                  const std::vector<uint8_t>& bc_dirichlet, int mm_mode, double mm_scalar,
                  const double* mm1, Csr* A, Csr* Pdg, const P1Plan* plan = nullptr);

// Smoothed-aggregation hierarchy down to at most `coarse_max` unknowns.
// `singular` adds a tiny diagonal shift before inverting the coarsest level
// (pure Neumann problems, whose constant nullspace the outer solver projects out).
// host_inverse = false leaves the inversion to the caller (coarse_dense holds the
// matrix to invert, with the 1e-8 relative diagonal shift of a singular problem;
// the inverse is then projected onto the complement of the constants).
AmgHierarchy build_amg(const Csr& A0, const Csr& Pdg, int coarse_max, double strength, bool singular,
                       bool host_inverse = true);

Csr transpose(const Csr& A);
Csr spgemm(const Csr& A, const Csr& B);

}  // namespace sipg
