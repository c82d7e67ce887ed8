// Device set-up of the algebraic coarse levels.
//
// The reference keeps its PETSc GAMG interpolation across time steps
// (`[petsc-amg] reuse-interpolation = 1`, examples/3d/oscillating_droplet/config.ini:59):
// only the operator values change with the density factor, so every later set-up
// recomputes the Galerkin products with the stored prolongators. Here the
// continuous P1 operator is assembled on the device from the element data, the
// Galerkin products run as precomputed term lists (one thread per output entry,
// terms summed in the order of the host sparse product, so the result is
// deterministic), and the coarsest level is inverted on the device.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "amg.hpp"

namespace sipg {

// Order-1 reference tables: derivative matrices, mass matrix and per-face
// masses embedded in the volume (row-major Np x Np, Np = dim + 1 <= 4).
struct P1Tables {
  int dim = 3;
  double D[3][16];
  double M[16];
  double MF[4][16];
};
P1Tables p1_tables(const RefElement& r);

// Per-element blocks of the continuous P1 operator (blk: K x Np x Np, row-major),
// the same terms as p1c_operator: volume J sum_d Dx_d^T M F Dx_d, Dirichlet face
// blocks sJ (tau MF - MF F Dn - Dn^T MF F) and the J M mm mass term.
// geof: K x ng; factor1, mm1: K x Np or null; tau1: K x Nf; nbr: K x Nf;
// bct: boundary-face types (Dirichlet = 0).
void p1c_blocks_device(const P1Tables& t, int K, const double* geof, const double* factor1, const double* tau1,
                       const int* nbr, const unsigned char* bct, int mm_mode, double mm_scalar, const double* mm1,
                       double* blk, cudaStream_t s);

// Sums of fixed terms: out[i] = sum_{t = ptr[i]}^{ptr[i+1]-1} in[idx[t]] * coef[t]
// (coef null: 1). out32, when given, receives the same values in FP32.
void term_sum_device(int n, const int* ptr, const int* idx, const double* coef, const double* in, double* out,
                     float* out32, cudaStream_t s);

// Inverse diagonal of a CSR matrix (0 where a row has no diagonal entry).
void csr_dinv_device(int n, const int* ptr, const int* idx, const double* v, double* d64, float* d32,
                     cudaStream_t s);

// Dense row-major copy of an n x n CSR matrix; `shift` adds 1e-8 max_i |a_ii| to
// the diagonal (the pure-Neumann coarsest level, as build_amg does on the host).
void csr_to_dense_device(int n, const int* ptr, const int* idx, const double* v, double* dense, bool shift,
                         cudaStream_t s);

// Term lists of C = A B with one operand fixed: every entry of C becomes a list of
// (position in the varying operand's values, value of the fixed operand's entry),
// in the order the host sparse product accumulates them. `Cs` receives the
// structure of C (values zero).
struct TermPlan {
  std::vector<int> ptr, idx;
  std::vector<double> coef;
};
TermPlan spgemm_plan(const Csr& A, const Csr& B, bool a_varies, Csr* Cs);

// The P1 assembly as term lists: entry k of the operator sums the element-block
// entries e * Np * Np + q with slot (e, q) = k, in element order.
TermPlan p1c_gather_plan(const P1Plan& plan, int K, int Np);

}  // namespace sipg
