// Fused matrix-free SIPG apply for nodal DG on simplices (CUDA cores, FP64/FP32).
//
// One launch computes y = A x for the variable-coefficient SIPG operator of
// FactorViscousMatrix3D::mult (src/solvers/3d/slip_matrix/factor_viscous_matrix.cpp:96-310)
// and its 2D twin, including the constant-coefficient Poisson, the Helmholtz
// (mass term) and the 3-component slip-coupled viscous operator. The reference
// runs ~45 separate OP2 loops per 3-component apply with every intermediate
// in HBM; here each CTA keeps a batch of elements in shared memory and goes
// from x to y in one pass:
//   P0  stage x (own and face neighbours), factor, geometry, penalty
//   P1  own gradient q_d = f * G^T (Dr x, Ds x, Dt x) at every node, and the
//       neighbour's normal flux n.q+ at the matched face nodes (recomputed
//       from the neighbour's x: no second pass, no face buffers in HBM)
//   P2  face fluxes: Fu = sJ (tau [x]/2 - n.{q}), Fq_d = -n_d sJ f [x]/2
//       (fvmf_3d_mult_flux.h), Dirichlet / Neumann / slip boundary traces
//       (vmf_3d_mult_avg_jump.h)
//   P3  q~_r = J sum_d G[r][d] q_d   (mass and geometric transform commute)
//   P4  W_r = M q~_r + EMAT (sum_d G[r][d] Fq_d)
//   P5  y = EMAT Fu + sum_r D_r^T W_r + J M (mm * x)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sipg {

__host__ __device__ constexpr int c_np(int dim, int p) {
  return dim == 2 ? (p + 1) * (p + 2) / 2 : (p + 1) * (p + 2) * (p + 3) / 6;
}
__host__ __device__ constexpr int c_nfp(int dim, int p) { return dim == 2 ? p + 1 : (p + 1) * (p + 2) / 2; }

template <int DIM, int P>
struct Cfg {
  static constexpr int NP = c_np(DIM, P);
  static constexpr int NFP = c_nfp(DIM, P);
  static constexpr int NF = DIM + 1;
  static constexpr int NFNFP = NF * NFP;
  static constexpr int LD = NP | 1;        // odd row stride: conflict-free column walks
  static constexpr int LDE = NFNFP | 1;
  static constexpr int NG = DIM == 3 ? 10 : 5;
  static constexpr int NPERM = DIM == 3 ? 6 : 2;
  // constant blob (T): Dr, Ds, [Dt], M (NP x LD each), EMAT (NP x LDE)
  static constexpr int OFF_D = 0;
  static constexpr int OFF_M = DIM * NP * LD;
  static constexpr int OFF_E = OFF_M + NP * LD;
  static constexpr int CONST_T = OFF_E + NP * LDE;
  // int8 tables: fmask (NF x NFP), perm_pos (NPERM x NFP)
  static constexpr int ITAB = NF * NFP + NPERM * NFP;
};

#ifdef __CUDACC__
// Outward unit normal n and surface Jacobian sJ of face f of an affine simplex
// from its geometric factors g (3D rx ry rz sx sy sz tx ty tz J, faces t = -1,
// s = -1, r + s + t = -1, r = -1; 2D rx ry sx sy J, faces s = -1, r + s = 0, r = -1).
template <int DIM>
__device__ __forceinline__ void simplex_face_normal(const double* g, int f, double n[3], double* sJ) {
  n[2] = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double* gr = g;        // d r / d x
    const double* gs = g + DIM;  // d s / d x
    double v;
    if (DIM == 3) {
      const double* gt = g + 6;
      v = f == 0 ? -gt[d] : f == 1 ? -gs[d] : f == 2 ? (gr[d] + gs[d]) + gt[d] : -gr[d];
    } else {
      v = f == 0 ? -gs[d] : f == 1 ? gr[d] + gs[d] : -gr[d];
    }
    n[d] = v;
  }
  const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  n[0] /= len;
  n[1] /= len;
  n[2] /= len;
  *sJ = len * g[DIM == 3 ? 9 : 4];
}
#endif

// Boundary condition types (problem_specific_3d.h: 0 Dirichlet, 1 Neumann; slip 2).
enum : int { BC_DIRICHLET = 0, BC_NEUMANN = 1, BC_SLIP = 2 };

// mm modes
enum : int { MM_NONE = 0, MM_SCALAR = 1, MM_NODAL = 2 };

template <typename T>
struct ApplyArgs {
  const T* consts;        // Cfg::CONST_T values
  const int8_t* itab;     // Cfg::ITAB values
  const T* geof;          // K x NG
  const int* nbr;         // K x NF: neighbour, or -(bface+1)
  const uint32_t* fcode;  // K: byte f = neighbour face | orientation << 2
  const T* tau;           // K x NF
  const T* factor;        // K x NP or null (constant 1)
  const T* mm;            // K x NP (MM_NODAL)
  T mm_scalar;
  int mm_mode;
  const uint8_t* bct;     // ncomp x Kb boundary types
  int Kb;
  int K;
  int ncomp;              // 1, or DIM for the slip-coupled vector operator
  const T* x;             // ncomp x K x NP
  T* y;
  int pin_elem, pin_node; // pinned DOF (row/column replaced by pin_scale * I), -1: none
  T pin_scale;
  int eb;                 // elements per CTA batch
  T alpha, beta;          // y = alpha * A x + beta * c (beta == 0: c is not read)
  const T* c;             // ncomp x K x NP; y unless the caller gives another vector
  const T* tcg;           // tensor-core path: tile-major element and face geometry (launch_tc_geom)
  int tcgen05 = 0;        // tensor-core path, FP32: tcgen05 kernels where the order has them (else mma.sync)
};

// Host-side launchers (sipg_apply.cu).
template <typename T>
cudaError_t launch_apply(int dim, int order, const ApplyArgs<T>& a, int num_sms, cudaStream_t s);
size_t apply_smem_bytes(int dim, int order, int ncomp, int eb, bool fp64);
int apply_pick_eb(int dim, int order, int ncomp, bool fp64);
// Vector operator (ncomp = dim): y_c += alpha x the component-coupling slip-face
// terms, over the elements that own boundary faces (after per-component scalar
// applies, which give slip faces no face terms).
template <typename T>
cudaError_t launch_slip(int dim, int order, const ApplyArgs<T>& a, const int* belems, int n_belem, cudaStream_t s);

// tau per element face (fvmf_3d_calc_tau_faces.h / fvmf_3d_calc_tau_bfaces.h).
template <typename T>
cudaError_t launch_tau(int dim, int order, const int8_t* itab, const T* geof, const int* nbr,
                       const uint32_t* fcode, const T* factor, int K, T* tau, cudaStream_t s);

}  // namespace sipg
