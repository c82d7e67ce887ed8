// Reference simplex element (triangle / tetrahedron) for nodal DG of order 1..4.
//
// Replaces the constant tables that INS-Solver takes from the unvendored
// OP2-DG-Toolkit (`dg_Dr_kernel`, `dg_Ds_kernel`, `dg_Dt_kernel`,
// `dg_Mass_kernel`, `dg_MM_F{0..3}_kernel`, `FMASK`, and the EMAT/LIFT
// operators used through `op2_gemv`; see src/kernels/fvmf_3d_op1_diag.h:2-5,
// src/kernels/fvmf_3d_op2_diag.h:4-10, src/kernels/fvmf_3d_calc_tau_faces.h:6,
// src/solvers/3d/slip_matrix/factor_viscous_matrix.cpp:109-117,243-276).
//
// Nodes follow the published warp-and-blend construction of Hesthaven and
// Warburton (Nodal Discontinuous Galerkin Methods, 2008, sec. 6.1 and 10.2).
// Operators are built from a tensor-Legendre polynomial basis spanning P_p and
// integrated with collapsed (Duffy) Gauss-Legendre rules that are exact for the
// polynomial degrees involved, so the matrices do not depend on the basis.
//
// All matrices are row-major: A[i * ncols + j].
#pragma once
#include <vector>
#include <cstdint>

namespace sipg {

constexpr int kMaxOrder = 4;

struct RefElement {
  int dim = 0;      // 2 or 3
  int order = 0;    // polynomial order p
  int Np = 0;       // nodes per element
  int Nfp = 0;      // nodes per face
  int Nfaces = 0;   // 3 (triangle) or 4 (tetrahedron)
  int Nverts = 0;   // 3 or 4
  int Nperm = 0;    // face orientation count: 2 (edges) or 6 (triangles)
  double ref_volume = 0.0;   // 2 (triangle) or 4/3 (tetrahedron)

  std::vector<double> r, s, t;                // node coordinates (t empty in 2D)
  std::vector<double> V;                      // Np x Np generalized Vandermonde
  std::vector<double> Dr, Ds, Dt;             // Np x Np differentiation matrices
  std::vector<double> M, Minv;                // Np x Np mass matrix and inverse
  std::vector<int> fmask;                     // Nfaces x Nfp volume node of each face node
  std::vector<double> MF;                     // Nfaces x (Nfp x Nfp) face mass (face node ordering)
  std::vector<double> MMF;                    // Nfaces x (Np x Np) face mass embedded in volume
  std::vector<double> EMAT;                   // Np x (Nfaces*Nfp): face-to-volume mass ("lift" without M^-1)
  std::vector<double> LIFT;                   // Np x (Nfaces*Nfp): Minv * EMAT
  // perm_pos[sigma * Nfp + j]: position k on the neighbour's face that touches
  // face node j of this face when the neighbour's face vertices are this face's
  // vertices permuted by sigma (see face_vertex_perm).
  std::vector<int> perm_pos;
  // face_verts[f * 3 + a]: local vertex a (0..dim-1) of face f.
  std::vector<int> face_verts;
};

// Build the reference element for dim in {2,3} and order in 1..4.
RefElement build_ref_element(int dim, int order);

// Interpolation from order q nodes to order p nodes (Np(p) x Np(q), row-major):
// evaluates the order-q Lagrange basis at the order-p nodes (prolongation P_{q->p}).
std::vector<double> interp_matrix(int dim, int q, int p);

// The 6 (3D) / 2 (2D) permutations of face vertices. sigma maps
// position a on this face to position sigma[a] on the neighbour's face.
const int* face_vertex_perm(int dim, int sigma);

// Collapsed Gauss-Legendre rule with n points per direction on the reference
// simplex (weights sum to its volume; exact for degree 2n - 3 in 3D, 2n - 2 in
// 2D; dim 1: the Gauss-Legendre rule on [-1, 1], exact for 2n - 1). Nodes a, b, c
// ascending, a outermost: r = (1+a)(1-b)(1-c)/4 - 1, s = (1+b)(1-c)/2 - 1, t = c
// (2D: r = (1+a)(1-b)/2 - 1, s = b).
void collapsed_rule(int dim, int n, std::vector<double>& qr, std::vector<double>& qs, std::vector<double>& qt,
                    std::vector<double>& qw);
// Reference coordinates of the face-parameter point (a, b) on face f (the
// parameter domain is the reference triangle in 3D, [-1, 1] in 2D).
void face_param_point(int dim, int f, double a, double b, double* r, double* s, double* t);
// Nodal basis (and its reference derivatives, 3 x n x Np, d/dr d/ds d/dt) at n points.
void lagrange_at_points(const RefElement& e, const std::vector<double>& r, const std::vector<double>& s,
                        const std::vector<double>& t, std::vector<double>& phi, std::vector<double>* dphi);

inline int np_of(int dim, int p) {
  return dim == 2 ? (p + 1) * (p + 2) / 2 : (p + 1) * (p + 2) * (p + 3) / 6;
}
inline int nfp_of(int dim, int p) { return dim == 2 ? p + 1 : (p + 1) * (p + 2) / 2; }

}  // namespace sipg
