// Over-integrated variable-coefficient SIPG operator: the factor given at
// cubature points instead of the nodes.
//
// Replaces FactorPoissonMatrixFreeDiagOI3D (OP2-DG-Toolkit, unvendored), which
// the reference selects with `[pressure-solve] over_int`
// (src/solvers/3d/mp_ins_solver.cpp:81-88) and feeds in
// MPINSSolver3D::update_pressure_matrices_oi (:524-544): 1/rho at the volume
// cubature points (mat_free_set_factor_oi, after mp_ins_3d_pr_fact_oi_0), at the
// surface cubature points of every face (mat_free_set_factor_surf_oi, after
// mp_ins_3d_pr_fact_oi_1), and its L2 projection onto the nodes
// (CUB3D_PROJ, set_factor) for the coarse levels.
//
// The bilinear form is the SIPG form of the nodal operator with every integral
// taken by cubature and the factor read at the cubature points:
//   volume     sum_q w_q J f_q grad(phi_i) . grad(phi_j)
//   each face  -1/2 int {f grad u} . n [v] - 1/2 int f- (n . grad v) [u] + tau/2 int [u][v]
//              (interior; Dirichlet faces: jump 2u, average from inside, weights 1)
// where each face integral that carries one side's factor is taken with that
// side's surface points (so no factor is needed at the other side's points and
// the operator is symmetric), and tau = 2(p+1)(p+2) max over both sides' points
// of fscale f (boundary faces: own side). The cubature rules (the toolkit's
// DG_CUB_3D_NP / DG_CUB_SURF_3D_NP rules are not in the reference tree) are
// collapsed Gauss-Legendre rules exact to degree 2p + 1 in the volume (p + 2
// points per direction) and 2p on the faces (p + 1 per direction), so with a
// constant factor the operator equals the nodal one.
#pragma once
#include <vector>

#include "refelem.hpp"

namespace sipg {

struct OiTables {
  int dim = 0, order = 0, Np = 0, Nf = 0, nq = 0, nqs = 0, nperm = 0;
  std::vector<double> rq, sq, tq, wq;  // volume points (reference coordinates) and weights
  std::vector<double> vphi;            // nq x Np basis at the volume points
  std::vector<double> vdphi;           // 3 x nq x Np reference derivatives there
  // face points by their barycentric coordinates in the face's vertex order
  // (the same on every face), so a point of face f is sum_a lam_a(s) v[face_verts[f][a]]
  std::vector<double> lam;             // nqs x dim
  std::vector<double> ws;              // nqs face-parameter weights (sum: 2, the mass matrices' face measure)
  std::vector<double> fr, fs, ft;      // Nf x nqs reference coordinates of each face's points
  std::vector<double> fphi;            // Nf x nqs x Np basis at a face's points
  std::vector<double> fdphi;           // Nf x 3 x nqs x Np reference derivatives there
  // the neighbour's basis and derivatives at this element's points of a face, for
  // the neighbour's face g and orientation sigma (this face's vertex a is the
  // neighbour's face vertex sigma[a]): [g][sigma] x nqs x Np and [g][sigma] x 3 x nqs x Np
  std::vector<double> xphi, xdphi;
  // this element's basis at the neighbour's points, for this element's face f and
  // orientation sigma: [f][sigma] x nqs x Np
  std::vector<double> yphi;
  std::vector<double> proj;            // Np x nq: M^-1 (w_q phi_i(x_q)), the L2 projection of point values
};

OiTables build_oi_tables(int dim, int order);

}  // namespace sipg
