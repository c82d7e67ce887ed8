// Simplicial DG mesh: connectivity, face orientation codes and affine
// geometric factors.
//
// Stands in for the unvendored DGMesh2D/DGMesh3D of OP2-DG-Toolkit, whose
// per-cell and per-face data the hot-path kernels consume: `geof` (10 values in
// 3D, 5 in 2D; src/kernels/fvmf_3d_grad.h:4-12), `nx_c/ny_c/nz_c/sJ_c`
// (src/solvers/3d/slip_matrix/factor_viscous_matrix.cpp:213-218), `fscale`,
// `faceNum`, `fmaskL/fmaskR`, `face2cells`, `bface2cells`, `bfaceNum`,
// `bnx/bny/bnz/bsJ/bfscale` (factor_viscous_matrix.cpp:47-92,316-366).
#pragma once
#include <cstdint>
#include <vector>

#include "refelem.hpp"

namespace sipg {

// geof layout (our own, stated once): 3D rx ry rz sx sy sz tx ty tz J;
// 2D rx ry sx sy J.
enum Geof3D { RX3 = 0, RY3, RZ3, SX3, SY3, SZ3, TX3, TY3, TZ3, J3, NGEOF3 };
enum Geof2D { RX2 = 0, RY2, SX2, SY2, J2, NGEOF2 };

struct Mesh {
  int dim = 0, order = 0, K = 0, Nv = 0, Nf = 0, Np = 0, Nfp = 0;
  std::vector<double> vx;       // Nv * dim vertex coordinates
  std::vector<int> e2v;         // K * (dim+1)
  std::vector<double> geof;     // K * ngeof
  std::vector<double> nx, ny, nz, sJ, fscale;  // K * Nf, outward, per element face
  std::vector<int> nbr;         // K * Nf: neighbour element, or -(bface+1) on the boundary
  std::vector<uint8_t> nbr_face;  // K * Nf: neighbour's local face (interior only)
  std::vector<uint8_t> nbr_perm;  // K * Nf: orientation code sigma (interior only)
  // Face lists in the reference's form (one entry per interior face, L < R).
  std::vector<int> face2cells;  // F * 2
  std::vector<int> faceNum;     // F * 2
  std::vector<int> fmaskL, fmaskR;  // F * Nfp volume node indices matched node by node
  std::vector<int> bface2cell, bfaceNum;  // Kb
  std::vector<double> bface_centroid;     // Kb * dim
  std::vector<double> x, y, z;  // K * Np physical node coordinates
  int ngeof() const { return dim == 3 ? (int)NGEOF3 : (int)NGEOF2; }
  int nfaces_interior() const { return (int)faceNum.size() / 2; }
  int nbfaces() const { return (int)bfaceNum.size(); }
};

// Build connectivity and geometry for a general simplicial mesh given vertex
// coordinates and element-to-vertex lists. Elements with negative Jacobian are
// reoriented. Throws on non-manifold input.
Mesh build_mesh(const RefElement& ref, int Nv, const double* vx, int K, const int* e2v);

// Synthetic structured meshes: the unit square split into n x n quads, each cut
// into 2 triangles along the (0,0)-(1,1) diagonal; the unit cube split into n^3
// hexes, each cut into 6 tetrahedra sharing the (0,0,0)-(1,1,1) diagonal (Kuhn
// split). Interior vertices are jittered uniformly by +-jitter*h per coordinate
// from `seed`; boundary vertices stay fixed.
void box_mesh(int dim, int n, double jitter, uint64_t seed, std::vector<double>& vx,
              std::vector<int>& e2v);

// Deterministic generator shared by every workload (splitmix64).
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
  double normal();
};

}  // namespace sipg
