// Mesh connectivity and geometric factors. See mesh.hpp.
#include "mesh.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <stdexcept>
#include <unordered_map>

namespace sipg {

double SplitMix64::normal() {
  // Box-Muller.
  double u1 = uniform(), u2 = uniform();
  if (u1 < 1e-300) u1 = 1e-300;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

void box_mesh(int dim, int n, double jitter, uint64_t seed, std::vector<double>& vx,
              std::vector<int>& e2v) {
  const double h = 1.0 / n;
  SplitMix64 rng(seed);
  vx.clear();
  e2v.clear();
  if (dim == 2) {
    auto vid = [&](int i, int j) { return i + (n + 1) * j; };
    for (int j = 0; j <= n; ++j)
      for (int i = 0; i <= n; ++i) {
        double x = i * h, y = j * h;
        bool interior = i > 0 && i < n && j > 0 && j < n;
        double dx = (2 * rng.uniform() - 1) * jitter * h;
        double dy = (2 * rng.uniform() - 1) * jitter * h;
        if (interior) { x += dx; y += dy; }
        vx.push_back(x); vx.push_back(y);
      }
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        int a = vid(i, j), b = vid(i + 1, j), c = vid(i + 1, j + 1), d = vid(i, j + 1);
        int t0[3] = {a, b, c}, t1[3] = {a, c, d};
        e2v.insert(e2v.end(), t0, t0 + 3);
        e2v.insert(e2v.end(), t1, t1 + 3);
      }
    return;
  }
  auto vid = [&](int i, int j, int k) { return i + (n + 1) * (j + (n + 1) * k); };
  for (int k = 0; k <= n; ++k)
    for (int j = 0; j <= n; ++j)
      for (int i = 0; i <= n; ++i) {
        double x = i * h, y = j * h, z = k * h;
        bool interior = i > 0 && i < n && j > 0 && j < n && k > 0 && k < n;
        double dx = (2 * rng.uniform() - 1) * jitter * h;
        double dy = (2 * rng.uniform() - 1) * jitter * h;
        double dz = (2 * rng.uniform() - 1) * jitter * h;
        if (interior) { x += dx; y += dy; z += dz; }
        vx.push_back(x); vx.push_back(y); vx.push_back(z);
      }
  static const int axes[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        for (int tt = 0; tt < 6; ++tt) {
          int c[3] = {0, 0, 0};
          int v[4];
          v[0] = vid(i, j, k);
          c[axes[tt][0]] = 1;
          v[1] = vid(i + c[0], j + c[1], k + c[2]);
          c[axes[tt][1]] = 1;
          v[2] = vid(i + c[0], j + c[1], k + c[2]);
          v[3] = vid(i + 1, j + 1, k + 1);
          e2v.insert(e2v.end(), v, v + 4);
        }
}

Mesh build_mesh(const RefElement& ref, int Nv, const double* vx_in, int K, const int* e2v_in) {
  Mesh m;
  const int dim = ref.dim;
  const int nv = dim + 1;
  m.dim = dim; m.order = ref.order; m.K = K; m.Nv = Nv;
  m.Nf = ref.Nfaces; m.Np = ref.Np; m.Nfp = ref.Nfp;
  m.vx.assign(vx_in, vx_in + (size_t)Nv * dim);
  m.e2v.assign(e2v_in, e2v_in + (size_t)K * nv);
  const int Nf = m.Nf, Np = m.Np, Nfp = m.Nfp, ng = m.ngeof();

  // Orientation: make every element's Jacobian positive.
  for (int e = 0; e < K; ++e) {
    int* v = &m.e2v[(size_t)e * nv];
    for (int a = 0; a < nv; ++a)
      if (v[a] < 0 || v[a] >= Nv) throw std::runtime_error("vertex index out of range");
    double det;
    if (dim == 2) {
      const double* p0 = &m.vx[v[0] * 2]; const double* p1 = &m.vx[v[1] * 2];
      const double* p2 = &m.vx[v[2] * 2];
      det = (p1[0] - p0[0]) * (p2[1] - p0[1]) - (p1[1] - p0[1]) * (p2[0] - p0[0]);
    } else {
      const double* p0 = &m.vx[v[0] * 3]; double a[3], b[3], c[3];
      for (int d = 0; d < 3; ++d) {
        a[d] = m.vx[v[1] * 3 + d] - p0[d]; b[d] = m.vx[v[2] * 3 + d] - p0[d];
        c[d] = m.vx[v[3] * 3 + d] - p0[d];
      }
      det = a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
            a[2] * (b[0] * c[1] - b[1] * c[0]);
    }
    if (det == 0.0) throw std::runtime_error("degenerate element");
    if (det < 0) std::swap(v[1], v[2]);
  }

  // Geometric factors and outward face normals (affine simplices).
  m.geof.assign((size_t)K * ng, 0.0);
  m.nx.assign((size_t)K * Nf, 0.0); m.ny = m.nx; m.nz = m.nx; m.sJ = m.nx; m.fscale = m.nx;
  m.x.assign((size_t)K * Np, 0.0); m.y = m.x; m.z = m.x;
  for (int e = 0; e < K; ++e) {
    const int* v = &m.e2v[(size_t)e * nv];
    double* g = &m.geof[(size_t)e * ng];
    if (dim == 2) {
      const double* p0 = &m.vx[v[0] * 2]; const double* p1 = &m.vx[v[1] * 2];
      const double* p2 = &m.vx[v[2] * 2];
      double xr = 0.5 * (p1[0] - p0[0]), xs = 0.5 * (p2[0] - p0[0]);
      double yr = 0.5 * (p1[1] - p0[1]), ys = 0.5 * (p2[1] - p0[1]);
      double J = xr * ys - xs * yr;
      g[RX2] = ys / J; g[RY2] = -xs / J; g[SX2] = -yr / J; g[SY2] = xr / J; g[J2] = J;
      double n[3][2] = {{-g[SX2], -g[SY2]}, {g[RX2] + g[SX2], g[RY2] + g[SY2]}, {-g[RX2], -g[RY2]}};
      for (int f = 0; f < 3; ++f) {
        double len = std::sqrt(n[f][0] * n[f][0] + n[f][1] * n[f][1]);
        size_t i = (size_t)e * Nf + f;
        m.nx[i] = n[f][0] / len; m.ny[i] = n[f][1] / len; m.nz[i] = 0.0;
        m.sJ[i] = len * J; m.fscale[i] = m.sJ[i] / J;
      }
      for (int k = 0; k < Np; ++k) {
        double r = ref.r[k], s = ref.s[k];
        double l0 = -(r + s) / 2, l1 = (1 + r) / 2, l2 = (1 + s) / 2;
        m.x[(size_t)e * Np + k] = l0 * p0[0] + l1 * p1[0] + l2 * p2[0];
        m.y[(size_t)e * Np + k] = l0 * p0[1] + l1 * p1[1] + l2 * p2[1];
      }
    } else {
      const double* P[4];
      for (int a = 0; a < 4; ++a) P[a] = &m.vx[v[a] * 3];
      double F[3][3];  // F[d][c] = d x_d / d r_c
      for (int d = 0; d < 3; ++d)
        for (int c = 0; c < 3; ++c) F[d][c] = 0.5 * (P[c + 1][d] - P[0][d]);
      double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                 F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                 F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
      double Gi[3][3];  // Gi[c][d] = d r_c / d x_d = inverse of F
      Gi[0][0] = (F[1][1] * F[2][2] - F[1][2] * F[2][1]) / J;
      Gi[0][1] = (F[0][2] * F[2][1] - F[0][1] * F[2][2]) / J;
      Gi[0][2] = (F[0][1] * F[1][2] - F[0][2] * F[1][1]) / J;
      Gi[1][0] = (F[1][2] * F[2][0] - F[1][0] * F[2][2]) / J;
      Gi[1][1] = (F[0][0] * F[2][2] - F[0][2] * F[2][0]) / J;
      Gi[1][2] = (F[0][2] * F[1][0] - F[0][0] * F[1][2]) / J;
      Gi[2][0] = (F[1][0] * F[2][1] - F[1][1] * F[2][0]) / J;
      Gi[2][1] = (F[0][1] * F[2][0] - F[0][0] * F[2][1]) / J;
      Gi[2][2] = (F[0][0] * F[1][1] - F[0][1] * F[1][0]) / J;
      for (int c = 0; c < 3; ++c)
        for (int d = 0; d < 3; ++d) g[c * 3 + d] = Gi[c][d];
      g[J3] = J;
      double n[4][3];
      for (int d = 0; d < 3; ++d) {
        n[0][d] = -Gi[2][d];
        n[1][d] = -Gi[1][d];
        n[2][d] = Gi[0][d] + Gi[1][d] + Gi[2][d];
        n[3][d] = -Gi[0][d];
      }
      for (int f = 0; f < 4; ++f) {
        double len = std::sqrt(n[f][0] * n[f][0] + n[f][1] * n[f][1] + n[f][2] * n[f][2]);
        size_t i = (size_t)e * Nf + f;
        m.nx[i] = n[f][0] / len; m.ny[i] = n[f][1] / len; m.nz[i] = n[f][2] / len;
        m.sJ[i] = len * J; m.fscale[i] = m.sJ[i] / J;
      }
      for (int k = 0; k < Np; ++k) {
        double r = ref.r[k], s = ref.s[k], t = ref.t[k];
        double l[4] = {-(1 + r + s + t) / 2, (1 + r) / 2, (1 + s) / 2, (1 + t) / 2};
        double X[3] = {0, 0, 0};
        for (int a = 0; a < 4; ++a)
          for (int d = 0; d < 3; ++d) X[d] += l[a] * P[a][d];
        m.x[(size_t)e * Np + k] = X[0]; m.y[(size_t)e * Np + k] = X[1]; m.z[(size_t)e * Np + k] = X[2];
      }
    }
  }

  // Face matching by sorted vertex ids.
  struct KeyHash {
    size_t operator()(const std::array<int, 3>& k) const {
      uint64_t h = 1469598103934665603ull;
      for (int x : k) { h ^= (uint64_t)(uint32_t)x; h *= 1099511628211ull; }
      return (size_t)h;
    }
  };
  std::unordered_map<std::array<int, 3>, int, KeyHash> open;  // key -> e*Nf+f
  open.reserve((size_t)K * Nf);
  m.nbr.assign((size_t)K * Nf, 0);
  m.nbr_face.assign((size_t)K * Nf, 0);
  m.nbr_perm.assign((size_t)K * Nf, 0);
  std::vector<char> matched((size_t)K * Nf, 0);
  auto face_global = [&](int e, int f, int a) {
    return m.e2v[(size_t)e * nv + ref.face_verts[f * 3 + a]];
  };
  for (int e = 0; e < K; ++e)
    for (int f = 0; f < Nf; ++f) {
      std::array<int, 3> key = {-1, -1, -1};
      for (int a = 0; a < dim; ++a) key[a] = face_global(e, f, a);
      std::sort(key.begin(), key.begin() + dim);
      auto it = open.find(key);
      if (it == open.end()) {
        open.emplace(key, e * Nf + f);
        continue;
      }
      int other = it->second;
      open.erase(it);
      int eL = other / Nf, fL = other % Nf, eR = e, fR = f;
      // sigma for each side: position a on own face -> position on neighbour face.
      auto sigma_of = [&](int e0, int f0, int e1, int f1) {
        int sg[3] = {0, 0, 0};
        for (int a = 0; a < dim; ++a) {
          int g0 = face_global(e0, f0, a);
          int b = 0;
          for (; b < dim; ++b)
            if (face_global(e1, f1, b) == g0) break;
          sg[a] = b;
        }
        for (int s = 0; s < ref.Nperm; ++s) {
          const int* p = face_vertex_perm(dim, s);
          bool same = true;
          for (int a = 0; a < dim; ++a) same &= p[a] == sg[a];
          if (same) return s;
        }
        throw std::runtime_error("face orientation not found");
      };
      int sLR = sigma_of(eL, fL, eR, fR), sRL = sigma_of(eR, fR, eL, fL);
      size_t iL = (size_t)eL * Nf + fL, iR = (size_t)eR * Nf + fR;
      m.nbr[iL] = eR; m.nbr_face[iL] = (uint8_t)fR; m.nbr_perm[iL] = (uint8_t)sLR;
      m.nbr[iR] = eL; m.nbr_face[iR] = (uint8_t)fL; m.nbr_perm[iR] = (uint8_t)sRL;
      matched[iL] = matched[iR] = 1;
      m.face2cells.push_back(eL); m.face2cells.push_back(eR);
      m.faceNum.push_back(fL); m.faceNum.push_back(fR);
      for (int j = 0; j < Nfp; ++j) {
        m.fmaskL.push_back(ref.fmask[fL * Nfp + j]);
        m.fmaskR.push_back(ref.fmask[fR * Nfp + ref.perm_pos[sLR * Nfp + j]]);
      }
    }
  // Remaining open faces are boundary faces, numbered in element order.
  for (int e = 0; e < K; ++e)
    for (int f = 0; f < Nf; ++f) {
      size_t i = (size_t)e * Nf + f;
      if (matched[i]) continue;
      int b = (int)m.bfaceNum.size();
      m.nbr[i] = -(b + 1);
      m.bface2cell.push_back(e);
      m.bfaceNum.push_back(f);
      for (int d = 0; d < dim; ++d) {
        double c = 0;
        for (int a = 0; a < dim; ++a) c += m.vx[face_global(e, f, a) * dim + d];
        m.bface_centroid.push_back(c / dim);
      }
    }
  return m;
}

}  // namespace sipg
