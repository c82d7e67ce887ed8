// Cubature tables of the over-integrated operator. See oi.hpp.
#include "oi.hpp"

#include <stdexcept>

namespace sipg {

namespace {

// Reference-simplex vertices (the bary() convention of refelem.cpp: vertex v is
// where barycentric coordinate v equals 1).
void ref_vertex(int dim, int v, double x[3]) {
  x[0] = x[1] = x[2] = -1.0;
  if (dim == 2) x[2] = 0.0;
  if (v >= 1) x[v - 1] = 1.0;
}

// Reference coordinates of sum_a lam[a] v[verts[a]].
void face_coords(int dim, const int* verts, const double* lam, double* r, double* s, double* t) {
  double x[3] = {0.0, 0.0, 0.0};
  for (int a = 0; a < dim; ++a) {
    double v[3];
    ref_vertex(dim, verts[a], v);
    for (int d = 0; d < 3; ++d) x[d] += lam[a] * v[d];
  }
  *r = x[0];
  *s = x[1];
  *t = dim == 3 ? x[2] : 0.0;
}

}  // namespace

OiTables build_oi_tables(int dim, int order) {
  const RefElement e = build_ref_element(dim, order);
  OiTables T;
  T.dim = dim;
  T.order = order;
  T.Np = e.Np;
  T.Nf = e.Nfaces;
  T.nperm = e.Nperm;
  const int Np = e.Np, Nf = e.Nfaces;
  // volume rule: exact to degree 2p + 1
  collapsed_rule(dim, order + 2, T.rq, T.sq, T.tq, T.wq);
  T.nq = (int)T.wq.size();
  lagrange_at_points(e, T.rq, T.sq, T.tq, T.vphi, &T.vdphi);
  // face rule: exact to degree 2p, points by face barycentrics
  std::vector<double> a, b, c;
  collapsed_rule(dim - 1, order + 1, a, b, c, T.ws);
  T.nqs = (int)T.ws.size();
  const int nqs = T.nqs;
  T.lam.assign((size_t)nqs * dim, 0.0);
  for (int q = 0; q < nqs; ++q) {
    if (dim == 3) {
      const double l1 = 0.5 * (1.0 + a[q]), l2 = 0.5 * (1.0 + b[q]);
      T.lam[q * 3 + 0] = 1.0 - l1 - l2;
      T.lam[q * 3 + 1] = l1;
      T.lam[q * 3 + 2] = l2;
    } else {
      T.lam[q * 2 + 0] = 0.5 * (1.0 - a[q]);
      T.lam[q * 2 + 1] = 0.5 * (1.0 + a[q]);
    }
  }
  auto points_on = [&](const int* verts, const std::vector<int>& order_of, std::vector<double>& r,
                       std::vector<double>& s, std::vector<double>& t) {
    // point q: sum_a lam_{order_of[a]}(q) v[verts[a]]
    r.resize(nqs);
    s.resize(nqs);
    t.resize(nqs);
    for (int q = 0; q < nqs; ++q) {
      double l[3] = {0.0, 0.0, 0.0};
      for (int x = 0; x < dim; ++x) l[x] = T.lam[q * dim + order_of[x]];
      face_coords(dim, verts, l, &r[q], &s[q], &t[q]);
    }
  };
  std::vector<int> ident(dim);
  for (int x = 0; x < dim; ++x) ident[x] = x;
  T.fr.resize((size_t)Nf * nqs);
  T.fs.resize((size_t)Nf * nqs);
  T.ft.resize((size_t)Nf * nqs);
  T.fphi.resize((size_t)Nf * nqs * Np);
  T.fdphi.resize((size_t)Nf * 3 * nqs * Np);
  for (int f = 0; f < Nf; ++f) {
    std::vector<double> r, s, t, phi, dphi;
    points_on(&e.face_verts[f * 3], ident, r, s, t);
    lagrange_at_points(e, r, s, t, phi, &dphi);
    for (int q = 0; q < nqs; ++q) {
      T.fr[f * nqs + q] = r[q];
      T.fs[f * nqs + q] = s[q];
      T.ft[f * nqs + q] = t[q];
    }
    std::copy(phi.begin(), phi.end(), T.fphi.begin() + (size_t)f * nqs * Np);
    std::copy(dphi.begin(), dphi.end(), T.fdphi.begin() + (size_t)f * 3 * nqs * Np);
  }
  // cross tables
  const int np = T.nperm;
  T.xphi.resize((size_t)Nf * np * nqs * Np);
  T.xdphi.resize((size_t)Nf * np * 3 * nqs * Np);
  T.yphi.resize((size_t)Nf * np * nqs * Np);
  for (int g = 0; g < Nf; ++g)
    for (int sg = 0; sg < np; ++sg) {
      const int* sigma = face_vertex_perm(dim, sg);
      // the neighbour's coordinates of this element's point q: sum_a lam_a(q) v[fv_g[sigma[a]]]
      std::vector<int> verts(dim);
      for (int x = 0; x < dim; ++x) verts[x] = e.face_verts[g * 3 + sigma[x]];
      std::vector<double> r, s, t, phi, dphi;
      points_on(verts.data(), ident, r, s, t);
      lagrange_at_points(e, r, s, t, phi, &dphi);
      std::copy(phi.begin(), phi.end(), T.xphi.begin() + ((size_t)g * np + sg) * nqs * Np);
      std::copy(dphi.begin(), dphi.end(), T.xdphi.begin() + ((size_t)g * np + sg) * 3 * nqs * Np);
      // this element (face g, orientation sigma) at the neighbour's point q:
      // barycentric a here is the neighbour's sigma[a]
      std::vector<int> ord(dim);
      for (int x = 0; x < dim; ++x) ord[x] = sigma[x];
      points_on(&e.face_verts[g * 3], ord, r, s, t);
      lagrange_at_points(e, r, s, t, phi, nullptr);
      std::copy(phi.begin(), phi.end(), T.yphi.begin() + ((size_t)g * np + sg) * nqs * Np);
    }
  // L2 projection of point values: M^-1 (w_q phi_i(x_q))
  T.proj.assign((size_t)Np * T.nq, 0.0);
  for (int i = 0; i < Np; ++i)
    for (int q = 0; q < T.nq; ++q) {
      double s = 0.0;
      for (int k = 0; k < Np; ++k) s += e.Minv[i * Np + k] * T.wq[q] * T.vphi[(size_t)q * Np + k];
      T.proj[(size_t)i * T.nq + q] = s;
    }
  return T;
}

}  // namespace sipg
