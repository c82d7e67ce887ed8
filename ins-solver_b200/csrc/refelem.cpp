// Reference simplex element construction. See refelem.hpp for what each table
// replaces in the reference and which published method it follows.
#include "refelem.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>

namespace sipg {
namespace {

constexpr double kPi = 3.14159265358979323846;

// Legendre polynomial P_n(x) and its derivative (unnormalised, P_n(1) = 1).
void legendre(int n, double x, double* p, double* dp) {
  double p0 = 1.0, p1 = x, d0 = 0.0, d1 = 1.0;
  if (n == 0) { *p = 1.0; *dp = 0.0; return; }
  for (int k = 2; k <= n; ++k) {
    double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
    double d2 = d0 + (2 * k - 1) * p1;  // P'_k = P'_{k-2} + (2k-1) P_{k-1}
    p0 = p1; p1 = p2; d0 = d1; d1 = d2;
  }
  *p = p1; *dp = d1;
}

// Gauss-Legendre rule with n points on [-1,1] (Newton on P_n).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0); w.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p, dp;
      legendre(n, z, &p, &dp);
      double dz = p / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p, dp;
    legendre(n, z, &p, &dp);
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Legendre-Gauss-Lobatto points (N+1 of them, ascending): -1, roots of P'_N, 1.
std::vector<double> lgl_points(int N) {
  std::vector<double> x(N + 1);
  x[0] = -1.0; x[N] = 1.0;
  for (int i = 1; i < N; ++i) {
    double z = -std::cos(kPi * i / N);
    for (int it = 0; it < 100; ++it) {
      // Newton on q(z) = P'_N(z); q'(z) = (2 z P'_N - N(N+1) P_N) / (1 - z^2).
      double p, dp;
      legendre(N, z, &p, &dp);
      double ddp = (2.0 * z * dp - N * (N + 1) * p) / (1.0 - z * z);
      double dz = dp / ddp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = z;
  }
  return x;
}

// Warp function of the warp-and-blend construction: the equidistant-node
// interpolant of (LGL - equidistant) displacement, divided by 1 - r^2.
double warp_factor(int N, double rout) {
  std::vector<double> lgl = lgl_points(N);
  double warp = 0.0;
  for (int k = 0; k <= N; ++k) {
    double xk = -1.0 + 2.0 * k / N;
    double lk = 1.0;
    for (int m = 0; m <= N; ++m) {
      if (m == k) continue;
      double xm = -1.0 + 2.0 * m / N;
      lk *= (rout - xm) / (xk - xm);
    }
    warp += lk * (lgl[k] - xk);
  }
  if (std::fabs(rout) < 1.0 - 1e-10) return warp / (1.0 - rout * rout);
  return 0.0;
}

// Warp-and-blend nodes on the equilateral triangle (Hesthaven-Warburton, Nodes2D),
// then mapped to the reference triangle (-1,-1),(1,-1),(-1,1).
void nodes_2d(int N, std::vector<double>& r, std::vector<double>& s) {
  static const double alpopt[15] = {0.0, 0.0, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999, 1.2832,
                                    1.3648, 1.4773, 1.4959, 1.5743, 1.5770, 1.6223, 1.6258};
  const double alpha = N < 16 ? alpopt[N - 1] : 5.0 / 3.0;
  r.clear(); s.clear();
  for (int n = 0; n <= N; ++n) {
    for (int m = 0; m <= N - n; ++m) {
      double L1 = double(n) / N, L3 = double(m) / N, L2 = 1.0 - L1 - L3;
      double x = -L2 + L3, y = (-L2 - L3 + 2.0 * L1) / std::sqrt(3.0);
      double b1 = 4.0 * L2 * L3, b2 = 4.0 * L1 * L3, b3 = 4.0 * L1 * L2;
      double w1 = b1 * warp_factor(N, L3 - L2) * (1.0 + (alpha * L1) * (alpha * L1));
      double w2 = b2 * warp_factor(N, L1 - L3) * (1.0 + (alpha * L2) * (alpha * L2));
      double w3 = b3 * warp_factor(N, L2 - L1) * (1.0 + (alpha * L3) * (alpha * L3));
      x += w1 + std::cos(2 * kPi / 3) * w2 + std::cos(4 * kPi / 3) * w3;
      y += std::sin(2 * kPi / 3) * w2 + std::sin(4 * kPi / 3) * w3;
      double l1 = (std::sqrt(3.0) * y + 1.0) / 3.0;
      double l2 = (-3.0 * x - std::sqrt(3.0) * y + 2.0) / 6.0;
      double l3 = (3.0 * x - std::sqrt(3.0) * y + 2.0) / 6.0;
      r.push_back(-l2 + l3 - l1);
      s.push_back(-l2 - l3 + l1);
    }
  }
}

// Face warp of the 3D construction (Hesthaven-Warburton, WarpShiftFace3D/evalshift).
double eval_warp(int p, const std::vector<double>& xnodes, double xout) {
  std::vector<double> xeq(p + 1);
  for (int i = 0; i <= p; ++i) xeq[i] = -1.0 + 2.0 * (p - i) / p;
  double warp = 0.0;
  for (int i = 0; i <= p; ++i) {
    double d = xnodes[i] - xeq[i];
    for (int j = 1; j < p; ++j)
      if (i != j) d *= (xout - xeq[j]) / (xeq[i] - xeq[j]);
    if (i != 0) d = -d / (xeq[i] - xeq[0]);
    if (i != p) d = d / (xeq[i] - xeq[p]);
    warp += d;
  }
  return warp;
}

void eval_shift(int p, double pval, double L1, double L2, double L3, double* dx, double* dy) {
  std::vector<double> lgl = lgl_points(p);
  std::vector<double> gx(p + 1);
  for (int i = 0; i <= p; ++i) gx[i] = -lgl[i];
  double b1 = L2 * L3, b2 = L1 * L3, b3 = L1 * L2;
  double wf1 = 4.0 * eval_warp(p, gx, L3 - L2);
  double wf2 = 4.0 * eval_warp(p, gx, L1 - L3);
  double wf3 = 4.0 * eval_warp(p, gx, L2 - L1);
  double w1 = b1 * wf1 * (1.0 + (pval * L1) * (pval * L1));
  double w2 = b2 * wf2 * (1.0 + (pval * L2) * (pval * L2));
  double w3 = b3 * wf3 * (1.0 + (pval * L3) * (pval * L3));
  *dx = w1 + std::cos(2 * kPi / 3) * w2 + std::cos(4 * kPi / 3) * w3;
  *dy = std::sin(2 * kPi / 3) * w2 + std::sin(4 * kPi / 3) * w3;
}

void nodes_3d(int p, std::vector<double>& r, std::vector<double>& s, std::vector<double>& t) {
  static const double alphastore[15] = {0.0, 0.0, 0.0, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577,
                                        1.1603, 1.10153, 0.6080, 0.4523, 0.8856, 0.8717, 0.9655};
  const double alpha = p <= 15 ? alphastore[p - 1] : 1.0;
  const double tol = 1e-10;
  const double sq3 = std::sqrt(3.0), sq6 = std::sqrt(6.0);
  const double v1[3] = {-1, -1 / sq3, -1 / sq6}, v2[3] = {1, -1 / sq3, -1 / sq6};
  const double v3[3] = {0, 2 / sq3, -1 / sq6}, v4[3] = {0, 0, 3 / sq6};
  double t1[4][3], t2[4][3];
  for (int d = 0; d < 3; ++d) {
    t1[0][d] = v2[d] - v1[d]; t1[1][d] = v2[d] - v1[d];
    t1[2][d] = v3[d] - v2[d]; t1[3][d] = v3[d] - v1[d];
    t2[0][d] = v3[d] - 0.5 * (v1[d] + v2[d]); t2[1][d] = v4[d] - 0.5 * (v1[d] + v2[d]);
    t2[2][d] = v4[d] - 0.5 * (v2[d] + v3[d]); t2[3][d] = v4[d] - 0.5 * (v1[d] + v3[d]);
  }
  for (int n = 0; n < 4; ++n) {
    double n1 = std::sqrt(t1[n][0] * t1[n][0] + t1[n][1] * t1[n][1] + t1[n][2] * t1[n][2]);
    double n2 = std::sqrt(t2[n][0] * t2[n][0] + t2[n][1] * t2[n][1] + t2[n][2] * t2[n][2]);
    for (int d = 0; d < 3; ++d) { t1[n][d] /= n1; t2[n][d] /= n2; }
  }
  r.clear(); s.clear(); t.clear();
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= p - n; ++m)
      for (int q = 0; q <= p - n - m; ++q) {
        double re = -1.0 + 2.0 * q / p, se = -1.0 + 2.0 * m / p, te = -1.0 + 2.0 * n / p;
        double L1 = (1 + te) / 2, L2 = (1 + se) / 2, L3 = -(1 + re + se + te) / 2, L4 = (1 + re) / 2;
        double X[3], shift[3] = {0, 0, 0};
        for (int d = 0; d < 3; ++d) X[d] = L3 * v1[d] + L4 * v2[d] + L2 * v3[d] + L1 * v4[d];
        for (int face = 0; face < 4; ++face) {
          double La, Lb, Lc, Ld;
          if (face == 0) { La = L1; Lb = L2; Lc = L3; Ld = L4; }
          else if (face == 1) { La = L2; Lb = L1; Lc = L3; Ld = L4; }
          else if (face == 2) { La = L3; Lb = L1; Lc = L4; Ld = L2; }
          else { La = L4; Lb = L1; Lc = L3; Ld = L2; }
          double w1, w2;
          eval_shift(p, alpha, Lb, Lc, Ld, &w1, &w2);
          double blend = Lb * Lc * Ld;
          double denom = (Lb + 0.5 * La) * (Lc + 0.5 * La) * (Ld + 0.5 * La);
          if (denom > tol) blend = (1 + (alpha * La) * (alpha * La)) * blend / denom;
          int nonzero = (Lb > tol) + (Lc > tol) + (Ld > tol);
          if (La < tol && nonzero < 3) {
            for (int d = 0; d < 3; ++d) shift[d] = w1 * t1[face][d] + w2 * t2[face][d];
          } else {
            for (int d = 0; d < 3; ++d) shift[d] += blend * w1 * t1[face][d] + blend * w2 * t2[face][d];
          }
        }
        for (int d = 0; d < 3; ++d) X[d] += shift[d];
        // Map equilateral tetrahedron to the reference one: solve A [r s t]^T = X - c.
        double rhs[3], A[3][3];
        for (int d = 0; d < 3; ++d) {
          rhs[d] = X[d] - 0.5 * (v2[d] + v3[d] + v4[d] - v1[d]);
          A[d][0] = 0.5 * (v2[d] - v1[d]);
          A[d][1] = 0.5 * (v3[d] - v1[d]);
          A[d][2] = 0.5 * (v4[d] - v1[d]);
        }
        double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                     A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                     A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
        double sol[3];
        for (int c = 0; c < 3; ++c) {
          double B[3][3];
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) B[i][j] = (j == c) ? rhs[i] : A[i][j];
          sol[c] = (B[0][0] * (B[1][1] * B[2][2] - B[1][2] * B[2][1]) -
                    B[0][1] * (B[1][0] * B[2][2] - B[1][2] * B[2][0]) +
                    B[0][2] * (B[1][0] * B[2][1] - B[1][1] * B[2][0])) / det;
        }
        r.push_back(sol[0]); s.push_back(sol[1]); t.push_back(sol[2]);
      }
}

// Polynomial basis of P_p: products of Legendre polynomials P_i(r)P_j(s)[P_k(t)]
// with total degree <= p. Evaluates value and gradient of every basis function.

void eval_basis(int dim, int p, double r, double s, double t, double* val, double* dr, double* ds,
                double* dt) {
  double Pr[kMaxOrder + 1], dPr[kMaxOrder + 1], Ps[kMaxOrder + 1], dPs[kMaxOrder + 1];
  double Pt[kMaxOrder + 1], dPt[kMaxOrder + 1];
  for (int i = 0; i <= p; ++i) {
    legendre(i, r, &Pr[i], &dPr[i]);
    legendre(i, s, &Ps[i], &dPs[i]);
    legendre(i, t, &Pt[i], &dPt[i]);
  }
  int n = 0;
  if (dim == 2) {
    for (int i = 0; i <= p; ++i)
      for (int j = 0; i + j <= p; ++j, ++n) {
        val[n] = Pr[i] * Ps[j];
        if (dr) dr[n] = dPr[i] * Ps[j];
        if (ds) ds[n] = Pr[i] * dPs[j];
        if (dt) dt[n] = 0.0;
      }
  } else {
    for (int i = 0; i <= p; ++i)
      for (int j = 0; i + j <= p; ++j)
        for (int k = 0; i + j + k <= p; ++k, ++n) {
          val[n] = Pr[i] * Ps[j] * Pt[k];
          if (dr) dr[n] = dPr[i] * Ps[j] * Pt[k];
          if (ds) ds[n] = Pr[i] * dPs[j] * Pt[k];
          if (dt) dt[n] = Pr[i] * Ps[j] * dPt[k];
        }
  }
}

// Dense inverse by Gauss-Jordan elimination with partial pivoting.
std::vector<double> inverse(const std::vector<double>& A, int n) {
  std::vector<double> a(A), inv(n * n, 0.0);
  for (int i = 0; i < n; ++i) inv[i * n + i] = 1.0;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int i = c + 1; i < n; ++i)
      if (std::fabs(a[i * n + c]) > std::fabs(a[piv * n + c])) piv = i;
    if (std::fabs(a[piv * n + c]) < 1e-300) throw std::runtime_error("singular matrix");
    if (piv != c)
      for (int j = 0; j < n; ++j) {
        std::swap(a[c * n + j], a[piv * n + j]);
        std::swap(inv[c * n + j], inv[piv * n + j]);
      }
    double d = a[c * n + c];
    for (int j = 0; j < n; ++j) { a[c * n + j] /= d; inv[c * n + j] /= d; }
    for (int i = 0; i < n; ++i) {
      if (i == c) continue;
      double f = a[i * n + c];
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) {
        a[i * n + j] -= f * a[c * n + j];
        inv[i * n + j] -= f * inv[c * n + j];
      }
    }
  }
  return inv;
}

// Collapsed Gauss-Legendre quadrature on the reference simplex; n points per
// direction integrates polynomials of degree <= 2n-3 exactly.
void simplex_quadrature(int dim, int n, std::vector<double>& qr, std::vector<double>& qs,
                        std::vector<double>& qt, std::vector<double>& qw) {
  std::vector<double> x, w;
  gauss_legendre(n, x, w);
  qr.clear(); qs.clear(); qt.clear(); qw.clear();
  if (dim == 2) {
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double a = x[i], b = x[j];
        qr.push_back((1 + a) * (1 - b) / 2 - 1);
        qs.push_back(b);
        qt.push_back(0.0);
        qw.push_back(w[i] * w[j] * (1 - b) / 2);
      }
  } else {
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        for (int k = 0; k < n; ++k) {
          double a = x[i], b = x[j], c = x[k];
          qr.push_back((1 + a) * (1 - b) * (1 - c) / 4 - 1);
          qs.push_back((1 + b) * (1 - c) / 2 - 1);
          qt.push_back(c);
          qw.push_back(w[i] * w[j] * w[k] * (1 - b) * (1 - c) * (1 - c) / 8);
        }
  }
}

// Barycentric coordinate of reference vertex v at (r,s,t).
double bary(int dim, int v, double r, double s, double t) {
  if (dim == 2) {
    if (v == 0) return -(r + s) / 2;
    if (v == 1) return (1 + r) / 2;
    return (1 + s) / 2;
  }
  if (v == 0) return -(1 + r + s + t) / 2;
  if (v == 1) return (1 + r) / 2;
  if (v == 2) return (1 + s) / 2;
  return (1 + t) / 2;
}

// Face -> vertices. 3D: face 0: t=-1, face 1: s=-1, face 2: r+s+t=-1, face 3: r=-1.
// 2D: face 0: s=-1, face 1: r+s=0, face 2: r=-1.
const int kFaceVerts3D[4][3] = {{0, 1, 2}, {0, 1, 3}, {1, 2, 3}, {0, 2, 3}};
const int kFaceVerts2D[3][2] = {{0, 1}, {1, 2}, {0, 2}};
const int kPerm3D[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
const int kPerm2D[2][2] = {{0, 1}, {1, 0}};

// Map from the face parameter domain (reference triangle / interval) to the face.
void face_point(int dim, int f, double a, double b, double* r, double* s, double* t) {
  if (dim == 2) {
    *t = 0.0;
    if (f == 0) { *r = a; *s = -1; }
    else if (f == 1) { *r = a; *s = -a; }
    else { *r = -1; *s = a; }
    return;
  }
  if (f == 0) { *r = a; *s = b; *t = -1; }
  else if (f == 1) { *r = a; *s = -1; *t = b; }
  else if (f == 2) { *r = a; *s = b; *t = -1 - a - b; }
  else { *r = -1; *s = a; *t = b; }
}

}  // namespace

const int* face_vertex_perm(int dim, int sigma) {
  return dim == 2 ? kPerm2D[sigma] : kPerm3D[sigma];
}

static void lagrange_at(const RefElement& e, const std::vector<double>& Vinv, double r, double s,
                        double t, double* phi, double* dphir, double* dphis, double* dphit) {
  const int Np = e.Np;
  std::vector<double> psi(Np), pr(Np), ps(Np), pt(Np);
  eval_basis(e.dim, e.order, r, s, t, psi.data(), pr.data(), ps.data(), pt.data());
  for (int i = 0; i < Np; ++i) {
    double v = 0, vr = 0, vs = 0, vt = 0;
    for (int n = 0; n < Np; ++n) {
      double c = Vinv[n * Np + i];
      v += psi[n] * c; vr += pr[n] * c; vs += ps[n] * c; vt += pt[n] * c;
    }
    phi[i] = v;
    if (dphir) { dphir[i] = vr; dphis[i] = vs; dphit[i] = vt; }
  }
}

void collapsed_rule(int dim, int n, std::vector<double>& qr, std::vector<double>& qs, std::vector<double>& qt,
                    std::vector<double>& qw) {
  // Gauss-Legendre nodes in ascending order, the first collapsed direction outermost
  std::vector<double> x, w;
  gauss_legendre(n, x, w);
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return x[a] < x[b]; });
  std::vector<double> xs(n), ws(n);
  for (int i = 0; i < n; ++i) { xs[i] = x[ord[i]]; ws[i] = w[ord[i]]; }
  qr.clear(); qs.clear(); qt.clear(); qw.clear();
  if (dim == 1) {
    qr = xs;
    qw = ws;
    qs.assign(n, 0.0);
    qt.assign(n, 0.0);
    return;
  }
  if (dim == 2) {
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        const double a = xs[i], b = xs[j];
        qr.push_back((1 + a) * (1 - b) / 2 - 1);
        qs.push_back(b);
        qt.push_back(0.0);
        qw.push_back(ws[i] * ws[j] * (1 - b) / 2);
      }
    return;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      for (int k = 0; k < n; ++k) {
        const double a = xs[i], b = xs[j], c = xs[k];
        qr.push_back((1 + a) * (1 - b) * (1 - c) / 4 - 1);
        qs.push_back((1 + b) * (1 - c) / 2 - 1);
        qt.push_back(c);
        qw.push_back(ws[i] * ws[j] * ws[k] * (1 - b) * (1 - c) * (1 - c) / 8);
      }
}

void face_param_point(int dim, int f, double a, double b, double* r, double* s, double* t) {
  face_point(dim, f, a, b, r, s, t);
}

void lagrange_at_points(const RefElement& e, const std::vector<double>& r, const std::vector<double>& s,
                        const std::vector<double>& t, std::vector<double>& phi, std::vector<double>* dphi) {
  const int Np = e.Np;
  const size_t n = r.size();
  const std::vector<double> Vinv = inverse(e.V, Np);
  phi.assign(n * Np, 0.0);
  if (dphi) dphi->assign(3 * n * Np, 0.0);
  std::vector<double> dr(Np), ds(Np), dt(Np);
  for (size_t q = 0; q < n; ++q) {
    lagrange_at(e, Vinv, r[q], s[q], t.empty() ? 0.0 : t[q], &phi[q * Np], dr.data(), ds.data(), dt.data());
    if (dphi)
      for (int i = 0; i < Np; ++i) {
        (*dphi)[(0 * n + q) * Np + i] = dr[i];
        (*dphi)[(1 * n + q) * Np + i] = ds[i];
        (*dphi)[(2 * n + q) * Np + i] = e.dim == 3 ? dt[i] : 0.0;
      }
  }
}

RefElement build_ref_element(int dim, int order) {
  if ((dim != 2 && dim != 3) || order < 1 || order > kMaxOrder)
    throw std::runtime_error("unsupported element: dim=" + std::to_string(dim) +
                             " order=" + std::to_string(order));
  RefElement e;
  e.dim = dim;
  e.order = order;
  e.Np = np_of(dim, order);
  e.Nfp = nfp_of(dim, order);
  e.Nfaces = dim + 1;
  e.Nverts = dim + 1;
  e.Nperm = dim == 2 ? 2 : 6;
  e.ref_volume = dim == 2 ? 2.0 : 4.0 / 3.0;
  const int Np = e.Np, Nfp = e.Nfp, Nf = e.Nfaces;

  if (dim == 2) {
    nodes_2d(order, e.r, e.s);
    e.t.assign(Np, 0.0);
  } else {
    nodes_3d(order, e.r, e.s, e.t);
  }
  // Snap coordinates that sit on a face to the exact face value.
  for (int i = 0; i < Np; ++i) {
    for (int v = 0; v < e.Nverts; ++v) {
      double b = bary(dim, v, e.r[i], e.s[i], e.t[i]);
      if (std::fabs(b) < 1e-12) {
        if (v == 1) e.r[i] = -1.0;
        else if (v == 2) e.s[i] = -1.0;
        else if (v == 3) e.t[i] = -1.0;
      }
    }
    if (std::fabs(bary(dim, 0, e.r[i], e.s[i], e.t[i])) < 1e-12) {
      if (dim == 2) e.s[i] = -e.r[i];
      else e.t[i] = -1.0 - e.r[i] - e.s[i];
    }
  }

  // Vandermonde and derivative matrices.
  e.V.assign(Np * Np, 0.0);
  std::vector<double> Vr(Np * Np), Vs(Np * Np), Vt(Np * Np);
  for (int m = 0; m < Np; ++m)
    eval_basis(dim, order, e.r[m], e.s[m], e.t[m], &e.V[m * Np], &Vr[m * Np], &Vs[m * Np],
               &Vt[m * Np]);
  std::vector<double> Vinv = inverse(e.V, Np);
  auto matmul = [&](const std::vector<double>& A, const std::vector<double>& B) {
    std::vector<double> C(Np * Np, 0.0);
    for (int i = 0; i < Np; ++i)
      for (int k = 0; k < Np; ++k) {
        double a = A[i * Np + k];
        for (int j = 0; j < Np; ++j) C[i * Np + j] += a * B[k * Np + j];
      }
    return C;
  };
  e.Dr = matmul(Vr, Vinv);
  e.Ds = matmul(Vs, Vinv);
  e.Dt = dim == 3 ? matmul(Vt, Vinv) : std::vector<double>(Np * Np, 0.0);

  // Mass matrix by exact quadrature.
  {
    std::vector<double> qr, qs, qt, qw;
    simplex_quadrature(dim, order + 3, qr, qs, qt, qw);
    e.M.assign(Np * Np, 0.0);
    std::vector<double> phi(Np);
    for (size_t q = 0; q < qw.size(); ++q) {
      lagrange_at(e, Vinv, qr[q], qs[q], qt[q], phi.data(), nullptr, nullptr, nullptr);
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j) e.M[i * Np + j] += qw[q] * phi[i] * phi[j];
    }
    e.Minv = inverse(e.M, Np);
  }

  // Face node masks, ordered canonically by face-barycentric coordinates so
  // every face lists its nodes in the same pattern (needed for perm tables).
  e.face_verts.assign(Nf * 3, -1);
  for (int f = 0; f < Nf; ++f)
    for (int a = 0; a < dim; ++a)
      e.face_verts[f * 3 + a] = dim == 2 ? kFaceVerts2D[f][a] : kFaceVerts3D[f][a];
  auto opposite_vertex = [&](int f) {
    for (int v = 0; v < e.Nverts; ++v) {
      bool on = false;
      for (int a = 0; a < dim; ++a) on |= e.face_verts[f * 3 + a] == v;
      if (!on) return v;
    }
    return -1;
  };
  std::vector<std::vector<std::vector<double>>> fbary(Nf);
  e.fmask.assign(Nf * Nfp, -1);
  for (int f = 0; f < Nf; ++f) {
    int ov = opposite_vertex(f);
    std::vector<std::pair<std::vector<double>, int>> items;
    for (int i = 0; i < Np; ++i) {
      if (std::fabs(bary(dim, ov, e.r[i], e.s[i], e.t[i])) > 1e-10) continue;
      std::vector<double> b(dim);
      for (int a = 0; a < dim; ++a) b[a] = bary(dim, e.face_verts[f * 3 + a], e.r[i], e.s[i], e.t[i]);
      items.push_back({b, i});
    }
    if ((int)items.size() != Nfp) throw std::runtime_error("face node count mismatch");
    std::sort(items.begin(), items.end(), [&](const auto& x, const auto& y) {
      for (int a = 0; a < dim; ++a) {
        if (std::fabs(x.first[a] - y.first[a]) > 1e-9) return x.first[a] < y.first[a];
      }
      return false;
    });
    for (int j = 0; j < Nfp; ++j) {
      e.fmask[f * Nfp + j] = items[j].second;
      fbary[f].push_back(items[j].first);
    }
  }
  // All faces must carry the same face node pattern.
  for (int f = 1; f < Nf; ++f)
    for (int j = 0; j < Nfp; ++j)
      for (int a = 0; a < dim; ++a)
        if (std::fabs(fbary[f][j][a] - fbary[0][j][a]) > 1e-9)
          throw std::runtime_error("face node sets differ between faces");

  // Orientation tables: neighbour face vertex sigma[a] coincides with our vertex a.
  e.perm_pos.assign(e.Nperm * Nfp, -1);
  for (int sg = 0; sg < e.Nperm; ++sg) {
    const int* sigma = face_vertex_perm(dim, sg);
    for (int j = 0; j < Nfp; ++j) {
      std::vector<double> target(dim);
      for (int a = 0; a < dim; ++a) target[sigma[a]] = fbary[0][j][a];
      for (int k = 0; k < Nfp; ++k) {
        bool same = true;
        for (int a = 0; a < dim; ++a) same &= std::fabs(fbary[0][k][a] - target[a]) < 1e-9;
        if (same) { e.perm_pos[sg * Nfp + j] = k; break; }
      }
      if (e.perm_pos[sg * Nfp + j] < 0) throw std::runtime_error("face nodes not symmetric");
    }
  }

  // Face mass matrices over the face parameter domain (area 2 in 3D, length 2 in 2D).
  {
    std::vector<double> x, w;
    gauss_legendre(order + 3, x, w);
    std::vector<double> pa, pb, pw;
    if (dim == 2) {
      for (size_t i = 0; i < x.size(); ++i) { pa.push_back(x[i]); pb.push_back(0); pw.push_back(w[i]); }
    } else {
      for (size_t i = 0; i < x.size(); ++i)
        for (size_t j = 0; j < x.size(); ++j) {
          pa.push_back((1 + x[i]) * (1 - x[j]) / 2 - 1);
          pb.push_back(x[j]);
          pw.push_back(w[i] * w[j] * (1 - x[j]) / 2);
        }
    }
    e.MMF.assign(Nf * Np * Np, 0.0);
    std::vector<double> phi(Np);
    for (int f = 0; f < Nf; ++f)
      for (size_t q = 0; q < pw.size(); ++q) {
        double r, s, t;
        face_point(dim, f, pa[q], pb[q], &r, &s, &t);
        lagrange_at(e, Vinv, r, s, t, phi.data(), nullptr, nullptr, nullptr);
        for (int i = 0; i < Np; ++i)
          for (int j = 0; j < Np; ++j) e.MMF[(f * Np + i) * Np + j] += pw[q] * phi[i] * phi[j];
      }
    e.MF.assign(Nf * Nfp * Nfp, 0.0);
    e.EMAT.assign(Np * Nf * Nfp, 0.0);
    for (int f = 0; f < Nf; ++f) {
      for (int a = 0; a < Nfp; ++a)
        for (int b = 0; b < Nfp; ++b)
          e.MF[(f * Nfp + a) * Nfp + b] = e.MMF[(f * Np + e.fmask[f * Nfp + a]) * Np + e.fmask[f * Nfp + b]];
      for (int i = 0; i < Np; ++i)
        for (int b = 0; b < Nfp; ++b)
          e.EMAT[i * (Nf * Nfp) + f * Nfp + b] = e.MMF[(f * Np + i) * Np + e.fmask[f * Nfp + b]];
    }
    e.LIFT.assign(Np * Nf * Nfp, 0.0);
    for (int i = 0; i < Np; ++i)
      for (int k = 0; k < Np; ++k)
        for (int c = 0; c < Nf * Nfp; ++c) e.LIFT[i * Nf * Nfp + c] += e.Minv[i * Np + k] * e.EMAT[k * Nf * Nfp + c];
  }
  return e;
}

std::vector<double> interp_matrix(int dim, int q, int p) {
  RefElement eq = build_ref_element(dim, q);
  RefElement ep = build_ref_element(dim, p);
  std::vector<double> Vinv = inverse(eq.V, eq.Np);
  std::vector<double> P(ep.Np * eq.Np);
  std::vector<double> phi(eq.Np);
  for (int m = 0; m < ep.Np; ++m) {
    lagrange_at(eq, Vinv, ep.r[m], ep.s[m], ep.t[m], phi.data(), nullptr, nullptr, nullptr);
    for (int n = 0; n < eq.Np; ++n) P[m * eq.Np + n] = phi[n];
  }
  return P;
}

}  // namespace sipg
