// Smoothed-aggregation hierarchy for the p=0 level. See amg.hpp.
#include "amg.hpp"

#include "refelem.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>

namespace sipg {

Csr p0_operator(int K, int Nf, const double* sJ, const double* tau, const int* nbr,
                const std::vector<uint8_t>& bc_dirichlet) {
  Csr A;
  A.rows = A.cols = K;
  A.ptr.assign(K + 1, 0);
  for (int e = 0; e < K; ++e) {
    double d = 0.0;
    std::vector<std::pair<int, double>> off;
    for (int f = 0; f < Nf; ++f) {
      size_t i = (size_t)e * Nf + f;
      double w = sJ[i] * tau[i];
      int nb = nbr[i];
      if (nb >= 0) {
        d += w;
        off.push_back({nb, -w});
      } else if (bc_dirichlet[-nb - 1]) {
        d += 2.0 * w;
      }
    }
    off.push_back({e, d});
    std::sort(off.begin(), off.end());
    for (auto& pr : off) {
      A.idx.push_back(pr.first);
      A.val.push_back(pr.second);
    }
    A.ptr[e + 1] = (int)A.idx.size();
  }
  return A;
}

P1Plan p1c_plan(int K, int Nv, int Np, const int* e2v) {
  P1Plan pl;
  pl.Nv = Nv;
  std::vector<std::vector<int>> cols(Nv);
  for (int e = 0; e < K; ++e)
    for (int i = 0; i < Np; ++i)
      for (int j = 0; j < Np; ++j) cols[e2v[(size_t)e * Np + i]].push_back(e2v[(size_t)e * Np + j]);
  pl.ptr.assign(Nv + 1, 0);
  for (int v = 0; v < Nv; ++v) {
    std::sort(cols[v].begin(), cols[v].end());
    cols[v].erase(std::unique(cols[v].begin(), cols[v].end()), cols[v].end());
    pl.ptr[v + 1] = pl.ptr[v] + (int)cols[v].size();
  }
  pl.idx.resize(pl.ptr[Nv]);
  for (int v = 0; v < Nv; ++v) std::copy(cols[v].begin(), cols[v].end(), pl.idx.begin() + pl.ptr[v]);
  pl.slot.resize((size_t)K * Np * Np);
  for (int e = 0; e < K; ++e)
    for (int i = 0; i < Np; ++i) {
      const int vi = e2v[(size_t)e * Np + i];
      const int* b = pl.idx.data() + pl.ptr[vi];
      const int* en = pl.idx.data() + pl.ptr[vi + 1];
      for (int j = 0; j < Np; ++j)
        pl.slot[((size_t)e * Np + i) * Np + j] = pl.ptr[vi] + (int)(std::lower_bound(b, en, e2v[(size_t)e * Np + j]) - b);
    }
  return pl;
}

void p1c_operator(const RefElement& r, int K, int Nv, const double* geof, const int* e2v,
                  const double* factor1, const double* tau1, const double* sJ, const double* nx,
                  const double* ny, const double* nz, const int* nbr,
                  const std::vector<uint8_t>& bc_dirichlet, int mm_mode, double mm_scalar,
                  const double* mm1, Csr* Aout, Csr* Pout, const P1Plan* plan) {
  const int dim = r.dim, Np = r.Np, Nf = r.Nfaces, Nfp = r.Nfp, ng = dim == 3 ? 10 : 5;
  if (Np != dim + 1) throw std::runtime_error("p1c_operator needs the order-1 element");
  const double* Dm[3] = {r.Dr.data(), r.Ds.data(), r.Dt.data()};
  // assemble into the planned sparsity (element order) or, without a plan, with a
  // per-row map of the vertex graph
  std::vector<std::vector<std::pair<int, double>>> rows(plan ? 0 : Nv);
  std::vector<double> pval(plan ? plan->idx.size() : 0, 0.0);
  std::vector<double> B(Np * Np), Dx(Np * Np), T(Np * Np), Dn(Np * Np);
  for (int e = 0; e < K; ++e) {
    const double* g = geof + (size_t)e * ng;
    const double J = g[dim == 3 ? 9 : 4];
    auto G = [&](int rr, int d) { return g[rr * dim + d]; };
    auto fac = [&](int i) { return factor1 ? factor1[(size_t)e * Np + i] : 1.0; };
    std::fill(B.begin(), B.end(), 0.0);
    for (int d = 0; d < dim; ++d) {
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j) {
          double s = 0.0;
          for (int rr = 0; rr < dim; ++rr) s += G(rr, d) * Dm[rr][i * Np + j];
          Dx[i * Np + j] = s;
        }
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j) {
          double s = 0.0;
          for (int k = 0; k < Np; ++k) s += r.M[i * Np + k] * fac(k) * Dx[k * Np + j];
          T[i * Np + j] = J * s;
        }
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j) {
          double s = 0.0;
          for (int k = 0; k < Np; ++k) s += Dx[k * Np + i] * T[k * Np + j];
          B[i * Np + j] += s;
        }
    }
    for (int f = 0; f < Nf; ++f) {
      size_t fi = (size_t)e * Nf + f;
      int nb = nbr[fi];
      if (nb >= 0 || !bc_dirichlet[-nb - 1]) continue;
      double n[3] = {nx[fi], ny[fi], dim == 3 ? nz[fi] : 0.0};
      double rf[3] = {0, 0, 0};
      for (int rr = 0; rr < dim; ++rr)
        for (int d = 0; d < dim; ++d) rf[rr] += n[d] * G(rr, d);
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j) {
          double s = 0.0;
          for (int rr = 0; rr < dim; ++rr) s += rf[rr] * Dm[rr][i * Np + j];
          Dn[i * Np + j] = s;  // n . grad, unscaled
        }
      const double* mf = r.MMF.data() + (size_t)f * Np * Np;
      const double scale = sJ[fi], gtau = tau1[fi];
      // exact Galerkin entries of the apply's Dirichlet face terms: the
      // consistency term carries the factor at the quadrature node (n.q = f dn u),
      // the symmetric term carries it at the trial node (Fq = -n sJ f [u] / 2)
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j) {
          double s = 0.0;
          for (int k = 0; k < Np; ++k)
            s += mf[i * Np + k] * fac(k) * Dn[k * Np + j] + Dn[k * Np + i] * mf[k * Np + j] * fac(j);
          B[i * Np + j] += scale * (gtau * mf[i * Np + j] - s);
        }
    }
    if (mm_mode != 0)
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j)
          B[i * Np + j] += J * r.M[i * Np + j] * (mm_mode == 1 ? mm_scalar : mm1[(size_t)e * Np + j]);
    const int* v = e2v + (size_t)e * Np;
    if (plan) {
      const int* sl = plan->slot.data() + (size_t)e * Np * Np;
      for (int q = 0; q < Np * Np; ++q) pval[sl[q]] += B[q];
    } else {
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j) rows[v[i]].push_back({v[j], B[i * Np + j]});
    }
    (void)Nfp;
  }
  Csr& A = *Aout;
  A.rows = A.cols = Nv;
  if (plan) {
    A.ptr = plan->ptr;
    A.idx = plan->idx;
    A.val = std::move(pval);
  }
  if (!plan) {
    A.ptr.assign(Nv + 1, 0);
    A.idx.clear();
    A.val.clear();
  }
  for (int i = 0; i < Nv && !plan; ++i) {
    auto& rw = rows[i];
    std::sort(rw.begin(), rw.end());
    for (size_t k = 0; k < rw.size();) {
      int c = rw[k].first;
      double s = 0.0;
      while (k < rw.size() && rw[k].first == c) s += rw[k++].second;
      A.idx.push_back(c);
      A.val.push_back(s);
    }
    A.ptr[i + 1] = (int)A.idx.size();
  }
  // injection of vertex values into the p=1 nodes: row (e, i) has one entry at e2v[e][i]
  Csr& P = *Pout;
  P.rows = K * Np;
  P.cols = Nv;
  P.ptr.resize(P.rows + 1);
  P.idx.resize(P.rows);
  P.val.assign(P.rows, 1.0);
  for (int k = 0; k <= P.rows; ++k) P.ptr[k] = k;
  for (int k = 0; k < P.rows; ++k) P.idx[k] = e2v[k];
}

Csr transpose(const Csr& A) {
  Csr T;
  T.rows = A.cols;
  T.cols = A.rows;
  T.ptr.assign(T.rows + 1, 0);
  for (int j : A.idx) T.ptr[j + 1]++;
  for (int r = 0; r < T.rows; ++r) T.ptr[r + 1] += T.ptr[r];
  T.idx.resize(A.nnz());
  T.val.resize(A.nnz());
  std::vector<int> pos(T.ptr.begin(), T.ptr.end() - 1);
  for (int i = 0; i < A.rows; ++i)
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
      int j = A.idx[k];
      T.idx[pos[j]] = i;
      T.val[pos[j]++] = A.val[k];
    }
  return T;
}

Csr spgemm(const Csr& A, const Csr& B) {
  if (A.cols != B.rows) throw std::runtime_error("spgemm shape mismatch");
  Csr C;
  C.rows = A.rows;
  C.cols = B.cols;
  C.ptr.assign(C.rows + 1, 0);
  std::vector<double> acc(B.cols, 0.0);
  std::vector<int> mark(B.cols, -1), cols;
  for (int i = 0; i < A.rows; ++i) {
    cols.clear();
    for (int ka = A.ptr[i]; ka < A.ptr[i + 1]; ++ka) {
      int k = A.idx[ka];
      double a = A.val[ka];
      for (int kb = B.ptr[k]; kb < B.ptr[k + 1]; ++kb) {
        int j = B.idx[kb];
        if (mark[j] != i) { mark[j] = i; acc[j] = 0.0; cols.push_back(j); }
        acc[j] += a * B.val[kb];
      }
    }
    std::sort(cols.begin(), cols.end());
    for (int j : cols) {
      C.idx.push_back(j);
      C.val.push_back(acc[j]);
    }
    C.ptr[i + 1] = (int)C.idx.size();
  }
  return C;
}

namespace {

// Greedy aggregation over strong connections |a_ij| >= theta sqrt(a_ii a_jj).
std::vector<int> aggregate(const Csr& A, double theta, int* n_agg) {
  const int n = A.rows;
  std::vector<double> diag(n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
      if (A.idx[k] == i) diag[i] = A.val[k];
  auto strong = [&](int i, int k) {
    int j = A.idx[k];
    return j != i && std::fabs(A.val[k]) >= theta * std::sqrt(std::fabs(diag[i] * diag[j]));
  };
  std::vector<int> agg(n, -1);
  int na = 0;
  // pass 1: seeds whose strong neighbours are all free
  for (int i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    bool free_nbhd = true;
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
      if (strong(i, k) && agg[A.idx[k]] >= 0) { free_nbhd = false; break; }
    if (!free_nbhd) continue;
    agg[i] = na;
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
      if (strong(i, k)) agg[A.idx[k]] = na;
    ++na;
  }
  // pass 2: join the strongest aggregated neighbour; else start a new aggregate
  for (int i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    int best = -1;
    double bw = 0.0;
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
      int j = A.idx[k];
      if (j == i || agg[j] < 0) continue;
      double w = std::fabs(A.val[k]);
      if (w > bw) { bw = w; best = agg[j]; }
    }
    agg[i] = best >= 0 ? best : na++;
  }
  *n_agg = na;
  return agg;
}

std::vector<double> dense_inverse(std::vector<double> a, int n) {
  std::vector<double> v((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int i = c + 1; i < n; ++i)
      if (std::fabs(a[(size_t)i * n + c]) > std::fabs(a[(size_t)piv * n + c])) piv = i;
    if (std::fabs(a[(size_t)piv * n + c]) < 1e-300) throw std::runtime_error("singular coarse matrix");
    if (piv != c)
      for (int j = 0; j < n; ++j) {
        std::swap(a[(size_t)c * n + j], a[(size_t)piv * n + j]);
        std::swap(v[(size_t)c * n + j], v[(size_t)piv * n + j]);
      }
    double d = 1.0 / a[(size_t)c * n + c];
    for (int j = 0; j < n; ++j) { a[(size_t)c * n + j] *= d; v[(size_t)c * n + j] *= d; }
    for (int i = 0; i < n; ++i) {
      if (i == c) continue;
      double f = a[(size_t)i * n + c];
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) {
        a[(size_t)i * n + j] -= f * a[(size_t)c * n + j];
        v[(size_t)i * n + j] -= f * v[(size_t)c * n + j];
      }
    }
  }
  return v;
}

}  // namespace

// A level must keep at most this fraction of its rows; the densely inverted
// coarsest level holds at most kMaxDenseCoarse rows.
constexpr double kMinCoarsening = 0.6;
constexpr int kMaxDenseCoarse = 8192;

namespace {
struct HostTimer {
  bool on = std::getenv("SIPG_SETUP_TIMES") != nullptr;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  void mark(const char* what, int level) {
    if (!on) return;
    const auto t1 = std::chrono::steady_clock::now();
    std::fprintf(stderr, "  amg %-20s level %2d %8.2f ms\n", what, level,
                 std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  }
};
}  // namespace

AmgHierarchy build_amg(const Csr& A0, const Csr& Pdg, int coarse_max, double strength, bool singular,
                       bool host_inverse) {
  HostTimer ht;
  AmgHierarchy H;
  H.singular = singular;
  H.Pdg = Pdg;
  H.Rdg = transpose(Pdg);
  H.levels.push_back({A0, {}, {}});
  while (H.levels.back().A.rows > coarse_max && H.levels.size() < 16) {
    const Csr& A = H.levels.back().A;
    // A threshold that leaves most connections weak coarsens little and makes the
    // Galerkin products dense; such a level is aggregated again with a lower threshold.
    int na = 0;
    double theta = strength;
    std::vector<int> agg = aggregate(A, theta, &na);
    for (int retry = 0; retry < 3 && na > kMinCoarsening * A.rows; ++retry) {
      theta *= 0.25;
      agg = aggregate(A, theta, &na);
    }
    if (na > kMinCoarsening * A.rows || na < 1) break;
    ht.mark("aggregate", (int)H.levels.size() - 1);
    // tentative prolongator: piecewise constant on aggregates
    Csr T;
    T.rows = A.rows;
    T.cols = na;
    T.ptr.resize(A.rows + 1);
    for (int i = 0; i < A.rows; ++i) {
      T.ptr[i] = i;
      T.idx.push_back(agg[i]);
      T.val.push_back(1.0);
    }
    T.ptr[A.rows] = A.rows;
    // smoothed prolongator P = (I - omega D^-1 A) T, omega = 4 / (3 rho(D^-1 A)),
    // rho bounded by the Gershgorin estimate max_i sum_j |a_ij| / a_ii.
    double rho = 0.0;
    std::vector<double> dinv(A.rows, 0.0);
    for (int i = 0; i < A.rows; ++i) {
      double d = 0.0, s = 0.0;
      for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) {
        if (A.idx[k] == i) d = A.val[k];
        s += std::fabs(A.val[k]);
      }
      dinv[i] = d != 0.0 ? 1.0 / d : 0.0;
      rho = std::max(rho, s * std::fabs(dinv[i]));
    }
    const double omega = 4.0 / (3.0 * rho);
    Csr S = A;  // S = I - omega D^-1 A
    for (int i = 0; i < S.rows; ++i)
      for (int k = S.ptr[i]; k < S.ptr[i + 1]; ++k) {
        double v = -omega * dinv[i] * S.val[k];
        if (S.idx[k] == i) v += 1.0;
        S.val[k] = v;
      }
    Csr P = spgemm(S, T);
    Csr R = transpose(P);
    ht.mark("prolongator", (int)H.levels.size() - 1);
    Csr Ac = spgemm(R, spgemm(A, P));
    ht.mark("galerkin product", (int)H.levels.size() - 1);
    H.levels.back().P = std::move(P);
    H.levels.back().R = std::move(R);
    H.levels.push_back({std::move(Ac), {}, {}});
  }
  const Csr& C = H.levels.back().A;
  const int n = C.rows;
  if (n > kMaxDenseCoarse)
    throw std::runtime_error("algebraic coarsening stalled: coarsest level too large for a dense inverse");
  std::vector<double> dense((size_t)n * n, 0.0);
  double dmax = 0.0;
  for (int i = 0; i < n; ++i)
    for (int k = C.ptr[i]; k < C.ptr[i + 1]; ++k) {
      dense[(size_t)i * n + C.idx[k]] = C.val[k];
      if (C.idx[k] == i) dmax = std::max(dmax, std::fabs(C.val[k]));
    }
  if (singular)
    for (int i = 0; i < n; ++i) dense[(size_t)i * n + i] += 1e-8 * dmax;
  ht.mark("coarse matrix", -1);
  H.coarse_n = n;
  if (!host_inverse) {
    H.coarse_dense = std::move(dense);
    return H;
  }
  std::vector<double> inv = dense_inverse(std::move(dense), n);
  ht.mark("dense inverse", -1);
  if (singular) {
    // pseudo-inverse on the complement of the constants: Q inv Q with Q = I - 11^T/n,
    // so the coarsest correction neither sees nor produces the nullspace
    std::vector<double> rm(n, 0.0), cm(n, 0.0);
    double all = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double v = inv[(size_t)i * n + j];
        rm[i] += v;
        cm[j] += v;
        all += v;
      }
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        inv[(size_t)i * n + j] += -rm[i] / n - cm[j] / n + all / ((double)n * n);
  }
  H.coarse_inv = std::move(inv);
  H.coarse_n = n;
  return H;
}

}  // namespace sipg
