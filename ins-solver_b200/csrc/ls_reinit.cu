// Level-set reinitialisation on the device: the closest-point reinitialisation of
// LevelSetSolver3D::reinitLS (src/solvers/3d/ls_solver.cpp:719-860,
// sampleInterface and the sampling Newton of src/solvers/3d/ls_solver_cpu.cpp:
// 291-316, 318-487, the closest-point Newton of ls_solver.cpp:259-480), in four
// launches and a host pass that keeps the converged samples:
//   cells    the elements whose nodal values change sign (s >= 0 against s < 0);
//   sample   Np points per such element, started at the reference nodes scaled by
//            0.75, moved onto the zero set of the element's polynomial by the
//            simplified Newton x -= s grad s / |grad s|^2 (100 steps, converged when
//            the step^2 < max(1e-18, 1e-4 h^2)) and kept if converged inside the
//            element;
//   nearest  the closest kept sample to every node, by brute force over the samples
//            staged through shared memory, four nodes per thread (the reference
//            queries a KD-tree);
//   newton   from that sample, the Lagrange-multiplier Newton iteration for the
//            closest point of the zero set of the sample element's polynomial (4 x 4
//            pivoted solve, steps clamped to h / 2, a fall-back step when the system
//            is singular, abandoned beyond 1.5 h, 50 steps, converged at step^2 <
//            1e-24); s = +-|x - closest point| (the sample's distance when Newton does
//            not converge), +-ls_cap for elements whose first node is farther than
//            ls_cap + 2 h from every sample; then clamped to +-ls_cap (ls_post_reinit).
// Departures, for a deterministic GPU form: the polynomial of an element is its own
// nodal interpolant (the reference fits a weighted least-squares polynomial over a
// face-neighbour stencil, weights exp(-|x - x_c|^2 / (0.001 h))); samples that do not
// converge are dropped (the reference restarts them from random points drawn from
// std::random_device); no kink detection and no edge-intersection starting points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/sipg_b200.h"
#include "capi_util.hpp"
#include "ins_step.cuh"
#include "runtime.hpp"
#include "vecops.cuh"

namespace sipg {
namespace {

constexpr int kRThreads = 128;

__device__ __forceinline__ double qnan() { return __longlong_as_double(0x7ff8000000000000LL); }

// Monomial coefficients of the nodal interpolant in reference coordinates:
// c = Vm^-1 s with Vm[i][k] = r_i^a s_i^b t_i^c over the exponents a + b + c <= p in
// the nested order of mono_exps.
std::vector<int> mono_exps(int p) {
  std::vector<int> e;
  for (int n = 0; n <= p; ++n)
    for (int a = n; a >= 0; --a)
      for (int b = n - a; b >= 0; --b) {
        e.push_back(a);
        e.push_back(b);
        e.push_back(n - a - b);
      }
  return e;
}

struct ReinitTables {
  DevBuf vminv;  // Np x Np
  DevBuf exps;   // Np x 3 ints
  DevBuf rst;    // 3 x Np reference node coordinates
};

const ReinitTables& reinit_tables(int order) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::unique_ptr<ReinitTables>> cache;
  int dev = 0;
  SIPG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  auto& slot = cache[{dev, order}];
  if (slot) return *slot;
  const RefElement& r = dev_ref(3, order).ref;
  const int Np = r.Np;
  const std::vector<int> ex = mono_exps(order);
  std::vector<double> A((size_t)Np * Np), I((size_t)Np * Np, 0.0);
  for (int i = 0; i < Np; ++i) {
    for (int k = 0; k < Np; ++k)
      A[(size_t)i * Np + k] = std::pow(r.r[i], ex[3 * k]) * std::pow(r.s[i], ex[3 * k + 1]) * std::pow(r.t[i], ex[3 * k + 2]);
    I[(size_t)i * Np + i] = 1.0;
  }
  // Gauss-Jordan with partial pivoting
  for (int c = 0; c < Np; ++c) {
    int p = c;
    for (int i = c + 1; i < Np; ++i)
      if (std::fabs(A[(size_t)i * Np + c]) > std::fabs(A[(size_t)p * Np + c])) p = i;
    for (int j = 0; j < Np; ++j) {
      std::swap(A[(size_t)c * Np + j], A[(size_t)p * Np + j]);
      std::swap(I[(size_t)c * Np + j], I[(size_t)p * Np + j]);
    }
    const double d = 1.0 / A[(size_t)c * Np + c];
    for (int j = 0; j < Np; ++j) {
      A[(size_t)c * Np + j] *= d;
      I[(size_t)c * Np + j] *= d;
    }
    for (int i = 0; i < Np; ++i) {
      if (i == c) continue;
      const double f = A[(size_t)i * Np + c];
      if (f == 0.0) continue;
      for (int j = 0; j < Np; ++j) {
        A[(size_t)i * Np + j] -= f * A[(size_t)c * Np + j];
        I[(size_t)i * Np + j] -= f * I[(size_t)c * Np + j];
      }
    }
  }
  auto t = std::make_unique<ReinitTables>();
  t->vminv = DevBuf(I.size() * sizeof(double));
  t->vminv.upload(I.data(), I.size() * sizeof(double));
  t->exps = DevBuf(ex.size() * sizeof(int));
  t->exps.upload(ex.data(), ex.size() * sizeof(int));
  std::vector<double> rst;
  rst.insert(rst.end(), r.r.begin(), r.r.end());
  rst.insert(rst.end(), r.s.begin(), r.s.end());
  rst.insert(rst.end(), r.t.begin(), r.t.end());
  t->rst = DevBuf(rst.size() * sizeof(double));
  t->rst.upload(rst.data(), rst.size() * sizeof(double));
  slot = std::move(t);
  return *slot;
}

struct ReinitArgs {
  const double* vminv;
  const int* exps;
  const double* rst;
  const double* geof;  // K x 10: dr/dx (row r, column d), J
  const double* xyz;   // 3 x K x Np node coordinates
  const double* s;     // level set before the reinitialisation
  double* s_out;
  int* cells;          // interface elements
  int* ncells;
  double* samples;     // ncells x Np x 3 (NaN: dropped)
  const double* csamples;  // the kept samples, in order (x, y, z)
  const int* cflat;        // their flat sample indices
  int* nearest;        // K x Np: flat sample index, or -1
  double h, ls_cap, tol;
  int K, Np, order;
};

// The element's polynomial in reference coordinates: value, gradient, Hessian
// (rr, ss, tt, rs, rt, st) at r.
template <int P>
__device__ void poly_eval(const double* c, const int* ex, int Np, const double r[3], double* val, double gr[3],
                          double hs[6]) {
  double pw[3][P + 1];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    pw[d][0] = 1.0;
#pragma unroll
    for (int k = 1; k <= P; ++k) pw[d][k] = pw[d][k - 1] * r[d];
  }
  double v = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0, h0 = 0.0, h1 = 0.0, h2 = 0.0, h3 = 0.0, h4 = 0.0, h5 = 0.0;
  for (int k = 0; k < Np; ++k) {
    const int a = ex[3 * k], b = ex[3 * k + 1], e = ex[3 * k + 2];
    const double ck = c[k];
    const double A = pw[0][a], B = pw[1][b], E = pw[2][e];
    const double dA = a > 0 ? a * pw[0][a - 1] : 0.0, dB = b > 0 ? b * pw[1][b - 1] : 0.0,
                 dE = e > 0 ? e * pw[2][e - 1] : 0.0;
    const double ddA = a > 1 ? a * (a - 1) * pw[0][a - 2] : 0.0, ddB = b > 1 ? b * (b - 1) * pw[1][b - 2] : 0.0,
                 ddE = e > 1 ? e * (e - 1) * pw[2][e - 2] : 0.0;
    v += ck * A * B * E;
    g0 += ck * dA * B * E;
    g1 += ck * A * dB * E;
    g2 += ck * A * B * dE;
    h0 += ck * ddA * B * E;
    h1 += ck * A * ddB * E;
    h2 += ck * A * B * ddE;
    h3 += ck * dA * dB * E;
    h4 += ck * dA * B * dE;
    h5 += ck * A * dB * dE;
  }
  *val = v;
  gr[0] = g0;
  gr[1] = g1;
  gr[2] = g2;
  hs[0] = h0;
  hs[1] = h1;
  hs[2] = h2;
  hs[3] = h3;
  hs[4] = h4;
  hs[5] = h5;
}

// s, its physical gradient and Hessian (xx, yy, zz, xy, xz, yz) at the physical point x
// of element e whose monomial coefficients are c.
template <int P>
__device__ void phys_eval(const ReinitArgs& a, int e, const double* c, const double x[3], double* val,
                          double gx[3], double hx[6]) {
  const double* g = a.geof + (size_t)e * 10;
  const size_t n = (size_t)a.K * a.Np, b = (size_t)e * a.Np;
  const double x0[3] = {a.xyz[b], a.xyz[n + b], a.xyz[2 * n + b]};
  const double r0[3] = {a.rst[0], a.rst[a.Np], a.rst[2 * a.Np]};
  double r[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r[i] = r0[i];
#pragma unroll
    for (int d = 0; d < 3; ++d) r[i] += g[i * 3 + d] * (x[d] - x0[d]);
  }
  double gr[3], hr[6];
  poly_eval<P>(c, a.exps, a.Np, r, val, gr, hr);
  const double H[3][3] = {{hr[0], hr[3], hr[4]}, {hr[3], hr[1], hr[5]}, {hr[4], hr[5], hr[2]}};
#pragma unroll
  for (int d = 0; d < 3; ++d) gx[d] = gr[0] * g[d] + gr[1] * g[3 + d] + gr[2] * g[6 + d];
  const int pd[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int d = pd[q][0], f = pd[q][1];
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) acc += g[i * 3 + d] * H[i][j] * g[j * 3 + f];
    hx[q] = acc;
  }
}

__device__ bool in_element(const ReinitArgs& a, int e, const double x[3]) {
  const double* g = a.geof + (size_t)e * 10;
  const size_t n = (size_t)a.K * a.Np, b = (size_t)e * a.Np;
  const double x0[3] = {a.xyz[b], a.xyz[n + b], a.xyz[2 * n + b]};
  double r[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    r[i] = a.rst[i * a.Np];
#pragma unroll
    for (int d = 0; d < 3; ++d) r[i] += g[i * 3 + d] * (x[d] - x0[d]);
  }
  const double eps = 1e-10;
  return r[0] >= -1.0 - eps && r[1] >= -1.0 - eps && r[2] >= -1.0 - eps && r[0] + r[1] + r[2] <= -1.0 + eps;
}

__device__ void cell_coeffs(const ReinitArgs& a, int e, double* c) {
  const double* se = a.s + (size_t)e * a.Np;
  for (int k = 0; k < a.Np; ++k) {
    double v = 0.0;
    for (int j = 0; j < a.Np; ++j) v += a.vminv[(size_t)k * a.Np + j] * se[j];
    c[k] = v;
  }
}

__global__ void k_reinit_cells(ReinitArgs a) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < a.K; e += gridDim.x * blockDim.x) {
    const double* se = a.s + (size_t)e * a.Np;
    const bool pos = se[0] >= 0.0;
    bool cut = false;
    for (int j = 1; j < a.Np; ++j) cut = cut || ((se[j] >= 0.0) != pos);
    if (cut) a.cells[atomicAdd(a.ncells, 1)] = e;
  }
}

template <int P>
__global__ void __launch_bounds__(kRThreads) k_reinit_sample(ReinitArgs a, int ncells) {
  constexpr int NP = (P + 1) * (P + 2) * (P + 3) / 6;
  const int total = ncells * NP;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int ci = t / NP, j = t - ci * NP;
    const int e = a.cells[ci];
    double c[NP];
    cell_coeffs(a, e, c);
    // start: the reference node scaled by 0.75, mapped to the element
    const double* g = a.geof + (size_t)e * 10;
    const size_t n = (size_t)a.K * NP, b = (size_t)e * NP;
    const double x0[3] = {a.xyz[b], a.xyz[n + b], a.xyz[2 * n + b]};
    const double rs[3] = {0.75 * a.rst[j], 0.75 * a.rst[NP + j], 0.75 * a.rst[2 * NP + j]};
    // x = x0 + G^-1 (r - r0): solve the 3 x 3 system of the affine map
    double dr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) dr[i] = rs[i] - a.rst[i * NP];
    const double m00 = g[0], m01 = g[1], m02 = g[2], m10 = g[3], m11 = g[4], m12 = g[5], m20 = g[6], m21 = g[7],
                 m22 = g[8];
    const double det = m00 * (m11 * m22 - m12 * m21) - m01 * (m10 * m22 - m12 * m20) + m02 * (m10 * m21 - m11 * m20);
    double x[3];
    x[0] = x0[0] + ((m11 * m22 - m12 * m21) * dr[0] - (m01 * m22 - m02 * m21) * dr[1] + (m01 * m12 - m02 * m11) * dr[2]) / det;
    x[1] = x0[1] + (-(m10 * m22 - m12 * m20) * dr[0] + (m00 * m22 - m02 * m20) * dr[1] - (m00 * m12 - m02 * m10) * dr[2]) / det;
    x[2] = x0[2] + ((m10 * m21 - m11 * m20) * dr[0] - (m00 * m21 - m01 * m20) * dr[1] + (m00 * m11 - m01 * m10) * dr[2]) / det;
    bool conv = false;
    for (int it = 0; it < 100; ++it) {
      double v, gx[3], hx[6];
      phys_eval<P>(a, e, c, x, &v, gx, hx);
      const double sq = gx[0] * gx[0] + gx[1] * gx[1] + gx[2] * gx[2];
      if (sq > 1e-14) {
#pragma unroll
        for (int d = 0; d < 3; ++d) gx[d] *= v / sq;
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) x[d] -= gx[d];
      if (gx[0] * gx[0] + gx[1] * gx[1] + gx[2] * gx[2] < a.tol) {
        conv = true;
        break;
      }
    }
    const bool keep = conv && in_element(a, e, x);
#pragma unroll
    for (int d = 0; d < 3; ++d) a.samples[(size_t)t * 3 + d] = keep ? x[d] : qnan();
  }
}

// closest kept sample to every node: brute force, the samples staged through shared
// memory and compared against NPT nodes per thread; ties go to the first sample
constexpr int kNpt = 4;
__global__ void __launch_bounds__(kRThreads) k_reinit_nearest(ReinitArgs a, int nkept) {
  __shared__ double sx[kRThreads], sy[kRThreads], sz[kRThreads];
  const size_t n = (size_t)a.K * a.Np;
  const size_t node0 = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) * kNpt;
  double px[kNpt], py[kNpt], pz[kNpt], best[kNpt];
  int bi[kNpt];
#pragma unroll
  for (int q = 0; q < kNpt; ++q) {
    const size_t node = node0 + q;
    const bool act = node < n;
    px[q] = act ? a.xyz[node] : 0.0;
    py[q] = act ? a.xyz[n + node] : 0.0;
    pz[q] = act ? a.xyz[2 * n + node] : 0.0;
    best[q] = INFINITY;
    bi[q] = -1;
  }
  for (int s0 = 0; s0 < nkept; s0 += kRThreads) {
    __syncthreads();
    const int sidx = s0 + threadIdx.x;
    sx[threadIdx.x] = sidx < nkept ? a.csamples[(size_t)sidx * 3] : 0.0;
    sy[threadIdx.x] = sidx < nkept ? a.csamples[(size_t)sidx * 3 + 1] : 0.0;
    sz[threadIdx.x] = sidx < nkept ? a.csamples[(size_t)sidx * 3 + 2] : 0.0;
    __syncthreads();
    const int m = min(kRThreads, nkept - s0);
    for (int k = 0; k < m; ++k) {
      const double qx = sx[k], qy = sy[k], qz = sz[k];
#pragma unroll
      for (int q = 0; q < kNpt; ++q) {
        const double dx = qx - px[q], dy = qy - py[q], dz = qz - pz[q];
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < best[q]) {
          best[q] = d2;
          bi[q] = s0 + k;
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kNpt; ++q)
    if (node0 + q < n) a.nearest[node0 + q] = bi[q] >= 0 ? a.cflat[bi[q]] : -1;
}

// 4 x 4 solve with partial pivoting; false when a pivot is below 1e4 machine epsilon
__device__ bool solve4(double A[4][4], double b[4]) {
  for (int i = 0; i < 4; ++i) {
    int j = i;
    for (int k = i + 1; k < 4; ++k)
      if (fabs(A[k][i]) > fabs(A[j][i])) j = k;
    if (j != i) {
      for (int k = 0; k < 4; ++k) {
        const double t = A[i][k];
        A[i][k] = A[j][k];
        A[j][k] = t;
      }
      const double t = b[i];
      b[i] = b[j];
      b[j] = t;
    }
    if (fabs(A[i][i]) < 1.0e4 * 2.220446049250313e-16) return false;
    const double f = 1.0 / A[i][i];
    for (int r = i + 1; r < 4; ++r) A[r][i] *= f;
    for (int r = i + 1; r < 4; ++r) {
      for (int k = i + 1; k < 4; ++k) A[r][k] -= A[r][i] * A[i][k];
      b[r] -= A[r][i] * b[i];
    }
  }
  for (int i = 3; i >= 0; --i) {
    double sum = 0.0;
    for (int j = i + 1; j < 4; ++j) sum += A[i][j] * b[j];
    b[i] = (b[i] - sum) / A[i][i];
  }
  return true;
}

template <int P>
__global__ void __launch_bounds__(kRThreads) k_reinit_newton(ReinitArgs a) {
  constexpr int NP = (P + 1) * (P + 2) * (P + 3) / 6;
  const size_t n = (size_t)a.K * NP;
  for (size_t node = blockIdx.x * (size_t)blockDim.x + threadIdx.x; node < n; node += (size_t)gridDim.x * blockDim.x) {
    const size_t first = node / NP * NP;  // the element's first node decides whether it is reinitialised
    const double sv = a.s[node];
    const double sgn = sv < 0.0 ? -1.0 : 1.0;
    const int b0 = a.nearest[first], bi = a.nearest[node];
    double out = sgn * a.ls_cap;
    if (b0 >= 0 && bi >= 0) {
      const double w = a.ls_cap + 2.0 * a.h;
      double d0 = 0.0, d1 = 0.0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double e0 = a.samples[(size_t)b0 * 3 + d] - a.xyz[d * n + first];
        const double e1 = a.samples[(size_t)bi * 3 + d] - a.xyz[d * n + node];
        d0 += e0 * e0;
        d1 += e1 * e1;
      }
      if (d0 < w * w) {
        const int e = a.cells[bi / NP];
        double c[NP];
        cell_coeffs(a, e, c);
        const double node_x[3] = {a.xyz[node], a.xyz[n + node], a.xyz[2 * n + node]};
        double pt[3] = {a.samples[(size_t)bi * 3], a.samples[(size_t)bi * 3 + 1], a.samples[(size_t)bi * 3 + 2]};
        const double init[3] = {pt[0], pt[1], pt[2]};
        double lambda = 0.0;
        bool conv = false;
        for (int step = 0; step < 50; ++step) {
          const double old[3] = {pt[0], pt[1], pt[2]};
          double v, gx[3], hx[6];
          phys_eval<P>(a, e, c, pt, &v, gx, hx);
          const double g2 = gx[0] * gx[0] + gx[1] * gx[1] + gx[2] * gx[2];
          if (g2 < 1e-14) break;
          if (step == 0)
            lambda = ((node_x[0] - pt[0]) * gx[0] + (node_x[1] - pt[1]) * gx[1] + (node_x[2] - pt[2]) * gx[2]) / g2;
          double f[4] = {pt[0] - node_x[0] + lambda * gx[0], pt[1] - node_x[1] + lambda * gx[1],
                         pt[2] - node_x[2] + lambda * gx[2], v};
          double H[4][4] = {{1.0 + lambda * hx[0], lambda * hx[3], lambda * hx[4], gx[0]},
                            {lambda * hx[3], 1.0 + lambda * hx[1], lambda * hx[5], gx[1]},
                            {lambda * hx[4], lambda * hx[5], 1.0 + lambda * hx[2], gx[2]},
                            {gx[0], gx[1], gx[2], 0.0}};
          if (!solve4(H, f)) {
            double d1v[3], d2v[3];
            const double lam = ((node_x[0] - pt[0]) * gx[0] + (node_x[1] - pt[1]) * gx[1] + (node_x[2] - pt[2]) * gx[2]) / g2;
            lambda = lam;
            double m2 = 0.0;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              d1v[d] = (v / g2) * gx[d];
              d2v[d] = pt[d] - node_x[d] + lam * gx[d];
              m2 += d2v[d] * d2v[d];
            }
            if (m2 > 0.01 * a.h * a.h) {
              const double sc = 0.1 * a.h / sqrt(m2);
#pragma unroll
              for (int d = 0; d < 3; ++d) d2v[d] *= sc;
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) pt[d] -= d1v[d] + d2v[d];
          } else {
            const double m2 = f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
            if (m2 > 0.25 * a.h * a.h) {
              const double sc = 0.5 * a.h / sqrt(m2);
#pragma unroll
              for (int k = 0; k < 4; ++k) f[k] *= sc;
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) pt[d] -= f[d];
            lambda -= f[3];
          }
          double mv = 0.0, st = 0.0;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            mv += (init[d] - pt[d]) * (init[d] - pt[d]);
            st += (old[d] - pt[d]) * (old[d] - pt[d]);
          }
          if (mv > 2.25 * a.h * a.h) {
#pragma unroll
            for (int d = 0; d < 3; ++d) pt[d] = old[d];
            break;
          }
          if (st < 1e-24) {
            conv = true;
            break;
          }
        }
        double dist2 = d1;
        if (conv) {
          dist2 = 0.0;
#pragma unroll
          for (int d = 0; d < 3; ++d) dist2 += (pt[d] - node_x[d]) * (pt[d] - node_x[d]);
        }
        out = sgn * sqrt(dist2);
      }
    }
    a.s_out[node] = fmax(fmin(a.ls_cap, out), -a.ls_cap);
  }
}

}  // namespace

void ls_reinit_device(sipg_mesh* m, int order, const double* xyz, double* s, double h, double ls_cap,
                      ReinitWork& w, cudaStream_t st) {
  if (m->dim != 3) throw Error(SIPG_INVALID_ARG, "the level-set reinitialisation is 3D");
  if (order < 1 || order > 4) throw Error(SIPG_INVALID_ARG, "order must be 1..4");
  m->ensure_device();
  const ReinitTables& t = reinit_tables(order);
  const int Np = np_of(3, order);
  const size_t n = (size_t)m->K * Np;
  ensure(w.cells, (size_t)m->K * sizeof(int));
  ensure(w.count, sizeof(int));
  ensure(w.nearest, n * sizeof(int));
  ensure(w.s_old, n * sizeof(double));
  ReinitArgs a{};
  a.vminv = t.vminv.as<double>();
  a.exps = t.exps.as<int>();
  a.rst = t.rst.as<double>();
  a.geof = m->geof64.as<double>();
  a.xyz = xyz;
  a.s = w.s_old.as<double>();
  a.s_out = s;
  a.cells = w.cells.as<int>();
  a.ncells = w.count.as<int>();
  a.h = h;
  a.ls_cap = ls_cap;
  a.tol = std::max(1e-18, 1e-4 * h * h);
  a.K = m->K;
  a.Np = Np;
  a.order = order;
  SIPG_CUDA(cudaMemcpyAsync(w.s_old.p, s, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  SIPG_CUDA(cudaMemsetAsync(w.count.p, 0, sizeof(int), st));
  const int g1 = std::max(1, std::min((m->K + 255) / 256, num_sms() * 8));
  k_reinit_cells<<<g1, 256, 0, st>>>(a);
  note_launch();
  SIPG_CUDA(cudaGetLastError());
  int ncells = 0;
  SIPG_CUDA(cudaMemcpyAsync(&ncells, w.count.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  SIPG_CUDA(cudaStreamSynchronize(st));
  const int nsamples = ncells * Np;
  ensure(w.samples, std::max<size_t>(1, (size_t)nsamples * 3) * sizeof(double));
  a.samples = w.samples.as<double>();
  a.nearest = w.nearest.as<int>();
  if (ncells > 0) {
    const int g2 = std::max(1, std::min((nsamples + kRThreads - 1) / kRThreads, num_sms() * 8));
    switch (order) {
      case 1: k_reinit_sample<1><<<g2, kRThreads, 0, st>>>(a, ncells); break;
      case 2: k_reinit_sample<2><<<g2, kRThreads, 0, st>>>(a, ncells); break;
      case 3: k_reinit_sample<3><<<g2, kRThreads, 0, st>>>(a, ncells); break;
      default: k_reinit_sample<4><<<g2, kRThreads, 0, st>>>(a, ncells); break;
    }
    note_launch();
    SIPG_CUDA(cudaGetLastError());
  }
  // keep the converged samples, in order (a host pass over the sample list)
  std::vector<double> hs((size_t)nsamples * 3), kept;
  std::vector<int> flat;
  if (nsamples) {
    SIPG_CUDA(cudaMemcpyAsync(hs.data(), w.samples.p, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    SIPG_CUDA(cudaStreamSynchronize(st));
  }
  for (int i = 0; i < nsamples; ++i)
    if (!std::isnan(hs[(size_t)i * 3])) {
      kept.insert(kept.end(), hs.begin() + (size_t)i * 3, hs.begin() + (size_t)i * 3 + 3);
      flat.push_back(i);
    }
  const int nkept = (int)flat.size();
  ensure(w.kept, std::max<size_t>(1, kept.size()) * sizeof(double));
  ensure(w.flat, std::max<size_t>(1, flat.size()) * sizeof(int));
  if (nkept) {
    w.kept.upload(kept.data(), kept.size() * sizeof(double), st);
    w.flat.upload(flat.data(), flat.size() * sizeof(int), st);
  }
  a.csamples = w.kept.as<double>();
  a.cflat = w.flat.as<int>();
  const size_t nthreads = (n + kNpt - 1) / kNpt;
  const int g3 = (int)((nthreads + kRThreads - 1) / kRThreads);
  k_reinit_nearest<<<g3, kRThreads, 0, st>>>(a, nkept);
  note_launch();
  SIPG_CUDA(cudaGetLastError());
  const int g4 = (int)std::max<size_t>(1, std::min<size_t>((n + kRThreads - 1) / kRThreads, (size_t)num_sms() * 16));
  switch (order) {
    case 1: k_reinit_newton<1><<<g4, kRThreads, 0, st>>>(a); break;
    case 2: k_reinit_newton<2><<<g4, kRThreads, 0, st>>>(a); break;
    case 3: k_reinit_newton<3><<<g4, kRThreads, 0, st>>>(a); break;
    default: k_reinit_newton<4><<<g4, kRThreads, 0, st>>>(a); break;
  }
  note_launch();
  SIPG_CUDA(cudaGetLastError());
}

}  // namespace sipg
