// Element-local velocity projection of the pressure step.
//
// INSSolverBase3D::project_velocity with `div_div = 1` (pr_projection_method 1,
// src/solvers/3d/ins_solver_base.cpp:1052-1124; 2D
// src/solvers/2d/ins_solver_base.cpp:894-955) runs four OP2 loops and two mass
// passes over the cells: ins_3d_proj_rhs (velTT = velT - dt grad p), mesh->mass
// (b = J M velTT), ins_3d_proj_pen (pen = factor h / (p + 1), h from
// ins_proj_setup_0/1 at set-up, ins_solver_base.cpp:201-214) and
// ins_3d_proj_cg_precon, a conjugate-gradient solve per element of
//   (J M + pen G^T D^T J M D G) velTT = b
// on the dim x Np velocity unknowns of the element, preconditioned by the
// inverse mass matrix (1/J) M^-1 in 3D (ins_3d_proj_cg_precon.h:1-160) and
// unpreconditioned in 2D (ins_proj_cg_2d.h), stopping on the absolute residual
// (3D |r|_2 < 1e-8, 2D |r|_2^2 < 1e-16) or after 100 iterations.
//
// Here the whole sequence is one kernel. A warp owns two elements (one at
// p = 4 in 3D), a lane per node: it reads velT, grad p, the geometric factors
// and h once, iterates both elements' CG in registers and shared memory, and
// writes velTT once. The solve is bound by shared-memory bandwidth (the
// reference-element matrices are read from shared memory at every product), so
// the kernel minimises shared traffic per multiply-add: each matrix entry read
// serves both elements of the warp, matrix entries and vector values are read
// in 16-byte pairs (column pairs of Np rows; vectors padded to an even length
// with zeros), and in 3D the mass term J M p of the operator is carried by the
// recursion J M p_new = r_new + beta J M p (since J M z = r for z = (1/J) M^-1 r)
// instead of three mass products per iteration. Dot products are xor-butterfly
// warp reductions, which leave the same bits in every lane, so the stopping
// tests are warp-uniform; an element that has stopped idles while the other
// finishes. The counters the reference accumulates (cells, converged cells,
// iterations) are summed per warp and added once per warp.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/sipg_b200.h"
#include "capi_util.hpp"
#include "vecops.cuh"

namespace sipg {
namespace {

constexpr int kProjWarps = 4;   // warps per CTA
constexpr int kProjMaxIter = 100;

__host__ __device__ constexpr int proj_np(int D, int P) {
  return D == 2 ? (P + 1) * (P + 2) / 2 : (P + 1) * (P + 2) * (P + 3) / 6;
}
// Np rounded up to even: vectors and matrix columns are read in pairs.
__host__ __device__ constexpr int proj_npe(int D, int P) { return (proj_np(D, P) + 1) & ~1; }
// Elements per warp: two while a node per lane covers the element, else one.
__host__ __device__ constexpr int proj_epw(int D, int P) { return proj_np(D, P) <= 32 ? 2 : 1; }
// Matrices in the blob: D_k for products (D), D_k^T for products (D), M, and M^-1 in 3D;
// each stored as Npe/2 column pairs of Np rows: A(i, 2q + t) at (q * Np + i) * 2 + t.
__host__ __device__ constexpr int proj_nmat(int D) { return 2 * D + 1 + (D == 3 ? 1 : 0); }
template <int D, int P>
__host__ __device__ constexpr int proj_mat_doubles() { return proj_np(D, P) * proj_npe(D, P); }
template <int D, int P>
__host__ __device__ constexpr int proj_smem_doubles() {
  // matrices + per warp and element: A (D x Npe), B (D x Npe), C (Npe)
  return proj_nmat(D) * proj_mat_doubles<D, P>() + kProjWarps * proj_epw(D, P) * (2 * D + 1) * proj_npe(D, P);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// y_e(i) = sum_j A(i, j) v_e(j) for the E vectors v_e (stride vs doubles apart),
// even and odd j summed separately (two independent FMA chains); A in the pair
// layout, v padded with zeros to Npe.
template <int NP, int NPE, int E>
__device__ __forceinline__ void mat_vec(const double* __restrict__ A, const double* v, int vs, int i,
                                        double (&y)[E]) {
  double y1[E];
#pragma unroll
  for (int e = 0; e < E; ++e) y[e] = y1[e] = 0.0;
#pragma unroll 5
  for (int q = 0; q < NPE / 2; ++q) {
    const double2 a = *reinterpret_cast<const double2*>(A + (q * NP + i) * 2);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const double2 x = *reinterpret_cast<const double2*>(v + e * vs + 2 * q);
      y[e] += a.x * x.x;
      y1[e] += a.y * x.y;
    }
  }
#pragma unroll
  for (int e = 0; e < E; ++e) y[e] += y1[e];
}

// E elements per warp (a lane per node, NPL nodes per lane).
template <int D, int P>
__global__ void __launch_bounds__(kProjWarps * 32)
k_proj_cg(int K, const double* __restrict__ geof, const double* __restrict__ hK,
          const double* __restrict__ mats, double dt, double factor, const double* __restrict__ dp,
          const double* __restrict__ velT, double* __restrict__ velTT,
          unsigned long long* __restrict__ stats) {
  constexpr int NP = proj_np(D, P), NPE = proj_npe(D, P), NPL = (NP + 31) / 32, NG = D == 3 ? 10 : 5;
  constexpr int E = proj_epw(D, P), MAT = proj_mat_doubles<D, P>();
  constexpr int WB = E * (2 * D + 1) * NPE;  // per-warp buffer
  constexpr bool kPre = D == 3;
  extern __shared__ double sm[];
  const double* sD = sm;                  // D_k, k < D
  const double* sDt = sm + D * MAT;       // D_k^T
  const double* sM = sm + 2 * D * MAT;    // M
  const double* sMi = sm + (2 * D + 1) * MAT;  // M^-1 (3D)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sA = sm + proj_nmat(D) * MAT + warp * WB;  // [E][D][NPE]
  double* sB = sA + E * D * NPE;                      // [E][D][NPE]
  double* sC = sB + E * D * NPE;                      // [E][NPE]
  for (int i = threadIdx.x; i < proj_nmat(D) * MAT; i += blockDim.x) sm[i] = mats[i];
  // zero the warp buffers once: their pad entries (Np..Npe-1) stay zero
  for (int i = lane; i < WB; i += 32) sA[i] = 0.0;
  __syncthreads();

  const size_t n = (size_t)K * NP;
  const double tol = kPre ? 1e-8 : 1e-16;
  unsigned long long n_conv = 0, n_iter = 0;

  for (int e0 = (blockIdx.x * kProjWarps + warp) * E; e0 < K; e0 += gridDim.x * kProjWarps * E) {
    double G[E][3][3], J[E], pen[E], inv_J[E];
    bool valid[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int el = e0 + e;
      valid[e] = el < K;
      const int ec = valid[e] ? el : e0;
      const double* g = geof + (size_t)ec * NG;
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) G[e][k][c] = 0.0;
      if (D == 3) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int c = 0; c < 3; ++c) G[e][k][c] = __ldg(g + k * 3 + c);
        J[e] = __ldg(g + 9);
      } else {
        G[e][0][0] = __ldg(g + 0); G[e][0][1] = __ldg(g + 1);
        G[e][1][0] = __ldg(g + 2); G[e][1][1] = __ldg(g + 3);
        J[e] = __ldg(g + 4);
      }
      pen[e] = factor * (__ldg(hK + ec) / ((double)P + 1.0));
      inv_J[e] = 1.0 / J[e];
    }

    double x[E][D][NPL], r[E][D][NPL], z[E][D][NPL], p[E][D][NPL], ap[E][D][NPL], q[E][D][NPL];

    // ap = pen * G^T D^T (J M (D G v)) + mass, v read from sB; mass = J M v when
    // explicit_mass (also returned in q), else the q carried by the caller.
    auto apply = [&](bool explicit_mass) {
#pragma unroll
      for (int u = 0; u < NPL; ++u) {  // (G v)_k -> sA
        const int i = lane + 32 * u;
        if (i < NP)
#pragma unroll
          for (int e = 0; e < E; ++e)
#pragma unroll
            for (int k = 0; k < D; ++k) {
              double s = 0.0;
#pragma unroll
              for (int c = 0; c < D; ++c) s += G[e][k][c] * sB[(e * D + c) * NPE + i];
              sA[(e * D + k) * NPE + i] = s;
            }
      }
      __syncwarp();
#pragma unroll
      for (int u = 0; u < NPL; ++u) {  // divergence d = sum_k D_k (G v)_k -> sC
        const int i = lane + 32 * u;
        if (i < NP) {
          double d[E];
#pragma unroll
          for (int e = 0; e < E; ++e) d[e] = 0.0;
#pragma unroll
          for (int k = 0; k < D; ++k) {
            double s[E];
            mat_vec<NP, NPE, E>(sD + k * MAT, sA + k * NPE, D * NPE, i, s);
#pragma unroll
            for (int e = 0; e < E; ++e) d[e] += s[e];
          }
#pragma unroll
          for (int e = 0; e < E; ++e) sC[e * NPE + i] = d[e];
        }
      }
      __syncwarp();
#pragma unroll
      for (int u = 0; u < NPL; ++u) {  // m = J M d -> sA[e][0]
        const int i = lane + 32 * u;
        if (i < NP) {
          double s[E];
          mat_vec<NP, NPE, E>(sM, sC, NPE, i, s);
#pragma unroll
          for (int e = 0; e < E; ++e) sA[e * D * NPE + i] = J[e] * s[e];
        }
      }
      __syncwarp();
#pragma unroll
      for (int u = 0; u < NPL; ++u) {  // w_k = D_k^T m; ap_c = pen sum_k G_kc w_k + mass_c
        const int i = lane + 32 * u;
        if (i < NP) {
          double w[D][E];
#pragma unroll
          for (int k = 0; k < D; ++k) mat_vec<NP, NPE, E>(sDt + k * MAT, sA, D * NPE, i, w[k]);
          if (explicit_mass)
#pragma unroll
            for (int c = 0; c < D; ++c) {
              double s[E];
              mat_vec<NP, NPE, E>(sM, sB + c * NPE, D * NPE, i, s);
#pragma unroll
              for (int e = 0; e < E; ++e) q[e][c][u] = J[e] * s[e];
            }
#pragma unroll
          for (int e = 0; e < E; ++e)
#pragma unroll
            for (int c = 0; c < D; ++c) {
              double s = 0.0;
#pragma unroll
              for (int k = 0; k < D; ++k) s += G[e][k][c] * w[k][e];
              ap[e][c][u] = pen[e] * s + q[e][c][u];
            }
        } else {
#pragma unroll
          for (int e = 0; e < E; ++e)
#pragma unroll
            for (int c = 0; c < D; ++c) { ap[e][c][u] = 0.0; q[e][c][u] = 0.0; }
        }
      }
    };
    auto stage = [&](const double (&v)[E][D][NPL]) {
      __syncwarp();
#pragma unroll
      for (int u = 0; u < NPL; ++u) {
        const int i = lane + 32 * u;
        if (i < NP)
#pragma unroll
          for (int e = 0; e < E; ++e)
#pragma unroll
            for (int c = 0; c < D; ++c) sB[(e * D + c) * NPE + i] = v[e][c][u];
      }
      __syncwarp();
    };
    // z = (1/J) M^-1 r (3D) or r (2D); rz = r . z per element (warp sums)
    auto precondition = [&](double (&rz)[E]) {
      if (kPre) stage(r);
#pragma unroll
      for (int e = 0; e < E; ++e) rz[e] = 0.0;
#pragma unroll
      for (int u = 0; u < NPL; ++u) {
        const int i = lane + 32 * u;
#pragma unroll
        for (int c = 0; c < D; ++c) {
          double s[E];
          if (kPre && i < NP) {
            mat_vec<NP, NPE, E>(sMi, sB + c * NPE, D * NPE, i, s);
#pragma unroll
            for (int e = 0; e < E; ++e) s[e] = inv_J[e] * s[e];
          } else {
#pragma unroll
            for (int e = 0; e < E; ++e) s[e] = i < NP ? r[e][c][u] : 0.0;
          }
#pragma unroll
          for (int e = 0; e < E; ++e) {
            z[e][c][u] = s[e];
            rz[e] += r[e][c][u] * s[e];
          }
        }
      }
#pragma unroll
      for (int e = 0; e < E; ++e) rz[e] = warp_sum(rz[e]);
    };

    // velTT = velT - dt grad p: the initial guess and, through J M, the right-hand side
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int u = 0; u < NPL; ++u) {
        const int i = lane + 32 * u;
#pragma unroll
        for (int c = 0; c < D; ++c) {
          const size_t g = c * n + (size_t)(e0 + e) * NP + i;
          x[e][c][u] = (valid[e] && i < NP) ? __ldg(velT + g) - dt * __ldg(dp + g) : 0.0;
        }
      }
    stage(x);
    apply(true);  // q = J M x is the right-hand side, ap = A x
    double res[E], rz[E];
    bool active[E];
    int it[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      double s = 0.0;
#pragma unroll
      for (int u = 0; u < NPL; ++u)
#pragma unroll
        for (int c = 0; c < D; ++c) {
          r[e][c][u] = q[e][c][u] - ap[e][c][u];
          s += r[e][c][u] * r[e][c][u];
        }
      s = warp_sum(s);
      res[e] = kPre ? sqrt(s) : s;
      it[e] = 0;
      active[e] = valid[e] && res[e] > tol;
    }
    precondition(rz);
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int u = 0; u < NPL; ++u)
#pragma unroll
        for (int c = 0; c < D; ++c) {
          p[e][c][u] = z[e][c][u];
          q[e][c][u] = r[e][c][u];  // J M p = J M z = r (3D)
        }

    bool any = false;
#pragma unroll
    for (int e = 0; e < E; ++e) any |= active[e];
    while (any) {
      stage(p);
      apply(!kPre);  // 3D: J M p is carried in q
      double pap[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        double s = 0.0;
#pragma unroll
        for (int u = 0; u < NPL; ++u)
#pragma unroll
          for (int c = 0; c < D; ++c) s += p[e][c][u] * ap[e][c][u];
        pap[e] = warp_sum(s);
      }
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const double alpha = rz[e] / pap[e];
        double s = 0.0;
#pragma unroll
        for (int u = 0; u < NPL; ++u)
#pragma unroll
          for (int c = 0; c < D; ++c) {
            if (active[e]) {
              x[e][c][u] += alpha * p[e][c][u];
              r[e][c][u] -= alpha * ap[e][c][u];
            }
            s += r[e][c][u] * r[e][c][u];
          }
        s = warp_sum(s);
        if (active[e]) {
          res[e] = kPre ? sqrt(s) : s;
          if (res[e] < tol) active[e] = false;  // the reference's break: not counted
        }
      }
      double rz_new[E];
      precondition(rz_new);
      any = false;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        if (active[e]) {
          const double beta = rz_new[e] / rz[e];
          rz[e] = rz_new[e];
#pragma unroll
          for (int u = 0; u < NPL; ++u)
#pragma unroll
            for (int c = 0; c < D; ++c) {
              p[e][c][u] = z[e][c][u] + beta * p[e][c][u];
              if (kPre) q[e][c][u] = r[e][c][u] + beta * q[e][c][u];
            }
          ++it[e];
          active[e] = res[e] > tol && it[e] < kProjMaxIter;
        }
        any |= active[e];
      }
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
      if (!valid[e]) continue;
#pragma unroll
      for (int u = 0; u < NPL; ++u) {
        const int i = lane + 32 * u;
        if (i < NP)
#pragma unroll
          for (int c = 0; c < D; ++c) velTT[c * n + (size_t)(e0 + e) * NP + i] = x[e][c][u];
      }
      n_iter += (unsigned long long)it[e];
      n_conv += (it[e] < kProjMaxIter && !isnan(res[e])) ? 1ull : 0ull;
    }
  }
  if (stats && lane == 0) {
    atomicAdd(stats + 0, n_conv);
    atomicAdd(stats + 1, n_iter);
  }
}

// Reference-element matrices in the kernel's layouts, per (device, dim, order).
struct ProjMats {
  DevBuf blob;
  int Np = 0;
};

const ProjMats& proj_mats(int dim, int order) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::unique_ptr<ProjMats>> cache;
  int dev = 0;
  SIPG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  auto& slot = cache[{dev, dim * 10 + order}];
  if (slot) return *slot;
  const DevRef& dr = dev_ref(dim, order);
  const RefElement& ref = dr.ref;
  const int Np = ref.Np, Npe = (Np + 1) & ~1;
  const size_t MAT = (size_t)Np * Npe;
  std::vector<double> b((size_t)proj_nmat(dim) * MAT, 0.0);  // pad columns stay zero
  // A(i, j) of matrix m at m * MAT + ((j / 2) * Np + i) * 2 + j % 2; rm: row-major source
  auto put = [&](int m, const std::vector<double>& rm, bool transpose) {
    for (int i = 0; i < Np; ++i)
      for (int j = 0; j < Np; ++j)
        b[m * MAT + ((size_t)(j / 2) * Np + i) * 2 + j % 2] = transpose ? rm[(size_t)j * Np + i] : rm[(size_t)i * Np + j];
  };
  const std::vector<double>* Dk[3] = {&ref.Dr, &ref.Ds, &ref.Dt};
  for (int k = 0; k < dim; ++k) {
    put(k, *Dk[k], false);
    put(dim + k, *Dk[k], true);
  }
  put(2 * dim, ref.M, false);
  if (dim == 3) put(2 * dim + 1, ref.Minv, false);
  auto pm = std::make_unique<ProjMats>();
  pm->Np = Np;
  pm->blob = DevBuf(b.size() * sizeof(double));
  pm->blob.upload(b.data(), b.size() * sizeof(double));
  SIPG_CUDA(cudaDeviceSynchronize());
  slot = std::move(pm);
  return *slot;
}

// 1 / (largest fscale over the element's interior faces), once per mesh
// (ins_proj_setup_0.h / ins_proj_setup_1.h).
const double* proj_h_device(sipg_mesh* m) {
  m->ensure_device();
  std::lock_guard<std::mutex> lk(m->dev_mu);
  if (!m->proj_h.p) {
    const Mesh& h = m->host_order(1);
    const int Nf = m->dim + 1;
    std::vector<double> hv(m->K);
    for (int e = 0; e < m->K; ++e) {
      double mx = 0.0;
      for (int f = 0; f < Nf; ++f)
        if (h.nbr[(size_t)e * Nf + f] >= 0) mx = std::fmax(mx, h.fscale[(size_t)e * Nf + f]);
      hv[e] = 1.0 / mx;
    }
    DevBuf b((size_t)m->K * sizeof(double));
    b.upload(hv.data(), hv.size() * sizeof(double));
    SIPG_CUDA(cudaDeviceSynchronize());
    m->proj_h = std::move(b);
  }
  return m->proj_h.as<double>();
}

template <int D, int P>
void launch_proj(sipg_mesh* m, const double* mats, const double* hK, double dt, double factor, const double* dp,
                 const double* velT, double* velTT, unsigned long long* stats, cudaStream_t s) {
  constexpr size_t smem = proj_smem_doubles<D, P>() * sizeof(double);
  static_assert(smem <= 227 * 1024, "projection shared memory");
  auto kern = k_proj_cg<D, P>;
  SIPG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  SIPG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kProjWarps * 32, smem));
  per_sm = std::max(per_sm, 1);
  const int need = (m->K + kProjWarps - 1) / kProjWarps;
  const int grid = std::max(1, std::min(need, per_sm * num_sms()));
  kern<<<grid, kProjWarps * 32, smem, s>>>(m->K, m->geof64.as<double>(), hK, mats, dt, factor, dp, velT, velTT,
                                           stats);
  SIPG_CUDA(cudaGetLastError());
  note_launch();
}

void project_device(sipg_mesh* m, int order, double dt, double factor, const double* dp, const double* velT,
                    double* velTT, unsigned long long* stats, cudaStream_t s) {
  if (!m || order < 1 || order > 4 || !dp || !velT || !velTT)
    throw Error(SIPG_INVALID_ARG, "project_velocity: null mesh/array or order outside 1..4");
  if (!std::isfinite(dt) || !std::isfinite(factor)) throw Error(SIPG_INVALID_ARG, "project_velocity: dt/factor");
  if (velTT == velT || velTT == dp) throw Error(SIPG_INVALID_ARG, "project_velocity: velTT must not alias its inputs");
  const double* hK = proj_h_device(m);
  const double* mats = proj_mats(m->dim, order).blob.as<double>();
  if (stats) SIPG_CUDA(cudaMemsetAsync(stats, 0, 2 * sizeof(unsigned long long), s));
  if (m->K == 0) return;
  switch (m->dim * 10 + order) {
    case 21: launch_proj<2, 1>(m, mats, hK, dt, factor, dp, velT, velTT, stats, s); break;
    case 22: launch_proj<2, 2>(m, mats, hK, dt, factor, dp, velT, velTT, stats, s); break;
    case 23: launch_proj<2, 3>(m, mats, hK, dt, factor, dp, velT, velTT, stats, s); break;
    case 24: launch_proj<2, 4>(m, mats, hK, dt, factor, dp, velT, velTT, stats, s); break;
    case 31: launch_proj<3, 1>(m, mats, hK, dt, factor, dp, velT, velTT, stats, s); break;
    case 32: launch_proj<3, 2>(m, mats, hK, dt, factor, dp, velT, velTT, stats, s); break;
    case 33: launch_proj<3, 3>(m, mats, hK, dt, factor, dp, velT, velTT, stats, s); break;
    case 34: launch_proj<3, 4>(m, mats, hK, dt, factor, dp, velT, velTT, stats, s); break;
    default: throw Error(SIPG_INVALID_ARG, "project_velocity: dimension");
  }
}

}  // namespace
}  // namespace sipg

using namespace sipg;

extern "C" int sipg_project_velocity(sipg_mesh* m, int order, double dt, double factor, const double* dp,
                                     const double* velT, double* velTT, unsigned long long* stats,
                                     void* stream) {
  return guarded([&] { project_device(m, order, dt, factor, dp, velT, velTT, stats, (cudaStream_t)stream); });
}

extern "C" int sipg_project_velocity_host(sipg_mesh* m, int order, double dt, double factor, const double* dp,
                                          const double* velT, double* velTT, double* stats) {
  return guarded([&] {
    if (!m || order < 1 || order > 4 || !dp || !velT || !velTT)
      throw Error(SIPG_INVALID_ARG, "project_velocity: null mesh/array or order outside 1..4");
    const size_t n = (size_t)m->dim * m->K * np_of(m->dim, order), bytes = n * sizeof(double);
    // device copies stay on the mesh between calls (grown on demand), so a time
    // step's projection allocates nothing after the first call
    std::lock_guard<std::mutex> lk(m->proj_mu);
    const size_t need = 3 * bytes + 2 * sizeof(unsigned long long);
    if (m->proj_io.bytes < need) {
      m->proj_io = DevBuf();
      m->proj_io = DevBuf(need);
    }
    char* base = m->proj_io.as<char>();
    double* d_dp = reinterpret_cast<double*>(base);
    double* d_v = reinterpret_cast<double*>(base + bytes);
    double* d_out = reinterpret_cast<double*>(base + 2 * bytes);
    auto* d_st = reinterpret_cast<unsigned long long*>(base + 3 * bytes);
    SIPG_CUDA(cudaMemcpy(d_dp, dp, bytes, cudaMemcpyHostToDevice));
    SIPG_CUDA(cudaMemcpy(d_v, velT, bytes, cudaMemcpyHostToDevice));
    project_device(m, order, dt, factor, d_dp, d_v, d_out, d_st, 0);
    unsigned long long st[2] = {0, 0};
    SIPG_CUDA(cudaMemcpy(velTT, d_out, bytes, cudaMemcpyDeviceToHost));
    SIPG_CUDA(cudaMemcpy(st, d_st, sizeof(st), cudaMemcpyDeviceToHost));
    if (stats) {
      stats[0] = (double)m->K;
      stats[1] = (double)st[0];
      stats[2] = (double)st[1];
    }
  });
}
