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
// Here the whole sequence is one kernel: a warp owns an element (a lane per
// node, two nodes per lane at p = 4), reads velT, grad p, its geometric factors
// and h once, iterates the CG entirely in registers and shared memory, and
// writes velTT once. The reference-element matrices sit in shared memory in the
// layouts that make every product conflict-free (lane i reads consecutive
// doubles; the vector operand is a broadcast), the warp's vectors are exchanged
// through a per-warp shared buffer, and the dot products are xor-butterfly warp
// reductions, which leave the same bits in every lane so the stopping test is
// warp-uniform. The counters the reference accumulates (cells, converged cells,
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

constexpr int kProjWarps = 8;   // warps (elements in flight) per CTA
constexpr int kProjMaxIter = 100;

__host__ __device__ constexpr int proj_np(int D, int P) {
  return D == 2 ? (P + 1) * (P + 2) / 2 : (P + 1) * (P + 2) * (P + 3) / 6;
}
// Matrices in the blob: D_k by columns (D of them), D_k by rows (D), M, and M^-1 in 3D.
__host__ __device__ constexpr int proj_nmat(int D) { return 2 * D + 1 + (D == 3 ? 1 : 0); }
template <int D, int P>
__host__ __device__ constexpr int proj_smem_doubles() {
  // matrices + per warp: A (D x Np), B (D x Np), C (Np)
  return proj_nmat(D) * proj_np(D, P) * proj_np(D, P) + kProjWarps * (2 * D + 1) * proj_np(D, P);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One element, one warp. NPL = nodes per lane.
template <int D, int P>
__global__ void __launch_bounds__(kProjWarps * 32)
k_proj_cg(int K, const double* __restrict__ geof, const double* __restrict__ hK,
          const double* __restrict__ mats, double dt, double factor, const double* __restrict__ dp,
          const double* __restrict__ velT, double* __restrict__ velTT,
          unsigned long long* __restrict__ stats) {
  constexpr int NP = proj_np(D, P), NPP = NP * NP, NPL = (NP + 31) / 32, NG = D == 3 ? 10 : 5;
  constexpr bool kPre = D == 3;
  extern __shared__ double sm[];
  double* sDc = sm;                       // D_k(i, j) at k*NPP + j*NP + i
  double* sDr = sm + D * NPP;             // D_k(j, i) at k*NPP + j*NP + i
  double* sM = sm + 2 * D * NPP;          // M(i, j) at j*NP + i
  double* sMi = sm + (2 * D + 1) * NPP;   // M^-1(i, j) at j*NP + i (3D)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sA = sm + proj_nmat(D) * NPP + warp * (2 * D + 1) * NP;
  double* sB = sA + D * NP;
  double* sC = sB + D * NP;
  for (int i = threadIdx.x; i < proj_nmat(D) * NPP; i += blockDim.x) sm[i] = mats[i];
  __syncthreads();

  const size_t n = (size_t)K * NP;
  const double tol = kPre ? 1e-8 : 1e-16;
  unsigned long long n_conv = 0, n_iter = 0;

  for (int e = blockIdx.x * kProjWarps + warp; e < K; e += gridDim.x * kProjWarps) {
    double G[3][3] = {};
    double J;
    if (D == 3) {
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) G[k][c] = __ldg(geof + (size_t)e * NG + k * 3 + c);
      J = __ldg(geof + (size_t)e * NG + 9);
    } else {
      G[0][0] = __ldg(geof + (size_t)e * NG + 0); G[0][1] = __ldg(geof + (size_t)e * NG + 1);
      G[1][0] = __ldg(geof + (size_t)e * NG + 2); G[1][1] = __ldg(geof + (size_t)e * NG + 3);
      J = __ldg(geof + (size_t)e * NG + 4);
    }
    const double pen = factor * (__ldg(hK + e) / ((double)P + 1.0));
    const double inv_J = 1.0 / J;

    double x[D][NPL], r[D][NPL], z[D][NPL], p[D][NPL], ap[D][NPL], mv[D][NPL];

    // out = pen * G^T D^T (J M (D G v)) + J M v; mvo = J M v. v is read from sB.
    auto apply = [&](double (&out)[D][NPL], double (&mvo)[D][NPL]) {
      // stage 1: (G v)_k at the lane's nodes -> sA (v already in sB)
#pragma unroll
      for (int q = 0; q < NPL; ++q) {
        const int i = lane + 32 * q;
        if (i < NP) {
#pragma unroll
          for (int k = 0; k < D; ++k) {
            double s = 0.0;
#pragma unroll
            for (int c = 0; c < D; ++c) s += G[k][c] * sB[c * NP + i];
            sA[k * NP + i] = s;
          }
        }
      }
      __syncwarp();
      // stage 2: divergence d = sum_k D_k (G v)_k -> sC
#pragma unroll
      for (int q = 0; q < NPL; ++q) {
        const int i = lane + 32 * q;
        if (i < NP) {
          double d = 0.0;
#pragma unroll
          for (int k = 0; k < D; ++k) {
            double s = 0.0;
#pragma unroll 4
            for (int j = 0; j < NP; ++j) s += sDc[k * NPP + j * NP + i] * sA[k * NP + j];
            d += s;
          }
          sC[i] = d;
        }
      }
      __syncwarp();
      // stage 3: m = J M d -> sA[0..NP)
#pragma unroll
      for (int q = 0; q < NPL; ++q) {
        const int i = lane + 32 * q;
        if (i < NP) {
          double s = 0.0;
#pragma unroll 4
          for (int j = 0; j < NP; ++j) s += sM[j * NP + i] * sC[j];
          sA[i] = J * s;
        }
      }
      __syncwarp();
      // stages 4-5: w_k = D_k^T m, out_c = pen * sum_k G_kc w_k + J (M v_c)
#pragma unroll
      for (int q = 0; q < NPL; ++q) {
        const int i = lane + 32 * q;
        if (i < NP) {
          double w[D];
#pragma unroll
          for (int k = 0; k < D; ++k) {
            double s = 0.0;
#pragma unroll 4
            for (int j = 0; j < NP; ++j) s += sDr[k * NPP + j * NP + i] * sA[j];
            w[k] = s;
          }
#pragma unroll
          for (int c = 0; c < D; ++c) {
            double s = 0.0, mm = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) s += G[k][c] * w[k];
#pragma unroll 4
            for (int j = 0; j < NP; ++j) mm += sM[j * NP + i] * sB[c * NP + j];
            mvo[c][q] = J * mm;
            out[c][q] = pen * s + mvo[c][q];
          }
        } else {
#pragma unroll
          for (int c = 0; c < D; ++c) { out[c][q] = 0.0; mvo[c][q] = 0.0; }
        }
      }
    };
    // z = (1/J) M^-1 r (3D) or r (2D); returns the lane's part of r . z
    auto precondition = [&]() {
      double rz = 0.0;
      if (kPre) {
        __syncwarp();
#pragma unroll
        for (int q = 0; q < NPL; ++q) {
          const int i = lane + 32 * q;
          if (i < NP)
#pragma unroll
            for (int c = 0; c < D; ++c) sB[c * NP + i] = r[c][q];
        }
        __syncwarp();
      }
#pragma unroll
      for (int q = 0; q < NPL; ++q) {
        const int i = lane + 32 * q;
#pragma unroll
        for (int c = 0; c < D; ++c) {
          double s = 0.0;
          if (i < NP) {
            if (kPre) {
#pragma unroll 4
              for (int j = 0; j < NP; ++j) s += sMi[j * NP + i] * sB[c * NP + j];
              s = inv_J * s;
            } else {
              s = r[c][q];
            }
          }
          z[c][q] = s;
          rz += r[c][q] * s;
        }
      }
      return rz;
    };
    auto stage_v = [&](const double (&v)[D][NPL]) {
      __syncwarp();
#pragma unroll
      for (int q = 0; q < NPL; ++q) {
        const int i = lane + 32 * q;
        if (i < NP)
#pragma unroll
          for (int c = 0; c < D; ++c) sB[c * NP + i] = v[c][q];
      }
      __syncwarp();
    };

    // velTT = velT - dt grad p: the initial guess and, through J M, the right-hand side
#pragma unroll
    for (int q = 0; q < NPL; ++q) {
      const int i = lane + 32 * q;
#pragma unroll
      for (int c = 0; c < D; ++c) {
        const size_t g = c * n + (size_t)e * NP + i;
        x[c][q] = i < NP ? __ldg(velT + g) - dt * __ldg(dp + g) : 0.0;
      }
    }
    stage_v(x);
    apply(ap, mv);
    double res = 0.0;
#pragma unroll
    for (int q = 0; q < NPL; ++q)
#pragma unroll
      for (int c = 0; c < D; ++c) {
        r[c][q] = mv[c][q] - ap[c][q];
        res += r[c][q] * r[c][q];
      }
    res = warp_sum(res);
    if (kPre) res = sqrt(res);
    double rz = warp_sum(precondition());
#pragma unroll
    for (int q = 0; q < NPL; ++q)
#pragma unroll
      for (int c = 0; c < D; ++c) p[c][q] = z[c][q];

    int it = 0;
    while (res > tol && it < kProjMaxIter) {
      stage_v(p);
      apply(ap, mv);
      double pap = 0.0;
#pragma unroll
      for (int q = 0; q < NPL; ++q)
#pragma unroll
        for (int c = 0; c < D; ++c) pap += p[c][q] * ap[c][q];
      pap = warp_sum(pap);
      const double alpha = rz / pap;
      res = 0.0;
#pragma unroll
      for (int q = 0; q < NPL; ++q)
#pragma unroll
        for (int c = 0; c < D; ++c) {
          x[c][q] += alpha * p[c][q];
          r[c][q] -= alpha * ap[c][q];
          res += r[c][q] * r[c][q];
        }
      res = warp_sum(res);
      if (kPre) res = sqrt(res);
      if (res < tol) break;
      const double rz_new = warp_sum(precondition());
      const double beta = rz_new / rz;
      rz = rz_new;
#pragma unroll
      for (int q = 0; q < NPL; ++q)
#pragma unroll
        for (int c = 0; c < D; ++c) p[c][q] = z[c][q] + beta * p[c][q];
      ++it;
    }
#pragma unroll
    for (int q = 0; q < NPL; ++q) {
      const int i = lane + 32 * q;
      if (i < NP)
#pragma unroll
        for (int c = 0; c < D; ++c) velTT[c * n + (size_t)e * NP + i] = x[c][q];
    }
    n_iter += (unsigned long long)it;
    n_conv += (it < kProjMaxIter && !isnan(res)) ? 1ull : 0ull;
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
  const int Np = ref.Np, NPP = Np * Np;
  const std::vector<double>* Dk[3] = {&ref.Dr, &ref.Ds, &ref.Dt};
  std::vector<double> b((size_t)proj_nmat(dim) * NPP);
  for (int k = 0; k < dim; ++k)
    for (int i = 0; i < Np; ++i)
      for (int j = 0; j < Np; ++j) {
        b[(size_t)k * NPP + j * Np + i] = (*Dk[k])[(size_t)i * Np + j];           // by columns
        b[(size_t)(dim + k) * NPP + j * Np + i] = (*Dk[k])[(size_t)j * Np + i];   // by rows
      }
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      b[(size_t)2 * dim * NPP + j * Np + i] = ref.M[(size_t)i * Np + j];
      if (dim == 3) b[(size_t)(2 * dim + 1) * NPP + j * Np + i] = ref.Minv[(size_t)i * Np + j];
    }
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
    DevBuf d_dp(std::max<size_t>(bytes, 8)), d_v(std::max<size_t>(bytes, 8)), d_out(std::max<size_t>(bytes, 8));
    DevBuf d_st(2 * sizeof(unsigned long long));
    SIPG_CUDA(cudaMemcpy(d_dp.p, dp, bytes, cudaMemcpyHostToDevice));
    SIPG_CUDA(cudaMemcpy(d_v.p, velT, bytes, cudaMemcpyHostToDevice));
    project_device(m, order, dt, factor, d_dp.as<double>(), d_v.as<double>(), d_out.as<double>(),
                   d_st.as<unsigned long long>(), 0);
    unsigned long long st[2] = {0, 0};
    SIPG_CUDA(cudaMemcpy(velTT, d_out.p, bytes, cudaMemcpyDeviceToHost));
    SIPG_CUDA(cudaMemcpy(st, d_st.p, sizeof(st), cudaMemcpyDeviceToHost));
    if (stats) {
      stats[0] = (double)m->K;
      stats[1] = (double)st[0];
      stats[2] = (double)st[1];
    }
  });
}
