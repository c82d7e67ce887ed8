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
#include "pdl.cuh"
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
__host__ __device__ constexpr int proj_nfp(int D, int P) { return D == 2 ? P + 1 : (P + 1) * (P + 2) / 2; }
__host__ __device__ constexpr int proj_nfpe(int D, int P) { return (proj_nfp(D, P) + 1) & ~1; }
// LIFT = M^-1 EMAT after the matrices, per face f: LIFT(i, f Nfp + k) in the pair
// layout of an Np x Nfpe block (the fused-gradient variant reads it)
template <int D, int P>
__host__ __device__ constexpr int proj_lift_doubles() { return (D + 1) * proj_np(D, P) * proj_nfpe(D, P); }
template <int D, int P>
__host__ __device__ constexpr int proj_blob_doubles() {
  return proj_nmat(D) * proj_mat_doubles<D, P>() + proj_lift_doubles<D, P>();
}
template <int D, int P>
__host__ __device__ constexpr int proj_warp_doubles() {
  // per element: A (D x Npe), B (D x Npe), C (Npe), face jumps ((D + 1) x Nfpe)
  return proj_epw(D, P) * ((2 * D + 1) * proj_npe(D, P) + (D + 1) * proj_nfpe(D, P));
}
template <int D, int P>
__host__ __device__ constexpr int proj_smem_doubles() {
  return proj_blob_doubles<D, P>() + kProjWarps * proj_warp_doubles<D, P>();
}

struct ProjArgs {
  int K;
  const double* geof;      // K x ngeof
  const double* hK;        // K: penalty length
  const double* mats;      // proj_blob_doubles
  double dt, factor;
  const double* dp;        // grad p, dim x K x Np (plain variant)
  const double* pr;        // pressure, K x Np (fused-gradient variant)
  const double* rho;       // density K x Np or null (fused-gradient variant: grad p / rho)
  const int* nbr;          // K x (dim + 1): neighbour or -(bface + 1)
  const uint32_t* fcode;   // K: byte f = neighbour face | orientation << 2
  const int8_t* itab;      // fmask ((dim + 1) x Nfp) then neighbour node positions (Nperm x Nfp)
  const double* velT;
  double* velTT;
  unsigned long long* stats;
};

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

// E elements per warp (a lane per node, NPL nodes per lane). GRAD: the pressure
// gradient is computed here from the pressure (central flux, then / rho) instead
// of being read.
template <int D, int P, bool GRAD>
__global__ void __launch_bounds__(kProjWarps * 32) k_proj_cg(const ProjArgs a) {
  constexpr int NP = proj_np(D, P), NPE = proj_npe(D, P), NPL = (NP + 31) / 32, NG = D == 3 ? 10 : 5;
  constexpr int NF = D + 1, NFP = proj_nfp(D, P), NFPE = proj_nfpe(D, P);
  constexpr int E = proj_epw(D, P), MAT = proj_mat_doubles<D, P>();
  constexpr int WB = proj_warp_doubles<D, P>();  // per-warp buffer
  constexpr bool kPre = D == 3;
  const int K = a.K;
  const double* __restrict__ geof = a.geof;
  const double* __restrict__ hK = a.hK;
  const double dt = a.dt, factor = a.factor;
  const double* __restrict__ velT = a.velT;
  double* __restrict__ velTT = a.velTT;
  extern __shared__ double sm[];
  const double* sD = sm;                  // D_k, k < D
  const double* sDt = sm + D * MAT;       // D_k^T
  const double* sM = sm + 2 * D * MAT;    // M
  const double* sMi = sm + (2 * D + 1) * MAT;  // M^-1 (3D)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double* sL = sm + proj_nmat(D) * MAT;  // LIFT, per face an Np x Nfpe pair block
  double* sA = sm + proj_blob_doubles<D, P>() + warp * WB;  // [E][D][NPE]
  double* sB = sA + E * D * NPE;                             // [E][D][NPE]
  double* sC = sB + E * D * NPE;                             // [E][NPE]
  double* sJ = sC + E * NPE;                                 // [E][NF][NFPE] face jumps
  for (int i = threadIdx.x; i < proj_blob_doubles<D, P>(); i += blockDim.x) sm[i] = a.mats[i];
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

    // grad p: read, or (GRAD) computed with the central flux and divided by rho
    double gp[E][D][NPL];
    if (GRAD) {
      const int8_t* fmask = a.itab;
      const int8_t* npos = a.itab + NF * NFP;
      __syncwarp();  // the previous element's last reads of sB are done
#pragma unroll
      for (int e = 0; e < E; ++e)
#pragma unroll
        for (int u = 0; u < NPL; ++u) {
          const int i = lane + 32 * u;
          if (i < NP) sB[e * D * NPE + i] = valid[e] ? __ldg(a.pr + (size_t)(e0 + e) * NP + i) : 0.0;
        }
      __syncwarp();
      // (p+ - p-) / 2 at every face node; boundary faces add nothing
#pragma unroll
      for (int e = 0; e < E; ++e)
        for (int m = lane; m < NF * NFP; m += 32) {
          const int f = m / NFP, k = m - f * NFP;
          double jv = 0.0;
          if (valid[e]) {
            const int el = e0 + e;
            const int nb = __ldg(a.nbr + (size_t)el * NF + f);
            if (nb >= 0) {
              const int code = (__ldg(a.fcode + el) >> (8 * f)) & 0xff;
              const int fr = code & 3, sg = code >> 2;
              const int nn = fmask[fr * NFP + npos[sg * NFP + k]];
              jv = 0.5 * (__ldg(a.pr + (size_t)nb * NP + nn) - sB[e * D * NPE + fmask[f * NFP + k]]);
            }
          }
          sJ[(e * NF + f) * NFPE + k] = jv;
        }
      __syncwarp();
#pragma unroll
      for (int u = 0; u < NPL; ++u) {
        const int i = lane + 32 * u;
        if (i < NP) {
          double dr[D][E], lf[NF][E];
#pragma unroll
          for (int k = 0; k < D; ++k) mat_vec<NP, NPE, E>(sD + k * MAT, sB, D * NPE, i, dr[k]);
#pragma unroll
          for (int f = 0; f < NF; ++f) mat_vec<NP, NFPE, E>(sL + f * NP * NFPE, sJ + f * NFPE, NF * NFPE, i, lf[f]);
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const double rinv = (valid[e] && a.rho) ? 1.0 / __ldg(a.rho + (size_t)(e0 + e) * NP + i) : 1.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
              double g = 0.0;
#pragma unroll
              for (int k = 0; k < D; ++k) g += G[e][k][d] * dr[k][e];
              // fscale n of each face (the unnormalised outward normal)
              if (D == 3) {
                g += -G[e][2][d] * lf[0][e];
                g += -G[e][1][d] * lf[1][e];
                g += ((G[e][0][d] + G[e][1][d]) + G[e][2][d]) * lf[2][e];
                g += -G[e][0][d] * lf[3][e];
              } else {
                g += -G[e][1][d] * lf[0][e];
                g += (G[e][0][d] + G[e][1][d]) * lf[1][e];
                g += -G[e][0][d] * lf[2][e];
              }
              gp[e][d][u] = g * rinv;
            }
          }
        } else {
#pragma unroll
          for (int e = 0; e < E; ++e)
#pragma unroll
            for (int d = 0; d < D; ++d) gp[e][d][u] = 0.0;
        }
      }
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e)
#pragma unroll
        for (int u = 0; u < NPL; ++u) {
          const int i = lane + 32 * u;
#pragma unroll
          for (int c = 0; c < D; ++c)
            gp[e][c][u] = (valid[e] && i < NP) ? __ldg(a.dp + c * n + (size_t)(e0 + e) * NP + i) : 0.0;
        }
    }
    // velTT = velT - dt grad p: the initial guess and, through J M, the right-hand side
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int u = 0; u < NPL; ++u) {
        const int i = lane + 32 * u;
#pragma unroll
        for (int c = 0; c < D; ++c) {
          const size_t g = c * n + (size_t)(e0 + e) * NP + i;
          x[e][c][u] = (valid[e] && i < NP) ? __ldg(velT + g) - dt * gp[e][c][u] : 0.0;
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
  if (a.stats && lane == 0) {
    atomicAdd(a.stats + 0, n_conv);
    atomicAdd(a.stats + 1, n_iter);
  }
}


// Right-hand side of the pressure solve, two elements per warp (one at p = 4 in 3D):
//   rhs = J M ( -(div_c velT) / dt + LIFT dPdN_new ),  dPdN_new = b0 dPdN + b1 dPdN_old,
// div_c the central-flux divergence (volume sum_k D_k (G u)_k plus LIFT of
// fscale n . (u+ - u-) / 2 on interior faces); dPdN_old <- dPdN_new.
struct PrRhsArgs {
  int K;
  const double* geof;
  const double* mats;
  double dt, b0, b1;
  const int* nbr;
  const uint32_t* fcode;
  const int8_t* itab;
  const double* velT;      // dim x K x Np
  const double* dPdN;      // K x (dim + 1) x Nfp or null
  double* dPdN_old;        // K x (dim + 1) x Nfp or null
  double* rhs;             // K x Np
};

template <int D, int P>
__global__ void __launch_bounds__(kProjWarps * 32) k_pr_rhs(const PrRhsArgs a) {
  constexpr int NP = proj_np(D, P), NPE = proj_npe(D, P), NPL = (NP + 31) / 32, NG = D == 3 ? 10 : 5;
  constexpr int NF = D + 1, NFP = proj_nfp(D, P), NFPE = proj_nfpe(D, P), MAT = proj_mat_doubles<D, P>();
  constexpr int E = proj_epw(D, P);  // elements per warp: each matrix read serves all of them
  constexpr int WB = E * ((D + 1) * NPE + 2 * NF * NFPE);
  extern __shared__ double sm[];
  const double* sD = sm;
  const double* sM = sm + 2 * D * MAT;
  const double* sL = sm + proj_nmat(D) * MAT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sGU = sm + proj_blob_doubles<D, P>() + warp * WB;  // [E][D][NPE]
  double* sPre = sGU + E * D * NPE;                          // [E][NPE]
  double* sF1 = sPre + E * NPE;                              // [E][NF][NFPE] fscale n . (u+ - u-) / 2
  double* sF2 = sF1 + E * NF * NFPE;                         // [E][NF][NFPE] dPdN_new
  for (int i = threadIdx.x; i < proj_blob_doubles<D, P>(); i += blockDim.x) sm[i] = a.mats[i];
  for (int i = lane; i < WB; i += 32) sGU[i] = 0.0;
  __syncthreads();
  const size_t n = (size_t)a.K * NP;
  const int8_t* fmask = a.itab;
  const int8_t* npos = a.itab + NF * NFP;
  const double inv_dt = 1.0 / a.dt;
  for (int e0 = (blockIdx.x * kProjWarps + warp) * E; e0 < a.K; e0 += gridDim.x * kProjWarps * E) {
    double G[E][3][3], J[E];
    bool valid[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      valid[e] = e0 + e < a.K;
      const double* g = a.geof + (size_t)(valid[e] ? e0 + e : e0) * NG;
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
    }
    __syncwarp();  // the previous elements' reads of the buffers are done
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int u = 0; u < NPL; ++u) {
        const int i = lane + 32 * u;
        if (i < NP) {
          double uc[D];
#pragma unroll
          for (int c = 0; c < D; ++c) uc[c] = valid[e] ? __ldg(a.velT + c * n + (size_t)(e0 + e) * NP + i) : 0.0;
#pragma unroll
          for (int k = 0; k < D; ++k) {
            double s = 0.0;
#pragma unroll
            for (int c = 0; c < D; ++c) s += G[e][k][c] * uc[c];
            sGU[(e * D + k) * NPE + i] = s;
          }
        }
      }
    // face terms: the warp's neighbour indices and face codes first (one lane per
    // element face), then every lane issues all of its face nodes' loads before it uses
    // any of them (the neighbour's velocities wait on the neighbour index)
    constexpr int NFN = NF * NFP, ITEMS = (E * NFN + 31) / 32;
    int nbv = -1;
    uint32_t codev = 0;
    if (lane < E * NF) {
      const int e = lane / NF, f = lane - (lane / NF) * NF;
      if (e0 + e < a.K) {
        nbv = __ldg(a.nbr + (size_t)(e0 + e) * NF + f);
        codev = __ldg(a.fcode + e0 + e);
      }
    }
    double vP[ITEMS][D], vM[ITEMS][D], dnv[ITEMS];
    int nbi[ITEMS];
#pragma unroll
    for (int u = 0; u < ITEMS; ++u) {
      const int it = lane + 32 * u;
      const int e = min(it / NFN, E - 1), m = it - (it / NFN) * NFN, f = m / NFP, k = m - f * NFP;
      const bool act = it < E * NFN && e0 + e < a.K;
      const int nb = __shfl_sync(0xffffffffu, nbv, e * NF + f);
      const uint32_t code = __shfl_sync(0xffffffffu, codev, e * NF + f);
      nbi[u] = act ? nb : -1;
      dnv[u] = 0.0;
#pragma unroll
      for (int d = 0; d < D; ++d) vP[u][d] = vM[u][d] = 0.0;
      if (act) {
        const int el = e0 + e;
        if (nb >= 0) {
          const int cf = (code >> (8 * f)) & 0xff;
          const int fr = cf & 3, sg = cf >> 2;
          const int nn = fmask[fr * NFP + npos[sg * NFP + k]], o = fmask[f * NFP + k];
#pragma unroll
          for (int d = 0; d < D; ++d) {
            vP[u][d] = __ldg(a.velT + d * n + (size_t)nb * NP + nn);
            vM[u][d] = __ldg(a.velT + d * n + (size_t)el * NP + o);
          }
        }
        const size_t fi = (size_t)el * NF * NFP + m;
        dnv[u] = (a.dPdN ? a.b0 * a.dPdN[fi] : 0.0) + (a.dPdN_old ? a.b1 * a.dPdN_old[fi] : 0.0);
      }
    }
#pragma unroll
    for (int u = 0; u < ITEMS; ++u) {
      const int it = lane + 32 * u;
      if (it >= E * NFN) continue;
      const int e = it / NFN, m = it - e * NFN, f = m / NFP, k = m - f * NFP;
      double un = 0.0;
      if (nbi[u] >= 0) {
#pragma unroll
        for (int ee = 0; ee < E; ++ee) {
          if (ee != e) continue;
#pragma unroll
          for (int d = 0; d < D; ++d) {
            double v;  // fscale n_d of face f (the unnormalised outward normal)
            if (D == 3)
              v = f == 0 ? -G[ee][2][d] : f == 1 ? -G[ee][1][d] : f == 2 ? (G[ee][0][d] + G[ee][1][d]) + G[ee][2][d]
                                                                           : -G[ee][0][d];
            else
              v = f == 0 ? -G[ee][1][d] : f == 1 ? G[ee][0][d] + G[ee][1][d] : -G[ee][0][d];
            un += v * (0.5 * (vP[u][d] - vM[u][d]));
          }
        }
      }
      if (e0 + e < a.K && a.dPdN_old) a.dPdN_old[(size_t)(e0 + e) * NF * NFP + m] = dnv[u];
      sF1[(e * NF + f) * NFPE + k] = un;
      sF2[(e * NF + f) * NFPE + k] = dnv[u];
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < NPL; ++u) {
      const int i = lane + 32 * u;
      if (i < NP) {
        double vol[E], l1[E], l2[E], y[E];
#pragma unroll
        for (int e = 0; e < E; ++e) vol[e] = l1[e] = l2[e] = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
          mat_vec<NP, NPE, E>(sD + k * MAT, sGU + k * NPE, D * NPE, i, y);
#pragma unroll
          for (int e = 0; e < E; ++e) vol[e] += y[e];
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          mat_vec<NP, NFPE, E>(sL + f * NP * NFPE, sF1 + f * NFPE, NF * NFPE, i, y);
#pragma unroll
          for (int e = 0; e < E; ++e) l1[e] += y[e];
          mat_vec<NP, NFPE, E>(sL + f * NP * NFPE, sF2 + f * NFPE, NF * NFPE, i, y);
#pragma unroll
          for (int e = 0; e < E; ++e) l2[e] += y[e];
        }
#pragma unroll
        for (int e = 0; e < E; ++e) sPre[e * NPE + i] = -(vol[e] + l1[e]) * inv_dt + l2[e];
      }
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < NPL; ++u) {
      const int i = lane + 32 * u;
      if (i < NP) {
        double y[E];
        mat_vec<NP, NPE, E>(sM, sPre, NPE, i, y);
#pragma unroll
        for (int e = 0; e < E; ++e)
          if (valid[e]) a.rhs[(size_t)(e0 + e) * NP + i] = J[e] * y[e];
      }
    }
  }
}

template <int D, int P>
__host__ __device__ constexpr int pr_rhs_smem_doubles() {
  return proj_blob_doubles<D, P>() +
         kProjWarps * proj_epw(D, P) * ((D + 1) * proj_npe(D, P) + 2 * (D + 1) * proj_nfpe(D, P));
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
  const int Nfpe0 = (ref.Nfp + 1) & ~1;
  std::vector<double> b((size_t)proj_nmat(dim) * MAT + (size_t)(dim + 1) * Np * Nfpe0, 0.0);  // pads stay zero
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
  const int Nf = dim + 1, Nfp = ref.Nfp, Nfpe = (Nfp + 1) & ~1;
  double* lift = b.data() + (size_t)proj_nmat(dim) * MAT;
  for (int f = 0; f < Nf; ++f)
    for (int i = 0; i < Np; ++i)
      for (int k = 0; k < Nfp; ++k)
        lift[(size_t)f * Np * Nfpe + ((size_t)(k / 2) * Np + i) * 2 + k % 2] = ref.LIFT[(size_t)i * Nf * Nfp + f * Nfp + k];
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

// Opt the kernel into its dynamic shared memory and return its resident CTAs per
// SM, once per (kernel, device): the attribute belongs to the current device.
template <typename Kern>
int kernel_setup(Kern kern, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> per_sm;  // (kernel, device)
  int dev = 0;
  SIPG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  int& n = per_sm[{reinterpret_cast<const void*>(kern), dev}];
  if (!n) {
    SIPG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int b = 0;
    SIPG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, kProjWarps * 32, smem));
    n = std::max(b, 1);
  }
  return n;
}

template <int D, int P, bool GRAD>
void launch_proj(const ProjArgs& a, cudaStream_t s) {
  constexpr size_t smem = proj_smem_doubles<D, P>() * sizeof(double);
  static_assert(smem <= 227 * 1024, "projection shared memory");
  auto kern = k_proj_cg<D, P, GRAD>;
  const int per_sm = kernel_setup(kern, smem);
  const int epc = kProjWarps * proj_epw(D, P);  // elements per CTA round
  const int need = (a.K + epc - 1) / epc;
  const int grid = std::max(1, std::min(need, per_sm * num_sms()));
  kern<<<grid, kProjWarps * 32, smem, s>>>(a);
  SIPG_CUDA(cudaGetLastError());
  note_launch();
}

// velTT from velT and either grad p (dp) or the pressure (pr, rho: GRAD).
void project_device(sipg_mesh* m, int order, double dt, double factor, const double* dp, const double* pr,
                    const double* rho, const double* velT, double* velTT, unsigned long long* stats,
                    cudaStream_t s) {
  const bool grad = pr != nullptr;
  if (!m || order < 1 || order > 4 || (!dp && !pr) || !velT || !velTT)
    throw Error(SIPG_INVALID_ARG, "project_velocity: null mesh/array or order outside 1..4");
  if (!std::isfinite(dt) || !std::isfinite(factor)) throw Error(SIPG_INVALID_ARG, "project_velocity: dt/factor");
  if (velTT == velT || (dp && velTT == dp) || (pr && velTT == pr) || (rho && velTT == rho))
    throw Error(SIPG_INVALID_ARG, "project_velocity: velTT must not alias its inputs");
  ProjArgs a{};
  a.K = m->K;
  a.hK = proj_h_device(m);  // also uploads the mesh
  a.geof = m->geof64.as<double>();
  a.mats = proj_mats(m->dim, order).blob.as<double>();
  a.dt = dt;
  a.factor = factor;
  a.dp = dp;
  a.pr = pr;
  a.rho = rho;
  a.nbr = m->nbr.as<int>();
  a.fcode = m->fcode.as<uint32_t>();
  a.itab = dev_ref(m->dim, order).itab.as<int8_t>();
  a.velT = velT;
  a.velTT = velTT;
  a.stats = stats;
  if (stats) SIPG_CUDA(cudaMemsetAsync(stats, 0, 2 * sizeof(unsigned long long), s));
  if (m->K == 0) return;
#define SIPG_PROJ(D, P)                        \
  (grad ? launch_proj<D, P, true>(a, s) : launch_proj<D, P, false>(a, s))
  switch (m->dim * 10 + order) {
    case 21: SIPG_PROJ(2, 1); break;
    case 22: SIPG_PROJ(2, 2); break;
    case 23: SIPG_PROJ(2, 3); break;
    case 24: SIPG_PROJ(2, 4); break;
    case 31: SIPG_PROJ(3, 1); break;
    case 32: SIPG_PROJ(3, 2); break;
    case 33: SIPG_PROJ(3, 3); break;
    case 34: SIPG_PROJ(3, 4); break;
    default: throw Error(SIPG_INVALID_ARG, "project_velocity: dimension");
  }
#undef SIPG_PROJ
}

// The host-buffer variants: inputs and output through device copies kept on the
// mesh between calls (grown on demand), so a time step allocates nothing after
// its first call. nin input arrays of in_bytes[i] bytes.
void project_host(sipg_mesh* m, int order, double dt, double factor, const double* dp, const double* pr,
                  const double* rho, const double* velT, double* velTT, double* stats) {
  if (!m || order < 1 || order > 4 || (!dp && !pr) || !velT || !velTT)
    throw Error(SIPG_INVALID_ARG, "project_velocity: null mesh/array or order outside 1..4");
  const size_t nv = (size_t)m->K * np_of(m->dim, order);
  const size_t vb = m->dim * nv * sizeof(double), sb = nv * sizeof(double);
  const size_t gb = pr ? sb : vb;  // grad p or pressure
  const size_t rb = rho ? sb : 0;
  std::lock_guard<std::mutex> lk(m->proj_mu);
  const size_t need = gb + rb + 2 * vb + 2 * sizeof(unsigned long long);
  if (m->proj_io.bytes < need) {
    m->proj_io = DevBuf();
    m->proj_io = DevBuf(need);
  }
  char* base = m->proj_io.as<char>();
  double* d_g = reinterpret_cast<double*>(base);
  double* d_r = rho ? reinterpret_cast<double*>(base + gb) : nullptr;
  double* d_v = reinterpret_cast<double*>(base + gb + rb);
  double* d_out = reinterpret_cast<double*>(base + gb + rb + vb);
  auto* d_st = reinterpret_cast<unsigned long long*>(base + gb + rb + 2 * vb);
  SIPG_CUDA(cudaMemcpy(d_g, pr ? pr : dp, gb, cudaMemcpyHostToDevice));
  if (rho) SIPG_CUDA(cudaMemcpy(d_r, rho, rb, cudaMemcpyHostToDevice));
  SIPG_CUDA(cudaMemcpy(d_v, velT, vb, cudaMemcpyHostToDevice));
  project_device(m, order, dt, factor, pr ? nullptr : d_g, pr ? d_g : nullptr, d_r, d_v, d_out, d_st, 0);
  unsigned long long st[2] = {0, 0};
  SIPG_CUDA(cudaMemcpy(velTT, d_out, vb, cudaMemcpyDeviceToHost));
  SIPG_CUDA(cudaMemcpy(st, d_st, sizeof(st), cudaMemcpyDeviceToHost));
  if (stats) {
    stats[0] = (double)m->K;
    stats[1] = (double)st[0];
    stats[2] = (double)st[1];
  }
}


template <int D, int P>
void launch_pr_rhs(const PrRhsArgs& a, cudaStream_t s) {
  constexpr size_t smem = pr_rhs_smem_doubles<D, P>() * sizeof(double);
  static_assert(smem <= 227 * 1024, "pressure rhs shared memory");
  auto kern = k_pr_rhs<D, P>;
  const int per_sm = kernel_setup(kern, smem);
  const int epc = kProjWarps * proj_epw(D, P);  // elements per CTA round
  const int need = (a.K + epc - 1) / epc;
  const int grid = std::max(1, std::min(need, per_sm * num_sms()));
  kern<<<grid, kProjWarps * 32, smem, s>>>(a);
  SIPG_CUDA(cudaGetLastError());
  note_launch();
}

void pressure_rhs_device(sipg_mesh* m, int order, double dt, double b0, double b1, const double* velT,
                         const double* dPdN, double* dPdN_old, double* rhs, cudaStream_t s) {
  if (!m || order < 1 || order > 4 || !velT || !rhs)
    throw Error(SIPG_INVALID_ARG, "pressure_rhs: null mesh/array or order outside 1..4");
  if (!std::isfinite(dt) || dt == 0.0 || !std::isfinite(b0) || !std::isfinite(b1))
    throw Error(SIPG_INVALID_ARG, "pressure_rhs: dt/b0/b1");
  if (rhs == velT || (dPdN_old && dPdN_old == dPdN)) throw Error(SIPG_INVALID_ARG, "pressure_rhs: aliasing");
  m->ensure_device();
  PrRhsArgs a{};
  a.K = m->K;
  a.geof = m->geof64.as<double>();
  a.mats = proj_mats(m->dim, order).blob.as<double>();
  a.dt = dt;
  a.b0 = b0;
  a.b1 = b1;
  a.nbr = m->nbr.as<int>();
  a.fcode = m->fcode.as<uint32_t>();
  a.itab = dev_ref(m->dim, order).itab.as<int8_t>();
  a.velT = velT;
  a.dPdN = dPdN;
  a.dPdN_old = dPdN_old;
  a.rhs = rhs;
  if (m->K == 0) return;
  switch (m->dim * 10 + order) {
    case 21: launch_pr_rhs<2, 1>(a, s); break;
    case 22: launch_pr_rhs<2, 2>(a, s); break;
    case 23: launch_pr_rhs<2, 3>(a, s); break;
    case 24: launch_pr_rhs<2, 4>(a, s); break;
    case 31: launch_pr_rhs<3, 1>(a, s); break;
    case 32: launch_pr_rhs<3, 2>(a, s); break;
    case 33: launch_pr_rhs<3, 3>(a, s); break;
    case 34: launch_pr_rhs<3, 4>(a, s); break;
    default: throw Error(SIPG_INVALID_ARG, "pressure_rhs: dimension");
  }
}

// Viscous right-hand side of the two-phase time step in one pass
// (MPINSSolver3D::viscosity, src/solvers/3d/mp_ins_solver.cpp:669-694:
// mp_ins_3d_vis_0 then mesh->mass on each component): per element
//   rhs_c = J M (fact0 rho u_c)  (c = 0 .. dim-1),   mm_factor = fact1 rho.
// A block takes 32 elements: their rho and velocity rows are staged with
// coalesced loads, thread (c, e) applies M (shared, broadcast reads) to one
// component of one element, and the rows go back coalesced.
template <int NP, int DIM>
__global__ void __launch_bounds__(96) k_vis_rhs(int K, const double* __restrict__ Mm, int ldm,
                                                 const double* __restrict__ geof, int ngeof, double fact0,
                                                 double fact1, const double* __restrict__ rho,
                                                 const double* __restrict__ vel, double* __restrict__ rhs,
                                                 double* __restrict__ mm) {
  constexpr int EB = 32;
  __shared__ double sM[NP * NP];
  __shared__ double sr[EB * NP];
  __shared__ double sv[3 * EB * NP];
  for (int i = threadIdx.x; i < NP * NP; i += blockDim.x) sM[i] = Mm[(i / NP) * ldm + i % NP];  // set-up data
  pdl_enter();
  for (int e0 = blockIdx.x * EB; e0 < K; e0 += gridDim.x * EB) {
    const int ne = min(EB, K - e0);
    __syncthreads();
    for (int i = threadIdx.x; i < ne * NP; i += blockDim.x) {
      const double r = rho[(size_t)e0 * NP + i];
      sr[i] = r;
      mm[(size_t)e0 * NP + i] = fact1 * r;
    }
    for (int c = 0; c < DIM; ++c)
      for (int i = threadIdx.x; i < ne * NP; i += blockDim.x)
        sv[c * EB * NP + i] = vel[((size_t)c * K + e0) * NP + i];
    __syncthreads();
    const int c = threadIdx.x / EB, el = threadIdx.x % EB;
    if (c < DIM && el < ne) {
      double w[NP];
      const double* ur = sv + c * EB * NP + el * NP;
      const double* rr = sr + el * NP;
#pragma unroll
      for (int j = 0; j < NP; ++j) w[j] = fact0 * rr[j] * ur[j];
      const double J = geof[(size_t)(e0 + el) * ngeof + ngeof - 1];
      double* out = sv + c * EB * NP + el * NP;  // each thread overwrites only its own row
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < NP; ++j) acc += sM[i * NP + j] * w[j];
        out[i] = J * acc;
      }
    }
    __syncthreads();
    for (int cc = 0; cc < DIM; ++cc)
      for (int i = threadIdx.x; i < ne * NP; i += blockDim.x)
        rhs[((size_t)cc * K + e0) * NP + i] = sv[cc * EB * NP + i];
  }
}

template <int DIM, int P>
void launch_vis_rhs(sipg_mesh* m, const double* Mm, int ldm, double fact0, double fact1, const double* rho,
                    const double* vel, double* rhs, double* mm, cudaStream_t s) {
  constexpr int NP = DIM == 2 ? (P + 1) * (P + 2) / 2 : (P + 1) * (P + 2) * (P + 3) / 6;
  const int grid = std::max(1, std::min((m->K + 31) / 32, 148 * 16));
  SIPG_CUDA(pdl_launch(k_vis_rhs<NP, DIM>, dim3(grid), dim3(96), 0, s, m->K, Mm, ldm, m->geof64.as<double>(),
                       DIM == 3 ? 10 : 5, fact0, fact1, rho, vel, rhs, mm));
  note_launch();
}

void viscous_rhs_device(sipg_mesh* m, int order, double fact0, double fact1, const double* rho, const double* vel,
                        double* rhs, double* mm, cudaStream_t s) {
  if (!m || order < 1 || order > 4 || !rho || !vel || !rhs || !mm)
    throw Error(SIPG_INVALID_ARG, "viscous_rhs: null mesh/array or order outside 1..4");
  if (!std::isfinite(fact0) || !std::isfinite(fact1)) throw Error(SIPG_INVALID_ARG, "viscous_rhs: factors");
  if (rhs == vel || mm == rho) throw Error(SIPG_INVALID_ARG, "viscous_rhs: aliasing");
  m->ensure_device();
  if (m->K == 0) return;
  const DevRef& dr = dev_ref(m->dim, order);
  const int Np = dr.Np, ld = Np | 1;
  const double* Mm = dr.c64.as<double>() + (size_t)m->dim * Np * ld;  // mass block of the constant blob
  switch (m->dim * 10 + order) {
    case 21: launch_vis_rhs<2, 1>(m, Mm, ld, fact0, fact1, rho, vel, rhs, mm, s); break;
    case 22: launch_vis_rhs<2, 2>(m, Mm, ld, fact0, fact1, rho, vel, rhs, mm, s); break;
    case 23: launch_vis_rhs<2, 3>(m, Mm, ld, fact0, fact1, rho, vel, rhs, mm, s); break;
    case 24: launch_vis_rhs<2, 4>(m, Mm, ld, fact0, fact1, rho, vel, rhs, mm, s); break;
    case 31: launch_vis_rhs<3, 1>(m, Mm, ld, fact0, fact1, rho, vel, rhs, mm, s); break;
    case 32: launch_vis_rhs<3, 2>(m, Mm, ld, fact0, fact1, rho, vel, rhs, mm, s); break;
    case 33: launch_vis_rhs<3, 3>(m, Mm, ld, fact0, fact1, rho, vel, rhs, mm, s); break;
    case 34: launch_vis_rhs<3, 4>(m, Mm, ld, fact0, fact1, rho, vel, rhs, mm, s); break;
    default: throw Error(SIPG_INVALID_ARG, "viscous_rhs: dimension");
  }
}

}  // namespace
}  // namespace sipg

using namespace sipg;

extern "C" int sipg_project_velocity(sipg_mesh* m, int order, double dt, double factor, const double* dp,
                                     const double* velT, double* velTT, unsigned long long* stats,
                                     void* stream) {
  return guarded([&] {
    if (!dp) throw Error(SIPG_INVALID_ARG, "project_velocity: null dp");
    project_device(m, order, dt, factor, dp, nullptr, nullptr, velT, velTT, stats, (cudaStream_t)stream);
  });
}

extern "C" int sipg_project_velocity_host(sipg_mesh* m, int order, double dt, double factor, const double* dp,
                                          const double* velT, double* velTT, double* stats) {
  return guarded([&] {
    if (!dp) throw Error(SIPG_INVALID_ARG, "project_velocity: null dp");
    project_host(m, order, dt, factor, dp, nullptr, nullptr, velT, velTT, stats);
  });
}

extern "C" int sipg_pressure_projection(sipg_mesh* m, int order, double dt, double factor, const double* pr,
                                        const double* rho, const double* velT, double* velTT,
                                        unsigned long long* stats, void* stream) {
  return guarded([&] {
    if (!pr) throw Error(SIPG_INVALID_ARG, "pressure_projection: null pr");
    project_device(m, order, dt, factor, nullptr, pr, rho, velT, velTT, stats, (cudaStream_t)stream);
  });
}

extern "C" int sipg_pressure_projection_host(sipg_mesh* m, int order, double dt, double factor, const double* pr,
                                             const double* rho, const double* velT, double* velTT, double* stats) {
  return guarded([&] {
    if (!pr) throw Error(SIPG_INVALID_ARG, "pressure_projection: null pr");
    project_host(m, order, dt, factor, nullptr, pr, rho, velT, velTT, stats);
  });
}

extern "C" int sipg_pressure_rhs(sipg_mesh* m, int order, double dt, double b0, double b1, const double* velT,
                                 const double* dPdN, double* dPdN_old, double* rhs, void* stream) {
  return guarded([&] { pressure_rhs_device(m, order, dt, b0, b1, velT, dPdN, dPdN_old, rhs, (cudaStream_t)stream); });
}

extern "C" int sipg_pressure_rhs_host(sipg_mesh* m, int order, double dt, double b0, double b1, const double* velT,
                                      const double* dPdN, double* dPdN_old, double* rhs) {
  return guarded([&] {
    if (!m || order < 1 || order > 4 || !velT || !rhs)
      throw Error(SIPG_INVALID_ARG, "pressure_rhs: null mesh/array or order outside 1..4");
    const int Np = np_of(m->dim, order), Nfp = m->dim == 2 ? order + 1 : (order + 1) * (order + 2) / 2;
    const size_t vb = (size_t)m->dim * m->K * Np * sizeof(double), sb = (size_t)m->K * Np * sizeof(double);
    const size_t fb = (size_t)m->K * (m->dim + 1) * Nfp * sizeof(double);
    std::lock_guard<std::mutex> lk(m->proj_mu);
    const size_t need = vb + sb + 2 * fb;
    if (m->proj_io.bytes < need) {
      m->proj_io = DevBuf();
      m->proj_io = DevBuf(need);
    }
    char* base = m->proj_io.as<char>();
    double* d_v = reinterpret_cast<double*>(base);
    double* d_rhs = reinterpret_cast<double*>(base + vb);
    double* d_n = dPdN ? reinterpret_cast<double*>(base + vb + sb) : nullptr;
    double* d_o = dPdN_old ? reinterpret_cast<double*>(base + vb + sb + fb) : nullptr;
    SIPG_CUDA(cudaMemcpy(d_v, velT, vb, cudaMemcpyHostToDevice));
    if (d_n) SIPG_CUDA(cudaMemcpy(d_n, dPdN, fb, cudaMemcpyHostToDevice));
    if (d_o) SIPG_CUDA(cudaMemcpy(d_o, dPdN_old, fb, cudaMemcpyHostToDevice));
    pressure_rhs_device(m, order, dt, b0, b1, d_v, d_n, d_o, d_rhs, 0);
    SIPG_CUDA(cudaMemcpy(rhs, d_rhs, sb, cudaMemcpyDeviceToHost));
    if (d_o) SIPG_CUDA(cudaMemcpy(dPdN_old, d_o, fb, cudaMemcpyDeviceToHost));
  });
}

extern "C" int sipg_viscous_rhs(sipg_mesh* m, int order, double fact0, double fact1, const double* rho,
                                const double* velTT, double* rhs, double* mm_factor, void* stream) {
  return guarded([&] { viscous_rhs_device(m, order, fact0, fact1, rho, velTT, rhs, mm_factor, (cudaStream_t)stream); });
}

extern "C" int sipg_viscous_rhs_host(sipg_mesh* m, int order, double fact0, double fact1, const double* rho,
                                     const double* velTT, double* rhs, double* mm_factor) {
  return guarded([&] {
    if (!m || order < 1 || order > 4 || !rho || !velTT || !rhs || !mm_factor)
      throw Error(SIPG_INVALID_ARG, "viscous_rhs: null mesh/array or order outside 1..4");
    const int Np = np_of(m->dim, order);
    const size_t sb = (size_t)m->K * Np * sizeof(double), vb = (size_t)m->dim * sb;
    std::lock_guard<std::mutex> lk(m->proj_mu);
    const size_t need = 2 * vb + 2 * sb;
    if (m->proj_io.bytes < need) {
      m->proj_io = DevBuf();
      m->proj_io = DevBuf(need);
    }
    char* base = m->proj_io.as<char>();
    double* d_v = reinterpret_cast<double*>(base);
    double* d_rhs = reinterpret_cast<double*>(base + vb);
    double* d_rho = reinterpret_cast<double*>(base + 2 * vb);
    double* d_mm = reinterpret_cast<double*>(base + 2 * vb + sb);
    SIPG_CUDA(cudaMemcpy(d_v, velTT, vb, cudaMemcpyHostToDevice));
    SIPG_CUDA(cudaMemcpy(d_rho, rho, sb, cudaMemcpyHostToDevice));
    viscous_rhs_device(m, order, fact0, fact1, d_rho, d_v, d_rhs, d_mm, 0);
    SIPG_CUDA(cudaMemcpy(rhs, d_rhs, vb, cudaMemcpyDeviceToHost));
    SIPG_CUDA(cudaMemcpy(mm_factor, d_mm, sb, cudaMemcpyDeviceToHost));
  });
}
