// Steps of the 3D incompressible time step around the solves. Non-linear
// advection, fused into one kernel: INSSolverBase3D::advec_current_non_linear + advec_standard
// (src/solvers/3d/ins_solver_base.cpp:224-329, 451-480), i.e. the flux tensor
// u (x) u (ins_3d_advec_0), its strong-form divergence (mesh->div), the
// Lax-Friedrichs face fluxes (ins_3d_advec_1 interior, ins_3d_advec_2 boundary:
// no-slip, slip, natural outflow), their LIFT, and the extrapolated velocity
// (ins_3d_advec_3): velT = a0 u + a1 u_old - dt (b0 N + b1 N_old).
// One warp per element (lane = node / face node), FP64; the reference matrices
// D_r and LIFT sit in shared memory. The boundary kernel's wave speed is the
// floor of the largest |n . u| over the face (the reference stores it in an int,
// ins_3d_advec_2.h:44), kept here so the results are the reference's.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <memory>
#include <mutex>

#include "../../include/sipg_b200.h"
#include "capi_util.hpp"
#include "ins_step.cuh"
#include "runtime.hpp"
#include "sipg_apply.cuh"
#include "vecops.cuh"

namespace sipg {
namespace {

constexpr int kAdvWarps = 8;

struct AdvTables {
  DevBuf mats;  // Dr, Ds, Dt (Np x Np), LIFT (Np x Nf Nfp), row-major
  DevBuf weak;  // Drw, Dsw, Dtw = M^-1 D_r^T M (Np x Np), LIFT: the weak-form divergence
};

const AdvTables& adv_tables(int order) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::unique_ptr<AdvTables>> cache;
  int dev = 0;
  SIPG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  auto& slot = cache[{dev, order}];
  if (slot) return *slot;
  const RefElement& r = dev_ref(3, order).ref;
  std::vector<double> m;
  m.insert(m.end(), r.Dr.begin(), r.Dr.end());
  m.insert(m.end(), r.Ds.begin(), r.Ds.end());
  m.insert(m.end(), r.Dt.begin(), r.Dt.end());
  m.insert(m.end(), r.LIFT.begin(), r.LIFT.end());
  auto t = std::make_unique<AdvTables>();
  t->mats = DevBuf(m.size() * sizeof(double));
  t->mats.upload(m.data(), m.size() * sizeof(double));
  // weak derivatives: (M D_w f)_i = int d(phi_i)/dr f, i.e. D_w = M^-1 D^T M
  const int Np = r.Np;
  std::vector<double> w;
  for (const std::vector<double>* D : {&r.Dr, &r.Ds, &r.Dt}) {
    std::vector<double> DtM((size_t)Np * Np, 0.0), Dw((size_t)Np * Np, 0.0);
    for (int i = 0; i < Np; ++i)
      for (int k = 0; k < Np; ++k) {
        double acc = 0.0;
        for (int j = 0; j < Np; ++j) acc += (*D)[(size_t)j * Np + i] * r.M[(size_t)j * Np + k];
        DtM[(size_t)i * Np + k] = acc;
      }
    for (int i = 0; i < Np; ++i)
      for (int k = 0; k < Np; ++k) {
        double acc = 0.0;
        for (int j = 0; j < Np; ++j) acc += r.Minv[(size_t)i * Np + j] * DtM[(size_t)j * Np + k];
        Dw[(size_t)i * Np + k] = acc;
      }
    w.insert(w.end(), Dw.begin(), Dw.end());
  }
  w.insert(w.end(), r.LIFT.begin(), r.LIFT.end());
  t->weak = DevBuf(w.size() * sizeof(double));
  t->weak.upload(w.data(), w.size() * sizeof(double));
  slot = std::move(t);
  return *slot;
}

struct AdvArgs {
  const double* mats;
  const int8_t* itab;  // fmask, perm_pos
  const double* geof;
  const int* nbr;
  const uint32_t* fcode;
  const int* vel_bc;  // Kb: 0 no-slip, 1 slip, 2 natural outflow
  const double *u, *u_old, *N_old;
  double *N, *velT;
  double dt, a0, a1, b0, b1;
  double grav;  // body force -grav along y, added to N_y in the extrapolation only
  int K;
};

template <int P>
__global__ void __launch_bounds__(kAdvWarps * 32) k_advection(const AdvArgs a) {
  using Cf = Cfg<3, P>;
  constexpr int NP = Cf::NP, NFP = Cf::NFP, NF = 4, NFNFP = NF * NFP, NG = 10;
  extern __shared__ double sm[];
  const double* sD = sm;                       // 3 x NP x NP
  const double* sL = sm + 3 * NP * NP;         // NP x NFNFP
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sU = sm + 3 * NP * NP + NP * NFNFP + warp * (12 * NP + 4 * NFNFP);
  double* sH = sU + 3 * NP;    // [3][3][NP]: H[c][r] = sum_d G[r][d] u_c u_d
  double* sF = sH + 9 * NP;    // [3][NFNFP] face fluxes
  double* sS = sF + 3 * NFNFP; // [NFNFP] boundary wave speeds
  for (int i = threadIdx.x; i < 3 * NP * NP + NP * NFNFP; i += blockDim.x) sm[i] = a.mats[i];
  __syncthreads();
  const int8_t* fmask = a.itab;
  const int8_t* perm = a.itab + NF * NFP;
  const size_t n = (size_t)a.K * NP;
  for (int e = blockIdx.x * kAdvWarps + warp; e < a.K; e += gridDim.x * kAdvWarps) {
    double g[NG];
#pragma unroll
    for (int k = 0; k < NG; ++k) g[k] = __ldg(a.geof + (size_t)e * NG + k);
    __syncwarp();
    for (int i = lane; i < NP; i += 32) {
      double uc[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        uc[c] = a.u[c * n + (size_t)e * NP + i];
        sU[c * NP + i] = uc[c];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          double s = 0.0;
#pragma unroll
          for (int d = 0; d < 3; ++d) s += g[r * 3 + d] * (uc[c] * uc[d]);
          sH[(c * 3 + r) * NP + i] = s;
        }
    }
    __syncwarp();
    // face fluxes (ins_3d_advec_1 / ins_3d_advec_2)
    for (int m = lane; m < NFNFP; m += 32) {
      const int f = m / NFP, j = m - f * NFP;
      double nv[3], sJ;
      simplex_face_normal<3>(g, f, nv, &sJ);
      const double fs = sJ / g[9];
      const int o = fmask[f * NFP + j];
      const double uM[3] = {sU[o], sU[NP + o], sU[2 * NP + o]};
      const double lvel = nv[0] * uM[0] + nv[1] * uM[1] + nv[2] * uM[2];
      const int nb = __ldg(a.nbr + (size_t)e * NF + f);
      if (nb >= 0) {
        const int code = (__ldg(a.fcode + e) >> (8 * f)) & 0xff;
        const int gf = code & 3, sg = code >> 2;
        const int nn = fmask[gf * NFP + perm[sg * NFP + j]];
        double uP[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) uP[c] = a.u[c * n + (size_t)nb * NP + nn];
        double gn[NG], np_[3], sJn;
#pragma unroll
        for (int k = 0; k < NG; ++k) gn[k] = __ldg(a.geof + (size_t)nb * NG + k);
        simplex_face_normal<3>(gn, gf, np_, &sJn);
        const double rvel = np_[0] * uP[0] + np_[1] * uP[1] + np_[2] * uP[2];
        const double nuP = nv[0] * uP[0] + nv[1] * uP[1] + nv[2] * uP[2];
        const double lam = fmax(fabs(lvel), fabs(rvel));
#pragma unroll
        for (int c = 0; c < 3; ++c) sF[c * NFNFP + m] = 0.5 * fs * (-(uM[c] * lvel - uP[c] * nuP) - lam * (uP[c] - uM[c]));
        sS[m] = -1.0;
      } else {
        const int kind = __ldg(a.vel_bc + (-nb - 1));
        double uR[3];
        if (kind == 0) {
          uR[0] = uR[1] = uR[2] = 0.0;
        } else if (kind == 1) {
#pragma unroll
          for (int c = 0; c < 3; ++c) uR[c] = uM[c] - lvel * nv[c];
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c) uR[c] = uM[c];
        }
        const double rvel = nv[0] * uR[0] + nv[1] * uR[1] + nv[2] * uR[2];
        sS[m] = fmax(fabs(lvel), fabs(rvel));
#pragma unroll
        for (int c = 0; c < 3; ++c) sF[c * NFNFP + m] = 0.5 * fs * (-(uM[c] * lvel - uR[c] * rvel));  // + wave term below
      }
    }
    __syncwarp();
    // boundary wave term: - floor(max over the face of the speeds) (uR - uM)
    for (int m = lane; m < NFNFP; m += 32) {
      if (sS[m] < 0.0) continue;
      const int f = m / NFP, j = m - f * NFP;
      double mx = 0.0;
      for (int k = 0; k < NFP; ++k) mx = fmax(mx, sS[f * NFP + k]);
      const double lam = (double)(int)mx;
      if (lam == 0.0) continue;
      double nv[3], sJ;
      simplex_face_normal<3>(g, f, nv, &sJ);
      const double fs = sJ / g[9];
      const int o = fmask[f * NFP + j];
      const double uM[3] = {sU[o], sU[NP + o], sU[2 * NP + o]};
      const double lvel = nv[0] * uM[0] + nv[1] * uM[1] + nv[2] * uM[2];
      const int kind = __ldg(a.vel_bc + (-__ldg(a.nbr + (size_t)e * NF + f) - 1));
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double uR = kind == 0 ? 0.0 : kind == 1 ? uM[c] - lvel * nv[c] : uM[c];
        sF[c * NFNFP + m] += 0.5 * fs * (-lam * (uR - uM[c]));
      }
    }
    __syncwarp();
    // N = sum_r D_r H_r + LIFT flux, then velT
    for (int i = lane; i < NP; i += 32) {
      double Nc[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const double* Dr = sD + r * NP * NP + i * NP;
        for (int k = 0; k < NP; ++k) {
          const double dv = Dr[k];
#pragma unroll
          for (int c = 0; c < 3; ++c) Nc[c] += dv * sH[(c * 3 + r) * NP + k];
        }
      }
      const double* Li = sL + i * NFNFP;
      for (int k = 0; k < NFNFP; ++k) {
        const double lv = Li[k];
#pragma unroll
        for (int c = 0; c < 3; ++c) Nc[c] += lv * sF[c * NFNFP + k];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const size_t idx = c * n + (size_t)e * NP + i;
        a.N[idx] = Nc[c];
        const double gc = c == 1 ? a.grav : 0.0;
        a.velT[idx] =
            (a.a0 * sU[c * NP + i] + a.a1 * a.u_old[idx]) - a.dt * (a.b0 * (Nc[c] + gc) + a.b1 * (a.N_old[idx] + gc));
      }
    }
  }
}

struct PnArgs {
  const double* mats;  // Dr, Ds, Dt first
  const int8_t* itab;
  const double* geof;
  const int* nbr;
  const int* belems;
  int n_belem;
  const int* vel_bc;
  const double *u, *N, *mu, *rho;
  double* dPdN;  // K x 4 x Nfp, zeroed before
  double reynolds;
  double grav;  // body force -grav along y: -N_y becomes -(N_y + grav)
  int K;
};

// Curl-curl Neumann data of the multiphase pressure step
// (MPINSSolver3D::apply_pressure_neumann_bc, src/solvers/3d/mp_ins_solver.cpp:450-493):
// w = mu curl u (mesh->curl, mp_ins_3d_pr_mu), then on no-slip and slip walls
// (mp_ins_3d_pr_0) dPdN = fscale n . (-N - curl w / (Re rho)) at the face nodes. One
// warp per element that owns a boundary face; the curls are the element-local
// strong-form derivatives.
template <int P>
__global__ void __launch_bounds__(kAdvWarps * 32) k_pressure_neumann(const PnArgs a) {
  using Cf = Cfg<3, P>;
  constexpr int NP = Cf::NP, NFP = Cf::NFP, NF = 4, NG = 10;
  extern __shared__ double sm[];
  const double* sD = sm;  // 3 x NP x NP
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sU = sm + 3 * NP * NP + warp * 6 * NP;  // [3][NP] u
  double* sW = sU + 3 * NP;                       // [3][NP] mu curl u
  for (int i = threadIdx.x; i < 3 * NP * NP; i += blockDim.x) sm[i] = a.mats[i];
  __syncthreads();
  const int8_t* fmask = a.itab;
  const size_t n = (size_t)a.K * NP;
  for (int it = blockIdx.x * kAdvWarps + warp; it < a.n_belem; it += gridDim.x * kAdvWarps) {
    const int e = __ldg(a.belems + it);
    double g[NG];
#pragma unroll
    for (int k = 0; k < NG; ++k) g[k] = __ldg(a.geof + (size_t)e * NG + k);
    __syncwarp();
    for (int i = lane; i < 3 * NP; i += 32) sU[i] = a.u[(i / NP) * n + (size_t)e * NP + i % NP];
    __syncwarp();
    // w = mu curl u at every node
    for (int i = lane; i < NP; i += 32) {
      double gr[3][3];  // gr[c][d] = d u_c / dx_d
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double dr[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < NP; ++k) {
          const double uk = sU[c * NP + k];
#pragma unroll
          for (int r = 0; r < 3; ++r) dr[r] += sD[r * NP * NP + i * NP + k] * uk;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) gr[c][d] = g[d] * dr[0] + g[3 + d] * dr[1] + g[6 + d] * dr[2];
      }
      const double mu = a.mu[(size_t)e * NP + i];
      sW[0 * NP + i] = mu * (gr[2][1] - gr[1][2]);
      sW[1 * NP + i] = mu * (gr[0][2] - gr[2][0]);
      sW[2 * NP + i] = mu * (gr[1][0] - gr[0][1]);
    }
    __syncwarp();
    for (int m = lane; m < NF * NFP; m += 32) {
      const int f = m / NFP, j = m - f * NFP;
      const int nb = __ldg(a.nbr + (size_t)e * NF + f);
      if (nb >= 0) continue;
      const int kind = __ldg(a.vel_bc + (-nb - 1));
      if (kind != 0 && kind != 1) continue;  // natural outflow: no Neumann data
      const int i = fmask[f * NFP + j];
      double gr[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double dr[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < NP; ++k) {
          const double wk = sW[c * NP + k];
#pragma unroll
          for (int r = 0; r < 3; ++r) dr[r] += sD[r * NP * NP + i * NP + k] * wk;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) gr[c][d] = g[d] * dr[0] + g[3 + d] * dr[1] + g[6 + d] * dr[2];
      }
      const double c2[3] = {gr[2][1] - gr[1][2], gr[0][2] - gr[2][0], gr[1][0] - gr[0][1]};
      double nv[3], sJ;
      simplex_face_normal<3>(g, f, nv, &sJ);
      const double fs = sJ / g[9];
      const double rr = a.reynolds * a.rho[(size_t)e * NP + i];
      double s = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        s += nv[c] * (-(a.N[c * n + (size_t)e * NP + i] + (c == 1 ? a.grav : 0.0)) - c2[c] / rr);
      a.dPdN[((size_t)e * NF + f) * NFP + j] = fs * s;
    }
  }
}

template <int P>
void launch_pressure_neumann_t(const PnArgs& a, cudaStream_t s) {
  constexpr int NP = Cfg<3, P>::NP;
  const size_t smem = (size_t)(3 * NP * NP + kAdvWarps * 6 * NP) * sizeof(double);
  auto k = k_pressure_neumann<P>;
  SIPG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = std::max(1, std::min((a.n_belem + kAdvWarps - 1) / kAdvWarps, num_sms() * 8));
  k<<<grid, kAdvWarps * 32, smem, s>>>(a);
  note_launch();
  SIPG_CUDA(cudaGetLastError());
}

template <int P>
void launch_advection_t(const AdvArgs& a, cudaStream_t s) {
  using Cf = Cfg<3, P>;
  constexpr int NP = Cf::NP, NFNFP = 4 * Cf::NFP;
  const size_t smem = (size_t)(3 * NP * NP + NP * NFNFP + kAdvWarps * (12 * NP + 4 * NFNFP)) * sizeof(double);
  auto k = k_advection<P>;
  SIPG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = std::max(1, std::min((a.K + kAdvWarps - 1) / kAdvWarps, num_sms() * 8));
  k<<<grid, kAdvWarps * 32, smem, s>>>(a);
  note_launch();
  SIPG_CUDA(cudaGetLastError());
}

// Level-set advection, AdvectionSolver3D::step / rhs (src/solvers/3d/advection_solver.cpp:
// 24-120) with the level-set boundary kernel (LevelSetAdvectionSolver3D::bc_kernel,
// src/solvers/3d/ls_solver.cpp:34-51): one stage of the three-stage Runge-Kutta
// scheme per launch. The right-hand side of q is
//   div_weak(u q) - LIFT(flux)                               (mesh->div_weak, op2_gemv -1 LIFT)
// with the upwind flux of advec_3d_flux on interior faces,
//   fscale (n.u- (q- + q+) / 2 + |n.u-| (q- - q+) / 2),
// and fscale n.u- q- on no-slip, slip and outflow faces (ls_advec_3d_bc takes the
// exterior value from the interior there). The stage combinations are runge_kutta_0/1:
//   stage 0: rk0 = L(s),  q1 = s + dt rk0
//   stage 1: rk1 = L(q1), q2 = s + dt (rk0 + rk1) / 8   (the reference's 0.5 dt (rk0/4 + rk1/4))
//   stage 2: rk2 = L(q2), s += dt (rk0 / 6 + rk1 / 6 + 2 rk2 / 3)
// and the last stage also applies ls_step (rho, mu from the smoothed Heaviside
// tanh(pi s / alpha)), 1 / rho (the pressure factor) and max |u|^2 (the time-step
// bound of INSSolverBase3D::max_vel, ins_solver_base.cpp:1398-1407).
struct LsArgs {
  const double* weak;  // Drw, Dsw, Dtw, LIFT
  const int8_t* itab;
  const double* geof;
  const int* nbr;
  const uint32_t* fcode;
  const int* vel_bc;
  const double* q;  // stage input
  const double* u;  // velocity, 3 x K x Np
  double* s;        // level set at the start of the step; written by the last stage
  double *rk0, *rk1;
  double* q_out;
  double *rho, *mu, *rrho;
  unsigned long long* vmax;  // bits of the largest |u|^2 (non-negative doubles order as integers)
  double dt, alpha, rho0, rho1, mu0, mu1;
  int stage, K;
};

__device__ __forceinline__ void ls_props(const LsArgs& a, double sv, size_t idx) {
  const double step = tanh(3.141592653589793238463 * sv / a.alpha);
  const double rho = 0.5 * a.rho0 * (1.0 + step) + 0.5 * a.rho1 * (1.0 - step);
  a.rho[idx] = rho;
  a.mu[idx] = 0.5 * a.mu0 * (1.0 + step) + 0.5 * a.mu1 * (1.0 - step);
  a.rrho[idx] = 1.0 / rho;
}

template <int P>
__global__ void __launch_bounds__(kAdvWarps * 32) k_ls_stage(const LsArgs a) {
  using Cf = Cfg<3, P>;
  constexpr int NP = Cf::NP, NFP = Cf::NFP, NF = 4, NFNFP = NF * NFP, NG = 10;
  extern __shared__ double sm[];
  const double* sD = sm;                // 3 x NP x NP weak derivatives
  const double* sL = sm + 3 * NP * NP;  // NP x NFNFP
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sU = sm + 3 * NP * NP + NP * NFNFP + warp * (7 * NP + NFNFP);
  double* sQ = sU + 3 * NP;  // [NP]
  double* sH = sQ + NP;      // [3][NP]: H_r = q sum_d G[r][d] u_d
  double* sF = sH + 3 * NP;  // [NFNFP]
  for (int i = threadIdx.x; i < 3 * NP * NP + NP * NFNFP; i += blockDim.x) sm[i] = a.weak[i];
  __syncthreads();
  const int8_t* fmask = a.itab;
  const int8_t* perm = a.itab + NF * NFP;
  const size_t n = (size_t)a.K * NP;
  double vmax = 0.0;
  for (int e = blockIdx.x * kAdvWarps + warp; e < a.K; e += gridDim.x * kAdvWarps) {
    double g[NG];
#pragma unroll
    for (int k = 0; k < NG; ++k) g[k] = __ldg(a.geof + (size_t)e * NG + k);
    __syncwarp();
    for (int i = lane; i < NP; i += 32) {
      const double q = a.q[(size_t)e * NP + i];
      double uc[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        uc[c] = a.u[c * n + (size_t)e * NP + i];
        sU[c * NP + i] = uc[c];
      }
      sQ[i] = q;
#pragma unroll
      for (int r = 0; r < 3; ++r) sH[r * NP + i] = q * (g[r * 3] * uc[0] + g[r * 3 + 1] * uc[1] + g[r * 3 + 2] * uc[2]);
      vmax = fmax(vmax, uc[0] * uc[0] + uc[1] * uc[1] + uc[2] * uc[2]);
    }
    __syncwarp();
    for (int m = lane; m < NFNFP; m += 32) {
      const int f = m / NFP, j = m - f * NFP;
      double nv[3], sJ;
      simplex_face_normal<3>(g, f, nv, &sJ);
      const double fs = sJ / g[9];
      const int o = fmask[f * NFP + j];
      const double qM = sQ[o];
      const double un = nv[0] * sU[o] + nv[1] * sU[NP + o] + nv[2] * sU[2 * NP + o];
      const int nb = __ldg(a.nbr + (size_t)e * NF + f);
      double fl;
      if (nb >= 0) {
        const int code = (__ldg(a.fcode + e) >> (8 * f)) & 0xff;
        const int gf = code & 3, sg = code >> 2;
        const double qP = a.q[(size_t)nb * NP + fmask[gf * NFP + perm[sg * NFP + j]]];
        fl = un * (0.5 * (qM + qP)) + 0.5 * fabs(un) * (qM - qP);
      } else {
        fl = un * qM;
      }
      sF[m] = fs * fl;
    }
    __syncwarp();
    for (int i = lane; i < NP; i += 32) {
      double r = 0.0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double* Dw = sD + d * NP * NP + i * NP;
        const double* H = sH + d * NP;
        for (int k = 0; k < NP; ++k) r += Dw[k] * H[k];
      }
      const double* Li = sL + i * NFNFP;
      double lf = 0.0;
      for (int k = 0; k < NFNFP; ++k) lf += Li[k] * sF[k];
      r -= lf;
      const size_t idx = (size_t)e * NP + i;
      if (a.stage == 0) {
        a.rk0[idx] = r;
        a.q_out[idx] = a.s[idx] + a.dt * r;
      } else if (a.stage == 1) {
        a.rk1[idx] = r;
        a.q_out[idx] = a.s[idx] + 0.5 * a.dt * (a.rk0[idx] / 4.0 + r / 4.0);
      } else {
        const double sv = a.s[idx] + a.dt * (a.rk0[idx] / 6.0 + a.rk1[idx] / 6.0 + 2.0 * r / 3.0);
        a.s[idx] = sv;
        ls_props(a, sv, idx);
      }
    }
  }
  if (a.stage == 2 && a.vmax) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    if (lane == 0) atomicMax(a.vmax, (unsigned long long)__double_as_longlong(vmax));
  }
}

// ls_step and max |u|^2 alone (the initial fields).
__global__ void k_ls_props(const LsArgs a, size_t n) {
  double vmax = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    ls_props(a, a.s[i], i);
    const double u = a.u[i], v = a.u[n + i], w = a.u[2 * n + i];
    vmax = fmax(vmax, u * u + v * v + w * w);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if ((threadIdx.x & 31) == 0) atomicMax(a.vmax, (unsigned long long)__double_as_longlong(vmax));
}

template <int P>
void launch_ls_t(const LsArgs& a, cudaStream_t s) {
  using Cf = Cfg<3, P>;
  constexpr int NP = Cf::NP, NFNFP = 4 * Cf::NFP;
  const size_t smem = (size_t)(3 * NP * NP + NP * NFNFP + kAdvWarps * (7 * NP + NFNFP)) * sizeof(double);
  auto k = k_ls_stage<P>;
  SIPG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = std::max(1, std::min((a.K + kAdvWarps - 1) / kAdvWarps, num_sms() * 8));
  k<<<grid, kAdvWarps * 32, smem, s>>>(a);
  note_launch();
  SIPG_CUDA(cudaGetLastError());
}

LsArgs ls_args(sipg_mesh* m, int order, const LsFields& f) {
  m->ensure_device();
  LsArgs a{};
  a.weak = adv_tables(order).weak.as<double>();
  a.itab = dev_ref(3, order).itab.as<int8_t>();
  a.geof = m->geof64.as<double>();
  a.nbr = m->nbr.as<int>();
  a.fcode = m->fcode.as<uint32_t>();
  a.u = f.u;
  a.s = f.s;
  a.rk0 = f.rk0;
  a.rk1 = f.rk1;
  a.rho = f.rho;
  a.mu = f.mu;
  a.rrho = f.rrho;
  a.vmax = f.vmax;
  a.alpha = f.alpha;
  a.rho0 = f.rho0;
  a.rho1 = f.rho1;
  a.mu0 = f.mu0;
  a.mu1 = f.mu1;
  a.K = m->K;
  return a;
}

}  // namespace

void ls_step_device(sipg_mesh* m, int order, double dt, const LsFields& f, cudaStream_t s) {
  if (m->dim != 3) throw Error(SIPG_INVALID_ARG, "the level-set step is 3D");
  if (order < 1 || order > 4) throw Error(SIPG_INVALID_ARG, "order must be 1..4");
  LsArgs a = ls_args(m, order, f);
  a.dt = dt;
  if (f.vmax) SIPG_CUDA(cudaMemsetAsync(f.vmax, 0, sizeof(unsigned long long), s));
  const double* qin[3] = {f.s, f.qa, f.qb};
  double* qout[3] = {f.qa, f.qb, nullptr};
  for (int st = 0; st < 3; ++st) {
    a.stage = st;
    a.q = qin[st];
    a.q_out = qout[st];
    switch (order) {
      case 1: launch_ls_t<1>(a, s); break;
      case 2: launch_ls_t<2>(a, s); break;
      case 3: launch_ls_t<3>(a, s); break;
      default: launch_ls_t<4>(a, s); break;
    }
  }
}

void ls_props_device(sipg_mesh* m, int order, const LsFields& f, cudaStream_t s) {
  LsArgs a = ls_args(m, order, f);
  const size_t n = (size_t)m->K * np_of(3, order);
  SIPG_CUDA(cudaMemsetAsync(f.vmax, 0, sizeof(unsigned long long), s));
  const int grid = (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)num_sms() * 8));
  k_ls_props<<<grid, 256, 0, s>>>(a, n);
  note_launch();
  SIPG_CUDA(cudaGetLastError());
}

void pressure_neumann_device(sipg_mesh* m, int order, double reynolds, double grav, const double* u,
                             const double* N, const double* mu, const double* rho, const int* vel_bc, double* dPdN,
                             cudaStream_t s) {
  if (m->dim != 3) throw Error(SIPG_INVALID_ARG, "the pressure Neumann data are 3D");
  if (order < 1 || order > 4) throw Error(SIPG_INVALID_ARG, "order must be 1..4");
  m->ensure_device();
  const int Nfp = nfp_of(3, order);
  SIPG_CUDA(cudaMemsetAsync(dPdN, 0, (size_t)m->K * 4 * Nfp * sizeof(double), s));
  if (m->n_belem == 0) return;
  PnArgs a;
  a.mats = adv_tables(order).mats.as<double>();
  a.itab = dev_ref(3, order).itab.as<int8_t>();
  a.geof = m->geof64.as<double>();
  a.nbr = m->nbr.as<int>();
  a.belems = m->belems.as<int>();
  a.n_belem = m->n_belem;
  a.vel_bc = vel_bc;
  a.u = u;
  a.N = N;
  a.mu = mu;
  a.rho = rho;
  a.dPdN = dPdN;
  a.reynolds = reynolds;
  a.grav = grav;
  a.K = m->K;
  switch (order) {
    case 1: launch_pressure_neumann_t<1>(a, s); break;
    case 2: launch_pressure_neumann_t<2>(a, s); break;
    case 3: launch_pressure_neumann_t<3>(a, s); break;
    default: launch_pressure_neumann_t<4>(a, s); break;
  }
}

void advection_device(sipg_mesh* m, int order, double dt, double a0, double a1, double b0, double b1, double grav,
                      const double* u, const double* u_old, const double* N_old, const int* vel_bc, double* N,
                      double* velT, cudaStream_t s) {
  if (m->dim != 3) throw Error(SIPG_INVALID_ARG, "the advection step is 3D");
  if (order < 1 || order > 4) throw Error(SIPG_INVALID_ARG, "order must be 1..4");
  m->ensure_device();
  AdvArgs a;
  a.mats = adv_tables(order).mats.as<double>();
  a.itab = dev_ref(3, order).itab.as<int8_t>();
  a.geof = m->geof64.as<double>();
  a.nbr = m->nbr.as<int>();
  a.fcode = m->fcode.as<uint32_t>();
  a.vel_bc = vel_bc;
  a.u = u;
  a.u_old = u_old;
  a.N_old = N_old;
  a.N = N;
  a.velT = velT;
  a.dt = dt;
  a.a0 = a0;
  a.a1 = a1;
  a.b0 = b0;
  a.b1 = b1;
  a.grav = grav;
  a.K = m->K;
  switch (order) {
    case 1: launch_advection_t<1>(a, s); break;
    case 2: launch_advection_t<2>(a, s); break;
    case 3: launch_advection_t<3>(a, s); break;
    default: launch_advection_t<4>(a, s); break;
  }
}

}  // namespace sipg

using namespace sipg;

extern "C" {

int sipg_ins_advection(sipg_mesh* m, int order, double dt, double a0, double a1, double b0, double b1,
                       const double* vel, const double* vel_old, const double* N_old, const int* vel_bc, double* N,
                       double* velT, void* stream) {
  return guarded([&] {
    if (!m || !vel || !vel_old || !N_old || !vel_bc || !N || !velT) throw Error(SIPG_INVALID_ARG, "advection arguments");
    advection_device(m, order, dt, a0, a1, b0, b1, 0.0, vel, vel_old, N_old, vel_bc, N, velT, (cudaStream_t)stream);
  });
}

int sipg_ins_advection_host(sipg_mesh* m, int order, double dt, double a0, double a1, double b0, double b1,
                            const double* vel, const double* vel_old, const double* N_old, const int* vel_bc,
                            double* N, double* velT) {
  return guarded([&] {
    if (!m || !vel || !vel_old || !N_old || !vel_bc || !N || !velT) throw Error(SIPG_INVALID_ARG, "advection arguments");
    m->ensure_device();
    const size_t n = (size_t)3 * m->K * np_of(3, order), bytes = n * sizeof(double);
    DevBuf du(bytes), duo(bytes), dno(bytes), dn(bytes), dv(bytes), db(std::max<size_t>(1, m->Kb) * sizeof(int));
    du.upload(vel, bytes);
    duo.upload(vel_old, bytes);
    dno.upload(N_old, bytes);
    if (m->Kb) db.upload(vel_bc, m->Kb * sizeof(int));
    advection_device(m, order, dt, a0, a1, b0, b1, 0.0, du.as<double>(), duo.as<double>(), dno.as<double>(), db.as<int>(),
                     dn.as<double>(), dv.as<double>(), 0);
    SIPG_CUDA(cudaMemcpy(N, dn.p, bytes, cudaMemcpyDeviceToHost));
    SIPG_CUDA(cudaMemcpy(velT, dv.p, bytes, cudaMemcpyDeviceToHost));
  });
}

int sipg_ins_pressure_neumann(sipg_mesh* m, int order, double reynolds, const double* vel, const double* N,
                              const double* mu, const double* rho, const int* vel_bc, double* dPdN, void* stream) {
  return guarded([&] {
    if (!m || !vel || !N || !mu || !rho || !vel_bc || !dPdN || !(reynolds > 0.0))
      throw Error(SIPG_INVALID_ARG, "pressure Neumann data arguments");
    pressure_neumann_device(m, order, reynolds, 0.0, vel, N, mu, rho, vel_bc, dPdN, (cudaStream_t)stream);
  });
}

int sipg_ins_pressure_neumann_host(sipg_mesh* m, int order, double reynolds, const double* vel, const double* N,
                                   const double* mu, const double* rho, const int* vel_bc, double* dPdN) {
  return guarded([&] {
    if (!m || !vel || !N || !mu || !rho || !vel_bc || !dPdN || !(reynolds > 0.0))
      throw Error(SIPG_INVALID_ARG, "pressure Neumann data arguments");
    m->ensure_device();
    const int Np = np_of(3, order), Nfp = nfp_of(3, order);
    const size_t nv = (size_t)3 * m->K * Np * sizeof(double), ns = (size_t)m->K * Np * sizeof(double);
    const size_t nd = (size_t)m->K * 4 * Nfp * sizeof(double);
    DevBuf du(nv), dn(nv), dmu(ns), drho(ns), dd(nd), db(std::max<size_t>(1, m->Kb) * sizeof(int));
    du.upload(vel, nv);
    dn.upload(N, nv);
    dmu.upload(mu, ns);
    drho.upload(rho, ns);
    if (m->Kb) db.upload(vel_bc, m->Kb * sizeof(int));
    pressure_neumann_device(m, order, reynolds, 0.0, du.as<double>(), dn.as<double>(), dmu.as<double>(),
                            drho.as<double>(), db.as<int>(), dd.as<double>(), 0);
    SIPG_CUDA(cudaMemcpy(dPdN, dd.p, nd, cudaMemcpyDeviceToHost));
  });
}

}  // extern "C"
