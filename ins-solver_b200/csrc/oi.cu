// Over-integrated operator: penalty, nodal projection of the factor and the
// element-row blocks from the cubature-point factor. See oi.hpp.
//
// The operator changes with the density at every time step, so it is assembled
// once per set_factor_oi into the block-sparse form of the low-order levels
// (self block and one block per face neighbour, FP64 and FP32) and applied as a
// block-sparse product, HBM-bound at (NF + 1) Np^2 values per element.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <memory>
#include <mutex>

#include "../../include/sipg_b200.h"
#include "bsr.cuh"
#include "capi_util.hpp"
#include "oi.hpp"
#include "runtime.hpp"
#include "sipg_apply.cuh"
#include "vecops.cuh"

namespace sipg {

struct OiDev {
  OiTables t;
  DevBuf vphi, vdphi, wq, ws, fphi, fdphi, xphi, xdphi, yphi, proj, mass;
};

namespace {

const OiDev& oi_dev(int dim, int order) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::unique_ptr<OiDev>> cache;
  int dev = 0;
  SIPG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  auto& slot = cache[{dev, dim * 10 + order}];
  if (slot) return *slot;
  auto d = std::make_unique<OiDev>();
  d->t = build_oi_tables(dim, order);
  auto up = [](DevBuf& b, const std::vector<double>& v) {
    b = DevBuf(std::max<size_t>(1, v.size()) * sizeof(double));
    if (!v.empty()) b.upload(v.data(), v.size() * sizeof(double));
  };
  up(d->vphi, d->t.vphi);
  up(d->vdphi, d->t.vdphi);
  up(d->wq, d->t.wq);
  up(d->ws, d->t.ws);
  up(d->fphi, d->t.fphi);
  up(d->fdphi, d->t.fdphi);
  up(d->xphi, d->t.xphi);
  up(d->xdphi, d->t.xdphi);
  up(d->yphi, d->t.yphi);
  up(d->proj, d->t.proj);
  up(d->mass, dev_ref(dim, order).ref.M);
  slot = std::move(d);
  return *slot;
}

struct OiArgs {
  const double *vdphi, *wq, *ws, *fphi, *fdphi, *xphi, *yphi, *mass;
  const double* geof;
  const int* nbr;
  const uint32_t* fcode;
  const uint8_t* bct;
  const double* fvol;   // K x nq
  const double* fsurf;  // K x NF x nqs
  const double* tau;    // K x NF
  int mm_mode;
  double mm_scalar;
  const double* mm;
  int K, nq, nqs, nperm;
  int pin_elem, pin_node;
  double* v;  // block values, layout of BsrOp
};

template <int DIM>
__device__ __forceinline__ double oi_J(const double* g) { return g[DIM == 3 ? 9 : 4]; }

// Penalty per element face from the surface-point factors of both sides:
// 2(p+1)(p+2) max(max_s fscale- f-_s, max_t fscale+ f+_t); boundary faces: own side.
template <int DIM>
__global__ void k_oi_tau(const double* __restrict__ geof, const int* __restrict__ nbr,
                         const uint32_t* __restrict__ fcode, const double* __restrict__ fsurf, int K, int nqs,
                         double c, double* __restrict__ tau64, float* __restrict__ tau32) {
  constexpr int NF = DIM + 1, NG = DIM == 3 ? 10 : 5;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < K * NF; i += gridDim.x * blockDim.x) {
    const int e = i / NF, f = i - (i / NF) * NF;
    const double* g = geof + (size_t)e * NG;
    double n[3], sJ;
    simplex_face_normal<DIM>(g, f, n, &sJ);
    const double fs = sJ / oi_J<DIM>(g);
    double m = 0.0;
    const double* fo = fsurf + ((size_t)e * NF + f) * nqs;
    for (int s = 0; s < nqs; ++s) m = fmax(m, fs * fo[s]);
    const int nb = nbr[i];
    if (nb >= 0) {
      const int gf = (fcode[e] >> (8 * f)) & 3;
      const double fsn = sJ / oi_J<DIM>(geof + (size_t)nb * NG);
      const double* fn = fsurf + ((size_t)nb * NF + gf) * nqs;
      for (int s = 0; s < nqs; ++s) m = fmax(m, fsn * fn[s]);
    }
    tau64[i] = c * m;
    tau32[i] = (float)(c * m);
  }
}

// Nodal factor = the L2 projection of the volume-point factor.
__global__ void k_oi_project(const double* __restrict__ proj, const double* __restrict__ fvol, int K, int Np,
                             int nq, double* __restrict__ f64, float* __restrict__ f32) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)K * Np;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t e = i / Np;
    const int r = (int)(i - e * Np);
    double s = 0.0;
    for (int q = 0; q < nq; ++q) s += proj[(size_t)r * nq + q] * fvol[e * nq + q];
    f64[i] = s;
    f32[i] = (float)s;
  }
}

constexpr int OI_THREADS = 128, OI_QC = 32;

// Element blocks, one CTA per element (grid-stride). Each thread owns the entries
// (i, j) = t, t + 128, ... of a block; the volume term runs over the cubature
// points in chunks of OI_QC whose physical gradients are staged in shared memory.
template <int DIM, int NP>
__global__ void __launch_bounds__(OI_THREADS) k_oi_blocks(OiArgs a) {
  constexpr int NF = DIM + 1, NG = DIM == 3 ? 10 : 5, NE = (NP * NP + OI_THREADS - 1) / OI_THREADS;
  extern __shared__ double sm[];
  const int nqs = a.nqs;
  double* Y = sm;                           // [DIM][OI_QC][NP]
  double* aq = Y + DIM * OI_QC * NP;        // [OI_QC]
  double* ph = aq + OI_QC;                  // [nqs][NP] own basis at own points
  double* dn = ph + nqs * NP;               // [nqs][NP] own normal derivative at own points
  double* ps = dn + nqs * NP;               // [nqs][NP] neighbour basis at own points
  double* dp = ps + nqs * NP;               // [nqs][NP] neighbour normal derivative at its points
  double* ch = dp + nqs * NP;               // [nqs][NP] own basis at the neighbour's points
  double* fm = ch + nqs * NP;               // [nqs] own factor x weight
  double* fp = fm + nqs;                    // [nqs] neighbour factor x weight
  double* g = fp + nqs;                     // [NG] own geometry
  double* gn = g + NG;                      // [NG] neighbour geometry
  const size_t K = (size_t)a.K;
  for (int e = blockIdx.x; e < a.K; e += gridDim.x) {
    __syncthreads();
    if (threadIdx.x < NG) g[threadIdx.x] = a.geof[(size_t)e * NG + threadIdx.x];
    __syncthreads();
    const double J = oi_J<DIM>(g);
    double acc[NE];
#pragma unroll
    for (int k = 0; k < NE; ++k) acc[k] = 0.0;
    // volume: sum_q w_q J f_q sum_d (dphi_i / dx_d)(dphi_j / dx_d)
    for (int q0 = 0; q0 < a.nq; q0 += OI_QC) {
      const int nc = min(OI_QC, a.nq - q0);
      for (int t = threadIdx.x; t < DIM * nc * NP; t += blockDim.x) {
        const int d = t / (nc * NP), qq = (t / NP) % nc, i = t % NP;
        double s = 0.0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) s += g[r * DIM + d] * a.vdphi[((size_t)r * a.nq + q0 + qq) * NP + i];
        Y[(d * OI_QC + qq) * NP + i] = s;
      }
      for (int qq = threadIdx.x; qq < nc; qq += blockDim.x)
        aq[qq] = a.wq[q0 + qq] * J * a.fvol[(size_t)e * a.nq + q0 + qq];
      __syncthreads();
#pragma unroll
      for (int k = 0; k < NE; ++k) {
        const int ent = threadIdx.x + k * OI_THREADS;
        if (ent >= NP * NP) break;
        const int i = ent / NP, j = ent % NP;
        double s = 0.0;
        for (int qq = 0; qq < nc; ++qq) {
          double t = 0.0;
#pragma unroll
          for (int d = 0; d < DIM; ++d) t += Y[(d * OI_QC + qq) * NP + i] * Y[(d * OI_QC + qq) * NP + j];
          s += aq[qq] * t;
        }
        acc[k] += s;
      }
      __syncthreads();
    }
    // faces
    for (int f = 0; f < NF; ++f) {
      const int nb = a.nbr[(size_t)e * NF + f];
      if (nb < 0 && a.bct[-nb - 1] != BC_DIRICHLET) continue;  // Neumann and (scalar) slip faces add nothing
      double n[3], sJ;
      simplex_face_normal<DIM>(g, f, n, &sJ);
      const double h = nb >= 0 ? 0.5 : 1.0, tau = a.tau[(size_t)e * NF + f];
      double cr[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int d = 0; d < DIM; ++d) cr[r] += n[d] * g[r * DIM + d];
      int gf = 0, sg = 0;
      if (nb >= 0) {
        const int code = (a.fcode[e] >> (8 * f)) & 0xff;
        gf = code & 3;
        sg = code >> 2;
        if (threadIdx.x < NG) gn[threadIdx.x] = a.geof[(size_t)nb * NG + threadIdx.x];
      }
      __syncthreads();
      double cn[3] = {0.0, 0.0, 0.0};
      if (nb >= 0)
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
          for (int d = 0; d < DIM; ++d) cn[r] += n[d] * gn[r * DIM + d];
      for (int t = threadIdx.x; t < nqs * NP; t += blockDim.x) {
        const int s = t / NP, i = t % NP;
        ph[t] = a.fphi[((size_t)f * nqs + s) * NP + i];
        double v = 0.0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) v += cr[r] * a.fdphi[(((size_t)f * 3 + r) * nqs + s) * NP + i];
        dn[t] = v;
        if (nb >= 0) {
          ps[t] = a.xphi[(((size_t)gf * a.nperm + sg) * nqs + s) * NP + i];
          double w = 0.0;
#pragma unroll
          for (int r = 0; r < DIM; ++r) w += cn[r] * a.fdphi[(((size_t)gf * 3 + r) * nqs + s) * NP + i];
          dp[t] = w;
          ch[t] = a.yphi[(((size_t)f * a.nperm + sg) * nqs + s) * NP + i];
        }
      }
      for (int s = threadIdx.x; s < nqs; s += blockDim.x) {
        fm[s] = a.ws[s] * a.fsurf[((size_t)e * NF + f) * nqs + s];
        if (nb >= 0) fp[s] = a.ws[s] * a.fsurf[((size_t)nb * NF + gf) * nqs + s];
      }
      __syncthreads();
      // self: sJ sum_s [-h f- (dn_j phi_i + dn_i phi_j) + h tau phi_i phi_j]
#pragma unroll
      for (int k = 0; k < NE; ++k) {
        const int ent = threadIdx.x + k * OI_THREADS;
        if (ent >= NP * NP) break;
        const int i = ent / NP, j = ent % NP;
        double s1 = 0.0;
        for (int s = 0; s < nqs; ++s) {
          const double pi = ph[s * NP + i], pj = ph[s * NP + j];
          s1 += -h * fm[s] * (dn[s * NP + j] * pi + dn[s * NP + i] * pj) + h * tau * a.ws[s] * pi * pj;
        }
        acc[k] += sJ * s1;
      }
      if (nb >= 0) {
        // neighbour: sJ [sum_s (f- dn_i psi_j - tau phi_i psi_j) / 2 - sum_t f+_t dn+_j(t) chi_i(t) / 2]
        for (int ent = threadIdx.x; ent < NP * NP; ent += blockDim.x) {
          const int i = ent / NP, j = ent % NP;
          double s1 = 0.0, s2 = 0.0;
          for (int s = 0; s < nqs; ++s) {
            s1 += (fm[s] * dn[s * NP + i] - tau * a.ws[s] * ph[s * NP + i]) * ps[s * NP + j];
            s2 += fp[s] * dp[s * NP + j] * ch[s * NP + i];
          }
          double val = 0.5 * sJ * (s1 - s2);
          if ((nb == a.pin_elem && j == a.pin_node) || (e == a.pin_elem && i == a.pin_node)) val = 0.0;
          a.v[((size_t)((1 + f) * NP + i) * NP + j) * K + e] = val;
        }
      }
      __syncthreads();
    }
    for (int f = 0; f < NF; ++f)
      if (a.nbr[(size_t)e * NF + f] < 0)
        for (int ent = threadIdx.x; ent < NP * NP; ent += blockDim.x)
          a.v[((size_t)((1 + f) * NP + ent / NP) * NP + ent % NP) * K + e] = 0.0;
#pragma unroll
    for (int k = 0; k < NE; ++k) {
      const int ent = threadIdx.x + k * OI_THREADS;
      if (ent >= NP * NP) break;
      const int i = ent / NP, j = ent % NP;
      double val = acc[k];
      if (a.mm_mode != MM_NONE)
        val += J * a.mass[i * NP + j] * (a.mm_mode == MM_SCALAR ? a.mm_scalar : a.mm[(size_t)e * NP + j]);
      // the pinned DOF: column zero, its row keeps only its own diagonal
      if (e == a.pin_elem && (j == a.pin_node || i == a.pin_node) && i != j) val = 0.0;
      a.v[((size_t)i * NP + j) * K + e] = val;
    }
  }
}

size_t oi_smem(int dim, int Np, int nqs) {
  const int NG = dim == 3 ? 10 : 5;
  return (size_t)(dim * OI_QC * Np + OI_QC + 5 * nqs * Np + 2 * nqs + 2 * NG) * sizeof(double);
}

template <int DIM, int NP>
void launch_oi_blocks_t(const OiArgs& a, size_t smem, cudaStream_t s) {
  auto k = k_oi_blocks<DIM, NP>;
  SIPG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = std::max(1, std::min(a.K, num_sms() * 16));
  k<<<grid, OI_THREADS, smem, s>>>(a);
  note_launch();
  SIPG_CUDA(cudaGetLastError());
}

}  // namespace

void oi_sizes(int dim, int order, int* nq, int* nqs) {
  const OiDev& d = oi_dev(dim, order);
  if (nq) *nq = d.t.nq;
  if (nqs) *nqs = d.t.nqs;
}

// 1/rho of the level set at the volume and surface cubature points:
// LevelSetSolver3D::getRhoVolOI / getRhoSurfOI (src/solvers/3d/ls_solver.cpp:202-233:
// s interpolated to the points, then ls_3d_step_rho_vol_oi / ls_3d_step_surf_oi_1)
// followed by mp_ins_3d_pr_fact_oi_0/1 (1 / rho). The surface values come from the
// element's own polynomial, whose trace the reference interpolates from the face
// nodes. One thread per point.
__global__ void k_oi_ls_factor(const double* __restrict__ vphi, const double* __restrict__ fphi,
                               const double* __restrict__ s, int K, int Np, int nq, int nfq, double alpha,
                               double rho0, double rho1, double* __restrict__ fvol, double* __restrict__ fsurf) {
  const size_t nv = (size_t)K * nq, ns = (size_t)K * nfq;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nv + ns; i += (size_t)gridDim.x * blockDim.x) {
    const bool vol = i < nv;
    const size_t j = vol ? i : i - nv;
    const int per = vol ? nq : nfq;
    const size_t e = j / per;
    const int q = (int)(j - e * per);
    const double* phi = (vol ? vphi : fphi) + (size_t)q * Np;
    const double* se = s + e * Np;
    double sv = 0.0;
    for (int k = 0; k < Np; ++k) sv += phi[k] * se[k];
    const double step = tanh(3.141592653589793238463 * sv / alpha);
    const double rho = 0.5 * rho0 * (1.0 + step) + 0.5 * rho1 * (1.0 - step);
    (vol ? fvol : fsurf)[j] = 1.0 / rho;
  }
}

void set_factor_oi_level_set(sipg_op* op, const double* s, double alpha, double rho0, double rho1,
                             cudaStream_t st) {
  if (op->ncomp != 1) throw Error(SIPG_INVALID_ARG, "the over-integrated operator is scalar");
  sipg_mesh* m = op->mesh;
  const int K = m->K, NF = m->dim + 1;
  const OiDev& d = oi_dev(m->dim, op->order);
  const int nq = d.t.nq, nqs = d.t.nqs;
  ensure(op->oi_fvol, (size_t)K * nq * sizeof(double));
  ensure(op->oi_fsurf, (size_t)K * NF * nqs * sizeof(double));
  const size_t n = (size_t)K * (nq + NF * nqs);
  const int g = (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)num_sms() * 16));
  k_oi_ls_factor<<<g, 256, 0, st>>>(d.vphi.as<double>(), d.fphi.as<double>(), s, K, op->Np, nq, NF * nqs, alpha,
                                    rho0, rho1, op->oi_fvol.as<double>(), op->oi_fsurf.as<double>());
  note_launch();
  SIPG_CUDA(cudaGetLastError());
  ++op->version;
  oi_assemble(op, st);
}

// Set the operator's cubature-point factor (host or device pointers): penalty,
// nodal projection (the coarse levels' factor), element blocks FP64 and FP32.
void set_factor_oi_device(sipg_op* op, const double* fvol, const double* fsurf, cudaStream_t s) {
  if (op->ncomp != 1) throw Error(SIPG_INVALID_ARG, "the over-integrated operator is scalar");
  sipg_mesh* m = op->mesh;
  const int K = m->K, NF = m->dim + 1;
  const OiDev& d = oi_dev(m->dim, op->order);
  const int nq = d.t.nq, nqs = d.t.nqs;
  ensure(op->oi_fvol, (size_t)K * nq * sizeof(double));
  ensure(op->oi_fsurf, (size_t)K * NF * nqs * sizeof(double));
  SIPG_CUDA(cudaMemcpyAsync(op->oi_fvol.p, fvol, (size_t)K * nq * sizeof(double), cudaMemcpyDefault, s));
  SIPG_CUDA(cudaMemcpyAsync(op->oi_fsurf.p, fsurf, (size_t)K * NF * nqs * sizeof(double), cudaMemcpyDefault, s));
  oi_assemble(op, s);
}

// Penalty, nodal projection and blocks from the operator's stored cubature-point
// factor (again after its boundary types, mass term or pinned DOF change).
void oi_assemble(sipg_op* op, cudaStream_t s) {
  sipg_mesh* m = op->mesh;
  const int dim = m->dim, K = m->K, NF = dim + 1, Np = op->Np;
  const OiDev& d = oi_dev(dim, op->order);
  const int nq = d.t.nq, nqs = d.t.nqs;
  // nodal projection of the factor (set_factor of the reference's OI matrix)
  const size_t n = (size_t)K * Np;
  if (!op->factor64.p) {
    op->factor64 = DevBuf(n * sizeof(double));
    op->factor32 = DevBuf(n * sizeof(float));
  }
  const int g1 = (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16));
  k_oi_project<<<g1, 256, 0, s>>>(d.proj.as<double>(), op->oi_fvol.as<double>(), K, Np, nq,
                                  op->factor64.as<double>(), op->factor32.as<float>());
  note_launch();
  op->has_factor = true;
  const double c = 2.0 * (op->order + 1) * (op->order + 2);
  const int g2 = std::max(1, std::min((K * NF + 255) / 256, 148 * 16));
  if (dim == 3)
    k_oi_tau<3><<<g2, 256, 0, s>>>(m->geof64.as<double>(), m->nbr.as<int>(), m->fcode.as<uint32_t>(),
                                   op->oi_fsurf.as<double>(), K, nqs, c, op->tau64.as<double>(),
                                   op->tau32.as<float>());
  else
    k_oi_tau<2><<<g2, 256, 0, s>>>(m->geof64.as<double>(), m->nbr.as<int>(), m->fcode.as<uint32_t>(),
                                   op->oi_fsurf.as<double>(), K, nqs, c, op->tau64.as<double>(),
                                   op->tau32.as<float>());
  note_launch();
  if (!op->oi_blocks) op->oi_blocks = std::make_shared<BsrOp>();
  BsrOp& B = *op->oi_blocks;
  B.K = K;
  B.Np = Np;
  B.NF = NF;
  B.dim = dim;
  B.nbr = m->nbr.as<int>();
  const size_t nv = (size_t)(NF + 1) * Np * Np * K;
  ensure(B.v64, nv * sizeof(double));
  ensure(B.v32, nv * sizeof(float));
  OiArgs a;
  a.vdphi = d.vdphi.as<double>();
  a.wq = d.wq.as<double>();
  a.ws = d.ws.as<double>();
  a.fphi = d.fphi.as<double>();
  a.fdphi = d.fdphi.as<double>();
  a.xphi = d.xphi.as<double>();
  a.yphi = d.yphi.as<double>();
  a.mass = d.mass.as<double>();
  a.geof = m->geof64.as<double>();
  a.nbr = m->nbr.as<int>();
  a.fcode = m->fcode.as<uint32_t>();
  a.bct = op->bct.as<uint8_t>();
  a.fvol = op->oi_fvol.as<double>();
  a.fsurf = op->oi_fsurf.as<double>();
  a.tau = op->tau64.as<double>();
  a.mm_mode = op->mm_mode;
  a.mm_scalar = op->mm_scalar;
  a.mm = op->mm_mode == MM_NODAL ? op->mm64.as<double>() : nullptr;
  a.K = K;
  a.nq = nq;
  a.nqs = nqs;
  a.nperm = d.t.nperm;
  a.pin_elem = op->pin_elem;
  a.pin_node = op->pin_node;
  a.v = B.v64.as<double>();
  const size_t smem = oi_smem(dim, Np, nqs);
  switch (dim * 100 + Np) {
    case 203: launch_oi_blocks_t<2, 3>(a, smem, s); break;
    case 206: launch_oi_blocks_t<2, 6>(a, smem, s); break;
    case 210: launch_oi_blocks_t<2, 10>(a, smem, s); break;
    case 215: launch_oi_blocks_t<2, 15>(a, smem, s); break;
    case 304: launch_oi_blocks_t<3, 4>(a, smem, s); break;
    case 310: launch_oi_blocks_t<3, 10>(a, smem, s); break;
    case 320: launch_oi_blocks_t<3, 20>(a, smem, s); break;
    case 335: launch_oi_blocks_t<3, 35>(a, smem, s); break;
    default: throw Error(SIPG_INVALID_ARG, "over-integrated operator: unsupported element");
  }
  to_f32(B.v32.as<float>(), B.v64.as<double>(), nv, s);
  op->oi = true;
}

}  // namespace sipg

using namespace sipg;

extern "C" {

int sipg_op_oi_sizes(const sipg_op* op, int* nq, int* nqs) {
  return guarded([&] {
    if (!op) throw Error(SIPG_INVALID_ARG, "null op");
    oi_sizes(op->mesh->dim, op->order, nq, nqs);
  });
}

int sipg_op_oi_points_host(sipg_op* op, double* xyz_vol, double* xyz_surf) {
  return guarded([&] {
    if (!op) throw Error(SIPG_INVALID_ARG, "null op");
    sipg_mesh* m = op->mesh;
    const int dim = m->dim, K = m->K, NF = dim + 1, nv = dim + 1;
    const OiDev& d = oi_dev(dim, op->order);
    const int nq = d.t.nq, nqs = d.t.nqs;
    // affine map: x = sum_v bary_v(r, s, t) X_v with the element's vertices
    auto bary = [&](double r, double s, double t, double* b) {
      if (dim == 2) {
        b[0] = -(r + s) / 2; b[1] = (1 + r) / 2; b[2] = (1 + s) / 2;
      } else {
        b[0] = -(1 + r + s + t) / 2; b[1] = (1 + r) / 2; b[2] = (1 + s) / 2; b[3] = (1 + t) / 2;
      }
    };
    auto map = [&](int e, double r, double s, double t, double* x) {
      double b[4];
      bary(r, s, t, b);
      for (int c = 0; c < dim; ++c) {
        double v = 0.0;
        for (int k = 0; k < nv; ++k) v += b[k] * m->vx[(size_t)m->e2v[(size_t)e * nv + k] * dim + c];
        x[c] = v;
      }
    };
    double x[3];
    for (int e = 0; e < K; ++e) {
      if (xyz_vol)
        for (int q = 0; q < nq; ++q) {
          map(e, d.t.rq[q], d.t.sq[q], dim == 3 ? d.t.tq[q] : 0.0, x);
          for (int c = 0; c < dim; ++c) xyz_vol[((size_t)c * K + e) * nq + q] = x[c];
        }
      if (xyz_surf)
        for (int f = 0; f < NF; ++f)
          for (int q = 0; q < nqs; ++q) {
            map(e, d.t.fr[f * nqs + q], d.t.fs[f * nqs + q], d.t.ft[f * nqs + q], x);
            for (int c = 0; c < dim; ++c) xyz_surf[(((size_t)c * K + e) * NF + f) * nqs + q] = x[c];
          }
    }
  });
}

int sipg_op_set_factor_oi(sipg_op* op, const double* fvol, const double* fsurf) {
  return guarded([&] {
    if (!op || !fvol || !fsurf) throw Error(SIPG_INVALID_ARG, "set_factor_oi arguments");
    ++op->version;
    set_factor_oi_device(op, fvol, fsurf, 0);
    SIPG_CUDA(cudaDeviceSynchronize());
    op->refresh_pin(0);  // the nodal twin's pinned row (p-multigrid levels)
    SIPG_CUDA(cudaDeviceSynchronize());
  });
}

int sipg_op_set_factor_oi_device(sipg_op* op, const double* fvol, const double* fsurf, void* stream) {
  return guarded([&] {
    if (!op || !fvol || !fsurf) throw Error(SIPG_INVALID_ARG, "set_factor_oi arguments");
    ++op->version;
    set_factor_oi_device(op, fvol, fsurf, (cudaStream_t)stream);
  });
}

}  // extern "C"
