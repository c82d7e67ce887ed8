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

constexpr int OI_QC = 16;

// One warp assembles one element's blocks. Every block is a sum of outer products
// over cubature points,
//   volume        sum_{q,d} a_q Y_d[q][i] Y_d[q][j]       (Y_d = dphi/dx_d, a_q = w_q J f_q)
//   self, face    sum_s P[s][i] Q[s][j] + E[s][i] P[s][j]  (P = phi, E = -h sJ f- dn,
//                                                          Q = E + h sJ tau w P)
//   neighbour     sum_s U[s][i] PS[s][j] + CH[s][i] DM[s][j]
//                 (U = sJ (f- dn - tau w phi) / 2, PS = the neighbour's basis, CH = the own
//                  basis at the neighbour's points, DM = -sJ f+ dn+ / 2),
// i.e. a product L^T R of two (points x Np) factors. The element-dependent factors
// (Y, E, Q, U, DM) are staged per point chunk or face in the warp's shared area (columns
// padded with zeros to NB 8-wide tiles, rows SS apart); the pure basis tables (P, PS, CH)
// are read in place through the read-only cache, which keeps the shared area at 12 KB per
// warp for p = 3 (four CTAs of four warps per SM). The warp multiplies them on the FP64
// tensor cores: one m8n8k4 MMA per (8 x 8 tile of the block, 4 points), A = L^T and B = R
// read straight from the rows (lane (g, t) reads row t, column g), accumulators in
// registers.
template <int NP>
struct OiTile {
  static constexpr int NB = (NP + 7) / 8;  // 8-wide tiles per block side
  static constexpr int S8 = NB * 8;        // staged columns (zeros beyond Np)
  // row stride = 8 (mod 16) doubles: the four rows t of a fragment load fall in
  // two distinct halves of the banks, two wavefronts per 32 x 8-byte load
  static constexpr int SS = S8 % 16 == 0 ? S8 + 8 : S8;
  static constexpr int W = NP > 20 ? 2 : 4;  // warps per CTA
};

// acc[bi][bj] += (L^T R) tile (bi, bj) over rows 0..nk-1 of L and R (row k of L scaled by
// w[k] when w is given). Lane (g = lane / 4, t = lane % 4) holds entries (8 bi + g,
// 8 bj + 2t) and (8 bi + g, 8 bj + 2t + 1). A staged operand has rows SS apart and zeros
// beyond Np; a table operand (LT / RT: a basis table in global memory, rows Np apart)
// is read through the read-only cache with the columns beyond Np masked.
template <int NP, bool LT = false, bool RT = false>
__device__ __forceinline__ void oi_mma(double (&acc)[OiTile<NP>::NB][OiTile<NP>::NB][2], const double* L,
                                       const double* R, const double* w, int nk, int lane) {
  constexpr int NB = OiTile<NP>::NB, SS = OiTile<NP>::SS;
  constexpr int LL = LT ? NP : SS, LR = RT ? NP : SS;
  const int g = lane >> 2, t = lane & 3;
  for (int k0 = 0; k0 < nk; k0 += 4) {
    const int k = k0 + t;
    const bool ok = k < nk;
    const int kc = ok ? k : nk - 1;  // rows past nk are never read
    const double ws = ok ? (w ? w[kc] : 1.0) : 0.0;
    double av[NB], bv[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const int c = b * 8 + g;
      const double l = LT ? (c < NP ? __ldg(L + kc * LL + c) : 0.0) : L[kc * LL + c];
      const double r = RT ? (c < NP ? __ldg(R + kc * LR + c) : 0.0) : R[kc * LR + c];
      av[b] = ok ? ws * l : 0.0;
      bv[b] = ok ? r : 0.0;
    }
#pragma unroll
    for (int bi = 0; bi < NB; ++bi)
#pragma unroll
      for (int bj = 0; bj < NB; ++bj)
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                     : "+d"(acc[bi][bj][0]), "+d"(acc[bi][bj][1])
                     : "d"(av[bi]), "d"(bv[bj]));
  }
}

template <int NP>
__device__ __forceinline__ void oi_zero(double (&acc)[OiTile<NP>::NB][OiTile<NP>::NB][2]) {
#pragma unroll
  for (int bi = 0; bi < OiTile<NP>::NB; ++bi)
#pragma unroll
    for (int bj = 0; bj < OiTile<NP>::NB; ++bj) acc[bi][bj][0] = acc[bi][bj][1] = 0.0;
}

// Writes this lane's entries (8 bi + lane / 4, 8 bj + 2 (lane % 4) + c) of block blk of
// element e: 0 the self block, 1 + f the neighbour block of face f. mode 0 writes the
// values, 1 a neighbour block with the pinned DOF's row and column zeroed, 2 the self
// block with the mass term added and the pinned DOF's off-diagonal entries zeroed.
template <int NP>
__device__ __forceinline__ void oi_store(const OiArgs& a, const double (&c)[OiTile<NP>::NB][OiTile<NP>::NB][2],
                                         int blk, int e, int nb, int mode, double J, int lane) {
  constexpr int NB = OiTile<NP>::NB;
  const size_t K = (size_t)a.K;
  const int g8 = lane >> 2, t2 = 2 * (lane & 3);
#pragma unroll
  for (int bi = 0; bi < NB; ++bi)
#pragma unroll
    for (int bj = 0; bj < NB; ++bj)
#pragma unroll
      for (int cc = 0; cc < 2; ++cc) {
        const int i = bi * 8 + g8, j = bj * 8 + t2 + cc;
        if (i >= NP || j >= NP) continue;
        double v = c[bi][bj][cc];
        if (mode == 1 && ((nb == a.pin_elem && j == a.pin_node) || (e == a.pin_elem && i == a.pin_node))) v = 0.0;
        if (mode == 2) {
          if (a.mm_mode != MM_NONE)
            v += J * a.mass[i * NP + j] * (a.mm_mode == MM_SCALAR ? a.mm_scalar : a.mm[(size_t)e * NP + j]);
          // the pinned DOF: column zero, its row keeps only its own diagonal
          if (e == a.pin_elem && (j == a.pin_node || i == a.pin_node) && i != j) v = 0.0;
        }
        a.v[((size_t)(blk * NP + i) * NP + j) * K + e] = v;
      }
}

// doubles of one warp's shared area: a volume chunk (Y and its weights) or the four
// staged face arrays, whichever is larger (the basis P, the neighbour's basis PS and the
// own basis at the neighbour's points CH are table rows, read in place)
template <int DIM, int NP>
__host__ __device__ size_t oi_warp_doubles(int nqs) {
  constexpr int SS = OiTile<NP>::SS;
  const size_t vol = (size_t)OI_QC * DIM * SS + OI_QC * DIM;
  const size_t face = (size_t)4 * nqs * SS;
  return vol > face ? vol : face;
}

template <int DIM, int NP>
__global__ void __launch_bounds__(32 * OiTile<NP>::W, OiTile<NP>::W == 4 ? 4 : 1) k_oi_blocks(OiArgs a) {
  constexpr int NF = DIM + 1, NG = DIM == 3 ? 10 : 5, NB = OiTile<NP>::NB, S8 = OiTile<NP>::S8;
  constexpr int SS = OiTile<NP>::SS, W = OiTile<NP>::W;
  extern __shared__ __align__(16) double sm[];
  const int nqs = a.nqs, nq = a.nq;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* Z = sm + (size_t)warp * oi_warp_doubles<DIM, NP>(nqs);
  // volume chunk: Y[(q * DIM + d) * SS + i], weights wv[q * DIM + d]
  double* Y = Z;
  double* wv = Z + (size_t)OI_QC * DIM * SS;
  // face arrays, nqs x SS each
  double* E = Z;
  double* Q = E + nqs * SS;
  double* U = Q + nqs * SS;
  double* DM = U + nqs * SS;
  for (int e = blockIdx.x * W + warp; e < a.K; e += gridDim.x * W) {
    double g[NG];
#pragma unroll
    for (int k = 0; k < NG; ++k) g[k] = __ldg(a.geof + (size_t)e * NG + k);
    const double J = oi_J<DIM>(g);
    double acc[NB][NB][2];
    oi_zero<NP>(acc);
    // volume
    for (int q0 = 0; q0 < nq; q0 += OI_QC) {
      const int nc = min(OI_QC, nq - q0);
      __syncwarp();
      // each reference derivative is loaded once and serves the DIM physical ones
      for (int idx = lane; idx < nc * S8; idx += 32) {
        const int i = idx % S8, qq = idx / S8;
        double dr[DIM];
#pragma unroll
        for (int r = 0; r < DIM; ++r) dr[r] = i < NP ? __ldg(a.vdphi + ((size_t)r * nq + q0 + qq) * NP + i) : 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          double v = 0.0;
#pragma unroll
          for (int r = 0; r < DIM; ++r) v += g[r * DIM + d] * dr[r];
          Y[(qq * DIM + d) * SS + i] = v;
        }
      }
      for (int idx = lane; idx < nc * DIM; idx += 32) {
        const int qq = idx / DIM;
        wv[idx] = __ldg(a.wq + q0 + qq) * J * a.fvol[(size_t)e * nq + q0 + qq];
      }
      __syncwarp();
      oi_mma<NP>(acc, Y, Y, wv, nc * DIM, lane);
    }
    // faces
    for (int f = 0; f < NF; ++f) {
      const int nb = a.nbr[(size_t)e * NF + f];
      const bool dir = nb < 0 && a.bct[-nb - 1] == BC_DIRICHLET;
      if (nb < 0) {
        // no neighbour block on a boundary face
        double zero[NB][NB][2];
        oi_zero<NP>(zero);
        oi_store<NP>(a, zero, 1 + f, e, nb, 0, J, lane);
        if (!dir) continue;  // Neumann and (scalar) slip faces add nothing
      }
      double n[3], sJ;
      simplex_face_normal<DIM>(g, f, n, &sJ);
      const double h = nb >= 0 ? 0.5 : 1.0, tau = a.tau[(size_t)e * NF + f];
      double cr[3] = {0.0, 0.0, 0.0}, cn[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int d = 0; d < DIM; ++d) cr[r] += n[d] * g[r * DIM + d];
      int gf = 0, sg = 0;
      if (nb >= 0) {
        const int code = (a.fcode[e] >> (8 * f)) & 0xff;
        gf = code & 3;
        sg = code >> 2;
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
          for (int d = 0; d < DIM; ++d) cn[r] += n[d] * __ldg(a.geof + (size_t)nb * NG + r * DIM + d);
      }
      __syncwarp();
      for (int idx = lane; idx < nqs * S8; idx += 32) {
        const int sq = idx / S8, i = idx % S8, o = sq * SS + i;
        double ph = 0.0, dn = 0.0, dp = 0.0;
        if (i < NP) {
          ph = __ldg(a.fphi + ((size_t)f * nqs + sq) * NP + i);
#pragma unroll
          for (int r = 0; r < DIM; ++r) dn += cr[r] * __ldg(a.fdphi + (((size_t)f * 3 + r) * nqs + sq) * NP + i);
          if (nb >= 0) {
#pragma unroll
            for (int r = 0; r < DIM; ++r) dp += cn[r] * __ldg(a.fdphi + (((size_t)gf * 3 + r) * nqs + sq) * NP + i);
          }
        }
        const double ws = __ldg(a.ws + sq);
        const double fm = ws * a.fsurf[((size_t)e * NF + f) * nqs + sq];
        const double ev = -h * sJ * fm * dn;
        E[o] = ev;
        Q[o] = ev + h * sJ * tau * ws * ph;
        if (nb >= 0) {
          const double fp = ws * a.fsurf[((size_t)nb * NF + gf) * nqs + sq];
          U[o] = 0.5 * sJ * (fm * dn - tau * ws * ph);
          DM[o] = -0.5 * sJ * fp * dp;
        }
      }
      __syncwarp();
      const double* P = a.fphi + (size_t)f * nqs * NP;
      oi_mma<NP, true, false>(acc, P, Q, nullptr, nqs, lane);
      oi_mma<NP, false, true>(acc, E, P, nullptr, nqs, lane);
      if (nb >= 0) {
        double nacc[NB][NB][2];
        oi_zero<NP>(nacc);
        oi_mma<NP, false, true>(nacc, U, a.xphi + ((size_t)gf * a.nperm + sg) * nqs * NP, nullptr, nqs, lane);
        oi_mma<NP, true, false>(nacc, a.yphi + ((size_t)f * a.nperm + sg) * nqs * NP, DM, nullptr, nqs, lane);
        oi_store<NP>(a, nacc, 1 + f, e, nb, 1, J, lane);
      }
    }
    oi_store<NP>(a, acc, 0, e, -1, 2, J, lane);
  }
}

template <int DIM, int NP>
void launch_oi_blocks_t(const OiArgs& a, cudaStream_t s) {
  constexpr int W = OiTile<NP>::W;
  const size_t smem = (size_t)W * oi_warp_doubles<DIM, NP>(a.nqs) * sizeof(double);
  auto k = k_oi_blocks<DIM, NP>;
  SIPG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = std::max(1, std::min((a.K + W - 1) / W, num_sms() * 16));
  k<<<grid, 32 * W, smem, s>>>(a);
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
  switch (dim * 100 + Np) {
    case 203: launch_oi_blocks_t<2, 3>(a, s); break;
    case 206: launch_oi_blocks_t<2, 6>(a, s); break;
    case 210: launch_oi_blocks_t<2, 10>(a, s); break;
    case 215: launch_oi_blocks_t<2, 15>(a, s); break;
    case 304: launch_oi_blocks_t<3, 4>(a, s); break;
    case 310: launch_oi_blocks_t<3, 10>(a, s); break;
    case 320: launch_oi_blocks_t<3, 20>(a, s); break;
    case 335: launch_oi_blocks_t<3, 35>(a, s); break;
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
