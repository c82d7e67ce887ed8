// Element diagonal blocks, diagonals, block inverses and boundary lifting.
//
// Replaces FactorViscousMatrix3D::calc_diag / calc_inv_block_diag
// (src/solvers/3d/slip_matrix/factor_viscous_matrix.cpp:312-451: fvmf_3d_op1(_diag),
// fvmf_3d_op2_(block_)diag, fvmf_3d_mm_(block_)diag, fvmf_3d_bop_(block_)diag and
// the host Armadillo inverse at :423-450) and apply_bc (:47-68, fvmf_3d_apply_bc.h).
// One CTA builds one element's Np x Np block in shared memory, FP64 throughout;
// the inverse is Gauss-Jordan with partial pivoting in shared memory, so the
// reference's host round trip disappears.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "runtime.hpp"
#include "sipg_blocks.cuh"
#include "vecops.cuh"

namespace sipg {
namespace {

template <int DIM>
__device__ void face_normal_d(const double* g, int f, double n[3], double* sJ) {
  if (DIM == 3) {
    for (int d = 0; d < 3; ++d) {
      double v;
      if (f == 0) v = -g[6 + d];
      else if (f == 1) v = -g[3 + d];
      else if (f == 2) v = (g[d] + g[3 + d]) + g[6 + d];
      else v = -g[d];
      n[d] = v;
    }
    double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    n[0] /= len; n[1] /= len; n[2] /= len;
    *sJ = len * g[9];
  } else {
    for (int d = 0; d < 2; ++d) {
      double v;
      if (f == 0) v = -g[2 + d];
      else if (f == 1) v = g[d] + g[2 + d];
      else v = -g[d];
      n[d] = v;
    }
    n[2] = 0.0;
    double len = sqrt(n[0] * n[0] + n[1] * n[1]);
    n[0] /= len; n[1] /= len;
    *sJ = len * g[4];
  }
}

// One warp builds one element's block: the reference matrices (consts64 layout of
// the apply, Cfg: Dr, Ds, [Dt], M with row stride LD) and the face masses are staged
// once per CTA, each warp keeps its element's block B and two Np x Np work arrays,
// and only warp barriers separate the steps (lanes stride over the entries, each
// entry summed in the same order as a plain loop).
template <int P>
struct BlockWarps {
  static constexpr int W = P >= 4 ? 2 : 4;
};

template <int NP>
struct BlockTile {
  static constexpr int S = (NP + 3) / 4 * 4, NTI = S / 4, NT = NTI * NTI;
};

// Shared-memory layout of block_kernel in doubles, every part starting on an even
// index (16 bytes) for the tiles' double2 loads: the staged reference matrices and
// face masses, then per warp the block B, the staging area (LT, Xd, Ts) and fac, fcol, g.
__host__ __device__ constexpr size_t even_up(size_t n) { return (n + 1) / 2 * 2; }

template <int DIM, int P>
struct BlockSmem {
  using C = Cfg<DIM, P>;
  static constexpr size_t BASE = even_up((size_t)(DIM + 1) * C::NP * C::LD + (size_t)C::NF * C::NFP * C::NFP);
  static constexpr size_t OFF_LT = even_up((size_t)C::NP * C::NP);
  static constexpr size_t WARP = OFF_LT + 3 * (size_t)C::NP * BlockTile<C::NP>::S + even_up(2 * C::NP + C::NG);
};

template <int DIM, int P>
__host__ __device__ constexpr size_t block_smem_doubles() {
  return BlockSmem<DIM, P>::BASE + (size_t)BlockWarps<P>::W * BlockSmem<DIM, P>::WARP;
}

// acc (4 x 4 tile at rows i0, columns j0) = sum_k L[k][i] R[k][j], rows of stride S
template <int S>
__device__ __forceinline__ void block_outer(double (&acc)[16], const double* L, const double* R, int nk, int i0,
                                            int j0) {
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] = 0.0;
  for (int k = 0; k < nk; ++k) {
    const double2 l01 = *reinterpret_cast<const double2*>(L + k * S + i0);
    const double2 l23 = *reinterpret_cast<const double2*>(L + k * S + i0 + 2);
    const double2 r01 = *reinterpret_cast<const double2*>(R + k * S + j0);
    const double2 r23 = *reinterpret_cast<const double2*>(R + k * S + j0 + 2);
    const double l[4] = {l01.x, l01.y, l23.x, l23.y};
    const double r[4] = {r01.x, r01.y, r23.x, r23.y};
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a * 4 + b] = fma(l[a], r[b], acc[a * 4 + b]);
  }
}

template <int DIM, int P>
__global__ void __launch_bounds__(32 * BlockWarps<P>::W) block_kernel(BlockArgs a, const double* __restrict__ U) {
  using C = Cfg<DIM, P>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, LD = C::LD, NG = C::NG, NPP = NP * NP;
  constexpr int W = BlockWarps<P>::W;
  extern __shared__ __align__(16) double smb[];
  __shared__ int fm[NF * NFP];
  double* Dm = smb;                               // DIM x NP x LD
  double* Mm = Dm + DIM * NP * LD;                // NP x LD
  double* MF = Mm + NP * LD;                      // NF x NFP x NFP
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int S = BlockTile<NP>::S, NTI = BlockTile<NP>::NTI, NT = BlockTile<NP>::NT;
  using L = BlockSmem<DIM, P>;
  double* B = smb + L::BASE + (size_t)warp * L::WARP;
  double* LT = B + L::OFF_LT;  // NP x S: (J M F)^T
  double* Xd = LT + NP * S;  // NP x S: X_d
  double* Ts = Xd + NP * S;  // NP x S: T = J M F X_d
  // Np x Np work arrays of the face terms and of the reference's volume variants,
  // over the staging area (NP * S >= NPP)
  double* X = LT;
  double* T = Xd;
  double* fac = Ts + NP * S;
  double* fcol = fac + NP;
  double* g = fcol + NP;
  for (int i = threadIdx.x; i < (DIM + 1) * NP * LD; i += blockDim.x) Dm[i] = a.consts[C::OFF_D + i];
  for (int i = threadIdx.x; i < NF * NFP * NFP; i += blockDim.x) MF[i] = a.mf[i];
  for (int i = threadIdx.x; i < NF * NFP; i += blockDim.x) fm[i] = a.itab[i];
  __syncthreads();
  const int total = a.K * a.ncomp;
  for (int item = blockIdx.x * W + warp; item < total; item += gridDim.x * W) {
    const int e = item % a.K, c = item / a.K;
    __syncwarp();
    for (int i = lane; i < NG; i += 32) g[i] = a.geof[(size_t)e * NG + i];
    for (int i = lane; i < NP; i += 32) fac[i] = a.factor ? a.factor[(size_t)e * NP + i] : 1.0;
    for (int i = lane; i < NPP; i += 32) B[i] = 0.0;
    __syncwarp();
    const double J = g[DIM == 3 ? 9 : 4];
    if (a.mode == BLOCK_DIAG_ONLY && !a.ref_volume) {
      // the diagonal alone: J sum_l f_l sum_{r<=s} K_rs U_rs[i][l] for the volume, with
      // K = G G^T and U_rs[i][l] = E_r[i][l] D_s[l][i] (+ the (s, r) term for r < s),
      // E_r = D_r^T M; the face terms touch the face nodes only (MF is symmetric)
      constexpr int NQ = DIM * (DIM + 1) / 2;
      double Kq[NQ];
      {
        int q = 0;
        for (int r = 0; r < DIM; ++r)
          for (int s2 = r; s2 < DIM; ++s2, ++q) {
            double v = 0.0;
            for (int d = 0; d < DIM; ++d) v += g[r * DIM + d] * g[s2 * DIM + d];
            Kq[q] = v;
          }
      }
      double* out_base = a.out + (size_t)item * NP;
      for (int i = lane; i < NP; i += 32) {
        double dv = 0.0;
        for (int l = 0; l < NP; ++l) {
          double u = 0.0;
#pragma unroll
          for (int q = 0; q < NQ; ++q) u += Kq[q] * __ldg(U + ((size_t)q * NP + i) * NP + l);
          dv += fac[l] * u;
        }
        dv *= J;
        for (int f = 0; f < NF; ++f) {
          const int nb = a.nbr[(size_t)e * NF + f];
          double n[3], sJ;
          face_normal_d<DIM>(g, f, n, &sJ);
          double scale;
          if (nb >= 0) {
            scale = 0.5 * sJ;
          } else {
            const int b = -nb - 1;
            bool all_slip = a.ncomp == DIM;
            for (int k = 0; k < a.ncomp; ++k) all_slip = all_slip && a.bct[(size_t)k * a.Kb + b] == 2;
            if (all_slip) scale = sJ * n[c] * n[c];
            else if (a.bct[(size_t)c * a.Kb + b] == 0) scale = sJ;
            else continue;  // Neumann
          }
          int aa = -1;
          for (int k = 0; k < NFP; ++k)
            if (fm[f * NFP + k] == i) aa = k;
          if (aa < 0) continue;
          double rf[3] = {0.0, 0.0, 0.0};
          for (int rr = 0; rr < DIM; ++rr)
            for (int d = 0; d < DIM; ++d) rf[rr] += n[d] * g[rr * DIM + d];
          const double* mf = MF + f * NFP * NFP;
          double s1 = 0.0;
          for (int bb = 0; bb < NFP; ++bb) {
            const int jn = fm[f * NFP + bb];
            double xv = 0.0;
            for (int rr = 0; rr < DIM; ++rr) xv += rf[rr] * Dm[rr * NP * LD + jn * LD + i];
            s1 += mf[aa * NFP + bb] * (xv * fac[jn]);
          }
          dv -= 2.0 * scale * s1;
          dv += scale * a.tau[(size_t)e * NF + f] * mf[aa * NFP + aa];
        }
        if (a.mm_mode != 0) dv += J * Mm[i * LD + i] * (a.mm_mode == 1 ? a.mm_scalar : a.mm[(size_t)e * NP + i]);
        if (e == a.pin_elem && i == a.pin_node) dv = a.pin_scale;
        out_base[i] = dv;
      }
      continue;
    }
    // volume: sum_d J Dx_d^T M F Dx_d (fvmf_3d_op1.h / fvmf_3d_op1_diag.h); the operator's
    // form as outer products in 4 x 4 lane tiles, the reference's variants entry by entry
    if (!a.ref_volume) {
      for (int i = lane; i < NP * S; i += 32) {
        const int k = i / S, r = i % S;
        LT[i] = r < NP ? J * Mm[r * LD + k] * fac[k] : 0.0;
      }
      for (int d = 0; d < DIM; ++d) {
        for (int i = lane; i < NP * S; i += 32) {
          const int k = i / S, cc = i % S;
          double v = 0.0;
          if (cc < NP)
            for (int rr = 0; rr < DIM; ++rr) v += g[rr * DIM + d] * Dm[rr * NP * LD + k * LD + cc];
          Xd[i] = v;
        }
        __syncwarp();
        for (int t = lane; t < NT; t += 32) {
          const int i0 = 4 * (t / NTI), j0 = 4 * (t % NTI);
          double acc[16];
          block_outer<S>(acc, LT, Xd, NP, i0, j0);
#pragma unroll
          for (int aa = 0; aa < 4; ++aa)
#pragma unroll
            for (int bb = 0; bb < 4; ++bb)
              if (i0 + aa < NP) Ts[(i0 + aa) * S + j0 + bb] = acc[aa * 4 + bb];
        }
        __syncwarp();
        for (int t = lane; t < NT; t += 32) {
          const int i0 = 4 * (t / NTI), j0 = 4 * (t % NTI);
          double acc[16];
          block_outer<S>(acc, Xd, Ts, NP, i0, j0);
#pragma unroll
          for (int aa = 0; aa < 4; ++aa)
#pragma unroll
            for (int bb = 0; bb < 4; ++bb)
              if (i0 + aa < NP && j0 + bb < NP) B[(i0 + aa) * NP + j0 + bb] += acc[aa * 4 + bb];
        }
        __syncwarp();
      }
    }
    for (int d = 0; d < (a.ref_volume ? DIM : 0); ++d) {
      for (int i = lane; i < NPP; i += 32) {
        int r = i / NP, cc = i % NP;
        double s = 0.0;
        for (int rr = 0; rr < DIM; ++rr) s += g[rr * DIM + d] * Dm[rr * NP * LD + r * LD + cc];
        X[i] = s;
      }
      __syncwarp();
      for (int i = lane; i < NPP; i += 32) {
        int r = i / NP, cc = i % NP;
        double s = 0.0;
        if (a.ref_volume && DIM == 2) {
          for (int k = 0; k < NP; ++k) s += Mm[r * LD + k] * X[k * NP + cc];
          s *= fac[r];
        } else {
          for (int k = 0; k < NP; ++k) s += Mm[r * LD + k] * fac[k] * X[k * NP + cc];
        }
        T[i] = J * s;
      }
      __syncwarp();
      for (int i = lane; i < NPP; i += 32) {
        int r = i / NP, cc = i % NP;
        double s = 0.0;
        if (a.ref_volume && DIM == 3)
          for (int k = 0; k < NP; ++k) s += X[r * NP + k] * T[k * NP + cc];
        else
          for (int k = 0; k < NP; ++k) s += X[k * NP + r] * T[k * NP + cc];
        B[i] += s;
      }
      __syncwarp();
    }
    // faces (fvmf_3d_op2_block_diag.h, fvmf_3d_bop_block_diag.h)
    for (int f = 0; f < NF; ++f) {
      const int nb = a.nbr[(size_t)e * NF + f];
      double n[3], sJ;
      face_normal_d<DIM>(g, f, n, &sJ);
      double scale;
      if (nb >= 0) {
        scale = 0.5 * sJ;
      } else {
        const int b = -nb - 1;
        bool all_slip = a.ncomp == DIM;
        for (int k = 0; k < a.ncomp; ++k) all_slip = all_slip && a.bct[(size_t)k * a.Kb + b] == 2;
        if (all_slip) scale = sJ * n[c] * n[c];
        else if (a.bct[(size_t)c * a.Kb + b] == 0) scale = sJ;
        else continue;  // Neumann
      }
      const double gtau = a.tau[(size_t)e * NF + f];
      // X = D_n: X[i][j] = f_i sum_r (n . grad r) D_r[i][j]
      double rf[3] = {0.0, 0.0, 0.0};
      for (int rr = 0; rr < DIM; ++rr)
        for (int d = 0; d < DIM; ++d) rf[rr] += n[d] * g[rr * DIM + d];
      for (int i = lane; i < NPP; i += 32) {
        int r = i / NP, cc = i % NP;
        double s = 0.0;
        for (int rr = 0; rr < DIM; ++rr) s += rf[rr] * Dm[rr * NP * LD + r * LD + cc];
        X[i] = s * fac[r];
      }
      __syncwarp();
      const double* mf = MF + f * NFP * NFP;
      const int* fmf = fm + f * NFP;
      // rows on the face: -scale * (MF D_n)[a][j]; and the penalty on face-face entries
      for (int i = lane; i < NFP * NP; i += 32) {
        int aa = i / NP, j = i % NP;
        double s = 0.0;
        for (int bb = 0; bb < NFP; ++bb) s += mf[aa * NFP + bb] * X[fmf[bb] * NP + j];
        B[fmf[aa] * NP + j] -= scale * s;
      }
      __syncwarp();
      // columns on the face: -scale * (D_n^T MF)[i][b]
      for (int i = lane; i < NP * NFP; i += 32) {
        int r = i / NFP, bb = i % NFP;
        double s = 0.0;
        for (int aa = 0; aa < NFP; ++aa) s += X[fmf[aa] * NP + r] * mf[aa * NFP + bb];
        B[r * NP + fmf[bb]] -= scale * s;
      }
      __syncwarp();
      for (int i = lane; i < NFP * NFP; i += 32) {
        int aa = i / NFP, bb = i % NFP;
        B[fmf[aa] * NP + fmf[bb]] += scale * gtau * mf[i];
      }
      __syncwarp();
    }
    // mass term (fvmf_3d_mm_block_diag.h: the reference scales rows; the operator scales columns)
    if (a.mm_mode != 0) {
      for (int i = lane; i < NPP; i += 32) {
        int r = i / NP, cc = i % NP;
        int k = a.ref_volume ? r : cc;
        double mmv = a.mm_mode == 1 ? a.mm_scalar : a.mm[(size_t)e * NP + k];
        B[i] += J * Mm[r * LD + cc] * mmv;
      }
      __syncwarp();
    }
    if (e == a.pin_elem) {
      const int pn = a.pin_node;
      for (int i = lane; i < NP; i += 32) {
        if (i != pn) { B[pn * NP + i] = 0.0; B[i * NP + pn] = 0.0; }
      }
      __syncwarp();
      if (lane == 0) B[pn * NP + pn] = a.pin_scale;
      __syncwarp();
    }
    double* out_base = a.out + (size_t)item * (a.mode == BLOCK_DIAG_ONLY ? NP : NPP);
    if (a.mode == BLOCK_DIAG_ONLY) {
      for (int i = lane; i < NP; i += 32) out_base[i] = B[i * NP + i];
      continue;
    }
    if (a.mode == BLOCK_INVERSE) {
      // Gauss-Jordan with partial pivoting: B -> I, X -> B^-1
      for (int i = lane; i < NPP; i += 32) X[i] = (i / NP == i % NP) ? 1.0 : 0.0;
      __syncwarp();
      for (int col = 0; col < NP; ++col) {
        // pivot: the first row (from col down) of largest |B[r][col]|, as a serial scan picks it
        double best = -1.0;
        int p = NP;
        for (int r = col + lane; r < NP; r += 32) {
          const double v = fabs(B[r * NP + col]);
          if (v > best) { best = v; p = r; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double ob = __shfl_xor_sync(0xffffffffu, best, o);
          const int op = __shfl_xor_sync(0xffffffffu, p, o);
          if (ob > best || (ob == best && op < p)) { best = ob; p = op; }
        }
        if (p != col)
          for (int j = lane; j < NP; j += 32) {
            double t0 = B[col * NP + j]; B[col * NP + j] = B[p * NP + j]; B[p * NP + j] = t0;
            double t1 = X[col * NP + j]; X[col * NP + j] = X[p * NP + j]; X[p * NP + j] = t1;
          }
        __syncwarp();
        const double dinv = 1.0 / B[col * NP + col];
        __syncwarp();
        for (int j = lane; j < NP; j += 32) {
          B[col * NP + j] *= dinv;
          X[col * NP + j] *= dinv;
        }
        __syncwarp();
        for (int r = lane; r < NP; r += 32) fcol[r] = B[r * NP + col];
        __syncwarp();
        for (int i = lane; i < NPP; i += 32) {
          int r = i / NP, j = i % NP;
          if (r == col) continue;
          B[i] -= fcol[r] * B[col * NP + j];
          X[i] -= fcol[r] * X[col * NP + j];
        }
        __syncwarp();
      }
      for (int i = lane; i < NPP; i += 32) out_base[i] = X[i];
    } else {
      for (int i = lane; i < NPP; i += 32) out_base[i] = B[i];
    }
  }
}

// Boundary lifting of Dirichlet / Neumann data into the right-hand side
// (fvmf_3d_apply_bc.h:29-85), one CTA per element that owns boundary faces;
// an element's faces are applied in order, so the sums are deterministic.
template <int DIM, int P>
__global__ void __launch_bounds__(128) apply_bc_kernel(ApplyBcArgs a) {
  using C = Cfg<DIM, P>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, LD = C::LD, NG = C::NG, NPP = NP * NP;
  __shared__ double X[NPP], tmp[NP], g[NG], fac[NP], acc[NP];
  const double* Dm = a.consts + C::OFF_D;
  for (int item = blockIdx.x; item < a.n_belem * a.ncomp; item += gridDim.x) {
    const int e = a.belems[item % a.n_belem], c = item / a.n_belem;
    __syncthreads();
    for (int i = threadIdx.x; i < NG; i += blockDim.x) g[i] = a.geof[(size_t)e * NG + i];
    for (int i = threadIdx.x; i < NP; i += blockDim.x) {
      fac[i] = a.factor ? a.factor[(size_t)e * NP + i] : 1.0;
      acc[i] = 0.0;
    }
    __syncthreads();
    for (int f = 0; f < NF; ++f) {
      const int nb = a.nbr[(size_t)e * NF + f];
      if (nb >= 0) continue;
      const int b = -nb - 1;
      const int t = a.bct[(size_t)c * a.Kb + b];
      if (t != 0 && t != 1) continue;  // slip: nothing
      double n[3], sJ;
      face_normal_d<DIM>(g, f, n, &sJ);
      const double* mf = a.mf + f * NFP * NFP;
      const int8_t* fmf = a.itab + f * NFP;
      const double* bc = a.bc + ((size_t)c * a.Kb + b) * NFP;
      if (t == 1) {
        for (int i = threadIdx.x; i < NFP; i += blockDim.x) {
          double s = 0.0;
          for (int j = 0; j < NFP; ++j) s += mf[i * NFP + j] * bc[j];
          acc[fmf[i]] += sJ * s;
        }
        __syncthreads();
        continue;
      }
      const double gtau = a.tau[(size_t)e * NF + f];
      double rf[3] = {0.0, 0.0, 0.0};
      for (int rr = 0; rr < DIM; ++rr)
        for (int d = 0; d < DIM; ++d) rf[rr] += n[d] * g[rr * DIM + d];
      for (int i = threadIdx.x; i < NPP; i += blockDim.x) {
        int r = i / NP, cc = i % NP;
        double s = 0.0;
        for (int rr = 0; rr < DIM; ++rr) s += rf[rr] * Dm[rr * NP * LD + r * LD + cc];
        X[i] = s * fac[r];
      }
      for (int i = threadIdx.x; i < NP; i += blockDim.x) tmp[i] = 0.0;
      __syncthreads();
      for (int i = threadIdx.x; i < NFP; i += blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < NFP; ++j) s += mf[i * NFP + j] * bc[j];
        tmp[fmf[i]] = sJ * s;
      }
      __syncthreads();
      for (int i = threadIdx.x; i < NP; i += blockDim.x) {
        double s = gtau * tmp[i];
        for (int j = 0; j < NP; ++j) s -= X[j * NP + i] * tmp[j];
        acc[i] += s;
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < NP; i += blockDim.x) a.rhs[((size_t)c * a.K + e) * NP + i] += acc[i];
  }
}

}  // namespace

#define SIPG_DISPATCH_B(DIM_, ORDER_, ...)                         \
  switch ((DIM_) * 10 + (ORDER_)) {                                \
    case 21: { constexpr int D = 2, P = 1; __VA_ARGS__; }          \
    case 22: { constexpr int D = 2, P = 2; __VA_ARGS__; }          \
    case 23: { constexpr int D = 2, P = 3; __VA_ARGS__; }          \
    case 24: { constexpr int D = 2, P = 4; __VA_ARGS__; }          \
    case 31: { constexpr int D = 3, P = 1; __VA_ARGS__; }          \
    case 32: { constexpr int D = 3, P = 2; __VA_ARGS__; }          \
    case 33: { constexpr int D = 3, P = 3; __VA_ARGS__; }          \
    case 34: { constexpr int D = 3, P = 4; __VA_ARGS__; }          \
    default: break;                                                \
  }

// U_rs[i][l] = E_r[i][l] D_s[l][i] (+ E_s[i][l] D_r[l][i] for r < s), E_r = D_r^T M: the
// volume diagonal's tables, per order (pairs r <= s in order), cached per device
static const double* diag_tables(int dim, int order) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::unique_ptr<DevBuf>> cache;
  int dev = 0;
  SIPG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  auto& slot = cache[{dev, dim * 10 + order}];
  if (slot) return slot->as<double>();
  const RefElement& r = dev_ref(dim, order).ref;
  const int Np = r.Np;
  const std::vector<double>* D[3] = {&r.Dr, &r.Ds, &r.Dt};
  std::vector<std::vector<double>> E(dim, std::vector<double>((size_t)Np * Np, 0.0));
  for (int q = 0; q < dim; ++q)
    for (int i = 0; i < Np; ++i)
      for (int l = 0; l < Np; ++l) {
        double v = 0.0;
        for (int k = 0; k < Np; ++k) v += (*D[q])[(size_t)k * Np + i] * r.M[(size_t)k * Np + l];
        E[q][(size_t)i * Np + l] = v;
      }
  std::vector<double> U;
  for (int a = 0; a < dim; ++a)
    for (int b = a; b < dim; ++b)
      for (int i = 0; i < Np; ++i)
        for (int l = 0; l < Np; ++l) {
          double v = E[a][(size_t)i * Np + l] * (*D[b])[(size_t)l * Np + i];
          if (b != a) v += E[b][(size_t)i * Np + l] * (*D[a])[(size_t)l * Np + i];
          U.push_back(v);
        }
  slot = std::make_unique<DevBuf>(U.size() * sizeof(double));
  slot->upload(U.data(), U.size() * sizeof(double));
  return slot->as<double>();
}

cudaError_t launch_blocks(int dim, int order, const BlockArgs& a, cudaStream_t s) {
  int total = a.K * a.ncomp;
  if (total <= 0) return cudaSuccess;
  SIPG_DISPATCH_B(dim, order, {
    constexpr int W = BlockWarps<P>::W;
    const size_t smem = block_smem_doubles<D, P>() * sizeof(double);
    auto k = block_kernel<D, P>;
    cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    const int grid = std::max(1, std::min((total + W - 1) / W, 148 * 8));
    const double* U = a.mode == BLOCK_DIAG_ONLY ? diag_tables(D, P) : nullptr;
    k<<<grid, 32 * W, smem, s>>>(a, U);
    note_launch();
    return cudaGetLastError();
  });
  return cudaErrorInvalidValue;
}

cudaError_t launch_apply_bc(int dim, int order, const ApplyBcArgs& a, cudaStream_t s) {
  int total = a.n_belem * a.ncomp;
  if (total <= 0) return cudaSuccess;
  int grid = std::min(total, 148 * 16);
  SIPG_DISPATCH_B(dim, order, apply_bc_kernel<D, P><<<grid, 128, 0, s>>>(a); note_launch(); return cudaGetLastError());
  return cudaErrorInvalidValue;
}

}  // namespace sipg
