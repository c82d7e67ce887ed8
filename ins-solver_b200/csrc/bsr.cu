// Element-block form of low-order SIPG operators: assembly and apply.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>
#include <vector>

#include "../../include/sipg_b200.h"
#include "bsr.cuh"
#include "capi_util.hpp"
#include "pdl.cuh"
#include "sipg_blocks.cuh"
#include "vecops.cuh"

namespace sipg {
namespace {

int grid_of(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }

// Element-row blocks of the operator straight from the terms of the apply
// (sipg_apply.cu; FactorViscousMatrix3D::mult, factor_viscous_matrix.cpp:96-310),
// one thread per (row r, element e), e fastest (coalesced block stores), 64 per block. With
// Dx_d = sum_r G[r][d] D_r, Dn = sum_r (n . G[r]) D_r, F the nodal factor, MF the
// face mass, m_j / m+_j the own / neighbour node at face node j, scale = sJ / 2 on
// interior faces and sJ on Dirichlet faces (jump 2u, average n.q):
//   self:      J sum_d Dx_d^T M F Dx_d + J M diag(mm)
//              + rows on the face: scale MF (tau I - F Dn) at the face nodes
//              + columns m_j:      -scale f(m_j) sum_a Dn[m_a][r] MF[a][j]
//   neighbour: rows on the face:   -scale MF (tau I + F+ Dn+) at the matched nodes
//              columns m+_j:       +scale f(m_j) sum_a Dn[m_a][r] MF[a][j]
// (Dn+ built from the neighbour's G with this element's normal). The apply reads
// a pinned DOF as zero and returns pin_scale times it in its row: its column is
// zero and its row holds pin_scale on the diagonal only.
template <int DIM, int P>
__global__ void __launch_bounds__(64) k_bsr_direct(BlockArgs a, const uint32_t* __restrict__ fcode,
                                                    double* __restrict__ v) {
  using C = Cfg<DIM, P>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, LD = C::LD, NG = C::NG, NPERM = C::NPERM;
  __shared__ double sD[DIM][NP][NP], sM[NP][NP], sMF[NF][NFP][NFP];
  __shared__ int sfm[NF][NFP], sperm[NPERM][NFP];
  // the thread's row of every block, one shared-memory column per thread (the
  // entries are addressed through the face-node tables)
  __shared__ double sacc[(NF + 1) * NP][64];
#define ACC(s_, c_) sacc[(s_) * NP + (c_)][threadIdx.x]
  for (int t = threadIdx.x; t < DIM * NP * NP; t += blockDim.x) {
    const int d = t / (NP * NP), i = (t / NP) % NP, j = t % NP;
    sD[d][i][j] = a.consts[C::OFF_D + d * NP * LD + i * LD + j];
  }
  for (int t = threadIdx.x; t < NP * NP; t += blockDim.x) sM[t / NP][t % NP] = a.consts[C::OFF_M + (t / NP) * LD + t % NP];
  for (int t = threadIdx.x; t < NF * NFP * NFP; t += blockDim.x) (&sMF[0][0][0])[t] = a.mf[t];
  for (int t = threadIdx.x; t < NF * NFP; t += blockDim.x) (&sfm[0][0])[t] = a.itab[t];
  for (int t = threadIdx.x; t < NPERM * NFP; t += blockDim.x) (&sperm[0][0])[t] = a.itab[NF * NFP + t];
  __syncthreads();
  const size_t K = (size_t)a.K;
  for (size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x; tid < K * NP; tid += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(tid / K), e = (int)(tid - (size_t)r * K);
    double g[NG], f[NP];
#pragma unroll
    for (int i = 0; i < NG; ++i) g[i] = a.geof[(size_t)e * NG + i];
#pragma unroll
    for (int i = 0; i < NP; ++i) f[i] = a.factor ? a.factor[(size_t)e * NP + i] : 1.0;
    for (int q = 0; q < (NF + 1) * NP; ++q) sacc[q][threadIdx.x] = 0.0;
    const double J = g[DIM == 3 ? 9 : 4];
    // volume row r: J sum_d sum_q t_d[q] Dx_d[q][p], t_d[q] = f(q) sum_m Dx_d[m][r] M[m][q],
    // summed as sum_rr sum_q u_rr[q] D_rr[q][p] with u_rr[q] = sum_d G[rr][d] t_d[q]
    {
      double u[DIM][NP];
      {
        double t[DIM][NP];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          double col[NP];
#pragma unroll
          for (int m = 0; m < NP; ++m) {
            double s = 0.0;
#pragma unroll
            for (int rr = 0; rr < DIM; ++rr) s += g[rr * DIM + d] * sD[rr][m][r];
            col[m] = s;
          }
#pragma unroll
          for (int q = 0; q < NP; ++q) {
            double s = 0.0;
#pragma unroll
            for (int m = 0; m < NP; ++m) s += col[m] * sM[m][q];
            t[d][q] = J * f[q] * s;
          }
        }
#pragma unroll
        for (int rr = 0; rr < DIM; ++rr)
#pragma unroll
          for (int q = 0; q < NP; ++q) {
            double s = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) s += g[rr * DIM + d] * t[d][q];
            u[rr][q] = s;
          }
      }
#pragma unroll 1
      for (int p = 0; p < NP; ++p) {
        double s = 0.0;
#pragma unroll
        for (int rr = 0; rr < DIM; ++rr)
#pragma unroll
          for (int q = 0; q < NP; ++q) s += u[rr][q] * sD[rr][q][p];
        ACC(0, p) += s;
      }
    }
#pragma unroll 1
    for (int fc = 0; fc < NF; ++fc) {
      const int nb = a.nbr[(size_t)e * NF + fc];
      if (nb < 0 && a.bct[-nb - 1] != BC_DIRICHLET) continue;  // Neumann (and scalar slip): no face terms
      double n[3], sJ;
      simplex_face_normal<DIM>(g, fc, n, &sJ);
      const double scale = nb >= 0 ? 0.5 * sJ : sJ;
      const double tau = a.tau[(size_t)e * NF + fc];
      double rf[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int rr = 0; rr < DIM; ++rr)
#pragma unroll
        for (int d = 0; d < DIM; ++d) rf[rr] += n[d] * g[rr * DIM + d];
      // neighbour data: matched nodes, factor, geometry
      int nm[NFP];
      double rfn[3] = {0.0, 0.0, 0.0};
      const double* gn = nullptr;
      if (nb >= 0) {
        const int code = (fcode[e] >> (8 * fc)) & 0xff;
#pragma unroll
        for (int j = 0; j < NFP; ++j) nm[j] = sfm[code & 3][sperm[code >> 2][j]];
        gn = a.geof + (size_t)nb * NG;
#pragma unroll
        for (int rr = 0; rr < DIM; ++rr)
#pragma unroll
          for (int d = 0; d < DIM; ++d) rfn[rr] += n[d] * gn[rr * DIM + d];
      }
      // columns: -/+ scale f(m_j) sum_a Dn[m_a][r] MF[a][j]
      double dnr[NFP];
#pragma unroll
      for (int aa = 0; aa < NFP; ++aa) {
        double s = 0.0;
#pragma unroll
        for (int rr = 0; rr < DIM; ++rr) s += rf[rr] * sD[rr][sfm[fc][aa]][r];
        dnr[aa] = s;
      }
#pragma unroll
      for (int j = 0; j < NFP; ++j) {
        double cj = 0.0;
#pragma unroll
        for (int aa = 0; aa < NFP; ++aa) cj += dnr[aa] * sMF[fc][aa][j];
        const double w = scale * f[sfm[fc][j]] * cj;
        ACC(0, sfm[fc][j]) -= w;
        if (nb >= 0) ACC(1 + fc, nm[j]) += w;
      }
      // rows on the face
      int ar = -1;
#pragma unroll
      for (int aa = 0; aa < NFP; ++aa)
        if (sfm[fc][aa] == r) ar = aa;
      if (ar < 0) continue;
#pragma unroll 1
      for (int j = 0; j < NFP; ++j) {
        const double w = scale * sMF[fc][ar][j];
        const int mj = sfm[fc][j];
        ACC(0, mj) += w * tau;
        const double wf = w * f[mj];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          double dn = 0.0;
#pragma unroll
          for (int rr = 0; rr < DIM; ++rr) dn += rf[rr] * sD[rr][mj][p];
          ACC(0, p) -= wf * dn;
        }
        if (nb >= 0) {
          const int q = nm[j];
          ACC(1 + fc, q) -= w * tau;
          const double wfn = w * (a.factor ? a.factor[(size_t)nb * NP + q] : 1.0);
#pragma unroll
          for (int c = 0; c < NP; ++c) {
            double dn = 0.0;
#pragma unroll
            for (int rr = 0; rr < DIM; ++rr) dn += rfn[rr] * sD[rr][q][c];
            ACC(1 + fc, c) -= wfn * dn;
          }
        }
      }
    }
    if (a.mm_mode != MM_NONE)
#pragma unroll
      for (int p = 0; p < NP; ++p) ACC(0, p) += J * sM[r][p] * (a.mm_mode == MM_SCALAR ? a.mm_scalar : a.mm[(size_t)e * NP + p]);
    // the pinned DOF is read as zero by every row (its column vanishes) ...
    if (a.pin_elem >= 0) {
      if (e == a.pin_elem) ACC(0, a.pin_node) = 0.0;
      for (int fc = 0; fc < NF; ++fc)
        if (a.nbr[(size_t)e * NF + fc] == a.pin_elem) ACC(1 + fc, a.pin_node) = 0.0;
    }
    // ... and its own row is pin_scale times itself
    if (e == a.pin_elem && r == a.pin_node) {
#pragma unroll
      for (int s = 0; s <= NF; ++s)
#pragma unroll
        for (int c = 0; c < NP; ++c) ACC(s, c) = (s == 0 && c == r) ? a.pin_scale : 0.0;
    }
#pragma unroll
    for (int s = 0; s <= NF; ++s)
#pragma unroll
      for (int c = 0; c < NP; ++c) v[((size_t)(s * NP + r) * NP + c) * K + e] = ACC(s, c);
  }
#undef ACC
}

__global__ void k_d2f(float* dst, const double* src, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

// One thread per (row r, element e), e fastest: block reads are coalesced and
// there are Np threads per element row to hide the gather latency.
// V4: x rows read as one 16-byte load (FP32, Np = 4, x 16-byte aligned).
template <typename T, int NP, int NF, bool V4 = false>
__global__ void __launch_bounds__(256) k_bsr(int K, const T* __restrict__ v, const int* __restrict__ nbr,
                                             const T* __restrict__ x, T* y, T alpha, T beta, const T* c) {
  pdl_enter();
  const size_t K_ = (size_t)K;
  const size_t total = K_ * NP;
  for (size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x; tid < total; tid += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(tid / K_);
    const int e = (int)(tid - (size_t)r * K_);
    int ks[NF + 1];
    ks[0] = e;
#pragma unroll
    for (int f = 0; f < NF; ++f) ks[f + 1] = nbr[(size_t)e * NF + f];
    T acc = T(0);
#pragma unroll
    for (int s = 0; s <= NF; ++s) {
      const int k = ks[s];
      if (k < 0) continue;
      const T* vs = v + ((size_t)(s * NP + r) * NP) * K_ + e;
      const T* xk = x + (size_t)k * NP;
      T xv[NP];
      if constexpr (V4 && std::is_same<T, float>::value && NP == 4) {
        const float4 q = *reinterpret_cast<const float4*>(xk);
        xv[0] = q.x; xv[1] = q.y; xv[2] = q.z; xv[3] = q.w;
      } else {
#pragma unroll
        for (int c = 0; c < NP; ++c) xv[c] = xk[c];
      }
#pragma unroll
      for (int c = 0; c < NP; ++c) acc += vs[(size_t)c * K_] * xv[c];
    }
    T o = alpha * acc;
    if (beta != T(0)) o += beta * c[(size_t)e * NP + r];
    y[(size_t)e * NP + r] = o;
  }
}

// Scaled FP16 copy of the blocks: per element the largest magnitude over its
// (NF + 1) Np^2 values is the scale, and v16 holds values / scale in the
// row-fastest layout of k_bsr16.
__global__ void k_bsr16_pack(const double* __restrict__ v64, int K, int Np, int NS, __half* __restrict__ v16,
                             float* __restrict__ scale) {
  const size_t K_ = (size_t)K;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < K; e += gridDim.x * blockDim.x) {
    double m = 0.0;
    for (int q = 0; q < NS * Np * Np; ++q) m = fmax(m, fabs(v64[(size_t)q * K_ + e]));
    const float sc = m > 0.0 ? (float)m : 1.0f;
    scale[e] = sc;
    for (int s = 0; s < NS; ++s)
      for (int r = 0; r < Np; ++r)
        for (int c = 0; c < Np; ++c)
          v16[(((size_t)s * Np + c) * K_ + e) * Np + r] =
              __double2half(v64[(((size_t)s * Np + r) * Np + c) * K_ + e] / (double)sc);
  }
}

// Two rows per thread: t2 = e Np/2 + r/2 (Np even), so the Np/2 threads of an
// element read consecutive FP16 pairs and the same x values (broadcast). The
// neighbour list is read first and every block value is loaded without a branch
// (boundary slots hold zero blocks and read the element's own x row), so all
// loads of a thread are independent. y = alpha scale[e] acc + beta c, FP32
// accumulation.
template <int NP, int NF>
__global__ void __launch_bounds__(256, 2) k_bsr16(int K, const __half* __restrict__ v, const float* __restrict__ scale,
                                               const int* __restrict__ nbr, const float* __restrict__ x, float* y,
                                               float alpha, float beta, const float* c) {
  static_assert(NP % 2 == 0, "two rows per thread");
  pdl_enter();
  constexpr int H = NP / 2;
  const size_t KH = (size_t)K * H;
  const __half2* v2 = reinterpret_cast<const __half2*>(v);
  for (size_t t2 = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t2 < KH; t2 += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(t2 / H);
    int ks[NF + 1];
    ks[0] = e;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const int k = nbr[(size_t)e * NF + f];
      ks[f + 1] = k < 0 ? e : k;
    }
    // all loads first (about 100 in flight per thread), then the products
    __half2 w[NF + 1][NP];
    float xv[NF + 1][NP];
#pragma unroll
    for (int s = 0; s <= NF; ++s)
#pragma unroll
      for (int cc = 0; cc < NP; ++cc) w[s][cc] = v2[(size_t)(s * NP + cc) * KH + t2];
#pragma unroll
    for (int s = 0; s <= NF; ++s)
#pragma unroll
      for (int cc = 0; cc < NP; ++cc) xv[s][cc] = x[(size_t)ks[s] * NP + cc];
    float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
    for (int s = 0; s <= NF; ++s)
#pragma unroll
      for (int cc = 0; cc < NP; ++cc) {
        const float2 wf = __half22float2(w[s][cc]);
        a0 += wf.x * xv[s][cc];
        a1 += wf.y * xv[s][cc];
      }
    const float sc = scale[e];
    float2 o = make_float2(alpha * (sc * a0), alpha * (sc * a1));
    if (beta != 0.0f) {
      const float2 cv = *reinterpret_cast<const float2*>(c + 2 * t2);
      o.x += beta * cv.x;
      o.y += beta * cv.y;
    }
    *reinterpret_cast<float2*>(y + 2 * t2) = o;
  }
}

// C = Bi A per element row block (FP64), Bi the inverse diagonal block as the
// smoother stores it: its symmetric part when sym (packed triangles,
// k_block_pack_sym), else as is. C[s][r][c][e] = sum_m Bi_e[r][m] A[s][m][c][e],
// one thread per (block entry, element), element fastest.
// C = Bd^-1 A block by block: one thread per (element, row r, block s) holds row r of
// the element's inverse diagonal block in registers (symmetrised when sym) and writes
// the Np entries of row r of C's block s; the loads of A and the stores of C are
// coalesced over the elements.
template <int NP>
__global__ void k_bsr_precond(const double* __restrict__ A, const double* __restrict__ binv, int K, int NS, int sym,
                              double* __restrict__ C) {
  const size_t K_ = (size_t)K, total = (size_t)NS * NP * K_;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t e = i % K_, q = i / K_;
    const int r = (int)(q % NP), s = (int)(q / NP);
    const double* be = binv + e * NP * NP;
    double b[NP];
#pragma unroll
    for (int m = 0; m < NP; ++m) b[m] = sym ? 0.5 * (be[r * NP + m] + be[m * NP + r]) : be[r * NP + m];
    for (int c = 0; c < NP; ++c) {
      double acc = 0.0;
#pragma unroll
      for (int m = 0; m < NP; ++m) acc += b[m] * A[(((size_t)s * NP + m) * NP + c) * K_ + e];
      C[(((size_t)s * NP + r) * NP + c) * K_ + e] = acc;
    }
  }
}

// One fused Chebyshev step (bsr_cheb_step), same thread layout and loads as k_bsr16.
template <int NP, int NF>
__global__ void __launch_bounds__(256, 2) k_bsr16_cheb(int K, const __half* __restrict__ v,
                                                       const float* __restrict__ scale, const int* __restrict__ nbr,
                                                       const float* __restrict__ din, float* __restrict__ dout,
                                                       float* sres, float* z, float c1, float c2, float s0_scale) {
  static_assert(NP % 2 == 0, "two rows per thread");
  pdl_enter();
  constexpr int H = NP / 2;
  const size_t KH = (size_t)K * H;
  const __half2* v2 = reinterpret_cast<const __half2*>(v);
  for (size_t t2 = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t2 < KH; t2 += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(t2 / H);
    int ks[NF + 1];
    ks[0] = e;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const int k = nbr[(size_t)e * NF + f];
      ks[f + 1] = k < 0 ? e : k;
    }
    __half2 w[NF + 1][NP];
    float xv[NF + 1][NP];
#pragma unroll
    for (int s = 0; s <= NF; ++s)
#pragma unroll
      for (int cc = 0; cc < NP; ++cc) w[s][cc] = v2[(size_t)(s * NP + cc) * KH + t2];
#pragma unroll
    for (int s = 0; s <= NF; ++s)
#pragma unroll
      for (int cc = 0; cc < NP; ++cc) xv[s][cc] = din[(size_t)ks[s] * NP + cc];
    float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
    for (int s = 0; s <= NF; ++s)
#pragma unroll
      for (int cc = 0; cc < NP; ++cc) {
        const float2 wf = __half22float2(w[s][cc]);
        a0 += wf.x * xv[s][cc];
        a1 += wf.y * xv[s][cc];
      }
    const float sc = scale[e];
    const float2 d0 = *reinterpret_cast<const float2*>(din + 2 * t2);
    float2 sr = s0_scale != 0.0f ? make_float2(s0_scale * d0.x, s0_scale * d0.y)
                                 : *reinterpret_cast<const float2*>(sres + 2 * t2);
    sr.x -= sc * a0;
    sr.y -= sc * a1;
    const float2 dn = make_float2(c1 * d0.x + c2 * sr.x, c1 * d0.y + c2 * sr.y);
    float2 zz = *reinterpret_cast<const float2*>(z + 2 * t2);
    zz.x += dn.x;
    zz.y += dn.y;
    *reinterpret_cast<float2*>(sres + 2 * t2) = sr;
    *reinterpret_cast<float2*>(dout + 2 * t2) = dn;
    *reinterpret_cast<float2*>(z + 2 * t2) = zz;
  }
}

}  // namespace

void element_blocks_device(const sipg_op* op, double* v, cudaStream_t s) {
  if (op->ncomp != 1) throw Error(SIPG_INVALID_ARG, "element blocks need a scalar operator");
  const sipg_mesh* m = op->mesh;
  const BlockArgs a = op->block_args(BLOCK_FULL, 0, v, true);
  const size_t n = (size_t)m->K * op->Np;
  const int g = (int)std::max<size_t>(1, std::min<size_t>((n + 63) / 64, 148 * 32));
  const uint32_t* fc = m->fcode.as<uint32_t>();
  switch (m->dim * 10 + op->order) {
    case 21: k_bsr_direct<2, 1><<<g, 64, 0, s>>>(a, fc, v); break;
    case 22: k_bsr_direct<2, 2><<<g, 64, 0, s>>>(a, fc, v); break;
    case 31: k_bsr_direct<3, 1><<<g, 64, 0, s>>>(a, fc, v); break;
    case 32: k_bsr_direct<3, 2><<<g, 64, 0, s>>>(a, fc, v); break;
    default: throw Error(SIPG_INVALID_ARG, "element blocks: orders 1 and 2 only");
  }
  note_launch();
  SIPG_CUDA(cudaGetLastError());
}

void bsr_assemble(sipg_op* op, BsrOp& B, bool want32, cudaStream_t s, const double* binv_rows, bool binv_sym) {
  if (op->ncomp != 1) throw Error(SIPG_INVALID_ARG, "assembled blocks need a scalar operator");
  sipg_mesh* m = op->mesh;
  const int K = m->K, Np = op->Np, NF = m->dim + 1;
  B.K = K;
  B.Np = Np;
  B.NF = NF;
  B.dim = m->dim;
  B.nbr = m->nbr.as<int>();
  const size_t nv = (size_t)(NF + 1) * Np * Np * K;
  ensure(B.v64, nv * sizeof(double));
  element_blocks_device(op, B.v64.as<double>(), s);
  const bool half = want32 && Np % 2 == 0;  // two rows per thread in k_bsr16
  if (half) {
    ensure(B.v16, nv * sizeof(__half));
    ensure(B.scale16, (size_t)K * sizeof(float));
    k_bsr16_pack<<<grid_of(K), 256, 0, s>>>(B.v64.as<double>(), K, Np, NF + 1, B.v16.as<__half>(),
                                            B.scale16.as<float>());
    note_launch();
    if (binv_rows) {
      ensure(B.c64, nv * sizeof(double));
      DevBuf& c64 = B.c64;
      const size_t nrows = (size_t)(NF + 1) * Np * K;
      const int sy = binv_sym ? 1 : 0;
      switch (Np) {  // the even orders that reach here: two rows per thread in k_bsr16
        case 4: k_bsr_precond<4><<<grid_of(nrows), 256, 0, s>>>(B.v64.as<double>(), binv_rows, K, NF + 1, sy, c64.as<double>()); break;
        case 6: k_bsr_precond<6><<<grid_of(nrows), 256, 0, s>>>(B.v64.as<double>(), binv_rows, K, NF + 1, sy, c64.as<double>()); break;
        case 10: k_bsr_precond<10><<<grid_of(nrows), 256, 0, s>>>(B.v64.as<double>(), binv_rows, K, NF + 1, sy, c64.as<double>()); break;
        case 20: k_bsr_precond<20><<<grid_of(nrows), 256, 0, s>>>(B.v64.as<double>(), binv_rows, K, NF + 1, sy, c64.as<double>()); break;
        default: throw Error(SIPG_INVALID_ARG, "block-preconditioned assembled level: unsupported Np");
      }
      note_launch();
      SIPG_CUDA(cudaGetLastError());
      ensure(B.c16, nv * sizeof(__half));
      ensure(B.cscale16, (size_t)K * sizeof(float));
      k_bsr16_pack<<<grid_of(K), 256, 0, s>>>(c64.as<double>(), K, Np, NF + 1, B.c16.as<__half>(),
                                              B.cscale16.as<float>());
      note_launch();
    }
  } else if (want32) {
    ensure(B.v32, nv * sizeof(float));
    k_d2f<<<grid_of(nv), 256, 0, s>>>(B.v32.as<float>(), B.v64.as<double>(), nv);
    note_launch();
  }
  SIPG_CUDA(cudaGetLastError());
}

template <typename T>
void bsr_apply(const BsrOp& B, const T* x, T* y, T alpha, T beta, cudaStream_t s, const T* c) {
  if (!c) c = y;
  if constexpr (std::is_same<T, float>::value) {
    if (B.v16.p) {
      if (((reinterpret_cast<uintptr_t>(y) | reinterpret_cast<uintptr_t>(c)) & 7) != 0)
        throw Error(SIPG_INVALID_ARG, "the FP16 assembled apply needs 8-byte aligned vectors");
      const int g = (int)std::max<size_t>(1, std::min<size_t>(((size_t)B.K * B.Np / 2 + 255) / 256, 148 * 32));
      const __half* v = B.v16.as<__half>();
      const float* sc = B.scale16.as<float>();
      if (B.dim == 3 && B.Np == 10)
        pdl_launch(k_bsr16<10, 4>, dim3(g), dim3(256), 0, s, B.K, v, sc, B.nbr, x, y, alpha, beta, c);
      else if (B.dim == 3 && B.Np == 4)
        pdl_launch(k_bsr16<4, 4>, dim3(g), dim3(256), 0, s, B.K, v, sc, B.nbr, x, y, alpha, beta, c);
      else if (B.dim == 2 && B.Np == 6)
        pdl_launch(k_bsr16<6, 3>, dim3(g), dim3(256), 0, s, B.K, v, sc, B.nbr, x, y, alpha, beta, c);
      else
        throw Error(SIPG_INVALID_ARG, "no FP16 assembled apply for this element");
      note_launch();
      SIPG_CUDA(cudaGetLastError());
      return;
    }
  }
  const T* v = std::is_same<T, double>::value ? (const T*)B.v64.p : (const T*)B.v32.p;
  if (!v) throw Error(SIPG_INVALID_ARG, "assembled blocks missing for this precision");
  const int g = (int)std::max<size_t>(1, std::min<size_t>(((size_t)B.K * B.Np + 255) / 256, 148 * 32));
  const bool v4 = std::is_same<T, float>::value && (reinterpret_cast<uintptr_t>(x) & 15) == 0;
  if (B.dim == 3 && B.Np == 4 && v4)
    pdl_launch(k_bsr<T, 4, 4, true>, dim3(g), dim3(256), 0, s, B.K, v, B.nbr, x, y, alpha, beta, c);
  else if (B.dim == 3 && B.Np == 4) pdl_launch(k_bsr<T, 4, 4>, dim3(g), dim3(256), 0, s, B.K, v, B.nbr, x, y, alpha, beta, c);
  else if (B.dim == 3 && B.Np == 10) pdl_launch(k_bsr<T, 10, 4>, dim3(g), dim3(256), 0, s, B.K, v, B.nbr, x, y, alpha, beta, c);
  else if (B.dim == 2 && B.Np == 3) pdl_launch(k_bsr<T, 3, 3>, dim3(g), dim3(256), 0, s, B.K, v, B.nbr, x, y, alpha, beta, c);
  else if (B.dim == 2 && B.Np == 6) pdl_launch(k_bsr<T, 6, 3>, dim3(g), dim3(256), 0, s, B.K, v, B.nbr, x, y, alpha, beta, c);
  // orders 3 and 4 (the over-integrated operator's blocks)
  else if (B.dim == 3 && B.Np == 20) pdl_launch(k_bsr<T, 20, 4>, dim3(g), dim3(256), 0, s, B.K, v, B.nbr, x, y, alpha, beta, c);
  else if (B.dim == 3 && B.Np == 35) pdl_launch(k_bsr<T, 35, 4>, dim3(g), dim3(256), 0, s, B.K, v, B.nbr, x, y, alpha, beta, c);
  else if (B.dim == 2 && B.Np == 10) pdl_launch(k_bsr<T, 10, 3>, dim3(g), dim3(256), 0, s, B.K, v, B.nbr, x, y, alpha, beta, c);
  else if (B.dim == 2 && B.Np == 15) pdl_launch(k_bsr<T, 15, 3>, dim3(g), dim3(256), 0, s, B.K, v, B.nbr, x, y, alpha, beta, c);
  else throw Error(SIPG_INVALID_ARG, "no assembled apply for this element");
  note_launch();
  SIPG_CUDA(cudaGetLastError());
}

void bsr_cheb_step(const BsrOp& B, const float* din, float* dout, float* sres, float* z, float c1, float c2,
                   float s0_scale, cudaStream_t s) {
  if (!B.c16.p) throw Error(SIPG_INVALID_ARG, "preconditioned FP16 blocks missing");
  if (((reinterpret_cast<uintptr_t>(din) | reinterpret_cast<uintptr_t>(dout) | reinterpret_cast<uintptr_t>(sres) |
        reinterpret_cast<uintptr_t>(z)) & 7) != 0)
    throw Error(SIPG_INVALID_ARG, "the fused Chebyshev step needs 8-byte aligned vectors");
  const int g = (int)std::max<size_t>(1, std::min<size_t>(((size_t)B.K * B.Np / 2 + 255) / 256, 148 * 32));
  const __half* v = B.c16.as<__half>();
  const float* sc = B.cscale16.as<float>();
  if (B.dim == 3 && B.Np == 10)
    pdl_launch(k_bsr16_cheb<10, 4>, dim3(g), dim3(256), 0, s, B.K, v, sc, B.nbr, din, dout, sres, z, c1, c2, s0_scale);
  else if (B.dim == 3 && B.Np == 4)
    pdl_launch(k_bsr16_cheb<4, 4>, dim3(g), dim3(256), 0, s, B.K, v, sc, B.nbr, din, dout, sres, z, c1, c2, s0_scale);
  else if (B.dim == 2 && B.Np == 6)
    pdl_launch(k_bsr16_cheb<6, 3>, dim3(g), dim3(256), 0, s, B.K, v, sc, B.nbr, din, dout, sres, z, c1, c2, s0_scale);
  else
    throw Error(SIPG_INVALID_ARG, "no fused Chebyshev step for this element");
  note_launch();
  SIPG_CUDA(cudaGetLastError());
}

template void bsr_apply<double>(const BsrOp&, const double*, double*, double, double, cudaStream_t, const double*);
template void bsr_apply<float>(const BsrOp&, const float*, float*, float, float, cudaStream_t, const float*);

}  // namespace sipg

extern "C" int sipg_op_element_blocks_host(sipg_op* op, double* blocks) {
  using namespace sipg;
  return guarded([&] {
    if (!op || !blocks) throw Error(SIPG_INVALID_ARG, "element_blocks arguments");
    const size_t n = (size_t)(op->mesh->dim + 2) * op->Np * op->Np * op->mesh->K;
    DevBuf d(n * sizeof(double));
    element_blocks_device(op, d.as<double>(), 0);
    SIPG_CUDA(cudaMemcpy(blocks, d.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  });
}
