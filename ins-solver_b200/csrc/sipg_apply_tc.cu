// Tensor-core SIPG apply (scalar operator): FP32 data on TF32 tensor cores or
// FP64 data on the FP64 tensor cores, in two passes over the elements.
//
// Same operator as sipg_apply.cu (FactorViscousMatrix3D::mult,
// src/solvers/3d/slip_matrix/factor_viscous_matrix.cpp:96-310, one component).
// The reference exchanges face data through 12 face buffers per component
// (mesh->jump / mesh->avg into K x Nf*Nfp op_dats); here each element publishes
// one trace record per face and every matrix product is batched over elements.
//
// Elements are the M dimension of mma.sync (16 per warp tile for TF32
// m16n8k8, 8 for FP64 m8n8k4); the reference-element matrices are the B
// operands, packed on the host in fragment order. An accumulator block is laid
// out exactly like an A block once the dummy summation index k is permuted
// (slot t <-> logical column 2t, slot t+4 <-> 2t+1, folded into the packing of
// B), so a product's result feeds the next product from registers and the
// elementwise steps (metric terms, fluxes) run on fragment registers.
//
//   pass 1 (traces): per face node k = (f, j) with volume node m = fmask(f, j):
//           g = f(m) sum_r c_r(f) (D_r x)(m), c_r = n_f . grad r, computed as
//           x (TE x Np) . BF_r (Np x Nf*Nfp), BF_r[n][k] = D_r[m(k)][n];
//           trace[e][f] = (x(m(f, j)) for j < Nfp, g(f, j) for j < Nfp).
//   pass 2 (apply): gr_r = x . B1_r (gradient in the reference directions),
//           w_r = J f sum_s K_rs gr_s (K = G G^T, the metric of the element),
//           fluxes from the own and the neighbour's traces
//             [u] = u- - u+, n.{q} = (g- - g+)/2 (n+ = -n-), boundary faces as
//             vmf_3d_mult_avg_jump.h:43-80,
//             Fu = sJ (tau [u]/2 - n.{q}), S = -sJ f [u]/2 (fvmf_3d_mult_flux.h:13-22),
//           Z_r = w_r . M^T + (c_r S) . EMAT^T,
//           y = sum_r Z_r . D_r + Fu . EMAT^T + (J mm x) . M^T.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "pdl.cuh"
#include "sipg_apply.cuh"
#include "sipg_apply_tc.cuh"
#include "vecops.cuh"

namespace sipg {
namespace {

__host__ __device__ constexpr int rup(int x, int m) { return (x + m - 1) / m * m; }

// MMA on logical blocks of 8R element rows x 8 columns. Lane (g = lane/4,
// t = lane%4) holds rows g + 8 ri (ri < R) and logical columns 2t + ci (ci < 2)
// of an A block and of an accumulator block, and rows 2t + ci, column g of a
// B block (one V2 per lane in the packed blobs).
template <typename T>
struct Frag;

template <>
struct Frag<float> {
  static constexpr int R = 2;
  using V2 = float2;
  // FP32 values go to the TF32 MMA as they are: the tensor core uses the sign,
  // exponent and top 10 mantissa bits (truncation, relative error below 2^-10
  // per operand instead of 2^-11 after a round-to-nearest conversion). Dropping
  // the conversion instruction (about 160 per warp tile and lane at p = 3) left
  // the iteration counts of the mixed-precision solves unchanged.
  __device__ static __forceinline__ float op(float x) { return x; }
  // m16n8k8: a0 (g, t) a1 (g+8, t) a2 (g, t+4) a3 (g+8, t+4); b0 (t, g) b1 (t+4, g);
  // c0 (g, 2t) c1 (g, 2t+1) c2 (g+8, 2t) c3 (g+8, 2t+1).
  __device__ static __forceinline__ void mma(float (&c)[2][2], const float (&a)[2][2], V2 b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0][0]), "+f"(c[0][1]), "+f"(c[1][0]), "+f"(c[1][1])
        : "r"(__float_as_uint(a[0][0])), "r"(__float_as_uint(a[1][0])), "r"(__float_as_uint(a[0][1])),
          "r"(__float_as_uint(a[1][1])), "r"(__float_as_uint(b.x)), "r"(__float_as_uint(b.y)));
  }
};

template <>
struct Frag<double> {
  static constexpr int R = 1;
  using V2 = double2;
  __device__ static __forceinline__ double op(double x) { return x; }
  // two m8n8k4 steps: a0 (g, t), b0 (t, g), c0 (g, 2t) c1 (g, 2t+1); the first
  // binds slot t to logical column 2t, the second to 2t+1.
  __device__ static __forceinline__ void mma(double (&c)[1][2], const double (&a)[1][2], V2 b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0][0]), "+d"(c[0][1])
                 : "d"(a[0][0]), "d"(b.x));
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0][0]), "+d"(c[0][1])
                 : "d"(a[0][1]), "d"(b.y));
  }
};

// Smallest m >= n with m = 8 (mod 16): row stride of staged element data for
// which the pair loads of a fragment (two adjacent columns per lane, element
// rows g) fall in distinct banks.
__host__ __device__ constexpr int pad816(int n) { return n <= 8 ? 8 : rup(n - 8, 16) + 8; }

template <typename T, int DIM, int P>
struct Tc {
  using C = Cfg<DIM, P>;
  static constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF;
  static constexpr int R = Frag<T>::R, TE = 8 * R;   // elements per warp tile
  static constexpr int NT = rup(NP, 8) / 8;          // node blocks
  static constexpr int KF = NF * NFP;                // face nodes of an element
  static constexpr int FT = rup(KF, 8) / 8;          // face-node blocks
  static constexpr int TRP = rup(NFP, 2);            // g part of a trace record starts here
  static constexpr int TR = rup(2 * TRP, 4);         // record length: a 16-byte multiple
  static constexpr int BLK = 64;                     // values per packed 8 x 8 block
  // pass-2 blob: B1_r (NT x NT blocks), BM, BE (FT x NT), B3_r; then the pass-1 blob BF_r (NT x FT)
  static constexpr int B1 = 0;
  static constexpr int BM = B1 + DIM * NT * NT * BLK;
  static constexpr int BE = BM + NT * NT * BLK;
  static constexpr int B3 = BE + FT * NT * BLK;
  static constexpr int N2 = B3 + DIM * NT * NT * BLK;
  static constexpr int BF = N2;
  static constexpr int N1 = DIM * NT * FT * BLK;
  static constexpr int NALL = N2 + N1;
  static constexpr int XS = pad816(NP);              // staged row stride of x and factor
  static constexpr int TS = pad816(NF * TR);         // staged row stride of an element's trace records
  // copy piece of an x / factor row (rows start on multiples of Np values)
  static constexpr int XCB = (NP * (int)sizeof(T)) % 16 == 0 ? 16 : (NP * (int)sizeof(T)) % 8 == 0 ? 8 : 4;
  // geometry block of a warp tile (launch_tc_geom), rows of TE values: NV volume
  // rows (J, then the metric K = G G^T by rows of its upper triangle, zero rows),
  // then NFG x NF face rows [q][f] (q: sJ, c_0, c_1, c_2)
  static constexpr int NV = 8, NFG = 4, GROWS = NV + NFG * NF;
  static constexpr int SFG = NFG * NF * TE;
  // element stage (T units, every part a multiple of 64 bytes): x, factor, then
  // the face rows of the geometry block (pass 1) or the whole block and tau (pass 2)
  static constexpr int SX = 0, SF = TE * XS, SG = 2 * TE * XS;
  static constexpr int ST1 = SG + SFG;
  static constexpr int STAU = SG + GROWS * TE, ST2 = STAU + TE * NF;
  static constexpr int SI = TE * NF + TE;            // int slot: nbr, face codes
  // pass 1 warp: 2 stages, output records
  static constexpr int W1_T = 2 * ST1 + TE * TS;
  static constexpr int W2_I = 3 * SI;
  static constexpr int CH = TR * (int)sizeof(T) / 16;  // 16-byte chunks per trace record
};

// Pass-2 warp area: NS element stages, own and neighbour trace records (one
// buffer each).
template <typename T, int DIM, int P, int NS>
struct W2 {
  using X = Tc<T, DIM, P>;
  static constexpr int STR = NS * X::ST2, SNB = STR + X::TE * X::TS, T_ = SNB + X::TE * X::TS;
};

// Row of the metric entry K_rs (r <= s) in the geometry block.
__host__ __device__ constexpr int kidx(int dim, int r, int s) { return 1 + r * dim - r * (r - 1) / 2 + (s - r); }

template <typename T>
__device__ __forceinline__ typename Frag<T>::V2 ldb(const T* blob, int blk, int lane) {
  return reinterpret_cast<const typename Frag<T>::V2*>(blob)[blk * 32 + lane];
}
template <typename T>
__device__ __forceinline__ typename Frag<T>::V2 ld2(const T* p) {
  return *reinterpret_cast<const typename Frag<T>::V2*>(p);
}

// CB-byte asynchronous copy (4, 8 or 16), zero-filled past `bytes`.
template <int CB>
__device__ __forceinline__ void cp_async_n(void* sdst, const void* gsrc, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  if (CB == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(bytes));
  else if (CB == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(bytes));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc), "r"(bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }
__device__ __forceinline__ void cp_wait_but_one() { asm volatile("cp.async.wait_group 1;\n" ::); }

// Copy `total` bytes (a multiple of 16) to shared memory: the first `valid`
// come from base + off (16-byte aligned), the rest is zero.
__device__ __forceinline__ void copy_block(void* s, const void* base, size_t off, int total, int valid, int lane) {
  const char* b = static_cast<const char*>(base);
  for (int c = lane * 16; c < total; c += 32 * 16) {
    const int n = min(16, max(0, valid - c));
    cp_async_n<16>(static_cast<char*>(s) + c, n > 0 ? b + off + c : b, n);
  }
}

// NR rows of LEN values (global rows contiguous from row0) into shared rows of
// stride DS; rows at or past nvalid are zero-filled (zero) or skipped. Lane
// handles row lane % NR and every (32 / NR)-th piece of it, so the row address is
// computed once.
template <typename T, int CB, int LEN, int DS, int NR>
__device__ __forceinline__ void copy_rows(T* dst, const T* base, size_t row0, int nvalid, int lane, bool zero) {
  constexpr int V = CB / (int)sizeof(T), CPR = LEN / V, LPR = 32 / NR;
  static_assert(LEN % V == 0, "row length must be a multiple of the copy piece");
  static_assert(32 % NR == 0, "rows must divide the warp");
  const int r = lane % NR, q = lane / NR;
  const bool v = r < nvalid;
  if (!v && !zero) return;
  T* d = dst + r * DS;
  const T* src = v ? base + (row0 + r) * LEN : base;
#pragma unroll
  for (int c0 = 0; c0 < CPR; c0 += LPR) {
    const int c = c0 + q;
    if (c < CPR) cp_async_n<CB>(d + c * V, v ? src + c * V : base, v ? CB : 0);
  }
}

template <typename T, int DIM, int P>
__device__ __forceinline__ void issue_elem(const ApplyArgs<T>& a, T* st, int tile, int lane, bool pass2) {
  using X = Tc<T, DIM, P>;
  constexpr int NP = X::NP, NF = X::NF, TE = X::TE, S = sizeof(T);
  const int e0 = tile * TE;
  const int ne = max(0, min(TE, a.K - e0));
  copy_rows<T, X::XCB, NP, X::XS, TE>(st + X::SX, a.x, (size_t)e0, ne, lane, true);
  if (a.factor) copy_rows<T, X::XCB, NP, X::XS, TE>(st + X::SF, a.factor, (size_t)e0, ne, lane, true);
  // the geometry block is zero past K, so a started tile copies it whole
  const size_t gb = (size_t)tile * X::GROWS * TE * S;
  if (pass2) {
    copy_block(st + X::SG, a.tcg, gb, X::GROWS * TE * S, ne > 0 ? X::GROWS * TE * S : 0, lane);
    copy_block(st + X::STAU, a.tau, (size_t)e0 * NF * S, TE * NF * S, ne * NF * S, lane);
  } else {
    copy_block(st + X::SG, a.tcg, gb + (size_t)X::NV * TE * S, X::SFG * S, ne > 0 ? X::SFG * S : 0, lane);
  }
}

template <typename T, int DIM, int P>
__device__ __forceinline__ void issue_ints(const ApplyArgs<T>& a, int* slot, int tile, int lane) {
  using X = Tc<T, DIM, P>;
  constexpr int NF = X::NF, TE = X::TE;
  const int e0 = tile * TE;
  const int ne = max(0, min(TE, a.K - e0));
  copy_block(slot, a.nbr, (size_t)e0 * NF * 4, TE * NF * 4, ne * NF * 4, lane);
  copy_block(slot + TE * NF, a.fcode, (size_t)e0 * 4, TE * 4, ne * 4, lane);
}

// Own and neighbour trace records of a tile whose connectivity has arrived
// (records that are never read are not copied).
template <typename T, int DIM, int P, int NS>
__device__ __forceinline__ void issue_traces(const ApplyArgs<T>& a, const T* trace, T* w, const int* slot, int tile,
                                             int lane) {
  using X = Tc<T, DIM, P>;
  using L = W2<T, DIM, P, NS>;
  constexpr int NF = X::NF, TE = X::TE, CH = X::CH, TR = X::TR, TS = X::TS, VPC = 16 / sizeof(T);
  const int e0 = tile * TE;
  const int ne = max(0, min(TE, a.K - e0));
  copy_rows<T, 16, NF * TR, TS, TE>(w + L::STR, trace, (size_t)e0, ne, lane, false);
  const int* nbr = slot;
  const int* code = slot + TE * NF;
  // one neighbour record (CH pieces) per lane and round
#pragma unroll
  for (int lf0 = 0; lf0 < TE * NF; lf0 += 32) {
    const int lf = lf0 + lane;
    if (lf < TE * NF) {
      const int el = lf / NF, f = lf % NF;
      const int nb = nbr[lf];
      if (el < ne && nb >= 0) {
        const int fr = (code[el] >> (8 * f)) & 3;
        T* d = w + L::SNB + el * TS + f * TR;
        const T* src = trace + ((size_t)nb * NF + fr) * TR;
#pragma unroll
        for (int c = 0; c < CH; ++c) cp_async_n<16>(d + c * VPC, src + c * VPC, 16);
      }
    }
  }
}

// 1/sqrt: the hardware approximation in FP32 (the TF32 path tolerates its ulps), exact in FP64.
__device__ __forceinline__ float inv_sqrt(float v) { return rsqrtf(v); }
__device__ __forceinline__ double inv_sqrt(double v) { return 1.0 / sqrt(v); }

// sJ and c_r = n . grad r of face f (n the outward unit normal) from the geometric factors g.
template <typename T, int DIM>
__device__ __forceinline__ void face_geom(const T* g, int f, T& sJ, T (&c)[3]) {
  T n[3];
  if (DIM == 3) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      T v;
      if (f == 0) v = -g[6 + d];
      else if (f == 1) v = -g[3 + d];
      else if (f == 2) v = (g[d] + g[3 + d]) + g[6 + d];
      else v = -g[d];
      n[d] = v;
    }
    const T len2 = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    const T inv = inv_sqrt(len2);
    n[0] *= inv; n[1] *= inv; n[2] *= inv;
    sJ = len2 * inv * g[9];
  } else {
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      T v;
      if (f == 0) v = -g[2 + d];
      else if (f == 1) v = g[d] + g[2 + d];
      else v = -g[d];
      n[d] = v;
    }
    n[2] = T(0);
    const T len2 = n[0] * n[0] + n[1] * n[1];
    const T inv = inv_sqrt(len2);
    n[0] *= inv; n[1] *= inv;
    sJ = len2 * inv * g[4];
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    T cr = T(0);
    if (r < DIM)
#pragma unroll
      for (int d = 0; d < DIM; ++d) cr += n[d] * g[r * DIM + d];
    c[r] = cr;
  }
}

template <typename T, int DIM, int P>
__device__ __forceinline__ T fgeo(const T* sfg, int q, int f, int el) {
  using X = Tc<T, DIM, P>;
  return sfg[(q * X::NF + f) * X::TE + el];
}

// Zero the padding columns (Np .. XS-1) of the x and factor rows of `nst` element
// stages `stride` values apart: the fragment loads read them and the copies never
// write them. Nothing else in a warp area is read before it is written.
template <typename T, int DIM, int P>
__device__ __forceinline__ void zero_row_padding(T* W, int nst, int stride, int lane) {
  using X = Tc<T, DIM, P>;
  constexpr int PAD = X::XS - X::NP, TE = X::TE;
  if (PAD == 0) return;
  for (int i = lane; i < nst * 2 * TE * PAD; i += 32) {
    const int row = i / PAD, c = i % PAD;  // row over (stage, x rows then factor rows)
    W[(row / (2 * TE)) * stride + (row % (2 * TE)) * X::XS + X::NP + c] = T(0);
  }
}

// A blocks of x: u[kb][ri][ci] = x[g + 8 ri][8 kb + 2t + ci]
// (staged rows are zero past Np).
template <typename T, int DIM, int P>
__device__ __forceinline__ void load_x_frags(const T* sx, T (&u)[Tc<T, DIM, P>::NT][Frag<T>::R][2], int g, int t) {
  using X = Tc<T, DIM, P>;
#pragma unroll
  for (int kb = 0; kb < X::NT; ++kb)
#pragma unroll
    for (int ri = 0; ri < X::R; ++ri) {
      const auto v = ld2(sx + (g + 8 * ri) * X::XS + 8 * kb + 2 * t);
      u[kb][ri][0] = Frag<T>::op(v.x);
      u[kb][ri][1] = Frag<T>::op(v.y);
    }
}

// ---------------------------------------------------------------- pass 1
template <typename T, int DIM, int P, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 1) sipg_trace_kernel(ApplyArgs<T> a, const T* __restrict__ blob,
                                                                 T* __restrict__ trace) {
  using X = Tc<T, DIM, P>;
  using F = Frag<T>;
  using V2 = typename F::V2;
  constexpr int NFP = X::NFP, NF = X::NF, NT = X::NT, FT = X::FT, R = X::R, TE = X::TE, TR = X::TR, KF = X::KF,
                XS = X::XS, TS = X::TS, TRP = X::TRP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* BFs = reinterpret_cast<T*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  T* W = BFs + X::N1 + warp * X::W1_T;
  int8_t* fmask = reinterpret_cast<int8_t*>(BFs + X::N1 + WARPS * X::W1_T);
  T* sout = W + 2 * X::ST1;
  const int ntiles = (a.K + TE - 1) / TE;
  const int stride = gridDim.x * WARPS;
  // warp-major tile order: the last, partial round of tiles is spread over all
  // CTAs (SMs) instead of filling the first ones
  int tile = warp * gridDim.x + blockIdx.x;
  pdl_trigger();
  zero_row_padding<T, DIM, P>(W, 2, X::ST1, lane);
  for (int i = threadIdx.x; i < X::N1; i += blockDim.x) BFs[i] = blob[X::BF + i];
  for (int i = threadIdx.x; i < NF * NFP; i += blockDim.x) fmask[i] = a.itab[i];
  pdl_wait();  // x, factor and the trace buffer belong to the preceding kernels
  __syncwarp();
  issue_elem<T, DIM, P>(a, W, tile, lane, false);
  cp_commit();
  __syncthreads();
  for (int it = 0; tile < ntiles; ++it, tile += stride) {
    T* st = W + (it & 1) * X::ST1;
    cp_wait_all();
    __syncwarp();
    issue_elem<T, DIM, P>(a, W + ((it & 1) ^ 1) * X::ST1, tile + stride, lane, false);
    cp_commit();
    const int e0 = tile * TE;
    const int ne = min(TE, a.K - e0);
    T* sx = st + X::SX;
    const T* sf = st + X::SF;
    const T* sfg = st + X::SG;  // face rows of the geometry block
    if (lane == 0 && a.pin_elem >= e0 && a.pin_elem < e0 + ne) sx[(a.pin_elem - e0) * XS + a.pin_node] = T(0);
    __syncwarp();
    T u[NT][R][2];
    load_x_frags<T, DIM, P>(sx, u, g, t);
#pragma unroll
    for (int fb = 0; fb < FT; ++fb) {
      T acc[DIM][R][2];
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int ri = 0; ri < R; ++ri) acc[r][ri][0] = acc[r][ri][1] = T(0);
#pragma unroll
      for (int kb = 0; kb < NT; ++kb)
#pragma unroll
        for (int r = 0; r < DIM; ++r) F::mma(acc[r], u[kb], ldb(BFs, (r * NT + kb) * FT + fb, lane));
      if constexpr (NFP % 2 == 0) {
        // the two columns of a lane lie on one face
        const int k0 = 8 * fb + 2 * t;
        if (k0 < KF) {
          const int f = k0 / NFP, j0 = k0 % NFP;
          const int m0 = fmask[k0], m1 = fmask[k0 + 1];
#pragma unroll
          for (int ri = 0; ri < R; ++ri) {
            const int el = g + 8 * ri;
            T s0 = T(0), s1 = T(0);
#pragma unroll
            for (int r = 0; r < DIM; ++r) {
              const T c = fgeo<T, DIM, P>(sfg, 1 + r, f, el);
              s0 += c * acc[r][ri][0];
              s1 += c * acc[r][ri][1];
            }
            const T* xr = sx + el * XS;
            const T fm0 = a.factor ? sf[el * XS + m0] : T(1), fm1 = a.factor ? sf[el * XS + m1] : T(1);
            T* rec = sout + el * TS + f * TR;
            *reinterpret_cast<V2*>(rec + j0) = V2{xr[m0], xr[m1]};
            *reinterpret_cast<V2*>(rec + TRP + j0) = V2{fm0 * s0, fm1 * s1};
          }
        }
      } else {
#pragma unroll
        for (int ri = 0; ri < R; ++ri)
#pragma unroll
          for (int ci = 0; ci < 2; ++ci) {
            const int k = 8 * fb + 2 * t + ci;
            if (k < KF) {
              const int el = g + 8 * ri;
              const int f = k / NFP, j = k % NFP;
              const int m = fmask[k];
              T s = T(0);
#pragma unroll
              for (int r = 0; r < DIM; ++r) s += fgeo<T, DIM, P>(sfg, 1 + r, f, el) * acc[r][ri][ci];
              const T fm = a.factor ? sf[el * XS + m] : T(1);
              T* rec = sout + el * TS + f * TR;
              rec[j] = sx[el * XS + m];
              rec[TRP + j] = fm * s;
            }
          }
      }
    }
    __syncwarp();
    // coalesced write-out of the tile's records
    {
      using V4 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
      constexpr int VPC = 16 / sizeof(T), CPE = NF * X::CH;
      const int n = ne * CPE;
      for (int i = lane; i < n; i += 32) {
        const int el = i / CPE, c = i % CPE;
        *reinterpret_cast<V4*>(trace + (size_t)(e0 + el) * NF * TR + c * VPC) =
            *reinterpret_cast<const V4*>(sout + el * TS + c * VPC);
      }
    }
    __syncwarp();
  }
  cp_wait_all();
}

// ---------------------------------------------------------------- pass 2
// NS = 2: the next tile's element data is fetched during the whole current tile
// (double-buffered stage); NS = 1: after the current tile's fluxes, which frees
// shared memory for more warps per SM.
template <typename T, int DIM, int P, int WARPS, int NS>
__global__ void __launch_bounds__(WARPS * 32, 1) sipg_apply_tc_kernel(ApplyArgs<T> a, const T* __restrict__ blob,
                                                                    const T* __restrict__ trace) {
  using X = Tc<T, DIM, P>;
  using L = W2<T, DIM, P, NS>;
  using F = Frag<T>;
  constexpr int NP = X::NP, NFP = X::NFP, NF = X::NF, NT = X::NT, FT = X::FT, R = X::R, TE = X::TE, TR = X::TR,
                KF = X::KF, TRP = X::TRP, XS = X::XS, TS = X::TS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* B = reinterpret_cast<T*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  T* W = B + X::N2 + warp * L::T_;
  int* ibase = reinterpret_cast<int*>(B + X::N2 + WARPS * L::T_);
  int* I = ibase + warp * X::W2_I;
  int8_t* itab = reinterpret_cast<int8_t*>(ibase + WARPS * X::W2_I);
  const int8_t* fmask = itab;
  const int8_t* perm = itab + NF * NFP;
  const T* str = W + L::STR;
  const T* snb = W + L::SNB;
  const int ntiles = (a.K + TE - 1) / TE;
  const int stride = gridDim.x * WARPS;
  // warp-major tile order: the last, partial round of tiles is spread over all
  // CTAs (SMs) instead of filling the first ones
  int tile = warp * gridDim.x + blockIdx.x;
  pdl_trigger();
  zero_row_padding<T, DIM, P>(W, NS, X::ST2, lane);
  __syncwarp();
  // prologue: constants and the connectivity of the first two tiles (set-up data),
  // then, once the preceding kernels are done, the first tile's element data
  issue_ints<T, DIM, P>(a, I, tile, lane);
  issue_ints<T, DIM, P>(a, I + X::SI, tile + stride, lane);
  for (int i = threadIdx.x; i < X::N2; i += blockDim.x) B[i] = blob[i];
  for (int i = threadIdx.x; i < Cfg<DIM, P>::ITAB; i += blockDim.x) itab[i] = a.itab[i];
  pdl_wait();
  issue_elem<T, DIM, P>(a, W, tile, lane, true);
  cp_commit();
  __syncthreads();
  cp_wait_all();
  __syncwarp();
  issue_traces<T, DIM, P, NS>(a, trace, W, I, tile, lane);
  cp_commit();
  // this lane's face-node columns per block: face | node in face << 4 | volume nodes << 10, << 18
  int fbi[FT];
#pragma unroll
  for (int fb = 0; fb < FT; ++fb) {
    const int k0 = 8 * fb + 2 * t;
    fbi[fb] = -1;
    if (NFP % 2 == 0 && k0 < KF) fbi[fb] = (k0 / NFP) | ((k0 % NFP) << 4) | (fmask[k0] << 10) | (fmask[k0 + 1] << 18);
  }
  for (int it = 0; tile < ntiles; ++it, tile += stride) {
    const int sb = NS == 2 ? (it & 1) : 0, slot = it % 3;
    T* st = W + sb * X::ST2;
    const int* ints = I + slot * X::SI;
    // element data of this tile and connectivity of the next one have arrived (the
    // tile's trace records, issued after the previous tile's fluxes, may still be in flight)
    cp_wait_but_one();
    __syncwarp();
    if (NS == 2) {
      issue_ints<T, DIM, P>(a, I + ((it + 2) % 3) * X::SI, tile + 2 * stride, lane);
      issue_elem<T, DIM, P>(a, W + (sb ^ 1) * X::ST2, tile + stride, lane, true);
      cp_commit();
    }

    const int e0 = tile * TE;
    const int ne = min(TE, a.K - e0);
    T* sx = st + X::SX;
    const T* sf = st + X::SF;
    const T* sg = st + X::SG;
    const T* stau = st + X::STAU;
    const int* snbr = ints;
    const int* scode = ints + TE * NF;
    if (lane == 0 && a.pin_elem >= e0 && a.pin_elem < e0 + ne) sx[(a.pin_elem - e0) * XS + a.pin_node] = T(0);
    // c values read by the epilogue (beta != 0), loaded now so that their latency
    // hides behind the tile's products
    T yold[NT][R][2];
    if (a.beta != T(0)) {
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int ri = 0; ri < R; ++ri) {
          const int el = g + 8 * ri, n0 = 8 * nt + 2 * t;
          const T* crow = a.c + (size_t)(e0 + el) * NP;
          if (NP % 2 == 0) {  // node pairs (n0, n0 + 1) are aligned
            typename F::V2 v{T(0), T(0)};
            if (el < ne && n0 < NP) v = ld2(crow + n0);
            yold[nt][ri][0] = v.x;
            yold[nt][ri][1] = v.y;
          } else {
#pragma unroll
            for (int ci = 0; ci < 2; ++ci) yold[nt][ri][ci] = (el < ne && n0 + ci < NP) ? crow[n0 + ci] : T(0);
          }
        }
    }
    const T* sfg = sg + X::NV * TE;  // face rows of the geometry block
    __syncwarp();

    // metric of the lane's elements: J and K = G G^T
    T Jm[R], Km[R][DIM][DIM];
#pragma unroll
    for (int ri = 0; ri < R; ++ri) {
      const int el = g + 8 * ri;
      Jm[ri] = sg[el];
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int s = r; s < DIM; ++s) {
          const T v = sg[kidx(DIM, r, s) * TE + el];
          Km[ri][r][s] = v;
          Km[ri][s][r] = v;
        }
    }

    // gr_r = x . B1_r
    T w[DIM][NT][R][2];
    {
      T u[NT][R][2];
      load_x_frags<T, DIM, P>(sx, u, g, t);
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
          for (int ri = 0; ri < R; ++ri) w[r][nt][ri][0] = w[r][nt][ri][1] = T(0);
#pragma unroll
      for (int kb = 0; kb < NT; ++kb)
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) F::mma(w[r][nt], u[kb], ldb(B + X::B1, (r * NT + kb) * NT + nt, lane));
    }
    // w_r = J f sum_s K_rs gr_s (A blocks of the next product)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int ri = 0; ri < R; ++ri) {
        const int el = g + 8 * ri;
        T fJ[2] = {Jm[ri], Jm[ri]};
        if (a.factor) {
          const auto fv = ld2(sf + el * XS + 8 * nt + 2 * t);
          fJ[0] *= fv.x;
          fJ[1] *= fv.y;
        }
#pragma unroll
        for (int ci = 0; ci < 2; ++ci) {
          T gr[DIM];
#pragma unroll
          for (int s = 0; s < DIM; ++s) gr[s] = w[s][nt][ri][ci];
#pragma unroll
          for (int r = 0; r < DIM; ++r) {
            T v = T(0);
#pragma unroll
            for (int s = 0; s < DIM; ++s) v += Km[ri][r][s] * gr[s];
            w[r][nt][ri][ci] = F::op(fJ[ci] * v);
          }
        }
      }
    // Z_r = w_r . M^T ; y = (J mm x) . M^T
    T z[DIM][NT][R][2], y[NT][R][2];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int ri = 0; ri < R; ++ri) {
        y[nt][ri][0] = y[nt][ri][1] = T(0);
#pragma unroll
        for (int r = 0; r < DIM; ++r) z[r][nt][ri][0] = z[r][nt][ri][1] = T(0);
      }
    const bool has_mm = a.mm_mode != MM_NONE;
#pragma unroll
    for (int kb = 0; kb < NT; ++kb) {
      T mx[R][2];
      if (has_mm) {
#pragma unroll
        for (int ri = 0; ri < R; ++ri)
#pragma unroll
          for (int ci = 0; ci < 2; ++ci) {
            const int el = g + 8 * ri, m = 8 * kb + 2 * t + ci;
            T v = T(0);
            if (m < NP && el < ne) {
              const T mmv = a.mm_mode == MM_SCALAR ? a.mm_scalar : a.mm[(size_t)(e0 + el) * NP + m];
              v = Jm[ri] * mmv * sx[el * XS + m];
            }
            mx[ri][ci] = F::op(v);
          }
      }
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const auto b = ldb(B + X::BM, kb * NT + nt, lane);
#pragma unroll
        for (int r = 0; r < DIM; ++r) F::mma(z[r][nt], w[r][kb], b);
        if (has_mm) F::mma(y[nt], mx, b);
      }
    }
    // the tile's trace records have arrived
    if (NS == 2) cp_wait_but_one();
    else cp_wait_all();
    __syncwarp();
    // face fluxes: y += Fu . EMAT^T ; Z_r += (c_r S) . EMAT^T
#pragma unroll
    for (int fb = 0; fb < FT; ++fb) {
      T fu[R][2], sv[DIM][R][2];
      if constexpr (NFP % 2 == 0) {
        // the two columns of a lane lie on one face
        const int fi = fbi[fb];
        const int f = fi & 15, j0 = (fi >> 4) & 63, m0 = (fi >> 10) & 255, m1 = (fi >> 18) & 255;
#pragma unroll
        for (int ri = 0; ri < R; ++ri) {
          const int el = g + 8 * ri;
          T vfu[2] = {T(0), T(0)}, vs[2] = {T(0), T(0)}, cr[DIM];
#pragma unroll
          for (int r = 0; r < DIM; ++r) cr[r] = T(0);
          if (fi >= 0 && el < ne) {
            const int lf = el * NF + f;
            const T* own = str + el * TS + f * TR;
            const auto um = ld2(own + j0);
            const auto gm = ld2(own + TRP + j0);
            const int nb = snbr[lf];
            T jump[2] = {T(0), T(0)}, navg[2] = {T(0), T(0)};
            if (nb >= 0) {
              const int8_t* pr = perm + ((scode[el] >> (8 * f + 2)) & 7) * NFP + j0;
              const T* rec = snb + el * TS + f * TR;
              const int kk0 = pr[0], kk1 = pr[1];
              jump[0] = um.x - rec[kk0];
              jump[1] = um.y - rec[kk1];
              navg[0] = T(0.5) * (gm.x - rec[TRP + kk0]);
              navg[1] = T(0.5) * (gm.y - rec[TRP + kk1]);
            } else if (a.bct[-nb - 1] == BC_DIRICHLET) {
              jump[0] = T(2) * um.x;
              jump[1] = T(2) * um.y;
              navg[0] = gm.x;
              navg[1] = gm.y;
            }
            const T sJ = fgeo<T, DIM, P>(sfg, 0, f, el);
#pragma unroll
            for (int r = 0; r < DIM; ++r) cr[r] = fgeo<T, DIM, P>(sfg, 1 + r, f, el);
            const T tau = stau[lf];
            const T fm0 = a.factor ? sf[el * XS + m0] : T(1);
            const T fm1 = a.factor ? sf[el * XS + m1] : T(1);
            const T h0 = T(0.5) * jump[0], h1 = T(0.5) * jump[1];
            vfu[0] = sJ * (tau * h0 - navg[0]);
            vfu[1] = sJ * (tau * h1 - navg[1]);
            vs[0] = -sJ * fm0 * h0;
            vs[1] = -sJ * fm1 * h1;
          }
#pragma unroll
          for (int ci = 0; ci < 2; ++ci) {
            fu[ri][ci] = F::op(vfu[ci]);
#pragma unroll
            for (int r = 0; r < DIM; ++r) sv[r][ri][ci] = F::op(cr[r] * vs[ci]);
          }
        }
      } else {
#pragma unroll
        for (int ri = 0; ri < R; ++ri)
#pragma unroll
          for (int ci = 0; ci < 2; ++ci) {
            const int el = g + 8 * ri, k = 8 * fb + 2 * t + ci;
            T vfu = T(0), vs = T(0), cr[DIM];
#pragma unroll
            for (int r = 0; r < DIM; ++r) cr[r] = T(0);
            if (k < KF && el < ne) {
              const int f = k / NFP, j = k % NFP;
              const int lf = el * NF + f;
              const T* own = str + el * TS + f * TR;
              const T um = own[j], gm = own[TRP + j];
              const int nb = snbr[lf];
              T jump = T(0), navg = T(0);
              if (nb >= 0) {
                const int kk = perm[((scode[el] >> (8 * f + 2)) & 7) * NFP + j];
                const T* rec = snb + el * TS + f * TR;
                jump = um - rec[kk];
                navg = T(0.5) * (gm - rec[TRP + kk]);
              } else if (a.bct[-nb - 1] == BC_DIRICHLET) {
                jump = T(2) * um;
                navg = gm;
              }
              const T hj = T(0.5) * jump;
              const T sJ = fgeo<T, DIM, P>(sfg, 0, f, el);
              const T fm = a.factor ? sf[el * XS + fmask[k]] : T(1);
              vfu = sJ * (stau[lf] * hj - navg);
              vs = -sJ * fm * hj;
#pragma unroll
              for (int r = 0; r < DIM; ++r) cr[r] = fgeo<T, DIM, P>(sfg, 1 + r, f, el);
            }
            fu[ri][ci] = F::op(vfu);
#pragma unroll
            for (int r = 0; r < DIM; ++r) sv[r][ri][ci] = F::op(cr[r] * vs);
          }
      }
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const auto b = ldb(B + X::BE, fb * NT + nt, lane);
        F::mma(y[nt], fu, b);
#pragma unroll
        for (int r = 0; r < DIM; ++r) F::mma(z[r][nt], sv[r], b);
      }
    }
    // the trace buffer (and with NS = 1 the element stage) is free: the next tile's
    // data lands during the rest of this tile and the next tile's volume products
    __syncwarp();
    if (NS == 1) {
      issue_ints<T, DIM, P>(a, I + ((it + 2) % 3) * X::SI, tile + 2 * stride, lane);
      issue_elem<T, DIM, P>(a, W, tile + stride, lane, true);
      cp_commit();
    }
    issue_traces<T, DIM, P, NS>(a, trace, W, I + ((it + 1) % 3) * X::SI, tile + stride, lane);
    cp_commit();
    // y += sum_r Z_r . D_r
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
      for (int kb = 0; kb < NT; ++kb) {
        T zr[R][2];
#pragma unroll
        for (int ri = 0; ri < R; ++ri) {
          zr[ri][0] = F::op(z[r][kb][ri][0]);
          zr[ri][1] = F::op(z[r][kb][ri][1]);
        }
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) F::mma(y[nt], zr, ldb(B + X::B3, (r * NT + kb) * NT + nt, lane));
      }
    // epilogue: pinned row, alpha / beta, store (pairs of nodes when Np is even)
    const bool pin_here = a.pin_elem >= e0 && a.pin_elem < e0 + ne;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int ri = 0; ri < R; ++ri) {
        const int el = g + 8 * ri;
        if (el >= ne) continue;
        const size_t row = (size_t)(e0 + el) * NP;
        T acc[2];
#pragma unroll
        for (int ci = 0; ci < 2; ++ci) {
          const int n = 8 * nt + 2 * t + ci;
          acc[ci] = y[nt][ri][ci];
          if (pin_here && e0 + el == a.pin_elem && n == a.pin_node) acc[ci] = a.pin_scale * a.x[row + n];
          acc[ci] *= a.alpha;
          if (a.beta != T(0)) acc[ci] += a.beta * yold[nt][ri][ci];
        }
        const int n0 = 8 * nt + 2 * t;
        if (NP % 2 == 0) {
          if (n0 < NP) *reinterpret_cast<typename F::V2*>(a.y + row + n0) = typename F::V2{acc[0], acc[1]};
        } else {
          if (n0 < NP) a.y[row + n0] = acc[0];
          if (n0 + 1 < NP) a.y[row + n0 + 1] = acc[1];
        }
      }
    __syncwarp();
  }
  cp_wait_all();
}

// Geometry blocks of the tensor-core apply, one thread per element slot of a
// warp tile: J, the metric K = G G^T and per face sJ and c_r = n . grad r (the
// same arithmetic for every apply, so it is done once per mesh).
template <typename T, int DIM, int TE>
__global__ void k_tc_geom(const T* __restrict__ geof, int K, T* __restrict__ out) {
  constexpr int NF = DIM + 1, NG = DIM == 3 ? 10 : 5, NV = 8, NFG = 4, GROWS = NV + NFG * NF;
  const int ntiles = (K + TE - 1) / TE;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ntiles * TE; e += gridDim.x * blockDim.x) {
    T v[GROWS];
#pragma unroll
    for (int i = 0; i < GROWS; ++i) v[i] = T(0);
    if (e < K) {
      const T* g = geof + (size_t)e * NG;
      v[0] = g[DIM * DIM];
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int s = r; s < DIM; ++s) {
          T k = T(0);
#pragma unroll
          for (int d = 0; d < DIM; ++d) k += g[r * DIM + d] * g[s * DIM + d];
          v[kidx(DIM, r, s)] = k;
        }
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        T sJ, c[3];
        face_geom<T, DIM>(g, f, sJ, c);
        v[NV + f] = sJ;
#pragma unroll
        for (int r = 0; r < 3; ++r) v[NV + (1 + r) * NF + f] = c[r];
      }
    }
    T* o = out + (size_t)(e / TE) * GROWS * TE + e % TE;
#pragma unroll
    for (int i = 0; i < GROWS; ++i) o[(size_t)i * TE] = v[i];
  }
}

constexpr int kSmemBudget = 227 * 1024;

template <typename T, int DIM, int P>
constexpr size_t smem1(int w) {
  using X = Tc<T, DIM, P>;
  return (size_t)(X::N1 + w * X::W1_T) * sizeof(T) + X::NF * X::NFP;
}
template <typename T, int DIM, int P, int NS>
constexpr size_t smem2(int w) {
  using X = Tc<T, DIM, P>;
  return (size_t)(X::N2 + w * W2<T, DIM, P, NS>::T_) * sizeof(T) + (size_t)w * X::W2_I * 4 + Cfg<DIM, P>::ITAB;
}
template <typename T, int DIM, int P>
constexpr int warps1() {
  int w = 16;
  while (w > 1 && smem1<T, DIM, P>(w) > (size_t)kSmemBudget) --w;
  return w;
}
// 0 when not even one warp tile fits next to the constants
template <typename T, int DIM, int P, int NS>
constexpr int warps2() {
  int w = 16;
  while (w > 0 && smem2<T, DIM, P, NS>(w) > (size_t)kSmemBudget) --w;
  return w;
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <typename T, int DIM, int P, int WARPS>
cudaError_t launch_pass1(const ApplyArgs<T>& a, const T* blob, T* trace, int ntiles, int num_sms, cudaStream_t s) {
  static_assert(WARPS >= 1 && smem1<T, DIM, P>(WARPS) <= (size_t)kSmemBudget, "pass-1 warps do not fit");
  auto k = sipg_trace_kernel<T, DIM, P, WARPS>;
  const size_t bytes = smem1<T, DIM, P>(WARPS);
  cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (err != cudaSuccess) return err;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, WARPS * 32, bytes);
  const int grid = std::min((ntiles + WARPS - 1) / WARPS, num_sms * std::max(per_sm, 1));
  if (grid > 0) {
    pdl_launch(k, dim3(grid), dim3(WARPS * 32), bytes, s, a, blob, trace);
    note_launch();
  }
  return cudaSuccess;
}

template <typename T, int DIM, int P, int NS, int WARPS>
cudaError_t launch_pass2(const ApplyArgs<T>& a, const T* blob, const T* trace, int ntiles, int num_sms,
                         cudaStream_t s) {
  static_assert(WARPS >= 1 && smem2<T, DIM, P, NS>(WARPS) <= (size_t)kSmemBudget, "pass-2 warps do not fit");
  auto k = sipg_apply_tc_kernel<T, DIM, P, WARPS, NS>;
  const size_t bytes = smem2<T, DIM, P, NS>(WARPS);
  cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (err != cudaSuccess) return err;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, WARPS * 32, bytes);
  const int grid = std::min((ntiles + WARPS - 1) / WARPS, num_sms * std::max(per_sm, 1));
  if (grid > 0) {
    pdl_launch(k, dim3(grid), dim3(WARPS * 32), bytes, s, a, blob, trace);
    note_launch();
  }
  return cudaSuccess;
}

constexpr int cmin(int a, int b) { return a < b ? a : b; }

// Launch shapes by the number of warp tiles: large meshes run as many warps per SM
// as shared memory allows (pass 2 single-buffered once every warp has at least two
// tiles); meshes with fewer tiles than a full-width wave over the SMs use narrow
// CTAs (4 or 2 warps), so that every SM gets work.
template <typename T, int DIM, int P>
cudaError_t launch_tc_t(const ApplyArgs<T>& a, const T* blob, T* trace, int num_sms, cudaStream_t s) {
  constexpr int WA = warps1<T, DIM, P>(), W2D = warps2<T, DIM, P, 2>(), W2S = warps2<T, DIM, P, 1>();
  if (W2D < 1) return cudaErrorInvalidConfiguration;
  using X = Tc<T, DIM, P>;
  if constexpr (std::is_same<T, float>::value) {
    // FP32: the tcgen05 kernels (their constants follow the mma.sync blob)
    if (a.tcgen05 && tc5_supported(DIM, P)) return launch_apply_tc5(DIM, P, a, blob + X::NALL, trace, num_sms, s);
  }
  // the kernels copy caller vectors in 16-byte pieces: other alignments take the CUDA-core kernel
  if (!aligned16(a.x) || !aligned16(a.y) || !aligned16(trace) || (a.factor && !aligned16(a.factor)) ||
      (a.beta != T(0) && !aligned16(a.c)))
    return launch_apply<T>(DIM, P, a, num_sms, s);
  const int ntiles = (a.K + X::TE - 1) / X::TE;
  const long long wave = (long long)num_sms;
  cudaError_t err;
  // pass 1 on large meshes: at most 12 warps per SM. It is latency-bound, so the
  // time goes with the number of tile rounds; at 24^3 x 6 tets (35 tiles per SM in
  // FP32, 70 in FP64) 12 warps give full rounds where 15 or 16 leave a partial one
  if (ntiles >= wave * WA) err = launch_pass1<T, DIM, P, cmin(12, WA)>(a, blob, trace, ntiles, num_sms, s);
  else if (ntiles >= wave * 4) err = launch_pass1<T, DIM, P, cmin(4, WA)>(a, blob, trace, ntiles, num_sms, s);
  else err = launch_pass1<T, DIM, P, cmin(2, WA)>(a, blob, trace, ntiles, num_sms, s);
  if (err != cudaSuccess) return err;
  if (W2S > W2D && ntiles >= 2 * wave * W2S) err = launch_pass2<T, DIM, P, 1, (W2S > W2D ? W2S : W2D)>(a, blob, trace, ntiles, num_sms, s);
  else if (ntiles >= wave * W2D) err = launch_pass2<T, DIM, P, 2, W2D>(a, blob, trace, ntiles, num_sms, s);
  else if (ntiles >= wave * 4) err = launch_pass2<T, DIM, P, 2, cmin(4, W2D)>(a, blob, trace, ntiles, num_sms, s);
  else err = launch_pass2<T, DIM, P, 2, cmin(2, W2D)>(a, blob, trace, ntiles, num_sms, s);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

// Host construction of the constant blob in fragment order (FP64 values).
template <typename T, int DIM, int P>
void build_tc_consts_t(const RefElement& r, std::vector<double>& out) {
  using X = Tc<T, DIM, P>;
  constexpr int NP = X::NP, NT = X::NT, FT = X::FT, KF = X::KF;
  out.assign(X::NALL, 0.0);
  // entry (row, col) of a logical matrix stored as 8 x 8 blocks, nblk_n blocks per block row
  auto put = [&](int base, int nblk_n, int row, int col, double v) {
    const int kb = row / 8, kr = row % 8, nt = col / 8, gg = col % 8;
    const int lane = gg * 4 + kr / 2;
    out[(size_t)base + ((size_t)(kb * nblk_n + nt) * 32 + lane) * 2 + (kr % 2)] = v;
  };
  const double* D[3] = {r.Dr.data(), r.Ds.data(), r.Dt.data()};
  for (int rr = 0; rr < DIM; ++rr)
    for (int m = 0; m < NP; ++m)
      for (int n = 0; n < NP; ++n) {
        put(X::B1 + rr * NT * NT * X::BLK, NT, n, m, D[rr][m * NP + n]);  // B1_r[n][m] = D_r[m][n]
        put(X::B3 + rr * NT * NT * X::BLK, NT, m, n, D[rr][m * NP + n]);  // B3_r[m][n] = D_r[m][n]
      }
  for (int m = 0; m < NP; ++m)
    for (int n = 0; n < NP; ++n) put(X::BM, NT, m, n, r.M[n * NP + m]);     // BM[m][n] = M[n][m]
  for (int k = 0; k < KF; ++k)
    for (int n = 0; n < NP; ++n) put(X::BE, NT, k, n, r.EMAT[n * KF + k]);  // BE[k][n] = EMAT[n][k]
  for (int rr = 0; rr < DIM; ++rr)
    for (int n = 0; n < NP; ++n)
      for (int k = 0; k < KF; ++k)
        put(X::BF + rr * NT * FT * X::BLK, FT, n, k, D[rr][r.fmask[k] * NP + n]);  // BF_r[n][k] = D_r[m(k)][n]
  if (std::is_same<T, float>::value) {
    std::vector<double> t5;  // empty where the order has no tcgen05 kernels
    build_tc5_consts(DIM, P, r, t5);
    out.insert(out.end(), t5.begin(), t5.end());
  }
}

}  // namespace

#define SIPG_DISPATCH_TC(DIM_, ORDER_, ...)                        \
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

template <typename T>
cudaError_t launch_apply_tc(int dim, int order, const ApplyArgs<T>& a, const T* tc_consts, T* trace,
                            int num_sms, cudaStream_t s) {
  SIPG_DISPATCH_TC(dim, order, return (launch_tc_t<T, D, P>(a, tc_consts, trace, num_sms, s)));
  return cudaErrorInvalidValue;
}

template <typename T>
void build_tc_consts(int dim, int order, const RefElement& r, std::vector<double>& out) {
  SIPG_DISPATCH_TC(dim, order, build_tc_consts_t<T, D, P>(r, out); return);
}

template <typename T>
int tc_warps_for(int dim, int order) {
  SIPG_DISPATCH_TC(dim, order, return warps2<T, D, P, 2>());
  return 0;
}

template <typename T>
size_t tc_geom_values(int dim, int K) {
  constexpr int TE = 8 * Frag<T>::R;
  const size_t ntiles = ((size_t)K + TE - 1) / TE;
  return ntiles * TE * (8 + 4 * (dim + 1));
}

template <typename T>
cudaError_t launch_tc_geom(int dim, const T* geof, int K, T* out, cudaStream_t s) {
  constexpr int TE = 8 * Frag<T>::R;
  const size_t n = ((size_t)K + TE - 1) / TE * TE;
  const int grid = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  if (grid == 0) return cudaSuccess;
  if (dim == 3) k_tc_geom<T, 3, TE><<<grid, 256, 0, s>>>(geof, K, out);
  else if (dim == 2) k_tc_geom<T, 2, TE><<<grid, 256, 0, s>>>(geof, K, out);
  else return cudaErrorInvalidValue;
  note_launch();
  return cudaGetLastError();
}

size_t tc_trace_values(int dim, int order, int K) {
  const int trp = rup(nfp_of(dim, order), 2);
  return (size_t)K * (dim + 1) * rup(2 * trp, 4);
}

template cudaError_t launch_apply_tc<float>(int, int, const ApplyArgs<float>&, const float*, float*, int,
                                            cudaStream_t);
template cudaError_t launch_apply_tc<double>(int, int, const ApplyArgs<double>&, const double*, double*, int,
                                             cudaStream_t);
template void build_tc_consts<float>(int, int, const RefElement&, std::vector<double>&);
template void build_tc_consts<double>(int, int, const RefElement&, std::vector<double>&);
template int tc_warps_for<float>(int, int);
template int tc_warps_for<double>(int, int);
template size_t tc_geom_values<float>(int, int);
template size_t tc_geom_values<double>(int, int);
template cudaError_t launch_tc_geom<float>(int, const float*, int, float*, cudaStream_t);
template cudaError_t launch_tc_geom<double>(int, const double*, int, double*, cudaStream_t);

}  // namespace sipg
