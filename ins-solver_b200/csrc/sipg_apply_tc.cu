// Tensor-core SIPG apply (scalar operator): FP32 data on TF32 tensor cores or
// FP64 data on the FP64 tensor cores, in two passes over the elements.
//
// Same operator as sipg_apply.cu (FactorViscousMatrix3D::mult,
// src/solvers/3d/slip_matrix/factor_viscous_matrix.cpp:96-310, one component).
// The reference exchanges face data through 12 face buffers per component
// (mesh->jump / mesh->avg into K x Nf*Nfp op_dats); here each element publishes
// one trace record per face, and the matrix products are batched over elements:
//   pass 1 (traces): grad_ref = [D_r] x (G1, 3Np x Np), then per face node
//           u = x(m) and g = f(m) n.grad x(m) with the element's own outward
//           normal -> trace[e][f] = (u[0..Nfp), g[0..Nfp)) in the element's
//           face-node order. 2 Nf Nfp values per element, L2-resident between
//           the passes.
//   pass 2 (apply): G1 again for the own gradient; the neighbour's trace gives
//           u+ and n-.q+ = -g+ (n+ = -n-), so no neighbour volume data is read;
//           fluxes Fu = sJ (tau [u]/2 - n.{q}), Fq = -n sJ f [u]/2
//           (fvmf_3d_mult_flux.h:13-22), boundary traces as
//           vmf_3d_mult_avg_jump.h:43-80; then one product
//             y_e = A2 b_e,  A2 = [D_r^T M | D_r^T EMAT | EMAT | M]  (Np x K2)
//           with b_e = [q~_r | F~_r | Fu | J mm x], q~_r = J sum_d G[r][d] q_d,
//           F~_r = sum_d G[r][d] Fq_d (geometry folded into the data; D_r^T M
//           and D_r^T EMAT precomputed).
// Each warp owns a tile of 8 elements (the MMA N dimension) and synchronises at
// warp level only; the constant operands live in shared memory per CTA.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "sipg_apply.cuh"
#include "sipg_apply_tc.cuh"
#include "vecops.cuh"

namespace sipg {
namespace {

constexpr int kEl = 8;  // elements per warp tile (MMA N)

__host__ __device__ constexpr int rup(int x, int m) { return (x + m - 1) / m * m; }
// Leading dimensions congruent to 4 (mod 32) 32-bit words: fragment loads of a
// warp touch 32 distinct banks.
__host__ __device__ constexpr int ld32(int x) { return rup(x - 4, 32) + 4 >= x ? rup(x - 4, 32) + 4 : rup(x - 4, 32) + 36; }
__host__ __device__ constexpr int ld64(int x) { return rup(x - 4, 16) + 4 >= x ? rup(x - 4, 16) + 4 : rup(x - 4, 16) + 20; }

template <typename T>
struct Mma;

// m16n8k8 TF32 inputs, FP32 accumulate.
template <>
struct Mma<float> {
  static constexpr int MT = 16, KT = 8, NC = 4;
  using A = uint32_t[4];
  using B = uint32_t[2];
  __device__ static __forceinline__ float to_op(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
  }
  __device__ static __forceinline__ void load_a(A& a, const float* M, int lda, int m0, int k0, int lane) {
    const int g = lane >> 2, t = lane & 3;
    a[0] = __float_as_uint(M[(m0 + g) * lda + k0 + t]);
    a[1] = __float_as_uint(M[(m0 + g + 8) * lda + k0 + t]);
    a[2] = __float_as_uint(M[(m0 + g) * lda + k0 + t + 4]);
    a[3] = __float_as_uint(M[(m0 + g + 8) * lda + k0 + t + 4]);
  }
  __device__ static __forceinline__ void load_b(B& b, const float* S, int ldb, int k0, int lane) {
    const int g = lane >> 2, t = lane & 3;
    b[0] = __float_as_uint(S[g * ldb + k0 + t]);
    b[1] = __float_as_uint(S[g * ldb + k0 + t + 4]);
  }
  __device__ static __forceinline__ void mma(float* c, const A& a, const B& b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
  }
  // accumulator C[m][n] -> S[n][m]
  __device__ static __forceinline__ void store_c(const float* c, float* S, int lds, int m0, int lane) {
    const int g = lane >> 2, t = lane & 3;
    S[(2 * t) * lds + m0 + g] = c[0];
    S[(2 * t + 1) * lds + m0 + g] = c[1];
    S[(2 * t) * lds + m0 + g + 8] = c[2];
    S[(2 * t + 1) * lds + m0 + g + 8] = c[3];
  }
};

// m8n8k4 FP64.
template <>
struct Mma<double> {
  static constexpr int MT = 8, KT = 4, NC = 2;
  using A = double[1];
  using B = double[1];
  __device__ static __forceinline__ double to_op(double x) { return x; }
  __device__ static __forceinline__ void load_a(A& a, const double* M, int lda, int m0, int k0, int lane) {
    a[0] = M[(m0 + (lane >> 2)) * lda + k0 + (lane & 3)];
  }
  __device__ static __forceinline__ void load_b(B& b, const double* S, int ldb, int k0, int lane) {
    b[0] = S[(lane >> 2) * ldb + k0 + (lane & 3)];
  }
  __device__ static __forceinline__ void mma(double* c, const A& a, const B& b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a[0]), "d"(b[0]));
  }
  __device__ static __forceinline__ void store_c(const double* c, double* S, int lds, int m0, int lane) {
    const int g = lane >> 2, t = lane & 3;
    S[(2 * t) * lds + m0 + g] = c[0];
    S[(2 * t + 1) * lds + m0 + g] = c[1];
  }
};

// Asynchronous global -> shared copies (cp.async), zero-filled when !valid.
template <typename T>
__device__ __forceinline__ void cp_async(T* sdst, const T* gsrc, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  const int n = valid ? (int)sizeof(T) : 0;
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(n));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename T, int DIM, int P>
struct TcCfg {
  using C = Cfg<DIM, P>;
  using M = Mma<T>;
  static constexpr bool F32 = std::is_same<T, float>::value;
  static constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, NFNFP = C::NFNFP, NG = C::NG;
  static constexpr int TR = 2 * NFP;                       // trace record per face: u, g
  static constexpr int M1 = rup(DIM * NP, M::MT);
  static constexpr int K1 = rup(NP, M::KT);
  static constexpr int M2 = rup(NP, M::MT);
  // G2 in two K-chunks: A = [q~_r | Fu | J mm x], B = [F~_r]
  static constexpr int KA = rup(DIM * NP + NFNFP + NP, M::KT);
  static constexpr int KB = rup(DIM * NFNFP, M::KT);
  static constexpr int OFU = DIM * NP, OMM = DIM * NP + NFNFP;
  static constexpr int LDA1 = F32 ? ld32(K1) : ld64(K1);
  static constexpr int LDA2A = F32 ? ld32(KA) : ld64(KA);
  static constexpr int LDA2B = F32 ? ld32(KB) : ld64(KB);
  static constexpr int LDB = F32 ? ld32(KA > KB ? KA : KB) : ld64(KA > KB ? KA : KB);
  static constexpr int LDC = F32 ? ld32(M1 > M2 ? M1 : M2) : ld64(M1 > M2 ? M1 : M2);
  static constexpr int CONST1 = M1 * LDA1;
  static constexpr int CONST_T = M1 * LDA1 + M2 * LDA2A + M2 * LDA2B;
  static constexpr int FG = 8;  // per (element, face): n (3), sJ, c_r = n.grad r (3)
  // element-data stage (T units): x, factor, geof, tau; ints: nbr, fcode word.
  // x is read past its end by the G1 operand (K1 > NP columns meet zero A1
  // columns), so factor follows x directly and stays finite.
  static constexpr int ST_T = kEl * NP * 2 + kEl * NG + kEl * NF;
  static constexpr int ST_I = kEl * NF + kEl;
  static constexpr int TRB = kEl * NF * TR;  // neighbour traces of one tile
  // pass 1: 2 stages + G1 output + face geometry
  static constexpr int W1_T = 2 * ST_T + kEl * LDC + kEl * NF * FG;
  static constexpr int W1_I = 2 * ST_I;
  // pass 2: 3 stages, 2 trace buffers, operand, G1/G2 output, face geometry, flux scalars
  static constexpr int W2_T = 3 * ST_T + 2 * TRB + kEl * LDB + kEl * LDC + kEl * NF * FG + kEl * NFNFP;
  static constexpr int W2_I = 3 * ST_I;
};

template <typename T, int DIM, int P>
struct Stage {
  using TC = TcCfg<T, DIM, P>;
  T* x; T* fac; T* geo; T* tau; int* nbr; int* code;
  __device__ Stage(T* tb, int* ib) {
    x = tb; fac = x + kEl * TC::NP; geo = fac + kEl * TC::NP; tau = geo + kEl * TC::NG;
    nbr = ib; code = nbr + kEl * TC::NF;
  }
};

// Issue the element data of a tile (zero-filled past the last element).
template <typename T, int DIM, int P>
__device__ __forceinline__ void issue_own(const ApplyArgs<T>& a, const Stage<T, DIM, P>& st, int tile, int lane) {
  using TC = TcCfg<T, DIM, P>;
  constexpr int NP = TC::NP, NG = TC::NG, NF = TC::NF;
  const int e0 = tile * kEl;
  const int ne = max(0, min(kEl, a.K - e0));
  const T* fsrc = a.factor ? a.factor : a.x;
  for (int i = lane; i < kEl * NP; i += 32) {
    const bool v = i < ne * NP;
    cp_async(st.x + i, v ? a.x + (size_t)e0 * NP + i : a.x, v);
    cp_async(st.fac + i, (v && a.factor) ? fsrc + (size_t)e0 * NP + i : a.x, v && a.factor);
  }
  for (int i = lane; i < kEl * NG; i += 32) {
    const bool v = i < ne * NG;
    cp_async(st.geo + i, v ? a.geof + (size_t)e0 * NG + i : a.geof, v);
  }
  for (int i = lane; i < kEl * NF; i += 32) {
    const bool v = i < ne * NF;
    cp_async(st.tau + i, v ? a.tau + (size_t)e0 * NF + i : a.tau, v);
    cp_async(st.nbr + i, v ? a.nbr + (size_t)e0 * NF + i : a.nbr, v);
  }
  if (lane < kEl) {
    const bool v = lane < ne;
    cp_async(st.code + lane, v ? (const int*)a.fcode + e0 + lane : (const int*)a.fcode, v);
  }
}

// Issue the neighbour trace records of a tile whose element data has arrived.
template <typename T, int DIM, int P>
__device__ __forceinline__ void issue_traces(const ApplyArgs<T>& a, const Stage<T, DIM, P>& st, const T* trace,
                                             T* dst, int tile, int lane) {
  using TC = TcCfg<T, DIM, P>;
  constexpr int NF = TC::NF, TR = TC::TR;
  const int ne = max(0, min(kEl, a.K - tile * kEl));
  for (int i = lane; i < kEl * NF * TR; i += 32) {
    const int lf = i / TR, k = i % TR;
    const int el = lf / NF;
    const int nb = st.nbr[lf];
    const bool v = el < ne && nb >= 0;
    const int fr = (st.code[el] >> (8 * (lf % NF))) & 3;
    cp_async(dst + i, v ? trace + ((size_t)nb * NF + fr) * TR + k : trace, v);
  }
}

// grad_ref (M1 rows, 8 columns) = A1 x B(8 x K1): all M-tiles in one k-loop.
template <typename T, int DIM, int P>
__device__ __forceinline__ void gemm1(const T* A1, const T* Bs, int ldb, T* Cs, int lane) {
  using TC = TcCfg<T, DIM, P>;
  using M = Mma<T>;
  constexpr int NMT = TC::M1 / M::MT;
  T c[NMT][M::NC];
#pragma unroll
  for (int m = 0; m < NMT; ++m)
#pragma unroll
    for (int i = 0; i < M::NC; ++i) c[m][i] = T(0);
#pragma unroll
  for (int k0 = 0; k0 < TC::K1; k0 += M::KT) {
    typename M::B b;
    M::load_b(b, Bs, ldb, k0, lane);
#pragma unroll
    for (int m = 0; m < NMT; ++m) {
      typename M::A a;
      M::load_a(a, A1, TC::LDA1, m * M::MT, k0, lane);
      M::mma(c[m], a, b);
    }
  }
#pragma unroll
  for (int m = 0; m < NMT; ++m) M::store_c(c[m], Cs, TC::LDC, m * M::MT, lane);
}

// acc += A (M2 x K) * B(8 x K)
template <typename T, int NMT, int K, int LDA, int LDB>
__device__ __forceinline__ void gemm_acc(T (&c)[NMT][Mma<T>::NC], const T* A, const T* Bs, int lane) {
  using M = Mma<T>;
#pragma unroll 4
  for (int k0 = 0; k0 < K; k0 += M::KT) {
    typename M::B b;
    M::load_b(b, Bs, LDB, k0, lane);
#pragma unroll
    for (int m = 0; m < NMT; ++m) {
      typename M::A af;
      M::load_a(af, A, LDA, m * M::MT, k0, lane);
      M::mma(c[m], af, b);
    }
  }
}

template <typename T, int DIM>
__device__ __forceinline__ void face_geom(const T* g, int f, T* out) {
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
    T len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    n[0] /= len; n[1] /= len; n[2] /= len;
    out[3] = len * g[9];
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
    T len = sqrt(n[0] * n[0] + n[1] * n[1]);
    n[0] /= len; n[1] /= len;
    out[3] = len * g[4];
  }
  out[0] = n[0]; out[1] = n[1]; out[2] = n[2];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    T cr = T(0);
    if (r < DIM)
#pragma unroll
      for (int d = 0; d < DIM; ++d) cr += n[d] * g[r * DIM + d];
    out[4 + r] = cr;
  }
}

// Element geometry of padded tile slots is the identity map (finite normals).
template <typename T, int DIM>
__device__ __forceinline__ void pad_geometry(T* geo, int ne, int lane) {
  constexpr int NG = DIM == 3 ? 10 : 5;
  for (int i = lane + ne * NG; i < kEl * NG; i += 32) {
    const int k = i % NG;
    T v = T(0);
    if (DIM == 3) v = (k == 0 || k == 4 || k == 8 || k == 9) ? T(1) : T(0);
    else v = (k == 0 || k == 3 || k == 4) ? T(1) : T(0);
    geo[i] = v;
  }
}

// ---------------------------------------------------------------- pass 1
template <typename T, int DIM, int P, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) sipg_trace_kernel(ApplyArgs<T> a, const T* __restrict__ tc_consts,
                                                              T* __restrict__ trace) {
  using TC = TcCfg<T, DIM, P>;
  constexpr int NP = TC::NP, NFP = TC::NFP, NF = TC::NF, NG = TC::NG, FG = TC::FG;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A1 = reinterpret_cast<T*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* W = A1 + TC::CONST1 + warp * TC::W1_T;
  int* I = reinterpret_cast<int*>(A1 + TC::CONST1 + WARPS * TC::W1_T) + warp * TC::W1_I;
  int8_t* fmask = reinterpret_cast<int8_t*>(reinterpret_cast<int*>(A1 + TC::CONST1 + WARPS * TC::W1_T) +
                                            WARPS * TC::W1_I);
  T* sC = W + 2 * TC::ST_T;
  T* sFG = sC + kEl * TC::LDC;
  for (int i = threadIdx.x; i < TC::CONST1; i += blockDim.x) A1[i] = tc_consts[i];
  for (int i = threadIdx.x; i < NF * NFP; i += blockDim.x) fmask[i] = a.itab[i];
  const int ntiles = (a.K + kEl - 1) / kEl;
  const int stride = gridDim.x * WARPS;
  int tile = blockIdx.x * WARPS + warp;
  issue_own<T, DIM, P>(a, Stage<T, DIM, P>(W, I), tile, lane);
  cp_commit();
  __syncthreads();
  for (int it = 0; tile < ntiles; ++it, tile += stride) {
    const int b = it & 1;
    const Stage<T, DIM, P> S(W + b * TC::ST_T, I + b * TC::ST_I);
    issue_own<T, DIM, P>(a, Stage<T, DIM, P>(W + (b ^ 1) * TC::ST_T, I + (b ^ 1) * TC::ST_I), tile + stride, lane);
    cp_commit();
    cp_wait<1>();
    __syncwarp();
    const int e0 = tile * kEl;
    const int ne = min(kEl, a.K - e0);
    if (a.pin_elem >= e0 && a.pin_elem < e0 + ne && lane == 0) S.x[(a.pin_elem - e0) * NP + a.pin_node] = T(0);
    pad_geometry<T, DIM>(S.geo, ne, lane);
    __syncwarp();
    if (lane < kEl * NF) face_geom<T, DIM>(S.geo + (lane / NF) * NG, lane % NF, sFG + lane * FG);
    gemm1<T, DIM, P>(A1, S.x, NP, sC, lane);
    __syncwarp();
    // trace[e][f] = (x at the face nodes, f n.grad x at the face nodes)
    for (int i = lane; i < ne * NF * NFP; i += 32) {
      const int el = i / (NF * NFP), k = i % (NF * NFP);
      const int f = k / NFP, j = k % NFP;
      const int m = fmask[f * NFP + j];
      const T* fg = sFG + (el * NF + f) * FG;
      T s = T(0);
#pragma unroll
      for (int r = 0; r < DIM; ++r) s += fg[4 + r] * sC[el * TC::LDC + r * NP + m];
      const T fm = a.factor ? S.fac[el * NP + m] : T(1);
      T* tr = trace + ((size_t)(e0 + el) * NF + f) * TC::TR;
      tr[j] = S.x[el * NP + m];
      tr[NFP + j] = fm * s;
    }
    __syncwarp();
  }
  cp_wait<0>();
}

// ---------------------------------------------------------------- pass 2
template <typename T, int DIM, int P, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) sipg_apply_tc_kernel(ApplyArgs<T> a, const T* __restrict__ tc_consts,
                                                                 const T* __restrict__ trace) {
  using TC = TcCfg<T, DIM, P>;
  using M = Mma<T>;
  constexpr int NP = TC::NP, NFP = TC::NFP, NF = TC::NF, NFNFP = TC::NFNFP, NG = TC::NG, FG = TC::FG,
                TR = TC::TR;
  constexpr int NMT = TC::M2 / M::MT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A1 = reinterpret_cast<T*>(smem_raw);
  T* A2a = A1 + TC::CONST1;
  T* A2b = A2a + TC::M2 * TC::LDA2A;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* W = A1 + TC::CONST_T + warp * TC::W2_T;
  int* ibase = reinterpret_cast<int*>(A1 + TC::CONST_T + WARPS * TC::W2_T);
  int* I = ibase + warp * TC::W2_I;
  int8_t* itab = reinterpret_cast<int8_t*>(ibase + WARPS * TC::W2_I);
  const int8_t* fmask = itab;
  const int8_t* perm = itab + NF * NFP;
  T* trb0 = W + 3 * TC::ST_T;
  T* sB = W + 3 * TC::ST_T + 2 * TC::TRB;
  T* sC = sB + kEl * TC::LDB;
  T* sFG = sC + kEl * TC::LDC;
  T* sS = sFG + kEl * NF * FG;
  for (int i = threadIdx.x; i < TC::CONST_T; i += blockDim.x) A1[i] = tc_consts[i];
  for (int i = threadIdx.x; i < Cfg<DIM, P>::ITAB; i += blockDim.x) itab[i] = a.itab[i];
  const int ntiles = (a.K + kEl - 1) / kEl;
  const int stride = gridDim.x * WARPS;
  int tile = blockIdx.x * WARPS + warp;
  // prologue: element data of tiles 0 and 1 in flight, traces of tile 0 behind them
  issue_own<T, DIM, P>(a, Stage<T, DIM, P>(W, I), tile, lane);
  cp_commit();
  issue_own<T, DIM, P>(a, Stage<T, DIM, P>(W + TC::ST_T, I + TC::ST_I), tile + stride, lane);
  cp_commit();
  cp_wait<1>();
  __syncwarp();
  issue_traces<T, DIM, P>(a, Stage<T, DIM, P>(W, I), trace, trb0, tile, lane);
  cp_commit();
  __syncthreads();
  int s0 = 0;  // stage of this tile; tile+1 in (s0+1)%3, tile+2 in (s0+2)%3
  for (int it = 0; tile < ntiles; ++it, tile += stride) {
    const int s1 = s0 == 2 ? 0 : s0 + 1, s2 = s1 == 2 ? 0 : s1 + 1;
    const Stage<T, DIM, P> S(W + s0 * TC::ST_T, I + s0 * TC::ST_I);
    T* TRc = trb0 + (it & 1) * TC::TRB;
    // element data of tile+1 and traces of tile have arrived
    cp_wait<0>();
    __syncwarp();
    issue_traces<T, DIM, P>(a, Stage<T, DIM, P>(W + s1 * TC::ST_T, I + s1 * TC::ST_I), trace,
                            trb0 + ((it + 1) & 1) * TC::TRB, tile + stride, lane);
    issue_own<T, DIM, P>(a, Stage<T, DIM, P>(W + s2 * TC::ST_T, I + s2 * TC::ST_I), tile + 2 * stride, lane);
    cp_commit();
    s0 = s1;
    const int e0 = tile * kEl;
    const int ne = min(kEl, a.K - e0);
    if (a.pin_elem >= e0 && a.pin_elem < e0 + ne && lane == 0) S.x[(a.pin_elem - e0) * NP + a.pin_node] = T(0);
    pad_geometry<T, DIM>(S.geo, ne, lane);
    __syncwarp();
    if (lane < kEl * NF) face_geom<T, DIM>(S.geo + (lane / NF) * NG, lane % NF, sFG + lane * FG);
    // ---- G1: own gradient in the reference directions
    gemm1<T, DIM, P>(A1, S.x, NP, sC, lane);
    __syncwarp();
    // ---- chunk A: q~_r, Fu, J mm x
    for (int i = lane; i < kEl * NP; i += 32) {
      const int el = i / NP, m = i % NP;
      const T* g = S.geo + el * NG;
      const T J = g[DIM == 3 ? 9 : 4], f = a.factor ? S.fac[i] : T(1);
      T gr[3], q[3];
#pragma unroll
      for (int r = 0; r < DIM; ++r) gr[r] = sC[el * TC::LDC + r * NP + m];
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        T sum = T(0);
#pragma unroll
        for (int r = 0; r < DIM; ++r) sum += g[r * DIM + d] * gr[r];
        q[d] = f * sum;
      }
#pragma unroll
      for (int r = 0; r < DIM; ++r) {
        T sum = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) sum += g[r * DIM + d] * q[d];
        sB[el * TC::LDB + r * NP + m] = M::to_op(J * sum);
      }
      T mv = T(0);
      if (a.mm_mode != MM_NONE && el < ne)
        mv = J * (a.mm_mode == MM_SCALAR ? a.mm_scalar : a.mm[(size_t)e0 * NP + i]) * S.x[i];
      sB[el * TC::LDB + TC::OMM + m] = M::to_op(mv);
    }
    constexpr int PADA = TC::KA - TC::OMM - NP;
    if (PADA > 0)
      for (int i = lane; i < kEl * PADA; i += 32) {
        const int el = i / (PADA > 0 ? PADA : 1), n = i % (PADA > 0 ? PADA : 1);
        sB[el * TC::LDB + TC::OMM + NP + n] = T(0);
      }
    for (int i = lane; i < kEl * NFNFP; i += 32) {
      const int el = i / NFNFP, k = i % NFNFP;
      const int f = k / NFP, j = k % NFP;
      const int lf = el * NF + f;
      const T* fg = sFG + lf * FG;
      const int m = fmask[f * NFP + j];
      const T fm = a.factor ? S.fac[el * NP + m] : T(1);
      T nq = T(0);
#pragma unroll
      for (int r = 0; r < DIM; ++r) nq += fg[4 + r] * sC[el * TC::LDC + r * NP + m];
      nq *= fm;
      const int nb = S.nbr[lf];
      const T um = S.x[el * NP + m];
      T jump = T(0), navg = T(0);
      if (el < ne) {
        if (nb >= 0) {
          const int kk = perm[((S.code[el] >> (8 * f + 2)) & 7) * NFP + j];
          jump = um - TRc[lf * TR + kk];
          navg = T(0.5) * (nq - TRc[lf * TR + NFP + kk]);
        } else if (a.bct[-nb - 1] == BC_DIRICHLET) {
          jump = T(2) * um;
          navg = nq;
        }
      }
      const T hj = T(0.5) * jump, sJ = fg[3];
      sS[i] = sJ * fm * -hj;
      sB[el * TC::LDB + TC::OFU + k] = M::to_op(sJ * (S.tau[lf] * hj - navg));
    }
    __syncwarp();
    T c[NMT][M::NC];
#pragma unroll
    for (int m = 0; m < NMT; ++m)
#pragma unroll
      for (int q = 0; q < M::NC; ++q) c[m][q] = T(0);
    gemm_acc<T, NMT, TC::KA, TC::LDA2A, TC::LDB>(c, A2a, sB, lane);
    __syncwarp();
    // ---- chunk B: F~_r = c_r(f) * sJ f (-[x]/2)
    for (int i = lane; i < kEl * TC::KB; i += 32) {
      const int el = i / TC::KB, col = i % TC::KB;
      T v = T(0);
      if (col < DIM * NFNFP) {
        const int r = col / NFNFP, k = col % NFNFP;
        v = sFG[(el * NF + k / NFP) * FG + 4 + r] * sS[el * NFNFP + k];
      }
      sB[el * TC::LDB + col] = M::to_op(v);
    }
    __syncwarp();
    gemm_acc<T, NMT, TC::KB, TC::LDA2B, TC::LDB>(c, A2b, sB, lane);
#pragma unroll
    for (int m = 0; m < NMT; ++m) M::store_c(c[m], sC, TC::LDC, m * M::MT, lane);
    __syncwarp();
    for (int i = lane; i < ne * NP; i += 32) {
      const int el = i / NP, m = i % NP;
      const int e = e0 + el;
      T acc = sC[el * TC::LDC + m];
      const size_t yi = (size_t)e0 * NP + i;
      if (e == a.pin_elem && m == a.pin_node) acc = a.pin_scale * a.x[yi];
      acc *= a.alpha;
      if (a.beta != T(0)) acc += a.beta * a.y[yi];
      a.y[yi] = acc;
    }
    __syncwarp();
  }
  cp_wait<0>();
}

constexpr int kSmemBudget = 220 * 1024;

template <typename T, int DIM, int P>
constexpr int warps1() {
  using TC = TcCfg<T, DIM, P>;
  return std::max(1, std::min(16, (int)((kSmemBudget - TC::CONST1 * (int)sizeof(T) - 64) /
                                        (TC::W1_T * (int)sizeof(T) + TC::W1_I * 4))));
}
// 0 when the constants leave no room for a warp tile
template <typename T, int DIM, int P>
constexpr int warps2() {
  using TC = TcCfg<T, DIM, P>;
  return std::min(16, (int)((kSmemBudget - TC::CONST_T * (int)sizeof(T) - 256) /
                            (TC::W2_T * (int)sizeof(T) + TC::W2_I * 4)));
}

template <typename T, int DIM, int P>
cudaError_t launch_tc_t(const ApplyArgs<T>& a, const T* tc_consts, T* trace, int num_sms, cudaStream_t s) {
  using TC = TcCfg<T, DIM, P>;
  constexpr int WA = warps1<T, DIM, P>(), WB = warps2<T, DIM, P>() < 1 ? 1 : warps2<T, DIM, P>();
  if (warps2<T, DIM, P>() < 1) return cudaErrorInvalidConfiguration;
  const int ntiles = (a.K + kEl - 1) / kEl;
  {
    auto k = sipg_trace_kernel<T, DIM, P, WA>;
    size_t bytes = (size_t)(TC::CONST1 + WA * TC::W1_T) * sizeof(T) + (size_t)WA * TC::W1_I * 4 + TC::NF * TC::NFP;
    cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (err != cudaSuccess) return err;
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, WA * 32, bytes);
    int grid = std::min((ntiles + WA - 1) / WA, num_sms * std::max(per_sm, 1));
    if (grid > 0) {
      k<<<grid, WA * 32, bytes, s>>>(a, tc_consts, trace);
      note_launch();
    }
  }
  {
    auto k = sipg_apply_tc_kernel<T, DIM, P, WB>;
    size_t bytes = (size_t)(TC::CONST_T + WB * TC::W2_T) * sizeof(T) + (size_t)WB * TC::W2_I * 4 +
                   Cfg<DIM, P>::ITAB;
    cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (err != cudaSuccess) return err;
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, WB * 32, bytes);
    int grid = std::min((ntiles + WB - 1) / WB, num_sms * std::max(per_sm, 1));
    if (grid > 0) {
      k<<<grid, WB * 32, bytes, s>>>(a, tc_consts, trace);
      note_launch();
    }
  }
  return cudaGetLastError();
}

// Host construction of the constant blob (A1 | A2a | A2b) in FP64.
template <typename T, int DIM, int P>
void build_tc_consts_t(const RefElement& r, std::vector<double>& out) {
  using TC = TcCfg<T, DIM, P>;
  constexpr int NP = TC::NP, NFNFP = TC::NFNFP;
  out.assign(TC::CONST_T, 0.0);
  const double* D[3] = {r.Dr.data(), r.Ds.data(), r.Dt.data()};
  double* A1 = out.data();
  double* A2a = A1 + TC::CONST1;
  double* A2b = A2a + TC::M2 * TC::LDA2A;
  for (int rr = 0; rr < DIM; ++rr)
    for (int m = 0; m < NP; ++m)
      for (int n = 0; n < NP; ++n) A1[(rr * NP + m) * TC::LDA1 + n] = D[rr][m * NP + n];
  for (int n = 0; n < NP; ++n) {
    for (int rr = 0; rr < DIM; ++rr) {
      for (int m = 0; m < NP; ++m) {
        double s = 0.0;
        for (int i = 0; i < NP; ++i) s += D[rr][i * NP + n] * r.M[i * NP + m];
        A2a[n * TC::LDA2A + rr * NP + m] = s;
      }
      for (int c = 0; c < NFNFP; ++c) {
        double s = 0.0;
        for (int i = 0; i < NP; ++i) s += D[rr][i * NP + n] * r.EMAT[i * NFNFP + c];
        A2b[n * TC::LDA2B + rr * NFNFP + c] = s;
      }
    }
    for (int c = 0; c < NFNFP; ++c) A2a[n * TC::LDA2A + TC::OFU + c] = r.EMAT[n * NFNFP + c];
    for (int m = 0; m < NP; ++m) A2a[n * TC::LDA2A + TC::OMM + m] = r.M[n * NP + m];
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
  SIPG_DISPATCH_TC(dim, order, return warps2<T, D, P>());
  return 0;
}

size_t tc_trace_values(int dim, int order, int K) {
  return (size_t)K * (dim + 1) * 2 * nfp_of(dim, order);
}

template cudaError_t launch_apply_tc<float>(int, int, const ApplyArgs<float>&, const float*, float*, int,
                                            cudaStream_t);
template cudaError_t launch_apply_tc<double>(int, int, const ApplyArgs<double>&, const double*, double*, int,
                                             cudaStream_t);
template void build_tc_consts<float>(int, int, const RefElement&, std::vector<double>&);
template void build_tc_consts<double>(int, int, const RefElement&, std::vector<double>&);
template int tc_warps_for<float>(int, int);
template int tc_warps_for<double>(int, int);

}  // namespace sipg
