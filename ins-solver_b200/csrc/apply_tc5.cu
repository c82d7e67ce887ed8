// SIPG apply (scalar operator, FP32 data) on the fifth-generation tensor cores:
// tcgen05.mma kind::tf32 with the accumulators in tensor memory (TMEM).
//
// Same operator as the mma.sync kernels of sipg_apply_tc.cu
// (FactorViscousMatrix3D::mult, src/solvers/3d/slip_matrix/factor_viscous_matrix.cpp:96-310,
// one component) and the same two passes and face-trace records between them.
// A tile is 128 elements, the M dimension of the MMAs; two threads per element
// (warps w and w + 4 read the same 32 TMEM lanes) do the elementwise work on
// whole rows, so no accumulator lives in registers.
//
//   pass 1: T = x . B1f (B1f: per face f and direction r the rows of D_r at the
//           face nodes), g = f(m) sum_r c_r(f) T_r at the face nodes, trace
//           record (u, g) per element face, written in the face-node order of
//           the neighbour that reads it (so pass 2 reads it without permuting).
//   pass 2: one MMA gives the reference gradients gr_r = x . D_r^T and the own
//           face traces T; each thread row then builds
//             w_r = J f sum_s K_rs gr_s                 (K = G G^T)
//             per face: Fu = sJ (tau [u]/2 - n.{q}),  c_r S with S = -sJ f [u]/2
//             (fvmf_3d_mult_flux.h:13-22, boundary traces vmf_3d_mult_avg_jump.h:43-80)
//             J mm x                                    (fvmf_3d_mult_mm_geof.h:5-19)
//           into one A row, and a second MMA against the reassociated constant
//           B2 = [M^T D_r ; EMAT^T D_r ; EMAT^T ; M^T] gives
//             y = sum_r (w_r M^T + (c_r S) EMAT^T) D_r + Fu EMAT^T + (J mm x) M^T,
//           the reference's mass, lift and D^T passes (factor_viscous_matrix.cpp:233-286)
//           as one product.
//
// Operands sit in shared memory in the K-major, unswizzled layout of the MMA
// (core matrices of 8 rows x 16 bytes; element (m, k) of an R-row operand at
// float (k / 4) * 4R + 4m + k % 4), so a thread's 16-byte chunk of a row is one
// vector store and the 32 threads of a warp store 512 contiguous bytes. The
// constant operands are laid out the same way on the host and copied once per
// CTA. Every wait on an MMA is bounded: after kWaitLimit polls the kernel
// records the timeout in g_tc5_timeouts and stops working on tiles.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "pdl.cuh"
#include "sipg_apply.cuh"
#include "sipg_apply_tc.cuh"
#include "vecops.cuh"

namespace sipg {

__device__ unsigned int g_tc5_timeouts = 0;

namespace {

__host__ __device__ constexpr int rup5(int x, int m) { return (x + m - 1) / m * m; }

constexpr int kM = 128;         // elements per tile = MMA M = TMEM lanes
constexpr int kThreads = 256;   // two threads per element
constexpr long kWaitLimit = 1 << 26;

template <int P>
struct T5 {
  static constexpr int NP = c_np(3, P), NFP = c_nfp(3, P), NF = 4, KF = NF * NFP;
  static constexpr int K1 = rup5(NP, 8);        // MMA-1 K: input nodes, zero padded
  static constexpr int NG = rup5(3 * NP, 16);   // MMA-1 columns of the reference gradients
  static constexpr int FT = rup5(3 * NFP, 16);  // MMA-1 columns of one face's traces
  static constexpr int N1 = NG + NF * FT;       // MMA-1 N
  static constexpr int N2 = rup5(NP, 16);       // MMA-2 N: output nodes
  // MMA-2 K sections: w_0..w_2, per face [c_0 S | c_1 S | c_2 S | Fu], J mm x
  static constexpr int KFACE = 4 * NFP;
  static constexpr int OFF_F = rup5(3 * NP, 8);
  static constexpr int OFF_MM = OFF_F + NF * KFACE;
  static constexpr int K2 = rup5(OFF_MM + NP, 8);
  // trace records: the mma.sync kernels' layout (u at [0, NFP), g at [TRP, TRP + NFP))
  static constexpr int TRP = rup5(NFP, 2), TR = rup5(2 * TRP, 4), TRV = TR / 4;
  // constant blob (floats, MMA layout): B1 (N1 x K1), B2 (N2 x K2)
  static constexpr int CB1 = 0, CB2 = N1 * K1, CALL = CB2 + N2 * K2;
  // geometry blocks of the mma.sync kernels (launch_tc_geom, FP32: tiles of 16 elements)
  static constexpr int GTE = 16, GROWS = 24, GBLK = GROWS * GTE;
  static constexpr int XS = NP | 1;             // row stride of the staged x / factor rows (odd: no bank conflicts)
  // pass-2 shared memory (bytes): constants, operands, x and factor rows, one
  // neighbour trace record per thread, the int8 tables, barriers
  static constexpr int SB1 = 0, SB2 = SB1 + N1 * K1 * 4, SA1 = SB2 + N2 * K2 * 4, SA2 = SA1 + kM * K1 * 4;
  static constexpr int SX = SA2 + kM * K2 * 4, SF = SX + kM * XS * 4;
  static constexpr int SITAB = SF + kM * XS * 4;
  static constexpr int SBAR = rup5(SITAB + NF * NFP + 6 * NFP, 16), SMEM2 = SBAR + 32;
  // pass 1: face rows of B1, x operand, x and factor rows, one record per thread
  // (reordered there), the int8 tables
  static constexpr int P1B = 0, P1A = P1B + NF * FT * K1 * 4, P1X = P1A + kM * K1 * 4, P1F = P1X + kM * XS * 4;
  static constexpr int P1S = P1F + kM * XS * 4, P1I = P1S + kThreads * TR * 4;
  static constexpr int P1BAR = rup5(P1I + NF * NFP + 6 * NFP, 16), SMEM1 = P1BAR + 32;
  static constexpr int TMEM2 = N1 + N2 <= 256 ? 256 : 512;
  static constexpr int TMEM1 = NF * FT <= 128 ? 128 : 256;
  static_assert(KFACE % 4 == 0, "face sections are whole 16-byte chunks");
  static_assert(N1 <= 256 && N1 % 16 == 0 && N2 % 16 == 0, "one MMA per K step");
  static_assert(FT % 16 == 0, "TMEM loads of a face group");
};

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory operand descriptor: K-major, no swizzle; lbo = byte distance of
// the two 16-byte K chunks of one MMA K step, sbo = byte distance of 8-row groups.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::tf32, FP32 accumulation, K-major A and B, M = 128.
__host__ __device__ constexpr uint32_t idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}
__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar));
}
__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar));
}
// Bounded wait for phase `parity` of an mbarrier; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity));
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// FP32 -> TF32 operand, rounded to nearest (a relative error below 2^-11).
__device__ __forceinline__ float tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Float index of element (row, k) of an operand with `rows` rows in the MMA layout.
__host__ __device__ constexpr int opidx(int rows, int row, int k) { return (k >> 2) * (rows * 4) + row * 4 + (k & 3); }

__device__ __forceinline__ void st4(float* s, int rows, int row, int k0, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(s + opidx(rows, row, k0)) = make_float4(tf32(a), tf32(b), tf32(c), tf32(d));
}

// Copy n floats (a multiple of 4) with 16-byte vectors; 16-byte aligned ends.
__device__ __forceinline__ void copy_f4(float* dst, const float* src, int n, int tid) {
  for (int i = tid * 4; i < n; i += kThreads * 4)
    *reinterpret_cast<float4*>(dst + i) = *reinterpret_cast<const float4*>(src + i);
}

// Face node -> volume node maps of the reference element (FMASK), as compile-time
// tables so that the flux code reads the staged rows at fixed offsets. The host
// checks them against the element the library builds (tc5_prepare); an order
// whose table differs is not run on these kernels.
template <int P>
struct FaceMask;
template <>
struct FaceMask<3> {
  __host__ __device__ static constexpr int at(int f, int j) {
    constexpr int8_t v[4][10] = {{9, 8, 6, 3, 7, 2, 5, 4, 1, 0},
                                 {19, 17, 12, 3, 16, 2, 11, 10, 1, 0},
                                 {19, 18, 15, 9, 17, 8, 14, 12, 6, 3},
                                 {19, 18, 15, 9, 16, 7, 13, 10, 4, 0}};
    return v[f][j];
  }
};

// A tile's x and factor rows: thread m of half 0 loads row m of x, of half 1 row m
// of the factor, into registers ahead of use (the next tile's while the current
// one finishes); they are stored as rows of stride XS (zero past the tile; the
// pinned DOF is zero, as in the operator's column) and the A1 operand (TF32,
// zero past Np) is built from the x rows.
template <int P>
struct Rows {
  float v[T5<P>::NP];
};

template <int P>
__device__ __forceinline__ void load_rows(const ApplyArgs<float>& a, int e0, int ne, int m, int half, Rows<P>& r) {
  using X = T5<P>;
  constexpr int NP = X::NP;
  const float* src = half == 0 ? a.x : a.factor;
  if (half == 1 && !src) {
#pragma unroll
    for (int i = 0; i < NP; ++i) r.v[i] = 1.f;
    return;
  }
  if (m >= ne) {
#pragma unroll
    for (int i = 0; i < NP; ++i) r.v[i] = 0.f;
    return;
  }
  const float* row = src + (size_t)(e0 + m) * NP;
  if constexpr (NP % 4 == 0) {
#pragma unroll
    for (int c = 0; c < NP / 4; ++c) {
      const float4 q = __ldg(reinterpret_cast<const float4*>(row) + c);
      r.v[4 * c] = q.x;
      r.v[4 * c + 1] = q.y;
      r.v[4 * c + 2] = q.z;
      r.v[4 * c + 3] = q.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < NP; ++i) r.v[i] = __ldg(row + i);
  }
}

template <int P>
__device__ __forceinline__ void store_rows(const ApplyArgs<float>& a, const Rows<P>& r, float* sX, float* sF,
                                           float* sA1, int e0, int m, int half) {
  using X = T5<P>;
  constexpr int NP = X::NP, XS = X::XS;
  float* dst = (half == 0 ? sX : sF) + m * XS;
  const int pin = (half == 0 && e0 + m == a.pin_elem) ? a.pin_node : -1;
#pragma unroll
  for (int i = 0; i < NP; ++i) dst[i] = i == pin ? 0.f : r.v[i];
  __syncthreads();
  // the two threads of row m write alternate 16-byte chunks of its A1 row
  const float* xr = sX + m * XS;
#pragma unroll
  for (int c = half * 4; c < X::K1; c += 8) {
    float v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = c + i < NP ? xr[c + i] : 0.f;
    st4(sA1, kM, m, c, v[0], v[1], v[2], v[3]);
  }
}

// Element e's column of the per-mesh geometry blocks (rows q at stride GTE).
template <int P>
__device__ __forceinline__ const float* geo_col(const float* __restrict__ tcg, int e) {
  using X = T5<P>;
  return tcg + (size_t)(e / X::GTE) * X::GBLK + (e % X::GTE);
}

// Face data of one element face, loaded into registers ahead of use: sJ, c_r,
// tau, the neighbour (or -(bface+1)) and its trace record.
template <int P>
struct FaceIn {
  float sJ, c[3], tau;
  int nb;
  bool dir;
  float4 rec[T5<P>::TRV];
};

template <int P>
__device__ __forceinline__ void load_face(const ApplyArgs<float>& a, const float* __restrict__ trace, const float* g,
                                          int e, int f, bool valid, FaceIn<P>& d) {
  using X = T5<P>;
  constexpr int NF = X::NF, GTE = X::GTE;
  d.sJ = d.tau = d.c[0] = d.c[1] = d.c[2] = 0.f;
  d.nb = -1;
  d.dir = false;
  if (!valid) return;
  d.sJ = __ldg(g + (8 + f) * GTE);
#pragma unroll
  for (int r = 0; r < 3; ++r) d.c[r] = __ldg(g + (8 + (1 + r) * NF + f) * GTE);
  d.tau = __ldg(a.tau + (size_t)e * NF + f);
  d.nb = __ldg(a.nbr + (size_t)e * NF + f);
  if (d.nb >= 0) {
    const uint32_t code = __ldg(a.fcode + e);
    const float4* src = reinterpret_cast<const float4*>(trace + ((size_t)d.nb * NF + ((code >> (8 * f)) & 3)) * X::TR);
#pragma unroll
    for (int c = 0; c < X::TRV; ++c) d.rec[c] = __ldg(src + c);
  } else {
    d.dir = a.bct[-d.nb - 1] == BC_DIRICHLET;
  }
}

// Face F of element row m: own traces from TMEM (T_r at the face nodes), the
// neighbour's record (already in this face's node order), the fluxes; writes the
// face's A2 section [c_r S | Fu].
template <int P, int F>
__device__ __forceinline__ void face_section(float* sA2, const float* xr, const float* fr, const FaceIn<P>& d,
                                             uint32_t tcol, int m) {
  using X = T5<P>;
  constexpr int NFP = X::NFP;
  float T[X::FT];
#pragma unroll
  for (int c = 0; c < X::FT; c += 16) tmem_ld16(tcol + c, *reinterpret_cast<float(*)[16]>(&T[c]));
  const bool inner = d.nb >= 0;
  const float* rec = reinterpret_cast<const float*>(d.rec);
  tmem_wait_ld();
  float sec[X::KFACE];
#pragma unroll
  for (int j = 0; j < NFP; ++j) {
    const int mj = FaceMask<P>::at(F, j);
    const float fm = fr[mj];
    const float gm = fm * (d.c[0] * T[j] + d.c[1] * T[NFP + j] + d.c[2] * T[2 * NFP + j]);
    const float um = xr[mj];
    float jump = 0.f, navg = 0.f;
    if (inner) {
      jump = um - rec[j];
      navg = 0.5f * (gm - rec[X::TRP + j]);
    } else if (d.dir) {
      jump = 2.0f * um;
      navg = gm;
    }
    const float h = 0.5f * jump;
    const float sv = -d.sJ * fm * h;
    sec[j] = d.c[0] * sv;
    sec[NFP + j] = d.c[1] * sv;
    sec[2 * NFP + j] = d.c[2] * sv;
    sec[3 * NFP + j] = d.sJ * (d.tau * h - navg);
  }
  constexpr int k0 = X::OFF_F + F * X::KFACE;
#pragma unroll
  for (int c = 0; c < X::KFACE; c += 4) st4(sA2, kM, m, k0 + c, sec[c], sec[c + 1], sec[c + 2], sec[c + 3]);
}

// Pass-1 record of face F: u and g at the face nodes, stored in the face-node
// order of the neighbour that reads it (position perm_pos[sigma][j] holds face
// node j; sigma: this face's orientation code), through the thread's slot.
template <int P, int F>
__device__ __forceinline__ void trace_record(float* __restrict__ trace, float* slot, const int8_t* perm,
                                             const float* xr, const float* fr, const float (&cg)[3], int pb,
                                             uint32_t tcol, size_t e, bool valid) {
  using X = T5<P>;
  constexpr int NFP = X::NFP;
  float T[X::FT];
#pragma unroll
  for (int c = 0; c < X::FT; c += 16) tmem_ld16(tcol + c, *reinterpret_cast<float(*)[16]>(&T[c]));
  tmem_wait_ld();
#pragma unroll
  for (int i = NFP; i < X::TRP; ++i) slot[i] = slot[X::TRP + i] = 0.f;
#pragma unroll
  for (int i = 2 * X::TRP; i < X::TR; ++i) slot[i] = 0.f;
#pragma unroll
  for (int j = 0; j < NFP; ++j) {
    const int mj = FaceMask<P>::at(F, j);
    const int pos = pb >= 0 ? perm[pb + j] : j;
    slot[pos] = xr[mj];
    slot[X::TRP + pos] = fr[mj] * (cg[0] * T[j] + cg[1] * T[NFP + j] + cg[2] * T[2 * NFP + j]);
  }
  if (valid) {
    float4* dst = reinterpret_cast<float4*>(trace + (e * X::NF + F) * X::TR);
#pragma unroll
    for (int c = 0; c < X::TRV; ++c) dst[c] = reinterpret_cast<const float4*>(slot)[c];
  }
}

// ---------------------------------------------------------------- pass 1
template <int P>
__global__ void __launch_bounds__(kThreads, 2) sipg_tc5_trace(ApplyArgs<float> a, const float* __restrict__ blob,
                                                             float* __restrict__ trace) {
  using X = T5<P>;
  constexpr int NFP = X::NFP, NF = X::NF, K1 = X::K1, XS = X::XS, GTE = X::GTE;
  extern __shared__ __align__(128) unsigned char smem[];
  float* sB = reinterpret_cast<float*>(smem + X::P1B);  // face rows of B1: NF*FT x K1
  float* sA1 = reinterpret_cast<float*>(smem + X::P1A);
  float* sX = reinterpret_cast<float*>(smem + X::P1X);
  float* sF = reinterpret_cast<float*>(smem + X::P1F);
  int8_t* itab = reinterpret_cast<int8_t*>(smem + X::P1I);
  const int8_t* perm = itab + NF * NFP;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + X::P1BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + X::P1BAR + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m = 32 * (warp & 3) + lane, half = warp >> 2;
  float* slot = reinterpret_cast<float*>(smem + X::P1S) + tid * X::TR;
  constexpr int NB = NF * X::FT;
  pdl_trigger();
  // face rows of B1 (rows NG .. N1 of the N1 x K1 operand) as an NB-row operand
  for (int q = tid; q < NB * K1; q += kThreads) {
    const int n = q / K1, k = q % K1;
    sB[opidx(NB, n, k)] = blob[X::CB1 + opidx(X::N1, X::NG + n, k)];
  }
  for (int i = tid; i < NF * NFP + 6 * NFP; i += kThreads) itab[i] = a.itab[i];
  if (tid == 0) {
    mbar_init(smem_u32(bar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(X::TMEM1));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  pdl_wait();
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t lane_base = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
  const int ntiles = (a.K + kM - 1) / kM;
  bool ok = true;
  uint32_t phase = 0;
  Rows<P> rows;
  if ((int)blockIdx.x < ntiles) load_rows<P>(a, blockIdx.x * kM, min(kM, a.K - (int)blockIdx.x * kM), m, half, rows);
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, phase ^= 1) {
    const int e0 = tile * kM, ne = min(kM, a.K - e0);
    const bool valid = m < ne;
    const int e = e0 + m;
    store_rows<P>(a, rows, sX, sF, sA1, e0, m, half);
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    {
      const int next = tile + gridDim.x;
      if (next < ntiles) load_rows<P>(a, next * kM, min(kM, a.K - next * kM), m, half, rows);
    }
    if (tid == 0) {
      const uint32_t a0 = smem_u32(sA1), b0 = smem_u32(sB);
#pragma unroll
      for (int kk = 0; kk < K1 / 8; ++kk)
        mma_tf32(tmem, sdesc(a0 + kk * 2 * kM * 16, kM * 16, 128), sdesc(b0 + kk * 2 * NB * 16, NB * 16, 128),
                 idesc_tf32(NB), kk > 0);
      mma_commit(smem_u32(bar));
    }
    // the face geometry and orientation while the MMA runs
    float cg[2][3];
    int pb[2] = {-1, -1};
    const float* g = geo_col<P>(a.tcg, e);
    const uint32_t code = valid ? __ldg(a.fcode + e) : 0u;
#pragma unroll
    for (int fi = 0; fi < 2; ++fi) {
      const int f = 2 * half + fi;
#pragma unroll
      for (int r = 0; r < 3; ++r) cg[fi][r] = valid ? __ldg(g + (8 + (1 + r) * NF + f) * GTE) : 0.f;
      if (valid && __ldg(a.nbr + (size_t)e * NF + f) >= 0) pb[fi] = (int)((code >> (8 * f + 2)) & 7) * NFP;
    }
    // one thread polls the MMA barrier, the others wait at the CTA barrier;
    // the whole CTA stops on a timeout
    ok = __syncthreads_and(tid == 0 ? mbar_wait(smem_u32(bar), phase) : true) != 0;
    tc_after_sync();
    if (!ok) {
      if (tid == 0) atomicAdd(&g_tc5_timeouts, 1u);
      break;
    }
    const float* xr = sX + m * XS;
    const float* fr = sF + m * XS;
    if (half == 0) {
      trace_record<P, 0>(trace, slot, perm, xr, fr, cg[0], pb[0], lane_base + 0 * X::FT, (size_t)e, valid);
      trace_record<P, 1>(trace, slot, perm, xr, fr, cg[1], pb[1], lane_base + 1 * X::FT, (size_t)e, valid);
    } else {
      trace_record<P, 2>(trace, slot, perm, xr, fr, cg[0], pb[0], lane_base + 2 * X::FT, (size_t)e, valid);
      trace_record<P, 3>(trace, slot, perm, xr, fr, cg[1], pb[1], lane_base + 3 * X::FT, (size_t)e, valid);
    }
    tc_before_sync();
    __syncthreads();  // the next tile's staging overwrites the rows, its MMA the accumulator
    tc_after_sync();
  }
  tc_before_sync();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(X::TMEM1));
}

// ---------------------------------------------------------------- pass 2
template <int P>
__global__ void __launch_bounds__(kThreads, 1) sipg_tc5_apply(ApplyArgs<float> a, const float* __restrict__ blob,
                                                             const float* __restrict__ trace) {
  using X = T5<P>;
  constexpr int NP = X::NP, NFP = X::NFP, NF = X::NF, K1 = X::K1, N1 = X::N1, N2 = X::N2, XS = X::XS;
  extern __shared__ __align__(128) unsigned char smem[];
  float* sB1 = reinterpret_cast<float*>(smem + X::SB1);
  float* sB2 = reinterpret_cast<float*>(smem + X::SB2);
  float* sA1 = reinterpret_cast<float*>(smem + X::SA1);
  float* sA2 = reinterpret_cast<float*>(smem + X::SA2);
  float* sX = reinterpret_cast<float*>(smem + X::SX);
  float* sF = reinterpret_cast<float*>(smem + X::SF);
  int8_t* itab = reinterpret_cast<int8_t*>(smem + X::SITAB);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + X::SBAR);  // [0] MMA 1, [1] MMA 2
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + X::SBAR + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m = 32 * (warp & 3) + lane, half = warp >> 2;
  pdl_trigger();
  copy_f4(sB1, blob + X::CB1, N1 * K1, tid);
  copy_f4(sB2, blob + X::CB2, N2 * X::K2, tid);
  for (int i = tid; i < NF * NFP + 6 * NFP; i += kThreads) itab[i] = a.itab[i];
  if (tid == 0) {
    mbar_init(smem_u32(bar));
    mbar_init(smem_u32(bar + 1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(X::TMEM2));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  pdl_wait();
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t lane_base = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
  const bool has_mm = a.mm_mode != MM_NONE;
  const int k2 = has_mm ? X::K2 : X::OFF_MM;
  const int ntiles = (a.K + kM - 1) / kM;
  bool ok = true;
  uint32_t phase = 0;
  Rows<P> rows;
  if ((int)blockIdx.x < ntiles) load_rows<P>(a, blockIdx.x * kM, min(kM, a.K - (int)blockIdx.x * kM), m, half, rows);
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, phase ^= 1) {
    const int e0 = tile * kM, ne = min(kM, a.K - e0);
    const bool valid = m < ne;
    const int e = e0 + m;
    store_rows<P>(a, rows, sX, sF, sA1, e0, m, half);
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (tid == 0) {
      const uint32_t a0 = smem_u32(sA1), b0 = smem_u32(sB1);
#pragma unroll
      for (int kk = 0; kk < K1 / 8; ++kk)
        mma_tf32(tmem, sdesc(a0 + kk * 2 * kM * 16, kM * 16, 128), sdesc(b0 + kk * 2 * N1 * 16, N1 * 16, 128),
                 idesc_tf32(N1), kk > 0);
      mma_commit(smem_u32(bar));
    }
    // this thread's faces (half 0: face 0 and the volume terms, half 1: faces 1..3)
    // and geometry, loaded while MMA 1 runs
    const float* g = geo_col<P>(a.tcg, e);
    constexpr int NFH = NF - 1;
    FaceIn<P> fd[NFH];
    if (half == 0) {
      load_face<P>(a, trace, g, e, 0, valid, fd[0]);
    } else {
#pragma unroll
      for (int i = 0; i < NFH; ++i) load_face<P>(a, trace, g, e, 1 + i, valid, fd[i]);
    }
    float J = 0.f, Km[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    if (half == 0 && valid) {
      J = __ldg(g);
      int q = 1;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int s2 = r; s2 < 3; ++s2) {
          Km[r][s2] = Km[s2][r] = __ldg(g + q * X::GTE);
          ++q;
        }
    }
    // one thread polls the MMA barrier, the others wait at the CTA barrier;
    // the whole CTA stops on a timeout
    ok = __syncthreads_and(tid == 0 ? mbar_wait(smem_u32(bar), phase) : true) != 0;
    tc_after_sync();
    if (!ok) {
      if (tid == 0) atomicAdd(&g_tc5_timeouts, 1u);
      break;
    }
    const float* xr = sX + m * XS;
    const float* fr = sF + m * XS;
    if (half == 0) {
      // w_r = J f sum_s K_rs gr_s
      float gr[X::NG];
#pragma unroll
      for (int c = 0; c < X::NG; c += 16) tmem_ld16(lane_base + c, *reinterpret_cast<float(*)[16]>(&gr[c]));
      tmem_wait_ld();
#pragma unroll
      for (int c = 0; c < X::OFF_F; c += 4) {
        float v[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int k = c + i;
          v[i] = 0.f;
          if (k < 3 * NP) {
            const int r = k / NP, n = k % NP;
            v[i] = J * fr[n] * (Km[r][0] * gr[n] + Km[r][1] * gr[NP + n] + Km[r][2] * gr[2 * NP + n]);
          }
        }
        st4(sA2, kM, m, c, v[0], v[1], v[2], v[3]);
      }
      if (has_mm) {
#pragma unroll
        for (int c = 0; c < X::K2 - X::OFF_MM; c += 4) {
          float v[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int n = c + i;
            v[i] = 0.f;
            if (n < NP && valid) {
              const float mmv = a.mm_mode == MM_SCALAR ? a.mm_scalar : __ldg(a.mm + (size_t)e * NP + n);
              v[i] = J * mmv * xr[n];
            }
          }
          st4(sA2, kM, m, X::OFF_MM + c, v[0], v[1], v[2], v[3]);
        }
      }
      face_section<P, 0>(sA2, xr, fr, fd[0], lane_base + X::NG, m);
    } else {
      face_section<P, 1>(sA2, xr, fr, fd[0], lane_base + X::NG + 1 * X::FT, m);
      face_section<P, 2>(sA2, xr, fr, fd[1], lane_base + X::NG + 2 * X::FT, m);
      face_section<P, 3>(sA2, xr, fr, fd[2], lane_base + X::NG + 3 * X::FT, m);
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (tid == 0) {
      const uint32_t a0 = smem_u32(sA2), b0 = smem_u32(sB2);
      for (int kk = 0; kk < k2 / 8; ++kk)
        mma_tf32(tmem + N1, sdesc(a0 + kk * 2 * kM * 16, kM * 16, 128), sdesc(b0 + kk * 2 * N2 * 16, N2 * 16, 128),
                 idesc_tf32(N2), kk > 0);
      mma_commit(smem_u32(bar + 1));
    }
    // the next tile's rows, and c for the epilogue (into the factor rows, free
    // now), while MMA 2 runs
    {
      const int next = tile + gridDim.x;
      if (next < ntiles) load_rows<P>(a, next * kM, min(kM, a.K - next * kM), m, half, rows);
    }
    if (a.beta != 0.f)
      for (int i = tid; i < ne * NP; i += kThreads) {
        const int mm_ = i / NP;
        sF[mm_ * XS + (i - mm_ * NP)] = __ldg(a.c + (size_t)e0 * NP + i);
      }
    ok = __syncthreads_and(tid == 0 ? mbar_wait(smem_u32(bar + 1), phase) : true) != 0;
    tc_after_sync();
    if (!ok) {
      if (tid == 0) atomicAdd(&g_tc5_timeouts, 1u);
      break;
    }
    constexpr int HALFN = N2 / 2;
    const int n0 = half * HALFN;
    float acc[HALFN];
#pragma unroll
    for (int c = 0; c < HALFN; c += 16)
      tmem_ld16(lane_base + N1 + n0 + c, *reinterpret_cast<float(*)[16]>(&acc[c]));
    tmem_wait_ld();
    // y row into the x rows (free now), then a coalesced store of the tile
    float* yr = sX + m * XS;
#pragma unroll
    for (int i = 0; i < HALFN; ++i) {
      const int n = n0 + i;
      if (n < NP) {
        float v = acc[i];
        if (e == a.pin_elem && n == a.pin_node) v = a.pin_scale * __ldg(a.x + (size_t)e * NP + n);
        v *= a.alpha;
        if (a.beta != 0.f) v += a.beta * fr[n];
        yr[n] = v;
      }
    }
    __syncthreads();
    for (int i = tid; i < ne * NP; i += kThreads) {
      const int mm_ = i / NP;
      a.y[(size_t)e0 * NP + i] = sX[mm_ * XS + (i - mm_ * NP)];
    }
    tc_before_sync();
    __syncthreads();  // shared operands, rows and accumulators are free for the next tile
    tc_after_sync();
  }
  tc_before_sync();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(X::TMEM2));
}

template <int P>
cudaError_t launch_t(const ApplyArgs<float>& a, const float* blob, float* trace, int num_sms, cudaStream_t s) {
  using X = T5<P>;
  static_assert(X::SMEM2 <= 227 * 1024, "pass-2 shared memory");
  const int ntiles = (a.K + kM - 1) / kM;
  if (ntiles == 0) return cudaSuccess;
  auto k1 = sipg_tc5_trace<P>;
  auto k2 = sipg_tc5_apply<P>;
  // the shared-memory opt-in is a per-device function attribute: set once per device
  static std::atomic<uint32_t> attr_done{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint32_t bit = 1u << (dev & 31);
  if (!(attr_done.load() & bit)) {
    e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, X::SMEM1);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, X::SMEM2);
    if (e != cudaSuccess) return e;
    attr_done.fetch_or(bit);
  }
  // persistent grids: every CTA is resident at once (two pass-1 CTAs per SM, one
  // pass-2 CTA), so a CTA of the next kernel that waits for tensor memory only
  // waits for CTAs that are already running
  const int g1 = std::min(ntiles, 2 * num_sms), g2 = std::min(ntiles, num_sms);
  e = pdl_launch(k1, dim3(g1), dim3(kThreads), (size_t)X::SMEM1, s, a, blob, trace);
  if (e != cudaSuccess) return e;
  note_launch();
  e = pdl_launch(k2, dim3(g2), dim3(kThreads), (size_t)X::SMEM2, s, a, blob, (const float*)trace);
  if (e != cudaSuccess) return e;
  note_launch();
  return cudaGetLastError();
}

template <int P>
void build_t(const RefElement& r, std::vector<double>& out) {
  using X = T5<P>;
  constexpr int NP = X::NP, NFP = X::NFP, NF = X::NF, KF = X::KF;
  out.assign(X::CALL, 0.0);
  const double* D[3] = {r.Dr.data(), r.Ds.data(), r.Dt.data()};
  auto b1 = [&](int n, int k, double v) { out[X::CB1 + opidx(X::N1, n, k)] = v; };
  auto b2 = [&](int n, int k, double v) { out[X::CB2 + opidx(X::N2, n, k)] = v; };
  for (int rr = 0; rr < 3; ++rr)
    for (int i = 0; i < NP; ++i)
      for (int k = 0; k < NP; ++k) b1(rr * NP + i, k, D[rr][i * NP + k]);  // gr_r[i] = sum_k D_r[i][k] x[k]
  for (int f = 0; f < NF; ++f)
    for (int rr = 0; rr < 3; ++rr)
      for (int j = 0; j < NFP; ++j) {
        const int mj = r.fmask[f * NFP + j];
        for (int k = 0; k < NP; ++k) b1(X::NG + f * X::FT + rr * NFP + j, k, D[rr][mj * NP + k]);
      }
  for (int i = 0; i < NP; ++i) {
    for (int rr = 0; rr < 3; ++rr) {
      for (int n = 0; n < NP; ++n) {  // (M^T D_r)[n][i]
        double s = 0.0;
        for (int mm = 0; mm < NP; ++mm) s += r.M[mm * NP + n] * D[rr][mm * NP + i];
        b2(i, rr * NP + n, s);
      }
      for (int f = 0; f < NF; ++f)
        for (int j = 0; j < NFP; ++j) {  // (EMAT^T D_r)[k][i]
          const int k = f * NFP + j;
          double s = 0.0;
          for (int mm = 0; mm < NP; ++mm) s += r.EMAT[mm * KF + k] * D[rr][mm * NP + i];
          b2(i, X::OFF_F + f * X::KFACE + rr * NFP + j, s);
        }
    }
    for (int f = 0; f < NF; ++f)
      for (int j = 0; j < NFP; ++j) b2(i, X::OFF_F + f * X::KFACE + 3 * NFP + j, r.EMAT[i * KF + f * NFP + j]);
    for (int n = 0; n < NP; ++n) b2(i, X::OFF_MM + n, r.M[i * NP + n]);
  }
}

}  // namespace

// Orders whose reference element matched the compile-time face masks (set by
// build_tc5_consts, which runs before any apply of that order).
static std::atomic<int> g_tc5_ready[5];

bool tc5_supported(int dim, int order) { return dim == 3 && order == 3 && g_tc5_ready[order].load() == 1; }

size_t tc5_const_values(int dim, int order) {
  if (dim == 3 && order == 3) return T5<3>::CALL;
  return 0;
}

void build_tc5_consts(int dim, int order, const RefElement& r, std::vector<double>& out) {
  out.clear();
  if (dim != 3 || order != 3) return;
  for (int f = 0; f < 4; ++f)
    for (int j = 0; j < T5<3>::NFP; ++j)
      if (r.fmask[f * T5<3>::NFP + j] != FaceMask<3>::at(f, j)) {
        g_tc5_ready[order].store(-1);
        return;
      }
  build_t<3>(r, out);
  g_tc5_ready[order].store(1);
}

cudaError_t launch_apply_tc5(int dim, int order, const ApplyArgs<float>& a, const float* blob, float* trace,
                             int num_sms, cudaStream_t s) {
  if (dim == 3 && order == 3) return launch_t<3>(a, blob, trace, num_sms, s);
  return cudaErrorNotSupported;
}

unsigned tc5_timeouts() {
  unsigned v = 0;
  cudaMemcpyFromSymbol(&v, g_tc5_timeouts, sizeof(v));
  return v;
}

}  // namespace sipg
