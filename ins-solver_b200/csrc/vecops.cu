// Vector kernels for the solvers. See vecops.cuh.

#include <stdexcept>
#include <string>

#include <algorithm>
#include <atomic>

#include <cuda_bf16.h>

#include "pdl.cuh"
#include "vecops.cuh"

namespace sipg {

static std::atomic<unsigned long long> g_launches{0};
static thread_local unsigned long long* t_recorded = nullptr;
void note_launch(unsigned n) {
  if (t_recorded) *t_recorded += n;
  else g_launches.fetch_add(n, std::memory_order_relaxed);
}
void record_launches(unsigned long long* counter) { t_recorded = counter; }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-reduce NK values; thread 0 returns the block totals in v[].
template <int NK>
__device__ __forceinline__ void block_sum(double (&v)[NK]) {
  __shared__ double sh[NK][kRedThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    double t = warp_sum(v[k]);
    if (lane == 0) sh[k][wid] = t;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      double t = lane < kRedThreads / 32 ? sh[k][lane] : 0.0;
      v[k] = warp_sum(t);
    }
  }
}

// Second stage: the last block to finish sums the partials in index order.
template <int NK>
__device__ __forceinline__ void finish(const double (&v)[NK], double* partial, unsigned* counter,
                                       double* out, int out_stride) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NK; ++k) partial[blockIdx.x * 4 + k] = v[k];
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double acc[NK];
#pragma unroll
  for (int k = 0; k < NK; ++k) acc[k] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < NK; ++k) acc[k] += ((volatile double*)partial)[b * 4 + k];
  block_sum<NK>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NK; ++k) out[k * out_stride] = acc[k];
    *counter = 0u;
  }
}

template <typename T, int NK>
__global__ void __launch_bounds__(kRedThreads) k_multi_dot(const T* a0, const T* b0, const T* a1,
                                                           const T* b1, const T* a2, const T* b2,
                                                           size_t n, double* partial,
                                                           unsigned* counter, double* out,
                                                           int out_stride) {
  pdl_enter();
  double v[NK];
#pragma unroll
  for (int k = 0; k < NK; ++k) v[k] = 0.0;
  #pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    v[0] += (double)a0[i] * (double)b0[i];
    if (NK > 1) v[1 % NK] += (double)a1[i] * (double)b1[i];
    if (NK > 2) v[2 % NK] += (double)a2[i] * (double)b2[i];
  }
  block_sum<NK>(v);
  finish<NK>(v, partial, counter, out, out_stride);
}

__global__ void __launch_bounds__(kRedThreads) k_dot_diff(const double* r, const double* z, const double* zo,
                                                          size_t n, double* partial, unsigned* counter,
                                                          double* out) {
  pdl_enter();
  double v[1] = {0.0};
  #pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    v[0] += r[i] * (z[i] - zo[i]);
  block_sum<1>(v);
  finish<1>(v, partial, counter, out, 1);
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_sum(const T* a, size_t n, double* partial,
                                                     unsigned* counter, double* out) {
  pdl_enter();
  double v[1] = {0.0};
  #pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    v[0] += (double)a[i];
  block_sum<1>(v);
  finish<1>(v, partial, counter, out, 1);
}

__global__ void __launch_bounds__(kRedThreads) k_cg_update_xr(double* x, double* r, const double* p,
                                                              const double* Ap, size_t n,
                                                              const double* scal, int num, int den,
                                                              double* partial, unsigned* counter,
                                                              double* rr_out) {
  pdl_enter();
  const double alpha = scal[num] / scal[den];
  double v[1] = {0.0};
  #pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    v[0] += ri * ri;
  }
  block_sum<1>(v);
  finish<1>(v, partial, counter, rr_out, 1);
}

// x += alpha p ; r -= alpha Ap ; out[0] = sum r, out[stride] = r . r
__global__ void __launch_bounds__(kRedThreads) k_cg_update_xr_sum(double* x, double* r, const double* p,
                                                                  const double* Ap, size_t n, const double* scal,
                                                                  int num, int den, double* partial,
                                                                  unsigned* counter, double* out, int stride) {
  pdl_enter();
  const double alpha = scal[num] / scal[den];
  double v[2] = {0.0, 0.0};
  #pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    v[0] += ri;
    v[1] += ri * ri;
  }
  block_sum<2>(v);
  finish<2>(v, partial, counter, out, stride);
}

// r -= mean (scal[mean_slot] / n; none when mean_slot < 0); r32 = (float) r;
// out[0] = r . r, out[stride] = r . zo
__global__ void __launch_bounds__(kRedThreads) k_resid_prep(double* r, float* r32, const double* zo, size_t n,
                                                            const double* scal, int mean_slot, double* partial,
                                                            unsigned* counter, double* out, int stride) {
  pdl_enter();
  const double m = mean_slot >= 0 ? scal[mean_slot] / (double)n : 0.0;
  double v[2] = {0.0, 0.0};
  #pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double ri = r[i];
    if (mean_slot >= 0) {
      ri -= m;
      r[i] = ri;
    }
    r32[i] = (float)ri;
    v[0] += ri * ri;
    v[1] += ri * zo[i];
  }
  block_sum<2>(v);
  finish<2>(v, partial, counter, out, stride);
}

// z = (double) z32 ; out = sum z
__global__ void __launch_bounds__(kRedThreads) k_to_f64_sum(double* z, const float* z32, size_t n, double* partial,
                                                            unsigned* counter, double* out) {
  pdl_enter();
  double v[1] = {0.0};
  #pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double zi = (double)z32[i];
    z[i] = zi;
    v[0] += zi;
  }
  block_sum<1>(v);
  finish<1>(v, partial, counter, out, 1);
}

// z = (z32 ? (double) z32 : z) - mean (scal[mean_slot] / n; none when mean_slot < 0); out = r . z
__global__ void __launch_bounds__(kRedThreads) k_finish_z_dot(double* z, const float* z32, const double* r,
                                                              size_t n, const double* scal, int mean_slot,
                                                              double* partial, unsigned* counter, double* out) {
  pdl_enter();
  const double m = mean_slot >= 0 ? scal[mean_slot] / (double)n : 0.0;
  double v[1] = {0.0};
  #pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double zi = z32 ? (double)z32[i] : z[i];
    if (mean_slot >= 0) zi -= m;
    z[i] = zi;
    v[0] += r[i] * zi;
  }
  block_sum<1>(v);
  finish<1>(v, partial, counter, out, 1);
}

// x += alpha p ; r -= alpha Ap ; out[0] = r . r, out[stride] = r . zo
__global__ void __launch_bounds__(kRedThreads) k_cg_update_xr_rzo(double* x, double* r, const double* p,
                                                                  const double* Ap, const double* zo, size_t n,
                                                                  const double* scal, int num, int den,
                                                                  double* partial, unsigned* counter, double* out,
                                                                  int stride) {
  pdl_enter();
  const double alpha = scal[num] / scal[den];
  double v[2] = {0.0, 0.0};
#pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    v[0] += ri * ri;
    v[1] += ri * zo[i];
  }
  block_sum<2>(v);
  finish<2>(v, partial, counter, out, stride);
}

// z = B r (row-major blocks; point Jacobi z = dinv r when Np == 0) ; out = r . z
__global__ void __launch_bounds__(kRedThreads) k_precond_dot(double* z, const double* r, const double* B, int Np,
                                                             size_t n, double* partial, unsigned* counter,
                                                             double* out) {
  pdl_enter();
  double v[1] = {0.0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double zi;
    if (Np > 0) {
      const size_t b = i / Np;
      const int row = (int)(i - b * Np);
      const double* Bb = B + (b * Np + row) * Np;
      const double* rb = r + b * Np;
      zi = 0.0;
      for (int j = 0; j < Np; ++j) zi += Bb[j] * rb[j];
    } else {
      zi = B[i] * r[i];
    }
    z[i] = zi;
    v[0] += r[i] * zi;
  }
  block_sum<1>(v);
  finish<1>(v, partial, counter, out, 1);
}

template <typename T>
__global__ void k_update_p(T* p, const T* z, size_t n, const double* scal, int num, int den) {
  pdl_enter();
  const T beta = (T)(scal[num] / scal[den]);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

template <typename T>
__global__ void k_sub_mean(T* v, size_t n, const double* scal, int slot) {
  pdl_enter();
  const T mean = (T)(scal[slot] / (double)n);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    v[i] -= mean;
}

template <typename T>
__global__ void k_copy(T* d, const T* s, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) d[i] = s[i];
}
template <typename T>
__global__ void k_zero(T* d, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) d[i] = T(0);
}
__global__ void k_to_f32(float* d, const double* s, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) d[i] = (float)s[i];
}
__global__ void k_to_f64(double* d, const float* s, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) d[i] = (double)s[i];
}
template <typename T>
__global__ void k_jacobi(T* z, const T* r, const T* dinv, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) z[i] = dinv[i] * r[i];
}
template <typename T>
__global__ void k_cheb(T* d, T* z, const T* res, const T* dinv, T c1, T c2, size_t n, int first) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    T di = (c1 != T(0) ? c1 * d[i] : T(0)) + c2 * dinv[i] * res[i];
    d[i] = di;
    z[i] = first ? di : z[i] + di;
  }
}

// Element-block Jacobi Chebyshev step with the inverse diagonal blocks stored as
// packed symmetric triangles (value t = c (c + 1) / 2 + r, r <= c): Np (Np + 1) / 2
// values per block instead of Np^2 (p = 3, BF16: 420 B instead of 800 B per
// element). The values are grouped in 16-byte chunks of CH = 16 / sizeof(TB),
// chunk k of block b at P[(k * nb + b) * CH], so one thread reads its block with
// 16-byte loads and a warp's loads of one chunk are contiguous. One thread per block:
//   d <- c1 d + c2 B res ; z += d  (first: z = d; c1 == 0 reads no d).
template <typename TB> struct Chunk;
template <> struct Chunk<__nv_bfloat16> {
  static constexpr int CH = 8;
  // value j (0..7) of a chunk: bf16 is the upper half of an fp32
  static __device__ __forceinline__ float at(const uint4& q, int j) {
    const unsigned w = j < 2 ? q.x : j < 4 ? q.y : j < 6 ? q.z : q.w;
    return __uint_as_float((j & 1) ? (w & 0xffff0000u) : (w << 16));
  }
};
template <> struct Chunk<double> {
  static constexpr int CH = 2;
  static __device__ __forceinline__ double at(const uint4& q, int j) {
    return j == 0 ? __hiloint2double((int)q.y, (int)q.x) : __hiloint2double((int)q.w, (int)q.z);
  }
};

// BT threads (= elements) per CTA (SymCfg::BT, or 16 on meshes too small to give
// every SM a CTA of that size); the res, d and z rows of the CTA's elements pass
// through shared memory (row stride NP + 1) so that global loads and stores are
// contiguous.
template <typename T, int NP>
struct SymCfg {
  static constexpr int BT = 3 * 64 * (NP + 1) * (int)sizeof(T) <= 40 * 1024 ? 64 : 32;
  static constexpr int LD = NP + 1;
};

template <typename T, typename TB, int NP, int BT>
__global__ void __launch_bounds__(BT) k_cheb_sym(T* d, T* z, const T* __restrict__ res, const TB* __restrict__ P,
                                                 T c1, T c2, int nb, int first) {
  pdl_enter();
  using C = Chunk<TB>;
  constexpr int LD = SymCfg<T, NP>::LD;
  constexpr int NK = (NP * (NP + 1) / 2 + C::CH - 1) / C::CH;  // 16-byte chunks per block
  // the first PF chunks (at most 56 registers) are requested before the staging
  // loads, so that their latency overlaps; the rest are read during the products
  constexpr int PF = NK < 14 ? NK : 14;
  __shared__ T sr[BT * LD], sd[BT * LD], sz[BT * LD];
  const int tid = threadIdx.x;
  const bool use_d = c1 != T(0);
  for (size_t e0 = (size_t)blockIdx.x * BT; e0 < (size_t)nb; e0 += (size_t)gridDim.x * BT) {
    const int ne = (size_t)nb - e0 < (size_t)BT ? (int)((size_t)nb - e0) : BT;
    const size_t g0 = e0 * NP;
    const uint4* pb = reinterpret_cast<const uint4*>(P) + e0 + tid;
    uint4 qa[PF];
    if (tid < ne) {
#pragma unroll
      for (int k = 0; k < PF; ++k) qa[k] = pb[(size_t)k * nb];
    }
    if (ne == BT) {  // full group: every load issued back to back
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        const int i = tid + k * BT, s = (i / NP) * LD + i % NP;
        sr[s] = res[g0 + i];
        if (use_d) sd[s] = d[g0 + i];
        if (!first) sz[s] = z[g0 + i];
      }
    } else {
      for (int i = tid; i < ne * NP; i += BT) {
        const int s = (i / NP) * LD + i % NP;
        sr[s] = res[g0 + i];
        if (use_d) sd[s] = d[g0 + i];
        if (!first) sz[s] = z[g0 + i];
      }
    }
    __syncthreads();
    if (tid < ne) {
      const T* rr = sr + tid * LD;
      T y[NP];
#pragma unroll
      for (int i = 0; i < NP; ++i) y[i] = T(0);
      uint4 q = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
      for (int c = 0; c < NP; ++c) {
        const T rc = rr[c];
#pragma unroll
        for (int k = 0; k <= c; ++k) {
          const int t = c * (c + 1) / 2 + k;
          if (t / C::CH < PF) q = qa[t / C::CH < PF ? t / C::CH : 0];
          else if (t % C::CH == 0) q = pb[(size_t)(t / C::CH) * nb];
          const T v = (T)C::at(q, t % C::CH);
          y[k] += v * rc;
          if (k != c) y[c] += v * rr[k];
        }
      }
      T* dd = sd + tid * LD;
      T* zz = sz + tid * LD;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const T di = (use_d ? c1 * dd[i] : T(0)) + c2 * y[i];
        dd[i] = di;
        zz[i] = first ? di : zz[i] + di;
      }
    }
    __syncthreads();
    if (ne == BT) {
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        const int i = tid + k * BT, s = (i / NP) * LD + i % NP;
        d[g0 + i] = sd[s];
        z[g0 + i] = sz[s];
      }
    } else {
      for (int i = tid; i < ne * NP; i += BT) {
        const int s = (i / NP) * LD + i % NP;
        d[g0 + i] = sd[s];
        z[g0 + i] = sz[s];
      }
    }
    __syncthreads();
  }
}

// Row-major FP64 blocks -> packed symmetric triangles in TB (the mean of the two
// triangles, so the stored block is exactly symmetric); chunk padding is zero.
__device__ __forceinline__ void blk_store(__nv_bfloat16* p, double v) { *p = __double2bfloat16(v); }
__device__ __forceinline__ void blk_store(float* p, double v) { *p = (float)v; }
__device__ __forceinline__ void blk_store(double* p, double v) { *p = v; }
template <typename TB>
__global__ void k_block_pack_sym(TB* P, const double* B, int nb, int Np) {
  pdl_enter();
  constexpr int CH = Chunk<TB>::CH;
  const int nt = Np * (Np + 1) / 2, nk = (nt + CH - 1) / CH;
  const size_t total = (size_t)nb * nk * CH;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(i % CH);
    const size_t kb = i / CH;
    const int k = (int)(kb / (size_t)nb);
    const size_t b = kb - (size_t)k * nb;
    const int t = k * CH + j;
    double v = 0.0;
    if (t < nt) {
      int c = 0;
      while ((c + 1) * (c + 2) / 2 <= t) ++c;
      const int r = t - c * (c + 1) / 2;
      const double* Bb = B + b * Np * Np;
      v = r == c ? Bb[r * Np + c] : 0.5 * (Bb[r * Np + c] + Bb[c * Np + r]);
    }
    blk_store(P + i, v);
  }
}

// Full-block form of the element-block Jacobi step (meshes too small for one thread
// per block to fill the GPU): d <- c1 d + c2 B res,
// z += d; B holds the inverse diagonal blocks column by column (Bc[b][c][r]) so
// that the threads of one block read consecutive addresses.
__device__ __forceinline__ float blk_val(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ float blk_val(const float* p) { return *p; }
__device__ __forceinline__ double blk_val(const double* p) { return *p; }

template <typename T, typename TB>
__global__ void k_cheb_block(T* d, T* z, const T* res, const TB* Bc, T c1, T c2, int nb, int Np, int first) {
  pdl_enter();
  const size_t total = (size_t)nb * Np;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t b = i / Np;
    const int r = (int)(i % Np);
    const TB* Bb = Bc + b * Np * Np + r;
    const T* rb = res + b * Np;
    T s = T(0);
    for (int c = 0; c < Np; ++c) s += (T)blk_val(Bb + (size_t)c * Np) * rb[c];
    const T di = (c1 != T(0) ? c1 * d[i] : T(0)) + c2 * s;
    d[i] = di;
    z[i] = first ? di : z[i] + di;
  }
}

template <typename TB> struct Pair;
template <> struct Pair<__nv_bfloat16> {
  static __device__ __forceinline__ float2 ld(const __nv_bfloat16* p) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
  }
};
template <> struct Pair<float> {
  static __device__ __forceinline__ float2 ld(const float* p) { return *reinterpret_cast<const float2*>(p); }
};
template <> struct Pair<double> {
  static __device__ __forceinline__ double2 ld(const double* p) { return *reinterpret_cast<const double2*>(p); }
};
template <typename T> struct Vec2;
template <> struct Vec2<float> { using t = float2; };
template <> struct Vec2<double> { using t = double2; };

// Same step, two rows per thread with paired loads (even Np).
template <typename T, typename TB>
__global__ void k_cheb_block2(T* d, T* z, const T* res, const TB* Bc, T c1, T c2, int nb, int Np, int first) {
  pdl_enter();
  using V = typename Vec2<T>::t;
  const int hp = Np / 2;
  const size_t total = (size_t)nb * hp;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t b = i / hp;
    const int r = 2 * (int)(i % hp);
    const TB* Bb = Bc + b * Np * Np + r;
    const T* rb = res + b * Np;
    T s0 = T(0), s1 = T(0);
    for (int c = 0; c < Np; ++c) {
      const auto v = Pair<TB>::ld(Bb + (size_t)c * Np);
      const T rc = rb[c];
      s0 += (T)v.x * rc;
      s1 += (T)v.y * rc;
    }
    const size_t o = b * Np + r;
    V dv{T(0), T(0)}, zv{T(0), T(0)};
    if (c1 != T(0)) dv = *reinterpret_cast<const V*>(d + o);
    if (!first) zv = *reinterpret_cast<const V*>(z + o);
    dv.x = c1 * dv.x + c2 * s0;
    dv.y = c1 * dv.y + c2 * s1;
    zv.x += dv.x;
    zv.y += dv.y;
    *reinterpret_cast<V*>(d + o) = dv;
    *reinterpret_cast<V*>(z + o) = zv;
  }
}

// Row-major FP64 blocks -> column-major blocks in T.
template <typename T>
__global__ void k_block_transpose(T* dst, const double* src, int nb, int Np) {
  pdl_enter();
  const size_t total = (size_t)nb * Np * Np;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t b = i / ((size_t)Np * Np);
    const int q = (int)(i % ((size_t)Np * Np));
    const int c = q / Np, r = q % Np;
    blk_store(dst + i, src[(b * Np + r) * Np + c]);
  }
}

// One warp per block row set: thread handles (block, row).
template <typename T>
__global__ void k_block_matvec(T* y, const T* B, const T* x, int nb, int Np) {
  pdl_enter();
  const size_t total = (size_t)nb * Np;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t b = i / Np;
    const int r = (int)(i % Np);
    const T* Bb = B + (b * Np + r) * Np;
    const T* xb = x + b * Np;
    double s = 0.0;
    for (int j = 0; j < Np; ++j) s += (double)Bb[j] * (double)xb[j];
    y[i] = (T)s;
  }
}

template <typename T>
__global__ void k_inv_mass(T* y, const T* x, const T* Minv, const T* geof, int ngeof, int jidx, int K,
                           int Np, int ncomp, T scale) {
  pdl_enter();
  const size_t total = (size_t)ncomp * K * Np;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t be = i / Np;
    const int r = (int)(i % Np);
    const int e = (int)(be % K);
    const T* xb = x + be * Np;
    T s = T(0);
    for (int j = 0; j < Np; ++j) s += Minv[r * Np + j] * xb[j];
    y[i] = scale * s / geof[(size_t)e * ngeof + jidx];
  }
}

// Fixed-size inverse mass: a block stages the rows of 128 elements with coalesced
// loads, each thread applies M^-1 (shared, broadcast reads) to one element's row
// and the block stores the rows back coalesced.
template <typename T, int NP>
__global__ void __launch_bounds__(128) k_inv_mass_n(T* __restrict__ y, const T* __restrict__ x,
                                                     const T* __restrict__ Minv, const T* __restrict__ geof,
                                                     int ngeof, int jidx, int K, int nrows, T scale) {
  __shared__ T sM[NP * NP];
  __shared__ T sx[128 * NP];
  for (int i = threadIdx.x; i < NP * NP; i += blockDim.x) sM[i] = Minv[i];  // set-up data
  pdl_enter();
  for (size_t b0 = (size_t)blockIdx.x * 128; b0 < (size_t)nrows; b0 += (size_t)gridDim.x * 128) {
    const int nb = (int)min((size_t)128, (size_t)nrows - b0);
    __syncthreads();
    for (int i = threadIdx.x; i < nb * NP; i += blockDim.x) sx[i] = x[b0 * NP + i];
    __syncthreads();
    if ((int)threadIdx.x < nb) {
      const size_t be = b0 + threadIdx.x;
      const T* xr = sx + threadIdx.x * NP;
      T xv[NP];
#pragma unroll
      for (int j = 0; j < NP; ++j) xv[j] = xr[j];
      const T sc = scale / geof[(be % (size_t)K) * ngeof + jidx];
      T* yr = sx + threadIdx.x * NP;
      // four rows at a time: independent accumulators hide the FMA latency
      constexpr int R4 = NP / 4 * 4;
#pragma unroll
      for (int r = 0; r < R4; r += 4) {
        T s0 = T(0), s1 = T(0), s2 = T(0), s3 = T(0);
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          const T v = xv[j];
          s0 += sM[r * NP + j] * v;
          s1 += sM[(r + 1) * NP + j] * v;
          s2 += sM[(r + 2) * NP + j] * v;
          s3 += sM[(r + 3) * NP + j] * v;
        }
        yr[r] = sc * s0;
        yr[r + 1] = sc * s1;
        yr[r + 2] = sc * s2;
        yr[r + 3] = sc * s3;
      }
#pragma unroll
      for (int r = R4; r < NP; ++r) {
        T s0 = T(0);
#pragma unroll
        for (int j = 0; j < NP; ++j) s0 += sM[r * NP + j] * xv[j];
        yr[r] = sc * s0;
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb * NP; i += blockDim.x) y[b0 * NP + i] = sx[i];
  }
}

// In-place blocked Gauss-Jordan inversion of a dense n x n matrix (row-major,
// FP64). For each pivot block K of GJB rows and columns, with P = A_KK^-1:
//   A_Kj <- P A_Kj                  (j not in K; k_gjb_row)
//   A_ij <- A_ij - A_iK A_Kj        (i, j not in K, with the new A_Kj; k_gjb_update)
//   A_iK <- -A_iK P, A_KK <- P      (i not in K; k_gjb_col)
// which is scalar Gauss-Jordan applied GJB pivots at a time: the trailing update
// is a rank-GJB product over 64 x 64 tiles instead of n rank-1 passes.
// No pivoting: the coarsest algebraic operator is symmetric positive definite
// (a singular one is shifted first), so every pivot block is.
constexpr int GJB = 32;

// P = A_KK^-1 by scalar Gauss-Jordan in one warp: lane i holds row i of the pivot block
// in registers and the pivot row reaches every lane by shuffles (no barriers); P is
// GJB x GJB (GJB = 32, one row per lane), zero outside the bs x bs block.
static_assert(GJB == 32, "one pivot-block row per lane");
__global__ void __launch_bounds__(32) k_gjb_pivot(const double* __restrict__ a, int n, int k0, int bs,
                                                  double* __restrict__ P) {
  const int i = threadIdx.x;
  double row[GJB];
#pragma unroll
  for (int j = 0; j < GJB; ++j) row[j] = (i < bs && j < bs) ? a[(size_t)(k0 + i) * n + k0 + j] : 0.0;
#pragma unroll
  for (int k = 0; k < GJB; ++k) {
    if (k >= bs) break;  // uniform across the warp
    const double r = 1.0 / __shfl_sync(0xffffffffu, row[k], k);
    // the pivot row scaled by r (its column k stays until the column step)
    if (i == k) {
#pragma unroll
      for (int j = 0; j < GJB; ++j)
        if (j != k) row[j] *= r;
    }
    const double aik = row[k];
#pragma unroll
    for (int j = 0; j < GJB; ++j) {
      const double akj = __shfl_sync(0xffffffffu, row[j], k);
      if (i != k && j != k) row[j] -= aik * akj;
    }
    row[k] = i == k ? r : row[k] * -r;
  }
#pragma unroll
  for (int j = 0; j < GJB; ++j) P[i * GJB + j] = (i < bs && j < bs) ? row[j] : 0.0;
}

// Row panel: one thread per column j outside K.
__global__ void __launch_bounds__(256) k_gjb_row(double* __restrict__ a, int n, int k0, int bs,
                                                 const double* __restrict__ P) {
  __shared__ double sp[GJB * GJB];
  for (int t = threadIdx.x; t < GJB * GJB; t += blockDim.x) sp[t] = P[t];
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n || (j >= k0 && j < k0 + bs)) return;
  double col[GJB];
#pragma unroll
  for (int m = 0; m < GJB; ++m) col[m] = m < bs ? a[(size_t)(k0 + m) * n + j] : 0.0;
#pragma unroll
  for (int i = 0; i < GJB; ++i) {
    if (i >= bs) break;
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < GJB; ++m) s += sp[i * GJB + m] * col[m];
    a[(size_t)(k0 + i) * n + j] = s;
  }
}

// Trailing update over 64 x 64 tiles, 256 threads, 4 x 4 entries per thread
// (rows ty + 16 u, columns tx + 16 v: coalesced loads and stores).
__global__ void __launch_bounds__(256) k_gjb_update(double* __restrict__ a, int n, int k0, int bs) {
  __shared__ double sc[64][GJB + 1];  // A_iK of the tile's rows
  __shared__ double sw[GJB][64 + 1];  // A_Kj of the tile's columns
  const int i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  for (int t = threadIdx.x; t < 64 * GJB; t += 256) {
    const int r = t / GJB, m = t % GJB;
    sc[r][m] = (i0 + r < n && m < bs) ? a[(size_t)(i0 + r) * n + k0 + m] : 0.0;
  }
  for (int t = threadIdx.x; t < GJB * 64; t += 256) {
    const int m = t / 64, c = t % 64;
    sw[m][c] = (j0 + c < n && m < bs) ? a[(size_t)(k0 + m) * n + j0 + c] : 0.0;
  }
  __syncthreads();
  double acc[4][4] = {};
#pragma unroll 8
  for (int m = 0; m < GJB; ++m) {
    double cv[4], wv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) cv[u] = sc[ty + 16 * u][m];
#pragma unroll
    for (int v = 0; v < 4; ++v) wv[v] = sw[m][tx + 16 * v];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] += cv[u] * wv[v];
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int i = i0 + ty + 16 * u;
    if (i >= n || (i >= k0 && i < k0 + bs)) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int j = j0 + tx + 16 * v;
      if (j >= n || (j >= k0 && j < k0 + bs)) continue;
      a[(size_t)i * n + j] -= acc[u][v];
    }
  }
}

// Column panel: one thread per row i; rows of K receive P.
__global__ void __launch_bounds__(128) k_gjb_col(double* __restrict__ a, int n, int k0, int bs,
                                                 const double* __restrict__ P) {
  __shared__ double sp[GJB * GJB];
  for (int t = threadIdx.x; t < GJB * GJB; t += blockDim.x) sp[t] = P[t];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* row = a + (size_t)i * n + k0;
  if (i >= k0 && i < k0 + bs) {
    for (int j = 0; j < bs; ++j) row[j] = sp[(i - k0) * GJB + j];
    return;
  }
  double rv[GJB];
#pragma unroll
  for (int m = 0; m < GJB; ++m) rv[m] = m < bs ? row[m] : 0.0;
#pragma unroll
  for (int j = 0; j < GJB; ++j) {
    if (j >= bs) break;
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < GJB; ++m) s += rv[m] * sp[m * GJB + j];
    row[j] = -s;
  }
}
// Row sums, column sums and the total of a dense matrix (one thread per row /
// column; the total from the row sums in a fixed order).
__global__ void k_dense_sums(const double* a, int n, double* rs, double* cs) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * n; t += gridDim.x * blockDim.x) {
    double s = 0.0;
    if (t < n)
      for (int j = 0; j < n; ++j) s += a[(size_t)t * n + j];
    else
      for (int i = 0; i < n; ++i) s += a[(size_t)i * n + (t - n)];
    (t < n ? rs[t] : cs[t - n]) = s;
  }
}
// Q a Q with Q = I - 11^T / n: a_ij - rs_i / n - cs_j / n + total / n^2.
__global__ void k_dense_project(double* a, int n, const double* rs, const double* cs) {
  __shared__ double total;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += rs[i];
    total = s;
  }
  __syncthreads();
  const double dn = (double)n;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)n * n;
       t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t / n), j = (int)(t - (size_t)i * n);
    a[t] += -rs[i] / dn - cs[j] / dn + total / (dn * dn);
  }
}

template <typename T>
__global__ void k_restrict(T* rc, const T* r, const T* P, int K, int Npf, int Npc, int ncomp) {
  pdl_enter();
  const size_t total = (size_t)ncomp * K * Npc;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t be = i / Npc;
    const int j = (int)(i % Npc);
    const T* rb = r + be * Npf;
    T s = T(0);
    for (int k = 0; k < Npf; ++k) s += P[k * Npc + j] * rb[k];
    rc[i] = s;
  }
}

// Fixed-size transfers: P (Npf x Npc) in shared memory, loops unrolled.
template <typename T, int NPF, int NPC>
__global__ void k_restrict_n(T* rc, const T* __restrict__ r, const T* __restrict__ P, size_t total) {
  __shared__ T sP[NPF * NPC];
  for (int i = threadIdx.x; i < NPF * NPC; i += blockDim.x) sP[i] = P[i];  // set-up data
  __syncthreads();
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t be = i / NPC;
    const int j = (int)(i - be * NPC);
    const T* rb = r + be * NPF;
    T s = T(0);
#pragma unroll
    for (int k = 0; k < NPF; ++k) s += sP[k * NPC + j] * rb[k];
    rc[i] = s;
  }
}
template <typename T, int NPF, int NPC>
__global__ void k_prolong_add_n(T* z, const T* __restrict__ zc, const T* __restrict__ P, size_t total) {
  __shared__ T sP[NPF * NPC];
  for (int i = threadIdx.x; i < NPF * NPC; i += blockDim.x) sP[i] = P[i];  // set-up data
  __syncthreads();
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t be = i / NPF;
    const int k = (int)(i - be * NPF);
    const T* zb = zc + be * NPC;
    T s = T(0);
#pragma unroll
    for (int j = 0; j < NPC; ++j) s += sP[k * NPC + j] * zb[j];
    z[i] += s;
  }
}

template <typename T>
__global__ void k_prolong_add(T* z, const T* zc, const T* P, int K, int Npf, int Npc, int ncomp) {
  pdl_enter();
  const size_t total = (size_t)ncomp * K * Npf;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t be = i / Npf;
    const int k = (int)(i % Npf);
    const T* zb = zc + be * Npc;
    T s = T(0);
    for (int j = 0; j < Npc; ++j) s += P[k * Npc + j] * zb[j];
    z[i] += s;
  }
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_coarse_update(T* z, T* r, T* sv, const T* p, const T* Ap,
                                                               const T* dinv, size_t n, double* scal,
                                                               double* partial, unsigned* counter) {
  pdl_enter();
  const double pap = scal[S_C_PAP];
  const bool ok = pap > 0.0 && scal[S_C_RZ] > 0.0;
  const T alpha = ok ? (T)(scal[S_C_RZ] / pap) : T(0);
  double v[1] = {0.0};
  #pragma unroll 4
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    z[i] += alpha * p[i];
    T ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    T si = dinv[i] * ri;
    sv[i] = si;
    v[0] += (double)ri * (double)si;
  }
  block_sum<1>(v);
  finish<1>(v, partial, counter, scal + S_C_RZN, 1);
}

template <typename T>
__global__ void k_coarse_update_p(T* p, const T* sv, size_t n, double* scal) {
  pdl_enter();
  const double rz = scal[S_C_RZ];
  const T beta = rz > 0.0 ? (T)(scal[S_C_RZN] / rz) : T(0);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] = sv[i] + beta * p[i];
}

__global__ void k_shift_scalar(double* scal, int from, int to) {
  pdl_enter(); scal[to] = scal[from]; }

// Eight lanes per row (the algebraic levels are small: parallelism, not bytes, limits them).
template <typename T>
__global__ void k_csr_spmv(int rows, const int* __restrict__ ptr, const int* __restrict__ idx,
                           const T* __restrict__ val, const T* __restrict__ x, T* y, T alpha, T beta, const T* c) {
  pdl_enter();
  const int lane = threadIdx.x & 31, sub = lane & 7;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; 4 * w < rows; w += warps) {
    const int r = 4 * w + (lane >> 3);
    T s = T(0);
    if (r < rows)
      for (int k = ptr[r] + sub; k < ptr[r + 1]; k += 8) s += val[k] * x[idx[k]];
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, 8);
    if (r < rows && sub == 0) y[r] = beta != T(0) ? alpha * s + beta * c[r] : alpha * s;
  }
}

// One Chebyshev step of an algebraic level fused with its residual update, eight
// lanes per row:  dn = c1 d + c2 dinv r ; z = (first ? 0 : z) + dn ; rn = r - A dn
// (rn skipped when null). d and r are only read (rows read their neighbours'
// entries), dn and rn are other buffers; c1 == 0 reads no d.
template <typename T>
__device__ __forceinline__ T cheb_dir(const T* d, const T* r, const T* dinv, int j, T c1, T c2) {
  return (c1 != T(0) ? c1 * d[j] : T(0)) + c2 * dinv[j] * r[j];
}
template <typename T>
__global__ void k_csr_cheb(int rows, const int* __restrict__ ptr, const int* __restrict__ idx,
                           const T* __restrict__ val, const T* __restrict__ d, const T* __restrict__ r,
                           const T* __restrict__ dinv, T* __restrict__ dn, T* __restrict__ rn, T* z, T c1, T c2,
                           int first) {
  pdl_enter();
  const int lane = threadIdx.x & 31, sub = lane & 7;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; 4 * w < rows; w += warps) {
    const int i = 4 * w + (lane >> 3);
    T s = T(0);
    if (i < rows && rn)
      for (int k = ptr[i] + sub; k < ptr[i + 1]; k += 8) s += val[k] * cheb_dir(d, r, dinv, idx[k], c1, c2);
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, 8);
    if (i < rows && sub == 0) {
      const T di = cheb_dir(d, r, dinv, i, c1, c2);
      dn[i] = di;
      z[i] = first ? di : z[i] + di;
      if (rn) rn[i] = r[i] - s;
    }
  }
}

// One warp per row of a dense matrix.
template <typename T>
__global__ void k_dense_mv(int n, const T* __restrict__ M, const T* __restrict__ x, T* y) {
  pdl_enter();
  const int lane = threadIdx.x & 31;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += (gridDim.x * blockDim.x) >> 5) {
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += (double)M[(size_t)r * n + j] * (double)x[j];
    s = warp_sum(s);
    if (lane == 0) y[r] = (T)s;
  }
}

template <typename T>
__global__ void k_vadd(T* y, const T* x, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) y[i] += x[i];
}

// Reduction grid: one element per thread for short vectors (up to 296 CTAs),
// about eight per thread for long ones, at most kRedBlocks CTAs (the partial sums
// depend on n only, so results stay reproducible).
inline int red_grid(size_t n) {
  const size_t short_grid = std::min<size_t>((n + kRedThreads - 1) / kRedThreads, 296);
  const size_t long_grid = (n + 8 * kRedThreads - 1) / (8 * kRedThreads);
  return (int)std::max<size_t>(1, std::min<size_t>(kRedBlocks, std::max(short_grid, long_grid)));
}
inline int grid_for(size_t n) {
  size_t g = (n + 255) / 256;
  return (int)std::max<size_t>(1, std::min<size_t>(g, 148 * 16));
}

}  // namespace

template <typename T>
void multi_dot(const T* const* a, const T* const* b, int nk, size_t n, double* out, int out_stride,
               const RedWork& w, cudaStream_t s) {
  if (nk == 1)
    pdl_launch(k_multi_dot<T, 1>, dim3(red_grid(n)), dim3(kRedThreads), 0, s, a[0], b[0], nullptr, nullptr, nullptr, nullptr, n,
                                                         w.partial, w.counter, out, out_stride);
  else if (nk == 2)
    pdl_launch(k_multi_dot<T, 2>, dim3(red_grid(n)), dim3(kRedThreads), 0, s, a[0], b[0], a[1], b[1], nullptr, nullptr, n,
                                                         w.partial, w.counter, out, out_stride);
  else
    pdl_launch(k_multi_dot<T, 3>, dim3(red_grid(n)), dim3(kRedThreads), 0, s, a[0], b[0], a[1], b[1], a[2], b[2], n,
                                                         w.partial, w.counter, out, out_stride);
  note_launch();
}

void dot_diff(const double* r, const double* z, const double* zo, size_t n, double* out,
              const RedWork& w, cudaStream_t s) {
  pdl_launch(k_dot_diff, dim3(red_grid(n)), dim3(kRedThreads), 0, s, r, z, zo, n, w.partial, w.counter, out);
  note_launch();
}

template <typename T>
void vsum(const T* a, size_t n, double* out, const RedWork& w, cudaStream_t s) {
  pdl_launch(k_sum<T>, dim3(red_grid(n)), dim3(kRedThreads), 0, s, a, n, w.partial, w.counter, out);
  note_launch();
}

void cg_update_xr(double* x, double* r, const double* p, const double* Ap, size_t n,
                  const double* scal, int num, int den, double* rr_out, const RedWork& w,
                  cudaStream_t s) {
  pdl_launch(k_cg_update_xr, dim3(red_grid(n)), dim3(kRedThreads), 0, s, x, r, p, Ap, n, scal, num, den, w.partial, w.counter, rr_out);
  note_launch();
}

void cg_update_xr_sum(double* x, double* r, const double* p, const double* Ap, size_t n, const double* scal, int num,
                      int den, double* out, int stride, const RedWork& w, cudaStream_t s) {
  pdl_launch(k_cg_update_xr_sum, dim3(red_grid(n)), dim3(kRedThreads), 0, s, x, r, p, Ap, n, scal, num, den, w.partial,
             w.counter, out, stride);
  note_launch();
}
void cg_update_xr_rzo(double* x, double* r, const double* p, const double* Ap, const double* zo, size_t n,
                      const double* scal, int num, int den, double* out, int stride, const RedWork& w,
                      cudaStream_t s) {
  pdl_launch(k_cg_update_xr_rzo, dim3(red_grid(n)), dim3(kRedThreads), 0, s, x, r, p, Ap, zo, n, scal, num, den,
             w.partial, w.counter, out, stride);
  note_launch();
}
void precond_dot(double* z, const double* r, const double* B, int Np, size_t n, double* out, const RedWork& w,
                 cudaStream_t s) {
  pdl_launch(k_precond_dot, dim3(red_grid(n)), dim3(kRedThreads), 0, s, z, r, B, Np, n, w.partial, w.counter, out);
  note_launch();
}
void resid_prep(double* r, float* r32, const double* zo, size_t n, const double* scal, int mean_slot, double* out,
                int stride, const RedWork& w, cudaStream_t s) {
  pdl_launch(k_resid_prep, dim3(red_grid(n)), dim3(kRedThreads), 0, s, r, r32, zo, n, scal, mean_slot, w.partial,
             w.counter, out, stride);
  note_launch();
}
void to_f64_sum(double* z, const float* z32, size_t n, double* out, const RedWork& w, cudaStream_t s) {
  pdl_launch(k_to_f64_sum, dim3(red_grid(n)), dim3(kRedThreads), 0, s, z, z32, n, w.partial, w.counter, out);
  note_launch();
}
void finish_z_dot(double* z, const float* z32, const double* r, size_t n, const double* scal, int mean_slot,
                  double* out, const RedWork& w, cudaStream_t s) {
  pdl_launch(k_finish_z_dot, dim3(red_grid(n)), dim3(kRedThreads), 0, s, z, z32, r, n, scal, mean_slot, w.partial,
             w.counter, out);
  note_launch();
}

template <typename T>
void update_p(T* p, const T* z, size_t n, const double* scal, int num, int den, cudaStream_t s) {
  pdl_launch(k_update_p<T>, dim3(grid_for(n)), dim3(256), 0, s, p, z, n, scal, num, den);
  note_launch();
}
template <typename T>
void sub_mean(T* v, size_t n, const double* scal, int slot, cudaStream_t s) {
  pdl_launch(k_sub_mean<T>, dim3(grid_for(n)), dim3(256), 0, s, v, n, scal, slot);
  note_launch();
}
template <typename T>
void vcopy(T* dst, const T* src, size_t n, cudaStream_t s) {
  pdl_launch(k_copy<T>, dim3(grid_for(n)), dim3(256), 0, s, dst, src, n);
  note_launch();
}
template <typename T>
void vzero(T* dst, size_t n, cudaStream_t s) {
  pdl_launch(k_zero<T>, dim3(grid_for(n)), dim3(256), 0, s, dst, n);
  note_launch();
}
void to_f32(float* dst, const double* src, size_t n, cudaStream_t s) {
  pdl_launch(k_to_f32, dim3(grid_for(n)), dim3(256), 0, s, dst, src, n);
  note_launch();
}
void to_f64(double* dst, const float* src, size_t n, cudaStream_t s) {
  pdl_launch(k_to_f64, dim3(grid_for(n)), dim3(256), 0, s, dst, src, n);
  note_launch();
}
template <typename T, typename TB>
void cheb_step_block(T* d, T* z, const T* res, const TB* Bc, T c1, T c2, int nb, int Np, cudaStream_t s,
                     bool first) {
  if (Np % 2 == 0)
    pdl_launch(k_cheb_block2<T, TB>, dim3(grid_for((size_t)nb * Np / 2)), dim3(256), 0, s, d, z, res, Bc, c1, c2,
               nb, Np, (int)first);
  else
    pdl_launch(k_cheb_block<T, TB>, dim3(grid_for((size_t)nb * Np)), dim3(256), 0, s, d, z, res, Bc, c1, c2, nb, Np,
               (int)first);
  note_launch();
}
template void cheb_step_block<float, __nv_bfloat16>(float*, float*, const float*, const __nv_bfloat16*, float, float,
                                                    int, int, cudaStream_t, bool);
template void block_transpose<__nv_bfloat16>(__nv_bfloat16*, const double*, int, int, cudaStream_t);
template <typename T>
void block_transpose(T* dst, const double* src, int nb, int Np, cudaStream_t s) {
  pdl_launch(k_block_transpose<T>, dim3(grid_for((size_t)nb * Np * Np)), dim3(256), 0, s, dst, src, nb, Np);
  note_launch();
}
bool block_sym_supported(int Np) {
  return Np == 3 || Np == 4 || Np == 6 || Np == 10 || Np == 15 || Np == 20 || Np == 35;
}
template <typename T, typename TB>
void cheb_step_sym(T* d, T* z, const T* res, const TB* P, T c1, T c2, int nb, int Np, cudaStream_t s, bool first) {
  const int f = first ? 1 : 0;
  auto go = [&](auto big, auto small, int bt) {
    const bool narrow = nb < 2 * 148 * bt;
    if (narrow) bt = 16;
    const dim3 g((unsigned)std::max(1, std::min((nb + bt - 1) / bt, 148 * 32)));
    if (narrow) pdl_launch(small, g, dim3(bt), 0, s, d, z, res, P, c1, c2, nb, f);
    else pdl_launch(big, g, dim3(bt), 0, s, d, z, res, P, c1, c2, nb, f);
  };
#define SIPG_SYM_CASE(N)                                                                              \
  case N:                                                                                            \
    go(k_cheb_sym<T, TB, N, SymCfg<T, N>::BT>, k_cheb_sym<T, TB, N, 16>, SymCfg<T, N>::BT);           \
    break;
  switch (Np) {
    SIPG_SYM_CASE(3)
    SIPG_SYM_CASE(4)
    SIPG_SYM_CASE(6)
    SIPG_SYM_CASE(10)
    SIPG_SYM_CASE(15)
    SIPG_SYM_CASE(20)
    SIPG_SYM_CASE(35)
    default: return;  // not reached: the solver checks block_sym_supported
  }
#undef SIPG_SYM_CASE
  note_launch();
}
template void cheb_step_sym<float, __nv_bfloat16>(float*, float*, const float*, const __nv_bfloat16*, float, float, int,
                                                  int, cudaStream_t, bool);
template void cheb_step_sym<double, double>(double*, double*, const double*, const double*, double, double, int, int,
                                            cudaStream_t, bool);
template <typename TB>
size_t block_sym_values(int nb, int Np) {
  constexpr int CH = Chunk<TB>::CH;
  return (size_t)nb * ((Np * (Np + 1) / 2 + CH - 1) / CH) * CH;
}
template size_t block_sym_values<__nv_bfloat16>(int, int);
template size_t block_sym_values<double>(int, int);
template <typename TB>
void block_pack_sym(TB* P, const double* B, int nb, int Np, cudaStream_t s) {
  pdl_launch(k_block_pack_sym<TB>, dim3(grid_for(block_sym_values<TB>(nb, Np))), dim3(256), 0, s, P, B, nb, Np);
  note_launch();
}
template void block_pack_sym<__nv_bfloat16>(__nv_bfloat16*, const double*, int, int, cudaStream_t);
template void block_pack_sym<double>(double*, const double*, int, int, cudaStream_t);
template <typename T>
void jacobi(T* z, const T* r, const T* dinv, size_t n, cudaStream_t s) {
  pdl_launch(k_jacobi<T>, dim3(grid_for(n)), dim3(256), 0, s, z, r, dinv, n);
  note_launch();
}
template <typename T>
void cheb_step(T* d, T* z, const T* res, const T* dinv, T c1, T c2, size_t n, cudaStream_t s, bool first) {
  pdl_launch(k_cheb<T>, dim3(grid_for(n)), dim3(256), 0, s, d, z, res, dinv, c1, c2, n, (int)first);
  note_launch();
}
template <typename T>
void block_matvec(T* y, const T* B, const T* x, int nb, int Np, cudaStream_t s) {
  pdl_launch(k_block_matvec<T>, dim3(grid_for((size_t)nb * Np)), dim3(256), 0, s, y, B, x, nb, Np);
  note_launch();
}
template <typename T>
void inv_mass(T* y, const T* x, const T* Minv, const T* geof, int ngeof, int jidx, int K, int Np,
              int ncomp, T scale, cudaStream_t s) {
  const int nrows = ncomp * K;
  const dim3 g((unsigned)std::max(1, std::min((nrows + 127) / 128, 148 * 8))), b(128);
  switch (Np) {  // 3D orders 2..4 and 2D orders 3..4: element rows staged in shared memory
    case 10: pdl_launch(k_inv_mass_n<T, 10>, g, b, 0, s, y, x, Minv, geof, ngeof, jidx, K, nrows, scale); break;
    case 15: pdl_launch(k_inv_mass_n<T, 15>, g, b, 0, s, y, x, Minv, geof, ngeof, jidx, K, nrows, scale); break;
    case 20: pdl_launch(k_inv_mass_n<T, 20>, g, b, 0, s, y, x, Minv, geof, ngeof, jidx, K, nrows, scale); break;
    case 35: pdl_launch(k_inv_mass_n<T, 35>, g, b, 0, s, y, x, Minv, geof, ngeof, jidx, K, nrows, scale); break;
    default:
      pdl_launch(k_inv_mass<T>, dim3(grid_for((size_t)ncomp * K * Np)), dim3(256), 0, s, y, x, Minv, geof, ngeof, jidx,
                 K, Np, ncomp, scale);
  }
  note_launch();
}
template <typename T>
void restrict_elem(T* rc, const T* r, const T* P, int K, int Npf, int Npc, int ncomp, cudaStream_t s) {
  const size_t total = (size_t)ncomp * K * Npc;
  const dim3 g(grid_for(total)), b(256);
  if (Npf == 20 && Npc == 10) pdl_launch(k_restrict_n<T, 20, 10>, g, b, 0, s, rc, r, P, total);
  else if (Npf == 10 && Npc == 4) pdl_launch(k_restrict_n<T, 10, 4>, g, b, 0, s, rc, r, P, total);
  else if (Npf == 20 && Npc == 4) pdl_launch(k_restrict_n<T, 20, 4>, g, b, 0, s, rc, r, P, total);
  else if (Npf == 10 && Npc == 6) pdl_launch(k_restrict_n<T, 10, 6>, g, b, 0, s, rc, r, P, total);
  else if (Npf == 6 && Npc == 3) pdl_launch(k_restrict_n<T, 6, 3>, g, b, 0, s, rc, r, P, total);
  else pdl_launch(k_restrict<T>, g, b, 0, s, rc, r, P, K, Npf, Npc, ncomp);
  note_launch();
}
template <typename T>
void prolong_add(T* z, const T* zc, const T* P, int K, int Npf, int Npc, int ncomp, cudaStream_t s) {
  const size_t total = (size_t)ncomp * K * Npf;
  const dim3 g(grid_for(total)), b(256);
  if (Npf == 20 && Npc == 10) pdl_launch(k_prolong_add_n<T, 20, 10>, g, b, 0, s, z, zc, P, total);
  else if (Npf == 10 && Npc == 4) pdl_launch(k_prolong_add_n<T, 10, 4>, g, b, 0, s, z, zc, P, total);
  else if (Npf == 20 && Npc == 4) pdl_launch(k_prolong_add_n<T, 20, 4>, g, b, 0, s, z, zc, P, total);
  else if (Npf == 10 && Npc == 6) pdl_launch(k_prolong_add_n<T, 10, 6>, g, b, 0, s, z, zc, P, total);
  else if (Npf == 6 && Npc == 3) pdl_launch(k_prolong_add_n<T, 6, 3>, g, b, 0, s, z, zc, P, total);
  else pdl_launch(k_prolong_add<T>, g, b, 0, s, z, zc, P, K, Npf, Npc, ncomp);
  note_launch();
}
template <typename T>
void coarse_update(T* z, T* r, T* sv, const T* p, const T* Ap, const T* dinv, size_t n, double* scal,
                   const RedWork& w, cudaStream_t s) {
  pdl_launch(k_coarse_update<T>, dim3(red_grid(n)), dim3(kRedThreads), 0, s, z, r, sv, p, Ap, dinv, n, scal, w.partial, w.counter);
  note_launch();
}
template <typename T>
void coarse_update_p(T* p, const T* sv, size_t n, double* scal, cudaStream_t s) {
  pdl_launch(k_coarse_update_p<T>, dim3(grid_for(n)), dim3(256), 0, s, p, sv, n, scal);
  note_launch();
  pdl_launch(k_shift_scalar, dim3(1), dim3(1), 0, s, scal, S_C_RZN, S_C_RZ);
  note_launch();
}

template <typename T>
void csr_spmv(int rows, const int* ptr, const int* idx, const T* val, const T* x, T* y, T alpha, T beta,
              cudaStream_t s, const T* c) {
  const int blocks = std::max(1, std::min((rows + 31) / 32, 148 * 16));
  pdl_launch(k_csr_spmv<T>, dim3(blocks), dim3(256), 0, s, rows, ptr, idx, val, x, y, alpha, beta, c ? c : y);
  note_launch();
}
template <typename T>
void csr_cheb(int rows, const int* ptr, const int* idx, const T* val, const T* d, const T* r, const T* dinv, T* dn,
              T* rn, T* z, T c1, T c2, bool first, cudaStream_t s) {
  const int blocks = std::max(1, std::min((rows + 31) / 32, 148 * 16));
  pdl_launch(k_csr_cheb<T>, dim3(blocks), dim3(256), 0, s, rows, ptr, idx, val, d, r, dinv, dn, rn, z, c1, c2,
             (int)first);
  note_launch();
}
void dense_inverse_device(double* a, int n, bool project_constants, double* work, cudaStream_t s) {
  const size_t nn = (size_t)n * n;
  const int g2 = (int)std::min<size_t>((nn + 255) / 256, 148 * 8);
  double* P = work + 2 * (size_t)n;  // GJB x GJB pivot-block inverse
  const int tiles = (n + 63) / 64;
  for (int k0 = 0; k0 < n; k0 += GJB) {
    const int bs = std::min(GJB, n - k0);
    k_gjb_pivot<<<1, 32, 0, s>>>(a, n, k0, bs, P);
    k_gjb_row<<<(n + 255) / 256, 256, 0, s>>>(a, n, k0, bs, P);
    k_gjb_update<<<dim3(tiles, tiles), 256, 0, s>>>(a, n, k0, bs);
    k_gjb_col<<<(n + 127) / 128, 128, 0, s>>>(a, n, k0, bs, P);
    note_launch(4);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("dense inverse: ") + cudaGetErrorString(e));
  if (project_constants) {
    k_dense_sums<<<(2 * n + 255) / 256, 256, 0, s>>>(a, n, work, work + n);
    k_dense_project<<<g2, 256, 0, s>>>(a, n, work, work + n);
    note_launch(2);
  }
}

// v_i = 2 U_i - 1 with U_i the i-th splitmix64 draw of `seed` (top 53 bits), as
// the host generator SplitMix64 gives them one after the other.
__global__ void k_splitmix_uniform(double* v, size_t n, unsigned long long seed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long z = seed + (unsigned long long)(i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    v[i] = 2.0 * ((double)(z >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
  }
}
void splitmix_uniform_device(double* v, size_t n, unsigned long long seed, cudaStream_t s) {
  k_splitmix_uniform<<<grid_for(n), 256, 0, s>>>(v, n, seed);
  note_launch();
}

template <typename T>
void dense_mv(int n, const T* M, const T* x, T* y, cudaStream_t s) {
  int blocks = std::max(1, std::min((n * 32 + 255) / 256, 148 * 8));
  pdl_launch(k_dense_mv<T>, dim3(blocks), dim3(256), 0, s, n, M, x, y);
  note_launch();
}
template <typename T>
void vadd(T* y, const T* x, size_t n, cudaStream_t s) {
  pdl_launch(k_vadd<T>, dim3(grid_for(n)), dim3(256), 0, s, y, x, n);
  note_launch();
}

#define SIPG_INST(T)                                                                              \
  template void multi_dot<T>(const T* const*, const T* const*, int, size_t, double*, int,         \
                             const RedWork&, cudaStream_t);                                      \
  template void vsum<T>(const T*, size_t, double*, const RedWork&, cudaStream_t);                \
  template void update_p<T>(T*, const T*, size_t, const double*, int, int, cudaStream_t);        \
  template void sub_mean<T>(T*, size_t, const double*, int, cudaStream_t);                       \
  template void vcopy<T>(T*, const T*, size_t, cudaStream_t);                                    \
  template void vzero<T>(T*, size_t, cudaStream_t);                                              \
  template void jacobi<T>(T*, const T*, const T*, size_t, cudaStream_t);                         \
  template void cheb_step<T>(T*, T*, const T*, const T*, T, T, size_t, cudaStream_t, bool);      \
  template void block_matvec<T>(T*, const T*, const T*, int, int, cudaStream_t);                 \
  template void inv_mass<T>(T*, const T*, const T*, const T*, int, int, int, int, int, T,        \
                            cudaStream_t);                                                       \
  template void restrict_elem<T>(T*, const T*, const T*, int, int, int, int, cudaStream_t);      \
  template void prolong_add<T>(T*, const T*, const T*, int, int, int, int, cudaStream_t);        \
  template void coarse_update<T>(T*, T*, T*, const T*, const T*, const T*, size_t, double*,      \
                                 const RedWork&, cudaStream_t);                                  \
  template void coarse_update_p<T>(T*, const T*, size_t, double*, cudaStream_t);                 \
  template void cheb_step_block<T, T>(T*, T*, const T*, const T*, T, T, int, int, cudaStream_t, bool); \
  template void block_transpose<T>(T*, const double*, int, int, cudaStream_t);                     \
  template void csr_spmv<T>(int, const int*, const int*, const T*, const T*, T*, T, T, cudaStream_t, const T*); \
  template void csr_cheb<T>(int, const int*, const int*, const T*, const T*, const T*, const T*, T*, T*, T*, T, T, \
                            bool, cudaStream_t);                                                   \
  template void dense_mv<T>(int, const T*, const T*, T*, cudaStream_t);                          \
  template void vadd<T>(T*, const T*, size_t, cudaStream_t);

SIPG_INST(double)
SIPG_INST(float)

}  // namespace sipg
