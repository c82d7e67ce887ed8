// Device set-up of the algebraic coarse levels. See amg_setup.cuh.
#include "amg_setup.cuh"

#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "refelem.hpp"
#include "sipg_apply.cuh"
#include "vecops.cuh"

namespace sipg {

P1Tables p1_tables(const RefElement& r) {
  if (r.Np != r.dim + 1 || r.Np > 4) throw std::runtime_error("p1_tables needs the order-1 element");
  P1Tables t{};
  t.dim = r.dim;
  const int npp = r.Np * r.Np;
  const std::vector<double>* D[3] = {&r.Dr, &r.Ds, &r.Dt};
  for (int d = 0; d < r.dim; ++d)
    for (int q = 0; q < npp; ++q) t.D[d][q] = (*D[d])[q];
  for (int q = 0; q < npp; ++q) t.M[q] = r.M[q];
  for (int f = 0; f < r.Nfaces; ++f)
    for (int q = 0; q < npp; ++q) t.MF[f][q] = r.MMF[(size_t)f * npp + q];
  return t;
}

namespace {

// One thread per element; the block stays in registers (Np <= 4).
template <int DIM>
__global__ void k_p1c_blocks(P1Tables t, int K, const double* __restrict__ geof, const double* __restrict__ factor1,
                             const double* __restrict__ tau1, const int* __restrict__ nbr,
                             const unsigned char* __restrict__ bct, int mm_mode, double mm_scalar,
                             const double* __restrict__ mm1, double* __restrict__ blk) {
  constexpr int NP = DIM + 1, NF = DIM + 1, NG = DIM == 3 ? 10 : 5;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= K) return;
  double g[NG], fac[NP], B[NP][NP], Dx[NP][NP], T[NP][NP];
  for (int i = 0; i < NG; ++i) g[i] = geof[(size_t)e * NG + i];
  for (int i = 0; i < NP; ++i) fac[i] = factor1 ? factor1[(size_t)e * NP + i] : 1.0;
  const double J = g[DIM == 3 ? 9 : 4];
#pragma unroll
  for (int i = 0; i < NP; ++i)
#pragma unroll
    for (int j = 0; j < NP; ++j) B[i][j] = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double s = 0.0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) s += g[r * DIM + d] * t.D[r][i * NP + j];
        Dx[i][j] = s;
      }
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) s += t.M[i * NP + k] * fac[k] * Dx[k][j];
        T[i][j] = J * s;
      }
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) s += Dx[k][i] * T[k][j];
        B[i][j] += s;
      }
  }
  for (int f = 0; f < NF; ++f) {
    const int nb = nbr[(size_t)e * NF + f];
    if (nb >= 0 || bct[-nb - 1] != 0) continue;  // interior jumps vanish; Neumann and slip add nothing
    double n[3], sJ;
    simplex_face_normal<DIM>(g, f, n, &sJ);
    double rf[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < DIM; ++r)
#pragma unroll
      for (int d = 0; d < DIM; ++d) rf[r] += n[d] * g[r * DIM + d];
    double Dn[NP][NP];
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double s = 0.0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) s += rf[r] * t.D[r][i * NP + j];
        Dn[i][j] = s;
      }
    const double* mf = t.MF[f];
    const double gtau = tau1[(size_t)e * NF + f];
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NP; ++k) s += mf[i * NP + k] * fac[k] * Dn[k][j] + Dn[k][i] * mf[k * NP + j] * fac[j];
        B[i][j] += sJ * (gtau * mf[i * NP + j] - s);
      }
  }
  if (mm_mode != 0)
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int j = 0; j < NP; ++j) B[i][j] += J * t.M[i * NP + j] * (mm_mode == 1 ? mm_scalar : mm1[(size_t)e * NP + j]);
#pragma unroll
  for (int i = 0; i < NP; ++i)
#pragma unroll
    for (int j = 0; j < NP; ++j) blk[(size_t)e * NP * NP + i * NP + j] = B[i][j];
}

__global__ void k_term_sum(int n, const int* __restrict__ ptr, const int* __restrict__ idx,
                           const double* __restrict__ coef, const double* __restrict__ in, double* __restrict__ out,
                           float* __restrict__ out32) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    const int b = ptr[i], e = ptr[i + 1];
    if (coef)
      for (int t = b; t < e; ++t) s += in[idx[t]] * coef[t];
    else
      for (int t = b; t < e; ++t) s += in[idx[t]];
    out[i] = s;
    if (out32) out32[i] = (float)s;
  }
}

__global__ void k_csr_dinv(int n, const int* __restrict__ ptr, const int* __restrict__ idx,
                           const double* __restrict__ v, double* __restrict__ d64, float* __restrict__ d32) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k)
      if (idx[k] == i) d = 1.0 / v[k];
    d64[i] = d;
    if (d32) d32[i] = (float)d;
  }
}

__global__ void k_csr_scatter(int n, const int* __restrict__ ptr, const int* __restrict__ idx,
                              const double* __restrict__ v, double* __restrict__ dense) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) dense[(size_t)i * n + idx[k]] = v[k];
}

// One block: dmax = max_i |a_ii|, then a_ii += 1e-8 dmax.
__global__ void k_dense_shift(int n, double* dense) {
  __shared__ double red[32];
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(dense[(size_t)i * n + i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  const double sh = 1e-8 * red[0];
  for (int i = threadIdx.x; i < n; i += blockDim.x) dense[(size_t)i * n + i] += sh;
}

int blocks_for(size_t n, int threads) {
  return (int)std::max<size_t>(1, std::min<size_t>((n + threads - 1) / threads, 148 * 16));
}

}  // namespace

void p1c_blocks_device(const P1Tables& t, int K, const double* geof, const double* factor1, const double* tau1,
                       const int* nbr, const unsigned char* bct, int mm_mode, double mm_scalar, const double* mm1,
                       double* blk, cudaStream_t s) {
  const int th = 128, grid = (K + th - 1) / th;
  if (K <= 0) return;
  if (t.dim == 3)
    k_p1c_blocks<3><<<grid, th, 0, s>>>(t, K, geof, factor1, tau1, nbr, bct, mm_mode, mm_scalar, mm1, blk);
  else
    k_p1c_blocks<2><<<grid, th, 0, s>>>(t, K, geof, factor1, tau1, nbr, bct, mm_mode, mm_scalar, mm1, blk);
  note_launch();
}

void term_sum_device(int n, const int* ptr, const int* idx, const double* coef, const double* in, double* out,
                     float* out32, cudaStream_t s) {
  if (n <= 0) return;
  k_term_sum<<<blocks_for(n, 256), 256, 0, s>>>(n, ptr, idx, coef, in, out, out32);
  note_launch();
}

void csr_dinv_device(int n, const int* ptr, const int* idx, const double* v, double* d64, float* d32,
                     cudaStream_t s) {
  if (n <= 0) return;
  k_csr_dinv<<<blocks_for(n, 256), 256, 0, s>>>(n, ptr, idx, v, d64, d32);
  note_launch();
}

void csr_to_dense_device(int n, const int* ptr, const int* idx, const double* v, double* dense, bool shift,
                         cudaStream_t s) {
  if (n <= 0) return;
  cudaMemsetAsync(dense, 0, (size_t)n * n * sizeof(double), s);
  k_csr_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, ptr, idx, v, dense);
  note_launch();
  if (shift) {
    k_dense_shift<<<1, 1024, 0, s>>>(n, dense);
    note_launch();
  }
}

TermPlan spgemm_plan(const Csr& A, const Csr& B, bool a_varies, Csr* Cs) {
  if (A.cols != B.rows) throw std::runtime_error("spgemm_plan shape mismatch");
  Csr& C = *Cs;
  C.rows = A.rows;
  C.cols = B.cols;
  C.ptr.assign(C.rows + 1, 0);
  C.idx.clear();
  TermPlan tp;
  tp.ptr.assign(1, 0);
  std::vector<int> mark(B.cols, -1), pos(B.cols, 0), cols, cnt;
  struct Term { int out, idx; double coef; };
  std::vector<Term> terms;
  for (int i = 0; i < A.rows; ++i) {
    cols.clear();
    terms.clear();
    for (int ka = A.ptr[i]; ka < A.ptr[i + 1]; ++ka) {
      const int k = A.idx[ka];
      for (int kb = B.ptr[k]; kb < B.ptr[k + 1]; ++kb) {
        const int j = B.idx[kb];
        if (mark[j] != i) { mark[j] = i; cols.push_back(j); }
        terms.push_back({j, a_varies ? ka : kb, a_varies ? B.val[kb] : A.val[ka]});
      }
    }
    std::sort(cols.begin(), cols.end());
    const int base = (int)C.idx.size();
    for (size_t c = 0; c < cols.size(); ++c) pos[cols[c]] = base + (int)c;
    cnt.assign(cols.size(), 0);
    for (const Term& t : terms) cnt[pos[t.out] - base]++;
    const int t0 = tp.ptr.back();
    for (size_t c = 0; c < cols.size(); ++c) {
      C.idx.push_back(cols[c]);
      tp.ptr.push_back(tp.ptr.back() + cnt[c]);
    }
    tp.idx.resize(tp.ptr.back());
    tp.coef.resize(tp.ptr.back());
    // fill in visiting order: per output the terms keep the order of the product's accumulation
    std::vector<int> fill(cols.size(), 0);
    for (const Term& t : terms) {
      const int c = pos[t.out] - base;
      const int at = tp.ptr[base + c] + fill[c]++;
      tp.idx[at] = t.idx;
      tp.coef[at] = t.coef;
    }
    (void)t0;
    C.ptr[i + 1] = (int)C.idx.size();
  }
  C.val.assign(C.idx.size(), 0.0);
  return tp;
}

TermPlan p1c_gather_plan(const P1Plan& plan, int K, int Np) {
  const size_t nnz = plan.idx.size(), ne = (size_t)K * Np * Np;
  TermPlan tp;
  tp.ptr.assign(nnz + 1, 0);
  for (size_t q = 0; q < ne; ++q) tp.ptr[plan.slot[q] + 1]++;
  for (size_t k = 0; k < nnz; ++k) tp.ptr[k + 1] += tp.ptr[k];
  tp.idx.resize(ne);
  std::vector<int> fill(tp.ptr.begin(), tp.ptr.end() - 1);
  for (size_t q = 0; q < ne; ++q) tp.idx[fill[plan.slot[q]]++] = (int)q;  // element order within each entry
  return tp;
}

}  // namespace sipg
