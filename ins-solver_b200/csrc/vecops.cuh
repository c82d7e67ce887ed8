// Vector kernels of the Krylov and multigrid loops (cg3_*.h / cg_*.h kernels of
// the reference, src/kernels/cg3_alpha_pre.h ... cg3_update_p.h), fused so that
// each CG step reads every vector once. Reductions are FP64 warp-shuffle sums
// with a fixed two-stage order (block partials, then the last block reduces the
// partials in index order), so results are bitwise reproducible run to run and
// the scalars never leave the device.
#pragma once
#include <cstddef>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace sipg {

// Count of kernel launches issued by this library (diagnostics).
void note_launch(unsigned n = 1);
// While counter is set, this thread's note_launch calls add to it instead (kernels
// recorded into a graph during a capture, not launched); null restores counting.
void record_launches(unsigned long long* counter);
unsigned long long launch_count();

// Device scalar slots used by the solvers.
enum Scal : int {
  S_RZ = 0,    // r . z           (alpha numerator, beta denominator)
  S_PAP = 1,   // p . A p
  S_RR = 2,    // r . r
  S_BETA = 3,  // r . (z - z_old)
  S_BB = 4,    // b . b
  S_SUM = 5,   // sum (nullspace projection)
  S_C_RZ = 6,  // coarse CG: r . s
  S_C_PAP = 7, // coarse CG: p . Ap
  S_C_RZN = 8, // coarse CG: new r . s
  S_C_FLAG = 9,
  S_TMP = 10,
  S_RZO = 11,    // r_(k+1) . z_k   (device-resident loop: beta without swapping z buffers)
  S_RZN = 12,    // r_(k+1) . z_(k+1)
  S_ITER = 13,   // iterations done
  S_STATUS = 14, // 0 running, 1 converged, 2 breakdown, 3 iteration limit, 4 chunk done
  S_TOL = 15,    // absolute tolerance on ||r||
  S_CHUNK = 16,  // iterations left in this launch
  S_RZP = 17,    // r_k . z_k of the previous iteration (beta denominator)
  S_COUNT = 24
};

struct RedWork {
  double* partial = nullptr;   // kRedBlocks x 4
  unsigned* counter = nullptr; // 1
};
constexpr int kRedBlocks = 148 * 8;
constexpr int kRedThreads = 256;

// out[k] = sum_i a_k[i] * b_k[i] for k < nk (nk <= 3); b_k may alias a_k.
template <typename T>
void multi_dot(const T* const* a, const T* const* b, int nk, size_t n, double* out, int out_stride,
               const RedWork& w, cudaStream_t s);

// out = sum_i r[i] * (z[i] - zo[i])   (cg3_compute_beta_pre_flex.h)
void dot_diff(const double* r, const double* z, const double* zo, size_t n, double* out,
              const RedWork& w, cudaStream_t s);

// Sum of entries (nullspace projection).
template <typename T>
void vsum(const T* a, size_t n, double* out, const RedWork& w, cudaStream_t s);

// x += alpha p ; r -= alpha Ap ; rr = r.r   with alpha = scal[num] / scal[den]
void cg_update_xr(double* x, double* r, const double* p, const double* Ap, size_t n,
                  const double* scal, int num, int den, double* rr_out, const RedWork& w,
                  cudaStream_t s);
// Fused steps of the mixed-precision outer iteration (two-output reductions write
// out[0] and out[stride]):
//   x += alpha p ; r -= alpha Ap ; out = (sum r, r . r)
void cg_update_xr_sum(double* x, double* r, const double* p, const double* Ap, size_t n, const double* scal, int num,
                      int den, double* out, int stride, const RedWork& w, cudaStream_t s);
//   r -= mean (scal[mean_slot] / n, none when mean_slot < 0) ; r32 = r ; out = (r . r, r . zo)
void resid_prep(double* r, float* r32, const double* zo, size_t n, const double* scal, int mean_slot, double* out,
                int stride, const RedWork& w, cudaStream_t s);
//   x += alpha p ; r -= alpha Ap ; out = (r . r, r . zo)
void cg_update_xr_rzo(double* x, double* r, const double* p, const double* Ap, const double* zo, size_t n,
                      const double* scal, int num, int den, double* out, int stride, const RedWork& w,
                      cudaStream_t s);
//   z = B r (row-major Np x Np blocks; Np == 0: z = B r elementwise, point Jacobi) ; out = r . z
void precond_dot(double* z, const double* r, const double* B, int Np, size_t n, double* out, const RedWork& w,
                 cudaStream_t s);
//   z = z32 ; out = sum z
void to_f64_sum(double* z, const float* z32, size_t n, double* out, const RedWork& w, cudaStream_t s);
//   z = (z32 ? z32 : z) - mean (as above) ; out = r . z
void finish_z_dot(double* z, const float* z32, const double* r, size_t n, const double* scal, int mean_slot,
                  double* out, const RedWork& w, cudaStream_t s);
// p = z + beta p   with beta = scal[num] / scal[den]
template <typename T>
void update_p(T* p, const T* z, size_t n, const double* scal, int num, int den, cudaStream_t s);
// y = a (constant copy), y -= mean (scal[S_SUM] / n)
template <typename T>
void sub_mean(T* v, size_t n, const double* scal, int slot, cudaStream_t s);

template <typename T>
void vcopy(T* dst, const T* src, size_t n, cudaStream_t s);
template <typename T>
void vzero(T* dst, size_t n, cudaStream_t s);
void to_f32(float* dst, const double* src, size_t n, cudaStream_t s);
void to_f64(double* dst, const float* src, size_t n, cudaStream_t s);

// z = dinv * r
template <typename T>
void jacobi(T* z, const T* r, const T* dinv, size_t n, cudaStream_t s);

// Chebyshev step: d = c1 * d + c2 * dinv * res ; z += d  (first: z = d; c1 == 0 reads no d)
template <typename T>
void cheb_step(T* d, T* z, const T* res, const T* dinv, T c1, T c2, size_t n, cudaStream_t s, bool first = false);
// Same step with full column-major blocks Bc (nb blocks of Np x Np): ten threads per
// block at p = 3, for meshes too small to fill the GPU with one thread per block.
template <typename T, typename TB>
void cheb_step_block(T* d, T* z, const T* res, const TB* Bc, T c1, T c2, int nb, int Np, cudaStream_t s,
                     bool first = false);
template <typename T>
void block_transpose(T* dst, const double* src, int nb, int Np, cudaStream_t s);
// Element-block Jacobi Chebyshev step: d <- c1 d + c2 B res, z += d (first: z = d;
// c1 == 0 reads no d), with the inverse diagonal blocks B stored as packed symmetric
// triangles (block_pack_sym) for Np in {3, 4, 6, 10, 15, 20, 35}.
bool block_sym_supported(int Np);
template <typename T, typename TB>
void cheb_step_sym(T* d, T* z, const T* res, const TB* P, T c1, T c2, int nb, int Np, cudaStream_t s,
                   bool first = false);
// Row-major FP64 blocks (nb x Np x Np) -> packed symmetric triangles (mean of the two),
// in 16-byte chunks of 16 / sizeof(TB) values: chunk k of block b at P[(k * nb + b) * CH].
template <typename TB>
void block_pack_sym(TB* P, const double* B, int nb, int Np, cudaStream_t s);
// Values (padding included) that block_pack_sym writes.
template <typename TB>
size_t block_sym_values(int nb, int Np);

// Element-block matvec: y_e = B_e x_e (B: nb x Np x Np row-major, nb blocks)
template <typename T>
void block_matvec(T* y, const T* B, const T* x, int nb, int Np, cudaStream_t s);

// Inverse mass: y_e = scale * Minv x_e / J_e (pre_inv_mass / pre_factor_inv_mass)
template <typename T>
void inv_mass(T* y, const T* x, const T* Minv, const T* geof, int ngeof, int jidx, int K, int Np,
              int ncomp, T scale, cudaStream_t s);

// Order transfer per element: restrict  rc_e = P^T r_e  (P: Npf x Npc row-major)
//                             prolong   z_e += P zc_e
template <typename T>
void restrict_elem(T* rc, const T* r, const T* P, int K, int Npf, int Npc, int ncomp, cudaStream_t s);
template <typename T>
void prolong_add(T* z, const T* zc, const T* P, int K, int Npf, int Npc, int ncomp, cudaStream_t s);

// Fixed-count coarse CG helpers (device scalars):
//   alpha = scal[S_C_RZ] / scal[S_C_PAP]; z += alpha p; r -= alpha Ap; s = dinv r; scal[S_C_RZN] = r.s
template <typename T>
void coarse_update(T* z, T* r, T* sv, const T* p, const T* Ap, const T* dinv, size_t n, double* scal,
                   const RedWork& w, cudaStream_t s);
// p = s + (scal[S_C_RZN]/scal[S_C_RZ]) p ; scal[S_C_RZ] = scal[S_C_RZN]
template <typename T>
void coarse_update_p(T* p, const T* sv, size_t n, double* scal, cudaStream_t s);

// y = alpha * A x + beta * c for a CSR matrix (c = y when null; beta == 0: c is not read)
template <typename T>
void csr_spmv(int rows, const int* ptr, const int* idx, const T* val, const T* x, T* y, T alpha, T beta,
              cudaStream_t s, const T* c = nullptr);
// Chebyshev step fused with the residual update on a CSR level:
//   dn = c1 d + c2 dinv r ; z = (first ? 0 : z) + dn ; rn = r - A dn (rn may be null)
// dn, rn must not alias d, r; c1 == 0 reads no d.
template <typename T>
void csr_cheb(int rows, const int* ptr, const int* idx, const T* val, const T* d, const T* r, const T* dinv, T* dn,
              T* rn, T* z, T c1, T c2, bool first, cudaStream_t s);
// y = M x for a dense row-major n x n matrix
template <typename T>
void dense_mv(int n, const T* M, const T* x, T* y, cudaStream_t s);
// In-place inverse of the dense SPD matrix a (n x n, FP64) by blocked Gauss-Jordan
// elimination (32 pivots per step, the trailing update as 64 x 64 tiles);
// project_constants applies Q a Q, Q = I - 11^T/n, after it. work: 2n + 1024 doubles.
void dense_inverse_device(double* a, int n, bool project_constants, double* work, cudaStream_t s);
// v_i = 2 U_i - 1, U_i the i-th splitmix64 draw from `seed` (the host SplitMix64 sequence).
void splitmix_uniform_device(double* v, size_t n, unsigned long long seed, cudaStream_t s);
// y += x
template <typename T>
void vadd(T* y, const T* x, size_t n, cudaStream_t s);

}  // namespace sipg
