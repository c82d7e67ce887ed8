// Krylov solvers and the p-multigrid preconditioner, all on the device.
//
// Replaces ViscousSolver3D::conjugate_gradient / preconditioned_conjugate_gradient
// (src/solvers/3d/slip_matrix/viscous_solver.cpp:89-301) with its preconditioners
// (:357-453), and the LinearSolver family created at
// src/solvers/3d/ins_solver_base.cpp:1522-1536 (PETScJacobiSolver,
// PETScBlockJacobiSolver, PETScInvMassSolver, PETScPMultigrid; unvendored, so the
// p-multigrid follows its configuration keys [p-multigrid] orders / cheb_orders /
// eigen_val_saftey_factor, examples/3d/oscillating_droplet/config.ini:24-31).
//
// Every scalar of the iteration (alpha, beta, norms) stays on the device; the
// host reads one FP64 residual norm per iteration to decide termination.
// Mixed precision: the V-cycle (smoother applies, transfers, coarse CG) runs in
// FP32 while the outer flexible CG, its residual update, inner products and step
// lengths, and the final defect r = b - A x stay FP64.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <type_traits>
#include <vector>

#include "../../include/sipg_b200.h"
#include "amg.hpp"
#include "amg_setup.cuh"
#include "capi_util.hpp"
#include "bsr.cuh"
#include "runtime.hpp"
#include "sipg_blocks.cuh"
#include "vecops.cuh"

using namespace sipg;

namespace {

struct PinnedScalars {
  double* h = nullptr;
  PinnedScalars() { SIPG_CUDA(cudaMallocHost(&h, S_COUNT * sizeof(double))); }
  ~PinnedScalars() { if (h) cudaFreeHost(h); }
};

struct Level {
  std::unique_ptr<sipg_op> own;  // levels > 0 own their operator
  sipg_op* op = nullptr;
  int order = 0, Np = 0;
  size_t n = 0;
  DevBuf dinv64, dinv32, factor64, mm64;
  double lmax = 0.0;
  DevBuf P64, P32;               // prolongation from the next level: Np x Np_next
  // work vectors in the V-cycle precision
  DevBuf rhs, z, res, d;
  DevBuf d2, sres;               // fused Chebyshev steps (bsr->c16): second d buffer, Bd^-1 r
  DevBuf cp, cs, cAp;            // coarse CG
  DevBuf bc64, bc32;             // inverse diagonal blocks (block-Jacobi smoothing; bc32 in bf16)
  bool bsym = false;             // bc* packed symmetric (large meshes) or full column-major blocks
  std::unique_ptr<BsrOp> bsr;    // assembled element blocks (low orders), else matrix-free
  int cheb = 4, pre = 1, post = 1;  // Chebyshev degree, smoothing sweeps before / after the coarse correction
  // y = alpha A x + beta c (c = y when null)
  template <typename T>
  void apply(const T* x, T* y, cudaStream_t s, T alpha = T(1), T beta = T(0), const T* c = nullptr) const {
    if (bsr) bsr_apply<T>(*bsr, x, y, alpha, beta, s, c);
    else op->apply<T>(x, y, s, alpha, beta, c);
  }
};

// Per-element interpolation kernel: out_e = I in_e (I: Npo x Npi row-major)
__global__ void k_interp(double* out, const double* in, const double* I, int K, int Npo, int Npi) {
  const size_t total = (size_t)K * Npo;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t e = i / Npo;
    const int r = (int)(i % Npo);
    double s = 0.0;
    for (int j = 0; j < Npi; ++j) s += I[r * Npi + j] * in[e * Npi + j];
    out[i] = s;
  }
}

__global__ void k_recip(double* d, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    d[i] = 1.0 / d[i];
}

template <typename T>
__global__ void k_scale(T* v, size_t n, const double* scal, int slot) {
  const T inv = (T)(1.0 / sqrt(scal[slot]));
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    v[i] *= inv;
}

__global__ void k_mul(double* v, const double* w, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    v[i] *= w[i];
}

struct DevCsr {
  int rows = 0, cols = 0;
  DevBuf ptr, idx, v64, v32;
  void upload(const Csr& c) {
    rows = c.rows;
    cols = c.cols;
    ptr = DevBuf((c.ptr.size()) * sizeof(int));
    ptr.upload(c.ptr.data(), c.ptr.size() * sizeof(int));
    size_t nz = std::max<size_t>(1, c.nnz());
    idx = DevBuf(nz * sizeof(int));
    v64 = DevBuf(nz * sizeof(double));
    v32 = DevBuf(nz * sizeof(float));
    if (c.nnz()) {
      idx.upload(c.idx.data(), c.nnz() * sizeof(int));
      v64.upload(c.val.data(), c.nnz() * sizeof(double));
      std::vector<float> f(c.val.begin(), c.val.end());
      v32.upload(f.data(), f.size() * sizeof(float));
    }
  }
  template <typename T>
  const T* vals() const {
    return std::is_same<T, float>::value ? (const T*)v32.p : (const T*)v64.p;
  }
  // y = alpha A x + beta c (c = y when null)
  template <typename T>
  void mv(const T* x, T* y, T alpha, T beta, cudaStream_t s, const T* c = nullptr) const {
    csr_spmv<T>(rows, ptr.as<int>(), idx.as<int>(), vals<T>(), x, y, alpha, beta, s, c);
  }
};

// Fixed term lists on the device (TermPlan): out[i] = sum_t in[idx[t]] * coef[t].
struct DevTerms {
  int n = 0;
  DevBuf ptr, idx, coef;
  void upload(const TermPlan& t) {
    n = (int)t.ptr.size() - 1;
    ptr = DevBuf(t.ptr.size() * sizeof(int));
    ptr.upload(t.ptr.data(), t.ptr.size() * sizeof(int));
    idx = DevBuf(std::max<size_t>(1, t.idx.size()) * sizeof(int));
    if (!t.idx.empty()) idx.upload(t.idx.data(), t.idx.size() * sizeof(int));
    coef = DevBuf();
    if (!t.coef.empty()) {
      coef = DevBuf(t.coef.size() * sizeof(double));
      coef.upload(t.coef.data(), t.coef.size() * sizeof(double));
    }
  }
  void run(const double* in, double* out, float* out32, cudaStream_t s) const {
    term_sum_device(n, ptr.as<int>(), idx.as<int>(), coef.p ? coef.as<double>() : nullptr, in, out, out32, s);
  }
};

struct AmgDevLevel {
  int n = 0;
  DevCsr A, P, R;
  DevTerms ap, rap;  // Galerkin product with the stored P: AP = A P, then R (AP) = the next level's operator
  DevBuf apv;        // values of A P
  DevBuf dinv64, dinv32;
  double lmax = 0.0;
  DevBuf rhs, z, res, d;
  DevBuf res2, d2;  // the fused Chebyshev steps alternate between (d, res) and (d2, res2)
};

int grid_for(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }

}  // namespace

// Set-up phase timer: with SIPG_SETUP_TIMES set in the environment, each phase
// of a solver set-up is synchronised and its wall time printed to stderr.
struct PhaseTimer {
  bool on = std::getenv("SIPG_SETUP_TIMES") != nullptr;
  cudaStream_t s;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  explicit PhaseTimer(cudaStream_t st) : s(st) {}
  void mark(const char* what, int level = -1) {
    if (!on) return;
    cudaStreamSynchronize(s);
    const auto t1 = std::chrono::steady_clock::now();
    std::fprintf(stderr, "setup %-22s level %2d %8.2f ms\n", what, level,
                 std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  }
};

// One capture at a time in the process (solvers of a serving loop capture from
// several threads), and no capture while another thread runs a solver's first
// solve or set-up: those launch kernels for the first time, and loading a kernel
// module while another thread captures a stream can fail or invalidate the capture.
static std::recursive_mutex g_graph_mu;

// Levels with at least this many element blocks store them packed symmetric
// (one thread per block fills the GPU from here on).
constexpr int kSymMinBlocks = 148 * 128;

// Device-resident outer loop: beta numerator of the flexible CG from two dots
// (r.z_new - r.z_old) and the per-iteration stopping test, which ends the
// conditional while-node of the loop graph.
__global__ void k_beta_flex(double* scal) {
  scal[S_BETA] = scal[S_RZN] - scal[S_RZO];
  scal[S_RZP] = scal[S_RZ];
  scal[S_RZ] = scal[S_RZN];
}

__global__ void k_loop_check(double* scal, cudaGraphConditionalHandle h, int max_iter) {
  const double it = scal[S_ITER] + 1.0;
  scal[S_ITER] = it;
  const double pap = scal[S_PAP], rr = scal[S_RR];
  double st = 0.0;
  if (!(pap > 0.0) || !isfinite(rr)) st = 2.0;
  else if (sqrt(rr) <= scal[S_TOL]) st = 1.0;
  else if (it >= (double)max_iter) st = 3.0;
  else if ((scal[S_CHUNK] -= 1.0) <= 0.0) st = 4.0;
  if (st != 0.0) {
    scal[S_STATUS] = st;
    cudaGraphSetConditional(h, 0);
  }
}

struct sipg_solver {
  sipg_op* op = nullptr;
  int kind = 0;
  sipg_solver_opts o{};
  size_t n = 0;
  cudaStream_t stream = nullptr;
  DevBuf r, z, p, Ap, bw, xw, r32, z32;
  DevBuf scal, partial, counter;
  RedWork rw;
  PinnedScalars hs;
  DevBuf dinv, blocks, minv;
  std::vector<Level> lv;
  std::vector<AmgDevLevel> al;
  DevCsr Pdg, Rdg;
  DevBuf cinv64, cinv32, cinv_work;
  int cinv_n = 0;
  DevBuf rows_ws;  // set-up workspace: FP64 inverse diagonal blocks of a level
  DevBuf pl_v, pl_w, pl_t;  // set-up workspace: power iteration
  DevBuf p1_blk, a0_tmp;     // set-up workspace: P1 element blocks, level-0 values before the hierarchy exists
  // the algebraic hierarchy (aggregates and prolongators) is kept across set-ups
  // while these stay the same (amg_reuse_interpolation)
  bool amg_frozen = false;
  std::vector<int> amg_bct;
  bool amg_singular = false;
  bool use_amg = false;
  bool dirty = true;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Graph replay of the outer iteration: one graph per parity of the roles of
  // z and z_old; the solution is iterated in xi so that no caller pointer is baked in.
  DevBuf xi;
  cudaGraphExec_t gx[2] = {nullptr, nullptr};
  unsigned long long gnodes[2] = {0, 0};
  unsigned gver = 0;
  bool graph_broken = false;
  const std::atomic<int>* cancel = nullptr;  // set by a serving loop: non-zero ends the solve
  // device-resident loop (conditional while-node around one iteration on fixed buffers)
  cudaGraphExec_t gloop = nullptr;
  unsigned long long gloop_nodes = 0;
  bool gloop_broken = false;
  bool warm = false;  // a solve has run since the last set-up: its kernels are loaded
  PinnedScalars hw;  // host staging of scalars written before a loop launch

  double* S() const { return scal.as<double>(); }
  void drop_graphs() {
    for (auto& g : gx)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
    if (gloop) {
      cudaGraphExecDestroy(gloop);
      gloop = nullptr;
    }
  }
  template <typename F>
  void capture_loop(F&& body);
  ~sipg_solver() {
    drop_graphs();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }

  double read_scalar(int slot) {
    SIPG_CUDA(cudaMemcpyAsync(hs.h + slot, S() + slot, sizeof(double), cudaMemcpyDeviceToHost, stream));
    SIPG_CUDA(cudaStreamSynchronize(stream));
    return hs.h[slot];
  }
  // all device scalars to the host with one synchronisation
  void read_scalars() {
    SIPG_CUDA(cudaMemcpyAsync(hs.h, S(), S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SIPG_CUDA(cudaStreamSynchronize(stream));
  }
  template <typename F>
  void capture_iteration(int par, F&& body);

  void dot(const double* a, const double* b, int slot) {
    const double* aa[1] = {a};
    const double* bb[1] = {b};
    multi_dot<double>(aa, bb, 1, n, S() + slot, 1, rw, stream);
  }

  void setup();
  void setup_body();
  void setup_pmg();
  template <typename T> void vcycle(int l);
  template <typename T> void chebyshev(Level& L, bool want_res, bool first);
  template <typename T> void smooth(Level& L, int sweeps, bool want_res, bool first);
  template <typename T> void coarse(Level& L);
  template <typename T> void amg_vcycle(int l);
  template <typename T> void last_level_amg(Level& L);
  template <typename T> const T* csr_chebyshev(AmgDevLevel& A, const T* rin, bool first, bool want_res);
  void setup_amg();
  void precondition(const double* rin, double* zout);
  int solve(const double* b, double* x, sipg_solve_info* info);
  double power_lmax(sipg_op* lop, const double* dinv64, size_t nl, const double* blocks = nullptr, int Np = 0);
  double power_lmax_csr(const AmgDevLevel& D);
  double power_lmax_f32(Level& L);
};

// Diagonal of an operator (FP64), with its pinned DOF.
static void op_diag(sipg_op* op, double* out, cudaStream_t s) {
  SIPG_CUDA(launch_blocks(op->mesh->dim, op->order, op->block_args(BLOCK_DIAG_ONLY, 0, out, true), s));
}

double sipg_solver::power_lmax(sipg_op* lop, const double* dinv64, size_t nl, const double* blocks, int Np) {
  // Power iteration on D^-1 A (D the diagonal, or the diagonal blocks when `blocks`
  // holds their inverses row by row) from v0_i = U(-1,1), splitmix64 seed 0x5eed.
  // work vectors kept across set-ups; the start vector is generated on the device
  if (pl_v.bytes < nl * sizeof(double)) {
    pl_v = DevBuf(nl * sizeof(double));
    pl_w = DevBuf(nl * sizeof(double));
    pl_t = DevBuf(nl * sizeof(double));
  }
  double* v = pl_v.as<double>();
  double* w = pl_w.as<double>();
  double* tb = pl_t.as<double>();
  splitmix_uniform_device(v, nl, 0x5eedull, stream);
  double lam = 0.0;
  for (int it = 0; it < o.eig_iters; ++it) {
    const double* a[1] = {v};
    multi_dot<double>(a, a, 1, nl, S() + S_TMP, 1, rw, stream);
    k_scale<double><<<grid_for(nl), 256, 0, stream>>>(v, nl, S(), S_TMP);
    note_launch();
    if (blocks) {
      lop->apply<double>(v, tb, stream);
      block_matvec<double>(w, blocks, tb, (int)(nl / Np), Np, stream);
    } else {
      lop->apply<double>(v, w, stream);
      k_mul<<<grid_for(nl), 256, 0, stream>>>(w, dinv64, nl);
      note_launch();
    }
    std::swap(v, w);
  }
  // lambda = ||S A v|| of the last step (no host synchronisation before it)
  const double* b[1] = {v};
  multi_dot<double>(b, b, 1, nl, S() + S_TMP, 1, rw, stream);
  lam = std::sqrt(read_scalar(S_TMP));
  return lam;
}

// The FP32 V-cycle's levels with element-block Jacobi smoothing: the same power
// iteration on the operator the smoother sees, B^-1 A with the level's FP32 apply
// (TF32 matrix-free, or the assembled FP16 blocks) and its BF16 inverse blocks.
double sipg_solver::power_lmax_f32(Level& L) {
  const size_t nl = L.n;
  if (pl_v.bytes < nl * sizeof(double)) {
    pl_v = DevBuf(nl * sizeof(double));
    pl_w = DevBuf(nl * sizeof(double));
    pl_t = DevBuf(nl * sizeof(double));
  }
  float* v = pl_v.as<float>();
  float* w = pl_w.as<float>();
  float* t = pl_t.as<float>();
  splitmix_uniform_device(pl_w.as<double>(), nl, 0x5eedull, stream);
  to_f32(v, pl_w.as<double>(), nl, stream);
  const int nb = (int)(nl / L.Np);
  for (int it = 0; it < o.eig_iters; ++it) {
    const float* a[1] = {v};
    multi_dot<float>(a, a, 1, nl, S() + S_TMP, 1, rw, stream);
    k_scale<float><<<grid_for(nl), 256, 0, stream>>>(v, nl, S(), S_TMP);
    note_launch();
    L.apply<float>(v, t, stream);
    // w = B^-1 t (a first Chebyshev step with c2 = 1; the level's z is scratch here)
    if (L.bsym)
      cheb_step_sym<float, __nv_bfloat16>(w, L.z.as<float>(), t, L.bc32.as<__nv_bfloat16>(), 0.0f, 1.0f, nb, L.Np,
                                          stream, true);
    else
      cheb_step_block<float, __nv_bfloat16>(w, L.z.as<float>(), t, L.bc32.as<__nv_bfloat16>(), 0.0f, 1.0f, nb,
                                            L.Np, stream, true);
    std::swap(v, w);
  }
  const float* b[1] = {v};
  multi_dot<float>(b, b, 1, nl, S() + S_TMP, 1, rw, stream);
  return std::sqrt(read_scalar(S_TMP));
}

// The same power iteration on D^-1 A for an algebraic level (CSR, FP64).
double sipg_solver::power_lmax_csr(const AmgDevLevel& D) {
  const size_t nl = (size_t)D.n;
  if (pl_v.bytes < nl * sizeof(double)) {
    pl_v = DevBuf(nl * sizeof(double));
    pl_w = DevBuf(nl * sizeof(double));
    pl_t = DevBuf(nl * sizeof(double));
  }
  double* v = pl_v.as<double>();
  double* w = pl_w.as<double>();
  splitmix_uniform_device(v, nl, 0x5eedull, stream);
  for (int it = 0; it < o.eig_iters; ++it) {
    const double* a[1] = {v};
    multi_dot<double>(a, a, 1, nl, S() + S_TMP, 1, rw, stream);
    k_scale<double><<<grid_for(nl), 256, 0, stream>>>(v, nl, S(), S_TMP);
    note_launch();
    D.A.mv<double>(v, w, 1.0, 0.0, stream);
    k_mul<<<grid_for(nl), 256, 0, stream>>>(w, D.dinv64.as<double>(), nl);
    note_launch();
    std::swap(v, w);
  }
  const double* b[1] = {v};
  multi_dot<double>(b, b, 1, nl, S() + S_TMP, 1, rw, stream);
  return std::sqrt(read_scalar(S_TMP));
}

void sipg_solver::setup_pmg() {
  const int nl = o.n_levels;
  if (nl < 1 || nl > 4) throw Error(SIPG_INVALID_ARG, "n_levels must be 1..4");
  if (o.orders[0] != op->order) throw Error(SIPG_INVALID_ARG, "orders[0] must equal the operator's order");
  for (int l = 1; l < nl; ++l)
    if (o.orders[l] < 1 || o.orders[l] >= o.orders[l - 1]) throw Error(SIPG_INVALID_ARG, "orders must decrease");
  const bool f32 = o.precision == SIPG_FP32;
  const size_t ts = f32 ? sizeof(float) : sizeof(double);
  sipg_mesh* m = op->mesh;
  const int K = m->K, nc = op->ncomp, dim = m->dim;
  PhaseTimer pt(stream);
  if (!lv.empty() && op->oi != (lv[0].own != nullptr)) {  // nodal <-> over-integrated factor: levels anew
    lv.clear();
    al.clear();
    amg_frozen = false;
  }
  if (lv.empty()) {
    lv.resize(nl);
    for (int l = 0; l < nl; ++l) {
      Level& L = lv[l];
      L.order = o.orders[l];
      if (l == 0 && !op->oi) {
        L.op = op;
      } else {
        L.own = create_op(m, L.order, nc);
        L.op = L.own.get();
        set_bc_types_host(L.op, op->bct_host);
      }
      L.Np = L.op->Np;
      L.n = (size_t)nc * K * L.Np;
      L.dinv64 = DevBuf(L.n * sizeof(double));
      if (f32) L.dinv32 = DevBuf(L.n * sizeof(float));
      L.rhs = DevBuf(L.n * ts);
      L.z = DevBuf(L.n * ts);
      L.res = DevBuf(L.n * ts);
      L.d = DevBuf(L.n * ts);
      if (l == nl - 1) {
        L.cp = DevBuf(L.n * ts);
        L.cs = DevBuf(L.n * ts);
        L.cAp = DevBuf(L.n * ts);
      }
      if (l < nl - 1) {
        std::vector<double> P = interp_matrix(dim, o.orders[l + 1], L.order);
        L.P64 = DevBuf(P.size() * sizeof(double));
        L.P64.upload(P.data(), P.size() * sizeof(double));
        std::vector<float> P32(P.begin(), P.end());
        L.P32 = DevBuf(P32.size() * sizeof(float));
        L.P32.upload(P32.data(), P32.size() * sizeof(float));
      }
    }
  }
  // An over-integrated operator is the outer solver's; the V-cycle's finest level
  // is its nodal twin with the projected factor (the factor of the reference's
  // coarse levels, mp_ins_solver.cpp:538-543), kept current here.
  if (op->oi) {
    Level& L0 = lv[0];
    set_bc_types_host(L0.op, op->bct_host);
    set_factor_device(L0.op, op->factor64.as<double>(), stream);
    if (op->mm_mode == SIPG_MM_NODAL) {
      if (!L0.mm64.p) L0.mm64 = DevBuf((size_t)K * L0.Np * sizeof(double));
      SIPG_CUDA(cudaMemcpyAsync(L0.mm64.p, op->mm64.p, (size_t)K * L0.Np * sizeof(double), cudaMemcpyDeviceToDevice,
                                stream));
      set_mm_device(L0.op, SIPG_MM_NODAL, 0.0, L0.mm64.as<double>(), stream);
    } else {
      set_mm_device(L0.op, op->mm_mode, op->mm_scalar, nullptr, stream);
    }
    L0.op->pin_elem = op->pin_elem;
    L0.op->pin_node = op->pin_node;
    SIPG_CUDA(cudaStreamSynchronize(stream));
    if (op->pin_elem >= 0) L0.op->refresh_pin(stream);
  }
  // Coefficients of the coarse levels: interpolate the fine nodal factor / mm.
  for (int l = 1; l < nl; ++l) {
    Level& L = lv[l];
    std::vector<double> I = interp_matrix(dim, o.orders[0], L.order);
    DevBuf Id(I.size() * sizeof(double));
    Id.upload(I.data(), I.size() * sizeof(double));
    if (op->has_factor) {
      if (!L.factor64.p) L.factor64 = DevBuf((size_t)K * L.Np * sizeof(double));
      k_interp<<<grid_for((size_t)K * L.Np), 256, 0, stream>>>(L.factor64.as<double>(), op->factor64.as<double>(),
                                                               Id.as<double>(), K, L.Np, op->Np);
      note_launch();
      set_factor_device(L.op, L.factor64.as<double>(), stream);
    } else {
      L.op->has_factor = false;
      L.op->refresh_tau(stream);
    }
    if (op->mm_mode == SIPG_MM_NODAL) {
      if (!L.mm64.p) L.mm64 = DevBuf((size_t)K * L.Np * sizeof(double));
      k_interp<<<grid_for((size_t)K * L.Np), 256, 0, stream>>>(L.mm64.as<double>(), op->mm64.as<double>(),
                                                               Id.as<double>(), K, L.Np, op->Np);
      note_launch();
      set_mm_device(L.op, SIPG_MM_NODAL, 0.0, L.mm64.as<double>(), stream);
    } else {
      set_mm_device(L.op, op->mm_mode, op->mm_scalar, nullptr, stream);
    }
    if (op->pin_elem >= 0) {
      L.op->pin_elem = op->pin_elem;
      L.op->pin_node = op->pin_node < L.Np ? op->pin_node : 0;
      SIPG_CUDA(cudaStreamSynchronize(stream));
      L.op->refresh_pin(stream);
    } else {
      L.op->pin_elem = -1;
    }
    SIPG_CUDA(cudaStreamSynchronize(stream));
  }
  pt.mark("levels and factors");
  // the point-Jacobi diagonal is read by the Chebyshev smoother without element blocks
  // and by the Jacobi-PCG on the lowest order; the element-block smoother with the
  // algebraic coarse solve reads none
  const bool amg_below = o.coarse_kind == 1 && nc == 1 && lv.back().order == 1;
  for (int l = 0; l < nl; ++l) {
    Level& L = lv[l];
    L.cheb = o.cheb_orders[l] > 0 ? o.cheb_orders[l] : o.cheb_order;
    L.pre = std::max(0, o.pre_it[l]);
    L.post = std::max(0, o.post_it[l]);
    // the Chebyshev bound is read only by a level's smoothing sweeps (a single level with
    // no sweeps is an inner Jacobi-PCG preconditioner)
    const bool smooths = L.pre > 0 || L.post > 0;
    if (o.smoother != 1 || (l == nl - 1 && !amg_below)) {
      op_diag(L.op, L.dinv64.as<double>(), stream);
      k_recip<<<grid_for(L.n), 256, 0, stream>>>(L.dinv64.as<double>(), L.n);
      note_launch();
      if (f32) to_f32(L.dinv32.as<float>(), L.dinv64.as<double>(), L.n, stream);
    }
    DevBuf& rows = rows_ws;  // FP64 inverse diagonal blocks, row-major per element (block-Jacobi smoothing)
    if (o.smoother == 1) {
      // element-block Jacobi: inverse diagonal blocks in the level precision (BF16 for
      // the FP32 V-cycle: the smoother tolerates 8 mantissa bits). Large meshes store
      // them as packed symmetric triangles (one thread per block, half the bytes);
      // small ones as full column-major blocks (ten threads per block at p = 3).
      const int nb = (int)(L.n / L.Np);
      L.bsym = block_sym_supported(L.Np) && nb >= kSymMinBlocks;
      const size_t rb = (size_t)nb * L.Np * L.Np * sizeof(double);
      if (rows.bytes < rb) rows = DevBuf(rb);  // shared by the levels, kept across set-ups
      SIPG_CUDA(launch_blocks(dim, L.order, L.op->block_args(BLOCK_INVERSE, 0, rows.as<double>(), true), stream));
      if (f32 && L.bsym) {
        ensure(L.bc32, block_sym_values<__nv_bfloat16>(nb, L.Np) * sizeof(__nv_bfloat16));
        block_pack_sym<__nv_bfloat16>(L.bc32.as<__nv_bfloat16>(), rows.as<double>(), nb, L.Np, stream);
      } else if (f32) {
        ensure(L.bc32, (size_t)nb * L.Np * L.Np * sizeof(__nv_bfloat16));
        block_transpose<__nv_bfloat16>(L.bc32.as<__nv_bfloat16>(), rows.as<double>(), nb, L.Np, stream);
      } else if (L.bsym) {
        ensure(L.bc64, block_sym_values<double>(nb, L.Np) * sizeof(double));
        block_pack_sym<double>(L.bc64.as<double>(), rows.as<double>(), nb, L.Np, stream);
      } else {
        ensure(L.bc64, (size_t)nb * L.Np * L.Np * sizeof(double));
        block_transpose<double>(L.bc64.as<double>(), rows.as<double>(), nb, L.Np, stream);
      }
      pt.mark("diagonal and blocks", l);
      // the FP32 V-cycle estimates its bound after the assembly, on its own operator
      if (!f32 && smooths) L.lmax = power_lmax(L.op, nullptr, L.n, rows.as<double>(), L.Np);
    } else {
      L.bc64 = DevBuf();
      L.bc32 = DevBuf();
      pt.mark("diagonal", l);
      if (smooths) L.lmax = power_lmax(L.op, L.dinv64.as<double>(), L.n);
    }
    if (!(f32 && o.smoother == 1)) pt.mark("eigenvalue bound", l);
    // -1: p = 2 and below in the FP32 V-cycle (p = 2 as scaled FP16 blocks: half the
    // bytes of the matrix-free apply's per-element work, same iteration counts), p = 1
    // in the FP64 V-cycle (FP64 blocks at p = 2 move more bytes than the matrix-free apply)
    const int amo = o.assembled_max_order >= 0 ? o.assembled_max_order : (f32 ? 2 : 1);
    if (l > 0 && L.order <= amo && bsr_supported(dim, L.order, nc)) {
      if (!L.bsr) L.bsr = std::make_unique<BsrOp>();  // its buffers are reused by later set-ups
      // FP32 V-cycle with packed symmetric block-Jacobi smoothing: also C = Bd^-1 A, so
      // that one kernel per Chebyshev step after the first updates Bd^-1 r directly
      const bool fused = f32 && o.smoother == 1 && L.Np % 2 == 0;
      bsr_assemble(L.op, *L.bsr, f32, stream, fused ? rows.as<double>() : nullptr, L.bsym);
      pt.mark("assembled blocks", l);
      if (L.bsr->c16.p) {
        ensure(L.d2, L.n * sizeof(float));
        ensure(L.sres, L.n * sizeof(float));
      }
    } else {
      L.bsr.reset();
    }
    if (f32 && o.smoother == 1 && smooths) {
      L.lmax = power_lmax_f32(L);
      pt.mark("eigenvalue bound", l);
    }
  }
  use_amg = o.coarse_kind == 1 && nc == 1 && lv.back().order == 1;
  if (use_amg) setup_amg();
  pt.mark("algebraic levels");
}

// Algebraic levels below the p = 1 level. The continuous P1 operator is assembled
// on the device from the level's factor and penalty. The first set-up (and any
// set-up after the boundary types or the singularity of the problem changed, or
// every set-up with amg_reuse_interpolation = 0) aggregates on the host and stores
// the prolongators and the Galerkin term lists; every set-up then recomputes the
// level operators, their inverse diagonals and eigenvalue bounds and the coarsest
// inverse on the device.
void sipg_solver::setup_amg() {
  Level& L = lv.back();
  sipg_op* lop = L.op;
  sipg_mesh* m = op->mesh;
  const int K = m->K, Np1 = L.Np;
  bool any_dirichlet = false;
  for (int b = 0; b < m->Kb; ++b) any_dirichlet |= op->bct_host[b] == SIPG_BC_DIRICHLET;
  const bool singular = !any_dirichlet && lop->mm_mode == SIPG_MM_NONE;
  PhaseTimer pt(stream);
  {
    std::lock_guard<std::mutex> lk(m->probe_mu);
    if (!m->p1_plan) m->p1_plan = std::make_shared<P1Plan>(p1c_plan(K, m->Nv, Np1, m->e2v.data()));
    if (!m->p1_gather) {
      auto g = std::make_shared<DevTerms>();
      g->upload(p1c_gather_plan(*m->p1_plan, K, Np1));
      m->p1_gather = g;
    }
  }
  const P1Plan& plan = *m->p1_plan;
  const DevTerms& gather = *std::static_pointer_cast<DevTerms>(m->p1_gather);
  const size_t nnz0 = plan.idx.size();
  ensure(p1_blk, (size_t)K * Np1 * Np1 * sizeof(double));
  p1c_blocks_device(p1_tables(dev_ref(m->dim, 1).ref), K, m->geof64.as<double>(),
                    lop->has_factor ? lop->factor64.as<double>() : nullptr, lop->tau64.as<double>(), m->nbr.as<int>(),
                    lop->bct.as<unsigned char>(), lop->mm_mode, lop->mm_scalar,
                    lop->mm_mode == SIPG_MM_NODAL ? lop->mm64.as<double>() : nullptr, p1_blk.as<double>(), stream);
  const bool reuse = o.amg_reuse_interpolation != 0 && amg_frozen && !al.empty() && amg_bct == op->bct_host &&
                     amg_singular == singular;
  const bool f32 = o.precision == SIPG_FP32;
  const size_t ts = f32 ? sizeof(float) : sizeof(double);
  if (!reuse) {
    amg_frozen = false;
    ensure(a0_tmp, nnz0 * sizeof(double));
    gather.run(p1_blk.as<double>(), a0_tmp.as<double>(), nullptr, stream);
    Csr A0;
    A0.rows = A0.cols = m->Nv;
    A0.ptr = plan.ptr;
    A0.idx = plan.idx;
    A0.val.resize(nnz0);
    SIPG_CUDA(cudaMemcpyAsync(A0.val.data(), a0_tmp.p, nnz0 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    SIPG_CUDA(cudaStreamSynchronize(stream));
    // injection of vertex values into the p = 1 nodes: row (e, i) has one entry at e2v[e][i]
    Csr Pd;
    Pd.rows = K * Np1;
    Pd.cols = m->Nv;
    Pd.ptr.resize(Pd.rows + 1);
    for (int k = 0; k <= Pd.rows; ++k) Pd.ptr[k] = k;
    Pd.idx.assign(m->e2v.begin(), m->e2v.begin() + Pd.rows);
    Pd.val.assign(Pd.rows, 1.0);
    pt.mark("P1 operator (device)");
    AmgHierarchy H = build_amg(A0, Pd, std::max(2, o.amg_coarse_max), o.amg_strength, singular, false);
    pt.mark("aggregation (host)");
    Pdg.upload(H.Pdg);
    Rdg.upload(H.Rdg);
    al.clear();
    al.resize(H.levels.size());
    for (size_t l = 0; l < H.levels.size(); ++l) {
      AmgDevLevel& D = al[l];
      const AmgLevel& HL = H.levels[l];
      D.n = HL.A.rows;
      D.A.upload(HL.A);
      if (l + 1 < H.levels.size()) {
        D.P.upload(HL.P);
        D.R.upload(HL.R);
        Csr APs, RAPs;
        const TermPlan tap = spgemm_plan(HL.A, HL.P, true, &APs);
        const TermPlan trap = spgemm_plan(HL.R, APs, false, &RAPs);
        const Csr& next = H.levels[l + 1].A;
        if (RAPs.ptr != next.ptr || RAPs.idx != next.idx)
          throw Error(SIPG_CUDA_ERROR, "algebraic set-up: Galerkin term lists do not match the coarse operator");
        D.ap.upload(tap);
        D.rap.upload(trap);
        D.apv = DevBuf(std::max<size_t>(1, APs.nnz()) * sizeof(double));
        D.dinv64 = DevBuf(D.n * sizeof(double));
        D.dinv32 = DevBuf(D.n * sizeof(float));
      }
      D.rhs = DevBuf(D.n * ts);
      D.z = DevBuf(D.n * ts);
      D.res = DevBuf(D.n * ts);
      D.d = DevBuf(D.n * ts);
      D.res2 = DevBuf(D.n * ts);
      D.d2 = DevBuf(D.n * ts);
    }
    cinv_n = H.coarse_n;
    const size_t nn = (size_t)cinv_n * cinv_n;
    ensure(cinv64, nn * sizeof(double));
    ensure(cinv32, nn * sizeof(float));
    ensure(cinv_work, ((size_t)2 * cinv_n + 1024) * sizeof(double));
    amg_bct = op->bct_host;
    amg_singular = singular;
    amg_frozen = true;
    pt.mark("hierarchy upload");
  }
  // level operators from the stored prolongators (Galerkin products on the device)
  gather.run(p1_blk.as<double>(), al[0].A.v64.as<double>(), al[0].A.v32.as<float>(), stream);
  for (size_t l = 0; l + 1 < al.size(); ++l) {
    AmgDevLevel& D = al[l];
    D.ap.run(D.A.v64.as<double>(), D.apv.as<double>(), nullptr, stream);
    D.rap.run(D.apv.as<double>(), al[l + 1].A.v64.as<double>(), al[l + 1].A.v32.as<float>(), stream);
    csr_dinv_device(D.n, D.A.ptr.as<int>(), D.A.idx.as<int>(), D.A.v64.as<double>(), D.dinv64.as<double>(),
                    D.dinv32.as<float>(), stream);
    D.lmax = power_lmax_csr(D);
  }
  pt.mark("algebraic levels (device)");
  // the coarsest level is inverted on the device (FP64 blocked Gauss-Jordan), then copied to FP32
  const AmgDevLevel& C = al.back();
  const size_t nn = (size_t)cinv_n * cinv_n;
  csr_to_dense_device(cinv_n, C.A.ptr.as<int>(), C.A.idx.as<int>(), C.A.v64.as<double>(), cinv64.as<double>(),
                      singular, stream);
  dense_inverse_device(cinv64.as<double>(), cinv_n, singular, cinv_work.as<double>(), stream);
  to_f32(cinv32.as<float>(), cinv64.as<double>(), nn, stream);
  pt.mark("coarsest inverse (device)");
}

// A set-up that fails part-way leaves no half-built levels behind: the next
// solve builds them again from the start.
void sipg_solver::setup() {
  std::lock_guard<std::recursive_mutex> first_use(g_graph_mu);
  warm = false;
  try {
    setup_body();
  } catch (...) {
    lv.clear();
    al.clear();
    amg_frozen = false;
    use_amg = false;
    dirty = true;
    throw;
  }
}

void sipg_solver::setup_body() {
  drop_graphs();
  graph_broken = false;
  gloop_broken = false;
  n = (size_t)op->ncomp * op->mesh->K * op->Np;
  if (!r.p) {
    size_t b = n * sizeof(double);
    r = DevBuf(b); z = DevBuf(b); p = DevBuf(b); Ap = DevBuf(b);
    scal = DevBuf(S_COUNT * sizeof(double));
    partial = DevBuf(kRedBlocks * 4 * sizeof(double));
    counter = DevBuf(sizeof(unsigned));
    SIPG_CUDA(cudaMemsetAsync(counter.p, 0, sizeof(unsigned), stream));
    SIPG_CUDA(cudaMemsetAsync(scal.p, 0, S_COUNT * sizeof(double), stream));
    rw.partial = partial.as<double>();
    rw.counter = counter.as<unsigned>();
    if (kind == SIPG_SOLVER_PMULTIGRID && o.precision == SIPG_FP32) {
      r32 = DevBuf(n * sizeof(float));
      z32 = DevBuf(n * sizeof(float));
    }
  }
  if (kind == SIPG_SOLVER_JACOBI) {
    if (!dinv.p) dinv = DevBuf(n * sizeof(double));
    op_diag(op, dinv.as<double>(), stream);
    k_recip<<<grid_for(n), 256, 0, stream>>>(dinv.as<double>(), n);
      note_launch();
  } else if (kind == SIPG_SOLVER_BLOCK_JACOBI) {
    if (!blocks.p) blocks = DevBuf(n * op->Np * sizeof(double));
    SIPG_CUDA(launch_blocks(op->mesh->dim, op->order,
                            op->block_args(BLOCK_INVERSE, o.ref_volume_block, blocks.as<double>(), true), stream));
  } else if (kind == SIPG_SOLVER_INV_MASS) {
    if (!minv.p) {
      const RefElement& re = op->dref->ref;
      std::vector<double> mi(re.Minv);
      minv = DevBuf(mi.size() * sizeof(double));
      minv.upload(mi.data(), mi.size() * sizeof(double), stream);
    }
  } else if (kind == SIPG_SOLVER_PMULTIGRID) {
    setup_pmg();
  }
  SIPG_CUDA(cudaStreamSynchronize(stream));
  dirty = false;
}

// One Chebyshev sweep on z with the residual res kept current (except, when
// !want_res, after the last step). `first`: z = 0 and res = rhs before the sweep,
// which the first step reads from rhs directly (no zeroing or copy).
template <typename T>
void sipg_solver::chebyshev(Level& L, bool want_res, bool first) {
  const double hi = L.lmax * o.eig_safety, lo = hi / o.eig_ratio;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
  double rho_old = 1.0 / sigma;
  const T* dinv = std::is_same<T, float>::value ? (const T*)L.dinv32.p : (const T*)L.dinv64.p;
  T* d = L.d.as<T>();
  T* z = L.z.as<T>();
  T* res = L.res.as<T>();
  if (std::is_same<T, float>::value && L.bsr && L.bsr->c16.p && L.bc32.p) {
    // first step from Bd^-1 r (block smoother kernel), then one fused kernel per step
    // on C = Bd^-1 A with s = Bd^-1 r kept current; the residual, where wanted, from rhs
    const bool from_rhs = first;
    const T* rin = from_rhs ? L.rhs.as<T>() : res;
    const int nb = (int)(L.n / L.Np);
    if (L.bsym)
      cheb_step_sym<float, __nv_bfloat16>((float*)d, (float*)z, (const float*)rin, L.bc32.as<__nv_bfloat16>(), 0.0f,
                                          (float)(1.0 / theta), nb, L.Np, stream, from_rhs);
    else
      cheb_step_block<float, __nv_bfloat16>((float*)d, (float*)z, (const float*)rin, L.bc32.as<__nv_bfloat16>(),
                                            0.0f, (float)(1.0 / theta), nb, L.Np, stream, from_rhs);
    float* dc = (float*)d;
    float* dn = L.d2.as<float>();
    for (int it = 1; it < L.cheb; ++it) {
      const double rho = 1.0 / (2.0 * sigma - rho_old);
      const double c1 = rho * rho_old, c2 = 2.0 * rho / delta;
      rho_old = rho;
      bsr_cheb_step(*L.bsr, dc, dn, L.sres.as<float>(), (float*)z, (float)c1, (float)c2,
                    it == 1 ? (float)theta : 0.0f, stream);
      std::swap(dc, dn);
    }
    if (want_res) L.apply<T>(z, res, stream, T(-1), T(1), L.rhs.as<T>());
    return;
  }
  for (int it = 0; it < L.cheb; ++it) {
    double c1 = 0.0, c2 = 1.0 / theta;
    if (it > 0) {
      double rho = 1.0 / (2.0 * sigma - rho_old);
      c1 = rho * rho_old;
      c2 = 2.0 * rho / delta;
      rho_old = rho;
    }
    const bool from_rhs = first && it == 0;
    const T* rin = from_rhs ? L.rhs.as<T>() : res;
    const int nb = (int)(L.n / L.Np);
    if (L.bc32.p && std::is_same<T, float>::value && L.bsym) {
      cheb_step_sym<float, __nv_bfloat16>((float*)d, (float*)z, (const float*)rin, L.bc32.as<__nv_bfloat16>(),
                                          (float)c1, (float)c2, nb, L.Np, stream, from_rhs);
    } else if (L.bc32.p && std::is_same<T, float>::value) {
      cheb_step_block<float, __nv_bfloat16>((float*)d, (float*)z, (const float*)rin, L.bc32.as<__nv_bfloat16>(),
                                            (float)c1, (float)c2, nb, L.Np, stream, from_rhs);
    } else if (L.bc64.p && std::is_same<T, double>::value && L.bsym) {
      cheb_step_sym<double, double>((double*)d, (double*)z, (const double*)rin, L.bc64.as<double>(), (double)c1,
                                    (double)c2, nb, L.Np, stream, from_rhs);
    } else if (L.bc64.p) {
      cheb_step_block<T, T>(d, z, rin, (const T*)L.bc64.p, (T)c1, (T)c2, nb, L.Np, stream, from_rhs);
    } else {
      cheb_step<T>(d, z, rin, dinv, (T)c1, (T)c2, L.n, stream, from_rhs);
    }
    if (it < L.cheb - 1 || want_res) L.apply<T>(d, res, stream, T(-1), T(1), rin);
  }
}

// `sweeps` Chebyshev sweeps on z with residual res; the residual is kept current
// except, when !want_res, after the last sweep. `first`: from z = 0, res = rhs.
template <typename T>
void sipg_solver::smooth(Level& L, int sweeps, bool want_res, bool first) {
  for (int k = 0; k < sweeps; ++k) chebyshev<T>(L, k < sweeps - 1 || want_res, first && k == 0);
}

template <typename T>
void sipg_solver::coarse(Level& L) {
  // Fixed-count Jacobi-PCG from zero on the coarsest order, scalars on device.
  const T* dinv = std::is_same<T, float>::value ? (const T*)L.dinv32.p : (const T*)L.dinv64.p;
  T* z = L.z.as<T>();
  T* res = L.res.as<T>();
  T* cp = L.cp.as<T>();
  T* cs = L.cs.as<T>();
  T* cAp = L.cAp.as<T>();
  vzero<T>(z, L.n, stream);
  vcopy<T>(res, L.rhs.as<T>(), L.n, stream);
  jacobi<T>(cs, res, dinv, L.n, stream);
  vcopy<T>(cp, cs, L.n, stream);
  {
    const T* a[1] = {res};
    const T* b[1] = {cs};
    multi_dot<T>(a, b, 1, L.n, S() + S_C_RZ, 1, rw, stream);
  }
  for (int it = 0; it < o.coarse_iters; ++it) {
    L.apply<T>(cp, cAp, stream);
    const T* a[1] = {cp};
    const T* b[1] = {cAp};
    multi_dot<T>(a, b, 1, L.n, S() + S_C_PAP, 1, rw, stream);
    coarse_update<T>(z, res, cs, cp, cAp, dinv, L.n, S(), rw, stream);
    coarse_update_p<T>(cp, cs, L.n, S(), stream);
  }
}

// Chebyshev sweep on an algebraic level from the residual rin (z = 0 before it when
// `first`), one fused kernel per step; returns the final residual (null when
// !want_res).
template <typename T>
const T* sipg_solver::csr_chebyshev(AmgDevLevel& A, const T* rin, bool first, bool want_res) {
  const double hi = A.lmax * o.eig_safety, lo = hi / o.eig_ratio;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
  double rho_old = 1.0 / sigma;
  const T* dinv = std::is_same<T, float>::value ? (const T*)A.dinv32.p : (const T*)A.dinv64.p;
  T* dbuf[2] = {A.d.as<T>(), A.d2.as<T>()};
  T* rbuf[2] = {A.res.as<T>(), A.res2.as<T>()};
  const T* dcur = nullptr;  // not read by the first step (c1 = 0)
  const T* rcur = rin;
  int ob = rin == rbuf[0] ? 1 : 0;
  const int deg = o.amg_cheb_order > 0 ? o.amg_cheb_order : o.cheb_order;
  for (int it = 0; it < deg; ++it) {
    double c1 = 0.0, c2 = 1.0 / theta;
    if (it > 0) {
      double rho = 1.0 / (2.0 * sigma - rho_old);
      c1 = rho * rho_old;
      c2 = 2.0 * rho / delta;
      rho_old = rho;
    }
    T* dn = dbuf[ob];
    T* rn = (it < deg - 1 || want_res) ? rbuf[ob] : nullptr;
    csr_cheb<T>(A.n, A.A.ptr.as<int>(), A.A.idx.as<int>(), A.A.vals<T>(), dcur ? dcur : dn, rcur, dinv, dn, rn,
                A.z.as<T>(), (T)c1, (T)c2, first && it == 0, stream);
    dcur = dn;
    rcur = rn;
    ob ^= 1;
  }
  return rcur;
}

template <typename T>
void sipg_solver::amg_vcycle(int l) {
  AmgDevLevel& A = al[l];
  if (l == (int)al.size() - 1) {
    const T* inv = std::is_same<T, float>::value ? (const T*)cinv32.p : (const T*)cinv64.p;
    dense_mv<T>(cinv_n, inv, A.rhs.as<T>(), A.z.as<T>(), stream);
    return;
  }
  AmgDevLevel& Cn = al[l + 1];
  const T* r = csr_chebyshev<T>(A, A.rhs.as<T>(), true, true);
  A.R.mv<T>(r, Cn.rhs.as<T>(), T(1), T(0), stream);
  amg_vcycle<T>(l + 1);
  A.P.mv<T>(Cn.z.as<T>(), A.z.as<T>(), T(1), T(1), stream);
  A.A.mv<T>(A.z.as<T>(), A.res2.as<T>(), T(-1), T(1), stream, A.rhs.as<T>());
  csr_chebyshev<T>(A, A.res2.as<T>(), false, false);
}

// Lowest order with the algebraic coarse space: Chebyshev, R_dg, AMG V-cycle,
// P_dg, Chebyshev.
template <typename T>
void sipg_solver::last_level_amg(Level& L) {
  if (L.pre > 0) {
    smooth<T>(L, L.pre, true, true);
    Rdg.mv<T>(L.res.as<T>(), al[0].rhs.as<T>(), T(1), T(0), stream);
  } else {
    vzero<T>(L.z.as<T>(), L.n, stream);
    Rdg.mv<T>(L.rhs.as<T>(), al[0].rhs.as<T>(), T(1), T(0), stream);
  }
  amg_vcycle<T>(0);
  Pdg.mv<T>(al[0].z.as<T>(), L.z.as<T>(), T(1), T(1), stream);
  if (L.post > 0) {
    L.apply<T>(L.z.as<T>(), L.res.as<T>(), stream, T(-1), T(1), L.rhs.as<T>());
    smooth<T>(L, L.post, false, false);
  }
}

template <typename T>
void sipg_solver::vcycle(int l) {
  Level& L = lv[l];
  const int nl = (int)lv.size();
  if (l == nl - 1) {
    if (use_amg) last_level_amg<T>(L);
    else coarse<T>(L);
    return;
  }
  Level& Cl = lv[l + 1];
  const bool f32 = std::is_same<T, float>::value;
  const T* P = f32 ? (const T*)L.P32.p : (const T*)L.P64.p;
  const int K = op->mesh->K, nc = op->ncomp;
  if (L.pre > 0) {
    smooth<T>(L, L.pre, true, true);
    restrict_elem<T>(Cl.rhs.as<T>(), L.res.as<T>(), P, K, L.Np, Cl.Np, nc, stream);
  } else {
    vzero<T>(L.z.as<T>(), L.n, stream);
    restrict_elem<T>(Cl.rhs.as<T>(), L.rhs.as<T>(), P, K, L.Np, Cl.Np, nc, stream);
  }
  vcycle<T>(l + 1);
  prolong_add<T>(L.z.as<T>(), Cl.z.as<T>(), P, K, L.Np, Cl.Np, nc, stream);
  if (L.post > 0) {
    L.apply<T>(L.z.as<T>(), L.res.as<T>(), stream, T(-1), T(1), L.rhs.as<T>());
    smooth<T>(L, L.post, false, false);
  }
}

void sipg_solver::precondition(const double* rin, double* zout) {
  switch (kind) {
    case SIPG_SOLVER_INV_MASS: {
      const int dim = op->mesh->dim;
      inv_mass<double>(zout, rin, minv.as<double>(), op->mesh->geof64.as<double>(), dim == 3 ? 10 : 5,
                       dim == 3 ? 9 : 4, op->mesh->K, op->Np, op->ncomp, o.inv_mass_factor, stream);
      break;
    }
    case SIPG_SOLVER_JACOBI:
      jacobi<double>(zout, rin, dinv.as<double>(), n, stream);
      break;
    case SIPG_SOLVER_BLOCK_JACOBI:
      block_matvec<double>(zout, blocks.as<double>(), rin, (int)(n / op->Np), op->Np, stream);
      break;
    case SIPG_SOLVER_PMULTIGRID:
      if (o.precision == SIPG_FP32) {
        to_f32(lv[0].rhs.as<float>(), rin, n, stream);
        vcycle<float>(0);
        to_f64(zout, lv[0].z.as<float>(), n, stream);
      } else {
        vcopy<double>(lv[0].rhs.as<double>(), rin, n, stream);
        vcycle<double>(0);
        vcopy<double>(zout, lv[0].z.as<double>(), n, stream);
      }
      break;
    default:
      vcopy<double>(zout, rin, n, stream);
  }
  if (o.nullspace) {
    vsum<double>(zout, n, S() + S_SUM, rw, stream);
    sub_mean<double>(zout, n, S(), S_SUM, stream);
  }
}

// Capture one outer iteration into gx[par]; on any failure the solver keeps
// launching kernels one by one.
template <typename F>
void sipg_solver::capture_iteration(int par, F&& body) {
  std::lock_guard<std::recursive_mutex> capture_lock(g_graph_mu);
  unsigned long long nodes = 0;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    cudaGetLastError();
    graph_broken = true;
    return;
  }
  bool ok = true;
  record_launches(&nodes);  // recorded, not launched
  try {
    body();
  } catch (...) {
    ok = false;
  }
  record_launches(nullptr);
  cudaError_t e = cudaStreamEndCapture(stream, &g);
  if (!ok || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    graph_broken = true;
    return;
  }
  e = cudaGraphInstantiate(&gx[par], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    gx[par] = nullptr;
    cudaGetLastError();
    graph_broken = true;
    return;
  }
  gnodes[par] = nodes;
}

// Build gloop: a conditional while-node whose body is one iteration followed by
// the stopping test. On any failure the solver falls back to per-iteration graphs.
template <typename F>
void sipg_solver::capture_loop(F&& body) {
  std::lock_guard<std::recursive_mutex> capture_lock(g_graph_mu);
  unsigned long long nodes = 0;
  cudaGraph_t g = nullptr;
  bool ok = cudaGraphCreate(&g, 0) == cudaSuccess;
  cudaGraphConditionalHandle h{};
  cudaGraphNodeParams cp{};
  cudaGraphNode_t node = nullptr;
  if (ok) ok = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
  if (ok) {
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    ok = cudaGraphAddNode(&node, g, nullptr, 0, &cp) == cudaSuccess;
  }
  if (ok) ok = cudaStreamBeginCaptureToGraph(stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeRelaxed) == cudaSuccess;
  if (ok) {
    bool body_ok = true;
    record_launches(&nodes);  // recorded, not launched
    try {
      body();
      k_loop_check<<<1, 1, 0, stream>>>(S(), h, o.max_iter);
      note_launch();
    } catch (...) {
      body_ok = false;
    }
    record_launches(nullptr);
    cudaGraph_t out = nullptr;
    ok = cudaStreamEndCapture(stream, &out) == cudaSuccess && body_ok;
  }
  if (ok) ok = cudaGraphInstantiate(&gloop, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    if (gloop) cudaGraphExecDestroy(gloop);
    gloop = nullptr;
    cudaGetLastError();
    gloop_broken = true;
    return;
  }
  gloop_nodes = nodes;
}

int sipg_solver::solve(const double* b, double* x_user, sipg_solve_info* info) {
  std::unique_lock<std::recursive_mutex> first_use(g_graph_mu, std::defer_lock);
  if (!warm || dirty) first_use.lock();
  auto t0 = std::chrono::steady_clock::now();
  if (dirty) setup();
  auto t1 = std::chrono::steady_clock::now();
  const bool graphs = o.graphs != 0 && kind != SIPG_SOLVER_CG;
  if (graphs && gver != op->version) {
    drop_graphs();
    gver = op->version;
  }
  if (graphs && !xi.p) xi = DevBuf(n * sizeof(double));
  SIPG_CUDA(cudaEventRecord(ev0, stream));
  double* x = graphs ? xi.as<double>() : x_user;
  if (graphs) vcopy<double>(x, x_user, n, stream);
  double* R = r.as<double>();
  double* Z = z.as<double>();
  double* Pv = p.as<double>();
  double* AP = Ap.as<double>();
  // r = b - A x (calc_res_explicit, viscous_solver.cpp:329-343)
  vcopy<double>(R, b, n, stream);
  op->apply<double>(x, R, stream, -1.0, 1.0);
  if (o.nullspace) {
    vsum<double>(R, n, S() + S_SUM, rw, stream);
    sub_mean<double>(R, n, S(), S_SUM, stream);
  }
  dot(b, b, S_BB);
  dot(R, R, S_RR);
  read_scalars();
  const double bnorm = std::sqrt(hs.h[S_BB]);
  double res = std::sqrt(hs.h[S_RR]);
  const double tol = std::max(o.abs_tol, o.rel_tol * bnorm);
  int iter = 0, status = SIPG_OK;
  if (!std::isfinite(bnorm) || !std::isfinite(res)) {
    status = SIPG_BREAKDOWN;
    res = NAN;
  }
  if (kind == SIPG_SOLVER_CG) {
    // conjugate_gradient: explicit residual every iteration (viscous_solver.cpp:115-160)
    vcopy<double>(Pv, R, n, stream);
    while (status == SIPG_OK && res > tol && iter < o.max_iter) {
      op->apply<double>(Pv, AP, stream);
      const double* a[2] = {R, Pv};
      const double* bb[2] = {R, AP};
      multi_dot<double>(a, bb, 2, n, S() + S_RZ, 1, rw, stream);  // S_RZ = r.r, S_PAP = p.Ap
      // x += alpha p; r is recomputed below, the rr output is unused here
      cg_update_xr(x, Z, Pv, AP, n, S(), S_RZ, S_PAP, S() + S_TMP, rw, stream);
      vcopy<double>(R, b, n, stream);
      op->apply<double>(x, R, stream, -1.0, 1.0);
      if (o.nullspace) {
        vsum<double>(R, n, S() + S_SUM, rw, stream);
        sub_mean<double>(R, n, S(), S_SUM, stream);
      }
      dot(R, R, S_RR);
      update_p<double>(Pv, R, n, S(), S_RR, S_RZ, stream);
      ++iter;
      read_scalars();
      const double pap = hs.h[S_PAP];
      res = std::sqrt(hs.h[S_RR]);
      if (!(pap > 0.0) || !std::isfinite(res)) { status = SIPG_BREAKDOWN; break; }
      if (cancel && cancel->load(std::memory_order_relaxed)) { status = SIPG_CANCELLED; break; }
    }
  } else {
    // flexible PCG (viscous_solver.cpp:177-301). One iteration on fixed buffers: z is
    // overwritten in place and beta = r.z_new - r.z_old comes from two dots.
    if (status == SIPG_OK) precondition(R, Z);
    vcopy<double>(Pv, Z, n, stream);
    dot(R, Z, S_RZ);
    // mixed p-multigrid: the nullspace projections, the FP32 / FP64 conversions and
    // the dots ride on the vector passes next to them
    const bool fused = kind == SIPG_SOLVER_PMULTIGRID && o.precision == SIPG_FP32;
    const int mean_slot = o.nullspace ? (int)S_SUM : -1;
    auto body = [&] {
      op->apply<double>(Pv, AP, stream);
      dot(Pv, AP, S_PAP);  // cg3_alpha_pre
      if (fused) {
        // update_ans + update_res, projection, r . r, r . z_old, r to FP32
        if (o.nullspace) cg_update_xr_sum(x, R, Pv, AP, n, S(), S_RZ, S_PAP, S() + S_SUM, S_TMP - S_SUM, rw, stream);
        else cg_update_xr(x, R, Pv, AP, n, S(), S_RZ, S_PAP, S() + S_TMP, rw, stream);
        resid_prep(R, lv[0].rhs.as<float>(), Z, n, S(), mean_slot, S() + S_RR, S_RZO - S_RR, rw, stream);
        vcycle<float>(0);
        // z to FP64, projection, r . z_new
        if (o.nullspace) to_f64_sum(Z, lv[0].z.as<float>(), n, S() + S_SUM, rw, stream);
        finish_z_dot(Z, o.nullspace ? nullptr : lv[0].z.as<float>(), R, n, S(), mean_slot, S() + S_RZN, rw, stream);
      } else if (!o.nullspace && (kind == SIPG_SOLVER_JACOBI || kind == SIPG_SOLVER_BLOCK_JACOBI)) {
        // update_ans + update_res with r . r and r . z_old; z = M^-1 r with r . z_new
        cg_update_xr_rzo(x, R, Pv, AP, Z, n, S(), S_RZ, S_PAP, S() + S_RR, S_RZO - S_RR, rw, stream);
        if (kind == SIPG_SOLVER_JACOBI) precond_dot(Z, R, dinv.as<double>(), 0, n, S() + S_RZN, rw, stream);
        else precond_dot(Z, R, blocks.as<double>(), op->Np, n, S() + S_RZN, rw, stream);
      } else {
        cg_update_xr(x, R, Pv, AP, n, S(), S_RZ, S_PAP, S() + S_RR, rw, stream);  // update_ans + update_res
        if (o.nullspace) {
          vsum<double>(R, n, S() + S_SUM, rw, stream);
          sub_mean<double>(R, n, S(), S_SUM, stream);
          dot(R, R, S_RR);
        }
        dot(R, Z, S_RZO);
        precondition(R, Z);
        dot(R, Z, S_RZN);
      }
      k_beta_flex<<<1, 1, 0, stream>>>(S());  // cg3_compute_beta_pre_flex
      note_launch();
      update_p<double>(Pv, Z, n, S(), S_BETA, S_RZP, stream);
    };
    auto after = [&](int it_now) {
      iter = it_now;
      const double pap = hs.h[S_PAP];
      res = std::sqrt(hs.h[S_RR]);
      if (!(pap > 0.0) || !std::isfinite(res)) status = SIPG_BREAKDOWN;
      else if (cancel && cancel->load(std::memory_order_relaxed)) status = SIPG_CANCELLED;
    };
    // graphs = 2: the iterations after the first run inside gloop, whose while-node
    // repeats the body until k_loop_check ends it; the host reads the scalars once
    // per launch of at most kLoopChunk iterations. graphs = 1: one graph launch per
    // iteration. The first iteration runs eagerly (lazy buffers are allocated there).
    constexpr int kLoopChunk = 64;
    while (status == SIPG_OK && res > tol && iter < o.max_iter) {
      if (graphs && iter >= 1 && o.graphs >= 2 && !gloop && !gloop_broken) capture_loop(body);
      if (graphs && iter >= 1 && gloop) {
        hw.h[S_ITER] = (double)iter;
        hw.h[S_STATUS] = 0.0;
        hw.h[S_TOL] = tol;
        hw.h[S_CHUNK] = (double)kLoopChunk;
        SIPG_CUDA(cudaMemcpyAsync(S() + S_ITER, hw.h + S_ITER, 4 * sizeof(double), cudaMemcpyHostToDevice, stream));
        SIPG_CUDA(cudaGraphLaunch(gloop, stream));
        read_scalars();
        const int done = (int)hs.h[S_ITER];
        note_launch((unsigned)((done - iter) * gloop_nodes));
        after(done);
        continue;
      }
      if (graphs && iter >= 1 && !gx[0] && !graph_broken) capture_iteration(0, body);
      if (graphs && iter >= 1 && gx[0]) {
        SIPG_CUDA(cudaGraphLaunch(gx[0], stream));
        note_launch((unsigned)gnodes[0]);
      } else {
        body();
      }
      read_scalars();
      after(iter + 1);
    }
  }
  if (status == SIPG_OK && res > tol) status = SIPG_NOT_CONVERGED;
  SIPG_CUDA(cudaEventRecord(ev1, stream));
  // final defect with an explicit FP64 apply
  vcopy<double>(AP, b, n, stream);
  op->apply<double>(x, AP, stream, -1.0, 1.0);
  if (o.nullspace) {
    vsum<double>(AP, n, S() + S_SUM, rw, stream);
    sub_mean<double>(AP, n, S(), S_SUM, stream);
  }
  dot(AP, AP, S_TMP);
  if (graphs) vcopy<double>(x_user, x, n, stream);
  double true_res = std::sqrt(read_scalar(S_TMP));
  float ms = 0.f;
  SIPG_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  if (info) {
    info->iters = iter;
    info->abs_res = res;
    info->rel_res = bnorm > 0 ? res / bnorm : res;
    info->true_rel_res = bnorm > 0 ? true_res / bnorm : true_res;
    info->setup_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    info->solve_ms = ms;
    info->status = status;
  }
  warm = true;
  return status;
}

namespace sipg {
void solver_set_cancel(sipg_solver* s, const std::atomic<int>* flag) { s->cancel = flag; }
cudaStream_t solver_stream(sipg_solver* s) { return s->stream; }
}  // namespace sipg

extern "C" {

int sipg_solver_default_opts(int kind, sipg_solver_opts* o) {
  return guarded([&] {
    if (!o) throw Error(SIPG_INVALID_ARG, "null opts");
    std::memset(o, 0, sizeof(*o));
    // set_tol_and_iter defaults of the pressure solve (ins_solver_base.cpp:153-160)
    o->rel_tol = 1e-8;
    o->abs_tol = 1e-9;
    o->max_iter = 500;
    o->precision = SIPG_FP64;
    o->inv_mass_factor = 1.0;
    o->n_levels = 3;
    o->orders[0] = 3; o->orders[1] = 2; o->orders[2] = 1;
    o->cheb_order = 4;
    o->eig_safety = 1.1;
    o->eig_ratio = 30.0;
    o->eig_iters = 20;
    o->coarse_iters = 20;
    o->check_every = 1;
    o->coarse_kind = 1;
    o->amg_coarse_max = 2048;
    o->amg_strength = 0.08;
    o->graphs = 2;
    o->assembled_max_order = -1;
    o->smoother = 1;
    o->amg_cheb_order = 2;
    o->amg_reuse_interpolation = 1;
    for (int l = 0; l < 4; ++l) {
      o->cheb_orders[l] = 0;
      o->pre_it[l] = 1;
      o->post_it[l] = 1;
    }
    (void)kind;
  });
}

int sipg_solver_create(sipg_op* op, int kind, const sipg_solver_opts* o, sipg_solver** out) {
  return guarded([&] {
    if (!op || !out || kind < 0 || kind > SIPG_SOLVER_PMULTIGRID) throw Error(SIPG_INVALID_ARG, "solver_create");
    auto s = std::make_unique<sipg_solver>();
    s->op = op;
    s->kind = kind;
    if (o) s->o = *o;
    else sipg_solver_default_opts(kind, &s->o);
    if (s->o.precision != SIPG_FP64 && s->o.precision != SIPG_FP32) throw Error(SIPG_INVALID_ARG, "precision");
    if (kind == SIPG_SOLVER_PMULTIGRID && s->o.n_levels >= 1) s->o.orders[0] = op->order;
    SIPG_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    SIPG_CUDA(cudaEventCreate(&s->ev0));
    SIPG_CUDA(cudaEventCreate(&s->ev1));
    *out = s.release();
  });
}

int sipg_solver_setup(sipg_solver* s) {
  return guarded([&] {
    if (!s) throw Error(SIPG_INVALID_ARG, "null solver");
    s->setup();
  });
}

int sipg_solver_solve(sipg_solver* s, const double* b, double* x, sipg_solve_info* info) {
  int st = SIPG_OK;
  int g = guarded([&] {
    if (!s || !b || !x) throw Error(SIPG_INVALID_ARG, "solve arguments");
    st = s->solve(b, x, info);
  });
  return g != SIPG_OK ? g : st;
}

int sipg_solver_solve_host(sipg_solver* s, const double* b, double* x, sipg_solve_info* info) {
  int st = SIPG_OK;
  int g = guarded([&] {
    if (!s || !b || !x) throw Error(SIPG_INVALID_ARG, "solve arguments");
    size_t bytes = (size_t)s->op->ncomp * s->op->mesh->K * s->op->Np * sizeof(double);
    if (!s->bw.p) { s->bw = DevBuf(bytes); s->xw = DevBuf(bytes); }
    SIPG_CUDA(cudaMemcpyAsync(s->bw.p, b, bytes, cudaMemcpyHostToDevice, s->stream));
    SIPG_CUDA(cudaMemcpyAsync(s->xw.p, x, bytes, cudaMemcpyHostToDevice, s->stream));
    st = s->solve(s->bw.as<double>(), s->xw.as<double>(), info);
    SIPG_CUDA(cudaMemcpyAsync(x, s->xw.p, bytes, cudaMemcpyDeviceToHost, s->stream));
    SIPG_CUDA(cudaStreamSynchronize(s->stream));
  });
  return g != SIPG_OK ? g : st;
}

void sipg_solver_destroy(sipg_solver* s) { delete s; }

int sipg_launch_count(unsigned long long* n) {
  return guarded([&] {
    if (!n) throw Error(SIPG_INVALID_ARG, "null pointer");
    *n = launch_count();
  });
}

int sipg_kernel_wait_timeouts(unsigned long long* n) {
  return guarded([&] {
    if (!n) throw Error(SIPG_INVALID_ARG, "null pointer");
    *n = tc5_timeouts();
  });
}

}  // extern "C"
