// Internal runtime objects behind the C ABI (include/sipg_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "amg.hpp"
#include "mesh.hpp"
#include "refelem.hpp"
#include "sipg_apply.cuh"
#include "sipg_apply_tc.cuh"
#include "sipg_blocks.cuh"

namespace sipg {

// Error carried up to the C ABI as (status, message).
struct Error : std::runtime_error {
  int status;
  Error(int st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};

void cuda_check(cudaError_t e, const char* what);
#define SIPG_CUDA(call) ::sipg::cuda_check((call), #call)

// Device allocation owned by a runtime object.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  explicit DevBuf(size_t n);
  ~DevBuf();
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept;
  template <typename T> T* as() const { return static_cast<T*>(p); }
  void upload(const void* src, size_t n, cudaStream_t s = 0);
};

// Keep b at exactly n bytes, reallocating only when the size changes (set-up
// buffers are rebuilt at every time step: no allocation, no implicit
// synchronisation of cudaFree when the mesh stays the same).
inline void ensure(DevBuf& b, size_t n) {
  if (b.bytes != n) b = DevBuf(n);
}

// Order-specific reference tables on the device (FP64 and FP32 copies).
struct DevRef {
  RefElement ref;
  DevBuf c64, c32, itab, mf;
  DevBuf tc64, tc32;   // tensor-core constant blobs (A1 | A2)
  bool tc_ok64 = false, tc_ok32 = false;
  int Np = 0, Nfp = 0;
};
const DevRef& dev_ref(int dim, int order);  // cached per device

int num_sms();

}  // namespace sipg

struct sipg_mesh {
  int dim = 0, K = 0, Kb = 0, F = 0, Nv = 0;
  std::vector<double> vx;
  std::vector<int> e2v;
  std::map<int, sipg::Mesh> host;  // per-order host tables (lazily built)
  std::mutex host_mu;
  sipg::DevBuf geof64, geof32, nbr, fcode, belems;
  sipg::DevBuf tcg64, tcg32;  // geometry blocks of the tensor-core apply (launch_tc_geom)
  std::shared_ptr<sipg::P1Plan> p1_plan;  // algebraic coarse space: sparsity of the P1 operator (set-up cache)
  std::shared_ptr<void> p1_gather;        // its assembly from element blocks as device term lists (set-up cache)
  std::mutex probe_mu;         // guards the set-up caches above
  sipg::DevBuf proj_h;        // velocity projection: 1 / max interior-face fscale per element
  sipg::DevBuf proj_io;       // velocity projection: device copies for the host-buffer entry point
  std::mutex proj_mu;         // serialises host-buffer projections on this mesh
  int n_belem = 0;
  bool geom_bf16 = false;  // FP32 geometric data rounded to BF16 (sipg_mesh_set_geometry_precision)
  bool device_ready = false;
  std::mutex dev_mu;
  const sipg::Mesh& host_order(int order);
  void ensure_device();  // upload geometry/connectivity on first device use
};

namespace sipg {
struct BsrOp;
}

struct sipg_op {
  sipg_mesh* mesh = nullptr;
  int order = 0, ncomp = 1, Np = 0, Nfp = 0;
  const sipg::DevRef* dref = nullptr;
  bool has_factor = false;
  sipg::DevBuf factor64, factor32, tau64, tau32;
  int mm_mode = 0;
  double mm_scalar = 0.0;
  sipg::DevBuf mm64, mm32;
  sipg::DevBuf bct;           // ncomp x Kb uint8
  std::vector<int> bct_host;  // ncomp x Kb
  int pin_elem = -1, pin_node = -1;
  double pin_scale = 1.0;
  int eb64 = 0, eb32 = 0;
  int kernel = 0;  // 0: tensor cores where available, 1: CUDA cores
  unsigned version = 0;  // bumped by every setter: solvers re-capture their graphs
  mutable sipg::DevBuf trace64, trace32;  // face traces of the two-pass tensor-core apply
  // over-integrated factor (sipg_op_set_factor_oi): the factor at the volume and
  // surface cubature points, and the element blocks the operator then applies;
  // factor64 holds its nodal projection (the p-multigrid levels' factor)
  bool oi = false;
  sipg::DevBuf oi_fvol, oi_fsurf;
  std::shared_ptr<sipg::BsrOp> oi_blocks;
  // Apply on device buffers in precision T.
  template <typename T>
  // y = alpha A x + beta c, c = y when null (beta == 0: c is not read)
  void apply(const T* x, T* y, cudaStream_t s, T alpha = T(1), T beta = T(0), const T* c = nullptr) const;
  void refresh_tau(cudaStream_t s);
  sipg::BlockArgs block_args(int mode, int ref_volume, double* out, bool with_pin) const;
  void apply_bc_device(const double* bc, double* rhs, cudaStream_t s) const;
  void refresh_pin(cudaStream_t s);
};

namespace sipg {
std::unique_ptr<sipg_op> create_op(sipg_mesh* m, int order, int ncomp);
void set_factor_device(sipg_op* op, const double* f64, cudaStream_t s);
void set_mm_device(sipg_op* op, int mode, double scalar, const double* mm64, cudaStream_t s);
void set_bc_types_host(sipg_op* op, const std::vector<int>& types);
// Over-integrated factor (oi.cu): copy the cubature-point factor (K x nq and
// K x Nf x nqs, host or device pointers), then assemble; oi_assemble again from
// the stored factor after the boundary types, mass term or pinned DOF change.
void set_factor_oi_device(sipg_op* op, const double* fvol, const double* fsurf, cudaStream_t s);
void oi_assemble(sipg_op* op, cudaStream_t s);
// The two-phase pressure factor 1/rho(s) at the cubature points straight from the
// level set s (K x Np, device), rho = the smoothed Heaviside of ls_step; then assemble.
void set_factor_oi_level_set(sipg_op* op, const double* s, double alpha, double rho0, double rho1, cudaStream_t st);
}  // namespace sipg
