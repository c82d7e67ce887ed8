// Runtime objects and the C ABI of include/sipg_b200.h (mesh, operator, blocks).
// The solver entry points live in solver.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "../../include/sipg_b200.h"
#include "capi_util.hpp"
#include "bsr.cuh"
#include "runtime.hpp"
#include "sipg_blocks.cuh"
#include "vecops.cuh"

namespace sipg {

thread_local std::string g_last_error;

void set_last_error(const std::string& s) { g_last_error = s; }

void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  int st = e == cudaErrorMemoryAllocation ? SIPG_OUT_OF_MEMORY
           : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? SIPG_NO_DEVICE
                                                                           : SIPG_CUDA_ERROR;
  throw Error(st, std::string(what) + ": " + cudaGetErrorString(e));
}

DevBuf::DevBuf(size_t n) : bytes(n) {
  if (n) SIPG_CUDA(cudaMalloc(&p, n));
}
DevBuf::~DevBuf() {
  if (p) cudaFree(p);
}
DevBuf& DevBuf::operator=(DevBuf&& o) noexcept {
  if (this != &o) {
    if (p) cudaFree(p);
    p = o.p; bytes = o.bytes;
    o.p = nullptr; o.bytes = 0;
  }
  return *this;
}
void DevBuf::upload(const void* src, size_t n, cudaStream_t s) {
  if (n > bytes) throw Error(SIPG_INVALID_ARG, "upload larger than buffer");
  SIPG_CUDA(cudaMemcpyAsync(p, src, n, cudaMemcpyHostToDevice, s));
  SIPG_CUDA(cudaStreamSynchronize(s));
}

int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    SIPG_CUDA(cudaGetDevice(&dev));
    SIPG_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  }
  return n;
}

template <int DIM, int P>
static void pack_consts(const RefElement& r, std::vector<double>& c, std::vector<int8_t>& it) {
  using C = Cfg<DIM, P>;
  c.assign(C::CONST_T, 0.0);
  const double* D[3] = {r.Dr.data(), r.Ds.data(), r.Dt.data()};
  for (int d = 0; d < DIM; ++d)
    for (int i = 0; i < C::NP; ++i)
      for (int j = 0; j < C::NP; ++j) c[C::OFF_D + d * C::NP * C::LD + i * C::LD + j] = D[d][i * C::NP + j];
  for (int i = 0; i < C::NP; ++i)
    for (int j = 0; j < C::NP; ++j) c[C::OFF_M + i * C::LD + j] = r.M[i * C::NP + j];
  for (int i = 0; i < C::NP; ++i)
    for (int k = 0; k < C::NFNFP; ++k) c[C::OFF_E + i * C::LDE + k] = r.EMAT[i * C::NFNFP + k];
  it.assign(C::ITAB, 0);
  for (int k = 0; k < C::NF * C::NFP; ++k) it[k] = (int8_t)r.fmask[k];
  for (int k = 0; k < C::NPERM * C::NFP; ++k) it[C::NF * C::NFP + k] = (int8_t)r.perm_pos[k];
}

const DevRef& dev_ref(int dim, int order) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::map<int, std::unique_ptr<DevRef>>> cache;
  int dev = 0;
  SIPG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  auto& slot = cache[{dev, dim * 10 + order}];
  auto it = slot.find(0);
  if (it != slot.end()) return *it->second;
  auto d = std::make_unique<DevRef>();
  d->ref = build_ref_element(dim, order);
  d->Np = d->ref.Np;
  d->Nfp = d->ref.Nfp;
  std::vector<double> c;
  std::vector<int8_t> itab;
  switch (dim * 10 + order) {
    case 21: pack_consts<2, 1>(d->ref, c, itab); break;
    case 22: pack_consts<2, 2>(d->ref, c, itab); break;
    case 23: pack_consts<2, 3>(d->ref, c, itab); break;
    case 24: pack_consts<2, 4>(d->ref, c, itab); break;
    case 31: pack_consts<3, 1>(d->ref, c, itab); break;
    case 32: pack_consts<3, 2>(d->ref, c, itab); break;
    case 33: pack_consts<3, 3>(d->ref, c, itab); break;
    case 34: pack_consts<3, 4>(d->ref, c, itab); break;
    default: throw Error(SIPG_INVALID_ARG, "unsupported dim/order");
  }
  std::vector<float> c32(c.begin(), c.end());
  d->c64 = DevBuf(c.size() * sizeof(double));
  d->c64.upload(c.data(), c.size() * sizeof(double));
  d->c32 = DevBuf(c32.size() * sizeof(float));
  d->c32.upload(c32.data(), c32.size() * sizeof(float));
  d->itab = DevBuf(itab.size());
  d->itab.upload(itab.data(), itab.size());
  d->mf = DevBuf(d->ref.MF.size() * sizeof(double));
  d->mf.upload(d->ref.MF.data(), d->ref.MF.size() * sizeof(double));
  {
    // tensor-core blobs: FP64 as is, FP32 rounded to nearest TF32
    std::vector<double> t64, t32d;
    build_tc_consts<double>(dim, order, d->ref, t64);
    build_tc_consts<float>(dim, order, d->ref, t32d);
    std::vector<float> t32(t32d.size());
    for (size_t i = 0; i < t32d.size(); ++i) {
      float f = (float)t32d[i];
      uint32_t b;
      std::memcpy(&b, &f, 4);
      b = (b + 0x1000u) & ~0x1FFFu;
      std::memcpy(&t32[i], &b, 4);
    }
    d->tc64 = DevBuf(t64.size() * sizeof(double));
    d->tc64.upload(t64.data(), t64.size() * sizeof(double));
    d->tc32 = DevBuf(t32.size() * sizeof(float));
    d->tc32.upload(t32.data(), t32.size() * sizeof(float));
    d->tc_ok64 = tc_warps_for<double>(dim, order) >= 2;
    d->tc_ok32 = tc_warps_for<float>(dim, order) >= 2;
  }
  auto* raw = d.get();
  slot[0] = std::move(d);
  return *raw;
}

}  // namespace sipg

using namespace sipg;

const Mesh& sipg_mesh::host_order(int order) {
  std::lock_guard<std::mutex> lk(host_mu);
  auto it = host.find(order);
  if (it != host.end()) return it->second;
  RefElement ref = build_ref_element(dim, order);
  auto res = host.emplace(order, build_mesh(ref, Nv, vx.data(), K, e2v.data()));
  return res.first->second;
}

namespace {
// v rounded to the nearest BF16 value (ties to even), kept in an FP32 word
float bf16_round(float v) {
  uint32_t u;
  std::memcpy(&u, &v, sizeof(u));
  if ((u & 0x7f800000u) != 0x7f800000u) {  // finite
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
  }
  float r;
  std::memcpy(&r, &u, sizeof(r));
  return r;
}
}  // namespace

void sipg_mesh::ensure_device() {
  std::lock_guard<std::mutex> lk(dev_mu);
  if (device_ready) return;
  const Mesh& h = host_order(1);
  const int Nf = dim + 1, ng = h.ngeof();
  std::vector<float> g32(h.geof.begin(), h.geof.end());
  if (geom_bf16)
    for (float& v : g32) v = bf16_round(v);
  std::vector<uint32_t> code(K, 0);
  for (int e = 0; e < K; ++e)
    for (int f = 0; f < Nf; ++f) {
      size_t i = (size_t)e * Nf + f;
      uint32_t c = h.nbr[i] >= 0 ? (uint32_t)(h.nbr_face[i] | (h.nbr_perm[i] << 2)) : 0u;
      code[e] |= c << (8 * f);
    }
  std::vector<int> be;
  for (int e = 0; e < K; ++e)
    for (int f = 0; f < Nf; ++f)
      if (h.nbr[(size_t)e * Nf + f] < 0) { be.push_back(e); break; }
  geof64 = DevBuf((size_t)K * ng * sizeof(double));
  geof64.upload(h.geof.data(), (size_t)K * ng * sizeof(double));
  geof32 = DevBuf((size_t)K * ng * sizeof(float));
  geof32.upload(g32.data(), (size_t)K * ng * sizeof(float));
  nbr = DevBuf((size_t)K * Nf * sizeof(int));
  nbr.upload(h.nbr.data(), (size_t)K * Nf * sizeof(int));
  fcode = DevBuf((size_t)K * sizeof(uint32_t));
  fcode.upload(code.data(), (size_t)K * sizeof(uint32_t));
  n_belem = (int)be.size();
  belems = DevBuf(std::max<size_t>(1, be.size()) * sizeof(int));
  if (!be.empty()) belems.upload(be.data(), be.size() * sizeof(int));
  tcg64 = DevBuf(tc_geom_values<double>(dim, K) * sizeof(double));
  tcg32 = DevBuf(tc_geom_values<float>(dim, K) * sizeof(float));
  SIPG_CUDA(launch_tc_geom<double>(dim, geof64.as<double>(), K, tcg64.as<double>(), 0));
  SIPG_CUDA(launch_tc_geom<float>(dim, geof32.as<float>(), K, tcg32.as<float>(), 0));
  SIPG_CUDA(cudaDeviceSynchronize());
  if (geom_bf16) {  // the derived geometry blocks are stored at the same precision
    std::vector<float> t(tc_geom_values<float>(dim, K));
    SIPG_CUDA(cudaMemcpy(t.data(), tcg32.p, t.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (float& v : t) v = bf16_round(v);
    tcg32.upload(t.data(), t.size() * sizeof(float));
  }
  device_ready = true;
}

template <typename T>
void sipg_op::apply(const T* x, T* y, cudaStream_t s, T alpha, T beta, const T* c) const {
  constexpr bool f64 = std::is_same<T, double>::value;
  if (oi) {  // over-integrated factor: the assembled element blocks
    bsr_apply<T>(*oi_blocks, x, y, alpha, beta, s, c);
    return;
  }
  ApplyArgs<T> a;
  a.consts = f64 ? (const T*)dref->c64.p : (const T*)dref->c32.p;
  a.itab = dref->itab.as<int8_t>();
  a.geof = f64 ? (const T*)mesh->geof64.p : (const T*)mesh->geof32.p;
  a.nbr = mesh->nbr.as<int>();
  a.fcode = mesh->fcode.as<uint32_t>();
  a.tau = f64 ? (const T*)tau64.p : (const T*)tau32.p;
  a.factor = has_factor ? (f64 ? (const T*)factor64.p : (const T*)factor32.p) : nullptr;
  a.mm = mm_mode == MM_NODAL ? (f64 ? (const T*)mm64.p : (const T*)mm32.p) : nullptr;
  a.mm_scalar = (T)mm_scalar;
  a.mm_mode = mm_mode;
  a.bct = bct.as<uint8_t>();
  a.Kb = mesh->Kb;
  a.K = mesh->K;
  a.ncomp = ncomp;
  a.x = x;
  a.y = y;
  a.pin_elem = pin_elem;
  a.pin_node = pin_node;
  a.pin_scale = (T)pin_scale;
  a.eb = f64 ? eb64 : eb32;
  a.alpha = alpha;
  a.beta = beta;
  a.c = c ? c : y;
  a.tcg = f64 ? (const T*)mesh->tcg64.p : (const T*)mesh->tcg32.p;
  a.tcgen05 = kernel == 3;
  const bool tc_ok = (kernel == 0 || kernel >= 2) && (f64 ? dref->tc_ok64 : dref->tc_ok32);
  if (tc_ok && ncomp > 1 && pin_elem < 0) {
    // vector operator: one tensor-core scalar apply per component (its own boundary
    // types; slip faces get no face terms there), then the slip faces' coupling terms
    const T* tcc = f64 ? (const T*)dref->tc64.p : (const T*)dref->tc32.p;
    DevBuf& tr = f64 ? trace64 : trace32;
    if (!tr.p) tr = DevBuf(tc_trace_values(mesh->dim, order, mesh->K) * sizeof(T));
    const size_t per = (size_t)mesh->K * Np;
    for (int comp = 0; comp < ncomp; ++comp) {
      ApplyArgs<T> ac = a;
      ac.ncomp = 1;
      ac.x = x + comp * per;
      ac.y = y + comp * per;
      ac.c = a.c + comp * per;
      ac.bct = bct.as<uint8_t>() + (size_t)comp * mesh->Kb;
      SIPG_CUDA(launch_apply_tc<T>(mesh->dim, order, ac, tcc, tr.as<T>(), num_sms(), s));
    }
    SIPG_CUDA(launch_slip<T>(mesh->dim, order, a, mesh->belems.as<int>(), mesh->n_belem, s));
    return;
  }
  const bool tc = tc_ok && ncomp == 1;
  if (tc) {
    const T* tcc = f64 ? (const T*)dref->tc64.p : (const T*)dref->tc32.p;
    DevBuf& tr = f64 ? trace64 : trace32;
    if (!tr.p) tr = DevBuf(tc_trace_values(mesh->dim, order, mesh->K) * sizeof(T));
    SIPG_CUDA(launch_apply_tc<T>(mesh->dim, order, a, tcc, tr.as<T>(), num_sms(), s));
    return;
  }
  SIPG_CUDA(launch_apply<T>(mesh->dim, order, a, num_sms(), s));
}
template void sipg_op::apply<double>(const double*, double*, cudaStream_t, double, double, const double*) const;
template void sipg_op::apply<float>(const float*, float*, cudaStream_t, float, float, const float*) const;

void sipg_op::refresh_tau(cudaStream_t s) {
  const double* f = has_factor ? factor64.as<double>() : nullptr;
  SIPG_CUDA(launch_tau<double>(mesh->dim, order, dref->itab.as<int8_t>(), mesh->geof64.as<double>(),
                               mesh->nbr.as<int>(), mesh->fcode.as<uint32_t>(), f, mesh->K,
                               tau64.as<double>(), s));
  const float* f32 = has_factor ? factor32.as<float>() : nullptr;
  SIPG_CUDA(launch_tau<float>(mesh->dim, order, dref->itab.as<int8_t>(), mesh->geof32.as<float>(),
                              mesh->nbr.as<int>(), mesh->fcode.as<uint32_t>(), f32, mesh->K,
                              tau32.as<float>(), s));
}

BlockArgs sipg_op::block_args(int mode, int ref_volume, double* out, bool with_pin) const {
  BlockArgs a;
  a.consts = dref->c64.as<double>();
  a.itab = dref->itab.as<int8_t>();
  a.mf = dref->mf.as<double>();
  a.geof = mesh->geof64.as<double>();
  a.nbr = mesh->nbr.as<int>();
  a.tau = tau64.as<double>();
  a.factor = has_factor ? factor64.as<double>() : nullptr;
  a.mm_mode = mm_mode;
  a.mm_scalar = mm_scalar;
  a.mm = mm_mode == MM_NODAL ? mm64.as<double>() : nullptr;
  a.bct = bct.as<uint8_t>();
  a.Kb = mesh->Kb;
  a.K = mesh->K;
  a.ncomp = ncomp;
  a.ref_volume = ref_volume;
  a.pin_elem = with_pin ? pin_elem : -1;
  a.pin_node = pin_node;
  a.pin_scale = pin_scale;
  a.mode = mode;
  a.out = out;
  return a;
}

void sipg_op::refresh_pin(cudaStream_t s) {
  if (pin_elem < 0) return;
  // pin scale = the unpinned diagonal entry at the pinned DOF
  DevBuf d((size_t)ncomp * mesh->K * Np * sizeof(double));
  BlockArgs a = block_args(BLOCK_DIAG_ONLY, 0, d.as<double>(), false);
  SIPG_CUDA(launch_blocks(mesh->dim, order, a, s));
  double v = 0;
  SIPG_CUDA(cudaMemcpyAsync(&v, d.as<double>() + (size_t)pin_elem * Np + pin_node, sizeof(double),
                            cudaMemcpyDeviceToHost, s));
  SIPG_CUDA(cudaStreamSynchronize(s));
  pin_scale = v;
}

namespace sipg {
std::unique_ptr<sipg_op> create_op(sipg_mesh* m, int order, int ncomp) {
  if (order < 1 || order > kMaxOrder) throw Error(SIPG_INVALID_ARG, "order must be 1..4");
  if (ncomp != 1 && ncomp != m->dim) throw Error(SIPG_INVALID_ARG, "ncomp must be 1 or dim");
  m->ensure_device();
  auto op = std::make_unique<sipg_op>();
  op->mesh = m;
  op->order = order;
  op->ncomp = ncomp;
  op->dref = &dev_ref(m->dim, order);
  op->Np = op->dref->Np;
  op->Nfp = op->dref->Nfp;
  const int Nf = m->dim + 1;
  op->tau64 = DevBuf((size_t)m->K * Nf * sizeof(double));
  op->tau32 = DevBuf((size_t)m->K * Nf * sizeof(float));
  op->bct_host.assign((size_t)ncomp * m->Kb, SIPG_BC_DIRICHLET);
  op->bct = DevBuf(std::max<size_t>(1, op->bct_host.size()));
  std::vector<uint8_t> b(op->bct_host.size(), 0);
  if (!b.empty()) op->bct.upload(b.data(), b.size());
  op->eb64 = apply_pick_eb(m->dim, order, ncomp, true);
  op->eb32 = apply_pick_eb(m->dim, order, ncomp, false);
  op->refresh_tau(0);
  SIPG_CUDA(cudaDeviceSynchronize());
  return op;
}

// Device-side factor update (p-multigrid levels): f64 is K x Np FP64 on the device.
void set_factor_device(sipg_op* op, const double* f64, cudaStream_t s) {
  size_t n = (size_t)op->mesh->K * op->Np;
  if (!op->factor64.p) {
    op->factor64 = DevBuf(n * sizeof(double));
    op->factor32 = DevBuf(n * sizeof(float));
  }
  SIPG_CUDA(cudaMemcpyAsync(op->factor64.p, f64, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  to_f32(op->factor32.as<float>(), op->factor64.as<double>(), n, s);
  op->has_factor = true;
  op->refresh_tau(s);
}

void set_mm_device(sipg_op* op, int mode, double scalar, const double* mm64, cudaStream_t s) {
  op->mm_mode = mode;
  op->mm_scalar = scalar;
  if (mode == SIPG_MM_NODAL) {
    size_t n = (size_t)op->mesh->K * op->Np;
    if (!op->mm64.p) {
      op->mm64 = DevBuf(n * sizeof(double));
      op->mm32 = DevBuf(n * sizeof(float));
    }
    SIPG_CUDA(cudaMemcpyAsync(op->mm64.p, mm64, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    to_f32(op->mm32.as<float>(), op->mm64.as<double>(), n, s);
  }
}

void set_bc_types_host(sipg_op* op, const std::vector<int>& types) {
  size_t n = (size_t)op->ncomp * op->mesh->Kb;
  std::vector<uint8_t> b(n);
  for (size_t i = 0; i < n; ++i) {
    b[i] = (uint8_t)types[i];
    op->bct_host[i] = types[i];
  }
  if (n) op->bct.upload(b.data(), n);
}
}  // namespace sipg

// ------------------------------------------------------------------ C ABI
extern "C" {

const char* sipg_last_error(void) { return g_last_error.c_str(); }
int sipg_version(void) { return 100; }

int sipg_device_count(int* n) {
  return guarded([&] {
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) c = 0;
    *n = c;
  });
}
int sipg_dev_alloc(size_t bytes, void** ptr) {
  return guarded([&] { SIPG_CUDA(cudaMalloc(ptr, bytes)); });
}
int sipg_dev_free(void* ptr) {
  return guarded([&] { SIPG_CUDA(cudaFree(ptr)); });
}
int sipg_memcpy_h2d(void* dst, const void* src, size_t bytes) {
  return guarded([&] { SIPG_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice)); });
}
int sipg_memcpy_d2h(void* dst, const void* src, size_t bytes) {
  return guarded([&] { SIPG_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost)); });
}
int sipg_device_synchronize(void) {
  return guarded([&] { SIPG_CUDA(cudaDeviceSynchronize()); });
}

int sipg_ref_sizes(int dim, int order, int* Np, int* Nfp, int* Nfaces, int* Nperm) {
  return guarded([&] {
    if ((dim != 2 && dim != 3) || order < 1 || order > kMaxOrder) throw Error(SIPG_INVALID_ARG, "dim/order");
    if (Np) *Np = np_of(dim, order);
    if (Nfp) *Nfp = nfp_of(dim, order);
    if (Nfaces) *Nfaces = dim + 1;
    if (Nperm) *Nperm = dim == 2 ? 2 : 6;
  });
}

int sipg_ref_tables(int dim, int order, double* r, double* s, double* t, double* Dr, double* Ds,
                    double* Dt, double* M, double* MMF, double* EMAT, int* fmask, int* perm_pos) {
  return guarded([&] {
    RefElement e = build_ref_element(dim, order);
    auto cp = [](double* dst, const std::vector<double>& v) {
      if (dst) std::copy(v.begin(), v.end(), dst);
    };
    cp(r, e.r); cp(s, e.s); cp(t, e.t); cp(Dr, e.Dr); cp(Ds, e.Ds); cp(Dt, e.Dt); cp(M, e.M);
    cp(MMF, e.MMF); cp(EMAT, e.EMAT);
    if (fmask) std::copy(e.fmask.begin(), e.fmask.end(), fmask);
    if (perm_pos) std::copy(e.perm_pos.begin(), e.perm_pos.end(), perm_pos);
  });
}

int sipg_interp_matrix(int dim, int q, int p, double* P) {
  return guarded([&] {
    std::vector<double> m = interp_matrix(dim, q, p);
    std::copy(m.begin(), m.end(), P);
  });
}

int sipg_box_mesh_sizes(int dim, int n, int* Nv, int* K) {
  return guarded([&] {
    if ((dim != 2 && dim != 3) || n < 1) throw Error(SIPG_INVALID_ARG, "dim/n");
    if (dim == 2) { *Nv = (n + 1) * (n + 1); *K = 2 * n * n; }
    else { *Nv = (n + 1) * (n + 1) * (n + 1); *K = 6 * n * n * n; }
  });
}

int sipg_box_mesh(int dim, int n, double jitter, uint64_t seed, double* vx, int* e2v) {
  return guarded([&] {
    std::vector<double> v;
    std::vector<int> c;
    box_mesh(dim, n, jitter, seed, v, c);
    std::copy(v.begin(), v.end(), vx);
    std::copy(c.begin(), c.end(), e2v);
  });
}

int sipg_mesh_set_geometry_precision(sipg_mesh* m, int bits) {
  return guarded([&] {
    if (!m || (bits != 16 && bits != 32)) throw Error(SIPG_INVALID_ARG, "geometry precision: 16 or 32 bits");
    std::lock_guard<std::mutex> lk(m->dev_mu);
    if (m->device_ready) throw Error(SIPG_INVALID_ARG, "geometry precision: set it before the mesh's first device use");
    m->geom_bf16 = bits == 16;
  });
}

int sipg_mesh_create(int dim, int Nv, const double* vx, int K, const int* e2v, sipg_mesh** out) {
  return guarded([&] {
    if ((dim != 2 && dim != 3) || Nv <= 0 || K <= 0 || !vx || !e2v || !out)
      throw Error(SIPG_INVALID_ARG, "mesh_create arguments");
    auto m = std::make_unique<sipg_mesh>();
    m->dim = dim; m->Nv = Nv; m->K = K;
    m->vx.assign(vx, vx + (size_t)Nv * dim);
    m->e2v.assign(e2v, e2v + (size_t)K * (dim + 1));
    const Mesh& h = m->host_order(1);
    // host_order may have reoriented elements: keep that orientation for later orders
    m->e2v = h.e2v;
    m->Kb = h.nbfaces();
    m->F = h.nfaces_interior();
    *out = m.release();
  });
}

int sipg_mesh_sizes(const sipg_mesh* m, int* K, int* F, int* Kb) {
  return guarded([&] {
    if (!m) throw Error(SIPG_INVALID_ARG, "null mesh");
    if (K) *K = m->K;
    if (F) *F = m->F;
    if (Kb) *Kb = m->Kb;
  });
}

int sipg_mesh_export(const sipg_mesh* mc, int order, double* geof, double* nx, double* ny,
                     double* nz, double* sJ, double* fscale, int* face2cells, int* faceNum,
                     int* fmaskL, int* fmaskR, int* bface2cell, int* bfaceNum,
                     double* bface_centroid, double* x, double* y, double* z) {
  return guarded([&] {
    if (!mc) throw Error(SIPG_INVALID_ARG, "null mesh");
    sipg_mesh* m = const_cast<sipg_mesh*>(mc);
    const Mesh& h = m->host_order(order);
    auto cpd = [](double* d, const std::vector<double>& v) { if (d) std::copy(v.begin(), v.end(), d); };
    auto cpi = [](int* d, const std::vector<int>& v) { if (d) std::copy(v.begin(), v.end(), d); };
    cpd(geof, h.geof); cpd(nx, h.nx); cpd(ny, h.ny); cpd(nz, h.nz); cpd(sJ, h.sJ); cpd(fscale, h.fscale);
    cpi(face2cells, h.face2cells); cpi(faceNum, h.faceNum); cpi(fmaskL, h.fmaskL); cpi(fmaskR, h.fmaskR);
    cpi(bface2cell, h.bface2cell); cpi(bfaceNum, h.bfaceNum); cpd(bface_centroid, h.bface_centroid);
    cpd(x, h.x); cpd(y, h.y); cpd(z, h.z);
  });
}

int sipg_mesh_device_bytes(const sipg_mesh* m, size_t* bytes) {
  return guarded([&] {
    *bytes = m->geof64.bytes + m->geof32.bytes + m->nbr.bytes + m->fcode.bytes + m->belems.bytes +
             m->tcg64.bytes + m->tcg32.bytes + m->proj_h.bytes + m->proj_io.bytes;
  });
}

void sipg_mesh_destroy(sipg_mesh* m) { delete m; }

int sipg_op_create(sipg_mesh* m, int order, int ncomp, sipg_op** out) {
  return guarded([&] {
    if (!m || !out) throw Error(SIPG_INVALID_ARG, "null argument");
    *out = sipg::create_op(m, order, ncomp).release();
  });
}

int sipg_op_set_factor(sipg_op* op, const double* factor) {
  return guarded([&] {
    if (!op) throw Error(SIPG_INVALID_ARG, "null op");
    ++op->version;
    op->oi = false;  // a nodal factor replaces a cubature-point one
    size_t n = (size_t)op->mesh->K * op->Np;
    if (!factor) {
      op->has_factor = false;
    } else {
      if (!op->factor64.p) {
        op->factor64 = DevBuf(n * sizeof(double));
        op->factor32 = DevBuf(n * sizeof(float));
      }
      std::vector<float> f32(factor, factor + n);
      op->factor64.upload(factor, n * sizeof(double));
      op->factor32.upload(f32.data(), n * sizeof(float));
      op->has_factor = true;
    }
    op->refresh_tau(0);
    op->refresh_pin(0);
    SIPG_CUDA(cudaDeviceSynchronize());
  });
}

int sipg_op_set_mm(sipg_op* op, int mode, double scalar, const double* mm) {
  return guarded([&] {
    if (!op || mode < 0 || mode > 2 || (mode == SIPG_MM_NODAL && !mm)) throw Error(SIPG_INVALID_ARG, "set_mm");
    ++op->version;
    op->mm_mode = mode;
    op->mm_scalar = scalar;
    if (mode == SIPG_MM_NODAL) {
      size_t n = (size_t)op->mesh->K * op->Np;
      if (!op->mm64.p) {
        op->mm64 = DevBuf(n * sizeof(double));
        op->mm32 = DevBuf(n * sizeof(float));
      }
      std::vector<float> m32(mm, mm + n);
      op->mm64.upload(mm, n * sizeof(double));
      op->mm32.upload(m32.data(), n * sizeof(float));
    }
    op->refresh_pin(0);
    if (op->oi) {
      oi_assemble(op, 0);
      SIPG_CUDA(cudaDeviceSynchronize());
    }
  });
}

int sipg_op_set_bc_types(sipg_op* op, const int* types) {
  return guarded([&] {
    if (!op || (!types && op->mesh->Kb)) throw Error(SIPG_INVALID_ARG, "set_bc_types");
    ++op->version;
    size_t n = (size_t)op->ncomp * op->mesh->Kb;
    std::vector<uint8_t> b(n);
    for (size_t i = 0; i < n; ++i) {
      if (types[i] < 0 || types[i] > 2) throw Error(SIPG_INVALID_ARG, "bc type must be 0, 1 or 2");
      b[i] = (uint8_t)types[i];
      op->bct_host[i] = types[i];
    }
    if (n) op->bct.upload(b.data(), n);
    op->refresh_pin(0);
    if (op->oi) {
      oi_assemble(op, 0);
      SIPG_CUDA(cudaDeviceSynchronize());
    }
  });
}

int sipg_op_set_pin(sipg_op* op, int elem, int node) {
  return guarded([&] {
    if (!op) throw Error(SIPG_INVALID_ARG, "null op");
    ++op->version;
    if (elem < 0) {
      op->pin_elem = -1;
      op->pin_node = -1;
    } else {
      if (elem >= op->mesh->K || node < 0 || node >= op->Np) throw Error(SIPG_INVALID_ARG, "pin out of range");
      op->pin_elem = elem;
      op->pin_node = node;
      op->refresh_pin(0);
    }
    if (op->oi) {
      oi_assemble(op, 0);
      SIPG_CUDA(cudaDeviceSynchronize());
    }
  });
}

int sipg_op_apply(sipg_op* op, int precision, const void* x, void* y, void* stream) {
  return guarded([&] {
    if (!op || !x || !y) throw Error(SIPG_INVALID_ARG, "apply arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (precision == SIPG_FP64) op->apply<double>((const double*)x, (double*)y, s);
    else if (precision == SIPG_FP32) op->apply<float>((const float*)x, (float*)y, s);
    else throw Error(SIPG_INVALID_ARG, "precision must be 64 or 32");
  });
}

int sipg_op_set_kernel(sipg_op* op, int kind) {
  return guarded([&] {
    if (!op || kind < 0 || kind > 3) throw Error(SIPG_INVALID_ARG, "set_kernel");
    ++op->version;
    op->kernel = kind;
  });
}

int sipg_op_apply_host(sipg_op* op, const double* x, double* y) {
  return guarded([&] {
    if (!op || !x || !y) throw Error(SIPG_INVALID_ARG, "apply arguments");
    size_t n = (size_t)op->ncomp * op->mesh->K * op->Np * sizeof(double);
    DevBuf dx(n), dy(n);
    SIPG_CUDA(cudaMemcpy(dx.p, x, n, cudaMemcpyHostToDevice));
    op->apply<double>(dx.as<double>(), dy.as<double>(), 0);
    SIPG_CUDA(cudaMemcpy(y, dy.p, n, cudaMemcpyDeviceToHost));
  });
}

int sipg_op_apply_bc_host(sipg_op* op, const double* bc, double* rhs) {
  return guarded([&] {
    if (!op || !bc || !rhs) throw Error(SIPG_INVALID_ARG, "apply_bc arguments");
    sipg_mesh* m = op->mesh;
    size_t nb = (size_t)op->ncomp * m->Kb * op->Nfp * sizeof(double);
    size_t nr = (size_t)op->ncomp * m->K * op->Np * sizeof(double);
    DevBuf dbc(std::max<size_t>(nb, 8)), drhs(nr);
    if (nb) SIPG_CUDA(cudaMemcpy(dbc.p, bc, nb, cudaMemcpyHostToDevice));
    SIPG_CUDA(cudaMemcpy(drhs.p, rhs, nr, cudaMemcpyHostToDevice));
    op->apply_bc_device(dbc.as<double>(), drhs.as<double>(), 0);
    SIPG_CUDA(cudaMemcpy(rhs, drhs.p, nr, cudaMemcpyDeviceToHost));
  });
}

int sipg_op_diag_host(sipg_op* op, double* diag) {
  return guarded([&] {
    if (!op || !diag) throw Error(SIPG_INVALID_ARG, "diag arguments");
    size_t n = (size_t)op->ncomp * op->mesh->K * op->Np;
    DevBuf d(n * sizeof(double));
    SIPG_CUDA(launch_blocks(op->mesh->dim, op->order, op->block_args(BLOCK_DIAG_ONLY, 0, d.as<double>(), true), 0));
    SIPG_CUDA(cudaMemcpy(diag, d.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  });
}

int sipg_op_block_diag_host(sipg_op* op, int invert, int ref_volume_block, double* blocks) {
  return guarded([&] {
    if (!op || !blocks) throw Error(SIPG_INVALID_ARG, "block_diag arguments");
    size_t n = (size_t)op->ncomp * op->mesh->K * op->Np * op->Np;
    DevBuf d(n * sizeof(double));
    SIPG_CUDA(launch_blocks(op->mesh->dim, op->order,
                            op->block_args(invert ? BLOCK_INVERSE : BLOCK_FULL, ref_volume_block, d.as<double>(), true), 0));
    SIPG_CUDA(cudaMemcpy(blocks, d.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  });
}

int sipg_op_sizes(const sipg_op* op, int* K, int* Np, int* Nfp, int* ncomp) {
  return guarded([&] {
    if (!op) throw Error(SIPG_INVALID_ARG, "null op");
    if (K) *K = op->mesh->K;
    if (Np) *Np = op->Np;
    if (Nfp) *Nfp = op->Nfp;
    if (ncomp) *ncomp = op->ncomp;
  });
}

void sipg_op_destroy(sipg_op* op) { delete op; }

}  // extern "C"

void sipg_op::apply_bc_device(const double* bc, double* rhs, cudaStream_t s) const {
  ApplyBcArgs a;
  a.consts = dref->c64.as<double>();
  a.itab = dref->itab.as<int8_t>();
  a.mf = dref->mf.as<double>();
  a.geof = mesh->geof64.as<double>();
  a.nbr = mesh->nbr.as<int>();
  a.tau = tau64.as<double>();
  a.factor = has_factor ? factor64.as<double>() : nullptr;
  a.bct = bct.as<uint8_t>();
  a.Kb = mesh->Kb;
  a.K = mesh->K;
  a.ncomp = ncomp;
  a.belems = mesh->belems.as<int>();
  a.n_belem = mesh->n_belem;
  a.bc = bc;
  a.rhs = rhs;
  SIPG_CUDA(launch_apply_bc(mesh->dim, order, a, s));
}
