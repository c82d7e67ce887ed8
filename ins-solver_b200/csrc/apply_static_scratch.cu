// Allocation-free operator apply: sipg_op_apply_static_scratch.
//
// sipg_op_apply runs the scalar tensor-core apply in two passes that hand face
// traces to each other through a scratch buffer, and it takes that buffer from
// cudaMalloc the first time an operator is applied in a precision. Some callers
// cannot make that allocation when they apply:
//  * a time-step loop whose memory is already handed out to another allocator
//    (the reference keeps its fields in OP2 dats and its temporaries in a dat
//    pool, and PETSc holds its own pools), so a late cudaMalloc can fail with
//    out-of-memory in the middle of a run;
//  * host code that must not stall other streams: cudaMalloc and cudaFree may
//    synchronise the device.
// This entry point runs the same two kernels with the trace scratch in a
// fixed-size array compiled into the library as a __device__ variable, so the
// call allocates nothing. Its price is a fixed kScratchBytes of device memory
// per device (reserved when the library's module is loaded in a context: at the
// first use of its kernels under lazy module loading, the CUDA default, or at
// context creation under CUDA_MODULE_LOADING=EAGER), and one scratch per device: two
// calls that overlap in time on the same device (different streams, different
// host threads without ordering) race on it and give wrong results.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <string>

#include "../../include/sipg_b200.h"
#include "capi_util.hpp"
#include "runtime.hpp"

namespace sipg {
namespace {

// 64 MiB holds the face traces of K * Nf * 2 * Nfp values: at p = 3 in 3D that is
// 209,715 tetrahedra in FP32 and 104,857 in FP64.
constexpr size_t kScratchBytes = SIPG_STATIC_SCRATCH_BYTES;
static_assert(kScratchBytes % 256 == 0, "scratch size must keep 256-byte alignment");

// Nothing in the scratch must start at zero: the first pass writes every trace
// entry of every element before the second pass reads any of them.
__device__ __align__(256) unsigned char g_trace_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::atomic<void*> g_scratch_ptr[kMaxDevices];
std::mutex g_setup_mu;

// Device address of the scratch on the current device, looked up once per device.
void* scratch_on_current_device() {
  int dev = 0;
  SIPG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw Error(SIPG_INVALID_ARG, "device ordinal beyond the static scratch table");
  void* p = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (p) return p;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  p = g_scratch_ptr[dev].load(std::memory_order_relaxed);
  if (!p) {
    cudaError_t e = cudaGetSymbolAddress(&p, g_trace_scratch);
    if (e != cudaSuccess || !p)
      throw Error(SIPG_CUDA_ERROR, std::string("static scratch set-up (cudaGetSymbolAddress): ") +
                                       cudaGetErrorString(e));
    g_scratch_ptr[dev].store(p, std::memory_order_release);
  }
  return p;
}

template <typename T>
ApplyArgs<T> args_of(const sipg_op* op, const T* x, T* y) {
  constexpr bool f64 = std::is_same<T, double>::value;
  ApplyArgs<T> a;
  a.consts = f64 ? (const T*)op->dref->c64.p : (const T*)op->dref->c32.p;
  a.itab = op->dref->itab.as<int8_t>();
  a.geof = f64 ? (const T*)op->mesh->geof64.p : (const T*)op->mesh->geof32.p;
  a.nbr = op->mesh->nbr.as<int>();
  a.fcode = op->mesh->fcode.as<uint32_t>();
  a.tau = f64 ? (const T*)op->tau64.p : (const T*)op->tau32.p;
  a.factor = op->has_factor ? (f64 ? (const T*)op->factor64.p : (const T*)op->factor32.p) : nullptr;
  a.mm = op->mm_mode == SIPG_MM_NODAL ? (f64 ? (const T*)op->mm64.p : (const T*)op->mm32.p) : nullptr;
  a.mm_scalar = (T)op->mm_scalar;
  a.mm_mode = op->mm_mode;
  a.bct = op->bct.as<uint8_t>();
  a.Kb = op->mesh->Kb;
  a.K = op->mesh->K;
  a.ncomp = op->ncomp;
  a.x = x;
  a.y = y;
  a.pin_elem = op->pin_elem;
  a.pin_node = op->pin_node;
  a.pin_scale = (T)op->pin_scale;
  a.eb = f64 ? op->eb64 : op->eb32;
  a.alpha = T(1);
  a.beta = T(0);
  a.c = y;
  a.tcg = f64 ? (const T*)op->mesh->tcg64.p : (const T*)op->mesh->tcg32.p;
  a.tcgen05 = op->kernel == 3;
  return a;
}

// Same kernel choice as sipg_op::apply; only the origin of the trace scratch differs.
template <typename T>
void apply_static(const sipg_op* op, const T* x, T* y, cudaStream_t s) {
  constexpr bool f64 = std::is_same<T, double>::value;
  const ApplyArgs<T> a = args_of<T>(op, x, y);
  const bool tc = (op->kernel == 0 || op->kernel >= 2) && op->ncomp == 1 &&
                  (f64 ? op->dref->tc_ok64 : op->dref->tc_ok32);
  if (!tc) {  // the single-pass kernels need no scratch
    SIPG_CUDA(launch_apply<T>(op->mesh->dim, op->order, a, num_sms(), s));
    return;
  }
  const size_t need = tc_trace_values(op->mesh->dim, op->order, op->mesh->K) * sizeof(T);
  if (need > kScratchBytes)
    throw Error(SIPG_INVALID_ARG, "sipg_op_apply_static_scratch: this operator needs " + std::to_string(need) +
                                      " bytes of trace scratch (K = " + std::to_string(op->mesh->K) +
                                      ", order " + std::to_string(op->order) + ") but the static scratch holds " +
                                      std::to_string(kScratchBytes) + "; use sipg_op_apply");
  T* trace = static_cast<T*>(scratch_on_current_device());
  const T* tcc = f64 ? (const T*)op->dref->tc64.p : (const T*)op->dref->tc32.p;
  SIPG_CUDA(launch_apply_tc<T>(op->mesh->dim, op->order, a, tcc, trace, num_sms(), s));
}

}  // namespace
}  // namespace sipg

using namespace sipg;

extern "C" int sipg_op_apply_static_scratch(sipg_op* op, int precision, const void* x, void* y, void* stream) {
  return guarded([&] {
    if (!op || !x || !y) throw Error(SIPG_INVALID_ARG, "apply arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (op->oi) {  // the over-integrated operator's block-sparse apply needs no scratch
      if (precision == SIPG_FP64) op->apply<double>((const double*)x, (double*)y, s);
      else if (precision == SIPG_FP32) op->apply<float>((const float*)x, (float*)y, s);
      else throw Error(SIPG_INVALID_ARG, "precision must be 64 or 32");
      return;
    }
    if (precision == SIPG_FP64) apply_static<double>(op, (const double*)x, (double*)y, s);
    else if (precision == SIPG_FP32) apply_static<float>(op, (const float*)x, (float*)y, s);
    else throw Error(SIPG_INVALID_ARG, "precision must be 64 or 32");
  });
}
