// Tensor-core SIPG apply launchers (sipg_apply_tc.cu).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "refelem.hpp"
#include "sipg_apply.cuh"

namespace sipg {

// Scalar operator (ncomp == 1) on the tensor cores: T = float runs TF32 MMAs
// with FP32 accumulation, T = double runs FP64 MMAs. tc_consts: device blob of
// build_tc_consts<T> converted to T.
// trace: scratch of tc_trace_values(dim, order, K) values (face traces between
// the two passes); applies sharing one trace buffer must be stream-ordered.
template <typename T>
cudaError_t launch_apply_tc(int dim, int order, const ApplyArgs<T>& a, const T* tc_consts, T* trace,
                            int num_sms, cudaStream_t s);
size_t tc_trace_values(int dim, int order, int K);
template <typename T>
void build_tc_consts(int dim, int order, const RefElement& r, std::vector<double>& out);
// Warps per CTA of the apply pass (below 2: use the CUDA-core kernel).
template <typename T>
int tc_warps_for(int dim, int order);
// Element and face geometry of the tensor-core apply (ApplyArgs::tcg), computed
// once per mesh from the K x NG geometric factors: tc_geom_values<T>(dim, K)
// values, one block per warp tile of elements (zero past K).
template <typename T>
size_t tc_geom_values(int dim, int K);
template <typename T>
cudaError_t launch_tc_geom(int dim, const T* geof, int K, T* out, cudaStream_t s);

// tcgen05 kernels of the FP32 scalar apply (apply_tc5.cu): their constants follow
// the mma.sync blob of build_tc_consts<float> (appended by it), the face traces
// use the same scratch layout (tc_trace_values).
bool tc5_supported(int dim, int order);
size_t tc5_const_values(int dim, int order);
void build_tc5_consts(int dim, int order, const RefElement& r, std::vector<double>& out);
cudaError_t launch_apply_tc5(int dim, int order, const ApplyArgs<float>& a, const float* blob, float* trace,
                             int num_sms, cudaStream_t s);
// MMA waits of the tcgen05 kernels that ran out (0 unless something hung).
unsigned tc5_timeouts();

}  // namespace sipg
