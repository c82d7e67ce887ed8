// Programmatic dependent launch: a kernel of the solve loop may start (launch,
// prologue, constant loads) while the previous kernel on its stream finishes;
// it waits for that kernel's completion before touching data it produces.
// Every kernel launched with pdl_launch calls pdl_wait before its first read of
// data written by earlier kernels and before its first global write.
#pragma once
#include <cuda_runtime.h>

#include <utility>

namespace sipg {

// Wait until the preceding kernel of the stream has completed and its writes are visible
// (a no-op for kernels launched without the attribute).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
// Allow the next kernel of the stream to be scheduled once every block of this one has started.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_enter() {
  pdl_trigger();
  pdl_wait();
}

template <typename... KArgs, typename... Args>
inline cudaError_t pdl_launch(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

}  // namespace sipg
