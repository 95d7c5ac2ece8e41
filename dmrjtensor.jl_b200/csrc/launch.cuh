// launch.cuh -- kernel launches with programmatic dependent launch (sm_90 and later).
//
// A bond step is two dozen short kernels in one stream, each depending on the one before. With
// an ordinary launch the next kernel is scheduled only after its predecessor has finished and
// its writes have been flushed, so every boundary costs a full launch latency on the device.
// Every kernel of this library therefore begins with grid_entry(): griddepcontrol.wait blocks
// until all kernels it depends on in the stream have COMPLETED and their memory operations are
// visible, then griddepcontrol.launch_dependents lets the next kernel in the stream be
// scheduled. Every launch goes through launch_k, which sets the programmatic-serialisation
// attribute, so the next kernel's launch and block set-up overlap the running kernel and its
// blocks start work the moment the running kernel completes.
//
// Ordering is unchanged: no thread touches global memory before its wait returns, so a kernel
// still sees every write of the kernels before it and never overwrites what they read. The
// trigger comes after the wait, so at most one kernel runs ahead in its set-up. A kernel whose
// predecessor in the stream is not a kernel (a copy, a memset, an event wait) is ordered after
// it as usual, and both instructions are no-ops in a kernel launched without the attribute.
#pragma once
#include <cuda_runtime.h>
#include <utility>

namespace dmrg {

__device__ __forceinline__ void grid_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// kernel<<<grid, block, smem, s>>>(args...) with programmatic stream serialisation allowed.
// Errors are left for the caller's cudaGetLastError().
template <typename... P, typename... A>
inline void launch_k(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                     A&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  (void)cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

}  // namespace dmrg
