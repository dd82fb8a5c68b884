/* cb_launch.cuh -- programmatic dependent launch for the step kernels.
 *
 * Consecutive steps of a run are consecutive kernels on the run's stream. A
 * step kernel is launched with programmatic stream serialisation: once every
 * block of the previous step has finished its sites (and said so with
 * griddepcontrol.launch_dependents), the next step may be scheduled -- its
 * blocks take the slots the finished blocks leave -- and it waits, in
 * hardware, for the previous grid to complete and its memory to be visible
 * (griddepcontrol.wait) before it reads anything that grid wrote. The launch
 * latency of a step so overlaps the tail of the one before, and waiting blocks
 * never hold slots that other streams' kernels could use for long. Without
 * the launch attribute both instructions do nothing.
 */
#ifndef CB_LAUNCH_CUH
#define CB_LAUNCH_CUH

#include <cuda_runtime.h>

#include <utility>

namespace cb {

/* wait for the preceding grid on the stream (all its memory operations done) */
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

/* let the next kernel on the stream be scheduled */
__device__ __forceinline__ void pdl_allow_next() { asm volatile("griddepcontrol.launch_dependents;" :::); }

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace cb

#endif
