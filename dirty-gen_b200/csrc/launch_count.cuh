// Count of this library's kernel launches issued from the calling thread, and
// the launch form of the step's kernels.
//
// silt_step reads the count before and after a step to report how many
// kernels the step launched (silt_step_parts.launches).
//
// Programmatic dependent launch: a kernel launched with launch_dep() (which,
// like <<<...>>>, leaves any launch error to cudaGetLastError) may be
// scheduled while the kernel before it on the stream is still finishing, so
// its launch latency hides behind that kernel's tail. Every kernel of the
// library calls dep_wait() before its first memory access; the wait returns
// once every kernel before it on the stream has completed and its writes are
// visible (and at once for an ordinary launch).
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace silt {

extern thread_local unsigned long long t_kernel_launches;

inline void count_launch() { ++t_kernel_launches; }

__device__ __forceinline__ void dep_wait() {
#if defined(__CUDA_ARCH__)
    asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

// Per-launch device timing (silt_set_kernel_timing, kernel_timer.cu): while
// it is on, every launch of the library is bracketed by two CUDA events on
// its own stream, and the elapsed time is booked to the kernel.
bool kernel_timing_on();
void kernel_timing_begin(cudaStream_t st);
void kernel_timing_end(cudaStream_t st, const void* kernel);

// cudaLaunchKernelEx with the optional timing around it.
template <typename... KArgs, typename... Args>
cudaError_t launch_ex(const cudaLaunchConfig_t& cfg, void (*kernel)(KArgs...), Args&&... args) {
    const bool timed = kernel_timing_on();
    if (timed) kernel_timing_begin(cfg.stream);
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
    if (timed) kernel_timing_end(cfg.stream, reinterpret_cast<const void*>(kernel));
    return e;
}

template <typename... KArgs, typename... Args>
cudaError_t launch_dep(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return launch_ex(cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace silt
