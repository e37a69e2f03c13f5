// Count of this library's kernel launches issued from the calling thread.
// silt_step reads it before and after a step to report how many kernels the
// step launched (silt_step_parts.launches).
#pragma once

namespace silt {

extern thread_local unsigned long long t_kernel_launches;

inline void count_launch() { ++t_kernel_launches; }

}  // namespace silt
