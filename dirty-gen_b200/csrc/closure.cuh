// Device entry points of the learned flux closure (closure_mma.cu,
// closure_step.cu) for the runtime.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace silt {
namespace closure {

const char* last_error();
int fail(int rc, const char* what);

cudaError_t conv3x3(const uint16_t* x, const uint16_t* w, const float* bias, const uint16_t* gate, uint16_t* y,
                    float* y32, int n_img, int h, int wd, int cin, int cout, int relu, cudaStream_t st);
cudaError_t conv3x3_wgrad(const uint16_t* x, const uint16_t* dy, float* dw, float* db, int n_img, int h, int wd,
                          int cin, int cout, cudaStream_t st);
// Copies the kernels' sticky timeout flag to *flag (host) after the stream's work.
int device_error(cudaStream_t st, int* flag);

}  // namespace closure
}  // namespace silt
