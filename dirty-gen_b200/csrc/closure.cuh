// The learned flux closure (closure_mma.cu: tensor-core kernels; closure_step.cu:
// the closure inside the step) as the runtime sees it.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/silt_closure.h"
#include "sheet_fine.cuh"

namespace silt {
namespace closure {

extern thread_local char g_err[200];
const char* last_error();
int fail(int rc, const char* what);

cudaError_t conv3x3(const uint16_t* x, const uint16_t* w, const float* bias, const uint16_t* gate, uint16_t* y,
                    float* y32, int n_img, int h, int wd, int cin, int cout, int relu, cudaStream_t st);
cudaError_t conv3x3_wgrad(const uint16_t* x, const uint16_t* dy, float* dw, float* db, int n_img, int h, int wd,
                          int cin, int cout, cudaStream_t st);
// Copies the kernels' sticky timeout flag to *flag (host) after the stream's work.
int device_error(cudaStream_t st, int* flag);

constexpr int MAX_CROP_TIRES = 8;

// The network on the device: packed forward weights, biases, normalisation.
struct Net {
    const uint16_t* w[3] = {nullptr, nullptr, nullptr};
    const float* b[3] = {nullptr, nullptr, nullptr};
    const float* norm = nullptr;
};

// One crop's input gather: the window, the crop's first cell, its tires.
struct FeatureJob {
    fine::SheetView W;
    int ci0, cj0;
    int ntires;
    silt_tire_push tires[MAX_CROP_TIRES];
};

// One crop's correction.
struct ApplyJob {
    fine::SheetView W;
    int ci0, cj0;
    float* resid;   // [clipped, predicted] transfer sums of the crop
    double* moved;  // FP64 volume moved across faces, m^3 (accumulated)
};

cudaError_t launch_features(const FeatureJob* d_jobs, int n, const float* d_norm, uint16_t* x, cudaStream_t st);
cudaError_t launch_apply(const ApplyJob* d_jobs, int n, const float* y, const float* d_norm, cudaStream_t st);

// Per-step records through pinned memory: a ring of slots, each reused only
// after its last copy has left it.
struct Staging {
    static constexpr int SLOTS = 4;  // a slot is reused four puts later: its copy is long done
    void* dev[SLOTS] = {};
    void* host[SLOTS] = {};
    cudaEvent_t ev[SLOTS] = {};
    size_t cap[SLOTS] = {};
    int flip = 0;
    cudaError_t put(const void* data, size_t bytes, cudaStream_t st, void** out);
    void release();
};

// Buffers and records of the closure over up to `cap` crops per step. The
// residual estimates of each correction come back through a ring of pinned
// slots, so the host reads the newest finished one without waiting and the
// GPU may run up to RING corrections ahead of it.
struct Runner {
    static constexpr int RING = 4;
    int cap = 0;
    uint16_t* x = nullptr;   // crops x 32 x 32 x 16 BF16 input
    uint16_t* a1 = nullptr;  // hidden activations
    uint16_t* a2 = nullptr;
    float* y = nullptr;      // crops x 32 x 32 x 16 FP32 output
    float* d_resid = nullptr;
    double* d_moved = nullptr;
    float* h_resid[RING] = {nullptr, nullptr, nullptr, nullptr};   // pinned, 2 floats per crop
    double* h_moved[RING] = {nullptr, nullptr, nullptr, nullptr};  // pinned
    cudaEvent_t ev[RING] = {nullptr, nullptr, nullptr, nullptr};
    int crops[RING] = {0, 0, 0, 0};
    std::vector<int> tag[RING];
    unsigned long long written = 0, read = 0;  // corrections issued / consumed
    Staging fjobs, ajobs;

    cudaError_t reserve(int n);
    // Gathers every job's crop into x (before the coarse step).
    cudaError_t features(const std::vector<FeatureJob>& jobs, const Net& net, cudaStream_t st);
    // Runs the network on the gathered crops and applies the corrections
    // (after the coarse step); the jobs' resid and moved pointers are set
    // here. `tag` (e.g. the crops' windows) comes back with the estimates.
    cudaError_t correct(std::vector<ApplyJob>& jobs, const Net& net, cudaStream_t st,
                        const std::vector<int>& tag = std::vector<int>());
    // The residual estimates (clipped / predicted transfer) of the newest
    // finished correction not read yet, with its tag and the FP64 volume
    // moved so far; false if none has finished.
    bool poll(std::vector<float>& resid, double* moved_m3, std::vector<int>* tag = nullptr);
    void release();
};

void crop_origin(const std::vector<silt_tire_push>& ps, float ox, float oz, float cell, int* ci0, int* cj0);

}  // namespace closure
}  // namespace silt

struct silt_closure {
    int device = 0;
    float* params = nullptr;
    float* norm_dev = nullptr;
    uint16_t* wpack[3] = {nullptr, nullptr, nullptr};
    silt::closure::Net net;
};
