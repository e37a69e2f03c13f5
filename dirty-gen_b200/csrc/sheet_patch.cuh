// Launch parameters of the nested-patch sheet step (sheet_patch.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace silt {
namespace patch {

// One layer of one patch: its planes and its persistent scratch.
struct Job {
    float* h;
    float* u;
    float* v;
    const float* bed;
    const uint8_t* grain;
    const float* moisture;
    float* sc[2][5];   // two scratch sets (the reference's sc and sc2): a, b, c, d, e
    float* f1;         // transient: vorticity, then edge fluxes
    float* f2;         // transient: edge fluxes, wet-body labels
    int32_t nu_const;  // 1 for the water layer
    float vort;
    int32_t active;
    int32_t pad;
};

struct Args {
    const Job* jobs;
    int32_t res;
    float cell, dt, sub_cap, eps;
    int32_t pace;
    int32_t has_sc2;
    float nu_c, mob_c;
    float decay_w[9];  // water damping factor for 1..8 substeps (index = substep count)
};

cudaError_t launch_patch_step(const Args& A, int njobs, cudaStream_t st);
size_t patch_static_smem();

}  // namespace patch
}  // namespace silt
