// Boundary drivers of the coarse water sheet in open water (sheet_drivers.cu):
// the paddle strip and the river reach. The host evaluates each step's
// scalars (the stroke with the host libm's sinf, the pull with its expf, the
// index ranges) exactly as the reference writes them.
#pragma once

#include <cuda_runtime.h>

#include "sheet_fine.cuh"

namespace silt {
namespace drivers {

struct WaveStep {
    int i0, i1, j0, j1;         // the strip's cells on the window
    float x0, x1, z0, z1;       // the strip, m
    float dx, dz;               // unit push direction
    float stroke, pull;         // this step's paddle velocity and relaxation
    float span_x, span_z;
};

struct ReachStep {
    int along_z, positive;
    int c0, c1, rows;           // cross band and end rows on the window
    float dx, dz;               // downstream unit vector
    float inlet_eta, outlet_eta, inlet_speed;
    float inflow_c;             // the inlet's suspended load as a fraction of the water column (0: none)
    float* susp;                // the suspended-solids plane (when inflow_c > 0)
    double* entrained;          // its FP64 book of solids that entered the window
};

cudaError_t wave_step(const fine::SheetView& W, const WaveStep& w, cudaStream_t st);
// bank: the reference's f32 bank (device); books[4]: its FP64 twin.
cudaError_t reach_step(const fine::SheetView& W, const ReachStep& r, float* bank, double* books, cudaStream_t st);

}  // namespace drivers
}  // namespace silt
