// The coarse window's wall mask (src/fluid_core.rs:7288-7360 solid_mask).
#include "sheet_walls.cuh"

#include <cmath>

#include "launch_count.cuh"

namespace silt {
namespace walls {

namespace {

__global__ void k_mask(uint8_t* mask, int res, float cell, float ox, float oz, const float* water, const float* bed,
                       const SolidGeom* geoms, int n) {
    ::silt::dep_wait();
    const int cells = res * res;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < cells; g += gridDim.x * blockDim.x)
        mask[g] = mask_value(geoms, n, g % res, g / res, res, cell, ox, oz, water, bed);
}

}  // namespace

SolidGeom make_geom(float x, float z, float yaw, float half_length, float half_width, float bottom_y, float top_y,
                    int contact) {
    SolidGeom s{};
    s.x = x;
    s.z = z;
    s.fx = std::sin(yaw);
    s.fz = std::cos(yaw);
    s.hl = std::fmax(half_length, 0.0f);
    s.hw = std::fmax(half_width, 0.0f);
    s.bottom = bottom_y;
    s.top = top_y;
    s.reach0 = std::hypot(s.hl, s.hw);
    s.contact = contact ? 1 : 0;
    s.valid = half_length > 1.0e-4f && half_width > 1.0e-4f && std::isfinite(x) && std::isfinite(z) ? 1 : 0;
    return s;
}

cudaError_t launch_mask(uint8_t* mask, int res, float cell, float ox, float oz, const float* water, const float* bed,
                        const SolidGeom* geoms, int n, cudaStream_t st) {
    const int cells = res * res;
    int blocks = (cells + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    ::silt::launch_dep(k_mask, dim3(blocks), dim3(256), 0, st, mask, res, cell, ox, oz, water, bed, geoms, n);
    ::silt::count_launch();
    return cudaGetLastError();
}

}  // namespace walls
}  // namespace silt
