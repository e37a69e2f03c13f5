// Walls in the sheet: the bodies' footprints (src/fluid_core.rs:213-240
// HydroSolid) and the wall mask the step reads (:7288-7360 solid_mask).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace silt {
namespace walls {

// One body as the mask kernels read it. The trigonometry and the hypot are
// evaluated once on the host with the C library (the reference's f32 methods
// call the same functions), so every grid sees the same bits.
struct SolidGeom {
    float x, z;
    float fx, fz;       // sin(yaw), cos(yaw): the long axis
    float hl, hw;       // max(half_length, 0), max(half_width, 0)
    float bottom, top;  // underside and top, world Y
    float reach0;       // hypot(hl, hw); the grid adds one cell
    int32_t contact;    // 1: tire contact (drawn over walls)
    int32_t valid;      // 0: skipped (degenerate extent, or x, z not finite)
    float ring;         // max(half_length, half_width) + 0.55: ring_surface's reach
};

constexpr int MAX_SOLIDS = 64;

// Whether body `s` covers cell (i, j) of a grid at origin (ox, oz) whose
// highest neighbouring surface is `eta` over bed `bedv`: the reference's
// bounding-box clip, then solid_overlaps (:4584-4604).
__device__ __forceinline__ bool covers(const SolidGeom& s, int i, int j, int res, float cell, float ox, float oz,
                                       float eta, float bedv) {
    if (!s.valid) return false;
    const float reach = s.reach0 + cell;
    if (!isfinite(reach)) return false;
    const float lo_i = floorf((s.x - reach - ox) / cell - 0.5f);
    const float hi_i = ceilf((s.x + reach - ox) / cell - 0.5f);
    const float lo_j = floorf((s.z - reach - oz) / cell - 0.5f);
    const float hi_j = ceilf((s.z + reach - oz) / cell - 0.5f);
    const float top = (float)(res - 1);
    if (hi_i < 0.0f || hi_j < 0.0f || lo_i > top || lo_j > top) return false;
    if ((float)i < fmaxf(lo_i, 0.0f) || (float)i > fminf(hi_i, top)) return false;
    if ((float)j < fmaxf(lo_j, 0.0f) || (float)j > fminf(hi_j, top)) return false;
    const float x = ox + ((float)i + 0.5f) * cell;
    const float z = oz + ((float)j + 0.5f) * cell;
    const float dx = x - s.x, dz = z - s.z;
    const float along = dx * s.fx + dz * s.fz;
    const float lat = dx * s.fz + dz * (-s.fx);
    if (!(fabsf(along) <= s.hl && fabsf(lat) <= s.hw)) return false;
    return eta > s.bottom + 1.0e-4f && bedv < s.top;
}

// The mask value of cell (i, j): 1 under a contact, else 2 under a wall, else
// 0. The surface tested is the highest of the cell and its four neighbours.
__device__ __forceinline__ uint8_t mask_value(const SolidGeom* geoms, int n, int i, int j, int res, float cell,
                                              float ox, float oz, const float* water, const float* bed) {
    const int g = j * res + i;
    float eta = bed[g] + water[g];
    if (i > 0) eta = fmaxf(eta, bed[g - 1] + water[g - 1]);
    if (i + 1 < res) eta = fmaxf(eta, bed[g + 1] + water[g + 1]);
    if (j > 0) eta = fmaxf(eta, bed[g - res] + water[g - res]);
    if (j + 1 < res) eta = fmaxf(eta, bed[g + res] + water[g + res]);
    uint8_t v = 0;
    for (int k = 0; k < n; ++k) {
        const SolidGeom& s = geoms[k];
        if (v == 1 || (v == 2 && !s.contact)) continue;
        if (covers(s, i, j, res, cell, ox, oz, eta, bed[g])) v = s.contact ? 1 : 2;
    }
    return v;
}

// scour_contacts (src/fluid_core.rs:7364-7420) on the coarse window, from its
// wall mask: the cut bed goes into the slurry sheet; `eroded` (FP64 m^3) and
// `hole_bits` (the deepest cut, float bits) accumulate.
struct ScourPlanes {
    const uint8_t* mask;
    const float* water;
    const float* uw;
    const float* vw;
    float* bed;
    float* slurry;
    float* us;
    float* vs;
    float* moisture;
    float* bed_drop;
    uint8_t* grain;
    int res;
    float area, dt;
    double* eroded;       // m^3: each cut cell's actual slurry change times its area
    double* slurry_sum;   // the step's FP64 slurry depth sum, kept current
    unsigned int* hole_bits;
};
cudaError_t launch_scour(const ScourPlanes& P, cudaStream_t st);

// hydro_load's sums (:7164-7249) from the window's wall mask: out[0..1]
// force x, z (N, FP64 sums of the reference's f32 terms), out[2..3] contact and
// wall cell counts, then per body k out[4 + 3k ..] the ring's bed sum, water
// sum and cell count (:7251-7286).
cudaError_t launch_load(const uint8_t* mask, const float* water, const float* uw, const float* vw, const float* bed,
                        int res, float cell, float ox, float oz, const SolidGeom* geoms, int n, double* out,
                        cudaStream_t st);

// The host form of one body (C library trigonometry and hypot).
SolidGeom make_geom(float x, float z, float yaw, float half_length, float half_width, float bottom_y, float top_y,
                    int contact);

// The coarse window's mask (res^2 bytes) from its water over its bed.
cudaError_t launch_mask(uint8_t* mask, int res, float cell, float ox, float oz, const float* water, const float* bed,
                        const SolidGeom* geoms, int n, cudaStream_t st);

}  // namespace walls
}  // namespace silt
