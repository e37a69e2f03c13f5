// The coarse window's wall mask (src/fluid_core.rs:7288-7360 solid_mask).
#include "sheet_walls.cuh"

#include <cmath>

#include "launch_count.cuh"
#include "sheet_math.cuh"

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

__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    return t;  // thread 0
}

__global__ void k_scour(ScourPlanes P) {
    ::silt::dep_wait();
    __shared__ double red[8];
    const int res = P.res;
    double moved = 0.0;
    unsigned int deepest = 0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < res * res; g += gridDim.x * blockDim.x) {
        const int i = g % res, j = g / res;
        if (i < 1 || j < 1 || i + 1 >= res || j + 1 >= res) continue;
        if (P.mask[g] != 0 || P.water[g] < 0.02f) continue;
        if (P.mask[g - 1] != 1 && P.mask[g + 1] != 1 && P.mask[g - res] != 1 && P.mask[g + res] != 1) continue;
        const float speed = hypot_rn(P.uw[g], P.vw[g]);
        if (!isfinite(speed)) continue;
        const float tau = 1000.0f * 0.03f * speed * speed;
        const float tau_c = 1.5f;
        if (tau <= tau_c) continue;
        const float rate = fminf(0.0035f * (tau / tau_c - 1.0f), 0.012f);
        const float room = fmaxf(0.08f - P.bed_drop[g], 0.0f);
        const float dh = fminf(rate * P.dt, room);
        if (!(dh > 0.0f)) continue;
        P.bed[g] -= dh;
        const float before = P.slurry[g];
        const float after = before + dh;
        P.slurry[g] = after;
        moved += (double)after - (double)before;
        P.us[g] = P.uw[g];
        P.vs[g] = P.vw[g];
        P.grain[g] = 1;  // Grain::Silt
        P.moisture[g] = fmaxf(P.moisture[g], 0.9f);
        const float drop = P.bed_drop[g] + dh;
        P.bed_drop[g] = drop;
        deepest = max(deepest, __float_as_uint(drop));
    }
    const double t = block_sum(moved, red);
    if (threadIdx.x == 0 && t != 0.0) {
        atomicAdd(P.slurry_sum, t);
        atomicAdd(P.eroded, t * (double)P.area);
    }
    if (deepest) atomicMax(P.hole_bits, deepest);
}

// Wall forces and block counts over the window; ring sums, block per body
// (blockIdx.y = 1 + k).
__global__ void k_load(const uint8_t* mask, const float* water, const float* uw, const float* vw, const float* bed,
                       int res, float cell, float ox, float oz, const SolidGeom* geoms, double* out) {
    ::silt::dep_wait();
    __shared__ double red[8];
    double a = 0.0, b = 0.0, c = 0.0;
    if (blockIdx.y == 0) {
        for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < res * res; g += gridDim.x * blockDim.x) {
            const uint8_t m = mask[g];
            if (m == 1) c += 1.0;
            if (m == 2) c += 1048576.0;  // the wall count rides above the contact count (< 2^20 cells)
            if (m != 0) continue;
            const float h = water[g];
            if (h < 1.0e-4f || !isfinite(h)) continue;
            const int i = g % res, j = g / res;
            for (int k = 0; k < 4; ++k) {
                const int di = k == 0 ? -1 : (k == 1 ? 1 : 0), dj = k == 2 ? -1 : (k == 3 ? 1 : 0);
                const int ni = i + di, nj = j + dj;
                if (ni < 0 || nj < 0 || ni >= res || nj >= res || mask[nj * res + ni] == 0) continue;
                const float nx = (float)di, nz = (float)dj;
                const float hydro = 1000.0f * 9.81f * h * h * 0.5f * cell;
                a += (double)(nx * hydro);
                b += (double)(nz * hydro);
                const float vn = uw[g] * nx + vw[g] * nz;
                if (vn > 0.0f) {
                    const float dyn_f = 0.5f * 1000.0f * vn * vn * h * cell;
                    a += (double)(nx * dyn_f);
                    b += (double)(nz * dyn_f);
                }
            }
        }
    } else {
        const SolidGeom& s = geoms[blockIdx.y - 1];
        const float reach = s.ring;
        const int i0 = (int)floorf((s.x - reach - ox) / cell), i1 = (int)floorf((s.x + reach - ox) / cell);
        const int j0 = (int)floorf((s.z - reach - oz) / cell), j1 = (int)floorf((s.z + reach - oz) / cell);
        const int w = i1 - i0 + 1;
        const int cells = w > 0 && j1 >= j0 ? w * (j1 - j0 + 1) : 0;
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cells; q += gridDim.x * blockDim.x) {
            const int i = i0 + q % w, j = j0 + q / w;
            if (i < 0 || j < 0 || i >= res || j >= res) continue;
            const float x = ox + ((float)i + 0.5f) * cell;
            const float z = oz + ((float)j + 0.5f) * cell;
            const float dx = x - s.x, dz = z - s.z;
            const float along = dx * s.fx + dz * s.fz;
            const float lat = dx * s.fz + dz * (-s.fx);
            if (fabsf(along) <= s.hl && fabsf(lat) <= s.hw) continue;  // solid_contains
            if (hypot_rn(dx, dz) > reach) continue;
            const int g = j * res + i;
            if (water[g] < 0.01f) continue;
            a += (double)bed[g];
            b += (double)water[g];
            c += 1.0;
        }
    }
    double* o = blockIdx.y == 0 ? out : out + 4 + 3 * (blockIdx.y - 1);
    const double ta = block_sum(a, red);
    const double tb = block_sum(b, red);
    const double tc = block_sum(c, red);
    if (threadIdx.x == 0) {
        atomicAdd(&o[0], ta);
        atomicAdd(&o[1], tb);
        if (blockIdx.y == 0) {
            const double walls = floor(tc / 1048576.0);
            atomicAdd(&o[2], tc - walls * 1048576.0);
            atomicAdd(&o[3], walls);
        } else {
            atomicAdd(&o[2], tc);
        }
    }
}

}  // namespace

cudaError_t launch_scour(const ScourPlanes& P, cudaStream_t st) {
    const int cells = P.res * P.res;
    int blocks = (cells + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    ::silt::launch_dep(k_scour, dim3(blocks), dim3(256), 0, st, P);
    ::silt::count_launch();
    return cudaGetLastError();
}

cudaError_t launch_load(const uint8_t* mask, const float* water, const float* uw, const float* vw, const float* bed,
                        int res, float cell, float ox, float oz, const SolidGeom* geoms, int n, double* out,
                        cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, (4 + 3 * (size_t)n) * sizeof(double), st);
    if (e != cudaSuccess) return e;
    ::silt::launch_dep(k_load, dim3(148, 1 + n), dim3(256), 0, st, mask, water, uw, vw, bed, res, cell, ox, oz, geoms,
                       out);
    ::silt::count_launch();
    return cudaGetLastError();
}

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
    s.ring = std::fmax(half_length, half_width) + 0.55f;
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
