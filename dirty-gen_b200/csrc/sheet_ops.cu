// Per-cell kernels around the sheet step: seeding (the reference's closure
// writes), the render-contract publish, map export, the FP64 ledger sum and
// the non-finite count. Each follows the reference function it names.
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "block_sum.cuh"
#include "sheet_math.cuh"
#include "sheet_ops.cuh"
#include "launch_count.cuh"

namespace silt {

#define GRID_STRIDE(i, n) for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

static int blocks_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b > 148 * 16 ? 148 * 16 : (b == 0 ? 1 : b));
}

// src/fluid_core.rs:5329-5356 map_water_bed, per cell.
__global__ void k_map_water_bed(const float* bed_in, const float* water_in, float* bed, float* water, float* moisture,
                                uint8_t* grain, size_t n) {
    ::silt::dep_wait();
    GRID_STRIDE(i, n) {
        float b = bed_in[i];
        bed[i] = finite_f(b) ? b : 0.0f;
        float w = water_in[i];
        w = finite_f(w) ? fmaxf(w, 0.0f) : 0.0f;
        water[i] = w;
        if (w > 0.0f) {
            moisture[i] = fmaxf(moisture[i], 0.8f);
            if (grain[i] == 4) grain[i] = 1;
        }
    }
}

// src/fluid_core.rs:5358-5372 map_water_velocity.
__global__ void k_map_water_velocity(const float* u_in, const float* v_in, const float* water, float* uw, float* vw,
                                     size_t n) {
    ::silt::dep_wait();
    GRID_STRIDE(i, n) {
        if (water[i] <= 1.0e-6f) continue;
        float u = u_in[i], v = v_in[i];
        uw[i] = finite_f(u) ? u : 0.0f;
        vw[i] = finite_f(v) ? v : 0.0f;
    }
}

// src/fluid_core.rs:5820-5849 paint (pour_water / pour_slurry).
__global__ void k_paint(float* depth_plane, float* moisture, uint8_t* grain, int res, float cell, float ox, float oz,
                        float x0, float x1, float z0, float z1, float depth, int water, int g, float m) {
    ::silt::dep_wait();
    size_t n = (size_t)res * res;
    GRID_STRIDE(k, n) {
        int i = (int)(k % res), j = (int)(k / res);
        float x = ox + ((float)i + 0.5f) * cell;
        float z = oz + ((float)j + 0.5f) * cell;
        if (x < x0 || x >= x1 || z < z0 || z >= z1) continue;
        depth_plane[k] = depth;
        if (!water) {
            grain[k] = (uint8_t)g;
            moisture[k] = m;
        }
    }
}

// src/fluid_core.rs:5854-5877 lay_slurry_mask.
__global__ void k_lay_slurry(const float* depth, float* slurry, float* moisture, uint8_t* grain, size_t n, int g,
                             float m) {
    ::silt::dep_wait();
    GRID_STRIDE(i, n) {
        float d = depth[i];
        if (!(finite_f(d) && d > 0.0f)) continue;
        slurry[i] += d;
        grain[i] = (uint8_t)g;
        moisture[i] = fmaxf(moisture[i], m);
    }
}

// src/fluid_core.rs:5236-5254 lay_slurry_on_water, per cell: a slurry film
// of `depth` on every cell holding more than 12 mm of water; `count` gets the
// number of such cells.
__global__ void k_lay_on_water(const float* water, float* slurry, float* moisture, uint8_t* grain, size_t n, float depth,
                               int g, unsigned int* count) {
    ::silt::dep_wait();
    unsigned int c = 0;
    GRID_STRIDE(i, n) {
        if (water[i] <= 0.012f) continue;
        slurry[i] = depth;
        grain[i] = (uint8_t)g;
        moisture[i] = fmaxf(moisture[i], 0.90f);
        ++c;
    }
    if (c) atomicAdd(count, c);
}

// src/fluid_core.rs:5928-5950 read_substrate_grid, per cell.
__global__ void k_read_substrate(const float* bed_in, const float* moist_in, const uint8_t* grain_in, float* bed,
                                 float* moisture, uint8_t* grain, const float* slurry, size_t n) {
    ::silt::dep_wait();
    GRID_STRIDE(i, n) {
        bed[i] = bed_in[i];
        moisture[i] = rclamp(moist_in[i], 0.0f, 1.0f);
        if (slurry[i] > 1.0e-5f) grain[i] = grain_in[i];
    }
}

// Inflow strip: depth added on one row over [x0, x1). A cell still waiting
// for the previous dry cut gets it first, so the water lands at rest.
__global__ void k_inflow(float* water, float* uw, float* vw, int cut_pending, int res, int j, int i0, int i1,
                         float add, int tiles_x, uint8_t* t_wet, uint8_t* t_zuv, uint8_t* t_zh) {
    ::silt::dep_wait();
    int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= i1) return;
    size_t c = (size_t)j * res + i;
    if (tiles_x) {  // the grid engine's tile of this cell now holds water
        const int t = (j / 32) * tiles_x + i / 32;
        t_wet[t] = 1;
        t_zuv[t] = 0;
        t_zh[t] = 0;
    }
    if (cut_pending && water[c] < 1.0e-6f) {
        uw[c] = 0.0f;
        vw[c] = 0.0f;
    }
    water[c] += add;
}

// coarse_cell (src/fluid_core.rs:6998-7035) feeding render_contract film/flow
// (src/render_contract.rs:457-496). Tracers are off the sheet path: turbidity 0.
__global__ void k_publish(const float* water, const float* slurry, const float* uw, const float* vw, const float* us,
                          const float* vs, const float* susp, const float* turbid, float* film, float* flow, size_t n) {
    ::silt::dep_wait();
    GRID_STRIDE(i, n) {
        float water_m = finite0(water[i]), slurry_m = finite0(slurry[i]);
        float fl = water_m + slurry_m;
        float u = 0.0f, v = 0.0f;
        if (!(fl < 1.0e-5f)) {
            u = finite0((uw[i] * water_m + us[i] * slurry_m) / fl);
            v = finite0((vw[i] * water_m + vs[i] * slurry_m) / fl);
        }
        bool dry = !finite_f(water_m) || !finite_f(slurry_m) || water_m + slurry_m < 1.0e-5f;
        if (dry) { u = 0.0f; v = 0.0f; }
        float speed = dry ? 0.0f : finite0(sqrtf(u * u + v * v));
        // coarse_cell's turbidity (src/fluid_core.rs:7024-7032): suspended load
        // and stirred silt over the water column; the publish clamps it again.
        const float turbidity =
            water_m < 1.0e-5f
                ? 0.0f
                : rclamp((fmaxf(finite0(susp[i]), 0.0f) + fmaxf(finite0(turbid[i]), 0.0f)) / water_m, 0.0f, 1.0f);
        const float turb = (!finite_f(water_m) || water_m < 1.0e-5f) ? 0.0f : rclamp(finite0(turbidity), 0.0f, 1.0f);
        reinterpret_cast<float2*>(film)[i] = make_float2(finite0(water_m), finite0(slurry_m));
        reinterpret_cast<float4*>(flow)[i] = make_float4(u, v, speed, turb);
    }
}

// export_maps (src/fluid_core.rs:6941-6975).
__global__ void k_export(const float* bed, const float* water, const float* slurry, const float* uw, const float* vw,
                         const float* us, const float* vs, const float* moist, float* height, float* vel_u,
                         float* vel_v, float* moisture, size_t n) {
    ::silt::dep_wait();
    GRID_STRIDE(i, n) {
        if (height) height[i] = bed[i] + water[i] + slurry[i];
        float hw = finite0(water[i]), hs = finite0(slurry[i]);
        float h = hw + hs;
        float u = 0.0f, v = 0.0f;
        if (!(h < 1.0e-5f)) {
            u = finite0((uw[i] * hw + us[i] * hs) / h);
            v = finite0((vw[i] * hw + vs[i] * hs) / h);
        }
        if (vel_u) vel_u[i] = u;
        if (vel_v) vel_v[i] = v;
        if (moisture) moisture[i] = moist[i];
    }
}

// FP64 sums of max(h, 0) for two planes (the ledger's column_sum, src/fluid_core.rs:4617).
__global__ void k_sum2(const float* a, const float* b, size_t n, double* out) {
    ::silt::dep_wait();
    double sa = 0.0, sb = 0.0;
    GRID_STRIDE(i, n) {
        sa += (double)fmaxf(a[i], 0.0f);
        sb += (double)fmaxf(b[i], 0.0f);
    }
    ::silt::block_add(sa, out);
    ::silt::block_add(sb, out + 1);
}

// The last block of a launch to finish (the ticket counts finished blocks)
// adds the blocks' partial pairs part[2k], part[2k + 1], k < nb, in a fixed
// order into out[0], out[1] and re-arms the ticket, so the sum does not
// depend on the order the blocks ran in. Every thread of the block calls it.
__device__ __forceinline__ void ordered_finish(double sa, double sb, double* part, unsigned int* ticket, int k,
                                               int nb, double* out) {
    __shared__ int last;
    sa = ::silt::block_sum(sa);
    sb = ::silt::block_sum(sb);
    if (threadIdx.x == 0) {
        part[2 * k] = sa;
        part[2 * k + 1] = sb;
        __threadfence();
        last = atomicAdd(ticket, 1u) == (unsigned int)(nb - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double ta = 0.0, tb = 0.0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) {
        ta += ((volatile double*)part)[2 * q];
        tb += ((volatile double*)part)[2 * q + 1];
    }
    ta = ::silt::block_sum(ta);
    tb = ::silt::block_sum(tb);
    if (threadIdx.x == 0) {
        out[0] = ta;
        out[1] = tb;
        *ticket = 0u;
    }
}

// k_sum2 with a fixed grid and an ordered finish: the same planes give the
// same bits on every call.
__global__ void k_sum2_ordered(const float* a, const float* b, size_t n, double* out, double* part,
                               unsigned int* ticket) {
    ::silt::dep_wait();
    double sa = 0.0, sb = 0.0;
    GRID_STRIDE(i, n) {
        sa += (double)fmaxf(a[i], 0.0f);
        sb += (double)fmaxf(b[i], 0.0f);
    }
    ordered_finish(sa, sb, part, ticket, blockIdx.x, gridDim.x, out);
}

__global__ void k_non_finite(const float* const* planes, int np, size_t n, unsigned int* out) {
    ::silt::dep_wait();
    unsigned int c = 0;
    GRID_STRIDE(i, n) {
        for (int p = 0; p < np; ++p) c += !finite_f(planes[p][i]);
    }
    ::silt::block_add(c, out);
}

// src/fluid_core.rs:7521-7581 eddy_shear, the snapshot pass: neighbours in
// the order (-1, 0), (1, 0), (0, -1), (0, 1); a wet neighbour (over 3 mm)
// gives its velocity, dry ground standing 3 cm above the surface gives 0 (no
// slip), a dry beach is skipped, the window edge too.
__global__ void k_eddy(const float* h, const float* u, const float* v, const float* bed, int res, float k, float* du,
                       float* dv) {
    ::silt::dep_wait();
    const size_t n = (size_t)res * res;
    GRID_STRIDE(idx, n) {
        const int i = (int)(idx % res), j = (int)(idx / res);
        float a = 0.0f, b = 0.0f;
        const float h0 = h[idx];
        if (h0 > 0.003f) {
            const float u0 = u[idx], v0 = v[idx];
            float lu = 0.0f, lv = 0.0f;
            const int di[4] = {-1, 1, 0, 0}, dj[4] = {0, 0, -1, 1};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int ni = i + di[q], nj = j + dj[q];
                if (ni < 0 || nj < 0 || ni >= res || nj >= res) continue;
                const size_t nidx = (size_t)nj * res + ni;
                float un, vn;
                if (h[nidx] > 0.003f) {
                    un = u[nidx];
                    vn = v[nidx];
                } else if (bed[nidx] > bed[idx] + h0 + 0.03f) {
                    un = 0.0f;
                    vn = 0.0f;
                } else {
                    continue;
                }
                lu += un - u0;
                lv += vn - v0;
            }
            a = k * lu;
            b = k * lv;
        }
        du[idx] = a;
        dv[idx] = b;
    }
}

// The eddy change applied (src/fluid_core.rs:7570-7580), then Manning bed
// friction (:7485-7512): keep = 1 / (1 + dt g n^2 |u| / max(h, 2 mm)^(4/3)).
__global__ void k_friction(const float* h, float* u, float* v, const float* du, const float* dv, size_t n, float gn2,
                           float dt) {
    ::silt::dep_wait();
    GRID_STRIDE(idx, n) {
        float uu = u[idx], vv = v[idx];
        const float a = du[idx], b = dv[idx];
        if (a != 0.0f || b != 0.0f) {
            const float nu = uu + a, nv = vv + b;
            if (isfinite(nu) && isfinite(nv)) {
                uu = nu;
                vv = nv;
            }
        }
        if (gn2 > 0.0f) {
            const float hv = h[idx];
            if (hv > 1.0e-4f) {
                const float speed = hypot_rn(uu, vv);
                if (speed > 0.0f) {
                    const float kk = gn2 * speed / pow_rn(fmaxf(hv, 0.002f), 4.0f / 3.0f);
                    const float keep = 1.0f / (1.0f + dt * kk);
                    uu = uu * keep;
                    vv = vv * keep;
                }
            }
        }
        u[idx] = uu;
        v[idx] = vv;
    }
}

// src/fluid_core.rs:7584-7636 diffuse_surface. The transfer across the face
// from cell a to its east or north neighbour b, both wet, is k (eta_a -
// eta_b) limited to a quarter of the donor. Each cell gathers its four faces
// in the order the reference's raster sweep adds them to it: from the cell
// below, from the cell to the west, then its own east and north faces.
__device__ __forceinline__ float surface_flux(const float* h, const float* bed, size_t a, size_t b, float k) {
    const float ha = h[a], hb = h[b];
    if (!(ha > 0.003f) || !(hb > 0.003f)) return 0.0f;
    float f = k * ((bed[a] + ha) - (bed[b] + hb));
    if (f > 0.0f) f = fminf(f, 0.25f * ha);
    else f = fmaxf(f, -0.25f * hb);
    return f;
}

__global__ void k_diffuse(const float* h, const float* bed, int res, float k, float* delta) {
    ::silt::dep_wait();
    const size_t n = (size_t)res * res;
    GRID_STRIDE(idx, n) {
        const int i = (int)(idx % res), j = (int)(idx / res);
        float d = 0.0f;
        if (j > 0) d += surface_flux(h, bed, idx - res, idx, k);
        if (i > 0) d += surface_flux(h, bed, idx - 1, idx, k);
        if (i + 1 < res) d -= surface_flux(h, bed, idx, idx + 1, k);
        if (j + 1 < res) d -= surface_flux(h, bed, idx, idx + res, k);
        delta[idx] = d;
    }
}

__global__ void k_diffuse_apply(float* h, const float* delta, size_t n, double* ledger) {
    ::silt::dep_wait();
    double part = 0.0;
    GRID_STRIDE(idx, n) {
        const float d = delta[idx];
        if (d != 0.0f && isfinite(d)) {
            const float h0 = h[idx], h1 = fmaxf(h0 + d, 0.0f);
            h[idx] = h1;
            part += (double)h1 - (double)h0;
        }
    }
    if (ledger) ::silt::block_add(part, ledger);
}

cudaError_t op_map_water_bed(const float* bed_in, const float* water_in, float* bed, float* water, float* moisture,
                             uint8_t* grain, size_t n, cudaStream_t st) {
    ::silt::launch_dep(k_map_water_bed, dim3(blocks_for(n)), dim3(256), 0, st, bed_in, water_in, bed, water, moisture, grain, n);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_map_water_velocity(const float* u_in, const float* v_in, const float* water, float* uw, float* vw,
                                  size_t n, cudaStream_t st) {
    ::silt::launch_dep(k_map_water_velocity, dim3(blocks_for(n)), dim3(256), 0, st, u_in, v_in, water, uw, vw, n);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_paint(float* depth_plane, float* moisture, uint8_t* grain, int res, float cell, float ox, float oz,
                     float x0, float x1, float z0, float z1, float depth, int water, int g, float m, cudaStream_t st) {
    ::silt::launch_dep(k_paint, dim3(blocks_for((size_t)res * res)), dim3(256), 0, st, depth_plane, moisture, grain, res, cell, ox, oz, x0, x1, z0,
                                                           z1, depth, water, g, m);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_lay_slurry(const float* depth, float* slurry, float* moisture, uint8_t* grain, size_t n, int g, float m,
                          cudaStream_t st) {
    ::silt::launch_dep(k_lay_slurry, dim3(blocks_for(n)), dim3(256), 0, st, depth, slurry, moisture, grain, n, g, m);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_lay_on_water(const float* water, float* slurry, float* moisture, uint8_t* grain, size_t n, float depth,
                            int g, unsigned int* count, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    ::silt::launch_dep(k_lay_on_water, dim3(blocks_for(n)), dim3(256), 0, st, water, slurry, moisture, grain, n, depth,
                       g, count);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_read_substrate(const float* bed_in, const float* moist_in, const uint8_t* grain_in, float* bed,
                              float* moisture, uint8_t* grain, const float* slurry, size_t n, cudaStream_t st) {
    ::silt::launch_dep(k_read_substrate, dim3(blocks_for(n)), dim3(256), 0, st, bed_in, moist_in, grain_in, bed, moisture, grain, slurry, n);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_inflow(float* water, float* uw, float* vw, int cut_pending, int res, int j, int i0, int i1, float add,
                      int tiles_x, uint8_t* t_wet, uint8_t* t_zuv, uint8_t* t_zh, cudaStream_t st) {
    if (i1 <= i0) return cudaSuccess;
    ::silt::launch_dep(k_inflow, dim3((i1 - i0 + 127) / 128), dim3(128), 0, st, water, uw, vw, cut_pending, res, j, i0, i1, add, tiles_x, t_wet,
                                                     t_zuv, t_zh);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_publish(const float* water, const float* slurry, const float* uw, const float* vw, const float* us,
                       const float* vs, const float* susp, const float* turbid, float* film, float* flow, size_t n,
                       cudaStream_t st) {
    ::silt::launch_dep(k_publish, dim3(blocks_for(n)), dim3(256), 0, st, water, slurry, uw, vw, us, vs, susp, turbid,
                       film, flow, n);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_export(const float* bed, const float* water, const float* slurry, const float* uw, const float* vw,
                      const float* us, const float* vs, const float* moist, float* height, float* vel_u, float* vel_v,
                      float* moisture, size_t n, cudaStream_t st) {
    ::silt::launch_dep(k_export, dim3(blocks_for(n)), dim3(256), 0, st, bed, water, slurry, uw, vw, us, vs, moist, height, vel_u, vel_v, moisture,
                                           n);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_sum2(const float* a, const float* b, size_t n, double* out, cudaStream_t st, double* scratch) {
    if (scratch) {
        const int nb = std::min(blocks_for(n), SUM_BLOCKS);
        unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + 2 * SUM_BLOCKS);
        ::silt::launch_dep(k_sum2_ordered, dim3(nb), dim3(256), 0, st, a, b, n, out, scratch, ticket);
        ::silt::count_launch();
        return cudaGetLastError();
    }
    cudaError_t e = cudaMemsetAsync(out, 0, 2 * sizeof(double), st);
    if (e != cudaSuccess) return e;
    ::silt::launch_dep(k_sum2, dim3(blocks_for(n)), dim3(256), 0, st, a, b, n, out);
    ::silt::count_launch();
    return cudaGetLastError();
}
__global__ void k_gather_ledgers(const double* const* acc, const double* const* books, int n, double* out) {
    ::silt::dep_wait();
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n) return;
    double* o = out + 16 * (size_t)w;
    o[0] = acc[w][0];
    o[1] = acc[w][1];
    o[2] = books[w][0];
    o[3] = books[w][1];
    o[4] = books[w][2];
    o[5] = books[w][3];
    o[6] = books[w][4];
    o[7] = books[w][6];
    for (int k = 0; k < 6; ++k) o[8 + k] = books[w][7 + k];  // the tracers' books
}
__global__ void k_gather_words(const unsigned int* const* src, int n, int words, unsigned int* out) {
    ::silt::dep_wait();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * words) return;
    out[q] = src[q / words][q % words];
}
// Every window's suspended and silt column sums (FP64 of the clamped cells)
// into out[16 w + 14], [16 w + 15], in a fixed order (ordered_finish per
// window; part holds gridDim.x pairs per window, then the windows' tickets).
__global__ void k_sum_tracers(const float* const* susp, const float* const* turbid, const int* cells, double* out,
                              double* part) {
    ::silt::dep_wait();
    const int w = blockIdx.y;
    const float* a = susp[w];
    const float* b = turbid[w];
    const size_t n = (size_t)cells[w];
    double sa = 0.0, sb = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        sa += (double)fmaxf(a[i], 0.0f);
        sb += (double)fmaxf(b[i], 0.0f);
    }
    unsigned int* tickets = reinterpret_cast<unsigned int*>(part + 2 * (size_t)gridDim.x * gridDim.y);
    ordered_finish(sa, sb, part + 2 * (size_t)gridDim.x * w, tickets + w, blockIdx.x, gridDim.x,
                   out + 16 * (size_t)w + 14);
}
size_t sum_tracers_scratch_bytes(int n) {
    const int per = std::max(1, std::min(64, 2368 / std::max(n, 1)));
    return (2 * (size_t)per * n) * sizeof(double) + (size_t)n * sizeof(unsigned int);
}
cudaError_t op_sum_tracers(const float* const* susp, const float* const* turbid, const int* cells, int n, double* out,
                           double* scratch, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int per = std::max(1, std::min(64, 2368 / n));
    ::silt::launch_dep(k_sum_tracers, dim3(per, n), dim3(256), 0, st, susp, turbid, cells, out, scratch);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_gather_ledgers(const double* const* acc, const double* const* books, int n, double* out,
                              cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    ::silt::launch_dep(k_gather_ledgers, dim3((n + 127) / 128), dim3(128), 0, st, acc, books, n, out);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_gather_words(const unsigned int* const* src, int n, int words, unsigned int* out, cudaStream_t st) {
    if (n <= 0 || words <= 0) return cudaSuccess;
    ::silt::launch_dep(k_gather_words, dim3((n * words + 255) / 256), dim3(256), 0, st, src, n, words, out);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_open_water(const float* h, float* u, float* v, const float* bed, int res, float k_visc, float gn2,
                          float dt, float* scratch, cudaStream_t st) {
    const size_t n = (size_t)res * res;
    float* du = scratch;
    float* dv = scratch + n;
    if (k_visc > 0.0f) {
        ::silt::launch_dep(k_eddy, dim3(blocks_for(n)), dim3(256), 0, st, h, (const float*)u, (const float*)v, bed,
                           res, k_visc, du, dv);
        ::silt::count_launch();
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    } else {
        cudaError_t e = cudaMemsetAsync(scratch, 0, 2 * n * sizeof(float), st);
        if (e != cudaSuccess) return e;
    }
    ::silt::launch_dep(k_friction, dim3(blocks_for(n)), dim3(256), 0, st, h, u, v, (const float*)du,
                       (const float*)dv, n, gn2, dt);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_diffuse_surface(float* h, const float* bed, int res, float k, float* scratch, double* ledger,
                               cudaStream_t st) {
    const size_t n = (size_t)res * res;
    ::silt::launch_dep(k_diffuse, dim3(blocks_for(n)), dim3(256), 0, st, (const float*)h, bed, res, k, scratch);
    ::silt::count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    ::silt::launch_dep(k_diffuse_apply, dim3(blocks_for(n)), dim3(256), 0, st, h, (const float*)scratch, n, ledger);
    ::silt::count_launch();
    return cudaGetLastError();
}
cudaError_t op_non_finite(const float* const* planes, int np, size_t n, unsigned int* out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    ::silt::launch_dep(k_non_finite, dim3(blocks_for(n)), dim3(256), 0, st, planes, np, n, out);
    ::silt::count_launch();
    return cudaGetLastError();
}

}  // namespace silt
