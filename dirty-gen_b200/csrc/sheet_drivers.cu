// The coarse window's boundary drivers of open water: the paddle strip
// (src/fluid_core.rs:7420-7480 drive_waves) and the river reach's inlet and
// outlet (:7638-7745 feed_reach).
#include "sheet_drivers.cuh"

#include "launch_count.cuh"

namespace silt {
namespace drivers {

namespace {

// Every water cell of the strip relaxes toward the paddle stroke along the
// push direction, the pull tapered over the strip's outer quarters; cells
// under 2 cm of water are left alone (so the lazy dry cut never matters).
__global__ void k_wave(fine::SheetView W, WaveStep w) {
    ::silt::dep_wait();
    const int ni = w.i1 - w.i0, nj = w.j1 - w.j0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ni * nj; q += gridDim.x * blockDim.x) {
        const int i = w.i0 + q % ni, j = w.j0 + q / ni;
        const float x = W.origin[0] + ((float)i + 0.5f) * W.cell;
        const float z = W.origin[1] + ((float)j + 0.5f) * W.cell;
        if (x < w.x0 || x > w.x1 || z < w.z0 || z > w.z1) continue;
        const size_t idx = (size_t)j * W.res + i;
        const float h = W.h[0][idx];
        if (h < 0.02f || !isfinite(h)) continue;
        const float tx = fminf(fmaxf(fminf(x - w.x0, w.x1 - x) / (0.25f * w.span_x), 0.0f), 1.0f);
        const float tz = fminf(fmaxf(fminf(z - w.z0, w.z1 - z) / (0.25f * w.span_z), 0.0f), 1.0f);
        const float k = w.pull * fminf(tx, tz);
        const float u = W.u[0][idx], v = W.v[0][idx];
        const float along = u * w.dx + v * w.dz;
        const float d = (w.stroke - along) * k;
        const float nu = u + d * w.dx, nv = v + d * w.dz;
        if (isfinite(nu) && isfinite(nv)) {
            W.u[0][idx] = nu;
            W.v[0][idx] = nv;
        }
    }
}

// One cell of the reach's inlet or outlet rows toward its stage, through the
// f32 bank exactly as the reference's sequential sweep does; the FP64 books
// receive the cell's actual change.
__device__ __forceinline__ void hold_stage(const fine::SheetView& W, size_t idx, float eta, float area, float* bank,
                                           double* moved, int i, int j) {
    const float target = fmaxf(eta - W.bed[idx], 0.0f);
    const float h = W.h[0][idx];
    if (!isfinite(h) || target <= 0.0f) return;
    float h1 = h;
    if (h > target) {
        *bank += (h - target) * area;
        h1 = target;
    } else if (*bank > 0.0f) {
        const float add = fminf(target - h, *bank / area);
        h1 = h + add;
        *bank -= add * area;
    }
    if (h1 != h) {
        W.h[0][idx] = h1;
        *moved += (double)h1 - (double)h;
        fine::mark_tile(W, 0, i, j);
    }
}

// The reach's sweep is sequential in the reference (each cell reads the bank
// the one before left): one thread walks it in the same order.
__global__ void k_reach(fine::SheetView W, ReachStep r, float* bank, double* books) {
    ::silt::dep_wait();
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int res = W.res;
    const float area = W.cell * W.cell;
    float b = *bank;
    double moved = 0.0;
    double inflow_m3 = 0.0;
    auto at = [&](int along, int cross) -> size_t {
        return r.along_z ? (size_t)along * res + cross : (size_t)cross * res + along;
    };
    auto row = [&](int k) { return r.positive ? k : res - 1 - k; };
    auto cell_i = [&](size_t idx) { return (int)(idx % res); };
    auto cell_j = [&](size_t idx) { return (int)(idx / res); };
    const int first_out = res - r.rows;
    for (int cross = r.c0; cross < r.c1; ++cross) {
        const size_t src = at(row(first_out - 1), cross);
        float su = W.u[0][src], sv = W.v[0][src];
        if (W.cut_pending && W.h[0][src] < 1.0e-6f) {  // the lazy dry cut of the copied cell
            su = 0.0f;
            sv = 0.0f;
        }
        const float along = fmaxf(su * r.dx + sv * r.dz, 0.0f);
        for (int k = first_out; k < res; ++k) {
            const size_t idx = at(row(k), cross);
            const float target = fmaxf(r.outlet_eta - W.bed[idx], 0.0f);
            const float h = W.h[0][idx];
            if (!isfinite(h) || target <= 0.0f) continue;
            hold_stage(W, idx, r.outlet_eta, area, &b, &moved, cell_i(idx), cell_j(idx));
            if (isfinite(su) && isfinite(sv)) {
                const float cross_v = r.along_z ? su : sv;
                W.u[0][idx] = r.along_z ? cross_v : along * r.dx;
                W.v[0][idx] = r.along_z ? along * r.dz : cross_v;
                fine::mark_tile(W, 0, cell_i(idx), cell_j(idx));
            }
        }
    }
    float deep = 0.0f;
    for (int cross = r.c0; cross < r.c1; ++cross) deep = fmaxf(deep, fmaxf(r.inlet_eta - W.bed[at(row(0), cross)], 0.0f));
    if (deep > 0.0f)
        for (int k = 0; k < r.rows; ++k)
            for (int cross = r.c0; cross < r.c1; ++cross) {
                const size_t idx = at(row(k), cross);
                const float target = fmaxf(r.inlet_eta - W.bed[idx], 0.0f);
                const float h = W.h[0][idx];
                if (!isfinite(h) || target <= 0.0f) continue;
                hold_stage(W, idx, r.inlet_eta, area, &b, &moved, cell_i(idx), cell_j(idx));
                const float speed = r.inlet_speed * sqrtf(fminf(fmaxf(W.h[0][idx] / deep, 0.0f), 1.0f));
                W.u[0][idx] = speed * r.dx;
                W.v[0][idx] = speed * r.dz;
                fine::mark_tile(W, 0, cell_i(idx), cell_j(idx));
                if (r.inflow_c > 0.0f) {
                    // The water arrives carrying its load (src/fluid_core.rs:7746-7755).
                    const float w = W.h[0][idx];
                    const float want = r.inflow_c * w;
                    const float have = r.susp[idx];
                    if (w >= 1.0e-5f && isfinite(have) && have < want) {
                        r.susp[idx] = want;
                        inflow_m3 += (double)((want - have) * area);
                    }
                }
            }
    if (inflow_m3 != 0.0) *r.entrained += inflow_m3;
    *bank = b;
    if (moved != 0.0) {
        if (W.d_acc) W.d_acc[0] += moved;
        books[4] -= moved * ((double)W.cell * (double)W.cell);
    }
}

}  // namespace

cudaError_t wave_step(const fine::SheetView& W, const WaveStep& w, cudaStream_t st) {
    const int n = (w.i1 - w.i0) * (w.j1 - w.j0);
    if (n <= 0) return cudaSuccess;
    const int blocks = (n + 255) / 256 < 296 ? (n + 255) / 256 : 296;
    ::silt::launch_dep(k_wave, dim3(blocks), dim3(256), 0, st, W, w);
    ::silt::count_launch();
    return cudaGetLastError();
}

cudaError_t reach_step(const fine::SheetView& W, const ReachStep& r, float* bank, double* books, cudaStream_t st) {
    if (r.c1 <= r.c0) return cudaSuccess;
    ::silt::launch_dep(k_reach, dim3(1), dim3(32), 0, st, W, r, bank, books);
    ::silt::count_launch();
    return cudaGetLastError();
}

}  // namespace drivers
}  // namespace silt
