// Nested 2 cm patches and their two-way coupling with the coarse window
// (x3-team/Dirty-gen src/fluid_core.rs:8152-8566 and src/fluid_core/near.rs).
//
// The host decides the geometry each step from the tire positions: patch
// origins, the fine-to-coarse axes, the held columns, the near-field columns
// and which tire shoves which grid. Those small tables go to the device in
// one copy; the kernels below then move all cell data on the device:
//
//   k_refine_lay    coarse -> fine copy of held columns, free-surface bed elsewhere,
//                   the slurry's material tables
//   k_lay_finish    empty the held coarse columns; lay the kept 10x10 residual
//                   tiles back on the patch (near_apply)
//   k_push_patches  tire shoves on every patch's velocity, pushes applied in
//                   call order; one more row of blocks ages the near-field tiles
//                   and recycles dropped slots (near_fade)
//   (sheet_window.cu k_window_step: the fine sheet step itself)
//   k_peel_patches  spray peeled off the fine water, events queued on the device
//   k_restrict      residual tiles of held columns (near_capture), then the
//                   volume- and momentum-weighted sum back into the columns
//   k_release       fine volume outside the window, booked as parked; fine depths cleared
//   k_push_cells, k_peel  the same shove and peel on the coarse grid
//
// Near-field tiles live in a device pool with a slot per coarse cell; slots
// are taken in the capture (k_restrict) and returned in the fade
// (k_push_patches, or k_near_fade without tires), so no kernel both pushes and
// pops the free stack.
#include <algorithm>
#include <array>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include <cuda_runtime.h>

#include "sheet_fine.cuh"
#include "sheet_host_math.h"
#include "sheet_math.cuh"
#include "sheet_window.cuh"
#include "sheet_park.cuh"
#include "launch_count.cuh"

namespace silt {
namespace fine {

namespace {

constexpr int MAX_PATCHES = 16;
constexpr int NEAR_POOL = 16384;
constexpr int SPRAY_CAP = 1 << 16;
constexpr float NEAR_LIFE_S = 1.5f;      // near.rs:37
constexpr float NEAR_DROP_M = 1.0e-5f;   // near.rs:39
constexpr float NEAR_FILM_M = 1.0e-6f;   // near.rs:41

thread_local char g_err[200] = "";

#define FCK(call)                                                                     \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            snprintf(g_err, sizeof g_err, "%s: %s", #call, cudaGetErrorString(e_));   \
            return SILT_ECUDA;                                                        \
        }                                                                             \
    } while (0)

}  // namespace

// Device planes of one patch.
struct PatchState {
    float* base = nullptr;
    float *water, *slurry, *uw, *vw, *us, *vs, *bed, *bed_slurry, *moisture;
    float *nu_s, *mob_s, *damp_s;  // slurry material of each cell, from grain and moisture at lay time
    uint8_t* grain;
    uint8_t* solid;       // the patch's wall mask
    float* win[2];        // [layer]: the window engine's scratch planes
    // Host geometry of the current step.
    float origin[2] = {0, 0};
    std::vector<int16_t> col, row;
};

struct PatchRef {
    float *water, *slurry, *uw, *vw, *us, *vs, *bed, *bed_slurry, *moisture;
    float *nu_s, *mob_s, *damp_s;
    uint8_t* grain;
    uint8_t* solid;
    const int16_t* col;
    const int16_t* row;
    float ox, oz;
};

struct NearCol {
    int cidx, patch, i0, j0, inner, pad;
};

struct RestrictEntry {
    int cidx, cnt, held, seg_off, seg_n, pad;
};

struct Segment {
    int patch, i0, i1, j0, j1, pad;
};

struct PushJob {
    float x, z, fx, fz, radius, width, speed, slip;
    int span_i0, span_i1, span_j0, span_j1;  // half-open index spans (index_span)
    int index;                               // position in the call order
    int pad[3];
};

struct SprayRec {
    float x, y, z, vx, vy, vz, volume;
    int kind;
    unsigned long long key;
};

struct NearMeta {
    int state;   // 0 free, 1 live, 2 released (back to the free stack at the next fade)
    int key;     // coarse cell index
    int fresh;
    float idle_s;
    float peak;
    int pad[3];
};

struct Impl {
    int res = 0;
    park::Table park;                 // parked cells by world key (allocated on first use)
    int8_t* owner = nullptr;          // per coarse cell: patch that holds it, -1 none
    std::vector<int8_t> h_owner;      // host mirror
    std::vector<int> held_now;        // coarse cells held by the last laid patches
    void* host = nullptr;             // HostState: the step plan and its table buffers
    // Near-field pool.
    int* slot_map = nullptr;          // per coarse cell
    float* pool = nullptr;            // NEAR_POOL x 4 x sub^2
    NearMeta* meta = nullptr;
    int* free_stack = nullptr;
    int* counters = nullptr;          // [0] free top, [1] live tiles, [2] overflow, [3] spray count
    bool near_maybe = false;
    bool spray_dirty = false;         // the spray count may be non-zero (a step with tires ran)
    // Spray.
    SprayRec* spray = nullptr;
    double* d_books = nullptr;        // [0] spray m3, [1] parked water m3, [2] parked slurry m3, [3] dry cut m3,
                                      // [4] river reach bank m3 (FP64 twin of the reference's f32 bank),
                                      // [5] eroded bed m3, [6] transport rounding m3, [7..10] the
                                      // tracers' entrained, settled suspended, stirred and settled silt,
                                      // [11] parked suspended, [12] parked silt
    double* h_books = nullptr;
    int* h_counters = nullptr;
};

static Impl& I(Patches& P) { return *reinterpret_cast<Impl*>(P.impl); }

// ------------------------------------------------------------------ kernels

__global__ void k_scatter_owner(int8_t* owner, const int* idx, const int8_t* val, int n) {
    ::silt::dep_wait();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) owner[idx[k]] = val[k];
}

// refine (src/fluid_core.rs:8358-8460), the copy into fine cell f of patch p.
__device__ __forceinline__ void refine_cell(const PatchRef& R, int p, int f, int fres, const SheetView& W,
                                            const int8_t* owner) {
    R.water[f] = 0.0f;
    R.slurry[f] = 0.0f;
    R.uw[f] = 0.0f;
    R.vw[f] = 0.0f;
    R.us[f] = 0.0f;
    R.vs[f] = 0.0f;
    const int ci = R.col[f % fres], cj = R.row[f / fres];
    if (ci >= 0 && cj >= 0) {
        const size_t c = (size_t)cj * W.res + ci;
        R.moisture[f] = W.moisture[c];
        R.grain[f] = W.grain[c];
    }
    // The slurry's material laws once per step here, spread over the whole
    // GPU, instead of once per cell and substep inside the patch's step.
    const float nu = dynamic_viscosity(R.grain[f], R.moisture[f]);
    R.nu_s[f] = nu;
    R.mob_s[f] = sheet_mobility_for(nu);
    R.damp_s[f] = sheet_damp(nu);
    if (ci < 0 || cj < 0) return;
    const size_t c = (size_t)cj * W.res + ci;
    if (owner[c] != p) {
        R.bed[f] = W.bed[c] + W.h[0][c];
        R.bed_slurry[f] = W.bed[c] + W.h[1][c];
        return;
    }
    R.bed[f] = W.bed[c];
    R.bed_slurry[f] = W.bed[c];
    const float hw = W.h[0][c], hs = W.h[1][c];
    R.water[f] = hw;
    R.slurry[f] = hs;
    // A coarse cell still waiting for the previous dry cut carries no velocity.
    const bool cw = W.cut_pending && hw < 1.0e-6f, cs = W.cut_pending && hs < 1.0e-6f;
    R.uw[f] = cw ? 0.0f : W.u[0][c];
    R.vw[f] = cw ? 0.0f : W.v[0][c];
    R.us[f] = cs ? 0.0f : W.u[1][c];
    R.vs[f] = cs ? 0.0f : W.v[1][c];
}

__global__ void k_refine_lay(const PatchRef* refs, int np, int fres, SheetView W, const int8_t* owner,
                             int* spray_count) {
    ::silt::dep_wait();
    const size_t fn = (size_t)fres * fres;
    if (blockIdx.x == 0 && threadIdx.x == 0) *spray_count = 0;  // this step's spray events start here
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < fn * np; k += (size_t)gridDim.x * blockDim.x)
        refine_cell(refs[k / fn], (int)(k / fn), (int)(k % fn), fres, W, owner);
}

__device__ __forceinline__ float tile_left(float idle) { return idle <= 0.0f ? 1.0f : exp_rn(-idle / NEAR_LIFE_S); }

// near.rs:139-148 floor_scale on one residual, given its lowest value
// (the minimum of 0 and every residual).
__device__ float floor_scale_min(float base, float low) {
    if (low >= 0.0f || base + low >= 0.0f) return 1.0f;
    if (base <= 0.0f) return 0.0f;
    return rclamp(base / -low, 0.0f, 1.0f);
}

// near_apply (near.rs:276-308): one block per held near column.
__device__ void near_apply_col(int q, const PatchRef* refs, int fres, int sub, const NearCol* cols, int ncol,
                               const int* slot_map, const float* pool, const NearMeta* meta) {
    if (q >= ncol) return;
    const NearCol C = cols[q];
    const int slot = slot_map[C.cidx];
    if (slot < 0 || meta[slot].state != 1) return;
    const int n2 = sub * sub;
    const float* tw = pool + (size_t)slot * 4 * n2;
    const float* ts = tw + n2;
    const float* tuw = ts + n2;
    const float* tvw = tuw + n2;
    const PatchRef& R = refs[C.patch];
    __shared__ float scale[2];
    const int f0 = C.j0 * fres + C.i0;
    const float bw = R.water[f0], bs = R.slurry[f0];
    const float left = tile_left(meta[slot].idle_s);
    if (threadIdx.x < 32) {
        // floor_scale's minimum residual of each layer over the first warp (a
        // minimum: any order gives the same value).
        float lw = 0.0f, ls = 0.0f;
        for (int k = threadIdx.x; k < n2; k += 32) {
            lw = fminf(lw, tw[k]);
            ls = fminf(ls, ts[k]);
        }
        for (int o = 16; o > 0; o >>= 1) {
            lw = fminf(lw, __shfl_down_sync(0xffffffffu, lw, o));
            ls = fminf(ls, __shfl_down_sync(0xffffffffu, ls, o));
        }
        if (threadIdx.x == 0) {
            scale[0] = left * floor_scale_min(bw / fmaxf(left, 1.0e-6f), lw);
            scale[1] = left * floor_scale_min(bs / fmaxf(left, 1.0e-6f), ls);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n2; k += blockDim.x) {
        const int b = k / sub, a = k % sub;
        const int f = (C.j0 + b) * fres + C.i0 + a;
        float w = fmaxf(bw + scale[0] * tw[k], 0.0f);
        float s = fmaxf(bs + scale[1] * ts[k], 0.0f);
        R.water[f] = w;
        R.slurry[f] = s;
        if (C.inner && w > NEAR_FILM_M) {
            R.uw[f] += left * tuw[k];
            R.vw[f] += left * tvw[k];
        }
    }
}

// The end of the lay in one launch: blocks [0, zero_blocks) empty the held
// coarse columns, the rest apply the near-field residual of one held column
// each (independent writes: coarse cells, fine cells).
__global__ void k_lay_finish(SheetView W, const int* held, int n_held, int zero_blocks, const PatchRef* refs,
                             int fres, int sub, const NearCol* cols, int ncol, const int* slot_map, const float* pool,
                             const NearMeta* meta) {
    ::silt::dep_wait();
    if ((int)blockIdx.x < zero_blocks) {
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_held; k += zero_blocks * blockDim.x) {
            const size_t c = held[k];
            W.h[0][c] = 0.0f;
            W.h[1][c] = 0.0f;
            W.u[0][c] = 0.0f;
            W.v[0][c] = 0.0f;
            W.u[1][c] = 0.0f;
            W.v[1][c] = 0.0f;
        }
        return;
    }
    near_apply_col((int)blockIdx.x - zero_blocks, refs, fres, sub, cols, ncol, slot_map, pool, meta);
}

// near_fade (near.rs:311-325) and slot recycling.
__device__ void near_fade_slot(int s, NearMeta* meta, int* slot_map, int* free_stack, int* counters, float dt) {
    NearMeta& M = meta[s];
    if (M.state == 1) {
        if (M.fresh) {
            M.fresh = 0;
        } else {
            M.idle_s += dt;
            if (!(M.peak * tile_left(M.idle_s) > NEAR_DROP_M)) {
                slot_map[M.key] = -1;
                M.state = 2;
                atomicSub(&counters[1], 1);
            }
        }
    }
    if (M.state == 2) {
        int top = atomicAdd(&counters[0], 1);
        free_stack[top] = s;
        M.state = 0;
    }
}

__global__ void k_near_fade(NearMeta* meta, int* slot_map, int* free_stack, int* counters, float dt) {
    ::silt::dep_wait();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < NEAR_POOL) near_fade_slot(s, meta, slot_map, free_stack, counters, dt);
}

// push_on (src/fluid_core.rs:8169-8239); every thread owns one cell of the
// pushes' joint span and applies the pushes in call order.
__device__ void push_cell(float* w, float* s, float* uw, float* vw, float* us, float* vs, int res, float cell,
                          float ox, float oz, const PushJob* jobs, int njobs, int i, int j) {
    const size_t idx = (size_t)j * res + i;
    for (int q = 0; q < njobs; ++q) {
        const PushJob p = jobs[q];
        if (i < p.span_i0 || i >= p.span_i1 || j < p.span_j0 || j >= p.span_j1) continue;
        float fx = p.fx, fz = p.fz;
        float len = fmaxf(sqrtf(fx * fx + fz * fz), 1.0e-4f);
        fx = fx / len;
        fz = fz / len;
        const float rx = fz, rz = -fx;
        const float speed = fmaxf(p.speed, 0.0f);
        const float x = ox + ((float)i + 0.5f) * cell;
        const float z = oz + ((float)j + 0.5f) * cell;
        const float dx = x - p.x, dz = z - p.z;
        const float along = dx * fx + dz * fz;
        const float lat = dx * rx + dz * rz;
        if (fabsf(lat) > p.width * 0.65f + cell) continue;
        if (along < -p.radius * 1.4f || along > p.radius * 1.1f) continue;
        const float flank = rclamp(fabsf(lat) / (p.width * 0.65f + cell), 0.0f, 1.0f);
        const float shove = fmaxf(speed, 0.4f) * (1.0f - flank * flank);
        const float sg = isnan(lat) ? lat : (signbit(lat) ? -1.0f : 1.0f);  // f32::signum
        if (w[idx] > 0.004f) {
            uw[idx] += fx * shove * 0.85f;
            vw[idx] += fz * shove * 0.85f;
            uw[idx] += rx * sg * shove * 0.18f * flank;
            vw[idx] += rz * sg * shove * 0.18f * flank;
        }
        if (s[idx] > 0.004f) {
            const float fore = along > 0.0f ? 1.0f : 0.72f;
            us[idx] += fx * shove * fore;
            vs[idx] += fz * shove * fore;
            us[idx] += rx * sg * shove * 0.28f * flank;
            vs[idx] += rz * sg * shove * 0.28f * flank;
        }
    }
}

__global__ void k_push_cells(float* w, float* s, float* uw, float* vw, float* us, float* vs, int res, float cell,
                             float ox, float oz, const PushJob* jobs, int njobs, int bi0, int bj0, int bw, int bh) {
    ::silt::dep_wait();
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < bw * bh; k += gridDim.x * blockDim.x)
        push_cell(w, s, uw, vw, us, vs, res, cell, ox, oz, jobs, njobs, bi0 + k % bw, bj0 + k / bw);
}

// One patch's shove or peel jobs within a launch over all patches (blockIdx.y).
struct JobGroup {
    int patch;          // PatchRef index
    float ox, oz;       // patch origin
    int job_off;        // byte offset of its PushJob list in the step table
    int njobs, i0, j0, w, h;
};

// The wall mask of every patch (blockIdx.y), src/fluid_core.rs:7288-7360
// with fine = true: the patch's water over its bed at its origin.
__global__ void k_patch_walls(const PatchRef* refs, int fres, float fcell, const walls::SolidGeom* geoms, int n) {
    ::silt::dep_wait();
    const PatchRef& r = refs[blockIdx.y];
    const int cells = fres * fres;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += gridDim.x * blockDim.x)
        r.solid[c] = walls::mask_value(geoms, n, c % fres, c / fres, fres, fcell, r.ox, r.oz, r.water, r.bed);
}

// The shoves of every patch (blockIdx.y = group). With `fade`, one more row
// of blocks runs near_fade over the tile pool (independent of the shoves).
__global__ void k_push_patches(const PatchRef* refs, const char* tab, const JobGroup* groups, int ngroups, int fres,
                               float fcell, int fade, NearMeta* meta, int* slot_map, int* free_stack, int* counters,
                               float dt) {
    ::silt::dep_wait();
    if ((int)blockIdx.y == ngroups) {
        if (fade)
            for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < NEAR_POOL; q += gridDim.x * blockDim.x)
                near_fade_slot(q, meta, slot_map, free_stack, counters, dt);
        return;
    }
    const JobGroup G = groups[blockIdx.y];
    const PatchRef& R = refs[G.patch];
    const PushJob* jobs = reinterpret_cast<const PushJob*>(tab + G.job_off);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < G.w * G.h; k += gridDim.x * blockDim.x)
        push_cell(R.water, R.slurry, R.uw, R.vw, R.us, R.vs, fres, fcell, G.ox, G.oz, jobs, G.njobs,
                  G.i0 + k % G.w, G.j0 + k / G.w);
}

// peel_spray (src/fluid_core.rs:8241-8314). Events carry a sort key that
// restores the reference's order (phase, patch, push, row, column).
__device__ void peel_cell(float* w, const float* uw, const float* vw, int res, float cell, float ox, float oz,
                          const PushJob* jobs, int njobs, int i, int j, const int8_t* owner, int coarse_res, float cox,
                          float coz, float coarse_cell, int phase, int patch, SprayRec* out, int* counters,
                          double* books, double* ledger_depth) {
    const size_t idx = (size_t)j * res + i;
    const float area = cell * cell;
    for (int q = 0; q < njobs; ++q) {
        const PushJob p = jobs[q];
        if (p.speed < 0.8f) continue;
        if (i < p.span_i0 || i >= p.span_i1 || j < p.span_j0 || j >= p.span_j1) continue;
        const float x = ox + ((float)i + 0.5f) * cell;
        const float z = oz + ((float)j + 0.5f) * cell;
        if (owner) {  // skip the held columns (coarse_held, src/fluid_core.rs:9664-9672)
            float ci = floorf((x - cox) / coarse_cell), cj = floorf((z - coz) / coarse_cell);
            if (!(ci < 0.0f || cj < 0.0f)) {
                int ii = (int)ci, jj = (int)cj;
                if (ii < coarse_res && jj < coarse_res && owner[(size_t)jj * coarse_res + ii] >= 0) continue;
            }
        }
        const float dx = x - p.x, dz = z - p.z;
        if (dx * dx + dz * dz > (p.radius * 1.3f) * (p.radius * 1.3f)) continue;
        if (w[idx] < 0.01f) continue;
        const float take = fminf(w[idx] * 0.04f, 0.004f);
        if (take * area < 1.0e-6f) continue;
        const float before = w[idx], after = before - take;
        w[idx] = after;
        int slot = atomicAdd(&counters[3], 1);
        // The spray book takes the cell's actual change, so the FP64 books close.
        atomicAdd(&books[0], ((double)before - (double)after) * ((double)cell * (double)cell));
        // The depth sum follows the cell's actual (rounded) change.
        if (ledger_depth) atomicAdd(ledger_depth, (double)after - (double)before);
        if (slot < SPRAY_CAP) {
            SprayRec r;
            r.x = x;
            r.y = 0.35f;
            r.z = z;
            r.vx = uw[idx] * 0.3f;
            r.vy = 1.4f + p.speed * 0.25f;
            r.vz = vw[idx] * 0.3f;
            r.volume = take * area;
            r.kind = 0;
            r.key = ((unsigned long long)phase << 60) | ((unsigned long long)patch << 54) |
                    ((unsigned long long)p.index << 44) | ((unsigned long long)j << 22) | (unsigned long long)i;
            out[slot] = r;
        }
    }
}

__global__ void k_peel(float* w, const float* uw, const float* vw, int res, float cell, float ox, float oz,
                       const PushJob* jobs, int njobs, int bi0, int bj0, int bw, int bh, const int8_t* owner,
                       int coarse_res, float cox, float coz, float coarse_cell, int phase, int patch, SprayRec* out,
                       int* counters, double* books, double* ledger_depth) {
    ::silt::dep_wait();
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < bw * bh; k += gridDim.x * blockDim.x)
        peel_cell(w, uw, vw, res, cell, ox, oz, jobs, njobs, bi0 + k % bw, bj0 + k / bw, owner, coarse_res, cox, coz,
                  coarse_cell, phase, patch, out, counters, books, ledger_depth);
}

// The fine peel of every patch in one launch (phase 0: no held-column test, no coarse ledger).
__global__ void k_peel_patches(const PatchRef* refs, const char* tab, const JobGroup* groups, int fres, float fcell,
                               SprayRec* out, int* counters, double* books) {
    ::silt::dep_wait();
    const JobGroup G = groups[blockIdx.y];
    const PatchRef& R = refs[G.patch];
    const PushJob* jobs = reinterpret_cast<const PushJob*>(tab + G.job_off);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < G.w * G.h; k += gridDim.x * blockDim.x)
        peel_cell(R.water, R.uw, R.vw, fres, fcell, G.ox, G.oz, jobs, G.njobs, G.i0 + k % G.w, G.j0 + k / G.w,
                  nullptr, 0, 0.0f, 0.0f, 1.0f, 0, G.patch, out, counters, books, nullptr);
}

// near_capture (near.rs:199-273): one block of 128 threads per held near column.
__device__ void near_capture_col(int q, const PatchRef* refs, int fres, int sub, const NearCol* cols, int ncol,
                                 int* slot_map, float* pool, NearMeta* meta, int* free_stack, int* counters) {
    if (q >= ncol) return;
    const NearCol C = cols[q];
    const PatchRef& R = refs[C.patch];
    const int n2 = sub * sub;
    __shared__ float bw_[1024], bs_[1024], bu_[1024], bv_[1024];
    __shared__ int decision;   // 0 remove, 1 keep
    __shared__ int slot_s;
    __shared__ float mw_s, ms_s, uu_s, vv_s, sw_s;
    __shared__ double mean_w, mean_s;
    for (int k = threadIdx.x; k < n2; k += blockDim.x) {
        const int f = (C.j0 + k / sub) * fres + C.i0 + k % sub;
        bw_[k] = R.water[f];
        bs_[k] = R.slurry[f];
        bu_[k] = R.uw[f];
        bv_[k] = R.vw[f];
    }
    __syncthreads();
    // The column's reductions, each in the reference's order, spread over the
    // first warp: per-row sums on `sub` lanes, then the rest on their own lanes.
    __shared__ float row_w[32], row_s[32];
    __shared__ float sw_sh, ss_sh, mu_sh, mv_sh, peak_sh;
    __shared__ double sum_w_sh, sum_s_sh;
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        if (lane < sub) {
            // Each row of `sub` summed from -0.0 (near.rs column sums).
            float rw = -0.0f, rs = -0.0f;
            for (int a = 0; a < sub; ++a) {
                rw += bw_[lane * sub + a];
                rs += bs_[lane * sub + a];
            }
            row_w[lane] = rw;
            row_s[lane] = rs;
        }
        __syncwarp();
        if (lane < 2) {  // rows added in order
            const float* rows = lane == 0 ? row_w : row_s;
            float acc = 0.0f;
            for (int b = 0; b < sub; ++b) acc += rows[b];
            if (lane == 0) sw_sh = acc; else ss_sh = acc;
        }
        __syncwarp();
        const float sw = sw_sh, ss = ss_sh;
        const float nn = (float)n2;
        const float mw = sw / nn, ms = ss / nn;
        // abs_peak (near.rs:128-137): the largest deviation over whole groups
        // of four, in any order (a maximum).
        float pk = 0.0f;
        const int whole = (n2 / 4) * 4;
        for (int k = lane; k < whole; k += 32) {
            float a = fabsf(bw_[k] - mw);
            pk = a > pk ? a : pk;
            float b2 = fabsf(bs_[k] - ms);
            pk = b2 > pk ? b2 : pk;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float x = __shfl_down_sync(0xffffffffu, pk, o);
            pk = x > pk ? x : pk;
        }
        if (lane == 0) peak_sh = pk;
        // recentre (near.rs:118-125): f64 sums of the residual, in order.
        if (lane == 1 || lane == 2) {
            const float* b = lane == 1 ? bw_ : bs_;
            const float m = lane == 1 ? mw : ms;
            double acc = 0.0;
            for (int k = 0; k < n2; ++k) acc += (double)(b[k] - m);
            if (lane == 1) sum_w_sh = acc; else sum_s_sh = acc;
        }
        if (lane == 3 || lane == 4) {  // momentum of the water, in order
            const float* vel = lane == 3 ? bu_ : bv_;
            float acc = 0.0f;
            if (C.inner && sw > 1.0e-10f)
                for (int k = 0; k < n2; ++k) acc += bw_[k] * vel[k];
            if (lane == 3) mu_sh = acc; else mv_sh = acc;
        }
        __syncwarp();
    }
    if (threadIdx.x == 0) {
        const float sw = sw_sh, ss = ss_sh;
        int keep = 1;
        if (sw <= 0.0f && ss <= 0.0f) keep = 0;
        const float nn = (float)n2;
        const float mw = sw / nn, ms = ss / nn;
        const float peak = peak_sh;
        if (keep && peak <= NEAR_DROP_M && !C.inner) keep = 0;
        mean_w = sum_w_sh / (double)n2;
        mean_s = sum_s_sh / (double)n2;
        const float mu = mu_sh, mv = mv_sh;
        uu_s = mu / sw;
        vv_s = mv / sw;
        mw_s = mw;
        ms_s = ms;
        sw_s = sw;
        int slot = slot_map[C.cidx];
        if (!keep) {
            if (slot >= 0) {
                meta[slot].state = 2;
                slot_map[C.cidx] = -1;
                atomicSub(&counters[1], 1);
            }
            slot = -1;
        } else if (slot < 0) {
            int top = atomicSub(&counters[0], 1);
            if (top <= 0) {
                atomicAdd(&counters[0], 1);
                atomicAdd(&counters[2], 1);
                keep = 0;
            } else {
                slot = free_stack[top - 1];
                slot_map[C.cidx] = slot;
                meta[slot].state = 1;
                meta[slot].key = C.cidx;
                atomicAdd(&counters[1], 1);
            }
        }
        decision = keep;
        slot_s = slot;
        if (keep) {
            meta[slot].peak = peak;
            meta[slot].idle_s = 0.0f;
            meta[slot].fresh = 1;
        }
    }
    __syncthreads();
    if (!decision) return;
    float* tw = pool + (size_t)slot_s * 4 * n2;
    float* ts = tw + n2;
    float* tuw = ts + n2;
    float* tvw = tuw + n2;
    const float mwf = (float)mean_w, msf = (float)mean_s;
    const bool vel = C.inner && sw_s > 1.0e-10f;
    for (int k = threadIdx.x; k < n2; k += blockDim.x) {
        tw[k] = (bw_[k] - mw_s) - mwf;
        ts[k] = (bs_[k] - ms_s) - msf;
        if (vel) {
            const bool wet = bw_[k] > NEAR_FILM_M;
            tuw[k] = wet ? bu_[k] - uu_s : 0.0f;
            tvw[k] = wet ? bv_[k] - vv_s : 0.0f;
        } else {
            tuw[k] = 0.0f;
            tvw[k] = 0.0f;
        }
    }
}

__device__ void restrict_column(const PatchRef* refs, int fres, const SheetView& W, const RestrictEntry& E,
                                const Segment* segs, float fine_area, float coarse_area, int lane) {
    float aw = 0.0f, as = 0.0f, auw = 0.0f, avw = 0.0f, aus = 0.0f, avs = 0.0f;
    for (int sgi = 0; sgi < E.seg_n; ++sgi) {
        const Segment S = segs[E.seg_off + sgi];
        const PatchRef& R = refs[S.patch];
        const int ni = S.i1 - S.i0 + 1, nc = ni * (S.j1 - S.j0 + 1);
        constexpr int G = 4;  // chunks loaded together before they are summed
        for (int g0 = 0; g0 < nc; g0 += 32 * G) {
            float pw[G], ps[G], puw[G], pvw[G], pus[G], pvs[G];
            unsigned takes[G];
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const int c = g0 + 32 * q + lane;
                pw[q] = ps[q] = puw[q] = pvw[q] = pus[q] = pvs[q] = 0.0f;
                int take = 0;
                if (c < nc) {
                    const int f = (S.j0 + c / ni) * fres + S.i0 + c % ni;
                    const float fw = R.water[f], fs = R.slurry[f];
                    if (!(fw == 0.0f && fs == 0.0f)) {
                        take = 1;
                        pw[q] = fw * fine_area;
                        ps[q] = fs * fine_area;
                        puw[q] = R.uw[f] * fw * fine_area;
                        pvw[q] = R.vw[f] * fw * fine_area;
                        pus[q] = R.us[f] * fs * fine_area;
                        pvs[q] = R.vs[f] * fs * fine_area;
                    }
                }
                takes[q] = __ballot_sync(0xffffffffu, take);
            }
#pragma unroll
            for (int q = 0; q < G; ++q) {
                const int m = min(32, nc - (g0 + 32 * q));
                for (int b = 0; b < m; ++b) {
                    const float xw = __shfl_sync(0xffffffffu, pw[q], b), xs = __shfl_sync(0xffffffffu, ps[q], b);
                    const float xuw = __shfl_sync(0xffffffffu, puw[q], b), xvw = __shfl_sync(0xffffffffu, pvw[q], b);
                    const float xus = __shfl_sync(0xffffffffu, pus[q], b), xvs = __shfl_sync(0xffffffffu, pvs[q], b);
                    if ((takes[q] >> b) & 1u) {
                        aw += xw;
                        as += xs;
                        auw += xuw;
                        avw += xvw;
                        aus += xus;
                        avs += xvs;
                    }
                }
            }
        }
    }
    if (lane != 0) return;
    const size_t idx = E.cidx;
    const float w = aw / coarse_area, s = as / coarse_area;
    mark_tile(W, 0, (int)(idx % W.res), (int)(idx / W.res));
    mark_tile(W, 1, (int)(idx % W.res), (int)(idx / W.res));
    // A column the patch does not hold keeps its depth and gains what flowed
    // onto its fine cells. For patches that are whole multiples of the coarse
    // cell every touched column is fully covered and this is the reference's
    // `!held && cnt >= full` branch; a partly covered rim column (64-cell
    // patches) must not lose the coarse depth it kept.
    if (!E.held) {
        if (w <= 0.0f && s <= 0.0f) return;
        const float old_w = W.h[0][idx], old_s = W.h[1][idx];
        const float new_w = old_w + w, new_s = old_s + s;
        // Pending dry cut: a cell under eps holds no velocity.
        if (W.cut_pending && old_w < 1.0e-6f) W.u[0][idx] = W.v[0][idx] = 0.0f;
        if (W.cut_pending && old_s < 1.0e-6f) W.u[1][idx] = W.v[1][idx] = 0.0f;
        if (new_w > 1.0e-6f) {
            W.u[0][idx] = (old_w * W.u[0][idx] * coarse_area + auw) / (new_w * coarse_area);
            W.v[0][idx] = (old_w * W.v[0][idx] * coarse_area + avw) / (new_w * coarse_area);
        }
        if (new_s > 1.0e-6f) {
            W.u[1][idx] = (old_s * W.u[1][idx] * coarse_area + aus) / (new_s * coarse_area);
            W.v[1][idx] = (old_s * W.v[1][idx] * coarse_area + avs) / (new_s * coarse_area);
        }
        W.h[0][idx] = new_w;
        W.h[1][idx] = new_s;
        return;
    }
    W.h[0][idx] = w;
    W.h[1][idx] = s;
    if (w > 1.0e-6f) {
        W.u[0][idx] = auw / (w * coarse_area);
        W.v[0][idx] = avw / (w * coarse_area);
    }
    if (s > 1.0e-6f) {
        W.u[1][idx] = aus / (s * coarse_area);
        W.v[1][idx] = avs / (s * coarse_area);
    }
}

// restrict_fine (src/fluid_core.rs:8462-8555): one warp per touched coarse
// column. The lanes load 32 fine cells at a time and form their products in
// parallel; the six sums then take the products one by one in the
// reference's raster order (every lane adds the same sequence).
// Blocks [0, ncap) capture the near-field residual of one held column each
// (with `ncap` = 0 when the near field is off); the rest restrict, a warp per
// touched coarse column. Both read the fine cells after the peel and write
// disjoint state (the tile pool, the coarse columns). 128 threads per block.
__global__ void k_restrict(const PatchRef* refs, int fres, int sub, SheetView W, const RestrictEntry* ents, int nent,
                           const Segment* segs, float fine_area, float coarse_area, const NearCol* cols, int ncap,
                           int* slot_map, float* pool, NearMeta* meta, int* free_stack, int* counters) {
    ::silt::dep_wait();
    if ((int)blockIdx.x < ncap) {
        near_capture_col(blockIdx.x, refs, fres, sub, cols, ncap, slot_map, pool, meta, free_stack, counters);
        return;
    }
    const int lane = threadIdx.x & 31;
    const int nb = (int)gridDim.x - ncap;
    const int warps = (int)((nb * (size_t)blockDim.x) >> 5);
    for (int q = (int)((((int)blockIdx.x - ncap) * (size_t)blockDim.x + threadIdx.x) >> 5); q < nent; q += warps)
        restrict_column(refs, fres, W, ents[q], segs, fine_area, coarse_area, lane);
}

// After the restrict: fine cells outside the coarse window have their volume
// parked (src/fluid_core.rs:8476-8484), and every fine depth is released.
// Empties the patches. With `park`, fine cells outside the window add their
// depth to the parked slot of the coarse world cell under them
// (src/fluid_core.rs:8484-8487: water * fine_area / coarse_area), and their
// volume to the parked books.
__device__ void release_cells(const PatchRef* refs, int np, int fres, float fcell, float ccell, double* books,
                              int park, park::Table T, size_t k0, size_t stride) {
    const size_t fn = (size_t)fres * fres;
    const float fine_area = fcell * fcell, coarse_area = ccell * ccell;
    double pw = 0.0, ps = 0.0;
    for (size_t k = k0; k < fn * np; k += stride) {
        const PatchRef& R = refs[k / fn];
        const int f = (int)(k % fn);
        if (park && !(R.col[f % fres] >= 0 && R.row[f / fres] >= 0)) {
            pw += (double)R.water[f] * fine_area;
            ps += (double)R.slurry[f] * fine_area;
            if (T.cap && (R.water[f] != 0.0f || R.slurry[f] != 0.0f)) {
                const float x = R.ox + ((float)(f % fres) + 0.5f) * fcell;
                const float z = R.oz + ((float)(f / fres) + 0.5f) * fcell;
                bool fresh = false;
                const int s = park::find_or_insert(T, park::key_of(park::world_axis(x, ccell), park::world_axis(z, ccell)),
                                                   &fresh);
                if (s >= 0) {
                    atomicAdd(&T.vals[(size_t)s * park::NVAL + 0], R.water[f] * fine_area / coarse_area);
                    atomicAdd(&T.vals[(size_t)s * park::NVAL + 1], R.slurry[f] * fine_area / coarse_area);
                }
            }
        }
        R.water[f] = 0.0f;
        R.slurry[f] = 0.0f;
    }
    for (int o = 16; o > 0; o >>= 1) {
        pw += __shfl_down_sync(0xffffffffu, pw, o);
        ps += __shfl_down_sync(0xffffffffu, ps, o);
    }
    if ((threadIdx.x & 31) == 0 && (pw != 0.0 || ps != 0.0)) {
        atomicAdd(&books[1], pw);
        atomicAdd(&books[2], ps);
    }
}

__global__ void k_release(const PatchRef* refs, int np, int fres, float fcell, float ccell, double* books, int park,
                          park::Table T) {
    ::silt::dep_wait();
    release_cells(refs, np, fres, fcell, ccell, books, park, T, blockIdx.x * (size_t)blockDim.x + threadIdx.x,
                  (size_t)gridDim.x * blockDim.x);
}

// A move of the window by (di, dj) cells: near-field tiles follow their
// coarse cells; tiles whose cell leaves the window (all of them when the
// window jumps) are released (their residual sums to zero, so no volume
// goes with them).
__global__ void k_near_unmap(int* slot_map, size_t n) {
    ::silt::dep_wait();
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        slot_map[c] = -1;
}

__global__ void k_near_move(NearMeta* meta, int* slot_map, int* counters, int res, int di, int dj, int keep) {
    ::silt::dep_wait();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= NEAR_POOL) return;
    NearMeta& M = meta[s];
    if (M.state != 1) return;
    const int i = M.key % res - di, j = M.key / res - dj;
    if (keep && i >= 0 && j >= 0 && i < res && j < res) {
        M.key = j * res + i;
        slot_map[M.key] = s;
    } else {
        M.state = 2;  // back to the free stack at the next fade
        atomicSub(&counters[1], 1);
    }
}

__global__ void k_init_pool(NearMeta* meta, int* free_stack, int* slot_map, size_t ncells, int* counters) {
    ::silt::dep_wait();
    size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k < NEAR_POOL) {
        meta[k].state = 0;
        free_stack[k] = NEAR_POOL - 1 - (int)k;
    }
    for (size_t c = k; c < ncells; c += (size_t)gridDim.x * blockDim.x) slot_map[c] = -1;
    if (k == 0) {
        counters[0] = NEAR_POOL;
        counters[1] = 0;
        counters[2] = 0;
        counters[3] = 0;
    }
}

// ------------------------------------------------------------------- host side

namespace {

std::pair<int, int> index_span(float origin, float cell, int res, float center, float reach) {
    if (!(cell > 0.0f) || res == 0) return {0, 0};
    float lo = std::fmax(std::floor((center - reach - origin) / cell - 1.0f), 0.0f);
    float hi = std::fmax(std::ceil((center + reach - origin) / cell + 2.0f), 0.0f);
    auto to_i = [](float v) { return v > 0.0f ? (v >= 2.0e9f ? 2000000000 : (int)v) : 0; };
    int l = std::min(to_i(lo), res);
    int h = std::max(std::min(to_i(hi), res), l);
    return {l, h};
}

float dist2_segment(float px, float pz, float ax, float az, float bx, float bz) {
    float abx = bx - ax, abz = bz - az;
    float ab2 = abx * abx + abz * abz;
    float t = ab2 < 1.0e-8f ? 0.0f : host::rclamp(((px - ax) * abx + (pz - az) * abz) / ab2, 0.0f, 1.0f);
    float dx = px - (ax + abx * t), dz = pz - (az + abz * t);
    return dx * dx + dz * dz;
}

// near_tire_zone (src/fluid_core.rs:9624-9640).
bool near_tire_zone(const std::vector<silt_tire_push>& ps, float x, float z, float r2) {
    for (const auto& p : ps) {
        float dx = x - p.x, dz = z - p.z;
        if (dx * dx + dz * dz <= r2) return true;
    }
    for (size_t i = 0; i < ps.size(); ++i)
        for (size_t j = i + 1; j < ps.size(); ++j) {
            if (std::fabs(ps[i].x - ps[j].x) >= 0.45f) continue;
            if (dist2_segment(x, z, ps[i].x, ps[i].z, ps[j].x, ps[j].z) <= r2) return true;
        }
    return false;
}

// coarse_axis (src/fluid_core.rs:9546-9557).
long coarse_axis(float origin, float cell, int res, float p) {
    float i = std::floor((p - origin) / cell);
    if (i < 0.0f) return -1;
    long ii = (long)i;
    return ii >= res ? -1 : ii;
}

struct Table {
    std::vector<char> buf;
    template <class T>
    size_t put(const T* p, size_t n) {
        size_t off = (buf.size() + 255) & ~size_t(255);
        buf.resize(off + std::max<size_t>(n, 1) * sizeof(T));
        if (n) memcpy(buf.data() + off, p, n * sizeof(T));
        return off;
    }
};

int launch_blocks(size_t n, int per = 256) {
    return (int)std::max<size_t>(1, std::min<size_t>((n + per - 1) / per, 148 * 8));
}

PushJob make_job(const silt_tire_push& p, int index, float origin_x, float origin_z, float cell, int res,
                 float reach) {
    PushJob J;
    J.x = p.x;
    J.z = p.z;
    J.fx = p.forward_x;
    J.fz = p.forward_z;
    J.radius = p.radius;
    J.width = p.width;
    J.speed = p.speed;
    J.slip = p.slip;
    auto si = index_span(origin_x, cell, res, p.x, reach);
    auto sj = index_span(origin_z, cell, res, p.z, reach);
    J.span_i0 = si.first;
    J.span_i1 = si.second;
    J.span_j0 = sj.first;
    J.span_j1 = sj.second;
    J.index = index;
    J.pad[0] = J.pad[1] = J.pad[2] = 0;
    return J;
}

float push_reach(const silt_tire_push& p, float cell) { return hypotf(p.radius * 1.4f, p.width * 0.65f + cell) + cell; }
float peel_reach(const silt_tire_push& p, float cell) { return p.radius * 1.3f + cell; }

struct JobList {
    size_t off = 0;
    int n = 0, i0 = 0, j0 = 0, w = 0, h = 0;
};

JobList job_list(Table& tab, const std::vector<PushJob>& jobs) {
    JobList L;
    L.n = (int)jobs.size();
    int a0 = 1 << 30, a1 = -1, b0 = 1 << 30, b1 = -1;
    for (auto& J : jobs) {
        if (J.span_i1 <= J.span_i0 || J.span_j1 <= J.span_j0) continue;
        a0 = std::min(a0, J.span_i0);
        a1 = std::max(a1, J.span_i1);
        b0 = std::min(b0, J.span_j0);
        b1 = std::max(b1, J.span_j1);
    }
    if (a1 < 0) {
        L.n = 0;
        return L;
    }
    L.i0 = a0;
    L.j0 = b0;
    L.w = a1 - a0;
    L.h = b1 - b0;
    L.off = tab.put(jobs.data(), jobs.size());
    return L;
}

}  // namespace

// Per-handle state of one step between laying the patches and packing them.
struct StepPlan {
    int np = 0;
    std::vector<int> held;
    bool any_park = false;
    int n_owner = 0, n_near = 0, n_ent = 0;
    size_t off_jobs = 0;
    size_t off_refs = 0, off_held = 0, off_oidx = 0, off_oval = 0, off_near = 0, off_ent = 0, off_seg = 0;
    std::vector<JobList> fine_push, fine_peel;
    JobList coarse_push, coarse_peel;
    std::vector<int> coarse_pushed;   // tires that shove coarse cells (their cell is not held)
    int b_apply = 0, b_fade = 0, b_ncap = 0;  // batched step: near-field apply, fade and capture counts
    size_t off_push_groups = 0, off_peel_groups = 0;
    int n_push_groups = 0, n_peel_groups = 0, push_cells_max = 0, peel_cells_max = 0;
    int slot = 0;
};

// Staging slots of the per-step tables: a slot is reused STAGING_SLOTS steps
// later, so the wait for its earlier copy finds it done and the host plans
// ahead of the device.
constexpr int STAGING_SLOTS = 4;

struct HostState {
    StepPlan plan;
    char* d_tab[STAGING_SLOTS] = {};
    char* h_tab[STAGING_SLOTS] = {};
    size_t cap[STAGING_SLOTS] = {};
    cudaEvent_t ev[STAGING_SLOTS] = {};
    int flip = 0;
};

static HostState& H(Patches& P) { return *reinterpret_cast<HostState*>(I(P).host); }

static int ensure_patches(Patches& P, int np, cudaStream_t st) {
    const size_t fn = (size_t)P.fres * P.fres;
    while ((int)P.patches.size() < np) {
        PatchState* S = new PatchState();
        // 12 planes + a spare + the window engine's scratch for two layers,
        // then grain and the wall mask.
        const size_t planes = 13 + 2 * (size_t)window::SCRATCH_PLANES;
        cudaError_t e = cudaMalloc(&S->base, planes * fn * sizeof(float) + 2 * fn + 256);
        if (e != cudaSuccess) {
            delete S;
            snprintf(g_err, sizeof g_err, "patch alloc: %s", cudaGetErrorString(e));
            return SILT_ENOMEM;
        }
        float* q = S->base;
        float** named[12] = {&S->water, &S->slurry, &S->uw, &S->vw, &S->us,      &S->vs,
                             &S->bed,   &S->bed_slurry, &S->moisture, &S->nu_s, &S->mob_s, &S->damp_s};
        for (int k = 0; k < 12; ++k) {
            *named[k] = q;
            q += fn;
        }
        q += fn;
        for (int l = 0; l < 2; ++l) {
            S->win[l] = q;
            q += (size_t)window::SCRATCH_PLANES * fn;
        }
        S->grain = reinterpret_cast<uint8_t*>(q);
        S->solid = S->grain + fn;
        FCK(cudaMemsetAsync(S->base, 0, planes * fn * sizeof(float), st));
        FCK(cudaMemsetAsync(S->grain, 4, fn, st));
        FCK(cudaMemsetAsync(S->solid, 0, fn, st));
        P.patches.push_back(S);
    }
    return SILT_OK;
}

// Plans one step's geometry on the host and ships it in one table copy.
static int plan_step(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& ps, float dt) {
    Impl& M = I(P);
    HostState& HS = H(P);
    StepPlan& L = HS.plan;
    L = StepPlan();
    SheetView W = view_of(s);
    const int res = W.res, fres = P.fres, sub = P.sub;
    const float extent = (float)fres * P.fcell;
    const int full = sub * sub;
    const float r2 = P.tire_r * P.tire_r;
    L.np = P.patches_off ? 0 : P.layout == SILT_FINE_MEAN_PATCH ? 1 : std::min((int)ps.size(), MAX_PATCHES);
    int rc = ensure_patches(P, L.np, W.st);
    if (rc) return rc;
    // Owner changes as one value per cell: last step's holds are released,
    // this step's holds override (a cell listed twice would race in the scatter).
    std::map<int, int8_t> changes;
    for (int c : M.held_now) {
        M.h_owner[c] = -1;
        changes[c] = -1;
    }
    M.held_now.clear();
    struct Touch {
        int cnt = 0;
        std::vector<Segment> segs;
    };
    std::map<int, Touch> touch;
    std::vector<int16_t> axes((size_t)L.np * 2 * fres);
    for (int p = 0; p < L.np; ++p) {
        PatchState* S = P.patches[p];
        if (P.layout == SILT_FINE_MEAN_PATCH) {
            float cx = 0.0f, cz = 0.0f;
            for (const auto& t : ps) {
                cx += t.x;
                cz += t.z;
            }
            float n = (float)ps.size();
            cx /= n;
            cz /= n;
            host::snap_origin(cx, cz, extent, W.cell, S->origin);
        } else {
            host::snap_origin(ps[p].x, ps[p].z, extent, W.cell, S->origin);
        }
        S->col.assign(fres, -1);
        S->row.assign(fres, -1);
        for (int i = 0; i < fres; ++i) {
            S->col[i] = (int16_t)coarse_axis(W.origin[0], W.cell, res, S->origin[0] + ((float)i + 0.5f) * P.fcell);
            S->row[i] = (int16_t)coarse_axis(W.origin[1], W.cell, res, S->origin[1] + ((float)i + 0.5f) * P.fcell);
            axes[(size_t)p * 2 * fres + i] = S->col[i];
            axes[(size_t)p * 2 * fres + fres + i] = S->row[i];
        }
        auto runs = [&](const std::vector<int16_t>& ax) {
            std::vector<std::array<int, 3>> out;
            int i = 0;
            while (i < fres) {
                int c = ax[i], n = 1;
                while (i + n < fres && ax[i + n] == c) ++n;
                if (c >= 0) out.push_back({c, i, i + n - 1});
                else L.any_park = true;
                i += n;
            }
            return out;
        };
        auto cr = runs(S->col), rr = runs(S->row);
        std::vector<silt_tire_push> own;
        if (P.layout == SILT_FINE_MEAN_PATCH)
            own = ps;
        else
            own.push_back(ps[p]);
        for (auto& r : rr)
            for (auto& c : cr) {
                const int cidx = r[0] * res + c[0];
                const int n = (c[2] - c[1] + 1) * (r[2] - r[1] + 1);
                Touch& T = touch[cidx];
                T.cnt += n;
                T.segs.push_back({p, c[1], c[2], r[1], r[2], 0});
                if (n != full || M.h_owner[cidx] >= 0) continue;
                float x = W.origin[0] + ((float)c[0] + 0.5f) * W.cell;
                float z = W.origin[1] + ((float)r[0] + 0.5f) * W.cell;
                if (near_tire_zone(own, x, z, r2)) {
                    M.h_owner[cidx] = (int8_t)p;
                    M.held_now.push_back(cidx);
                    L.held.push_back(cidx);
                    changes[cidx] = (int8_t)p;
                }
            }
    }
    std::vector<NearCol> ncols;
    for (int p = 0; p < L.np; ++p) {
        PatchState* S = P.patches[p];
        auto runs = [&](const std::vector<int16_t>& ax) {
            std::vector<std::pair<int, int>> out;
            int i = 0;
            while (i < fres) {
                int c = ax[i], n = 1;
                while (i + n < fres && ax[i + n] == c) ++n;
                if (c >= 0 && n == sub) out.push_back({c, i});
                i += n;
            }
            return out;
        };
        auto cols = runs(S->col), rows = runs(S->row);
        for (auto& r : rows)
            for (auto& c : cols) {
                const int cidx = r.first * res + c.first;
                if (M.h_owner[cidx] != p) continue;
                const int i = c.first, j = r.first;
                int inner = 0;
                if (i > 0 && j > 0 && i + 1 < res && j + 1 < res)
                    inner = M.h_owner[cidx - 1] >= 0 && M.h_owner[cidx + 1] >= 0 && M.h_owner[cidx - res] >= 0 &&
                            M.h_owner[cidx + res] >= 0;
                ncols.push_back({cidx, p, c.second, r.second, inner, 0});
            }
    }
    std::vector<RestrictEntry> ents;
    std::vector<Segment> segs;
    for (auto& kv : touch) {
        RestrictEntry E;
        E.cidx = kv.first;
        E.cnt = kv.second.cnt;
        E.held = M.h_owner[kv.first] >= 0;
        E.seg_off = (int)segs.size();
        E.seg_n = (int)kv.second.segs.size();
        E.pad = 0;
        for (auto& sg : kv.second.segs) segs.push_back(sg);
        ents.push_back(E);
    }
    std::vector<int> oidx;
    std::vector<int8_t> oval;
    for (auto& kv : changes) {
        oidx.push_back(kv.first);
        oval.push_back(kv.second);
    }
    if (L.any_park && !M.park.cap) FCK(park::alloc(M.park, 1u << 16, W.st));
    Table tab;
    // Axes first: the refs below point into the device copy of this table.
    const size_t off_axes = tab.put(axes.data(), axes.size());
    L.off_held = tab.put(L.held.data(), L.held.size());
    L.off_oidx = tab.put(oidx.data(), oidx.size());
    L.off_oval = tab.put(oval.data(), oval.size());
    L.off_near = tab.put(ncols.data(), ncols.size());
    L.off_ent = tab.put(ents.data(), ents.size());
    L.off_seg = tab.put(segs.data(), segs.size());
    L.n_owner = (int)oidx.size();
    L.n_near = (int)ncols.size();
    L.n_ent = (int)ents.size();
    // Tire jobs: shove and peel per patch, shove outside, peel on the coarse window.
    for (int p = 0; p < L.np; ++p) {
        PatchState* S = P.patches[p];
        std::vector<PushJob> push, peel;
        for (size_t q = 0; q < ps.size(); ++q) {
            peel.push_back(make_job(ps[q], (int)q, S->origin[0], S->origin[1], P.fcell, fres,
                                    peel_reach(ps[q], P.fcell)));
            // cell_is_refined (src/fluid_core.rs:8338-8356): held by this patch and inside its rectangle.
            long ci = coarse_axis(W.origin[0], W.cell, res, ps[q].x);
            long cj = coarse_axis(W.origin[1], W.cell, res, ps[q].z);
            if (ci < 0 || cj < 0 || M.h_owner[cj * res + ci] != p) continue;
            float x0 = W.origin[0] + (float)ci * W.cell, z0 = W.origin[1] + (float)cj * W.cell;
            float x1 = x0 + W.cell, z1 = z0 + W.cell;
            if (!(x0 >= S->origin[0] - 1.0e-4f && z0 >= S->origin[1] - 1.0e-4f &&
                  x1 <= S->origin[0] + extent + 1.0e-4f && z1 <= S->origin[1] + extent + 1.0e-4f))
                continue;
            push.push_back(make_job(ps[q], (int)q, S->origin[0], S->origin[1], P.fcell, fres,
                                    push_reach(ps[q], P.fcell)));
        }
        L.fine_push.push_back(job_list(tab, push));
        L.fine_peel.push_back(job_list(tab, peel));
    }
    {
        std::vector<JobGroup> pg, qg;
        L.push_cells_max = L.peel_cells_max = 0;
        for (int p = 0; p < L.np; ++p) {
            const PatchState* S = P.patches[p];
            for (int which = 0; which < 2; ++which) {
                const JobList& J = which ? L.fine_peel[p] : L.fine_push[p];
                if (!J.n) continue;
                JobGroup G;
                G.patch = p;
                G.ox = S->origin[0];
                G.oz = S->origin[1];
                G.job_off = (int)J.off;
                G.njobs = J.n;
                G.i0 = J.i0;
                G.j0 = J.j0;
                G.w = J.w;
                G.h = J.h;
                (which ? qg : pg).push_back(G);
                int& mx = which ? L.peel_cells_max : L.push_cells_max;
                mx = std::max(mx, J.w * J.h);
            }
        }
        L.n_push_groups = (int)pg.size();
        L.n_peel_groups = (int)qg.size();
        L.off_push_groups = tab.put(pg.data(), pg.size());
        L.off_peel_groups = tab.put(qg.data(), qg.size());
    }
    {
        std::vector<PushJob> push, peel;
        for (size_t q = 0; q < ps.size(); ++q) {
            peel.push_back(make_job(ps[q], (int)q, W.origin[0], W.origin[1], W.cell, res, peel_reach(ps[q], W.cell)));
            long ci = coarse_axis(W.origin[0], W.cell, res, ps[q].x);
            long cj = coarse_axis(W.origin[1], W.cell, res, ps[q].z);
            if (ci >= 0 && cj >= 0 && M.h_owner[cj * res + ci] >= 0) continue;
            if (P.coarse_shove_off) continue;
            const PushJob J = make_job(ps[q], (int)q, W.origin[0], W.origin[1], W.cell, res, push_reach(ps[q], W.cell));
            push.push_back(J);
            // A shove whose span misses the window touches no coarse cell.
            if (J.span_i0 < J.span_i1 && J.span_j0 < J.span_j1) L.coarse_pushed.push_back((int)q);
        }
        L.coarse_push = job_list(tab, push);
        L.coarse_peel = job_list(tab, peel);
    }
    // Patch references, pointing at the axes inside the device table.
    const int slot = HS.flip;
    HS.flip = (HS.flip + 1) % STAGING_SLOTS;
    L.slot = slot;
    size_t need = tab.buf.size() + (size_t)L.np * (sizeof(PatchRef) + 2 * sizeof(window::Job)) + 1024;
    if (need > HS.cap[slot]) {
        if (HS.ev[slot]) FCK(cudaEventSynchronize(HS.ev[slot]));
        if (HS.d_tab[slot]) cudaFree(HS.d_tab[slot]);
        if (HS.h_tab[slot]) cudaFreeHost(HS.h_tab[slot]);
        HS.d_tab[slot] = nullptr;
        HS.h_tab[slot] = nullptr;
        HS.cap[slot] = std::max(need * 2, (size_t)1 << 20);
        FCK(cudaMalloc(&HS.d_tab[slot], HS.cap[slot]));
        FCK(cudaMallocHost(&HS.h_tab[slot], HS.cap[slot]));
        if (!HS.ev[slot]) FCK(cudaEventCreateWithFlags(&HS.ev[slot], cudaEventDisableTiming));
    }
    std::vector<PatchRef> refs;
    for (int p = 0; p < L.np; ++p) {
        PatchState* S = P.patches[p];
        PatchRef r;
        r.water = S->water;
        r.slurry = S->slurry;
        r.uw = S->uw;
        r.vw = S->vw;
        r.us = S->us;
        r.vs = S->vs;
        r.bed = S->bed;
        r.bed_slurry = S->bed_slurry;
        r.moisture = S->moisture;
        r.nu_s = S->nu_s;
        r.mob_s = S->mob_s;
        r.damp_s = S->damp_s;
        r.grain = S->grain;
        r.solid = S->solid;
        const int16_t* dax = reinterpret_cast<const int16_t*>(HS.d_tab[slot] + off_axes);
        r.col = dax + (size_t)p * 2 * fres;
        r.row = dax + (size_t)p * 2 * fres + fres;
        r.ox = S->origin[0];
        r.oz = S->origin[1];
        refs.push_back(r);
    }
    L.off_refs = tab.put(refs.data(), refs.size());
    // The fine pair (src/fluid_core.rs:7942-8150 with fine = true): one window
    // job per patch and layer.
    {
        std::vector<window::Job> jobs;
        const float nu_w = P.open_mobility >= 0.0f ? -std::fmax(P.open_mobility, 1.0e-4f) : host::dynamic_viscosity(3, 1.0f);
        const size_t fn = (size_t)fres * fres;
        for (int p = 0; p < L.np; ++p) {
            PatchState* S = P.patches[p];
            for (int l = 0; l < 2; ++l) {
                window::Job J;
                memset(&J, 0, sizeof J);
                J.h = l == 0 ? S->water : S->slurry;
                J.u = l == 0 ? S->uw : S->us;
                J.v = l == 0 ? S->vw : S->vs;
                J.bed = l == 0 ? S->bed : S->bed_slurry;
                J.grain = S->grain;
                J.moisture = S->moisture;
                window::attach_scratch(J, S->win[l], fn);
                J.res = fres;
                J.cell = P.fcell;
                J.div = P.fdivs;
                J.solid = P.n_solids > 0 ? S->solid : nullptr;
                J.cut = M.d_books + 3;
                J.round = M.d_books + 6;
                J.cut_area = (double)P.fcell * (double)P.fcell;
                J.dt = dt;
                J.vort = l == 0 ? 0.08f : 0.05f;
                J.sub_cap = P.sub_cap;
                J.eps = 1.0e-6f;
                J.nu_mode = l == 0 ? window::NU_CONST : window::NU_TABLE;
                J.nu_plane = S->nu_s;
                J.mob_plane = S->mob_s;
                J.damp_plane = S->damp_s;
                J.nu_c = nu_w;
                J.mob_c = host::sheet_mobility_for(nu_w);
                for (int k = 1; k <= 8; ++k) J.decay_c[k] = expf(-host::sheet_damp(nu_w) * (dt / (float)k));
                J.pace = P.pace;
                J.has_sc2 = 1;
                J.active = 1;
                jobs.push_back(J);
            }
        }
        L.off_jobs = tab.put(jobs.data(), jobs.size());
    }
    // The pinned slot in use STAGING_SLOTS steps ago may still feed its copy.
    FCK(cudaEventSynchronize(HS.ev[slot]));
    memcpy(HS.h_tab[slot], tab.buf.data(), tab.buf.size());
    FCK(cudaMemcpyAsync(HS.d_tab[slot], HS.h_tab[slot], tab.buf.size(), cudaMemcpyHostToDevice, W.st));
    FCK(cudaEventRecord(HS.ev[slot], W.st));
    return SILT_OK;
}

#define TAB(T, off) (reinterpret_cast<const T*>(HS.d_tab[L.slot] + (off)))

// The coarse speed bound's growth from this step's coupling. The restrict
// hands each column a depth-weighted mean of its fine cells' velocities and
// its own, so it adds nothing above the largest fine speed; after the patch
// step every wet fine cell faster than 0.05 m/s lies in a work box and is
// clamped to the film cap, and drier cells carry only the laid coarse velocity
// (shoves need 4 mm of depth). So only the shoves of tires outside the patches
// raise it: each by at most 1.04 max(speed, 0.4) (|fore f + 0.28 flank r| <=
// sqrt(1 + 0.28^2)), summed where the tires' spans overlap.
static float coarse_shove_bound(const StepPlan& L, const std::vector<silt_tire_push>& ps, const SheetView& W) {
    float add = 0.0f;
    for (int a : L.coarse_pushed) {
        float reach_a = push_reach(ps[a], W.cell);
        auto ai = index_span(W.origin[0], W.cell, W.res, ps[a].x, reach_a);
        auto aj = index_span(W.origin[1], W.cell, W.res, ps[a].z, reach_a);
        float sum = 0.0f;
        for (int b : L.coarse_pushed) {
            float reach_b = push_reach(ps[b], W.cell);
            auto bi = index_span(W.origin[0], W.cell, W.res, ps[b].x, reach_b);
            auto bj = index_span(W.origin[1], W.cell, W.res, ps[b].z, reach_b);
            bool overlap = ai.first < bi.second && bi.first < ai.second && aj.first < bj.second && bj.first < aj.second;
            if (a == b || overlap) sum += 1.04f * std::max(ps[b].speed, 0.4f);
        }
        add = std::max(add, sum);
    }
    return add;
}

static int lay_patches(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& ps, float dt) {
    Impl& M = I(P);
    int rc = plan_step(P, s, ps, dt);
    if (rc) return rc;
    HostState& HS = H(P);
    const StepPlan& L = HS.plan;
    SheetView W = view_of(s);
    const PatchRef* refs = TAB(PatchRef, L.off_refs);
    if (L.n_owner) {
        ::silt::launch_dep(k_scatter_owner, dim3(launch_blocks(L.n_owner)), dim3(256), 0, W.st, M.owner, TAB(int, L.off_oidx),
                                                                     TAB(int8_t, L.off_oval), L.n_owner);
        ::silt::count_launch();
        FCK(cudaGetLastError());
    }
    if (L.np == 0) {  // no patch: the released holds above are all there is to lay
        FCK(cudaMemsetAsync(M.counters + 3, 0, sizeof(int), W.st));  // the spray count k_refine_lay would clear
        P.active = 0;
        return SILT_OK;
    }
    ::silt::launch_dep(k_refine_lay, dim3(launch_blocks((size_t)L.np * P.fres * P.fres)), dim3(256), 0, W.st, refs, L.np, P.fres, W, M.owner,
                                                                                 M.counters + 3);
    ::silt::count_launch();
    FCK(cudaGetLastError());
    P.fine_on = true;
    P.active = L.np;
    // Empty the held coarse columns and apply the near-field residuals in one
    // launch (the fade runs with the shoves).
    const int n_held = (int)L.held.size();
    const int n_apply = M.near_maybe ? L.n_near : 0;
    if (n_held || n_apply) {
        const int zero_blocks = n_held ? launch_blocks((size_t)n_held, 128) : 0;
        ::silt::launch_dep(k_lay_finish, dim3(zero_blocks + n_apply), dim3(128), 0, W.st, W, TAB(int, L.off_held), n_held, zero_blocks, refs,
                                                             P.fres, P.sub, TAB(NearCol, L.off_near), n_apply,
                                                             M.slot_map, M.pool, M.meta);
        ::silt::count_launch();
        FCK(cudaGetLastError());
    }
    return SILT_OK;
}

int restrict_all(Patches& P, silt_sheet* s) {
    if (!P.fine_on) return SILT_OK;
    Impl& M = I(P);
    HostState& HS = H(P);
    const StepPlan& L = HS.plan;
    SheetView W = view_of(s);
    const PatchRef* refs = TAB(PatchRef, L.off_refs);
    // The near-field capture and the restrict in one launch.
    const int ncap = (P.near_on && L.n_near) ? L.n_near : 0;
    if (ncap) M.near_maybe = true;
    if (ncap || L.n_ent) {
        const int rblocks = L.n_ent ? launch_blocks((size_t)L.n_ent * 32, 128) : 0;
        ::silt::launch_dep(k_restrict, dim3(ncap + rblocks), dim3(128), 0, W.st, refs, P.fres, P.sub, W, TAB(RestrictEntry, L.off_ent), L.n_ent,
                                                     TAB(Segment, L.off_seg), P.fcell * P.fcell, W.cell * W.cell,
                                                     TAB(NearCol, L.off_near), ncap, M.slot_map, M.pool, M.meta,
                                                     M.free_stack, M.counters);
        ::silt::count_launch();
        FCK(cudaGetLastError());
    }
    ::silt::launch_dep(k_release, dim3(launch_blocks((size_t)L.np * P.fres * P.fres)), dim3(256), 0, W.st, refs, L.np,
                       P.fres, P.fcell, W.cell, M.d_books, L.any_park ? 1 : 0, M.park);
    ::silt::count_launch();
    FCK(cudaGetLastError());
    P.fine_on = false;
    invalidate_ledger(s);
    return SILT_OK;
}

static int fade_only(Patches& P, silt_sheet* s, float dt) {
    Impl& M = I(P);
    if (!M.near_maybe) return SILT_OK;
    SheetView W = view_of(s);
    ::silt::launch_dep(k_near_fade, dim3((NEAR_POOL + 255) / 256), dim3(256), 0, W.st, M.meta, M.slot_map, M.free_stack, M.counters,
                                                          dt > 0.0f && std::isfinite(dt) ? dt : 0.0f);
    ::silt::count_launch();
    FCK(cudaGetLastError());
    return SILT_OK;
}

int step_patches(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& ps, float dt, StepOut& out) {
    Impl& M = I(P);
    int rc = restrict_all(P, s);
    if (rc) return rc;
    SheetView W = view_of(s);
    if (ps.empty()) {
        if (M.spray_dirty) {
            FCK(cudaMemsetAsync(M.counters + 3, 0, sizeof(int), W.st));
            M.spray_dirty = false;
        }
        return fade_only(P, s, dt);
    }
    // With tires, k_refine_lay clears the spray count.
    M.spray_dirty = true;
    // The coarse planes may still wait for the previous dry cut: the lay,
    // restrict and shove kernels apply it to the cells they touch.
    if ((rc = lay_patches(P, s, ps, dt))) return rc;
    HostState& HS = H(P);
    const StepPlan& L = HS.plan;
    W = view_of(s);
    const PatchRef* refs = TAB(PatchRef, L.off_refs);
    const char* tab = TAB(char, 0);
    // The shoves of every patch, and the near-field fade in one more row of blocks.
    const int fade = M.near_maybe ? 1 : 0;
    if (L.n_push_groups || fade) {
        dim3 grid(launch_blocks((size_t)std::max(L.push_cells_max, 1)), L.n_push_groups + fade);
        ::silt::launch_dep(k_push_patches, dim3(grid), dim3(256), 0, W.st, refs, tab, TAB(JobGroup, L.off_push_groups), L.n_push_groups, P.fres,
                                               P.fcell, fade, M.meta, M.slot_map, M.free_stack, M.counters,
                                               dt > 0.0f && std::isfinite(dt) ? dt : 0.0f);
        ::silt::count_launch();
        FCK(cudaGetLastError());
    }
    if (P.n_solids > 0) {
        // Each patch's wall mask from its water over its bed (solid_mask(true)).
        dim3 grid(launch_blocks((size_t)P.fres * P.fres), L.np);
        ::silt::launch_dep(k_patch_walls, dim3(grid), dim3(256), 0, W.st, refs, P.fres, P.fcell, P.d_solids,
                           P.n_solids);
        ::silt::count_launch();
        FCK(cudaGetLastError());
    }
    FCK(window::launch_window_step(TAB(window::Job, L.off_jobs), 2 * L.np, P.fres, W.st));
    if (L.n_peel_groups) {
        dim3 grid(launch_blocks((size_t)L.peel_cells_max), L.n_peel_groups);
        ::silt::launch_dep(k_peel_patches, dim3(grid), dim3(256), 0, W.st, refs, tab, TAB(JobGroup, L.off_peel_groups), P.fres, P.fcell, M.spray,
                                               M.counters, M.d_books);
        ::silt::count_launch();
        FCK(cudaGetLastError());
    }
    if ((rc = restrict_all(P, s))) return rc;
    if (L.coarse_push.n) {
        const JobList& J = L.coarse_push;
        ::silt::launch_dep(k_push_cells, dim3(launch_blocks((size_t)J.w * J.h)), dim3(256), 0, W.st, W.h[0], W.h[1], W.u[0], W.v[0], W.u[1],
                                                                         W.v[1], W.res, W.cell, W.origin[0],
                                                                         W.origin[1], TAB(PushJob, J.off), J.n, J.i0,
                                                                         J.j0, J.w, J.h);
        ::silt::count_launch();
        FCK(cudaGetLastError());
    }
    add_speed(s, coarse_shove_bound(L, ps, W));
    out.spray_events = 1;
    return SILT_OK;
}

int peel_coarse(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& ps, StepOut& out) {
    if (ps.empty()) return SILT_OK;
    Impl& M = I(P);
    HostState& HS = H(P);
    const StepPlan& L = HS.plan;
    const JobList& J = L.coarse_peel;
    if (!J.n) return SILT_OK;
    SheetView W = view_of(s);
    ::silt::launch_dep(k_peel, dim3(launch_blocks((size_t)J.w * J.h)), dim3(256), 0, W.st, W.h[0], W.u[0], W.v[0], W.res, W.cell, W.origin[0],
                                                               W.origin[1], TAB(PushJob, J.off), J.n, J.i0, J.j0, J.w,
                                                               J.h, M.owner, W.res, W.origin[0], W.origin[1], W.cell,
                                                               1, 0, M.spray, M.counters, M.d_books, W.d_acc);
    ::silt::count_launch();
    FCK(cudaGetLastError());
    return SILT_OK;
}

int collect_spray(Patches& P, silt_sheet* s, const StepOut& out, silt_spray_event* host, int cap, int* n_out) {
    Impl& M = I(P);
    SheetView W = view_of(s);
    if (!host && !n_out) return SILT_OK;
    FCK(cudaMemcpyAsync(M.h_counters, M.counters, 8 * sizeof(int), cudaMemcpyDeviceToHost, W.st));
    FCK(cudaStreamSynchronize(W.st));
    int n = std::min(M.h_counters[3], SPRAY_CAP);
    if (n_out) *n_out = n;
    if (host && cap > 0 && n > 0) {
        std::vector<SprayRec> recs(n);
        FCK(cudaMemcpyAsync(recs.data(), M.spray, n * sizeof(SprayRec), cudaMemcpyDeviceToHost, W.st));
        FCK(cudaStreamSynchronize(W.st));
        std::sort(recs.begin(), recs.end(), [](const SprayRec& a, const SprayRec& b) { return a.key < b.key; });
        for (int k = 0; k < n && k < cap; ++k)
            host[k] = {recs[k].x, recs[k].y, recs[k].z, recs[k].vx, recs[k].vy, recs[k].vz, recs[k].volume,
                       recs[k].kind};
    }
    return SILT_OK;
}

double* books(Patches& P) { return I(P).d_books; }

park::Table& park_table(Patches& P) { return I(P).park; }

int move_window(Patches& P, silt_sheet* s, int di, int dj, bool scroll) {
    Impl& M = I(P);
    if (!M.near_maybe) return SILT_OK;
    SheetView W = view_of(s);
    ::silt::launch_dep(k_near_unmap, dim3(launch_blocks(W.n)), dim3(256), 0, W.st, M.slot_map, W.n);
    ::silt::count_launch();
    FCK(cudaGetLastError());
    ::silt::launch_dep(k_near_move, dim3((NEAR_POOL + 255) / 256), dim3(256), 0, W.st, M.meta, M.slot_map, M.counters,
                       W.res, di, dj, scroll ? 1 : 0);
    ::silt::count_launch();
    FCK(cudaGetLastError());
    return SILT_OK;
}

int ledger_parts(Patches& P, silt_sheet* s, double* spray, double* park_w, double* park_s, double* cut,
                 double* reach, double* eroded, double* round) {
    Impl& M = I(P);
    SheetView W = view_of(s);
    FCK(cudaMemcpyAsync(M.h_books, M.d_books, 16 * sizeof(double), cudaMemcpyDeviceToHost, W.st));
    FCK(cudaStreamSynchronize(W.st));
    *spray = M.h_books[0];
    *park_w = M.h_books[1];
    *park_s = M.h_books[2];
    if (cut) *cut = M.h_books[3];
    if (reach) *reach = M.h_books[4];
    if (eroded) *eroded = M.h_books[5];
    if (round) *round = M.h_books[6];
    return SILT_OK;
}

int books_enqueue(Patches& P, silt_sheet* s) {
    Impl& M = I(P);
    FCK(cudaMemcpyAsync(M.h_books, M.d_books, 16 * sizeof(double), cudaMemcpyDeviceToHost, view_of(s).st));
    return SILT_OK;
}

const double* books_host(Patches& P) { return I(P).h_books; }

int debug_patch(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& ps, int patch, float* host,
                float* origin2) {
    int rc = restrict_all(P, s);
    if (rc) return rc;
    SheetView W = view_of(s);
    if (ps.empty()) {
        if ((rc = fade_only(P, s, 0.0f))) return rc;
        memset(host, 0, (size_t)P.fres * P.fres * sizeof(float));
        FCK(cudaStreamSynchronize(W.st));
        return SILT_OK;
    }
    if ((rc = flush(s))) return rc;
    if ((rc = lay_patches(P, s, ps, 0.0f))) return rc;
    if (patch >= 0 && patch < P.active) {
        PatchState* S = P.patches[patch];
        FCK(cudaMemcpyAsync(host, S->water, (size_t)P.fres * P.fres * sizeof(float), cudaMemcpyDeviceToHost, W.st));
        if (origin2) {
            origin2[0] = S->origin[0];
            origin2[1] = S->origin[1];
        }
    }
    rc = restrict_all(P, s);
    FCK(cudaStreamSynchronize(W.st));
    return rc;
}

int near_tiles(Patches& P, silt_sheet* s, int* out) {
    Impl& M = I(P);
    SheetView W = view_of(s);
    FCK(cudaMemcpyAsync(M.h_counters, M.counters, 8 * sizeof(int), cudaMemcpyDeviceToHost, W.st));
    FCK(cudaStreamSynchronize(W.st));
    *out = M.h_counters[1];
    return SILT_OK;
}

int set_near_field(Patches& P, silt_sheet* s, bool on) {
    Impl& M = I(P);
    P.near_on = on;
    if (!on) {
        SheetView W = view_of(s);
        ::silt::launch_dep(k_init_pool, dim3(launch_blocks(std::max<size_t>(W.n, NEAR_POOL))), dim3(256), 0, W.st, M.meta, M.free_stack,
                                                                                       M.slot_map, W.n, M.counters);
        ::silt::count_launch();
        FCK(cudaGetLastError());
        M.near_maybe = false;
    }
    return SILT_OK;
}

int create(Patches& P, const silt_cfg& cfg, int res, cudaStream_t st) {
    P.layout = cfg.fine_layout == SILT_FINE_PER_TIRE ? SILT_FINE_PER_TIRE : SILT_FINE_MEAN_PATCH;
    P.fres = cfg.fine_res;
    P.fcell = cfg.fine_cell;
    P.fdivs = cell_divisors(cfg.fine_cell, st);
    P.sub = (int)std::lround(cfg.cell / cfg.fine_cell);
    P.tire_r = cfg.tire_r;
    if (P.fres > 512 || P.sub > 32) {
        snprintf(g_err, sizeof g_err, "fine_res above 512 or cell ratio above 32");
        return SILT_EINVAL;
    }
    Impl* M = new Impl();
    P.impl = M;
    M->host = new HostState();
    M->res = res;
    const size_t n = (size_t)res * res;
    M->h_owner.assign(n, -1);
    const int n2 = P.sub * P.sub;
    FCK(cudaMalloc(&M->owner, n));
    FCK(cudaMemsetAsync(M->owner, 0xff, n, st));
    FCK(cudaMalloc(&M->slot_map, n * sizeof(int)));
    FCK(cudaMalloc(&M->pool, (size_t)NEAR_POOL * 4 * n2 * sizeof(float)));
    FCK(cudaMalloc(&M->meta, NEAR_POOL * sizeof(NearMeta)));
    FCK(cudaMalloc(&M->free_stack, NEAR_POOL * sizeof(int)));
    FCK(cudaMalloc(&M->counters, 8 * sizeof(int)));
    FCK(cudaMalloc(&M->spray, SPRAY_CAP * sizeof(SprayRec)));
    FCK(cudaMalloc(&M->d_books, 16 * sizeof(double)));
    FCK(cudaMemsetAsync(M->d_books, 0, 16 * sizeof(double), st));
    FCK(cudaMallocHost(&M->h_books, 16 * sizeof(double)));
    FCK(cudaMallocHost(&M->h_counters, 8 * sizeof(int)));
    ::silt::launch_dep(k_init_pool, dim3(launch_blocks(std::max<size_t>(n, NEAR_POOL))), dim3(256), 0, st, M->meta, M->free_stack, M->slot_map, n,
                                                                               M->counters);
    ::silt::count_launch();
    FCK(cudaGetLastError());
    return SILT_OK;
}

void destroy(Patches& P) {
    for (PatchState* S : P.patches) {
        cudaFree(S->base);
        delete S;
    }
    P.patches.clear();
    if (!P.impl) return;
    Impl* M = (Impl*)P.impl;
    if (M->host) {
        HostState* HS = (HostState*)M->host;
        for (int k = 0; k < STAGING_SLOTS; ++k) {
            if (HS->ev[k]) cudaEventDestroy(HS->ev[k]);
            cudaFree(HS->d_tab[k]);
            if (HS->h_tab[k]) cudaFreeHost(HS->h_tab[k]);
        }
        delete HS;
    }
    park::release(M->park);
    cudaFree(M->owner);
    cudaFree(M->slot_map);
    cudaFree(M->pool);
    cudaFree(M->meta);
    cudaFree(M->free_stack);
    cudaFree(M->counters);
    cudaFree(M->spray);
    cudaFree(M->d_books);
    if (M->h_books) cudaFreeHost(M->h_books);
    if (M->h_counters) cudaFreeHost(M->h_counters);
    delete M;
    P.impl = nullptr;
}

const char* last_error() { return g_err; }


// ------------------------------------------------------------ batched windows
// Many windows' nested patches stepped by one launch per kernel: each window's
// tables are planned and uploaded per window (on any host thread), then one
// record per window tells the batched kernels (blockIdx.z = record) where its
// tables, planes and books are.

struct FineRec {
    SheetView W;
    const PatchRef* refs;
    const char* tab;
    int np, fres, sub, park;
    float fcell, dt;
    int8_t* owner;
    const int* oidx;
    const int8_t* oval;
    int n_owner;
    const int* held;
    int n_held, zero_blocks;
    const NearCol* near;
    int n_apply, ncap, fade;
    const JobGroup* push_groups;
    int n_push_groups;
    const JobGroup* peel_groups;
    int n_peel_groups;
    const RestrictEntry* ents;
    int n_ent, rblocks;
    const Segment* segs;
    const PushJob* cpush;
    int cpush_n, cpush_i0, cpush_j0, cpush_w, cpush_h;
    int* slot_map;
    float* pool;
    NearMeta* meta;
    int* free_stack;
    int* counters;
    SprayRec* spray;
    double* books;
    park::Table park_table;
};

struct PeelRec {
    SheetView W;
    const PushJob* jobs;
    int n, i0, j0, w, h;
    int8_t* owner;
    SprayRec* spray;
    int* counters;
    double* books;
};

__global__ void kb_scatter(const FineRec* recs) {
    ::silt::dep_wait();
    const FineRec& r = recs[blockIdx.z];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < r.n_owner; k += gridDim.x * blockDim.x)
        r.owner[r.oidx[k]] = r.oval[k];
}

__global__ void kb_refine(const FineRec* recs) {
    ::silt::dep_wait();
    const FineRec& r = recs[blockIdx.z];
    const size_t fn = (size_t)r.fres * r.fres;
    if (blockIdx.x == 0 && threadIdx.x == 0) r.counters[3] = 0;  // this step's spray events start here
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < fn * r.np; k += (size_t)gridDim.x * blockDim.x)
        refine_cell(r.refs[k / fn], (int)(k / fn), (int)(k % fn), r.fres, r.W, r.owner);
}

__global__ void kb_lay_finish(const FineRec* recs) {
    ::silt::dep_wait();
    const FineRec& r = recs[blockIdx.z];
    const int b = (int)blockIdx.x;
    if (b < r.zero_blocks) {
        for (int k = b * blockDim.x + threadIdx.x; k < r.n_held; k += r.zero_blocks * blockDim.x) {
            const size_t c = r.held[k];
            r.W.h[0][c] = 0.0f;
            r.W.h[1][c] = 0.0f;
            r.W.u[0][c] = 0.0f;
            r.W.v[0][c] = 0.0f;
            r.W.u[1][c] = 0.0f;
            r.W.v[1][c] = 0.0f;
        }
        return;
    }
    near_apply_col(b - r.zero_blocks, r.refs, r.fres, r.sub, r.near, r.n_apply, r.slot_map, r.pool, r.meta);
}

__global__ void kb_push(const FineRec* recs) {
    ::silt::dep_wait();
    const FineRec& r = recs[blockIdx.z];
    const int y = (int)blockIdx.y;
    if (y == r.n_push_groups) {
        if (r.fade)
            for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < NEAR_POOL; q += gridDim.x * blockDim.x)
                near_fade_slot(q, r.meta, r.slot_map, r.free_stack, r.counters, r.dt);
        return;
    }
    if (y > r.n_push_groups) return;
    const JobGroup G = r.push_groups[y];
    const PatchRef& R = r.refs[G.patch];
    const PushJob* jobs = reinterpret_cast<const PushJob*>(r.tab + G.job_off);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < G.w * G.h; k += gridDim.x * blockDim.x)
        push_cell(R.water, R.slurry, R.uw, R.vw, R.us, R.vs, r.fres, r.fcell, G.ox, G.oz, jobs, G.njobs,
                  G.i0 + k % G.w, G.j0 + k / G.w);
}

__global__ void kb_peel_patches(const FineRec* recs) {
    ::silt::dep_wait();
    const FineRec& r = recs[blockIdx.z];
    if ((int)blockIdx.y >= r.n_peel_groups) return;
    const JobGroup G = r.peel_groups[blockIdx.y];
    const PatchRef& R = r.refs[G.patch];
    const PushJob* jobs = reinterpret_cast<const PushJob*>(r.tab + G.job_off);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < G.w * G.h; k += gridDim.x * blockDim.x)
        peel_cell(R.water, R.uw, R.vw, r.fres, r.fcell, G.ox, G.oz, jobs, G.njobs, G.i0 + k % G.w, G.j0 + k / G.w,
                  nullptr, 0, 0.0f, 0.0f, 1.0f, 0, G.patch, r.spray, r.counters, r.books, nullptr);
}

__global__ void kb_restrict(const FineRec* recs) {
    ::silt::dep_wait();
    const FineRec& r = recs[blockIdx.z];
    const int b = (int)blockIdx.x;
    if (b < r.ncap) {
        near_capture_col(b, r.refs, r.fres, r.sub, r.near, r.ncap, r.slot_map, r.pool, r.meta, r.free_stack,
                         r.counters);
        return;
    }
    if (b - r.ncap >= r.rblocks) return;
    const int lane = threadIdx.x & 31;
    const int warps = (int)((r.rblocks * (size_t)blockDim.x) >> 5);
    for (int q = (int)(((b - r.ncap) * (size_t)blockDim.x + threadIdx.x) >> 5); q < r.n_ent; q += warps)
        restrict_column(r.refs, r.fres, r.W, r.ents[q], r.segs, r.fcell * r.fcell, r.W.cell * r.W.cell, lane);
}

__global__ void kb_release(const FineRec* recs) {
    ::silt::dep_wait();
    const FineRec& r = recs[blockIdx.z];
    release_cells(r.refs, r.np, r.fres, r.fcell, r.W.cell, r.books, r.park, r.park_table,
                  blockIdx.x * (size_t)blockDim.x + threadIdx.x, (size_t)gridDim.x * blockDim.x);
}

__global__ void kb_coarse_push(const FineRec* recs) {
    ::silt::dep_wait();
    const FineRec& r = recs[blockIdx.z];
    const SheetView& W = r.W;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < r.cpush_w * r.cpush_h; k += gridDim.x * blockDim.x)
        push_cell(W.h[0], W.h[1], W.u[0], W.v[0], W.u[1], W.v[1], W.res, W.cell, W.origin[0], W.origin[1], r.cpush,
                  r.cpush_n, r.cpush_i0 + k % r.cpush_w, r.cpush_j0 + k / r.cpush_w);
}

__global__ void kb_coarse_peel(const PeelRec* recs) {
    ::silt::dep_wait();
    const PeelRec& r = recs[blockIdx.z];
    const SheetView& W = r.W;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < r.w * r.h; k += gridDim.x * blockDim.x)
        peel_cell(W.h[0], W.u[0], W.v[0], W.res, W.cell, W.origin[0], W.origin[1], r.jobs, r.n, r.i0 + k % r.w,
                  r.j0 + k / r.w, r.owner, W.res, W.origin[0], W.origin[1], W.cell, 1, 0, r.spray, r.counters,
                  r.books, W.d_acc);
}

struct FineBatch {
    // Pinned and device staging in a ring of slots: records, then job pointers.
    char* h_buf[STAGING_SLOTS] = {};
    char* d_buf[STAGING_SLOTS] = {};
    size_t cap[STAGING_SLOTS] = {};
    cudaEvent_t ev[STAGING_SLOTS] = {};
    int flip = 0;
    PeelRec* h_peel[STAGING_SLOTS] = {};
    PeelRec* d_peel[STAGING_SLOTS] = {};
    size_t peel_cap[STAGING_SLOTS] = {};
    cudaEvent_t peel_ev[STAGING_SLOTS] = {};
    int peel_flip = 0;
};

FineBatch* batch_new() { return new FineBatch(); }

void batch_free(FineBatch* B) {
    if (!B) return;
    for (int k = 0; k < STAGING_SLOTS; ++k) {
        if (B->ev[k]) cudaEventSynchronize(B->ev[k]);
        if (B->peel_ev[k]) cudaEventSynchronize(B->peel_ev[k]);
        cudaFree(B->d_buf[k]);
        if (B->h_buf[k]) cudaFreeHost(B->h_buf[k]);
        cudaFree(B->d_peel[k]);
        if (B->h_peel[k]) cudaFreeHost(B->h_peel[k]);
        if (B->ev[k]) cudaEventDestroy(B->ev[k]);
        if (B->peel_ev[k]) cudaEventDestroy(B->peel_ev[k]);
    }
    delete B;
}

int batch_prepare(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& ps, float dt, StepOut& out,
                  bool* has_work) {
    *has_work = false;
    Impl& M = I(P);
    int rc = restrict_all(P, s);
    if (rc) return rc;
    if (ps.empty()) {
        if (M.spray_dirty) {
            FCK(cudaMemsetAsync(M.counters + 3, 0, sizeof(int), view_of(s).st));
            M.spray_dirty = false;
        }
        return fade_only(P, s, dt);
    }
    M.spray_dirty = true;
    if ((rc = plan_step(P, s, ps, dt))) return rc;
    StepPlan& L = H(P).plan;
    // The flags the single-window step reads between its launches.
    L.b_apply = M.near_maybe ? L.n_near : 0;
    L.b_fade = M.near_maybe ? 1 : 0;
    L.b_ncap = (P.near_on && L.n_near) ? L.n_near : 0;
    if (L.b_ncap) M.near_maybe = true;
    P.active = L.np;
    P.fine_on = false;  // the batched launches restrict the patches this step
    invalidate_ledger(s);
    add_speed(s, coarse_shove_bound(L, ps, view_of(s)));
    out.spray_events = 1;
    *has_work = true;
    return SILT_OK;
}

int batch_launch(FineBatch* B, const std::vector<silt_sheet*>& sheets, const std::vector<Patches*>& patches, float dt,
                 cudaStream_t st) {
    const int n = (int)sheets.size();
    if (n == 0) return SILT_OK;
    size_t njobs = 0;
    int max_fres = 0;
    for (Patches* P : patches) {
        njobs += 2 * (size_t)H(*P).plan.np;
        max_fres = std::max(max_fres, P->fres);
    }
    const size_t rec_bytes = ((n * sizeof(FineRec)) + 255) & ~size_t(255);
    const size_t need = rec_bytes + njobs * sizeof(window::Job*);
    const int slot = B->flip;
    B->flip = (B->flip + 1) % STAGING_SLOTS;
    if (B->ev[slot]) FCK(cudaEventSynchronize(B->ev[slot]));
    if (need > B->cap[slot]) {
        cudaFree(B->d_buf[slot]);
        if (B->h_buf[slot]) cudaFreeHost(B->h_buf[slot]);
        B->d_buf[slot] = nullptr;
        B->h_buf[slot] = nullptr;
        B->cap[slot] = 0;
        const size_t cap = std::max(need * 2, (size_t)1 << 16);
        FCK(cudaMalloc(&B->d_buf[slot], cap));
        FCK(cudaMallocHost(&B->h_buf[slot], cap));
        B->cap[slot] = cap;
    }
    if (!B->ev[slot]) FCK(cudaEventCreateWithFlags(&B->ev[slot], cudaEventDisableTiming));
    FineRec* recs = reinterpret_cast<FineRec*>(B->h_buf[slot]);
    window::Job** jl = reinterpret_cast<window::Job**>(B->h_buf[slot] + rec_bytes);
    int mx_owner = 1, mx_cells = 1, mx_finish = 1, mx_push = 1, mx_pgroups = 0, mx_peel = 1, mx_qgroups = 0;
    int mx_restrict = 1, mx_cpush = 1;
    size_t q = 0;
    for (int w = 0; w < n; ++w) {
        silt_sheet* s = sheets[w];
        Patches& P = *patches[w];
        Impl& M = I(P);
        HostState& HS = H(P);
        const StepPlan& L = HS.plan;
        FineRec& r = recs[w];
        memset(&r, 0, sizeof r);
        r.W = view_of(s);
        r.refs = TAB(PatchRef, L.off_refs);
        r.tab = TAB(char, 0);
        r.np = L.np;
        r.fres = P.fres;
        r.sub = P.sub;
        r.park = L.any_park ? 1 : 0;
        r.fcell = P.fcell;
        r.dt = dt > 0.0f && std::isfinite(dt) ? dt : 0.0f;
        r.owner = M.owner;
        r.oidx = TAB(int, L.off_oidx);
        r.oval = TAB(int8_t, L.off_oval);
        r.n_owner = L.n_owner;
        r.held = TAB(int, L.off_held);
        r.n_held = (int)L.held.size();
        r.zero_blocks = r.n_held ? launch_blocks((size_t)r.n_held, 128) : 0;
        r.near = TAB(NearCol, L.off_near);
        r.n_apply = L.b_apply;
        r.ncap = L.b_ncap;
        r.fade = L.b_fade;
        r.push_groups = TAB(JobGroup, L.off_push_groups);
        r.n_push_groups = L.n_push_groups;
        r.peel_groups = TAB(JobGroup, L.off_peel_groups);
        r.n_peel_groups = L.n_peel_groups;
        r.ents = TAB(RestrictEntry, L.off_ent);
        r.n_ent = L.n_ent;
        r.rblocks = L.n_ent ? launch_blocks((size_t)L.n_ent * 32, 128) : 0;
        r.segs = TAB(Segment, L.off_seg);
        r.cpush = TAB(PushJob, L.coarse_push.off);
        r.cpush_n = L.coarse_push.n;
        r.cpush_i0 = L.coarse_push.i0;
        r.cpush_j0 = L.coarse_push.j0;
        r.cpush_w = L.coarse_push.n ? L.coarse_push.w : 0;
        r.cpush_h = L.coarse_push.n ? L.coarse_push.h : 0;
        r.slot_map = M.slot_map;
        r.pool = M.pool;
        r.meta = M.meta;
        r.free_stack = M.free_stack;
        r.counters = M.counters;
        r.spray = M.spray;
        r.books = M.d_books;
        r.park_table = M.park;
        window::Job* jobs = const_cast<window::Job*>(TAB(window::Job, L.off_jobs));
        for (int k = 0; k < 2 * L.np; ++k) jl[q++] = jobs + k;
        mx_owner = std::max(mx_owner, r.n_owner);
        mx_cells = std::max(mx_cells, r.np * r.fres * r.fres);
        mx_finish = std::max(mx_finish, r.zero_blocks + r.n_apply);
        mx_push = std::max(mx_push, L.push_cells_max);
        mx_pgroups = std::max(mx_pgroups, L.n_push_groups);
        mx_peel = std::max(mx_peel, L.peel_cells_max);
        mx_qgroups = std::max(mx_qgroups, L.n_peel_groups);
        mx_restrict = std::max(mx_restrict, r.ncap + r.rblocks);
        mx_cpush = std::max(mx_cpush, r.cpush_w * r.cpush_h);
    }
    FCK(cudaMemcpyAsync(B->d_buf[slot], B->h_buf[slot], need, cudaMemcpyHostToDevice, st));
    FCK(cudaEventRecord(B->ev[slot], st));
    const FineRec* d = reinterpret_cast<const FineRec*>(B->d_buf[slot]);
    window::Job* const* djl = reinterpret_cast<window::Job* const*>(B->d_buf[slot] + rec_bytes);
    const unsigned nz = (unsigned)n;
#define BLAUNCH(kern, gx, gy, threads)                                           \
    do {                                                                          \
        ::silt::launch_dep(kern, dim3(dim3((unsigned)(gx), (unsigned)(gy), nz)), dim3((threads)), 0, st, d); \
        ::silt::count_launch();                                                   \
        FCK(cudaGetLastError());                                                  \
    } while (0)
    BLAUNCH(kb_scatter, launch_blocks((size_t)mx_owner), 1, 256);
    BLAUNCH(kb_refine, launch_blocks((size_t)mx_cells), 1, 256);
    BLAUNCH(kb_lay_finish, mx_finish, 1, 128);
    BLAUNCH(kb_push, launch_blocks((size_t)mx_push), mx_pgroups + 1, 256);
    FCK(window::launch_window_step_list(djl, (int)njobs, max_fres, st));
    if (mx_qgroups) BLAUNCH(kb_peel_patches, launch_blocks((size_t)mx_peel), mx_qgroups, 256);
    BLAUNCH(kb_restrict, mx_restrict, 1, 128);
    BLAUNCH(kb_release, launch_blocks((size_t)mx_cells), 1, 256);
    BLAUNCH(kb_coarse_push, launch_blocks((size_t)mx_cpush), 1, 256);
#undef BLAUNCH
    return SILT_OK;
}

int batch_peel(FineBatch* B, const std::vector<silt_sheet*>& sheets, const std::vector<Patches*>& patches,
               cudaStream_t st) {
    const int n = (int)sheets.size();
    if (n == 0) return SILT_OK;
    const int slot = B->peel_flip;
    B->peel_flip = (B->peel_flip + 1) % STAGING_SLOTS;
    if (B->peel_ev[slot]) FCK(cudaEventSynchronize(B->peel_ev[slot]));
    if ((size_t)n > B->peel_cap[slot]) {
        cudaFree(B->d_peel[slot]);
        if (B->h_peel[slot]) cudaFreeHost(B->h_peel[slot]);
        B->d_peel[slot] = nullptr;
        B->h_peel[slot] = nullptr;
        B->peel_cap[slot] = 0;
        FCK(cudaMalloc(&B->d_peel[slot], 2 * (size_t)n * sizeof(PeelRec)));
        FCK(cudaMallocHost(&B->h_peel[slot], 2 * (size_t)n * sizeof(PeelRec)));
        B->peel_cap[slot] = 2 * (size_t)n;
    }
    if (!B->peel_ev[slot]) FCK(cudaEventCreateWithFlags(&B->peel_ev[slot], cudaEventDisableTiming));
    int mx = 1;
    for (int w = 0; w < n; ++w) {
        silt_sheet* s = sheets[w];
        Patches& P = *patches[w];
        Impl& M = I(P);
        HostState& HS = H(P);
        const StepPlan& L = HS.plan;
        PeelRec& r = B->h_peel[slot][w];
        memset(&r, 0, sizeof r);
        r.W = view_of(s);
        r.jobs = TAB(PushJob, L.coarse_peel.off);
        r.n = L.coarse_peel.n;
        r.i0 = L.coarse_peel.i0;
        r.j0 = L.coarse_peel.j0;
        r.w = L.coarse_peel.n ? L.coarse_peel.w : 0;
        r.h = L.coarse_peel.n ? L.coarse_peel.h : 0;
        r.owner = M.owner;
        r.spray = M.spray;
        r.counters = M.counters;
        r.books = M.d_books;
        mx = std::max(mx, r.w * r.h);
    }
    FCK(cudaMemcpyAsync(B->d_peel[slot], B->h_peel[slot], n * sizeof(PeelRec), cudaMemcpyHostToDevice, st));
    FCK(cudaEventRecord(B->peel_ev[slot], st));
    ::silt::launch_dep(kb_coarse_peel, dim3(dim3((unsigned)launch_blocks((size_t)mx), 1, (unsigned)n)), dim3(256), 0, st, B->d_peel[slot]);
    ::silt::count_launch();
    FCK(cudaGetLastError());
    return SILT_OK;
}

}  // namespace fine
}  // namespace silt
