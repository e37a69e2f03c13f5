// The sheet's tracers on the coarse window: foam, stirred silt (`turbid`)
// and wheel-lifted suspended solids (`susp`), as x3-team/Dirty-gen steps them
// (src/fluid_core.rs:6210-6739 step_tracers and its parts, :8758-8815
// entrain_wake, :8817-9002 advect_suspended).
//
// The reference walks index lists and applies each update in place, in order.
// Here every update is a per-cell kernel that reproduces that order:
//   * a cell's foam and silt sources (every tire in push order, then the
//     shore, then Froude breaking) run in one thread for that cell;
//   * the silt transport (flux_thickness) accumulates each donor's removals
//     in the reference's edge order, so a cell recomputes, for itself and its
//     four neighbours, the donor sequence up to the edge it shares;
//   * the suspended transport lets a receiver take from its neighbours in the
//     reference's raster order of donors (a receiver's room depends on what
//     earlier donors gave it): receivers write each accepted give into the
//     donor's slot, then each donor subtracts its slots in its own order.
// Books that the reference sums in f32 in list order are FP64 sums of the
// same f32 terms. Index boxes (the live silt span, the visit box) are device
// reductions, and every kernel reads the step's control flags on the device,
// so the host never waits.
#include "sheet_tracers.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "block_sum.cuh"
#include "launch_count.cuh"
#include "sheet_math.cuh"

namespace silt {
namespace tracers {

namespace {

constexpr float FOAM_EQ = 0.85f;             // src/fluid_core.rs:115
constexpr float FOAM_TAU_S = 0.35f;          // :117
constexpr float SUSP_FALL_M_S = 0.004f;      // :122
constexpr float SILT_COLUMN_CAP_M = 0.028f;  // :124

enum : uint8_t { WET = 1, SHORE = 2, LIVE = 4 };

// Per-step control, in State plus these words (kept after State in memory).
struct Ctl {
    int active;     // the tracer step runs at all (wake, live silt or live foam)
    int cbox[4];    // the step's collection box
    int tspan2[4];  // silt span after the transport
    int tspan3[4];  // silt span after the sources
    int mbox[4];    // where wet and shore marks may be set (the last collection box)
    int ssup[4];    // this step's suspended pass: a box holding every cell whose load is not 0
    int ssup_next[4];  // the same for the next step, grown by every writer of the load
    unsigned int live_foam_prev;
};

__device__ __forceinline__ Ctl* ctl_of(State* s) { return reinterpret_cast<Ctl*>(s + 1); }

// The tracer step goes on past the wet set (:6226-6229): it runs at all and
// has wet cells or live silt. Final once the wet-set pass has ended.
__device__ __forceinline__ bool step_goes(const State* st) {
    const Ctl* c = reinterpret_cast<const Ctl*>(st + 1);
    return c->active && (st->wet_any || st->live_silt);
}

__device__ __forceinline__ float vel(const float* u, const Sheet& S, size_t g) {
    // The grid engine's pending dry cut: a cell under eps carries no velocity.
    return (S.cut_pending && S.water[g] < 1.0e-6f) ? 0.0f : u[g];
}

__device__ __forceinline__ float smoothstep_f(float e0, float e1, float x) {  // :9688-9691
    float t = rclamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

__device__ __forceinline__ float breaking_foam(float speed, float thickness) {  // :9676-9686
    if (!finite_f(speed) || !finite_f(thickness) || thickness < 0.004f || speed <= 0.05f) return 0.0f;
    const float froude = speed / sqrtf(9.81f * thickness);
    return smoothstep_f(0.85f, 1.45f, froude);
}

__device__ __forceinline__ float sample_foam(const float* src, int res, float x, float z) {  // :9693-9712
    if (!finite_f(x) || !finite_f(z) || x < 0.0f || z < 0.0f) return 0.0f;
    const float fx = floorf(x), fz = floorf(z);
    if (fx >= (float)res || fz >= (float)res) return 0.0f;
    const int i0 = (int)fx, j0 = (int)fz;
    const int i1 = min(i0 + 1, res - 1), j1 = min(j0 + 1, res - 1);
    const float tx = rclamp(x - (float)i0, 0.0f, 1.0f), tz = rclamp(z - (float)j0, 0.0f, 1.0f);
    const float a = src[(size_t)j0 * res + i0], b = src[(size_t)j0 * res + i1];
    const float c = src[(size_t)j1 * res + i0], d = src[(size_t)j1 * res + i1];
    const float v = a + (b - a) * tx + (c - a) * tz + (a - b - c + d) * tx * tz;
    return finite_f(v) ? rclamp(v, 0.0f, 1.0f) : 0.0f;
}

// shore_cell (:9826-9872): foam production and silt lift rate of a wet cell.
__device__ __forceinline__ void shore_cell(const Sheet& S, int i, int j, float& foam, float& rate) {
    foam = 0.0f;
    rate = 0.0f;
    const int res = S.res;
    if (i == 0 || j == 0 || i + 1 >= res || j + 1 >= res) return;
    const size_t g = (size_t)j * res + i;
    const float h = S.water[g];
    if (!finite_f(h) || h < 0.004f) return;
    float nx = 0.0f, nz = 0.0f;
    bool edge = false;
    const int di[4] = {-1, 1, 0, 0}, dj[4] = {0, 0, -1, 1};
    for (int k = 0; k < 4; ++k) {
        const float nh = S.water[(size_t)(j + dj[k]) * res + (i + di[k])];
        if (finite_f(nh) && nh < 0.004f) {
            edge = true;
            nx += (float)di[k];
            nz += (float)dj[k];
        }
    }
    if (!edge) return;
    const float u = vel(S.uw, S, g), v = vel(S.vw, S, g);
    if (!finite_f(u) || !finite_f(v)) return;
    const float film = hypot_rn(u, v);
    const float nlen = fmaxf(hypot_rn(nx, nz), 1.0e-4f);
    const float into = fmaxf((u * nx + v * nz) / nlen, 0.0f);
    const float strain = fabsf(vel(S.uw, S, g + 1) - vel(S.uw, S, g - 1)) + fabsf(vel(S.vw, S, g + res) - vel(S.vw, S, g - res));
    const float shear_v = fmaxf(film, strain);
    if (shear_v < 0.2f && into < 0.2f) return;
    const float prod = fmaxf(breaking_foam(fmaxf(shear_v, into), h), smoothstep_f(0.25f, 1.1f, into));
    foam = prod > 0.02f ? prod : 0.0f;
    if (h > 0.012f && h < 0.055f && (shear_v > 0.45f || into > 0.4f)) {
        const float tau = 1000.0f * 0.025f * shear_v * shear_v;
        if (tau > 3.0f || into > 0.45f) rate = fminf(0.006f * (into + shear_v * 0.35f), 0.01f);
    }
}

// add_foam (:6400-6418) on the cell's value.
__device__ __forceinline__ void add_foam(float& f, float prod, float dt) {
    if (prod <= 0.0f || !finite_f(prod) || !(dt > 0.0f)) return;
    const float cur = finite_f(f) ? rclamp(f, 0.0f, FOAM_EQ) : 0.0f;
    const float room = FOAM_EQ - cur;
    if (room <= 1.0e-5f) return;
    const float grown = cur + room * prod * fminf(dt / FOAM_TAU_S, 1.0f);
    f = finite_f(grown) ? fminf(grown, FOAM_EQ) : 0.0f;
}

// add_silt (:6699-6710); the stirred volume goes to `book`.
__device__ __forceinline__ void add_silt(float& t, float dh, float area, double& book) {
    if (dh <= 0.0f || !finite_f(dh)) return;
    const float room = fmaxf(SILT_COLUMN_CAP_M - fmaxf(t, 0.0f), 0.0f);
    const float add = fminf(dh, room);
    if (add <= 0.0f) return;
    t += add;
    book += (double)(add * area);
}

__device__ __forceinline__ void block_book(double v, double* book) { ::silt::block_add(v, book); }
__device__ __forceinline__ void block_count(unsigned int v, unsigned int* to) { ::silt::block_add(v, to); }

// Sets *flag when any thread of the block passes `any`.
__device__ __forceinline__ void block_flag(bool any, unsigned int* flag) {
    if (__syncthreads_or(any) && threadIdx.x == 0) *flag = 1u;
}


// A thread's own box of cells, merged over the warp and added with one
// atomic per bound.
struct LocalBox {
    int b[4] = {0x7fffffff, -1, 0x7fffffff, -1};
    __device__ __forceinline__ void add(int i, int j) {
        b[0] = min(b[0], i);
        b[1] = max(b[1], i);
        b[2] = min(b[2], j);
        b[3] = max(b[3], j);
    }
    // Merged over the block, then one atomic per bound. Every thread of the
    // block calls it.
    __device__ __forceinline__ void commit(int* box) {
        __shared__ int part[4][32];
        for (int o = 16; o > 0; o >>= 1) {
            b[0] = min(b[0], __shfl_down_sync(0xffffffffu, b[0], o));
            b[1] = max(b[1], __shfl_down_sync(0xffffffffu, b[1], o));
            b[2] = min(b[2], __shfl_down_sync(0xffffffffu, b[2], o));
            b[3] = max(b[3], __shfl_down_sync(0xffffffffu, b[3], o));
        }
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0)
            for (int k = 0; k < 4; ++k) part[k][warp] = b[k];
        __syncthreads();
        if (warp == 0) {
            const bool have = lane < (int)(blockDim.x >> 5);
            b[0] = have ? part[0][lane] : 0x7fffffff;
            b[1] = have ? part[1][lane] : -1;
            b[2] = have ? part[2][lane] : 0x7fffffff;
            b[3] = have ? part[3][lane] : -1;
            for (int o = 16; o > 0; o >>= 1) {
                b[0] = min(b[0], __shfl_down_sync(0xffffffffu, b[0], o));
                b[1] = max(b[1], __shfl_down_sync(0xffffffffu, b[1], o));
                b[2] = min(b[2], __shfl_down_sync(0xffffffffu, b[2], o));
                b[3] = max(b[3], __shfl_down_sync(0xffffffffu, b[3], o));
            }
            if (lane == 0 && b[1] >= 0) {
                atomicMin(&box[0], b[0]);
                atomicMax(&box[1], b[1]);
                atomicMin(&box[2], b[2]);
                atomicMax(&box[3], b[3]);
            }
        }
        __syncthreads();
    }
};

__device__ __forceinline__ void box_clear(int* box, int res) {
    box[0] = res;
    box[1] = -1;
    box[2] = res;
    box[3] = -1;
}

__device__ __forceinline__ bool box_empty(const int* b) { return b[0] > b[1]; }

// turbid_span's result (:9766-9795): the box grown by one, clamped.
__device__ __forceinline__ void grown(const int* b, int res, int& i0, int& i1, int& j0, int& j1) {
    i0 = max(b[0] - 1, 0);
    i1 = min(b[1] + 1, res - 1);
    j0 = max(b[2] - 1, 0);
    j1 = min(b[3] + 1, res - 1);
}

// Every cell of the job's window (blockIdx.y is the job, blockIdx.x strides
// its cells). Indices are 32-bit: a window holds fewer than 2^32 cells.
#define CELLS(S)                                                                                                  \
    for (unsigned g = blockIdx.x * blockDim.x + threadIdx.x, n_ = (unsigned)(S).res * (unsigned)(S).res; g < n_; \
         g += gridDim.x * blockDim.x)

// The cells (i, j, g) of the box [i0, i1] x [j0, j1] (inclusive) of a window
// `res` cells wide; `continue` moves to the next cell.
#define BOX_CELLS(res, i0, i1, j0, j1)                                                                  \
    for (unsigned q_ = blockIdx.x * blockDim.x + threadIdx.x, w_ = (unsigned)max((i1) - (i0) + 1, 0),    \
                  n_ = w_ * (unsigned)max((j1) - (j0) + 1, 0);                                          \
         q_ < n_; q_ += gridDim.x * blockDim.x)                                                        \
        for (int once_ = 1, i = (i0) + (int)(q_ % w_), j = (j0) + (int)(q_ / w_); once_; once_ = 0)        \
            for (unsigned g = (unsigned)j * (unsigned)(res) + (unsigned)i; once_; once_ = 0)

// The 128-cell segments of a row of a `res`-wide window (cells 128 s .. 128 s + 127).
__host__ __device__ __forceinline__ int segments(int res) { return (res + 127) / 128; }

// QUAD_ROWS over whole segments: every segment that meets the columns
// [i0, i1], in the rows [j0, j1], one per warp iteration. Declares j, s and
// ib = 128 s + lane; the cells outside [i0, i1] are the caller's to skip.
#define QUAD_SEGS(res, i0, i1, j0, j1)                                                                          \
    for (unsigned it_ = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, s0_ = (unsigned)max((i0), 0) >> 7,        \
                  nx_ = (i1) >= (i0) ? ((unsigned)(i1) >> 7) - s0_ + 1u : 0u,                                 \
                  n_ = nx_ * (unsigned)max((j1) - (j0) + 1, 0);                                               \
         it_ < n_; it_ += (gridDim.x * blockDim.x) >> 5)                                                        \
        for (int once_ = 1, j = (j0) + (int)(it_ / nx_), s = (int)(s0_ + it_ % nx_), ib = s * 128 + (int)(threadIdx.x & 31); \
             once_; once_ = 0)

// Four cells per thread for the passes over whole windows: a warp takes 128
// consecutive cells of a row of the box, lane l the cells ib, ib + 32,
// ib + 64, ib + 96 with ib = start + l (each load coalesced; a thread's four
// loads independent). Declares j and ib.
#define QUAD_ROWS(res, i0, i1, j0, j1)                                                                          \
    for (unsigned it_ = (blockIdx.x * blockDim.x + threadIdx.x) >> 5,                                           \
                  nx_ = (unsigned)max((i1) - (i0) + 128, 0) / 128u, n_ = nx_ * (unsigned)max((j1) - (j0) + 1, 0); \
         it_ < n_; it_ += (gridDim.x * blockDim.x) >> 5)                                                        \
        for (int once_ = 1, j = (j0) + (int)(it_ / nx_), ib = (i0) + (int)(it_ % nx_) * 128 + (int)(threadIdx.x & 31); \
             once_; once_ = 0)

// The job is copied into registers: the planes' stores would otherwise make
// the compiler reload its fields from memory after every write.
#define JOB                              \
    const Job J = jobs[blockIdx.y];      \
    const Sheet& S = J.S;                \
    const Planes& T = J.T;               \
    (void)S;                             \
    (void)T

// A box read from device memory into registers.
struct Box {
    int i0, i1, j0, j1;
    __device__ __forceinline__ bool empty() const { return i0 > i1 || j0 > j1; }
};
__device__ __forceinline__ Box box_of(const int* b) { return Box{b[0], b[1], b[2], b[3]}; }
__device__ __forceinline__ Box grown_box(const int* b, int res) {
    Box r;
    grown(b, res, r.i0, r.i1, r.j0, r.j1);
    return r;
}
__device__ __forceinline__ Box box_union(Box a, Box b) {
    if (a.empty()) return b;
    if (b.empty()) return a;
    return Box{min(a.i0, b.i0), max(a.i1, b.i1), min(a.j0, b.j0), max(a.j1, b.j1)};
}

// True when the warp's 128 cells of row j from column ib0 on hold no wet or
// foam-live mark (the flags of the one or two segments they meet, as this
// step's wet-set pass left them) and meet no cell of box b: a pass that acts
// only on such marks and on the cells of b has nothing to do there. Flags of
// segments the wet-set pass did not visit may be stale, but such segments
// lie outside its box, where no cell carries a mark.
__device__ __forceinline__ bool quiet_run(const uint8_t* occ, int res, int j, int ib0, const Box& b) {
    const int ns = segments(res);
    const int s0 = ib0 >> 7, s1 = min((ib0 + 127) >> 7, ns - 1);
    if (occ[j * ns + s0] | occ[j * ns + s1]) return false;
    return b.empty() || j < b.j0 || j > b.j1 || ib0 + 127 < b.i0 || ib0 > b.i1;
}
__device__ __forceinline__ bool in_box(const Box& b, int i, int j) {
    return i >= b.i0 && i <= b.i1 && j >= b.j0 && j <= b.j1;
}

// ------------------------------------------------------------ entrain_wake

__global__ void k_entrain(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    float* susp = T.susp[0];
    const float dt = J.dt;
    const int res = S.res;
    const float cell = S.cell, area = cell * cell;
    double b = 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0 && J.ebox[0] <= J.ebox[1]) {
        int* sup = ctl_of(T.st)->ssup_next;  // the wake's cells may now hold a load
        atomicMin(&sup[0], J.ebox[0]);
        atomicMax(&sup[1], J.ebox[1]);
        atomicMin(&sup[2], J.ebox[2]);
        atomicMax(&sup[3], J.ebox[3]);
    }
    BOX_CELLS(res, J.ebox[0], J.ebox[1], J.ebox[2], J.ebox[3]) {
        for (int k = 0; k < J.npush; ++k) {
            const silt_tire_push& p = J.push[k];
            if (p.speed < 0.3f) continue;
            const float fl = fmaxf(sqrtf(p.forward_x * p.forward_x + p.forward_z * p.forward_z), 1.0e-4f);
            const float fx = p.forward_x / fl, fz = p.forward_z / fl;
            const float rx = fz, rz = -fx;
            const float reach = p.radius * 3.4f + cell;
            const int i0 = (int)floorf(((p.x - reach) - S.ox) / cell);
            const int i1 = (int)floorf(((p.x + reach) - S.ox) / cell);
            const int j0 = (int)floorf(((p.z - reach) - S.oz) / cell);
            const int j1 = (int)floorf(((p.z + reach) - S.oz) / cell);
            if (i < max(i0, 0) || i > min(i1, res - 1) || j < max(j0, 0) || j > min(j1, res - 1)) continue;
            const float aft = p.radius * 3.2f;
            const float half = p.width * 0.55f + 0.08f;
            const float x = S.ox + ((float)i + 0.5f) * cell;
            const float z = S.oz + ((float)j + 0.5f) * cell;
            const float dx = x - p.x, dz = z - p.z;
            const float along = dx * fx + dz * fz;
            if (along > -0.05f || along < -aft) continue;
            const float lat = fabsf(dx * rx + dz * rz);
            if (lat > half) continue;
            const float water = S.water[g];
            if (!finite_f(water) || water < 0.004f) continue;
            const float along_t = rclamp((-along) / aft, 0.0f, 1.0f);
            const float lat_t = rclamp(lat / half, 0.0f, 1.0f);
            const float core = (1.0f - along_t) * (1.0f - lat_t);
            const float room = fmaxf(water - susp[g], 0.0f);
            const float add = fminf(4.0f * dt * core * water, room);
            if (add <= 1.0e-8f) continue;
            susp[g] += add;
            b += (double)(add * area);
        }
    }
    block_book(b, T.books + 0);
}

// ------------------------------------------------------------ step_tracers
//
// The silt span at a step's start (turbid_span, :9766-9795) is kept exact
// between steps instead of scanned: every kernel that changes silt records
// the box of the cells it leaves above 1e-8, and a cell outside the region a
// kernel touches keeps a value that was already at most 1e-8. A scan of the
// whole window runs only after the planes were rewritten wholesale (attach,
// window moves). Launches: [scan], begin (control words and the collection
// box), collect (with the foam advection into scratch), the silt advection
// into scratch, commit, settle (with the sync's start), spawn, clear and sync.

// The start span of the jobs whose planes were rewritten (`rescan`); the
// reset that rewrote them left the span empty.
__global__ void k_scan(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    if (!J.rescan) return;
    const float* turbid = T.turbid[0];
    const int res = S.res;
    LocalBox lb;
    CELLS(S) {
        if (turbid[g] > 1.0e-8f) lb.add((int)(g % res), (int)(g / res));
    }
    lb.commit(T.st->tspan);
}

// The step's control words, then collect_tracer_wet's box (:6248-6293) and
// tracer_visit_box (:6296-6337). `wake`: a tire with speed or slip, or a
// surface drive (host-known); `pbox`: the tires' reach boxes (host-computed;
// empty when none).
__global__ void k_begin(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    State* st = T.st;
    const int res = S.res, wake = J.wake;
    Ctl* c = ctl_of(st);
    box_clear(c->tspan2, res);
    box_clear(c->tspan3, res);
    box_clear(c->cbox, res);
    st->live_silt = box_empty(st->tspan) ? 0u : 1u;
    st->wet_any = 0;
    c->live_foam_prev = st->live_foam;
    c->active = (wake || st->live_silt || c->live_foam_prev) ? 1 : 0;
    if (!c->active) return;
    if (wake) {
        c->cbox[0] = 0;
        c->cbox[1] = res - 1;
        c->cbox[2] = 0;
        c->cbox[3] = res - 1;
        return;
    }
    int b[4] = {res, -1, res, -1};
    bool any = false;
    auto take = [&](int i0, int i1, int j0, int j1) {
        b[0] = min(b[0], i0);
        b[1] = max(b[1], i1);
        b[2] = min(b[2], j0);
        b[3] = max(b[3], j1);
        any = true;
    };
    if (c->live_foam_prev) take(st->live_box[0], st->live_box[1], st->live_box[2], st->live_box[3]);
    if (!box_empty(st->tspan)) {
        int i0, i1, j0, j1;
        grown(st->tspan, res, i0, i1, j0, j1);
        take(i0, i1, j0, j1);
    }
    if (J.pbox[0] <= J.pbox[1]) take(J.pbox[0], J.pbox[1], J.pbox[2], J.pbox[3]);
    if (!any) return;  // cbox stays empty
    c->cbox[0] = max(b[0] - 2, 0);
    c->cbox[1] = min(b[1] + 2, res - 1);
    c->cbox[2] = max(b[2] - 2, 0);
    c->cbox[3] = min(b[3] + 2, res - 1);
}


// The silt a donor cell gives across its four edges in flux_thickness's
// order (x edges before z edges, each axis in index order): to the left,
// right, up and down neighbour (0 where it is not the donor or the edge lies
// outside the box). flux_edge (:9857-9876) with the donor's running removal.
__device__ __forceinline__ void donor_flux(const Sheet& S, const float* T, int i, int j, int bi0, int bi1, int bj0,
                                           int bj1, float dt, float out[4]) {
    const int res = S.res;
    const size_t d = (size_t)j * res + i;
    const float column = finite_f(T[d]) ? T[d] : 0.0f;
    float removed = 0.0f;
    out[0] = out[1] = out[2] = out[3] = 0.0f;
    if (column <= 1.0e-8f) return;  // every edge finds no room: nothing to read
    auto edge = [&](float v, bool donor_is_me) -> float {
        if (!finite_f(v) || fabsf(v) < 1.0e-5f || !donor_is_me) return 0.0f;
        const float room = column - removed;
        if (room <= 1.0e-8f) return 0.0f;
        const float frac = fminf(fabsf(v) * dt / S.cell, 0.45f);
        const float dh = fminf(column * frac, room);
        if (dh <= 1.0e-8f || !finite_f(dh)) return 0.0f;
        removed += dh;
        return dh;
    };
    if (i - 1 >= bi0 && i <= bi1) {  // edge (i-1, i): this cell donates when the face speed is not positive
        const float v = 0.5f * (vel(S.uw, S, d - 1) + vel(S.uw, S, d));
        out[0] = edge(v, !(v > 0.0f));
    }
    if (i >= bi0 && i <= bi1 - 1) {  // edge (i, i+1)
        const float v = 0.5f * (vel(S.uw, S, d) + vel(S.uw, S, d + 1));
        out[1] = edge(v, v > 0.0f);
    }
    if (j - 1 >= bj0 && j <= bj1) {  // edge (j-1, j)
        const float v = 0.5f * (vel(S.vw, S, d - res) + vel(S.vw, S, d));
        out[2] = edge(v, !(v > 0.0f));
    }
    if (j >= bj0 && j <= bj1 - 1) {  // edge (j, j+1)
        const float v = 0.5f * (vel(S.vw, S, d) + vel(S.vw, S, d + res));
        out[3] = edge(v, v > 0.0f);
    }
}

// advect_turbid (:6421-6470) of cell (i, j) of the grown span: its new silt.
__device__ __forceinline__ float turbid_after(const Sheet& S, const float* T, int i, int j, int bi0, int bi1, int bj0,
                                              int bj1, float dt) {
    const size_t g = (size_t)j * S.res + i;
    float own[4], nb[4];
    donor_flux(S, T, i, j, bi0, bi1, bj0, bj1, dt, own);
    float removed = 0.0f;
    for (int k = 0; k < 4; ++k)
        if (own[k] > 0.0f) removed += own[k];
    // What the neighbours give this cell, in the reference's edge order.
    float added = 0.0f;
    if (i - 1 >= bi0) {
        donor_flux(S, T, i - 1, j, bi0, bi1, bj0, bj1, dt, nb);
        if (nb[1] > 0.0f) added += nb[1];
    }
    if (i + 1 <= bi1) {
        donor_flux(S, T, i + 1, j, bi0, bi1, bj0, bj1, dt, nb);
        if (nb[0] > 0.0f) added += nb[0];
    }
    if (j - 1 >= bj0) {
        donor_flux(S, T, i, j - 1, bi0, bi1, bj0, bj1, dt, nb);
        if (nb[3] > 0.0f) added += nb[3];
    }
    if (j + 1 <= bj1) {
        donor_flux(S, T, i, j + 1, bi0, bi1, bj0, bj1, dt, nb);
        if (nb[2] > 0.0f) added += nb[2];
    }
    float t = T[g];
    if (removed == 0.0f && added == 0.0f) {
        if (!finite_f(t)) t = 0.0f;
    } else {
        const float next = t - removed + added;
        t = finite_f(next) ? fmaxf(next, 0.0f) : 0.0f;
    }
    return t;
}

// The wet set (marks) and, into scratch, advect_foam (:6352-6397) of every
// wet or foam-live cell; k_turbid_advect puts advect_turbid of the grown span
// beside it. Both read only fields no step kernel has changed yet; whether
// they take effect is decided once the wet set is known (k_go, k_commit).
__global__ void __launch_bounds__(256, 3) k_collect(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    uint8_t* mark = T.mark;
    State* st = T.st;
    Ctl* c = ctl_of(st);
    if (!c->active) return;
    const int res = S.res;
    const float dt = J.dt, decay = J.foam_decay;
    const float* foam = T.foam[0];
    float* ftmp = T.foam[1];
    const bool foam_on = c->live_foam_prev != 0;
    // Wet and shore marks are cleared where the last collection may have set
    // them and set inside this step's box; live marks stay.
    const Box b = box_of(c->cbox);
    const Box u = box_union(b, box_of(c->mbox));
    bool any = false;
    const int ns = segments(res);
    QUAD_SEGS(res, u.i0, u.i1, u.j0, u.j1) {
        // The four cells' loads in two rounds: marks and depths, then, for the
        // wet cells only, the four neighbours' water of the shore test
        // (shore_wet_cell, :9752-9764: a cell on the window's border is never
        // shore) and the velocity the foam advection reads.
        uint8_t mk[4];
        float hw[4], hs[4], nb[4][4], uw4[4], vw4[4];
        bool here[4], wet[4], inner[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = ib + 32 * k;
            const unsigned g = (unsigned)j * (unsigned)res + (unsigned)i;
            here[k] = i >= u.i0 && i <= u.i1;
            wet[k] = false;
            if (here[k]) mk[k] = mark[g];
            if (here[k] && in_box(b, i, j)) {
                hw[k] = S.water[g];
                hs[k] = S.slurry[g];
                wet[k] = true;
            }
        }
        // A segment with no wet cell and no foam-live mark: its cells' marks
        // become 0 and nothing else happens there.
        bool busy = false;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (here[k] && (mk[k] & LIVE)) busy = true;
            if (wet[k]) {
                const float h = hw[k] + hs[k];
                if (finite_f(h) && !(h < 0.004f)) busy = true;
            }
        }
        if (!__any_sync(0xffffffffu, busy)) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (here[k] && mk[k] != 0) mark[(unsigned)j * (unsigned)res + (unsigned)(ib + 32 * k)] = 0;
            if ((threadIdx.x & 31) == 0) T.occ[j * ns + s] = 0;
            continue;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = ib + 32 * k;
            const unsigned g = (unsigned)j * (unsigned)res + (unsigned)i;
            if (wet[k]) {
                const float h = hw[k] + hs[k];
                wet[k] = finite_f(h) && !(h < 0.004f);
            }
            inner[k] = i > 0 && j > 0 && i + 1 < res && j + 1 < res;
            if (!wet[k]) continue;
            if (inner[k]) {
                nb[k][0] = S.water[g - 1];
                nb[k][1] = S.water[g + 1];
                nb[k][2] = S.water[g - res];
                nb[k][3] = S.water[g + res];
            }
            if (foam_on) {
                uw4[k] = S.uw[g];
                vw4[k] = S.vw[g];
            }
        }
        bool marked = false;  // a wet or foam-live mark among this thread's cells
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (!here[k]) continue;
            const int i = ib + 32 * k;
            const unsigned g = (unsigned)j * (unsigned)res + (unsigned)i;
            uint8_t m = mk[k] & LIVE;
            if (wet[k]) {
                m |= WET;
                any = true;
                bool shore = false;
                if (inner[k])
                    for (int q = 0; q < 4; ++q) shore = shore || (finite_f(nb[k][q]) && nb[k][q] < 0.004f);
                if (shore) m |= SHORE;
            }
            mark[g] = m;
            marked = marked || m != 0;
            if (foam_on) {
                if (m & WET) {
                    const float uu = uw4[k], vv = vw4[k];  // wet cells are far above the dry cut
                    float sample = 0.0f;
                    if (finite_f(uu) && finite_f(vv)) {
                        const float x = (float)i - uu * dt / S.cell;
                        const float z = (float)j - vv * dt / S.cell;
                        sample = sample_foam(foam, res, x, z);
                    }
                    const float fv = sample * decay;
                    ftmp[g] = (fv > 1.0e-4f && finite_f(fv)) ? fminf(fv, FOAM_EQ) : 0.0f;
                } else if (m & LIVE) {
                    ftmp[g] = 0.0f;
                }
            }
        }
        // The warp holds the whole segment (the cells outside the box carry no mark).
        const unsigned seg = __ballot_sync(0xffffffffu, marked);
        if ((threadIdx.x & 31) == 0) T.occ[j * ns + s] = seg != 0u ? 1 : 0;
    }
    block_flag(any, &st->wet_any);
}

// advect_turbid of the grown span into scratch, spread over every block of
// the launch (a cell's donor sequences are long; in the wet-set pass the
// few warps holding the span's rows would carry all of them).
__global__ void k_turbid_advect(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    State* st = T.st;
    if (!ctl_of(st)->active || box_empty(st->tspan)) return;
    const int res = S.res;
    const Box tb = grown_box(st->tspan, res);
    const float* silt = T.turbid[0];
    float* ttmp = T.turbid[1];
    BOX_CELLS(res, tb.i0, tb.i1, tb.j0, tb.j1) {
        // A cell without silt beside neighbours without silt (those inside the
        // span) keeps its value: every edge of those columns gives 0.
        const bool still = silt[g] == 0.0f && (i - 1 < tb.i0 || silt[g - 1] == 0.0f) &&
                           (i + 1 > tb.i1 || silt[g + 1] == 0.0f) && (j - 1 < tb.j0 || silt[g - res] == 0.0f) &&
                           (j + 1 > tb.j1 || silt[g + res] == 0.0f);
        ttmp[g] = still ? silt[g] : turbid_after(S, silt, i, j, tb.i0, tb.i1, tb.j0, tb.j1, J.dt);
    }
}

// The advections take effect: foam on every wet or foam-live cell, silt on
// the grown span, whose cells above 1e-8 are the span after the transport
// (outside it no cell holds more than 1e-8).
__global__ void k_commit(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    State* st = T.st;
    Ctl* c = ctl_of(st);
    if (!step_goes(st)) return;
    const int res = S.res;
    const bool foam_on = c->live_foam_prev != 0, silt_on = !box_empty(st->tspan);
    if (!foam_on && !silt_on) return;
    const Box fb = foam_on ? box_of(c->cbox) : Box{0, -1, 0, -1};
    const Box tb = silt_on ? grown_box(st->tspan, res) : Box{0, -1, 0, -1};
    const Box u = box_union(fb, tb);
    float* foam = T.foam[0];
    const float* ftmp = T.foam[1];
    float* silt = T.turbid[0];
    const float* ttmp = T.turbid[1];
    const uint8_t* mark = T.mark;
    LocalBox lb;
    QUAD_ROWS(res, u.i0, u.i1, u.j0, u.j1) {
        if (quiet_run(T.occ, res, j, ib - (int)(threadIdx.x & 31), tb)) continue;
        bool fo[4];
        float fv[4], tv[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = ib + 32 * k;
            fo[k] = i <= u.i1 && in_box(fb, i, j) && (mark[(unsigned)j * (unsigned)res + (unsigned)i] & (WET | LIVE));
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = ib + 32 * k;
            const unsigned g = (unsigned)j * (unsigned)res + (unsigned)i;
            if (fo[k]) fv[k] = ftmp[g];
            if (i <= u.i1 && in_box(tb, i, j)) tv[k] = ttmp[g];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = ib + 32 * k;
            const unsigned g = (unsigned)j * (unsigned)res + (unsigned)i;
            if (fo[k]) foam[g] = fv[k];
            if (i <= u.i1 && in_box(tb, i, j)) {
                silt[g] = tv[k];
                if (tv[k] > 1.0e-8f) lb.add(i, j);
            }
        }
    }
    lb.commit(c->tspan2);
}

// settle_turbid (:6473-6509) on the span after the transport; the cells it
// leaves above 1e-8 go into the span after the sources.
__global__ void k_settle(const Job* jobs) {
    ::silt::dep_wait();
    const Job J = jobs[blockIdx.y];
    const Sheet& S = J.S;
    float* T = J.T.turbid[0];
    State* st = J.T.st;
    const float keep = J.silt_keep;
    double* book = J.T.books + 3;
    Ctl* c = ctl_of(st);
    if (blockIdx.x == 0 && threadIdx.x == 0 && c->active) {
        // The sync's start (:6339): the marks' box for the next step's wet
        // set, and the live set and start span, rebuilt by k_clear_sync.
        for (int k = 0; k < 4; ++k) c->mbox[k] = c->cbox[k];
        if (step_goes(st)) {
            st->live_foam = 0;
            box_clear(st->live_box, S.res);
            box_clear(st->tspan, S.res);
        }
    }
    if (!step_goes(st) || box_empty(c->tspan2)) return;
    const int res = S.res;
    const float area = S.cell * S.cell;
    int bi0, bi1, bj0, bj1;
    grown(c->tspan2, res, bi0, bi1, bj0, bj1);
    double b = 0.0;
    LocalBox lb;
    BOX_CELLS(res, bi0, bi1, bj0, bj1) {
        const float h = S.water[g] + S.slurry[g];
        const float column = finite_f(T[g]) ? fmaxf(T[g], 0.0f) : 0.0f;
        if (column <= 0.0f) {
            T[g] = 0.0f;
            continue;
        }
        if (!finite_f(h) || h < 1.0e-5f) {
            b += (double)(column * area);
            T[g] = 0.0f;
            continue;
        }
        const float stay = column * keep;
        b += (double)((column - stay) * area);
        T[g] = stay;
        if (stay > 1.0e-8f) lb.add(i, j);
    }
    lb.commit(c->tspan3);
    block_book(b, book);
}

// A tire push's constants for spawn_tire_tracers (:6599-6665), computed once
// per block; `live`: the tire moves or slips.
struct PushK {
    float x, z, speed, radius, fx, fz, rx, rz, reach2, slip_v, width;
    int live;
};

__device__ __forceinline__ PushK push_k(const silt_tire_push& p, float cell) {
    PushK q;
    q.speed = finite_f(p.speed) ? fmaxf(p.speed, 0.0f) : 0.0f;
    const float slip = finite_f(p.slip) ? fminf(fabsf(p.slip), 1.5f) : 0.0f;
    q.live = !(q.speed < 0.25f && slip < 0.05f);
    q.radius = fmaxf(p.radius, 0.05f);
    const float len = fmaxf(sqrtf(p.forward_x * p.forward_x + p.forward_z * p.forward_z), 1.0e-4f);
    q.fx = p.forward_x / len;
    q.fz = p.forward_z / len;
    q.rx = q.fz;
    q.rz = -q.fx;
    const float reach = q.radius * 1.15f + cell;
    q.reach2 = reach * reach;
    q.slip_v = q.speed * slip;
    q.x = p.x;
    q.z = p.z;
    q.width = p.width;
    return q;
}

constexpr int SPAWN_SHARED_PUSHES = 32;

// spawn_foam_and_silt (:6511-6520) on one wet cell (water h, film velocity
// u, v, slurry hs): the tires in push order (spawn_tire_tracers :6599-6665),
// then the shore (spawn_shore_tracers :6667-6684) and Froude breaking
// (spawn_breaking_speed :6545-6558). `table`: the pushes' constants, or null
// to compute them from `push` here.
__device__ __forceinline__ void spawn_cell(const Sheet& S, int i, int j, uint8_t m, float h, float hs, float u,
                                           float v, const PushK* table, const silt_tire_push* push, int np, float dt,
                                           float& f, float& t, double& b) {
    const float cell = S.cell, area = cell * cell;
    for (int k = 0; k < np; ++k) {
        const PushK q = table ? table[k] : push_k(push[k], cell);
        if (!q.live) continue;
        if (!finite_f(h) || h < 0.004f) continue;
        const float x = S.ox + ((float)i + 0.5f) * cell;
        const float z = S.oz + ((float)j + 0.5f) * cell;
        const float dx = x - q.x, dz = z - q.z;
        if (dx * dx + dz * dz > q.reach2) continue;
        const float along = dx * q.fx + dz * q.fz;
        const float lat = dx * q.rx + dz * q.rz;
        const float dist = hypot_rn(dx, dz);
        float film = hypot_rn(u, v);
        film = finite_f(film) ? film : 0.0f;
        const float immerse = fminf(h, q.radius * 0.9f);
        const float r_line = sqrtf(fmaxf(2.0f * q.radius * immerse - immerse * immerse, 0.0f));
        const float band = 1.0f - rclamp(fabsf(dist - r_line) / (cell * 1.35f), 0.0f, 1.0f);
        if (band > 0.0f) {
            const float motion = fmaxf(fmaxf(q.slip_v, q.speed * 0.45f), film);
            add_foam(f, breaking_foam(motion, h) * band, dt);
        }
        const bool on_patch = fabsf(lat) <= q.width * 0.55f + cell * 0.35f && along >= -q.radius * 0.55f &&
                              along <= q.radius * 0.35f;
        if (on_patch && h > 0.02f) {
            // lift_silt (:6686-6697), rate cap 0.015, critical stress 6 Pa.
            const float shear_v = fmaxf(q.slip_v, film * 0.35f);
            if (finite_f(shear_v) && shear_v > 0.0f) {
                const float tau = 1000.0f * 0.035f * shear_v * shear_v;
                if (tau > 6.0f) {
                    const float rate = fminf(0.008f * (tau / 6.0f - 1.0f), 0.015f);
                    add_silt(t, fminf(rate * dt, 0.0025f), area, b);
                }
            }
        }
    }
    if (m & SHORE) {
        float prod, silt_add;
        shore_cell(S, i, j, prod, silt_add);
        add_foam(f, prod, dt);
        if (silt_add > 0.0f) add_silt(t, fminf(silt_add * dt, 0.0012f), area, b);
    }
    const float hh = h + hs;
    if (finite_f(hh) && !(hh < 0.004f)) {
        if (finite_f(u) && finite_f(v) && !(hypot_rn(u, v) <= 0.05f)) add_foam(f, breaking_foam(hypot_rn(u, v), hh), dt);
    }
}

// The sources on every wet cell. They only add silt, so a cell above 1e-8
// after the settling stays above it; the wet cells that end above it join
// the span after the sources.
__global__ void __launch_bounds__(256, 3) k_spawn(const Job* jobs) {
    ::silt::dep_wait();
    const Job J = jobs[blockIdx.y];
    const Sheet& S = J.S;
    float* foam = J.T.foam[0];
    float* T = J.T.turbid[0];
    const uint8_t* mark = J.T.mark;
    const float dt = J.dt;
    double* book = J.T.books + 2;
    Ctl* c = ctl_of(J.T.st);
    if (!step_goes(J.T.st)) return;
    __shared__ PushK table[SPAWN_SHARED_PUSHES];
    const int np = J.npush;
    const bool shared_table = np <= SPAWN_SHARED_PUSHES;
    if (shared_table && (int)threadIdx.x < np) table[threadIdx.x] = push_k(J.push[threadIdx.x], S.cell);
    __syncthreads();
    const int res = S.res;
    double b = 0.0;
    LocalBox lb;
    const Box cb = box_of(c->cbox);  // the wet cells lie inside
    QUAD_ROWS(res, cb.i0, cb.i1, cb.j0, cb.j1) {
        if (quiet_run(J.T.occ, res, j, ib - (int)(threadIdx.x & 31), Box{0, -1, 0, -1})) continue;
        uint8_t mk[4];
        float hw[4], hs[4], u4[4], v4[4], f4[4], t4[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = ib + 32 * k;
            mk[k] = i <= cb.i1 ? mark[(unsigned)j * (unsigned)res + (unsigned)i] : (uint8_t)0;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (!(mk[k] & WET)) continue;
            const unsigned g = (unsigned)j * (unsigned)res + (unsigned)(ib + 32 * k);
            hw[k] = S.water[g];
            hs[k] = S.slurry[g];
            u4[k] = S.uw[g];
            v4[k] = S.vw[g];
            f4[k] = foam[g];
            t4[k] = T[g];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (!(mk[k] & WET)) continue;
            const int i = ib + 32 * k;
            const unsigned g = (unsigned)j * (unsigned)res + (unsigned)i;
            float f = f4[k], t = t4[k];
            spawn_cell(S, i, j, mk[k], hw[k], hs[k], u4[k], v4[k], shared_table ? table : nullptr, J.push, np, dt, f,
                       t, b);
            foam[g] = f;
            T[g] = t;
            if (t > 1.0e-8f) lb.add(i, j);
        }
    }
    lb.commit(c->tspan3);  // with the settled cells': the silt span after the sources
    block_book(b, book);
}

// clear_dry_tracers (:6712-6739) then sync_foam_live (:6339-6349), per cell.
// The clear only lowers silt, so the grown span after the sources holds every
// cell above 1e-8 after it: those cells are the next step's start span.
// Outside the collection box no cell is wet, and the live cells of the last
// sync lie inside it (it covers their box), so every mark there is 0.
__global__ void __launch_bounds__(256, 4) k_clear_sync(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    float* foam = T.foam[0];
    float* silt = T.turbid[0];
    uint8_t* mark = T.mark;
    State* st = T.st;
    Ctl* c = ctl_of(st);
    double* book = T.books + 3;
    if (!step_goes(st)) return;
    const int res = S.res;
    const float area = S.cell * S.cell;
    const Box cb = box_of(c->cbox);
    const Box sb = box_empty(c->tspan3) ? Box{0, -1, 0, -1} : grown_box(c->tspan3, res);
    const Box u = box_union(cb, sb);
    double b = 0.0;
    unsigned int cnt = 0;
    LocalBox live, span;
    QUAD_ROWS(res, u.i0, u.i1, u.j0, u.j1) {
        if (quiet_run(T.occ, res, j, ib - (int)(threadIdx.x & 31), sb)) continue;
        // Loads in two rounds: the marks, then what the wet cells and the
        // span's cells read.
        float hw[4], hs[4], f4[4], t4[4];
        uint8_t mk[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = ib + 32 * k;
            mk[k] = i <= u.i1 ? mark[(unsigned)j * (unsigned)res + (unsigned)i] : (uint8_t)0;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = ib + 32 * k;
            const unsigned g = (unsigned)j * (unsigned)res + (unsigned)i;
            if (i > u.i1) continue;
            const bool in_span = in_box(sb, i, j);
            if (!(mk[k] & WET) && !in_span) continue;
            hw[k] = S.water[g];
            hs[k] = S.slurry[g];
            if (mk[k] & WET) f4[k] = foam[g];
            if (in_span) t4[k] = silt[g];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = ib + 32 * k;
            const unsigned g = (unsigned)j * (unsigned)res + (unsigned)i;
            if (i > u.i1) continue;
            const uint8_t m = mk[k];
            const bool in_span = in_box(sb, i, j);
            if (!(m & WET) && !in_span) {
                if (m != 0 && in_box(cb, i, j)) mark[g] = 0;  // a dry cell's marks (sync below)
                continue;
            }
            const float h = hw[k] + hs[k];
            float f = (m & WET) ? f4[k] : 0.0f;
            if (m & WET) {
                if (!finite_f(h) || h < 0.004f || !finite_f(f)) {
                    f = 0.0f;
                    foam[g] = 0.0f;
                }
            }
            if (in_span) {
                float t = t4[k];
                if (!finite_f(h) || h < 1.0e-5f) {
                    if (t > 0.0f) {
                        b += (double)(t * area);
                        t = 0.0f;
                        silt[g] = 0.0f;
                    }
                } else if (!finite_f(t)) {
                    t = 0.0f;
                    silt[g] = 0.0f;
                }
                if (t > 1.0e-8f) span.add(i, j);
            }
            if (in_box(cb, i, j)) {
                uint8_t mm = m & (WET | SHORE);
                if ((mm & WET) && finite_f(f) && f > 1.0e-4f) {
                    mm |= LIVE;
                    ++cnt;
                    live.add(i, j);
                }
                mark[g] = mm;
            }
        }
    }
    live.commit(st->live_box);
    span.commit(st->tspan);
    block_count(cnt, &st->live_foam);
    block_book(b, book);
}

// ---------------------------------------------------------- step_suspended

__global__ void k_susp_begin(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    State* st = T.st;
    const int res = S.res;
    Ctl* c = ctl_of(st);
    box_clear(st->sbox, res);
    st->capped = 0;
    // The cells that may hold a load: every writer since the last pass grew
    // the next box; a river inlet carrying a load writes its rows.
    for (int k = 0; k < 4; ++k) c->ssup[k] = c->ssup_next[k];
    if (J.sup_all) {
        c->ssup[0] = 0;
        c->ssup[1] = res - 1;
        c->ssup[2] = 0;
        c->ssup[3] = res - 1;
    }
    box_clear(c->ssup_next, res);
}

// advect_suspended's first loop (:8826-8870): grains fall out at their fall
// speed; a dry cell or a load above the water settles whole. Cells outside
// the support box hold no load, and the loop leaves them as they are.
__global__ void k_susp_settle(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    float* susp = T.susp[0];
    State* st = T.st;
    Ctl* c = ctl_of(st);
    const float dt = J.dt;
    double* book = T.books + 1;
    const int res = S.res;
    const float area = S.cell * S.cell;
    const Box sup = box_of(c->ssup);
    double b = 0.0;
    LocalBox lb, held;
    BOX_CELLS(res, sup.i0, sup.i1, sup.j0, sup.j1) {
        float s = susp[g];
        if (!finite_f(s) || s <= 1.0e-12f) {
            if (__float_as_uint(s) != 0u) susp[g] = 0.0f;
            continue;
        }
        const float w = S.water[g];
        if (!finite_f(w) || w < 1.0e-5f || s > w) {
            b += (double)(s * area);
            susp[g] = 0.0f;
            continue;
        }
        const float keep = exp_rn(-dt * SUSP_FALL_M_S / w);
        const float landed = s * (1.0f - keep);
        if (landed > 0.0f) {
            b += (double)landed * (double)area;
            s -= landed;
            susp[g] = s;
        }
        if (s > 1.0e-8f) lb.add(i, j);
        if (s != 0.0f) held.add(i, j);
    }
    lb.commit(st->sbox);
    held.commit(c->ssup_next);
    block_book(b, book);
}

// One donor's part of advect_suspended's transport (:8894-8969).
struct Donor {
    bool live;
    float depth, w, c, fu, fv, fd;
    int up_i, up_j;  // receivers of the advected gives (-1: off the window)
};

__device__ __forceinline__ Donor donor_of(const Sheet& S, const float* susp, int i, int j, float dt) {
    const int res = S.res;
    const size_t d = (size_t)j * res + i;
    Donor D;
    D.depth = susp[d];
    D.w = S.water[d];
    D.live = !(D.depth <= 1.0e-12f || !finite_f(D.depth) || !finite_f(D.w) || D.w < 1.0e-5f);
    if (!D.live) return D;
    // film_uv(water, 0, uw, vw, 0, 0) (:3490-3501): the water film's own velocity.
    float u = 0.0f, v = 0.0f;
    const float hh = D.w + 0.0f;
    if (finite_f(hh) && !(hh < 1.0e-5f)) {
        u = finite0((S.uw[d] * D.w + 0.0f * 0.0f) / hh);
        v = finite0((S.vw[d] * D.w + 0.0f * 0.0f) / hh);
    }
    u = S.surface_driven && finite_f(u) ? u : 0.0f;
    v = finite_f(v) ? v : 0.0f;
    D.c = D.depth / D.w;
    float fu = fabsf(u) * dt / S.cell, fv = fabsf(v) * dt / S.cell;
    const float sum = fu + fv;
    if (sum > 0.45f) {
        fu *= 0.45f / sum;
        fv *= 0.45f / sum;
    }
    D.fu = fu;
    D.fv = fv;
    D.up_i = u > 0.0f ? (i + 1 < res ? (int)d + 1 : -1) : (i > 0 ? (int)d - 1 : -1);
    D.up_j = v > 0.0f ? (j + 1 < res ? (int)d + res : -1) : (j > 0 ? (int)d - res : -1);
    const float speed = sqrtf(u * u + v * v);
    const float k = 0.01f + 0.2f * speed * D.w;
    D.fd = fminf(k * dt / (S.cell * S.cell), 0.1f);
    return D;
}

// Receivers: each cell takes from its neighbour donors in raster order of
// the donors, each donor's gives in its own order (advection x, z, then
// mixing +x, -x, +z, -z), and records every accepted give in the donor's
// slot; its total goes to `taken`.
__global__ void k_susp_take(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    const float* susp = T.susp[0];
    float* taken = T.taken;
    float* acc = T.acc;
    State* st = T.st;
    const float dt = J.dt;
    if (box_empty(st->sbox)) return;
    const int res = S.res;
    const size_t n = (size_t)res * res;
    int bi0, bi1, bj0, bj1;
    grown(st->sbox, res, bi0, bi1, bj0, bj1);
    const bool open = S.surface_driven != 0;
    BOX_CELLS(res, max(bi0 - 1, 0), min(bi1 + 1, res - 1), max(bj0 - 1, 0), min(bj1 + 1, res - 1)) {
        const float wr = S.water[g];
        const bool can = finite_f(wr) && !(wr < 1.0e-5f);
        float tk = 0.0f;
        const int di[4] = {0, -1, 1, 0}, dj[4] = {-1, 0, 0, 1};  // donors in raster order
        for (int q = 0; q < 4; ++q) {
            const int a = i + di[q], c2 = j + dj[q];
            if (a < bi0 || a > bi1 || c2 < bj0 || c2 > bj1) continue;  // donors are the box's cells
            const Donor D = donor_of(S, susp, a, c2, dt);
            if (!D.live) continue;
            const size_t d = (size_t)c2 * res + a;
            const float fr[2] = {D.fu, D.fv};
            const int rv[2] = {D.up_i, D.up_j};
            for (int s = 0; s < 2; ++s) {
                if (rv[s] != (int)g) continue;
                const float give = D.depth * fr[s];
                if (give <= 1.0e-12f) continue;
                float accept = 0.0f;
                if (can) {
                    const float have = susp[g] + tk;
                    const float room = fmaxf(D.c * wr - have, 0.0f);
                    accept = fminf(fminf(give, room), fmaxf(wr - have, 0.0f));
                    if (accept <= 1.0e-12f) accept = 0.0f;
                    else tk += accept;
                }
                acc[(size_t)s * n + d] = accept;
            }
            if (!open) continue;
            // The donor's mixing neighbours: +x, -x, +z, -z.
            const int mk = (g == d + 1) ? 0 : (g + 1 == d ? 1 : (g == d + res ? 2 : 3));
            float accept = 0.0f;
            if (can) {
                const float cn = susp[g] / wr;
                if (D.c > cn) {
                    const float give = D.fd * (D.c - cn) * fminf(D.w, wr);
                    const float have = susp[g] + tk;
                    accept = fminf(give, fmaxf(wr - have, 0.0f));
                    if (accept <= 1.0e-12f) accept = 0.0f;
                    else tk += accept;
                }
            }
            acc[(size_t)(2 + mk) * n + d] = accept;
        }
        taken[g] = tk;
    }
}

// Donors: each box cell gives its slots away in its own order, takes what
// its neighbours gave it, then the load above the water or on a dry cell
// settles (:8971-9000).
__global__ void k_susp_give(const Job* jobs) {
    ::silt::dep_wait();
    JOB;
    float* susp = T.susp[0];
    const float* taken = T.taken;
    const float* acc = T.acc;
    State* st = T.st;
    const float dt = J.dt;
    double* book = T.books + 1;
    if (box_empty(st->sbox)) return;
    const int res = S.res;
    const size_t n = (size_t)res * res;
    const float area = S.cell * S.cell;
    int bi0, bi1, bj0, bj1;
    grown(st->sbox, res, bi0, bi1, bj0, bj1);
    const bool open = S.surface_driven != 0;
    double b = 0.0;
    unsigned int capped = 0;
    LocalBox held;
    BOX_CELLS(res, bi0, bi1, bj0, bj1) {
        float next = susp[g];
        const Donor D = donor_of(S, susp, i, j, dt);
        if (D.live) {
            const float fr[2] = {D.fu, D.fv};
            const int rv[2] = {D.up_i, D.up_j};
            for (int s = 0; s < 2; ++s) {
                const float give = D.depth * fr[s];
                if (give <= 1.0e-12f) continue;
                if (rv[s] < 0) {
                    b += (double)(give * area);
                    next -= give;
                    continue;
                }
                const float wrr = S.water[rv[s]];
                if (!finite_f(wrr) || wrr < 1.0e-5f) continue;
                const float a = acc[(size_t)s * n + g];
                if (a > 0.0f) next -= a;
            }
            if (open) {
                const bool has[4] = {i + 1 < res, i > 0, j + 1 < res, j > 0};
                const int off[4] = {1, -1, res, -res};
                for (int k = 0; k < 4; ++k) {
                    if (!has[k]) continue;
                    const float wrr = S.water[g + off[k]];
                    if (!finite_f(wrr) || wrr < 1.0e-5f) continue;
                    const float a = acc[(size_t)(2 + k) * n + g];
                    if (a > 0.0f) next -= a;
                }
            }
        }
        next += taken[g];
        float s = next;
        if (!finite_f(s) || s <= 0.0f) {
            susp[g] = 0.0f;
            continue;
        }
        const float w = S.water[g];
        if (!finite_f(w) || w < 1.0e-5f) {
            b += (double)(s * area);
            s = 0.0f;
        } else if (s > w) {
            const float excess = s - w;
            b += (double)(excess * area);
            if (excess > 1.0e-5f) ++capped;
            s = w;
        }
        susp[g] = s;
        if (s != 0.0f) held.add(i, j);
    }
    held.commit(ctl_of(st)->ssup_next);
    block_book(b, book);
    block_count(capped, &st->capped);
}

// The idle report of every job with a report word: `last` 0 = the jobs
// without a suspended pass (after step_tracers), 1 = the rest (after
// step_suspended).
__global__ void k_idle(const Job* jobs, int last) {
    ::silt::dep_wait();
    const Job& J = jobs[blockIdx.y];
    if (threadIdx.x != 0 || blockIdx.x != 0 || !J.idle_out || (J.susp_on != 0) != (last != 0)) return;
    const State* st = J.T.st;
    const Ctl* c = reinterpret_cast<const Ctl*>(st + 1);
    const bool idle = st->live_foam == 0u && box_empty(st->tspan) && !J.rescan &&
                      (!J.susp_on || box_empty(c->ssup_next));
    *J.idle_out = idle ? 1u : 0u;
}

__global__ void k_reset_live(uint8_t* mark, State* st, int res, size_t n) {
    ::silt::dep_wait();
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x)
        mark[g] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // The planes were rewritten: the silt span is scanned again before the
        // next tracer step, and any cell may hold a suspended load.
        Ctl* c = ctl_of(st);
        st->live_foam = 0;
        box_clear(st->live_box, res);
        box_clear(st->tspan, res);
        box_clear(c->mbox, res);
        c->ssup_next[0] = 0;
        c->ssup_next[1] = res - 1;
        c->ssup_next[2] = 0;
        c->ssup_next[3] = res - 1;
    }
}

// tracer_visit_box's tire part (:6320-6331) on the host: each tire inside
// the window reaches ceil(8 m / cell) cells around its own.
void push_box(const Sheet& S, const silt_tire_push* p, int n, int* b) {
    b[0] = S.res;
    b[1] = -1;
    b[2] = S.res;
    b[3] = -1;
    const int reach = (int)ceilf(8.0f / S.cell);
    for (int k = 0; k < n; ++k) {
        const float fi = floorf((p[k].x - S.ox) / S.cell), fj = floorf((p[k].z - S.oz) / S.cell);
        if (!(fi >= 0.0f) || !(fj >= 0.0f) || fi >= (float)S.res || fj >= (float)S.res) continue;
        const int ci = (int)fi, cj = (int)fj;
        b[0] = std::min(b[0], std::max(ci - reach, 0));
        b[1] = std::max(b[1], std::min(ci + reach, S.res - 1));
        b[2] = std::min(b[2], std::max(cj - reach, 0));
        b[3] = std::max(b[3], std::min(cj + reach, S.res - 1));
    }
}

// entrain_wake's cells (:8766-8776): the union of the tires' reach boxes,
// one cell wider on each side and clamped to the window (each cell still
// tests every tire's own box, so the margin only covers host rounding).
void entrain_box(const Sheet& S, const silt_tire_push* p, int n, int* b) {
    b[0] = S.res;
    b[1] = -1;
    b[2] = S.res;
    b[3] = -1;
    for (int k = 0; k < n; ++k) {
        if (!(p[k].speed >= 0.3f)) continue;
        const float reach = p[k].radius * 3.4f + S.cell;
        const float lo_x = floorf(((p[k].x - reach) - S.ox) / S.cell), hi_x = floorf(((p[k].x + reach) - S.ox) / S.cell);
        const float lo_z = floorf(((p[k].z - reach) - S.oz) / S.cell), hi_z = floorf(((p[k].z + reach) - S.oz) / S.cell);
        if (!(lo_x <= hi_x) || !(lo_z <= hi_z)) continue;
        if (hi_x < 0.0f || hi_z < 0.0f || lo_x >= (float)S.res || lo_z >= (float)S.res) continue;
        b[0] = std::min(b[0], (int)std::max(lo_x - 1.0f, 0.0f));
        b[1] = std::max(b[1], (int)std::min(hi_x + 1.0f, (float)(S.res - 1)));
        b[2] = std::min(b[2], (int)std::max(lo_z - 1.0f, 0.0f));
        b[3] = std::max(b[3], (int)std::min(hi_z + 1.0f, (float)(S.res - 1)));
    }
}

// Blocks per window of a launch over n windows: enough for the largest
// window, about `total` blocks of 256 threads in all.
int blocks_x(const Window* w, int n, int total) {
    size_t most = 1;
    for (int k = 0; k < n; ++k) most = std::max(most, (size_t)w[k].S.res * w[k].S.res);
    const size_t per = std::max<size_t>(1, (size_t)std::max(total, 1) / (size_t)std::max(n, 1));
    return (int)std::min((most + 255) / 256, per);
}

// Uploads the jobs (and their pushes) of one launch sequence; returns the
// device array.
cudaError_t upload(Runner& R, const Window* w, int n, float dt, float foam_decay, float silt_keep, cudaStream_t st,
                   const Job** out) {
    const int slot = R.next;
    R.next = (R.next + 1) % Runner::SLOTS;
    cudaError_t e;
    if (R.ev[slot]) {
        if ((e = cudaEventSynchronize(R.ev[slot])) != cudaSuccess) return e;  // this slot's last copy is done
    } else if ((e = cudaEventCreateWithFlags(&R.ev[slot], cudaEventDisableTiming)) != cudaSuccess) {
        return e;
    }
    size_t np = 0;
    for (int k = 0; k < n; ++k) np += (size_t)w[k].npush;
    if ((size_t)n > R.cap_jobs[slot]) {
        cudaFree(R.d_jobs[slot]);
        if (R.h_jobs[slot]) cudaFreeHost(R.h_jobs[slot]);
        R.d_jobs[slot] = nullptr;
        R.h_jobs[slot] = nullptr;
        R.cap_jobs[slot] = 0;
        const size_t cap = (size_t)n * 2;
        if ((e = cudaMalloc(&R.d_jobs[slot], cap * sizeof(Job))) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&R.h_jobs[slot], cap * sizeof(Job))) != cudaSuccess) return e;
        R.cap_jobs[slot] = cap;
    }
    if (np > R.cap_push[slot]) {
        cudaFree(R.d_push[slot]);
        if (R.h_push[slot]) cudaFreeHost(R.h_push[slot]);
        R.d_push[slot] = nullptr;
        R.h_push[slot] = nullptr;
        R.cap_push[slot] = 0;
        const size_t cap = np * 2 + 16;
        if ((e = cudaMalloc(&R.d_push[slot], cap * sizeof(silt_tire_push))) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&R.h_push[slot], cap * sizeof(silt_tire_push))) != cudaSuccess) return e;
        R.cap_push[slot] = cap;
    }
    size_t q = 0;
    for (int k = 0; k < n; ++k) {
        Job& J = R.h_jobs[slot][k];
        memset(&J, 0, sizeof J);
        J.S = w[k].S;
        J.T = w[k].T;
        J.npush = w[k].npush;
        J.push = w[k].npush ? R.d_push[slot] + q : nullptr;
        if (w[k].npush) memcpy(R.h_push[slot] + q, w[k].push, (size_t)w[k].npush * sizeof(silt_tire_push));
        q += (size_t)w[k].npush;
        bool wake = w[k].S.surface_driven != 0;
        for (int t = 0; t < w[k].npush; ++t) {
            const silt_tire_push& p = w[k].push[t];
            wake = wake || (std::isfinite(p.speed) && p.speed >= 0.25f) ||
                   (std::isfinite(p.slip) && fabsf(p.slip) >= 0.05f);
        }
        J.wake = wake ? 1 : 0;
        J.rescan = w[k].rescan;
        J.sup_all = w[k].sup_all;
        J.susp_on = w[k].susp_on;
        J.idle_out = w[k].idle_out;
        push_box(w[k].S, w[k].push, w[k].npush, J.pbox);
        entrain_box(w[k].S, w[k].push, w[k].npush, J.ebox);
        J.dt = dt;
        J.foam_decay = foam_decay;
        J.silt_keep = silt_keep;
    }
    if (np && (e = cudaMemcpyAsync(R.d_push[slot], R.h_push[slot], np * sizeof(silt_tire_push),
                                   cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(R.d_jobs[slot], R.h_jobs[slot], (size_t)n * sizeof(Job), cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
        return e;
    if ((e = cudaEventRecord(R.ev[slot], st)) != cudaSuccess) return e;
    *out = R.d_jobs[slot];
    return cudaSuccess;
}

#define LAUNCH(kernel, bx, ...)                                                                \
    do {                                                                                       \
        ::silt::launch_dep(kernel, dim3((bx), (unsigned)n), dim3(256), 0, st, __VA_ARGS__);    \
        ::silt::count_launch();                                                                \
        const cudaError_t e_ = cudaGetLastError();                                             \
        if (e_ != cudaSuccess) return e_;                                                      \
    } while (0)

}  // namespace

size_t plane_bytes(int res) {
    const size_t n = (size_t)res * res;
    return 256 + 6 * n * sizeof(float) + 6 * n * sizeof(float) + n + (size_t)res * segments(res) + 256;
}

cudaError_t attach(Planes& T, void* mem, int res, double* books, cudaStream_t st) {
    const size_t n = (size_t)res * res;
    char* q = (char*)mem;
    T.st = reinterpret_cast<State*>(q);  // State then Ctl, within the first 256 bytes
    static_assert(sizeof(State) + sizeof(Ctl) <= 256, "tracer state");
    q += 256;
    float* f = reinterpret_cast<float*>(q);
    T.foam[0] = f;
    T.foam[1] = f + n;
    T.turbid[0] = f + 2 * n;
    T.turbid[1] = f + 3 * n;
    T.susp[0] = f + 4 * n;
    T.susp[1] = f + 5 * n;
    T.taken = T.susp[1];
    T.acc = f + 6 * n;
    T.mark = reinterpret_cast<uint8_t*>(f + 12 * n);
    T.occ = T.mark + n;
    T.books = books;
    cudaError_t e = cudaMemsetAsync(mem, 0, plane_bytes(res), st);
    if (e != cudaSuccess) return e;
    return reset_indices(T, res, st);
}

void Runner::release() {
    for (int k = 0; k < SLOTS; ++k) {
        cudaFree(d_jobs[k]);
        cudaFree(d_push[k]);
        if (h_jobs[k]) cudaFreeHost(h_jobs[k]);
        if (h_push[k]) cudaFreeHost(h_push[k]);
        if (ev[k]) cudaEventDestroy(ev[k]);
        d_jobs[k] = h_jobs[k] = nullptr;
        d_push[k] = h_push[k] = nullptr;
        cap_jobs[k] = cap_push[k] = 0;
        ev[k] = nullptr;
    }
}

cudaError_t entrain(Runner& R, const Window* w, int n, float dt, cudaStream_t st) {
    if (n <= 0 || !(dt > 0.0f) || !std::isfinite(dt)) return cudaSuccess;
    const Job* jobs = nullptr;
    cudaError_t e = upload(R, w, n, dt, 0.0f, 0.0f, st, &jobs);
    if (e != cudaSuccess) return e;
    LAUNCH(k_entrain, blocks_x(w, n, R.blocks_total), jobs);
    return cudaSuccess;
}

cudaError_t step_tracers(Runner& R, const Window* w, int n, float dt, cudaStream_t st) {
    if (n <= 0 || !(dt > 0.0f) || !std::isfinite(dt)) return cudaSuccess;
    // The per-step factors, with the C library's expf as the reference's f32::exp.
    const float foam_decay = expf(-dt / 1.8f);  // FOAM_LIFE_S :112
    const float silt_keep = expf(-dt / 4.0f);   // SILT_SETTLE_S :119
    const Job* jobs = nullptr;
    cudaError_t e = upload(R, w, n, dt, foam_decay, silt_keep, st, &jobs);
    if (e != cudaSuccess) return e;
    const int bx = blocks_x(w, n, R.blocks_total);
    bool rescan = false;
    for (int k = 0; k < n; ++k) rescan = rescan || w[k].rescan;
    if (rescan) LAUNCH(k_scan, bx, jobs);
    LAUNCH(k_begin, 1, jobs);
    LAUNCH(k_collect, bx, jobs);
    LAUNCH(k_turbid_advect, bx, jobs);
    LAUNCH(k_commit, bx, jobs);
    LAUNCH(k_settle, bx, jobs);
    LAUNCH(k_spawn, bx, jobs);
    LAUNCH(k_clear_sync, bx, jobs);
    bool report = false;
    for (int k = 0; k < n; ++k) report = report || (w[k].idle_out && !w[k].susp_on);
    if (report) LAUNCH(k_idle, 1, jobs, 0);
    return cudaSuccess;
}

cudaError_t step_suspended(Runner& R, const Window* w, int n, float dt, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const Job* jobs = nullptr;
    cudaError_t e = upload(R, w, n, dt, 0.0f, 0.0f, st, &jobs);
    if (e != cudaSuccess) return e;
    LAUNCH(k_susp_begin, 1, jobs);
    if (!(dt > 0.0f) || !std::isfinite(dt)) return cudaSuccess;
    const int bx = blocks_x(w, n, R.blocks_total);
    LAUNCH(k_susp_settle, bx, jobs);
    LAUNCH(k_susp_take, bx, jobs);
    LAUNCH(k_susp_give, bx, jobs);
    bool report = false;
    for (int k = 0; k < n; ++k) report = report || w[k].idle_out;
    if (report) LAUNCH(k_idle, 1, jobs, 1);
    return cudaSuccess;
}

cudaError_t reset_indices(Planes& T, int res, cudaStream_t st) {
    const size_t cells = (size_t)res * res;
    const size_t b = (cells + 255) / 256;
    ::silt::launch_dep(k_reset_live, dim3((unsigned)std::min<size_t>(std::max<size_t>(b, 1), 1184)), dim3(256), 0, st,
                       T.mark, T.st, res, cells);
    ::silt::count_launch();
    return cudaGetLastError();
}

}  // namespace tracers
}  // namespace silt
