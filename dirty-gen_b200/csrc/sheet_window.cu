// Window engine: one CTA steps one layer of one window (up to 512 x 512
// cells) exactly as the reference's step_sheet does (x3-team/Dirty-gen
// src/fluid_core.rs:821-2082): work boxes chosen per step, the CFL substep
// count, then every substep box by box with the per-sheet scratch planes the
// reference keeps between calls. It serves the nested 2 cm patches, the
// coarse 20 cm window and batches of windows (one CTA per window layer).
//
// Exactness notes, each a property of the reference this engine keeps:
// * A box-edge cell reads pressure and blur values an earlier box or an
//   earlier step left in the scratch; the same scratch planes with the same
//   writes reproduce those reads.
// * The coarse pair confines vorticity in a raster-order Gauss-Seidel sweep
//   (force_gravity_open, :2234-2260). Here the sweep is solved as a fixed
//   point: every wet cell's final velocity is u_grav + kick(final values of
//   the cells before it, its own post-gravity value, pre-gravity values of
//   the cells after it). Passes run until one changes no bit, which makes
//   every cell satisfy its own sweep equation, i.e. the sequential result;
//   past a pass limit one thread runs the sweep itself.
// * Fine sheets and the free operator's large boxes confine from a snapshot
//   (Jacobi), as the reference does there.
#include <algorithm>
#include <cooperative_groups.h>
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>

#include "sheet_math.cuh"
#include "sheet_window.cuh"
#include "launch_count.cuh"

namespace silt {
namespace window {

constexpr int NT = 512;            // threads per CTA
constexpr int SLEEP_TILE = 8;      // src/fluid_core.rs:1528
constexpr int MAX_TILES = (MAX_RES / SLEEP_TILE) * (MAX_RES / SLEEP_TILE);
constexpr int MAX_BOXES = 512;
constexpr int GS_MAX_PASSES = 256;

struct Box {
    int i0, i1, j0, j1;
};

static_assert(NT % 32 == 0 && NT / 32 <= 32, "one warp reduces the per-warp partials");

struct Shared {
    int lab[MAX_TILES];
    unsigned char hot[MAX_TILES];
    unsigned char grown[MAX_TILES];
    int bbox[4][MAX_BOXES];
    int row_count[MAX_RES];
    int nbox;
    int changed;
    int chg[3];      // Gauss-Seidel pass verdicts, rotating (pass k uses chg[k % 3])
    int lchg[3];     // wet-body label rounds' verdicts, rotating the same way
    float red_f[NT / 32];
    double red_d[NT / 32];
    double crew_d;   // this CTA's share of a crew-wide sum or maximum, read by the crew
    int crew_ext[5]; // this CTA's share of the wet extent: count, i0, -i1, j0, j1
    float crew_f;
    int red_i[4][NT / 32];
};

// Every cell of the inclusive rectangle, one warp per row and the lanes along
// x (no division per cell). Bodies may `continue` to the next cell.
#define CTA_RECT(I0, I1, J0, J1, ...)                                               \
    {                                                                               \
        const int ri0_ = (I0), ri1_ = (I1), rj1_ = (J1);                            \
        for (int j = (J0) + (int)(threadIdx.x >> 5); j <= rj1_; j += NT / 32)       \
            for (int i = ri0_ + (int)(threadIdx.x & 31); i <= ri1_; i += 32) {      \
                const int g = j * res + i;                                          \
                (void)g;                                                            \
                __VA_ARGS__                                                         \
            }                                                                       \
    }

namespace cg = cooperative_groups;

// A job is stepped by a cluster of CTAs (its crew). The step's phases split
// the box rows over every warp of the crew and end at the cluster barrier
// (release/acquire at cluster scope, so each phase sees the planes the crew
// wrote in the one before). Work-box selection, the wet and CFL reductions
// and the ledger read whole planes and run per CTA (identical in every CTA,
// so the crew's control flow stays uniform) or on rank 0 alone.
__device__ __forceinline__ int crew_rank() { return (int)cg::this_cluster().block_rank(); }
__device__ __forceinline__ int crew_size() { return (int)cg::this_cluster().num_blocks(); }
__device__ __forceinline__ void crew_sync() { cg::this_cluster().sync(); }

// Every cell of the inclusive rectangle, shared by the crew: work items are
// (row, 32-cell chunk) pairs dealt round-robin to the crew's warps, lanes
// along x. Bodies may `continue` to the next cell.
#define CLU_RECT(I0, I1, J0, J1, ...)                                                    \
    {                                                                                    \
        const int ri0_ = (I0), ri1_ = (I1), rj0_ = (J0), rj1_ = (J1);                    \
        if (ri1_ >= ri0_ && rj1_ >= rj0_) {                                              \
            const int ch_ = (ri1_ - ri0_ + 32) >> 5;                                     \
            const int items_ = (rj1_ - rj0_ + 1) * ch_;                                  \
            const int gs_ = crew_size() * (NT / 32);                                     \
            for (int it_ = crew_rank() * (NT / 32) + (int)(threadIdx.x >> 5); it_ < items_; \
                 it_ += gs_) {                                                           \
                const int r_ = it_ / ch_;                                                \
                const int j = rj0_ + r_;                                                 \
                const int i = ri0_ + (it_ - r_ * ch_) * 32 + (int)(threadIdx.x & 31);   \
                if (i <= ri1_) {                                                         \
                    const int g = j * res + i;                                           \
                    (void)g;                                                             \
                    __VA_ARGS__                                                          \
                }                                                                        \
            }                                                                            \
        }                                                                                \
    }

__device__ __forceinline__ double block_sum_d(Shared& S, double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) S.red_d[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < NT / 32 ? S.red_d[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) S.red_d[0] = t;
    }
    __syncthreads();
    double r = S.red_d[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ float block_max_f(Shared& S, float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) S.red_f[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        float t = threadIdx.x < NT / 32 ? S.red_f[threadIdx.x] : 0.0f;  // values reduced here are >= 0
        for (int o = 16; o > 0; o >>= 1) t = fmaxf(t, __shfl_down_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) S.red_f[0] = t;
    }
    __syncthreads();
    float r = S.red_f[0];
    __syncthreads();
    return r;
}

// Every crew CTA's copy of one shared-memory value, combined in rank order:
// lane r of each warp loads rank r's copy (the loads overlap instead of
// following one another), then the values are folded through shuffles in rank
// order, so the result is exactly the one a loop over the ranks gives. Called
// by every thread after the barrier that published the copies; at most 32
// CTAs in a crew.
template <typename T, typename F>
__device__ __forceinline__ T crew_fold(const T* mine, T init, F combine) {
    cg::cluster_group crew = cg::this_cluster();
    const int lane = threadIdx.x & 31, n = crew_size();
    T got = init;
    if (lane < n) got = *crew.map_shared_rank(mine, lane);
    T acc = init;
    for (int r = 0; r < n; ++r) acc = combine(acc, __shfl_sync(0xffffffffu, got, r));
    return acc;
}

// A crew-wide sum of per-thread partials: each CTA reduces its own, then every
// CTA adds the CTAs' results in rank order (the same value in every CTA).
__device__ double crew_sum_d(Shared& S, double v) {
    const double part = block_sum_d(S, v);
    if (threadIdx.x == 0) S.crew_d = part;
    crew_sync();
    const double tot = crew_fold(&S.crew_d, 0.0, [](double a, double b) { return a + b; });
    crew_sync();  // every CTA has read the shares before they are reused
    return tot;
}

// A crew-wide maximum of non-negative per-thread values.
__device__ float crew_max_f(Shared& S, float v) {
    const float part = block_max_f(S, v);
    if (threadIdx.x == 0) S.crew_f = part;
    crew_sync();
    const float m = crew_fold(&S.crew_f, 0.0f, [](float a, float b) { return fmaxf(a, b); });
    crew_sync();
    return m;
}

// Four ints reduced together: op 0 = sum, 1 = min, 2 = max.
__device__ void block_reduce4(Shared& S, int v[4], const int op[4]) {
    for (int q = 0; q < 4; ++q)
        for (int o = 16; o > 0; o >>= 1) {
            int w = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = op[q] == 0 ? v[q] + w : (op[q] == 1 ? min(v[q], w) : max(v[q], w));
        }
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 4; ++q) S.red_i[q][threadIdx.x >> 5] = v[q];
    __syncthreads();
    if (threadIdx.x < 32) {
        for (int q = 0; q < 4; ++q) {
            const int ident = op[q] == 0 ? 0 : (op[q] == 1 ? 0x7fffffff : (int)0x80000000);
            int t = threadIdx.x < NT / 32 ? S.red_i[q][threadIdx.x] : ident;
            for (int o = 16; o > 0; o >>= 1) {
                int w = __shfl_down_sync(0xffffffffu, t, o);
                t = op[q] == 0 ? t + w : (op[q] == 1 ? min(t, w) : max(t, w));
            }
            if (threadIdx.x == 0) S.red_i[q][0] = t;
        }
    }
    __syncthreads();
    for (int q = 0; q < 4; ++q) v[q] = S.red_i[q][0];
    __syncthreads();
}

// The crew-wide wet sum and wet extent of one pass: ws summed as crew_sum_d
// does; ext = {wet cells, min i, -max i, min j, max j} over the crew, in the
// same barriers.
__device__ double crew_sum_extent(Shared& S, double v, int ext[5]) {
    const double part = block_sum_d(S, v);
    int a[4] = {ext[0], ext[1], ext[2], ext[3]};
    const int op[4] = {0, 1, 1, 1};
    block_reduce4(S, a, op);
    int b[4] = {ext[4], 0, 0, 0};
    const int op2[4] = {2, 2, 2, 2};
    block_reduce4(S, b, op2);
    if (threadIdx.x == 0) {
        S.crew_d = part;
        for (int q = 0; q < 4; ++q) S.crew_ext[q] = a[q];
        S.crew_ext[4] = b[0];
    }
    crew_sync();
    const double tot = crew_fold(&S.crew_d, 0.0, [](double a, double b) { return a + b; });
    auto mn = [](int a, int b) { return min(a, b); };
    ext[0] = crew_fold(&S.crew_ext[0], 0, [](int a, int b) { return a + b; });
    ext[1] = crew_fold(&S.crew_ext[1], 0x7fffffff, mn);
    ext[2] = crew_fold(&S.crew_ext[2], 0x7fffffff, mn);
    ext[3] = crew_fold(&S.crew_ext[3], 0x7fffffff, mn);
    ext[4] = crew_fold(&S.crew_ext[4], -1, [](int a, int b) { return max(a, b); });
    crew_sync();  // every CTA has read the shares before they are reused
    return tot;
}


// Five taps along one axis, clamped at the grid edge. Cells at least 2 from
// the edge start from the first product (accum5), others from 0.0
// (accum5_clamped), src/fluid_core.rs:3680-3697.
__device__ __forceinline__ float tap5c(const float* line, int res, int i, float k0, float k1, float k2, int stride) {
    const bool in = i >= 2 && i <= res - 3;
    const int i0 = i < 2 ? 0 : i - 2, i1 = i < 1 ? 0 : i - 1;
    const int i3 = i + 1 > res - 1 ? res - 1 : i + 1, i4 = i + 2 > res - 1 ? res - 1 : i + 2;
    float a0 = line[i0 * stride], a1 = line[i1 * stride], a2 = line[i * stride], a3 = line[i3 * stride],
          a4 = line[i4 * stride];
    float a = in ? a0 * k0 : 0.0f + a0 * k0;
    a += a1 * k1;
    a += a2 * k2;
    a += a3 * k1;
    a += a4 * k0;
    return a;
}

// tap5c down column i where rows [lo, hi] come from `in_box` and the other
// rows from `outside`.
__device__ __forceinline__ float tap5c_pick(const float* in_box, const float* outside, int lo, int hi, int res, int i,
                                            int j, float k0, float k1, float k2) {
    const bool in = j >= 2 && j <= res - 3;
    const int r0 = j < 2 ? 0 : j - 2, r1 = j < 1 ? 0 : j - 1;
    const int r3 = j + 1 > res - 1 ? res - 1 : j + 1, r4 = j + 2 > res - 1 ? res - 1 : j + 2;
    auto at = [&](int r) { return (r >= lo && r <= hi ? in_box : outside)[r * res + i]; };
    float a0 = at(r0), a1 = at(r1), a2 = at(j), a3 = at(r3), a4 = at(r4);
    float a = in ? a0 * k0 : 0.0f + a0 * k0;
    a += a1 * k1;
    a += a2 * k2;
    a += a3 * k1;
    a += a4 * k0;
    return a;
}

// The reference's two blurs of one source in a row, blur_box with GAUSS into
// dst_g and then with STEEP into dst_s, both through the scratch `tmp`
// (src/fluid_core.rs:3541-3569), in two crew phases instead of four. The x
// passes of the box rows go to tmp_g (GAUSS, a transient plane) and tmp
// (STEEP, where the reference's second blur leaves it). Each z pass reads box
// rows from its own x pass and the rows outside the box from tmp as they are:
// the reference's x passes write only the box, so both of its z passes see
// the same stale rows there. `combine(g, gauss, steep)` runs on each box cell
// in the z phase.
template <class Comb>
__device__ void cta_blur_pair(const float* __restrict__ src, float* __restrict__ dst_g, float* __restrict__ dst_s,
                              float* __restrict__ tmp, float* __restrict__ tmp_g, int res, const Box& b,
                              Comb combine) {
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        const float* line = src + j * res;
        tmp_g[g] = tap5c(line, res, i, kG0, kG1, kG2, 1);
        tmp[g] = tap5c(line, res, i, kS0, kS1, kS2, 1);
    })
    crew_sync();
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        const float gv = tap5c_pick(tmp_g, tmp, b.j0, b.j1, res, i, j, kG0, kG1, kG2);
        const float sv = tap5c(tmp + i, res, j, kS0, kS1, kS2, res);
        dst_g[g] = gv;
        dst_s[g] = sv;
        combine(g, gv, sv);
    })
    crew_sync();
}

__device__ __forceinline__ float job_nu(const Job& J, int g) {
    if (J.nu_mode == NU_CONST) return J.nu_c;
    if (J.nu_mode == NU_PLANE || J.nu_mode == NU_TABLE) return J.nu_plane[g];
    return dynamic_viscosity(J.grain[g], J.moisture[g]);
}

// sheet_mobility_for(nu) of the cell.
__device__ __forceinline__ float job_mob(const Job& J, int g) {
    if (J.nu_mode == NU_CONST) return J.mob_c;
    if (J.nu_mode == NU_TABLE) return J.mob_plane[g];
    return sheet_mobility_for(job_nu(J, g));
}

// The cell's damping factor over dt: exp(-sheet_damp(nu) dt).
__device__ __forceinline__ float job_decay(const Job& J, int g, float dt, float decay_c) {
    if (J.nu_mode == NU_CONST) return decay_c;
    const float rate = J.nu_mode == NU_TABLE ? J.damp_plane[g] : sheet_damp(job_nu(J, g));
    return exp_rn(-rate * dt);
}

// transport_open_rows (src/fluid_core.rs:3025-3137) on one box, banks off;
// on a walled sheet the same edges as transport/move_edge_bufs (:3894-3963,
// :4178-4223): an edge touching a wall moves nothing, and a dry bank above the
// donor's surface takes nothing (banks on the layer's bed).
__device__ void cta_transport(const Job& J, const Box& b, float dt) {
    // Two crew phases. Each cell recomputes the fluxes of the edges it needs
    // (its own two and, for the donor's room, the left flux one edge further)
    // from the depths before the pass, exactly as the reference's flux
    // buffers hold them, so no flux plane and no barrier sits between the
    // fluxes and the update. The x pass writes its depths to f1; the z pass
    // reads them there and writes h.
    const int res = J.res;
    float* __restrict__ h = J.h;
    const float* __restrict__ U = J.u;
    const float* __restrict__ V = J.v;
    float* __restrict__ HX = J.f1;
    const FixedDiv cell = J.div.cell;
    const uint8_t* __restrict__ gate = J.gate;
    const uint8_t* __restrict__ W = J.solid;
    const float* __restrict__ bed = J.bed;
    const bool walled = W != nullptr;
    // The rounding book: each updated cell's f32 change less the exact
    // (FP64) sum of the fluxes across its faces.
    const bool book_round = J.round != nullptr;
    double rnd = 0.0;
    // dh of the edge from donor d to receiver r on depths hp, 0 across a wall.
    auto edge = [&](const float* hp, int d, int r, float remd, float speed) {
        const float dh = open_edge_dh(walled, hp[d], hp[r], remd, gate ? gate[r] : 1, walled ? bed[d] : 0.0f,
                                      walled ? bed[r] : 0.0f, speed, dt, cell, 0.45f);
        return walled && (W[d] | W[r]) ? 0.0f : dh;
    };
    // x pass. Edge e joins cells e and e+1 of the row, e in [i0, i1 - 1]: its
    // left-going flux (donor e+1) when the face speed is not positive, else
    // its right-going flux (donor e, after what e gave across edge e-1).
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        const int row = j * res;
        auto speed = [&](int e) { return 0.5f * (U[row + e] + U[row + e + 1]); };
        auto left = [&](int e) {
            const float sp = speed(e);
            const float dh = edge(h, row + e + 1, row + e, 0.0f, sp);
            return sp > 0.0f ? 0.0f : dh;
        };
        auto right = [&](int e) {
            const float sp = speed(e);
            const float prev = e > b.i0 ? left(e - 1) : 0.0f;
            const float dh = edge(h, row + e, row + e + 1, 0.0f + prev, sp);
            return sp > 0.0f ? dh : 0.0f;
        };
        const float flm = i > b.i0 ? left(i - 1) : 0.0f, frm = i > b.i0 ? right(i - 1) : 0.0f;
        const float flc = i < b.i1 ? left(i) : 0.0f, frc = i < b.i1 ? right(i) : 0.0f;
        const float rem = (0.0f + flm) + frc, add = (0.0f + frm) + flc;
        const float hv = h[g];
        const float moved = fmaxf(hv - rem + add, 0.0f);
        const float hx = (rem > 0.0f || add > 0.0f) ? moved : hv;
        HX[g] = hx;
        if (book_round) rnd += ((double)hx - (double)hv) - (((double)frm + (double)flc) - ((double)flm + (double)frc));
    })
    crew_sync();
    // z pass on the x pass's depths: row pair r joins rows r and r+1, r in [j0, j1 - 1].
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        auto speed = [&](int r) { return 0.5f * (V[r * res + i] + V[(r + 1) * res + i]); };
        auto up = [&](int r) {
            const float sp = speed(r);
            const float dh = edge(HX, (r + 1) * res + i, r * res + i, 0.0f, sp);
            return sp > 0.0f ? 0.0f : dh;
        };
        auto down = [&](int r) {
            const float sp = speed(r);
            const float ra = r > b.j0 ? 0.0f + up(r - 1) : 0.0f;
            const float dh = edge(HX, r * res + i, (r + 1) * res + i, ra, sp);
            return sp > 0.0f ? dh : 0.0f;
        };
        const float upm = j > b.j0 ? up(j - 1) : 0.0f, dnm = j > b.j0 ? down(j - 1) : 0.0f;
        const float upc = j < b.j1 ? up(j) : 0.0f, dnc = j < b.j1 ? down(j) : 0.0f;
        const float rem = (0.0f + upm) + dnc, add = (0.0f + dnm) + upc;
        const float hv = HX[g];
        const float moved = fmaxf(hv - rem + add, 0.0f);
        const float hn = (rem > 0.0f || add > 0.0f) ? moved : hv;
        h[g] = hn;
        if (book_round) rnd += ((double)hn - (double)hv) - (((double)dnm + (double)upc) - ((double)upm + (double)dnc));
    })
    if (book_round) {
        for (int o = 16; o > 0; o >>= 1) rnd += __shfl_down_sync(0xffffffffu, rnd, o);
        if ((threadIdx.x & 31) == 0 && rnd != 0.0) atomicAdd(J.round, rnd * J.cut_area);
    }
    crew_sync();
}

__device__ void cta_dry_cut(const Job& J, const Box& b) {
    const int res = J.res;
    const float eps = J.eps;
    if (!(eps > 0.0f)) return;
    float* __restrict__ h = J.h;
    float* __restrict__ u = J.u;
    float* __restrict__ v = J.v;
    double cut = 0.0;  // depth the cut removes, booked so the FP64 books still close
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        if (h[g] < eps) {
            if (h[g] > 0.0f) cut += (double)h[g];
            h[g] = 0.0f;
            u[g] = 0.0f;
            v[g] = 0.0f;
        }
    })
    for (int o = 16; o > 0; o >>= 1) cut += __shfl_down_sync(0xffffffffu, cut, o);
    if ((threadIdx.x & 31) == 0 && cut > 0.0 && J.cut) atomicAdd(J.cut, cut * J.cut_area);
    crew_sync();
}

// ---------------------------------------------------------------- walls
// The walled sheet's passes (src/fluid_core.rs:4225-4582). Each writes only
// cells that the pass itself never reads (wall cells from open ones, or a cell
// from its own values), so it runs in place on the crew; redirect, which
// moves depth between neighbours, books into scratch first.

// Four-neighbour offsets in the reference's order: (-1,0), (1,0), (0,-1), (0,1).
__device__ __forceinline__ int nb_di(int k) { return k == 0 ? -1 : (k == 1 ? 1 : 0); }
__device__ __forceinline__ int nb_dj(int k) { return k == 2 ? -1 : (k == 3 ? 1 : 0); }

__device__ __forceinline__ bool wall_at(const uint8_t* W, int res, int i, int j) {
    return i >= 0 && j >= 0 && i < res && j < res && W[j * res + i] != 0;
}
__device__ __forceinline__ bool open_at(const uint8_t* W, int res, int i, int j) {
    return i >= 0 && j >= 0 && i < res && j < res && W[j * res + i] == 0;
}

// solid_near (:4565-4582, radius 1): a wall among the eight neighbours.
__device__ __forceinline__ bool wall_near(const uint8_t* W, int res, int i, int j) {
    for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di)
            if ((di | dj) && wall_at(W, res, i + di, j + dj)) return true;
    return false;
}

// displace_occupied (:4382-4444) on the whole window: a covered column goes,
// in equal shares, to its open four-neighbours (to the open cells of its 5 x 5
// block when none is open) and the cell empties; with nowhere to go it stays.
// Each open cell gathers its shares in the reference's order (sources in
// raster order) into f1, then every cell applies its change.
__device__ void cta_displace(const Job& J) {
    const int res = J.res;
    const uint8_t* __restrict__ W = J.solid;
    float* __restrict__ H = J.h;
    float* __restrict__ give = J.f1;
    // Open cells a wall cell at (si, sj) would give to: its four-neighbours,
    // or its 5 x 5 block when none of those is open.
    auto share_count = [&](int si, int sj, bool& four) {
        int n = 0;
        for (int k = 0; k < 4; ++k) n += open_at(W, res, si + nb_di(k), sj + nb_dj(k)) ? 1 : 0;
        four = n > 0;
        if (four) return n;
        for (int dj = -2; dj <= 2; ++dj)
            for (int di = -2; di <= 2; ++di) n += open_at(W, res, si + di, sj + dj) ? 1 : 0;
        return n;
    };
    CLU_RECT(0, res - 1, 0, res - 1, {
        if (W[g] == 0) {
            float acc = 0.0f;
            for (int sj = j - 2; sj <= j + 2; ++sj)
                for (int si = i - 2; si <= i + 2; ++si) {
                    if (!wall_at(W, res, si, sj)) continue;
                    const float vol = H[sj * res + si];
                    if (vol <= 1.0e-8f) continue;
                    bool four;
                    const int n = share_count(si, sj, four);
                    if (four && abs(si - i) + abs(sj - j) != 1) continue;
                    acc += vol / (float)n;
                }
            give[g] = acc;
        }
    })
    crew_sync();
    CLU_RECT(0, res - 1, 0, res - 1, {
        if (W[g] != 0) {
            const float vol = H[g];
            bool four;
            if (vol <= 1.0e-8f || share_count(i, j, four) > 0) {
                H[g] = 0.0f;
                J.u[g] = 0.0f;
                J.v[g] = 0.0f;
            }
        } else if (give[g] > 0.0f) {
            H[g] += give[g];
        }
    })
    crew_sync();
}

// lift_solid_surface (:4225-4276): a wall cell's surface is the mean of the
// wet open cells within two cells, its own when there are none.
__device__ void cta_lift(const Job& J, const Box& b, float* eta) {
    const int res = J.res;
    const uint8_t* __restrict__ W = J.solid;
    const float eps = J.eps;
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        if (W[g] != 0) {
            float acc = 0.0f, n = 0.0f;
            for (int dj = -2; dj <= 2; ++dj)
                for (int di = -2; di <= 2; ++di) {
                    if (!(di | dj) || !open_at(W, res, i + di, j + dj)) continue;
                    const int q = (j + dj) * res + i + di;
                    if (J.h[q] <= eps) continue;
                    acc += eta[q];
                    n += 1.0f;
                }
            if (n > 0.0f) eta[g] = acc / n;
        }
    })
}

// write_noslip_ghost (:4278-4326): a wall cell takes minus the mean velocity
// of its wet open four-neighbours, zero when there are none.
__device__ void cta_ghost(const Job& J, const Box& b) {
    const int res = J.res;
    const uint8_t* __restrict__ W = J.solid;
    const float eps = J.eps;
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        if (W[g] != 0) {
            float au = 0.0f, av = 0.0f, n = 0.0f;
            for (int k = 0; k < 4; ++k) {
                const int ni = i + nb_di(k), nj = j + nb_dj(k);
                if (!open_at(W, res, ni, nj)) continue;
                const int q = nj * res + ni;
                if (J.h[q] <= eps) continue;
                au += J.u[q];
                av += J.v[q];
                n += 1.0f;
            }
            J.u[g] = n > 0.0f ? -au / n : 0.0f;
            J.v[g] = n > 0.0f ? -av / n : 0.0f;
        }
    })
}

// block_into_solid (:4328-4380): a wet open cell drops the part of its
// velocity that points into a wall neighbour, direction by direction.
__device__ void cta_block(const Job& J, const Box& b) {
    const int res = J.res;
    const uint8_t* __restrict__ W = J.solid;
    const float eps = J.eps;
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        if (W[g] == 0 && J.h[g] > eps) {
            float ux = J.u[g], vx = J.v[g];
            bool hit = false;
            for (int k = 0; k < 4; ++k) {
                if (!wall_at(W, res, i + nb_di(k), j + nb_dj(k))) continue;
                const float nx = (float)nb_di(k), nz = (float)nb_dj(k);
                const float vn = ux * nx + vx * nz;
                if (vn > 0.0f) {
                    ux -= vn * nx;
                    vx -= vn * nz;
                    hit = true;
                }
            }
            if (hit) {
                J.u[g] = ux;
                J.v[g] = vx;
            }
        }
    })
}

// redirect_into_walls (:4446-4563). Sources are the box's open cells with 2 cm
// of water; each books its removal and, per direction, the share each accepted
// flank receives. Receivers (the box and a one-cell rim) then add their shares
// in the reference's order -- sources in raster order, directions in neighbour
// order -- and the new depths land in f1 before they are copied back. The
// books live in the transient planes (the Gauss-Seidel snapshots and f2): the
// scratch sets keep what the reference's blurs left there, which the next
// step's blurs read beyond its box.
__device__ void cta_redirect(const Job& J, const Box& b, float dt) {
    const int res = J.res;
    const uint8_t* __restrict__ W = J.solid;
    float* __restrict__ H = J.h;
    const float* __restrict__ bed = J.bed;
    float* __restrict__ removed = J.gs[0];
    float* const book[4] = {J.gs[1], J.gs[2], J.gs[3], J.f2};
    // A flank q of source s takes water unless it is a wall or a dry bank
    // above the source's surface.
    auto accepts = [&](int q, int s) {
        return W[q] == 0 && !(H[q] <= 1.0e-6f && bed[q] > bed[s] + H[s] + 1.0e-3f);
    };
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        float rem = 0.0f;
        float share[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (W[g] == 0 && !(H[g] < 0.02f)) {
            for (int k = 0; k < 4; ++k) {
                const int di = nb_di(k), dj = nb_dj(k);
                if (!wall_at(W, res, i + di, j + dj)) continue;
                float vn = J.u[g] * (float)di + J.v[g] * (float)dj;
                if (open_at(W, res, i - di, j - dj)) {
                    const int up = (j - dj) * res + (i - di);
                    const float feed = J.u[up] * (float)di + J.v[up] * (float)dj;
                    if (feed > vn) vn = feed;
                }
                if (vn < 0.05f) continue;
                // The flanks: across the direction, lower index first.
                const int pi = di != 0 ? 0 : 1, pj = di != 0 ? 1 : 0;
                int n_dest = 0;
                float flank = 0.0f;
                for (int side = -1; side <= 1; side += 2) {
                    const int qi = i + side * pi, qj = j + side * pj;
                    if (qi < 0 || qj < 0 || qi >= res || qj >= res) continue;
                    const int q = qj * res + qi;
                    if (!accepts(q, g)) continue;
                    flank += H[q];
                    ++n_dest;
                }
                if (n_dest == 0) continue;
                const float excess = H[g] - flank / (float)n_dest;
                if (excess < 2.0e-3f) continue;
                const float room = H[g] - rem;
                if (room < 1.0e-6f) continue;
                const float frac = fminf(fdiv(vn * dt, J.div.cell), 0.45f);
                const float dh = fminf(fminf(excess, H[g] * frac), room);
                if (dh < 1.0e-8f) continue;
                rem += dh;
                share[k] = dh / (float)n_dest;
            }
        }
        removed[g] = rem;
        for (int k = 0; k < 4; ++k) book[k][g] = share[k];
    })
    crew_sync();
    const int ri0 = max(b.i0 - 1, 0), ri1 = min(b.i1 + 1, res - 1);
    const int rj0 = max(b.j0 - 1, 0), rj1 = min(b.j1 + 1, res - 1);
    auto in_box = [&](int i, int j) { return i >= b.i0 && i <= b.i1 && j >= b.j0 && j <= b.j1; };
    CLU_RECT(ri0, ri1, rj0, rj1, {
        // Sources whose flank this cell is: the cell above (horizontal
        // directions), left and right (vertical directions), below
        // (horizontal directions), in raster order.
        float add = 0.0f;
        const int si[4] = {i, i - 1, i + 1, i};
        const int sj[4] = {j - 1, j, j, j + 1};
        for (int t = 0; t < 4; ++t) {
            if (!in_box(si[t], sj[t])) continue;
            const int s = sj[t] * res + si[t];
            const int k0 = (t == 0 || t == 3) ? 0 : 2;
            for (int k = k0; k < k0 + 2; ++k) {
                const float sh = book[k][s];
                if (sh > 0.0f && accepts(g, s)) add += sh;
            }
        }
        const float rem = in_box(i, j) ? removed[g] : 0.0f;
        const float hv = H[g];
        J.f1[g] = (rem > 0.0f || add > 0.0f) ? fmaxf(hv - rem + add, 0.0f) : hv;
    })
    crew_sync();
    CLU_RECT(ri0, ri1, rj0, rj1, { H[g] = J.f1[g]; })
    crew_sync();
}

// Gravity then the raster-order Gauss-Seidel confinement on one box
// (force_gravity_open's serial sweep, src/fluid_core.rs:2234-2260).
__device__ int cta_gravity_gs(Shared& S, const Job& J, const Box& b, const float* p, float dt) {
    const int res = J.res;
    const float eps = J.eps;
    const FixedDiv two = J.div.two;
    float* U0 = J.gs[0];
    float* V0 = J.gs[1];
    float* UG = J.gs[2];
    float* VG = J.gs[3];
    {
        // The starting velocity on the box and its 2-cell rim, and gravity on
        // the box's wet cells, in one phase: each cell's thread copies its
        // velocity before it changes it, and gravity reads only p.
        const int x0 = max(b.i0 - 2, 0), x1 = min(b.i1 + 2, res - 1), y0 = max(b.j0 - 2, 0),
                  y1 = min(b.j1 + 2, res - 1);
        if (threadIdx.x == 0) S.chg[0] = S.chg[1] = S.chg[2] = 0;
        CLU_RECT(x0, x1, y0, y1, {
            const float u0 = J.u[g], v0 = J.v[g];
            U0[g] = u0;
            V0[g] = v0;
            if (i >= b.i0 && i <= b.i1 && j >= b.j0 && j <= b.j1 && J.h[g] > eps) {
                const int ip = min(i + 1, res - 1), im = max(i - 1, 0), jp = min(j + 1, res - 1), jm = max(j - 1, 0);
                float px = fdiv(p[j * res + ip] - p[j * res + im], two);
                float pz = fdiv(p[jp * res + i] - p[jm * res + i], two);
                float mob = job_mob(J, g);
                // force_gravity_solid (:2084-2129): at least 1 beside a wall.
                if (J.solid && J.h[g] > 0.08f && wall_near(J.solid, res, i, j)) mob = fmaxf(mob, 1.0f);
                float ug = u0 + -kGravity * px * mob * dt;
                float vg = v0 + -kGravity * pz * mob * dt;
                UG[g] = ug;
                VG[g] = vg;
                J.u[g] = ug;
                J.v[g] = vg;
            }
        })
    }
    crew_sync();
    if (!(J.vort > 0.0f)) return 0;
    // Fixed point of the sweep: cells before (i, j) in raster order read their
    // final values, (i, j) itself its post-gravity value, cells after it their
    // pre-gravity values.
    // A pass ends at the crew barrier; its verdict is the OR of every CTA's
    // flag for that pass, read from their shared memory. Flags rotate over
    // three slots, so a pass needs one barrier: pass k sets chg[k % 3] and
    // clears chg[(k + 1) % 3], which the crew last read before the barrier
    // that ended pass k - 1.
    cg::cluster_group crew = cg::this_cluster();
    int passes = 0;
    for (; passes < GS_MAX_PASSES; ++passes) {
        const int slot = passes % 3;
        if (threadIdx.x == 0) S.chg[(slot + 1) % 3] = 0;
        CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
            if (J.h[g] > eps) {
                auto pick = [&](const float* X, const float* G0, const float* SG, int a, int c) {
                    if (a == i && c == j) return SG[g];
                    const bool before = c < j || (c == j && a < i);
                    return before ? X[c * res + a] : G0[c * res + a];
                };
                auto uu = [&](int a, int c) { return pick(J.u, U0, UG, a, c); };
                auto vv = [&](int a, int c) { return pick(J.v, V0, VG, a, c); };
                float du, dv;
                float nu_ = UG[g], nv_ = VG[g];
                // Two cells inside the window no stencil index is clamped.
                const bool inner = i >= 2 && j >= 2 && i + 2 < res && j + 2 < res;
                if (inner ? conf_kick_inner(two, dt, J.vort, SweepRead{J.u, U0, UG, g, res},
                                            SweepRead{J.v, V0, VG, g, res}, du, dv)
                          : conf_kick(i, j, res, two, dt, J.vort, uu, vv, du, dv)) {
                    nu_ = UG[g] + du;
                    nv_ = VG[g] + dv;
                }
                if (__float_as_uint(nu_) != __float_as_uint(J.u[g]) || __float_as_uint(nv_) != __float_as_uint(J.v[g])) {
                    J.u[g] = nu_;
                    J.v[g] = nv_;
                    S.chg[slot] = 1;
                }
            }
        })
        crew_sync();
        const int any = crew_fold(&S.chg[slot], 0, [](int a, int b) { return a | b; });
        if (!any) break;
    }
    if (passes < GS_MAX_PASSES) return passes + 1;
    // Pass limit reached: the sweep itself, in raster order, on one thread of the crew.
    if (crew_rank() == 0 && threadIdx.x == 0) {
        for (int j = b.j0; j <= b.j1; ++j)
            for (int i = b.i0; i <= b.i1; ++i) {
                const int g = j * res + i;
                if (!(J.h[g] > eps)) continue;
                auto pick = [&](const float* X, const float* G0, const float* SG, int a, int c) {
                    if (a == i && c == j) return SG[g];
                    const bool before = c < j || (c == j && a < i);
                    return before ? X[c * res + a] : G0[c * res + a];
                };
                auto uu = [&](int a, int c) { return pick(J.u, U0, UG, a, c); };
                auto vv = [&](int a, int c) { return pick(J.v, V0, VG, a, c); };
                float du, dv;
                if (conf_kick(i, j, res, two, dt, J.vort, uu, vv, du, dv)) {
                    J.u[g] = UG[g] + du;
                    J.v[g] = VG[g] + dv;
                } else {
                    J.u[g] = UG[g];
                    J.v[g] = VG[g];
                }
            }
    }
    crew_sync();
    return -1;
}

// Gravity then snapshot-Jacobi confinement (force_gravity_par :2263-2378,
// gravity_jacobi_serial :2530-2595).
__device__ void cta_gravity_jacobi(const Job& J, const Box& b, const float* __restrict__ p, float dt) {
    // Distinct planes; each phase writes only its own cell of u, v or W.
    const int res = J.res;
    const float eps = J.eps;
    const FixedDiv two = J.div.two;
    const float* __restrict__ H = J.h;
    float* __restrict__ U = J.u;
    float* __restrict__ V = J.v;
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        if (H[g] > eps) {
            const int ip = min(i + 1, res - 1), im = max(i - 1, 0), jp = min(j + 1, res - 1), jm = max(j - 1, 0);
            float px = fdiv(p[j * res + ip] - p[j * res + im], two);
            float pz = fdiv(p[jp * res + i] - p[jm * res + i], two);
            float mob = job_mob(J, g);
            U[g] += -kGravity * px * mob * dt;
            V[g] += -kGravity * pz * mob * dt;
        }
    })
    crew_sync();
    if (!(J.vort > 0.0f)) return;
    float* __restrict__ W = J.f1;
    {
        const int wi0 = max(b.i0 - 1, 0), wi1 = min(b.i1 + 1, res - 1);
        const int wj0 = max(b.j0 - 1, 0), wj1 = min(b.j1 + 1, res - 1);
        CLU_RECT(wi0, wi1, wj0, wj1, {
            const int ip = min(i + 1, res - 1), im = max(i - 1, 0), jp = min(j + 1, res - 1), jm = max(j - 1, 0);
            float dvdx = fdiv(V[j * res + ip] - V[j * res + im], two);
            float dudz = fdiv(U[jp * res + i] - U[jm * res + i], two);
            W[g] = dvdx - dudz;
        })
    }
    crew_sync();
    const float vort = J.vort;
    CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
        if (H[g] > eps) {
            float w = W[g];
            if (finite_f(w) && !(fabsf(w) < 1.0e-4f)) {
                const int ip = min(i + 1, res - 1), im = max(i - 1, 0), jp = min(j + 1, res - 1), jm = max(j - 1, 0);
                float wxp = fabsf(W[j * res + ip]), wxm = fabsf(W[j * res + im]);
                float wzp = fabsf(W[jp * res + i]), wzm = fabsf(W[jm * res + i]);
                float nx = fdiv(wxp - wxm, two);
                float nz = fdiv(wzp - wzm, two);
                float du = vort * dt * (-nz * w);
                float dv = vort * dt * (nx * w);
                if (finite_f(du) && finite_f(dv) && du * du + dv * dv <= 0.0625f) {
                    U[g] += du;
                    V[g] += dv;
                }
            }
        }
    })
    crew_sync();
}

// substep (src/fluid_core.rs:1879-2082), open sheet, gravity drive.
__device__ __forceinline__ int cta_substep(Shared& S, const Job& J, const Box& b, float* const* sc, float dt, float decay_c,
                           bool do_flux, bool inner_par) {
    const int res = J.res;
    float* __restrict__ sa = sc[0];
    float* __restrict__ sb = sc[1];
    float* __restrict__ scc = sc[2];
    float* __restrict__ sd = sc[3];
    float* __restrict__ se = sc[4];
    const float eps = J.eps, cell = J.cell;
    const bool fine = cell <= kFineCell + 1.0e-6f;
    const bool walled = J.solid != nullptr;
    {
        const float* __restrict__ bed = J.bed;
        const float* __restrict__ H = J.h;
        const int hi0 = max(b.i0 - 2, 0), hi1 = min(b.i1 + 2, res - 1);
        const int hj0 = max(b.j0 - 2, 0), hj1 = min(b.j1 + 2, res - 1);
        CLU_RECT(hi0, hi1, hj0, hj1, { sa[g] = bed[g] + H[g]; })
    }
    crew_sync();
    if (walled) {
        cta_lift(J, b, sa);
        crew_sync();
    }
    cta_blur_pair(sa, sb, scc, se, J.f1, res, b, [&](int g, float gauss, float steep) {
        float filtered = 0.62f * gauss + 0.38f * steep;
        sd[g] = 0.45f * filtered + 0.55f * sa[g];
    });
    const bool par = (b.j1 - b.j0 >= 47) && (b.i1 - b.i0 >= 31) && inner_par;
    int passes = 0;
    if (walled) {
        // A walled sheet sweeps serially on every grid (the step pair's
        // serial inner loops; the free operator takes no walls).
        cta_ghost(J, b);
        crew_sync();
        passes = cta_gravity_gs(S, J, b, sd, dt);
    } else if (fine || par) {
        cta_gravity_jacobi(J, b, sd, dt);
    } else {
        passes = cta_gravity_gs(S, J, b, sd, dt);
    }
    const bool project = !fine || walled;
    if (project) {
        CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
            const int ip = min(i + 1, res - 1), im = max(i - 1, 0), jp = min(j + 1, res - 1), jm = max(j - 1, 0);
            float ux = fdiv(J.u[j * res + ip] - J.u[j * res + im], J.div.two);
            float vz = fdiv(J.v[jp * res + i] - J.v[jm * res + i], J.div.two);
            float div = ux + vz;
            float s = sa[j * res + ip] + sa[j * res + im] + sa[jp * res + i] + sa[jm * res + i] - 4.0f * sa[g];
            float lap_h = fdiv(s, J.div.cell2);
            float overload = 1.0f + rclamp(fdiv(job_nu(J, g), J.div.d231), 0.0f, 6.0f);
            sb[g] = div * overload - 0.015f * overload * lap_h;
        })
        crew_sync();
        cta_blur_pair(sb, scc, sa, se, J.f1, res, b,
                      [&](int g, float gauss, float steep) { sd[g] = 0.62f * gauss + 0.38f * steep; });
    }
    {
        const float* __restrict__ H = J.h;
        float* __restrict__ U = J.u;
        float* __restrict__ V = J.v;
        CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
            if (H[g] > eps) {
                float uu = U[g], vv = V[g];
                if (project) {
                    const int ip = min(i + 1, res - 1), im = max(i - 1, 0), jp = min(j + 1, res - 1),
                              jm = max(j - 1, 0);
                    float qx = fdiv(sd[j * res + ip] - sd[j * res + im], J.div.two);
                    float qz = fdiv(sd[jp * res + i] - sd[jm * res + i], J.div.two);
                    uu += 0.012f * dt * qx;
                    vv += 0.012f * dt * qz;
                }
                float decay = job_decay(J, g, dt, decay_c);
                U[g] = finite_speed(uu * decay, kSpeedCap);
                V[g] = finite_speed(vv * decay, kSpeedCap);
            }
        })
    }
    crew_sync();
    if (walled) {
        cta_redirect(J, b, dt);
        cta_block(J, b);
        crew_sync();
        cta_ghost(J, b);
        crew_sync();
    }
    if (do_flux) {
        cta_transport(J, b, dt);
        cta_dry_cut(J, b);
    }
    return passes;
}

// awake_work_boxes (src/fluid_core.rs:1537-1657).
// Called by the whole crew: the crew marks rank 0's hot tiles, rank 0 does
// the rest (labels and boxes in its shared memory).
__device__ void cta_awake_boxes(Shared& S, const Job& J) {
    const int res = J.res;
    const int tiles = (res + SLEEP_TILE - 1) / SLEEP_TILE;
    const int ntile = tiles * tiles;
    if (crew_rank() == 0)
        for (int t = threadIdx.x; t < ntile; t += NT) {
            S.hot[t] = 0;
            S.grown[t] = 0;
        }
    crew_sync();
    Shared* S0 = cg::this_cluster().map_shared_rank(&S, 0);
    const float eps = J.eps, cell = J.cell;
    CLU_RECT(0, res - 1, 0, res - 1, {
        float hv = J.h[g];
        if (hv > eps) {
            bool awake = hypot_rn(J.u[g], J.v[g]) > 0.05f;
            if (!awake) {
                float eta = J.bed[g] + hv;
                int ip = i + 1 < res ? g + 1 : g;
                int jp = j + 1 < res ? g + res : g;
                float dex = fabsf(J.bed[ip] + J.h[ip] - eta);
                float dez = fabsf(J.bed[jp] + J.h[jp] - eta);
                awake = fmaxf(dex, dez) > 0.02f * cell;
            }
            if (awake) S0->hot[(j / SLEEP_TILE) * tiles + i / SLEEP_TILE] = 1;
        }
    })
    crew_sync();
    if (crew_rank() != 0) return;
    for (int t = threadIdx.x; t < ntile; t += NT) {
        int ti = t % tiles, tj = t / tiles;
        unsigned char gr = 0;
        for (int dj = -1; dj <= 1; ++dj)
            for (int di = -1; di <= 1; ++di) {
                int ni = ti + di, nj = tj + dj;
                if (ni >= 0 && nj >= 0 && ni < tiles && nj < tiles && S.hot[nj * tiles + ni]) gr = 1;
            }
        S.grown[t] = gr;
        S.lab[t] = gr ? t : 0x7fffffff;
    }
    __syncthreads();
    // Component label = first tile in raster order, the order the reference's scan finds them.
    for (int iter = 0; iter < 4 * MAX_TILES; ++iter) {
        if (threadIdx.x == 0) S.changed = 0;
        __syncthreads();
        for (int t = threadIdx.x; t < ntile; t += NT) {
            if (!S.grown[t]) continue;
            int ti = t % tiles, tj = t / tiles;
            int m = S.lab[t];
            if (ti > 0 && S.grown[t - 1]) m = min(m, S.lab[t - 1]);
            if (ti + 1 < tiles && S.grown[t + 1]) m = min(m, S.lab[t + 1]);
            if (tj > 0 && S.grown[t - tiles]) m = min(m, S.lab[t - tiles]);
            if (tj + 1 < tiles && S.grown[t + tiles]) m = min(m, S.lab[t + tiles]);
            m = min(m, S.lab[m]);
            if (m < S.lab[t]) {
                atomicMin(&S.lab[t], m);
                S.changed = 1;
            }
        }
        __syncthreads();
        if (!S.changed) break;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        int nb = 0;
        for (int t = 0; t < ntile; ++t)
            if (S.grown[t] && S.lab[t] == t && nb < MAX_BOXES) {
                S.bbox[0][nb] = t % tiles;
                S.bbox[1][nb] = t % tiles;
                S.bbox[2][nb] = t / tiles;
                S.bbox[3][nb] = t / tiles;
                S.lab[t] = -(nb + 1);
                ++nb;
            }
        S.nbox = nb;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < ntile; t += NT) {
        if (!S.grown[t]) continue;
        int r = S.lab[t];
        int slot = r < 0 ? -r - 1 : -S.lab[r] - 1;
        if (slot < 0 || slot >= MAX_BOXES) continue;
        int ti = t % tiles, tj = t / tiles;
        atomicMin(&S.bbox[0][slot], ti);
        atomicMax(&S.bbox[1][slot], ti);
        atomicMin(&S.bbox[2][slot], tj);
        atomicMax(&S.bbox[3][slot], tj);
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < S.nbox; ++k) {
            int ti0 = S.bbox[0][k], ti1 = S.bbox[1][k], tj0 = S.bbox[2][k], tj1 = S.bbox[3][k];
            S.bbox[0][k] = ti0 * SLEEP_TILE;
            S.bbox[1][k] = min((ti1 + 1) * SLEEP_TILE, res) - 1;
            S.bbox[2][k] = tj0 * SLEEP_TILE;
            S.bbox[3][k] = min((tj1 + 1) * SLEEP_TILE, res) - 1;
        }
    __syncthreads();
}

__device__ __forceinline__ bool boxes_touch(int a0, int a1, int a2, int a3, int b0, int b1, int b2, int b3) {
    auto ss = [](int x) { return x > 0 ? x - 1 : 0; };
    return ss(a0) <= b1 + 1 && ss(b0) <= a1 + 1 && ss(a2) <= b3 + 1 && ss(b2) <= a3 + 1;
}

__device__ void set_whole(Shared& S, int x0, int x1, int y0, int y1) {
    if (threadIdx.x == 0) {
        S.nbox = 1;
        S.bbox[0][0] = x0;
        S.bbox[1][0] = x1;
        S.bbox[2][0] = y0;
        S.bbox[3][0] = y1;
    }
    __syncthreads();
}

// sheet_work_boxes (src/fluid_core.rs:1325-1447). Wet bodies are labelled in
// the f2 plane (as ints) by hooking and pointer jumping; a body's root is its
// first wet cell in raster order, the order the reference's run merge keeps.
// The wet-body labels of sheet_work_boxes (src/fluid_core.rs:1378-1457) over
// the wet extent, by the whole crew, into the plane f2: every wet cell ends
// holding its body's smallest index (its first raster cell). Hook and jump:
// each round lowers the label of the larger of two neighbours' labels to the
// smaller root (each cell walks to its root first), then points every cell
// at its root. Labels only fall and stay inside the body, so the rounds end
// at that fixed point, in a few rounds. A run's cells start with the same
// label, which only shortens the rounds: the fixed point is the same. Nothing
// to label when no cell is wet or
// every cell of the extent is (cta_wet_boxes then takes the whole box).
__device__ void crew_label_bodies(Shared& S, const Job& J, const int ext[5]) {
    const int res = J.res;
    const float eps = J.eps;
    const int wet = ext[0], i0 = ext[1], i1 = -ext[2], j0 = ext[3], j1 = ext[4];
    if (wet == 0 || wet == (i1 - i0 + 1) * (j1 - j0 + 1)) return;
    int* L = reinterpret_cast<int*>(J.f2);
    // Start from runs: a wet cell takes the index of the first cell of its
    // horizontal run within its warp's 32-cell chunk (a ballot finds it), so
    // the rounds only join runs.
    {
        const int ch = (i1 - i0 + 32) >> 5;
        const int items = (j1 - j0 + 1) * ch;
        const int lane = (int)(threadIdx.x & 31);
        for (int it = crew_rank() * (NT / 32) + (int)(threadIdx.x >> 5); it < items; it += crew_size() * (NT / 32)) {
            const int r = it / ch;
            const int j = j0 + r;
            const int ib = i0 + (it - r * ch) * 32;
            const int i = ib + lane;
            const bool in = i <= i1;
            const int g = j * res + i;
            const bool wet = in && J.h[g] > eps;
            const unsigned m = __ballot_sync(0xffffffffu, wet);
            // The run's first lane: the lowest lane at or below this one such
            // that every lane from it up to this one is wet.
            const unsigned dry_below = ~m & ((lane == 31) ? 0xffffffffu : ((1u << (lane + 1)) - 1u));
            const int first = dry_below ? (32 - __clz(dry_below)) : 0;
            if (in) L[g] = wet ? j * res + ib + first : -1;
        }
    }
    if (threadIdx.x == 0) S.lchg[0] = S.lchg[1] = S.lchg[2] = 0;
    crew_sync();
    // A cell's root: follow the labels down (they only fall, so the walk
    // ends; the cap only bounds a walk, the rounds still reach the fixed point).
    auto root = [&](int x) {
        for (int k = 0; k < 4096; ++k) {
            const int y = ((volatile int*)L)[x];
            if (y == x) break;
            x = y;
        }
        return x;
    };
    for (int round = 0; round < 4096; ++round) {
        const int slot = round % 3;
        // Round k sets lchg[k % 3] and clears lchg[(k + 1) % 3], which the
        // crew last read in round k - 2, two barriers ago.
        if (threadIdx.x == 0) S.lchg[(slot + 1) % 3] = 0;
        // Hook: two wet neighbours with different roots hang the larger root
        // under the smaller.
        CLU_RECT(i0, i1, j0, j1, {
            const int a = L[g];
            if (a >= 0) {
                const int ra = root(a);
                if (i < i1 && L[g + 1] >= 0) {
                    const int rc = root(L[g + 1]);
                    if (rc != ra) {
                        atomicMin(&L[max(ra, rc)], min(ra, rc));
                        S.lchg[slot] = 1;
                    }
                }
                if (j < j1 && L[g + res] >= 0) {
                    const int rc = root(L[g + res]);
                    if (rc != ra) {
                        atomicMin(&L[max(ra, rc)], min(ra, rc));
                        S.lchg[slot] = 1;
                    }
                }
            }
        })
        crew_sync();
        // Compress: every cell points at its root.
        CLU_RECT(i0, i1, j0, j1, {
            const int a = L[g];
            if (a >= 0) {
                const int r = root(a);
                if (r != a) {
                    L[g] = r;
                    S.lchg[slot] = 1;
                }
            }
        })
        crew_sync();
        if (!crew_fold(&S.lchg[slot], 0, [](int x, int y) { return x | y; })) break;
    }
}

// `ext`: the crew's wet extent of the layer (crew_sum_extent).
__device__ void cta_wet_boxes(Shared& S, const Job& J, const int ext[5]) {
    const int res = J.res;
    const int wet = ext[0], i0 = ext[1], i1 = -ext[2], j0 = ext[3], j1 = ext[4];
    if (wet == 0) {
        if (threadIdx.x == 0) S.nbox = 0;
        __syncthreads();
        return;
    }
    const int x0 = max(i0 - 3, 0), x1 = min(i1 + 3, res - 1), y0 = max(j0 - 3, 0), y1 = min(j1 + 3, res - 1);
    if (wet == (i1 - i0 + 1) * (j1 - j0 + 1)) {
        set_whole(S, x0, x1, y0, y1);
        return;
    }
    // The crew has labelled every wet cell of the box with its body's first
    // raster cell (crew_label_bodies).
    int* L = reinterpret_cast<int*>(J.f2);
    // Roots in raster order: count per row, scan, then number them.
    const int rows = j1 - j0 + 1;
    for (int r = threadIdx.x; r < rows; r += NT) {
        int c = 0;
        const int j = j0 + r;
        for (int i = i0; i <= i1; ++i) c += L[j * res + i] == j * res + i;
        S.row_count[r] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int r = 0; r < rows; ++r) {
            int c = S.row_count[r];
            S.row_count[r] = acc;
            acc += c;
        }
        S.nbox = acc;
    }
    __syncthreads();
    const int nbodies = S.nbox;
    // More than MAX_BOXES bodies: step the whole box. The reference merges the
    // grown bodies first and only then falls back at more than 8 boxes, so
    // this differs from it only when over 512 separate bodies would merge
    // into 8 or fewer boxes.
    if (nbodies > MAX_BOXES) {
        __syncthreads();
        set_whole(S, x0, x1, y0, y1);
        return;
    }
    for (int r = threadIdx.x; r < rows; r += NT) {
        int slot = S.row_count[r];
        const int j = j0 + r;
        for (int i = i0; i <= i1; ++i) {
            const int g = j * res + i;
            if (L[g] == g) {
                S.bbox[0][slot] = i;
                S.bbox[1][slot] = i;
                S.bbox[2][slot] = j;
                S.bbox[3][slot] = j;
                L[g] = -(slot + 2);
                ++slot;
            }
        }
    }
    __syncthreads();
    CTA_RECT(i0, i1, j0, j1, {
        int r = L[g];
        if (r >= 0 || r <= -2) {
            int slot = r >= 0 ? -L[r] - 2 : -r - 2;
            if (slot >= 0 && slot < MAX_BOXES) {
                atomicMin(&S.bbox[0][slot], i);
                atomicMax(&S.bbox[1][slot], i);
                atomicMin(&S.bbox[2][slot], j);
                atomicMax(&S.bbox[3][slot], j);
            }
        }
    })
    __syncthreads();
    if (threadIdx.x == 0) {
        int nb = nbodies;
        for (int k = 0; k < nb; ++k) {
            S.bbox[0][k] = max(S.bbox[0][k] - 6, 0);
            S.bbox[1][k] = min(S.bbox[1][k] + 6, res - 1);
            S.bbox[2][k] = max(S.bbox[2][k] - 6, 0);
            S.bbox[3][k] = min(S.bbox[3][k] + 6, res - 1);
        }
        // merge_boxes (src/fluid_core.rs:1459-1487), swap_remove order.
        for (;;) {
            bool did = false;
            int a = 0;
            while (a < nb) {
                int c = a + 1;
                while (c < nb) {
                    if (boxes_touch(S.bbox[0][a], S.bbox[1][a], S.bbox[2][a], S.bbox[3][a], S.bbox[0][c],
                                    S.bbox[1][c], S.bbox[2][c], S.bbox[3][c])) {
                        S.bbox[0][a] = min(S.bbox[0][a], S.bbox[0][c]);
                        S.bbox[1][a] = max(S.bbox[1][a], S.bbox[1][c]);
                        S.bbox[2][a] = min(S.bbox[2][a], S.bbox[2][c]);
                        S.bbox[3][a] = max(S.bbox[3][a], S.bbox[3][c]);
                        for (int q = 0; q < 4; ++q) S.bbox[q][c] = S.bbox[q][nb - 1];
                        --nb;
                        did = true;
                    } else {
                        ++c;
                    }
                }
                ++a;
            }
            if (!did) break;
        }
        if (nb == 1 || nb > 8) {
            nb = 1;
            S.bbox[0][0] = x0;
            S.bbox[1][0] = x1;
            S.bbox[2][0] = y0;
            S.bbox[3][0] = y1;
        }
        S.nbox = nb;
    }
    __syncthreads();
}

// soften_border (src/fluid_core.rs:9594-9622) on the whole layer.
__device__ void cta_soften(const Job& J) {
    const int res = J.res, edge = J.soften_edge;
    // The band's rows and columns: [0, lo] and [hi, res).
    const int lo = min(edge, res) - 1, hi = min(max(edge, res - edge), res);
#define SOFTEN_CELL                                                     \
    {                                                                   \
        const int dx_ = min(i, res - 1 - i), dz_ = min(j, res - 1 - j); \
        int d = min(dx_, dz_);                                          \
        if (J.open_axis == 1 && j >= J.open_c0 && j < J.open_c1)        \
            d = dz_;                                                    \
        else if (J.open_axis == 2 && i >= J.open_c0 && i < J.open_c1)   \
            d = dx_;                                                    \
        if (d < edge) {                                                 \
            float t = (float)d / (float)edge;                           \
            float w = t * t * (3.0f - 2.0f * t);                        \
            J.u[g] *= w;                                                \
            J.v[g] *= w;                                                \
        }                                                               \
    }
    // Only the band within `edge` of the border: the top and bottom rows,
    // then the left and right columns of the rows between.
    CLU_RECT(0, res - 1, 0, lo, SOFTEN_CELL)
    CLU_RECT(0, res - 1, hi, res - 1, SOFTEN_CELL)
    CLU_RECT(0, lo, lo + 1, hi - 1, SOFTEN_CELL)
    CLU_RECT(hi, res - 1, lo + 1, hi - 1, SOFTEN_CELL)
#undef SOFTEN_CELL
    crew_sync();
}

// The layer's FP64 depth sum over the crew; rank 0 writes it.
__device__ void cta_ledger(Shared& S, const Job& J) {
    const int res = J.res;
    double part = 0.0;
    CLU_RECT(0, res - 1, 0, res - 1, { part += (double)fmaxf(J.h[g], 0.0f); })
    part = crew_sum_d(S, part);
    if (threadIdx.x == 0 && J.ledger && crew_rank() == 0) *J.ledger = part;
}

// step_sheet_eps_in + step_sheet_scratch (src/fluid_core.rs:821-852, :1659-1831).
// One window layer's step; returns the Gauss-Seidel passes of its last box.
__device__ __forceinline__ int window_body(Shared& S, const Job& J) {
    int gs_passes = 0;
    const int res = J.res;
    const float eps = J.eps;
    if (J.soften_edge > 0) cta_soften(J);
    if (J.solid) cta_displace(J);
    // wet_sum early out (src/fluid_core.rs:1306-1319, :840-844), over the crew.
    double ws = 0.0;
    int ext[5] = {0, res, 1, res, -1};  // wet cells, min i, -max i, min j, max j
    CLU_RECT(0, res - 1, 0, res - 1, {
        float hv = J.h[g];
        if (hv > eps) {
            ws += (double)hv;
            ext[0] += 1;
            ext[1] = min(ext[1], i);
            ext[2] = min(ext[2], -i);
            ext[3] = min(ext[3], j);
            ext[4] = max(ext[4], j);
        }
    })
    ws = crew_sum_extent(S, ws, ext);
    if (!(ws > (double)eps)) {
        cta_ledger(S, J);
        return 0;
    }
    const bool open_fine = !J.solid && J.cell <= kFineCell + 1.0e-6f;
    const bool fine_open = open_fine && J.pace == 0;
    const bool whole_wet = open_fine && (J.pace == 2 || J.pace == 3);
    const bool awake = open_fine && !whole_wet && !fine_open;
    // Work boxes on rank 0 (the wet-body labels use a global plane; the awake
    // scan is shared by the crew), then every other CTA copies them from its
    // shared memory.
    if (fine_open || awake) {
        cta_awake_boxes(S, J);
    } else {
        crew_label_bodies(S, J, ext);
        if (crew_rank() == 0) cta_wet_boxes(S, J, ext);
    }
    crew_sync();
    if (crew_rank() != 0) {
        const Shared* S0 = cg::this_cluster().map_shared_rank(&S, 0);
        const int n0 = S0->nbox;
        for (int k = threadIdx.x; k < 4 * n0; k += NT) S.bbox[k / n0][k % n0] = S0->bbox[k / n0][k % n0];
        if (threadIdx.x == 0) S.nbox = n0;
        __syncthreads();
    }
    const int nb = S.nbox;
    if (nb <= 0) {
        cta_ledger(S, J);
        return 0;
    }
    const float cap = finite_f(J.sub_cap) ? rclamp(J.sub_cap, 1.0f, 8.0f) : 8.0f;
    int nsub = 1;
    if (!fine_open) {
        float m2 = 0.0f;
        for (int k = 0; k < nb; ++k) {
            const Box b = {S.bbox[0][k], S.bbox[1][k], S.bbox[2][k], S.bbox[3][k]};
            CLU_RECT(b.i0, b.i1, b.j0, b.j1, {
                float uu = J.u[g], vv = J.v[g];
                float s2 = uu * uu + vv * vv;
                if (s2 > m2) m2 = s2;
            })
        }
        m2 = crew_max_f(S, m2);
        float max_s = fmaxf(0.15f, sqrtf(m2));
        nsub = (int)rclamp(ceilf((J.dt * max_s) / (0.42f * fmaxf(J.cell, 1.0e-3f))), 1.0f, cap);
    }
    const float dts = J.dt / (float)nsub;
    float* set0[5] = {J.sc[0][0], J.sc[0][1], J.sc[0][2], J.sc[0][3], J.sc[0][4]};
    float* set1[5] = {J.sc[1][0], J.sc[1][1], J.sc[1][2], J.sc[1][3], J.sc[1][4]};
    auto ap = [](int a0, int a1, int b0, int b1) { return a1 + 6 < b0 || b1 + 6 < a0; };
    const bool two_apart = J.has_sc2 && nb == 2 &&
                           (ap(S.bbox[0][0], S.bbox[1][0], S.bbox[0][1], S.bbox[1][1]) ||
                            ap(S.bbox[2][0], S.bbox[3][0], S.bbox[2][1], S.bbox[3][1]));
    // Two far-apart boxes run on two workers with the inner loops serial.
    const bool inner = two_apart ? false : (J.inner_par != 0);
    if (J.pace == 3 && whole_wet && nsub > 1) {
        for (int k = 0; k < nb; ++k) {
            const Box b = {S.bbox[0][k], S.bbox[1][k], S.bbox[2][k], S.bbox[3][k]};
            float* const* sc = (two_apart && k == 1) ? set1 : set0;
            gs_passes = cta_substep(S, J, b, sc, J.dt, J.decay_c[1], false, inner);
            for (int s = 0; s < nsub; ++s) cta_transport(J, b, dts);
            cta_dry_cut(J, b);
        }
    } else {
        for (int s = 0; s < nsub; ++s)
            for (int k = 0; k < nb; ++k) {
                const Box b = {S.bbox[0][k], S.bbox[1][k], S.bbox[2][k], S.bbox[3][k]};
                float* const* sc = (two_apart && k == 1) ? set1 : set0;
                int p = cta_substep(S, J, b, sc, dts, J.decay_c[nsub], true, inner);
                gs_passes = p < 0 || gs_passes < 0 ? -1 : max(gs_passes, p);
            }
    }
    cta_ledger(S, J);
    return gs_passes;
}

__device__ __forceinline__ void window_job(Job* jp) {
    __shared__ Shared S;
    __shared__ Job Js;
    // The job's fields live in shared memory for the step: every phase reads
    // them, and a copy on the thread's stack would be reloaded from local
    // memory after each store through a plane pointer.
    if (threadIdx.x == 0) Js = *jp;
    __syncthreads();
    if (!Js.active) return;  // the same for the whole crew
    const int gs_passes = window_body(S, Js);
    if (threadIdx.x == 0 && crew_rank() == 0) jp->gs_iters = gs_passes;
    crew_sync();  // no CTA leaves while another may still read its shared memory
}

// Job k of an array.
__global__ void __launch_bounds__(NT, 1) k_window_step(Job* jobs) {
    ::silt::dep_wait();
    window_job(jobs + blockIdx.x / (unsigned)crew_size());
}

// Job k of a list of jobs that live in different tables (batched windows).
__global__ void __launch_bounds__(NT, 1) k_window_step_list(Job* const* jobs) {
    ::silt::dep_wait();
    window_job(jobs[blockIdx.x / (unsigned)crew_size()]);
}

// Largest crew: 16 CTAs, the non-portable cluster size B200 allows.
constexpr int MAX_CREW = 16;

// CTAs per job: enough warps for one (row, 32-cell chunk) item each on a
// 64-cell patch, up to the largest crew.
static int crew_for(int max_res) {
    const int items = max_res * ((max_res + 31) / 32);
    int c = items / (NT / 32);
    if (c < 1) c = 1;
    if (c > MAX_CREW) c = MAX_CREW;
    return c;
}

// The largest crew the device can hold at once (a cluster of full-SM CTAs).
static int crew_limit_query(cudaStream_t st) {
    if (cudaFuncSetAttribute(k_window_step, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
        cudaFuncSetAttribute(k_window_step_list, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 8;  // the portable size
    }
    for (int c = MAX_CREW; c >= 1; --c) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)c, 1, 1);
        cfg.blockDim = dim3(NT, 1, 1);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, k_window_step, &cfg) == cudaSuccess && n > 0) return c;
        cudaGetLastError();
    }
    return 1;
}

static int crew_limit(cudaStream_t st) {
    static std::once_flag once;
    static int limit = 1;
    std::call_once(once, [st] { limit = crew_limit_query(st); });
    return limit;
}

// The crew for `njobs` jobs: as large as the window and the device allow, and
// small enough that all the jobs' CTAs fit on the GPU about twice over.
static int crew_of(int njobs, int max_res, cudaStream_t st) {
    return std::max(1, std::min({crew_for(max_res), crew_limit(st), 296 / std::max(njobs, 1)}));
}

cudaError_t launch_window_step_list(Job* const* d_job_list, int njobs, int max_res, cudaStream_t st) {
    if (njobs <= 0) return cudaSuccess;
    const int crew = crew_of(njobs, max_res, st);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(njobs * crew), 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)crew;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;  // the kernel starts with dep_wait()
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    cudaError_t e = ::silt::launch_ex(cfg, k_window_step_list, d_job_list);
    ::silt::count_launch();
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_window_step(const Job* d_jobs, int njobs, int max_res, cudaStream_t st) {
    if (njobs <= 0) return cudaSuccess;
    const int crew = crew_of(njobs, max_res, st);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(njobs * crew), 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)crew;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;  // the kernel starts with dep_wait()
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    cudaError_t e = ::silt::launch_ex(cfg, k_window_step, const_cast<Job*>(d_jobs));
    ::silt::count_launch();
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

size_t window_static_smem() { return sizeof(Shared); }

}  // namespace window
}  // namespace silt
