// Launch parameters of the full-grid sheet kernels (sheet_grid.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "sheet_div.cuh"

namespace silt {

enum NuMode : int32_t {
    NU_CONST = 0,   // one viscosity for the whole layer (the water sheet, 0.9 Pa s)
    NU_PLANE = 1,   // a float viscosity per cell (the free step_sheet operator)
    NU_GRAIN = 2,   // dynamic_viscosity(grain, moisture) per cell
    NU_TABLE = 3,   // nu_plane, mob_plane, damp_plane: the laws evaluated once per cell beforehand (the slurry sheet)
};

struct LayerParams {
    const float* h;
    const float* bed;
    const float* u;
    const float* v;
    float* u_out;
    float* v_out;
    const uint8_t* grain;
    const float* moisture;
    const float* nu_plane;
    const float* mob_plane;   // NU_TABLE
    const float* damp_plane;  // NU_TABLE
    int32_t nu_mode;
    float nu_c, mob_c, decay_c;  // NU_CONST: viscosity, mobility and damping factor
    int32_t res;
    float cell, dt, vort, eps;
    FixedDiv div_two;      // 2 * cell (the centred differences)
    FixedDiv div_cell2;    // cell * cell (the laplacian)
    FixedDiv div_231;      // 231 (the projection's overload)
    int32_t project;       // divergence projection (cells wider than 2 cm)
    int32_t soften_edge;   // soft window band width in cells, 0 = off
    int32_t open_axis;     // a river reach's band through the window ends: 0 none, 1 rows [open_c0, open_c1)
    int32_t open_c0, open_c1;  // (reach along X), 2 columns (along Z); there only one edge distance softens
    int32_t apply_cut;     // zero u, v where h < eps on load (the previous dry cut)
    int32_t skip;          // layer has nothing to do this substep
    // Confinement form. sweep = 1: the reference's raster-order Gauss-Seidel
    // sweep (force_gravity_open, src/fluid_core.rs:2234-2260), solved on the
    // grid as a fixed point in the planes fu, fv; sweep = 0: the snapshot
    // (Jacobi) form of force_gravity_par (:2263).
    int32_t sweep;
    float* fu;
    float* fv;
};

// Device state of one Gauss-Seidel sweep launch: the grid barrier's arrival
// count and the pass verdicts (cleared by the tile-list kernel before every
// force launch), a sticky error for a barrier wait that gave up, and pass
// statistics.
struct SweepState {
    unsigned int bar;         // CTAs arrived at the grid barrier in this launch
    unsigned int flag[3];     // pass p's verdict in flag[p % 3]: some tile changed
    unsigned int err;         // sticky: bit 0 a barrier wait ran past its limit, bit 1 a transport tile's
                              // TMA copies did not arrive within theirs
    unsigned int passes_max;  // most passes one launch needed
    unsigned int fallbacks;   // launches that ran the sequential sweep after the pass limit
    unsigned int launches;    // sweep launches
    unsigned int epoch;       // launches ever (never reset): the base of the tiles' change stamps
    unsigned int solves;      // tile solves (a tile in a pass) since step timing was last set
    unsigned int local_passes;  // local passes of those solves
};

// Active-tile bookkeeping of the grid engine, per layer and ping-pong buffer,
// one byte per 32 x 32 tile. A tile is stepped only when some tile of its
// 3 x 3 neighbourhood may hold water; every other tile is provably unchanged
// (no depth within the force and transport halos, no velocity after the dry
// cut) and is written once with zeros, then skipped while its buffer stays zero.
struct TileFlags {
    uint8_t* wet[2][2];      // [layer][buffer]: the tile may hold water
    uint8_t* zero_uv[2][2];  // [layer][buffer]: u and v of the tile are all zero
    uint8_t* zero_h[2][2];   // [layer][buffer]: h of the tile is all zero
    int* list;               // entries (layer << 30) | (zero_fill << 29) | tile
    int* count;
    unsigned long long* stepped;  // per layer: running total of tiles stepped (may be nullptr)
    int32_t tiles_x;
    SweepState* sweep;       // cleared by the tile-list kernel (may be nullptr)
    // Per layer and tile (stamp[l * tiles_x^2 + t]): when the sweep last
    // changed the tile, as epoch * 256 + pass + 1. A later pass solves a tile
    // again only when its 3 x 3 neighbourhood changed since it was solved.
    unsigned int* stamp;
};

// Substep count decided on the device (src/fluid_core.rs:1715-1744). The
// largest squared speed of each layer, reduced over the tiles that may hold
// water, gives the layer's count n = clamp(ceil(dt max(0.15, s) / (0.42 cell)),
// 1, cap); the tile-list, force and transport kernels of substep k read it and
// step with dt / n while k < n. The host launches `launched` substeps from its
// own speed bound; a layer that needs fewer copies its tiles through the rest
// (identity substeps), and one that needs more sets `overflow`.
struct SubstepCount {
    const unsigned int* speed2;  // [2] float bits; nullptr = the host's count (LayerParams.dt, skip)
    unsigned int* overflow;
    float dt, cell, cap;
    int32_t k, launched;
    float water_decay[9];        // [n]: damping factor of the water layer over dt / n
};

struct ForceLaunch {
    LayerParams lay[2];
    TileFlags tf;
    SubstepCount sc;
    int32_t nxt;             // buffer being written
};

struct TransportParams {
    const float* h;
    const float* u;
    const float* v;
    float* h_out;
    const uint8_t* gate;      // nullptr = every receiver open
    const float* bank_bed;    // nullptr = no dry-bank test (banks off)
    double* ledger;           // FP64 sum of the new depth, may be nullptr
    double* cut;              // FP64 volume the dry cut removed, m^3 (accumulated), may be nullptr
    double cut_area;          // m^2 of one cell for the cut and rounding books
    double* round;            // FP64 rounding book, m^3 (accumulated), may be nullptr: each updated
                              // cell's f32 change minus the exact sum of its face fluxes
    int32_t res;
    float cell, dt, eps;
    FixedDiv div_cell;        // cell (the face fraction speed dt / cell)
    int32_t skip;
};

struct TransportLaunch {
    TransportParams lay[2];
    TileFlags tf;
    SubstepCount sc;
    int32_t nxt;
};

// TMA descriptors of a transport launch's input planes: h, u, v of each
// layer (valid where on[layer]; built by launch_transport).
struct TransportMaps {
    CUtensorMap map[2][3];
    int32_t on[2];
};

constexpr int GRID_TILE = 32;

// One window's part of a batched substep (many independent windows stepped by
// the same launches). The list kernel reads it by window (blockIdx.y); the
// force, speed and transport kernels by each list entry's window.
struct WindowSubstep {
    ForceLaunch F;            // layers, the window's tile flags, device count, buffer written
    TransportLaunch T;
    int32_t cur, all;
    int32_t skip;             // the window sits this substep out
    int32_t apply_cut;        // speed pass: cells below eps are skipped
    double* zero_ledger;      // the window's ledger sums, cleared by the list kernel
    unsigned int* zero_bits;  // the window's speed bits, cleared before substep 0's speed pass (or nullptr)
};

// Batched substep over `nwin` windows: one tile list (entries and their
// window indices), cleared count slot for the next substep.
cudaError_t launch_batch_tile_list(const WindowSubstep* d_ws, int nwin, int max_tiles, int* list, int* entry_win,
                                   int* count, int* count_next, SweepState* sweep, cudaStream_t st);
cudaError_t launch_batch_speed2(const WindowSubstep* d_ws, const int* list, const int* entry_win, const int* count,
                                cudaStream_t st);
// `sweep` non-null: some window confines by the Gauss-Seidel sweep, and the
// force pass runs as one cooperative launch (pre-sweep tiles, the sweep's
// fixed point, projection) over every window.
// `ctas_per_sm` caps the cooperative launch's CTAs per SM (at most what the
// device holds at once; 0 = that maximum); `blocks` sizes the transport's
// persistent grid (0 = four per SM). Every setting gives the same bits.
cudaError_t launch_batch_force(const WindowSubstep* d_ws, int nwin, const int* list, const int* entry_win,
                               const int* count, SweepState* sweep, cudaStream_t st, int ctas_per_sm = 0);
cudaError_t launch_batch_transport(const WindowSubstep* d_ws, const int* list, const int* entry_win,
                                   const int* count, cudaStream_t st, int blocks = 0);

size_t force_smem_bytes();
// Builds the tile list of one substep: active tiles of both layers, then the
// quiet tiles whose output buffer is not yet zero. `all` marks every tile active.
// The list's count must be zero on entry. With `count_next` the kernel zeroes
// the other count slot for the next substep (and `zero_ledger[0..1]`,
// `zero_bits[0..1]` when given), so a step needs no memset; without it the
// count is cleared by a memset first.
cudaError_t launch_tile_list(const TileFlags& tf, int cur, int nxt, int all, int skip0, int skip1,
                             const SubstepCount& sc, int* count_next, double* zero_ledger, unsigned int* zero_bits,
                             cudaStream_t st);
// Largest squared speed of each layer over the stepped tiles of the current
// tile list, which must be substep 0's (cells below eps skipped when
// apply_cut): atomicMax into bits[0..1], which start at zero.
cudaError_t launch_tile_speed2(const TileFlags& tf, const float* const h[2], const float* const u[2],
                               const float* const v[2], int res, float eps, int apply_cut, unsigned int* bits,
                               cudaStream_t st);
size_t transport_smem_bytes();
// A layer with `sweep` set runs the Gauss-Seidel form: one cooperative
// launch (every CTA resident) that computes the post-gravity velocity of
// every stepped tile, solves the raster-order sweep as a fixed point across
// tiles (grid barriers between passes, bounded waits; L.tf.sweep holds the
// barrier state), then projects, damps and clamps.
cudaError_t launch_force(const ForceLaunch& L, int res, int layers, cudaStream_t st);
cudaError_t launch_transport(const TransportLaunch& L, int res, int layers, cudaStream_t st);
// The slurry's material laws per cell: viscosity, mobility and damping rate
// from grain and moisture (dynamic_viscosity, sheet_mobility_for, sheet_damp).
cudaError_t launch_material(const uint8_t* grain, const float* moisture, float* nu, float* mob, float* damp, size_t n,
                            cudaStream_t st);
cudaError_t launch_apply_cut(const float* h, float* u, float* v, size_t n, float eps, cudaStream_t st);
cudaError_t launch_max_speed2(const float* h, const float* u, const float* v, size_t n, float eps, int apply_cut,
                              unsigned int* out_bits, cudaStream_t st);

}  // namespace silt
