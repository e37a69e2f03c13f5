// TEST INFRASTRUCTURE ONLY. CPU restatement of the reference's sheet step
// (x3-team/Dirty-gen "Silt", src/fluid_core.rs and src/fluid_core/near.rs),
// used as the parity checker for the CUDA path and as the timed CPU
// baseline. Nothing in the product links or calls this code.
//
// Parity pinning: the reference is Rust and no Rust toolchain exists on this
// machine, so this restatement is pinned by re-running the reference's own
// unit tests (restated under tests/) against it; see tests/test_oracle_*.py.
//
// Arithmetic follows the reference exactly: f32 everywhere, the same
// evaluation order, no FMA contraction (build with -ffp-contract=off) and
// glibc expf/powf/hypotf, which is what Rust's f32::exp/powf/hypot call.
#pragma once
#include <cstddef>
#include <cstdint>

extern "C" {

// ---- free one-sheet operator (src/fluid_core.rs:770 `step_sheet`) -------------
// A scratch handle stands in for the reference's thread-local SCRATCH
// (src/fluid_core.rs:581-589): repeated calls on one handle see the scratch
// contents the previous call left, as the reference's calls on one thread do.
void* oracle_scratch_new(void);
void oracle_scratch_free(void* sc);

// Full step_sheet_eps (src/fluid_core.rs:856) on caller arrays, res*res each.
// inner_par = 1 is the free operator outside a two-sheet pair (row splits
// allowed, Jacobi confinement on big boxes); 0 is inside `step_pair`.
void oracle_step_sheet(float* h, float* u, float* v, const float* bed, const float* nu,
                       const uint8_t* gate, int res, float cell, float dt, float vorticity,
                       float eps, int banks, float sub_cap, int pace, int inner_par, void* sc);

// transport_open_rows_body / transport_open_ref (src/fluid_core.rs:3025, :3140)
// on one box; `serial` selects the serial edge-loop definition. removed/added
// receive the scratch sums.
void oracle_transport_open(float* h, const float* vel, const uint8_t* gate, int res,
                           float cell, float dt, int i0, int i1, int j0, int j1, int along_x,
                           const float* bed, float frac_cap, int serial, float* removed,
                           float* added);

// sheet_work_boxes (src/fluid_core.rs:1325); out holds 4*cap ints (i0,i1,j0,j1).
// flood = 1 runs the test-only flood-fill definition (src/fluid_core.rs:11134).
int oracle_sheet_work_boxes(const float* h, int res, float eps, int allow_split, int flood,
                            int* out, int cap);
// awake_work_boxes (src/fluid_core.rs:1537).
int oracle_awake_work_boxes(const float* h, const float* u, const float* v, const float* bed,
                            int res, float cell, float eps, int* out, int cap);

float oracle_dynamic_viscosity(int grain, float moisture);
float oracle_sheet_mobility_for(float nu);
float oracle_sheet_damp(float nu);
void oracle_soften_border(float* u, float* v, int res);

// rut_heal (src/fluid_core.rs:4673): out = level_s, relief0, relief_8s, still_deep.
void oracle_rut_heal(int grain, float moisture, float* out4);

// ---- window core (FluidCore subset on the sheet path) ---------------------------
typedef struct {
    int res;           // coarse cells per side (reference: 200)
    float cell;        // coarse cell, m (reference: 0.20)
    int fine_res;      // fine cells per patch side (reference: 160)
    float fine_cell;   // fine cell, m (reference: 0.02)
    int layout;        // 0: one patch at the mean tire (reference); 1: one patch per tire
    float tire_r;      // held-column radius around a tire, m (reference: 0.56)
    int soften;        // 1: soften_border on the coarse velocity (reference: 1)
    int inner_par;     // 0: coarse pair runs serial inner loops (reference step_pair)
    float center_x, center_z;
    int threads;       // >1: each sheet of a pair on its own thread (the reference's rayon::join)
} oracle_core_cfg;

typedef struct {
    float x, z, forward_x, forward_z, radius, width, speed, slip;
} oracle_tire;

typedef struct {
    float x, y, z, vx, vy, vz, volume;
    int kind;
} oracle_spray;

void* oracle_core_new(const oracle_core_cfg* cfg);
void oracle_core_free(void* core);
float oracle_core_map_water_bed(void* core, const float* bed, const float* water);
void oracle_core_map_grain(void* core, const uint8_t* grain);
void oracle_core_map_water_velocity(void* core, const float* u, const float* v);
float oracle_core_pour(void* core, float x0, float x1, float z0, float z1, float depth,
                       int water, int grain, float moisture);
float oracle_core_lay_slurry_mask(void* core, const float* depth, int grain, float moisture);
void oracle_core_read_substrate(void* core, const float* bed, const float* moisture,
                                const uint8_t* grain);
void oracle_core_push_tire(void* core, const oracle_tire* t);
int oracle_core_step(void* core, float dt, oracle_spray* out, int cap);
// out[0..4]: water_m3, slurry_m3, frozen_water_m3, frozen_slurry_m3, spray_m3,
// in f32 as the reference sums them; out64[0..2]: water, slurry in f64.
void oracle_core_ledger(void* core, float* out5, double* out64_2);
// which: 0 water 1 slurry 2 uw 3 vw 4 us 5 vs 6 bed 7 moisture 8 foam 9 turbid
// (stirred silt) 10 susp (suspended solids); dst res*res floats.
void oracle_core_get(void* core, int which, float* dst);
void oracle_core_set(void* core, int which, const float* src);
void oracle_core_get_grain(void* core, uint8_t* dst);
void oracle_core_publish(void* core, float* film, float* flow);
void oracle_core_set_fine_pace(void* core, int pace);
void oracle_core_set_turbidity(void* core, int on);
void oracle_core_set_reach_turbidity(void* core, float inlet_turbidity);
void oracle_core_tracer_books(void* core, float* out8, double* out64_8);
void oracle_core_set_fine_sub_cap(void* core, float cap);
void oracle_core_set_near_field(void* core, int on);
int oracle_core_near_tiles(void* core);
float oracle_core_spray_m3(void* core);
uint32_t oracle_core_non_finite(void* core);
void oracle_core_sample(void* core, float x, float z, float* out7);
// Lays the fine patch down for these tires, copies patch k's water to dst
// (fine_res^2 floats), reads its origin, and packs it back (near.rs:341).
void oracle_core_fine_water_debug(void* core, const oracle_tire* tires, int n, int patch,
                                  float* dst, float* origin2);
void oracle_core_inflow(void* core, int j, float x0, float x1, float depth);
}
