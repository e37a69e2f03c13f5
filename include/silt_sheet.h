/* silt_sheet.h -- C ABI of the B200 two-layer (water + slurry) sheet step.
 *
 * Drop-in for the sheet path of x3-team/Dirty-gen's `FluidCore`
 * (src/fluid_core.rs). Each entry point names the reference interface it
 * replaces. The handle owns the device state (SoA float planes in HBM); the
 * caller owns every host buffer passed in. Seeding arrays are the values the
 * reference's closures would return, one per coarse cell, row-major j*res+i.
 *
 * Threading: one handle per CUDA stream, not thread-safe. All work is queued
 * on the handle's stream; calls that return host data synchronise it.
 *
 * Errors: the reference returns silently on dt <= 0 and similar no-ops; here
 * those return SILT_OK_NOOP. Bad pointers or sizes return SILT_EINVAL, a CUDA
 * failure SILT_ECUDA, a device wait past its limit SILT_ETIMEOUT. SILT_EBOUND
 * (from silt_sheet_sync and silt_get_ledger, and sticky) means a step needed
 * more substeps than the host's speed bound launched for it.
 */
#ifndef SILT_SHEET_H
#define SILT_SHEET_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SILT_OK 0
#define SILT_OK_NOOP 1
#define SILT_EINVAL (-1)
#define SILT_ECUDA (-2)
#define SILT_ETIMEOUT (-3)
#define SILT_ENOMEM (-4)
#define SILT_EBOUND (-5)

/* Grain codes, src/fluid_core.rs:116-124 (`Grain`). */
#define SILT_GRAIN_CLAY 0
#define SILT_GRAIN_SILT 1
#define SILT_GRAIN_SAND 2
#define SILT_GRAIN_WATER 3
#define SILT_GRAIN_OTHER 4

/* Nested 2 cm layout: 0 = one patch centred on the mean tire (the reference,
 * src/fluid_core.rs:8358), 1 = one patch per tire. */
#define SILT_FINE_MEAN_PATCH 0
#define SILT_FINE_PER_TIRE 1

typedef struct silt_sheet silt_sheet;

/* Window geometry and options. Defaults (silt_cfg_default) are the
 * reference constants: 200 cells of 0.20 m (src/fluid_core.rs:69-72), a 160
 * cell 2 cm patch (:73-76), held radius 0.56 m (:80), soft window border
 * (:9594). */
typedef struct {
    int32_t res;          /* coarse cells per side */
    float cell;           /* coarse cell, m */
    int32_t fine_res;     /* fine cells per patch side */
    float fine_cell;      /* fine cell, m; cell / fine_cell must be a whole number */
    int32_t fine_layout;  /* SILT_FINE_MEAN_PATCH or SILT_FINE_PER_TIRE */
    float tire_r;         /* held-column radius around a tire, m */
    int32_t soften_border;/* 1: slow the velocity in the window's edge band each step */
    float center_x;       /* window centre, m (FluidCore::new(center)) */
    float center_z;
    int32_t device;       /* CUDA device ordinal */
    void* stream;         /* cudaStream_t to queue on; NULL makes a private stream */
    int32_t engine;       /* SILT_ENGINE_*: how the coarse pair is stepped */
} silt_cfg;

/* Coarse-pair engines. WINDOW steps each layer box by box exactly as the
 * reference (work boxes, Gauss-Seidel confinement, per-sheet scratch), one
 * crew of CTAs per layer, windows up to 512 cells per side. GRID steps the
 * whole grid with tiled kernels on every SM, for grids of any size; it
 * confines by the reference step pair's raster-order Gauss-Seidel sweep
 * unless silt_set_confinement selects the snapshot form. AUTO picks WINDOW
 * up to 512 cells per side and GRID above. The nested patches always use WINDOW. */
#define SILT_ENGINE_AUTO 0
#define SILT_ENGINE_WINDOW 1
#define SILT_ENGINE_GRID 2

/* One tire shoving the sheet, src/fluid_core.rs:359-368 (`TirePush`). */
typedef struct {
    float x, z, forward_x, forward_z, radius, width, speed, slip;
} silt_tire_push;

/* Volume peeled off the water sheet, src/fluid_core.rs:372-382 (`SprayEvent`). */
typedef struct {
    float x, y, z, vx, vy, vz, volume;
    int32_t kind;
} silt_spray_event;

/* Volume books, src/fluid_core.rs:485-509 (`FluidLedger`), the sheet part,
 * accumulated in FP64. `opened_m3` is water added by an inflow strip. */
typedef struct {
    double water_m3, slurry_m3, frozen_water_m3, frozen_slurry_m3, spray_m3, opened_m3, total_m3;
    /* Volume the dry cut (src/fluid_core.rs:2072-2081, films under 1e-6 m)
     * has removed since creation; not in total_m3, which keeps the
     * reference's books. total_m3 + cut_m3 - opened_m3 is conserved. */
    double cut_m3;
    /* The river reach's bank (FluidLedger::reach_m3, :6863), in total_m3. */
    double reach_m3;
    /* Volume the f32 transport updates created (+) or removed (-) by
     * rounding since creation: each updated cell's f32 depth change less the
     * exact (FP64) sum of the fluxes across its faces, summed in FP64. The
     * state is the reference's f32 arithmetic, so this is the part of the
     * books' per-step gap its transport explains; not in total_m3.
     * total_m3 + cut_m3 - opened_m3 - round_m3 is conserved but for the
     * rounding of the other f32 updates (coupling, seeding). */
    double round_m3;
    /* The tracers' books (FluidLedger's suspended part, src/fluid_core.rs:
     * 496-505, and the silt book, :6171-6195), FP64: suspended solids in the
     * water column, settled out of it, parked off the window, and lifted into
     * suspension in all (wheel wakes, a river reach's inlet load); stirred silt
     * in the column, settled, parked, and stirred in all. The reference adds
     * the suspended account to its total; total_m3 here keeps the water and
     * slurry books only, so it closes without them (the lifted solids come
     * from the bed, not from the water). Each account closes on its own:
     * suspended + settled + parked = entrained, and the same for the silt. */
    double suspended_m3, settled_suspended_m3, frozen_suspended_m3, entrained_m3;
    double turbid_m3, turbid_settled_m3, frozen_turbid_m3, stirred_m3;
} silt_ledger;

/* src/fluid_core.rs:289-320 (`RiverReach`); with turbidity on, the inlet's
 * water arrives carrying inlet_turbidity of its column as suspended solids. */
typedef struct {
    int32_t along_z, positive;
    float cross0, cross1;
    int32_t rows;
    float inlet_eta, outlet_eta, inlet_speed_m_s, inlet_turbidity;
} silt_river_reach;

/* src/fluid_core.rs:274-287 (`WaveMaker`). */
typedef struct {
    float x0, x1, z0, z1, dir_x, dir_z, amplitude_m_s, period_s, ramp_s;
} silt_wave_maker;

/* src/fluid_core.rs:213-240 (`HydroSolid`): a wheel's or a belly panel's
 * footprint, a wall in the sheet wherever the free surface stands above
 * bottom_y (and the bed below top_y). yaw 0 points the long axis along +Z.
 * contact != 0 marks a tire contact (drawn over walls). radius and width
 * (the cylinder of a wheel) are kept for the caller; the sheet uses the box. */
typedef struct {
    float x, z, yaw, half_length, half_width, bottom_y, top_y;
    int32_t contact;
    float radius, width;
} silt_hydro_solid;

/* src/fluid_core.rs:242-255 (`HydroLoad`): what the walls feel, read back
 * after a step. */
typedef struct {
    float force_x, force_z;   /* N: hydrostatic plus dynamic pressure on the wall faces */
    float buoyancy_n, hull_buoyancy_n, wheel_buoyancy_n;
    float displaced_m3;
    float eroded_m3;          /* bed scoured beside tire contacts since creation */
    float hole_m;             /* the deepest scour */
    uint32_t wheel_blocks, belly_blocks;  /* contact and wall cells of the coarse mask */
} silt_hydro_load;

/* src/fluid_core.rs:440-448 (`GroundSample`); settled dust is off this path (0). */
typedef struct {
    float water_m, slurry_m, u, v, settled_dust_m, moisture, bed_m;
} silt_ground_sample;

/* src/fluid_core.rs:452-465 (`CoarseCell`), sheet fields. */
typedef struct {
    float x, z, bed_m, water_m, slurry_m, moisture, u, v;
    float turbidity;  /* suspended load plus stirred silt over the water column, 0..1 */
} silt_coarse_cell;

/* -------------------------------------------------------------- lifecycle */
void silt_cfg_default(silt_cfg* cfg);
/* FluidCore::new (src/fluid_core.rs:4958). */
int silt_sheet_create(const silt_cfg* cfg, silt_sheet** out);
int silt_sheet_destroy(silt_sheet* s);
/* Waits for all queued work. */
int silt_sheet_sync(silt_sheet* s);
/* Last CUDA error string for this thread ("" when none). */
const char* silt_last_error(void);

/* ---------------------------------------------------------------- seeding */
/* FluidCore::map_water_bed (src/fluid_core.rs:5329); vol_out may be NULL. */
int silt_map_water_bed(silt_sheet* s, const float* bed, const float* water, float* vol_out);
/* FluidCore::map_grain (src/fluid_core.rs:5318). */
int silt_map_grain(silt_sheet* s, const uint8_t* grain);
/* FluidCore::map_water_velocity (src/fluid_core.rs:5358). */
int silt_map_water_velocity(silt_sheet* s, const float* u, const float* v);
/* FluidCore::pour_water / pour_slurry (src/fluid_core.rs:5424, :5428). */
int silt_pour_water(silt_sheet* s, float x0, float x1, float z0, float z1, float depth, float* vol_out);
int silt_pour_slurry(silt_sheet* s, float x0, float x1, float z0, float z1, float depth, int32_t grain,
                     float moisture, float* vol_out);
/* FluidCore::lay_slurry_mask (src/fluid_core.rs:5857). */
int silt_lay_slurry_mask(silt_sheet* s, const float* depth, int32_t grain, float moisture, float* vol_out);
/* FluidCore::lay_slurry_on_water (src/fluid_core.rs:5236-5254): the slurry
 * depth becomes `depth` on every cell holding more than 12 mm of water (grain
 * `grain`, moisture at least 0.90); *vol_out gets depth * cell area summed
 * over those cells as the reference's f32 running sum. Synchronises. */
int silt_lay_slurry_on_water(silt_sheet* s, float depth, int32_t grain, float* vol_out);
/* FluidCore::read_substrate_grid (src/fluid_core.rs:5928). */
int silt_read_substrate_grid(silt_sheet* s, const float* bed, const float* moisture, const uint8_t* grain);
/* Inflow strip on coarse row j over world x in [x0, x1), rate m^3/s; rate 0 turns it off.
 * No reference counterpart (the reference has no inflow source); booked as opened_m3. */
int silt_set_inflow(silt_sheet* s, int32_t j, float x0, float x1, float rate_m3_s);

/* --------------------------------------------------------------- per step */
/* FluidCore::push_tire (src/fluid_core.rs:5964). */
int silt_push_tire(silt_sheet* s, const silt_tire_push* push);
/* FluidCore::step (src/fluid_core.rs:6034), sheet path. Writes up to `cap`
 * spray events to `out` (may be NULL when cap is 0) and the total count to
 * n_out (may be NULL). Synchronises only when events are requested. */
int silt_step(silt_sheet* s, float dt, silt_spray_event* out, int32_t cap, int32_t* n_out);

/* ------------------------------------------------------------------ reads */
/* FluidCore::ledger (src/fluid_core.rs:6821), FP64. */
int silt_get_ledger(silt_sheet* s, silt_ledger* out);
/* FluidCore::coarse_cell (src/fluid_core.rs:6998). Returns SILT_OK_NOOP outside the window. */
int silt_get_coarse_cell(silt_sheet* s, int32_t i, int32_t j, silt_coarse_cell* out);
/* FluidCore::export_maps (src/fluid_core.rs:6941): height, vel_u, vel_v, moisture (res*res each; any may be NULL). */
int silt_export_maps(silt_sheet* s, float* height, float* vel_u, float* vel_v, float* moisture);
/* render_contract::publish_with_snow film/flow (src/render_contract.rs:483-496):
 * film = (water, slurry) per cell, flow = (vx, vz, speed, turbidity), the
 * turbidity from the tracers' suspended load and stirred silt. Host pointers. */
int silt_publish_film_flow(silt_sheet* s, float* film, float* flow);
/* Same maps into device memory the caller owns (2*res*res and 4*res*res floats). */
int silt_publish_film_flow_device(silt_sheet* s, float* d_film, float* d_flow);
/* FluidCore::non_finite_count (src/fluid_core.rs:5374), sheet planes. */
int silt_non_finite_count(silt_sheet* s, uint32_t* out);
/* FluidCore::spray_m3 (src/fluid_core.rs:6817). */
int silt_spray_m3(silt_sheet* s, double* out);
/* FluidCore::sample (src/fluid_core.rs:6806-6813, sample_coarse :9428-9454)
 * between steps (the patches are handed back): the coarse cell under (x, z);
 * SILT_OK_NOOP and zeros outside the window. */
int silt_sample(silt_sheet* s, float x, float z, silt_ground_sample* out);
/* FluidCore::recenter (src/fluid_core.rs:5409-5421): moves the window to
 * the one centred on (cx, cz). Cells that slide off are parked (in a device
 * table keyed by world cell, booked as frozen volume), cells that slide on
 * are restored; bed and grain stay on their index (the caller re-reads the
 * substrate). A whole-cell move scrolls (shift_coarse_scroll :9024), any
 * other jump re-keys every cell (shift_coarse_hash :9147). Near-field tiles
 * follow their cells; tiles leaving the window are released. */
int silt_recenter(silt_sheet* s, float cx, float cz);
/* FluidCore::set_center (src/fluid_core.rs:5403): track the chase point
 * without sliding the window. */
int silt_set_center(silt_sheet* s, float cx, float cz);
/* FluidCore::window_bounds (src/fluid_core.rs:6977): origin x, origin z, extent. */
int silt_window_bounds(silt_sheet* s, float* ox, float* oz, float* extent);
/* FluidCore::window_origin (src/fluid_core.rs:6987-6990): the minimum corner
 * of a res x res window of `cell` around the centre, snapped like
 * silt_sheet_create (snap_origin :9877-9892). Host only. */
int silt_window_origin(float center_x, float center_z, int32_t res, float cell, float* origin2);
/* Raw plane copy to host for tests and tools: which = 0 water, 1 slurry, 2 uw,
 * 3 vw, 4 us, 5 vs, 6 bed, 7 moisture, 8 foam, 9 stirred silt (m), 10
 * suspended solids (m). */
int silt_read_plane(silt_sheet* s, int32_t which, float* host);
int silt_write_plane(silt_sheet* s, int32_t which, const float* host);
/* Device pointer of plane `which` (same indices) in the handle's current
 * buffers, valid until the next step or write; the caller orders its reads
 * after the handle's stream. */
int silt_plane_device(silt_sheet* s, int32_t which, void** out);
/* Device-to-device copy of src's window state (depths, velocities, bed,
 * moisture, grain) into dst (same size and device); dst's nested patches and
 * near field are untouched. Used to step one state two ways. */
int silt_sheet_copy_state(silt_sheet* dst, silt_sheet* src);
/* Diagnostic of the grid engine's division by a fixed divisor d > 0 (x times
 * the rounded reciprocal, refined once by the FMA remainder): counts of float
 * x, over all 2^32 bit patterns, whose result differs from IEEE x / d, written
 * to the host array counts6: [0] all, [1] x zero, [2] x subnormal, [3] x
 * infinite or NaN, [4] a subnormal or zero IEEE quotient, [5] the rest. The
 * engine divides by the product only for divisors whose [0] is 0 (checked
 * once per divisor at silt_sheet_create). No counterpart in the reference,
 * which divides by IEEE division throughout. Synchronises `stream`. */
int silt_check_fixed_division(float d, unsigned long long* counts6, void* stream);
/* The divisors the library treats as checked without running the check:
 * 2 cell, cell^2, 231 and cell for the standard cells of 0.2 m and 0.02 m,
 * as the float products the step forms. The check's verdict depends only on
 * IEEE single-precision arithmetic, not on the GPU; every other divisor is
 * checked once per process and device. Writes up to cap values to out and
 * returns how many there are (no device work). */
int silt_known_exact_divisors(float* out, int32_t cap);
/* FluidCore::fine_water_debug (src/fluid_core/near.rs:341): lays the patch
 * down for these tires, copies patch `patch` (fine_res^2 floats) and its
 * origin, and packs it back. */
int silt_fine_water_debug(silt_sheet* s, const silt_tire_push* tires, int32_t n, int32_t patch, float* host,
                          float* origin2);
/* FluidCore::near_tiles (src/fluid_core/near.rs:328). */
int silt_near_tiles(silt_sheet* s, int32_t* out);

/* Device time per kernel family since timing was last switched on, measured
 * with CUDA events on the handle's stream. The GPU counterpart of
 * FluidCore::step_parts (src/fluid_core.rs:4782-4795, :6130). `launches`
 * counts this library's kernel launches (always counted); `force_cells` the
 * cell-layers the force kernel stepped (the grid engine's active tiles, or
 * every window cell on the window engine), `force_cells_water` the water
 * layer's share. */
typedef struct {
    double force_ms, transport_ms, fine_ms;
    int64_t steps, launches, force_launches, force_cells, force_cells_water;
    int64_t device_counts;  /* steps whose substep count the device decided */
    double host_step_ms, host_fine_ms;  /* host time inside silt_step, and its nested-patch share */
    /* Grid engine, Gauss-Seidel sweep: launches, the most fixed-point passes
     * one launch needed, launches that reached the pass limit and ran the
     * sequential sweep, tile solves (a tile in one pass) and their local
     * passes in shared memory. */
    int64_t sweep_launches, sweep_passes_max, sweep_fallbacks, sweep_solves, sweep_local_passes;
    /* Host time per phase of a step (ms, summed over the steps; with step
     * timing on): [0] closure crops and wake entrainment, [1] per-window
     * planning on a batch's workers, [2] the nested patches (a single sheet:
     * their planning and launches, with the inflow), [3] the coarse pair and
     * open-water drivers, [4] the patches' peel (and scour), [5] tracers and
     * reach, [6] the closure's correction, spray and the books. */
    double host_phase_ms[8];
} silt_step_parts;
int silt_set_step_timing(silt_sheet* s, int32_t on);
int silt_get_step_parts(silt_sheet* s, silt_step_parts* out);

/* Device time of every kernel this library launches, from any handle or
 * thread, while on: each launch is bracketed by two CUDA events on its own
 * stream (which costs the overlap of back-to-back launches, so time a pass of
 * its own). on = 1 clears earlier totals. silt_get_kernel_times waits for the
 * device and writes up to cap rows, largest total first; *n_out is the
 * number of kernels seen. A GPU counterpart of the reference's per-part step
 * timing (FluidCore::step_parts, src/fluid_core.rs:4782-4795), by kernel. */
typedef struct {
    char name[96];     /* qualified kernel name, no argument list */
    int64_t launches;
    double ms;         /* summed device time */
} silt_kernel_time;
int silt_set_kernel_timing(int32_t on);
int silt_get_kernel_times(silt_kernel_time* out, int32_t cap, int32_t* n_out);

/* ------------------------------------------------------- batched windows */
/* Many independent windows stepped together (vehicles or scenes, each its own
 * FluidCore in the reference, which steps them one after another). A batch
 * groups sheets created with SILT_ENGINE_GRID on one device and one stream;
 * each keeps its own state, seeding, tires, ledger and reads through the
 * calls above. silt_batch_step(b, dt) equals silt_step(s, dt) on every sheet
 * (same kernels and arithmetic), except that spray events are not returned
 * (their volume still goes to each sheet's books): the nested patches and
 * inflow run per sheet, then every window's coarse pair advances through one
 * tile list and one launch of each grid kernel per substep. */
typedef struct silt_batch silt_batch;
int silt_batch_create(silt_sheet* const* sheets, int32_t n, silt_batch** out);
int silt_batch_destroy(silt_batch* b);
int silt_batch_step(silt_batch* b, float dt);
/* silt_push_tire for many windows at once: pushes[k] goes to the window at
 * batch index windows[k] (in call order within each window). */
int silt_batch_push_tires(silt_batch* b, const int32_t* windows, const silt_tire_push* pushes, int32_t n);
/* Every window's ledger (out: one per window, in batch order) with one copy
 * back and one wait, as silt_get_ledger gives them one at a time. */
int silt_batch_get_ledgers(silt_batch* b, silt_ledger* out);
/* Device time of the batched force and transport launches, tiles stepped,
 * launches and host time, as silt_get_step_parts reports for one sheet. */
int silt_batch_set_timing(silt_batch* b, int32_t on);
int silt_batch_get_parts(silt_batch* b, silt_step_parts* out);
/* The batch's launch settings, picked by timed trials. No counterpart in the
 * reference, which steps its windows one after another. Every setting gives
 * the same bits, so the autotuner times ordinary steps: after six untimed
 * steps it varies one setting at a time (coordinate descent), runs each
 * candidate for two steps, keeps the faster candidate's best time, fixes the
 * best candidate before the next setting, and stops after 16 timed steps.
 * The choice is kept for the process per device and size class (window
 * count and coarse cells), and appended to the file named by the
 * environment variable SILT_TUNE_CACHE when set (read at the first tuning);
 * a later batch of the same class takes it without trials. */
typedef struct {
    int32_t sweep_ctas_per_sm;  /* CTAs per SM of the batched Gauss-Seidel launch (1 or 2) */
    int32_t transport_blocks;   /* blocks of the batched transport's persistent grid */
    int32_t tracer_blocks;      /* blocks of a tracer pass over all the windows */
    int32_t tuned;              /* 1: chosen by trials or taken from the cache; 0: defaults or set */
    int32_t trials;             /* candidates timed */
    float trial_ms[16];         /* each candidate's best step time (device, ms), in trial order */
} silt_batch_tune;
/* on != 0 starts the trials with the next steps (or takes a cached choice);
 * 0 stops them and keeps the settings in force. */
int silt_batch_autotune(silt_batch* b, int32_t on);
int silt_batch_get_tune(silt_batch* b, silt_batch_tune* out);
/* Sets the three settings directly (0 keeps a setting's default). */
int silt_batch_set_tune(silt_batch* b, const silt_batch_tune* in);

/* ------------------------------------------------------------------ knobs */
/* FluidCore::set_fine_sub_cap / set_fine_pace (src/fluid_core.rs:5072, :5085). */
int silt_set_fine_sub_cap(silt_sheet* s, float cap);
int silt_set_fine_pace(silt_sheet* s, int32_t pace);
/* FluidCore::set_near_field (src/fluid_core/near.rs:332). */
int silt_set_near_field(silt_sheet* s, int32_t on);
/* Vorticity confinement of the grid engine's coarse pair. SWEEP (default) is
 * the reference step pair's form: step_pair runs its sheets' inner loops
 * serially, so force_gravity_open (src/fluid_core.rs:2234-2260) confines in a
 * raster-order Gauss-Seidel sweep; the grid engine solves that sweep as a
 * fixed point across tiles and gives its result bit for bit. SNAPSHOT is the
 * Jacobi form of force_gravity_par (:2263), which the reference takes for
 * boxes of at least 48 x 32 outside a step pair. The window engine always
 * sweeps as the reference does; this knob does not change it. */
#define SILT_CONFINE_SWEEP 0
#define SILT_CONFINE_SNAPSHOT 1
int silt_set_confinement(silt_sheet* s, int32_t form);
/* FluidCore::set_open_water (src/fluid_core.rs:5293-5303; on = 0 is None):
 * the water sheet runs at `mobility` (clamped to [0, 1]) with Manning bed
 * friction `manning_n` and eddy viscosity `eddy_m2_s` (m^2/s) after each
 * coarse pair (bed_friction / eddy_shear, :7485-7581). */
int silt_set_open_water(silt_sheet* s, int32_t on, float mobility, float manning_n, float eddy_m2_s);
/* FluidCore::set_surface_diffusion (src/fluid_core.rs:5284-5286, applied by
 * diffuse_surface :7584-7636), m^2/s; 0 is off. */
int silt_set_surface_diffusion(silt_sheet* s, float m2_s);
/* FluidCore::set_river_reach (src/fluid_core.rs:5273-5275; NULL is None):
 * an inlet and an outlet at the window ends (feed_reach :7638-7745, after the
 * coarse pair) and a border band that lets the current through (:8018-8033). */
int silt_set_river_reach(silt_sheet* s, const silt_river_reach* reach);
/* FluidCore::set_wave_maker (src/fluid_core.rs:5306-5309; NULL is None):
 * a paddle strip (drive_waves :7420-7480, before the coarse pair); restarts
 * the paddle clock. */
int silt_set_wave_maker(silt_sheet* s, const silt_wave_maker* wave);
/* FluidCore::set_turbidity_enabled (src/fluid_core.rs:5097; on by default,
 * :4994): the tires' wake lifts solids into suspension, which the sheet
 * carries and settles (step_suspended :8750). Foam and stirred silt
 * (step_tracers :6210) run either way. */
int silt_set_turbidity_enabled(silt_sheet* s, int32_t on);
/* FluidCore::set_hydro_solids (src/fluid_core.rs:5257-5260): the walls of the
 * next steps (n = 0 removes them). Each step builds the wall mask of the
 * coarse window and of every tire patch from the water over its bed
 * (:7288-7360 solid_mask), pushes covered columns to their open neighbours
 * (:4382 displace_occupied) and steps the walled sheet (:1879-2082 with
 * `solid`): lifted surface, no-slip ghosts, the Gauss-Seidel gravity sweep
 * with the wall mobility, redirect and block at the walls, walled transport.
 * Up to 64 bodies; the window engine only (SILT_EINVAL on the grid engine). */
int silt_set_hydro_solids(silt_sheet* s, const silt_hydro_solid* solids, int32_t n);
/* FluidCore::hydro_load (src/fluid_core.rs:7164-7249): the coarse mask of the
 * current state, the hydrostatic (rho g h^2 / 2 per face metre) and dynamic
 * (rho vn^2 h / 2) force on every open wet cell's wall faces, and each body's
 * buoyancy from the mean surface of its wet ring (:7251-7286; a wheel's
 * submerged circular segment, a belly's box at 0.36 fill). The reference's
 * f32 running sums are FP64 sums here. Synchronises the handle's stream.
 * With walls the step also scours (scour_contacts :7364-7420): shear above
 * 1.5 Pa beside a contact cuts up to 8 cm of bed per cell into the slurry as
 * silt; the ledger books that volume in opened_m3. */
int silt_get_hydro_load(silt_sheet* s, silt_hydro_load* out);

/* ------------------------------------------------------ one-sheet operator */
/* Free `step_sheet` (src/fluid_core.rs:770) with the gravity drive on caller
 * device arrays (res*res each): h, u, v updated in place; bed, nu, gate read.
 * `scratch` is device memory of silt_step_sheet_scratch_bytes(res) bytes the
 * caller allocates once and passes to every call (zeroed before the first):
 * it plays the reference's per-thread sheet scratch, whose contents one call
 * leaves for the next. Up to 512 cells per side the window engine steps the
 * sheet exactly as the reference; above, the grid engine. stream is a
 * cudaStream_t (NULL = legacy stream). */
size_t silt_step_sheet_scratch_bytes(int32_t res);
int silt_step_sheet(float* h, float* u, float* v, const float* bed, const float* nu, const uint8_t* gate,
                    int32_t res, float cell, float dt, float vorticity, void* scratch, void* stream);

/* The same operator for callers that cannot allocate GPU memory. No
 * counterpart in the reference: it exists for code on a fixed-budget frame
 * loop (a game or simulation tick) where cudaMalloc/cudaFree may not run,
 * since cudaFree waits for the whole device and an allocation can stall or
 * fail mid-frame, and for hosts whose GPU memory is all owned by another
 * allocator. Its scratch is a fixed array compiled into the library, sized
 * for grids up to SILT_STEP_SHEET_STATIC_MAX_RES cells per side (4 MiB per
 * GPU that loads the library, held until the process exits); larger grids
 * return SILT_EINVAL. The first call on each device does a one-time set-up:
 * with that device current it looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it for the rest of the process, so make
 * that first call before any stream capture begins. After cudaDeviceReset
 * the kept address is stale: do not call this entry point on a device that
 * was reset. The array keeps what the last call left in it, as the
 * reference's per-thread sheet scratch does.
 * Every call shares the one array: calls whose work overlaps on the GPU race
 * and must be ordered by the caller (one stream, or events). Calls no
 * cudaMalloc, cudaFree or other allocating routine. */
#define SILT_STEP_SHEET_STATIC_MAX_RES 256
int silt_step_sheet_noalloc(float* h, float* u, float* v, const float* bed, const float* nu, const uint8_t* gate,
                            int32_t res, float cell, float dt, float vorticity, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SILT_SHEET_H */
