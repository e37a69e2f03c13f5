// Host runtime of the B200 sheet step: the `silt_*` C ABI (include/silt_sheet.h).
//
// A handle owns the device state of one window: ping-pong SoA planes for the
// water and slurry depth and velocity, the bed, moisture and grain, the
// nested 2 cm patches, and small device accumulators. Every call queues work
// on the handle's stream; only calls that return host data synchronise.
//
// Step order follows FluidCore::step (x3-team/Dirty-gen src/fluid_core.rs:6034),
// sheet subset: inflow, refine (restrict, lay the patches, near field), tire
// shove on the patches, fine pair, fine spray, restrict, shove outside the
// patches, coarse pair, coarse spray.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <condition_variable>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/silt_sheet.h"
#include "../../include/silt_closure.h"
#include "closure.cuh"
#include "sheet_drivers.cuh"
#include "sheet_fine.cuh"
#include "launch_count.cuh"
#include "sheet_grid.cuh"
#include "sheet_host_math.h"
#include "sheet_ops.cuh"
#include "sheet_walls.cuh"
#include "sheet_park.cuh"
#include "sheet_tracers.cuh"
#include "sheet_window.cuh"

namespace {

thread_local char g_err[256] = "";

int fail_cuda(cudaError_t e, const char* what) {
    snprintf(g_err, sizeof g_err, "%s: %s", what, cudaGetErrorString(e));
    return SILT_ECUDA;
}
int fail_arg(const char* what) {
    snprintf(g_err, sizeof g_err, "invalid argument: %s", what);
    return SILT_EINVAL;
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return fail_cuda(e_, #call);   \
    } while (0)

struct DevicePlane {
    void* p = nullptr;
    ~DevicePlane() {
        if (p) cudaFree(p);
    }
};

}  // namespace

using silt::fine::Patches;

struct silt_sheet {
    silt_cfg cfg;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    int res = 0;
    size_t n = 0;
    float origin[2] = {0, 0};
    // [layer][buffer]: layer 0 water, 1 slurry.
    float* h[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    float* u[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    float* v[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int cur = 0;
    float* bed = nullptr;
    float* moisture = nullptr;
    uint8_t* grain = nullptr;
    float* mat = nullptr;         // slurry material per cell: viscosity, mobility, damping rate (3 planes)
    bool mat_dirty = true;        // grain or moisture changed since the planes were computed
    float* staging = nullptr;     // n floats for host uploads
    float* staging2 = nullptr;
    uint8_t* staging_u8 = nullptr;
    double* d_acc = nullptr;      // [0..1] step ledger sums, [2..3] reductions, [4..7] spare
    unsigned int* d_u32 = nullptr;   // [0..1] speed bits, [2] substep overflow, [3] non-finite count, [4..7] tile counters
    const float** d_planes = nullptr;
    double* h_acc = nullptr;      // pinned mirror of d_acc
    double* d_sum_scratch = nullptr;  // the ordered plane sums' partials (SUM_SCRATCH_BYTES)
    // d_u32: [0, 2) speed bits, [2] substep overflow, [4, 8) tiles stepped
    // (two u64), [SWEEP_AT, SWEEP_AT + 11) the sweep launch state, [COUNT_AT]
    // a seeding call's cell count.
    static constexpr int SWEEP_AT = 8;
    static constexpr int COUNT_AT = 20;
    static_assert(SWEEP_AT + sizeof(silt::SweepState) / sizeof(unsigned int) <= COUNT_AT, "d_u32 slots");
    unsigned int* h_flags = nullptr;  // pinned: d_u32[2, 16) as last read (FLAG_* below)
    bool cut_pending = false;
    bool ledger_fresh = false;    // h_acc[0..1] hold the current depth sums
    float vmax_bound = 0.0f;      // bound on any cell's speed |(u, v)|, for the one-substep shortcut
    float moisture_ambient = 0.0f;
    std::vector<silt_tire_push> pushes;
    double opened_m3 = 0.0;
    int inflow_j = -1, inflow_i0 = 0, inflow_i1 = 0;
    float inflow_rate = 0.0f;
    Patches fine;
    // Step timing (silt_set_step_timing): event triples around force/transport.
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<cudaEvent_t> ev_used;   // groups of three: start, after force, after transport
    // The step's divisors (2 cell, cell^2, 231, cell), set at creation; each
    // is exact only once checked against IEEE division for every float.
    silt::CellDivisors div{};
    silt_step_parts parts;
    // Window engine for the coarse pair (SILT_ENGINE_WINDOW).
    int engine = SILT_ENGINE_GRID;
    float* win_planes = nullptr;                  // 2 layers x SCRATCH_PLANES x n
    static constexpr int WIN_SLOTS = 4;           // a slot is reused 4 steps later: the host runs ahead
    silt::window::Job* d_win_jobs = nullptr;      // WIN_SLOTS slots x 2 layers
    silt::window::Job* h_win_jobs = nullptr;      // pinned staging
    cudaEvent_t win_ev[WIN_SLOTS] = {};
    int win_flip = 0;
    // Walls (silt_set_hydro_solids): the bodies in two device slots, each
    // filled from its pinned half once the copy two updates ago is done.
    int n_solids = 0;
    silt::walls::SolidGeom* d_solids = nullptr;  // 2 x MAX_SOLIDS
    silt::walls::SolidGeom* h_solids = nullptr;  // pinned, 2 x MAX_SOLIDS
    cudaEvent_t solid_ev[2] = {nullptr, nullptr};
    int solid_slot = 0;
    uint8_t* d_wall_mask = nullptr;  // the coarse window's mask (res^2)
    std::vector<silt_hydro_solid> solids;        // as set, for the buoyancy read-back
    float* d_bed_drop = nullptr;                 // scour depth per coarse cell (res^2)
    double* d_wall_out = nullptr;                // hydro_load sums: 4 + 3 x MAX_SOLIDS
    unsigned int* d_hole_bits = nullptr;         // the deepest scour (float bits)
    // Grid engine: active-tile flags and the substep's tile list.
    silt::TileFlags tf;
    uint8_t* tile_mem = nullptr;
    int* tile_count = nullptr;   // two count slots, used alternately by successive substeps
    unsigned long long tile_seq = 0;
    bool tiles_all = true;     // next substep steps every tile (after any outside write)
    // Confinement form of the grid engine (silt_set_confinement): the
    // reference step pair's Gauss-Seidel sweep by default, solved in the
    // iterate planes (2 layers x u, v) with the launch state in d_u32.
    int confine = SILT_CONFINE_SWEEP;
    float* sweep_planes = nullptr;
    unsigned int* sweep_stamp = nullptr;  // the sweep's per-tile change stamps (2 layers)
    silt::SweepState* sweep_state() { return reinterpret_cast<silt::SweepState*>(d_u32 + SWEEP_AT); }

    // Open-water mode of the water sheet (FluidCore::set_open_water,
    // src/fluid_core.rs:5293-5303) and the surface diffusion (:5284-5286).
    bool open_water = false;
    float ow_mobility = 0.0f, ow_manning = 0.0f, ow_eddy = 0.0f;
    float surface_diffusion = 0.0f;
    float* ow_scratch = nullptr;   // 2 n floats for the drivers' snapshots
    // FluidCore::set_turbidity_enabled (src/fluid_core.rs:5097, on by
    // default :4994): the wake's suspended load and its transport.
    bool turbidity = true;
    // The tracers on the coarse window: foam, stirred silt, suspended solids.
    void* tr_mem = nullptr;
    silt::tracers::Planes tr;
    silt::tracers::Runner tr_run;
    bool tr_rescan = true;  // the tracer planes were rewritten (attach, move): scan the silt span once
    // What the host knows of the tracers' idleness from the device's reports
    // (silt::tracers::step_suspended), so that silt_step can skip tracer
    // steps that would change nothing.
    struct TracerIdle {
        static constexpr int SLOTS = 8;
        unsigned int* d_flag = nullptr;   // SLOTS report words
        unsigned int* h_flag = nullptr;   // their pinned mirror
        cudaEvent_t ev[SLOTS] = {};
        long long step_of[SLOTS] = {-1, -1, -1, -1, -1, -1, -1, -1};  // the step a slot reports (-1: none)
        int next = 0;
        long long steps = 0;          // steps counted at their start
        long long last_trigger = 0;   // the last step with a wake, rewritten planes or a tracer switch
        long long idle_through = -1;  // the tracers are known idle after this step
    } tri;
    bool tr_poke = false;  // something outside a step changed what the tracers would do
    float center[2] = {0.0f, 0.0f};  // the chase point (set_center / recenter)
    bool reach_on = false;           // FluidCore::set_river_reach
    silt_river_reach reach;
    float* d_reach_bank = nullptr;   // the reference's f32 bank (device)
    bool wave_on = false;            // FluidCore::set_wave_maker
    silt_wave_maker wave;
    float wave_t = 0.0f;
    // Tire coupling (silt_set_coupling): nested sheets, none, or the learned closure.
    int coupling = SILT_COUPLING_NESTED;
    silt_closure* net = nullptr;
    float clos_threshold = 0.25f;
    silt::closure::Runner* clos = nullptr;
    bool clos_fallback_next = false;   // the last residual estimate was above the threshold
    silt_closure_stats cstats = {0, 0, 0.0f, 0.0};

    float* H(int l) { return h[l][cur]; }
    float* U(int l) { return u[l][cur]; }
    float* V(int l) { return v[l][cur]; }
};

namespace {

float water_nu() { return silt::host::dynamic_viscosity(3, 1.0f); }
void reach_band(const silt_sheet* s, int* axis, int* c0, int* c1);

// The water row's viscosity entry: in open-water mode a negative entry, the
// mobility itself (src/fluid_core.rs:8015-8017, sheet_mobility_for :169-172).
float water_nu(const silt_sheet* s) {
    return s->open_water ? -std::fmax(s->ow_mobility, 1.0e-4f) : water_nu();
}

// After a write from outside the step (seeding, plane writes) every tile may
// hold water and no buffer is known to be zero.
int tiles_dirty(silt_sheet* s) {
    s->tiles_all = true;
    s->mat_dirty = true;
    if (!s->tile_mem) return SILT_OK;
    const size_t nt = (size_t)s->tf.tiles_x * s->tf.tiles_x;
    for (int l = 0; l < 2; ++l)
        for (int b = 0; b < 2; ++b) {
            CK(cudaMemsetAsync(s->tf.wet[l][b], 1, nt, s->st));
            CK(cudaMemsetAsync(s->tf.zero_uv[l][b], 0, nt, s->st));
            CK(cudaMemsetAsync(s->tf.zero_h[l][b], 0, nt, s->st));
        }
    return SILT_OK;
}

// Materialise the lazy dry cut before anything reads or writes the planes.
int flush_cut(silt_sheet* s) {
    if (!s->cut_pending) return SILT_OK;
    for (int l = 0; l < 2; ++l) CK(silt::launch_apply_cut(s->H(l), s->U(l), s->V(l), s->n, 1.0e-6f, s->st));
    s->cut_pending = false;
    return SILT_OK;
}

int upload(silt_sheet* s, float* dst, const float* host) {
    CK(cudaMemcpyAsync(dst, host, s->n * sizeof(float), cudaMemcpyHostToDevice, s->st));
    return SILT_OK;
}

// The slurry's per-cell material planes, recomputed after grain or moisture
// changed (seeding calls only: the step never changes them).
int refresh_material(silt_sheet* s) {
    if (!s->mat_dirty) return SILT_OK;
    CK(silt::launch_material(s->grain, s->moisture, s->mat, s->mat + s->n, s->mat + 2 * s->n, s->n, s->st));
    s->mat_dirty = false;
    return SILT_OK;
}

// The coarse window as the tracers see it (the current planes).
silt::tracers::Window tracer_window(silt_sheet* s, const std::vector<silt_tire_push>& ps) {
    silt::tracers::Window w;
    w.S.water = s->H(0);
    w.S.slurry = s->H(1);
    w.S.uw = s->U(0);
    w.S.vw = s->V(0);
    w.S.res = s->res;
    w.S.cell = s->cfg.cell;
    w.S.ox = s->origin[0];
    w.S.oz = s->origin[1];
    w.S.cut_pending = s->cut_pending ? 1 : 0;
    w.S.surface_driven = (s->wave_on || s->reach_on) ? 1 : 0;
    w.T = s->tr;
    w.push = ps.empty() ? nullptr : ps.data();
    w.npush = (int)ps.size();
    w.rescan = s->tr_rescan ? 1 : 0;
    // A river inlet carrying a load writes its rows' suspended solids.
    w.sup_all = (s->reach_on && s->reach.inlet_turbidity != 0.0f) ? 1 : 0;
    return w;
}

// At a step's start: whether its tracer kernels can be skipped. They can when
// the tracers are known idle after the previous step (a device report of an
// earlier step said idle, and no step since had a trigger) and this step has
// no trigger: without a wake the tracer step does not run at all
// (src/fluid_core.rs:6213-6218), the suspended pass finds no load, and an
// idle state stays idle. Triggers: tire pushes, a surface drive, rewritten
// planes, the tracer switch. Reports arrive through pinned memory and are
// only polled, so the host never waits for one.
bool tracers_skip(silt_sheet* s, bool wake) {
    silt_sheet::TracerIdle& I = s->tri;
    if (!I.d_flag) return false;
    const long long n = ++I.steps;
    for (int k = 0; k < silt_sheet::TracerIdle::SLOTS; ++k) {
        if (I.step_of[k] < 0) continue;
        const cudaError_t q = cudaEventQuery(I.ev[k]);
        if (q == cudaErrorNotReady) continue;
        if (q == cudaSuccess && I.h_flag[k] && I.step_of[k] >= I.last_trigger) I.idle_through = n - 1;
        if (q != cudaSuccess) cudaGetLastError();
        I.step_of[k] = -1;
    }
    const bool trigger = wake || s->tr_rescan || s->tr_poke;
    s->tr_poke = false;
    if (trigger) I.last_trigger = n;
    if (!trigger && I.idle_through == n - 1) {
        I.idle_through = n;
        return true;
    }
    return false;
}

// The report word of this step's tracer launches (nullptr: no report).
unsigned int* tracers_report_word(silt_sheet* s) {
    silt_sheet::TracerIdle& I = s->tri;
    return I.d_flag ? I.d_flag + I.next : nullptr;
}

// After this step's tracer launches: bring the report back.
int tracers_report(silt_sheet* s) {
    silt_sheet::TracerIdle& I = s->tri;
    if (!I.d_flag) return SILT_OK;
    const int k = I.next;
    I.next = (I.next + 1) % silt_sheet::TracerIdle::SLOTS;
    CK(cudaMemcpyAsync(I.h_flag + k, I.d_flag + k, sizeof(unsigned int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaEventRecord(I.ev[k], s->st));
    I.step_of[k] = I.steps;
    return SILT_OK;
}

// Host plan of one sheet's coarse pair for one step: how many substeps to
// launch and whether the device decides the count.
struct CoarsePlan {
    int launched = 1;
    silt::SubstepCount sc;
    int soften_edge = 0;
    float nu_w = 0.0f;
};

// Substep count (src/fluid_core.rs:1715-1744). With every speed under the
// host's bound one substep is certain. Otherwise the device measures each
// layer's largest speed and decides its count; the host launches as many
// substeps as the bound allows, without waiting for the answer.
void coarse_plan(silt_sheet* s, float dt, CoarsePlan& cp) {
    const float cell = s->cfg.cell;
    const float cap = 8.0f;
    const float bound = s->vmax_bound;
    const float courant_len = 0.42f * std::max(cell, 1.0e-3f);
    memset(&cp.sc, 0, sizeof cp.sc);
    cp.launched = 1;
    cp.sc.dt = dt;
    cp.sc.cell = cell;
    cp.sc.cap = cap;
    cp.nu_w = water_nu(s);
    for (int q = 1; q <= 8; ++q) cp.sc.water_decay[q] = expf(-silt::host::sheet_damp(cp.nu_w) * (dt / (float)q));
    cp.sc.water_decay[0] = cp.sc.water_decay[1];
    if (!(dt * std::max(0.15f, bound) <= courant_len)) {
        const float nb = ceilf((dt * std::max(0.15f, bound)) / courant_len);
        cp.launched = std::isfinite(nb) ? (int)silt::host::rclamp(nb, 1.0f, cap) : (int)cap;
        cp.sc.speed2 = s->d_u32;
        cp.sc.overflow = s->d_u32 + 2;
        cp.sc.launched = cp.launched;
        s->parts.device_counts += 1;
    }
    cp.soften_edge = s->cfg.soften_border ? std::max(s->res / 12, 2) : 0;
}

// Parameters of substep k of FluidCore::step_pair (src/fluid_core.rs:7942-8150)
// on the sheet's current buffers, writing the other ones. `all`: step every
// tile (the first substep after an outside write, whose dry cells may carry
// velocity).
void coarse_substep(silt_sheet* s, const CoarsePlan& cp, float dt, int k, silt::ForceLaunch& F,
                    silt::TransportLaunch& T, int& all) {
    const int res = s->res;
    const float cell = s->cfg.cell;
    const float eps = 1.0e-6f;
    memset(&F, 0, sizeof F);
    memset(&T, 0, sizeof T);
    const int nxt = s->cur ^ 1;
    F.sc = cp.sc;
    F.sc.k = k;
    T.sc = F.sc;
    for (int l = 0; l < 2; ++l) {
        silt::LayerParams& P = F.lay[l];
        P.h = s->h[l][s->cur];
        P.bed = s->bed;
        P.u = s->u[l][s->cur];
        P.v = s->v[l][s->cur];
        P.u_out = s->u[l][nxt];
        P.v_out = s->v[l][nxt];
        P.res = res;
        P.cell = cell;
        P.div_two = s->div.two;
        P.div_cell2 = s->div.cell2;
        P.div_231 = s->div.d231;
        P.dt = dt;  // the device divides by its count when it decides one
        P.vort = l == 0 ? 0.08f : 0.05f;  // src/fluid_core.rs:8074, :8116
        P.eps = eps;
        P.project = cell > silt::host::kFineCell + 1.0e-6f;
        P.soften_edge = k == 0 ? cp.soften_edge : 0;
        reach_band(s, &P.open_axis, &P.open_c0, &P.open_c1);
        P.apply_cut = (k > 0 || s->cut_pending) ? 1 : 0;
        P.skip = 0;
        // The step pair runs serial inner loops, so coarse cells confine by
        // the raster sweep (force_gravity_open :2234-2260); 2 cm cells always
        // take the snapshot form (gravity_jacobi_serial, :2223-2228).
        P.sweep = s->confine == SILT_CONFINE_SWEEP && P.project && s->sweep_planes ? 1 : 0;
        P.fu = s->sweep_planes ? s->sweep_planes + (size_t)(2 * l) * s->n : nullptr;
        P.fv = s->sweep_planes ? s->sweep_planes + (size_t)(2 * l + 1) * s->n : nullptr;
        if (l == 0) {
            P.nu_mode = silt::NU_CONST;
            P.nu_c = cp.nu_w;
            P.mob_c = silt::host::sheet_mobility_for(cp.nu_w);
            P.decay_c = cp.sc.water_decay[1];
        } else {
            P.nu_mode = silt::NU_TABLE;
            P.grain = s->grain;
            P.moisture = s->moisture;
            P.nu_plane = s->mat;
            P.mob_plane = s->mat + s->n;
            P.damp_plane = s->mat + 2 * s->n;
        }
        silt::TransportParams& Q = T.lay[l];
        Q.h = s->h[l][s->cur];
        Q.u = P.u_out;
        Q.v = P.v_out;
        Q.h_out = s->h[l][nxt];
        Q.gate = nullptr;
        Q.bank_bed = nullptr;
        Q.ledger = s->d_acc + l;
        Q.cut = silt::fine::books(s->fine) + 3;
        Q.round = silt::fine::books(s->fine) + 6;
        Q.cut_area = (double)cell * (double)cell;
        Q.res = res;
        Q.cell = cell;
        Q.div_cell = s->div.cell;
        Q.dt = dt;
        Q.eps = eps;
        Q.skip = 0;
    }
    F.tf = s->tf;
    F.nxt = nxt;
    T.tf = s->tf;
    T.nxt = nxt;
    all = (s->tiles_all || !(k > 0 || s->cut_pending)) ? 1 : 0;
}

// After substep k: the other buffers are current and wait for the dry cut.
void coarse_advance(silt_sheet* s) {
    s->cur ^= 1;
    s->cut_pending = true;
    s->tiles_all = false;
}

// One coarse-sized pair of sheets for one step (FluidCore::step_pair, src/fluid_core.rs:7942-8150).
int step_coarse_pair(silt_sheet* s, float dt) {
    const int res = s->res;
    const float eps = 1.0e-6f;
    int rc0 = refresh_material(s);
    if (rc0) return rc0;
    CoarsePlan cp;
    coarse_plan(s, dt, cp);
    for (int k = 0; k < cp.launched; ++k) {
        silt::ForceLaunch F;
        silt::TransportLaunch T;
        int all = 0;
        coarse_substep(s, cp, dt, k, F, T, all);
        // The list kernel clears this substep's ledger sums, the next
        // substep's list count and, before the speed pass, the speed bits.
        const int slot = (int)(s->tile_seq++ & 1);
        s->tf.count = s->tile_count + slot;
        F.tf.count = s->tf.count;
        T.tf.count = s->tf.count;
        CK(silt::launch_tile_list(s->tf, s->cur, F.nxt, all, 0, 0, F.sc, s->tile_count + (slot ^ 1), s->d_acc,
                                  (k == 0 && F.sc.speed2) ? s->d_u32 : nullptr, s->st));
        if (k == 0 && F.sc.speed2) {
            // The substep count, from the tiles substep 0 steps.
            const float* hh[2] = {s->H(0), s->H(1)};
            const float* uu[2] = {s->U(0), s->U(1)};
            const float* vv[2] = {s->V(0), s->V(1)};
            CK(silt::launch_tile_speed2(s->tf, hh, uu, vv, res, eps, s->cut_pending ? 1 : 0, s->d_u32, s->st));
        }
        cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
        if (s->timing) {
            for (int q = 0; q < 3; ++q) {
                if (s->ev_pool.empty()) {
                    cudaEvent_t e;
                    CK(cudaEventCreate(&e));
                    s->ev_pool.push_back(e);
                }
                ev[q] = s->ev_pool.back();
                s->ev_pool.pop_back();
                s->ev_used.push_back(ev[q]);
            }
            CK(cudaEventRecord(ev[0], s->st));
        }
        CK(silt::launch_force(F, res, 2, s->st));
        if (s->timing) CK(cudaEventRecord(ev[1], s->st));
        CK(silt::launch_transport(T, res, 2, s->st));
        if (s->timing) CK(cudaEventRecord(ev[2], s->st));
        s->parts.force_launches += 1;
        coarse_advance(s);
    }
    // Every component is now clamped to the film speed cap.
    s->vmax_bound = silt::host::kSpeedCap * 1.4142137f;
    return SILT_OK;
}

// The coarse pair on the window engine: one CTA per layer steps it box by
// box exactly as FluidCore::step_pair does (serial inner loops, so the
// Gauss-Seidel confinement), in place on the current planes.
int step_coarse_pair_window(silt_sheet* s, float dt) {
    int rc = flush_cut(s);
    if (rc) return rc;
    if ((rc = refresh_material(s))) return rc;
    const int slot = s->win_flip;
    s->win_flip = (s->win_flip + 1) % silt_sheet::WIN_SLOTS;
    CK(cudaEventSynchronize(s->win_ev[slot]));
    silt::window::Job* jobs = s->h_win_jobs + 2 * slot;
    const float nu_w = water_nu(s);
    for (int l = 0; l < 2; ++l) {
        silt::window::Job& J = jobs[l];
        memset(&J, 0, sizeof J);
        J.h = s->H(l);
        J.u = s->U(l);
        J.v = s->V(l);
        J.bed = s->bed;
        J.grain = s->grain;
        J.moisture = s->moisture;
        silt::window::attach_scratch(J, s->win_planes + (size_t)l * silt::window::SCRATCH_PLANES * s->n, s->n);
        J.ledger = s->d_acc + l;
        J.cut = silt::fine::books(s->fine) + 3;
        J.round = silt::fine::books(s->fine) + 6;
        J.cut_area = (double)s->cfg.cell * (double)s->cfg.cell;
        J.res = s->res;
        J.cell = s->cfg.cell;
        J.div = s->div;
        J.solid = s->n_solids > 0 ? s->d_wall_mask : nullptr;
        J.dt = dt;
        J.vort = l == 0 ? 0.08f : 0.05f;  // src/fluid_core.rs:8074, :8116
        J.sub_cap = 8.0f;
        J.eps = 1.0e-6f;
        J.nu_mode = l == 0 ? silt::window::NU_CONST : silt::window::NU_TABLE;
        J.nu_plane = s->mat;
        J.mob_plane = s->mat + s->n;
        J.damp_plane = s->mat + 2 * s->n;
        J.nu_c = nu_w;
        J.mob_c = silt::host::sheet_mobility_for(nu_w);
        for (int k = 1; k <= 8; ++k) J.decay_c[k] = expf(-silt::host::sheet_damp(nu_w) * (dt / (float)k));
        J.soften_edge = s->cfg.soften_border ? std::max(s->res / 12, 2) : 0;
        reach_band(s, &J.open_axis, &J.open_c0, &J.open_c1);
        J.has_sc2 = 1;
        J.active = 1;
    }
    CK(cudaMemcpyAsync(s->d_win_jobs + 2 * slot, jobs, 2 * sizeof(silt::window::Job), cudaMemcpyHostToDevice, s->st));
    CK(cudaEventRecord(s->win_ev[slot], s->st));
    if (s->n_solids > 0) {
        // One mask for both sheets, from the water before either steps
        // (src/fluid_core.rs:7954-7967).
        CK(silt::walls::launch_mask(s->d_wall_mask, s->res, s->cfg.cell, s->origin[0], s->origin[1], s->H(0), s->bed,
                                    s->fine.d_solids, s->n_solids, s->st));
    }
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    if (s->timing) {
        for (int q = 0; q < 3; ++q) {
            if (s->ev_pool.empty()) {
                cudaEvent_t x;
                CK(cudaEventCreate(&x));
                s->ev_pool.push_back(x);
            }
            ev[q] = s->ev_pool.back();
            s->ev_pool.pop_back();
            s->ev_used.push_back(ev[q]);
        }
        CK(cudaEventRecord(ev[0], s->st));
    }
    CK(silt::window::launch_window_step(s->d_win_jobs + 2 * slot, 2, s->res, s->st));
    if (s->timing) {
        // Force time only: the transport runs inside the same kernel, so the
        // third event closes an empty transport interval.
        CK(cudaEventRecord(ev[1], s->st));
        CK(cudaEventRecord(ev[2], s->st));
        // The Gauss-Seidel passes each layer's last box needed (diagnostics;
        // timing mode only, as this read waits for the step).
        silt::window::Job done[2];
        CK(cudaMemcpyAsync(done, s->d_win_jobs + 2 * slot, sizeof done, cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
        for (int l = 0; l < 2; ++l) {
            s->parts.sweep_launches += 1;
            s->parts.sweep_solves += 1;
            s->parts.sweep_local_passes += done[l].gs_iters > 0 ? done[l].gs_iters : 0;
            s->parts.sweep_passes_max = std::max<int64_t>(s->parts.sweep_passes_max, done[l].gs_iters);
            if (done[l].gs_iters < 0) s->parts.sweep_fallbacks += 1;
        }
    }
    s->parts.force_launches += 1;
    s->parts.force_cells += 2 * (int64_t)s->n;
    s->parts.force_cells_water += (int64_t)s->n;
    s->vmax_bound = silt::host::kSpeedCap * 1.4142137f;
    return SILT_OK;
}

}  // namespace

namespace silt {
thread_local unsigned long long t_kernel_launches = 0;
}

extern "C" {

const char* silt_last_error(void) {
    if (g_err[0]) return g_err;
    if (const char* c = silt::closure::last_error()) return c;
    return silt::fine::last_error();
}

void silt_cfg_default(silt_cfg* c) {
    if (!c) return;
    c->res = 200;
    c->cell = 0.20f;
    c->fine_res = 160;
    c->fine_cell = 0.02f;
    c->fine_layout = SILT_FINE_MEAN_PATCH;
    c->tire_r = 0.56f;
    c->soften_border = 1;
    c->center_x = 0.0f;
    c->center_z = 0.0f;
    c->device = 0;
    c->stream = nullptr;
    c->engine = SILT_ENGINE_AUTO;
}

int silt_sheet_create(const silt_cfg* cfg, silt_sheet** out) {
    if (!cfg || !out) return fail_arg("cfg/out");
    if (cfg->res < 8 || cfg->res > 32768 || !(cfg->cell > 0.0f)) return fail_arg("res/cell");
    if (cfg->fine_res < 8 || cfg->fine_res > 1024 || !(cfg->fine_cell > 0.0f)) return fail_arg("fine_res/fine_cell");
    float ratio = cfg->cell / cfg->fine_cell;
    if (fabsf(ratio - roundf(ratio)) > 1.0e-3f || roundf(ratio) < 1.0f) return fail_arg("cell/fine_cell not whole");
    *out = nullptr;
    CK(cudaSetDevice(cfg->device));
    silt_sheet* s = new silt_sheet();
    s->cfg = *cfg;
    memset(&s->parts, 0, sizeof s->parts);
    s->res = cfg->res;
    s->n = (size_t)cfg->res * cfg->res;
    silt::host::snap_origin(cfg->center_x, cfg->center_z, (float)cfg->res * cfg->cell, cfg->cell, s->origin);
    if (cfg->stream) {
        s->st = (cudaStream_t)cfg->stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete s;
            return fail_cuda(e, "cudaStreamCreate");
        }
        s->own_stream = true;
    }
    const size_t nb = s->n * sizeof(float);
    cudaError_t e = cudaSuccess;
    for (int l = 0; l < 2 && e == cudaSuccess; ++l)
        for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
            e = cudaMalloc(&s->h[l][b], nb);
            if (e == cudaSuccess) e = cudaMalloc(&s->u[l][b], nb);
            if (e == cudaSuccess) e = cudaMalloc(&s->v[l][b], nb);
        }
    if (e == cudaSuccess) e = cudaMalloc(&s->bed, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->moisture, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->grain, s->n);
    if (e == cudaSuccess) e = cudaMalloc(&s->mat, 3 * nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->staging, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->staging2, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->staging_u8, s->n);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_acc, 8 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_sum_scratch, silt::SUM_SCRATCH_BYTES);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_sum_scratch, 0, silt::SUM_SCRATCH_BYTES, s->st);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_u32, 24 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_planes, 8 * sizeof(float*));
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_acc, 8 * sizeof(double));
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_flags, 16 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(s->d_u32, 0, 24 * sizeof(unsigned int));
    if (e == cudaSuccess) memset(s->h_flags, 0, 16 * sizeof(unsigned int));
    s->engine = cfg->engine == SILT_ENGINE_WINDOW || cfg->engine == SILT_ENGINE_GRID
                    ? cfg->engine
                    : (cfg->res <= silt::window::MAX_RES ? SILT_ENGINE_WINDOW : SILT_ENGINE_GRID);
    if (s->engine == SILT_ENGINE_WINDOW && cfg->res > silt::window::MAX_RES) {
        silt_sheet_destroy(s);
        return fail_arg("window engine serves windows up to 512 cells per side");
    }
    if (s->engine == SILT_ENGINE_GRID) {
        const int tx = (cfg->res + silt::GRID_TILE - 1) / silt::GRID_TILE;
        const size_t nt = (size_t)tx * tx;
        if (e == cudaSuccess) e = cudaMalloc(&s->tile_mem, 12 * nt + 2 * nt * sizeof(int) + 256);
        if (e == cudaSuccess) {
            uint8_t* q = s->tile_mem;
            for (int l = 0; l < 2; ++l)
                for (int b = 0; b < 2; ++b) {
                    s->tf.wet[l][b] = q;
                    q += nt;
                    s->tf.zero_uv[l][b] = q;
                    q += nt;
                    s->tf.zero_h[l][b] = q;
                    q += nt;
                }
            q = (uint8_t*)(((uintptr_t)q + 15) & ~uintptr_t(15));
            s->tf.list = (int*)q;
            s->tile_count = s->tf.list + 2 * nt;
            s->tf.count = s->tile_count;
            s->tf.stepped = reinterpret_cast<unsigned long long*>(s->d_u32 + 4);
            s->tf.tiles_x = tx;
            s->tf.sweep = s->sweep_state();
            e = cudaMemsetAsync(s->tile_count, 0, 2 * sizeof(int), s->st);
        }
        if (e == cudaSuccess) e = cudaMalloc(&s->sweep_planes, 4 * nb);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->sweep_planes, 0, 4 * nb, s->st);
        if (e == cudaSuccess) e = cudaMalloc(&s->sweep_stamp, 2 * nt * sizeof(unsigned int));
        if (e == cudaSuccess) e = cudaMemsetAsync(s->sweep_stamp, 0, 2 * nt * sizeof(unsigned int), s->st);
        s->tf.stamp = s->sweep_stamp;
    }
    if (s->engine == SILT_ENGINE_WINDOW) {
        const size_t wp = 2 * (size_t)silt::window::SCRATCH_PLANES * s->n * sizeof(float);
        if (e == cudaSuccess) e = cudaMalloc(&s->win_planes, wp);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->win_planes, 0, wp, s->st);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_win_jobs, 2 * silt_sheet::WIN_SLOTS * sizeof(silt::window::Job));
        if (e == cudaSuccess) e = cudaMallocHost(&s->h_win_jobs, 2 * silt_sheet::WIN_SLOTS * sizeof(silt::window::Job));
        for (int k = 0; k < silt_sheet::WIN_SLOTS && e == cudaSuccess; ++k)
            e = cudaEventCreateWithFlags(&s->win_ev[k], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        silt_sheet_destroy(s);
        return e == cudaErrorMemoryAllocation ? SILT_ENOMEM : fail_cuda(e, "allocate window");
    }
    for (int l = 0; l < 2; ++l)
        for (int b = 0; b < 2; ++b) {
            cudaMemsetAsync(s->h[l][b], 0, nb, s->st);
            cudaMemsetAsync(s->u[l][b], 0, nb, s->st);
            cudaMemsetAsync(s->v[l][b], 0, nb, s->st);
        }
    cudaMemsetAsync(s->bed, 0, nb, s->st);
    cudaMemsetAsync(s->moisture, 0, nb, s->st);
    cudaMemsetAsync(s->grain, 4, s->n, s->st);  // Grain::Other
    if (e == cudaSuccess && tiles_dirty(s) != SILT_OK) e = cudaErrorUnknown;
    int rc = silt::fine::create(s->fine, *cfg, s->res, s->st);
    if (rc != SILT_OK) {
        silt_sheet_destroy(s);
        return rc;
    }
    e = cudaMalloc(&s->tr_mem, silt::tracers::plane_bytes(s->res));
    if (e == cudaSuccess) e = silt::tracers::attach(s->tr, s->tr_mem, s->res, silt::fine::books(s->fine) + 7, s->st);
    if (e == cudaSuccess) e = cudaMalloc(&s->tri.d_flag, silt_sheet::TracerIdle::SLOTS * sizeof(unsigned int));
    if (e == cudaSuccess)
        e = cudaMallocHost(&s->tri.h_flag, silt_sheet::TracerIdle::SLOTS * sizeof(unsigned int));
    for (int k = 0; k < silt_sheet::TracerIdle::SLOTS && e == cudaSuccess; ++k)
        e = cudaEventCreateWithFlags(&s->tri.ev[k], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        silt_sheet_destroy(s);
        return e == cudaErrorMemoryAllocation ? SILT_ENOMEM : fail_cuda(e, "allocate tracers");
    }
    s->div = silt::cell_divisors(cfg->cell, s->st);
    e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) {
        silt_sheet_destroy(s);
        return fail_cuda(e, "init window");
    }
    *out = s;
    return SILT_OK;
}

int silt_sheet_destroy(silt_sheet* s) {
    if (!s) return SILT_OK;
    cudaSetDevice(s->cfg.device);
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->clos) {
        s->clos->release();
        delete s->clos;
    }
    cudaFree(s->ow_scratch);
    cudaFree(s->d_reach_bank);
    s->tr_run.release();
    cudaFree(s->tr_mem);
    cudaFree(s->tri.d_flag);
    if (s->tri.h_flag) cudaFreeHost(s->tri.h_flag);
    for (int k = 0; k < silt_sheet::TracerIdle::SLOTS; ++k)
        if (s->tri.ev[k]) cudaEventDestroy(s->tri.ev[k]);
    silt::fine::destroy(s->fine);
    for (int l = 0; l < 2; ++l)
        for (int b = 0; b < 2; ++b) {
            cudaFree(s->h[l][b]);
            cudaFree(s->u[l][b]);
            cudaFree(s->v[l][b]);
        }
    cudaFree(s->bed);
    cudaFree(s->moisture);
    cudaFree(s->grain);
    cudaFree(s->mat);
    cudaFree(s->staging);
    cudaFree(s->staging2);
    cudaFree(s->staging_u8);
    cudaFree(s->d_acc);
    cudaFree(s->d_sum_scratch);
    cudaFreeHost(s->h_flags);
    cudaFree(s->d_u32);
    cudaFree(s->d_planes);
    if (s->h_acc) cudaFreeHost(s->h_acc);
    cudaFree(s->win_planes);
    cudaFree(s->tile_mem);
    cudaFree(s->sweep_planes);
    cudaFree(s->sweep_stamp);
    cudaFree(s->d_win_jobs);
    if (s->h_win_jobs) cudaFreeHost(s->h_win_jobs);
    cudaFree(s->d_solids);
    if (s->h_solids) cudaFreeHost(s->h_solids);
    for (int k = 0; k < 2; ++k)
        if (s->solid_ev[k]) cudaEventDestroy(s->solid_ev[k]);
    cudaFree(s->d_wall_mask);
    cudaFree(s->d_bed_drop);
    cudaFree(s->d_wall_out);
    cudaFree(s->d_hole_bits);
    for (int k = 0; k < silt_sheet::WIN_SLOTS; ++k)
        if (s->win_ev[k]) cudaEventDestroy(s->win_ev[k]);
    for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : s->ev_used) cudaEventDestroy(e);
    if (s->own_stream) cudaStreamDestroy(s->st);
    delete s;
    return SILT_OK;
}

// After a wait on the stream, with h_flags read back: a sweep launch whose
// grid barrier gave up (the state of that step is incomplete), or a step
// whose layer needed more substeps than the host's speed bound launched (the
// state is off the reference's path).
static int check_substep_overflow(silt_sheet* s) {
    if (const unsigned int err = s->h_flags[silt_sheet::SWEEP_AT + 4 - 2]) {
        snprintf(g_err, sizeof g_err, "%s",
                 (err & 1u) ? "a Gauss-Seidel sweep launch gave up waiting at its grid barrier"
                            : "a transport tile's TMA copies did not arrive in time");
        return SILT_ETIMEOUT;
    }
    if (!s->h_flags[0]) return SILT_OK;
    snprintf(g_err, sizeof g_err, "%s",
             "a step needed more substeps than its speed bound launched; the state is no longer the reference's");
    return SILT_EBOUND;
}

int silt_sheet_sync(silt_sheet* s) {
    if (!s) return fail_arg("handle");
    CK(cudaMemcpyAsync(s->h_flags, s->d_u32 + 2, 14 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return check_substep_overflow(s);
}

// Host-side volume of what a seeding call writes, summed in f32 cell order like the reference.
static float host_volume(const float* w, size_t n, float area, bool clamp_nonneg) {
    float vol = 0.0f;
    for (size_t i = 0; i < n; ++i) {
        float x = w[i];
        if (clamp_nonneg) x = std::isfinite(x) ? std::max(x, 0.0f) : 0.0f;
        vol += x * area;
    }
    return vol;
}

int silt_map_water_bed(silt_sheet* s, const float* bed, const float* water, float* vol_out) {
    if (!s || !bed || !water) return fail_arg("map_water_bed");
    int rc = silt::fine::restrict_all(s->fine, s);
    if (rc) return rc;
    if ((rc = flush_cut(s))) return rc;
    if ((rc = upload(s, s->staging, bed))) return rc;
    if ((rc = upload(s, s->staging2, water))) return rc;
    CK(silt::op_map_water_bed(s->staging, s->staging2, s->bed, s->H(0), s->moisture, s->grain, s->n, s->st));
    CK(cudaStreamSynchronize(s->st));  // the host arrays may be freed on return
    if (vol_out) *vol_out = host_volume(water, s->n, s->cfg.cell * s->cfg.cell, true);
    s->ledger_fresh = false;
    if (int rc2 = tiles_dirty(s)) return rc2;
    return SILT_OK;
}

int silt_map_grain(silt_sheet* s, const uint8_t* grain) {
    if (!s || !grain) return fail_arg("map_grain");
    int rc = silt::fine::restrict_all(s->fine, s);
    if (rc) return rc;
    CK(cudaMemcpyAsync(s->grain, grain, s->n, cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->mat_dirty = true;
    return SILT_OK;
}

int silt_map_water_velocity(silt_sheet* s, const float* u, const float* v) {
    if (!s || !u || !v) return fail_arg("map_water_velocity");
    int rc = silt::fine::restrict_all(s->fine, s);
    if (rc) return rc;
    if ((rc = flush_cut(s))) return rc;
    if ((rc = upload(s, s->staging, u))) return rc;
    if ((rc = upload(s, s->staging2, v))) return rc;
    CK(silt::op_map_water_velocity(s->staging, s->staging2, s->H(0), s->U(0), s->V(0), s->n, s->st));
    CK(cudaStreamSynchronize(s->st));
    float m = 0.0f;
    for (size_t i = 0; i < s->n; ++i) {
        if (std::isfinite(u[i])) m = std::max(m, fabsf(u[i]));
        if (std::isfinite(v[i])) m = std::max(m, fabsf(v[i]));
    }
    s->vmax_bound = std::max(s->vmax_bound, m * 1.4142137f);
    return tiles_dirty(s);
}

static int paint(silt_sheet* s, float x0, float x1, float z0, float z1, float depth, int water, int grain, float m,
                 float* vol_out) {
    if (!s) return fail_arg("handle");
    int rc = flush_cut(s);
    if (rc) return rc;
    depth = std::max(depth, 0.0f);  // NaN becomes 0 like f32::max
    if (std::isnan(depth)) depth = 0.0f;
    m = silt::host::rclamp(m, 0.0f, 1.0f);
    CK(silt::op_paint(water ? s->H(0) : s->H(1), s->moisture, s->grain, s->res, s->cfg.cell, s->origin[0],
                      s->origin[1], x0, x1, z0, z1, depth, water, grain, m, s->st));
    if (vol_out) {
        float vol = 0.0f, area = s->cfg.cell * s->cfg.cell;
        for (int j = 0; j < s->res; ++j)
            for (int i = 0; i < s->res; ++i) {
                float x = s->origin[0] + ((float)i + 0.5f) * s->cfg.cell;
                float z = s->origin[1] + ((float)j + 0.5f) * s->cfg.cell;
                if (x < x0 || x >= x1 || z < z0 || z >= z1) continue;
                vol += depth * area;
            }
        *vol_out = vol;
    }
    s->ledger_fresh = false;
    return tiles_dirty(s);
}

int silt_pour_water(silt_sheet* s, float x0, float x1, float z0, float z1, float depth, float* vol_out) {
    return paint(s, x0, x1, z0, z1, depth, 1, SILT_GRAIN_WATER, 1.0f, vol_out);
}

int silt_pour_slurry(silt_sheet* s, float x0, float x1, float z0, float z1, float depth, int32_t grain, float moisture,
                     float* vol_out) {
    return paint(s, x0, x1, z0, z1, depth, 0, grain, moisture, vol_out);
}

int silt_lay_slurry_mask(silt_sheet* s, const float* depth, int32_t grain, float moisture, float* vol_out) {
    if (!s || !depth) return fail_arg("lay_slurry_mask");
    int rc = silt::fine::restrict_all(s->fine, s);
    if (rc) return rc;
    if ((rc = flush_cut(s))) return rc;
    if ((rc = upload(s, s->staging, depth))) return rc;
    CK(silt::op_lay_slurry(s->staging, s->H(1), s->moisture, s->grain, s->n, grain,
                           silt::host::rclamp(moisture, 0.0f, 1.0f), s->st));
    CK(cudaStreamSynchronize(s->st));
    if (vol_out) {
        float vol = 0.0f, area = s->cfg.cell * s->cfg.cell;
        for (size_t i = 0; i < s->n; ++i)
            if (std::isfinite(depth[i]) && depth[i] > 0.0f) vol += depth[i] * area;
        *vol_out = vol;
    }
    s->ledger_fresh = false;
    return tiles_dirty(s);
}

int silt_lay_slurry_on_water(silt_sheet* s, float depth, int32_t grain, float* vol_out) {
    if (!s) return fail_arg("lay_slurry_on_water");
    if (vol_out) *vol_out = 0.0f;
    if (!(std::isfinite(depth) && depth > 0.0f)) return SILT_OK_NOOP;
    int rc = silt::fine::restrict_all(s->fine, s);
    if (rc) return rc;
    if ((rc = flush_cut(s))) return rc;
    CK(silt::op_lay_on_water(s->H(0), s->H(1), s->moisture, s->grain, s->n, depth, grain, s->d_u32 + silt_sheet::COUNT_AT, s->st));
    unsigned int cells = 0;
    CK(cudaMemcpyAsync(&cells, s->d_u32 + silt_sheet::COUNT_AT, sizeof cells, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (vol_out) {
        // The reference's f32 running sum of depth * area over those cells.
        const float each = depth * (s->cfg.cell * s->cfg.cell);
        float vol = 0.0f;
        for (unsigned int k = 0; k < cells; ++k) vol += each;
        *vol_out = vol;
    }
    s->mat_dirty = true;
    s->ledger_fresh = false;
    return tiles_dirty(s);
}

int silt_window_origin(float center_x, float center_z, int32_t res, float cell, float* origin2) {
    if (!origin2 || res <= 0 || !(cell > 0.0f)) return fail_arg("window_origin");
    silt::host::snap_origin(center_x, center_z, (float)res * cell, cell, origin2);
    return SILT_OK;
}

int silt_read_substrate_grid(silt_sheet* s, const float* bed, const float* moisture, const uint8_t* grain) {
    if (!s || !bed || !moisture || !grain) return fail_arg("read_substrate_grid");
    int rc = silt::fine::restrict_all(s->fine, s);
    if (rc) return rc;
    if ((rc = upload(s, s->staging, bed))) return rc;
    if ((rc = upload(s, s->staging2, moisture))) return rc;
    CK(cudaMemcpyAsync(s->staging_u8, grain, s->n, cudaMemcpyHostToDevice, s->st));
    CK(silt::op_read_substrate(s->staging, s->staging2, s->staging_u8, s->bed, s->moisture, s->grain, s->H(1), s->n,
                               s->st));
    // The pad moisture: the most common whole percent (src/fluid_core.rs:5937-5961).
    uint32_t hist[101] = {0};
    for (size_t i = 0; i < s->n; ++i) {
        float m = silt::host::rclamp(moisture[i], 0.0f, 1.0f);
        float pct = m * 100.0f;
        size_t whole = pct > 0.0f ? (size_t)pct : 0;
        size_t bucket = pct - (float)whole >= 0.5f ? whole + 1 : whole;
        hist[std::min(bucket, (size_t)100)] += 1;
    }
    size_t best = 0;
    uint32_t best_n = 0;
    for (size_t i = 0; i < 101; ++i)
        if (hist[i] > best_n) {
            best = i;
            best_n = hist[i];
        }
    s->moisture_ambient = (float)best * 0.01f;
    CK(cudaStreamSynchronize(s->st));
    s->mat_dirty = true;
    return SILT_OK;
}

int silt_set_inflow(silt_sheet* s, int32_t j, float x0, float x1, float rate) {
    if (!s) return fail_arg("handle");
    if (!(rate > 0.0f) || j < 0 || j >= s->res) {
        s->inflow_j = -1;
        return SILT_OK;
    }
    int i0 = s->res, i1 = 0;
    for (int i = 0; i < s->res; ++i) {
        float x = s->origin[0] + ((float)i + 0.5f) * s->cfg.cell;
        if (x >= x0 && x < x1) {
            i0 = std::min(i0, i);
            i1 = std::max(i1, i + 1);
        }
    }
    if (i1 <= i0) return fail_arg("inflow strip covers no cell");
    s->inflow_j = j;
    s->inflow_i0 = i0;
    s->inflow_i1 = i1;
    s->inflow_rate = rate;
    return SILT_OK;
}

int silt_push_tire(silt_sheet* s, const silt_tire_push* p) {
    if (!s || !p) return fail_arg("push_tire");
    s->pushes.push_back(*p);
    return SILT_OK;
}

}  // extern "C"

namespace {

// The parts of silt_step before the coarse pair: the tire pushes of the step,
// the inflow strip, the nested patches (refine, shove, fine pair, peel,
// restrict, shove outside).
int step_inflow(silt_sheet* s, float dt);

int step_before_coarse(silt_sheet* s, float dt, std::vector<silt_tire_push>& ps, silt::fine::StepOut& fo) {
    ps.clear();
    ps.swap(s->pushes);
    int rc = step_inflow(s, dt);
    if (rc) return rc;
    return silt::fine::step_patches(s->fine, s, ps, dt, fo);
}

// The inflow strip's share of the step (a build addition, booked as opened).
int step_inflow(silt_sheet* s, float dt) {
    if (s->inflow_j >= 0) {
        int nc = s->inflow_i1 - s->inflow_i0;
        float add = s->inflow_rate * dt / ((float)nc * s->cfg.cell * s->cfg.cell);
        silt::fine::SheetView W = silt::fine::view_of(s);
        CK(silt::op_inflow(s->H(0), s->U(0), s->V(0), s->cut_pending ? 1 : 0, s->res, s->inflow_j, s->inflow_i0,
                           s->inflow_i1, add, W.tiles_x, W.t_wet[0], W.t_zuv[0], W.t_zh[0], s->st));
        s->opened_m3 += (double)add * (double)s->cfg.cell * (double)s->cfg.cell * (double)nc;
    }
    return SILT_OK;
}

// Open-water drivers after the coarse pair (src/fluid_core.rs:6073-6074):
// bed_friction (eddy shear, then Manning) in open-water mode, then the
// surface diffusion when it is set.
int open_water_step(silt_sheet* s, float dt) {
    if (!s->open_water && !(s->surface_diffusion > 0.0f)) return SILT_OK;
    if (!s->ow_scratch) CK(cudaMalloc(&s->ow_scratch, 2 * s->n * sizeof(float)));
    const float cell = s->cfg.cell;
    if (s->open_water) {
        const float k = s->ow_eddy > 0.0f ? std::fmin(s->ow_eddy * dt / (cell * cell), 0.2f) : 0.0f;
        const float gn2 = s->ow_manning > 0.0f ? silt::host::kGravityHost * s->ow_manning * s->ow_manning : 0.0f;
        if (k > 0.0f || gn2 > 0.0f)
            CK(silt::op_open_water(s->H(0), s->U(0), s->V(0), s->bed, s->res, k, gn2, dt, s->ow_scratch, s->st));
    }
    if (s->surface_diffusion > 0.0f) {
        const float k = std::fmin(s->surface_diffusion * dt / (cell * cell), 0.12f);
        CK(silt::op_diffuse_surface(s->H(0), s->bed, s->res, k, s->ow_scratch, s->d_acc, s->st));
    }
    return SILT_OK;
}

// The reach's band on the window (src/fluid_core.rs:8018-8033): 0 none, 1 a
// band of rows (a reach along X), 2 a band of columns (along Z).
void reach_band(const silt_sheet* s, int* axis, int* c0, int* c1) {
    *axis = 0;
    *c0 = *c1 = 0;
    if (!s->reach_on) return;
    const float cell = s->cfg.cell;
    const float o = s->reach.along_z ? s->origin[0] : s->origin[1];
    const float a = std::fmax(std::floor((s->reach.cross0 - o) / cell), 0.0f);
    const float b = std::fmax(std::ceil((s->reach.cross1 - o) / cell), 0.0f);
    *c0 = (int)std::fmin(a, 2.0e9f);
    *c1 = (int)std::fmin(std::fmin(b, 2.0e9f), (float)s->res);
    *axis = s->reach.along_z ? 2 : 1;
}

// drive_waves (src/fluid_core.rs:7420-7480): the step's scalars on the host.
int wave_step(silt_sheet* s, float dt) {
    if (!s->wave_on) return SILT_OK;
    const silt_wave_maker& w = s->wave;
    if (dt <= 0.0f || w.period_s <= 0.0f) return SILT_OK;
    s->wave_t += dt;
    const float len = std::hypot(w.dir_x, w.dir_z);
    if (len < 1.0e-6f || !std::isfinite(len)) return SILT_OK;
    silt::drivers::WaveStep q;
    q.dx = w.dir_x / len;
    q.dz = w.dir_z / len;
    const float ramp = w.ramp_s > 0.0f ? silt::host::rclamp(s->wave_t / w.ramp_s, 0.0f, 1.0f) : 1.0f;
    const float phase = 6.28318548f * s->wave_t / w.period_s;  // TAU in f32
    q.stroke = w.amplitude_m_s * ramp * std::sin(phase);
    q.pull = 1.0f - std::exp(-dt / 0.08f);
    const float cell = s->cfg.cell;
    q.span_x = std::fmax(w.x1 - w.x0, cell);
    q.span_z = std::fmax(w.z1 - w.z0, cell);
    auto idx = [](float f) { return (int)std::fmax(std::fmin(f, 2.0e9f), -2.0e9f); };
    q.i0 = std::max(idx(std::floor((w.x0 - s->origin[0]) / cell)), 0);
    q.i1 = std::min(idx(std::ceil((w.x1 - s->origin[0]) / cell)), s->res);
    q.j0 = std::max(idx(std::floor((w.z0 - s->origin[1]) / cell)), 0);
    q.j1 = std::min(idx(std::ceil((w.z1 - s->origin[1]) / cell)), s->res);
    q.x0 = w.x0;
    q.x1 = w.x1;
    q.z0 = w.z0;
    q.z1 = w.z1;
    if (q.i1 <= q.i0 || q.j1 <= q.j0) return SILT_OK;
    CK(silt::drivers::wave_step(silt::fine::view_of(s), q, s->st));
    return SILT_OK;
}

// scour_contacts (src/fluid_core.rs:7364-7420) after the coarse peel, from
// the mask of the state the step left.
int scour_step(silt_sheet* s, float dt) {
    if (s->n_solids == 0 || !(dt > 0.0f)) return SILT_OK;
    CK(silt::walls::launch_mask(s->d_wall_mask, s->res, s->cfg.cell, s->origin[0], s->origin[1], s->H(0), s->bed,
                                s->fine.d_solids, s->n_solids, s->st));
    silt::walls::ScourPlanes P;
    P.mask = s->d_wall_mask;
    P.water = s->H(0);
    P.uw = s->U(0);
    P.vw = s->V(0);
    P.bed = s->bed;
    P.slurry = s->H(1);
    P.us = s->U(1);
    P.vs = s->V(1);
    P.moisture = s->moisture;
    P.bed_drop = s->d_bed_drop;
    P.grain = s->grain;
    P.res = s->res;
    P.area = s->cfg.cell * s->cfg.cell;
    P.dt = dt;
    P.eroded = silt::fine::books(s->fine) + 5;
    P.slurry_sum = s->d_acc + 1;
    P.hole_bits = s->d_hole_bits;
    CK(silt::walls::launch_scour(P, s->st));
    s->mat_dirty = true;
    return SILT_OK;
}

// feed_reach (src/fluid_core.rs:7638-7745).
int reach_step(silt_sheet* s) {
    if (!s->reach_on) return SILT_OK;
    silt::drivers::ReachStep r;
    int axis;
    reach_band(s, &axis, &r.c0, &r.c1);
    if (r.c1 <= r.c0) return SILT_OK;
    r.along_z = s->reach.along_z ? 1 : 0;
    r.positive = s->reach.positive ? 1 : 0;
    r.rows = std::min(std::max(s->reach.rows, 1), s->res / 4);
    if (r.rows < 1) return SILT_OK;
    r.dx = r.along_z ? 0.0f : (r.positive ? 1.0f : -1.0f);
    r.dz = r.along_z ? (r.positive ? 1.0f : -1.0f) : 0.0f;
    r.inlet_eta = s->reach.inlet_eta;
    r.outlet_eta = s->reach.outlet_eta;
    r.inlet_speed = s->reach.inlet_speed_m_s;
    const float c = s->reach.inlet_turbidity;
    r.inflow_c = s->turbidity && std::isfinite(c) ? silt::host::rclamp(c, 0.0f, 1.0f) : 0.0f;
    r.susp = s->tr.susp[0];
    r.entrained = silt::fine::books(s->fine) + 7;
    CK(silt::drivers::reach_step(silt::fine::view_of(s), r, s->d_reach_bank, silt::fine::books(s->fine), s->st));
    return SILT_OK;
}

// The coupling of this step's tires: sets whether the nested patches are laid
// and returns true when the learned closure corrects the step.
bool closure_begin(silt_sheet* s) {
    s->fine.patches_off = false;
    s->fine.coarse_shove_off = false;
    if (s->coupling == SILT_COUPLING_NESTED) return false;
    if (s->coupling == SILT_COUPLING_NONE) {
        s->fine.patches_off = true;
        return false;
    }
    std::vector<float> r;
    double moved = 0.0;
    if (s->clos->poll(r, &moved) && !r.empty()) {
        s->cstats.last_residual = r[0];
        s->cstats.moved_m3 = moved;
        s->clos_fallback_next = r[0] > s->clos_threshold;
    }
    if (s->pushes.empty()) {  // no tire, nothing to correct: the plain coarse step
        s->fine.patches_off = true;
        return false;
    }
    if (s->clos_fallback_next) {  // the nested sheets take this step
        s->clos_fallback_next = false;
        s->cstats.fallback_steps += 1;
        return false;
    }
    s->fine.patches_off = true;
    s->fine.coarse_shove_off = true;  // the network carries the tires' effect on the window
    s->cstats.closure_steps += 1;
    return true;
}

silt::closure::FeatureJob closure_job(silt_sheet* s, const std::vector<silt_tire_push>& ps) {
    silt::closure::FeatureJob J;
    memset(&J, 0, sizeof J);
    J.W = silt::fine::view_of(s);
    silt::closure::crop_origin(ps, s->origin[0], s->origin[1], s->cfg.cell, &J.ci0, &J.cj0);
    J.ntires = (int)std::min(ps.size(), (size_t)silt::closure::MAX_CROP_TIRES);
    for (int t = 0; t < J.ntires; ++t) J.tires[t] = ps[t];
    return J;
}

int closure_correct(silt_sheet* s, const silt::closure::FeatureJob& F) {
    std::vector<silt::closure::ApplyJob> A(1);
    memset(A.data(), 0, sizeof(silt::closure::ApplyJob));
    A[0].W = silt::fine::view_of(s);
    A[0].ci0 = F.ci0;
    A[0].cj0 = F.cj0;
    CK(s->clos->correct(A, s->net->net, s->st));
    return SILT_OK;
}

}  // namespace

extern "C" {

int silt_step(silt_sheet* s, float dt, silt_spray_event* out, int32_t cap, int32_t* n_out) {
    if (!s) return fail_arg("handle");
    if (n_out) *n_out = 0;
    if (!(dt > 0.0f) || !std::isfinite(dt)) {
        s->pushes.clear();
        return SILT_OK_NOOP;
    }
    const unsigned long long launches0 = silt::t_kernel_launches;
    using clock = std::chrono::steady_clock;
    const clock::time_point t0 = clock::now();
    clock::time_point tp = t0;
    // Host time per phase (with timing on): the time since the last mark goes
    // to phase k (the same slots as a batch's, where they apply).
    auto phase = [&](int k) {
        if (!s->timing) return;
        const clock::time_point t = clock::now();
        s->parts.host_phase_ms[k] += std::chrono::duration<double, std::milli>(t - tp).count();
        tp = t;
    };
    std::vector<silt_tire_push> ps;
    silt::fine::StepOut fo;
    int rc;
    const bool skip_tracers = tracers_skip(s, !s->pushes.empty() || s->wave_on || s->reach_on);
    // Lift from the column the tire rolls into, before the sheet shoves it
    // (entrain_wake, src/fluid_core.rs:6051-6053).
    if (s->turbidity && !s->pushes.empty()) {
        const silt::tracers::Window w = tracer_window(s, s->pushes);
        CK(silt::tracers::entrain(s->tr_run, &w, 1, dt, s->st));
    }
    // The learned closure reads the state the nested sheets would start from.
    const bool net_on = closure_begin(s);
    silt::closure::FeatureJob F;
    if (net_on) {
        F = closure_job(s, s->pushes);
        CK(s->clos->features({F}, s->net->net, s->st));
    }
    phase(0);
    rc = step_before_coarse(s, dt, ps, fo);
    if (rc) return rc;
    phase(2);
    const clock::time_point t2 = clock::now();
    if ((rc = wave_step(s, dt))) return rc;
    rc = s->engine == SILT_ENGINE_WINDOW ? step_coarse_pair_window(s, dt) : step_coarse_pair(s, dt);
    if (rc) return rc;
    if ((rc = open_water_step(s, dt))) return rc;
    phase(3);
    rc = silt::fine::peel_coarse(s->fine, s, ps, fo);
    if (rc) return rc;
    if ((rc = scour_step(s, dt))) return rc;
    phase(4);
    if (!skip_tracers) {
        // step_tracers (src/fluid_core.rs:6080), then the reach, then the
        // suspended load (:6082-6089).
        silt::tracers::Window w = tracer_window(s, ps);
        w.susp_on = s->turbidity ? 1 : 0;
        w.idle_out = tracers_report_word(s);
        CK(silt::tracers::step_tracers(s->tr_run, &w, 1, dt, s->st));
        s->tr_rescan = false;
    }
    if ((rc = reach_step(s))) return rc;
    if (s->turbidity && !skip_tracers) {
        silt::tracers::Window w = tracer_window(s, ps);
        w.susp_on = 1;
        w.idle_out = tracers_report_word(s);
        CK(silt::tracers::step_suspended(s->tr_run, &w, 1, dt, s->st));
    }
    if (!skip_tracers && (rc = tracers_report(s))) return rc;
    phase(5);
    if (net_on && (rc = closure_correct(s, F))) return rc;
    int32_t nev = 0;
    if (out || n_out) {
        rc = silt::fine::collect_spray(s->fine, s, fo, out, cap, &nev);
        if (rc) return rc;
    }
    if (n_out) *n_out = nev;
    phase(6);
    s->parts.steps += 1;
    s->parts.launches += (int64_t)(silt::t_kernel_launches - launches0);
    if (s->timing) {
        const clock::time_point t3 = clock::now();
        s->parts.host_step_ms += std::chrono::duration<double, std::milli>(t3 - t0).count();
        s->parts.host_fine_ms += std::chrono::duration<double, std::milli>(t2 - t0).count();
    }
    s->ledger_fresh = true;  // d_acc holds the post-step depth sums (spray already taken off)
    return SILT_OK;
}

}  // extern "C"

namespace {

// world_key's axis (src/fluid_core.rs:9894-9896) on the host: floor(p / cell)
// as a saturating i32 cast.
long long world_axis_host(float p, float cell) {
    const float f = std::floor(p / cell);
    if (std::isnan(f)) return 0;
    if (f >= 2147483648.0f) return 2147483647LL;
    if (f < -2147483648.0f) return -2147483648LL;
    return (long long)f;
}

// uniform_cell_shift (src/fluid_core.rs:9899-9933): the move is a whole number
// of cells for the window's corners and middle alike.
bool uniform_cell_shift(const float* o, const float* nw, float cell, int res, int* di, int* dj) {
    if (res <= 0 || !(std::isfinite(cell) && cell > 0.0f)) return false;
    auto key = [&](const float* org, int i, int j, long long* kx, long long* kz) {
        *kx = world_axis_host(org[0] + ((float)i + 0.5f) * cell, cell);
        *kz = world_axis_host(org[1] + ((float)j + 0.5f) * cell, cell);
    };
    long long o0x, o0z, n0x, n0z, o1x, o1z, n1x, n1z, omx, omz, nmx, nmz;
    key(o, 0, 0, &o0x, &o0z);
    key(nw, 0, 0, &n0x, &n0z);
    const long long ddi = n0x - o0x, ddj = n0z - o0z;
    const int last = res - 1, mid = res / 2;
    key(o, last, last, &o1x, &o1z);
    key(nw, last, last, &n1x, &n1z);
    if (o1x - o0x != last || o1z - o0z != last) return false;
    if (n1x - n0x != last || n1z - n0z != last) return false;
    if (n1x - o1x != ddi || n1z - o1z != ddj) return false;
    key(o, mid, mid, &omx, &omz);
    key(nw, mid, mid, &nmx, &nmz);
    if (nmx - omx != ddi || nmz - omz != ddj) return false;
    if (ddi > INT_MAX || ddi < INT_MIN || ddj > INT_MAX || ddj < INT_MIN) return false;
    *di = (int)ddi;
    *dj = (int)ddj;
    return true;
}

// Room in the parked table for `incoming` more keys, rebuilding it larger
// (and without tombstones) when taken slots would pass half of it.
int park_room(silt_sheet* s, size_t incoming) {
    silt::park::Table& T = silt::fine::park_table(s->fine);
    unsigned int used = 0, overflow = 0;
    if (T.cap) CK(silt::park::usage(T, &used, &overflow, s->st));
    if (overflow) return fail_cuda(cudaErrorMemoryAllocation, "parked cells: table overflow");
    size_t want = 2 * ((size_t)used + incoming);
    if (T.cap && want <= T.cap) return SILT_OK;
    size_t cap = 1u << 16;
    while (cap < want) cap <<= 1;
    if (cap > (1u << 30)) return fail_cuda(cudaErrorMemoryAllocation, "parked cells: table too large");
    CK(silt::park::rebuild(T, (unsigned int)cap, s->st));
    return SILT_OK;
}

}  // namespace

extern "C" {

int silt_set_center(silt_sheet* s, float cx, float cz) {
    if (!s) return fail_arg("handle");
    s->center[0] = cx;
    s->center[1] = cz;
    return SILT_OK;
}

int silt_recenter(silt_sheet* s, float cx, float cz) {
    if (!s) return fail_arg("handle");
    if (!std::isfinite(cx) || !std::isfinite(cz)) return fail_arg("recenter: centre");
    int rc = silt::fine::restrict_all(s->fine, s);  // the patches go back first (src/fluid_core.rs:5410-5412)
    if (rc) return rc;
    s->center[0] = cx;
    s->center[1] = cz;
    float nw[2];
    silt::host::snap_origin(cx, cz, (float)s->res * s->cfg.cell, s->cfg.cell, nw);
    if (std::fabs(nw[0] - s->origin[0]) < 1.0e-4f && std::fabs(nw[1] - s->origin[1]) < 1.0e-4f) return SILT_OK;
    if ((rc = flush_cut(s))) return rc;
    int di = 0, dj = 0;
    const bool scroll = uniform_cell_shift(s->origin, nw, s->cfg.cell, s->res, &di, &dj);
    const size_t n = s->n;
    size_t incoming = n;
    if (scroll) {
        const size_t ai = (size_t)std::min(std::abs(di), s->res), aj = (size_t)std::min(std::abs(dj), s->res);
        incoming = std::min(n, ai * (size_t)s->res + aj * (size_t)s->res);
    }
    if ((rc = park_room(s, incoming))) return rc;
    silt::park::Table& T = silt::fine::park_table(s->fine);
    silt::park::Planes P;
    memset(&P, 0, sizeof P);
    const int nx = s->cur ^ 1;
    for (int l = 0; l < 2; ++l) {
        P.h[l] = s->h[l][s->cur];
        P.u[l] = s->u[l][s->cur];
        P.v[l] = s->v[l][s->cur];
        P.h_out[l] = s->h[l][nx];
        P.u_out[l] = s->u[l][nx];
        P.v_out[l] = s->v[l][nx];
    }
    P.moisture = s->moisture;
    P.moisture_out = s->staging;
    P.foam = s->tr.foam[0];
    P.turbid = s->tr.turbid[0];
    P.susp = s->tr.susp[0];
    P.foam_out = s->tr.foam[1];
    P.turbid_out = s->tr.turbid[1];
    P.susp_out = s->tr.susp[1];
    P.track_susp = s->turbidity ? 1 : 0;
    P.res = s->res;
    P.cell = s->cfg.cell;
    P.ambient = s->moisture_ambient;
    P.books = silt::fine::books(s->fine);
    if (scroll) {
        // shift_coarse_scroll (src/fluid_core.rs:9024-9145).
        CK(silt::park::park_cells(P, T, s->origin[0], s->origin[1], di, dj, 0, s->st));
        CK(silt::park::scroll_cells(P, di, dj, s->st));
        s->cur = nx;
        std::swap(s->moisture, s->staging);
        // The tracers scrolled into their scratch planes; the fields keep their addresses.
        for (int q = 0; q < 3; ++q) {
            float* const* pl = q == 0 ? s->tr.foam : (q == 1 ? s->tr.turbid : s->tr.susp);
            CK(cudaMemcpyAsync(pl[0], pl[1], s->n * sizeof(float), cudaMemcpyDeviceToDevice, s->st));
        }
        for (int l = 0; l < 2; ++l) {
            P.h[l] = s->h[l][s->cur];
            P.u[l] = s->u[l][s->cur];
            P.v[l] = s->v[l][s->cur];
        }
        P.moisture = s->moisture;
        s->origin[0] = nw[0];
        s->origin[1] = nw[1];
        CK(silt::park::restore_cells(P, T, s->origin[0], s->origin[1], di, dj, 0, s->st));
    } else {
        // shift_coarse_hash (src/fluid_core.rs:9147-9222).
        CK(silt::park::park_cells(P, T, s->origin[0], s->origin[1], 0, 0, 1, s->st));
        s->origin[0] = nw[0];
        s->origin[1] = nw[1];
        CK(silt::park::restore_cells(P, T, s->origin[0], s->origin[1], 0, 0, 1, s->st));
    }
    if ((rc = silt::fine::move_window(s->fine, s, di, dj, scroll))) return rc;
    CK(silt::tracers::reset_indices(s->tr, s->res, s->st));  // reset_tracer_indices (src/fluid_core.rs:9125, :9225)
    s->tr_rescan = true;
    unsigned int used = 0, overflow = 0;
    CK(silt::park::usage(T, &used, &overflow, s->st));
    if (overflow) return fail_cuda(cudaErrorMemoryAllocation, "parked cells: table overflow");
    s->vmax_bound = std::max(s->vmax_bound, silt::host::kSpeedCap * 1.4142137f);
    s->ledger_fresh = false;
    return tiles_dirty(s);
}

int silt_set_open_water(silt_sheet* s, int32_t on, float mobility, float manning_n, float eddy_m2_s) {
    if (!s) return fail_arg("handle");
    s->open_water = on != 0 && std::isfinite(mobility) && std::isfinite(manning_n) && std::isfinite(eddy_m2_s);
    if (s->open_water) {
        s->ow_mobility = std::fmin(std::fmax(mobility, 0.0f), 1.0f);
        s->ow_manning = std::fmax(manning_n, 0.0f);
        s->ow_eddy = std::fmax(eddy_m2_s, 0.0f);
    }
    s->fine.open_mobility = s->open_water ? s->ow_mobility : -1.0f;
    return SILT_OK;
}

int silt_set_surface_diffusion(silt_sheet* s, float m2_s) {
    if (!s) return fail_arg("handle");
    s->surface_diffusion = std::isfinite(m2_s) ? std::fmax(m2_s, 0.0f) : 0.0f;
    return SILT_OK;
}

int silt_set_river_reach(silt_sheet* s, const silt_river_reach* reach) {
    if (!s) return fail_arg("handle");
    s->reach_on = reach != nullptr;
    if (reach) {
        s->reach = *reach;
        if (!s->d_reach_bank) {
            CK(cudaMalloc(&s->d_reach_bank, sizeof(float)));
            CK(cudaMemsetAsync(s->d_reach_bank, 0, sizeof(float), s->st));
        }
    }
    return SILT_OK;
}

int silt_set_wave_maker(silt_sheet* s, const silt_wave_maker* wave) {
    if (!s) return fail_arg("handle");
    s->wave_on = wave != nullptr;
    if (wave) s->wave = *wave;
    s->wave_t = 0.0f;
    return SILT_OK;
}

int silt_set_hydro_solids(silt_sheet* s, const silt_hydro_solid* solids, int32_t n) {
    if (!s || n < 0 || (n > 0 && !solids)) return fail_arg("set_hydro_solids");
    if (n > silt::walls::MAX_SOLIDS) return fail_arg("set_hydro_solids: more than 64 bodies");
    if (n > 0 && s->engine != SILT_ENGINE_WINDOW) return fail_arg("set_hydro_solids: walls need the window engine");
    CK(cudaSetDevice(s->cfg.device));
    if (n > 0 && !s->d_solids) {
        const size_t bytes = 2 * silt::walls::MAX_SOLIDS * sizeof(silt::walls::SolidGeom);
        CK(cudaMalloc(&s->d_solids, bytes));
        CK(cudaMallocHost(&s->h_solids, bytes));
        for (int k = 0; k < 2; ++k) CK(cudaEventCreateWithFlags(&s->solid_ev[k], cudaEventDisableTiming));
        CK(cudaMalloc(&s->d_wall_mask, s->n));
        CK(cudaMalloc(&s->d_bed_drop, s->n * sizeof(float)));
        CK(cudaMemsetAsync(s->d_bed_drop, 0, s->n * sizeof(float), s->st));
        CK(cudaMalloc(&s->d_wall_out, (4 + 3 * silt::walls::MAX_SOLIDS) * sizeof(double)));
        CK(cudaMalloc(&s->d_hole_bits, sizeof(unsigned int)));
        CK(cudaMemsetAsync(s->d_hole_bits, 0, sizeof(unsigned int), s->st));
    }
    if (n > 0) {
        const int slot = s->solid_slot ^ 1;
        CK(cudaEventSynchronize(s->solid_ev[slot]));
        silt::walls::SolidGeom* h = s->h_solids + (size_t)slot * silt::walls::MAX_SOLIDS;
        for (int k = 0; k < n; ++k) {
            const silt_hydro_solid& b = solids[k];
            h[k] = silt::walls::make_geom(b.x, b.z, b.yaw, b.half_length, b.half_width, b.bottom_y, b.top_y,
                                          b.contact);
        }
        silt::walls::SolidGeom* d = s->d_solids + (size_t)slot * silt::walls::MAX_SOLIDS;
        CK(cudaMemcpyAsync(d, h, (size_t)n * sizeof *h, cudaMemcpyHostToDevice, s->st));
        CK(cudaEventRecord(s->solid_ev[slot], s->st));
        s->solid_slot = slot;
    }
    s->n_solids = n;
    s->solids.assign(solids, solids + n);
    s->fine.d_solids = n > 0 ? s->d_solids + (size_t)s->solid_slot * silt::walls::MAX_SOLIDS : nullptr;
    s->fine.n_solids = n;
    return SILT_OK;
}

// src/fluid_core.rs:4606-4615 cylinder_segment_volume (C library acosf, sqrtf).
static float cylinder_segment_volume(float depth, float radius, float width) {
    const float d = silt::host::rclamp(depth, 0.0f, radius * 2.0f);
    if (d <= 1.0e-4f || width <= 0.0f || radius <= 1.0e-3f) return 0.0f;
    const float c = silt::host::rclamp((radius - d) / radius, -1.0f, 1.0f);
    const float area =
        radius * radius * std::acos(c) - (radius - d) * std::sqrt(std::fmax(2.0f * radius * d - d * d, 0.0f));
    return std::fmax(area, 0.0f) * width;
}

int silt_get_hydro_load(silt_sheet* s, silt_hydro_load* out) {
    if (!s || !out) return fail_arg("hydro_load");
    CK(cudaSetDevice(s->cfg.device));
    memset(out, 0, sizeof *out);
    const int n = s->n_solids;
    std::vector<double> acc(4 + 3 * (size_t)n, 0.0);
    unsigned int hole_bits = 0;
    if (n > 0) {
        CK(silt::walls::launch_mask(s->d_wall_mask, s->res, s->cfg.cell, s->origin[0], s->origin[1], s->H(0), s->bed,
                                    s->fine.d_solids, n, s->st));
        CK(silt::walls::launch_load(s->d_wall_mask, s->H(0), s->U(0), s->V(0), s->bed, s->res, s->cfg.cell,
                                    s->origin[0], s->origin[1], s->fine.d_solids, n, s->d_wall_out, s->st));
        CK(cudaMemcpyAsync(acc.data(), s->d_wall_out, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    }
    if (s->d_hole_bits)
        CK(cudaMemcpyAsync(&hole_bits, s->d_hole_bits, sizeof hole_bits, cudaMemcpyDeviceToHost, s->st));
    double spray = 0.0, park_w = 0.0, park_s = 0.0, eroded = 0.0;
    int rc = silt::fine::ledger_parts(s->fine, s, &spray, &park_w, &park_s, nullptr, nullptr, &eroded);
    if (rc) return rc;
    out->force_x = (float)acc[0];
    out->force_z = (float)acc[1];
    out->wheel_blocks = (uint32_t)acc[2];
    out->belly_blocks = (uint32_t)acc[3];
    const float rho_g = 1000.0f * 9.81f;
    float wheel_b = 0.0f, hull_b = 0.0f, displaced = 0.0f;
    for (int k = 0; k < n; ++k) {
        const double cnt = acc[4 + 3 * (size_t)k + 2];
        if (cnt < 1.0) continue;
        const float bed = (float)(acc[4 + 3 * (size_t)k] / cnt);
        const float water = (float)(acc[4 + 3 * (size_t)k + 1] / cnt);
        const silt_hydro_solid& b = s->solids[k];
        if (b.radius > 0.0f) {
            const float vol = cylinder_segment_volume(water, b.radius, b.width);
            displaced += vol;
            wheel_b += rho_g * vol;
        } else {
            const float eta = bed + water;
            const float height = std::fmax(b.top_y - b.bottom_y, 0.0f);
            const float sub = silt::host::rclamp(eta - b.bottom_y, 0.0f, height);
            const float vol = (b.half_length * 2.0f) * (b.half_width * 2.0f) * sub * 0.36f;
            displaced += vol;
            hull_b += rho_g * vol;
        }
    }
    out->buoyancy_n = wheel_b + hull_b;
    out->hull_buoyancy_n = hull_b;
    out->wheel_buoyancy_n = wheel_b;
    out->displaced_m3 = displaced;
    out->eroded_m3 = (float)eroded;
    float hole;
    memcpy(&hole, &hole_bits, sizeof hole);
    out->hole_m = hole;
    return SILT_OK;
}

int silt_set_turbidity_enabled(silt_sheet* s, int32_t on) {
    if (!s) return fail_arg("handle");
    s->turbidity = on != 0;
    s->tr_poke = true;
    return SILT_OK;
}

int silt_sample(silt_sheet* s, float x, float z, silt_ground_sample* out) {
    if (!s || !out) return fail_arg("sample");
    memset(out, 0, sizeof *out);
    auto axis = [&](float o, float p) -> long {  // coarse_axis, src/fluid_core.rs:9546-9557
        const float i = std::floor((p - o) / s->cfg.cell);
        if (i < 0.0f) return -1;
        const double ii = std::isnan(i) ? 0.0 : (double)i;
        return ii >= (double)s->res ? -1 : (long)ii;
    };
    const long i = axis(s->origin[0], x), j = axis(s->origin[1], z);
    if (i < 0 || j < 0) return SILT_OK_NOOP;  // outside the window: nothing parked per cell here
    int rc = flush_cut(s);
    if (rc) return rc;
    const size_t c = (size_t)j * s->res + (size_t)i;
    float vals[6];
    const float* src[6] = {s->H(0) + c, s->H(1) + c, s->U(1) + c, s->V(1) + c, s->moisture + c, s->bed + c};
    for (int k = 0; k < 6; ++k)
        CK(cudaMemcpyAsync(vals + k, src[k], sizeof(float), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    out->water_m = vals[0];
    out->slurry_m = vals[1];
    out->u = vals[2];
    out->v = vals[3];
    out->settled_dust_m = 0.0f;
    out->moisture = vals[4];
    out->bed_m = vals[5];
    return SILT_OK;
}

int silt_set_coupling(silt_sheet* s, int32_t mode, silt_closure* net, float threshold) {
    if (!s) return fail_arg("handle");
    if (mode != SILT_COUPLING_NESTED && mode != SILT_COUPLING_NONE && mode != SILT_COUPLING_CLOSURE)
        return fail_arg("coupling mode");
    if (mode == SILT_COUPLING_CLOSURE && !net) return fail_arg("closure coupling needs a network");
    if (!(threshold >= 0.0f) || !std::isfinite(threshold)) return fail_arg("closure threshold");
    if (net && net->device != s->cfg.device) return fail_arg("closure network on another device");
    if (mode == SILT_COUPLING_CLOSURE && !s->clos) {
        s->clos = new silt::closure::Runner();
        CK(s->clos->reserve(1));
    }
    s->coupling = mode;
    s->net = mode == SILT_COUPLING_CLOSURE ? net : nullptr;
    s->clos_threshold = threshold;
    s->clos_fallback_next = false;
    s->fine.patches_off = mode != SILT_COUPLING_NESTED;
    s->fine.coarse_shove_off = false;
    return SILT_OK;
}

int silt_closure_features(silt_sheet* s, silt_closure* net, void* x, int32_t* origin) {
    if (!s || !net || !x || !origin) return fail_arg("closure_features");
    if (((uintptr_t)x & 15u) != 0) return fail_arg("closure_features: x must be 16-byte aligned");
    if (!s->clos) {
        s->clos = new silt::closure::Runner();
        CK(s->clos->reserve(1));
    }
    const silt::closure::FeatureJob F = closure_job(s, s->pushes);
    CK(s->clos->features({F}, net->net, s->st));
    CK(cudaMemcpyAsync(x, s->clos->x, (size_t)SILT_CLOSURE_CROP * SILT_CLOSURE_CROP * SILT_CLOSURE_CIN * 2,
                       cudaMemcpyDeviceToDevice, s->st));
    origin[0] = F.ci0;
    origin[1] = F.cj0;
    return SILT_OK;
}

int silt_get_closure_stats(silt_sheet* s, silt_closure_stats* out) {
    if (!s || !out) return fail_arg("closure_stats");
    if (s->clos) {
        CK(cudaStreamSynchronize(s->st));
        std::vector<float> r;
        double moved = 0.0;
        if (s->clos->poll(r, &moved) && !r.empty()) {
            s->cstats.last_residual = r[0];
            s->cstats.moved_m3 = moved;
            s->clos_fallback_next = r[0] > s->clos_threshold;
        }
    }
    *out = s->cstats;
    return SILT_OK;
}

int silt_get_ledger(silt_sheet* s, silt_ledger* out) {
    if (!s || !out) return fail_arg("ledger");
    double w = 0.0, sl = 0.0;
    if (s->ledger_fresh) {
        CK(cudaMemcpyAsync(s->h_acc, s->d_acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    } else {
        CK(silt::op_sum2(s->H(0), s->H(1), s->n, s->d_acc + 2, s->st, s->d_sum_scratch));
        CK(cudaMemcpyAsync(s->h_acc, s->d_acc + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    }
    CK(silt::op_sum2(s->tr.susp[0], s->tr.turbid[0], s->n, s->d_acc + 4, s->st, s->d_sum_scratch));
    CK(cudaMemcpyAsync(s->h_acc + 4, s->d_acc + 4, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    // Every copy is queued first and the stream waited on once.
    int rc = silt::fine::books_enqueue(s->fine, s);
    if (rc) return rc;
    CK(cudaMemcpyAsync(s->h_flags, s->d_u32 + 2, 14 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if ((rc = check_substep_overflow(s))) return rc;
    const double* bk = silt::fine::books_host(s->fine);
    const double spray = bk[0], park_w = bk[1], park_s = bk[2], cut = bk[3], reach = bk[4], eroded = bk[5],
                 rounding = bk[6];
    const double area = (double)s->cfg.cell * (double)s->cfg.cell;
    w = s->h_acc[0] * area;
    sl = s->h_acc[1] * area;
    out->water_m3 = w;
    out->slurry_m3 = sl;
    out->frozen_water_m3 = park_w;
    out->frozen_slurry_m3 = park_s;
    out->spray_m3 = spray;
    out->opened_m3 = s->opened_m3 + eroded;
    out->total_m3 = w + sl + park_w + park_s + spray + reach;
    out->cut_m3 = cut;
    out->reach_m3 = reach;
    out->round_m3 = rounding;
    // The tracers' books take the reference's f32 cell area (cell * cell in
    // f32), so the standing load and its running books use one area.
    const double tracer_area = (double)(s->cfg.cell * s->cfg.cell);
    out->suspended_m3 = s->h_acc[4] * tracer_area;
    out->settled_suspended_m3 = bk[8];
    out->frozen_suspended_m3 = bk[11];
    out->entrained_m3 = bk[7];
    out->turbid_m3 = s->h_acc[5] * tracer_area;
    out->turbid_settled_m3 = bk[10];
    out->frozen_turbid_m3 = bk[12];
    out->stirred_m3 = bk[9];
    return SILT_OK;
}

int silt_get_coarse_cell(silt_sheet* s, int32_t i, int32_t j, silt_coarse_cell* out) {
    if (!s || !out) return fail_arg("coarse_cell");
    if (i < 0 || j < 0 || i >= s->res || j >= s->res) return SILT_OK_NOOP;
    int rc = flush_cut(s);
    if (rc) return rc;
    size_t idx = (size_t)j * s->res + i;
    float vals[10];
    const float* src[10] = {s->bed + idx, s->H(0) + idx, s->H(1) + idx, s->moisture + idx,
                            s->U(0) + idx, s->V(0) + idx, s->U(1) + idx, s->V(1) + idx,
                            s->tr.susp[0] + idx, s->tr.turbid[0] + idx};
    for (int k = 0; k < 10; ++k) CK(cudaMemcpyAsync(&vals[k], src[k], 4, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    using silt::host::finite0;
    float water_m = finite0(vals[1]), slurry_m = finite0(vals[2]);
    float film = water_m + slurry_m;
    float u = 0.0f, v = 0.0f;
    if (!(film < 1.0e-5f)) {
        u = finite0((vals[4] * water_m + vals[6] * slurry_m) / film);
        v = finite0((vals[5] * water_m + vals[7] * slurry_m) / film);
    }
    out->x = s->origin[0] + ((float)i + 0.5f) * s->cfg.cell;
    out->z = s->origin[1] + ((float)j + 0.5f) * s->cfg.cell;
    out->bed_m = finite0(vals[0]);
    out->water_m = water_m;
    out->slurry_m = slurry_m;
    out->moisture = finite0(vals[3]);
    out->u = u;
    out->v = v;
    // Suspended load plus stirred silt over the water column (:7024-7032).
    out->turbidity = water_m < 1.0e-5f
                         ? 0.0f
                         : silt::host::rclamp((std::fmax(finite0(vals[8]), 0.0f) + std::fmax(finite0(vals[9]), 0.0f)) /
                                                  water_m,
                                              0.0f, 1.0f);
    return SILT_OK;
}

int silt_export_maps(silt_sheet* s, float* height, float* vel_u, float* vel_v, float* moisture) {
    if (!s) return fail_arg("handle");
    int rc = silt::fine::restrict_all(s->fine, s);
    if (rc) return rc;
    if ((rc = flush_cut(s))) return rc;
    // Four planes through the two staging buffers, two at a time.
    float* outs[4] = {height, vel_u, vel_v, moisture};
    for (int pass = 0; pass < 2; ++pass) {
        float* d[4] = {nullptr, nullptr, nullptr, nullptr};
        d[pass * 2] = s->staging;
        d[pass * 2 + 1] = s->staging2;
        if (!outs[pass * 2] && !outs[pass * 2 + 1]) continue;
        CK(silt::op_export(s->bed, s->H(0), s->H(1), s->U(0), s->V(0), s->U(1), s->V(1), s->moisture, d[0], d[1],
                           d[2], d[3], s->n, s->st));
        if (outs[pass * 2])
            CK(cudaMemcpyAsync(outs[pass * 2], s->staging, s->n * 4, cudaMemcpyDeviceToHost, s->st));
        if (outs[pass * 2 + 1])
            CK(cudaMemcpyAsync(outs[pass * 2 + 1], s->staging2, s->n * 4, cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    return SILT_OK;
}

int silt_publish_film_flow_device(silt_sheet* s, float* d_film, float* d_flow) {
    if (!s || !d_film || !d_flow) return fail_arg("publish");
    int rc = flush_cut(s);
    if (rc) return rc;
    CK(silt::op_publish(s->H(0), s->H(1), s->U(0), s->V(0), s->U(1), s->V(1), s->tr.susp[0], s->tr.turbid[0], d_film,
                        d_flow, s->n, s->st));
    return SILT_OK;
}

int silt_publish_film_flow(silt_sheet* s, float* film, float* flow) {
    if (!s || !film || !flow) return fail_arg("publish");
    float* d_film = nullptr;
    float* d_flow = nullptr;
    CK(cudaMallocAsync((void**)&d_film, s->n * 2 * sizeof(float), s->st));
    CK(cudaMallocAsync((void**)&d_flow, s->n * 4 * sizeof(float), s->st));
    int rc = silt_publish_film_flow_device(s, d_film, d_flow);
    if (rc == SILT_OK) {
        CK(cudaMemcpyAsync(film, d_film, s->n * 2 * sizeof(float), cudaMemcpyDeviceToHost, s->st));
        CK(cudaMemcpyAsync(flow, d_flow, s->n * 4 * sizeof(float), cudaMemcpyDeviceToHost, s->st));
    }
    cudaFreeAsync(d_film, s->st);
    cudaFreeAsync(d_flow, s->st);
    CK(cudaStreamSynchronize(s->st));
    return rc;
}

int silt_non_finite_count(silt_sheet* s, uint32_t* out) {
    if (!s || !out) return fail_arg("non_finite_count");
    const float* planes[8] = {s->H(0), s->H(1), s->U(0), s->V(0), s->U(1), s->V(1), s->bed, s->moisture};
    CK(cudaMemcpyAsync(s->d_planes, planes, sizeof planes, cudaMemcpyHostToDevice, s->st));
    CK(silt::op_non_finite(s->d_planes, 8, s->n, s->d_u32 + 3, s->st));
    unsigned int c = 0;
    CK(cudaMemcpyAsync(&c, s->d_u32 + 3, 4, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    *out = c;
    return SILT_OK;
}

int silt_spray_m3(silt_sheet* s, double* out) {
    if (!s || !out) return fail_arg("spray_m3");
    double pw = 0.0, ps = 0.0;
    int rc = silt::fine::ledger_parts(s->fine, s, out, &pw, &ps);
    return rc;
}

int silt_window_bounds(silt_sheet* s, float* ox, float* oz, float* extent) {
    if (!s) return fail_arg("handle");
    if (ox) *ox = s->origin[0];
    if (oz) *oz = s->origin[1];
    if (extent) *extent = (float)s->res * s->cfg.cell;
    return SILT_OK;
}

static float* plane_of(silt_sheet* s, int which) {
    switch (which) {
        case 0: return s->H(0);
        case 1: return s->H(1);
        case 2: return s->U(0);
        case 3: return s->V(0);
        case 4: return s->U(1);
        case 5: return s->V(1);
        case 6: return s->bed;
        case 7: return s->moisture;
        case 8: return s->tr.foam[0];
        case 9: return s->tr.turbid[0];
        case 10: return s->tr.susp[0];
        default: return nullptr;
    }
}

int silt_read_plane(silt_sheet* s, int32_t which, float* host) {
    if (!s || !host) return fail_arg("read_plane");
    float* p = plane_of(s, which);
    if (!p) return fail_arg("plane index");
    int rc = flush_cut(s);
    if (rc) return rc;
    CK(cudaMemcpyAsync(host, p, s->n * 4, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return SILT_OK;
}

int silt_write_plane(silt_sheet* s, int32_t which, const float* host) {
    if (!s || !host) return fail_arg("write_plane");
    float* p = plane_of(s, which);
    if (!p) return fail_arg("plane index");
    int rc = flush_cut(s);
    if (rc) return rc;
    s->tr_poke = true;  // a tracer plane, or the water they ride on, changed outside a step
    CK(cudaMemcpyAsync(p, host, s->n * 4, cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (which >= 2 && which <= 5) {
        float m = 0.0f;
        for (size_t i = 0; i < s->n; ++i)
            if (std::isfinite(host[i])) m = std::max(m, fabsf(host[i]));
        s->vmax_bound = std::max(s->vmax_bound, m * 1.4142137f);
    }
    s->ledger_fresh = false;
    return tiles_dirty(s);
}

int silt_plane_device(silt_sheet* s, int32_t which, void** out) {
    if (!s || !out) return fail_arg("plane_device");
    float* p = plane_of(s, which);
    if (!p) return fail_arg("plane index");
    int rc = flush_cut(s);
    if (rc) return rc;
    *out = p;
    return SILT_OK;
}

int silt_sheet_copy_state(silt_sheet* dst, silt_sheet* src) {
    if (!dst || !src || dst == src) return fail_arg("copy_state");
    if (dst->res != src->res || dst->cfg.device != src->cfg.device) return fail_arg("copy_state: different windows");
    int rc = flush_cut(src);
    if (rc) return rc;
    CK(cudaStreamSynchronize(src->st));
    rc = flush_cut(dst);
    if (rc) return rc;
    for (int which = 0; which < 8; ++which)
        CK(cudaMemcpyAsync(plane_of(dst, which), plane_of(src, which), dst->n * 4, cudaMemcpyDeviceToDevice, dst->st));
    CK(cudaMemcpyAsync(dst->grain, src->grain, dst->n, cudaMemcpyDeviceToDevice, dst->st));
    dst->vmax_bound = src->vmax_bound;
    dst->moisture_ambient = src->moisture_ambient;
    dst->ledger_fresh = false;
    return tiles_dirty(dst);
}

int silt_check_fixed_division(float d, unsigned long long* counts6, void* stream) {
    if (!counts6 || !(d > 0.0f) || !std::isfinite(d)) return fail_arg("check_fixed_division");
    CK(silt::check_fixed_div(d, counts6, (cudaStream_t)stream));
    return SILT_OK;
}

int silt_known_exact_divisors(float* out, int32_t cap) {
    if (cap < 0 || (cap > 0 && !out)) return fail_arg("known_exact_divisors");
    return silt::known_exact_divisors(out, cap);
}

int silt_fine_water_debug(silt_sheet* s, const silt_tire_push* tires, int32_t n, int32_t patch, float* host,
                          float* origin2) {
    if (!s || (n > 0 && !tires) || !host) return fail_arg("fine_water_debug");
    std::vector<silt_tire_push> ps(tires, tires + n);
    return silt::fine::debug_patch(s->fine, s, ps, patch, host, origin2);
}

int silt_near_tiles(silt_sheet* s, int32_t* out) {
    if (!s || !out) return fail_arg("near_tiles");
    return silt::fine::near_tiles(s->fine, s, out);
}

int silt_set_step_timing(silt_sheet* s, int32_t on) {
    if (!s) return fail_arg("handle");
    CK(cudaStreamSynchronize(s->st));
    if (s->tile_mem) {
        CK(cudaMemsetAsync(s->d_u32 + 4, 0, 16, s->st));
        CK(cudaMemsetAsync(&s->sweep_state()->passes_max, 0, 3 * sizeof(unsigned int), s->st));
        CK(cudaMemsetAsync(&s->sweep_state()->solves, 0, 2 * sizeof(unsigned int), s->st));
    }
    for (cudaEvent_t e : s->ev_used) s->ev_pool.push_back(e);
    s->ev_used.clear();
    memset(&s->parts, 0, sizeof s->parts);
    s->timing = on != 0;
    return SILT_OK;
}

int silt_get_step_parts(silt_sheet* s, silt_step_parts* out) {
    if (!s || !out) return fail_arg("step_parts");
    CK(cudaStreamSynchronize(s->st));
    for (size_t k = 0; k + 2 < s->ev_used.size(); k += 3) {
        float a = 0.0f, b = 0.0f;
        CK(cudaEventElapsedTime(&a, s->ev_used[k], s->ev_used[k + 1]));
        CK(cudaEventElapsedTime(&b, s->ev_used[k + 1], s->ev_used[k + 2]));
        s->parts.force_ms += a;
        s->parts.transport_ms += b;
    }
    for (cudaEvent_t e : s->ev_used) s->ev_pool.push_back(e);
    s->ev_used.clear();
    if (s->tile_mem) {
        // Cells of the tiles the force kernel stepped (32 x 32 per tile layer).
        unsigned long long stepped[2] = {0, 0};
        CK(cudaMemcpy(stepped, s->d_u32 + 4, 16, cudaMemcpyDeviceToHost));
        s->parts.force_cells = (int64_t)(stepped[0] + stepped[1]) * silt::GRID_TILE * silt::GRID_TILE;
        s->parts.force_cells_water = (int64_t)stepped[0] * silt::GRID_TILE * silt::GRID_TILE;
        silt::SweepState st;
        CK(cudaMemcpy(&st, s->sweep_state(), sizeof st, cudaMemcpyDeviceToHost));
        s->parts.sweep_launches = st.launches;
        s->parts.sweep_passes_max = st.passes_max;
        s->parts.sweep_fallbacks = st.fallbacks;
        s->parts.sweep_solves = st.solves;
        s->parts.sweep_local_passes = st.local_passes;
    }
    *out = s->parts;
    return SILT_OK;
}

int silt_set_fine_sub_cap(silt_sheet* s, float cap) {
    if (!s) return fail_arg("handle");
    s->fine.sub_cap = std::isfinite(cap) ? silt::host::rclamp(cap, 1.0f, 8.0f) : 8.0f;
    return SILT_OK;
}

int silt_set_fine_pace(silt_sheet* s, int32_t pace) {
    if (!s) return fail_arg("handle");
    s->fine.pace = std::min(std::max(pace, 0), 3);
    return SILT_OK;
}

int silt_set_near_field(silt_sheet* s, int32_t on) {
    if (!s) return fail_arg("handle");
    return silt::fine::set_near_field(s->fine, s, on != 0);
}

int silt_set_confinement(silt_sheet* s, int32_t form) {
    if (!s) return fail_arg("handle");
    if (form != SILT_CONFINE_SWEEP && form != SILT_CONFINE_SNAPSHOT) return fail_arg("confinement form");
    s->confine = form;
    return SILT_OK;
}

// ---------------------------------------------------------------- batched windows
}  // extern "C"

// Host threads for the per-window parts of a batched step (tire pushes,
// inflow, the nested patches: host planning and a dozen small launches per
// window with tires). Each worker owns a stream; its windows' work goes there
// between an event from the batch stream and one back to it.
struct BatchWorkers {
    std::vector<std::thread> threads;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> done;
    std::vector<int> rc;
    std::vector<std::string> err;
    std::vector<unsigned long long> launches;
    std::mutex m;
    std::condition_variable go, finished;
    std::function<void(int)> job;
    unsigned long long gen = 0;
    int pending = 0;
    bool quit = false;
    int device = 0;

    void loop(int k) {
        cudaSetDevice(device);
        unsigned long long seen = 0;
        for (;;) {
            std::function<void(int)> f;
            {
                std::unique_lock<std::mutex> lk(m);
                go.wait(lk, [&] { return quit || gen != seen; });
                if (quit) return;
                seen = gen;
                f = job;
            }
            const unsigned long long l0 = silt::t_kernel_launches;
            f(k);
            {
                std::lock_guard<std::mutex> lk(m);
                launches[k] += silt::t_kernel_launches - l0;
                if (--pending == 0) finished.notify_all();
            }
        }
    }
    // Runs f(k) on every worker and returns when all are done.
    void run(std::function<void(int)> f) {
        std::unique_lock<std::mutex> lk(m);
        job = std::move(f);
        pending = (int)threads.size();
        ++gen;
        go.notify_all();
        finished.wait(lk, [&] { return pending == 0; });
    }
    ~BatchWorkers() {
        {
            std::lock_guard<std::mutex> lk(m);
            quit = true;
        }
        go.notify_all();
        for (auto& t : threads) t.join();
        for (cudaStream_t st : streams) cudaStreamDestroy(st);
        for (cudaEvent_t e : done) cudaEventDestroy(e);
    }
};

// Batch autotuner state (silt_batch_autotune).
struct BatchTuner {
    static constexpr int KNOBS = 3, REPS = 2, SKIP = 6;
    bool active = false;
    int knob = 0, cand = 0, rep = 0, skip = SKIP;
    float best_rep = 0.0f;     // the current candidate's best step so far
    cudaEvent_t e0[REPS] = {}, e1[REPS] = {};
    std::vector<float> cand_ms;  // the current knob's candidates' best times
};

struct silt_batch {
    std::vector<silt_sheet*> sheets;
    silt_batch_tune tune = {2, 148 * 4, 2368, 0, 0, {}};  // launch settings in force
    BatchTuner tuner;
    BatchWorkers* workers = nullptr;
    silt::fine::FineBatch* fine = nullptr;  // staging of the batched nested-patch launches
    cudaEvent_t ev_start = nullptr;
    cudaStream_t st = nullptr;
    int device = 0;
    int max_tiles = 0;              // the largest window's tile count per layer
    int* list = nullptr;            // tile list of every window, and each entry's window
    int* entry_win = nullptr;
    int* count = nullptr;           // two count slots, used alternately by successive substeps
    unsigned long long seq = 0;
    // Substep descriptors in a ring of slots, reused WS_SLOTS steps later, so
    // the wait for a slot's earlier copy finds it done and the host plans ahead.
    static constexpr int WS_SLOTS = 4;
    silt::WindowSubstep* d_ws[WS_SLOTS] = {};
    silt::WindowSubstep* h_ws[WS_SLOTS] = {};  // pinned
    size_t ws_cap[WS_SLOTS] = {};
    cudaEvent_t ev[WS_SLOTS] = {};
    int flip = 0;
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool, ev_used;  // groups of three: start, after force, after transport
    silt_step_parts parts;
    // The learned closure over the windows coupled by it: one crop per window
    // with tires, every crop through the same launches.
    silt::closure::Runner* clos = nullptr;
    // Ledger gather: per window the depth sums and the books, one copy back.
    const double** d_ledger_src = nullptr;  // [0, n) depth sums, [n, 2n) books
    double* d_ledgers = nullptr;            // 16 doubles per window
    silt::tracers::Runner tr_run;           // the windows' tracer launches
    const float** d_tr_src = nullptr;       // [0, n) suspended planes, [n, 2n) silt planes
    int* d_tr_cells = nullptr;              // cells per window
    double* d_tr_sum = nullptr;             // the ordered tracer sums' scratch
    double* h_ledgers = nullptr;            // pinned
    // Every window's 14 flag words (d_u32[2, 16)) in one block, one copy back.
    const unsigned int** d_flag_src = nullptr;
    unsigned int* d_flags = nullptr;
    unsigned int* h_flags = nullptr;        // pinned
};

namespace {

int batch_free(silt_batch* b) {
    if (!b) return SILT_OK;
    if (b->st) cudaStreamSynchronize(b->st);
    for (int r = 0; r < BatchTuner::REPS; ++r) {
        if (b->tuner.e0[r]) cudaEventDestroy(b->tuner.e0[r]);
        if (b->tuner.e1[r]) cudaEventDestroy(b->tuner.e1[r]);
    }
    if (b->clos) {
        b->clos->release();
        delete b->clos;
    }
    delete b->workers;
    silt::fine::batch_free(b->fine);
    if (b->ev_start) cudaEventDestroy(b->ev_start);
    cudaFree(b->list);
    cudaFree(b->entry_win);
    cudaFree(b->count);
    cudaFree(b->d_ledger_src);
    cudaFree(b->d_ledgers);
    cudaFree(b->d_tr_src);
    cudaFree(b->d_tr_cells);
    cudaFree(b->d_tr_sum);
    b->tr_run.release();
    if (b->h_ledgers) cudaFreeHost(b->h_ledgers);
    cudaFree(b->d_flag_src);
    cudaFree(b->d_flags);
    if (b->h_flags) cudaFreeHost(b->h_flags);
    for (int k = 0; k < silt_batch::WS_SLOTS; ++k) {
        cudaFree(b->d_ws[k]);
        if (b->h_ws[k]) cudaFreeHost(b->h_ws[k]);
        if (b->ev[k]) cudaEventDestroy(b->ev[k]);
    }
    for (cudaEvent_t e : b->ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : b->ev_used) cudaEventDestroy(e);
    delete b;
    return SILT_OK;
}

cudaEvent_t batch_event(silt_batch* b) {
    cudaEvent_t e = nullptr;
    if (b->ev_pool.empty()) {
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    } else {
        e = b->ev_pool.back();
        b->ev_pool.pop_back();
    }
    b->ev_used.push_back(e);
    return e;
}

// Per window of the batch: whether its nested patches are laid this step and
// whether the closure corrects it (the residual estimates of the last
// correction decide the fallbacks, as in the single-window step).
int batch_closure_begin(silt_batch* b, std::vector<int>& net_win, std::vector<silt::closure::FeatureJob>& feats,
                        const silt_closure** net) {
    std::vector<float> r;
    std::vector<int> wins;
    double moved = 0.0;
    if (b->clos && b->clos->poll(r, &moved, &wins))
        for (size_t k = 0; k < r.size() && k < wins.size(); ++k) {
            silt_sheet* s = b->sheets[wins[k]];
            s->cstats.last_residual = r[k];
            s->clos_fallback_next = r[k] > s->clos_threshold;
        }
    for (int w = 0; w < (int)b->sheets.size(); ++w) {
        silt_sheet* s = b->sheets[w];
        s->fine.patches_off = s->coupling != SILT_COUPLING_NESTED;
        s->fine.coarse_shove_off = false;
        if (s->coupling != SILT_COUPLING_CLOSURE || s->pushes.empty()) continue;
        if (s->clos_fallback_next) {
            s->clos_fallback_next = false;
            s->fine.patches_off = false;
            s->cstats.fallback_steps += 1;
            continue;
        }
        if (*net && *net != s->net) return fail_arg("batch: closure windows must share one network");
        *net = s->net;
        s->fine.coarse_shove_off = true;
        s->cstats.closure_steps += 1;
        net_win.push_back(w);
        feats.push_back(closure_job(s, s->pushes));
    }
    if (!net_win.empty()) {
        if (!b->clos) b->clos = new silt::closure::Runner();
        CK(b->clos->reserve((int)net_win.size()));
    }
    return SILT_OK;
}

// The coarse pairs of every window, `launched` substeps at most, through the
// batched list, speed, force and transport kernels.
// ------------------------------------------------------- batch autotuner
// Candidates of each launch setting, the default first.
const std::vector<int>& tune_cands(int knob) {
    static const std::vector<int> c[BatchTuner::KNOBS] = {{2, 1}, {148 * 4, 148 * 2, 148 * 8}, {2368, 1184, 4736}};
    return c[knob];
}

int& tune_field(silt_batch_tune& t, int knob) {
    return knob == 0 ? t.sweep_ctas_per_sm : (knob == 1 ? t.transport_blocks : t.tracer_blocks);
}

// The size class a choice is kept for: device, window count, coarse cells.
std::string tune_key(silt_batch* b) {
    size_t cells = 0;
    for (silt_sheet* s : b->sheets) cells += s->n;
    char k[96];
    snprintf(k, sizeof k, "dev%d_win%zu_cells%zu", b->device, b->sheets.size(), cells);
    return k;
}

std::mutex g_tune_mu;
std::map<std::string, silt_batch_tune> g_tune_cache;
bool g_tune_loaded = false;

// SILT_TUNE_CACHE: one line per choice, "key sweep_ctas_per_sm transport_blocks tracer_blocks".
void tune_cache_load() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = getenv("SILT_TUNE_CACHE");
    if (!path || !*path) return;
    FILE* f = fopen(path, "r");
    if (!f) return;
    char key[96];
    int a = 0, c = 0, d = 0;
    while (fscanf(f, "%95s %d %d %d", key, &a, &c, &d) == 4) {
        if (a < 1 || a > 2 || c < 1 || d < 1) continue;
        silt_batch_tune t = {a, c, d, 1, 0, {}};
        g_tune_cache[key] = t;
    }
    fclose(f);
}

void tune_cache_store(const std::string& key, const silt_batch_tune& t) {
    g_tune_cache[key] = t;
    const char* path = getenv("SILT_TUNE_CACHE");
    if (!path || !*path) return;
    if (FILE* f = fopen(path, "a")) {
        fprintf(f, "%s %d %d %d\n", key.c_str(), t.sweep_ctas_per_sm, t.transport_blocks, t.tracer_blocks);
        fclose(f);
    }
}

// Before a step's work: set the candidate under trial and mark the start.
// Returns whether this step is timed.
int tune_before(silt_batch* b, bool* timed) {
    *timed = false;
    BatchTuner& T = b->tuner;
    if (!T.active) return SILT_OK;
    if (T.skip > 0) {
        --T.skip;
        return SILT_OK;
    }
    tune_field(b->tune, T.knob) = tune_cands(T.knob)[T.cand];
    for (int r = 0; r < BatchTuner::REPS; ++r) {
        if (!T.e0[r]) CK(cudaEventCreate(&T.e0[r]));
        if (!T.e1[r]) CK(cudaEventCreate(&T.e1[r]));
    }
    CK(cudaEventRecord(T.e0[T.rep], b->st));
    *timed = true;
    return SILT_OK;
}

// After a timed step: once a candidate has run its steps, keep its best
// time; once a setting's candidates are done, fix the fastest.
int tune_after(silt_batch* b) {
    BatchTuner& T = b->tuner;
    CK(cudaEventRecord(T.e1[T.rep], b->st));
    if (++T.rep < BatchTuner::REPS) return SILT_OK;
    T.rep = 0;
    CK(cudaEventSynchronize(T.e1[BatchTuner::REPS - 1]));
    float best = 0.0f;
    for (int r = 0; r < BatchTuner::REPS; ++r) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, T.e0[r], T.e1[r]));
        best = r == 0 ? ms : std::min(best, ms);
    }
    if (b->tune.trials < 16) b->tune.trial_ms[b->tune.trials] = best;
    b->tune.trials += 1;
    T.cand_ms.push_back(best);
    const std::vector<int>& c = tune_cands(T.knob);
    if (++T.cand < (int)c.size()) return SILT_OK;
    const int pick = (int)(std::min_element(T.cand_ms.begin(), T.cand_ms.end()) - T.cand_ms.begin());
    tune_field(b->tune, T.knob) = c[pick];
    T.cand_ms.clear();
    T.cand = 0;
    if (++T.knob < BatchTuner::KNOBS) return SILT_OK;
    T.active = false;
    b->tune.tuned = 1;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_cache_store(tune_key(b), b->tune);
    return SILT_OK;
}

int batch_coarse(silt_batch* b, float dt) {
    const int n = (int)b->sheets.size();
    std::vector<CoarsePlan> plans(n);
    int steps = 1;
    bool device_count = false;
    for (int w = 0; w < n; ++w) {
        int rc = refresh_material(b->sheets[w]);
        if (rc) return rc;
        coarse_plan(b->sheets[w], dt, plans[w]);
        steps = std::max(steps, plans[w].launched);
        device_count = device_count || plans[w].sc.speed2 != nullptr;
    }
    const int slot = b->flip;
    b->flip = (b->flip + 1) % silt_batch::WS_SLOTS;
    const size_t need = (size_t)steps * n;
    // The batch's sweep launches keep their state in the first window's
    // slot, so their errors come back through that window's flags.
    silt::SweepState* sweep = b->sheets[0]->sweep_state();
    bool sweeping = false;
    if (b->ev[slot]) CK(cudaEventSynchronize(b->ev[slot]));  // this slot's last copy has left its pinned half
    if (need > b->ws_cap[slot]) {
        cudaFree(b->d_ws[slot]);
        if (b->h_ws[slot]) cudaFreeHost(b->h_ws[slot]);
        b->d_ws[slot] = nullptr;
        b->h_ws[slot] = nullptr;
        b->ws_cap[slot] = 0;
        CK(cudaMalloc(&b->d_ws[slot], need * sizeof(silt::WindowSubstep)));
        CK(cudaMallocHost(&b->h_ws[slot], need * sizeof(silt::WindowSubstep)));
        b->ws_cap[slot] = need;
    }
    if (!b->ev[slot]) CK(cudaEventCreateWithFlags(&b->ev[slot], cudaEventDisableTiming));
    for (int k = 0; k < steps; ++k)
        for (int w = 0; w < n; ++w) {
            silt_sheet* s = b->sheets[w];
            silt::WindowSubstep& D = b->h_ws[slot][(size_t)k * n + w];
            memset(&D, 0, sizeof D);
            if (k >= plans[w].launched) {
                D.skip = 1;
                continue;
            }
            int all = 0;
            coarse_substep(s, plans[w], dt, k, D.F, D.T, all);
            sweeping = sweeping || D.F.lay[0].sweep || D.F.lay[1].sweep;
            D.cur = s->cur;
            D.all = all;
            D.apply_cut = s->cut_pending ? 1 : 0;
            D.zero_ledger = s->d_acc;
            D.zero_bits = (k == 0 && D.F.sc.speed2) ? s->d_u32 : nullptr;
            s->parts.force_launches += 1;
            coarse_advance(s);
        }
    CK(cudaMemcpyAsync(b->d_ws[slot], b->h_ws[slot], need * sizeof(silt::WindowSubstep), cudaMemcpyHostToDevice,
                       b->st));
    CK(cudaEventRecord(b->ev[slot], b->st));
    for (int k = 0; k < steps; ++k) {
        const silt::WindowSubstep* d = b->d_ws[slot] + (size_t)k * n;
        int* count = b->count + (b->seq & 1);
        int* count_next = b->count + ((b->seq + 1) & 1);
        ++b->seq;
        CK(silt::launch_batch_tile_list(d, n, b->max_tiles, b->list, b->entry_win, count, count_next,
                                        sweeping ? sweep : nullptr, b->st));
        if (k == 0 && device_count) CK(silt::launch_batch_speed2(d, b->list, b->entry_win, count, b->st));
        cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
        if (b->timing) {
            e0 = batch_event(b);
            e1 = batch_event(b);
            e2 = batch_event(b);
            if (!e0 || !e1 || !e2) return fail_cuda(cudaErrorMemoryAllocation, "batch timing events");
            CK(cudaEventRecord(e0, b->st));
        }
        CK(silt::launch_batch_force(d, n, b->list, b->entry_win, count, sweeping ? sweep : nullptr, b->st,
                                    b->tune.sweep_ctas_per_sm));
        if (b->timing) CK(cudaEventRecord(e1, b->st));
        CK(silt::launch_batch_transport(d, b->list, b->entry_win, count, b->st, b->tune.transport_blocks));
        if (b->timing) CK(cudaEventRecord(e2, b->st));
        b->parts.force_launches += 1;
    }
    for (int w = 0; w < n; ++w) b->sheets[w]->vmax_bound = silt::host::kSpeedCap * 1.4142137f;
    return SILT_OK;
}

}  // namespace

extern "C" {

int silt_batch_create(silt_sheet* const* sheets, int32_t n, silt_batch** out) {
    if (!sheets || n <= 0 || !out) return fail_arg("batch");
    *out = nullptr;
    silt_batch* b = new silt_batch();
    memset(&b->parts, 0, sizeof b->parts);
    size_t tiles = 0;
    for (int w = 0; w < n; ++w) {
        silt_sheet* s = sheets[w];
        if (!s) {
            batch_free(b);
            return fail_arg("batch: null sheet");
        }
        if (s->engine != SILT_ENGINE_GRID || !s->tile_mem) {
            batch_free(b);
            return fail_arg("batch: every sheet must step on the grid engine (SILT_ENGINE_GRID)");
        }
        if (w > 0 && (s->st != b->st || s->cfg.device != b->device)) {
            batch_free(b);
            return fail_arg("batch: every sheet must share one device and one stream");
        }
        if (w == 0) {
            b->st = s->st;
            b->device = s->cfg.device;
        }
        const int nt = s->tf.tiles_x * s->tf.tiles_x;
        b->max_tiles = std::max(b->max_tiles, nt);
        tiles += 2 * (size_t)nt;
        b->sheets.push_back(s);
    }
    if (n > 65535) {
        batch_free(b);
        return fail_arg("batch: at most 65535 windows");
    }
    cudaSetDevice(b->device);
    cudaError_t e = cudaMalloc(&b->list, tiles * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->entry_win, tiles * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->count, 2 * sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(b->count, 0, 2 * sizeof(int), b->st);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ledger_src, 2 * (size_t)n * sizeof(double*));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ledgers, 16 * (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_ledgers, 16 * (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_flag_src, (size_t)n * sizeof(unsigned int*));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_flags, 14 * (size_t)n * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_flags, 14 * (size_t)n * sizeof(unsigned int));
    if (e == cudaSuccess) {
        std::vector<const unsigned int*> src(n);
        for (int w = 0; w < n; ++w) src[w] = b->sheets[w]->d_u32 + 2;
        e = cudaMemcpy(b->d_flag_src, src.data(), src.size() * sizeof(unsigned int*), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tr_src, 2 * (size_t)n * sizeof(float*));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tr_cells, (size_t)n * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tr_sum, silt::sum_tracers_scratch_bytes(n));
    if (e == cudaSuccess) e = cudaMemset(b->d_tr_sum, 0, silt::sum_tracers_scratch_bytes(n));
    if (e == cudaSuccess) {
        std::vector<const float*> src(2 * (size_t)n);
        std::vector<int> cells(n);
        for (int w = 0; w < n; ++w) {
            src[w] = b->sheets[w]->tr.susp[0];
            src[n + w] = b->sheets[w]->tr.turbid[0];
            cells[w] = (int)b->sheets[w]->n;
        }
        e = cudaMemcpy(b->d_tr_src, src.data(), src.size() * sizeof(float*), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b->d_tr_cells, cells.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) {
        std::vector<const double*> src(2 * (size_t)n);
        for (int w = 0; w < n; ++w) {
            src[w] = b->sheets[w]->d_acc;
            src[n + w] = silt::fine::books(b->sheets[w]->fine);
        }
        e = cudaMemcpy(b->d_ledger_src, src.data(), src.size() * sizeof(double*), cudaMemcpyHostToDevice);
    }
    b->fine = silt::fine::batch_new();
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_start, cudaEventDisableTiming);
    if (e == cudaSuccess) {
        unsigned hw = std::thread::hardware_concurrency();
        const int k = std::max(1, std::min({8, (int)(hw ? hw : 1), n}));
        BatchWorkers* W = new BatchWorkers();
        W->device = b->device;
        b->workers = W;
        for (int q = 0; q < k && e == cudaSuccess; ++q) {
            cudaStream_t st = nullptr;
            cudaEvent_t ev = nullptr;
            e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (st) W->streams.push_back(st);
            if (ev) W->done.push_back(ev);
        }
        if (e == cudaSuccess) {
            W->rc.assign(k, 0);
            W->err.assign(k, std::string());
            W->launches.assign(k, 0);
            for (int q = 0; q < k; ++q) W->threads.emplace_back([W, q] { W->loop(q); });
        }
    }
    if (e != cudaSuccess) {
        batch_free(b);
        return fail_cuda(e, "batch alloc");
    }
    *out = b;
    return SILT_OK;
}

int silt_batch_destroy(silt_batch* b) { return batch_free(b); }

int silt_batch_step(silt_batch* b, float dt) {
    int rc;
    if (!b) return fail_arg("batch");
    if (!(dt > 0.0f) || !std::isfinite(dt)) {
        for (silt_sheet* s : b->sheets) s->pushes.clear();
        return SILT_OK_NOOP;
    }
    const unsigned long long launches0 = silt::t_kernel_launches;
    using clock = std::chrono::steady_clock;
    const clock::time_point t0 = clock::now();
    clock::time_point tp = t0;
    bool tune_timed = false;
    if ((rc = tune_before(b, &tune_timed))) return rc;
    b->tr_run.blocks_total = b->tune.tracer_blocks;
    // Host time per phase of the step (with timing on): the time since the
    // last mark goes to phase k.
    auto phase = [&](int k) {
        if (!b->timing) return;
        const clock::time_point t = clock::now();
        b->parts.host_phase_ms[k] += std::chrono::duration<double, std::milli>(t - tp).count();
        tp = t;
    };
    const int n = (int)b->sheets.size();
    std::vector<std::vector<silt_tire_push>> ps(n);
    std::vector<silt::fine::StepOut> fo(n);
    BatchWorkers& Wk = *b->workers;
    const int nk = (int)Wk.threads.size();
    std::vector<char> work(n, 0);
    for (auto& c : Wk.launches) c = 0;
    // Windows the learned closure corrects this step: their crops are read
    // from the state before anything of the step touches it.
    std::vector<int> net_win;
    std::vector<silt::closure::FeatureJob> feats;
    const silt_closure* net = nullptr;
    if ((rc = batch_closure_begin(b, net_win, feats, &net))) return rc;
    if (!feats.empty()) CK(b->clos->features(feats, net->net, b->st));
    {
        // entrain_wake (src/fluid_core.rs:6051-6053) of every window with tires, one launch.
        std::vector<silt::tracers::Window> tw;
        for (silt_sheet* s : b->sheets)
            if (s->turbidity && !s->pushes.empty()) tw.push_back(tracer_window(s, s->pushes));
        if (!tw.empty()) CK(silt::tracers::entrain(b->tr_run, tw.data(), (int)tw.size(), dt, b->st));
    }
    phase(0);
    CK(cudaEventRecord(b->ev_start, b->st));  // the workers' streams start after the batch's previous work
    // Each window's tire pushes, inflow and nested-patch planning on the
    // workers (the planning uploads the window's tables on the worker's
    // stream); the patches themselves step in the batched launches below.
    Wk.run([&](int k) {
        Wk.rc[k] = 0;
        cudaStream_t wst = Wk.streams[k];
        cudaError_t e = cudaStreamWaitEvent(wst, b->ev_start, 0);
        for (int w = k; w < n && e == cudaSuccess && Wk.rc[k] == 0; w += nk) {
            silt_sheet* s = b->sheets[w];
            cudaStream_t own = s->st;
            s->st = wst;
            ps[w].clear();
            ps[w].swap(s->pushes);
            bool has = false;
            Wk.rc[k] = step_inflow(s, dt);
            if (!Wk.rc[k]) Wk.rc[k] = silt::fine::batch_prepare(s->fine, s, ps[w], dt, fo[w], &has);
            work[w] = has ? 1 : 0;
            s->st = own;
            if (Wk.rc[k]) Wk.err[k] = silt_last_error();
        }
        if (e == cudaSuccess) e = cudaEventRecord(Wk.done[k], wst);
        if (e != cudaSuccess && Wk.rc[k] == 0) {
            Wk.rc[k] = SILT_ECUDA;
            Wk.err[k] = std::string("batch worker: ") + cudaGetErrorString(e);
        }
    });
    for (int k = 0; k < nk; ++k)
        if (Wk.rc[k]) {
            snprintf(g_err, sizeof g_err, "%s", Wk.err[k].c_str());
            return Wk.rc[k];
        }
    for (int k = 0; k < nk; ++k) CK(cudaStreamWaitEvent(b->st, Wk.done[k], 0));
    phase(1);
    std::vector<silt_sheet*> fs;
    std::vector<silt::fine::Patches*> fp;
    for (int w = 0; w < n; ++w)
        if (work[w]) {
            fs.push_back(b->sheets[w]);
            fp.push_back(&b->sheets[w]->fine);
        }
    if ((rc = silt::fine::batch_launch(b->fine, fs, fp, dt, b->st))) return rc;
    phase(2);
    const clock::time_point t1 = clock::now();
    for (silt_sheet* s : b->sheets)
        if ((rc = wave_step(s, dt))) return rc;
    if ((rc = batch_coarse(b, dt))) return rc;
    for (silt_sheet* s : b->sheets)
        if ((rc = open_water_step(s, dt))) return rc;
    phase(3);
    if ((rc = silt::fine::batch_peel(b->fine, fs, fp, b->st))) return rc;
    phase(4);
    {
        // step_tracers of every window in one launch sequence, the reach, then
        // the suspended load of the windows with turbidity on.
        std::vector<silt::tracers::Window> tw;
        tw.reserve(n);
        for (int w = 0; w < n; ++w) tw.push_back(tracer_window(b->sheets[w], ps[w]));
        CK(silt::tracers::step_tracers(b->tr_run, tw.data(), n, dt, b->st));
        for (silt_sheet* s : b->sheets) {
            s->tr_rescan = false;
            s->tr_poke = true;  // stepped by the batch, which sends no idle reports
        }
        for (silt_sheet* s : b->sheets)
            if ((rc = reach_step(s))) return rc;
        std::vector<silt::tracers::Window> sw;
        for (int w = 0; w < n; ++w)
            if (b->sheets[w]->turbidity) sw.push_back(tracer_window(b->sheets[w], ps[w]));
        if (!sw.empty()) CK(silt::tracers::step_suspended(b->tr_run, sw.data(), (int)sw.size(), dt, b->st));
    }
    phase(5);
    if (!net_win.empty()) {
        std::vector<silt::closure::ApplyJob> A(net_win.size());
        memset(A.data(), 0, A.size() * sizeof(silt::closure::ApplyJob));
        for (size_t k = 0; k < net_win.size(); ++k) {
            A[k].W = silt::fine::view_of(b->sheets[net_win[k]]);
            A[k].ci0 = feats[k].ci0;
            A[k].cj0 = feats[k].cj0;
        }
        CK(b->clos->correct(A, net->net, b->st, net_win));
    }
    for (int w = 0; w < n; ++w) {
        silt_sheet* s = b->sheets[w];
        s->parts.steps += 1;
        s->ledger_fresh = true;
    }
    b->parts.steps += 1;
    b->parts.launches += (int64_t)(silt::t_kernel_launches - launches0);
    for (auto c : Wk.launches) b->parts.launches += (int64_t)c;
    phase(6);
    if (tune_timed && (rc = tune_after(b))) return rc;
    if (b->timing) {
        const clock::time_point t2 = clock::now();
        b->parts.host_step_ms += std::chrono::duration<double, std::milli>(t2 - t0).count();
        b->parts.host_fine_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    return SILT_OK;
}

int silt_batch_get_ledgers(silt_batch* b, silt_ledger* out) {
    if (!b || !out) return fail_arg("batch ledgers");
    const int n = (int)b->sheets.size();
    bool fresh = true;
    for (silt_sheet* s : b->sheets) fresh = fresh && s->ledger_fresh;
    if (!fresh) {  // before the first step: each window sums its planes
        for (int w = 0; w < n; ++w) {
            int rc = silt_get_ledger(b->sheets[w], out + w);
            if (rc) return rc;
        }
        return SILT_OK;
    }
    CK(cudaMemsetAsync(b->d_ledgers, 0, 16 * (size_t)n * sizeof(double), b->st));
    CK(silt::op_sum_tracers(b->d_tr_src, b->d_tr_src + n, b->d_tr_cells, n, b->d_ledgers, b->d_tr_sum, b->st));
    CK(silt::op_gather_ledgers(b->d_ledger_src, b->d_ledger_src + n, n, b->d_ledgers, b->st));
    CK(cudaMemcpyAsync(b->h_ledgers, b->d_ledgers, 16 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, b->st));
    CK(silt::op_gather_words(b->d_flag_src, n, 14, b->d_flags, b->st));
    CK(cudaMemcpyAsync(b->h_flags, b->d_flags, 14 * (size_t)n * sizeof(unsigned int), cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));
    for (int w = 0; w < n; ++w) {
        silt_sheet* s = b->sheets[w];
        memcpy(s->h_flags, b->h_flags + 14 * (size_t)w, 14 * sizeof(unsigned int));
        int rc = check_substep_overflow(s);
        if (rc) return rc;
        const double* g = b->h_ledgers + 16 * (size_t)w;
        const double area = (double)s->cfg.cell * (double)s->cfg.cell;
        silt_ledger& L = out[w];
        L.water_m3 = g[0] * area;
        L.slurry_m3 = g[1] * area;
        L.spray_m3 = g[2];
        L.frozen_water_m3 = g[3];
        L.frozen_slurry_m3 = g[4];
        L.opened_m3 = s->opened_m3;
        L.reach_m3 = g[6];
        L.total_m3 = L.water_m3 + L.slurry_m3 + L.frozen_water_m3 + L.frozen_slurry_m3 + L.spray_m3 + L.reach_m3;
        L.cut_m3 = g[5];
        L.round_m3 = g[7];
        L.entrained_m3 = g[8];
        L.settled_suspended_m3 = g[9];
        L.stirred_m3 = g[10];
        L.turbid_settled_m3 = g[11];
        L.frozen_suspended_m3 = g[12];
        L.frozen_turbid_m3 = g[13];
        L.suspended_m3 = g[14] * (double)(s->cfg.cell * s->cfg.cell);  // the tracers' f32 cell area
        L.turbid_m3 = g[15] * (double)(s->cfg.cell * s->cfg.cell);
    }
    return SILT_OK;
}

int silt_batch_push_tires(silt_batch* b, const int32_t* windows, const silt_tire_push* pushes, int32_t n) {
    if (!b || n < 0 || (n > 0 && (!windows || !pushes))) return fail_arg("batch_push_tires");
    const int nw = (int)b->sheets.size();
    for (int k = 0; k < n; ++k)
        if (windows[k] < 0 || windows[k] >= nw) return fail_arg("batch_push_tires: window index");
    for (int k = 0; k < n; ++k) b->sheets[windows[k]]->pushes.push_back(pushes[k]);
    return SILT_OK;
}

int silt_batch_set_timing(silt_batch* b, int32_t on) {
    if (!b) return fail_arg("batch");
    CK(cudaStreamSynchronize(b->st));
    b->timing = on != 0;
    memset(&b->parts, 0, sizeof b->parts);
    for (cudaEvent_t e : b->ev_used) b->ev_pool.push_back(e);
    b->ev_used.clear();
    for (silt_sheet* s : b->sheets)
        if (s->tile_mem) {
            CK(cudaMemsetAsync(s->d_u32 + 4, 0, 16, b->st));
            CK(cudaMemsetAsync(&s->sweep_state()->passes_max, 0, 3 * sizeof(unsigned int), b->st));
            CK(cudaMemsetAsync(&s->sweep_state()->solves, 0, 2 * sizeof(unsigned int), b->st));
        }
    return SILT_OK;
}

int silt_batch_autotune(silt_batch* b, int32_t on) {
    if (!b) return fail_arg("batch");
    BatchTuner& T = b->tuner;
    if (!on) {
        T.active = false;
        return SILT_OK;
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tune_cache_load();
        auto it = g_tune_cache.find(tune_key(b));
        if (it != g_tune_cache.end()) {
            b->tune = it->second;
            b->tune.tuned = 1;
            b->tune.trials = 0;
            T.active = false;
            return SILT_OK;
        }
    }
    T.active = true;
    T.knob = T.cand = T.rep = 0;
    T.skip = BatchTuner::SKIP;
    T.cand_ms.clear();
    b->tune = silt_batch_tune{2, 148 * 4, 2368, 0, 0, {}};
    return SILT_OK;
}

int silt_batch_get_tune(silt_batch* b, silt_batch_tune* out) {
    if (!b || !out) return fail_arg("batch tune");
    *out = b->tune;
    return SILT_OK;
}

int silt_batch_set_tune(silt_batch* b, const silt_batch_tune* in) {
    if (!b || !in) return fail_arg("batch tune");
    if (in->sweep_ctas_per_sm < 0 || in->sweep_ctas_per_sm > 2 || in->transport_blocks < 0 ||
        in->transport_blocks > 65535 || in->tracer_blocks < 0 || in->tracer_blocks > 65535)
        return fail_arg("batch tune: sweep_ctas_per_sm 1..2, blocks 1..65535 (0 keeps the default)");
    b->tuner.active = false;
    b->tune = silt_batch_tune{in->sweep_ctas_per_sm > 0 ? in->sweep_ctas_per_sm : 2,
                              in->transport_blocks > 0 ? in->transport_blocks : 148 * 4,
                              in->tracer_blocks > 0 ? in->tracer_blocks : 2368, 0, 0, {}};
    return SILT_OK;
}

int silt_batch_get_parts(silt_batch* b, silt_step_parts* out) {
    if (!b || !out) return fail_arg("batch parts");
    CK(cudaStreamSynchronize(b->st));
    for (size_t k = 0; k + 2 < b->ev_used.size(); k += 3) {
        float x = 0.0f, y = 0.0f;
        CK(cudaEventElapsedTime(&x, b->ev_used[k], b->ev_used[k + 1]));
        CK(cudaEventElapsedTime(&y, b->ev_used[k + 1], b->ev_used[k + 2]));
        b->parts.force_ms += x;
        b->parts.transport_ms += y;
    }
    for (cudaEvent_t e : b->ev_used) b->ev_pool.push_back(e);
    b->ev_used.clear();
    b->parts.force_cells = 0;
    b->parts.force_cells_water = 0;
    for (silt_sheet* s : b->sheets) {
        unsigned long long stepped[2] = {0, 0};
        CK(cudaMemcpy(stepped, s->d_u32 + 4, 16, cudaMemcpyDeviceToHost));
        b->parts.force_cells += (int64_t)(stepped[0] + stepped[1]) * silt::GRID_TILE * silt::GRID_TILE;
        b->parts.force_cells_water += (int64_t)stepped[0] * silt::GRID_TILE * silt::GRID_TILE;
        if (s == b->sheets[0]) {
            silt::SweepState st;
            CK(cudaMemcpy(&st, s->sweep_state(), sizeof st, cudaMemcpyDeviceToHost));
            b->parts.sweep_launches = st.launches;
            b->parts.sweep_passes_max = st.passes_max;
            b->parts.sweep_fallbacks = st.fallbacks;
            b->parts.sweep_solves = st.solves;
            b->parts.sweep_local_passes = st.local_passes;
        }
    }
    *out = b->parts;
    return SILT_OK;
}

// ---------------------------------------------------------------- free operator
// Free-operator scratch: up to 512 cells per side, a 4 KiB header holding
// the window job, then the window engine's planes; above, 256 bytes of
// reduction words and the grid engine's three planes.
static size_t step_sheet_scratch(int32_t res) {
    if (res <= 0) return 0;
    size_t n = (size_t)res * res;
    if (res <= silt::window::MAX_RES) return 4096 + (size_t)silt::window::SCRATCH_PLANES * n * sizeof(float);
    const size_t tx = (size_t)(res + silt::GRID_TILE - 1) / silt::GRID_TILE;
    return 256 + 3 * n * sizeof(float) + 12 * tx * tx + 2 * tx * tx * sizeof(int) + 64;
}

size_t silt_step_sheet_scratch_bytes(int32_t res) { return step_sheet_scratch(res); }

// The free operator on the window engine: exact, asynchronous (the substep
// count and the wet test are decided on the device).
static int step_sheet_window(float* h, float* u, float* v, const float* bed, const float* nu, const uint8_t* gate,
                             int32_t res, float cell, float dt, float vorticity, void* scratch, cudaStream_t st) {
    const size_t n = (size_t)res * res;
    silt::window::Job J;
    memset(&J, 0, sizeof J);
    J.h = h;
    J.u = u;
    J.v = v;
    J.bed = bed;
    J.nu_plane = nu;
    J.gate = gate;
    silt::window::attach_scratch(J, reinterpret_cast<float*>((char*)scratch + 4096), n);
    J.res = res;
    J.cell = cell;
    J.div = silt::ieee_cell_divisors(cell);  // no check runs here
    J.dt = dt;
    J.vort = vorticity;
    J.sub_cap = 8.0f;
    J.eps = 1.0e-6f;
    J.nu_mode = silt::window::NU_PLANE;
    J.inner_par = 1;
    J.has_sc2 = 0;
    J.active = 1;
    silt::window::Job* d_job = reinterpret_cast<silt::window::Job*>(scratch);
    // From the stack: the copy is staged before this call returns.
    CK(cudaMemcpyAsync(d_job, &J, sizeof J, cudaMemcpyHostToDevice, st));
    CK(silt::window::launch_window_step(d_job, 1, res, st));
    return SILT_OK;
}

int silt_step_sheet(float* h, float* u, float* v, const float* bed, const float* nu, const uint8_t* gate, int32_t res,
                    float cell, float dt, float vorticity, void* scratch, void* stream) {
    if (!h || !u || !v || !bed || !nu || !scratch || res <= 0) return fail_arg("step_sheet");
    if (!(dt > 0.0f)) return SILT_OK_NOOP;
    if (!(cell > silt::host::kFineCell + 1.0e-6f))
        return fail_arg("step_sheet: 2 cm sheets step through the window's nested patch");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)res * res;
    if (((uintptr_t)scratch & 15) != 0) return fail_arg("step_sheet: scratch must be 16-byte aligned");
    if (res <= silt::window::MAX_RES)
        return step_sheet_window(h, u, v, bed, nu, gate, res, cell, dt, vorticity, scratch, (cudaStream_t)stream);
    // Scratch layout: [0, 32) speed bits, [32, 48) two FP64 sums, [256, ...) u, v, h planes.
    unsigned int* d_bits = (unsigned int*)scratch;
    double* d_sum = (double*)((char*)scratch + 32);
    float* u_mid = (float*)((char*)scratch + 256);
    float* v_mid = u_mid + n;
    float* h_next = v_mid + n;
    // Tile flags after the planes: every tile is stepped on every call (no sweep state).
    silt::TileFlags tf = {};
    {
        const int tx = (res + silt::GRID_TILE - 1) / silt::GRID_TILE;
        const size_t nt = (size_t)tx * tx;
        uint8_t* q = reinterpret_cast<uint8_t*>(h_next + n);
        for (int l = 0; l < 2; ++l)
            for (int b = 0; b < 2; ++b) {
                tf.wet[l][b] = q;
                q += nt;
                tf.zero_uv[l][b] = q;
                q += nt;
                tf.zero_h[l][b] = q;
                q += nt;
            }
        q = (uint8_t*)(((uintptr_t)q + 15) & ~uintptr_t(15));
        tf.list = (int*)q;
        tf.count = tf.list + 2 * nt;
        tf.tiles_x = tx;
    }
    CK(cudaMemsetAsync(d_bits, 0, 32, st));
    CK(silt::launch_max_speed2(h, u, v, n, 1.0e-6f, 0, d_bits, st));
    CK(silt::op_sum2(h, h, n, d_sum, st));
    unsigned int bits = 0;
    double sums[2];
    CK(cudaMemcpyAsync(&bits, d_bits, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(sums, d_sum, 16, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (!(sums[0] > 1.0e-6)) return SILT_OK_NOOP;  // nothing wet (src/fluid_core.rs:873-879)
    float m2;
    memcpy(&m2, &bits, 4);
    float max_s = std::max(0.15f, sqrtf(m2));
    int nsub = (int)silt::host::rclamp(ceilf((dt * max_s) / (0.42f * std::max(cell, 1.0e-3f))), 1.0f, 8.0f);
    float dts = dt / (float)nsub;
    for (int k = 0; k < nsub; ++k) {
        silt::ForceLaunch F;
        silt::TransportLaunch T;
        memset(&F, 0, sizeof F);
        memset(&T, 0, sizeof T);
        silt::LayerParams& P = F.lay[0];
        P.h = h;
        P.bed = bed;
        P.u = u;
        P.v = v;
        P.u_out = u_mid;
        P.v_out = v_mid;
        P.nu_plane = nu;
        P.nu_mode = silt::NU_PLANE;
        P.res = res;
        P.cell = cell;
        // The free operator divides by IEEE division (no check runs here).
        const silt::CellDivisors ieee = silt::ieee_cell_divisors(cell);
        P.div_two = ieee.two;
        P.div_cell2 = ieee.cell2;
        P.div_231 = ieee.d231;
        P.dt = dts;
        P.vort = vorticity;
        P.eps = 1.0e-6f;
        P.project = 1;
        silt::TransportParams& Q = T.lay[0];
        Q.h = h;
        Q.u = u_mid;
        Q.v = v_mid;
        Q.h_out = h_next;
        Q.gate = gate;
        Q.res = res;
        Q.cell = cell;
        Q.div_cell = ieee.cell;
        Q.dt = dts;
        Q.eps = 1.0e-6f;
        F.lay[1].skip = 1;
        T.lay[1].skip = 1;
        F.tf = tf;
        T.tf = tf;
        F.nxt = 1;
        T.nxt = 1;
        silt::SubstepCount host_count;
        memset(&host_count, 0, sizeof host_count);
        CK(silt::launch_tile_list(tf, 0, 1, 1, 0, 1, host_count, nullptr, nullptr, nullptr, st));
        CK(silt::launch_force(F, res, 1, st));
        CK(silt::launch_transport(T, res, 1, st));
        CK(cudaMemcpyAsync(h, h_next, n * 4, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(u, u_mid, n * 4, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(v, v_mid, n * 4, cudaMemcpyDeviceToDevice, st));
        CK(silt::launch_apply_cut(h, u, v, n, 1.0e-6f, st));
    }
    return SILT_OK;
}

// ------------------------------------------------------ free operator, no alloc
// Scratch for silt_step_sheet_noalloc: the layout silt_step_sheet expects
// (a 4 KiB job header, then the window engine's scratch planes) for the
// largest grid it serves. Zero at load, as a caller's scratch must be before
// its first use; the header is rewritten by every call and the planes keep
// what the last call left, like the reference's per-thread sheet scratch.
// Every GPU that loads the library holds this array until the process
// exits. In host code `g_step_sheet_scratch` is only a
// stand-in symbol, never a device address: the address comes from
// cudaGetSymbolAddress, looked up once per device with that device current.
static __device__ __align__(256) unsigned char
    g_step_sheet_scratch[4096 + (size_t)silt::window::SCRATCH_PLANES * SILT_STEP_SHEET_STATIC_MAX_RES *
                                    SILT_STEP_SHEET_STATIC_MAX_RES * sizeof(float)];

static std::mutex g_scratch_mu;
static void* g_scratch_addr[64] = {nullptr};

int silt_step_sheet_noalloc(float* h, float* u, float* v, const float* bed, const float* nu, const uint8_t* gate,
                            int32_t res, float cell, float dt, float vorticity, void* stream) {
    if (res <= 0) return fail_arg("step_sheet_noalloc: res");
    if (res > SILT_STEP_SHEET_STATIC_MAX_RES) {
        snprintf(g_err, sizeof g_err,
                 "invalid argument: step_sheet_noalloc serves grids up to %d cells per side, got %d "
                 "(use silt_step_sheet with caller scratch)",
                 SILT_STEP_SHEET_STATIC_MAX_RES, (int)res);
        return SILT_EINVAL;
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail_arg("step_sheet_noalloc: device ordinal");
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_addr[dev]) {
            // First call on this device (it is current): resolve the array's device address.
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_step_sheet_scratch);
            if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress(g_step_sheet_scratch)");
            g_scratch_addr[dev] = p;
        }
        scratch = g_scratch_addr[dev];
    }
    return silt_step_sheet(h, u, v, bed, nu, gate, res, cell, dt, vorticity, scratch, stream);
}

}  // extern "C"

// Accessors the nested-patch module uses (sheet_fine.cu).
namespace silt {
namespace fine {
SheetView view_of(silt_sheet* s) {
    SheetView w;
    w.st = s->st;
    w.res = s->res;
    w.n = s->n;
    w.cell = s->cfg.cell;
    w.origin[0] = s->origin[0];
    w.origin[1] = s->origin[1];
    for (int l = 0; l < 2; ++l) {
        w.h[l] = s->H(l);
        w.u[l] = s->U(l);
        w.v[l] = s->V(l);
    }
    w.bed = s->bed;
    w.moisture = s->moisture;
    w.grain = s->grain;
    w.d_acc = s->d_acc;
    w.cut_pending = s->cut_pending ? 1 : 0;
    w.tiles_x = s->tile_mem ? s->tf.tiles_x : 0;
    for (int l = 0; l < 2; ++l) {
        w.t_wet[l] = s->tile_mem ? s->tf.wet[l][s->cur] : nullptr;
        w.t_zuv[l] = s->tile_mem ? s->tf.zero_uv[l][s->cur] : nullptr;
        w.t_zh[l] = s->tile_mem ? s->tf.zero_h[l][s->cur] : nullptr;
    }
    return w;
}
int flush(silt_sheet* s) { return flush_cut(s); }
void add_speed(silt_sheet* s, float add) { s->vmax_bound += add; }
void invalidate_ledger(silt_sheet* s) { s->ledger_fresh = false; }
}  // namespace fine
}  // namespace silt
