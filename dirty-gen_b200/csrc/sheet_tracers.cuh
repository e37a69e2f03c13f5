// The sheet's tracers on the coarse window (sheet_tracers.cu): foam, stirred
// silt and wheel-lifted suspended solids (x3-team/Dirty-gen
// src/fluid_core.rs:6136-6800 step_tracers, :8750-9003 step_suspended and
// entrain_wake). They never write depth or velocity; they feed the published
// turbidity and the suspended part of the ledger.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/silt_sheet.h"

namespace silt {
namespace tracers {

// Device state of one window's tracers between launches.
struct State {
    int tspan[4];     // turbid cells above 1e-8 (i0, i1, j0, j1; empty when i0 > i1)
    int live_box[4];  // foam-live cells after the last sync
    int sbox[4];      // suspended cells above 1e-8 after the settle pass
    unsigned int live_foam;   // foam-live cells after the last sync
    unsigned int live_silt;   // some turbid cell above 1e-8 at the start of the tracer step
    unsigned int wet_any;     // the tracer step's wet set is not empty
    unsigned int capped;      // suspended cells booked down onto the water in the last step
};

// One window's tracer planes (res^2 each unless noted) and its books.
struct Planes {
    float* foam[2];     // [0] the field, [1] scratch
    float* turbid[2];
    float* susp[2];
    float* taken;       // suspended solids a cell takes from its neighbours this step
    float* acc;         // 6 planes: each donor's accepted gives (advection x, z; mixing +x, -x, +z, -z)
    uint8_t* mark;      // bit 0 wet, bit 1 shore, bit 2 foam-live
    uint8_t* occ;       // per row and 128-cell segment (cells 128 s .. 128 s + 127): 1 when the wet-set pass
                        // left a wet or foam-live mark in it (res x ceil(res / 128))
    State* st;
    double* books;      // [0] entrained, [1] settled suspended, [2] stirred, [3] settled silt (m^3, FP64)
};

// The coarse window the tracers ride on.
struct Sheet {
    const float* water;
    const float* slurry;
    const float* uw;     // water velocity; cells under eps read 0 while a dry cut is pending
    const float* vw;
    int res;
    float cell;
    float ox, oz;        // window origin, m
    int cut_pending;
    int surface_driven;  // a wave maker or a river reach drives the sheet
};

// One window's part of a tracer launch.
struct Job {
    Sheet S;
    Planes T;
    const silt_tire_push* push;  // this window's tire pushes of the step (device), in push order
    int npush;
    int wake;                    // a tire with speed or slip, or a surface drive
    int pbox[4];                 // the tires' reach boxes (tracer_visit_box's tire part; empty when none)
    int ebox[4];                 // entrain_wake's cells: the union of the tires' wake boxes (empty when none)
    int rescan;                  // the planes were rewritten: scan the silt span before the step
    int susp_on;                 // the suspended load is stepped (turbidity on)
    unsigned int* idle_out;      // device word: after the step, 1 when the tracers have nothing left to do
    int sup_all;                 // something outside the tracer kernels wrote the suspended load (a river inlet)
    float dt, foam_decay, silt_keep;
};

// Host staging of the jobs of a launch sequence: windows and their pushes,
// uploaded once per sequence into a ring of slots. A step uploads up to three
// sequences, so a slot is reused about three steps later and its wait for
// the earlier copy finds it long done: the host runs ahead of the device.
struct Runner {
    static constexpr int SLOTS = 10;
    Job* d_jobs[SLOTS] = {};
    Job* h_jobs[SLOTS] = {};
    silt_tire_push* d_push[SLOTS] = {};
    silt_tire_push* h_push[SLOTS] = {};
    size_t cap_jobs[SLOTS] = {}, cap_push[SLOTS] = {};
    cudaEvent_t ev[SLOTS] = {};
    int next = 0;
    // Blocks of a pass over all the windows of a launch: 8 per SM (measured
    // on config 2 against 16 and 32; any value gives the same planes).
    int blocks_total = 1184;
    void release();
};

// One window of a step: its sheet, planes and pushes (host).
struct Window {
    Sheet S;
    Planes T;
    const silt_tire_push* push;
    int npush;
    int rescan = 0;   // the planes were rewritten since the last tracer step (attach, window move)
    int sup_all = 0;  // a river inlet writes the suspended load outside the tracer kernels
    int susp_on = 0;  // turbidity on: step_suspended follows step_tracers this step
    unsigned int* idle_out = nullptr;  // device word for the idle report (see step_tracers)
};

size_t plane_bytes(int res);  // device bytes of one window's tracer planes
cudaError_t attach(Planes& T, void* mem, int res, double* books, cudaStream_t st);  // zeroes them

// entrain_wake (src/fluid_core.rs:8758-8815) on every window, before the step.
cudaError_t entrain(Runner& R, const Window* w, int n, float dt, cudaStream_t st);
// step_tracers (src/fluid_core.rs:6210-6237) after the coarse pair and its peel.
// A window without turbidity then reports whether it is idle (below).
cudaError_t step_tracers(Runner& R, const Window* w, int n, float dt, cudaStream_t st);
// step_suspended (src/fluid_core.rs:8750-8756 with advect_suspended :8817-9002),
// then every window reports whether it is idle: no live foam, no silt above
// 1e-8 and no suspended load. An idle window whose next step has no wake (no
// tire, no surface drive) and no rewritten planes stays idle through that
// step, whose tracer kernels would change nothing, so the caller may skip
// them; a window stays idle until such a trigger.
cudaError_t step_suspended(Runner& R, const Window* w, int n, float dt, cudaStream_t st);
// Clears the foam-live set (reset_tracer_indices, src/fluid_core.rs:9228-9233) after a window move.
cudaError_t reset_indices(Planes& T, int res, cudaStream_t st);

}  // namespace tracers
}  // namespace silt
