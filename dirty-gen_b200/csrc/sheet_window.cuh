// Window engine: one CTA steps one layer of one window exactly as the
// reference's step_sheet does (sheet_window.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "sheet_div.cuh"

namespace silt {
namespace window {

constexpr int MAX_RES = 512;  // largest window side the engine steps (tile and row tables)

// NU_TABLE: nu_plane, mob_plane and damp_plane hold each cell's viscosity,
// mobility and damping rate (the material laws applied once beforehand).
enum : int32_t { NU_CONST = 0, NU_PLANE = 1, NU_GRAIN = 2, NU_TABLE = 3 };

// One layer of one window: its planes, its persistent scratch, its options.
struct Job {
    float* h;
    float* u;
    float* v;
    const float* bed;
    const uint8_t* grain;
    const float* moisture;
    const float* nu_plane;
    const float* mob_plane;   // NU_TABLE only
    const float* damp_plane;  // NU_TABLE only
    const uint8_t* gate;   // nullptr: every receiver open
    const uint8_t* solid;  // wall mask (0 open, 1 contact, 2 wall), nullptr: an open sheet
    float* sc[2][5];       // the reference's two scratch sets (sc, sc2): a, b, c, d, e
    float* f1;             // transient: vorticity, edge fluxes
    float* f2;             // transient: edge fluxes, wet-body labels
    float* gs[4];          // Gauss-Seidel confinement: u0, v0, u after gravity, v after gravity
    double* ledger;        // FP64 sum of max(h, 0) after the step, may be nullptr
    double* cut;           // FP64 volume the dry cut removed, m^3 (accumulated), may be nullptr
    double cut_area;       // m^2 of one cell for the cut and rounding books
    double* round;         // FP64 rounding book, m^3 (accumulated), may be nullptr: each updated
                           // cell's f32 change minus the exact sum of its face fluxes
    int32_t res;
    float cell, dt, vort, sub_cap, eps;
    CellDivisors div;      // 2 cell, cell^2, 231, cell (fdiv)
    int32_t nu_mode;
    float nu_c, mob_c;
    float decay_c[9];      // NU_CONST damping factor for 1..8 substeps
    int32_t pace;          // fine-sheet pace (cells of 2 cm)
    int32_t inner_par;     // 1: the free operator (Jacobi confinement on boxes >= 48 x 32)
    int32_t soften_edge;   // soft window band in cells, 0 = off (step_pair's soften_border)
    int32_t open_axis;     // a river reach's band through the window ends: 0 none, 1 rows [open_c0, open_c1)
    int32_t open_c0, open_c1;  // (reach along X), 2 columns (along Z); there only one edge distance softens
    int32_t has_sc2;       // two far-apart boxes step on the second scratch set
    int32_t active;
    int32_t gs_iters;      // out: Gauss-Seidel passes used by the last box (diagnostics)
};

// One cluster of CTAs steps each job, its size chosen from `max_res`, the
// largest window side among the jobs.
cudaError_t launch_window_step(const Job* d_jobs, int njobs, int max_res, cudaStream_t st);
// The same for jobs addressed through a device array of pointers.
cudaError_t launch_window_step_list(Job* const* d_job_list, int njobs, int max_res, cudaStream_t st);
size_t window_static_smem();

// Planes of scratch one window layer needs beyond its own h, u, v: two
// scratch sets of five planes, two transient planes, four for the
// Gauss-Seidel confinement.
constexpr int SCRATCH_PLANES = 16;

// Points a job's scratch at `planes` (SCRATCH_PLANES x res*res floats).
inline void attach_scratch(Job& J, float* planes, size_t n) {
    float* q = planes;
    for (int s = 0; s < 2; ++s)
        for (int a = 0; a < 5; ++a) {
            J.sc[s][a] = q;
            q += n;
        }
    J.f1 = q;
    q += n;
    J.f2 = q;
    q += n;
    for (int k = 0; k < 4; ++k) {
        J.gs[k] = q;
        q += n;
    }
}

}  // namespace window
}  // namespace silt
