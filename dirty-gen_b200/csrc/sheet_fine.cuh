// Nested 2 cm patches and their two-way coupling with the coarse window
// (x3-team/Dirty-gen src/fluid_core.rs:8152-8566, src/fluid_core/near.rs).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/silt_sheet.h"
#include "sheet_div.cuh"
#include "sheet_park.cuh"
#include "sheet_walls.cuh"

namespace silt {
namespace fine {

// The coarse window as the patch module sees it (current buffers).
struct SheetView {
    cudaStream_t st;
    int res;
    size_t n;
    float cell;
    float origin[2];
    float* h[2];
    float* u[2];
    float* v[2];
    float* bed;
    float* moisture;
    uint8_t* grain;
    double* d_acc;
    int cut_pending;   // u, v of cells with h < eps still hold their pre-cut values
    // Grid engine tile flags of the current buffers (tiles_x = 0 on the window
    // engine): a kernel that writes a coarse cell marks its tile.
    int tiles_x;
    uint8_t* t_wet[2];
    uint8_t* t_zuv[2];
    uint8_t* t_zh[2];
};

// Marks the tile of coarse cell (i, j) of layer l as possibly wet and not zero.
__device__ __forceinline__ void mark_tile(const SheetView& W, int l, int i, int j) {
    if (!W.tiles_x) return;
    const int t = (j / 32) * W.tiles_x + i / 32;
    W.t_wet[l][t] = 1;
    W.t_zuv[l][t] = 0;
    W.t_zh[l][t] = 0;
}

struct StepOut {
    int spray_events = 0;   // events queued on the device this step
};

struct PatchState;  // device planes of one patch (sheet_fine.cu)

struct Patches {
    int layout = SILT_FINE_MEAN_PATCH;
    int fres = 160;
    float fcell = 0.02f;
    CellDivisors fdivs{};  // the patch step's divisors for fcell (set by create)
    int sub = 10;
    float tire_r = 0.56f;
    float sub_cap = 8.0f;
    int pace = 0;
    bool near_on = true;
    bool patches_off = false;  // lay no patch this step: every tire shoves the coarse cells (closure coupling)
    bool coarse_shove_off = false;  // and not even that: the learned closure carries the tires' effect
    float open_mobility = -1.0f;    // >= 0: open-water mode, the water row's mobility (src/fluid_core.rs:8015-8017)
    const walls::SolidGeom* d_solids = nullptr;  // the walls (silt_set_hydro_solids), device
    int n_solids = 0;
    bool fine_on = false;
    int active = 0;
    std::vector<PatchState*> patches;
    void* impl = nullptr;   // device tables owned by sheet_fine.cu
};

SheetView view_of(silt_sheet* s);
int flush(silt_sheet* s);
// Raises the bound on any cell speed by `add` m/s (a tire shove).
void add_speed(silt_sheet* s, float add);
void invalidate_ledger(silt_sheet* s);

int create(Patches& P, const silt_cfg& cfg, int res, cudaStream_t st);
void destroy(Patches& P);
// restrict_fine (src/fluid_core.rs:8462) when a patch is laid down.
int restrict_all(Patches& P, silt_sheet* s);
// refine, shove, fine pair, fine spray, restrict, shove outside (src/fluid_core.rs:6058-6066).
int step_patches(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& pushes, float dt, StepOut& out);
// peel_spray on the coarse window, held columns skipped (src/fluid_core.rs:6071).
int peel_coarse(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& pushes, StepOut& out);

// Batched windows: step_patches and peel_coarse split so that many windows
// share each launch. batch_prepare (per window, on any host thread, with the
// sheet's stream pointing at that thread's stream) plans the patches and
// uploads the window's tables, or runs the tire-less path; it sets *has_work
// when the window's patches go to the batched launches. batch_launch then
// steps every such window's patches on `st` (after the uploads), and
// batch_peel, after the coarse step, peels their coarse cells.
struct FineBatch;
FineBatch* batch_new();
void batch_free(FineBatch* B);
int batch_prepare(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& pushes, float dt, StepOut& out,
                  bool* has_work);
int batch_launch(FineBatch* B, const std::vector<silt_sheet*>& sheets, const std::vector<Patches*>& patches, float dt,
                 cudaStream_t st);
int batch_peel(FineBatch* B, const std::vector<silt_sheet*>& sheets, const std::vector<Patches*>& patches,
               cudaStream_t st);
int collect_spray(Patches& P, silt_sheet* s, const StepOut& out, silt_spray_event* host, int cap, int* n_out);
// FP64 books kept on the device: spray volume and parked (off-window) water and slurry.
int ledger_parts(Patches& P, silt_sheet* s, double* spray, double* park_w, double* park_s, double* cut = nullptr,
                 double* reach = nullptr, double* eroded = nullptr, double* round = nullptr);
// Queues the copy of all 16 books to their host copy on the sheet's stream
// without waiting: books_host holds them once the stream has reached it.
int books_enqueue(Patches& P, silt_sheet* s);
// The host copy of all 16 books as the last ledger_parts (or books_enqueue,
// after a wait on the stream) brought them.
const double* books_host(Patches& P);
// Device address of the books: [0] spray, [1] parked water, [2] parked slurry,
// [3] dry cut, [4] river reach bank, [5] bed scoured into the slurry (m^3, FP64).
double* books(Patches& P);
// The window's parked cells (allocated on first use).
park::Table& park_table(Patches& P);
// The near field's part of a window move by (di, dj) cells (scroll = false:
// a jump, every tile is released).
int move_window(Patches& P, silt_sheet* s, int di, int dj, bool scroll);
const char* last_error();
int debug_patch(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& pushes, int patch, float* host,
                float* origin2);
int near_tiles(Patches& P, silt_sheet* s, int* out);
int set_near_field(Patches& P, silt_sheet* s, bool on);

}  // namespace fine
}  // namespace silt
