// Nested 2 cm patches (placeholder until the patch kernels land): the window
// steps without tires; a tire push is refused.
#include "sheet_fine.cuh"

namespace silt {
namespace fine {

struct PatchState {};

int create(Patches& P, const silt_cfg& cfg, int res, cudaStream_t st) {
    P.layout = cfg.fine_layout;
    P.fres = cfg.fine_res;
    P.fcell = cfg.fine_cell;
    P.tire_r = cfg.tire_r;
    return SILT_OK;
}
void destroy(Patches& P) {}
int restrict_all(Patches& P, silt_sheet* s) { return SILT_OK; }
int step_patches(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& pushes, float dt, StepOut& out) {
    return pushes.empty() ? SILT_OK : SILT_EINVAL;
}
int peel_coarse(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& pushes, StepOut& out) {
    return SILT_OK;
}
int collect_spray(Patches& P, silt_sheet* s, const StepOut& out, silt_spray_event* host, int cap, int* n_out,
                  double* spray_m3) {
    *n_out = 0;
    return SILT_OK;
}
int ledger_parts(Patches& P, silt_sheet* s, double* fine_w, double* fine_s, double* park_w, double* park_s) {
    *fine_w = *fine_s = *park_w = *park_s = 0.0;
    return SILT_OK;
}
int debug_patch(Patches& P, silt_sheet* s, const std::vector<silt_tire_push>& pushes, int patch, float* host,
                float* origin2) {
    return SILT_EINVAL;
}
int near_tiles(Patches& P, silt_sheet* s, int* out) {
    *out = 0;
    return SILT_OK;
}
int set_near_field(Patches& P, silt_sheet* s, bool on) {
    P.near_on = on;
    return SILT_OK;
}

}  // namespace fine
}  // namespace silt
