// Per-cell kernels around the sheet step (sheet_ops.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace silt {

cudaError_t op_map_water_bed(const float* bed_in, const float* water_in, float* bed, float* water, float* moisture,
                             uint8_t* grain, size_t n, cudaStream_t st);
cudaError_t op_map_water_velocity(const float* u_in, const float* v_in, const float* water, float* uw, float* vw,
                                  size_t n, cudaStream_t st);
cudaError_t op_paint(float* depth_plane, float* moisture, uint8_t* grain, int res, float cell, float ox, float oz,
                     float x0, float x1, float z0, float z1, float depth, int water, int g, float m, cudaStream_t st);
// lay_slurry_on_water: slurry `depth` on cells with more than 12 mm of water;
// `count` (device) receives how many.
cudaError_t op_lay_on_water(const float* water, float* slurry, float* moisture, uint8_t* grain, size_t n, float depth,
                            int g, unsigned int* count, cudaStream_t st);
cudaError_t op_lay_slurry(const float* depth, float* slurry, float* moisture, uint8_t* grain, size_t n, int g, float m,
                          cudaStream_t st);
cudaError_t op_read_substrate(const float* bed_in, const float* moist_in, const uint8_t* grain_in, float* bed,
                              float* moisture, uint8_t* grain, const float* slurry, size_t n, cudaStream_t st);
cudaError_t op_inflow(float* water, float* uw, float* vw, int cut_pending, int res, int j, int i0, int i1, float add,
                      int tiles_x, uint8_t* t_wet, uint8_t* t_zuv, uint8_t* t_zh, cudaStream_t st);
cudaError_t op_publish(const float* water, const float* slurry, const float* uw, const float* vw, const float* us,
                       const float* vs, const float* susp, const float* turbid, float* film, float* flow, size_t n,
                       cudaStream_t st);
cudaError_t op_export(const float* bed, const float* water, const float* slurry, const float* uw, const float* vw,
                      const float* us, const float* vs, const float* moist, float* height, float* vel_u, float* vel_v,
                      float* moisture, size_t n, cudaStream_t st);
// Blocks of an ordered plane sum; its scratch holds 2 * SUM_BLOCKS doubles and
// a ticket (SUM_SCRATCH_BYTES, zeroed once).
constexpr int SUM_BLOCKS = 1184;
constexpr size_t SUM_SCRATCH_BYTES = (2 * SUM_BLOCKS + 2) * sizeof(double);
// out[0..1] = FP64 sums of max(a, 0) and max(b, 0). With `scratch` the sum
// is ordered (the same bits on every call); without it, blocks add atomically.
cudaError_t op_sum2(const float* a, const float* b, size_t n, double* out, cudaStream_t st, double* scratch = nullptr);
// Every window's suspended and silt column sums into out[16 w + 14, 15], in
// a fixed order; `scratch` (sum_tracers_scratch_bytes(n), zeroed once).
size_t sum_tracers_scratch_bytes(int n);
cudaError_t op_sum_tracers(const float* const* susp, const float* const* turbid, const int* cells, int n, double* out,
                           double* scratch, cudaStream_t st);
// out[16 w + 0..1] = acc[w][0..1] (depth sums), out[16 w + 2..6] = books[w][0..4],
// out[16 w + 7] = books[w][6] (the transport rounding book), out[16 w + 8..13] = books[w][7..12] (tracers).
cudaError_t op_gather_ledgers(const double* const* acc, const double* const* books, int n, double* out,
                              cudaStream_t st);
// out[words w + k] = src[w][k] for k < words: each window's flag words in one block.
cudaError_t op_gather_words(const unsigned int* const* src, int n, int words, unsigned int* out, cudaStream_t st);
cudaError_t op_non_finite(const float* const* planes, int np, size_t n, unsigned int* out, cudaStream_t st);

// Open-water drivers of the coarse water sheet (src/fluid_core.rs:7482-7636).
// eddy: the velocity change of one explicit Laplacian from a snapshot into
// du, dv (k = min(nu_t dt / cell^2, 0.2)). friction: adds du, dv, then (gn2 >
// 0) Manning friction, implicit. diffuse: surface-slope transfers between wet
// neighbours from a snapshot into delta; diffuse_apply adds them and the
// exact depth change to ledger[0]. scratch: 2 res^2 floats.
cudaError_t op_open_water(const float* h, float* u, float* v, const float* bed, int res, float k_visc, float gn2,
                          float dt, float* scratch, cudaStream_t st);
cudaError_t op_diffuse_surface(float* h, const float* bed, int res, float k, float* scratch, double* ledger,
                               cudaStream_t st);

}  // namespace silt
