// Parked cells: the window's state that has left it, keyed by world cell
// (src/fluid_core.rs:4763-4805 `Parked`, `park_slot`; :9894 `world_key`), in a
// device hash table so a moving window parks and restores cells with no host
// round trip. Open addressing, linear probing; a removed key leaves a
// tombstone, inserts take only empty slots (so two threads inserting the same
// key cannot both succeed), and the table is rebuilt on the host's request
// once live keys plus tombstones pass half of it.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace silt {
namespace park {

constexpr unsigned long long EMPTY = ~0ull;
constexpr unsigned long long TOMB = ~0ull - 1ull;
// water, slurry, uw, vw, us, vs, moisture, unused, foam, stirred silt, suspended solids, unused
constexpr int NVAL = 12;

struct Table {
    unsigned long long* keys = nullptr;
    float* vals = nullptr;          // NVAL per slot
    unsigned int cap = 0;           // power of two
    unsigned int* used = nullptr;   // [0] slots ever taken (live + tombstones), [1] probe overflow flag
};

__device__ __forceinline__ unsigned long long key_of(int ix, int iz) {
    return ((unsigned long long)(unsigned int)ix << 32) | (unsigned long long)(unsigned int)iz;
}

// world_key (src/fluid_core.rs:9894-9896): floor(x / cell), floor(z / cell)
// as i32 (a saturating cast; NaN gives 0).
__device__ __forceinline__ int world_axis(float p, float cell) {
    const float f = floorf(p / cell);
    if (f != f) return 0;
    if (f >= 2147483648.0f) return 2147483647;
    if (f < -2147483648.0f) return (int)0x80000000u;
    return (int)f;
}

__device__ __forceinline__ unsigned int slot_hash(unsigned long long k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (unsigned int)k;
}

// The slot holding `k`, or -1.
__device__ __forceinline__ int lookup(const Table& T, unsigned long long k) {
    const unsigned int mask = T.cap - 1;
    unsigned int s = slot_hash(k) & mask;
    for (unsigned int probe = 0; probe < T.cap; ++probe, s = (s + 1) & mask) {
        const unsigned long long cur = *(volatile unsigned long long*)&T.keys[s];
        if (cur == k) return (int)s;
        if (cur == EMPTY) return -1;
    }
    return -1;
}

// The slot holding `k`, inserting it into an empty slot when absent (values
// of a new slot are the ones a previous occupant left: the caller writes
// them). *fresh tells whether this call inserted it. -1: the table is full.
__device__ __forceinline__ int find_or_insert(const Table& T, unsigned long long k, bool* fresh) {
    const unsigned int mask = T.cap - 1;
    unsigned int s = slot_hash(k) & mask;
    *fresh = false;
    for (unsigned int probe = 0; probe < T.cap; ++probe, s = (s + 1) & mask) {
        unsigned long long cur = *(volatile unsigned long long*)&T.keys[s];
        if (cur == k) return (int)s;
        if (cur != EMPTY) continue;
        cur = atomicCAS(&T.keys[s], EMPTY, k);
        if (cur == EMPTY) {
            *fresh = true;
            atomicAdd(&T.used[0], 1u);
            return (int)s;
        }
        if (cur == k) return (int)s;
    }
    atomicOr(&T.used[1], 1u);
    return -1;
}

cudaError_t alloc(Table& T, unsigned int cap, cudaStream_t st);
void release(Table& T);
// Rebuilds T at `cap` slots without its tombstones (synchronises st).
cudaError_t rebuild(Table& T, unsigned int cap, cudaStream_t st);
// Slots taken (live + tombstones) and the overflow flag (synchronises st).
cudaError_t usage(const Table& T, unsigned int* used, unsigned int* overflow, cudaStream_t st);

// One window's planes for a move (current buffers, and the buffers a scroll
// writes).
struct Planes {
    float* h[2];
    float* u[2];
    float* v[2];
    float* moisture;
    float* h_out[2];
    float* u_out[2];
    float* v_out[2];
    float* moisture_out;
    // The tracers (src/fluid_core.rs:4763-4782 Parked: foam, turbid, susp),
    // and the planes a scroll writes them to; track_susp is the turbidity
    // switch (a scroll carries the suspended load only with it on).
    float* foam;
    float* turbid;
    float* susp;
    float* foam_out;
    float* turbid_out;
    float* susp_out;
    int track_susp;
    int res;
    float cell;
    float ambient;
    double* books;  // [1] parked water m^3, [2] parked slurry m^3, [11] parked suspended, [12] parked silt
};

// Parks the cells of the window at origin (ox, oz) that leave it when its
// origin moves by (di, dj) cells (all of them when all != 0): cells worth
// keeping are written to the table, the others' keys are removed.
cudaError_t park_cells(const Planes& P, const Table& T, float ox, float oz, int di, int dj, int all, cudaStream_t st);
// shift_coarse_scroll's copy: the overlap moves by (di, dj) into the output
// buffers; cells that bring nothing worth keeping, and cells that enter, are
// cleared (moisture to the ambient value).
cudaError_t scroll_cells(const Planes& P, int di, int dj, cudaStream_t st);
// Restores the cells that enter the window at origin (ox, oz) after a move by
// (di, dj) (all cells when all != 0; then cells with no parked slot are
// cleared) from the table, removing their keys.
cudaError_t restore_cells(const Planes& P, const Table& T, float ox, float oz, int di, int dj, int all,
                          cudaStream_t st);

}  // namespace park
}  // namespace silt
