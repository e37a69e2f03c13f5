// Parked cells of a moving window (src/fluid_core.rs:9004-9222:
// shift_coarse, shift_coarse_scroll, shift_coarse_hash) on the device.
#include "sheet_park.cuh"

#include <cstdio>

#include "launch_count.cuh"

namespace silt {
namespace park {

namespace {

// each_leaving (src/fluid_core.rs:9936-9990) as a set: the columns and rows
// a move by (di, dj) pushes out of an n-cell window.
__device__ __forceinline__ bool leaving(int i, int j, int n, int di, int dj) {
    if (di > 0 && i < min(di, n)) return true;
    if (di < 0 && i >= n - min(-di, n)) return true;
    if (dj > 0 && j < min(dj, n)) return true;
    if (dj < 0 && j >= n - min(-dj, n)) return true;
    return false;
}

__device__ __forceinline__ void book(double w, double s, double* books) {
    for (int o = 16; o > 0; o >>= 1) {
        w += __shfl_down_sync(0xffffffffu, w, o);
        s += __shfl_down_sync(0xffffffffu, s, o);
    }
    if ((threadIdx.x & 31) == 0 && books && (w != 0.0 || s != 0.0)) {
        atomicAdd(&books[1], w);
        atomicAdd(&books[2], s);
    }
}

// The parked stirred silt a slot books: its finite, non-negative part.
__device__ __forceinline__ double silt_of(float t) { return isfinite(t) && t > 0.0f ? (double)t : 0.0; }

// The parked tracer books: suspended solids [11], stirred silt [12]. They take
// the tracers' own cell area, the reference's f32 cell * cell.
__device__ __forceinline__ void book_tracers(double su, double tu, double* books) {
    for (int o = 16; o > 0; o >>= 1) {
        su += __shfl_down_sync(0xffffffffu, su, o);
        tu += __shfl_down_sync(0xffffffffu, tu, o);
    }
    if ((threadIdx.x & 31) == 0 && books && (su != 0.0 || tu != 0.0)) {
        atomicAdd(&books[11], su);
        atomicAdd(&books[12], tu);
    }
}

__global__ void k_park(Planes P, Table T, float ox, float oz, int di, int dj, int all) {
    ::silt::dep_wait();
    const int n = P.res;
    const double area = (double)P.cell * (double)P.cell;
    const double tarea = (double)(P.cell * P.cell);
    double dw = 0.0, ds = 0.0, dsu = 0.0, dtu = 0.0;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < (size_t)n * n;
         c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % n), j = (int)(c / n);
        if (!all && !leaving(i, j, n, di, dj)) continue;
        const unsigned long long k = key_of(world_axis(ox + ((float)i + 0.5f) * P.cell, P.cell),
                                            world_axis(oz + ((float)j + 0.5f) * P.cell, P.cell));
        float v[NVAL] = {P.h[0][c], P.h[1][c], P.u[0][c], P.v[0][c], P.u[1][c], P.v[1][c], P.moisture[c], 0.0f,
                         P.foam[c], P.turbid[c], P.susp[c], 0.0f};
        // park_slot (src/fluid_core.rs:4797-4805; settled dust is off this path).
        const bool keep = v[0] > 1.0e-8f || v[1] > 1.0e-8f || v[10] > 1.0e-8f || fabsf(v[6] - P.ambient) > 6.0e-3f ||
                          v[8] > 1.0e-4f || v[9] > 1.0e-8f;
        if (keep) {
            bool fresh = false;
            const int s = find_or_insert(T, k, &fresh);
            if (s < 0) continue;
            float* slot = T.vals + (size_t)s * NVAL;
            const float ow = fresh ? 0.0f : slot[0], os = fresh ? 0.0f : slot[1];
            const float osu = fresh ? 0.0f : slot[10], otu = fresh ? 0.0f : slot[9];
            for (int q = 0; q < NVAL; ++q) slot[q] = v[q];
            dw += ((double)v[0] - (double)ow) * area;
            ds += ((double)v[1] - (double)os) * area;
            dsu += ((double)v[10] - (double)osu) * tarea;
            dtu += (silt_of(v[9]) - silt_of(otu)) * tarea;
        } else {
            const int s = lookup(T, k);
            if (s < 0) continue;
            const float* slot = T.vals + (size_t)s * NVAL;
            dw -= (double)slot[0] * area;
            ds -= (double)slot[1] * area;
            dsu -= (double)slot[10] * tarea;
            dtu -= silt_of(slot[9]) * tarea;
            T.keys[s] = TOMB;
        }
    }
    book(dw, ds, P.books);
    book_tracers(dsu, dtu, P.books);
}

__global__ void k_scroll(Planes P, int di, int dj) {
    ::silt::dep_wait();
    const int n = P.res;
    for (size_t dst = blockIdx.x * (size_t)blockDim.x + threadIdx.x; dst < (size_t)n * n;
         dst += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(dst % n), j = (int)(dst / n);
        const int si = i + di, sj = j + dj;
        bool keep = false;
        size_t src = 0;
        if (si >= 0 && si < n && sj >= 0 && sj < n) {
            src = (size_t)sj * n + si;
            keep = P.h[0][src] > 1.0e-8f || P.h[1][src] > 1.0e-8f || P.moisture[src] > 1.0e-4f ||
                   P.foam[src] > 1.0e-5f || P.turbid[src] > 1.0e-8f || (P.track_susp && P.susp[src] > 1.0e-8f);
        }
        for (int l = 0; l < 2; ++l) {
            P.h_out[l][dst] = keep ? P.h[l][src] : 0.0f;
            P.u_out[l][dst] = keep ? P.u[l][src] : 0.0f;
            P.v_out[l][dst] = keep ? P.v[l][src] : 0.0f;
        }
        P.moisture_out[dst] = keep ? P.moisture[src] : P.ambient;
        P.foam_out[dst] = keep ? P.foam[src] : 0.0f;
        P.turbid_out[dst] = keep ? P.turbid[src] : 0.0f;
        P.susp_out[dst] = keep && P.track_susp ? P.susp[src] : 0.0f;
    }
}

__global__ void k_restore(Planes P, Table T, float ox, float oz, int di, int dj, int all) {
    ::silt::dep_wait();
    const int n = P.res;
    const double area = (double)P.cell * (double)P.cell;
    const double tarea = (double)(P.cell * P.cell);
    double dw = 0.0, ds = 0.0, dsu = 0.0, dtu = 0.0;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < (size_t)n * n;
         c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % n), j = (int)(c / n);
        if (!all && !leaving(i, j, n, -di, -dj)) continue;
        const unsigned long long k = key_of(world_axis(ox + ((float)i + 0.5f) * P.cell, P.cell),
                                            world_axis(oz + ((float)j + 0.5f) * P.cell, P.cell));
        const int s = lookup(T, k);
        float v[NVAL] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, P.ambient, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (s >= 0) {
            const float* slot = T.vals + (size_t)s * NVAL;
            for (int q = 0; q < NVAL; ++q) v[q] = slot[q];
            T.keys[s] = TOMB;
            dw -= (double)v[0] * area;
            ds -= (double)v[1] * area;
            dsu -= (double)v[10] * tarea;
            dtu -= silt_of(v[9]) * tarea;
        } else if (!all) {
            continue;  // nothing parked here: the scroll left the cell cleared
        }
        P.h[0][c] = v[0];
        P.h[1][c] = v[1];
        P.u[0][c] = v[2];
        P.v[0][c] = v[3];
        P.u[1][c] = v[4];
        P.v[1][c] = v[5];
        P.moisture[c] = v[6];
        P.foam[c] = v[8];
        P.turbid[c] = v[9];
        P.susp[c] = v[10];
    }
    book(dw, ds, P.books);
    book_tracers(dsu, dtu, P.books);
}

__global__ void k_rehash(Table old, Table T) {
    ::silt::dep_wait();
    for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; s < old.cap; s += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long k = old.keys[s];
        if (k == EMPTY || k == TOMB) continue;
        bool fresh = false;
        const int d = find_or_insert(T, k, &fresh);
        if (d < 0) continue;
        for (int q = 0; q < NVAL; ++q) T.vals[(size_t)d * NVAL + q] = old.vals[s * NVAL + q];
    }
}

__global__ void k_clear_keys(unsigned long long* keys, unsigned int cap) {
    ::silt::dep_wait();
    for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; s < cap; s += (size_t)gridDim.x * blockDim.x)
        keys[s] = EMPTY;
}

int grid_for(size_t n) {
    const size_t b = (n + 255) / 256;
    return (int)(b < 148 * 8 ? (b ? b : 1) : 148 * 8);
}

}  // namespace

cudaError_t alloc(Table& T, unsigned int cap, cudaStream_t st) {
    T = Table();
    cudaError_t e = cudaMalloc(&T.keys, (size_t)cap * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&T.vals, (size_t)cap * NVAL * sizeof(float));
    // An empty slot's values are zero, so a slot that deposits add into
    // starts from zero whichever thread inserted its key.
    if (e == cudaSuccess) e = cudaMemsetAsync(T.vals, 0, (size_t)cap * NVAL * sizeof(float), st);
    if (e == cudaSuccess) e = cudaMalloc(&T.used, 2 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemsetAsync(T.used, 0, 2 * sizeof(unsigned int), st);
    if (e != cudaSuccess) {
        release(T);
        return e;
    }
    T.cap = cap;
    ::silt::launch_dep(k_clear_keys, dim3(grid_for(cap)), dim3(256), 0, st, T.keys, cap);
    ::silt::count_launch();
    return cudaGetLastError();
}

void release(Table& T) {
    cudaFree(T.keys);
    cudaFree(T.vals);
    cudaFree(T.used);
    T = Table();
}

cudaError_t rebuild(Table& T, unsigned int cap, cudaStream_t st) {
    Table N;
    cudaError_t e = alloc(N, cap, st);
    if (e != cudaSuccess) return e;
    if (T.cap) {
        ::silt::launch_dep(k_rehash, dim3(grid_for(T.cap)), dim3(256), 0, st, T, N);
        ::silt::count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) {
            release(N);
            return e;
        }
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) {
        release(N);
        return e;
    }
    release(T);
    T = N;
    return cudaSuccess;
}

cudaError_t usage(const Table& T, unsigned int* used, unsigned int* overflow, cudaStream_t st) {
    unsigned int h[2] = {0, 0};
    if (T.cap) {
        cudaError_t e = cudaMemcpyAsync(h, T.used, sizeof h, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
    }
    *used = h[0];
    *overflow = h[1];
    return cudaSuccess;
}

cudaError_t park_cells(const Planes& P, const Table& T, float ox, float oz, int di, int dj, int all, cudaStream_t st) {
    ::silt::launch_dep(k_park, dim3(grid_for((size_t)P.res * P.res)), dim3(256), 0, st, P, T, ox, oz, di, dj, all);
    ::silt::count_launch();
    return cudaGetLastError();
}

cudaError_t scroll_cells(const Planes& P, int di, int dj, cudaStream_t st) {
    ::silt::launch_dep(k_scroll, dim3(grid_for((size_t)P.res * P.res)), dim3(256), 0, st, P, di, dj);
    ::silt::count_launch();
    return cudaGetLastError();
}

cudaError_t restore_cells(const Planes& P, const Table& T, float ox, float oz, int di, int dj, int all,
                          cudaStream_t st) {
    ::silt::launch_dep(k_restore, dim3(grid_for((size_t)P.res * P.res)), dim3(256), 0, st, P, T, ox, oz, di, dj,
                       all);
    ::silt::count_launch();
    return cudaGetLastError();
}

}  // namespace park
}  // namespace silt
