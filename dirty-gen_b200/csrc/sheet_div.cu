// Exhaustive check of the fixed-divisor division against IEEE division.
#include "sheet_div.cuh"

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include "launch_count.cuh"

namespace silt {

namespace {

__global__ void k_check_div(float d, float r, unsigned long long* counts) {
    ::silt::dep_wait();
    unsigned long long local[6] = {0, 0, 0, 0, 0, 0};
    const FixedDiv D{d, r, 1};
    const unsigned long long total = 1ull << 32;
    for (unsigned long long b = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; b < total;
         b += (unsigned long long)gridDim.x * blockDim.x) {
        const float x = __uint_as_float((unsigned int)b);
        const float want = x / d;
        const float got = fdiv(x, D);
        const bool same = __float_as_uint(want) == __float_as_uint(got) || (want != want && got != got);
        if (same) continue;
        local[0] += 1;
        const float ax = fabsf(x);
        if (ax == 0.0f) local[1] += 1;
        else if (ax < 1.17549435e-38f) local[2] += 1;
        else if (!(ax <= 3.40282347e38f)) local[3] += 1;
        else if (fabsf(want) < 1.17549435e-38f) local[4] += 1;
        else local[5] += 1;
    }
    for (int k = 0; k < 6; ++k) {
        unsigned long long v = local[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&counts[k], v);
    }
}

std::mutex g_div_mutex;
std::map<std::pair<int, unsigned int>, int> g_div_exact;  // (device, bits of d) -> exact

// Divisors already known to pass the exhaustive check: the four of each
// standard cell width, 0.2 m (coarse) and 0.02 m (tire sheets), as the float
// products 2 * cell and cell * cell that cell_divisors forms. The check's
// verdict depends only on IEEE single-precision arithmetic (a correctly
// rounded product, fused multiply-add and division, no flush to zero), not
// on the device, so it holds on every GPU; tests/test_gpu_division.py runs
// the full check on each entry to keep the table honest. A divisor outside
// the table is checked once per process and device.
bool known_exact(float d) {
    const float cells[2] = {0.2f, 0.02f};
    for (float c : cells) {
        const float ds[4] = {2.0f * c, c * c, 231.0f, c};
        for (float x : ds)
            if (x == d) return true;
    }
    return false;
}

}  // namespace

int known_exact_divisors(float* out, int cap) {
    const float cells[2] = {0.2f, 0.02f};
    float uniq[8];
    int n = 0;
    for (float c : cells) {
        const float ds[4] = {2.0f * c, c * c, 231.0f, c};
        for (float x : ds) {
            bool seen = false;
            for (int k = 0; k < n; ++k) seen = seen || uniq[k] == x;
            if (!seen) uniq[n++] = x;
        }
    }
    for (int k = 0; k < n && k < cap; ++k) out[k] = uniq[k];
    return n;
}

cudaError_t check_fixed_div(float d, unsigned long long* counts6, cudaStream_t st) {
    unsigned long long* dc = nullptr;
    cudaError_t e = cudaMalloc(&dc, 6 * sizeof(unsigned long long));
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(dc, 0, 6 * sizeof(unsigned long long), st);
    const float r = 1.0f / d;
    if (e == cudaSuccess) {
        ::silt::launch_dep(k_check_div, dim3(148 * 16), dim3(256), 0, st, d, r, dc);
        ::silt::count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(counts6, dc, 6 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(dc);
    return e;
}

FixedDiv fixed_div_for(float d, cudaStream_t st) {
    FixedDiv D{d, 1.0f / d, 0};
    if (!(d > 0.0f) || !std::isfinite(d)) return D;
    int dev = 0;
    cudaGetDevice(&dev);
    unsigned int bits;
    memcpy(&bits, &d, sizeof bits);
    if (known_exact(d)) {
        D.exact = 1;
        return D;
    }
    std::lock_guard<std::mutex> lock(g_div_mutex);
    const auto key = std::make_pair(dev, bits);
    auto it = g_div_exact.find(key);
    if (it != g_div_exact.end()) {
        D.exact = it->second;
        return D;
    }
    unsigned long long c[6] = {1, 0, 0, 0, 0, 0};
    const cudaError_t e = check_fixed_div(d, c, st);
    // Only a completed check is remembered: a failed one (no memory, a call
    // under stream capture) leaves this divisor on IEEE division for now and
    // is retried at the next sheet creation.
    if (e == cudaSuccess) g_div_exact.emplace(key, c[0] == 0 ? 1 : 0);
    else cudaGetLastError();
    D.exact = e == cudaSuccess && c[0] == 0 ? 1 : 0;
    return D;
}

CellDivisors cell_divisors(float cell, cudaStream_t st) {
    CellDivisors D;
    D.two = fixed_div_for(2.0f * cell, st);
    D.cell2 = fixed_div_for(cell * cell, st);
    D.d231 = fixed_div_for(231.0f, st);
    D.cell = fixed_div_for(cell, st);
    return D;
}

}  // namespace silt
