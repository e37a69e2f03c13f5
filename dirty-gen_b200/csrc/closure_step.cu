// The learned closure inside the step: the network input gathered from a
// window's coarse state around its vehicle, the three convolutions, and the
// correction applied as depth moved across coarse faces.
//
// Input channels per crop cell (before normalisation): water depth, slurry
// depth, water u and v (0 where the water is under the dry-cut depth), bed,
// and the tire shove field: for every tire, the shove speed
// `max(speed, 0.4) * (1 - flank^2)` of push_on (src/fluid_core.rs:8169-8239)
// over the cells its shove covers, summed.
//
// Correction: output channels 0..3 (times the output scales) are the depth
// moved across the +x and +z faces of each crop cell for water and slurry
// (m); channels 4..7 the change of water u, v and slurry u, v (m/s) of the
// cells that are wet after the depth moves, clamped like the step's speeds. A face inside the window and the crop moves at most a quarter of its
// donor's depth, so no cell can lose more than it holds; each face's transfer
// is computed once and added to one cell and taken from the other, so the
// window's volume is unchanged up to FP32 rounding of the two depths, and the
// FP64 ledger sums are updated with the exact change of every cell. The part
// of the predicted transfers the limiter removed, over all that was
// predicted, is the crop's residual estimate.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/silt_closure.h"
#include "closure.cuh"
#include "launch_count.cuh"
#include "sheet_math.cuh"

namespace silt {
namespace closure {

namespace {

constexpr int CROP = SILT_CLOSURE_CROP;
constexpr int CROP_CELLS = CROP * CROP;
constexpr float DRY_M = 1.0e-6f;     // the sheet's dry-cut depth
constexpr float DONOR_SHARE = 0.25f; // a face moves at most this share of its donor's depth

__device__ __forceinline__ uint16_t bf16_bits(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }

__global__ void __launch_bounds__(CROP_CELLS) k_features(const FeatureJob* jobs, const float* norm, uint16_t* x) {
    ::silt::dep_wait();
    const FeatureJob& J = jobs[blockIdx.x];
    const int p = threadIdx.x, cx = p % CROP, cy = p / CROP;
    const int i = J.ci0 + cx, j = J.cj0 + cy;
    uint16_t* out = x + ((size_t)blockIdx.x * CROP_CELLS + p) * SILT_CLOSURE_CIN;
    float raw[SILT_CLOSURE_IN_USED];
    const bool in = i >= 0 && j >= 0 && i < J.W.res && j < J.W.res;
    if (in) {
        const size_t c = (size_t)j * J.W.res + i;
        const float hw = J.W.h[0][c];
        raw[0] = hw;
        raw[1] = J.W.h[1][c];
        const bool wet = hw >= DRY_M;
        raw[2] = wet ? J.W.u[0][c] : 0.0f;
        raw[3] = wet ? J.W.v[0][c] : 0.0f;
        raw[4] = J.W.bed[c];
        const float cell = J.W.cell;
        const float x0 = J.W.origin[0] + ((float)i + 0.5f) * cell, z0 = J.W.origin[1] + ((float)j + 0.5f) * cell;
        float shove = 0.0f;
        for (int t = 0; t < J.ntires; ++t) {
            const silt_tire_push& T = J.tires[t];
            const float len = fmaxf(sqrtf(T.forward_x * T.forward_x + T.forward_z * T.forward_z), 1.0e-4f);
            const float fx = T.forward_x / len, fz = T.forward_z / len;
            const float dx = x0 - T.x, dz = z0 - T.z;
            const float along = dx * fx + dz * fz, lat = dx * fz - dz * fx;
            const float half = T.width * 0.65f + cell;
            if (fabsf(lat) > half || along < -T.radius * 1.4f || along > T.radius * 1.1f) continue;
            const float flank = fminf(fmaxf(fabsf(lat) / half, 0.0f), 1.0f);
            shove += fmaxf(T.speed, 0.4f) * (1.0f - flank * flank);
        }
        raw[5] = shove;
    }
    uint32_t packed[SILT_CLOSURE_CIN / 2];
#pragma unroll
    for (int k = 0; k < SILT_CLOSURE_CIN / 2; ++k) {
        float a = 0.0f, b = 0.0f;
        if (in && 2 * k < SILT_CLOSURE_IN_USED) a = (raw[2 * k] - norm[2 * k]) * norm[6 + 2 * k];
        if (in && 2 * k + 1 < SILT_CLOSURE_IN_USED) b = (raw[2 * k + 1] - norm[2 * k + 1]) * norm[6 + 2 * k + 1];
        packed[k] = (uint32_t)bf16_bits(a) | ((uint32_t)bf16_bits(b) << 16);
    }
    uint4* o = reinterpret_cast<uint4*>(out);
    o[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
    o[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
}

__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    return s;  // valid in thread 0
}

__global__ void __launch_bounds__(CROP_CELLS) k_apply(const ApplyJob* jobs, const float* y, const float* norm) {
    ::silt::dep_wait();
    const ApplyJob& J = jobs[blockIdx.x];
    __shared__ float gx[2][CROP_CELLS], gz[2][CROP_CELLS];
    __shared__ double red[CROP_CELLS / 32];
    const int p = threadIdx.x, cx = p % CROP, cy = p / CROP;
    const int res = J.W.res;
    const int i = J.ci0 + cx, j = J.cj0 + cy;
    const bool in = i >= 0 && j >= 0 && i < res && j < res;
    const bool in_x = in && cx + 1 < CROP && i + 1 < res;  // the +x face joins two crop cells of the window
    const bool in_z = in && cy + 1 < CROP && j + 1 < res;
    const size_t c = in ? (size_t)j * res + i : 0;
    const float* yo = y + ((size_t)blockIdx.x * CROP_CELLS + p) * SILT_CLOSURE_COUT;
    float clipped = 0.0f, total = 0.0f;
#pragma unroll
    for (int l = 0; l < 2; ++l) {
        float tx = 0.0f, tz = 0.0f;
        if (in_x) {
            const float raw = yo[2 * l] * norm[12 + 2 * l];
            const float hl = J.W.h[l][c], hr = J.W.h[l][c + 1];
            tx = fminf(fmaxf(raw, -DONOR_SHARE * hr), DONOR_SHARE * hl);
            clipped += fabsf(raw - tx);
            total += fabsf(raw);
        }
        if (in_z) {
            const float raw = yo[2 * l + 1] * norm[12 + 2 * l + 1];
            const float hl = J.W.h[l][c], hu = J.W.h[l][c + res];
            tz = fminf(fmaxf(raw, -DONOR_SHARE * hu), DONOR_SHARE * hl);
            clipped += fabsf(raw - tz);
            total += fabsf(raw);
        }
        gx[l][p] = tx;
        gz[l][p] = tz;
    }
    __syncthreads();
    double change[2] = {0.0, 0.0}, moved = 0.0;
    if (in) {
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const float inflow = (cx > 0 ? gx[l][p - 1] : 0.0f) + (cy > 0 ? gz[l][p - CROP] : 0.0f);
            const float outflow = gx[l][p] + gz[l][p];
            const float d = inflow - outflow;
            moved += (double)fabsf(gx[l][p]) + (double)fabsf(gz[l][p]);
            if (d == 0.0f) continue;
            const float h0 = J.W.h[l][c];
            if (J.W.cut_pending && h0 < DRY_M && d > 0.0f) {
                J.W.u[l][c] = 0.0f;  // the lazy dry cut of a cell that is about to hold water
                J.W.v[l][c] = 0.0f;
            }
            const float h1 = fmaxf(h0 + d, 0.0f);
            J.W.h[l][c] = h1;
            change[l] = (double)h1 - (double)h0;
            if (h1 > 0.0f) mark_tile(J.W, l, i, j);
        }
        // Velocity change of the wet cells, within the step's speed clamp
        // (finite_speed, src/fluid_core.rs:3473).
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            const float h1 = J.W.h[l][c];
            if (!(h1 >= DRY_M)) continue;
            const float du = yo[4 + 2 * l] * norm[16 + 2 * l], dv = yo[5 + 2 * l] * norm[17 + 2 * l];
            if (du == 0.0f && dv == 0.0f) continue;
            J.W.u[l][c] = finite_speed(J.W.u[l][c] + du, kSpeedCap);
            J.W.v[l][c] = finite_speed(J.W.v[l][c] + dv, kSpeedCap);
            mark_tile(J.W, l, i, j);
        }
    }
    const double area = (double)J.W.cell * (double)J.W.cell;
    const double s0 = block_sum(change[0], red);
    const double s1 = block_sum(change[1], red);
    const double sm = block_sum(moved, red);
    const double sc = block_sum((double)clipped, red);
    const double st = block_sum((double)total, red);
    if (p == 0) {
        if (J.W.d_acc) {
            atomicAdd(J.W.d_acc + 0, s0);
            atomicAdd(J.W.d_acc + 1, s1);
        }
        if (J.moved) atomicAdd(J.moved, sm * area);
        if (J.resid) {
            J.resid[0] = (float)sc;
            J.resid[1] = (float)st;
        }
    }
}

}  // namespace

cudaError_t launch_features(const FeatureJob* d_jobs, int n, const float* d_norm, uint16_t* x, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    ::silt::launch_dep(k_features, dim3(n), dim3(CROP_CELLS), 0, st, d_jobs, d_norm, x);
    ::silt::count_launch();
    return cudaGetLastError();
}

cudaError_t launch_apply(const ApplyJob* d_jobs, int n, const float* y, const float* d_norm, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    ::silt::launch_dep(k_apply, dim3(n), dim3(CROP_CELLS), 0, st, d_jobs, y, d_norm);
    ::silt::count_launch();
    return cudaGetLastError();
}

// ---- Staging of per-step job records ---------------------------------------

void Staging::release() {
    for (int k = 0; k < SLOTS; ++k) {
        if (ev[k]) cudaEventSynchronize(ev[k]);
        cudaFree(dev[k]);
        if (host[k]) cudaFreeHost(host[k]);
        if (ev[k]) cudaEventDestroy(ev[k]);
        dev[k] = nullptr;
        host[k] = nullptr;
        ev[k] = nullptr;
        cap[k] = 0;
    }
}

cudaError_t Staging::put(const void* data, size_t bytes, cudaStream_t st, void** out) {
    const int k = flip;
    flip = (flip + 1) % SLOTS;
    cudaError_t e = cudaSuccess;
    if (ev[k]) e = cudaEventSynchronize(ev[k]);  // this slot's last copy has left the pinned buffer
    if (e != cudaSuccess) return e;
    if (bytes > cap[k]) {
        cudaFree(dev[k]);
        if (host[k]) cudaFreeHost(host[k]);
        dev[k] = nullptr;
        host[k] = nullptr;
        cap[k] = 0;
        const size_t want = std::max(bytes * 2, (size_t)4096);
        if ((e = cudaMalloc(&dev[k], want)) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&host[k], want)) != cudaSuccess) return e;
        cap[k] = want;
    }
    if (!ev[k] && (e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming)) != cudaSuccess) return e;
    memcpy(host[k], data, bytes);
    if ((e = cudaMemcpyAsync(dev[k], host[k], bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(ev[k], st)) != cudaSuccess) return e;
    *out = dev[k];
    return cudaSuccess;
}

// ---- Crop runner ------------------------------------------------------------

void Runner::release() {
    for (int k = 0; k < RING; ++k) {
        if (ev[k]) cudaEventSynchronize(ev[k]);
        if (h_resid[k]) cudaFreeHost(h_resid[k]);
        if (h_moved[k]) cudaFreeHost(h_moved[k]);
        if (ev[k]) cudaEventDestroy(ev[k]);
    }
    cudaFree(x);
    cudaFree(a1);
    cudaFree(a2);
    cudaFree(y);
    cudaFree(d_resid);
    cudaFree(d_moved);
    fjobs.release();
    ajobs.release();
    *this = Runner();
}

cudaError_t Runner::reserve(int n) {
    if (n <= cap) return cudaSuccess;
    for (int k = 0; k < RING; ++k)
        if (ev[k]) cudaEventSynchronize(ev[k]);
    cudaFree(x);
    cudaFree(a1);
    cudaFree(a2);
    cudaFree(y);
    cudaFree(d_resid);
    x = a1 = a2 = nullptr;
    y = nullptr;
    d_resid = nullptr;
    for (int k = 0; k < RING; ++k) {
        if (h_resid[k]) cudaFreeHost(h_resid[k]);
        h_resid[k] = nullptr;
    }
    cap = 0;
    read = written;  // estimates still in flight are dropped with their buffers
    const size_t px = (size_t)n * CROP_CELLS;
    cudaError_t e;
    if ((e = cudaMalloc(&x, px * SILT_CLOSURE_CIN * 2)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&a1, px * SILT_CLOSURE_HIDDEN * 2)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&a2, px * SILT_CLOSURE_HIDDEN * 2)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&y, px * SILT_CLOSURE_COUT * sizeof(float))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&d_resid, (size_t)n * 2 * sizeof(float))) != cudaSuccess) return e;
    for (int k = 0; k < RING; ++k) {
        if ((e = cudaMallocHost(&h_resid[k], (size_t)n * 2 * sizeof(float))) != cudaSuccess) return e;
        if (!h_moved[k] && (e = cudaMallocHost(&h_moved[k], sizeof(double))) != cudaSuccess) return e;
        if (!ev[k] && (e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    if (!d_moved) {
        if ((e = cudaMalloc(&d_moved, sizeof(double))) != cudaSuccess) return e;
        if ((e = cudaMemset(d_moved, 0, sizeof(double))) != cudaSuccess) return e;
    }
    cap = n;
    return cudaSuccess;
}

cudaError_t Runner::features(const std::vector<FeatureJob>& jobs, const Net& net, cudaStream_t st) {
    const int n = (int)jobs.size();
    if (n == 0) return cudaSuccess;
    cudaError_t e = reserve(n);
    if (e != cudaSuccess) return e;
    void* d = nullptr;
    if ((e = fjobs.put(jobs.data(), jobs.size() * sizeof(FeatureJob), st, &d)) != cudaSuccess) return e;
    return launch_features(static_cast<const FeatureJob*>(d), n, net.norm, x, st);
}

cudaError_t Runner::correct(std::vector<ApplyJob>& jobs, const Net& net, cudaStream_t st,
                            const std::vector<int>& tags) {
    const int n = (int)jobs.size();
    if (n == 0) return cudaSuccess;
    if (n > cap) return cudaErrorInvalidValue;  // features() reserved the crops
    cudaError_t e;
    for (int k = 0; k < n; ++k) {
        jobs[k].resid = d_resid + 2 * k;
        jobs[k].moved = d_moved;
    }
    const int H = CROP, W = CROP;
    if ((e = conv3x3(x, net.w[0], net.b[0], nullptr, a1, nullptr, n, H, W, SILT_CLOSURE_CIN, SILT_CLOSURE_HIDDEN, 1,
                     st)) != cudaSuccess)
        return e;
    if ((e = conv3x3(a1, net.w[1], net.b[1], nullptr, a2, nullptr, n, H, W, SILT_CLOSURE_HIDDEN, SILT_CLOSURE_HIDDEN,
                     1, st)) != cudaSuccess)
        return e;
    if ((e = conv3x3(a2, net.w[2], net.b[2], nullptr, nullptr, y, n, H, W, SILT_CLOSURE_HIDDEN, SILT_CLOSURE_COUT, 0,
                     st)) != cudaSuccess)
        return e;
    void* d = nullptr;
    if ((e = ajobs.put(jobs.data(), jobs.size() * sizeof(ApplyJob), st, &d)) != cudaSuccess) return e;
    if ((e = launch_apply(static_cast<const ApplyJob*>(d), n, y, net.norm, st)) != cudaSuccess) return e;
    // The estimates come back without a wait; a slot is reused only after
    // its previous copy has landed.
    const int slot = (int)(written % RING);
    if ((e = cudaEventSynchronize(ev[slot])) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(h_resid[slot], d_resid, (size_t)n * 2 * sizeof(float), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(h_moved[slot], d_moved, sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
    if ((e = cudaEventRecord(ev[slot], st)) != cudaSuccess) return e;
    crops[slot] = n;
    tag[slot] = tags;
    ++written;
    if (written - read > (unsigned long long)RING) read = written - RING;
    return cudaSuccess;
}

bool Runner::poll(std::vector<float>& resid, double* moved_m3, std::vector<int>* out_tag) {
    // The newest finished correction among those not read yet.
    long long found = -1;
    for (unsigned long long q = read; q < written; ++q)
        if (cudaEventQuery(ev[q % RING]) == cudaSuccess) found = (long long)q;
    if (found < 0) return false;
    const int slot = (int)(found % RING);
    resid.resize(crops[slot]);
    for (int k = 0; k < crops[slot]; ++k) {
        const float c = h_resid[slot][2 * k], t = h_resid[slot][2 * k + 1];
        resid[k] = t > 0.0f ? c / t : 0.0f;
    }
    if (moved_m3) *moved_m3 = *h_moved[slot];
    if (out_tag) *out_tag = tag[slot];
    read = (unsigned long long)found + 1;
    return true;
}

// The crop's first coarse cell: centred on the mean tire position.
void crop_origin(const std::vector<silt_tire_push>& ps, float ox, float oz, float cell, int* ci0, int* cj0) {
    float mx = 0.0f, mz = 0.0f;
    for (const auto& t : ps) {
        mx += t.x;
        mz += t.z;
    }
    const float n = ps.empty() ? 1.0f : (float)ps.size();
    mx /= n;
    mz /= n;
    *ci0 = (int)std::floor((mx - ox) / cell) - CROP / 2;
    *cj0 = (int)std::floor((mz - oz) / cell) - CROP / 2;
}

}  // namespace closure
}  // namespace silt

using namespace silt::closure;

extern "C" {

int silt_closure_create(const float* params, int32_t n_params, const float* norm, int32_t device,
                        silt_closure** out) {
    if (!params || !norm || !out || n_params != SILT_CLOSURE_NPARAM)
        return fail(SILT_EINVAL, "invalid argument: closure_create");
    *out = nullptr;
    for (int k = 0; k < n_params; ++k)
        if (!std::isfinite(params[k])) return fail(SILT_EINVAL, "invalid argument: closure parameters not finite");
    for (int k = 0; k < SILT_CLOSURE_NNORM; ++k)
        if (!std::isfinite(norm[k])) return fail(SILT_EINVAL, "invalid argument: closure normalisation not finite");
    silt_closure* c = new silt_closure();
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    Net& N = c->net;
    const int cin[3] = {SILT_CLOSURE_CIN, SILT_CLOSURE_HIDDEN, SILT_CLOSURE_HIDDEN};
    const int cout[3] = {SILT_CLOSURE_HIDDEN, SILT_CLOSURE_HIDDEN, SILT_CLOSURE_COUT};
    if (e == cudaSuccess) e = cudaMalloc(&c->params, (size_t)n_params * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(c->params, params, (size_t)n_params * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&c->norm_dev, SILT_CLOSURE_NNORM * sizeof(float));
    if (e == cudaSuccess)
        e = cudaMemcpy(c->norm_dev, norm, SILT_CLOSURE_NNORM * sizeof(float), cudaMemcpyHostToDevice);
    size_t off = 0;
    for (int l = 0; l < 3 && e == cudaSuccess; ++l) {
        uint16_t* w = nullptr;
        e = cudaMalloc(&w, (size_t)9 * cin[l] * cout[l] * 2);
        c->wpack[l] = w;
        if (e != cudaSuccess) break;
        int rc = silt_closure_pack(c->params + off, w, nullptr, cin[l], cout[l], nullptr);
        if (rc) e = cudaErrorUnknown;
        N.w[l] = w;
        off += (size_t)9 * cin[l] * cout[l];
        N.b[l] = c->params + off;
        off += cout[l];
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    N.norm = c->norm_dev;
    if (e != cudaSuccess) {
        silt_closure_destroy(c);
        snprintf(g_err, sizeof g_err, "closure_create: %s", cudaGetErrorString(e));
        return SILT_ECUDA;
    }
    *out = c;
    return SILT_OK;
}

int silt_closure_destroy(silt_closure* c) {
    if (!c) return SILT_OK;
    cudaFree(c->params);
    cudaFree(c->norm_dev);
    for (auto* w : c->wpack) cudaFree(w);
    delete c;
    return SILT_OK;
}

}  // extern "C"
