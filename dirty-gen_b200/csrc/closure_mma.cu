// Tensor-core kernels of the learned flux closure: 3 x 3 convolutions as
// implicit GEMMs on tcgen05 (BF16 operands staged in shared memory, FP32
// accumulators in tensor memory), their weight gradient, the loss gradient,
// Adam and weight packing.
//
// Forward / input gradient (k_conv3x3): one CTA of 128 threads per 8 x 16
// pixel tile (M = 128 rows = pixels). K runs over (tap, input channel): for
// each of the 9 taps the tile's shifted pixels are copied into shared memory
// in the K-major no-swizzle core-matrix layout (8 rows x 16 bytes per core
// matrix), and one elected thread issues 9 x cin/16 MMAs of 128 x cout x 16
// into one TMEM accumulator; a commit to an mbarrier tells the CTA when the
// accumulator is complete, and each warp reads its 32 rows back with
// tcgen05.ld for the epilogue (bias, ReLU or the ReLU-derivative gate,
// BF16/FP32 store).
//
// Weight gradient (k_conv3x3_wgrad): M = (tap, input channel) rows (padded to
// a multiple of 128), N = output channels, K = pixels. Each CTA accumulates
// its tiles' 128-pixel K slices in TMEM and adds its partial sums to the
// global gradient once at the end.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "../../include/silt_closure.h"
#include "closure.cuh"
#include "launch_count.cuh"

namespace silt {
namespace closure {

thread_local char g_err[200] = "";

const char* last_error() { return g_err[0] ? g_err : nullptr; }

int fail(int rc, const char* what) {
    snprintf(g_err, sizeof g_err, "%s", what);
    return rc;
}

namespace {

constexpr int TILE_H = 8, TILE_W = 16, TILE_M = 128;
constexpr int THREADS = 128;
constexpr int WAIT_LIMIT = 1 << 22;  // mbarrier polls before a kernel gives up and flags an error

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (between the two 8-element K chunks of one MMA), stride byte offset
// (between 8-row groups), all in 16-byte units; bit 46 = descriptor version 1.
__device__ __forceinline__ uint64_t mat_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TILE_M >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Generic-proxy shared-memory writes become visible to the tensor core's reads.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the barrier phase with a bounded number of polls; false if it
// never completed.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, int limit = WAIT_LIMIT) {
    uint32_t done = 0;
    for (int k = 0; k < limit && !done; ++k)
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
    return done != 0;
}

// 8 consecutive FP32 columns of this thread's TMEM lane (32x32b shape: warp w
// of the warpgroup reads lanes 32w..32w+31).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* out) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int k = 0; k < 8; ++k) out[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint16_t to_bf16(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }
__device__ __forceinline__ float from_bf16(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }

struct ConvArgs {
    const uint16_t* x;
    const uint16_t* w;
    const float* bias;
    const uint16_t* gate;
    uint16_t* y;
    float* y32;
    int n_img, H, W, relu;
    int* err;
};

template <int CIN, int COUT>
struct ConvShape {
    static constexpr int TAP_BYTES = TILE_M * CIN * 2;  // one tap's 128 x cin slice of A
    static constexpr int A_BYTES = 9 * TAP_BYTES;
    static constexpr int KC = 9 * CIN / 8;              // 8-element K chunks of a weight row
    static constexpr int B_BYTES = COUT * 9 * CIN * 2;
    static constexpr int SMEM = A_BYTES + B_BYTES;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(THREADS) k_conv3x3(ConvArgs a) {
    ::silt::dep_wait();
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 32, "shape");
    using S = ConvShape<CIN, COUT>;
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* As = smem;
    uint8_t* Bs = smem + S::A_BYTES;
    __shared__ uint64_t bar;
    __shared__ uint32_t tslot;
    __shared__ float bias_s[COUT];
    const int tid = threadIdx.x, warp = tid >> 5;
    // Weights, row n = output channel, K = tap * CIN + c, in 8-element chunks.
    for (int q = tid; q < COUT * S::KC; q += THREADS) {
        const int n = q / S::KC, kc = q - n * S::KC;
        const uint4 v = *reinterpret_cast<const uint4*>(a.w + ((size_t)n * 9 * CIN + (size_t)kc * 8));
        *reinterpret_cast<uint4*>(Bs + (n >> 3) * (S::KC * 128) + kc * 128 + (n & 7) * 16) = v;
    }
    if (tid < COUT) bias_s[tid] = a.bias ? a.bias[tid] : 0.0f;
    if (tid == 0) bar_init(&bar, 1);
    if (warp == 0) tmem_alloc(&tslot, 32);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    const int tiles_x = (a.W + TILE_W - 1) / TILE_W, tiles_y = (a.H + TILE_H - 1) / TILE_H;
    const int per_img = tiles_x * tiles_y, ntiles = a.n_img * per_img;
    constexpr uint32_t IDESC = idesc_bf16(COUT);
    uint32_t parity = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const int img = t / per_img, r = t - img * per_img, ty = r / tiles_x, tx = r - ty * tiles_x;
        const int py = ty * TILE_H + (tid >> 4), px = tx * TILE_W + (tid & 15);  // row m = tid of A and D
        for (int tap = 0; tap < 9; ++tap) {
            const int yy = py + tap / 3 - 1, xx = px + tap % 3 - 1;
            const bool in = yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
            const uint4* src = reinterpret_cast<const uint4*>(a.x + (((size_t)img * a.H + yy) * a.W + xx) * CIN);
            uint8_t* dst = As + tap * S::TAP_BYTES + (tid >> 3) * (CIN * 16) + (tid & 7) * 16;
#pragma unroll
            for (int c = 0; c < CIN / 8; ++c)
                *reinterpret_cast<uint4*>(dst + c * 128) = in ? src[c] : make_uint4(0u, 0u, 0u, 0u);
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs);
            uint32_t acc = 0;
            for (int tap = 0; tap < 9; ++tap)
#pragma unroll
                for (int s = 0; s < CIN / 16; ++s) {
                    const uint64_t ad = mat_desc(a0 + tap * S::TAP_BYTES + s * 256, 128, CIN * 16);
                    const uint64_t bd = mat_desc(b0 + (tap * (CIN / 8) + 2 * s) * 128, 128, S::KC * 128);
                    mma_bf16(tmem, ad, bd, IDESC, acc);
                    acc = 1;
                }
            mma_commit(&bar);
        }
        ok = __syncthreads_and(bar_wait(&bar, parity) ? 1 : 0) != 0;  // uniform across the CTA
        parity ^= 1u;
        tc_fence_after();
        float v[COUT];
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 8) tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v + c0);
        tmem_wait_ld();
        if (ok && py < a.H && px < a.W) {
            const size_t pix = ((size_t)img * a.H + py) * a.W + px;
            const uint16_t* g = a.gate ? a.gate + pix * COUT : nullptr;
#pragma unroll
            for (int c = 0; c < COUT; ++c) {
                float o = v[c] + bias_s[c];
                if (a.relu) o = fmaxf(o, 0.0f);
                if (g && !(from_bf16(g[c]) > 0.0f)) o = 0.0f;
                v[c] = o;
            }
            if (a.y32) {
                float4* d = reinterpret_cast<float4*>(a.y32 + pix * COUT);
#pragma unroll
                for (int c = 0; c < COUT; c += 4) d[c / 4] = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
            }
            if (a.y) {
                uint4* d = reinterpret_cast<uint4*>(a.y + pix * COUT);
#pragma unroll
                for (int c = 0; c < COUT; c += 8) {
                    uint4 o;
                    o.x = (uint32_t)to_bf16(v[c]) | ((uint32_t)to_bf16(v[c + 1]) << 16);
                    o.y = (uint32_t)to_bf16(v[c + 2]) | ((uint32_t)to_bf16(v[c + 3]) << 16);
                    o.z = (uint32_t)to_bf16(v[c + 4]) | ((uint32_t)to_bf16(v[c + 5]) << 16);
                    o.w = (uint32_t)to_bf16(v[c + 6]) | ((uint32_t)to_bf16(v[c + 7]) << 16);
                    d[c / 8] = o;
                }
            }
        }
        tc_fence_before();
        __syncthreads();
    }
    if (!ok && tid == 0 && a.err) atomicExch(a.err, 1);
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(tmem, 32);
}

struct WgradArgs {
    const uint16_t* x;
    const uint16_t* dy;
    float* dw;
    float* db;
    int n_img, H, W;
    int* err;
};

template <int CIN, int COUT>
struct WgradShape {
    static constexpr int ROWS = 9 * CIN;                    // (tap, cin)
    static constexpr int MT = (ROWS + TILE_M - 1) / TILE_M;  // 128-row M tiles
    static constexpr int SBO = (TILE_M / 8) * 128;           // 16 pixel chunks per row group
    static constexpr int A_BYTES = MT * TILE_M * TILE_M * 2;
    static constexpr int B_BYTES = COUT * TILE_M * 2;
    static constexpr int SMEM = A_BYTES + B_BYTES;
    static constexpr int COLS = MT * COUT <= 32 ? 32 : (MT * COUT <= 64 ? 64 : 128);
};

// Eight pixels' 8-channel vectors (v[j] = pixel j) -> eight channels'
// 8-pixel vectors (out[r] = channel r), BF16 lanes.
__device__ __forceinline__ void transpose8(const uint4 (&v)[8], uint4 (&out)[8]) {
    uint16_t e[8][8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t w[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            e[j][2 * q] = (uint16_t)(w[q] & 0xFFFFu);
            e[j][2 * q + 1] = (uint16_t)(w[q] >> 16);
        }
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        out[r].x = (uint32_t)e[0][r] | ((uint32_t)e[1][r] << 16);
        out[r].y = (uint32_t)e[2][r] | ((uint32_t)e[3][r] << 16);
        out[r].z = (uint32_t)e[4][r] | ((uint32_t)e[5][r] << 16);
        out[r].w = (uint32_t)e[6][r] | ((uint32_t)e[7][r] << 16);
    }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(THREADS) k_conv3x3_wgrad(WgradArgs a) {
    ::silt::dep_wait();
    using S = WgradShape<CIN, COUT>;
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* As = smem;
    uint8_t* Bs = smem + S::A_BYTES;
    __shared__ uint64_t bar;
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5;
    // Rows past 9 * CIN are zero for the whole kernel.
    for (int q = S::ROWS * 16 + tid; q < S::MT * TILE_M * 16; q += THREADS)
        *reinterpret_cast<uint4*>(As + (q / 16 >> 3) * S::SBO + (q % 16) * 128 + (q / 16 & 7) * 16) =
            make_uint4(0u, 0u, 0u, 0u);
    if (tid == 0) bar_init(&bar, 1);
    if (warp == 0) tmem_alloc(&tslot, S::COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    const int tiles_x = (a.W + TILE_W - 1) / TILE_W, tiles_y = (a.H + TILE_H - 1) / TILE_H;
    const int per_img = tiles_x * tiles_y, ntiles = a.n_img * per_img;
    constexpr uint32_t IDESC = idesc_bf16(COUT);
    constexpr int B_ITEMS = (COUT / 8) * 16;  // (channel chunk, pixel chunk)
    float bsum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t parity = 0;
    bool ok = true, any = false;
    for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const int img = t / per_img, r = t - img * per_img, ty = r / tiles_x, tx = r - ty * tiles_x;
        // A: row (tap, cin), K = the tile's 128 pixels (pixel m at (m / 16, m % 16)).
        for (int q = tid; q < 9 * (CIN / 8) * 16; q += THREADS) {
            const int pc = q & 15, cc = (q >> 4) % (CIN / 8), tap = (q >> 4) / (CIN / 8);
            uint4 v[8], o[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int m = pc * 8 + j;
                const int yy = ty * TILE_H + (m >> 4) + tap / 3 - 1, xx = tx * TILE_W + (m & 15) + tap % 3 - 1;
                const bool in = yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
                v[j] = in ? *reinterpret_cast<const uint4*>(a.x + (((size_t)img * a.H + yy) * a.W + xx) * CIN + cc * 8)
                          : make_uint4(0u, 0u, 0u, 0u);
            }
            transpose8(v, o);
            uint8_t* dst = As + (tap * (CIN / 8) + cc) * S::SBO + pc * 128;
#pragma unroll
            for (int k = 0; k < 8; ++k) *reinterpret_cast<uint4*>(dst + k * 16) = o[k];
        }
        // B: row = output channel, K = pixels; pixels outside the image give 0.
        if (tid < B_ITEMS) {
            const int pc = tid & 15, cc = tid >> 4;
            uint4 v[8], o[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int m = pc * 8 + j;
                const int yy = ty * TILE_H + (m >> 4), xx = tx * TILE_W + (m & 15);
                const bool in = yy < a.H && xx < a.W;
                v[j] = in ? *reinterpret_cast<const uint4*>(a.dy + (((size_t)img * a.H + yy) * a.W + xx) * COUT + cc * 8)
                          : make_uint4(0u, 0u, 0u, 0u);
            }
            transpose8(v, o);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                *reinterpret_cast<uint4*>(Bs + cc * S::SBO + pc * 128 + k * 16) = o[k];
                const uint32_t w[4] = {o[k].x, o[k].y, o[k].z, o[k].w};
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    bsum[k] += from_bf16((uint16_t)(w[q] & 0xFFFFu)) + from_bf16((uint16_t)(w[q] >> 16));
            }
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs);
#pragma unroll
            for (int mt = 0; mt < S::MT; ++mt)
#pragma unroll
                for (int s = 0; s < TILE_M / 16; ++s) {
                    const uint64_t ad = mat_desc(a0 + mt * (TILE_M / 8) * S::SBO + s * 256, 128, S::SBO);
                    const uint64_t bd = mat_desc(b0 + s * 256, 128, S::SBO);
                    mma_bf16(tmem + (uint32_t)(mt * COUT), ad, bd, IDESC, (any || s > 0) ? 1u : 0u);
                }
            mma_commit(&bar);
        }
        any = true;
        // Uniform across the CTA; the shared operands are rewritten by the next tile.
        ok = __syncthreads_and(bar_wait(&bar, parity) ? 1 : 0) != 0;
        parity ^= 1u;
        tc_fence_after();
    }
    if (ok && any) {
#pragma unroll
        for (int mt = 0; mt < S::MT; ++mt) {
            float v[COUT];
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 8)
                tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * COUT + c0), v + c0);
            tmem_wait_ld();
            const int row = mt * TILE_M + tid;
            if (row < S::ROWS)
#pragma unroll
                for (int c = 0; c < COUT; ++c) atomicAdd(a.dw + (size_t)row * COUT + c, v[c]);
        }
        if (tid < B_ITEMS && a.db)
#pragma unroll
            for (int k = 0; k < 8; ++k) atomicAdd(a.db + (tid >> 4) * 8 + k, bsum[k]);
    }
    if (!ok && tid == 0 && a.err) atomicExch(a.err, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(tmem, S::COLS);
}

__global__ void k_loss_grad(const float* y, const float* t, const float* wgt, uint16_t* dy, double* loss, int n_pix,
                            int cpad, int n_out, float scale) {
    ::silt::dep_wait();
    double part = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_pix; p += gridDim.x * blockDim.x) {
        const float w = wgt ? wgt[p] : 1.0f;
        for (int c = 0; c < cpad; ++c) {
            float g = 0.0f;
            if (c < n_out) {
                const float d = y[(size_t)p * cpad + c] - t[(size_t)p * n_out + c];
                part += (double)(w * d * d) * (double)scale;
                g = 2.0f * w * d * scale;
            }
            dy[(size_t)p * cpad + c] = to_bf16(g);
        }
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    __shared__ double ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0 && loss) atomicAdd(loss, v);
    }
}

// One crop per block, one cell per thread (the crop edge has no outgoing face).
__global__ void __launch_bounds__(SILT_CLOSURE_CROP * SILT_CLOSURE_CROP)
    k_step_loss(const float* y, const float* t, const float* scale, const float* inv_var, float lam, uint16_t* dy,
                double* loss, float norm) {
    ::silt::dep_wait();
    constexpr int N = SILT_CLOSURE_CROP, NC = N * N, CO = SILT_CLOSURE_COUT, NT = 8;
    __shared__ float g[4][NC];
    __shared__ float e[2][NC];
    __shared__ double red[NC / 32];
    const int p = threadIdx.x, cx = p % N, cy = p / N;
    const size_t pix = (size_t)blockIdx.x * NC + p;
    const float* yo = y + pix * CO;
    const float* to = t + pix * NT;
    float yv[8], sc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        yv[c] = yo[c];
        sc[c] = scale[c];
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const bool edge = (c % 2 == 0) ? cx == N - 1 : cy == N - 1;
        g[c][p] = edge ? 0.0f : yv[c] * sc[c];
    }
    __syncthreads();
    double part = 0.0;
#pragma unroll
    for (int l = 0; l < 2; ++l) {
        const float in = (cx > 0 ? g[2 * l][p - 1] : 0.0f) + (cy > 0 ? g[2 * l + 1][p - N] : 0.0f);
        const float div = in - g[2 * l][p] - g[2 * l + 1][p];
        const float r = div - to[l];
        e[l][p] = r;
        part += (double)(inv_var[l] * r * r);
    }
    float gv[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float w = to[6 + k / 2];
        const float r = yv[4 + k] * sc[4 + k] - to[2 + k];
        part += (double)(inv_var[2 + k] * w * r * r);
        gv[k] = 2.0f * inv_var[2 + k] * w * r * sc[4 + k];
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) part += (double)(lam * yv[c] * yv[c]);
    __syncthreads();
    uint16_t* out = dy + pix * CO;
#pragma unroll
    for (int l = 0; l < 2; ++l) {
        const float gx = cx < N - 1 ? 2.0f * inv_var[l] * (e[l][p + 1] - e[l][p]) : 0.0f;
        const float gz = cy < N - 1 ? 2.0f * inv_var[l] * (e[l][p + N] - e[l][p]) : 0.0f;
        out[2 * l] = to_bf16((gx * sc[2 * l] + 2.0f * lam * yv[2 * l]) * norm);
        out[2 * l + 1] = to_bf16((gz * sc[2 * l + 1] + 2.0f * lam * yv[2 * l + 1]) * norm);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) out[4 + k] = to_bf16((gv[k] + 2.0f * lam * yv[4 + k]) * norm);
#pragma unroll
    for (int c = 8; c < CO; ++c) out[c] = 0;
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((p & 31) == 0) red[p >> 5] = part;
    __syncthreads();
    if (p == 0 && loss) {
        double s = 0.0;
        for (int w = 0; w < NC / 32; ++w) s += red[w];
        atomicAdd(loss, s * (double)norm);
    }
}

__global__ void k_adam(float* p, float* m, float* v, const float* g, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    ::silt::dep_wait();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void k_pack(const float* w, uint16_t* fwd, uint16_t* bwd, int cin, int cout) {
    ::silt::dep_wait();
    const int n = 9 * cin * cout;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = i % cout, c = (i / cout) % cin, tap = i / (cout * cin);
        const uint16_t b = to_bf16(w[i]);
        if (fwd) fwd[((size_t)o * 9 + tap) * cin + c] = b;
        if (bwd) bwd[((size_t)c * 9 + (8 - tap)) * cout + o] = b;
    }
}

// The bounded wait on a barrier phase that never completes (nothing arrives
// on it): every thread gives up after `polls` polls and the error slot is
// set, as a convolution's wait would set it. Nothing is in flight and no
// tensor memory is held, so the kernel ends and the context stays usable.
__global__ void k_wait_probe(int* err, int polls) {
    ::silt::dep_wait();
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) bar_init(&bar, 1);
    __syncthreads();
    const bool ok = bar_wait(&bar, 0, polls);
    if (!ok && threadIdx.x == 0 && err) atomicExch(err, 1);
}

template <class K>
cudaError_t set_smem(K kernel, int bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    }
    return n;
}

template <int CIN, int COUT>
cudaError_t conv_launch(const ConvArgs& a, cudaStream_t st) {
    using S = ConvShape<CIN, COUT>;
    static cudaError_t attr = set_smem(k_conv3x3<CIN, COUT>, S::SMEM);
    if (attr != cudaSuccess) return attr;
    const int tiles = a.n_img * ((a.H + TILE_H - 1) / TILE_H) * ((a.W + TILE_W - 1) / TILE_W);
    const int grid = tiles < 2 * sm_count() ? tiles : 2 * sm_count();
    ::silt::launch_dep(k_conv3x3<CIN, COUT>, dim3(grid), dim3(THREADS), S::SMEM, st, a);
    ::silt::count_launch();
    return cudaGetLastError();
}

template <int CIN, int COUT>
cudaError_t wgrad_launch(const WgradArgs& a, cudaStream_t st) {
    using S = WgradShape<CIN, COUT>;
    static cudaError_t attr = set_smem(k_conv3x3_wgrad<CIN, COUT>, S::SMEM);
    if (attr != cudaSuccess) return attr;
    const int tiles = a.n_img * ((a.H + TILE_H - 1) / TILE_H) * ((a.W + TILE_W - 1) / TILE_W);
    const int grid = tiles < sm_count() ? tiles : sm_count();
    ::silt::launch_dep(k_conv3x3_wgrad<CIN, COUT>, dim3(grid), dim3(THREADS), S::SMEM, st, a);
    ::silt::count_launch();
    return cudaGetLastError();
}

int* err_slot() {
    static int* d = nullptr;
    if (!d && cudaMalloc(&d, sizeof(int)) == cudaSuccess) cudaMemset(d, 0, sizeof(int));
    return d;
}

}  // namespace

cudaError_t conv3x3(const uint16_t* x, const uint16_t* w, const float* bias, const uint16_t* gate, uint16_t* y,
                    float* y32, int n_img, int h, int wd, int cin, int cout, int relu, cudaStream_t st) {
    ConvArgs a{x, w, bias, gate, y, y32, n_img, h, wd, relu, err_slot()};
    if (n_img <= 0 || h <= 0 || wd <= 0) return cudaSuccess;
    if (cin == 16 && cout == 32) return conv_launch<16, 32>(a, st);
    if (cin == 32 && cout == 32) return conv_launch<32, 32>(a, st);
    if (cin == 32 && cout == 16) return conv_launch<32, 16>(a, st);
    if (cin == 16 && cout == 16) return conv_launch<16, 16>(a, st);
    return cudaErrorInvalidValue;
}

cudaError_t conv3x3_wgrad(const uint16_t* x, const uint16_t* dy, float* dw, float* db, int n_img, int h, int wd,
                          int cin, int cout, cudaStream_t st) {
    WgradArgs a{x, dy, dw, db, n_img, h, wd, err_slot()};
    if (n_img <= 0 || h <= 0 || wd <= 0) return cudaSuccess;
    if (cin == 16 && cout == 32) return wgrad_launch<16, 32>(a, st);
    if (cin == 32 && cout == 32) return wgrad_launch<32, 32>(a, st);
    if (cin == 32 && cout == 16) return wgrad_launch<32, 16>(a, st);
    return cudaErrorInvalidValue;
}

int device_error(cudaStream_t st, int* flag) {
    int* d = err_slot();
    if (!d) return 0;
    if (cudaMemcpyAsync(flag, d, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
    return 0;
}

}  // namespace closure
}  // namespace silt

using namespace silt::closure;

namespace {

bool shape_ok(int cin, int cout) {
    return (cin == 16 && cout == 32) || (cin == 32 && cout == 32) || (cin == 32 && cout == 16) ||
           (cin == 16 && cout == 16);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

int cuda_rc(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return SILT_OK;
    snprintf(g_err, sizeof g_err, "%s: %s", what, cudaGetErrorString(e));
    return SILT_ECUDA;
}

}  // namespace

extern "C" {

int silt_conv3x3_forward(const void* x, const void* w, const float* bias, const void* gate, void* y, float* y32,
                         int32_t n_img, int32_t h, int32_t wd, int32_t cin, int32_t cout, int32_t relu,
                         void* stream) {
    if (!x || !w || (!y && !y32) || n_img < 0 || h < 0 || wd < 0 || !shape_ok(cin, cout))
        return fail(SILT_EINVAL, "invalid argument: conv3x3_forward");
    if (!aligned16(x) || !aligned16(w) || (y && !aligned16(y)) || (y32 && !aligned16(y32)))
        return fail(SILT_EINVAL, "invalid argument: conv3x3_forward needs 16-byte aligned tensors");
    return cuda_rc(conv3x3((const uint16_t*)x, (const uint16_t*)w, bias, (const uint16_t*)gate, (uint16_t*)y, y32,
                           n_img, h, wd, cin, cout, relu, (cudaStream_t)stream),
                   "conv3x3_forward");
}

int silt_conv3x3_wgrad(const void* x, const void* dy, float* dw, float* db, int32_t n_img, int32_t h, int32_t wd,
                       int32_t cin, int32_t cout, void* stream) {
    if (!x || !dy || !dw || n_img < 0 || h < 0 || wd < 0 || !shape_ok(cin, cout) || (cin == 16 && cout == 16))
        return fail(SILT_EINVAL, "invalid argument: conv3x3_wgrad");
    if (!aligned16(x) || !aligned16(dy)) return fail(SILT_EINVAL, "invalid argument: conv3x3_wgrad alignment");
    return cuda_rc(conv3x3_wgrad((const uint16_t*)x, (const uint16_t*)dy, dw, db, n_img, h, wd, cin, cout,
                                 (cudaStream_t)stream),
                   "conv3x3_wgrad");
}

int silt_closure_loss_grad(const float* y, const float* target, const float* pixel_weight, void* dy, double* loss,
                           int32_t n_pix, int32_t cout_pad, int32_t n_out, float scale, void* stream) {
    if (!y || !target || !dy || n_pix < 0 || cout_pad <= 0 || n_out <= 0 || n_out > cout_pad)
        return fail(SILT_EINVAL, "invalid argument: closure_loss_grad");
    if (n_pix == 0) return SILT_OK;
    const int blocks = (n_pix + 255) / 256 < 1184 ? (n_pix + 255) / 256 : 1184;
    ::silt::launch_dep(k_loss_grad, dim3(blocks), dim3(256), 0, (cudaStream_t)stream, y, target, pixel_weight, (uint16_t*)dy, loss, n_pix,
                                                          cout_pad, n_out, scale);
    ::silt::count_launch();
    return cuda_rc(cudaGetLastError(), "closure_loss_grad");
}

int silt_closure_step_loss_grad(const float* y, const float* t, const float* scale, const float* inv_var,
                                float lambda, void* dy, double* loss, int32_t n_img, float norm, void* stream) {
    if (!y || !t || !scale || !inv_var || !dy || n_img < 0)
        return fail(SILT_EINVAL, "invalid argument: closure_step_loss_grad");
    if (n_img == 0) return SILT_OK;
    ::silt::launch_dep(k_step_loss, dim3(n_img), dim3(SILT_CLOSURE_CROP * SILT_CLOSURE_CROP), 0, (cudaStream_t)stream, 
        y, t, scale, inv_var, lambda, (uint16_t*)dy, loss, norm);
    ::silt::count_launch();
    return cuda_rc(cudaGetLastError(), "closure_step_loss_grad");
}

int silt_closure_adam(float* param, float* m, float* v, const float* grad, int32_t n, float lr, float beta1,
                      float beta2, float eps, int32_t step, void* stream) {
    if (!param || !m || !v || !grad || n < 0 || step < 1) return fail(SILT_EINVAL, "invalid argument: closure_adam");
    if (n == 0) return SILT_OK;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    ::silt::launch_dep(k_adam, dim3((n + 255) / 256), dim3(256), 0, (cudaStream_t)stream, param, m, v, grad, n, lr, beta1, beta2, eps, c1, c2);
    ::silt::count_launch();
    return cuda_rc(cudaGetLastError(), "closure_adam");
}

int silt_closure_wait_status(int32_t* gave_up, void* stream) {
    if (!gave_up) return fail(SILT_EINVAL, "invalid argument: closure_wait_status");
    int* d = err_slot();
    if (!d) return fail(SILT_ECUDA, "closure_wait_status: no error slot");
    int flag = 0;
    const cudaStream_t st = (cudaStream_t)stream;
    int rc = cuda_rc(cudaMemcpyAsync(&flag, d, sizeof(int), cudaMemcpyDeviceToHost, st), "closure_wait_status");
    if (rc == SILT_OK) rc = cuda_rc(cudaMemsetAsync(d, 0, sizeof(int), st), "closure_wait_status");
    if (rc == SILT_OK) rc = cuda_rc(cudaStreamSynchronize(st), "closure_wait_status");
    *gave_up = flag;
    return rc;
}

int silt_closure_wait_probe(int32_t polls, void* stream) {
    if (polls < 1 || polls > (1 << 20)) return fail(SILT_EINVAL, "invalid argument: closure_wait_probe polls");
    int* d = err_slot();
    if (!d) return fail(SILT_ECUDA, "closure_wait_probe: no error slot");
    ::silt::launch_dep(k_wait_probe, dim3(1), dim3(32), 0, (cudaStream_t)stream, d, (int)polls);
    ::silt::count_launch();
    return cuda_rc(cudaGetLastError(), "closure_wait_probe");
}

int silt_closure_pack(const float* w, void* w_fwd, void* w_bwd, int32_t cin, int32_t cout, void* stream) {
    if (!w || (!w_fwd && !w_bwd) || cin <= 0 || cout <= 0) return fail(SILT_EINVAL, "invalid argument: closure_pack");
    const int n = 9 * cin * cout;
    ::silt::launch_dep(k_pack, dim3((n + 255) / 256), dim3(256), 0, (cudaStream_t)stream, w, (uint16_t*)w_fwd, (uint16_t*)w_bwd, cin, cout);
    ::silt::count_launch();
    return cuda_rc(cudaGetLastError(), "closure_pack");
}

}  // extern "C"
