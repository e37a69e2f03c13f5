// One CTA per (patch, layer) steps a nested 2 cm sheet exactly as the
// reference does (x3-team/Dirty-gen src/fluid_core.rs:1659-2082): work boxes
// chosen per step (awake 8x8 tiles for pace 0/1, wet bodies for pace 2/3),
// the CFL substep count, then every substep box by box with the per-sheet
// scratch planes the reference keeps between steps. A box-edge cell of the
// reference reads pressure and blur values that an earlier box or an earlier
// step left in that scratch; keeping the same planes with the same writes
// reproduces those reads. The patch planes are small (64^2..160^2) and stay
// in L2; each phase is a CTA-wide pass separated by __syncthreads.
#include <cstdint>
#include <cuda_runtime.h>

#include "sheet_math.cuh"
#include "sheet_patch.cuh"

namespace silt {
namespace patch {

constexpr int NT = 1024;          // threads per CTA
constexpr int SLEEP_TILE = 8;     // src/fluid_core.rs:1528
constexpr int MAX_TILES = 64 * 64;
constexpr int MAX_BOXES = 512;

struct Box {
    int i0, i1, j0, j1;
};

struct Shared {
    int lab[MAX_TILES];           // tile component labels / wet-body scratch
    unsigned char hot[MAX_TILES];
    unsigned char grown[MAX_TILES];
    int bbox[4][MAX_BOXES];       // per box: i0, i1, j0, j1
    int nbox;
    int changed;
    float red_f[NT / 32];
    double red_d[NT / 32];
    int red_i[4][NT / 32];
};

#define CTA_RECT(I0, I1, J0, J1, ...)                                              \
    {                                                                               \
        const int ri0_ = (I0), rj0_ = (J0);                                         \
        const int rw_ = (I1) - ri0_ + 1, rh_ = (J1) - rj0_ + 1;                    \
        if (rw_ > 0 && rh_ > 0) {                                                   \
            const int rn_ = rw_ * rh_;                                              \
            for (int k_ = threadIdx.x; k_ < rn_; k_ += NT) {                        \
                const int j = rj0_ + k_ / rw_;                                      \
                const int i = ri0_ + k_ % rw_;                                      \
                const int g = j * res + i;                                          \
                (void)g;                                                            \
                __VA_ARGS__                                                         \
            }                                                                       \
        }                                                                           \
    }

__device__ __forceinline__ float block_sum_f(Shared& S, float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) S.red_f[threadIdx.x >> 5] = v;
    __syncthreads();
    float t = 0.0f;
    if (threadIdx.x < 32) {
        t = S.red_f[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) S.red_f[0] = t;
    }
    __syncthreads();
    return S.red_f[0];
}

__device__ __forceinline__ double block_sum_d(Shared& S, double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) S.red_d[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = S.red_d[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) S.red_d[0] = t;
    }
    __syncthreads();
    return S.red_d[0];
}

__device__ __forceinline__ float block_max_f(Shared& S, float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) S.red_f[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        float t = S.red_f[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) t = fmaxf(t, __shfl_down_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) S.red_f[0] = t;
    }
    __syncthreads();
    return S.red_f[0];
}

// Reduces four ints: op 0 = sum, 1 = min, 2 = max, per slot.
__device__ void block_reduce4(Shared& S, int v[4], const int op[4]) {
    for (int q = 0; q < 4; ++q)
        for (int o = 16; o > 0; o >>= 1) {
            int w = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = op[q] == 0 ? v[q] + w : (op[q] == 1 ? min(v[q], w) : max(v[q], w));
        }
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 4; ++q) S.red_i[q][threadIdx.x >> 5] = v[q];
    __syncthreads();
    if (threadIdx.x < 32) {
        for (int q = 0; q < 4; ++q) {
            int t = S.red_i[q][threadIdx.x];
            for (int o = 16; o > 0; o >>= 1) {
                int w = __shfl_down_sync(0xffffffffu, t, o);
                t = op[q] == 0 ? t + w : (op[q] == 1 ? min(t, w) : max(t, w));
            }
            if (threadIdx.x == 0) S.red_i[q][0] = t;
        }
    }
    __syncthreads();
    for (int q = 0; q < 4; ++q) v[q] = S.red_i[q][0];
    __syncthreads();
}

__device__ __forceinline__ float tap5c(const float* row, int res, int i, float k0, float k1, float k2, int stride) {
    // Five taps along one axis with clamped indices; interior cells start from
    // the first product (accum5), edge cells from 0.0 (accum5_clamped).
    const bool in = i >= 2 && i <= res - 3;
    const int i0 = i < 2 ? 0 : i - 2, i1 = i < 1 ? 0 : i - 1;
    const int i3 = i + 1 > res - 1 ? res - 1 : i + 1, i4 = i + 2 > res - 1 ? res - 1 : i + 2;
    float a0 = row[i0 * stride], a1 = row[i1 * stride], a2 = row[i * stride], a3 = row[i3 * stride],
          a4 = row[i4 * stride];
    float a = in ? a0 * k0 : 0.0f + a0 * k0;
    a += a1 * k1;
    a += a2 * k2;
    a += a3 * k1;
    a += a4 * k0;
    return a;
}

// One blur_box (src/fluid_core.rs:3541-3569): x pass of the box rows into
// tmp, then z pass into dst; the z pass reads tmp rows outside the box as the
// scratch holds them.
__device__ void cta_blur(const float* src, float* dst, float* tmp, int res, const Box& b, float k0, float k1,
                         float k2) {
    CTA_RECT(b.i0, b.i1, b.j0, b.j1, { tmp[g] = tap5c(src + j * res, res, i, k0, k1, k2, 1); })
    __syncthreads();
    CTA_RECT(b.i0, b.i1, b.j0, b.j1, { dst[g] = tap5c(tmp + i, res, j, k0, k1, k2, res); })
    __syncthreads();
}

// Cell material of the layer: viscosity for mobility and damping.
__device__ __forceinline__ float job_nu(const Job& J, const Args& A, int g) {
    return J.nu_const ? A.nu_c : dynamic_viscosity(J.grain[g], J.moisture[g]);
}

// transport_open_rows (src/fluid_core.rs:3025-3137) on one box, gates open.
__device__ void cta_transport(const Job& J, const Args& A, int res, const Box& b, float dt) {
    float* h = J.h;
    float* F1 = J.f1;
    float* F2 = J.f2;
    const float cell = A.cell;
    // x pass: left-going, right-going, update.
    CTA_RECT(b.i0, b.i1 - 1, b.j0, b.j1, {
        float speed = 0.5f * (J.u[g] + J.u[g + 1]);
        float dh = open_edge_dh(false, h[g + 1], h[g], 0.0f, 1, 0.0f, 0.0f, speed, dt, cell, 0.45f);
        F1[g] = speed > 0.0f ? 0.0f : dh;
    })
    __syncthreads();
    CTA_RECT(b.i0, b.i1 - 1, b.j0, b.j1, {
        float speed = 0.5f * (J.u[g] + J.u[g + 1]);
        float prev = i > b.i0 ? F1[g - 1] : 0.0f;
        float dh = open_edge_dh(false, h[g], h[g + 1], 0.0f + prev, 1, 0.0f, 0.0f, speed, dt, cell, 0.45f);
        F2[g] = speed > 0.0f ? dh : 0.0f;
    })
    __syncthreads();
    CTA_RECT(b.i0, b.i1, b.j0, b.j1, {
        float flm = i > b.i0 ? F1[g - 1] : 0.0f, frm = i > b.i0 ? F2[g - 1] : 0.0f;
        float flc = i < b.i1 ? F1[g] : 0.0f, frc = i < b.i1 ? F2[g] : 0.0f;
        float rem = (0.0f + flm) + frc, add = (0.0f + frm) + flc;
        float hv = h[g];
        float moved = fmaxf(hv - rem + add, 0.0f);
        h[g] = (rem > 0.0f || add > 0.0f) ? moved : hv;
    })
    __syncthreads();
    // z pass: up-going (donor row j+1), down-going (donor row j, removed = up of the pair above).
    CTA_RECT(b.i0, b.i1, b.j0, b.j1 - 1, {
        float speed = 0.5f * (J.v[g] + J.v[g + res]);
        float dh = open_edge_dh(false, h[g + res], h[g], 0.0f, 1, 0.0f, 0.0f, speed, dt, cell, 0.45f);
        F1[g] = speed > 0.0f ? 0.0f : dh;
    })
    __syncthreads();
    CTA_RECT(b.i0, b.i1, b.j0, b.j1 - 1, {
        float speed = 0.5f * (J.v[g] + J.v[g + res]);
        float ra = j > b.j0 ? 0.0f + F1[g - res] : 0.0f;
        float dh = open_edge_dh(false, h[g], h[g + res], ra, 1, 0.0f, 0.0f, speed, dt, cell, 0.45f);
        F2[g] = speed > 0.0f ? dh : 0.0f;
    })
    __syncthreads();
    CTA_RECT(b.i0, b.i1, b.j0, b.j1, {
        float upm = j > b.j0 ? F1[g - res] : 0.0f, dnm = j > b.j0 ? F2[g - res] : 0.0f;
        float upc = j < b.j1 ? F1[g] : 0.0f, dnc = j < b.j1 ? F2[g] : 0.0f;
        float rem = (0.0f + upm) + dnc, add = (0.0f + dnm) + upc;
        float hv = h[g];
        float moved = fmaxf(hv - rem + add, 0.0f);
        h[g] = (rem > 0.0f || add > 0.0f) ? moved : hv;
    })
    __syncthreads();
}

__device__ void cta_dry_cut(const Job& J, int res, const Box& b, float eps) {
    if (!(eps > 0.0f)) return;
    CTA_RECT(b.i0, b.i1, b.j0, b.j1, {
        if (J.h[g] < eps) {
            J.h[g] = 0.0f;
            J.u[g] = 0.0f;
            J.v[g] = 0.0f;
        }
    })
    __syncthreads();
}

// substep (src/fluid_core.rs:1879-2082) for an open 2 cm sheet: no projection,
// snapshot-Jacobi confinement (gravity_jacobi_serial, :2530-2595).
__device__ void cta_substep(const Job& J, const Args& A, int res, const Box& b, float* const* sc, float dt,
                            float decay_w, bool do_flux) {
    float* sa = sc[0];
    float* sb = sc[1];
    float* scc = sc[2];
    float* sd = sc[3];
    float* se = sc[4];
    const float eps = A.eps, cell = A.cell;
    const float two = 2.0f * cell;
    {
        const int hi0 = max(b.i0 - 2, 0), hi1 = min(b.i1 + 2, res - 1);
        const int hj0 = max(b.j0 - 2, 0), hj1 = min(b.j1 + 2, res - 1);
        CTA_RECT(hi0, hi1, hj0, hj1, { sa[g] = J.bed[g] + J.h[g]; })
    }
    __syncthreads();
    cta_blur(sa, sb, se, res, b, kG0, kG1, kG2);
    cta_blur(sa, scc, se, res, b, kS0, kS1, kS2);
    CTA_RECT(b.i0, b.i1, b.j0, b.j1, {
        float filtered = 0.62f * sb[g] + 0.38f * scc[g];
        sd[g] = 0.45f * filtered + 0.55f * sa[g];
    })
    __syncthreads();
    CTA_RECT(b.i0, b.i1, b.j0, b.j1, {
        if (J.h[g] > eps) {
            const int ip = min(i + 1, res - 1), im = max(i - 1, 0), jp = min(j + 1, res - 1), jm = max(j - 1, 0);
            float px = (sd[j * res + ip] - sd[j * res + im]) / two;
            float pz = (sd[jp * res + i] - sd[jm * res + i]) / two;
            float mob = J.nu_const ? A.mob_c : sheet_mobility_for(job_nu(J, A, g));
            J.u[g] += -kGravity * px * mob * dt;
            J.v[g] += -kGravity * pz * mob * dt;
        }
    })
    __syncthreads();
    if (J.vort > 0.0f) {
        float* W = J.f1;
        const int wi0 = max(b.i0 - 1, 0), wi1 = min(b.i1 + 1, res - 1);
        const int wj0 = max(b.j0 - 1, 0), wj1 = min(b.j1 + 1, res - 1);
        CTA_RECT(wi0, wi1, wj0, wj1, {
            const int ip = min(i + 1, res - 1), im = max(i - 1, 0), jp = min(j + 1, res - 1), jm = max(j - 1, 0);
            float dvdx = (J.v[j * res + ip] - J.v[j * res + im]) / two;
            float dudz = (J.u[jp * res + i] - J.u[jm * res + i]) / two;
            W[g] = dvdx - dudz;
        })
        __syncthreads();
        CTA_RECT(b.i0, b.i1, b.j0, b.j1, {
            if (J.h[g] > eps) {
                float w = W[g];
                if (finite_f(w) && !(fabsf(w) < 1.0e-4f)) {
                    const int ip = min(i + 1, res - 1), im = max(i - 1, 0), jp = min(j + 1, res - 1),
                              jm = max(j - 1, 0);
                    float wxp = fabsf(W[j * res + ip]), wxm = fabsf(W[j * res + im]);
                    float wzp = fabsf(W[jp * res + i]), wzm = fabsf(W[jm * res + i]);
                    float nx = (wxp - wxm) / two;
                    float nz = (wzp - wzm) / two;
                    float du = J.vort * dt * (-nz * w);
                    float dv = J.vort * dt * (nx * w);
                    if (finite_f(du) && finite_f(dv) && du * du + dv * dv <= 0.0625f) {
                        J.u[g] += du;
                        J.v[g] += dv;
                    }
                }
            }
        })
        __syncthreads();
    }
    CTA_RECT(b.i0, b.i1, b.j0, b.j1, {
        if (J.h[g] > eps) {
            float decay = J.nu_const ? decay_w : expf(-sheet_damp(job_nu(J, A, g)) * dt);
            J.u[g] = finite_speed(J.u[g] * decay, kSpeedCap);
            J.v[g] = finite_speed(J.v[g] * decay, kSpeedCap);
        }
    })
    __syncthreads();
    if (!do_flux) return;
    cta_transport(J, A, res, b, dt);
    cta_dry_cut(J, res, b, eps);
}

// awake_work_boxes (src/fluid_core.rs:1537-1657) into S.bbox / S.nbox.
__device__ void cta_awake_boxes(Shared& S, const Job& J, const Args& A, int res) {
    const int tiles = (res + SLEEP_TILE - 1) / SLEEP_TILE;
    const int ntile = tiles * tiles;
    for (int t = threadIdx.x; t < ntile; t += NT) {
        S.hot[t] = 0;
        S.grown[t] = 0;
    }
    __syncthreads();
    const float eps = A.eps, cell = A.cell;
    CTA_RECT(0, res - 1, 0, res - 1, {
        float hv = J.h[g];
        if (hv > eps) {
            bool awake = hypotf(J.u[g], J.v[g]) > 0.05f;
            if (!awake) {
                float eta = J.bed[g] + hv;
                int ip = i + 1 < res ? g + 1 : g;
                int jp = j + 1 < res ? g + res : g;
                float dex = fabsf(J.bed[ip] + J.h[ip] - eta);
                float dez = fabsf(J.bed[jp] + J.h[jp] - eta);
                awake = fmaxf(dex, dez) > 0.02f * cell;
            }
            if (awake) S.hot[(j / SLEEP_TILE) * tiles + i / SLEEP_TILE] = 1;
        }
    })
    __syncthreads();
    for (int t = threadIdx.x; t < ntile; t += NT) {
        int ti = t % tiles, tj = t / tiles;
        unsigned char gr = 0;
        for (int dj = -1; dj <= 1; ++dj)
            for (int di = -1; di <= 1; ++di) {
                int ni = ti + di, nj = tj + dj;
                if (ni >= 0 && nj >= 0 && ni < tiles && nj < tiles && S.hot[nj * tiles + ni]) gr = 1;
            }
        S.grown[t] = gr;
        S.lab[t] = gr ? t : 0x7fffffff;
    }
    __syncthreads();
    // Components of grown tiles by min-label propagation; the label is the
    // component's first tile in raster order, the order the reference's scan finds them.
    for (int iter = 0; iter < 4 * MAX_TILES; ++iter) {
        if (threadIdx.x == 0) S.changed = 0;
        __syncthreads();
        for (int t = threadIdx.x; t < ntile; t += NT) {
            if (!S.grown[t]) continue;
            int ti = t % tiles, tj = t / tiles;
            int m = S.lab[t];
            if (ti > 0 && S.grown[t - 1]) m = min(m, S.lab[t - 1]);
            if (ti + 1 < tiles && S.grown[t + 1]) m = min(m, S.lab[t + 1]);
            if (tj > 0 && S.grown[t - tiles]) m = min(m, S.lab[t - tiles]);
            if (tj + 1 < tiles && S.grown[t + tiles]) m = min(m, S.lab[t + tiles]);
            m = min(m, S.lab[m]);
            if (m < S.lab[t]) {
                atomicMin(&S.lab[t], m);
                S.changed = 1;
            }
        }
        __syncthreads();
        if (!S.changed) break;
        __syncthreads();
    }
    // Boxes in root order.
    if (threadIdx.x == 0) {
        int nb = 0;
        for (int t = 0; t < ntile; ++t)
            if (S.grown[t] && S.lab[t] == t && nb < MAX_BOXES) {
                S.bbox[0][nb] = t % tiles;
                S.bbox[1][nb] = t % tiles;
                S.bbox[2][nb] = t / tiles;
                S.bbox[3][nb] = t / tiles;
                S.lab[t] = -(nb + 1);  // root slot marker, read below through the label chain
                ++nb;
            }
        S.nbox = nb;
    }
    __syncthreads();
    // Every grown tile joins its root's box (roots now hold -(box+1)).
    for (int t = threadIdx.x; t < ntile; t += NT) {
        if (!S.grown[t]) continue;
        int r = S.lab[t];
        int slot = r < 0 ? -r - 1 : -S.lab[r] - 1;
        if (slot < 0 || slot >= MAX_BOXES) continue;
        int ti = t % tiles, tj = t / tiles;
        atomicMin(&S.bbox[0][slot], ti);
        atomicMax(&S.bbox[1][slot], ti);
        atomicMin(&S.bbox[2][slot], tj);
        atomicMax(&S.bbox[3][slot], tj);
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < S.nbox; ++k) {
            int ti0 = S.bbox[0][k], ti1 = S.bbox[1][k], tj0 = S.bbox[2][k], tj1 = S.bbox[3][k];
            S.bbox[0][k] = ti0 * SLEEP_TILE;
            S.bbox[1][k] = min((ti1 + 1) * SLEEP_TILE, res) - 1;
            S.bbox[2][k] = tj0 * SLEEP_TILE;
            S.bbox[3][k] = min((tj1 + 1) * SLEEP_TILE, res) - 1;
        }
    __syncthreads();
}

__device__ __forceinline__ bool boxes_touch(int a0, int a1, int a2, int a3, int b0, int b1, int b2, int b3) {
    auto ss = [](int x) { return x > 0 ? x - 1 : 0; };
    return ss(a0) <= b1 + 1 && ss(b0) <= a1 + 1 && ss(a2) <= b3 + 1 && ss(b2) <= a3 + 1;
}

// sheet_work_boxes (src/fluid_core.rs:1325-1447) into S.bbox / S.nbox. Wet
// bodies are labelled in the f2 plane (as ints) by min-label propagation; a
// body's label is its first wet cell in raster order.
__device__ void cta_wet_boxes(Shared& S, const Job& J, const Args& A, int res) {
    const float eps = A.eps;
    int v[4] = {0, res, 0, res};  // wet count, i0, (i1 via -), j0
    int vi1 = -1, vj1 = -1;
    CTA_RECT(0, res - 1, 0, res - 1, {
        if (J.h[g] > eps) {
            v[0] += 1;
            v[1] = min(v[1], i);
            vi1 = max(vi1, i);
            v[3] = min(v[3], j);
            vj1 = max(vj1, j);
        }
    })
    v[2] = -vi1;
    {
        const int op[4] = {0, 1, 1, 1};
        int t[4] = {v[0], v[1], v[2], v[3]};
        block_reduce4(S, t, op);
        v[0] = t[0];
        v[1] = t[1];
        vi1 = -t[2];
        v[3] = t[3];
    }
    {
        const int op[4] = {2, 2, 2, 2};
        int t[4] = {vj1, 0, 0, 0};
        block_reduce4(S, t, op);
        vj1 = t[0];
    }
    const int wet = v[0], i0 = v[1], i1 = vi1, j0 = v[3], j1 = vj1;
    if (wet == 0) {
        if (threadIdx.x == 0) S.nbox = 0;
        __syncthreads();
        return;
    }
    const int x0 = max(i0 - 3, 0), x1 = min(i1 + 3, res - 1), y0 = max(j0 - 3, 0), y1 = min(j1 + 3, res - 1);
    const bool solid = wet == (i1 - i0 + 1) * (j1 - j0 + 1);
    if (solid) {
        if (threadIdx.x == 0) {
            S.nbox = 1;
            S.bbox[0][0] = x0;
            S.bbox[1][0] = x1;
            S.bbox[2][0] = y0;
            S.bbox[3][0] = y1;
        }
        __syncthreads();
        return;
    }
    int* L = reinterpret_cast<int*>(J.f2);
    CTA_RECT(0, res - 1, 0, res - 1, { L[g] = J.h[g] > eps ? g : -1; })
    __syncthreads();
    for (int iter = 0; iter < res * res; ++iter) {
        if (threadIdx.x == 0) S.changed = 0;
        __syncthreads();
        CTA_RECT(i0, i1, j0, j1, {
            int m = L[g];
            if (m >= 0) {
                if (i > 0 && L[g - 1] >= 0) m = min(m, L[g - 1]);
                if (i + 1 < res && L[g + 1] >= 0) m = min(m, L[g + 1]);
                if (j > 0 && L[g - res] >= 0) m = min(m, L[g - res]);
                if (j + 1 < res && L[g + res] >= 0) m = min(m, L[g + res]);
                m = min(m, L[m]);
                if (m < L[g]) {
                    atomicMin(&L[g], m);
                    S.changed = 1;
                }
            }
        })
        __syncthreads();
        if (!S.changed) break;
        __syncthreads();
    }
    // Bodies in first-cell order, with their bounding boxes and the split halo of 6.
    if (threadIdx.x == 0) {
        int nb = 0;
        bool over = false;
        for (int j = j0; j <= j1 && !over; ++j)
            for (int i = i0; i <= i1; ++i) {
                int g = j * res + i;
                if (L[g] == g) {
                    if (nb >= MAX_BOXES) {
                        over = true;
                        break;
                    }
                    S.bbox[0][nb] = i;
                    S.bbox[1][nb] = i;
                    S.bbox[2][nb] = j;
                    S.bbox[3][nb] = j;
                    L[g] = -(nb + 2);
                    ++nb;
                }
            }
        S.nbox = over ? -1 : nb;
    }
    __syncthreads();
    if (S.nbox < 0) {  // more bodies than slots: merged boxes would exceed 8, the whole box applies
        if (threadIdx.x == 0) {
            S.nbox = 1;
            S.bbox[0][0] = x0;
            S.bbox[1][0] = x1;
            S.bbox[2][0] = y0;
            S.bbox[3][0] = y1;
        }
        __syncthreads();
        return;
    }
    CTA_RECT(i0, i1, j0, j1, {
        int r = L[g];
        if (r >= 0 || r <= -2) {
            int slot = r >= 0 ? -L[r] - 2 : -r - 2;
            if (slot >= 0 && slot < MAX_BOXES) {
                atomicMin(&S.bbox[0][slot], i);
                atomicMax(&S.bbox[1][slot], i);
                atomicMin(&S.bbox[2][slot], j);
                atomicMax(&S.bbox[3][slot], j);
            }
        }
    })
    __syncthreads();
    if (threadIdx.x == 0) {
        int nb = S.nbox;
        for (int k = 0; k < nb; ++k) {
            S.bbox[0][k] = max(S.bbox[0][k] - 6, 0);
            S.bbox[1][k] = min(S.bbox[1][k] + 6, res - 1);
            S.bbox[2][k] = max(S.bbox[2][k] - 6, 0);
            S.bbox[3][k] = min(S.bbox[3][k] + 6, res - 1);
        }
        // merge_boxes (src/fluid_core.rs:1459-1487), swap_remove order.
        for (;;) {
            bool did = false;
            int a = 0;
            while (a < nb) {
                int c = a + 1;
                while (c < nb) {
                    if (boxes_touch(S.bbox[0][a], S.bbox[1][a], S.bbox[2][a], S.bbox[3][a], S.bbox[0][c],
                                    S.bbox[1][c], S.bbox[2][c], S.bbox[3][c])) {
                        S.bbox[0][a] = min(S.bbox[0][a], S.bbox[0][c]);
                        S.bbox[1][a] = max(S.bbox[1][a], S.bbox[1][c]);
                        S.bbox[2][a] = min(S.bbox[2][a], S.bbox[2][c]);
                        S.bbox[3][a] = max(S.bbox[3][a], S.bbox[3][c]);
                        for (int q = 0; q < 4; ++q) S.bbox[q][c] = S.bbox[q][nb - 1];
                        --nb;
                        did = true;
                    } else {
                        ++c;
                    }
                }
                ++a;
            }
            if (!did) break;
        }
        if (nb == 1 || nb > 8) {
            nb = 1;
            S.bbox[0][0] = x0;
            S.bbox[1][0] = x1;
            S.bbox[2][0] = y0;
            S.bbox[3][0] = y1;
        }
        S.nbox = nb;
    }
    __syncthreads();
}

// step_sheet_eps_in + step_sheet_scratch (src/fluid_core.rs:821-852, :1659-1831)
// for one open 2 cm layer of one patch.
__global__ void __launch_bounds__(NT, 1) k_patch_step(Args A) {
    const Job J = A.jobs[blockIdx.x];
    if (!J.active) return;
    __shared__ Shared S;
    const int res = A.res;
    const float eps = A.eps;
    // Early out on an effectively dry sheet (wet_sum, src/fluid_core.rs:1306-1319).
    double ws = 0.0;
    CTA_RECT(0, res - 1, 0, res - 1, {
        float hv = J.h[g];
        if (hv > eps) ws += (double)hv;
    })
    ws = block_sum_d(S, ws);
    if (!(ws > (double)eps)) return;
    const bool fine_open = A.pace == 0;
    const bool whole_wet = A.pace == 2 || A.pace == 3;
    if (whole_wet)
        cta_wet_boxes(S, J, A, res);
    else
        cta_awake_boxes(S, J, A, res);
    const int nb = S.nbox;
    if (nb <= 0) return;
    const float cap = rclamp(A.sub_cap, 1.0f, 8.0f);
    int nsub = 1;
    if (!fine_open) {
        float m2 = 0.0f;
        for (int k = 0; k < nb; ++k) {
            Box b = {S.bbox[0][k], S.bbox[1][k], S.bbox[2][k], S.bbox[3][k]};
            CTA_RECT(b.i0, b.i1, b.j0, b.j1, {
                float uu = J.u[g], vv = J.v[g];
                float s2 = uu * uu + vv * vv;
                if (s2 > m2) m2 = s2;
            })
        }
        m2 = block_max_f(S, m2);
        float max_s = fmaxf(0.15f, sqrtf(m2));
        nsub = (int)rclamp(ceilf((A.dt * max_s) / (0.42f * fmaxf(A.cell, 1.0e-3f))), 1.0f, cap);
    }
    const float dts = A.dt / (float)nsub;
    const float decay_w = A.decay_w[nsub];
    float* set0[5] = {J.sc[0][0], J.sc[0][1], J.sc[0][2], J.sc[0][3], J.sc[0][4]};
    float* set1[5] = {J.sc[1][0], J.sc[1][1], J.sc[1][2], J.sc[1][3], J.sc[1][4]};
    auto apart = [&](int a, int c) {
        auto ap = [](int a0, int a1, int b0, int b1) { return a1 + 6 < b0 || b1 + 6 < a0; };
        return ap(S.bbox[0][a], S.bbox[1][a], S.bbox[0][c], S.bbox[1][c]) ||
               ap(S.bbox[2][a], S.bbox[3][a], S.bbox[2][c], S.bbox[3][c]);
    };
    const bool two_apart = A.has_sc2 && nb == 2 && apart(0, 1);
    if (A.pace == 3 && whole_wet && nsub > 1) {
        for (int k = 0; k < nb; ++k) {
            Box b = {S.bbox[0][k], S.bbox[1][k], S.bbox[2][k], S.bbox[3][k]};
            float* const* sc = (two_apart && k == 1) ? set1 : set0;
            cta_substep(J, A, res, b, sc, A.dt, A.decay_w[1], false);
            for (int s = 0; s < nsub; ++s) cta_transport(J, A, res, b, dts);
            cta_dry_cut(J, res, b, eps);
        }
        return;
    }
    for (int s = 0; s < nsub; ++s)
        for (int k = 0; k < nb; ++k) {
            Box b = {S.bbox[0][k], S.bbox[1][k], S.bbox[2][k], S.bbox[3][k]};
            float* const* sc = (two_apart && k == 1) ? set1 : set0;
            cta_substep(J, A, res, b, sc, dts, decay_w, true);
        }
}

cudaError_t launch_patch_step(const Args& A, int njobs, cudaStream_t st) {
    if (njobs <= 0) return cudaSuccess;
    k_patch_step<<<njobs, NT, 0, st>>>(A);
    return cudaGetLastError();
}

size_t patch_static_smem() { return sizeof(Shared); }

}  // namespace patch
}  // namespace silt
