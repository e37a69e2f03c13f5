// Full-grid sheet substep for the coarse window and large grids.
//
// One substep of the reference (`substep`, x3-team/Dirty-gen
// src/fluid_core.rs:1879-2082) is split in two fused, tiled kernels:
//
//   k_force      eta = bed + h, the two 5-tap pressure blurs, gravity,
//                snapshot-Jacobi vorticity confinement, the divergence
//                "overload" projection (its own two blurs), damping and the
//                speed clamp. Reads h, bed, u, v (and grain/moisture for the
//                slurry), writes the new u, v. All intermediates live in
//                shared memory; the tile carries a 9-cell halo.
//   k_transport  donor-cell transport of depth, x pass then z pass, the dry
//                cut, and the FP64 ledger partial sum. Reads h, u, v, writes h.
//
// Both layers (water, slurry) go in one launch (blockIdx.z). Every stencil
// clamps its index at the grid edge exactly as the reference's edge branches
// do, so interior and border cells follow one formula.
//
// Work-box semantics: the reference steps only cells inside its work boxes
// (wet bounding box + 3, or split bodies + 6). A wet cell is always at least 3
// cells inside its box when a step has one substep, so every value a wet cell
// reads is a value the full-grid pass computes the same way; dry cells carry
// no flux and no force. The full-grid pass therefore gives the reference's
// depths and velocities on every cell that holds fluid.
#include <cstdint>
#include <mutex>
#include <vector>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include "sheet_grid.cuh"
#include "sheet_math.cuh"
#include "launch_count.cuh"

namespace silt {

constexpr int FT = 32;       // force tile edge
constexpr int FH = 9;        // force halo: p (2) + gravity (1) + vorticity (2) + projection (4)
constexpr int FW = FT + 2 * FH;
constexpr int FPLANE = FW * FW;
constexpr int FORCE_THREADS = 512;

constexpr int TT = 32;       // transport tile edge
constexpr int TW = TT + 3;   // rows [t0-2, t1+1)
// A transport plane in shared memory: rows [ty0-2, ty0+33), each TS cells from
// column tx0-4 (16 bytes below tx0-2, so that a 2D TMA box can start there),
// padded to 128 bytes.
constexpr int TS = TT + 8;
constexpr int TPL = (TS * TW + 31) / 32 * 32;
static_assert((TS * sizeof(float)) % 16 == 0, "a TMA box row is a multiple of 16 bytes");
static_assert((TPL * sizeof(float)) % 128 == 0, "each transport plane starts 128-byte aligned");
static_assert(TS * TW * sizeof(float) <= TPL * sizeof(float), "a TMA box fits its plane");
constexpr int TRANSPORT_THREADS = 256;

size_t force_smem_bytes() { return sizeof(float) * FPLANE * 8; }
size_t transport_smem_bytes() { return sizeof(float) * TPL * 8; }

// Five taps left to right. Away from the edge the reference starts from the
// first product (accum5); near it from 0.0 (accum5_clamped,
// src/fluid_core.rs:3680-3697).
__device__ __forceinline__ float tap5(float a0, float a1, float a2, float a3, float a4, float k0, float k1, float k2,
                                      bool interior) {
    float a = interior ? a0 * k0 : 0.0f + a0 * k0;
    a += a1 * k1;
    a += a2 * k2;
    a += a3 * k1;
    a += a4 * k0;
    return a;
}

__device__ __forceinline__ int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

// The layer's substep count from its largest squared speed, in the host's
// arithmetic (IEEE sqrt and divide, no contraction).
__device__ __forceinline__ int device_nsub(const SubstepCount& c, int l) {
    const float m2 = __uint_as_float(c.speed2[l]);
    const float max_s = fmaxf(0.15f, sqrtf(m2));
    const float ns = ceilf((c.dt * max_s) / (0.42f * fmaxf(c.cell, 1.0e-3f)));
    return (int)rclamp(ns, 1.0f, c.cap);
}

// One flag plane by layer and buffer, without indexing the parameter array
// by a runtime value (which would copy it to local memory).
__device__ __forceinline__ uint8_t* pick(uint8_t* const (&a)[2][2], int l, int b) {
    return l ? (b ? a[1][1] : a[1][0]) : (b ? a[0][1] : a[0][0]);
}

// Tile-list entry: layer, zero-fill and copy bits over the tile index.
constexpr int ENTRY_ZERO = 1 << 29;
constexpr int ENTRY_COPY = 1 << 28;
constexpr int ENTRY_TILE = (1 << 28) - 1;

// Clears a sweep launch's barrier count and pass verdicts (the tile-list
// kernel does, before each force launch).
__device__ __forceinline__ void clear_sweep(SweepState* S) {
    if (!S) return;
    S->bar = 0u;
    S->flag[0] = S->flag[1] = S->flag[2] = 0u;
}

// Cell material: viscosity, mobility and damping factor.
__device__ __forceinline__ float cell_nu(const LayerParams& P, size_t g) {
    if (P.nu_mode == NU_CONST) return P.nu_c;
    if (P.nu_mode == NU_PLANE || P.nu_mode == NU_TABLE) return P.nu_plane[g];
    return dynamic_viscosity(P.grain[g], P.moisture[g]);
}

// sheet_mobility_for(nu) of the cell.
__device__ __forceinline__ float cell_mob(const LayerParams& P, size_t g) {
    if (P.nu_mode == NU_CONST) return P.mob_c;
    if (P.nu_mode == NU_TABLE) return P.mob_plane[g];
    return sheet_mobility_for(cell_nu(P, g));
}

// The cell's damping factor over dt: exp(-sheet_damp(nu) dt), the
// double-precision exponential rounded once (as the window engine does).
__device__ __forceinline__ float cell_decay(const LayerParams& P, size_t g, float dt) {
    if (P.nu_mode == NU_CONST) return P.decay_c;
    const float rate = P.nu_mode == NU_TABLE ? P.damp_plane[g] : sheet_damp(cell_nu(P, g));
    return exp_rn(-rate * dt);
}

// Every cell of the tile's region of radius (RX, RY): f(gx, gy, s, g) with s
// the shared-memory index and g the global one. Edge tiles clip the region to
// the grid and walk it one warp per row; interior tiles walk the rectangle as
// one flat range (a compile-time width), which keeps every lane busy.
template <bool EDGE, int RX, int RY, class F>
__device__ __forceinline__ void region(int tx0, int ty0, int res, F f) {
    const int ox = tx0 - FH, oy = ty0 - FH;
    if (EDGE) {
        const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
        constexpr int NW = FORCE_THREADS / 32;
        const int x0 = max(0, tx0 - RX), x1 = min(res, tx0 + FT + RX);
        const int y0 = max(0, ty0 - RY), y1 = min(res, ty0 + FT + RY);
        for (int gy = y0 + wy; gy < y1; gy += NW)
            for (int gx = x0 + lane; gx < x1; gx += 32)
                f(gx, gy, (gy - oy) * FW + (gx - ox), (size_t)gy * res + gx);
    } else {
        constexpr int W = FT + 2 * RX, H = FT + 2 * RY;
        for (int k = threadIdx.x; k < W * H; k += FORCE_THREADS) {
            const int r = k / W;
            const int gy = ty0 - RY + r, gx = tx0 - RX + (k - r * W);
            f(gx, gy, (gy - oy) * FW + (gx - ox), (size_t)gy * res + gx);
        }
    }
}

// The velocity a substep starts from at (gx, gy): the lazy dry cut of the
// previous substep, then the soft window border (src/fluid_core.rs:9594-9622;
// a river reach's band keeps its current through the window ends).
__device__ __forceinline__ void start_velocity(const LayerParams& P, int gx, int gy, size_t g, float hv, float& uu,
                                               float& vv) {
    uu = P.u[g];
    vv = P.v[g];
    if (P.apply_cut && hv < P.eps) {
        uu = 0.0f;
        vv = 0.0f;
    }
    if (P.soften_edge > 0) {
        const int res = P.res;
        const int dx = min(gx, res - 1 - gx), dz = min(gy, res - 1 - gy);
        int d = min(dx, dz);
        if (P.open_axis == 1 && gy >= P.open_c0 && gy < P.open_c1) d = dz;
        else if (P.open_axis == 2 && gx >= P.open_c0 && gx < P.open_c1) d = dx;
        if (d < P.soften_edge) {
            float t = (float)d / (float)P.soften_edge;
            float w = t * t * (3.0f - 2.0f * t);
            uu *= w;
            vv *= w;
        }
    }
}

// Shared-memory planes of a force tile (FW x FW floats each, origin at the
// tile corner minus FH).
struct ForcePlanes {
    float* E;   // eta
    float* TG;  // x-pass scratch
    float* TS;
    float* PB;  // pressure p, then projection b
    float* U;   // u, v
    float* V;
    float* HS;  // depth
    float* WQ;  // vorticity, then q
    __device__ explicit ForcePlanes(float* sm)
        : E(sm), TG(sm + FPLANE), TS(sm + 2 * FPLANE), PB(sm + 3 * FPLANE), U(sm + 4 * FPLANE), V(sm + 5 * FPLANE),
          HS(sm + 6 * FPLANE), WQ(sm + 7 * FPLANE) {}
};

#define NX(d) (EDGE ? (gy - oy) * FW + (clampi(gx + (d), 0, res - 1) - ox) : s + (d))
#define NZ(d) (EDGE ? (clampi(gy + (d), 0, res - 1) - oy) * FW + (gx - ox) : s + (d) * FW)

// Depth and eta on radius R + 2, then the pressure p = 0.45 (0.62 G + 0.38 S)
// + 0.55 eta on radius R (src/fluid_core.rs:1950-1985): the two 5-tap blurs,
// x pass then z pass. Ends with a barrier.
template <bool EDGE, int R>
__device__ __forceinline__ void pressure_field(const LayerParams& P, const ForcePlanes& F, int tx0, int ty0) {
    const int res = P.res;
    const int ox = tx0 - FH, oy = ty0 - FH;
    region<EDGE, R + 2, R + 2>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
        float hv = P.h[g];
        F.HS[s] = hv;
        F.E[s] = P.bed[g] + hv;
    });
    __syncthreads();
    region<EDGE, R, R + 2>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
        const bool in = EDGE ? (gx >= 2 && gx <= res - 3) : true;
        float e0 = F.E[NX(-2)], e1 = F.E[NX(-1)], e2 = F.E[s], e3 = F.E[NX(1)], e4 = F.E[NX(2)];
        F.TG[s] = tap5(e0, e1, e2, e3, e4, kG0, kG1, kG2, in);
        F.TS[s] = tap5(e0, e1, e2, e3, e4, kS0, kS1, kS2, in);
    });
    __syncthreads();
    region<EDGE, R, R>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
        const bool in = EDGE ? (gy >= 2 && gy <= res - 3) : true;
        const int s0 = NZ(-2), s1 = NZ(-1), s3 = NZ(1), s4 = NZ(2);
        float gb = tap5(F.TG[s0], F.TG[s1], F.TG[s], F.TG[s3], F.TG[s4], kG0, kG1, kG2, in);
        float sc = tap5(F.TS[s0], F.TS[s1], F.TS[s], F.TS[s3], F.TS[s4], kS0, kS1, kS2, in);
        float filtered = 0.62f * gb + 0.38f * sc;
        F.PB[s] = 0.45f * filtered + 0.55f * F.E[s];
    });
    __syncthreads();
}

// Projection, damping and the speed clamp from the confined velocity in U, V
// (radius 4), depth and eta (radius 4) (src/fluid_core.rs:1992-2037). Writes
// every cell of the tile to u_out, v_out.
template <bool EDGE>
__device__ __forceinline__ void finish_tile(const LayerParams& P, const ForcePlanes& F, int tx0, int ty0) {
    const int res = P.res;
    const int ox = tx0 - FH, oy = ty0 - FH;
    const float dt = P.dt, eps = P.eps;
    if (P.project) {
        // b = div * overload - 0.015 * overload * lap(eta), radius 3 (:1992-2003).
        region<EDGE, 3, 3>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
            const int sxp = NX(1), sxm = NX(-1), szp = NZ(1), szm = NZ(-1);
            float ux = fdiv(F.U[sxp] - F.U[sxm], P.div_two);
            float vz = fdiv(F.V[szp] - F.V[szm], P.div_two);
            float div = ux + vz;
            float lsum = F.E[sxp] + F.E[sxm] + F.E[szp] + F.E[szm] - 4.0f * F.E[s];
            float lap_h = fdiv(lsum, P.div_cell2);
            float overload = 1.0f + rclamp(fdiv(cell_nu(P, g), P.div_231), 0.0f, 6.0f);
            F.PB[s] = div * overload - 0.015f * overload * lap_h;
        });
        __syncthreads();
        // x pass of both blurs of b: rows radius 3, columns radius 1.
        region<EDGE, 1, 3>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
            const bool in = EDGE ? (gx >= 2 && gx <= res - 3) : true;
            float b0 = F.PB[NX(-2)], b1 = F.PB[NX(-1)], b2 = F.PB[s], b3 = F.PB[NX(1)], b4 = F.PB[NX(2)];
            F.TG[s] = tap5(b0, b1, b2, b3, b4, kG0, kG1, kG2, in);
            F.TS[s] = tap5(b0, b1, b2, b3, b4, kS0, kS1, kS2, in);
        });
        __syncthreads();
        // q = 0.62 G(b) + 0.38 S(b), radius 1 (:2004-2011).
        region<EDGE, 1, 1>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
            const bool in = EDGE ? (gy >= 2 && gy <= res - 3) : true;
            const int s0 = NZ(-2), s1 = NZ(-1), s3 = NZ(1), s4 = NZ(2);
            float gq = tap5(F.TG[s0], F.TG[s1], F.TG[s], F.TG[s3], F.TG[s4], kG0, kG1, kG2, in);
            float sq = tap5(F.TS[s0], F.TS[s1], F.TS[s], F.TS[s3], F.TS[s4], kS0, kS1, kS2, in);
            F.WQ[s] = 0.62f * gq + 0.38f * sq;
        });
        __syncthreads();
    }
    // Projection kick, damping and the speed clamp on wet cells (:2015-2037).
    region<EDGE, 0, 0>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
        float uu = F.U[s], vv = F.V[s];
        if (F.HS[s] > eps) {
            if (P.project) {
                float qx = fdiv(F.WQ[NX(1)] - F.WQ[NX(-1)], P.div_two);
                float qz = fdiv(F.WQ[NZ(1)] - F.WQ[NZ(-1)], P.div_two);
                uu += 0.012f * dt * qx;
                vv += 0.012f * dt * qz;
            }
            float decay = cell_decay(P, g, dt);
            uu = finite_speed(uu * decay, kSpeedCap);
            vv = finite_speed(vv * decay, kSpeedCap);
        }
        P.u_out[g] = uu;
        P.v_out[g] = vv;
    });
}

// One force tile in the snapshot (Jacobi) form. EDGE = false for tiles whose
// whole radius-9 region lies at least 2 cells inside the grid: no index is
// ever clamped there and every blur uses the interior form, so the stencils
// are plain offsets. Threads walk the regions as rows (one warp per row,
// lanes along x).
template <bool EDGE>
__device__ __forceinline__ void force_tile(const LayerParams& P, float* sm, int tx0, int ty0) {
    const int res = P.res;
    const ForcePlanes F(sm);
    const int ox = tx0 - FH, oy = ty0 - FH;
    const float dt = P.dt, eps = P.eps;
    // 1-3. Depth, eta (radius 9) and the pressure (radius 7).
    pressure_field<EDGE, 7>(P, F, tx0, ty0);
    // Velocity on radius 6 and gravity down the pressure gradient on wet
    // cells (src/fluid_core.rs:2234-2253).
    region<EDGE, 6, 6>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
        float uu, vv;
        start_velocity(P, gx, gy, g, F.HS[s], uu, vv);
        if (F.HS[s] > eps) {
            float px = fdiv(F.PB[NX(1)] - F.PB[NX(-1)], P.div_two);
            float pz = fdiv(F.PB[NZ(1)] - F.PB[NZ(-1)], P.div_two);
            float mob = cell_mob(P, g);
            uu += -kGravity * px * mob * dt;
            vv += -kGravity * pz * mob * dt;
        }
        F.U[s] = uu;
        F.V[s] = vv;
    });
    __syncthreads();
    // Vorticity of the post-gravity snapshot, radius 5 (src/fluid_core.rs:3498-3506).
    if (P.vort > 0.0f) {
        region<EDGE, 5, 5>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
            float dvdx = fdiv(F.V[NX(1)] - F.V[NX(-1)], P.div_two);
            float dudz = fdiv(F.U[NZ(1)] - F.U[NZ(-1)], P.div_two);
            F.WQ[s] = dvdx - dudz;
        });
        __syncthreads();
        // Confinement kick from that snapshot, in place, radius 4
        // (src/fluid_core.rs:2348-2375, :2441-2470).
        region<EDGE, 4, 4>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
            if (F.HS[s] > eps) {
                float w = F.WQ[s];
                if (finite_f(w) && !(fabsf(w) < 1.0e-4f)) {
                    float wxp = fabsf(F.WQ[NX(1)]), wxm = fabsf(F.WQ[NX(-1)]);
                    float wzp = fabsf(F.WQ[NZ(1)]), wzm = fabsf(F.WQ[NZ(-1)]);
                    float nx_ = fdiv(wxp - wxm, P.div_two);
                    float nz_ = fdiv(wzp - wzm, P.div_two);
                    float du = P.vort * dt * (-nz_ * w);
                    float dv = P.vort * dt * (nx_ * w);
                    if (finite_f(du) && finite_f(dv) && du * du + dv * dv <= 0.0625f) {
                        F.U[s] += du;
                        F.V[s] += dv;
                    }
                }
            }
        });
        __syncthreads();
    }
    finish_tile<EDGE>(P, F, tx0, ty0);
}

// Sweep form, part 1: the post-gravity velocity G of every cell of the tile
// (gravity on wet cells only; a dry cell keeps its starting velocity), written
// to u_out, v_out, and the sweep's first iterate F = G to fu, fv.
template <bool EDGE>
__device__ __forceinline__ void pre_tile(const LayerParams& P, float* sm, int tx0, int ty0) {
    const int res = P.res;
    const ForcePlanes F(sm);
    const int ox = tx0 - FH, oy = ty0 - FH;
    const float dt = P.dt, eps = P.eps;
    pressure_field<EDGE, 1>(P, F, tx0, ty0);
    region<EDGE, 0, 0>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
        float uu, vv;
        start_velocity(P, gx, gy, g, F.HS[s], uu, vv);
        if (F.HS[s] > eps) {
            float px = fdiv(F.PB[NX(1)] - F.PB[NX(-1)], P.div_two);
            float pz = fdiv(F.PB[NZ(1)] - F.PB[NZ(-1)], P.div_two);
            float mob = cell_mob(P, g);
            uu += -kGravity * px * mob * dt;
            vv += -kGravity * pz * mob * dt;
        }
        P.u_out[g] = uu;
        P.v_out[g] = vv;
        P.fu[g] = uu;
        P.fv[g] = vv;
    });
}

// Local passes of the sweep's fixed point on one tile before its values go
// back to global memory.
#ifndef SILT_SWEEP_LOCAL_PASSES
#define SILT_SWEEP_LOCAL_PASSES 16
#endif
constexpr int SWEEP_LOCAL_PASSES = SILT_SWEEP_LOCAL_PASSES;

// Sweep form, part 2: one pass of the raster-order Gauss-Seidel confinement
// (force_gravity_open, src/fluid_core.rs:2234-2260) solved as a fixed point.
// In the reference's sweep a wet cell's final velocity is its post-gravity
// value G plus the kick computed from the final values of the cells before it
// in raster order, its own G, and the starting values of the cells after it;
// dry cells never change. The tile iterates that equation for its own wet
// cells in shared memory, reading the current iterate of other tiles' cells
// from fu, fv, until a local pass changes no bit, and writes back what
// changed. Returns true (block-uniform) when any value of the tile changed.
// When a whole pass over every tile changes nothing, every cell satisfies its
// equation with the values it read, and since each cell depends only on
// earlier cells that solution is the sequential sweep's, bit for bit.
// `reuse`: this CTA's shared memory still holds this tile from an earlier
// pass of the launch (the CTA solves no other tile), so only the ring of
// other tiles' wet cells around it is read again; the starting and
// post-gravity velocities and the tile's own iterate are current.
template <bool EDGE>
__device__ bool sweep_tile(const LayerParams& P, float* sm, int tx0, int ty0, bool reuse, int& passes) {
    const int res = P.res;
    float* PU = sm;              // starting velocity (the values of cells after a cell)
    float* PV = sm + FPLANE;
    float* FU = sm + 2 * FPLANE;  // current iterate (the values of cells before it)
    float* FV = sm + 3 * FPLANE;
    float* GU = sm + 4 * FPLANE;  // post-gravity velocity of the tile's own cells
    float* GV = sm + 5 * FPLANE;
    float* WT = sm + 6 * FPLANE;  // 1: wet
    const int ox = tx0 - FH, oy = ty0 - FH;
    const float eps = P.eps;
    if (reuse) {
        region<EDGE, 2, 2>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
            if (gx >= tx0 && gx < tx0 + FT && gy >= ty0 && gy < ty0 + FT) return;
            if (WT[s] != 0.0f) {
                FU[s] = P.fu[g];
                FV[s] = P.fv[g];
            }
        });
    } else region<EDGE, 2, 2>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
        const float hv = P.h[g];
        float uu, vv;
        start_velocity(P, gx, gy, g, hv, uu, vv);
        const bool wet = hv > eps;
        PU[s] = uu;
        PV[s] = vv;
        WT[s] = wet ? 1.0f : 0.0f;
        // A wet cell's tile is always stepped this substep, so its iterate
        // is current; a dry cell keeps its starting velocity.
        FU[s] = wet ? P.fu[g] : uu;
        FV[s] = wet ? P.fv[g] : vv;
        if (wet && gx >= tx0 && gx < tx0 + FT && gy >= ty0 && gy < ty0 + FT) {
            GU[s] = P.u_out[g];
            GV[s] = P.v_out[g];
        }
    });
    __syncthreads();
    bool tile_changed = false;
    passes = 0;
    // Interior tiles recompute, after the first local pass, only the cells
    // one of whose earlier-cell reads changed since they were last computed:
    // a cell whose inputs did not change keeps its value. A change at c
    // marks the cells that read c's iterate: c + (1,0), (2,0), (0,1),
    // (-1,1), (1,1), (0,2). Marks for pass it + 1 go to one byte plane while
    // pass it reads the other (plane 7 of the force layout, unused here).
    uint8_t* const marks = reinterpret_cast<uint8_t*>(sm + 7 * FPLANE);
    for (int it = 0; it < SWEEP_LOCAL_PASSES; ++it) {
        ++passes;
        int changed = 0;
        const uint8_t* dirty = marks + (it & 1) * FPLANE;
        uint8_t* dirty_next = marks + ((it + 1) & 1) * FPLANE;
        if (!EDGE) {
            region<false, 0, 0>(tx0, ty0, res, [&](int, int, int s, size_t) { dirty_next[s] = 0; });
            __syncthreads();
        }
        region<EDGE, 0, 0>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
            if (WT[s] == 0.0f) return;
            if (!EDGE) {
                // Interior tile: no stencil index is clamped.
                if (it > 0 && !dirty[s]) return;
                float du, dv, nu_ = GU[s], nv_ = GV[s];
                if (conf_kick_inner(P.div_two, P.dt, P.vort, SweepRead{FU, PU, GU, s, FW},
                                    SweepRead{FV, PV, GV, s, FW}, du, dv)) {
                    nu_ = GU[s] + du;
                    nv_ = GV[s] + dv;
                }
                if (__float_as_uint(nu_) != __float_as_uint(FU[s]) || __float_as_uint(nv_) != __float_as_uint(FV[s])) {
                    FU[s] = nu_;
                    FV[s] = nv_;
                    changed = 1;
                    dirty_next[s + 1] = 1;
                    dirty_next[s + 2] = 1;
                    dirty_next[s + FW - 1] = 1;
                    dirty_next[s + FW] = 1;
                    dirty_next[s + FW + 1] = 1;
                    dirty_next[s + 2 * FW] = 1;
                }
                return;
            }
            auto at = [&](int a, int b) { return (b - oy) * FW + (a - ox); };
            auto before = [&](int a, int b) { return b < gy || (b == gy && a < gx); };
            auto uu = [&](int a, int b) {
                if (a == gx && b == gy) return GU[s];
                return before(a, b) ? FU[at(a, b)] : PU[at(a, b)];
            };
            auto vv = [&](int a, int b) {
                if (a == gx && b == gy) return GV[s];
                return before(a, b) ? FV[at(a, b)] : PV[at(a, b)];
            };
            float du, dv, nu_ = GU[s], nv_ = GV[s];
            if (conf_kick(gx, gy, res, P.div_two, P.dt, P.vort, uu, vv, du, dv)) {
                nu_ = GU[s] + du;
                nv_ = GV[s] + dv;
            }
            if (__float_as_uint(nu_) != __float_as_uint(FU[s]) || __float_as_uint(nv_) != __float_as_uint(FV[s])) {
                FU[s] = nu_;
                FV[s] = nv_;
                changed = 1;
            }
        });
        if (!__syncthreads_or(changed)) break;
        tile_changed = true;
    }
    if (tile_changed) {
        region<EDGE, 0, 0>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
            if (WT[s] != 0.0f) {
                P.fu[g] = FU[s];
                P.fv[g] = FV[s];
            }
        });
    }
    __syncthreads();  // shared memory is read again by the next tile or pass
    return tile_changed;
}

// Sweep form, part 3: projection, damping and clamp from the solved sweep.
template <bool EDGE>
__device__ __forceinline__ void post_tile(const LayerParams& P, float* sm, int tx0, int ty0) {
    const int res = P.res;
    const ForcePlanes F(sm);
    const float eps = P.eps;
    region<EDGE, 4, 4>(tx0, ty0, res, [&](int gx, int gy, int s, size_t g) {
        const float hv = P.h[g];
        F.HS[s] = hv;
        F.E[s] = P.bed[g] + hv;
        float uu, vv;
        if (hv > eps) {
            uu = P.fu[g];
            vv = P.fv[g];
        } else {
            start_velocity(P, gx, gy, g, hv, uu, vv);
        }
        F.U[s] = uu;
        F.V[s] = vv;
    });
    __syncthreads();
    finish_tile<EDGE>(P, F, tx0, ty0);
}

#undef NX
#undef NZ

// A layer's force parameters for this substep: with a device count, its dt
// and (constant-viscosity layers) damping factor for that count.
__device__ __forceinline__ LayerParams force_params(const LayerParams& P0, const SubstepCount& sc, int l,
                                                    bool report_overflow) {
    LayerParams P = P0;
    if (sc.speed2) {
        const int ns = device_nsub(sc, l);
        P.dt = sc.dt / (float)ns;
        if (P.nu_mode == NU_CONST) P.decay_c = sc.water_decay[ns];
        if (report_overflow && sc.k == 0 && ns > sc.launched) atomicOr(sc.overflow, 1u);
    }
    return P;
}

// A tile whose whole radius-9 region lies at least 2 cells inside the grid:
// no stencil index is clamped there and every blur uses the interior form.
__device__ __forceinline__ bool tile_interior(int res, int tx0, int ty0) {
    return tx0 - FH >= 2 && ty0 - FH >= 2 && tx0 + FT + FH <= res - 2 && ty0 + FT + FH <= res - 2;
}

// One list entry of the force pass (the sweep form's first part for a
// sweeping layer). Returns true when it used shared memory.
__device__ __forceinline__ bool force_entry(const LayerParams& P, const TileFlags& tf, int nxt, int e, float* sm) {
    const int l = e >> 30, zero_fill = (e & ENTRY_ZERO) != 0, copy = (e & ENTRY_COPY) != 0, t = e & ENTRY_TILE;
    const int res = P.res;
    const int tx0 = (t % tf.tiles_x) * FT, ty0 = (t / tf.tiles_x) * FT;
    if (copy) {
        // Identity substep of a layer that has taken all its substeps.
        const int w = min(FT, res - tx0), h = min(FT, res - ty0);
        for (int q = threadIdx.x; q < w * h; q += blockDim.x) {
            const size_t g = (size_t)(ty0 + q / w) * res + tx0 + q % w;
            P.u_out[g] = P.u[g];
            P.v_out[g] = P.v[g];
        }
        if (threadIdx.x == 0) pick(tf.zero_uv, l, nxt)[t] = pick(tf.zero_uv, l, nxt ^ 1)[t];
        return false;
    }
    if (zero_fill) {
        // A quiet tile: dry in its whole neighbourhood, so after the dry cut
        // its velocity is zero.
        const int w = min(FT, res - tx0), h = min(FT, res - ty0);
        for (int q = threadIdx.x; q < w * h; q += blockDim.x) {
            const size_t g = (size_t)(ty0 + q / w) * res + tx0 + q % w;
            P.u_out[g] = 0.0f;
            P.v_out[g] = 0.0f;
        }
        if (threadIdx.x == 0) pick(tf.zero_uv, l, nxt)[t] = 1;
        return false;
    }
    const bool interior = tile_interior(res, tx0, ty0);
    if (P.sweep) {
        // Sweep form: this launch's first part; the sweep and the projection follow.
        if (interior)
            pre_tile<false>(P, sm, tx0, ty0);
        else
            pre_tile<true>(P, sm, tx0, ty0);
    } else if (interior) {
        force_tile<false>(P, sm, tx0, ty0);
    } else {
        force_tile<true>(P, sm, tx0, ty0);
    }
    if (threadIdx.x == 0) pick(tf.zero_uv, l, nxt)[t] = 0;
    return true;
}

// A list entry that steps its tile (neither a zero fill nor an identity copy).
__device__ __forceinline__ bool entry_steps(int e) { return (e & (ENTRY_ZERO | ENTRY_COPY)) == 0; }

// Sweep-form pass `pass` over one list entry: the fixed-point pass of a
// stepped tile of a sweeping layer with confinement on. After the first
// pass a tile is solved again only when some tile of its 3 x 3
// neighbourhood (itself included) changed since the previous pass began: it
// is otherwise still at the fixed point of the values around it. Returns
// whether the tile changed (block-uniform) and stamps it when it did.
// `reuse`: the CTA solves only this entry in the launch, so its shared
// memory keeps the tile between passes.
__device__ __forceinline__ bool sweep_entry(const LayerParams& P, const TileFlags& tf, int e, float* sm, int pass,
                                            unsigned int epoch, bool reuse) {
    if (!entry_steps(e) || !P.sweep || !(P.vort > 0.0f)) return false;
    const int l = e >> 30, t = e & ENTRY_TILE;
    const int nt = tf.tiles_x * tf.tiles_x;
    const int ti = t % tf.tiles_x, tj = t / tf.tiles_x;
    unsigned int* stamp = tf.stamp ? tf.stamp + (size_t)l * nt : nullptr;
    if (pass > 0 && stamp) {
        // Nine threads read the nine stamps at once.
        bool hit = false;
        if (threadIdx.x < 9) {
            const int x = ti + (int)(threadIdx.x % 3) - 1, y = tj + (int)(threadIdx.x / 3) - 1;
            const unsigned int since = epoch * 256u + (unsigned int)pass;
            hit = x >= 0 && y >= 0 && x < tf.tiles_x && y < tf.tiles_x &&
                  *(volatile unsigned int*)&stamp[y * tf.tiles_x + x] >= since;
        }
        if (!__syncthreads_or(hit)) return false;
    }
    const int tx0 = ti * FT, ty0 = tj * FT;
    int passes = 0;
    const bool keep = reuse && pass > 0;
    const bool changed = tile_interior(P.res, tx0, ty0) ? sweep_tile<false>(P, sm, tx0, ty0, keep, passes)
                                                        : sweep_tile<true>(P, sm, tx0, ty0, keep, passes);
    if (threadIdx.x == 0) {
        if (changed && stamp) {
            __threadfence();
            stamp[t] = epoch * 256u + (unsigned int)pass + 1u;
        }
        if (tf.sweep) {
            atomicAdd(&tf.sweep->solves, 1u);
            atomicAdd(&tf.sweep->local_passes, (unsigned int)passes);
        }
    }
    return changed;
}

// Sweep-form projection of one list entry. Returns true when it used shared memory.
__device__ __forceinline__ bool post_entry(const LayerParams& P, const TileFlags& tf, int e, float* sm) {
    if (!entry_steps(e) || !P.sweep) return false;
    const int t = e & ENTRY_TILE;
    const int tx0 = (t % tf.tiles_x) * FT, ty0 = (t / tf.tiles_x) * FT;
    if (tile_interior(P.res, tx0, ty0))
        post_tile<false>(P, sm, tx0, ty0);
    else
        post_tile<true>(P, sm, tx0, ty0);
    return true;
}

// ----------------------------------------------- Gauss-Seidel sweep launches
//
// The sweep's fixed point couples every stepped tile, so its passes run in
// one cooperative launch (every CTA resident at once) separated by a grid
// barrier. Each wait is bounded: past the limit the CTA records the failure
// in SweepState::err and the launch ends; the host reports SILT_ETIMEOUT.

constexpr int SWEEP_MAX_PASSES = 64;                  // then the sequential sweep
constexpr unsigned int SWEEP_SPIN_LIMIT = 1u << 22;   // polls of ~0.1 us: about half a second

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier of a cooperative launch: the arrival count only grows within
// a launch (the tile-list kernel clears it before), so barrier number k waits
// for k * gridDim.x arrivals. False when the wait gave up.
__device__ bool grid_barrier(SweepState* S, unsigned int& target) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        target += gridDim.x;
        __threadfence();
        atomicAdd(&S->bar, 1u);
        int good = 1;
        unsigned int spins = 0;
        while (ld_acquire_u32(&S->bar) < target) {
            if (++spins > SWEEP_SPIN_LIMIT) {
                atomicOr(&S->err, 1u);
                good = 0;
                break;
            }
            if (spins > 256) __nanosleep(64);  // short waits poll without sleeping
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Passes of the fixed point until one changes nothing anywhere. `visit(k)`
// runs list entry k's pass and returns whether it changed a value. Returns
// the number of passes, 0 at the pass limit, -1 after a failed barrier.
template <class Visit>
__device__ int sweep_fixed_point(SweepState* S, unsigned int& target, int n, Visit visit) {
    __shared__ unsigned int verdict;
    for (int pass = 0; pass < SWEEP_MAX_PASSES; ++pass) {
        bool changed = false;
        for (int k = blockIdx.x; k < n; k += gridDim.x) changed |= visit(k, pass);
        if (threadIdx.x == 0) {
            if (changed) atomicOr(&S->flag[pass % 3], 1u);
            // The next pass's verdict starts clear; the one cleared here was
            // last read before the previous barrier.
            if (blockIdx.x == 0) S->flag[(pass + 1) % 3] = 0u;
        }
        if (!grid_barrier(S, target)) return -1;
        if (threadIdx.x == 0) verdict = ld_acquire_u32(&S->flag[pass % 3]);
        __syncthreads();
        if (verdict == 0u) return pass + 1;
    }
    return 0;
}

// The sequential sweep of one layer on one thread (past the pass limit):
// every wet cell in raster order, as force_gravity_open does.
__device__ void sweep_serial(const LayerParams& P) {
    const int res = P.res;
    const float eps = P.eps;
    for (int j = 0; j < res; ++j)
        for (int i = 0; i < res; ++i) {
            const size_t g = (size_t)j * res + i;
            if (!(P.h[g] > eps)) continue;
            auto val = [&](bool is_u, int a, int b) {
                const size_t q = (size_t)b * res + a;
                if (a == i && b == j) return is_u ? P.u_out[q] : P.v_out[q];
                const float hq = P.h[q];
                if (hq > eps && (b < j || (b == j && a < i))) return is_u ? P.fu[q] : P.fv[q];
                float uu, vv;
                start_velocity(P, a, b, q, hq, uu, vv);
                return is_u ? uu : vv;
            };
            auto uu = [&](int a, int b) { return val(true, a, b); };
            auto vv = [&](int a, int b) { return val(false, a, b); };
            float du, dv, nu_ = P.u_out[g], nv_ = P.v_out[g];
            if (conf_kick(i, j, res, P.div_two, P.dt, P.vort, uu, vv, du, dv)) {
                nu_ = P.u_out[g] + du;
                nv_ = P.v_out[g] + dv;
            }
            P.fu[g] = nu_;
            P.fv[g] = nv_;
        }
}

// True when layer l takes a real (not identity) substep in this launch.
__device__ __forceinline__ bool layer_steps(const SubstepCount& sc, int l) {
    return !(sc.speed2 && sc.k > 0 && sc.k >= device_nsub(sc, l));
}

__device__ __forceinline__ void sweep_stats(SweepState* S, int passes) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(&S->launches, 1u);
        atomicAdd(&S->epoch, 1u);  // every CTA read the epoch at the launch's start, two barriers ago
        atomicMax(&S->passes_max, (unsigned int)(passes > 0 ? passes : SWEEP_MAX_PASSES));
        if (passes == 0) atomicAdd(&S->fallbacks, 1u);
    }
}

// One sheet's force pass in the sweep form (cooperative launch): pre-sweep
// tiles (and the list's zero and copy entries), the fixed point, projection.
__global__ void __launch_bounds__(FORCE_THREADS) k_force_sweep(ForceLaunch L) {
    ::silt::dep_wait();
    extern __shared__ float sm[];
    __shared__ LayerParams Ps[2];
    if (threadIdx.x < 2) Ps[threadIdx.x] = force_params(L.lay[threadIdx.x], L.sc, threadIdx.x, blockIdx.x == 0);
    __syncthreads();
    SweepState* S = L.tf.sweep;
    const unsigned int epoch = ld_acquire_u32(&S->epoch);
    const int n = *L.tf.count;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int e = L.tf.list[k];
        if (force_entry(Ps[e >> 30], L.tf, L.nxt, e, sm)) __syncthreads();
    }
    unsigned int target = 0;
    if (!grid_barrier(S, target)) return;
    const bool reuse = n <= (int)gridDim.x;  // one entry per CTA: its tile stays in shared memory
    const int passes = sweep_fixed_point(S, target, n, [&](int k, int pass) {
        const int e = L.tf.list[k];
        return sweep_entry(Ps[e >> 30], L.tf, e, sm, pass, epoch, reuse);
    });
    if (passes < 0) return;
    if (passes == 0) {
        if (threadIdx.x == 0 && blockIdx.x < 2) {
            const LayerParams& P = Ps[blockIdx.x];
            if (P.sweep && P.vort > 0.0f && !P.skip && layer_steps(L.sc, blockIdx.x)) sweep_serial(P);
        }
        if (!grid_barrier(S, target)) return;
    }
    sweep_stats(S, passes);
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int e = L.tf.list[k];
        if (post_entry(Ps[e >> 30], L.tf, e, sm)) __syncthreads();
    }
}

// Persistent over the substep's tile list.
__global__ void __launch_bounds__(FORCE_THREADS) k_force(ForceLaunch L) {
    ::silt::dep_wait();
    extern __shared__ float sm[];
    __shared__ LayerParams Ps[2];
    if (threadIdx.x < 2) Ps[threadIdx.x] = force_params(L.lay[threadIdx.x], L.sc, threadIdx.x, blockIdx.x == 0);
    __syncthreads();
    const int n = *L.tf.count;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int e = L.tf.list[k];
        if (force_entry(Ps[e >> 30], L.tf, L.nxt, e, sm)) __syncthreads();  // shared memory is reused by the next tile
    }
}

// The list entry of tile t of layer l for this substep, or -1 for none.
__device__ __forceinline__ int tile_entry(const TileFlags& tf, int cur, int nxt, int all, const SubstepCount& sc,
                                          int l, int t) {
    if (sc.speed2 && sc.k > 0) {  // substep 0 steps every layer; its list precedes the speed pass
        const int ns = device_nsub(sc, l);
        if (sc.k >= ns) {
            // Identity substep: carry every tile not known to be zero.
            if (!(pick(tf.zero_h, l, cur)[t] && pick(tf.zero_uv, l, cur)[t])) return (l << 30) | ENTRY_COPY | t;
            if (!(pick(tf.zero_h, l, nxt)[t] && pick(tf.zero_uv, l, nxt)[t])) return (l << 30) | ENTRY_ZERO | t;
            return -1;
        }
    }
    const int ti = t % tf.tiles_x, tj = t / tf.tiles_x;
    bool active = all != 0;
    for (int dj = -1; dj <= 1 && !active; ++dj)
        for (int di = -1; di <= 1; ++di) {
            const int a = ti + di, b = tj + dj;
            if (a < 0 || b < 0 || a >= tf.tiles_x || b >= tf.tiles_x) continue;
            if (pick(tf.wet, l, cur)[b * tf.tiles_x + a]) {
                active = true;
                break;
            }
        }
    if (active) {
        if (tf.stepped) atomicAdd(&tf.stepped[l], 1ull);
        return (l << 30) | t;
    }
    if (!pick(tf.zero_uv, l, nxt)[t] || !pick(tf.zero_h, l, nxt)[t]) return (l << 30) | ENTRY_ZERO | t;
    return -1;
}

__global__ void k_tile_list(TileFlags tf, int cur, int nxt, int all, int skip0, int skip1, SubstepCount sc,
                            int* count_next, double* zero_ledger, unsigned int* zero_bits) {
    ::silt::dep_wait();
    const int nt = tf.tiles_x * tf.tiles_x;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) {
        if (count_next) *count_next = 0;
        if (zero_ledger) zero_ledger[0] = zero_ledger[1] = 0.0;
        if (zero_bits) zero_bits[0] = zero_bits[1] = 0u;
        clear_sweep(tf.sweep);
    }
    if (k >= 2 * nt) return;
    const int l = k / nt, t = k % nt;
    if (l == 0 ? skip0 : skip1) return;
    const int e = tile_entry(tf, cur, nxt, all, sc, l, t);
    if (e >= 0) tf.list[atomicAdd(tf.count, 1)] = e;
}

cudaError_t launch_tile_list(const TileFlags& tf, int cur, int nxt, int all, int skip0, int skip1,
                             const SubstepCount& sc, int* count_next, double* zero_ledger, unsigned int* zero_bits,
                             cudaStream_t st) {
    if (!count_next) {
        cudaError_t e = cudaMemsetAsync(tf.count, 0, sizeof(int), st);
        if (e != cudaSuccess) return e;
    }
    const int n = 2 * tf.tiles_x * tf.tiles_x;
    ::silt::launch_dep(k_tile_list, dim3((n + 255) / 256), dim3(256), 0, st, tf, cur, nxt, all, skip0, skip1, sc, count_next, zero_ledger,
                                                 zero_bits);
    ::silt::count_launch();
    return cudaGetLastError();
}

// ------------------------------------------------- TMA staging of halo tiles

constexpr int TMA_WAIT_LIMIT = 1 << 22;  // mbarrier polls before a CTA gives up on a copy

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Waits for the barrier phase with a bounded number of polls; false if it
// never completed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done = 0;
    for (int k = 0; k < TMA_WAIT_LIMIT && !done; ++k)
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
    return done != 0;
}

// One 2D tile copy global -> this CTA's own shared memory only, counted
// on `bar`. x must be a multiple of 4 floats (16 bytes).
__device__ __forceinline__ void tma_load_2d(float* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// The mbarrier of a CTA's tile copies and the parity of its next phase.
struct TileStage {
    uint64_t* bar;
    uint32_t phase;
    bool off;  // a copy did not arrive in time: this CTA loads its tiles itself
};

// h, u and v of a transport tile, rows [ty0-2, ty0+33) x columns
// [tx0-4, tx0+36), into their shared planes: three TMA copies (h, u, v
// tensor maps of the layer) completing one phase of the stage's barrier.
// Columns past the grid's edge read 0 and are not used. False when the copies
// did not arrive within the poll limit, twice: the error word gets bit 1 and
// the caller loads the planes itself.
__device__ bool tma_stage_transport(const CUtensorMap* maps, float* HSm, float* US, float* VS, int tx0, int ty0,
                                    TileStage& ts, unsigned int* err) {
    // Every thread's earlier writes of these planes come before the copies' writes.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(ts.bar)),
                     "r"(3 * TS * TW * (int)sizeof(float))
                     : "memory");
        tma_load_2d(HSm, maps + 0, tx0 - 4, ty0 - 2, ts.bar);
        tma_load_2d(US, maps + 1, tx0 - 4, ty0 - 2, ts.bar);
        tma_load_2d(VS, maps + 2, tx0 - 4, ty0 - 2, ts.bar);
    }
    bool ok = __syncthreads_and(mbar_wait(ts.bar, ts.phase) ? 1 : 0) != 0;
    if (!ok) ok = __syncthreads_and(mbar_wait(ts.bar, ts.phase) ? 1 : 0) != 0;
    if (!ok) {
        if (threadIdx.x == 0 && err) atomicOr(err, 2u);
        ts.off = true;  // the phases are no longer known: no more copies
        return false;
    }
    ts.phase ^= 1u;
    return true;
}

// Cells [x0, x0 + W) x [y0, y0 + H) of a transport tile: edge tiles walk
// clipped rows one warp per row; interior tiles (W, H exact) one flat range
// of compile-time width, so every lane is busy on the 33-35 wide passes.
template <bool EDGE, int W, int H, class F>
__device__ __forceinline__ void trows(int x0, int x1, int y0, int y1, F f) {
    if (EDGE) {
        const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
        constexpr int NW = TRANSPORT_THREADS / 32;
        for (int gy = y0 + wy; gy < y1; gy += NW)
            for (int gx = x0 + lane; gx < x1; gx += 32) f(gx, gy);
    } else {
        for (int k = threadIdx.x; k < W * H; k += TRANSPORT_THREADS) {
            const int r = k / W;
            f(x0 + (k - r * W), y0 + r);
        }
    }
}

// Donor-cell transport (src/fluid_core.rs:3025-3137), x pass then z pass on
// the updated depth, dry cut (src/fluid_core.rs:2072-2081), FP64 ledger sum.
// An edge moves depth one way only (the sign of its face speed picks the
// donor), so each flux pass evaluates the edges whose donor it is and writes
// 0 for the others. EDGE = false: the tile is full and its cells
// [t0-2, t1+1) lie inside the grid with t1 <= res-1, so no range is clipped.
template <bool EDGE>
__device__ __forceinline__ void transport_tile(const TransportParams& P, float* sm, int tx0, int ty0,
                                               const TileFlags& tf, int l, int nxt, int t, const CUtensorMap* maps,
                                               TileStage* ts) {
    const int res = P.res;
    const int tx1 = min(res, tx0 + TT), ty1 = min(res, ty0 + TT);
    constexpr int PL = TPL;
    float* HSm = sm;            // h on rows [ty0-2, ty1+1), cols [tx0-2, tx1+1)
    float* US = sm + PL;        // u on the same cells
    float* FL = sm + 2 * PL;    // left-going flux of edge e (cells e, e+1)
    float* FR = sm + 3 * PL;    // right-going flux
    float* HX = sm + 4 * PL;    // depth after the x pass
    float* VS = sm + 5 * PL;    // v
    float* UP = sm + 6 * PL;    // up-going flux of row pair (r, r+1)
    float* DN = sm + 7 * PL;    // down-going flux
    const int ox = tx0 - 4, oy = ty0 - 2;
#define TIDX(gx, gy) (((gy) - oy) * TS + ((gx) - ox))
    const int ry0 = max(0, ty0 - 2), ry1 = min(res, ty1 + 1);
    const int cx0 = max(0, tx0 - 2), cx1 = min(res, tx1 + 1);
    const FixedDiv& cell = P.div_cell;
    const float dt = P.dt;
    const bool with_bed = P.bank_bed != nullptr;
    const uint8_t* gate = P.gate;
    // An interior tile of a layer with tensor maps arrives by TMA.
    const bool staged = !EDGE && maps && ts && !ts->off &&
                        tma_stage_transport(maps, HSm, US, VS, tx0, ty0, *ts, tf.sweep ? &tf.sweep->err : nullptr);
    if (!staged) {
        trows<EDGE, TT + 3, TT + 3>(cx0, cx1, ry0, ry1, [&](int gx, int gy) {
            size_t g = (size_t)gy * res + gx;
            HSm[TIDX(gx, gy)] = P.h[g];
            US[TIDX(gx, gy)] = P.u[g];
            if (gx >= tx0 && gx < tx1) VS[TIDX(gx, gy)] = P.v[g];
        });
        __syncthreads();
    }
    // x pass. Edge e joins cells e and e+1 and exists for 0 <= e < res-1.
    // Left-going flux first (its donor e+1 has removed nothing yet).
    const int e0 = max(0, tx0 - 2), e1 = min(res - 2, tx1 - 1);  // inclusive edge range
    trows<EDGE, TT + 2, TT + 3>(e0, e1 + 1, ry0, ry1, [&](int e, int gy) {
        float speed = 0.5f * (US[TIDX(e, gy)] + US[TIDX(e + 1, gy)]);
        float dh = 0.0f;
        if (!(speed > 0.0f)) {
            size_t g = (size_t)gy * res + e;
            float bd = with_bed ? P.bank_bed[g + 1] : 0.0f, bc = with_bed ? P.bank_bed[g] : 0.0f;
            dh = open_edge_dh(with_bed, HSm[TIDX(e + 1, gy)], HSm[TIDX(e, gy)], 0.0f, gate ? gate[g] : 1, bd, bc,
                              speed, dt, cell, 0.45f);
        }
        FL[TIDX(e, gy)] = dh;
    });
    __syncthreads();
    // Right-going: donor e has removed the left-going flux of edge e-1.
    trows<EDGE, TT + 1, TT + 3>(max(e0, tx0 - 1), e1 + 1, ry0, ry1, [&](int e, int gy) {
        float speed = 0.5f * (US[TIDX(e, gy)] + US[TIDX(e + 1, gy)]);
        float dh = 0.0f;
        if (speed > 0.0f) {
            float prev = e > 0 ? FL[TIDX(e - 1, gy)] : 0.0f;
            size_t g = (size_t)gy * res + e;
            float bd = with_bed ? P.bank_bed[g] : 0.0f, bc = with_bed ? P.bank_bed[g + 1] : 0.0f;
            dh = open_edge_dh(with_bed, HSm[TIDX(e, gy)], HSm[TIDX(e + 1, gy)], 0.0f + prev, gate ? gate[g + 1] : 1,
                              bd, bc, speed, dt, cell, 0.45f);
        }
        FR[TIDX(e, gy)] = dh;
    });
    __syncthreads();
    // Depth after the x pass on rows [ry0, ry1), tile columns. The rounding
    // book takes, for the tile's own cells, each cell's f32 change less the
    // exact (FP64) sum of the fluxes across its faces.
    double rnd = 0.0;
    const bool book_round = P.round != nullptr;
    trows<EDGE, TT, TT + 3>(tx0, tx1, ry0, ry1, [&](int c, int gy) {
        float flm = c - 1 >= 0 ? FL[TIDX(c - 1, gy)] : 0.0f;
        float frm = c - 1 >= 0 ? FR[TIDX(c - 1, gy)] : 0.0f;
        float flc = c <= res - 2 ? FL[TIDX(c, gy)] : 0.0f;
        float frc = c <= res - 2 ? FR[TIDX(c, gy)] : 0.0f;
        float rem = (0.0f + flm) + frc;
        float add = (0.0f + frm) + flc;
        float hv = HSm[TIDX(c, gy)];
        float moved = fmaxf(hv - rem + add, 0.0f);
        const float hx = (rem > 0.0f || add > 0.0f) ? moved : hv;
        HX[TIDX(c, gy)] = hx;
        if (book_round && gy >= ty0 && gy < ty1)
            rnd += ((double)hx - (double)hv) - (((double)frm + (double)flc) - ((double)flm + (double)frc));
    });
    __syncthreads();
    // z pass. Pair r joins rows r and r+1 and exists for 0 <= r < res-1.
    const int p0 = max(0, ty0 - 2), p1 = min(res - 2, ty1 - 1);
    trows<EDGE, TT, TT + 2>(tx0, tx1, p0, p1 + 1, [&](int c, int r) {
        float speed = 0.5f * (VS[TIDX(c, r)] + VS[TIDX(c, r + 1)]);
        float dh = 0.0f;
        if (!(speed > 0.0f)) {
            size_t g = (size_t)r * res + c;
            float bd = with_bed ? P.bank_bed[g + res] : 0.0f, bc = with_bed ? P.bank_bed[g] : 0.0f;
            dh = open_edge_dh(with_bed, HX[TIDX(c, r + 1)], HX[TIDX(c, r)], 0.0f, gate ? gate[g] : 1, bd, bc, speed,
                              dt, cell, 0.45f);
        }
        UP[TIDX(c, r)] = dh;
    });
    __syncthreads();
    trows<EDGE, TT, TT + 1>(tx0, tx1, max(p0, ty0 - 1), p1 + 1, [&](int c, int r) {
        float speed = 0.5f * (VS[TIDX(c, r)] + VS[TIDX(c, r + 1)]);
        float dh = 0.0f;
        if (speed > 0.0f) {
            float ra = r > 0 ? 0.0f + UP[TIDX(c, r - 1)] : 0.0f;
            size_t g = (size_t)r * res + c;
            float bd = with_bed ? P.bank_bed[g] : 0.0f, bc = with_bed ? P.bank_bed[g + res] : 0.0f;
            dh = open_edge_dh(with_bed, HX[TIDX(c, r)], HX[TIDX(c, r + 1)], ra, gate ? gate[g + res] : 1, bd, bc,
                              speed, dt, cell, 0.45f);
        }
        DN[TIDX(c, r)] = dh;
    });
    __syncthreads();
    double part = 0.0, cut = 0.0;
    trows<EDGE, TT, TT>(tx0, tx1, ty0, ty1, [&](int c, int r) {
        float upm = r - 1 >= 0 ? UP[TIDX(c, r - 1)] : 0.0f;
        float dnm = r - 1 >= 0 ? DN[TIDX(c, r - 1)] : 0.0f;
        float upc = r <= res - 2 ? UP[TIDX(c, r)] : 0.0f;
        float dnc = r <= res - 2 ? DN[TIDX(c, r)] : 0.0f;
        float rem = (0.0f + upm) + dnc;
        float add = (0.0f + dnm) + upc;
        float hv = HX[TIDX(c, r)];
        float moved = fmaxf(hv - rem + add, 0.0f);
        float hn = (rem > 0.0f || add > 0.0f) ? moved : hv;
        if (book_round)
            rnd += ((double)hn - (double)hv) - (((double)dnm + (double)upc) - ((double)upm + (double)dnc));
        if (P.eps > 0.0f && hn < P.eps) {
            if (hn > 0.0f) cut += (double)hn;  // booked: the dry cut's volume
            hn = 0.0f;
        }
        P.h_out[(size_t)r * res + c] = hn;
        part += (double)fmaxf(hn, 0.0f);
    });
    for (int o = 16; o > 0; o >>= 1) cut += __shfl_down_sync(0xffffffffu, cut, o);
    if ((threadIdx.x & 31) == 0 && cut > 0.0 && P.cut) atomicAdd(P.cut, cut * P.cut_area);
    if (book_round) {
        for (int o = 16; o > 0; o >>= 1) rnd += __shfl_down_sync(0xffffffffu, rnd, o);
        if ((threadIdx.x & 31) == 0 && rnd != 0.0) atomicAdd(P.round, rnd * P.cut_area);
    }
#undef TIDX
    // Block sum of the depth (FP64), one atomic per tile; the tile's flags.
    const int any = __syncthreads_or(part > 0.0);
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    __shared__ double warp_sum[TRANSPORT_THREADS / 32];
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? warp_sum[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) {
            if (P.ledger) atomicAdd(P.ledger, v);
            pick(tf.wet, l, nxt)[t] = any ? 1 : 0;
            pick(tf.zero_h, l, nxt)[t] = any ? 0 : 1;
        }
    }
    __syncthreads();  // shared memory is reused by the next tile
}

// Identity substep of one depth tile: copy, ledger sum and flags as
// transport_tile leaves them.
__device__ void copy_tile(const TransportParams& P, int tx0, int ty0, const TileFlags& tf, int l, int nxt, int t) {
    const int res = P.res;
    const int w = min(TT, res - tx0), h = min(TT, res - ty0);
    double part = 0.0;
    for (int q = threadIdx.x; q < w * h; q += blockDim.x) {
        const size_t g = (size_t)(ty0 + q / w) * res + tx0 + q % w;
        const float hv = P.h[g];
        P.h_out[g] = hv;
        part += (double)fmaxf(hv, 0.0f);
    }
    const int any = __syncthreads_or(part > 0.0);
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    __shared__ double warp_sum[TRANSPORT_THREADS / 32];
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? warp_sum[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) {
            if (P.ledger) atomicAdd(P.ledger, v);
            pick(tf.wet, l, nxt)[t] = any ? 1 : 0;
            pick(tf.zero_h, l, nxt)[t] = any ? 0 : 1;
        }
    }
    __syncthreads();
}

// One list entry of the transport pass.
__device__ __forceinline__ void transport_entry(const TransportParams& P, const TileFlags& tf, int nxt, int e,
                                                float* sm, const CUtensorMap* maps = nullptr,
                                                TileStage* ts = nullptr) {
    const int l = e >> 30, zero_fill = (e & ENTRY_ZERO) != 0, copy = (e & ENTRY_COPY) != 0, t = e & ENTRY_TILE;
    const int res = P.res;
    const int tx0 = (t % tf.tiles_x) * TT, ty0 = (t / tf.tiles_x) * TT;
    if (copy) {
        copy_tile(P, tx0, ty0, tf, l, nxt, t);
        return;
    }
    if (zero_fill) {
        const int w = min(TT, res - tx0), h = min(TT, res - ty0);
        for (int q = threadIdx.x; q < w * h; q += blockDim.x)
            P.h_out[(size_t)(ty0 + q / w) * res + tx0 + q % w] = 0.0f;
        if (threadIdx.x == 0) {
            pick(tf.wet, l, nxt)[t] = 0;
            pick(tf.zero_h, l, nxt)[t] = 1;
        }
        return;
    }
    const bool interior = tx0 >= 2 && ty0 >= 2 && tx0 + TT + 1 <= res && ty0 + TT + 1 <= res;
    if (interior)
        transport_tile<false>(P, sm, tx0, ty0, tf, l, nxt, t, maps, ts);
    else
        transport_tile<true>(P, sm, tx0, ty0, tf, l, nxt, t, nullptr, nullptr);
}

// Persistent over the substep's tile list.
__global__ void __launch_bounds__(TRANSPORT_THREADS) k_transport(TransportLaunch L,
                                                                   const __grid_constant__ TransportMaps M) {
    ::silt::dep_wait();
    extern __shared__ __align__(128) float sm[];
    __shared__ TransportParams Ps[2];
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x < 2) {
        const int l = threadIdx.x;
        TransportParams P = L.lay[l];
        if (L.sc.speed2) P.dt = L.sc.dt / (float)device_nsub(L.sc, l);
        Ps[l] = P;
    }
    const bool tma = (M.on[0] || M.on[1]) && (smem_addr(sm) & 127u) == 0;
    if (tma && threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&bar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    TileStage ts{&bar, 0u, !tma};
    const int n = *L.tf.count;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int e = L.tf.list[k];
        const int l = e >> 30;
        transport_entry(Ps[l], L.tf, L.nxt, e, sm, M.on[l] ? M.map[l] : nullptr, &ts);
    }
}

// Materialises the lazy dry cut: u = v = 0 where h < eps.
__global__ void k_apply_cut(const float* h, float* u, float* v, size_t n, float eps) {
    ::silt::dep_wait();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (h[i] < eps) { u[i] = 0.0f; v[i] = 0.0f; }
}

// Largest squared speed, for the CFL substep count (src/fluid_core.rs:1723-1744).
__global__ void k_max_speed2(const float* h, const float* u, const float* v, size_t n, float eps, int apply_cut,
                             unsigned int* out_bits) {
    ::silt::dep_wait();
    float m = 0.0f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float uu = u[i], vv = v[i];
        if (apply_cut && h[i] < eps) continue;
        float s2 = uu * uu + vv * vv;
        if (s2 > m) m = s2;
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_uint(m));
}

// k_max_speed2 over the stepped tiles of substep 0's list (every tile that
// may hold water is one of them; a tile without water has no cell at or above
// eps and, after the dry cut, no velocity). Each thread loads its four cells
// before comparing, so a tile costs one memory round trip.
__global__ void __launch_bounds__(256) k_tile_speed2(TileFlags tf, const float* h0, const float* u0, const float* v0,
                                                     const float* h1, const float* u1, const float* v1, int res,
                                                     float eps, int apply_cut, unsigned int* bits) {
    ::silt::dep_wait();
    const int n = *tf.count;
    const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int e = tf.list[k];
        if (e & (ENTRY_ZERO | ENTRY_COPY)) continue;
        const int l = e >> 30, t = e & ENTRY_TILE;
        const float* h = l ? h1 : h0;
        const float* u = l ? u1 : u0;
        const float* v = l ? v1 : v0;
        const int tx0 = (t % tf.tiles_x) * GRID_TILE, ty0 = (t / tf.tiles_x) * GRID_TILE;
        const int gx = tx0 + lane;
        float hv[4], uv[4], vv[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int gy = ty0 + wy + 8 * r;
            const bool in = gx < res && gy < res;
            const size_t g = in ? (size_t)gy * res + gx : 0;
            hv[r] = in ? h[g] : 0.0f;
            uv[r] = in ? u[g] : 0.0f;
            vv[r] = in ? v[g] : 0.0f;
        }
        float m = 0.0f;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (apply_cut && hv[r] < eps) continue;
            const float s2 = uv[r] * uv[r] + vv[r] * vv[r];
            if (s2 > m) m = s2;
        }
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
        if (lane == 0 && m > 0.0f) atomicMax(&bits[l], __float_as_uint(m));
    }
}

cudaError_t launch_tile_speed2(const TileFlags& tf, const float* const h[2], const float* const u[2],
                               const float* const v[2], int res, float eps, int apply_cut, unsigned int* bits,
                               cudaStream_t st) {
    ::silt::launch_dep(k_tile_speed2, dim3(148 * 8), dim3(256), 0, st, tf, h[0], u[0], v[0], h[1], u[1], v[1], res, eps, apply_cut, bits);
    ::silt::count_launch();
    return cudaGetLastError();
}

// ------------------------------------------------------------ batched windows

__global__ void k_batch_tile_list(const WindowSubstep* ws, int* list, int* entry_win, int* count, int* count_next,
                                  SweepState* sweep) {
    ::silt::dep_wait();
    const int w = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (w == 0 && k == 0) {
        *count_next = 0;
        clear_sweep(sweep);
    }
    const WindowSubstep& D = ws[w];
    if (D.skip) return;
    const TileFlags& tf = D.F.tf;
    if (k == 0) {
        if (D.zero_ledger) D.zero_ledger[0] = D.zero_ledger[1] = 0.0;
        if (D.zero_bits) D.zero_bits[0] = D.zero_bits[1] = 0u;
    }
    const int nt = tf.tiles_x * tf.tiles_x;
    if (k >= 2 * nt) return;
    const int l = k / nt, t = k % nt;
    const int e = tile_entry(tf, D.cur, D.F.nxt, D.all, D.F.sc, l, t);
    if (e >= 0) {
        const int q = atomicAdd(count, 1);
        list[q] = e;
        entry_win[q] = w;
    }
}

__global__ void __launch_bounds__(256) k_batch_speed2(const WindowSubstep* ws, const int* list, const int* entry_win,
                                                      const int* count) {
    ::silt::dep_wait();
    const int n = *count;
    const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int e = list[k];
        if (e & (ENTRY_ZERO | ENTRY_COPY)) continue;
        const WindowSubstep& D = ws[entry_win[k]];
        if (!D.zero_bits) continue;
        const int l = e >> 30, t = e & ENTRY_TILE;
        const LayerParams& P = D.F.lay[l];
        const int res = P.res, tiles_x = D.F.tf.tiles_x;
        const int tx0 = (t % tiles_x) * GRID_TILE, ty0 = (t / tiles_x) * GRID_TILE;
        const int gx = tx0 + lane;
        float hv[4], uv[4], vv[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int gy = ty0 + wy + 8 * r;
            const bool in = gx < res && gy < res;
            const size_t g = in ? (size_t)gy * res + gx : 0;
            hv[r] = in ? P.h[g] : 0.0f;
            uv[r] = in ? P.u[g] : 0.0f;
            vv[r] = in ? P.v[g] : 0.0f;
        }
        float m = 0.0f;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (D.apply_cut && hv[r] < P.eps) continue;
            const float s2 = uv[r] * uv[r] + vv[r] * vv[r];
            if (s2 > m) m = s2;
        }
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
        if (lane == 0 && m > 0.0f) atomicMax(&D.zero_bits[l], __float_as_uint(m));
    }
}

__global__ void __launch_bounds__(FORCE_THREADS) k_batch_force(const WindowSubstep* ws, const int* list,
                                                               const int* entry_win, const int* count) {
    ::silt::dep_wait();
    extern __shared__ float sm[];
    __shared__ LayerParams Ps;
    __shared__ TileFlags Tf;
    __shared__ int nxt_s;
    const int n = *count;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int e = list[k];
        if (threadIdx.x == 0) {
            const WindowSubstep& D = ws[entry_win[k]];
            Ps = force_params(D.F.lay[e >> 30], D.F.sc, e >> 30, true);
            Tf = D.F.tf;
            nxt_s = D.F.nxt;
        }
        __syncthreads();
        force_entry(Ps, Tf, nxt_s, e, sm);
        __syncthreads();  // the parameters and shared memory are reused by the next entry
    }
}

// Every window's force pass in the sweep form (cooperative launch), as
// k_force_sweep does for one sheet; windows without the sweep take the
// snapshot form in the first part and sit out the rest.
__global__ void __launch_bounds__(FORCE_THREADS) k_batch_force_sweep(const WindowSubstep* ws, int nwin, const int* list,
                                                                     const int* entry_win, const int* count,
                                                                     SweepState* S) {
    ::silt::dep_wait();
    extern __shared__ float sm[];
    __shared__ LayerParams Ps;
    __shared__ TileFlags Tf;
    __shared__ int nxt_s;
    const int n = *count;
    auto fetch = [&](int k, bool report) {
        const int e = list[k];
        if (threadIdx.x == 0) {
            const WindowSubstep& D = ws[entry_win[k]];
            Ps = force_params(D.F.lay[e >> 30], D.F.sc, e >> 30, report);
            Tf = D.F.tf;
            nxt_s = D.F.nxt;
        }
        __syncthreads();
        return e;
    };
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int e = fetch(k, true);
        force_entry(Ps, Tf, nxt_s, e, sm);
        __syncthreads();  // the parameters and shared memory are reused by the next entry
    }
    unsigned int target = 0;
    const unsigned int epoch = ld_acquire_u32(&S->epoch);
    if (!grid_barrier(S, target)) return;
    const bool reuse = n <= (int)gridDim.x;  // one entry per CTA: its tile stays in shared memory
    const int passes = sweep_fixed_point(S, target, n, [&](int k, int pass) {
        const int e = fetch(k, false);
        const bool r = sweep_entry(Ps, Tf, e, sm, pass, epoch, reuse);
        __syncthreads();
        return r;
    });
    if (passes < 0) return;
    if (passes == 0) {
        for (int u = blockIdx.x; u < 2 * nwin; u += gridDim.x) {
            if (threadIdx.x != 0) continue;
            const WindowSubstep& D = ws[u >> 1];
            const int l = u & 1;
            if (D.skip) continue;
            const LayerParams P = force_params(D.F.lay[l], D.F.sc, l, false);
            if (P.sweep && P.vort > 0.0f && !P.skip && layer_steps(D.F.sc, l)) sweep_serial(P);
        }
        if (!grid_barrier(S, target)) return;
    }
    sweep_stats(S, passes);
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int e = fetch(k, false);
        post_entry(Ps, Tf, e, sm);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(TRANSPORT_THREADS) k_batch_transport(const WindowSubstep* ws, const int* list,
                                                                       const int* entry_win, const int* count) {
    ::silt::dep_wait();
    extern __shared__ float sm[];
    __shared__ TransportParams Ps;
    __shared__ TileFlags Tf;
    __shared__ int nxt_s;
    const int n = *count;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int e = list[k];
        if (threadIdx.x == 0) {
            const WindowSubstep& D = ws[entry_win[k]];
            const int l = e >> 30;
            TransportParams P = D.T.lay[l];
            if (D.T.sc.speed2) P.dt = D.T.sc.dt / (float)device_nsub(D.T.sc, l);
            Ps = P;
            Tf = D.T.tf;
            nxt_s = D.T.nxt;
        }
        __syncthreads();
        transport_entry(Ps, Tf, nxt_s, e, sm);
        __syncthreads();
    }
}

cudaError_t launch_batch_tile_list(const WindowSubstep* d_ws, int nwin, int max_tiles, int* list, int* entry_win,
                                   int* count, int* count_next, SweepState* sweep, cudaStream_t st) {
    if (nwin <= 0) return cudaSuccess;
    dim3 grid((2 * max_tiles + 255) / 256, nwin);
    ::silt::launch_dep(k_batch_tile_list, dim3(grid), dim3(256), 0, st, d_ws, list, entry_win, count, count_next,
                       sweep);
    ::silt::count_launch();
    return cudaGetLastError();
}

cudaError_t launch_batch_speed2(const WindowSubstep* d_ws, const int* list, const int* entry_win, const int* count,
                                cudaStream_t st) {
    ::silt::launch_dep(k_batch_speed2, dim3(148 * 8), dim3(256), 0, st, d_ws, list, entry_win, count);
    ::silt::count_launch();
    return cudaGetLastError();
}

// Grid of a cooperative force launch: every CTA the device holds at once.
template <class K>
int coop_grid(K kernel, size_t smem) {
    int dev = 0, nsm = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, FORCE_THREADS, smem) != cudaSuccess) return 0;
    return nsm * per;
}

template <class K, class... Args>
cudaError_t launch_coop(K kernel, int grid, cudaStream_t st, Args... args) {
    if (grid <= 0) return cudaErrorInvalidConfiguration;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(FORCE_THREADS);
    cfg.dynamicSmemBytes = force_smem_bytes();
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = ::silt::launch_ex(cfg, kernel, args...);
    ::silt::count_launch();
    return e;
}

cudaError_t launch_batch_force(const WindowSubstep* d_ws, int nwin, const int* list, const int* entry_win,
                               const int* count, SweepState* sweep, cudaStream_t st, int ctas_per_sm) {
    if (sweep) {
        static std::once_flag sattr;
        static int grid = 0, nsm = 148;
        std::call_once(sattr, [] {
            cudaFuncSetAttribute(k_batch_force_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)force_smem_bytes());
            grid = coop_grid(k_batch_force_sweep, force_smem_bytes());
            int dev = 0;
            if (cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0)
                nsm = 148;
            cudaGetLastError();
        });
        // Fewer CTAs than the device holds stay co-resident: the launch is still cooperative.
        const int g = ctas_per_sm > 0 ? std::min(grid, ctas_per_sm * nsm) : grid;
        const cudaError_t e = launch_coop(k_batch_force_sweep, g, st, d_ws, nwin, list, entry_win, count, sweep);
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    static std::once_flag attr;
    std::call_once(attr, [] { cudaFuncSetAttribute(k_batch_force, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)force_smem_bytes()); });
    ::silt::launch_dep(k_batch_force, dim3(148 * 2), dim3(FORCE_THREADS), force_smem_bytes(), st, d_ws, list, entry_win, count);
    ::silt::count_launch();
    return cudaGetLastError();
}

cudaError_t launch_batch_transport(const WindowSubstep* d_ws, const int* list, const int* entry_win,
                                   const int* count, cudaStream_t st, int blocks) {
    static std::once_flag attr;
    std::call_once(attr, [] { cudaFuncSetAttribute(k_batch_transport, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)transport_smem_bytes()); });
    const unsigned grid = blocks > 0 ? (unsigned)blocks : 148u * 4u;
    ::silt::launch_dep(k_batch_transport, dim3(grid), dim3(TRANSPORT_THREADS), transport_smem_bytes(), st, d_ws, list, entry_win, count);
    ::silt::count_launch();
    return cudaGetLastError();
}

cudaError_t launch_force(const ForceLaunch& L, int res, int layers, cudaStream_t st) {
    if (L.lay[0].sweep || L.lay[1].sweep) {
        if (!L.tf.sweep) return cudaErrorInvalidValue;
        static std::once_flag sattr;
        static int grid = 0;
        std::call_once(sattr, [] {
            cudaFuncSetAttribute(k_force_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)force_smem_bytes());
            grid = coop_grid(k_force_sweep, force_smem_bytes());
        });
        const cudaError_t e = launch_coop(k_force_sweep, grid, st, L);
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    static std::once_flag attr;
    std::call_once(attr, [] { cudaFuncSetAttribute(k_force, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)force_smem_bytes()); });
    (void)res;
    (void)layers;
    ::silt::launch_dep(k_force, dim3(148 * 2), dim3(FORCE_THREADS), force_smem_bytes(), st, L);
    ::silt::count_launch();
    return cudaGetLastError();
}

namespace {

// cuTensorMapEncodeTiled from the driver (through the runtime: no link to libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// The transport's tensor map of a res x res FP32 plane: boxes of TS x TW
// cells, out-of-grid cells read as 0. Maps are kept per (plane, res): the
// step alternates between a few fixed buffers.
bool transport_map(const float* plane, int res, CUtensorMap* out) {
    struct Entry {
        const float* plane;
        int res;
        CUtensorMap map;
    };
    static std::mutex m;
    static std::vector<Entry> cache;
    std::lock_guard<std::mutex> lock(m);
    for (const Entry& e : cache)
        if (e.plane == plane && e.res == res) {
            *out = e.map;
            return true;
        }
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || (res % 4) != 0 || (reinterpret_cast<uintptr_t>(plane) % 16) != 0) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)res, (cuuint64_t)res};
    const cuuint64_t strides[1] = {(cuuint64_t)res * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)TS, (cuuint32_t)TW};
    const cuuint32_t elem[2] = {1, 1};
    Entry e{plane, res, {}};
    if (enc(&e.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(plane), dims, strides, box, elem,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    if (cache.size() >= 64) cache.erase(cache.begin());
    cache.push_back(e);
    *out = e.map;
    return true;
}

}  // namespace

cudaError_t launch_transport(const TransportLaunch& L, int res, int layers, cudaStream_t st) {
    static std::once_flag attr;
    std::call_once(attr, [] { cudaFuncSetAttribute(k_transport, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)transport_smem_bytes()); });
    (void)layers;
    // Interior tiles of a grid a multiple of 4 cells wide arrive by TMA.
    TransportMaps M;
    for (int l = 0; l < 2; ++l) {
        const TransportParams& P = L.lay[l];
        M.on[l] = P.res == res && P.h && P.u && P.v && transport_map(P.h, res, &M.map[l][0]) &&
                  transport_map(P.u, res, &M.map[l][1]) && transport_map(P.v, res, &M.map[l][2]);
    }
    ::silt::launch_dep(k_transport, dim3(148 * 4), dim3(TRANSPORT_THREADS), transport_smem_bytes(), st, L, M);
    ::silt::count_launch();
    return cudaGetLastError();
}

__global__ void k_material(const uint8_t* grain, const float* moisture, float* nu, float* mob, float* damp, size_t n) {
    ::silt::dep_wait();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float x = dynamic_viscosity(grain[i], moisture[i]);
        nu[i] = x;
        mob[i] = sheet_mobility_for(x);
        damp[i] = sheet_damp(x);
    }
}

cudaError_t launch_material(const uint8_t* grain, const float* moisture, float* nu, float* mob, float* damp, size_t n,
                            cudaStream_t st) {
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    ::silt::launch_dep(k_material, dim3(blocks), dim3(256), 0, st, grain, moisture, nu, mob, damp, n);
    ::silt::count_launch();
    return cudaGetLastError();
}

cudaError_t launch_apply_cut(const float* h, float* u, float* v, size_t n, float eps, cudaStream_t st) {
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    ::silt::launch_dep(k_apply_cut, dim3(blocks), dim3(256), 0, st, h, u, v, n, eps);
    ::silt::count_launch();
    return cudaGetLastError();
}

cudaError_t launch_max_speed2(const float* h, const float* u, const float* v, size_t n, float eps, int apply_cut,
                              unsigned int* out_bits, cudaStream_t st) {
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    ::silt::launch_dep(k_max_speed2, dim3(blocks), dim3(256), 0, st, h, u, v, n, eps, apply_cut, out_bits);
    ::silt::count_launch();
    return cudaGetLastError();
}

}  // namespace silt
