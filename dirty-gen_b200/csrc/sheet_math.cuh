// Device-side scalar laws of the sheet step, written to give the same f32
// results as the reference (x3-team/Dirty-gen src/fluid_core.rs). The whole
// library is compiled with -fmad=false so no multiply and add are fused,
// matching the reference's build (src/fluid_core.rs:2983-2984).
#pragma once
#include <cstdint>

#include "sheet_div.cuh"

namespace silt {

constexpr float kGravity = 9.81f;          // src/fluid_core.rs:111
constexpr float kFineCell = 0.02f;         // :73
constexpr float kSpeedCap = 1.6f;          // FILM_SPEED_CAP_MPS :10003
constexpr float kG0 = 0.06f, kG1 = 0.24f, kG2 = 0.40f;   // GAUSS :108
constexpr float kS0 = 0.02f, kS1 = 0.08f, kS2 = 0.80f;   // STEEP :109

// f32::clamp: NaN passes through.
__device__ __forceinline__ float rclamp(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
__device__ __forceinline__ bool finite_f(float x) { return isfinite(x); }

// src/fluid_core.rs:150-161
__device__ __forceinline__ float dynamic_viscosity(uint8_t grain, float moisture) {
    float x = rclamp((rclamp(moisture, 0.0f, 1.0f) - 0.22f) / 0.70f, 0.0f, 1.0f);
    float thin = x * x * (3.0f - 2.0f * x);
    float stiff, fluid;
    switch (grain) {
        case 1: stiff = 220.0f; fluid = 4.0f; break;
        case 2: stiff = 28.0f; fluid = 0.55f; break;
        case 3: stiff = 0.9f; fluid = 0.9f; break;
        case 4: stiff = 1.5f; fluid = 0.08f; break;
        default: stiff = 420.0f; fluid = 0.35f; break;
    }
    return stiff + (fluid - stiff) * thin;
}

// src/fluid_core.rs:169-180
__device__ __forceinline__ float sheet_mobility_for(float nu) {
    if (nu < 0.0f) return -nu;
    float boost = 0.0f;
    if (nu < 12.0f) {
        float t = rclamp((12.0f - fmaxf(nu, 0.0f)) / 12.0f, 0.0f, 1.0f);
        boost = t * t * 1.6f;
    }
    return 0.042f * (1.0f + boost);
}

// x^y and e^x as floats: the double-precision function rounded once to
// float. The reference calls the C library's powf and expf, which are
// correctly rounded on all but a few inputs in 10^4 over the ranges the
// sheet uses (an exhaustive comparison with the rounded double results:
// expf on [-100, 0] differs on 0.009% of floats, powf(r, 0.3) on [0.002, 12]
// on 0.06%); CUDA's single-precision powf and expf differ far more often.
__device__ __forceinline__ float pow_rn(float x, float y) { return (float)pow((double)x, (double)y); }
__device__ __forceinline__ float exp_rn(float x) { return (float)exp((double)x); }
// hypot(x, y) as the C library's hypotf gives it (the double-precision root
// of the exact double sum of squares, rounded once): identical to glibc's
// on 2e8 random pairs.
__device__ __forceinline__ float hypot_rn(float x, float y) {
    const double dx = (double)x, dy = (double)y;
    return (float)sqrt(dx * dx + dy * dy);
}

// src/fluid_core.rs:184-192
__device__ __forceinline__ float sheet_damp(float nu) {
    float rel = rclamp(fmaxf(nu, 0.05f) / 231.0f, 0.002f, 12.0f);
    if (rel >= 0.42f) return 1.70f * pow_rn(rel, 0.30f);
    const float at_silt = 1.70f * pow_rn(0.42f, 0.30f);
    float t = rclamp(rel / 0.42f, 0.0f, 1.0f);
    return at_silt * pow_rn(t, 1.15f);
}

// src/fluid_core.rs:3473-3479
__device__ __forceinline__ float finite_speed(float v, float lim) {
    return finite_f(v) ? rclamp(v, -lim, lim) : 0.0f;
}
__device__ __forceinline__ float finite0(float v) { return finite_f(v) ? v : 0.0f; }

__device__ __forceinline__ float divide_by(float x, float d) { return x / d; }
__device__ __forceinline__ float divide_by(float x, const FixedDiv& d) { return fdiv(x, d); }

// src/fluid_core.rs:2867-2911 open_edge_dh: depth one donor gives across one
// edge, 0 where the serial loop would skip the edge. `cell` is a float or a
// FixedDiv of the cell width.
template <class Cell>
__device__ __forceinline__ float open_edge_dh(bool with_bed, float hd, float hr, float remd, uint8_t gate_r,
                                              float bed_d, float bed_r, float speed, float dt, const Cell& cell,
                                              float frac_cap) {
    bool live = !(fabsf(speed) < 1.0e-5f);
    bool bank = with_bed && hr <= 1.0e-6f && bed_r > bed_d + hd + 1.0e-3f;
    float room = hd - remd;
    bool gate_shut = gate_r == 0 && hr <= 1.0e-6f;
    float frac = fminf(divide_by(fabsf(speed) * dt, cell), frac_cap);
    float dh = fminf(hd * frac, room);
    bool ok = live & !bank & !(room <= 1.0e-8f) & !gate_shut & !(dh <= 1.0e-8f);
    return ok ? dh : 0.0f;
}

// The confinement kick at (i, j) from the velocities `uu`, `vv` return for
// any cell (src/fluid_core.rs:3442-3471 with clamped indices; the interior
// form :2805-2831 gives the same values).
template <class UF, class VF>
__device__ __forceinline__ bool conf_kick(int i, int j, int res, const FixedDiv& two, float dt, float vort, UF uu, VF vv,
                                          float& du, float& dv) {
    auto vort_at = [&](int a, int c) {
        const int ip = min(a + 1, res - 1), im = max(a - 1, 0), jp = min(c + 1, res - 1), jm = max(c - 1, 0);
        float dvdx = fdiv(vv(ip, c) - vv(im, c), two);
        float dudz = fdiv(uu(a, jp) - uu(a, jm), two);
        return dvdx - dudz;
    };
    float w = vort_at(i, j);
    if (!finite_f(w) || fabsf(w) < 1.0e-4f) return false;
    float wxp = fabsf(vort_at(min(i + 1, res - 1), j));
    float wxm = fabsf(vort_at(max(i - 1, 0), j));
    float wzp = fabsf(vort_at(i, min(j + 1, res - 1)));
    float wzm = fabsf(vort_at(i, max(j - 1, 0)));
    float nx = fdiv(wxp - wxm, two);
    float nz = fdiv(wzp - wzm, two);
    du = vort * dt * (-nz * w);
    dv = vort * dt * (nx * w);
    return finite_f(du) && finite_f(dv) && du * du + dv * dv <= 0.0625f;
}

// What one cell of the Gauss-Seidel sweep reads at offset (DX, DY) from it
// (force_gravity_open's raster order, src/fluid_core.rs:2234-2260): its own
// post-gravity value at (0, 0), the current iterate of a cell before it, the
// starting value of a cell after it. The offsets are compile-time constants,
// so each read is one load at a fixed distance from the cell.
struct SweepRead {
    const float* cur;    // current iterate
    const float* start;  // starting values
    const float* own;    // post-gravity values
    int s;               // the cell's index
    int stride;          // the row stride
    template <int DX, int DY>
    __device__ __forceinline__ float at() const {
        if constexpr (DX == 0 && DY == 0)
            return own[s];
        else if constexpr (DY < 0 || (DY == 0 && DX < 0))
            return cur[s + DY * stride + DX];
        else
            return start[s + DY * stride + DX];
    }
};

// conf_kick at a cell at least two cells inside the grid, where no stencil
// index is clamped: the same arithmetic in the same order, reading the nine
// neighbours through SweepRead's fixed offsets.
__device__ __forceinline__ bool conf_kick_inner(const FixedDiv& two, float dt, float vort, const SweepRead& uu,
                                                const SweepRead& vv, float& du, float& dv) {
    auto vort_of = [&](float vp, float vm, float up, float um) {
        float dvdx = fdiv(vp - vm, two);
        float dudz = fdiv(up - um, two);
        return dvdx - dudz;
    };
    float w = vort_of(vv.at<1, 0>(), vv.at<-1, 0>(), uu.at<0, 1>(), uu.at<0, -1>());
    if (!finite_f(w) || fabsf(w) < 1.0e-4f) return false;
    float wxp = fabsf(vort_of(vv.at<2, 0>(), vv.at<0, 0>(), uu.at<1, 1>(), uu.at<1, -1>()));
    float wxm = fabsf(vort_of(vv.at<0, 0>(), vv.at<-2, 0>(), uu.at<-1, 1>(), uu.at<-1, -1>()));
    float wzp = fabsf(vort_of(vv.at<1, 1>(), vv.at<-1, 1>(), uu.at<0, 2>(), uu.at<0, 0>()));
    float wzm = fabsf(vort_of(vv.at<1, -1>(), vv.at<-1, -1>(), uu.at<0, 0>(), uu.at<0, -2>()));
    float nx = fdiv(wxp - wxm, two);
    float nz = fdiv(wzp - wzm, two);
    du = vort * dt * (-nz * w);
    dv = vort * dt * (nx * w);
    return finite_f(du) && finite_f(dv) && du * du + dv * dv <= 0.0625f;
}

}  // namespace silt
