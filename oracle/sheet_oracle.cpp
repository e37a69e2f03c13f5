// TEST INFRASTRUCTURE ONLY: CPU restatement of the reference sheet step used
// as the parity checker and the timed CPU baseline. Every function cites the
// reference file:line it restates (paths inside x3-team/Dirty-gen). The
// product never links this file.
//
// Build: g++ -O2 -ffp-contract=off -fno-fast-math (see oracle/Makefile).
//
// With -DORACLE_F64 the same source builds the FP64 restatement (the nested-
// sheet oracle the learned closure is judged against): every float of the
// step, the interface included, becomes a double and each single-precision
// libm call its double form. The model's constants keep their float values
// (the `f` literals), so only the arithmetic's precision changes.
//
// With -DORACLE_ELEM_RN it builds the step with the device's elementary
// functions (below), which attributes a book difference to them.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <thread>
#include <tuple>
#include <utility>
#include <vector>

#ifdef ORACLE_F64
#define float double
#define expf exp
#define powf pow
#define sqrtf sqrt
#define hypotf hypot
#define floorf floor
#define ceilf ceil
#define fabsf fabs
#define fminf fmin
#define fmaxf fmax
#define acosf acos
#define cosf cos
#define sinf sin
#define finite oracle_finite  // glibc declares finite(double)
#endif

#ifdef ORACLE_ELEM_RN
// The same step with e^x, x^y and hypot taken as the double-precision result
// rounded once to float, as the device computes them: the C library's expf,
// powf and hypotf differ from that on a few inputs in 10^4. Used only to
// attribute an FP64 book difference to those functions; the parity oracle is
// the default build.
static inline float oracle_exp_rn(float x) { return (float)std::exp((double)x); }
static inline float oracle_pow_rn(float x, float y) { return (float)std::pow((double)x, (double)y); }
static inline float oracle_hypot_rn(float x, float y) {
    const double dx = (double)x, dy = (double)y;
    return (float)std::sqrt(dx * dx + dy * dy);
}
#define expf oracle_exp_rn
#define powf oracle_pow_rn
#define hypotf oracle_hypot_rn
#endif

#include "sheet_oracle.h"

namespace {

typedef uint8_t u8;
typedef size_t usize;

// ---------------------------------------------------------------- constants
// src/fluid_core.rs:69-124
const float GAUSS[5] = {0.06f, 0.24f, 0.40f, 0.24f, 0.06f};
const float STEEP[5] = {0.02f, 0.08f, 0.80f, 0.08f, 0.02f};
const float GRAVITY = 9.81f;
const float FINE_CELL_M = 0.02f;
const usize FINE_RES = 160;
const usize SERIAL_SHEET_MAX = 96;          // :2480
const float FILM_SPEED_CAP_MPS = 1.6f;      // :10003
const usize BOX_PAR_GAP = 6;                // :1870
const usize SLEEP_TILE = 8;                 // :1528
const float SLEEP_SPEED = 0.05f;            // :1531
const float SLEEP_SLOPE = 0.02f;            // :1533
const usize NU_FILL_MARGIN = 8;             // :791
const float NEAR_RESIDUAL_LIFE_S = 1.5f;    // near.rs:37
const float NEAR_DROP_M = 1.0e-5f;          // near.rs:39
const float NEAR_FILM_M = 1.0e-6f;          // near.rs:41
const float FOAM_LIFE_S = 1.8f;             // :112
const float FOAM_EQ = 0.85f;                // :115
const float FOAM_TAU_S = 0.35f;             // :117
const float SILT_SETTLE_S = 4.0f;           // :119
const float SUSP_FALL_M_S = 0.004f;         // :122
const float SILT_COLUMN_CAP_M = 0.028f;     // :124

// ------------------------------------------------- Rust f32 helper semantics
inline float rmax(float a, float b) { return fmaxf(a, b); }   // f32::max (NaN-ignoring)
inline float rmin(float a, float b) { return fminf(a, b); }   // f32::min
inline float rclamp(float x, float lo, float hi) {           // f32::clamp (NaN stays)
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
inline bool finite(float x) { return std::isfinite(x); }
inline float rsignum(float x) {  // f32::signum: +1 for +0.0, -1 for -0.0
    if (std::isnan(x)) return x;
    return std::signbit(x) ? -1.0f : 1.0f;
}
inline usize sat_sub(usize a, usize b) { return a > b ? a - b : 0; }
inline usize f2usize(float x) {  // `as usize`, saturating, NaN -> 0
    if (!(x > 0.0f)) return 0;
    if (x >= 1.8e19f) return (usize)-1;
    return (usize)x;
}
// The bit pattern of a value (memo keys compare values bit for bit).
inline uint64_t fbits(float x) {
    uint64_t b = 0;
    memcpy(&b, &x, sizeof x);
    return b;
}
// Iterator::sum for f32 folds from -0.0 in the reference toolchain.
inline float rsum(const float* p, usize n) {
    float s = -0.0f;
    for (usize k = 0; k < n; ++k) s += p[k];
    return s;
}

struct Box {
    usize i0, i1, j0, j1;
    bool operator==(const Box& o) const {
        return i0 == o.i0 && i1 == o.i1 && j0 == o.j0 && j1 == o.j1;
    }
};

// -------------------------------------------------------------- material laws
// src/fluid_core.rs:150-161
float dynamic_viscosity(u8 grain, float moisture) {
    float x = rclamp((rclamp(moisture, 0.0f, 1.0f) - 0.22f) / 0.70f, 0.0f, 1.0f);
    float thin = x * x * (3.0f - 2.0f * x);
    float stiff, fluid;
    switch (grain) {
        case 1: stiff = 220.0f; fluid = 4.0f; break;     // Silt
        case 2: stiff = 28.0f; fluid = 0.55f; break;     // Sand
        case 3: stiff = 0.9f; fluid = 0.9f; break;       // Water
        case 4: stiff = 1.5f; fluid = 0.08f; break;      // Other
        default: stiff = 420.0f; fluid = 0.35f; break;   // Clay (0 and unknown)
    }
    return stiff + (fluid - stiff) * thin;
}

// src/fluid_core.rs:169-180
float sheet_mobility_for(float nu) {
    if (nu < 0.0f) return -nu;
    float boost;
    if (nu < 12.0f) {
        float t = rclamp((12.0f - rmax(nu, 0.0f)) / 12.0f, 0.0f, 1.0f);
        boost = t * t * 1.6f;
    } else {
        boost = 0.0f;
    }
    return 0.042f * (1.0f + boost);
}

// src/fluid_core.rs:184-192
float sheet_damp(float nu) {
    float rel = rclamp(rmax(nu, 0.05f) / 231.0f, 0.002f, 12.0f);
    if (rel >= 0.42f) return 1.70f * powf(rel, 0.30f);
    float at_silt = 1.70f * powf(0.42f, 0.30f);
    float t = rclamp(rel / 0.42f, 0.0f, 1.0f);
    return at_silt * powf(t, 1.15f);
}

// src/fluid_core.rs:3473-3479
float finite_speed(float v, float lim) { return finite(v) ? rclamp(v, -lim, lim) : 0.0f; }
float finite0(float v) { return finite(v) ? v : 0.0f; }

// ------------------------------------------------------- tracer helpers
// src/fluid_core.rs:9688-9691
float smoothstep(float e0, float e1, float x) {
    float t = rclamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
// src/fluid_core.rs:9676-9686
float breaking_foam(float speed, float thickness) {
    if (!finite(speed) || !finite(thickness) || thickness < 0.004f || speed <= 0.05f) return 0.0f;
    float froude = speed / sqrtf(9.81f * thickness);
    return smoothstep(0.85f, 1.45f, froude);
}
// src/fluid_core.rs:9693-9712
float sample_foam(const float* src, usize res, float x, float z) {
    if (!finite(x) || !finite(z) || x < 0.0f || z < 0.0f) return 0.0f;
    usize i0 = f2usize(floorf(x)), j0 = f2usize(floorf(z));
    if (i0 >= res || j0 >= res) return 0.0f;
    usize i1 = std::min(i0 + 1, res - 1), j1 = std::min(j0 + 1, res - 1);
    float tx = rclamp(x - (float)i0, 0.0f, 1.0f), tz = rclamp(z - (float)j0, 0.0f, 1.0f);
    float a = src[j0 * res + i0], b = src[j0 * res + i1], c = src[j1 * res + i0], d = src[j1 * res + i1];
    float v = a + (b - a) * tx + (c - a) * tz + (a - b - c + d) * tx * tz;
    return finite(v) ? rclamp(v, 0.0f, 1.0f) : 0.0f;
}
// src/fluid_core.rs:9857-9876 flux_edge
void flux_edge(const float* h, float* scratch, usize n, usize a, usize b, float vel, float cell, float dt) {
    if (!finite(vel) || fabsf(vel) < 1.0e-5f) return;
    usize donor = vel > 0.0f ? a : b, recv = vel > 0.0f ? b : a;
    float column = finite(h[donor]) ? h[donor] : 0.0f;
    float room = column - scratch[donor];
    if (room <= 1.0e-8f) return;
    float frac = rmin(fabsf(vel) * dt / cell, 0.45f);
    float dh = rmin(column * frac, room);
    if (dh <= 1.0e-8f || !finite(dh)) return;
    scratch[donor] += dh;
    scratch[n + recv] += dh;
}
// src/fluid_core.rs:9716-9748 flux_thickness
void flux_thickness(const float* h, const float* u, const float* v, usize res, float cell, float dt, usize i0,
                    usize i1, usize j0, usize j1, float* scratch) {
    usize n = res * res;
    for (usize j = j0; j <= j1; ++j) {
        usize row = j * res;
        for (usize i = i0; i < std::min(i1, res - 1); ++i) {
            usize a = row + i, b = a + 1;
            float vel = 0.5f * (u[a] + u[b]);
            flux_edge(h, scratch, n, a, b, vel, cell, dt);
        }
    }
    for (usize j = j0; j < std::min(j1, res - 1); ++j)
        for (usize i = i0; i <= i1; ++i) {
            usize a = j * res + i, b = a + res;
            float vel = 0.5f * (v[a] + v[b]);
            flux_edge(h, scratch, n, a, b, vel, cell, dt);
        }
}
// src/fluid_core.rs:9752-9764
bool shore_wet_cell(const float* water, usize res, usize i, usize j) {
    if (i == 0 || j == 0 || i + 1 >= res || j + 1 >= res) return false;
    const int d[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
    for (auto& o : d) {
        float nh = water[(usize)((int)j + o[1]) * res + (usize)((int)i + o[0])];
        if (finite(nh) && nh < 0.004f) return true;
    }
    return false;
}
// src/fluid_core.rs:9766-9795 (inclusive box of cells above 1e-8, grown by one)
bool turbid_span(const float* h, usize res, usize& i0, usize& i1, usize& j0, usize& j1) {
    i0 = res; i1 = 0; j0 = res; j1 = 0;
    for (usize j = 0; j < res; ++j) {
        const float* row = h + j * res;
        float m = 0.0f;
        for (usize i = 0; i < res; ++i) m = rmax(m, row[i]);
        if (m <= 1.0e-8f) continue;
        usize first = 0, last = 0;
        for (usize i = 0; i < res; ++i) if (row[i] > 1.0e-8f) { first = i; break; }
        for (usize i = res; i-- > 0;) if (row[i] > 1.0e-8f) { last = i; break; }
        i0 = std::min(i0, first); i1 = std::max(i1, last); j0 = std::min(j0, j); j1 = std::max(j1, j);
    }
    if (i0 > i1) return false;
    i0 = sat_sub(i0, 1); i1 = std::min(i1 + 1, res - 1); j0 = sat_sub(j0, 1); j1 = std::min(j1 + 1, res - 1);
    return true;
}
// src/fluid_core.rs:9826-9872 shore_cell: (foam production, silt lift rate)
void shore_cell(const float* water, const float* uw, const float* vw, usize res, usize idx, float& foam,
                float& rate) {
    foam = 0.0f; rate = 0.0f;
    usize i = idx % res, j = idx / res;
    if (i == 0 || j == 0 || i + 1 >= res || j + 1 >= res) return;
    float h = water[idx];
    if (!finite(h) || h < 0.004f) return;
    float nx = 0.0f, nz = 0.0f;
    bool edge = false;
    const int d[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
    for (auto& o : d) {
        float nh = water[(usize)((int)j + o[1]) * res + (usize)((int)i + o[0])];
        if (finite(nh) && nh < 0.004f) { edge = true; nx += (float)o[0]; nz += (float)o[1]; }
    }
    if (!edge) return;
    float u = uw[idx], v = vw[idx];
    if (!finite(u) || !finite(v)) return;
    float film = hypotf(u, v);
    float nlen = rmax(hypotf(nx, nz), 1.0e-4f);
    float into = rmax((u * nx + v * nz) / nlen, 0.0f);
    float strain = fabsf(uw[idx + 1] - uw[idx - 1]) + fabsf(vw[idx + res] - vw[idx - res]);
    float shear_v = rmax(film, strain);
    if (shear_v < 0.2f && into < 0.2f) return;
    float prod = rmax(breaking_foam(rmax(shear_v, into), h), smoothstep(0.25f, 1.1f, into));
    foam = prod > 0.02f ? prod : 0.0f;
    if (h > 0.012f && h < 0.055f && (shear_v > 0.45f || into > 0.4f)) {
        float tau = 1000.0f * 0.025f * shear_v * shear_v;
        if (tau > 3.0f || into > 0.45f) rate = rmin(0.006f * (into + shear_v * 0.35f), 0.01f);
    }
}

// ------------------------------------------------------------------- scratch
// src/fluid_core.rs:536-579
struct Scratch {
    usize n = 0;
    std::vector<float> a, b, c, d, e, removed, added, flux_l, flux_r;
    void fit(usize n_) {
        if (n == n_) return;
        n = n_;
        a.resize(n, 0.0f); b.resize(n, 0.0f); c.resize(n, 0.0f); d.resize(n, 0.0f);
        e.resize(n, 0.0f); removed.resize(n, 0.0f); added.resize(n, 0.0f);
    }
};

// ------------------------------------------------------------------ stencils
// src/fluid_core.rs:3498-3540
float vorticity_at(const float* u, const float* v, usize res, usize i, usize j, float cell) {
    usize ip = std::min(i + 1, res - 1), im = sat_sub(i, 1);
    usize jp = std::min(j + 1, res - 1), jm = sat_sub(j, 1);
    float dvdx = (v[j * res + ip] - v[j * res + im]) / (2.0f * cell);
    float dudz = (u[jp * res + i] - u[jm * res + i]) / (2.0f * cell);
    return dvdx - dudz;
}
void grad(const float* p, usize res, usize i, usize j, float cell, float& dx, float& dz) {
    usize ip = std::min(i + 1, res - 1), im = sat_sub(i, 1);
    usize jp = std::min(j + 1, res - 1), jm = sat_sub(j, 1);
    dx = (p[j * res + ip] - p[j * res + im]) / (2.0f * cell);
    dz = (p[jp * res + i] - p[jm * res + i]) / (2.0f * cell);
}
void grad_vel(const float* u, const float* v, usize res, usize i, usize j, float cell,
              float& dux, float& dvz) {
    usize ip = std::min(i + 1, res - 1), im = sat_sub(i, 1);
    usize jp = std::min(j + 1, res - 1), jm = sat_sub(j, 1);
    dux = (u[j * res + ip] - u[j * res + im]) / (2.0f * cell);
    dvz = (v[jp * res + i] - v[jm * res + i]) / (2.0f * cell);
}
float lap(const float* p, usize res, usize i, usize j, float cell) {
    usize idx = j * res + i;
    usize ip = std::min(i + 1, res - 1), im = sat_sub(i, 1);
    usize jp = std::min(j + 1, res - 1), jm = sat_sub(j, 1);
    float s = p[j * res + ip] + p[j * res + im] + p[jp * res + i] + p[jm * res + i] - 4.0f * p[idx];
    return s / (cell * cell);
}
// src/fluid_core.rs:2833-2838
inline float vort_interior(const float* u, const float* v, usize res, usize i, usize j, float two) {
    float dvdx = (v[j * res + i + 1] - v[j * res + i - 1]) / two;
    float dudz = (u[(j + 1) * res + i] - u[(j - 1) * res + i]) / two;
    return dvdx - dudz;
}

// Confinement kick shared by the four variants: src/fluid_core.rs:3442-3471,
// :2805-2831, :2348-2375, :2446-2470. `su,sv` are read, `u,v` written.
void confine_one(const float* su, const float* sv, float* u, float* v, usize res, usize i,
                 usize j, float cell, float dt, float eps) {
    float w = vorticity_at(su, sv, res, i, j, cell);
    if (!finite(w) || fabsf(w) < 1.0e-4f) return;
    float wxp = fabsf(vorticity_at(su, sv, res, std::min(i + 1, res - 1), j, cell));
    float wxm = fabsf(vorticity_at(su, sv, res, sat_sub(i, 1), j, cell));
    float wzp = fabsf(vorticity_at(su, sv, res, i, std::min(j + 1, res - 1), cell));
    float wzm = fabsf(vorticity_at(su, sv, res, i, sat_sub(j, 1), cell));
    float nx = (wxp - wxm) / (2.0f * cell);
    float nz = (wzp - wzm) / (2.0f * cell);
    float du = eps * dt * (-nz * w);
    float dv = eps * dt * (nx * w);
    if (finite(du) && finite(dv) && du * du + dv * dv <= 0.0625f) {
        usize idx = j * res + i;
        u[idx] += du;
        v[idx] += dv;
    }
}
void confine_interior(const float* su, const float* sv, float* u, float* v, usize res, usize i,
                      usize j, float dt, float eps, float two) {
    float w = vort_interior(su, sv, res, i, j, two);
    if (!finite(w) || fabsf(w) < 1.0e-4f) return;
    float wxp = fabsf(vort_interior(su, sv, res, i + 1, j, two));
    float wxm = fabsf(vort_interior(su, sv, res, i - 1, j, two));
    float wzp = fabsf(vort_interior(su, sv, res, i, j + 1, two));
    float wzm = fabsf(vort_interior(su, sv, res, i, j - 1, two));
    float nx = (wxp - wxm) / two;
    float nz = (wzp - wzm) / two;
    float du = eps * dt * (-nz * w);
    float dv = eps * dt * (nx * w);
    if (finite(du) && finite(dv) && du * du + dv * dv <= 0.0625f) {
        usize idx = j * res + i;
        u[idx] += du;
        v[idx] += dv;
    }
}

// ---------------------------------------------------------------------- blur
// src/fluid_core.rs:3680-3758 (accum5, accum5_clamped, blur_axis_x/z)
inline float accum5(float a0, float a1, float a2, float a3, float a4, const float* k) {
    float a = a0 * k[0];
    a += a1 * k[1];
    a += a2 * k[2];
    a += a3 * k[3];
    a += a4 * k[4];
    return a;
}
inline float accum5_clamped(const float* row, usize r, usize i, const float* k) {
    float a = 0.0f;
    for (int t = -2; t <= 2; ++t) {
        long ii = (long)i + t;
        if (ii < 0) ii = 0;
        if (ii > (long)r - 1) ii = (long)r - 1;
        a += row[ii] * k[t + 2];
    }
    return a;
}
void blur_axis_x(const float* src, float* tmp, usize res, usize j, usize i0, usize i1, const float* k) {
    const float* row = src + j * res;
    float* dst = tmp + j * res;
    usize lo = std::max(i0, (usize)2);
    usize hi = std::min(i1, sat_sub(res, 3));
    for (usize i = i0; i < std::min(lo, i1 + 1); ++i) dst[i] = accum5_clamped(row, res, i, k);
    if (lo <= hi)
        for (usize i = lo; i <= hi; ++i)
            dst[i] = accum5(row[i - 2], row[i - 1], row[i], row[i + 1], row[i + 2], k);
    usize tail = std::max(hi + 1, lo);
    for (usize i = tail; i <= i1; ++i) dst[i] = accum5_clamped(row, res, i, k);
}
void blur_axis_z(const float* src, float* dst, usize res, usize j, usize i0, usize i1, const float* k) {
    if (j >= 2 && j <= sat_sub(res, 3)) {
        const float* r0 = src + (j - 2) * res;
        const float* r1 = src + (j - 1) * res;
        const float* r2 = src + j * res;
        const float* r3 = src + (j + 1) * res;
        const float* r4 = src + (j + 2) * res;
        for (usize i = i0; i <= i1; ++i) dst[j * res + i] = accum5(r0[i], r1[i], r2[i], r3[i], r4[i], k);
    } else {
        for (usize i = i0; i <= i1; ++i) {
            float a = 0.0f;
            for (int t = -2; t <= 2; ++t) {
                long jj = (long)j + t;
                if (jj < 0) jj = 0;
                if (jj > (long)res - 1) jj = (long)res - 1;
                a += src[jj * res + i] * k[t + 2];
            }
            dst[j * res + i] = a;
        }
    }
}
// src/fluid_core.rs:3541-3569
void blur_box(const float* src, float* dst, float* tmp, usize res, usize i0, usize i1, usize j0,
              usize j1, const float* k) {
    if (i0 > i1 || j0 > j1 || res == 0) return;
    for (usize j = j0; j <= j1; ++j) blur_axis_x(src, tmp, res, j, i0, i1, k);
    for (usize j = j0; j <= j1; ++j) blur_axis_z(tmp, dst, res, j, i0, i1, k);
}

// ------------------------------------------------------------ gravity + confine
// Snapshot-Jacobi confinement: force_gravity_par (src/fluid_core.rs:2263-2378) and
// gravity_jacobi_serial/jacobi_confine_box (:2530-2595, :2415-2473) give the same
// values: every cell reads the post-gravity snapshot.
void jacobi_confine(const float* h, float* u, float* v, usize res, float cell, float dt,
                    float vorticity, float eps, usize i0, usize i1, usize j0, usize j1) {
    usize n = res * res;
    std::vector<float> su(u, u + n), sv(v, v + n);
    float two = 2.0f * cell;
    for (usize j = j0; j <= j1; ++j)
        for (usize i = i0; i <= i1; ++i) {
            usize idx = j * res + i;
            if (h[idx] <= eps) continue;
            if (i >= 2 && j >= 2 && i + 2 < res && j + 2 < res)
                confine_interior(su.data(), sv.data(), u, v, res, i, j, dt, vorticity, two);
            else
                confine_one(su.data(), sv.data(), u, v, res, i, j, cell, dt, vorticity);
        }
}

// src/fluid_core.rs:2204-2261 (serial sweep) with its two Jacobi branches.
void force_gravity_open(const float* h, float* u, float* v, const float* nu, const float* p,
                        usize res, float cell, float dt, float vorticity, float eps, usize i0,
                        usize i1, usize j0, usize j1, bool inner_par) {
    float two = 2.0f * cell;
    bool fine = cell <= FINE_CELL_M + 1.0e-6f;
    bool par = (j1 - j0 >= 47) && (i1 - i0 >= 31) && inner_par;
    bool jacobi = fine || par;
    for (usize j = j0; j <= j1; ++j)
        for (usize i = i0; i <= i1; ++i) {
            usize idx = j * res + i;
            if (h[idx] <= eps) continue;
            float px, pz;
            if (i >= 2 && j >= 2 && i + 2 < res && j + 2 < res) {
                px = (p[idx + 1] - p[idx - 1]) / two;
                pz = (p[idx + res] - p[idx - res]) / two;
            } else {
                grad(p, res, i, j, cell, px, pz);
            }
            float mob = sheet_mobility_for(nu[idx]);
            u[idx] += -GRAVITY * px * mob * dt;
            v[idx] += -GRAVITY * pz * mob * dt;
            if (!jacobi && vorticity > 0.0f) {
                if (i >= 2 && j >= 2 && i + 2 < res && j + 2 < res)
                    confine_interior(u, v, u, v, res, i, j, dt, vorticity, two);
                else
                    confine_one(u, v, u, v, res, i, j, cell, dt, vorticity);
            }
        }
    if (jacobi && vorticity > 0.0f) jacobi_confine(h, u, v, res, cell, dt, vorticity, eps, i0, i1, j0, j1);
}

// ------------------------------------------------------------------ transport
// src/fluid_core.rs:2867-2911 open_edge_dh
inline float open_edge_dh(bool BED, float hd, float hr, float remd, u8 gate_r, float bed_d,
                          float bed_r, float speed, float dt, float cell, float frac_cap) {
    bool live = !(fabsf(speed) < 1.0e-5f);
    bool bank = BED && hr <= 1.0e-6f && bed_r > bed_d + hd + 1.0e-3f;
    float room = hd - remd;
    bool gate_shut = gate_r == 0 && hr <= 1.0e-6f;
    float frac = rmin(fabsf(speed) * dt / cell, frac_cap);
    float dh = rmin(hd * frac, room);
    bool ok = live & !bank & !(room <= 1.0e-8f) & !gate_shut & !(dh <= 1.0e-8f);
    return ok ? dh : 0.0f;
}

// src/fluid_core.rs:3025-3137 transport_open_rows_body
void transport_open_rows(bool BED, float* h, const float* vel, const u8* gate, usize res, float cell,
                         float dt, usize i0, usize i1, usize j0, usize j1, bool along_x,
                         const float* bed, float frac_cap, Scratch& sc) {
    usize m = i1 + 1 - i0;
    if (along_x) {
        if (sc.flux_l.size() < m) {
            sc.flux_l.resize(m, 0.0f);
            sc.flux_r.resize(m, 0.0f);
        }
        for (usize j = j0; j <= j1; ++j) {
            usize lo = j * res + i0;
            float* hr = h + lo;
            const float* vr = vel + lo;
            const u8* gr = gate + lo;
            const float* br = BED ? bed + lo : nullptr;
            float* fl = sc.flux_l.data();
            float* fr = sc.flux_r.data();
            usize edges = m - 1;
            for (usize k = 0; k < edges; ++k) {
                float speed = 0.5f * (vr[k] + vr[k + 1]);
                float bd = BED ? br[k + 1] : 0.0f, bc = BED ? br[k] : 0.0f;
                float dh = open_edge_dh(BED, hr[k + 1], hr[k], 0.0f, gr[k], bd, bc, speed, dt, cell, frac_cap);
                fl[k] = speed > 0.0f ? 0.0f : dh;
            }
            for (usize k = 0; k < edges; ++k) {
                float speed = 0.5f * (vr[k] + vr[k + 1]);
                float prev = k > 0 ? fl[k - 1] : 0.0f;
                float bd = BED ? br[k] : 0.0f, bc = BED ? br[k + 1] : 0.0f;
                float dh = open_edge_dh(BED, hr[k], hr[k + 1], 0.0f + prev, gr[k + 1], bd, bc, speed, dt, cell, frac_cap);
                fr[k] = speed > 0.0f ? dh : 0.0f;
            }
            fl[edges] = 0.0f;
            fr[edges] = 0.0f;
            float* rem = sc.removed.data() + lo;
            float* add = sc.added.data() + lo;
            rem[0] = (0.0f + 0.0f) + fr[0];
            add[0] = (0.0f + 0.0f) + fl[0];
            for (usize c = 1; c < m; ++c) {
                rem[c] = (0.0f + fl[c - 1]) + fr[c];
                add[c] = (0.0f + fr[c - 1]) + fl[c];
            }
            for (usize c = 0; c < m; ++c) {
                float moved = rmax(hr[c] - rem[c] + add[c], 0.0f);
                hr[c] = (rem[c] > 0.0f || add[c] > 0.0f) ? moved : hr[c];
            }
        }
        return;
    }
    for (usize j = j0; j <= j1; ++j) {
        usize lo = j * res + i0;
        std::fill(sc.removed.begin() + lo, sc.removed.begin() + lo + m, 0.0f);
        std::fill(sc.added.begin() + lo, sc.added.begin() + lo + m, 0.0f);
    }
    for (usize j = j0; j < j1; ++j) {
        usize lo = j * res + i0;
        const float* ha = h + lo;
        const float* hb = h + lo + res;
        const float* va = vel + lo;
        const float* vb = vel + lo + res;
        const u8* ga = gate + lo;
        const u8* gb = gate + lo + res;
        float* ra = sc.removed.data() + lo;
        float* rb = sc.removed.data() + lo + res;
        float* aa = sc.added.data() + lo;
        float* ab = sc.added.data() + lo + res;
        const float* ba = BED ? bed + lo : nullptr;
        const float* bb = BED ? bed + lo + res : nullptr;
        // src/fluid_core.rs:2916-2960 open_row_pair
        for (usize i = 0; i < m; ++i) {
            float speed = 0.5f * (va[i] + vb[i]);
            float bd = BED ? bb[i] : 0.0f, bc = BED ? ba[i] : 0.0f;
            float dh = open_edge_dh(BED, hb[i], ha[i], 0.0f, ga[i], bd, bc, speed, dt, cell, frac_cap);
            float up = speed > 0.0f ? 0.0f : dh;
            rb[i] += up;
            aa[i] += up;
        }
        for (usize i = 0; i < m; ++i) {
            float speed = 0.5f * (va[i] + vb[i]);
            float bd = BED ? ba[i] : 0.0f, bc = BED ? bb[i] : 0.0f;
            float dh = open_edge_dh(BED, ha[i], hb[i], ra[i], gb[i], bd, bc, speed, dt, cell, frac_cap);
            float down = speed > 0.0f ? dh : 0.0f;
            ra[i] += down;
            ab[i] += down;
        }
    }
    for (usize j = j0; j <= j1; ++j) {
        usize lo = j * res + i0;
        for (usize c = 0; c < m; ++c) {
            float r = sc.removed[lo + c], a = sc.added[lo + c];
            float moved = rmax(h[lo + c] - r + a, 0.0f);
            h[lo + c] = (r > 0.0f || a > 0.0f) ? moved : h[lo + c];
        }
    }
}

// src/fluid_core.rs:3140-3206 transport_open_ref + flux_open :3411-3440 (serial definition)
void transport_open_serial(float* h, const float* vel, const u8* gate, usize res, float cell,
                           float dt, usize i0, usize i1, usize j0, usize j1, bool along_x,
                           const float* bed, float frac_cap, Scratch& sc) {
    for (usize j = j0; j <= j1; ++j)
        for (usize i = i0; i <= i1; ++i) sc.removed[j * res + i] = sc.added[j * res + i] = 0.0f;
    auto flux = [&](usize a, usize b, float speed) {
        usize donor = speed > 0.0f ? a : b, recv = speed > 0.0f ? b : a;
        float room = h[donor] - sc.removed[donor];
        if (room <= 1.0e-8f) return;
        if (gate[recv] == 0 && h[recv] <= 1.0e-6f) return;
        float frac = rmin(fabsf(speed) * dt / cell, frac_cap);
        float dh = rmin(h[donor] * frac, room);
        if (dh <= 1.0e-8f) return;
        sc.removed[donor] += dh;
        sc.added[recv] += dh;
    };
    auto edge = [&](usize a, usize b) {
        float speed = 0.5f * (vel[a] + vel[b]);
        if (fabsf(speed) < 1.0e-5f) return;
        if (bed) {
            usize donor = speed > 0.0f ? a : b, recv = speed > 0.0f ? b : a;
            if (h[recv] <= 1.0e-6f && bed[recv] > bed[donor] + h[donor] + 1.0e-3f) return;
        }
        flux(a, b, speed);
    };
    if (along_x) {
        for (usize j = j0; j <= j1; ++j)
            for (usize i = i0; i < i1; ++i) edge(j * res + i, j * res + i + 1);
    } else {
        for (usize j = j0; j < j1; ++j)
            for (usize i = i0; i <= i1; ++i) edge(j * res + i, j * res + i + res);
    }
    for (usize j = j0; j <= j1; ++j)
        for (usize i = i0; i <= i1; ++i) {
            usize idx = j * res + i;
            float r = sc.removed[idx], a = sc.added[idx];
            float moved = rmax(h[idx] - r + a, 0.0f);
            h[idx] = (r > 0.0f || a > 0.0f) ? moved : h[idx];
        }
}

// ---------------------------------------------------------------------- walls
// A body's footprint in the sheet (src/fluid_core.rs:213-240 HydroSolid).
struct HydroSolid {
    float x, z, yaw, half_length, half_width, bottom_y, top_y;
    bool contact;
    float radius, width;
};

// src/fluid_core.rs:4584-4594: inside the yawed rectangle (yaw 0 = long axis +Z).
bool solid_contains(const HydroSolid& s, float x, float z) {
    const float dx = x - s.x, dz = z - s.z;
    const float fx = sinf(s.yaw), fz = cosf(s.yaw);
    const float along = dx * fx + dz * fz;
    const float lat = dx * fz + dz * (-fx);
    return fabsf(along) <= rmax(s.half_length, 0.0f) && fabsf(lat) <= rmax(s.half_width, 0.0f);
}

// src/fluid_core.rs:4596-4604: a wall only where the free surface stands above
// the underside and the bed below the top.
bool solid_overlaps(const HydroSolid& s, float x, float z, float eta, float bed) {
    if (s.half_length <= 1.0e-4f || s.half_width <= 1.0e-4f) return false;
    if (!solid_contains(s, x, z)) return false;
    return eta > s.bottom_y + 1.0e-4f && bed < s.top_y;
}

// src/fluid_core.rs:7288-7360 solid_mask: 2 = wall, 1 = tire contact (contacts
// are drawn second and win a shared cell). The surface tested is the highest
// of the cell and its four neighbours (water layer over its bed).
std::vector<u8> solid_mask(const std::vector<HydroSolid>& solids, usize res, float cell, const float* origin,
                           const float* water, const float* bed) {
    std::vector<u8> mask(res * res, 0);
    for (int pass = 0; pass < 2; ++pass) {
        const bool contact = pass == 1;
        const u8 value = contact ? 1 : 2;
        for (const HydroSolid& s : solids) {
            if (s.contact != contact) continue;
            if (s.half_length <= 1.0e-4f || s.half_width <= 1.0e-4f) continue;
            const float reach = hypotf(rmax(s.half_length, 0.0f), rmax(s.half_width, 0.0f)) + cell;
            if (!finite(reach) || !finite(s.x) || !finite(s.z)) continue;
            const float lo_i = floorf((s.x - reach - origin[0]) / cell - 0.5f);
            const float hi_i = ceilf((s.x + reach - origin[0]) / cell - 0.5f);
            const float lo_j = floorf((s.z - reach - origin[1]) / cell - 0.5f);
            const float hi_j = ceilf((s.z + reach - origin[1]) / cell - 0.5f);
            const float top = (float)(res - 1);
            if (hi_i < 0.0f || hi_j < 0.0f || lo_i > top || lo_j > top) continue;
            const usize i0 = f2usize(rmax(lo_i, 0.0f)), i1 = f2usize(rmin(hi_i, top));
            const usize j0 = f2usize(rmax(lo_j, 0.0f)), j1 = f2usize(rmin(hi_j, top));
            for (usize j = j0; j <= j1; ++j)
                for (usize i = i0; i <= i1; ++i) {
                    const usize idx = j * res + i;
                    if (mask[idx] == value) continue;
                    const float x = origin[0] + ((float)i + 0.5f) * cell;
                    const float z = origin[1] + ((float)j + 0.5f) * cell;
                    float eta = bed[idx] + water[idx];
                    if (i > 0) eta = rmax(eta, bed[idx - 1] + water[idx - 1]);
                    if (i + 1 < res) eta = rmax(eta, bed[idx + 1] + water[idx + 1]);
                    if (j > 0) eta = rmax(eta, bed[idx - res] + water[idx - res]);
                    if (j + 1 < res) eta = rmax(eta, bed[idx + res] + water[idx + res]);
                    if (solid_overlaps(s, x, z, eta, bed[idx])) mask[idx] = value;
                }
        }
    }
    return mask;
}

// The four neighbours in the reference's order: (-1,0), (1,0), (0,-1), (0,1).
static const int NB4[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};

inline bool in_grid(long i, long j, usize res) { return i >= 0 && j >= 0 && i < (long)res && j < (long)res; }

// src/fluid_core.rs:4382-4444 displace_occupied: a covered column moves, in
// equal shares, to its open neighbours (the 5 x 5 block when no four-neighbour
// is open); a column with nowhere to go stays.
void displace_occupied(float* h, float* u, float* v, const u8* solid, usize res) {
    std::vector<float> give(res * res, 0.0f);
    std::vector<usize> neigh;
    for (usize j = 0; j < res; ++j)
        for (usize i = 0; i < res; ++i) {
            const usize idx = j * res + i;
            if (!solid[idx]) continue;
            const float vol = h[idx];
            if (vol <= 1.0e-8f) {
                h[idx] = u[idx] = v[idx] = 0.0f;
                continue;
            }
            neigh.clear();
            for (const auto& d : NB4) {
                const long ni = (long)i + d[0], nj = (long)j + d[1];
                if (!in_grid(ni, nj, res)) continue;
                const usize q = (usize)nj * res + (usize)ni;
                if (!solid[q]) neigh.push_back(q);
            }
            if (neigh.empty())
                for (long dj = -2; dj <= 2; ++dj)
                    for (long di = -2; di <= 2; ++di) {
                        const long ni = (long)i + di, nj = (long)j + dj;
                        if (!in_grid(ni, nj, res)) continue;
                        const usize q = (usize)nj * res + (usize)ni;
                        if (!solid[q]) neigh.push_back(q);
                    }
            if (neigh.empty()) continue;
            h[idx] = u[idx] = v[idx] = 0.0f;
            const float share = vol / (float)neigh.size();
            for (usize q : neigh) give[q] += share;
        }
    for (usize k = 0; k < res * res; ++k)
        if (give[k] > 0.0f) h[k] += give[k];
}

// src/fluid_core.rs:4225-4276 lift_solid_surface: a wall cell's surface is the
// mean of the wet open cells within two cells (its own when there are none).
void lift_solid_surface(float* eta, const float* h, const u8* solid, usize res, const Box& b, float eps,
                        float* tmp) {
    for (usize j = b.j0; j <= b.j1; ++j)
        for (usize i = b.i0; i <= b.i1; ++i) {
            const usize idx = j * res + i;
            if (!solid[idx]) continue;
            float acc = 0.0f, n = 0.0f;
            for (long dj = -2; dj <= 2; ++dj)
                for (long di = -2; di <= 2; ++di) {
                    if (di == 0 && dj == 0) continue;
                    const long ni = (long)i + di, nj = (long)j + dj;
                    if (!in_grid(ni, nj, res)) continue;
                    const usize q = (usize)nj * res + (usize)ni;
                    if (solid[q] || h[q] <= eps) continue;
                    acc += eta[q];
                    n += 1.0f;
                }
            tmp[idx] = n > 0.0f ? acc / n : eta[idx];
        }
    for (usize j = b.j0; j <= b.j1; ++j)
        for (usize i = b.i0; i <= b.i1; ++i)
            if (solid[j * res + i]) eta[j * res + i] = tmp[j * res + i];
}

// src/fluid_core.rs:4278-4326 write_noslip_ghost: a wall cell takes minus the
// mean velocity of its wet open four-neighbours (zero when there are none).
void write_noslip_ghost(float* u, float* v, const float* h, const u8* solid, usize res, const Box& b, float eps) {
    std::vector<std::tuple<usize, float, float>> ghosts;
    for (usize j = b.j0; j <= b.j1; ++j)
        for (usize i = b.i0; i <= b.i1; ++i) {
            const usize idx = j * res + i;
            if (!solid[idx]) continue;
            float au = 0.0f, av = 0.0f, n = 0.0f;
            for (const auto& d : NB4) {
                const long ni = (long)i + d[0], nj = (long)j + d[1];
                if (!in_grid(ni, nj, res)) continue;
                const usize q = (usize)nj * res + (usize)ni;
                if (solid[q] || h[q] <= eps) continue;
                au += u[q];
                av += v[q];
                n += 1.0f;
            }
            if (n > 0.0f)
                ghosts.emplace_back(idx, -au / n, -av / n);
            else
                ghosts.emplace_back(idx, 0.0f, 0.0f);
        }
    for (const auto& g : ghosts) {
        u[std::get<0>(g)] = std::get<1>(g);
        v[std::get<0>(g)] = std::get<2>(g);
    }
}

// src/fluid_core.rs:4328-4380 block_into_solid: a wet open cell loses the
// part of its velocity that points into a wall neighbour, direction by
// direction in the neighbour order.
void block_into_solid(float* u, float* v, const float* h, const u8* solid, usize res, const Box& b, float eps) {
    std::vector<std::tuple<usize, float, float>> next;
    for (usize j = b.j0; j <= b.j1; ++j)
        for (usize i = b.i0; i <= b.i1; ++i) {
            const usize idx = j * res + i;
            if (solid[idx] || h[idx] <= eps) continue;
            float ux = u[idx], vx = v[idx];
            bool hit = false;
            for (const auto& d : NB4) {
                const long ni = (long)i + d[0], nj = (long)j + d[1];
                if (!in_grid(ni, nj, res)) continue;
                if (!solid[(usize)nj * res + (usize)ni]) continue;
                const float nx = (float)d[0], nz = (float)d[1];
                const float vn = ux * nx + vx * nz;
                if (vn > 0.0f) {
                    ux -= vn * nx;
                    vx -= vn * nz;
                    hit = true;
                }
            }
            if (hit) next.emplace_back(idx, ux, vx);
        }
    for (const auto& t : next) {
        u[std::get<0>(t)] = std::get<1>(t);
        v[std::get<0>(t)] = std::get<2>(t);
    }
}

// src/fluid_core.rs:4446-4563 redirect_into_walls: the discharge aimed at a
// wall (the cell's own, or the stream feeding it when that is faster) turns
// aside to the open flanks, as much as stands above their mean depth.
void redirect_into_walls(float* h, const float* u, const float* v, const u8* solid, const float* bed, usize res,
                         float cell, float dt, const Box& b, Scratch& sc) {
    const usize ri0 = sat_sub(b.i0, 1), ri1 = std::min(b.i1 + 1, res - 1);
    const usize rj0 = sat_sub(b.j0, 1), rj1 = std::min(b.j1 + 1, res - 1);
    for (usize j = rj0; j <= rj1; ++j)
        for (usize i = ri0; i <= ri1; ++i) sc.removed[j * res + i] = sc.added[j * res + i] = 0.0f;
    for (usize j = b.j0; j <= b.j1; ++j)
        for (usize i = b.i0; i <= b.i1; ++i) {
            const usize idx = j * res + i;
            if (solid[idx] || h[idx] < 0.02f) continue;
            for (const auto& d : NB4) {
                const long di = d[0], dj = d[1];
                const long ni = (long)i + di, nj = (long)j + dj;
                if (!in_grid(ni, nj, res)) continue;
                if (!solid[(usize)nj * res + (usize)ni]) continue;
                float vn = u[idx] * (float)di + v[idx] * (float)dj;
                const long ui = (long)i - di, uj = (long)j - dj;
                if (in_grid(ui, uj, res)) {
                    const usize up = (usize)uj * res + (usize)ui;
                    if (!solid[up]) {
                        const float feed = u[up] * (float)di + v[up] * (float)dj;
                        if (feed > vn) vn = feed;
                    }
                }
                if (vn < 0.05f) continue;
                const long perp[2][2] = {{di != 0 ? 0 : -1, di != 0 ? -1 : 0}, {di != 0 ? 0 : 1, di != 0 ? 1 : 0}};
                usize dest[2] = {0, 0};
                usize n_dest = 0;
                float flank = 0.0f;
                for (const auto& pq : perp) {
                    const long qi = (long)i + pq[0], qj = (long)j + pq[1];
                    if (!in_grid(qi, qj, res)) continue;
                    const usize q = (usize)qj * res + (usize)qi;
                    if (solid[q]) continue;
                    if (h[q] <= 1.0e-6f && bed[q] > bed[idx] + h[idx] + 1.0e-3f) continue;
                    dest[n_dest++] = q;
                    flank += h[q];
                }
                if (n_dest == 0) continue;
                const float excess = h[idx] - flank / (float)n_dest;
                if (excess < 2.0e-3f) continue;
                const float room = h[idx] - sc.removed[idx];
                if (room < 1.0e-6f) continue;
                const float frac = rmin(vn * dt / cell, 0.45f);
                const float dh = rmin(rmin(excess, h[idx] * frac), room);
                if (dh < 1.0e-8f) continue;
                sc.removed[idx] += dh;
                const float share = dh / (float)n_dest;
                for (usize k = 0; k < n_dest; ++k) sc.added[dest[k]] += share;
            }
        }
    for (usize j = rj0; j <= rj1; ++j)
        for (usize i = ri0; i <= ri1; ++i) {
            const usize idx = j * res + i;
            if (sc.removed[idx] > 0.0f || sc.added[idx] > 0.0f)
                h[idx] = rmax(h[idx] - sc.removed[idx] + sc.added[idx], 0.0f);
        }
}

// src/fluid_core.rs:4565-4582 solid_near (radius 1): a wall among the eight neighbours.
bool solid_near(const u8* mask, usize res, usize i, usize j) {
    for (long dj = -1; dj <= 1; ++dj)
        for (long di = -1; di <= 1; ++di) {
            if (di == 0 && dj == 0) continue;
            const long ni = (long)i + di, nj = (long)j + dj;
            if (in_grid(ni, nj, res) && mask[(usize)nj * res + (usize)ni]) return true;
        }
    return false;
}

// src/fluid_core.rs:2084-2129 force_gravity_solid, the serial sweep (the step
// pair runs its sheets with serial inner loops): gravity, with the mobility
// raised to at least 1 beside a wall under 8 cm of water, then the
// confinement kick, cell by cell in raster order.
void force_gravity_solid(const float* h, float* u, float* v, const float* nu, const float* p, const u8* mask,
                         usize res, float cell, float dt, float vorticity, float eps, const Box& b, bool inner_par) {
    if (b.j1 - b.j0 >= 47 && b.i1 - b.i0 >= 31 && inner_par) {
        // force_gravity_solid_par (:2131-2202): gravity on every cell first,
        // then the same forward confinement sweep.
        for (usize j = b.j0; j <= b.j1; ++j)
            for (usize i = b.i0; i <= b.i1; ++i) {
                const usize idx = j * res + i;
                if (h[idx] <= eps) continue;
                float px, pz;
                grad(p, res, i, j, cell, px, pz);
                float mob = sheet_mobility_for(nu[idx]);
                if (h[idx] > 0.08f && solid_near(mask, res, i, j)) mob = rmax(mob, 1.0f);
                u[idx] += -GRAVITY * px * mob * dt;
                v[idx] += -GRAVITY * pz * mob * dt;
            }
        if (vorticity <= 0.0f) return;
        for (usize j = b.j0; j <= b.j1; ++j)
            for (usize i = b.i0; i <= b.i1; ++i)
                if (h[j * res + i] > eps) confine_one(u, v, u, v, res, i, j, cell, dt, vorticity);
        return;
    }
    for (usize j = b.j0; j <= b.j1; ++j)
        for (usize i = b.i0; i <= b.i1; ++i) {
            const usize idx = j * res + i;
            if (h[idx] <= eps) continue;
            float px, pz;
            grad(p, res, i, j, cell, px, pz);
            float mob = sheet_mobility_for(nu[idx]);
            if (h[idx] > 0.08f && solid_near(mask, res, i, j)) mob = rmax(mob, 1.0f);
            u[idx] += -GRAVITY * px * mob * dt;
            v[idx] += -GRAVITY * pz * mob * dt;
            if (vorticity > 0.0f) confine_one(u, v, u, v, res, i, j, cell, dt, vorticity);
        }
}

// src/fluid_core.rs:3894-3963 transport with move_edge_bufs (:4178-4223): the
// walled donor-cell flux. An edge touching a wall moves nothing; a dry bank
// above the donor's surface takes nothing.
void transport_walled(float* h, const float* vel, const u8* gate, usize res, float cell, float dt, const Box& b,
                      bool along_x, const u8* solid, const float* bed, Scratch& sc) {
    for (usize j = b.j0; j <= b.j1; ++j)
        for (usize i = b.i0; i <= b.i1; ++i) sc.removed[j * res + i] = sc.added[j * res + i] = 0.0f;
    auto edge = [&](usize a, usize c) {
        if (solid[a] || solid[c]) return;
        const float speed = 0.5f * (vel[a] + vel[c]);
        if (fabsf(speed) < 1.0e-5f) return;
        const usize donor = speed > 0.0f ? a : c, recv = speed > 0.0f ? c : a;
        if (h[recv] <= 1.0e-6f && bed[recv] > bed[donor] + h[donor] + 1.0e-3f) return;
        const float room = h[donor] - sc.removed[donor];
        if (room <= 1.0e-8f) return;
        if (gate[recv] == 0 && h[recv] <= 1.0e-6f) return;
        const float frac = rmin(fabsf(speed) * dt / cell, 0.45f);
        const float dh = rmin(h[donor] * frac, room);
        if (dh <= 1.0e-8f) return;
        sc.removed[donor] += dh;
        sc.added[recv] += dh;
    };
    if (along_x) {
        for (usize j = b.j0; j <= b.j1; ++j)
            for (usize i = b.i0; i < b.i1; ++i) edge(j * res + i, j * res + i + 1);
    } else {
        for (usize j = b.j0; j < b.j1; ++j)
            for (usize i = b.i0; i <= b.i1; ++i) edge(j * res + i, (j + 1) * res + i);
    }
    for (usize j = b.j0; j <= b.j1; ++j)
        for (usize i = b.i0; i <= b.i1; ++i) {
            const usize idx = j * res + i;
            if (sc.removed[idx] > 0.0f || sc.added[idx] > 0.0f)
                h[idx] = rmax(h[idx] - sc.removed[idx] + sc.added[idx], 0.0f);
        }
}

// -------------------------------------------------------------------- substep
// src/fluid_core.rs:1879-2082, open sheet (no walls), gravity drive.
void substep(float* h, float* u, float* v, const float* bed, const float* nu, const u8* gate,
             usize res, float cell, float dt, float vorticity, float eps, usize i0, usize i1,
             usize j0, usize j1, bool banks, bool do_flux, Scratch& sc, bool inner_par,
             const u8* solid = nullptr) {
    const Box box{i0, i1, j0, j1};
    usize hi0 = sat_sub(i0, 2), hi1 = std::min(i1 + 2, res - 1);
    usize hj0 = sat_sub(j0, 2), hj1 = std::min(j1 + 2, res - 1);
    for (usize j = hj0; j <= hj1; ++j)
        for (usize i = hi0; i <= hi1; ++i) sc.a[j * res + i] = bed[j * res + i] + h[j * res + i];
    if (solid) lift_solid_surface(sc.a.data(), h, solid, res, box, eps, sc.e.data());
    blur_box(sc.a.data(), sc.b.data(), sc.e.data(), res, i0, i1, j0, j1, GAUSS);
    blur_box(sc.a.data(), sc.c.data(), sc.e.data(), res, i0, i1, j0, j1, STEEP);
    for (usize j = j0; j <= j1; ++j)
        for (usize i = i0; i <= i1; ++i) {
            usize idx = j * res + i;
            float filtered = 0.62f * sc.b[idx] + 0.38f * sc.c[idx];
            sc.d[idx] = 0.45f * filtered + 0.55f * sc.a[idx];
        }
    if (solid) {
        write_noslip_ghost(u, v, h, solid, res, box, eps);
        force_gravity_solid(h, u, v, nu, sc.d.data(), solid, res, cell, dt, vorticity, eps, box, inner_par);
    } else {
        force_gravity_open(h, u, v, nu, sc.d.data(), res, cell, dt, vorticity, eps, i0, i1, j0, j1, inner_par);
    }
    bool project = solid || cell > FINE_CELL_M + 1.0e-6f;
    if (project) {
        for (usize j = j0; j <= j1; ++j)
            for (usize i = i0; i <= i1; ++i) {
                usize idx = j * res + i;
                float ux, vz;
                grad_vel(u, v, res, i, j, cell, ux, vz);
                float div = ux + vz;
                float lap_h = lap(sc.a.data(), res, i, j, cell);
                float overload = 1.0f + rclamp(nu[idx] / 231.0f, 0.0f, 6.0f);
                sc.b[idx] = div * overload - 0.015f * overload * lap_h;
            }
        blur_box(sc.b.data(), sc.c.data(), sc.e.data(), res, i0, i1, j0, j1, GAUSS);
        blur_box(sc.b.data(), sc.a.data(), sc.e.data(), res, i0, i1, j0, j1, STEEP);
        for (usize j = j0; j <= j1; ++j)
            for (usize i = i0; i <= i1; ++i) {
                usize idx = j * res + i;
                sc.d[idx] = 0.62f * sc.c[idx] + 0.38f * sc.a[idx];
            }
    }
    uint64_t memo_nu = fbits(std::numeric_limits<float>::quiet_NaN());  // f32::NAN
    float memo_decay = 1.0f;
    for (usize j = j0; j <= j1; ++j)
        for (usize i = i0; i <= i1; ++i) {
            usize idx = j * res + i;
            if (h[idx] <= eps) continue;
            if (project) {
                float qx, qz;
                grad(sc.d.data(), res, i, j, cell, qx, qz);
                u[idx] += 0.012f * dt * qx;
                v[idx] += 0.012f * dt * qz;
            }
            float nu_here = nu[idx];
            if (fbits(nu_here) != memo_nu) {
                memo_nu = fbits(nu_here);
                memo_decay = expf(-sheet_damp(nu_here) * dt);
            }
            float decay = memo_decay;
            u[idx] = finite_speed(u[idx] * decay, FILM_SPEED_CAP_MPS);
            v[idx] = finite_speed(v[idx] * decay, FILM_SPEED_CAP_MPS);
        }
    if (solid) {
        redirect_into_walls(h, u, v, solid, bed, res, cell, dt, box, sc);
        block_into_solid(u, v, h, solid, res, box, eps);
        write_noslip_ghost(u, v, h, solid, res, box, eps);
    }
    if (!do_flux) return;
    if (solid) {
        transport_walled(h, u, gate, res, cell, dt, box, true, solid, bed, sc);
        transport_walled(h, v, gate, res, cell, dt, box, false, solid, bed, sc);
    } else {
        const float* open_bed = banks ? bed : nullptr;
        transport_open_rows(banks, h, u, gate, res, cell, dt, i0, i1, j0, j1, true, open_bed, 0.45f, sc);
        transport_open_rows(banks, h, v, gate, res, cell, dt, i0, i1, j0, j1, false, open_bed, 0.45f, sc);
    }
    for (usize j = j0; j <= j1; ++j)
        for (usize i = i0; i <= i1; ++i) {
            usize idx = j * res + i;
            if (eps > 0.0f && h[idx] < eps) h[idx] = u[idx] = v[idx] = 0.0f;
        }
}

// ---------------------------------------------------------------- work boxes
// src/fluid_core.rs:1306-1319
float wet_sum(const float* h, usize n, float eps) {
    float lanes[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    usize chunks = n / 8;
    for (usize c = 0; c < chunks; ++c)
        for (int k = 0; k < 8; ++k) {
            float x = h[c * 8 + k];
            lanes[k] += x > eps ? x : 0.0f;
        }
    float sum = rsum(lanes, 8);
    for (usize k = chunks * 8; k < n; ++k) {
        float x = h[k];
        sum += x > eps ? x : 0.0f;
    }
    return sum;
}

// src/fluid_core.rs:794-818
bool wet_bounds(const float* h, usize res, usize margin, Box& out) {
    usize j0 = (usize)-1, j1 = 0, i0 = (usize)-1, i1 = 0;
    for (usize j = 0; j < res; ++j) {
        const float* row = h + j * res;
        long first = -1, last = -1;
        for (usize i = 0; i < res; ++i)
            if (row[i] > 0.0f) {
                if (first < 0) first = (long)i;
                last = (long)i;
            }
        if (first < 0) continue;
        j0 = std::min(j0, j);
        j1 = j;
        i0 = std::min(i0, (usize)first);
        i1 = std::max(i1, (usize)last);
    }
    if (j0 == (usize)-1) return false;
    out = {sat_sub(i0, margin), std::min(i1 + margin, res - 1), sat_sub(j0, margin), std::min(j1 + margin, res - 1)};
    return true;
}

// src/fluid_core.rs:1449-1479
bool boxes_touch(const Box& a, const Box& b) {
    return sat_sub(a.i0, 1) <= b.i1 + 1 && sat_sub(b.i0, 1) <= a.i1 + 1 &&
           sat_sub(a.j0, 1) <= b.j1 + 1 && sat_sub(b.j0, 1) <= a.j1 + 1;
}
void merge_boxes(std::vector<Box>& boxes) {
    for (;;) {
        bool did = false;
        usize i = 0;
        while (i < boxes.size()) {
            usize j = i + 1;
            while (j < boxes.size()) {
                if (boxes_touch(boxes[i], boxes[j])) {
                    Box a = boxes[i], b = boxes[j];
                    boxes[i] = {std::min(a.i0, b.i0), std::max(a.i1, b.i1), std::min(a.j0, b.j0), std::max(a.j1, b.j1)};
                    boxes[j] = boxes.back();  // swap_remove
                    boxes.pop_back();
                    did = true;
                } else {
                    ++j;
                }
            }
            ++i;
        }
        if (!did) break;
    }
}

const usize SPLIT_HALO = 6;

// src/fluid_core.rs:1325-1447 (run-length bodies)
std::vector<Box> sheet_work_boxes(const float* h, usize res, float eps, bool allow_split) {
    usize i0 = res, i1 = 0, j0 = res, j1 = 0, wet = 0;
    for (usize j = 0; j < res; ++j) {
        const float* row = h + j * res;
        usize c = 0;
        for (usize i = 0; i < res; ++i) c += row[i] > eps;
        if (c == 0) continue;
        wet += c;
        usize first = 0, last = 0;
        for (usize i = 0; i < res; ++i) if (row[i] > eps) { first = i; break; }
        for (usize i = res; i-- > 0;) if (row[i] > eps) { last = i; break; }
        i0 = std::min(i0, first);
        i1 = std::max(i1, last);
        j0 = std::min(j0, j);
        j1 = std::max(j1, j);
    }
    if (wet == 0) return {};
    Box whole = {sat_sub(i0, 3), std::min(i1 + 3, res - 1), sat_sub(j0, 3), std::min(j1 + 3, res - 1)};
    bool solid = wet == (i1 - i0 + 1) * (j1 - j0 + 1);
    if (!allow_split || solid) return {whole};
    std::vector<std::pair<usize, usize>> all;
    std::vector<uint32_t> parent;
    std::vector<Box> bbox;
    std::vector<usize> first;
    auto root = [&](uint32_t x) {
        while (parent[x] != x) {
            uint32_t up = parent[parent[x]];
            parent[x] = up;
            x = up;
        }
        return x;
    };
    usize prev0 = 0, prev1 = 0;
    for (usize j = j0; j <= j1; ++j) {
        const float* row = h + j * res;
        usize start = all.size();
        usize i = i0;
        while (i <= i1) {
            if (!(row[i] > eps)) { ++i; continue; }
            usize a = i;
            while (i <= i1 && row[i] > eps) ++i;
            usize b = i - 1;
            uint32_t id = (uint32_t)all.size();
            all.push_back({a, b});
            parent.push_back(id);
            bbox.push_back({a, b, j, j});
            first.push_back(j * res + a);
            for (usize k = prev0; k < prev1; ++k) {
                usize pa = all[k].first, pb = all[k].second;
                if (pa <= b && a <= pb) {
                    uint32_t ra = root((uint32_t)k), rb = root(id);
                    if (ra != rb) {
                        uint32_t keep = ra < rb ? ra : rb, gone = ra < rb ? rb : ra;
                        parent[gone] = keep;
                        Box g = bbox[gone];
                        Box& kb = bbox[keep];
                        kb.i0 = std::min(kb.i0, g.i0);
                        kb.i1 = std::max(kb.i1, g.i1);
                        kb.j0 = std::min(kb.j0, g.j0);
                        kb.j1 = std::max(kb.j1, g.j1);
                        first[keep] = std::min(first[keep], first[gone]);
                    }
                }
            }
        }
        prev0 = start;
        prev1 = all.size();
    }
    std::vector<std::pair<usize, Box>> bodies;
    for (usize k = 0; k < all.size(); ++k)
        if (parent[k] == (uint32_t)k) bodies.push_back({first[k], bbox[k]});
    std::sort(bodies.begin(), bodies.end(), [](const std::pair<usize, Box>& x, const std::pair<usize, Box>& y) { return x.first < y.first; });
    std::vector<Box> boxes;
    for (auto& bd : bodies) {
        Box c = bd.second;
        boxes.push_back({sat_sub(c.i0, SPLIT_HALO), std::min(c.i1 + SPLIT_HALO, res - 1),
                         sat_sub(c.j0, SPLIT_HALO), std::min(c.j1 + SPLIT_HALO, res - 1)});
    }
    merge_boxes(boxes);
    if (boxes.size() == 1 || boxes.size() > 8) return {whole};
    return boxes;
}

// src/fluid_core.rs:11134-11227 (test-only flood-fill definition)
std::vector<Box> sheet_work_boxes_flood(const float* h, usize res, float eps, bool allow_split) {
    usize i0 = res, i1 = 0, j0 = res, j1 = 0, wet = 0;
    for (usize j = 0; j < res; ++j) {
        const float* row = h + j * res;
        usize c = 0;
        for (usize i = 0; i < res; ++i) c += row[i] > eps;
        if (c == 0) continue;
        wet += c;
        usize first = 0, last = 0;
        for (usize i = 0; i < res; ++i) if (row[i] > eps) { first = i; break; }
        for (usize i = res; i-- > 0;) if (row[i] > eps) { last = i; break; }
        i0 = std::min(i0, first); i1 = std::max(i1, last);
        j0 = std::min(j0, j); j1 = std::max(j1, j);
    }
    if (wet == 0) return {};
    Box whole = {sat_sub(i0, 3), std::min(i1 + 3, res - 1), sat_sub(j0, 3), std::min(j1 + 3, res - 1)};
    bool solid = wet == (i1 - i0 + 1) * (j1 - j0 + 1);
    if (!allow_split || solid) return {whole};
    std::vector<u8> mark(res * res, 0);
    std::vector<usize> queue;
    std::vector<Box> boxes;
    for (usize j = j0; j <= j1; ++j)
        for (usize i = i0; i <= i1; ++i) {
            usize s = j * res + i;
            if (h[s] <= eps || mark[s]) continue;
            usize ci0 = i, ci1 = i, cj0 = j, cj1 = j;
            mark[s] = 1;
            queue.clear();
            queue.push_back(s);
            while (!queue.empty()) {
                usize cur = queue.back();
                queue.pop_back();
                usize cj = cur / res, ci = cur - cj * res;
                ci0 = std::min(ci0, ci); ci1 = std::max(ci1, ci);
                cj0 = std::min(cj0, cj); cj1 = std::max(cj1, cj);
                long neigh[4] = {ci > 0 ? (long)cur - 1 : -1, ci + 1 < res ? (long)cur + 1 : -1,
                                 cj > 0 ? (long)(cur - res) : -1, cj + 1 < res ? (long)(cur + res) : -1};
                for (long nidx : neigh)
                    if (nidx >= 0 && !mark[nidx] && h[nidx] > eps) {
                        mark[nidx] = 1;
                        queue.push_back((usize)nidx);
                    }
            }
            boxes.push_back({sat_sub(ci0, SPLIT_HALO), std::min(ci1 + SPLIT_HALO, res - 1),
                             sat_sub(cj0, SPLIT_HALO), std::min(cj1 + SPLIT_HALO, res - 1)});
        }
    merge_boxes(boxes);
    if (boxes.size() == 1 || boxes.size() > 8) return {whole};
    return boxes;
}

// src/fluid_core.rs:1537-1657
std::vector<Box> awake_work_boxes(const float* h, const float* u, const float* v, const float* bed,
                                  usize res, float cell, float eps) {
    usize tiles = (res + SLEEP_TILE - 1) / SLEEP_TILE;
    usize ntile = tiles * tiles;
    std::vector<u8> hot(ntile, 0), grown(ntile, 0);
    for (usize tj = 0; tj < tiles; ++tj)
        for (usize ti = 0; ti < tiles; ++ti) {
            usize i0 = ti * SLEEP_TILE, j0 = tj * SLEEP_TILE;
            usize i1 = std::min(i0 + SLEEP_TILE, res), j1 = std::min(j0 + SLEEP_TILE, res);
            bool awake = false;
            for (usize j = j0; j < j1 && !awake; ++j) {
                usize row = j * res;
                for (usize i = i0; i < i1; ++i) {
                    usize idx = row + i;
                    if (h[idx] <= eps) continue;
                    if (hypotf(u[idx], v[idx]) > SLEEP_SPEED) { awake = true; break; }
                    float eta = bed[idx] + h[idx];
                    usize ip = i + 1 < res ? row + i + 1 : idx;
                    usize jp = j + 1 < res ? (j + 1) * res + i : idx;
                    float dex = fabsf(bed[ip] + h[ip] - eta);
                    float dez = fabsf(bed[jp] + h[jp] - eta);
                    if (rmax(dex, dez) > SLEEP_SLOPE * cell) { awake = true; break; }
                }
            }
            if (awake) hot[tj * tiles + ti] = 1;
        }
    for (usize tj = 0; tj < tiles; ++tj)
        for (usize ti = 0; ti < tiles; ++ti) {
            if (!hot[tj * tiles + ti]) continue;
            for (int dj = -1; dj <= 1; ++dj)
                for (int di = -1; di <= 1; ++di) {
                    long ni = (long)ti + di, nj = (long)tj + dj;
                    if (ni >= 0 && nj >= 0 && ni < (long)tiles && nj < (long)tiles) grown[nj * tiles + ni] = 1;
                }
        }
    std::vector<u8> seen(ntile, 0);
    std::vector<usize> stack;
    std::vector<Box> boxes;
    for (usize s = 0; s < ntile; ++s) {
        if (!grown[s] || seen[s]) continue;
        seen[s] = 1;
        stack.clear();
        stack.push_back(s);
        usize ti0 = s % tiles, ti1 = ti0, tj0 = s / tiles, tj1 = tj0;
        while (!stack.empty()) {
            usize cur = stack.back();
            stack.pop_back();
            usize tj = cur / tiles, ti = cur - tj * tiles;
            ti0 = std::min(ti0, ti); ti1 = std::max(ti1, ti);
            tj0 = std::min(tj0, tj); tj1 = std::max(tj1, tj);
            auto visit = [&](usize nidx) {
                if (grown[nidx] && !seen[nidx]) { seen[nidx] = 1; stack.push_back(nidx); }
            };
            if (ti > 0) visit(tj * tiles + ti - 1);
            if (ti + 1 < tiles) visit(tj * tiles + ti + 1);
            if (tj > 0) visit((tj - 1) * tiles + ti);
            if (tj + 1 < tiles) visit((tj + 1) * tiles + ti);
        }
        boxes.push_back({ti0 * SLEEP_TILE, std::min((ti1 + 1) * SLEEP_TILE, res) - 1,
                         tj0 * SLEEP_TILE, std::min((tj1 + 1) * SLEEP_TILE, res) - 1});
    }
    return boxes;
}

// src/fluid_core.rs:1873-1877
bool boxes_apart(const Box& a, const Box& b, usize gap) {
    auto apart = [gap](usize a0, usize a1, usize b0, usize b1) { return a1 + gap < b0 || b1 + gap < a0; };
    return apart(a.i0, a.i1, b.i0, b.i1) || apart(a.j0, a.j1, b.j0, b.j1);
}

// src/fluid_core.rs:1836-1868
void pace3_slices(float* h, float* u, float* v, const u8* gate, usize res, float cell, float dts,
                  uint32_t nsub, float eps, const Box& bx, Scratch& sc) {
    for (uint32_t s = 0; s < nsub; ++s) {
        transport_open_rows(false, h, u, gate, res, cell, dts, bx.i0, bx.i1, bx.j0, bx.j1, true, nullptr, 0.45f, sc);
        transport_open_rows(false, h, v, gate, res, cell, dts, bx.i0, bx.i1, bx.j0, bx.j1, false, nullptr, 0.45f, sc);
    }
    if (eps > 0.0f)
        for (usize j = bx.j0; j <= bx.j1; ++j)
            for (usize i = bx.i0; i <= bx.i1; ++i) {
                usize idx = j * res + i;
                if (h[idx] < eps) h[idx] = u[idx] = v[idx] = 0.0f;
            }
}

// src/fluid_core.rs:1659-1831 step_sheet_scratch (open sheet, gravity drive).
void step_sheet_scratch(float* h, float* u, float* v, const float* bed, const float* nu,
                        const u8* gate, usize res, float cell, float dt, float vorticity, float eps,
                        bool banks, float sub_cap, int pace, Scratch& sc, Scratch* sc2,
                        bool inner_par, const u8* solid = nullptr) {
    bool open_fine = !solid && cell <= FINE_CELL_M + 1.0e-6f;
    bool fine_open = open_fine && pace == 0;
    bool whole_wet = open_fine && (pace == 2 || pace == 3);
    bool awake = open_fine && !whole_wet && !fine_open;
    std::vector<Box> boxes = (fine_open || awake) ? awake_work_boxes(h, u, v, bed, res, cell, eps)
                                                  : sheet_work_boxes(h, res, eps, true);
    if (boxes.empty()) return;
    float cap = finite(sub_cap) ? rclamp(sub_cap, 1.0f, 8.0f) : 8.0f;
    uint32_t nsub;
    if (fine_open) {
        nsub = 1;
    } else {
        float max_s = 0.15f;
        float max_s2 = 0.0f;
        for (const Box& b : boxes)
            for (usize j = b.j0; j <= b.j1; ++j)
                for (usize i = b.i0; i <= b.i1; ++i) {
                    float uu = u[j * res + i], vv = v[j * res + i];
                    float s2 = uu * uu + vv * vv;
                    if (s2 > max_s2) max_s2 = s2;
                }
        max_s = rmax(max_s, sqrtf(max_s2));
        float courant = 0.42f;
        nsub = (uint32_t)rclamp(ceilf((dt * max_s) / (courant * rmax(cell, 1.0e-3f))), 1.0f, cap);
    }
    float dts = dt / (float)nsub;
    if (pace == 3 && whole_wet && nsub > 1) {
        auto run = [&](const Box& b, Scratch& s) {
            substep(h, u, v, bed, nu, gate, res, cell, dt, vorticity, eps, b.i0, b.i1, b.j0, b.j1, banks, false, s, inner_par, solid);
            pace3_slices(h, u, v, gate, res, cell, dts, nsub, eps, b, s);
        };
        if (sc2 && boxes.size() == 2 && boxes_apart(boxes[0], boxes[1], BOX_PAR_GAP)) {
            run(boxes[0], sc);
            run(boxes[1], *sc2);
            return;
        }
        for (const Box& b : boxes) run(b, sc);
        return;
    }
    if (sc2 && boxes.size() == 2 && boxes_apart(boxes[0], boxes[1], BOX_PAR_GAP)) {
        for (uint32_t s = 0; s < nsub; ++s) {
            // The two boxes step on two workers with serial inner loops.
            substep(h, u, v, bed, nu, gate, res, cell, dts, vorticity, eps, boxes[0].i0, boxes[0].i1, boxes[0].j0, boxes[0].j1, banks, true, sc, false, solid);
            substep(h, u, v, bed, nu, gate, res, cell, dts, vorticity, eps, boxes[1].i0, boxes[1].i1, boxes[1].j0, boxes[1].j1, banks, true, *sc2, false, solid);
        }
        return;
    }
    for (uint32_t s = 0; s < nsub; ++s)
        for (const Box& b : boxes)
            substep(h, u, v, bed, nu, gate, res, cell, dts, vorticity, eps, b.i0, b.i1, b.j0, b.j1, banks, true, sc, inner_par, solid);
}

// src/fluid_core.rs:821-889 step_sheet_eps_in / step_sheet_eps
void step_sheet_eps(float* h, float* u, float* v, const float* bed, const float* nu, const u8* gate,
                    usize res, float cell, float dt, float vorticity, float eps, bool banks,
                    float sub_cap, int pace, Scratch& sc, Scratch* sc2, bool inner_par, const u8* solid = nullptr) {
    if (dt <= 0.0f || res == 0) return;
    float sum = wet_sum(h, res * res, eps);
    if (sum <= eps) return;
    sc.fit(res * res);
    if (sc2) sc2->fit(res * res);
    step_sheet_scratch(h, u, v, bed, nu, gate, res, cell, dt, vorticity, eps, banks, sub_cap, pace, sc, sc2, inner_par,
                       solid);
}

// src/fluid_core.rs:9594-9622 (no reach band)
// open_axis: -1 none; 0 a reach along X (its band [c0, c1) of rows keeps its
// current through the window ends: only the row distance counts); 1 along Z.
void soften_border(float* u, float* v, usize res, int open_axis = -1, usize c0 = 0, usize c1 = 0) {
    usize edge = std::max(res / 12, (usize)2);
    usize ends = std::min(edge, res);
    for (usize j = 0; j < res; ++j) {
        bool row_band = std::min(j, res - 1 - j) < edge;
        usize left = row_band ? res : ends, right = row_band ? res : res - ends;
        auto visit = [&](usize i) {
            usize di = std::min(i, res - 1 - i), dj = std::min(j, res - 1 - j);
            usize d = std::min(di, dj);
            if (open_axis == 0 && j >= c0 && j < c1) d = dj;
            else if (open_axis == 1 && i >= c0 && i < c1) d = di;
            if (d >= edge) return;
            float t = (float)d / (float)edge;
            float w = t * t * (3.0f - 2.0f * t);
            usize idx = j * res + i;
            u[idx] *= w;
            v[idx] *= w;
        };
        for (usize i = 0; i < left; ++i) visit(i);
        for (usize i = std::max(right, left); i < res; ++i) visit(i);
    }
}

// --------------------------------------------------------------- window core
struct TirePush {
    float x, z, forward_x, forward_z, radius, width, speed, slip;
};
struct Spray {
    float x, y, z, vx, vy, vz, volume;
    int kind;
};

// src/fluid_core.rs:9877-9897
std::pair<usize, usize> index_span(float origin, float cell, usize res, float center, float reach) {
    if (!(cell > 0.0f) || res == 0) return {0, 0};
    float lo = rmax(floorf((center - reach - origin) / cell - 1.0f), 0.0f);
    float hi = rmax(ceilf((center + reach - origin) / cell + 2.0f), 0.0f);
    usize l = std::min(f2usize(lo), res);
    usize hh = std::max(std::min(f2usize(hi), res), l);
    return {l, hh};
}
void snap_origin(float cx, float cz, float extent, float cell, float* out) {
    float x = cx - extent * 0.5f, z = cz - extent * 0.5f;
    out[0] = floorf(x / cell) * cell;
    out[1] = floorf(z / cell) * cell;
}
std::pair<int, int> world_key(float x, float z, float cell) {
    return {(int)floorf(x / cell), (int)floorf(z / cell)};
}
// src/fluid_core.rs:9641-9662
float dist2_segment(float px, float pz, float ax, float az, float bx, float bz) {
    float abx = bx - ax, abz = bz - az;
    float ab2 = abx * abx + abz * abz;
    float t = ab2 < 1.0e-8f ? 0.0f : rclamp(((px - ax) * abx + (pz - az) * abz) / ab2, 0.0f, 1.0f);
    float dx = px - (ax + abx * t), dz = pz - (az + abz * t);
    return dx * dx + dz * dz;
}
// src/fluid_core.rs:9624-9640
bool near_tire_zone(const std::vector<TirePush>& pushes, float x, float z, float r2) {
    for (const auto& p : pushes) {
        float dx = x - p.x, dz = z - p.z;
        if (dx * dx + dz * dz <= r2) return true;
    }
    for (usize i = 0; i < pushes.size(); ++i)
        for (usize j = i + 1; j < pushes.size(); ++j) {
            const TirePush &a = pushes[i], &b = pushes[j];
            if (fabsf(a.x - b.x) >= 0.45f) continue;
            if (dist2_segment(x, z, a.x, a.z, b.x, b.z) <= r2) return true;
        }
    return false;
}

// near.rs:43-80
struct NearTile {
    std::vector<float> w, s, uw, vw;
    bool fresh = false;
    float idle_s = 0.0f;
    float peak = 0.0f;
    explicit NearTile(usize n2) : w(n2, 0.0f), s(n2, 0.0f), uw(n2, 0.0f), vw(n2, 0.0f) {}
    float left() const { return idle_s <= 0.0f ? 1.0f : expf(-idle_s / NEAR_RESIDUAL_LIFE_S); }
};

// near.rs:118-125
void recentre(std::vector<float>& r) {
    double sum = 0.0;
    for (float x : r) sum += (double)x;
    float mean = (float)(sum / (double)r.size());
    for (float& x : r) x -= mean;
}
// near.rs:128-137
float abs_peak(const std::vector<float>& r) {
    float hi[4] = {0, 0, 0, 0};
    for (usize c = 0; c + 4 <= r.size(); c += 4)
        for (int l = 0; l < 4; ++l) {
            float a = fabsf(r[c + l]);
            hi[l] = a > hi[l] ? a : hi[l];
        }
    return rmax(rmax(rmax(hi[0], hi[1]), hi[2]), hi[3]);
}
// near.rs:139-148
float floor_scale(float base, const std::vector<float>& r) {
    float low = 0.0f;
    for (float x : r) low = rmin(low, x);
    if (low >= 0.0f || base + low >= 0.0f) return 1.0f;
    if (base <= 0.0f) return 0.0f;
    return rclamp(base / -low, 0.0f, 1.0f);
}

struct Patch {
    float origin[2] = {0, 0};
    std::vector<float> water, slurry, uw, vw, us, vs, bed, bed_slurry, moisture;
    std::vector<u8> grain;
    std::vector<uint16_t> col, row;
    Scratch sc[2][2];  // [water, slurry][sc, sc2]
};

struct Core {
    oracle_core_cfg cfg;
    usize res, fres, sub;
    float origin[2];
    std::vector<float> water, slurry, uw, vw, us, vs, bed, moisture;
    std::vector<u8> grain, fine_hold;
    float moisture_ambient = 0.0f;
    std::vector<Patch> patches;
    std::vector<int> hold_owner;   // patch that holds each coarse column (per-tire layout)
    bool fine_on = false;
    bool near_on = true;
    std::map<std::pair<int, int>, NearTile> near;
    // src/fluid_core.rs:4763-4782 Parked (the sheet fields and the tracers;
    // settled dust is off this path).
    struct Parked {
        float water = 0, slurry = 0, uw = 0, vw = 0, us = 0, vs = 0, moisture = 0, foam = 0, turbid = 0, susp = 0;
    };
    std::map<std::pair<int, int>, Parked> parked;
    float spray_m3 = 0.0f;
    std::vector<TirePush> pushes;
    float fine_sub_cap = 8.0f;
    int fine_pace = 0;
    Scratch coarse_sc[2][2];
    std::vector<float> nu_w, nu_s;  // PairScratch rows (src/fluid_core.rs:621-647)
    std::vector<float> fnu_w, fnu_s;
    std::vector<std::vector<float>> fnu_s_rows;
    std::vector<u8> gate, fgate;
    int inflow_j = -1;
    float inflow_x0 = 0, inflow_x1 = 0, inflow_rate = 0;
    double opened_m3 = 0.0;
    // src/fluid_core.rs:333-340 OpenWater, :5284-5303 the setters.
    bool open_water = false;
    float ow_mobility = 0.0f, ow_manning = 0.0f, ow_eddy = 0.0f;
    float surface_diffusion = 0.0f;
    // src/fluid_core.rs:289-320 RiverReach (inlet turbidity is off this path),
    // :274-287 WaveMaker.
    bool reach_on = false;
    bool reach_along_z = false, reach_positive = true;
    float reach_cross0 = 0, reach_cross1 = 0, reach_inlet_eta = 0, reach_outlet_eta = 0, reach_speed = 0;
    usize reach_rows = 1;
    float reach_bank_m3 = 0.0f;
    bool wave_on = false;
    float wave_x0 = 0, wave_x1 = 0, wave_z0 = 0, wave_z1 = 0, wave_dx = 0, wave_dz = 0, wave_amp = 0, wave_period = 0,
          wave_ramp = 0, wave_t = 0;
    // src/fluid_core.rs:5257-5264 set_hydro_solids: walls in the sheet.
    std::vector<HydroSolid> solids;
    // src/fluid_core.rs:4907-4909: scour beside tire contacts.
    std::vector<float> bed_drop;
    float eroded_m3 = 0.0f, scour_hole_m = 0.0f;
    // src/fluid_core.rs:4832-4860: the tracers. Foam (a 0..1 cover), stirred
    // silt (`turbid`, metres of soil in the water) and wheel-lifted suspended
    // solids (`susp`, metres), with their books in f32 as the reference keeps
    // them and FP64 twins of the same terms.
    std::vector<float> foam, turbid, susp, susp_next, susp_taken, tracer_scratch;
    std::vector<uint32_t> foam_live, wet_idx, shore_idx;
    std::vector<u8> foam_live_mark;
    float turbid_settled_m3 = 0.0f, stirred_m3 = 0.0f, entrained_m3 = 0.0f, settled_suspended_m3 = 0.0f;
    double turbid_settled64 = 0.0, stirred64 = 0.0, entrained64 = 0.0, settled_suspended64 = 0.0;
    uint32_t last_susp_capped = 0;
    bool turbidity_enabled = true;   // :4994
    float reach_inlet_turbidity = 0.0f;

    explicit Core(const oracle_core_cfg& c) : cfg(c) {
        res = (usize)c.res;
        fres = (usize)c.fine_res;
        sub = (usize)lroundf(c.cell / c.fine_cell);
        usize n = res * res, fn = fres * fres;
        bed_drop.assign(n, 0.0f);
        foam.assign(n, 0.0f); turbid.assign(n, 0.0f); susp.assign(n, 0.0f);
        susp_next.assign(n, 0.0f); susp_taken.assign(n, 0.0f); foam_live_mark.assign(n, 0);
        water.assign(n, 0); slurry.assign(n, 0); uw.assign(n, 0); vw.assign(n, 0);
        us.assign(n, 0); vs.assign(n, 0); bed.assign(n, 0); moisture.assign(n, 0);
        grain.assign(n, 4);
        fine_hold.assign(n, 0);
        hold_owner.assign(n, -1);
        snap_origin(c.center_x, c.center_z, (float)res * c.cell, c.cell, origin);
        float nuw = dynamic_viscosity(3, 1.0f);
        nu_w.assign(n, nuw); nu_s.assign(n, 0.0f); gate.assign(n, 1);
        fnu_w.assign(fn, nuw); fnu_s.assign(fn, 0.0f); fgate.assign(fn, 1);
    }
    void coarse_xz(usize i, usize j, float& x, float& z) const {
        x = origin[0] + ((float)i + 0.5f) * cfg.cell;
        z = origin[1] + ((float)j + 0.5f) * cfg.cell;
    }
    long coarse_axis(float o, float p) const {  // src/fluid_core.rs:9546-9557
        float i = floorf((p - o) / cfg.cell);
        if (i < 0.0f) return -1;
        usize ii = f2usize(i);
        return ii >= res ? -1 : (long)ii;
    }
    bool coarse_ij(float x, float z, usize& i, usize& j) const {
        long a = coarse_axis(origin[0], x), b = coarse_axis(origin[1], z);
        if (a < 0 || b < 0) return false;
        i = (usize)a; j = (usize)b;
        return true;
    }
    void make_patch_axes(Patch& P) const {  // src/fluid_core.rs:9518-9535
        P.col.assign(fres, 0xffff);
        P.row.assign(fres, 0xffff);
        for (usize i = 0; i < fres; ++i) {
            float x = P.origin[0] + ((float)i + 0.5f) * cfg.fine_cell;
            long ci = coarse_axis(origin[0], x);
            if (ci >= 0) P.col[i] = (uint16_t)ci;
        }
        for (usize j = 0; j < fres; ++j) {
            float z = P.origin[1] + ((float)j + 0.5f) * cfg.fine_cell;
            long cj = coarse_axis(origin[1], z);
            if (cj >= 0) P.row[j] = (uint16_t)cj;
        }
    }
    void ensure_patches(usize k) {
        usize fn = fres * fres;
        while (patches.size() < k) {
            Patch P;
            P.water.assign(fn, 0); P.slurry.assign(fn, 0); P.uw.assign(fn, 0); P.vw.assign(fn, 0);
            P.us.assign(fn, 0); P.vs.assign(fn, 0); P.bed.assign(fn, 0); P.bed_slurry.assign(fn, 0);
            P.moisture.assign(fn, 0); P.grain.assign(fn, 4);
            patches.push_back(std::move(P));
        }
    }
    usize active_patches() const { return cfg.layout == 0 ? (fine_on ? 1 : 0) : (fine_on ? pushes_in_use : 0); }
    usize pushes_in_use = 0;

    // near.rs:152-185 near_columns, per patch
    struct NearCol { usize cidx; std::pair<int, int> key; usize i0, j0; };
    std::vector<NearCol> near_columns(const Patch& P, int pidx) const {
        auto runs = [&](const std::vector<uint16_t>& axis) {
            std::vector<std::pair<uint16_t, usize>> out;
            usize i = 0;
            while (i < fres) {
                uint16_t c = axis[i];
                usize n = 1;
                while (i + n < fres && axis[i + n] == c) ++n;
                if (c != 0xffff && n == sub) out.push_back({c, i});
                i += n;
            }
            return out;
        };
        auto cols = runs(P.col), rows = runs(P.row);
        std::vector<NearCol> out;
        for (auto& r : rows)
            for (auto& c : cols) {
                usize cidx = (usize)r.first * res + c.first;
                if (fine_hold[cidx] != 1 || hold_owner[cidx] != pidx) continue;
                float x, z;
                coarse_xz(c.first, r.first, x, z);
                out.push_back({cidx, world_key(x, z, cfg.cell), c.second, r.second});
            }
        return out;
    }
    bool near_inner(usize cidx) const {  // near.rs:188-197
        usize i = cidx % res, j = cidx / res;
        if (i == 0 || j == 0 || i + 1 >= res || j + 1 >= res) return false;
        usize nb[4] = {cidx - 1, cidx + 1, cidx - res, cidx + res};
        for (usize q : nb)
            if (fine_hold[q] != 1) return false;
        return true;
    }
    // near.rs:199-273
    void near_capture() {
        if (!fine_on || !near_on) return;
        usize n2 = sub * sub;
        for (usize pk = 0; pk < active_patches(); ++pk) {
            Patch& P = patches[pk];
            for (const NearCol& nc : near_columns(P, cfg.layout == 0 ? -1 : (int)pk)) {
                float sw = 0.0f, ss = 0.0f;
                for (usize b = 0; b < sub; ++b) {
                    usize f = (nc.j0 + b) * fres + nc.i0;
                    sw += rsum(&P.water[f], sub);
                    ss += rsum(&P.slurry[f], sub);
                }
                if (sw <= 0.0f && ss <= 0.0f) { near.erase(nc.key); continue; }
                float nn = (float)n2;
                float mw = sw / nn, ms = ss / nn;
                std::vector<float> rw(n2), rs(n2);
                for (usize b = 0; b < sub; ++b) {
                    usize f = (nc.j0 + b) * fres + nc.i0;
                    for (usize a = 0; a < sub; ++a) {
                        rw[b * sub + a] = P.water[f + a] - mw;
                        rs[b * sub + a] = P.slurry[f + a] - ms;
                    }
                }
                float peak = rmax(abs_peak(rw), abs_peak(rs));
                bool inner = near_inner(nc.cidx);
                if (peak <= NEAR_DROP_M && !inner) { near.erase(nc.key); continue; }
                recentre(rw);
                recentre(rs);
                auto it = near.find(nc.key);
                if (it == near.end()) it = near.emplace(nc.key, NearTile(n2)).first;
                NearTile& tile = it->second;
                tile.w = rw;
                tile.s = rs;
                if (inner && sw > 1.0e-10f) {
                    float mu = 0.0f, mv = 0.0f;
                    for (usize b = 0; b < sub; ++b) {
                        usize f = (nc.j0 + b) * fres + nc.i0;
                        for (usize a = 0; a < sub; ++a) {
                            float w = P.water[f + a];
                            mu += w * P.uw[f + a];
                            mv += w * P.vw[f + a];
                        }
                    }
                    float uu = mu / sw, vv = mv / sw;
                    for (usize b = 0; b < sub; ++b) {
                        usize f = (nc.j0 + b) * fres + nc.i0;
                        for (usize a = 0; a < sub; ++a) {
                            bool wet = P.water[f + a] > NEAR_FILM_M;
                            tile.uw[b * sub + a] = wet ? P.uw[f + a] - uu : 0.0f;
                            tile.vw[b * sub + a] = wet ? P.vw[f + a] - vv : 0.0f;
                        }
                    }
                } else {
                    std::fill(tile.uw.begin(), tile.uw.end(), 0.0f);
                    std::fill(tile.vw.begin(), tile.vw.end(), 0.0f);
                }
                tile.peak = peak;
                tile.idle_s = 0.0f;
                tile.fresh = true;
            }
        }
    }
    // near.rs:311-325
    void near_fade(float dt) {
        if (near.empty()) return;
        dt = (dt > 0.0f && finite(dt)) ? dt : 0.0f;
        for (auto it = near.begin(); it != near.end();) {
            NearTile& t = it->second;
            if (t.fresh) { t.fresh = false; ++it; continue; }
            t.idle_s += dt;
            if (t.peak * t.left() > NEAR_DROP_M) ++it;
            else it = near.erase(it);
        }
    }
    // near.rs:276-308
    void near_apply(float dt) {
        if (!near.empty()) {
            for (usize pk = 0; pk < active_patches(); ++pk) {
                Patch& P = patches[pk];
                for (const NearCol& nc : near_columns(P, cfg.layout == 0 ? -1 : (int)pk)) {
                    auto it = near.find(nc.key);
                    if (it == near.end()) continue;
                    const NearTile& tile = it->second;
                    usize f0 = nc.j0 * fres + nc.i0;
                    float bw = P.water[f0], bs = P.slurry[f0];
                    bool inner = near_inner(nc.cidx);
                    float left = tile.left();
                    float aw = left * floor_scale(bw / rmax(left, 1.0e-6f), tile.w);
                    float as_ = left * floor_scale(bs / rmax(left, 1.0e-6f), tile.s);
                    for (usize b = 0; b < sub; ++b)
                        for (usize a = 0; a < sub; ++a) {
                            usize f = (nc.j0 + b) * fres + nc.i0 + a;
                            usize k = b * sub + a;
                            float w = rmax(bw + aw * tile.w[k], 0.0f);
                            float s = rmax(bs + as_ * tile.s[k], 0.0f);
                            P.water[f] = w;
                            P.slurry[f] = s;
                            if (inner && w > NEAR_FILM_M) {
                                P.uw[f] += left * tile.uw[k];
                                P.vw[f] += left * tile.vw[k];
                            }
                        }
                }
            }
        }
        near_fade(dt);
    }

    // src/fluid_core.rs:8462-8555 restrict_fine (all patches)
    void restrict_fine() {
        if (!fine_on) return;
        near_capture();
        float fine_area = cfg.fine_cell * cfg.fine_cell;
        float coarse_area = cfg.cell * cfg.cell;
        std::map<usize, usize> touch_pos;
        std::vector<usize> touch;
        std::vector<float> aw, as, auw, avw, aus, avs;
        std::vector<uint32_t> cnt;
        auto mark = [&](usize cidx) {
            auto it = touch_pos.find(cidx);
            if (it == touch_pos.end()) {
                touch_pos[cidx] = touch.size();
                touch.push_back(cidx);
                aw.push_back(0); as.push_back(0); auw.push_back(0); avw.push_back(0); aus.push_back(0); avs.push_back(0);
                cnt.push_back(0);
                return touch.size() - 1;
            }
            return it->second;
        };
        for (usize pk = 0; pk < active_patches(); ++pk) {
            Patch& P = patches[pk];
            for (usize j = 0; j < fres; ++j) {
                uint16_t cj = P.row[j];
                for (usize i = 0; i < fres; ++i) {
                    uint16_t ci = P.col[i];
                    usize fidx = j * fres + i;
                    if (cj == 0xffff || ci == 0xffff) {
                        float x = P.origin[0] + ((float)i + 0.5f) * cfg.fine_cell;
                        float z = P.origin[1] + ((float)j + 0.5f) * cfg.fine_cell;
                        auto& slot = parked[world_key(x, z, cfg.cell)];
                        slot.water += P.water[fidx] * fine_area / coarse_area;
                        slot.slurry += P.slurry[fidx] * fine_area / coarse_area;
                        continue;
                    }
                    usize cidx = (usize)cj * res + ci;
                    usize t = mark(cidx);
                    cnt[t] += 1;
                    float fw = P.water[fidx], fs = P.slurry[fidx];
                    if (fw == 0.0f && fs == 0.0f) continue;
                    aw[t] += P.water[fidx] * fine_area;
                    as[t] += P.slurry[fidx] * fine_area;
                    auw[t] += P.uw[fidx] * P.water[fidx] * fine_area;
                    avw[t] += P.vw[fidx] * P.water[fidx] * fine_area;
                    aus[t] += P.us[fidx] * P.slurry[fidx] * fine_area;
                    avs[t] += P.vs[fidx] * P.slurry[fidx] * fine_area;
                }
            }
        }
        for (usize t = 0; t < touch.size(); ++t) {
            usize idx = touch[t];
            bool held = fine_hold[idx] == 1;
            float w = aw[t] / coarse_area, s = as[t] / coarse_area;
            // Unheld columns keep their depth and gain what flowed onto their fine
            // cells. With patches that are whole multiples of the coarse cell (the
            // reference's 160-cell patch) every touched column is fully covered, so
            // this is the reference's `!held && cnt >= full` branch; a partly
            // covered rim column of a 64-cell patch must not lose its coarse depth.
            if (!held) {
                if (w <= 0.0f && s <= 0.0f) continue;
                float old_w = water[idx], old_s = slurry[idx];
                float new_w = old_w + w, new_s = old_s + s;
                if (new_w > 1.0e-6f) {
                    uw[idx] = (old_w * uw[idx] * coarse_area + auw[t]) / (new_w * coarse_area);
                    vw[idx] = (old_w * vw[idx] * coarse_area + avw[t]) / (new_w * coarse_area);
                }
                if (new_s > 1.0e-6f) {
                    us[idx] = (old_s * us[idx] * coarse_area + aus[t]) / (new_s * coarse_area);
                    vs[idx] = (old_s * vs[idx] * coarse_area + avs[t]) / (new_s * coarse_area);
                }
                water[idx] = new_w;
                slurry[idx] = new_s;
                continue;
            }
            water[idx] = w;
            slurry[idx] = s;
            if (w > 1.0e-6f) {
                uw[idx] = auw[t] / (w * coarse_area);
                vw[idx] = avw[t] / (w * coarse_area);
            }
            if (s > 1.0e-6f) {
                us[idx] = aus[t] / (s * coarse_area);
                vs[idx] = avs[t] / (s * coarse_area);
            }
        }
        for (usize pk = 0; pk < active_patches(); ++pk) {
            std::fill(patches[pk].water.begin(), patches[pk].water.end(), 0.0f);
            std::fill(patches[pk].slurry.begin(), patches[pk].slurry.end(), 0.0f);
        }
        fine_on = false;
    }

    // src/fluid_core.rs:8358-8460 refine. Layout 0 follows the reference (one
    // patch at the mean tire); layout 1 lays one patch per tire and holds a
    // column for the first patch that covers it and lies near its own tire.
    // All holds are decided first, then every patch is laid from the coarse
    // state before any held column is emptied (for one patch this is the
    // reference's order).
    void refine(const std::vector<TirePush>& ps, float dt) {
        restrict_fine();
        if (ps.empty()) { near_fade(dt); return; }
        usize np = cfg.layout == 0 ? 1 : std::min(ps.size(), (usize)16);
        ensure_patches(np);
        pushes_in_use = np;
        float extent = (float)fres * cfg.fine_cell;
        std::fill(fine_hold.begin(), fine_hold.end(), 0);
        std::fill(hold_owner.begin(), hold_owner.end(), -1);
        usize full = sub * sub;
        float r2 = cfg.tire_r * cfg.tire_r;
        std::vector<std::vector<usize>> touches(np);
        std::vector<std::vector<std::pair<usize, usize>>> hits(np);
        for (usize pk = 0; pk < np; ++pk) {
            Patch& P = patches[pk];
            if (cfg.layout == 0) {
                float cx = 0.0f, cz = 0.0f;
                for (auto& p : ps) { cx += p.x; cz += p.z; }
                float n = (float)ps.size();
                cx /= n; cz /= n;
                snap_origin(cx, cz, extent, cfg.cell, P.origin);
            } else {
                snap_origin(ps[pk].x, ps[pk].z, extent, cfg.cell, P.origin);
            }
            std::fill(P.water.begin(), P.water.end(), 0.0f);
            std::fill(P.slurry.begin(), P.slurry.end(), 0.0f);
            std::fill(P.uw.begin(), P.uw.end(), 0.0f);
            std::fill(P.vw.begin(), P.vw.end(), 0.0f);
            std::fill(P.us.begin(), P.us.end(), 0.0f);
            std::fill(P.vs.begin(), P.vs.end(), 0.0f);
            make_patch_axes(P);
            std::map<usize, uint32_t> cnt;
            for (usize j = 0; j < fres; ++j) {
                uint16_t cj = P.row[j];
                if (cj == 0xffff) continue;
                for (usize i = 0; i < fres; ++i) {
                    uint16_t ci = P.col[i];
                    if (ci == 0xffff) continue;
                    usize cidx = (usize)cj * res + ci;
                    if (cnt[cidx] == 0) touches[pk].push_back(cidx);
                    cnt[cidx] += 1;
                    hits[pk].push_back({j * fres + i, cidx});
                }
            }
            std::vector<TirePush> own;
            if (cfg.layout == 0) own = ps; else own.push_back(ps[pk]);
            for (usize cidx : touches[pk]) {
                if (cnt[cidx] != full) continue;
                if (fine_hold[cidx] == 1) continue;
                float x, z;
                coarse_xz(cidx % res, cidx / res, x, z);
                if (near_tire_zone(own, x, z, r2)) {
                    fine_hold[cidx] = 1;
                    hold_owner[cidx] = cfg.layout == 0 ? -1 : (int)pk;
                }
            }
        }
        for (usize pk = 0; pk < np; ++pk) {
            Patch& P = patches[pk];
            int me = cfg.layout == 0 ? -1 : (int)pk;
            for (auto& hp : hits[pk]) {
                usize fidx = hp.first, cidx = hp.second;
                P.moisture[fidx] = moisture[cidx];
                P.grain[fidx] = grain[cidx];
                if (!(fine_hold[cidx] == 1 && hold_owner[cidx] == me)) {
                    P.bed[fidx] = bed[cidx] + water[cidx];
                    P.bed_slurry[fidx] = bed[cidx] + slurry[cidx];
                    continue;
                }
                P.bed[fidx] = bed[cidx];
                P.bed_slurry[fidx] = bed[cidx];
                P.water[fidx] = water[cidx];
                P.slurry[fidx] = slurry[cidx];
                P.uw[fidx] = uw[cidx];
                P.vw[fidx] = vw[cidx];
                P.us[fidx] = us[cidx];
                P.vs[fidx] = vs[cidx];
            }
        }
        for (usize pk = 0; pk < np; ++pk)
            for (usize cidx : touches[pk])
                if (fine_hold[cidx] == 1)
                    water[cidx] = slurry[cidx] = uw[cidx] = vw[cidx] = us[cidx] = vs[cidx] = 0.0f;
        fine_on = true;
        near_apply(dt);
    }

    bool fine_held_at(float x, float z) const {
        usize i, j;
        if (!coarse_ij(x, z, i, j)) return false;
        return fine_hold[j * res + i] == 1;
    }
    // src/fluid_core.rs:8318-8356 cell_is_refined; returns the patch that holds it or -1.
    int refined_patch(float x, float z) const {
        if (!fine_on || !fine_held_at(x, z)) return -1;
        usize i, j;
        if (!coarse_ij(x, z, i, j)) return -1;
        float x0 = origin[0] + (float)i * cfg.cell, z0 = origin[1] + (float)j * cfg.cell;
        float x1 = x0 + cfg.cell, z1 = z0 + cfg.cell;
        int pk = cfg.layout == 0 ? 0 : hold_owner[j * res + i];
        if (pk < 0) return -1;
        const Patch& P = patches[pk];
        float extent = (float)fres * cfg.fine_cell;
        float rect[4] = {P.origin[0], P.origin[0] + extent, P.origin[1], P.origin[1] + extent};
        if (x0 >= rect[0] - 1.0e-4f && z0 >= rect[2] - 1.0e-4f && x1 <= rect[1] + 1.0e-4f && z1 <= rect[3] + 1.0e-4f)
            return pk;
        return -1;
    }

    // src/fluid_core.rs:8169-8239 push_on
    void push_on(const TirePush& p, float* w, float* s, float* fuw, float* fvw, float* fus, float* fvs,
                 usize r, float cell, const float* org) {
        float fx = p.forward_x, fz = p.forward_z;
        float len = rmax(sqrtf(fx * fx + fz * fz), 1.0e-4f);
        fx = fx / len;
        fz = fz / len;
        float rx = fz, rz = -fx;
        float speed = rmax(p.speed, 0.0f);
        float reach = hypotf(p.radius * 1.4f, p.width * 0.65f + cell) + cell;
        auto si = index_span(org[0], cell, r, p.x, reach);
        auto sj = index_span(org[1], cell, r, p.z, reach);
        for (usize j = sj.first; j < sj.second; ++j)
            for (usize i = si.first; i < si.second; ++i) {
                float x = org[0] + ((float)i + 0.5f) * cell;
                float z = org[1] + ((float)j + 0.5f) * cell;
                float dx = x - p.x, dz = z - p.z;
                float along = dx * fx + dz * fz;
                float lat = dx * rx + dz * rz;
                if (fabsf(lat) > p.width * 0.65f + cell) continue;
                if (along < -p.radius * 1.4f || along > p.radius * 1.1f) continue;
                usize idx = j * r + i;
                float flank = rclamp(fabsf(lat) / (p.width * 0.65f + cell), 0.0f, 1.0f);
                float shove = rmax(speed, 0.4f) * (1.0f - flank * flank);
                if (w[idx] > 0.004f) {
                    fuw[idx] += fx * shove * 0.85f;
                    fvw[idx] += fz * shove * 0.85f;
                    fuw[idx] += rx * rsignum(lat) * shove * 0.18f * flank;
                    fvw[idx] += rz * rsignum(lat) * shove * 0.18f * flank;
                }
                if (s[idx] > 0.004f) {
                    float fore = along > 0.0f ? 1.0f : 0.72f;
                    fus[idx] += fx * shove * fore;
                    fvs[idx] += fz * shove * fore;
                    fus[idx] += rx * rsignum(lat) * shove * 0.28f * flank;
                    fvs[idx] += rz * rsignum(lat) * shove * 0.28f * flank;
                }
            }
    }

    // src/fluid_core.rs:8241-8314 peel_spray
    void peel(const std::vector<TirePush>& ps, float* w, const float* fuw, const float* fvw, usize r,
              float cell, const float* org, bool skip_held, std::vector<Spray>& out) {
        float area = cell * cell;
        for (const auto& p : ps) {
            if (p.speed < 0.8f) continue;
            float reach = p.radius * 1.3f + cell;
            auto si = index_span(org[0], cell, r, p.x, reach);
            auto sj = index_span(org[1], cell, r, p.z, reach);
            for (usize j = sj.first; j < sj.second; ++j)
                for (usize i = si.first; i < si.second; ++i) {
                    float x = org[0] + ((float)i + 0.5f) * cell;
                    float z = org[1] + ((float)j + 0.5f) * cell;
                    if (skip_held) {
                        float ci = floorf((x - origin[0]) / cfg.cell), cj = floorf((z - origin[1]) / cfg.cell);
                        if (!(ci < 0.0f || cj < 0.0f)) {
                            usize ii = f2usize(ci), jj = f2usize(cj);
                            if (ii < res && jj < res && fine_hold[jj * res + ii] == 1) continue;
                        }
                    }
                    float dx = x - p.x, dz = z - p.z;
                    if (dx * dx + dz * dz > (p.radius * 1.3f) * (p.radius * 1.3f)) continue;
                    usize idx = j * r + i;
                    if (w[idx] < 0.01f) continue;
                    float take = rmin(w[idx] * 0.04f, 0.004f);
                    if (take * area < 1.0e-6f) continue;
                    w[idx] -= take;
                    out.push_back({x, 0.35f, z, fuw[idx] * 0.3f, 1.4f + p.speed * 0.25f, fvw[idx] * 0.3f, take * area, 0});
                }
        }
    }

    // src/fluid_core.rs:7942-8150 step_pair (open sheets, no bodies).
    void step_pair(float dt, bool fine) {
        if (fine && !fine_on) return;
        // An open reach runs the water row at its own mobility (a negative
        // entry, src/fluid_core.rs:8015-8017) and puts the water value back
        // after the pair (:8142-8145).
        struct RestoreWater {
            Core& c;
            ~RestoreWater() {
                if (!c.open_water) return;
                float nuw = dynamic_viscosity(3, 1.0f);
                std::fill(c.nu_w.begin(), c.nu_w.end(), nuw);
                std::fill(c.fnu_w.begin(), c.fnu_w.end(), nuw);
            }
        } restore{*this};
        if (open_water) {
            float m = -rmax(ow_mobility, 1.0e-4f);
            std::fill(nu_w.begin(), nu_w.end(), m);
            std::fill(fnu_w.begin(), fnu_w.end(), m);
        }
        float cap = fine ? fine_sub_cap : 8.0f;
        int pace = fine ? fine_pace : 0;
        if (!fine) {
            // An open reach keeps its current through the window ends (src/fluid_core.rs:8018-8033).
            int open_axis = -1;
            usize oc0 = 0, oc1 = 0;
            if (reach_on) {
                float o = reach_along_z ? origin[0] : origin[1];
                oc0 = f2usize(rmax(floorf((reach_cross0 - o) / cfg.cell), 0.0f));
                oc1 = std::min(f2usize(rmax(ceilf((reach_cross1 - o) / cfg.cell), 0.0f)), res);
                open_axis = reach_along_z ? 1 : 0;
            }
            // src/fluid_core.rs:7954-7967: one wall mask for both sheets, from
            // the water before either steps; each sheet first pushes its
            // columns out of the covered cells (:8057-8059, :8098-8100).
            std::vector<u8> cmask;
            if (!solids.empty()) cmask = solid_mask(solids, res, cfg.cell, origin, water.data(), bed.data());
            const u8* cm = cmask.empty() ? nullptr : cmask.data();
            auto run_water = [&]() {
                if (cfg.soften) soften_border(uw.data(), vw.data(), res, open_axis, oc0, oc1);
                if (cm) displace_occupied(water.data(), uw.data(), vw.data(), cm, res);
                step_sheet_eps(water.data(), uw.data(), vw.data(), bed.data(), nu_w.data(), gate.data(), res, cfg.cell, dt, 0.08f, 1.0e-6f, false, cap, pace, coarse_sc[0][0], &coarse_sc[0][1], cfg.inner_par != 0, cm);
            };
            auto run_slurry = [&]() {
                Box wb;
                if (wet_bounds(slurry.data(), res, NU_FILL_MARGIN, wb))
                    for (usize j = wb.j0; j <= wb.j1; ++j)
                        for (usize i = wb.i0; i <= wb.i1; ++i) {
                            usize idx = j * res + i;
                            nu_s[idx] = dynamic_viscosity(grain[idx], moisture[idx]);
                        }
                if (cfg.soften) soften_border(us.data(), vs.data(), res, open_axis, oc0, oc1);
                if (cm) displace_occupied(slurry.data(), us.data(), vs.data(), cm, res);
                step_sheet_eps(slurry.data(), us.data(), vs.data(), bed.data(), nu_s.data(), gate.data(), res, cfg.cell, dt, 0.05f, 1.0e-6f, false, cap, pace, coarse_sc[1][0], &coarse_sc[1][1], cfg.inner_par != 0, cm);
            };
            // src/fluid_core.rs:8127-8131: the two sheets on two workers.
            if (cfg.threads > 1) {
                std::thread t(run_slurry);
                run_water();
                t.join();
            } else {
                run_water();
                run_slurry();
            }
            return;
        }
        // Each patch's slurry reads its own viscosity row (patches run on
        // their own workers when threads > 1; results do not depend on it).
        if (fnu_s_rows.size() < active_patches()) fnu_s_rows.resize(active_patches(), std::vector<float>(fres * fres, 0.0f));
        // Each patch's wall mask, from its water over its bed (solid_mask(true)).
        std::vector<std::vector<u8>> fmask(active_patches());
        if (!solids.empty())
            for (usize pk = 0; pk < active_patches(); ++pk)
                fmask[pk] = solid_mask(solids, fres, cfg.fine_cell, patches[pk].origin, patches[pk].water.data(),
                                       patches[pk].bed.data());
        auto run_patch = [&](usize pk, int layer) {
            Patch& P = patches[pk];
            const u8* fm = fmask[pk].empty() ? nullptr : fmask[pk].data();
            if (layer == 0) {
                if (fm) displace_occupied(P.water.data(), P.uw.data(), P.vw.data(), fm, fres);
                step_sheet_eps(P.water.data(), P.uw.data(), P.vw.data(), P.bed.data(), fnu_w.data(), fgate.data(), fres, cfg.fine_cell, dt, 0.08f, 1.0e-6f, false, cap, pace, P.sc[0][0], &P.sc[0][1], false, fm);
                return;
            }
            std::vector<float>& nu = fnu_s_rows[pk];
            Box wb;
            if (wet_bounds(P.slurry.data(), fres, NU_FILL_MARGIN, wb))
                for (usize j = wb.j0; j <= wb.j1; ++j)
                    for (usize i = wb.i0; i <= wb.i1; ++i) {
                        usize idx = j * fres + i;
                        nu[idx] = dynamic_viscosity(P.grain[idx], P.moisture[idx]);
                    }
            if (fm) displace_occupied(P.slurry.data(), P.us.data(), P.vs.data(), fm, fres);
            step_sheet_eps(P.slurry.data(), P.us.data(), P.vs.data(), P.bed_slurry.data(), nu.data(), fgate.data(), fres, cfg.fine_cell, dt, 0.05f, 1.0e-6f, false, cap, pace, P.sc[1][0], &P.sc[1][1], false, fm);
        };
        if (cfg.threads > 1) {
            std::vector<std::thread> pool;
            for (usize pk = 0; pk < active_patches(); ++pk)
                for (int l = 0; l < 2; ++l) pool.emplace_back(run_patch, pk, l);
            for (auto& t : pool) t.join();
        } else {
            for (usize pk = 0; pk < active_patches(); ++pk) {
                run_patch(pk, 0);
                run_patch(pk, 1);
            }
        }
    }

    // src/fluid_core.rs:6034-6128, sheet subset.
    std::vector<Spray> step(float dt) {
        std::vector<TirePush> ps;
        ps.swap(pushes);
        // Lift from the column the tire rolls into, before the sheet shoves it (:6051-6053).
        if (turbidity_enabled && dt > 0.0f && finite(dt) && !ps.empty()) entrain_wake(ps, dt);
        if (inflow_j >= 0 && dt > 0.0f) apply_inflow(dt);
        refine(ps, dt);
        // apply_pushes(fine): src/fluid_core.rs:8152-8158
        for (const auto& p : ps) {
            int pk = refined_patch(p.x, p.z);
            if (pk < 0) continue;
            Patch& P = patches[pk];
            push_on(p, P.water.data(), P.slurry.data(), P.uw.data(), P.vw.data(), P.us.data(), P.vs.data(), fres, cfg.fine_cell, P.origin);
        }
        step_pair(dt, true);
        std::vector<Spray> spray;
        if (fine_on)
            for (usize pk = 0; pk < active_patches(); ++pk) {
                Patch& P = patches[pk];
                peel(ps, P.water.data(), P.uw.data(), P.vw.data(), fres, cfg.fine_cell, P.origin, false, spray);
            }
        restrict_fine();
        for (const auto& p : ps) {  // apply_pushes_outside :8160-8167
            if (fine_held_at(p.x, p.z)) continue;
            push_on(p, water.data(), slurry.data(), uw.data(), vw.data(), us.data(), vs.data(), res, cfg.cell, origin);
        }
        drive_waves(dt);
        step_pair(dt, false);
        bed_friction(dt);
        diffuse_surface(dt);
        if (!ps.empty()) peel(ps, water.data(), uw.data(), vw.data(), res, cfg.cell, origin, true, spray);
        if (!solids.empty()) scour_contacts(dt);
        step_tracers(dt, ps);         // :6080
        feed_reach();
        if (turbidity_enabled) step_suspended(dt);  // :6087-6089
        for (const auto& s : spray) spray_m3 += s.volume;
        return spray;
    }

    // src/fluid_core.rs:7364-7420 scour_contacts: shear above 1.5 Pa on a wet
    // open cell beside a tire contact cuts the bed into the slurry sheet, at
    // most 8 cm per cell over the run.
    void scour_contacts(float dt) {
        if (dt <= 0.0f || solids.empty()) return;
        std::vector<u8> mask = solid_mask(solids, res, cfg.cell, origin, water.data(), bed.data());
        const float area = cfg.cell * cfg.cell;
        std::vector<float> cut(res * res, 0.0f);
        for (usize j = 1; j + 1 < res; ++j)
            for (usize i = 1; i + 1 < res; ++i) {
                const usize idx = j * res + i;
                if (mask[idx] != 0 || water[idx] < 0.02f) continue;
                bool touch = false;
                for (const auto& d : NB4)
                    if (mask[(usize)((long)j + d[1]) * res + (usize)((long)i + d[0])] == 1) {
                        touch = true;
                        break;
                    }
                if (!touch) continue;
                const float speed = hypotf(uw[idx], vw[idx]);
                if (!finite(speed)) continue;
                const float tau = 1000.0f * 0.03f * speed * speed;
                const float tau_c = 1.5f;
                if (tau <= tau_c) continue;
                const float rate = rmin(0.0035f * (tau / tau_c - 1.0f), 0.012f);
                const float room = rmax(0.08f - bed_drop[idx], 0.0f);
                cut[idx] = rmin(rate * dt, room);
            }
        for (usize idx = 0; idx < res * res; ++idx) {
            const float dh = cut[idx];
            if (dh <= 0.0f) continue;
            bed[idx] -= dh;
            slurry[idx] += dh;
            us[idx] = uw[idx];
            vs[idx] = vw[idx];
            grain[idx] = 1;  // Grain::Silt
            moisture[idx] = rmax(moisture[idx], 0.9f);
            bed_drop[idx] += dh;
            eroded_m3 += dh * area;
            scour_hole_m = rmax(scour_hole_m, bed_drop[idx]);
        }
    }

    // src/fluid_core.rs:7251-7286 ring_surface: mean bed and water of the wet
    // cells in a ring around the body.
    bool ring_surface(const HydroSolid& s, float& bed_out, float& water_out) const {
        const float reach = rmax(s.half_length, s.half_width) + 0.55f;
        const long i0 = (long)floorf((s.x - reach - origin[0]) / cfg.cell);
        const long i1 = (long)floorf((s.x + reach - origin[0]) / cfg.cell);
        const long j0 = (long)floorf((s.z - reach - origin[1]) / cfg.cell);
        const long j1 = (long)floorf((s.z + reach - origin[1]) / cfg.cell);
        float bsum = 0.0f, wsum = 0.0f, n = 0.0f;
        for (long j = j0; j <= j1; ++j)
            for (long i = i0; i <= i1; ++i) {
                if (!in_grid(i, j, res)) continue;
                const float x = origin[0] + ((float)i + 0.5f) * cfg.cell;
                const float z = origin[1] + ((float)j + 0.5f) * cfg.cell;
                if (solid_contains(s, x, z)) continue;
                if (hypotf(x - s.x, z - s.z) > reach) continue;
                const usize idx = (usize)j * res + (usize)i;
                if (water[idx] < 0.01f) continue;
                bsum += bed[idx];
                wsum += water[idx];
                n += 1.0f;
            }
        if (n < 1.0f) return false;
        bed_out = bsum / n;
        water_out = wsum / n;
        return true;
    }

    // src/fluid_core.rs:4606-4615 cylinder_segment_volume
    static float cylinder_segment_volume(float depth, float radius, float width) {
        const float d = rclamp(depth, 0.0f, radius * 2.0f);
        if (d <= 1.0e-4f || width <= 0.0f || radius <= 1.0e-3f) return 0.0f;
        const float c = rclamp((radius - d) / radius, -1.0f, 1.0f);
        const float area = radius * radius * acosf(c) - (radius - d) * sqrtf(rmax(2.0f * radius * d - d * d, 0.0f));
        return rmax(area, 0.0f) * width;
    }

    // src/fluid_core.rs:7164-7249 hydro_load: out = force_x, force_z,
    // buoyancy, hull buoyancy, wheel buoyancy, displaced m^3, eroded m^3,
    // hole m, wheel blocks, belly blocks.
    void hydro_load(float* out) const {
        std::vector<u8> mask = solids.empty() ? std::vector<u8>(res * res, 0)
                                              : solid_mask(solids, res, cfg.cell, origin, water.data(), bed.data());
        float fx = 0.0f, fz = 0.0f;
        uint32_t wheel_blocks = 0, belly_blocks = 0;
        for (u8 m : mask) {
            if (m == 1) ++wheel_blocks;
            else if (m == 2) ++belly_blocks;
        }
        const float cell = cfg.cell;
        for (usize j = 0; j < res; ++j)
            for (usize i = 0; i < res; ++i) {
                const usize idx = j * res + i;
                if (mask[idx] != 0) continue;
                const float h = water[idx];
                if (h < 1.0e-4f || !finite(h)) continue;
                for (const auto& d : NB4) {
                    const long ni = (long)i + d[0], nj = (long)j + d[1];
                    if (!in_grid(ni, nj, res)) continue;
                    if (mask[(usize)nj * res + (usize)ni] == 0) continue;
                    const float nx = (float)d[0], nz = (float)d[1];
                    const float hydro = 1000.0f * GRAVITY * h * h * 0.5f * cell;
                    fx += nx * hydro;
                    fz += nz * hydro;
                    const float vn = uw[idx] * nx + vw[idx] * nz;
                    if (vn > 0.0f) {
                        const float dyn_f = 0.5f * 1000.0f * vn * vn * h * cell;
                        fx += nx * dyn_f;
                        fz += nz * dyn_f;
                    }
                }
            }
        float wheel_b = 0.0f, hull_b = 0.0f, displaced = 0.0f;
        for (const HydroSolid& s : solids) {
            float rb, rw;
            if (!ring_surface(s, rb, rw)) continue;
            if (s.radius > 0.0f) {
                const float vol = cylinder_segment_volume(rw, s.radius, s.width);
                displaced += vol;
                wheel_b += 1000.0f * GRAVITY * vol;
            } else {
                const float eta = rb + rw;
                const float height = rmax(s.top_y - s.bottom_y, 0.0f);
                const float sub = rclamp(eta - s.bottom_y, 0.0f, height);
                const float vol = (s.half_length * 2.0f) * (s.half_width * 2.0f) * sub * 0.36f;
                displaced += vol;
                hull_b += 1000.0f * GRAVITY * vol;
            }
        }
        const float vals[10] = {fx, fz, wheel_b + hull_b, hull_b, wheel_b, displaced, eroded_m3, scour_hole_m,
                                (float)wheel_blocks, (float)belly_blocks};
        memcpy(out, vals, sizeof vals);
    }

    // src/fluid_core.rs:7482-7512 bed_friction: the eddy shear, then Manning
    // friction, implicit, on the coarse water in open-water mode.
    void bed_friction(float dt) {
        if (!open_water) return;
        if (dt <= 0.0f) return;
        eddy_shear(ow_eddy, dt);
        if (ow_manning <= 0.0f) return;
        float gn2 = GRAVITY * ow_manning * ow_manning;
        for (usize idx = 0; idx < res * res; ++idx) {
            float h = water[idx];
            if (!(h > 1.0e-4f)) continue;
            float u = uw[idx], v = vw[idx];
            float speed = hypotf(u, v);
            if (!(speed > 0.0f)) continue;
            float k = gn2 * speed / powf(rmax(h, 0.002f), 4.0f / 3.0f);
            float keep = 1.0f / (1.0f + dt * k);
            uw[idx] = u * keep;
            vw[idx] = v * keep;
        }
    }

    // src/fluid_core.rs:7514-7581 eddy_shear: one explicit Laplacian of the
    // water velocity from a snapshot; dry ground standing 3 cm above the
    // surface is no slip, a beach is skipped.
    void eddy_shear(float nu_t, float dt) {
        if (nu_t <= 0.0f) return;
        const float WET = 0.003f, STANDS_OUT = 0.03f;
        usize n = res * res;
        float k = rmin(nu_t * dt / (cfg.cell * cfg.cell), 0.2f);
        std::vector<float> du(n, 0.0f), dv(n, 0.0f);
        for (usize j = 0; j < res; ++j)
            for (usize i = 0; i < res; ++i) {
                usize idx = j * res + i;
                if (!(water[idx] > WET)) continue;
                float u0 = uw[idx], v0 = vw[idx];
                float lu = 0.0f, lv = 0.0f;
                const int nb[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
                for (auto& d : nb) {
                    long ni = (long)i + d[0], nj = (long)j + d[1];
                    if (ni < 0 || nj < 0 || ni >= (long)res || nj >= (long)res) continue;
                    usize nidx = (usize)nj * res + (usize)ni;
                    float un, vn;
                    if (water[nidx] > WET) {
                        un = uw[nidx];
                        vn = vw[nidx];
                    } else if (bed[nidx] > bed[idx] + water[idx] + STANDS_OUT) {
                        un = 0.0f;
                        vn = 0.0f;
                    } else {
                        continue;
                    }
                    lu += un - u0;
                    lv += vn - v0;
                }
                du[idx] = k * lu;
                dv[idx] = k * lv;
            }
        for (usize idx = 0; idx < n; ++idx)
            if (du[idx] != 0.0f || dv[idx] != 0.0f) {
                float nu = uw[idx] + du[idx], nv = vw[idx] + dv[idx];
                if (finite(nu) && finite(nv)) {
                    uw[idx] = nu;
                    vw[idx] = nv;
                }
            }
    }

    // src/fluid_core.rs:7582-7636 diffuse_surface: surface-slope fluxes from
    // one snapshot, each east and north face once, a quarter-column donor limit.
    void diffuse_surface(float dt) {
        if (surface_diffusion <= 0.0f || dt <= 0.0f) return;
        float k = rmin(surface_diffusion * dt / (cfg.cell * cfg.cell), 0.12f);
        const float WET = 0.003f;
        usize n = res * res;
        std::vector<float> delta(n, 0.0f);
        for (usize j = 0; j < res; ++j)
            for (usize i = 0; i < res; ++i) {
                usize a = j * res + i;
                float ha = water[a];
                if (!(ha > WET)) continue;
                float ea = bed[a] + ha;
                for (int face = 0; face < 2; ++face) {
                    if (face == 0 && !(i + 1 < res)) continue;
                    if (face == 1 && !(j + 1 < res)) continue;
                    usize b = face == 0 ? a + 1 : a + res;
                    float hb = water[b];
                    if (!(hb > WET)) continue;
                    float eb = bed[b] + hb;
                    float f = k * (ea - eb);
                    if (f > 0.0f) f = rmin(f, 0.25f * ha);
                    else f = rmax(f, -0.25f * hb);
                    delta[a] -= f;
                    delta[b] += f;
                }
            }
        for (usize idx = 0; idx < n; ++idx) {
            float d = delta[idx];
            if (d != 0.0f && finite(d)) water[idx] = rmax(water[idx] + d, 0.0f);
        }
    }

    // src/fluid_core.rs:7420-7480 drive_waves: the paddle strip's water
    // velocity relaxes toward the stroke, tapered over the strip's outer
    // quarters.
    void drive_waves(float dt) {
        if (!wave_on) return;
        if (dt <= 0.0f || wave_period <= 0.0f) return;
        wave_t += dt;
        float len = hypotf(wave_dx, wave_dz);
        if (len < 1.0e-6f || !finite(len)) return;
        float dx = wave_dx / len, dz = wave_dz / len;
        float ramp = wave_ramp > 0.0f ? rmin(rmax(wave_t / wave_ramp, 0.0f), 1.0f) : 1.0f;
        float phase = 6.28318548f * wave_t / wave_period;
        float stroke = wave_amp * ramp * sinf(phase);
        float pull = 1.0f - expf(-dt / 0.08f);
        float cell = cfg.cell;
        float span_x = rmax(wave_x1 - wave_x0, cell), span_z = rmax(wave_z1 - wave_z0, cell);
        long i0 = std::max((long)floorf((wave_x0 - origin[0]) / cell), 0L);
        long i1 = std::min((long)ceilf((wave_x1 - origin[0]) / cell), (long)res);
        long j0 = std::max((long)floorf((wave_z0 - origin[1]) / cell), 0L);
        long j1 = std::min((long)ceilf((wave_z1 - origin[1]) / cell), (long)res);
        for (long j = j0; j < j1; ++j)
            for (long i = i0; i < i1; ++i) {
                float x, z;
                coarse_xz((usize)i, (usize)j, x, z);
                if (x < wave_x0 || x > wave_x1 || z < wave_z0 || z > wave_z1) continue;
                usize idx = (usize)j * res + (usize)i;
                if (water[idx] < 0.02f || !finite(water[idx])) continue;
                float tx = rmin(rmax(rmin(x - wave_x0, wave_x1 - x) / (0.25f * span_x), 0.0f), 1.0f);
                float tz = rmin(rmax(rmin(z - wave_z0, wave_z1 - z) / (0.25f * span_z), 0.0f), 1.0f);
                float k = pull * rmin(tx, tz);
                float u = uw[idx], v = vw[idx];
                float along = u * dx + v * dz;
                float d = (stroke - along) * k;
                float nu = u + d * dx, nv = v + d * dz;
                if (finite(nu) && finite(nv)) {
                    uw[idx] = nu;
                    vw[idx] = nv;
                }
            }
    }

    // src/fluid_core.rs:7638-7745 feed_reach: the outlet rows hold their stage
    // and copy the interior velocity, banking the excess; the inlet rows fill
    // from the bank toward their stage and push the water in.
    void feed_reach() {
        if (!reach_on) return;
        usize rows = std::min(std::max(reach_rows, (usize)1), res / 4);
        float cell = cfg.cell, area = cell * cell;
        float co = reach_along_z ? origin[0] : origin[1];
        usize c0 = f2usize(rmax(floorf((reach_cross0 - co) / cell), 0.0f));
        float c1f = ceilf((reach_cross1 - co) / cell);
        usize c1 = f2usize(rmin(rmax(c1f, 0.0f), (float)res));
        if (c1 <= c0) return;
        auto at = [&](usize along, usize cross) { return reach_along_z ? along * res + cross : cross * res + along; };
        auto row = [&](usize k) { return reach_positive ? k : res - 1 - k; };
        float dx = reach_along_z ? 0.0f : (reach_positive ? 1.0f : -1.0f);
        float dz = reach_along_z ? (reach_positive ? 1.0f : -1.0f) : 0.0f;
        usize first_out = res - rows;
        for (usize cross = c0; cross < c1; ++cross) {
            usize src = at(row(first_out - 1), cross);
            float su = uw[src], sv = vw[src];
            float along = rmax(su * dx + sv * dz, 0.0f);
            for (usize k = first_out; k < res; ++k) {
                usize idx = at(row(k), cross);
                float target = rmax(reach_outlet_eta - bed[idx], 0.0f);
                float h = water[idx];
                if (!finite(h) || target <= 0.0f) continue;
                if (h > target) {
                    reach_bank_m3 += (h - target) * area;
                    water[idx] = target;
                } else if (reach_bank_m3 > 0.0f) {
                    float add = rmin(target - h, reach_bank_m3 / area);
                    water[idx] = h + add;
                    reach_bank_m3 -= add * area;
                }
                if (finite(su) && finite(sv)) {
                    float cross_v = reach_along_z ? su : sv;
                    if (reach_along_z) {
                        uw[idx] = cross_v;
                        vw[idx] = along * dz;
                    } else {
                        uw[idx] = along * dx;
                        vw[idx] = cross_v;
                    }
                }
            }
        }
        float inflow_c = turbidity_enabled && finite(reach_inlet_turbidity) ? rclamp(reach_inlet_turbidity, 0.0f, 1.0f) : 0.0f;
        double inflow_m3 = 0.0;
        float deep = 0.0f;
        for (usize cross = c0; cross < c1; ++cross) deep = rmax(deep, rmax(reach_inlet_eta - bed[at(row(0), cross)], 0.0f));
        if (deep <= 0.0f) return;
        for (usize k = 0; k < rows; ++k)
            for (usize cross = c0; cross < c1; ++cross) {
                usize idx = at(row(k), cross);
                float target = rmax(reach_inlet_eta - bed[idx], 0.0f);
                float h = water[idx];
                if (!finite(h) || target <= 0.0f) continue;
                if (h > target) {
                    reach_bank_m3 += (h - target) * area;
                    water[idx] = target;
                } else if (reach_bank_m3 > 0.0f) {
                    float add = rmin(target - h, reach_bank_m3 / area);
                    water[idx] = h + add;
                    reach_bank_m3 -= add * area;
                }
                float speed = reach_speed * sqrtf(rmin(rmax(water[idx] / deep, 0.0f), 1.0f));
                uw[idx] = speed * dx;
                vw[idx] = speed * dz;
                if (inflow_c > 0.0f) {  // :7712-7757, the inlet's suspended load
                    float w = water[idx];
                    float want = inflow_c * w;
                    float have = susp[idx];
                    if (w >= 1.0e-5f && finite(have) && have < want) {
                        susp[idx] = want;
                        inflow_m3 += (double)((want - have) * area);
                    }
                }
            }
        entrained_m3 += (float)inflow_m3;
        entrained64 += inflow_m3;
    }

    // src/fluid_core.rs:4797-4805 park_slot (settled dust is off this path and 0).
    bool park_slot(const Parked& p) const {
        return p.water > 1.0e-8f || p.slurry > 1.0e-8f || p.susp > 1.0e-8f ||
               fabsf(p.moisture - moisture_ambient) > 6.0e-3f || p.foam > 1.0e-4f || p.turbid > 1.0e-8f;
    }
    Parked slot_of(usize idx) const {
        Parked p;
        p.water = water[idx]; p.slurry = slurry[idx]; p.uw = uw[idx]; p.vw = vw[idx];
        p.us = us[idx]; p.vs = vs[idx]; p.moisture = moisture[idx];
        p.foam = foam[idx]; p.turbid = turbid[idx]; p.susp = susp[idx];
        return p;
    }
    void put_slot(usize idx, const Parked& p) {
        water[idx] = p.water; slurry[idx] = p.slurry; uw[idx] = p.uw; vw[idx] = p.vw;
        us[idx] = p.us; vs[idx] = p.vs; moisture[idx] = p.moisture;
        foam[idx] = p.foam; turbid[idx] = p.turbid; susp[idx] = p.susp;
    }
    // src/fluid_core.rs:9228-9233 reset_tracer_indices.
    void reset_tracer_indices() {
        wet_idx.clear();
        shore_idx.clear();
        foam_live.clear();
        std::fill(foam_live_mark.begin(), foam_live_mark.end(), 0);
    }
    std::pair<int, int> cell_key(const float* o, usize i, usize j) const {
        return world_key(o[0] + ((float)i + 0.5f) * cfg.cell, o[1] + ((float)j + 0.5f) * cfg.cell, cfg.cell);
    }
    void park(usize idx, std::pair<int, int> key) {
        Parked p = slot_of(idx);
        if (park_slot(p)) parked[key] = p;
        else parked.erase(key);
    }

    // src/fluid_core.rs:9899-9933 uniform_cell_shift.
    bool uniform_cell_shift(const float* o, const float* nw, int& di, int& dj) const {
        if (res == 0 || !(finite(cfg.cell) && cfg.cell > 0.0f)) return false;
        auto o00 = cell_key(o, 0, 0), n00 = cell_key(nw, 0, 0);
        di = n00.first - o00.first;
        dj = n00.second - o00.second;
        usize last = res - 1;
        auto o11 = cell_key(o, last, last), n11 = cell_key(nw, last, last);
        if (o11.first - o00.first != (int)last || o11.second - o00.second != (int)last) return false;
        if (n11.first - n00.first != (int)last || n11.second - n00.second != (int)last) return false;
        if (n11.first - o11.first != di || n11.second - o11.second != dj) return false;
        usize mid = res / 2;
        auto om = cell_key(o, mid, mid), nm = cell_key(nw, mid, mid);
        return nm.first - om.first == di && nm.second - om.second == dj;
    }

    // src/fluid_core.rs:9936-9990 each_leaving.
    template <class F>
    void each_leaving(int di, int dj, F f) const {
        int n = (int)res;
        if (di > 0) {
            int w = std::min(di, n);
            for (int j = 0; j < n; ++j) for (int i = 0; i < w; ++i) f(i, j);
        } else if (di < 0) {
            int w = std::min(-di, n);
            for (int j = 0; j < n; ++j) for (int i = n - w; i < n; ++i) f(i, j);
        }
        auto covered = [&](int i) { return di > 0 ? i < di : (di < 0 ? i >= n + di : false); };
        if (dj > 0) {
            int h = std::min(dj, n);
            for (int j = 0; j < h; ++j) for (int i = 0; i < n; ++i) if (!covered(i)) f(i, j);
        } else if (dj < 0) {
            int h = std::min(-dj, n);
            for (int j = n - h; j < n; ++j) for (int i = 0; i < n; ++i) if (!covered(i)) f(i, j);
        }
    }

    // src/fluid_core.rs:5409-5421 recenter (the sheet part) and :9004-9020 shift_coarse.
    void recenter(float cx, float cz) {
        if (fine_on) restrict_fine();
        float nw[2];
        snap_origin(cx, cz, (float)res * cfg.cell, cfg.cell, nw);
        if (fabsf(nw[0] - origin[0]) < 1.0e-4f && fabsf(nw[1] - origin[1]) < 1.0e-4f) return;
        int di, dj;
        if (uniform_cell_shift(origin, nw, di, dj)) shift_scroll(nw, di, dj);
        else shift_hash(nw);
    }

    // src/fluid_core.rs:9024-9145 shift_coarse_scroll: park the strip that
    // leaves, copy the overlap by index (bed and grain stay on their index),
    // restore the strip that enters.
    void shift_scroll(const float* nw, int di, int dj) {
        usize n = res * res;
        each_leaving(di, dj, [&](int i, int j) { park((usize)j * res + i, cell_key(origin, i, j)); });
        std::vector<float> cw = water, cs = slurry, cuw = uw, cvw = vw, cus = us, cvs = vs, cm = moisture;
        std::vector<float> cf = foam, ct = turbid, cp = susp;
        const bool track_susp = turbidity_enabled;
        int rn = (int)res;
        for (int j = 0; j < rn; ++j)
            for (int i = 0; i < rn; ++i) {
                usize dst = (usize)j * res + i;
                int si = i + di, sj = j + dj;
                bool keep = false;
                usize src = 0;
                if (si >= 0 && si < rn && sj >= 0 && sj < rn) {
                    src = (usize)sj * res + si;
                    keep = cw[src] > 1.0e-8f || cs[src] > 1.0e-8f || cm[src] > 1.0e-4f || cf[src] > 1.0e-5f ||
                           ct[src] > 1.0e-8f || (track_susp && cp[src] > 1.0e-8f);
                }
                if (keep) {
                    water[dst] = cw[src]; slurry[dst] = cs[src]; uw[dst] = cuw[src]; vw[dst] = cvw[src];
                    us[dst] = cus[src]; vs[dst] = cvs[src]; moisture[dst] = cm[src];
                    foam[dst] = cf[src]; turbid[dst] = ct[src]; susp[dst] = track_susp ? cp[src] : 0.0f;
                } else {
                    water[dst] = 0; slurry[dst] = 0; uw[dst] = 0; vw[dst] = 0; us[dst] = 0; vs[dst] = 0;
                    moisture[dst] = moisture_ambient;
                    foam[dst] = 0; turbid[dst] = 0; susp[dst] = 0;
                }
            }
        (void)n;
        origin[0] = nw[0];
        origin[1] = nw[1];
        reset_tracer_indices();
        each_leaving(-di, -dj, [&](int i, int j) {
            auto it = parked.find(cell_key(origin, i, j));
            if (it == parked.end()) return;
            put_slot((usize)j * res + i, it->second);
            parked.erase(it);
        });
    }

    // src/fluid_core.rs:9147-9222 shift_coarse_hash: park everything, restore
    // what the new window covers.
    void shift_hash(const float* nw) {
        for (usize j = 0; j < res; ++j)
            for (usize i = 0; i < res; ++i) park(j * res + i, cell_key(origin, i, j));
        origin[0] = nw[0];
        origin[1] = nw[1];
        reset_tracer_indices();
        for (usize j = 0; j < res; ++j)
            for (usize i = 0; i < res; ++i) {
                usize idx = j * res + i;
                Parked p;
                p.moisture = moisture_ambient;
                auto it = parked.find(cell_key(origin, i, j));
                if (it != parked.end()) {
                    p = it->second;
                    parked.erase(it);
                }
                put_slot(idx, p);
            }
    }

    // ------------------------------------------------------------ tracers
    bool surface_driven() const { return wave_on || reach_on; }  // :6240-6244
    static bool wake_push(const TirePush& p) {
        return (finite(p.speed) && p.speed >= 0.25f) || (finite(p.slip) && fabsf(p.slip) >= 0.05f);
    }

    // src/fluid_core.rs:8758-8815 entrain_wake: the aft plume of each tire
    // lifts solids into the water column it rolls through.
    void entrain_wake(const std::vector<TirePush>& ps, float dt) {
        const int r = (int)res;
        const float cell = cfg.cell, area = cell * cell;
        for (const auto& p : ps) {
            if (p.speed < 0.3f) continue;
            float fl = rmax(sqrtf(p.forward_x * p.forward_x + p.forward_z * p.forward_z), 1.0e-4f);
            float fx = p.forward_x / fl, fz = p.forward_z / fl;
            float rx = fz, rz = -fx;
            float reach = p.radius * 3.4f + cell;
            int i0 = (int)floorf(((p.x - reach) - origin[0]) / cell);
            int i1 = (int)floorf(((p.x + reach) - origin[0]) / cell);
            int j0 = (int)floorf(((p.z - reach) - origin[1]) / cell);
            int j1 = (int)floorf(((p.z + reach) - origin[1]) / cell);
            float aft = p.radius * 3.2f;
            float half = p.width * 0.55f + 0.08f;
            for (int j = std::max(j0, 0); j <= std::min(j1, r - 1); ++j)
                for (int i = std::max(i0, 0); i <= std::min(i1, r - 1); ++i) {
                    float x = origin[0] + ((float)i + 0.5f) * cell;
                    float z = origin[1] + ((float)j + 0.5f) * cell;
                    float dx = x - p.x, dz = z - p.z;
                    float along = dx * fx + dz * fz;
                    if (along > -0.05f || along < -aft) continue;
                    float lat = fabsf(dx * rx + dz * rz);
                    if (lat > half) continue;
                    usize idx = (usize)j * res + (usize)i;
                    float w = water[idx];
                    if (!finite(w) || w < 0.004f) continue;
                    float along_t = rclamp((-along) / aft, 0.0f, 1.0f);
                    float lat_t = rclamp(lat / half, 0.0f, 1.0f);
                    float core = (1.0f - along_t) * (1.0f - lat_t);
                    float room = rmax(w - susp[idx], 0.0f);
                    float add = rmin(4.0f * dt * core * w, room);
                    if (add <= 1.0e-8f) continue;
                    susp[idx] += add;
                    entrained_m3 += add * area;
                    entrained64 += (double)(add * area);
                }
        }
    }

    // src/fluid_core.rs:6210-6237 step_tracers.
    void step_tracers(float dt, const std::vector<TirePush>& ps) {
        if (dt <= 0.0f || !finite(dt)) return;
        bool wake = surface_driven();
        for (const auto& p : ps) wake = wake || wake_push(p);
        bool live_silt = false;
        for (float t : turbid) live_silt = live_silt || (finite(t) && t > 1.0e-8f);
        bool live_foam = !foam_live.empty();
        if (!wake && !live_silt && !live_foam) return;
        collect_tracer_wet(ps);
        if (wet_idx.empty() && !live_silt) return;
        if (live_foam) advect_foam(dt);
        advect_turbid(dt);
        settle_turbid(dt);
        for (const auto& p : ps) spawn_tire_tracers(p, dt, cfg.cell * cfg.cell);
        spawn_shore_tracers(dt, cfg.cell * cfg.cell);
        spawn_breaking_speed(dt);
        clear_dry_tracers();
        sync_foam_live();
    }

    // src/fluid_core.rs:6248-6293 collect_tracer_wet.
    void collect_tracer_wet(const std::vector<TirePush>& ps) {
        wet_idx.clear();
        shore_idx.clear();
        bool wake = surface_driven();
        for (const auto& p : ps) wake = wake || wake_push(p);
        usize i0, i1, j0, j1;
        if (wake) {
            i0 = 0; i1 = res - 1; j0 = 0; j1 = res - 1;
        } else if (tracer_visit_box(ps, i0, i1, j0, j1)) {
            const usize M = 2;
            i0 = sat_sub(i0, M); j0 = sat_sub(j0, M);
            i1 = std::min(i1 + M, res - 1); j1 = std::min(j1 + M, res - 1);
        } else {
            return;
        }
        for (usize j = j0; j <= j1; ++j) {
            usize row = j * res;
            float peak = 0.0f;
            for (usize i = i0; i <= i1; ++i) peak = rmax(peak, water[row + i] + slurry[row + i]);
            if (peak < 0.004f) continue;
            for (usize i = i0; i <= i1; ++i) {
                usize idx = row + i;
                float h = water[idx] + slurry[idx];
                if (!finite(h) || h < 0.004f) continue;
                wet_idx.push_back((uint32_t)idx);
                if (shore_wet_cell(water.data(), res, i, j)) shore_idx.push_back((uint32_t)idx);
            }
        }
    }

    // src/fluid_core.rs:6296-6337 tracer_visit_box.
    bool tracer_visit_box(const std::vector<TirePush>& ps, usize& i0, usize& i1, usize& j0, usize& j1) const {
        i0 = res; i1 = 0; j0 = res; j1 = 0;
        bool any = false;
        for (uint32_t id : foam_live) {
            usize i = id % res, j = id / res;
            i0 = std::min(i0, i); i1 = std::max(i1, i); j0 = std::min(j0, j); j1 = std::max(j1, j);
            any = true;
        }
        usize ti0, ti1, tj0, tj1;
        if (turbid_span(turbid.data(), res, ti0, ti1, tj0, tj1)) {
            i0 = std::min(i0, ti0); i1 = std::max(i1, ti1); j0 = std::min(j0, tj0); j1 = std::max(j1, tj1);
            any = true;
        }
        int reach = (int)ceilf(8.0f / cfg.cell);
        for (const auto& p : ps) {
            usize ci, cj;
            if (!coarse_ij(p.x, p.z, ci, cj)) continue;
            int a = (int)ci, b = (int)cj, r = (int)res;
            i0 = std::min(i0, (usize)std::max(a - reach, 0)); i1 = std::max(i1, (usize)std::min(a + reach, r - 1));
            j0 = std::min(j0, (usize)std::max(b - reach, 0)); j1 = std::max(j1, (usize)std::min(b + reach, r - 1));
            any = true;
        }
        return any;
    }

    // src/fluid_core.rs:6339-6349 sync_foam_live.
    void sync_foam_live() {
        foam_live.clear();
        std::fill(foam_live_mark.begin(), foam_live_mark.end(), 0);
        for (uint32_t id : wet_idx)
            if (finite(foam[id]) && foam[id] > 1.0e-4f) {
                foam_live_mark[id] = 1;
                foam_live.push_back(id);
            }
    }

    // src/fluid_core.rs:6352-6397 advect_foam: semi-Lagrangian on the wet cells.
    void advect_foam(float dt) {
        const float cell = cfg.cell;
        std::vector<float> src = foam;
        std::vector<float> samp(wet_idx.size(), 0.0f);
        for (usize k = 0; k < wet_idx.size(); ++k) {
            usize idx = wet_idx[k];
            float u = uw[idx], v = vw[idx];
            float sample = 0.0f;
            if (finite(u) && finite(v)) {
                usize i = idx % res, j = idx / res;
                float x = (float)i - u * dt / cell;
                float z = (float)j - v * dt / cell;
                sample = sample_foam(src.data(), res, x, z);
            }
            samp[k] = sample;
        }
        std::vector<float> next = src;
        for (uint32_t id : foam_live) next[id] = 0.0f;
        for (uint32_t id : wet_idx) next[id] = 0.0f;
        float decay = expf(-dt / FOAM_LIFE_S);
        for (usize k = 0; k < wet_idx.size(); ++k) {
            float v = samp[k] * decay;
            if (v > 1.0e-4f && finite(v)) next[wet_idx[k]] = rmin(v, FOAM_EQ);
        }
        foam = next;
    }

    // src/fluid_core.rs:6400-6418 add_foam.
    void add_foam(usize idx, float prod, float dt) {
        if (prod <= 0.0f || !finite(prod) || !(dt > 0.0f)) return;
        float cur = finite(foam[idx]) ? rclamp(foam[idx], 0.0f, FOAM_EQ) : 0.0f;
        float room = FOAM_EQ - cur;
        if (room <= 1.0e-5f) return;
        float grown = cur + room * prod * rmin(dt / FOAM_TAU_S, 1.0f);
        foam[idx] = finite(grown) ? rmin(grown, FOAM_EQ) : 0.0f;
    }

    // src/fluid_core.rs:6421-6470 advect_turbid: donor-cell transport of the silt column.
    void advect_turbid(float dt) {
        usize i0, i1, j0, j1;
        if (!turbid_span(turbid.data(), res, i0, i1, j0, j1)) return;
        usize n = res * res;
        std::vector<float> scratch(2 * n, 0.0f);
        flux_thickness(turbid.data(), uw.data(), vw.data(), res, cfg.cell, dt, i0, i1, j0, j1, scratch.data());
        for (usize j = j0; j <= j1; ++j)
            for (usize i = i0; i <= i1; ++i) {
                usize idx = j * res + i;
                float removed = scratch[idx], added = scratch[n + idx];
                if (removed == 0.0f && added == 0.0f) {
                    if (!finite(turbid[idx])) turbid[idx] = 0.0f;
                    continue;
                }
                float next = turbid[idx] - removed + added;
                turbid[idx] = finite(next) ? rmax(next, 0.0f) : 0.0f;
            }
    }

    // src/fluid_core.rs:6473-6509 settle_turbid.
    void settle_turbid(float dt) {
        const float area = cfg.cell * cfg.cell;
        float keep = expf(-dt / SILT_SETTLE_S);
        float settled = 0.0f;
        double settled64 = 0.0;
        usize i0, i1, j0, j1;
        if (!turbid_span(turbid.data(), res, i0, i1, j0, j1)) return;
        for (usize j = j0; j <= j1; ++j)
            for (usize i = i0; i <= i1; ++i) {
                usize idx = j * res + i;
                float h = water[idx] + slurry[idx];
                float column = finite(turbid[idx]) ? rmax(turbid[idx], 0.0f) : 0.0f;
                if (column <= 0.0f) { turbid[idx] = 0.0f; continue; }
                if (!finite(h) || h < 1.0e-5f) {
                    settled += column * area;
                    settled64 += (double)(column * area);
                    turbid[idx] = 0.0f;
                    continue;
                }
                float stay = column * keep;
                settled += (column - stay) * area;
                settled64 += (double)((column - stay) * area);
                turbid[idx] = stay;
            }
        if (finite(settled)) {
            turbid_settled_m3 += settled;
            turbid_settled64 += settled64;
        }
    }

    // src/fluid_core.rs:6545-6558 spawn_breaking_speed.
    void spawn_breaking_speed(float dt) {
        for (uint32_t id : wet_idx) {
            float h = water[id] + slurry[id];
            if (!finite(h) || h < 0.004f) continue;
            float u = uw[id], v = vw[id];
            if (!finite(u) || !finite(v) || hypotf(u, v) <= 0.05f) continue;
            float speed = hypotf(u, v);
            add_foam(id, breaking_foam(speed, h), dt);
        }
    }

    // src/fluid_core.rs:6599-6665 spawn_tire_tracers.
    void spawn_tire_tracers(const TirePush& p, float dt, float area) {
        float speed = finite(p.speed) ? rmax(p.speed, 0.0f) : 0.0f;
        float slip = finite(p.slip) ? rmin(fabsf(p.slip), 1.5f) : 0.0f;
        if (speed < 0.25f && slip < 0.05f) return;
        float radius = rmax(p.radius, 0.05f);
        float len = rmax(sqrtf(p.forward_x * p.forward_x + p.forward_z * p.forward_z), 1.0e-4f);
        float fx = p.forward_x / len, fz = p.forward_z / len;
        float rx = fz, rz = -fx;
        const float cell = cfg.cell;
        float reach = radius * 1.15f + cell;
        float reach2 = reach * reach;
        float slip_v = speed * slip;
        for (uint32_t id : wet_idx) {
            usize idx = id;
            float h = water[idx];
            if (!finite(h) || h < 0.004f) continue;
            usize i = idx % res, j = idx / res;
            float x = origin[0] + ((float)i + 0.5f) * cell;
            float z = origin[1] + ((float)j + 0.5f) * cell;
            float dx = x - p.x, dz = z - p.z;
            if (dx * dx + dz * dz > reach2) continue;
            float along = dx * fx + dz * fz;
            float lat = dx * rx + dz * rz;
            float dist = hypotf(dx, dz);
            float film = hypotf(uw[idx], vw[idx]);
            film = finite(film) ? film : 0.0f;
            float immerse = rmin(h, radius * 0.9f);
            float r_line = sqrtf(rmax(2.0f * radius * immerse - immerse * immerse, 0.0f));
            float band = 1.0f - rclamp(fabsf(dist - r_line) / (cell * 1.35f), 0.0f, 1.0f);
            if (band > 0.0f) {
                float motion = rmax(rmax(slip_v, speed * 0.45f), film);
                float prod = breaking_foam(motion, h) * band;
                add_foam(idx, prod, dt);
            }
            bool on_patch = fabsf(lat) <= p.width * 0.55f + cell * 0.35f && along >= -radius * 0.55f &&
                            along <= radius * 0.35f;
            if (on_patch && h > 0.02f) {
                float shear_v = rmax(slip_v, film * 0.35f);
                lift_silt(idx, shear_v, dt, area, 0.015f, 6.0f);
            }
        }
    }

    // src/fluid_core.rs:6667-6684 spawn_shore_tracers.
    void spawn_shore_tracers(float dt, float area) {
        for (uint32_t id : shore_idx) {
            float prod, silt_add;
            shore_cell(water.data(), uw.data(), vw.data(), res, id, prod, silt_add);
            add_foam(id, prod, dt);
            if (silt_add > 0.0f) add_silt(id, rmin(silt_add * dt, 0.0012f), area);
        }
    }

    // src/fluid_core.rs:6686-6697 lift_silt.
    void lift_silt(usize idx, float shear_v, float dt, float area, float rate_cap, float tau_c) {
        if (!finite(shear_v) || shear_v <= 0.0f) return;
        float tau = 1000.0f * 0.035f * shear_v * shear_v;
        if (tau <= tau_c) return;
        float rate = rmin(0.008f * (tau / tau_c - 1.0f), rate_cap);
        add_silt(idx, rmin(rate * dt, 0.0025f), area);
    }

    // src/fluid_core.rs:6699-6710 add_silt.
    void add_silt(usize idx, float dh, float area) {
        if (dh <= 0.0f || !finite(dh)) return;
        float room = rmax(SILT_COLUMN_CAP_M - rmax(turbid[idx], 0.0f), 0.0f);
        float add = rmin(dh, room);
        if (add <= 0.0f) return;
        turbid[idx] += add;
        stirred_m3 += add * area;
        stirred64 += (double)(add * area);
    }

    // src/fluid_core.rs:6712-6739 clear_dry_tracers.
    void clear_dry_tracers() {
        const float area = cfg.cell * cfg.cell;
        for (uint32_t id : wet_idx) {
            float h = water[id] + slurry[id];
            if (!finite(h) || h < 0.004f) foam[id] = 0.0f;
            else if (!finite(foam[id])) foam[id] = 0.0f;
        }
        usize i0, i1, j0, j1;
        if (!turbid_span(turbid.data(), res, i0, i1, j0, j1)) return;
        for (usize j = j0; j <= j1; ++j)
            for (usize i = i0; i <= i1; ++i) {
                usize idx = j * res + i;
                float h = water[idx] + slurry[idx];
                if (!finite(h) || h < 1.0e-5f) {
                    if (turbid[idx] > 0.0f) {
                        turbid_settled_m3 += turbid[idx] * area;
                        turbid_settled64 += (double)(turbid[idx] * area);
                        turbid[idx] = 0.0f;
                    }
                } else if (!finite(turbid[idx])) {
                    turbid[idx] = 0.0f;
                }
            }
    }

    // src/fluid_core.rs:8817-9002 advect_suspended (step_suspended :8750-8756).
    void step_suspended(float dt) {
        last_susp_capped = 0;
        if (dt <= 0.0f || !finite(dt)) return;
        const float cell = cfg.cell, area = cell * cell;
        usize i0 = res, i1 = 0, j0 = res, j1 = 0;
        double landed_m3 = 0.0;
        for (usize j = 0; j < res; ++j)
            for (usize i = 0; i < res; ++i) {
                usize idx = j * res + i;
                float sv = susp[idx];
                if (!finite(sv) || sv <= 1.0e-12f) { susp[idx] = 0.0f; continue; }
                float w = water[idx];
                if (!finite(w) || w < 1.0e-5f || sv > w) {
                    settled_suspended_m3 += sv * area;
                    settled_suspended64 += (double)(sv * area);
                    susp[idx] = 0.0f;
                    continue;
                }
                float keep = expf(-dt * SUSP_FALL_M_S / w);
                float landed = sv * (1.0f - keep);
                if (landed > 0.0f) {
                    landed_m3 += (double)landed * (double)area;
                    sv -= landed;
                    susp[idx] = sv;
                }
                if (sv > 1.0e-8f) {
                    i0 = std::min(i0, i); i1 = std::max(i1, i); j0 = std::min(j0, j); j1 = std::max(j1, j);
                }
            }
        settled_suspended_m3 += (float)landed_m3;
        settled_suspended64 += landed_m3;
        if (i0 > i1) return;
        i0 = sat_sub(i0, 1); j0 = sat_sub(j0, 1);
        i1 = std::min(i1 + 1, res - 1); j1 = std::min(j1 + 1, res - 1);
        susp_next = susp;
        std::fill(susp_taken.begin(), susp_taken.end(), 0.0f);
        const bool open = surface_driven();
        for (usize j = j0; j <= j1; ++j)
            for (usize i = i0; i <= i1; ++i) {
                usize idx = j * res + i;
                float depth = susp[idx], w = water[idx];
                if (depth <= 1.0e-12f || !finite(depth) || !finite(w) || w < 1.0e-5f) continue;
                // film_uv(water, 0, uw, vw, 0, 0) (:3490-3501)
                float u = 0.0f, v = 0.0f;
                {
                    float hh = w + 0.0f;
                    if (finite(hh) && !(hh < 1.0e-5f)) {
                        u = finite0((uw[idx] * w + 0.0f * 0.0f) / hh);
                        v = finite0((vw[idx] * w + 0.0f * 0.0f) / hh);
                    }
                }
                u = open && finite(u) ? u : 0.0f;
                v = finite(v) ? v : 0.0f;
                float c = depth / w;
                float fu = fabsf(u) * dt / cell, fv = fabsf(v) * dt / cell;
                float sum = fu + fv;
                if (sum > 0.45f) { fu *= 0.45f / sum; fv *= 0.45f / sum; }
                long up_i = u > 0.0f ? (i + 1 < res ? (long)(idx + 1) : -1) : (i > 0 ? (long)(idx - 1) : -1);
                long up_j = v > 0.0f ? (j + 1 < res ? (long)(idx + res) : -1) : (j > 0 ? (long)(idx - res) : -1);
                const float fr[2] = {fu, fv};
                const long rv[2] = {up_i, up_j};
                for (int q = 0; q < 2; ++q) {
                    float give = depth * fr[q];
                    if (give <= 1.0e-12f) continue;
                    if (rv[q] < 0) {
                        settled_suspended_m3 += give * area;
                        settled_suspended64 += (double)(give * area);
                        susp_next[idx] -= give;
                        continue;
                    }
                    usize nn = (usize)rv[q];
                    float wr = water[nn];
                    if (!finite(wr) || wr < 1.0e-5f) continue;
                    float have = susp[nn] + susp_taken[nn];
                    float room = rmax(c * wr - have, 0.0f);
                    float accept = rmin(rmin(give, room), rmax(wr - have, 0.0f));
                    if (accept <= 1.0e-12f) continue;
                    susp_next[idx] -= accept;
                    susp_taken[nn] += accept;
                }
                if (!open) continue;
                float speed = sqrtf(u * u + v * v);
                float k = 0.01f + 0.2f * speed * w;
                float fd = rmin(k * dt / (cell * cell), 0.1f);
                const long nb[4] = {i + 1 < res ? (long)(idx + 1) : -1, i > 0 ? (long)(idx - 1) : -1,
                                    j + 1 < res ? (long)(idx + res) : -1, j > 0 ? (long)(idx - res) : -1};
                for (long nl : nb) {
                    if (nl < 0) continue;
                    usize nn = (usize)nl;
                    float wr = water[nn];
                    if (!finite(wr) || wr < 1.0e-5f) continue;
                    float cn = susp[nn] / wr;
                    if (!(c > cn)) continue;
                    float give = fd * (c - cn) * rmin(w, wr);
                    float have = susp[nn] + susp_taken[nn];
                    float accept = rmin(give, rmax(wr - have, 0.0f));
                    if (accept <= 1.0e-12f) continue;
                    susp_next[idx] -= accept;
                    susp_taken[nn] += accept;
                }
            }
        for (usize j = j0; j <= j1; ++j)
            for (usize i = i0; i <= i1; ++i) susp_next[j * res + i] += susp_taken[j * res + i];
        uint32_t capped = 0;
        for (usize j = j0; j <= j1; ++j)
            for (usize i = i0; i <= i1; ++i) {
                usize idx = j * res + i;
                float sv = susp_next[idx];
                if (!finite(sv) || sv <= 0.0f) { susp_next[idx] = 0.0f; continue; }
                float w = water[idx];
                if (!finite(w) || w < 1.0e-5f) {
                    settled_suspended_m3 += sv * area;
                    settled_suspended64 += (double)(sv * area);
                    sv = 0.0f;
                } else if (sv > w) {
                    float excess = sv - w;
                    settled_suspended_m3 += excess * area;
                    settled_suspended64 += (double)(excess * area);
                    if (excess > 1.0e-5f) capped += 1;
                    sv = w;
                }
                susp_next[idx] = sv;
            }
        last_susp_capped += capped;
        std::swap(susp, susp_next);
    }

    // Inflow strip: one coarse row, water added as depth, booked as opened volume.
    void apply_inflow(float dt) {
        std::vector<usize> cells;
        for (usize i = 0; i < res; ++i) {
            float x, z;
            coarse_xz(i, (usize)inflow_j, x, z);
            if (x >= inflow_x0 && x < inflow_x1) cells.push_back((usize)inflow_j * res + i);
        }
        if (cells.empty()) return;
        float add = inflow_rate * dt / ((float)cells.size() * cfg.cell * cfg.cell);
        for (usize idx : cells) water[idx] += add;
        opened_m3 += (double)add * (double)cfg.cell * (double)cfg.cell * (double)cells.size();
    }
};

float column_sum(const std::vector<float>& h, float cell) {  // src/fluid_core.rs:4617-4620
    float area = cell * cell;
    float s = -0.0f;
    for (float x : h) s += rmax(x, 0.0f);
    return s * area;
}

}  // namespace

// ============================================================== C interface
extern "C" {

void* oracle_scratch_new(void) { return new Scratch(); }
void oracle_scratch_free(void* sc) { delete (Scratch*)sc; }

void oracle_step_sheet(float* h, float* u, float* v, const float* bed, const float* nu, const uint8_t* gate,
                       int res, float cell, float dt, float vorticity, float eps, int banks, float sub_cap,
                       int pace, int inner_par, void* sc) {
    if (res <= 0) return;
    step_sheet_eps(h, u, v, bed, nu, gate, (usize)res, cell, dt, vorticity, eps, banks != 0, sub_cap, pace,
                   *(Scratch*)sc, nullptr, inner_par != 0);
}

void oracle_transport_open(float* h, const float* vel, const uint8_t* gate, int res, float cell, float dt,
                           int i0, int i1, int j0, int j1, int along_x, const float* bed, float frac_cap,
                           int serial, float* removed, float* added) {
    Scratch sc;
    sc.fit((usize)res * res);
    if (serial)
        transport_open_serial(h, vel, gate, res, cell, dt, i0, i1, j0, j1, along_x != 0, bed, frac_cap, sc);
    else
        transport_open_rows(bed != nullptr, h, vel, gate, res, cell, dt, i0, i1, j0, j1, along_x != 0, bed, frac_cap, sc);
    memcpy(removed, sc.removed.data(), sizeof(float) * res * res);
    memcpy(added, sc.added.data(), sizeof(float) * res * res);
}

static int put_boxes(const std::vector<Box>& b, int* out, int cap) {
    int n = (int)b.size();
    for (int k = 0; k < n && k < cap; ++k) {
        out[4 * k] = (int)b[k].i0; out[4 * k + 1] = (int)b[k].i1;
        out[4 * k + 2] = (int)b[k].j0; out[4 * k + 3] = (int)b[k].j1;
    }
    return n;
}
int oracle_sheet_work_boxes(const float* h, int res, float eps, int allow_split, int flood, int* out, int cap) {
    return put_boxes(flood ? sheet_work_boxes_flood(h, res, eps, allow_split != 0) : sheet_work_boxes(h, res, eps, allow_split != 0), out, cap);
}
int oracle_awake_work_boxes(const float* h, const float* u, const float* v, const float* bed, int res, float cell,
                            float eps, int* out, int cap) {
    return put_boxes(awake_work_boxes(h, u, v, bed, res, cell, eps), out, cap);
}
float oracle_dynamic_viscosity(int grain, float moisture) { return dynamic_viscosity((u8)grain, moisture); }
float oracle_sheet_mobility_for(float nu) { return sheet_mobility_for(nu); }
float oracle_sheet_damp(float nu) { return sheet_damp(nu); }
void oracle_soften_border(float* u, float* v, int res) { soften_border(u, v, (usize)res); }

// src/fluid_core.rs:4673-4760 rut_heal + relief
static float relief(const std::vector<float>& h, const std::vector<float>& bed, usize res, float cell) {
    float c = (float)(res / 2);
    float center = 0, cn = 0, ring = 0, rn = 0;
    for (usize j = 0; j < res; ++j)
        for (usize i = 0; i < res; ++i) {
            float x = ((float)i + 0.5f - c) * cell, z = ((float)j + 0.5f - c) * cell;
            float r = sqrtf(x * x + z * z);
            float eta = bed[j * res + i] + h[j * res + i];
            if (r < 0.12f) { center += eta; cn += 1.0f; }
            else if (r >= 0.48f && r < 0.68f) { ring += eta; rn += 1.0f; }
        }
    if (cn < 1.0f || rn < 1.0f) return 0.0f;
    return (ring / rn) - (center / cn);
}
void oracle_rut_heal(int grain, float moisture, float* out4) {
    usize res = 48;
    float cell = 0.06f;
    usize n = res * res;
    std::vector<float> h(n, 0), u(n, 0), v(n, 0), bed(n, 0);
    float nu_v = dynamic_viscosity((u8)grain, moisture);
    std::vector<float> nu(n, nu_v);
    std::vector<u8> gate(n, 1);
    float c = (float)(res / 2);
    for (usize j = 0; j < res; ++j)
        for (usize i = 0; i < res; ++i) {
            float x = ((float)i + 0.5f - c) * cell, z = ((float)j + 0.5f - c) * cell;
            float r = sqrtf(x * x + z * z);
            usize idx = j * res + i;
            float bowl = expf(-(r * r) / (2.0f * 0.42f * 0.42f));
            bed[idx] = -0.07f * bowl;
            h[idx] = 0.012f + 0.028f * (1.0f - bowl);
        }
    float relief0 = relief(h, bed, res, cell);
    float level_s = 20.0f, relief_8s = relief0, t = 0.0f, dt = 0.05f;
    Scratch sc;
    while (t < 20.0f - 1.0e-4f) {
        step_sheet_eps(h.data(), u.data(), v.data(), bed.data(), nu.data(), gate.data(), res, cell, dt, 0.0f, 1.0e-6f, false, 8.0f, 0, sc, nullptr, true);
        t += dt;
        float r = relief(h, bed, res, cell);
        if (fabsf(t - 8.0f) <= dt * 0.51f) relief_8s = r;
        if (level_s > 19.0f && r < relief0 * 0.28f) level_s = t;
        if (t >= 8.0f && level_s < 19.0f) break;
    }
    out4[0] = level_s; out4[1] = relief0; out4[2] = relief_8s; out4[3] = relief_8s > relief0 * 0.38f ? 1.0f : 0.0f;
}

void* oracle_core_new(const oracle_core_cfg* cfg) { return new Core(*cfg); }
void oracle_core_free(void* core) { delete (Core*)core; }

// src/fluid_core.rs:5329-5356 map_water_bed (closure values passed per cell)
float oracle_core_map_water_bed(void* cp, const float* bedv, const float* waterv) {
    Core& C = *(Core*)cp;
    C.restrict_fine();
    float vol = 0.0f, area = C.cfg.cell * C.cfg.cell;
    for (usize idx = 0; idx < C.res * C.res; ++idx) {
        C.bed[idx] = finite(bedv[idx]) ? bedv[idx] : 0.0f;
        float w = finite(waterv[idx]) ? rmax(waterv[idx], 0.0f) : 0.0f;
        C.water[idx] = w;
        if (w > 0.0f) {
            C.moisture[idx] = rmax(C.moisture[idx], 0.8f);
            if (C.grain[idx] == 4) C.grain[idx] = 1;
        }
        vol += w * area;
    }
    return vol;
}
void oracle_core_map_grain(void* cp, const uint8_t* g) {  // :5318-5327
    Core& C = *(Core*)cp;
    C.restrict_fine();
    memcpy(C.grain.data(), g, C.res * C.res);
}
void oracle_core_map_water_velocity(void* cp, const float* u, const float* v) {  // :5358-5372
    Core& C = *(Core*)cp;
    C.restrict_fine();
    for (usize idx = 0; idx < C.res * C.res; ++idx) {
        if (C.water[idx] <= 1.0e-6f) continue;
        C.uw[idx] = finite(u[idx]) ? u[idx] : 0.0f;
        C.vw[idx] = finite(v[idx]) ? v[idx] : 0.0f;
    }
}
// :5424-5435 pour_water / pour_slurry via paint :5820-5849
float oracle_core_pour(void* cp, float x0, float x1, float z0, float z1, float depth, int water, int grain,
                       float moisture) {
    Core& C = *(Core*)cp;
    depth = rmax(depth, 0.0f);
    float vol = 0.0f, area = C.cfg.cell * C.cfg.cell;
    for (usize j = 0; j < C.res; ++j)
        for (usize i = 0; i < C.res; ++i) {
            float x, z;
            C.coarse_xz(i, j, x, z);
            if (x < x0 || x >= x1 || z < z0 || z >= z1) continue;
            usize idx = j * C.res + i;
            if (water) C.water[idx] = depth;
            else {
                C.slurry[idx] = depth;
                C.grain[idx] = (u8)grain;
                C.moisture[idx] = rclamp(moisture, 0.0f, 1.0f);
            }
            vol += depth * area;
        }
    return vol;
}
// :5854-5877 lay_slurry_mask
float oracle_core_lay_slurry_mask(void* cp, const float* depth, int grain, float moisture) {
    Core& C = *(Core*)cp;
    C.restrict_fine();
    float vol = 0.0f, area = C.cfg.cell * C.cfg.cell;
    for (usize idx = 0; idx < C.res * C.res; ++idx) {
        float d = depth[idx];
        if (!(finite(d) && d > 0.0f)) continue;
        C.slurry[idx] += d;
        C.grain[idx] = (u8)grain;
        C.moisture[idx] = rmax(C.moisture[idx], rclamp(moisture, 0.0f, 1.0f));
        vol += d * area;
    }
    return vol;
}
// :5928-5962 read_substrate_grid
void oracle_core_read_substrate(void* cp, const float* bedv, const float* moist, const uint8_t* g) {
    Core& C = *(Core*)cp;
    C.restrict_fine();
    uint32_t hist[101] = {0};
    for (usize idx = 0; idx < C.res * C.res; ++idx) {
        float m = rclamp(moist[idx], 0.0f, 1.0f);
        C.bed[idx] = bedv[idx];
        C.moisture[idx] = m;
        float pct = m * 100.0f;
        usize whole = f2usize(pct);
        usize bucket = pct - (float)whole >= 0.5f ? whole + 1 : whole;
        hist[std::min(bucket, (usize)100)] += 1;
        if (C.slurry[idx] > 1.0e-5f) C.grain[idx] = g[idx];
    }
    usize best = 0;
    uint32_t best_n = 0;
    for (usize i = 0; i < 101; ++i)
        if (hist[i] > best_n) { best = i; best_n = hist[i]; }
    C.moisture_ambient = (float)best * 0.01f;
}
void oracle_core_push_tire(void* cp, const oracle_tire* t) {
    ((Core*)cp)->pushes.push_back({t->x, t->z, t->forward_x, t->forward_z, t->radius, t->width, t->speed, t->slip});
}
int oracle_core_step(void* cp, float dt, oracle_spray* out, int cap) {
    std::vector<Spray> s = ((Core*)cp)->step(dt);
    for (int k = 0; k < (int)s.size() && k < cap; ++k)
        out[k] = {s[k].x, s[k].y, s[k].z, s[k].vx, s[k].vy, s[k].vz, s[k].volume, s[k].kind};
    return (int)s.size();
}
// :6821-6883, sheet books only (no dust, fog, reach, suspended)
void oracle_core_ledger(void* cp, float* out5, double* out64) {
    Core& C = *(Core*)cp;
    float water = column_sum(C.water, C.cfg.cell), slurry = column_sum(C.slurry, C.cfg.cell);
    if (C.fine_on)
        for (usize pk = 0; pk < C.active_patches(); ++pk) {
            water += column_sum(C.patches[pk].water, C.cfg.fine_cell);
            slurry += column_sum(C.patches[pk].slurry, C.cfg.fine_cell);
        }
    float fw = 0.0f, fs = 0.0f, area = C.cfg.cell * C.cfg.cell;
    for (auto& kv : C.parked) { fw += kv.second.water * area; fs += kv.second.slurry * area; }
    out5[0] = water; out5[1] = slurry; out5[2] = fw; out5[3] = fs; out5[4] = C.spray_m3;
    double w64 = 0.0, s64 = 0.0;
    for (float x : C.water) w64 += (double)rmax(x, 0.0f);
    for (float x : C.slurry) s64 += (double)rmax(x, 0.0f);
    out64[0] = w64 * (double)C.cfg.cell * (double)C.cfg.cell;
    out64[1] = s64 * (double)C.cfg.cell * (double)C.cfg.cell;
}
static std::vector<float>* core_field(Core& C, int which) {
    switch (which) {
        case 0: return &C.water; case 1: return &C.slurry; case 2: return &C.uw; case 3: return &C.vw;
        case 4: return &C.us; case 5: return &C.vs; case 6: return &C.bed; case 8: return &C.foam;
        case 9: return &C.turbid; case 10: return &C.susp; default: return &C.moisture;
    }
}
void oracle_core_get(void* cp, int which, float* dst) {
    Core& C = *(Core*)cp;
    std::vector<float>* f = core_field(C, which);
    memcpy(dst, f->data(), f->size() * sizeof(float));
}
void oracle_core_set(void* cp, int which, const float* src) {
    Core& C = *(Core*)cp;
    std::vector<float>* f = core_field(C, which);
    memcpy(f->data(), src, f->size() * sizeof(float));
}
void oracle_core_get_grain(void* cp, uint8_t* dst) { Core& C = *(Core*)cp; memcpy(dst, C.grain.data(), C.grain.size()); }
// src/render_contract.rs:457-496 film/flow via coarse_cell (:6998-7035), the
// turbidity channel from the suspended and stirred columns (:7024-7032).
void oracle_core_publish(void* cp, float* film, float* flow) {
    Core& C = *(Core*)cp;
    for (usize idx = 0; idx < C.res * C.res; ++idx) {
        float water_m = finite0(C.water[idx]), slurry_m = finite0(C.slurry[idx]);
        float turbidity = water_m < 1.0e-5f
                              ? 0.0f
                              : rclamp((rmax(finite0(C.susp[idx]), 0.0f) + rmax(finite0(C.turbid[idx]), 0.0f)) /
                                           water_m,
                                       0.0f, 1.0f);
        float turb = (!finite(water_m) || water_m < 1.0e-5f) ? 0.0f : rclamp(finite0(turbidity), 0.0f, 1.0f);
        float fl = water_m + slurry_m;
        float u = 0.0f, v = 0.0f;
        if (!(fl < 1.0e-5f)) {
            u = finite0((C.uw[idx] * water_m + C.us[idx] * slurry_m) / fl);
            v = finite0((C.vw[idx] * water_m + C.vs[idx] * slurry_m) / fl);
        }
        bool dry = !finite(water_m) || !finite(slurry_m) || water_m + slurry_m < 1.0e-5f;
        if (dry) { u = 0.0f; v = 0.0f; } else { u = finite0(u); v = finite0(v); }
        float speed = dry ? 0.0f : finite0(sqrtf(u * u + v * v));
        film[2 * idx] = finite0(water_m);
        film[2 * idx + 1] = finite0(slurry_m);
        flow[4 * idx] = u; flow[4 * idx + 1] = v; flow[4 * idx + 2] = speed; flow[4 * idx + 3] = turb;
    }
}
// src/fluid_core.rs:5097-5099 set_turbidity_enabled.
void oracle_core_set_turbidity(void* cp, int on) { ((Core*)cp)->turbidity_enabled = on != 0; }
// RiverReach::inlet_turbidity (src/fluid_core.rs:319).
void oracle_core_set_reach_turbidity(void* cp, float c) { ((Core*)cp)->reach_inlet_turbidity = c; }
// The tracer books (src/fluid_core.rs:6171-6195 silt book, :6821-6884 the
// suspended part of the ledger), out8 in f32 as the reference keeps them and
// out64 the same terms in FP64: [0] suspended in the column, [1] settled
// suspended, [2] parked suspended, [3] entrained, [4] stirred silt in the
// column, [5] settled silt, [6] stirred, [7] parked silt.
void oracle_core_tracer_books(void* cp, float* out8, double* out64) {
    Core& C = *(Core*)cp;
    const float area = C.cfg.cell * C.cfg.cell;
    float susp_sum = -0.0f, turbid_sum = 0.0f;
    double susp64 = 0.0, turbid64 = 0.0;
    for (usize k = 0; k < C.res * C.res; ++k) {
        susp_sum += rmax(C.susp[k], 0.0f);
        susp64 += (double)rmax(C.susp[k], 0.0f);
        float t = finite(C.turbid[k]) ? rmax(C.turbid[k], 0.0f) : 0.0f;
        turbid_sum = turbid_sum + t;
        turbid64 += (double)t;
    }
    float fsusp = 0.0f, fturb = 0.0f;
    double fsusp64 = 0.0, fturb64 = 0.0;
    for (const auto& kv : C.parked) {
        fsusp += kv.second.susp * area;
        fsusp64 += (double)kv.second.susp * (double)area;
        if (finite(kv.second.turbid)) {
            fturb += rmax(kv.second.turbid, 0.0f) * area;
            fturb64 += (double)rmax(kv.second.turbid, 0.0f) * (double)area;
        }
    }
    out8[0] = susp_sum * area; out64[0] = susp64 * (double)area;
    out8[1] = C.settled_suspended_m3; out64[1] = C.settled_suspended64;
    out8[2] = fsusp; out64[2] = fsusp64;
    out8[3] = C.entrained_m3; out64[3] = C.entrained64;
    out8[4] = turbid_sum * area; out64[4] = turbid64 * (double)area;
    out8[5] = C.turbid_settled_m3; out64[5] = C.turbid_settled64;
    out8[6] = C.stirred_m3; out64[6] = C.stirred64;
    out8[7] = fturb; out64[7] = fturb64;
}
void oracle_core_set_fine_pace(void* cp, int pace) { ((Core*)cp)->fine_pace = std::min(pace, 3); }
void oracle_core_set_fine_sub_cap(void* cp, float cap) { ((Core*)cp)->fine_sub_cap = finite(cap) ? rclamp(cap, 1.0f, 8.0f) : 8.0f; }
// src/fluid_core.rs:5293-5303 set_open_water (on = 0: None).
void oracle_core_set_open_water(void* cp, int on, float mobility, float manning_n, float eddy_m2_s) {
    Core& C = *(Core*)cp;
    C.open_water = on != 0 && finite(mobility) && finite(manning_n) && finite(eddy_m2_s);
    if (!C.open_water) return;
    C.ow_mobility = rmin(rmax(mobility, 0.0f), 1.0f);
    C.ow_manning = rmax(manning_n, 0.0f);
    C.ow_eddy = rmax(eddy_m2_s, 0.0f);
}
// src/fluid_core.rs:5273-5275 set_river_reach (on = 0: None).
void oracle_core_set_river_reach(void* cp, int on, int along_z, int positive, float cross0, float cross1, int rows,
                                 float inlet_eta, float outlet_eta, float inlet_speed) {
    Core& C = *(Core*)cp;
    C.reach_on = on != 0;
    C.reach_along_z = along_z != 0;
    C.reach_positive = positive != 0;
    C.reach_cross0 = cross0;
    C.reach_cross1 = cross1;
    C.reach_rows = rows > 0 ? (usize)rows : 0;
    C.reach_inlet_eta = inlet_eta;
    C.reach_outlet_eta = outlet_eta;
    C.reach_speed = inlet_speed;
}
float oracle_core_reach_bank(void* cp) { return ((Core*)cp)->reach_bank_m3; }
// Solids as 10 floats each: x, z, yaw, half_length, half_width, bottom_y,
// top_y, contact (0/1), radius, width.
void oracle_core_set_hydro_solids(void* cp, const float* packed, int n) {
    Core& C = *(Core*)cp;
    C.solids.clear();
    for (int k = 0; k < n; ++k) {
        const float* f = packed + 10 * k;
        C.solids.push_back(HydroSolid{f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7] != 0.0f, f[8], f[9]});
    }
}
// src/fluid_core.rs:5236-5254 lay_slurry_on_water.
float oracle_core_lay_slurry_on_water(void* cp, float depth, int grain) {
    Core& C = *(Core*)cp;
    if (!(finite(depth) && depth > 0.0f)) return 0.0f;
    C.restrict_fine();
    const float area = C.cfg.cell * C.cfg.cell;
    float vol = 0.0f;
    for (usize idx = 0; idx < C.water.size(); ++idx) {
        if (C.water[idx] <= 0.012f) continue;
        C.slurry[idx] = depth;
        C.grain[idx] = (u8)grain;
        C.moisture[idx] = rmax(C.moisture[idx], 0.90f);
        vol += depth * area;
    }
    return vol;
}
void oracle_core_hydro_load(void* cp, float* out10) { ((Core*)cp)->hydro_load(out10); }
// The wall mask the next coarse step pair would use (res^2 bytes).
void oracle_core_solid_mask(void* cp, uint8_t* out) {
    Core& C = *(Core*)cp;
    std::vector<u8> m = solid_mask(C.solids, C.res, C.cfg.cell, C.origin, C.water.data(), C.bed.data());
    memcpy(out, m.data(), m.size());
}
// src/fluid_core.rs:5306-5309 set_wave_maker (restarts the paddle clock).
void oracle_core_set_wave_maker(void* cp, int on, float x0, float x1, float z0, float z1, float dir_x, float dir_z,
                                float amplitude, float period, float ramp) {
    Core& C = *(Core*)cp;
    C.wave_on = on != 0;
    C.wave_x0 = x0; C.wave_x1 = x1; C.wave_z0 = z0; C.wave_z1 = z1;
    C.wave_dx = dir_x; C.wave_dz = dir_z;
    C.wave_amp = amplitude; C.wave_period = period; C.wave_ramp = ramp;
    C.wave_t = 0.0f;
}
// src/fluid_core.rs:5409-5421 recenter.
void oracle_core_recenter(void* cp, float cx, float cz) { ((Core*)cp)->recenter(cx, cz); }
void oracle_core_origin(void* cp, float* out2) {
    Core& C = *(Core*)cp;
    out2[0] = C.origin[0];
    out2[1] = C.origin[1];
}
int oracle_core_parked_count(void* cp) { return (int)((Core*)cp)->parked.size(); }
// src/fluid_core.rs:5284-5286 set_surface_diffusion.
void oracle_core_set_surface_diffusion(void* cp, float m2_s) {
    Core& C = *(Core*)cp;
    C.surface_diffusion = finite(m2_s) ? rmax(m2_s, 0.0f) : 0.0f;
}
void oracle_core_set_near_field(void* cp, int on) {
    Core& C = *(Core*)cp;
    C.near_on = on != 0;
    if (!on) C.near.clear();
}
int oracle_core_near_tiles(void* cp) { return (int)((Core*)cp)->near.size(); }
float oracle_core_spray_m3(void* cp) { return ((Core*)cp)->spray_m3; }
uint32_t oracle_core_non_finite(void* cp) {
    Core& C = *(Core*)cp;
    uint32_t n = 0;
    for (auto* f : {&C.water, &C.slurry, &C.uw, &C.vw, &C.us, &C.vs, &C.bed, &C.moisture})
        for (float x : *f) n += !finite(x);
    return n;
}
// :6806-6815 sample (coarse only between steps; the patch is packed)
void oracle_core_sample(void* cp, float x, float z, float* out7) {
    Core& C = *(Core*)cp;
    usize i, j;
    for (int k = 0; k < 7; ++k) out7[k] = 0.0f;
    if (!C.coarse_ij(x, z, i, j)) return;
    usize idx = j * C.res + i;
    out7[0] = C.water[idx]; out7[1] = C.slurry[idx]; out7[2] = C.us[idx]; out7[3] = C.vs[idx];
    out7[4] = 0.0f; out7[5] = C.moisture[idx]; out7[6] = C.bed[idx];
}
void oracle_core_fine_water_debug(void* cp, const oracle_tire* tires, int n, int patch, float* dst, float* origin2) {
    Core& C = *(Core*)cp;
    std::vector<TirePush> ps;
    for (int k = 0; k < n; ++k)
        ps.push_back({tires[k].x, tires[k].z, tires[k].forward_x, tires[k].forward_z, tires[k].radius, tires[k].width, tires[k].speed, tires[k].slip});
    C.refine(ps, 0.0f);
    if (patch < (int)C.active_patches()) {
        memcpy(dst, C.patches[patch].water.data(), C.fres * C.fres * sizeof(float));
        origin2[0] = C.patches[patch].origin[0];
        origin2[1] = C.patches[patch].origin[1];
    }
    C.restrict_fine();
}
void oracle_core_inflow(void* cp, int j, float x0, float x1, float rate) {
    Core& C = *(Core*)cp;
    C.inflow_j = j; C.inflow_x0 = x0; C.inflow_x1 = x1; C.inflow_rate = rate;
}
}
