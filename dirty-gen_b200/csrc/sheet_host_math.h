// Host copies of the reference's scalar laws (x3-team/Dirty-gen
// src/fluid_core.rs:150-192, :9888-9897). The host evaluates the water
// sheet's constant damping factor with the same libm the reference uses, so
// the water layer's damping is bit-identical.
#pragma once
#include <algorithm>
#include <cmath>

namespace silt {
namespace host {

constexpr float kFineCell = 0.02f;
constexpr float kSpeedCap = 1.6f;
constexpr float kGravityHost = 9.81f;  // GRAVITY, src/fluid_core.rs:111

inline float rclamp(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
inline float finite0(float v) { return std::isfinite(v) ? v : 0.0f; }

inline float dynamic_viscosity(int grain, float moisture) {
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

inline float sheet_mobility_for(float nu) {
    if (nu < 0.0f) return -nu;
    float boost = 0.0f;
    if (nu < 12.0f) {
        float t = rclamp((12.0f - std::fmax(nu, 0.0f)) / 12.0f, 0.0f, 1.0f);
        boost = t * t * 1.6f;
    }
    return 0.042f * (1.0f + boost);
}

inline float sheet_damp(float nu) {
    float rel = rclamp(std::fmax(nu, 0.05f) / 231.0f, 0.002f, 12.0f);
    if (rel >= 0.42f) return 1.70f * powf(rel, 0.30f);
    float at_silt = 1.70f * powf(0.42f, 0.30f);
    float t = rclamp(rel / 0.42f, 0.0f, 1.0f);
    return at_silt * powf(t, 1.15f);
}

inline void snap_origin(float cx, float cz, float extent, float cell, float* out) {
    float x = cx - extent * 0.5f, z = cz - extent * 0.5f;
    out[0] = std::floor(x / cell) * cell;
    out[1] = std::floor(z / cell) * cell;
}

}  // namespace host
}  // namespace silt
