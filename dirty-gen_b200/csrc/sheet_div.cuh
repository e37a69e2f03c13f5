// Division by a divisor that is fixed for a whole launch (2 * cell, cell^2,
// 231, cell): q = x * r with r = RN(1 / d), one refinement with the exact
// remainder rem = fma(-q, d, x), q' = fma(rem, r, q) (Markstein's FMA
// correction: P. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990), and the
// sign of x (d > 0, so a zero quotient keeps x's sign as IEEE division does),
// for |x| in [2^-90, 2^90] and zeros; other x divide by IEEE division.
// The runtime enables it for a divisor only after checking it against IEEE
// division for every one of the 2^32 float bit patterns of x
// (fixed_div_for); any mismatch keeps that divisor on IEEE division.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace silt {

struct FixedDiv {
    float d;
    float r;
    int32_t exact;  // 1: the refined product equals IEEE x / d for every float x
};

__device__ __forceinline__ float fdiv(float x, const FixedDiv& D) {
    const float ax = fabsf(x);
    // Outside [2^-90, 2^90] (zeros aside) the product can overflow or the
    // remainder fall below the normal range: IEEE division there.
    if (!D.exact || !(ax <= 0x1p90f) || (ax < 0x1p-90f && ax != 0.0f)) return x / D.d;
    const float q = x * D.r;
    const float rem = __fmaf_rn(-q, D.d, x);
    return copysignf(__fmaf_rn(rem, D.r, q), x);
}

// The divisors of one sheet's step for its cell width: 2 cell (the centred
// differences), cell^2 (the laplacian), 231 (the projection's overload) and
// cell (the face fraction speed dt / cell).
struct CellDivisors {
    FixedDiv two, cell2, d231, cell;
};

// Every divisor on IEEE division (no check, no device work).
inline CellDivisors ieee_cell_divisors(float cell) {
    CellDivisors D;
    D.two = FixedDiv{2.0f * cell, 1.0f / (2.0f * cell), 0};
    D.cell2 = FixedDiv{cell * cell, 1.0f / (cell * cell), 0};
    D.d231 = FixedDiv{231.0f, 1.0f / 231.0f, 0};
    D.cell = FixedDiv{cell, 1.0f / cell, 0};
    return D;
}

// The same divisors, each checked (fixed_div_for).
CellDivisors cell_divisors(float cell, cudaStream_t st);

// The divisor d with its reciprocal, exact only when the exhaustive check
// passed: divisors of the standard cell widths are known to pass; any other
// is checked once per distinct d and device, on `st`, and a completed check
// is cached.
FixedDiv fixed_div_for(float d, cudaStream_t st);
// The divisors known to pass without a check at run time (out[0, cap));
// returns how many there are.
int known_exact_divisors(float* out, int cap);

// Mismatch counts of fdiv against IEEE division over all 2^32 x: [0] all,
// [1] x zero, [2] x subnormal, [3] x infinite or NaN, [4] x normal with a
// subnormal or zero IEEE quotient, [5] the rest.
cudaError_t check_fixed_div(float d, unsigned long long* counts6, cudaStream_t st);

}  // namespace silt
