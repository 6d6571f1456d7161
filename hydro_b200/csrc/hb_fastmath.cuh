// hb_fastmath.cuh -- FP64 reciprocal and reciprocal square root from the
// hardware approximations, for the stage sets that do not need IEEE-rounded
// division and square root (the mixed-precision and the FMA FP64 sets).
#pragma once

#include <cuda_runtime.h>

namespace hb {

// Reciprocal and reciprocal square root in FP64: the hardware approximation
// (PTX rcp.approx.ftz.f64 / rsqrt.approx.ftz.f64) refined by two
// Newton-Raphson steps, each of which doubles the number of correct bits, to
// the FP64 rounding level.  Inputs are positive normal numbers (every
// divisor and radicand of a valid state is).
__device__ __forceinline__ double rcp64(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

__device__ __forceinline__ double rsqrt64(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double h = 0.5 * y;
    double r = fma(-(x * y), h, 0.5);  // 1/2 - x y^2 / 2
    y = fma(y, r, y);
    h = 0.5 * y;
    r = fma(-(x * y), h, 0.5);
    return fma(y, r, y);
}

}  // namespace hb
