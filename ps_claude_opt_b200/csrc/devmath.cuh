// devmath.cuh -- small device math helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>

namespace psb {

// 1/d without special-case branches, for finite normal d: the PTX
// rcp.approx.ftz.f64 estimate refined by two Newton-Raphson steps for the
// reciprocal, r <- r + r (1 - d r), each of which doubles the number of
// correct bits.  The facet terms only ever see d = mu + mu0 in (2e-8, 2] or
// the stand-in 1.  Agrees with the correctly rounded 1.0 / d to within one
// unit in the last place (checked by the test suite).
__device__ __forceinline__ double rcp_nr(double d)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}

}  // namespace psb
