// Unit-Gaussian bin integrals shared by the forward raster and the adjoint.
#pragma once

#include <cuda_runtime.h>

namespace wctb200 {

// erfc(z) for z >= 0 by the Chebyshev fit of W. H. Press et al., Numerical
// Recipes (2nd ed.), section 6.2, function erfcc: fractional error below
// 1.2e-7 over the whole range.  The reciprocal is the hardware
// approximation (a few ulp), well inside that; the frame and gradient
// parity tests against the FP64 oracle cover the result.
__device__ __forceinline__ float erfc_nr(float z)
{
    const float t = __fdividef(1.0f, fmaf(0.5f, z, 1.0f));
    float p = 0.17087277f;
    p = fmaf(t, p, -0.82215223f);
    p = fmaf(t, p, 1.48851587f);
    p = fmaf(t, p, -1.13520398f);
    p = fmaf(t, p, 0.27886807f);
    p = fmaf(t, p, -0.18628806f);
    p = fmaf(t, p, 0.09678418f);
    p = fmaf(t, p, 0.37409196f);
    p = fmaf(t, p, 1.00002368f);
    p = fmaf(t, p, -1.26551223f);
    return t * __expf(fmaf(-z, z, p));
}

__device__ __forceinline__ float edge_erfc(float k, float bs, float cr, float inv)
{
    const float x = (k * bs - cr) * inv;
    return copysignf(erfc_nr(fabsf(x)), x);  // sign of x carried on the (non-negative) erfc value
}
__device__ __forceinline__ float bin_from_edges(float a, float b)
{
    const float ea = fabsf(a), eb = fabsf(b);
    const bool na = signbit(a), nb = signbit(b);
    if (!na) return 0.5f * (ea - eb);         // both edges at or above the centre
    if (nb) return 0.5f * (eb - ea);          // both below
    return 0.5f * ((2.0f - ea) - eb);         // bin straddles the centre
}

// Standard normal density.
__device__ __forceinline__ float norm_pdf(float u) { return 0.39894228040143268f * __expf(-0.5f * u * u); }

}  // namespace wctb200
