// interp_weights.hpp -- the point-sampling weights of the affine and mapim
// interpolators, InterpolationKernel::interpolate (kernel.rs:133-214), for host
// and device.  The host builds per-axis weight tables with these functions for
// the separable walk of an axis-aligned affine; the device evaluates them per
// pixel elsewhere.  Both sides compile without floating-point contraction (fma
// appears only where written), so a table entry equals the device's value.
#pragma once

#include <cmath>

#include "sin_rn.cuh"

namespace viprs {

VIPRS_SIN_HD double bicubic_w(double x) {
    x = fabs(x);
    if (x < 1.0) return fma(2.5 * x, -x, 1.5 * x * x * x) + 1.0;
    if (x < 2.0) return fma(4.0, -x, fma(2.5 * x, x, -0.5 * x * x * x)) + 2.0;
    return 0.0;
}

// The Lanczos sines are rounded to nearest (sin_rn.cuh), as the platform sin
// viprs calls rounds them.
VIPRS_SIN_HD double kernel_w(int k, double x) {
    const double eps = 2.220446049250313e-16;
    const double pi = 3.141592653589793;
    switch (k) {
    case 0: return fabs(x) < 0.5 ? 1.0 : 0.0;
    case 1: x = fabs(x); return x < 1.0 ? 1.0 - x : 0.0;
    case 2: case 7: case 5: return bicubic_w(x);
    case 3:
        x = fabs(x);
        if (x < 0.5) return fma(2.0 * x, -x, 1.0);
        if (x < 1.5) return fma(2.5, -x, x * x) + 1.5;
        return 0.0;
    case 8: {
        x = fabs(x);
        if (x < eps) return 1.0;
        if (x < 2.0) { const double p = pi * x; return 2.0 * sinrn::sin_rn(p) * sinrn::sin_rn(p / 2.0) / (p * p); }
        return 0.0;
    }
    case 9: {
        x = fabs(x);
        if (x < eps) return 1.0;
        if (x < 3.0) { const double p = pi * x; return 3.0 * sinrn::sin_rn(p) * sinrn::sin_rn(p / 3.0) / (p * p); }
        return 0.0;
    }
    default: return 0.0;
    }
}

// Taps per axis of the separable samplers: support 3 for Lanczos3, else 2.
VIPRS_SIN_HD int separable_taps(int k) { return k == 9 ? 6 : 4; }

}  // namespace viprs
