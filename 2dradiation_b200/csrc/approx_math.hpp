// Polynomial trigonometry of the reference (src/Utility.hh:128-471), usable
// from host and device code.  The reference evaluates its stencil directions,
// rotations and departure angles with these approximations instead of libm;
// the departure-angle computation of the curved stream must see the same
// values, so they are restated here with the same coefficients (published in
// Hastings, "Approximations for Digital Computers", 1955, as the reference
// notes) and the same argument reductions.
#pragma once
#include <cmath>
#include <cstdlib>

#ifdef __CUDACC__
#define GRLBM_HD __host__ __device__ __forceinline__
#else
#define GRLBM_HD inline
#endif

namespace grlbm
{
constexpr double kPi = 3.14159265358979323846;
constexpr double kHalfPi = 1.57079632679489661923;

// MyAtan<9>: odd polynomial on [-1, 1] (src/Utility.hh:179-188)
GRLBM_HD double atan_poly9(double z)
{
    const double zz = z * z;
    return z * (0.9998660 + zz * (-0.3302995 + zz * (0.1801410 + zz * (-0.0851330 + zz * 0.0208351))));
}

// MyAtan2<9> (src/Utility.hh:220-254): the octant test compares |x| and |y|
// after rounding both to float, as the reference's fabsf calls do.
GRLBM_HD double approx_atan2(double y, double x)
{
    if (x != 0.0)
    {
        if (fabsf((float)x) > fabsf((float)y))
        {
            const double z = y / x;
            if (x > 0.0)
                return atan_poly9(z);
            return (y >= 0.0) ? atan_poly9(z) + kPi : atan_poly9(z) - kPi;
        }
        const double z = x / y;
        return (y > 0.0) ? -atan_poly9(z) + kHalfPi : -atan_poly9(z) - kHalfPi;
    }
    if (y > 0.0)
        return kHalfPi;
    if (y < 0.0)
        return -kHalfPi;
    return 0.0;
}

// Tensor2::Phi (src/DataTypes.hh:166-170): angle in [0, 2 pi)
GRLBM_HD double approx_phi(double x, double y)
{
    const double p = approx_atan2(y, x);
    return (p < 0) ? p + 2.0 * kPi : p;
}

// MySin<9> on [-pi/2, 5 pi/2] (src/Utility.hh:272-323).  Outside that range
// the reference aborts; this returns NaN and callers check.
GRLBM_HD double approx_sin(double x)
{
    if (-kHalfPi <= x && x <= kHalfPi)
    {
    }
    else if (kHalfPi <= x && x <= 3.0 * kHalfPi)
        x = -(x - kPi);
    else if (3.0 * kHalfPi <= x && x <= 5.0 * kHalfPi)
        x = x - 2.0 * kPi;
    else
        return NAN;
    x *= 2.0 / kPi;
    const double xx = x * x;
    return x * (1.57079631847 + xx * (-0.64596371106 + xx * (0.07968967928 + xx * (-0.00467376557 + xx * 0.00015148419))));
}

// MyCos: float argument, float result (src/Utility.hh:340-360).
GRLBM_HD double approx_cos(double xd)
{
    const float x = (float)xd;
    const float pi = (float)kPi;
    const float half = (float)kHalfPi;
    if (x >= pi)
        return (double)(float)(-approx_sin((double)(x - half)));
    return (double)(float)approx_sin((double)(x + half));
}

// MyAcos (src/Utility.hh:453-471) over MyAsin<4> (:366-395).  In the
// reference MyAsin's unqualified abs() resolves to the C library's
// int abs(int), so its argument is truncated to an integer first; this keeps
// that behaviour because the flux look-up table is built on it.
inline double approx_acos(double xd)
{
    auto asin4 = [](double x) {
        const double sign = (double)((0.0 < x) - (x < 0.0));
        x = (double)std::abs((int)x);
        const double p = 1.57078786 + x * (-0.21412453 + x * (0.08466649 + x * (-0.03575663 + x * 0.00864884)));
        return sign * (kHalfPi - std::sqrt(1.0 - x) * p);
    };
    const float x = (float)xd;
    const float r = (x >= 0) ? (float)(kHalfPi - asin4((double)x)) : (float)(kHalfPi + asin4((double)(-x)));
    return (double)r;
}
} // namespace grlbm
