/*
 * orc_math.h -- host stand-ins for the CUDA device math that the reference's update rules call
 * (rsqrt, cospi, sinpi).  TEST INFRASTRUCTURE ONLY.
 *
 * The reference calls rsqrt (algorithms/OrUpdate.hxx:72, SaUpdate.hxx:109, SrUpdate.hxx:88,
 * GaugeFixingSubgroupStep.hxx:333,566, Quaternion.hxx:222) and cospi/sinpi
 * (algorithms/SaUpdate.hxx:119-133, RandomUpdate.hxx:50-58).  Host C has none of them, so both
 * the C oracle (gf_oracle.c) and the build of the reference's own templates (ref_pin.cpp) use
 * these definitions; that keeps the two bit-identical.  cospi/sinpi reduce the argument
 * exactly (x - 2*round(x/2) is exact in binary floating point) and then call cos/sin of pi*r.
 */
#ifndef ORC_MATH_H
#define ORC_MATH_H

#include <math.h>

#define ORC_PI 3.14159265358979323846

static inline double orc_rsqrt_d(double x) { return 1.0 / sqrt(x); }
static inline float orc_rsqrt_f(float x) { return 1.0f / sqrtf(x); }

static inline double orc_cospi_d(double x)
{
    double r = x - 2.0 * nearbyint(0.5 * x); /* r in [-1, 1] */
    if (r == 0.5 || r == -0.5) return 0.0;
    return cos(ORC_PI * r);
}

static inline double orc_sinpi_d(double x)
{
    double r = x - 2.0 * nearbyint(0.5 * x);
    if (r == 1.0 || r == -1.0 || r == 0.0) return 0.0 * r;
    return sin(ORC_PI * r);
}

static inline float orc_cospi_f(float x) { return (float)orc_cospi_d((double)x); }
static inline float orc_sinpi_f(float x) { return (float)orc_sinpi_d((double)x); }

#endif
