/*
 * oracle/refmath.h -- TEST INFRASTRUCTURE ONLY (the oracle's CPU math).
 *
 * CPU versions of the single-precision math functions that the reference RCA
 * kernel calls (MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.cu:79-98,
 * 258-268, 299, 308, 319, 329-380).  Each one is evaluated in double precision
 * from its mathematical definition and rounded once to float, so the results
 * are the correctly rounded value in all but rare double-rounding cases.  They
 * are NOT NVIDIA's implementations (whose steps are not reproduced here); the
 * GPU reference build calls CUDA's own functions instead.
 *
 * Used by two things only:
 *   - oracle/ref_shim.h, which compiles the reference kernel source as C++;
 *   - oracle/rca_oracle.c, the plain-C restatement of the same arithmetic.
 * Both therefore see identical transcendental values, which lets the
 * restatement be checked bit-for-bit against the reference kernel on the CPU.
 */
#ifndef RCABF_ORACLE_REFMATH_H
#define RCABF_ORACLE_REFMATH_H

#include <math.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define RM_INLINE static inline

/* Exact reduction of x to r in [-1, 1] with x = r + 2k (k integer).  For
 * |x| >= 2^23 every float is an even integer or odd integer; those return the
 * exact zero/one pattern of sin(pi x). */
RM_INLINE double rm_reduce_pi(float x, int *exact_int)
{
    double d = (double)x;
    double k = nearbyint(d * 0.5);
    double r = d - 2.0 * k; /* exact in double: |d| < 2^128, r in [-1, 1] */
    *exact_int = (r == floor(r));
    return r;
}

/* sin(pi x), float in / float out (CUDA name: sinpif, also sinpi(float)). */
RM_INLINE float rm_sinpif(float x)
{
    int is_int;
    double r = rm_reduce_pi(x, &is_int);
    if (is_int) {
        /* sin(pi * integer) is an exact zero carrying the sign of x. */
        return copysignf(0.0f, x);
    }
    double a = fabs(r);
    double s = (a > 0.5) ? sin(M_PI * (1.0 - a)) : sin(M_PI * a);
    return (float)(r < 0 ? -s : s);
}

/* cos(pi x), float in / float out (CUDA name: cospif). */
RM_INLINE float rm_cospif(float x)
{
    int is_int;
    double r = rm_reduce_pi(x, &is_int);
    double a = fabs(r);
    if (a == 0.5) return 0.0f;
    if (is_int) return (a == 0.0) ? 1.0f : -1.0f;
    double c = (a < 0.5) ? sin(M_PI * (0.5 - a)) : -sin(M_PI * (a - 0.5));
    return (float)c;
}

/* a / b for the reference's fdividef: correctly rounded quotient. */
RM_INLINE float rm_fdividef(float a, float b) { return (float)((double)a / (double)b); }

/* sqrt(a^2 + b^2 + c^2): squares are exact in double. */
RM_INLINE float rm_norm3df(float a, float b, float c)
{
    double da = a, db = b, dc = c;
    return (float)sqrt(da * da + db * db + dc * dc);
}

/* sqrt(a^2 + b^2). */
RM_INLINE float rm_hypotf(float a, float b)
{
    double da = a, db = b;
    return (float)sqrt(da * da + db * db);
}

/* cos / sin of a float argument, evaluated in double (libm's double
 * functions reduce the argument exactly). */
RM_INLINE float rm_cosf(float x) { return (float)cos((double)x); }
RM_INLINE float rm_sinf(float x) { return (float)sin((double)x); }
RM_INLINE float rm_acosf(float x) { return (float)acos((double)x); }

/* exp, asin, atan2, sqrt, fabs of float arguments, evaluated in double
 * (the simulator kernels, SimUS_CUDARCA.cu). */
RM_INLINE float rm_expf(float x) { return (float)exp((double)x); }
RM_INLINE float rm_asinf(float x) { return (float)asin((double)x); }
RM_INLINE float rm_atan2f(float y, float x) { return (float)atan2((double)y, (double)x); }
RM_INLINE float rm_sqrtf(float x) { return (float)sqrt((double)x); }
RM_INLINE float rm_fabsf(float x) { return fabsf(x); }

/* 1 / sqrt(x) in double (the reference passes a double argument). */
RM_INLINE double rm_rsqrt(double x) { return 1.0 / sqrt(x); }

#endif /* RCABF_ORACLE_REFMATH_H */
