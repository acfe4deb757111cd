/* The library's transcendental functions, identical on host and device.
 *
 * The reference evaluates SIN/COS/EXP with the GLSL builtins (tape/point.comp,
 * tape/interval.comp, tape/gradient.comp), whose precision is left to the
 * driver, so no bit pattern can be matched there. This library instead DEFINES
 * frep_sinf/frep_cosf/frep_expf below and uses them in the CUDA kernels; the
 * CPU oracle includes this header so both sides compute the same bits.
 *
 * Method (published, restated here in my own code):
 *   - argument reduction after Cody & Waite (1980): x = k*(pi/2) + r with pi/2
 *     split into three parts (33 + 33 + 53 significant bits), so k*part is
 *     exact for |k| < 2^20; exp uses x = k*ln2 + r with ln2 split 33 + 53 bits;
 *   - truncated Taylor series on the reduced range (|r| <= pi/4 resp. ln2/2),
 *     evaluated in double precision, then one rounding to float.
 * The double result is within ~3e-14 relative of the true value, so the float
 * result is the correctly rounded value except in near-halfway cases, and is
 * within 1 ulp (the widening the outward interval mode applies) for every
 * finite argument of exp and every |x| < 2^20 of sin / cos (tested against
 * long double on host and device: largest error 0.49999 ulp). For
 * |x| >= 2^20 the sine/cosine reduction first takes fmod(x, 2*pi_double) and
 * loses accuracy but stays in [-1, 1]; the outward intervals use [-1, 1]
 * there.
 *
 * Every operation is a plain IEEE double operation (no FMA: host code is built
 * with -ffp-contract=off, device code with -fmad=false), so results are
 * bit-identical across CPU and GPU.
 */
#ifndef FREP_MATH_H
#define FREP_MATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define FREP_HD __host__ __device__ __forceinline__
#else
#define FREP_HD inline
#endif

namespace frep_math {

FREP_HD double sin_poly(double r) {
    /* r - r^3/3! + r^5/5! - ... - r^15/15!  (Horner in r^2) */
    const double r2 = r * r;
    double p = -0x1.ae7f3e733b81fp-41;          /* -1/15! */
    p = p * r2 + 0x1.6124613a86d09p-33;          /* +1/13! */
    p = p * r2 - 0x1.ae64567f544e4p-26;          /* -1/11! */
    p = p * r2 + 0x1.71de3a556c734p-19;          /* +1/9!  */
    p = p * r2 - 0x1.a01a01a01a01ap-13;          /* -1/7!  */
    p = p * r2 + 0x1.1111111111111p-7;           /* +1/5!  */
    p = p * r2 - 0x1.5555555555555p-3;           /* -1/3!  */
    return r + (r * r2) * p;
}

FREP_HD double cos_poly(double r) {
    /* 1 - r^2/2! + r^4/4! - ... + r^16/16! */
    const double r2 = r * r;
    double p = 0x1.ae7f3e733b81fp-45;            /* +1/16! */
    p = p * r2 - 0x1.93974a8c07c9dp-37;          /* -1/14! */
    p = p * r2 + 0x1.1eed8eff8d898p-29;          /* +1/12! */
    p = p * r2 - 0x1.27e4fb7789f5cp-22;          /* -1/10! */
    p = p * r2 + 0x1.a01a01a01a01ap-16;          /* +1/8!  */
    p = p * r2 - 0x1.6c16c16c16c17p-10;          /* -1/6!  */
    p = p * r2 + 0x1.5555555555555p-5;           /* +1/4!  */
    p = p * r2 - 0x1.0000000000000p-1;           /* -1/2!  */
    return 1.0 + r2 * p;
}

/* Reduces x to r in [-pi/4, pi/4] (approximately) and the quadrant k mod 4. */
FREP_HD double reduce_pio2(double x, int* quadrant) {
    const double two_over_pi = 0x1.45f306dc9c883p-1;
    const double pio2_1 = 0x1.921fb54400000p+0;
    const double pio2_2 = 0x1.0b4611a600000p-34;
    const double pio2_3 = 0x1.3198a2e037073p-69;
    if (fabs(x) >= 1048576.0) {
        x = fmod(x, 0x1.921fb54442d18p+2); /* 2*pi rounded to double */
    }
    const double k = floor(x * two_over_pi + 0.5);
    double r = x - k * pio2_1;
    r = r - k * pio2_2;
    r = r - k * pio2_3;
    const int ki = (int)k;
    *quadrant = ki & 3;
    return r;
}

}  // namespace frep_math

FREP_HD float frep_sinf(float xf) {
    const double x = (double)xf;
    if (!(fabs(x) < INFINITY)) return xf - xf; /* NaN for inf and NaN */
    int q;
    const double r = frep_math::reduce_pio2(x, &q);
    double v;
    switch (q) {
        case 0: v = frep_math::sin_poly(r); break;
        case 1: v = frep_math::cos_poly(r); break;
        case 2: v = -frep_math::sin_poly(r); break;
        default: v = -frep_math::cos_poly(r); break;
    }
    return (float)v;
}

FREP_HD float frep_cosf(float xf) {
    const double x = (double)xf;
    if (!(fabs(x) < INFINITY)) return xf - xf;
    int q;
    const double r = frep_math::reduce_pio2(x, &q);
    double v;
    switch (q) {
        case 0: v = frep_math::cos_poly(r); break;
        case 1: v = -frep_math::sin_poly(r); break;
        case 2: v = -frep_math::cos_poly(r); break;
        default: v = frep_math::sin_poly(r); break;
    }
    return (float)v;
}

FREP_HD float frep_expf(float xf) {
    const double x = (double)xf;
    if (x != x) return xf;                 /* NaN */
    if (x > 128.0) return INFINITY;        /* e^128 overflows float */
    if (x < -150.0) return 0.0f;           /* below half the smallest subnormal */
    const double inv_ln2 = 0x1.71547652b82fep+0;
    const double ln2_1 = 0x1.62e42ff000000p-1;
    const double ln2_2 = -0x1.718432a1b0e26p-35;
    const double k = floor(x * inv_ln2 + 0.5);
    double r = x - k * ln2_1;
    r = r - k * ln2_2;
    /* e^r, |r| <= ln2/2: sum_{i<=12} r^i / i! */
    double p = 0x1.1eed8eff8d898p-29;            /* 1/12! */
    p = p * r + 0x1.ae64567f544e4p-26;           /* 1/11! */
    p = p * r + 0x1.27e4fb7789f5cp-22;           /* 1/10! */
    p = p * r + 0x1.71de3a556c734p-19;           /* 1/9!  */
    p = p * r + 0x1.a01a01a01a01ap-16;           /* 1/8!  */
    p = p * r + 0x1.a01a01a01a01ap-13;           /* 1/7!  */
    p = p * r + 0x1.6c16c16c16c17p-10;           /* 1/6!  */
    p = p * r + 0x1.1111111111111p-7;            /* 1/5!  */
    p = p * r + 0x1.5555555555555p-5;            /* 1/4!  */
    p = p * r + 0x1.5555555555555p-3;            /* 1/3!  */
    p = p * r + 0x1.0000000000000p-1;            /* 1/2!  */
    p = p * r + 1.0;
    p = p * r + 1.0;
    return (float)ldexp(p, (int)k);
}

/* Neighbouring floats by bit manipulation (no rounding-mode dependence). */
FREP_HD float frep_next_up(float x) {
    if (x != x || x == INFINITY) return x;
    if (x == 0.0f) return 1.40129846e-45f; /* smallest positive subnormal */
    uint32_t u;
    memcpy(&u, &x, 4);
    u = (x > 0.0f) ? u + 1 : u - 1;
    memcpy(&x, &u, 4);
    return x;
}

FREP_HD float frep_next_down(float x) { return -frep_next_up(-x); }

#endif /* FREP_MATH_H */
