/*
 * gprm_sincos64.h - double-precision sin/cos shared by the CUDA kernels and
 * the CPU oracle, so that the FP64 band recheck is bit-reproducible on both.
 *
 * Method: Cody-Waite argument reduction by pi/2 with a three-part split of
 * pi/2 (each part holds 32 significant bits, so k*P1 and k*P2 are exact for
 * |k| < 2^21), then the Taylor series of sin and cos on |r| <= pi/4
 * evaluated by Horner's rule in r^2.  The truncation error of the series
 * (first omitted terms r^25/25! and r^24/24!) is below 1e-27, far under
 * half an ulp; rounding gives about 1-2 ulp, which the tests bound against
 * libm.  The coefficients are 1/n! rounded to double, written as exact
 * hexadecimal literals.  Every operation is a plain IEEE add or multiply and
 * the translation units that include this header are compiled without FMA
 * contraction, so the host and the device produce identical bits.
 *
 * Valid for |x| < 2^20 * pi/2; joint angles are far inside that range.  NaN
 * and infinities propagate as NaN.
 */
#ifndef GPRM_SINCOS64_H
#define GPRM_SINCOS64_H

#ifdef __CUDACC__
#define GPRM_HD __host__ __device__ __forceinline__
#else
#define GPRM_HD static inline
#include <math.h>
#endif

/* 2/pi rounded to double */
#define GPRM_TWO_OVER_PI  0x1.45f306dc9c883p-1
/* pi/2 = P1 + P2 + P3 (+ < 2^-100) */
#define GPRM_PIO2_P1      0x1.921fb544p+0
#define GPRM_PIO2_P2      0x1.0b4611a6p-34
#define GPRM_PIO2_P3      0x1.3198a2e037073p-69

GPRM_HD void gprm_sincos64(double x, double* s_out, double* c_out)
{
    double k = x * GPRM_TWO_OVER_PI;
#ifdef __CUDA_ARCH__
    k = rint(k);
#else
    k = nearbyint(k);
#endif
    double r = x - k * GPRM_PIO2_P1;
    r = r - k * GPRM_PIO2_P2;
    r = r - k * GPRM_PIO2_P3;
    double r2 = r * r;
    /* sin r = r + r*r2*ps, ps = -1/3! + r2/5! - ... + r2^10/23! */
    double ps = -0x1.761b41316381ap-75;         /* -1/23! */
    ps = ps * r2 + 0x1.71b8ef6dcf572p-66;       /*  1/21! */
    ps = ps * r2 + -0x1.2f49b46814157p-57;      /* -1/19! */
    ps = ps * r2 + 0x1.952c77030ad4ap-49;       /*  1/17! */
    ps = ps * r2 + -0x1.ae7f3e733b81fp-41;      /* -1/15! */
    ps = ps * r2 + 0x1.6124613a86d09p-33;       /*  1/13! */
    ps = ps * r2 + -0x1.ae64567f544e4p-26;      /* -1/11! */
    ps = ps * r2 + 0x1.71de3a556c734p-19;       /*  1/9!  */
    ps = ps * r2 + -0x1.a01a01a01a01ap-13;      /* -1/7!  */
    ps = ps * r2 + 0x1.1111111111111p-7;        /*  1/5!  */
    ps = ps * r2 + -0x1.5555555555555p-3;       /* -1/3!  */
    double sr = r + r * (r2 * ps);
    /* cos r = 1 - r2/2 + r2^2*pc, pc = 1/4! - r2/6! + ... - r2^9/22! */
    double pc = -0x1.0ce396db7f853p-70;         /* -1/22! */
    pc = pc * r2 + 0x1.e542ba4020225p-62;       /*  1/20! */
    pc = pc * r2 + -0x1.6827863b97d97p-53;      /* -1/18! */
    pc = pc * r2 + 0x1.ae7f3e733b81fp-45;       /*  1/16! */
    pc = pc * r2 + -0x1.93974a8c07c9dp-37;      /* -1/14! */
    pc = pc * r2 + 0x1.1eed8eff8d898p-29;       /*  1/12! */
    pc = pc * r2 + -0x1.27e4fb7789f5cp-22;      /* -1/10! */
    pc = pc * r2 + 0x1.a01a01a01a01ap-16;       /*  1/8!  */
    pc = pc * r2 + -0x1.6c16c16c16c17p-10;      /* -1/6!  */
    pc = pc * r2 + 0x1.5555555555555p-5;        /*  1/4!  */
    double cr = 1.0 - 0.5 * r2 + r2 * r2 * pc;
    /* NaN/inf arguments give NaN in sr and cr; pick quadrant 0 for them so
     * the integer conversion below is always defined. */
    double kq = (k == k && k < 4.0e15 && k > -4.0e15) ? k : 0.0;
    long long q = (long long)kq;
    int quad = (int)(q & 3);
    double s, c;
    if (quad == 0)      { s = sr;  c = cr;  }
    else if (quad == 1) { s = cr;  c = -sr; }
    else if (quad == 2) { s = -sr; c = -cr; }
    else                { s = -cr; c = sr;  }
    *s_out = s;
    *c_out = c;
}

#endif /* GPRM_SINCOS64_H */
