/*
 * sfb200_sphmath.h -- bit-reproducible FP64 transcendentals for the spherical pair path.
 *
 * The reference evaluates `sincosd` (degrees) in unit_position / local_east_north
 * (src/HelperFunctions.jl:133-153, 404-409), `sincos` (radians) for SphericalAngle, and
 * `atan(y, x)` in geodesic_frame (src/HelperFunctions.jl:196). Those come from Julia's own libm,
 * which is not available here, and CUDA's and glibc's versions differ from each other in the last
 * ulp. A pair whose separation sits within an ulp of a bin edge would then land in different bins
 * on the GPU and on the CPU check. To make the distance bin a deterministic function of the inputs,
 * this header implements the three functions once, from textbook methods, using only IEEE-exact
 * operations (+, -, *, /, sqrt, fma, fmod, rint) written through the SFB_* macros below. The same
 * source compiles for the host (C, -ffp-contract=off) and the device (explicit __d*_rn intrinsics),
 * so both produce identical bits.
 *
 * Methods (accuracy checked against 300-bit mpmath in the test suite, <= 1.5 ulp):
 *   sincosd: exact reduction of the angle modulo 360 and to [-45, 45] degrees (exact in binary64),
 *            conversion to radians with a double-double pi/180, Taylor series to degree 19 (sin) and
 *            18 (cos) on |y| <= pi/4 with first-order correction for the low word.
 *   sincos:  three-part Cody-Waite reduction by pi/2 (exact products for |x| < 2^19 pi/2), same
 *            kernels.
 *   atan2:   for y, x >= 0: t = min/max, k = rint(8 t), s = (a - c_k b) / (b + c_k a) with
 *            c_k = k/8, atan(t) = atan(c_k) + atan(s), |s| <= 1/16, Taylor series to s^17;
 *            atan(c_k) stored as double-double (computed with mpmath). Other quadrants by symmetry.
 * Constants are exact binary64 hex literals (Taylor coefficients (-1)^n/(2n+1)!, 1/(2n+1);
 * atan(k/8), pi/180, pi/2 rounded from 300-bit values).
 */
#ifndef SFB200_SPHMATH_H
#define SFB200_SPHMATH_H

#ifdef __CUDACC__
#define SFB_HD __host__ __device__ __forceinline__
#else
#define SFB_HD static inline
#include <math.h>
#endif

#if defined(__CUDA_ARCH__)
#define SFB_ADD(a, b) __dadd_rn((a), (b))
#define SFB_SUB(a, b) __dsub_rn((a), (b))
#define SFB_MUL(a, b) __dmul_rn((a), (b))
#define SFB_DIV(a, b) __ddiv_rn((a), (b))
#define SFB_FMA(a, b, c) __fma_rn((a), (b), (c))
#define SFB_SQRT(a) __dsqrt_rn(a)
#else
#define SFB_ADD(a, b) ((a) + (b))
#define SFB_SUB(a, b) ((a) - (b))
#define SFB_MUL(a, b) ((a) * (b))
#define SFB_DIV(a, b) ((a) / (b))
#define SFB_FMA(a, b, c) fma((a), (b), (c))
#define SFB_SQRT(a) sqrt(a)
#endif

/* sin and cos of y = yh + yl, |y| <= pi/4 (+ tiny). */
SFB_HD void sfb_sincos_kernel(double yh, double yl, double* s, double* c)
{
    const double z = SFB_MUL(yh, yh);
    /* sin: yh + (yh^3 P(z) + yl (1 - z/2)),  P = sum_{n>=1} (-1)^n z^(n-1) / (2n+1)! */
    double p = -0x1.2f49b46814157p-57;
    p = SFB_FMA(p, z, 0x1.952c77030ad4ap-49);
    p = SFB_FMA(p, z, -0x1.ae7f3e733b81fp-41);
    p = SFB_FMA(p, z, 0x1.6124613a86d09p-33);
    p = SFB_FMA(p, z, -0x1.ae64567f544e4p-26);
    p = SFB_FMA(p, z, 0x1.71de3a556c734p-19);
    p = SFB_FMA(p, z, -0x1.a01a01a01a01ap-13);
    p = SFB_FMA(p, z, 0x1.1111111111111p-7);
    p = SFB_FMA(p, z, -0x1.5555555555555p-3);
    const double v = SFB_MUL(z, yh);
    const double corr = SFB_MUL(yl, SFB_FMA(-0.5, z, 1.0));
    *s = SFB_ADD(yh, SFB_FMA(v, p, corr));
    /* cos: 1 - z/2 + z^2 Q(z) - yh*yl, evaluated as w + ((1 - w) - hz + (z^2 Q - yh yl)) */
    double q = -0x1.6827863b97d97p-53;
    q = SFB_FMA(q, z, 0x1.ae7f3e733b81fp-45);
    q = SFB_FMA(q, z, -0x1.93974a8c07c9dp-37);
    q = SFB_FMA(q, z, 0x1.1eed8eff8d898p-29);
    q = SFB_FMA(q, z, -0x1.27e4fb7789f5cp-22);
    q = SFB_FMA(q, z, 0x1.a01a01a01a01ap-16);
    q = SFB_FMA(q, z, -0x1.6c16c16c16c17p-10);
    q = SFB_FMA(q, z, 0x1.5555555555555p-5);
    const double hz = SFB_MUL(0.5, z);
    const double w = SFB_SUB(1.0, hz);
    const double tail = SFB_SUB(SFB_MUL(SFB_MUL(z, z), q), SFB_MUL(yh, yl));
    *c = SFB_ADD(w, SFB_ADD(SFB_SUB(SFB_SUB(1.0, w), hz), tail));
}

/* Place the kernel results in quadrant k (angle = k*90deg + y). */
SFB_HD void sfb_sincos_quadrant(int k, double sy, double cy, double* s, double* c)
{
    switch (k & 3) {
    case 0: *s = sy;  *c = cy;  break;
    case 1: *s = cy;  *c = -sy; break;
    case 2: *s = -sy; *c = -cy; break;
    default: *s = -cy; *c = sy; break;
    }
}

/* sin and cos of an angle in degrees (the angle unit of Distances.Haversine coordinates). */
SFB_HD void sfb_sincosd(double x, double* s, double* c)
{
    if (!(x - x == 0.0)) { /* inf or NaN */
        const double nan = x - x;
        *s = nan; *c = nan;
        return;
    }
    const double r = fmod(x, 360.0);              /* exact */
    const double q = rint(SFB_DIV(r, 90.0));      /* nearest quadrant, |q| <= 4 */
    const double y = SFB_SUB(r, SFB_MUL(q, 90.0)); /* exact: |y| <= 45 and |y| <= |r| */
    const double P_HI = 0x1.1df46a2529d39p-6, P_LO = 0x1.5c1d8becdd291p-62; /* pi/180 */
    const double yh = SFB_MUL(y, P_HI);
    const double yl = SFB_FMA(y, P_LO, SFB_FMA(y, P_HI, -yh));
    double sy, cy;
    sfb_sincos_kernel(yh, yl, &sy, &cy);
    if (y == 0.0) { sy = 0.0; cy = 1.0; }          /* multiples of 90 degrees are exact */
    sfb_sincos_quadrant((int)q, sy, cy, s, c);
    if (*s == 0.0) *s = 0.0 * x;                  /* signed zero follows the input, like sind */
    if (*c == 0.0) *c = 0.0;                      /* cosd of an odd multiple of 90 is +0 */
}

/* sin and cos of an angle in radians (Distances.SphericalAngle coordinates). Accurate for
 * |x| < 2^19 * pi/2; the sphere path only sees longitudes and latitudes. */
SFB_HD void sfb_sincos(double x, double* s, double* c)
{
    if (!(x - x == 0.0)) {
        const double nan = x - x;
        *s = nan; *c = nan;
        return;
    }
    const double k = rint(SFB_MUL(x, 0x1.45f306dc9c883p-1)); /* x * 2/pi */
    const double P1 = 0x1.921fb54400000p+0, P2 = 0x1.0b4611a600000p-34, P3 = 0x1.3198a2e037073p-69;
    const double w = SFB_FMA(-k, P1, x);           /* exact for |k| < 2^20 */
    const double t = SFB_MUL(k, P2);               /* exact */
    const double yh = SFB_SUB(w, t);
    const double yl = SFB_FMA(-k, P3, SFB_SUB(SFB_SUB(w, yh), t));
    double sy, cy;
    sfb_sincos_kernel(yh, yl, &sy, &cy);
    sfb_sincos_quadrant((int)(long long)k, sy, cy, s, c);
}

/* atan(s) for |s| <= 1/16 + tiny, returned as s + s^3 Q(s^2) (without the leading term). */
SFB_HD double sfb_atan_tail(double s)
{
    const double z = SFB_MUL(s, s);
    double q = 0x1.e1e1e1e1e1e1ep-5;
    q = SFB_FMA(q, z, -0x1.1111111111111p-4);
    q = SFB_FMA(q, z, 0x1.3b13b13b13b14p-4);
    q = SFB_FMA(q, z, -0x1.745d1745d1746p-4);
    q = SFB_FMA(q, z, 0x1.c71c71c71c71cp-4);
    q = SFB_FMA(q, z, -0x1.2492492492492p-3);
    q = SFB_FMA(q, z, 0x1.999999999999ap-3);
    q = SFB_FMA(q, z, -0x1.5555555555555p-2);
    return SFB_MUL(SFB_MUL(s, z), q);
}

/* atan2(y, x) for finite y >= 0, x >= 0 (the only quadrant geodesic_frame uses: both arguments
 * are square roots). atan2(0, 0) = 0 as in Julia. */
SFB_HD double sfb_atan2_pos(double y, double x)
{
    if (y != y || x != x) return y + x;
    if (y == 0.0) return 0.0;
    if (x == 0.0) return 0x1.921fb54442d18p+0;
    const int swap = y > x;
    const double a = swap ? x : y;
    const double b = swap ? y : x;
    const double t = SFB_DIV(a, b);                /* in [0, 1] */
    const int k = (int)rint(SFB_MUL(t, 8.0));
    double hi, lo, s;
    switch (k) {
    case 0: hi = 0.0; lo = 0.0; break;
    case 1: hi = 0x1.fd5ba9aac2f6ep-4; lo = -0x1.cd37686760c17p-59; break;
    case 2: hi = 0x1.f5b75f92c80ddp-3; lo = 0x1.8ab6e3cf7afbdp-57; break;
    case 3: hi = 0x1.6f61941e4def1p-2; lo = -0x1.c63aae6f6e918p-56; break;
    case 4: hi = 0x1.dac670561bb4fp-2; lo = 0x1.a2b7f222f65e2p-56; break;
    case 5: hi = 0x1.1e00babdefeb4p-1; lo = -0x1.928df287a668fp-58; break;
    case 6: hi = 0x1.4978fa3269ee1p-1; lo = 0x1.2419a87f2a458p-56; break;
    case 7: hi = 0x1.700a7c5784634p-1; lo = -0x1.8c34d25aadef6p-56; break;
    default: hi = 0x1.921fb54442d18p-1; lo = 0x1.1a62633145c07p-55; break;
    }
    if (k == 0) {
        s = t;
    } else {
        const double ck = SFB_MUL((double)k, 0.125);
        s = SFB_DIV(SFB_FMA(-ck, b, a), SFB_FMA(ck, a, b));
    }
    double res = SFB_ADD(hi, SFB_ADD(s, SFB_ADD(lo, sfb_atan_tail(s))));
    if (swap) {
        res = SFB_ADD(SFB_SUB(0x1.921fb54442d18p+0, res), 0x1.1a62633145c07p-54);
    }
    return res;
}

/* General atan2 by symmetry (used only by tests of this header). */
SFB_HD double sfb_atan2(double y, double x)
{
    if (y != y || x != x) return y + x;
    const double ay = y < 0.0 ? -y : y;
    const double ax = x < 0.0 ? -x : x;
    double r = sfb_atan2_pos(ay, ax);
    if (x < 0.0 || (x == 0.0 && 1.0 / x < 0.0)) {
        r = SFB_ADD(SFB_SUB(0x1.921fb54442d18p+1, r), 0x1.1a62633145c07p-53);
    }
    return (y < 0.0 || (y == 0.0 && 1.0 / y < 0.0)) ? -r : r;
}

#endif /* SFB200_SPHMATH_H */
