/*
 * javarand.c -- java.util.Random, restated from the Java SE API specification of
 * the class (a 48-bit linear congruential generator, multiplier 0x5DEECE66D,
 * addend 0xB), so the seeded inputs of the reference's tests are regenerated
 * exactly: e.g. FlipTest.column(new Random(71)) at FlipTest.java:134-150 and
 * ScatterTest.Particles.jittered at ScatterTest.java:460-478.
 *
 * Test infrastructure only (see oracle.h).
 *
 * nextGaussian is the specification's polar method; it calls StrictMath.log and
 * StrictMath.sqrt. sqrt is correctly rounded everywhere; StrictMath.log is fdlibm's
 * __ieee754_log (Sun's published e_log.c), restated below, since the C library's log
 * differs from it in the last bit for some arguments.
 */
#include "oracle.h"
#include <math.h>
#include <string.h>

/* fdlibm __ieee754_log: x = 2^k (1+f), log(1+f) from s = f/(2+f) and a degree-14 odd
 * polynomial in s (coefficients Lg1..Lg7), ln2 split in two parts. */
static double fdlibm_log(double x) {
    static const double ln2_hi = 6.93147180369123816490e-01, ln2_lo = 1.90821492927058770002e-10,
                        two54 = 1.80143985094819840000e+16,
                        Lg1 = 6.666666666666735130e-01, Lg2 = 3.999999999940941908e-01,
                        Lg3 = 2.857142874366239149e-01, Lg4 = 2.222219843214978396e-01,
                        Lg5 = 1.818357216161805012e-01, Lg6 = 1.531383769920937332e-01,
                        Lg7 = 1.479819860511658591e-01;
    uint64_t b;
    memcpy(&b, &x, 8);
    int32_t hx = (int32_t)(b >> 32);
    uint32_t lx = (uint32_t)b;
    int32_t k = 0;
    if (hx < 0x00100000) {
        if (((hx & 0x7fffffff) | lx) == 0) return -INFINITY;
        if (hx < 0) return NAN;
        k -= 54;
        x *= two54;
        memcpy(&b, &x, 8);
        hx = (int32_t)(b >> 32);
    }
    if (hx >= 0x7ff00000) return x + x;
    k += (hx >> 20) - 1023;
    hx &= 0x000fffff;
    int32_t i = (hx + 0x95f64) & 0x100000;
    memcpy(&b, &x, 8);
    b = ((uint64_t)(uint32_t)(hx | (i ^ 0x3ff00000)) << 32) | (b & 0xffffffffULL);
    memcpy(&x, &b, 8);
    k += (i >> 20);
    double f = x - 1.0, dk, R;
    if ((0x000fffff & (2 + hx)) < 3) {
        if (f == 0.0) {
            if (k == 0) return 0.0;
            dk = (double)k;
            return dk * ln2_hi + dk * ln2_lo;
        }
        R = f * f * (0.5 - 0.33333333333333333 * f);
        if (k == 0) return f - R;
        dk = (double)k;
        return dk * ln2_hi - ((R - dk * ln2_lo) - f);
    }
    double s = f / (2.0 + f);
    dk = (double)k;
    double z = s * s;
    i = hx - 0x6147a;
    double w = z * z;
    int32_t j = 0x6b851 - hx;
    double t1 = w * (Lg2 + w * (Lg4 + w * Lg6));
    double t2 = z * (Lg1 + w * (Lg3 + w * (Lg5 + w * Lg7)));
    i |= j;
    R = t2 + t1;
    if (i > 0) {
        double hfsq = 0.5 * f * f;
        if (k == 0) return f - (hfsq - s * (hfsq + R));
        return dk * ln2_hi - ((hfsq - (s * (hfsq + R) + dk * ln2_lo)) - f);
    }
    if (k == 0) return f - s * (f - R);
    return dk * ln2_hi - ((s * (f - R) - dk * ln2_lo) - f);
}

static const int64_t MULT = 0x5DEECE66DLL;
static const int64_t MASK = (1LL << 48) - 1;

void or_jrand_init(or_jrand* r, int64_t seed) {
    r->seed = (seed ^ MULT) & MASK;
    r->have_next_gaussian = 0;
    r->next_gaussian = 0;
}

int32_t or_jrand_next(or_jrand* r, int bits) {
    r->seed = (int64_t)(((uint64_t)r->seed * (uint64_t)MULT + 0xBULL) & (uint64_t)MASK);
    return (int32_t)((uint64_t)r->seed >> (48 - bits));
}

float or_jrand_float(or_jrand* r) {
    return (float)or_jrand_next(r, 24) / (float)(1 << 24);
}

double or_jrand_double(or_jrand* r) {
    int64_t hi = (int64_t)or_jrand_next(r, 26);
    int64_t lo = (int64_t)or_jrand_next(r, 27);
    return (double)((hi << 27) + lo) * (1.0 / (double)(1LL << 53));
}

int32_t or_jrand_int(or_jrand* r, int32_t bound) {
    if (bound <= 0) return 0;
    if ((bound & -bound) == bound) {                 /* a power of two */
        return (int32_t)(((int64_t)bound * (int64_t)or_jrand_next(r, 31)) >> 31);
    }
    int32_t bits, val;
    do {
        bits = or_jrand_next(r, 31);
        val = bits % bound;
    } while ((int32_t)((uint32_t)bits - (uint32_t)val + (uint32_t)(bound - 1)) < 0);
    return val;
}

double or_jrand_gaussian(or_jrand* r) {
    if (r->have_next_gaussian) {
        r->have_next_gaussian = 0;
        return r->next_gaussian;
    }
    double v1, v2, s;
    do {
        v1 = 2 * or_jrand_double(r) - 1;
        v2 = 2 * or_jrand_double(r) - 1;
        s = v1 * v1 + v2 * v2;
    } while (s >= 1 || s == 0);
    double multiplier = sqrt(-2 * fdlibm_log(s) / s);
    r->next_gaussian = v2 * multiplier;
    r->have_next_gaussian = 1;
    return v1 * multiplier;
}

void or_jrand_floats(or_jrand* r, float* out, int64_t n) {
    for (int64_t k = 0; k < n; k++) out[k] = or_jrand_float(r);
}
