// Reproducible transcendental functions for the renderer's float arithmetic.
//
// The renderer's branch decisions (which triangle a ray hits, which child an
// edge-tree walk picks, whether a line sample survives its tests) depend on
// the last bits of sines, cosines, arc tangents and powers.  CUDA's math
// library and the host's libm each round those differently, so a GPU render
// and a CPU render of the same sample could take different branches.  These
// functions give the same bits on both: each evaluates in IEEE double
// precision with additions, subtractions, multiplications, divisions and
// square roots only, every one rounded to nearest and none fused (explicit
// __d*_rn intrinsics on the device; on the host the translation units that use
// this header are compiled with -ffp-contract=off), in a fixed order, and
// rounds the double result to float once.
//
// Methods (textbook ones, with coefficients that are exact Taylor
// coefficients rounded to double):
//   log  x = 2^k m, m in [sqrt(1/2), sqrt(2)]; log m = 2 atanh(s),
//        s = (m - 1) / (m + 1), |s| <= 0.172, series to s^21.
//   exp  x = k ln2 + r, |r| <= ln2 / 2 (Cody-Waite: ln2 split into a 33-bit
//        head and a tail), Taylor series to r^13, then times 2^k.
//   pow  exp(y log x) for x > 0; integer y for x < 0.
//   atan table reduction atan x = k pi/32 + atan((x - c) / (1 + x c)),
//        c = tan(k pi/32), |t| <= tan(pi/64); series to t^15.
//   atan2, acos  from atan (acos x = 2 atan(sqrt((1 - x) / (1 + x)))).
//   sin, cos  x = k pi/2 + r (Cody-Waite, 33-bit head of pi/2), |r| <= pi/4,
//        Taylor series to r^17 / r^16; meant for |x| < 2^20.
// Before the final rounding the relative error is a few units of 2^-52, so
// the float results are the correctly rounded values except when the exact
// value lies within ~1e-15 (relative) of a rounding boundary of float.
#pragma once

#include <stdint.h>
#include <cstring>

#if defined(__CUDACC__)
#define DRM_FN __host__ __device__ __forceinline__
#else
#define DRM_FN inline
#endif

namespace drm {

#ifdef __CUDA_ARCH__
DRM_FN double add(double a, double b) { return __dadd_rn(a, b); }
DRM_FN double sub(double a, double b) { return __dsub_rn(a, b); }
DRM_FN double mul(double a, double b) { return __dmul_rn(a, b); }
DRM_FN double div(double a, double b) { return __ddiv_rn(a, b); }
DRM_FN double root(double a) { return __dsqrt_rn(a); }
DRM_FN int64_t bits(double a) { return __double_as_longlong(a); }
DRM_FN double from_bits(int64_t b) { return __longlong_as_double(b); }
#else
DRM_FN double add(double a, double b) { return a + b; }
DRM_FN double sub(double a, double b) { return a - b; }
DRM_FN double mul(double a, double b) { return a * b; }
DRM_FN double div(double a, double b) { return a / b; }
DRM_FN double root(double a) { return __builtin_sqrt(a); }
DRM_FN int64_t bits(double a) {
    int64_t b;
    std::memcpy(&b, &a, 8);
    return b;
}
DRM_FN double from_bits(int64_t b) {
    double a;
    std::memcpy(&a, &b, 8);
    return a;
}
#endif

constexpr double kPi = 3.141592653589793;
constexpr double kPio2 = 1.5707963267948966;
constexpr double kPio2Hi = 1.5707963267341256;   // 33 significant bits: k * kPio2Hi is exact for |k| < 2^20
constexpr double kPio2Lo = 6.077100506506192e-11;  // pi/2 - kPio2Hi
constexpr double kTwoOverPi = 0.6366197723675814;
constexpr double kLn2 = 0.6931471805599453;
constexpr double kLn2Hi = 0.6931471804855391;    // 33 significant bits
constexpr double kLn2Lo = 7.440617110012397e-11;   // ln 2 - kLn2Hi
constexpr double kInvLn2 = 1.4426950408889634;
constexpr double kSqrt2 = 1.4142135623730951;
constexpr double kInf = __builtin_huge_val();

DRM_FN bool is_nan(double x) { return x != x; }
DRM_FN double absd(double x) { return from_bits(bits(x) & 0x7fffffffffffffffLL); }
DRM_FN bool sign_bit(double x) { return bits(x) < 0; }
// nearest integer (ties to even) of |x| < 2^51, exactly
DRM_FN double round_int(double x) {
    const double big = 6755399441055744.0;  // 1.5 * 2^52
    return sub(add(x, big), big);
}
// 2^k for -2044 <= k <= 2046, as two exact powers of two
DRM_FN double scale2(double v, int k) {
    int k1 = k / 2, k2 = k - k1;
    v = mul(v, from_bits((int64_t)(k1 + 1023) << 52));
    return mul(v, from_bits((int64_t)(k2 + 1023) << 52));
}

// natural logarithm of a double
DRM_FN double log_d(double x) {
    if (is_nan(x) || x < 0.0) return kInf - kInf;
    if (x == 0.0) return -kInf;
    if (x == kInf) return kInf;
    int64_t b = bits(x);
    int e = (int)((b >> 52) & 0x7ff);
    int k = 0;
    if (e == 0) {  // subnormal: scale by 2^54 first
        x = mul(x, 18014398509481984.0);
        b = bits(x);
        e = (int)((b >> 52) & 0x7ff);
        k = -54;
    }
    k += e - 1023;
    double m = from_bits((b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);  // [1, 2)
    if (m > kSqrt2) {
        m = mul(m, 0.5);
        k += 1;
    }
    double s = div(sub(m, 1.0), add(m, 1.0));
    double z = mul(s, s);
    double p = 0.047619047619047616;
    p = add(mul(p, z), 0.05263157894736842);
    p = add(mul(p, z), 0.058823529411764705);
    p = add(mul(p, z), 0.06666666666666667);
    p = add(mul(p, z), 0.07692307692307693);
    p = add(mul(p, z), 0.09090909090909091);
    p = add(mul(p, z), 0.1111111111111111);
    p = add(mul(p, z), 0.14285714285714285);
    p = add(mul(p, z), 0.2);
    p = add(mul(p, z), 0.3333333333333333);
    p = add(mul(p, z), 1.0);
    double lm = mul(2.0, mul(s, p));
    double dk = (double)k;
    return add(add(mul(dk, kLn2Hi), lm), mul(dk, kLn2Lo));
}

// e^x of a double
DRM_FN double exp_d(double x) {
    if (is_nan(x)) return x;
    if (x > 709.0) return kInf;
    if (x < -745.5) return 0.0;
    double k = round_int(mul(x, kInvLn2));
    double r = sub(sub(x, mul(k, kLn2Hi)), mul(k, kLn2Lo));
    double p = 1.6059043836821613e-10;
    p = add(mul(p, r), 2.08767569878681e-09);
    p = add(mul(p, r), 2.505210838544172e-08);
    p = add(mul(p, r), 2.755731922398589e-07);
    p = add(mul(p, r), 2.7557319223985893e-06);
    p = add(mul(p, r), 2.48015873015873e-05);
    p = add(mul(p, r), 0.0001984126984126984);
    p = add(mul(p, r), 0.001388888888888889);
    p = add(mul(p, r), 0.008333333333333333);
    p = add(mul(p, r), 0.041666666666666664);
    p = add(mul(p, r), 0.16666666666666666);
    p = add(mul(p, r), 0.5);
    p = add(mul(p, r), 1.0);
    p = add(mul(p, r), 1.0);
    return scale2(p, (int)k);
}

// Tables of the arc tangent's argument reduction: c_k = tan(k pi/32) and
// k pi/32, k = 0..15, rounded to double.
#define DRM_ATAN_C {0.0, 0.09849140335716425, 0.198912367379658, 0.3033466836073424, 0.41421356237309503, \
                    0.5345111359507917, 0.6681786379192989, 0.8206787908286604, 1.0, 1.2185035255879764, \
                    1.496605762665489, 1.8708684117893895, 2.414213562373095, 3.2965582089383205, \
                    5.027339492125848, 10.15317038760886}
#define DRM_ATAN_A {0.0, 0.09817477042468103, 0.19634954084936207, 0.2945243112740431, 0.39269908169872414, \
                    0.4908738521234052, 0.5890486225480862, 0.6872233929727672, 0.7853981633974483, \
                    0.8835729338221293, 0.9817477042468103, 1.0799224746714915, 1.1780972450961724, \
                    1.2762720155208536, 1.3744467859455345, 1.4726215563702156}
#if defined(__CUDACC__)
static __device__ const double drm_atan_c_dev[16] = DRM_ATAN_C;
static __device__ const double drm_atan_a_dev[16] = DRM_ATAN_A;
#endif
static const double drm_atan_c_host[16] = DRM_ATAN_C;
static const double drm_atan_a_host[16] = DRM_ATAN_A;

// atan t for |t| <= 0.055, series to t^15
DRM_FN double atan_series(double t) {
    double z = mul(t, t);
    double p = -0.06666666666666667;
    p = add(mul(p, z), 0.07692307692307693);
    p = add(mul(p, z), -0.09090909090909091);
    p = add(mul(p, z), 0.1111111111111111);
    p = add(mul(p, z), -0.14285714285714285);
    p = add(mul(p, z), 0.2);
    p = add(mul(p, z), -0.3333333333333333);
    p = add(mul(p, z), 1.0);
    return mul(t, p);
}

// arc tangent of a double: atan a = k pi/32 + atan((a - c_k) / (1 + a c_k))
// with k the nearest multiple (16 comparisons against tan((2k + 1) pi/64)),
// so that |t| <= tan(pi/64); a > tan(31 pi/64) as pi/2 - atan(1/a).
DRM_FN double atan_d(double x) {
    if (is_nan(x)) return x;
    bool neg = sign_bit(x);
    double a = absd(x);
    double r;
    if (a > 20.355467624987188) {
        r = sub(kPio2, atan_series(div(1.0, a)));
    } else {
        int k = (a > 0.049126849769467254) + (a > 0.14833598753834742) + (a > 0.25048696019130545) +
                (a > 0.3578057213145241) + (a > 0.4729647758913199) + (a > 0.5993769336819238) +
                (a > 0.7416505462720354) + (a > 0.9063471690191471) + (a > 1.1033299757334756) +
                (a > 1.3483439134867201) + (a > 1.668399205583507) + (a > 2.1143223575486405) +
                (a > 2.7948127724904768) + (a > 3.9922237837700845) + (a > 6.7414524054149885);
#ifdef __CUDA_ARCH__
        double c = __ldg(&drm_atan_c_dev[k]), ang = __ldg(&drm_atan_a_dev[k]);
#else
        double c = drm_atan_c_host[k], ang = drm_atan_a_host[k];
#endif
        double t = div(sub(a, c), add(1.0, mul(a, c)));
        r = add(ang, atan_series(t));
    }
    return neg ? -r : r;
}

// atan2 with the C99 conventions for zeros and infinities
DRM_FN double atan2_d(double y, double x) {
    if (is_nan(x) || is_nan(y)) return x + y;
    bool ny = sign_bit(y), nx = sign_bit(x);
    double ay = absd(y), ax = absd(x);
    double r;
    if (ay == 0.0) {
        r = nx ? kPi : 0.0;
    } else if (ax == 0.0) {
        r = kPio2;
    } else if (ay == kInf && ax == kInf) {
        r = nx ? 2.356194490192345 : 0.7853981633974483;
    } else {
        r = ay <= ax ? atan_d(div(ay, ax)) : sub(kPio2, atan_d(div(ax, ay)));
        if (nx) r = sub(kPi, r);
    }
    return ny ? -r : r;
}

DRM_FN double acos_d(double x) {
    if (is_nan(x) || x > 1.0 || x < -1.0) return kInf - kInf;
    return mul(2.0, atan_d(root(div(sub(1.0, x), add(1.0, x)))));
}

// sine and cosine of r, |r| <= pi/4 (+ rounding)
DRM_FN double sin_poly(double r) {
    double z = mul(r, r);
    double p = 2.8114572543455206e-15;
    p = add(mul(p, z), -7.647163731819816e-13);
    p = add(mul(p, z), 1.6059043836821613e-10);
    p = add(mul(p, z), -2.505210838544172e-08);
    p = add(mul(p, z), 2.7557319223985893e-06);
    p = add(mul(p, z), -0.0001984126984126984);
    p = add(mul(p, z), 0.008333333333333333);
    p = add(mul(p, z), -0.16666666666666666);
    p = add(mul(p, z), 1.0);
    return mul(r, p);
}
DRM_FN double cos_poly(double r) {
    double z = mul(r, r);
    double p = 4.779477332387385e-14;
    p = add(mul(p, z), -1.1470745597729725e-11);
    p = add(mul(p, z), 2.08767569878681e-09);
    p = add(mul(p, z), -2.755731922398589e-07);
    p = add(mul(p, z), 2.48015873015873e-05);
    p = add(mul(p, z), -0.001388888888888889);
    p = add(mul(p, z), 0.041666666666666664);
    p = add(mul(p, z), -0.5);
    p = add(mul(p, z), 1.0);
    return p;
}
// quadrant q = k mod 4 and remainder r of x = k pi/2 + r
DRM_FN double reduce_pio2(double x, int &q) {
    double k = round_int(mul(x, kTwoOverPi));
    q = (int)((int64_t)k & 3);
    return sub(sub(x, mul(k, kPio2Hi)), mul(k, kPio2Lo));
}
DRM_FN double sin_d(double x) {
    if (is_nan(x) || absd(x) == kInf) return kInf - kInf;
    int q;
    double r = reduce_pio2(x, q);
    double v = (q & 1) ? cos_poly(r) : sin_poly(r);
    return (q & 2) ? -v : v;
}
DRM_FN double cos_d(double x) {
    if (is_nan(x) || absd(x) == kInf) return kInf - kInf;
    int q;
    double r = reduce_pio2(x, q);
    double v = (q & 1) ? sin_poly(r) : cos_poly(r);
    return ((q + 1) & 2) ? -v : v;
}

// x^y for doubles (the float power calls it with float arguments)
DRM_FN double pow_d(double x, double y) {
    if (y == 0.0 || x == 1.0) return 1.0;
    if (is_nan(x) || is_nan(y)) return x + y;
    bool neg = false;
    if (x < 0.0) {
        // a negative base has a real power only for integer exponents
        double fy = round_int(y);
        if (absd(y) >= 4503599627370496.0) fy = y;  // |y| >= 2^52: an even integer
        if (fy != y) return kInf - kInf;
        if (absd(y) < 4503599627370496.0) neg = ((int64_t)fy & 1) != 0;
        x = -x;
    }
    double r;
    if (x == 0.0) r = y > 0.0 ? 0.0 : kInf;
    else if (x == kInf) r = y > 0.0 ? kInf : 0.0;
    else r = exp_d(mul(y, log_d(x)));
    return neg ? -r : r;
}

}  // namespace drm

DRM_FN float dr_sinf(float x) { return (float)drm::sin_d((double)x); }
DRM_FN float dr_cosf(float x) { return (float)drm::cos_d((double)x); }
DRM_FN float dr_atanf(float x) { return (float)drm::atan_d((double)x); }
DRM_FN float dr_atan2f(float y, float x) { return (float)drm::atan2_d((double)y, (double)x); }
DRM_FN float dr_acosf(float x) { return (float)drm::acos_d((double)x); }
DRM_FN float dr_expf(float x) { return (float)drm::exp_d((double)x); }
DRM_FN float dr_logf(float x) { return (float)drm::log_d((double)x); }
DRM_FN float dr_powf(float x, float y) { return (float)drm::pow_d((double)x, (double)y); }

// Dispatch by function number (0 sin, 1 cos, 2 atan, 3 atan2(x, y), 4 acos,
// 5 exp, 6 log, 7 pow(x, y)): the check hooks of the library and of the host
// test build evaluate the functions through this one switch.
DRM_FN float dr_math_eval(int fn, float x, float y) {
    switch (fn) {
    case 0: return dr_sinf(x);
    case 1: return dr_cosf(x);
    case 2: return dr_atanf(x);
    case 3: return dr_atan2f(x, y);
    case 4: return dr_acosf(x);
    case 5: return dr_expf(x);
    case 6: return dr_logf(x);
    case 7: return dr_powf(x, y);
    default: return 0.f;
    }
}
