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
// The arc tangent family (atan, atan2, acos) is evaluated in float, see
// below.  Methods (textbook ones, with coefficients that are exact Taylor
// coefficients rounded to double):
//   log  x = 2^k m, m in [sqrt(1/2), sqrt(2)]; log m = 2 atanh(s),
//        s = (m - 1) / (m + 1), |s| <= 0.172, series to s^21.
//   exp  x = k ln2 + r, |r| <= ln2 / 2 (Cody-Waite: ln2 split into a 33-bit
//        head and a tail), Taylor series to r^13, then times 2^k.
//   pow  exp(y log x) for x > 0; integer y for x < 0.
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

// The arc tangent family in float (the renderer's line samples call atan in
// their Newton loop and its edge-tree walks call acos and atan per node, so
// these stay in single precision; every operation is an IEEE float operation
// without contraction, so the bits are still the same on the GPU and the
// host).  atan a = k pi/32 + atan t, t = (a - c_k) / (1 + a c_k), with c_k
// the float nearest tan(k pi/32), k picked by 16 comparisons so that
// |t| <= ~tan(pi/64), the angle atan(c_k) as a head and a tail float, and the
// series to t^9; a > ~tan(31 pi/64) as pi/2 - atan(1/a).  Within about 2 ulp.
namespace drm {
#define DRM_ATANF_C {0.0f, 0.09849140048027039f, 0.1989123672246933f, 0.3033466935157776f, 0.4142135679721832f, \
                     0.534511148929596f, 0.6681786179542542f, 0.8206787705421448f, 1.0f, 1.218503475189209f, \
                     1.4966057538986206f, 1.870868444442749f, 2.4142136573791504f, 3.296558141708374f, \
                     5.027339458465576f, 10.153170585632324f}
#define DRM_ATANF_AH {0.0f, 0.09817476570606232f, 0.19634954631328583f, 0.29452431201934814f, \
                      0.39269909262657166f, 0.49087387323379517f, 0.5890486240386963f, 0.6872233748435974f, \
                      0.7853981852531433f, 0.8835729360580444f, 0.9817476868629456f, 1.0799224376678467f, \
                      1.1780972480773926f, 1.2762720584869385f, 1.3744467496871948f, 1.4726215600967407f}
#define DRM_ATANF_AL {0.0f, 1.8693642189759885e-09f, -5.612990516823402e-09f, 8.32819413432162e-09f, \
                      -6.148726860999432e-09f, -1.1015669265646011e-08f, -1.5293277755290546e-08f, \
                      6.007060626700422e-09f, -2.1855694143368964e-08f, -2.2519143882959725e-08f, \
                      1.4677898008130796e-08f, 4.425970701049664e-08f, 1.0932094340887488e-08f, \
                      -4.863122882170501e-08f, 3.4977222895804516e-08f, -1.8240424726201354e-09f}
#if defined(__CUDACC__)
static __device__ const float drm_atanf_c_dev[16] = DRM_ATANF_C;
static __device__ const float drm_atanf_ah_dev[16] = DRM_ATANF_AH;
static __device__ const float drm_atanf_al_dev[16] = DRM_ATANF_AL;
#endif
static const float drm_atanf_c_host[16] = DRM_ATANF_C;
static const float drm_atanf_ah_host[16] = DRM_ATANF_AH;
static const float drm_atanf_al_host[16] = DRM_ATANF_AL;
constexpr float kPio2Hf = 1.5707963705062866f, kPio2Lf = -4.371138828673793e-08f;
constexpr float kPiHf = 3.1415927410125732f, kPiLf = -8.742277657347586e-08f;

#ifdef __CUDA_ARCH__
DRM_FN float fadd(float a, float b) { return __fadd_rn(a, b); }
DRM_FN float fsub(float a, float b) { return __fsub_rn(a, b); }
DRM_FN float fmul(float a, float b) { return __fmul_rn(a, b); }
DRM_FN float fdiv(float a, float b) { return __fdiv_rn(a, b); }
DRM_FN float froot(float a) { return __fsqrt_rn(a); }
DRM_FN uint32_t fbits(float a) { return __float_as_uint(a); }
DRM_FN float fabs_(float a) { return __uint_as_float(__float_as_uint(a) & 0x7fffffffu); }
#else
DRM_FN float fadd(float a, float b) { return a + b; }
DRM_FN float fsub(float a, float b) { return a - b; }
DRM_FN float fmul(float a, float b) { return a * b; }
DRM_FN float fdiv(float a, float b) { return a / b; }
DRM_FN float froot(float a) { return __builtin_sqrtf(a); }
DRM_FN uint32_t fbits(float a) {
    uint32_t b;
    std::memcpy(&b, &a, 4);
    return b;
}
DRM_FN float fabs_(float a) {
    uint32_t b = fbits(a) & 0x7fffffffu;
    float r;
    std::memcpy(&r, &b, 4);
    return r;
}
#endif

// atan t - t for |t| <= 0.055: t^3 (-1/3 + t^2/5 - t^4/7 + t^6/9)
DRM_FN float atanf_tail(float t) {
    float z = fmul(t, t);
    float q = 0.1111111119389534f;
    q = fsub(fmul(q, z), 0.1428571492433548f);
    q = fadd(fmul(q, z), 0.20000000298023224f);
    q = fsub(fmul(q, z), 0.3333333432674408f);
    return fmul(fmul(t, z), q);
}
// atan of a >= 0 as head + tail (hi + lo), for the callers that add to it
DRM_FN float atanf_pos(float a) {
    if (a > 20.355466842651367f) {
        float t = fdiv(1.f, a);
        return fadd(kPio2Hf, fsub(kPio2Lf, fadd(t, atanf_tail(t))));
    }
    int k = (a > 0.049126848578453064f) + (a > 0.1483359932899475f) + (a > 0.25048696994781494f) +
            (a > 0.3578057289123535f) + (a > 0.4729647636413574f) + (a > 0.599376916885376f) +
            (a > 0.7416505217552185f) + (a > 0.9063471555709839f) + (a > 1.1033300161361694f) +
            (a > 1.3483439683914185f) + (a > 1.6683992147445679f) + (a > 2.1143224239349365f) +
            (a > 2.7948126792907715f) + (a > 3.9922237396240234f) + (a > 6.741452217102051f);
#ifdef __CUDA_ARCH__
    float c = __ldg(&drm_atanf_c_dev[k]), ah = __ldg(&drm_atanf_ah_dev[k]), al = __ldg(&drm_atanf_al_dev[k]);
#else
    float c = drm_atanf_c_host[k], ah = drm_atanf_ah_host[k], al = drm_atanf_al_host[k];
#endif
    float t = fdiv(fsub(a, c), fadd(1.f, fmul(a, c)));
    return fadd(ah, fadd(al, fadd(t, atanf_tail(t))));
}
}  // namespace drm

DRM_FN float dr_atanf(float x) {
    if (x != x) return x;
    float r = drm::atanf_pos(drm::fabs_(x));
    return (drm::fbits(x) & 0x80000000u) ? -r : r;
}
// atan2 with the C99 conventions for zeros and infinities
DRM_FN float dr_atan2f(float y, float x) {
    if (x != x || y != y) return x + y;
    bool ny = (drm::fbits(y) & 0x80000000u) != 0, nx = (drm::fbits(x) & 0x80000000u) != 0;
    float ay = drm::fabs_(y), ax = drm::fabs_(x);
    const float inf = __builtin_huge_valf();
    float r;
    if (ay == 0.f) {
        r = nx ? drm::kPiHf : 0.f;
    } else if (ax == 0.f) {
        r = drm::kPio2Hf;
    } else if (ay == inf && ax == inf) {
        r = nx ? 2.356194496154785f : 0.7853981852531433f;
    } else {
        if (ay <= ax) {
            r = drm::atanf_pos(drm::fdiv(ay, ax));
        } else {
            float q = drm::fdiv(ax, ay);
            r = drm::fadd(drm::kPio2Hf, drm::fsub(drm::kPio2Lf, drm::atanf_pos(q)));
        }
        if (nx) r = drm::fadd(drm::kPiHf, drm::fsub(drm::kPiLf, r));
    }
    return ny ? -r : r;
}
// acos x = 2 atan(sqrt((1 - x) / (1 + x)))
DRM_FN float dr_acosf(float x) {
    if (x != x || x > 1.f || x < -1.f) return __builtin_nanf("");
    if (x == -1.f) return drm::kPiHf;
    return drm::fmul(2.f, drm::atanf_pos(drm::froot(drm::fdiv(drm::fsub(1.f, x), drm::fadd(1.f, x)))));
}
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
