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
//   log  Tang's table-driven method: x = 2^k m, log m = log c_j +
//        log1p(m / c_j - 1) over 64 centres c_j, series to r^8.
//   exp  Tang's table-driven method: x = (64 m + j) ln2/64 + r (Cody-Waite),
//        e^x = 2^m 2^(j/64) e^r, series to r^6.
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

// Tables of the logarithm and the exponential (Tang's table-driven method):
// DRM_LOG_INV[j] = 1 / c_j rounded to double, c_0 = 1 and c_j = 1 + (j + 1/2)
// / 64 for j > 0, and DRM_LOG_L[j] = -log(DRM_LOG_INV[j]); DRM_EXP_T[j] =
// 2^(j/64).  All rounded to double from 60-digit values.
#define DRM_LOG_INV {1.0, 0.9770992366412213, 0.9624060150375939, 0.9481481481481482, \
    0.9343065693430657, 0.920863309352518, 0.9078014184397163, 0.8951048951048951, \
    0.8827586206896552, 0.8707482993197279, 0.8590604026845637, 0.847682119205298, \
    0.8366013071895425, 0.8258064516129032, 0.8152866242038217, 0.8050314465408805, \
    0.7950310559006211, 0.7852760736196319, 0.7757575757575758, 0.7664670658682635, \
    0.757396449704142, 0.7485380116959064, 0.7398843930635838, 0.7314285714285714, \
    0.7231638418079096, 0.7150837988826816, 0.7071823204419889, 0.6994535519125683, \
    0.6918918918918919, 0.6844919786096256, 0.6772486772486772, 0.6701570680628273, \
    0.6632124352331606, 0.6564102564102564, 0.649746192893401, 0.6432160804020101, \
    0.6368159203980099, 0.6305418719211823, 0.624390243902439, 0.6183574879227053, \
    0.6124401913875598, 0.6066350710900474, 0.6009389671361502, 0.5953488372093023, \
    0.5898617511520737, 0.5844748858447488, 0.579185520361991, 0.5739910313901345, \
    0.5688888888888889, 0.5638766519823789, 0.5589519650655022, 0.5541125541125541, \
    0.5493562231759657, 0.5446808510638298, 0.540084388185654, 0.5355648535564853, \
    0.5311203319502075, 0.5267489711934157, 0.5224489795918368, 0.5182186234817814, \
    0.5140562248995983, 0.5099601593625498, 0.5059288537549407, 0.5019607843137255}
#define DRM_LOG_L {0.0, 0.023167059281534418, 0.03831886430213666, 0.05324451451881224, \
    0.06795066190850778, 0.08244366921107454, 0.09672962645855114, 0.11081436634029011, \
    0.12470347850095725, 0.1384023228591192, 0.151916042025842, 0.16524957289530717, \
    0.17840765747281825, 0.19139485299962947, 0.20421554142869083, 0.2168739383006143, \
    0.2293741010648459, 0.24171993688714513, 0.25391520998096345, 0.2659635484971379, \
    0.2778684510034563, 0.2896332925830427, 0.30126133057816185, 0.3127557100038969, \
    0.324119468654212, 0.3353555419211378, 0.3464667673462086, 0.3574558889218038, \
    0.36832556115870757, 0.3790783529349695, 0.38971675114002524, 0.40024316412701266, \
    0.4106599249852683, 0.42096929464412963, 0.43117346481837143, 0.4412745608048752, \
    0.4512746441394586, 0.46117571512217015, 0.470979715218791, 0.48068852934575196, \
    0.4903039880451939, 0.49982786955644926, 0.5092619017898079, 0.5186077642080457, \
    0.5278670896208424, 0.5370414658968837, 0.5461324375981356, 0.5551415075405016, \
    0.564070138284803, 0.5729197535617854, 0.5816917396346225, 0.5903874466021763, \
    0.5990081896460834, 0.6075552502245418, 0.616029877215514, 0.6244332880118936, \
    0.6327666695710378, 0.6410311794209312, 0.6492279466251097, 0.65735807270836, \
    0.6654226325450905, 0.6734226752121667, 0.6813592248079031, 0.689233281238809}
#define DRM_EXP_T {1.0, 1.0108892860517005, 1.0218971486541166, 1.0330248790212284, \
    1.0442737824274138, 1.0556451783605572, 1.0671404006768237, 1.0787607977571199, \
    1.0905077326652577, 1.102382583307841, 1.1143867425958924, 1.1265216186082418, \
    1.1387886347566916, 1.1511892299529827, 1.1637248587775775, 1.1763969916502812, \
    1.189207115002721, 1.202156731452703, 1.215247359980469, 1.22848053610687, \
    1.241857812073484, 1.255380757024691, 1.2690509571917332, 1.2828700160787783, \
    1.2968395546510096, 1.3109612115247644, 1.3252366431597413, 1.339667524053303, \
    1.3542555469368927, 1.3690024229745905, 1.383909881963832, 1.3989796725383112, \
    1.4142135623730951, 1.42961333839197, 1.4451808069770467, 1.460917794180647, \
    1.4768261459394993, 1.4929077282912648, 1.5091644275934228, 1.5255981507445384, \
    1.5422108254079407, 1.559004400237837, 1.5759808451078865, 1.593142151342267, \
    1.6104903319492543, 1.6280274218573478, 1.645755478153965, 1.6636765803267364, \
    1.681792830507429, 1.7001063537185235, 1.718619298122478, 1.7373338352737062, \
    1.7562521603732995, 1.7753764925265212, 1.7947090750031072, 1.8142521755003989, \
    1.8340080864093424, 1.8539791250833855, 1.8741676341103, 1.8945759815869656, \
    1.9152065613971474, 1.9360617934922943, 1.9571441241754002, 1.978456026387951}
#if defined(__CUDACC__)
static __device__ const double drm_log_inv_dev[64] = DRM_LOG_INV;
static __device__ const double drm_log_l_dev[64] = DRM_LOG_L;
static __device__ const double drm_exp_t_dev[64] = DRM_EXP_T;
#endif
static const double drm_log_inv_host[64] = DRM_LOG_INV;
static const double drm_log_l_host[64] = DRM_LOG_L;
static const double drm_exp_t_host[64] = DRM_EXP_T;
#ifdef __CUDA_ARCH__
#define DRM_TABLE(name, j) __ldg(drm_##name##_dev + (j))
#else
#define DRM_TABLE(name, j) (drm_##name##_host[(j)])
#endif
constexpr double kLn2By64Hi = 0.01083042469326756;  // ln2 / 64, 32 significant bits
constexpr double kLn2By64Lo = 2.9815858269852933e-12;
constexpr double k64ByLn2 = 92.33248261689366;

// natural logarithm of a double: x = 2^k m, m in [1, 2); j = the top 6 bits
// of m's fraction; log x = k ln2 + L[j] + log1p(m INV[j] - 1), |m INV[j] - 1|
// < 1/64, log1p by its series to r^8
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
    int j = (int)((b >> 46) & 63);
    double r = sub(mul(m, DRM_TABLE(log_inv, j)), 1.0);
    double q = -0.125;
    q = add(mul(q, r), 0.14285714285714285);
    q = add(mul(q, r), -0.16666666666666666);
    q = add(mul(q, r), 0.2);
    q = add(mul(q, r), -0.25);
    q = add(mul(q, r), 0.3333333333333333);
    q = add(mul(q, r), -0.5);
    q = add(mul(mul(q, r), r), r);
    double dk = (double)k;
    return add(add(mul(dk, kLn2Hi), DRM_TABLE(log_l, j)), add(q, mul(dk, kLn2Lo)));
}

// e^x of a double: x = (64 m + j) ln2/64 + r, |r| <= ln2/128 (Cody-Waite);
// e^x = 2^m T[j] e^r, e^r by its series to r^6
DRM_FN double exp_d(double x) {
    if (is_nan(x)) return x;
    if (x > 709.0) return kInf;
    if (x < -745.5) return 0.0;
    double kd = round_int(mul(x, k64ByLn2));
    double r = sub(sub(x, mul(kd, kLn2By64Hi)), mul(kd, kLn2By64Lo));
    double p = 0.001388888888888889;
    p = add(mul(p, r), 0.008333333333333333);
    p = add(mul(p, r), 0.041666666666666664);
    p = add(mul(p, r), 0.16666666666666666);
    p = add(mul(p, r), 0.5);
    p = add(mul(p, r), 1.0);
    p = add(mul(p, r), 1.0);
    int k = (int)kd;
    int j = k & 63;
    return scale2(mul(DRM_TABLE(exp_t, j), p), (k - j) / 64);
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
