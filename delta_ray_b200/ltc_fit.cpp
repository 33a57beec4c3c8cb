// Fits linearly transformed cosines (LTC) to the renderer's specular lobes.
//
// Heitz, Dupuy, Hill and Neubelt, "Real-Time Polygonal-Light Shading with
// Linearly Transformed Cosines" (SIGGRAPH 2016): a clamped cosine
// D_o(w_o) = max(w_o.z, 0) / pi, pushed through a 3x3 matrix M
// (w = M w_o / |M w_o|), has the density
//     D(w) = D_o(w_o) |det M^-1| / |M^-1 w|^3,   w_o = M^-1 w / |M^-1 w|.
// For a view direction V = (sin t, 0, cos t) in the xz-plane, an isotropic
// lobe is symmetric about that plane, so M = [[a, 0, b], [0, c, 0], [d, 0, 1]]
// (the scale of M does not change D).  The fit minimises, over (a, b, c, d),
//     E = integral |D(w) - f(w) / |f||^3 dw
// where f is the lobe's cosine-weighted BRDF without Fresnel and |f| its
// integral, estimated with stratified samples drawn half from D and half from
// the lobe's own half-vector sampling, weighted by the balance heuristic.  The
// optimiser is Nelder-Mead (Nelder and Mead, 1965); along each row of the
// table (fixed view angle) the fit runs from roughness 1 down to 0, each fit
// starting from the previous one.
//
// Lobes (roughness r):
//   model 0, Blinn-Phong: D(h) = (e + 2) / (2 pi) cos^e(h), e = 2 / r, with the
//       renderer's rational Smith G1 term;
//   model 1, GGX (Walter et al. 2007): alpha = max(r^2, 1e-4),
//       D(h) = alpha^2 / (pi ((n.h)^2 (alpha^2 - 1) + 1)^2), exact Smith G1.
//
// Table layout, as the renderer reads it: entry (ir + it * n), ir for
// roughness ir / (n - 1), it for view angle (it / (n - 1)) * pi / 2, each a
// row-major 3x3 M.
#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace {

const double kPi = 3.14159265358979323846;

struct V3 {
    double x, y, z;
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
double len(V3 a) { return std::sqrt(dot(a, a)); }
V3 norm(V3 a) { return (1.0 / len(a)) * a; }

// ---------------------------------------------------------------- lobes
struct Lobe {
    int model;
    double r;  // roughness
    V3 v;      // view direction

    double alpha() const { return std::max(r * r, 1e-4); }
    double phong_e() const { return std::max(2.0 / std::max(r, 1e-4), 0.0); }

    double D(double ch) const {
        if (ch <= 0.0) return 0.0;
        if (model == 0) {
            double e = phong_e();
            return (e + 2.0) / (2.0 * kPi) * std::pow(ch, e);
        }
        double a2 = alpha() * alpha();
        double k = ch * ch * (a2 - 1.0) + 1.0;
        return a2 / (kPi * k * k);
    }

    double G1(V3 w, V3 h) const {
        double c = w.z;
        if (dot(w, h) * c <= 0.0) return 0.0;
        if (model == 1) {
            double a2 = alpha() * alpha();
            return 2.0 * c / (c + std::sqrt(a2 + (1.0 - a2) * c * c));
        }
        // the renderer's rational approximation (isotropic: projected roughness sqrt(r))
        double tan_t = std::sqrt(std::max(1.0 / (c * c) - 1.0, 0.0));
        if (tan_t == 0.0) return 1.0;
        double a = 1.0 / (std::sqrt(r) * tan_t);
        if (a >= 1.6) return 1.0;
        return (3.535 * a + 2.181 * a * a) / (1.0 + 2.276 * a + 2.577 * a * a);
    }

    // cosine-weighted BRDF value (no Fresnel)
    double f(V3 w) const {
        if (w.z <= 0.0 || v.z <= 0.0) return 0.0;
        V3 h = norm(v + w);
        return D(h.z) * G1(v, h) * G1(w, h) / (4.0 * v.z);
    }

    // half vector with density D(h) cos(h)
    V3 sample(double u0, double u1, double *pdf) const {
        double ch;
        if (model == 0) {
            ch = std::pow(u0, 1.0 / (phong_e() + 2.0));
        } else {
            double a2 = alpha() * alpha();
            ch = std::sqrt((1.0 - u0) / (1.0 + (a2 - 1.0) * u0));
        }
        double sh = std::sqrt(std::max(1.0 - ch * ch, 0.0)), phi = 2.0 * kPi * u1;
        V3 h{sh * std::cos(phi), sh * std::sin(phi), ch};
        V3 w = 2.0 * dot(v, h) * h - v;
        double vh = std::fabs(dot(v, h));
        *pdf = vh > 0.0 ? D(ch) * ch / (4.0 * vh) : 0.0;
        return w;
    }

    double pdf(V3 w) const {
        V3 h = v + w;
        if (len(h) == 0.0) return 0.0;
        h = norm(h);
        double vh = std::fabs(dot(v, h));
        return vh > 0.0 ? D(h.z) * h.z / (4.0 * vh) : 0.0;
    }
};

// ---------------------------------------------------------------- LTC
struct Ltc {
    double m[9], inv[9], det_inv;
    bool set(const double *p) {  // p = (a, b, c, d)
        double a = p[0], b = p[1], c = p[2], d = p[3];
        if (!(a > 1e-6 && c > 1e-6)) return false;
        double det = c * (a - b * d);  // det [[a,0,b],[0,c,0],[d,0,1]]
        if (!(det > 1e-12)) return false;
        m[0] = a; m[1] = 0; m[2] = b;
        m[3] = 0; m[4] = c; m[5] = 0;
        m[6] = d; m[7] = 0; m[8] = 1;
        double id = 1.0 / det;
        inv[0] = c * id;  inv[1] = 0;                  inv[2] = -b * c * id;
        inv[3] = 0;       inv[4] = (a - b * d) * id;   inv[5] = 0;
        inv[6] = -d * c * id; inv[7] = 0;              inv[8] = a * c * id;
        det_inv = id;
        return true;
    }
    static V3 mul(const double *M, V3 w) {
        return {M[0] * w.x + M[1] * w.y + M[2] * w.z, M[3] * w.x + M[4] * w.y + M[5] * w.z,
                M[6] * w.x + M[7] * w.y + M[8] * w.z};
    }
    double pdf(V3 w) const {
        V3 wo = mul(inv, w);
        double l = len(wo);
        double z = wo.z / l;
        if (z <= 0.0) return 0.0;
        return z / kPi * std::fabs(det_inv) / (l * l * l);
    }
    V3 sample(double u0, double u1) const {
        double phi = 2.0 * kPi * u0, s = std::sqrt(1.0 - u1);
        V3 wo{std::cos(phi) * s, std::sin(phi) * s, std::sqrt(u1)};
        return norm(mul(m, wo));
    }
};

// ---------------------------------------------------------------- error
struct Fit {
    Lobe lobe;
    int ns;       // strata per axis
    double norm;  // integral of the lobe

    double amplitude() const {
        double acc = 0.0;
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) {
                double p;
                V3 w = lobe.sample((i + 0.5) / ns, (j + 0.5) / ns, &p);
                if (p > 0.0) acc += lobe.f(w) / p;
            }
        return acc / (ns * ns);
    }

    double error(const double *params) const {
        Ltc l;
        if (!l.set(params)) return 1e30;
        double err = 0.0;
        for (int s = 0; s < 2; s++)
            for (int i = 0; i < ns; i++)
                for (int j = 0; j < ns; j++) {
                    double u0 = (i + 0.5) / ns, u1 = (j + 0.5) / ns;
                    V3 w;
                    if (s == 0) {
                        w = l.sample(u0, u1);
                    } else {
                        double p;
                        w = lobe.sample(u0, u1, &p);
                    }
                    double pl = l.pdf(w), pb = lobe.pdf(w);
                    double q = 0.5 * (pl + pb);
                    if (q <= 0.0) continue;
                    double target = lobe.f(w) / norm;
                    double e = std::fabs(pl - target);
                    err += e * e * e / q;
                }
        return err / (2.0 * ns * ns);
    }
};

// Nelder-Mead over 4 parameters, from x (updated in place); returns the error.
double nelder_mead(const Fit &fit, double *x, int iters, double step) {
    const int n = 4;
    double p[n + 1][n], fv[n + 1];
    for (int i = 0; i <= n; i++) {
        for (int k = 0; k < n; k++) p[i][k] = x[k];
        if (i > 0) p[i][i - 1] += step * std::max(std::fabs(x[i - 1]), 0.05);
        fv[i] = fit.error(p[i]);
    }
    for (int it = 0; it < iters; it++) {
        int lo = 0, hi = 0, nh = 0;
        for (int i = 0; i <= n; i++) {
            if (fv[i] < fv[lo]) lo = i;
            if (fv[i] > fv[hi]) hi = i;
        }
        nh = lo;
        for (int i = 0; i <= n; i++)
            if (i != hi && fv[i] > fv[nh]) nh = i;
        if (std::fabs(fv[hi] - fv[lo]) <= 1e-9 * (std::fabs(fv[lo]) + 1e-12)) break;
        double c[n] = {0, 0, 0, 0};
        for (int i = 0; i <= n; i++)
            if (i != hi)
                for (int k = 0; k < n; k++) c[k] += p[i][k] / n;
        auto point = [&](double t, double *out) {
            for (int k = 0; k < n; k++) out[k] = c[k] + t * (p[hi][k] - c[k]);
        };
        double r[n], e[n], k2[n];
        point(-1.0, r);
        double fr = fit.error(r);
        if (fr < fv[lo]) {
            point(-2.0, e);
            double fe = fit.error(e);
            if (fe < fr) {
                std::copy(e, e + n, p[hi]);
                fv[hi] = fe;
            } else {
                std::copy(r, r + n, p[hi]);
                fv[hi] = fr;
            }
        } else if (fr < fv[nh]) {
            std::copy(r, r + n, p[hi]);
            fv[hi] = fr;
        } else {
            bool outside = fr < fv[hi];
            point(outside ? -0.5 : 0.5, k2);
            double fk = fit.error(k2);
            if (fk < (outside ? fr : fv[hi])) {
                std::copy(k2, k2 + n, p[hi]);
                fv[hi] = fk;
            } else {  // shrink towards the best point
                for (int i = 0; i <= n; i++) {
                    if (i == lo) continue;
                    for (int k = 0; k < n; k++) p[i][k] = p[lo][k] + 0.5 * (p[i][k] - p[lo][k]);
                    fv[i] = fit.error(p[i]);
                }
            }
        }
    }
    int lo = 0;
    for (int i = 1; i <= n; i++)
        if (fv[i] < fv[lo]) lo = i;
    std::copy(p[lo], p[lo] + n, x);
    return fv[lo];
}

void fit_row(int model, int n, int it, int strata, int iters, float *out_m, float *out_err) {
    double theta = (double)it / (n - 1) * kPi / 2.0;
    theta = std::min(theta, kPi / 2.0 - 1e-3);  // grazing views: the lobe is still defined
    V3 v{std::sin(theta), 0.0, std::cos(theta)};
    double x[4] = {1.0, 0.0, 1.0, 0.0};
    for (int ir = n - 1; ir >= 0; ir--) {
        Fit fit{Lobe{model, std::max((double)ir / (n - 1), 1e-3), v}, strata, 0.0};
        fit.norm = fit.amplitude();
        double err = 0.0;
        if (fit.norm > 0.0) {
            // a restart from the previous solution with a small and a larger step
            err = nelder_mead(fit, x, iters, 0.05);
            err = nelder_mead(fit, x, iters, 0.2);
        }
        float *m = out_m + 9 * (size_t)(ir + it * n);
        const double M[9] = {x[0], 0.0, x[1], 0.0, x[2], 0.0, x[3], 0.0, 1.0};
        for (int k = 0; k < 9; k++) m[k] = (float)M[k];
        if (out_err) out_err[ir + it * n] = (float)err;
    }
}

}  // namespace

extern "C" {

// Fits the n x n table of `model` (0 Blinn-Phong, 1 GGX) into out_m
// [n * n * 9] (and the final error of each entry into out_err [n * n] when
// not NULL), rows on `threads` threads.
__attribute__((visibility("default"))) int ltc_fit_table(int model, int n, int strata, int iters, float *out_m,
                                                         float *out_err, int threads) {
    if (n < 2 || (model != 0 && model != 1) || !out_m) return 1;
    threads = std::max(1, threads);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++)
        pool.emplace_back([=]() {
            for (int it = t; it < n; it += threads) fit_row(model, n, it, strata, iters, out_m, out_err);
        });
    for (auto &th : pool) th.join();
    return 0;
}

// Distance between the fitted LTC and the normalised lobe for one entry:
// integral |D_ltc - f / |f|| (L1, 0 = exact, 2 = disjoint), for tests.
__attribute__((visibility("default"))) double ltc_fit_l1(int model, double roughness, double theta, const float *m9,
                                                         int strata) {
    V3 v{std::sin(theta), 0.0, std::cos(theta)};
    Fit fit{Lobe{model, std::max(roughness, 1e-3), v}, strata, 0.0};
    fit.norm = fit.amplitude();
    Ltc l;
    double p[4] = {m9[0] / m9[8], m9[2] / m9[8], m9[4] / m9[8], m9[6] / m9[8]};
    if (!l.set(p) || fit.norm <= 0.0) return 2.0;
    double acc = 0.0;
    int ns = strata;
    for (int s = 0; s < 2; s++)
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) {
                double u0 = (i + 0.5) / ns, u1 = (j + 0.5) / ns, pb;
                V3 w = s == 0 ? l.sample(u0, u1) : fit.lobe.sample(u0, u1, &pb);
                double pl = l.pdf(w), pbb = fit.lobe.pdf(w), q = 0.5 * (pl + pbb);
                if (q > 0.0) acc += std::fabs(pl - fit.lobe.f(w) / fit.norm) / q;
            }
    return acc / (2.0 * ns * ns);
}

}  // extern "C"
