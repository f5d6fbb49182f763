// ORACLE — test infrastructure only. Only tests/, the smoke check and bench.py's CPU baseline
// load the library built from this file; the product path never does.
//
// FP64 CPU restatement of Larmor's FOD peak search (larmor-dmri 2.2.0): the amplitude of a
// tournier-basis SH series and its derivatives on the sphere (cpp/src/sh/harmonics.cpp), the
// Newton climb to a peak (cpp/src/sh/peaks.cpp:31-78) and the search of one voxel from the local
// maxima of its amplitudes on a sphere (cpp/src/sh/peaks.cpp:80-133), with the chunk loop of
// _core.peaks_chunk (cpp/src/python/sh.cpp:112-176). The steps, constants, tie rules and merge
// order are the reference's; the code is this project's own.
//
// Parity pins: tests/golden/peaks.npz holds the outputs of the reference's numpy peak oracle
// (tests/sd/reference_peaks.py) and MRtrix sh2peaks' peaks of the same FOD block;
// tests/test_peaks.py checks this file against them.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <thread>
#include <vector>

namespace oracle_peaks {

constexpr int kMaxLmax = 20;
constexpr int kDim = kMaxLmax + 1;
constexpr double kPi = 3.14159265358979323846;
constexpr double kSqrt2 = 1.41421356237309504880;
// Two peaks closer than this in cosine are one (cpp/src/sh/peaks.cpp:12).
constexpr double kSamePeak = 0.99;

int coefficient_index(int degree, int order, bool full) {
    return full ? degree * degree + degree + order : degree * (degree + 1) / 2 + order;
}

// base^exponent by squaring (cpp/src/sh/harmonics.cpp:13-27).
double power_int(double base, int exponent) {
    double result = 1.0;
    for (;;) {
        if (exponent % 2 == 1) result *= base;
        exponent /= 2;
        if (exponent == 0) break;
        base *= base;
    }
    return result;
}

double ladder_up(int l, int m) { return std::sqrt(double((l - m) * (l + m + 1))); }
double ladder_down(int l, int m) { return std::sqrt(double((l + m) * (l - m + 1))); }

// The recurrence constants (cpp/src/sh/harmonics.cpp:39-66): P(m, m) / sin^m theta with the
// Condon-Shortley sign, and sqrt((4 l^2 - 1) / (l^2 - m^2)) for l > m.
struct Constants {
    double diagonal[kDim];
    double factor[kDim][kDim];
    Constants() {
        double ratio = 1.0;
        for (int m = 0; m <= kMaxLmax; ++m) {
            const double mf = m;
            if (m > 0) ratio *= (2.0 * mf - 1.0) / (2.0 * mf);
            diagonal[m] = (m % 2 == 1 ? -1.0 : 1.0) * std::sqrt((2.0 * mf + 1.0) / (4.0 * kPi) * ratio);
            for (int l = 0; l <= kMaxLmax; ++l) factor[l][m] = 0.0;
            for (int l = m + 1; l <= kMaxLmax; ++l) {
                const double lf = l;
                factor[l][m] = std::sqrt((4.0 * lf * lf - 1.0) / (lf * lf - mf * mf));
            }
        }
    }
};

const Constants& constants() {
    static const Constants c;
    return c;
}

// The normalised associated Legendre table P(l, m)(cos theta) (cpp/src/sh/harmonics.cpp:70-88).
struct Table {
    double p[kDim][kDim] = {};
    Table(int lmax, double c, double s) {
        const Constants& k = constants();
        for (int m = 0; m <= lmax; ++m) {
            p[m][m] = k.diagonal[m] * power_int(s, m);
            if (m < lmax) p[m + 1][m] = std::sqrt(2.0 * m + 3.0) * c * p[m][m];
            for (int l = m + 2; l <= lmax; ++l)
                p[l][m] = k.factor[l][m] * (c * p[l - 1][m] - p[l - 2][m] / k.factor[l - 1][m]);
        }
    }
    // dP/dtheta and d2P/dtheta2 (cpp/src/sh/harmonics.cpp:102-137).
    double d1(int l, int m) const {
        if (l == 0) return 0.0;
        if (m == 0) return ladder_up(l, 0) * p[l][1];
        const double above = m < l ? ladder_up(l, m) * p[l][m + 1] : 0.0;
        return (above - ladder_down(l, m) * p[l][m - 1]) / 2.0;
    }
    double d2(int l, int m) const {
        if (l == 0) return 0.0;
        if (m == 0) {
            const double u0 = ladder_up(l, 0);
            return (u0 * ladder_up(l, 1) * p[l][2] - u0 * u0 * p[l][0]) / 2.0;
        }
        const double u = ladder_up(l, m), d = ladder_down(l, m);
        double total = -(u * u + d * d) * p[l][m];
        if (m == 1)
            total -= ladder_down(l, 1) * ladder_down(l, 0) * p[l][1];
        else
            total += ladder_down(l, m) * ladder_down(l, m - 1) * p[l][m - 2];
        if (m + 2 <= l) total += ladder_up(l, m) * ladder_up(l, m + 1) * p[l][m + 2];
        return total / 4.0;
    }
};

struct Derivatives {
    double f, t, p, tt, tp, pp;
};

// cpp/src/sh/harmonics.cpp:139-196: f, df/dtheta, df/dphi / sin, d2f/dtheta2,
// d2f/dtheta dphi / sin, d2f/dphi2 / sin^2; the pole limits where sin theta < 1e-4.
Derivatives derivatives(const double* sh, int lmax, bool full, double theta, double phi) {
    const Table tab(lmax, std::cos(theta), std::sin(theta));
    const double st = std::sin(theta);
    const bool pole = st < 1e-4;
    Derivatives r{0, 0, 0, 0, 0, 0};
    for (int l = 0; l <= lmax; l += full ? 1 : 2) {
        const double zonal = sh[coefficient_index(l, 0, full)];
        r.f += zonal * tab.p[l][0];
        r.t += zonal * tab.d1(l, 0);
        r.tt += zonal * tab.d2(l, 0);
        for (int m = 1; m <= l; ++m) {
            const double mf = m;
            const double cc = sh[coefficient_index(l, m, full)], sc = sh[coefficient_index(l, -m, full)];
            const double sp = std::sin(mf * phi), cp = std::cos(mf * phi);
            const double ang = kSqrt2 * (cc * cp + sc * sp);
            const double ang_p = kSqrt2 * (sc * cp - cc * sp);
            const double pv = tab.p[l][m], pt = tab.d1(l, m);
            r.f += ang * pv;
            r.t += ang * pt;
            r.tt += ang * tab.d2(l, m);
            if (pole) {
                r.p += ang_p * pt;
            } else {
                r.p += mf * ang_p * pv;
                r.tp += mf * ang_p * pt;
                r.pp -= mf * mf * ang * pv;
            }
        }
    }
    if (!pole) {
        r.p /= st;
        r.tp /= st;
        r.pp /= st * st;
    }
    return r;
}

// cpp/src/sh/peaks.cpp:31-78. True with the direction after the first step shorter than tol
// and the amplitude before it; false after max_iters steps.
bool climb(const double* sh, int lmax, bool full, const double* start, int max_iters, double tol, double max_step,
           double* dir, double* amp) {
    double d[3] = {start[0], start[1], start[2]};
    for (int it = 0; it < max_iters; ++it) {
        const double theta = std::acos(std::clamp(d[2], -1.0, 1.0));
        const double phi = std::atan2(d[1], d[0]);
        const Derivatives h = derivatives(sh, lmax, full, theta, phi);
        const double gnorm = std::sqrt(h.t * h.t + h.p * h.p);
        double at = 0.0, ap = 0.0;
        if (gnorm != 0.0) {
            at = h.t / gnorm;
            ap = h.p / gnorm;
        }
        const double slope = at * h.t + ap * h.p;
        const double curv = at * at * h.tt + 2.0 * at * ap * h.tp + ap * ap * h.pp;
        double step = curv != 0.0 ? std::abs(slope / curv) : 0.0;
        step = std::fmin(step, max_step);
        const double s_t = std::sin(theta), c_t = std::cos(theta), s_p = std::sin(phi), c_p = std::cos(phi);
        const double tt[3] = {c_t * c_p, c_t * s_p, -s_t};
        const double tp[3] = {-s_p, c_p, 0.0};
        for (int a = 0; a < 3; ++a) d[a] += step * (at * tt[a] + ap * tp[a]);
        const double n = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (int a = 0; a < 3; ++a) d[a] /= n;
        if (step < tol) {
            for (int a = 0; a < 3; ++a) dir[a] = d[a];
            *amp = h.f;
            return true;
        }
    }
    return false;
}

struct Peak {
    double d[3];
    double a;
};

// cpp/src/sh/peaks.cpp:80-133: climbs from every vertex with a positive amplitude and no
// neighbour above it, in vertex order; merges climbs closer than 0.99 in |cos| (signed cos when
// full), keeping the larger; a stable sort by amplitude; the first n_peaks above both thresholds.
void voxel_peaks(const double* sh, int lmax, bool full, const double* on_sphere, const double* vertices,
                 const int64_t* neighbours, int64_t nv, int n_peaks, double rel, double thr, double* dirs,
                 double* amps, std::vector<Peak>& found) {
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (int k = 0; k < 3 * n_peaks; ++k) dirs[k] = nan;
    for (int k = 0; k < n_peaks; ++k) amps[k] = nan;
    if (nv == 0 || !std::isfinite(on_sphere[0])) return;
    found.clear();
    for (int64_t v = 0; v < nv; ++v) {
        const double here = on_sphere[v];
        bool is_max = here > 0.0;
        for (int j = 0; j < 6 && is_max; ++j) is_max = on_sphere[neighbours[v * 6 + j]] <= here;
        if (!is_max) continue;
        Peak pk;
        if (!climb(sh, lmax, full, vertices + 3 * v, 50, 1e-4, 0.2, pk.d, &pk.a)) continue;
        if (!(pk.a > 0.0)) continue;
        auto match = std::find_if(found.begin(), found.end(), [&](const Peak& o) {
            const double c = pk.d[0] * o.d[0] + pk.d[1] * o.d[1] + pk.d[2] * o.d[2];
            return (full ? c : std::abs(c)) > kSamePeak;
        });
        if (match == found.end())
            found.push_back(pk);
        else if (pk.a > match->a)
            *match = pk;
    }
    if (found.empty()) return;
    std::stable_sort(found.begin(), found.end(), [](const Peak& x, const Peak& y) { return x.a > y.a; });
    const double largest = found.front().a;
    const int kept = std::min<int>(n_peaks, int(found.size()));
    for (int r = 0; r < kept; ++r) {
        const Peak& pk = found[r];
        if (pk.a < thr || pk.a < rel * largest) break;
        const bool flip = !full && pk.d[2] < 0.0;
        for (int a = 0; a < 3; ++a) dirs[3 * r + a] = flip ? -pk.d[a] : pk.d[a];
        amps[r] = pk.a;
    }
}

}  // namespace oracle_peaks

extern "C" {

void oracle_sh_derivatives(const double* sh, int64_t lmax, int full, double theta, double phi, double* out) {
    const auto r = oracle_peaks::derivatives(sh, int(lmax), full != 0, theta, phi);
    out[0] = r.f;
    out[1] = r.t;
    out[2] = r.p;
    out[3] = r.tt;
    out[4] = r.tp;
    out[5] = r.pp;
}

// NaN direction and amplitude when the climb does not stop within max_iters
// (cpp/src/python/sh.cpp:84-108).
void oracle_climb(const double* sh, int64_t lmax, int full, const double* start, int64_t max_iters, double tol,
                  double max_step, double* dir, double* amp) {
    if (!oracle_peaks::climb(sh, int(lmax), full != 0, start, int(max_iters), tol, max_step, dir, amp)) {
        const double nan = std::numeric_limits<double>::quiet_NaN();
        dir[0] = dir[1] = dir[2] = nan;
        *amp = nan;
    }
}

// coeffs (n, C), on_sphere (n, nv), vertices (nv, 3), neighbours (nv, 6) -> dirs (n, n_peaks, 3),
// amps (n, n_peaks); voxels split over n_threads threads in blocks of 16
// (cpp/src/python/sh.cpp:157-171). The caller checks the arguments.
void oracle_peaks_chunk(const double* coeffs, int64_t n, int64_t ncoef, int64_t lmax, int full,
                        const double* on_sphere, const double* vertices, const int64_t* neighbours, int64_t nv,
                        int64_t n_peaks, double rel, double thr, int64_t n_threads, double* dirs, double* amps) {
    const int64_t block = 16;
    const int64_t n_blocks = (n + block - 1) / block;
    auto work = [&](int64_t t) {
        std::vector<oracle_peaks::Peak> found;
        for (int64_t b = t; b < n_blocks; b += n_threads)
            for (int64_t v = b * block; v < std::min(n, (b + 1) * block); ++v)
                oracle_peaks::voxel_peaks(coeffs + v * ncoef, int(lmax), full != 0, on_sphere + v * nv, vertices,
                                          neighbours, nv, int(n_peaks), rel, thr, dirs + v * n_peaks * 3,
                                          amps + v * n_peaks, found);
    };
    std::vector<std::thread> pool;
    for (int64_t t = 1; t < n_threads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
}

}  // extern "C"
