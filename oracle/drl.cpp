// ORACLE — test infrastructure only. Only tests/, the smoke check and bench.py's CPU baseline
// load the library built from this file; the product path never does.
//
// FP64 CPU restatement of damped Richardson-Lucy deconvolution (larmor-dmri 2.2.0): the dRL
// solver's start and block solve (cpp/src/sd/solver.cpp:9-12) over damped_richardson_lucy
// (cpp/src/sd/drl.cpp:39-100), one voxel at a time (a voxel's iterations never depend on the
// others of its block). Dell'Acqua F et al., NeuroImage 49 (2010) 1446-1458.
//
// Parity pins: tests/golden/drl.npz holds the reference's numpy solver
// (tests/sd/reference_solvers.py:drl_solver) on the cases of tests/sd/test_drl.py;
// tests/test_drl.py checks this file against them at the reference's bound (rtol 1e-10).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

namespace oracle_rl {

constexpr double kFloor = 1e-6;           // cpp/src/sd/drl.cpp:13
constexpr double kOffset = 1e-16;         // cpp/src/sd/drl.cpp:16
constexpr double kConvergeShare = 1e-4;   // cpp/src/sd/drl.cpp:20

double power_8(double x) {
    const double x2 = x * x, x4 = x2 * x2;
    return x4 * x4;
}

// One voxel: signal (m,), fod (c,) holding the start on entry and the result on exit.
void solve(const double* k_t, const double* gram, int c, int m, double nu, int n_iter, const double* s,
           double* fod) {
    // Sample standard deviation (n - 1) and the largest non-NaN value of the signal.
    double mean = 0.0;
    for (int i = 0; i < m; ++i) mean += s[i];
    mean /= m;
    double ss = 0.0, largest = -INFINITY;
    bool any = false;
    for (int i = 0; i < m; ++i) {
        ss += (s[i] - mean) * (s[i] - mean);
        if (!std::isnan(s[i])) {
            largest = any ? std::max(largest, s[i]) : s[i];
            any = true;
        }
    }
    const double strength = std::fmax(1.0 - 4.0 * std::sqrt(ss / double(m - 1)), 0.0);
    const double threshold = kConvergeShare * (any ? largest : NAN);
    const double nu8 = power_8(nu);
    std::vector<double> ks(static_cast<size_t>(c));
    std::vector<double> pred(static_cast<size_t>(c));
    std::vector<double> prev(fod, fod + c);
    for (int d = 0; d < c; ++d) {
        double acc = 0.0;
        for (int i = 0; i < m; ++i) acc += k_t[size_t(d) * m + i] * s[i];
        ks[size_t(d)] = acc;
    }
    for (int it = 0; it < n_iter; ++it) {
        // pred = (K^T K) f, each entry summed over q in increasing order from 0; q outer, so that
        // the inner loop runs over independent entries.
        std::fill(pred.begin(), pred.end(), 0.0);
        for (int q = 0; q < c; ++q) {
            const double fq = fod[q];
            const double* row = gram + size_t(q) * c;
            for (int d = 0; d < c; ++d) pred[size_t(d)] += fq * row[d];
        }
        double change = 0.0;
        for (int d = 0; d < c; ++d) {
            const double a = fod[d], a8 = power_8(a);
            const double damping = 1.0 - strength * (1.0 - a8 / (a8 + nu8));
            const double ratio = (ks[size_t(d)] - pred[size_t(d)]) / (pred[size_t(d)] + kOffset);
            const double updated = std::fmax(a * (1.0 + damping * ratio), kFloor);
            fod[d] = updated;
            change += std::fabs(updated - prev[size_t(d)]);
        }
        if (change <= threshold) return;
        std::copy(fod, fod + c, prev.begin());
    }
}

}  // namespace oracle_rl

extern "C" {

// _core.fit_single_tissue with a dRL solver (cpp/src/python/sd.cpp, cpp/src/sd/solver.cpp:9-12):
// fods (v, c) from the signals (v, m), K^T (c, m), K^T K (c, c), each voxel started at init.
void oracle_drl(const double* signals, int64_t v, int64_t m, const double* k_t, const double* gram, int64_t c,
                double nu, int64_t n_iter, double init, int64_t n_threads, double* fods) {
    auto work = [&](int64_t t) {
        for (int64_t voxel = t; voxel < v; voxel += n_threads) {
            double* f = fods + voxel * c;
            std::fill(f, f + c, init);
            oracle_rl::solve(k_t, gram, int(c), int(m), nu, int(n_iter), signals + voxel * m, f);
        }
    };
    std::vector<std::thread> pool;
    for (int64_t t = 1; t < n_threads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
}

}  // extern "C"
