// ORACLE — test infrastructure only. Only tests/, the smoke check and bench.py's CPU baseline
// load the library built from this file; the product path never does.
//
// FP64 CPU restatement of single-shell constrained spherical deconvolution (larmor-dmri 2.2.0):
// the problem's Gram matrix (cpp/src/sd/csd.cpp:11-22) and the per-voxel solve
// (cpp/src/sd/csd.cpp:24-65): the linear estimate initial * s, then repeated solves of
// (M^T M + norm_weight I + C_S^T C_S) f = M^T s, S the constraint rows where C f < threshold,
// until S repeats or after max_iter solves; with the chunk loop of _core.fit_csd
// (cpp/src/python/sd.cpp:171-209). The steps and the stopping rule are the reference's; the
// Cholesky factorisation and the triangular solves are this project's own code (the reference
// uses Eigen's LLT, which is not available here).
//
// Parity pins: the reference's compiled solve cannot run here (it needs Eigen), and its tests
// hold no golden solves (their MRtrix comparisons need dwi2fod). The solve is pinned by the
// reference's known-answer tests of tests/sd/test_csd.py (directions of one fibre and of
// crossings within 2 degrees, negative lobes suppressed) and by its fixed point, which
// tests/test_csd.py checks; the problem's matrices are pinned against the reference's own
// csd_problem (tests/golden/csd.npz).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

namespace oracle_csd {

// In-place Cholesky of the (n, n) row-major SPD matrix a into its lower factor, and the solve
// of L L^T x = b.
void cholesky_solve(std::vector<double>& a, int n, const std::vector<double>& b, std::vector<double>& x) {
    for (int j = 0; j < n; ++j) {
        double d = a[size_t(j) * n + j];
        for (int q = 0; q < j; ++q) d -= a[size_t(j) * n + q] * a[size_t(j) * n + q];
        d = std::sqrt(d);
        a[size_t(j) * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double s = a[size_t(i) * n + j];
            for (int q = 0; q < j; ++q) s -= a[size_t(i) * n + q] * a[size_t(j) * n + q];
            a[size_t(i) * n + j] = s / d;
        }
    }
    std::vector<double> y(size_t(n), 0.0);
    for (int i = 0; i < n; ++i) {
        double s = b[size_t(i)];
        for (int q = 0; q < i; ++q) s -= a[size_t(i) * n + q] * y[size_t(q)];
        y[size_t(i)] = s / a[size_t(i) * n + i];
    }
    x.assign(size_t(n), 0.0);
    for (int i = n - 1; i >= 0; --i) {
        double s = y[size_t(i)];
        for (int q = i + 1; q < n; ++q) s -= a[size_t(q) * n + i] * x[size_t(q)];
        x[size_t(i)] = s / a[size_t(i) * n + i];
    }
}

struct Problem {
    const double *initial, *forward, *constraint;  // (c0, m), (m, c), (k, c)
    int c0, m, c, k, max_iter;
    double threshold;
    std::vector<double> gram;  // (c, c): M^T M + norm_weight I
};

// cpp/src/sd/csd.cpp:24-65 for one signal (m,): the FOD (c,) and whether S repeated.
bool solve(const Problem& p, const double* s, double* fod_out) {
    const int c = p.c, m = p.m, k = p.k;
    std::vector<double> fod(size_t(c), 0.0), projected(size_t(c), 0.0);
    for (int r = 0; r < p.c0; ++r) {
        double acc = 0.0;
        for (int i = 0; i < m; ++i) acc += p.initial[size_t(r) * m + i] * s[i];
        fod[size_t(r)] = acc;
    }
    for (int j = 0; j < c; ++j) {
        double acc = 0.0;
        for (int i = 0; i < m; ++i) acc += p.forward[size_t(i) * c + j] * s[i];
        projected[size_t(j)] = acc;
    }
    std::vector<int> constrained, previous;
    std::vector<double> system;
    bool first = true;
    bool converged = p.max_iter == 0;
    for (int it = 0; it < p.max_iter; ++it) {
        constrained.clear();
        for (int d = 0; d < k; ++d) {
            double a = 0.0;
            for (int j = 0; j < c; ++j) a += p.constraint[size_t(d) * c + j] * fod[size_t(j)];
            if (a < p.threshold) constrained.push_back(d);
        }
        if (!first && constrained == previous) {
            converged = true;
            break;
        }
        first = false;
        system = p.gram;
        for (int d : constrained) {
            const double* row = p.constraint + size_t(d) * c;
            for (int i = 0; i < c; ++i)
                for (int j = 0; j <= i; ++j) system[size_t(i) * c + j] += row[i] * row[j];
        }
        cholesky_solve(system, c, projected, fod);
        std::swap(previous, constrained);
    }
    std::copy(fod.begin(), fod.end(), fod_out);
    return converged;
}

}  // namespace oracle_csd

extern "C" {

// _core.fit_csd (cpp/src/python/sd.cpp:171-209): fods (v, c) and converged (v,) of the signals
// (v, m); voxels split over n_threads threads. The caller checks the arguments.
void oracle_fit_csd(const double* signals, int64_t v, int64_t m, const double* initial, int64_t c0,
                    const double* forward, int64_t c, const double* constraint, int64_t k, double norm_weight,
                    double threshold, int64_t max_iter, int64_t n_threads, double* fods, uint8_t* converged) {
    oracle_csd::Problem p{initial, forward, constraint, int(c0), int(m), int(c), int(k), int(max_iter), threshold, {}};
    p.gram.assign(size_t(c * c), 0.0);
    for (int64_t i = 0; i < c; ++i)
        for (int64_t j = 0; j < c; ++j) {
            double acc = 0.0;
            for (int64_t r = 0; r < m; ++r) acc += forward[r * c + i] * forward[r * c + j];
            p.gram[size_t(i * c + j)] = acc;
        }
    for (int64_t i = 0; i < c; ++i) p.gram[size_t(i * c + i)] += norm_weight;
    auto work = [&](int64_t t) {
        for (int64_t voxel = t; voxel < v; voxel += n_threads)
            converged[voxel] = oracle_csd::solve(p, signals + voxel * m, fods + voxel * c);
    };
    std::vector<std::thread> pool;
    for (int64_t t = 1; t < n_threads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
}

}  // extern "C"
