// ORACLE — test infrastructure only. Only tests/, the smoke check and bench.py's CPU baseline
// load the library built from this file; the product path never does.
//
// FP64 CPU restatement of Larmor's voxelwise fitting hot path (larmor-dmri 2.2.0). Each
// function names the reference file:line it follows (paths within the reference project).
// The algorithms, tolerances, tie rules and iteration caps are the reference's; the code is
// this project's own, on the small dense LA of dense.hpp instead of Eigen.
//
// Parity pins: tests/golden holds the reference's own fixtures (MRtrix DT/DKT fits of the CFIN
// block, the MRIToolkit mFOD fit) and outputs of the reference's numpy oracles on the same
// inputs; tests/test_oracle.py checks this file against them.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <limits>
#include <mutex>
#include <optional>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "dense.hpp"

namespace oracle_rl {
// Damped Richardson-Lucy of one voxel (drl.cpp): fod holds the start on entry.
void solve(const double* k_t, const double* gram, int c, int m, double nu, int n_iter, const double* s,
           double* fod);
}  // namespace oracle_rl

namespace oracle {

namespace {

constexpr double INF = std::numeric_limits<double>::infinity();

// Runs body(begin, end) over blocks of items on n_threads threads with an atomic block counter;
// the per-item work is independent, so the result does not depend on n_threads.
// Follows cpp/src/common/parallel.hpp:26-86.
template <class Body>
void parallel_blocks(Index n_items, Index block, int n_threads, Body body) {
    const Index n_blocks = (n_items + block - 1) / block;
    if (n_blocks == 0) return;
    std::atomic<Index> next{0};
    std::exception_ptr error;
    std::mutex error_mutex;
    auto run = [&] {
        try {
            for (;;) {
                const Index b = next.fetch_add(1);
                if (b >= n_blocks) break;
                body(b * block, std::min(n_items, (b + 1) * block));
            }
        } catch (...) {
            std::lock_guard<std::mutex> lock(error_mutex);
            if (!error) error = std::current_exception();
        }
    };
    const Index workers = std::max<Index>(1, std::min<Index>(n_threads, n_blocks));
    std::vector<std::thread> threads;
    for (Index w = 1; w < workers; ++w) threads.emplace_back(run);
    run();
    for (auto& t : threads) t.join();
    if (error) std::rethrow_exception(error);
}

// ---------------------------------------------------------------------------------------
// NNLS (cpp/src/sd/nnls.cpp)
// ---------------------------------------------------------------------------------------

using Active = std::vector<char>;

// 10 eps norm1(C) max(rows, cols) (cpp/src/sd/nnls.cpp:177-181).
double default_gradient_tolerance(const Mat& c) {
    double norm1 = 0.0;
    for (Index j = 0; j < c.cols; ++j) {
        double s = 0.0;
        for (Index i = 0; i < c.rows; ++i) s += std::fabs(c(i, j));
        norm1 = std::max(norm1, s);
    }
    return 10.0 * EPS * norm1 * static_cast<double>(std::max(c.rows, c.cols));
}

// Inactive column with the largest gradient, the first on a tie; -1 if none
// (cpp/src/sd/nnls.cpp:94-102).
Index steepest_inactive(const Vec& g, const Active& active) {
    Index best = -1;
    for (Index j = 0; j < static_cast<Index>(g.size()); ++j)
        if (!active[static_cast<size_t>(j)] && (best < 0 || g[static_cast<size_t>(j)] > g[static_cast<size_t>(best)])) best = j;
    return best;
}

// Least squares on the columns of `design` through a column-pivoted QR with threshold
// max(rows, cols) eps; columns beyond the rank get zero (cpp/src/sd/nnls.cpp:119-139).
Vec least_squares(const Mat& design, const Vec& data) {
    ColPivQR qr(design, static_cast<double>(std::max(design.rows, design.cols)) * EPS);
    const Index rank = qr.rank();
    Vec rotated = data;
    qr.apply_qt(rotated, rank);
    Vec head(rotated.begin(), rotated.begin() + rank);
    upper_solve(qr.qr, rank, head);
    Vec coef(static_cast<size_t>(design.cols), 0.0);
    for (Index p = 0; p < rank; ++p) coef[static_cast<size_t>(qr.perm[static_cast<size_t>(p)])] = head[static_cast<size_t>(p)];
    return coef;
}

struct Blocking {
    double step = INF;
    Index column = -1;
};

// Smallest x/(x - z) over active columns with z <= 0, the first on a tie; a column at zero
// in both gives 0 (cpp/src/sd/nnls.cpp:160-173, cpp/src/sd/lsi.cpp:234-248).
Blocking blocking_step(const Vec& x, const Vec& z, const Active& active) {
    Blocking b;
    for (Index j = 0; j < static_cast<Index>(x.size()); ++j) {
        if (!active[static_cast<size_t>(j)] || z[static_cast<size_t>(j)] > 0.0) continue;
        const double d = x[static_cast<size_t>(j)] - z[static_cast<size_t>(j)];
        const double s = d > 0.0 ? x[static_cast<size_t>(j)] / d : 0.0;
        if (s < b.step) b = {s, j};
    }
    return b;
}

struct NnlsResult {
    Vec x;
    bool converged = true;
};

// The Lawson-Hanson loop (cpp/src/sd/nnls.cpp:187-221).
template <class GradientAt, class FitOn>
NnlsResult lawson_hanson(Index n, double tol, Index max_inner, GradientAt gradient_at, FitOn fit_on) {
    Active active(static_cast<size_t>(n), 0);
    Vec x(static_cast<size_t>(n), 0.0);
    Vec g = gradient_at(x);
    Index inner = 0;
    for (;;) {
        const Index e = steepest_inactive(g, active);
        if (e < 0 || g[static_cast<size_t>(e)] <= tol) break;
        active[static_cast<size_t>(e)] = 1;
        Vec z = fit_on(active);
        for (;;) {
            bool any = false;
            for (Index j = 0; j < n; ++j)
                if (active[static_cast<size_t>(j)] && z[static_cast<size_t>(j)] <= 0.0) any = true;
            if (!any) break;
            if (++inner > max_inner) return {z, false};
            const Blocking b = blocking_step(x, z, active);
            for (Index j = 0; j < n; ++j) x[static_cast<size_t>(j)] += b.step * (z[static_cast<size_t>(j)] - x[static_cast<size_t>(j)]);
            x[static_cast<size_t>(b.column)] = 0.0;
            active[static_cast<size_t>(b.column)] = 0;
            for (Index j = 0; j < n; ++j)
                if (active[static_cast<size_t>(j)] && !(std::fabs(x[static_cast<size_t>(j)]) >= tol)) active[static_cast<size_t>(j)] = 0;
            z = fit_on(active);
        }
        x = z;
        g = gradient_at(x);
    }
    return {x, true};
}

// NNLS with the least-squares fits by QR on the active columns (cpp/src/sd/nnls.cpp:332-346).
NnlsResult solve_nnls_with_limit(const Mat& c, const Vec& d, double tol, Index max_inner) {
    const Index n = c.cols;
    auto fit_on = [&](const Active& active) {
        std::vector<Index> idx;
        for (Index j = 0; j < n; ++j)
            if (active[static_cast<size_t>(j)]) idx.push_back(j);
        Vec full(static_cast<size_t>(n), 0.0);
        if (idx.empty()) return full;
        Mat sub(c.rows, static_cast<Index>(idx.size()));
        for (Index i = 0; i < c.rows; ++i)
            for (size_t k = 0; k < idx.size(); ++k) sub(i, static_cast<Index>(k)) = c(i, idx[k]);
        const Vec coef = least_squares(sub, d);
        for (size_t k = 0; k < idx.size(); ++k) full[static_cast<size_t>(idx[k])] = coef[k];
        return full;
    };
    auto gradient_at = [&](const Vec& x) {
        Vec r = d;
        const Vec cx = matvec(c, x);
        for (Index i = 0; i < c.rows; ++i) r[static_cast<size_t>(i)] -= cx[static_cast<size_t>(i)];
        return matTvec(c, r);
    };
    return lawson_hanson(n, tol, max_inner, gradient_at, fit_on);
}

Vec solve_nnls(const Mat& c, const Vec& d, double tol) {
    return solve_nnls_with_limit(c, d, tol, 3 * c.cols).x;
}

// Removes the column at `position` from the lower Cholesky factor of n columns, keeping
// L L^T, by a row shift and Givens rotations (cpp/src/sd/nnls.cpp:305-324).
void remove_cholesky_column(Mat& f, Index n, Index position) {
    for (Index row = position; row < n - 1; ++row)
        for (Index j = 0; j < n; ++j) f(row, j) = f(row + 1, j);
    for (Index col = position; col < n - 1; ++col) {
        const double diag = f(col, col), above = f(col, col + 1);
        const double len = std::hypot(diag, above);
        const double c = diag / len, s = above / len;
        for (Index row = col; row < n - 1; ++row) {
            const double l = f(row, col), r = f(row, col + 1);
            f(row, col) = c * l + s * r;
            f(row, col + 1) = c * r - s * l;
        }
    }
}

constexpr double MIN_RELATIVE_PIVOT = 1e-12;
constexpr double MAX_NORMAL_EQUATIONS_CONDITION = 1e8;

struct RidgeDesign {
    Mat kernel;  // (m, c)
    Mat gram;    // K^T K + ridge^2 I
    double ridge = 0.0;
    bool normal_equations = false;
};

// cpp/src/sd/nnls.cpp:348-360.
RidgeDesign make_ridge_design(const Mat& k, double ridge) {
    RidgeDesign d;
    d.kernel = k;
    d.ridge = ridge;
    d.gram = Mat(k.cols, k.cols);
    double sq = 0.0;
    for (Index i = 0; i < k.rows; ++i)
        for (Index j = 0; j < k.cols; ++j) sq += k(i, j) * k(i, j);
    for (Index a = 0; a < k.cols; ++a)
        for (Index b = 0; b < k.cols; ++b) {
            double s = 0.0;
            for (Index i = 0; i < k.rows; ++i) s += k(i, a) * k(i, b);
            d.gram(a, b) = s;
        }
    for (Index a = 0; a < k.cols; ++a) d.gram(a, a) += ridge * ridge;
    const double r2 = ridge * ridge;
    d.normal_equations = r2 == 0.0 || sq + r2 <= MAX_NORMAL_EQUATIONS_CONDITION * r2;
    return d;
}

// Cholesky factor of the Gram matrix on the active columns in joining order
// (cpp/src/sd/nnls.cpp:237-301, cpp/src/sd/lsi.cpp:145-200).
template <class Gram>
struct ActiveCholesky {
    Gram gram;
    Mat factor;
    std::vector<Index> columns;
    Active in_factor;
    ActiveCholesky(Gram g, Index n) : gram(g), factor(n, n), in_factor(static_cast<size_t>(n), 0) {}

    bool append(Index column) {
        const Index pos = static_cast<Index>(columns.size());
        Vec cross(static_cast<size_t>(pos));
        for (Index r = 0; r < pos; ++r) cross[static_cast<size_t>(r)] = gram(columns[static_cast<size_t>(r)], column);
        for (Index i = 0; i < pos; ++i) {  // L w = cross
            double s = cross[static_cast<size_t>(i)];
            for (Index j = 0; j < i; ++j) s -= factor(i, j) * cross[static_cast<size_t>(j)];
            cross[static_cast<size_t>(i)] = s / factor(i, i);
        }
        double sq = 0.0;
        for (double v : cross) sq += v * v;
        const double gcc = gram(column, column);
        const double pivot = gcc - sq;
        if (!(pivot > MIN_RELATIVE_PIVOT * gcc)) return false;
        for (Index j = 0; j < pos; ++j) factor(pos, j) = cross[static_cast<size_t>(j)];
        factor(pos, pos) = std::sqrt(pivot);
        columns.push_back(column);
        in_factor[static_cast<size_t>(column)] = 1;
        return true;
    }
    void keep(const Active& active) {
        for (size_t p = columns.size(); p-- > 0;) {
            const Index col = columns[p];
            if (!active[static_cast<size_t>(col)]) {
                remove_cholesky_column(factor, static_cast<Index>(columns.size()), static_cast<Index>(p));
                columns.erase(columns.begin() + static_cast<std::ptrdiff_t>(p));
                in_factor[static_cast<size_t>(col)] = 0;
            }
        }
    }
    bool update(const Active& active) {
        keep(active);
        for (Index j = 0; j < static_cast<Index>(active.size()); ++j)
            if (active[static_cast<size_t>(j)] && !in_factor[static_cast<size_t>(j)] && !append(j)) return false;
        return true;
    }
    Vec solve(const Vec& rhs) const {
        const Index n = static_cast<Index>(columns.size());
        Vec a(static_cast<size_t>(n));
        for (Index p = 0; p < n; ++p) a[static_cast<size_t>(p)] = rhs[static_cast<size_t>(columns[static_cast<size_t>(p)])];
        for (Index i = 0; i < n; ++i) {
            double s = a[static_cast<size_t>(i)];
            for (Index j = 0; j < i; ++j) s -= factor(i, j) * a[static_cast<size_t>(j)];
            a[static_cast<size_t>(i)] = s / factor(i, i);
        }
        for (Index i = n - 1; i >= 0; --i) {
            double s = a[static_cast<size_t>(i)];
            for (Index j = i + 1; j < n; ++j) s -= factor(j, i) * a[static_cast<size_t>(j)];
            a[static_cast<size_t>(i)] = s / factor(i, i);
        }
        Vec full(rhs.size(), 0.0);
        for (Index p = 0; p < n; ++p) full[static_cast<size_t>(columns[static_cast<size_t>(p)])] = a[static_cast<size_t>(p)];
        return full;
    }
};

struct MatGram {
    const Mat* g;
    double operator()(Index r, Index c) const { return (*g)(r, c); }
};

// min ||K x - s||^2 + ridge^2 ||x||^2 + 2 l1 sum(x), x >= 0 (cpp/src/sd/nnls.cpp:362-418).
Vec solve_ridge_nnls(const RidgeDesign& d, const Vec& s, double l1, double tol) {
    if (l1 > 0 && d.ridge == 0) throw std::invalid_argument("l1 > 0 needs ridge > 0.");
    const Index m = d.kernel.rows, n = d.kernel.cols;
    Vec corr = matTvec(d.kernel, s);
    for (double& v : corr) v -= l1;
    auto gradient_at = [&](const Vec& x) {
        Vec g = corr;
        for (Index c = 0; c < n; ++c) {
            const double xc = x[static_cast<size_t>(c)];
            if (xc != 0.0)
                for (Index r = 0; r < n; ++r) g[static_cast<size_t>(r)] -= xc * d.gram(r, c);
        }
        return g;
    };
    auto fit_by_qr = [&](const Active& active) {
        std::vector<Index> idx;
        for (Index j = 0; j < n; ++j)
            if (active[static_cast<size_t>(j)]) idx.push_back(j);
        Vec full(static_cast<size_t>(n), 0.0);
        const Index na = static_cast<Index>(idx.size());
        if (na == 0) return full;
        const bool has_ridge = d.ridge > 0.0;
        Mat sub(m + (has_ridge ? na : 0), na);
        Vec data(static_cast<size_t>(sub.rows), 0.0);
        for (Index i = 0; i < m; ++i) {
            for (Index k = 0; k < na; ++k) sub(i, k) = d.kernel(i, idx[static_cast<size_t>(k)]);
            data[static_cast<size_t>(i)] = s[static_cast<size_t>(i)];
        }
        if (has_ridge)
            for (Index k = 0; k < na; ++k) {
                sub(m + k, k) = d.ridge;
                data[static_cast<size_t>(m + k)] = -l1 / d.ridge;
            }
        const Vec coef = least_squares(sub, data);
        for (Index k = 0; k < na; ++k) full[static_cast<size_t>(idx[static_cast<size_t>(k)])] = coef[static_cast<size_t>(k)];
        return full;
    };
    if (!d.normal_equations) return lawson_hanson(n, tol, 3 * n, gradient_at, fit_by_qr).x;
    ActiveCholesky<MatGram> chol(MatGram{&d.gram}, n);
    bool failed = false;
    auto fit_on = [&](const Active& active) {
        failed = failed || !chol.update(active);
        return failed ? fit_by_qr(active) : chol.solve(corr);
    };
    return lawson_hanson(n, tol, 3 * n, gradient_at, fit_on).x;
}

// ---------------------------------------------------------------------------------------
// Log-signal fit (cpp/src/dwi/log_fit.cpp)
// ---------------------------------------------------------------------------------------

constexpr double FEASIBILITY_MARGIN = 1e-12;
constexpr Index INNER_STEPS_PER_CONSTRAINT = 50;
constexpr double CONSTRAINT_TOLERANCE = 1e-9;

struct LogDesign {
    Vec scales;      // (P,)
    Mat x;           // scaled design (N, P)
    Mat pinv;        // (P, N)
    Mat g;           // scaled constraints (M, P)
};

// cpp/src/dwi/log_fit.cpp:220-236.
LogDesign make_log_design(const Mat& x, const Mat& g) {
    LogDesign d;
    const Index n = x.rows, p = x.cols;
    d.scales.assign(static_cast<size_t>(p), 0.0);
    for (Index j = 0; j < p; ++j) {
        double s = 0.0;
        for (Index i = 0; i < n; ++i) s += x(i, j) * x(i, j);
        d.scales[static_cast<size_t>(j)] = s == 0.0 ? 1.0 : std::sqrt(s);
    }
    d.x = Mat(n, p);
    for (Index i = 0; i < n; ++i)
        for (Index j = 0; j < p; ++j) d.x(i, j) = x(i, j) * (1.0 / d.scales[static_cast<size_t>(j)]);
    d.pinv = pseudo_inverse_full_rank(d.x);
    d.g = Mat(g.rows, p);
    for (Index i = 0; i < g.rows; ++i)
        for (Index j = 0; j < p; ++j) d.g(i, j) = g(i, j) * (1.0 / d.scales[static_cast<size_t>(j)]);
    return d;
}

// IRLS from the ordinary fit (cpp/src/dwi/log_fit.cpp:114-147).
Vec reweighted_fit(const LogDesign& d, Index max_rw, double tol, const Vec& y, const Vec& ordinary,
                   int* iterations) {
    *iterations = 0;
    if (!all_finite(ordinary)) return ordinary;
    const Index n = d.x.rows, p = d.x.cols;
    Vec params = ordinary;
    Vec pred = matvec(d.x, params);
    for (Index it = 0; it < max_rw; ++it) {
        const double mx = *std::max_element(pred.begin(), pred.end());
        Vec w(static_cast<size_t>(n));
        for (Index i = 0; i < n; ++i) w[static_cast<size_t>(i)] = std::exp(2.0 * (pred[static_cast<size_t>(i)] - mx));
        Mat normal(p, p);
        Vec rhs(static_cast<size_t>(p), 0.0);
        for (Index a = 0; a < p; ++a) {
            for (Index b = 0; b < p; ++b) {
                double s = 0.0;
                for (Index i = 0; i < n; ++i) s += d.x(i, a) * (w[static_cast<size_t>(i)] * d.x(i, b));
                normal(a, b) = s;
            }
            double r = 0.0;
            for (Index i = 0; i < n; ++i) r += (w[static_cast<size_t>(i)] * d.x(i, a)) * y[static_cast<size_t>(i)];
            rhs[static_cast<size_t>(a)] = r;
        }
        PartialPivLU lu(normal);
        ++*iterations;
        if (lu.zero_pivot) return ordinary;
        const Vec next = lu.solve(rhs);
        if (!all_finite(next)) return ordinary;
        const Vec next_pred = matvec(d.x, next);
        double change = 0.0;
        for (Index i = 0; i < n; ++i) change = std::max(change, std::fabs(next_pred[static_cast<size_t>(i)] - pred[static_cast<size_t>(i)]));
        params = next;
        pred = next_pred;
        if (!(change > tol)) break;
    }
    return params;
}

bool breaks_a_constraint(const LogDesign& d, const Vec& p) {
    const Vec v = matvec(d.g, p);
    return *std::min_element(v.begin(), v.end()) < 0.0;
}

// cpp/src/dwi/log_fit.cpp:156-163.
bool meets_the_constraints(const LogDesign& d, const Vec& p, const Vec& start) {
    const Vec v = matvec(d.g, p);
    double size = 0.0;
    for (Index i = 0; i < d.g.rows; ++i) {
        double s = 0.0;
        for (Index j = 0; j < d.g.cols; ++j)
            s += std::fabs(d.g(i, j)) * (std::fabs(p[static_cast<size_t>(j)]) + std::fabs(start[static_cast<size_t>(j)]));
        size = std::max(size, s);
    }
    return *std::min_element(v.begin(), v.end()) >= -CONSTRAINT_TOLERANCE * size;
}

// The constrained re-fit through least distance and NNLS (cpp/src/dwi/log_fit.cpp:170-216).
Vec constrained_fit(const LogDesign& d, const Vec& y, const Vec& root_w, const Vec& params) {
    const Index n = d.x.rows, p = d.x.cols, m = d.g.rows;
    Mat wx(n, p);
    for (Index i = 0; i < n; ++i)
        for (Index j = 0; j < p; ++j) wx(i, j) = root_w[static_cast<size_t>(i)] * d.x(i, j);
    HouseholderQR qr(wx);
    Vec rotated(static_cast<size_t>(n));
    for (Index i = 0; i < n; ++i) rotated[static_cast<size_t>(i)] = root_w[static_cast<size_t>(i)] * y[static_cast<size_t>(i)];
    qr.apply_qt(rotated);
    double dmax = 0.0, dmin = INF;
    for (Index k = 0; k < p; ++k) {
        dmax = std::max(dmax, std::fabs(qr.qr(k, k)));
        dmin = std::min(dmin, std::fabs(qr.qr(k, k)));
    }
    const double rank_tol = static_cast<double>(n) * EPS * dmax;
    if (!(dmin > rank_tol)) return params;
    Vec free_sol(rotated.begin(), rotated.begin() + p);
    upper_solve(qr.qr, p, free_sol);

    Mat ld(p + 1, m);
    for (Index c = 0; c < m; ++c) {
        Vec col(static_cast<size_t>(p));
        for (Index j = 0; j < p; ++j) col[static_cast<size_t>(j)] = d.g(c, j);
        upper_transpose_solve(qr.qr, p, col);
        for (Index j = 0; j < p; ++j) ld(j, c) = col[static_cast<size_t>(j)];
    }
    const Vec gf = matvec(d.g, free_sol);
    for (Index c = 0; c < m; ++c) ld(p, c) = -gf[static_cast<size_t>(c)];
    Vec unit(static_cast<size_t>(p + 1), 0.0);
    unit[static_cast<size_t>(p)] = 1.0;
    const NnlsResult u = solve_nnls_with_limit(ld, unit, default_gradient_tolerance(ld), INNER_STEPS_PER_CONSTRAINT * m);
    if (!u.converged) return params;
    Vec res = matvec(ld, u.x);
    for (Index i = 0; i <= p; ++i) res[static_cast<size_t>(i)] -= unit[static_cast<size_t>(i)];
    if (res[static_cast<size_t>(p)] >= -FEASIBILITY_MARGIN) return params;
    Vec dist(static_cast<size_t>(p));
    for (Index j = 0; j < p; ++j) dist[static_cast<size_t>(j)] = -res[static_cast<size_t>(j)] / res[static_cast<size_t>(p)];
    upper_solve(qr.qr, p, dist);
    Vec out(static_cast<size_t>(p));
    for (Index j = 0; j < p; ++j) out[static_cast<size_t>(j)] = free_sol[static_cast<size_t>(j)] + dist[static_cast<size_t>(j)];
    if (!all_finite(out) || !meets_the_constraints(d, out, free_sol)) return params;
    return out;
}

// One voxel of fit_log_signal_block (cpp/src/dwi/log_fit.cpp:245-269).
void fit_log_voxel(const LogDesign& d, bool weighted, Index max_rw, double tol, const double* y_row,
                   double* out_params, unsigned char* out_broke, int* out_iters) {
    const Index n = d.x.rows, p = d.x.cols;
    Vec y(y_row, y_row + n);
    const Vec ordinary = matvec(d.pinv, y);
    int iters = 0;
    Vec params = weighted ? reweighted_fit(d, max_rw, tol, y, ordinary, &iters) : ordinary;
    const bool constrain = d.g.rows > 0 && all_finite(params) && breaks_a_constraint(d, params);
    if (constrain) {
        Vec root_w(static_cast<size_t>(n), 1.0);
        if (weighted) {
            const Vec pred = matvec(d.x, params);
            const double mx = *std::max_element(pred.begin(), pred.end());
            for (Index i = 0; i < n; ++i) root_w[static_cast<size_t>(i)] = std::exp(pred[static_cast<size_t>(i)] - mx);
        }
        params = constrained_fit(d, y, root_w, params);
    }
    for (Index j = 0; j < p; ++j) out_params[j] = params[static_cast<size_t>(j)] / d.scales[static_cast<size_t>(j)];
    *out_broke = constrain ? 1 : 0;
    if (out_iters) *out_iters = iters;
}

// ---------------------------------------------------------------------------------------
// LSI (cpp/src/sd/lsi.cpp)
// ---------------------------------------------------------------------------------------

struct LsiDesign {
    Mat q_t;        // (n, m)
    Mat back;       // (n, n)
    Mat e;          // (k, n) unit rows
    Mat gram;       // (k, k)
    Vec abs_sums;   // (k,)
};

// cpp/src/sd/lsi.cpp:75-125.
LsiDesign make_lsi_design(const Mat& a, const Mat& g, double ridge) {
    const Index m = a.rows, n = a.cols;
    if (g.cols != n) throw std::invalid_argument("the constraints have " + std::to_string(g.cols) + " columns but the design has " + std::to_string(n));
    if (!(ridge >= 0.0)) throw std::invalid_argument("the ridge must be at least 0");
    const bool has_ridge = ridge > 0.0;
    Mat stacked(m + (has_ridge ? n : 0), n);
    for (Index i = 0; i < m; ++i)
        for (Index j = 0; j < n; ++j) stacked(i, j) = a(i, j);
    if (has_ridge)
        for (Index j = 0; j < n; ++j) stacked(m + j, j) = ridge;
    ColPivQR qr(stacked, static_cast<double>(std::max(stacked.rows, stacked.cols)) * EPS);
    if (stacked.rows < n || qr.rank() < n)
        throw std::invalid_argument("the design does not have full column rank: the measurements cannot determine all " + std::to_string(n) + " parameters");
    LsiDesign d;
    // Thin Q: columns Q e_k, k < n.
    d.q_t = Mat(n, m);
    for (Index k = 0; k < n; ++k) {
        Vec e(static_cast<size_t>(stacked.rows), 0.0);
        e[static_cast<size_t>(k)] = 1.0;
        for (Index r = n - 1; r >= 0; --r) apply_householder_vec(qr.qr, r, r, qr.tau[static_cast<size_t>(r)], e);
        for (Index i = 0; i < m; ++i) d.q_t(k, i) = e[static_cast<size_t>(i)];
    }
    // R^-1, then P R^-1 (row perm[k] of the result is row k of R^-1).
    Mat rinv(n, n);
    for (Index c = 0; c < n; ++c) {
        Vec e(static_cast<size_t>(n), 0.0);
        e[static_cast<size_t>(c)] = 1.0;
        upper_solve(qr.qr, n, e);
        for (Index r = 0; r < n; ++r) rinv(r, c) = e[static_cast<size_t>(r)];
    }
    d.back = Mat(n, n);
    for (Index k = 0; k < n; ++k)
        for (Index c = 0; c < n; ++c) d.back(qr.perm[static_cast<size_t>(k)], c) = rinv(k, c);
    const Index kc = g.rows;
    d.e = Mat(kc, n);
    for (Index i = 0; i < kc; ++i) {
        double nrm = 0.0;
        for (Index c = 0; c < n; ++c) {
            double s = 0.0;
            for (Index j = 0; j < n; ++j) s += g(i, j) * d.back(j, c);
            d.e(i, c) = s;
            nrm += s * s;
        }
        nrm = std::sqrt(nrm);
        if (nrm > 0.0)
            for (Index c = 0; c < n; ++c) d.e(i, c) /= nrm;
    }
    d.gram = Mat(kc, kc);
    d.abs_sums.assign(static_cast<size_t>(kc), 0.0);
    for (Index i = 0; i < kc; ++i) {
        for (Index j = 0; j < kc; ++j) {
            double s = 0.0;
            for (Index c = 0; c < n; ++c) s += d.e(i, c) * d.e(j, c);
            d.gram(i, j) = s;
        }
        double s = 0.0;
        for (Index c = 0; c < n; ++c) s += std::fabs(d.e(i, c));
        d.abs_sums[static_cast<size_t>(i)] = s;
    }
    return d;
}

struct LdpGram {
    const Mat* gram;
    const Vec* f;
    double operator()(Index r, Index c) const { return (*gram)(r, c) + (*f)[static_cast<size_t>(r)] * (*f)[static_cast<size_t>(c)]; }
};

// cpp/src/sd/lsi.cpp:253-297; the count of outer steps goes to *outer.
std::optional<Vec> ldp_multipliers(const LsiDesign& d, const Vec& f, int* outer) {
    const Index k = static_cast<Index>(f.size());
    double norm1 = 0.0;
    for (Index i = 0; i < k; ++i) norm1 = std::max(norm1, d.abs_sums[static_cast<size_t>(i)] + std::fabs(f[static_cast<size_t>(i)]));
    const double tol = 10.0 * EPS * norm1 * static_cast<double>(std::max(d.back.rows + 1, k));
    const Index max_inner = 3 * k;
    Active active(static_cast<size_t>(k), 0);
    ActiveCholesky<LdpGram> chol(LdpGram{&d.gram, &f}, k);
    Vec u(static_cast<size_t>(k), 0.0);
    Index inner = 0;
    *outer = 0;
    for (;;) {
        double fu = 0.0;
        for (Index i = 0; i < k; ++i) fu += f[static_cast<size_t>(i)] * u[static_cast<size_t>(i)];
        Vec grad(static_cast<size_t>(k));
        for (Index i = 0; i < k; ++i) grad[static_cast<size_t>(i)] = f[static_cast<size_t>(i)] * (1.0 - fu);
        for (Index c = 0; c < k; ++c) {
            const double uc = u[static_cast<size_t>(c)];
            if (uc != 0.0)
                for (Index i = 0; i < k; ++i) grad[static_cast<size_t>(i)] -= uc * d.gram(c, i);
        }
        const Index e = steepest_inactive(grad, active);
        if (e < 0 || grad[static_cast<size_t>(e)] <= tol) return u;
        ++*outer;
        active[static_cast<size_t>(e)] = 1;
        if (!chol.append(e)) return std::nullopt;
        Vec z = chol.solve(f);
        for (Blocking b = blocking_step(u, z, active); b.column >= 0; b = blocking_step(u, z, active)) {
            if (++inner > max_inner) return std::nullopt;
            for (Index i = 0; i < k; ++i) u[static_cast<size_t>(i)] += b.step * (z[static_cast<size_t>(i)] - u[static_cast<size_t>(i)]);
            u[static_cast<size_t>(b.column)] = 0.0;
            for (Index i = 0; i < k; ++i)
                if (i == b.column || std::fabs(u[static_cast<size_t>(i)]) < tol) {
                    active[static_cast<size_t>(i)] = 0;
                    u[static_cast<size_t>(i)] = 0.0;
                }
            chol.keep(active);
            z = chol.solve(f);
        }
        u = z;
    }
}

// cpp/src/sd/lsi.cpp:301-338. *status: 0 fast path, 1 QR fallback, 2 f = 0.
bool solve_lsi(const LsiDesign& d, const double* s, bool only_qr, double* out, int* status,
               int* outer, unsigned char* active_out) {
    const Index n = d.back.rows, k = d.e.rows, m = d.q_t.cols;
    Vec data(s, s + m);
    const Vec rot = matvec(d.q_t, data);
    Vec raw = matvec(d.e, rot);
    double scale = 0.0;
    for (double& v : raw) {
        v = -v;
        scale = std::max(scale, std::fabs(v));
    }
    *outer = 0;
    if (!(scale > 0.0)) {
        const Vec x = matvec(d.back, rot);
        std::copy(x.begin(), x.end(), out);
        *status = 2;
        if (active_out) std::fill(active_out, active_out + k, 0);
        return true;
    }
    Vec f(static_cast<size_t>(k));
    for (Index i = 0; i < k; ++i) f[static_cast<size_t>(i)] = raw[static_cast<size_t>(i)] / scale;
    Vec u;
    bool converged = true;
    std::optional<Vec> fast = only_qr ? std::nullopt : ldp_multipliers(d, f, outer);
    if (fast) {
        u = *fast;
        *status = 0;
    } else {
        Mat c(n + 1, k);
        for (Index i = 0; i < n; ++i)
            for (Index j = 0; j < k; ++j) c(i, j) = d.e(j, i);
        for (Index j = 0; j < k; ++j) c(n, j) = f[static_cast<size_t>(j)];
        Vec target(static_cast<size_t>(n + 1), 0.0);
        target[static_cast<size_t>(n)] = 1.0;
        NnlsResult r = solve_nnls_with_limit(c, target, default_gradient_tolerance(c), 3 * k);
        u = r.x;
        converged = r.converged;
        *status = 1;
    }
    double fu = 0.0;
    for (Index i = 0; i < k; ++i) fu += f[static_cast<size_t>(i)] * u[static_cast<size_t>(i)];
    const Vec etu = matTvec(d.e, u);
    Vec z(static_cast<size_t>(n));
    for (Index i = 0; i < n; ++i) z[static_cast<size_t>(i)] = scale * etu[static_cast<size_t>(i)] / (1.0 - fu) + rot[static_cast<size_t>(i)];
    const Vec x = matvec(d.back, z);
    std::copy(x.begin(), x.end(), out);
    if (active_out)
        for (Index i = 0; i < k; ++i) active_out[i] = u[static_cast<size_t>(i)] != 0.0 ? 1 : 0;
    return converged;
}

// ---------------------------------------------------------------------------------------
// Fractions and the multi-tissue loop (cpp/src/sd/fractions.cpp, cpp/src/sd/multi_tissue.cpp)
// ---------------------------------------------------------------------------------------

constexpr double MEDIAN_TIE_TOLERANCE = 1e-9;
constexpr double FRACTION_SUM_OFFSET = 1e-16;

bool less_nan_last(double l, double r) { return std::isnan(r) ? !std::isnan(l) : l < r; }

// cpp/src/sd/fractions.cpp:56-68.
double median(const Vec& values) {
    Vec s = values;
    if (s.empty()) return std::numeric_limits<double>::quiet_NaN();
    auto mid = s.begin() + static_cast<std::ptrdiff_t>(s.size() / 2);
    std::nth_element(s.begin(), mid, s.end(), less_nan_last);
    if (s.size() % 2 == 1) return *mid;
    const double lower = *std::max_element(s.begin(), mid, less_nan_last);
    return (lower + *mid) / 2.0;
}

struct TissueKernel {
    Mat aniso;       // (m, ca)
    Mat iso;         // (m, ci)
    Mat w_iso;       // (m, ci)
    std::vector<std::pair<Index, Index>> blocks;
};

// cpp/src/sd/fractions.cpp:70-101. per_block false: one lumped anisotropic column.
Vec compute_fractions(const Vec& fod, const TissueKernel& k, const double* signal, bool per_block,
                      const double* tol) {
    const double threshold = median(fod) * (1.0 - MEDIAN_TIE_TOLERANCE);
    Vec th = fod;
    for (double& v : th)
        if (v < threshold) v = 0.0;
    std::vector<std::pair<Index, Index>> groups;
    if (per_block) groups = k.blocks;
    else groups.push_back({0, k.aniso.cols});
    const Index ng = static_cast<Index>(groups.size()), ci = k.iso.cols, m = k.aniso.rows;
    Mat cols(m, ng + ci);
    for (Index gi = 0; gi < ng; ++gi) {
        const auto [b, e] = groups[static_cast<size_t>(gi)];
        Vec gs(static_cast<size_t>(m), 0.0);
        for (Index i = 0; i < m; ++i) {
            double s = 0.0;
            for (Index j = b; j < e; ++j) s += k.aniso(i, j) * th[static_cast<size_t>(j)];
            gs[static_cast<size_t>(i)] = s;
        }
        if (m > 0) {
            double largest = -INF;
            bool any = false;
            for (double v : gs)
                if (!std::isnan(v)) {
                    largest = any ? std::max(largest, v) : v;
                    any = true;
                }
            if (!any) largest = std::numeric_limits<double>::quiet_NaN();
            if (largest > 0.0)
                for (double& v : gs) v /= largest;
        }
        for (Index i = 0; i < m; ++i) cols(i, gi) = gs[static_cast<size_t>(i)];
    }
    for (Index i = 0; i < m; ++i)
        for (Index j = 0; j < ci; ++j) cols(i, ng + j) = k.iso(i, j);
    const double t = tol ? *tol : default_gradient_tolerance(cols);
    return solve_nnls(cols, Vec(signal, signal + m), t);
}

Vec anisotropic_signal(const double* ws, const Mat& w_iso, const Vec& f_iso) {
    const Index m = w_iso.rows;
    Vec r(static_cast<size_t>(m));
    for (Index i = 0; i < m; ++i) {
        double s = 0.0;
        for (Index j = 0; j < w_iso.cols; ++j) s += w_iso(i, j) * f_iso[static_cast<size_t>(j)];
        r[static_cast<size_t>(i)] = std::fmax(ws[i] - s, 0.0);
    }
    return r;
}

// The FOD solve of one stage of the multi-tissue fit: the ridge NNLS (L2NNLS, plain NNLS in the
// rounds) or, when k_t is set, damped Richardson-Lucy from init (GRL;
// cpp/src/sd/solver.cpp:9-12).
struct StageSolver {
    const RidgeDesign* design = nullptr;
    double tol = 0.0;
    const double* k_t = nullptr;   // (c, m)
    const double* gram = nullptr;  // (c, c)
    Index c = 0, m = 0;
    double nu = 0.0, init = 0.0;
    Index n_iter = 0;
    Vec operator()(const Vec& as) const {
        if (k_t == nullptr) return solve_ridge_nnls(*design, as, 0.0, tol);
        Vec fod(static_cast<size_t>(c), init);
        oracle_rl::solve(k_t, gram, int(c), int(m), nu, int(n_iter), as.data(), fod.data());
        return fod;
    }
};

// One voxel of fit_multi_tissue_block (cpp/src/sd/multi_tissue.cpp:76-148); the loop's rounds
// are independent per voxel, so a voxel alone gives the block's result
// (cpp/tests/sd/test_multi_tissue.cpp:56).
void fit_multi_tissue_voxel(const double* signal, const Vec& weights, const TissueKernel& lr,
                            const StageSolver& lr_solve, const TissueKernel& hr, const StageSolver& hr_solve,
                            Index max_rounds, double fraction_tol, double final_tol, double* out_fod,
                            double* out_fractions, int* out_rounds) {
    const Index m = lr.aniso.rows, ci = lr.iso.cols;
    Vec ws(static_cast<size_t>(m));
    for (Index i = 0; i < m; ++i) ws[static_cast<size_t>(i)] = signal[i] * weights[static_cast<size_t>(i)];
    Vec f_iso(static_cast<size_t>(ci), 0.0);
    Vec prev(static_cast<size_t>(1 + ci), INF);
    int rounds = 0;
    for (Index round = 0; round < max_rounds; ++round) {
        ++rounds;
        const Vec as = anisotropic_signal(ws.data(), lr.w_iso, f_iso);
        const Vec fod = lr_solve(as);
        const Vec fr = compute_fractions(fod, lr, signal, false, nullptr);
        for (Index j = 0; j < ci; ++j) f_iso[static_cast<size_t>(j)] = fr[static_cast<size_t>(1 + j)];
        bool converged = true;
        for (Index j = 0; j < 1 + ci; ++j)
            if (!(std::fabs(fr[static_cast<size_t>(j)] - prev[static_cast<size_t>(j)]) < fraction_tol)) converged = false;
        if (converged) break;
        prev = fr;
    }
    const Vec as = anisotropic_signal(ws.data(), hr.w_iso, f_iso);
    const Vec fod = hr_solve(as);
    std::copy(fod.begin(), fod.end(), out_fod);
    const Vec fr = compute_fractions(fod, hr, signal, true, &final_tol);
    double total = FRACTION_SUM_OFFSET;
    for (double v : fr) total += v;
    for (size_t j = 0; j < fr.size(); ++j) out_fractions[j] = fr[j] / total;
    if (out_rounds) *out_rounds = rounds;
}

std::string last_error;

template <class F>
int guarded(F f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        last_error = e.what();
        return 1;
    }
}

}  // namespace

}  // namespace oracle

using namespace oracle;

extern "C" {

const char* oracle_last_error() { return oracle::last_error.c_str(); }

// fit_log_signal over v voxels (cpp/src/python/dwi.cpp:42-82): x (n, p), g (m, p), log_s (v, n);
// params (v, p), broke (v,), iterations (v,) or null.
int oracle_fit_log_signal(const double* x, Index n, Index p, const double* g, Index m,
                          const double* log_s, Index v, int weighted, Index max_rw, double tol,
                          int n_threads, double* params, unsigned char* broke, int* iterations) {
    return guarded([&] {
        if (n < p) throw std::invalid_argument("x must be (n, p) with n >= p");
        if (max_rw < 0) throw std::invalid_argument("max_iter must be at least 0");
        const LogDesign d = make_log_design(Mat::from(x, n, p), Mat::from(g, m, p));
        parallel_blocks(v, 64, n_threads, [&](Index b, Index e) {
            for (Index i = b; i < e; ++i)
                fit_log_voxel(d, weighted != 0, max_rw, tol, log_s + i * n, params + i * p, broke + i,
                              iterations ? iterations + i : nullptr);
        });
    });
}

// Scaled design, pseudo-inverse and scales, for tests of the design preparation.
int oracle_log_design(const double* x, Index n, Index p, double* scales, double* pinv) {
    return guarded([&] {
        const LogDesign d = make_log_design(Mat::from(x, n, p), Mat(0, p));
        std::copy(d.scales.begin(), d.scales.end(), scales);
        std::copy(d.pinv.a.begin(), d.pinv.a.end(), pinv);
    });
}

// LsiDesign (cpp/src/sd/lsi.cpp:75): a (m, n), g (k, n). Writes q_t (n, m), back (n, n),
// e (k, n), gram (k, k), abs_sums (k,).
int oracle_lsi_design(const double* a, Index m, Index n, const double* g, Index k, double ridge,
                      double* q_t, double* back, double* e, double* gram, double* abs_sums) {
    return guarded([&] {
        const LsiDesign d = make_lsi_design(Mat::from(a, m, n), Mat::from(g, k, n), ridge);
        std::copy(d.q_t.a.begin(), d.q_t.a.end(), q_t);
        std::copy(d.back.a.begin(), d.back.a.end(), back);
        std::copy(d.e.a.begin(), d.e.a.end(), e);
        std::copy(d.gram.a.begin(), d.gram.a.end(), gram);
        std::copy(d.abs_sums.begin(), d.abs_sums.end(), abs_sums);
    });
}

// fit_lsi (cpp/src/python/sd.cpp:370): signals (v, m) -> x (v, n), converged (v,); status
// (v,) 0 fast, 1 QR fallback, 2 f = 0; outer (v,) outer steps; active (v, k) or null.
int oracle_fit_lsi(const double* a, Index m, Index n, const double* g, Index k, double ridge,
                   const double* signals, Index v, int only_qr, int n_threads, double* x,
                   unsigned char* converged, int* status, int* outer, unsigned char* active) {
    return guarded([&] {
        const LsiDesign d = make_lsi_design(Mat::from(a, m, n), Mat::from(g, k, n), ridge);
        parallel_blocks(v, 128, n_threads, [&](Index b, Index e) {
            for (Index i = b; i < e; ++i)
                converged[i] = solve_lsi(d, signals + i * m, only_qr != 0, x + i * n, status + i,
                                         outer + i, active ? active + i * k : nullptr)
                                   ? 1 : 0;
        });
    });
}

// solve_nnls_with_limit (cpp/src/sd/nnls.cpp:332): c (rows, cols), d (rows,), tol < 0 for the
// default tolerance, max_inner < 0 for 3 * cols.
int oracle_nnls(const double* c, Index rows, Index cols, const double* d, double tol,
                Index max_inner, double* x, unsigned char* converged) {
    return guarded([&] {
        const Mat cm = Mat::from(c, rows, cols);
        const double t = tol < 0 ? default_gradient_tolerance(cm) : tol;
        const NnlsResult r = solve_nnls_with_limit(cm, Vec(d, d + rows), t, max_inner < 0 ? 3 * cols : max_inner);
        std::copy(r.x.begin(), r.x.end(), x);
        *converged = r.converged ? 1 : 0;
    });
}

// FodSolver.l2nnls + fit_single_tissue (cpp/src/sd/solver.cpp:422-429): k (m, c), signals
// (v, m) -> fods (v, c).
int oracle_ridge_nnls(const double* k, Index m, Index c, double ridge, double tol_x,
                      const double* signals, Index v, int n_threads, double* fods) {
    return guarded([&] {
        const RidgeDesign d = make_ridge_design(Mat::from(k, m, c), ridge);
        parallel_blocks(v, 128, n_threads, [&](Index b, Index e) {
            for (Index i = b; i < e; ++i) {
                const Vec f = solve_ridge_nnls(d, Vec(signals + i * m, signals + (i + 1) * m), 0.0, tol_x);
                std::copy(f.begin(), f.end(), fods + i * c);
            }
        });
    });
}

// fit_multi_tissue (cpp/src/python/sd.cpp:310). Kernels: k_aniso (m, ca), k_iso and w_k_iso
// (m, ci); blocks as (start, stop) pairs. Each stage solves by the ridge NNLS of its weighted
// kernel w_aniso, or, when its k_t is not NULL, by damped Richardson-Lucy with K^T = k_t
// (ca, m), K^T K = gram (ca, ca), nu, n_iter and init.
int oracle_fit_multi_tissue(const double* signals, Index v, Index m, const double* weights,
                            const double* lr_aniso, Index lr_ca, const double* lr_iso,
                            const double* lr_w_iso, const double* lr_w_aniso, double lr_ridge,
                            double lr_tol, const double* hr_aniso, Index hr_ca,
                            const double* hr_iso, const double* hr_w_iso,
                            const double* hr_w_aniso, double hr_ridge, double hr_tol, Index ci,
                            const Index* blocks, Index n_blocks, Index max_rounds,
                            double fraction_tol, double final_tol, int n_threads, double* fods,
                            double* fractions, int* rounds, const double* lr_k_t, const double* lr_gram,
                            double lr_nu, Index lr_n_iter, double lr_init, const double* hr_k_t,
                            const double* hr_gram, double hr_nu, Index hr_n_iter, double hr_init) {
    return guarded([&] {
        TissueKernel lr{Mat::from(lr_aniso, m, lr_ca), Mat::from(lr_iso, m, ci), Mat::from(lr_w_iso, m, ci), {}};
        TissueKernel hr{Mat::from(hr_aniso, m, hr_ca), Mat::from(hr_iso, m, ci), Mat::from(hr_w_iso, m, ci), {}};
        for (Index b = 0; b < n_blocks; ++b) hr.blocks.push_back({blocks[2 * b], blocks[2 * b + 1]});
        lr.blocks = {{0, lr_ca}};
        const RidgeDesign lr_d = make_ridge_design(Mat::from(lr_w_aniso, m, lr_ca), lr_ridge);
        const RidgeDesign hr_d = make_ridge_design(Mat::from(hr_w_aniso, m, hr_ca), hr_ridge);
        const StageSolver lr_s{&lr_d, lr_tol, lr_k_t, lr_gram, lr_ca, m, lr_nu, lr_init, lr_n_iter};
        const StageSolver hr_s{&hr_d, hr_tol, hr_k_t, hr_gram, hr_ca, m, hr_nu, hr_init, hr_n_iter};
        const Vec w(weights, weights + m);
        const Index nf = n_blocks + ci;
        parallel_blocks(v, 128, n_threads, [&](Index b, Index e) {
            for (Index i = b; i < e; ++i)
                fit_multi_tissue_voxel(signals + i * m, w, lr, lr_s, hr, hr_s, max_rounds, fraction_tol, final_tol,
                                       fods + i * hr_ca, fractions + i * nf, rounds ? rounds + i : nullptr);
        });
    });
}

// median (cpp/src/sd/fractions.cpp:56), for tests.
double oracle_median(const double* values, Index n) { return median(Vec(values, values + n)); }

}  // extern "C"
