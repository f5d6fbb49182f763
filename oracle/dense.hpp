// ORACLE — test infrastructure only. Nothing in the product path links or calls this file.
//
// Small dense FP64 linear algebra for the CPU restatement of Larmor's fitting hot path:
// row-major matrices, Householder QR (plain and with column pivoting), LU with partial
// pivoting, triangular solves. The decompositions follow the published algorithms that
// Larmor's C++ core relies on through Eigen 5.0.1 (cpp/cmake/third_party.cmake:5-7), with the
// same pivot rules, so that the rank decisions and tie-breaks of the reference carry over:
//   - Householder reflector: beta = -sign(c0) ||x||, tau = (beta - c0) / beta,
//     essential part = tail / (c0 - beta) (Golub & Van Loan 5.1.2; LAPACK dlarfg).
//   - Column-pivoted QR (Businger & Golub 1965): the column of largest remaining norm, the
//     first on a tie; norms downdated as in LAPACK dgeqp3 (Drmac & Bujanovic 2008) and
//     recomputed when the downdate loses more than half the digits.
//   - LU with partial pivoting: the row of largest magnitude, the first on a tie; a zero
//     pivot is kept and reported through the diagonal.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

namespace oracle {

using Index = std::int64_t;
constexpr double EPS = std::numeric_limits<double>::epsilon();

// A row-major matrix of doubles.
struct Mat {
    Index rows = 0, cols = 0;
    std::vector<double> a;
    Mat() = default;
    Mat(Index r, Index c, double fill = 0.0) : rows(r), cols(c), a(static_cast<size_t>(r * c), fill) {}
    double& operator()(Index i, Index j) { return a[static_cast<size_t>(i * cols + j)]; }
    double operator()(Index i, Index j) const { return a[static_cast<size_t>(i * cols + j)]; }
    static Mat from(const double* p, Index r, Index c) {
        Mat m(r, c);
        std::copy(p, p + r * c, m.a.begin());
        return m;
    }
};

using Vec = std::vector<double>;

inline Vec matvec(const Mat& m, const Vec& x) {
    Vec y(static_cast<size_t>(m.rows), 0.0);
    for (Index i = 0; i < m.rows; ++i) {
        double s = 0.0;
        for (Index j = 0; j < m.cols; ++j) s += m(i, j) * x[static_cast<size_t>(j)];
        y[static_cast<size_t>(i)] = s;
    }
    return y;
}

inline Vec matTvec(const Mat& m, const Vec& x) {
    Vec y(static_cast<size_t>(m.cols), 0.0);
    for (Index i = 0; i < m.rows; ++i) {
        const double xi = x[static_cast<size_t>(i)];
        for (Index j = 0; j < m.cols; ++j) y[static_cast<size_t>(j)] += m(i, j) * xi;
    }
    return y;
}

inline bool all_finite(const Vec& v) {
    for (double x : v)
        if (!std::isfinite(x)) return false;
    return true;
}

// Makes the reflector H = I - tau v v^T, v = (1, essential), with H x = (beta, 0, ...), for the
// column x = m(row0.., col) in place: m(row0, col) is left untouched (the caller writes beta),
// the essential part replaces the entries below it.
inline void make_householder(Mat& m, Index row0, Index col, double& tau, double& beta) {
    const double c0 = m(row0, col);
    double tail_sq = 0.0;
    for (Index i = row0 + 1; i < m.rows; ++i) tail_sq += m(i, col) * m(i, col);
    if (tail_sq <= std::numeric_limits<double>::min()) {
        tau = 0.0;
        beta = c0;
        for (Index i = row0 + 1; i < m.rows; ++i) m(i, col) = 0.0;
        return;
    }
    beta = std::sqrt(c0 * c0 + tail_sq);
    if (c0 >= 0.0) beta = -beta;
    const double denom = c0 - beta;
    for (Index i = row0 + 1; i < m.rows; ++i) m(i, col) /= denom;
    tau = (beta - c0) / beta;
}

// Applies H = I - tau v v^T (v = (1, m(row0+1.., col))) from the left to columns
// [c_begin, c_end) of m, rows row0...
inline void apply_householder_cols(Mat& m, Index row0, Index col, double tau, Index c_begin,
                                   Index c_end) {
    if (tau == 0.0) return;
    for (Index j = c_begin; j < c_end; ++j) {
        double dot = m(row0, j);
        for (Index i = row0 + 1; i < m.rows; ++i) dot += m(i, col) * m(i, j);
        m(row0, j) -= tau * dot;
        for (Index i = row0 + 1; i < m.rows; ++i) m(i, j) -= tau * m(i, col) * dot;
    }
}

// Applies the same reflector to a vector b (length m.rows).
inline void apply_householder_vec(const Mat& m, Index row0, Index col, double tau, Vec& b) {
    if (tau == 0.0) return;
    double dot = b[static_cast<size_t>(row0)];
    for (Index i = row0 + 1; i < m.rows; ++i) dot += m(i, col) * b[static_cast<size_t>(i)];
    b[static_cast<size_t>(row0)] -= tau * dot;
    for (Index i = row0 + 1; i < m.rows; ++i) b[static_cast<size_t>(i)] -= tau * m(i, col) * dot;
}

// Householder QR without pivoting: the upper triangle holds R, the lower the reflectors.
struct HouseholderQR {
    Mat qr;
    Vec tau;
    explicit HouseholderQR(Mat m) : qr(std::move(m)) {
        const Index size = std::min(qr.rows, qr.cols);
        tau.assign(static_cast<size_t>(size), 0.0);
        for (Index k = 0; k < size; ++k) {
            double beta;
            make_householder(qr, k, k, tau[static_cast<size_t>(k)], beta);
            qr(k, k) = beta;
            apply_householder_cols(qr, k, k, tau[static_cast<size_t>(k)], k + 1, qr.cols);
        }
    }
    // b <- Q^T b.
    void apply_qt(Vec& b) const {
        for (Index k = 0; k < static_cast<Index>(tau.size()); ++k)
            apply_householder_vec(qr, k, k, tau[static_cast<size_t>(k)], b);
    }
};

// Householder QR with column pivoting, with a rank threshold relative to the largest pivot.
struct ColPivQR {
    Mat qr;
    Vec tau;
    std::vector<Index> perm;  // perm[k] = original column now at position k
    Index nonzero_pivots = 0;
    double max_pivot = 0.0;
    double threshold = -1.0;  // < 0: default, eps * min(rows, cols)

    explicit ColPivQR(Mat m, double thr = -1.0) : qr(std::move(m)), threshold(thr) {
        const Index rows = qr.rows, cols = qr.cols;
        const Index size = std::min(rows, cols);
        tau.assign(static_cast<size_t>(size), 0.0);
        perm.resize(static_cast<size_t>(cols));
        for (Index j = 0; j < cols; ++j) perm[static_cast<size_t>(j)] = j;
        Vec updated(static_cast<size_t>(cols)), direct(static_cast<size_t>(cols));
        double maxnorm = 0.0;
        for (Index j = 0; j < cols; ++j) {
            double s = 0.0;
            for (Index i = 0; i < rows; ++i) s += qr(i, j) * qr(i, j);
            updated[static_cast<size_t>(j)] = direct[static_cast<size_t>(j)] = std::sqrt(s);
            maxnorm = std::max(maxnorm, updated[static_cast<size_t>(j)]);
        }
        const double t = maxnorm * EPS;
        const double threshold_helper = t * t / static_cast<double>(rows);
        const double downdate_threshold = std::sqrt(EPS);
        nonzero_pivots = size;
        max_pivot = 0.0;
        for (Index k = 0; k < size; ++k) {
            Index best = k;
            double best_sq = updated[static_cast<size_t>(k)] * updated[static_cast<size_t>(k)];
            for (Index j = k + 1; j < cols; ++j) {
                const double v = updated[static_cast<size_t>(j)] * updated[static_cast<size_t>(j)];
                if (v > best_sq) {
                    best_sq = v;
                    best = j;
                }
            }
            if (nonzero_pivots == size && best_sq < threshold_helper * static_cast<double>(rows - k))
                nonzero_pivots = k;
            if (best != k) {
                for (Index i = 0; i < rows; ++i) std::swap(qr(i, k), qr(i, best));
                std::swap(updated[static_cast<size_t>(k)], updated[static_cast<size_t>(best)]);
                std::swap(direct[static_cast<size_t>(k)], direct[static_cast<size_t>(best)]);
                std::swap(perm[static_cast<size_t>(k)], perm[static_cast<size_t>(best)]);
            }
            double beta;
            make_householder(qr, k, k, tau[static_cast<size_t>(k)], beta);
            qr(k, k) = beta;
            max_pivot = std::max(max_pivot, std::fabs(beta));
            apply_householder_cols(qr, k, k, tau[static_cast<size_t>(k)], k + 1, cols);
            for (Index j = k + 1; j < cols; ++j) {
                double& u = updated[static_cast<size_t>(j)];
                if (u != 0.0) {
                    double tmp = std::fabs(qr(k, j)) / u;
                    tmp = (1.0 + tmp) * (1.0 - tmp);
                    if (tmp < 0.0) tmp = 0.0;
                    const double ratio = u / direct[static_cast<size_t>(j)];
                    const double tmp2 = tmp * ratio * ratio;
                    if (tmp2 <= downdate_threshold) {
                        double s = 0.0;
                        for (Index i = k + 1; i < rows; ++i) s += qr(i, j) * qr(i, j);
                        direct[static_cast<size_t>(j)] = std::sqrt(s);
                        u = direct[static_cast<size_t>(j)];
                    } else {
                        u *= std::sqrt(tmp);
                    }
                }
            }
        }
    }

    Index rank() const {
        const double thr = threshold < 0.0 ? EPS * static_cast<double>(std::min(qr.rows, qr.cols))
                                           : threshold;
        const double pre = std::fabs(max_pivot) * thr;
        Index r = 0;
        for (Index i = 0; i < nonzero_pivots; ++i)
            if (std::fabs(qr(i, i)) > pre) ++r;
        return r;
    }

    // b <- H_{len-1} ... H_0 b, the first len reflectors of Q^T.
    void apply_qt(Vec& b, Index len) const {
        for (Index k = 0; k < len; ++k) apply_householder_vec(qr, k, k, tau[static_cast<size_t>(k)], b);
    }
};

// Solves R x = b in place with R the upper triangle of the top-left n x n corner of m.
inline void upper_solve(const Mat& m, Index n, Vec& b) {
    for (Index i = n - 1; i >= 0; --i) {
        double s = b[static_cast<size_t>(i)];
        for (Index j = i + 1; j < n; ++j) s -= m(i, j) * b[static_cast<size_t>(j)];
        b[static_cast<size_t>(i)] = s / m(i, i);
    }
}

// Solves R^T x = b in place (forward substitution with the transposed upper triangle).
inline void upper_transpose_solve(const Mat& m, Index n, Vec& b) {
    for (Index i = 0; i < n; ++i) {
        double s = b[static_cast<size_t>(i)];
        for (Index j = 0; j < i; ++j) s -= m(j, i) * b[static_cast<size_t>(j)];
        b[static_cast<size_t>(i)] = s / m(i, i);
    }
}

// LU with partial pivoting of a square matrix, in place. zero_pivot is true when a pivot of
// the decomposition is exactly zero.
struct PartialPivLU {
    Mat lu;
    std::vector<Index> row_perm;  // row_perm[i] = original row at position i
    bool zero_pivot = false;
    explicit PartialPivLU(Mat m) : lu(std::move(m)) {
        const Index n = lu.rows;
        row_perm.resize(static_cast<size_t>(n));
        for (Index i = 0; i < n; ++i) row_perm[static_cast<size_t>(i)] = i;
        for (Index k = 0; k < n; ++k) {
            Index best = k;
            double big = std::fabs(lu(k, k));
            for (Index i = k + 1; i < n; ++i)
                if (std::fabs(lu(i, k)) > big) {
                    big = std::fabs(lu(i, k));
                    best = i;
                }
            if (big != 0.0) {
                if (best != k) {
                    for (Index j = 0; j < n; ++j) std::swap(lu(k, j), lu(best, j));
                    std::swap(row_perm[static_cast<size_t>(k)], row_perm[static_cast<size_t>(best)]);
                }
                for (Index i = k + 1; i < n; ++i) lu(i, k) /= lu(k, k);
            } else {
                zero_pivot = true;
            }
            for (Index i = k + 1; i < n; ++i) {
                const double l = lu(i, k);
                for (Index j = k + 1; j < n; ++j) lu(i, j) -= l * lu(k, j);
            }
        }
        for (Index k = 0; k < n; ++k)
            if (lu(k, k) == 0.0) zero_pivot = true;
    }
    Vec solve(const Vec& b) const {
        const Index n = lu.rows;
        Vec x(static_cast<size_t>(n));
        for (Index i = 0; i < n; ++i) x[static_cast<size_t>(i)] = b[static_cast<size_t>(row_perm[static_cast<size_t>(i)])];
        for (Index i = 0; i < n; ++i) {
            double s = x[static_cast<size_t>(i)];
            for (Index j = 0; j < i; ++j) s -= lu(i, j) * x[static_cast<size_t>(j)];
            x[static_cast<size_t>(i)] = s;
        }
        upper_solve(lu, n, x);
        return x;
    }
};

// The pseudo-inverse (cols, rows) of a matrix of full column rank, P R^-1 Q1^T from the
// column-pivoted QR.
inline Mat pseudo_inverse_full_rank(const Mat& m) {
    ColPivQR qr(m);
    const Index rows = m.rows, cols = m.cols;
    Mat pinv(cols, rows);
    for (Index r = 0; r < rows; ++r) {
        Vec e(static_cast<size_t>(rows), 0.0);
        e[static_cast<size_t>(r)] = 1.0;
        qr.apply_qt(e, std::min(rows, cols));
        upper_solve(qr.qr, cols, e);
        for (Index k = 0; k < cols; ++k) pinv(qr.perm[static_cast<size_t>(k)], r) = e[static_cast<size_t>(k)];
    }
    return pinv;
}

}  // namespace oracle
