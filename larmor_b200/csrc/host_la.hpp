// Host-side FP64 preparation of the per-table designs: column scaling, the pseudo-inverse of
// the log-signal design, the LSI reduction and the ridge Gram matrices. These run once per
// gradient table (or per table and responses) and are cached on the device afterwards; the
// per-voxel work is in the CUDA kernels.
//
// The decompositions are the ones Larmor's core uses through Eigen, with the same pivot and
// rank rules (Householder QR with column pivoting: the column of largest remaining norm, first
// on a tie, LAPACK-style norm downdating; rank = pivots above threshold * |largest pivot|), so
// the prepared matrices agree with the reference's to rounding.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace lar::host {

using i64 = std::int64_t;
constexpr double kEps = std::numeric_limits<double>::epsilon();

// Column-major dense matrix.
struct ColMat {
    i64 rows = 0, cols = 0;
    std::vector<double> v;
    ColMat() = default;
    ColMat(i64 r, i64 c) : rows(r), cols(c), v(static_cast<size_t>(r * c), 0.0) {}
    double& at(i64 i, i64 j) { return v[static_cast<size_t>(j * rows + i)]; }
    double at(i64 i, i64 j) const { return v[static_cast<size_t>(j * rows + i)]; }
    double* col(i64 j) { return v.data() + j * rows; }
    const double* col(i64 j) const { return v.data() + j * rows; }
    // From a row-major (r, c) array.
    static ColMat from_rows(const double* p, i64 r, i64 c) {
        ColMat m(r, c);
        for (i64 i = 0; i < r; ++i)
            for (i64 j = 0; j < c; ++j) m.at(i, j) = p[i * c + j];
        return m;
    }
    // To a row-major (rows, cols) vector.
    std::vector<double> to_rows() const {
        std::vector<double> out(static_cast<size_t>(rows * cols));
        for (i64 i = 0; i < rows; ++i)
            for (i64 j = 0; j < cols; ++j) out[static_cast<size_t>(i * cols + j)] = at(i, j);
        return out;
    }
};

// Householder QR with column pivoting, in place on a column-major copy.
class PivotedQR {
public:
    PivotedQR(ColMat a, double rank_threshold) : qr_(std::move(a)), threshold_(rank_threshold) {
        const i64 m = qr_.rows, n = qr_.cols, size = std::min(m, n);
        tau_.assign(static_cast<size_t>(size), 0.0);
        perm_.resize(static_cast<size_t>(n));
        std::vector<double> norm_upd(static_cast<size_t>(n)), norm_dir(static_cast<size_t>(n));
        double biggest = 0.0;
        for (i64 j = 0; j < n; ++j) {
            perm_[static_cast<size_t>(j)] = j;
            double s = 0.0;
            for (i64 i = 0; i < m; ++i) s += qr_.at(i, j) * qr_.at(i, j);
            norm_upd[static_cast<size_t>(j)] = norm_dir[static_cast<size_t>(j)] = std::sqrt(s);
            biggest = std::max(biggest, std::sqrt(s));
        }
        const double small_sq = (biggest * kEps) * (biggest * kEps) / static_cast<double>(m);
        nonzero_ = size;
        for (i64 k = 0; k < size; ++k) {
            i64 piv = k;
            double piv_sq = norm_upd[static_cast<size_t>(k)] * norm_upd[static_cast<size_t>(k)];
            for (i64 j = k + 1; j < n; ++j) {
                const double sq = norm_upd[static_cast<size_t>(j)] * norm_upd[static_cast<size_t>(j)];
                if (sq > piv_sq) { piv_sq = sq; piv = j; }
            }
            if (nonzero_ == size && piv_sq < small_sq * static_cast<double>(m - k)) nonzero_ = k;
            if (piv != k) {
                std::swap_ranges(qr_.col(k), qr_.col(k) + m, qr_.col(piv));
                std::swap(norm_upd[static_cast<size_t>(k)], norm_upd[static_cast<size_t>(piv)]);
                std::swap(norm_dir[static_cast<size_t>(k)], norm_dir[static_cast<size_t>(piv)]);
                std::swap(perm_[static_cast<size_t>(k)], perm_[static_cast<size_t>(piv)]);
            }
            reflect(k);
            for (i64 j = k + 1; j < n; ++j) {
                double& u = norm_upd[static_cast<size_t>(j)];
                if (u == 0.0) continue;
                double t = std::fabs(qr_.at(k, j)) / u;
                t = std::max(0.0, (1.0 + t) * (1.0 - t));
                const double r = u / norm_dir[static_cast<size_t>(j)];
                if (t * r * r <= std::sqrt(kEps)) {
                    double s = 0.0;
                    for (i64 i = k + 1; i < m; ++i) s += qr_.at(i, j) * qr_.at(i, j);
                    norm_dir[static_cast<size_t>(j)] = u = std::sqrt(s);
                } else {
                    u *= std::sqrt(t);
                }
            }
        }
    }

    i64 rank() const {
        const double cut = max_pivot_ * threshold_;
        i64 r = 0;
        for (i64 i = 0; i < nonzero_; ++i)
            if (std::fabs(qr_.at(i, i)) > cut) ++r;
        return r;
    }
    const ColMat& factors() const { return qr_; }
    const std::vector<i64>& perm() const { return perm_; }

    // b <- Q^T b with the first `len` reflectors.
    void apply_qt(double* b, i64 len) const {
        for (i64 k = 0; k < len; ++k) apply(k, b);
    }
    // b <- Q b with the first `len` reflectors (reverse order).
    void apply_q(double* b, i64 len) const {
        for (i64 k = len; k-- > 0;) apply(k, b);
    }
    // Solves R x = b on the leading n x n block, in place.
    void r_solve(double* b, i64 n) const {
        for (i64 i = n - 1; i >= 0; --i) {
            double s = b[i];
            for (i64 j = i + 1; j < n; ++j) s -= qr_.at(i, j) * b[j];
            b[i] = s / qr_.at(i, i);
        }
    }

private:
    // Householder reflector of column k below the diagonal, applied to the trailing columns.
    void reflect(i64 k) {
        const i64 m = qr_.rows, n = qr_.cols;
        double* c = qr_.col(k);
        double tail = 0.0;
        for (i64 i = k + 1; i < m; ++i) tail += c[i] * c[i];
        double tau, beta;
        if (tail <= std::numeric_limits<double>::min()) {
            tau = 0.0;
            beta = c[k];
            for (i64 i = k + 1; i < m; ++i) c[i] = 0.0;
        } else {
            beta = std::sqrt(c[k] * c[k] + tail);
            if (c[k] >= 0.0) beta = -beta;
            const double d = c[k] - beta;
            for (i64 i = k + 1; i < m; ++i) c[i] /= d;
            tau = (beta - c[k]) / beta;
        }
        c[k] = beta;
        tau_[static_cast<size_t>(k)] = tau;
        max_pivot_ = std::max(max_pivot_, std::fabs(beta));
        if (tau == 0.0) return;
        for (i64 j = k + 1; j < n; ++j) {
            double* t = qr_.col(j);
            double dot = t[k];
            for (i64 i = k + 1; i < m; ++i) dot += c[i] * t[i];
            t[k] -= tau * dot;
            for (i64 i = k + 1; i < m; ++i) t[i] -= tau * c[i] * dot;
        }
    }
    void apply(i64 k, double* b) const {
        const double tau = tau_[static_cast<size_t>(k)];
        if (tau == 0.0) return;
        const double* c = qr_.col(k);
        double dot = b[k];
        for (i64 i = k + 1; i < qr_.rows; ++i) dot += c[i] * b[i];
        b[k] -= tau * dot;
        for (i64 i = k + 1; i < qr_.rows; ++i) b[i] -= tau * c[i] * dot;
    }

    ColMat qr_;
    std::vector<double> tau_;
    std::vector<i64> perm_;
    i64 nonzero_ = 0;
    double max_pivot_ = 0.0;
    double threshold_;
};

// The prepared log-signal design: unit-norm columns, their scales, the pseudo-inverse, and the
// constraints with the same column scales. Follows cpp/src/dwi/log_fit.cpp:220-236.
struct LogDesignHost {
    i64 n = 0, p = 0, m = 0;
    std::vector<double> scales;   // (p,)
    std::vector<double> x;        // (n, p) row-major, scaled
    std::vector<double> pinv;     // (p, n) row-major
    std::vector<double> g;        // (m, p) row-major, scaled
};

inline LogDesignHost prepare_log_design(const double* x, i64 n, i64 p, const double* g, i64 m) {
    if (n < p || p < 1) {
        throw std::invalid_argument("x must be (n, p) with n >= p >= 1: got (" + std::to_string(n) +
                                    ", " + std::to_string(p) + ")");
    }
    LogDesignHost d;
    d.n = n; d.p = p; d.m = m;
    d.scales.resize(static_cast<size_t>(p));
    for (i64 j = 0; j < p; ++j) {
        double s = 0.0;
        for (i64 i = 0; i < n; ++i) s += x[i * p + j] * x[i * p + j];
        d.scales[static_cast<size_t>(j)] = s == 0.0 ? 1.0 : std::sqrt(s);
    }
    d.x.resize(static_cast<size_t>(n * p));
    for (i64 i = 0; i < n; ++i)
        for (i64 j = 0; j < p; ++j) d.x[static_cast<size_t>(i * p + j)] = x[i * p + j] * (1.0 / d.scales[static_cast<size_t>(j)]);
    d.g.resize(static_cast<size_t>(m * p));
    for (i64 i = 0; i < m; ++i)
        for (i64 j = 0; j < p; ++j) d.g[static_cast<size_t>(i * p + j)] = g[i * p + j] * (1.0 / d.scales[static_cast<size_t>(j)]);
    // Pseudo-inverse P R^-1 Q1^T of the scaled design (full column rank).
    PivotedQR qr(ColMat::from_rows(d.x.data(), n, p), kEps * static_cast<double>(std::min(n, p)));
    if (qr.rank() < p) {
        throw std::invalid_argument("the design does not have full column rank");
    }
    d.pinv.assign(static_cast<size_t>(p * n), 0.0);
    std::vector<double> e(static_cast<size_t>(n));
    for (i64 r = 0; r < n; ++r) {
        std::fill(e.begin(), e.end(), 0.0);
        e[static_cast<size_t>(r)] = 1.0;
        qr.apply_qt(e.data(), p);
        qr.r_solve(e.data(), p);
        for (i64 k = 0; k < p; ++k) d.pinv[static_cast<size_t>(qr.perm()[static_cast<size_t>(k)] * n + r)] = e[static_cast<size_t>(k)];
    }
    return d;
}

// The prepared LSI problem (cpp/src/sd/lsi.cpp:75-125): q_t (n, m) = rows of the thin Q that
// multiply the measurements, back = P R^-1 (n, n), e = G P R^-1 with unit rows (k, n), its Gram
// (k, k) and absolute row sums (k,). All row-major.
struct LsiDesignHost {
    i64 m = 0, n = 0, k = 0;
    std::vector<double> q_t, back, e, gram, abs_sums;
};

inline LsiDesignHost prepare_lsi_design(const double* a, i64 m, i64 n, const double* g, i64 k,
                                        double ridge) {
    if (!(ridge >= 0.0)) throw std::invalid_argument("the ridge must be at least 0");
    const bool has_ridge = ridge > 0.0;
    const i64 rows = m + (has_ridge ? n : 0);
    ColMat stacked(rows, n);
    for (i64 i = 0; i < m; ++i)
        for (i64 j = 0; j < n; ++j) stacked.at(i, j) = a[i * n + j];
    if (has_ridge)
        for (i64 j = 0; j < n; ++j) stacked.at(m + j, j) = ridge;
    PivotedQR qr(stacked, static_cast<double>(std::max(rows, n)) * kEps);
    if (rows < n || qr.rank() < n) {
        throw std::invalid_argument(
            "the design does not have full column rank: the measurements cannot determine all " +
            std::to_string(n) + " parameters");
    }
    LsiDesignHost d;
    d.m = m; d.n = n; d.k = k;
    d.q_t.assign(static_cast<size_t>(n * m), 0.0);
    std::vector<double> e(static_cast<size_t>(rows));
    for (i64 c = 0; c < n; ++c) {
        std::fill(e.begin(), e.end(), 0.0);
        e[static_cast<size_t>(c)] = 1.0;
        qr.apply_q(e.data(), n);
        for (i64 i = 0; i < m; ++i) d.q_t[static_cast<size_t>(c * m + i)] = e[static_cast<size_t>(i)];
    }
    d.back.assign(static_cast<size_t>(n * n), 0.0);
    std::vector<double> col(static_cast<size_t>(n));
    for (i64 c = 0; c < n; ++c) {
        std::fill(col.begin(), col.end(), 0.0);
        col[static_cast<size_t>(c)] = 1.0;
        qr.r_solve(col.data(), n);
        for (i64 r = 0; r < n; ++r) d.back[static_cast<size_t>(qr.perm()[static_cast<size_t>(r)] * n + c)] = col[static_cast<size_t>(r)];
    }
    d.e.assign(static_cast<size_t>(k * n), 0.0);
    for (i64 i = 0; i < k; ++i) {
        double nrm = 0.0;
        for (i64 c = 0; c < n; ++c) {
            double s = 0.0;
            for (i64 j = 0; j < n; ++j) s += g[i * n + j] * d.back[static_cast<size_t>(j * n + c)];
            d.e[static_cast<size_t>(i * n + c)] = s;
            nrm += s * s;
        }
        nrm = std::sqrt(nrm);
        if (nrm > 0.0)
            for (i64 c = 0; c < n; ++c) d.e[static_cast<size_t>(i * n + c)] /= nrm;
    }
    d.gram.assign(static_cast<size_t>(k * k), 0.0);
    d.abs_sums.assign(static_cast<size_t>(k), 0.0);
    for (i64 i = 0; i < k; ++i) {
        for (i64 j = 0; j < k; ++j) {
            double s = 0.0;
            for (i64 c = 0; c < n; ++c) s += d.e[static_cast<size_t>(i * n + c)] * d.e[static_cast<size_t>(j * n + c)];
            d.gram[static_cast<size_t>(i * k + j)] = s;
        }
        double s = 0.0;
        for (i64 c = 0; c < n; ++c) s += std::fabs(d.e[static_cast<size_t>(i * n + c)]);
        d.abs_sums[static_cast<size_t>(i)] = s;
    }
    return d;
}

// Gram matrix K^T K + ridge^2 I (c, c) of a kernel (m, c), and whether the ridge fits may use
// the normal equations (cpp/src/sd/nnls.cpp:348-360).
struct RidgeDesignHost {
    i64 m = 0, c = 0;
    double ridge = 0.0;
    bool normal_equations = false;
    std::vector<double> kernel;  // (m, c) row-major
    std::vector<double> gram;    // (c, c)
};

inline RidgeDesignHost prepare_ridge_design(const double* k, i64 m, i64 c, double ridge) {
    RidgeDesignHost d;
    d.m = m; d.c = c; d.ridge = ridge;
    d.kernel.assign(k, k + m * c);
    d.gram.assign(static_cast<size_t>(c * c), 0.0);
    double sq = 0.0;
    for (i64 i = 0; i < m; ++i)
        for (i64 j = 0; j < c; ++j) sq += k[i * c + j] * k[i * c + j];
    for (i64 a = 0; a < c; ++a)
        for (i64 b = 0; b < c; ++b) {
            double s = 0.0;
            for (i64 i = 0; i < m; ++i) s += k[i * c + a] * k[i * c + b];
            d.gram[static_cast<size_t>(a * c + b)] = s;
        }
    const double r2 = ridge * ridge;
    for (i64 a = 0; a < c; ++a) d.gram[static_cast<size_t>(a * c + a)] += r2;
    d.normal_equations = r2 == 0.0 || sq + r2 <= 1e8 * r2;
    return d;
}

}  // namespace lar::host
