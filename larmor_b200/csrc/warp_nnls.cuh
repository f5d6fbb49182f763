// Warp-level non-negative least squares: the Lawson-Hanson active-set method with least-squares
// fits by column-pivoted Householder QR on the active columns, one warp per problem.
//
// Follows cpp/src/sd/nnls.cpp: least_squares (:119-139; threshold max(rows, k) eps on the pivots,
// columns past the numerical rank get 0), largest_feasible_step (:160-173; the first on a tie),
// lawson_hanson (:187-221; an inner-step limit, the blocking column leaves and so does any whose
// coefficient rounding left below the gradient tolerance). The pivoting (largest remaining
// column norm, the first on a tie, LAPACK-style norm downdating) is that of the column-pivoted QR
// the reference uses, so rank decisions and ties carry over.
//
// Lanes split the rows of the matrix (dot products by warp reductions) and the columns for the
// gradient C^T (d - C x). All state lives in memory the caller provides (shared or global).
#pragma once

#include <cfloat>
#include <cstdint>

#include "common.cuh"

namespace lar {

constexpr double kEps64 = 2.220446049250313e-16;

// Index of the largest value among the lanes' candidates, the smallest index on a tie; lanes
// without a candidate pass index -1. Every lane gets the result.
__device__ __forceinline__ int warp_argmax_first(double v, int idx) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        const bool take = oi >= 0 && (idx < 0 || ov > v || (ov == v && oi < idx));
        v = take ? ov : v;
        idx = take ? oi : idx;
    }
    return idx;
}

// Index of the smallest value, the smallest index on a tie, with the value in *best.
__device__ __forceinline__ int warp_argmin_first(double v, int idx, double* best) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        const bool take = oi >= 0 && (idx < 0 || ov < v || (ov == v && oi < idx));
        v = take ? ov : v;
        idx = take ? oi : idx;
    }
    *best = v;
    return idx;
}

// Workspace of warp_qr_least_squares for up to `kcap` active columns of `rows` rows.
struct QrScratch {
    double* sub;   // (kcap, rows), column-major: the active columns, then the QR factors
    double* tau;   // (kcap,)
    double* nu;    // (kcap,) updated column norms
    double* nd;    // (kcap,) directly computed column norms
    int* perm;     // (kcap,) position -> index into the active list
    double* rv;    // (rows,) rotated data, then the solution
};

// Column loader of a row-major matrix: entry (r, col).
struct RowMajorColumns {
    const double* c;
    int ldc;
    __device__ __forceinline__ double operator()(int r, int col, int /*q*/) const { return c[size_t(r) * ldc + col]; }
};

// Least squares of d (rows) on the columns act[0..k) of a matrix whose entry (r, act[q]) the
// loader gives: writes the coefficients of those columns into z (indexed by column; other
// entries untouched).
template <class Columns>
__device__ __forceinline__ void warp_qr_least_squares_cols(const Columns cols, int rows, const int* act, int k,
                                                  const double* d, QrScratch s, double* z, int lane) {
    if (k == 0) return;
    for (int q = 0; q < k; ++q) {
        const int col = act[q];
        double sq = 0.0;
        for (int r = lane; r < rows; r += 32) {
            const double x = cols(r, col, q);
            s.sub[size_t(q) * rows + r] = x;
            sq += x * x;
        }
        sq = warp_sum(sq);
        if (lane == 0) {
            s.nu[q] = s.nd[q] = sqrt(sq);
            s.perm[q] = q;
        }
    }
    __syncwarp();
    double biggest = 0.0;
    for (int q = 0; q < k; ++q) biggest = fmax(biggest, s.nu[q]);
    const double th = biggest * kEps64;
    const double small_sq = th * th / double(rows);
    const int size = min(rows, k);
    int nonzero = size;
    double maxpivot = 0.0;
    for (int kk = 0; kk < size; ++kk) {
        int best = kk;
        double best_sq = s.nu[kk] * s.nu[kk];
        for (int q = kk + 1; q < k; ++q) {
            const double sq = s.nu[q] * s.nu[q];
            if (sq > best_sq) { best_sq = sq; best = q; }
        }
        if (nonzero == size && best_sq < small_sq * double(rows - kk)) nonzero = kk;
        if (best != kk) {
            for (int r = lane; r < rows; r += 32) {
                const double t = s.sub[size_t(kk) * rows + r];
                s.sub[size_t(kk) * rows + r] = s.sub[size_t(best) * rows + r];
                s.sub[size_t(best) * rows + r] = t;
            }
            __syncwarp();
            if (lane == 0) {
                double t = s.nu[kk]; s.nu[kk] = s.nu[best]; s.nu[best] = t;
                t = s.nd[kk]; s.nd[kk] = s.nd[best]; s.nd[best] = t;
                const int pt = s.perm[kk]; s.perm[kk] = s.perm[best]; s.perm[best] = pt;
            }
        }
        __syncwarp();
        double* col = s.sub + size_t(kk) * rows;
        const double c0 = col[kk];
        double tail = 0.0;
        for (int r = kk + 1 + lane; r < rows; r += 32) tail += col[r] * col[r];
        tail = warp_sum(tail);
        double tau, beta;
        if (tail <= DBL_MIN) {
            tau = 0.0;
            beta = c0;
            for (int r = kk + 1 + lane; r < rows; r += 32) col[r] = 0.0;
        } else {
            beta = sqrt(c0 * c0 + tail);
            if (c0 >= 0.0) beta = -beta;
            const double den = c0 - beta;
            for (int r = kk + 1 + lane; r < rows; r += 32) col[r] /= den;
            tau = (beta - c0) / beta;
        }
        __syncwarp();
        if (lane == 0) {
            col[kk] = beta;
            s.tau[kk] = tau;
        }
        maxpivot = fmax(maxpivot, fabs(beta));
        __syncwarp();
        for (int q = kk + 1; q < k; ++q) {
            double* other = s.sub + size_t(q) * rows;
            if (tau != 0.0) {
                double dot = 0.0;
                for (int r = kk + 1 + lane; r < rows; r += 32) dot += col[r] * other[r];
                dot = warp_sum(dot) + other[kk];
                __syncwarp();
                if (lane == 0) other[kk] -= tau * dot;
                for (int r = kk + 1 + lane; r < rows; r += 32) other[r] -= tau * col[r] * dot;
                __syncwarp();
            }
            const double u = s.nu[q];
            if (u != 0.0) {
                double t = fabs(other[kk]) / u;
                t = fmax(0.0, (1.0 + t) * (1.0 - t));
                const double ratio = u / s.nd[q];
                if (t * ratio * ratio <= sqrt(kEps64)) {
                    double sq = 0.0;
                    for (int r = kk + 1 + lane; r < rows; r += 32) sq += other[r] * other[r];
                    sq = warp_sum(sq);
                    __syncwarp();
                    if (lane == 0) s.nd[q] = s.nu[q] = sqrt(sq);
                } else {
                    __syncwarp();
                    if (lane == 0) s.nu[q] = u * sqrt(t);
                }
            }
            __syncwarp();
        }
    }
    const double thr = double(max(rows, k)) * kEps64;
    int rank = 0;
    for (int i = 0; i < nonzero; ++i)
        if (fabs(s.sub[size_t(i) * rows + i]) > maxpivot * thr) ++rank;
    for (int r = lane; r < rows; r += 32) s.rv[r] = d[r];
    __syncwarp();
    for (int kk = 0; kk < rank; ++kk) {
        const double tau = s.tau[kk];
        if (tau == 0.0) continue;
        const double* col = s.sub + size_t(kk) * rows;
        double dot = 0.0;
        for (int r = kk + 1 + lane; r < rows; r += 32) dot += col[r] * s.rv[r];
        dot = warp_sum(dot) + s.rv[kk];
        __syncwarp();
        if (lane == 0) s.rv[kk] -= tau * dot;
        for (int r = kk + 1 + lane; r < rows; r += 32) s.rv[r] -= tau * col[r] * dot;
        __syncwarp();
    }
    // R11 b = rotated[:rank] by column-oriented back substitution.
    for (int i = rank - 1; i >= 0; --i) {
        __syncwarp();
        const double bi = s.rv[i] / s.sub[size_t(i) * rows + i];
        __syncwarp();
        if (lane == 0) s.rv[i] = bi;
        for (int r = lane; r < i; r += 32) s.rv[r] -= s.sub[size_t(i) * rows + r] * bi;
    }
    __syncwarp();
    for (int i = lane; i < rank; i += 32) z[act[s.perm[i]]] = s.rv[i];
    for (int i = rank + lane; i < k; i += 32) z[act[s.perm[i]]] = 0.0;
    __syncwarp();
}

// Least squares of d on the columns act[0..k) of c (rows x ldc, row-major).
__device__ __forceinline__ void warp_qr_least_squares(const double* __restrict__ c, int rows, int ldc,
                                             const int* act, int k, const double* d, QrScratch s,
                                             double* z, int lane) {
    warp_qr_least_squares_cols(RowMajorColumns{c, ldc}, rows, act, k, d, s, z, lane);
}

// Workspace of warp_nnls_explicit for an m-column problem with at most `acap` active columns.
struct NnlsScratch {
    double* u;      // (m,) solution
    double* z;      // (m,) candidate
    uint8_t* flag;  // (m,) active flags
    int* act;       // (acap,) active columns, increasing
    int* n_act;     // one int
    double* res;    // (rows,) residual
    QrScratch qr;
    int acap;
};

// Solves min ||c u - d|| over u >= 0 for c (rows x m, row-major) by Lawson-Hanson with QR fits
// (cpp/src/sd/nnls.cpp:187-221, :332-346). Returns 1 when the method ended by its rule, 0 when
// the inner-step limit ran out (u is then the last fit), -1 when more than acap columns became
// active (u undefined). u is in s.u.
__device__ __forceinline__ int warp_nnls_explicit(const double* __restrict__ c, int rows, int m, const double* d,
                                         double tol, int max_inner, NnlsScratch s, int lane) {
    for (int j = lane; j < m; j += 32) {
        s.u[j] = 0.0;
        s.z[j] = 0.0;
        s.flag[j] = 0;
    }
    if (lane == 0) *s.n_act = 0;
    __syncwarp();
    int inner = 0;
    for (;;) {
        const int na = *s.n_act;
        for (int r = lane; r < rows; r += 32) {
            double acc = d[r];
            for (int q = 0; q < na; ++q) acc -= c[size_t(r) * m + s.act[q]] * s.u[s.act[q]];
            s.res[r] = acc;
        }
        __syncwarp();
        double bv = 0.0;
        int bi = -1;
        int e = -1;
        double ge = 0.0;
        if (m <= 8) {
            // Few columns of many rows: lanes split the rows, one reduction per column.
            for (int j = 0; j < m; ++j) {
                double g = 0.0;
                for (int r = lane; r < rows; r += 32) g += c[size_t(r) * m + j] * s.res[r];
                g = warp_sum(g);
                if (!s.flag[j] && (bi < 0 || g > bv)) { bv = g; bi = j; }
            }
            e = bi;
            ge = bv;
        } else {
            // Lanes over the columns, four at a time so that their dot products overlap; each
            // lane takes its columns in increasing order (the first on a tie).
            for (int j0 = lane; j0 < m; j0 += 4 * 32) {
                double g[4] = {0.0, 0.0, 0.0, 0.0};
                bool open[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) open[q] = j0 + 32 * q < m && !s.flag[j0 + 32 * q];
                for (int r = 0; r < rows; ++r) {
                    const double rr = s.res[r];
                    const double* cr = c + size_t(r) * m;
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (open[q]) g[q] += cr[j0 + 32 * q] * rr;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (open[q] && (bi < 0 || g[q] > bv)) { bv = g[q]; bi = j0 + 32 * q; }
            }
            e = warp_argmax_first(bv, bi);
            ge = e >= 0 ? __shfl_sync(0xffffffffu, bv, e & 31) : 0.0;
        }
        if (e < 0 || ge <= tol) return 1;
        if (na >= s.acap) return -1;
        __syncwarp();
        if (lane == 0) {
            int q = na;
            while (q > 0 && s.act[q - 1] > e) { s.act[q] = s.act[q - 1]; --q; }
            s.act[q] = e;
            *s.n_act = na + 1;
            s.flag[e] = 1;
        }
        __syncwarp();
        warp_qr_least_squares(c, rows, m, s.act, *s.n_act, d, s.qr, s.z, lane);
        for (;;) {
            const int n2 = *s.n_act;
            bool any = false;
            for (int q = lane; q < n2; q += 32) any |= s.z[s.act[q]] <= 0.0;
            if (!__any_sync(0xffffffffu, any)) break;
            if (++inner > max_inner) {
                // The last least-squares fit is the answer (zero off the active set).
                for (int j = lane; j < m; j += 32) s.u[j] = s.flag[j] ? s.z[j] : 0.0;
                __syncwarp();
                return 0;
            }
            double sv = 0.0;
            int si = -1;
            for (int q = lane; q < n2; q += 32) {
                const int col = s.act[q];
                if (s.z[col] > 0.0) continue;
                const double dist = s.u[col] - s.z[col];
                const double st = dist > 0.0 ? s.u[col] / dist : 0.0;
                if (si < 0 || st < sv || (st == sv && col < si)) { sv = st; si = col; }
            }
            double step;
            const int bcol = warp_argmin_first(sv, si, &step);
            // u += step (z - u) on every column: inactive ones may still hold values rounding
            // left below the tolerance, which move towards their zero candidate.
            for (int j = lane; j < m; j += 32) {
                const double zj = s.flag[j] ? s.z[j] : 0.0;
                s.u[j] += step * (zj - s.u[j]);
            }
            __syncwarp();
            if (lane == 0) {
                s.u[bcol] = 0.0;
                int w = 0;
                for (int q = 0; q < n2; ++q) {
                    const int col = s.act[q];
                    if (col == bcol || !(fabs(s.u[col]) >= tol)) {
                        s.flag[col] = 0;
                        continue;
                    }
                    s.act[w++] = col;
                }
                *s.n_act = w;
            }
            __syncwarp();
            warp_qr_least_squares(c, rows, m, s.act, *s.n_act, d, s.qr, s.z, lane);
        }
        for (int j = lane; j < m; j += 32) s.u[j] = s.flag[j] ? s.z[j] : 0.0;
        __syncwarp();
    }
}

}  // namespace lar
