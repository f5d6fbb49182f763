// A growing and shrinking Cholesky factor L of a Gram matrix on an active set of columns, held by
// one warp: the factor of the reference's ActiveCholesky / GrowingCholesky
// (cpp/src/sd/nnls.cpp:237-324, cpp/src/sd/lsi.cpp:145-200).
//
// Storage: packed rows, row r at offset r (r + 3) / 2 with r + 2 slots (the columns 0..r and one
// slot above the diagonal that a column removal uses transiently). The reciprocal of each
// diagonal entry is kept beside the factor, so the triangular solves multiply instead of
// dividing. The right-hand side of a solve lives in registers, VPL values per lane (entry
// r = lane + 32 t), and moves between lanes by shuffles: each substitution step costs one
// shuffle and no memory round trip or warp barrier.
#pragma once

#include "common.cuh"

namespace lar {

__host__ __device__ constexpr int packed_row(int r) { return r * (r + 3) / 2; }
__host__ __device__ constexpr int packed_size(int cap) { return packed_row(cap); }

struct WarpFactor {
    double* L;    // packed rows
    double* inv;  // (cap,) 1 / L(r, r)
    int* cols;    // (cap,) the factor's columns in joining order
    int cap;
    __device__ __forceinline__ double& at(int r, int c) const { return L[packed_row(r) + c]; }
};

template <int VPL>
__device__ __forceinline__ double reg_get(const double (&v)[VPL], int j) {
    const int t = j >> 5;
    double x = v[0];
#pragma unroll
    for (int i = 1; i < VPL; ++i) x = (t == i) ? v[i] : x;
    return __shfl_sync(0xffffffffu, x, j & 31);
}

template <int VPL>
__device__ __forceinline__ void reg_set(double (&v)[VPL], int j, double x, int lane) {
    if ((j & 31) == lane) {
        const int t = j >> 5;
#pragma unroll
        for (int i = 0; i < VPL; ++i)
            if (t == i) v[i] = x;
    }
}

// w <- L^-1 w on the first na rows (forward substitution, column by column).
template <int VPL>
__device__ __forceinline__ void reg_forward(const WarpFactor& f, int na, double (&w)[VPL], int lane) {
    for (int j = 0; j < na; ++j) {
        const double wj = reg_get<VPL>(w, j) * f.inv[j];
        reg_set<VPL>(w, j, wj, lane);
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int r = lane + 32 * t;
            if (r > j && r < na) w[t] = fma(-f.at(r, j), wj, w[t]);
        }
    }
}

// w <- L^-T w on the first na rows (back substitution).
template <int VPL>
__device__ __forceinline__ void reg_backward(const WarpFactor& f, int na, double (&w)[VPL], int lane) {
    for (int j = na - 1; j >= 0; --j) {
        const double xj = reg_get<VPL>(w, j) * f.inv[j];
        reg_set<VPL>(w, j, xj, lane);
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int r = lane + 32 * t;
            if (r < j) w[t] = fma(-f.at(j, r), xj, w[t]);
        }
    }
}

// Appends column `col` with cross entries h_r = H(cols[r], col) (r < na, in registers) and
// diagonal h_cc: L w = h, pivot = h_cc - w.w; returns false (leaving the factor as it was) when
// the pivot is not above min_relative * h_cc or the factor is full.
template <int VPL>
__device__ __noinline__ bool factor_append(const WarpFactor& f, int& na, double (&h)[VPL], double h_cc, int col,
                                           double min_relative, int lane) {
    if (na >= f.cap) return false;
    reg_forward<VPL>(f, na, h, lane);
    double sq = 0.0;
#pragma unroll
    for (int t = 0; t < VPL; ++t) {
        const int r = lane + 32 * t;
        if (r < na) sq += h[t] * h[t];
    }
    sq = warp_sum(sq);
    const double pivot = h_cc - sq;
    if (!(pivot > min_relative * h_cc)) return false;
#pragma unroll
    for (int t = 0; t < VPL; ++t) {
        const int r = lane + 32 * t;
        if (r < na) f.at(na, r) = h[t];
    }
    if (lane == 0) {
        const double d = sqrt(pivot);
        f.at(na, na) = d;
        f.inv[na] = 1.0 / d;
        f.cols[na] = col;
    }
    ++na;
    __syncwarp();
    return true;
}

// Removes the column at position `pos` of `na`: the rows below move up and Givens rotations of
// two columns clear the entry each leaves above the diagonal (cpp/src/sd/nnls.cpp:305-324).
static __device__ __noinline__ void factor_remove(const WarpFactor& f, int na, int pos, int lane) {
    for (int row = pos; row < na - 1; ++row) {
        for (int c = lane; c <= row + 1; c += 32) f.at(row, c) = f.at(row + 1, c);
        __syncwarp();
    }
    if (lane == 0)
        for (int q = pos; q < na - 1; ++q) f.cols[q] = f.cols[q + 1];
    for (int col = pos; col < na - 1; ++col) {
        const double diag = f.at(col, col), above = f.at(col, col + 1);
        const double len = hypot(diag, above);
        const double c = diag / len, s = above / len;
        __syncwarp();
        for (int row = col + lane; row < na - 1; row += 32) {
            const double l = f.at(row, col), r = f.at(row, col + 1);
            f.at(row, col) = c * l + s * r;
            f.at(row, col + 1) = c * r - s * l;
        }
        __syncwarp();
        if (lane == 0) f.inv[col] = 1.0 / f.at(col, col);
    }
    __syncwarp();
}

// z (zlen, zero off the factor's columns) <- H_AA^-1 rhs_A.
template <int VPL>
__device__ __noinline__ void factor_solve(const WarpFactor& f, int na, const double* rhs, double* z, int zlen,
                                          int lane) {
    double a[VPL];
#pragma unroll
    for (int t = 0; t < VPL; ++t) {
        const int r = lane + 32 * t;
        a[t] = r < na ? rhs[f.cols[r]] : 0.0;
    }
    for (int j = lane; j < zlen; j += 32) z[j] = 0.0;
    reg_forward<VPL>(f, na, a, lane);
    reg_backward<VPL>(f, na, a, lane);
    __syncwarp();
#pragma unroll
    for (int t = 0; t < VPL; ++t) {
        const int r = lane + 32 * t;
        if (r < na) z[f.cols[r]] = a[t];
    }
    __syncwarp();
}

}  // namespace lar

namespace lar {

// The inverse M = L^-1 of a growing Cholesky factor L of a Gram matrix on an active set, held by
// one warp next to L itself, with y = M rhs_A: the active-set solve z_A = G_AA^-1 rhs_A = M^T y
// becomes one triangular matrix-vector product (lanes over the columns of M, its rows read
// whole), and an appended column two such products and a reduction, instead of serial
// substitutions.
//
// Appending column e with cross entries h = G(A, e) and diagonal g_ee: w = M h, the pivot
// d^2 = g_ee - w.w, L's new row is [w^T d], M's is [-(w^T M) / d, 1 / d], and
// y_e = (rhs_e - w.y) / d, since L_new = [L 0; w^T d].
//
// Removing the column at position p (ActiveCholesky's downdate, cpp/src/sd/nnls.cpp:305-324):
// L's rows below p move up and Givens rotations G_k of its columns (k, k+1), k = p..na-2, clear
// the entries left above the diagonal: L~ Q = [L' 0] with Q = G_p ... G_{na-2}. Then
// L'^-1 is Q^T M without its last row and without column p (which Q^T M holds as zeros there):
// the same rotations, transposed, act on the rows (k, k+1) of M and on y.
//
// Storage: L and M as packed rows (row r at r (r + 3) / 2 with r + 2 slots: the columns 0..r
// and the one a rotation fills transiently); h, w and y in shared memory.
struct InvFactor {
    double* L;    // packed rows
    double* M;    // packed rows
    double* h;    // (cap,) the cross entries of the column being appended
    double* w;    // (cap,) M h
    double* y;    // (cap,) M rhs_A
    int* cols;    // (cap,) the factor's columns in joining order
    int cap;
};

// Appends column `col` (cross entries already in f.h[0..na)): false, leaving the factor as it
// was, when the pivot is not above min_relative * h_cc or the factor is full.
template <int VPL>
__device__ __forceinline__ bool inv_append(const InvFactor f, int& na, double h_cc, double rhs_c, int col,
                                           double min_relative, int lane) {
    if (na >= f.cap) return false;
    const int nt = (na + 31) >> 5;
    double w[VPL];
#pragma unroll
    for (int t = 0; t < VPL; ++t) w[t] = 0.0;
    // w_r = sum_{j <= r} M(r, j) h_j: each lane its own rows.
    for (int j = 0; j < na; ++j) {
        const double hj = f.h[j];
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int r = lane + 32 * t;
            if (t < nt && r >= j && r < na) w[t] = fma(f.M[packed_row(r) + j], hj, w[t]);
        }
    }
    double sq = 0.0, wy = 0.0;
#pragma unroll
    for (int t = 0; t < VPL; ++t) {
        const int r = lane + 32 * t;
        if (t < nt && r < na) {
            f.w[r] = w[t];
            sq = fma(w[t], w[t], sq);
            wy = fma(w[t], f.y[r], wy);
        }
    }
    sq = warp_sum(sq);
    wy = warp_sum(wy);
    const double pivot = h_cc - sq;
    if (!(pivot > min_relative * h_cc)) return false;
    const double d = sqrt(pivot), inv_d = 1.0 / d;
    __syncwarp();
    // Row na of M: -(w^T M)_j / d for j < na (rows of M read whole), 1 / d on the diagonal;
    // row na of L: w, d.
    double u[VPL];
#pragma unroll
    for (int t = 0; t < VPL; ++t) u[t] = 0.0;
    for (int r = 0; r < na; ++r) {
        const double wr = f.w[r];
        const double* row = f.M + packed_row(r);
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int j = lane + 32 * t;
            if (t < nt && j <= r) u[t] = fma(wr, row[j], u[t]);
        }
    }
    double* mrow = f.M + packed_row(na);
    double* lrow = f.L + packed_row(na);
#pragma unroll
    for (int t = 0; t < VPL; ++t) {
        const int j = lane + 32 * t;
        if (t < nt && j < na) {
            mrow[j] = -u[t] * inv_d;
            lrow[j] = f.w[j];
        }
    }
    if (lane == 0) {
        mrow[na] = inv_d;
        lrow[na] = d;
        f.y[na] = (rhs_c - wy) * inv_d;
        f.cols[na] = col;
    }
    ++na;
    __syncwarp();
    return true;
}

// Removes the factor column at position pos of na (see above), VPL * 32 >= na. One pass over the
// rotations: L~'s row r is read where L's row r + 1 lies until rotation r, its last, moves it up
// into row r; M's row k is final after rotation k and is written there without column pos.
// Each rotation: c = diag / hypot(diag, above), s = above / hypot, by one reciprocal hypot.
template <int VPL>
__device__ __forceinline__ void inv_remove(const InvFactor f, int na, int pos, int lane) {
    if (lane == 0)
        for (int q = pos; q < na - 1; ++q) f.cols[q] = f.cols[q + 1];
    for (int k = pos; k < na - 1; ++k) {
        double* lk = f.L + packed_row(k + 1);  // L~ row k
        const double diag = lk[k], above = lk[k + 1];
        const double rh = rhypot(diag, above);
        const double c = diag * rh, s = above * rh;
        __syncwarp();
        // L~ rows k..na-2 (stored one row down): columns (k, k + 1) by G_k.
        for (int row = k + lane; row < na - 1; row += 32) {
            double* lr = f.L + packed_row(row + 1);
            const double l = lr[k], r = lr[k + 1];
            lr[k] = c * l + s * r;
            lr[k + 1] = c * r - s * l;
        }
        // M rows (k, k + 1) by G_k^T (row k's column k + 1 is zero before), y likewise.
        double a[VPL], b[VPL];
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int j = lane + 32 * t;
            a[t] = b[t] = 0.0;
            if (j <= k + 1) {
                const double ma = j <= k ? f.M[packed_row(k) + j] : 0.0, mb = f.M[packed_row(k + 1) + j];
                a[t] = c * ma + s * mb;
                b[t] = c * mb - s * ma;
            }
        }
        if (lane == 0) {
            const double ya = f.y[k], yb = f.y[k + 1];
            f.y[k] = c * ya + s * yb;
            f.y[k + 1] = c * yb - s * ya;
        }
        __syncwarp();
        // Row k of L~ is final: move it up (columns 0..k; its column k + 1 is now zero).
        for (int j = lane; j <= k; j += 32) f.L[packed_row(k) + j] = lk[j];
        // Row k of M is final: without column pos. Row k + 1 stays whole for the next rotation.
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int j = lane + 32 * t;
            if (j <= k + 1) {
                if (j != pos) f.M[packed_row(k) + (j < pos ? j : j - 1)] = a[t];
                f.M[packed_row(k + 1) + j] = b[t];
            }
        }
        __syncwarp();
    }
}

// z (zlen, zero off the factor's columns) <- M^T y = G_AA^-1 rhs_A.
template <int VPL>
__device__ __forceinline__ void inv_solve(const InvFactor f, int na, double* z, int zlen, int lane) {
    const int nt = (na + 31) >> 5;
    double acc[VPL];
#pragma unroll
    for (int t = 0; t < VPL; ++t) acc[t] = 0.0;
    for (int r = 0; r < na; ++r) {
        const double yr = f.y[r];
        const double* row = f.M + packed_row(r);
#pragma unroll
        for (int t = 0; t < VPL; ++t) {
            const int j = lane + 32 * t;
            if (t < nt && j <= r) acc[t] = fma(row[j], yr, acc[t]);
        }
    }
    for (int j = lane; j < zlen; j += 32) z[j] = 0.0;
    __syncwarp();
#pragma unroll
    for (int t = 0; t < VPL; ++t) {
        const int j = lane + 32 * t;
        if (t < nt && j < na) z[f.cols[j]] = acc[t];
    }
    __syncwarp();
}

}  // namespace lar
