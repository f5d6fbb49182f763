// The ridge NNLS of small kernels (at most 48 directions, the low-resolution mFOD fit) with two
// voxels per warp: each half-warp (16 lanes) runs one voxel's Lawson-Hanson steps on the Gram
// matrix, the same steps as ridge_nnls in multi_tissue.cu (cpp/src/sd/nnls.cpp:362-418), with
// the factor kept as its inverse (InvFactor in warp_chol.cuh: two rows per lane, up to 32
// active columns). A warp-wide step is mostly idle lanes when a voxel has ~10 active columns of
// 44; two voxels per warp do twice the work per instruction.
//
// The two halves run their own control flow (their masks name only their own lanes). A voxel
// whose fit needs the QR fallback (a pivot below the tolerance, more than 32 active columns, or
// a solver without normal equations) is not finished here: its half appends it to a list that
// the one-warp-per-voxel kernel then fits from the start, so it gets exactly that kernel's
// result.
#pragma once

#include "common.cuh"
#include "warp_chol.cuh"

namespace lar {

constexpr int kHalf = 16;

struct HalfWarp {
    int lane;       // 0..15 within the half
    int base;       // 0 or 16
    unsigned mask;  // the half's lanes
    __device__ __forceinline__ explicit HalfWarp(int warp_lane)
        : lane(warp_lane & 15), base(warp_lane & 16), mask(0xFFFFu << (warp_lane & 16)) {}
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    __device__ __forceinline__ double sum(double v) const {
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
        return v;
    }
    template <class T>
    __device__ __forceinline__ T from(T v, int src) const { return __shfl_sync(mask, v, base + src); }
    __device__ __forceinline__ bool any(bool p) const { return __any_sync(mask, p); }
    __device__ __forceinline__ unsigned ballot(bool p) const { return (__ballot_sync(mask, p) >> base) & 0xFFFFu; }
    // The largest v over the half and its index, the smallest index on a tie (idx < 0: none).
    __device__ __forceinline__ int argmax_first(double v, int idx) const {
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(mask, v, o);
            const int oi = __shfl_xor_sync(mask, idx, o);
            const bool take = oi >= 0 && (idx < 0 || ov > v || (ov == v && oi < idx));
            v = take ? ov : v;
            idx = take ? oi : idx;
        }
        return idx;
    }
    __device__ __forceinline__ int argmin_first(double v, int idx, double* best) const {
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(mask, v, o);
            const int oi = __shfl_xor_sync(mask, idx, o);
            const bool take = oi >= 0 && (idx < 0 || ov < v || (ov == v && oi < idx));
            v = take ? ov : v;
            idx = take ? oi : idx;
        }
        *best = v;
        return idx;
    }
};

// The InvFactor operations of warp_chol.cuh for a half-warp: rows r = lane + 16 t, t < 2.
__device__ __forceinline__ bool half_append(const InvFactor f, int& na, double h_cc, double rhs_c, int col,
                                            double min_relative, const HalfWarp& hw) {
    if (na >= f.cap) return false;
    const int nt = (na + 15) >> 4;
    double w[2] = {0.0, 0.0};
    for (int j = 0; j < na; ++j) {
        const double hj = f.h[j];
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int r = hw.lane + kHalf * t;
            if (t < nt && r >= j && r < na) w[t] = fma(f.M[packed_row(r) + j], hj, w[t]);
        }
    }
    double sq = 0.0, wy = 0.0;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const int r = hw.lane + kHalf * t;
        if (t < nt && r < na) {
            f.w[r] = w[t];
            sq = fma(w[t], w[t], sq);
            wy = fma(w[t], f.y[r], wy);
        }
    }
    sq = hw.sum(sq);
    wy = hw.sum(wy);
    const double pivot = h_cc - sq;
    if (!(pivot > min_relative * h_cc)) return false;
    const double d = sqrt(pivot), inv_d = 1.0 / d;
    hw.sync();
    double u[2] = {0.0, 0.0};
    for (int r = 0; r < na; ++r) {
        const double wr = f.w[r];
        const double* row = f.M + packed_row(r);
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int j = hw.lane + kHalf * t;
            if (t < nt && j <= r) u[t] = fma(wr, row[j], u[t]);
        }
    }
    double* mrow = f.M + packed_row(na);
    double* lrow = f.L + packed_row(na);
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const int j = hw.lane + kHalf * t;
        if (t < nt && j < na) {
            mrow[j] = -u[t] * inv_d;
            lrow[j] = f.w[j];
        }
    }
    if (hw.lane == 0) {
        mrow[na] = inv_d;
        lrow[na] = d;
        f.y[na] = (rhs_c - wy) * inv_d;
        f.cols[na] = col;
    }
    ++na;
    hw.sync();
    return true;
}

__device__ __forceinline__ void half_solve(const InvFactor f, int na, double* z, int zlen, const HalfWarp& hw) {
    const int nt = (na + 15) >> 4;
    double acc[2] = {0.0, 0.0};
    for (int r = 0; r < na; ++r) {
        const double yr = f.y[r];
        const double* row = f.M + packed_row(r);
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int j = hw.lane + kHalf * t;
            if (t < nt && j <= r) acc[t] = fma(row[j], yr, acc[t]);
        }
    }
    for (int j = hw.lane; j < zlen; j += kHalf) z[j] = 0.0;
    hw.sync();
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const int j = hw.lane + kHalf * t;
        if (t < nt && j < na) z[f.cols[j]] = acc[t];
    }
    hw.sync();
}

__device__ __forceinline__ void half_remove(const InvFactor f, int na, int pos, const HalfWarp& hw) {
    if (hw.lane == 0)
        for (int q = pos; q < na - 1; ++q) f.cols[q] = f.cols[q + 1];
    for (int k = pos; k < na - 1; ++k) {
        double* lk = f.L + packed_row(k + 1);
        const double diag = lk[k], above = lk[k + 1];
        const double rh = rhypot(diag, above);
        const double c = diag * rh, s = above * rh;
        hw.sync();
        for (int row = k + hw.lane; row < na - 1; row += kHalf) {
            double* lr = f.L + packed_row(row + 1);
            const double l = lr[k], r = lr[k + 1];
            lr[k] = c * l + s * r;
            lr[k + 1] = c * r - s * l;
        }
        double a[2], b[2];
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int j = hw.lane + kHalf * t;
            a[t] = b[t] = 0.0;
            if (j <= k + 1) {
                const double ma = j <= k ? f.M[packed_row(k) + j] : 0.0, mb = f.M[packed_row(k + 1) + j];
                a[t] = c * ma + s * mb;
                b[t] = c * mb - s * ma;
            }
        }
        if (hw.lane == 0) {
            const double ya = f.y[k], yb = f.y[k + 1];
            f.y[k] = c * ya + s * yb;
            f.y[k + 1] = c * yb - s * ya;
        }
        hw.sync();
        for (int j = hw.lane; j <= k; j += kHalf) f.L[packed_row(k) + j] = lk[j];
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int j = hw.lane + kHalf * t;
            if (j <= k + 1) {
                if (j != pos) f.M[packed_row(k) + (j < pos ? j : j - 1)] = a[t];
                f.M[packed_row(k + 1) + j] = b[t];
            }
        }
        hw.sync();
    }
}

}  // namespace lar
