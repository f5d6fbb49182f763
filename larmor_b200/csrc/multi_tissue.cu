// Multi-tissue spherical deconvolution (SDModel's mFOD method) on the GPU, one warp per voxel.
//
// Follows cpp/src/sd/multi_tissue.cpp:76-148 per voxel (a voxel's rounds do not depend on the
// other voxels of its block, cpp/tests/sd/test_multi_tissue.cpp:56): up to max_rounds rounds of
//   the anisotropic signal max(s_w - W_iso f_iso, 0) (:68-72),
//   its low-resolution FOD by non-negative least squares (solve_ridge_nnls, cpp/src/sd/nnls.cpp
//   :362-418, with the normal equations and an active-set Cholesky factor, :237-301, falling
//   back to QR on the stacked matrix from the first pivot that fails),
//   the fractions: FOD values below their median set to zero, all anisotropic tissues as one
//   column scaled to a maximum of 1, next to the isotropic columns, fitted by NNLS with QR fits
//   (compute_fractions, cpp/src/sd/fractions.cpp:70-101),
// until no fraction changes by fraction_tol; then the high-resolution FOD (ridge NNLS) and the
// per-block fractions with the final tolerance, normalised to sum to 1 (+1e-16).
//
// Work distribution: a persistent grid of warps pulls voxels from a device counter (the rounds
// and active-set steps differ between voxels). Lanes split the kernel's columns for the
// correlations K^T s and the NNLS gradients, the measurements for the fraction columns, and the
// factor's rows for the triangular solves. Each warp owns a slot of global scratch: the
// signals, the FOD vectors, the Cholesky factor (up to kCholCap active columns) and the QR
// workspaces.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "host_la.hpp"
#include "warp_nnls.cuh"

namespace lar {

namespace {

constexpr int kMtWarps = 4;
constexpr int kCholCap = 256;   // active columns the Cholesky factor holds
constexpr int kQrCap = 64;      // active columns of the ridge QR fallback
constexpr int kMaxGroups = 16;  // fraction columns (anisotropic groups + isotropic tissues)
constexpr double kMinPivot = 1e-12;
constexpr double kMedianTie = 1e-9;
constexpr double kFractionSumOffset = 1e-16;

struct RidgeDev {
    int m, c;
    double ridge, tol;
    int normal_equations;
    const double* k;     // (m, c) row-major
    const double* gram;  // (c, c)
};

struct TissueDev {
    int m, ca, ci, nb;
    const double* kt;    // (ca, m): the unweighted anisotropic kernel, transposed
    const double* iso;   // (m, ci)
    const double* wiso;  // (m, ci)
    const int* blocks;   // (nb, 2)
};

struct Slot {
    double *s, *ws, *as, *corr, *x, *z, *th, *L, *cols, *fu, *fz, *fsub, *qsub, *qd, *qrv, *frv;
    uint8_t *flag, *inf, *fflag;
};

inline size_t slot_doubles(int m, int cmax, int ng) {
    return 3 * size_t(m) + 4 * size_t(cmax) + size_t(kCholCap) * kCholCap + size_t(m) * ng + 2 * size_t(ng) +
           size_t(ng) * m + size_t(m + kQrCap) * kQrCap + 2 * size_t(m + kQrCap) + size_t(m) +
           (2 * size_t(cmax) + ng + 7) / 8 + 64;
}

__device__ Slot carve(double* base, int m, int cmax, int ng) {
    Slot s;
    double* p = base;
    s.s = p; p += m;
    s.ws = p; p += m;
    s.as = p; p += m;
    s.corr = p; p += cmax;
    s.x = p; p += cmax;
    s.z = p; p += cmax;
    s.th = p; p += cmax;
    s.L = p; p += size_t(kCholCap) * kCholCap;
    s.cols = p; p += size_t(m) * ng;
    s.fu = p; p += ng;
    s.fz = p; p += ng;
    s.fsub = p; p += size_t(ng) * m;
    s.qsub = p; p += size_t(m + kQrCap) * kQrCap;
    s.qd = p; p += m + kQrCap;
    s.qrv = p; p += m + kQrCap;
    s.frv = p; p += m;
    s.flag = reinterpret_cast<uint8_t*>(p);
    s.inf = s.flag + cmax;
    s.fflag = s.inf + cmax;
    return s;
}

struct WarpState {
    int cols[kCholCap];    // factor columns, joining order
    int sorted[kCholCap];  // active columns with x != 0 candidates, increasing (the factor's set)
    int qact[kQrCap];      // QR fallback active columns, increasing
    double qtau[kQrCap], qnu[kQrCap], qnd[kQrCap];
    int qperm[kQrCap];
    double fres[kMaxGroups];
    int fact[kMaxGroups], fn_act;
    double ftau[kMaxGroups], fnu[kMaxGroups], fnd[kMaxGroups];
    int fperm[kMaxGroups];
    double fiso[kMaxGroups], prev[kMaxGroups], fr[kMaxGroups];
    double med[2];
    double a[kCholCap];
};

// ---- the active-set Cholesky factor of a Gram matrix (cpp/src/sd/nnls.cpp:237-301) ------

// Appends `col`: L w = G_{A,col}, pivot = G_col,col - w.w; false when the pivot is not clearly
// positive.
__device__ bool chol_append(const RidgeDev& R, double* L, int& na, WarpState& st, int col, int lane) {
    double* w = st.a;
    for (int r = lane; r < na; r += 32) w[r] = R.gram[size_t(st.cols[r]) * R.c + col];
    __syncwarp();
    for (int j = 0; j < na; ++j) {
        const double wj = w[j] / L[j * kCholCap + j];
        __syncwarp();
        if (lane == 0) w[j] = wj;
        for (int r = j + 1 + lane; r < na; r += 32) w[r] -= L[r * kCholCap + j] * wj;
        __syncwarp();
    }
    double sq = 0.0;
    for (int r = lane; r < na; r += 32) sq += w[r] * w[r];
    sq = warp_sum(sq);
    const double gcc = R.gram[size_t(col) * R.c + col];
    const double pivot = gcc - sq;
    if (!(pivot > kMinPivot * gcc) || na >= kCholCap) return false;
    for (int r = lane; r < na; r += 32) L[na * kCholCap + r] = w[r];
    __syncwarp();
    if (lane == 0) {
        L[na * kCholCap + na] = sqrt(pivot);
        st.cols[na] = col;
    }
    ++na;
    __syncwarp();
    return true;
}

__device__ void chol_remove(double* L, int na, int pos, int lane) {
    for (int j = lane; j < na; j += 32)
        for (int row = pos; row < na - 1; ++row) L[row * kCholCap + j] = L[(row + 1) * kCholCap + j];
    __syncwarp();
    for (int col = pos; col < na - 1; ++col) {
        const double diag = L[col * kCholCap + col], above = L[col * kCholCap + col + 1];
        const double len = hypot(diag, above);
        const double c = diag / len, s = above / len;
        for (int row = col + lane; row < na - 1; row += 32) {
            const double l = L[row * kCholCap + col], r = L[row * kCholCap + col + 1];
            L[row * kCholCap + col] = c * l + s * r;
            L[row * kCholCap + col + 1] = c * r - s * l;
        }
        __syncwarp();
    }
}

// z <- G_AA^-1 rhs_A, zero off the factor's columns.
__device__ void chol_solve(const double* L, int na, const WarpState& st, const double* rhs, double* z, int c,
                           double* a, int lane) {
    for (int j = lane; j < c; j += 32) z[j] = 0.0;
    for (int p = lane; p < na; p += 32) a[p] = rhs[st.cols[p]];
    __syncwarp();
    for (int j = 0; j < na; ++j) {
        const double aj = a[j] / L[j * kCholCap + j];
        __syncwarp();
        if (lane == 0) a[j] = aj;
        for (int r = j + 1 + lane; r < na; r += 32) a[r] -= L[r * kCholCap + j] * aj;
        __syncwarp();
    }
    for (int j = na - 1; j >= 0; --j) {
        const double aj = a[j] / L[j * kCholCap + j];
        __syncwarp();
        if (lane == 0) a[j] = aj;
        for (int r = lane; r < j; r += 32) a[r] -= L[j * kCholCap + r] * aj;
        __syncwarp();
    }
    for (int p = lane; p < na; p += 32) z[st.cols[p]] = a[p];
    __syncwarp();
}

// The stacked columns [K_A; ridge I] of the ridge QR fallback.
struct StackedColumns {
    const double* k;
    int m, c;
    double ridge;
    __device__ __forceinline__ double operator()(int r, int col, int q) const {
        return r < m ? k[size_t(r) * c + col] : (r - m == q ? ridge : 0.0);
    }
};

// Least squares on the active columns by QR (fit_by_qr, cpp/src/sd/nnls.cpp:385-401); false
// when more columns are active than the QR workspace holds.
__device__ bool ridge_qr_fit(const RidgeDev& R, const double* sig, const uint8_t* flag, Slot& sl, WarpState& st,
                             int lane) {
    int k = 0;
    if (lane == 0) {
        for (int j = 0; j < R.c; ++j)
            if (flag[j]) {
                if (k < kQrCap) st.qact[k] = j;
                ++k;
            }
    }
    k = __shfl_sync(0xffffffffu, k, 0);
    for (int j = lane; j < R.c; j += 32) sl.z[j] = 0.0;
    __syncwarp();
    if (k > kQrCap) return false;
    const bool has_ridge = R.ridge > 0.0;
    const int rows = R.m + (has_ridge ? k : 0);
    for (int r = lane; r < rows; r += 32) sl.qd[r] = r < R.m ? sig[r] : 0.0;
    __syncwarp();
    QrScratch qs{sl.qsub, st.qtau, st.qnu, st.qnd, st.qperm, sl.qrv};
    warp_qr_least_squares_cols(StackedColumns{R.k, R.m, R.c, R.ridge}, rows, st.qact, k, sl.qd, qs, sl.z, lane);
    return true;
}

// min ||K x - sig||^2 + ridge^2 ||x||^2 over x >= 0 (solve_ridge_nnls with l1 = 0,
// cpp/src/sd/nnls.cpp:362-418), the result in sl.x. Returns false only when the QR fallback's
// workspace overflowed (x is then the last fit).
__device__ bool ridge_nnls(const RidgeDev& R, const double* sig, Slot& sl, WarpState& st, int lane) {
    const int c = R.c, m = R.m;
    for (int j = lane; j < c; j += 32) {
        double acc = 0.0;
        for (int i = 0; i < m; ++i) acc += R.k[size_t(i) * c + j] * sig[i];
        sl.corr[j] = acc;
        sl.x[j] = 0.0;
        sl.z[j] = 0.0;
        sl.flag[j] = 0;
        sl.inf[j] = 0;
    }
    __syncwarp();
    const bool use_qr_only = !R.normal_equations;
    bool failed = false, overflow = false;
    int na = 0, n_sorted = 0, inner = 0;
    const int max_inner = 3 * c;
    // fit_on: the factor brought to the active set, or QR from the first failing pivot on.
    auto fit_on = [&]() {
        if (!use_qr_only && !failed) {
            for (int pos = na - 1; pos >= 0; --pos) {
                const int col = st.cols[pos];
                if (sl.flag[col]) continue;
                chol_remove(sl.L, na, pos, lane);
                if (lane == 0) {
                    for (int q = pos; q < na - 1; ++q) st.cols[q] = st.cols[q + 1];
                    sl.inf[col] = 0;
                }
                --na;
                __syncwarp();
            }
            for (int j = 0; j < c && !failed; ++j) {
                if (!sl.flag[j] || sl.inf[j]) continue;
                if (!chol_append(R, sl.L, na, st, j, lane)) {
                    failed = true;
                } else {
                    if (lane == 0) sl.inf[j] = 1;
                    __syncwarp();
                }
            }
        }
        if (use_qr_only || failed) {
            overflow |= !ridge_qr_fit(R, sig, sl.flag, sl, st, lane);
        } else {
            chol_solve(sl.L, na, st, sl.corr, sl.z, c, st.a, lane);
        }
    };
    for (;;) {
        // Gradient corr - G x over the non-zero x, columns in increasing order; the steepest
        // inactive entry, the first on a tie.
        if (lane == 0) {
            n_sorted = 0;
            for (int j = 0; j < c; ++j)
                if (sl.x[j] != 0.0) st.sorted[n_sorted++] = j;
        }
        n_sorted = __shfl_sync(0xffffffffu, n_sorted, 0);
        __syncwarp();
        double bv = 0.0;
        int bi = -1;
        for (int j = lane; j < c; j += 32) {
            if (sl.flag[j]) continue;
            double g = sl.corr[j];
            for (int q = 0; q < n_sorted; ++q) {
                const int col = st.sorted[q];
                g -= sl.x[col] * R.gram[size_t(col) * c + j];
            }
            if (bi < 0 || g > bv) { bv = g; bi = j; }
        }
        const int e = warp_argmax_first(bv, bi);
        const double ge = e >= 0 ? __shfl_sync(0xffffffffu, bv, e & 31) : 0.0;
        if (e < 0 || ge <= R.tol) break;
        if (lane == 0) sl.flag[e] = 1;
        __syncwarp();
        fit_on();
        for (;;) {
            bool any = false;
            for (int j = lane; j < c; j += 32) any |= sl.flag[j] && sl.z[j] <= 0.0;
            if (!__any_sync(0xffffffffu, any)) break;
            if (++inner > max_inner) {
                // The last least-squares fit is the answer (cpp/src/sd/nnls.cpp:204-207).
                for (int j = lane; j < c; j += 32) sl.x[j] = sl.z[j];
                __syncwarp();
                return !overflow;
            }
            double sv = 0.0;
            int si = -1;
            for (int j = lane; j < c; j += 32) {
                if (!sl.flag[j] || sl.z[j] > 0.0) continue;
                const double dist = sl.x[j] - sl.z[j];
                const double stp = dist > 0.0 ? sl.x[j] / dist : 0.0;
                if (si < 0 || stp < sv) { sv = stp; si = j; }
            }
            double step;
            const int b = warp_argmin_first(sv, si, &step);
            for (int j = lane; j < c; j += 32) sl.x[j] += step * (sl.z[j] - sl.x[j]);
            __syncwarp();
            if (lane == 0) {
                sl.x[b] = 0.0;
                sl.flag[b] = 0;
            }
            __syncwarp();
            for (int j = lane; j < c; j += 32)
                if (sl.flag[j] && !(fabs(sl.x[j]) >= R.tol)) sl.flag[j] = 0;
            __syncwarp();
            fit_on();
        }
        for (int j = lane; j < c; j += 32) sl.x[j] = sl.z[j];
        __syncwarp();
    }
    return !overflow;
}

// Median of v[0..n), the mean of the two middle values for even n (cpp/src/sd/fractions.cpp:56-68),
// by ranks: the element of stable rank r is the r-th smallest.
__device__ double warp_median(const double* v, int n, WarpState& st, int lane) {
    const int hi = n / 2, lo = n % 2 ? n / 2 : n / 2 - 1;
    for (int i = lane; i < n; i += 32) {
        const double vi = v[i];
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const double vj = v[j];
            rank += (vj < vi) || (vj == vi && j < i);
        }
        if (rank == hi) st.med[0] = vi;
        if (rank == lo) st.med[1] = vi;
    }
    __syncwarp();
    return n % 2 ? st.med[0] : (st.med[1] + st.med[0]) / 2.0;
}

// compute_fractions (cpp/src/sd/fractions.cpp:70-101): tol < 0 uses the default tolerance of the
// fraction columns. Writes the fractions (groups, then isotropic tissues) to st.fr.
__device__ void fractions(const TissueDev& T, const double* fod, const double* sig, bool per_block, double tol,
                          Slot& sl, WarpState& st, int lane) {
    const int m = T.m, ca = T.ca, ci = T.ci;
    const double threshold = warp_median(fod, ca, st, lane) * (1.0 - kMedianTie);
    for (int j = lane; j < ca; j += 32) sl.th[j] = fod[j] < threshold ? 0.0 : fod[j];
    __syncwarp();
    const int ng = per_block ? T.nb : 1;
    const int ncol = ng + ci;
    double colmax = 0.0;
    for (int g = 0; g < ng; ++g) {
        const int b = per_block ? T.blocks[2 * g] : 0, e = per_block ? T.blocks[2 * g + 1] : ca;
        double largest = -INFINITY;
        bool any = false;
        for (int i = lane; i < m; i += 32) {
            double acc = 0.0;
            for (int j = b; j < e; ++j) {
                const double t = sl.th[j];
                if (t != 0.0) acc += T.kt[size_t(j) * m + i] * t;
            }
            sl.cols[size_t(i) * ncol + g] = acc;
            if (!isnan(acc)) {
                largest = any ? fmax(largest, acc) : acc;
                any = true;
            }
        }
        // The largest non-NaN value over the lanes (Eigen's maxCoeff<PropagateNumbers>).
        const bool lane_any = any;
        largest = lane_any ? largest : -INFINITY;
        largest = warp_max(largest);
        const bool all_nan = !__any_sync(0xffffffffu, lane_any);
        __syncwarp();
        if (!all_nan && largest > 0.0)
            for (int i = lane; i < m; i += 32) sl.cols[size_t(i) * ncol + g] /= largest;
        __syncwarp();
    }
    for (int i = lane; i < m; i += 32)
        for (int j = 0; j < ci; ++j) sl.cols[size_t(i) * ncol + ng + j] = T.iso[size_t(i) * ci + j];
    __syncwarp();
    if (tol < 0.0) {
        // 10 eps norm1(C) max(rows, columns) (cpp/src/sd/nnls.cpp:177-181).
        for (int g = 0; g < ncol; ++g) {
            double sum = 0.0;
            for (int i = lane; i < m; i += 32) sum += fabs(sl.cols[size_t(i) * ncol + g]);
            colmax = fmax(colmax, warp_sum(sum));
        }
        tol = 10.0 * kEps64 * colmax * double(max(m, ncol));
    }
    NnlsScratch ns{sl.fu, sl.fz, sl.fflag, st.fact, &st.fn_act, sl.frv,
                   QrScratch{sl.fsub, st.ftau, st.fnu, st.fnd, st.fperm, sl.frv}, kMaxGroups};
    // The residual and the QR's rotated data must not share memory.
    ns.res = sl.qrv;
    warp_nnls_explicit(sl.cols, m, ncol, sig, tol, 3 * ncol, ns, lane);
    for (int g = lane; g < ncol; g += 32) st.fr[g] = sl.fu[g];
    __syncwarp();
}

__global__ void __launch_bounds__(kMtWarps * 32) multi_tissue_kernel(
    const double* __restrict__ signals, int64_t v, const double* __restrict__ weights, TissueDev lr,
    RidgeDev lr_solver, TissueDev hr, RidgeDev hr_solver, int max_rounds, double fraction_tol, double final_tol,
    int* queue, double* __restrict__ workspace, size_t slot_size, int cmax, int ng_max,
    double* __restrict__ fods, double* __restrict__ fractions_out, int32_t* __restrict__ rounds_out,
    uint8_t* __restrict__ status) {
    __shared__ WarpState states[kMtWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpState& st = states[warp];
    Slot sl = carve(workspace + (size_t(blockIdx.x) * kMtWarps + warp) * slot_size, lr.m, cmax, ng_max);
    const int m = lr.m, ci = lr.ci;
    for (;;) {
        int64_t voxel = 0;
        if (lane == 0) voxel = atomicAdd(queue, 1);
        voxel = __shfl_sync(0xffffffffu, voxel, 0);
        if (voxel >= v) break;
        for (int i = lane; i < m; i += 32) {
            const double s = signals[voxel * m + i];
            sl.s[i] = s;
            sl.ws[i] = s * weights[i];
        }
        if (lane < kMaxGroups) {
            st.fiso[lane] = 0.0;
            st.prev[lane] = INFINITY;
        }
        __syncwarp();
        bool ok = true;
        int rounds = 0;
        for (int round = 0; round < max_rounds; ++round) {
            ++rounds;
            for (int i = lane; i < m; i += 32) {
                double r = 0.0;
                for (int j = 0; j < ci; ++j) r += lr.wiso[size_t(i) * ci + j] * st.fiso[j];
                sl.as[i] = fmax(sl.ws[i] - r, 0.0);
            }
            __syncwarp();
            ok &= ridge_nnls(lr_solver, sl.as, sl, st, lane);
            fractions(lr, sl.x, sl.s, false, -1.0, sl, st, lane);
            bool converged = true;
            for (int j = 0; j <= ci; ++j) converged &= fabs(st.fr[j] - st.prev[j]) < fraction_tol;
            __syncwarp();
            if (lane < ci) st.fiso[lane] = st.fr[1 + lane];
            __syncwarp();
            if (converged) break;
            if (lane <= ci) st.prev[lane] = st.fr[lane];
            __syncwarp();
        }
        for (int i = lane; i < m; i += 32) {
            double r = 0.0;
            for (int j = 0; j < ci; ++j) r += hr.wiso[size_t(i) * ci + j] * st.fiso[j];
            sl.as[i] = fmax(sl.ws[i] - r, 0.0);
        }
        __syncwarp();
        ok &= ridge_nnls(hr_solver, sl.as, sl, st, lane);
        for (int j = lane; j < hr.ca; j += 32) fods[voxel * hr.ca + j] = sl.x[j];
        __syncwarp();
        fractions(hr, sl.x, sl.s, true, final_tol, sl, st, lane);
        const int nf = hr.nb + ci;
        double total = kFractionSumOffset;
        for (int g = 0; g < nf; ++g) total += st.fr[g];
        for (int g = lane; g < nf; g += 32) fractions_out[voxel * nf + g] = st.fr[g] / total;
        if (lane == 0) {
            if (rounds_out) rounds_out[voxel] = rounds;
            if (status) status[voxel] = ok ? 0 : 1;
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kMtWarps * 32) single_tissue_kernel(
    const double* __restrict__ signals, int64_t v, RidgeDev solver, int* queue, double* __restrict__ workspace,
    size_t slot_size, int cmax, double* __restrict__ fods, uint8_t* __restrict__ status) {
    __shared__ WarpState states[kMtWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpState& st = states[warp];
    Slot sl = carve(workspace + (size_t(blockIdx.x) * kMtWarps + warp) * slot_size, solver.m, cmax, 1);
    for (;;) {
        int64_t voxel = 0;
        if (lane == 0) voxel = atomicAdd(queue, 1);
        voxel = __shfl_sync(0xffffffffu, voxel, 0);
        if (voxel >= v) break;
        for (int i = lane; i < solver.m; i += 32) sl.s[i] = signals[voxel * solver.m + i];
        __syncwarp();
        const bool ok = ridge_nnls(solver, sl.s, sl, st, lane);
        for (int j = lane; j < solver.c; j += 32) fods[voxel * solver.c + j] = sl.x[j];
        if (lane == 0 && status) status[voxel] = ok ? 0 : 1;
        __syncwarp();
    }
}

}  // namespace

}  // namespace lar

// FodSolver.l2nnls (cpp/src/python/sd.cpp:89-102, cpp/src/sd/solver.cpp:464-467).
struct lar_fod_solver_s {
    lar::host::RidgeDesignHost host;
    double tol = 0.0;
    lar::DeviceArray<double> k, gram;
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    ~lar_fod_solver_s() {
        if (scratch) cudaFree(scratch);
    }
    lar::RidgeDev view() const {
        return lar::RidgeDev{int(host.m), int(host.c), host.ridge, tol, host.normal_equations ? 1 : 0, k.ptr, gram.ptr};
    }
    void* reserve(size_t need) {
        if (need > scratch_bytes) {
            if (scratch) lar::cuda_check(cudaFree(scratch), "cudaFree");
            scratch = nullptr;
            scratch_bytes = 0;
            lar::cuda_check(cudaMalloc(&scratch, need), "cudaMalloc (SD scratch)");
            scratch_bytes = need;
        }
        return scratch;
    }
};

// DeconvKernel (cpp/src/python/sd.cpp:260-292): one resolution of a multi-tissue kernel.
struct lar_deconv_kernel_s {
    int64_t m = 0, ca = 0, ci = 0, nb = 0;
    lar::DeviceArray<double> kt, iso, wiso;
    lar::DeviceArray<int> blocks;
    lar::TissueDev view() const {
        return lar::TissueDev{int(m), int(ca), int(ci), int(nb), kt.ptr, iso.ptr, wiso.ptr, blocks.ptr};
    }
};

using namespace lar;

extern "C" {

int lar_l2nnls_create(const double* k, int64_t m, int64_t c, double reg, double tol_x, lar_fod_solver* out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        require(reg >= 0.0, "reg must be at least 0");
        require(tol_x > 0.0, "tol_x must be positive");
        require(k != nullptr && m > 0 && c > 0, "k must be a non-empty (m, c) array");
        require(c <= (int64_t(1) << 16) && m <= 4096, "the kernel is too large");
        auto h = std::make_unique<lar_fod_solver_s>();
        h->host = host::prepare_ridge_design(k, m, c, reg);
        h->tol = tol_x;
        h->k.upload(h->host.kernel.data(), h->host.kernel.size());
        h->gram.upload(h->host.gram.data(), h->host.gram.size());
        *out = h.release();
    });
}

void lar_fod_solver_destroy(lar_fod_solver solver) { delete solver; }

int lar_deconv_kernel_create(const double* k_aniso, int64_t m, int64_t ca, const double* k_iso,
                             const double* w_k_iso, int64_t ci, const int64_t* blocks, int64_t nb,
                             lar_deconv_kernel* out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        require(k_aniso != nullptr && m > 0 && ca > 0, "k_aniso must be a non-empty (m, ca) array");
        require(ci >= 0 && (ci == 0 || (k_iso && w_k_iso)), "k_iso and w_k_iso must be (m, ci) arrays");
        require(nb >= 1 && blocks != nullptr, "aniso_blocks must hold at least one block");
        require(nb + ci <= kMaxGroups, "at most 16 tissues");
        std::string text;
        for (int64_t b = 0; b < nb; ++b) {
            const int64_t s = blocks[2 * b], e = blocks[2 * b + 1];
            require(s >= 0 && s < e && e <= ca, "aniso_blocks must be non-empty ranges within 0.." +
                                                    std::to_string(ca));
        }
        auto h = std::make_unique<lar_deconv_kernel_s>();
        h->m = m; h->ca = ca; h->ci = ci; h->nb = nb;
        std::vector<double> kt(size_t(ca * m));
        for (int64_t i = 0; i < m; ++i)
            for (int64_t j = 0; j < ca; ++j) kt[size_t(j * m + i)] = k_aniso[i * ca + j];
        h->kt.upload(kt.data(), kt.size());
        std::vector<double> iso(size_t(std::max<int64_t>(1, m * ci)), 0.0), wiso(iso.size(), 0.0);
        if (ci > 0) {
            std::copy(k_iso, k_iso + m * ci, iso.begin());
            std::copy(w_k_iso, w_k_iso + m * ci, wiso.begin());
        }
        h->iso.upload(iso.data(), iso.size());
        h->wiso.upload(wiso.data(), wiso.size());
        std::vector<int> bl(size_t(2 * nb));
        for (int64_t b = 0; b < 2 * nb; ++b) bl[size_t(b)] = int(blocks[b]);
        h->blocks.upload(bl.data(), bl.size());
        *out = h.release();
    });
}

void lar_deconv_kernel_destroy(lar_deconv_kernel kernel) { delete kernel; }

int lar_fit_multi_tissue(const double* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                         lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver,
                         int64_t max_outer, double fraction_tol, double final_tol_x, double* fods,
                         double* fractions, int32_t* rounds, uint8_t* status, void* stream) {
    return guarded([&] {
        require(lr && hr && lr_solver && hr_solver, "kernels and solvers must not be NULL");
        require(weights != nullptr, "weights must not be NULL");
        const int64_t m = hr->m;
        require(lr->m == m && lr_solver->host.m == m && hr_solver->host.m == m,
                "signals, weights and the kernels' measurements do not match");
        require(lr->ci == hr->ci, "the two kernels have different numbers of isotropic tissues");
        require(lr_solver->host.c == lr->ca, "the low-resolution solver does not match its kernel");
        require(hr_solver->host.c == hr->ca, "the high-resolution solver does not match its kernel");
        require(max_outer >= 0, "max_outer must be at least 0");
        require(v >= 0, "v must be at least 0");
        if (v == 0) return;
        require(signals && fods && fractions, "signals, fods and fractions must not be NULL");
        const int cmax = int(std::max(lr->ca, hr->ca));
        const int ng = int(hr->nb + hr->ci);
        const size_t slot = slot_doubles(int(m), cmax, std::max(ng, 2));
        const int slots = int(std::max<int64_t>(kMtWarps, std::min<int64_t>((v + kMtWarps - 1) / kMtWarps * kMtWarps,
                                                                            int64_t(sm_count()) * 8)));
        const size_t head = 256 + ((size_t(m) * sizeof(double) + 255) / 256) * 256;
        char* base = static_cast<char*>(hr_solver->reserve(head + size_t(slots) * slot * sizeof(double)));
        auto st = static_cast<cudaStream_t>(stream);
        cuda_check(cudaMemsetAsync(base, 0, sizeof(int), st), "cudaMemsetAsync");
        double* dweights = reinterpret_cast<double*>(base + 256);
        cuda_check(cudaMemcpyAsync(dweights, weights, size_t(m) * sizeof(double), cudaMemcpyHostToDevice, st),
                   "cudaMemcpyAsync (weights)");
        multi_tissue_kernel<<<slots / kMtWarps, kMtWarps * 32, 0, st>>>(
            signals, v, dweights, lr->view(), lr_solver->view(), hr->view(), hr_solver->view(),
            int(std::min<int64_t>(max_outer, 1 << 20)), fraction_tol, final_tol_x, reinterpret_cast<int*>(base),
            reinterpret_cast<double*>(base + head), slot, cmax, std::max(ng, 2), fods, fractions, rounds, status);
        cuda_check(cudaGetLastError(), "multi_tissue_kernel launch");
        // The weights' host buffer is the caller's; the copy must finish before it returns.
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    });
}

int lar_fit_single_tissue(const double* signals, int64_t v, lar_fod_solver solver, double* fods, uint8_t* status,
                          void* stream) {
    return guarded([&] {
        require(solver != nullptr, "solver must not be NULL");
        require(v >= 0, "v must be at least 0");
        if (v == 0) return;
        require(signals && fods, "signals and fods must not be NULL");
        const int m = int(solver->host.m), c = int(solver->host.c);
        const size_t slot = slot_doubles(m, c, 2);
        const int slots = int(std::max<int64_t>(kMtWarps, std::min<int64_t>((v + kMtWarps - 1) / kMtWarps * kMtWarps,
                                                                            int64_t(sm_count()) * 8)));
        char* base = static_cast<char*>(solver->reserve(256 + size_t(slots) * slot * sizeof(double)));
        auto st = static_cast<cudaStream_t>(stream);
        cuda_check(cudaMemsetAsync(base, 0, sizeof(int), st), "cudaMemsetAsync");
        single_tissue_kernel<<<slots / kMtWarps, kMtWarps * 32, 0, st>>>(
            signals, v, solver->view(), reinterpret_cast<int*>(base), reinterpret_cast<double*>(base + 256), slot, c,
            fods, status);
        cuda_check(cudaGetLastError(), "single_tissue_kernel launch");
    });
}

}  // extern "C"
