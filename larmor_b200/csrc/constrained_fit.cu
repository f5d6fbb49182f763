// The constrained re-fit of log-signal fits that break a constraint (DKI's D(n) >= 0,
// K(n) >= 0, K(n) <= 3 / (b_max D(n)) on 256 directions), one warp per violating voxel.
//
// Follows constrained_fit (cpp/src/dwi/log_fit.cpp:170-216): the weighted design
// W^(1/2) X = Q R (Householder, unpivoted), the least-distance problem min ||z|| subject to
// A z >= c with A = G R^-1 and c = -G p_free, solved as the NNLS problem
// min ||[A^T; c^T] u - e|| over u >= 0 by the Lawson-Hanson active-set method with the
// least-squares fits by column-pivoted Householder QR on the active columns
// (cpp/src/sd/nnls.cpp:119-139, :187-221), at most 50 inner steps per constraint, then the
// feasibility margin, the back substitution and the check that the result meets the
// constraints up to rounding. Where any step fails the voxel keeps its unconstrained fit, as
// in the reference.
//
// Work distribution: the violators were compacted into a list by the unconstrained fit; a
// fixed number of warps take them from a device work counter (no host round trip, so the pair
// of launches can be captured in a CUDA graph). Each warp owns a slot of global scratch
// memory: the QR of the weighted design (n x p), the NNLS matrix ((p+1) x m), the active
// columns' QR ((p+1) x 64), and the NNLS vectors. Lanes split the rows of the design for the
// reflections, the m constraint columns for gradients and steps, and the active columns for
// the small QR.

#include <cfloat>
#include <cstdint>

#include "common.cuh"
#include "log_fit.cuh"
#include "log_fit_warp.cuh"

namespace lar {

namespace {

constexpr int kCWarps = 4;
constexpr double kEps = 2.220446049250313e-16;
constexpr double kFeasibilityMargin = 1e-12;
constexpr int kInnerStepsPerConstraint = 50;
constexpr double kConstraintTolerance = 1e-9;

__device__ __forceinline__ double wsum(double v) { return warp_sum(v); }
__device__ __forceinline__ double wmax(double v) { return warp_max(v); }

// Index of the largest value among the lanes' candidates, the smallest index on a tie;
// lanes without a candidate pass index -1.
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

// Index of the smallest value, the smallest index on a tie; -1 candidates are ignored.
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

// Per-warp shared state.
struct WarpShared {
    double vec[4][64];  // p-sized vectors: free solution, scratch
    double tau[64];
    double rvec[64];    // NNLS residual rows / rotated data of the small QR
    double nrm_u[kMaxActive], nrm_d[kMaxActive];
    int act[kMaxActive];   // active columns, increasing
    int perm[kMaxActive];
    int n_act;
};

// Least squares on the active columns of c ((rows) x m, row-major) for the data e_{rows-1}:
// column-pivoted Householder QR with threshold max(rows, k) eps (cpp/src/sd/nnls.cpp:119-139);
// columns past the numerical rank get 0. Writes the coefficients of all m columns into z
// (zero off the active set).
__device__ void active_least_squares(const double* c, int rows, int m, double* sub, WarpShared& sh,
                                     double* z, int lane) {
    const int k = sh.n_act;
    for (int j = lane; j < m; j += 32) z[j] = 0.0;
    __syncwarp();
    if (k == 0) return;
    // sub (rows x kMaxActive) <- the active columns; column norms.
    for (int q = lane; q < k; q += 32) {
        const int col = sh.act[q];
        double s = 0.0;
        for (int r = 0; r < rows; ++r) {
            const double x = c[size_t(r) * m + col];
            sub[r * kMaxActive + q] = x;
            s += x * x;
        }
        sh.nrm_u[q] = sh.nrm_d[q] = sqrt(s);
        sh.perm[q] = q;
    }
    __syncwarp();
    double biggest = 0.0;
    for (int q = 0; q < k; ++q) biggest = fmax(biggest, sh.nrm_u[q]);
    const double th = biggest * kEps;
    const double small_sq = th * th / double(rows);
    const int size = min(rows, k);
    int nonzero = size;
    double maxpivot = 0.0;
    for (int kk = 0; kk < size; ++kk) {
        // Pivot: the largest remaining norm, the first on a tie.
        double v = -1.0;
        int idx = -1;
        for (int q = kk + lane; q < k; q += 32) {
            const double sq = sh.nrm_u[q] * sh.nrm_u[q];
            if (idx < 0 || sq > v) { v = sq; idx = q; }
        }
        const int best = warp_argmax_first(v, idx);
        const double best_sq = sh.nrm_u[best] * sh.nrm_u[best];
        if (nonzero == size && best_sq < small_sq * double(rows - kk)) nonzero = kk;
        __syncwarp();
        if (best != kk) {
            for (int r = lane; r < rows; r += 32) {
                const double t = sub[r * kMaxActive + kk];
                sub[r * kMaxActive + kk] = sub[r * kMaxActive + best];
                sub[r * kMaxActive + best] = t;
            }
            if (lane == 0) {
                double t = sh.nrm_u[kk]; sh.nrm_u[kk] = sh.nrm_u[best]; sh.nrm_u[best] = t;
                t = sh.nrm_d[kk]; sh.nrm_d[kk] = sh.nrm_d[best]; sh.nrm_d[best] = t;
                const int pt = sh.perm[kk]; sh.perm[kk] = sh.perm[best]; sh.perm[best] = pt;
            }
        }
        __syncwarp();
        // Householder reflector of column kk, rows kk.. (LAPACK dlarfg convention).
        const double c0 = sub[kk * kMaxActive + kk];
        double tail = 0.0;
        for (int r = kk + 1 + lane; r < rows; r += 32) tail += sub[r * kMaxActive + kk] * sub[r * kMaxActive + kk];
        tail = wsum(tail);
        double tau, beta;
        if (tail <= DBL_MIN) {
            tau = 0.0;
            beta = c0;
            for (int r = kk + 1 + lane; r < rows; r += 32) sub[r * kMaxActive + kk] = 0.0;
        } else {
            beta = sqrt(c0 * c0 + tail);
            if (c0 >= 0.0) beta = -beta;
            const double den = c0 - beta;
            for (int r = kk + 1 + lane; r < rows; r += 32) sub[r * kMaxActive + kk] /= den;
            tau = (beta - c0) / beta;
        }
        __syncwarp();
        if (lane == 0) {
            sub[kk * kMaxActive + kk] = beta;
            sh.tau[kk] = tau;
        }
        maxpivot = fmax(maxpivot, fabs(beta));
        __syncwarp();
        // Apply to the remaining columns and downdate their norms; lanes over columns.
        for (int q = kk + 1 + lane; q < k; q += 32) {
            if (tau != 0.0) {
                double dot = sub[kk * kMaxActive + q];
                for (int r = kk + 1; r < rows; ++r) dot += sub[r * kMaxActive + kk] * sub[r * kMaxActive + q];
                sub[kk * kMaxActive + q] -= tau * dot;
                for (int r = kk + 1; r < rows; ++r) sub[r * kMaxActive + q] -= tau * sub[r * kMaxActive + kk] * dot;
            }
            double& u = sh.nrm_u[q];
            if (u != 0.0) {
                double t = fabs(sub[kk * kMaxActive + q]) / u;
                t = fmax(0.0, (1.0 + t) * (1.0 - t));
                const double ratio = u / sh.nrm_d[q];
                if (t * ratio * ratio <= sqrt(kEps)) {
                    double s = 0.0;
                    for (int r = kk + 1; r < rows; ++r) s += sub[r * kMaxActive + q] * sub[r * kMaxActive + q];
                    sh.nrm_d[q] = sqrt(s);
                    u = sh.nrm_d[q];
                } else {
                    u *= sqrt(t);
                }
            }
        }
        __syncwarp();
    }
    const double thr = double(max(rows, k)) * kEps;
    int rank = 0;
    for (int i = 0; i < nonzero; ++i)
        if (fabs(sub[i * kMaxActive + i]) > maxpivot * thr) ++rank;
    // rotated = Q^T e_last with the first `rank` reflectors.
    for (int r = lane; r < rows; r += 32) sh.rvec[r] = (r == rows - 1) ? 1.0 : 0.0;
    __syncwarp();
    for (int kk = 0; kk < rank; ++kk) {
        const double tau = sh.tau[kk];
        if (tau == 0.0) continue;
        double dot = 0.0;
        for (int r = kk + 1 + lane; r < rows; r += 32) dot += sub[r * kMaxActive + kk] * sh.rvec[r];
        dot = wsum(dot) + sh.rvec[kk];
        __syncwarp();
        if (lane == 0) sh.rvec[kk] -= tau * dot;
        for (int r = kk + 1 + lane; r < rows; r += 32) sh.rvec[r] -= tau * sub[r * kMaxActive + kk] * dot;
        __syncwarp();
    }
    // R11 b = rotated[:rank], then scatter through the pivots.
    if (lane == 0) {
        for (int i = rank - 1; i >= 0; --i) {
            double s = sh.rvec[i];
            for (int j = i + 1; j < rank; ++j) s -= sub[i * kMaxActive + j] * sh.rvec[j];
            sh.rvec[i] = s / sub[i * kMaxActive + i];
        }
    }
    __syncwarp();
    for (int i = lane; i < rank; i += 32) z[sh.act[sh.perm[i]]] = sh.rvec[i];
    __syncwarp();
}

template <class Src>
__global__ void __launch_bounds__(kCWarps * 32) constrained_fit_kernel(
    LogDesignDevice<double> d, Src src, int weighted, ViolatorList<double> list, int* queue,
    double* __restrict__ workspace, size_t slot_doubles, double* __restrict__ params) {
    __shared__ WarpShared shared[kCWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpShared& sh = shared[warp];
    const int n = d.n, p = d.p, m = d.m, rows = p + 1;
    double* slot = workspace + (size_t(blockIdx.x) * kCWarps + warp) * slot_doubles;
    double* qr = slot;                          // (n, p) row-major
    double* cm = qr + size_t(n) * p;            // (rows, m) row-major
    double* sub = cm + size_t(rows) * m;        // (rows, kMaxActive)
    double* u = sub + size_t(rows) * kMaxActive;  // (m,)
    double* z = u + m;                          // (m,)
    double* ys = z + m;                         // (n,) log signals, then root weights after
    double* rw = ys + n;                        // (n,) root weights; also the rotated data
    const int total = min(*list.count, list.capacity);
    for (;;) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(queue, 1);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= total) break;
        const int64_t voxel = list.voxel[idx];
        double* pu = sh.vec[0];
        if (lane < p) pu[lane] = list.params[size_t(idx) * p + lane];
        src.template warp_stage<double>(voxel, ys, lane);
        __syncwarp();
        // Root weights exp(pred - max pred) of the unconstrained solution (:259-263).
        double mx = -INFINITY;
        for (int j = lane; j < n; j += 32) {
            double pred = 0.0;
            for (int a = 0; a < p; ++a) pred += d.x[size_t(j) * p + a] * pu[a];
            rw[j] = pred;
            mx = fmax(mx, pred);
        }
        mx = wmax(mx);
        __syncwarp();
        for (int j = lane; j < n; j += 32) rw[j] = weighted ? exp(rw[j] - mx) : 1.0;
        __syncwarp();
        // W^(1/2) X and W^(1/2) y.
        for (int i = lane; i < n * p; i += 32) qr[i] = rw[i / p] * d.x[i];
        for (int j = lane; j < n; j += 32) ys[j] = rw[j] * ys[j];
        __syncwarp();
        // Householder QR (unpivoted), rotating ys along.
        double* tau = sh.tau;
        for (int k = 0; k < p; ++k) {
            const double c0 = qr[size_t(k) * p + k];
            double tail = 0.0;
            for (int r = k + 1 + lane; r < n; r += 32) tail += qr[size_t(r) * p + k] * qr[size_t(r) * p + k];
            tail = wsum(tail);
            double tk, beta;
            if (tail <= DBL_MIN) {
                tk = 0.0;
                beta = c0;
                for (int r = k + 1 + lane; r < n; r += 32) qr[size_t(r) * p + k] = 0.0;
            } else {
                beta = sqrt(c0 * c0 + tail);
                if (c0 >= 0.0) beta = -beta;
                const double den = c0 - beta;
                for (int r = k + 1 + lane; r < n; r += 32) qr[size_t(r) * p + k] /= den;
                tk = (beta - c0) / beta;
            }
            __syncwarp();
            if (lane == 0) {
                qr[size_t(k) * p + k] = beta;
                tau[k] = tk;
            }
            __syncwarp();
            if (tk != 0.0) {
                // Columns j > k and the data: dot products by warp reductions over rows.
                for (int j = k + 1; j <= p; ++j) {
                    double dot = 0.0;
                    if (j < p) {
                        for (int r = k + 1 + lane; r < n; r += 32) dot += qr[size_t(r) * p + k] * qr[size_t(r) * p + j];
                        dot = wsum(dot) + qr[size_t(k) * p + j];
                        __syncwarp();
                        if (lane == 0) qr[size_t(k) * p + j] -= tk * dot;
                        for (int r = k + 1 + lane; r < n; r += 32) qr[size_t(r) * p + j] -= tk * qr[size_t(r) * p + k] * dot;
                    } else {
                        for (int r = k + 1 + lane; r < n; r += 32) dot += qr[size_t(r) * p + k] * ys[r];
                        dot = wsum(dot) + ys[k];
                        __syncwarp();
                        if (lane == 0) ys[k] -= tk * dot;
                        for (int r = k + 1 + lane; r < n; r += 32) ys[r] -= tk * qr[size_t(r) * p + k] * dot;
                    }
                    __syncwarp();
                }
            }
        }
        // Rank check on the diagonal of R (:183-188).
        double dmax = 0.0, dmin = INFINITY;
        for (int k = 0; k < p; ++k) {
            dmax = fmax(dmax, fabs(qr[size_t(k) * p + k]));
            dmin = fmin(dmin, fabs(qr[size_t(k) * p + k]));
        }
        if (!(dmin > double(n) * kEps * dmax)) continue;
        // p_free = R^-1 (Q^T W^(1/2) y)[:p].
        double* pfree = sh.vec[1];
        if (lane == 0) {
            for (int i = p - 1; i >= 0; --i) {
                double s = ys[i];
                for (int j = i + 1; j < p; ++j) s -= qr[size_t(i) * p + j] * pfree[j];
                pfree[i] = s / qr[size_t(i) * p + i];
            }
        }
        __syncwarp();
        // NNLS matrix: rows 0..p-1 = R^-T G^T, row p = -(G p_free)^T; lanes over constraints.
        double colsum_max = 0.0;
        for (int c = lane; c < m; c += 32) {
            const double* gr = d.g + size_t(c) * p;
            double acc_abs = 0.0, gf = 0.0;
            for (int i = 0; i < p; ++i) {
                double s = gr[i];
                for (int k = 0; k < i; ++k) s -= qr[size_t(k) * p + i] * cm[size_t(k) * m + c];
                s /= qr[size_t(i) * p + i];
                cm[size_t(i) * m + c] = s;
                acc_abs += fabs(s);
                gf += gr[i] * pfree[i];
            }
            cm[size_t(p) * m + c] = -gf;
            acc_abs += fabs(gf);
            colsum_max = fmax(colsum_max, acc_abs);
            u[c] = 0.0;
        }
        colsum_max = wmax(colsum_max);
        const double tol = 10.0 * kEps * colsum_max * double(max(rows, m));
        if (lane == 0) sh.n_act = 0;
        __syncwarp();
        // Lawson-Hanson (cpp/src/sd/nnls.cpp:187-221) on C u ~ e_p.
        const int max_inner = kInnerStepsPerConstraint * m;
        int inner = 0;
        bool converged = true, overflow = false;
        double* res = sh.vec[2];
        for (;;) {
            // r = e_p - C u over the active columns (u is zero elsewhere); lane = row.
            if (lane < rows) {
                double s = (lane == p) ? 1.0 : 0.0;
                for (int q = 0; q < sh.n_act; ++q) {
                    const int col = sh.act[q];
                    s -= cm[size_t(lane) * m + col] * u[col];
                }
                res[lane] = s;
            }
            __syncwarp();
            // The steepest inactive gradient C^T r, the first on a tie.
            double bestv = 0.0;
            int besti = -1;
            for (int c = lane; c < m; c += 32) {
                bool active = false;
                for (int q = 0; q < sh.n_act; ++q) active |= (sh.act[q] == c);
                if (active) continue;
                double gval = 0.0;
                for (int i = 0; i < rows; ++i) gval += cm[size_t(i) * m + c] * res[i];
                if (besti < 0 || gval > bestv) { bestv = gval; besti = c; }
            }
            const int e = warp_argmax_first(bestv, besti);
            double ge = __shfl_sync(0xffffffffu, bestv, 0);
            {
                // The value of the winner: recompute on every lane (uniform).
                double gval = 0.0;
                if (e >= 0)
                    for (int i = 0; i < rows; ++i) gval += cm[size_t(i) * m + e] * res[i];
                ge = gval;
            }
            if (e < 0 || ge <= tol) break;
            if (sh.n_act >= kMaxActive) { overflow = true; break; }
            // Insert e keeping the list increasing.
            if (lane == 0) {
                int q = sh.n_act;
                while (q > 0 && sh.act[q - 1] > e) { sh.act[q] = sh.act[q - 1]; --q; }
                sh.act[q] = e;
                ++sh.n_act;
            }
            __syncwarp();
            active_least_squares(cm, rows, m, sub, sh, z, lane);
            for (;;) {
                bool any = false;
                for (int q = lane; q < sh.n_act; q += 32) any |= z[sh.act[q]] <= 0.0;
                if (!__any_sync(0xffffffffu, any)) break;
                if (++inner > max_inner) { converged = false; break; }
                // Blocking step: the smallest u/(u - z) over active columns with z <= 0.
                double sv = INFINITY;
                int si = -1;
                for (int q = lane; q < sh.n_act; q += 32) {
                    const int col = sh.act[q];
                    if (z[col] > 0.0) continue;
                    const double dist = u[col] - z[col];
                    const double st = dist > 0.0 ? u[col] / dist : 0.0;
                    if (si < 0 || st < sv || (st == sv && col < si)) { sv = st; si = col; }
                }
                double step;
                const int bcol = warp_argmin_first(sv, si, &step);
                step = __shfl_sync(0xffffffffu, step, 0);
                for (int q = lane; q < sh.n_act; q += 32) {
                    const int col = sh.act[q];
                    u[col] += step * (z[col] - u[col]);
                }
                __syncwarp();
                if (lane == 0) {
                    u[bcol] = 0.0;
                    // Drop the blocking column and any whose coefficient rounding left below tol.
                    int w = 0;
                    for (int q = 0; q < sh.n_act; ++q) {
                        const int col = sh.act[q];
                        if (col == bcol || !(fabs(u[col]) >= tol)) {
                            if (col != bcol) { /* stays at its value, inactive */ }
                            continue;
                        }
                        sh.act[w++] = col;
                    }
                    sh.n_act = w;
                }
                __syncwarp();
                active_least_squares(cm, rows, m, sub, sh, z, lane);
            }
            if (!converged) break;
            // u = z (zero off the active set).
            for (int c = lane; c < m; c += 32) u[c] = z[c];
            __syncwarp();
        }
        if (!converged || overflow) continue;
        // Residual C u - e_p over all columns with non-zero u.
        if (lane < rows) {
            double s = (lane == p) ? -1.0 : 0.0;
            for (int c = 0; c < m; ++c) {
                const double uc = u[c];
                if (uc != 0.0) s += cm[size_t(lane) * m + c] * uc;
            }
            res[lane] = s;
        }
        __syncwarp();
        const double last = res[p];
        if (last >= -kFeasibilityMargin) continue;
        // p = p_free + R^-1 (-res[:p] / res[p]).
        double* pc = sh.vec[3];
        if (lane == 0) {
            for (int i = p - 1; i >= 0; --i) {
                double s = -res[i] / last;
                for (int j = i + 1; j < p; ++j) s -= qr[size_t(i) * p + j] * pc[j];
                pc[i] = s / qr[size_t(i) * p + i];
            }
            for (int i = 0; i < p; ++i) pc[i] = pfree[i] + pc[i];
        }
        __syncwarp();
        bool finite = true;
        for (int a = 0; a < p; ++a) finite &= bool(isfinite(pc[a]));
        if (!finite) continue;
        // meets_the_constraints (:156-163).
        double vmin = INFINITY, size = 0.0;
        for (int c = lane; c < m; c += 32) {
            const double* gr = d.g + size_t(c) * p;
            double val = 0.0, sz = 0.0;
            for (int a = 0; a < p; ++a) {
                val += gr[a] * pc[a];
                sz += fabs(gr[a]) * (fabs(pc[a]) + fabs(pfree[a]));
            }
            vmin = fmin(vmin, val);
            size = fmax(size, sz);
        }
        vmin = -wmax(-vmin);
        size = wmax(size);
        if (!(vmin >= -kConstraintTolerance * size)) continue;
        if (lane < p) params[voxel * p + lane] = pc[lane] / d.scales64[lane];
        __syncwarp();
    }
}

}  // namespace

template <class Src>
void launch_constrained(const LogDesignDevice<double>& d, const Src& src, int weighted,
                        const ViolatorList<double>& list, int /*list_count_host_bound*/, int* queue,
                        double* workspace, int slots, double* params, cudaStream_t stream) {
    require(d.p + 1 <= 32, "the constrained fit takes at most 31 parameters");
    const int blocks = std::max(1, slots / kCWarps);
    constrained_fit_kernel<Src><<<blocks, kCWarps * 32, 0, stream>>>(
        d, src, weighted, list, queue, workspace, constrained_slot_doubles(d.n, d.p, d.m), params);
    cuda_check(cudaGetLastError(), "constrained_fit_kernel launch");
}

template void launch_constrained<LogSource>(const LogDesignDevice<double>&, const LogSource&, int,
                                            const ViolatorList<double>&, int, int*, double*, int, double*,
                                            cudaStream_t);
template void launch_constrained<CappedSource>(const LogDesignDevice<double>&, const CappedSource&, int,
                                               const ViolatorList<double>&, int, int*, double*, int, double*,
                                               cudaStream_t);

}  // namespace lar
