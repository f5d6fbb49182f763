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

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "common.cuh"
#include "log_fit.cuh"
#include "log_fit_warp.cuh"
#include "warp_nnls.cuh"

namespace lar {

namespace {

constexpr int kCWarps = 4;
constexpr double kEps = kEps64;
constexpr double kFeasibilityMargin = 1e-12;
constexpr int kInnerStepsPerConstraint = 50;
constexpr double kConstraintTolerance = 1e-9;

__device__ __forceinline__ double wsum(double v) { return warp_sum(v); }
__device__ __forceinline__ double wmax(double v) { return warp_max(v); }

// Per-warp shared state.
struct WarpShared {
    double vec[4][64];  // p-sized vectors: unconstrained and free solutions, scratch
    double tau[64];     // reflectors of the weighted design
    double qtau[kMaxActive], qnu[kMaxActive], qnd[kMaxActive], rv[64], res[64];
    int qperm[kMaxActive];
    int act[kMaxActive];
    int n_act;
};

template <class Src>
__global__ void __launch_bounds__(kCWarps * 32, 4) constrained_fit_kernel(
    LogDesignDevice<double> d, Src src, int weighted, ViolatorList<double> list, int* queue,
    double* __restrict__ workspace, size_t slot_doubles, double* __restrict__ params) {
    __shared__ WarpShared shared[kCWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpShared& sh = shared[warp];
    const int n = d.n, p = d.p, m = d.m, rows = p + 1;
    double* slot = workspace + (size_t(blockIdx.x) * kCWarps + warp) * slot_doubles;
    double* qr = slot;                          // (n, p) row-major
    double* cm = qr + size_t(n) * p;            // (rows, m) row-major
    double* sub = cm + size_t(rows) * m;        // (kMaxActive, rows) QR of the active columns
    double* u = sub + size_t(rows) * kMaxActive;  // (m,)
    double* z = u + m;                          // (m,)
    double* ys = z + m;                         // (n,) log signals, then weighted
    double* rw = ys + n;                        // (n,) root weights
    uint8_t* flag = reinterpret_cast<uint8_t*>(rw + n);  // (m,) active flags
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
                // Columns j > k and the data (column p), eight at a time: the dot products of a
                // group in one pass over the rows and independent warp reductions, then the
                // updates. Each dot keeps its rows' order and its reduction's.
                for (int j0 = k + 1; j0 <= p; j0 += 8) {
                    double dv[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) dv[q] = 0.0;
                    for (int r = k + 1 + lane; r < n; r += 32) {
                        const double vr = qr[size_t(r) * p + k];
                        const double* row = qr + size_t(r) * p;
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int j = j0 + q;
                            if (j < p) dv[q] += vr * row[j];
                            else if (j == p) dv[q] += vr * ys[r];
                        }
                    }
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int j = j0 + q;
                        if (j <= p) dv[q] = wsum(dv[q]) + (j < p ? qr[size_t(k) * p + j] : ys[k]);
                    }
                    __syncwarp();
                    if (lane == 0) {
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int j = j0 + q;
                            if (j < p) qr[size_t(k) * p + j] -= tk * dv[q];
                            else if (j == p) ys[k] -= tk * dv[q];
                        }
                    }
                    for (int r = k + 1 + lane; r < n; r += 32) {
                        double* row = qr + size_t(r) * p;
                        const double vr = row[k];
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int j = j0 + q;
                            if (j < p) row[j] -= tk * vr * dv[q];
                            else if (j == p) ys[r] -= tk * vr * dv[q];
                        }
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
        // NNLS matrix: rows 0..p-1 = R^-T G^T, row p = -(G p_free)^T; lanes over constraints, four
        // columns at a time so that their substitution chains overlap.
        double colsum_max = 0.0;
        for (int c0 = lane; c0 < m; c0 += 4 * 32) {
            int cc[4];
            bool in[4];
            double acc_abs[4], gf[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                cc[q] = c0 + 32 * q;
                in[q] = cc[q] < m;
                acc_abs[q] = 0.0;
                gf[q] = 0.0;
            }
            for (int i = 0; i < p; ++i) {
                double sv[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) sv[q] = in[q] ? d.g[size_t(cc[q]) * p + i] : 0.0;
                for (int k = 0; k < i; ++k) {
                    const double rki = qr[size_t(k) * p + i];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (in[q]) sv[q] -= rki * cm[size_t(k) * m + cc[q]];
                }
                const double rii = qr[size_t(i) * p + i];
                const double pf = pfree[i];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (!in[q]) continue;
                    const double si = sv[q] / rii;
                    cm[size_t(i) * m + cc[q]] = si;
                    acc_abs[q] += fabs(si);
                    gf[q] += d.g[size_t(cc[q]) * p + i] * pf;
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (!in[q]) continue;
                cm[size_t(p) * m + cc[q]] = -gf[q];
                acc_abs[q] += fabs(gf[q]);
                colsum_max = fmax(colsum_max, acc_abs[q]);
                u[cc[q]] = 0.0;
            }
        }
        colsum_max = wmax(colsum_max);
        const double tol = 10.0 * kEps * colsum_max * double(max(rows, m));
        // Lawson-Hanson (cpp/src/sd/nnls.cpp:187-221) on C u ~ e_p.
        double* unit = sh.rv;  // e_p, then the residual rows below
        for (int r = lane; r < rows; r += 32) unit[r] = (r == p) ? 1.0 : 0.0;
        __syncwarp();
        double* unit_copy = sh.vec[2];
        for (int r = lane; r < rows; r += 32) unit_copy[r] = unit[r];
        __syncwarp();
        NnlsScratch ns{u, z, flag, sh.act, &sh.n_act, sh.res,
                       QrScratch{sub, sh.qtau, sh.qnu, sh.qnd, sh.qperm, sh.rv}, kMaxActive};
        const int outcome = warp_nnls_explicit(cm, rows, m, unit_copy, tol, kInnerStepsPerConstraint * m, ns, lane);
        if (outcome != 1) continue;
        double* res = sh.vec[2];
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

int constrained_resident_warps() {
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, constrained_fit_kernel<CappedSource>,
                                                             kCWarps * 32, 0),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    return sm_count() * ctas_per_sm(per_sm, "dki.refit.ctas_per_sm") * kCWarps;
}

template <class Src>
void launch_constrained(const LogDesignDevice<double>& d, const Src& src, int weighted,
                        const ViolatorList<double>& list, int /*list_count_host_bound*/, int* queue,
                        double* workspace, int slots, double* params, cudaStream_t stream) {
    require(d.p + 1 <= 32, "the constrained fit takes at most 31 parameters");
    const int blocks = std::max(1, slots / kCWarps);
    LaunchScope scope("constrained_fit_kernel", stream);
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
