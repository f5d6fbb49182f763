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
// The NNLS matrix C = [R^-T G^T; -(G p_free)^T] ((p+1) x m) is never formed whole. Its
// gradient C^T r is G t with t = R^-1 r[:p] - r[p] p_free (G, shared by every voxel, stays in
// L2), and only the columns that join the active set are formed, each once per voxel, into a
// column cache. So a voxel moves its design's QR and the few columns it uses, not the 768-column
// system (which made the kernel move ~300x its algorithmic bytes).
//
// Work distribution: the violators were compacted into a list by the unconstrained fit; a
// fixed number of warps take them from a device work counter (no host round trip, so the pair
// of launches can be captured in a CUDA graph). Each warp owns a slot of global scratch
// memory: the QR of the weighted design (n x p), the column cache (m x (p+1), touched only for
// the columns used), the active columns' QR ((p+1) x 64), and the NNLS vectors. Lanes split
// the rows of the design for the reflections, the m constraint columns for gradients and
// steps, and the active columns for the small QR.

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "batch.cuh"
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

// Per-warp shared state (p + 1 <= 32).
struct WarpState {
    double vec[4][32];  // p- or (p+1)-sized vectors: unconstrained and free solutions, scratch
    double tau[32];     // reflectors of the weighted design
    double qtau[kMaxActive], qnu[kMaxActive], qnd[kMaxActive], rv[32], res[32];
    double t[32];       // R^-1 r[:p] - r[p] p_free of the gradient
    int qperm[kMaxActive];
    int act[kMaxActive];
    int n_act;
};

// With the column sums' forward substitutions (one per lane, entry i at [i * 32 + lane]).
struct WarpShared : WarpState {
    double ysub[31 * 32];
};

constexpr int kSmemActive = 32;  // active NNLS columns whose QR fits can run in shared memory

// Where a violator's re-fit keeps its arrays: the weighted design's QR (n, p), the log signals and
// root weights (n each), the column sums' substitutions (31 x 32), the NNLS system's formed
// columns (m, p + 1), the QR of the active columns (kMaxActive, p + 1; ssub, when set, holds
// that of up to kSmemActive columns in shared memory), the NNLS vectors and flags (m each).
struct RefitMem {
    double *qr, *ys, *rw, *ysub, *ssub, *cache, *sub, *u, *z;
    uint8_t *flag, *ready;
};

// The slot layout of a warp (constrained_slot_doubles), with qr, ys and rw in it.
__device__ __forceinline__ RefitMem slot_refit_mem(double* slot, int n, int p, int m) {
    RefitMem r;
    const int rows = p + 1;
    r.qr = slot;
    r.cache = r.qr + size_t(n) * p;
    r.sub = r.cache + size_t(rows) * m;
    r.u = r.sub + size_t(rows) * kMaxActive;
    r.z = r.u + m;
    r.ys = r.z + m;
    r.rw = r.ys + n;
    r.flag = reinterpret_cast<uint8_t*>(r.rw + n);
    r.ready = r.flag + m;
    r.ysub = nullptr;
    r.ssub = nullptr;
    return r;
}

// Whether the column sums' substitutions fit in the QR's rows below R (dead by then).
__host__ __device__ inline bool refit_ysub_aliased(int n, int p) { return size_t(n - p) * p >= 31 * 32; }

// A warp's shared-memory doubles when its QR, signals, weights and small NNLS fits live there.
__host__ __device__ inline size_t refit_smem_doubles(int n, int p) {
    return size_t(n) * p + 2 * size_t(n) + size_t(p + 1) * kSmemActive + (refit_ysub_aliased(n, p) ? 0 : 31 * 32);
}

// The NNLS system C = [R^-T G^T; -(G p_free)^T] of one voxel, formed column by column on demand.
struct ImplicitSystem {
    const double* g;      // (m, p) constraints
    const double* gt;     // (p, m) the same, transposed
    const double* qr;     // (n, p): R in its upper triangle
    const double* pfree;  // (p,)
    double* cache;        // (m, p + 1)
    uint8_t* ready;       // (m,)
    int p, m;
    // Column c into the cache, unless it is there: the forward substitution R^T y = g_c with
    // lane i holding entry i (column-oriented: entry k is final once the rows above it are
    // subtracted), then y_p = -g_c p_free.
    __device__ void form(int c, int lane) const {
        if (ready[c]) return;
        const double* gc = g + size_t(c) * p;
        double* col = cache + size_t(c) * (p + 1);
        const double gi = lane < p ? gc[lane] : 0.0;
        double si = gi;
        for (int k = 0; k < p; ++k) {
            const double yk = __shfl_sync(0xffffffffu, si, k) / qr[size_t(k) * p + k];
            if (lane > k && lane < p) si -= qr[size_t(k) * p + lane] * yk;
            if (lane == k) si = yk;
        }
        const double gf = warp_sum(lane < p ? gi * pfree[lane] : 0.0);
        if (lane < p) col[lane] = si;
        if (lane == 0) {
            col[p] = -gf;
            ready[c] = 1;
        }
        __syncwarp();
    }
};

struct CachedColumns {
    const double* cache;
    int rows;
    __device__ __forceinline__ double operator()(int r, int col, int /*q*/) const {
        return cache[size_t(col) * rows + r];
    }
};

// Lawson-Hanson with QR fits on C (rows = p + 1, m columns) and d, as warp_nnls_explicit, with
// C's gradient C^T (d - C u) = G t and the active columns from the cache. Returns 1 when the
// method ended by its rule, 0 when the inner-step limit ran out, -1 past acap active columns.
__device__ int implicit_nnls(const ImplicitSystem& sys, const double* d, double tol, int max_inner, NnlsScratch s,
                             double* t, double* ssub, int lane) {
    const int m = sys.m, p = sys.p, rows = p + 1;
    const CachedColumns cols{sys.cache, rows};
    // The fit on the active columns, its QR in shared memory (ssub) when given and large enough.
    auto fit = [&]() {
        QrScratch q = s.qr;
        if (ssub != nullptr && *s.n_act <= kSmemActive) q.sub = ssub;
        warp_qr_least_squares_cols(cols, rows, s.act, *s.n_act, d, q, s.z, lane);
    };
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
            for (int q = 0; q < na; ++q) acc -= sys.cache[size_t(s.act[q]) * rows + r] * s.u[s.act[q]];
            s.res[r] = acc;
        }
        __syncwarp();
        // t = R^-1 res[:p] - res[p] p_free: column-oriented back substitution, lane i holding
        // entry i (entry k is final once the columns right of it are subtracted).
        {
            double yi = lane < p ? s.res[lane] : 0.0;
            for (int k = p - 1; k >= 0; --k) {
                const double tk = __shfl_sync(0xffffffffu, yi, k) / sys.qr[size_t(k) * p + k];
                if (lane < k) yi -= sys.qr[size_t(lane) * p + k] * tk;
                if (lane == k) yi = tk;
            }
            if (lane < p) t[lane] = yi - s.res[p] * sys.pfree[lane];
        }
        __syncwarp();
        // The gradient of every inactive column, g_c . t, lanes over the columns (each lane in
        // increasing order: the first on a tie).
        double bv = 0.0;
        int bi = -1;
        for (int c = lane; c < m; c += 32) {
            if (s.flag[c]) continue;
            double w = 0.0;
            for (int a = 0; a < p; ++a) w += sys.gt[size_t(a) * m + c] * t[a];
            if (bi < 0 || w > bv) {
                bv = w;
                bi = c;
            }
        }
        const int e = warp_argmax_first(bv, bi);
        const double ge = e >= 0 ? __shfl_sync(0xffffffffu, bv, e & 31) : 0.0;
        if (e < 0 || ge <= tol) return 1;
        if (na >= s.acap) return -1;
        sys.form(e, lane);
        if (lane == 0) {
            int q = na;
            while (q > 0 && s.act[q - 1] > e) {
                s.act[q] = s.act[q - 1];
                --q;
            }
            s.act[q] = e;
            *s.n_act = na + 1;
            s.flag[e] = 1;
        }
        __syncwarp();
        fit();
        for (;;) {
            const int n2 = *s.n_act;
            bool any = false;
            for (int q = lane; q < n2; q += 32) any |= s.z[s.act[q]] <= 0.0;
            if (!__any_sync(0xffffffffu, any)) break;
            if (++inner > max_inner) {
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
                if (si < 0 || st < sv || (st == sv && col < si)) {
                    sv = st;
                    si = col;
                }
            }
            double step;
            const int bcol = warp_argmin_first(sv, si, &step);
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
            fit();
        }
        for (int j = lane; j < m; j += 32) s.u[j] = s.flag[j] ? s.z[j] : 0.0;
        __syncwarp();
    }
}

// The constrained re-fit of one violator on a warp (its unconstrained scaled parameters in
// pin): where every step succeeds, out (p) gets the constrained parameters.
template <class Src>
__device__ __forceinline__ void refit_violator(const LogDesignDevice<double>& d, const Src& src, int weighted,
                                               int64_t voxel, const double* pin, const RefitMem& mem, WarpState& sh,
                                               double* out, int lane) {
    const int n = d.n, p = d.p, m = d.m, rows = p + 1;
    double* const qr = mem.qr;
    double* const cache = mem.cache;
    double* const sub = mem.sub;
    double* const u = mem.u;
    double* const z = mem.z;
    double* const ys = mem.ys;
    double* const rw = mem.rw;
    uint8_t* const flag = mem.flag;
    uint8_t* const ready = mem.ready;
    double* pu = sh.vec[0];
    if (lane < p) pu[lane] = pin[lane];
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
    if (!(dmin > double(n) * kEps * dmax)) return;
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
    // The NNLS tolerance 10 eps norm1(C) max(p + 1, m) needs every column's absolute sum:
    // sum_i |(R^-T g_c)_i| + |g_c p_free|. Lanes over constraints, each substitution's
    // entries in the warp's shared column of ysub; the columns themselves are not kept.
    double colsum_max = 0.0;
    double* ysub = mem.ysub;
    for (int c = lane; c < m; c += 32) {
        const double* gc = d.g + size_t(c) * p;
        double acc_abs = 0.0, gf = 0.0;
        for (int i = 0; i < p; ++i) {
            double s0 = gc[i], s1 = 0.0;
            int k = 0;
            for (; k + 1 < i; k += 2) {
                s0 -= qr[size_t(k) * p + i] * ysub[k * 32 + lane];
                s1 -= qr[size_t(k + 1) * p + i] * ysub[(k + 1) * 32 + lane];
            }
            if (k < i) s0 -= qr[size_t(k) * p + i] * ysub[k * 32 + lane];
            const double si = (s0 + s1) / qr[size_t(i) * p + i];
            ysub[i * 32 + lane] = si;
            acc_abs += fabs(si);
            gf += gc[i] * pfree[i];
        }
        acc_abs += fabs(gf);
        colsum_max = fmax(colsum_max, acc_abs);
    }
    colsum_max = wmax(colsum_max);
    const double tol = 10.0 * kEps * colsum_max * double(max(rows, m));
    for (int c = lane; c < m; c += 32) ready[c] = 0;
    __syncwarp();
    // Lawson-Hanson (cpp/src/sd/nnls.cpp:187-221) on C u ~ e_p.
    double* unit = sh.vec[2];
    for (int r = lane; r < rows; r += 32) unit[r] = (r == p) ? 1.0 : 0.0;
    __syncwarp();
    const ImplicitSystem sys{d.g, d.gt, qr, pfree, cache, ready, p, m};
    NnlsScratch ns{u, z, flag, sh.act, &sh.n_act, sh.res,
                   QrScratch{sub, sh.qtau, sh.qnu, sh.qnd, sh.qperm, sh.rv}, kMaxActive};
    const int outcome = implicit_nnls(sys, unit, tol, kInnerStepsPerConstraint * m, ns, sh.t, mem.ssub, lane);
    if (outcome != 1) return;
    double* res = sh.vec[2];
    // Residual C u - e_p over the active columns (u is zero elsewhere).
    if (lane < rows) {
        double s = (lane == p) ? -1.0 : 0.0;
        for (int q = 0; q < sh.n_act; ++q) {
            const int c = sh.act[q];
            const double uc = u[c];
            if (uc != 0.0) s += cache[size_t(c) * rows + lane] * uc;
        }
        res[lane] = s;
    }
    __syncwarp();
    const double last = res[p];
    if (last >= -kFeasibilityMargin) return;
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
    if (!finite) return;
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
    if (!(vmin >= -kConstraintTolerance * size)) return;
    if (lane < p) out[lane] = pc[lane] / d.scales64[lane];
    __syncwarp();
}

template <class Src>
__global__ void __launch_bounds__(kCWarps * 32, 4) constrained_fit_kernel(
    LogDesignDevice<double> d, Src src, int weighted, ViolatorList<double> list, int* queue,
    double* __restrict__ workspace, size_t slot_doubles, double* __restrict__ params) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WarpShared* shared = reinterpret_cast<WarpShared*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpShared& sh = shared[warp];
    const int p = d.p;
    double* slot = workspace + (size_t(blockIdx.x) * kCWarps + warp) * slot_doubles;
    const int total = min(*list.count, list.capacity);
    for (;;) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(queue, 1);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= total) break;
        const int64_t voxel = list.voxel[idx];
        RefitMem mem = slot_refit_mem(slot, d.n, p, d.m);
        mem.ysub = sh.ysub;
        refit_violator<Src>(d, src, weighted, voxel, list.params + size_t(idx) * p, mem, sh, params + voxel * p,
                            lane);
    }
}

// The same re-fit with one warp per CTA and the weighted design's QR, signals, weights and the
// QR of up to kSmemActive active NNLS columns in shared memory (refit_smem_doubles): a violator
// takes ~3x fewer warp cycles than with them in the global slot, at fewer warps per SM, which
// pays while a warp's state stays small (a modest table; see launch_constrained).
template <class Src>
__global__ void __launch_bounds__(32) constrained_fit_smem_kernel(
    LogDesignDevice<double> d, Src src, int weighted, ViolatorList<double> list, int* queue,
    double* __restrict__ workspace, size_t slot_doubles, double* __restrict__ params) {
    __shared__ WarpState sh;
    extern __shared__ __align__(16) double wsm[];
    const int lane = threadIdx.x & 31;
    const int n = d.n, p = d.p, rows = p + 1;
    double* slot = workspace + size_t(blockIdx.x) * slot_doubles;
    RefitMem mem = slot_refit_mem(slot, n, p, d.m);
    mem.qr = wsm;
    mem.ys = mem.qr + size_t(n) * p;
    mem.rw = mem.ys + n;
    mem.ssub = mem.rw + n;
    mem.ysub = refit_ysub_aliased(n, p) ? mem.qr + size_t(p) * p : mem.ssub + size_t(rows) * kSmemActive;
    const int total = min(*list.count, list.capacity);
    for (;;) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(queue, 1);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= total) break;
        const int64_t voxel = list.voxel[idx];
        refit_violator<Src>(d, src, weighted, voxel, list.params + size_t(idx) * p, mem, sh, params + voxel * p,
                            lane);
    }
}

// The DKI family of a batch (batch.cuh): warps take the violators of every DKI volume from one
// list, each with its volume's design, signals and outputs.
__global__ void __launch_bounds__(kCWarps * 32, 4) batch_refit_kernel(
    const DkiBatchJob* __restrict__ jobs, BatchViolators list, int weighted, int* queue,
    double* __restrict__ workspace, size_t slot_doubles) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WarpShared* shared = reinterpret_cast<WarpShared*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpShared& sh = shared[warp];
    double* slot = workspace + (size_t(blockIdx.x) * kCWarps + warp) * slot_doubles;
    const int total = min(*list.count, list.capacity);
    for (;;) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(queue, 1);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= total) break;
        const DkiBatchJob& job = jobs[list.job[idx]];
        const LogDesignDevice<double> d = job.d;
        const CappedSource src{job.s, job.s0, job.floor, job.is_b0, d.n};
        const int64_t voxel = list.voxel[idx];
        RefitMem mem = slot_refit_mem(slot, d.n, d.p, d.m);
        mem.ysub = sh.ysub;
        refit_violator<CappedSource>(d, src, weighted, voxel, list.params + size_t(idx) * d.p, mem, sh,
                                     job.params + voxel * d.p, lane);
    }
}

}  // namespace

constexpr size_t kCSmem = kCWarps * sizeof(WarpShared);

template <class Src>
void allow_smem() {
    static_assert(kCSmem <= 200 * 1024, "the re-fit's shared state outgrows an SM");
    cuda_check(cudaFuncSetAttribute(constrained_fit_kernel<Src>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(kCSmem)),
               "cudaFuncSetAttribute");
}

// The shared-memory re-fit is used while a warp's state stays within this many bytes (at least
// five warps per SM): on the 134-measurement DKI table (35 KB, six warps per SM) it took 187 ms
// against 213 ms with the state in the global slot at sixteen warps per SM, on the 288-measurement
// tables (65 KB, three warps per SM) it lost.
constexpr size_t kSmemRefitMaxBytes = 40 * 1024;

bool use_smem_refit(int n, int p) {
    return refit_smem_doubles(n, p) * sizeof(double) + sizeof(WarpState) <= kSmemRefitMaxBytes;
}

int global_resident_warps() {
    int per_sm = 0;
    allow_smem<CappedSource>();
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, constrained_fit_kernel<CappedSource>,
                                                             kCWarps * 32, kCSmem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    return sm_count() * ctas_per_sm(per_sm, "dki.refit.ctas_per_sm") * kCWarps;
}

template <class Kernel>
void allow_refit_smem(Kernel kernel, size_t bytes) {
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)),
               "cudaFuncSetAttribute");
}

int constrained_resident_warps(int n, int p) {
    if (!use_smem_refit(n, p)) return global_resident_warps();
    const size_t bytes = refit_smem_doubles(n, p) * sizeof(double);
    allow_refit_smem(constrained_fit_smem_kernel<CappedSource>, bytes);
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, constrained_fit_smem_kernel<CappedSource>, 32,
                                                             bytes),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    return sm_count() * ctas_per_sm(per_sm, "dki.refit.ctas_per_sm") / 4 * 4;
}

size_t batch_refit_slot_doubles(int n_max, int p, int m_max) { return constrained_slot_doubles(n_max, p, m_max); }

// Batches keep the global slot: their shared memory would be sized for the largest table.
int batch_refit_slots() { return global_resident_warps(); }

void launch_batch_refit(const DkiBatchJob* jobs, const BatchViolators& violators, int weighted, int* queue,
                        double* workspace, int slots, size_t slot_doubles, cudaStream_t stream) {
    const int blocks = std::max(1, slots / kCWarps);
    cuda_check(cudaFuncSetAttribute(batch_refit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kCSmem)),
               "cudaFuncSetAttribute");
    cuda_check(cudaMemsetAsync(queue, 0, sizeof(int), stream), "cudaMemsetAsync");
    LaunchScope scope("batch_refit_kernel", stream);
    batch_refit_kernel<<<blocks, kCWarps * 32, kCSmem, stream>>>(jobs, violators, weighted, queue, workspace,
                                                                 slot_doubles);
    cuda_check(cudaGetLastError(), "batch_refit_kernel launch");
}

template <class Src>
void launch_constrained(const LogDesignDevice<double>& d, const Src& src, int weighted,
                        const ViolatorList<double>& list, int /*list_count_host_bound*/, int* queue,
                        double* workspace, int slots, double* params, cudaStream_t stream) {
    require(d.p + 1 <= 32, "the constrained fit takes at most 31 parameters");
    if (use_smem_refit(d.n, d.p)) {
        const size_t bytes = refit_smem_doubles(d.n, d.p) * sizeof(double);
        allow_refit_smem(constrained_fit_smem_kernel<Src>, bytes);
        LaunchScope scope("constrained_fit_kernel", stream);
        constrained_fit_smem_kernel<Src><<<std::max(1, slots), 32, bytes, stream>>>(
            d, src, weighted, list, queue, workspace, constrained_slot_doubles(d.n, d.p, d.m), params);
        cuda_check(cudaGetLastError(), "constrained_fit_smem_kernel launch");
        return;
    }
    const int blocks = std::max(1, slots / kCWarps);
    allow_smem<Src>();
    LaunchScope scope("constrained_fit_kernel", stream);
    constrained_fit_kernel<Src><<<blocks, kCWarps * 32, kCSmem, stream>>>(
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
