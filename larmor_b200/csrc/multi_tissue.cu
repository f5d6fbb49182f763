// Multi-tissue spherical deconvolution (SDModel's mFOD method) on the GPU.
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
// Work distribution: the voxels go through the rounds together, each round as three kernels
// over the list of voxels still iterating:
//   correlate_kernel  K^T max(s_w - W_iso f_iso, 0) for 32 voxels x 16 RC columns per CTA, the
//                     signals built while the tile is staged in shared memory (a tiled FP64
//                     product, each entry summed over the measurements in increasing order);
//   ridge_nnls_kernel the active-set NNLS on the Gram matrix and those correlations, one warp per
//                     voxel (no work of the measurements' length unless the QR fallback runs);
//   lr_fractions_kernel  the fractions, the convergence test and the next round's voxel list.
// The high-resolution FOD then runs the first two for all voxels, and hr_fractions_kernel the
// final fractions. Each kernel's code is small (the warps of an SM share their instruction
// cache), and the per-voxel state between kernels lives in HBM.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "host_la.hpp"
#include "drl.cuh"
#include "group_nnls.cuh"
#include "plain_fp32.cuh"
#include "warp_chol.cuh"
#include "warp_nnls.cuh"

namespace lar {

namespace {

constexpr int kMtWarps = 4;
constexpr int kCholCap = 256;   // active columns the Cholesky factor holds
constexpr int kQrCap = 64;      // active columns of the ridge QR fallback
constexpr int kMaxGroups = 16;  // fraction columns (anisotropic groups + isotropic tissues)
constexpr double kMinPivot = 1e-12;
constexpr int kMaxColumns = 640;  // kernel columns (directions) a solver may have
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

// The signal a ridge NNLS fits, entry i of voxel v: s(v, i) itself (single tissue), or
// max(s(v, i) w_i - sum_t W_iso(i, t) f_iso(v, t), 0) (cpp/src/sd/multi_tissue.cpp:68-72).
struct SignalDev {
    const double* s;     // (v, m)
    const double* w;     // (m,) or null: the plain signal
    const double* wiso;  // (m, ci)
    const double* fiso;  // (v, ci)
    int m, ci;
    __device__ __forceinline__ double operator()(int64_t voxel, int i) const {
        const double si = s[voxel * m + i];
        if (w == nullptr) return si;
        const double ws = __dmul_rn(si, w[i]);
        double r = 0.0;
        for (int t = 0; t < ci; ++t) r = fma(wiso[size_t(i) * ci + t], fiso[voxel * ci + t], r);
        return fmax(ws - r, 0.0);
    }
};

// The voxel at position p of a round's list (the identity when there is no list).
__device__ __forceinline__ int64_t listed(const int* list, int64_t p) { return list ? int64_t(list[p]) : p; }

// ---- correlations ----------------------------------------------------------------------

constexpr int kCorrVoxels = 32;  // voxels per CTA tile
constexpr int kCorrResidentCtas = 8;  // CTAs per SM of a correlation grid whose count is on the device
constexpr int kCorrDepth = 16;   // measurements per shared-memory stage

// corr(v, j) = sum_i K(i, j) signal(v, i), i increasing, for the listed voxels: 128 threads as
// 8 voxel lanes x 16 column lanes, each with 4 voxels x RC columns of the tile.
// corr(v, j) for the kCorrVoxels voxels vox[] (shared; -1: none) and the columns col0 .. col0 +
// 16 RC - 1 of the tile: 128 threads as 8 voxel lanes x 16 column lanes, each with 4 voxels x RC
// columns; each entry summed in increasing measurement order.
template <int RC>
__device__ __forceinline__ void correlate_tile(const SignalDev& S, const int64_t* vox, const double* __restrict__ k,
                                               int c, int col0, double* __restrict__ corr, int ldc) {
    constexpr int TC = 16 * RC;
    __shared__ double sig_t[kCorrDepth][kCorrVoxels + 1];
    __shared__ double k_t[kCorrDepth][TC];
    const int tid = threadIdx.x, tv = tid & 7, tc = tid >> 3;
    const int m = S.m;
    double acc[4][RC];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < RC; ++b) acc[a][b] = 0.0;
    for (int i0 = 0; i0 < m; i0 += kCorrDepth) {
        const int depth = min(kCorrDepth, m - i0);
        for (int e = tid; e < kCorrVoxels * kCorrDepth; e += 128) {
            const int vv = e / kCorrDepth, ii = e % kCorrDepth;
            const int64_t voxel = vox[vv];
            sig_t[ii][vv] = (voxel >= 0 && ii < depth) ? S(voxel, i0 + ii) : 0.0;
        }
        for (int e = tid; e < kCorrDepth * TC; e += 128) {
            const int ii = e / TC, cc = e % TC;
            const int col = col0 + cc;
            k_t[ii][cc] = (ii < depth && col < c) ? k[size_t(i0 + ii) * c + col] : 0.0;
        }
        __syncthreads();
        for (int ii = 0; ii < depth; ++ii) {
            double sv[4], kv[RC];
#pragma unroll
            for (int a = 0; a < 4; ++a) sv[a] = sig_t[ii][tv + 8 * a];
#pragma unroll
            for (int b = 0; b < RC; ++b) kv[b] = k_t[ii][tc + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < RC; ++b) acc[a][b] = fma(kv[b], sv[a], acc[a][b]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int64_t voxel = vox[tv + 8 * a];
        if (voxel < 0) continue;
#pragma unroll
        for (int b = 0; b < RC; ++b) {
            const int col = col0 + tc + 16 * b;
            if (col < c) corr[voxel * ldc + col] = acc[a][b];
        }
    }
}

// corr(v, j) = sum_i K(i, j) signal(v, i) for the listed voxels: tiles of kCorrVoxels voxels x
// 16 RC columns, a CTA's tiles strided by the grid (a round whose count lives on the device is
// launched with a resident-sized grid, so an empty round costs little).
template <int RC>
__global__ void __launch_bounds__(128) correlate_kernel(SignalDev S, const int* __restrict__ list, int64_t count,
                                                        const int* __restrict__ count_dev,
                                                        const double* __restrict__ k, int c,
                                                        double* __restrict__ corr, int ldc) {
    __shared__ int64_t vox[kCorrVoxels];
    const int tid = threadIdx.x;
    if (count_dev) count = min(count, int64_t(*count_dev));
    for (int64_t p0 = int64_t(blockIdx.x) * kCorrVoxels; p0 < count; p0 += int64_t(gridDim.x) * kCorrVoxels) {
        __syncthreads();  // the previous tile's voxels are read
        if (tid < kCorrVoxels) vox[tid] = p0 + tid < count ? listed(list, p0 + tid) : -1;
        __syncthreads();
        correlate_tile<RC>(S, vox, k, c, blockIdx.y * 16 * RC, corr, ldc);
    }
}

// ---- ridge NNLS ------------------------------------------------------------------------

// A warp's NNLS workspace. Shared memory: the solution x, its candidate z, the factor's vectors
// h, w and y (InvFactor), the active and in-factor flags. Global slot: the packed factor and
// its inverse, the signal (for the QR fallback) and the QR workspace.
struct NnlsSlot {
    double *x, *z, *h, *w, *y, *L, *M, *sig, *qsub, *qd, *qrv;
    uint8_t *flag, *inf;
};

inline size_t nnls_slot_doubles(int m, int cap) {
    return 2 * size_t(packed_size(cap)) + size_t(m) + size_t(m + kQrCap) * kQrCap + 2 * size_t(m + kQrCap) + 8;
}

__host__ __device__ inline size_t nnls_smem_bytes(int c, int cap) {
    return ((2 * size_t(c) + 3 * size_t(cap)) * sizeof(double) + 2 * size_t(c) + 15) / 16 * 16;
}

__device__ NnlsSlot carve_nnls(double* base, unsigned char* smem, int m, int c, int cap) {
    NnlsSlot s;
    double* p = base;
    s.L = p; p += packed_size(cap);
    s.M = p; p += packed_size(cap);
    s.sig = p; p += m;
    s.qsub = p; p += size_t(m + kQrCap) * kQrCap;
    s.qd = p; p += m + kQrCap;
    s.qrv = p;
    double* q = reinterpret_cast<double*>(smem);
    s.x = q; q += c;
    s.z = q; q += c;
    s.h = q; q += cap;
    s.w = q; q += cap;
    s.y = q; q += cap;
    s.flag = reinterpret_cast<uint8_t*>(q);
    s.inf = s.flag + c;
    return s;
}

template <int CAP, int CMAX>
struct NnlsState {
    int cols[CAP];     // factor columns, joining order
    int sorted[CMAX];  // columns with x != 0, increasing; the columns to append again in a fit
    int qact[kQrCap];  // QR fallback active columns, increasing
    double qtau[kQrCap], qnu[kQrCap], qnd[kQrCap];
    int qperm[kQrCap];
};

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
template <class State>
__device__ __noinline__ bool ridge_qr_fit(const RidgeDev R, const double* sig, const NnlsSlot sl, State& st, int lane) {
    int k = 0;
    if (lane == 0) {
        for (int j = 0; j < R.c; ++j)
            if (sl.flag[j]) {
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
// cpp/src/sd/nnls.cpp:362-418) from corr = K^T sig, the result in sl.x. The signal itself is
// built only when a QR fit needs it. Returns false only when the QR fallback's workspace
// overflowed (x is then the last fit). VPL * 32 is the factor's capacity, CPL * 32 >= c.
//
// Inlined into its kernel with every argument by value, so that its state (the active count,
// the flags, the workspace pointers) stays in registers; the outer (entering column) and inner
// (blocking step) iterations of Lawson-Hanson share one loop with one fit, so the factor code
// is emitted once.
//
// With REDO, a fit the factor cannot take (more than VPL * 32 active columns, or a pivot below the
// relative tolerance) stops at once with *redo set, instead of continuing by QR: the caller refits
// that voxel from the start with a larger factor, which takes the same steps up to that point.
template <int VPL, int CPL, bool REDO = false, class State>
__device__ __forceinline__ bool ridge_nnls(const RidgeDev R, const SignalDev S, int64_t voxel,
                                           const double* __restrict__ corr, const NnlsSlot sl, State& st,
                                           int lane, bool* redo = nullptr) {
    const int c = R.c;
    const InvFactor fac{sl.L, sl.M, sl.h, sl.w, sl.y, st.cols, VPL * 32};
    for (int j = lane; j < c; j += 32) {
        sl.x[j] = 0.0;
        sl.z[j] = 0.0;
        sl.flag[j] = 0;
        sl.inf[j] = 0;
    }
    __syncwarp();
    const bool use_qr_only = !R.normal_equations;
    bool failed = false, overflow = false, have_sig = false;
    int na = 0, inner = 0;
    const int max_inner = 3 * c;
    bool blocked = false;  // the last fit left an active column at or below zero: an inner step
    for (;;) {
        int entering = -1;
        if (!blocked) {
            // Outer step: the gradient corr - G x over the non-zero x, columns in increasing
            // order; the steepest inactive entry, the first on a tie.
            int n_sorted = 0;
            for (int base = 0; base < c; base += 32) {
                const int j = base + lane;
                const bool nz = j < c && sl.x[j] != 0.0;
                const unsigned ballot = __ballot_sync(0xffffffffu, nz);
                if (nz) st.sorted[n_sorted + __popc(ballot & ((1u << lane) - 1u))] = j;
                n_sorted += __popc(ballot);
            }
            __syncwarp();
            double g[CPL];
#pragma unroll
            for (int t = 0; t < CPL; ++t) {
                const int j = lane + 32 * t;
                g[t] = j < c ? corr[j] : 0.0;
            }
            for (int q = 0; q < n_sorted; ++q) {
                const int col = st.sorted[q];
                const double xc = sl.x[col];
                const double* row = R.gram + size_t(col) * c;
#pragma unroll
                for (int t = 0; t < CPL; ++t) {
                    const int j = lane + 32 * t;
                    if (j < c) g[t] -= xc * row[j];
                }
            }
            double bv = 0.0;
            int bi = -1;
#pragma unroll
            for (int t = 0; t < CPL; ++t) {
                const int j = lane + 32 * t;
                if (j < c && !sl.flag[j] && (bi < 0 || g[t] > bv)) { bv = g[t]; bi = j; }
            }
            const int e = warp_argmax_first(bv, bi);
            const double ge = e >= 0 ? __shfl_sync(0xffffffffu, bv, e & 31) : 0.0;
            if (e < 0 || ge <= R.tol) break;
            if (lane == 0) sl.flag[e] = 1;
            __syncwarp();
            entering = e;
        } else {
            // Inner step: move towards the fit until the first active column reaches zero,
            // drop it and every active column below the tolerance.
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
        }
        // The fit on the active set (ActiveCholesky::update, :246-262), or QR from the first
        // failing pivot on: the columns that left the active set leave the factor (from the
        // last position down), then the entering column joins (every other active column is
        // in the factor already, so update()'s scan appends only it).
        if (!use_qr_only && !failed) {
            for (int pos = na - 1; pos >= 0; --pos) {
                const int col = st.cols[pos];
                if (sl.flag[col]) continue;
                if (VPL == 1 || na <= 32) inv_remove<1>(fac, na, pos, lane);
                else inv_remove<VPL>(fac, na, pos, lane);
                if (lane == 0) sl.inf[col] = 0;
                --na;
                __syncwarp();
            }
            if (entering >= 0) {
                for (int r = lane; r < na; r += 32) sl.h[r] = R.gram[size_t(st.cols[r]) * c + entering];
                __syncwarp();
                // Below 32 active columns one row slice per lane holds the factor's rows: the
                // one-slice code skips the unrolled empty slices of the larger capacity.
                const double gee = R.gram[size_t(entering) * c + entering];
                const bool appended =
                    (VPL == 1 || na < 32)
                        ? inv_append<1>(fac, na, gee, corr[entering], entering, kMinPivot, lane)
                        : inv_append<VPL>(fac, na, gee, corr[entering], entering, kMinPivot, lane);
                if (!appended) {
                    if constexpr (REDO) {
                        *redo = true;
                        return true;
                    }
                    failed = true;
                } else {
                    if (lane == 0) sl.inf[entering] = 1;
                    __syncwarp();
                }
            }
        }
        if (use_qr_only || failed) {
            if (!have_sig) {
                for (int i = lane; i < R.m; i += 32) sl.sig[i] = S(voxel, i);
                __syncwarp();
                have_sig = true;
            }
            overflow |= !ridge_qr_fit(R, sl.sig, sl, st, lane);
        } else if (VPL == 1 || na <= 32) {
            inv_solve<1>(fac, na, sl.z, c, lane);
        } else {
            inv_solve<VPL>(fac, na, sl.z, c, lane);
        }
        bool any = false;
        for (int j = lane; j < c; j += 32) any |= sl.flag[j] && sl.z[j] <= 0.0;
        blocked = __any_sync(0xffffffffu, any);
        if (!blocked) {
            for (int j = lane; j < c; j += 32) sl.x[j] = sl.z[j];
            __syncwarp();
        }
    }
    return !overflow;
}

// One warp per listed voxel, pulled from a device counter: x(v) <- the ridge NNLS of corr(v);
// bad(v) <- 1 when the QR fallback overflowed.
template <int VPL, int CPL>
__global__ void __launch_bounds__(kMtWarps * 32, (CPL <= 2 ? 6 : 4)) ridge_nnls_kernel(
    RidgeDev R, SignalDev S, const int* __restrict__ list, int64_t count, const int* __restrict__ count_dev,
    const double* __restrict__ corr, int ldc, double* __restrict__ x_out, int ldx, uint8_t* __restrict__ bad,
    int* queue, double* __restrict__ workspace, size_t slot_size) {
    using State = NnlsState<VPL * 32, CPL * 32>;
    if (count_dev) count = min(count, int64_t(*count_dev));
    __shared__ State states[kMtWarps];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    State& st = states[warp];
    NnlsSlot sl = carve_nnls(workspace + (size_t(blockIdx.x) * kMtWarps + warp) * slot_size,
                             smem_raw + warp * nnls_smem_bytes(R.c, VPL * 32), R.m, R.c, VPL * 32);
    for (;;) {
        int64_t p = 0;
        if (lane == 0) p = atomicAdd(queue, 1);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= count) break;
        const int64_t voxel = listed(list, p);
        const bool ok = ridge_nnls<VPL, CPL>(R, S, voxel, corr + voxel * ldc, sl, st, lane);
        for (int j = lane; j < R.c; j += 32) x_out[voxel * ldx + j] = sl.x[j];
        if (lane == 0 && !ok && bad) bad[voxel] = 1;
        __syncwarp();
    }
}

// The first pass of the high-resolution NNLS: one warp per voxel with a factor of VPL * 32 columns
// (the active sets of the 300-direction FODs stay below 32; a larger factor takes more shared
// memory and registers and fewer warps per SM); a voxel whose fit outgrows it, or needs the QR
// fallback, goes on `redo` for ridge_nnls_kernel with the full factor, which fits it from the
// start. Below the capacity the two take the same steps with the same factor code, so every
// voxel gets the result the full-factor kernel gives.
template <int VPL, int CPL>
__global__ void __launch_bounds__(kMtWarps * 32, 4) ridge_nnls_first_kernel(
    RidgeDev R, SignalDev S, int64_t count, const double* __restrict__ corr, int ldc, double* __restrict__ x_out,
    int ldx, int* __restrict__ redo, int* redo_count, int* queue, double* __restrict__ workspace, size_t slot_size) {
    using State = NnlsState<VPL * 32, CPL * 32>;
    __shared__ State states[kMtWarps];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    State& st = states[warp];
    NnlsSlot sl = carve_nnls(workspace + (size_t(blockIdx.x) * kMtWarps + warp) * slot_size,
                             smem_raw + warp * nnls_smem_bytes(R.c, VPL * 32), R.m, R.c, VPL * 32);
    for (;;) {
        int64_t voxel = 0;
        if (lane == 0) voxel = atomicAdd(queue, 1);
        voxel = __shfl_sync(0xffffffffu, voxel, 0);
        if (voxel >= count) break;
        bool again = false;
        ridge_nnls<VPL, CPL, true>(R, S, voxel, corr + voxel * ldc, sl, st, lane, &again);
        if (again) {
            if (lane == 0) redo[atomicAdd(redo_count, 1)] = int(voxel);
        } else {
            for (int j = lane; j < R.c; j += 32) x_out[voxel * ldx + j] = sl.x[j];
        }
        __syncwarp();
    }
}

// ---- ridge NNLS, two voxels per warp (at most 48 directions) ---------------------------------

// A half-warp's workspace: x, z (c each), the factor's vectors h, w, y (32 each) and the two
// flag arrays in shared memory; the factor and its inverse (32 columns) in its global slot.
struct HalfSlot {
    double *x, *z, *h, *w, *y, *L, *M;
    uint8_t *flag, *inf;
};

inline size_t half_slot_doubles() { return 2 * size_t(packed_size(2 * kHalf)) + 8; }

__host__ __device__ inline size_t half_smem_bytes(int c) {
    return ((2 * size_t(c) + 3 * 2 * kHalf) * sizeof(double) + 2 * size_t(c) + 15) / 16 * 16;
}

__device__ HalfSlot carve_half(double* base, unsigned char* smem, int c) {
    HalfSlot s;
    s.L = base;
    s.M = base + packed_size(2 * kHalf);
    double* q = reinterpret_cast<double*>(smem);
    s.x = q; q += c;
    s.z = q; q += c;
    s.h = q; q += 2 * kHalf;
    s.w = q; q += 2 * kHalf;
    s.y = q; q += 2 * kHalf;
    s.flag = reinterpret_cast<uint8_t*>(q);
    s.inf = s.flag + c;
    return s;
}

template <int CPL>
struct HalfState {
    int cols[2 * kHalf];      // factor columns, joining order
    int sorted[kHalf * CPL];  // columns with x != 0, increasing
};

// ridge_nnls for one voxel on a half-warp (see group_nnls.cuh): the same steps, rules and
// tolerances. False when the voxel needs the QR fallback (a pivot below the tolerance or more
// than 32 active columns); the caller then hands it to the one-warp kernel.
template <int CPL>
__device__ __forceinline__ bool ridge_nnls_half(const RidgeDev R, const double* __restrict__ corr, const HalfSlot sl,
                                                HalfState<CPL>& st, const HalfWarp hw) {
    const int c = R.c;
    const InvFactor fac{sl.L, sl.M, sl.h, sl.w, sl.y, st.cols, 2 * kHalf};
    for (int j = hw.lane; j < c; j += kHalf) {
        sl.x[j] = 0.0;
        sl.z[j] = 0.0;
        sl.flag[j] = 0;
        sl.inf[j] = 0;
    }
    hw.sync();
    int na = 0, inner = 0;
    const int max_inner = 3 * c;
    bool blocked = false;
    for (;;) {
        int entering = -1;
        if (!blocked) {
            int n_sorted = 0;
            for (int base = 0; base < c; base += kHalf) {
                const int j = base + hw.lane;
                const bool nz = j < c && sl.x[j] != 0.0;
                const unsigned ballot = hw.ballot(nz);
                if (nz) st.sorted[n_sorted + __popc(ballot & ((1u << hw.lane) - 1u))] = j;
                n_sorted += __popc(ballot);
            }
            hw.sync();
            double g[CPL];
#pragma unroll
            for (int t = 0; t < CPL; ++t) {
                const int j = hw.lane + kHalf * t;
                g[t] = j < c ? corr[j] : 0.0;
            }
            for (int q = 0; q < n_sorted; ++q) {
                const int col = st.sorted[q];
                const double xc = sl.x[col];
                const double* row = R.gram + size_t(col) * c;
#pragma unroll
                for (int t = 0; t < CPL; ++t) {
                    const int j = hw.lane + kHalf * t;
                    if (j < c) g[t] -= xc * row[j];
                }
            }
            double bv = 0.0;
            int bi = -1;
#pragma unroll
            for (int t = 0; t < CPL; ++t) {
                const int j = hw.lane + kHalf * t;
                if (j < c && !sl.flag[j] && (bi < 0 || g[t] > bv)) { bv = g[t]; bi = j; }
            }
            const int e = hw.argmax_first(bv, bi);
            const double ge = e >= 0 ? hw.from(bv, e & (kHalf - 1)) : 0.0;
            if (e < 0 || ge <= R.tol) break;
            if (hw.lane == 0) sl.flag[e] = 1;
            hw.sync();
            entering = e;
        } else {
            if (++inner > max_inner) {
                for (int j = hw.lane; j < c; j += kHalf) sl.x[j] = sl.z[j];
                hw.sync();
                return true;
            }
            double sv = 0.0;
            int si = -1;
            for (int j = hw.lane; j < c; j += kHalf) {
                if (!sl.flag[j] || sl.z[j] > 0.0) continue;
                const double dist = sl.x[j] - sl.z[j];
                const double stp = dist > 0.0 ? sl.x[j] / dist : 0.0;
                if (si < 0 || stp < sv) { sv = stp; si = j; }
            }
            double step;
            const int b = hw.argmin_first(sv, si, &step);
            for (int j = hw.lane; j < c; j += kHalf) sl.x[j] += step * (sl.z[j] - sl.x[j]);
            hw.sync();
            if (hw.lane == 0) {
                sl.x[b] = 0.0;
                sl.flag[b] = 0;
            }
            hw.sync();
            for (int j = hw.lane; j < c; j += kHalf)
                if (sl.flag[j] && !(fabs(sl.x[j]) >= R.tol)) sl.flag[j] = 0;
            hw.sync();
        }
        for (int pos = na - 1; pos >= 0; --pos) {
            const int col = st.cols[pos];
            if (sl.flag[col]) continue;
            half_remove(fac, na, pos, hw);
            if (hw.lane == 0) sl.inf[col] = 0;
            --na;
            hw.sync();
        }
        if (entering >= 0) {
            if (na >= 2 * kHalf) return false;
            for (int r = hw.lane; r < na; r += kHalf) sl.h[r] = R.gram[size_t(st.cols[r]) * c + entering];
            hw.sync();
            if (!half_append(fac, na, R.gram[size_t(entering) * c + entering], corr[entering], entering, kMinPivot,
                             hw))
                return false;
            if (hw.lane == 0) sl.inf[entering] = 1;
            hw.sync();
        }
        half_solve(fac, na, sl.z, c, hw);
        bool any = false;
        for (int j = hw.lane; j < c; j += kHalf) any |= sl.flag[j] && sl.z[j] <= 0.0;
        blocked = hw.any(any);
        if (!blocked) {
            for (int j = hw.lane; j < c; j += kHalf) sl.x[j] = sl.z[j];
            hw.sync();
        }
    }
    return true;
}

// Two listed voxels per warp, one per half, pulled from a device counter: x(v) <- the ridge
// NNLS of corr(v), or v appended to `redo` when it needs the QR fallback.
template <int CPL>
__global__ void __launch_bounds__(kMtWarps * 32, 8) ridge_nnls_half_kernel(
    RidgeDev R, const int* __restrict__ list, int64_t count, const int* __restrict__ count_dev,
    const double* __restrict__ corr, int ldc, double* __restrict__ x_out, int ldx, int* __restrict__ redo,
    int* redo_count, int* queue, double* __restrict__ workspace, size_t slot_size) {
    if (count_dev) count = min(count, int64_t(*count_dev));
    __shared__ HalfState<CPL> states[2 * kMtWarps];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const HalfWarp hw(threadIdx.x & 31);
    const int gid = int(threadIdx.x >> 4);  // half-warp within the CTA
    HalfState<CPL>& st = states[gid];
    const HalfSlot sl = carve_half(workspace + (size_t(blockIdx.x) * 2 * kMtWarps + gid) * slot_size,
                                   smem_raw + gid * half_smem_bytes(R.c), R.c);
    for (;;) {
        long long p = 0;
        if (hw.lane == 0) p = atomicAdd(queue, 1);
        p = hw.from(p, 0);
        if (p >= count) break;
        const int64_t voxel = listed(list, p);
        const bool done = ridge_nnls_half<CPL>(R, corr + voxel * ldc, sl, st, hw);
        if (done) {
            for (int j = hw.lane; j < R.c; j += kHalf) x_out[voxel * ldx + j] = sl.x[j];
        } else if (hw.lane == 0) {
            redo[atomicAdd(redo_count, 1)] = int(voxel);
        }
        hw.sync();
    }
}

// ---- fractions -------------------------------------------------------------------------

// A warp's fraction workspace in its global slot: the thresholded FOD, the fraction columns
// (row-major) and the NNLS / QR workspace.
struct FracSlot {
    double *th, *cols, *fu, *fz, *fsub, *frv, *res;
    uint8_t* fflag;
};

inline size_t frac_slot_doubles(int m, int ca, int ng) {
    return size_t(ca) + size_t(m) * ng + 2 * size_t(ng) + size_t(ng) * m + 2 * size_t(m) + (size_t(ng) + 7) / 8 + 8;
}

__device__ FracSlot carve_frac(double* base, int m, int ca, int ng) {
    FracSlot s;
    double* p = base;
    s.th = p; p += ca;
    s.cols = p; p += size_t(m) * ng;
    s.fu = p; p += ng;
    s.fz = p; p += ng;
    s.fsub = p; p += size_t(ng) * m;
    s.frv = p; p += m;
    s.res = p; p += m;
    s.fflag = reinterpret_cast<uint8_t*>(p);
    return s;
}

struct FracState {
    int fact[kMaxGroups], fn_act;
    double ftau[kMaxGroups], fnu[kMaxGroups], fnd[kMaxGroups];
    int fperm[kMaxGroups];
    double fr[kMaxGroups];
    double med[2];
};

// Median of v[0..n), the mean of the two middle values for even n (cpp/src/sd/fractions.cpp:56-68),
// by ranks: the element of stable rank r is the r-th smallest.
__device__ __forceinline__ double warp_median(const double* v, int n, FracState& st, int lane) {
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

constexpr int kFastRowsPerLane = 10;  // measurements per lane of the register fraction fit (m <= 320)

// Lawson-Hanson (cpp/src/sd/nnls.cpp:187-221) on the normal equations G u = b of at most four
// columns, every lane running the same scalar steps: the gradient b - G u over the active
// columns, the steepest inactive column (the first on a tie), the least-squares fit of the
// active block by Cholesky, the blocking step and the drops below tol, at most max_inner inner
// steps. Inactive rows of the active block's system are the identity, so each solve runs on
// compile-time indices. False when a pivot is not positive (the caller then fits by QR).
__device__ __forceinline__ bool small_nnls(const double (&G)[4][4], const double (&b)[4], int n, double tol,
                                           int max_inner, double (&u)[4]) {
    bool flag[4];
    double z[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        flag[j] = false;
        u[j] = 0.0;
        z[j] = 0.0;
    }
    auto solve = [&]() -> bool {
        double L[4][4], y[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
#pragma unroll
            for (int c = 0; c <= a; ++c) {
                double sum = flag[a] && flag[c] ? G[a][c] : (a == c ? 1.0 : 0.0);
#pragma unroll
                for (int k = 0; k < c; ++k) sum -= L[a][k] * L[c][k];
                if (a == c) {
                    if (!(sum > 0.0)) return false;
                    L[a][a] = sqrt(sum);
                } else {
                    L[a][c] = sum / L[c][c];
                }
            }
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            double sum = flag[a] ? b[a] : 0.0;
#pragma unroll
            for (int k = 0; k < a; ++k) sum -= L[a][k] * y[k];
            y[a] = sum / L[a][a];
        }
#pragma unroll
        for (int a = 3; a >= 0; --a) {
            double sum = y[a];
#pragma unroll
            for (int k = a + 1; k < 4; ++k) sum -= L[k][a] * z[k];
            z[a] = flag[a] ? sum / L[a][a] : 0.0;
        }
        return true;
    };
    int inner = 0;
    for (;;) {
        int e = -1;
        double best = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (j >= n) continue;
            double w = b[j];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (flag[q]) w -= G[j][q] * u[q];
            if (!flag[j] && (e < 0 || w > best)) {
                best = w;
                e = j;
            }
        }
        if (e < 0 || best <= tol) return true;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (j == e) flag[j] = true;
        if (!solve()) return false;
        for (;;) {
            bool any = false;
#pragma unroll
            for (int j = 0; j < 4; ++j) any |= flag[j] && z[j] <= 0.0;
            if (!any) break;
            if (++inner > max_inner) {
#pragma unroll
                for (int j = 0; j < 4; ++j) u[j] = flag[j] ? z[j] : 0.0;
                return true;
            }
            double sv = 0.0;
            int si = -1;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (!flag[j] || z[j] > 0.0) continue;
                const double dist = u[j] - z[j];
                const double stp = dist > 0.0 ? u[j] / dist : 0.0;
                if (si < 0 || stp < sv) {
                    sv = stp;
                    si = j;
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double zj = flag[j] ? z[j] : 0.0;
                u[j] += sv * (zj - u[j]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (j == si) u[j] = 0.0;
                if (flag[j] && (j == si || !(fabs(u[j]) >= tol))) flag[j] = false;
            }
            if (!solve()) return false;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) u[j] = flag[j] ? z[j] : 0.0;
    }
}

// compute_fractions for one anisotropic column next to at most three isotropic ones and at most
// 320 measurements: the column K th scaled to a maximum of 1 in registers, then C^T C, C^T s and
// the columns' norm1 in one reduction, and the NNLS on those (small_nnls). False when that
// needs the QR fit.
__device__ __forceinline__ bool fractions_small(const TissueDev T, const double* sig, int gb, int ge, double tol,
                                                const FracSlot sl, FracState& st, int lane) {
    const int m = T.m, ci = T.ci, n = 1 + ci;
    double col[kFastRowsPerLane];
#pragma unroll
    for (int t = 0; t < kFastRowsPerLane; ++t) col[t] = 0.0;
    for (int j = gb; j < ge; ++j) {
        const double tj = sl.th[j];
        if (tj == 0.0) continue;
        const double* kr = T.kt + size_t(j) * m;
#pragma unroll
        for (int t = 0; t < kFastRowsPerLane; ++t) {
            const int i = lane + 32 * t;
            if (i < m) col[t] += kr[i] * tj;
        }
    }
    double largest = -INFINITY;
    bool any = false;
#pragma unroll
    for (int t = 0; t < kFastRowsPerLane; ++t) {
        const int i = lane + 32 * t;
        if (i < m && !isnan(col[t])) {
            largest = any ? fmax(largest, col[t]) : col[t];
            any = true;
        }
    }
    // The largest non-NaN value over the lanes (Eigen's maxCoeff<PropagateNumbers>).
    largest = warp_max(any ? largest : -INFINITY);
    const bool all_nan = !__any_sync(0xffffffffu, any);
    if (!all_nan && largest > 0.0) {
#pragma unroll
        for (int t = 0; t < kFastRowsPerLane; ++t) col[t] /= largest;
    }
    // Partial sums: G (upper triangle, 10), C^T s (4), norm1 (4).
    double part[18];
#pragma unroll
    for (int k = 0; k < 18; ++k) part[k] = 0.0;
#pragma unroll
    for (int t = 0; t < kFastRowsPerLane; ++t) {
        const int i = lane + 32 * t;
        if (i >= m) continue;
        double v[4];
        v[0] = col[t];
#pragma unroll
        for (int q = 1; q < 4; ++q) v[q] = q <= ci ? T.iso[size_t(i) * ci + q - 1] : 0.0;
        const double si = sig[i];
        int k = 0;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int c = a; c < 4; ++c) part[k++] += v[a] * v[c];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            part[10 + a] += v[a] * si;
            part[14 + a] += fabs(v[a]);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 18; ++k) part[k] += __shfl_xor_sync(0xffffffffu, part[k], off);
    double G[4][4], b[4], u[4];
    {
        int k = 0;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int c = a; c < 4; ++c) {
                G[a][c] = part[k];
                G[c][a] = part[k];
                ++k;
            }
    }
    double colmax = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        b[a] = part[10 + a];
        if (a < n) colmax = fmax(colmax, part[14 + a]);
    }
    if (tol < 0.0) tol = 10.0 * kEps64 * colmax * double(max(m, n));
    if (!small_nnls(G, b, n, tol, 3 * n, u)) return false;
    if (lane < n) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (q == lane) st.fr[q] = u[q];
    }
    __syncwarp();
    return true;
}

// compute_fractions (cpp/src/sd/fractions.cpp:70-101): tol < 0 uses the default tolerance of the
// fraction columns. Writes the fractions (groups, then isotropic tissues) to st.fr. One
// anisotropic group, at most three isotropic tissues and at most 320 measurements take the
// register fit (fractions_small); otherwise, or when its normal equations are not positive
// definite, the columns are built in the warp's slot and fitted by QR.
__device__ __forceinline__ void fractions(const TissueDev T, const double* fod, const double* sig, bool per_block,
                                          double tol, const FracSlot sl, FracState& st, int lane) {
    const int m = T.m, ca = T.ca, ci = T.ci;
    const double threshold = warp_median(fod, ca, st, lane) * (1.0 - kMedianTie);
    for (int j = lane; j < ca; j += 32) sl.th[j] = fod[j] < threshold ? 0.0 : fod[j];
    __syncwarp();
    const int ng = per_block ? T.nb : 1;
    const int ncol = ng + ci;
    if (ng == 1 && ci <= 3 && m <= 32 * kFastRowsPerLane) {
        const int gb = per_block ? T.blocks[0] : 0, ge = per_block ? T.blocks[1] : ca;
        if (fractions_small(T, sig, gb, ge, tol, sl, st, lane)) return;
    }
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
    NnlsScratch ns{sl.fu, sl.fz, sl.fflag, st.fact, &st.fn_act, sl.res,
                   QrScratch{sl.fsub, st.ftau, st.fnu, st.fnd, st.fperm, sl.frv}, kMaxGroups};
    warp_nnls_explicit(sl.cols, m, ncol, sig, tol, 3 * ncol, ns, lane);
    for (int g = lane; g < ncol; g += 32) st.fr[g] = sl.fu[g];
    __syncwarp();
}

// One round's fractions of the listed voxels (cpp/src/sd/multi_tissue.cpp:100-125): f_iso(v)
// takes the isotropic fractions; a voxel whose fractions all moved by less than fraction_tol, or
// that used its last round, records its round count, the others join the next round's list
// with their fractions kept for the next comparison.
__global__ void __launch_bounds__(kMtWarps * 32, 5) lr_fractions_kernel(
    TissueDev T, const double* __restrict__ signals, const double* __restrict__ fods, int ldf,
    const int* __restrict__ list, int64_t count, const int* __restrict__ count_dev, int round, int max_rounds,
    double fraction_tol, double* __restrict__ fiso, double* __restrict__ prev, int32_t* __restrict__ rounds,
    int* __restrict__ next, int* next_count, int* queue, double* __restrict__ workspace, size_t slot_size) {
    if (count_dev) count = min(count, int64_t(*count_dev));
    __shared__ FracState states[kMtWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    FracState& st = states[warp];
    FracSlot sl = carve_frac(workspace + (size_t(blockIdx.x) * kMtWarps + warp) * slot_size, T.m, T.ca, 1 + T.ci);
    const int ci = T.ci;
    for (;;) {
        int64_t p = 0;
        if (lane == 0) p = atomicAdd(queue, 1);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= count) break;
        const int64_t voxel = listed(list, p);
        fractions(T, fods + voxel * ldf, signals + voxel * T.m, false, -1.0, sl, st, lane);
        // The first round has nothing to compare with (its previous fractions are infinite).
        bool converged = round > 0;
        for (int j = 0; j <= ci; ++j) converged &= fabs(st.fr[j] - prev[voxel * (ci + 1) + j]) < fraction_tol;
        __syncwarp();
        if (lane < ci) fiso[voxel * ci + lane] = st.fr[1 + lane];
        if (converged || round + 1 >= max_rounds) {
            if (lane == 0) rounds[voxel] = round + 1;
        } else {
            if (lane <= ci) prev[voxel * (ci + 1) + lane] = st.fr[lane];
            if (lane == 0) next[atomicAdd(next_count, 1)] = int(voxel);
        }
        __syncwarp();
    }
}

// The final per-block fractions of every voxel, normalised to sum to 1 (+1e-16), with the round
// counts and statuses (cpp/src/sd/multi_tissue.cpp:127-148).
__global__ void __launch_bounds__(kMtWarps * 32, 5) hr_fractions_kernel(
    TissueDev T, const double* __restrict__ signals, const double* __restrict__ fods, int64_t count,
    double final_tol, const int32_t* __restrict__ rounds_in, const uint8_t* __restrict__ bad,
    double* __restrict__ fractions_out, int32_t* __restrict__ rounds_out, uint8_t* __restrict__ status, int* queue,
    double* __restrict__ workspace, size_t slot_size) {
    __shared__ FracState states[kMtWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    FracState& st = states[warp];
    FracSlot sl = carve_frac(workspace + (size_t(blockIdx.x) * kMtWarps + warp) * slot_size, T.m, T.ca,
                             T.nb + T.ci);
    const int nf = T.nb + T.ci;
    for (;;) {
        int64_t voxel = 0;
        if (lane == 0) voxel = atomicAdd(queue, 1);
        voxel = __shfl_sync(0xffffffffu, voxel, 0);
        if (voxel >= count) break;
        fractions(T, fods + voxel * T.ca, signals + voxel * T.m, true, final_tol, sl, st, lane);
        double total = kFractionSumOffset;
        for (int g = 0; g < nf; ++g) total += st.fr[g];
        for (int g = lane; g < nf; g += 32) fractions_out[voxel * nf + g] = st.fr[g] / total;
        if (lane == 0) {
            if (rounds_out) rounds_out[voxel] = rounds_in[voxel];
            if (status) status[voxel] = bad[voxel];
        }
        __syncwarp();
    }
}

// ---- batches (batch.cuh): every mFOD volume of a batch through one queue per stage ------------

// A volume of a batch: its solvers and kernels, signals, shell weights and outputs.
struct MfodBatchJob {
    int64_t v, off;  // voxels; the row of its first voxel in the batch's per-voxel state
    RidgeDev lr, hr;
    TissueDev lrt, hrt;
    const double* s;   // (v, m) S0-normalised signals
    const double* w;   // (m,) shell weights
    double* fods;      // (v, hr.c)
    double* fractions; // (v, hrt.nb + hrt.ci)
    int32_t* rounds;   // (v,) or null
    uint8_t* status;   // (v,) or null
};

// The per-voxel state of a batch (volume j's voxel v at row off_j + v) and the stage's tickets.
struct MfodBatchState {
    const MfodBatchJob* jobs;
    int n_jobs, ci, ldc, ldx;  // isotropic tissues; row strides of corr and of the low-resolution FODs
    double *fiso, *prev, *corr, *xlr;
    int32_t* rounds;
    uint8_t* bad;
    int64_t* vfirst;   // (n_jobs + 1) this stage's first voxel ticket per volume
    int64_t* tfirst;   // (n_jobs + 1) its first correlation tile per volume
    int64_t* redo;     // volume << 32 | voxel, for the one-warp NNLS
    int* redo_count;
};

// A round's lists are per-volume segments of one array (volume j's at row off_j), null for
// every voxel of every volume.
struct BatchItem {
    int job;
    int64_t voxel;
};

__device__ __forceinline__ BatchItem batch_item(const MfodBatchState& B, const int* list, int64_t p) {
    const int j = ticket_job(B.vfirst, B.n_jobs, p);
    const int64_t q = p - B.vfirst[j];
    return BatchItem{j, list ? int64_t(list[B.jobs[j].off + q]) : q};
}

__device__ __forceinline__ SignalDev batch_signal(const MfodBatchState& B, const MfodBatchJob& J, const TissueDev& T) {
    return SignalDev{J.s, J.w, T.wiso, B.fiso + J.off * B.ci, T.m, B.ci};
}

// The tickets of a stage from each volume's count (null: every voxel).
__global__ void batch_plan_kernel(MfodBatchState B, const int* __restrict__ counts) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int64_t a = 0, b = 0;
    for (int j = 0; j < B.n_jobs; ++j) {
        B.vfirst[j] = a;
        B.tfirst[j] = b;
        const int64_t c = counts ? int64_t(counts[j]) : B.jobs[j].v;
        a += c;
        b += (c + kCorrVoxels - 1) / kCorrVoxels;
    }
    B.vfirst[B.n_jobs] = a;
    B.tfirst[B.n_jobs] = b;
}

// correlate_kernel over every volume: a CTA per (volume, tile of kCorrVoxels listed voxels).
template <int RC, bool HR>
__global__ void __launch_bounds__(128) batch_correlate_kernel(MfodBatchState B, const int* __restrict__ list) {
    __shared__ int64_t vox[kCorrVoxels];
    const int tid = threadIdx.x;
    const int64_t total = B.tfirst[B.n_jobs];
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
        const int j = ticket_job(B.tfirst, B.n_jobs, t);
        const MfodBatchJob& J = B.jobs[j];
        const int64_t count = B.vfirst[j + 1] - B.vfirst[j];
        const int64_t p0 = (t - B.tfirst[j]) * kCorrVoxels;
        __syncthreads();  // the previous tile's voxels are read
        if (tid < kCorrVoxels) {
            const int64_t q = p0 + tid;
            vox[tid] = q < count ? (list ? int64_t(list[J.off + q]) : q) : -1;
        }
        __syncthreads();
        const RidgeDev R = HR ? J.hr : J.lr;
        const TissueDev T = HR ? J.hrt : J.lrt;
        correlate_tile<RC>(batch_signal(B, J, T), vox, R.k, R.c, blockIdx.y * 16 * RC, B.corr + J.off * B.ldc,
                           B.ldc);
    }
}

// ridge_nnls_half_kernel over every volume's list.
template <int CPL>
__global__ void __launch_bounds__(kMtWarps * 32, 8) batch_half_kernel(MfodBatchState B, const int* __restrict__ list,
                                                                     int c_max, int* queue,
                                                                     double* __restrict__ workspace,
                                                                     size_t slot_size) {
    __shared__ HalfState<CPL> states[2 * kMtWarps];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const HalfWarp hw(threadIdx.x & 31);
    const int gid = int(threadIdx.x >> 4);
    HalfState<CPL>& st = states[gid];
    const HalfSlot sl = carve_half(workspace + (size_t(blockIdx.x) * 2 * kMtWarps + gid) * slot_size,
                                   smem_raw + gid * half_smem_bytes(c_max), c_max);
    const int64_t total = B.vfirst[B.n_jobs];
    for (;;) {
        long long p = 0;
        if (hw.lane == 0) p = atomicAdd(queue, 1);
        p = hw.from(p, 0);
        if (p >= total) break;
        const BatchItem it = batch_item(B, list, p);
        const MfodBatchJob& J = B.jobs[it.job];
        const RidgeDev R = J.lr;
        const int64_t row = J.off + it.voxel;
        if (ridge_nnls_half<CPL>(R, B.corr + row * B.ldc, sl, st, hw)) {
            for (int j = hw.lane; j < R.c; j += kHalf) B.xlr[row * B.ldx + j] = sl.x[j];
        } else if (hw.lane == 0) {
            B.redo[atomicAdd(B.redo_count, 1)] = (int64_t(it.job) << 32) | it.voxel;
        }
        hw.sync();
    }
}

// ridge_nnls_kernel over the voxels the first passes handed back, from every volume.
template <int VPL, int CPL, bool HR>
__global__ void __launch_bounds__(kMtWarps * 32, (CPL <= 2 ? 6 : 4)) batch_redo_kernel(
    MfodBatchState B, int c_max, int* queue, double* __restrict__ workspace, size_t slot_size) {
    using State = NnlsState<VPL * 32, CPL * 32>;
    __shared__ State states[kMtWarps];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    State& st = states[warp];
    double* slot = workspace + (size_t(blockIdx.x) * kMtWarps + warp) * slot_size;
    unsigned char* wsm = smem_raw + warp * nnls_smem_bytes(c_max, VPL * 32);
    const int total = *B.redo_count;
    for (;;) {
        int p = 0;
        if (lane == 0) p = atomicAdd(queue, 1);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= total) break;
        const int64_t e = B.redo[p];
        const MfodBatchJob& J = B.jobs[int(e >> 32)];
        const int64_t voxel = e & 0xffffffffll;
        const RidgeDev R = HR ? J.hr : J.lr;
        const TissueDev T = HR ? J.hrt : J.lrt;
        NnlsSlot sl = carve_nnls(slot, wsm, R.m, R.c, VPL * 32);
        const int64_t row = J.off + voxel;
        const bool ok = ridge_nnls<VPL, CPL>(R, batch_signal(B, J, T), voxel, B.corr + row * B.ldc, sl, st, lane);
        double* x = HR ? J.fods + voxel * R.c : B.xlr + row * B.ldx;
        for (int j = lane; j < R.c; j += 32) x[j] = sl.x[j];
        if (lane == 0 && !ok) B.bad[row] = 1;
        __syncwarp();
    }
}

// ridge_nnls_first_kernel<1, 10> over every voxel of every volume.
__global__ void __launch_bounds__(kMtWarps * 32, 5) batch_first_kernel(MfodBatchState B, int c_max, int* queue,
                                                                      double* __restrict__ workspace,
                                                                      size_t slot_size) {
    using State = NnlsState<32, 10 * 32>;
    __shared__ State states[kMtWarps];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    State& st = states[warp];
    double* slot = workspace + (size_t(blockIdx.x) * kMtWarps + warp) * slot_size;
    unsigned char* wsm = smem_raw + warp * nnls_smem_bytes(c_max, 32);
    const int64_t total = B.vfirst[B.n_jobs];
    for (;;) {
        long long p = 0;
        if (lane == 0) p = atomicAdd(queue, 1);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= total) break;
        const BatchItem it = batch_item(B, nullptr, p);
        const MfodBatchJob& J = B.jobs[it.job];
        const RidgeDev R = J.hr;
        NnlsSlot sl = carve_nnls(slot, wsm, R.m, R.c, 32);
        const int64_t row = J.off + it.voxel;
        bool again = false;
        ridge_nnls<1, 10, true>(R, batch_signal(B, J, J.hrt), it.voxel, B.corr + row * B.ldc, sl, st, lane, &again);
        if (again) {
            if (lane == 0) B.redo[atomicAdd(B.redo_count, 1)] = (int64_t(it.job) << 32) | it.voxel;
        } else {
            for (int j = lane; j < R.c; j += 32) J.fods[it.voxel * R.c + j] = sl.x[j];
        }
        __syncwarp();
    }
}

// lr_fractions_kernel over every volume's list; the next round's list goes to each volume's
// segment.
__global__ void __launch_bounds__(kMtWarps * 32, 4) batch_lr_fractions_kernel(
    MfodBatchState B, const int* __restrict__ list, int round, int max_rounds, double fraction_tol,
    int* __restrict__ next, int* next_counts, int* queue, double* __restrict__ workspace, size_t slot_size) {
    __shared__ FracState states[kMtWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    FracState& st = states[warp];
    double* slot = workspace + (size_t(blockIdx.x) * kMtWarps + warp) * slot_size;
    const int ci = B.ci;
    const int64_t total = B.vfirst[B.n_jobs];
    for (;;) {
        long long p = 0;
        if (lane == 0) p = atomicAdd(queue, 1);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= total) break;
        const BatchItem it = batch_item(B, list, p);
        const MfodBatchJob& J = B.jobs[it.job];
        const TissueDev T = J.lrt;
        const FracSlot sl = carve_frac(slot, T.m, T.ca, 1 + T.ci);
        const int64_t row = J.off + it.voxel;
        fractions(T, B.xlr + row * B.ldx, J.s + it.voxel * T.m, false, -1.0, sl, st, lane);
        bool converged = round > 0;
        for (int j = 0; j <= ci; ++j) converged &= fabs(st.fr[j] - B.prev[row * (ci + 1) + j]) < fraction_tol;
        __syncwarp();
        if (lane < ci) B.fiso[row * ci + lane] = st.fr[1 + lane];
        if (converged || round + 1 >= max_rounds) {
            if (lane == 0) B.rounds[row] = round + 1;
        } else {
            if (lane <= ci) B.prev[row * (ci + 1) + lane] = st.fr[lane];
            if (lane == 0) next[J.off + atomicAdd(next_counts + it.job, 1)] = int(it.voxel);
        }
        __syncwarp();
    }
}

// hr_fractions_kernel over every voxel of every volume.
__global__ void __launch_bounds__(kMtWarps * 32, 4) batch_hr_fractions_kernel(MfodBatchState B, double final_tol,
                                                                             int* queue,
                                                                             double* __restrict__ workspace,
                                                                             size_t slot_size) {
    __shared__ FracState states[kMtWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    FracState& st = states[warp];
    double* slot = workspace + (size_t(blockIdx.x) * kMtWarps + warp) * slot_size;
    const int64_t total = B.vfirst[B.n_jobs];
    for (;;) {
        long long p = 0;
        if (lane == 0) p = atomicAdd(queue, 1);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= total) break;
        const BatchItem it = batch_item(B, nullptr, p);
        const MfodBatchJob& J = B.jobs[it.job];
        const TissueDev T = J.hrt;
        const int nf = T.nb + T.ci;
        const FracSlot sl = carve_frac(slot, T.m, T.ca, nf);
        const int64_t row = J.off + it.voxel;
        fractions(T, J.fods + it.voxel * T.ca, J.s + it.voxel * T.m, true, final_tol, sl, st, lane);
        double sum = kFractionSumOffset;
        for (int g = 0; g < nf; ++g) sum += st.fr[g];
        for (int g = lane; g < nf; g += 32) J.fractions[it.voxel * nf + g] = st.fr[g] / sum;
        if (lane == 0) {
            if (J.rounds) J.rounds[it.voxel] = B.rounds[row];
            if (J.status) J.status[it.voxel] = B.bad[row];
        }
        __syncwarp();
    }
}

// ---- host side -------------------------------------------------------------------------

// The warps of a persistent grid: as many as the SMs hold at once (or one per item), in whole
// CTAs of kMtWarps.
template <class Kernel>
int64_t resident_slots(Kernel kernel, size_t smem, int64_t items, const char* setting) {
    require(smem <= 200 * 1024, "the kernel has too many columns for the shared-memory solver");
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "cudaFuncSetAttribute");
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kMtWarps * 32, smem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((items + kMtWarps - 1) / kMtWarps,
                                                                  int64_t(sm_count()) * ctas_per_sm(per_sm, setting)));
    return blocks * kMtWarps;
}

// A bump allocator over one device buffer, 256-byte aligned pieces.
struct Carver {
    char* base;
    size_t used = 0;
    template <class T>
    T* take(size_t n) {
        T* p = reinterpret_cast<T*>(base ? base + used : nullptr);
        used += (n * sizeof(T) + 255) / 256 * 256;
        return p;
    }
};

// Launches the ridge NNLS of `count` listed voxels on the instantiation that fits the solver.
struct NnlsLaunch {
    void (*kernel)(RidgeDev, SignalDev, const int*, int64_t, const int*, const double*, int, double*, int, uint8_t*,
                   int*, double*, size_t);
    int cap;
    const char* name;
};

inline NnlsLaunch nnls_variant(int c) {
    // Up to 64 directions (the low-resolution kernels): a 32-column factor, the active sets
    // being far smaller (past 32 active columns the fit continues by QR).
    if (c <= 64) return {ridge_nnls_kernel<1, 2>, 32, "ridge_nnls_kernel<1,2>"};
    if (c <= 320) return {ridge_nnls_kernel<kCholCap / 32, 10>, kCholCap, "ridge_nnls_kernel<8,10>"};
    return {ridge_nnls_kernel<kCholCap / 32, kMaxColumns / 32>, kCholCap, "ridge_nnls_kernel<8,20>"};
}

inline void launch_correlate(const SignalDev& S, const int* list, int64_t count, const int* count_dev,
                             const RidgeDev& R, double* corr, int ldc, cudaStream_t st) {
    if (count == 0) return;
    // count is exact unless the round's count lives on the device (count_dev): then it is an
    // upper bound and the grid stays resident-sized, the CTAs striding over the live tiles.
    int64_t tiles = (count + kCorrVoxels - 1) / kCorrVoxels;
    if (count_dev) tiles = std::min<int64_t>(tiles, int64_t(sm_count()) * kCorrResidentCtas);
    const unsigned gx = unsigned(tiles);
    LaunchScope scope("correlate_kernel", st);
    if (R.c <= 48) {
        correlate_kernel<3><<<dim3(gx, 1), 128, 0, st>>>(S, list, count, count_dev, R.k, R.c, corr, ldc);
    } else {
        correlate_kernel<4><<<dim3(gx, unsigned((R.c + 63) / 64)), 128, 0, st>>>(S, list, count, count_dev, R.k, R.c,
                                                                                 corr, ldc);
    }
    cuda_check(cudaGetLastError(), "correlate_kernel launch");
}

// lsqnonneg (cpp/src/python/sd.cpp:208-228): one warp solves min ||c x - d|| over x >= 0 for c
// (m, n) row-major by the fraction fits' Lawson-Hanson with QR fits (cpp/src/sd/nnls.cpp:187-258),
// at most 3 n inner steps. default_tol: tol = 10 eps norm1(c) max(m, n) (nnls.cpp:177-181).
__global__ void __launch_bounds__(32) lsqnonneg_kernel(const double* __restrict__ c, int m, int n,
                                                       const double* __restrict__ d, bool default_tol, double tol,
                                                       double* __restrict__ x, double* __restrict__ workspace) {
    __shared__ FracState st;
    const int lane = threadIdx.x;
    const FracSlot sl = carve_frac(workspace, m, 0, n);
    if (default_tol) {
        double colmax = 0.0;
        for (int g = 0; g < n; ++g) {
            double sum = 0.0;
            for (int i = lane; i < m; i += 32) sum += fabs(c[size_t(i) * n + g]);
            colmax = fmax(colmax, warp_sum(sum));
        }
        tol = 10.0 * kEps64 * colmax * double(max(m, n));
    }
    NnlsScratch ns{sl.fu, sl.fz, sl.fflag, st.fact, &st.fn_act, sl.res,
                   QrScratch{sl.fsub, st.ftau, st.fnu, st.fnd, st.fperm, sl.frv}, kMaxGroups};
    warp_nnls_explicit(c, m, n, d, tol, 3 * n, ns, lane);
    for (int g = lane; g < n; g += 32) x[g] = sl.fu[g];
}

}  // namespace

}  // namespace lar

namespace lar {
// A device FP32 copy of an FP64 host array (rounded to nearest).
inline void upload_fp32(DeviceArray<float>& dst, const std::vector<double>& src) {
    std::vector<float> f(src.begin(), src.end());
    dst.upload(f.data(), f.size());
}
}  // namespace lar

// FodSolver.l2nnls (cpp/src/python/sd.cpp:89-102, cpp/src/sd/solver.cpp:464-467).
struct lar_fod_solver_s {
    // 0: the ridge NNLS (L2NNLS) with its design below; 1: damped Richardson-Lucy (dRL).
    int kind = 0;
    lar::DeviceArray<double> drl_kt, drl_gram;
    lar::DeviceArray<float> drl_gtc;  // K^T K for the tensor-core dRL (precision LAR_TF32X3)
    lar::DeviceArray<int> drl_err;    // where the tensor-core dRL records a wait that ran out
    lar::DrlDev drl{};
    lar::host::RidgeDesignHost host;
    double tol = 0.0;
    lar::DeviceArray<double> k, gram;
    lar::DeviceArray<float> k32, gram32;  // FP32 copies for the plain single-precision fit
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    int* pinned = nullptr;  // one host int the round loop reads the next round's count into
    ~lar_fod_solver_s() {
        if (scratch) cudaFree(scratch);
        if (pinned) cudaFreeHost(pinned);
    }
    int* count_buffer() {
        if (!pinned) lar::cuda_check(cudaMallocHost(&pinned, sizeof(int)), "cudaMallocHost");
        return pinned;
    }
    // The shell weights on the device, uploaded when they differ from the last call's. Under
    // stream capture nothing may be uploaded, so they must match an earlier uncaptured call.
    std::vector<double> weights_host;
    lar::DeviceArray<double> weights_dev;
    const double* device_weights(const double* w, int64_t m, bool capturing) {
        if (weights_host.size() != size_t(m) || !std::equal(w, w + m, weights_host.begin())) {
            lar::require(!capturing, "under stream capture the weights must be those of an earlier uncaptured "
                                     "call with this solver");
            weights_host.assign(w, w + m);
            weights_dev.upload(weights_host.data(), weights_host.size());
        }
        return weights_dev.ptr;
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
    lar::DeviceArray<float> kt32, iso32, wiso32;  // FP32 copies for the plain single-precision fit
    lar::DeviceArray<int> blocks;
    lar::TissueDev view() const {
        return lar::TissueDev{int(m), int(ca), int(ci), int(nb), kt.ptr, iso.ptr, wiso.ptr, blocks.ptr};
    }
};

using namespace lar;

// The multi-tissue fit behind both entry points. device_rounds: enqueue every round with its
// voxel count read on the device (as under stream capture) instead of reading each count back.
static int fit_multi_tissue(const double* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                            lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver,
                            int64_t max_outer, double fraction_tol, double final_tol_x, double* fods,
                            double* fractions, int32_t* rounds, uint8_t* status, void* stream,
                            bool device_rounds) {
    return guarded([&] {
        require(lr && hr && lr_solver && hr_solver, "kernels and solvers must not be NULL");
        require(weights != nullptr, "weights must not be NULL");
        const int64_t m = hr->m;
        require(lr->m == m, "signals, weights and the kernels' measurements do not match");
        require(lr->ci == hr->ci, "the two kernels have different numbers of isotropic tissues");
        // require_matching_solver (cpp/src/python/sd.cpp:294-307), with its message.
        auto matching = [m](const char* name, const lar_deconv_kernel_s& k, const lar_fod_solver_s& sv) {
            require(sv.host.c == k.ca && sv.host.m == m,
                    std::string("the ") + name + " solver (" + std::to_string(sv.host.c) + " directions, " +
                        std::to_string(sv.host.m) + " measurements) does not match its kernel (" +
                        std::to_string(k.ca) + " directions, " + std::to_string(m) + " measurements)");
        };
        matching("low-resolution", *lr, *lr_solver);
        matching("high-resolution", *hr, *hr_solver);
        require(max_outer >= 0, "max_outer must be at least 0");
        require(v >= 0, "v must be at least 0");
        if (v == 0) return;
        require(signals && fods && fractions, "signals, fods and fractions must not be NULL");
        const int mi = int(m), ci = int(lr->ci), c_lr = int(lr->ca), c_hr = int(hr->ca);
        const int nf = int(hr->nb + hr->ci);
        const int max_rounds = int(std::min<int64_t>(max_outer, 1 << 20));
        const RidgeDev lrs = lr_solver->view(), hrs = hr_solver->view();
        const TissueDev lrt = lr->view(), hrt = hr->view();
        // A dRL solver (GRL) replaces the correlations and the NNLS of its stage by drl_kernel on
        // the stage's anisotropic signals; the fractions are the same.
        const bool lr_drl = lr_solver->kind == 1, hr_drl = hr_solver->kind == 1;
        const NnlsLaunch lr_nnls = nnls_variant(c_lr), hr_nnls = nnls_variant(c_hr);
        const size_t lr_smem = nnls_smem_bytes(c_lr, lr_nnls.cap) * kMtWarps;
        const size_t hr_smem = nnls_smem_bytes(c_hr, hr_nnls.cap) * kMtWarps;
        // Voxels per pass: the per-voxel state of a pass (correlations, the low-resolution FOD,
        // f_iso and the previous fractions, two list entries, the round count and status) within
        // 4 GiB.
        const size_t per_voxel = (size_t(std::max(c_lr, c_hr)) + size_t(c_lr) + 2 * size_t(ci) + 1) * sizeof(double) +
                                 3 * sizeof(int) + 1;
        const int64_t n_max = std::min<int64_t>(v, std::max<int64_t>(4096, int64_t((size_t(4) << 30) / per_voxel)));
        const int64_t lr_slots = lr_drl ? 0 : resident_slots(lr_nnls.kernel, lr_smem, n_max, "sd.nnls.ctas_per_sm");
        // Low-resolution kernels of at most 48 directions with normal equations: two voxels per
        // warp (ridge_nnls_half_kernel), the voxels that need the QR fallback then refitted by
        // the one-warp kernel.
        const bool half = !lr_drl && lrs.normal_equations && c_lr <= 48;
        auto half_kernel = ridge_nnls_half_kernel<3>;
        const size_t half_smem = half_smem_bytes(c_lr) * 2 * kMtWarps;
        const int64_t half_warps = half ? resident_slots(half_kernel, half_smem, n_max, "sd.nnls.ctas_per_sm") : 0;
        const int64_t hr_slots = hr_drl ? 0 : resident_slots(hr_nnls.kernel, hr_smem, n_max, "sd.nnls.ctas_per_sm");
        // High-resolution kernels of 65 to 320 directions with normal equations: a first pass with
        // a 32-column factor, the voxels that outgrow it refitted by the full-factor kernel.
        const bool hr_first = !hr_drl && hrs.normal_equations && c_hr > 64 && c_hr <= 320;
        auto first_kernel = ridge_nnls_first_kernel<1, 10>;
        const size_t first_smem = nnls_smem_bytes(c_hr, 32) * kMtWarps;
        const int64_t first_slots = hr_first ? resident_slots(first_kernel, first_smem, n_max, "sd.nnls.ctas_per_sm") : 0;
        const size_t first_slot = nnls_slot_doubles(mi, 32);
        const int64_t lf_slots = resident_slots(lr_fractions_kernel, 0, n_max, "sd.fractions.ctas_per_sm");
        const int64_t hf_slots = resident_slots(hr_fractions_kernel, 0, n_max, "sd.fractions.ctas_per_sm");
        const size_t lr_slot = nnls_slot_doubles(mi, lr_nnls.cap), hr_slot = nnls_slot_doubles(mi, hr_nnls.cap);
        const size_t lf_slot = frac_slot_doubles(mi, c_lr, 1 + ci), hf_slot = frac_slot_doubles(mi, c_hr, nf);
        const size_t slot_doubles =
            std::max(std::max(std::max(std::max(size_t(lr_slots) * lr_slot, size_t(hr_slots) * hr_slot),
                                       std::max(size_t(lf_slots) * lf_slot, size_t(hf_slots) * hf_slot)),
                              size_t(2 * half_warps) * half_slot_doubles()),
                     size_t(first_slots) * first_slot);
        struct Pieces {
            int* counters;  // [0] the persistent kernels' work counter, [2], [3] the two lists' counts,
                            // [4] the voxels to refit by the one-warp NNLS
            int* list[2];
            int* redo;
            double *fiso, *prev, *corr, *xlr, *slots;
            int32_t* rounds;
            uint8_t* bad;
        };
        auto carve_all = [&](Carver& cv) {
            Pieces p;
            p.counters = cv.take<int>(8);
            p.list[0] = cv.take<int>(size_t(n_max));
            p.list[1] = cv.take<int>(size_t(n_max));
            p.redo = cv.take<int>(size_t(n_max));
            p.fiso = cv.take<double>(size_t(n_max) * std::max(ci, 1));
            p.prev = cv.take<double>(size_t(n_max) * (ci + 1));
            p.corr = cv.take<double>(size_t(n_max) * std::max(c_lr, c_hr));
            p.xlr = cv.take<double>(size_t(n_max) * c_lr);
            p.rounds = cv.take<int32_t>(size_t(n_max));
            p.bad = cv.take<uint8_t>(size_t(n_max));
            p.slots = cv.take<double>(slot_doubles);
            return p;
        };
        Carver sizing{nullptr};
        carve_all(sizing);
        Carver cv{static_cast<char*>(hr_solver->reserve(sizing.used))};
        const Pieces P = carve_all(cv);
        auto st = static_cast<cudaStream_t>(stream);
        // Under stream capture (a CUDA graph) nothing may wait on the host: every round is
        // enqueued and reads its voxel count on the device, exiting at once when it is 0.
        cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
        cuda_check(cudaStreamIsCapturing(st, &capture), "cudaStreamIsCapturing");
        const bool capturing = capture != cudaStreamCaptureStatusNone;
        const bool graph = capturing || device_rounds;
        const double* dweights = hr_solver->device_weights(weights, m, capturing);
        int* host_count = graph ? nullptr : hr_solver->count_buffer();
        auto blocks = [](int64_t slots, int64_t count) {
            return unsigned(std::max<int64_t>(1, std::min<int64_t>(slots / kMtWarps, (count + kMtWarps - 1) / kMtWarps)));
        };
        auto reset_queue = [&] { cuda_check(cudaMemsetAsync(P.counters, 0, sizeof(int), st), "cudaMemsetAsync"); };
        for (int64_t v0 = 0; v0 < v; v0 += n_max) {
            const int64_t n = std::min(n_max, v - v0);
            const double* sig = signals + v0 * m;
            if (ci > 0) cuda_check(cudaMemsetAsync(P.fiso, 0, size_t(n) * ci * sizeof(double), st), "cudaMemsetAsync");
            cuda_check(cudaMemsetAsync(P.rounds, 0, size_t(n) * sizeof(int32_t), st), "cudaMemsetAsync");
            cuda_check(cudaMemsetAsync(P.bad, 0, size_t(n), st), "cudaMemsetAsync");
            const SignalDev lr_sig{sig, dweights, lrt.wiso, P.fiso, mi, ci};
            // The first round takes every voxel; later rounds the list the previous one wrote,
            // with its count read back on the host (or, under capture, on the device).
            const int* cur = nullptr;
            const int* cur_count = nullptr;
            int side = 0;
            int64_t count = n;
            for (int round = 0; round < max_rounds && count > 0; ++round) {
                int* nxt = P.list[side];
                int* nxt_count = P.counters + 2 + side;
                if (!lr_drl) launch_correlate(lr_sig, cur, count, cur_count, lrs, P.corr, c_lr, st);
                reset_queue();
                cuda_check(cudaMemsetAsync(nxt_count, 0, sizeof(int), st), "cudaMemsetAsync");
                if (lr_drl) {
                    const DrlSignal lr_as{sig, dweights, lrt.wiso, P.fiso, mi, ci};
                    launch_drl_listed(lr_solver->drl, lr_as, cur, count, cur_count, P.xlr, c_lr, st);
                } else if (half) {
                    cuda_check(cudaMemsetAsync(P.counters + 4, 0, sizeof(int), st), "cudaMemsetAsync");
                    {
                        LaunchScope scope("ridge_nnls_half_kernel<3>", st);
                        half_kernel<<<blocks(half_warps, (count + 1) / 2), kMtWarps * 32, half_smem, st>>>(
                            lrs, cur, count, cur_count, P.corr, c_lr, P.xlr, c_lr, P.redo, P.counters + 4, P.counters,
                            P.slots, half_slot_doubles());
                        cuda_check(cudaGetLastError(), "ridge_nnls_half_kernel launch");
                    }
                    reset_queue();
                    // The voxels the two-voxel kernel handed back are rare (its QR fallback): a
                    // persistent grid of one CTA per SM takes them.
                    LaunchScope scope(lr_nnls.name, st);
                    const unsigned redo_blocks = std::min<unsigned>(blocks(lr_slots, count), unsigned(sm_count()));
                    lr_nnls.kernel<<<redo_blocks, kMtWarps * 32, lr_smem, st>>>(
                        lrs, lr_sig, P.redo, count, P.counters + 4, P.corr, c_lr, P.xlr, c_lr, P.bad, P.counters,
                        P.slots, lr_slot);
                    cuda_check(cudaGetLastError(), "ridge_nnls_kernel launch");
                } else {
                    LaunchScope scope(lr_nnls.name, st);
                    lr_nnls.kernel<<<blocks(lr_slots, count), kMtWarps * 32, lr_smem, st>>>(
                        lrs, lr_sig, cur, count, cur_count, P.corr, c_lr, P.xlr, c_lr, P.bad, P.counters, P.slots,
                        lr_slot);
                    cuda_check(cudaGetLastError(), "ridge_nnls_kernel launch");
                }
                reset_queue();
                {
                    LaunchScope scope("lr_fractions_kernel", st);
                    lr_fractions_kernel<<<blocks(lf_slots, count), kMtWarps * 32, 0, st>>>(
                        lrt, sig, P.xlr, c_lr, cur, count, cur_count, round, max_rounds, fraction_tol, P.fiso, P.prev,
                        P.rounds, nxt, nxt_count, P.counters, P.slots, lf_slot);
                    cuda_check(cudaGetLastError(), "lr_fractions_kernel launch");
                }
                if (!graph) {
                    cuda_check(cudaMemcpyAsync(host_count, nxt_count, sizeof(int), cudaMemcpyDeviceToHost, st),
                               "cudaMemcpyAsync (round count)");
                    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
                    count = *host_count;
                } else {
                    cur_count = nxt_count;
                }
                cur = nxt;
                side ^= 1;
            }
            const SignalDev hr_sig{sig, dweights, hrt.wiso, P.fiso, mi, ci};
            if (hr_drl) {
                const DrlSignal hr_as{sig, dweights, hrt.wiso, P.fiso, mi, ci};
                launch_drl_listed(hr_solver->drl, hr_as, nullptr, n, nullptr, fods + v0 * c_hr, c_hr, st);
            } else {
                launch_correlate(hr_sig, nullptr, n, nullptr, hrs, P.corr, c_hr, st);
                reset_queue();
                if (hr_first) {
                    cuda_check(cudaMemsetAsync(P.counters + 4, 0, sizeof(int), st), "cudaMemsetAsync");
                    {
                        LaunchScope scope("ridge_nnls_first_kernel<1,10>", st);
                        first_kernel<<<blocks(first_slots, n), kMtWarps * 32, first_smem, st>>>(
                            hrs, hr_sig, n, P.corr, c_hr, fods + v0 * c_hr, c_hr, P.redo, P.counters + 4, P.counters,
                            P.slots, first_slot);
                        cuda_check(cudaGetLastError(), "ridge_nnls_first_kernel launch");
                    }
                    reset_queue();
                    // The voxels the first pass handed back (rare): a grid of one CTA per SM.
                    LaunchScope scope(hr_nnls.name, st);
                    const unsigned redo_blocks = std::min<unsigned>(blocks(hr_slots, n), unsigned(sm_count()));
                    hr_nnls.kernel<<<redo_blocks, kMtWarps * 32, hr_smem, st>>>(
                        hrs, hr_sig, P.redo, n, P.counters + 4, P.corr, c_hr, fods + v0 * c_hr, c_hr, P.bad,
                        P.counters, P.slots, hr_slot);
                    cuda_check(cudaGetLastError(), "ridge_nnls_kernel launch");
                } else {
                    LaunchScope scope(hr_nnls.name, st);
                    hr_nnls.kernel<<<blocks(hr_slots, n), kMtWarps * 32, hr_smem, st>>>(
                        hrs, hr_sig, nullptr, n, nullptr, P.corr, c_hr, fods + v0 * c_hr, c_hr, P.bad, P.counters,
                        P.slots, hr_slot);
                    cuda_check(cudaGetLastError(), "ridge_nnls_kernel launch");
                }
            }
            reset_queue();
            LaunchScope scope("hr_fractions_kernel", st);
            hr_fractions_kernel<<<blocks(hf_slots, n), kMtWarps * 32, 0, st>>>(
                hrt, sig, fods + v0 * c_hr, n, final_tol_x, P.rounds, P.bad, fractions + v0 * nf,
                rounds ? rounds + v0 : nullptr, status ? status + v0 : nullptr, P.counters, P.slots, hf_slot);
            cuda_check(cudaGetLastError(), "hr_fractions_kernel launch");
        }
    });
}

// ---- batches (batch.cuh): the mFOD family --------------------------------------------------

namespace lar {

struct MfodBatch {
    std::vector<MfodBatchJob> jobs;
    std::vector<std::vector<double>> weights;
    std::vector<std::unique_ptr<DeviceArray<double>>> weights_dev;
    int max_rounds = -1;
    double fraction_tol = 0.0, final_tol = 0.0;
    int ci = -1, m_max = 0, c_lr_max = 0, c_hr_max = 0, nf_max = 0;
    int64_t voxels = 0, tiles = 0;
    // Finalized: the device job table, the per-voxel state and the launch shapes.
    DeviceArray<MfodBatchJob> d_jobs;
    void* scratch = nullptr;
    MfodBatchState B{};
    int *list[2] = {nullptr, nullptr}, *counts[2] = {nullptr, nullptr}, *queue = nullptr;
    double* slots = nullptr;
    int64_t half_warps = 0, lr_slots = 0, first_slots = 0, hr_slots = 0, lf_slots = 0, hf_slots = 0;
    size_t half_smem = 0, lr_smem = 0, first_smem = 0, hr_smem = 0;
    size_t lr_slot = 0, first_slot = 0, hr_slot = 0, lf_slot = 0, hf_slot = 0;
    ~MfodBatch() {
        if (scratch) cudaFree(scratch);
    }
};

MfodBatch* mfod_batch_create() { return new MfodBatch(); }

void mfod_batch_destroy(MfodBatch* b) { delete b; }

void mfod_batch_add(MfodBatch* b, const double* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                    lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver, int64_t max_outer,
                    double fraction_tol, double final_tol_x, double* fods, double* fractions, int32_t* rounds,
                    uint8_t* status) {
    require(lr && hr && lr_solver && hr_solver, "kernels and solvers must not be NULL");
    require(weights != nullptr, "weights must not be NULL");
    const int64_t m = hr->m;
    require(lr->m == m, "signals, weights and the kernels' measurements do not match");
    require(lr->ci == hr->ci, "the two kernels have different numbers of isotropic tissues");
    require(lr_solver->host.c == lr->ca && lr_solver->host.m == m && hr_solver->host.c == hr->ca &&
                hr_solver->host.m == m,
            "a solver does not match its kernel");
    require(lr_solver->kind == 0 && hr_solver->kind == 0 && lr_solver->host.normal_equations &&
                hr_solver->host.normal_equations,
            "a batch takes ridge NNLS (L2NNLS) solvers with normal equations");
    require(lr->ca <= 48 && hr->ca > 64 && hr->ca <= 320,
            "a batch takes low-resolution kernels of at most 48 directions and high-resolution ones of 65 to 320");
    require(max_outer >= 0 && v >= 0, "max_outer and v must be at least 0");
    require(v == 0 || (signals && fods && fractions), "signals, fods and fractions must not be NULL");
    const int rounds_cap = int(std::min<int64_t>(max_outer, 1 << 20));
    if (b->max_rounds < 0) {
        b->max_rounds = rounds_cap;
        b->fraction_tol = fraction_tol;
        b->final_tol = final_tol_x;
        b->ci = int(lr->ci);
    }
    require(rounds_cap == b->max_rounds && fraction_tol == b->fraction_tol && final_tol_x == b->final_tol,
            "every mFOD job of a batch takes the same max_outer, fraction_tol and final_tol_x");
    require(int(lr->ci) == b->ci, "every mFOD job of a batch has the same isotropic tissues");
    MfodBatchJob j{};
    j.v = v;
    j.off = b->voxels;
    j.lr = lr_solver->view();
    j.hr = hr_solver->view();
    j.lrt = lr->view();
    j.hrt = hr->view();
    j.s = signals;
    j.fods = fods;
    j.fractions = fractions;
    j.rounds = rounds;
    j.status = status;
    b->jobs.push_back(j);
    b->weights.emplace_back(weights, weights + m);
    b->voxels += v;
    b->tiles += (v + kCorrVoxels - 1) / kCorrVoxels;
    b->m_max = std::max(b->m_max, int(m));
    b->c_lr_max = std::max(b->c_lr_max, int(lr->ca));
    b->c_hr_max = std::max(b->c_hr_max, int(hr->ca));
    b->nf_max = std::max(b->nf_max, int(hr->nb + hr->ci));
}

void mfod_batch_finalize(MfodBatch* b) {
    if (b->jobs.empty()) return;
    require(b->voxels < (int64_t(1) << 31), "at most 2^31 - 1 mFOD voxels per batch");
    for (size_t k = 0; k < b->jobs.size(); ++k) {
        b->weights_dev.push_back(std::make_unique<DeviceArray<double>>());
        b->weights_dev.back()->upload(b->weights[k].data(), b->weights[k].size());
        b->jobs[k].w = b->weights_dev.back()->ptr;
    }
    b->d_jobs.upload(b->jobs.data(), b->jobs.size());
    const int64_t V = b->voxels, nj = int64_t(b->jobs.size());
    const int ci = b->ci, mi = b->m_max, ldc = std::max(b->c_lr_max, b->c_hr_max), ldx = b->c_lr_max;
    // Launch shapes: the single-volume fit's persistent grids, sized for the whole batch.
    b->half_smem = half_smem_bytes(b->c_lr_max) * 2 * kMtWarps;
    b->half_warps = resident_slots(batch_half_kernel<3>, b->half_smem, V, "sd.nnls.ctas_per_sm");
    b->lr_smem = nnls_smem_bytes(b->c_lr_max, 32) * kMtWarps;
    b->lr_slots = resident_slots(batch_redo_kernel<1, 2, false>, b->lr_smem, V, "sd.nnls.ctas_per_sm");
    b->first_smem = nnls_smem_bytes(b->c_hr_max, 32) * kMtWarps;
    b->first_slots = resident_slots(batch_first_kernel, b->first_smem, V, "sd.nnls.ctas_per_sm");
    b->hr_smem = nnls_smem_bytes(b->c_hr_max, kCholCap) * kMtWarps;
    b->hr_slots = resident_slots(batch_redo_kernel<kCholCap / 32, 10, true>, b->hr_smem, V, "sd.nnls.ctas_per_sm");
    b->lf_slots = resident_slots(batch_lr_fractions_kernel, 0, V, "sd.fractions.ctas_per_sm");
    b->hf_slots = resident_slots(batch_hr_fractions_kernel, 0, V, "sd.fractions.ctas_per_sm");
    b->lr_slot = nnls_slot_doubles(mi, 32);
    b->first_slot = nnls_slot_doubles(mi, 32);
    b->hr_slot = nnls_slot_doubles(mi, kCholCap);
    b->lf_slot = frac_slot_doubles(mi, b->c_lr_max, 1 + ci);
    b->hf_slot = frac_slot_doubles(mi, b->c_hr_max, b->nf_max);
    const size_t slot_doubles = std::max(
        {size_t(2 * b->half_warps) * half_slot_doubles(), size_t(b->lr_slots) * b->lr_slot,
         size_t(b->first_slots) * b->first_slot, size_t(b->hr_slots) * b->hr_slot, size_t(b->lf_slots) * b->lf_slot,
         size_t(b->hf_slots) * b->hf_slot});
    auto carve_all = [&](Carver& cv) {
        MfodBatchState s{};
        s.jobs = b->d_jobs.ptr;
        s.n_jobs = int(nj);
        s.ci = ci;
        s.ldc = ldc;
        s.ldx = ldx;
        s.fiso = cv.take<double>(size_t(V) * std::max(ci, 1));
        s.prev = cv.take<double>(size_t(V) * (ci + 1));
        s.corr = cv.take<double>(size_t(V) * ldc);
        s.xlr = cv.take<double>(size_t(V) * ldx);
        s.rounds = cv.take<int32_t>(size_t(V));
        s.bad = cv.take<uint8_t>(size_t(V));
        s.vfirst = cv.take<int64_t>(size_t(nj) + 1);
        s.tfirst = cv.take<int64_t>(size_t(nj) + 1);
        s.redo = cv.take<int64_t>(size_t(V));
        s.redo_count = cv.take<int>(1);
        b->list[0] = cv.take<int>(size_t(V));
        b->list[1] = cv.take<int>(size_t(V));
        b->counts[0] = cv.take<int>(size_t(nj));
        b->counts[1] = cv.take<int>(size_t(nj));
        b->queue = cv.take<int>(1);
        b->slots = cv.take<double>(slot_doubles);
        return s;
    };
    Carver sizing{nullptr};
    carve_all(sizing);
    cuda_check(cudaMalloc(&b->scratch, sizing.used), "cudaMalloc (mFOD batch state)");
    Carver cv{static_cast<char*>(b->scratch)};
    b->B = carve_all(cv);
}

void mfod_batch_run(MfodBatch* b, cudaStream_t st) {
    if (b->jobs.empty() || b->voxels == 0) return;
    const MfodBatchState& B = b->B;
    const int64_t V = b->voxels, nj = int64_t(b->jobs.size());
    const int ci = b->ci;
    auto blocks = [](int64_t slots, int64_t count) {
        return unsigned(std::max<int64_t>(1, std::min<int64_t>(slots / kMtWarps, (count + kMtWarps - 1) / kMtWarps)));
    };
    auto zero = [&](void* p, size_t bytes) { cuda_check(cudaMemsetAsync(p, 0, bytes, st), "cudaMemsetAsync"); };
    auto launched = [](const char* what) { cuda_check(cudaGetLastError(), what); };
    if (ci > 0) zero(B.fiso, size_t(V) * ci * sizeof(double));
    zero(B.rounds, size_t(V) * sizeof(int32_t));
    zero(B.bad, size_t(V));
    // The correlation grids stay resident-sized: a round's tiles are only known on the device.
    const unsigned corr_grid = unsigned(std::min<int64_t>(b->tiles, int64_t(sm_count()) * kCorrResidentCtas));
    const unsigned lr_redo_blocks = std::min<unsigned>(blocks(b->lr_slots, V), unsigned(sm_count()));
    const unsigned hr_redo_blocks = std::min<unsigned>(blocks(b->hr_slots, V), unsigned(sm_count()));
    // Every round is enqueued: each stage reads its tickets on the device, so a round whose
    // lists are all empty costs only its launches.
    const int* cur = nullptr;
    const int* cur_counts = nullptr;
    int side = 0;
    for (int round = 0; round < b->max_rounds; ++round) {
        int* nxt = b->list[side];
        int* nxt_counts = b->counts[side];
        {
            LaunchScope scope("batch_plan_kernel", st);
            batch_plan_kernel<<<1, 32, 0, st>>>(B, cur_counts);
            launched("batch_plan_kernel launch");
        }
        {
            LaunchScope scope("batch_correlate_kernel", st);
            batch_correlate_kernel<3, false><<<corr_grid, 128, 0, st>>>(B, cur);
            launched("batch_correlate_kernel launch");
        }
        zero(b->queue, sizeof(int));
        zero(nxt_counts, size_t(nj) * sizeof(int));
        zero(B.redo_count, sizeof(int));
        {
            LaunchScope scope("batch_half_kernel<3>", st);
            batch_half_kernel<3><<<blocks(b->half_warps, (V + 1) / 2), kMtWarps * 32, b->half_smem, st>>>(
                B, cur, b->c_lr_max, b->queue, b->slots, half_slot_doubles());
            launched("batch_half_kernel launch");
        }
        zero(b->queue, sizeof(int));
        {
            LaunchScope scope("batch_redo_kernel<1,2>", st);
            batch_redo_kernel<1, 2, false><<<lr_redo_blocks, kMtWarps * 32, b->lr_smem, st>>>(
                B, b->c_lr_max, b->queue, b->slots, b->lr_slot);
            launched("batch_redo_kernel launch");
        }
        zero(b->queue, sizeof(int));
        {
            LaunchScope scope("batch_lr_fractions_kernel", st);
            batch_lr_fractions_kernel<<<blocks(b->lf_slots, V), kMtWarps * 32, 0, st>>>(
                B, cur, round, b->max_rounds, b->fraction_tol, nxt, nxt_counts, b->queue, b->slots, b->lf_slot);
            launched("batch_lr_fractions_kernel launch");
        }
        cur = nxt;
        cur_counts = nxt_counts;
        side ^= 1;
    }
    {
        LaunchScope scope("batch_plan_kernel", st);
        batch_plan_kernel<<<1, 32, 0, st>>>(B, nullptr);
        launched("batch_plan_kernel launch");
    }
    {
        LaunchScope scope("batch_correlate_kernel", st);
        batch_correlate_kernel<4, true><<<dim3(corr_grid, unsigned((b->c_hr_max + 63) / 64)), 128, 0, st>>>(
            B, nullptr);
        launched("batch_correlate_kernel launch");
    }
    zero(b->queue, sizeof(int));
    zero(B.redo_count, sizeof(int));
    {
        LaunchScope scope("batch_first_kernel<1,10>", st);
        batch_first_kernel<<<blocks(b->first_slots, V), kMtWarps * 32, b->first_smem, st>>>(
            B, b->c_hr_max, b->queue, b->slots, b->first_slot);
        launched("batch_first_kernel launch");
    }
    zero(b->queue, sizeof(int));
    {
        LaunchScope scope("batch_redo_kernel<8,10>", st);
        batch_redo_kernel<kCholCap / 32, 10, true><<<hr_redo_blocks, kMtWarps * 32, b->hr_smem, st>>>(
            B, b->c_hr_max, b->queue, b->slots, b->hr_slot);
        launched("batch_redo_kernel launch");
    }
    zero(b->queue, sizeof(int));
    LaunchScope scope("batch_hr_fractions_kernel", st);
    batch_hr_fractions_kernel<<<blocks(b->hf_slots, V), kMtWarps * 32, 0, st>>>(B, b->final_tol, b->queue, b->slots,
                                                                              b->hf_slot);
    launched("batch_hr_fractions_kernel launch");
}

}  // namespace lar

extern "C" {

int lar_fit_multi_tissue(const double* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                         lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver,
                         int64_t max_outer, double fraction_tol, double final_tol_x, double* fods,
                         double* fractions, int32_t* rounds, uint8_t* status, void* stream) {
    return fit_multi_tissue(signals, v, weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol, final_tol_x,
                            fods, fractions, rounds, status, stream, false);
}

int lar_fit_multi_tissue_async(const double* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                               lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver,
                               int64_t max_outer, double fraction_tol, double final_tol_x, double* fods,
                               double* fractions, int32_t* rounds, uint8_t* status, void* stream) {
    return fit_multi_tissue(signals, v, weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol, final_tol_x,
                            fods, fractions, rounds, status, stream, true);
}

int lar_fit_multi_tissue_plain_fp32(const float* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                                    lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver,
                                    int64_t max_outer, double fraction_tol, double final_tol_x, float* fods,
                                    float* fractions, int32_t* rounds, uint8_t* status, void* stream) {
    return guarded([&] {
        require(lr && hr && lr_solver && hr_solver, "kernels and solvers must not be NULL");
        require(weights != nullptr, "weights must not be NULL");
        require(lr_solver->kind == 0 && hr_solver->kind == 0, "the plain FP32 fit takes L2NNLS solvers");
        const int64_t m = hr->m;
        require(lr->m == m && lr_solver->host.m == m && hr_solver->host.m == m,
                "signals, weights and the kernels' measurements do not match");
        require(lr_solver->host.c == lr->ca && hr_solver->host.c == hr->ca, "a solver does not match its kernel");
        require(lr->ci == hr->ci && lr->nb == 1, "the low-resolution kernel must have one anisotropic block and the "
                                                 "isotropic tissues of the high-resolution one");
        require(m <= kPlainMaxMeasurements && std::max(lr->ca, hr->ca) <= kPlainMaxColumns &&
                    hr->nb + hr->ci <= kPlainMaxGroups && 1 + lr->ci <= kPlainMaxGroups,
                "the plain FP32 fit takes at most 512 measurements, 320 directions and 4 fraction columns");
        require(max_outer >= 0 && v >= 0, "max_outer and v must be at least 0");
        if (v == 0) return;
        require(signals && fods && fractions, "signals, fods and fractions must not be NULL");
        auto st = static_cast<cudaStream_t>(stream);
        auto stage = [](const lar_deconv_kernel_s& k, const lar_fod_solver_s& sv) {
            return PlainStage{int(k.m), int(k.ca), int(k.ci), int(k.nb), float(sv.tol), sv.k32.ptr, sv.gram32.ptr,
                              k.kt32.ptr, k.iso32.ptr, k.wiso32.ptr, k.blocks.ptr};
        };
        std::vector<float> w32(weights, weights + m);
        float* dw = nullptr;
        cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&dw), size_t(m) * sizeof(float), st), "cudaMallocAsync");
        cuda_check(cudaMemcpyAsync(dw, w32.data(), size_t(m) * sizeof(float), cudaMemcpyHostToDevice, st),
                   "cudaMemcpyAsync");
        launch_plain_fp32(stage(*lr, *lr_solver), stage(*hr, *hr_solver), signals, v, dw,
                          int(std::min<int64_t>(max_outer, 1 << 20)), float(fraction_tol), float(final_tol_x), fods,
                          fractions, rounds, status, st);
        // The weights' host copy must outlive the copy above.
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        cuda_check(cudaFreeAsync(dw, st), "cudaFreeAsync");
    });
}

int lar_lsqnonneg(const double* c, int64_t m, int64_t n, const double* d, int default_tol, double tol_x, double* x,
                  void* stream) {
    return guarded([&] {
        require(m >= 1 && n >= 1 && n <= kMaxGroups, "lsqnonneg takes c of (m, n), m >= 1, 1 <= n <= 16");
        require(c && d && x, "c, d and x must not be NULL");
        auto st = static_cast<cudaStream_t>(stream);
        double* ws = nullptr;
        const size_t bytes = frac_slot_doubles(int(m), 0, int(n)) * sizeof(double);
        cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&ws), bytes, st), "cudaMallocAsync");
        {
            LaunchScope scope("lsqnonneg_kernel", st);
            lsqnonneg_kernel<<<1, 32, 0, st>>>(c, int(m), int(n), d, default_tol != 0, tol_x, x, ws);
            cuda_check(cudaGetLastError(), "lsqnonneg_kernel launch");
        }
        cuda_check(cudaFreeAsync(ws, st), "cudaFreeAsync");
    });
}


int lar_drl_create(const double* k_t, const double* k_t_k, int64_t c, int64_t m, double nu, int64_t n_iter,
                   double init, lar_fod_solver* out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        require(k_t != nullptr && k_t_k != nullptr && c > 0 && m > 1, "k_t must be a non-empty (c, m) array, m > 1");
        require(drl_fits(int(c)), "dRL takes at most 640 directions");
        require(n_iter >= 0, "n_iter must be at least 0");
        auto h = std::make_unique<lar_fod_solver_s>();
        h->kind = 1;
        h->host.m = m;
        h->host.c = c;
        h->drl_kt.upload(k_t, size_t(c * m));
        h->drl_gram.upload(k_t_k, size_t(c * c));
        h->drl = DrlDev{h->drl_kt.ptr, h->drl_gram.ptr, int(c), int(m), int(n_iter), nu, init};
        *out = h.release();
    });
}

int lar_l2nnls_create(const double* k, int64_t m, int64_t c, double reg, double tol_x, lar_fod_solver* out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        require(reg >= 0.0, "reg must be at least 0");
        require(tol_x > 0.0, "tol_x must be positive");
        require(k != nullptr && m > 0 && c > 0, "k must be a non-empty (m, c) array");
        require(c <= 640 && m <= 4096, "the kernel has more than 640 directions or 4096 measurements");
        auto h = std::make_unique<lar_fod_solver_s>();
        h->host = host::prepare_ridge_design(k, m, c, reg);
        h->tol = tol_x;
        h->k.upload(h->host.kernel.data(), h->host.kernel.size());
        h->gram.upload(h->host.gram.data(), h->host.gram.size());
        upload_fp32(h->k32, h->host.kernel);
        upload_fp32(h->gram32, h->host.gram);
        *out = h.release();
    });
}

int lar_drl_set_precision(lar_fod_solver solver, int precision) {
    return guarded([&] {
        require(solver != nullptr && solver->kind == 1, "solver must be a dRL solver");
        require(precision == LAR_FP64 || precision == LAR_TF32X3, "precision must be LAR_FP64 or LAR_TF32X3");
        if (precision == LAR_FP64) {
            solver->drl.gtc = nullptr;
            solver->drl.err = nullptr;
            return;
        }
        const int c = int(solver->host.c);
        require(drl_tc_fits(c) && drl_tc_fits_measurements(c, int(solver->host.m)),
                "the tensor-core dRL takes 65 to 320 directions and at most " +
                    std::to_string(drl_tc_smem_bytes(c) / (48 * 8)) + " measurements");
        std::vector<double> gram(size_t(c) * c);
        cuda_check(cudaMemcpy(gram.data(), solver->drl_gram.ptr, gram.size() * sizeof(double), cudaMemcpyDeviceToHost),
                   "cudaMemcpy");
        const std::vector<float> layout = drl_tc_layout(gram.data(), c);
        solver->drl_gtc.upload(layout.data(), layout.size());
        const int zero = 0;
        solver->drl_err.upload(&zero, 1);
        solver->drl.gtc = solver->drl_gtc.ptr;
        solver->drl.err = solver->drl_err.ptr;
    });
}

int lar_drl_errors(lar_fod_solver solver, int* out) {
    return guarded([&] {
        require(solver != nullptr && out != nullptr, "solver and out must not be NULL");
        *out = 0;
        if (solver->drl.err == nullptr) return;
        cuda_check(cudaMemcpy(out, solver->drl.err, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
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
        upload_fp32(h->kt32, kt);
        std::vector<double> iso(size_t(std::max<int64_t>(1, m * ci)), 0.0), wiso(iso.size(), 0.0);
        if (ci > 0) {
            std::copy(k_iso, k_iso + m * ci, iso.begin());
            std::copy(w_k_iso, w_k_iso + m * ci, wiso.begin());
        }
        h->iso.upload(iso.data(), iso.size());
        h->wiso.upload(wiso.data(), wiso.size());
        upload_fp32(h->iso32, iso);
        upload_fp32(h->wiso32, wiso);
        std::vector<int> bl(size_t(2 * nb));
        for (int64_t b = 0; b < 2 * nb; ++b) bl[size_t(b)] = int(blocks[b]);
        h->blocks.upload(bl.data(), bl.size());
        *out = h.release();
    });
}

void lar_deconv_kernel_destroy(lar_deconv_kernel kernel) { delete kernel; }

int lar_fit_single_tissue(const double* signals, int64_t v, lar_fod_solver solver, double* fods, uint8_t* status,
                          void* stream) {
    return guarded([&] {
        require(solver != nullptr, "solver must not be NULL");
        require(v >= 0, "v must be at least 0");
        if (v == 0) return;
        require(signals && fods, "signals and fods must not be NULL");
        if (solver->kind == 1) {
            if (status) cuda_check(cudaMemsetAsync(status, 0, size_t(v), static_cast<cudaStream_t>(stream)),
                                   "cudaMemsetAsync");
            launch_drl(solver->drl, signals, v, fods, static_cast<cudaStream_t>(stream));
            return;
        }
        const int m = int(solver->host.m), c = int(solver->host.c);
        const RidgeDev R = solver->view();
        const NnlsLaunch nn = nnls_variant(c);
        const size_t smem = nnls_smem_bytes(c, nn.cap) * kMtWarps;
        const int64_t n_max = std::min<int64_t>(v, std::max<int64_t>(4096, int64_t((size_t(2) << 30) / (size_t(c) * 8))));
        const int64_t slots = resident_slots(nn.kernel, smem, n_max, "sd.nnls.ctas_per_sm");
        const size_t slot = nnls_slot_doubles(m, nn.cap);
        auto carve_all = [&](Carver& cv, int*& counters, double*& corr, double*& work) {
            counters = cv.take<int>(8);
            corr = cv.take<double>(size_t(n_max) * c);
            work = cv.take<double>(size_t(slots) * slot);
        };
        int* counters = nullptr;
        double *corr = nullptr, *work = nullptr;
        Carver sizing{nullptr};
        carve_all(sizing, counters, corr, work);
        Carver cv{static_cast<char*>(solver->reserve(sizing.used))};
        carve_all(cv, counters, corr, work);
        auto st = static_cast<cudaStream_t>(stream);
        for (int64_t v0 = 0; v0 < v; v0 += n_max) {
            const int64_t n = std::min(n_max, v - v0);
            const SignalDev S{signals + v0 * m, nullptr, nullptr, nullptr, m, 0};
            launch_correlate(S, nullptr, n, nullptr, R, corr, c, st);
            if (status) cuda_check(cudaMemsetAsync(status + v0, 0, size_t(n), st), "cudaMemsetAsync");
            cuda_check(cudaMemsetAsync(counters, 0, sizeof(int), st), "cudaMemsetAsync");
            const unsigned nb = unsigned(std::max<int64_t>(1, std::min<int64_t>(slots / kMtWarps, (n + kMtWarps - 1) / kMtWarps)));
            LaunchScope scope(nn.name, st);
            nn.kernel<<<nb, kMtWarps * 32, smem, st>>>(R, S, nullptr, n, nullptr, corr, c, fods + v0 * c, c,
                                                       status ? status + v0 : nullptr, counters, work, slot);
            cuda_check(cudaGetLastError(), "ridge_nnls_kernel launch");
        }
    });
}

}  // extern "C"
