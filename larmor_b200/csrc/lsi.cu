// Least squares with inequality constraints (MSMT-CSD) on the GPU, one warp per voxel.
//
// Follows cpp/src/sd/lsi.cpp. The design is prepared once on the host in FP64 (make_lsi_design
// :75-125, host_la.hpp): q_t (n x m), back = P R^-1 (n x n), E = G P R^-1 with unit rows
// (k x n), its Gram E E^T (k x k) and absolute row sums. Per voxel (solve_lsi_by :301-338):
//   rotated = q_t s; f = -E rotated scaled to max |f| = 1 (or the unconstrained solution when
//   f = 0); the LDP multipliers u >= 0 by the Lawson-Hanson steps on H = E E^T + f f^T with a
//   growing Cholesky factor and Givens downdates (ldp_multipliers :253-297: the steepest
//   inactive gradient f (1 - f.u) - E E^T u enters, the first on a tie; a pivot below 1e-12 of
//   its diagonal or more than 3 k inner steps sends the voxel to the fallback); the fallback is
//   the QR-based NNLS on the explicit [E^T; f^T] (warp_nnls.cuh); then
//   x = back (scale E^T u / (1 - f.u) + rotated).
//
// Work distribution: a persistent grid of warps takes voxels from a device counter, since the
// number of active-set steps differs from voxel to voxel. The Gram matrix (shared by every
// voxel) is read row by row from L2; lanes split the k constraint columns for gradients and
// steps, the n parameters for the projections, and the factor's rows for the triangular
// solves. Each warp owns a slot of global scratch for its Cholesky factor and the fallback.

#include <algorithm>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "host_la.hpp"
#include "warp_nnls.cuh"

namespace lar {

namespace {

constexpr int kLsiWarps = 4;
constexpr int kFactorCap = 64;   // columns the Cholesky factor can hold (> n + 1)
constexpr double kMinRelativePivot = 1e-12;

struct LsiDevice {
    int m, n, k;
    const double* qt;      // (m, n): q_t transposed, row j holds column j of q_t
    const double* back;    // (n, n)
    const double* et;      // (n, k): E transposed
    const double* e;       // (k, n)
    const double* gram;    // (k, k)
    const double* abs_sums;  // (k,)
};

inline size_t lsi_slot_doubles(int n, int k) {
    return size_t(kFactorCap) * kFactorCap  // L
           + 5 * size_t(k)                  // f, u, z, fallback u, z
           + size_t(n + 1) * k              // fallback matrix
           + size_t(kFactorCap) * (n + 1)   // fallback QR columns
           + (2 * size_t(k) + 7) / 8        // flag bytes (two arrays)
           + 256;
}

struct LsiShared {
    double rot[64];
    double a[kFactorCap];    // triangular-solve vector
    double t[64];            // E^T u
    double qtau[kFactorCap], qnu[kFactorCap], qnd[kFactorCap], rv[kFactorCap + 1], res[kFactorCap + 1];
    double d[kFactorCap + 1];
    int qperm[kFactorCap];
    int act[kFactorCap];     // fallback active list
    int n_act;
    int cols[kFactorCap];    // factor columns in joining order
    int sorted[kFactorCap];  // the same, increasing
};

// H(r, c) = (E E^T)(r, c) + f_r f_c.
__device__ __forceinline__ double ldp_h(const LsiDevice& D, const double* f, int r, int c) {
    return D.gram[size_t(r) * D.k + c] + f[r] * f[c];
}

// Removes position `pos` from the lower factor L (ld = kFactorCap) of `na` columns, keeping
// L L^T of the others: a row shift and Givens rotations (cpp/src/sd/nnls.cpp:305-324).
__device__ void remove_factor_column(double* L, int na, int pos, int lane) {
    for (int j = lane; j < na; j += 32)
        for (int row = pos; row < na - 1; ++row) L[row * kFactorCap + j] = L[(row + 1) * kFactorCap + j];
    __syncwarp();
    for (int col = pos; col < na - 1; ++col) {
        const double diag = L[col * kFactorCap + col], above = L[col * kFactorCap + col + 1];
        const double len = hypot(diag, above);
        const double c = diag / len, s = above / len;
        for (int row = col + lane; row < na - 1; row += 32) {
            const double l = L[row * kFactorCap + col], r = L[row * kFactorCap + col + 1];
            L[row * kFactorCap + col] = c * l + s * r;
            L[row * kFactorCap + col + 1] = c * r - s * l;
        }
        __syncwarp();
    }
}

// z <- the solution of H_AA z_A = f_A (zero elsewhere) from the factor.
__device__ void factor_solve(const double* L, int na, const int* cols, const double* f, double* z, int k,
                             double* a, int lane) {
    for (int j = lane; j < k; j += 32) z[j] = 0.0;
    for (int p = lane; p < na; p += 32) a[p] = f[cols[p]];
    __syncwarp();
    for (int j = 0; j < na; ++j) {
        const double aj = a[j] / L[j * kFactorCap + j];
        __syncwarp();
        if (lane == 0) a[j] = aj;
        for (int r = j + 1 + lane; r < na; r += 32) a[r] -= L[r * kFactorCap + j] * aj;
        __syncwarp();
    }
    for (int j = na - 1; j >= 0; --j) {
        const double aj = a[j] / L[j * kFactorCap + j];
        __syncwarp();
        if (lane == 0) a[j] = aj;
        for (int r = lane; r < j; r += 32) a[r] -= L[j * kFactorCap + r] * aj;
        __syncwarp();
    }
    for (int p = lane; p < na; p += 32) z[cols[p]] = a[p];
    __syncwarp();
}

// The LDP multipliers (cpp/src/sd/lsi.cpp:253-297). Returns false when a Cholesky pivot fails
// or the inner steps run out (the caller falls back to the QR-based NNLS).
__device__ bool ldp_multipliers(const LsiDevice& D, const double* f, double* u, double* z, uint8_t* flag,
                                double* L, LsiShared& sh, int* outer_steps, int lane) {
    const int k = D.k;
    double norm1 = 0.0;
    for (int j = lane; j < k; j += 32) {
        norm1 = fmax(norm1, D.abs_sums[j] + fabs(f[j]));
        u[j] = 0.0;
        z[j] = 0.0;
        flag[j] = 0;
    }
    norm1 = warp_max(norm1);
    const double tol = 10.0 * kEps64 * norm1 * double(max(D.n + 1, k));
    const int max_inner = 3 * k;
    int na = 0, inner = 0, outer = 0;
    __syncwarp();
    for (;;) {
        double fu = 0.0;
        for (int j = lane; j < k; j += 32) fu += f[j] * u[j];
        fu = warp_sum(fu);
        // Steepest inactive gradient f (1 - f.u) - sum_c u_c (E E^T)_c, columns c in increasing order.
        double bv = 0.0;
        int bi = -1;
        for (int j = lane; j < k; j += 32) {
            if (flag[j]) continue;
            double g = f[j] * (1.0 - fu);
            for (int q = 0; q < na; ++q) {
                const int c = sh.sorted[q];
                const double uc = u[c];
                if (uc != 0.0) g -= uc * D.gram[size_t(c) * k + j];
            }
            if (bi < 0 || g > bv) { bv = g; bi = j; }
        }
        const int e = warp_argmax_first(bv, bi);
        const double ge = e >= 0 ? __shfl_sync(0xffffffffu, bv, e & 31) : 0.0;
        if (e < 0 || ge <= tol) break;
        ++outer;
        if (na >= kFactorCap) { *outer_steps = outer; return false; }
        // Append e to the factor: L w = H_{A,e}, pivot = H_ee - w.w.
        double* w = sh.a;
        for (int r = lane; r < na; r += 32) w[r] = ldp_h(D, f, sh.cols[r], e);
        __syncwarp();
        for (int j = 0; j < na; ++j) {
            const double wj = w[j] / L[j * kFactorCap + j];
            __syncwarp();
            if (lane == 0) w[j] = wj;
            for (int r = j + 1 + lane; r < na; r += 32) w[r] -= L[r * kFactorCap + j] * wj;
            __syncwarp();
        }
        double sq = 0.0;
        for (int r = lane; r < na; r += 32) sq += w[r] * w[r];
        sq = warp_sum(sq);
        const double hee = ldp_h(D, f, e, e);
        const double pivot = hee - sq;
        if (!(pivot > kMinRelativePivot * hee)) { *outer_steps = outer; return false; }
        for (int r = lane; r < na; r += 32) L[na * kFactorCap + r] = w[r];
        __syncwarp();
        if (lane == 0) {
            L[na * kFactorCap + na] = sqrt(pivot);
            sh.cols[na] = e;
            int q = na;
            while (q > 0 && sh.sorted[q - 1] > e) { sh.sorted[q] = sh.sorted[q - 1]; --q; }
            sh.sorted[q] = e;
            flag[e] = 1;
        }
        ++na;
        __syncwarp();
        factor_solve(L, na, sh.cols, f, z, k, sh.a, lane);
        for (;;) {
            // Blocking step over active columns with z <= 0, the first on a tie.
            double sv = 0.0;
            int si = -1;
            for (int q = lane; q < na; q += 32) {
                const int col = sh.cols[q];
                if (z[col] > 0.0) continue;
                const double dist = u[col] - z[col];
                const double st = dist > 0.0 ? u[col] / dist : 0.0;
                if (si < 0 || st < sv || (st == sv && col < si)) { sv = st; si = col; }
            }
            double step;
            const int b = warp_argmin_first(sv, si, &step);
            if (b < 0) break;
            if (++inner > max_inner) { *outer_steps = outer; return false; }
            for (int q = lane; q < na; q += 32) {
                const int col = sh.cols[q];
                u[col] += step * (z[col] - u[col]);
            }
            __syncwarp();
            if (lane == 0) {
                u[b] = 0.0;
                for (int q = 0; q < na; ++q) {
                    const int col = sh.cols[q];
                    if (col == b || fabs(u[col]) < tol) {
                        flag[col] = 0;
                        u[col] = 0.0;
                    }
                }
            }
            __syncwarp();
            // keep(): drop the factor columns that left, from the last position to the first.
            for (int pos = na - 1; pos >= 0; --pos) {
                const int col = sh.cols[pos];
                if (flag[col]) continue;
                remove_factor_column(L, na, pos, lane);
                if (lane == 0) {
                    for (int q = pos; q < na - 1; ++q) sh.cols[q] = sh.cols[q + 1];
                    int w2 = 0;
                    for (int q = 0; q < na; ++q)
                        if (sh.sorted[q] != col) sh.sorted[w2++] = sh.sorted[q];
                }
                --na;
                __syncwarp();
            }
            factor_solve(L, na, sh.cols, f, z, k, sh.a, lane);
        }
        for (int j = lane; j < k; j += 32) u[j] = z[j];
        __syncwarp();
    }
    *outer_steps = outer;
    return true;
}

__global__ void __launch_bounds__(kLsiWarps * 32) lsi_kernel(LsiDevice D, const double* __restrict__ signals,
                                                             int64_t v, int only_qr, int* queue,
                                                             double* __restrict__ workspace, size_t slot_doubles,
                                                             double* __restrict__ x, uint8_t* __restrict__ converged,
                                                             uint8_t* __restrict__ status,
                                                             int32_t* __restrict__ outer_out,
                                                             uint8_t* __restrict__ active_out) {
    __shared__ LsiShared shared[kLsiWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    LsiShared& sh = shared[warp];
    const int m = D.m, n = D.n, k = D.k, rows = n + 1;
    double* slot = workspace + (size_t(blockIdx.x) * kLsiWarps + warp) * slot_doubles;
    double* L = slot;
    double* f = L + kFactorCap * kFactorCap;
    double* u = f + k;
    double* z = u + k;
    double* u2 = z + k;
    double* z2 = u2 + k;
    double* cmat = z2 + k;                        // (rows, k)
    double* sub = cmat + size_t(rows) * k;        // (kFactorCap, rows)
    uint8_t* flag = reinterpret_cast<uint8_t*>(sub + size_t(kFactorCap) * rows);
    uint8_t* flag2 = flag + k;
    for (;;) {
        int64_t voxel = 0;
        if (lane == 0) voxel = atomicAdd(queue, 1);
        voxel = __shfl_sync(0xffffffffu, voxel, 0);
        if (voxel >= v) break;
        const double* s = signals + voxel * m;
        // rotated = q_t s.
        for (int i = lane; i < n; i += 32) {
            double acc = 0.0;
            for (int j = 0; j < m; ++j) acc += D.qt[size_t(j) * n + i] * s[j];
            sh.rot[i] = acc;
        }
        __syncwarp();
        // f = -E rotated, scaled by max |f|.
        double scale = 0.0;
        for (int j = lane; j < k; j += 32) {
            double acc = 0.0;
            for (int i = 0; i < n; ++i) acc += D.et[size_t(i) * k + j] * sh.rot[i];
            f[j] = -acc;
            scale = fmax(scale, fabs(acc));
        }
        scale = warp_max(scale);
        __syncwarp();
        uint8_t st = 0, conv = 1;
        int outer = 0;
        if (!(scale > 0.0)) {
            // f = 0: the unconstrained solution back * rotated.
            for (int i = lane; i < n; i += 32) {
                double acc = 0.0;
                for (int j = 0; j < n; ++j) acc += D.back[size_t(i) * n + j] * sh.rot[j];
                x[voxel * n + i] = acc;
            }
            if (active_out)
                for (int j = lane; j < k; j += 32) active_out[voxel * k + j] = 0;
            st = 2;
        } else {
            for (int j = lane; j < k; j += 32) f[j] /= scale;
            __syncwarp();
            const double* mult = u;
            bool fast = !only_qr && ldp_multipliers(D, f, u, z, flag, L, sh, &outer, lane);
            if (!fast) {
                // QR-based NNLS on the explicit [E^T; f^T] (cpp/src/sd/lsi.cpp:321-332).
                double colmax = 0.0;
                for (int j = lane; j < k; j += 32) {
                    double cs = fabs(f[j]);
                    for (int i = 0; i < n; ++i) {
                        const double eij = D.e[size_t(j) * n + i];
                        cmat[size_t(i) * k + j] = eij;
                        cs += fabs(eij);
                    }
                    cmat[size_t(n) * k + j] = f[j];
                    colmax = fmax(colmax, cs);
                }
                colmax = warp_max(colmax);
                for (int r = lane; r < rows; r += 32) sh.d[r] = (r == n) ? 1.0 : 0.0;
                __syncwarp();
                const double tol = 10.0 * kEps64 * colmax * double(max(rows, k));
                NnlsScratch ns{u2, z2, flag2, sh.act, &sh.n_act, sh.res,
                               QrScratch{sub, sh.qtau, sh.qnu, sh.qnd, sh.qperm, sh.rv}, kFactorCap};
                const int outcome = warp_nnls_explicit(cmat, rows, k, sh.d, tol, 3 * k, ns, lane);
                conv = outcome == 1 ? 1 : 0;
                if (outcome < 0)
                    for (int j = lane; j < k; j += 32) u2[j] = 0.0;
                __syncwarp();
                mult = u2;
                st = 1;
            }
            // x = back (scale E^T u / (1 - f.u) + rotated).
            double fu = 0.0;
            for (int j = lane; j < k; j += 32) fu += f[j] * mult[j];
            fu = warp_sum(fu);
            for (int i = lane; i < n; i += 32) {
                double acc = 0.0;
                for (int j = 0; j < k; ++j) {
                    const double mj = mult[j];
                    if (mj != 0.0) acc += D.e[size_t(j) * n + i] * mj;
                }
                sh.t[i] = scale * acc / (1.0 - fu) + sh.rot[i];
            }
            __syncwarp();
            for (int i = lane; i < n; i += 32) {
                double acc = 0.0;
                for (int j = 0; j < n; ++j) acc += D.back[size_t(i) * n + j] * sh.t[j];
                x[voxel * n + i] = acc;
            }
            if (active_out)
                for (int j = lane; j < k; j += 32) active_out[voxel * k + j] = mult[j] != 0.0 ? 1 : 0;
        }
        if (lane == 0) {
            converged[voxel] = conv;
            if (status) status[voxel] = st;
            if (outer_out) outer_out[voxel] = outer;
        }
        __syncwarp();
    }
}

}  // namespace

}  // namespace lar

struct lar_lsi_design_s {
    lar::host::LsiDesignHost host;
    lar::DeviceArray<double> qt, back, et, e, gram, abs_sums;
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    ~lar_lsi_design_s() {
        if (scratch) cudaFree(scratch);
    }
};

using namespace lar;

extern "C" {

int lar_lsi_design_create(const double* a, int64_t m, int64_t n, const double* g, int64_t k, double ridge,
                          lar_lsi_design* out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        require(a != nullptr && m > 0 && n > 0, "a must be a non-empty (m, n) array");
        require(g != nullptr && k > 0, "g must be a non-empty (k, n) array");
        require(n + 1 <= 64, "the LSI fit takes at most 63 parameters");
        require(m <= (int64_t(1) << 20) && k <= (int64_t(1) << 16), "the LSI design is too large");
        auto h = std::make_unique<lar_lsi_design_s>();
        h->host = host::prepare_lsi_design(a, m, n, g, k, ridge);
        const auto& d = h->host;
        std::vector<double> qt(size_t(m * n)), et(size_t(n * k));
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < m; ++j) qt[size_t(j * n + i)] = d.q_t[size_t(i * m + j)];
        for (int64_t j = 0; j < k; ++j)
            for (int64_t i = 0; i < n; ++i) et[size_t(i * k + j)] = d.e[size_t(j * n + i)];
        h->qt.upload(qt.data(), qt.size());
        h->back.upload(d.back.data(), d.back.size());
        h->et.upload(et.data(), et.size());
        h->e.upload(d.e.data(), d.e.size());
        h->gram.upload(d.gram.data(), d.gram.size());
        h->abs_sums.upload(d.abs_sums.data(), d.abs_sums.size());
        *out = h.release();
    });
}

void lar_lsi_design_destroy(lar_lsi_design design) { delete design; }

int lar_lsi_design_matrices(lar_lsi_design design, double* q_t, double* back, double* e, double* gram,
                            double* abs_sums) {
    return guarded([&] {
        require(design != nullptr, "design must not be NULL");
        const auto& d = design->host;
        if (q_t) std::copy(d.q_t.begin(), d.q_t.end(), q_t);
        if (back) std::copy(d.back.begin(), d.back.end(), back);
        if (e) std::copy(d.e.begin(), d.e.end(), e);
        if (gram) std::copy(d.gram.begin(), d.gram.end(), gram);
        if (abs_sums) std::copy(d.abs_sums.begin(), d.abs_sums.end(), abs_sums);
    });
}

int lar_fit_lsi(lar_lsi_design design, const double* signals, int64_t v, int only_qr, double* x,
                uint8_t* converged, uint8_t* status, int32_t* outer, uint8_t* active, void* stream) {
    return guarded([&] {
        require(design != nullptr, "design must not be NULL");
        require(v >= 0, "v must be at least 0");
        if (v == 0) return;
        require(signals && x && converged, "signals, x and converged must not be NULL");
        const auto& h = design->host;
        const int slots = int(std::max<int64_t>(kLsiWarps, std::min<int64_t>(
                                                              (v + kLsiWarps - 1) / kLsiWarps * kLsiWarps,
                                                              int64_t(sm_count()) * 8)));
        const size_t slot = lsi_slot_doubles(int(h.n), int(h.k));
        const size_t need = 256 + size_t(slots) * slot * sizeof(double);
        if (need > design->scratch_bytes) {
            if (design->scratch) cuda_check(cudaFree(design->scratch), "cudaFree");
            design->scratch = nullptr;
            design->scratch_bytes = 0;
            cuda_check(cudaMalloc(&design->scratch, need), "cudaMalloc (LSI scratch)");
            design->scratch_bytes = need;
        }
        auto st = static_cast<cudaStream_t>(stream);
        char* base = static_cast<char*>(design->scratch);
        cuda_check(cudaMemsetAsync(base, 0, sizeof(int), st), "cudaMemsetAsync");
        LsiDevice D{int(h.m), int(h.n), int(h.k), design->qt.ptr, design->back.ptr, design->et.ptr,
                    design->e.ptr, design->gram.ptr, design->abs_sums.ptr};
        lsi_kernel<<<slots / kLsiWarps, kLsiWarps * 32, 0, st>>>(
            D, signals, v, only_qr, reinterpret_cast<int*>(base), reinterpret_cast<double*>(base + 256), slot, x,
            converged, status, outer, active);
        cuda_check(cudaGetLastError(), "lsi_kernel launch");
    });
}

}  // extern "C"
