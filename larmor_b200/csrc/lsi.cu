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
// Work distribution: a persistent grid of warps, as many as fit on the SMs at once, takes voxels
// from a device counter, since the number of active-set steps differs from voxel to voxel. Each
// warp keeps its bounds, multipliers, candidate and packed Cholesky factor in shared memory
// (warp_chol.cuh: the triangular solves run in registers with shuffles); the Gram matrix
// (shared by every voxel) is read row by row from L2. Lanes split the k constraint columns for
// gradients and steps, the n parameters for the projections. The rare QR fallback works in a
// per-warp slot of global scratch.

#include <algorithm>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "host_la.hpp"
#include "plain_fp32.cuh"
#include "warp_chol.cuh"
#include "warp_nnls.cuh"

namespace lar {

namespace {

constexpr int kLsiWarps = 4;
constexpr int kFactorCap = 64;   // active columns the Cholesky factor can hold (>= n + 1)
constexpr double kMinRelativePivot = 1e-12;
constexpr int kColsPerLane = 16;  // constraint columns a lane holds gradients for (k <= 512)

struct LsiDevice {
    int m, n, k;
    const double* qt;      // (m, n): q_t transposed, row j holds column j of q_t
    const double* back;    // (n, n)
    const double* et;      // (n, k): E transposed
    const double* e;       // (k, n)
    const double* gram;    // (k, k)
    const double* abs_sums;  // (k,)
};

// Global scratch of one warp: the Cholesky factor and its inverse, the QR-based fallback's
// explicit matrix and workspaces.
inline size_t lsi_slot_doubles(int n, int k) {
    return 2 * size_t(packed_size(kFactorCap))  // L, M
           + 2 * size_t(k)                  // fallback u, z
           + size_t(n + 1) * k              // fallback matrix
           + size_t(kFactorCap) * (n + 1)   // fallback QR columns
           + (size_t(k) + 7) / 8            // fallback flags
           + 64;
}

// Shared memory of one warp: bounds f, multipliers u, candidate z (k each), the factor's vectors
// h, w, y (cap each), small vectors, then the int and byte arrays.
struct LsiWarpLayout {
    int k, cap;
    __host__ __device__ size_t doubles() const { return 3 * size_t(k) + 3 * size_t(cap) + 4 * 64; }
    __host__ __device__ size_t ints() const { return 2 * size_t(cap) + 2 * 64 + 8; }
    __host__ __device__ size_t bytes() const {
        return (doubles() * sizeof(double) + ints() * sizeof(int) + size_t(k) + 15) / 16 * 16;
    }
};

struct LsiWarp {
    double *f, *u, *z, *h, *wv, *y, *L, *M, *rot, *t, *d, *res;
    int *cols, *sorted, *act, *perm;
    int* n_act;
    uint8_t* flag;
};

__device__ LsiWarp carve_lsi(unsigned char* base, const LsiWarpLayout& lay) {
    LsiWarp w;
    double* p = reinterpret_cast<double*>(base);
    w.f = p; p += lay.k;
    w.u = p; p += lay.k;
    w.z = p; p += lay.k;
    w.h = p; p += lay.cap;
    w.wv = p; p += lay.cap;
    w.y = p; p += lay.cap;
    w.L = nullptr;  // in the warp's global slot
    w.M = nullptr;
    w.rot = p; p += 64;
    w.t = p; p += 64;
    w.d = p; p += 64;
    w.res = p; p += 64;
    int* q = reinterpret_cast<int*>(p);
    w.cols = q; q += lay.cap;
    w.sorted = q; q += lay.cap;
    w.act = q; q += 64;
    w.perm = q; q += 64;
    w.n_act = q; q += 8;
    w.flag = reinterpret_cast<uint8_t*>(q);
    return w;
}

// The small per-warp QR state of the fallback.
struct LsiQrShared {
    double tau[kFactorCap], nu[kFactorCap], nd[kFactorCap], rv[kFactorCap + 1];
};

// The LDP multipliers (cpp/src/sd/lsi.cpp:253-297) in w.u. Returns false when a Cholesky pivot
// fails or the inner steps run out (the caller falls back to the QR-based NNLS). The factor of
// H_AA is kept with its inverse (warp_chol.cuh, InvFactor): y = M f_A grows with each append, a
// solve is one triangular matrix-vector product, and a removal is the Givens downdate of both.
// Inlined into the kernel with every argument by value, so that its state stays in registers.
template <int CPL>
__device__ __forceinline__ bool ldp_multipliers(const LsiDevice D, const LsiWarp w, int cap, int* outer_steps,
                                                int lane) {
    constexpr int VPL = kFactorCap / 32;
    const int k = D.k;
    const InvFactor fac{w.L, w.M, w.h, w.wv, w.y, w.cols, cap};
    double norm1 = 0.0;
    for (int j = lane; j < k; j += 32) {
        norm1 = fmax(norm1, D.abs_sums[j] + fabs(w.f[j]));
        w.u[j] = 0.0;
        w.z[j] = 0.0;
        w.flag[j] = 0;
    }
    norm1 = warp_max(norm1);
    const double tol = 10.0 * kEps64 * norm1 * double(max(D.n + 1, k));
    const int max_inner = 3 * k;
    int na = 0, inner = 0, outer = 0;
    __syncwarp();
    auto solve = [&]() {
        if (na <= 32) inv_solve<1>(fac, na, w.z, k, lane);
        else inv_solve<VPL>(fac, na, w.z, k, lane);
    };
    for (;;) {
        double fu = 0.0;
        for (int j = lane; j < k; j += 32) fu += w.f[j] * w.u[j];
        fu = warp_sum(fu);
        // Steepest inactive gradient f (1 - f.u) - sum_c u_c (E E^T)_c over the active columns in
        // increasing order (u is zero elsewhere), the first on a tie.
        double g[CPL];
#pragma unroll
        for (int t = 0; t < CPL; ++t) {
            const int j = lane + 32 * t;
            g[t] = j < k ? w.f[j] * (1.0 - fu) : 0.0;
        }
        for (int q = 0; q < na; ++q) {
            const int c = w.sorted[q];
            const double uc = w.u[c];
            if (uc == 0.0) continue;
            const double* row = D.gram + size_t(c) * k;
#pragma unroll
            for (int t = 0; t < CPL; ++t) {
                const int j = lane + 32 * t;
                if (j < k) g[t] -= uc * row[j];
            }
        }
        double bv = 0.0;
        int bi = -1;
#pragma unroll
        for (int t = 0; t < CPL; ++t) {
            const int j = lane + 32 * t;
            if (j < k && !w.flag[j] && (bi < 0 || g[t] > bv)) { bv = g[t]; bi = j; }
        }
        const int e = warp_argmax_first(bv, bi);
        const double ge = e >= 0 ? __shfl_sync(0xffffffffu, bv, e & 31) : 0.0;
        if (e < 0 || ge <= tol) break;
        ++outer;
        // H(cols[r], e) = (E E^T)(cols[r], e) + f_cols[r] f_e, then append.
        const double fe = w.f[e];
        for (int r = lane; r < na; r += 32) {
            const int c = w.cols[r];
            w.h[r] = D.gram[size_t(c) * k + e] + w.f[c] * fe;
        }
        __syncwarp();
        const double hee = D.gram[size_t(e) * k + e] + fe * fe;
        const bool appended = na < 32 ? inv_append<1>(fac, na, hee, fe, e, kMinRelativePivot, lane)
                                      : inv_append<VPL>(fac, na, hee, fe, e, kMinRelativePivot, lane);
        if (!appended) {
            *outer_steps = outer;
            return false;
        }
        if (lane == 0) {
            w.flag[e] = 1;
            int q = na - 1;
            while (q > 0 && w.sorted[q - 1] > e) { w.sorted[q] = w.sorted[q - 1]; --q; }
            w.sorted[q] = e;
        }
        __syncwarp();
        solve();
        for (;;) {
            // Blocking step over active columns with z <= 0, the first on a tie.
            double sv = 0.0;
            int si = -1;
            for (int q = lane; q < na; q += 32) {
                const int col = w.sorted[q];
                if (w.z[col] > 0.0) continue;
                const double dist = w.u[col] - w.z[col];
                const double st = dist > 0.0 ? w.u[col] / dist : 0.0;
                if (si < 0 || st < sv) { sv = st; si = col; }
            }
            double step;
            const int b = warp_argmin_first(sv, si, &step);
            if (b < 0) break;
            if (++inner > max_inner) {
                *outer_steps = outer;
                return false;
            }
            for (int q = lane; q < na; q += 32) {
                const int col = w.sorted[q];
                w.u[col] += step * (w.z[col] - w.u[col]);
            }
            __syncwarp();
            // The blocking coefficient leaves, and so does any that rounding left near zero.
            if (lane == 0) {
                w.u[b] = 0.0;
                int kept = 0;
                for (int q = 0; q < na; ++q) {
                    const int col = w.sorted[q];
                    if (col == b || fabs(w.u[col]) < tol) {
                        w.flag[col] = 0;
                        w.u[col] = 0.0;
                    } else {
                        w.sorted[kept++] = col;
                    }
                }
            }
            __syncwarp();
            // keep(): drop the factor columns that left, from the last position to the first.
            for (int pos = na - 1; pos >= 0; --pos) {
                if (w.flag[w.cols[pos]]) continue;
                if (na <= 32) inv_remove<1>(fac, na, pos, lane);
                else inv_remove<VPL>(fac, na, pos, lane);
                --na;
                __syncwarp();
            }
            solve();
        }
        for (int j = lane; j < k; j += 32) w.u[j] = w.z[j];
        __syncwarp();
    }
    *outer_steps = outer;
    return true;
}

template <int CPL>
__global__ void __launch_bounds__(kLsiWarps * 32, 4) lsi_kernel(LsiDevice D, const double* __restrict__ signals,
                                                             int64_t v, int only_qr, int* queue, int cap,
                                                             double* __restrict__ workspace, size_t slot_doubles,
                                                             double* __restrict__ x, uint8_t* __restrict__ converged,
                                                             uint8_t* __restrict__ status,
                                                             int32_t* __restrict__ outer_out,
                                                             uint8_t* __restrict__ active_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ LsiQrShared qr_shared[kLsiWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const LsiWarpLayout lay{D.k, cap};
    LsiQrShared& qsh = qr_shared[warp];
    const int m = D.m, n = D.n, k = D.k, rows = n + 1;
    double* slot = workspace + (size_t(blockIdx.x) * kLsiWarps + warp) * slot_doubles;
    LsiWarp w = carve_lsi(smem_raw + warp * lay.bytes(), lay);
    w.L = slot;
    w.M = slot + packed_size(kFactorCap);
    double* u2 = w.M + packed_size(kFactorCap);
    double* z2 = u2 + k;
    double* cmat = z2 + k;                        // (rows, k)
    double* sub = cmat + size_t(rows) * k;        // (kFactorCap, rows)
    uint8_t* flag2 = reinterpret_cast<uint8_t*>(sub + size_t(kFactorCap) * rows);
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
            w.rot[i] = acc;
        }
        __syncwarp();
        // f = -E rotated, scaled by max |f|.
        double scale = 0.0;
        for (int j = lane; j < k; j += 32) {
            double acc = 0.0;
            for (int i = 0; i < n; ++i) acc += D.et[size_t(i) * k + j] * w.rot[i];
            w.f[j] = -acc;
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
                for (int j = 0; j < n; ++j) acc += D.back[size_t(i) * n + j] * w.rot[j];
                x[voxel * n + i] = acc;
            }
            if (active_out)
                for (int j = lane; j < k; j += 32) active_out[voxel * k + j] = 0;
            st = 2;
        } else {
            for (int j = lane; j < k; j += 32) w.f[j] /= scale;
            __syncwarp();
            const double* mult = w.u;
            const bool fast = !only_qr && ldp_multipliers<CPL>(D, w, cap, &outer, lane);
            if (!fast) {
                // QR-based NNLS on the explicit [E^T; f^T] (cpp/src/sd/lsi.cpp:321-332).
                double colmax = 0.0;
                for (int j = lane; j < k; j += 32) {
                    double cs = fabs(w.f[j]);
                    for (int i = 0; i < n; ++i) {
                        const double eij = D.e[size_t(j) * n + i];
                        cmat[size_t(i) * k + j] = eij;
                        cs += fabs(eij);
                    }
                    cmat[size_t(n) * k + j] = w.f[j];
                    colmax = fmax(colmax, cs);
                }
                colmax = warp_max(colmax);
                for (int r = lane; r < rows; r += 32) w.d[r] = (r == n) ? 1.0 : 0.0;
                __syncwarp();
                const double tol = 10.0 * kEps64 * colmax * double(max(rows, k));
                NnlsScratch ns{u2, z2, flag2, w.act, w.n_act, w.res,
                               QrScratch{sub, qsh.tau, qsh.nu, qsh.nd, w.perm, qsh.rv}, kFactorCap};
                const int outcome = warp_nnls_explicit(cmat, rows, k, w.d, tol, 3 * k, ns, lane);
                conv = outcome == 1 ? 1 : 0;
                if (outcome < 0)
                    for (int j = lane; j < k; j += 32) u2[j] = 0.0;
                __syncwarp();
                mult = u2;
                st = 1;
            }
            // x = back (scale E^T u / (1 - f.u) + rotated).
            double fu = 0.0;
            for (int j = lane; j < k; j += 32) fu += w.f[j] * mult[j];
            fu = warp_sum(fu);
            for (int i = lane; i < n; i += 32) {
                double acc = 0.0;
                for (int j = 0; j < k; ++j) {
                    const double mj = mult[j];
                    if (mj != 0.0) acc += D.e[size_t(j) * n + i] * mj;
                }
                w.t[i] = scale * acc / (1.0 - fu) + w.rot[i];
            }
            __syncwarp();
            for (int i = lane; i < n; i += 32) {
                double acc = 0.0;
                for (int j = 0; j < n; ++j) acc += D.back[size_t(i) * n + j] * w.t[j];
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
    // FP32 copies for the plain single-precision fit (the comparison baseline).
    lar::DeviceArray<float> qt32, back32, et32, e32, gram32, abs_sums32;
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
        require(k <= 512, "the LSI fit takes at most 512 constraints");
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
        auto upload32 = [](DeviceArray<float>& dst, const std::vector<double>& src) {
            const std::vector<float> f(src.begin(), src.end());
            dst.upload(f.data(), f.size());
        };
        upload32(h->qt32, qt);
        upload32(h->back32, d.back);
        upload32(h->et32, et);
        upload32(h->e32, d.e);
        upload32(h->gram32, d.gram);
        upload32(h->abs_sums32, d.abs_sums);
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
        const int cap = int(std::min<int64_t>(kFactorCap, (h.n + 1 + 7) / 8 * 8));
        const LsiWarpLayout lay{int(h.k), cap};
        const size_t smem = lay.bytes() * kLsiWarps;
        require(smem <= 200 * 1024, "the LSI problem has too many constraints for the shared-memory solver");
        // Constraint columns per lane: 10 up to 320 constraints (302 with the 300-direction grid),
        // else kColsPerLane.
        auto kernel = h.k <= 320 ? lsi_kernel<10> : lsi_kernel<kColsPerLane>;
        cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                   "cudaFuncSetAttribute");
        int per_sm = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kLsiWarps * 32, smem),
                   "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((v + kLsiWarps - 1) / kLsiWarps,
                                                                      int64_t(sm_count()) * ctas_per_sm(per_sm, "lsi.ctas_per_sm")));
        const int slots = int(blocks) * kLsiWarps;
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
        LaunchScope scope("lsi_kernel", st);
        kernel<<<unsigned(blocks), kLsiWarps * 32, smem, st>>>(
            D, signals, v, only_qr, reinterpret_cast<int*>(base), cap, reinterpret_cast<double*>(base + 256), slot,
            x, converged, status, outer, active);
        cuda_check(cudaGetLastError(), "lsi_kernel launch");
    });
}

int lar_fit_lsi_plain_fp32(lar_lsi_design design, const float* signals, int64_t v, float* x, uint8_t* status,
                           void* stream) {
    return guarded([&] {
        require(design != nullptr, "design must not be NULL");
        require(v >= 0, "v must be at least 0");
        if (v == 0) return;
        require(signals && x, "signals and x must not be NULL");
        const auto& h = design->host;
        const PlainLsi D{int(h.m), int(h.n), int(h.k), design->qt32.ptr, design->back32.ptr, design->et32.ptr,
                         design->e32.ptr, design->gram32.ptr, design->abs_sums32.ptr};
        launch_plain_lsi(D, signals, v, x, status, static_cast<cudaStream_t>(stream));
    });
}

}  // extern "C"
