// Single-shell constrained spherical deconvolution (CSD) on the GPU: _core.fit_csd
// (cpp/src/python/sd.cpp:171-209) over cpp/src/sd/csd.cpp. Per voxel: the linear estimate
// f = initial s, the projection M^T s, then up to max_iter solves of
// (M^T M + norm_weight I + C_S^T C_S) f = M^T s, S the rows of C where C f < threshold, until
// S repeats (Tournier et al., NeuroImage 35 (2007) 1459-1472).
//
// Mapping: one warp per voxel, voxels grid-strided over a resident grid. The system is kept
// packed (lower triangle, row-major) in the warp's shared memory. Each iteration rebuilds it as
// the Gram matrix plus the outer products of the constrained rows. Those rows are staged eight at
// a time, and each lane accumulates its packed entries. A right-looking Cholesky factorisation
// and two column-oriented triangular solves follow. The amplitudes C f read C^T so that the lanes
// (one direction each) load coalesced. The work per voxel-iteration is about |S| c^2/2 + c^3/6
// FMAs on data resident in shared memory and L1; FP64-bound.

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "common.cuh"

namespace lar {
namespace {

constexpr int kCsdStage = 8;  // constraint rows staged per pass of the system build

struct CsdDev {
    const double* initial_t;     // (m, c0)
    const double* forward;       // (m, c)
    const double* constraint;    // (k, c)
    const double* constraint_t;  // (c, k)
    const double* gram;          // packed (c (c + 1) / 2): M^T M + norm_weight I
    int m, c, c0, k, max_iter;
    double threshold;
};

__host__ __device__ inline int packed_count(int c) { return c * (c + 1) / 2; }

// Shared memory of one warp: the packed system, f, the right-hand side, the staged rows, then
// the two lists of constrained directions.
__host__ __device__ inline size_t csd_warp_bytes(int c, int k) {
    const size_t doubles = size_t(packed_count(c)) + 3 * size_t(c) + size_t(kCsdStage) * c;
    return (doubles * 8 + 2 * size_t(k) * 2 + 15) / 16 * 16;
}

__global__ void csd_kernel(CsdDev P, const double* __restrict__ signals, int64_t v, double* __restrict__ fods,
                           uint8_t* __restrict__ converged_out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const int c = P.c, k = P.k, npk = packed_count(c);
    // The (row, column) of each packed entry, shared by the CTA's warps.
    auto* tri = reinterpret_cast<uint16_t*>(smem);
    for (int e = threadIdx.x; e < npk; e += blockDim.x) {
        int i = int((sqrt(8.0 * e + 1.0) - 1.0) / 2.0);
        while (i * (i + 1) / 2 > e) --i;
        while ((i + 1) * (i + 2) / 2 <= e) ++i;
        tri[e] = uint16_t((i << 8) | (e - i * (i + 1) / 2));
    }
    __syncthreads();
    unsigned char* base = smem + (size_t(npk) * 2 + 15) / 16 * 16 + size_t(w) * csd_warp_bytes(c, k);
    double* H = reinterpret_cast<double*>(base);
    double* f = H + npk;
    double* rhs = f + c;
    double* y = rhs + c;
    double* rows = y + c;
    auto* list_a = reinterpret_cast<uint16_t*>(rows + kCsdStage * c);
    uint16_t* list_b = list_a + k;
    const int64_t n_warps = int64_t(gridDim.x) * warps;
    for (int64_t voxel = int64_t(blockIdx.x) * warps + w; voxel < v; voxel += n_warps) {
        const double* s = signals + voxel * P.m;
        for (int j = lane; j < c; j += 32) {
            double pj = 0.0, fj = 0.0;
            for (int i = 0; i < P.m; ++i) {
                const double si = s[i];
                pj = fma(P.forward[size_t(i) * c + j], si, pj);
                if (j < P.c0) fj = fma(P.initial_t[size_t(i) * P.c0 + j], si, fj);
            }
            rhs[j] = pj;
            f[j] = fj;
        }
        __syncwarp();
        uint16_t* cur = list_a;
        uint16_t* prev = list_b;
        int n_prev = -1;
        bool conv = P.max_iter == 0;
        for (int it = 0; it < P.max_iter; ++it) {
            // The constrained directions, in increasing order.
            int n_cur = 0;
            for (int d0 = 0; d0 < k; d0 += 32) {
                const int d = d0 + lane;
                bool below = false;
                if (d < k) {
                    double a = 0.0;
                    for (int j = 0; j < c; ++j) a = fma(P.constraint_t[size_t(j) * k + d], f[j], a);
                    below = a < P.threshold;
                }
                const unsigned b = __ballot_sync(0xffffffffu, below);
                if (below) cur[n_cur + __popc(b & ((1u << lane) - 1u))] = uint16_t(d);
                n_cur += __popc(b);
            }
            __syncwarp();
            if (n_prev == n_cur) {
                bool same = true;
                for (int q = lane; q < n_cur; q += 32) same &= cur[q] == prev[q];
                if (__all_sync(0xffffffffu, same)) {
                    conv = true;
                    break;
                }
            }
            // The system: the Gram matrix plus the constrained rows' outer products.
            for (int e = lane; e < npk; e += 32) H[e] = P.gram[e];
            for (int q0 = 0; q0 < n_cur; q0 += kCsdStage) {
                const int nr = min(kCsdStage, n_cur - q0);
                __syncwarp();
                for (int t = lane; t < nr * c; t += 32) {
                    const int r = t / c, j = t - r * c;
                    rows[t] = P.constraint[size_t(cur[q0 + r]) * c + j];
                }
                __syncwarp();
                for (int e = lane; e < npk; e += 32) {
                    const int i = tri[e] >> 8, j = tri[e] & 0xFF;
                    double h = H[e];
                    for (int r = 0; r < nr; ++r) h = fma(rows[r * c + i], rows[r * c + j], h);
                    H[e] = h;
                }
            }
            __syncwarp();
            // Right-looking Cholesky, packed in place.
            for (int j = 0; j < c; ++j) {
                const int jj = j * (j + 1) / 2 + j;
                const double d = sqrt(H[jj]);
                __syncwarp();
                if (lane == 0) H[jj] = d;
                for (int i = j + 1 + lane; i < c; i += 32) H[i * (i + 1) / 2 + j] /= d;
                __syncwarp();
                for (int e = (j + 1) * (j + 2) / 2 + lane; e < npk; e += 32) {
                    const int i = tri[e] >> 8, q = tri[e] & 0xFF;
                    if (q > j) H[e] -= H[i * (i + 1) / 2 + j] * H[q * (q + 1) / 2 + j];
                }
                __syncwarp();
            }
            // L y = rhs, then L^T f = y.
            for (int q = lane; q < c; q += 32) y[q] = rhs[q];
            __syncwarp();
            for (int i = 0; i < c; ++i) {
                const double yi = y[i] / H[i * (i + 1) / 2 + i];
                __syncwarp();
                if (lane == 0) y[i] = yi;
                for (int r = i + 1 + lane; r < c; r += 32) y[r] -= H[r * (r + 1) / 2 + i] * yi;
                __syncwarp();
            }
            for (int i = c - 1; i >= 0; --i) {
                const int row = i * (i + 1) / 2;
                const double fi = y[i] / H[row + i];
                __syncwarp();
                if (lane == 0) f[i] = fi;
                for (int r = lane; r < i; r += 32) y[r] -= H[row + r] * fi;
                __syncwarp();
            }
            uint16_t* t = prev;
            prev = cur;
            cur = t;
            n_prev = n_cur;
        }
        for (int j = lane; j < c; j += 32) fods[voxel * c + j] = f[j];
        if (lane == 0) converged_out[voxel] = conv;
        __syncwarp();
    }
}

}  // namespace
}  // namespace lar

// The matrices of one shell's CSD fit on the device (the reference's CsdProblem,
// cpp/src/sd/csd.hpp:10-24).
struct lar_csd_s {
    int m = 0, c = 0, c0 = 0, k = 0, max_iter = 0;
    double threshold = 0.0;
    lar::DeviceArray<double> initial_t, forward, constraint, constraint_t, gram;
};

using namespace lar;

extern "C" {

int lar_csd_create(const double* initial, int64_t c0, int64_t m, const double* forward, int64_t c,
                   const double* constraint, int64_t k, double norm_weight, double threshold, int64_t max_iter,
                   lar_csd* out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        require(m > 0 && c > 0 && k > 0 && c0 >= 0, "the matrices must not be empty");
        require(c0 <= c, "initial must not have more rows than forward has columns");
        require(c <= 255 && k <= 65535, "at most 255 coefficients and 65535 constraint directions");
        require(max_iter >= 0, "max_iter must be at least 0");
        require(forward && constraint && (c0 == 0 || initial), "the matrices must not be NULL");
        const size_t tri_bytes = (size_t(packed_count(int(c))) * 2 + 15) / 16 * 16;
        require(tri_bytes + csd_warp_bytes(int(c), int(k)) <= 220 * 1024,
                "the system does not fit one warp's shared memory: too many coefficients or directions");
        auto h = std::make_unique<lar_csd_s>();
        h->m = int(m);
        h->c = int(c);
        h->c0 = int(c0);
        h->k = int(k);
        h->max_iter = int(max_iter);
        h->threshold = threshold;
        std::vector<double> it(static_cast<size_t>(m * std::max<int64_t>(c0, 1)), 0.0);
        std::vector<double> ct(static_cast<size_t>(c * k));
        std::vector<double> gram(static_cast<size_t>(packed_count(int(c))));
        for (int64_t r = 0; r < c0; ++r)
            for (int64_t i = 0; i < m; ++i) it[size_t(i * c0 + r)] = initial[r * m + i];
        for (int64_t d = 0; d < k; ++d)
            for (int64_t j = 0; j < c; ++j) ct[size_t(j * k + d)] = constraint[d * c + j];
        // cpp/src/sd/csd.cpp:13-14: M^T M with norm_weight on its diagonal.
        for (int64_t i = 0; i < c; ++i)
            for (int64_t j = 0; j <= i; ++j) {
                double acc = 0.0;
                for (int64_t r = 0; r < m; ++r) acc += forward[r * c + i] * forward[r * c + j];
                gram[size_t(i * (i + 1) / 2 + j)] = acc + (i == j ? norm_weight : 0.0);
            }
        h->initial_t.upload(it.data(), it.size());
        h->forward.upload(forward, size_t(m * c));
        h->constraint.upload(constraint, size_t(k * c));
        h->constraint_t.upload(ct.data(), ct.size());
        h->gram.upload(gram.data(), gram.size());
        *out = h.release();
    });
}

void lar_csd_destroy(lar_csd csd) { delete csd; }

int lar_fit_csd(lar_csd csd, const double* signals, int64_t v, double* fods, uint8_t* converged, void* stream) {
    return guarded([&] {
        require(csd != nullptr, "csd must not be NULL");
        require(v >= 0, "v must be at least 0");
        if (v == 0) return;
        require(signals && fods && converged, "signals, fods and converged must not be NULL");
        auto st = static_cast<cudaStream_t>(stream);
        const CsdDev P{csd->initial_t.ptr, csd->forward.ptr, csd->constraint.ptr, csd->constraint_t.ptr,
                       csd->gram.ptr, csd->m, csd->c, csd->c0, csd->k, csd->max_iter, csd->threshold};
        const size_t tri_bytes = (size_t(packed_count(csd->c)) * 2 + 15) / 16 * 16;
        const size_t per_warp = csd_warp_bytes(csd->c, csd->k);
        const int warps = int(std::max<size_t>(1, std::min<size_t>(4, (200 * 1024 - tri_bytes) / per_warp)));
        const size_t smem = tri_bytes + per_warp * warps;
        cuda_check(cudaFuncSetAttribute(csd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                   "cudaFuncSetAttribute");
        int per_sm = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, csd_kernel, warps * 32, smem),
                   "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        const int64_t blocks = std::max<int64_t>(
            1, std::min<int64_t>((v + warps - 1) / warps, int64_t(sm_count()) * ctas_per_sm(per_sm, "csd.ctas_per_sm")));
        LaunchScope scope("csd_kernel", st);
        csd_kernel<<<unsigned(blocks), warps * 32, smem, st>>>(P, signals, v, fods, converged);
        cuda_check(cudaGetLastError(), "csd_kernel launch");
    });
}

}  // extern "C"
