// Single-shell constrained spherical deconvolution (CSD) on the GPU: _core.fit_csd
// (cpp/src/python/sd.cpp:171-209) over cpp/src/sd/csd.cpp. Per voxel: the linear estimate
// f = initial s, the projection M^T s, then up to max_iter solves of
// (M^T M + norm_weight I + C_S^T C_S) f = M^T s, S the rows of C where C f < threshold, until
// S repeats (Tournier et al., NeuroImage 35 (2007) 1459-1472).
//
// Mapping: one warp per voxel, voxels grid-strided over a resident grid. The system is kept
// packed (lower triangle, row-major) in the warp's shared memory. Each iteration rebuilds it as
// the Gram matrix plus C_S^T C_S, the product of the constrained rows on the FP64 tensor cores
// (mma.sync m8n8k4, the lower 8x8 tiles, rows staged eight at a time in shared memory). A
// left-looking Cholesky factorisation (one row per lane) and two column-oriented triangular solves
// follow. The amplitudes C f read C^T, so that the lanes (one direction each) load coalesced. The
// work per voxel-iteration is about |S| c^2/2 tensor-core FMAs plus c^3/6 FMAs, on data resident
// in shared memory and L1.

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "common.cuh"

namespace lar {
namespace {

constexpr int kCsdStage = 8;   // constraint rows staged per pass of the system build (two k-steps of 4)
constexpr int kCsdFixed = 6;   // tile rows of the systems of c <= 48 (lmax <= 8), all 21 lower tiles at once
constexpr int kCsdBatch = 8;   // tiles accumulated at once for larger systems

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

// The staged rows' stride: 48 for the systems of c <= 48 (six whole tile rows), else c rounded up
// to whole 8-column tiles.
__host__ __device__ inline int padded8(int c) { return c <= 8 * kCsdFixed ? 8 * kCsdFixed : (c + 7) / 8 * 8; }

// Shared memory of one warp: the packed system, f, the right-hand side, y, the staged rows
// (padded to whole 8-column tiles), then the two lists of constrained directions.
__host__ __device__ inline size_t csd_warp_bytes(int c, int k) {
    const size_t doubles = size_t(packed_count(c)) + 3 * size_t(c) + size_t(kCsdStage) * padded8(c);
    return (doubles * 8 + 2 * size_t(k) * 2 + 15) / 16 * 16;
}

// D += A B for one 8x8x4 FP64 tile on the tensor cores: a lane holds A(lane / 4, lane % 4),
// B(lane % 4, lane / 4) and D(lane / 4, 2 (lane % 4) + {0, 1}).
__device__ __forceinline__ void mma_f64(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Stages the constrained rows cur[q0, q0 + kCsdStage) of C into rows (kCsdStage, cp), zero-padded.
__device__ __forceinline__ int stage_rows(const CsdDev& P, const uint16_t* cur, int n_cur, int q0, double* rows,
                                          int cp, int lane) {
    const int nr = min(kCsdStage, n_cur - q0);
    __syncwarp();
    for (int t = lane; t < kCsdStage * cp; t += 32) {
        const int r = t / cp, j = t - r * cp;
        rows[t] = (r < nr && j < P.c) ? P.constraint[size_t(cur[q0 + r]) * P.c + j] : 0.0;
    }
    __syncwarp();
    return nr;
}

// H = gram + C_S^T C_S for c <= 48: the 21 lower tiles of six tile rows, indices fixed at compile
// time, accumulated in registers over all the constrained rows.
__device__ __forceinline__ void build_fixed(const CsdDev& P, const uint16_t* cur, int n_cur, double* rows, double* H,
                                            int lane) {
    constexpr int T = kCsdFixed, cp = 8 * kCsdFixed;
    double acc[T * (T + 1) / 2][2];
#pragma unroll
    for (int t = 0; t < T * (T + 1) / 2; ++t) acc[t][0] = acc[t][1] = 0.0;
    for (int q0 = 0; q0 < n_cur; q0 += kCsdStage) {
        stage_rows(P, cur, n_cur, q0, rows, cp, lane);
#pragma unroll
        for (int kk = 0; kk < kCsdStage; kk += 4) {
            const double* rk = rows + (kk + (lane & 3)) * cp + (lane >> 2);
            double v[T];
#pragma unroll
            for (int b = 0; b < T; ++b) v[b] = rk[8 * b];
            int t = 0;
#pragma unroll
            for (int bi = 0; bi < T; ++bi)
#pragma unroll
                for (int bj = 0; bj <= bi; ++bj, ++t) mma_f64(acc[t][0], acc[t][1], v[bi], v[bj]);
        }
    }
    const int c = P.c;
    int t = 0;
#pragma unroll
    for (int bi = 0; bi < T; ++bi)
#pragma unroll
        for (int bj = 0; bj <= bi; ++bj, ++t) {
            const int i = 8 * bi + (lane >> 2);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = 8 * bj + 2 * (lane & 3) + h;
                if (i < c && j <= i) {
                    const int e = i * (i + 1) / 2 + j;
                    H[e] = P.gram[e] + acc[t][h];
                }
            }
        }
}

// H = gram + C_S^T C_S for larger c: the lower tiles kCsdBatch at a time, the rows staged again
// for each batch.
__device__ __noinline__ void build_batched(const CsdDev& P, const uint16_t* cur, int n_cur, double* rows, double* H,
                                           int lane) {
    const int c = P.c, cp = padded8(c), tiles = cp / 8, n_tiles = tiles * (tiles + 1) / 2;
    for (int t0 = 0; t0 < n_tiles; t0 += kCsdBatch) {
        double acc[kCsdBatch][2];
        int off_r[kCsdBatch], off_c[kCsdBatch];
#pragma unroll
        for (int t = 0; t < kCsdBatch; ++t) {
            acc[t][0] = acc[t][1] = 0.0;
            int idx = t0 + t, r = 0;  // tile t0 + t of the lower triangle, row by row
            while (idx > r) {
                idx -= r + 1;
                ++r;
            }
            off_r[t] = 8 * r;
            off_c[t] = 8 * idx;
        }
        for (int q0 = 0; q0 < n_cur; q0 += kCsdStage) {
            stage_rows(P, cur, n_cur, q0, rows, cp, lane);
#pragma unroll
            for (int kk = 0; kk < kCsdStage; kk += 4) {
                const double* rk = rows + (kk + (lane & 3)) * cp + (lane >> 2);
#pragma unroll
                for (int t = 0; t < kCsdBatch; ++t)
                    if (t0 + t < n_tiles) mma_f64(acc[t][0], acc[t][1], rk[off_r[t]], rk[off_c[t]]);
            }
        }
#pragma unroll
        for (int t = 0; t < kCsdBatch; ++t) {
            if (t0 + t >= n_tiles) continue;
            const int i = off_r[t] + (lane >> 2);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = off_c[t] + 2 * (lane & 3) + h;
                if (i < c && j <= i) {
                    const int e = i * (i + 1) / 2 + j;
                    H[e] = P.gram[e] + acc[t][h];
                }
            }
        }
    }
}

template <bool FIXED>
__global__ void csd_kernel(CsdDev P, const double* __restrict__ signals, int64_t v, double* __restrict__ fods,
                           uint8_t* __restrict__ converged_out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const int c = P.c, k = P.k, npk = packed_count(c);
    unsigned char* base = smem + size_t(w) * csd_warp_bytes(c, k);
    double* H = reinterpret_cast<double*>(base);
    double* f = H + npk;
    double* rhs = f + c;
    double* y = rhs + c;
    double* rows = y + c;
    auto* list_a = reinterpret_cast<uint16_t*>(rows + kCsdStage * padded8(c));
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
            // The system: the Gram matrix plus C_S^T C_S, the constrained rows' product on the
            // tensor cores over the rows staged kCsdStage at a time (zero-padded to whole tiles
            // and k-steps).
            if (FIXED)
                build_fixed(P, cur, n_cur, rows, H, lane);
            else
                build_batched(P, cur, n_cur, rows, H, lane);
            __syncwarp();
            // Left-looking Cholesky, packed in place: column j's entries from the finished
            // columns, one row per lane; lane 0 holds the diagonal.
            for (int j = 0; j < c; ++j) {
                const double* lj = H + j * (j + 1) / 2;
                double val[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int i = j + lane + 32 * u;
                    val[u] = 0.0;
                    if (i < c) {
                        const double* li = H + i * (i + 1) / 2;
                        double a = li[j];
                        for (int q = 0; q < j; ++q) a -= li[q] * lj[q];
                        val[u] = a;
                    }
                }
                const double d = sqrt(__shfl_sync(0xffffffffu, val[0], 0));
                __syncwarp();
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int i = j + lane + 32 * u;
                    if (i < c) H[i * (i + 1) / 2 + j] = i == j ? d : val[u] / d;
                }
                for (int i = j + 64 + lane; i < c; i += 32) {
                    const double* li = H + i * (i + 1) / 2;
                    double a = li[j];
                    for (int q = 0; q < j; ++q) a -= li[q] * lj[q];
                    H[i * (i + 1) / 2 + j] = a / d;
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
        require(csd_warp_bytes(int(c), int(k)) <= 220 * 1024,
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
        const size_t per_warp = csd_warp_bytes(csd->c, csd->k);
        const int warps = int(std::max<size_t>(1, std::min<size_t>(4, (200 * 1024) / per_warp)));
        const size_t smem = per_warp * warps;
        auto kernel = csd->c <= 8 * kCsdFixed ? csd_kernel<true> : csd_kernel<false>;
        cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                   "cudaFuncSetAttribute");
        int per_sm = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, warps * 32, smem),
                   "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        const int64_t blocks = std::max<int64_t>(
            1, std::min<int64_t>((v + warps - 1) / warps, int64_t(sm_count()) * ctas_per_sm(per_sm, "csd.ctas_per_sm")));
        LaunchScope scope("csd_kernel", st);
        kernel<<<unsigned(blocks), warps * 32, smem, st>>>(P, signals, v, fods, converged);
        cuda_check(cudaGetLastError(), "csd_kernel launch");
    });
}

}  // extern "C"
