// Damped Richardson-Lucy (dRL) deconvolution on the GPU: FodSolver.drl + fit_single_tissue
// (cpp/src/python/sd.cpp:127-145, cpp/src/sd/solver.cpp:9-12) over damped_richardson_lucy
// (cpp/src/sd/drl.cpp:39-100). Dell'Acqua F et al., NeuroImage 49 (2010) 1446-1458.
//
// Each voxel starts every amplitude at `init`. An iteration computes the prediction p = K^T K f
// and moves each amplitude to max(f (1 + u (K^T s - p) / (p + 1e-16)), 1e-6). The damping is
// u = 1 - strength (1 - f^8 / (f^8 + nu^8)), with strength = max(1 - 4 std(s), 0). A voxel
// stops when its amplitudes change in total by no more than 1e-4 of its largest signal value.
//
// Mapping: a CTA of 8 warps takes 8 RT voxels at a time (32 up to 320 directions, 8 up to 640)
// and keeps their FODs F (8 RT, c) and K^T s (8 RT, c) in shared memory for all their
// iterations. An iteration is one product F K^T K on the FP64 tensor cores: mma.sync m8n8k4
// over the RT 8-voxel row tiles and the 8-direction column tiles, which the warps take
// round-robin. K^T K (c x c, 720 KB at c = 300) stays in L2 and streams through each CTA once
// per iteration for its voxels, 8 rows at a time, into a double-buffered shared-memory stage by
// cp.async while the tensor cores work on the previous 8 rows. The rows of F, K^T s and the
// stage are padded, so the fragment loads of a warp fall in distinct banks. The update is the
// epilogue, on the accumulators, after a barrier, since every warp reads all of F. Each voxel's
// change is reduced in a fixed order, so the stopping test does not depend on the schedule.
// Converged voxels keep their FOD while the tile's others iterate.
//
// Up to 64 directions the whole K^T K (at most 36 KB) is loaded once per CTA instead, and an
// iteration needs one barrier; the CTA then fits in half an SM.
//
// The multi-tissue rounds (GRL, cpp/src/sd/multi_tissue.cpp:40-95) run the same solve on a list
// of voxels whose signal is the anisotropic part max(s w - W_iso f_iso, 0) of the round.

#include <algorithm>
#include <cmath>

#include <math_constants.h>

#include "common.cuh"
#include "drl.cuh"

namespace lar {
namespace {

constexpr int kDrlWarps = 8;
constexpr int kDrlChunk = 8;   // rows of K^T K per stage (two k-steps), one per warp
// The two tilings: RT 8-voxel row tiles per CTA, MAXCT column tiles per warp, for
// c <= 8 * kDrlWarps * MAXCT directions.
constexpr int kNarrowRt = 4, kNarrowCt = 5;   // 32 voxels, c <= 320
constexpr int kWideRt = 1, kWideCt = 10;      // 8 voxels, c <= 640
constexpr int kNarrowMaxC = 8 * kDrlWarps * kNarrowCt;
constexpr int kWideMaxC = 8 * kDrlWarps * kWideCt;
// Up to 64 directions (the low-resolution kernels of the multi-tissue rounds) all of K^T K stays
// in shared memory for the CTA's life: 32 voxels, one column tile per warp, two CTAs per SM.
constexpr int kResidentMaxC = 8 * kDrlWarps;

// Row strides (doubles) of F and K^T s, and of the K^T K stage, for cp columns: the padding puts
// the 8 rows of an A fragment, and the 4 rows of a B fragment, in different banks.
__host__ __device__ inline int drl_ldf(int cp) { return cp + 4; }
__host__ __device__ inline int drl_ldg(int cp) { return cp + 8; }

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async16(double* dst, const double* src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N));
}

__device__ __forceinline__ double power_8(double x) {
    const double x2 = x * x, x4 = x2 * x2;
    return x4 * x4;
}

__device__ __forceinline__ void mma_f64(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Entry i of the signal of `voxel` that dRL deconvolves.
__device__ __forceinline__ double signal_at(const DrlSignal& S, int64_t voxel, int i) {
    const double si = S.s[voxel * S.m + i];
    if (S.w == nullptr) return si;
    const double ws = __dmul_rn(si, S.w[i]);
    double r = 0.0;
    for (int t = 0; t < S.ci; ++t) r = fma(S.wiso[size_t(i) * S.ci + t], S.fiso[voxel * S.ci + t], r);
    return fmax(ws - r, 0.0);
}

// x(list[p], :) = the dRL FOD of voxel list[p] for p < count (min(count, *count_dev) when
// count_dev is given); no list: voxel p itself.
template <int RT, int MAXCT, bool RESIDENT>
__global__ void __launch_bounds__(kDrlWarps * 32, RESIDENT ? 2 : 1)
    drl_kernel(DrlDev P, DrlSignal S, const int* __restrict__ list, int64_t count, const int* __restrict__ count_dev,
               double* __restrict__ x, int64_t ldx) {
    constexpr int kRows = 8 * RT;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double part[kDrlWarps][kRows];
    __shared__ double strength[kRows], threshold[kRows];
    __shared__ int active[kRows];
    __shared__ int64_t vox[kRows];
    __shared__ int n_active;
    if (count_dev) count = min(count, int64_t(*count_dev));
    const int c = P.c, m = P.m, cp = (c + 7) / 8 * 8, n_ct = cp / 8, ldf = drl_ldf(cp), ldg = drl_ldg(cp);
    double* F = reinterpret_cast<double*>(smem);  // (kRows, ldf)
    double* KS = F + kRows * ldf;                 // (kRows, ldf)
    double* GS = KS + kRows * ldf;                // (2, kDrlChunk, ldg): the K^T K stage; resident: (cp, ldg)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double nu8 = power_8(P.nu);
    if constexpr (RESIDENT) {
        // All of K^T K, zero past c (made visible by the barrier at the first tile's start).
        for (int e = threadIdx.x; e < cp * ldg; e += blockDim.x) {
            const int k = e / ldg, d = e - k * ldg;
            GS[e] = (k < c && d < c) ? P.gram[size_t(k) * c + d] : 0.0;
        }
    } else {
        // The stage's columns past c stay 0.
        for (int e = threadIdx.x; e < 2 * kDrlChunk * ldg; e += blockDim.x)
            if (e % ldg >= c) GS[e] = 0.0;
    }
    const int n_chunks = cp / kDrlChunk;
    // Rows [8 q, 8 q + 8) of K^T K into stage buffer b, one row per 32 threads: cp.async of 16
    // bytes when the rows are 16-byte aligned (c even; the stage's row stride is a multiple of 16
    // bytes), else of 8; zeros for the rows past c.
    const bool wide = c % 2 == 0;
    auto stage = [&](int q, int b) {
        const int r = threadIdx.x >> 5, k = q * kDrlChunk + r;
        double* dst = GS + (b * kDrlChunk + r) * ldg;
        const double* src = P.gram + size_t(k) * c;
        if (k >= c) {
            for (int d = lane; d < c; d += 32) dst[d] = 0.0;
        } else if (wide) {
            for (int d = 2 * lane; d < c; d += 64) cp_async16(dst + d, src + d);
        } else {
            for (int d = lane; d < c; d += 32) cp_async8(dst + d, src + d);
        }
        cp_async_commit();
    };
    for (int64_t p0 = int64_t(blockIdx.x) * kRows; p0 < count; p0 += int64_t(gridDim.x) * kRows) {
        if (tid < kRows) vox[tid] = p0 + tid < count ? (list ? int64_t(list[p0 + tid]) : p0 + tid) : -1;
        __syncthreads();
        // Each voxel's damping strength (1 - 4 x the sample standard deviation, at least 0) and
        // stopping threshold (1e-4 x its largest non-NaN signal value).
        for (int r = warp; r < kRows; r += kDrlWarps) {
            const int64_t voxel = vox[r];
            if (voxel < 0) {
                if (lane == 0) {
                    active[r] = 0;
                    strength[r] = threshold[r] = 0.0;
                }
                continue;
            }
            double sum = 0.0, mx = -CUDART_INF;
            bool any = false;
            for (int i = lane; i < m; i += 32) {
                const double si = signal_at(S, voxel, i);
                sum += si;
                if (!isnan(si)) {
                    mx = any ? fmax(mx, si) : si;
                    any = true;
                }
            }
            const double mean = warp_sum(sum) / m;
            double ss = 0.0;
            for (int i = lane; i < m; i += 32) {
                const double si = signal_at(S, voxel, i);
                ss += (si - mean) * (si - mean);
            }
            ss = warp_sum(ss);
            const bool all_nan = !__any_sync(0xffffffffu, any);
            mx = warp_max(any ? mx : -CUDART_INF);
            if (lane == 0) {
                strength[r] = fmax(1.0 - 4.0 * sqrt(ss / double(m - 1)), 0.0);
                threshold[r] = 1e-4 * (all_nan ? CUDART_NAN : mx);
                active[r] = 1;
            }
        }
        // K^T s and the start.
        for (int e = tid; e < kRows * ldf; e += blockDim.x) {
            const int r = e / ldf, d = e - r * ldf;
            const int64_t voxel = vox[r];
            const bool real = voxel >= 0 && d < c;
            double ks = 0.0;
            if (real) {
                const double* kt = P.k_t + size_t(d) * m;
                for (int i = 0; i < m; ++i) ks = fma(kt[i], signal_at(S, voxel, i), ks);
            }
            KS[e] = ks;
            F[e] = real ? P.init : 0.0;
        }
        __syncthreads();
        for (int it = 0; it < P.n_iter; ++it) {
            if (tid == 0) {
                int a = 0;
                for (int r = 0; r < kRows; ++r) a += active[r];
                n_active = a;
            }
            __syncthreads();
            if (n_active == 0) break;
            // The prediction K^T K f of every voxel of the tile (K^T K is symmetric: its column
            // block is read as rows).
            double acc[RT][MAXCT][2];
#pragma unroll
            for (int rt = 0; rt < RT; ++rt)
#pragma unroll
                for (int t = 0; t < MAXCT; ++t) acc[rt][t][0] = acc[rt][t][1] = 0.0;
            if constexpr (RESIDENT) {
                const int ct = warp;
                if (ct < n_ct) {
                    for (int k0 = 0; k0 < cp; k0 += 4) {
                        const int kk = k0 + (lane & 3);
                        const double b = GS[kk * ldg + 8 * ct + (lane >> 2)];
#pragma unroll
                        for (int rt = 0; rt < RT; ++rt)
                            mma_f64(acc[rt][0][0], acc[rt][0][1], F[(8 * rt + (lane >> 2)) * ldf + kk], b);
                    }
                }
                // The update overwrites F: every warp is done reading it first.
                __syncthreads();
            } else {
                stage(0, 0);
                for (int q = 0; q < n_chunks; ++q) {
                    if (q + 1 < n_chunks) {
                        stage(q + 1, (q + 1) & 1);
                        cp_async_wait<1>();
                    } else {
                        cp_async_wait<0>();
                    }
                    __syncthreads();
                    const double* g = GS + (q & 1) * kDrlChunk * ldg;
#pragma unroll
                    for (int ks = 0; ks < kDrlChunk; ks += 4) {
                        const int kk = q * kDrlChunk + ks + (lane & 3);
                        const double* grow = g + (ks + (lane & 3)) * ldg + (lane >> 2);
                        double a[RT];
#pragma unroll
                        for (int rt = 0; rt < RT; ++rt) a[rt] = F[(8 * rt + (lane >> 2)) * ldf + kk];
#pragma unroll
                        for (int t = 0; t < MAXCT; ++t) {
                            const int ct = warp + kDrlWarps * t;
                            if (ct < n_ct) {
                                const double b = grow[8 * ct];
#pragma unroll
                                for (int rt = 0; rt < RT; ++rt) mma_f64(acc[rt][t][0], acc[rt][t][1], a[rt], b);
                            }
                        }
                    }
                    // The next stage overwrites this buffer: every warp is done with it first.
                    __syncthreads();
                }
            }
            // The damped update of the still-active voxels, and each one's total change.
            double change[RT];
#pragma unroll
            for (int rt = 0; rt < RT; ++rt) change[rt] = 0.0;
#pragma unroll
            for (int t = 0; t < MAXCT; ++t) {
                const int ct = warp + kDrlWarps * t;
                if (ct >= n_ct) continue;
#pragma unroll
                for (int rt = 0; rt < RT; ++rt) {
                    const int r = 8 * rt + (lane >> 2);
                    if (!active[r]) continue;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int d = 8 * ct + 2 * (lane & 3) + h;
                        if (d >= c) continue;
                        const double f = F[r * ldf + d], f8 = power_8(f);
                        const double damping = 1.0 - strength[r] * (1.0 - f8 / (f8 + nu8));
                        const double pred = acc[rt][t][h];
                        const double ratio = (KS[r * ldf + d] - pred) / (pred + 1e-16);
                        const double updated = fmax(f * (1.0 + damping * ratio), 1e-6);
                        F[r * ldf + d] = updated;
                        change[rt] += fabs(updated - f);
                    }
                }
            }
#pragma unroll
            for (int rt = 0; rt < RT; ++rt) {
                change[rt] += __shfl_xor_sync(0xffffffffu, change[rt], 1);
                change[rt] += __shfl_xor_sync(0xffffffffu, change[rt], 2);
                if ((lane & 3) == 0) part[warp][8 * rt + (lane >> 2)] = change[rt];
            }
            __syncthreads();
            if (tid < kRows && active[tid]) {
                double total = 0.0;
                for (int w = 0; w < kDrlWarps; ++w) total += part[w][tid];
                if (total <= threshold[tid]) active[tid] = 0;
            }
            __syncthreads();
        }
        for (int e = tid; e < kRows * ldf; e += blockDim.x) {
            const int r = e / ldf, d = e - r * ldf;
            const int64_t voxel = vox[r];
            if (voxel >= 0 && d < c) x[voxel * ldx + d] = F[e];
        }
        __syncthreads();
    }
}

template <int RT, int MAXCT, bool RESIDENT>
void launch_variant(const DrlDev& P, const DrlSignal& S, const int* list, int64_t count, const int* count_dev,
                    double* x, int64_t ldx, cudaStream_t st, const char* name) {
    auto kernel = drl_kernel<RT, MAXCT, RESIDENT>;
    const size_t smem = drl_smem_bytes(P.c);
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "cudaFuncSetAttribute");
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kDrlWarps * 32, smem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    const int64_t tiles = (count + 8 * RT - 1) / (8 * RT);
    const int64_t blocks =
        std::max<int64_t>(1, std::min<int64_t>(tiles, int64_t(sm_count()) * ctas_per_sm(per_sm, "drl.ctas_per_sm")));
    LaunchScope scope(name, st);
    kernel<<<unsigned(blocks), kDrlWarps * 32, smem, st>>>(P, S, list, count, count_dev, x, ldx);
    cuda_check(cudaGetLastError(), "drl_kernel launch");
}

}  // namespace

size_t drl_smem_bytes(int c) {
    const int cp = (c + 7) / 8 * 8;
    if (c <= kResidentMaxC) return (2 * size_t(8 * kNarrowRt) * drl_ldf(cp) + size_t(cp) * drl_ldg(cp)) * sizeof(double);
    const size_t rows = c <= kNarrowMaxC ? 8 * kNarrowRt : 8 * kWideRt;
    return (2 * rows * drl_ldf(cp) + 2 * size_t(kDrlChunk) * drl_ldg(cp)) * sizeof(double);
}

bool drl_fits(int c) { return c >= 1 && c <= kWideMaxC; }

void launch_drl_listed(const DrlDev& P, const DrlSignal& S, const int* list, int64_t count, const int* count_dev,
                       double* x, int64_t ldx, cudaStream_t st) {
    if (count == 0) return;
    if (P.gtc != nullptr && drl_tc_fits(P.c) && drl_tc_fits_measurements(P.c, P.m)) {
        launch_drl_tc(P, P.gtc, S, list, count, count_dev, x, ldx, P.err, st);
        return;
    }
    if (P.c <= kResidentMaxC)
        launch_variant<kNarrowRt, 1, true>(P, S, list, count, count_dev, x, ldx, st, "drl_kernel_resident");
    else if (P.c <= kNarrowMaxC)
        launch_variant<kNarrowRt, kNarrowCt, false>(P, S, list, count, count_dev, x, ldx, st, "drl_kernel");
    else
        launch_variant<kWideRt, kWideCt, false>(P, S, list, count, count_dev, x, ldx, st, "drl_kernel_wide");
}

void launch_drl(const DrlDev& P, const double* signals, int64_t v, double* fods, cudaStream_t st) {
    launch_drl_listed(P, DrlSignal{signals, nullptr, nullptr, nullptr, P.m, 0}, nullptr, v, nullptr, fods, P.c, st);
}

}  // namespace lar
