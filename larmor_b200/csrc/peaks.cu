// FOD peaks on the GPU: the amplitude of a tournier-basis SH series and its derivatives on the
// sphere (cpp/src/sh/harmonics.cpp:139-196), the Newton climb to a peak (cpp/src/sh/peaks.cpp:
// 31-78) and the peak search of each voxel from the local maxima of its amplitudes on a sphere
// (cpp/src/sh/peaks.cpp:80-133), behind _core.sh_derivatives, _core.climb and _core.peaks_chunk
// (cpp/src/python/sh.cpp:69-176).
//
// Layout and mapping:
// - The Legendre table is built one degree at a time: row l of P(l, m) needs only rows l-1 and
//   l-2 (the recurrence runs along the degree for each order), and the derivative terms of
//   degree l need only row l (the ladder formulas mix orders m-2..m+2 of one degree). So three
//   rows of LCAP+1 values stay in registers instead of a (lmax+1)^2 table, with the same
//   arithmetic per entry as the reference's order-by-order fill.
// - The constants that depend only on (l, m) (the diagonal start, the recurrence factors, the
//   ladder factors) are tables in constant memory, computed on the host with the reference's
//   formulas and uploaded once per device.
// - The search runs in passes over one list of all the chunk's climbs (see "the peak search in
//   passes" below): a voxel has ~5-15 local maxima of very uneven climb lengths, so one warp
//   per voxel left most lanes idle; the pool of climbs keeps every lane on a climb, and the
//   merge per voxel runs on one thread in the reference's order.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include <math_constants.h>

#include "common.cuh"

namespace lar {
namespace {

constexpr int kShMaxLmax = 20;
constexpr int kShDim = kShMaxLmax + 1;
constexpr double kSamePeak = 0.99;  // cpp/src/sh/peaks.cpp:12

struct ShConstants {
    double diagonal[kShDim];         // P(m, m) / sin^m theta, with the Condon-Shortley sign
    double factor[kShDim][kShDim];   // sqrt((4 l^2 - 1) / (l^2 - m^2)), l > m
    double first_up[kShDim];         // sqrt(2 m + 3): P(m + 1, m) = first_up[m] cos P(m, m)
    double up[kShDim][kShDim + 1];   // sqrt((l - m) (l + m + 1))
    double down[kShDim][kShDim + 1]; // sqrt((l + m) (l - m + 1))
};

__constant__ ShConstants c_sh;

// cpp/src/sh/harmonics.cpp:39-66 and :29-37: the same formulas, in double on the host.
ShConstants host_constants() {
    ShConstants k;
    std::memset(&k, 0, sizeof(k));
    const double pi = 3.14159265358979323846;
    double ratio = 1.0;
    for (int m = 0; m <= kShMaxLmax; ++m) {
        const double mf = m;
        if (m > 0) ratio *= (2.0 * mf - 1.0) / (2.0 * mf);
        k.diagonal[m] = (m % 2 == 1 ? -1.0 : 1.0) * std::sqrt((2.0 * mf + 1.0) / (4.0 * pi) * ratio);
        k.first_up[m] = std::sqrt(2.0 * mf + 3.0);
        for (int l = m + 1; l <= kShMaxLmax; ++l) {
            const double lf = l;
            k.factor[l][m] = std::sqrt((4.0 * lf * lf - 1.0) / (lf * lf - mf * mf));
        }
    }
    for (int l = 0; l <= kShMaxLmax; ++l)
        for (int m = 0; m <= l; ++m) {
            k.up[l][m] = std::sqrt(double((l - m) * (l + m + 1)));
            k.down[l][m] = std::sqrt(double((l + m) * (l - m + 1)));
        }
    return k;
}

void ensure_constants() {
    static std::mutex mu;
    static bool ready[64] = {};
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    require(dev >= 0 && dev < 64, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (ready[dev]) return;
    static const ShConstants k = host_constants();
    cuda_check(cudaMemcpyToSymbol(c_sh, &k, sizeof(k)), "cudaMemcpyToSymbol");
    ready[dev] = true;
}

// The workspaces of the peak search come from a stream-ordered pool of the library's own per
// device that keeps freed memory for the next call (the device's default pool returns it to the
// driver at every synchronisation, and the search synchronises once per call).
cudaMemPool_t workspace_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    require(dev >= 0 && dev < 64, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        cuda_check(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
        uint64_t keep = ~uint64_t(0);
        cuda_check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
        pools[dev] = pool;
    }
    return pools[dev];
}

__host__ __device__ inline int n_coeffs(int lmax, bool full) {
    return full ? (lmax + 1) * (lmax + 1) : (lmax + 1) * (lmax + 2) / 2;
}

__device__ __forceinline__ int coefficient_index(int l, int m, bool full) {
    return full ? l * l + l + m : l * (l + 1) / 2 + m;
}

// base^e by squaring, the reference's order of products (cpp/src/sh/harmonics.cpp:13-27).
__device__ __forceinline__ double power_int(double base, int e) {
    double result = 1.0;
    for (;;) {
        if (e % 2 == 1) result *= base;
        e /= 2;
        if (e == 0) break;
        base *= base;
    }
    return result;
}

struct ShDerivatives {
    double f, t, p, tt, tp, pp;
};

// f, df/dtheta, df/dphi / sin, d2f/dtheta2, d2f/dtheta dphi / sin, d2f/dphi2 / sin^2 at
// (theta, phi), given sin and cos of both; the pole limits where sin theta < 1e-4. lmax <= LCAP.
template <int LCAP>
__device__ __forceinline__ ShDerivatives sh_derivatives(const double* __restrict__ sh, int lmax, bool full,
                                                        double st, double ct, double phi) {
    const bool pole = st < 1e-4;
    double sm[LCAP + 1], cm[LCAP + 1];
#pragma unroll
    for (int m = 1; m <= LCAP; ++m)
        if (m <= lmax) sincos(double(m) * phi, &sm[m], &cm[m]);
    double p2[LCAP + 1], p1[LCAP + 1], p0[LCAP + 1];
    ShDerivatives r{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int l = 0; l <= LCAP; ++l) {
        if (l > lmax) break;
        // Row l of the table (cpp/src/sh/harmonics.cpp:70-88, the same products per entry).
#pragma unroll
        for (int m = 0; m <= l; ++m) {
            if (m == l)
                p0[m] = c_sh.diagonal[m] * power_int(st, m);
            else if (m == l - 1)
                p0[m] = c_sh.first_up[m] * ct * p1[m];
            else
                p0[m] = c_sh.factor[l][m] * (ct * p1[m] - p2[m] / c_sh.factor[l - 1][m]);
        }
        if (full || l % 2 == 0) {
            // The terms of degree l (cpp/src/sh/harmonics.cpp:102-137, 150-186).
            const double zonal = __ldg(sh + coefficient_index(l, 0, full));
            r.f += zonal * p0[0];
            if (l > 0) {
                const double u0 = c_sh.up[l][0];
                const double p_2 = l >= 2 ? p0[2] : 0.0;
                r.t += zonal * (u0 * p0[1]);
                r.tt += zonal * ((u0 * c_sh.up[l][1] * p_2 - u0 * u0 * p0[0]) / 2.0);
            }
#pragma unroll
            for (int m = 1; m <= l; ++m) {
                const double mf = m;
                const double cc = __ldg(sh + coefficient_index(l, m, full));
                const double sc = __ldg(sh + coefficient_index(l, -m, full));
                const double ang = 1.41421356237309504880 * (cc * cm[m] + sc * sm[m]);
                const double ang_p = 1.41421356237309504880 * (sc * cm[m] - cc * sm[m]);
                const double u = c_sh.up[l][m], d = c_sh.down[l][m];
                const double above = m < l ? u * p0[m < l ? m + 1 : m] : 0.0;
                const double pv = p0[m];
                const double pt = (above - d * p0[m - 1]) / 2.0;
                double total = -(u * u + d * d) * pv;
                if (m == 1)
                    total -= c_sh.down[l][1] * c_sh.down[l][0] * p0[1];
                else
                    total += c_sh.down[l][m] * c_sh.down[l][m - 1] * p0[m >= 2 ? m - 2 : 0];
                if (m + 2 <= l) total += c_sh.up[l][m] * c_sh.up[l][m + 1] * p0[m + 2 <= l ? m + 2 : m];
                r.f += ang * pv;
                r.t += ang * pt;
                r.tt += ang * (total / 4.0);
                if (pole) {
                    r.p += ang_p * pt;
                } else {
                    r.p += mf * ang_p * pv;
                    r.tp += mf * ang_p * pt;
                    r.pp -= mf * mf * ang * pv;
                }
            }
        }
#pragma unroll
        for (int m = 0; m <= l; ++m) {
            p2[m] = p1[m];
            p1[m] = p0[m];
        }
    }
    if (!pole) {
        r.p /= st;
        r.tp /= st;
        r.pp /= st * st;
    }
    return r;
}

// One step of the Newton climb of cpp/src/sh/peaks.cpp:36-72 from the unit vector (x, y, z):
// moves it along the gradient by the capped Newton step and renormalises it; returns the step
// and, in *f, the amplitude before it.
template <int LCAP>
__device__ __forceinline__ double climb_step(const double* __restrict__ sh, int lmax, bool full, double& x, double& y,
                                             double& z, double max_step, double* f) {
    const double zc = z < -1.0 ? -1.0 : (1.0 < z ? 1.0 : z);  // std::clamp
    const double theta = acos(zc);
    const double phi = atan2(y, x);
    double st, ct, sp, cp;
    sincos(theta, &st, &ct);
    sincos(phi, &sp, &cp);
    const ShDerivatives h = sh_derivatives<LCAP>(sh, lmax, full, st, ct, phi);
    const double gnorm = sqrt(h.t * h.t + h.p * h.p);
    double at = 0.0, ap = 0.0;
    if (gnorm != 0.0) {
        at = h.t / gnorm;
        ap = h.p / gnorm;
    }
    const double slope = at * h.t + ap * h.p;
    const double curv = at * at * h.tt + 2.0 * at * ap * h.tp + ap * ap * h.pp;
    double step = curv != 0.0 ? fabs(slope / curv) : 0.0;
    step = fmin(step, max_step);
    x += step * (at * (ct * cp) + ap * (-sp));
    y += step * (at * (ct * sp) + ap * cp);
    z += step * (at * (-st) + ap * 0.0);
    const double n = sqrt(x * x + y * y + z * z);
    x /= n;
    y /= n;
    z /= n;
    *f = h.f;
    return step;
}

// The Newton climb of cpp/src/sh/peaks.cpp:31-78: true with the direction after the first step
// shorter than tol and the amplitude before it; false after max_iters steps.
template <int LCAP>
__device__ bool climb(const double* __restrict__ sh, int lmax, bool full, double x, double y, double z, int max_iters,
                      double tol, double max_step, double* out, double* amp) {
    for (int it = 0; it < max_iters; ++it) {
        double f;
        if (climb_step<LCAP>(sh, lmax, full, x, y, z, max_step, &f) < tol) {
            out[0] = x;
            out[1] = y;
            out[2] = z;
            *amp = f;
            return true;
        }
    }
    return false;
}

template <int LCAP>
__global__ void __launch_bounds__(128) sh_derivatives_kernel(const double* __restrict__ coeffs, int64_t n, int64_t ldc,
                                                             int lmax, int full, const double* __restrict__ theta,
                                                             const double* __restrict__ phi, double* __restrict__ out) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // Legendre::at_elevation takes cos and sin of theta (cpp/src/sh/harmonics.cpp:92-94).
    double st, ct;
    sincos(theta[i], &st, &ct);
    const ShDerivatives r = sh_derivatives<LCAP>(coeffs + i * ldc, lmax, full != 0, st, ct, phi[i]);
    double* o = out + i * 6;
    o[0] = r.f;
    o[1] = r.t;
    o[2] = r.p;
    o[3] = r.tt;
    o[4] = r.tp;
    o[5] = r.pp;
}

template <int LCAP>
__global__ void __launch_bounds__(128) climb_kernel(const double* __restrict__ coeffs, int64_t n, int64_t ldc, int lmax,
                                                    int full, const double* __restrict__ starts, int max_iters,
                                                    double tol, double max_step, double* __restrict__ dirs,
                                                    double* __restrict__ amps) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d[3], a;
    if (!climb<LCAP>(coeffs + i * ldc, lmax, full != 0, starts[3 * i], starts[3 * i + 1], starts[3 * i + 2],
                     max_iters, tol, max_step, d, &a)) {
        d[0] = d[1] = d[2] = a = CUDART_NAN;
    }
    dirs[3 * i] = d[0];
    dirs[3 * i + 1] = d[1];
    dirs[3 * i + 2] = d[2];
    amps[i] = a;
}

// ---- the peak search in passes ------------------------------------------------------------
//
// (1) peak_count_kernel: per voxel the number of its local maxima with a positive amplitude (0
//     when nv is 0 or the first amplitude is not finite: cpp/src/sh/peaks.cpp:87-89);
// (2) scan_blocks_kernel + scan_sums_kernel: their exclusive prefix sums, the offsets of the
//     voxels' climbs in one list, and the total;
// (3) peak_fill_kernel: the starts (voxel, vertex) at those offsets, in vertex order;
// (4) climb_pool_kernel: every climb of the list, one Newton step per pass of a lane, a lane
//     whose climb ends taking the next from a device counter, so the lanes stay busy however
//     uneven the climbs' lengths and the voxels' start counts are;
// (5) peak_merge_kernel: per voxel its climbs merged in start order into a found list kept in
//     place at the front of its span (cpp/src/sh/peaks.cpp:94-116), then the n_peaks largest,
//     ties to the earlier entry (a stable sort), above both thresholds (:118-132).

constexpr int kScanItems = 4;
constexpr int kScanBlock = 1024;
constexpr int kScanSpan = kScanItems * kScanBlock;  // voxels per scan block

__device__ __forceinline__ bool local_max(const double* __restrict__ amp, const int* __restrict__ nb, int v) {
    const double here = amp[v];
    bool is_max = here > 0.0;
    for (int j = 0; j < 6 && is_max; ++j) is_max = amp[nb[6 * v + j]] <= here;
    return is_max;
}

__global__ void __launch_bounds__(128) peak_count_kernel(const double* __restrict__ on_sphere, int64_t n, int64_t lds,
                                                         const int* __restrict__ neighbours, int nv,
                                                         int* __restrict__ counts) {
    const int lane = threadIdx.x & 31;
    const int64_t voxel = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (voxel >= n) return;
    const double* amp = on_sphere + voxel * lds;
    int count = 0;
    if (nv > 0 && isfinite(amp[0])) {
        for (int base = 0; base < nv; base += 32) {
            const int v = base + lane;
            count += __popc(__ballot_sync(0xffffffffu, v < nv && local_max(amp, neighbours, v)));
        }
    }
    if (lane == 0) counts[voxel] = count;
}

// Exclusive prefix sums of counts within blocks of kScanSpan voxels, and each block's sum.
__global__ void __launch_bounds__(kScanBlock) scan_blocks_kernel(const int* __restrict__ counts, int64_t n,
                                                                 int64_t* __restrict__ offsets,
                                                                 int64_t* __restrict__ block_sums) {
    __shared__ int64_t warp_sums[kScanBlock / 32];
    const int64_t first = int64_t(blockIdx.x) * kScanSpan + int64_t(threadIdx.x) * kScanItems;
    int64_t local[kScanItems];
    int64_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        local[k] = sum;
        sum += first + k < n ? counts[first + k] : 0;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t up = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += up;
    }
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0) {
        int64_t ws = warp_sums[lane];
        int64_t wi = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t up = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += up;
        }
        warp_sums[lane] = wi - ws;
        if (lane == 31) block_sums[blockIdx.x] = wi;
    }
    __syncthreads();
    const int64_t before = warp_sums[w] + incl - sum;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (first + k < n) offsets[first + k] = before + local[k];
}

// The blocks' sums to exclusive block offsets, in place, and the total; one block.
__global__ void __launch_bounds__(kScanBlock) scan_sums_kernel(int64_t* __restrict__ block_sums, int64_t blocks,
                                                               int64_t* __restrict__ total) {
    __shared__ int64_t warp_sums[kScanBlock / 32];
    __shared__ int64_t carry;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t b0 = 0; b0 < blocks; b0 += kScanBlock) {
        const int64_t b = b0 + threadIdx.x;
        const int64_t x = b < blocks ? block_sums[b] : 0;
        int64_t incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t up = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += up;
        }
        if (lane == 31) warp_sums[w] = incl;
        __syncthreads();
        if (w == 0) {
            const int64_t ws = warp_sums[lane];
            int64_t wi = ws;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t up = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += up;
            }
            warp_sums[lane] = wi - ws;
        }
        __syncthreads();
        const int64_t base = carry;
        if (b < blocks) block_sums[b] = base + warp_sums[w] + incl - x;
        __syncthreads();
        if (threadIdx.x == kScanBlock - 1) carry = base + warp_sums[w] + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__device__ __forceinline__ int64_t climb_offset(const int64_t* __restrict__ offsets,
                                                const int64_t* __restrict__ block_offsets, int64_t voxel) {
    return offsets[voxel] + block_offsets[voxel / kScanSpan];
}

__global__ void __launch_bounds__(128) peak_fill_kernel(const double* __restrict__ on_sphere, int64_t n, int64_t lds,
                                                        const int* __restrict__ neighbours, int nv,
                                                        const int64_t* __restrict__ offsets,
                                                        const int64_t* __restrict__ block_offsets,
                                                        int2* __restrict__ starts) {
    const int lane = threadIdx.x & 31;
    const int64_t voxel = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (voxel >= n) return;
    const double* amp = on_sphere + voxel * lds;
    if (nv == 0 || !isfinite(amp[0])) return;
    int64_t at = climb_offset(offsets, block_offsets, voxel);
    for (int base = 0; base < nv; base += 32) {
        const int v = base + lane;
        const bool is_max = v < nv && local_max(amp, neighbours, v);
        const unsigned b = __ballot_sync(0xffffffffu, is_max);
        if (is_max) starts[at + __popc(b & ((1u << lane) - 1u))] = make_int2(int(voxel), v);
        at += __popc(b);
    }
}

// Every climb of the list (cpp/src/sh/peaks.cpp:31-78 with the search's settings: 50 steps,
// tolerance 1e-4, steps of at most 0.2): results (total, 4) = the direction and the amplitude,
// the amplitude NaN when the climb has not stopped.
template <int LCAP>
__global__ void __launch_bounds__(128, 4) climb_pool_kernel(const double* __restrict__ coeffs, int64_t ldc, int lmax,
                                                            int full, const double* __restrict__ vertices,
                                                            const int2* __restrict__ starts, int64_t total,
                                                            double4* __restrict__ results,
                                                            unsigned long long* __restrict__ next) {
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const bool is_full = full != 0;
    int64_t k = -1;
    int it = 0;
    double x = 0.0, y = 0.0, z = 0.0;
    const double* sh = coeffs;
    bool exhausted = false;
    for (;;) {
        // Lanes without a climb take the next ones, one atomic per warp.
        const unsigned want = __ballot_sync(0xffffffffu, k < 0 && !exhausted);
        if (want) {
            unsigned long long base = 0;
            const int leader = __ffs(want) - 1;
            if (lane == leader) base = atomicAdd(next, (unsigned long long)__popc(want));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (base + __popc(want) >= (unsigned long long)total) exhausted = true;
            if (k < 0) {
                const unsigned long long mine = base + __popc(want & below);
                if (mine < (unsigned long long)total) {
                    k = int64_t(mine);
                    const int2 s = starts[k];
                    x = vertices[3 * s.y];
                    y = vertices[3 * s.y + 1];
                    z = vertices[3 * s.y + 2];
                    sh = coeffs + int64_t(s.x) * ldc;
                    it = 0;
                }
            }
        }
        if (!__any_sync(0xffffffffu, k >= 0)) break;
        if (k >= 0) {
            double f;
            const double step = climb_step<LCAP>(sh, lmax, is_full, x, y, z, 0.2, &f);
            if (step < 1e-4) {
                results[k] = make_double4(x, y, z, f);
                k = -1;
            } else if (++it >= 50) {
                results[k] = make_double4(CUDART_NAN, CUDART_NAN, CUDART_NAN, CUDART_NAN);
                k = -1;
            }
        }
    }
}

__global__ void __launch_bounds__(128) peak_merge_kernel(int64_t n, int full, const int* __restrict__ counts,
                                                         const int64_t* __restrict__ offsets,
                                                         const int64_t* __restrict__ block_offsets,
                                                         double4* __restrict__ results, int n_peaks, double rel,
                                                         double thr, double* __restrict__ dirs,
                                                         double* __restrict__ amps) {
    const int64_t voxel = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (voxel >= n) return;
    double* dv = dirs + voxel * int64_t(n_peaks) * 3;
    double* av = amps + voxel * int64_t(n_peaks);
    for (int k = 0; k < 3 * n_peaks; ++k) dv[k] = CUDART_NAN;
    for (int k = 0; k < n_peaks; ++k) av[k] = CUDART_NAN;
    const int count = counts[voxel];
    if (count == 0) return;
    double4* found = results + climb_offset(offsets, block_offsets, voxel);
    const bool is_full = full != 0;
    int n_found = 0;
    for (int i = 0; i < count; ++i) {
        const double4 c = found[i];
        // Written so that a NaN amplitude is dropped too.
        if (!(c.w > 0.0)) continue;
        int match = -1;
        for (int j = 0; j < n_found; ++j) {
            const double4 o = found[j];
            const double cosine = c.x * o.x + c.y * o.y + c.z * o.z;
            if ((is_full ? cosine : fabs(cosine)) > kSamePeak) {
                match = j;
                break;
            }
        }
        // The found list occupies entries [0, n_found), n_found <= i: entry i is read already.
        if (match < 0)
            found[n_found++] = c;
        else if (c.w > found[match].w)
            found[match] = c;
    }
    if (n_found == 0) return;
    double largest = 0.0;
    const int kept = min(n_peaks, n_found);
    for (int r = 0; r < kept; ++r) {
        int bi = 0;
        double best = -CUDART_INF;
        for (int j = 0; j < n_found; ++j)
            if (found[j].w > best) {
                best = found[j].w;
                bi = j;
            }
        if (r == 0) largest = best;
        if (best < thr || best < rel * largest) break;
        const double4 c = found[bi];
        const bool flip = !is_full && c.z < 0.0;
        dv[3 * r] = flip ? -c.x : c.x;
        dv[3 * r + 1] = flip ? -c.y : c.y;
        dv[3 * r + 2] = flip ? -c.z : c.z;
        av[r] = best;
        found[bi].w = -CUDART_INF;  // taken
    }
}

int lcap_for(int lmax) { return lmax <= 8 ? 8 : (lmax <= 12 ? 12 : 20); }

void check_lmax(int lmax, bool full, int64_t ldc) {
    require(lmax >= 0 && lmax <= kShMaxLmax && (full || lmax % 2 == 0),
            "lmax must be at most 20, and even unless full, got " + std::to_string(lmax));
    require(ldc >= n_coeffs(lmax, full), "ldc must be at least the series' coefficient count");
}

}  // namespace
}  // namespace lar

// A sphere for the peak search: unit vertices and the 6 neighbours of each, on the device.
struct lar_peak_sphere_s {
    int64_t nv = 0;
    lar::DeviceArray<double> vertices;  // (nv, 3)
    lar::DeviceArray<int> neighbours;   // (nv, 6)
};

using namespace lar;

extern "C" {

int lar_peak_sphere_create(const double* vertices, const int64_t* neighbours, int64_t nv, lar_peak_sphere* out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        require(nv >= 0 && nv < (int64_t(1) << 31), "nv must be between 0 and 2^31 - 1");
        require(nv == 0 || (vertices != nullptr && neighbours != nullptr), "vertices and neighbours must not be NULL");
        std::vector<int> nb(size_t(nv) * 6);
        for (int64_t k = 0; k < nv * 6; ++k) {
            require(neighbours[k] >= 0 && neighbours[k] < nv, "a neighbour index is outside the sphere");
            nb[size_t(k)] = int(neighbours[k]);
        }
        auto h = std::make_unique<lar_peak_sphere_s>();
        h->nv = nv;
        h->vertices.upload(vertices, size_t(nv) * 3);
        h->neighbours.upload(nb.data(), nb.size());
        *out = h.release();
    });
}

void lar_peak_sphere_destroy(lar_peak_sphere sphere) { delete sphere; }

int lar_sh_derivatives(const double* coeffs, int64_t n, int64_t ldc, int lmax, int full, const double* theta,
                       const double* phi, double* out, void* stream) {
    return guarded([&] {
        check_lmax(lmax, full != 0, ldc);
        require(n >= 0, "n must be at least 0");
        if (n == 0) return;
        ensure_constants();
        auto st = static_cast<cudaStream_t>(stream);
        const unsigned blocks = unsigned((n + 127) / 128);
        LaunchScope scope("sh_derivatives_kernel", st);
        switch (lcap_for(lmax)) {
            case 8: sh_derivatives_kernel<8><<<blocks, 128, 0, st>>>(coeffs, n, ldc, lmax, full, theta, phi, out); break;
            case 12: sh_derivatives_kernel<12><<<blocks, 128, 0, st>>>(coeffs, n, ldc, lmax, full, theta, phi, out); break;
            default: sh_derivatives_kernel<20><<<blocks, 128, 0, st>>>(coeffs, n, ldc, lmax, full, theta, phi, out);
        }
        cuda_check(cudaGetLastError(), "sh_derivatives_kernel launch");
    });
}

int lar_climb(const double* coeffs, int64_t n, int64_t ldc, int lmax, int full, const double* starts, int max_iters,
              double tol, double max_step, double* directions, double* amplitudes, void* stream) {
    return guarded([&] {
        check_lmax(lmax, full != 0, ldc);
        require(n >= 0, "n must be at least 0");
        require(max_iters >= 0, "max_iters must be at least 0");
        if (n == 0) return;
        ensure_constants();
        auto st = static_cast<cudaStream_t>(stream);
        const unsigned blocks = unsigned((n + 127) / 128);
        LaunchScope scope("climb_kernel", st);
        switch (lcap_for(lmax)) {
            case 8:
                climb_kernel<8><<<blocks, 128, 0, st>>>(coeffs, n, ldc, lmax, full, starts, max_iters, tol, max_step,
                                                        directions, amplitudes);
                break;
            case 12:
                climb_kernel<12><<<blocks, 128, 0, st>>>(coeffs, n, ldc, lmax, full, starts, max_iters, tol, max_step,
                                                         directions, amplitudes);
                break;
            default:
                climb_kernel<20><<<blocks, 128, 0, st>>>(coeffs, n, ldc, lmax, full, starts, max_iters, tol, max_step,
                                                         directions, amplitudes);
        }
        cuda_check(cudaGetLastError(), "climb_kernel launch");
    });
}

int lar_find_peaks(lar_peak_sphere sphere, const double* coeffs, int64_t n, int64_t ldc, int lmax, int full,
                   const double* on_sphere, int64_t lds, int n_peaks, double relative_threshold, double threshold,
                   double* directions, double* amplitudes, void* stream) {
    return guarded([&] {
        require(sphere != nullptr, "sphere must not be NULL");
        check_lmax(lmax, full != 0, ldc);
        require(n >= 0, "n must be at least 0");
        require(n_peaks >= 1, "n_peaks must be at least 1");
        require(lds >= sphere->nv, "lds must be at least the sphere's vertex count");
        require(n < (int64_t(1) << 31), "n must be below 2^31");
        if (n == 0) return;
        ensure_constants();
        auto st = static_cast<cudaStream_t>(stream);
        const int nv = int(sphere->nv);
        const int64_t scan_blocks = (n + kScanSpan - 1) / kScanSpan;
        // Workspace: counts (n), offsets (n), block offsets, the total and the climbs' counter.
        const size_t ws_bytes = size_t(n) * sizeof(int) + (size_t(n) + size_t(scan_blocks) + 2) * sizeof(int64_t) + 64;
        char* ws = nullptr;
        cudaMemPool_t pool = workspace_pool();
        cuda_check(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ws), ws_bytes, pool, st), "cudaMallocFromPoolAsync");
        auto* offsets = reinterpret_cast<int64_t*>(ws);
        auto* block_offsets = offsets + n;
        auto* total_dev = block_offsets + scan_blocks;
        auto* next = reinterpret_cast<unsigned long long*>(total_dev + 1);
        int* counts = reinterpret_cast<int*>(next + 1);
        const unsigned warp_blocks = unsigned((n * 32 + 127) / 128);
        {
            LaunchScope scope("peak_count_kernel", st);
            peak_count_kernel<<<warp_blocks, 128, 0, st>>>(on_sphere, n, lds, sphere->neighbours.ptr, nv, counts);
            cuda_check(cudaGetLastError(), "peak_count_kernel launch");
        }
        {
            LaunchScope scope("scan_blocks_kernel", st);
            scan_blocks_kernel<<<unsigned(scan_blocks), kScanBlock, 0, st>>>(counts, n, offsets, block_offsets);
            cuda_check(cudaGetLastError(), "scan_blocks_kernel launch");
        }
        {
            LaunchScope scope("scan_sums_kernel", st);
            scan_sums_kernel<<<1, kScanBlock, 0, st>>>(block_offsets, scan_blocks, total_dev);
            cuda_check(cudaGetLastError(), "scan_sums_kernel launch");
        }
        // The climb list's length sizes its buffers: the one wait of the call.
        int64_t total = 0;
        cuda_check(cudaMemcpyAsync(&total, total_dev, sizeof(total), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        char* lists = nullptr;
        if (total > 0) {
            cuda_check(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&lists),
                                               size_t(total) * (sizeof(int2) + sizeof(double4)), pool, st),
                       "cudaMallocFromPoolAsync");
            auto* results = reinterpret_cast<double4*>(lists);
            auto* starts = reinterpret_cast<int2*>(results + total);
            {
                LaunchScope scope("peak_fill_kernel", st);
                peak_fill_kernel<<<warp_blocks, 128, 0, st>>>(on_sphere, n, lds, sphere->neighbours.ptr, nv, offsets,
                                                              block_offsets, starts);
                cuda_check(cudaGetLastError(), "peak_fill_kernel launch");
            }
            cuda_check(cudaMemsetAsync(next, 0, sizeof(*next), st), "cudaMemsetAsync");
            const int lcap = lcap_for(lmax);
            auto climber =
                lcap == 8 ? climb_pool_kernel<8> : (lcap == 12 ? climb_pool_kernel<12> : climb_pool_kernel<20>);
            int per_sm = 0;
            cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, climber, 128, 0),
                       "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
            const int64_t pool_blocks = std::max<int64_t>(
                1, std::min<int64_t>((total + 127) / 128, int64_t(sm_count()) * ctas_per_sm(per_sm, "peaks.ctas_per_sm")));
            {
                LaunchScope scope("climb_pool_kernel", st);
                climber<<<unsigned(pool_blocks), 128, 0, st>>>(coeffs, ldc, lmax, full, sphere->vertices.ptr, starts,
                                                               total, results, next);
                cuda_check(cudaGetLastError(), "climb_pool_kernel launch");
            }
        }
        {
            LaunchScope scope("peak_merge_kernel", st);
            peak_merge_kernel<<<unsigned((n + 127) / 128), 128, 0, st>>>(
                n, full, counts, offsets, block_offsets, reinterpret_cast<double4*>(lists), n_peaks, relative_threshold,
                threshold, directions, amplitudes);
            cuda_check(cudaGetLastError(), "peak_merge_kernel launch");
        }
        if (lists) cuda_check(cudaFreeAsync(lists, st), "cudaFreeAsync");
        cuda_check(cudaFreeAsync(ws, st), "cudaFreeAsync");
    });
}

}  // extern "C"
