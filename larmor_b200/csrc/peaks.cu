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
// - One warp per voxel: the lanes test 32 vertices at a time for local maxima and collect the
//   starts in vertex order; each lane then climbs from one start; the warp merges the climbs
//   into the voxel's found list in start order (the reference's merge order), with the lanes
//   searching the list for the first match; the n_peaks largest are chosen by repeated
//   warp-wide maxima, ties to the earlier entry (the reference's stable sort).
// - The found list is per-warp global scratch of nv entries, the most climbs a voxel can have.

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
constexpr int kPeakWarps = 4;
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

// The Newton climb of cpp/src/sh/peaks.cpp:31-78: true with the direction after the first step
// shorter than tol and the amplitude before it; false after max_iters steps.
template <int LCAP>
__device__ bool climb(const double* __restrict__ sh, int lmax, bool full, double x, double y, double z, int max_iters,
                      double tol, double max_step, double* out, double* amp) {
    for (int it = 0; it < max_iters; ++it) {
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
        if (step < tol) {
            out[0] = x;
            out[1] = y;
            out[2] = z;
            *amp = h.f;
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

// A climb's result, per lane of a warp.
struct ClimbSlot {
    double d[3];
    double a;
};

template <int LCAP>
__global__ void __launch_bounds__(kPeakWarps * 32) peaks_kernel(
    const double* __restrict__ coeffs, int64_t n, int64_t ldc, int lmax, int full, const double* __restrict__ on_sphere,
    int64_t lds, const double* __restrict__ vertices, const int* __restrict__ neighbours, int nv, int n_peaks,
    double rel, double thr, double* __restrict__ dirs, double* __restrict__ amps, double* __restrict__ scratch) {
    __shared__ ClimbSlot slots[kPeakWarps][32];
    __shared__ int starts[kPeakWarps][32];
    __shared__ unsigned char valid[kPeakWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t warp = int64_t(blockIdx.x) * kPeakWarps + w;
    const int64_t n_warps = int64_t(gridDim.x) * kPeakWarps;
    // The found list: nv entries of (x, y, z, amplitude).
    double* found = scratch + warp * int64_t(nv) * 4;
    const bool is_full = full != 0;
    for (int64_t voxel = warp; voxel < n; voxel += n_warps) {
        const double* sh = coeffs + voxel * ldc;
        const double* amp_v = on_sphere + voxel * lds;
        double* dv = dirs + voxel * int64_t(n_peaks) * 3;
        double* av = amps + voxel * int64_t(n_peaks);
        for (int k = lane; k < 3 * n_peaks; k += 32) dv[k] = CUDART_NAN;
        for (int k = lane; k < n_peaks; k += 32) av[k] = CUDART_NAN;
        if (nv == 0 || !isfinite(amp_v[0])) continue;
        int n_found = 0, pending = 0;
        // Climbs from starts[w][0..pending) and merges them in order.
        auto climb_and_merge = [&]() {
            if (lane < pending) {
                const int v = starts[w][lane];
                ClimbSlot s;
                const bool ok = climb<LCAP>(sh, lmax, is_full, vertices[3 * v], vertices[3 * v + 1],
                                            vertices[3 * v + 2], 50, 1e-4, 0.2, s.d, &s.a);
                // Written so that a NaN amplitude is dropped too.
                valid[w][lane] = ok && s.a > 0.0;
                slots[w][lane] = s;
            }
            __syncwarp();
            for (int i = 0; i < pending; ++i) {
                if (!valid[w][i]) continue;
                const ClimbSlot s = slots[w][i];
                int match = -1;
                for (int j0 = 0; j0 < n_found && match < 0; j0 += 32) {
                    const int j = j0 + lane;
                    bool same = false;
                    if (j < n_found) {
                        const double* f = found + 4 * j;
                        const double c = s.d[0] * f[0] + s.d[1] * f[1] + s.d[2] * f[2];
                        same = (is_full ? c : fabs(c)) > kSamePeak;
                    }
                    const unsigned b = __ballot_sync(0xffffffffu, same);
                    if (b) match = j0 + __ffs(b) - 1;
                }
                if (lane == 0) {
                    double* f = nullptr;
                    if (match < 0)
                        f = found + 4 * n_found;
                    else if (s.a > found[4 * match + 3])
                        f = found + 4 * match;
                    if (f) {
                        f[0] = s.d[0];
                        f[1] = s.d[1];
                        f[2] = s.d[2];
                        f[3] = s.a;
                    }
                }
                if (match < 0) ++n_found;
                __syncwarp();
            }
            pending = 0;
        };
        for (int base = 0; base < nv; base += 32) {
            const int v = base + lane;
            bool is_max = false;
            if (v < nv) {
                const double here = amp_v[v];
                is_max = here > 0.0;
                for (int j = 0; j < 6 && is_max; ++j) is_max = amp_v[neighbours[6 * v + j]] <= here;
            }
            const unsigned b = __ballot_sync(0xffffffffu, is_max);
            const int k = __popc(b);
            if (pending + k > 32) climb_and_merge();
            if (is_max) starts[w][pending + __popc(b & ((1u << lane) - 1u))] = v;
            pending += k;
            __syncwarp();
        }
        if (pending > 0) climb_and_merge();
        if (n_found == 0) continue;
        // The n_peaks largest in a stable order, above both thresholds
        // (cpp/src/sh/peaks.cpp:118-132).
        double largest = 0.0;
        const int kept = min(n_peaks, n_found);
        for (int r = 0; r < kept; ++r) {
            double best = -CUDART_INF;
            int bi = -1;
            for (int j = lane; j < n_found; j += 32) {
                const double a = found[4 * j + 3];
                if (a > best) {
                    best = a;
                    bi = j;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (oi >= 0 && (bi < 0 || ob > best || (ob == best && oi < bi))) {
                    best = ob;
                    bi = oi;
                }
            }
            if (r == 0) largest = best;
            if (best < thr || best < rel * largest) break;
            if (lane == 0) {
                double* f = found + 4 * bi;
                const bool flip = !is_full && f[2] < 0.0;
                for (int a = 0; a < 3; ++a) dv[3 * r + a] = flip ? -f[a] : f[a];
                av[r] = best;
                f[3] = -CUDART_INF;  // taken
            }
            __syncwarp();
        }
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
        if (n == 0) return;
        ensure_constants();
        auto st = static_cast<cudaStream_t>(stream);
        const int lcap = lcap_for(lmax);
        auto kernel = lcap == 8 ? peaks_kernel<8> : (lcap == 12 ? peaks_kernel<12> : peaks_kernel<20>);
        int per_sm = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPeakWarps * 32, 0),
                   "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        const int64_t blocks = std::max<int64_t>(
            1, std::min<int64_t>((n + kPeakWarps - 1) / kPeakWarps,
                                 int64_t(sm_count()) * ctas_per_sm(per_sm, "peaks.ctas_per_sm")));
        const size_t scratch_bytes = size_t(blocks) * kPeakWarps * size_t(std::max<int64_t>(sphere->nv, 1)) * 4 *
                                     sizeof(double);
        double* scratch = nullptr;
        cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&scratch), scratch_bytes, st), "cudaMallocAsync");
        {
            LaunchScope scope("peaks_kernel", st);
            kernel<<<unsigned(blocks), kPeakWarps * 32, 0, st>>>(
                coeffs, n, ldc, lmax, full, on_sphere, lds, sphere->vertices.ptr, sphere->neighbours.ptr,
                int(sphere->nv), n_peaks, relative_threshold, threshold, directions, amplitudes, scratch);
        }
        const cudaError_t launch = cudaGetLastError();
        cuda_check(cudaFreeAsync(scratch, st), "cudaFreeAsync");
        cuda_check(launch, "peaks_kernel launch");
    });
}

}  // extern "C"
