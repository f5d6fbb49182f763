// The log-signal fit for designs of up to 32 parameters (DKI: p = 22), one warp per voxel.
//
// Follows cpp/src/dwi/log_fit.cpp: the ordinary fit pinv y (:251), the reweighted fit
// (reweighted_fit :114-147) and the constraint check (breaks_a_constraint :150). The design
// (unit-norm columns, pseudo-inverse) sits in shared memory, shared by the CTA's warps; each
// warp keeps its voxel's log signals, weights and normal matrix in its own shared-memory
// slice. Lanes split the measurements for predictions and weights, the normal-matrix entries
// for the weighted Gram, and the rows for the L D L^T solve.
//
// Voxels whose unconstrained solution breaks a constraint are appended to a compacted list
// (voxel index and scaled parameters) for the constrained re-fit (constrained_fit.cu).

#include <cstdint>

#include "common.cuh"
#include "log_fit.cuh"
#include "batch.cuh"
#include "log_fit_warp.cuh"

namespace lar {

namespace {

constexpr int kWarps = 4;

template <class T>
struct WarpLayout {
    int n, p, px, pp;
    // Shared memory: X (n, px), pinv^T (n, p), the (a, b) of each normal-matrix entry,
    // then per warp: y (n), w (n), normal matrix (p, px), 4 vectors of 32.
    __host__ __device__ size_t design_elems() const { return size_t(n) * px + size_t(n) * p; }
    __host__ __device__ size_t warp_elems() const { return 2 * size_t(n) + size_t(p) * px + 4 * 32; }
    __host__ __device__ size_t bytes(int warps) const {
        return (design_elems() + warps * warp_elems()) * sizeof(T) + 2 * size_t(pp) + 16;
    }
};

// Solves the symmetric system held in the lower triangle of a (p x px, shared) by L D L^T in
// place, with b (shared, p) overwritten by the solution. Returns false on an exactly zero pivot
// (singular weighted normal equations; cpp/src/dwi/log_fit.cpp:128-133). All lanes return the
// same value.
template <class T>
__device__ bool warp_ldlt_solve(T* a, int p, int px, T* b, T* col, int lane) {
    for (int k = 0; k < p; ++k) {
        __syncwarp();
        const T d = a[k * px + k];
        if (d == T(0)) return false;
        const int i = k + 1 + lane;
        T l = T(0);
        if (i < p) {
            const T c = a[i * px + k];
            col[i] = c;
            l = c / d;
        }
        __syncwarp();
        if (i < p) {
            for (int j = k + 1; j <= i; ++j) a[i * px + j] = fma(-l, col[j], a[i * px + j]);
            a[i * px + k] = l;
        }
    }
    // L z = b, then z / d, then L^T x = z.
    for (int k = 0; k < p; ++k) {
        __syncwarp();
        const T zk = b[k];
        const int i = k + 1 + lane;
        if (i < p) b[i] = fma(-a[i * px + k], zk, b[i]);
    }
    __syncwarp();
    if (lane < p) b[lane] = b[lane] / a[lane * px + lane];
    for (int k = p - 1; k >= 0; --k) {
        __syncwarp();
        const T zk = b[k];
        if (lane < k) b[lane] = fma(-a[k * px + lane], zk, b[lane]);
    }
    __syncwarp();
    return true;
}

// A CTA's shared memory for the warp fits: the design (X with its rows padded to px, pinv^T,
// the (a, b) of each normal-matrix entry), then each warp's slice (y, w, normal matrix, four
// 32-vectors).
template <class T>
struct WarpSmem {
    T *xs, *pinvt, *ys, *ws, *gm, *pv, *rv, *ov, *cv;
    uint8_t *ea, *eb;
};

template <class T>
__device__ __forceinline__ WarpSmem<T> carve_warp(unsigned char* smem_raw, const WarpLayout<T>& lay, int warps,
                                                  int warp) {
    WarpSmem<T> w;
    T* base = reinterpret_cast<T*>(smem_raw);
    w.xs = base;
    w.pinvt = base + size_t(lay.n) * lay.px;
    w.ea = reinterpret_cast<uint8_t*>(base + lay.design_elems() + warps * lay.warp_elems());
    w.eb = w.ea + lay.pp;
    w.ys = base + lay.design_elems() + warp * lay.warp_elems();
    w.ws = w.ys + lay.n;
    w.gm = w.ws + lay.n;
    w.pv = w.gm + size_t(lay.p) * lay.px;  // current parameters
    w.rv = w.pv + 32;                      // right-hand side / next parameters
    w.ov = w.rv + 32;                      // ordinary fit
    w.cv = w.ov + 32;                      // column scratch of the solve
    return w;
}

// The CTA stages the design (the caller synchronises before and after).
template <class T>
__device__ __forceinline__ void stage_warp_design(const LogDesignDevice<T>& d, const WarpLayout<T>& lay,
                                                  const WarpSmem<T>& w) {
    const int n = lay.n, p = lay.p, px = lay.px, pp = lay.pp;
    for (int i = threadIdx.x; i < n * p; i += blockDim.x) {
        const int r = i / p, c = i % p;
        w.xs[r * px + c] = d.x[i];
        w.pinvt[i] = d.pinvt[i];
    }
    for (int e = threadIdx.x; e < pp; e += blockDim.x) {
        // Entry e of the packed upper triangle, row by row.
        int a = 0, rem = e;
        while (rem >= p - a) { rem -= p - a; ++a; }
        w.ea[e] = uint8_t(a);
        w.eb[e] = uint8_t(a + rem);
    }
}

// One voxel's fit on a warp: its scaled parameters end in w.pv. Returns the number of weighted
// fits and sets *violated_out when the (finite) solution breaks a constraint.
template <class T, class Src>
__device__ __forceinline__ int log_warp_voxel(const LogDesignDevice<T>& d, const WarpLayout<T>& lay,
                                              const WarpSmem<T>& w, const Src& src, int64_t voxel,
                                              int weighted, int max_rw, T tol, bool* violated_out,
                                              int lane) {
    const int n = lay.n, p = lay.p, px = lay.px, pp = lay.pp;
    T* const xs = w.xs;
    T* const pinvt = w.pinvt;
    const uint8_t* const ea = w.ea;
    const uint8_t* const eb = w.eb;
    T* const ys = w.ys;
    T* const ws = w.ws;
    T* const gm = w.gm;
    T* const pv = w.pv;
    T* const rv = w.rv;
    T* const ov = w.ov;
    T* const cv = w.cv;
        src.template warp_stage<T>(voxel, ys, lane);
    __syncwarp();
    // Ordinary fit.
    if (lane < p) {
        T acc = T(0);
        for (int j = 0; j < n; ++j) acc = fma(pinvt[j * p + lane], ys[j], acc);
        ov[lane] = acc;
        pv[lane] = acc;
    }
    __syncwarp();
    bool finite = true;
    for (int a = 0; a < p; ++a) finite &= bool(isfinite(pv[a]));
    int it = 0;
    if (weighted && finite) {
        T mx = -INFINITY;
        for (int j = lane; j < n; j += 32) {
            T pred = T(0);
            for (int a = 0; a < p; ++a) pred = fma(xs[j * px + a], pv[a], pred);
            mx = fmax(mx, pred);
        }
        mx = warp_max(mx);
        for (; it < max_rw; ++it) {
            for (int j = lane; j < n; j += 32) {
                T pred = T(0);
                for (int a = 0; a < p; ++a) pred = fma(xs[j * px + a], pv[a], pred);
                ws[j] = dev_exp<T>(T(2) * (pred - mx));
            }
            __syncwarp();
            // Four entries per lane at a time, so that their sums over the measurements
            // overlap (each in its own order).
            for (int e0 = lane; e0 < pp; e0 += 4 * 32) {
                int ia[4], ib[4];
                T acc[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int e = e0 + 32 * q;
                    ia[q] = e < pp ? ea[e] : 0;
                    ib[q] = e < pp ? eb[e] : 0;
                    acc[q] = T(0);
                }
                for (int j = 0; j < n; ++j) {
                    const T wj = ws[j];
                    const T* xr = xs + j * px;
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[q] = fma(wj * xr[ia[q]], xr[ib[q]], acc[q]);
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (e0 + 32 * q < pp) gm[ib[q] * px + ia[q]] = acc[q];  // lower triangle
            }
            if (lane < p) {
                T acc = T(0);
                for (int j = 0; j < n; ++j) acc = fma(ws[j] * xs[j * px + lane], ys[j], acc);
                rv[lane] = acc;
            }
            __syncwarp();
            bool ok = warp_ldlt_solve<T>(gm, p, px, rv, cv, lane);
            if (ok) {
                for (int a = 0; a < p; ++a) ok &= bool(isfinite(rv[a]));
            }
            if (!ok) {
                if (lane < p) pv[lane] = ov[lane];
                __syncwarp();
                ++it;
                break;
            }
            T change = T(0), mxn = -INFINITY;
            for (int j = lane; j < n; j += 32) {
                T po = T(0), pn = T(0);
                for (int a = 0; a < p; ++a) {
                    po = fma(xs[j * px + a], pv[a], po);
                    pn = fma(xs[j * px + a], rv[a], pn);
                }
                change = fmax(change, fabs(pn - po));
                mxn = fmax(mxn, pn);
            }
            change = warp_max(change);
            mxn = warp_max(mxn);
            __syncwarp();
            if (lane < p) pv[lane] = rv[lane];
            __syncwarp();
            mx = mxn;
            if (!(change > tol)) {
                ++it;
                break;
            }
        }
    }
    // Constraint check on the scaled parameters (cpp/src/dwi/log_fit.cpp:150,256).
    bool violated = false;
    if (d.m > 0) {
        bool fin = true;
        for (int a = 0; a < p; ++a) fin &= bool(isfinite(pv[a]));
        if (fin) {
            bool neg = false;
            for (int i = lane; i < d.m; i += 32) {
                T val = T(0);
                for (int a = 0; a < p; ++a) val = fma(d.g[size_t(i) * p + a], pv[a], val);
                neg |= val < T(0);
            }
            violated = __any_sync(0xffffffffu, neg);
        }
    }
    *violated_out = violated;
    return it;
}

// WARPS warps per CTA share one staged design; the launcher picks the count that keeps the most
// warps resident (the design dominates a CTA's shared memory at DKI's table sizes).
template <class T, class Src, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) fit_log_warp_kernel(
    LogDesignDevice<T> d, Src src, int64_t v, int weighted, int max_rw, T tol,
    double* __restrict__ params, uint8_t* __restrict__ broke, int32_t* __restrict__ iterations,
    ViolatorList<T> violators) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int p = d.p;
    const WarpLayout<T> lay{d.n, p, p | 1, p * (p + 1) / 2};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const WarpSmem<T> w = carve_warp<T>(smem_raw, lay, WARPS, warp);
    stage_warp_design<T>(d, lay, w);
    __syncthreads();
    for (int64_t voxel = int64_t(blockIdx.x) * WARPS + warp; voxel < v;
         voxel += int64_t(gridDim.x) * WARPS) {
        bool violated = false;
        const int it = log_warp_voxel<T>(d, lay, w, src, voxel, weighted, max_rw, tol, &violated, lane);
        const T* pv = w.pv;
        if (lane < p) params[voxel * p + lane] = double(pv[lane]) / d.scales64[lane];
        if (lane == 0) {
            broke[voxel] = violated ? 1 : 0;
            if (iterations) iterations[voxel] = it;
        }
        if (violated && violators.count != nullptr) {
            int slot = 0;
            if (lane == 0) slot = atomicAdd(violators.count, 1);
            slot = __shfl_sync(0xffffffffu, slot, 0);
            if (slot < violators.capacity) {
                if (lane == 0) violators.voxel[slot] = voxel;
                if (lane < p) violators.params[size_t(slot) * p + lane] = double(pv[lane]);
            }
        }
        __syncwarp();
    }
}

// The DKI family of a batch (batch.cuh): CTAs of WARPS warps take tickets of
// kDkiVoxelsPerWarp * WARPS voxels of one volume from a device counter across every DKI volume
// (each warp fits every WARPS-th voxel of the ticket) and restage the design when the ticket
// moves to another volume. The shared memory is sized for the family's largest table, so the
// CTAs are wider than the single-volume fit's: more warps share one staged design. Violators go
// to one list for the whole family, with their volume.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) batch_log_warp_kernel(
    const DkiBatchJob* __restrict__ jobs, const int64_t* __restrict__ first, int n_jobs, int weighted,
    int max_rw, double tol, int* __restrict__ queue, BatchViolators violators) {
    using T = double;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ long long ticket;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t total = first[n_jobs];
    int cur = -1;
    WarpLayout<T> lay{0, 0, 1, 0};
    WarpSmem<T> w{};
    for (;;) {
        if (threadIdx.x == 0) ticket = atomicAdd(reinterpret_cast<unsigned long long*>(queue), 1ull);
        __syncthreads();
        const int64_t t = ticket;
        if (t >= total) break;
        const int j = ticket_job(first, n_jobs, t);
        const DkiBatchJob& job = jobs[j];
        const LogDesignDevice<T> d = job.d;
        if (j != cur) {
            const int p = d.p;
            lay = WarpLayout<T>{d.n, p, p | 1, p * (p + 1) / 2};
            w = carve_warp<T>(smem_raw, lay, WARPS, warp);
            stage_warp_design<T>(d, lay, w);
            cur = j;
        }
        __syncthreads();
        const CappedSource src{job.s, job.s0, job.floor, job.is_b0, d.n};
        const int64_t v = job.v, block_first = (t - first[j]) * (kDkiVoxelsPerWarp * WARPS);
        const int p = d.p;
        for (int k = warp; k < kDkiVoxelsPerWarp * WARPS; k += WARPS) {
            const int64_t voxel = block_first + k;
            if (voxel >= v) break;
            bool violated = false;
            log_warp_voxel<T>(d, lay, w, src, voxel, weighted, max_rw, T(tol), &violated, lane);
            const T* pv = w.pv;
            if (lane < p) job.params[voxel * p + lane] = pv[lane] / d.scales64[lane];
            if (lane == 0) job.broke[voxel] = violated ? 1 : 0;
            if (violated) {
                int slot = 0;
                if (lane == 0) slot = atomicAdd(violators.count, 1);
                slot = __shfl_sync(0xffffffffu, slot, 0);
                if (slot < violators.capacity) {
                    if (lane == 0) {
                        violators.job[slot] = j;
                        violators.voxel[slot] = voxel;
                    }
                    if (lane < p) violators.params[size_t(slot) * p + lane] = pv[lane];
                }
            }
            __syncwarp();
        }
        __syncthreads();
    }
}

// The resident warps of fit_log_warp_kernel with WARPS warps per CTA (0 when its shared memory
// does not fit a CTA), setting the kernel's shared-memory limit.
template <class T, class Src, int WARPS>
int64_t warp_fit_residency(const WarpLayout<T>& lay) {
    const size_t smem = lay.bytes(WARPS);
    if (smem > 227 * 1024) return 0;
    auto kernel = fit_log_warp_kernel<T, Src, WARPS>;
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "cudaFuncSetAttribute");
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, WARPS * 32, smem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    return int64_t(per_sm) * WARPS;
}

template <class T, class Src, int WARPS>
void launch_warp_w(const LogDesignDevice<T>& d, const Src& src, int64_t v, int weighted, int max_rw, double tol,
                   double* params, uint8_t* broke, int32_t* iterations, const ViolatorList<T>& violators,
                   cudaStream_t stream) {
    const WarpLayout<T> lay{d.n, d.p, d.p | 1, d.p * (d.p + 1) / 2};
    const size_t smem = lay.bytes(WARPS);
    const int64_t per_sm = warp_fit_residency<T, Src, WARPS>(lay) / WARPS;
    const int64_t need = (v + WARPS - 1) / WARPS;
    const int64_t waves = launch_setting("log.warp.waves") > 0 ? launch_setting("log.warp.waves") : 4;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(need, int64_t(sm_count()) * std::max<int64_t>(per_sm, 1) * waves));
    LaunchScope scope("fit_log_warp_kernel", stream);
    fit_log_warp_kernel<T, Src, WARPS><<<unsigned(grid), WARPS * 32, smem, stream>>>(
        d, src, v, weighted, max_rw, T(tol), params, broke, iterations, violators);
    cuda_check(cudaGetLastError(), "fit_log_warp_kernel launch");
}

template <class T, class Src>
void launch_warp_impl(const LogDesignDevice<T>& d, const Src& src, int64_t v, int weighted, int max_rw,
                      double tol, double* params, uint8_t* broke, int32_t* iterations,
                      const ViolatorList<T>& violators, cudaStream_t stream) {
    const WarpLayout<T> lay{d.n, d.p, d.p | 1, d.p * (d.p + 1) / 2};
    require(lay.bytes(kWarps) <= 227 * 1024, "the design is too large for the shared-memory log fit");
    // The warps per CTA that keep the most warps resident (the fewest on a tie).
    const int64_t r4 = warp_fit_residency<T, Src, 4>(lay), r8 = warp_fit_residency<T, Src, 8>(lay),
                  r16 = warp_fit_residency<T, Src, 16>(lay);
    if (r16 > std::max(r4, r8))
        launch_warp_w<T, Src, 16>(d, src, v, weighted, max_rw, tol, params, broke, iterations, violators, stream);
    else if (r8 > r4)
        launch_warp_w<T, Src, 8>(d, src, v, weighted, max_rw, tol, params, broke, iterations, violators, stream);
    else
        launch_warp_w<T, Src, 4>(d, src, v, weighted, max_rw, tol, params, broke, iterations, violators, stream);
}

}  // namespace

template <class T>
void launch_log_warp(const LogDesignDevice<T>& d, const LogSource& src, int64_t v, int weighted, int max_rw,
                     double tol, double* params, uint8_t* broke, int32_t* iterations,
                     const ViolatorList<T>& violators, cudaStream_t stream) {
    launch_warp_impl<T, LogSource>(d, src, v, weighted, max_rw, tol, params, broke, iterations, violators, stream);
}

template <class T>
void launch_log_warp(const LogDesignDevice<T>& d, const CappedSource& src, int64_t v, int weighted, int max_rw,
                     double tol, double* params, uint8_t* broke, int32_t* iterations,
                     const ViolatorList<T>& violators, cudaStream_t stream) {
    launch_warp_impl<T, CappedSource>(d, src, v, weighted, max_rw, tol, params, broke, iterations, violators,
                                      stream);
}

size_t batch_log_warp_smem(int n_max, int p, int warps) {
    return WarpLayout<double>{n_max, p, p | 1, p * (p + 1) / 2}.bytes(warps);
}

int batch_log_warp_warps(int n_max, int p) {
    for (int warps : {12, 8, 4})
        if (batch_log_warp_smem(n_max, p, warps) <= 227 * 1024) return warps;
    return 0;
}

template <int WARPS>
void launch_batch_log_warp_impl(const DkiBatchJob* jobs, const int64_t* first, int n_jobs, size_t smem,
                                int64_t tickets, int weighted, int max_rw, double tol, int* queue,
                                const BatchViolators& violators, cudaStream_t stream) {
    auto kernel = batch_log_warp_kernel<WARPS>;
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "cudaFuncSetAttribute");
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, WARPS * 32, smem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    const int64_t grid = std::min<int64_t>(tickets, int64_t(sm_count()) * std::max(per_sm, 1));
    cuda_check(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), stream), "cudaMemsetAsync");
    LaunchScope scope("batch_log_warp_kernel", stream);
    kernel<<<unsigned(grid), WARPS * 32, smem, stream>>>(jobs, first, n_jobs, weighted, max_rw, tol, queue,
                                                         violators);
    cuda_check(cudaGetLastError(), "batch_log_warp_kernel launch");
}

void launch_batch_log_warp(const DkiBatchJob* jobs, const int64_t* first, int n_jobs, int n_max, int p, int warps,
                           int64_t tickets, int weighted, int max_rw, double tol, int* queue,
                           const BatchViolators& violators, cudaStream_t stream) {
    if (n_jobs == 0 || tickets == 0) return;
    const size_t smem = batch_log_warp_smem(n_max, p, warps);
    require(smem <= 227 * 1024, "the design is too large for the shared-memory log fit");
    if (warps == 12)
        launch_batch_log_warp_impl<12>(jobs, first, n_jobs, smem, tickets, weighted, max_rw, tol, queue, violators,
                                       stream);
    else if (warps == 8)
        launch_batch_log_warp_impl<8>(jobs, first, n_jobs, smem, tickets, weighted, max_rw, tol, queue, violators,
                                      stream);
    else
        launch_batch_log_warp_impl<4>(jobs, first, n_jobs, smem, tickets, weighted, max_rw, tol, queue, violators,
                                      stream);
}

template void launch_log_warp<double>(const LogDesignDevice<double>&, const LogSource&, int64_t, int, int, double,
                                      double*, uint8_t*, int32_t*, const ViolatorList<double>&, cudaStream_t);
template void launch_log_warp<float>(const LogDesignDevice<float>&, const LogSource&, int64_t, int, int, double,
                                     double*, uint8_t*, int32_t*, const ViolatorList<float>&, cudaStream_t);
template void launch_log_warp<double>(const LogDesignDevice<double>&, const CappedSource&, int64_t, int, int,
                                      double, double*, uint8_t*, int32_t*, const ViolatorList<double>&,
                                      cudaStream_t);
template void launch_log_warp<float>(const LogDesignDevice<float>&, const CappedSource&, int64_t, int, int,
                                     double, double*, uint8_t*, int32_t*, const ViolatorList<float>&,
                                     cudaStream_t);

}  // namespace lar
