// Log-signal least-squares fits of DTI and DKI on the GPU: ordinary, iteratively reweighted
// (IRLS) and, for DKI, re-fitted under constraints. Follows the per-voxel algorithm of
// cpp/src/dwi/log_fit.cpp (reweighted_fit :114-147, fit_log_signal_block :245-269) and the
// maps of src/larmor/dwi/dti.py:170-235.
//
// Layout: the masked signals are (v, n) row-major, one voxel's n samples contiguous, as the
// reference's chunk arrays are. The per-table design (unit-norm columns X (n, p), its
// pseudo-inverse, the products Z[n][ab] = X_na X_nb of the normal matrix, constraints) is small
// and shared by every voxel: each CTA stages it once into shared memory.
//
// DTI (p = 7): one thread per voxel. Each thread accumulates its 28 normal-matrix entries and
// 7 right-hand sides in registers over the measurements (design operands are warp-uniform
// shared-memory broadcasts), solves the 7 x 7 system by LU with partial pivoting in registers,
// and finishes with the tensor's eigen-decomposition (cyclic Jacobi) and the DTI maps.

#include <cmath>
#include <cstdio>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "host_la.hpp"
#include "log_fit.cuh"
#include "batch.cuh"
#include "log_fit_warp.cuh"
#include "tensor_maps.cuh"

// Device scratch of a design handle: the violator list and the constrained re-fit's warp
// slots, grown on demand. Calls on one handle must not overlap on the GPU.
struct LogScratch {
    void* base = nullptr;
    size_t bytes = 0;
    ~LogScratch() {
        if (base) cudaFree(base);
    }
    void* reserve(size_t need) {
        if (need > bytes) {
            if (base) lar::cuda_check(cudaFree(base), "cudaFree");
            base = nullptr;
            bytes = 0;
            lar::cuda_check(cudaMalloc(&base, need), "cudaMalloc (log-fit scratch)");
            bytes = need;
        }
        return base;
    }
};

struct lar_log_design_s {
    lar::host::LogDesignHost host;
    LogScratch scratch;
    lar::LogDesignDevice<double> d64;
    lar::LogDesignDevice<float> d32;
    lar::DeviceArray<double> x64, pinvt64, z64, g64, scales64;
    lar::DeviceArray<float> x32, pinvt32, z32, g32, scales32;
};

namespace lar {

namespace {

// ---- per-thread helpers ----------------------------------------------------------------

template <class T, int P>
__device__ __forceinline__ bool all_finite(const T (&v)[P]) {
    bool ok = true;
#pragma unroll
    for (int i = 0; i < P; ++i) ok &= isfinite(v[i]);
    return ok;
}

// ---- the small-p thread-per-voxel IRLS --------------------------------------------------

template <class T, int P>
struct SmallFit {
    static constexpr int PP = P * (P + 1) / 2;
    // Shared memory: x, z, pinv^T (T), the CTA's log signals (T), its raw rows.
    static size_t bytes(int n, int block, int raw_bytes) {
        return size_t(n) * (2 * P + PP) * sizeof(T) + size_t(n) * block * sizeof(T) +
               size_t(n) * block * raw_bytes + 16;
    }
};

// Packed index of (a, b), a <= b, in the upper triangle stored row by row.
__host__ __device__ constexpr int packed(int a, int b, int p) { return a * p - a * (a - 1) / 2 + (b - a); }

// Solves the symmetric system g x = b (g packed, P x P) in place in b by L D L^T. Returns false
// when a pivot is exactly zero, the weighted normal equations being singular (weights that
// underflow to zero on most measurements), as the reference's zero LU pivot test does
// (cpp/src/dwi/log_fit.cpp:128-133).
template <class T, int P>
__device__ __forceinline__ bool ldlt_solve(T (&g)[P * (P + 1) / 2], T (&b)[P]) {
    // In place: g(j, j) <- d_j, g(j, i) (j < i) <- L(i, j).
    bool ok = true;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        T d = g[packed(j, j, P)];
#pragma unroll
        for (int k = 0; k < j; ++k) {
            const T l = g[packed(k, j, P)];
            d = fma(-l * g[packed(k, k, P)], l, d);
        }
        ok &= (d != T(0));
        g[packed(j, j, P)] = d;
        const T inv = T(1) / d;
#pragma unroll
        for (int i = j + 1; i < P; ++i) {
            T s = g[packed(j, i, P)];
#pragma unroll
            for (int k = 0; k < j; ++k) s = fma(-g[packed(k, i, P)] * g[packed(k, k, P)], g[packed(k, j, P)], s);
            g[packed(j, i, P)] = s * inv;
        }
    }
    if (!ok) return false;
#pragma unroll
    for (int i = 0; i < P; ++i)
#pragma unroll
        for (int k = 0; k < i; ++k) b[i] = fma(-g[packed(k, i, P)], b[k], b[i]);
#pragma unroll
    for (int i = 0; i < P; ++i) b[i] = b[i] / g[packed(i, i, P)];
#pragma unroll
    for (int i = P - 1; i >= 0; --i)
#pragma unroll
        for (int k = i + 1; k < P; ++k) b[i] = fma(-g[packed(i, k, P)], b[k], b[i]);
    return true;
}

// Fits one voxel from its log signals ys[j * stride] and leaves its scaled parameters in p;
// returns the number of weighted fits. Follows reweighted_fit (cpp/src/dwi/log_fit.cpp:114-147)
// from the ordinary fit pinv y (:251).
template <class T, int P>
__device__ __forceinline__ int fit_voxel_small(const T* __restrict__ xs, const T* __restrict__ zs,
                                               const T* __restrict__ pinvt, int n,
                                               const T* __restrict__ ys, int stride, bool weighted,
                                               int max_rw, T tol, T (&p)[P]) {
    constexpr int PP = P * (P + 1) / 2;
    T ord[P];
#pragma unroll
    for (int a = 0; a < P; ++a) ord[a] = T(0);
#pragma unroll 2
    for (int j = 0; j < n; ++j) {
        const T y = ys[j * stride];
#pragma unroll
        for (int a = 0; a < P; ++a) ord[a] = fma(pinvt[j * P + a], y, ord[a]);
    }
#pragma unroll
    for (int a = 0; a < P; ++a) p[a] = ord[a];
    if (!weighted || !all_finite(ord)) return 0;

    T mx = -INFINITY;
#pragma unroll 2
    for (int j = 0; j < n; ++j) {
        T pred = T(0);
#pragma unroll
        for (int a = 0; a < P; ++a) pred = fma(xs[j * P + a], p[a], pred);
        mx = fmax(mx, pred);
    }
    int it = 0;
    for (; it < max_rw; ++it) {
        T g[PP], r[P];
#pragma unroll
        for (int k = 0; k < PP; ++k) g[k] = T(0);
#pragma unroll
        for (int a = 0; a < P; ++a) r[a] = T(0);
#pragma unroll 2
        for (int j = 0; j < n; ++j) {
            T pred = T(0);
#pragma unroll
            for (int a = 0; a < P; ++a) pred = fma(xs[j * P + a], p[a], pred);
            const T w = dev_exp<T>(T(2) * (pred - mx));
            const T wy = w * ys[j * stride];
#pragma unroll
            for (int k = 0; k < PP; ++k) g[k] = fma(w, zs[j * PP + k], g[k]);
#pragma unroll
            for (int a = 0; a < P; ++a) r[a] = fma(wy, xs[j * P + a], r[a]);
        }
        if (!ldlt_solve<T, P>(g, r) || !all_finite(r)) {
#pragma unroll
            for (int a = 0; a < P; ++a) p[a] = ord[a];
            return it + 1;
        }
        T change = T(0), mx_next = -INFINITY;
#pragma unroll 2
        for (int j = 0; j < n; ++j) {
            T po = T(0), pn = T(0);
#pragma unroll
            for (int a = 0; a < P; ++a) {
                po = fma(xs[j * P + a], p[a], po);
                pn = fma(xs[j * P + a], r[a], pn);
            }
            change = fmax(change, fabs(pn - po));
            mx_next = fmax(mx_next, pn);
        }
#pragma unroll
        for (int a = 0; a < P; ++a) p[a] = r[a];
        mx = mx_next;
        if (!(change > tol)) return it + 1;
    }
    return it;
}

// Stages x (n, p), z (n, pp) and pinv^T (n, p) into shared memory; returns the end.
template <class T, int P>
__device__ __forceinline__ T* stage_design(const LogDesignDevice<T>& d, T* sm) {
    constexpr int PP = P * (P + 1) / 2;
    const int n = d.n;
    for (int i = threadIdx.x; i < n * P; i += blockDim.x) sm[i] = d.x[i];
    for (int i = threadIdx.x; i < n * PP; i += blockDim.x) sm[n * P + i] = d.z[i];
    for (int i = threadIdx.x; i < n * P; i += blockDim.x) sm[n * (P + PP) + i] = d.pinvt[i];
    return sm + n * (2 * P + PP);
}

template <class T, int P, int BLOCK, class Src>
__global__ void __launch_bounds__(BLOCK) fit_log_small_kernel(LogDesignDevice<T> d, Src src, int64_t v,
                                                              int weighted, int max_rw, T tol,
                                                              double* __restrict__ params,
                                                              uint8_t* __restrict__ broke,
                                                              int32_t* __restrict__ iterations) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    constexpr int PP = P * (P + 1) / 2;
    const int n = d.n;
    T* ys = stage_design<T, P>(d, sm);
    unsigned char* raw = reinterpret_cast<unsigned char*>(ys + n * BLOCK);
    const int64_t first = int64_t(blockIdx.x) * BLOCK;
    const int count = int(v - first < int64_t(BLOCK) ? v - first : int64_t(BLOCK));
    src.template stage<T, BLOCK>(first, count, raw, ys);
    __syncthreads();
    if (threadIdx.x >= count) return;
    const int64_t voxel = first + threadIdx.x;
    T p[P];
    const int it = fit_voxel_small<T, P>(sm, sm + n * P, sm + n * (P + PP), n, ys + threadIdx.x, BLOCK,
                                         weighted != 0, max_rw, tol, p);
#pragma unroll
    for (int a = 0; a < P; ++a) params[voxel * P + a] = double(p[a]) / d.scales64[a];
    broke[voxel] = 0;
    if (iterations) iterations[voxel] = it;
}

template <class T, int BLOCK>
__global__ void __launch_bounds__(BLOCK) fit_dti_maps_kernel(LogDesignDevice<T> d, FlooredSource src,
                                                             int64_t v, int weighted, int max_rw, T tol,
                                                             float* __restrict__ maps,
                                                             uint8_t* __restrict__ npd,
                                                             double* __restrict__ params) {
    constexpr int P = 7, PP = 28;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    const int n = d.n;
    T* ys = stage_design<T, P>(d, sm);
    unsigned char* raw = reinterpret_cast<unsigned char*>(ys + n * BLOCK);
    const int64_t first = int64_t(blockIdx.x) * BLOCK;
    const int count = int(v - first < int64_t(BLOCK) ? v - first : int64_t(BLOCK));
    src.template stage<T, BLOCK>(first, count, raw, ys);
    __syncthreads();
    if (threadIdx.x >= count) return;
    const int64_t voxel = first + threadIdx.x;
    T p[P];
    fit_voxel_small<T, P>(sm, sm + n * P, sm + n * (P + PP), n, ys + threadIdx.x, BLOCK, weighted != 0,
                          max_rw, tol, p);
    T dt[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) dt[a] = p[a + 1] / d.scales[a + 1];
    if (params) {
#pragma unroll
        for (int a = 0; a < P; ++a) params[voxel * P + a] = double(p[a]) / d.scales64[a];
    }
    dti_maps<T>(dt, voxel, v, maps, npd);
}

// The DTI family of a batch (batch.cuh): a persistent grid whose CTAs take tickets of
// kDtiBatchBlock voxels of one volume from a device counter across every DTI volume; a CTA
// restages the design when its ticket moves to another volume. Per voxel the same fit and maps
// as fit_dti_maps_kernel (FP64).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) batch_dti_kernel(const DtiBatchJob* __restrict__ jobs,
                                                          const int64_t* __restrict__ first, int n_jobs,
                                                          int weighted, int max_rw, double tol,
                                                          int* __restrict__ queue) {
    using T = double;
    constexpr int P = 7;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ long long ticket;
    T* sm = reinterpret_cast<T*>(smem_raw);
    const int64_t total = first[n_jobs];
    int cur = -1;
    for (;;) {
        if (threadIdx.x == 0) ticket = atomicAdd(reinterpret_cast<unsigned long long*>(queue), 1ull);
        __syncthreads();
        const int64_t t = ticket;
        if (t >= total) break;
        const int j = ticket_job(first, n_jobs, t);
        const DtiBatchJob& job = jobs[j];
        const LogDesignDevice<T> d = job.d;
        const int n = d.n;
        T* ys = sm + n * (2 * P + P * (P + 1) / 2);
        if (j != cur) {
            stage_design<T, P>(d, sm);
            cur = j;
        }
        unsigned char* raw = reinterpret_cast<unsigned char*>(ys + n * BLOCK);
        const int64_t v = job.v;
        const int64_t block_first = (t - first[j]) * BLOCK;
        const int count = int(v - block_first < int64_t(BLOCK) ? v - block_first : int64_t(BLOCK));
        const FlooredSource src{job.s, job.floor, n};
        src.template stage<T, BLOCK>(block_first, count, raw, ys);
        __syncthreads();
        if (threadIdx.x < count) {
            const int64_t voxel = block_first + threadIdx.x;
            T p[P];
            fit_voxel_small<T, P>(sm, sm + n * P, sm + n * (P + P * (P + 1) / 2), n, ys + threadIdx.x, BLOCK,
                                  weighted != 0, max_rw, T(tol), p);
            T dt[6];
#pragma unroll
            for (int a = 0; a < 6; ++a) dt[a] = p[a + 1] / d.scales[a + 1];
            dti_maps<T>(dt, voxel, v, job.maps, job.npd);
        }
        __syncthreads();
    }
}

template <class T>
const LogDesignDevice<T>& device_view(const lar_log_design_s* h);
template <>
const LogDesignDevice<double>& device_view<double>(const lar_log_design_s* h) { return h->d64; }
template <>
const LogDesignDevice<float>& device_view<float>(const lar_log_design_s* h) { return h->d32; }

// Voxels per CTA of the shared-memory fits: 64, or 32 / 16 when the design and a CTA's signals
// of 64 voxels do not fit in shared memory (tables of more than about 200 measurements).
inline int small_block(int n, int raw_bytes, size_t per_value) {
    auto fits = [&](int block) {
        return size_t(n) * (2 * 7 + 28) * per_value + size_t(n) * block * per_value + size_t(n) * block * raw_bytes +
                   16 <= 227 * 1024;
    };
    const int64_t want = launch_setting("dti.voxels_per_cta");
    if ((want == 16 || want == 32 || want == 64) && fits(int(want))) return int(want);
    for (int block : {64, 32, 16}) {
        const size_t bytes = size_t(n) * (2 * 7 + 28) * per_value + size_t(n) * block * per_value +
                             size_t(n) * block * raw_bytes + 16;
        if (bytes <= 227 * 1024) return block;
    }
    return 16;
}

template <class Kernel>
void set_smem(Kernel kernel, size_t bytes) {
    require(bytes <= 227 * 1024, "the design has too many measurements for the shared-memory fit");
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)),
               "cudaFuncSetAttribute");
}

// Scratch layout for a constrained fit of v voxels: [count, queue] ints, voxel ids, scaled
// parameters, then the warp slots of the re-fit.
struct ScratchPlan {
    size_t ids_off, params_off, slots_off, total;
    int slots;
};

inline ScratchPlan plan_scratch(const lar::host::LogDesignHost& h, int64_t v) {
    ScratchPlan s{};
    const size_t align = 256;
    auto up = [&](size_t x) { return (x + align - 1) / align * align; };
    s.ids_off = align;
    s.params_off = up(s.ids_off + size_t(v) * sizeof(int64_t));
    s.slots_off = up(s.params_off + size_t(v) * h.p * sizeof(double));
    // As many warp slots as warps of the re-fit fit on the GPU at once.
    const int64_t cap = constrained_resident_warps(int(h.n), int(h.p));
    s.slots = int(std::max<int64_t>(4, std::min<int64_t>((v + 3) / 4 * 4, cap)));
    s.total = s.slots_off + size_t(s.slots) * constrained_slot_doubles(int(h.n), int(h.p), int(h.m)) * sizeof(double);
    return s;
}

template <class T, class Src>
void launch_general(lar_log_design_s* h, const Src& src, int64_t v, int weighted, int max_rw, double tol,
                    double* params, uint8_t* broke, int32_t* iterations, cudaStream_t stream) {
    const auto& d = device_view<T>(h);
    require(h->host.p <= 32, "the log fit takes at most 32 parameters");
    ViolatorList<T> vl;
    ViolatorList<double> vl64;
    ScratchPlan plan{};
    char* base = nullptr;
    if (h->host.m > 0) {
        require(h->host.p <= 31, "the constrained log fit takes at most 31 parameters");
        require(v < (int64_t(1) << 31), "at most 2^31 - 1 voxels per constrained call");
        plan = plan_scratch(h->host, v);
        base = static_cast<char*>(h->scratch.reserve(plan.total));
        cuda_check(cudaMemsetAsync(base, 0, 2 * sizeof(int), stream), "cudaMemsetAsync");
        vl.count = reinterpret_cast<int*>(base);
        vl.capacity = int(v);
        vl.voxel = reinterpret_cast<int64_t*>(base + plan.ids_off);
        vl.params = reinterpret_cast<double*>(base + plan.params_off);
        vl64.count = vl.count;
        vl64.capacity = vl.capacity;
        vl64.voxel = vl.voxel;
        vl64.params = vl.params;
    }
    launch_log_warp<T>(d, src, v, weighted, max_rw, tol, params, broke, iterations, vl, stream);
    if (h->host.m > 0) {
        launch_constrained<Src>(h->d64, src, weighted, vl64, int(v), reinterpret_cast<int*>(base) + 1,
                                reinterpret_cast<double*>(base + plan.slots_off), plan.slots, params, stream);
    }
}

template <class T>
void launch_fit(lar_log_design_s* h, const double* log_s, int64_t v, int weighted,
                int max_rw, double tol, double* params, uint8_t* broke, int32_t* iterations,
                cudaStream_t stream) {
    const auto& d = device_view<T>(h);
    const int p = int(h->host.p);
    LogSource src{log_s, h->host.n};
    if (p == 7 && h->host.m == 0) {
        auto run = [&](auto kernel, int block) {
            const size_t sm = SmallFit<T, 7>::bytes(d.n, block, LogSource::raw_bytes);
            set_smem(kernel, sm);
            const int64_t grid = (v + block - 1) / block;
            LaunchScope scope("fit_log_small_kernel", stream);
            kernel<<<unsigned(grid), block, sm, stream>>>(d, src, v, weighted, max_rw, T(tol), params, broke,
                                                          iterations);
            cuda_check(cudaGetLastError(), "fit_log_small_kernel launch");
        };
        const int block = small_block(d.n, LogSource::raw_bytes, sizeof(T));
        if (block == 64) run(fit_log_small_kernel<T, 7, 64, LogSource>, 64);
        else if (block == 32) run(fit_log_small_kernel<T, 7, 32, LogSource>, 32);
        else run(fit_log_small_kernel<T, 7, 16, LogSource>, 16);
        return;
    }
    launch_general<T>(h, src, v, weighted, max_rw, tol, params, broke, iterations, stream);
}

template <class T>
void launch_dti_maps(const lar_log_design_s* h, const float* s, const double* floor, int64_t v,
                     int weighted, int max_rw, double tol, float* maps, uint8_t* npd,
                     double* params, cudaStream_t stream) {
    const auto& d = device_view<T>(h);
    FlooredSource src{s, floor, h->host.n};
    auto run = [&](auto kernel, int block) {
        const size_t sm = SmallFit<T, 7>::bytes(d.n, block, FlooredSource::raw_bytes);
        set_smem(kernel, sm);
        const int64_t grid = (v + block - 1) / block;
        LaunchScope scope("fit_dti_maps_kernel", stream);
        kernel<<<unsigned(grid), block, sm, stream>>>(d, src, v, weighted, max_rw, T(tol), maps, npd, params);
        cuda_check(cudaGetLastError(), "fit_dti_maps_kernel launch");
    };
    const int block = small_block(d.n, FlooredSource::raw_bytes, sizeof(T));
    if (block == 64) run(fit_dti_maps_kernel<T, 64>, 64);
    else if (block == 32) run(fit_dti_maps_kernel<T, 32>, 32);
    else run(fit_dti_maps_kernel<T, 16>, 16);
}

}  // namespace

size_t batch_dti_smem(int n_max) { return SmallFit<double, 7>::bytes(n_max, kDtiBatchBlock, FlooredSource::raw_bytes); }

void launch_batch_dti(const DtiBatchJob* jobs, const int64_t* first, int n_jobs, int n_max, int64_t tickets,
                      int weighted, int max_rw, double tol, int* queue, cudaStream_t stream) {
    if (n_jobs == 0 || tickets == 0) return;
    auto kernel = batch_dti_kernel<kDtiBatchBlock>;
    const size_t sm = batch_dti_smem(n_max);
    set_smem(kernel, sm);
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kDtiBatchBlock, sm),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    const int64_t grid = std::min<int64_t>(tickets, int64_t(sm_count()) * std::max(per_sm, 1));
    cuda_check(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), stream), "cudaMemsetAsync");
    LaunchScope scope("batch_dti_kernel", stream);
    kernel<<<unsigned(grid), kDtiBatchBlock, sm, stream>>>(jobs, first, n_jobs, weighted, max_rw, tol, queue);
    cuda_check(cudaGetLastError(), "batch_dti_kernel launch");
}

namespace {

template <class T>
void upload_design(lar_log_design_s* h, DeviceArray<T>& x, DeviceArray<T>& pinvt, DeviceArray<T>& z,
                   DeviceArray<T>& g, DeviceArray<T>& scales, LogDesignDevice<T>& view) {
    const auto& hd = h->host;
    const int64_t n = hd.n, p = hd.p, m = hd.m, pp = p * (p + 1) / 2;
    std::vector<T> xv(static_cast<size_t>(n * p)), pt(static_cast<size_t>(n * p)), zv(static_cast<size_t>(n * pp)),
        gv(static_cast<size_t>(2 * m * p)), sv(static_cast<size_t>(p));
    for (int64_t i = 0; i < n; ++i)
        for (int64_t a = 0; a < p; ++a) {
            xv[size_t(i * p + a)] = T(hd.x[size_t(i * p + a)]);
            pt[size_t(i * p + a)] = T(hd.pinv[size_t(a * n + i)]);
        }
    for (int64_t i = 0; i < n; ++i) {
        int64_t k = 0;
        for (int64_t a = 0; a < p; ++a)
            for (int64_t b = a; b < p; ++b) zv[size_t(i * pp + k++)] = T(hd.x[size_t(i * p + a)] * hd.x[size_t(i * p + b)]);
    }
    // g (m, p) row-major, then its transpose (p, m).
    for (int64_t c = 0; c < m; ++c)
        for (int64_t a = 0; a < p; ++a) {
            gv[size_t(c * p + a)] = T(hd.g[size_t(c * p + a)]);
            gv[size_t(m * p + a * m + c)] = T(hd.g[size_t(c * p + a)]);
        }
    for (int64_t a = 0; a < p; ++a) sv[size_t(a)] = T(hd.scales[size_t(a)]);
    x.upload(xv.data(), xv.size());
    pinvt.upload(pt.data(), pt.size());
    z.upload(zv.data(), zv.size());
    g.upload(gv.data(), gv.size());
    scales.upload(sv.data(), sv.size());
    view.n = int(n);
    view.p = int(p);
    view.m = int(m);
    view.x = x.ptr;
    view.pinvt = pinvt.ptr;
    view.z = z.ptr;
    view.g = g.ptr;
    view.gt = m > 0 ? g.ptr + m * p : nullptr;
    view.scales = scales.ptr;
}

}  // namespace

void launch_dki_maps(const double* params, int64_t v, float* maps, uint8_t* npd, cudaStream_t stream);

}  // namespace lar

using namespace lar;

namespace lar {
LogDesignDevice<double> log_design_view(const lar_log_design_s* h) { return h->d64; }
}  // namespace lar

extern "C" {

int lar_log_design_create(const double* x, int64_t n, int64_t p, const double* g, int64_t m,
                          lar_log_design* out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        require(x != nullptr && n > 0 && p > 0, "x must be a non-empty (n, p) array");
        require(m >= 0 && (m == 0 || g != nullptr), "g must be (m, p) with m >= 0");
        require(n >= p, "x must be (n, p) with n >= p: got (" + std::to_string(n) + ", " + std::to_string(p) + ")");
        auto h = std::make_unique<lar_log_design_s>();
        h->host = host::prepare_log_design(x, n, p, g, m);
        upload_design<double>(h.get(), h->x64, h->pinvt64, h->z64, h->g64, h->scales64, h->d64);
        upload_design<float>(h.get(), h->x32, h->pinvt32, h->z32, h->g32, h->scales32, h->d32);
        h->d64.scales64 = h->scales64.ptr;
        h->d32.scales64 = h->scales64.ptr;
        *out = h.release();
    });
}

void lar_log_design_destroy(lar_log_design design) { delete design; }

int lar_log_design_violators(lar_log_design design, int64_t* count) {
    return guarded([&] {
        require(design != nullptr && count != nullptr, "design and count must not be NULL");
        int n = 0;
        if (design->host.m > 0 && design->scratch.base != nullptr)
            cuda_check(cudaMemcpy(&n, design->scratch.base, sizeof(int), cudaMemcpyDeviceToHost),
                       "cudaMemcpy (violator count)");
        *count = n;
    });
}

int lar_fit_log_signal(lar_log_design design, const double* log_s, int64_t v, int weighted,
                       int64_t max_iter, double tol, int precision, double* params,
                       uint8_t* broke, int32_t* iterations, void* stream) {
    return guarded([&] {
        require(design != nullptr, "design must not be NULL");
        require(v >= 0, "v must be at least 0");
        require(max_iter >= 0, "max_iter must be at least 0");
        require(precision == LAR_FP64 || precision == LAR_FP32, "precision must be LAR_FP64 or LAR_FP32");
        if (v == 0) return;
        require(log_s && params && broke, "log_s, params and broke must not be NULL");
        const int rw = int(std::min<int64_t>(max_iter, 1 << 20));
        auto s = static_cast<cudaStream_t>(stream);
        if (precision == LAR_FP64)
            launch_fit<double>(design, log_s, v, weighted, rw, tol, params, broke, iterations, s);
        else
            launch_fit<float>(design, log_s, v, weighted, rw, tol, params, broke, iterations, s);
    });
}

int lar_fit_dti_maps(lar_log_design design, const float* signals, const double* floor,
                     int64_t v, int weighted, int64_t max_iter, double tol, int precision,
                     float* maps, uint8_t* npd, double* params, void* stream) {
    return guarded([&] {
        require(design != nullptr, "design must not be NULL");
        require(design->host.p == 7 && design->host.m == 0,
                "the DTI maps need the 7-column DTI design without constraints");
        require(v >= 0, "v must be at least 0");
        require(max_iter >= 0, "max_iter must be at least 0");
        require(precision == LAR_FP64 || precision == LAR_FP32, "precision must be LAR_FP64 or LAR_FP32");
        if (v == 0) return;
        require(signals && floor && maps && npd, "signals, floor, maps and npd must not be NULL");
        const int rw = int(std::min<int64_t>(max_iter, 1 << 20));
        auto s = static_cast<cudaStream_t>(stream);
        if (precision == LAR_FP64)
            launch_dti_maps<double>(design, signals, floor, v, weighted, rw, tol, maps, npd, params, s);
        else
            launch_dti_maps<float>(design, signals, floor, v, weighted, rw, tol, maps, npd, params, s);
    });
}

int lar_dki_maps(const double* params, int64_t v, float* maps, uint8_t* npd, void* stream) {
    return guarded([&] {
        require(v >= 0, "v must be at least 0");
        if (v == 0) return;
        require(params && maps && npd, "params, maps and npd must not be NULL");
        launch_dki_maps(params, v, maps, npd, static_cast<cudaStream_t>(stream));
    });
}

int lar_fit_dki_maps(lar_log_design design, const float* signals, const double* s0, const double* floor,
                     const uint8_t* is_b0, int64_t v, int weighted, int64_t max_iter, double tol,
                     int precision, float* maps, uint8_t* npd, uint8_t* broke, double* params,
                     void* stream) {
    return guarded([&] {
        require(design != nullptr, "design must not be NULL");
        require(design->host.p == 22, "the DKI maps need the 22-column DKI design");
        require(v >= 0, "v must be at least 0");
        require(max_iter >= 0, "max_iter must be at least 0");
        require(precision == LAR_FP64 || precision == LAR_FP32, "precision must be LAR_FP64 or LAR_FP32");
        if (v == 0) return;
        require(signals && floor && is_b0 && maps && npd && broke && params,
                "signals, floor, is_b0, maps, npd, broke and params must not be NULL");
        const int rw = int(std::min<int64_t>(max_iter, 1 << 20));
        auto st = static_cast<cudaStream_t>(stream);
        CappedSource src{signals, s0, floor, is_b0, design->host.n};
        if (precision == LAR_FP64)
            launch_general<double>(design, src, v, weighted, rw, tol, params, broke, nullptr, st);
        else
            launch_general<float>(design, src, v, weighted, rw, tol, params, broke, nullptr, st);
        launch_dki_maps(params, v, maps, npd, st);
    });
}

}  // extern "C"
