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

struct lar_log_design_s {
    lar::host::LogDesignHost host;
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

// ---- signal sources ---------------------------------------------------------------------
//
// A CTA owns `count` consecutive voxels, whose rows are contiguous in memory: it copies them
// into shared memory with coalesced loads, then each thread turns its own row into log
// signals (T) in a thread-strided shared array ys[j * BLOCK + tid], computed once per voxel.

// log_s (v, n) double, as larmor._core.fit_log_signal receives it.
struct LogSource {
    const double* log_s;
    int64_t n;
    static constexpr int raw_bytes = 8;
    template <class T, int BLOCK>
    __device__ __forceinline__ void stage(int64_t first, int count, unsigned char* raw, T* ys) const {
        const double* src = log_s + first * n;
        double* dst = reinterpret_cast<double*>(raw);
        const int total = count * int(n);
        for (int i = threadIdx.x; i < total; i += BLOCK) dst[i] = src[i];
        __syncthreads();
        if (threadIdx.x < count)
            for (int j = 0; j < n; ++j) ys[j * BLOCK + threadIdx.x] = T(dst[threadIdx.x * n + j]);
    }
};

// float32 signals (v, n) with a per-voxel floor for samples that are not finite and positive
// (src/larmor/dwi/inputs.py:227-252), logged in T.
struct FlooredSource {
    const float* s;
    const double* floor;
    int64_t n;
    static constexpr int raw_bytes = 4;
    template <class T, int BLOCK>
    __device__ __forceinline__ void stage(int64_t first, int count, unsigned char* raw, T* ys) const {
        const float* src = s + first * n;
        float* dst = reinterpret_cast<float*>(raw);
        const int total = count * int(n);
        for (int i = threadIdx.x; i < total; i += BLOCK) dst[i] = src[i];
        __syncthreads();
        if (threadIdx.x < count) {
            const T log_floor = dev_log<T>(T(floor[first + threadIdx.x]));
            for (int j = 0; j < n; ++j) {
                const float v = dst[threadIdx.x * n + j];
                ys[j * BLOCK + threadIdx.x] = (isfinite(v) && v > 0.0f) ? dev_log<T>(T(v)) : log_floor;
            }
        }
    }
};

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

// ---- DTI maps ---------------------------------------------------------------------------

// Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations (Jacobi 1846;
// Golub & Van Loan 8.5): eigenvalues in w, eigenvectors in the columns of q.
template <class T>
__device__ __forceinline__ T eps_of();
template <>
__device__ __forceinline__ double eps_of<double>() { return 2.220446049250313e-16; }
template <>
__device__ __forceinline__ float eps_of<float>() { return 1.1920929e-07f; }

template <class T>
__device__ __forceinline__ void jacobi3(T (&a)[3][3], T (&w)[3], T (&q)[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) q[i][j] = i == j ? T(1) : T(0);
    for (int sweep = 0; sweep < 12; ++sweep) {
        bool rotated = false;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0;
            const int r = pq == 0 ? 1 : 2;
            const T apq = a[p][r];
            const T app = a[p][p], arr = a[r][r];
            // An off-diagonal entry below rounding of its diagonal pair is zero.
            if (fabs(apq) <= T(1e-3) * eps_of<T>() * (fabs(app) + fabs(arr)) ||
                apq == T(0)) {
                a[p][r] = a[r][p] = T(0);
                continue;
            }
            rotated = true;
            const T theta = (arr - app) / (T(2) * apq);
            const T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
            const T c = T(1) / sqrt(t * t + T(1));
            const T s = t * c;
            a[p][p] = app - t * apq;
            a[r][r] = arr + t * apq;
            a[p][r] = a[r][p] = T(0);
            const int o = 3 - p - r;
            const T aop = a[o][p], aor = a[o][r];
            a[o][p] = a[p][o] = c * aop - s * aor;
            a[o][r] = a[r][o] = s * aop + c * aor;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const T qp = q[i][p], qr = q[i][r];
                q[i][p] = c * qp - s * qr;
                q[i][r] = s * qp + c * qr;
            }
        }
        if (!rotated) break;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) w[i] = a[i][i];
}

template <class T>
__device__ __forceinline__ T zero_nan(T x) { return isnan(x) ? T(0) : x; }

// The maps of compute_dti_metrics (src/larmor/dwi/dti.py:170-235) of one voxel's tensor
// elements d (xx, xy, xz, yy, yz, zz), written as 16 rows of maps (stride v).
template <class T>
__device__ __forceinline__ void dti_maps(const T (&d)[6], int64_t voxel, int64_t v,
                                         float* __restrict__ maps, uint8_t* __restrict__ npd) {
    T ev[3] = {T(0), T(0), T(0)};
    T pe[3] = {T(NAN), T(NAN), T(NAN)};
    bool finite = true;
#pragma unroll
    for (int i = 0; i < 6; ++i) finite &= isfinite(d[i]);
    if (finite) {
        T a[3][3] = {{d[0], d[1], d[2]}, {d[1], d[3], d[4]}, {d[2], d[4], d[5]}};
        T w[3], q[3][3];
        jacobi3<T>(a, w, q);
        // Descending order by a sorting network on (value, column) pairs; selects keep
        // everything in registers.
        T c0[3] = {q[0][0], q[1][0], q[2][0]}, c1[3] = {q[0][1], q[1][1], q[2][1]},
          c2[3] = {q[0][2], q[1][2], q[2][2]};
        T w0 = w[0], w1 = w[1], w2 = w[2];
        auto swap_if = [](T& wa, T (&ca)[3], T& wb, T (&cb)[3]) {
            const bool s = wa < wb;
            const T t = wa; wa = s ? wb : wa; wb = s ? t : wb;
#pragma unroll
            for (int i = 0; i < 3; ++i) { const T u = ca[i]; ca[i] = s ? cb[i] : ca[i]; cb[i] = s ? u : cb[i]; }
        };
        swap_if(w0, c0, w1, c1);
        swap_if(w1, c1, w2, c2);
        swap_if(w0, c0, w1, c1);
        ev[0] = w0; ev[1] = w1; ev[2] = w2;
#pragma unroll
        for (int i = 0; i < 3; ++i) pe[i] = c0[i];
    }
    const T l1 = zero_nan(ev[0]), l2 = zero_nan(ev[1]), l3 = zero_nan(ev[2]);
    const T md = zero_nan((d[0] + d[3] + d[5]) / T(3));
    const T num_sq = (l1 - l2) * (l1 - l2) + (l2 - l3) * (l2 - l3) + (l3 - l1) * (l3 - l1);
    const T num = sqrt(fmax(num_sq, T(0)));
    const T den = sqrt(l1 * l1 + l2 * l2 + l3 * l3);
    T fa = den > T(1e-12) ? sqrt(T(0.5)) * (num / den) : T(0);
    fa = zero_nan(fmin(fmax(fa, T(0)), T(1)));
#pragma unroll
    for (int i = 0; i < 6; ++i) maps[i * v + voxel] = float(d[i]);
    maps[6 * v + voxel] = float(fa);
    maps[7 * v + voxel] = float(md);
    maps[8 * v + voxel] = float(l1);
    maps[9 * v + voxel] = float((l2 + l3) / T(2));
#pragma unroll
    for (int i = 0; i < 3; ++i) maps[(10 + i) * v + voxel] = float(pe[i]);
    maps[13 * v + voxel] = float(l1);
    maps[14 * v + voxel] = float(l2);
    maps[15 * v + voxel] = float(l3);
    npd[voxel] = l3 <= T(0) ? 1 : 0;
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

template <class T>
const LogDesignDevice<T>& device_view(const lar_log_design_s* h);
template <>
const LogDesignDevice<double>& device_view<double>(const lar_log_design_s* h) { return h->d64; }
template <>
const LogDesignDevice<float>& device_view<float>(const lar_log_design_s* h) { return h->d32; }

constexpr int kSmallBlock = 64;

template <class Kernel>
void set_smem(Kernel kernel, size_t bytes) {
    require(bytes <= 227 * 1024, "the design has too many measurements for the shared-memory fit");
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)),
               "cudaFuncSetAttribute");
}

template <class T>
void launch_fit(const lar_log_design_s* h, const double* log_s, int64_t v, int weighted,
                int max_rw, double tol, double* params, uint8_t* broke, int32_t* iterations,
                cudaStream_t stream) {
    const auto& d = device_view<T>(h);
    const int p = int(h->host.p);
    if (p == 7 && h->host.m == 0) {
        LogSource src{log_s, h->host.n};
        const size_t sm = SmallFit<T, 7>::bytes(d.n, kSmallBlock, LogSource::raw_bytes);
        auto kernel = fit_log_small_kernel<T, 7, kSmallBlock, LogSource>;
        set_smem(kernel, sm);
        const int64_t grid = (v + kSmallBlock - 1) / kSmallBlock;
        kernel<<<unsigned(grid), kSmallBlock, sm, stream>>>(d, src, v, weighted, max_rw, T(tol), params,
                                                            broke, iterations);
        cuda_check(cudaGetLastError(), "fit_log_small_kernel launch");
        return;
    }
    throw Error(LAR_ERR_INVALID, "this build fits designs with p = 7 and no constraints; got p = " +
                                     std::to_string(p) + ", m = " + std::to_string(h->host.m));
}

template <class T>
void launch_dti_maps(const lar_log_design_s* h, const float* s, const double* floor, int64_t v,
                     int weighted, int max_rw, double tol, float* maps, uint8_t* npd,
                     double* params, cudaStream_t stream) {
    const auto& d = device_view<T>(h);
    FlooredSource src{s, floor, h->host.n};
    const size_t sm = SmallFit<T, 7>::bytes(d.n, kSmallBlock, FlooredSource::raw_bytes);
    auto kernel = fit_dti_maps_kernel<T, kSmallBlock>;
    set_smem(kernel, sm);
    const int64_t grid = (v + kSmallBlock - 1) / kSmallBlock;
    kernel<<<unsigned(grid), kSmallBlock, sm, stream>>>(d, src, v, weighted, max_rw, T(tol), maps, npd, params);
    cuda_check(cudaGetLastError(), "fit_dti_maps_kernel launch");
}

template <class T>
void upload_design(lar_log_design_s* h, DeviceArray<T>& x, DeviceArray<T>& pinvt, DeviceArray<T>& z,
                   DeviceArray<T>& g, DeviceArray<T>& scales, LogDesignDevice<T>& view) {
    const auto& hd = h->host;
    const int64_t n = hd.n, p = hd.p, m = hd.m, pp = p * (p + 1) / 2;
    std::vector<T> xv(static_cast<size_t>(n * p)), pt(static_cast<size_t>(n * p)), zv(static_cast<size_t>(n * pp)),
        gv(static_cast<size_t>(m * p)), sv(static_cast<size_t>(p));
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
    for (size_t i = 0; i < gv.size(); ++i) gv[i] = T(hd.g[i]);
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
    view.scales = scales.ptr;
}

}  // namespace

}  // namespace lar

using namespace lar;

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

}  // extern "C"
