// Device view of a prepared log-signal design (see log_fit.cu).
#pragma once

#include <cstdint>

#include "common.cuh"

namespace lar {

template <class T>
struct LogDesignDevice {
    int n = 0, p = 0, m = 0;
    const T* x = nullptr;          // (n, p) unit-norm columns
    const T* pinvt = nullptr;      // (n, p) transposed pseudo-inverse
    const T* z = nullptr;          // (n, p(p+1)/2) products x_na x_nb, a <= b
    const T* g = nullptr;          // (m, p) constraints, column-scaled
    const T* gt = nullptr;         // (p, m) the same, transposed (lanes over constraints read it coalesced)
    const T* scales = nullptr;     // (p,) column norms
    const double* scales64 = nullptr;  // (p,) column norms in double, for the outputs
};

// ---- signal sources ---------------------------------------------------------------------
//
// A CTA owns `count` consecutive voxels, whose rows are contiguous in memory: it copies them
// into shared memory with coalesced loads, then each thread turns its own row into log
// signals (T) in a thread-strided shared array ys[j * BLOCK + tid], computed once per voxel.

// log_s (v, n) double, as larmor._core.fit_log_signal receives it.
struct LogSource {
    const double* log_s;
    int64_t n;
    // Warp-cooperative: ys[j] = y_j of one voxel, lanes over j (coalesced).
    template <class T>
    __device__ __forceinline__ void warp_stage(int64_t voxel, T* ys, int lane) const {
        for (int j = lane; j < n; j += 32) ys[j] = T(log_s[voxel * n + j]);
    }
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
    template <class T>
    __device__ __forceinline__ void warp_stage(int64_t voxel, T* ys, int lane) const {
        const T lf = dev_log<T>(T(floor[voxel]));
        for (int j = lane; j < n; j += 32) {
            const float x = s[voxel * n + j];
            ys[j] = (isfinite(x) && x > 0.0f) ? dev_log<T>(T(x)) : lf;
        }
    }
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

// float32 signals (v, n) prepared as DKIModel.fit does before its log fit
// (src/larmor/dwi/dki.py:243-250): where the voxel's S0 differs from the mean of its own b0s
// (relative 1e-9), the b0 samples become S0; diffusion-weighted samples are capped at S0; then
// samples that are not finite and positive become floor[voxel]. Without S0 (s0 == NULL) only
// the floor applies.
struct CappedSource {
    const float* s;
    const double* s0;      // (v,) or NULL
    const double* floor;   // (v,)
    const uint8_t* is_b0;  // (n,) device
    int64_t n;
    template <class T>
    __device__ __forceinline__ void warp_stage(int64_t voxel, T* ys, int lane) const {
        const T lf = dev_log<T>(T(floor[voxel]));
        if (s0 == nullptr) {
            for (int j = lane; j < n; j += 32) {
                const float x = s[voxel * n + j];
                ys[j] = (isfinite(x) && x > 0.0f) ? dev_log<T>(T(x)) : lf;
            }
            return;
        }
        const double s0v = s0[voxel];
        // The mean of the voxel's own b0s, summed in measurement order as numpy does for short
        // rows: lane 0 adds them up.
        double own = 0.0;
        int count = 0;
        if (lane == 0) {
            for (int j = 0; j < n; ++j)
                if (is_b0[j]) { own += double(s[voxel * n + j]); ++count; }
            own = count ? own / count : 0.0;
        }
        own = __shfl_sync(0xffffffffu, own, 0);
        const bool repaired = !(fabs(s0v - own) <= 1e-9 * fabs(own));
        for (int j = lane; j < n; j += 32) {
            double x = double(s[voxel * n + j]);
            if (is_b0[j]) {
                if (repaired) x = s0v;
            } else {
                x = isnan(x) ? x : fmin(x, s0v);
            }
            ys[j] = (isfinite(x) && x > 0.0) ? dev_log<T>(T(x)) : lf;
        }
    }
};

}  // namespace lar
