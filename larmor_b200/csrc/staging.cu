// Device input staging of the voxelwise fits: the masked voxels' samples of a DWI volume read
// on the device from the raw volume, with the reference's input preparation
// (src/larmor/dwi/inputs.py):
// - the float32 conversion and the float32 scaling by slope and intercept of Volume.as_float /
//   signal_rows (src/larmor/types/volume.py:116-123, src/larmor/dwi/inputs.py:137-172);
// - estimate_s0: the mean b0, and for a mask voxel whose mean b0 is at or below its mean
//   diffusion-weighted signal, the mean S0 of the plausible mask voxels in its 3x3x3, else
//   5x5x5, neighbourhood, NaN when there is none (src/larmor/dwi/inputs.py:78-134);
// - largest_finite_signal and the per-voxel floor of floor_bad_samples
//   (src/larmor/dwi/inputs.py:212-252);
// - the SD models' S0-normalised signals, capped at 1 (src/larmor/sd/model.py:184-200).
//
// Mapping: one warp per voxel reads its contiguous row of N samples (the volume is C-ordered
// (X, Y, Z, N)), writes the scaled row and reduces its b0 and total sums in FP64, its largest
// finite sample and whether all are finite. A grid map of mask indices then lets one thread per
// dark-b0 voxel visit its neighbourhoods. HBM-bound: each sample is read once.

#include <cmath>
#include <cstring>
#include <vector>

#include <math_constants.h>

#include "common.cuh"

namespace lar {
namespace {

constexpr uint8_t kNotFinite = 0, kPlausible = 1, kRepair = 2;

template <class T>
__device__ __forceinline__ float to_float(T x) {
    return float(x);
}
template <>
__device__ __forceinline__ float to_float<double>(double x) {
    return __double2float_rn(x);
}
template <>
__device__ __forceinline__ float to_float<int32_t>(int32_t x) {
    return __int2float_rn(x);
}
template <>
__device__ __forceinline__ float to_float<uint32_t>(uint32_t x) {
    return __uint2float_rn(x);
}

template <class T>
__global__ void __launch_bounds__(256) stage_gather_kernel(const T* __restrict__ volume, int64_t n, float slope,
                                                           float intercept, int scale,
                                                           const int64_t* __restrict__ voxels, int64_t v,
                                                           const uint8_t* __restrict__ is_b0, int n_b0,
                                                           float* __restrict__ signals, double* __restrict__ s0_raw,
                                                           uint8_t* __restrict__ state, double* __restrict__ row_max,
                                                           uint8_t* __restrict__ finite) {
    const int lane = threadIdx.x & 31;
    const int64_t i = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (i >= v) return;
    const T* row = volume + voxels[i] * n;
    float* out = signals + i * n;
    double b0 = 0.0, all = 0.0, mx = -CUDART_INF;
    bool ok = true;
    for (int64_t j = lane; j < n; j += 32) {
        float x = to_float<T>(row[j]);
        // Two float32 roundings, as numpy's x *= slope; x += intercept (no fused multiply-add).
        if (scale) x = __fadd_rn(__fmul_rn(x, slope), intercept);
        out[j] = x;
        const double d = x;
        all += d;
        if (is_b0[j]) b0 += d;
        if (isfinite(x))
            mx = fmax(mx, d);
        else
            ok = false;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        all += __shfl_xor_sync(0xffffffffu, all, o);
        b0 += __shfl_xor_sync(0xffffffffu, b0, o);
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    ok = __all_sync(0xffffffffu, ok);
    if (lane != 0) return;
    row_max[i] = mx;
    finite[i] = ok;
    if (n_b0 == 0) return;
    const double s0 = b0 / n_b0;
    s0_raw[i] = s0;
    const int64_t n_dw = n - n_b0;
    if (n_dw == 0) {
        state[i] = kPlausible;  // no diffusion weighting: the mean b0 as it is
        return;
    }
    const double mean_dw = (all - b0) / double(n_dw);
    state[i] = !(isfinite(s0) && isfinite(mean_dw)) ? kNotFinite : (s0 > mean_dw ? kPlausible : kRepair);
}

__global__ void stage_index_kernel(const int64_t* __restrict__ voxels, int64_t v, int* __restrict__ index) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < v) index[voxels[i]] = int(i);
}

// S0 of each mask voxel: its mean b0, or for a dark-b0 voxel the mean S0 of the plausible mask
// voxels within 3x3x3, else 5x5x5 (outside the grid counts as none), NaN when there is none.
__global__ void __launch_bounds__(128) stage_repair_kernel(const int64_t* __restrict__ voxels, int64_t v, int64_t ny,
                                                           int64_t nz, int64_t nx, const int* __restrict__ index,
                                                           const double* __restrict__ s0_raw,
                                                           const uint8_t* __restrict__ state, double* __restrict__ s0) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= v) return;
    if (state[i] != kRepair) {
        s0[i] = s0_raw[i];
        return;
    }
    const int64_t flat = voxels[i];
    const int64_t z = flat % nz, y = (flat / nz) % ny, x = flat / (nz * ny);
    double value = CUDART_NAN;
    for (int r = 1; r <= 2; ++r) {
        double sum = 0.0;
        int count = 0;
        for (int64_t a = max(x - r, int64_t(0)); a <= min(x + r, nx - 1); ++a)
            for (int64_t b = max(y - r, int64_t(0)); b <= min(y + r, ny - 1); ++b)
                for (int64_t c = max(z - r, int64_t(0)); c <= min(z + r, nz - 1); ++c) {
                    const int j = index[(a * ny + b) * nz + c];
                    if (j >= 0 && state[j] == kPlausible) {
                        sum += s0_raw[j];
                        ++count;
                    }
                }
        if (count > 0) {
            value = sum / count;
            break;
        }
    }
    s0[i] = value;
}

// largest_finite_signal: the largest finite sample of all rows, or 1 when none is positive;
// then each voxel's floor, 1e-3 S0 where S0 is finite and positive, else 1e-3 largest.
__global__ void __launch_bounds__(1024) stage_floor_kernel(const double* __restrict__ row_max, int64_t v,
                                                           const double* __restrict__ s0, double* __restrict__ floor,
                                                           double* __restrict__ largest) {
    __shared__ double warp_max[32];
    double mx = -CUDART_INF;
    for (int64_t i = threadIdx.x; i < v; i += blockDim.x) mx = fmax(mx, row_max[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        mx = warp_max[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (threadIdx.x == 0) warp_max[0] = mx > 0.0 ? mx : 1.0;
    }
    __syncthreads();
    const double big = warp_max[0];
    if (threadIdx.x == 0 && largest) *largest = big;
    for (int64_t i = threadIdx.x; i < v; i += blockDim.x) {
        const bool usable = s0 && isfinite(s0[i]) && s0[i] > 0.0;
        floor[i] = 1e-3 * (usable ? s0[i] : big);
    }
}

__global__ void __launch_bounds__(256) normalise_kernel(const float* __restrict__ signals, const double* __restrict__ s0,
                                                        int64_t v, int64_t n, double* __restrict__ out,
                                                        uint8_t* __restrict__ finite) {
    const int lane = threadIdx.x & 31;
    const int64_t i = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (i >= v) return;
    const double d = s0[i];
    bool ok = true;
    for (int64_t j = lane; j < n; j += 32) {
        const double q = double(signals[i * n + j]) / d;
        ok &= bool(isfinite(q));
        out[i * n + j] = fmin(q, 1.0);
    }
    ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) finite[i] = ok;
}

template <class T>
void launch_gather(const void* volume, int64_t n, float slope, float intercept, int scale, const int64_t* voxels,
                   int64_t v, const uint8_t* is_b0, int n_b0, float* signals, double* s0_raw, uint8_t* state,
                   double* row_max, uint8_t* finite, cudaStream_t st) {
    const unsigned blocks = unsigned((v * 32 + 255) / 256);
    stage_gather_kernel<T><<<blocks, 256, 0, st>>>(static_cast<const T*>(volume), n, slope, intercept, scale, voxels,
                                                   v, is_b0, n_b0, signals, s0_raw, state, row_max, finite);
}

// out(voxels[i], r) = values(r, i): the rows of a map-major (rows, v) array put back on the grid,
// voxel-major (grid, rows), as unmask does on the host (src/larmor/dwi/mask.py:139). Consecutive
// threads take consecutive voxels of one row: coalesced reads, writes strided by `rows`.
__global__ void __launch_bounds__(256) unmask_rows_kernel(const float* __restrict__ values, int64_t rows, int64_t v,
                                                          const int64_t* __restrict__ voxels, float* __restrict__ out) {
    const int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= rows * v) return;
    const int64_t r = e / v, i = e - r * v;
    out[voxels[i] * rows + r] = values[e];
}

}  // namespace
}  // namespace lar

using namespace lar;

extern "C" {

int lar_stage_dwi(const void* volume, int dtype, int64_t nx, int64_t ny, int64_t nz, int64_t n, double slope,
                  double intercept, const int64_t* voxels, int64_t v, const uint8_t* is_b0, float* signals, double* s0,
                  uint8_t* finite, double* floor, double* largest, void* stream) {
    return guarded([&] {
        require(nx > 0 && ny > 0 && nz > 0 && n > 0, "the volume must have a non-empty (X, Y, Z, N) shape");
        require(nx * ny * nz < (int64_t(1) << 31), "the grid must have fewer than 2^31 voxels");
        require(v >= 0 && v <= nx * ny * nz, "v must be between 0 and the grid's voxel count");
        require(is_b0 != nullptr, "is_b0 must not be NULL");
        require(dtype >= LAR_DTYPE_F32 && dtype <= LAR_DTYPE_U32, "unknown dtype code");
        int n_b0 = 0;
        for (int64_t j = 0; j < n; ++j) n_b0 += is_b0[j] != 0;
        require(n_b0 == 0 || s0 != nullptr, "s0 must not be NULL for a table with b0s");
        if (v == 0) return;
        auto st = static_cast<cudaStream_t>(stream);
        // Scaling as signal_rows: only when it is not the identity (Volume makes a slope of 0 or
        // not finite the identity).
        float fslope = float(slope), fintercept = float(intercept);
        const int scale = std::isfinite(slope) && slope != 0.0 && (slope != 1.0 || intercept != 0.0);
        // Workspace: the b0 flags, the raw S0, per-voxel states, row maxima and the grid map.
        const int64_t grid = nx * ny * nz;
        const size_t bytes = size_t(n) + size_t(v) * (8 + 1 + 8) + size_t(grid) * 4 + 256;
        char* ws = nullptr;
        cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&ws), bytes, st), "cudaMallocAsync");
        auto* s0_raw = reinterpret_cast<double*>(ws);
        auto* row_max = s0_raw + v;
        auto* index = reinterpret_cast<int*>(row_max + v);
        auto* state = reinterpret_cast<uint8_t*>(index + grid);
        auto* flags = state + v;
        std::vector<uint8_t> host_flags(static_cast<size_t>(n));
        for (int64_t j = 0; j < n; ++j) host_flags[size_t(j)] = is_b0[j] != 0;
        cuda_check(cudaMemcpyAsync(flags, host_flags.data(), size_t(n), cudaMemcpyHostToDevice, st), "cudaMemcpyAsync");
        {
            LaunchScope scope("stage_gather_kernel", st);
            switch (dtype) {
                case LAR_DTYPE_F32: launch_gather<float>(volume, n, fslope, fintercept, scale, voxels, v, flags, n_b0, signals, s0_raw, state, row_max, finite, st); break;
                case LAR_DTYPE_F64: launch_gather<double>(volume, n, fslope, fintercept, scale, voxels, v, flags, n_b0, signals, s0_raw, state, row_max, finite, st); break;
                case LAR_DTYPE_I16: launch_gather<int16_t>(volume, n, fslope, fintercept, scale, voxels, v, flags, n_b0, signals, s0_raw, state, row_max, finite, st); break;
                case LAR_DTYPE_U16: launch_gather<uint16_t>(volume, n, fslope, fintercept, scale, voxels, v, flags, n_b0, signals, s0_raw, state, row_max, finite, st); break;
                case LAR_DTYPE_I8: launch_gather<int8_t>(volume, n, fslope, fintercept, scale, voxels, v, flags, n_b0, signals, s0_raw, state, row_max, finite, st); break;
                case LAR_DTYPE_U8: launch_gather<uint8_t>(volume, n, fslope, fintercept, scale, voxels, v, flags, n_b0, signals, s0_raw, state, row_max, finite, st); break;
                case LAR_DTYPE_I32: launch_gather<int32_t>(volume, n, fslope, fintercept, scale, voxels, v, flags, n_b0, signals, s0_raw, state, row_max, finite, st); break;
                default: launch_gather<uint32_t>(volume, n, fslope, fintercept, scale, voxels, v, flags, n_b0, signals, s0_raw, state, row_max, finite, st);
            }
            cuda_check(cudaGetLastError(), "stage_gather_kernel launch");
        }
        if (n_b0 > 0) {
            cuda_check(cudaMemsetAsync(index, 0xFF, size_t(grid) * 4, st), "cudaMemsetAsync");
            {
                LaunchScope scope("stage_index_kernel", st);
                stage_index_kernel<<<unsigned((v + 255) / 256), 256, 0, st>>>(voxels, v, index);
                cuda_check(cudaGetLastError(), "stage_index_kernel launch");
            }
            LaunchScope scope("stage_repair_kernel", st);
            stage_repair_kernel<<<unsigned((v + 127) / 128), 128, 0, st>>>(voxels, v, ny, nz, nx, index, s0_raw,
                                                                            state, s0);
            cuda_check(cudaGetLastError(), "stage_repair_kernel launch");
        }
        if (floor) {
            LaunchScope scope("stage_floor_kernel", st);
            stage_floor_kernel<<<1, 1024, 0, st>>>(row_max, v, n_b0 > 0 ? s0 : nullptr, floor, largest);
            cuda_check(cudaGetLastError(), "stage_floor_kernel launch");
        }
        cuda_check(cudaFreeAsync(ws, st), "cudaFreeAsync");
    });
}

int lar_unmask_rows(const float* values, int64_t rows, int64_t v, const int64_t* voxels, int64_t grid, float* out,
                    void* stream) {
    return guarded([&] {
        require(rows >= 1 && v >= 0 && grid >= v, "rows must be at least 1 and v between 0 and the grid's size");
        if (v == 0) return;
        require(values && voxels && out, "values, voxels and out must not be NULL");
        auto st = static_cast<cudaStream_t>(stream);
        LaunchScope scope("unmask_rows_kernel", st);
        const int64_t total = rows * v;
        unmask_rows_kernel<<<unsigned((total + 255) / 256), 256, 0, st>>>(values, rows, v, voxels, out);
        cuda_check(cudaGetLastError(), "unmask_rows_kernel launch");
    });
}

int lar_normalise_signals(const float* signals, const double* s0, int64_t v, int64_t n, double* normalised,
                          uint8_t* finite, void* stream) {
    return guarded([&] {
        require(v >= 0 && n > 0, "v must be at least 0 and n at least 1");
        if (v == 0) return;
        auto st = static_cast<cudaStream_t>(stream);
        LaunchScope scope("normalise_kernel", st);
        normalise_kernel<<<unsigned((v * 32 + 255) / 256), 256, 0, st>>>(signals, s0, v, n, normalised, finite);
        cuda_check(cudaGetLastError(), "normalise_kernel launch");
    });
}

}  // extern "C"
