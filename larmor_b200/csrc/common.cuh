// Shared definitions of the larmor_b200 CUDA library: status codes, the thread-local error
// message, device helpers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/larmor_b200.h"

namespace lar {

// The message of the last failed call on this host thread (lar_last_error).
void set_error(const std::string& message);

// Thrown by the C-ABI internals; the entry points turn it into a status code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw Error(LAR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

inline void require(bool ok, const std::string& message) {
    if (!ok) throw Error(LAR_ERR_INVALID, message);
}

// Runs f and maps exceptions to status codes for the C ABI.
template <class F>
int guarded(F&& f) {
    try {
        f();
        return LAR_OK;
    } catch (const Error& e) {
        set_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_error("out of host memory");
        return LAR_ERR_MEMORY;
    } catch (const std::exception& e) {
        set_error(e.what());
        return LAR_ERR_INVALID;
    }
}

// A device buffer owned by a design handle.
template <class T>
struct DeviceArray {
    T* ptr = nullptr;
    size_t count = 0;
    DeviceArray() = default;
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    ~DeviceArray() {
        if (ptr) cudaFree(ptr);
    }
    void upload(const T* host, size_t n) {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = n;
        if (n == 0) return;
        cuda_check(cudaMalloc(&ptr, n * sizeof(T)), "cudaMalloc");
        cuda_check(cudaMemcpy(ptr, host, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
    }
};

// Launch accounting: every kernel launch of the library is made inside a LaunchScope, which
// counts it and, while kernel timing is on (lar_kernel_timing), brackets it with CUDA events
// on its stream.
struct LaunchScope {
    LaunchScope(const char* name, cudaStream_t stream);
    ~LaunchScope();
    LaunchScope(const LaunchScope&) = delete;
    LaunchScope& operator=(const LaunchScope&) = delete;
    const char* name;
    cudaStream_t stream;
    cudaEvent_t start = nullptr;
};

// Launch settings (lar_set_launch_setting): 0 when a setting is unset, which keeps the
// library's own choice. A tuner sets them; results never depend on them.
int64_t launch_setting(const char* name);

// Resident CTAs per SM of a persistent grid: the occupancy limit, or less when the named setting
// asks for fewer.
inline int ctas_per_sm(int occupancy, const char* setting) {
    const int64_t want = launch_setting(setting);
    const int occ = occupancy > 0 ? occupancy : 1;
    return want > 0 && want < occ ? int(want) : occ;
}

inline int sm_count() {
    int dev = 0, n = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    return n;
}

// ---- device helpers --------------------------------------------------------------------

template <class T>
__device__ __forceinline__ T dev_exp(T x);
template <>
__device__ __forceinline__ double dev_exp<double>(double x) { return exp(x); }
template <>
__device__ __forceinline__ float dev_exp<float>(float x) { return expf(x); }

template <class T>
__device__ __forceinline__ T dev_log(T x);
template <>
__device__ __forceinline__ double dev_log<double>(double x) { return log(x); }
template <>
__device__ __forceinline__ float dev_log<float>(float x) { return logf(x); }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

}  // namespace lar
