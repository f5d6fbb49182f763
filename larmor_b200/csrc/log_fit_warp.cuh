// The warp-per-voxel log fit and the constrained re-fit of its violators (see
// log_fit_warp.cu, constrained_fit.cu).
#pragma once

#include <cstdint>

#include "log_fit.cuh"

namespace lar {

// A compacted list of the voxels whose unconstrained solution breaks a constraint: their
// indices and scaled parameters, filled by atomic append. Entries past `capacity` are dropped
// (the count still counts them; the caller sizes the list for every voxel).
template <class T>
struct ViolatorList {
    int* count = nullptr;
    int capacity = 0;
    int64_t* voxel = nullptr;
    double* params = nullptr;  // (capacity, p) scaled parameters
};

template <class T>
void launch_log_warp(const LogDesignDevice<T>& d, const LogSource& src, int64_t v, int weighted, int max_rw,
                     double tol, double* params, uint8_t* broke, int32_t* iterations,
                     const ViolatorList<T>& violators, cudaStream_t stream);
template <class T>
void launch_log_warp(const LogDesignDevice<T>& d, const CappedSource& src, int64_t v, int weighted, int max_rw,
                     double tol, double* params, uint8_t* broke, int32_t* iterations,
                     const ViolatorList<T>& violators, cudaStream_t stream);

// Largest number of active NNLS columns the constrained re-fit keeps in its QR workspace.
constexpr int kMaxActive = 64;

// Doubles of global workspace one warp of the constrained re-fit uses.
inline size_t constrained_slot_doubles(int n, int p, int m) {
    return size_t(n) * p + size_t(p + 1) * m + size_t(p + 1) * kMaxActive + 2 * size_t(m) + 2 * size_t(n) +
           (2 * size_t(m) + 7) / 8 + 64;
}

// Re-fits the violators of `list` subject to g p >= 0 (cpp/src/dwi/log_fit.cpp:170-216), in
// FP64, writing the constrained parameters (divided by the column scales) over `params` where
// the re-fit succeeds. `workspace` holds `slots` warp slots of constrained_slot_doubles()
// doubles; `queue` is a device int the kernel uses as its work counter (zeroed by the caller).
// The warps of the constrained re-fit of designs of n measurements and p parameters that fit
// on the GPU at once (its grid's size), a multiple of 4.
int constrained_resident_warps(int n, int p);

template <class Src>
void launch_constrained(const LogDesignDevice<double>& d, const Src& src, int weighted,
                        const ViolatorList<double>& list, int list_count_host_bound, int* queue,
                        double* workspace, int slots, double* params, cudaStream_t stream);

}  // namespace lar
