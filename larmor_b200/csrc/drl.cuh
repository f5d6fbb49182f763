// Damped Richardson-Lucy on the GPU (drl.cu): the solver's device matrices and the launcher the
// FOD solver handle uses.
#pragma once

#include <vector>

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace lar {

// The dRL solver's matrices on the device (cpp/src/sd/drl.hpp:9-20, cpp/src/sd/solver.hpp).
struct DrlDev {
    const double* k_t;   // (c, m): K^T
    const double* gram;  // (c, c): K^T K
    int c, m, n_iter;
    double nu, init;
    // The tensor-core mode (LAR_TF32X3): K^T K split and laid out for drl_tc.cu, and a device
    // int where that kernel records a wait that ran out; null for the FP64 kernels.
    const float* gtc = nullptr;
    int* err = nullptr;
};

// The signal dRL deconvolves, entry i of voxel v: s(v, i) itself (a single-tissue fit), or the
// anisotropic part max(s(v, i) w_i - sum_t W_iso(i, t) f_iso(v, t), 0) of a multi-tissue round
// (cpp/src/sd/multi_tissue.cpp:68-72).
struct DrlSignal {
    const double* s;     // (v, m)
    const double* w;     // (m,) shell weights, or null: the plain signal
    const double* wiso;  // (m, ci): the weighted isotropic kernel
    const double* fiso;  // (v, ci): the isotropic fractions of the round
    int m, ci;
};

// Whether drl_kernel takes c directions (1 to 640).
bool drl_fits(int c);

// The tensor-core dRL (drl_tc.cu): whether it takes c directions (65 to 320), its shared
// memory, the layout of K^T K it reads (TF32 heads and remainders in 8-direction chunks), and
// its launch over a voxel list as launch_drl_listed.
bool drl_tc_fits(int c);
bool drl_tc_fits_measurements(int c, int m);
size_t drl_tc_smem_bytes(int c);
std::vector<float> drl_tc_layout(const double* gram, int c);
void launch_drl_tc(const DrlDev& P, const float* gtc, const DrlSignal& S, const int* list, int64_t count,
                   const int* count_dev, double* x, int64_t ldx, int* err, cudaStream_t st);

// The shared memory drl_kernel takes for c directions.
size_t drl_smem_bytes(int c);

// fods (v, c) of the signals (v, m), all device arrays: every voxel started at P.init.
void launch_drl(const DrlDev& P, const double* signals, int64_t v, double* fods, cudaStream_t stream);

// x(voxel, :) (row stride ldx) = the dRL FOD of each voxel list[p], p < count (the voxels
// 0..count-1 when list is null; count capped by *count_dev when that is given), every voxel
// started at P.init.
void launch_drl_listed(const DrlDev& P, const DrlSignal& S, const int* list, int64_t count, const int* count_dev,
                       double* x, int64_t ldx, cudaStream_t stream);

}  // namespace lar
