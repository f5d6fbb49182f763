// Damped Richardson-Lucy on the GPU (drl.cu): the solver's device matrices and the launcher the
// FOD solver handle uses.
#pragma once

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
};

// Whether drl_kernel takes c directions (1 to 320).
bool drl_fits(int c);

// The shared memory drl_kernel takes for c directions.
size_t drl_smem_bytes(int c);

// fods (v, c) of the signals (v, m), all device arrays: every voxel started at P.init.
void launch_drl(const DrlDev& P, const double* signals, int64_t v, double* fods, cudaStream_t stream);

}  // namespace lar
