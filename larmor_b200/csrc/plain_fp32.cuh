// The plain single-precision multi-tissue fit (the comparison baseline of the FP64 path): the
// interface between the SD handles (multi_tissue.cu) and its kernel (plain_fp32.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace lar {

// One resolution's matrices in FP32: the solver's weighted kernel and Gram matrix, the deconv
// kernel's unweighted anisotropic kernel (transposed) and isotropic columns.
struct PlainStage {
    int m, c, ci, nb;
    float tol;           // the NNLS gradient tolerance (the solver's tol_x)
    const float* k;      // (m, c) row-major, weighted
    const float* gram;   // (c, c): K^T K + ridge^2 I
    const float* kt;     // (c, m): the unweighted anisotropic kernel, transposed
    const float* iso;    // (m, ci) unweighted
    const float* wiso;   // (m, ci) weighted
    const int* blocks;   // (nb, 2)
};

// Largest sizes the plain kernel takes (its per-warp state lives in shared memory).
constexpr int kPlainMaxMeasurements = 512;
constexpr int kPlainMaxColumns = 320;
constexpr int kPlainMaxActive = 64;
constexpr int kPlainMaxGroups = 4;

// The LSI design of MSMT-CSD in FP32 (lsi.cu's matrices, the same layouts).
struct PlainLsi {
    int m, n, k;
    const float* qt;        // (m, n): q_t transposed
    const float* back;      // (n, n)
    const float* et;        // (n, k): E transposed
    const float* e;         // (k, n)
    const float* gram;      // (k, k): E E^T
    const float* abs_sums;  // (k,)
};

constexpr int kPlainLsiMaxConstraints = 512;
constexpr int kPlainLsiMaxParameters = 63;

void launch_plain_lsi(const PlainLsi& D, const float* signals, int64_t v, float* x, uint8_t* status,
                      cudaStream_t stream);

void launch_plain_fp32(const PlainStage& lr, const PlainStage& hr, const float* signals, int64_t v,
                       const float* weights, int max_rounds, float fraction_tol, float final_tol, float* fods,
                       float* fractions, int32_t* rounds, uint8_t* status, cudaStream_t stream);

}  // namespace lar
