// FOD amplitudes on a sphere grid to spherical-harmonic coefficients on the GPU: the SD fit's
// _to_sh step (src/larmor/sd/model.py:412-440), which least-squares fits the basis to each
// voxel's amplitudes (fit_sh, src/larmor/sd/sh.py:134) and scales by the grid's density; with
// exact_integral c00 is the amplitudes' sum / sqrt(4 pi).
//
// The basis matrix has full column rank, so the least-squares coefficients are pinv(B) a: the
// host forms P = density pinv(B) (ncoef, ca) once per (grid, lmax, basis), and the kernel is a
// tiled FP64 product over 32 voxels x 48 coefficients per CTA, each coefficient summed over
// the directions in increasing order.

#include <cmath>
#include <memory>
#include <vector>

#include "common.cuh"

namespace lar {
namespace {

constexpr int kShVoxels = 32;
constexpr int kShCoeffs = 48;
constexpr int kShDepth = 16;

// out(v, k) = sum_j P(k, j) a(v, j) for 32 voxels x 48 coefficients: 128 threads as 8 voxel
// lanes x 16 coefficient lanes, 4 x 3 outputs each.
__global__ void __launch_bounds__(128) project_sh_kernel(const double* __restrict__ amp, int64_t v, int64_t lda,
                                                         int ca, const double* __restrict__ pt, int ncoef,
                                                         int exact_integral, double* __restrict__ out,
                                                         int64_t ldo) {
    __shared__ double a_t[kShDepth][kShVoxels + 1];
    __shared__ double p_t[kShDepth][kShCoeffs];
    const int tid = threadIdx.x, tv = tid & 7, tc = tid >> 3;
    const int64_t v0 = int64_t(blockIdx.x) * kShVoxels;
    const int k0 = blockIdx.y * kShCoeffs;
    double acc[4][3], sum[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        sum[a] = 0.0;
#pragma unroll
        for (int b = 0; b < 3; ++b) acc[a][b] = 0.0;
    }
    for (int j0 = 0; j0 < ca; j0 += kShDepth) {
        const int depth = min(kShDepth, ca - j0);
        for (int e = tid; e < kShVoxels * kShDepth; e += 128) {
            const int vv = e / kShDepth, jj = e % kShDepth;
            const int64_t voxel = v0 + vv;
            a_t[jj][vv] = (voxel < v && jj < depth) ? amp[voxel * lda + j0 + jj] : 0.0;
        }
        for (int e = tid; e < kShDepth * kShCoeffs; e += 128) {
            const int jj = e / kShCoeffs, kk = e % kShCoeffs;
            p_t[jj][kk] = (jj < depth && k0 + kk < ncoef) ? pt[size_t(j0 + jj) * ncoef + k0 + kk] : 0.0;
        }
        __syncthreads();
        for (int jj = 0; jj < depth; ++jj) {
            double av[4], pv[3];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = a_t[jj][tv + 8 * a];
#pragma unroll
            for (int b = 0; b < 3; ++b) pv[b] = p_t[jj][tc + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                sum[a] += av[a];
#pragma unroll
                for (int b = 0; b < 3; ++b) acc[a][b] = fma(pv[b], av[a], acc[a][b]);
            }
        }
        __syncthreads();
    }
    // 1 / sqrt(4 pi), the l = 0 basis function's value.
    const double y00 = 0.28209479177387814;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int64_t voxel = v0 + tv + 8 * a;
        if (voxel >= v) continue;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const int k = k0 + tc + 16 * b;
            if (k >= ncoef) continue;
            out[voxel * ldo + k] = (exact_integral && k == 0) ? sum[a] * y00 : acc[a][b];
        }
    }
}

}  // namespace
}  // namespace lar

// The projector of one (sphere grid, lmax, basis): P transposed on the device.
struct lar_sh_projector_s {
    int64_t ncoef = 0, ca = 0;
    lar::DeviceArray<double> pt;  // (ca, ncoef)
};

using namespace lar;

extern "C" {

int lar_sh_projector_create(const double* projector, int64_t ncoef, int64_t ca, lar_sh_projector* out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        require(projector != nullptr && ncoef > 0 && ca > 0, "projector must be a non-empty (ncoef, ca) array");
        auto h = std::make_unique<lar_sh_projector_s>();
        h->ncoef = ncoef;
        h->ca = ca;
        std::vector<double> pt(size_t(ncoef * ca));
        for (int64_t k = 0; k < ncoef; ++k)
            for (int64_t j = 0; j < ca; ++j) pt[size_t(j * ncoef + k)] = projector[k * ca + j];
        h->pt.upload(pt.data(), pt.size());
        *out = h.release();
    });
}

void lar_sh_projector_destroy(lar_sh_projector projector) { delete projector; }

int lar_project_sh(lar_sh_projector projector, const double* amplitudes, int64_t v, int64_t lda,
                   int exact_integral, double* out, int64_t ldo, void* stream) {
    return guarded([&] {
        require(projector != nullptr, "projector must not be NULL");
        require(v >= 0, "v must be at least 0");
        require(lda >= projector->ca && ldo >= projector->ncoef,
                "lda must be at least the directions and ldo at least the coefficients");
        if (v == 0) return;
        require(amplitudes != nullptr && out != nullptr, "amplitudes and out must not be NULL");
        auto st = static_cast<cudaStream_t>(stream);
        const dim3 grid(unsigned((v + kShVoxels - 1) / kShVoxels), unsigned((projector->ncoef + kShCoeffs - 1) / kShCoeffs));
        LaunchScope scope("project_sh_kernel", st);
        project_sh_kernel<<<grid, 128, 0, st>>>(amplitudes, v, lda, int(projector->ca), projector->pt.ptr,
                                                int(projector->ncoef), exact_integral, out, ldo);
        cuda_check(cudaGetLastError(), "project_sh_kernel launch");
    });
}

}  // extern "C"
