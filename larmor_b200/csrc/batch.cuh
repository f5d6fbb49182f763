// Batches of volumes fitted through one work queue per model family (the batched-uneven
// workload: many volumes of different sizes, gradient tables and models).
//
// A family's volumes ("jobs") sit in a device job table. Each launch of a family stage covers
// every job of the family: its CTAs (or warps) take tickets from one device counter, a ticket
// being a block of voxels of one job. first[j] is job j's first ticket (first[n_jobs] the
// total), so the job of ticket t is the last j with first[j] <= t; a CTA whose ticket moves to
// another job restages that job's design. Uneven volumes and uneven per-voxel costs are absorbed
// by the one queue, as the reference's block queue does across a volume
// (cpp/src/common/parallel.hpp:26-84).
#pragma once

#include <cstdint>

#include "common.cuh"
#include "log_fit.cuh"

struct lar_log_design_s;

namespace lar {

// The FP64 device view of a prepared log-signal design (log_fit.cu).
LogDesignDevice<double> log_design_view(const lar_log_design_s* h);

// The job of ticket t: the last j in [0, n_jobs) with first[j] <= t (empty jobs are skipped).
__device__ __forceinline__ int ticket_job(const int64_t* __restrict__ first, int n_jobs, int64_t t) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// A DTI volume: floored float32 signals (v, n) in, the 16 maps (16, v) and the non-positive-
// definite flags out.
struct DtiBatchJob {
    LogDesignDevice<double> d;
    const float* s;
    const double* floor;
    int64_t v;
    float* maps;
    uint8_t* npd;
};

// A DKI volume: float32 signals (v, n) with S0, floors and the b0 mask (n,), as
// lar_fit_dki_maps takes them; the 36 maps, the flags, the broke flags and the parameters out.
struct DkiBatchJob {
    LogDesignDevice<double> d;
    const float* s;
    const double* s0;
    const double* floor;
    const uint8_t* is_b0;
    int64_t v;
    float* maps;
    uint8_t* npd;
    uint8_t* broke;
    double* params;
};

// The violators of a DKI batch: job, voxel and scaled unconstrained parameters per entry.
struct BatchViolators {
    int* count = nullptr;
    int capacity = 0;
    int* job = nullptr;
    int64_t* voxel = nullptr;
    double* params = nullptr;  // (capacity, p)
};

// Voxels per ticket of the family stages.
constexpr int kDtiBatchBlock = 32;   // one CTA of the DTI fit (thread per voxel)
constexpr int kDkiVoxelsPerWarp = 4;  // a ticket of the DKI log fit: 4 voxels per warp of its CTA
constexpr int kMapsBatchVoxels = 128;

// Launch shapes and shared memory of the family stages (sized for the largest table).
size_t batch_dti_smem(int n_max);
// Warps per CTA of the DKI log fit (12, 8 or 4; 0: the largest table does not fit) and its
// shared memory.
int batch_log_warp_warps(int n_max, int p);
size_t batch_log_warp_smem(int n_max, int p, int warps);
void launch_batch_dti(const DtiBatchJob* jobs, const int64_t* first, int n_jobs, int n_max, int64_t tickets,
                      int weighted, int max_rw, double tol, int* queue, cudaStream_t stream);
void launch_batch_log_warp(const DkiBatchJob* jobs, const int64_t* first, int n_jobs, int n_max, int p, int warps,
                           int64_t tickets, int weighted, int max_rw, double tol, int* queue,
                           const BatchViolators& violators, cudaStream_t stream);
size_t batch_refit_slot_doubles(int n_max, int p, int m_max);
int batch_refit_slots();
void launch_batch_refit(const DkiBatchJob* jobs, const BatchViolators& violators, int weighted, int* queue,
                        double* workspace, int slots, size_t slot_doubles, cudaStream_t stream);
void launch_batch_dki_maps(const DkiBatchJob* jobs, const int64_t* first, int n_jobs, int64_t tickets,
                           cudaStream_t stream);

// The multi-tissue (mFOD) family (multi_tissue.cu): the round kernels of lar_fit_multi_tissue,
// each launched once per round over every volume's list.
struct MfodBatch;
MfodBatch* mfod_batch_create();
void mfod_batch_destroy(MfodBatch* b);
void mfod_batch_add(MfodBatch* b, const double* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                    lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver, int64_t max_outer,
                    double fraction_tol, double final_tol_x, double* fods, double* fractions, int32_t* rounds,
                    uint8_t* status);
void mfod_batch_finalize(MfodBatch* b);
void mfod_batch_run(MfodBatch* b, cudaStream_t stream);

}  // namespace lar
