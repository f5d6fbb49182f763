// The C ABI of batches: many volumes of the DTI, DKI and multi-tissue (mFOD) models, each
// family fitted through one device work queue across all of its volumes (batch.cuh).
//
// Jobs are added family by family with device pointers to their inputs and outputs;
// lar_batch_finalize uploads the job tables and allocates the scratch the families use; after
// that lar_batch_run enqueues the stages of the chosen families on a stream with no allocation
// and no host synchronisation, so one CUDA graph can hold a whole batch.

#include <algorithm>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "batch.cuh"
#include "common.cuh"

namespace lar {
namespace {

struct CudaFree {
    void operator()(void* p) const {
        if (p) cudaFree(p);
    }
};

template <class T>
void upload_vector(DeviceArray<T>& dst, const std::vector<T>& src) {
    dst.upload(src.data(), src.size());
}

// Tickets of `block` voxels per job: first[j] and, last, the total.
std::vector<int64_t> ticket_starts(const std::vector<int64_t>& voxels, int64_t block) {
    std::vector<int64_t> first(voxels.size() + 1, 0);
    for (size_t j = 0; j < voxels.size(); ++j) first[j + 1] = first[j] + (voxels[j] + block - 1) / block;
    return first;
}

// The log-fit settings every job of a family shares.
struct LogFitSettings {
    int weighted = -1;
    int max_rw = 0;
    double tol = 0.0;
    void check(int w, int64_t max_iter, double t, const char* family) {
        const int rw = int(std::min<int64_t>(max_iter, 1 << 20));
        if (weighted < 0) {
            weighted = w != 0;
            max_rw = rw;
            tol = t;
            return;
        }
        require((w != 0) == (weighted != 0) && rw == max_rw && t == tol,
                std::string("every ") + family + " job of a batch takes the same weighted, max_iter and tol");
    }
};

}  // namespace
}  // namespace lar

using namespace lar;

struct lar_batch_s {
    bool finalized = false;
    // DTI
    LogFitSettings dti_fit;
    std::vector<DtiBatchJob> dti;
    DeviceArray<DtiBatchJob> d_dti;
    DeviceArray<int64_t> dti_first;
    int64_t dti_tickets = 0;
    int dti_nmax = 0;
    // DKI
    LogFitSettings dki_fit;
    std::vector<DkiBatchJob> dki;
    DeviceArray<DkiBatchJob> d_dki;
    DeviceArray<int64_t> dki_fit_first, dki_maps_first;
    int64_t dki_fit_tickets = 0, dki_maps_tickets = 0;
    int dki_nmax = 0, dki_mmax = 0, dki_warps = 0;
    BatchViolators violators;
    double* refit_slots = nullptr;
    int refit_nslots = 0;
    size_t refit_slot_doubles = 0;
    // mFOD
    std::unique_ptr<MfodBatch, void (*)(MfodBatch*)> mfod{nullptr, mfod_batch_destroy};
    // Device scratch: counters, then the violator list and the re-fit slots.
    std::unique_ptr<void, CudaFree> scratch;
    int* counters = nullptr;  // [0, 1] DTI queue, [2, 3] DKI fit queue, [4] violators, [5] re-fit queue
};

extern "C" {

int lar_batch_create(lar_batch* out) {
    return guarded([&] {
        require(out != nullptr, "out must not be NULL");
        *out = new lar_batch_s();
    });
}

void lar_batch_destroy(lar_batch batch) { delete batch; }

int lar_batch_add_dti(lar_batch batch, lar_log_design design, const float* signals, const double* floor, int64_t v,
                      int weighted, int64_t max_iter, double tol, float* maps, uint8_t* npd) {
    return guarded([&] {
        require(batch != nullptr && design != nullptr, "batch and design must not be NULL");
        require(!batch->finalized, "the batch is finalized: add every job before lar_batch_finalize");
        const LogDesignDevice<double> d = log_design_view(design);
        require(d.p == 7 && d.m == 0, "the DTI maps need the 7-column DTI design without constraints");
        require(v >= 0 && max_iter >= 0, "v and max_iter must be at least 0");
        require(v == 0 || (signals && floor && maps && npd), "signals, floor, maps and npd must not be NULL");
        batch->dti_fit.check(weighted, max_iter, tol, "DTI");
        batch->dti.push_back(DtiBatchJob{d, signals, floor, v, maps, npd});
    });
}

int lar_batch_add_dki(lar_batch batch, lar_log_design design, const float* signals, const double* s0,
                      const double* floor, const uint8_t* is_b0, int64_t v, int weighted, int64_t max_iter, double tol,
                      float* maps, uint8_t* npd, uint8_t* broke, double* params) {
    return guarded([&] {
        require(batch != nullptr && design != nullptr, "batch and design must not be NULL");
        require(!batch->finalized, "the batch is finalized: add every job before lar_batch_finalize");
        const LogDesignDevice<double> d = log_design_view(design);
        require(d.p == 22, "the DKI maps need the 22-column DKI design");
        require(v >= 0 && max_iter >= 0, "v and max_iter must be at least 0");
        require(v == 0 || (signals && floor && is_b0 && maps && npd && broke && params),
                "signals, floor, is_b0, maps, npd, broke and params must not be NULL");
        batch->dki_fit.check(weighted, max_iter, tol, "DKI");
        batch->dki.push_back(DkiBatchJob{d, signals, s0, floor, is_b0, v, maps, npd, broke, params});
    });
}

int lar_batch_add_mfod(lar_batch batch, const double* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                       lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver, int64_t max_outer,
                       double fraction_tol, double final_tol_x, double* fods, double* fractions, int32_t* rounds,
                       uint8_t* status) {
    return guarded([&] {
        require(batch != nullptr, "batch must not be NULL");
        require(!batch->finalized, "the batch is finalized: add every job before lar_batch_finalize");
        if (!batch->mfod) batch->mfod.reset(mfod_batch_create());
        mfod_batch_add(batch->mfod.get(), signals, v, weights, lr, lr_solver, hr, hr_solver, max_outer, fraction_tol,
                       final_tol_x, fods, fractions, rounds, status);
    });
}

int lar_batch_finalize(lar_batch batch) {
    return guarded([&] {
        require(batch != nullptr, "batch must not be NULL");
        require(!batch->finalized, "the batch is already finalized");
        lar_batch_s& b = *batch;
        // DTI: tickets of kDtiBatchBlock voxels.
        std::vector<int64_t> voxels;
        for (const auto& j : b.dti) {
            voxels.push_back(j.v);
            b.dti_nmax = std::max(b.dti_nmax, j.d.n);
        }
        if (!b.dti.empty()) {
            require(batch_dti_smem(b.dti_nmax) <= 227 * 1024,
                    "a DTI table of the batch has too many measurements for the shared-memory fit");
            const auto first = ticket_starts(voxels, kDtiBatchBlock);
            b.dti_tickets = first.back();
            upload_vector(b.d_dti, b.dti);
            upload_vector(b.dti_first, first);
        }
        // DKI: tickets of kDkiVoxelsPerWarp voxels per warp of the fit's CTA, kMapsBatchVoxels for the maps; one violator
        // list for the family (every voxel may break a constraint) and the re-fit's warp slots.
        voxels.clear();
        int64_t dki_voxels = 0;
        for (const auto& j : b.dki) {
            voxels.push_back(j.v);
            dki_voxels += j.v;
            b.dki_nmax = std::max(b.dki_nmax, j.d.n);
            b.dki_mmax = std::max(b.dki_mmax, j.d.m);
        }
        size_t viol_bytes = 0, slot_bytes = 0;
        if (!b.dki.empty()) {
            b.dki_warps = batch_log_warp_warps(b.dki_nmax, 22);
            require(b.dki_warps > 0, "a DKI table of the batch is too large for the shared-memory log fit");
            require(dki_voxels < (int64_t(1) << 31), "at most 2^31 - 1 DKI voxels per batch");
            const auto fit_first = ticket_starts(voxels, int64_t(kDkiVoxelsPerWarp) * b.dki_warps);
            const auto maps_first = ticket_starts(voxels, kMapsBatchVoxels);
            b.dki_fit_tickets = fit_first.back();
            b.dki_maps_tickets = maps_first.back();
            upload_vector(b.d_dki, b.dki);
            upload_vector(b.dki_fit_first, fit_first);
            upload_vector(b.dki_maps_first, maps_first);
            b.violators.capacity = int(dki_voxels);
            // Rounded up to 256 bytes: the re-fit's slots (doubles) follow.
            viol_bytes = (size_t(dki_voxels) * (sizeof(int) + sizeof(int64_t) + 22 * sizeof(double)) + 255) / 256 * 256;
            if (b.dki_mmax > 0) {
                b.refit_slot_doubles = batch_refit_slot_doubles(b.dki_nmax, 22, b.dki_mmax);
                b.refit_nslots = int(std::max<int64_t>(4, std::min<int64_t>((dki_voxels + 3) / 4 * 4,
                                                                            batch_refit_slots())));
                slot_bytes = size_t(b.refit_nslots) * b.refit_slot_doubles * sizeof(double);
            }
        }
        const size_t counter_bytes = 256;
        void* base = nullptr;
        cuda_check(cudaMalloc(&base, counter_bytes + viol_bytes + slot_bytes), "cudaMalloc (batch scratch)");
        b.scratch.reset(base);
        char* p = static_cast<char*>(base);
        b.counters = reinterpret_cast<int*>(p);
        cuda_check(cudaMemset(b.counters, 0, counter_bytes), "cudaMemset");
        p += counter_bytes;
        if (!b.dki.empty()) {
            const size_t cap = size_t(b.violators.capacity);
            b.violators.count = b.counters + 4;
            b.violators.params = reinterpret_cast<double*>(p);
            b.violators.voxel = reinterpret_cast<int64_t*>(p + cap * 22 * sizeof(double));
            b.violators.job = reinterpret_cast<int*>(p + cap * (22 * sizeof(double) + sizeof(int64_t)));
            p += viol_bytes;
            b.refit_slots = slot_bytes ? reinterpret_cast<double*>(p) : nullptr;
        }
        if (b.mfod) mfod_batch_finalize(b.mfod.get());
        b.finalized = true;
    });
}

int lar_batch_run(lar_batch batch, int families, void* stream) {
    return guarded([&] {
        require(batch != nullptr, "batch must not be NULL");
        require(batch->finalized, "lar_batch_finalize the batch before running it");
        require((families & ~(LAR_BATCH_DTI | LAR_BATCH_DKI | LAR_BATCH_MFOD)) == 0, "unknown family bits");
        lar_batch_s& b = *batch;
        auto st = static_cast<cudaStream_t>(stream);
        if ((families & LAR_BATCH_DTI) && !b.dti.empty())
            launch_batch_dti(b.d_dti.ptr, b.dti_first.ptr, int(b.dti.size()), b.dti_nmax, b.dti_tickets,
                             b.dti_fit.weighted, b.dti_fit.max_rw, b.dti_fit.tol, b.counters, st);
        if ((families & LAR_BATCH_DKI) && !b.dki.empty()) {
            cuda_check(cudaMemsetAsync(b.violators.count, 0, sizeof(int), st), "cudaMemsetAsync");
            launch_batch_log_warp(b.d_dki.ptr, b.dki_fit_first.ptr, int(b.dki.size()), b.dki_nmax, 22, b.dki_warps,
                                  b.dki_fit_tickets, b.dki_fit.weighted, b.dki_fit.max_rw, b.dki_fit.tol,
                                  b.counters + 2, b.violators, st);
            if (b.dki_mmax > 0)
                launch_batch_refit(b.d_dki.ptr, b.violators, b.dki_fit.weighted, b.counters + 5, b.refit_slots,
                                   b.refit_nslots, b.refit_slot_doubles, st);
            launch_batch_dki_maps(b.d_dki.ptr, b.dki_maps_first.ptr, int(b.dki.size()), b.dki_maps_tickets, st);
        }
        if ((families & LAR_BATCH_MFOD) && b.mfod) mfod_batch_run(b.mfod.get(), st);
    });
}

}  // extern "C"
