// Library-wide C-ABI entry points: error reporting, version, launch accounting.
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"

namespace lar {

namespace {
thread_local std::string last_error;

std::atomic<int64_t> launches{0};
std::atomic<bool> timing{false};
std::mutex timing_mutex;
// Kernel name -> (start, end) event pairs of its timed launches.
std::map<std::string, std::vector<std::pair<cudaEvent_t, cudaEvent_t>>> timed;

void clear_timed() {
    for (auto& entry : timed)
        for (auto& ev : entry.second) {
            cudaEventDestroy(ev.first);
            cudaEventDestroy(ev.second);
        }
    timed.clear();
}
}  // namespace

void set_error(const std::string& message) { last_error = message; }

namespace {
std::mutex settings_mutex;
std::map<std::string, int64_t> settings;
// name -> largest accepted value
const std::map<std::string, int64_t> kSettings = {
    {"dti.voxels_per_cta", 64},     // voxels per CTA of the shared-memory DTI fit: 16, 32 or 64
    {"log.warp.waves", 64},         // waves of resident CTAs in the warp-per-voxel log fit's grid
    {"dki.refit.ctas_per_sm", 32},  // CTAs per SM of the constrained re-fit
    {"lsi.ctas_per_sm", 32},        // CTAs per SM of the LSI
    {"sd.nnls.ctas_per_sm", 32},    // CTAs per SM of the ridge NNLS
    {"sd.fractions.ctas_per_sm", 32},  // CTAs per SM of the fraction kernels
    {"peaks.ctas_per_sm", 32},      // CTAs per SM of the peak search
    {"csd.ctas_per_sm", 32},        // CTAs per SM of the CSD fit
    {"drl.ctas_per_sm", 32},        // CTAs per SM of damped Richardson-Lucy
};
}  // namespace

int64_t launch_setting(const char* name) {
    std::lock_guard<std::mutex> lock(settings_mutex);
    auto it = settings.find(name);
    return it == settings.end() ? 0 : it->second;
}

LaunchScope::LaunchScope(const char* n, cudaStream_t s) : name(n), stream(s) {
    launches.fetch_add(1, std::memory_order_relaxed);
    if (timing.load(std::memory_order_relaxed) && cudaEventCreate(&start) == cudaSuccess) {
        if (cudaEventRecord(start, stream) != cudaSuccess) {
            cudaEventDestroy(start);
            start = nullptr;
        }
    }
}

LaunchScope::~LaunchScope() {
    if (start == nullptr) return;
    cudaEvent_t end = nullptr;
    if (cudaEventCreate(&end) != cudaSuccess || cudaEventRecord(end, stream) != cudaSuccess) {
        if (end) cudaEventDestroy(end);
        cudaEventDestroy(start);
        return;
    }
    std::lock_guard<std::mutex> lock(timing_mutex);
    timed[name].emplace_back(start, end);
}

}  // namespace lar

extern "C" {

const char* lar_last_error(void) { return lar::last_error.c_str(); }

const char* lar_version(void) { return "larmor_b200 0.1.0 (sm_100a)"; }

int64_t lar_launch_count(void) { return lar::launches.load(); }

int lar_set_launch_setting(const char* name, int64_t value) {
    return lar::guarded([&] {
        lar::require(name != nullptr, "name must not be NULL");
        auto it = lar::kSettings.find(name);
        lar::require(it != lar::kSettings.end(), std::string("unknown launch setting ") + name);
        lar::require(value >= 0 && value <= it->second,
                     std::string(name) + " takes 0 (the library's choice) to " + std::to_string(it->second));
        std::lock_guard<std::mutex> lock(lar::settings_mutex);
        if (value == 0) lar::settings.erase(name);
        else lar::settings[name] = value;
    });
}

int lar_get_launch_setting(const char* name, int64_t* value) {
    return lar::guarded([&] {
        lar::require(name != nullptr && value != nullptr, "name and value must not be NULL");
        lar::require(lar::kSettings.count(name) == 1, std::string("unknown launch setting ") + name);
        *value = lar::launch_setting(name);
    });
}

int lar_kernel_timing(int enable) {
    return lar::guarded([&] {
        std::lock_guard<std::mutex> lock(lar::timing_mutex);
        lar::clear_timed();
        lar::timing.store(enable != 0);
    });
}

int lar_kernel_time(const char* name, double* total_ms, int64_t* count) {
    return lar::guarded([&] {
        lar::require(name != nullptr && total_ms != nullptr && count != nullptr,
                     "name, total_ms and count must not be NULL");
        std::lock_guard<std::mutex> lock(lar::timing_mutex);
        double sum = 0.0;
        int64_t n = 0;
        auto it = lar::timed.find(name);
        if (it != lar::timed.end()) {
            for (auto& ev : it->second) {
                lar::cuda_check(cudaEventSynchronize(ev.second), "cudaEventSynchronize");
                float ms = 0.0f;
                lar::cuda_check(cudaEventElapsedTime(&ms, ev.first, ev.second), "cudaEventElapsedTime");
                sum += ms;
                ++n;
            }
        }
        *total_ms = sum;
        *count = n;
    });
}

}  // extern "C"
