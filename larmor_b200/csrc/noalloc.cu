// lar_fit_log_signal_noalloc: the log-signal fit (with the constrained re-fit) for callers that
// cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: an application whose device memory is owned by its own
// allocator or budget (a server that reserves all memory up front), code running where an
// allocation would synchronise the device or is not allowed, or a plugin host that hands
// out only its own buffers. lar_fit_log_signal needs a design handle, whose creation allocates
// device memory, and it grows a scratch buffer on first use. This entry point allocates
// nothing on the device: the prepared design, the list of constraint violators and the
// constrained re-fit's per-warp workspace all live in one file-scope static device array of
// kNoAllocScratchBytes (32 MiB). Every GPU that loads the library holds that array until the
// process exits.
//
// Set-up: the first call on a device looks up the array's device address there with
// cudaGetSymbolAddress (host code cannot use the symbol itself: in host code its name is only
// a stand-in for the device array); make that first call before any stream capture. Every call
// shares the array and overwrites what the previous call left in it; the counters that must
// start at zero are cleared on the stream at the start of each call. Two calls whose work
// overlaps on the GPU (on different streams, or from different host threads) race on the array:
// serialise them.

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "host_la.hpp"
#include "log_fit.cuh"
#include "log_fit_warp.cuh"

namespace lar {

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The device address of g_noalloc_scratch on the current device, looked up once per device.
unsigned char* noalloc_scratch_address() {
    static std::mutex mutex;
    static std::map<int, unsigned char*> by_device;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(mutex);
    auto it = by_device.find(dev);
    if (it != by_device.end()) return it->second;
    void* ptr = nullptr;
    cuda_check(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress (no-alloc scratch)");
    auto* base = static_cast<unsigned char*>(ptr);
    by_device.emplace(dev, base);
    return base;
}

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

}  // namespace lar

using namespace lar;

extern "C" int lar_fit_log_signal_noalloc(const double* x, int64_t n, int64_t p, const double* g, int64_t m,
                                          const double* log_s, int64_t v, int weighted, int64_t max_iter,
                                          double tol, double* params, uint8_t* broke, void* stream) {
    return guarded([&] {
        require(x != nullptr && n > 0 && p > 0, "x must be a non-empty (n, p) host array");
        require(n >= p, "x must be (n, p) with n >= p: got (" + std::to_string(n) + ", " + std::to_string(p) + ")");
        require(m >= 0 && (m == 0 || g != nullptr), "g must be an (m, p) host array with m >= 0");
        require(p <= (m > 0 ? 31 : 32), "the no-alloc fit takes at most 31 parameters with constraints, 32 without");
        require(v >= 0, "v must be at least 0");
        require(v < (int64_t(1) << 31), "at most 2^31 - 1 voxels per call");
        require(max_iter >= 0, "max_iter must be at least 0");
        if (v == 0) return;

        // Scratch layout: [count, queue] ints | design (x, pinv^T, g, scales) | violator ids |
        // violator parameters | warp slots of the constrained re-fit.
        const size_t design_doubles = size_t(2 * n * p + 2 * m * p + p);
        const size_t design_off = 256;
        const size_t ids_off = up256(design_off + design_doubles * sizeof(double));
        const size_t params_off = up256(ids_off + (m > 0 ? size_t(v) * sizeof(int64_t) : 0));
        const size_t slots_off = up256(params_off + (m > 0 ? size_t(v) * size_t(p) * sizeof(double) : 0));
        const size_t slot_bytes = constrained_slot_doubles(int(n), int(p), int(m)) * sizeof(double);
        int slots = 0;
        if (m > 0) {
            const size_t room = slots_off < kNoAllocScratchBytes ? kNoAllocScratchBytes - slots_off : 0;
            slots = int(std::min<size_t>(room / slot_bytes, 1 << 20)) / 4 * 4;
        }
        const size_t need = m > 0 ? slots_off + 4 * slot_bytes : params_off;
        if (need > kNoAllocScratchBytes || (m > 0 && slots < 4)) {
            const size_t fixed = (m > 0 ? 4 * slot_bytes : 0) + up256(design_doubles * sizeof(double)) + 1024;
            const size_t per_voxel = m > 0 ? sizeof(int64_t) + size_t(p) * sizeof(double) : 0;
            if (per_voxel == 0 || fixed >= kNoAllocScratchBytes)
                // No voxel count fits: the design (and the re-fit's smallest workspace) alone
                // outgrow the array.
                throw Error(LAR_ERR_INVALID,
                            "lar_fit_log_signal_noalloc: a design of (n, p, m) = (" + std::to_string(n) + ", " +
                                std::to_string(p) + ", " + std::to_string(m) + ") needs " + std::to_string(fixed) +
                                " bytes of scratch before any voxel, more than the " +
                                std::to_string(kNoAllocScratchBytes) +
                                "-byte (32 MiB) static array; the design itself is too large for this entry point");
            const long long max_v = (long long)((kNoAllocScratchBytes - fixed) / per_voxel);
            throw Error(LAR_ERR_INVALID,
                        "lar_fit_log_signal_noalloc: a design of (n, p, m) = (" + std::to_string(n) + ", " +
                            std::to_string(p) + ", " + std::to_string(m) + ") with " + std::to_string(v) +
                            " voxels needs " + std::to_string(need) + " bytes of scratch, more than the " +
                            std::to_string(kNoAllocScratchBytes) + "-byte (32 MiB) static array; fit at most " +
                            std::to_string(max_v) + " voxels per call");
        }

        require(log_s && params && broke, "log_s, params and broke must not be NULL");
        // As many warp slots as the re-fit keeps resident, as far as the array has room.
        if (m > 0) slots = std::max(4, std::min(slots, constrained_resident_warps(int(n), int(p))) / 4 * 4);
        unsigned char* base = noalloc_scratch_address();
        auto st = static_cast<cudaStream_t>(stream);

        // The prepared design, in FP64, copied into the static array.
        const host::LogDesignHost h = host::prepare_log_design(x, n, p, g, m);
        std::vector<double> packed(design_doubles);
        double* px_ = packed.data();
        double* ppinvt = px_ + n * p;
        double* pg = ppinvt + n * p;
        double* pgt = pg + m * p;
        double* pscales = pgt + m * p;
        std::memcpy(px_, h.x.data(), sizeof(double) * size_t(n * p));
        for (int64_t i = 0; i < n; ++i)
            for (int64_t a = 0; a < p; ++a) ppinvt[i * p + a] = h.pinv[size_t(a * n + i)];
        if (m > 0) std::memcpy(pg, h.g.data(), sizeof(double) * size_t(m * p));
        for (int64_t c = 0; c < m; ++c)
            for (int64_t a = 0; a < p; ++a) pgt[a * m + c] = h.g[size_t(c * p + a)];
        std::memcpy(pscales, h.scales.data(), sizeof(double) * size_t(p));
        cuda_check(cudaMemcpyAsync(base + design_off, packed.data(), packed.size() * sizeof(double),
                                   cudaMemcpyHostToDevice, st),
                   "cudaMemcpyAsync (no-alloc design)");
        // The host staging buffer must outlive the copy.
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");

        const double* dx = reinterpret_cast<const double*>(base + design_off);
        LogDesignDevice<double> d;
        d.n = int(n);
        d.p = int(p);
        d.m = int(m);
        d.x = dx;
        d.pinvt = dx + n * p;
        d.z = nullptr;
        d.g = dx + 2 * n * p;
        d.gt = m > 0 ? dx + 2 * n * p + m * p : nullptr;
        d.scales = dx + 2 * n * p + 2 * m * p;
        d.scales64 = d.scales;

        ViolatorList<double> list;
        if (m > 0) {
            cuda_check(cudaMemsetAsync(base, 0, 2 * sizeof(int), st), "cudaMemsetAsync (no-alloc counters)");
            list.count = reinterpret_cast<int*>(base);
            list.capacity = int(v);
            list.voxel = reinterpret_cast<int64_t*>(base + ids_off);
            list.params = reinterpret_cast<double*>(base + params_off);
        }
        const LogSource src{log_s, n};
        const int rw = int(std::min<int64_t>(max_iter, 1 << 20));
        launch_log_warp<double>(d, src, v, weighted, rw, tol, params, broke, nullptr, list, st);
        if (m > 0) {
            launch_constrained<LogSource>(d, src, weighted, list, int(v), reinterpret_cast<int*>(base) + 1,
                                          reinterpret_cast<double*>(base + slots_off), slots, params, st);
        }
    });
}
