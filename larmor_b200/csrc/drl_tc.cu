// Damped Richardson-Lucy with its product F K^T K on the 5th-generation tensor cores
// (tcgen05.mma, kind::tf32, accumulators in tensor memory): the precision mode LAR_TF32X3 of
// FodSolver.drl.
//
// The iteration is that of drl.cu (cpp/src/sd/drl.cpp:39-100): p = K^T K f, then
// f <- max(f (1 + u (K^T s - p) / (p + 1e-16)), 1e-6) with the damping u of f and nu, until a
// voxel's total change is at most 1e-4 of its largest signal. Here the product runs as three
// TF32 products with FP32 accumulation, P = G_hi F_hi + G_hi F_lo + G_lo F_hi, where each
// operand is split into its TF32 head (the low 13 mantissa bits cleared) and the FP32
// remainder: the split recovers the bits TF32 drops (the "3xTF32" scheme), so P carries FP32
// accuracy (~1e-6 relative) instead of TF32's ~5e-4. The state F and the update are FP32; K^T s
// is summed in FP64 and kept in FP32. The results match the FP64 path to ~1e-5 of a voxel's
// largest amplitude (the tests bound them at the FOD tolerance 1e-4).
//
// Mapping: one CTA of 4 warps per SM (it takes all 512 columns of tensor memory) fits 48 voxels
// at a time. The MMA computes P^T = G F^T: M = 128 directions per tile (ceil(c / 128) tiles),
// N = 48 voxels, K = 8 directions per instruction. F^T's two parts (48 x c, K-major, the
// canonical no-swizzle layout of 8 x 16-byte core matrices) stay in shared memory; G's two
// parts are read from a copy prepared once per solver in the same layout, chunk by chunk
// (8 directions of every tile and part, 24 KB), by bulk copies (cp.async.bulk, the TMA engine)
// into a 4-stage ring. Thread 0 issues the copies and the MMAs, completion is tracked with
// mbarriers (the copies' transaction bytes, tcgen05.commit for the MMAs). P and K^T s live in
// tensor memory (lane = direction, column = voxel); after each product every warp reads its
// 32-lane quadrant (tcgen05.ld), applies the update, writes F's parts back to shared memory
// and sums each voxel's change in a fixed order.
//
// Every wait on an mbarrier is bounded (about a second); past the bound the kernel records an
// error in *err, stops issuing work, frees its tensor memory and returns.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <math_constants.h>

#include "common.cuh"
#include "drl.cuh"

namespace lar {
namespace {

constexpr int kTcThreads = 256;   // 8 warps: warp w reads tensor-memory lanes 32 (w % 4).., voxels 24 (w / 4)..
constexpr int kTcHalf = 24;       // voxels of a tile each of a quadrant's two warps updates
constexpr int kTcN = 48;          // voxels per tile (the MMA's N)
constexpr int kTcM = 128;         // directions per MMA tile (the MMA's M)
constexpr int kTcK = 8;           // directions per MMA step (K of kind::tf32)
constexpr int kTcStages = 4;
constexpr int kTcMaxTiles = 3;    // up to 384 padded directions
constexpr int kTcTmemCols = 512;
constexpr int kTcKsCol = 256;     // K^T s at tensor-memory columns [256, 256 + tiles * N)
constexpr long long kTcWaitCycles = 2000000000LL;  // about a second at 1.9 GHz

// Bytes of one prepared chunk of G: every tile's two parts, 128 rows x 8 directions each.
constexpr int kTcBlockBytes = kTcM * kTcK * 4;

__host__ __device__ inline int tc_kpad(int c) { return (c + kTcK - 1) / kTcK * kTcK; }
__host__ __device__ inline int tc_tiles(int c) { return (c + kTcM - 1) / kTcM; }
__host__ __device__ inline size_t tc_chunk_bytes(int c) { return size_t(tc_tiles(c)) * 2 * kTcBlockBytes; }
// Bytes of one part of F^T in shared memory.
// F^T's direction groups of 4 are 36 floats (144 bytes, the MMA's leading byte offset) apart
// instead of 32: the epilogue's 32 lanes (32 consecutive directions of one voxel) then hit 32
// different banks.
constexpr int kTcFGroupFloats = 36;
__host__ __device__ inline size_t tc_f_bytes(int c) { return size_t(kTcN / 8) * (tc_kpad(c) / 4) * kTcFGroupFloats * 4; }

// Offset (floats) of entry (row r, direction k) in a K-major layout of 8 x 4 core matrices
// (8 rows x 16 bytes, 32 floats each): 8-row groups `group` floats apart, direction groups of 4
// `kstride` floats apart.
__host__ __device__ inline size_t kmajor_offset(int r, int k, size_t group, int kstride = 32) {
    return size_t(r >> 3) * group + size_t(k >> 2) * kstride + size_t(r & 7) * 4 + size_t(k & 3);
}

struct TcShared {
    unsigned long long full[kTcStages];   // a stage's bulk copy has landed
    unsigned long long empty[kTcStages];  // the MMAs that read a stage have finished
    unsigned long long done;              // every MMA of an iteration has finished
    unsigned tmem_base;
    int n_active;
    int abort;
    float strength[kTcN], threshold[kTcN];
    int active[kTcN];
    long long vox[kTcN];
    float part[4][kTcN];  // each lane quadrant's share of a voxel's change
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of the given parity; false when the wait outlasts the bound.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    const long long start = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - start > kTcWaitCycles) return false;
    return true;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Chunk `chunk_index` of G into a stage: one bulk copy per 4 KB block (tile and part), so that
// the copy engines fetch the blocks in parallel; the mbarrier expects the whole chunk.
__device__ __forceinline__ void load_chunk(unsigned char* stage, const float* gtc, int chunk_index, int tiles,
                                           unsigned long long* bar) {
    const unsigned bytes = unsigned(tiles) * 2 * kTcBlockBytes;
    mbar_expect_tx(bar, bytes);
    const unsigned char* src = reinterpret_cast<const unsigned char*>(gtc) + size_t(chunk_index) * bytes;
    for (int b = 0; b < 2 * tiles; ++b)
        bulk_load(stage + size_t(b) * kTcBlockBytes, src + size_t(b) * kTcBlockBytes, kTcBlockBytes, bar);
}

// The shared-memory matrix descriptor of a K-major operand without swizzling: 8-row groups
// `sbo` bytes apart, the two 16-byte direction chunks of an MMA step `lbo` bytes apart.
__device__ __forceinline__ unsigned long long umma_desc(const void* p, unsigned sbo, unsigned lbo = 128) {
    const unsigned long long addr = smem_u32(p);
    return ((addr >> 4) & 0x3FFFull) | ((unsigned long long)((lbo >> 4) & 0x3FFF) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// kind::tf32, FP32 accumulators, both operands K-major, M = 128, N = kTcN.
constexpr unsigned kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | (unsigned(kTcN >> 3) << 17) |
                              (unsigned(kTcM >> 4) << 24);

__device__ __forceinline__ void umma_tf32(unsigned d_tmem, unsigned long long a, unsigned long long b,
                                          unsigned accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kTcIdesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(unsigned taddr, float (&v)[8]) {
    unsigned r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_st8(unsigned taddr, const float (&v)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
                 "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
                 "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// The TF32 head of x (its low 13 mantissa bits cleared) and the FP32 remainder.
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
    hi = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
    lo = x - hi;
}

__device__ __forceinline__ float pow8f(float x) {
    const float x2 = x * x, x4 = x2 * x2;
    return x4 * x4;
}

// Entry i of the signal dRL deconvolves for `voxel` (as drl.cu's signal_at).
__device__ __forceinline__ double tc_signal(const DrlSignal& S, int64_t voxel, int i) {
    const double si = S.s[voxel * S.m + i];
    if (S.w == nullptr) return si;
    const double ws = __dmul_rn(si, S.w[i]);
    double r = 0.0;
    for (int t = 0; t < S.ci; ++t) r = fma(S.wiso[size_t(i) * S.ci + t], S.fiso[voxel * S.ci + t], r);
    return fmax(ws - r, 0.0);
}

__global__ void __launch_bounds__(kTcThreads, 1)
    drl_tc_kernel(DrlDev P, const float* __restrict__ gtc, DrlSignal S, const int* __restrict__ list, int64_t count,
                  const int* __restrict__ count_dev, double* __restrict__ x, int64_t ldx, int* err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ TcShared sh;
    if (count_dev) count = min(count, int64_t(*count_dev));
    const int c = P.c, m = P.m, kpad = tc_kpad(c), tiles = tc_tiles(c), nq = kpad / kTcK;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const size_t fbytes = tc_f_bytes(c);
    float* FH = reinterpret_cast<float*>(smem);
    float* FL = reinterpret_cast<float*>(smem + fbytes);
    unsigned char* stage_base = smem + 2 * fbytes;
    const size_t chunk = tc_chunk_bytes(c);
    const size_t fgroup = size_t(kpad / 4) * kTcFGroupFloats;  // floats between 8-voxel groups of F^T
    constexpr unsigned kFLbo = kTcFGroupFloats * 4;          // bytes between its direction groups
    const float nu = float(P.nu);

    if (tid == 0) {
        for (int s = 0; s < kTcStages; ++s) {
            mbar_init(&sh.full[s], 1);
            mbar_init(&sh.empty[s], 1);
        }
        mbar_init(&sh.done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        sh.abort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh.tmem_base)),
                     "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = sh.tmem_base;
    const int quad = warp & 3, half = warp >> 2;
    const unsigned lane_base = unsigned(32 * quad) << 16;
    // G streams through the stage ring continuously, across iterations and tiles (it does not
    // change): chunk R of the stream is data chunk R % nq in stage R % kTcStages, the (R /
    // kTcStages)-th use of that stage, so its barriers' phase parity is (R / kTcStages) & 1.
    // Thread 0 issues the MMAs and counts the chunks consumed (`used`); thread 32 (the producer)
    // issues the copies and counts the chunks loaded (`loaded`), kTcStages ahead; everyone
    // tracks `done`.
    constexpr int kProducer = 32;
    long long used = 0, loaded = 0;
    unsigned done_phase = 0;
    if (tid == kProducer) {
        for (; loaded < kTcStages; ++loaded)
            load_chunk(stage_base + size_t(loaded) * chunk, gtc, int(loaded % nq), tiles, &sh.full[loaded]);
    }

    for (int64_t p0 = int64_t(blockIdx.x) * kTcN; p0 < count && !sh.abort; p0 += int64_t(gridDim.x) * kTcN) {
        if (tid < kTcN) sh.vox[tid] = p0 + tid < count ? (list ? int64_t(list[p0 + tid]) : p0 + tid) : -1;
        __syncthreads();
        // Each voxel's damping strength and stopping threshold (drl.cu), a warp per voxel.
        for (int j = warp; j < kTcN; j += kTcThreads / 32) {
            const int64_t voxel = sh.vox[j];
            if (voxel < 0) {
                if (lane == 0) {
                    sh.active[j] = 0;
                    sh.strength[j] = sh.threshold[j] = 0.f;
                }
                continue;
            }
            double sum = 0.0, mx = -CUDART_INF;
            bool any = false;
            for (int i = lane; i < m; i += 32) {
                const double si = tc_signal(S, voxel, i);
                sum += si;
                if (!isnan(si)) {
                    mx = any ? fmax(mx, si) : si;
                    any = true;
                }
            }
            const double mean = warp_sum(sum) / m;
            double ss = 0.0;
            for (int i = lane; i < m; i += 32) {
                const double si = tc_signal(S, voxel, i);
                ss += (si - mean) * (si - mean);
            }
            ss = warp_sum(ss);
            const bool all_nan = !__any_sync(0xffffffffu, any);
            mx = warp_max(any ? mx : -CUDART_INF);
            if (lane == 0) {
                sh.strength[j] = float(fmax(1.0 - 4.0 * sqrt(ss / double(m - 1)), 0.0));
                sh.threshold[j] = float(1e-4 * (all_nan ? CUDART_NAN : mx));
                sh.active[j] = 1;
            }
        }
        // K^T s of the tile into tensor memory (FP64 sums, kept in FP32), 16 voxels at a time:
        // their signals (FP64) staged in the F area, then a thread per direction lane of each
        // tile reads its row of K^T once for the 16.
        double* sig = reinterpret_cast<double*>(smem);
        for (int j0 = 0; j0 < kTcN; j0 += 16) {
            for (int e = tid; e < 16 * m; e += kTcThreads) {
                const int jj = e / m, i = e - jj * m;
                const int64_t voxel = sh.vox[j0 + jj];
                sig[e] = voxel >= 0 ? tc_signal(S, voxel, i) : 0.0;
            }
            __syncthreads();
            for (int t = 0; t < tiles; ++t) {
                const int d = kTcM * t + 32 * quad + lane;
                double acc[8];
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) acc[jj] = 0.0;
                if (d < c) {
                    const double* kt = P.k_t + size_t(d) * m;
                    const double* sh8 = sig + size_t(8 * half) * m;
                    for (int i = 0; i < m; ++i) {
                        const double k = kt[i];
#pragma unroll
                        for (int jj = 0; jj < 8; ++jj) acc[jj] = fma(k, sh8[jj * m + i], acc[jj]);
                    }
                }
                float ks[8];
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) ks[jj] = float(acc[jj]);
                tmem_st8(tmem + lane_base + unsigned(kTcKsCol + t * kTcN + j0 + 8 * half), ks);
            }
            tmem_wait_st();
            __syncthreads();
        }
        {
            float hi, lo;
            split_tf32(float(P.init), hi, lo);
            for (int e = tid; e < kTcN * kpad; e += kTcThreads) {
                const int j = e / kpad, k = e - j * kpad;
                const bool real = sh.vox[j] >= 0 && k < c;
                const size_t off = kmajor_offset(j, k, fgroup, kTcFGroupFloats);
                FH[off] = real ? hi : 0.f;
                FL[off] = real ? lo : 0.f;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();

        for (int it = 0; it < P.n_iter; ++it) {
            if (tid == 0) {
                int a = 0;
                for (int j = 0; j < kTcN; ++j) a += sh.active[j];
                sh.n_active = a;
            }
            __syncthreads();
            if (sh.n_active == 0 || sh.abort) break;
            // The product: thread 0 issues the MMAs of the iteration's nq chunks as they land,
            // while the producer refills each stage with chunk R + kTcStages of the stream as
            // soon as the MMAs of chunk R are done with it.
            if (tid == kProducer) {
                bool ok = true;
                for (int i = 0; i < nq && ok; ++i) {
                    const long long R = loaded, Rw = R - kTcStages;
                    const int s = int(R % kTcStages);
                    ok = mbar_wait(&sh.empty[s], unsigned(Rw / kTcStages) & 1u);
                    if (!ok) break;
                    load_chunk(stage_base + size_t(s) * chunk, gtc, int(R % nq), tiles, &sh.full[s]);
                    ++loaded;
                }
                if (!ok) {
                    sh.abort = 1;
                    atomicExch(err, 1);
                }
            }
            if (tid == 0) {
                tc_fence_after();
                bool ok = true;
                for (int q = 0; q < nq && ok; ++q) {
                    const long long R = used;
                    const int s = int(R % kTcStages);
                    ok = mbar_wait(&sh.full[s], unsigned(R / kTcStages) & 1u);
                    if (!ok) break;
                    tc_fence_after();
                    const unsigned char* st = stage_base + size_t(s) * chunk;
                    const unsigned long long bh = umma_desc(
                        reinterpret_cast<const unsigned char*>(FH) + size_t(q) * 2 * kFLbo, unsigned(fgroup * 4), kFLbo);
                    const unsigned long long bl = umma_desc(
                        reinterpret_cast<const unsigned char*>(FL) + size_t(q) * 2 * kFLbo, unsigned(fgroup * 4), kFLbo);
                    for (int t = 0; t < tiles; ++t) {
                        const unsigned long long ah = umma_desc(st + size_t(2 * t) * kTcBlockBytes, 256);
                        const unsigned long long al = umma_desc(st + size_t(2 * t + 1) * kTcBlockBytes, 256);
                        const unsigned d_tmem = tmem + unsigned(t * kTcN);
                        umma_tf32(d_tmem, ah, bh, q > 0 ? 1u : 0u);
                        umma_tf32(d_tmem, ah, bl, 1u);
                        umma_tf32(d_tmem, al, bh, 1u);
                    }
                    umma_commit(&sh.empty[s]);
                    ++used;
                }
                umma_commit(&sh.done);
                if (!ok) {
                    sh.abort = 1;
                    atomicExch(err, 1);
                }
            }
            __syncthreads();
            if (sh.abort) break;
            // Everyone waits for the product.
            if (!mbar_wait(&sh.done, done_phase & 1u)) {
                atomicExch(err, 1);
                sh.abort = 1;
            }
            done_phase ^= 1u;
            tc_fence_after();
            __syncthreads();
            if (sh.abort) break;
            // The damped update of the still-active voxels: a thread holds one direction lane of
            // each tile and the 24 voxels of its warp's half.
            float change[kTcHalf];
#pragma unroll
            for (int j = 0; j < kTcHalf; ++j) change[j] = 0.f;
            for (int t = 0; t < tiles; ++t) {
                const int d = kTcM * t + 32 * quad + lane;
#pragma unroll
                for (int g = 0; g < kTcHalf; g += 8) {
                    const int j0 = kTcHalf * half + g;
                    float pv[8], kv[8];
                    tmem_ld8(tmem + lane_base + unsigned(t * kTcN + j0), pv);
                    tmem_ld8(tmem + lane_base + unsigned(kTcKsCol + t * kTcN + j0), kv);
                    tmem_wait_ld();
                    if (d >= c) continue;
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj) {
                        const int j = j0 + jj;
                        if (!sh.active[j]) continue;
                        const size_t off = kmajor_offset(j, d, fgroup, kTcFGroupFloats);
                        const float f = FH[off] + FL[off];
                        // f^8 / (f^8 + nu^8) as 1 / (1 + (nu / f)^8): no underflow of f^8.
                        // Fast divisions (about 2 ulp): the product carries ~1e-6 already.
                        const float q8 = pow8f(__fdividef(nu, f));
                        const float damping = 1.f - sh.strength[j] * (1.f - __fdividef(1.f, 1.f + q8));
                        const float ratio = __fdividef(kv[jj] - pv[jj], pv[jj] + 1e-16f);
                        const float updated = fmaxf(f * (1.f + damping * ratio), 1e-6f);
                        float hi, lo;
                        split_tf32(updated, hi, lo);
                        FH[off] = hi;
                        FL[off] = lo;
                        change[g + jj] += fabsf(updated - f);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < kTcHalf; ++j) {
                const float v = warp_sum(change[j]);
                if (lane == 0) sh.part[quad][kTcHalf * half + j] = v;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_fence_before();
            __syncthreads();
            if (tid < kTcN && sh.active[tid]) {
                const float total = sh.part[0][tid] + sh.part[1][tid] + sh.part[2][tid] + sh.part[3][tid];
                if (total <= sh.threshold[tid]) sh.active[tid] = 0;
            }
            __syncthreads();
        }
        if (sh.abort) break;
        for (int e = tid; e < kTcN * c; e += kTcThreads) {
            const int j = e / c, k = e - j * c;
            const int64_t voxel = sh.vox[j];
            if (voxel >= 0) {
                const size_t off = kmajor_offset(j, k, fgroup, kTcFGroupFloats);
                x[voxel * ldx + k] = double(FH[off] + FL[off]);
            }
        }
        __syncthreads();
    }
    // The stream's copies still in flight (the kTcStages loaded past the last chunk consumed)
    // land before the CTA exits (bounded waits).
    if (tid == kProducer)
        for (long long R = loaded - kTcStages; R < loaded; ++R)
            if (!mbar_wait(&sh.full[R % kTcStages], unsigned(R / kTcStages) & 1u)) {
                atomicExch(err, 1);
                break;
            }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols));
}

}  // namespace

bool drl_tc_fits(int c) { return c > 64 && c <= kTcMaxTiles * kTcM && c <= 320; }

// 16 voxels' FP64 signals are staged in the F area of the kernel's shared memory for K^T s.
bool drl_tc_fits_measurements(int c, int m) { return size_t(16) * m * 8 <= 2 * tc_f_bytes(c); }

size_t drl_tc_smem_bytes(int c) { return 2 * tc_f_bytes(c) + size_t(kTcStages) * tc_chunk_bytes(c); }

// G = K^T K in the layout the kernel's bulk copies read: chunk q (directions 8q..8q+7) holds,
// for every tile t of 128 directions, the TF32 head then the remainder of rows 128t..128t+127,
// each a K-major block of 8 x 4 core matrices; rows and directions past c are zero.
std::vector<float> drl_tc_layout(const double* gram, int c) {
    const int kpad = tc_kpad(c), tiles = tc_tiles(c), nq = kpad / kTcK;
    const size_t block = size_t(kTcM) * kTcK;
    std::vector<float> out(size_t(nq) * tiles * 2 * block, 0.f);
    for (int q = 0; q < nq; ++q)
        for (int t = 0; t < tiles; ++t)
            for (int r = 0; r < kTcM; ++r)
                for (int kk = 0; kk < kTcK; ++kk) {
                    const int row = kTcM * t + r, k = kTcK * q + kk;
                    const float v = (row < c && k < c) ? float(gram[size_t(row) * c + k]) : 0.f;
                    uint32_t bits;
                    std::memcpy(&bits, &v, 4);
                    bits &= 0xFFFFE000u;
                    float hi;
                    std::memcpy(&hi, &bits, 4);
                    const float lo = v - hi;
                    const size_t base = (size_t(q) * tiles + t) * 2 * block;
                    const size_t off = kmajor_offset(r, kk, 64);
                    out[base + off] = hi;
                    out[base + block + off] = lo;
                }
    return out;
}

void launch_drl_tc(const DrlDev& P, const float* gtc, const DrlSignal& S, const int* list, int64_t count,
                   const int* count_dev, double* x, int64_t ldx, int* err, cudaStream_t st) {
    if (count == 0) return;
    require(drl_tc_fits(P.c), "the tensor-core dRL takes 65 to 320 directions");
    const size_t smem = drl_tc_smem_bytes(P.c);
    require(smem <= 227 * 1024, "the tensor-core dRL's shared memory outgrows an SM");
    cuda_check(cudaFuncSetAttribute(drl_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "cudaFuncSetAttribute");
    const int64_t tiles = (count + kTcN - 1) / kTcN;
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>(tiles, sm_count()));
    LaunchScope scope("drl_tc_kernel", st);
    drl_tc_kernel<<<unsigned(blocks), kTcThreads, smem, st>>>(P, gtc, S, list, count, count_dev, x, ldx, err);
    cuda_check(cudaGetLastError(), "drl_tc_kernel launch");
}

}  // namespace lar
