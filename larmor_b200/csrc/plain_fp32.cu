// The plain single-precision multi-tissue fit: the comparison baseline of the FP64 path.
//
// It is the direct GPU port of the reference's per-voxel loop (cpp/src/sd/multi_tissue.cpp:76-148)
// that a first CUDA version would be: one warp per voxel runs every round of its voxel in one
// kernel, in FP32, with the textbook forms of each step:
//   - the anisotropic signal max(s w - W_iso f_iso, 0) and its correlations K^T s with the
//     lanes over the kernel's columns;
//   - Lawson-Hanson NNLS on the normal equations (cpp/src/sd/nnls.cpp:187-221 with the
//     Cholesky fits of :237-301), the Cholesky factor of the active Gram block formed anew
//     for every fit (no updates or downdates), in shared memory, up to 64 active columns;
//   - the fractions (cpp/src/sd/fractions.cpp:56-101): the median threshold, the lumped (or
//     per-block) columns scaled to a maximum of 1, and their NNLS on the normal equations.
// It keeps the reference's constants, tie rules and step limits, with a relative pivot of 1e-6
// (FP32) in place of 1e-12 and a limit of 3c outer steps (FP32 gradients can cycle at the
// FP64 tolerance). It has no QR fallback: a voxel whose active set outgrows the factor or
// whose pivot fails keeps its last iterate and gets status 1 (2 when a step limit stops it).
//
// The FP64 path (multi_tissue.cu) differs in everything this kernel leaves plain: round
// kernels over a shrinking voxel list, the inverse factor kept across the active-set changes
// with Givens downdates, two voxels per warp at low resolution, register fraction fits.

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "plain_fp32.cuh"

namespace lar {

namespace {

constexpr int kPlainWarps = 4;
constexpr unsigned kFull = 0xffffffffu;
constexpr float kPlainMinPivot = 1e-6f;
constexpr float kPlainMedianTie = 1e-9f;
constexpr float kPlainFractionOffset = 1e-16f;
constexpr float kEps32 = 1.1920929e-7f;
constexpr int NA = kPlainMaxActive;

struct Scratch {
    float *ws, *sig, *as, *gs, *corr, *x, *z, *g, *L, *y, *small;
    int* idx;
    int* meta;  // [0] the active count of the last solve
    unsigned char* act;
};

__host__ __device__ inline size_t plain_warp_bytes(int m, int c, int ng) {
    const size_t floats = size_t(3) * m + size_t(ng) * m + size_t(4) * c + size_t(NA) * NA + NA + 64;
    return (floats * 4 + (NA + 4) * 4 + size_t(c) + 15) / 16 * 16;
}

__device__ Scratch carve(unsigned char* base, int m, int c, int ng) {
    Scratch s;
    float* f = reinterpret_cast<float*>(base);
    s.ws = f;
    s.sig = s.ws + m;
    s.as = s.sig + m;
    s.gs = s.as + m;
    s.corr = s.gs + size_t(ng) * m;
    s.x = s.corr + c;
    s.z = s.x + c;
    s.g = s.z + c;
    s.L = s.g + c;
    s.y = s.L + NA * NA;
    s.small = s.y + NA;
    s.idx = reinterpret_cast<int*>(s.small + 64);
    s.meta = s.idx + NA;
    s.act = reinterpret_cast<unsigned char*>(s.meta + 4);
    return s;
}

__device__ __forceinline__ float wsum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ float wmax(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// The inactive column with the largest gradient, the first on a tie; -1 if none.
__device__ int steepest(const float* g, const unsigned char* act, int c, int lane, float& best) {
    float bv = -INFINITY;
    int bi = -1;
    for (int j = lane; j < c; j += 32)
        if (!act[j] && (bi < 0 || g[j] > bv)) {
            bv = g[j];
            bi = j;
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(kFull, bv, o);
        const int oi = __shfl_xor_sync(kFull, bi, o);
        if (oi >= 0 && (bi < 0 || ov > bv || (ov == bv && oi < bi))) {
            bv = ov;
            bi = oi;
        }
    }
    best = bv;
    return bi;
}

// A Gram matrix stored whole, (c, c) row-major.
struct DenseGram {
    const float* g;
    int c;
    __device__ __forceinline__ float operator()(int i, int j) const { return g[size_t(i) * c + j]; }
};

// z = the solution of G_AA z_A = corr_A on the active columns (0 elsewhere), by a Cholesky
// factor of G_AA formed anew; false when the active set exceeds NA or a pivot fails.
template <class Gram>
__device__ bool solve_active(const Gram& G, int c, const Scratch& s, int lane) {
    int na = 0;
    for (int base = 0; base < c; base += 32) {
        const int j = base + lane;
        const bool a = j < c && s.act[j];
        const unsigned mask = __ballot_sync(kFull, a);
        if (a) {
            const int pos = na + __popc(mask & ((1u << lane) - 1u));
            if (pos < NA) s.idx[pos] = j;
        }
        na += __popc(mask);
    }
    if (na > NA) return false;
    if (lane == 0) s.meta[0] = na;
    __syncwarp();
    for (int e = lane; e < na * na; e += 32) {
        const int r = e / na, q = e - r * na;
        if (q <= r) s.L[r * NA + q] = G(s.idx[r], s.idx[q]);
    }
    __syncwarp();
    // Left-looking Cholesky, one column at a time.
    for (int k = 0; k < na; ++k) {
        float part = 0.f;
        for (int j = lane; j < k; j += 32) part += s.L[k * NA + j] * s.L[k * NA + j];
        const float gkk = s.L[k * NA + k];
        const float pivot = gkk - wsum(part);
        if (!(pivot > kPlainMinPivot * gkk)) return false;
        const float d = sqrtf(pivot);
        for (int i = k + 1 + lane; i < na; i += 32) {
            float acc = s.L[i * NA + k];
            for (int j = 0; j < k; ++j) acc -= s.L[i * NA + j] * s.L[k * NA + j];
            s.L[i * NA + k] = acc / d;
        }
        __syncwarp();
        if (lane == 0) s.L[k * NA + k] = d;
        __syncwarp();
    }
    for (int k = 0; k < na; ++k) {  // L y = corr_A
        float part = 0.f;
        for (int j = lane; j < k; j += 32) part += s.L[k * NA + j] * s.y[j];
        const float sum = wsum(part);
        if (lane == 0) s.y[k] = (s.corr[s.idx[k]] - sum) / s.L[k * NA + k];
        __syncwarp();
    }
    for (int k = na - 1; k >= 0; --k) {  // L^T z_A = y
        float part = 0.f;
        for (int j = k + 1 + lane; j < na; j += 32) part += s.L[j * NA + k] * s.y[j];
        const float sum = wsum(part);
        if (lane == 0) s.y[k] = (s.y[k] - sum) / s.L[k * NA + k];
        __syncwarp();
    }
    for (int j = lane; j < c; j += 32) s.z[j] = 0.f;
    __syncwarp();
    for (int k = lane; k < na; k += 32) s.z[s.idx[k]] = s.y[k];
    __syncwarp();
    return true;
}

// Lawson-Hanson on (G, corr): x >= 0. 0: converged; 1: the factor failed; 2: a step limit.
template <class Gram>
__device__ int plain_nnls(const Gram& G, int c, float tol, const Scratch& s, int lane) {
    for (int j = lane; j < c; j += 32) {
        s.x[j] = 0.f;
        s.act[j] = 0;
        s.g[j] = s.corr[j];
    }
    __syncwarp();
    const int cap = 3 * c;
    int inner = 0, outer = 0;
    for (;;) {
        float best;
        const int e = steepest(s.g, s.act, c, lane, best);
        if (e < 0 || !(best > tol)) return 0;
        if (++outer > cap) return 2;
        if (lane == 0) s.act[e] = 1;
        __syncwarp();
        if (!solve_active(G, c, s, lane)) return 1;
        for (;;) {
            bool any = false;
            for (int j = lane; j < c; j += 32) any |= s.act[j] && s.z[j] <= 0.f;
            if (!__any_sync(kFull, any)) break;
            if (++inner > cap) {
                for (int j = lane; j < c; j += 32) s.x[j] = s.z[j];
                __syncwarp();
                return 2;
            }
            float bs = INFINITY;
            int bc = -1;
            for (int j = lane; j < c; j += 32)
                if (s.act[j] && s.z[j] <= 0.f) {
                    const float d = s.x[j] - s.z[j];
                    const float stp = d > 0.f ? s.x[j] / d : 0.f;
                    if (stp < bs) {
                        bs = stp;
                        bc = j;
                    }
                }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float ov = __shfl_xor_sync(kFull, bs, o);
                const int oc = __shfl_xor_sync(kFull, bc, o);
                if (oc >= 0 && (bc < 0 || ov < bs || (ov == bs && oc < bc))) {
                    bs = ov;
                    bc = oc;
                }
            }
            for (int j = lane; j < c; j += 32) s.x[j] += bs * (s.z[j] - s.x[j]);
            __syncwarp();
            if (lane == 0) {
                s.x[bc] = 0.f;
                s.act[bc] = 0;
            }
            __syncwarp();
            for (int j = lane; j < c; j += 32)
                if (s.act[j] && !(fabsf(s.x[j]) >= tol)) s.act[j] = 0;
            __syncwarp();
            if (!solve_active(G, c, s, lane)) return 1;
        }
        for (int j = lane; j < c; j += 32) s.x[j] = s.z[j];
        __syncwarp();
        // g = corr - G x over the active columns (G symmetric: row i read along j).
        const int na = s.meta[0];
        for (int j = lane; j < c; j += 32) {
            float acc = s.corr[j];
            for (int k = 0; k < na; ++k) {
                const int i = s.idx[k];
                acc -= G(i, j) * s.x[i];
            }
            s.g[j] = acc;
        }
        __syncwarp();
    }
}

// The median of v[0..n): the middle order statistic, or the mean of the two middle ones.
__device__ float plain_median(const float* v, int n, int lane) {
    const int k1 = (n - 1) / 2, k2 = n / 2;
    float a = -INFINITY, b = -INFINITY;
    for (int i = lane; i < n; i += 32) {
        const float vi = v[i];
        int less = 0, eq = 0;
        for (int j = 0; j < n; ++j) {
            less += v[j] < vi;
            eq += v[j] == vi;
        }
        if (less <= k1 && k1 < less + eq) a = vi;
        if (less <= k2 && k2 < less + eq) b = vi;
    }
    a = wmax(a);
    b = wmax(b);
    return n % 2 == 1 ? b : (a + b) / 2.f;
}

// NNLS of at most four columns on lane 0, on the normal equations N x = b.
__device__ void small_nnls(const float (&N)[kPlainMaxGroups][kPlainMaxGroups], const float (&b)[kPlainMaxGroups],
                           int n, float tol, float (&x)[kPlainMaxGroups]) {
    bool act[kPlainMaxGroups] = {};
    float z[kPlainMaxGroups], g[kPlainMaxGroups];
    for (int j = 0; j < n; ++j) {
        x[j] = 0.f;
        g[j] = b[j];
    }
    auto solve = [&](float (&out)[kPlainMaxGroups]) {
        float L[kPlainMaxGroups][kPlainMaxGroups] = {}, y[kPlainMaxGroups] = {};
        for (int a2 = 0; a2 < n; ++a2) {
            out[a2] = 0.f;
            if (!act[a2]) continue;
            for (int c2 = 0; c2 <= a2; ++c2) {
                if (!act[c2]) continue;
                float sum = N[a2][c2];
                for (int k = 0; k < c2; ++k)
                    if (act[k]) sum -= L[a2][k] * L[c2][k];
                if (c2 == a2)
                    L[a2][a2] = sqrtf(fmaxf(sum, 1e-30f));
                else
                    L[a2][c2] = sum / L[c2][c2];
            }
        }
        for (int a2 = 0; a2 < n; ++a2) {
            if (!act[a2]) continue;
            float sum = b[a2];
            for (int k = 0; k < a2; ++k)
                if (act[k]) sum -= L[a2][k] * y[k];
            y[a2] = sum / L[a2][a2];
        }
        for (int a2 = n - 1; a2 >= 0; --a2) {
            if (!act[a2]) continue;
            float sum = y[a2];
            for (int k = a2 + 1; k < n; ++k)
                if (act[k]) sum -= L[k][a2] * out[k];
            out[a2] = sum / L[a2][a2];
        }
    };
    int inner = 0, outer = 0;
    for (;;) {
        int e = -1;
        for (int j = 0; j < n; ++j)
            if (!act[j] && (e < 0 || g[j] > g[e])) e = j;
        if (e < 0 || !(g[e] > tol) || ++outer > 3 * n) return;
        act[e] = true;
        solve(z);
        for (;;) {
            bool any = false;
            for (int j = 0; j < n; ++j) any |= act[j] && z[j] <= 0.f;
            if (!any) break;
            if (++inner > 3 * n) {
                for (int j = 0; j < n; ++j) x[j] = z[j];
                return;
            }
            float bs = INFINITY;
            int bc = -1;
            for (int j = 0; j < n; ++j)
                if (act[j] && z[j] <= 0.f) {
                    const float d = x[j] - z[j];
                    const float stp = d > 0.f ? x[j] / d : 0.f;
                    if (stp < bs) {
                        bs = stp;
                        bc = j;
                    }
                }
            for (int j = 0; j < n; ++j) x[j] += bs * (z[j] - x[j]);
            x[bc] = 0.f;
            act[bc] = false;
            for (int j = 0; j < n; ++j)
                if (act[j] && !(fabsf(x[j]) >= tol)) act[j] = false;
            solve(z);
        }
        for (int j = 0; j < n; ++j) x[j] = z[j];
        for (int j = 0; j < n; ++j) {
            float acc = b[j];
            for (int k = 0; k < n; ++k) acc -= N[j][k] * x[k];
            g[j] = acc;
        }
    }
}

// The fractions of one voxel (cpp/src/sd/fractions.cpp:70-101) into s.small[8..8+n): the FOD
// thresholded at its median, one lumped column (or one per block) scaled to a maximum of 1,
// next to the isotropic columns, fitted to the signal by NNLS. tol < 0: the default
// 10 eps norm1 max(m, n).
__device__ int plain_fractions(const PlainStage& T, const float* fod, const Scratch& s, bool per_block, float tol,
                               int lane) {
    const int m = T.m, c = T.c, ci = T.ci;
    const float threshold = plain_median(fod, c, lane) * (1.f - kPlainMedianTie);
    const int ng = per_block ? T.nb : 1;
    const int n = ng + ci;
    for (int gi = 0; gi < ng; ++gi) {
        const int b0 = per_block ? T.blocks[2 * gi] : 0, b1 = per_block ? T.blocks[2 * gi + 1] : c;
        float* col = s.gs + size_t(gi) * m;
        float largest = -INFINITY;
        for (int i = lane; i < m; i += 32) {
            float acc = 0.f;
            for (int j = b0; j < b1; ++j) {
                const float f = fod[j];
                if (!(f < threshold)) acc += T.kt[size_t(j) * m + i] * f;
            }
            col[i] = acc;
            if (!isnan(acc)) largest = fmaxf(largest, acc);
        }
        largest = wmax(largest);
        __syncwarp();
        if (largest > 0.f)
            for (int i = lane; i < m; i += 32) col[i] /= largest;
        __syncwarp();
    }
    auto column = [&](int j, int i) { return j < ng ? s.gs[size_t(j) * m + i] : T.iso[size_t(i) * ci + (j - ng)]; };
    float N[kPlainMaxGroups][kPlainMaxGroups] = {}, b[kPlainMaxGroups] = {}, x[kPlainMaxGroups] = {};
    float norm1 = 0.f;
    for (int a = 0; a < n; ++a) {
        float pb = 0.f, pn = 0.f;
        for (int i = lane; i < m; i += 32) {
            const float ca = column(a, i);
            pb += ca * s.sig[i];
            pn += fabsf(ca);
        }
        b[a] = wsum(pb);
        norm1 = fmaxf(norm1, wsum(pn));
        for (int q = 0; q <= a; ++q) {
            float p = 0.f;
            for (int i = lane; i < m; i += 32) p += column(a, i) * column(q, i);
            N[a][q] = N[q][a] = wsum(p);
        }
    }
    if (tol < 0.f) tol = 10.f * kEps32 * norm1 * float(max(m, n));
    if (lane == 0) {
        small_nnls(N, b, n, tol, x);
        for (int j = 0; j < n; ++j) s.small[8 + j] = x[j];
    }
    __syncwarp();
    return n;
}

// s.as = max(s.ws - W_iso f_iso, 0) and s.corr = K^T s.as for one stage.
__device__ void stage_correlations(const PlainStage& T, const float* f_iso, const Scratch& s, int lane) {
    for (int i = lane; i < T.m; i += 32) {
        float r = 0.f;
        for (int t = 0; t < T.ci; ++t) r += T.wiso[size_t(i) * T.ci + t] * f_iso[t];
        s.as[i] = fmaxf(s.ws[i] - r, 0.f);
    }
    __syncwarp();
    for (int j = lane; j < T.c; j += 32) {
        float acc = 0.f;
        for (int i = 0; i < T.m; ++i) acc += T.k[size_t(i) * T.c + j] * s.as[i];
        s.corr[j] = acc;
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kPlainWarps * 32) plain_fp32_mfod_kernel(
    PlainStage lr, PlainStage hr, const float* __restrict__ signals, int64_t v, const float* __restrict__ weights,
    int max_rounds, float fraction_tol, float final_tol, float* __restrict__ fods, float* __restrict__ fractions,
    int32_t* __restrict__ rounds_out, uint8_t* __restrict__ status_out, int ng) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m = lr.m, cmax = max(lr.c, hr.c);
    const Scratch s = carve(smem + size_t(warp) * plain_warp_bytes(m, cmax, ng), m, cmax, ng);
    const int ci = lr.ci;
    float* f_iso = s.small;      // [0, 4)
    float* prev = s.small + 4;   // [4, 8)
    float* fr = s.small + 8;     // [8, 12): the last fractions
    const int64_t warps = int64_t(gridDim.x) * kPlainWarps;
    for (int64_t voxel = int64_t(blockIdx.x) * kPlainWarps + warp; voxel < v; voxel += warps) {
        const float* row = signals + voxel * m;
        for (int i = lane; i < m; i += 32) {
            const float si = row[i];
            s.sig[i] = si;
            s.ws[i] = si * weights[i];
        }
        if (lane < kPlainMaxGroups) {
            f_iso[lane] = 0.f;
            prev[lane] = INFINITY;
        }
        __syncwarp();
        int status = 0, rounds = 0;
        for (int round = 0; round < max_rounds; ++round) {
            ++rounds;
            stage_correlations(lr, f_iso, s, lane);
            status = max(status, plain_nnls(DenseGram{lr.gram, lr.c}, lr.c, lr.tol, s, lane));
            plain_fractions(lr, s.x, s, false, -1.f, lane);
            bool converged = true;
            for (int j = 0; j < 1 + ci; ++j) converged &= fabsf(fr[j] - prev[j]) < fraction_tol;
            __syncwarp();
            if (lane < ci) f_iso[lane] = fr[1 + lane];
            __syncwarp();
            if (converged) break;
            if (lane < 1 + ci) prev[lane] = fr[lane];
            __syncwarp();
        }
        stage_correlations(hr, f_iso, s, lane);
        status = max(status, plain_nnls(DenseGram{hr.gram, hr.c}, hr.c, hr.tol, s, lane));
        for (int j = lane; j < hr.c; j += 32) fods[voxel * hr.c + j] = s.x[j];
        const int nf = plain_fractions(hr, s.x, s, true, final_tol, lane);
        float total = kPlainFractionOffset;
        for (int j = 0; j < nf; ++j) total += fr[j];
        if (lane < nf) fractions[voxel * nf + lane] = fr[lane] / total;
        if (lane == 0) {
            if (rounds_out) rounds_out[voxel] = rounds;
            if (status_out) status_out[voxel] = uint8_t(status);
        }
        __syncwarp();
    }
}

// ---- MSMT-CSD (LSI) -------------------------------------------------------------------------

// The plain single-precision LSI fit, the comparison baseline of lsi_kernel: one warp per voxel in
// FP32 with the textbook forms of the reference's steps (cpp/src/sd/lsi.cpp:253-338):
// rotated = q_t s; f = -E rotated scaled to max |f| = 1 (the unconstrained solution back rotated
// when f = 0); the LDP multipliers u >= 0 by Lawson-Hanson on H = E E^T + f f^T with right-hand
// side f (plain_nnls: the gradient f - H u is the LDP's f (1 - f.u) - E E^T u, the Cholesky factor
// of H_AA formed anew for every fit); x = back (scale E^T u / (1 - f.u) + rotated). No QR
// fallback: a voxel whose factor fails (or outgrows kPlainMaxActive) gets status 1, a step
// limit status 3, f = 0 status 2.
struct LdpGram {
    const float* gram;  // (k, k) E E^T
    const float* f;     // (k,) the voxel's scaled bounds
    int k;
    __device__ __forceinline__ float operator()(int i, int j) const { return gram[size_t(i) * k + j] + f[i] * f[j]; }
};

__host__ __device__ inline size_t plain_lsi_warp_bytes(int k) {
    const size_t floats = 2 * 64 + size_t(4) * k + size_t(NA) * NA + NA + 64;
    return (floats * 4 + (NA + 4) * 4 + size_t(k) + 15) / 16 * 16;
}

__device__ Scratch carve_lsi(unsigned char* base, int k, float*& rot, float*& tv) {
    Scratch s{};
    float* f = reinterpret_cast<float*>(base);
    rot = f;
    tv = rot + 64;
    s.corr = tv + 64;  // the bounds f: the NNLS right-hand side
    s.x = s.corr + k;  // the multipliers u
    s.z = s.x + k;
    s.g = s.z + k;
    s.L = s.g + k;
    s.y = s.L + NA * NA;
    s.small = s.y + NA;
    s.idx = reinterpret_cast<int*>(s.small + 64);
    s.meta = s.idx + NA;
    s.act = reinterpret_cast<unsigned char*>(s.meta + 4);
    return s;
}

__global__ void __launch_bounds__(kPlainWarps * 32) plain_lsi_kernel(PlainLsi D, const float* __restrict__ signals,
                                                                     int64_t v, float* __restrict__ x_out,
                                                                     uint8_t* __restrict__ status_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m = D.m, n = D.n, k = D.k;
    float *rot, *tv;
    const Scratch s = carve_lsi(smem_raw + warp * plain_lsi_warp_bytes(k), k, rot, tv);
    float* f = s.corr;
    for (int64_t voxel = int64_t(blockIdx.x) * kPlainWarps + warp; voxel < v;
         voxel += int64_t(gridDim.x) * kPlainWarps) {
        const float* sv = signals + voxel * m;
        for (int i = lane; i < n; i += 32) {
            float acc = 0.f;
            for (int j = 0; j < m; ++j) acc += D.qt[size_t(j) * n + i] * sv[j];
            rot[i] = acc;
        }
        __syncwarp();
        float scale = 0.f;
        for (int j = lane; j < k; j += 32) {
            float acc = 0.f;
            for (int i = 0; i < n; ++i) acc += D.et[size_t(i) * k + j] * rot[i];
            f[j] = -acc;
            scale = fmaxf(scale, fabsf(acc));
        }
        scale = wmax(scale);
        __syncwarp();
        uint8_t st = 0;
        if (!(scale > 0.f)) {
            for (int i = lane; i < n; i += 32) {
                float acc = 0.f;
                for (int j = 0; j < n; ++j) acc += D.back[size_t(i) * n + j] * rot[j];
                x_out[voxel * n + i] = acc;
            }
            st = 2;
        } else {
            float norm1 = 0.f;
            for (int j = lane; j < k; j += 32) {
                f[j] /= scale;
                norm1 = fmaxf(norm1, D.abs_sums[j] + fabsf(f[j]));
            }
            norm1 = wmax(norm1);
            __syncwarp();
            const float tol = 10.f * kEps32 * norm1 * float(max(n + 1, k));
            const int r = plain_nnls(LdpGram{D.gram, f, k}, k, tol, s, lane);
            st = r == 0 ? 0 : (r == 1 ? 1 : 3);
            float fu = 0.f;
            for (int j = lane; j < k; j += 32) fu += f[j] * s.x[j];
            fu = wsum(fu);
            for (int i = lane; i < n; i += 32) {
                float acc = 0.f;
                for (int j = 0; j < k; ++j) acc += D.e[size_t(j) * n + i] * s.x[j];
                tv[i] = scale * acc / (1.f - fu) + rot[i];
            }
            __syncwarp();
            for (int i = lane; i < n; i += 32) {
                float acc = 0.f;
                for (int j = 0; j < n; ++j) acc += D.back[size_t(i) * n + j] * tv[j];
                x_out[voxel * n + i] = acc;
            }
        }
        if (lane == 0 && status_out) status_out[voxel] = st;
        __syncwarp();
    }
}

}  // namespace

void launch_plain_lsi(const PlainLsi& D, const float* signals, int64_t v, float* x, uint8_t* status,
                      cudaStream_t stream) {
    if (v == 0) return;
    require(D.n <= kPlainLsiMaxParameters && D.k <= kPlainLsiMaxConstraints,
            "the plain FP32 LSI fit takes at most 63 parameters and 512 constraints");
    const size_t smem = plain_lsi_warp_bytes(D.k) * kPlainWarps;
    cuda_check(cudaFuncSetAttribute(plain_lsi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "cudaFuncSetAttribute");
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, plain_lsi_kernel, kPlainWarps * 32, smem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    const int64_t blocks = std::max<int64_t>(
        1, std::min<int64_t>((v + kPlainWarps - 1) / kPlainWarps, int64_t(sm_count()) * std::max(per_sm, 1)));
    LaunchScope scope("plain_lsi_kernel", stream);
    plain_lsi_kernel<<<unsigned(blocks), kPlainWarps * 32, smem, stream>>>(D, signals, v, x, status);
    cuda_check(cudaGetLastError(), "plain_lsi_kernel launch");
}

void launch_plain_fp32(const PlainStage& lr, const PlainStage& hr, const float* signals, int64_t v,
                       const float* weights, int max_rounds, float fraction_tol, float final_tol, float* fods,
                       float* fractions, int32_t* rounds, uint8_t* status, cudaStream_t stream) {
    if (v == 0) return;
    const int ng = std::max(1, hr.nb);
    const size_t smem = plain_warp_bytes(lr.m, std::max(lr.c, hr.c), ng) * kPlainWarps;
    require(smem <= 200 * 1024, "the plain FP32 fit's per-warp state does not fit in shared memory");
    cuda_check(cudaFuncSetAttribute(plain_fp32_mfod_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "cudaFuncSetAttribute");
    int per_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, plain_fp32_mfod_kernel, kPlainWarps * 32, smem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    const int64_t blocks = std::max<int64_t>(
        1, std::min<int64_t>((v + kPlainWarps - 1) / kPlainWarps, int64_t(sm_count()) * std::max(per_sm, 1)));
    LaunchScope scope("plain_fp32_mfod_kernel", stream);
    plain_fp32_mfod_kernel<<<unsigned(blocks), kPlainWarps * 32, smem, stream>>>(
        lr, hr, signals, v, weights, max_rounds, fraction_tol, final_tol, fods, fractions, rounds, status, ng);
    cuda_check(cudaGetLastError(), "plain_fp32_mfod_kernel launch");
}

}  // namespace lar
