// The DKI maps on the GPU, one thread per voxel: the DTI maps of the diffusion tensor, the
// kurtosis tensor W = (MD^2 W) / MD^2, S0, and MK, AK, RK, KA of compute_kurtosis_metrics
// (src/larmor/dwi/dki.py:261-282, :285-342, :517-540), in FP64.
//
// MK and RK use the closed forms of Tabesh et al. (2011) in the eigenframe of D, with
// Carlson's R_F and R_D (dki_metrics.cuh); where two eigenvalues are closer than 3e-4 MD they
// are extrapolated from three shifted eigenvalue sets (3 f(h) - 3 f(2h) + f(3h)), as the
// reference does. KA is the standard deviation of K(n) = MD^2 W(n) / D(n)^2 over the
// 16 x 32 node half-sphere quadrature (Gauss-Legendre in cos(theta), uniform in phi).
//
// Layout of maps (36, v): rows 0-15 the DTI maps (dt 6, fa, md, ad, rd, pe 3, eigen_vals 3),
// rows 16-30 kt, row 31 s0, rows 32-35 mk, ak, rk, ka.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "dki_metrics.cuh"
#include "tensor_maps.cuh"

namespace lar {

namespace {

constexpr int kKaTheta = 16, kKaPhi = 32, kKaNodes = kKaTheta * kKaPhi;
constexpr double kDegenerateGap = 3e-4;
constexpr double kPi = 3.14159265358979323846;

// The unique element of W for the multiset of indices with n0 zeros, n1 ones, n2 twos, in
// the order of DKIFit.kt (src/larmor/dwi/dki.py:30-46).
__host__ __device__ constexpr int kt_index(int n0, int n1, int n2) {
    return n0 == 4 ? 0 : n1 == 4 ? 1 : n2 == 4 ? 2
         : (n0 == 3 && n1 == 1) ? 3 : (n0 == 3 && n2 == 1) ? 4
         : (n1 == 3 && n0 == 1) ? 5 : (n1 == 3 && n2 == 1) ? 6
         : (n2 == 3 && n0 == 1) ? 7 : (n2 == 3 && n1 == 1) ? 8
         : (n0 == 2 && n1 == 2) ? 9 : (n0 == 2 && n2 == 2) ? 10 : (n1 == 2 && n2 == 2) ? 11
         : n0 == 2 ? 12 : n1 == 2 ? 13 : 14;
}

__device__ __forceinline__ double w_elem(const double* w, int a, int b, int c, int d) {
    const int n0 = (a == 0) + (b == 0) + (c == 0) + (d == 0);
    const int n1 = (a == 1) + (b == 1) + (c == 1) + (d == 1);
    return w[kt_index(n0, n1, 4 - n0 - n1)];
}

// W(u, u, v, v) = sum_abcd W_abcd u_a u_b v_c v_d.
__device__ __forceinline__ double w_uuvv(const double* w, const double* u, const double* v) {
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            double inner = 0.0;
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int d = 0; d < 3; ++d) inner += w_elem(w, a, b, c, d) * v[c] * v[d];
            s += u[a] * u[b] * inner;
        }
    return s;
}

struct KaQuadrature {
    const double* dbasis;  // (nodes, 6)
    const double* wbasis;  // (nodes, 15)
    const double* weight;  // (nodes,)
};

// The 36 DKI maps of one voxel from its 22 parameters.
__device__ __forceinline__ void dki_maps_voxel(const double* __restrict__ params, int64_t voxel, int64_t v,
                                               const KaQuadrature& quad, float* __restrict__ maps,
                                               uint8_t* __restrict__ npd) {
    const double* p = params + voxel * 22;
    double d[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) d[i] = p[1 + i];
    const double md_fit = (d[0] + d[3] + d[5]) / 3.0;
    double w[15];
#pragma unroll
    for (int i = 0; i < 15; ++i) w[i] = md_fit > 0.0 ? p[7 + i] / (md_fit * md_fit) : 0.0;
    double vec[3][3], val[4];
    dti_maps<double>(d, voxel, v, maps, npd, vec, val);
#pragma unroll
    for (int i = 0; i < 15; ++i) maps[(16 + i) * v + voxel] = float(w[i]);
    maps[31 * v + voxel] = float(exp(p[0]));

    double mk = 0.0, ak = 0.0, rk = 0.0, ka = 0.0;
    bool finite = val[3] != 0.0;
#pragma unroll
    for (int i = 0; i < 15; ++i) finite &= bool(isfinite(w[i]));
    const double l1 = val[0], l2 = val[1], l3 = val[2];
    if (finite && l3 > 0.0) {
        double wt[6];
        wt[0] = w_uuvv(w, vec[0], vec[0]);
        wt[1] = w_uuvv(w, vec[1], vec[1]);
        wt[2] = w_uuvv(w, vec[2], vec[2]);
        wt[3] = w_uuvv(w, vec[0], vec[1]);
        wt[4] = w_uuvv(w, vec[0], vec[2]);
        wt[5] = w_uuvv(w, vec[1], vec[2]);
        const double md = (l1 + l2 + l3) / 3.0;
        ak = md * md * wt[0] / (l1 * l1);
        const double gap = fmin(l1 - l2, l2 - l3);
        if (!(gap < kDegenerateGap * md)) {
            mk = mean_kurtosis(l1, l2, l3, wt);
            rk = radial_kurtosis(l1, l2, l3, wt);
        } else {
            const double h = kDegenerateGap * md;
            double mkk[3], rkk[3];
#pragma unroll
            for (int k = 1; k <= 3; ++k) {
                const double a = l1 + k * 2.0 * h, b = l2 + k * h, c = l3;
                mkk[k - 1] = mean_kurtosis(a, b, c, wt);
                rkk[k - 1] = radial_kurtosis(a, b, c, wt);
            }
            mk = 3.0 * mkk[0] - 3.0 * mkk[1] + mkk[2];
            rk = 3.0 * rkk[0] - 3.0 * rkk[1] + rkk[2];
        }
        // KA: the spread of K(n) over the half-sphere quadrature (src/larmor/dwi/dki.py:517-540).
        const double md2 = md_fit * md_fit;
        double mean = 0.0, second = 0.0;
        for (int i = 0; i < kKaNodes; ++i) {
            const double* db = quad.dbasis + i * 6;
            const double* wb = quad.wbasis + i * 15;
            double dn = 0.0, wn = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) dn += d[k] * db[k];
#pragma unroll
            for (int k = 0; k < 15; ++k) wn += w[k] * wb[k];
            const double kn = md2 * wn / (dn * dn);
            mean += kn * quad.weight[i];
        }
        for (int i = 0; i < kKaNodes; ++i) {
            const double* db = quad.dbasis + i * 6;
            const double* wb = quad.wbasis + i * 15;
            double dn = 0.0, wn = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) dn += d[k] * db[k];
#pragma unroll
            for (int k = 0; k < 15; ++k) wn += w[k] * wb[k];
            const double dev = md2 * wn / (dn * dn) - mean;
            second += dev * dev * quad.weight[i];
        }
        ka = sqrt(fmax(second, 0.0));
    }
    maps[32 * v + voxel] = float(mk);
    maps[33 * v + voxel] = float(ak);
    maps[34 * v + voxel] = float(rk);
    maps[35 * v + voxel] = float(ka);
}

__global__ void __launch_bounds__(128) dki_maps_kernel(const double* __restrict__ params, int64_t v,
                                                       KaQuadrature quad, float* __restrict__ maps,
                                                       uint8_t* __restrict__ npd) {
    const int64_t voxel = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (voxel < v) dki_maps_voxel(params, voxel, v, quad, maps, npd);
}

// The DKI family of a batch (batch.cuh): one launch over every DKI volume, a CTA per ticket of
// kMapsBatchVoxels voxels of one volume.
__global__ void __launch_bounds__(kMapsBatchVoxels) batch_dki_maps_kernel(const DkiBatchJob* __restrict__ jobs,
                                                                          const int64_t* __restrict__ first,
                                                                          int n_jobs, KaQuadrature quad) {
    const int64_t t = blockIdx.x;
    if (t >= first[n_jobs]) return;
    const int j = ticket_job(first, n_jobs, t);
    const DkiBatchJob& job = jobs[j];
    const int64_t voxel = (t - first[j]) * kMapsBatchVoxels + threadIdx.x;
    if (voxel < job.v) dki_maps_voxel(job.params, voxel, job.v, quad, job.maps, job.npd);
}

// Gauss-Legendre nodes and weights on [-1, 1] by Newton's method on P_n with the three-term
// recurrence (Golub & Welsch 1969 give the same nodes as eigenvalues).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(size_t(n), 0.0);
    w.assign(size_t(n), 0.0);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5)), dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);
        x[size_t(i)] = z;
        w[size_t(i)] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

// The quadrature of _half_sphere_quadrature (src/larmor/dwi/dki.py:498-514) with the D and W
// basis rows of each node, uploaded once per device.
KaQuadrature ka_quadrature() {
    static std::mutex mutex;
    static std::map<int, double*> per_device;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(mutex);
    auto it = per_device.find(dev);
    if (it == per_device.end()) {
        std::vector<double> t, wt;
        gauss_legendre(2 * kKaTheta, t, wt);
        std::vector<std::pair<double, double>> upper;
        for (size_t i = 0; i < t.size(); ++i)
            if (t[i] > 0.0) upper.push_back({t[i], wt[i]});
        std::sort(upper.begin(), upper.end());
        std::vector<double> host(size_t(kKaNodes) * 22);
        double total = 0.0;
        for (const auto& u : upper) total += u.second * kKaPhi;
        static const int quads[15][4] = {{0, 0, 0, 0}, {1, 1, 1, 1}, {2, 2, 2, 2}, {0, 0, 0, 1}, {0, 0, 0, 2},
                                         {1, 1, 1, 0}, {1, 1, 1, 2}, {2, 2, 2, 0}, {2, 2, 2, 1}, {0, 0, 1, 1},
                                         {0, 0, 2, 2}, {1, 1, 2, 2}, {0, 0, 1, 2}, {1, 1, 0, 2}, {2, 2, 0, 1}};
        static const double mult[15] = {1, 1, 1, 4, 4, 4, 4, 4, 4, 6, 6, 6, 12, 12, 12};
        for (int it_ = 0; it_ < kKaTheta; ++it_) {
            const double ct = upper[size_t(it_)].first, st = std::sqrt(1.0 - ct * ct);
            for (int ip = 0; ip < kKaPhi; ++ip) {
                const double phi = 2.0 * kPi * ip / kKaPhi;
                const double n3[3] = {st * std::cos(phi), st * std::sin(phi), ct};
                const int node = it_ * kKaPhi + ip;
                double* db = host.data() + size_t(node) * 6;
                db[0] = n3[0] * n3[0]; db[1] = 2 * n3[0] * n3[1]; db[2] = 2 * n3[0] * n3[2];
                db[3] = n3[1] * n3[1]; db[4] = 2 * n3[1] * n3[2]; db[5] = n3[2] * n3[2];
                double* wb = host.data() + size_t(kKaNodes) * 6 + size_t(node) * 15;
                for (int k = 0; k < 15; ++k)
                    wb[k] = mult[k] * n3[quads[k][0]] * n3[quads[k][1]] * n3[quads[k][2]] * n3[quads[k][3]];
                host[size_t(kKaNodes) * 21 + size_t(node)] = upper[size_t(it_)].second / total;
            }
        }
        double* d = nullptr;
        cuda_check(cudaMalloc(&d, host.size() * sizeof(double)), "cudaMalloc");
        cuda_check(cudaMemcpy(d, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
        it = per_device.emplace(dev, d).first;
    }
    double* base = it->second;
    return KaQuadrature{base, base + size_t(kKaNodes) * 6, base + size_t(kKaNodes) * 21};
}

}  // namespace

void launch_batch_dki_maps(const DkiBatchJob* jobs, const int64_t* first, int n_jobs, int64_t tickets,
                           cudaStream_t stream) {
    if (n_jobs == 0 || tickets == 0) return;
    const KaQuadrature quad = ka_quadrature();
    LaunchScope scope("batch_dki_maps_kernel", stream);
    batch_dki_maps_kernel<<<unsigned(tickets), kMapsBatchVoxels, 0, stream>>>(jobs, first, n_jobs, quad);
    cuda_check(cudaGetLastError(), "batch_dki_maps_kernel launch");
}

void launch_dki_maps(const double* params, int64_t v, float* maps, uint8_t* npd, cudaStream_t stream) {
    if (v == 0) return;
    const KaQuadrature quad = ka_quadrature();
    const int64_t grid = (v + 127) / 128;
    LaunchScope scope("dki_maps_kernel", stream);
    dki_maps_kernel<<<unsigned(grid), 128, 0, stream>>>(params, v, quad, maps, npd);
    cuda_check(cudaGetLastError(), "dki_maps_kernel launch");
}

}  // namespace lar
