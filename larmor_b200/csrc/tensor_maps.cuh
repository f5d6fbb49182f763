// Eigen-decomposition of the diffusion tensor and the DTI maps of compute_dti_metrics
// (src/larmor/dwi/dti.py:170-235), shared by the DTI and DKI epilogues.
#pragma once

#include <cmath>
#include <cstdint>

namespace lar {

// Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations (Jacobi 1846;
// Golub & Van Loan 8.5): eigenvalues in w, eigenvectors in the columns of q.
template <class T>
__device__ __forceinline__ T eps_of();
template <>
__device__ __forceinline__ double eps_of<double>() { return 2.220446049250313e-16; }
template <>
__device__ __forceinline__ float eps_of<float>() { return 1.1920929e-07f; }

template <class T>
__device__ __forceinline__ void jacobi3(T (&a)[3][3], T (&w)[3], T (&q)[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) q[i][j] = i == j ? T(1) : T(0);
    for (int sweep = 0; sweep < 12; ++sweep) {
        bool rotated = false;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0;
            const int r = pq == 0 ? 1 : 2;
            const T apq = a[p][r];
            const T app = a[p][p], arr = a[r][r];
            // An off-diagonal entry below rounding of its diagonal pair is zero.
            if (fabs(apq) <= T(1e-3) * eps_of<T>() * (fabs(app) + fabs(arr)) ||
                apq == T(0)) {
                a[p][r] = a[r][p] = T(0);
                continue;
            }
            rotated = true;
            const T theta = (arr - app) / (T(2) * apq);
            const T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
            const T c = T(1) / sqrt(t * t + T(1));
            const T s = t * c;
            a[p][p] = app - t * apq;
            a[r][r] = arr + t * apq;
            a[p][r] = a[r][p] = T(0);
            const int o = 3 - p - r;
            const T aop = a[o][p], aor = a[o][r];
            a[o][p] = a[p][o] = c * aop - s * aor;
            a[o][r] = a[r][o] = s * aop + c * aor;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const T qp = q[i][p], qr = q[i][r];
                q[i][p] = c * qp - s * qr;
                q[i][r] = s * qp + c * qr;
            }
        }
        if (!rotated) break;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) w[i] = a[i][i];
}

template <class T>
__device__ __forceinline__ T zero_nan(T x) { return isnan(x) ? T(0) : x; }

// The maps of compute_dti_metrics (src/larmor/dwi/dti.py:170-235) of one voxel's tensor
// elements d (xx, xy, xz, yy, yz, zz), written as 16 rows of maps (stride v).
template <class T>
__device__ __forceinline__ void dti_maps(const T (&d)[6], int64_t voxel, int64_t v,
                                         float* __restrict__ maps, uint8_t* __restrict__ npd,
                                         T (*vec_out)[3] = nullptr, T* val_out = nullptr) {
    T ev[3] = {T(0), T(0), T(0)};
    T pe[3] = {T(NAN), T(NAN), T(NAN)};
    bool finite = true;
#pragma unroll
    for (int i = 0; i < 6; ++i) finite &= isfinite(d[i]);
    if (finite) {
        T a[3][3] = {{d[0], d[1], d[2]}, {d[1], d[3], d[4]}, {d[2], d[4], d[5]}};
        T w[3], q[3][3];
        jacobi3<T>(a, w, q);
        // Descending order by a sorting network on (value, column) pairs; selects keep
        // everything in registers.
        T c0[3] = {q[0][0], q[1][0], q[2][0]}, c1[3] = {q[0][1], q[1][1], q[2][1]},
          c2[3] = {q[0][2], q[1][2], q[2][2]};
        T w0 = w[0], w1 = w[1], w2 = w[2];
        auto swap_if = [](T& wa, T (&ca)[3], T& wb, T (&cb)[3]) {
            const bool s = wa < wb;
            const T t = wa; wa = s ? wb : wa; wb = s ? t : wb;
#pragma unroll
            for (int i = 0; i < 3; ++i) { const T u = ca[i]; ca[i] = s ? cb[i] : ca[i]; cb[i] = s ? u : cb[i]; }
        };
        swap_if(w0, c0, w1, c1);
        swap_if(w1, c1, w2, c2);
        swap_if(w0, c0, w1, c1);
        ev[0] = w0; ev[1] = w1; ev[2] = w2;
#pragma unroll
        for (int i = 0; i < 3; ++i) pe[i] = c0[i];
        if (vec_out) {
#pragma unroll
            for (int i = 0; i < 3; ++i) { vec_out[0][i] = c0[i]; vec_out[1][i] = c1[i]; vec_out[2][i] = c2[i]; }
        }
    }
    if (val_out) { val_out[0] = ev[0]; val_out[1] = ev[1]; val_out[2] = ev[2]; val_out[3] = finite ? T(1) : T(0); }
    const T l1 = zero_nan(ev[0]), l2 = zero_nan(ev[1]), l3 = zero_nan(ev[2]);
    const T md = zero_nan((d[0] + d[3] + d[5]) / T(3));
    const T num_sq = (l1 - l2) * (l1 - l2) + (l2 - l3) * (l2 - l3) + (l3 - l1) * (l3 - l1);
    const T num = sqrt(fmax(num_sq, T(0)));
    const T den = sqrt(l1 * l1 + l2 * l2 + l3 * l3);
    T fa = den > T(1e-12) ? sqrt(T(0.5)) * (num / den) : T(0);
    fa = zero_nan(fmin(fmax(fa, T(0)), T(1)));
#pragma unroll
    for (int i = 0; i < 6; ++i) maps[i * v + voxel] = float(d[i]);
    maps[6 * v + voxel] = float(fa);
    maps[7 * v + voxel] = float(md);
    maps[8 * v + voxel] = float(l1);
    maps[9 * v + voxel] = float((l2 + l3) / T(2));
#pragma unroll
    for (int i = 0; i < 3; ++i) maps[(10 + i) * v + voxel] = float(pe[i]);
    maps[13 * v + voxel] = float(l1);
    maps[14 * v + voxel] = float(l2);
    maps[15 * v + voxel] = float(l3);
    npd[voxel] = l3 <= T(0) ? 1 : 0;
}

}  // namespace lar
