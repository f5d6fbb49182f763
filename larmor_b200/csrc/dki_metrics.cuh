// Device math of the DKI maps: Carlson's symmetric elliptic integrals and the tensor metrics
// of src/larmor/dwi/dki.py:285-540 (compute_kurtosis_metrics).
#pragma once

#include <cmath>

namespace lar {

// Carlson's R_F(x, y, z) by the duplication theorem and the fifth-order series of
// B. C. Carlson, "Numerical computation of real or complex elliptic integrals",
// Numerical Algorithms 10 (1995) 13-26, eq. (2.2)-(2.7); x, y, z >= 0, at most one zero.
__host__ __device__ inline double carlson_rf(double x, double y, double z) {
    const double r = 1e-16;
    double a0 = (x + y + z) / 3.0;
    double q = pow(3.0 * r, -1.0 / 6.0) * fmax(fabs(a0 - x), fmax(fabs(a0 - y), fabs(a0 - z)));
    double a = a0, xm = x, ym = y, zm = z, f = 1.0;  // f = 4^-m
    for (int m = 0; m < 40 && f * q >= fabs(a); ++m) {
        const double sx = sqrt(xm), sy = sqrt(ym), sz = sqrt(zm);
        const double lam = sx * sy + sx * sz + sy * sz;
        a = 0.25 * (a + lam);
        xm = 0.25 * (xm + lam);
        ym = 0.25 * (ym + lam);
        zm = 0.25 * (zm + lam);
        f *= 0.25;
    }
    const double X = (a0 - x) * f / a, Y = (a0 - y) * f / a, Z = -X - Y;
    const double e2 = X * Y - Z * Z, e3 = X * Y * Z;
    return (1.0 - e2 / 10.0 + e3 / 14.0 + e2 * e2 / 24.0 - 3.0 * e2 * e3 / 44.0) / sqrt(a);
}

// Carlson's R_D(x, y, z) (ibid., eq. (2.28)-(2.29)); x, y >= 0 (not both zero), z > 0.
__host__ __device__ inline double carlson_rd(double x, double y, double z) {
    const double r = 1e-16;
    double a0 = (x + y + 3.0 * z) / 5.0;
    double q = pow(0.25 * r, -1.0 / 6.0) * fmax(fabs(a0 - x), fmax(fabs(a0 - y), fabs(a0 - z)));
    double a = a0, xm = x, ym = y, zm = z, f = 1.0, sum = 0.0;
    for (int m = 0; m < 40 && f * q >= fabs(a); ++m) {
        const double sx = sqrt(xm), sy = sqrt(ym), sz = sqrt(zm);
        const double lam = sx * sy + sx * sz + sy * sz;
        sum += f / (sz * (zm + lam));
        a = 0.25 * (a + lam);
        xm = 0.25 * (xm + lam);
        ym = 0.25 * (ym + lam);
        zm = 0.25 * (zm + lam);
        f *= 0.25;
    }
    const double X = (a0 - x) * f / a, Y = (a0 - y) * f / a, Z = -(X + Y) / 3.0;
    const double xy = X * Y, z2 = Z * Z;
    const double e2 = xy - 6.0 * z2, e3 = (3.0 * xy - 8.0 * z2) * Z, e4 = 3.0 * (xy - z2) * z2,
                 e5 = xy * z2 * Z;
    const double series = 1.0 - 3.0 * e2 / 14.0 + e3 / 6.0 + 9.0 * e2 * e2 / 88.0 - 3.0 * e4 / 22.0 -
                          9.0 * e2 * e3 / 52.0 + 3.0 * e5 / 26.0;
    return f * series / (a * sqrt(a)) + 3.0 * sum;
}

// The weight of W1111 in MK for eigenvalues a, b, c (a != b, a != c) (Tabesh et al. 2011;
// src/larmor/dwi/dki.py:453-460).
__host__ __device__ inline double mk_f1(double a, double b, double c) {
    const double rf = carlson_rf(a / b, a / c, 1.0), rd = carlson_rd(a / b, a / c, 1.0);
    const double bc = sqrt(b * c);
    const double bracket = bc / a * rf + (3.0 * a * a - a * b - a * c - b * c) / (3.0 * a * bc) * rd - 1.0;
    return (a + b + c) * (a + b + c) / (18.0 * (a - b) * (a - c)) * bracket;
}

// The weight of W2233 in MK (b != c) (src/larmor/dwi/dki.py:463-470).
__host__ __device__ inline double mk_f2(double a, double b, double c) {
    const double rf = carlson_rf(a / b, a / c, 1.0), rd = carlson_rd(a / b, a / c, 1.0);
    const double bc = sqrt(b * c);
    const double bracket = (b + c) / bc * rf + (2.0 * a - b - c) / (3.0 * bc) * rd - 2.0;
    return (a + b + c) * (a + b + c) / (3.0 * (b - c) * (b - c)) * bracket;
}

// MK from eigenvalues (descending) and the eigenframe components
// wt = (W1111, W2222, W3333, W1122, W1133, W2233) (src/larmor/dwi/dki.py:473-484).
__host__ __device__ inline double mean_kurtosis(double l1, double l2, double l3, const double* wt) {
    return mk_f1(l1, l2, l3) * wt[0] + mk_f1(l2, l1, l3) * wt[1] + mk_f1(l3, l2, l1) * wt[2] +
           mk_f2(l1, l2, l3) * wt[5] + mk_f2(l2, l1, l3) * wt[4] + mk_f2(l3, l2, l1) * wt[3];
}

// RK (src/larmor/dwi/dki.py:487-495).
__host__ __device__ inline double radial_kurtosis(double l1, double l2, double l3, const double* wt) {
    const double pre = (l1 + l2 + l3) * (l1 + l2 + l3) / ((l2 - l3) * (l2 - l3));
    const double s23 = sqrt(l2 * l3);
    const double g12 = pre / (18.0 * l2) * (2.0 * l2 + (l3 * l3 - 3.0 * l2 * l3) / s23);
    const double g13 = pre / (18.0 * l3) * (2.0 * l3 + (l2 * l2 - 3.0 * l2 * l3) / s23);
    const double g2 = pre / 3.0 * ((l2 + l3) / s23 - 2.0);
    return g12 * wt[1] + g13 * wt[2] + g2 * wt[5];
}

}  // namespace lar
