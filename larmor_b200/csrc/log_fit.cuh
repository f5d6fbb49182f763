// Device view of a prepared log-signal design (see log_fit.cu).
#pragma once

#include <cstdint>

namespace lar {

template <class T>
struct LogDesignDevice {
    int n = 0, p = 0, m = 0;
    const T* x = nullptr;          // (n, p) unit-norm columns
    const T* pinvt = nullptr;      // (n, p) transposed pseudo-inverse
    const T* z = nullptr;          // (n, p(p+1)/2) products x_na x_nb, a <= b
    const T* g = nullptr;          // (m, p) constraints, column-scaled
    const T* scales = nullptr;     // (p,) column norms
    const double* scales64 = nullptr;  // (p,) column norms in double, for the outputs
};

}  // namespace lar
