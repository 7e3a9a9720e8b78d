// C entry point over pic::band_inverse for tests/test_band_inverse.py.
#include "band_inverse.h"

extern "C" int band_inverse_c(double* a, int n, int bw) {
    std::vector<double> v(a, a + size_t(n) * n);
    if (!pic::band_inverse(v, n, bw)) return 1;
    std::copy(v.begin(), v.end(), a);
    return 0;
}
