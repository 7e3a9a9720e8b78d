// Host-side inverse of a band matrix, for the direct solve of the first coarse
// multigrid level (multigrid.cu).  Plain C++: the tests build it with g++ and
// check it against numpy.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <vector>

namespace pic {

// Inverse of a band matrix (every coupling within bw of the diagonal) by LU
// factorisation without pivoting, then one forward and one back substitution
// per column of the identity: O(n bw^2 + n^2 bw).  The level operators are
// M-matrices (weakly diagonally dominant, dominant on the rows next to a
// Dirichlet node), for which elimination without pivoting is stable.
inline bool band_inverse(std::vector<double>& a, int n, int bw) {
    auto A = [&](int r, int c) -> double& { return a[size_t(r) * n + c]; };
    for (int k = 0; k < n; ++k) {
        const double p = A(k, k);
        if (!(std::fabs(p) > 1e-300)) return false;
        const int last = std::min(n - 1, k + bw);
        for (int r = k + 1; r <= last; ++r) {
            const double m = A(r, k) / p;
            if (m == 0.0) continue;
            A(r, k) = m;
            for (int c = k + 1; c <= last; ++c) A(r, c) -= m * A(k, c);
        }
    }
    std::vector<double> inv(size_t(n) * n), x(n);
    for (int col = 0; col < n; ++col) {
        // L y = e_col (unit lower triangle; y is zero above col)
        std::fill(x.begin(), x.end(), 0.0);
        x[col] = 1.0;
        for (int i = col + 1; i < n; ++i) {
            double s = 0.0;
            for (int k = std::max(col, i - bw); k < i; ++k) s += A(i, k) * x[k];
            x[i] = -s;
        }
        // U x = y
        for (int i = n - 1; i >= 0; --i) {
            double s = x[i];
            const int last = std::min(n - 1, i + bw);
            for (int k = i + 1; k <= last; ++k) s -= A(i, k) * x[k];
            x[i] = s / A(i, i);
        }
        for (int i = 0; i < n; ++i) inv[size_t(i) * n + col] = x[i];
    }
    a.swap(inv);
    return true;
}

}  // namespace pic
