// Image-geometry matrices on the host, compiled with -ffp-contract=off.
//
// The physical→index matrix decides every sample's continuous index, so it must be
// the host reference's matrix to the bit: direction·diag(spacing) formed entry by
// entry (core/coord.rs:50-75), then inverted by Gauss–Jordan elimination with
// partial pivoting and a 1e-12 singularity threshold, in the reference's row and
// column order (core/matrix.rs:44-104).

#include <cmath>
#include <utility>

#include "internal.h"

namespace mi {

void index_to_physical(const mi_geometry& g, double* m) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m[r * 3 + c] = g.direction[r * 3 + c] * g.spacing[c];
}

bool invert3(const double* m, double* inv) {
    double a[3][6];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            a[r][c] = m[r * 3 + c];
            a[r][3 + c] = (r == c) ? 1.0 : 0.0;
        }
    }
    for (int col = 0; col < 3; ++col) {
        int piv = col;
        double best = std::fabs(a[col][col]);
        for (int r = col + 1; r < 3; ++r) {
            const double v = std::fabs(a[r][col]);
            if (v > best) {
                best = v;
                piv = r;
            }
        }
        if (best < 1e-12) return false;
        if (piv != col)
            for (int c = 0; c < 6; ++c) std::swap(a[col][c], a[piv][c]);
        const double diag = a[col][col];
        for (int c = 0; c < 6; ++c) a[col][c] /= diag;
        for (int r = 0; r < 3; ++r) {
            if (r == col) continue;
            const double factor = a[r][col];
            if (factor == 0.0) continue;
            for (int c = 0; c < 6; ++c) a[r][c] -= factor * a[col][c];
        }
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) inv[r * 3 + c] = a[r][3 + c];
    return true;
}

}  // namespace mi
