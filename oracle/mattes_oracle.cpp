// CPU ORACLE — test infrastructure only.
//
// This file restates, in plain serial FP64 C++, the reference CPU algorithm for the
// Mattes mutual-information metric of sitk-rs (crate `sitk` v0.0.3). It is the
// checker for the CUDA library under sitk-rs_b200/: only tests/, the smoke check in
// __graft_entry__.py and the CPU-baseline legs of bench.py load it. Nothing in the
// product links or calls it.
//
// Parity status: the reference is Rust and cannot be built in this environment
// (no cargo/rustc, no network for its crates), and its own tests hold no golden
// vectors for this metric (all of its Mattes pins are relational). This oracle is
// therefore "parity unpinned" against the reference binary. It is pinned instead by
// (a) published SplitMix64 vectors, (b) the reference's relational tests re-created
// in tests/test_oracle.py, and (c) an independent numpy FP64 implementation
// (oracle/np_oracle.py) that must agree with this file.
//
// Arithmetic order follows the reference exactly. Rust never fuses a*b+c, so this
// file is compiled with -ffp-contract=off, and every sum is written in the
// reference's accumulation order. Citations are paths inside the reference crate
// (crates/sitk/src/...).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cfloat>
#include <vector>
#include <algorithm>
#include <limits>
#include <thread>

extern "C" {

typedef struct {
    int64_t size[3];
    double spacing[3];
    double origin[3];
    double direction[9];  // row-major
} or_geometry;

enum {
    OR_OK = 0,
    OR_TOO_FEW_BINS = 1,
    OR_CONSTANT_FIXED = 2,
    OR_CONSTANT_MOVING = 3,
    OR_SINGULAR_DIRECTION = 4,
    OR_BAD_ARGUMENT = 5,
};

enum { OR_AFFINE = 0, OR_EULER3D = 1, OR_VERSOR_RIGID3D = 2, OR_TRANSLATION = 3 };

}  // extern "C"

namespace {

const int PADDING = 2;  // registration/mattes.rs:92

// core/matrix.rs:9-21 — accumulator starts at 0.0, terms added in column order.
void mat_vec(const double* m, const double* v, double* out) {
    for (int r = 0; r < 3; ++r) {
        double acc = 0.0;
        for (int c = 0; c < 3; ++c) acc += m[r * 3 + c] * v[c];
        out[r] = acc;
    }
}

// core/matrix.rs:24-40 — zero entries of `a` are skipped.
void matmul(const double* a, const double* b, double* out) {
    for (int i = 0; i < 9; ++i) out[i] = 0.0;
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
            double ark = a[r * 3 + k];
            if (ark == 0.0) continue;
            for (int c = 0; c < 3; ++c) out[r * 3 + c] += ark * b[k * 3 + c];
        }
}

// core/matrix.rs:44-104 — Gauss–Jordan with partial pivoting, singular below 1e-12.
bool invert3(const double* m, double* inv) {
    const int n = 3, w = 6;
    double a[18];
    for (int r = 0; r < n; ++r) {
        for (int c = 0; c < w; ++c) a[r * w + c] = 0.0;
        for (int c = 0; c < n; ++c) a[r * w + c] = m[r * n + c];
        a[r * w + n + r] = 1.0;
    }
    for (int col = 0; col < n; ++col) {
        int pivot = col;
        double best = std::fabs(a[col * w + col]);
        for (int r = col + 1; r < n; ++r) {
            double val = std::fabs(a[r * w + col]);
            if (val > best) { best = val; pivot = r; }
        }
        if (best < 1e-12) return false;
        if (pivot != col)
            for (int c = 0; c < w; ++c) std::swap(a[col * w + c], a[pivot * w + c]);
        double diag = a[col * w + col];
        for (int c = 0; c < w; ++c) a[col * w + c] /= diag;
        for (int r = 0; r < n; ++r) {
            if (r == col) continue;
            double factor = a[r * w + col];
            if (factor == 0.0) continue;
            for (int c = 0; c < w; ++c) a[r * w + c] -= factor * a[col * w + c];
        }
    }
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) inv[r * n + c] = a[r * w + n + c];
    return true;
}

// core/coord.rs:50-88 — index→physical = direction·diag(spacing); physical→index is
// the Gauss–Jordan inverse of that composed matrix.
void index_to_physical(const or_geometry& g, double* m) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m[r * 3 + c] = g.direction[r * 3 + c] * g.spacing[c];
}

// ---------------------------------------------------------------------------
// Transforms (transform/parametric.rs). Each yields the stored (matrix, offset)
// its transform_point multiplies, and a per-point dense Jacobian.
// ---------------------------------------------------------------------------
struct Transform {
    int kind = OR_AFFINE;
    int nparams = 12;
    double matrix[9];
    double offset[3];
    double center[3];
    double p[12];
    bool compute_zyx = false;
    double vx = 0, vy = 0, vz = 0, vw = 1;  // versor (normalised)

    // transform/parametric.rs:549-553 (and :1103-1107, :1331-1335):
    // mat_vec(matrix, p) then + offset.
    void transform_point(const double* x, double* y) const {
        double mx[3];
        mat_vec(matrix, x, mx);
        for (int d = 0; d < 3; ++d) y[d] = mx[d] + offset[d];
    }

    // Jacobian of the mapped point w.r.t. the parameters at point x, row-major 3×P.
    void jacobian(const double* x, double* j) const {
        const int P = nparams;
        for (int i = 0; i < 3 * P; ++i) j[i] = 0.0;
        if (kind == OR_AFFINE) {
            // parametric.rs:589-602
            for (int i = 0; i < 3; ++i) {
                for (int c = 0; c < 3; ++c) j[i * P + (i * 3 + c)] = x[c] - center[c];
                j[i * P + (9 + i)] = 1.0;
            }
        } else if (kind == OR_TRANSLATION) {
            for (int i = 0; i < 3; ++i) j[i * P + i] = 1.0;
        } else if (kind == OR_EULER3D) {
            // parametric.rs:1125-1166
            double cx = std::cos(p[0]), sx = std::sin(p[0]);
            double cy = std::cos(p[1]), sy = std::sin(p[1]);
            double cz = std::cos(p[2]), sz = std::sin(p[2]);
            double px = x[0] - center[0], py = x[1] - center[1], pz = x[2] - center[2];
            if (compute_zyx) {
                j[0] = (cz * sy * cx + sz * sx) * py + (-cz * sy * sx + sz * cx) * pz;
                j[6] = (sz * sy * cx - cz * sx) * py + (-sz * sy * sx - cz * cx) * pz;
                j[12] = (cy * cx) * py + (-cy * sx) * pz;
                j[1] = (-cz * sy) * px + (cz * cy * sx) * py + (cz * cy * cx) * pz;
                j[7] = (-sz * sy) * px + (sz * cy * sx) * py + (sz * cy * cx) * pz;
                j[13] = (-cy) * px + (-sy * sx) * py + (-sy * cx) * pz;
                j[2] = (-sz * cy) * px + (-sz * sy * sx - cz * cx) * py + (-sz * sy * cx + cz * sx) * pz;
                j[8] = (cz * cy) * px + (cz * sy * sx - sz * cx) * py + (cz * sy * cx + sz * sx) * pz;
                j[14] = 0.0;
            } else {
                j[0] = (-sz * cx * sy) * px + (sz * sx) * py + (sz * cx * cy) * pz;
                j[6] = (cz * cx * sy) * px + (-cz * sx) * py + (-cz * cx * cy) * pz;
                j[12] = (sx * sy) * px + (cx) * py + (-sx * cy) * pz;
                j[1] = (-cz * sy - sz * sx * cy) * px + (cz * cy - sz * sx * sy) * pz;
                j[7] = (-sz * sy + cz * sx * cy) * px + (sz * cy + cz * sx * sy) * pz;
                j[13] = (-cx * cy) * px + (-cx * sy) * pz;
                j[2] = (-sz * cy - cz * sx * sy) * px + (-cz * cx) * py + (-sz * sy + cz * sx * cy) * pz;
                j[8] = (cz * cy - sz * sx * sy) * px + (-sz * cx) * py + (cz * sy + sz * sx * cy) * pz;
                j[14] = 0.0;
            }
            j[3] = 1.0; j[10] = 1.0; j[17] = 1.0;
        } else {
            // parametric.rs:1355-1384
            double px = x[0] - center[0], py = x[1] - center[1], pz = x[2] - center[2];
            double vxx = vx * vx, vyy = vy * vy, vzz = vz * vz, vww = vw * vw;
            double vxy = vx * vy, vxz = vx * vz, vxw = vx * vw;
            double vyz = vy * vz, vyw = vy * vw, vzw = vz * vw;
            j[0] = 2.0 * ((vyw + vxz) * py + (vzw - vxy) * pz) / vw;
            j[6] = 2.0 * ((vyw - vxz) * px - 2.0 * vxw * py + (vxx - vww) * pz) / vw;
            j[12] = 2.0 * ((vzw + vxy) * px + (vww - vxx) * py - 2.0 * vxw * pz) / vw;
            j[1] = 2.0 * (-2.0 * vyw * px + (vxw + vyz) * py + (vww - vyy) * pz) / vw;
            j[7] = 2.0 * ((vxw - vyz) * px + (vzw + vxy) * pz) / vw;
            j[13] = 2.0 * ((vyy - vww) * px + (vzw - vxy) * py - 2.0 * vyw * pz) / vw;
            j[2] = 2.0 * (-2.0 * vzw * px + (vzz - vww) * py + (vxw - vyz) * pz) / vw;
            j[8] = 2.0 * ((vww - vzz) * px - 2.0 * vzw * py + (vyw + vxz) * pz) / vw;
            j[14] = 2.0 * ((vxw + vyz) * px + (vyw - vxz) * py) / vw;
            j[3] = 1.0; j[10] = 1.0; j[17] = 1.0;
        }
    }
};

// Build a transform from (kind, params, fixed params) the way each family's
// set_parameters / recompute does.
bool make_transform(int kind, const double* params, const double* fixed, int nfixed, Transform& t) {
    t.kind = kind;
    for (int d = 0; d < 3; ++d) t.center[d] = (fixed && nfixed >= 3) ? fixed[d] : 0.0;
    if (kind == OR_AFFINE) {
        // parametric.rs:566-573, compute_offset :522-527
        t.nparams = 12;
        for (int i = 0; i < 12; ++i) t.p[i] = params[i];
        for (int i = 0; i < 9; ++i) t.matrix[i] = params[i];
        double ac[3];
        mat_vec(t.matrix, t.center, ac);
        for (int d = 0; d < 3; ++d) t.offset[d] = t.center[d] + params[9 + d] - ac[d];
    } else if (kind == OR_TRANSLATION) {
        // parametric.rs:378-391: p + t; the identity matrix form is bitwise equal.
        t.nparams = 3;
        for (int i = 0; i < 3; ++i) t.p[i] = params[i];
        for (int i = 0; i < 9; ++i) t.matrix[i] = (i % 4 == 0) ? 1.0 : 0.0;
        for (int d = 0; d < 3; ++d) t.offset[d] = params[d];
    } else if (kind == OR_EULER3D) {
        // parametric.rs:1063-1086
        t.nparams = 6;
        for (int i = 0; i < 6; ++i) t.p[i] = params[i];
        t.compute_zyx = (fixed && nfixed == 4) ? (fixed[3] != 0.0) : false;
        double cx = std::cos(params[0]), sx = std::sin(params[0]);
        double cy = std::cos(params[1]), sy = std::sin(params[1]);
        double cz = std::cos(params[2]), sz = std::sin(params[2]);
        double rx[9] = {1.0, 0.0, 0.0, 0.0, cx, -sx, 0.0, sx, cx};
        double ry[9] = {cy, 0.0, sy, 0.0, 1.0, 0.0, -sy, 0.0, cy};
        double rz[9] = {cz, -sz, 0.0, sz, cz, 0.0, 0.0, 0.0, 1.0};
        double tmp[9];
        if (t.compute_zyx) { matmul(rz, ry, tmp); matmul(tmp, rx, t.matrix); }
        else { matmul(rz, rx, tmp); matmul(tmp, ry, t.matrix); }
        double mc[3];
        mat_vec(t.matrix, t.center, mc);
        for (int i = 0; i < 3; ++i) t.offset[i] = params[3 + i] + t.center[i] - mc[i];
    } else if (kind == OR_VERSOR_RIGID3D) {
        // parametric.rs:1310-1345 (set_versor, recompute)
        t.nparams = 6;
        for (int i = 0; i < 6; ++i) t.p[i] = params[i];
        const double EPS = 1e-10;
        double vx = params[0], vy = params[1], vz = params[2];
        double norm = std::sqrt(vx * vx + vy * vy + vz * vz);
        double ax = vx, ay = vy, az = vz;
        if (norm >= 1.0 - EPS) {
            double d = norm + EPS * norm;
            ax = vx / d; ay = vy / d; az = vz / d;
        }
        t.vx = ax; t.vy = ay; t.vz = az;
        double s = 1.0 - (ax * ax + ay * ay + az * az);
        t.vw = std::sqrt(s > 0.0 ? s : 0.0);
        double x = t.vx, y = t.vy, z = t.vz, w = t.vw;
        double xx = x * x, yy = y * y, zz = z * z;
        double xy = x * y, xz = x * z, xw = x * w;
        double yz = y * z, yw = y * w, zw = z * w;
        double m[9] = {
            1.0 - 2.0 * (yy + zz), 2.0 * (xy - zw), 2.0 * (xz + yw),
            2.0 * (xy + zw), 1.0 - 2.0 * (xx + zz), 2.0 * (yz - xw),
            2.0 * (xz - yw), 2.0 * (yz + xw), 1.0 - 2.0 * (xx + yy)};
        double mc[3];
        mat_vec(m, t.center, mc);
        for (int i = 0; i < 3; ++i) t.offset[i] = params[3 + i] + t.center[i] - mc[i];
        for (int i = 0; i < 9; ++i) t.matrix[i] = m[i];
    } else {
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Mattes pieces (registration/mattes.rs)
// ---------------------------------------------------------------------------

// mattes.rs:96-107
double cubic_bspline(double u) {
    double a = std::fabs(u);
    if (a < 1.0) {
        double sq = a * a;
        return (4.0 - 6.0 * sq + 3.0 * sq * a) / 6.0;
    } else if (a < 2.0) {
        double sq = a * a;
        return (8.0 - 12.0 * a + 6.0 * sq - sq * a) / 6.0;
    }
    return 0.0;
}

// mattes.rs:112-124
double cubic_bspline_derivative(double u) {
    if (u >= 0.0 && u < 1.0) return -2.0 * u + 1.5 * u * u;
    if (u > -1.0 && u < 0.0) return -2.0 * u - 1.5 * u * u;
    if (u >= 1.0 && u < 2.0) return -2.0 + 2.0 * u - 0.5 * u * u;
    if (u > -2.0 && u <= -1.0) return 2.0 + 2.0 * u + 0.5 * u * u;
    return 0.0;
}

struct Geometry {
    int bins;
    double moving_true_min, moving_true_max;
    double fixed_bin_size, moving_bin_size;
    double fixed_normalized_min, moving_normalized_min;
};

// mattes.rs:152-186
int make_geometry(double fmin, double fmax, double mmin, double mmax, int bins, Geometry& g) {
    if (bins < 2 * PADDING + 1) return OR_TOO_FEW_BINS;
    if (fmax - fmin <= DBL_EPSILON) return OR_CONSTANT_FIXED;
    if (mmax - mmin <= DBL_EPSILON) return OR_CONSTANT_MOVING;
    double denom = (double)(bins - 2 * PADDING);
    g.bins = bins;
    g.moving_true_min = mmin;
    g.moving_true_max = mmax;
    g.fixed_bin_size = (fmax - fmin) / denom;
    g.moving_bin_size = (mmax - mmin) / denom;
    g.fixed_normalized_min = fmin / g.fixed_bin_size - (double)PADDING;
    g.moving_normalized_min = mmin / g.moving_bin_size - (double)PADDING;
    return OR_OK;
}

// mattes.rs:193-206 — truncate toward zero, clamp to [padding, bins − padding − 1].
int parzen_index(double value, double bin_size, double nmin, int bins) {
    double term = value / bin_size - nmin;
    long long index = (long long)term;
    long long lo = PADDING, hi = (long long)bins - PADDING - 1;
    if (index < lo) index = lo;
    else if (index > hi) index = hi;
    return (int)index;
}

// core/compensated.rs:112-123 (ITK's Kahan recurrence; the sum is returned
// without folding the last compensation back in).
double kahan_sum(const double* v, size_t n) {
    double sum = 0.0, comp = 0.0;
    for (size_t i = 0; i < n; ++i) {
        double ci = v[i] - comp;
        double t = sum + ci;
        comp = (t - sum) - ci;
        sum = t;
    }
    return sum;
}

// The prepared sample set and moving image (registration/metric.rs:494-581, 722-924).
struct Problem {
    const float* fixed;
    or_geometry fg;
    const float* moving;
    or_geometry mg;
    const uint8_t* mmask;
    double f_i2p[9];
    double m_p2i[9];
    int64_t mstride[3];
    std::vector<int64_t> flats;  // selected voxels (after the fixed-mask filter); empty = full grid
    bool grid;
    int64_t n;  // sample count
};

// registration/scales.rs:259-271 — origin-seeded accumulation.
inline void grid_point(const Problem& P, int64_t flat, double* out) {
    double idx[3];
    int64_t f = flat;
    for (int d = 0; d < 3; ++d) {
        idx[d] = (double)(f % P.fg.size[d]);
        f /= P.fg.size[d];
    }
    for (int r = 0; r < 3; ++r) {
        double acc = P.fg.origin[r];
        for (int c = 0; c < 3; ++c) acc += P.f_i2p[r * 3 + c] * idx[c];
        out[r] = acc;
    }
}

// metric.rs:795-806 — c = M·(p − origin), the difference formed first.
inline void continuous_index(const Problem& P, const double* p, double* c) {
    for (int r = 0; r < 3; ++r) {
        double acc = -0.0;  // Rust's f64 Sum starts from −0.0; a finite result is unaffected
        for (int j = 0; j < 3; ++j) acc += P.m_p2i[r * 3 + j] * (p[j] - P.mg.origin[j]);
        c[r] = acc;
    }
}

// metric.rs:817-833 + core/coord.rs:185-191 — floor(c + 0.5), reject outside.
inline bool mask_allows(const Problem& P, const double* c) {
    if (!P.mmask) return true;
    int64_t flat = 0;
    for (int d = 0; d < 3; ++d) {
        int64_t r = (int64_t)std::floor(c[d] + 0.5);
        if (r < 0 || r >= P.mg.size[d]) return false;
        flat += r * P.mstride[d];
    }
    return P.mmask[flat] != 0;
}

// transform/interpolator.rs:29-34
inline bool is_inside(const Problem& P, const double* c) {
    for (int d = 0; d < 3; ++d)
        if (!(c[d] >= -0.5 && c[d] < (double)P.mg.size[d] - 0.5)) return false;
    return true;
}

// transform/interpolator.rs:103-152 + metric.rs:848-861 (physical gradient).
// Returns false when the point is outside the buffer or masked.
inline bool moving_value_grad(const Problem& P, const double* p, double* value, double* gphys,
                              bool want_grad) {
    double c[3];
    continuous_index(P, p, c);
    if (!mask_allows(P, c)) return false;
    if (!is_inside(P, c)) return false;
    double frac[3];
    int64_t base[3];
    for (int d = 0; d < 3; ++d) {
        double f = std::floor(c[d]);
        base[d] = (int64_t)f;
        frac[d] = c[d] - f;
    }
    double v = 0.0;
    double g[3] = {0.0, 0.0, 0.0};
    for (int corner = 0; corner < 8; ++corner) {
        int64_t off = 0;
        double weight = 1.0;
        for (int d = 0; d < 3; ++d) {
            int bit = (corner >> d) & 1;
            weight *= bit ? frac[d] : 1.0 - frac[d];
            int64_t idx = base[d] + bit;
            if (idx < 0) idx = 0;
            if (idx > P.mg.size[d] - 1) idx = P.mg.size[d] - 1;
            off += idx * P.mstride[d];
        }
        double b = (double)P.moving[off];
        v += weight * b;
        if (want_grad) {
            for (int j = 0; j < 3; ++j) {
                double wj = 1.0;
                for (int d = 0; d < 3; ++d) {
                    if (d == j) continue;
                    int bit = (corner >> d) & 1;
                    wj *= bit ? frac[d] : 1.0 - frac[d];
                }
                double sign = ((corner >> j) & 1) ? 1.0 : -1.0;
                g[j] += sign * wj * b;
            }
        }
    }
    *value = v;
    if (want_grad) {
        for (int d = 0; d < 3; ++d) {
            double acc = -0.0;
            for (int j = 0; j < 3; ++j) acc += g[j] * P.m_p2i[j * 3 + d];
            gphys[d] = acc;
        }
    }
    return true;
}

int prepare(const float* fixed, const or_geometry* fg, const float* moving, const or_geometry* mg,
            const uint8_t* fmask, const uint8_t* mmask, const int64_t* draw, int64_t ndraw,
            Problem& P) {
    P.fixed = fixed;
    P.fg = *fg;
    P.moving = moving;
    P.mg = *mg;
    P.mmask = mmask;
    index_to_physical(*fg, P.f_i2p);
    double m_i2p[9];
    index_to_physical(*mg, m_i2p);
    if (!invert3(m_i2p, P.m_p2i)) return OR_SINGULAR_DIRECTION;
    P.mstride[0] = 1;
    P.mstride[1] = mg->size[0];
    P.mstride[2] = mg->size[0] * mg->size[1];
    int64_t nvox = fg->size[0] * fg->size[1] * fg->size[2];
    // metric.rs:528-540 — the draw, then the fixed-mask filter; no list for the
    // unmasked full grid.
    if (!draw && !fmask) {
        P.grid = true;
        P.n = nvox;
        return OR_OK;
    }
    P.grid = false;
    P.flats.clear();
    if (!draw) {
        for (int64_t s = 0; s < nvox; ++s)
            if (fmask[s]) P.flats.push_back(s);
    } else {
        for (int64_t i = 0; i < ndraw; ++i) {
            int64_t f = draw[i];
            if (f < 0 || f >= nvox) return OR_BAD_ARGUMENT;
            if (!fmask || fmask[f]) P.flats.push_back(f);
        }
    }
    P.n = (int64_t)P.flats.size();
    return OR_OK;
}

inline int64_t sample_flat(const Problem& P, int64_t s) { return P.grid ? s : P.flats[s]; }

// Ranges that size the histogram (metric.rs:633-640 SampledPoints, :913-924 masked moving).
void ranges(const Problem& P, double* fmin, double* fmax, double* mmin, double* mmax) {
    double lo = INFINITY, hi = -INFINITY;
    for (int64_t s = 0; s < P.n; ++s) {
        double v = (double)P.fixed[sample_flat(P, s)];
        lo = std::fmin(lo, v);
        hi = std::fmax(hi, v);
    }
    if (P.n == 0) { lo = 0.0; hi = 0.0; }
    *fmin = lo; *fmax = hi;
    int64_t nm = P.mg.size[0] * P.mg.size[1] * P.mg.size[2];
    lo = INFINITY; hi = -INFINITY;
    bool any = false;
    for (int64_t i = 0; i < nm; ++i) {
        if (P.mmask && !P.mmask[i]) continue;
        double v = (double)P.moving[i];
        lo = std::fmin(lo, v);
        hi = std::fmax(hi, v);
        any = true;
    }
    if (!any) { lo = 0.0; hi = 0.0; }
    *mmin = lo; *mmax = hi;
}

struct Accum {
    std::vector<double> joint, fixed_marginal, jpd;
    int64_t valid = 0;
};

// The per-sample body of evaluate_global_support (mattes.rs:536-588), or of
// build_histogram (mattes.rs:451-483) when want_deriv is false.
template <class TransformT>
inline void sample_body(const Problem& P, const Geometry& G, const TransformT& T, int64_t s,
                        bool want_deriv, Accum& A, int8_t* status, int32_t* fi_out,
                        int32_t* mi_out) {
    const int bins = G.bins;
    const int np = T.nparams;
    int64_t flat = sample_flat(P, s);
    double fp[3], mp[3];
    if (P.grid) grid_point(P, flat, fp);
    else grid_point(P, flat, fp);  // metric.rs:339-348 — explicit points are write_point's
    double fv = (double)P.fixed[flat];
    T.transform_point(fp, mp);
    double mv, g[3];
    if (!moving_value_grad(P, mp, &mv, g, want_deriv)) {
        if (status) status[s] = 0;
        return;
    }
    if (mv < G.moving_true_min || mv > G.moving_true_max) {
        if (status) status[s] = 1;
        return;
    }
    double moving_term = mv / G.moving_bin_size - G.moving_normalized_min;
    int mi = parzen_index(mv, G.moving_bin_size, G.moving_normalized_min, bins);
    int fi = parzen_index(fv, G.fixed_bin_size, G.fixed_normalized_min, bins);
    if (status) status[s] = 2;
    if (fi_out) fi_out[s] = fi;
    if (mi_out) mi_out[s] = mi;
    A.fixed_marginal[fi] += 1.0;
    double jac[36];
    if (want_deriv) T.jacobian(fp, jac);
    int start = mi - 1;
    for (int m = start; m < start + 4; ++m) {
        double arg = (double)m - moving_term;
        double val = cubic_bspline(arg);
        A.joint[(size_t)fi * bins + m] += val;
        if (want_deriv) {
            double dw = cubic_bspline_derivative(arg);
            size_t base = ((size_t)fi * bins + m) * np;
            for (int k = 0; k < np; ++k) {
                double inner = 0.0;
                for (int d = 0; d < 3; ++d) inner += jac[d * np + k] * g[d];
                A.jpd[base + k] += inner * dw;
            }
        }
    }
    A.valid += 1;
}

// mattes.rs:590-676 (derivative) and mattes.rs:273-328 (value-only tail).
void finish(const Geometry& G, Accum& A, int np, bool want_deriv, double* value, double* deriv,
            int64_t* valid) {
    const int bins = G.bins;
    *valid = A.valid;
    for (int k = 0; k < np && deriv; ++k) deriv[k] = 0.0;
    if (A.valid == 0) { *value = DBL_MAX; return; }
    double joint_sum = kahan_sum(A.joint.data(), A.joint.size());
    if (joint_sum < DBL_EPSILON) { *value = DBL_MAX; return; }
    double n_factor = 1.0 / (G.moving_bin_size * (double)A.valid);
    if (want_deriv)
        for (auto& d : A.jpd) d *= n_factor;
    double inv_sum = 1.0 / joint_sum;
    for (auto& p : A.joint) p *= inv_sum;
    for (auto& p : A.fixed_marginal) p *= inv_sum;
    std::vector<double> mm(bins, 0.0);
    for (int f = 0; f < bins; ++f)
        for (int m = 0; m < bins; ++m) mm[m] += A.joint[(size_t)f * bins + m];
    const double close = DBL_EPSILON;
    double sum = 0.0;
    for (int f = 0; f < bins; ++f) {
        double fm = A.fixed_marginal[f];
        if (fm <= close) continue;
        double log_fm = std::log(fm);
        for (int m = 0; m < bins; ++m) {
            double mmv = mm[m];
            double jp = A.joint[(size_t)f * bins + m];
            if (mmv > close && jp > close) {
                double pr = std::log(jp / mmv);
                sum += jp * (pr - log_fm);
                if (want_deriv) {
                    size_t base = ((size_t)f * bins + m) * np;
                    for (int k = 0; k < np; ++k) deriv[k] += A.jpd[base + k] * pr;
                }
            }
        }
    }
    *value = -sum;
}

// A point map given as stages (matrix row-major, offset; 12 doubles each), replayed
// one by one as p ← mat_vec(M, p) + offset (transform/matrix_offset.rs:102-109), with
// a parameter Jacobian that is affine in the fixed point, J(x) = J0 + Σ_e x_e·C_e
// (the form registration/cuda.rs:294-363 affine_form recovers from a transform).
struct StageMap {
    int nstage = 0;
    int nparams = 0;
    double st[8][12];
    double jac0[36];
    double jacc[3][36];
    void transform_point(const double* x, double* y) const {
        double p[3] = {x[0], x[1], x[2]};
        for (int k = 0; k < nstage; ++k) {
            double q[3];
            mat_vec(st[k], p, q);
            for (int d = 0; d < 3; ++d) p[d] = q[d] + st[k][9 + d];
        }
        for (int d = 0; d < 3; ++d) y[d] = p[d];
    }
    void jacobian(const double* x, double* j) const {
        for (int i = 0; i < 3 * nparams; ++i) j[i] = jac0[i] + x[0] * jacc[0][i] + x[1] * jacc[1][i] + x[2] * jacc[2][i];
    }
};

// `draw` is the sampling strategy's draw BEFORE the fixed-mask filter (NULL = the
// whole grid). Per-sample outputs, when non-null, are indexed in post-filter sample
// order: status 0 = outside/masked, 1 = moving value out of range, 2 = valid; fi/mi
// are the Parzen bins of a valid sample. `nthreads` > 1 splits the samples into
// contiguous chunks with private accumulators folded in thread-index order (the
// reference's deterministic rayon rule, core/parallel.rs:766); 1 is the serial walk.
template <class TransformT>
int evaluate_with(const Problem& P, int bins, const TransformT& T, int want_derivative, int nthreads,
                  double* value, double* deriv, int64_t* valid, int8_t* status, int32_t* fi_out, int32_t* mi_out,
                  double* joint_out, double* fixed_marginal_out) {
    double fmin, fmax, mmin, mmax;
    ranges(P, &fmin, &fmax, &mmin, &mmax);
    Geometry G;
    int st = make_geometry(fmin, fmax, mmin, mmax, bins, G);
    if (st) return st;
    const bool wd = want_derivative != 0;
    const int np = T.nparams;
    if (nthreads < 1) nthreads = 1;
    std::vector<Accum> parts(nthreads);
    for (auto& a : parts) {
        a.joint.assign((size_t)bins * bins, 0.0);
        a.fixed_marginal.assign(bins, 0.0);
        if (wd) a.jpd.assign((size_t)bins * bins * np, 0.0);
    }
    const int64_t n = P.n;
    if (nthreads == 1) {
        for (int64_t s = 0; s < n; ++s) sample_body(P, G, T, s, wd, parts[0], status, fi_out, mi_out);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; ++t) {
            pool.emplace_back([&, t]() {
                int64_t lo = n * t / nthreads, hi = n * (t + 1) / nthreads;
                for (int64_t s = lo; s < hi; ++s)
                    sample_body(P, G, T, s, wd, parts[t], status, fi_out, mi_out);
            });
        }
        for (auto& th : pool) th.join();
        for (int t = 1; t < nthreads; ++t) {
            for (size_t i = 0; i < parts[0].joint.size(); ++i) parts[0].joint[i] += parts[t].joint[i];
            for (int i = 0; i < bins; ++i) parts[0].fixed_marginal[i] += parts[t].fixed_marginal[i];
            for (size_t i = 0; i < parts[0].jpd.size(); ++i) parts[0].jpd[i] += parts[t].jpd[i];
            parts[0].valid += parts[t].valid;
        }
    }
    Accum& A = parts[0];
    if (joint_out) std::memcpy(joint_out, A.joint.data(), A.joint.size() * sizeof(double));
    if (fixed_marginal_out) std::memcpy(fixed_marginal_out, A.fixed_marginal.data(), bins * sizeof(double));
    finish(G, A, np, wd, value, deriv, valid);
    return OR_OK;
}

}  // namespace

extern "C" {

// One SplitMix64 output (registration/metric.rs:110-116) after `state` has been
// advanced; exposed so a test can pin it against published vectors.
uint64_t or_splitmix64_next(uint64_t* state) {
    *state += 0x9E3779B97F4A7C15ULL;
    uint64_t z = *state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// registration/metric.rs:419-437. strategy: 0 None, 1 Regular, 2 Random.
// Returns the number of drawn voxels (written to `out` when non-null and cap allows),
// or −1 for the None strategy (the identity selection has no list).
int64_t or_draw_samples(int64_t voxels, int strategy, double percentage, uint64_t seed,
                        int64_t* out, int64_t cap) {
    if (strategy == 0) return -1;
    if (strategy == 1) {
        double inv = std::ceil(1.0 / percentage);
        int64_t stride = (int64_t)inv;
        if (stride < 1) stride = 1;
        int64_t n = 0;
        for (int64_t v = 0; v < voxels; v += stride, ++n)
            if (out && n < cap) out[n] = v;
        return n;
    }
    int64_t count = (int64_t)((double)voxels * percentage);
    uint64_t state = seed;
    for (int64_t i = 0; i < count; ++i) {
        uint64_t r = or_splitmix64_next(&state) % (uint64_t)voxels;
        if (out && i < cap) out[i] = (int64_t)r;
    }
    return count;
}

// Histogram geometry for a problem: [fixed_min, fixed_max, moving_min, moving_max,
// fixed_bin_size, moving_bin_size, fixed_normalized_min, moving_normalized_min],
// plus the sample count after the fixed-mask filter.
int or_metric_geometry(const float* fixed, const or_geometry* fg, const float* moving,
                       const or_geometry* mg, const uint8_t* fmask, const uint8_t* mmask,
                       const int64_t* draw, int64_t ndraw, int bins, double* out8,
                       int64_t* nsamples) {
    Problem P;
    int st = prepare(fixed, fg, moving, mg, fmask, mmask, draw, ndraw, P);
    if (st) return st;
    double fmin, fmax, mmin, mmax;
    ranges(P, &fmin, &fmax, &mmin, &mmax);
    Geometry G;
    out8[0] = fmin; out8[1] = fmax; out8[2] = mmin; out8[3] = mmax;
    if (nsamples) *nsamples = P.n;
    st = make_geometry(fmin, fmax, mmin, mmax, bins, G);
    if (st) return st;
    out8[4] = G.fixed_bin_size; out8[5] = G.moving_bin_size;
    out8[6] = G.fixed_normalized_min; out8[7] = G.moving_normalized_min;
    return OR_OK;
}

// The whole metric: value = −MI, derivative = +∇(−MI) (mattes.rs:522-676), or the
// value-only walk (mattes.rs:442-500) when want_derivative is 0.
//
int or_mattes_evaluate(const float* fixed, const or_geometry* fg, const float* moving,
                       const or_geometry* mg, const uint8_t* fmask, const uint8_t* mmask,
                       const int64_t* draw, int64_t ndraw, int bins, int kind,
                       const double* params, const double* fixed_params, int nfixed,
                       int want_derivative, int nthreads, double* value, double* deriv,
                       int64_t* valid, int8_t* status, int32_t* fi_out, int32_t* mi_out,
                       double* joint_out, double* fixed_marginal_out) {
    Problem P;
    int st = prepare(fixed, fg, moving, mg, fmask, mmask, draw, ndraw, P);
    if (st) return st;
    Transform T;
    if (!make_transform(kind, params, fixed_params, nfixed, T)) return OR_BAD_ARGUMENT;
    return evaluate_with(P, bins, T, want_derivative, nthreads, value, deriv, valid, status, fi_out, mi_out,
                         joint_out, fixed_marginal_out);
}

// The same metric at a point map of 1..8 stages with an affine-in-x Jacobian form
// (jac0: 3×nparams row-major; jacc: three such blocks).
int or_mattes_evaluate_stages(const float* fixed, const or_geometry* fg, const float* moving,
                              const or_geometry* mg, const uint8_t* fmask, const uint8_t* mmask,
                              const int64_t* draw, int64_t ndraw, int bins, const double* stages, int nstage,
                              const double* jac0, const double* jacc, int nparams, int nthreads, double* value,
                              double* deriv, int64_t* valid, int8_t* status, int32_t* fi_out, int32_t* mi_out) {
    if (nstage < 1 || nstage > 8 || nparams < 1 || nparams > 12) return OR_BAD_ARGUMENT;
    Problem P;
    int st = prepare(fixed, fg, moving, mg, fmask, mmask, draw, ndraw, P);
    if (st) return st;
    StageMap T;
    T.nstage = nstage;
    T.nparams = nparams;
    for (int k = 0; k < nstage; ++k)
        for (int i = 0; i < 12; ++i) T.st[k][i] = stages[k * 12 + i];
    for (int i = 0; i < 3 * nparams; ++i) {
        T.jac0[i] = jac0[i];
        for (int e = 0; e < 3; ++e) T.jacc[e][i] = jacc[e * 3 * nparams + i];
    }
    return evaluate_with(P, bins, T, 1, nthreads, value, deriv, valid, status, fi_out, mi_out, nullptr, nullptr);
}

// One level of registration with the reference's regular-step gradient descent
// (registration/optimizer.rs:352-440) as its driver runs it (method.rs:3140-3400):
// physical-shift scales over the fixed grid's corners (scales.rs:423-441, 668-722)
// and, when estimate_lr, the learning rate estimated once (scales.rs:779-824;
// method.rs EstimateLearningRate::Once). The objective is this file's metric.
// stop: 0 MaxIterations, 1 StepTooSmall, 3 GradientConverged.
int or_register(const float* fixed, const or_geometry* fg, const float* moving, const or_geometry* mg,
                const uint8_t* fmask, const uint8_t* mmask, const int64_t* draw, int64_t ndraw, int bins,
                int kind, double* params_inout, const double* fixed_params, int nfixed, int iterations,
                double minimum_step, double gradient_tolerance, double relaxation_factor, double learning_rate,
                int estimate_lr, int shift_scales, int nthreads, double* value_out, int* iterations_out,
                int* stop_out) {
    Problem P;
    int st = prepare(fixed, fg, moving, mg, fmask, mmask, draw, ndraw, P);
    if (st) return st;
    double fmin, fmax, mmin, mmax;
    ranges(P, &fmin, &fmax, &mmin, &mmax);
    Geometry G;
    st = make_geometry(fmin, fmax, mmin, mmax, bins, G);
    if (st) return st;
    Transform T0;
    if (!make_transform(kind, params_inout, fixed_params, nfixed, T0)) return OR_BAD_ARGUMENT;
    const int n = T0.nparams;
    if (nthreads < 1) nthreads = 1;
    std::vector<double> grad(n), scales(n, 1.0), scaled(n), prev(n, 0.0), p(params_inout, params_inout + n);
    double value = 0.0;
    auto eval = [&](const double* at) {
        Transform T;
        make_transform(kind, at, fixed_params, nfixed, T);
        std::vector<Accum> parts(nthreads);
        for (auto& a : parts) {
            a.joint.assign((size_t)bins * bins, 0.0);
            a.fixed_marginal.assign(bins, 0.0);
            a.jpd.assign((size_t)bins * bins * n, 0.0);
        }
        const int64_t ns = P.n;
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; ++t)
            pool.emplace_back([&, t]() {
                const int64_t lo = ns * t / nthreads, hi = ns * (t + 1) / nthreads;
                for (int64_t s = lo; s < hi; ++s) sample_body(P, G, T, s, true, parts[t], nullptr, nullptr, nullptr);
            });
        for (auto& th : pool) th.join();
        for (int t = 1; t < nthreads; ++t) {
            for (size_t i = 0; i < parts[0].joint.size(); ++i) parts[0].joint[i] += parts[t].joint[i];
            for (int i = 0; i < bins; ++i) parts[0].fixed_marginal[i] += parts[t].fixed_marginal[i];
            for (size_t i = 0; i < parts[0].jpd.size(); ++i) parts[0].jpd[i] += parts[t].jpd[i];
            parts[0].valid += parts[t].valid;
        }
        int64_t valid = 0;
        finish(G, parts[0], n, true, &value, grad.data(), &valid);
    };
    // the estimator's Jacobians at the initial transform, at the 8 grid corners
    std::vector<double> jac((size_t)8 * 3 * n);
    double i2p[9];
    index_to_physical(*fg, i2p);
    for (int corner = 0; corner < 8; ++corner) {
        double idx[3], x[3];
        for (int d = 0; d < 3; ++d) idx[d] = ((corner >> d) & 1) ? (double)(fg->size[d] - 1) : 0.0;
        for (int r = 0; r < 3; ++r) {
            double v = fg->origin[r];
            for (int c = 0; c < 3; ++c) v += i2p[r * 3 + c] * idx[c];
            x[r] = v;
        }
        T0.jacobian(x, jac.data() + (size_t)corner * 3 * n);
    }
    const double dsmall = 0.01;
    if (shift_scales) {
        std::vector<double> shifts(n, 0.0);
        for (int s = 0; s < 8; ++s)
            for (int k = 0; k < n; ++k) {
                double sq = 0.0;
                for (int r = 0; r < 3; ++r) {
                    double v = jac[(size_t)s * 3 * n + r * n + k];
                    sq += v * v;
                }
                shifts[k] = std::fmax(shifts[k], dsmall * std::sqrt(sq));
            }
        double mn = INFINITY;
        for (int k = 0; k < n; ++k)
            if (shifts[k] > DBL_EPSILON) mn = std::fmin(mn, shifts[k]);
        if (std::isfinite(mn)) {
            double inv_d2 = 1.0 / (dsmall * dsmall);
            for (int k = 0; k < n; ++k)
                scales[k] = (shifts[k] <= DBL_EPSILON ? mn * mn : shifts[k] * shifts[k]) * inv_d2;
        }
    }
    double max_step_size = INFINITY;
    for (int d = 0; d < 3; ++d) max_step_size = std::fmin(max_step_size, fg->spacing[d]);
    auto est_lr = [&](const double* step) {
        double max_step = 0.0;
        for (int k = 0; k < n; ++k) max_step = std::fmax(max_step, std::fabs(step[k]));
        if (max_step <= DBL_EPSILON) return 1.0;
        double factor = dsmall / max_step;
        double max_sq = 0.0;
        for (int s = 0; s < 8; ++s) {
            double sq = 0.0;
            for (int r = 0; r < 3; ++r) {
                double dot = -0.0;
                for (int c = 0; c < n; ++c) dot += jac[(size_t)s * 3 * n + r * n + c] * (step[c] * factor);
                sq += dot * dot;
            }
            max_sq = std::fmax(max_sq, sq);
        }
        double step_scale = std::sqrt(max_sq) / factor;
        return step_scale <= DBL_EPSILON ? 1.0 : max_step_size / step_scale;
    };
    eval(p.data());
    double lr = learning_rate;
    if (estimate_lr) {
        for (int k = 0; k < n; ++k) scaled[k] = grad[k] / scales[k];
        double sq = -0.0;
        for (int k = 0; k < n; ++k) sq += scaled[k] * scaled[k];
        lr = est_lr(scaled.data()) * std::sqrt(sq);
    }
    double relaxation = 1.0;
    int stop = 0, taken = 0;
    for (;;) {
        for (int k = 0; k < n; ++k) scaled[k] = grad[k] / scales[k];
        std::vector<double> sq(n);
        for (int k = 0; k < n; ++k) sq[k] = scaled[k] * scaled[k];
        const double gm = std::sqrt(kahan_sum(sq.data(), n));
        if (gm < gradient_tolerance) { stop = 3; break; }
        for (int k = 0; k < n; ++k) sq[k] = scaled[k] * prev[k];
        if (kahan_sum(sq.data(), n) < 0.0) relaxation *= relaxation_factor;
        const double step_length = relaxation * lr;
        if (step_length < minimum_step) { stop = 1; break; }
        if (taken >= iterations) break;
        const double factor = step_length / gm;
        for (int k = 0; k < n; ++k) p[k] -= factor * scaled[k];
        prev = scaled;
        ++taken;
        eval(p.data());
    }
    std::memcpy(params_inout, p.data(), sizeof(double) * n);
    *value_out = value;
    *iterations_out = taken;
    *stop_out = stop;
    return OR_OK;
}

// The transform's stored matrix/offset (one point-map stage) and its Jacobian at a
// point — exposed so tests can check the product's host-side transform code.
int or_transform(int kind, const double* params, const double* fixed_params, int nfixed,
                 const double* point, double* matrix9, double* offset3, double* jac,
                 double* mapped3) {
    Transform T;
    if (!make_transform(kind, params, fixed_params, nfixed, T)) return OR_BAD_ARGUMENT;
    if (matrix9) std::memcpy(matrix9, T.matrix, sizeof(T.matrix));
    if (offset3) std::memcpy(offset3, T.offset, sizeof(T.offset));
    if (point && jac) T.jacobian(point, jac);
    if (point && mapped3) T.transform_point(point, mapped3);
    return OR_OK;
}

int or_cubic_bspline(const double* u, double* val, double* dval, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        if (val) val[i] = cubic_bspline(u[i]);
        if (dval) dval[i] = cubic_bspline_derivative(u[i]);
    }
    return OR_OK;
}

double or_kahan_sum(const double* v, int64_t n) { return kahan_sum(v, (size_t)n); }

int64_t or_round_half_integer_up(double x) { return (int64_t)std::floor(x + 0.5); }

int or_invert3(const double* m, double* inv) { return invert3(m, inv) ? OR_OK : OR_SINGULAR_DIRECTION; }

}  // extern "C"

namespace {

// ---------------------------------------------------------------------------
// The cubic B-spline transform (transform/bspline.rs), 3-D, order 3.
// ---------------------------------------------------------------------------

// bspline.rs:94-106 (the deformation kernel; same basis as the Parzen window, its own
// expression order)
double bs_cubic(double u) {
    double a = std::fabs(u);
    if (a < 1.0) {
        double sq = a * a;
        return (4.0 - 6.0 * sq + 3.0 * sq * a) / 6.0;
    } else if (a < 2.0) {
        double sq = a * a;
        return (8.0 - 12.0 * a + 6.0 * sq - sq * a) / 6.0;
    }
    return 0.0;
}

struct BSpline {
    int64_t gsize[3];
    double gorigin[3], gspacing[3], gdir[9], p2i[9];
    int64_t gstride[3];
    int64_t nper = 0;
    const double* coef = nullptr;

    // set_fixed_parameters / from_grid_geometry (bspline.rs:275-321, :638-656):
    // [gridSize(3), gridOrigin(3), gridSpacing(3), gridDirection(9)]
    bool init(const double* fp, const double* c, int64_t ncoef) {
        for (int d = 0; d < 3; ++d) {
            gsize[d] = fp[d] >= 1.0 ? (int64_t)fp[d] : 0;
            if (gsize[d] == 0) return false;
            gorigin[d] = fp[3 + d];
            gspacing[d] = fp[6 + d];
        }
        for (int i = 0; i < 9; ++i) gdir[i] = fp[9 + i];
        double m[9];
        for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc) m[r * 3 + cc] = gdir[r * 3 + cc] * gspacing[cc];
        if (!invert3(m, p2i)) return false;
        gstride[0] = 1;
        gstride[1] = gsize[0];
        gstride[2] = gsize[0] * gsize[1];
        nper = gsize[0] * gsize[1] * gsize[2];
        if (ncoef != 3 * nper) return false;
        coef = c;
        return true;
    }

    // bspline.rs:488-499
    void continuous_index(const double* p, double* idx) const {
        for (int r = 0; r < 3; ++r) {
            double acc = -0.0;
            for (int cc = 0; cc < 3; ++cc) acc += p2i[r * 3 + cc] * (p[cc] - gorigin[cc]);
            idx[r] = acc;
        }
    }

    // bspline.rs:504-520 (the far limit snapped inward)
    bool inside_valid_region(double* idx) const {
        const double min_limit = 0.5 * (3.0 - 1.0);
        for (int d = 0; d < 3; ++d) {
            const double max_limit = (double)gsize[d] - 0.5 * (3.0 - 1.0) - 1.0;
            const double ulp = 4.0 * DBL_EPSILON * std::max(std::fabs(max_limit), 1.0);
            if (std::fabs(idx[d] - max_limit) <= ulp)
                idx[d] = max_limit - 6.0 * DBL_EPSILON * std::max(std::fabs(max_limit), 1.0);
            else if (idx[d] >= max_limit || idx[d] < min_limit)
                return false;
        }
        return true;
    }

    // bspline.rs:525-557: 64 weights, first axis fastest, and the support start
    void weights(const double* idx, double* w, int64_t* start) const {
        double w1[3][4];
        for (int d = 0; d < 3; ++d) {
            start[d] = (int64_t)std::floor(idx[d] + 0.5 - 3.0 / 2.0);
            double x = idx[d] - (double)start[d];
            for (int t = 0; t < 4; ++t) {
                w1[d][t] = bs_cubic(x);
                x -= 1.0;
            }
        }
        for (int k = 0; k < 64; ++k) {
            double prod = 1.0;
            int rem = k;
            for (int d = 0; d < 3; ++d) {
                prod *= w1[d][rem % 4];
                rem /= 4;
            }
            w[k] = prod;
        }
    }

    int64_t support_flat(const int64_t* start, int k) const {
        int rem = k;
        int64_t flat = 0;
        for (int d = 0; d < 3; ++d) {
            flat += (start[d] + rem % 4) * gstride[d];
            rem /= 4;
        }
        return flat;
    }

    // bspline.rs:561-585
    void transform_point(const double* x, double* y) const {
        double idx[3];
        continuous_index(x, idx);
        if (!inside_valid_region(idx)) {
            for (int d = 0; d < 3; ++d) y[d] = x[d];
            return;
        }
        double w[64];
        int64_t start[3];
        weights(idx, w, start);
        double disp[3] = {0.0, 0.0, 0.0};
        for (int k = 0; k < 64; ++k) {
            const int64_t flat = support_flat(start, k);
            for (int d = 0; d < 3; ++d) disp[d] += w[k] * coef[d * nper + flat];
        }
        for (int d = 0; d < 3; ++d) y[d] = x[d] + disp[d];
    }

    static constexpr int nparams = 0;  // the sparse path never asks for a dense Jacobian
    void jacobian(const double*, double*) const {}
};

// mattes_tail's pRatio table (mattes.rs:273-328) beside the value: pratio[f·B + m] =
// ln(jp/mm)·nFactor where both are above ε, else 0. Returns false when degenerate.
bool tail_with_pratio(const Geometry& G, Accum& A, double* value, std::vector<double>& pratio) {
    const int bins = G.bins;
    pratio.assign((size_t)bins * bins, 0.0);
    if (A.valid == 0) return false;
    double joint_sum = kahan_sum(A.joint.data(), A.joint.size());
    if (joint_sum < DBL_EPSILON) return false;
    double n_factor = 1.0 / (G.moving_bin_size * (double)A.valid);
    double inv_sum = 1.0 / joint_sum;
    for (auto& p : A.joint) p *= inv_sum;
    for (auto& p : A.fixed_marginal) p *= inv_sum;
    std::vector<double> mm(bins, 0.0);
    for (int f = 0; f < bins; ++f)
        for (int m = 0; m < bins; ++m) mm[m] += A.joint[(size_t)f * bins + m];
    double sum = 0.0;
    for (int f = 0; f < bins; ++f) {
        double fm = A.fixed_marginal[f];
        if (fm <= DBL_EPSILON) continue;
        double log_fm = std::log(fm);
        for (int m = 0; m < bins; ++m) {
            double mmv = mm[m], jp = A.joint[(size_t)f * bins + m];
            if (mmv > DBL_EPSILON && jp > DBL_EPSILON) {
                double pr = std::log(jp / mmv);
                sum += jp * (pr - log_fm);
                pratio[(size_t)f * bins + m] = pr * n_factor;
            }
        }
    }
    *value = -sum;
    return true;
}

}  // namespace

extern "C" {

// A point through the B-spline transform (bspline.rs:561-585); for tests.
int or_bspline_transform_point(const double* fixed18, const double* coef, int64_t ncoef, const double* x,
                               double* y) {
    BSpline T;
    if (!T.init(fixed18, coef, ncoef)) return OR_BAD_ARGUMENT;
    T.transform_point(x, y);
    return OR_OK;
}

// The Mattes metric through a B-spline transform: evaluate_sparse_support
// (mattes.rs:722-796). Pass 1 is build_histogram (the same per-sample body as the
// global-support path, through the B-spline point map); the value and pRatio come
// from mattes_tail; pass 2 re-walks the samples and, for every valid sample inside the
// transform's valid region, adds inner·acc to each of its 64·3 coefficients in
// support order (k, then d), with inner = weight·∇M[d] and acc = Σ_taps B₃′·pRatio.
// Per-sample status / bins as or_mattes_evaluate.
int or_bspline_mattes_evaluate(const float* fixed, const or_geometry* fg, const float* moving,
                               const or_geometry* mg, const uint8_t* fmask, const uint8_t* mmask,
                               const int64_t* draw, int64_t ndraw, int bins, const double* fixed18,
                               const double* coef, int64_t ncoef, int want_derivative, double* value,
                               double* deriv, int64_t* valid, int8_t* status, int32_t* fi_out, int32_t* mi_out) {
    Problem P;
    int st = prepare(fixed, fg, moving, mg, fmask, mmask, draw, ndraw, P);
    if (st) return st;
    double fmin, fmax, mmin, mmax;
    ranges(P, &fmin, &fmax, &mmin, &mmax);
    Geometry G;
    st = make_geometry(fmin, fmax, mmin, mmax, bins, G);
    if (st) return st;
    BSpline T;
    if (!T.init(fixed18, coef, ncoef)) return OR_BAD_ARGUMENT;
    Accum A;
    A.joint.assign((size_t)bins * bins, 0.0);
    A.fixed_marginal.assign(bins, 0.0);
    for (int64_t s = 0; s < P.n; ++s) sample_body(P, G, T, s, false, A, status, fi_out, mi_out);
    if (want_derivative)
        for (int64_t k = 0; k < ncoef; ++k) deriv[k] = 0.0;
    *valid = A.valid;
    std::vector<double> pratio;
    if (!tail_with_pratio(G, A, value, pratio)) {
        *value = DBL_MAX;
        return OR_OK;
    }
    if (!want_derivative) return OR_OK;
    for (int64_t s = 0; s < P.n; ++s) {
        const int64_t flat = sample_flat(P, s);
        double fp[3], mp[3], mv, g[3];
        grid_point(P, flat, fp);
        const double fv = (double)P.fixed[flat];
        T.transform_point(fp, mp);
        if (!moving_value_grad(P, mp, &mv, g, true)) continue;
        if (mv < G.moving_true_min || mv > G.moving_true_max) continue;
        double idx[3];
        T.continuous_index(fp, idx);
        if (!T.inside_valid_region(idx)) continue;  // empty sparse Jacobian
        double w[64];
        int64_t start[3];
        T.weights(idx, w, start);
        const double moving_term = mv / G.moving_bin_size - G.moving_normalized_min;
        const int mi = parzen_index(mv, G.moving_bin_size, G.moving_normalized_min, bins);
        const int fi = parzen_index(fv, G.fixed_bin_size, G.fixed_normalized_min, bins);
        for (int k = 0; k < 64; ++k) {
            const int64_t cp = T.support_flat(start, k);
            for (int d = 0; d < 3; ++d) {
                // inner = Σ_e col[e]·∇M[e] with col = w·e_d
                double inner = -0.0;
                for (int e = 0; e < 3; ++e) inner += (e == d ? w[k] : 0.0) * g[e];
                double acc = 0.0;
                for (int m = mi - 1; m < mi + 3; ++m) {
                    const double arg = (double)m - moving_term;
                    acc += cubic_bspline_derivative(arg) * pratio[(size_t)fi * bins + m];
                }
                deriv[d * T.nper + cp] += inner * acc;
            }
        }
    }
    return OR_OK;
}

// ---------------------------------------------------------------------------
// The shared-sampler siblings of the Mattes metric, over the same Problem (sample
// set, masks, moving image) and the same per-sample sampler (moving_value_grad).
// ---------------------------------------------------------------------------

// Mean squares: CpuBackend::mean_squares, dense branch (registration/metric.rs:1064-
// 1160), and mean_squares_value (:1162-1196) when want_derivative is 0. Per valid
// sample, in sample order: diff = mv − f; value_sum += diff²; for each parameter k,
// deriv[k] += 2·diff·(Σ_d ∇M[d]·J[d][k]) (the Σ from 0.0, d ascending). Then both
// are scaled by 1/valid; no valid sample gives f64::MAX and a zero derivative.
int or_ms_evaluate(const float* fixed, const or_geometry* fg, const float* moving, const or_geometry* mg,
                   const uint8_t* fmask, const uint8_t* mmask, const int64_t* draw, int64_t ndraw, int kind,
                   const double* params, const double* fixed_params, int nfixed, int want_derivative,
                   double* value, double* deriv, int64_t* valid) {
    Problem P;
    int st = prepare(fixed, fg, moving, mg, fmask, mmask, draw, ndraw, P);
    if (st) return st;
    Transform T;
    if (!make_transform(kind, params, fixed_params, nfixed, T)) return OR_BAD_ARGUMENT;
    const int np = T.nparams;
    const bool wd = want_derivative != 0;
    double value_sum = 0.0;
    std::vector<double> d(np, 0.0);
    int64_t nv = 0;
    double jac[36];
    for (int64_t s = 0; s < P.n; ++s) {
        const int64_t flat = sample_flat(P, s);
        double fp[3], mp[3], mv, g[3];
        grid_point(P, flat, fp);
        T.transform_point(fp, mp);
        if (!moving_value_grad(P, mp, &mv, g, wd)) continue;
        const double diff = mv - (double)P.fixed[flat];
        value_sum += diff * diff;
        if (wd) {
            T.jacobian(fp, jac);
            for (int k = 0; k < np; ++k) {
                double gk = 0.0;
                for (int q = 0; q < 3; ++q) gk += g[q] * jac[q * np + k];
                d[k] += 2.0 * diff * gk;
            }
        }
        nv += 1;
    }
    *valid = nv;
    if (nv == 0) {
        *value = DBL_MAX;
        if (wd) for (int k = 0; k < np; ++k) deriv[k] = 0.0;
        return OR_OK;
    }
    const double inv = 1.0 / (double)nv;
    if (wd) {
        *value = value_sum * inv;
        for (int k = 0; k < np; ++k) deriv[k] = d[k] * inv;
    } else {
        *value = value_sum / (double)nv;  // mean_squares_value divides
    }
    return OR_OK;
}

// Normalised cross-correlation: CorrelationMetric (registration/correlation.rs).
// Pass 1, means() (:260-295): Σf, Σm over the valid samples in sample order, each
// divided by the count. Pass 2, evaluate() (:297-410): f1 = f − f̄, m1 = m − m̄;
// fm += f1·m1, f2 += f1², m2 += m1², fdm[k] += f1·inner, mdm[k] += m1·inner with
// inner = Σ_d ∇M[d]·J[d][k]; value = −fm²/(m2·f2), derivative
// −2·fm/(f2·m2)·(fdm − fm/m2·mdm). value() (:200-257) is pass 2 without the
// derivative sums. No valid sample, or m2·f2 ≤ ε, gives f64::MAX and a zero
// derivative (valid = the count in the second case).
int or_ncc_evaluate(const float* fixed, const or_geometry* fg, const float* moving, const or_geometry* mg,
                    const uint8_t* fmask, const uint8_t* mmask, const int64_t* draw, int64_t ndraw, int kind,
                    const double* params, const double* fixed_params, int nfixed, int want_derivative,
                    double* value, double* deriv, int64_t* valid) {
    Problem P;
    int st = prepare(fixed, fg, moving, mg, fmask, mmask, draw, ndraw, P);
    if (st) return st;
    Transform T;
    if (!make_transform(kind, params, fixed_params, nfixed, T)) return OR_BAD_ARGUMENT;
    const int np = T.nparams;
    const bool wd = want_derivative != 0;
    if (wd) for (int k = 0; k < np; ++k) deriv[k] = 0.0;
    double fix_sum = 0.0, mov_sum = 0.0;
    int64_t n1 = 0;
    for (int64_t s = 0; s < P.n; ++s) {
        const int64_t flat = sample_flat(P, s);
        double fp[3], mp[3], mv, g[3];
        grid_point(P, flat, fp);
        T.transform_point(fp, mp);
        if (!moving_value_grad(P, mp, &mv, g, false)) continue;
        fix_sum += (double)P.fixed[flat];
        mov_sum += mv;
        n1 += 1;
    }
    if (n1 == 0) {
        *value = DBL_MAX;
        *valid = 0;
        return OR_OK;
    }
    const double avg_fix = fix_sum / (double)n1, avg_mov = mov_sum / (double)n1;
    double fm = 0.0, f2 = 0.0, m2 = 0.0;
    std::vector<double> fdm(np, 0.0), mdm(np, 0.0);
    int64_t nv = 0;
    double jac[36];
    for (int64_t s = 0; s < P.n; ++s) {
        const int64_t flat = sample_flat(P, s);
        double fp[3], mp[3], mv, g[3];
        grid_point(P, flat, fp);
        T.transform_point(fp, mp);
        if (!moving_value_grad(P, mp, &mv, g, wd)) continue;
        const double f1 = (double)P.fixed[flat] - avg_fix;
        const double m1 = mv - avg_mov;
        fm += f1 * m1;
        f2 += f1 * f1;
        m2 += m1 * m1;
        if (wd) {
            T.jacobian(fp, jac);
            for (int k = 0; k < np; ++k) {
                double inner = 0.0;
                for (int q = 0; q < 3; ++q) inner += g[q] * jac[q * np + k];
                fdm[k] += f1 * inner;
                mdm[k] += m1 * inner;
            }
        }
        nv += 1;
    }
    *valid = nv;
    const double m2f2 = m2 * f2;
    if (nv == 0 || m2f2 <= DBL_EPSILON) {
        *value = DBL_MAX;
        return OR_OK;
    }
    *value = -fm * fm / m2f2;
    if (wd)
        for (int k = 0; k < np; ++k) deriv[k] = -2.0 * fm / (f2 * m2) * (fdm[k] - fm / m2 * mdm[k]);
    return OR_OK;
}

}  // extern "C"
