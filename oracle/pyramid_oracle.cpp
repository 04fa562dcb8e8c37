// CPU ORACLE — test infrastructure only (see mattes_oracle.cpp for the status of
// the oracle as a whole). Serial FP64 restatement of one multi-resolution pyramid
// level of the reference (crate `sitk`, paths inside crates/sitk/src/):
//
//   recursive Gaussian   filters/recursive_gaussian.rs:81-290, :472-529;
//                        coefficients core/deriche.rs (zero order)
//   shrink geometry      filters/shrink.rs:51-95
//   linear resample      transform/resample.rs:226-290, transform/interpolator.rs:27-88
//
// Compiled with -ffp-contract=off: every a*b+c is two roundings, as in Rust.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

extern "C" {
typedef struct {
    int64_t size[3];
    double spacing[3];
    double origin[3];
    double direction[9];
} or_pgeometry;  // same layout as or_geometry in mattes_oracle.cpp
}

namespace {

struct Coeff {
    double n0, n1, n2, n3, d1, d2, d3, d4, m1, m2, m3, m4, bn1, bn2, bn3, bn4, bm1, bm2, bm3, bm4;
};

// core/deriche.rs: compute_d_coefficients, compute_n_coefficients with the
// zero-order column, then the zero-order normalisation (unit DC gain) and the
// symmetric anti-causal / boundary coefficients.
Coeff zero_order(double sigmad) {
    const double pw1 = 0.6681, pl1 = -1.3932, pw2 = 2.0787, pl2 = -1.3732;
    const double ca1 = 1.3530, cb1 = 1.8151, ca2 = -0.3531, cb2 = 0.0902;
    double cos1 = std::cos(pw1 / sigmad);
    double cos2 = std::cos(pw2 / sigmad);
    double exp1 = std::exp(pl1 / sigmad);
    double exp2 = std::exp(pl2 / sigmad);
    double d4 = exp1 * exp1 * exp2 * exp2;
    double d3 = -2.0 * cos1 * exp1 * exp2 * exp2 - 2.0 * cos2 * exp2 * exp1 * exp1;
    double d2 = 4.0 * cos2 * cos1 * exp1 * exp2 + exp1 * exp1 + exp2 * exp2;
    double d1 = -2.0 * (exp2 * cos2 + exp1 * cos1);
    double sd = 1.0 + d1 + d2 + d3 + d4;
    double sin1 = std::sin(pw1 / sigmad);
    double sin2 = std::sin(pw2 / sigmad);
    double n0 = ca1 + ca2;
    double n1 = exp2 * (cb2 * sin2 - (ca2 + 2.0 * ca1) * cos2) + exp1 * (cb1 * sin1 - (ca1 + 2.0 * ca2) * cos1);
    double n2 = ((ca1 + ca2) * cos2 * cos1 - cb1 * cos2 * sin1 - cb2 * cos1 * sin2) * 2.0 * exp1 * exp2 +
                ca2 * exp1 * exp1 + ca1 * exp2 * exp2;
    double n3 = exp2 * exp1 * exp1 * (cb2 * sin2 - ca2 * cos2) + exp1 * exp2 * exp2 * (cb1 * sin1 - ca1 * cos1);
    double sn_raw = n0 + n1 + n2 + n3;
    double alpha0 = 2.0 * sn_raw / sd - n0;
    Coeff c;
    c.n0 = n0 / alpha0;
    c.n1 = n1 / alpha0;
    c.n2 = n2 / alpha0;
    c.n3 = n3 / alpha0;
    c.d1 = d1;
    c.d2 = d2;
    c.d3 = d3;
    c.d4 = d4;
    c.m1 = c.n1 - d1 * c.n0;
    c.m2 = c.n2 - d2 * c.n0;
    c.m3 = c.n3 - d3 * c.n0;
    c.m4 = -d4 * c.n0;
    double sn = c.n0 + c.n1 + c.n2 + c.n3;
    double sm = c.m1 + c.m2 + c.m3 + c.m4;
    c.bn1 = d1 * sn / sd;
    c.bn2 = d2 * sn / sd;
    c.bn3 = d3 * sn / sd;
    c.bn4 = d4 * sn / sd;
    c.bm1 = d1 * sm / sd;
    c.bm2 = d2 * sm / sd;
    c.bm3 = d3 * sm / sd;
    c.bm4 = d4 * sm / sd;
    return c;
}

// recursive_gaussian.rs:472-529 (ITK FilterDataArray), literally: the causal pass
// into outs, the anti-causal pass into scratch, then outs[i] += scratch[i].
void filter_line(const std::vector<double>& data, const Coeff& c, std::vector<double>& outs,
                 std::vector<double>& scratch) {
    const size_t ln = data.size();
    double out_v1 = data[0];
    outs[0] = out_v1 * c.n0 + out_v1 * c.n1 + out_v1 * c.n2 + out_v1 * c.n3;
    outs[1] = data[1] * c.n0 + out_v1 * c.n1 + out_v1 * c.n2 + out_v1 * c.n3;
    outs[2] = data[2] * c.n0 + data[1] * c.n1 + out_v1 * c.n2 + out_v1 * c.n3;
    outs[3] = data[3] * c.n0 + data[2] * c.n1 + data[1] * c.n2 + out_v1 * c.n3;
    outs[0] -= out_v1 * c.bn1 + out_v1 * c.bn2 + out_v1 * c.bn3 + out_v1 * c.bn4;
    outs[1] -= outs[0] * c.d1 + out_v1 * c.bn2 + out_v1 * c.bn3 + out_v1 * c.bn4;
    outs[2] -= outs[1] * c.d1 + outs[0] * c.d2 + out_v1 * c.bn3 + out_v1 * c.bn4;
    outs[3] -= outs[2] * c.d1 + outs[1] * c.d2 + outs[0] * c.d3 + out_v1 * c.bn4;
    for (size_t i = 4; i < ln; ++i) {
        outs[i] = data[i] * c.n0 + data[i - 1] * c.n1 + data[i - 2] * c.n2 + data[i - 3] * c.n3;
        outs[i] -= outs[i - 1] * c.d1 + outs[i - 2] * c.d2 + outs[i - 3] * c.d3 + outs[i - 4] * c.d4;
    }
    double out_v2 = data[ln - 1];
    scratch[ln - 1] = out_v2 * c.m1 + out_v2 * c.m2 + out_v2 * c.m3 + out_v2 * c.m4;
    scratch[ln - 2] = data[ln - 1] * c.m1 + out_v2 * c.m2 + out_v2 * c.m3 + out_v2 * c.m4;
    scratch[ln - 3] = data[ln - 2] * c.m1 + data[ln - 1] * c.m2 + out_v2 * c.m3 + out_v2 * c.m4;
    scratch[ln - 4] = data[ln - 3] * c.m1 + data[ln - 2] * c.m2 + data[ln - 1] * c.m3 + out_v2 * c.m4;
    scratch[ln - 1] -= out_v2 * c.bm1 + out_v2 * c.bm2 + out_v2 * c.bm3 + out_v2 * c.bm4;
    scratch[ln - 2] -= scratch[ln - 1] * c.d1 + out_v2 * c.bm2 + out_v2 * c.bm3 + out_v2 * c.bm4;
    scratch[ln - 3] -= scratch[ln - 2] * c.d1 + scratch[ln - 1] * c.d2 + out_v2 * c.bm3 + out_v2 * c.bm4;
    scratch[ln - 4] -=
        scratch[ln - 3] * c.d1 + scratch[ln - 2] * c.d2 + scratch[ln - 1] * c.d3 + out_v2 * c.bm4;
    for (size_t i = ln - 4; i > 0; --i) {
        scratch[i - 1] = data[i] * c.m1 + data[i + 1] * c.m2 + data[i + 2] * c.m3 + data[i + 3] * c.m4;
        scratch[i - 1] -= scratch[i] * c.d1 + scratch[i + 1] * c.d2 + scratch[i + 2] * c.d3 + scratch[i + 3] * c.d4;
    }
    for (size_t i = 0; i < ln; ++i) outs[i] += scratch[i];
}

}  // namespace

extern "C" {

// recursive_gaussian (zero order, normalize_across_scale = false) of an f32 volume;
// sigma3 physical. Returns 0, or 5 (bad argument) for an axis shorter than 4 with
// sigma > 0.
int or_recursive_gaussian(const float* in, const or_pgeometry* g, const double* sigma3, float* out) {
    const int64_t n = g->size[0] * g->size[1] * g->size[2];
    std::vector<double> buf(in, in + n);
    const int64_t stride[3] = {1, g->size[0], g->size[0] * g->size[1]};
    for (int d = 0; d < 3; ++d) {
        if (sigma3[d] <= 0.0) continue;
        if (g->size[d] < 4) return 5;
        const Coeff c = zero_order(sigma3[d] / g->spacing[d]);
        const int64_t ln = g->size[d];
        std::vector<double> line(ln), outs(ln), scratch(ln);
        // every line along axis d: start voxels are those with coordinate d = 0
        for (int64_t s = 0; s < n; ++s) {
            if ((s / stride[d]) % g->size[d] != 0) continue;
            for (int64_t k = 0; k < ln; ++k) line[k] = buf[s + k * stride[d]];
            filter_line(line, c, outs, scratch);
            for (int64_t k = 0; k < ln; ++k) buf[s + k * stride[d]] = outs[k];
        }
    }
    for (int64_t i = 0; i < n; ++i) out[i] = (float)buf[i];
    return 0;
}

// shrink.rs:51-95 — the output grid only.
int or_shrink_geometry(const or_pgeometry* in, const int64_t* factors, or_pgeometry* out) {
    *out = *in;
    double delta[3];
    for (int d = 0; d < 3; ++d) {
        const int64_t f = factors[d];
        if (f <= 0) return 5;
        out->size[d] = std::max<int64_t>(in->size[d] / f, 1);
        out->spacing[d] = in->spacing[d] * (double)f;
        delta[d] = ((double)in->size[d] - 1.0) / 2.0 - (double)f * ((double)out->size[d] - 1.0) / 2.0;
    }
    for (int i = 0; i < 3; ++i) {
        double acc = 0.0;
        for (int j = 0; j < 3; ++j) acc += in->direction[i * 3 + j] * in->spacing[j] * delta[j];
        out->origin[i] = in->origin[i] + acc;
    }
    return 0;
}

int or_invert3(const double* m, double* inv);  // mattes_oracle.cpp (core/matrix.rs Gauss–Jordan)

// ResampleImageFilter::execute through the identity, linear interpolator.
static int resample(const float* in, const or_pgeometry* gin, const or_pgeometry* gout, double fill, bool linear,
                    float* out);

// ResampleImageFilter through the identity with the linear interpolator
// (transform/resample.rs:226-290, transform/interpolator.rs:103-152).
int or_resample_linear(const float* in, const or_pgeometry* gin, const or_pgeometry* gout, double fill,
                       float* out) {
    return resample(in, gin, gout, fill, true, out);
}

// The same with the nearest-neighbour interpolator (interpolator.rs:36-54): inside
// test, then floor(c + 0.5) per axis clamped to the grid; the level mask of the
// device driver (registration/method.rs:3068-3110 level_mask_on_device).
int or_resample_nearest(const float* in, const or_pgeometry* gin, const or_pgeometry* gout, double fill,
                        float* out) {
    return resample(in, gin, gout, fill, false, out);
}

static int resample(const float* in, const or_pgeometry* gin, const or_pgeometry* gout, double fill, bool linear,
                    float* out) {
    double m_in[9], inv[9], m_out[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            m_in[r * 3 + c] = gin->direction[r * 3 + c] * gin->spacing[c];
            m_out[r * 3 + c] = gout->direction[r * 3 + c] * gout->spacing[c];
        }
    if (or_invert3(m_in, inv) != 0) return 4;
    const int64_t on = gout->size[0] * gout->size[1] * gout->size[2];
    const int64_t istr[3] = {1, gin->size[0], gin->size[0] * gin->size[1]};
    for (int64_t q = 0; q < on; ++q) {
        const double idx[3] = {(double)(q % gout->size[0]), (double)((q / gout->size[0]) % gout->size[1]),
                               (double)(q / (gout->size[0] * gout->size[1]))};
        double phys[3];
        for (int r = 0; r < 3; ++r) {
            double acc = gout->origin[r];  // index_to_physical_point_f64: origin first
            for (int c = 0; c < 3; ++c) acc += m_out[r * 3 + c] * idx[c];
            phys[r] = acc;
        }
        // identity AffineTransform: M·p + offset, M = I, offset = 0
        double mapped[3];
        for (int r = 0; r < 3; ++r) {
            double acc = 0.0;
            for (int c = 0; c < 3; ++c) acc += (r == c ? 1.0 : 0.0) * phys[c];
            mapped[r] = acc + 0.0;
        }
        double diff[3], ci[3];
        for (int d = 0; d < 3; ++d) diff[d] = mapped[d] - gin->origin[d];
        for (int r = 0; r < 3; ++r) {
            double acc = 0.0;
            for (int c = 0; c < 3; ++c) acc += inv[r * 3 + c] * diff[c];
            ci[r] = acc;
        }
        bool inside = true;
        for (int d = 0; d < 3; ++d) inside = inside && ci[d] >= -0.5 && ci[d] < (double)gin->size[d] - 0.5;
        double v = fill;
        if (inside && !linear) {
            int64_t off = 0;
            for (int d = 0; d < 3; ++d) {
                int64_t i = (int64_t)std::floor(ci[d] + 0.5);
                i = std::min<int64_t>(std::max<int64_t>(i, 0), gin->size[d] - 1);
                off += i * istr[d];
            }
            v = (double)in[off];
        } else if (inside) {
            int64_t base[3];
            double frac[3];
            for (int d = 0; d < 3; ++d) {
                double f = std::floor(ci[d]);
                base[d] = (int64_t)f;
                frac[d] = ci[d] - f;
            }
            double acc = 0.0;
            for (int corner = 0; corner < 8; ++corner) {
                double w = 1.0;
                int64_t off = 0;
                for (int d = 0; d < 3; ++d) {
                    int bit = (corner >> d) & 1;
                    w *= bit ? frac[d] : 1.0 - frac[d];
                    int64_t k = std::min<int64_t>(std::max<int64_t>(base[d] + bit, 0), gin->size[d] - 1);
                    off += k * istr[d];
                }
                if (w != 0.0) acc += w * (double)in[off];
            }
            v = acc;
        }
        out[q] = (float)v;
    }
    return 0;
}

}  // extern "C"
