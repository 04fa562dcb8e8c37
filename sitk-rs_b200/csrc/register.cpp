// The registration driver around the device metric: regular-step gradient descent
// with physical-shift scales and a once-estimated learning rate, and the centred
// transform initializer. Host C++, compiled with -ffp-contract=off; every objective
// evaluation is one mi_metric_value_and_derivative call (two kernels on the device).
//
//   RSGD loop                registration/optimizer.rs:352-440
//   scales / learning rate   registration/scales.rs:572-871 (corner sampling for
//                            the linear families, scales.rs:423-441)
//   driver wiring            registration/method.rs:3140-3400 (EstimateLearningRate::Once:
//                            lr = estimate_learning_rate(g0/scales)·|g0/scales|)
//   centred initializer      registration/initializer.rs:56-105

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

namespace mi {
void index_to_physical(const mi_geometry& g, double* m);
}  // namespace mi

namespace {

constexpr double SMALL_PARAMETER_VARIATION = 0.01;  // scales.rs:137

// ITK's Kahan recurrence; the sum is returned without the final compensation
// (core/compensated.rs:112-123).
struct Kahan {
    double sum = 0.0, comp = 0.0;
    void add(double x) {
        const double ci = x - comp;
        const double t = sum + ci;
        comp = (t - sum) - ci;
        sum = t;
    }
};

// The physical-shift estimator over the fixed grid's 8 corner points (scales.rs:
// 423-441 picks corner sampling for linear transforms; VirtualGrid::point is
// origin-seeded).
struct ShiftEstimator {
    int P = 0;
    std::vector<double> jac;  // [8][3][P]
    double max_step_size = 1.0;

    mi_status init(int kind, const double* params, int nparams, const double* fixed, int nfixed,
                   const mi_geometry& fg) {
        P = nparams;
        double i2p[9];
        mi::index_to_physical(fg, i2p);
        jac.assign((size_t)8 * 3 * P, 0.0);
        for (int corner = 0; corner < 8; ++corner) {
            double idx[3];
            for (int d = 0; d < 3; ++d) idx[d] = ((corner >> d) & 1) ? (double)(fg.size[d] - 1) : 0.0;
            double x[3];
            for (int r = 0; r < 3; ++r) {
                double v = fg.origin[r];
                for (int c = 0; c < 3; ++c) v += i2p[r * 3 + c] * idx[c];
                x[r] = v;
            }
            const mi_status s = mi::transform_jacobian(kind, params, nparams, fixed, nfixed, x,
                                                       jac.data() + (size_t)corner * 3 * P);
            if (s != MI_OK) return s;
        }
        // FixedSamples::min_spacing: the smallest fixed spacing
        max_step_size = INFINITY;
        for (int d = 0; d < 3; ++d) max_step_size = std::fmin(max_step_size, fg.spacing[d]);
        return MI_OK;
    }

    // shift_scales (scales.rs:668-722)
    void scales(double* out) const {
        const double d = SMALL_PARAMETER_VARIATION, eps = DBL_EPSILON;
        std::vector<double> shifts(P, 0.0);
        for (int s = 0; s < 8; ++s) {
            const double* j = jac.data() + (size_t)s * 3 * P;
            for (int p = 0; p < P; ++p) {
                double sq = 0.0;
                for (int r = 0; r < 3; ++r) {
                    const double v = j[r * P + p];
                    sq += v * v;
                }
                shifts[p] = std::fmax(shifts[p], d * std::sqrt(sq));
            }
        }
        double min_nonzero = INFINITY;
        for (int p = 0; p < P; ++p)
            if (shifts[p] > eps) min_nonzero = std::fmin(min_nonzero, shifts[p]);
        if (!std::isfinite(min_nonzero)) {
            for (int p = 0; p < P; ++p) out[p] = 1.0;
            return;
        }
        const double inv_d2 = 1.0 / (d * d);
        for (int p = 0; p < P; ++p) {
            const double base = shifts[p] <= eps ? min_nonzero * min_nonzero : shifts[p] * shifts[p];
            out[p] = base * inv_d2;
        }
    }

    // max over the corners of |J·delta| (scales.rs:795-815, squared_shift :516-527)
    double max_shift(const double* delta) const {
        double max_sq = 0.0;
        for (int s = 0; s < 8; ++s) {
            const double* j = jac.data() + (size_t)s * 3 * P;
            double sq = 0.0;
            for (int r = 0; r < 3; ++r) {
                double dot = -0.0;
                for (int c = 0; c < P; ++c) dot += j[r * P + c] * delta[c];
                sq += dot * dot;
            }
            max_sq = std::fmax(max_sq, sq);
        }
        return std::sqrt(max_sq);
    }

    // shift_step_scale (scales.rs:779-793) and estimate_learning_rate (:817-824)
    double learning_rate(const double* step) const {
        double max_step = 0.0;
        for (int p = 0; p < P; ++p) max_step = std::fmax(max_step, std::fabs(step[p]));
        double step_scale = 0.0;
        if (max_step > DBL_EPSILON) {
            const double factor = SMALL_PARAMETER_VARIATION / max_step;
            std::vector<double> small(P);
            for (int p = 0; p < P; ++p) small[p] = step[p] * factor;
            step_scale = max_shift(small.data()) / factor;
        }
        return step_scale <= DBL_EPSILON ? 1.0 : max_step_size / step_scale;
    }
};

}  // namespace

extern "C" {

mi_status mi_register_rsgd(mi_metric* m, int kind, const double* fixed_params, int nfixed, const mi_rsgd_config* cfg,
                           double* params_inout, int nparams, mi_rsgd_result* out) {
    if (!m || !cfg || !params_inout || !out || nparams < 1 || nparams > MI_MAX_PARAMS) return MI_ERR_INVALID_ARGUMENT;
    const int n = nparams;
    std::vector<double> p(params_inout, params_inout + n), grad(n), scales(n, 1.0), scaled(n), prev(n, 0.0);
    int evaluations = 0;
    double value = 0.0;
    int64_t valid = 0;
    auto eval = [&](const double* at) -> mi_status {
        const mi_status st =
            mi_metric_value_and_derivative(m, kind, at, n, fixed_params, nfixed, &value, grad.data(), &valid);
        if (st == MI_OK && cfg->trace && evaluations < cfg->trace_rows) {
            double* row = cfg->trace + (size_t)evaluations * (1 + 2 * n);
            row[0] = value;
            std::memcpy(row + 1, at, sizeof(double) * n);
            std::memcpy(row + 1 + n, grad.data(), sizeof(double) * n);
        }
        ++evaluations;
        return st;
    };
    ShiftEstimator est;
    const bool need_est = cfg->physical_shift_scales || cfg->estimate_learning_rate;
    if (need_est) {
        const mi_status s = est.init(kind, p.data(), n, fixed_params, nfixed, m->fgeo);
        if (s != MI_OK) return s;
    }
    if (cfg->physical_shift_scales) est.scales(scales.data());

    mi_status s = eval(p.data());
    if (s != MI_OK) return s;
    double lr = cfg->learning_rate;
    if (cfg->estimate_learning_rate) {
        // method.rs: EstimateLearningRate::Once — lr = est(g0/scales)·|g0/scales|
        for (int k = 0; k < n; ++k) scaled[k] = grad[k] / scales[k];
        double sq = 0.0;
        for (int k = 0; k < n; ++k) sq += scaled[k] * scaled[k];
        lr = est.learning_rate(scaled.data()) * std::sqrt(sq);
    }

    double relaxation = 1.0;
    int stop = MI_STOP_MAX_ITERATIONS;
    int taken = 0;
    for (;;) {
        for (int k = 0; k < n; ++k) scaled[k] = grad[k] / scales[k];
        Kahan mag;
        for (int k = 0; k < n; ++k) mag.add(scaled[k] * scaled[k]);
        const double gradient_magnitude = std::sqrt(mag.sum);
        if (gradient_magnitude < cfg->gradient_tolerance) {
            stop = MI_STOP_GRADIENT_CONVERGED;
            break;
        }
        Kahan dot;
        for (int k = 0; k < n; ++k) dot.add(scaled[k] * prev[k]);
        if (dot.sum < 0.0) relaxation *= cfg->relaxation;
        const double step_length = relaxation * lr;
        if (step_length < cfg->minimum_step) {
            stop = MI_STOP_STEP_TOO_SMALL;
            break;
        }
        if (taken >= cfg->iterations) break;
        const double factor = step_length / gradient_magnitude;
        for (int k = 0; k < n; ++k) p[k] -= factor * scaled[k];
        prev = scaled;
        ++taken;
        s = eval(p.data());
        if (s != MI_OK) return s;
    }
    std::memcpy(params_inout, p.data(), sizeof(double) * n);
    out->value = value;
    out->valid = valid;
    out->iterations = taken;
    out->stop_reason = stop;
    out->evaluations = evaluations;
    return MI_OK;
}

mi_status mi_centered_initialize(const mi_geometry* fixed, const mi_geometry* moving, double* center3,
                                 double* translation3) {
    if (!fixed || !moving || !center3 || !translation3) return MI_ERR_INVALID_ARGUMENT;
    // geometric_center: continuous_index_to_physical_point((size − 1)/2), the origin
    // added last (core/coord.rs continuous_index_to_physical_point)
    auto centre = [](const mi_geometry& g, double* out) {
        double m[9];
        mi::index_to_physical(g, m);
        double idx[3];
        for (int d = 0; d < 3; ++d) idx[d] = ((double)g.size[d] - 1.0) / 2.0;
        for (int r = 0; r < 3; ++r) {
            double acc = 0.0;
            for (int c = 0; c < 3; ++c) acc += m[r * 3 + c] * idx[c];
            out[r] = acc + g.origin[r];
        }
    };
    double fc[3], mc[3];
    centre(*fixed, fc);
    centre(*moving, mc);
    for (int d = 0; d < 3; ++d) {
        center3[d] = fc[d];
        translation3[d] = mc[d] - fc[d];
    }
    return MI_OK;
}

}  // extern "C"
