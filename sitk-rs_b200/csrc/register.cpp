// The registration driver around the device metric: regular-step gradient descent
// with physical-shift scales and a once-estimated learning rate (the step logic is
// rsgd.h, shared with the batched device driver), and the centred transform
// initializer. Host C++, compiled with -ffp-contract=off; every objective evaluation
// is one mi_metric_value_and_derivative call.
//
//   driver wiring            registration/method.rs:3140-3400
//   centred initializer      registration/initializer.rs:56-105

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"
#include "rsgd.h"

namespace mi {

void index_to_physical(const mi_geometry& g, double* m);

// The transform's Jacobian at the fixed grid's 8 corner points (scales.rs:423-441
// picks corner sampling for the linear transforms; VirtualGrid::point is
// origin-seeded), and the smallest fixed spacing.
mi_status shift_corners(int kind, const double* params, int nparams, const double* fixed, int nfixed,
                        const mi_geometry& fg, rsgd::Corners& c) {
    c.P = nparams;
    double i2p[9];
    index_to_physical(fg, i2p);
    for (int corner = 0; corner < 8; ++corner) {
        double idx[3];
        for (int d = 0; d < 3; ++d) idx[d] = ((corner >> d) & 1) ? (double)(fg.size[d] - 1) : 0.0;
        double x[3];
        for (int r = 0; r < 3; ++r) {
            double v = fg.origin[r];
            for (int k = 0; k < 3; ++k) v += i2p[r * 3 + k] * idx[k];
            x[r] = v;
        }
        const mi_status s = transform_jacobian(kind, params, nparams, fixed, nfixed, x, c.jac + corner * 3 * nparams);
        if (s != MI_OK) return s;
    }
    c.max_step_size = INFINITY;
    for (int d = 0; d < 3; ++d) c.max_step_size = std::fmin(c.max_step_size, fg.spacing[d]);
    return MI_OK;
}

}  // namespace mi

extern "C" {

mi_status mi_register_rsgd(mi_metric* m, int kind, const double* fixed_params, int nfixed, const mi_rsgd_config* cfg,
                           double* params_inout, int nparams, mi_rsgd_result* out) {
    using namespace mi;
    if (!m || !cfg || !params_inout || !out || nparams < 1 || nparams > MI_MAX_PARAMS) return MI_ERR_INVALID_ARGUMENT;
    const int n = nparams;
    std::vector<double> p(params_inout, params_inout + n), grad(n), scales(n, 1.0);
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
    rsgd::Corners corners;
    mi_status s = shift_corners(kind, p.data(), n, fixed_params, nfixed, m->fgeo, corners);
    if (s != MI_OK) return s;
    if (cfg->physical_shift_scales) rsgd::shift_scales(corners, scales.data());
    rsgd::State state;
    rsgd::start(state, *cfg, n);
    for (;;) {
        s = eval(p.data());
        if (s != MI_OK) return s;
        if (rsgd::after_evaluation(state, *cfg, corners, scales.data(), grad.data(), p.data())) break;
    }
    std::memcpy(params_inout, p.data(), sizeof(double) * n);
    out->value = value;
    out->valid = valid;
    out->iterations = state.taken;
    out->stop_reason = state.stop;
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
