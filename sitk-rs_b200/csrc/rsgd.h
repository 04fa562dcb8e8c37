// Regular-step gradient descent with physical-shift scales and an estimated learning
// rate, written once for the host driver (register.cpp) and the batched device
// driver (batch.cu), so the two take the same steps bit for bit.
//
//   RSGD loop                registration/optimizer.rs:352-440
//   scales / learning rate   registration/scales.rs:572-871 (corner sampling for the
//                            linear families, scales.rs:423-441)
//   driver wiring            registration/method.rs:3140-3400 (EstimateLearningRate::Once:
//                            lr = estimate_learning_rate(g0/scales)·|g0/scales|)
//
// Every FP64 operation is separately rounded: plain operators on the host (compiled
// with -ffp-contract=off), __dmul_rn-style intrinsics on the device.
#pragma once

#include <cfloat>
#include <cmath>

#include "mi_b200.h"

#if defined(__CUDACC__)
#define MI_HD __host__ __device__
#else
#define MI_HD
#endif

namespace mi {
namespace rsgd {

MI_HD inline double mul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
MI_HD inline double add(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
MI_HD inline double sub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
MI_HD inline double div(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
MI_HD inline double root(double a) {
#if defined(__CUDA_ARCH__)
    return __dsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
}

constexpr double SMALL_PARAMETER_VARIATION = 0.01;  // scales.rs:137

// ITK's Kahan recurrence; the sum is returned without the final compensation
// (core/compensated.rs:112-123).
struct Kahan {
    double sum = 0.0, comp = 0.0;
    MI_HD void put(double x) {
        const double ci = sub(x, comp);
        const double t = add(sum, ci);
        comp = sub(sub(t, sum), ci);
        sum = t;
    }
};

// The transform's Jacobian at the fixed grid's 8 corner points ([8][3][P]), the
// physical-shift estimator's whole input for the linear families.
struct Corners {
    int P;
    double max_step_size;  // the smallest fixed spacing (FixedSamples::min_spacing)
    double jac[8 * 3 * MI_MAX_PARAMS];
};

// shift_scales (scales.rs:668-722)
MI_HD inline void shift_scales(const Corners& c, double* out) {
    const int P = c.P;
    const double d = SMALL_PARAMETER_VARIATION, eps = DBL_EPSILON;
    double shifts[MI_MAX_PARAMS];
    for (int p = 0; p < P; ++p) shifts[p] = 0.0;
    for (int s = 0; s < 8; ++s) {
        const double* j = c.jac + s * 3 * P;
        for (int p = 0; p < P; ++p) {
            double sq = 0.0;
            for (int r = 0; r < 3; ++r) sq = add(sq, mul(j[r * P + p], j[r * P + p]));
            shifts[p] = fmax(shifts[p], mul(d, root(sq)));
        }
    }
    double min_nonzero = INFINITY;
    for (int p = 0; p < P; ++p)
        if (shifts[p] > eps) min_nonzero = fmin(min_nonzero, shifts[p]);
    if (!(min_nonzero < INFINITY)) {
        for (int p = 0; p < P; ++p) out[p] = 1.0;
        return;
    }
    const double inv_d2 = div(1.0, mul(d, d));
    for (int p = 0; p < P; ++p) {
        const double base = shifts[p] <= eps ? mul(min_nonzero, min_nonzero) : mul(shifts[p], shifts[p]);
        out[p] = mul(base, inv_d2);
    }
}

// max over the corners of |J·delta| (scales.rs:795-815, squared_shift :516-527)
MI_HD inline double max_shift(const Corners& c, const double* delta) {
    const int P = c.P;
    double max_sq = 0.0;
    for (int s = 0; s < 8; ++s) {
        const double* j = c.jac + s * 3 * P;
        double sq = 0.0;
        for (int r = 0; r < 3; ++r) {
            double dot = -0.0;
            for (int k = 0; k < P; ++k) dot = add(dot, mul(j[r * P + k], delta[k]));
            sq = add(sq, mul(dot, dot));
        }
        max_sq = fmax(max_sq, sq);
    }
    return root(max_sq);
}

// shift_step_scale (scales.rs:779-793) and estimate_learning_rate (:817-824)
MI_HD inline double learning_rate(const Corners& c, const double* step) {
    const int P = c.P;
    double max_step = 0.0;
    for (int p = 0; p < P; ++p) max_step = fmax(max_step, fabs(step[p]));
    double step_scale = 0.0;
    if (max_step > DBL_EPSILON) {
        const double factor = div(SMALL_PARAMETER_VARIATION, max_step);
        double small[MI_MAX_PARAMS];
        for (int p = 0; p < P; ++p) small[p] = mul(step[p], factor);
        step_scale = div(max_shift(c, small), factor);
    }
    return step_scale <= DBL_EPSILON ? 1.0 : div(c.max_step_size, step_scale);
}

// The optimizer between two evaluations.
struct State {
    double prev[MI_MAX_PARAMS];  // the previous scaled gradient (ITK seeds it with zeros)
    double relaxation;
    double lr;
    int taken;      // steps taken
    int stop;       // mi_stop_reason once stopped
    int lr_pending; // the learning rate is still to be estimated from the first gradient
};

MI_HD inline void start(State& s, const mi_rsgd_config& cfg, int P) {
    for (int k = 0; k < P; ++k) s.prev[k] = 0.0;
    s.relaxation = 1.0;
    s.lr = cfg.learning_rate;
    s.taken = 0;
    s.stop = -1;
    s.lr_pending = cfg.estimate_learning_rate ? 1 : 0;
}

// One decision after an evaluation (optimizer.rs:383-440): with the derivative at p,
// either stop (returns true, s.stop set) or step p in place (returns false).
MI_HD inline bool after_evaluation(State& s, const mi_rsgd_config& cfg, const Corners& c, const double* scales,
                                   const double* grad, double* p) {
    const int n = c.P;
    double scaled[MI_MAX_PARAMS];
    for (int k = 0; k < n; ++k) scaled[k] = div(grad[k], scales[k]);
    if (s.lr_pending) {
        // method.rs: EstimateLearningRate::Once — lr = est(g0/scales)·|g0/scales|
        double sq = 0.0;
        for (int k = 0; k < n; ++k) sq = add(sq, mul(scaled[k], scaled[k]));
        s.lr = mul(learning_rate(c, scaled), root(sq));
        s.lr_pending = 0;
    }
    Kahan mag;
    for (int k = 0; k < n; ++k) mag.put(mul(scaled[k], scaled[k]));
    const double gradient_magnitude = root(mag.sum);
    if (gradient_magnitude < cfg.gradient_tolerance) {
        s.stop = MI_STOP_GRADIENT_CONVERGED;
        return true;
    }
    Kahan dot;
    for (int k = 0; k < n; ++k) dot.put(mul(scaled[k], s.prev[k]));
    if (dot.sum < 0.0) s.relaxation = mul(s.relaxation, cfg.relaxation);
    const double step_length = mul(s.relaxation, s.lr);
    if (step_length < cfg.minimum_step) {
        s.stop = MI_STOP_STEP_TOO_SMALL;
        return true;
    }
    if (s.taken >= cfg.iterations) {
        s.stop = MI_STOP_MAX_ITERATIONS;
        return true;
    }
    const double factor = div(step_length, gradient_magnitude);
    for (int k = 0; k < n; ++k) p[k] = sub(p[k], mul(factor, scaled[k]));
    for (int k = 0; k < n; ++k) s.prev[k] = scaled[k];
    s.taken += 1;
    return false;
}

}  // namespace rsgd
}  // namespace mi
