// Host-side transform families: parameters → the point-map stage the device replays,
// and the Jacobian's affine form J(x) = J(0) + Σ_e x_e·C_e.
//
// The stage is the matrix and offset each family stores and multiplies in its own
// transform_point (transform/parametric.rs:549-553, :1103-1107, :1331-1335), computed
// in the same operation order, so the device's continuous index is the host's to the
// bit (matrix_offset.rs:1-60 explains why the stored fields, not a probe, are used).
// This file is compiled with -ffp-contract=off: the reference never fuses.
//
// The Jacobian form replaces the reference's probed affine_form
// (registration/cuda.rs:294-363): each family's analytic Jacobian is linear in
// p = x − center, so C_e is read off at p = e_e and J(0) at p = −center.

#include <cmath>
#include <cstring>

#include "internal.h"

namespace {

void mat_vec3(const double* m, const double* v, double* out) {
    for (int r = 0; r < 3; ++r) {
        double acc = 0.0;
        for (int c = 0; c < 3; ++c) acc += m[r * 3 + c] * v[c];
        out[r] = acc;
    }
}

// Zero entries of the left factor are skipped, as core/matrix.rs:24-40 does; the
// skipped terms are exact zeros, so this only matters for the sign of zero.
void mat_mul3(const double* a, const double* b, double* out) {
    for (int i = 0; i < 9; ++i) out[i] = 0.0;
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
            const double ark = a[r * 3 + k];
            if (ark == 0.0) continue;
            for (int c = 0; c < 3; ++c) out[r * 3 + c] += ark * b[k * 3 + c];
        }
}

struct Family {
    int kind;
    int P;
    double m[9], off[3], center[3];
    double ang[3];
    bool zyx = false;
    double vx = 0, vy = 0, vz = 0, vw = 1;

    // Jacobian at p = x − center, row-major 3×P (parametric.rs:589-602, :1125-1166,
    // :1355-1384).
    void jac_centered(double px, double py, double pz, double* j) const {
        for (int i = 0; i < 3 * P; ++i) j[i] = 0.0;
        if (kind == MI_TRANSFORM_AFFINE) {
            const double p[3] = {px, py, pz};
            for (int i = 0; i < 3; ++i) {
                for (int c = 0; c < 3; ++c) j[i * P + i * 3 + c] = p[c];
                j[i * P + 9 + i] = 1.0;
            }
            return;
        }
        if (kind == MI_TRANSFORM_TRANSLATION) {
            for (int i = 0; i < 3; ++i) j[i * P + i] = 1.0;
            return;
        }
        if (kind == MI_TRANSFORM_EULER3D) {
            const double cx = std::cos(ang[0]), sx = std::sin(ang[0]);
            const double cy = std::cos(ang[1]), sy = std::sin(ang[1]);
            const double cz = std::cos(ang[2]), sz = std::sin(ang[2]);
            if (zyx) {
                j[0] = (cz * sy * cx + sz * sx) * py + (-cz * sy * sx + sz * cx) * pz;
                j[6] = (sz * sy * cx - cz * sx) * py + (-sz * sy * sx - cz * cx) * pz;
                j[12] = (cy * cx) * py + (-cy * sx) * pz;
                j[1] = (-cz * sy) * px + (cz * cy * sx) * py + (cz * cy * cx) * pz;
                j[7] = (-sz * sy) * px + (sz * cy * sx) * py + (sz * cy * cx) * pz;
                j[13] = (-cy) * px + (-sy * sx) * py + (-sy * cx) * pz;
                j[2] = (-sz * cy) * px + (-sz * sy * sx - cz * cx) * py + (-sz * sy * cx + cz * sx) * pz;
                j[8] = (cz * cy) * px + (cz * sy * sx - sz * cx) * py + (cz * sy * cx + sz * sx) * pz;
            } else {
                j[0] = (-sz * cx * sy) * px + (sz * sx) * py + (sz * cx * cy) * pz;
                j[6] = (cz * cx * sy) * px + (-cz * sx) * py + (-cz * cx * cy) * pz;
                j[12] = (sx * sy) * px + (cx) * py + (-sx * cy) * pz;
                j[1] = (-cz * sy - sz * sx * cy) * px + (cz * cy - sz * sx * sy) * pz;
                j[7] = (-sz * sy + cz * sx * cy) * px + (sz * cy + cz * sx * sy) * pz;
                j[13] = (-cx * cy) * px + (-cx * sy) * pz;
                j[2] = (-sz * cy - cz * sx * sy) * px + (-cz * cx) * py + (-sz * sy + cz * sx * cy) * pz;
                j[8] = (cz * cy - sz * sx * sy) * px + (-sz * cx) * py + (cz * sy + sz * sx * cy) * pz;
            }
            j[3] = 1.0; j[10] = 1.0; j[17] = 1.0;
            return;
        }
        // versor rigid
        const double vxx = vx * vx, vyy = vy * vy, vzz = vz * vz, vww = vw * vw;
        const double vxy = vx * vy, vxz = vx * vz, vxw = vx * vw;
        const double vyz = vy * vz, vyw = vy * vw, vzw = vz * vw;
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
};

mi_status build_family(int kind, const double* params, int nparams, const double* fixed, int nfixed,
                       Family& f);

}  // namespace

namespace mi {

mi_status transform_form(int kind, const double* params, int nparams, const double* fixed,
                         int nfixed, AffineForm* out) {
    if (!params || !out) return MI_ERR_INVALID_ARGUMENT;
    Family f{};
    const mi_status s = build_family(kind, params, nparams, fixed, nfixed, f);
    if (s != MI_OK) return s;
    out->nparams = f.P;
    for (int i = 0; i < 9; ++i) out->stage[i] = f.m[i];
    for (int d = 0; d < 3; ++d) out->stage[9 + d] = f.off[d];
    // J is linear in p = x − center plus a constant translation block.
    double jt[3 * MI_MAX_PARAMS];
    f.jac_centered(0.0, 0.0, 0.0, jt);  // the constant part
    for (int e = 0; e < 3; ++e) {
        double unit[3] = {0.0, 0.0, 0.0};
        unit[e] = 1.0;
        double je[3 * MI_MAX_PARAMS];
        f.jac_centered(unit[0], unit[1], unit[2], je);
        for (int i = 0; i < 3 * f.P; ++i) out->jacc[e][i] = je[i] - jt[i];
    }
    f.jac_centered(-f.center[0], -f.center[1], -f.center[2], out->jac0);
    return MI_OK;
}

mi_status transform_jacobian(int kind, const double* params, int nparams, const double* fixed, int nfixed,
                             const double* x, double* jac) {
    if (!params || !x || !jac) return MI_ERR_INVALID_ARGUMENT;
    Family f{};
    const mi_status s = build_family(kind, params, nparams, fixed, nfixed, f);
    if (s != MI_OK) return s;
    // jacobian_wrt_parameters(point): p = point − center first, as each family does
    f.jac_centered(x[0] - f.center[0], x[1] - f.center[1], x[2] - f.center[2], jac);
    return MI_OK;
}

}  // namespace mi

namespace {

mi_status build_family(int kind, const double* params, int nparams, const double* fixed, int nfixed,
                       Family& f) {
    f.kind = kind;
    for (int d = 0; d < 3; ++d) f.center[d] = (fixed && nfixed >= 3) ? fixed[d] : 0.0;
    switch (kind) {
        case MI_TRANSFORM_AFFINE: {
            // AffineTransform::set_parameters + compute_offset (parametric.rs:522-527, :566-573)
            if (nparams != 12) return MI_ERR_INVALID_ARGUMENT;
            f.P = 12;
            for (int i = 0; i < 9; ++i) f.m[i] = params[i];
            double ac[3];
            mat_vec3(f.m, f.center, ac);
            for (int d = 0; d < 3; ++d) f.off[d] = f.center[d] + params[9 + d] - ac[d];
            break;
        }
        case MI_TRANSFORM_TRANSLATION: {
            // p + t equals the identity-matrix stage bit for bit (matrix_offset.rs:62-70)
            if (nparams != 3) return MI_ERR_INVALID_ARGUMENT;
            f.P = 3;
            for (int i = 0; i < 9; ++i) f.m[i] = (i % 4 == 0) ? 1.0 : 0.0;
            for (int d = 0; d < 3; ++d) f.off[d] = params[d];
            break;
        }
        case MI_TRANSFORM_EULER3D: {
            // Euler3DTransform::recompute (parametric.rs:1063-1086): Rz·Rx·Ry by default
            if (nparams != 6) return MI_ERR_INVALID_ARGUMENT;
            f.P = 6;
            f.zyx = (fixed && nfixed == 4) ? (fixed[3] != 0.0) : false;
            for (int i = 0; i < 3; ++i) f.ang[i] = params[i];
            const double cx = std::cos(params[0]), sx = std::sin(params[0]);
            const double cy = std::cos(params[1]), sy = std::sin(params[1]);
            const double cz = std::cos(params[2]), sz = std::sin(params[2]);
            const double rx[9] = {1.0, 0.0, 0.0, 0.0, cx, -sx, 0.0, sx, cx};
            const double ry[9] = {cy, 0.0, sy, 0.0, 1.0, 0.0, -sy, 0.0, cy};
            const double rz[9] = {cz, -sz, 0.0, sz, cz, 0.0, 0.0, 0.0, 1.0};
            double t[9];
            if (f.zyx) { mat_mul3(rz, ry, t); mat_mul3(t, rx, f.m); }
            else { mat_mul3(rz, rx, t); mat_mul3(t, ry, f.m); }
            double mc[3];
            mat_vec3(f.m, f.center, mc);
            for (int i = 0; i < 3; ++i) f.off[i] = params[3 + i] + f.center[i] - mc[i];
            break;
        }
        case MI_TRANSFORM_VERSOR_RIGID3D: {
            // VersorRigid3DTransform::set_versor + recompute (parametric.rs:1310-1345)
            if (nparams != 6) return MI_ERR_INVALID_ARGUMENT;
            f.P = 6;
            const double eps = 1e-10;
            double ax = params[0], ay = params[1], az = params[2];
            const double norm = std::sqrt(ax * ax + ay * ay + az * az);
            if (norm >= 1.0 - eps) {
                const double d = norm + eps * norm;
                ax = params[0] / d; ay = params[1] / d; az = params[2] / d;
            }
            f.vx = ax; f.vy = ay; f.vz = az;
            const double s = 1.0 - (ax * ax + ay * ay + az * az);
            f.vw = std::sqrt(s > 0.0 ? s : 0.0);
            const double x = f.vx, y = f.vy, z = f.vz, w = f.vw;
            const double xx = x * x, yy = y * y, zz = z * z;
            const double xy = x * y, xz = x * z, xw = x * w;
            const double yz = y * z, yw = y * w, zw = z * w;
            const double m[9] = {1.0 - 2.0 * (yy + zz), 2.0 * (xy - zw), 2.0 * (xz + yw),
                                 2.0 * (xy + zw), 1.0 - 2.0 * (xx + zz), 2.0 * (yz - xw),
                                 2.0 * (xz - yw), 2.0 * (yz + xw), 1.0 - 2.0 * (xx + yy)};
            double mc[3];
            mat_vec3(m, f.center, mc);
            for (int i = 0; i < 3; ++i) f.off[i] = params[3 + i] + f.center[i] - mc[i];
            std::memcpy(f.m, m, sizeof(m));
            break;
        }
        default:
            return MI_ERR_INVALID_ARGUMENT;
    }
    return MI_OK;
}

}  // namespace
