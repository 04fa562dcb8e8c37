"""Second, independent CPU oracle in vectorised numpy FP64 (test infrastructure only).

It restates the same reference algorithm as oracle/mattes_oracle.cpp
(crates/sitk/src/registration/mattes.rs:522-676 with metric.rs:795-861,
transform/interpolator.rs:29-152, scales.rs:259-271) but is written separately, as
array code: every per-sample quantity is a numpy expression evaluated with the same
operation order (numpy never fuses a multiply and an add), and every histogram bin
is summed in sample order through np.bincount. The two oracles must therefore agree
on every per-sample decision exactly and on the value to the last bits; a
transcription error in either shows up as a disagreement. Only tests import it.
"""
from __future__ import annotations

import math

import numpy as np

PADDING = 2
EPS = np.finfo(np.float64).eps


def _i2p(geo):
    d = np.asarray(geo["direction"], dtype=np.float64).reshape(3, 3)
    s = np.asarray(geo["spacing"], dtype=np.float64)
    return d * s[None, :]


def _invert3(m):
    """Gauss–Jordan with partial pivoting (core/matrix.rs:44-104), same order."""
    a = np.zeros((3, 6))
    a[:, :3] = m
    a[:, 3:] = np.eye(3)
    for col in range(3):
        piv = col
        best = abs(a[col, col])
        for r in range(col + 1, 3):
            if abs(a[r, col]) > best:
                best, piv = abs(a[r, col]), r
        if best < 1e-12:
            raise ValueError("singular direction")
        if piv != col:
            a[[col, piv]] = a[[piv, col]]
        a[col] = a[col] / a[col, col]
        for r in range(3):
            if r == col or a[r, col] == 0.0:
                continue
            a[r] = a[r] - a[r, col] * a[col]
    return a[:, 3:].copy()


def _matvec(m, v):
    # zero-seeded accumulation in column order (core/matrix.rs:9-21)
    out = []
    for r in range(3):
        acc = 0.0
        for c in range(3):
            acc = acc + m[r][c] * v[c]
        out.append(acc)
    return out


def _matmul(a, b):
    out = [[0.0] * 3 for _ in range(3)]
    for r in range(3):
        for k in range(3):
            if a[r][k] == 0.0:
                continue
            for c in range(3):
                out[r][c] = out[r][c] + a[r][k] * b[k][c]
    return out


def transform_parts(kind, params, fixed_params=None):
    """(matrix 3×3 list, offset list, jacobian callable) per transform family."""
    c = [0.0, 0.0, 0.0] if fixed_params is None else [float(x) for x in fixed_params[:3]]
    p = [float(x) for x in params]
    if kind == 0:  # affine
        m = [p[0:3], p[3:6], p[6:9]]
        ac = _matvec(m, c)
        off = [c[d] + p[9 + d] - ac[d] for d in range(3)]

        def jac(x):  # x: (3, n)
            n = x.shape[1]
            j = np.zeros((3, 12, n))
            for i in range(3):
                for cc in range(3):
                    j[i, i * 3 + cc] = x[cc] - c[cc]
                j[i, 9 + i] = 1.0
            return j
        return m, off, jac
    if kind == 3:  # translation
        m = [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]

        def jac(x):
            j = np.zeros((3, 3, x.shape[1]))
            for i in range(3):
                j[i, i] = 1.0
            return j
        return m, [p[0], p[1], p[2]], jac
    if kind == 1:  # Euler3D
        zyx = fixed_params is not None and len(fixed_params) == 4 and fixed_params[3] != 0.0
        cx, sx = math.cos(p[0]), math.sin(p[0])
        cy, sy = math.cos(p[1]), math.sin(p[1])
        cz, sz = math.cos(p[2]), math.sin(p[2])
        rx = [[1.0, 0.0, 0.0], [0.0, cx, -sx], [0.0, sx, cx]]
        ry = [[cy, 0.0, sy], [0.0, 1.0, 0.0], [-sy, 0.0, cy]]
        rz = [[cz, -sz, 0.0], [sz, cz, 0.0], [0.0, 0.0, 1.0]]
        m = _matmul(_matmul(rz, ry), rx) if zyx else _matmul(_matmul(rz, rx), ry)
        mc = _matvec(m, c)
        off = [p[3 + i] + c[i] - mc[i] for i in range(3)]

        def jac(x):
            px, py, pz = x[0] - c[0], x[1] - c[1], x[2] - c[2]
            j = np.zeros((3, 6, x.shape[1]))
            if zyx:
                j[0, 0] = (cz * sy * cx + sz * sx) * py + (-cz * sy * sx + sz * cx) * pz
                j[1, 0] = (sz * sy * cx - cz * sx) * py + (-sz * sy * sx - cz * cx) * pz
                j[2, 0] = (cy * cx) * py + (-cy * sx) * pz
                j[0, 1] = (-cz * sy) * px + (cz * cy * sx) * py + (cz * cy * cx) * pz
                j[1, 1] = (-sz * sy) * px + (sz * cy * sx) * py + (sz * cy * cx) * pz
                j[2, 1] = (-cy) * px + (-sy * sx) * py + (-sy * cx) * pz
                j[0, 2] = (-sz * cy) * px + (-sz * sy * sx - cz * cx) * py + (-sz * sy * cx + cz * sx) * pz
                j[1, 2] = (cz * cy) * px + (cz * sy * sx - sz * cx) * py + (cz * sy * cx + sz * sx) * pz
            else:
                j[0, 0] = (-sz * cx * sy) * px + (sz * sx) * py + (sz * cx * cy) * pz
                j[1, 0] = (cz * cx * sy) * px + (-cz * sx) * py + (-cz * cx * cy) * pz
                j[2, 0] = (sx * sy) * px + (cx) * py + (-sx * cy) * pz
                j[0, 1] = (-cz * sy - sz * sx * cy) * px + (cz * cy - sz * sx * sy) * pz
                j[1, 1] = (-sz * sy + cz * sx * cy) * px + (sz * cy + cz * sx * sy) * pz
                j[2, 1] = (-cx * cy) * px + (-cx * sy) * pz
                j[0, 2] = (-sz * cy - cz * sx * sy) * px + (-cz * cx) * py + (-sz * sy + cz * sx * cy) * pz
                j[1, 2] = (cz * cy - sz * sx * sy) * px + (-sz * cx) * py + (cz * sy + sz * sx * cy) * pz
            j[0, 3] = 1.0
            j[1, 4] = 1.0
            j[2, 5] = 1.0
            return j
        return m, off, jac
    if kind == 2:  # VersorRigid3D
        vx, vy, vz = p[0], p[1], p[2]
        norm = math.sqrt(vx * vx + vy * vy + vz * vz)
        if norm >= 1.0 - 1e-10:
            dd = norm + 1e-10 * norm
            vx, vy, vz = vx / dd, vy / dd, vz / dd
        vw = math.sqrt(max(1.0 - (vx * vx + vy * vy + vz * vz), 0.0))
        xx, yy, zz = vx * vx, vy * vy, vz * vz
        xy, xz, xw = vx * vy, vx * vz, vx * vw
        yz, yw, zw = vy * vz, vy * vw, vz * vw
        m = [[1.0 - 2.0 * (yy + zz), 2.0 * (xy - zw), 2.0 * (xz + yw)],
             [2.0 * (xy + zw), 1.0 - 2.0 * (xx + zz), 2.0 * (yz - xw)],
             [2.0 * (xz - yw), 2.0 * (yz + xw), 1.0 - 2.0 * (xx + yy)]]
        mc = _matvec(m, c)
        off = [p[3 + i] + c[i] - mc[i] for i in range(3)]

        def jac(x):
            px, py, pz = x[0] - c[0], x[1] - c[1], x[2] - c[2]
            vxx, vyy, vzz, vww = vx * vx, vy * vy, vz * vz, vw * vw
            vxy, vxz, vxw = vx * vy, vx * vz, vx * vw
            vyz, vyw, vzw = vy * vz, vy * vw, vz * vw
            j = np.zeros((3, 6, x.shape[1]))
            j[0, 0] = 2.0 * ((vyw + vxz) * py + (vzw - vxy) * pz) / vw
            j[1, 0] = 2.0 * ((vyw - vxz) * px - 2.0 * vxw * py + (vxx - vww) * pz) / vw
            j[2, 0] = 2.0 * ((vzw + vxy) * px + (vww - vxx) * py - 2.0 * vxw * pz) / vw
            j[0, 1] = 2.0 * (-2.0 * vyw * px + (vxw + vyz) * py + (vww - vyy) * pz) / vw
            j[1, 1] = 2.0 * ((vxw - vyz) * px + (vzw + vxy) * pz) / vw
            j[2, 1] = 2.0 * ((vyy - vww) * px + (vzw - vxy) * py - 2.0 * vyw * pz) / vw
            j[0, 2] = 2.0 * (-2.0 * vzw * px + (vzz - vww) * py + (vxw - vyz) * pz) / vw
            j[1, 2] = 2.0 * ((vww - vzz) * px - 2.0 * vzw * py + (vyw + vxz) * pz) / vw
            j[2, 2] = 2.0 * ((vxw + vyz) * px + (vyw - vxz) * py) / vw
            j[0, 3] = 1.0
            j[1, 4] = 1.0
            j[2, 5] = 1.0
            return j
        return m, off, jac
    raise ValueError(f"unknown transform kind {kind}")


def _bspline3(u):
    a = np.abs(u)
    sq = a * a
    inner = (4.0 - 6.0 * sq + 3.0 * sq * a) / 6.0
    outer = (8.0 - 12.0 * a + 6.0 * sq - sq * a) / 6.0
    return np.where(a < 1.0, inner, np.where(a < 2.0, outer, 0.0))


def _bspline3_deriv(u):
    r = np.zeros_like(u)
    m1 = (u >= 0.0) & (u < 1.0)
    m2 = (u > -1.0) & (u < 0.0)
    m3 = (u >= 1.0) & (u < 2.0)
    m4 = (u > -2.0) & (u <= -1.0)
    r = np.where(m1, -2.0 * u + 1.5 * u * u, r)
    r = np.where(m2, -2.0 * u - 1.5 * u * u, r)
    r = np.where(m3, -2.0 + 2.0 * u - 0.5 * u * u, r)
    r = np.where(m4, 2.0 + 2.0 * u + 0.5 * u * u, r)
    return r


def _parzen(values, bin_size, nmin, bins):
    term = values / bin_size - nmin
    idx = np.trunc(term).astype(np.int64)
    return np.clip(idx, PADDING, bins - PADDING - 1), term


def evaluate(fixed, fgeo, moving, mgeo, bins, kind, params, fixed_params=None, fmask=None,
             mmask=None, draw=None, derivative=True):
    """Returns dict(value, derivative, valid, status, fi, mi) — status per sample in
    post-filter order: 0 outside/masked, 1 out of moving range, 2 valid."""
    fixed = np.asarray(fixed, dtype=np.float32).ravel()
    moving = np.asarray(moving, dtype=np.float32).ravel()
    fsize = [int(v) for v in fgeo["size"]]
    msize = [int(v) for v in mgeo["size"]]
    nvox = fsize[0] * fsize[1] * fsize[2]
    if bins < 2 * PADDING + 1:
        raise ValueError("too few bins")

    # sample set: draw then fixed-mask filter (metric.rs:528-540)
    if draw is None:
        flats = np.arange(nvox, dtype=np.int64)
    else:
        flats = np.asarray(draw, dtype=np.int64)
    if fmask is not None:
        flats = flats[np.asarray(fmask).ravel()[flats] != 0]
    n = flats.size
    fv = fixed[flats].astype(np.float64)

    # histogram ranges
    fmin, fmax = (float(fv.min()), float(fv.max())) if n else (0.0, 0.0)
    mvals = moving.astype(np.float64)
    if mmask is not None:
        mvals = mvals[np.asarray(mmask).ravel() != 0]
    mmin, mmax = (float(mvals.min()), float(mvals.max())) if mvals.size else (0.0, 0.0)
    if fmax - fmin <= EPS:
        raise ValueError("constant fixed")
    if mmax - mmin <= EPS:
        raise ValueError("constant moving")
    denom = float(bins - 2 * PADDING)
    fbs = (fmax - fmin) / denom
    mbs = (mmax - mmin) / denom
    fnm = fmin / fbs - PADDING
    mnm = mmin / mbs - PADDING

    # fixed points (scales.rs:259-271): origin-seeded
    i = (flats % fsize[0]).astype(np.float64)
    j = ((flats // fsize[0]) % fsize[1]).astype(np.float64)
    k = (flats // (fsize[0] * fsize[1])).astype(np.float64)
    m_f = _i2p(fgeo)
    fo = np.asarray(fgeo["origin"], dtype=np.float64)
    x = np.empty((3, n))
    for r in range(3):
        acc = fo[r] + m_f[r, 0] * i
        acc = acc + m_f[r, 1] * j
        acc = acc + m_f[r, 2] * k
        x[r] = acc

    # transform point: mat_vec then + offset
    tm, toff, jacfn = transform_parts(kind, params, fixed_params)
    y = np.empty((3, n))
    for d in range(3):
        acc = 0.0 + tm[d][0] * x[0]
        acc = acc + tm[d][1] * x[1]
        acc = acc + tm[d][2] * x[2]
        y[d] = acc + toff[d]

    # continuous index c = M·(y − o)
    p2i = _invert3(_i2p(mgeo))
    mo = np.asarray(mgeo["origin"], dtype=np.float64)
    diff = y - mo[:, None]
    c = np.empty((3, n))
    for r in range(3):
        acc = p2i[r, 0] * diff[0]
        acc = acc + p2i[r, 1] * diff[1]
        acc = acc + p2i[r, 2] * diff[2]
        c[r] = acc

    ok = np.ones(n, dtype=bool)
    if mmask is not None:
        mm = np.asarray(mmask).ravel()
        r = np.floor(c + 0.5)
        inb = np.all((r >= 0) & (r < np.asarray(msize)[:, None]), axis=0)
        rr = np.where(inb[None, :], r, 0).astype(np.int64)
        flat_m = rr[0] + msize[0] * (rr[1] + msize[1] * rr[2])
        ok &= inb & (mm[flat_m] != 0)
    for d in range(3):
        ok &= (c[d] >= -0.5) & (c[d] < float(msize[d]) - 0.5)

    fl = np.floor(c)
    frac = c - fl
    base = fl.astype(np.int64)
    one_m = 1.0 - frac
    val = np.zeros(n)
    g = np.zeros((3, n))
    for corner in range(8):
        bits = [(corner >> d) & 1 for d in range(3)]
        w = 1.0
        for d in range(3):
            w = w * (frac[d] if bits[d] else one_m[d])
        idx = [np.clip(base[d] + bits[d], 0, msize[d] - 1) for d in range(3)]
        off = idx[0] + msize[0] * (idx[1] + msize[1] * idx[2])
        off = np.where(ok, off, 0)
        b = moving[off].astype(np.float64)
        val = val + w * b
        for jj in range(3):
            wj = 1.0
            for d in range(3):
                if d == jj:
                    continue
                wj = wj * (frac[d] if bits[d] else one_m[d])
            sign = 1.0 if bits[jj] else -1.0
            g[jj] = g[jj] + sign * wj * b
    gphys = np.empty((3, n))
    for d in range(3):
        acc = g[0] * p2i[0, d]
        acc = acc + g[1] * p2i[1, d]
        acc = acc + g[2] * p2i[2, d]
        gphys[d] = acc

    status = np.where(ok, 2, 0).astype(np.int8)
    inr = ok & (val >= mmin) & (val <= mmax)
    status = np.where(ok & ~inr, 1, status).astype(np.int8)
    mi, mterm = _parzen(val, mbs, mnm, bins)
    fi, _ = _parzen(fv, fbs, fnm, bins)
    valid = int(inr.sum())

    sel = np.nonzero(inr)[0]
    fi_v, mi_v, mt_v = fi[sel], mi[sel], mterm[sel]
    taps = mi_v[:, None] - 1 + np.arange(4)[None, :]
    args = taps.astype(np.float64) - mt_v[:, None]
    keys = (fi_v[:, None] * bins + taps).ravel()
    joint = np.bincount(keys, weights=_bspline3(args).ravel(), minlength=bins * bins)
    fmarg = np.bincount(fi_v, minlength=bins).astype(np.float64)

    nparams = {0: 12, 1: 6, 2: 6, 3: 3}[kind]
    out_fi = np.where(inr, fi, -1).astype(np.int32)
    out_mi = np.where(inr, mi, -1).astype(np.int32)
    res = {"valid": valid, "status": status, "fi": out_fi, "mi": out_mi,
           "derivative": np.zeros(nparams), "joint": joint.copy(), "fixed_marginal": fmarg.copy()}
    if valid == 0:
        res["value"] = float(np.finfo(np.float64).max)
        return res
    # Kahan (core/compensated.rs:112-123)
    s = 0.0
    comp = 0.0
    for v in joint.tolist():
        ci = v - comp
        t = s + ci
        comp = (t - s) - ci
        s = t
    if s < EPS:
        res["value"] = float(np.finfo(np.float64).max)
        return res
    nf = 1.0 / (mbs * valid)
    jpd = None
    if derivative:
        jac = jacfn(x[:, sel])  # (3, P, nv)
        inner = np.zeros((nparams, sel.size))
        for kk in range(nparams):
            acc = 0.0 + jac[0, kk] * gphys[0, sel]
            acc = acc + jac[1, kk] * gphys[1, sel]
            acc = acc + jac[2, kk] * gphys[2, sel]
            inner[kk] = acc
        dw = _bspline3_deriv(args)  # (nv, 4)
        jpd = np.zeros((bins * bins, nparams))
        for kk in range(nparams):
            contrib = (inner[kk][:, None] * dw).ravel()
            jpd[:, kk] = np.bincount(keys, weights=contrib, minlength=bins * bins)
        jpd = jpd * nf
    inv = 1.0 / s
    jp = joint * inv
    fm = fmarg * inv
    jp2 = jp.reshape(bins, bins)
    mm_ = np.zeros(bins)
    for f in range(bins):
        mm_ = mm_ + jp2[f]
    total = 0.0
    deriv = np.zeros(nparams)
    for f in range(bins):
        if fm[f] <= EPS:
            continue
        lf = math.log(fm[f])
        for m in range(bins):
            if mm_[m] > EPS and jp2[f, m] > EPS:
                pr = math.log(jp2[f, m] / mm_[m])
                total += jp2[f, m] * (pr - lf)
                if derivative:
                    deriv = deriv + jpd[f * bins + m] * pr
    res["value"] = -total
    res["derivative"] = deriv
    return res
