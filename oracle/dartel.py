"""ORACLE (test infrastructure): NumPy restatement of the reference's 2-D DARTEL.

Every function follows the reference's torch CPU path operation by operation
(``src/cat_surface_gpu/dartel_grid.py`` and ``surface_warp.py``), one IEEE
rounding per operation and the same association order, so float64 and
float32 results are reproducible bit-for-bit by a kernel that keeps that
order.  Fields are ``[channels, ny, nx]`` arrays; maps use CAT's one-based
coordinates; Jacobians are stored ``(j00, j10, j01, j11)``.

Boundary rule (``dartel_grid.py:190-208``): x is periodic, y is reflected
with period ``2 ny`` (``ny == 1`` collapses y to 0).
"""

from __future__ import annotations

import numpy as np


# --------------------------------------------------------------------------- basics


def bound_indices(ix, iy, nx, ny):
    """dartel_grid.py:190-208 (_bound_indices)."""

    x = np.remainder(ix, nx)
    if ny == 1:
        return x, np.zeros_like(iy)
    period = 2 * ny
    reflected = np.remainder(iy, period)
    return x, np.where(reflected >= ny, period - reflected - 1, reflected)


def shift(field, dx, dy):
    """dartel_grid.py:211-226 (_shift): value at (x + dx, y + dy) with the boundary rule."""

    ny, nx = field.shape[-2:]
    shifted = np.roll(field, -dx, axis=-1)
    y = np.arange(ny) + dy
    if ny == 1:
        yi = np.zeros_like(y)
    else:
        period = 2 * ny
        r = np.remainder(y, period)
        yi = np.where(r >= ny, period - r - 1, r)
    return np.take(shifted, yi, axis=-2)


def identity_map(nx, ny, dtype=np.float64):
    """dartel_grid.py:174-187 (make_identity_map), one-based."""

    x = np.broadcast_to(np.arange(1, nx + 1, dtype=dtype)[None, :], (ny, nx))
    y = np.broadcast_to(np.arange(1, ny + 1, dtype=dtype)[:, None], (ny, nx))
    return np.stack((x, y)).astype(dtype)


def interpolation_indices(x, y, nx, ny):
    """dartel_grid.py:348-366 (_interpolation_indices)."""

    ix = np.floor(x).astype(np.int64)
    iy = np.floor(y).astype(np.int64)
    dx1 = x - ix.astype(x.dtype)
    dy1 = y - iy.astype(y.dtype)
    one = x.dtype.type(1.0)
    dx2 = one - dx1
    dy2 = one - dy1
    x22, y22 = bound_indices(ix, iy, nx, ny)
    x12, y12 = bound_indices(ix + 1, iy, nx, ny)
    x21, y21 = bound_indices(ix, iy + 1, nx, ny)
    x11, y11 = bound_indices(ix + 1, iy + 1, nx, ny)
    return x22, y22, x12, y12, x21, y21, x11, y11, dx1, dx2, dy1, dy2


def interpolate_channels(field, idx):
    """dartel_grid.py:369-394: (k22 dx2 + k12 dx1) dy2 + (k21 dx2 + k11 dx1) dy1."""

    x22, y22, x12, y12, x21, y21, x11, y11, dx1, dx2, dy1, dy2 = idx
    k22 = field[:, y22, x22]
    k12 = field[:, y12, x12]
    k21 = field[:, y21, x21]
    k11 = field[:, y11, x11]
    return (k22 * dx2 + k12 * dx1) * dy2 + (k21 * dx2 + k11 * dx1) * dy1


def _unwrap(c, c22, periods):
    return c - np.floor((c - c22) / periods + c.dtype.type(0.5)) * periods


def composition(a, b):
    """dartel_grid.py:407-440 (_composition_optimized): (B o A) with period unwrapping."""

    ny, nx = a.shape[1:]
    dt = a.dtype.type
    x = a[0] - dt(1.0)
    y = a[1] - dt(1.0)
    idx = interpolation_indices(x, y, nx, ny)
    periods = np.array((nx, ny), dtype=a.dtype).reshape(2, 1, 1)
    x22, y22, x12, y12, x21, y21, x11, y11, dx1, dx2, dy1, dy2 = idx
    cf = b - dt(1.0)
    c22 = cf[:, y22, x22]
    c12 = _unwrap(cf[:, y12, x12], c22, periods)
    c21 = _unwrap(cf[:, y21, x21], c22, periods)
    c11 = _unwrap(cf[:, y11, x11], c22, periods)
    return (c22 * dx2 + c12 * dx1) * dy2 + (c21 * dx2 + c11 * dx1) * dy1 + dt(1.0)


def composition_jacobian(a, ja, b, jb):
    """dartel_grid.py:443-507 (_composition_jacobian_optimized)."""

    ny, nx = a.shape[1:]
    dt = a.dtype.type
    x = a[0] - dt(1.0)
    y = a[1] - dt(1.0)
    idx = interpolation_indices(x, y, nx, ny)
    sampled = interpolate_channels(jb, idx)
    coordinates = composition(a, b)
    jb00, jb01, jb10, jb11 = sampled
    jac = np.stack(
        (
            jb00 * ja[0] + jb10 * ja[1],
            jb01 * ja[0] + jb11 * ja[1],
            jb00 * ja[2] + jb10 * ja[3],
            jb01 * ja[2] + jb11 * ja[3],
        )
    )
    return coordinates, jac


def jacobian_of_displacement(v, scale):
    """dartel_grid.py:624-652: central differences times scale / 2 (plus identity)."""

    ny, nx = v.shape[1:]
    dt = v.dtype.type
    s = dt(float(scale) * 0.5)
    xm = shift(v, -1, 0)
    xp = shift(v, 1, 0)
    ym = shift(v, 0, -1)
    yp = shift(v, 0, 1)
    j00 = (xm[0] * dt(-1.0) + xp[0]) * s + dt(1.0)
    j10 = (xm[1] * dt(-1.0) + xp[1]) * s
    j01 = (ym[0] * dt(-1.0) + yp[0]) * s
    j11 = (ym[1] * dt(-1.0) + yp[1]) * s + dt(1.0)
    return np.stack((j00, j10, j01, j11))


def smalldef_jac(v, scale):
    """dartel_grid.py:655-675: (id + v * scale, Jacobian)."""

    ny, nx = v.shape[1:]
    t = identity_map(nx, ny, v.dtype) + v * v.dtype.type(float(scale))
    return t, jacobian_of_displacement(v, scale)


def jac_div_smalldef(jac, v, scale):
    """dartel_grid.py:678-720: J . (I + s grad v)^-1."""

    d00, d10, d01, d11 = jacobian_of_displacement(v, scale)
    det = d00 * d11 - d01 * d10
    i00 = d11 / det
    i10 = -d10 / det
    i01 = -d01 / det
    i11 = d00 / det
    o00, o10, o01, o11 = jac
    return np.stack((o00 * i00 + o01 * i10, o10 * i00 + o11 * i10, o00 * i01 + o01 * i11, o10 * i01 + o11 * i11))


def initialise_objfun(source, target, t, jac, weights=None):
    """dartel_grid.py:723-775: Gauss-Newton gradient and Hessian of the SSD term."""

    ny, nx = source.shape
    dt = source.dtype.type
    if weights is None:
        weights = np.ones_like(target)
    x = t[0] - dt(1.0)
    y = t[1] - dt(1.0)
    idx = interpolation_indices(x, y, nx, ny)
    x22, y22, x12, y12, x21, y21, x11, y11, dx1, dx2, dy1, dy2 = idx
    k22 = source[y22, x22]
    k12 = source[y12, x12]
    k21 = source[y21, x21]
    k11 = source[y11, x11]
    sampled = (k22 * dx2 + k12 * dx1) * dy2 + (k21 * dx2 + k11 * dx1) * dy1
    diff = sampled - target
    ddx = (k11 - k21) * dy1 + (k12 - k22) * dy2
    ddy = (k11 * dx1 + k21 * dx2) - (k12 * dx1 + k22 * dx2)
    gx = jac[0] * ddx + jac[1] * ddy
    gy = jac[2] * ddx + jac[3] * ddy
    hess = np.stack((gx * gx * weights, gy * gy * weights, gx * gy * weights))
    rhs = np.stack((gx * diff * weights, gy * diff * weights))
    objective = dt(0.5) * np.sum(diff * diff * weights)
    return objective, rhs, hess


def _squaring_increment(b, a, t, jac):
    """One fused increment of dartel_grid.py:832-893 (optimized torch path)."""

    ny, nx = t.shape[1:]
    dt = t.dtype.type
    x = t[0] - dt(1.0)
    y = t[1] - dt(1.0)
    j00, j10, j01, j11 = jac
    det = j00 * j11 - j01 * j10
    s = interpolate_channels(np.concatenate((b, a)), interpolation_indices(x, y, nx, ny))
    sbx, sby, sa00, sa11, sa01 = s
    binc = np.stack((det * (sbx * j00 + sby * j10), det * (sbx * j01 + sby * j11)))
    tmp1 = sa00 * j00 + sa01 * j10
    tmp2 = sa01 * j00 + sa11 * j10
    tmp3 = sa00 * j01 + sa01 * j11
    tmp4 = sa01 * j01 + sa11 * j11
    ainc = np.stack((det * (tmp1 * j00 + tmp2 * j10), det * (tmp3 * j01 + tmp4 * j11), det * (tmp1 * j01 + tmp2 * j11)))
    return binc, ainc


def squaring_update(rhs, hess, t, jac, k, save_transformation=False):
    """dartel_grid.py:778-914.  Returns (b, A, map, J, scratch).

    ``scratch`` is the reference's ``map_buffers[0]`` after the loop (used by
    dartel_step as the multigrid initial guess): the input map when k <= 1 or
    when the final map is saved... see the slot bookkeeping below, which is
    the reference's, step for step.
    """

    b = rhs.copy()
    a = hess.copy()
    maps = [t, None]
    jacs = [jac, None]
    cur, other = 0, 1
    for step in range(k):
        binc, ainc = _squaring_increment(b, a, maps[cur], jacs[cur])
        b = b + binc
        a = a + ainc
        maps[other] = binc
        if save_transformation or step < k - 1:
            cm, cj = composition_jacobian(maps[cur], jacs[cur], maps[cur], jacs[cur])
            maps[other] = cm
            jacs[other] = cj
            cur, other = other, cur
    if save_transformation and cur != 0:
        maps[other] = maps[cur].copy()
        jacs[other] = jacs[cur].copy()
    return b, a, maps[cur], jacs[cur], maps[0]


def regularization_operator(v, params, rtype=1):
    """dartel_grid.py:917-1015 (rtype 0 linear-elastic, 1 membrane, 2 bending)."""

    dt = v.dtype.type
    sx, sy, mu, lam, ident = (float(p) for p in params)
    sx2, sy2 = sx * sx, sy * sy
    xm, xp, ym, yp = shift(v, -1, 0), shift(v, 1, 0), shift(v, 0, -1), shift(v, 0, 1)
    if rtype == 1:
        w00 = dt(mu * (2.0 * sx2 + 2.0 * sy2) + ident)
        w01 = dt(-mu * sy2)
        w10 = dt(-mu * sx2)
        return np.stack([w00 * v[c] + w01 * (ym[c] + yp[c]) + w10 * (xm[c] + xp[c]) for c in range(2)])
    if rtype == 0:
        wx0 = dt(mu * (2.0 * sy2 + 4.0 * sx2) + 2.0 * lam * sx2 + ident)
        wy0 = dt(mu * (2.0 * sx2 + 4.0 * sy2) + 2.0 * lam * sy2 + ident)
        wx1 = dt(-(2.0 * mu + lam) * sx2)
        wy1 = dt(-(2.0 * mu + lam) * sy2)
        wx2 = dt(-mu * sx2)
        wy2 = dt(-mu * sy2)
        wxy = dt(0.25 * (lam + mu) * sx * sy)
        xym, xyp, xpm, xpp = shift(v, -1, -1), shift(v, -1, 1), shift(v, 1, -1), shift(v, 1, 1)
        cross_x = xym[1] - xyp[1] - xpm[1] + xpp[1]
        cross_y = xym[0] - xyp[0] - xpm[0] + xpp[0]
        return np.stack(
            (
                wx0 * v[0] + wy2 * (ym[0] + yp[0]) + wx1 * (xm[0] + xp[0]) + wxy * cross_x,
                wy0 * v[1] + wy1 * (ym[1] + yp[1]) + wx2 * (xm[1] + xp[1]) + wxy * cross_y,
            )
        )
    sx4, sy4 = sx2 * sx2, sy2 * sy2
    w00 = dt(mu * (6.0 * sx4 + 6.0 * sy4 + 8.0 * sx2 * sy2) + ident)
    w01 = dt(mu * (-4.0 * sx2 * sy2 - 4.0 * sy4))
    w02 = dt(mu * sy4)
    w10 = dt(mu * (-4.0 * sx4 - 4.0 * sx2 * sy2))
    w11 = dt(mu * (2.0 * sx2 * sy2))
    w20 = dt(mu * sx4)
    xmm, xpp2, ymm, ypp = shift(v, -2, 0), shift(v, 2, 0), shift(v, 0, -2), shift(v, 0, 2)
    xmy, xpy, xmyp, xpyp = shift(v, -1, -1), shift(v, 1, -1), shift(v, -1, 1), shift(v, 1, 1)
    return np.stack(
        [
            w00 * v[c] + w01 * (ym[c] + yp[c]) + w02 * (ymm[c] + ypp[c]) + w10 * (xm[c] + xp[c])
            + w11 * (xmy[c] + xpy[c] + xmyp[c] + xpyp[c]) + w20 * (xmm[c] + xpp2[c])
            for c in range(2)
        ]
    )


def membrane_weights(params, dtype):
    sx, sy, mu, _lam, ident = (float(p) for p in params)
    return dtype(mu * (2.0 * sx * sx + 2.0 * sy * sy) + ident), dtype(-mu * sy * sy), dtype(-mu * sx * sx)


def apply_membrane_system(hess, v, params):
    """dartel_grid.py:1018-1070: (H + L_membrane) v."""

    reg = regularization_operator(v, params, rtype=1)
    return np.stack((reg[0] + hess[0] * v[0] + hess[2] * v[1], reg[1] + hess[2] * v[0] + hess[1] * v[1]))


def relax_membrane(hess, rhs, params, nit, initial=None):
    """dartel_grid.py:1073-1208: red-black Gauss-Seidel with a 2x2 point solve.

    Even nx (or nx == 1): the vectorised red-black path (1187-1208) -- cells
    with (x + y) odd first.  Odd nx > 1: the sequential scalar path
    (1154-1186), which updates in row-major order within each colour.
    """

    ny, nx = rhs.shape[1:]
    dt = rhs.dtype.type
    u = np.zeros_like(rhs) if initial is None else initial.copy()
    w00, w01, w10 = membrane_weights(params, dt)
    near = dt(1.0000000001)
    if nx % 2 == 1 and nx != 1:
        for it in range(2 * nit):
            for row in range(ny):
                start = int((it % 2) == (row % 2))
                for col in range(start, nx, 2):
                    xm, ym_ = bound_indices(col - 1, row, nx, ny)
                    xp, yp_ = bound_indices(col + 1, row, nx, ny)
                    x0, y0 = bound_indices(col, row - 1, nx, ny)
                    x1, y1 = bound_indices(col, row + 1, nx, ny)
                    rx = rhs[0, row, col] - w01 * (u[0, y0, x0] + u[0, y1, x1]) - w10 * (u[0, ym_, xm] + u[0, yp_, xp])
                    ry = rhs[1, row, col] - w01 * (u[1, y0, x0] + u[1, y1, x1]) - w10 * (u[1, ym_, xm] + u[1, yp_, xp])
                    dxx = hess[0, row, col] + w00
                    dyy = hess[1, row, col] + w00
                    cr = hess[2, row, col]
                    det = dxx * dyy * near - cr * cr
                    u[0, row, col] = (dyy * rx - cr * ry) / det
                    u[1, row, col] = (-cr * rx + dxx * ry) / det
        return u
    x = np.arange(nx)[None, :]
    y = np.arange(ny)[:, None]
    checker = ((x + y) & 1).astype(bool)
    for it in range(2 * nit):
        xm, xp, ym, yp = shift(u, -1, 0), shift(u, 1, 0), shift(u, 0, -1), shift(u, 0, 1)
        rx = rhs[0] - w01 * (ym[0] + yp[0]) - w10 * (xm[0] + xp[0])
        ry = rhs[1] - w01 * (ym[1] + yp[1]) - w10 * (xm[1] + xp[1])
        dxx = hess[0] + w00
        dyy = hess[1] + w00
        cr = hess[2]
        det = dxx * dyy * near - cr * cr
        nxv = (dyy * rx - cr * ry) / det
        nyv = (-cr * rx + dxx * ry) / det
        active = checker if it % 2 == 0 else ~checker
        u = np.stack((np.where(active, nxv, u[0]), np.where(active, nyv, u[1])))
    return u


def _wt2(d):
    a = np.abs(d)
    dt = d.dtype.type
    inner = dt(0.75) - a * a
    od = dt(1.5) - a
    outer = dt(0.5) * od * od
    return np.where(a < dt(0.5), inner, np.where(a < dt(1.5), outer, dt(0.0)))


def resize_field(field, tnx, tny):
    """dartel_grid.py:239-305: separable quadratic B-spline resize (y then x)."""

    c, sny, snx = field.shape
    dt = field.dtype.type
    yt = np.arange(tny, dtype=field.dtype)
    yl = (yt + dt(0.5)) * dt(sny) / dt(tny) - dt(0.5)
    yo = np.floor(yl + dt(0.5)).astype(np.int64)
    yw = _wt2(yo.astype(field.dtype) - yl)
    ywm = _wt2(yo.astype(field.dtype) - dt(1.0) - yl)
    ywp = _wt2(yo.astype(field.dtype) + dt(1.0) - yl)
    z = np.zeros_like(yo)
    _, ym = bound_indices(z, yo - 1, snx, sny)
    _, yc = bound_indices(z, yo, snx, sny)
    _, yp = bound_indices(z, yo + 1, snx, sny)
    inter = ywm[None, :, None] * field[:, ym, :] + yw[None, :, None] * field[:, yc, :] + ywp[None, :, None] * field[:, yp, :]
    xt = np.arange(tnx, dtype=field.dtype)
    xl = (xt + dt(0.5)) * dt(snx) / dt(tnx) - dt(0.5)
    xo = np.floor(xl + dt(0.5)).astype(np.int64)
    xw = _wt2(xo.astype(field.dtype) - xl)
    xwm = _wt2(xo.astype(field.dtype) - dt(1.0) - xl)
    xwp = _wt2(xo.astype(field.dtype) + dt(1.0) - xl)
    z = np.zeros_like(xo)
    xm, _ = bound_indices(xo - 1, z, snx, sny)
    xc, _ = bound_indices(xo, z, snx, sny)
    xp, _ = bound_indices(xo + 1, z, snx, sny)
    return xwm[None, None, :] * inter[:, :, xm] + xw[None, None, :] * inter[:, :, xc] + xwp[None, None, :] * inter[:, :, xp]


def grid_levels(nx, ny):
    """dartel_grid.py:1243-1249: halve (rounding up) until both sides are < 2."""

    specs = [(nx, ny)]
    while specs[-1][0] >= 2 or specs[-1][1] >= 2:
        px, py = specs[-1]
        coarse = ((px + 1) // 2, (py + 1) // 2)
        specs.append(coarse)
        if coarse[0] < 2 and coarse[1] < 2:
            break
    return specs


def fmg2_membrane(hess, rhs, params, cycles=3, nit=3, initial=None, assume_initial_nonzero=False):
    """dartel_grid.py:1211-1417: full multigrid for (H + L_membrane) u = b."""

    dt = rhs.dtype.type
    ny, nx = rhs.shape[1:]
    specs = grid_levels(nx, ny)
    base = tuple(float(p) for p in params)
    A = [hess]
    B0 = [rhs]
    for level in range(1, len(specs)):
        A.append(resize_field(A[-1], *specs[level]))
        B0.append(resize_field(B0[-1], *specs[level]))

    def lp(level):
        return (base[0] * specs[level][0] / nx, base[1] * specs[level][1] / ny, base[2], base[3], base[4])

    B = [rhs] + [np.zeros((2, s[1], s[0]), dtype=rhs.dtype) for s in specs[1:]]
    U = [np.zeros_like(b) for b in B]
    if initial is not None:
        U[0] = initial.copy()
        for level in range(1, len(specs)):
            U[level] = resize_field(U[level - 1], *specs[level])
    last = len(specs) - 1

    def residual(level):
        return B[level] - apply_membrane_system(A[level], U[level], lp(level))

    def cycle(start):
        for level in range(start, last):
            U[level] = relax_membrane(A[level], B[level], lp(level), nit, U[level])
            B[level + 1] = resize_field(residual(level), *specs[level + 1])
            U[level + 1] = np.zeros_like(B[level + 1])
        U[last] = relax_membrane(A[last], B[last], lp(last), nit, U[last])
        for level in range(last - 1, start - 1, -1):
            U[level] = U[level] + resize_field(U[level + 1], *specs[level])
            U[level] = relax_membrane(A[level], B[level], lp(level), nit, U[level])

    if initial is None:
        coarse_init = True
    elif assume_initial_nonzero:
        coarse_init = False
    else:
        coarse_init = not bool(np.any(U[0]))
    if coarse_init:
        ca, cb = A[last], B0[last]
        dxx = ca[0] + dt(base[4])
        dyy = ca[1] + dt(base[4])
        cr = ca[2]
        det = dxx * dyy * dt(1.0000000001) - cr * cr
        U[last] = np.stack(((dyy * cb[0] - cr * cb[1]) / det, (-cr * cb[0] + dxx * cb[1]) / det))
        U[last] = relax_membrane(ca, B[last], lp(last), nit, U[last])
        for level in range(last - 1, -1, -1):
            U[level] = resize_field(U[level + 1], *specs[level])
            if level > 0:
                B[level] = B0[level].copy()
            for _ in range(cycles):
                cycle(level)
    else:
        for _ in range(cycles):
            cycle(0)
    return U[0]


def expdef(v, k, return_jacobian=False):
    """dartel_grid.py:1619-1666: scaling and squaring from id + v / 2^k."""

    ny, nx = v.shape[1:]
    scale = 1.0 / float(2 ** k)
    cur = identity_map(nx, ny, v.dtype) + v * v.dtype.type(scale)
    if return_jacobian:
        jac = jacobian_of_displacement(v, scale)
        for _ in range(k):
            cur, jac = composition_jacobian(cur, jac, cur, jac)
        return cur, jac
    for _ in range(k):
        cur = composition(cur, cur)
    return cur


def dartel_step(source, target, v, k, params=(1.0, 1.0, 0.125, 0.0, 0.0), lmreg=1e-3, cycles=3, nit=3, code=1,
                assume_initial_nonzero=False):
    """dartel_grid.py:1420-1616 (rtype 1, no distortion weights)."""

    dt = v.dtype.type
    scale = 1.0 / float(2 ** k)
    t, jac = expdef(v, k, return_jacobian=True)
    jac = jac_div_smalldef(jac, v, scale)
    objective, rhs, hess = initialise_objfun(source, target, t, jac)
    t, jac = smalldef_jac(v, -scale)
    rhs, hess, t, jac, initial = squaring_update(rhs, hess, t, jac, k, save_transformation=code == 1)
    if code == 1:
        rjac = jac_div_smalldef(jac, v, -scale)
        robj, rrhs, rhess = initialise_objfun(target, source, t, rjac)
        objective = objective + robj
        rt, rj = smalldef_jac(v, scale)
        rrhs, rhess, _, _, initial = squaring_update(rrhs, rhess, rt, rj, k, save_transformation=False)
        rhs = rhs - rrhs
        hess = hess + rhess
    base = tuple(float(p) for p in params)
    reg = regularization_operator(v, base, rtype=1)
    rhs = rhs * dt(scale) + reg
    reg_objective = np.sum(reg * v)
    norm_rhs = np.sqrt(np.sum(rhs * rhs))
    hess = hess * dt(scale)
    solver_params = list(base)
    solver_params[4] += float(lmreg)
    u = fmg2_membrane(hess, rhs, solver_params, cycles=cycles, nit=nit, initial=initial,
                      assume_initial_nonzero=assume_initial_nonzero)
    return v - u, np.array((objective, reg_objective * dt(0.5), norm_rhs), dtype=v.dtype)


def default_dartel_parameters(loop=6, mu=0.125, lambda_=0.0, muchange=4, murate=1.25):
    """surface_warp.py:76-107."""

    values = []
    cm, cl = float(mu), float(lambda_)
    for index in range(loop):
        values.append((1.0, 1.0, cm, cl, cl / 2.0))
        if (index + 1) % muchange == 0:
            cm /= murate
        cl /= 5.0
    return tuple(values)


def solve_dartel_maps(source_maps, target_maps, loop=6, lmreg=1e-3, cycles=3, nit=3, its=3, code=1,
                      assume_initial_nonzero=False):
    """surface_warp.py:239-367 (the eager loop): each step map solved from zero velocity;
    the flow is expdef(k=10) of the LAST step's velocity."""

    params = default_dartel_parameters(loop)
    velocities, diagnostics = [], []
    for step in range(source_maps.shape[0]):
        v = np.zeros((2,) + source_maps.shape[1:], dtype=source_maps.dtype)
        metrics = []
        for index, p in enumerate(params):
            for _ in range(its):
                v, m = dartel_step(source_maps[step], target_maps[step], v, index, params=p, lmreg=lmreg,
                                   cycles=cycles, nit=nit, code=code, assume_initial_nonzero=assume_initial_nonzero)
                metrics.append(m)
        velocities.append(v)
        diagnostics.append(np.stack(metrics))
    flow = expdef(velocities[-1], 10)
    return flow, np.stack(diagnostics), velocities


def sample_field(field, x, y):
    """dartel_grid.py:590-621 (sample_field): bilinear with the boundary rule."""

    ny, nx = field.shape
    idx = interpolation_indices(x, y, nx, ny)
    return interpolate_channels(field[None], idx)[0]


def wrap_displacement(value):
    """surface_warp.py:491-497."""

    value = np.where(value >= 1.0, value - np.floor(value), value)
    value = np.where(value <= -1.0, value + np.floor(-value), value)
    value = np.where(value >= 0.5, value - 1.0, value)
    return np.where(value <= -0.5, value + 1.0, value)


def apply_flow_to_sphere(unit_sphere, flow, inverse=True):
    """surface_warp.py:500-584 with ``unit_sphere_vertices`` given (float32 input)."""

    points = np.asarray(unit_sphere, dtype=np.float32).astype(flow.dtype)
    x, y = points[:, 0], points[:, 1]
    z = np.clip(points[:, 2], -1.0, 1.0)
    theta = np.arccos(z)
    cw = -np.arctan2(x, y)
    cw = np.where(cw < 0.0, cw + 2.0 * np.pi, cw)
    u = (cw + np.pi / 2.0) / (2.0 * np.pi)
    u = np.where(u > 1.0, u - 1.0, u)
    v = theta / np.pi
    ny, nx = flow.shape[1:]
    row = np.broadcast_to(np.arange(ny, dtype=flow.dtype)[:, None], (ny, nx))
    col = np.broadcast_to(np.arange(nx, dtype=flow.dtype)[None, :], (ny, nx))
    weight = np.sin(((row + 0.5) / float(ny)) * np.pi)
    ud = wrap_displacement((flow[0] - col - 1.0) / float(nx)) * weight
    vd = wrap_displacement((flow[1] - row - 1.0) / float(ny)) * weight
    gx = u * float(nx) - 0.5
    gy = v * float(ny) - 0.5
    su = sample_field(ud, gx, gy)
    sv = sample_field(vd, gx, gy)
    if inverse:
        su, sv = -su, -sv
    u = u + su
    v = v + sv
    u = np.where(v < 0.0, u + 0.5, u)
    v = np.where(v < 0.0, -v, v)
    u = np.where(v > 1.0, u + 0.5, u)
    v = np.where(v > 1.0, 2.0 - v, v)
    u = u - np.floor(u)
    v = np.clip(v, 0.0, 1.0)
    phi = u * (2.0 * np.pi)
    th = v * np.pi
    st = np.sin(th)
    warped = np.stack((st * np.cos(phi), st * np.sin(phi), np.cos(th)), axis=-1)
    norm = np.linalg.norm(warped, axis=-1, keepdims=True)
    return warped / np.maximum(norm, np.finfo(flow.dtype).eps)


def average_xz_surfaces(x_surface, z_surface):
    """gpu_pipeline.py:248-271: blend of the x-pole and z-pole solutions."""

    xv = np.asarray(x_surface, dtype=np.float64)
    zv = np.asarray(z_surface, dtype=np.float64)
    phi_x = np.arccos(np.clip(xv[:, 0], -1.0, 1.0)) / np.pi
    phi_z = np.arccos(np.clip(zv[:, 2], -1.0, 1.0)) / np.pi
    wx = np.maximum(np.exp(-((2.0 * phi_x - 1.0) ** 2) / 0.1), 1e-19)
    wz = np.maximum(np.exp(-((2.0 * phi_z - 1.0) ** 2) / 0.1), 1e-19)
    total = wx + wz
    avg = (wx[:, None] * xv + wz[:, None] * zv) / total[:, None]
    avg = avg / np.maximum(np.linalg.norm(avg, axis=-1, keepdims=True), np.finfo(np.float64).eps)
    return avg.astype(np.float32)


# --------------------------------------------------------------------------- data-term adjoint


def data_term(v, source, target, k):
    """E(v) = 1/2 sum (S(exp(v)) - T)^2, exp = expdef's k squarings, S bilinear with the boundary rule.

    Forward of the hand-written adjoint (no reference counterpart; the
    sample is initialise_objfun's, dartel_grid.py:723-775)."""

    ny, nx = source.shape
    phi = expdef(v, k)
    idx = interpolation_indices(phi[0] - v.dtype.type(1), phi[1] - v.dtype.type(1), nx, ny)
    r = interpolate_channels(source[None], idx)[0] - target
    return v.dtype.type(0.5) * np.sum(r * r)


def data_term_gradient(v, source, target, k):
    """Exact reverse-mode derivative dE/dv of :func:`data_term` (sequential scatter order)."""

    ny, nx = source.shape
    dt = v.dtype.type
    s = dt(1.0 / 2 ** k)
    maps = [identity_map(nx, ny, v.dtype) + v * s]
    for _ in range(k):
        maps.append(composition(maps[-1], maps[-1]))
    phi = maps[-1]
    x22, y22, x12, y12, x21, y21, x11, y11, dx1, dx2, dy1, dy2 = interpolation_indices(phi[0] - dt(1), phi[1] - dt(1),
                                                                                        nx, ny)
    k22, k12, k21, k11 = source[y22, x22], source[y12, x12], source[y21, x21], source[y11, x11]
    r = ((k22 * dx2 + k12 * dx1) * dy2 + (k21 * dx2 + k11 * dx1) * dy1) - target
    abar = np.stack((r * ((k11 - k21) * dy1 + (k12 - k22) * dy2),
                     r * ((k11 * dx1 + k21 * dx2) - (k12 * dx1 + k22 * dx2))))
    periods = np.array((nx, ny), dtype=v.dtype).reshape(2, 1, 1)
    for i in reversed(range(k)):
        f = maps[i]
        x22, y22, x12, y12, x21, y21, x11, y11, dx1, dx2, dy1, dy2 = interpolation_indices(f[0] - dt(1), f[1] - dt(1),
                                                                                            nx, ny)
        cf = f - dt(1)
        c22 = cf[:, y22, x22]
        c12 = _unwrap(cf[:, y12, x12], c22, periods)
        c21 = _unwrap(cf[:, y21, x21], c22, periods)
        c11 = _unwrap(cf[:, y11, x11], c22, periods)
        dcx = (c12 - c22) * dy2 + (c11 - c21) * dy1
        dcy = (c21 * dx2 + c11 * dx1) - (c22 * dx2 + c12 * dx1)
        pbar = np.zeros_like(f)
        pbar[0] += abar[0] * dcx[0] + abar[1] * dcx[1]
        pbar[1] += abar[0] * dcy[0] + abar[1] * dcy[1]
        for ch in range(2):
            for yy, xx, weight in ((y22, x22, dx2 * dy2), (y12, x12, dx1 * dy2), (y21, x21, dx2 * dy1),
                                   (y11, x11, dx1 * dy1)):
                np.add.at(pbar[ch], (yy, xx), abar[ch] * weight)
        abar = pbar
    return abar * s


def gauss_newton_gradient(v, source, target, k):
    """The reference's DARTEL gradient of the same term (code 0): initialise_objfun at exp(v)
    pulled back by squaring_update, times 2^-k (dartel_grid.py:1420-1616 before the regulariser)."""

    s = 1.0 / 2 ** k
    t, jac = expdef(v, k, return_jacobian=True)
    jac = jac_div_smalldef(jac, v, s)
    _, rhs, hess = initialise_objfun(source, target, t, jac)
    t2, j2 = smalldef_jac(v, -s)
    rhs, _, _, _, _ = squaring_update(rhs, hess, t2, j2, k)
    return rhs * v.dtype.type(s)
