"""NumPy restatement of the reference's raw CUDA kernels (TEST INFRASTRUCTURE ONLY).

This module is part of the oracle: only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg may use it, and only as the checker.  It is
never on the product path.

Every function restates one kernel of ``src/holotomocupy/cuda_kernels.py``
(the reference keeps its CUDA C inside Python strings).  The arithmetic follows
the kernel line by line:

* the same index math (integer ``n/2`` divisions, ``floorf`` bases, the
  ``(n + ell + 2n) % 2n`` wrap of the USFFT grid, ``r[2*tz+1]`` = x shift and
  ``r[2*tz]`` = y shift);
* the same tap order (outer loop over the y tap, inner loop over the x tap);
* atomics are replaced by sequential accumulation (``np.add.at``).

The functions are written on flat buffers because the kernels receive raw
pointers.  They compute in the precision of the arrays they are given: float32
/ complex64 arrays reproduce the reference's FP32 arithmetic (up to FMA
contraction and the fast ``__expf/__cosf/__sinf`` intrinsics), float64 /
complex128 arrays give the FP64 oracle.
"""
import numpy as np


def _real_dtype(a):
    return np.float64 if a.dtype in (np.float64, np.complex128) else np.float32


# ----------------------------------------------------------------------------
# USFFT gather / scatter  -- src/holotomocupy/cuda_kernels.py:3-76
# ----------------------------------------------------------------------------
def gather(g, f, theta, m, mu, n, ntheta, nz, direction):
    """dir=0: g[ty,tz,tx] = 1/n * sum_{i1,i0} w * f[tz, iy, ix]   (cuda_kernels.py:22-71)
    dir=1: f[tz, iy, ix] += w * g[ty, tz, tx]                    (cuda_kernels.py:60-64)

    g: [ntheta, nz, n] complex (flat or shaped), f: [nz, 2n, 2n] complex.
    """
    rt = _real_dtype(g)
    gf = g.reshape(-1)
    ff = f.reshape(-1)
    twon = 2 * n
    ftwon = rt(twon)
    mu0 = rt(np.asarray(mu).reshape(-1)[0])
    PI = rt(3.141592653589793238)
    coeff0 = PI / mu0
    coeff1 = -PI * PI / mu0
    inv_twon = rt(1.0) / ftwon
    th = np.asarray(theta).reshape(-1)[:ntheta].astype(rt)
    tx = np.arange(n)
    # (tx - n / 2) / (float)n * __cosf(theta[ty])  -- integer n/2
    rho = (tx - n // 2).astype(rt) / rt(n)
    x0 = rho[None, :] * np.cos(th)[:, None]          # [ntheta, n]
    y0 = -rho[None, :] * np.sin(th)[:, None]
    base_x = np.floor(ftwon * x0).astype(np.int64) - m
    base_y = np.floor(ftwon * y0).astype(np.int64) - m
    length = 2 * m + 1
    ex = []
    for i0 in range(length):
        w0 = (base_x + i0).astype(rt) * inv_twon - x0
        ex.append(np.exp(coeff1 * w0 * w0))
    g_idx = (tx[None, None, :] + np.arange(nz)[None, :, None] * n
             + np.arange(ntheta)[:, None, None] * n * nz)   # [ntheta, nz, n]
    tz_off = (np.arange(nz) * twon * twon)[None, :, None]
    if direction == 0:
        acc = np.zeros((ntheta, nz, n), dtype=g.dtype)
    else:
        g0 = gf[g_idx]
    for i1 in range(length):
        ell1 = base_y + i1
        w1 = ell1.astype(rt) * inv_twon - y0
        ey = coeff0 * np.exp(coeff1 * w1 * w1)
        f_indy = (n + ell1 + twon) % twon
        row_off = (twon * f_indy)[:, None, :] + tz_off
        for i0 in range(length):
            w = (ex[i0] * ey)[:, None, :]
            ell0 = base_x + i0
            f_ind = ((n + ell0 + twon) % twon)[:, None, :] + row_off
            if direction == 0:
                acc += w * ff[f_ind]
            else:
                np.add.at(ff, f_ind.reshape(-1), (w * g0).reshape(-1))
    if direction == 0:
        gf[g_idx] = acc / rt(n)


# ----------------------------------------------------------------------------
# Mirror padding for the Fresnel propagator -- cuda_kernels.py:78-127
# ----------------------------------------------------------------------------
def pad_fwd(g, f, n, nz, ntheta):
    """g[tz, ty, tx] (2nz x 2n) = f[tz, tyy, txx] with the symmetric mirror map
    of cuda_kernels.py:89-94."""
    tx = np.arange(2 * n)
    ty = np.arange(2 * nz)
    txx = np.where(tx < n // 2, n // 2 - tx - 1,
                   np.where(tx >= n + n // 2, 2 * n - tx + n // 2 - 1, tx - n // 2))
    tyy = np.where(ty < nz // 2, nz // 2 - ty - 1,
                   np.where(ty >= nz + nz // 2, 2 * nz - ty + nz // 2 - 1, ty - nz // 2))
    fs = f.reshape(ntheta, nz, n)
    gs = g.reshape(-1)[: ntheta * 4 * n * nz].reshape(ntheta, 2 * nz, 2 * n)
    gs[...] = fs[:, tyy[:, None], txx[None, :]]


def pad_adj(g, f, n, nz, ntheta):
    """f[tz, ty, tx] = sum of the 4 mirror locations in g (cuda_kernels.py:113-123)."""
    tx = np.arange(n)
    ty = np.arange(nz)
    gx_c = tx + n // 2
    gx_m = np.where(tx < n // 2, n // 2 - 1 - tx, 2 * n + n // 2 - 1 - tx)
    gy_c = ty + nz // 2
    gy_m = np.where(ty < nz // 2, nz // 2 - 1 - ty, 2 * nz + nz // 2 - 1 - ty)
    gs = g.reshape(-1)[: ntheta * 4 * n * nz].reshape(ntheta, 2 * nz, 2 * n)
    v0 = gs[:, gy_c[:, None], gx_c[None, :]]
    v1 = gs[:, gy_c[:, None], gx_m[None, :]]
    v2 = gs[:, gy_m[:, None], gx_c[None, :]]
    v3 = gs[:, gy_m[:, None], gx_m[None, :]]
    f.reshape(ntheta, nz, n)[...] = v0 + v1 + v2 + v3


# ----------------------------------------------------------------------------
# Cubic B-spline basis -- cuda_kernels.py:131-159 (the x6-scaled cubic B-spline)
# ----------------------------------------------------------------------------
def bphi(t):
    a = np.abs(t)
    out = np.where((t > -2) & (t <= -1), (t + 2) ** 3, 0)
    out = np.where((t > -1) & (t <= 1), 4 - 6 * t * t + 3 * a * t * t, out)
    out = np.where((t > 1) & (t <= 2), (2 - t) ** 3, out)
    return out.astype(t.dtype)


def bdphi(t):
    a = np.abs(t)
    out = np.where((t > -2) & (t <= -1), 3 * (t + 2) ** 2, 0)
    out = np.where((t > -1) & (t <= 1), -12 * t + 9 * a * t, out)
    out = np.where((t > 1) & (t <= 2), -3 * (2 - t) ** 2, out)
    return out.astype(t.dtype)


def bd2phi(t):
    a = np.abs(t)
    out = np.where((t > -2) & (t <= -1), 6 * (t + 2), 0)
    out = np.where((t > -1) & (t <= 1), -12 + 18 * a, out)
    out = np.where((t > 1) & (t <= 2), 6 * (2 - t), out)
    return out.astype(t.dtype)


def _spline_geometry(r, mag, n, npsi, nz, nzpsi, ntheta, rt):
    """Sample positions of the shift kernels (cuda_kernels.py:177-186):
    x = (mag*(tx - n/2) - r[2tz+1] + (mag-1)/2) + npsi/2, same for y with r[2tz]."""
    rr = np.asarray(r).reshape(-1)[: 2 * ntheta].reshape(ntheta, 2).astype(rt)
    mg = np.asarray(mag).reshape(-1)[:ntheta].astype(rt)
    half = (mg - rt(1)) / rt(2)
    tx = np.arange(n)
    ty = np.arange(nz)
    x = (mg[:, None] * (tx - n // 2).astype(rt)[None, :] - rr[:, 1:2] + half[:, None]) + rt(npsi // 2)
    y = (mg[:, None] * (ty - nz // 2).astype(rt)[None, :] - rr[:, 0:1] + half[:, None]) + rt(nzpsi // 2)
    ix = np.floor(x).astype(np.int64)
    iy = np.floor(y).astype(np.int64)
    dx = x - ix.astype(rt)
    dy = y - iy.astype(rt)
    return ix, iy, dx, dy          # [ntheta, n], [ntheta, nz], ...


def _taps(ix, iy, dx, dy, npsi, nzpsi, jy, jx):
    """Index/validity of tap (jy, jx) for every output pixel: [ntheta, nz, n]."""
    ntheta = ix.shape[0]
    indy = iy + jy                                   # [ntheta, nz]
    indx = ix + jx                                   # [ntheta, n]
    valid = ((indy >= 0) & (indy < nzpsi))[:, :, None] & ((indx >= 0) & (indx < npsi))[:, None, :]
    tz_off = (np.arange(ntheta) * npsi * nzpsi)[:, None, None]
    idx = np.clip(indx, 0, npsi - 1)[:, None, :] + (np.clip(indy, 0, nzpsi - 1) * npsi)[:, :, None] + tz_off
    return idx, valid


# ----------------------------------------------------------------------------
# Shift S / S^T -- cuda_kernels.py:161-290 (complex `s`, real `sf`)
# ----------------------------------------------------------------------------
def s_kernel(g, f, r, mag, n, npsi, nz, nzpsi, ntheta, direction):
    """dir=0: g = S(f); dir=1: f += S^T(g).  g: [ntheta, nz, n], f: [ntheta, nzpsi, npsi]."""
    rt = _real_dtype(g)
    ix, iy, dx, dy = _spline_geometry(r, mag, n, npsi, nz, nzpsi, ntheta, rt)
    gf = g.reshape(-1)
    ff = f.reshape(-1)
    gsh = gf[: ntheta * nz * n].reshape(ntheta, nz, n)
    px = [bphi(dx - rt(jx)) for jx in range(-1, 3)]
    if direction == 0:
        acc = np.zeros((ntheta, nz, n), dtype=g.dtype)
    else:
        g0 = gsh.copy()
    for jy in range(-1, 3):
        pdym = bphi(dy - rt(jy))                     # [ntheta, nz]
        for jx in range(-1, 3):
            idx, valid = _taps(ix, iy, dx, dy, npsi, nzpsi, jy, jx)
            w = px[jx + 1][:, None, :] * pdym[:, :, None]
            if direction == 0:
                acc += np.where(valid, w * ff[idx], 0)
            else:
                np.add.at(ff, idx[valid], (w * g0)[valid])
    if direction == 0:
        gsh[...] = acc


def ds_kernel(res, c, c1, r, mag, Deltar, n, npsi, nz, nzpsi, ntheta):
    """First derivative (cuda_kernels.py:547-617):
    res = sum phi*phi*c1 - (dphi_x*phi_y*Drx + phi_x*dphi_y*Dry)*c."""
    rt = _real_dtype(res)
    ix, iy, dx, dy = _spline_geometry(r, mag, n, npsi, nz, nzpsi, ntheta, rt)
    dr = np.asarray(Deltar).reshape(-1)[: 2 * ntheta].reshape(ntheta, 2).astype(rt)
    drx = dr[:, 1][:, None, None]
    dry = dr[:, 0][:, None, None]
    cf = c.reshape(-1)
    c1f = c1.reshape(-1)
    px = [bphi(dx - rt(jx)) for jx in range(-1, 3)]
    dpx = [bdphi(dx - rt(jx)) for jx in range(-1, 3)]
    acc = np.zeros((ntheta, nz, n), dtype=res.dtype)
    for jy in range(-1, 3):
        dym = dy - rt(jy)
        pdym = bphi(dym)[:, :, None]
        dpdym = bdphi(dym)[:, :, None]
        for jx in range(-1, 3):
            idx, valid = _taps(ix, iy, dx, dy, npsi, nzpsi, jy, jx)
            w = dpx[jx + 1][:, None, :] * pdym * drx + dpdym * px[jx + 1][:, None, :] * dry
            w1 = px[jx + 1][:, None, :] * pdym
            acc -= np.where(valid, w * cf[idx], 0)
            acc += np.where(valid, w1 * c1f[idx], 0)
    res.reshape(-1)[: ntheta * nz * n] = acc.reshape(-1)


def d2s_kernel(res, c, c1, c2, r, mag, Deltar1, Deltar2, n, npsi, nz, nzpsi, ntheta):
    """Second derivative (cuda_kernels.py:377-459), including the reference's
    pairing of c1 with Deltar1 and c2 with Deltar2 (cuda_kernels.py:437-450)."""
    rt = _real_dtype(res)
    ix, iy, dx, dy = _spline_geometry(r, mag, n, npsi, nz, nzpsi, ntheta, rt)
    d1 = np.asarray(Deltar1).reshape(-1)[: 2 * ntheta].reshape(ntheta, 2).astype(rt)
    d2 = np.asarray(Deltar2).reshape(-1)[: 2 * ntheta].reshape(ntheta, 2).astype(rt)
    d1x, d1y = d1[:, 1][:, None, None], d1[:, 0][:, None, None]
    d2x, d2y = d2[:, 1][:, None, None], d2[:, 0][:, None, None]
    cross = d1x * d2y + d1y * d2x
    cf, c1f, c2f = c.reshape(-1), c1.reshape(-1), c2.reshape(-1)
    px = [bphi(dx - rt(jx)) for jx in range(-1, 3)]
    dpx = [bdphi(dx - rt(jx)) for jx in range(-1, 3)]
    d2px = [bd2phi(dx - rt(jx)) for jx in range(-1, 3)]
    acc = np.zeros((ntheta, nz, n), dtype=res.dtype)
    for jy in range(-1, 3):
        dym = dy - rt(jy)
        pdym = bphi(dym)[:, :, None]
        dpdym = bdphi(dym)[:, :, None]
        d2pdym = bd2phi(dym)[:, :, None]
        for jx in range(-1, 3):
            idx, valid = _taps(ix, iy, dx, dy, npsi, nzpsi, jy, jx)
            P, DP, D2P = px[jx + 1][:, None, :], dpx[jx + 1][:, None, :], d2px[jx + 1][:, None, :]
            w = D2P * pdym * d1x * d2x + DP * dpdym * cross + P * d2pdym * d1y * d2y
            w1 = DP * pdym * d1x + dpdym * P * d1y
            w2 = DP * pdym * d2x + dpdym * P * d2y
            acc += np.where(valid, w * cf[idx], 0)
            acc -= np.where(valid, w1 * c1f[idx], 0)
            acc -= np.where(valid, w2 * c2f[idx], 0)
    res.reshape(-1)[: ntheta * nz * n] = acc.reshape(-1)


def dsadj_kernel(f, dt1, dt2, c, g, r, mag, n, npsi, nz, nzpsi, ntheta):
    """Adjoint derivative (cuda_kernels.py:690-766): f += S^T(g);
    dt1 = sum -dphi_y*phi_x*c, dt2 = sum -dphi_x*phi_y*c."""
    rt = _real_dtype(g)
    ix, iy, dx, dy = _spline_geometry(r, mag, n, npsi, nz, nzpsi, ntheta, rt)
    cf = c.reshape(-1)
    ff = f.reshape(-1)
    g0 = g.reshape(-1)[: ntheta * nz * n].reshape(ntheta, nz, n).copy()
    px = [bphi(dx - rt(jx)) for jx in range(-1, 3)]
    dpx = [bdphi(dx - rt(jx)) for jx in range(-1, 3)]
    a1 = np.zeros((ntheta, nz, n), dtype=g.dtype)
    a2 = np.zeros((ntheta, nz, n), dtype=g.dtype)
    for jy in range(-1, 3):
        dym = dy - rt(jy)
        pdym = bphi(dym)[:, :, None]
        dpdym = bdphi(dym)[:, :, None]
        for jx in range(-1, 3):
            idx, valid = _taps(ix, iy, dx, dy, npsi, nzpsi, jy, jx)
            P, DP = px[jx + 1][:, None, :], dpx[jx + 1][:, None, :]
            w1 = -dpdym * P
            w2 = -DP * pdym
            cv = np.where(valid, cf[idx], 0)
            a1 += w1 * cv
            a2 += w2 * cv
            w3 = P * pdym
            np.add.at(ff, idx[valid], (w3 * g0)[valid])
    dt1.reshape(-1)[: ntheta * nz * n] = a1.reshape(-1)
    dt2.reshape(-1)[: ntheta * nz * n] = a2.reshape(-1)


# ----------------------------------------------------------------------------
# Back-projection shift -- cuda_kernels.py:294-370 (`sback`, Paganin init)
# ----------------------------------------------------------------------------
def sback_kernel(g, f, r, mag, n, npsi, nz, nzpsi, ntheta, direction):
    """dir=1: f += Sback^T(g) with the B-spline stretched by mag, phi(t / mag),
    over the taps jx in [ceil(dx - 2 mag), (int)(dx + 2 mag)) (the kernel's
    bounds: the upper one drops a tap of non-zero weight when dx + 2 mag is not
    an integer), likewise jy; dir=0: g = the matching gather.
    g: [ntheta, nz, n], f: [ntheta, nzpsi, npsi]."""
    rt = _real_dtype(g)
    mg = np.asarray(mag, dtype=rt).reshape(-1)
    mg = np.broadcast_to(mg, (ntheta,)) if mg.size == 1 else mg[:ntheta]   # one magnification for all
    ix, iy, dx, dy = _spline_geometry(r, mg, n, npsi, nz, nzpsi, ntheta, rt)
    gsh = g.reshape(-1)[: ntheta * nz * n].reshape(ntheta, nz, n)
    fsh = f.reshape(-1)[: ntheta * nzpsi * npsi].reshape(ntheta, nzpsi, npsi)
    for tz in range(ntheta):
        m0 = mg[tz]
        span = rt(2) * m0
        lox = np.ceil(dx[tz] - span).astype(np.int64)
        hix = np.trunc(dx[tz] + span).astype(np.int64)
        loy = np.ceil(dy[tz] - span).astype(np.int64)
        hiy = np.trunc(dy[tz] + span).astype(np.int64)
        acc = np.zeros((nz, n), dtype=g.dtype) if direction == 0 else None
        g0 = gsh[tz].copy() if direction != 0 else None
        ff = fsh[tz].reshape(-1)
        for jy in range(int(loy.min()), int(hiy.max())):
            indy = iy[tz] + jy
            oky = (jy >= loy) & (jy < hiy) & (indy >= 0) & (indy < nzpsi)
            pdym = bphi(((dy[tz] - rt(jy)) / m0).astype(rt))
            for jx in range(int(lox.min()), int(hix.max())):
                indx = ix[tz] + jx
                okx = (jx >= lox) & (jx < hix) & (indx >= 0) & (indx < npsi)
                w = (bphi(((dx[tz] - rt(jx)) / m0).astype(rt))[None, :] * pdym[:, None]).astype(rt)
                ok = oky[:, None] & okx[None, :]
                idx = np.clip(indy, 0, nzpsi - 1)[:, None] * npsi + np.clip(indx, 0, npsi - 1)[None, :]
                if direction == 0:
                    acc += np.where(ok, w * ff[idx], 0)
                else:
                    np.add.at(ff, idx[ok], (w * g0)[ok])
        if direction == 0:
            gsh[tz] = acc
