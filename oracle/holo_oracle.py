"""CPU oracle: NumPy restatement of holotomocupy's operator chain and BH cascade.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py`` (its CPU-baseline leg and ``--impl reference`` arm) may import
this module, and only as the checker or as the timed reference CPU
implementation.  Nothing in ``holotomocupy_b200`` imports it.

The classes restate the reference's algorithm in plain NumPy/SciPy with the
reference's discretisation (USFFT Gaussian gridding with eps=1e-3, the x6
cubic B-spline with a periodic FFT prefilter, the mirror-padded Fresnel
propagator) and with the reference's call structure (the F/dF/d2F_dF/gF
cascade of ``rec_mpi.py``).  Each method cites the reference lines it follows.
Precision is a constructor argument: ``dtype='complex128'`` is the FP64 oracle,
``dtype='complex64'`` reproduces the reference's FP32 arithmetic and is what
the CPU baseline times.

Pinning: ``tests/golden/make_golden.py`` runs the reference's own Python code
(through ``oracle/refshim.py``) on seeded inputs; ``tests/test_oracle.py``
checks this module against those fixtures.
"""
import math
import os

import numpy as np
import scipy.fft as sfft

from . import kernels_np as K

_WORKERS = int(os.environ.get("HOLO_ORACLE_WORKERS", os.cpu_count() or 1))


def _dtypes(dtype):
    cdt = np.dtype(dtype)
    if cdt == np.complex128:
        return np.complex128, np.float64
    if cdt == np.complex64:
        return np.complex64, np.float32
    raise ValueError(f"unsupported dtype {dtype}")


def fft2(x, **k):
    return sfft.fft2(x, workers=_WORKERS, **k)


def ifft2(x, **k):
    return sfft.ifft2(x, workers=_WORKERS, **k)


def reprod(a, b):
    """utils.py:96-97"""
    return a.real * b.real + a.imag * b.imag


def redot(a, b, axis=None):
    """utils.py:100-103 (accumulated in float64 here)."""
    return np.sum(reprod(a, b), axis=axis, dtype=np.float64)


class Tomo:
    """USFFT Radon transform (tomo.py:9-116)."""

    def __init__(self, n, nz, theta, mask_r, dtype="complex128"):
        self.cdt, self.rdt = _dtypes(dtype)
        rdt = self.rdt
        eps = 1e-3                                                     # tomo.py:14
        mu = -math.log(eps) / (2 * n * n)                              # tomo.py:15
        m = math.ceil(2 * n / math.pi * math.sqrt(-mu * math.log(eps) + (mu * n) ** 2 / 4))
        t = np.linspace(-1 / 2, 1 / 2, n, endpoint=False).astype(rdt)  # tomo.py:19
        dx, dy = np.meshgrid(t, t)
        phi = np.exp((mu * (n * n) * (dx * dx + dy * dy)).astype(rdt)) * (1 - n % 4)
        self.c1d = (1 - 2 * (np.arange(1, n + 1) % 2)).astype(rdt)      # tomo.py:24
        c2 = (1 - 2 * (np.arange(1, 2 * n + 1) % 2)).astype(rdt)
        self.c2d = np.outer(c2, c2)
        self.n, self.nz = n, nz
        self.ntheta = len(theta)
        self.theta = np.asarray(theta, dtype=rdt)
        if mask_r > 0:                                                  # tomo.py:34-44
            t1d = np.linspace(-1, 1, n)
            x, y = np.meshgrid(t1d, t1d)
            circ = (x ** 2 + y ** 2 < mask_r).astype("float64")
            g = np.exp(-(20 ** 2) * (x ** 2 + y ** 2))
            fcirc = np.fft.fftshift(np.fft.fft2(np.fft.fftshift(circ)))
            fg = np.fft.fftshift(np.fft.fft2(np.fft.fftshift(g)))
            mask = np.fft.fftshift(np.fft.ifft2(np.fft.fftshift(fcirc * fg))).real
            mask = (mask / np.amax(mask)).astype(rdt)
        else:
            mask = np.ones((n, n), dtype=rdt)
        self.mask = mask
        self.phi = (phi * (mask / (n * np.sqrt(n * self.ntheta)))).astype(rdt)  # tomo.py:47
        self.m = m
        self.mu = np.array([mu], dtype=rdt)

    def R(self, obj):
        """tomo.py:56-86"""
        nz = obj.shape[0]
        n = self.n
        fde = np.zeros((nz, 2 * n, 2 * n), dtype=self.cdt)
        fde[:, n // 2: 3 * n // 2, n // 2: 3 * n // 2] = obj * self.phi
        fde *= self.c2d
        fde = fft2(fde).astype(self.cdt)
        fde *= self.c2d
        sino = np.zeros((self.ntheta, nz, n), dtype=self.cdt)
        K.gather(sino, fde, self.theta, self.m, self.mu, n, self.ntheta, nz, 0)
        sino *= self.c1d
        sino = sfft.ifft(sino, workers=_WORKERS).astype(self.cdt)
        sino *= self.c1d
        res = sino / 4
        if np.isrealobj(obj):
            res = res.real
        return np.ascontiguousarray(res)

    def RT(self, data):
        """tomo.py:88-116"""
        nz = data.shape[1]
        n = self.n
        sino = (data * self.c1d).astype(self.cdt)
        sino = sfft.fft(sino, workers=_WORKERS).astype(self.cdt)
        sino *= self.c1d
        fde = np.zeros((nz, 2 * n, 2 * n), dtype=self.cdt)
        K.gather(sino, fde, self.theta, self.m, self.mu, n, self.ntheta, nz, 1)
        fde *= self.c2d
        fde = ifft2(fde).astype(self.cdt)
        fde *= self.c2d
        res = fde[:, n // 2: 3 * n // 2, n // 2: 3 * n // 2] * self.phi
        if np.isrealobj(data):
            res = res.real
        return np.ascontiguousarray(res)

    def filter_sino(self, data, filter_name):
        """tomo.py:118-161"""
        n = self.n
        f = np.fft.fftfreq(n).astype(self.rdt)
        af = np.abs(f) * 4 * n
        if filter_name == "ramp":
            h = af
        elif filter_name == "shepp":
            h = af * np.sinc(f)
        elif filter_name == "parzen":
            u = 2 * af
            w = np.where(u <= 0.5, 1 - 6 * u ** 2 + 6 * u ** 3, 2 * (1 - u) ** 3)
            h = af * w
        else:
            raise ValueError(f"Unknown filter '{filter_name}'. Choose: ramp, shepp, parzen.")
        res = sfft.ifft(sfft.fft(data, axis=-1) * h, axis=-1)
        return res if np.iscomplexobj(data) else res.real

    def fbp(self, data, filter_name="ramp"):
        """tomo.py:163-183"""
        norm_const = np.sqrt(self.n / self.ntheta)
        return self.RT(self.filter_sino(data, filter_name)) * norm_const

    def rec_tomo(self, d, niter=1):
        """tomo.py:185-210: conjugate gradients on ||R u - d||^2 from u = 0."""
        u = np.zeros((d.shape[1], self.n, self.n), dtype=d.dtype)
        Ru = self.R(u)
        eta = Reta = None
        for k in range(niter):
            grad = self.RT(2 * (Ru - d))
            Rgrad = self.R(grad)
            if k == 0:
                eta, Reta = -grad, -Rgrad
            else:
                beta = redot(Rgrad, Reta) / redot(Reta, Reta)
                eta = beta * eta - grad
                Reta = beta * Reta - Rgrad
            alpha = -redot(grad, eta) / (2 * redot(Reta, Reta))
            u = u + alpha * eta
            Ru = Ru + alpha * Reta
        return u


class Shift:
    """Cubic B-spline shift (shift.py:15-221)."""

    def __init__(self, n, npsi, nz, nzpsi, obj_dtype, dtype="complex128"):
        self.cdt, self.rdt = _dtypes(dtype)
        self.n, self.npsi, self.nz, self.nzpsi = n, npsi, nz, nzpsi
        self.obj_dtype = obj_dtype
        self.odt = self.cdt if obj_dtype == "complex64" else self.rdt
        rdt = self.rdt
        x = np.linspace(-1 / 2, 1 / 2 - 1 / npsi, npsi).astype(rdt)    # shift.py:26-30
        y = np.linspace(-1 / 2, 1 / 2 - 1 / nzpsi, nzpsi).astype(rdt)
        divx = (4 + 2 * 1 * np.cos(2 * np.pi * x)).astype(rdt)
        divy = (4 + 2 * 1 * np.cos(2 * np.pi * y)).astype(rdt)
        self.ifB3 = (1 / np.fft.fftshift(np.outer(divy, divx), axes=(-1, -2))).astype(rdt)

    def coeff(self, psi):
        """shift.py:74-82"""
        out = ifft2(fft2(psi) * self.ifB3).astype(self.cdt)
        if self.obj_dtype == "float32":
            out = out.real
        return out

    def S(self, c, r, m):
        """shift.py:102-111 / 159-168"""
        nt = c.shape[0]
        out = np.zeros((nt, self.nz, self.n), dtype=self.odt)
        K.s_kernel(out, np.ascontiguousarray(c), r, m, self.n, self.npsi, self.nz, self.nzpsi, nt, 0)
        return out

    curlySc = S

    def Sadj(self, spsi, r, m):
        """shift.py:113-122"""
        nt = spsi.shape[0]
        c = np.zeros((nt, self.nzpsi, self.npsi), dtype=self.odt)
        K.s_kernel(np.ascontiguousarray(spsi), c, r, m, self.n, self.npsi, self.nz, self.nzpsi, nt, 1)
        return c

    def curlyS(self, psi, r, m):
        """shift.py:128-132"""
        return self.S(self.coeff(psi), r, m)

    @staticmethod
    def phi(t):
        """shift.py:54-59 (the host-side x6 cubic B-spline)"""
        return ((-2 < t) * (t <= -1) * (t + 2) ** 3 + (-1 < t) * (t <= 1) * (4 - 6 * t ** 2 + 3 * t ** 3 * np.sign(t))
                + (1 < t) * (t <= 2) * (2 - t) ** 3)

    def coeffback(self, psi, m):
        """shift.py:84-96: the prefilter of the B-spline stretched by m (one
        magnification: the first if an array is given), periodic, in the
        Fourier domain."""
        rdt = self.rdt
        m = float(np.asarray(m).reshape(-1)[0])
        x = np.linspace(-1 / 2, 1 / 2 - 1 / self.npsi, self.npsi).astype(rdt)
        y = np.linspace(-1 / 2, 1 / 2 - 1 / self.nzpsi, self.nzpsi).astype(rdt)
        dx = self.phi(rdt(0))
        dy = self.phi(rdt(0))
        for k in range(1, 5):
            pk = self.phi(rdt(k / m))
            dx = (dx + 2 * pk * np.cos(2 * np.pi * k * x)).astype(rdt)
            dy = (dy + 2 * pk * np.cos(2 * np.pi * k * y)).astype(rdt)
        ifb = (1 / np.fft.fftshift(np.outer(dy, dx), axes=(-1, -2))).astype(rdt)
        return ifft2(fft2(psi) * ifb).astype(self.cdt)

    def Sback(self, spsi, r, m):
        """shift.py:138-148 + sback (cuda_kernels.py:294-370): [B, nz, n] ->
        [B, nzpsi, npsi] (complex) with the B-spline stretched by m."""
        nt = spsi.shape[0]
        c = np.zeros((nt, self.nzpsi, self.npsi), dtype=self.cdt)
        K.sback_kernel(np.ascontiguousarray(spsi).astype(self.cdt), c, r, m, self.n, self.npsi, self.nz,
                       self.nzpsi, nt, 1)
        return c

    def curlySback(self, psi, r, m):
        """shift.py:152-153"""
        return self.coeffback(self.Sback(psi, r, m), m)

    def dcurlySc(self, c, r, m, c1, Deltar):
        """shift.py:170-183"""
        nt = c.shape[0]
        res = np.zeros((nt, self.nz, self.n), dtype=self.odt)
        K.ds_kernel(res, np.ascontiguousarray(c), np.ascontiguousarray(c1), r, m, Deltar,
                    self.n, self.npsi, self.nz, self.nzpsi, nt)
        return res

    def dcurlySadjc(self, c, r, m, Deltaphi):
        """shift.py:185-204"""
        nt = c.shape[0]
        out1 = np.zeros((nt, self.nzpsi, self.npsi), dtype=self.odt)
        dt1 = np.zeros(Deltaphi.shape, dtype=self.odt)
        dt2 = np.zeros(Deltaphi.shape, dtype=self.odt)
        K.dsadj_kernel(out1, dt1, dt2, np.ascontiguousarray(c), np.ascontiguousarray(Deltaphi),
                       r, m, self.n, self.npsi, self.nz, self.nzpsi, nt)
        out2 = np.zeros((nt, 2), dtype=self.rdt)
        out2[:, 0] = redot(Deltaphi, dt1, axis=(1, 2))
        out2[:, 1] = redot(Deltaphi, dt2, axis=(1, 2))
        return [out1, out2]

    def d2curlySc(self, c, r, m, c1, Deltar1, c2, Deltar2):
        """shift.py:206-221"""
        nt = c.shape[0]
        res = np.zeros((nt, self.nz, self.n), dtype=self.odt)
        K.d2s_kernel(res, np.ascontiguousarray(c), np.ascontiguousarray(c1), np.ascontiguousarray(c2),
                     r, m, Deltar1, Deltar2, self.n, self.npsi, self.nz, self.nzpsi, nt)
        return res


def fresnel_kernel(n, nz, wavelength, voxelsize, distance, table="exact"):
    """propagation.py:20-28: fker[j] = exp(-1j*pi*lambda*z_j*(fx^2+fy^2)) / (4*n*nz)
    on the 2nz x 2n fftfreq grid.  table='ref32' repeats the reference's FP32
    table arithmetic (float32 frequencies and f2, complex64 storage);
    table='exact' evaluates the same formula in float64."""
    ndist = len(distance)
    if table == "ref32":
        fx = np.fft.fftfreq(2 * n, d=voxelsize).astype("float32")
        fy = np.fft.fftfreq(2 * nz, d=voxelsize).astype("float32")
        fx, fy = np.meshgrid(fx, fy)
        f2 = fx ** 2 + fy ** 2
        out = np.empty((ndist, 2 * nz, 2 * n), dtype="complex64")
        for j in range(ndist):
            out[j] = np.exp(-1j * np.pi * wavelength * np.float64(distance[j]) * f2) / float(4 * n * nz)
        return out
    fx = np.fft.fftfreq(2 * n, d=voxelsize)
    fy = np.fft.fftfreq(2 * nz, d=voxelsize)
    fx, fy = np.meshgrid(fx, fy)
    f2 = fx ** 2 + fy ** 2
    return np.stack([np.exp(-1j * np.pi * wavelength * distance[j] * f2) / (4 * n * nz)
                     for j in range(ndist)])


class Propagation:
    """Fresnel propagator (propagation.py:11-112)."""

    def __init__(self, n, nz, ntheta, ndist, wavelength, voxelsize, distance,
                 dtype="complex128", table=None):
        self.cdt, self.rdt = _dtypes(dtype)
        self.n, self.nz = n, nz
        if table is None:
            table = "exact" if self.cdt == np.complex128 else "ref32"
        self.fker = fresnel_kernel(n, nz, wavelength, voxelsize, distance, table).astype(self.cdt)

    def _conv(self, big, j, conj):
        h = np.conj(self.fker[j]) if conj else self.fker[j]
        return ifft2(fft2(big) * h, norm="forward").astype(self.cdt)

    def D(self, psi, j):
        """propagation.py:70-89"""
        added = psi.ndim == 2
        if added:
            psi = psi[None]
        nt = psi.shape[0]
        big = np.empty((nt, 2 * self.nz, 2 * self.n), dtype=self.cdt)
        K.pad_fwd(big, np.ascontiguousarray(psi, dtype=self.cdt), self.n, self.nz, nt)
        big = self._conv(big, j, False)
        res = big[:, self.nz // 2: -self.nz // 2, self.n // 2: -self.n // 2].copy()
        return res[0] if added else res

    def DT(self, psi, j):
        """propagation.py:91-112"""
        added = psi.ndim == 2
        if added:
            psi = psi[None]
        nt = psi.shape[0]
        big = np.zeros((nt, 2 * self.nz, 2 * self.n), dtype=self.cdt)
        big[:, self.nz // 2: -self.nz // 2, self.n // 2: -self.n // 2] = psi
        big = self._conv(big, j, True)
        res = np.zeros((nt, self.nz, self.n), dtype=self.cdt)
        K.pad_adj(big, res, self.n, self.nz, nt)
        return res[0] if added else res


class Rec:
    """The BH data-fidelity cascade and solver loop of rec_mpi.py (single rank).

    ``args`` carries the reference's keys (rec_mpi.py:22-26).  Optional keys
    ``distance`` (metres, per distance), ``wavelength``, ``voxelsize`` and
    ``norm_magnifications`` override the values derived from z1 and the
    focus distance (rec_mpi.py:55-60), which the synthetic workloads use to pass
    distances directly with unit magnification.
    """

    def __init__(self, args, dtype="complex128"):
        for k, v in vars(args).items():
            setattr(self, k, v)
        self.dtype = dtype
        self.cdt, self.rdt = _dtypes(dtype)
        if not hasattr(self, "lam_laplacian"):
            self.lam_laplacian = 0
        if getattr(self, "distance", None) is None:                   # rec_mpi.py:55-60
            wavelength = 1.24e-09 / self.energy
            z2 = self.focustodetectordistance - self.z1
            magnifications = self.focustodetectordistance / self.z1
            norm_magnifications = magnifications / magnifications[0]
            distance = (self.z1 * z2) / self.focustodetectordistance * norm_magnifications ** 2
            voxelsize = self.detector_pixelsize / magnifications[0]
        else:
            wavelength, voxelsize, distance = self.wavelength, self.voxelsize, self.distance
            norm_magnifications = getattr(self, "norm_magnifications", np.ones(self.ndist))
        self.rho_sq = {"obj": args.rho[0] ** 2, "prb": args.rho[1] ** 2, "pos": args.rho[2] ** 2}
        self.cl_tomo = Tomo(self.nobj, self.nzobj, self.theta, self.mask, dtype)
        self.cl_prop = Propagation(self.n, self.nz, self.ntheta, self.ndist, wavelength,
                                   voxelsize, distance, dtype)
        self.cl_shift = Shift(self.n, self.nobj, self.nz, self.nzobj, self.obj_dtype, dtype)
        self.norm_const = np.sqrt(self.nobj / self.ntheta)            # rec_mpi.py:88
        self.norm_magnifications = np.asarray(norm_magnifications, dtype=np.float64)
        self.data_size = self.ntheta * self.ndist * self.nz * self.n  # rec_mpi.py:91
        self.prb_size = self.ndist * self.nz * self.n
        self.obj_size = self.nzobj * self.nobj ** 2
        self.odt = self.cdt if self.obj_dtype == "complex64" else self.rdt
        # rec_mpi.py:135-136: shrink_nd and eff_demagnifications are ONE array,
        # zero until BH() fills it (rec_mpi.py:146); a forward model evaluated
        # before BH() (gen_sqrt_data) therefore samples with magnification 0.
        self.shrink_nd = np.zeros((self.ntheta, self.ndist), dtype=self.rdt)
        self.eff_demagnifications = self.shrink_nd
        self.F = [self.F0, self.F1, self.F2, self.F3]
        self.gF = [self.gF0, self.gF1, self.gF2, self.gF3]
        self.dF = [self.dF0, self.dF1, self.dF2, self.dF3]
        self.d2F_dF = [self.d2F_dF0, self.d2F_dF1, self.d2F_dF2, self.d2F_dF3]
        self.alloc_arrays()

    def alloc_arrays(self):
        """rec_mpi.py:105-136"""
        prb_shape = (self.ndist, self.nz, self.n)
        self.vars = {
            "obj": np.zeros((self.nzobj, self.nobj, self.nobj), self.odt),
            "pos": np.zeros((self.ntheta, self.ndist, 2), self.rdt),
            "prb": np.zeros(prb_shape, self.cdt),
            "proj": np.zeros((self.ntheta, self.nzobj, self.nobj), self.odt),
        }
        self.data = np.zeros((self.ntheta, self.ndist, self.nz, self.n), self.rdt)
        self.ref = np.zeros(prb_shape, self.rdt)
        self.grads, self.etas = {}, {}
        for ge in (self.grads, self.etas):
            ge["obj"] = np.zeros((self.nzobj, self.nobj, self.nobj), self.odt)
            ge["pos"] = np.zeros((self.ntheta, self.ndist, 2), self.rdt)
            ge["proj"] = np.zeros((self.ntheta, self.nzobj, self.nobj), self.odt)
            ge["prb"] = np.zeros(prb_shape, self.cdt)

    # -------------------------------------------------------------- cascade
    def F0(self, x, d):
        """rec_mpi.py:517-527"""
        t = np.abs(x) - d
        return np.sum(t * t, dtype=np.float64) / self.data_size

    def dF0(self, x, y, d, return_x=False):
        """rec_mpi.py:529-537"""
        return 2 / self.data_size * redot(x - d * (x / np.abs(x)), y)

    def d2F_dF0(self, x, y, z, w, d):
        """rec_mpi.py:539-553"""
        absval = np.abs(x)
        l0 = x / absval
        d0 = d / absval
        v = (1 - d0) * reprod(y, z) + d0 * reprod(l0, y) * reprod(l0, z)
        if w is not None:
            v = v + reprod(x - d * l0, w)
        return 2 / self.data_size * np.sum(v, dtype=np.float64)

    def gF0(self, x, y):
        """rec_mpi.py:555-569"""
        for i in range(1, 4)[::-1]:
            x = self.F[i](x)
        scale = self.rdt(2 / self.data_size)
        return scale * (x - y * (x / np.abs(x)))

    def F1(self, x):
        """rec_mpi.py:572-582"""
        x11, x12 = x
        x0 = np.empty((x12.shape[0], self.ndist, self.nz, self.n), self.cdt)
        for j in range(self.ndist):
            x0[:, j] = self.cl_prop.D(x11[j] * x12[:, j], j)
        return x0

    def dF1(self, x, y, return_x=True):
        """rec_mpi.py:584-600"""
        x11, x12 = x
        y11, y12 = y
        y0 = (y11[None] * x12 + x11[None] * y12).astype(self.cdt)
        for j in range(self.ndist):
            y0[:, j] = self.cl_prop.D(y0[:, j], j)
        if return_x:
            x0 = (x11[None] * x12).astype(self.cdt)
            for j in range(self.ndist):
                x0[:, j] = self.cl_prop.D(x0[:, j], j)
            return x0, y0
        return y0

    def d2F_dF1(self, x, y, z, w):
        """rec_mpi.py:602-624"""
        x11, x12 = x
        y11, y12 = y
        z11, z12 = z
        w11, w12 = w
        if y12 is z12:
            y0 = 2 * y11[None] * y12
        else:
            y0 = y11[None] * z12 + z11[None] * y12
        if w11 is not None:
            y0 = y0 + w11[None] * x12
        if w12 is not None:
            y0 = y0 + x11[None] * w12
        y0 = y0.astype(self.cdt)
        for j in range(self.ndist):
            y0[:, j] = self.cl_prop.D(y0[:, j], j)
        return y0

    def gF1(self, x, y):
        """rec_mpi.py:626-643"""
        y0 = y
        for i in range(2, 4)[::-1]:
            x = self.F[i](x)
        x11, x12 = x
        y12 = np.empty((y0.shape[0], self.ndist, self.nz, self.n), self.cdt)
        for j in range(self.ndist):
            y12[:, j] = self.cl_prop.DT(y0[:, j], j)
        y11 = np.sum(y12 * np.conj(x12), axis=0)
        y12 = y12 * np.conj(x11[None])
        return y11, y12

    def F2(self, x):
        """rec_mpi.py:646-658"""
        x21, x22 = x
        return x21, np.exp(1j * x22).astype(self.cdt)

    def dF2(self, x, y, return_x=True):
        """rec_mpi.py:660-678"""
        x21, x22 = x
        y21, y22 = y
        x12 = np.exp(1j * x22).astype(self.cdt)
        y12 = x12 * 1j * y22
        return ([x21, x12], [y21, y12]) if return_x else [y21, y12]

    def d2F_dF2(self, x, y, z, w):
        """rec_mpi.py:682-702"""
        x21, x22 = x
        y21, y22 = y
        z21, z22 = z
        w21, w22 = w
        e = np.exp(1j * x22)
        y12 = e * (-y22 * z22)
        if w22 is not None:
            y12 = y12 + e * 1j * w22
        return [w21, y12.astype(self.cdt)]

    def gF2(self, x, y):
        """rec_mpi.py:704-724"""
        y11, y12 = y
        x = self.F3(x)
        x21, x22 = x
        y22 = (-1j) * y12 * np.conj(np.exp(1j * x22))
        y22 = y22.real if self.obj_dtype == "float32" else y22.astype(self.cdt)
        return [y11, y22]

    def F3(self, x):
        """rec_mpi.py:727-739"""
        x31, x32, x33 = x
        x22 = np.empty((len(x33), self.ndist, self.nz, self.n), self.odt)
        c = self.cl_shift.coeff(x32)
        for k in range(self.ndist):
            x22[:, k] = self.cl_shift.curlySc(c, x33[:, k], self.eff_demagnifications[:, k])
        return [x31, x22]

    def dF3(self, x, y, return_x=True):
        """rec_mpi.py:741-761"""
        x31, x32, x33 = x
        y31, y32, y33 = y
        y22 = np.zeros((len(y32), self.ndist, self.nz, self.n), self.odt)
        c = self.cl_shift.coeff(x32)
        c1 = self.cl_shift.coeff(y32)
        if return_x:
            x22 = np.zeros((len(x32), self.ndist, self.nz, self.n), self.odt)
            for k in range(self.ndist):
                x22[:, k] = self.cl_shift.curlySc(c, x33[:, k], self.eff_demagnifications[:, k])
        for k in range(self.ndist):
            y22[:, k] = self.cl_shift.dcurlySc(c, x33[:, k], self.eff_demagnifications[:, k], c1, y33[:, k])
        return ([x31, x22], [y31, y22]) if return_x else [y31, y22]

    def d2F_dF3(self, x, y, z, w):
        """rec_mpi.py:765-788"""
        x31, x32, x33 = x
        y31, y32, y33 = y
        z31, z32, z33 = z
        w31, w32, w33 = w
        y22 = np.zeros((len(y32), self.ndist, self.nz, self.n), self.odt)
        c = self.cl_shift.coeff(x32)
        cy = self.cl_shift.coeff(y32)
        cz = self.cl_shift.coeff(z32)
        for k in range(self.ndist):
            y22[:, k] = self.cl_shift.d2curlySc(c, x33[:, k], self.eff_demagnifications[:, k],
                                                cy, y33[:, k], cz, z33[:, k])
        if w32 is not None:
            cy = self.cl_shift.coeff(w32)
            for k in range(self.ndist):
                y22[:, k] += self.cl_shift.dcurlySc(c, x33[:, k], self.eff_demagnifications[:, k], cy, w33[:, k])
        return [w31, y22]

    def gF3(self, x, y):
        """rec_mpi.py:790-813"""
        y21, y22 = y
        x31, x32, x33 = x
        y32 = np.zeros((y22.shape[0], self.nzobj, self.nobj), self.odt)
        y33 = np.empty((y22.shape[0], self.ndist, 2), self.rdt)
        c = self.cl_shift.coeff(x32)
        for k in range(self.ndist):
            dpsi, dr = self.cl_shift.dcurlySadjc(c, x33[:, k], self.eff_demagnifications[:, k],
                                                 np.ascontiguousarray(y22[:, k]))
            y32 += dpsi
            y33[:, k] = dr
        y32 = self.cl_shift.coeff(y32)
        return [y21, y32, y33]

    # ------------------------------------------------------------- solver
    def fwd_tomo(self, obj):
        """rec_mpi.py:498-507"""
        return self.cl_tomo.R(obj)

    def hessian_cascade(self, vars, grads, etas):
        """rec_mpi.py:250-303"""
        x = [vars["prb"], vars["proj"], vars["pos"]]
        y = [grads["prb"], grads["proj"], grads["pos"]]
        z = [etas["prb"], etas["proj"], etas["pos"]]
        w = [None, None, None]
        y_is_z = y[0] is z[0]
        for i in range(1, len(self.F))[::-1]:
            w = self.d2F_dF[i](x, y, z, w)
            fx, y = self.dF[i](x, y)
            if y_is_z:
                z = y
            else:
                z = self.dF[i](x, z, return_x=False)
            x = fx
        return self.d2F_dF[0](x, y, z, w, self.data)

    def hessian(self, vars, grads, etas):
        """rec_mpi.py:234-248"""
        w = self.hessian_cascade(vars, grads, etas)
        if self.lam_prbfit != 0:
            w += self.hessian_prbfit(vars["prb"], grads["prb"], etas["prb"])
        return w + self.hessian_laplacian(grads["obj"])

    def gradients_cascade(self, vars, grads):
        """rec_mpi.py:327-353"""
        x = [vars["prb"], vars["proj"], vars["pos"]]
        y = self.data
        for i in range(len(self.gF)):
            y = self.gF[i](x, y)
        grads["prb"][:] = y[0] * self.rho_sq["prb"]
        grads["proj"][:] = y[1] * self.rho_sq["obj"]
        grads["pos"][:] = y[2] * self.rho_sq["pos"]

    def gradients(self, vars, grads):
        """rec_mpi.py:305-325"""
        self.gradients_cascade(vars, grads)
        grads["obj"][:] = self.cl_tomo.RT(grads["proj"])               # gF4, rec_mpi.py:355-362
        self.gradient_laplacian(grads["obj"])
        if self.lam_prbfit != 0:
            self.gradient_prbfit(grads["prb"], vars["prb"])

    # ------------------------------------------ 3-D Laplacian regulariser
    # rec_mpi.py:402-496: the 7-point Laplacian, periodic in y and x, applied
    # to the object zero-padded by two slices in z.  The gradient and the
    # Hessian form apply it twice (the inner Laplacian also on the two ghost
    # slices next to the object), the energy once (object slices only).
    @staticmethod
    def _lap(a, b, c):
        """rec_mpi.py:432-436"""
        return (a + c + np.roll(b, -1, axis=1) + np.roll(b, 1, axis=1) + np.roll(b, -1, axis=2)
                + np.roll(b, 1, axis=2) - 6 * b)

    def _biharmonic(self, u):
        p = np.zeros((u.shape[0] + 4,) + u.shape[1:], u.dtype)
        p[2:-2] = u
        lm = self._lap(p[:-4], p[1:-3], p[2:-2])
        lz = self._lap(p[1:-3], p[2:-2], p[3:-1])
        lp = self._lap(p[2:-2], p[3:-1], p[4:])
        return self._lap(lm, lz, lp)

    def gradient_laplacian(self, grad_obj):
        """rec_mpi.py:419-442: grad_obj += 2 lam / obj_size (lap lap) vars obj."""
        if self.lam_laplacian == 0:
            return
        grad_obj += (2.0 * self.lam_laplacian / self.obj_size) * self._biharmonic(self.vars["obj"])

    def hessian_laplacian(self, dobj1):
        """rec_mpi.py:444-470: 2 lam / obj_size Re<dobj1, (lap lap) etas obj> (always the
        current etas obj, whatever directions the caller's Hessian form has)."""
        if self.lam_laplacian == 0:
            return 0.0
        return 2.0 * self.lam_laplacian / self.obj_size * redot(dobj1, self._biharmonic(self.etas["obj"]))

    def _lap_energy_local(self):
        """rec_mpi.py:472-496: lam / obj_size ||lap vars obj||^2 over the object slices."""
        if self.lam_laplacian == 0:
            return 0.0
        p = np.zeros((self.nzobj + 4, self.nobj, self.nobj), self.vars["obj"].dtype)
        p[2:-2] = self.vars["obj"]
        lap = self._lap(p[1:-3], p[2:-2], p[3:-1])
        return self.lam_laplacian / self.obj_size * redot(lap, lap)

    def gradient_prbfit(self, grad_prb, prb):
        """rec_mpi.py:365-377"""
        for j in range(self.ndist):
            tmp = self.cl_prop.D(prb[j: j + 1], j)
            td = self.ref[j: j + 1] * (tmp / np.abs(tmp))
            td = self.lam_prbfit / self.prb_size * self.cl_prop.DT(2 * (tmp - td), j)
            grad_prb[j: j + 1] += td * self.rho_sq["prb"]

    def hessian_prbfit(self, prb, dprb1, dprb2):
        """rec_mpi.py:379-398"""
        out = 0.0
        for j in range(self.ndist):
            Dprb = self.cl_prop.D(prb[j: j + 1], j)
            Dd1 = self.cl_prop.D(dprb1[j: j + 1], j)
            Dd2 = self.cl_prop.D(dprb2[j: j + 1], j)
            l0 = Dprb / np.abs(Dprb)
            d0 = self.ref[j: j + 1] / np.abs(Dprb)
            v1 = np.sum((1 - d0) * reprod(Dd1, Dd2), dtype=np.float64)
            v2 = np.sum(d0 * reprod(l0, Dd1) * reprod(l0, Dd2), dtype=np.float64)
            out += 2 * (v1 + v2)
        return self.lam_prbfit * out / self.prb_size

    def min(self, prb, obj, pos, proj):
        """rec_mpi.py:815-835 (data term + probe-fit term)"""
        y = [prb, proj, pos]
        for i in range(1, len(self.F))[::-1]:
            y = self.F[i](y)
        out = self.F0(y, self.data)
        for j in range(self.ndist):
            if self.lam_prbfit != 0:
                Dprb = self.cl_prop.D(prb[j: j + 1], j)[0]
                out += self.lam_prbfit / self.prb_size * np.linalg.norm(np.abs(Dprb) - self.ref[j]) ** 2
        return out + self._lap_energy_local()

    def gen_sqrt_data(self, vars, out):
        """rec_mpi.py:882-897"""
        obj = vars["obj"] / self.norm_const
        vars["proj"][:] = self.fwd_tomo(obj)
        y = [vars["prb"], vars["proj"], vars["pos"]]
        for i in range(1, len(self.F))[::-1]:
            y = self.F[i](y)
        out[:] = np.abs(y)

    def gen_sqrt_ref(self, prb, out):
        """rec_mpi.py:899-902"""
        for j in range(self.ndist):
            out[j] = np.abs(self.cl_prop.D(prb[j: j + 1], j)[0])

    def BH(self, niter=None, record=None):
        """rec_mpi.py:138-232.  ``record`` (a list) receives per-iteration
        (iteration, alpha, beta) for parity checks."""
        vars, grads, etas = self.vars, self.grads, self.etas
        self.eff_demagnifications[:] = (1 + self.shrink_nd) / self.norm_magnifications[None, :]
        vars["obj"] /= self.norm_const
        if self.start_iter == 0:
            vars["obj"] *= self.cl_tomo.mask
        vars["proj"][:] = self.fwd_tomo(vars["obj"])
        niter = self.niter if niter is None else niter
        for i in range(self.start_iter, niter):
            self.gradients(vars, grads)
            grads["proj"][:] = self.fwd_tomo(grads["obj"])
            if i == self.start_iter:
                beta = 0.0
            else:
                top = self.hessian(vars, grads, etas)
                bottom = self.hessian(vars, etas, etas)
                beta = top / bottom
            top = 0.0
            for v in ["obj", "pos"]:
                etas[v][:] = beta * etas[v] - grads[v]
                top -= redot(grads[v], etas[v]) / self.rho_sq[v]
            etas["prb"][:] = beta * etas["prb"] - grads["prb"]
            top -= redot(grads["prb"], etas["prb"]) / self.rho_sq["prb"]
            etas["proj"][:] = beta * etas["proj"] - grads["proj"]
            bottom = self.hessian(vars, etas, etas)
            alpha = top / bottom
            for v in ["obj", "prb", "pos", "proj"]:
                vars[v][:] = vars[v] + alpha * etas[v]
            if record is not None:
                record.append((i, float(alpha), float(beta)))
        vars["obj"] *= self.norm_const
        return vars
