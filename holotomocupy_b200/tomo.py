"""USFFT Radon transform on the B200 (drop-in for holotomocupy's Tomo).

Reference: ``src/holotomocupy/tomo.py:9-210``.  Same constructor
``Tomo(n, nz, theta, mask_r)``, same ``R`` / ``RT`` / ``fbp`` / ``rec_tomo``
and attributes ``n``, ``ntheta``, ``theta``, ``mask``, ``pars`` (CUDA torch
tensors in place of CuPy arrays).  ``nz`` is the slice capacity of one call,
as in the reference (its buffers are sized by it).
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib


def usfft_params(n):
    """eps, mu and the gridding half-width m of tomo.py:14-16."""
    eps = 1e-3
    mu = -math.log(eps) / (2 * n * n)
    m = math.ceil(2 * n / math.pi * math.sqrt(-mu * math.log(eps) + (mu * n) ** 2 / 4))
    return eps, mu, m


def support_mask(n, mask_r):
    """Gaussian-smoothed disc of tomo.py:34-44 (float32 [n, n]), or None."""
    if not mask_r > 0:
        return None
    t1d = np.linspace(-1, 1, n)
    x, y = np.meshgrid(t1d, t1d)
    circ = (x ** 2 + y ** 2 < mask_r).astype("float32")
    g = np.exp(-(20 ** 2) * (x ** 2 + y ** 2))
    fcirc = np.fft.fftshift(np.fft.fft2(np.fft.fftshift(circ)))
    fg = np.fft.fftshift(np.fft.fft2(np.fft.fftshift(g)))
    mask = np.fft.fftshift(np.fft.ifft2(np.fft.fftshift(fcirc * fg))).real.astype("float32")
    mask /= np.amax(mask)
    return mask


def deapodisation(n, ntheta, mask):
    """phi of tomo.py:19-21, 47 with the reference's float32/float64 steps."""
    _, mu, _ = usfft_params(n)
    t = np.linspace(-1 / 2, 1 / 2, n, endpoint=False).astype("float32")
    dx, dy = np.meshgrid(t, t)
    phi = np.exp((mu * (n * n) * (dx * dx + dy * dy)).astype("float32")) * np.float32(1 - n % 4)
    factor = (1.0 if mask is None else mask.astype(np.float64)) / (n * np.sqrt(n * ntheta))
    return (phi.astype(np.float64) * factor).astype("float32")


class Tomo:
    """Functionality for Radon transforms (tomo.py:9)."""

    def __init__(self, n, nz, theta, mask_r, device=None, norm_ntheta=None):
        """``norm_ntheta`` (default: the number of angles) is the angle count
        in the 1/(n sqrt(n ntheta)) scaling of R; a Tomo over a chunk of a
        larger angle set passes the full count so that its R is a slice of
        the full R."""
        self.n = n
        self._nz = nz
        theta = np.asarray(theta.cpu() if isinstance(theta, torch.Tensor) else theta).astype("float32")
        self.ntheta = len(theta)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.theta = torch.from_numpy(theta).to(self.device)
        mask = support_mask(n, mask_r)
        self.mask = 1.0 if mask is None else torch.from_numpy(mask).to(self.device)
        phi = deapodisation(n, self.ntheta if norm_ntheta is None else norm_ntheta, mask)
        _, mu, m = usfft_params(n)
        self._phi = phi
        self.pars = (m, torch.tensor([mu], dtype=torch.float32, device=self.device),
                     torch.from_numpy(phi).to(self.device))
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("ht_tomo_create", n, nz, self.ntheta, theta.ctypes.data_as(ctypes.c_void_p),
                      phi.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h))
        self._h = h
        self._filters = {}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().ht_tomo_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------ slabs of object slices
    # The handle's workspace holds `nz` slices (the constructor's nz); a taller
    # volume is transformed slab by slab, each slab's sinogram rows written in
    # place inside the full sinogram (row stride ldz = the volume's height).
    def _slabs(self, nz):
        for z0 in range(0, nz, self._nz):
            yield z0, min(self._nz, nz - z0)

    def _R_into(self, x, res, coeffx=False):
        """res[ntheta, nz, n] = R(x[nz, n, n]) (complex64, contiguous), with the
        detector-axis B-spline prefilter when coeffx (ht_tomo_R_slab)."""
        nz, st = x.shape[0], _lib.stream_ptr()
        row = self.n * 8
        with torch.cuda.device(x.device):
            for z0, nzs in self._slabs(nz):
                _lib.call("ht_tomo_R_slab", self._h, _lib.ptr(x[z0]), ctypes.c_void_p(res.data_ptr() + z0 * row), nzs,
                          nz, int(coeffx), st)
        return res

    def _RT_into(self, d, res, coeffx=False, scale=1.0):
        """res[nz, n, n] = scale R^T(d[ntheta, nz, n]) (complex64, contiguous)."""
        nz, st = d.shape[1], _lib.stream_ptr()
        row = self.n * 8
        with torch.cuda.device(d.device):
            for z0, nzs in self._slabs(nz):
                _lib.call("ht_tomo_RT_slab", self._h, ctypes.c_void_p(d.data_ptr() + z0 * row), _lib.ptr(res[z0]),
                          nzs, nz, int(coeffx), float(scale), st)
        return res

    def R(self, obj, out=None):
        """Radon transform (tomo.py:56-86): [nz, n, n] -> [ntheta, nz, n] (any nz:
        volumes taller than the handle's slab run slab by slab)."""
        _lib.require_cuda(obj, "obj")
        nz = obj.shape[0]
        if tuple(obj.shape[1:]) != (self.n, self.n):
            raise ValueError(f"obj must be [nz, {self.n}, {self.n}], got {tuple(obj.shape)}")
        real = not obj.is_complex()
        x = obj.to(torch.complex64).contiguous()
        res = out if (out is not None and not real) else torch.empty(self.ntheta, nz, self.n, dtype=torch.complex64,
                                                                     device=x.device)
        self._R_into(x, res)
        if real:
            res = res.real.contiguous()
            if out is not None:
                out.copy_(res)
                return out
        return res

    def RT(self, data, out=None):
        """Adjoint Radon transform (tomo.py:88-116): [ntheta, nz, n] -> [nz, n, n]."""
        _lib.require_cuda(data, "data")
        nz = data.shape[1]
        if data.shape[0] != self.ntheta or data.shape[2] != self.n:
            raise ValueError(f"data must be [{self.ntheta}, nz, {self.n}], got {tuple(data.shape)}")
        real = not data.is_complex()
        x = data.to(torch.complex64).contiguous()
        res = out if (out is not None and not real) else torch.empty(nz, self.n, self.n, dtype=torch.complex64,
                                                                     device=x.device)
        self._RT_into(x, res)
        if real:
            res = res.real.contiguous()
            if out is not None:
                out.copy_(res)
                return out
        return res

    def _filter_sino(self, data, filter_name):
        """1-D detector filter of tomo.py:118-161 (ramp, shepp, parzen)."""
        n = self.n
        if filter_name not in self._filters:
            f = np.fft.fftfreq(n).astype("float32")
            af = np.abs(f) * 4 * n
            if filter_name == "ramp":
                h = af
            elif filter_name == "shepp":
                h = af * np.sinc(f)
            elif filter_name == "parzen":
                u = 2 * af
                h = af * np.where(u <= 0.5, 1 - 6 * u ** 2 + 6 * u ** 3, 2 * (1 - u) ** 3)
            else:
                raise ValueError(f"Unknown filter '{filter_name}'. Choose: ramp, shepp, parzen.")
            self._filters[filter_name] = torch.from_numpy((h / n).astype("float32")).to(self.device)
        sym = self._filters[filter_name]
        real = not data.is_complex()
        x = data.to(torch.complex64).contiguous()
        out = torch.empty_like(x)
        with torch.cuda.device(x.device):
            _lib.call("ht_filter_rows", n, _lib.ptr(x), _lib.ptr(out), x.numel() // n, _lib.ptr(sym),
                      _lib.stream_ptr())
        return out.real.contiguous() if real else out

    def fbp(self, data, filter_name="ramp"):
        """Filtered back-projection (tomo.py:163-183)."""
        if isinstance(data, np.ndarray):
            data = torch.from_numpy(data).to(self.device)
        norm_const = float(np.float32(np.sqrt(self.n / self.ntheta)))
        res = self.RT(self._filter_sino(data, filter_name))
        res *= norm_const
        return res

    def rec_tomo(self, d, niter=1):
        """Conjugate-gradient tomography (tomo.py:185-210), FP64 inner products."""
        def redot(a, b):
            return float(torch.sum(a.real.double() * b.real.double() + (a.imag.double() * b.imag.double()
                                                                          if a.is_complex() else 0)))
        u = torch.zeros(d.shape[1], self.n, self.n, dtype=d.dtype, device=d.device)
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
            u += alpha * eta
            Ru += alpha * Reta
        return u
