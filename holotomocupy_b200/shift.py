"""Cubic B-spline shift family on the B200 (drop-in for holotomocupy's Shift).

Reference: ``src/holotomocupy/shift.py:15-221``.  Same constructor
``Shift(n, npsi, nz, nzpsi, obj_dtype, nchunk=None)`` and methods ``phi``,
``coeff``, ``S``, ``Sadj``, ``curlyS``, ``curlySc``, ``dcurlySc``,
``dcurlySadjc`` (returns ``[out1, out2]``), ``d2curlySc`` and the Paganin
back-projection helpers ``Sback``, ``coeffback``, ``curlySback``, on CUDA torch
tensors.  Positions are ``[..., 0] = y``, ``[..., 1] = x`` pixel shifts and
``m`` the per-angle magnification, exactly as in the reference.
"""
import ctypes

import numpy as np
import torch

from . import _lib


def _f32(t, dev):
    if isinstance(t, np.ndarray):
        t = torch.from_numpy(t)
    return t.to(device=dev, dtype=torch.float32).contiguous()


class Shift:
    """Cubic B-spline shift operator (shift.py:15)."""

    def __init__(self, n, npsi, nz, nzpsi, obj_dtype, nchunk=None, device=None):
        self.n, self.npsi, self.nz, self.nzpsi = n, npsi, nz, nzpsi
        self.obj_dtype = obj_dtype
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self._complex = obj_dtype == "complex64"
        self._tdt = torch.complex64 if self._complex else torch.float32
        # forward B-spline denominator (shift.py:26-30), kept for API parity
        x = np.linspace(-1 / 2, 1 / 2 - 1 / npsi, npsi).astype("float32")
        y = np.linspace(-1 / 2, 1 / 2 - 1 / nzpsi, nzpsi).astype("float32")
        divx = (self.phi(0) + 2 * self.phi(1) * np.cos(2 * np.pi * x)).astype("float32")
        divy = (self.phi(0) + 2 * self.phi(1) * np.cos(2 * np.pi * y)).astype("float32")
        self.ifB3 = torch.from_numpy(1 / np.fft.fftshift(np.outer(divy, divx), axes=(-1, -2))).to(self.device)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("ht_shift_create", n, npsi, nz, nzpsi, 1 if self._complex else 0, ctypes.byref(h))
            # the prefilter always runs on complex samples
            hc = ctypes.c_void_p()
            _lib.call("ht_shift_create", n, npsi, nz, nzpsi, 1, ctypes.byref(hc))
        self._h, self._hc = h, hc

    def __del__(self):
        for name in ("_h", "_hc"):
            h = getattr(self, name, None)
            if h is not None and h.value:
                try:
                    _lib.lib().ht_shift_destroy(h)
                except Exception:
                    pass
                setattr(self, name, None)

    @staticmethod
    def phi(t):
        """The x6 cubic B-spline (shift.py:54-59)."""
        t = np.asarray(t, dtype=np.float64)
        out = ((-2 < t) * (t <= -1) * (t + 2) ** 3 + (-1 < t) * (t <= 1) * (4 - 6 * t ** 2 + 3 * t ** 3 * np.sign(t))
               + (1 < t) * (t <= 2) * (2 - t) ** 3)
        return out.item() if out.ndim == 0 else out

    # ------------------------------------------------------------ helpers
    def _coef(self, c, name):
        _lib.require_cuda(c, name)
        if c.ndim != 3 or tuple(c.shape[1:]) != (self.nzpsi, self.npsi):
            raise ValueError(f"{name} must be [batch, {self.nzpsi}, {self.npsi}], got {tuple(c.shape)}")
        return c.to(self._tdt).contiguous()

    def _img(self, g, name):
        _lib.require_cuda(g, name)
        if g.ndim != 3 or tuple(g.shape[1:]) != (self.nz, self.n):
            raise ValueError(f"{name} must be [batch, {self.nz}, {self.n}], got {tuple(g.shape)}")
        return g.to(self._tdt).contiguous()

    def _call(self, name, *args):
        with torch.cuda.device(self.device):
            _lib.call(name, *args, _lib.stream_ptr())

    # --------------------------------------------------------- operators
    def coeff(self, psi):
        """B-spline prefilter ifft2(fft2(psi) * ifB3) (shift.py:74-82)."""
        _lib.require_cuda(psi, "psi")
        x = psi.to(torch.complex64).contiguous()
        out = torch.empty_like(x)
        b = x.numel() // (self.nzpsi * self.npsi)
        self._call("ht_shift_coeff", self._hc, _lib.ptr(x), _lib.ptr(out), b)
        if self.obj_dtype == "float32":
            out = out.real.contiguous()
        return out

    def S(self, c, r, m):
        """Shift S (shift.py:102-111)."""
        c = self._coef(c, "c")
        r, m = _f32(r, c.device), _f32(m, c.device)
        out = torch.empty(c.shape[0], self.nz, self.n, dtype=self._tdt, device=c.device)
        self._call("ht_shift_S", self._h, _lib.ptr(c), _lib.ptr(r), _lib.ptr(m), _lib.ptr(out), c.shape[0])
        return out

    curlySc = S

    def Sadj(self, spsi, r, m):
        """Adjoint shift S^T (shift.py:113-122)."""
        g = self._img(spsi, "spsi")
        r, m = _f32(r, g.device), _f32(m, g.device)
        out = torch.empty(g.shape[0], self.nzpsi, self.npsi, dtype=self._tdt, device=g.device)
        self._call("ht_shift_Sadj", self._h, _lib.ptr(g), _lib.ptr(r), _lib.ptr(m), _lib.ptr(out), g.shape[0])
        return out

    def curlyS(self, psi, r, m):
        """S o coeff (shift.py:128-132)."""
        return self.S(self.coeff(psi), r, m)

    def dcurlySc(self, c, r, m, c1, Deltar):
        """First derivative (shift.py:170-183)."""
        c, c1 = self._coef(c, "c"), self._coef(c1, "c1")
        r, m, dr = _f32(r, c.device), _f32(m, c.device), _f32(Deltar, c.device)
        out = torch.empty(c.shape[0], self.nz, self.n, dtype=self._tdt, device=c.device)
        self._call("ht_shift_dS", self._h, _lib.ptr(c), _lib.ptr(r), _lib.ptr(m), _lib.ptr(c1), _lib.ptr(dr),
                   _lib.ptr(out), c.shape[0])
        return out

    def dcurlySadjc(self, c, r, m, Deltaphi, out2_dtype=torch.float32):
        """Adjoint derivative (shift.py:185-204): [S^T(Deltaphi), position part]."""
        c = self._coef(c, "c")
        g = self._img(Deltaphi, "Deltaphi")
        r, m = _f32(r, c.device), _f32(m, c.device)
        out1 = torch.empty(c.shape[0], self.nzpsi, self.npsi, dtype=self._tdt, device=c.device)
        out2 = torch.empty(c.shape[0], 2, dtype=torch.float64, device=c.device)
        self._call("ht_shift_dSadj", self._h, _lib.ptr(c), _lib.ptr(r), _lib.ptr(m), _lib.ptr(g), _lib.ptr(out1),
                   _lib.ptr(out2), c.shape[0])
        return [out1, out2.to(out2_dtype)]

    # ------------------------------------- Paganin back-projection helpers
    def coeffback(self, psi, m):
        """The prefilter of the B-spline stretched by the magnification m
        (shift.py:84-96): ifft2(fft2(psi) / (B_m(y) B_m(x))) with
        B_m = phi(0) + 2 sum_{k=1..4} phi(k / m) cos(2 pi k f).  One
        magnification, as the reference's callers pass it (the first element
        when m holds several)."""
        _lib.require_cuda(psi, "psi")
        m = float(np.asarray(m.cpu() if isinstance(m, torch.Tensor) else m, dtype=np.float64).reshape(-1)[0])
        x = np.linspace(-1 / 2, 1 / 2 - 1 / self.npsi, self.npsi).astype("float32")
        y = np.linspace(-1 / 2, 1 / 2 - 1 / self.nzpsi, self.nzpsi).astype("float32")
        dx = np.float32(self.phi(0))
        dy = np.float32(self.phi(0))
        for k in range(1, 5):
            pk = np.float32(self.phi(np.float32(k / m)))
            dx = (dx + 2 * pk * np.cos(2 * np.pi * k * x)).astype("float32")
            dy = (dy + 2 * pk * np.cos(2 * np.pi * k * y)).astype("float32")
        # FFT order, each axis carrying its 1/N
        symx = torch.from_numpy((1.0 / (self.npsi * np.fft.fftshift(dx).astype(np.float64))).astype("float32"))
        symy = torch.from_numpy((1.0 / (self.nzpsi * np.fft.fftshift(dy).astype(np.float64))).astype("float32"))
        symx, symy = symx.to(psi.device), symy.to(psi.device)
        x = psi.to(torch.complex64).contiguous()
        out = torch.empty_like(x)
        b = x.numel() // (self.nzpsi * self.npsi)
        self._call("ht_shift_filter", self._hc, _lib.ptr(x), _lib.ptr(out), b, _lib.ptr(symx), _lib.ptr(symy))
        return out

    def Sback(self, spsi, r, m):
        """Back-projection shift (shift.py:138-148): detector images
        [batch, nz, n] onto the coefficient grid [batch, nzpsi, npsi]
        (complex64) with the B-spline stretched by m -- one magnification, or
        one per image."""
        _lib.require_cuda(spsi, "spsi")
        if spsi.ndim != 3 or tuple(spsi.shape[1:]) != (self.nz, self.n):
            raise ValueError(f"spsi must be [batch, {self.nz}, {self.n}], got {tuple(spsi.shape)}")
        g = spsi.to(torch.complex64).contiguous()
        r = _f32(r, g.device).reshape(-1)
        m = _f32(m if isinstance(m, (torch.Tensor, np.ndarray)) else np.asarray(m, np.float32), g.device).reshape(-1)
        if m.numel() not in (1, g.shape[0]):
            raise ValueError(f"m must hold 1 or {g.shape[0]} magnifications, got {m.numel()}")
        if r.numel() != 2 * g.shape[0]:
            raise ValueError(f"r must be [{g.shape[0]}, 2]")
        out = torch.empty(g.shape[0], self.nzpsi, self.npsi, dtype=torch.complex64, device=g.device)
        self._call("ht_shift_Sback", self._hc, _lib.ptr(g), _lib.ptr(r), _lib.ptr(m), int(m.numel()), _lib.ptr(out),
                   g.shape[0])
        return out

    def curlySback(self, psi, r, m):
        """coeffback o Sback (shift.py:152-153)."""
        return self.coeffback(self.Sback(psi, r, m), m)

    def d2curlySc(self, c, r, m, c1, Deltar1, c2, Deltar2):
        """Second-order term (shift.py:206-221)."""
        c, c1, c2 = self._coef(c, "c"), self._coef(c1, "c1"), self._coef(c2, "c2")
        dev = c.device
        r, m, d1, d2 = _f32(r, dev), _f32(m, dev), _f32(Deltar1, dev), _f32(Deltar2, dev)
        out = torch.empty(c.shape[0], self.nz, self.n, dtype=self._tdt, device=dev)
        self._call("ht_shift_d2S", self._h, _lib.ptr(c), _lib.ptr(r), _lib.ptr(m), _lib.ptr(c1), _lib.ptr(d1),
                   _lib.ptr(c2), _lib.ptr(d2), _lib.ptr(out), c.shape[0])
        return out
