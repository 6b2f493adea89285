"""Fresnel propagator D / DT on the B200 (drop-in for holotomocupy's Propagation).

Reference: ``src/holotomocupy/propagation.py:11-112``.  Same constructor
arguments, same ``D(psi, j)`` / ``DT(psi, j)`` calls on 2-D ``[nz, n]`` or 3-D
``[ntheta, nz, n]`` complex64 arrays (CUDA torch tensors here instead of CuPy
arrays), same ``fker`` table.  The work is done by ``ht_prop_D`` /
``ht_prop_DT`` of ``libholotomo_b200.so``: a DCT-domain form of the reference's
mirror-padded FFT convolution that never builds the padded 2nz x 2n buffer.

The attributes the reference's own tests reach into are kept
(tests/propagation/test_propagation.py:25-29, 154-191): ``_use_cufftdx``
(True: the library's propagator; False: the padded-grid path through torch's
cuFFT, the reference's CuPy branch, kept as the comparison point),
``_fwd_pad`` / ``_adj_pad`` (mirror padding and its adjoint, library
kernels), ``_conv2d.run`` (the padded-grid convolution, a library kernel) and
``_buf_big`` (the padded work buffer, allocated on first use because only the
padded-grid path needs it).
"""
import ctypes

import numpy as np
import torch

from . import _lib


def fresnel_table(n, nz, wavelength, voxelsize, distance):
    """The reference's Fresnel kernels (propagation.py:20-28), evaluated with the
    same arithmetic: float32 frequencies and squared radius, the phase in
    double precision, stored as complex64.  Shape [ndist, 2nz, 2n]."""
    fx = np.fft.fftfreq(2 * n, d=voxelsize).astype("float32")
    fy = np.fft.fftfreq(2 * nz, d=voxelsize).astype("float32")
    fx, fy = np.meshgrid(fx, fy)
    f2 = fx ** 2 + fy ** 2
    norm = float(4 * n * nz)
    out = np.empty((len(distance), 2 * nz, 2 * n), dtype="complex64")
    for j in range(len(distance)):
        out[j] = np.exp(-1j * np.pi * wavelength * np.float64(distance[j]) * f2) / norm
    return out


class Conv2D:
    """The padded-grid convolution ``y[b] = IFFT2(FFT2(x[b]) * H)`` (inverse
    unnormalised) of the reference's cuFFTDx wrapper
    (conv2d_cufftdx.py:150-196), on ``ht_conv2d_run``."""

    def __init__(self, nx, ny, device):
        self.nx, self.ny = nx, ny          # rows, columns of one image
        self.device = device
        h = ctypes.c_void_p()
        with torch.cuda.device(device):
            _lib.call("ht_conv2d_create", nx, ny, ctypes.byref(h))
        self._h = h

    def run(self, x, H, y, stream=None):
        """y[b] = IFFT2_unnorm(FFT2(x[b]) * H); x, y [batch, nx, ny] complex64
        contiguous (y may be x), H [nx, ny]; on ``stream`` (a torch stream,
        default the current one)."""
        x, H = x.resolve_conj(), H.resolve_conj()
        for name, t in (("x", x), ("H", H), ("y", y)):
            _lib.require_cuda(t, name, torch.complex64)
            if not t.is_contiguous():
                raise ValueError(f"{name} must be contiguous")
        if tuple(x.shape[-2:]) != (self.nx, self.ny) or tuple(H.shape) != (self.nx, self.ny) or y.shape != x.shape:
            raise ValueError(f"expected x, y [batch, {self.nx}, {self.ny}] and H [{self.nx}, {self.ny}]")
        st = _vp_stream(stream, x.device)
        with torch.cuda.device(x.device):
            _lib.call("ht_conv2d_run", self._h, _lib.ptr(x), _lib.ptr(H), _lib.ptr(y), x.shape[0], st)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().ht_conv2d_destroy(h)
            except Exception:
                pass
            self._h = None


def _vp_stream(stream, device):
    if stream is None:
        return _lib.stream_ptr(device)
    return ctypes.c_void_p(stream.cuda_stream)


class Propagation:
    """Functionality for Propagation (propagation.py:11)."""

    def __init__(self, n, nz, ntheta, ndist, wavelength, voxelsize, distance, device=None):
        self.n = n
        self.nz = nz
        self._ntheta = ntheta
        self.ndist = ndist
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        table = fresnel_table(n, nz, wavelength, voxelsize, np.asarray(distance)[:ndist])
        self.fker = torch.from_numpy(table).to(self.device)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("ht_prop_create", n, nz, ndist, table.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h))
        self._h = h
        self._use_cufftdx = True
        self._buf = None
        self._conv = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().ht_prop_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------- the reference's internals
    @property
    def _buf_big(self):
        """Padded work buffer [ntheta, 2nz, 2n] complex64 (propagation.py:31)."""
        if self._buf is None:
            self._buf = torch.empty(self._ntheta, 2 * self.nz, 2 * self.n, dtype=torch.complex64, device=self.device)
        return self._buf

    @property
    def _conv2d(self):
        """The padded-grid convolution object (propagation.py:36-40)."""
        if self._conv is None:
            self._conv = Conv2D(2 * self.nz, 2 * self.n, self.device)
        return self._conv

    def _fwd_pad(self, f, fpad):
        """Symmetric padding f [ntheta, nz, n] -> fpad [ntheta, 2nz, 2n] (propagation.py:46-56)."""
        _lib.require_cuda(f, "f", torch.complex64)
        _lib.require_cuda(fpad, "fpad", torch.complex64)
        f = f.contiguous()
        nt, nz, n = f.shape
        if tuple(fpad.shape) != (nt, 2 * nz, 2 * n) or not fpad.is_contiguous():
            raise ValueError(f"fpad must be a contiguous [{nt}, {2 * nz}, {2 * n}] array")
        with torch.cuda.device(f.device):
            _lib.call("ht_pad_mirror", _lib.ptr(f), _lib.ptr(fpad), nt, nz, n, _lib.stream_ptr())

    def _adj_pad(self, fpad, f):
        """Adjoint padding fpad [ntheta, 2nz, 2n] -> f [ntheta, nz, n] (propagation.py:58-68)."""
        _lib.require_cuda(f, "f", torch.complex64)
        _lib.require_cuda(fpad, "fpad", torch.complex64)
        fpad = fpad.contiguous()
        nt, nz2, n2 = fpad.shape
        if tuple(f.shape) != (nt, nz2 // 2, n2 // 2) or not f.is_contiguous():
            raise ValueError(f"f must be a contiguous [{nt}, {nz2 // 2}, {n2 // 2}] array")
        with torch.cuda.device(f.device):
            _lib.call("ht_pad_fold", _lib.ptr(fpad), _lib.ptr(f), nt, nz2 // 2, n2 // 2, _lib.stream_ptr())

    def _padded(self, x, j, adjoint):
        """The reference's CuPy branch on torch's cuFFT (propagation.py:77-86,
        98-110): the comparison point for the library's propagator."""
        nt = x.shape[0]
        buf = self._buf_big[:nt]
        h = self.fker[j].conj() if adjoint else self.fker[j]
        if adjoint:
            buf.zero_()
            buf[:, self.nz // 2: -self.nz // 2, self.n // 2: -self.n // 2] = x
        else:
            self._fwd_pad(x, buf)
        y = torch.fft.ifft2(torch.fft.fft2(buf) * h, norm="forward")
        if not adjoint:
            return y[:, self.nz // 2: -self.nz // 2, self.n // 2: -self.n // 2].contiguous()
        out = torch.empty_like(x)
        self._adj_pad(y, out)
        return out

    def _apply(self, name, psi, j, out=None):
        _lib.require_cuda(psi, "psi")
        added = psi.ndim == 2
        x = psi.unsqueeze(0) if added else psi
        if x.ndim != 3 or tuple(x.shape[1:]) != (self.nz, self.n):
            raise ValueError(f"expected [..., {self.nz}, {self.n}] input, got {tuple(psi.shape)}")
        x = x.to(torch.complex64).contiguous()
        if not (0 <= j < self.ndist):
            raise IndexError(f"distance index {j} out of range [0, {self.ndist})")
        if not self._use_cufftdx:
            res = self._padded(x, j, name == "ht_prop_DT")
            return res[0] if added else res
        if out is None:
            out = torch.empty_like(x)
        with torch.cuda.device(x.device):
            _lib.call(name, self._h, _lib.ptr(x), _lib.ptr(out), x.shape[0], int(j), _lib.stream_ptr())
        return out[0] if added else out

    def D(self, psi, j):
        """Forward propagator (propagation.py:70-89)."""
        return self._apply("ht_prop_D", psi, j)

    def DT(self, big_psi, j):
        """Adjoint propagator (propagation.py:91-112)."""
        return self._apply("ht_prop_DT", big_psi, j)
