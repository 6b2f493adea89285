"""Fresnel propagator D / DT on the B200 (drop-in for holotomocupy's Propagation).

Reference: ``src/holotomocupy/propagation.py:11-112``.  Same constructor
arguments, same ``D(psi, j)`` / ``DT(psi, j)`` calls on 2-D ``[nz, n]`` or 3-D
``[ntheta, nz, n]`` complex64 arrays (CUDA torch tensors here instead of CuPy
arrays), same ``fker`` table.  The work is done by ``ht_prop_D`` /
``ht_prop_DT`` of ``libholotomo_b200.so``: a DCT-domain form of the reference's
mirror-padded FFT convolution that never builds the padded 2nz x 2n buffer.
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

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().ht_prop_destroy(h)
            except Exception:
                pass
            self._h = None

    def _apply(self, name, psi, j, out=None):
        _lib.require_cuda(psi, "psi")
        added = psi.ndim == 2
        x = psi.unsqueeze(0) if added else psi
        if x.ndim != 3 or tuple(x.shape[1:]) != (self.nz, self.n):
            raise ValueError(f"expected [..., {self.nz}, {self.n}] input, got {tuple(psi.shape)}")
        x = x.to(torch.complex64).contiguous()
        if out is None:
            out = torch.empty_like(x)
        if not (0 <= j < self.ndist):
            raise IndexError(f"distance index {j} out of range [0, {self.ndist})")
        with torch.cuda.device(x.device):
            _lib.call(name, self._h, _lib.ptr(x), _lib.ptr(out), x.shape[0], int(j), _lib.stream_ptr())
        return out[0] if added else out

    def D(self, psi, j):
        """Forward propagator (propagation.py:70-89)."""
        return self._apply("ht_prop_D", psi, j)

    def DT(self, big_psi, j):
        """Adjoint propagator (propagation.py:91-112)."""
        return self._apply("ht_prop_DT", big_psi, j)
