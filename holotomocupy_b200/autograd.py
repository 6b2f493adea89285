"""Differentiable forms of the operator chain for torch.autograd.

Each operator is a ``torch.autograd.Function`` whose backward pass is the
hand-written adjoint kernel (PyTorch's convention for a complex-linear map is
that the backward of ``y = A x`` is ``A^H grad_y``; for a real input ``p`` of
a complex output it is ``Re <grad_y, dy/dp>``):

* ``radon(obj, tomo)``: ``R obj`` (tomo.py:56-86); backward ``R^T``
  (``ht_tomo_RT``, tomo.py:88-116);
* ``shift(psi, pos, mag, sh)``: ``S(coeff(psi); pos, mag)`` (shift.py:128-132);
  backward for ``psi``: ``coeff(S^T g)``, for ``pos``: the position
  derivative ``Re <g, dS/dpos>`` -- both from ``ht_shift_dSadj``
  (shift.py:185-204) -- the prefilter being self-adjoint;
* ``propagate(psi, j, prop)``: ``D_j psi`` (propagation.py:70-89); backward
  ``D_j^T`` (``ht_prop_DT``, propagation.py:91-112).

``DataFidelity`` composes them (with the probe product, whose gradient sum
over angles is taken in complex128) into the BH data term
(rec_mpi.py:517-813): ``F = 1/N sum (|D_k(prb_k exp(i S_k(coeff(R obj))))| - d)^2``
over (angle, distance) images, optionally in angle chunks whose forward is
recomputed in the backward pass (``torch.utils.checkpoint``), so that only one
chunk's intermediates are held at a time.
"""
import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

from .propagation import Propagation
from .shift import Shift
from .tomo import Tomo


class _Radon(torch.autograd.Function):
    @staticmethod
    def forward(ctx, obj, tomo):
        ctx.tomo = tomo
        return tomo.R(obj.contiguous())

    @staticmethod
    def backward(ctx, g):
        return ctx.tomo.RT(g.contiguous()), None


class _Shift(torch.autograd.Function):
    @staticmethod
    def forward(ctx, psi, pos, mag, sh):
        c = sh.coeff(psi.contiguous())
        ctx.sh = sh
        ctx.save_for_backward(c, pos, mag)
        return sh.S(c, pos, mag)

    @staticmethod
    def backward(ctx, g):
        c, pos, mag = ctx.saved_tensors
        sh = ctx.sh
        gc, gpos = sh.dcurlySadjc(c, pos, mag, g.contiguous())
        gpsi = sh.coeff(gc) if ctx.needs_input_grad[0] else None
        return gpsi, (gpos.to(pos.dtype) if ctx.needs_input_grad[1] else None), None, None


class _Propagate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, psi, j, prop):
        ctx.prop, ctx.j = prop, j
        return prop.D(psi.contiguous(), j)

    @staticmethod
    def backward(ctx, g):
        return ctx.prop.DT(g.contiguous(), ctx.j), None, None


class _ProbeMul(torch.autograd.Function):
    """prb [nz, n] times x12 [B, nz, n]; the probe gradient, a sum over the B
    angles, is accumulated in complex128 (as the fused cascade's is)."""

    @staticmethod
    def forward(ctx, prb, x12):
        ctx.save_for_backward(prb, x12)
        return prb.unsqueeze(0) * x12

    @staticmethod
    def backward(ctx, g):
        prb, x12 = ctx.saved_tensors
        gprb = gx = None
        if ctx.needs_input_grad[0]:
            gprb = torch.sum((g * x12.conj()).to(torch.complex128), dim=0).to(prb.dtype)
        if ctx.needs_input_grad[1]:
            gx = g * prb.conj().unsqueeze(0)
        return gprb, gx


def radon(obj, tomo):
    """R obj for obj [nz, n, n] complex64 -> [ntheta, nz, n]."""
    return _Radon.apply(obj, tomo)


def shift(psi, pos, mag, sh):
    """S(coeff(psi)) for psi [B, nzpsi, npsi], pos [B, 2] (y, x), mag [B]."""
    return _Shift.apply(psi, pos, mag, sh)


def propagate(psi, j, prop):
    """D_j psi for psi [B, nz, n]."""
    return _Propagate.apply(psi, j, prop)


class DataFidelity(torch.nn.Module):
    """The BH data term as a differentiable function of (obj or proj, prb, pos).

    Sizes as for Rec: object [nzobj, nobj, nobj], detector [nz, n], angles
    ``theta``, ``ndist`` distances (metres), probe [ndist, nz, n], positions
    [ntheta, ndist, 2] (y, x) and magnifications [ntheta, ndist].  With
    ``chunk`` the angles are processed ``chunk`` at a time and each chunk's
    forward is recomputed during the backward pass."""

    def __init__(self, sh, prop, theta, mask_r, nobj, nzobj, chunk=None):
        super().__init__()
        theta = np.asarray(theta.cpu() if isinstance(theta, torch.Tensor) else theta, dtype="float32")
        self.n, self.nz, self.ndist = prop.n, prop.nz, prop.ndist
        self.nobj, self.nzobj = nobj, nzobj
        self.ntheta = len(theta)
        self.data_size = self.ntheta * self.ndist * self.nz * self.n
        self.chunk = chunk or self.ntheta
        self.bounds = [(a, min(a + self.chunk, self.ntheta)) for a in range(0, self.ntheta, self.chunk)]
        self.tomos = [Tomo(nobj, nzobj, theta[a:b], mask_r, norm_ntheta=self.ntheta) for a, b in self.bounds]
        self.sh, self.prop = sh, prop

    @classmethod
    def create(cls, n, nz, nobj, nzobj, theta, ndist, wavelength, voxelsize, distance, mask_r=None, chunk=None,
               obj_dtype="complex64"):
        """Operators built from the geometry."""
        ntheta = len(theta)
        return cls(Shift(n, nobj, nz, nzobj, obj_dtype),
                   Propagation(n, nz, chunk or ntheta, ndist, wavelength, voxelsize, distance),
                   theta, mask_r, nobj, nzobj, chunk)

    @classmethod
    def from_rec(cls, rec, chunk=None):
        """The data term of a Rec (its shift and propagation operators, angles
        and object mask)."""
        return cls(rec.cl_shift, rec.cl_prop, rec.cl_tomo.theta, rec.mask, rec.nobj, rec.nzobj, chunk)

    def _term(self, proj, prb, pos, mag, data):
        out = proj.new_zeros((), dtype=torch.float32).real
        for k in range(self.ndist):
            x22 = shift(proj, pos[:, k].contiguous(), mag[:, k].contiguous(), self.sh)
            x12 = torch.exp(1j * x22)
            x0 = propagate(_ProbeMul.apply(prb[k], x12), k, self.prop)
            out = out + torch.sum((torch.abs(x0) - data[:, k]) ** 2)
        return out

    def _chunk_obj(self, i, obj, prb, pos, mag, data):
        return self._term(radon(obj, self.tomos[i]), prb, pos, mag, data)

    def forward(self, x, prb, pos, mag, data, proj=False):
        """F at (x, prb, pos): x is the object, or with proj=True the
        projections [ntheta, nzobj, nobj] (the BH variable proj)."""
        total = None
        for i, (a, b) in enumerate(self.bounds):
            args = (prb, pos[a:b], mag[a:b], data[a:b])
            if proj:
                f = self._term
                args = (x[a:b],) + args
            else:
                f = self._chunk_obj
                args = (i, x) + args
            t = checkpoint(f, *args, use_reentrant=False) if len(self.bounds) > 1 else f(*args)
            total = t if total is None else total + t
        return total / self.data_size
