"""Bilinear-Hessian holotomography solver on the B200 (drop-in for holotomocupy's Rec).

Reference: ``src/holotomocupy/rec_mpi.py:21-902`` (single rank).  Same
constructor ``Rec(args)`` with the reference's argument keys, the same
``vars`` / ``grads`` / ``etas`` dictionaries (CUDA torch tensors, resident on
the device instead of pinned host arrays), the cascade functions ``F*``,
``dF*``, ``d2F_dF*``, ``gF*`` (operator-by-operator, for derivative checks),
and ``gradients``, ``hessian``, ``BH``, ``min``, ``gen_sqrt_data``,
``gen_sqrt_ref``.

The solver itself runs the fused cascade of ``libholotomo_b200.so``
(``ht_rec_gradient`` / ``ht_rec_hessian``): one gradient pass and one Hessian
pass per iteration evaluate every quadratic form the reference's three
Hessian cascades produce, with the B-spline coefficients of vars/grads/etas
``proj`` kept alongside ``proj`` (the prefilter is linear, so the BH updates
apply to them directly).  Inner products, quadratic forms and the step sizes
are accumulated in float64.

Optional argument keys beyond the reference's: ``distance``, ``wavelength``,
``voxelsize`` and ``norm_magnifications`` give the propagation geometry
directly instead of deriving it from ``z1``/``energy`` (rec_mpi.py:55-60).
"""
import ctypes
import gc
import logging
import math
import time

import numpy as np
import torch

from . import _lib
from .convtable import log_error, new_table
from .propagation import Propagation
from .shift import Shift
from .tomo import Tomo

_log = logging.getLogger("holotomocupy_b200")


def _t(x, device, dtype=None):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype or x.dtype)
    return torch.as_tensor(np.asarray(x), device=device, dtype=dtype)


def position_drift(pos, pos_init):
    """Mean over the angles of |pos - pos_init|: [ndist, 2] float64 (y, x in
    pixels) from [ntheta, ndist, 2] position arrays."""
    return (pos - pos_init).abs().double().sum(dim=0).cpu().numpy() / pos.shape[0]


def reprod(a, b):
    """utils.py:96-97"""
    if a.is_complex() or b.is_complex():
        a = a if a.is_complex() else torch.complex(a, torch.zeros_like(a))
        b = b if b.is_complex() else torch.complex(b, torch.zeros_like(b))
        return a.real * b.real + a.imag * b.imag
    return a * b


def redot(a, b):
    """utils.py:100-103, accumulated in float64."""
    return float(torch.sum(reprod(a, b).double()))


class Rec:
    """BH reconstruction (rec_mpi.py:21)."""

    def __init__(self, args):
        for key, value in vars(args).items():
            setattr(self, key, value)
        if not hasattr(self, "lam_laplacian"):
            self.lam_laplacian = 0
        if not hasattr(self, "lam_prbfit"):
            self.lam_prbfit = 0
        self.device = torch.device("cuda", torch.cuda.current_device())
        dev = self.device
        if getattr(self, "distance", None) is None:                      # rec_mpi.py:55-60
            wavelength = 1.24e-09 / self.energy
            z1 = np.asarray(self.z1)
            z2 = self.focustodetectordistance - z1
            magnifications = self.focustodetectordistance / z1
            norm_magnifications = magnifications / magnifications[0]
            distance = (z1 * z2) / self.focustodetectordistance * norm_magnifications ** 2
            voxelsize = self.detector_pixelsize / magnifications[0]
        else:
            wavelength, voxelsize, distance = self.wavelength, self.voxelsize, np.asarray(self.distance)
            norm_magnifications = np.asarray(getattr(self, "norm_magnifications", np.ones(self.ndist)))
        self.rho_sq = {"obj": args.rho[0] ** 2, "prb": args.rho[1] ** 2, "pos": args.rho[2] ** 2}
        self.complex_obj = self.obj_dtype == "complex64"
        self.odt = torch.complex64 if self.complex_obj else torch.float32
        theta = np.asarray(self.theta.cpu() if isinstance(self.theta, torch.Tensor) else self.theta)
        # angle chunks of the fused cascade and object slabs of the Radon
        # transform (None: all at once); the chunked iteration recomputes each
        # angle chunk's forward pass before its Hessian pass
        self.angle_chunk = min(int(getattr(self, "angle_chunk", None) or self.ntheta), self.ntheta)
        self.slab_chunk = min(int(getattr(self, "slab_chunk", None) or self.nzobj), self.nzobj)
        self.cl_tomo = Tomo(self.nobj, self.slab_chunk, theta, self.mask)
        self.cl_prop = Propagation(self.n, self.nz, self.ntheta, self.ndist, wavelength, voxelsize, distance)
        self.cl_shift = Shift(self.n, self.nobj, self.nz, self.nzobj, self.obj_dtype)
        self.norm_const = float(np.float32(np.sqrt(self.nobj / self.ntheta)))   # rec_mpi.py:88
        self.norm_magnifications = norm_magnifications
        self.data_size = self.ntheta * self.ndist * self.nz * self.n
        self.prb_size = self.ndist * self.nz * self.n
        self.obj_size = self.nzobj * self.nobj ** 2
        self.table = new_table()
        self.alloc_arrays()
        h = ctypes.c_void_p()
        _lib.call("ht_rec_create", self.n, self.nz, self.nobj, self.nzobj, self.angle_chunk, self.ndist,
                  1 if self.complex_obj else 0, self.cl_prop._h, ctypes.byref(h))
        self._h = h
        # a handle processes exactly its own number of angles: the last, shorter
        # chunk has a handle of its own
        self._hrest = None
        rest = self.ntheta % self.angle_chunk
        if rest:
            hr = ctypes.c_void_p()
            _lib.call("ht_rec_create", self.n, self.nz, self.nobj, self.nzobj, rest, self.ndist,
                      1 if self.complex_obj else 0, self.cl_prop._h, ctypes.byref(hr))
            self._hrest = hr
        if self.angle_chunk < self.ntheta:
            for hh in (h, self._hrest):
                if hh is not None:
                    _lib.call("ht_rec_set_data_size", hh, float(self.data_size))
        self._scal = torch.zeros(8, dtype=torch.float64, device=dev)

    # the reference's operator lists (rec_mpi.py:38-45), built on access so
    # that the object holds no reference to itself and is freed when dropped
    @property
    def F(self):
        return [self.F0, self.F1, self.F2, self.F3]

    @property
    def gF(self):
        return [self.gF0, self.gF1, self.gF2, self.gF3]

    @property
    def dF(self):
        return [self.dF0, self.dF1, self.dF2, self.dF3]

    @property
    def d2F_dF(self):
        return [self.d2F_dF0, self.d2F_dF1, self.d2F_dF2, self.d2F_dF3]

    def close(self):
        """Release the device state now (the handle, the recorded graph and
        the arrays); the object is unusable afterwards."""
        try:
            self.release_graph()
        except Exception:
            pass
        for name in ("_h", "_hrest"):
            h = getattr(self, name, None)
            if h is not None and h.value:
                try:
                    _lib.lib().ht_rec_destroy(h)
                except Exception:
                    pass
                setattr(self, name, None)
        try:
            for name in ("vars", "grads", "etas", "data", "ref"):
                if isinstance(getattr(self, name, None), (dict, torch.Tensor)):
                    setattr(self, name, None)
        except Exception:   # interpreter shutdown
            pass

    def __del__(self):
        self.close()

    def reset(self):
        """Return to the state of a new Rec of the same arguments -- every
        array zero, no recorded graph, an empty convergence table -- keeping
        the device memory, the library handles and the operator tables: a
        server hands a finished reconstruction's Rec to the next request of
        the same arguments without freeing and allocating (each free
        synchronises the device).  Runs on the current stream."""
        self.release_graph()
        for d in (self.vars, self.grads, self.etas, self._c):
            for t in d.values():
                t.zero_()
        for t in (self.data, self.ref, self.shrink_nd, self._gc, self._gpos, self._gprb, self._H, self._dots,
                  self._bh, self._hist, self._count, self._vol, self._lapw, self._pfw, self._pf3, self._scal):
            if t is not None:
                t.zero_()
        self.table = new_table()

    # ------------------------------------------------------------ state
    def alloc_arrays(self):
        """rec_mpi.py:105-136 (device-resident, zero-initialised)."""
        dev, odt = self.device, self.odt
        prb_shape = (self.ndist, self.nz, self.n)
        z = lambda *s, dt=odt: torch.zeros(*s, dtype=dt, device=dev)
        self.vars = {"obj": z(self.nzobj, self.nobj, self.nobj), "pos": z(self.ntheta, self.ndist, 2, dt=torch.float32),
                     "prb": z(*prb_shape, dt=torch.complex64), "proj": z(self.ntheta, self.nzobj, self.nobj)}
        self.data = z(self.ntheta, self.ndist, self.nz, self.n, dt=torch.float32)
        self.ref = z(*prb_shape, dt=torch.float32)
        self.grads, self.etas = {}, {}
        for ge in (self.grads, self.etas):
            ge["obj"] = z(self.nzobj, self.nobj, self.nobj)
            ge["pos"] = z(self.ntheta, self.ndist, 2, dt=torch.float32)
            ge["proj"] = z(self.ntheta, self.nzobj, self.nobj)
            ge["prb"] = z(*prb_shape, dt=torch.complex64)
        # rec_mpi.py:135-136: one array, zero until BH() sets it (rec_mpi.py:146)
        self.shrink_nd = z(self.ntheta, self.ndist, dt=torch.float32)
        self.eff_demagnifications = self.shrink_nd
        # B-spline coefficients of vars/grads/etas proj
        self._c = {"vars": z(self.ntheta, self.nzobj, self.nobj), "grads": z(self.ntheta, self.nzobj, self.nobj),
                   "etas": z(self.ntheta, self.nzobj, self.nobj)}
        # persistent outputs of the fused passes and the device-side BH state:
        # nothing in an iteration allocates, so it can be recorded in a graph
        self._gc = z(self.ntheta, self.nzobj, self.nobj)
        self._gpos = z(self.ntheta, self.ndist, 2, dt=torch.float32)
        self._gprb = z(*prb_shape, dt=torch.complex64)
        self._H = z(4, dt=torch.float64)
        self._dots = z(4, dt=torch.float64)
        self._bh = z(2, dt=torch.float64)            # beta, alpha
        self._hist_cap = 4096
        self._hist = z(self._hist_cap, 2, dt=torch.float64)
        self._count = z(1, dt=torch.int32)
        self._graph = None
        # BH keeps only the B-spline coefficients of proj up to date and applies
        # the prefilter as Cx inside R / R^T and Cz on the volume (complex
        # objects); vars/grads/etas "proj" are recomputed by bh_finish()
        self._fold = self.complex_obj
        # the folded (complex-object) iteration allocates nothing, so it may be
        # recorded into a CUDA graph
        self.graphable = self._fold
        self._vol = z(self.nzobj, self.nobj, self.nobj) if self._fold else None
        # Laplacian regulariser workspace: the inner Laplacian on nzobj + 2 slices, then
        # 64 KiB of per-block partial sums from the next 16-byte boundary
        lap_bytes = -(-(self.nzobj + 2) * self.nobj * self.nobj * (8 if self.complex_obj else 4) // 16) * 16
        self._lapw = z(lap_bytes + 64 * 1024, dt=torch.uint8) if self.lam_laplacian != 0 else None
        # probe-fit workspace: three propagated probe-sized arrays and 32 KiB of partial sums
        self._pfw = (z(3 * self.ndist * self.nz * self.n + 4096, dt=torch.complex64)
                     if self.lam_prbfit != 0 else None)
        self._pf3 = z(3, dt=torch.float64)

    def _coeff_into(self, src, dst):
        """dst = coeff(src) (shift.py:74-82) for a [ntheta, nzobj, nobj] array."""
        if self.complex_obj:
            _lib.call("ht_shift_coeff", self.cl_shift._hc, _lib.ptr(src), _lib.ptr(dst), src.shape[0],
                      _lib.stream_ptr())
        else:
            dst.copy_(self.cl_shift.coeff(src))
        return dst

    def _axpby(self, x, y, a, b, dot=None):
        n = x.numel() * (2 if x.is_complex() else 1)
        _lib.call("ht_axpby", _lib.ptr(x), _lib.ptr(y), float(a), float(b), n,
                  _lib.ptr(dot) if dot is not None else None, _lib.stream_ptr())

    # -------------------------------------------------- fused cascade
    # ---------------------------------------------------- angle chunks
    def _chunks(self):
        """(first angle, handle) of each angle chunk of the fused cascade."""
        for th0 in range(0, self.ntheta, self.angle_chunk):
            yield th0, (self._h if th0 + self.angle_chunk <= self.ntheta else self._hrest)

    @staticmethod
    def _at(t, th0):
        """Address of angle th0 of an angle-major array (an angle chunk)."""
        return ctypes.c_void_p(t.data_ptr() + th0 * (t.numel() // t.shape[0]) * t.element_size())

    def _forward(self, c, pos, mag, prb, data=None, amp=None):
        """ht_rec_forward over the angle chunks: amplitudes into amp, or the
        objective sum (|x0| - data)^2 returned as a float."""
        total, st = 0.0, _lib.stream_ptr()
        for th0, h in self._chunks():
            _lib.call("ht_rec_forward", h, self._at(c, th0), self._at(pos, th0), self._at(mag, th0),
                      _lib.ptr(prb), self._at(data, th0) if data is not None else None,
                      self._at(amp, th0) if amp is not None else None,
                      _lib.ptr(self._scal) if data is not None else None, st)
            if data is not None:
                total += float(self._scal[0])
        return total

    def _gradient_pass(self, c, pos, prb, persistent=False, gpos=None, gprb=None, scale_pos=1.0, scale_prb=1.0):
        """Fused gF0..gF3 (rec_mpi.py:327-353): returns (sum_k S^T Y22, gpos, gprb), F in _scal[0].
        persistent=True writes gc into the Rec's own array (no allocation);
        gpos / gprb given: written there, times scale_pos / scale_prb.  Angle
        chunks run in turn, the probe gradient and F accumulated."""
        gc = self._gc if persistent else torch.empty_like(c)
        if gpos is None:
            gpos = self._gpos if persistent else torch.empty(self.ntheta, self.ndist, 2, dtype=torch.float32,
                                                             device=self.device)
        if gprb is None:
            gprb = self._gprb if persistent else torch.empty(self.ndist, self.nz, self.n, dtype=torch.complex64,
                                                             device=self.device)
        mag, st = self.eff_demagnifications, _lib.stream_ptr()
        for k, (th0, h) in enumerate(self._chunks()):
            _lib.call("ht_rec_gradient", h, self._at(c, th0), self._at(pos, th0), self._at(mag, th0),
                      _lib.ptr(prb), self._at(self.data, th0), self._at(gc, th0), self._at(gpos, th0), _lib.ptr(gprb),
                      _lib.ptr(self._scal), float(scale_pos), float(scale_prb), int(k > 0), st)
        return gc, gpos, gprb

    def _hessian_pass(self, c, pos, prb, y, z=None, out=None):
        """Fused Hessian forms; y, z = (coefficients, pos, prb) of the directions.
        Returns float64 tensor [H(y,y), H_ref(y,z), H(z,z), H_sym(y,z)].  With
        angle chunks, each chunk's forward and adjoint caches are recomputed
        (its gradient call, outputs discarded) before its Hessian call."""
        if out is None:
            out = torch.zeros(4, dtype=torch.float64, device=self.device)
        zz = z if z is not None else (None, None, None)
        mag, st = self.eff_demagnifications, _lib.stream_ptr()
        chunked = self.angle_chunk < self.ntheta
        if chunked and getattr(self, "_scratch", None) is None:
            self._scratch = (torch.empty((self.angle_chunk,) + tuple(c.shape[1:]), dtype=c.dtype, device=self.device),
                             torch.empty(self.angle_chunk, self.ndist, 2, dtype=torch.float32, device=self.device),
                             torch.empty(self.ndist, self.nz, self.n, dtype=torch.complex64, device=self.device))
        at = self._at
        for k, (th0, h) in enumerate(self._chunks()):
            if chunked:
                sc, sp, sq = self._scratch
                _lib.call("ht_rec_gradient", h, at(c, th0), at(pos, th0), at(mag, th0), _lib.ptr(prb),
                          at(self.data, th0), _lib.ptr(sc), _lib.ptr(sp), _lib.ptr(sq),
                          ctypes.c_void_p(self._scal.data_ptr() + 8), 1.0, 1.0, 0, st)
            _lib.call("ht_rec_hessian", h, at(c, th0), at(pos, th0), at(mag, th0), _lib.ptr(prb),
                      at(self.data, th0), 2 if z is not None else 1, at(y[0], th0), at(y[1], th0), _lib.ptr(y[2]),
                      at(zz[0], th0) if z is not None else None, at(zz[1], th0) if z is not None else None,
                      _lib.ptr(zz[2]) if z is not None else None, _lib.ptr(out), int(k > 0), st)
        return out

    def _contig(self, d):
        return {k: v.contiguous() for k, v in d.items()}

    def gradients_cascade(self, vars, grads):
        """rec_mpi.py:327-353 (data term; writes grads prb/proj/pos)."""
        v = self._contig(vars)
        c = self._coeff_into(v["proj"], torch.empty_like(v["proj"]))
        gc, gpos, gprb = self._gradient_pass(c, v["pos"], v["prb"])
        grads["prb"][:] = gprb * self.rho_sq["prb"]
        grads["proj"][:] = self.cl_shift.coeff(gc) * self.rho_sq["obj"]
        grads["pos"][:] = gpos * self.rho_sq["pos"]

    def hessian_cascade(self, vars, grads, etas):
        """rec_mpi.py:250-303: the data-term Hessian form at vars for (grads, etas)."""
        v = self._contig(vars)
        c = self._coeff_into(v["proj"], torch.empty_like(v["proj"]))
        self._gradient_pass(c, v["pos"], v["prb"])
        y_is_z = grads["prb"] is etas["prb"]
        g, e = self._contig(grads), self._contig(etas)
        cy = self._coeff_into(g["proj"], torch.empty_like(g["proj"]))
        y = (cy, g["pos"], g["prb"])
        if y_is_z:
            return float(self._hessian_pass(c, v["pos"], v["prb"], y)[0])
        cz = self._coeff_into(e["proj"], torch.empty_like(e["proj"]))
        return float(self._hessian_pass(c, v["pos"], v["prb"], y, (cz, e["pos"], e["prb"]))[1])

    # ------------------------------------------------- probe-fit term
    def gradient_prbfit(self, grad_prb, prb):
        """rec_mpi.py:365-377: grad_prb += rho lam/N D^H(2 (D prb - ref D prb/|D prb|)) (ht_prbfit_grad)."""
        if self.lam_prbfit == 0:
            return
        scale = float(np.float32(self.lam_prbfit / self.prb_size) * np.float32(self.rho_sq["prb"]))
        _lib.call("ht_prbfit_grad", self.cl_prop._h, _lib.ptr(prb.contiguous()), _lib.ptr(self.ref),
                  _lib.ptr(self._pfw), _lib.ptr(grad_prb), scale, _lib.stream_ptr())

    def _prbfit_forms_dev(self, prb, d1, d2, out, hess_slots):
        """hessian_prbfit (rec_mpi.py:379-398) on the device (ht_prbfit_forms): the
        forms of (d1,d1), (d1,d2), (d2,d2) into out[0..2], or added to the BH
        Hessian slots of out (hess_slots)."""
        _lib.call("ht_prbfit_forms", self.cl_prop._h, _lib.ptr(prb.contiguous()), _lib.ptr(d1.contiguous()),
                  _lib.ptr(d2.contiguous()) if d2 is not None else None, _lib.ptr(self.ref), _lib.ptr(self._pfw),
                  out, self.lam_prbfit / self.prb_size, int(hess_slots), _lib.stream_ptr())

    def hessian_prbfit(self, prb, dprb1, dprb2):
        """rec_mpi.py:380-398: the probe-fit term's Hessian form at prb for
        (dprb1, dprb2), summed in float64; 0 when lam_prbfit is 0."""
        return self._prbfit_forms(prb, dprb1, dprb2)[1]

    def _prbfit_forms(self, prb, d1, d2):
        """hessian_prbfit (rec_mpi.py:379-398) for the pairs (d1,d1), (d1,d2), (d2,d2)
        (d2 None: d1 for both)."""
        if self.lam_prbfit == 0:
            return 0.0, 0.0, 0.0
        self._prbfit_forms_dev(prb, d1, d2, _lib.ptr(self._pf3), 0)
        f = [float(v) for v in self._pf3.cpu().numpy()]
        return (f[0], f[1], f[2]) if d2 is not None else (f[0], f[0], f[0])

    # ------------------------------------------ 3-D Laplacian regulariser
    # rec_mpi.py:402-496 (ht_laplacian_*): gradient 2 lam/N B vars obj, Hessian
    # form 2 lam/N Re<d, B etas obj> (the current etas obj, as the reference
    # has it), energy lam/N |L vars obj|^2 over the object slices.
    def _lap_args(self):
        return self.nzobj, self.nobj, self.nobj, 1 if self.complex_obj else 0

    def gradient_laplacian(self, grad_obj):
        """rec_mpi.py:419-442"""
        if self.lam_laplacian == 0:
            return
        scale = float(np.float32(2.0 * self.lam_laplacian / self.obj_size))
        _lib.call("ht_laplacian_grad", _lib.ptr(self.vars["obj"]), _lib.ptr(grad_obj), *self._lap_args(), scale,
                  _lib.ptr(self._lapw), _lib.stream_ptr())

    def _lap_form(self, y, z, out, y2=None, out2=None):
        """out += 2 lam/N Re<y, B z> (and out2 += ... for y2) on the device."""
        _lib.call("ht_laplacian_dot", _lib.ptr(y), _lib.ptr(z), *self._lap_args(),
                  2.0 * self.lam_laplacian / self.obj_size, _lib.ptr(self._lapw), out,
                  _lib.ptr(y2) if y2 is not None else None, out2, _lib.stream_ptr())

    def hessian_laplacian(self, dobj1):
        """rec_mpi.py:444-470"""
        if self.lam_laplacian == 0:
            return 0.0
        acc = torch.zeros(1, dtype=torch.float64, device=self.device)
        self._lap_form(dobj1.contiguous(), self.etas["obj"], _lib.ptr(acc))
        return float(acc)

    def _lap_energy_local(self):
        """rec_mpi.py:472-496 under the reference's name (one GPU holds the
        whole object, so the local energy is the energy)."""
        return self._lap_energy()

    def _lap_energy(self):
        """rec_mpi.py:472-496"""
        if self.lam_laplacian == 0:
            return 0.0
        acc = torch.zeros(1, dtype=torch.float64, device=self.device)
        _lib.call("ht_laplacian_energy", _lib.ptr(self.vars["obj"]), *self._lap_args(),
                  self.lam_laplacian / self.obj_size, _lib.ptr(self._lapw), _lib.ptr(acc), _lib.stream_ptr())
        return float(acc)

    # ----------------------------------------------------- forward use
    def fwd_tomo(self, obj, out=None):
        """rec_mpi.py:498-507"""
        return self.cl_tomo.R(obj, out=out)

    def min(self, prb, obj, pos, proj, prbfit_only=False):
        """rec_mpi.py:815-835: data term + probe-fit term."""
        out = 0.0
        if not prbfit_only:
            c = self._coeff_into(proj.contiguous(), torch.empty_like(proj))
            out = self._forward(c, pos.contiguous(), self.eff_demagnifications, prb.contiguous(),
                                data=self.data) / self.data_size
        if self.lam_prbfit != 0:
            for j in range(self.ndist):
                Dprb = self.cl_prop.D(prb[j: j + 1].contiguous(), j)[0]
                out += self.lam_prbfit / self.prb_size * float(torch.linalg.norm(torch.abs(Dprb) - self.ref[j])) ** 2
        if not prbfit_only:
            out += self._lap_energy()   # of vars obj, as the reference's min has it
        return out

    def gen_sqrt_data(self, vars, out):
        """rec_mpi.py:882-897 (note: before the first BH() call the reference's
        eff_demagnifications is still zero, rec_mpi.py:135-136, and so is it here)."""
        vars["obj"] /= self.norm_const
        self.fwd_tomo(vars["obj"], out=vars["proj"])
        c = self._coeff_into(vars["proj"], torch.empty_like(vars["proj"]))
        self._forward(c, vars["pos"], self.eff_demagnifications, vars["prb"], amp=out)
        vars["obj"] *= self.norm_const

    def forward_amplitudes(self, obj, prb, pos, out=None):
        """|F1(F2(F3(prb, R(obj / norm_const), pos)))| with the physical
        magnifications 1 / norm_magnifications: the synthetic-data forward model
        (gen_sqrt_data without the zero-magnification start state)."""
        eff = torch.empty(self.ntheta, self.ndist, dtype=torch.float32, device=self.device)
        eff[:] = _t(1.0 / np.asarray(self.norm_magnifications, dtype=np.float64)[None, :], self.device, torch.float32)
        proj = self.fwd_tomo((obj / self.norm_const).to(self.odt).contiguous())
        c = self._coeff_into(proj, torch.empty_like(proj))
        del proj
        if out is None:
            out = torch.empty(self.ntheta, self.ndist, self.nz, self.n, dtype=torch.float32, device=self.device)
        self._forward(c, pos.contiguous(), eff, prb.contiguous(), amp=out)
        return out

    def gen_sqrt_ref(self, prb, out):
        """rec_mpi.py:899-902"""
        for j in range(self.ndist):
            out[j] = torch.abs(self.cl_prop.D(prb[j: j + 1].contiguous(), j)[0])

    # ------------------------------------------------------------ BH
    def BH(self, writer=None, niter=None, record=None, mode="host"):
        """rec_mpi.py:138-232.  ``record`` (a list) receives (iteration, alpha, beta).

        mode="host" iterates as the reference does (step sizes on the host).
        mode="graph" keeps the step sizes on the device and replays the
        steady-state iteration from a CUDA graph (same arithmetic; complex
        objects, no error table and no checkpoints -- otherwise it iterates as
        "host": the real-object iteration allocates temporaries, which a
        recorded graph must not refer to).  ``writer``
        (checkpoint.Writer) saves obj/prb/pos every vis_step iterations
        (rec_mpi.py:837-860, vis_debug)."""
        self.bh_setup()
        niter = self.niter if niter is None else niter
        checkpoints = writer is not None and getattr(self, "vis_step", -1) not in (-1, 0, None)
        if (mode == "graph" and self.graphable and self.err_step == -1 and not checkpoints
                and niter > self.start_iter):
            self.reserve_history(niter - self.start_iter)
            cur = torch.cuda.current_stream(self.device)
            side = torch.cuda.Stream(device=self.device)
            side.wait_stream(cur)
            with torch.cuda.stream(side):
                self.bh_iteration(self.start_iter, sync=False)
                if niter - self.start_iter > 1:
                    self.capture_iteration()
                    for _ in range(self.start_iter + 1, niter):
                        self.replay_iteration()
                    self.release_graph()
            cur.wait_stream(side)
            if record is not None:
                for k, (a, b) in enumerate(self.bh_history()):
                    record.append((self.start_iter + k, float(a), float(b)))
            return self.bh_finish()
        for i in range(self.start_iter, niter):
            a, b = self.bh_iteration(i)
            if record is not None:
                record.append((i, a, b))
            self.error_debug(self.vars, i)
            if checkpoints:
                self.vis_debug(self.vars, i, writer)
        return self.bh_finish()

    def bh_setup(self):
        """Start of BH (rec_mpi.py:139-162): magnifications, normalisation, mask,
        proj = R(obj) and its B-spline coefficients."""
        vars, C = self.vars, self._c
        self.eff_demagnifications[:] = (1 + self.shrink_nd) / _t(self.norm_magnifications[None, :], self.device,
                                                                 torch.float32)
        vars["obj"] /= self.norm_const
        if self.start_iter == 0:
            vars["obj"] *= self.cl_tomo.mask
        self.pos_init = vars["pos"].clone()   # rec_mpi.py:153, for vis_debug's drift
        self.fwd_tomo(vars["obj"], out=vars["proj"])
        self._coeff_into(vars["proj"], C["vars"])
        self.error_debug(vars, -1)
        self.time_start = time.time()
        self._count.zero_()

    def bh_finish(self):
        """End of BH (rec_mpi.py:229-232).  With the folded prefilter the proj
        arrays, which are R of the obj arrays, are recomputed here."""
        if self._fold:
            for d in (self.vars, self.grads, self.etas):
                self.fwd_tomo(d["obj"], out=d["proj"])
        self.vars["obj"] *= self.norm_const
        return self.vars

    def bh_iteration(self, i, sync=True):
        """One BH iteration (rec_mpi.py:163-227); returns (alpha, beta).

        sync=False keeps alpha and beta on the device (ht_bh_scalars,
        ht_axpby_dev): the iteration then makes no host round trip and can be
        recorded into a CUDA graph; it returns None and appends the step sizes
        to the device history (bh_history())."""
        vars, grads, etas, C = self.vars, self.grads, self.etas, self._c
        rho = self.rho_sq
        dots = self._dots
        first = i == self.start_iter
        # ---- gradients (rec_mpi.py:305-325); the variable scalings rho are
        # applied inside the library passes, so no separate elementwise pass runs
        gc, _, _ = self._gradient_pass(C["vars"], vars["pos"], vars["prb"], persistent=True, gpos=grads["pos"],
                                       gprb=grads["prb"], scale_pos=rho["pos"], scale_prb=rho["prb"])
        if self._fold:
            # grads obj = rho R^T coeff(gc) = rho Cz R^T Cx gc;  C grads = coeff(R grads obj) = Cx R Cz grads obj
            st, nc = _lib.stream_ptr(), self.nobj * self.nobj
            self.cl_tomo._RT_into(gc, grads["obj"], coeffx=True, scale=rho["obj"])
            _lib.call("ht_shift_coeff_z", self.cl_shift._hc, _lib.ptr(grads["obj"]), _lib.ptr(grads["obj"]), nc, st)
            self.gradient_laplacian(grads["obj"])
            self.gradient_prbfit(grads["prb"], vars["prb"])
            _lib.call("ht_shift_coeff_z", self.cl_shift._hc, _lib.ptr(grads["obj"]), _lib.ptr(self._vol), nc, st)
            self.cl_tomo._R_into(self._vol, C["grads"], coeffx=True)
        else:
            self._coeff_into(gc, grads["proj"])
            grads["proj"] *= rho["obj"]
            self.cl_tomo.RT(grads["proj"], out=grads["obj"])               # gF4
            self.gradient_laplacian(grads["obj"])
            self.gradient_prbfit(grads["prb"], vars["prb"])
            self.fwd_tomo(grads["obj"], out=grads["proj"])
            self._coeff_into(grads["proj"], C["grads"])
        # ---- Hessian forms (rec_mpi.py:180-213)
        y = (C["grads"], grads["pos"], grads["prb"])
        z = None if first else (C["etas"], etas["pos"], etas["prb"])
        H = self._hessian_pass(C["vars"], vars["pos"], vars["prb"], y, z, out=self._H)
        if self.lam_laplacian != 0:
            # the regulariser's forms (B symmetric): H(g,g); H(g,eta) in both the
            # reference's and the symmetric slot; H(eta,eta)
            hp = H.data_ptr()
            self._lap_form(grads["obj"], grads["obj"], ctypes.c_void_p(hp))
            if not first:
                self._lap_form(grads["obj"], etas["obj"], ctypes.c_void_p(hp + 8), etas["obj"],
                               ctypes.c_void_p(hp + 16))
                self._lap_form(grads["obj"], etas["obj"], ctypes.c_void_p(hp + 24))
        if sync:
            return self._bh_update_host(H.cpu().numpy(), first)
        if self.lam_prbfit != 0:
            # the probe-fit forms added to the Hessian slots on the device
            self._prbfit_forms_dev(vars["prb"], grads["prb"], None if first else etas["prb"], _lib.ptr(H), 1)
        # ---- the same with the step sizes on the device
        st = _lib.stream_ptr()
        bh = self._bh
        rr = (float(rho["obj"]), float(rho["pos"]), float(rho["prb"]))
        # phase 0: beta, and the dots cleared for the direction updates below
        _lib.call("ht_bh_scalars", _lib.ptr(H), _lib.ptr(dots), int(first), 0, *rr, _lib.ptr(bh), None, 0, None, st)
        beta = _lib.ptr(bh)
        for k, v in enumerate(("obj", "pos", "prb")):
            self._axpby_dev(etas[v], grads[v], beta, 1.0, None, -1.0, dots[k:k + 1])
        if not self._fold:
            self._axpby_dev(etas["proj"], grads["proj"], beta, 1.0, None, -1.0)
        self._axpby_dev(C["etas"], C["grads"], beta, 1.0, None, -1.0)
        _lib.call("ht_bh_scalars", _lib.ptr(H), _lib.ptr(dots), int(first), 1, *rr, _lib.ptr(bh),
                  _lib.ptr(self._hist), self._hist_cap, _lib.ptr(self._count), st)
        alpha = ctypes.c_void_p(bh.data_ptr() + 8)
        for v in ("obj", "prb", "pos") + (() if self._fold else ("proj",)):
            self._axpby_dev(vars[v], etas[v], None, 1.0, alpha, 1.0)
        self._axpby_dev(C["vars"], C["etas"], None, 1.0, alpha, 1.0)
        return None

    def _axpby_dev(self, x, y, A, sa, B, sb, dot=None):
        n = x.numel() * (2 if x.is_complex() else 1)
        _lib.call("ht_axpby_dev", _lib.ptr(x), _lib.ptr(y), A, float(sa), B, float(sb), n,
                  _lib.ptr(dot) if dot is not None else None, _lib.stream_ptr())

    def _bh_update_host(self, H, first):
        """Direction and variable updates with host step sizes (rec_mpi.py:180-218)."""
        vars, grads, etas, C = self.vars, self.grads, self.etas, self._c
        rho = self.rho_sq
        dots = self._dots
        if first:
            beta = 0.0
            pf = self._prbfit_forms(vars["prb"], grads["prb"], None)
            Hgg = H[0] + pf[0]
        else:
            pf = self._prbfit_forms(vars["prb"], grads["prb"], etas["prb"])
            Hgg, Hge, Hee, Hge_sym = H[0] + pf[0], H[1] + pf[1], H[2] + pf[2], H[3] + pf[1]
            beta = Hge / Hee
        # ---- conjugate direction and step (rec_mpi.py:196-218)
        dots.zero_()
        self._axpby(etas["obj"], grads["obj"], beta, -1, dots[0:1])
        self._axpby(etas["pos"], grads["pos"], beta, -1, dots[1:2])
        self._axpby(etas["prb"], grads["prb"], beta, -1, dots[2:3])
        if not self._fold:
            self._axpby(etas["proj"], grads["proj"], beta, -1)
        self._axpby(C["etas"], C["grads"], beta, -1)
        d = dots.cpu().numpy()
        top = -(d[0] / rho["obj"] + d[1] / rho["pos"] + d[2] / rho["prb"])
        bottom = Hgg if first else beta * beta * Hee - 2 * beta * Hge_sym + Hgg
        alpha = top / bottom
        for v in ("obj", "prb", "pos") + (() if self._fold else ("proj",)):
            self._axpby(vars[v], etas[v], 1, alpha)
        self._axpby(C["vars"], C["etas"], 1, alpha)
        return float(alpha), float(beta)

    def bh_history(self):
        """(alpha, beta) of the device-scalar iterations since bh_setup()."""
        n = min(int(self._count.item()), self._hist_cap)
        return [tuple(r) for r in self._hist[:n].cpu().numpy()]

    def reserve_history(self, n):
        """Room for n device-side (alpha, beta) pairs (4096 by default; the
        pairs beyond the room are counted but not kept).  A larger history
        replaces the buffer, so the recorded graph, which refers to the old
        one, is released: call before recording."""
        if n > self._hist_cap:
            self.release_graph()
            old, k = self._hist, self._hist_cap
            self._hist_cap = int(n)
            self._hist = torch.zeros(self._hist_cap, 2, dtype=torch.float64, device=self.device)
            self._hist[:k].copy_(old)

    def capture_iteration(self):
        """Record one steady-state device-scalar iteration (not the first) on
        the current stream into a CUDA graph; replay_iteration() then runs it
        with one launch.  Call after one iteration has run on this device (so
        every kernel's launch attributes are set).  Recording runs nothing.
        Complex objects only (graphable): the real-object iteration allocates
        temporaries from the caching allocator, which may hand that memory to
        another tensor, or release it, while the graph still writes there."""
        if not self.graphable:
            raise ValueError("capture_iteration: the real-object (float32) iteration allocates temporaries "
                             "and cannot be recorded; use bh_iteration(i, sync=False)")
        self.release_graph()
        st = _lib.stream_ptr()
        gc_on = gc.isenabled()
        gc.disable()   # no collector-driven destructors (device frees) while recording
        _lib.call("ht_graph_begin", st)
        try:
            self.bh_iteration(self.start_iter + 1, sync=False)
        finally:
            ex = ctypes.c_void_p()
            _lib.call("ht_graph_end", st, ctypes.byref(ex))
            if gc_on:
                gc.enable()
        self._graph = ex
        return ex

    def replay_iteration(self):
        """Run the recorded iteration on the current stream."""
        _lib.call("ht_graph_launch", self._graph, _lib.stream_ptr())

    def release_graph(self):
        if getattr(self, "_graph", None) is not None:
            _lib.lib().ht_graph_destroy(self._graph)
            self._graph = None

    def vis_debug(self, vars, i, writer=None):
        """rec_mpi.py:837-860: every vis_step iterations after the first, the
        state goes to the checkpoint writer and the mean absolute drift of the
        positions from their values at the start of BH is logged for each
        distance.  Without a writer nothing happens (the reference draws the
        state with matplotlib there)."""
        if writer is None or self.vis_step in (-1, 0, None) or i % self.vis_step != 0 or i <= self.start_iter:
            return
        writer.write_checkpoint(vars, i, self.norm_const)
        if getattr(self, "pos_init", None) is not None:
            d = position_drift(vars["pos"], self.pos_init)
            _log.warning("iteration %d: mean absolute position drift [px] %s", i,
                         "; ".join(f"distance {j}: y {d[j, 0]:.4f} x {d[j, 1]:.4f}" for j in range(len(d))))

    def error_debug(self, vars, i):
        """rec_mpi.py:862-880: a row of the convergence table self.table."""
        if self.err_step == -1 or i % self.err_step != 0:
            return
        if self._fold and i >= 0:   # proj is not kept up to date inside BH: use its coefficients
            err = self._forward(self._c["vars"], vars["pos"], self.eff_demagnifications, vars["prb"],
                                data=self.data) / self.data_size + self._lap_energy()
            if self.lam_prbfit != 0:
                err += self.min(vars["prb"], None, vars["pos"], None, prbfit_only=True)
        else:
            err = self.min(vars["prb"], vars["obj"], vars["pos"], vars["proj"])
        log_error(self, i, err, "conv.csv")

    def gradients(self, vars, grads):
        """rec_mpi.py:305-325"""
        self.gradients_cascade(vars, grads)
        self.cl_tomo.RT(grads["proj"].contiguous(), out=grads["obj"])
        self.gradient_laplacian(grads["obj"])
        self.gradient_prbfit(grads["prb"], vars["prb"])

    def hessian(self, vars, grads, etas):
        """rec_mpi.py:234-248"""
        w = self.hessian_cascade(vars, grads, etas)
        if self.lam_prbfit != 0:
            w += self._prbfit_forms(vars["prb"], grads["prb"], etas["prb"])[1]
        return w + self.hessian_laplacian(grads["obj"])

    # ====================== cascade functions, operator by operator
    # (rec_mpi.py:517-813; used for derivative checks, not by BH())
    # F0 and its derivatives are scalar reductions: evaluated in float64
    @staticmethod
    def _d64(*a):
        return [None if v is None else (v.to(torch.complex128) if v.is_complex() else v.double()) for v in a]

    def F0(self, x, d):
        x, d = self._d64(x, d)
        t = torch.abs(x) - d
        return float(torch.sum(t * t)) / self.data_size

    def dF0(self, x, y, d, return_x=False):
        x, y, d = self._d64(x, y, d)
        return 2 / self.data_size * redot(x - d * (x / torch.abs(x)), y)

    def d2F_dF0(self, x, y, z, w, d):
        x, y, z, w, d = self._d64(x, y, z, w, d)
        absval = torch.abs(x)
        l0 = x / absval
        d0 = d / absval
        v = (1 - d0) * reprod(y, z) + d0 * reprod(l0, y) * reprod(l0, z)
        if w is not None:
            v = v + reprod(x - d * l0, w)
        return 2 / self.data_size * float(torch.sum(v))

    def gF0(self, x, y):
        for i in range(1, 4)[::-1]:
            x = self.F[i](x)
        return np.float32(2 / self.data_size) * (x - y * (x / torch.abs(x)))

    def _D(self, a, j, adj=False):
        a = a.contiguous()
        return self.cl_prop.DT(a, j) if adj else self.cl_prop.D(a, j)

    def F1(self, x):
        x11, x12 = x
        x0 = torch.empty(x12.shape[0], self.ndist, self.nz, self.n, dtype=torch.complex64, device=x12.device)
        for j in range(self.ndist):
            x0[:, j] = self._D(x11[j] * x12[:, j], j)
        return x0

    def dF1(self, x, y, return_x=True):
        x11, x12 = x
        y11, y12 = y
        y0 = (y11[None] * x12 + x11[None] * y12).to(torch.complex64)
        for j in range(self.ndist):
            y0[:, j] = self._D(y0[:, j], j)
        if return_x:
            return self.F1(x), y0
        return y0

    def d2F_dF1(self, x, y, z, w):
        x11, x12 = x
        y11, y12 = y
        z11, z12 = z
        w11, w12 = w
        y0 = 2 * y11[None] * y12 if y12 is z12 else y11[None] * z12 + z11[None] * y12
        if w11 is not None:
            y0 = y0 + w11[None] * x12
        if w12 is not None:
            y0 = y0 + x11[None] * w12
        y0 = y0.to(torch.complex64)
        for j in range(self.ndist):
            y0[:, j] = self._D(y0[:, j], j)
        return y0

    def gF1(self, x, y):
        y0 = y
        for i in range(2, 4)[::-1]:
            x = self.F[i](x)
        x11, x12 = x
        y12 = torch.empty(y0.shape[0], self.ndist, self.nz, self.n, dtype=torch.complex64, device=y0.device)
        for j in range(self.ndist):
            y12[:, j] = self._D(y0[:, j], j, adj=True)
        y11 = torch.sum(y12 * torch.conj(x12), dim=0)
        y12 = y12 * torch.conj(x11[None])
        return y11, y12

    @staticmethod
    def _cexp(x22):
        return torch.exp(1j * x22.to(torch.complex64))

    def F2(self, x):
        x21, x22 = x
        return x21, self._cexp(x22)

    def dF2(self, x, y, return_x=True):
        x21, x22 = x
        y21, y22 = y
        x12 = self._cexp(x22)
        y12 = x12 * 1j * y22
        return ([x21, x12], [y21, y12]) if return_x else [y21, y12]

    def d2F_dF2(self, x, y, z, w):
        x21, x22 = x
        y21, y22 = y
        z21, z22 = z
        w21, w22 = w
        e = self._cexp(x22)
        y12 = e * (-y22 * z22)
        if w22 is not None:
            y12 = y12 + e * 1j * w22
        return [w21, y12]

    def gF2(self, x, y):
        y11, y12 = y
        x21, x22 = self.F3(x)
        y22 = (-1j) * y12 * torch.conj(self._cexp(x22))
        y22 = y22.real if not self.complex_obj else y22
        return [y11, y22]

    def _eff(self, k):
        return self.eff_demagnifications[:, k].contiguous()

    def F3(self, x):
        x31, x32, x33 = x
        x22 = torch.empty(len(x33), self.ndist, self.nz, self.n, dtype=self.odt, device=x32.device)
        c = self.cl_shift.coeff(x32)
        for k in range(self.ndist):
            x22[:, k] = self.cl_shift.curlySc(c, x33[:, k], self._eff(k))
        return [x31, x22]

    def dF3(self, x, y, return_x=True):
        x31, x32, x33 = x
        y31, y32, y33 = y
        y22 = torch.zeros(len(y32), self.ndist, self.nz, self.n, dtype=self.odt, device=y32.device)
        c = self.cl_shift.coeff(x32)
        c1 = self.cl_shift.coeff(y32)
        for k in range(self.ndist):
            y22[:, k] = self.cl_shift.dcurlySc(c, x33[:, k], self._eff(k), c1, y33[:, k])
        if return_x:
            return self.F3(x), [y31, y22]
        return [y31, y22]

    def d2F_dF3(self, x, y, z, w):
        x31, x32, x33 = x
        y31, y32, y33 = y
        z31, z32, z33 = z
        w31, w32, w33 = w
        y22 = torch.zeros(len(y32), self.ndist, self.nz, self.n, dtype=self.odt, device=y32.device)
        c = self.cl_shift.coeff(x32)
        cy = self.cl_shift.coeff(y32)
        cz = self.cl_shift.coeff(z32)
        for k in range(self.ndist):
            y22[:, k] = self.cl_shift.d2curlySc(c, x33[:, k], self._eff(k), cy, y33[:, k], cz, z33[:, k])
        if w32 is not None:
            cw = self.cl_shift.coeff(w32)
            for k in range(self.ndist):
                y22[:, k] += self.cl_shift.dcurlySc(c, x33[:, k], self._eff(k), cw, w33[:, k])
        return [w31, y22]

    def gF4(self, gradu, gradproj):
        """rec_mpi.py:356-362: gradu = R^T gradproj, the object gradient from
        the projections' gradient."""
        self.cl_tomo.RT(gradproj.contiguous(), out=gradu)
        return gradu

    def gF3(self, x, y):
        y21, y22 = y
        x31, x32, x33 = x
        y32 = torch.zeros(y22.shape[0], self.nzobj, self.nobj, dtype=self.odt, device=y22.device)
        y33 = torch.empty(y22.shape[0], self.ndist, 2, dtype=torch.float32, device=y22.device)
        c = self.cl_shift.coeff(x32)
        for k in range(self.ndist):
            dpsi, dr = self.cl_shift.dcurlySadjc(c, x33[:, k], self._eff(k), y22[:, k].contiguous())
            y32 += dpsi
            y33[:, k] = dr
        y32 = self.cl_shift.coeff(y32)
        return [y21, y32, y33]
