"""Near-field ptychography (drop-in for holotomocupy's RecNFP).

Reference: ``src/holotomocupy/rec_nfp_mpi.py:20-469`` (single rank).  One 2-D
projection ``proj`` [nzobj, nobj] is illuminated by the probe ``prb`` [nz, n]
at ``ntheta`` scan positions ``pos`` [ntheta, 2] and recorded at one
propagation distance:

    x0[theta] = D( prb * exp(i S_{pos[theta]}(coeff(proj))) ),   F = 1/N sum (|x0| - d)^2

with the Bilinear-Hessian (BH) solver over (prb, proj, pos).  The same fused
cascade as ``Rec`` does the work (``ht_rec_gradient`` / ``ht_rec_hessian``):
the handle is created for ntheta "angles" at one distance and told that the
coefficient array is shared by every position
(``ht_rec_set_shared_coefficients``), so the projection's gradient comes back
summed over the positions and nothing is tiled.  Inner products, the Hessian
forms and the step sizes are float64.

Kept from the reference: the constructor ``RecNFP(args)`` with its argument
keys, the ``vars`` / ``grads`` / ``etas`` dictionaries (CUDA torch tensors),
``BH``, ``gradients``, ``gradients_cascade``, ``hessian``,
``hessian_cascade``, ``min``, ``gen_sqrt_data`` and the convergence table.
The operator-by-operator ``F*`` / ``dF*`` / ``d2F_dF*`` / ``gF*`` functions are
not kept (the fused passes replace them; ``Rec`` has them for the 3-D case).
"""
import ctypes
import gc
import time

import numpy as np
import torch

from . import _lib
from .convtable import log_error, new_table
from .propagation import Propagation
from .shift import Shift


class RecNFP:
    """Near-field ptychography reconstruction (rec_nfp_mpi.py:20)."""

    def __init__(self, args):
        for key, value in vars(args).items():
            setattr(self, key, value)
        self.device = torch.device("cuda", torch.cuda.current_device())
        if getattr(self, "distance", None) is None:                 # rec_nfp_mpi.py:56-61
            wavelength = 1.24e-09 / self.energy
            z1 = float(np.asarray(self.z1).ravel()[0])
            z2 = self.focustodetectordistance - z1
            magnification = self.focustodetectordistance / z1
            distance = z1 * z2 / self.focustodetectordistance
            voxelsize = self.detector_pixelsize / magnification
        else:
            wavelength, voxelsize = self.wavelength, self.voxelsize
            distance = float(np.asarray(self.distance).ravel()[0])
        self.rho_sq = {"proj": args.rho[0] ** 2, "prb": args.rho[1] ** 2, "pos": args.rho[2] ** 2}
        self.complex_obj = self.obj_dtype == "complex64"
        self.odt = torch.complex64 if self.complex_obj else torch.float32
        self.cl_prop = Propagation(self.n, self.nz, self.ntheta, 1, wavelength, voxelsize, np.array([distance]))
        self.cl_shift = Shift(self.n, self.nobj, self.nz, self.nzobj, self.obj_dtype)
        self.data_size = self.ntheta * self.nz * self.n
        self.prb_size = self.nz * self.n
        self.table = new_table()
        self.alloc_arrays()
        h = ctypes.c_void_p()
        _lib.call("ht_rec_create", self.n, self.nz, self.nobj, self.nzobj, self.ntheta, 1,
                  1 if self.complex_obj else 0, self.cl_prop._h, ctypes.byref(h))
        self._h = h
        _lib.call("ht_rec_set_shared_coefficients", h, 1)

    def alloc_arrays(self):
        """rec_nfp_mpi.py:86-98 (device-resident, zero-initialised)."""
        dev, odt = self.device, self.odt
        z = lambda *s, dt=odt: torch.zeros(*s, dtype=dt, device=dev)
        self.vars = {"prb": z(self.nz, self.n, dt=torch.complex64), "proj": z(self.nzobj, self.nobj),
                     "pos": z(self.ntheta, 2, dt=torch.float32)}
        self.data = z(self.ntheta, self.nz, self.n, dt=torch.float32)
        self.grads, self.etas = {}, {}
        for ge in (self.grads, self.etas):
            ge["prb"] = z(self.nz, self.n, dt=torch.complex64)
            ge["proj"] = z(self.nzobj, self.nobj)
            ge["pos"] = z(self.ntheta, 2, dt=torch.float32)
        self._mag = torch.ones(self.ntheta, 1, dtype=torch.float32, device=dev)   # rec_nfp_mpi.py:357
        self._c = {k: z(self.nzobj, self.nobj) for k in ("vars", "grads", "etas")}
        self._gc = z(self.nzobj, self.nobj)
        self._scal = torch.zeros(2, dtype=torch.float64, device=dev)
        self._H = torch.zeros(4, dtype=torch.float64, device=dev)
        self._dots = torch.zeros(4, dtype=torch.float64, device=dev)
        self._bh = torch.zeros(2, dtype=torch.float64, device=dev)
        self._scratch = (z(self.ntheta, 2, dt=torch.float32), z(self.nz, self.n, dt=torch.complex64))
        # the device-side step-size history of the graph-replayed iterations
        self._hist_cap = 4096
        self._hist = z(self._hist_cap, 2, dt=torch.float64)
        self._count = z(1, dt=torch.int32)
        self._graph = None

    def close(self):
        try:
            self.release_graph()
        except Exception:
            pass
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().ht_rec_destroy(h)
            except Exception:
                pass
            self._h = None

    def __del__(self):
        self.close()

    # ------------------------------------------------------------- passes
    def _coeff(self, proj, out):
        """out = coeff(proj) (shift.py:74-82) for one [nzobj, nobj] array."""
        if self.complex_obj:
            _lib.call("ht_shift_coeff", self.cl_shift._hc, _lib.ptr(proj), _lib.ptr(out), 1, _lib.stream_ptr())
        else:
            out.copy_(self.cl_shift.coeff(proj[None])[0])
        return out

    def _gradient_pass(self, c, pos, prb, gpos, gprb, spos=1.0, sprb=1.0):
        """Fused gF0..gF3 (rec_nfp_mpi.py:186-216): gc (summed over positions)
        into self._gc, gpos, gprb (times spos, sprb); F's sum in _scal[0]."""
        _lib.call("ht_rec_gradient", self._h, _lib.ptr(c), _lib.ptr(pos), _lib.ptr(self._mag), _lib.ptr(prb),
                  _lib.ptr(self.data), _lib.ptr(self._gc), _lib.ptr(gpos), _lib.ptr(gprb), _lib.ptr(self._scal),
                  float(spos), float(sprb), 0, _lib.stream_ptr())

    def _hessian_pass(self, c, pos, prb, y, z=None):
        """Hessian forms at the last gradient pass's point for the directions
        y, z = (coefficients, pos, prb): [H(y,y), H_ref(y,z), H(z,z), H_sym(y,z)]."""
        zz = z if z is not None else (None, None, None)
        _lib.call("ht_rec_hessian", self._h, _lib.ptr(c), _lib.ptr(pos), _lib.ptr(self._mag), _lib.ptr(prb),
                  _lib.ptr(self.data), 2 if z is not None else 1, _lib.ptr(y[0]), _lib.ptr(y[1]), _lib.ptr(y[2]),
                  _lib.ptr(zz[0]) if z is not None else None, _lib.ptr(zz[1]) if z is not None else None,
                  _lib.ptr(zz[2]) if z is not None else None, _lib.ptr(self._H), 0, _lib.stream_ptr())
        return self._H

    # ----------------------------------------------------- reference API
    def gradients_cascade(self, vars, grads):
        """rec_nfp_mpi.py:192-216: grads prb / proj / pos (unscaled)."""
        c = self._coeff(vars["proj"].contiguous(), torch.empty_like(self._gc))
        self._gradient_pass(c, vars["pos"].contiguous(), vars["prb"].contiguous(), grads["pos"], grads["prb"])
        self._coeff(self._gc, grads["proj"])

    def gradients(self, vars, grads):
        """rec_nfp_mpi.py:186-189 (one rank: the reductions are the identity)."""
        self.gradients_cascade(vars, grads)

    def hessian_cascade(self, vars, grads, etas):
        """rec_nfp_mpi.py:151-184: the Hessian form at vars for (grads, etas)."""
        c = self._coeff(vars["proj"].contiguous(), torch.empty_like(self._gc))
        sp, sq = self._scratch
        pos, prb = vars["pos"].contiguous(), vars["prb"].contiguous()
        self._gradient_pass(c, pos, prb, sp, sq)
        cy = self._coeff(grads["proj"].contiguous(), torch.empty_like(self._gc))
        y = (cy, grads["pos"].contiguous(), grads["prb"].contiguous())
        if grads["prb"] is etas["prb"]:
            return float(self._hessian_pass(c, pos, prb, y)[0])
        cz = self._coeff(etas["proj"].contiguous(), torch.empty_like(self._gc))
        return float(self._hessian_pass(c, pos, prb, y, (cz, etas["pos"].contiguous(), etas["prb"].contiguous()))[1])

    def hessian(self, vars, grads, etas):
        """rec_nfp_mpi.py:146-147"""
        return self.hessian_cascade(vars, grads, etas)

    def min(self, prb, proj, pos):
        """rec_nfp_mpi.py:407-420: the data term."""
        c = self._coeff(proj.contiguous(), torch.empty_like(self._gc))
        _lib.call("ht_rec_forward", self._h, _lib.ptr(c), _lib.ptr(pos.contiguous()), _lib.ptr(self._mag),
                  _lib.ptr(prb.contiguous()), _lib.ptr(self.data), None, _lib.ptr(self._scal), _lib.stream_ptr())
        return float(self._scal[0]) / self.data_size

    def gen_sqrt_data(self, vars, out):
        """rec_nfp_mpi.py:460-469: out = |x0| at vars."""
        c = self._coeff(vars["proj"].contiguous(), torch.empty_like(self._gc))
        _lib.call("ht_rec_forward", self._h, _lib.ptr(c), _lib.ptr(vars["pos"].contiguous()), _lib.ptr(self._mag),
                  _lib.ptr(vars["prb"].contiguous()), None, _lib.ptr(out), None, _lib.stream_ptr())

    def error_debug(self, vars, i):
        """rec_nfp_mpi.py:442-458: a row of the convergence table self.table."""
        if self.err_step == -1 or i % self.err_step != 0:
            return
        err = self.min(vars["prb"], vars["proj"], vars["pos"])
        log_error(self, i, err, "conv_nfp.csv")

    # ------------------------------------------------------------------ BH
    def _axpby(self, x, y, a, b, dot=None):
        n = x.numel() * (2 if x.is_complex() else 1)
        _lib.call("ht_axpby", _lib.ptr(x), _lib.ptr(y), float(a), float(b), n,
                  _lib.ptr(dot) if dot is not None else None, _lib.stream_ptr())

    def _axpby_dev(self, x, y, A, sa, B, sb, dot=None):
        n = x.numel() * (2 if x.is_complex() else 1)
        _lib.call("ht_axpby_dev", _lib.ptr(x), _lib.ptr(y), A, float(sa), B, float(sb), n,
                  _lib.ptr(dot) if dot is not None else None, _lib.stream_ptr())

    def bh_iteration(self, i, sync=True):
        """One BH iteration (rec_nfp_mpi.py:100-144), with the Hessian forms of
        one fused pass: H(g,e) and H(e,e) give beta, and the bottom of alpha
        follows from them and H(g,g) by bilinearity (beta^2 H(e,e) - 2 beta
        H_sym(g,e) + H(g,g)), which is H(eta, eta) of the updated direction.
        Returns (alpha, beta).  sync=False keeps alpha and beta on the device
        (ht_bh_scalars, ht_axpby_dev: the same formulas), so the iteration
        makes no host round trip and can be recorded into a CUDA graph; the
        step sizes then go to the device history (bh_history())."""
        vars, grads, etas, C = self.vars, self.grads, self.etas, self._c
        rho = self.rho_sq
        first = i == self.start_iter
        self._coeff(vars["proj"], C["vars"])
        # gradients, scaled (rec_nfp_mpi.py:106-109)
        self._gradient_pass(C["vars"], vars["pos"], vars["prb"], grads["pos"], grads["prb"], rho["pos"], rho["prb"])
        self._coeff(self._gc, grads["proj"])
        if rho["proj"] != 1:
            grads["proj"] *= rho["proj"]
        self._coeff(grads["proj"], C["grads"])
        y = (C["grads"], grads["pos"], grads["prb"])
        z = None if first else (C["etas"], etas["pos"], etas["prb"])
        H = self._hessian_pass(C["vars"], vars["pos"], vars["prb"], y, z)
        dots = self._dots
        if sync:
            H = H.cpu().numpy()
            beta = 0.0 if first else H[1] / H[2]
            dots.zero_()
            for k, v in enumerate(("proj", "pos", "prb")):
                self._axpby(etas[v], grads[v], beta, -1.0, dots[k:k + 1])
            self._axpby(C["etas"], C["grads"], beta, -1.0)
            d = dots.cpu().numpy()
            top = -(d[1] / rho["pos"] + d[2] / rho["prb"] + d[0] / rho["proj"])
            bottom = H[0] if first else beta * beta * H[2] - 2 * beta * H[3] + H[0]
            alpha = top / bottom
            for v in ("prb", "proj", "pos"):
                self._axpby(vars[v], etas[v], 1.0, alpha)
            return float(alpha), float(beta)
        st = _lib.stream_ptr()
        bh = self._bh
        rr = (float(rho["proj"]), float(rho["pos"]), float(rho["prb"]))
        # phase 0: beta, and the dots cleared for the direction updates below
        _lib.call("ht_bh_scalars", _lib.ptr(H), _lib.ptr(dots), int(first), 0, *rr, _lib.ptr(bh), None, 0, None, st)
        beta = _lib.ptr(bh)
        for k, v in enumerate(("proj", "pos", "prb")):
            self._axpby_dev(etas[v], grads[v], beta, 1.0, None, -1.0, dots[k:k + 1])
        self._axpby_dev(C["etas"], C["grads"], beta, 1.0, None, -1.0)
        _lib.call("ht_bh_scalars", _lib.ptr(H), _lib.ptr(dots), int(first), 1, *rr, _lib.ptr(bh),
                  _lib.ptr(self._hist), self._hist_cap, _lib.ptr(self._count), st)
        alpha = ctypes.c_void_p(bh.data_ptr() + 8)
        for v in ("prb", "proj", "pos"):
            self._axpby_dev(vars[v], etas[v], None, 1.0, alpha, 1.0)
        return None

    def capture_iteration(self):
        """Record one steady-state device-scalar iteration (not the first) on
        the current stream into a CUDA graph; replay_iteration() then runs it
        with one launch.  Call after one iteration has run on this device.
        Recording runs nothing."""
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

    def bh_history(self):
        """(alpha, beta) of the device-scalar iterations since BH started."""
        n = min(int(self._count.item()), self._hist_cap)
        return [tuple(r) for r in self._hist[:n].cpu().numpy()]

    def reserve_history(self, n):
        """Room for n device-side (alpha, beta) pairs, as Rec.reserve_history."""
        if n > self._hist_cap:
            self.release_graph()
            old, k = self._hist, self._hist_cap
            self._hist_cap = int(n)
            self._hist = torch.zeros(self._hist_cap, 2, dtype=torch.float64, device=self.device)
            self._hist[:k].copy_(old)

    def BH(self, writer=None, niter=None, record=None, mode="host"):
        """rec_nfp_mpi.py:100-144.  ``record`` (a list) receives (iteration,
        alpha, beta).  mode="host" iterates as the reference does (step sizes
        on the host); mode="graph" keeps them on the device and replays the
        steady-state iteration from a CUDA graph (same arithmetic; complex
        projections, no error table -- otherwise it iterates as "host")."""
        vars = self.vars
        niter = self.niter if niter is None else niter
        self.time_start = time.time()
        self.error_debug(vars, -1)
        self._count.zero_()
        if mode == "graph" and self.complex_obj and self.err_step == -1 and niter > self.start_iter:
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
            return vars
        for i in range(self.start_iter, niter):
            alpha, beta = self.bh_iteration(i)
            if record is not None:
                record.append((i, alpha, beta))
            self.error_debug(vars, i)
        return vars
