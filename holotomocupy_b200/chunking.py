"""Chunked processing of host-resident arrays on one GPU (drop-in for
holotomocupy's ``Chunking``, src/holotomocupy/chunking.py:5-290).

``Chunking(nbytes, chunk)`` owns one device pool of ``nbytes`` and three
streams.  ``gpu_batch(axis_out, axis_inp, nout, inp_pad)`` decorates a
function ``f(cl, out1, ..., inp1, ...)`` written for device arrays so that it
also takes host (NumPy) arrays larger than the device: the arrays whose
``shape[axis]`` equals the chunked size ("proper" arguments, outputs first)
are streamed through the pool ``chunk`` rows at a time -- the host-to-device
copies, the compute and the device-to-host copies of consecutive chunks
overlap on three streams, double-buffered and ordered by events only -- while
the other arguments are passed whole (NumPy ones copied to the device once).  With ``inp_pad`` the
first input holds ``size + inp_pad`` rows and every chunk receives
``chunk + inp_pad`` of them (a halo).  Without any host array the function
runs directly.  These are the reference's argument rules (chunking.py:12-98).

Differences from the reference, by design: the pool and the chunk buffers
are torch tensors on the given device; host arrays are page-locked
(cudaHostRegister) for the duration of a call so that their copies are truly
asynchronous; the BLAS-1 helpers accumulate inner products in double
precision on the device with the library's kernels (the reference sums in
float32).
"""
import ctypes

import numpy as np
import torch

from . import _lib

_TORCH = {np.dtype("complex64"): torch.complex64, np.dtype("complex128"): torch.complex128,
          np.dtype("float32"): torch.float32, np.dtype("float64"): torch.float64,
          np.dtype("int32"): torch.int32, np.dtype("int64"): torch.int64, np.dtype("uint8"): torch.uint8}
_ALIGN = 256


def _is_array(a):
    return isinstance(a, np.ndarray) or (isinstance(a, torch.Tensor) and a.is_cuda)


def _tdtype(a):
    return a.dtype if isinstance(a, torch.Tensor) else _TORCH[np.dtype(a.dtype)]


def _itemsize(a):
    return a.element_size() if isinstance(a, torch.Tensor) else a.dtype.itemsize


class _HostPin:
    """Page-locks the memory of host arrays while a chunked call runs (ranges
    that are already page-locked are left as they are)."""

    def __init__(self, arrays):
        self.ptrs = []
        for a in arrays:
            if not isinstance(a, np.ndarray) or a.nbytes == 0:
                continue
            base = a
            while isinstance(base.base, np.ndarray):
                base = base.base
            if not base.flags["C_CONTIGUOUS"]:
                continue
            ptr = base.__array_interface__["data"][0]
            if any(p == ptr for p in self.ptrs):
                continue
            reg = ctypes.c_int(0)
            _lib.call("ht_host_register", ptr, base.nbytes, ctypes.byref(reg))
            if reg.value:
                self.ptrs.append(ptr)

    def close(self):
        for p in self.ptrs:
            _lib.call("ht_host_unregister", p)
        self.ptrs = []


class Chunking:
    """Chunked H2D / compute / D2H on one GPU (chunking.py:5-10)."""

    def __init__(self, nbytes, chunk, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.gpu_mem = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
        self.stream = [torch.cuda.Stream(device=self.device) for _ in range(3)]
        self.chunk = int(chunk)

    # --------------------------------------------------------- decorator
    def gpu_batch(self, axis_out=0, axis_inp=0, nout=1, inp_pad=0):
        """chunking.py:12-98 (same argument classification)."""

        def decorator(func):
            def inner(*args):
                if not any(isinstance(a, np.ndarray) for a in args):
                    func(*args)
                    return
                cl = args[0]
                out = list(args[1:1 + nout])
                inp = list(args[1 + nout:])
                size = inp[0].shape[axis_inp] - inp_pad
                proper_out = nonproper_out = 0
                for a in out:
                    if _is_array(a) and a.ndim > axis_out + 1 and a.shape[axis_out] == size:
                        proper_out += 1
                    elif isinstance(a, torch.Tensor):
                        nonproper_out += 1
                padded_first = 1 if inp_pad > 0 else 0
                proper_inp, nonproper_inp = padded_first, 0
                for a in inp[padded_first:]:
                    if _is_array(a) and a.ndim > axis_inp + 1 and a.shape[axis_inp] == size:
                        proper_inp += 1
                    elif _is_array(a):
                        nonproper_inp += 1
                if int(np.prod(out[0].shape)) == 0:
                    return
                self.run(cl, out, inp, proper_inp, nonproper_inp, proper_out, nonproper_out, axis_out, axis_inp,
                         func, inp_pad)

            return inner

        return decorator

    # ------------------------------------------------------------ buffers
    def _buffers(self, arrs, axis, offset, rows):
        """Two device buffers per array (rows along axis), carved from the pool."""
        bufs = [[], []]
        for j in (0, 1):
            for a in arrs:
                shape = list(a.shape)
                shape[axis] = rows
                nbytes = int(np.prod(shape)) * _itemsize(a)
                offset = (offset + _ALIGN - 1) // _ALIGN * _ALIGN
                if offset + nbytes > self.gpu_mem.numel():
                    raise RuntimeError(f"Chunking pool of {self.gpu_mem.numel()} bytes is too small for chunks of "
                                       f"{self.chunk} rows")
                bufs[j].append(self.gpu_mem[offset:offset + nbytes].view(_tdtype(a)).view(shape))
                offset += nbytes
        return bufs, offset

    @staticmethod
    def _sl(axis, sl, ndim):
        res = [slice(None)] * ndim
        res[axis] = sl
        return tuple(res)

    @staticmethod
    def _copy(dst, src):
        """dst <- src on the current stream (host sides as torch views)."""
        if isinstance(src, np.ndarray):
            src = torch.from_numpy(src)
        if isinstance(dst, np.ndarray):
            dst = torch.from_numpy(dst)
        dst.copy_(src, non_blocking=True)

    # --------------------------------------------------------------- run
    def run(self, cl, out, inp, proper_inp, nonproper_inp, proper_out, nonproper_out, axis_out, axis_inp, func,
            inp_pad=0):
        """The pipeline over the chunks (the work of chunking.py:100-200)."""
        size = inp[0].shape[axis_inp] - inp_pad
        nchunk = (size + self.chunk - 1) // self.chunk
        out_gpu, off = self._buffers(out[:proper_out], axis_out, 0, self.chunk)
        if inp_pad > 0 and proper_inp > 0:
            pad_gpu, off = self._buffers(inp[:1], axis_inp, off, self.chunk + inp_pad)
            rest_gpu, off = self._buffers(inp[1:proper_inp], axis_inp, off, self.chunk)
            inp_gpu = [pad_gpu[j] + rest_gpu[j] for j in (0, 1)]
        else:
            inp_gpu, off = self._buffers(inp[:proper_inp], axis_inp, off, self.chunk)
        for k in range(proper_inp, proper_inp + nonproper_inp):
            if isinstance(inp[k], np.ndarray):
                inp[k] = torch.from_numpy(np.ascontiguousarray(inp[k])).to(self.device)
        pin = _HostPin(out[:proper_out] + inp[:proper_inp])

        def bounds(k):
            return k * self.chunk, min(size, (k + 1) * self.chunk)

        def p2g(b, k):
            st, end = bounds(k)
            for j in range(proper_inp):
                extra = inp_pad if (j == 0 and inp_pad > 0) else 0
                nd = inp[j].ndim
                self._copy(inp_gpu[b][j][self._sl(axis_inp, slice(0, end - st + extra), nd)],
                           inp[j][self._sl(axis_inp, slice(st, end + extra), nd)])

        def g2p(b, k):
            st, end = bounds(k)
            for j in range(proper_out):
                nd = out[j].ndim
                self._copy(out[j][self._sl(axis_out, slice(st, end), nd)],
                           out_gpu[b][j][self._sl(axis_out, slice(0, end - st), nd)])

        def compute(b, k):
            st, end = bounds(k)
            n = end - st
            ic = []
            for j in range(proper_inp):
                extra = inp_pad if (j == 0 and inp_pad > 0) else 0
                ic.append(inp_gpu[b][j][self._sl(axis_inp, slice(0, n + extra), inp_gpu[b][j].ndim)])
            oc = [o[self._sl(axis_out, slice(0, n), o.ndim)] for o in out_gpu[b]]
            func(cl, *oc, *out[proper_out:], *ic, *inp[proper_inp:proper_inp + nonproper_inp],
                 *inp[proper_inp + nonproper_inp:])

        # The chunks flow through three streams -- copy in, compute, copy out --
        # ordered only by events, so the host issues every chunk's work in one
        # pass and waits once, at the end.  Buffer set b = k % 2 is reused by
        # chunk k + 2: its copy-in waits until chunk k's compute has read the
        # inputs, its compute until chunk k's copy-out has drained the outputs.
        s_in, s_comp, s_out = self.stream
        cur = torch.cuda.current_stream(self.device)
        for st in self.stream:
            st.wait_stream(cur)   # device inputs written before the call are visible
        ev = lambda: torch.cuda.Event()
        loaded, computed, drained = [None] * nchunk, [None] * nchunk, [None] * nchunk
        try:
            for k in range(nchunk):
                b = k % 2
                with torch.cuda.stream(s_in):
                    if k >= 2:
                        s_in.wait_event(computed[k - 2])
                    p2g(b, k)
                    loaded[k] = ev()
                    loaded[k].record(s_in)
                with torch.cuda.stream(s_comp):
                    s_comp.wait_event(loaded[k])
                    if k >= 2:
                        s_comp.wait_event(drained[k - 2])
                    compute(b, k)
                    computed[k] = ev()
                    computed[k].record(s_comp)
                with torch.cuda.stream(s_out):
                    s_out.wait_event(computed[k])
                    g2p(b, k)
                    drained[k] = ev()
                    drained[k].record(s_out)
        finally:
            # host outputs must be complete before the call returns (and before
            # the host pages are unlocked); device outputs follow on `cur`
            for st in self.stream:
                st.synchronize()
            cur.wait_stream(s_comp)
            pin.close()

    # ------------------------------------------- batched BLAS-1 (chunking.py:233-290)
    @staticmethod
    def _nfloat(t):
        return t.numel() * (2 if t.is_complex() else 1)

    def redot_batch(self, x, y):
        """Re<x, y>, accumulated in double (chunking.py:233-244)."""
        acc = torch.zeros(1, dtype=torch.float64, device=self.device)
        if isinstance(x, torch.Tensor) and isinstance(y, torch.Tensor):
            _lib.call("ht_dot", _lib.ptr(x.contiguous()), _lib.ptr(y.contiguous()), self._nfloat(x), _lib.ptr(acc),
                      _lib.stream_ptr())
            return float(acc)

        @self.gpu_batch(axis_out=0, axis_inp=0, nout=1)
        def _redot(cl, res, xc, yc):
            _lib.call("ht_dot", _lib.ptr(xc), _lib.ptr(yc), cl._nfloat(xc), _lib.ptr(res), _lib.stream_ptr())

        _redot(self, acc, x, y)
        return float(acc)

    def linear_batch(self, x, y, a, b, out=None):
        """out = a x + b y (chunking.py:246-257); out defaults to x."""
        if out is None:
            out = x
        if isinstance(x, torch.Tensor) and isinstance(y, torch.Tensor) and isinstance(out, torch.Tensor):
            if out is not x:
                out.copy_(x)
            _lib.call("ht_axpby", _lib.ptr(out), _lib.ptr(y.contiguous()), float(a), float(b), self._nfloat(out),
                      None, _lib.stream_ptr())
            return

        @self.gpu_batch(axis_out=0, axis_inp=0, nout=1)
        def _linear(cl, oc, xc, yc):
            oc.copy_(xc)
            _lib.call("ht_axpby", _lib.ptr(oc), _lib.ptr(yc), float(a), float(b), cl._nfloat(oc), None,
                      _lib.stream_ptr())

        _linear(self, out, x, y)

    def linear_redot_batch(self, x, y, a, b):
        """x = a x + b y in place; returns Re<y, x_new> in one pass (chunking.py:259-272)."""
        acc = torch.zeros(1, dtype=torch.float64, device=self.device)
        if isinstance(x, torch.Tensor) and isinstance(y, torch.Tensor):
            _lib.call("ht_axpby", _lib.ptr(x), _lib.ptr(y.contiguous()), float(a), float(b), self._nfloat(x),
                      _lib.ptr(acc), _lib.stream_ptr())
            return float(acc)

        @self.gpu_batch(axis_out=0, axis_inp=0, nout=2)
        def _linear_redot(cl, oc, res, xc, yc):
            oc.copy_(xc)
            _lib.call("ht_axpby", _lib.ptr(oc), _lib.ptr(yc), float(a), float(b), cl._nfloat(oc), _lib.ptr(res),
                      _lib.stream_ptr())

        _linear_redot(self, x, acc, x, y)
        return float(acc)

    def mulc_batch(self, out, x, a):
        """out = a x (chunking.py:274-285)."""
        if isinstance(x, torch.Tensor) and isinstance(out, torch.Tensor):
            torch.mul(x, a, out=out)
            return out

        @self.gpu_batch(axis_out=0, axis_inp=0, nout=1)
        def _mulc(cl, oc, xc):
            torch.mul(xc, a, out=oc)

        _mulc(self, out, x)
        return out
