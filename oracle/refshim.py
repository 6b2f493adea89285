"""Run the reference's own Python operators on the CPU (TEST INFRASTRUCTURE ONLY).

The reference (holotomocupy) is CuPy + mpi4py code.  Neither package exists in
this image, so this module installs small stand-ins in ``sys.modules`` and then
imports the reference's ``tomo.py``, ``shift.py``, ``propagation.py``,
``rec_mpi.py`` and ``rec_nfp_mpi.py`` UNCHANGED from a source tree given by
the caller:

* ``cupy``            -> NumPy, with arrays of a small ndarray subclass that has
                         CuPy's ``.get()``; ``cp.RawKernel`` -> the NumPy kernel
                         restatements of ``oracle/kernels_np.py`` (picked by the
                         kernel name and by float2/float in its source);
                         ``cp.fuse`` -> identity.
* ``cupyx.scipy.fft`` -> ``scipy.fft`` (honouring ``overwrite_x=True`` by writing
                         the result back, which ``tomo.py:68`` relies on).
* ``mpi4py`` / ``holotomocupy.mpi_functions`` -> a single-rank communicator
                         (``redist`` becomes a copy, reductions the identity).
* ``holotomocupy.conv2d_cufftdx`` -> "not available", so ``propagation.py`` takes
                         its CuPy FFT branch (``propagation.py:36-44``).
* ``Chunking.gpu_batch`` -> calls the wrapped function directly, the reference's
                         own no-host-array branch (``chunking.py:39-42``).
* ``nvtx``, ``matplotlib``, ``matplotlib_scalebar``, ``tifffile``, ``h5py`` -> no-ops.

It is used only here, to generate golden vectors under ``tests/golden``; the
reference source tree does not exist where the GPU tests run.
"""
import contextlib
import importlib
import sys
import types

import numpy as np
import scipy.fft as sfft

from . import kernels_np as K


class GArr(np.ndarray):
    """ndarray with CuPy's host-transfer methods; keeps 0-d results as arrays so
    that ``x[0].get()`` and ``cp.sum(...).get()`` work as in CuPy."""

    def __array_wrap__(self, arr, context=None, return_scalar=False):
        return np.asarray(arr).view(GArr)

    def __getitem__(self, k):
        r = super().__getitem__(k)
        return r if isinstance(r, np.ndarray) else np.asarray(r).view(GArr)

    def get(self, out=None, blocking=True, stream=None):
        a = np.array(np.asarray(self))
        if out is not None:
            out[...] = a
            return out
        return a

    def set(self, arr, stream=None):
        self[...] = arr


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, GArr):
        return x.view(GArr)
    if isinstance(x, (np.generic,)):
        return np.asarray(x).view(GArr)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


def _wrapfn(fn):
    def inner(*a, **k):
        return _wrap(fn(*a, **k))
    inner.__name__ = getattr(fn, "__name__", "fn")
    return inner


class _FakeModule(types.ModuleType):
    """Module whose unknown attributes fall through to a NumPy namespace."""

    def __init__(self, name, base):
        super().__init__(name)
        self._base = base

    def __getattr__(self, name):
        attr = getattr(self._base, name)
        if isinstance(attr, np.ufunc) or isinstance(attr, type):
            return attr
        if callable(attr):
            return _wrapfn(attr)
        if isinstance(attr, types.ModuleType):
            return _FakeModule(self.__name__ + "." + name, attr)
        return attr


class _KernelStandIn:
    """cp.RawKernel replacement: kernel(grid, block, args)."""

    def __init__(self, code, name, *a, **k):
        self.name = name
        self.complex = "float2" in code.split("(")[1] if "(" in code else True
        self.code = code

    def __call__(self, grid, block, args, **kw):
        a = list(args)
        n = self.name
        if n == "gather":
            g, f, theta, m, mu, nn, ntheta, nz, d = a
            K.gather(g, f, theta, int(m), mu, int(nn), int(ntheta), int(nz), int(d))
        elif n == "pad_fwd":
            K.pad_fwd(*a[:2], *[int(v) for v in a[2:]])
        elif n == "pad_adj":
            K.pad_adj(*a[:2], *[int(v) for v in a[2:]])
        elif n == "s":
            g, f, r, mag = a[:4]
            K.s_kernel(g, f, r, mag, *[int(v) for v in a[4:]])
        elif n == "ds":
            res, c, c1, r, mag, dr = a[:6]
            K.ds_kernel(res, c, c1, r, mag, dr, *[int(v) for v in a[6:]])
        elif n == "d2s":
            res, c, c1, c2, r, mag, d1, d2 = a[:8]
            K.d2s_kernel(res, c, c1, c2, r, mag, d1, d2, *[int(v) for v in a[8:]])
        elif n == "dsadj":
            f, dt1, dt2, c, g, r, mag = a[:7]
            K.dsadj_kernel(f, dt1, dt2, c, g, r, mag, *[int(v) for v in a[7:]])
        elif n == "sback":
            g, f, r, mag = a[:4]
            K.sback_kernel(g, f, r, mag, *[int(v) for v in a[4:]])
        else:
            raise NotImplementedError(f"kernel {n} has no stand-in")


class _NullCtx(contextlib.AbstractContextManager):
    def __exit__(self, *exc):
        return False

    def synchronize(self):
        pass

    @property
    def ptr(self):
        return 0


def _cufft_fn(fn):
    def inner(x, *a, overwrite_x=False, plan=None, **k):
        r = fn(np.asarray(x), *a, **k)
        if overwrite_x:
            x[...] = r
            return x
        return _wrap(r)
    return inner


def _make_cupy():
    cp = _FakeModule("cupy", np)
    cp.ndarray = np.ndarray
    cp.RawKernel = _KernelStandIn
    cp.fuse = lambda *a, **k: (lambda f: f)
    cp.asnumpy = lambda x, *a, **k: np.array(np.asarray(x))
    cp.array = _wrapfn(np.array)
    cp.asarray = _wrapfn(np.asarray)
    cp.vdot = _wrapfn(np.vdot)
    cp.newaxis = None

    cuda = types.SimpleNamespace()
    cuda.Stream = lambda *a, **k: _NullCtx()
    cuda.alloc = lambda nbytes: None
    cuda.alloc_pinned_memory = lambda nbytes: bytearray(int(nbytes))
    cuda.get_current_stream = lambda: _NullCtx()
    cuda.Event = lambda *a, **k: _NullCtx()
    cuda.runtime = types.SimpleNamespace(memGetInfo=lambda: (0, 0),
                                         memcpyHostToDevice=1, memcpyDeviceToHost=2)
    cp.cuda = cuda

    fftmod = _FakeModule("cupy.fft", np.fft)
    fftmod.config = types.SimpleNamespace(
        get_plan_cache=lambda: types.SimpleNamespace(set_size=lambda n: None))
    cp.fft = fftmod
    cp.linalg = _FakeModule("cupy.linalg", np.linalg)
    return cp, fftmod


def _make_cupyx():
    cupyx = types.ModuleType("cupyx")
    cscipy = types.ModuleType("cupyx.scipy")
    cfft = types.ModuleType("cupyx.scipy.fft")
    for name in ("fft", "ifft", "fft2", "ifft2", "fftn", "ifftn"):
        setattr(cfft, name, _cufft_fn(getattr(sfft, name)))
    cfft.get_fft_plan = lambda *a, **k: _NullCtx()
    cupyx.scipy = cscipy
    cscipy.fft = cfft
    return cupyx, cscipy, cfft


class _Comm:
    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def Barrier(self):
        pass

    def allreduce(self, x):
        return x

    def Sendrecv(self, sendbuf=None, dest=None, recvbuf=None, source=None, **kw):
        # one rank: both neighbours are MPI.PROC_NULL, nothing is exchanged
        pass


def _make_mpi():
    mpi4py = types.ModuleType("mpi4py")
    MPI = types.SimpleNamespace(COMM_WORLD=_Comm(), PROC_NULL=-1, IN_PLACE=None, SUM=None,
                                Is_finalized=lambda: False)
    mpi4py.MPI = MPI
    return mpi4py


def _make_mpi_functions():
    """Single-rank stand-in for pkg/mpi_functions.py (MPIClass, get_local_chunk)."""
    m = types.ModuleType("holotomocupy.mpi_functions")

    def get_local_chunk(total_size, rank, size):
        return 0, total_size

    class MPIClass:
        def __init__(self, comm, nzobj, ntheta, nobj, dtype):
            self.comm = comm
            self.rank, self.size = 0, 1
            self.st_obj, self.end_obj = 0, int(nzobj)
            self.st_theta, self.end_theta = 0, int(ntheta)
            self.local_nzobj, self.local_ntheta = int(nzobj), int(ntheta)

        def redist(self, src, dst, direction="forward"):
            dst[...] = src

        def allreduce(self, arr):
            return arr

        def allreduce2(self, a, b):
            return float(a), float(b)

    m.get_local_chunk = get_local_chunk
    m.MPIClass = MPIClass
    m.MPI = _make_mpi().MPI
    m.__all__ = ["get_local_chunk", "MPIClass", "MPI"]
    return m


def _stub(name, **attrs):
    mod = types.ModuleType(name)
    for k, v in attrs.items():
        setattr(mod, k, v)
    return mod


_LOADED = {}


def load_reference(src_dir):
    """Import the reference package from ``src_dir`` (the directory holding
    ``holotomocupy/``) with the stand-ins installed.  Returns a namespace with
    the modules ``tomo``, ``shift``, ``propagation``, ``rec_mpi``, ``rec_nfp_mpi`` and ``utils``."""
    if src_dir in _LOADED:
        return _LOADED[src_dir]
    cp, cpfft = _make_cupy()
    cupyx, cscipy, cfft = _make_cupyx()
    noop = lambda *a, **k: None
    deco = lambda *a, **k: (lambda f: f)
    mods = {
        "cupy": cp, "cupy.fft": cpfft, "cupyx": cupyx, "cupyx.scipy": cscipy,
        "cupyx.scipy.fft": cfft, "mpi4py": _make_mpi(),
        "nvtx": _stub("nvtx", push_range=noop, pop_range=noop, annotate=deco),
        "matplotlib": _stub("matplotlib"),
        "matplotlib.pyplot": _stub("matplotlib.pyplot"),
        "matplotlib_scalebar": _stub("matplotlib_scalebar"),
        "matplotlib_scalebar.scalebar": _stub("matplotlib_scalebar.scalebar", ScaleBar=object),
        "tifffile": _stub("tifffile"),
        "h5py": _stub("h5py"),
        "holotomocupy.conv2d_cufftdx": _stub(
            "holotomocupy.conv2d_cufftdx", CUFFTDX_AVAILABLE=False,
            precompile=noop, Conv2DCUFFTDX=None),
        "holotomocupy.mpi_functions": _make_mpi_functions(),
    }
    saved = {k: sys.modules.get(k) for k in mods}
    sys.modules.update(mods)
    sys.path.insert(0, src_dir)
    try:
        pkg = importlib.import_module("holotomocupy")
        ns = types.SimpleNamespace()
        for name in ("utils", "tomo", "shift", "propagation", "chunking", "rec_mpi", "rec_nfp_mpi"):
            setattr(ns, name, importlib.import_module("holotomocupy." + name))
        # Chunking: call the wrapped function directly (chunking.py:39-42 branch)
        ns.chunking.Chunking.__init__ = lambda self, nbytes, chunk: setattr(self, "chunk", chunk)
        ns.chunking.Chunking.gpu_batch = (
            lambda self, axis_out=0, axis_inp=0, nout=1, inp_pad=0:
            (lambda func: (lambda *args: func(*args))))
        ns.pkg = pkg
        ns.cp = cp
    finally:
        sys.path.remove(src_dir)
    _LOADED[src_dir] = ns
    return ns
