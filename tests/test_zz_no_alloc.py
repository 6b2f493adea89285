"""The objective entry point that allocates nothing, against the one that does.

Some callers cannot allocate device memory: their memory belongs to another
allocator (a framework's caching pool, a serving loop with a fixed budget), or
they must not call cudaMalloc/cudaFree because those calls can synchronise the
whole device.  ht_rec_objective_noalloc serves them from one fixed 32 MiB
device array.  This file is collected last so that a run stopping at its first
failure has already run every other test; it also passes on its own.
"""
import ctypes
import types

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _args(n, ntheta, ndist):
    return types.SimpleNamespace(
        theta=np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32"), ndist=ndist, ntheta=ntheta,
        nz=n, n=n, nzobj=n, nobj=n, obj_dtype="complex64", mask=0, lam_prbfit=0.0, rho=[1, 0.05, 0.02],
        niter=1, nchunk=n, vis_step=-1, err_step=-1, start_iter=0, distance=np.array([3e-3, 4e-3, 5e-3, 6e-3])[:ndist],
        wavelength=7.3e-11, voxelsize=20e-9, norm_magnifications=np.ones(ndist))


def _noalloc(prop_h, nobj, ntheta, c, pos, mag, prb, data):
    from holotomocupy_b200 import _lib
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    st = _lib.lib().ht_rec_objective_noalloc(prop_h, nobj, nobj, ntheta, 1, _lib.ptr(c), _lib.ptr(pos),
                                             _lib.ptr(mag), _lib.ptr(prb), _lib.ptr(data), _lib.ptr(out),
                                             _lib.stream_ptr())
    return st, out


def test_noalloc_objective_matches_the_allocating_entry_point():
    """Two calls in a row with different data: each must equal ht_rec_forward's
    objective (the array keeps the previous call's contents, so the second call
    also shows that the accumulators start from zero)."""
    from holotomocupy_b200 import _lib
    from holotomocupy_b200.rec import Rec
    n, ntheta, ndist = 512, 10, 4      # 3 angles fit the scratch at this size: chunks 3, 3, 3, 1
    rec = Rec(_args(n, ntheta, ndist))
    g = torch.Generator(device="cuda").manual_seed(5)
    proj = (0.05 * torch.randn(ntheta, n, n, dtype=torch.complex64, device="cuda", generator=g)).contiguous()
    c = rec._coeff_into(proj, torch.empty_like(proj))
    pos = (2 * torch.rand(ntheta, ndist, 2, device="cuda", generator=g) - 1).contiguous()
    mag = torch.ones(ntheta, ndist, device="cuda")
    prb = (1 + 0.1 * torch.randn(ndist, n, n, dtype=torch.complex64, device="cuda", generator=g)).contiguous()
    for call in range(2):
        data = (0.5 + torch.rand(ntheta, ndist, n, n, device="cuda", generator=g)).contiguous()
        ref = torch.zeros(1, dtype=torch.float64, device="cuda")
        _lib.call("ht_rec_forward", rec._h, _lib.ptr(c), _lib.ptr(pos), _lib.ptr(mag), _lib.ptr(prb),
                  _lib.ptr(data), None, _lib.ptr(ref), _lib.stream_ptr())
        st, out = _noalloc(rec.cl_prop._h, n, ntheta, c, pos, mag, prb, data)
        torch.cuda.synchronize()
        assert st == 0, _lib.lib().ht_last_error()
        r, v = float(ref), float(out)
        assert np.isfinite(v) and abs(v / r - 1) < 1e-6, (call, v, r)
    # the sums are reduced in a fixed order: the same inputs give the same bits
    st, again = _noalloc(rec.cl_prop._h, n, ntheta, c, pos, mag, prb, data)
    torch.cuda.synchronize()
    assert st == 0 and float(again) == v


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from holotomocupy_b200 import Propagation, _lib
    n, ndist = 1024, 4                 # one angle needs 4*1024*1024*8 bytes: above 32 MiB - 256
    p = Propagation(n, n, 1, ndist, 7.3e-11, 20e-9, [3e-3, 4e-3, 5e-3, 6e-3])
    z = torch.zeros(1, n, n, dtype=torch.complex64, device="cuda")
    pos = torch.zeros(1, ndist, 2, device="cuda")
    mag = torch.ones(1, ndist, device="cuda")
    prb = torch.ones(ndist, n, n, dtype=torch.complex64, device="cuda")
    data = torch.ones(1, ndist, n, n, device="cuda")
    st, out = _noalloc(p._h, n, 1, z, pos, mag, prb, data)
    assert st == 1
    assert b"32 MiB" in _lib.lib().ht_last_error()
