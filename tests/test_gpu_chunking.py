"""Chunking.gpu_batch (src/holotomocupy/chunking.py:12-290): host arrays
streamed through the device pool in chunks give the same results as the
device path, with the reference's argument rules (proper / non-proper
arguments, halo rows with inp_pad, chunking along axis 0 or 1)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype("complex64")


def test_propagator_over_host_arrays_equals_device_path():
    from holotomocupy_b200 import Propagation
    from holotomocupy_b200.chunking import Chunking
    rng = np.random.default_rng(0)
    n = nz = 64
    nb = 37
    prop = Propagation(n, nz, 8, 2, 7.3e-11, 20e-9, np.array([3e-3, 5e-3]))
    psi = _crand(rng, (nb, nz, n))
    prb = _crand(rng, (nz, n))                 # non-proper host input: copied to the device once
    out = np.zeros_like(psi)
    ch = Chunking(64 << 20, 8)

    @ch.gpu_batch(axis_out=0, axis_inp=0, nout=1)
    def _d(cl, o, x, p):
        o.copy_(prop.D(x * p, 1))

    _d(ch, out, psi, prb)
    ref = prop.D(torch.from_numpy(psi).cuda() * torch.from_numpy(prb).cuda(), 1).cpu().numpy()
    np.testing.assert_array_equal(out, ref)      # the same kernels on the same images


def test_halo_rows_with_inp_pad():
    """inp_pad = 4: each chunk receives its rows plus 4 (the Laplacian's use,
    rec_mpi.py:418-440); here out[i] = sum of padded rows i .. i+4."""
    from holotomocupy_b200.chunking import Chunking
    rng = np.random.default_rng(1)
    size, pad = 29, 4
    u = rng.standard_normal((size + pad, 16, 16)).astype("float32")
    out = np.zeros((size, 16, 16), "float32")
    ch = Chunking(16 << 20, 6)

    @ch.gpu_batch(axis_out=0, axis_inp=0, nout=1, inp_pad=pad)
    def _box(cl, o, up):
        o.copy_(sum(up[j:j + o.shape[0]] for j in range(pad + 1)))

    _box(ch, out, u)
    ref = sum(u[j:j + size] for j in range(pad + 1))
    np.testing.assert_allclose(out, ref, rtol=1e-6, atol=1e-5)


def test_chunking_along_axis_1():
    from holotomocupy_b200.chunking import Chunking
    rng = np.random.default_rng(2)
    x = rng.standard_normal((3, 41, 8, 8)).astype("float32")
    out = np.zeros_like(x)
    ch = Chunking(16 << 20, 10)

    @ch.gpu_batch(axis_out=1, axis_inp=1, nout=1)
    def _sq(cl, o, xc):
        torch.mul(xc, xc, out=o)

    _sq(ch, out, x)
    np.testing.assert_array_equal(out, x * x)


def test_blas1_batches_match_fp64():
    from holotomocupy_b200.chunking import Chunking
    rng = np.random.default_rng(3)
    x = _crand(rng, (53, 32, 32))
    y = _crand(rng, (53, 32, 32))
    ch = Chunking(32 << 20, 7)
    ref = float(np.sum(x.real.astype(np.float64) * y.real + x.imag.astype(np.float64) * y.imag))
    assert abs(ch.redot_batch(x, y) / ref - 1) < 1e-6
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    assert abs(ch.redot_batch(xd, yd) / ref - 1) < 1e-6
    # out = a x + b y
    out = np.zeros_like(x)
    ch.linear_batch(x, y, 0.5, -2.0, out=out)
    assert rel_l2(out, 0.5 * x.astype(np.complex128) - 2.0 * y) < 1e-6
    # x = a x + b y in place, returning Re<y, x_new>
    xx = x.copy()
    d = ch.linear_redot_batch(xx, y, 1.5, 0.25)
    xn = 1.5 * x.astype(np.complex128) + 0.25 * y
    assert rel_l2(xx, xn) < 1e-6
    dn = float(np.sum(y.real * xn.real + y.imag * xn.imag))
    assert abs(d / dn - 1) < 1e-6
    # out = a x
    o2 = np.zeros_like(x)
    ch.mulc_batch(o2, x, 3.0)
    assert rel_l2(o2, 3.0 * x.astype(np.complex128)) < 1e-6
    # the device path of the same helpers
    od = torch.empty_like(xd)
    ch.linear_batch(xd, yd, 0.5, -2.0, out=od)
    assert rel_l2(od.cpu().numpy(), 0.5 * x.astype(np.complex128) - 2.0 * y) < 1e-6


def test_pool_too_small_is_an_error():
    from holotomocupy_b200.chunking import Chunking
    x = np.zeros((10, 64, 64), "complex64")
    ch = Chunking(1 << 16, 8)

    @ch.gpu_batch(axis_out=0, axis_inp=0, nout=1)
    def _cp(cl, o, xc):
        o.copy_(xc)

    with pytest.raises(RuntimeError, match="too small"):
        _cp(ch, np.zeros_like(x), x)
