"""The reference's propagation test script against the drop-in Propagation.

tests/propagation/test_propagation.py of the reference drives Propagation at
n = nz = 1024, 4 images, 4 distances, and reaches into its internals:
``_use_cufftdx`` (a second instance with it off is the comparison point),
``_fwd_pad``, ``_conv2d.run``, ``_adj_pad`` and ``_buf_big``.  Its sections run
here unchanged apart from cupy -> torch, with its printed checks turned into
assertions: adjointness, energy, shapes, the backend comparison, and the
sub-steps of its profiling section, which must compose back to D and D^T.
The pad and convolution kernels are also checked against the oracle's
restatements of the reference kernels (pad_fwd / pad_adj) and a float64 FFT
convolution."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import kernels_np as K

pytestmark = pytest.mark.gpu

n = nz = 1024
ntheta = 4
energy = 17.1
wavelength = 1.24e-9 / energy
voxelsize = 20e-9
sx0 = -3.135e-3
z1 = np.array([5.110, 5.464, 6.879, 9.817]) * 1e-3 - sx0
focustodetectordistance = 1.217
z2 = focustodetectordistance - z1
distances = (z1 * z2) / focustodetectordistance
ndist = len(distances)


def crandn(*shape, g):
    return (torch.randn(*shape, device="cuda", generator=g) + 1j * torch.randn(*shape, device="cuda", generator=g)
            ).to(torch.complex64)


@pytest.fixture(scope="module")
def props():
    from holotomocupy_b200 import Propagation
    cl = Propagation(n, nz, ntheta, ndist, wavelength, voxelsize, distances)
    cl_cupy = Propagation(n, nz, ntheta, ndist, wavelength, voxelsize, distances)
    cl_cupy._use_cufftdx = False
    assert cl._use_cufftdx
    return cl, cl_cupy


def test_adjoint(props):
    cl, _ = props
    g = torch.Generator(device="cuda").manual_seed(1)
    for j in range(ndist):
        psi, phi = crandn(ntheta, nz, n, g=g), crandn(ntheta, nz, n, g=g)
        lhs = complex(torch.sum(cl.D(psi, j).to(torch.complex128) * phi.conj()))
        rhs = complex(torch.sum(psi.to(torch.complex128) * cl.DT(phi, j).conj()))
        assert abs(lhs - rhs) / abs(lhs) < 1e-5, (j, lhs, rhs)


def test_energy(props):
    cl, _ = props
    g = torch.Generator(device="cuda").manual_seed(2)
    for j in range(ndist):
        psi = crandn(ntheta, nz, n, g=g)
        e_in = float(torch.sum(torch.abs(psi) ** 2))
        e_out = float(torch.sum(torch.abs(cl.D(psi, j)) ** 2))
        assert abs(e_out / e_in - 1) < 0.02, (j, e_out / e_in)


def test_shapes(props):
    cl, _ = props
    psi_2d = torch.ones(nz, n, dtype=torch.complex64, device="cuda")
    psi_3d = torch.ones(ntheta, nz, n, dtype=torch.complex64, device="cuda")
    assert tuple(cl.D(psi_2d, 0).shape) == (nz, n)
    assert tuple(cl.D(psi_3d, 0).shape) == (ntheta, nz, n)
    assert tuple(cl.DT(psi_2d, 0).shape) == (nz, n)
    assert tuple(cl.DT(psi_3d, 0).shape) == (ntheta, nz, n)


def test_backends_agree(props):
    """max|D - D_cupy| / max|D_cupy| (the script prints it; here < 1e-5)."""
    cl, cl_cupy = props
    g = torch.Generator(device="cuda").manual_seed(3)
    for j in range(ndist):
        psi = crandn(ntheta, nz, n, g=g)
        for f, fc in ((cl.D, cl_cupy.D), (cl.DT, cl_cupy.DT)):
            ref, out = fc(psi, j), f(psi, j)
            err = float(torch.abs(out - ref).max()) / float(torch.abs(ref).max())
            assert err < 1e-5, (j, err)


def test_substeps_compose_to_D_and_DT(props):
    """The script's profiling section: _fwd_pad, _conv2d.run and the crop give
    D; the zero-embedding into _buf_big, _conv2d.run and _adj_pad give D^T."""
    cl, _ = props
    g = torch.Generator(device="cuda").manual_seed(4)
    j = 0
    psi, phi = crandn(ntheta, nz, n, g=g), crandn(ntheta, nz, n, g=g)
    ff_pad = torch.empty(ntheta, 2 * nz, 2 * n, dtype=torch.complex64, device="cuda")
    cl._fwd_pad(psi, ff_pad)
    y_buf = torch.empty_like(ff_pad)
    cl._conv2d.run(ff_pad, cl.fker[j], y_buf)
    crop = y_buf[:, cl.nz // 2: -cl.nz // 2, cl.n // 2: -cl.n // 2]
    assert rel_l2(crop.cpu().numpy(), cl.D(psi, j).cpu().numpy()) < 1e-5
    ff_zpad = torch.zeros(ntheta, 2 * nz, 2 * n, dtype=torch.complex64, device="cuda")
    ff_zpad[:, cl.nz // 2: -cl.nz // 2, cl.n // 2: -cl.n // 2] = phi
    y_buf2 = torch.empty_like(ff_zpad)
    cl._conv2d.run(ff_zpad, cl.fker[j].conj().contiguous(), y_buf2)
    out = torch.empty(ntheta, nz, n, dtype=torch.complex64, device="cuda")
    cl._adj_pad(y_buf2, out)
    assert rel_l2(out.cpu().numpy(), cl.DT(phi, j).cpu().numpy()) < 1e-5
    cl._buf_big[:ntheta].fill_(0)
    cl._buf_big[:ntheta][:, cl.nz // 2: -cl.nz // 2, cl.n // 2: -cl.n // 2] = phi
    assert tuple(cl._buf_big.shape) == (ntheta, 2 * nz, 2 * n)


@pytest.mark.parametrize("shape", [(2, 24, 32), (3, 64, 48), (1, 96, 96)])
def test_pad_kernels_match_the_reference_kernels(shape):
    from holotomocupy_b200 import Propagation
    nt, h, w = shape
    rng = np.random.default_rng(h + w)
    f = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype("complex64")
    G = (rng.standard_normal((nt, 2 * h, 2 * w)) + 1j * rng.standard_normal((nt, 2 * h, 2 * w))).astype("complex64")
    p = Propagation(w, h, nt, 1, wavelength, voxelsize, distances[:1])
    fp = torch.empty(nt, 2 * h, 2 * w, dtype=torch.complex64, device="cuda")
    p._fwd_pad(torch.from_numpy(f).cuda(), fp)
    ref = np.zeros((nt, 2 * h, 2 * w), "complex64")
    K.pad_fwd(ref, f, w, h, nt)
    np.testing.assert_array_equal(fp.cpu().numpy(), ref)
    fa = torch.empty(nt, h, w, dtype=torch.complex64, device="cuda")
    p._adj_pad(torch.from_numpy(G).cuda(), fa)
    ref = np.zeros((nt, h, w), "complex64")
    K.pad_adj(G, ref, w, h, nt)
    assert rel_l2(fa.cpu().numpy(), ref) < 1e-7


@pytest.mark.parametrize("rows,cols", [(36, 48), (256, 512), (2048, 2048)])
def test_conv2d_against_fp64(rows, cols):
    from holotomocupy_b200.propagation import Conv2D
    rng = np.random.default_rng(rows)
    b = 2
    x = (rng.standard_normal((b, rows, cols)) + 1j * rng.standard_normal((b, rows, cols))).astype("complex64")
    H = np.exp(1j * rng.uniform(0, 2 * np.pi, (rows, cols))).astype("complex64")
    c = Conv2D(rows, cols, torch.device("cuda", 0))
    y = torch.empty(b, rows, cols, dtype=torch.complex64, device="cuda")
    c.run(torch.from_numpy(x).cuda(), torch.from_numpy(H).cuda(), y)
    ref = np.fft.ifft2(np.fft.fft2(x.astype("complex128")) * H, norm="forward")
    assert rel_l2(y.cpu().numpy(), ref) < 1e-5
    xt = torch.from_numpy(x).cuda()
    c.run(xt, torch.from_numpy(H).cuda(), xt)          # in place
    assert rel_l2(xt.cpu().numpy(), ref) < 1e-5
