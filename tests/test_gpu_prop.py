"""Fresnel propagator on the GPU against the reference (golden vectors made by
running the reference's propagation.py) and against the FP64 oracle.

Tolerances: rel L2 <= 1e-5 against the reference (its own FP32 table and
arithmetic); against the FP64 oracle, whose Fresnel table is exact, the bound
is 1e-4 (the reference's FP32 table alone differs from it by 2-5e-5)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import holo_oracle as O

pytestmark = pytest.mark.gpu
TOL_REF = 1e-5
TOL_FP64 = 1e-4


def _prop(g, tag):
    from holotomocupy_b200 import Propagation
    n, nz = int(g[f"{tag}_n"]), int(g[f"{tag}_nz"])
    return Propagation(n, nz, 3, 3, float(g[f"{tag}_wavelength"]), float(g[f"{tag}_voxelsize"]),
                       g[f"{tag}_distance"])


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_D_DT_match_reference(golden, tag):
    g = golden("prop")
    p = _prop(g, tag)
    np.testing.assert_array_equal(p.fker.cpu().numpy(), g[f"{tag}_fker"])
    a = torch.from_numpy(g[f"{tag}_a"]).cuda()
    b = torch.from_numpy(g[f"{tag}_b"]).cuda()
    for j in range(3):
        assert rel_l2(p.D(a, j).cpu().numpy(), g[f"{tag}_D{j}"]) < TOL_REF
        assert rel_l2(p.DT(b, j).cpu().numpy(), g[f"{tag}_DT{j}"]) < TOL_REF
    d2 = p.D(a[0], 1)
    assert tuple(d2.shape) == g[f"{tag}_D2d"].shape
    assert rel_l2(d2.cpu().numpy(), g[f"{tag}_D2d"]) < TOL_REF


@pytest.mark.parametrize("n,nz", [(128, 128), (512, 512), (36, 512), (384, 256), (36, 18), (18, 36), (48, 1024), (64, 2048),
                                  (32, 4096)])
def test_D_against_fp64_oracle(n, nz):
    from holotomocupy_b200 import Propagation
    rng = np.random.default_rng(n + nz)
    dist = np.array([3e-3, 6e-3])
    p = Propagation(n, nz, 2, 2, 7.3e-11, 20e-9, dist)
    o = O.Propagation(n, nz, 2, 2, 7.3e-11, 20e-9, dist)
    o32 = O.Propagation(n, nz, 2, 2, 7.3e-11, 20e-9, dist, dtype="complex64")
    x = (rng.standard_normal((2, nz, n)) + 1j * rng.standard_normal((2, nz, n))).astype("complex64")
    xt = torch.from_numpy(x).cuda()
    for j in range(2):
        d = p.D(xt, j).cpu().numpy()
        assert rel_l2(d, o32.D(x, j)) < TOL_REF
        assert rel_l2(d, o.D(x.astype(np.complex128), j)) < TOL_FP64
        dt = p.DT(xt, j).cpu().numpy()
        assert rel_l2(dt, o32.DT(x, j)) < TOL_REF


def test_adjoint_energy_shape():
    """tests/propagation/test_propagation.py:42-88 of the reference, asserted."""
    from holotomocupy_b200 import Propagation
    n = nz = 256
    ntheta = 4
    wavelength = 1.24e-9 / 17.1
    sx0 = -3.135e-3
    z1 = np.array([5.110, 5.464, 6.879, 9.817]) * 1e-3 - sx0
    z2 = 1.217 - z1
    distances = (z1 * z2) / 1.217
    p = Propagation(n, nz, ntheta, 4, wavelength, 20e-9, distances)
    g = torch.Generator(device="cuda").manual_seed(0)
    for j in range(4):
        psi = torch.randn(ntheta, nz, n, dtype=torch.complex64, device="cuda", generator=g)
        phi = torch.randn(ntheta, nz, n, dtype=torch.complex64, device="cuda", generator=g)
        lhs = torch.sum(p.D(psi, j).to(torch.complex128) * phi.conj().to(torch.complex128)).item()
        rhs = torch.sum(psi.to(torch.complex128) * p.DT(phi, j).conj().to(torch.complex128)).item()
        assert abs(lhs - rhs) / abs(lhs) < 1e-5
        e_in = torch.sum(psi.abs() ** 2).item()
        e_out = torch.sum(p.D(psi, j).abs() ** 2).item()
        assert 0.9 < e_out / e_in < 1.1
    assert tuple(p.D(torch.ones(nz, n, dtype=torch.complex64, device="cuda"), 0).shape) == (nz, n)
    assert tuple(p.DT(torch.ones(ntheta, nz, n, dtype=torch.complex64, device="cuda"), 0).shape) == (ntheta, nz, n)


def test_in_place_and_aliasing():
    from holotomocupy_b200 import Propagation, _lib
    n = nz = 64
    p = Propagation(n, nz, 3, 1, 7.3e-11, 20e-9, [4e-3])
    x = torch.randn(3, nz, n, dtype=torch.complex64, device="cuda")
    ref = p.D(x, 0)
    y = x.clone()
    _lib.call("ht_prop_D", p._h, _lib.ptr(y), _lib.ptr(y), 3, 0, _lib.stream_ptr())
    torch.testing.assert_close(y, ref, rtol=0, atol=0)
