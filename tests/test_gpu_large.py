"""Operators at the 2048 size of the large configuration (2048^2 detector,
1800 angles) against the FP64 oracle on a few slices / images.  Bound:
rel L2 <= 1e-4 against the FP64 oracle (the propagator's FP32 table alone
differs from the exact one by 2-5e-5)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import holo_oracle as O

pytestmark = pytest.mark.gpu


def test_propagator_at_2048():
    from holotomocupy_b200 import Propagation
    n, dist = 2048, np.array([3e-3, 6e-3])
    rng = np.random.default_rng(2048)
    p = Propagation(n, n, 2, 2, 7.3e-11, 20e-9, dist)
    o = O.Propagation(n, n, 2, 2, 7.3e-11, 20e-9, dist)
    x = (rng.standard_normal((1, n, n)) + 1j * rng.standard_normal((1, n, n))).astype("complex64")
    for j in range(2):
        d = p.D(torch.from_numpy(x).cuda(), j).cpu().numpy()
        assert rel_l2(d, o.D(x.astype(np.complex128), j)) < 1e-4


def test_radon_at_2048_1800_angles():
    from holotomocupy_b200 import Tomo
    n, ntheta, nz = 2048, 1800, 2
    theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype("float32")
    rng = np.random.default_rng(1800)
    t = Tomo(n, nz, theta, 0.9)
    o = O.Tomo(n, nz, theta, 0.9, "complex128")
    x = (rng.standard_normal((nz, n, n)) + 1j * rng.standard_normal((nz, n, n))).astype("complex64")
    y = (rng.standard_normal((ntheta, nz, n)) + 1j * rng.standard_normal((ntheta, nz, n))).astype("complex64")
    assert rel_l2(t.R(torch.from_numpy(x).cuda()).cpu().numpy(), o.R(x.astype(np.complex128))) < 1e-4
    assert rel_l2(t.RT(torch.from_numpy(y).cuda()).cpu().numpy(), o.RT(y.astype(np.complex128))) < 1e-4
