"""Host-side logic of the reconstruction server that needs no GPU: the
argument key that decides which retired Rec a request may take over, and the
device-memory estimate admission uses."""
import types

import numpy as np

from holotomocupy_b200.serving import args_key, estimate_bytes
from holotomocupy_b200.synthetic import workload_args


def test_equal_arguments_share_a_key():
    assert args_key(workload_args(128, 224, 4)) == args_key(workload_args(128, 224, 4))
    hash(args_key(workload_args(128, 224, 4)))


def test_any_differing_argument_changes_the_key():
    base = workload_args(128, 224, 4)
    key = args_key(base)
    assert args_key(workload_args(256, 448, 4)) != key
    assert args_key(workload_args(128, 224, 3)) != key
    for name, value in (("distance", np.array([3e-3, 4e-3, 5e-3, 7e-3])), ("rho", [1, 0.05, 0.03]),
                        ("mask", 0.8), ("lam_prbfit", 1e-3)):
        other = types.SimpleNamespace(**vars(base))
        setattr(other, name, value)
        assert args_key(other) != key, name
    # a theta array with one angle moved
    other = types.SimpleNamespace(**vars(base))
    other.theta = base.theta.copy()
    other.theta[5] += 1e-6
    assert args_key(other) != key


def test_estimate_grows_with_the_problem():
    small, large = estimate_bytes(workload_args(128, 224, 4)), estimate_bytes(workload_args(256, 448, 4))
    assert 0 < small < large
    # n^4 work, n^3-and-more memory: a 512^3 x 900 x 4 reconstruction needs tens of GB
    assert 40e9 < estimate_bytes(workload_args(512, 900, 4)) < 120e9
