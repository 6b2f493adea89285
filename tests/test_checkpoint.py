"""Checkpoint layout and resume (writer.py:57-110, reader.py:260-340): the
state written by Writer reads back exactly, and a checkpoint of a coarser
reconstruction comes back upsampled the way the reference's reader does it.
Runs on the CPU (the .npz layout; .h5 where h5py exists)."""
import numpy as np
import pytest
import torch

from holotomocupy_b200.checkpoint import Writer, h5py, read_checkpoint


def _state(rng, nz, n, ntheta, ndist, dt):
    obj = rng.standard_normal((nz, n, n)) + (1j * rng.standard_normal((nz, n, n)) if dt == "complex64" else 0)
    return {"obj": torch.from_numpy(obj.astype(dt)),
            "prb": torch.from_numpy((rng.standard_normal((ndist, n, n)) + 1j * rng.standard_normal((ndist, n, n)))
                                    .astype("complex64")),
            "pos": torch.from_numpy(rng.uniform(-2, 2, (ntheta, ndist, 2)).astype("float32"))}


@pytest.mark.parametrize("dt", ["complex64", "float32"])
@pytest.mark.parametrize("fmt", ["npz", "h5"])
def test_round_trip(tmp_path, dt, fmt):
    if fmt == "h5" and h5py is None:
        pytest.skip("h5py is not installed")
    rng = np.random.default_rng(1)
    v = _state(rng, 6, 16, 5, 2, dt)
    w = Writer(str(tmp_path), dt, fmt=fmt)
    path = w.write_checkpoint(v, 7, norm_const=2.0)
    assert path.endswith(f"checkpoint_0007.{fmt}")
    r = read_checkpoint(path, 16, 6, dt)
    assert r["iter"] == 7
    np.testing.assert_allclose(r["obj"].numpy(), 2.0 * v["obj"].numpy(), rtol=1e-6)
    np.testing.assert_allclose(r["prb"].numpy(), v["prb"].numpy(), rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(r["pos"].numpy(), v["pos"].numpy())


def test_resume_from_a_coarser_reconstruction(tmp_path):
    rng = np.random.default_rng(2)
    v = _state(rng, 4, 8, 3, 2, "complex64")
    path = Writer(str(tmp_path), "complex64", fmt="npz").write_checkpoint(v, 3)
    r = read_checkpoint(path, 16, 8, "complex64")
    obj, prb, pos = v["obj"].numpy(), v["prb"].numpy(), v["pos"].numpy()
    up = np.repeat(np.repeat(obj, 2, axis=2), 2, axis=1)[np.arange(8) * 4 // 8]
    np.testing.assert_array_equal(r["obj"].numpy(), up)
    np.testing.assert_allclose(r["prb"].numpy(), np.repeat(np.repeat(prb, 2, axis=2), 2, axis=1), rtol=1e-5,
                               atol=1e-6)
    exp = pos * 2
    exp[..., 1] += 0.5
    np.testing.assert_allclose(r["pos"].numpy(), exp)
    assert r["obj"].shape == (8, 16, 16) and r["prb"].shape == (2, 16, 16)


def test_h5_needs_h5py(tmp_path):
    if h5py is not None:
        pytest.skip("h5py is installed")
    with pytest.raises(ImportError):
        Writer(str(tmp_path), fmt="h5")
