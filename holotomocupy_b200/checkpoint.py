"""Reconstruction checkpoints: write the BH state, resume from it.

Reference: ``src/holotomocupy/writer.py:9-110`` (``Writer.write_checkpoint``)
and ``src/holotomocupy/reader.py:260-340`` (``Reader.read_checkpoint``).  Same
file layout and names:

    checkpoint_{iter:04}   /obj_re, /obj_im (complex objects)  [nzobj, nobj, nobj] float32
                           /prb_abs, /prb_phase                 [ndist, nz, n]      float32
                           /pos                                 [ntheta, ndist, 2]  float32
                           attributes iter, obj_dtype

written as HDF5 (``.h5``) when h5py is importable, else as a NumPy archive
(``.npz``) with the same dataset names and the attributes as 0-d arrays.
Reading infers a resolution scale from the probe width, as the reference
does: probe and object repeated by the scale in y and x, object slices mapped
nearest-neighbour, positions multiplied by the scale with half a pixel per
extra sample added in x.  One process writes the whole state (the reference's
MPI ranks write their slabs of one file collectively).
"""
import os

import numpy as np
import torch

try:
    import h5py
except ImportError:   # the image may lack it: the .npz layout carries the same datasets
    h5py = None


def _host(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


class Writer:
    """Checkpoint writer (writer.py:9).  ``fmt`` 'h5' needs h5py; 'npz' always works."""

    def __init__(self, path_out, obj_dtype="complex64", fmt=None):
        self.path_out = path_out
        self.obj_dtype = obj_dtype
        self.fmt = fmt or ("h5" if h5py is not None else "npz")
        if self.fmt == "h5" and h5py is None:
            raise ImportError("h5py is not installed: write checkpoints with fmt='npz'")
        os.makedirs(path_out, exist_ok=True)

    def path(self, i):
        return os.path.join(self.path_out, f"checkpoint_{i:04}.{self.fmt}")

    def write_checkpoint(self, vars, i, norm_const=1.0):
        """Save obj (times norm_const, as the iteration holds it divided), prb
        and pos of iteration i (writer.py:57-110); returns the file path."""
        obj = _host(vars["obj"]) * np.float32(norm_const)
        prb = _host(vars["prb"])
        data = {"obj_re": np.ascontiguousarray(obj.real, dtype="float32"),
                "prb_abs": np.abs(prb).astype("float32"), "prb_phase": np.angle(prb).astype("float32"),
                "pos": _host(vars["pos"]).astype("float32")}
        if self.obj_dtype == "complex64":
            data["obj_im"] = np.ascontiguousarray(obj.imag, dtype="float32")
        path = self.path(i)
        if self.fmt == "h5":
            with h5py.File(path, "w") as f:
                f.attrs["iter"] = i
                f.attrs["obj_dtype"] = self.obj_dtype
                for k, v in data.items():
                    f.create_dataset(k, data=v)
        else:
            np.savez(path, iter=np.array(i), obj_dtype=np.array(self.obj_dtype), **data)
        return path


def _load(path):
    if path.endswith(".h5"):
        if h5py is None:
            raise ImportError("h5py is not installed: cannot read " + path)
        with h5py.File(path, "r") as f:
            d = {k: f[k][:] for k in f.keys()}
            d["obj_dtype"] = f.attrs["obj_dtype"]
            d["iter"] = int(f.attrs["iter"])
        return d
    with np.load(path) as f:
        d = {k: f[k] for k in f.files}
    d["obj_dtype"] = str(d["obj_dtype"])
    d["iter"] = int(d["iter"])
    return d


def read_checkpoint(path, n, nzobj, obj_dtype="complex64", device=None):
    """Read a checkpoint, upsampled to detector width n and nzobj object slices
    (reader.py:260-340).  Returns {'obj', 'prb', 'pos', 'iter'} as torch
    tensors on `device` (obj scaled as written: multiply by 1/norm_const
    yourself if the solver expects it divided)."""
    d = _load(path)
    scale = n // d["prb_abs"].shape[-1]
    if scale < 1:
        raise ValueError(f"checkpoint probe width {d['prb_abs'].shape[-1]} exceeds n = {n}")
    prb = (d["prb_abs"] * np.exp(1j * d["prb_phase"])).astype("complex64")
    block = d["obj_re"] + 1j * d["obj_im"] if d["obj_dtype"] == "complex64" else d["obj_re"]
    for axis in (2, 1):
        prb = np.repeat(prb, scale, axis=axis)
        block = np.repeat(block, scale, axis=axis)
    nz_src = block.shape[0]
    idx = np.clip((np.arange(nzobj) * nz_src / nzobj).astype(np.intp), 0, nz_src - 1)
    obj = block[idx].astype(obj_dtype)
    pos = d["pos"].astype("float32") * scale
    pos[..., 1] += 0.5 * (scale - 1)
    dev = device if device is not None else "cpu"
    return {"obj": torch.from_numpy(np.ascontiguousarray(obj)).to(dev),
            "prb": torch.from_numpy(np.ascontiguousarray(prb)).to(dev),
            "pos": torch.from_numpy(np.ascontiguousarray(pos)).to(dev), "iter": d["iter"]}
