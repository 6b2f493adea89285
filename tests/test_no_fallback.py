"""The operators have no CPU fallback: without the library, without a GPU,
or given host tensors, they raise instead of computing elsewhere."""
import numpy as np
import pytest
import torch


def test_missing_library_raises(monkeypatch):
    from holotomocupy_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libholotomo_b200.so")
    with pytest.raises(ImportError, match="no CPU fallback"):
        _lib.lib()


def test_host_tensors_are_refused():
    from holotomocupy_b200 import _lib
    with pytest.raises(TypeError, match="CUDA torch tensor"):
        _lib.require_cuda(torch.zeros(3), "x")
    with pytest.raises(TypeError, match="CUDA torch tensor"):
        _lib.require_cuda(np.zeros(3), "x")


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour on a machine without a GPU")
def test_operators_raise_without_a_gpu():
    from holotomocupy_b200 import Propagation, Tomo
    with pytest.raises(RuntimeError):
        Propagation(16, 16, 1, 1, 1e-10, 1e-8, np.array([1e-3]))
    with pytest.raises(RuntimeError):
        Tomo(16, 16, np.linspace(0, np.pi, 4, endpoint=False).astype("float32"), 1)
