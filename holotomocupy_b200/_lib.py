"""ctypes binding of ``lib/libholotomo_b200.so`` (declared in include/holotomo_b200.h).

The library is required: importing an operator without it raises at once,
there is no fallback implementation.
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libholotomo_b200.so")

_c_int, _c_long, _vp = ctypes.c_int, ctypes.c_long, ctypes.c_void_p
_c_float, _c_double = ctypes.c_float, ctypes.c_double

# name -> argtypes (all return int status unless listed in _RESTYPE)
SIGNATURES = {
    "ht_version": [],
    "ht_last_error": [],
    "ht_launch_count": [],
    "ht_host_register": [_vp, _c_long, _vp],
    "ht_host_unregister": [_vp],
    "ht_prop_create": [_c_int, _c_int, _c_int, _vp, ctypes.POINTER(_vp)],
    "ht_prop_destroy": [_vp],
    "ht_prop_D": [_vp, _vp, _vp, _c_long, _c_int, _vp],
    "ht_prop_DT": [_vp, _vp, _vp, _c_long, _c_int, _vp],
    "ht_conv2d_create": [_c_int, _c_int, ctypes.POINTER(_vp)],
    "ht_conv2d_destroy": [_vp],
    "ht_conv2d_run": [_vp, _vp, _vp, _vp, _c_long, _vp],
    "ht_pad_mirror": [_vp, _vp, _c_long, _c_int, _c_int, _vp],
    "ht_pad_fold": [_vp, _vp, _c_long, _c_int, _c_int, _vp],
    "ht_tomo_create": [_c_int, _c_int, _c_int, _vp, _vp, ctypes.POINTER(_vp)],
    "ht_tomo_destroy": [_vp],
    "ht_tomo_R": [_vp, _vp, _vp, _c_int, _vp],
    "ht_tomo_RT": [_vp, _vp, _vp, _c_int, _vp],
    "ht_tomo_R_coeffx": [_vp, _vp, _vp, _c_int, _vp],
    "ht_tomo_RT_coeffx": [_vp, _vp, _vp, _c_int, _c_float, _vp],
    "ht_tomo_R_slab": [_vp, _vp, _vp, _c_int, _c_int, _c_int, _vp],
    "ht_tomo_RT_slab": [_vp, _vp, _vp, _c_int, _c_int, _c_int, _c_float, _vp],
    "ht_shift_create": [_c_int, _c_int, _c_int, _c_int, _c_int, ctypes.POINTER(_vp)],
    "ht_shift_destroy": [_vp],
    "ht_shift_coeff": [_vp, _vp, _vp, _c_long, _vp],
    "ht_shift_filter": [_vp, _vp, _vp, _c_long, _vp, _vp, _vp],
    "ht_shift_Sback": [_vp, _vp, _vp, _vp, ctypes.c_int, _vp, _c_long, _vp],
    "ht_shift_coeff_z": [_vp, _vp, _vp, _c_long, _vp],
    "ht_shift_S": [_vp, _vp, _vp, _vp, _vp, _c_long, _vp],
    "ht_shift_Sadj": [_vp, _vp, _vp, _vp, _vp, _c_long, _vp],
    "ht_shift_dS": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_long, _vp],
    "ht_shift_d2S": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_long, _vp],
    "ht_shift_dSadj": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_long, _vp],
    "ht_filter_rows": [_c_int, _vp, _vp, _c_long, _vp, _vp],
    "ht_prbfit_grad": [_vp, _vp, _vp, _vp, _vp, _c_float, _vp],
    "ht_prbfit_forms": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_double, _c_int, _vp],
    "ht_laplacian_grad": [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_float, _vp, _vp],
    "ht_laplacian_dot": [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_double, _vp, _vp, _vp, _vp, _vp],
    "ht_laplacian_energy": [_vp, _c_int, _c_int, _c_int, _c_int, _c_double, _vp, _vp, _vp],
    "ht_axpby": [_vp, _vp, _c_float, _c_float, _c_long, _vp, _vp],
    "ht_dot": [_vp, _vp, _c_long, _vp, _vp],
    "ht_axpby_dev": [_vp, _vp, _vp, _c_float, _vp, _c_float, _c_long, _vp, _vp],
    "ht_bh_scalars": [_vp, _vp, _c_int, _c_int, _c_double, _c_double, _c_double, _vp, _vp, _c_int, _vp, _vp],
    "ht_graph_begin": [_vp],
    "ht_graph_end": [_vp, ctypes.POINTER(_vp)],
    "ht_graph_launch": [_vp, _vp],
    "ht_graph_destroy": [_vp],
    "ht_ktimer_arm": [ctypes.c_char_p, _c_int],
    "ht_ktimer_read": [ctypes.c_char_p, ctypes.POINTER(_c_double), ctypes.POINTER(_c_long), ctypes.POINTER(_c_double)],
    "ht_rec_create": [_c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _vp, ctypes.POINTER(_vp)],
    "ht_rec_destroy": [_vp],
    "ht_rec_forward": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "ht_rec_gradient": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_float, _c_float, _c_int, _vp],
    "ht_rec_set_data_size": [_vp, _c_double],
    "ht_rec_set_shared_coefficients": [_vp, _c_int],
    "ht_rec_objective_noalloc": [_vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "ht_rec_hessian": [_vp, _vp, _vp, _vp, _vp, _vp, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_int, _vp],
}
_RESTYPE = {"ht_last_error": ctypes.c_char_p, "ht_launch_count": ctypes.c_long}

_lib = None


class HoloError(RuntimeError):
    """A holotomo_b200 entry point returned a non-zero status."""


def lib():
    """Load the shared library once; raise if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m holotomocupy_b200.build` "
                "(the operators have no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, argt in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = argt
            fn.restype = _RESTYPE.get(name, _c_int)
        _lib = L
    return _lib


def call(name, *args):
    """Call an entry point and raise HoloError on a non-zero status."""
    L = lib()
    st = getattr(L, name)(*args)
    if st != 0:
        msg = L.ht_last_error().decode(errors="replace")
        raise HoloError(f"{name} failed with status {st}: {msg}")
    return st


def stream_ptr(device=None):
    return _vp(torch.cuda.current_stream(device).cuda_stream)


def ptr(t):
    """Device address of a tensor's storage.  A lazily conjugated or negated
    view (torch's conj/neg bits) would hand the kernel the unconjugated data,
    so such views are refused: resolve_conj() / resolve_neg() them first."""
    if t.is_conj() or t.is_neg():
        raise ValueError("lazily conjugated/negated tensor: call resolve_conj()/resolve_neg() before passing it")
    return _vp(t.data_ptr())


def require_cuda(t, name, dtype=None):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA torch tensor")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must have dtype {dtype}, got {t.dtype}")
