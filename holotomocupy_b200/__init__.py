"""B200-native operator chain of holotomocupy's Bilinear-Hessian solver.

Drop-in classes with the reference's Python API (CUDA torch tensors in place
of CuPy arrays): ``Propagation`` (Fresnel D/DT), ``Tomo`` (USFFT R/RT),
``Shift`` (B-spline shift family), ``Rec`` (the BH cascade and solver) and
``RecNFP`` (near-field ptychography on the same cascade).
All compute runs in ``lib/libholotomo_b200.so`` (sm_100a).
"""
from .propagation import Propagation, fresnel_table  # noqa: F401
from .shift import Shift  # noqa: F401
from .tomo import Tomo  # noqa: F401
from .rec import Rec  # noqa: F401
from .rec_nfp import RecNFP  # noqa: F401

__version__ = "0.1.0"
