"""polyspec_b200 -- B200-native (sm_100a) backend of PolySpec's hot path.

``PolySpec(..., backend="cuda")``, ``Weightings``, ``CGD`` and ``PSpecBin``
mirror the reference classes of polyspec/base.py, polyspec/weighting.py and
polyspec/pspec_bin.py; the spherical harmonic transforms, pixel products and
solver kernels run on the GPU through the C ABI of libpscuda.so
(include/pscuda.h).  There is no CPU fallback.
"""
from .base import PolySpec
from .weighting import Weightings, CGD
from .pspec_bin import PSpecBin

__all__ = ["PolySpec", "Weightings", "CGD", "PSpecBin"]
