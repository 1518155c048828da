"""B200-native completeness scorer and grain grower for GrainRecon (LabDCT grain mapping).

* ``grainrecon_b200.geometry`` -- B matrix, reflections, detector rotation, MEX param vectors.
* ``grainrecon_b200._lib``     -- ctypes binding of the C ABI (libgrainrecon_b200.so).
* ``grainrecon_b200.forward``  -- mirrors of the MATLAB GPU wrappers on top of the C ABI.
* ``grainrecon_b200.synth``    -- seeded synthetic samples, spot masks and distance maps.
* ``grainrecon_b200.build``    -- in-tree nvcc build for sm_100a.
"""
from . import geometry  # noqa: F401

__all__ = ["geometry", "Context", "load"]


def __getattr__(name):
    if name in ("Context", "load", "GrcError"):
        from . import _lib
        return getattr(_lib, name)
    raise AttributeError(name)
