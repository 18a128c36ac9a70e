"""aprict_b200: B200-native (sm_100a) cone-beam CT projection and reconstruction.

A drop-in for the projection / reconstruction path of aprict
(murdock-grewar/aprict 0.1.5, src/aprict/__init__.py:134-159): ``Volume``,
``FBVolume``, ``cb.flatpanel`` (ProjGeom, ProjectionSet, ConfigProject,
ConfigBackproject, project, backproject) and ``iterators`` (SIRT_flatpanel,
Landweber_flatpanel). Kernels live in libaprict_b200.so, reached through the C
ABI in include/aprict_b200.h.
"""

from .volume import FBVolume, Volume  # noqa: I001  (iterators import Volume from here)
from . import cb, iterators, phantoms, volume
from . import _structs as dtypes
from . import gbc, geometry, recon

__version__ = "0.1.0"

__all__ = ["FBVolume", "Volume", "__version__", "cb", "dtypes", "gbc", "geometry", "iterators", "phantoms", "recon",
           "volume"]
