"""geobrain_b200: GeoBrain's 2-D acoustic finite-difference propagator,
rebuilt for NVIDIA B200 (sm_100a).

``geobrain_b200.wave`` mirrors the acoustic part of ``geobrain.physics.wave``
(same names and call signatures); the compute is the CUDA library declared in
include/geobrain_b200.h, loaded from ``geobrain_b200/_so``.
"""
__version__ = "0.1.0"

from . import wave  # noqa: E402,F401
