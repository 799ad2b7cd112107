"""natinterp3d_b200: natural-neighbour (Sibson) interpolation in 3-D with the
query phase on an NVIDIA B200.

Drop-in for natinterp3d's API (``import natinterp3d_b200 as natinterp3d``):
``Interpolator``, ``get_weights`` and ``interpolate`` keep natinterp3d's
signatures and results.
"""
from .natinterp3d import Interpolator, interpolate, get_weights  # noqa: F401

__version__ = '0.1.0'
