"""nlfiber-b200: B200-native (sm_100a) voxel homogenization hot path of nlfiber.

linear   drop-in for nlfiber/linear.py (small-strain corrector solve, C, dC/drho) on libnlf.so
"""
from . import _lib  # noqa: F401  (loads libnlf.so; raises ImportError when it is missing)

__version__ = "0.1.0"
