"""mumax2 -- B200-native micromagnetic hot path behind MuMax2's quantity/module API.

`Plan` is the low-level handle of the fused CUDA path (libmm_b200.so).  The script
API (load/setv/run/...) mirroring src/python/mumax2.py lives in `engine`.
"""
from . import _native  # noqa: F401
from .plan import Ensemble, Plan  # noqa: F401
