"""B200-native set-intersection engine.

Behind the reference's per-technique entry points (one executable per
technique, see set_intersection_b200/apps) and its dataset format
(set_intersection_b200.dataset), the compute runs in hand-written sm_100a
kernels in libsi_b200.so, reached through the C ABI of include/si.h.
"""
from ._lib import LIB_PATH, SiError, Status, Technique, declared_symbols, lib  # noqa: F401
from . import dataset, tiling  # noqa: F401

__version__ = "0.1.0"


def __getattr__(name):
    # api/generate import torch/numpy lazily so the format helpers stay light.
    if name in ("api", "generate"):
        import importlib
        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
