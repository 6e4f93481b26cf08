"""ctypes binding of libsi_b200.so (the C ABI declared in include/si.h).

The library is built in-tree (``make -C set_intersection_b200``); importing
this module fails loudly when it is missing -- there is no fallback path.
"""
from __future__ import annotations

import ctypes
import enum
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsi_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "si.h")


class Status(enum.IntEnum):
    OK = 0
    INVALID_ARGUMENT = 1
    WORKSPACE_TOO_SMALL = 2
    CUDA = 3
    UNSUPPORTED = 4
    TIMEOUT = 5
    INVALID_INPUT = 6
    OUTPUT_OVERFLOW = 7


class Technique(enum.IntEnum):
    IP = 0
    OBS = 1
    HI = 2
    BITMAP = 3
    BITMAP_NAIVE = 4
    MM = 5
    AUTO = 6


class SiError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = Status(status)
        msg = f"{where}: {self.status.name.lower()}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


def declared_symbols(header: str = HEADER_PATH) -> list[str]:
    """Names of the functions include/si.h declares."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(si_[a-z0-9_]+)\s*\(", text)))


_u32p = ctypes.POINTER(ctypes.c_uint32)
_vp = ctypes.c_void_p
_u64 = ctypes.c_uint64
_sz = ctypes.c_size_t
_int = ctypes.c_int


class SetRange(ctypes.Structure):
    """si_set_range: sets [start, end) of a collection."""
    _fields_ = [("start", ctypes.c_uint32), ("end", ctypes.c_uint32)]


_SIGNATURES = {
    "si_version": (ctypes.c_char_p, []),
    "si_status_string": (ctypes.c_char_p, [_int]),
    "si_last_error_string": (ctypes.c_char_p, []),
    "si_sisi_workspace_size": (_sz, [_u64, _u64, _int]),
    "si_sisi": (_int, [_vp, _u64, _vp, _u64, _int, _vp, _vp, _u64, _vp, _sz, _vp]),
    "si_sisi_noalloc": (_int, [_vp, _u64, _vp, _u64, _vp, _vp, _u64, _vp]),
    "si_sisi_noalloc_check": (_int, [_vp]),
    "si_sisi_host_workspace_size": (_sz, [_vp, _u64, _vp, _u64, _int, ctypes.c_uint32]),
    "si_sisi_host": (_int, [_vp, _u64, _vp, _u64, _int, ctypes.c_uint32, ctypes.POINTER(_u64), _vp, _u64, _vp, _sz,
                            _vp]),
    "si_host_ctx_create": (_int, [ctypes.POINTER(_vp)]),
    "si_host_ctx_destroy": (None, [_vp]),
    "si_sisi_host_ctx": (_int, [_vp, _vp, _u64, _vp, _u64, _int, ctypes.c_uint32, ctypes.POINTER(_u64), _vp, _u64,
                                _vp, _sz, _vp]),
    "si_workspace_check": (_int, [_vp, _vp]),
    "si_workspace_diagnostic": (_int, [_vp, _vp, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    "si_validate_sorted": (_int, [_vp, _u64, _vp, _vp]),
    "si_wait_selftest": (_int, [_vp, _u64, _vp]),
    "si_gen_uniform": (_int, [_u64, _u64, _u64, _u64, _vp, _int]),
    "si_gen_bernoulli": (_int, [_u64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, _vp, _vp, _int]),
    "si_gen_powerlaw": (_int, [_u64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double,
                               ctypes.c_uint32, ctypes.c_double, _vp, _vp, _int]),
    "si_misi_workspace_size": (_sz, [SetRange, SetRange, _int]),
    "si_gen_loguniform": (_int, [_u64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _vp, _vp,
                                 _int]),
    "si_batch_workspace_size": (_sz, [_u64]),
    "si_batch_count": (_int, [_vp, _vp, ctypes.c_uint32, _vp, _u64, _int, _vp, _vp, _vp, _sz, _vp]),
    "si_batch_tune": (_int, [_vp, _vp, ctypes.c_uint32, _vp, _u64, ctypes.c_uint32, _vp, _vp, _sz, _vp, _vp]),
    "si_batch_graph_create": (_int, [_vp, _vp, ctypes.c_uint32, _vp, _u64, _int, _vp, _vp, _vp, _sz,
                                     ctypes.POINTER(_vp)]),
    "si_batch_graph_launch": (_int, [_vp, _vp]),
    "si_batch_graph_destroy": (None, [_vp]),
    "si_degree_stats_workspace_size": (_sz, []),
    "si_degree_stats": (_int, [_vp, _vp, ctypes.c_uint32, _u64, _u64, _vp, _vp, _vp, _sz, _vp]),
    "si_misi": (_int, [_vp, _vp, SetRange, SetRange, _u64, _int, _vp, _vp, _sz, _vp]),
    "si_misi_dense_workspace_size": (_sz, [ctypes.c_uint32, ctypes.c_uint32, _int]),
    "si_misi_dense": (_int, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, _int, _int, _vp, _vp, _sz, _vp]),
    "si_timer_enable": (None, [_int]),
    "si_timer_reset": (None, []),
    "si_timer_read": (_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_u64)]),
}


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is not built; run `make -C set_intersection_b200` "
            "(or __graft_entry__.build()) first"
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int, where: str) -> None:
    if status != Status.OK:
        detail = lib.si_last_error_string().decode() if status == Status.CUDA else ""
        raise SiError(status, where, detail)
