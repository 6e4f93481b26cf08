"""CPU oracle for the set-intersection engine -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
reference legs, as the checker; the product package never imports it.

Two layers:
  * liboracle.so: si_oracle.c, a C restatement of the reference's CPU
    techniques (std::set_intersection, serial_intersect, boost_bitset), each
    function citing the reference file:line it follows;
  * _ref/: the reference's own CPU executables compiled from its sources
    (stdintersection, serial_intersect, boost_bitset, txt2bin, bin2txt) plus
    ref_elements, built by `make -C oracle ref` where the reference checkout
    exists.  They pin the restatement (tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

STD, SERIAL, BITSET = 0, 1, 2
_TECH = {"std": STD, "std_set_intersection": STD, "stdintersection": STD,
         "serial": SERIAL, "serial_intersect": SERIAL,
         "bitset": BITSET, "boost_bitset": BITSET}

_lib = None


def build() -> None:
    subprocess.run(["make", "-C", HERE, "all"], check=True, capture_output=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, u64, u32, i = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int
        L.si_oracle_set_intersection.restype = u64
        L.si_oracle_set_intersection.argtypes = [vp, u64, vp, u64, vp]
        L.si_oracle_serial_intersect.restype = u64
        L.si_oracle_serial_intersect.argtypes = [vp, u64, vp, u64]
        L.si_oracle_all_pairs.restype = i
        L.si_oracle_all_pairs.argtypes = [vp, vp, u32, u32, i, i, vp]
        L.si_oracle_pairs.restype = i
        L.si_oracle_pairs.argtypes = [vp, vp, u32, vp, u64, i, vp]
        L.si_oracle_triangular_index.restype = u64
        L.si_oracle_triangular_index.argtypes = [u64, u64, u64]
        L.si_oracle_is_strictly_increasing.restype = i
        L.si_oracle_is_strictly_increasing.argtypes = [vp, u64]
        L.si_oracle_gen_uniform.restype = i
        L.si_oracle_gen_uniform.argtypes = [u64, u64, u64, u64, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> ctypes.c_void_p:
    return a.ctypes.data_as(ctypes.c_void_p)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def set_intersection(a, b) -> np.ndarray:
    """Elements of a ∩ b in std::set_intersection order."""
    a, b = _u32(a), _u32(b)
    out = np.empty(max(1, min(a.size, b.size)), dtype=np.uint32)
    n = lib().si_oracle_set_intersection(_p(a), a.size, _p(b), b.size, _p(out))
    return out[:n].copy()


def count(a, b, technique: str = "std") -> int:
    a, b = _u32(a), _u32(b)
    if _TECH[technique] == SERIAL:
        return int(lib().si_oracle_serial_intersect(_p(a), a.size, _p(b), b.size))
    return int(lib().si_oracle_set_intersection(_p(a), a.size, _p(b), b.size, None))


def all_pairs(elements, offsets, k: int, universe: int, technique: str = "std", threads: int = 0) -> np.ndarray:
    """uint32 counts of every pair a<b in triangular order (include/util.hpp:68-70)."""
    e = _u32(elements)
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    out = np.zeros(max(1, k * (k - 1) // 2), dtype=np.uint32)
    rc = lib().si_oracle_all_pairs(_p(e), _p(off), k, universe, _TECH[technique], threads, _p(out))
    if rc != 0:
        raise RuntimeError("si_oracle_all_pairs failed")
    return out[: k * (k - 1) // 2]


def pairs(elements, offsets, k: int, pair_list, threads: int = 0) -> np.ndarray:
    e = _u32(elements)
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    pl = np.ascontiguousarray(pair_list, dtype=np.uint32).reshape(-1)
    out = np.zeros(max(1, pl.size // 2), dtype=np.uint32)
    rc = lib().si_oracle_pairs(_p(e), _p(off), k, _p(pl), pl.size // 2, threads, _p(out))
    if rc != 0:
        raise RuntimeError("si_oracle_pairs failed")
    return out[: pl.size // 2]


def gen_uniform(seed: int, n: int, hi: int, lo: int = 0) -> np.ndarray:
    """The engine's seeded uniform n-subset of [lo, hi), ascending, restated in
    C (si_oracle_gen_uniform), so a reference run reads the very sets the
    engine is timed on without loading the engine's library."""
    out = np.empty(max(n, 1), dtype=np.uint32)
    rc = lib().si_oracle_gen_uniform(seed, n, lo, hi, _p(out))
    if rc != 0:
        raise RuntimeError(f"si_oracle_gen_uniform failed ({rc})")
    return out[:n]


def write_dataset(path: str, sets, universe: int) -> None:
    """A dataset file in the reference's binary format (include/io.hpp:70-89:
    u32 cardinality, u32 universe, u64 total elements, u32 sizes[], u32
    elements[]), written with numpy only."""
    sizes = np.array([len(x) for x in sets], dtype=np.uint32)
    with open(path, "wb") as f:
        np.array([len(sets), universe], dtype=np.uint32).tofile(f)
        np.array([int(sizes.sum(dtype=np.uint64))], dtype=np.uint64).tofile(f)
        sizes.tofile(f)
        for x in sets:
            np.ascontiguousarray(x, dtype=np.uint32).tofile(f)


def is_strictly_increasing(x) -> bool:
    x = _u32(x)
    return bool(lib().si_oracle_is_strictly_increasing(_p(x), x.size))


# ------------------------------------------------------------ reference run --
def ref_binary(name: str) -> str | None:
    p = os.path.join(REF_DIR, name)
    return p if os.access(p, os.X_OK) else None


def run_ref(name: str, dataset_path: str, output_path: str | None = None, threads: int | None = None,
            timeout: float = 600.0) -> dict:
    """Runs a reference CPU executable (oracle/_ref/<name>) on a dataset file.

    Returns {"stdout": ..., "host_ms": {interval name: ms}} where host_ms are
    the reference's own HostTimer figures (include/host_timer.hpp:48-61)."""
    exe = ref_binary(name)
    if exe is None:
        raise FileNotFoundError(f"{REF_DIR}/{name} not built (make -C oracle ref)")
    cmd = [exe, "--input", dataset_path]
    if output_path:
        cmd += ["--output", output_path]
    if threads:
        cmd += ["--threads", str(threads)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{name} exited {r.returncode}: {r.stdout[-500:]} {r.stderr[-500:]}")
    host_ms = {}
    for m in re.finditer(r"│\s*([^|│]+?)\s*\|\s*([0-9.]+)\s*│", r.stdout):
        host_ms[m.group(1)] = float(m.group(2))
    return {"stdout": r.stdout, "host_ms": host_ms}
