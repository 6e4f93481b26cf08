"""The C-ABI library loads and exports what include/si.h declares; host-side
argument checks and host generators work without a GPU."""
import ctypes
import subprocess

import numpy as np
import pytest

import set_intersection_b200 as si
from set_intersection_b200 import _lib
from set_intersection_b200._lib import Status, Technique


def test_every_declared_symbol_is_exported():
    declared = si.declared_symbols()
    assert "si_sisi" in declared
    out = subprocess.run(["nm", "-D", "--defined-only", si.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared if s not in exported]
    assert not missing, f"declared in include/si.h but not exported: {missing}"
    for s in declared:
        assert getattr(si.lib, s) is not None


def test_exports_are_plain_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", si.LIB_PATH], capture_output=True, text=True, check=True).stdout
    names = [line.split()[-1] for line in out.splitlines() if " T " in line]
    si_names = [n for n in names if n.startswith("si_")]
    assert si_names and all("_Z" not in n for n in si_names)


def test_version_and_status_strings():
    assert b"sm_100a" in si.lib.si_version()
    for s in Status:
        assert si.lib.si_status_string(int(s))
    assert si.lib.si_status_string(99) == b"unknown status"


def test_invalid_arguments_rejected_on_host():
    L = si.lib
    nul = ctypes.c_void_p(None)
    fake = ctypes.c_void_p(0x1000)
    # null count / workspace
    assert L.si_sisi(fake, 4, fake, 4, int(Technique.IP), nul, nul, 0, fake, 1 << 20, nul) == Status.INVALID_ARGUMENT
    assert L.si_sisi(fake, 4, fake, 4, int(Technique.IP), fake, nul, 0, nul, 1 << 20, nul) == Status.INVALID_ARGUMENT
    # misaligned set pointer
    assert L.si_sisi(ctypes.c_void_p(0x1002), 4, fake, 4, int(Technique.IP), fake, nul, 0, fake, 1 << 20,
                     nul) == Status.INVALID_ARGUMENT
    # output capacity below min(nA, nB)
    assert L.si_sisi(fake, 40, fake, 50, int(Technique.IP), fake, fake, 39, fake, 1 << 20,
                     nul) == Status.INVALID_ARGUMENT
    # workspace too small is detected before any launch
    assert L.si_sisi(fake, 1 << 20, fake, 1 << 20, int(Technique.IP), fake, nul, 0, fake, 64,
                     nul) == Status.WORKSPACE_TOO_SMALL
    # unknown technique
    assert L.si_sisi(fake, 4, fake, 4, 42, fake, nul, 0, fake, 1 << 20, nul) == Status.INVALID_ARGUMENT
    assert L.si_validate_sorted(fake, 4, nul, nul) == Status.INVALID_ARGUMENT
    assert L.si_workspace_check(nul, nul) == Status.INVALID_ARGUMENT


def test_batch_arguments_and_table_layout_on_host():
    """si_batch_count takes the four per-pair techniques and AUTO; the table
    layout (density class, log2 smaller size, log2 ratio) as si.h states it."""
    from set_intersection_b200 import api
    L = si.lib
    nul = ctypes.c_void_p(None)
    fake = ctypes.c_void_p(0x1000)
    for t in (Technique.BITMAP_NAIVE, Technique.MM, 42):
        assert L.si_batch_count(fake, fake, 2, fake, 1, int(t), None, fake, fake, 1 << 20,
                                nul) == Status.INVALID_ARGUMENT
    assert L.si_batch_count(fake, fake, 2, fake, 1, int(Technique.IP), None, fake, fake, 64,
                            nul) != Status.OK
    assert api.BATCH_TABLE_SIZE == 1024 and api.BATCH_CODES == 6
    assert api.batch_bucket(100, 100, 0, 99 * 300) == (3 << 8) | (6 << 4) | 0      # gap 300
    assert api.batch_bucket(100, 1600, 0, 1599 * 3) == (0 << 8) | (6 << 4) | 4     # gap 3, ratio 16
    assert api.batch_bucket(1600, 100, 10, 10 + 1599 * 31) == (1 << 8) | (6 << 4) | 4
    assert api.batch_bucket(0, 7, 0, 6000) == (3 << 8) | 15
    assert api.batch_bucket(5, 1, 0, 4000) == (3 << 8) | (0 << 4) | 2
    assert api.batch_bucket(1, 1) == (3 << 8) | (0 << 4) | 0
    with pytest.raises(ValueError):
        api._table(bytes(256))
    # the vectorised form over a host collection agrees with the scalar one
    rng = np.random.default_rng(1)
    sizes = rng.integers(0, 900, 300)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    el = np.concatenate([np.sort(rng.choice(int(rng.choice([1 << 10, 1 << 16, 1 << 26])), size=int(n), replace=False))
                         for n in sizes]).astype(np.uint32)
    pairs = rng.integers(0, 300, (3000, 2)).astype(np.uint32)
    want = []
    for a, b in pairs:
        na, nb = off[a + 1] - off[a], off[b + 1] - off[b]
        big = a if na >= nb else b
        n = off[big + 1] - off[big]
        want.append(api.batch_bucket(int(na), int(nb), int(el[off[big]]) if n else 0,
                                     int(el[off[big + 1] - 1]) if n else 0))
    np.testing.assert_array_equal(api.batch_buckets(el, off, pairs), want)


def test_dense_invalid_arguments_rejected_on_host():
    L = si.lib
    nul = ctypes.c_void_p(None)
    fake = ctypes.c_void_p(0x1000)
    mm, naive = int(Technique.MM), int(Technique.BITMAP_NAIVE)
    assert L.si_misi_dense(fake, fake, 10, 100, int(Technique.IP), 0, fake, fake, 1 << 20, nul) == Status.UNSUPPORTED
    assert L.si_misi_dense(fake, fake, 10, 100, mm, 2, fake, fake, 1 << 20, nul) == Status.INVALID_ARGUMENT
    assert L.si_misi_dense(fake, nul, 10, 100, mm, 0, fake, fake, 1 << 20, nul) == Status.INVALID_ARGUMENT
    assert L.si_misi_dense(fake, fake, 10, 100, mm, 0, nul, fake, 1 << 20, nul) == Status.INVALID_ARGUMENT
    assert L.si_misi_dense(fake, fake, 10, 100, mm, 0, fake, ctypes.c_void_p(0x1010), 1 << 20,
                           nul) == Status.INVALID_ARGUMENT
    assert L.si_misi_dense(fake, fake, 10, 1 << 24, mm, 0, fake, fake, 1 << 40, nul) == Status.UNSUPPORTED
    for t in (mm, naive):
        need = L.si_misi_dense_workspace_size(16384, 65535, t)
        assert L.si_misi_dense(fake, fake, 16384, 65535, t, 0, fake, fake, need - 1, nul) == \
            Status.WORKSPACE_TOO_SMALL
    # tensor-core operand: one byte per (set, value), rows padded to 256, values to 128
    assert L.si_misi_dense_workspace_size(16384, 65535, mm) == 256 + 16384 * 65536
    assert L.si_misi_dense_workspace_size(300, 200, mm) == 256 + 512 * 256
    # plain bitmaps: one bit per (set, value)
    assert L.si_misi_dense_workspace_size(16384, 65535, naive) == 256 + 16384 * 65536 // 8
    assert L.si_misi_dense_workspace_size(10, 100, int(Technique.IP)) == 0


def test_bernoulli_generator_density_and_determinism():
    from set_intersection_b200 import generate
    el, off = generate.bernoulli(9, 300, 4000, 0.05, threads=3)
    el2, off2 = generate.bernoulli(9, 300, 4000, 0.05, threads=11)
    assert np.array_equal(el, el2) and np.array_equal(off, off2)
    assert off[0] == 0 and np.all(np.diff(off) >= 0) and off[-1] == el.size
    assert abs(el.size / (300 * 4000) - 0.05) < 0.005
    for a in range(300):
        s = el[off[a]:off[a + 1]]
        assert np.all(np.diff(s.astype(np.int64)) > 0) and (s.size == 0 or s[-1] < 4000)
    full_el, full_off = generate.bernoulli(1, 3, 50, 1.0)
    assert np.array_equal(full_el, np.tile(np.arange(50, dtype=np.uint32), 3))
    empty_el, empty_off = generate.bernoulli(1, 3, 50, 0.0)
    assert empty_el.size == 0 and np.all(empty_off == 0)


def test_misi_invalid_arguments_rejected_on_host():
    L = si.lib
    R = _lib.SetRange
    nul = ctypes.c_void_p(None)
    fake = ctypes.c_void_p(0x1000)
    bm = int(Technique.BITMAP)
    ws = 1 << 30
    # dense techniques belong to si_misi_dense
    assert L.si_misi(fake, fake, R(0, 10), R(0, 10), 10, int(Technique.MM), fake, fake, ws, nul) == Status.UNSUPPORTED
    assert L.si_misi(fake, fake, R(0, 10), R(0, 10), 10, 42, fake, fake, ws, nul) == Status.INVALID_ARGUMENT
    assert L.si_misi(fake, nul, R(0, 10), R(0, 10), 10, bm, fake, fake, ws, nul) == Status.INVALID_ARGUMENT
    assert L.si_misi(fake, fake, R(0, 10), R(0, 10), 10, bm, nul, fake, ws, nul) == Status.INVALID_ARGUMENT
    # overlapping cross ranges, reversed range, stride below the tile
    assert L.si_misi(fake, fake, R(0, 10), R(5, 15), 10, bm, fake, fake, ws, nul) == Status.INVALID_ARGUMENT
    assert L.si_misi(fake, fake, R(10, 5), R(10, 5), 10, bm, fake, fake, ws, nul) == Status.INVALID_ARGUMENT
    assert L.si_misi(fake, fake, R(0, 10), R(0, 10), 9, bm, fake, fake, ws, nul) == Status.INVALID_ARGUMENT
    assert L.si_misi(fake, fake, R(0, 10), R(10, 30), 19, bm, fake, fake, ws, nul) == Status.INVALID_ARGUMENT
    # workspace too small is detected before any launch
    need = L.si_misi_workspace_size(R(0, 8192), R(0, 8192), bm)
    assert need > 8192 * 8
    assert L.si_misi(fake, fake, R(0, 8192), R(0, 8192), 8192, bm, fake, fake, need - 1,
                     nul) == Status.WORKSPACE_TOO_SMALL
    assert L.si_misi_workspace_size(R(0, 10), R(0, 10), int(Technique.MM)) == 0


def test_powerlaw_generator_sizes_values_and_determinism():
    from set_intersection_b200 import generate
    el, off = generate.powerlaw(5, 400, 16, 4096, 1.1, 1 << 16, 0.8, threads=3)
    el2, off2 = generate.powerlaw(5, 400, 16, 4096, 1.1, 1 << 16, 0.8, threads=7)
    assert np.array_equal(el, el2) and np.array_equal(off, off2)
    sizes = np.diff(off)
    assert sizes.min() >= 16 and sizes.max() <= 4096 and off[-1] == el.size
    # a power law with exponent 1.1 puts most sets near the lower end
    assert np.median(sizes) < sizes.mean() < 4096 / 2
    for a in range(400):
        s = el[off[a]:off[a + 1]]
        assert np.all(np.diff(s.astype(np.int64)) > 0) and s[0] >= 1 and s[-1] <= 1 << 16
    # Zipf popularity: small values are far more common than large ones
    assert np.count_nonzero(el <= 64) > 20 * np.count_nonzero((el > (1 << 16) - 64))
    # set a depends only on (seed, a): a prefix of the collection is the smaller collection
    el3, off3 = generate.powerlaw(5, 100, 16, 4096, 1.1, 1 << 16, 0.8)
    assert np.array_equal(el3, el[:off[100]]) and np.array_equal(off3, off[:101])


def test_workspace_size_grows_with_input():
    f = si.lib.si_sisi_workspace_size
    small = f(1000, 1000, int(Technique.IP))
    big = f(1 << 28, 1 << 28, int(Technique.IP))
    assert 0 < small < big
    # scratch is a small fraction of the input it partitions
    assert big < (2 << 28) * 4 // 100


def test_uniform_generator_is_exact_and_deterministic():
    from set_intersection_b200 import generate as g
    for n, hi in ((1000, 1 << 12), (5000, 1 << 30), (1 << 16, 1 << 18)):
        x = g.uniform(11, n, hi)
        assert x.size == n and x.dtype == np.uint32
        assert np.all(x[1:] > x[:-1]) and int(x[-1]) < hi
        np.testing.assert_array_equal(x, g.uniform(11, n, hi, threads=3))
        assert not np.array_equal(x, g.uniform(12, n, hi))
    full = g.uniform(1, 4096, 4096)
    np.testing.assert_array_equal(full, np.arange(4096, dtype=np.uint32))


def test_uniform_generator_rejects_bad_ranges():
    from set_intersection_b200 import generate as g
    with pytest.raises(_lib.SiError):
        g.uniform(1, 10, 5)
    with pytest.raises(_lib.SiError):
        g.uniform(1, 1, (1 << 32) + 1)


def test_skewed_generator_plants_overlap():
    import oracle
    from set_intersection_b200 import generate as g
    a, b = g.sisi_skewed(seed=9, n_small=1 << 10, n_large=1 << 16, universe=1 << 24)
    assert a.size == 1 << 10 and b.size == 1 << 16
    assert np.all(b[1:] > b[:-1])
    assert oracle.count(a, b) >= int(round(0.2 * a.size))


def test_host_pair_call_checks_arguments_on_host():
    """si_sisi_host: argument errors and a too-small workspace come back before
    any copy or launch; its workspace holds both sets, the output and the
    per-range scratch, and grows with the input."""
    L = si.lib
    nul = ctypes.c_void_p(None)
    fake = ctypes.c_void_p(0x10000)  # 256-byte aligned, never dereferenced
    a = np.arange(0, 4000, 2, dtype=np.uint32)
    b = np.arange(0, 3000, 3, dtype=np.uint32)
    pa, pb = a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p)
    out = np.zeros(min(a.size, b.size), dtype=np.uint32)
    po = out.ctypes.data_as(ctypes.c_void_p)
    cnt = ctypes.c_uint64(7)
    t = int(Technique.AUTO)
    need = L.si_sisi_host_workspace_size(pa, a.size, pb, b.size, t, 4)
    assert need >= 4 * (a.size + b.size + min(a.size, b.size))
    assert L.si_sisi_host_workspace_size(pa, a.size << 1, pa, a.size << 1, t, 4) > 0
    # null count, null workspace, misaligned workspace, short output, short workspace
    assert L.si_sisi_host(pa, a.size, pb, b.size, t, 4, None, po, out.size, fake, need, nul) == Status.INVALID_ARGUMENT
    assert L.si_sisi_host(pa, a.size, pb, b.size, t, 4, ctypes.byref(cnt), po, out.size, nul, need,
                          nul) == Status.INVALID_ARGUMENT
    assert L.si_sisi_host(pa, a.size, pb, b.size, t, 4, ctypes.byref(cnt), po, out.size, ctypes.c_void_p(0x10010),
                          need, nul) == Status.INVALID_ARGUMENT
    assert L.si_sisi_host(pa, a.size, pb, b.size, t, 4, ctypes.byref(cnt), po, out.size - 1, fake, need,
                          nul) == Status.INVALID_ARGUMENT
    assert L.si_sisi_host(pa, a.size, pb, b.size, t, 4, ctypes.byref(cnt), po, out.size, fake, need - 1,
                          nul) == Status.WORKSPACE_TOO_SMALL
    # an empty set: count 0 without touching the device
    assert L.si_sisi_host(pa, 0, pb, b.size, t, 0, ctypes.byref(cnt), po, out.size, fake,
                          L.si_sisi_host_workspace_size(pa, 0, pb, b.size, t, 0), nul) == Status.OK
    assert cnt.value == 0


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_reports(cuda):
    """A device wait on a phase that nothing completes gives up after its
    limit (here 0.2 s), reports SI_ERR_TIMEOUT through the workspace's error
    word, and the context stays usable for the next call."""
    import time
    import torch
    from set_intersection_b200 import api
    ws = torch.zeros(64, dtype=torch.int32, device=cuda)
    nul = ctypes.c_void_p(None)
    t0 = time.time()
    assert si.lib.si_wait_selftest(ctypes.c_void_p(ws.data_ptr()), 200_000_000, nul) == Status.TIMEOUT
    assert time.time() - t0 < 3.0
    site, detail = ctypes.c_uint32(0), ctypes.c_uint32(0)
    assert si.lib.si_workspace_diagnostic(ctypes.c_void_p(ws.data_ptr()), nul, ctypes.byref(site),
                                          ctypes.byref(detail)) == Status.TIMEOUT
    assert site.value == 31
    a = torch.arange(0, 1000, 2, dtype=torch.int32, device=cuda)
    b = torch.arange(0, 1000, 3, dtype=torch.int32, device=cuda)
    c, _ = api.intersect(a, b, "auto")
    assert c == 167
