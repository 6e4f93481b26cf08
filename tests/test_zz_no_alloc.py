"""si_sisi_noalloc: the single-pair call for callers that cannot allocate
device memory (FFI hosts handed buffers by another runtime, engines whose
memory manager owns all of HBM, paths where cudaMalloc would synchronise the
device).  It must give exactly what si_sisi gives, call after call, while
taking its scratch from the library's own fixed device array.

Collected last on purpose (file name), so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from set_intersection_b200._lib import Status, lib


def _sorted_unique(rng, n, hi):
    return np.sort(rng.choice(hi, size=n, replace=False)).astype(np.uint32)


def test_rejects_pairs_beyond_the_scratch_limit():
    """|A| + |B| above 2^29 is refused on the host, before any GPU work (fake
    device pointers are never dereferenced)."""
    fake = ctypes.c_void_p(0x100000)
    nul = ctypes.c_void_p(None)
    big = (1 << 29) - 10
    assert lib.si_sisi_noalloc(fake, big, fake, 11, fake, nul, 0, nul) == Status.WORKSPACE_TOO_SMALL
    assert lib.si_sisi_noalloc(fake, 1 << 30, fake, 0, fake, nul, 0, nul) == Status.WORKSPACE_TOO_SMALL
    assert lib.si_sisi_noalloc(fake, 10, fake, 10, nul, nul, 0, nul) == Status.INVALID_ARGUMENT


def test_documented_limit_fits_the_scratch_array():
    """The limit |A| + |B| <= 2^29 is what the 4 MiB array holds: the
    intersect-path workspace of any such pair fits it."""
    ip = 0  # SI_TECH_IP
    for na, nb in [(1 << 28, 1 << 28), (1 << 29, 0), (0, 1 << 29), ((1 << 29) - 1, 1)]:
        assert lib.si_sisi_workspace_size(na, nb, ip) <= 4 << 20, (na, nb)


@pytest.mark.gpu
def test_matches_si_sisi_on_two_calls_in_a_row(cuda):
    import torch
    from set_intersection_b200 import api

    def dev(x):
        return torch.from_numpy(x.view(np.int32)).to(cuda)

    rng = np.random.default_rng(2024)
    # two calls in a row: a large pair, then a smaller one that finds the
    # first call's leftovers in the shared scratch array
    pairs = [(_sorted_unique(rng, 3_000_000, 1 << 25), _sorted_unique(rng, 2_000_000, 1 << 25)),
             (_sorted_unique(rng, 70_001, 1 << 20), _sorted_unique(rng, 50_003, 1 << 20))]
    stream = torch.cuda.current_stream(cuda)
    for a, b in pairs:
        da, db = dev(a), dev(b)
        want_count, want_out = api.intersect(da, db, "ip")  # the existing entry point, si_sisi
        want = want_out.cpu().numpy()

        count = torch.full((1,), -1, dtype=torch.int64, device=cuda)
        cap = max(1, min(a.size, b.size))
        out = torch.full((cap,), -1, dtype=torch.int32, device=cuda)
        st = lib.si_sisi_noalloc(ctypes.c_void_p(da.data_ptr()), a.size, ctypes.c_void_p(db.data_ptr()), b.size,
                                 ctypes.c_void_p(count.data_ptr()), ctypes.c_void_p(out.data_ptr()), cap,
                                 ctypes.c_void_p(stream.cuda_stream))
        assert st == Status.OK
        torch.cuda.synchronize(cuda)
        got_count = int(count.item())
        assert got_count == want_count
        np.testing.assert_array_equal(out[:got_count].cpu().numpy(), want)

        # ... and with the oracle
        import oracle
        np.testing.assert_array_equal(out[:got_count].cpu().numpy().view(np.uint32), oracle.set_intersection(a, b))
        assert lib.si_sisi_noalloc_check(ctypes.c_void_p(stream.cuda_stream)) == Status.OK

        count.fill_(-1)
        st = lib.si_sisi_noalloc(ctypes.c_void_p(da.data_ptr()), a.size, ctypes.c_void_p(db.data_ptr()), b.size,
                                 ctypes.c_void_p(count.data_ptr()), ctypes.c_void_p(None), 0,
                                 ctypes.c_void_p(stream.cuda_stream))
        assert st == Status.OK
        torch.cuda.synchronize(cuda)
        assert int(count.item()) == want_count
        assert lib.si_sisi_noalloc_check(ctypes.c_void_p(stream.cuda_stream)) == Status.OK
