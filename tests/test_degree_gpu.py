"""Degree statistics on the GPU (si_degree_stats): the inverted-list length of
every value and each set's sum of them, equal to numpy's on the same
collection; a value past the slots is reported."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _collection(el, off):
    import torch
    from set_intersection_b200 import api
    return api.Collection(torch.from_numpy(np.ascontiguousarray(el, np.uint32).view(np.int32)).cuda(),
                          torch.from_numpy(np.asarray(off, np.int64)).cuda(), int(el.max()) if el.size else 0)


@pytest.mark.parametrize("k,n_min,n_max,universe,seed", [(1, 1, 5, 16, 1), (500, 16, 5000, 1 << 14, 2),
                                                         (3000, 32, 1 << 16, 1 << 22, 3)])
def test_degree_stats_match_numpy(cuda, k, n_min, n_max, universe, seed):
    from set_intersection_b200 import api, generate
    el, off = generate.loguniform(seed, k, n_min, n_max, universe)
    inv, sums = api.degree_stats(_collection(el, off), universe)
    want_inv = np.bincount(el.astype(np.int64), minlength=universe)
    np.testing.assert_array_equal(inv.cpu().numpy().view(np.uint32), want_inv)
    per_el = want_inv[el.astype(np.int64)]
    want_sums = np.add.reduceat(per_el, off[:-1]) if el.size else np.zeros(k, np.int64)
    want_sums[np.diff(off) == 0] = 0
    np.testing.assert_array_equal(sums.cpu().numpy(), want_sums)


def test_empty_sets_and_value_past_the_slots(cuda):
    from set_intersection_b200 import api
    from set_intersection_b200._lib import SiError, Status
    el = np.array([1, 2, 3, 2, 9], np.uint32)
    off = np.array([0, 3, 3, 5], np.int64)
    inv, sums = api.degree_stats(_collection(el, off), 10)
    np.testing.assert_array_equal(inv.cpu().numpy(), [0, 1, 2, 1, 0, 0, 0, 0, 0, 1])
    np.testing.assert_array_equal(sums.cpu().numpy(), [4, 0, 3])
    with pytest.raises(SiError) as e:
        api.degree_stats(_collection(el, off), 9)
    assert e.value.status == Status.INVALID_INPUT
