"""emp_sort_pairs_static (the allocation-free sort: working set in a static
device array) against the existing entry point emp_sort_pairs on the same
inputs, two calls in a row (the second call reuses the static array the first
one left behind)."""
import numpy as np
import pytest
import torch

import empanada_b200
from empanada_b200 import _native

P1, P2 = 536870909, 536870879


def _pairs(seed, n, distinct):
    rng = np.random.default_rng(seed)
    f1 = rng.integers(0, P1, size=distinct, dtype=np.uint64)
    f2 = rng.integers(0, P2, size=distinct, dtype=np.uint64)
    pool = (f1 << np.uint64(32)) | f2
    keys = pool[rng.integers(0, distinct, size=n)]
    vals = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    return keys, vals


def _device(keys, vals):
    return torch.from_numpy(keys.view(np.int64)).cuda(), torch.from_numpy(vals.view(np.int32)).cuda()


def test_static_sort_rejects_more_than_its_maximum():
    """Checked before any device work: no GPU needed."""
    n = empanada_b200.SORT_STATIC_MAX_PAIRS + 1
    with pytest.raises(_native.EmpError) as e:
        empanada_b200.sort_pairs_static(0x1000, 0x2000, n)
    assert e.value.code == -1  # EMP_E_INVAL


@pytest.mark.gpu
def test_static_sort_matches_emp_sort_pairs_twice(engine):
    cases = [(11, empanada_b200.SORT_STATIC_MAX_PAIRS, 700_000), (12, 300_007, 5_000)]
    for seed, n, distinct in cases:
        keys, vals = _pairs(seed, n, distinct)
        sk, sv = _device(keys, vals)
        rk, rv = _device(keys, vals)
        torch.cuda.synchronize()
        empanada_b200.sort_pairs_static(sk.data_ptr(), sv.data_ptr(), n)
        engine.sort_pairs(rk.data_ptr(), rv.data_ptr(), n)
        torch.cuda.synchronize()
        assert torch.equal(sk, rk), f"keys differ (n={n})"
        assert torch.equal(sv, rv), f"values differ (n={n})"
        # the inputs were not already sorted: the call did reorder them
        assert not np.array_equal(sk.cpu().numpy().view(np.uint64), keys)
