"""emp_sort_pairs_static: the sort for callers that must not allocate device
memory (a host program that owns the device through its own arena or
allocator, or a latency-bound loop in which cudaMalloc / cudaFree would
synchronise the device).  Its working set is a static device array of the
library, so these tests check

* its output against a stable numpy sort by (fp1, fp2, value>>31), the key
  order of the reference's thrust::sort_by_key on fingerprints
  (cqutils.cuh:195), and against the allocating entry point emp_sort_pairs;
* two calls in a row (the second reuses what the first left in the array),
  a small call right after a large one, the one-CTA path (n <= 4096) and the
  tile edge (4096 / 4097), and a caller's own stream;
* that a call changes neither the device's free memory nor the torch
  allocator's;
* the size limit, checked before any device work.

This file is collected last so that a failure here leaves every other test
already run.
"""
import os
import re

import numpy as np
import pytest

import empanada_b200
from empanada_b200 import _native

P1, P2 = 536870909, 536870879
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _pairs(seed, n, distinct):
    rng = np.random.default_rng(seed)
    f1 = rng.integers(0, P1, size=distinct, dtype=np.uint64)
    f2 = rng.integers(0, P2, size=distinct, dtype=np.uint64)
    pool = (f1 << np.uint64(32)) | f2
    keys = pool[rng.integers(0, distinct, size=n)]
    vals = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    return keys, vals


def _expected(keys, vals):
    sk = ((keys >> np.uint64(32)) << np.uint64(30)) | ((keys & np.uint64(0x1FFFFFFF)) << np.uint64(1)) | (
        vals.astype(np.uint64) >> np.uint64(31))
    order = np.argsort(sk, kind="stable")
    return keys[order], vals[order]


def _device(keys, vals):
    import torch

    return torch.from_numpy(keys.view(np.int64)).cuda(), torch.from_numpy(vals.view(np.int32)).cuda()


def test_static_limit_matches_the_header():
    """The Python bound is the C constant EMP_SORT_STATIC_MAX_PAIRS."""
    hdr = open(os.path.join(ROOT, "include", "empanada.h")).read()
    m = re.search(r"#define\s+EMP_SORT_STATIC_MAX_PAIRS\s+\(1u\s*<<\s*(\d+)\)", hdr)
    assert m, "EMP_SORT_STATIC_MAX_PAIRS not found in include/empanada.h"
    assert empanada_b200.SORT_STATIC_MAX_PAIRS == _native.SORT_STATIC_MAX_PAIRS == 1 << int(m.group(1))


def test_static_sort_rejects_more_than_its_maximum():
    """Checked before any device work: no GPU needed."""
    n = empanada_b200.SORT_STATIC_MAX_PAIRS + 1
    with pytest.raises(_native.EmpError) as e:
        empanada_b200.sort_pairs_static(0x1000, 0x2000, n)
    assert e.value.code == -1  # EMP_E_INVAL


def test_static_sort_rejects_null_pointers():
    """n >= 1 with a NULL key or value pointer is EMP_E_INVAL, as for
    emp_sort_pairs; n = 0 is a no-op.  Checked before any device work."""
    for n in (1, 2):
        with pytest.raises(_native.EmpError) as e:
            empanada_b200.sort_pairs_static(0, 0x2000, n)
        assert e.value.code == -1
        with pytest.raises(_native.EmpError) as e:
            empanada_b200.sort_pairs_static(0x1000, 0, n)
        assert e.value.code == -1
    empanada_b200.sort_pairs_static(0, 0, 0)


def _sort_static_and_check(keys, vals, stream=None):
    import torch

    sk, sv = _device(keys, vals)
    torch.cuda.synchronize()
    sptr = stream.cuda_stream if stream is not None else 0
    empanada_b200.sort_pairs_static(sk.data_ptr(), sv.data_ptr(), len(keys), sptr)
    ek, ev = _expected(keys, vals)
    gk = sk.cpu().numpy().view(np.uint64)
    gv = sv.cpu().numpy().view(np.uint32)
    assert (gk == ek).all(), f"keys differ from the stable numpy order (n={len(keys)})"
    assert (gv == ev).all(), f"values differ from the stable numpy order (n={len(keys)})"
    return sk, sv


@pytest.mark.gpu
def test_static_sort_matches_numpy_and_emp_sort_pairs_twice(engine):
    """Two calls in a row, each checked against numpy and against the
    allocating entry point on the same input."""
    import torch

    cases = [(11, empanada_b200.SORT_STATIC_MAX_PAIRS, 700_000), (12, 300_007, 5_000)]
    for seed, n, distinct in cases:
        keys, vals = _pairs(seed, n, distinct)
        sk, sv = _sort_static_and_check(keys, vals)
        rk, rv = _device(keys, vals)
        torch.cuda.synchronize()
        engine.sort_pairs(rk.data_ptr(), rv.data_ptr(), n)
        torch.cuda.synchronize()
        assert torch.equal(sk, rk), f"keys differ from emp_sort_pairs (n={n})"
        assert torch.equal(sv, rv), f"values differ from emp_sort_pairs (n={n})"
        # the inputs were not already sorted: the call did reorder them
        assert not np.array_equal(sk.cpu().numpy().view(np.uint64), keys)


@pytest.mark.gpu
def test_static_sort_sizes_and_order_of_calls():
    """The one-CTA path (n <= 4096), the tile edge, and a small call right
    after the largest one (only the small call's look-back words are
    cleared, which must be enough)."""
    seq = [(21, 2, 2), (22, 4096, 300), (23, 4097, 7), (24, empanada_b200.SORT_STATIC_MAX_PAIRS, 1_000_000),
           (25, 4097, 4097), (26, 3, 1), (27, 70_001, 70_001)]
    for seed, n, distinct in seq:
        keys, vals = _pairs(seed, n, distinct)
        _sort_static_and_check(keys, vals)


@pytest.mark.gpu
def test_static_sort_on_a_caller_stream():
    import torch

    s = torch.cuda.Stream()
    keys, vals = _pairs(31, 123_457, 40_000)
    with torch.cuda.stream(s):
        _sort_static_and_check(keys, vals, stream=s)


@pytest.mark.gpu
def test_static_sort_allocates_nothing():
    """After a first call on the device (which loads the kernels), a call
    changes neither the device's free memory nor the torch allocator's
    counters."""
    import torch

    keys, vals = _pairs(41, 500_000, 200_000)
    _sort_static_and_check(keys, vals)
    sk, sv = _device(keys, vals)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    resv0 = torch.cuda.memory_reserved()
    empanada_b200.sort_pairs_static(sk.data_ptr(), sv.data_ptr(), len(keys))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    assert torch.cuda.memory_allocated() == alloc0 and torch.cuda.memory_reserved() == resv0
    ek, ev = _expected(keys, vals)
    assert (sk.cpu().numpy().view(np.uint64) == ek).all()
    assert (sv.cpu().numpy().view(np.uint32) == ev).all()
