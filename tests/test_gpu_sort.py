"""K3 (onesweep radix sort) through the C ABI (emp_sort_pairs) against a
stable numpy sort by (fp1, fp2, value>>31), the key order of the reference's
thrust::sort_by_key on fingerprints (cqutils.cuh:195)."""
import numpy as np
import pytest
import torch

P1, P2 = 536870909, 536870879


def _keys(rng, n, distinct):
    f1 = rng.integers(0, P1, size=distinct, dtype=np.uint64)
    f2 = rng.integers(0, P2, size=distinct, dtype=np.uint64)
    pool = (f1 << np.uint64(32)) | f2
    return pool[rng.integers(0, distinct, size=n)]


def _expected(keys, vals):
    sk = ((keys >> np.uint64(32)) << np.uint64(30)) | ((keys & np.uint64(0x1FFFFFFF)) << np.uint64(1)) | (
        vals.astype(np.uint64) >> np.uint64(31))
    order = np.argsort(sk, kind="stable")
    return keys[order], vals[order]


@pytest.mark.gpu
@pytest.mark.parametrize("n,distinct", [(1, 1), (2, 2), (4095, 100), (4096, 4096), (4097, 7), (100_000, 1000),
                                        (1_000_003, 900_000), (3_000_000, 3_000_000)])
def test_sort_pairs_stable(engine, n, distinct):
    rng = np.random.default_rng(n)
    keys = _keys(rng, n, distinct)
    vals = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    dv = torch.from_numpy(vals.view(np.int32)).cuda()
    torch.cuda.synchronize()
    engine.sort_pairs(dk.data_ptr(), dv.data_ptr(), n)
    gk = dk.cpu().numpy().view(np.uint64)
    gv = dv.cpu().numpy().view(np.uint32)
    ek, ev = _expected(keys, vals)
    assert (gk == ek).all()
    assert (gv == ev).all()
