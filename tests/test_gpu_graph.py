"""The unitig layer over output.bin (emp_graph_*) against its CPU
restatement (oracle/graph_oracle.c): the same unitigs and the same GFA bytes
on golden cases and on built graphs with cycles, branches and isolated
read-ends."""
import struct

import numpy as np
import pytest

import empanada_b200
from cases import BY_NAME
from oracle import bind


def _records(recs):
    out = b""
    for ovlp, pairs in recs:
        out += struct.pack("<Qi", len(pairs), ovlp)
        out += struct.pack(f"<{len(pairs)}I", *[p[0] for p in pairs])
        out += struct.pack(f"<{len(pairs)}I", *[p[1] for p in pairs])
    return out


def _check(engine, out_bin, n_reads, read_len, tmp_path):
    want = bind.gfa(out_bin, n_reads, read_len)
    order_o, starts_o = bind.unitigs(out_bin, n_reads)
    with empanada_b200.Graph(engine, out_bin, n_reads) as g:
        order, starts = g.unitigs()
        assert (order == order_o).all() and (starts == starts_o).all()
        p = tmp_path / "g.gfa"
        g.write_gfa(str(p), read_len)
        got = p.read_bytes()
        st = g.stats()
    assert got == want
    assert st["unitigs"] == len(starts_o) - 1
    return st


@pytest.mark.gpu
def test_built_graphs(engine, tmp_path):
    # a 3-cycle of read-ends, its reverse path, a branch, a self loop, isolated ends
    recs = [(40, [(0, 2), (2, 4), (4, 0), (5, 3), (3, 1)]),
            (39, [(6, 8), (6, 10), (8, 12), (10, 12), (14, 14)]),
            (38, []),
            (37, [(16, 18), (18, 20), (20, 22)])]
    st = _check(engine, _records(recs), 13, 50, tmp_path)
    assert st["cycles"] == 2  # the 3-cycle and the self loop


@pytest.mark.gpu
def test_random_graphs(engine, tmp_path):
    rng = np.random.default_rng(5)
    for n_reads, n_edges in [(50, 30), (500, 400), (20_000, 25_000)]:
        v = 2 * n_reads
        recs, left = [], n_edges
        ovlp = 99
        while left:
            k = int(min(left, rng.integers(0, 500)))
            pairs = list(zip(rng.integers(0, v, size=k).tolist(), rng.integers(0, v, size=k).tolist()))
            recs.append((ovlp, pairs))
            left -= k
            ovlp -= 1
        _check(engine, _records(recs), n_reads, 100, tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "dups_palindromes", "sub_errors", "split_r128k", "read_len_255", "small"])
def test_golden_outputs(engine, tmp_path, name):
    case = BY_NAME[name]
    out, st = empanada_b200.run_bytes(case.fastq(), engine=engine, min_ovlp=case.min_ovlp(),
                                      reduce_mem=case.reduce_mem())
    g = _check(engine, out, st["n_reads"], st["read_len"], tmp_path)
    assert g["edges"] == st["n_edges"]


def test_graph_arguments_without_a_gpu():
    import ctypes

    from empanada_b200 import _native

    lib = _native.lib()
    h = ctypes.c_void_p()
    assert lib.emp_graph_build(None, None, 0, 1, ctypes.byref(h)) == _native.EMP_E_INVAL
    assert lib.emp_graph_destroy(None) == _native.EMP_E_INVAL
    assert lib.emp_graph_write_gfa(None, b"x", 1) == _native.EMP_E_INVAL


def test_oracle_graph_basics():
    b = _records([(10, [(0, 2), (2, 4), (4, 0)]), (9, [(1, 3)])])
    order, starts = bind.unitigs(b, 3)
    assert order.tolist() == [0, 2, 4, 1, 3, 5] and starts.tolist() == [0, 3, 5, 6]
    text = bind.gfa(b, 3, 20).decode()
    assert "P\tutg0\t0+,1+,2+\t*" in text and "L\t0\t-\t1\t-\t9M" in text
