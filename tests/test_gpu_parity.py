"""CUDA path vs the reference's own output (golden digests) and the oracle.

Every case of tests/golden/cases.py runs through the C ABI (emp_job_*); the
output.bin bytes must equal the reference's (sha256 from golden.json, and the
verbatim fixture where committed) and the oracle's.
"""
import dataclasses
import hashlib
import json
import os

import pytest

import empanada_b200
from cases import BY_NAME, CASES
from oracle import bind

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN = json.load(open(os.path.join(HERE, "golden.json")))

FAST_CASES = [c.name for c in CASES if not c.big]
OUT_OF_CORE = [c.name for c in CASES if c.name.startswith("out_of_core")]


def _run(engine, case):
    data = case.fastq()
    a = list(case.args)
    opts = dict(zip(a[::2], a[1::2]))
    out, st = empanada_b200.run_bytes(
        data, engine=engine, min_ovlp=int(opts.get("-o", 31)), map_mem=opts.get("-m", "1g"),
        reduce_mem=opts.get("-r", "1g"), base_blocksz=opts.get("-b", "32m"), kv_chunksz=opts.get("-c", "64m"))
    return data, out, st


@pytest.mark.gpu
@pytest.mark.parametrize("name", FAST_CASES)
def test_case_matches_reference(engine, name):
    case = BY_NAME[name]
    g = GOLDEN[name]
    data, out, st = _run(engine, case)
    assert hashlib.sha256(data).hexdigest() == g["fastq_sha256"], "input generator drifted"
    assert len(out) == g["size"]
    assert hashlib.sha256(out).hexdigest() == g["sha256"]
    if g.get("inline"):
        assert out == open(os.path.join(HERE, f"{name}.bin"), "rb").read()
    ref, rst = bind.run(data, case.min_ovlp(), case.reduce_mem())
    assert out == ref
    assert st["n_edges"] == rst["n_edges"]
    assert st["n_records"] == rst["n_records"]
    assert st["n_unique"] == rst["n_unique"]
    assert st["gpu_launches"] > 0 or st["n_reads"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small", "larger", "repeats_10m", "repeats_10m_r100m"])
def test_full_size_workload_matches_reference(engine, name):
    """Configs 1 and 2 at full size, config 3 at a tenth (in core, and out of
    core at -r 100m): byte-identical to the reference's output.bin."""
    case = BY_NAME[name]
    g = GOLDEN[name]
    data, out, st = _run(engine, case)
    assert hashlib.sha256(data).hexdigest() == g["fastq_sha256"]
    assert st["n_edges"] == g["edges"]
    assert st["n_records"] == g["records"]
    assert len(out) == g["size"]
    assert hashlib.sha256(out).hexdigest() == g["sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["config3_hbm", "config3_r1g"])
def test_config3_full_size_matches_reference(engine, name):
    """Config 3 at full size (100 Mbp genome with 5 % repeat families, 33.3M
    x 150 bp reads, 10.5 GB of FASTQ): HBM-sized (-m 160g -r 160g, every
    table in one chunk and one search window) and -m 1g -r 1g (the
    fingerprint sort chunked, the first rounds split into records of M/2
    windows).  output.bin must equal the reference's byte for byte."""
    import numpy as np

    from empanada_b200 import synth

    case = BY_NAME[name]
    g = GOLDEN.get(name)
    if not g or "sha256" not in g:
        pytest.fail(f"no golden digest for {name}: run tests/golden/make_golden.py {name}")
    w = dataclasses.replace(synth.SMALL, **case.synth)
    buf = np.empty(synth.fastq_size(w), dtype=np.uint8)
    synth.fastq_into(w, buf)
    assert buf.size == g["fastq_size"]
    a = list(case.args)
    opts = dict(zip(a[::2], a[1::2]))
    with engine.job(min_ovlp=int(opts["-o"]), map_mem=opts["-m"], reduce_mem=opts["-r"]) as job:
        job.feed(buf)
        del buf
        job.run()
        st = job.stats()
        out = job.output()
    assert st["n_edges"] == g["edges"]
    assert st["n_records"] == g["records"]
    assert len(out) == g["size"]
    assert hashlib.sha256(out).hexdigest() == g["sha256"]


ROUND_MODES = {
    "default": {},
    "sync_rounds": {"round_driver": 1},
    "edge_restart": {"edge_cap": 8},
    "sync_edge_restart": {"round_driver": 1, "edge_cap": 8},
    "region_spill": {"region_cap": 7},
    "region_spill_some": {"region_cap": 40},
    "small_buckets": {"bucket_mean": 512},
    "sort_dedup": {"dedup_driver": 1},
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "sub_errors", "dups_palindromes", "split_r128k", "read_len_1"])
@pytest.mark.parametrize("mode", sorted(ROUND_MODES))
def test_round_paths_agree(engine, name, mode):
    """Every round driver and engine choice gives the reference's bytes:
    host-synchronised rounds (full sort per round), the bucket kernel (the
    default), each restarted after an edge-buffer overflow, the bucket kernel
    with list regions so small that most (or some) entries go to the spill
    area, and with smaller buckets."""
    case = BY_NAME[name]
    with engine.tuned(**ROUND_MODES[mode]):
        data, out, st = _run(engine, case)
    assert hashlib.sha256(out).hexdigest() == GOLDEN[name]["sha256"]


@pytest.mark.gpu
def test_many_buckets_direct_binning(engine):
    """More than 2048 key buckets in a round (the 1.2M x 250 bp workload at
    512 entries per bucket): entries take their list positions straight from
    the bin counters instead of a shared-memory histogram."""
    case = BY_NAME["larger"]
    with engine.tuned(bucket_mean=512):
        data, out, st = _run(engine, case)
    assert hashlib.sha256(out).hexdigest() == GOLDEN["larger"]["sha256"]


@pytest.mark.gpu
def test_grid_barrier_timeout_is_reported(engine):
    """A grid-barrier wait that runs out (a barrier no arrival completes,
    with a 2 ms limit) ends the launch with EMP_E_TIMEOUT on the host; the
    engine then runs the same job, and another, correctly."""
    case = BY_NAME["tiny"]
    with engine.tuned(wait_limit_ns=2_000_000, block_next_wait=1):
        with engine.job(min_ovlp=case.min_ovlp()) as job:
            job.feed(case.fastq())
            with pytest.raises(empanada_b200._native.EmpError) as e:
                job.run()
            assert e.value.code == empanada_b200._native.EMP_E_TIMEOUT
            assert engine.tuning()["block_next_wait"] == 0  # used up by that launch
            job.reset()
            job.feed(case.fastq())
            job.run()
            assert hashlib.sha256(job.output()).hexdigest() == GOLDEN["tiny"]["sha256"]
    data, out, st = _run(engine, BY_NAME["sub_errors"])
    assert hashlib.sha256(out).hexdigest() == GOLDEN["sub_errors"]["sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", OUT_OF_CORE)
@pytest.mark.parametrize("mode", ["default", "sync_rounds", "edge_restart"])
def test_out_of_core_order(engine, name, mode):
    """2n > M: the reference's chunked sort (M-entry chunks merged through a
    FIFO) decides the duplicate survivors and the tie order of the large
    rounds; every round driver gives the reference's bytes."""
    with engine.tuned(**ROUND_MODES[mode]):
        data, out, st = _run(engine, BY_NAME[name])
    g = GOLDEN[name]
    assert hashlib.sha256(out).hexdigest() == g["sha256"]
    assert st["n_unique"] == g["unique"]
    assert st["n_records"] == g["records"]


@pytest.mark.gpu
def test_duplicate_walk_hang_is_reported(engine):
    """Where the reference's duplicate-removal walk never advances, the job
    fails with EMP_E_HANG and the engine stays usable."""
    import cases

    with engine.job(min_ovlp=20, reduce_mem="16k") as job:
        job.feed(cases.edge_ooc_hang())
        with pytest.raises(empanada_b200._native.EmpError) as e:
            job.run()
        assert e.value.code == empanada_b200._native.EMP_E_HANG
    out, _ = empanada_b200.run_bytes(cases.edge_ooc_hang(), engine=engine, min_ovlp=20)
    ref, _ = bind.run(cases.edge_ooc_hang(), 20, 1 << 30)
    assert out == ref


def _long_reads(L, n, seed, sub=0.002):
    """Reads beyond the reference's MAX_RD_LEN (its result is undefined
    there): checked against the oracle's extension of the same hash."""
    from empanada_b200 import synth

    w = synth.Workload(f"L{L}", seed=seed, genome_len=max(4 * L, n * L // 12), n_reads=n, read_len=L, sub_rate=sub)
    return synth.fastq_bytes(w)


@pytest.mark.gpu
@pytest.mark.parametrize("L,o", [(256, 31), (300, 31), (384, 200), (512, 31), (512, 500)])
def test_long_reads_match_oracle(engine, L, o):
    data = _long_reads(L, 3000, seed=L + o)
    out, st = empanada_b200.run_bytes(data, engine=engine, min_ovlp=o)
    ref, rst = bind.run(data, o)
    assert st["read_len"] == L
    assert out == ref
    assert st["n_edges"] == rst["n_edges"] and st["n_rounds"] == rst["n_rounds"]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["sync_rounds", "small_buckets", "split_r64k"])
def test_long_reads_round_paths(engine, mode):
    r = 64 << 10 if mode == "split_r64k" else 1 << 30
    data = _long_reads(300, 2500, seed=7)
    with engine.tuned(**ROUND_MODES.get(mode, {})):
        out, _ = empanada_b200.run_bytes(data, engine=engine, min_ovlp=40, reduce_mem=r)
    ref, _ = bind.run(data, 40, r)
    assert out == ref


@pytest.mark.gpu
def test_read_longer_than_512_is_unsupported(engine):
    with engine.job() as job:
        job.feed(_long_reads(513, 50, seed=3))
        with pytest.raises(empanada_b200._native.EmpError) as e:
            job.run()
        assert e.value.code == empanada_b200._native.EMP_E_UNSUPPORTED


@pytest.mark.gpu
def test_fingerprints_match_oracle(engine):
    for name in ["tiny", "odd_len", "lowercase", "read_len_255", "read_len_1", "dups_palindromes", 257, 300, 512]:
        data = _long_reads(name, 700, seed=name) if isinstance(name, int) else BY_NAME[name].fastq()
        with engine.job(min_ovlp=31 if isinstance(name, int) else BY_NAME[name].min_ovlp()) as job:
            job.feed(data)
            job.run()
            got = job.fingerprints()
        want, n, L = bind.fingerprints(data)
        assert got.size == 2 * n
        assert (got == want).all(), name


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "split_r128k", "out_of_core_r4k", "empty_input", "o_ge_L"])
def test_edge_sink_walks_output_records(engine, name):
    """emp_job_edges hands out exactly the records of output.bin, in order."""
    case = BY_NAME[name]
    a = list(case.args)
    o = dict(zip(a[::2], a[1::2]))
    with engine.job(min_ovlp=int(o.get("-o", 31)), reduce_mem=o.get("-r", "1g")) as job:
        job.feed(case.fastq())
        job.run()
        recs = job.edges()
        want = empanada_b200.decode_output(job.output())
    assert len(recs) == len(want)
    for (ov, f, t), (ov2, f2, t2) in zip(recs, want):
        assert ov == ov2 and (f == f2).all() and (t == t2).all()


@pytest.mark.gpu
@pytest.mark.parametrize("seqs", [["ACGT", "ACG"], ["ACG", "ACGTACGTACGTACGTACGT"], ["ACGTACGTACGTACGTACGTA", "ACGT"],
                                  ["ACGR", "ACGT"], ["ACGT", "AC-T"]])
def test_ragged_or_foreign_reads_are_a_format_error(engine, seqs):
    """Kept reads of unequal length, or a base outside ACGTacgt that is not
    N-class: the reference's result is undefined (it asserts equal lengths,
    fingerprint.cu:134-135), the oracle reports EMP_E_FORMAT, and so does the
    engine, which then runs the next job correctly."""
    from cases import fastq

    data = fastq(seqs)
    with pytest.raises(bind.OracleError) as o:
        bind.run(data, 1)
    assert o.value.code == bind.E_FORMAT
    with engine.job(min_ovlp=1) as job:
        job.feed(data)
        with pytest.raises(empanada_b200._native.EmpError) as e:
            job.run()
        assert e.value.code == empanada_b200._native.EMP_E_FORMAT
    data, out, st = _run(engine, BY_NAME["tiny"])
    assert hashlib.sha256(out).hexdigest() == GOLDEN["tiny"]["sha256"]
