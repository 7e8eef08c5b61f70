"""emp_batch_run: every job of a batch gives the bytes it gives alone.

The golden cases (reference digests) run as one batch, including jobs with
no reads or no rounds and out-of-core ones (2n > M); a failing job leaves
the others their results; synthetic read
sets of the batched workload's kind (mixed genome sizes, read lengths and
coverages) are compared with their own emp_job_run outputs.
"""
import hashlib
import json
import os

import pytest

import empanada_b200
from cases import BY_NAME, CASES
from empanada_b200 import _native, synth

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN = json.load(open(os.path.join(HERE, "golden.json")))

BATCH_CASES = [c.name for c in CASES if not c.big] + ["small"]


def _job(engine, case):
    a = list(case.args)
    o = dict(zip(a[::2], a[1::2]))
    job = engine.job(min_ovlp=int(o.get("-o", 31)), map_mem=o.get("-m", "1g"), reduce_mem=o.get("-r", "1g"),
                     base_blocksz=o.get("-b", "32m"), kv_chunksz=o.get("-c", "64m"))
    job.feed(case.fastq())
    return job


def _digest(job):
    return hashlib.sha256(job.output()).hexdigest()


@pytest.mark.gpu
def test_batch_of_golden_cases_matches_reference(engine):
    jobs = [_job(engine, BY_NAME[n]) for n in BATCH_CASES]
    try:
        engine.run_batch(jobs)
        for name, job in zip(BATCH_CASES, jobs):
            g = GOLDEN[name]
            assert _digest(job) == g["sha256"], name
            st = job.stats()
            if "edges" in g:
                assert st["n_edges"] == g["edges"], name
    finally:
        for j in jobs:
            j.close()


@pytest.mark.gpu
def test_batch_failure_leaves_other_jobs(engine):
    """A job that fails (here: input on which the reference never
    terminates) fails alone: the batch returns its status and the other jobs
    have their results."""
    import cases

    jobs = [_job(engine, BY_NAME["tiny"]), engine.job(min_ovlp=20, reduce_mem="16k"),
            _job(engine, BY_NAME["sub_errors"])]
    jobs[1].feed(cases.edge_ooc_hang())
    try:
        with pytest.raises(_native.EmpError) as ei:
            engine.run_batch(jobs)
        assert ei.value.code == _native.EMP_E_HANG
        assert _digest(jobs[0]) == GOLDEN["tiny"]["sha256"]
        assert _digest(jobs[2]) == GOLDEN["sub_errors"]["sha256"]
        with pytest.raises(_native.EmpError):
            jobs[1].output()
    finally:
        for j in jobs:
            j.close()


@pytest.mark.gpu
def test_batch_edge_restart(engine):
    """Edge buffers too small for every job: each runs again alone."""
    names = ["tiny", "sub_errors", "dups_palindromes", "read_len_255"]
    jobs = [_job(engine, BY_NAME[n]) for n in names]
    try:
        with engine.tuned(edge_cap=8):
            engine.run_batch(jobs)
        for name, job in zip(names, jobs):
            assert _digest(job) == GOLDEN[name]["sha256"], name
    finally:
        for j in jobs:
            j.close()


@pytest.mark.gpu
def test_batch_reuse_and_repeat(engine):
    """The same jobs run twice as a batch, then alone: identical bytes."""
    names = ["tiny", "odd_len", "read_len_1", "split_r128k"]
    jobs = [_job(engine, BY_NAME[n]) for n in names]
    try:
        engine.run_batch(jobs)
        first = [j.output() for j in jobs]
        engine.run_batch(jobs[::-1])
        assert [j.output() for j in jobs] == first
        for j, f in zip(jobs, first):
            j.run()
            assert j.output() == f
    finally:
        for j in jobs:
            j.close()


@pytest.mark.gpu
def test_batch_of_synthetic_sets_matches_single_runs(engine):
    """64 read sets of mixed genome size (20-300 kbp), read length (100-300)
    and coverage (10-80x) with 0.1 % substitutions, as one batch and one by
    one; two of them also against the oracle."""
    sets = synth.batched_sets(n_sets=64, seed=11, genome_min=20_000, genome_max=300_000, len_max=300)
    jobs = []
    try:
        for w in sets:
            j = engine.job(min_ovlp=w.min_ovlp)
            j.feed(synth.fastq_bytes(w))
            jobs.append(j)
        engine.run_batch(jobs)
        got = [j.output() for j in jobs]
        for w, j, g in zip(sets, jobs, got):
            j.run()
            assert j.output() == g, w.name
        from oracle import bind

        small = sorted(range(len(sets)), key=lambda k: sets[k].n_reads)[:2]
        for k in small:
            ref, _ = bind.run(synth.fastq_bytes(sets[k]), sets[k].min_ovlp)
            assert got[k] == ref, sets[k].name
    finally:
        for j in jobs:
            j.close()


@pytest.mark.gpu
def test_batch_rejects_bad_arguments(engine):
    with engine.job() as a:
        arr = (_native.ctypes.c_void_p * 2)(a.handle, a.handle)
        assert engine._lib.emp_batch_run(engine.handle, arr, 2, None) == _native.EMP_E_INVAL
        assert engine._lib.emp_batch_run(engine.handle, None, 1, None) == _native.EMP_E_INVAL
        assert engine._lib.emp_batch_run(engine.handle, None, 0, None) == _native.EMP_OK
