"""emp_server: jobs submitted over time, batched at round granularity, each
with the bytes it gives alone (the reference's for the golden cases)."""
import hashlib
import json
import os

import pytest

import empanada_b200
from cases import BY_NAME, CASES
from empanada_b200 import _native, synth

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN = json.load(open(os.path.join(HERE, "golden.json")))
NAMES = [c.name for c in CASES if not c.big]


def _job(engine, name):
    a = list(BY_NAME[name].args)
    o = dict(zip(a[::2], a[1::2]))
    job = engine.job(min_ovlp=int(o.get("-o", 31)), map_mem=o.get("-m", "1g"), reduce_mem=o.get("-r", "1g"))
    job.feed(BY_NAME[name].fastq())
    return job


def _drain(srv, limit=100000):
    out = []
    for _ in range(limit):
        q, f, d = srv.counts()
        if q == 0 and f == 0 and d == 0:
            return out
        out += srv.step()
    raise AssertionError("server did not drain")


@pytest.mark.gpu
@pytest.mark.parametrize("rounds_per_launch,share_min", [(1, 1), (3, 1), (16, 1), (1000, 1), (1, 0), (2, 200_000)])
def test_served_golden_cases_staggered(engine, rounds_per_launch, share_min):
    """Jobs arrive while others are mid-rounds (a few submitted per step):
    every output is the reference's.  share_min = 1: every job runs
    rounds_per_launch rounds a launch; 0: every job the launch's rounds;
    200k: the larger cases a share, the smaller all their rounds at once."""
    jobs = {n: _job(engine, n) for n in NAMES}
    order = NAMES[::2] + NAMES[1::2]
    with empanada_b200.Server(engine, rounds_per_launch=rounds_per_launch, rounds_per_launch_idle=rounds_per_launch,
                              max_jobs=8, share_min_entries=share_min) as srv:
        done = []
        for k in range(0, len(order), 3):
            for n in order[k:k + 3]:
                srv.submit(jobs[n])
            done += srv.step()
        done += _drain(srv)
    assert len(done) == len(order)
    for n, j in jobs.items():
        assert j.status() == 0, n
        assert hashlib.sha256(j.output()).hexdigest() == GOLDEN[n]["sha256"], n
        j.close()


@pytest.mark.gpu
def test_served_idle_launches_run_longer(engine):
    """With no job waiting, a launch runs up to rounds_per_launch_idle rounds:
    two jobs admitted together need one launch, and their bytes do not change."""
    names = ("sub_errors", "odd_len")
    jobs = [_job(engine, n) for n in names]
    with empanada_b200.Server(engine, rounds_per_launch=2, rounds_per_launch_idle=1000) as srv:
        for j in jobs:
            srv.submit(j)
        _drain(srv)
        st = srv.stats()
    assert st["launches"] == 1 and st["batch_jobs"] == 2 and st["alone"] == 0
    for n, j in zip(names, jobs):
        assert hashlib.sha256(j.output()).hexdigest() == GOLDEN[n]["sha256"], n
        j.close()


@pytest.mark.gpu
def test_served_lone_job_in_idle_server_runs_alone(engine):
    """A job admitted alone into an idle server runs as emp_job_run runs it
    (no batched launch); a job admitted while another is in flight joins the
    batch."""
    a, b = _job(engine, "sub_errors"), _job(engine, "odd_len")
    with empanada_b200.Server(engine, rounds_per_launch=1, rounds_per_launch_idle=1, share_min_entries=1) as srv:
        srv.submit(a)
        done = srv.step()
        st = srv.stats()
        assert done == [a] and st["alone"] == 1 and st["launches"] == 0
        a2 = _job(engine, "sub_errors")
        srv.submit(a2)
        srv.submit(b)
        srv.step()  # both admitted together: they join the batch
        done = _drain(srv)
        st = srv.stats()
    assert sorted(j.handle.value for j in done) == sorted((a2.handle.value, b.handle.value))
    assert st["alone"] == 1 and st["launches"] >= 1
    for n, j in (("sub_errors", a), ("sub_errors", a2), ("odd_len", b)):
        assert j.status() == 0
        assert hashlib.sha256(j.output()).hexdigest() == GOLDEN[n]["sha256"], n
        j.close()


@pytest.mark.gpu
def test_served_batch_max_entries_sends_jobs_alone(engine):
    """With batch_max_entries below every job's list, jobs admitted together
    all run alone (no batched launch) and give the reference's bytes."""
    names = ("sub_errors", "odd_len", "tiny")
    jobs = [_job(engine, n) for n in names]
    with empanada_b200.Server(engine, batch_max_entries=1) as srv:
        for j in jobs:
            srv.submit(j)
        _drain(srv)
        st = srv.stats()
    assert st["alone"] == len(names) and st["launches"] == 0
    for n, j in zip(names, jobs):
        assert j.status() == 0
        assert hashlib.sha256(j.output()).hexdigest() == GOLDEN[n]["sha256"], n
        j.close()


@pytest.mark.gpu
@pytest.mark.parametrize("share_min", [1, 8_000_000])
def test_served_mix_equals_alone(engine, share_min):
    """Mixed read sets (20-300 kbp genomes, 100-300 bp reads) submitted in
    waves: each output equals the job run alone, whether every job runs 8
    rounds a launch or each all its rounds in the launch it joins."""
    sets = synth.batched_sets(n_sets=40, seed=12, genome_min=20_000, genome_max=300_000, len_max=300)
    data = [synth.fastq_bytes(w) for w in sets]
    alone = []
    for w, d in zip(sets, data):
        out, _ = empanada_b200.run_bytes(d, engine=engine, min_ovlp=w.min_ovlp)
        alone.append(out)
    jobs = []
    with empanada_b200.Server(engine, rounds_per_launch=8, share_min_entries=share_min) as srv:
        for k, (w, d) in enumerate(zip(sets, data)):
            j = engine.job(min_ovlp=w.min_ovlp)
            j.feed(d)
            jobs.append(j)
            srv.submit(j)
            if k % 5 == 4:
                srv.step()
        _drain(srv)
    for j, a in zip(jobs, alone):
        assert j.status() == 0
        assert j.output() == a
        j.close()


@pytest.mark.gpu
def test_served_failure_and_edge_restart(engine):
    """A failing job completes with its status; jobs whose edge buffer
    overflows run again alone; the others are unaffected."""
    import cases

    bad = engine.job(min_ovlp=20, reduce_mem="16k")
    bad.feed(cases.edge_ooc_hang())
    good = [_job(engine, n) for n in ("tiny", "sub_errors", "read_len_255")]
    with engine.tuned(edge_cap=8), empanada_b200.Server(engine, rounds_per_launch=4, share_min_entries=1) as srv:
        srv.submit(good[0])
        srv.submit(bad)
        srv.step()
        srv.submit(good[1])
        srv.submit(good[2])
        _drain(srv)
    assert bad.status() == _native.EMP_E_HANG
    with pytest.raises(_native.EmpError):
        bad.output()
    for j, n in zip(good, ("tiny", "sub_errors", "read_len_255")):
        assert j.status() == 0
        assert hashlib.sha256(j.output()).hexdigest() == GOLDEN[n]["sha256"]
    for j in good + [bad]:
        j.close()


@pytest.mark.gpu
def test_served_admission_budget(engine):
    """A budget that fits one job's estimate at a time still completes every
    job, one after another."""
    jobs = [_job(engine, n) for n in ("tiny", "odd_len", "dups_palindromes")]
    budget = max(4 * len(BY_NAME[n].fastq()) for n in ("tiny", "odd_len", "dups_palindromes")) + (64 << 20)
    with empanada_b200.Server(engine, rounds_per_launch=2, hbm_budget_bytes=budget, share_min_entries=1) as srv:
        for j in jobs:
            srv.submit(j)
        srv.step()
        q, f, _ = srv.counts()
        assert f <= 1 and q >= 1
        _drain(srv)
    for j, n in zip(jobs, ("tiny", "odd_len", "dups_palindromes")):
        assert hashlib.sha256(j.output()).hexdigest() == GOLDEN[n]["sha256"]
        j.close()


@pytest.mark.gpu
def test_served_job_is_held(engine):
    """A submitted job accepts no other call until a step hands it out; a
    server destroyed with queued jobs releases them without a result."""
    j = _job(engine, "tiny")
    srv = empanada_b200.Server(engine)
    srv.submit(j)
    with pytest.raises(_native.EmpError) as e:
        srv.submit(j)
    assert e.value.code == _native.EMP_E_STATE
    with pytest.raises(_native.EmpError) as e:
        j.run()
    assert e.value.code == _native.EMP_E_STATE
    assert engine._lib.emp_job_destroy(j.handle) == _native.EMP_E_STATE
    srv.close()
    assert j.status() == _native.EMP_E_STATE
    j.run()
    assert hashlib.sha256(j.output()).hexdigest() == GOLDEN["tiny"]["sha256"]
    j.close()


@pytest.mark.gpu
def test_trim_returns_buffers_and_job_runs_again(engine):
    """emp_job_trim drops the result and the device buffers; the job then
    takes another read set (a larger one) and gives the same bytes as a
    fresh job."""
    j = _job(engine, "tiny")
    j.run()
    first = j.output()
    j.trim()
    with pytest.raises(_native.EmpError) as e:
        j.output()
    assert e.value.code == _native.EMP_E_STATE
    other = synth.fastq_bytes(synth.batched_sets(n_sets=1, seed=13, genome_max=200_000)[0])
    j.feed(other)
    j.run()
    fresh, _ = empanada_b200.run_bytes(other, engine=engine, min_ovlp=31)
    assert j.output() == fresh
    j.trim()
    j.feed(BY_NAME["tiny"].fastq())
    j.run()
    assert j.output() == first
    j.close()


@pytest.mark.gpu
def test_feed_async_pieces(engine):
    """Asynchronous feeds (page-locked pieces, split at arbitrary bytes, mixed
    with a synchronous one) give the reference's bytes."""
    import numpy as np
    import torch

    data = BY_NAME["sub_errors"].fastq()
    host = torch.empty(len(data), dtype=torch.uint8, pin_memory=True).numpy()
    host[:] = np.frombuffer(data, dtype=np.uint8)
    a, b = len(data) // 3, 2 * len(data) // 3
    with engine.job(min_ovlp=40) as j:
        j.feed_async(host[:a], last=False)
        j.feed_async(host[a:b], last=False)
        j.feed(host[b:], last=True)
        j.run()
        assert hashlib.sha256(j.output()).hexdigest() == GOLDEN["sub_errors"]["sha256"]
        j.reset()
        j.feed_async(host[:b], last=False)
        j.feed_async(host[b:], last=True)
        j.run()
        assert hashlib.sha256(j.output()).hexdigest() == GOLDEN["sub_errors"]["sha256"]
        assert j.stats()["ms_h2d"] >= 0.0
