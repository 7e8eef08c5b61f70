"""The autotuner's host logic (empanada_b200/tune.py) without a GPU: the
candidate space, the selection of the fastest, the output check and the
cache; and, on a GPU, that every candidate gives the reference's bytes."""
import hashlib
import json
import os

import pytest

from empanada_b200 import tune


def test_candidates_cover_the_space_default_first():
    c = tune.candidates({"a": [1, 2], "b": [7, 8, 9]})
    assert len(c) == 6 and c[0] == {"a": 1, "b": 7}
    assert {tune.label(x) for x in c} == {f"a={a},b={b}" for a in (1, 2) for b in (7, 8, 9)}


def test_select_fastest_and_ties_keep_the_earlier():
    order = ["x", "y", "z"]
    assert tune.select({"x": 3.0, "y": 1.0, "z": 2.0}, order) == "y"
    assert tune.select({"x": 1.0, "y": 1.0, "z": 2.0}, order) == "x"


def test_search_times_each_candidate_and_checks_outputs(monkeypatch):
    state = {"mean": None}
    cost = {1450: 0.003, 2175: 0.001, 2900: 0.002}
    clock = [0.0]
    monkeypatch.setattr(tune.time, "perf_counter", lambda: clock[0])

    def run():
        clock[0] += cost[state["mean"]]

    best, timings = tune.search({"bucket_mean": [2900, 2175, 1450]}, lambda c: state.update(mean=c["bucket_mean"]),
                                run, lambda: b"same bytes", repeats=2)
    assert best == {"bucket_mean": 2175}
    assert timings == pytest.approx({"bucket_mean=2900": 2.0, "bucket_mean=2175": 1.0, "bucket_mean=1450": 3.0})

    outs = iter([b"a", b"b"])
    with pytest.raises(RuntimeError, match="changed the output"):
        tune.search({"bucket_mean": [2900, 2175]}, lambda c: None, lambda: None, lambda: next(outs))


def test_cache_round_trip_and_shape_keys(tmp_path):
    p = str(tmp_path / "t" / "tune.json")
    c = tune.Cache(p)
    k = tune.shape_key("job", 33_333_333, 150)
    assert k == tune.shape_key("job", 30_000_000, 140) != tune.shape_key("job", 1_200_000, 250)
    assert c.get(k) is None
    c.put(k, {"bucket_mean": 2175}, {"bucket_mean=2175": 1.0})
    assert tune.Cache(p).get(k) == {"bucket_mean": 2175}
    assert json.load(open(p))[k]["timings_ms"] == {"bucket_mean=2175": 1.0}


def test_cache_ignores_what_it_cannot_read(tmp_path):
    """A damaged or foreign cache file means no cached choice, not an error."""
    p = tmp_path / "tune.json"
    k = tune.shape_key("job", 1_200_000, 250)
    for text in ("{not json", "[1, 2]", json.dumps({k: 3}), json.dumps({k: {"timings_ms": {}}}),
                 json.dumps({k: {"choice": [2900]}})):
        p.write_text(text)
        c = tune.Cache(str(p))
        assert c.get(k) is None, text
        c.put(k, {"bucket_mean": 2900}, {})  # and it is rewritten whole
        assert tune.Cache(str(p)).get(k) == {"bucket_mean": 2900}


def test_cached_choice_the_engine_does_not_take_is_timed_again(tmp_path):
    """A cached choice with a field this version lacks (or a value it rejects)
    is a miss: the candidates are timed and the cache entry replaced."""
    class FakeEngine:
        def __init__(self):
            self.t = {"bucket_mean": 2900, "dedup_driver": 0}

        def tuning(self):
            return dict(self.t)

        def set_tuning(self, **c):
            for k in c:
                if k not in self.t:
                    raise KeyError(k)
            self.t.update(c)

    class FakeJob:
        def run(self):
            pass

        def output(self):
            return b"same"

    c = tune.Cache(str(tmp_path / "tune.json"))
    k = tune.shape_key("job", 1000, 100)
    c.put(k, {"bucket_mean": 1450, "retired_field": 3}, {})
    eng = FakeEngine()
    res = tune.tune_job(eng, FakeJob(), 1000, 100, cache=c, space={"bucket_mean": [2175, 1450]}, repeats=1)
    assert res["source"] == "timed" and set(res["choice"]) == {"bucket_mean"}
    assert eng.t["dedup_driver"] == 0 and "retired_field" not in tune.Cache(c.path).get(k)


def test_tune_job_uses_the_cache_without_timing(tmp_path):
    class FakeEngine:
        def __init__(self):
            self.set = []

        def set_tuning(self, **kw):
            self.set.append(kw)

    c = tune.Cache(str(tmp_path / "tune.json"))
    k = tune.shape_key("job", 1000, 100)
    c.put(k, {"bucket_mean": 1450}, {})
    eng = FakeEngine()
    r = tune.tune_job(eng, job=None, reads=1000, read_len=100, cache=c)
    assert r["source"] == "cache" and eng.set == [{"bucket_mean": 1450}]


def test_env_switches(monkeypatch, tmp_path):
    monkeypatch.setenv("EMP_TUNE", "0")
    assert not tune.enabled()
    monkeypatch.setenv("EMP_TUNE", "1")
    assert tune.enabled()
    monkeypatch.setenv("EMP_TUNE_CACHE", str(tmp_path / "x.json"))
    assert tune.cache_path() == str(tmp_path / "x.json")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tiny", "sub_errors", "split_r128k", "out_of_core_r16k", "read_len_255"])
def test_every_candidate_gives_the_reference_bytes(engine, tmp_path, name):
    """The tuner times every candidate of the job space on a golden case (it
    raises if any changes the output); the chosen one gives the reference's
    bytes."""
    from cases import BY_NAME
    from test_gpu_parity import GOLDEN

    case = BY_NAME[name]
    before = engine.tuning()
    try:
        with engine.job(min_ovlp=case.min_ovlp(), reduce_mem=case.reduce_mem()) as job:
            job.feed(case.fastq())
            r = tune.tune_job(engine, job, reads=3000, read_len=100, cache=tune.Cache(str(tmp_path / "t.json")),
                              repeats=1)
            assert r["source"] == "timed" and len(r["timings_ms"]) == len(tune.candidates(tune.JOB_CANDIDATES))
            job.run()
            assert hashlib.sha256(job.output()).hexdigest() == GOLDEN[name]["sha256"]
    finally:
        engine.set_tuning(**before)
