"""Autotuner of the engine's choices (``emp_tuning``).

Every choice gives the same ``output.bin`` (the tuner checks that it does on
the workload it times); they differ in speed:

``bucket_mean``  entries per key bucket of the round kernel: its tile size.
                 Smaller buckets give more of them per round (better balance
                 across the SMs, more buckets in flight), larger ones fewer
                 per-bucket fixed costs.
``map_streams``  streams a batch's map phase spreads its jobs over (batches
                 only): more streams run more small jobs' kernels side by
                 side, at more launch and synchronisation overhead.
``dedup_driver`` duplicate removal by key buckets and hash sets (0) or by
                 sorting every fingerprint (1).

The tuner times each candidate on the caller's own workload (a fed job, or a
list of fed jobs for a batch), keeps the fastest and records it in a JSON
cache keyed by the workload's shape (kind, read count to a power of two,
read length to 50 bases), so that later runs of the same shape reuse the
choice without timing.  ``EMP_TUNE_CACHE`` names the cache file (default
``~/.cache/empanada_b200/tune.json``); ``EMP_TUNE=0`` turns the tuner off
(the defaults stay).
"""
from __future__ import annotations

import json
import math
import os
import time
import zlib
from typing import Callable, Iterable

from . import _native

# the defaults first: they win ties
JOB_CANDIDATES = {"bucket_mean": [2900, 2175, 1450], "dedup_driver": [0, 1]}
BATCH_CANDIDATES = {"bucket_mean": [2900, 2175, 1450], "map_streams": [8, 16, 32, 4]}


def enabled() -> bool:
    return os.environ.get("EMP_TUNE", "1") != "0"


def cache_path() -> str:
    return os.environ.get("EMP_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "empanada_b200",
                                                            "tune.json")


def shape_key(kind: str, reads: int, read_len: int) -> str:
    """The workload shape a choice is cached under."""
    r = max(1, int(reads))
    return f"{kind}:reads~2^{round(math.log2(r))}:L~{max(50, (int(read_len) + 25) // 50 * 50)}"


class Cache:
    """Choices per workload shape, in a JSON file."""

    def __init__(self, path: str | None = None):
        self.path = path or cache_path()
        self.data: dict = {}
        if os.path.exists(self.path):
            try:
                with open(self.path) as f:
                    data = json.load(f)
                self.data = data if isinstance(data, dict) else {}
            except (OSError, ValueError):
                self.data = {}

    def get(self, key: str) -> dict | None:
        """The cached choice, or None (also for an entry this version cannot read)."""
        e = self.data.get(key)
        if not isinstance(e, dict) or not isinstance(e.get("choice"), dict):
            return None
        return dict(e["choice"])

    def put(self, key: str, choice: dict, timings: dict) -> None:
        self.data[key] = {"choice": choice, "timings_ms": timings}
        os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def candidates(space: dict) -> list[dict]:
    """Every combination of the space's values (the first value of each
    field first), as a list of partial tunings."""
    out = [{}]
    for field, values in space.items():
        out = [dict(c, **{field: v}) for c in out for v in values]
    return out


def label(choice: dict) -> str:
    return ",".join(f"{k}={v}" for k, v in sorted(choice.items()))


def select(timings: dict[str, float], order: list[str]) -> str:
    """The fastest candidate; among equal times the earlier one in `order`."""
    return min(order, key=lambda lab: (timings[lab], order.index(lab)))


def search(space: dict, apply: Callable[[dict], None], run: Callable[[], None], output: Callable[[], bytes],
           repeats: int = 2) -> tuple[dict, dict]:
    """Time run() under every candidate of `space` (best of `repeats`, after
    one untimed run whose output() is checked: every candidate must give the
    same bytes).  Returns (best choice, {label: ms})."""
    cands = candidates(space)
    timings: dict[str, float] = {}
    digest = None
    for c in cands:
        apply(c)
        run()  # untimed: warms the candidate (allocations, first launches)
        d = zlib.crc32(output())
        if digest is None:
            digest = d
        elif d != digest:
            raise RuntimeError(f"tuning candidate {label(c)} changed the output")
        best = math.inf
        for _ in range(repeats):
            t0 = time.perf_counter()
            run()
            best = min(best, time.perf_counter() - t0)
        timings[label(c)] = 1000.0 * best
    order = [label(c) for c in cands]
    lab = select(timings, order)
    return cands[order.index(lab)], timings


def _apply_cached(engine, choice: dict) -> bool:
    """Apply a cached choice; False (nothing changed) when the engine does not
    take it: a field this version does not have, or a value it rejects."""
    before = engine.tuning() if hasattr(engine, "tuning") else None
    try:
        engine.set_tuning(**choice)
        return True
    except (KeyError, TypeError, ValueError, _native.EmpError):
        if before is not None:
            engine.set_tuning(**before)
        return False


def tune_job(engine, job, reads: int, read_len: int, cache: Cache | None = None, space: dict | None = None,
             repeats: int = 2) -> dict:
    """Choose the engine's tuning for runs like `job` (fed, not yet run):
    from the cache when the shape is known, else by timing every candidate
    on the job itself.  Applies the choice to the engine and returns
    {"choice", "source", "timings_ms"}."""
    key = shape_key("job", reads, read_len)
    cache = cache if cache is not None else Cache()
    hit = cache.get(key)
    if hit is not None and _apply_cached(engine, hit):
        return {"key": key, "choice": hit, "source": "cache", "timings_ms": None}

    best, timings = search(space or JOB_CANDIDATES, lambda c: engine.set_tuning(**c), job.run, job.output, repeats)
    engine.set_tuning(**best)
    cache.put(key, best, timings)
    return {"key": key, "choice": best, "source": "timed", "timings_ms": timings}


def tune_batch(engine, jobs: Iterable, reads: int, read_len: int, cache: Cache | None = None,
               space: dict | None = None, repeats: int = 1) -> dict:
    """tune_job for a batch: the candidates are timed on engine.run_batch(jobs)."""
    jobs = list(jobs)
    key = shape_key(f"batch{len(jobs)}", reads, read_len)
    cache = cache if cache is not None else Cache()
    hit = cache.get(key)
    if hit is not None and _apply_cached(engine, hit):
        return {"key": key, "choice": hit, "source": "cache", "timings_ms": None}

    def outputs() -> bytes:
        crcs = [zlib.crc32(j.output()) for j in jobs]
        return json.dumps(crcs).encode()

    best, timings = search(space or BATCH_CANDIDATES, lambda c: engine.set_tuning(**c),
                           lambda: engine.run_batch(jobs), outputs, repeats)
    engine.set_tuning(**best)
    cache.put(key, best, timings)
    return {"key": key, "choice": best, "source": "timed", "timings_ms": timings}
