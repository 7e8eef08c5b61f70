#!/usr/bin/env python
"""Throughput of empanada's read-overlap path (fingerprint + sort + overlap) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload NAME]

Workload (default): the largest single-GPU configuration, out_of_core_hbm:
a seeded 100 Mbp genome with 5 % repeat families (1-5 kbp copies, 2-50 each,
1 % divergence), 33.3M error-free reads x 150 bp at 50x (10.5 GB of FASTQ),
-o 31 with HBM-sized blocks (-m 160g -r 160g), generated on the host by the
seeded C generator.  A step is one complete job over that read set.
--workload larger runs the 1.2M x 250 bp set (-o 75 -m 8g -r 12g -b 16m -c 64m).

impl b200 (default), one process per GPU (torchrun for N > 1; replicas only,
each rank runs its own job, no data-path collective):
  value     reads/s with the FASTQ already in HBM: device time of emp_job_run
            (CUDA events on the launching stream); the FASTQ is larger than L2
            and a 256 MB buffer is written before each step
  e2e       reads/s through the C ABI with host buffers, wall clock: read
            sets back to back on two jobs, each step issuing the next set's
            emp_job_feed_fastq_async (pinned host -> HBM on the copy engine,
            beside this step's kernels), then emp_job_run and the copy of
            output.bin to host; e2e.serial_value: feed, run and copy out one
            after another
  roofline  the dominant kernel (the cooperative kernel that runs every
            overlap round in one launch, timed with the prologue launch that
            bins a large job's first list): its algorithmic bytes per launch
            (per round 16 B gathered per entry, 16 B written per entry kept
            for the next round, 8 B per edge) / its event-timed duration,
            against the measured HBM copy bandwidth
  cpu_baseline  rank 0 at N=1: the reference's own sources built as a CPU
            program (oracle/_ref, Thrust on OpenMP) on a bounded sample at the
            workload's coverage
impl reference: that CPU build alone, timed per step on the bounded sample
(rank 0 only under torchrun).
"""
from __future__ import annotations

import argparse
import collections
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
import zlib

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "reads/s (fingerprint+sort+overlap) on 1 B200; served-mix p50/p99 latency vs plain"
CPU_SAMPLE_READS = 200_000
CPU_SAMPLE_READS_1T = 50_000  # the one-thread run of the reference CPU build


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(
        os.environ.get("WORLD_SIZE", "1"))


def reduce_max_over_ranks(x: float, dist, device) -> float:
    """The largest x over all ranks (every rank gets it); x itself without a
    process group.  Timings of replicas are combined this way: the job is as
    slow as its slowest rank."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, reads_per_rank: int, steps: int, seconds: float) -> float:
    """Whole-job reads/s of `world` replicas, each running `steps` jobs of
    `reads_per_rank` reads in `seconds` (the slowest rank's time)."""
    return world * reads_per_rank * steps / seconds


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_summary(workload_key: str, field: str = "dram_bytes_per_algorithmic_byte"):
    """DRAM (or, with field="l2_bytes_per_algorithmic_byte", L2) traffic per
    algorithmic byte of each kernel profiled on this workload, from the
    committed ncu summary (profiles/traffic.json)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        try:
            return {v["kernel"]: float(v[field]) for v in json.load(open(p)).values()
                    if v.get("workload_key") == workload_key and field in v}
        except Exception:
            return None
    return None


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(rows), "reasons": reasons}


def cpu_reference_run(fastq_path: str, args: list[str], threads: int, cwd: str):
    """One run of the reference CPU build; -> (compute seconds, wall seconds).
    compute = wall minus the reference's own read_input rows of timings.csv."""
    from oracle import bind

    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    t0 = time.perf_counter()
    p = subprocess.run([bind.REF_CPU, fastq_path, os.path.join(cwd, "out.bin")] + args, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL, env=env, cwd=cwd)
    wall = time.perf_counter() - t0
    if p.returncode != 0:
        raise RuntimeError(f"reference CPU build exited {p.returncode}")
    read_us = 0
    tpath = os.path.join(cwd, "timings.csv")
    if os.path.exists(tpath):
        for line in open(tpath):
            if line.startswith("read_input,"):
                read_us += int(line.split(",")[1])
    return max(wall - read_us / 1e6, 1e-9), wall


def cpu_baseline_block(workload, steps: int = 1):
    """Bounded sample of the workload through the reference CPU build (or the oracle port)."""
    from empanada_b200 import synth
    from oracle import bind

    sample = workload.sampled(min(CPU_SAMPLE_READS, workload.n_reads))
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        fq = os.path.join(td, "sample.fq")
        synth.write_fastq(sample, fq)
        single = None
        if os.path.exists(bind.REF_CPU):
            times = [cpu_reference_run(fq, workload.cli_args(), threads, td)[0] for _ in range(steps)]
            kind, cores = "reference", threads
            # the same build on one host thread (OMP_NUM_THREADS=1), a smaller sample
            one = workload.sampled(min(CPU_SAMPLE_READS_1T, workload.n_reads))
            fq1 = os.path.join(td, "sample1.fq")
            synth.write_fastq(one, fq1)
            t1 = cpu_reference_run(fq1, workload.cli_args(), 1, td)[0]
            single = {"value": one.n_reads / t1, "unit": "reads/s", "cores": 1, "sample": one.name}
        else:
            data = open(fq, "rb").read()
            times = []
            for _ in range(steps):
                t0 = time.perf_counter()
                bind.run(data, workload.min_ovlp, 12 << 30)
                times.append(time.perf_counter() - t0)
            kind, cores = "port", 1
    v = sample.n_reads / statistics.median(times)
    return {"value": v, "unit": "reads/s", "cores": cores, "kind": kind,
            "sample": f"{sample.name}; "
                      f"{'reference sources built with Thrust on OpenMP' if kind == 'reference' else 'oracle C port'}; "
                      f"compute time = wall minus the reference's read_input; median of {len(times)}",
            "single_thread": single}, times


def run_reference_arm(args, workload):
    rank, _, world = env_rank()
    if rank != 0:
        return
    from oracle import bind
    from empanada_b200 import synth

    sample = workload.sampled(min(CPU_SAMPLE_READS, workload.n_reads))
    threads = os.cpu_count() or 1
    times = []
    with tempfile.TemporaryDirectory() as td:
        fq = os.path.join(td, "sample.fq")
        synth.write_fastq(sample, fq)
        have_ref = os.path.exists(bind.REF_CPU)
        data = None if have_ref else open(fq, "rb").read()
        for i in range(args.warmup + args.steps):
            if have_ref:
                t = cpu_reference_run(fq, workload.cli_args(), threads, td)[0]
            else:
                t0 = time.perf_counter()
                bind.run(data, workload.min_ovlp, 12 << 30)
                t = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(t)
    total = sum(times)
    v = sample.n_reads * len(times) / total
    kind = "reference" if have_ref else "port"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "reads/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded generator empanada_b200/csrc/synth_reads.c)",
            "config": {"workload": workload.name, "sample_reads": sample.n_reads, "read_len": workload.read_len,
                       "parallelism": "host threads"},
            "cpu_baseline": {"value": v, "unit": "reads/s", "cores": threads if have_ref else 1, "kind": kind,
                             "sample": f"{sample.name}, per step"},
            "e2e": {"value": v, "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def sort_microbench(args):
    """The radix sort alone (emp_sort_pairs) on N random (fingerprint, id) pairs."""
    import numpy as np
    import torch

    import empanada_b200

    n = args.pairs
    rng = np.random.default_rng(0)
    f1 = rng.integers(0, 536870909, size=n, dtype=np.uint64)
    f2 = rng.integers(0, 536870879, size=n, dtype=np.uint64)
    keys = torch.from_numpy(((f1 << np.uint64(32)) | f2).view(np.int64)).cuda()
    vals = torch.arange(n, dtype=torch.int32).cuda()
    wk, wv = keys.clone(), vals.clone()
    eng = empanada_b200.Engine(0)
    stream = torch.cuda.current_stream()
    ms = []
    for i in range(args.warmup + args.steps):
        wk.copy_(keys)
        wv.copy_(vals)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.sort_pairs(wk.data_ptr(), wv.data_ptr(), n, stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        if i >= args.warmup:
            ms.append(e0.elapsed_time(e1))
    peak, kind = measured_peaks()
    med = statistics.median(ms)
    print(json.dumps({"kernel": "emp_sort_pairs", "pairs": n, "ms_median": med, "pairs_per_s": n / med * 1e3,
                      "bytes_per_pair_algorithmic": 12 + 8 * 24, "achieved_GBps": (12 + 8 * 24) * n / med / 1e6,
                      "peak_GBps": peak, "peak_source": kind}), flush=True)
    eng.close()


def batched_bench(args):
    """Config 4: independent read sets as one batch (emp_batch_run) per step,
    against the same sets run job by job (emp_job_run each)."""
    import numpy as np
    import torch

    import empanada_b200
    from empanada_b200 import synth

    sets = synth.batched_sets(n_sets=args.batch_sets, genome_max=args.batch_genome_max)
    sizes = [synth.fastq_size(w) for w in sets]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    t0 = time.perf_counter()
    host = torch.empty(int(offs[-1]), dtype=torch.uint8, pin_memory=True)
    host_np = host.numpy()
    for w, a, b in zip(sets, offs[:-1], offs[1:]):
        synth.fastq_into(w, host_np[a:b])
    gen_s = time.perf_counter() - t0
    reads = sum(w.n_reads for w in sets)
    device = 0
    torch.cuda.set_device(device)
    stream = torch.cuda.current_stream(device)
    sptr = stream.cuda_stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")
    eng = empanada_b200.Engine(device)
    jobs = [eng.job(min_ovlp=w.min_ovlp) for w in sets]
    for j, a, b in zip(jobs, offs[:-1], offs[1:]):
        j.reserve(int(b - a))
        j.feed(host_np[a:b], last=True)
    from empanada_b200 import tune

    tuning = {"source": "defaults", "choice": eng.tuning()}
    if not args.no_tune and tune.enabled():
        tuning = tune.tune_batch(eng, jobs, reads, int(np.median([w.read_len for w in sets])))
        tuning["choice"] = eng.tuning()

    def timed(fn, steps, warmup):
        ms = []
        for i in range(warmup + steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            if i >= warmup:
                ms.append(e0.elapsed_time(e1))
        return ms

    with ClockSampler(device) as clk:
        batch_ms = timed(lambda: eng.run_batch(jobs, sptr), args.steps, args.warmup)
    clocks = clk.summary()
    outs = [j.output() for j in jobs]
    jst = [j.stats() for j in jobs]
    launches = jst[0]["gpu_launches"]  # the first job's counter spans the whole batch
    # the batched bucket-kernel launch of the last step (every job in the batch carries its time)
    batch_kernel_ms = float(np.median([x["ms_round_kernel"] for x in jst]))
    plain_steps = max(1, min(args.steps, 3))

    def plain():
        for j in jobs:
            j.run(sptr)

    plain_ms = timed(plain, plain_steps, 1)
    same = all(j.output() == o for j, o in zip(jobs, outs))
    for j in jobs:
        j.close()
    # e2e: every set's FASTQ from pinned host memory (asynchronous copies), the batch, every output.bin back
    out_cap = max(len(o) for o in outs) + 16
    out_host = torch.empty(out_cap, dtype=torch.uint8, pin_memory=True).numpy()
    jobs = [eng.job(min_ovlp=w.min_ovlp) for w in sets]
    for j, a, b in zip(jobs, offs[:-1], offs[1:]):
        j.reserve(int(b - a))
    e2e_s = []
    d2h = 0
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        for j, a, b in zip(jobs, offs[:-1], offs[1:]):
            j.reset()
            j.feed_async(host_np[a:b], last=True)  # on the copy engine; each job's map phase waits for its own
        eng.run_batch(jobs)
        d2h = sum(j.output_into(out_host) for j in jobs)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_s.append(dt)
    for j in jobs:
        j.close()
    eng.close()
    tb = sum(batch_ms) / len(batch_ms)
    tp = sum(plain_ms) / len(plain_ms)
    line = {"metric": "reads/s, batched read sets (fingerprint+sort+overlap)", "value": reads / (tb / 1e3),
            "unit": "reads/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": tb,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded generator empanada_b200/csrc/synth_reads.c)",
            "config": {"workload": f"batched: {len(sets)} read sets, genome log-uniform 50 kbp-"
                                   f"{args.batch_genome_max // 1000} kbp, read length 100-300, coverage 10-80x, "
                                   "0.1% substitutions, -o 31",
                       "reads": reads, "fastq_bytes": int(offs[-1]),
                       "l2": "inputs larger than L2; 256 MB L2 flush before every timed step"},
            "plain": {"value": reads / (tp / 1e3), "ms_per_step": tp, "steps": plain_steps,
                      "what": "the same sets job by job (emp_job_run each), device time"},
            "batched_over_plain": tp / tb, "batch_kernel_ms": batch_kernel_ms, "outputs_identical": same, "gpu_launches": launches,
            "e2e": {"value": reads * len(e2e_s) / sum(e2e_s), "unit": "reads/s",
                    "h2d_bytes_per_step": int(offs[-1]), "d2h_bytes_per_step": int(d2h),
                    "mode": "every set's FASTQ copied in from pinned host memory with emp_job_feed_fastq_async "
                            "(the first sets' map phase runs beside the later copies), one emp_batch_run, every "
                            "output.bin copied out (wall clock)"},
            "clocks": clocks, "host_generate_s": gen_s, "tuning": tuning}
    print(json.dumps(line), flush=True)


def served_bench(args):
    """Config 5: Poisson arrivals of read-set jobs (sizes as the batched sets,
    2 % heavy jobs of a 50 Mbp genome at 30x) into an emp_server, per
    arrival rate; the same arrival stream run job by job (emp_job_run in
    arrival order) for comparison.  Latency: scheduled arrival -> output.bin
    on the host (the request's FASTQ is copied in at arrival)."""
    import numpy as np
    import torch

    import empanada_b200
    from empanada_b200 import synth

    pool = synth.batched_sets(n_sets=args.serve_pool, seed=6, genome_max=args.batch_genome_max)
    heavy = [synth.Workload(f"heavy{k}: 50 Mbp genome at 30x, {L} bp", seed=7_000 + k, genome_len=50_000_000,
                            n_reads=50_000_000 * 30 // L, read_len=L, sub_rate=0.001, min_ovlp=31)
             for k, L in enumerate((150, 250))]
    sets = pool + heavy
    sizes = [synth.fastq_size(w) for w in sets]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    t0 = time.perf_counter()
    host = torch.empty(int(offs[-1]), dtype=torch.uint8, pin_memory=True)
    host_np = host.numpy()
    for w, a, b in zip(sets, offs[:-1], offs[1:]):
        synth.fastq_into(w, host_np[a:b])
    gen_s = time.perf_counter() - t0
    device = 0
    torch.cuda.set_device(device)
    eng = empanada_b200.Engine(device)
    # each set alone: the outputs every served job must reproduce
    digests = []
    with eng.job() as j:
        for w, a, b in zip(sets, offs[:-1], offs[1:]):
            j.reset()
            j.feed(host_np[a:b], last=True)
            j.run()
            digests.append(zlib.crc32(j.output()))
    out_host = torch.empty(1 << 30, dtype=torch.uint8, pin_memory=True).numpy()
    # idle jobs hold no device memory (trimmed after each request: their
    # buffers go back to the engine's pool, which keeps them for the next)
    free_jobs = []

    def get_job(k):
        return free_jobs.pop() if free_jobs else eng.job(min_ovlp=31)

    def stream(lam, n):
        # seeded by the rate alone: both arms (and a re-run) see the same arrivals
        rng = np.random.default_rng([5, int(round(lam * 1000))])
        t = np.cumsum(rng.exponential(1.0 / lam, size=n))
        kinds = np.where(rng.random(n) < 0.02, len(pool) + rng.integers(0, len(heavy), n),
                         rng.integers(0, len(pool), n))
        return t, kinds

    def run(lam, served):
        """Requests wait on the host until they are taken: one at a time for
        the job-by-job arm, up to 64 per step for the server while its own
        queue is empty (it admitted everything submitted so far)."""
        t_arr, kinds = stream(lam, int(min(max(args.serve_min_jobs, lam * args.serve_seconds), args.serve_max_jobs)))
        n = len(t_arr)
        lat = np.zeros(n)
        ok = True
        reads = 0
        srv = (empanada_b200.Server(eng, rounds_per_launch=args.serve_rounds, rounds_per_launch_idle=args.serve_rounds_idle,
                                    hbm_budget_bytes=args.serve_budget << 30,
                                    batch_max_entries=args.serve_batch_max, share_min_entries=args.serve_share_min)
               if served else None)
        pending = collections.deque()
        held = {}
        nxt = done = 0
        t_feed = t_step = t_out = 0.0
        steps = 0
        dev_ms = dict.fromkeys(("ms_map", "ms_dedup", "ms_rounds", "ms_round_kernel", "ms_total"), 0.0)
        start = time.perf_counter()
        while done < n:
            now = time.perf_counter() - start
            while nxt < n and t_arr[nxt] <= now:
                pending.append((nxt, int(kinds[nxt])))
                nxt += 1
            fin = []
            if served:
                t1 = time.perf_counter()
                if pending and srv.counts()[0] == 0:
                    for _ in range(min(64, len(pending))):
                        i, k = pending.popleft()
                        j = get_job(k)
                        j.reset()
                        j.feed_async(host_np[offs[k]:offs[k + 1]], last=True)
                        srv.submit(j)
                        held[j.handle.value] = (i, k)
                t2 = time.perf_counter()
                if held:
                    fin = [(j,) + held.pop(j.handle.value) for j in srv.step()]
                    steps += 1
                t_feed += t2 - t1
                t_step += time.perf_counter() - t2
            elif pending:
                i, k = pending.popleft()
                t1 = time.perf_counter()
                j = get_job(k)
                j.reset()
                j.feed(host_np[offs[k]:offs[k + 1]], last=True)
                t2 = time.perf_counter()
                j.run()
                t_feed += t2 - t1
                t_step += time.perf_counter() - t2
                steps += 1
                fin = [(j, i, k)]
            if not fin and not held and not pending and nxt < n:
                time.sleep(max(0.0, min(t_arr[nxt] - (time.perf_counter() - start), 0.002)))
            t3 = time.perf_counter()
            for j, i, k in fin:
                nbytes = j.output_into(out_host) if j.status() == 0 else -1
                lat[i] = time.perf_counter() - start - t_arr[i]
                js = j.stats()
                for f in dev_ms:
                    dev_ms[f] += js[f]
                ok = ok and nbytes >= 0 and zlib.crc32(out_host[:nbytes]) == digests[k]
                reads += sets[k].n_reads
                j.trim()
                free_jobs.append(j)
                done += 1
            t_out += time.perf_counter() - t3
        span = time.perf_counter() - start
        sst = None
        if srv:
            sst = srv.stats()
            srv.close()
        return {"jobs": n, "heavy_jobs": int((kinds >= len(pool)).sum()), "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "reads_per_s": reads / span, "seconds": span, "outputs_identical": bool(ok),
                "host_s": {"feed": t_feed, "run_or_step": t_step, "output": t_out, "steps": steps},
                "job_device_ms": dev_ms,
                "server": sst}

    rates = [float(x) for x in args.serve_rates.split(",")]
    # warm-up (untimed): the engine's memory pool grows to the peak a served
    # run holds, as it would in a long-running server
    run(max(rates), True)
    with ClockSampler(device) as clk:
        served = {str(l): run(l, True) for l in rates}
        plain = {str(l): run(l, False) for l in rates}
    clocks = clk.summary()
    for j in free_jobs:
        j.close()
    eng.close()
    line = {"metric": "served: p50/p99 latency (arrival -> output.bin on host) and reads/s per arrival rate",
            "value": served[str(rates[-1])]["reads_per_s"], "unit": "reads/s", "n_gpus": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded generator empanada_b200/csrc/synth_reads.c)",
            "config": {"workload": f"served: Poisson arrivals; a pool of {len(pool)} read sets drawn as the batched "
                                   f"sets (genome 50 kbp-{args.batch_genome_max // 1000} kbp log-uniform, 100-300 bp, "
                                   "10-80x, 0.1% substitutions) plus 2% heavy jobs (50 Mbp genome at 30x, 150 or "
                                   "250 bp), -o 31; jobs per rate: rate x "
                                   f"{args.serve_seconds} s within [{args.serve_min_jobs}, {args.serve_max_jobs}]",
                       "rounds_per_launch": args.serve_rounds, "rounds_per_launch_idle": args.serve_rounds_idle,
                       "admission_budget_gib": args.serve_budget,
                       "batch_max_entries": args.serve_batch_max, "share_min_entries": args.serve_share_min,
                       "rates_per_s": rates},
            "served": served, "plain": plain, "clocks": clocks, "host_generate_s": gen_s,
            "e2e": {"value": served[str(rates[-1])]["reads_per_s"], "unit": "reads/s",
                    "what": "every request's FASTQ copied in at arrival and its output.bin copied out"}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="out_of_core_hbm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the engine's default choices (no autotuning)")
    ap.add_argument("--no-graph", action="store_true", help="skip the unitig layer's measurement")
    ap.add_argument("--reads", type=int, default=0,
                    help="run a sample of the workload at the same coverage (genome shrunk with the read count)")
    ap.add_argument("--kernel", default=None, choices=[None, "sort"],
                    help="microbenchmark one kernel instead of the whole path")
    ap.add_argument("--pairs", type=int, default=1 << 24)
    ap.add_argument("--batch-sets", type=int, default=256, help="read sets of --workload batched")
    ap.add_argument("--batch-genome-max", type=int, default=5_000_000,
                    help="largest genome of --workload batched (log-uniform from 50 kbp)")
    ap.add_argument("--serve-rates", default="1,2,5,10,20,50,100,200", help="arrival rates (jobs/s) of --workload served")
    ap.add_argument("--serve-seconds", type=float, default=4.0)
    ap.add_argument("--serve-min-jobs", type=int, default=20)
    ap.add_argument("--serve-max-jobs", type=int, default=400)
    ap.add_argument("--serve-pool", type=int, default=48)
    ap.add_argument("--serve-rounds", type=int, default=16, help="bucket-kernel rounds per launch")
    ap.add_argument("--serve-rounds-idle", type=int, default=64,
                    help="served: rounds per launch while no job waits to join")
    ap.add_argument("--serve-share-min", type=int, default=8_000_000,
                    help="served: jobs with a first list at least this long run rounds_per_launch rounds a launch, "
                         "shorter ones all their rounds (0: every job the launch's rounds)")
    ap.add_argument("--serve-batch-max", type=int, default=0,
                    help="served jobs with a longer first round list run alone (0: the bucket kernel's limit)")
    ap.add_argument("--serve-budget", type=int, default=100, help="admission budget of the server, GiB")
    args = ap.parse_args()
    if args.warmup < 3:
        print(f"bench.py: --warmup {args.warmup} is below the 3 warm-up steps a valid measurement needs",
              file=sys.stderr)
    if args.impl == "reference" and args.workload in ("served", "batched"):
        if env_rank()[0] == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference runs one read set per process and "
                              "has no batched or served mode; bench.py --impl reference times its CPU build on "
                              "the single-set workloads"}), flush=True)
        return
    if args.workload == "served":
        served_bench(args)
        return
    if args.workload == "batched":
        batched_bench(args)
        return

    from empanada_b200 import synth

    workload = synth.WORKLOADS[args.workload]
    if args.reads:
        workload = workload.sampled(args.reads)
    if args.kernel == "sort":
        sort_microbench(args)
        return
    if args.impl == "reference":
        run_reference_arm(args, workload)
        return

    import numpy as np
    import torch

    import empanada_b200
    from empanada_b200 import tune

    rank, local_rank, world = env_rank()
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = local_rank
    torch.cuda.set_device(device)

    F = synth.fastq_size(workload)
    host = torch.empty(F, dtype=torch.uint8, pin_memory=True)
    host_np = host.numpy()
    synth.fastq_into(workload, host_np)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")  # > 126 MB L2

    eng = empanada_b200.Engine(device)
    params = dict(min_ovlp=workload.min_ovlp, map_mem=workload.map_mem, reduce_mem=workload.reduce_mem,
                  base_blocksz=workload.base_blocksz, kv_chunksz=workload.kv_chunksz)
    stream = torch.cuda.current_stream(device)
    sptr = stream.cuda_stream

    def barrier():
        torch.cuda.synchronize(device)
        if dist is not None:
            dist.barrier()

    # ---- value: FASTQ resident in HBM, device time of the whole job
    job = eng.job(**params)
    job.reserve(F)
    job.feed(host_np, last=True)
    tuning = {"source": "defaults", "choice": eng.tuning()}
    if not args.no_tune and tune.enabled():  # the engine's choices for this workload (empanada_b200/tune.py)
        tuning = tune.tune_job(eng, job, workload.n_reads, workload.read_len)
        tuning["choice"] = eng.tuning()
    for _ in range(args.warmup):
        flush.zero_()
        job.run(sptr)
    barrier()
    step_ms = []
    launches = 0
    sort_ms = 0.0
    sort_elems = 0
    sort_passes = 0
    upd_ms = 0.0
    upd_bytes = 0
    upd_launches = 0
    rk_ms = 0.0
    rk_bytes = 0.0
    with ClockSampler(device) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            job.run(sptr)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            st = job.stats()
            launches += st["gpu_launches"]
            sort_ms += st["ms_sort_passes"]
            sort_elems += st["sort_pass_elems"]
            sort_passes += st["sort_passes"]
            upd_ms += st["ms_update"]
            upd_bytes += st["update_bytes"]
            upd_launches += st["update_launches"]
            rk_ms += st["ms_round_kernel"]
            rk_bytes += st["round_kernel_bytes"]
    barrier()
    clocks = clk.summary()
    total_ms = sum(step_ms)
    out_bytes = st["output_bytes"]
    total_ms = reduce_max_over_ranks(total_ms, dist, f"cuda:{device}")
    value = replica_throughput(world, workload.n_reads, args.steps, total_ms / 1000.0)
    out_bin = job.output()
    ref_crc = zlib.crc32(out_bin)  # every end-to-end step must give these bytes
    job.close()
    # ---- the unitig layer over this output.bin (device time), beside its CPU restatement
    graph = None
    if not args.no_graph:
        with empanada_b200.Graph(eng, out_bin, st["n_reads"]) as g:
            gst = g.stats()
        graph = {"ms_build": gst["ms_build"], "edges": gst["edges"], "unitigs": gst["unitigs"],
                 "long_unitigs": gst["long_unitigs"], "cycles": gst["cycles"],
                 "what": "unitigs (maximal paths of edges u->v with out-degree(u) = in-degree(v) = 1) of the "
                         "job's output.bin on the device: edge scatter, degrees, one walk per unitig head, cycles "
                         "cut at their smallest read-end, placement"}
        if rank == 0 and world == 1:
            from oracle import bind

            t0 = time.perf_counter()
            bind.unitigs(out_bin, st["n_reads"])
            graph["cpu_oracle_ms"] = 1000 * (time.perf_counter() - t0)
            graph["cpu_oracle"] = "oracle/graph_oracle.c, one host thread, serial walk"
    del out_bin

    # ---- e2e: host FASTQ in, output.bin out, through the C ABI
    out_host = torch.empty(out_bytes + 4096, dtype=torch.uint8, pin_memory=True).numpy()
    # serial: each step copies its read set in, runs, copies output.bin out
    job = eng.job(**params)
    job.reserve(F)
    e2e_s = []
    for i in range(args.warmup + args.steps):
        barrier()
        t0 = time.perf_counter()
        job.reset()
        job.feed(host_np, last=True)
        job.run()
        n_out = job.output_into(out_host)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_s.append(dt)
    job.close()
    e2e_serial = replica_throughput(world, workload.n_reads, len(e2e_s),
                                    reduce_max_over_ranks(sum(e2e_s), dist, f"cuda:{device}"))
    # pipelined: read sets back to back on two jobs; each step issues the
    # asynchronous copy of the next step's read set (the copy engine runs it
    # beside this step's kernels), runs its own, and copies its output.bin
    # out.  The K timed steps form one region with no device-wide
    # synchronisation inside it (that would finish the next set's copy
    # outside the clock): one barrier before it, one after.
    pair = [eng.job(**params), eng.job(**params)]
    for j in pair:
        j.reserve(F)

    def pipelined_step(i):
        cur, nxt = pair[i % 2], pair[(i + 1) % 2]
        if i == 0:
            cur.reset()
            cur.feed_async(host_np, last=True)
        nxt.reset()
        nxt.feed_async(host_np, last=True)
        cur.run()
        got = cur.output_into(out_host)
        if got != out_bytes:
            raise RuntimeError(f"end-to-end step {i}: {got} output bytes, the device-resident run gave {out_bytes}")
        return got

    for i in range(args.warmup):
        pipelined_step(i)
    barrier()
    t0 = time.perf_counter()
    for i in range(args.warmup, args.warmup + args.steps):
        n_out = pipelined_step(i)
    e2e_elapsed = time.perf_counter() - t0
    barrier()
    if zlib.crc32(out_host[:n_out]) != ref_crc:
        raise RuntimeError("end-to-end: output.bin differs from the device-resident run's")
    for j in pair:
        j.close()
    e2e_total = reduce_max_over_ranks(e2e_elapsed, dist, f"cuda:{device}")
    e2e_value = replica_throughput(world, workload.n_reads, args.steps, e2e_total)

    peak, peak_kind = measured_peaks()
    traffic = traffic_summary(args.workload)
    if rk_ms >= max(sort_ms, upd_ms):  # the all-rounds cooperative kernel dominates
        per_launch = rk_bytes / args.steps
        ms, nl = rk_ms, args.steps
        if os.environ.get("EMP_NO_BUCKET"):
            kname = "coop_rounds_kernel"
            what = ("all rounds, Bloom-filter driver: per round 13 B + 1/4 B per entry in, 24 B per kept entry, "
                    "72 B per candidate, 8 B per edge")
        else:
            kname = "bucket_rounds_kernel"
            what = ("all rounds in one launch (with the prologue launch of a directly binned job, timed together): "
                    "per round 16 B gathered per entry, 16 B written per entry kept for the next round, 8 B per edge")
    elif sort_ms >= upd_ms:  # the radix-sort digit pass dominates
        per_launch = 24.0 * sort_elems / max(sort_passes, 1)
        ms, nl, kname = sort_ms, sort_passes, "onesweep_kernel"
        what = "radix-sort digit pass: 24 B per pair (12 read, 12 written)"
    else:  # the per-round table update of the pipeline dominates
        per_launch = upd_bytes / max(upd_launches, 1)
        ms, nl, kname = upd_ms, upd_launches, "pl_update_filter_kernel"
        what = "round update: 13 B read + 1/4 B of bases per entry in, 12 B written per entry out"
    achieved = per_launch * nl / (ms / 1000.0) / 1e9 if ms > 0 else 0.0
    tb = traffic.get(kname) if traffic else None
    l2_tb = (traffic_summary(args.workload, "l2_bytes_per_algorithmic_byte") or {}).get(kname)
    l2 = None
    if l2_tb and ms > 0:  # the lists stay in L2 here: L2 bytes (ncu) / time against the measured L2 read rate
        l2_peak = empanada_b200.measure_l2_read(64 << 20, device)
        l2_ach = l2_tb * per_launch * nl / (ms / 1000.0) / 1e9
        l2 = {"achieved": l2_ach, "peak": l2_peak, "unit": "GB/s", "frac": l2_ach / l2_peak if l2_peak else None,
              "traffic": l2_tb * per_launch,
              "peak_source": "measured live: emp_measure_l2_read, a 64 MiB buffer read 20 times from L2"}
    roofline = {"bound": "hbm", "kernel": kname, "algorithmic": what, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": f"{peak_kind} (HBM copy, burst)",
                "traffic": (tb * per_launch) if tb else None, "algorithmic_bytes_per_launch": per_launch,
                "avg_launch_us": 1000.0 * ms / max(nl, 1), "launches": nl,
                "l2": l2, "round_kernel_ms_per_step": rk_ms / args.steps,
                "sort_pass_ms_per_step": sort_ms / args.steps, "update_ms_per_step": upd_ms / args.steps}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu, _ = cpu_baseline_block(workload, steps=1)
        except Exception as e:  # reported, never fatal
            cpu = {"value": None, "unit": "reads/s", "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "reads/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u64",
                "data": "synthetic (seeded generator empanada_b200/csrc/synth_reads.c)",
                "config": {"workload": workload.name, "reads": workload.n_reads, "read_len": workload.read_len,
                           "fastq_bytes": F, "options": " ".join(workload.cli_args()),
                           "l2": "input (FASTQ) larger than L2; 256 MB L2 flush before every timed step",
                           "parallelism": f"replicas x{world}"},
                "bases_per_s": value * workload.read_len,
                "e2e": {"value": e2e_value, "unit": "reads/s", "h2d_bytes_per_step": F, "d2h_bytes_per_step": n_out,
                        "mode": "read sets back to back through the C ABI from pinned host memory: each step issues "
                                "the next set's asynchronous FASTQ copy, runs its own set and copies its output.bin "
                                "out (wall clock)",
                        "serial_value": e2e_serial},
                "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clocks,
                "tuning": tuning, "graph": graph,
                "job": {k: st[k] for k in ("n_reads", "n_unique", "n_edges", "n_records", "n_rounds", "ms_map",
                                           "ms_dedup", "ms_rounds")},
                "live_entries": int(sum(st["sfx_live"]) + sum(st["pfx_live"]))}
        print(json.dumps(line), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
