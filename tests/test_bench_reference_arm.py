"""bench.py's reference arm on the host CPU: the reference's own CPU build (or
the oracle when that build is absent) on a bounded sample of config 1, one
JSON line with the bench contract's keys; no GPU is touched."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args):
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, stdout=subprocess.PIPE,
                       stderr=subprocess.PIPE, text=True, timeout=600, env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert p.returncode == 0, p.stderr[-2000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_reference_arm_line():
    line = _bench("--impl", "reference", "--workload", "small", "--steps", "1", "--warmup", "1")
    assert line["impl"] == "reference"
    assert line["unit"] == "reads/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["warmup"] == 1  # as asked (below 3 bench.py warns on stderr)
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "reads/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["sample_reads"] == 100_000


def test_reference_arm_has_no_batched_or_served_mode():
    for w in ("batched", "served"):
        line = _bench("--impl", "reference", "--workload", w)
        assert line["impl"] == "reference" and "batched or served" in line["unavailable"]
