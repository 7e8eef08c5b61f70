"""Regenerate tests/golden/golden.json (and the small *.bin fixtures) by running
the reference's own sources, built as a CPU program by `make -C oracle ref-cpu`,
on every case in tests/golden/cases.py.

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py tiny small # selected cases

Each record holds the reference's output.bin digest and size; outputs up to
64 KiB are also stored verbatim as tests/golden/<case>.bin.  The CPU
restatement (oracle/) is run beside it and must agree byte for byte.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import CASES  # noqa: E402
from oracle import bind  # noqa: E402

GOLDEN = os.path.join(HERE, "golden.json")
INLINE_LIMIT = 64 * 1024


def main(names: list[str]) -> int:
    if not os.path.exists(bind.REF_CPU):
        print("oracle/_ref/empanada_ref_cpu is missing: run `make -C oracle ref-cpu` first")
        return 2
    golden = json.load(open(GOLDEN)) if os.path.exists(GOLDEN) else {}
    for case in CASES:
        if names and case.name not in names:
            continue
        data = case.fastq()
        with tempfile.TemporaryDirectory() as td:
            inp, out = os.path.join(td, "in.fq"), os.path.join(td, "out.bin")
            with open(inp, "wb") as f:
                f.write(data)
            t0 = time.time()
            ref_args = list(case.ref_args or case.args)
            p = bind.run_reference_cpu(inp, out, ref_args, cwd=td)
            dt = time.time() - t0
            rec = {"args": list(case.args), "fastq_sha256": hashlib.sha256(data).hexdigest(),
                   "fastq_size": len(data), "reference_exit": p.returncode, "reference_seconds": round(dt, 2)}
            if case.ref_args:
                rec["reference_args"] = ref_args
            if p.returncode == 0 and os.path.exists(out):
                ref = open(out, "rb").read()
                rec["sha256"] = hashlib.sha256(ref).hexdigest()
                rec["size"] = len(ref)
                try:
                    orc, st = bind.run(data, case.min_ovlp(), case.reduce_mem())
                    rec["oracle_matches"] = orc == ref
                    rec["edges"] = st["n_edges"]
                    rec["records"] = st["n_records"]
                    rec["rounds"] = st["n_rounds"]
                    rec["unique"] = st["n_unique"]
                except bind.OracleError as e:
                    rec["oracle_matches"] = False
                    rec["oracle_status"] = e.code
                path = os.path.join(HERE, f"{case.name}.bin")
                if len(ref) <= INLINE_LIMIT and not case.big:
                    with open(path, "wb") as f:
                        f.write(ref)
                    rec["inline"] = True
            golden[case.name] = rec
            print(case.name, json.dumps(rec))
    with open(GOLDEN, "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    bad = [k for k, v in golden.items() if v.get("reference_exit") == 0 and not v.get("oracle_matches")]
    if bad:
        print("oracle disagrees with the reference on:", bad)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
