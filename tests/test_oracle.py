"""The oracle (CPU restatement) pinned against the reference.

* known-answer tests of the hash arithmetic (assembly.cuh:29-34,
  fingerprint.cu:36-65, overlap.cu:30-39,57-91), including PrevPfx's
  wrapping 64-bit subtraction;
* every golden case: the oracle's output.bin equals the reference's own
  output (digest in golden.json, verbatim *.bin where committed);
* when the reference has been built here (oracle/_ref), fresh seeded inputs
  with random -o / -r are run through both and compared byte for byte.
"""
import hashlib
import json
import os
import random
import subprocess
import tempfile

import pytest

from cases import BY_NAME, CASES, fastq, revcomp
from oracle import bind

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN = json.load(open(os.path.join(HERE, "golden.json")))
P1, P2 = 536870909, 536870879


def H(s: str) -> int:
    enc = lambda c: ((ord(c) >> 1) & 3) + 1
    h1 = h2 = 0
    for c in s:
        h1 = (h1 * 5 + enc(c)) % P1
        h2 = (h2 * 7 + enc(c)) % P2
    return (h1 << 32) | h2


def test_known_answers():
    assert bind.hash_of("A") == (1 << 32) | 1
    assert bind.hash_of("AC") == (7 << 32) | 9
    assert bind.hash_of("ACGT") == (198 << 32) | 472
    assert bind.hash_of("acgt") == bind.hash_of("ACGT")
    inv1, inv2 = bind.radix_inv(1), bind.radix_inv(2)
    assert inv1 * 5 % P1 == 1 and inv2 * 7 % P2 == 1


def test_rolling_steps_match_direct_hashes():
    rng = random.Random(5)
    for _ in range(200):
        s = "".join(rng.choice("ACGT") for _ in range(rng.randint(2, 512)))  # 256-512: extended range
        assert bind.hash_of(s) == H(s)
        assert bind.next_sfx(H(s), s[0], len(s)) == H(s[1:])
        k = H(s)
        if (k >> 32) >= ((ord(s[-1]) >> 1) & 3) + 1 and (k & 0xFFFFFFFF) >= ((ord(s[-1]) >> 1) & 3) + 1:
            assert bind.prev_pfx(k, s[-1]) == H(s[:-1])


def test_prev_pfx_wraps_like_the_reference():
    inv1, inv2 = bind.radix_inv(1), bind.radix_inv(2)
    for f1, f2, b in [(0, 5, "A"), (1, 0, "G"), (3, 2, "T"), (0, 0, "C")]:
        e = ((ord(b) >> 1) & 3) + 1
        w1 = (inv1 * ((f1 - e) % 2**64)) % 2**64 % P1
        w2 = (inv2 * ((f2 - e) % 2**64)) % 2**64 % P2
        assert bind.prev_pfx((f1 << 32) | f2, b) == (w1 << 32) | w2


@pytest.mark.parametrize("name", [c.name for c in CASES if not c.big])
def test_oracle_matches_reference_golden(name):
    case = BY_NAME[name]
    g = GOLDEN[name]
    data = case.fastq()
    assert hashlib.sha256(data).hexdigest() == g["fastq_sha256"]
    out, st = bind.run(data, case.min_ovlp(), case.reduce_mem())
    assert hashlib.sha256(out).hexdigest() == g["sha256"]
    if g.get("inline"):
        assert out == open(os.path.join(HERE, f"{name}.bin"), "rb").read()


def test_oracle_matches_reference_golden_config1():
    case = BY_NAME["small"]
    g = GOLDEN["small"]
    out, st = bind.run(case.fastq(), 31, 1 << 30)
    assert st["n_edges"] == g["edges"] and st["n_records"] == g["records"]
    assert hashlib.sha256(out).hexdigest() == g["sha256"]


def test_oracle_errors():
    with pytest.raises(bind.OracleError) as e:
        bind.run(fastq(["ACGT", "ACG"]), 1)
    assert e.value.code == bind.E_FORMAT
    with pytest.raises(bind.OracleError) as e:
        bind.run(fastq(["ACGR", "ACGT"]), 1)
    assert e.value.code == bind.E_FORMAT
    with pytest.raises(bind.OracleError) as e:
        bind.run(fastq(["A" * 513, "C" * 513]), 31)
    assert e.value.code == bind.E_UNSUPPORTED
    with pytest.raises(bind.OracleError) as e:
        bind.run(fastq(["ACGT"]), 1, reduce_mem=16)
    assert e.value.code == bind.E_INVAL


def test_oracle_long_reads_follow_the_hash_definition():
    """Reads of 256-512 bases (beyond the reference's MAX_RD_LEN, where its
    result is undefined): the oracle's fingerprints are the exact hash of
    each read-end and its edges join exactly the overlapping read-ends."""
    rng = random.Random(23)
    for L in (256, 300, 512):
        g = "".join(rng.choice("ACGT") for _ in range(3 * L))
        reads = []
        for _ in range(12):
            p = rng.randrange(0, len(g) - L + 1)
            s = g[p:p + L]
            reads.append(revcomp(s) if rng.random() < 0.5 else s)
        data = fastq(reads)
        keys, n, LL = bind.fingerprints(data)
        assert (n, LL) == (len(reads), L)
        for i, s in enumerate(reads):
            assert int(keys[2 * i]) == H(s) and int(keys[2 * i + 1]) == H(revcomp(s))
        o = L // 2
        out, st = bind.run(data, o)
        ends = [x for s in reads for x in (s, revcomp(s))]
        got = set()
        for ov, frm, to in _records(out):
            for a, b in zip(frm, to):
                assert ends[a][L - ov:] == ends[b][:ov]  # suffix of a equals prefix of b
                got.add((int(a), int(b)))
        assert st["n_edges"] == len(got) > 0


def _records(data: bytes):
    import struct

    out, p = [], 0
    while p < len(data):
        n, ov = struct.unpack_from("<Qi", data, p)
        p += 12
        frm = struct.unpack_from(f"<{n}I", data, p)
        p += 4 * n
        to = struct.unpack_from(f"<{n}I", data, p)
        p += 4 * n
        out.append((ov, frm, to))
    return out


def test_oracle_duplicate_walk_hang():
    """A run of equal keys that fills the reference's duplicate-removal window
    (cq_get_partitions never advances): the oracle reports the hang."""
    import cases

    with pytest.raises(bind.OracleError) as e:
        bind.run(cases.edge_ooc_hang(), 20, 16 << 10)
    assert e.value.code == bind.E_HANG
    out, _ = bind.run(cases.edge_ooc_hang(), 20, 1 << 30)  # in core: no walk
    assert len(out) > 0


def _random_case(seed: int):
    """A seeded input for the reference-vs-oracle sweep: read length 1-255,
    a genome that may hold a repeat family (some copies reverse-complemented),
    substitutions and N bytes, lowercase reads, duplicated reads, palindromes,
    and -o / -r drawn so that small windows split tables and records."""
    rng = random.Random(50000 + seed)
    L = rng.choice([rng.randint(1, 40), rng.randint(20, 160), rng.randint(150, 255)])
    G = rng.randint(max(2 * L, 50), 30 * L + 100)
    g = [rng.choice("ACGT") for _ in range(G)]
    if rng.random() < 0.6 and G > 3 * L:
        rl = rng.randint(L // 2 + 1, 2 * L)
        rep = "".join(rng.choice("ACGT") for _ in range(rl))
        for _ in range(rng.randint(2, 8)):
            at = rng.randrange(0, max(1, G - rl))
            g[at:at + rl] = list(rep if rng.random() < 0.5 else revcomp(rep))
        g = g[:G]
    g = "".join(g)
    reads = []
    for _ in range(rng.randint(1, 1200)):
        p = rng.randrange(0, len(g) - L + 1)
        s = g[p:p + L]
        if rng.random() < 0.2:
            j = rng.randrange(L)
            s = s[:j] + rng.choice("ACGTNn") + s[j + 1:]
        if rng.random() < 0.05:
            s = s.lower()
        reads.append(revcomp(s) if rng.random() < 0.5 else s)
    if rng.random() < 0.3:
        for _ in range(rng.randint(1, 20)):
            reads.insert(rng.randrange(len(reads) + 1), rng.choice(reads))
    if rng.random() < 0.2 and L % 2 == 0:
        h = "".join(rng.choice("ACGT") for _ in range(L // 2))
        reads += [h + revcomp(h)] * rng.randint(1, 3)
    o = rng.randint(0, max(0, L - 1))
    r = rng.choice(["1g", "64k", "16k", "4k", "1k", str(rng.randint(8, 4096) * 16)])
    return fastq(reads), o, r


@pytest.mark.skipif(not os.path.exists(bind.REF_CPU), reason="reference not built here (needs its sources)")
@pytest.mark.parametrize("seed", range(40))
def test_oracle_matches_reference_random(seed):
    data, o, r = _random_case(seed)
    mult = {"k": 10, "m": 20, "g": 30}.get(r[-1], 0)
    rm = int(r[:-1] if mult else r) << mult
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.fq"), os.path.join(td, "out.bin")
        open(inp, "wb").write(data)
        try:
            p = bind.run_reference_cpu(inp, out, ["-o", str(o), "-r", r], cwd=td, timeout=60, threads=4)
        except subprocess.TimeoutExpired:  # the reference's endless partition walk
            with pytest.raises(bind.OracleError) as e:
                bind.run(data, o, rm)
            assert e.value.code == bind.E_HANG
            return
        if p.returncode != 0:
            pytest.skip("reference aborted on this input")
        ref = open(out, "rb").read()
    try:
        got, _ = bind.run(data, o, rm)
    except bind.OracleError as e:
        assert e.code == bind.E_HANG
        return
    assert got == ref
