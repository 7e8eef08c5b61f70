"""The oracle's variable-length extension (emp_oracle_run_var).

The reference asserts that all reads have one length (fingerprint.cu:134-135);
the extension defines the result for reads of unequal length: overlap lengths
ell run from the longest read's L-1 down to min_ovlp, a read-end of length len
joins the suffix and prefix tables at ell = len-1, and each round is the
reference's round on the read-ends in the tables.  Pinned here by:

* identity with the reference-pinned equal-length run on every golden case;
* an independent pure-Python model (string suffixes and prefixes, no rolling
  hashes, one search partition) on seeded variable-length read sets;
* the per-round edge sets not depending on -r (chunked sorts, merges and
  search partitions only change how records are cut);
* string-level invariants of every edge.
"""
import hashlib
import json
import os
import random
import struct
from collections import defaultdict

import pytest

from cases import BY_NAME, CASES, fastq, revcomp
from oracle import bind

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN = json.load(open(os.path.join(HERE, "golden.json")))
P1, P2 = 536870909, 536870879


def H(s: str) -> int:
    h1 = h2 = 0
    for c in s:
        e = ((ord(c) >> 1) & 3) + 1
        h1 = (h1 * 5 + e) % P1
        h2 = (h2 * 7 + e) % P2
    return (h1 << 32) | h2


def decode(out: bytes) -> list[tuple[int, list[int], list[int]]]:
    recs, pos = [], 0
    while pos < len(out):
        n, ov = struct.unpack_from("<Qi", out, pos)
        pos += 12
        frm = list(struct.unpack_from(f"<{n}I", out, pos))
        pos += 4 * n
        to = list(struct.unpack_from(f"<{n}I", out, pos))
        pos += 4 * n
        recs.append((ov, frm, to))
    return recs


def model(reads: list[str], min_ovlp: int) -> bytes:
    """The extension restated on strings, for one search partition per round
    (-r large): read-end 2i is read i, 2i+1 its reverse complement; full-length
    duplicates keep the lowest id; at each ell the live read-ends longer than
    ell are ordered by (key, id parity, id), the reference's tie order."""
    ends = []
    for s in reads:
        ends += [s, revcomp(s)]
    first = {}
    for rid in sorted(range(len(ends)), key=lambda r: (H(ends[r]), r)):
        first.setdefault(H(ends[rid]), rid)
    S, P = set(first.values()), set(first.values())
    L = max((len(s) for s in reads), default=0)
    out = bytearray()
    for ell in range(L - 1, min_ovlp - 1, -1):
        sa = [r for r in S if len(ends[r]) > ell]
        pa = [r for r in P if len(ends[r]) > ell]
        if not sa or not pa:
            continue
        sk = {r: H(ends[r][len(ends[r]) - ell:]) for r in sa}
        pk = {r: H(ends[r][:ell]) for r in pa}
        by_key = defaultdict(list)
        for r in sorted(pa, key=lambda r: (pk[r], r & 1, r)):
            by_key[pk[r]].append(r)
        frm, to = [], []
        for r in sorted(sa, key=lambda r: (sk[r], r & 1, r)):
            for q in by_key.get(sk[r], ()):
                if r // 2 != q // 2:
                    frm.append(r)
                    to.append(q)
        out += struct.pack("<Qi", len(frm), ell) + struct.pack(f"<{len(frm)}I", *frm)
        out += struct.pack(f"<{len(to)}I", *to)
        S -= set(frm)
        P -= set(to)
    return bytes(out)


def var_reads(seed: int, n: int = 160, genome: int = 1500, lens=(20, 64), dup_every: int = 0) -> list[str]:
    """Reads of random lengths sampled from one random genome, half of them
    reverse-complemented (so read-ends overlap across lengths)."""
    rng = random.Random(seed)
    g = "".join(rng.choice("ACGT") for _ in range(genome))
    out = []
    for i in range(n):
        L = rng.randint(*lens)
        p = rng.randrange(0, genome - L + 1)
        s = g[p:p + L]
        if rng.random() < 0.5:
            s = revcomp(s)
        out.append(s)
        if dup_every and i % dup_every == 0:
            out.append(s if rng.random() < 0.5 else revcomp(s))  # a duplicate read-end
    return out


@pytest.mark.parametrize("name", [c.name for c in CASES if not c.big])
def test_equal_lengths_give_the_reference_run(name):
    case = BY_NAME[name]
    data = case.fastq()
    try:
        want, st = bind.run(data, case.min_ovlp(), case.reduce_mem())
    except bind.OracleError as e:
        with pytest.raises(bind.OracleError) as got:
            bind.run(data, case.min_ovlp(), case.reduce_mem(), variable=True)
        assert got.value.code == e.code
        return
    out, st_var = bind.run(data, case.min_ovlp(), case.reduce_mem(), variable=True)
    assert hashlib.sha256(out).hexdigest() == GOLDEN[name]["sha256"]
    assert out == want and st_var == st


@pytest.mark.parametrize("seed,min_ovlp,lens,dup_every", [
    (1, 12, (20, 64), 0),
    (2, 8, (10, 40), 5),
    (3, 30, (25, 90), 0),
    (4, 5, (1, 30), 3),
    (5, 20, (60, 64), 0),
])
def test_variable_lengths_match_the_string_model(seed, min_ovlp, lens, dup_every):
    reads = var_reads(seed, lens=lens, dup_every=dup_every)
    assert len({len(s) for s in reads}) > 1
    out, st = bind.run(fastq(reads), min_ovlp, 1 << 30, variable=True)
    assert st["read_len"] == max(len(s) for s in reads)
    assert st["n_edges"] > 0
    assert out == model(reads, min_ovlp)


@pytest.mark.parametrize("seed", [6, 7, 8])
def test_variable_length_edges_do_not_depend_on_reduce_mem(seed):
    """Chunked rid sorts, merge partitions and search partitions cut the
    records differently, but each round's edges are the same pairs."""
    reads = var_reads(seed, n=400, genome=3000, lens=(30, 80))
    data = fastq(reads)

    def per_round(out):
        d = defaultdict(set)
        for ov, frm, to in decode(out):
            d[ov] |= set(zip(frm, to))
        return d

    big, _ = bind.run(data, 15, 1 << 30, variable=True)
    for rm in (16 * 64, 16 * 257, 16 * 1024):
        small, _ = bind.run(data, 15, rm, variable=True)
        assert per_round(small) == per_round(big), rm
        assert len(decode(small)) >= len(decode(big))


def test_variable_length_edge_invariants():
    reads = var_reads(9, n=300, genome=2000, lens=(15, 70), dup_every=11)
    min_ovlp = 10
    out, st = bind.run(fastq(reads), min_ovlp, 16 * 128, variable=True)
    ends = []
    for s in reads:
        ends += [s, revcomp(s)]
    srcs, dsts, last = set(), set(), None
    n_edges = 0
    for ov, frm, to in decode(out):
        assert min_ovlp <= ov <= max(len(s) for s in reads) - 1
        assert last is None or ov <= last  # ovlp_len never grows
        last = ov
        for a, b in zip(frm, to):
            assert a // 2 != b // 2
            assert len(ends[a]) > ov and len(ends[b]) > ov  # proper suffix and prefix
            assert ends[a][len(ends[a]) - ov:] == ends[b][:ov]
            assert a not in srcs and b not in dsts  # a suffix emits, and a prefix receives, in one round only
        srcs |= set(frm)
        dsts |= set(to)
        n_edges += len(frm)
    assert n_edges == st["n_edges"] > 0


def test_short_reads_never_join():
    """A read no longer than min_ovlp keeps its id but takes part in no round."""
    rng = random.Random(10)
    g = "".join(rng.choice("ACGT") for _ in range(400))
    reads = [g[i:i + 50] for i in range(0, 340, 10)] + [g[100:112], g[200:209]]
    out, st = bind.run(fastq(reads), 12, 1 << 30, variable=True)
    short = {2 * (len(reads) - 2), 2 * (len(reads) - 2) + 1, 2 * (len(reads) - 1), 2 * (len(reads) - 1) + 1}
    for _, frm, to in decode(out):
        assert not short & (set(frm) | set(to))
    assert st["n_reads"] == len(reads) and out == model(reads, 12)


def test_variable_length_errors():
    assert bind.run(fastq(["ACGTACGT", "ACG"]), 1, variable=True)[1]["read_len"] == 8
    with pytest.raises(bind.OracleError) as e:
        bind.run(fastq(["ACGT", "ACG"]), 1)
    assert e.value.code == bind.E_FORMAT
    with pytest.raises(bind.OracleError) as e:
        bind.run(fastq(["ACGR", "ACG"]), 1, variable=True)
    assert e.value.code == bind.E_FORMAT
    with pytest.raises(bind.OracleError) as e:
        bind.run(fastq(["A" * 513, "C" * 40]), 31, variable=True)
    assert e.value.code == bind.E_UNSUPPORTED
    out, st = bind.run(b"", 31, variable=True)
    assert out == b"" and st["n_reads"] == 0
