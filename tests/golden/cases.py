"""Input cases for the golden output.bin fixtures and the parity tests.

Each case is a FASTQ byte string plus the reference command-line options.
Synthetic workloads come from the seeded C generator (empanada_b200.synth);
edge cases are built here with a local seeded PRNG so they need nothing but
Python.
"""
from __future__ import annotations

import dataclasses
import random

COMP = {"A": "T", "C": "G", "G": "C", "T": "A", "a": "t", "c": "g", "g": "c", "t": "a", "N": "N", "n": "n"}


def revcomp(s: str) -> str:
    return "".join(COMP[c] for c in reversed(s))


def fastq(seqs, quals=None, trailing_newline=True) -> bytes:
    out = []
    for i, s in enumerate(seqs):
        q = quals[i] if quals else "I" * len(s)
        out.append(f"@r{i}\n{s}\n+\n{q}\n")
    data = "".join(out)
    if not trailing_newline:
        data = data[:-1]
    return data.encode()


def _genome(rng: random.Random, g: int) -> str:
    return "".join(rng.choice("ACGT") for _ in range(g))


def _reads(rng: random.Random, genome: str, n: int, L: int, sub: float = 0.0) -> list[str]:
    out = []
    for _ in range(n):
        p = rng.randrange(0, len(genome) - L + 1)
        s = list(genome[p:p + L])
        if sub:
            for j in range(L):
                if rng.random() < sub:
                    s[j] = rng.choice([b for b in "ACGT" if b != s[j]])
        s = "".join(s)
        if rng.random() < 0.5:
            s = revcomp(s)
        out.append(s)
    return out


def edge_n_reads() -> bytes:
    rng = random.Random(11)
    reads = _reads(rng, _genome(rng, 5000), 300, 60)
    for i in range(0, len(reads), 7):
        j = rng.randrange(60)
        reads[i] = reads[i][:j] + rng.choice("Nn") + reads[i][j + 1:]
    return fastq(reads)


def edge_lowercase() -> bytes:
    rng = random.Random(12)
    reads = _reads(rng, _genome(rng, 4000), 300, 50)
    for i in range(len(reads)):
        if i % 3 == 0:
            reads[i] = reads[i].lower()
        elif i % 3 == 1:
            reads[i] = "".join(c.lower() if rng.random() < 0.3 else c for c in reads[i])
    return fastq(reads)


def edge_no_trailing_newline() -> bytes:
    rng = random.Random(13)
    return fastq(_reads(rng, _genome(rng, 3000), 200, 40), trailing_newline=False)


def edge_dups_palindromes() -> bytes:
    rng = random.Random(14)
    g = _genome(rng, 3000)
    reads = _reads(rng, g, 150, 48)
    pal = []
    for _ in range(6):
        h = "".join(rng.choice("ACGT") for _ in range(24))
        pal.append(h + revcomp(h))  # its own reverse complement
    dups = [reads[3]] * 4 + [revcomp(reads[5])] * 3 + pal + pal[:2]
    out = reads[:]
    for k, d in enumerate(dups):
        out.insert((k * 17) % len(out), d)
    return fastq(out)


def edge_empty_seq_lines() -> bytes:
    rng = random.Random(15)
    reads = _reads(rng, _genome(rng, 3000), 120, 45)
    data = fastq(reads).decode().split("\n")
    for rec in (3, 40, 77):
        data[4 * rec + 1] = ""
        data[4 * rec + 3] = ""
    return "\n".join(data).encode()


def edge_header_only_tail() -> bytes:
    rng = random.Random(16)
    return fastq(_reads(rng, _genome(rng, 3000), 100, 44)) + b"@tail_without_sequence\n"


def edge_seq_line_unterminated() -> bytes:
    rng = random.Random(17)
    return fastq(_reads(rng, _genome(rng, 3000), 100, 44)) + b"@last\n" + _reads(rng, _genome(rng, 100), 1, 44)[0].encode()


def edge_empty() -> bytes:
    return b""


def edge_L1() -> bytes:
    rng = random.Random(18)
    return fastq([rng.choice("ACGT") for _ in range(20)])


def edge_L255() -> bytes:
    rng = random.Random(19)
    return fastq(_reads(rng, _genome(rng, 20000), 400, 255, sub=0.001))


def edge_sub_errors() -> bytes:
    rng = random.Random(20)
    return fastq(_reads(rng, _genome(rng, 15000), 2000, 120, sub=0.01))


def edge_ooc_dups() -> bytes:
    """Duplicated and reverse-complemented reads spread over the file, so equal
    fingerprints fall into different M-chunks of the reference's sort."""
    rng = random.Random(21)
    g = _genome(rng, 6000)
    reads = _reads(rng, g, 1500, 64, sub=0.002)
    out = reads[:]
    for k in range(400):
        d = reads[rng.randrange(len(reads))]
        out.insert(rng.randrange(len(out) + 1), revcomp(d) if k % 3 == 0 else d)
    return fastq(out)


def edge_ooc_hang() -> bytes:
    """1100 copies of one read among others: with -r 16k (M = 1024) the
    reference's duplicate-removal partition walk meets a run of 1100 equal
    keys that fills its window and stops advancing."""
    rng = random.Random(22)
    g = _genome(rng, 4000)
    reads = _reads(rng, g, 300, 50)
    out = reads + [reads[7]] * 1100
    rng.shuffle(out)
    return fastq(out)


@dataclasses.dataclass(frozen=True)
class Case:
    name: str
    args: tuple = ()            # reference CLI options
    edge: str | None = None     # name of an edge_* builder
    synth: dict | None = None   # empanada_b200.synth.Workload fields
    big: bool = False           # digest only (output too large to commit)
    # options the reference itself is run with when they must differ from
    # `args` (same output by construction; the reason is given at the case)
    ref_args: tuple | None = None

    def min_ovlp(self) -> int:
        a = list(self.args)
        return int(a[a.index("-o") + 1]) if "-o" in a else 31

    def reduce_mem(self) -> int:
        a = list(self.args)
        if "-r" not in a:
            return 1 << 30
        s = a[a.index("-r") + 1]
        mult = {"k": 10, "m": 20, "g": 30}.get(s[-1].lower(), 0)
        return int(s[:-1] if mult else s) << mult

    def fastq(self) -> bytes:
        if self.edge:
            return globals()[f"edge_{self.edge}"]()
        from empanada_b200 import synth
        w = dataclasses.replace(synth.SMALL, **self.synth)
        return synth.fastq_bytes(w)


TINY = {"seed": 101, "genome_len": 50_000, "n_reads": 3000, "read_len": 100}
CONFIG3_TENTH = {"seed": 3, "genome_len": 10_000_000, "n_reads": 3_333_333, "read_len": 150, "repeat_frac": 0.05,
                 "rep_min_len": 1000, "rep_max_len": 5000, "rep_min_copies": 2, "rep_max_copies": 50,
                 "rep_divergence": 0.01}
CONFIG3 = {"seed": 3, "genome_len": 100_000_000, "n_reads": 33_333_333, "read_len": 150, "repeat_frac": 0.05,
           "rep_min_len": 1000, "rep_max_len": 5000, "rep_min_copies": 2, "rep_max_copies": 50,
           "rep_divergence": 0.01}
CASES = [
    Case("tiny", ("-o", "31"), synth=TINY),
    Case("tiny_m16k_b1k", ("-o", "31", "-m", "16k", "-b", "1k", "-c", "1k"), synth=TINY),
    Case("odd_len", ("-o", "20"), synth={"seed": 102, "genome_len": 20_000, "n_reads": 2000, "read_len": 77,
                                         "sub_rate": 0.002}),
    Case("n_reads", ("-o", "21"), edge="n_reads"),
    Case("lowercase", ("-o", "15"), edge="lowercase"),
    Case("no_trailing_newline", ("-o", "11"), edge="no_trailing_newline"),
    Case("dups_palindromes", ("-o", "12"), edge="dups_palindromes"),
    Case("empty_seq_lines", ("-o", "13"), edge="empty_seq_lines"),
    Case("header_only_tail", ("-o", "13"), edge="header_only_tail"),
    Case("seq_line_unterminated", ("-o", "13"), edge="seq_line_unterminated"),
    Case("empty_input", ("-o", "31"), edge="empty"),
    Case("read_len_1", ("-o", "0"), edge="L1"),
    Case("read_len_255", ("-o", "120"), edge="L255"),
    Case("sub_errors", ("-o", "40"), edge="sub_errors"),
    Case("o_ge_L", ("-o", "100"), edge="lowercase"),
    Case("split_r128k", ("-o", "31", "-r", "128k"), synth=TINY),
    Case("out_of_core_r16k", ("-o", "31", "-r", "16k"), synth=TINY),
    Case("out_of_core_r4k", ("-o", "31", "-r", "4k"), synth=TINY),
    Case("out_of_core_r1k_odd", ("-o", "27", "-r", "1040"), synth={"seed": 103, "genome_len": 8_000,
                                                                    "n_reads": 700, "read_len": 60,
                                                                    "sub_rate": 0.002}),
    Case("out_of_core_dups_r16k", ("-o", "20", "-r", "16k"), edge="ooc_dups"),
    Case("out_of_core_repeats_r32k", ("-o", "25", "-r", "32k"),
         synth={"seed": 104, "genome_len": 60_000, "n_reads": 5000, "read_len": 90, "sub_rate": 0.001,
                "repeat_frac": 0.2, "rep_min_len": 300, "rep_max_len": 900, "rep_min_copies": 2,
                "rep_max_copies": 12, "rep_divergence": 0.002}),
    # config 3 at a tenth of its size: 10 Mbp genome, 5 % repeat families
    # (1-5 kbp copies, 2-50 each, 1 % divergence), 150 bp reads at 50x;
    # at -r 100m (M = 6.55M < 2n) the fingerprint sort goes out of core
    Case("repeats_10m_r100m", ("-o", "31", "-r", "100m"), synth=CONFIG3_TENTH, big=True),
    Case("repeats_10m", ("-o", "31"), synth=CONFIG3_TENTH, big=True),
    # config 3 at full size: 100 Mbp genome with 5 % repeat families, 33.3M
    # x 150 bp reads (10.5 GB FASTQ).  At -m 1g -r 1g the reference streams
    # 64 MiB blocks and M = 64Mi pairs < 2n, so its fingerprint sort is
    # chunked and the first rounds split into records of M/2 windows.
    Case("config3_r1g", ("-o", "31", "-m", "1g", "-r", "1g"), synth=CONFIG3, big=True),
    # HBM-sized: every table fits one chunk (2n <= M) and every round table
    # fits one search window (|table| <= M/2), so the output is the same for
    # every -r of at least 4g and any -m.  The reference's host build is run
    # at -m 1g -r 4g: at -r 160g its match buffer (13 B x M = 130 GB,
    # overlap.cu:120) exceeds host memory, and at -m 160g one 10 GB block
    # overflows its int offsets (preprocess.cu:98-182).
    Case("config3_hbm", ("-o", "31", "-m", "160g", "-r", "160g"), synth=CONFIG3, big=True,
         ref_args=("-o", "31", "-m", "1g", "-r", "4g")),
    Case("small", ("-o", "31"), synth={}, big=True),
    Case("larger", ("-o", "75", "-m", "8g", "-r", "12g", "-b", "16m", "-c", "64m"),
         synth={"seed": 2, "genome_len": 5_000_000, "n_reads": 1_200_000, "read_len": 250, "sub_rate": 0.001},
         big=True),
]
BY_NAME = {c.name: c for c in CASES}
