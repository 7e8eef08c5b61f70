"""The exchange plan for sharding one job over several GPUs, run on gloo ranks.

One job's read-ends are owned by key range (the top bits of the key's first
residue); rows of bases are replicated.  Per round every rank applies the hash
step to the entries it owns, sends each entry to the owner of its new key
(one all-to-all), joins locally in the reference's tie order (key, id parity,
id) and drops the suffixes that emitted and the prefixes that received: every
entry with a given key is on one rank, so join and removal need nothing from
the others.  The round's record is the ranks' edges in rank order (key ranges
ascend with the rank), written when both global tables are non-empty; the
loop stops when no suffix is left anywhere (an all-reduce of the two table
sizes).  Duplicate removal before the rounds is the same exchange of the
full-length keys, keeping the lowest id of each key.

This is the plan for the tables that fit one search window (every table under
M/2 entries, 2n <= M), where the reference writes one record per round.  Its
local steps here are numpy restatements; the test checks that two and three
ranks give the oracle's output.bin byte for byte, so what a device
implementation must reproduce (ownership, exchange, tie order, record order,
termination) is pinned before one is written.
"""
import os
import random
import socket
import subprocess
import sys

import pytest

from cases import fastq, revcomp
from oracle import bind

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import datetime, struct, sys
import numpy as np
import torch
import torch.distributed as dist

P1, P2 = 536870909, 536870879
INV1, INV2 = pow(5, P1 - 2, P1), pow(7, P2 - 2, P2)
U = np.uint64
COMP = {"A": "T", "C": "G", "G": "C", "T": "A"}


def enc(c):
    return ((ord(c) >> 1) & 3) + 1


def full_key(s):
    h1 = h2 = 0
    for c in s:
        h1 = (h1 * 5 + enc(c)) % P1
        h2 = (h2 * 7 + enc(c)) % P2
    return (h1 << 32) | h2


def next_sfx(k, e, length):  # drop the first base of a suffix of `length` bases
    m1, m2 = U(pow(5, length - 1, P1)), U(pow(7, length - 1, P2))
    f1, f2 = k >> U(32), k & U(0xFFFFFFFF)
    f1 = (f1 + U(P1) - (e * m1) % U(P1)) % U(P1)
    f2 = (f2 + U(P2) - (e * m2) % U(P2)) % U(P2)
    return (f1 << U(32)) | f2


def prev_pfx(k, e):  # drop the last base of a prefix (wrapping 64-bit arithmetic)
    f1, f2 = k >> U(32), k & U(0xFFFFFFFF)
    with np.errstate(over="ignore"):
        f1 = (U(INV1) * (f1 - e)) % U(P1)
        f2 = (U(INV2) * (f2 - e)) % U(P2)
    return (f1 << U(32)) | f2


def main():
    fq, min_ovlp, out_path = sys.argv[1], int(sys.argv[2]), sys.argv[3]
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))  # a lost rank ends the others
    rank, W = dist.get_rank(), dist.get_world_size()
    lines = open(fq).read().split("\n")
    reads = [lines[i] for i in range(1, len(lines), 4) if lines[i]]
    n, L = len(reads), len(reads[0])
    ends = []
    for s in reads:
        ends += [s, "".join(COMP[c] for c in reversed(s))]
    codes = np.array([[enc(c) for c in e] for e in ends], dtype=U)  # replicated rows, read-end order

    def owner(k):
        return ((k >> U(32)) * U(W)) >> U(29)

    def exchange(k, v):
        dest = owner(k).astype(np.int64)
        o = np.argsort(dest, kind="stable")
        k, v, dest = k[o], v[o], dest[o]
        send = np.bincount(dest, minlength=W).astype(np.int64)
        recv = torch.empty(W, dtype=torch.int64)
        dist.all_to_all_single(recv, torch.from_numpy(send))
        payload = torch.from_numpy(np.stack([k.view(np.int64), v.view(np.int64)], 1).reshape(-1).copy())
        out = torch.empty(2 * int(recv.sum()), dtype=torch.int64)
        dist.all_to_all_single(out, payload, (2 * recv).tolist(), (2 * send).tolist())
        pairs = out.numpy().reshape(-1, 2)
        return pairs[:, 0].copy().view(U), pairs[:, 1].copy().view(U)

    # map phase: a contiguous slice of the reads per rank, full keys to their owners
    lo, hi = rank * n // W, (rank + 1) * n // W
    rids = np.arange(2 * lo, 2 * hi, dtype=U)
    keys = np.array([full_key(ends[int(r)]) for r in rids], dtype=U)
    keys, rids = exchange(keys, rids)
    o = np.lexsort((rids, keys))  # in-core tie order of the reference's stable sort: lowest id first
    keys, rids = keys[o], rids[o]
    first = np.ones(len(keys), bool)
    first[1:] = keys[1:] != keys[:-1]
    Sk, Sv = keys[first], rids[first]
    Pk, Pv = Sk.copy(), Sv.copy()

    out = bytearray()
    for rnd in range(L - min_ovlp):
        ell = L - 1 - rnd
        cnt = torch.tensor([len(Sk), len(Pk)], dtype=torch.int64)
        dist.all_reduce(cnt)
        if int(cnt[0]) == 0:
            break
        Sk = next_sfx(Sk, codes[Sv.astype(np.int64), L - 1 - ell], ell + 1)
        Pk = prev_pfx(Pk, codes[Pv.astype(np.int64), ell])
        Sk, Sv = exchange(Sk, Sv)
        Pk, Pv = exchange(Pk, Pv)
        o = np.lexsort((Sv, Sv & U(1), Sk))
        Sk, Sv = Sk[o], Sv[o]
        o = np.lexsort((Pv, Pv & U(1), Pk))
        Pk, Pv = Pk[o], Pv[o]
        a, b = np.searchsorted(Pk, Sk, "left"), np.searchsorted(Pk, Sk, "right")
        frm, to = [], []
        for i in range(len(Sk)):
            for j in range(a[i], b[i]):
                if Sv[i] // U(2) != Pv[j] // U(2):
                    frm.append(int(Sv[i]))
                    to.append(int(Pv[j]))
        used_s, used_p = set(frm), set(to)
        ks = np.array([int(v) not in used_s for v in Sv], bool)
        kp = np.array([int(v) not in used_p for v in Pv], bool)
        Sk, Sv, Pk, Pv = Sk[ks], Sv[ks], Pk[kp], Pv[kp]
        parts = [None] * W
        dist.all_gather_object(parts, (frm, to))
        if rank == 0 and int(cnt[0]) and int(cnt[1]):
            F = [x for f, _ in parts for x in f]
            T = [x for _, t in parts for x in t]
            out += struct.pack("<Qi", len(F), ell) + struct.pack(f"<{len(F)}I", *F) + struct.pack(f"<{len(T)}I", *T)
    if rank == 0:
        open(out_path, "wb").write(bytes(out))
    dist.destroy_process_group()


main()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_sharded(tmp_path, data: bytes, min_ovlp: int, world: int) -> bytes:
    fq = tmp_path / "in.fq"
    fq.write_bytes(data)
    out = tmp_path / f"out_{world}.bin"
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), OMP_NUM_THREADS="1")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD, str(fq), str(min_ovlp), str(out)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    try:
        for p in procs:
            _, err = p.communicate(timeout=300)
            assert p.returncode == 0, err[-2000:]
    finally:
        for p in procs:  # the exact processes started here
            if p.poll() is None:
                p.kill()
                p.wait()
    return out.read_bytes()


def reads_with_repeats(seed: int, n: int, L: int, genome: int) -> list[str]:
    """Reads of one length from a random genome that holds five copies of one
    segment, some in reverse complement (so equal keys of different read-ends
    and parities meet in a round), plus duplicated reads and a palindrome."""
    rng = random.Random(seed)
    rep = "".join(rng.choice("ACGT") for _ in range(L + L // 2))
    g = "".join(rng.choice("ACGT") for _ in range(genome))
    for c in range(5):
        at = (c + 1) * genome // 7
        g = g[:at] + (rep if c % 2 == 0 else revcomp(rep)) + g[at + len(rep):]
    out = []
    for _ in range(n):
        p = rng.randrange(0, genome - L + 1)
        s = g[p:p + L]
        out.append(revcomp(s) if rng.random() < 0.5 else s)
    h = "".join(rng.choice("ACGT") for _ in range(L // 2))
    out += [out[3]] * 3 + [revcomp(out[7])] * 2 + [h + revcomp(h)] * 2  # duplicates and a palindrome
    rng.shuffle(out)
    return out


@pytest.mark.parametrize("seed,n,L,genome,min_ovlp,world", [
    (21, 240, 40, 700, 12, 2),
    (22, 300, 56, 900, 20, 3),  # this case and the next fail with the tie order (key, id) instead
    (23, 120, 30, 600, 8, 2),
])
def test_sharded_rounds_give_the_reference_bytes(tmp_path, seed, n, L, genome, min_ovlp, world):
    data = fastq(reads_with_repeats(seed, n, L, genome))
    want, st = bind.run(data, min_ovlp, 1 << 30)
    assert st["n_edges"] > 0 and st["n_unique"] < 2 * st["n_reads"]
    assert run_sharded(tmp_path, data, min_ovlp, world) == want
