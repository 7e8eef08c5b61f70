"""The device algorithm for a table of more than M entries (k_chunked.cu,
engine.cu chunked_sort), restated in Python, against a direct restatement of
the reference's chunked sort (cq_sort_by_key / cq_merge_by_key /
cq_get_merge_partitions, cqutils.cuh:37-84,140-247) on random tables with
many equal keys.  The device side: chunks from read-end ranks, a stable
sort by key then by chunk, the FIFO of merges over a ring of 2n entries
(checking that a merge's output never overlaps a queued table), each merge
placing A entries after the smaller B keys of their partition and B entries
after the A keys not larger.  The GPU tests check the CUDA code itself on
golden cases."""
import bisect
import random
from collections import deque


def ref_merge_parts(A, B, M):
    nA, nB, h = len(A), len(B), M // 2
    offA = offB = 0
    ps = []
    while offA < nA and offB < nB:
        pa, pb = min(nA - offA, h), min(nB - offB, h)
        if pa < h and pb < h:
            ps.append((pa, pb))
            offA += pa
            offB += pb
            break
        if A[offA + pa - 1][0] <= B[offB][0]:
            ps.append((pa, 0))
            offA += pa
        elif B[offB + pb - 1][0] <= A[offA][0]:
            ps.append((0, pb))
            offB += pb
        else:
            la, lb = A[offA + pa - 1][0], B[offB + pb - 1][0]
            if la < lb:
                pb = bisect.bisect_right([x[0] for x in B[offB:offB + pb]], la)
            elif lb < la:
                pa = bisect.bisect_right([x[0] for x in A[offA:offA + pa]], lb)
            ps.append((pa, pb))
            offA += pa
            offB += pb
    if offA == nA and offB < nB:
        ps.append((0, nB - offB))
    elif offB == nB and offA < nA:
        ps.append((nA - offA, 0))
    return ps


def ref_sort(T, M):
    if len(T) <= M:
        return sorted(T, key=lambda x: x[0])
    q = deque(sorted(T[o:o + M], key=lambda x: x[0]) for o in range(0, len(T), M))
    while len(q) > 1:
        A, B = q.popleft(), q.popleft()
        out, oa, ob = [], 0, 0
        for pa, pb in ref_merge_parts(A, B, M):
            out += sorted(A[oa:oa + pa] + B[ob:ob + pb], key=lambda x: x[0])
            oa += pa
            ob += pb
        q.append(out)
    return q[0]


def regen_order(T, M):  # id-sorted, each M-chunk: even ids then odd ids
    T = sorted(T, key=lambda x: x[1])
    out = []
    for o in range(0, len(T), M):
        c = T[o:o + M]
        out += [x for x in c if x[1] % 2 == 0] + [x for x in c if x[1] % 2 == 1]
    return out


def ring_bound(k, C, start, lo, hi, x, upper):
    while lo < hi:
        m = lo + (hi - lo) // 2
        v = k[(start + m) % C]
        if (v <= x) if upper else (v < x):
            lo = m + 1
        else:
            hi = m
    return lo


def dev_parts(k, C, sa, nA, sb, nB, h):
    offA = offB = 0
    parts = []

    def push(pa, pb):
        nonlocal offA, offB
        parts.append((offA, pa, offB, pb))
        offA += pa
        offB += pb

    while offA < nA and offB < nB:
        pa, pb = min(nA - offA, h), min(nB - offB, h)
        if pa < h and pb < h:
            push(pa, pb)
            break
        a_last, b_first = k[(sa + offA + pa - 1) % C], k[(sb + offB) % C]
        if a_last <= b_first:
            push(pa, 0)
            continue
        b_last, a_first = k[(sb + offB + pb - 1) % C], k[(sa + offA) % C]
        if b_last <= a_first:
            push(0, pb)
            continue
        if a_last < b_last:
            pb = ring_bound(k, C, sb, offB, offB + pb, a_last, True) - offB
        elif b_last < a_last:
            pa = ring_bound(k, C, sa, offA, offA + pa, b_last, True) - offA
        push(pa, pb)
    if offA == nA and offB < nB:
        push(0, nB - offB)
    elif offB == nB and offA < nA:
        push(nA - offA, 0)
    return parts


def dev_sort(lst, M, by_rank):
    n, C, h = len(lst), 2 * len(lst), M // 2
    T1 = sorted(lst, key=lambda x: x[0])
    if by_rank:
        ev = [x[1] for x in lst if x[1] % 2 == 0]
        od = [x[1] for x in lst if x[1] % 2 == 1]
        ranks = [bisect.bisect_left(ev, x[1]) + bisect.bisect_left(od, x[1]) for x in T1]
    else:
        ranks = [x[1] for x in T1]
    idx = sorted(range(n), key=lambda i: ranks[i] // M)
    k, v = [0] * C, [0] * C
    for i, s in enumerate(idx):
        k[i], v[i] = T1[s]
    q = deque((o, min(M, n - o)) for o in range(0, n, M))
    tail = n
    while len(q) > 1:
        (sa, nA), (sb, nB) = q.popleft(), q.popleft()
        parts = dev_parts(k, C, sa, nA, sb, nB, h)
        assert len(parts) <= n // max(h, 1) + 8
        writes = {}
        for e in range(nA + nB):
            isA = e < nA
            i = e if isA else e - nA
            lo, hi = 0, len(parts)
            while hi - lo > 1:
                m = (lo + hi) >> 1
                if (parts[m][0] if isA else parts[m][2]) <= i:
                    lo = m
                else:
                    hi = m
            a0, pa, b0, pb = parts[lo]
            src = ((sa if isA else sb) + i) % C
            key = k[src]
            if isA:
                pos = a0 + b0 + (i - a0) + ring_bound(k, C, sb, b0, b0 + pb, key, False) - b0
            else:
                pos = a0 + b0 + (i - b0) + ring_bound(k, C, sa, a0, a0 + pa, key, True) - a0
            dst = (tail + pos) % C
            assert dst not in writes and pos < nA + nB
            writes[dst] = (key, v[src])
        live = {(s + i) % C for s, ln in q for i in range(ln)}
        assert not live & set(writes), "a merge overwrote a queued table"
        for dst, (key, val) in writes.items():
            k[dst], v[dst] = key, val
        q.append((tail, nA + nB))
        tail = (tail + nA + nB) % C
    st = q[0][0]
    return [(k[(st + i) % C], v[(st + i) % C]) for i in range(n)]


def test_initial_table_order():
    rng = random.Random(1)
    for _ in range(150):
        n, M, kr = rng.randint(3, 260), rng.randint(2, 48), rng.randint(1, 30)
        T = [(rng.randrange(kr), i) for i in range(n)]
        want = ref_sort(T, M)
        got = dev_sort(T, M, False) if n > M else sorted(T, key=lambda x: x[0])
        assert got == want, (n, M)


def test_round_table_order():
    rng = random.Random(2)
    for _ in range(150):
        n, M, kr = rng.randint(3, 260), rng.randint(2, 48), rng.randint(1, 30)
        T = [(rng.randrange(kr), r) for r in rng.sample(range(4 * n + 10), n)]
        lst = (sorted([x for x in T if x[1] % 2 == 0], key=lambda x: x[1]) +
               sorted([x for x in T if x[1] % 2 == 1], key=lambda x: x[1]))
        want = ref_sort(regen_order(T, M), M)
        got = dev_sort(lst, M, True) if n > M else sorted(lst, key=lambda x: x[0])
        assert got == want, (n, M)
