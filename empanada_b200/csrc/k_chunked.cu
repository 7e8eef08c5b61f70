// k_chunked.cu -- the reference's fingerprint sort of a table larger than
// its chunk size M (-r / 16 entries), and its duplicate-removal walk.
//
// cq_sort_by_key (cqutils.cuh:180-247) sorts a table of more than M entries
// as M-entry chunks, each sorted on its own, then merged two at a time
// through a FIFO queue (the two oldest tables merge, the result joins the
// back).  cq_merge_by_key (140-177) cuts each merge into the partitions of
// cq_get_merge_partitions (37-84): a two-sided partition is the stable sort
// of [A part, B part], a one-sided one passes through.  Equal keys then end
// in the order of that merge tree rather than in input order, which decides
// the duplicate survivor and the order of edges within a record.
//
// On the device: chunk ids come from each entry's read-end rank, one stable
// sort by key and one by chunk give the sorted chunks back to back, and the
// FIFO runs over a ring of 2n entries (the queue holds n entries at every
// step, so a merge's output never overlaps a table still queued).  Each
// merge is one single-thread kernel for the partitions (a sequential walk in
// the reference too) and one kernel that places every entry at its final
// position by binary search: an A entry after the B entries with a smaller
// key in its partition, a B entry after the A entries with a key not larger.
#include "kernels.h"

namespace emp {
namespace {

EMP_DEV uint64_t ring_at(uint64_t start, uint64_t i, uint64_t C) {
    const uint64_t x = start + i;
    return x >= C ? x - C : x;
}

// first i in [lo, hi) with key(i) > x (upper) or >= x (lower), keys of the
// table that starts at ring position `start`
template <bool Upper>
EMP_DEV uint64_t ring_bound(const uint64_t *k, uint64_t C, uint64_t start, uint64_t lo, uint64_t hi, uint64_t x) {
    while (lo < hi) {
        const uint64_t m = lo + ((hi - lo) >> 1);
        const uint64_t v = k[ring_at(start, m, C)];
        if (Upper ? v <= x : v < x) lo = m + 1;
        else hi = m;
    }
    return lo;
}

// read-end id of a list value (table bit masked)
EMP_DEV uint32_t rid_of(uint32_t v) { return v & 0x7fffffffu; }

// first i in [lo, hi) with rid(lst[i]) >= x
EMP_DEV uint64_t rid_lower(const uint32_t *lst, uint64_t lo, uint64_t hi, uint32_t x) {
    while (lo < hi) {
        const uint64_t m = lo + ((hi - lo) >> 1);
        if (rid_of(lst[m]) < x) lo = m + 1;
        else hi = m;
    }
    return lo;
}

// Chunk of every entry: its read-end rank / M.  lst == nullptr: the table
// holds every read end once, in id order (the initial fingerprint table), so
// the rank is the id.  Otherwise lst is the table in list order (even ids
// ascending, then odd ids ascending) and the rank is the number of its ids
// below the entry's -- the position in the id-sorted table that the
// reference cuts into chunks (regenerate_fingerprints, overlap.cu:605-667).
__global__ void chunk_keys_kernel(const uint32_t *__restrict__ v, uint64_t n, const uint32_t *__restrict__ lst,
                                  uint64_t M, uint64_t *__restrict__ ck, uint32_t *__restrict__ ci) {
    uint64_t n_even = 0;
    if (lst) {  // the parity boundary of the list
        uint64_t lo = 0, hi = n;
        while (lo < hi) {
            const uint64_t m = lo + ((hi - lo) >> 1);
            if ((rid_of(lst[m]) & 1u) == 0) lo = m + 1;
            else hi = m;
        }
        n_even = lo;
    }
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t rid = rid_of(v[i]);
        const uint64_t rank = lst ? rid_lower(lst, 0, n_even, rid) + (rid_lower(lst, n_even, n, rid) - n_even) : rid;
        ck[i] = (rank / M) << 32;  // sort_key keeps the chunk order (chunk < 2^34)
        ci[i] = (uint32_t)i;
    }
}

__global__ void ring_gather_kernel(const uint64_t *__restrict__ k, const uint32_t *__restrict__ v,
                                   const uint32_t *__restrict__ idx, uint64_t n, uint64_t *__restrict__ rk,
                                   uint32_t *__restrict__ rv) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = idx[i];
        rk[i] = k[s];
        rv[i] = v[s];
    }
}

__global__ void ring_copy_kernel(const uint64_t *__restrict__ rk, const uint32_t *__restrict__ rv, uint64_t C,
                                 uint64_t start, uint64_t n, uint64_t *__restrict__ k, uint32_t *__restrict__ v) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t q = ring_at(start, i, C);
        k[i] = rk[q];
        v[i] = rv[q];
    }
}

// cq_get_merge_partitions (cqutils.cuh:37-84) of tables A (ring start sa, nA
// entries) and B, windows of h = M/2.  Every partition but the last takes a
// full window of A or of B, so at most nA/h + nB/h + 2 are written.
__global__ void merge_parts_kernel(const uint64_t *k, uint64_t C, uint64_t sa, uint64_t nA, uint64_t sb, uint64_t nB,
                                   uint64_t h, ChunkPart *parts, uint64_t cap, uint64_t *count, uint32_t *err) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint64_t offA = 0, offB = 0, np = 0;
    auto push = [&](uint64_t pa, uint64_t pb) {
        if (np < cap) parts[np] = ChunkPart{offA, pa, offB, pb};
        else atomicOr(err, kErrCapacity);
        ++np;
        offA += pa;
        offB += pb;
    };
    for (uint64_t guard = 0; offA < nA && offB < nB && guard <= nA + nB; ++guard) {
        uint64_t pa = nA - offA < h ? nA - offA : h, pb = nB - offB < h ? nB - offB : h;
        if (pa < h && pb < h) {  // both tails fit one window
            push(pa, pb);
            break;
        }
        const uint64_t a_last = k[ring_at(sa, offA + pa - 1, C)], b_first = k[ring_at(sb, offB, C)];
        if (a_last <= b_first) {  // all of A's window first
            push(pa, 0);
            continue;
        }
        const uint64_t b_last = k[ring_at(sb, offB + pb - 1, C)], a_first = k[ring_at(sa, offA, C)];
        if (b_last <= a_first) {  // all of B's window first
            push(0, pb);
            continue;
        }
        if (a_last < b_last) pb = ring_bound<true>(k, C, sb, offB, offB + pb, a_last) - offB;
        else if (b_last < a_last) pa = ring_bound<true>(k, C, sa, offA, offA + pa, b_last) - offA;
        push(pa, pb);
    }
    if (offA == nA && offB < nB) push(0, nB - offB);
    else if (offB == nB && offA < nA) push(nA - offA, 0);
    *count = np;
}

// Every entry of A and B at its place in the merged table (ring start so):
// within its partition, a stable sort of [A part, B part].
__global__ void merge_place_kernel(uint64_t *k, uint32_t *v, uint64_t C, uint64_t sa, uint64_t nA, uint64_t sb,
                                   uint64_t nB, uint64_t so, const ChunkPart *__restrict__ parts,
                                   const uint64_t *__restrict__ count) {
    const uint64_t np = *count;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nA + nB;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const bool isA = e < nA;
        const uint64_t i = isA ? e : e - nA;
        uint64_t lo = 0, hi = np;  // last partition starting at or before i on this side
        while (hi - lo > 1) {
            const uint64_t m = (lo + hi) >> 1;
            if ((isA ? parts[m].a0 : parts[m].b0) <= i) lo = m;
            else hi = m;
        }
        const ChunkPart p = parts[lo];
        const uint64_t src = ring_at(isA ? sa : sb, i, C);
        const uint64_t key = k[src];
        const uint32_t val = v[src];
        const uint64_t pos = isA ? p.a0 + p.b0 + (i - p.a0) + (ring_bound<false>(k, C, sb, p.b0, p.b0 + p.pb, key) - p.b0)
                                 : p.a0 + p.b0 + (i - p.b0) + (ring_bound<true>(k, C, sa, p.a0, p.a0 + p.pa, key) - p.a0);
        const uint64_t dst = ring_at(so, pos, C);
        k[dst] = key;
        v[dst] = val;
    }
}

// cq_get_partitions (cqutils.cuh:87-105) as cq_unique_by_key (272-306) walks
// it: a window of M ending inside a run of equal keys that fills it makes
// the reference's loop stop advancing.
__global__ void unique_walk_kernel(const uint64_t *__restrict__ k, uint64_t n, uint64_t M, uint32_t *err) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint64_t off = 0;
    while (n - off > M) {
        const uint64_t x = k[off + M - 1];
        uint64_t lo = off, hi = off + M;
        while (lo < hi) {
            const uint64_t m = lo + ((hi - lo) >> 1);
            if (k[m] < x) lo = m + 1;
            else hi = m;
        }
        if (lo == off) {
            atomicOr(err, kErrHang);
            return;
        }
        off = lo;
    }
}

int grid_for(uint64_t n) {
    const uint64_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

void launch_chunk_keys(const uint32_t *v, uint64_t n, const uint32_t *lst, uint64_t M, uint64_t *ck, uint32_t *ci,
                       cudaStream_t s) {
    count_launch();
    chunk_keys_kernel<<<grid_for(n), 256, 0, s>>>(v, n, lst, M, ck, ci);
}

void launch_ring_gather(const uint64_t *k, const uint32_t *v, const uint32_t *idx, uint64_t n, uint64_t *rk,
                        uint32_t *rv, cudaStream_t s) {
    count_launch();
    ring_gather_kernel<<<grid_for(n), 256, 0, s>>>(k, v, idx, n, rk, rv);
}

void launch_ring_copy(const uint64_t *rk, const uint32_t *rv, uint64_t C, uint64_t start, uint64_t n, uint64_t *k,
                      uint32_t *v, cudaStream_t s) {
    count_launch();
    ring_copy_kernel<<<grid_for(n), 256, 0, s>>>(rk, rv, C, start, n, k, v);
}

void launch_merge(uint64_t *rk, uint32_t *rv, uint64_t C, uint64_t sa, uint64_t nA, uint64_t sb, uint64_t nB,
                  uint64_t so, uint64_t h, ChunkPart *parts, uint64_t cap, uint64_t *count, uint32_t *err,
                  cudaStream_t s) {
    count_launch();
    merge_parts_kernel<<<1, 32, 0, s>>>(rk, C, sa, nA, sb, nB, h, parts, cap, count, err);
    count_launch();
    merge_place_kernel<<<grid_for(nA + nB), 256, 0, s>>>(rk, rv, C, sa, nA, sb, nB, so, parts, count);
}

void launch_unique_walk(const uint64_t *k, uint64_t n, uint64_t M, uint32_t *err, cudaStream_t s) {
    count_launch();
    unique_walk_kernel<<<1, 32, 0, s>>>(k, n, M, err);
}

}  // namespace emp
