// coop_common.cuh -- pieces of the cooperative persistent round kernel
// (k_bucket.cu): 256-thread CTAs, two per SM, all co-resident (cooperative
// launch), bounded grid barriers, tile tickets over the tiles of many jobs.
#pragma once

#include "sort_block.cuh"

namespace emp {

constexpr int kT = kBktThreads;         // 256
constexpr int kC = kBktTile / kT;       // 8 entries per thread per prologue tile
constexpr int kTW = kT / 32;            // warps of a CTA

// L1 is not coherent across SMs: everything another CTA of this launch may
// have written (job state, lists, candidates, used marks) is read around L1,
// job state through volatile loads and bulk data through ld.global.cg.
template <class T>
EMP_DEV T vld(const T &x) {
    return *(const volatile T *)&x;
}

EMP_DEV uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier (all CTAs co-resident: cooperative launch).  Bounded wait: on
// timeout the error bit is raised and false returned; the kernel then exits.
// The arrival counter only grows (zero at launch, like the rest of the
// control block): *s_gen (shared, zero at kernel start) holds the barriers
// this CTA has passed, so barrier g is passed once the counter reaches
// (g + 1) x grid.  Arriving costs one atomic and waiting one poll loop, with
// no reset on the last arrival's path; another CTA's timeout is seen while
// polling.
EMP_DEV bool grid_barrier_raw(CoopCtl *ctl, uint32_t *s_flag, uint32_t *s_gen) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile uint32_t *count = &ctl->bar_count;
        const uint32_t g = *s_gen;
        const uint32_t target = (g + 1) * gridDim.x + ctl->bar_extra;
        const uint64_t limit = ctl->wait_ns ? ctl->wait_ns : kBarrierTimeoutNs;
        __threadfence();
        const uint32_t arrived = atomicAdd(&ctl->bar_count, 1u) + 1;
        uint32_t ok = 1;
        if (arrived < target) {
            const uint64_t t0 = globaltimer();
            uint32_t polls = 0;
            while (*count < target) {
                if ((++polls & 255) == 0 &&
                    (globaltimer() - t0 > limit || (*(volatile uint32_t *)&ctl->err & kErrSpin))) {
                    atomicOr(&ctl->err, kErrSpin);
                    ok = 0;
                    break;
                }
                __nanosleep(20);
            }
        }
        __threadfence();
        *s_gen = g + 1;
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

// profiling: stamp point p of this CTA in the probed iteration (a later tile
// of the same phase overwrites the stamps of an earlier one)
EMP_DEV void probe(const CoopCtl *ctl, uint32_t iter, int p) {
    if (threadIdx.x == 0 && ctl->probe && iter == ctl->probe_iter)
        ctl->probe[(uint64_t)blockIdx.x * kCoopProbePoints + p] = globaltimer();
}

// barrier + optional phase timestamp (ctl->trace) for profiling
EMP_DEV bool grid_barrier(CoopCtl *ctl, uint32_t *s_flag, uint32_t *s_gen, uint32_t iter, int phase) {
    const bool ok = grid_barrier_raw(ctl, s_flag, s_gen);
    if (blockIdx.x == 0 && threadIdx.x == 0 && ctl->trace && iter < ctl->trace_cap)
        ctl->trace[(uint64_t)iter * kCoopTracePhases + phase] = globaltimer();
    return ok;
}



// prefix of per-job tile counts; count(j) evaluated for every job
template <class S, class F>
EMP_DEV uint32_t build_prefix(S &sh, int J, F count) {
    // each thread takes kPer consecutive jobs (J <= kCoopMaxJobs)
    constexpr int kPer = (kCoopMaxJobs + kT - 1) / kT;
    const int j0 = kPer * threadIdx.x;
    uint32_t c[kPer], run = 0;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        c[q] = j0 + q < J ? count(j0 + q) : 0u;
        run += c[q];
    }
    uint32_t tot;
    uint32_t ex = block_exclusive_scan<kT, uint32_t>(run, sh.scan32, &tot);
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        if (j0 + q <= J) sh.pref[j0 + q] = ex;
        ex += c[q];
    }
    if (threadIdx.x == 0) sh.pref[J] = tot;
    __syncthreads();
    return tot;
}

// tile t of the prefix -> (job, local tile)
template <class S, class F>
EMP_DEV void run_tile(S &sh, int J, uint32_t t, F f) {
    int lo = 0, hi = J;
    while (hi - lo > 1) {
        const int m = (lo + hi) >> 1;
        if (sh.pref[m] <= t) lo = m;
        else hi = m;
    }
    f(lo, t - sh.pref[lo]);
}

// Tiles without an order between them: CTA i takes tile i first, then the
// rest from the ticket (offset by the grid); no ticket round trip at all
// when there are at most as many tiles as CTAs.
template <class S, class F>
EMP_DEV void tile_loop_static(S &sh, uint32_t *ticket, int J, uint32_t total, F f) {
    if (blockIdx.x < total) run_tile(sh, J, blockIdx.x, f);
    if (total <= gridDim.x) return;
    for (;;) {
        if (threadIdx.x == 0) sh.tile = gridDim.x + atomicAdd(ticket, 1u);
        __syncthreads();
        const uint32_t t = sh.tile;
        __syncthreads();
        if (t >= total) break;
        run_tile(sh, J, t, f);
    }
}

// tile_loop_static that takes its next tile before it runs the current one,
// so that the current one can start fetching the next one's data:
// f(job, local tile, the next tile's global index or ~0u).
template <class S, class F>
EMP_DEV void tile_loop_ahead(S &sh, uint32_t *ticket, int J, uint32_t total, F f) {
    if (blockIdx.x >= total) return;
    const bool more = total > gridDim.x;
    uint32_t cur = blockIdx.x;
    for (;;) {
        uint32_t nxt = ~0u;
        if (more) {
            if (threadIdx.x == 0) sh.tile = gridDim.x + atomicAdd(ticket, 1u);
            __syncthreads();
            nxt = sh.tile;
            __syncthreads();
            if (nxt >= total) nxt = ~0u;
        }
        run_tile(sh, J, cur, [&](int j, uint32_t b) { f(j, b, nxt); });
        if (nxt == ~0u) return;
        cur = nxt;
    }
}

// take tiles from the ticket until all `total` are gone; f(job, local tile)
template <class S, class F>
EMP_DEV void tile_loop(S &sh, uint32_t *ticket, int J, uint32_t total, F f) {
    for (;;) {
        if (threadIdx.x == 0) sh.tile = atomicAdd(ticket, 1u);
        __syncthreads();
        const uint32_t t = sh.tile;
        __syncthreads();
        if (t >= total) break;
        int lo = 0, hi = J;
        while (hi - lo > 1) {
            const int m = (lo + hi) >> 1;
            if (sh.pref[m] <= t) lo = m;
            else hi = m;
        }
        f(lo, t - sh.pref[lo]);
    }
}

}  // namespace emp
