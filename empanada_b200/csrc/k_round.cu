// k_round.cu -- duplicate removal and the per-round overlap kernels.
//
// Table representation.  Each table (suffixes, prefixes) is kept as a list
// of (key, value) pairs in read-end-id order -- even ids ascending, then odd
// ids ascending -- which is exactly the order the reference's
// regenerate_fingerprints hands to the next fingerprint sort
// (overlap.cu:613-656: sort by id, partition even/odd, sort each part).  The
// two lists sit back to back [suffixes | prefixes]; value = id | table<<31.
// Keeping the lists in id order removes the reference's per-round id sort.
//
// Kernels
//   dedup_mark      first entry of each equal-key run survives
//                   (cq_unique_by_key, cqutils.cuh:272-306; in-core the
//                   survivor is the smallest id because the sort is stable)
//   init_list       ids of survivors in (even, odd) order + their keys
//   update_compact  drop entries whose id was used in the previous round
//                   (remove_used, overlap.cu:694-710) and apply NextSfx /
//                   PrevPfx with the base gathered from the 2-bit column store
//                   (filter_bases, overlap.cu:670-692); order-preserving
//                   compaction by single-pass chained scan.
//   join_count      in the merged sorted list every equal-key run holds its
//                   suffixes then its prefixes; per suffix count the prefixes
//                   of the same key from another read (get_edges self-edge
//                   filter, overlap.cu:594-598)
//   join_write      write (suffix id, prefix id) at the scanned offsets in
//                   (suffix order, prefix order) -- the order of get_edges
//                   (overlap.cu:557-603) -- and mark used ids.
#include "kernels.h"

namespace emp {

__global__ void dedup_mark_kernel(const uint64_t *__restrict__ k, const uint32_t *__restrict__ v, uint64_t n,
                                  uint8_t *__restrict__ alive) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        alive[v[i] & 0x7fffffffu] = (i == 0 || k[i] != k[i - 1]) ? 1 : 0;
}

constexpr int kChunks = kUpdTile / 256;  // 8

__global__ void __launch_bounds__(256) init_list_kernel(const uint64_t *__restrict__ keys0,
                                                        const uint8_t *__restrict__ alive, uint64_t n,
                                                        uint64_t *__restrict__ lk, uint32_t *__restrict__ lv,
                                                        uint64_t *status, uint32_t *tile_ctr, uint64_t *count,
                                                        uint32_t *err) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[8];
    __shared__ uint64_t s_base;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * kUpdTile, n2 = 2 * n;
    uint32_t rid[kChunks], ex[kChunks];
    bool keep[kChunks];
    uint32_t running = 0;
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
        const uint64_t q = base + c * 256 + threadIdx.x;
        keep[c] = false;
        rid[c] = 0;
        if (q < n2) {
            rid[c] = q < n ? (uint32_t)(2 * q) : (uint32_t)(2 * (q - n) + 1);
            keep[c] = alive[rid[c]] != 0;
        }
        uint32_t tot;
        ex[c] = running + block_exclusive_scan<256, uint32_t>(keep[c] ? 1u : 0u, s_warp, &tot);
        running += tot;
    }
    if (threadIdx.x == 0) s_base = lookback_exclusive(status, tile, running, err);
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
        if (keep[c]) {
            const uint64_t o = s_base + ex[c];
            lk[o] = keys0[rid[c]];
            lv[o] = rid[c];
        }
    }
    if (threadIdx.x == 0 && (uint64_t)tile == upd_tiles(n2) - 1) *count = s_base + running;
}

__global__ void iota_kernel(uint32_t *__restrict__ v, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        v[i] = (uint32_t)i;
}

__global__ void dup_prefix_half_kernel(uint64_t *__restrict__ lk, uint32_t *__restrict__ lv, uint64_t u) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < u; i += (uint64_t)gridDim.x * blockDim.x) {
        lk[u + i] = lk[i];
        lv[u + i] = lv[i] | 0x80000000u;
    }
}

EMP_DEV uint32_t column_code(const uint32_t *__restrict__ cols, uint64_t wpc, int col, uint32_t i) {
    return (__ldg(cols + (uint64_t)col * wpc + (i >> 4)) >> ((i & 15u) * 2u)) & 3u;
}

__global__ void __launch_bounds__(256) update_compact_kernel(RoundArgs a) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[8];
    __shared__ uint64_t s_base;
    __shared__ uint32_t s_sfx;
    if (threadIdx.x == 0) {
        s_tile = atomicAdd(a.tile_ctr, 1u);
        s_sfx = 0;
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * kUpdTile;
    const int L = a.L, r = a.round;
    const int cf = r, cb = L - 1 - r;
    const uint32_t pw1 = a.tables->pow1[L - r - 1], pw2 = a.tables->pow2[L - r - 1];
    const uint32_t inv1 = a.tables->inv1, inv2 = a.tables->inv2;
    uint64_t key[kChunks];
    uint32_t val[kChunks], ex[kChunks];
    bool keep[kChunks];
    uint32_t running = 0, sfx_kept = 0;
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
        const uint64_t e = base + c * 256 + threadIdx.x;
        keep[c] = false;
        key[c] = 0;
        val[c] = 0;
        if (e < a.n_in) {
            uint64_t k = a.kin[e];
            const uint32_t v = a.vin[e];
            const uint32_t rid = v & 0x7fffffffu, t = v >> 31, s = rid & 1u, i = rid >> 1;
            const bool used = t ? a.used_p[rid] : a.used_s[rid];
            if (!used) {
                const int col = t == 0 ? (s ? cb : cf) : (s ? cf : cb);
                const uint32_t b = column_code(a.cols, a.wpc, col, i) ^ (s << 1);
                k = t == 0 ? next_sfx(k, b, pw1, pw2) : prev_pfx(k, b, inv1, inv2);
                keep[c] = true;
                sfx_kept += t == 0;
            }
            key[c] = k;
            val[c] = v;
        }
        uint32_t tot;
        ex[c] = running + block_exclusive_scan<256, uint32_t>(keep[c] ? 1u : 0u, s_warp, &tot);
        running += tot;
    }
    if (sfx_kept) atomicAdd(&s_sfx, sfx_kept);
    if (threadIdx.x == 0) s_base = lookback_exclusive(a.status, tile, running, a.err);
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
        if (keep[c]) {
            const uint64_t o = s_base + ex[c];
            a.kout[o] = key[c];
            a.vout[o] = val[c];
        }
    }
    if (threadIdx.x == 0) {
        if (s_sfx) atomicAdd(reinterpret_cast<unsigned long long *>(a.s_out), (unsigned long long)s_sfx);
        if ((uint64_t)tile == upd_tiles(a.n_in) - 1) *a.n_out = s_base + running;
    }
}

__global__ void join_count_kernel(const uint64_t *__restrict__ k, const uint32_t *__restrict__ v, uint64_t n,
                                  uint32_t *__restrict__ cnt) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t vi = v[i];
        uint32_t c = 0;
        if ((vi >> 31) == 0) {
            const uint64_t ki = k[i];
            const uint32_t ri = (vi & 0x7fffffffu) >> 1;
            for (uint64_t j = i + 1; j < n && k[j] == ki; ++j) {
                const uint32_t vj = v[j];
                if ((vj >> 31) && ((vj & 0x7fffffffu) >> 1) != ri) ++c;
            }
        }
        cnt[i] = c;
    }
}

__global__ void join_write_kernel(const uint64_t *__restrict__ k, const uint32_t *__restrict__ v, uint64_t n,
                                  const uint32_t *__restrict__ cnt, const uint64_t *__restrict__ offs,
                                  uint32_t *__restrict__ from, uint32_t *__restrict__ to, uint8_t *__restrict__ used_s,
                                  uint8_t *__restrict__ used_p) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (!cnt[i]) continue;
        const uint64_t ki = k[i];
        const uint32_t si = v[i] & 0x7fffffffu, ri = si >> 1;
        uint64_t o = offs[i];
        for (uint64_t j = i + 1; j < n && k[j] == ki; ++j) {
            const uint32_t vj = v[j];
            const uint32_t pj = vj & 0x7fffffffu;
            if ((vj >> 31) && (pj >> 1) != ri) {
                from[o] = si;
                to[o] = pj;
                used_p[pj] = 1;
                ++o;
            }
        }
        used_s[si] = 1;
    }
}

__global__ void __launch_bounds__(256) split_tables_kernel(const uint64_t *__restrict__ k,
                                                           const uint32_t *__restrict__ v, uint64_t n,
                                                           uint64_t *__restrict__ akeys, uint32_t *__restrict__ apos,
                                                           uint64_t *__restrict__ bkeys, uint64_t *status,
                                                           uint32_t *tile_ctr, uint32_t *err) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[8];
    __shared__ uint64_t s_base;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * kUpdTile;
    uint32_t ex[kChunks];
    bool isa[kChunks];
    uint32_t running = 0;
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
        const uint64_t e = base + c * 256 + threadIdx.x;
        isa[c] = e < n && (v[e] >> 31) == 0;
        uint32_t tot;
        ex[c] = running + block_exclusive_scan<256, uint32_t>(isa[c] ? 1u : 0u, s_warp, &tot);
        running += tot;
    }
    if (threadIdx.x == 0) s_base = lookback_exclusive(status, tile, running, err);
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
        const uint64_t e = base + c * 256 + threadIdx.x;
        if (e >= n) continue;
        const uint64_t ra = s_base + ex[c];
        if (isa[c]) {
            akeys[ra] = k[e];
            apos[ra] = (uint32_t)e;
        } else {
            bkeys[e - ra] = k[e];
        }
    }
}

EMP_DEV uint64_t lower_bound_dev(const uint64_t *a, uint64_t lo, uint64_t hi, uint64_t key) {
    while (lo < hi) {
        const uint64_t m = lo + (hi - lo) / 2;
        if (a[m] < key) lo = m + 1;
        else hi = m;
    }
    return lo;
}

__global__ void search_partitions_kernel(const uint64_t *__restrict__ A, uint64_t S, const uint64_t *__restrict__ B,
                                         uint64_t P, uint64_t h, const uint32_t *__restrict__ apos,
                                         const uint64_t *__restrict__ offs, uint64_t E, SearchPart *parts,
                                         uint64_t cap, uint64_t *count, uint32_t *err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint64_t offA = 0, offB = 0, np = 0;
    bool failed = false;
    auto eoff = [&](uint64_t rank) -> uint64_t { return rank < S ? offs[apos[rank]] : E; };
    auto push = [&](uint64_t pa, uint64_t pb) -> bool {
        if (np >= cap) {
            atomicOr(err, kErrCapacity);
            failed = true;
            return false;
        }
        parts[np].pa = pa;
        parts[np].pb = pb;
        parts[np].e0 = eoff(offA);
        parts[np].e1 = eoff(offA + pa);
        ++np;
        return true;
    };
    while (offA < S && offB < P) {
        uint64_t pa = S - offA < h ? S - offA : h, pb = P - offB < h ? P - offB : h;
        if (pa < h && pb < h) {
            if (!push(pa, pb)) break;
            offA += pa;
            offB += pb;
            break;
        }
        const uint64_t la = A[offA + pa - 1], lb = B[offB + pb - 1];
        const uint64_t m = la < lb ? la : lb;
        pa = lower_bound_dev(A, offA, offA + pa, m) - offA;
        pb = lower_bound_dev(B, offB, offB + pb, m) - offB;
        if (pa == 0 && pb == 0) {
            atomicOr(err, kErrHang);
            failed = true;
            break;
        }
        if (!push(pa, pb)) break;
        offA += pa;
        offB += pb;
    }
    if (!failed) {
        if (offA == S && offB < P) push(0, P - offB);
        else if (offB == P && offA < S) push(S - offA, 0);
    }
    *count = np;
}

static unsigned grid_for(uint64_t work, unsigned per_block, unsigned cap) {
    uint64_t g = (work + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

void launch_dedup_mark(const uint64_t *skeys, const uint32_t *svals, uint64_t n2, uint8_t *alive, cudaStream_t s) {
    if (!n2) return;
    count_launch();
    dedup_mark_kernel<<<grid_for(n2, 256, 148 * 8), 256, 0, s>>>(skeys, svals, n2, alive);
}

void launch_init_list(const uint64_t *keys0, const uint8_t *alive, uint64_t n, uint64_t *lkeys, uint32_t *lvals,
                      uint64_t *status, uint32_t *tile_ctr, uint64_t *count, uint32_t *err, cudaStream_t s) {
    if (!n) {
        cudaMemsetAsync(count, 0, sizeof(uint64_t), s);
        return;
    }
    count_launch();
    init_list_kernel<<<(unsigned)upd_tiles(2 * n), 256, 0, s>>>(keys0, alive, n, lkeys, lvals, status, tile_ctr,
                                                                 count, err);
}

void launch_iota(uint32_t *v, uint64_t n, cudaStream_t s) {
    if (!n) return;
    count_launch();
    iota_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(v, n);
}

void launch_dup_prefix_half(uint64_t *lkeys, uint32_t *lvals, uint64_t u, cudaStream_t s) {
    if (!u) return;
    count_launch();
    dup_prefix_half_kernel<<<grid_for(u, 256, 148 * 8), 256, 0, s>>>(lkeys, lvals, u);
}

void launch_update_compact(const RoundArgs &a, cudaStream_t s) {
    if (!a.n_in) {
        cudaMemsetAsync(a.n_out, 0, sizeof(uint64_t), s);
        return;
    }
    count_launch();
    update_compact_kernel<<<(unsigned)upd_tiles(a.n_in), 256, 0, s>>>(a);
}

void launch_split_tables(const uint64_t *skeys, const uint32_t *svals, uint64_t n, uint64_t *akeys, uint32_t *apos,
                         uint64_t *bkeys, uint64_t *status, uint32_t *tile_ctr, uint32_t *err, cudaStream_t s) {
    if (!n) return;
    count_launch();
    split_tables_kernel<<<(unsigned)upd_tiles(n), 256, 0, s>>>(skeys, svals, n, akeys, apos, bkeys, status, tile_ctr,
                                                               err);
}

void launch_search_partitions(const uint64_t *akeys, uint64_t S, const uint64_t *bkeys, uint64_t P, uint64_t h,
                              const uint32_t *apos, const uint64_t *offs, uint64_t E, SearchPart *parts,
                              uint64_t cap, uint64_t *count, uint32_t *err, cudaStream_t s) {
    count_launch();
    search_partitions_kernel<<<1, 32, 0, s>>>(akeys, S, bkeys, P, h, apos, offs, E, parts, cap, count, err);
}

void launch_join_count(const uint64_t *skeys, const uint32_t *svals, uint64_t n, uint32_t *cnt, cudaStream_t s) {
    if (!n) return;
    count_launch();
    join_count_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(skeys, svals, n, cnt);
}

void launch_join_write(const uint64_t *skeys, const uint32_t *svals, uint64_t n, const uint32_t *cnt,
                       const uint64_t *offs, uint32_t *from, uint32_t *to, uint8_t *used_s, uint8_t *used_p,
                       cudaStream_t s) {
    if (!n) return;
    count_launch();
    join_write_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(skeys, svals, n, cnt, offs, from, to, used_s,
                                                                  used_p);
}

}  // namespace emp
