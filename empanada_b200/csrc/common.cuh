// common.cuh -- device helpers shared by the overlap-path kernels.
//
// Fingerprint arithmetic follows the reference exactly:
//   primes and radices           assembly.cuh:29-32
//   ENCODING(c) = ((c>>1)&3)+1   assembly.cuh:34   (A1 C2 T3 G4)
//   key = fp1 << 32 | fp2        assembly.cuh:50-52 (APPEND64)
//   NextSfx                      overlap.cu:57-75
//   PrevPfx (wrapping u64)       overlap.cu:77-91
// A base is carried as its 2-bit code v = (c>>1)&3 (A0 C1 T2 G3); the
// Watson-Crick complement is v^2 and ENCODING is v+1.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define EMP_DEV __device__ __forceinline__

namespace emp {

constexpr uint32_t kP1 = 536870909u;  // 2^29 - 3
constexpr uint32_t kP2 = 536870879u;  // 2^29 - 33
constexpr uint32_t kR1 = 5u;
constexpr uint32_t kR2 = 7u;
constexpr uint32_t kMask29 = (1u << 29) - 1u;
// Longest read.  The reference's MAX_RD_LEN (assembly.cuh:17) is 255: its u8
// lengths and 256-entry power tables overflow beyond it, so its results are
// undefined there.  Here the same exact hash runs on to 512 bases, with the
// power tables extended to match.
constexpr int kMaxReadLen = 512;
constexpr int kRefMaxReadLen = 255;

// Error bits raised by kernels into the job's device error word.
enum ErrBits : uint32_t {
    kErrSpin = 1u,      // a look-back wait ran out of iterations
    kErrBadBase = 2u,   // a kept read holds a byte outside ACGTacgt
    kErrCapacity = 4u,  // an output would overflow its buffer
    kErrHang = 8u,      // the reference would loop forever on this input
    kErrDedupFull = 16u,  // a duplicate-removal bucket had too many distinct keys (the sort takes over)
};

// Powers R^i mod P for i <= kMaxReadLen and the radix inverses (fingerprint.cu:26-34,
// overlap.cu:121-122).  Lives in device memory; staged into shared memory by
// the kernels that need it.
struct HashTables {
    uint32_t pow1[kMaxReadLen + 1];
    uint32_t pow2[kMaxReadLen + 1];
    uint32_t inv1;
    uint32_t inv2;
};
// Weights of read positions 16c .. 16c+15 for the read pass (Rinv = R^-1 mod
// P), w[c] = Rinv1^(16c+7), Rinv1^(16c+15), Rinv2^(16c+7), Rinv2^(16c+15),
// R1^(16c), R1^(16c+8), R2^(16c), R2^(16c+8).  In device memory right after
// the HashTables.
struct ChunkWeights {
    uint32_t w[kMaxReadLen / 16][8];
};

// x mod (2^29 - C) for any 64-bit x: two pseudo-Mersenne folds then one
// conditional subtraction (after the folds x < 2^29 + 2^18 < 2P).
template <uint32_t C, uint32_t P>
EMP_DEV uint32_t mod_fold(uint64_t x) {
    uint64_t y = (x & kMask29) + (x >> 29) * C;
    y = (y & kMask29) + (y >> 29) * C;
    uint32_t z = (uint32_t)y;
    return z >= P ? z - P : z;
}
EMP_DEV uint32_t mod1(uint64_t x) { return mod_fold<3u, kP1>(x); }
EMP_DEV uint32_t mod2(uint64_t x) { return mod_fold<33u, kP2>(x); }

// 32-bit fold for h*R + e with h < P, R <= 7, e <= 4 (value < 2^32).
template <uint32_t C, uint32_t P>
EMP_DEV uint32_t mod_fold32(uint32_t x) {
    uint32_t y = (x & kMask29) + (x >> 29) * C;
    return y >= P ? y - P : y;
}
EMP_DEV uint32_t horner1(uint32_t h, uint32_t e) { return mod_fold32<3u, kP1>(h * kR1 + e); }
EMP_DEV uint32_t horner2(uint32_t h, uint32_t e) { return mod_fold32<33u, kP2>(h * kR2 + e); }

EMP_DEV uint32_t base_code(uint8_t c) { return (c >> 1) & 3u; }

EMP_DEV bool is_acgt(uint8_t c) {
    c |= 0x20;  // fold case
    return c == 'a' || c == 'c' || c == 'g' || c == 't';
}

// markNs (preprocess.cu:119-121) == 9  <=>  64 <= c <= 127 with bit 3 set.
EMP_DEV bool is_n_class(uint8_t c) { return (c & 0xC0u) == 0x40u && (c & 8u); }

// NextSfx: drop the first base (code v) of a length-len suffix; pw = R^(len-1).
EMP_DEV uint64_t next_sfx(uint64_t key, uint32_t v, uint32_t pw1, uint32_t pw2) {
    uint32_t f1 = (uint32_t)(key >> 32), f2 = (uint32_t)key;
    uint32_t e = v + 1u;
    uint32_t t1 = mod1((uint64_t)(e * pw1));  // 32-bit product < 2^31, as in the reference
    uint32_t t2 = mod2((uint64_t)(e * pw2));
    f1 = f1 >= t1 ? f1 - t1 : f1 + kP1 - t1;
    f2 = f2 >= t2 ? f2 - t2 : f2 + kP2 - t2;
    return ((uint64_t)f1 << 32) | f2;
}

// PrevPfx: drop the last base (code v).  Subtraction and product wrap mod 2^64
// exactly like the reference's uint64_t expression.
EMP_DEV uint64_t prev_pfx(uint64_t key, uint32_t v, uint32_t inv1, uint32_t inv2) {
    uint64_t f1 = key >> 32, f2 = key & 0xffffffffull;
    uint64_t e = v + 1u;
    uint64_t x1 = (uint64_t)inv1 * (f1 - e);
    uint64_t x2 = (uint64_t)inv2 * (f2 - e);
    return ((uint64_t)mod1(x1) << 32) | mod2(x2);
}

// 59-bit sort key: (fp1, fp2) order-preserving in 58 bits, table bit below.
EMP_DEV uint64_t sort_key(uint64_t key, uint32_t val) {
    return ((key >> 32) << 30) | ((key & kMask29) << 1) | (val >> 31);
}

// ---------------------------------------------------------------- bulk copies
// One-dimensional TMA copies global -> shared completed on an mbarrier (the
// copy engine moves the bytes; one thread issues them).  Both addresses and
// the size must be multiples of 16 bytes.
EMP_DEV uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
EMP_DEV void mbar_init(uint64_t *bar, uint32_t arrivals) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(arrivals) : "memory");
}
// generic-proxy accesses of shared memory before this point are ordered
// before later async-proxy (bulk copy) accesses, and mbarrier inits are seen
EMP_DEV void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
EMP_DEV void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// arrive, expecting `bytes` of bulk copies, and start one copy of `bytes`
EMP_DEV void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// start pulling `bytes` of global memory into L2 (a hint: no completion)
EMP_DEV void prefetch_l2(const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}
// wait for the barrier's phase `parity` to complete; false after `limit` polls
EMP_DEV bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// ---------------------------------------------------------------- look-back
// Single-pass chained scan status words: flag in bits 62-63, value below.
constexpr uint64_t kStAgg = 1ull << 62;
constexpr uint64_t kStInc = 2ull << 62;
constexpr uint64_t kStVal = (1ull << 62) - 1;
constexpr uint32_t kSpinLimit = 1u << 22;

EMP_DEV void st_status(uint64_t *p, uint64_t v) { *(volatile uint64_t *)p = v; }
EMP_DEV uint64_t ld_status(const uint64_t *p) { return *(const volatile uint64_t *)p; }

// Publish this tile's aggregate, walk back to the nearest inclusive prefix and
// publish this tile's inclusive prefix.  Called by ONE thread.  Every wait is
// bounded: on timeout the error bit is raised and the tile publishes what it
// has so that no successor waits forever.
EMP_DEV uint64_t lookback_exclusive(uint64_t *status, uint32_t tile, uint64_t aggregate, uint32_t *err) {
    if (tile == 0) {
        st_status(status, kStInc | aggregate);
        return 0;
    }
    st_status(status + tile, kStAgg | aggregate);
    uint64_t excl = 0;
    int64_t t = (int64_t)tile - 1;
    while (t >= 0) {
        uint64_t s;
        uint32_t spins = 0;
        while (((s = ld_status(status + t)) >> 62) == 0) {
            if (++spins > kSpinLimit) {
                atomicOr(err, kErrSpin);
                st_status(status + tile, kStInc | (excl + aggregate));
                return excl;
            }
            __nanosleep(64);
        }
        excl += s & kStVal;
        if ((s >> 62) == 2) break;
        --t;
    }
    st_status(status + tile, kStInc | (excl + aggregate));
    return excl;
}

// Epoch-tagged status words: epoch in bits 44-63, flag in 42-43, value below.
// A word whose epoch differs from the caller's is "not ready", so status
// arrays never need clearing between uses (each use has a fresh epoch).
constexpr uint64_t kEpAgg = 1ull << 42;
constexpr uint64_t kEpInc = 2ull << 42;
constexpr uint64_t kEpVal = (1ull << 42) - 1;
EMP_DEV uint64_t ep_word(uint32_t epoch, uint64_t flag, uint64_t v) { return ((uint64_t)epoch << 44) | flag | v; }
EMP_DEV uint32_t ep_flag(uint64_t w, uint32_t epoch) {
    return (uint32_t)(w >> 44) == (epoch & 0xfffffu) ? (uint32_t)((w >> 42) & 3u) : 0u;
}

// lookback_exclusive with epoch-tagged words; reads up to 4 predecessors at
// a time.  One thread; bounded waits as above.
EMP_DEV uint64_t lookback_epoch(uint64_t *status, uint32_t tile, uint64_t aggregate, uint32_t epoch,
                                uint32_t *err) {
    epoch &= 0xfffffu;
    if (tile == 0) {
        st_status(status, ep_word(epoch, kEpInc, aggregate));
        return 0;
    }
    st_status(status + tile, ep_word(epoch, kEpAgg, aggregate));
    uint64_t excl = 0;
    int64_t t = (int64_t)tile - 1;
    while (t >= 0) {
        const int k = t >= 3 ? 4 : (int)t + 1;
        uint64_t w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i < k) w[i] = ld_status(status + (t - i));
        bool inc = false;
        for (int i = 0; i < k && !inc; ++i) {
            uint32_t f, spins = 0;
            while ((f = ep_flag(w[i], epoch)) == 0) {
                if (++spins > kSpinLimit) {
                    atomicOr(err, kErrSpin);
                    st_status(status + tile, ep_word(epoch, kEpInc, excl + aggregate));
                    return excl;
                }
                if (spins > 32) __nanosleep(32);
                w[i] = ld_status(status + (t - i));
            }
            excl += w[i] & kEpVal;
            inc = f == 2;
        }
        if (inc) break;
        t -= k;
    }
    st_status(status + tile, ep_word(epoch, kEpInc, excl + aggregate));
    return excl;
}

// Warp-parallel lookback_epoch: called by all 32 lanes of ONE warp; each probe
// reads the 32 nearest unresolved predecessors at once, waits (bounded) until
// all of them have published, and stops at the nearest inclusive prefix.
// Returns the exclusive prefix in every lane.
EMP_DEV uint64_t lookback_epoch_warp(uint64_t *status, uint32_t tile, uint64_t aggregate, uint32_t epoch,
                                     uint32_t *err) {
    const int lane = threadIdx.x & 31;
    epoch &= 0xfffffu;
    if (tile == 0) {
        if (lane == 0) st_status(status, ep_word(epoch, kEpInc, aggregate));
        return 0;
    }
    if (lane == 0) st_status(status + tile, ep_word(epoch, kEpAgg, aggregate));
    uint64_t excl = 0;
    int64_t t = (int64_t)tile - 1;  // nearest predecessor not yet folded in
    bool failed = false;
    while (!failed) {
        const int64_t idx = t - lane;
        uint64_t w = 0;
        uint32_t f = 2;  // before tile 0: an inclusive prefix of 0
        if (idx >= 0) {
            uint32_t spins = 0;
            w = ld_status(status + idx);
            while ((f = ep_flag(w, epoch)) == 0) {
                if (++spins > kSpinLimit) {
                    failed = true;
                    f = 2;
                    w = 0;
                    break;
                }
                if (spins > 32) __nanosleep(32);
                w = ld_status(status + idx);
            }
        }
        failed = __any_sync(0xffffffffu, failed);
        const uint32_t inc = __ballot_sync(0xffffffffu, f == 2);
        const int stop = inc ? __ffs(inc) - 1 : 31;  // nearest inclusive prefix in the window
        uint64_t v = lane <= stop ? (w & kEpVal) : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        if (inc) break;
        t -= 32;
    }
    if (failed && lane == 0) atomicOr(err, kErrSpin);
    if (lane == 0) st_status(status + tile, ep_word(epoch, kEpInc, excl + aggregate));
    return excl;
}

// Block-wide exclusive scan of one value per thread (blockDim.x = NT).
template <int NT, typename T>
EMP_DEV T block_exclusive_scan(T v, T *smem_warp /* NT/32 */, T *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if constexpr (NT <= 256) {  // every thread adds up the (at most 8) warp totals itself
        T before = T(0), all = T(0);
#pragma unroll
        for (int w = 0; w < NT / 32; ++w) {
            const T t = smem_warp[w];
            all += t;
            if (w < warp) before += t;
        }
        *total = all;
        __syncthreads();  // smem_warp is written again by the next scan
        return before + x - v;
    } else {
        if (warp == 0) {
            T w = lane < NT / 32 ? smem_warp[lane] : T(0);
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                T y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < NT / 32) smem_warp[lane] = w;
        }
        __syncthreads();
        T warp_excl = warp ? smem_warp[warp - 1] : T(0);
        *total = smem_warp[NT / 32 - 1];
        __syncthreads();
        return warp_excl + x - v;
    }
}

}  // namespace emp
