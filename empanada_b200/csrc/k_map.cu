// k_map.cu -- map phase: FASTQ bytes in HBM -> kept reads -> fingerprints of
// every read-end + read-major 2-bit bases (+ the column-major store when a
// round must run outside the bucket kernel).
//
// Reference behaviour restated (file:line in the reference project):
//   line ids / sequence lines   preprocess.cu:26-37, 70-87 (line g%4 == 1)
//   N filter                    preprocess.cu:98-182 (markNs == 9 drops the read)
//   equal read length           fingerprint.cu:125-153 (transpose_reads)
//   read-end ids                fingerprint.cu:75-115 (rid = 2i fwd, 2i+1 RC)
//   fingerprints                fingerprint.cu:36-65 (FingerprintMul, Horner form)
//   transposed bases            fingerprint.cu:125-153, blocks.cuh:11-128
//
// Kernels
//   nl_count      newline count of each 16 KB tile (16-byte vector loads);
//                 tile 0 also measures the first record's sequence line
//   read_pass     one CTA per tile staged in shared memory: the records'
//                 sequence lines, N filter, ACGT check, length, both
//                 fingerprints and the read-major 2-bit words, at each
//                 record's own index
//   compact_reads the kept records to consecutive indices (only when the
//                 N filter or an empty line dropped one)
//   columns       read-major words -> column-major words (only when needed)
#include <atomic>

#include "sort_block.cuh"

namespace emp {

EMP_DEV uint32_t nl_in_word(uint32_t w) { return __popc(__vcmpeq4(w, 0x0a0a0a0au)) >> 3; }

// smallest newline position of a 16-byte block above `after` (or ~0)
EMP_DEV uint32_t first_nl_after(const uint4 &v, uint32_t off, uint32_t after) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    uint32_t best = 0xffffffffu;
#pragma unroll
    for (int q = 3; q >= 0; --q) {
        uint32_t m = __vcmpeq4(w[q], 0x0a0a0a0au);
        while (m) {
            const uint32_t pos = off + 4 * q + ((__ffs(m) - 1) >> 3);
            m &= m - 1;
            m &= ~(0xffu << (8 * ((pos - off) & 3)));
            if (pos + 1 > after + 1 || after == 0xffffffffu) best = min(best, pos);
        }
    }
    return best;
}

__global__ void __launch_bounds__(256) nl_count_kernel(const uint8_t *__restrict__ fq, uint64_t F,
                                                       uint32_t *__restrict__ tile_counts, uint64_t *len0) {
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_nl[2];
    const uint64_t base = (uint64_t)blockIdx.x * kParseTile;
    uint32_t c = 0;
    uint4 blk[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint64_t off = base + ((uint64_t)k * 256 + threadIdx.x) * 16;
        blk[k] = make_uint4(0, 0, 0, 0);
        if (off + 16 <= F) {
            blk[k] = *reinterpret_cast<const uint4 *>(fq + off);
        } else {
            uint32_t *wb = reinterpret_cast<uint32_t *>(&blk[k]);
            for (int b = 0; b < 16; ++b)
                if (off + b < F) wb[b >> 2] |= (uint32_t)fq[off + b] << (8 * (b & 3));
        }
        c += nl_in_word(blk[k].x) + nl_in_word(blk[k].y) + nl_in_word(blk[k].z) + nl_in_word(blk[k].w);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = c;
    if (blockIdx.x == 0 && threadIdx.x == 0) s_nl[0] = s_nl[1] = 0xffffffffu;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < 8; ++w) t += s_warp[w];
        tile_counts[blockIdx.x] = t;
    }
    if (blockIdx.x != 0) return;
    // tile 0: the first record's sequence line lies between newlines 0 and 1
    // (a hint for sizing the read-major word store; 0 when not found here)
    uint32_t a = 0xffffffffu;
#pragma unroll
    for (int k = 0; k < 4; ++k) a = min(a, first_nl_after(blk[k], (uint32_t)(k * 256 + threadIdx.x) * 16, 0xffffffffu));
    if (a != 0xffffffffu) atomicMin(&s_nl[0], a);
    __syncthreads();
    const uint32_t p0 = s_nl[0];
    if (p0 != 0xffffffffu) {
        uint32_t b = 0xffffffffu;
#pragma unroll
        for (int k = 0; k < 4; ++k) b = min(b, first_nl_after(blk[k], (uint32_t)(k * 256 + threadIdx.x) * 16, p0));
        if (b != 0xffffffffu) atomicMin(&s_nl[1], b);
    }
    __syncthreads();
    if (threadIdx.x == 0) *len0 = (s_nl[0] != 0xffffffffu && s_nl[1] != 0xffffffffu) ? s_nl[1] - s_nl[0] - 1 : 0;
}

// 0x80 in every byte of t that is zero, 0 elsewhere (no carries between bytes)
EMP_DEV uint32_t zero_bytes(uint32_t t) { return ~(((t & 0x7f7f7f7fu) + 0x7f7f7f7fu) | t | 0x7f7f7f7fu); }

// ---------------------------------------------------------------- reads
// One CTA per 16 KB FASTQ tile (the tiles of nl_count), the tile and the
// 1 KB after it staged in shared memory.  A record belongs to the tile that
// holds the newline ending its header (line 4k); its sequence line runs from
// there to newline 4k+1, or to the end of the input.
//
//   locate   each thread counts the newlines of 64 tile bytes and 4 halo
//            bytes; one block scan gives every newline its line id, and the
//            tile's records their sequence bounds (window offsets)
//   records  G lanes per record (G from the tile's record count), 16 bases
//            a lane:
//            * a byte is one of ACGTacgt iff it equals "ACTG"[(b >> 1) & 3]
//              up to case (two byte permutes per 4 bytes); only a read that
//              fails this is searched for N-class bytes (markNs == 9).  The
//              record is kept when it holds no N-class byte and is not empty;
//            * the lane's bases give one read-major 2-bit word and, per
//              fingerprint, two 8-base dot products (dp4a / dp2a) weighted
//              by the chunk's constants:
//                H(read)    = R^(L-1) * sum_t enc(b_t) R^-t      mod P
//                H(revcomp) =           sum_t enc(comp b_t) R^t  mod P
//              (FingerprintMul's Horner form regrouped: the same residues);
//              64-bit partial sums meet in a shuffle reduction.
// Outputs go to the record's own index k (keys[2k], seq2[k * wpr ..]) with
// keep[k]; the kept count is summed with one atomic per tile.  When a record
// was dropped, compact_reads moves the kept ones to consecutive indices.  A
// sequence line that does not end inside the window (over 1 KB: never
// hashed) is checked by one lane straight from global memory.
constexpr int kRT = 256;
constexpr uint32_t kHalo = 528;  // a line of kMaxReadLen bases starting at the tile's end, rounded to 16
constexpr uint32_t kWin = (uint32_t)kParseTile + kHalo;
constexpr uint32_t kWinWords = kWin / 4;
constexpr uint32_t kRecCap = 2048;  // records per batch (a tile owns up to 4096: four newlines each)
constexpr uint16_t kNoEnd = 0xffffu;
constexpr int kChunks = kMaxReadLen / 16;
static_assert(kParseTile == 64 * kRT, "64 tile bytes per thread");
static_assert(kHalo % 16 == 0 && kHalo / 16 <= kRT && kHalo >= kMaxReadLen + 1, "one halo chunk per thread at most");
static_assert(kWin < kNoEnd, "window offsets fit 16 bits");
static_assert(kMaxReadLen % 16 == 0, "whole read-major words");

struct __align__(16) ReadSmem {
    uint32_t win[2][kWinWords + 8];  // two windows (zero past the input), each then zero padding
    uint32_t chunk[kChunks][8];      // ChunkWeights::w
    uint16_t start[kRecCap];         // sequence line [start, end) of the batch's records (window offsets)
    uint16_t end[kRecCap];           // kNoEnd: no newline ends it inside the window
    uint32_t scan32[kRT / 32];
    uint64_t bar[2];  // bulk-copy barriers of the two windows
};

// newline bytes of a word as 4 bits (byte b -> bit b): the bytes' top bits
// gathered by one multiply (partial products land on distinct bits)
EMP_DEV uint32_t nl_bits(uint32_t w) { return ((zero_bytes(w ^ 0x0a0a0a0au) >> 7) * 0x00204081u) >> 21 & 0xfu; }
// newline bytes of 16 bytes as 16 bits, byte order
EMP_DEV uint32_t nl_mask16(const uint4 &v) {
    return nl_bits(v.x) | (nl_bits(v.y) << 4) | (nl_bits(v.z) << 8) | (nl_bits(v.w) << 12);
}

// 16 window bytes from byte offset off (any alignment): x[q] = bytes off+4q ..
EMP_DEV void win16(const uint32_t *win, uint32_t off, uint32_t x[4]) {
    const uint32_t w = off >> 2, sh = (off & 3u) * 8u;
    uint32_t a = win[w];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint32_t b = win[w + q + 1];
        x[q] = __funnelshift_r(a, b, sh);
        a = b;
    }
}
// 0xff in the first n bytes of a word (n clamped to 0..4)
EMP_DEV uint32_t lead_bytes(int n) { return n >= 4 ? 0xffffffffu : n <= 0 ? 0u : (1u << (8 * n)) - 1u; }
// nonzero iff a byte of x selected by vm is not one of ACGTacgt
EMP_DEV uint32_t not_acgt(uint32_t x, uint32_t vm) {
    const uint32_t c = (x >> 1) & 0x03030303u;
    const uint32_t sel = __byte_perm(c | (c >> 4), 0u, 0x4420u);  // the codes as byte selectors
    const uint32_t want = __byte_perm(0x47544341u, 0u, sel);       // "ACTG"[code]
    return (x ^ want) & 0xdfdfdfdfu & vm;
}
// nonzero iff a byte of x selected by vm is N-class (bits 7-6 = 01, bit 3 set)
EMP_DEV uint32_t n_class(uint32_t x, uint32_t vm) { return zero_bytes((x & 0xc8c8c8c8u) ^ 0x48484848u) & vm; }
// x mod P = 2^29 - C for a P chosen at run time (mod1 / mod2 with their
// constants as arguments, so that the lanes of a group reduce different
// residues in one instruction stream)
constexpr uint32_t kP1C = (1u << 29) - kP1, kP2C = (1u << 29) - kP2;
EMP_DEV uint32_t mod_rt(uint64_t x, uint32_t C, uint32_t P) {
    uint64_t y = (x & kMask29) + (x >> 29) * C;
    y = (y & kMask29) + (y >> 29) * C;
    const uint32_t z = (uint32_t)y;
    return z >= P ? z - P : z;
}

// 4-base dot products of enc values in bytes (first base first), added to acc
EMP_DEV uint32_t fw1(uint32_t e, uint32_t acc) { return __dp4a(e, 0x0105197Du, acc); }  // 125 25 5 1
EMP_DEV uint32_t rc1(uint32_t e, uint32_t acc) { return __dp4a(e, 0x7D190501u, acc); }  // 1 5 25 125
EMP_DEV uint32_t fw2(uint32_t e, uint32_t acc) {  // 343 49 7 1
    return __dp2a_lo(0x00310157u, e, __dp2a_hi(0x00010007u, e, acc));
}
EMP_DEV uint32_t rc2(uint32_t e, uint32_t acc) {  // 1 7 49 343
    return __dp2a_lo(0x00070001u, e, __dp2a_hi(0x01570031u, e, acc));
}

// One lane's 16 bases (x: the chunk's bytes, nv of them in the read; kFull:
// all 16): the bytes' mismatches against "ACTG"[code] ORed into bad (a
// mismatch outside bit 5, the case bit, is a byte outside ACGTacgt), the
// read-major word, and the weighted 8-base sums into the fingerprint
// accumulators.  Each 8-base sum is below 2^22 and each weight below 2^29; a
// read adds at most 64 products.
template <bool kFull>
EMP_DEV void read_chunk(const uint32_t x[4], int nv, const uint32_t *kc, uint32_t &bad, uint32_t &word, uint64_t &f1,
                        uint64_t &f2, uint64_t &g1, uint64_t &g2) {
    uint32_t e[4], ec[4], p[4];
    const uint32_t s8 = (uint32_t)(nv > 16 ? 16 : nv) * 8u;  // valid bits of the chunk
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint32_t vm = kFull ? 0xffffffffu : __funnelshift_lc(0xffffffffu, 0u, s8 > 32u * q ? s8 - 32u * q : 0u);
        const uint32_t c = (x[q] >> 1) & 0x03030303u;
        const uint32_t want = __byte_perm(0x47544341u, 0u, __byte_perm(c | (c >> 4), 0u, 0x4420u));  // "ACTG"[code]
        bad |= kFull ? x[q] ^ want : (x[q] ^ want) & vm;
        const uint32_t cq = c & vm;  // A0 C1 T2 G3
        e[q] = kFull ? cq + 0x01010101u : (cq + 0x01010101u) & vm;
        ec[q] = kFull ? (cq ^ 0x02020202u) + 0x01010101u : ((cq ^ 0x02020202u) + 0x01010101u) & vm;
        p[q] = cq * 0x01041040u;  // byte 3: the four codes, 2 bits each, first lowest
    }
    word = __byte_perm(__byte_perm(p[0], p[1], 0x0073u), __byte_perm(p[2], p[3], 0x0073u), 0x5410u);
    f1 += (uint64_t)fw1(e[1], fw1(e[0], 0u) * 625u) * kc[0];
    f1 += (uint64_t)fw1(e[3], fw1(e[2], 0u) * 625u) * kc[1];
    f2 += (uint64_t)fw2(e[1], fw2(e[0], 0u) * 2401u) * kc[2];
    f2 += (uint64_t)fw2(e[3], fw2(e[2], 0u) * 2401u) * kc[3];
    g1 += (uint64_t)rc1(ec[0], rc1(ec[1], 0u) * 625u) * kc[4];
    g1 += (uint64_t)rc1(ec[2], rc1(ec[3], 0u) * 625u) * kc[5];
    g2 += (uint64_t)rc2(ec[0], rc2(ec[1], 0u) * 2401u) * kc[6];
    g2 += (uint64_t)rc2(ec[2], rc2(ec[3], 0u) * 2401u) * kc[7];
}

// The window of tile `tile` into dst: thread 0 starts one bulk copy of the
// input's whole 16-byte blocks (completing on bar); the bytes after them up
// to kWin (the input's last partial block, then zeros) are written by all
// threads.  Called by every thread of the CTA.
EMP_DEV void stage_window(const uint8_t *fq, uint64_t F, uint64_t tile, uint32_t *dst, uint64_t *bar) {
    const uint64_t T0 = tile * kParseTile, avail = F - T0;  // tile < parse_tiles(F): avail >= 1
    const uint32_t nbulk = (uint32_t)(avail < kWin ? avail : kWin) & ~15u;
    if (threadIdx.x == 0) {
        fence_proxy_async();  // the buffer's last reads (generic) before the copy's writes
        if (nbulk) bulk_load(dst, fq + T0, nbulk, bar);
        else mbar_arrive(bar);
    }
    for (uint32_t w = nbulk / 4 + threadIdx.x; w < kWinWords; w += kRT) {  // only near the input's end
        uint32_t v = 0;
        for (uint32_t b = 0; b < 4; ++b)
            if (4ull * w + b < avail) v |= (uint32_t)fq[T0 + 4ull * w + b] << (8 * b);
        dst[w] = v;
    }
}

__global__ void __launch_bounds__(kRT, 4) read_pass_kernel(const uint8_t *__restrict__ fq, uint64_t F,
                                                        const uint64_t *__restrict__ tile_excl,
                                                        const HashTables *__restrict__ tables,
                                                        const ChunkWeights *__restrict__ weights,
                                                        uint64_t *__restrict__ keys, uint32_t *__restrict__ seq2,
                                                        int wpr, uint32_t *__restrict__ keep_out, uint64_t *n_kept,
                                                        uint32_t *len_minmax, uint32_t *err) {
    extern __shared__ __align__(16) uint8_t read_smem[];
    ReadSmem &sm = *reinterpret_cast<ReadSmem *>(read_smem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < kChunks * 8; i += kRT) sm.chunk[i >> 3][i & 7] = weights->w[i >> 3][i & 7];
    for (int i = tid; i < (int)kRecCap; i += kRT) sm.end[i] = kNoEnd;  // each use resets its slots
    if (tid < 16) sm.win[tid >> 3][kWinWords + (tid & 7)] = 0;
    if (tid == 0) {
        mbar_init(&sm.bar[0], 1);
        mbar_init(&sm.bar[1], 1);
        fence_proxy_async();
    }
    __syncthreads();
    const uint64_t ntiles = parse_tiles(F);
    uint32_t lmin = 0xffffffffu, lmax = 0u, bad_kept = 0u, kept = 0u;
    if (blockIdx.x < ntiles) stage_window(fq, F, blockIdx.x, sm.win[0], &sm.bar[0]);
    int buf = 0;
    uint32_t parity = 0;  // bit b: the phase buffer b's barrier completes next
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, buf ^= 1) {
        const uint64_t T0 = tile * kParseTile;
        const bool win_eof = T0 + kWin >= F;  // the window holds the rest of the input
        const uint64_t E = tile_excl[tile];   // newlines before the tile
        const bool arrived = mbar_wait(&sm.bar[buf], (parity >> buf) & 1u, kSpinLimit);
        parity ^= 1u << buf;
        if (__syncthreads_or(!arrived)) {  // a copy that never lands: report it, give it one more wait
            if (tid == 0) {
                atomicOr(err, kErrSpin);
                mbar_wait(&sm.bar[buf], (parity >> buf) & 1u ^ 1u, kSpinLimit);
            }
            return;
        }
        if (tile + gridDim.x < ntiles) stage_window(fq, F, tile + gridDim.x, sm.win[buf ^ 1], &sm.bar[buf ^ 1]);
        const uint32_t *win = sm.win[buf];
        // ---- locate.  Thread t holds tile bytes [64t, 64t + 64) (four 16-byte
        // chunks, read in an order rotated by t so that a quarter-warp's
        // shared-memory reads spread over the banks) and, for t < 33, halo chunk
        // t.  Newline masks in byte order (one bit per byte), their counts, one
        // block scan of (tile count | halo count << 16): no carries (16384, 528).
        uint64_t m64 = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t q = (uint32_t)(k + tid) & 3u;
            m64 |= (uint64_t)nl_mask16(*reinterpret_cast<const uint4 *>(win + 16 * tid + 4 * q)) << (16 * q);
        }
        const uint32_t mh =
            tid < (int)(kHalo / 16) ? nl_mask16(*reinterpret_cast<const uint4 *>(win + kParseTile / 4 + 4 * tid)) : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan<kRT, uint32_t>((uint32_t)__popcll(m64) | ((uint32_t)__popc(mh) << 16),
                                                                sm.scan32, &tot);
        const uint32_t tile_nl = tot & 0xffffu;
        const uint64_t k0 = (E + 3) >> 2, k1 = (E + tile_nl + 3) >> 2;
        const uint32_t n_own = (uint32_t)(k1 - k0);
        // Newline j of the window (j = 0, 1, .. from the tile's start) ends line
        // E + j; with e3 = E & 3 it is newline (e3 + j) & 3 of record
        // (E >> 2) + ((e3 + j) >> 2), the tile's record ((e3 + j) >> 2) - adj.
        const uint32_t e3 = (uint32_t)E & 3u, adj = e3 ? 1u : 0u;
        for (uint32_t b0 = 0; b0 < n_own; b0 += kRecCap) {  // records in batches of kRecCap (one, but for tiny reads)
            const uint32_t nb = n_own - b0 < kRecCap ? n_own - b0 : kRecCap;
            uint32_t j = e3 + (ex & 0xffffu);  // e3 + the index of the thread's first newline
            for (uint64_t m = m64; m;) {
                const uint32_t pos = 64u * tid + (uint32_t)(__ffsll(m) - 1);
                m &= m - 1;
                const uint32_t slot = (j >> 2) - adj - b0, r4 = j & 3u;
                if ((j >> 2) >= adj + b0 && slot < nb) {
                    if (r4 == 0) sm.start[slot] = (uint16_t)(pos + 1);
                    else if (r4 == 1) sm.end[slot] = (uint16_t)pos;
                }
                ++j;
            }
            j = e3 + tile_nl + (ex >> 16);  // the halo: only sequence ends matter there
            for (uint32_t m = mh; m;) {
                const uint32_t pos = (uint32_t)kParseTile + 16u * tid + (uint32_t)(__ffs(m) - 1);
                m &= m - 1;
                const uint32_t slot = (j >> 2) - adj - b0;
                if ((j & 3u) == 1u && (j >> 2) >= adj + b0 && slot < nb) sm.end[slot] = (uint16_t)pos;
                ++j;
            }
            __syncthreads();
            // ---- records: G lanes each
            const int G = nb > 128 ? 1 : nb > 64 ? 2 : nb > 32 ? 4 : nb > 16 ? 8 : 16;
            const uint32_t lg = (uint32_t)tid & (G - 1), grp = (uint32_t)tid / G, ngrp = kRT / G;
            const uint32_t gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << (lane & ~(G - 1));
            for (uint32_t r0 = 0; r0 < nb; r0 += ngrp) {
                const uint32_t r = r0 + grp;
                const bool own = r < nb;
                uint32_t a = 0, b = 0;
                bool in_win = false;
                if (own) {
                    a = sm.start[r];
                    b = sm.end[r];
                    in_win = b != kNoEnd || win_eof;
                    if (b == kNoEnd && win_eof) b = (uint32_t)(F - T0);
                }
                const uint32_t L = in_win ? b - a : 0u;
                const bool hashed = own && L >= 1 && L <= (uint32_t)kMaxReadLen;
                const uint64_t k = k0 + b0 + r;
                const uint32_t nch = (L + 15) / 16;
                const uint32_t lim = own ? (nch > (uint32_t)wpr ? nch : (uint32_t)wpr) : 0u;  // words up to wpr
                uint32_t bad = 0;
                uint64_t f1 = 0, f2 = 0, g1 = 0, g2 = 0;
                // warp-uniform trips, so that a warp whose chunks are all whole
                // takes the unmasked path together
                const uint32_t trips = __reduce_max_sync(0xffffffffu, (lim + G - 1) / G);
                for (uint32_t it = 0; it < trips; ++it) {
                    const uint32_t c = lg + it * G;
                    const bool has = c < nch;
                    const int nv = (int)(L - 16 * c);
                    const bool whole = __all_sync(0xffffffffu, !has || !hashed || nv >= 16);
                    uint32_t word = 0;
                    if (has) {
                        uint32_t xw[4];
                        win16(win, a + 16 * c, xw);
                        if (!hashed) {
#pragma unroll
                            for (int q = 0; q < 4; ++q) bad |= not_acgt(xw[q], lead_bytes(nv - 4 * q));
                        } else if (whole) {
                            read_chunk<true>(xw, nv, sm.chunk[c], bad, word, f1, f2, g1, g2);
                        } else {
                            read_chunk<false>(xw, nv, sm.chunk[c], bad, word, f1, f2, g1, g2);
                        }
                    }
                    if (c < lim && c < (uint32_t)wpr) seq2[k * (uint64_t)wpr + c] = word;
                }
                bad &= 0xdfdfdfdfu;
                const bool gbad = (__ballot_sync(0xffffffffu, bad != 0) & gmask) != 0;
                uint32_t nm = 0;
                if (__any_sync(0xffffffffu, gbad) && gbad) {  // rare: are the odd bytes N-class?
                    for (uint32_t c = lg; c < nch; c += G) {
                        uint32_t xw[4];
                        win16(win, a + 16 * c, xw);
                        const int nv = (int)(L - 16 * c);
#pragma unroll
                        for (int q = 0; q < 4; ++q) nm |= n_class(xw[q], lead_bytes(nv - 4 * q));
                    }
                }
                const bool gn = (__ballot_sync(0xffffffffu, nm != 0) & gmask) != 0;
                for (int o = G >> 1; o; o >>= 1) {
                    f1 += __shfl_xor_sync(0xffffffffu, f1, o);
                    f2 += __shfl_xor_sync(0xffffffffu, f2, o);
                    g1 += __shfl_xor_sync(0xffffffffu, g1, o);
                    g2 += __shfl_xor_sync(0xffffffffu, g2, o);
                }
                if (own && lg == 0) {
                    sm.end[r] = kNoEnd;  // every lane of the group has read it
                    bool keep, bd;
                    uint64_t len;
                    if (in_win) {
                        keep = !gn && L > 0;
                        bd = gbad;
                        len = L;
                    } else {  // the line runs past the window: one lane walks it in global memory
                        const uint64_t p0 = T0 + a;
                        uint64_t p = p0;
                        bool hn = false;
                        bd = false;
                        for (; p < F; ++p) {
                            const uint32_t c8 = fq[p];
                            if (c8 == 0x0au) break;
                            hn |= n_class(c8, 0xffu) != 0;
                            bd |= not_acgt(c8, 0xffu) != 0;
                        }
                        len = p - p0;
                        keep = !hn && len > 0;
                    }
                    keep_out[k] = keep ? 1u : 0u;
                    if (keep) {
                        const uint32_t l32 = len > 0xffffffffull ? 0xffffffffu : (uint32_t)len;
                        lmin = min(lmin, l32);
                        lmax = max(lmax, l32);
                        bad_kept |= bd ? 1u : 0u;
                        ++kept;
                    }
                }
                if (hashed && !gn) {  // kept: its four residues, one lane each (f = lg, lg + G, ..)
                    uint32_t *kw = reinterpret_cast<uint32_t *>(keys + 2 * k);
                    for (uint32_t f = lg; f < 4; f += G) {
                        const bool p2 = (f & 1u) != 0;  // f: 0 fp1, 1 fp2 of the read; 2, 3 of its complement
                        const uint64_t sum = f == 0 ? f1 : f == 1 ? f2 : f == 2 ? g1 : g2;
                        const uint32_t C = p2 ? kP2C : kP1C, P = p2 ? kP2 : kP1;
                        const uint32_t pw = f < 2 ? __ldg((p2 ? tables->pow2 : tables->pow1) + L - 1) : 1u;
                        kw[f ^ 1u] = mod_rt((uint64_t)mod_rt(sum, C, P) * pw, C, P);  // key = fp1 << 32 | fp2
                    }
                }
            }
            __syncthreads();  // start / end (and, after the last batch, the window) are reused
        }
    }
    // kept count, length extremes of the kept reads, the bad-base flag
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        kept += __shfl_xor_sync(0xffffffffu, kept, o);
        lmin = min(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
        lmax = max(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    }
    const bool anybad = __any_sync(0xffffffffu, bad_kept != 0);
    if (lane == 0) {
        if (kept) atomicAdd(reinterpret_cast<unsigned long long *>(n_kept), (unsigned long long)kept);
        if (lmax) {
            atomicMin(len_minmax, lmin);
            atomicMax(len_minmax + 1, lmax);
        }
        if (anybad) atomicOr(err, kErrBadBase);
    }
}

// Kept records to consecutive indices: pos = exclusive scan of keep (a
// record is kept iff pos[k+1] > pos[k], the last one iff its pos < n_kept).
__global__ void __launch_bounds__(256) compact_reads_kernel(const uint32_t *__restrict__ pos, uint64_t n_rec,
                                                            uint64_t n_kept, const uint64_t *__restrict__ keys,
                                                            const uint32_t *__restrict__ seq2, int wpr,
                                                            uint64_t *__restrict__ keys_out,
                                                            uint32_t *__restrict__ seq2_out) {
    for (uint64_t k = (uint64_t)blockIdx.x * 256 + threadIdx.x; k < n_rec; k += (uint64_t)gridDim.x * 256) {
        const uint32_t i = pos[k];
        const uint64_t nxt = k + 1 < n_rec ? pos[k + 1] : n_kept;
        if (nxt == i) continue;
        keys_out[2ull * i] = keys[2 * k];
        keys_out[2ull * i + 1] = keys[2 * k + 1];
        for (int w = 0; w < wpr; ++w) seq2_out[(uint64_t)i * wpr + w] = seq2[k * wpr + w];
    }
}

// Read-major words of n reads (wpr per read) -> column-major words: cols[c *
// wpc + i/16] holds base c of read i at bits 2*(i%16).  One CTA per 256 reads.
__global__ void __launch_bounds__(256) columns_kernel(const uint32_t *__restrict__ seq2, uint64_t n, int L, int wpr,
                                                      uint32_t *__restrict__ cols, uint64_t wpc) {
    extern __shared__ uint32_t s_rows[];  // [256][wpr | 1]
    const int stride = wpr | 1;
    const uint64_t i0 = (uint64_t)blockIdx.x * 256;
    const uint32_t nr = n - i0 < 256 ? (uint32_t)(n - i0) : 256u;
    for (uint32_t q = threadIdx.x; q < 256u * (uint32_t)wpr; q += 256) {
        const uint32_t rr = q / (uint32_t)wpr, w = q - rr * (uint32_t)wpr;
        s_rows[rr * stride + w] = rr < nr ? seq2[(i0 + rr) * wpr + w] : 0u;
    }
    __syncthreads();
    const uint64_t w0 = i0 >> 4;
    for (uint32_t p = threadIdx.x; p < (uint32_t)L * 16u; p += 256) {
        const uint32_t col = p >> 4, wl = p & 15u;
        if (w0 + wl >= wpc) continue;
        uint32_t word = 0;
#pragma unroll
        for (int m = 0; m < 16; ++m)
            word |= ((s_rows[(16 * wl + m) * stride + (col >> 4)] >> (2 * (col & 15u))) & 3u) << (2 * m);
        cols[(uint64_t)col * wpc + w0 + wl] = word;
    }
}

static unsigned grid_for(uint64_t work, unsigned per_block, unsigned cap) {
    uint64_t g = (work + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

void launch_nl_count(const uint8_t *fq, uint64_t F, uint32_t *tile_counts, uint64_t *len0, cudaStream_t s) {
    if (!F) return;
    count_launch();
    nl_count_kernel<<<(unsigned)parse_tiles(F), 256, 0, s>>>(fq, F, tile_counts, len0);
}

void launch_read_pass(const uint8_t *fq, uint64_t F, const uint64_t *tile_excl, const HashTables *tables,
                      const ChunkWeights *weights, uint64_t *keys, uint32_t *seq2, int wpr, uint32_t *keep, uint64_t *n_kept, uint32_t *len_minmax,
                      uint32_t *err, cudaStream_t s) {
    if (!F) return;
    // persistent grid (SMs x resident CTAs) and the shared-memory attribute, once per device
    constexpr int kDevs = 64;
    static std::atomic<int> grid[kDevs] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) {
        cudaGetLastError();
        dev = 0;
    }
    int g = grid[dev].load(std::memory_order_acquire);
    if (!g) {
        int sms = 148, occ = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(read_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(ReadSmem));
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, read_pass_kernel, kRT, sizeof(ReadSmem)) !=
                cudaSuccess ||
            occ < 1)
            occ = 1;
        cudaGetLastError();
        g = sms * occ;
        grid[dev].store(g, std::memory_order_release);
    }
    count_launch();
    read_pass_kernel<<<grid_for(parse_tiles(F), 1, (unsigned)g), kRT, sizeof(ReadSmem), s>>>(
        fq, F, tile_excl, tables, weights, keys, seq2, wpr, keep, n_kept, len_minmax, err);
}

void launch_compact_reads(const uint32_t *pos, uint64_t n_rec, uint64_t n_kept, const uint64_t *keys,
                          const uint32_t *seq2, int wpr, uint64_t *keys_out, uint32_t *seq2_out, cudaStream_t s) {
    if (!n_rec) return;
    count_launch();
    compact_reads_kernel<<<grid_for(n_rec, 256, 148 * 16), 256, 0, s>>>(pos, n_rec, n_kept, keys, seq2, wpr, keys_out,
                                                                      seq2_out);
}

void launch_columns(const uint32_t *seq2, uint64_t n, int L, int wpr, uint32_t *cols, uint64_t wpc, cudaStream_t s) {
    if (!n) return;
    count_launch();
    const size_t smem = 256u * (size_t)(wpr | 1) * 4u;
    columns_kernel<<<(unsigned)((n + 255) / 256), 256, smem, s>>>(seq2, n, L, wpr, cols, wpc);
}

}  // namespace emp
