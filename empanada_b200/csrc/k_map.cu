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
//   nl_locate     global line id of every newline -> start/end of each
//                 record's sequence line
//   read_hash     one thread per record: N filter, ACGT check, length, both
//                 fingerprints and the read-major 2-bit words in one walk
//                 over the sequence line; kept reads get their index from a
//                 decoupled look-back over the tiles' kept counts
//   columns       read-major words -> column-major words (only when needed)
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

// Newline g ends line g.  Line 4k+1 is record k's sequence: it starts after
// newline 4k and ends at newline 4k+1.  Thread t of a tile takes its 64
// consecutive bytes (4 x 16-byte loads): one CTA scan of the per-thread
// newline counts gives each thread the line id of its first newline.
__global__ void __launch_bounds__(256) nl_locate_kernel(const uint8_t *__restrict__ fq, uint64_t F,
                                                        const uint64_t *__restrict__ tile_excl,
                                                        uint64_t *__restrict__ seq_start,
                                                        uint64_t *__restrict__ seq_end) {
    __shared__ uint32_t s_warp[8];
    const uint64_t base = (uint64_t)blockIdx.x * kParseTile + (uint64_t)threadIdx.x * 64;
    uint32_t w[16];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint64_t off = base + 16 * k;
        if (off + 16 <= F) {
            const uint4 v = __ldg(reinterpret_cast<const uint4 *>(fq + off));
            w[4 * k] = v.x;
            w[4 * k + 1] = v.y;
            w[4 * k + 2] = v.z;
            w[4 * k + 3] = v.w;
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) w[4 * k + q] = 0;
            for (int bb = 0; bb < 16; ++bb)
                if (off + bb < F) w[4 * k + (bb >> 2)] |= (uint32_t)fq[off + bb] << (8 * (bb & 3));
        }
    }
    uint32_t cnt = 0;
#pragma unroll
    for (int q = 0; q < 16; ++q) cnt += nl_in_word(w[q]);
    uint32_t tot;
    uint64_t my = tile_excl[blockIdx.x] + block_exclusive_scan<256, uint32_t>(cnt, s_warp, &tot);
    if (!cnt) return;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        uint32_t m = __vcmpeq4(w[q], 0x0a0a0a0au);  // 0xff in each newline byte
        while (m) {
            const int bb = (__ffs(m) - 1) >> 3;
            m &= ~(0xffu << (8 * bb));
            const uint64_t pos = base + 4 * q + bb;
            const uint32_t r = (uint32_t)(my & 3u);
            if (r == 0) seq_start[my >> 2] = pos + 1;
            else if (r == 1) seq_end[my >> 2] = pos;
            ++my;
        }
    }
}

// 0x80 in every byte of t that is zero, 0 elsewhere (no carries between bytes)
EMP_DEV uint32_t zero_bytes(uint32_t t) { return ~(((t & 0x7f7f7f7fu) + 0x7f7f7f7fu) | t | 0x7f7f7f7fu); }

// N-class bytes (markNs == 9, preprocess.cu:119-121: bits 7-6 = 01 and bit 3
// set) and bytes outside ACGTacgt among the bytes of x selected by m (0x80
// per byte)
EMP_DEV void check4(uint32_t x, uint32_t m, uint32_t &nm, uint32_t &bm) {
    const uint32_t f = x | 0x20202020u;  // case folded
    nm |= zero_bytes((x & 0xc8c8c8c8u) ^ 0x48484848u) & m;
    const uint32_t ok = zero_bytes(f ^ 0x61616161u) | zero_bytes(f ^ 0x63636363u) | zero_bytes(f ^ 0x67676767u) |
                        zero_bytes(f ^ 0x74747474u);  // a c g t
    bm |= ~ok & m;
}

// ---------------------------------------------------------------- reads
// One thread per FASTQ record, kReadTile records per tile, tiles taken in
// order from a ticket.  Per record, one walk over its sequence line in
// aligned 16-byte blocks gives
//   * the N filter and the ACGT check;
//   * both fingerprints as sums of per-word terms (the Horner form of
//     FingerprintMul expanded):
//         H(read)    = sum_t enc(b_t) R^(L-1-t)         mod P
//         H(revcomp) = sum_t enc(comp b_t) R^t          mod P
//     a memory word holding bases t .. t+3 of the read adds
//         (e0 R^3 + e1 R^2 + e2 R + e3) R^(L-4-t)  and  (e'0 + e'1 R + e'2 R^2 + e'3 R^3) R^t,
//     each below 2^41, to 64-bit sums (at most 129 words per read: below
//     2^49) that are reduced once; the words cut by the read's ends go byte
//     by byte;
//   * the read-major 2-bit words (16 bases per word, first base in bits 1-0).
// The kept records of a tile get consecutive read indices after the kept
// records of all earlier tiles (decoupled look-back on the kept count).
constexpr int kReadTile = 256;
constexpr int kSeqWordsMax = kMaxReadLen / 16;
static_assert(kMaxReadLen % 16 == 0, "whole read-major words");

__global__ void __launch_bounds__(kReadTile) read_hash_kernel(
    const uint8_t *__restrict__ fq, const uint64_t *__restrict__ seq_start, const uint64_t *__restrict__ seq_end,
    uint64_t n_rec, const HashTables *__restrict__ tables, uint64_t *__restrict__ keys, uint32_t *__restrict__ seq2,
    int wpr, uint64_t *status, uint32_t *tile_ctr, uint64_t *n_kept, uint32_t *len_minmax, uint32_t *err) {
    __shared__ uint32_t s_pow1[kMaxReadLen + 1], s_pow2[kMaxReadLen + 1];
    __shared__ uint32_t s_words[kSeqWordsMax][kReadTile + 1];  // [word][thread]
    __shared__ uint16_t s_who[kReadTile];                      // kept rank -> thread
    __shared__ uint32_t s_wcnt[kReadTile / 32];
    __shared__ uint32_t s_tile, s_kept;
    __shared__ uint64_t s_base;
    for (int i = threadIdx.x; i <= kMaxReadLen; i += kReadTile) {
        s_pow1[i] = tables->pow1[i];
        s_pow2[i] = tables->pow2[i];
    }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t ntiles = (n_rec + kReadTile - 1) / kReadTile;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t r = (uint64_t)tile * kReadTile + tid;
        const bool live = r < n_rec;
        const uint64_t a = live ? seq_start[r] : 0, b = live ? seq_end[r] : 0;
        const uint64_t len64 = b > a ? b - a : 0;
        const int L = len64 > (uint64_t)kMaxReadLen ? kMaxReadLen + 1 : (int)len64;  // > kMaxReadLen: not hashed
        const bool hash = L <= kMaxReadLen;
        uint32_t nm = 0, bm = 0;
        uint64_t f1 = 0, f2 = 0, g1 = 0, g2 = 0;
        uint64_t pend = 0;  // 2-bit codes of bases 16 jw .. (the words not yet emitted)
        int jw = 0;
        for (uint64_t A = a & ~15ull; A < b; A += 16) {
            const uint4 v = __ldg(reinterpret_cast<const uint4 *>(fq + A));
            const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint64_t W = A + 4 * q;
                if (W + 4 <= a || W >= b) continue;
                const uint32_t x = wv[q];
                const int t = (int)((int64_t)W - (int64_t)a);  // read position of the word's first byte
                const uint32_t c = (x >> 1) & 0x03030303u;     // base codes A0 C1 T2 G3
                if (t >= 0 && (uint64_t)W + 4 <= b) {          // the whole word lies inside the read
                    check4(x, 0x80808080u, nm, bm);
                    if (hash) {
                        const uint32_t e = c + 0x01010101u, ec = (c ^ 0x02020202u) + 0x01010101u;
                        const uint32_t h1 = __dp4a(e, 0x0105197Du, 0u);                       // 125 25 5 1
                        const uint32_t h2 = __dp4a(e, 0x01073100u, 0u) + (e & 0xffu) * 343u;  // 343 49 7 1
                        const uint32_t r1 = __dp4a(ec, 0x7D190501u, 0u);                      // 1 5 25 125
                        const uint32_t r2 = __dp4a(ec, 0x00310701u, 0u) + (ec >> 24) * 343u;  // 1 7 49 343
                        f1 += (uint64_t)h1 * s_pow1[L - 4 - t];
                        f2 += (uint64_t)h2 * s_pow2[L - 4 - t];
                        g1 += (uint64_t)r1 * s_pow1[t];
                        g2 += (uint64_t)r2 * s_pow2[t];
                    }
                } else {  // cut by an end of the read: byte by byte
                    uint32_t m = 0;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int tu = t + u;
                        if (tu < 0 || (uint64_t)(W + u) >= b) continue;
                        m |= 0x80u << (8 * u);
                        if (hash) {
                            const uint32_t cu = (c >> (8 * u)) & 3u, eu = cu + 1u, ecu = (cu ^ 2u) + 1u;
                            f1 += (uint64_t)eu * s_pow1[L - 1 - tu];
                            f2 += (uint64_t)eu * s_pow2[L - 1 - tu];
                            g1 += (uint64_t)ecu * s_pow1[tu];
                            g2 += (uint64_t)ecu * s_pow2[tu];
                        }
                    }
                    check4(x, m, nm, bm);
                }
                if (hash) {  // the word's bases into the pending 2-bit words
                    const uint32_t y = (c | (c >> 6)) & 0x000f000fu;
                    uint64_t c8 = (y & 0xfu) | ((y >> 12) & 0xf0u);  // bases t .. t+3, 2 bits each
                    if (t + 4 > L) c8 &= (1u << (2 * (L - t))) - 1u;  // past the read's end
                    if (t < 0) c8 >>= 2 * -t;
                    pend |= c8 << (2 * (t < 0 ? 0 : t - 16 * jw));
                    if (t + 4 >= 16 * (jw + 1)) {  // bases up to 16 (jw + 1) - 1 are in
                        s_words[jw][tid] = (uint32_t)pend;
                        pend >>= 32;
                        ++jw;
                    }
                }
            }
        }
        const bool keep = live && !nm && len64 > 0;
        if (hash && keep && 16 * jw < L) s_words[jw++][tid] = (uint32_t)pend;  // the last, partial word
        for (int w = hash ? jw : 0; w < wpr; ++w) s_words[w][tid] = 0;
        // ---- read indices: this tile's kept records after those of earlier tiles
        const uint32_t bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_wcnt[warp] = __popc(bal);
        __syncthreads();
        if (tid == 0) {
            uint32_t run = 0;
            for (int w = 0; w < kReadTile / 32; ++w) {
                const uint32_t c = s_wcnt[w];
                s_wcnt[w] = run;
                run += c;
            }
            s_kept = run;
            s_base = lookback_exclusive(status, tile, run, err);
            if (tile == ntiles - 1) *n_kept = s_base + run;
        }
        __syncthreads();
        const uint32_t rank = s_wcnt[warp] + __popc(bal & lanemask_lt_u32());
        const uint64_t i = s_base + rank;
        if (keep) {
            s_who[rank] = (uint16_t)tid;
            ulonglong2 kv;
            kv.x = ((uint64_t)mod1(f1) << 32) | mod2(f2);
            kv.y = ((uint64_t)mod1(g1) << 32) | mod2(g2);
            if (hash) *reinterpret_cast<ulonglong2 *>(keys + 2 * i) = kv;
            if (bm) atomicOr(err, kErrBadBase);
        }
        // length extremes of the kept reads
        uint32_t lmin = keep ? (len64 > 0xffffffffull ? 0xffffffffu : (uint32_t)len64) : 0xffffffffu;
        uint32_t lmax = keep ? lmin : 0u;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            lmin = min(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
            lmax = max(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
        }
        if (lane == 0 && lmax) {
            atomicMin(len_minmax, lmin);
            atomicMax(len_minmax + 1, lmax);
        }
        __syncthreads();
        // read-major words of the kept reads: one contiguous run of kept x wpr
        const uint32_t kept = s_kept;
        const uint64_t o0 = s_base * (uint64_t)wpr;
        for (uint32_t q = tid; q < kept * (uint32_t)wpr; q += kReadTile) {
            const uint32_t rk = q / (uint32_t)wpr, w = q - rk * (uint32_t)wpr;
            seq2[o0 + q] = s_words[w][s_who[rk]];
        }
        __syncthreads();
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

void launch_nl_locate(const uint8_t *fq, uint64_t F, const uint64_t *tile_excl, uint64_t *seq_start,
                      uint64_t *seq_end, cudaStream_t s) {
    if (!F) return;
    count_launch();
    nl_locate_kernel<<<(unsigned)parse_tiles(F), 256, 0, s>>>(fq, F, tile_excl, seq_start, seq_end);
}

void launch_read_hash(const uint8_t *fq, const uint64_t *seq_start, const uint64_t *seq_end, uint64_t n_rec,
                      const HashTables *tables, uint64_t *keys, uint32_t *seq2, int wpr, uint64_t *status,
                      uint32_t *tile_ctr, uint64_t *n_kept, uint32_t *len_minmax, uint32_t *err, cudaStream_t s) {
    if (!n_rec) return;
    static int grid = 0;  // persistent: SMs x resident CTAs (the same on every B200)
    if (!grid) {
        int dev = 0, sms = 148, occ = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, read_hash_kernel, kReadTile, 0) != cudaSuccess ||
            occ < 1)
            occ = 1;
        cudaGetLastError();
        grid = sms * occ;
    }
    const uint64_t tiles = (n_rec + kReadTile - 1) / kReadTile;
    count_launch();
    read_hash_kernel<<<grid_for(tiles, 1, (unsigned)grid), kReadTile, 0, s>>>(
        fq, seq_start, seq_end, n_rec, tables, keys, seq2, wpr, status, tile_ctr, n_kept, len_minmax, err);
}

void launch_columns(const uint32_t *seq2, uint64_t n, int L, int wpr, uint32_t *cols, uint64_t wpc, cudaStream_t s) {
    if (!n) return;
    count_launch();
    const size_t smem = 256u * (size_t)(wpr | 1) * 4u;
    columns_kernel<<<(unsigned)((n + 255) / 256), 256, smem, s>>>(seq2, n, L, wpr, cols, wpc);
}

}  // namespace emp
