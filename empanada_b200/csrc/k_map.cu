// k_map.cu -- map phase: FASTQ bytes in HBM -> kept reads -> fingerprints of
// every read-end + 2-bit column-major ("transposed") base store.
//
// Reference behaviour restated (file:line in the reference project):
//   line ids / sequence lines   preprocess.cu:26-37, 70-87 (line g%4 == 1)
//   N filter                    preprocess.cu:98-182 (markNs == 9 drops the read)
//   equal read length           fingerprint.cu:125-153 (transpose_reads)
//   read-end ids                fingerprint.cu:75-115 (rid = 2i fwd, 2i+1 RC)
//   fingerprints                fingerprint.cu:36-65 (Horner form of FingerprintMul)
//   transposed bases            fingerprint.cu:125-153, blocks.cuh:11-128
//
// Kernels
//   nl_count      newline count of each 16 KB tile (16-byte vector loads)
//   nl_locate     global line id of every newline -> start/end of each
//                 record's sequence line
//   classify      one warp per record, lane j taking bytes 16j..16j+15 of the
//                 sequence line (aligned 16-byte loads, neighbours shared by
//                 shuffle): N filter, ACGT check, length
//   scatter_hq    kept read i -> record index
//   fingerprint_pack
//                 one warp per read (two per warp-iteration when L <= 256),
//                 lane j taking bases 16j..16j+15: Horner hashes of its chunk
//                 for the read and its reverse complement, combined with R^k
//                 from shared memory; the chunk is also the read-major 2-bit
//                 word j, and each lane gathers its 16 column words of the
//                 warp's 16 reads in registers; the CTA writes 128 reads x L
//                 columns as whole 32-byte column segments.
#include "kernels.h"

namespace emp {

EMP_DEV uint32_t nl_in_word(uint32_t w) { return __popc(__vcmpeq4(w, 0x0a0a0a0au)) >> 3; }

__global__ void __launch_bounds__(256) nl_count_kernel(const uint8_t *__restrict__ fq, uint64_t F,
                                                       uint32_t *__restrict__ tile_counts) {
    __shared__ uint32_t s_warp[8];
    const uint64_t base = (uint64_t)blockIdx.x * kParseTile;
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint64_t off = base + ((uint64_t)k * 256 + threadIdx.x) * 16;
        if (off + 16 <= F) {
            uint4 w = *reinterpret_cast<const uint4 *>(fq + off);
            c += nl_in_word(w.x) + nl_in_word(w.y) + nl_in_word(w.z) + nl_in_word(w.w);
        } else {
            for (int b = 0; b < 16; ++b)
                if (off + b < F && fq[off + b] == '\n') ++c;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < 8; ++w) t += s_warp[w];
        tile_counts[blockIdx.x] = t;
    }
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

// Bytes [s, s + 16) of the FASTQ (only those below `end` are meaningful),
// for a group of consecutive lanes whose starts s differ by 16 from lane to
// lane (lane j: s = a + 16 j): each lane loads the aligned 16 bytes at or
// before s, takes the following aligned 16 from the next lane (the group's
// last lane, `last`, loads them), and funnels.  Every lane of the warp must
// call it.  Loads touch only 16-byte blocks that hold a byte below `end` (the
// buffer starts 16-byte aligned and holds 16 bytes of slack past the data).
EMP_DEV void load16(const uint8_t *__restrict__ fq, uint64_t s, uint64_t end, bool last, uint32_t w[4]) {
    const uint64_t A = s & ~15ull;
    const uint32_t o = (uint32_t)(s & 15ull);  // the same in every lane
    uint4 c0 = make_uint4(0, 0, 0, 0), c1;
    if (A < end) c0 = *reinterpret_cast<const uint4 *>(fq + A);
    c1.x = __shfl_down_sync(0xffffffffu, c0.x, 1);
    c1.y = __shfl_down_sync(0xffffffffu, c0.y, 1);
    c1.z = __shfl_down_sync(0xffffffffu, c0.z, 1);
    c1.w = __shfl_down_sync(0xffffffffu, c0.w, 1);
    if (last) {  // the block after the group's last lane's
        c1 = make_uint4(0, 0, 0, 0);
        if (o && A + 16 < end) c1 = *reinterpret_cast<const uint4 *>(fq + A + 16);
    }
    const uint32_t v[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    const uint32_t q = o >> 2, sh = (o & 3u) * 8u;
#pragma unroll
    for (int k = 0; k < 4; ++k) {  // word q + k of the pair, shifted by sh bits
        uint32_t lo = v[k], hi = v[k + 1];
        if (q == 1) { lo = v[k + 1]; hi = v[k + 2]; }
        if (q == 2) { lo = v[k + 2]; hi = v[k + 3]; }
        if (q == 3) { lo = v[k + 3]; hi = v[k + 4]; }
        w[k] = __funnelshift_r(lo, hi, sh);
    }
}
EMP_DEV uint32_t byte_of(const uint32_t w[4], int t) { return (w[t >> 2] >> (8 * (t & 3))) & 0xffu; }

// 0x80 in every byte of t that is zero, 0 elsewhere (no carries between bytes)
EMP_DEV uint32_t zero_bytes(uint32_t t) { return ~(((t & 0x7f7f7f7fu) + 0x7f7f7f7fu) | t | 0x7f7f7f7fu); }

// N-class and non-ACGT bytes among the first `valid` of w (any of each)
EMP_DEV void check16(const uint32_t w[4], int valid, bool &has_n, bool &bad) {
    uint32_t nm = 0, bm = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int vb = valid - 4 * k;
        const uint32_t m = vb >= 4 ? 0x80808080u : (vb <= 0 ? 0u : ((1u << (8 * vb)) - 1u) & 0x80808080u);
        const uint32_t x = w[k], f = x | 0x20202020u;  // case folded
        // markNs == 9 (is_n_class): bits 7-6 = 01 and bit 3 set
        nm |= zero_bytes((x & 0xc8c8c8c8u) ^ 0x48484848u) & m;
        const uint32_t ok = zero_bytes(f ^ 0x61616161u) | zero_bytes(f ^ 0x63636363u) |
                            zero_bytes(f ^ 0x67676767u) | zero_bytes(f ^ 0x74747474u);  // a c g t
        bm |= ~ok & m;
    }
    has_n |= nm != 0;
    bad |= bm != 0;
}

// One warp per 32 consecutive records: their sequence-line bounds in one
// load, then two records at a time, one per half-warp (lanes 16h + j take
// bytes 16j .. 16j+15 of record 2p + h, 256 bytes per pass), the next pair's
// first pass loaded while the current pair is checked; hq written for the 32
// at once.
__global__ void __launch_bounds__(256) classify_kernel(const uint8_t *__restrict__ fq,
                                                       const uint64_t *__restrict__ seq_start,
                                                       const uint64_t *__restrict__ seq_end, uint64_t n_rec,
                                                       uint32_t *__restrict__ hq, uint32_t *len_minmax,
                                                       uint32_t *err) {
    const uint32_t full = 0xffffffffu;
    const int lane = threadIdx.x & 31, h = lane >> 4, j = lane & 15;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t groups = (n_rec + 31) / 32;
    uint32_t lmin = 0xffffffffu, lmax = 0, bad_any = 0;
    for (uint64_t g = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < groups; g += warps) {
        const uint64_t k0 = g * 32, kl = k0 + lane;
        uint64_t ma = 0, mb = 0;
        if (kl < n_rec) {
            ma = seq_start[kl];
            mb = seq_end[kl];
        }
        const int cnt = (int)(n_rec - k0 < 32 ? n_rec - k0 : 32);
        uint32_t w[4];
        {
            const uint64_t a = __shfl_sync(full, ma, h), b = __shfl_sync(full, mb, h);
            load16(fq, a + 16 * (uint64_t)j, h < cnt ? b : 0, j == 15, w);
        }
        bool my_keep = false;
        for (int p = 0; 2 * p < cnt; ++p) {
            const int r = 2 * p + h;  // this half's record
            const bool live = r < cnt;
            const uint64_t a = __shfl_sync(full, ma, r), br = __shfl_sync(full, mb, r);  // every lane shuffles
            const uint64_t b = live ? br : 0;
            uint32_t wn[4] = {0, 0, 0, 0};
            if (2 * p + 2 < cnt) {
                const int rn = r + 2;
                const uint64_t an = __shfl_sync(full, ma, rn & 31), bn = __shfl_sync(full, mb, rn & 31);
                load16(fq, an + 16 * (uint64_t)j, rn < cnt ? bn : 0, j == 15, wn);
            }
            const uint64_t len = b > a ? b - a : 0;
            const uint32_t np = (uint32_t)((len + 255) / 256);
            const uint32_t passes = max(np, __shfl_xor_sync(full, np, 16));
            bool has_n = false, bad = false;
            for (uint32_t c0 = 0; c0 < passes; ++c0) {  // 16 chunks of 16 bytes per pass and half
                const uint64_t s = a + 256 * (uint64_t)c0 + 16 * (uint64_t)j;
                if (c0) load16(fq, s, b, j == 15, w);
                check16(w, s < b ? (int)(b - s < 16 ? b - s : 16) : 0, has_n, bad);
            }
            const uint32_t mn = __ballot_sync(full, has_n), mbad = __ballot_sync(full, bad);
            const bool hn = ((mn >> (16 * h)) & 0xffffu) != 0, hb = ((mbad >> (16 * h)) & 0xffffu) != 0;
            const bool keep = live && !hn && len > 0;
            const uint32_t kb = __ballot_sync(full, keep);
            if (lane == 2 * p) my_keep = kb & 1u;
            if (lane == 2 * p + 1) my_keep = (kb >> 16) & 1u;
            if (keep) {
                const uint32_t l32 = len > 0xffffffffull ? 0xffffffffu : (uint32_t)len;
                lmin = min(lmin, l32);
                lmax = max(lmax, l32);
                bad_any |= hb ? 1u : 0u;
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) w[k] = wn[k];
        }
        if (kl < n_rec) hq[kl] = my_keep ? 1u : 0u;
    }
    // both halves' extremes
    lmin = min(lmin, __shfl_xor_sync(full, lmin, 16));
    lmax = max(lmax, __shfl_xor_sync(full, lmax, 16));
    bad_any |= __shfl_xor_sync(full, bad_any, 16);
    if (lane == 0) {
        if (lmax) {
            atomicMin(len_minmax, lmin);
            atomicMax(len_minmax + 1, lmax);
        }
        if (bad_any) atomicOr(err, kErrBadBase);
    }
}

__global__ void scatter_hq_kernel(const uint32_t *__restrict__ hq, const uint32_t *__restrict__ idx,
                                  uint64_t n_rec, uint32_t *__restrict__ rec_of) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_rec;
         k += (uint64_t)gridDim.x * blockDim.x)
        if (hq[k]) rec_of[idx[k]] = (uint32_t)k;
}

// One warp, 16 reads of the CTA's 128 (rows warp*16 .. warp*16+15).  TWO:
// L <= 256, so the two half-warps take two reads at once (lanes 16h + j take
// chunk j of read m + h).  Lane chunk j holds bases 16j .. 16j+15.
template <bool TWO>
__global__ void __launch_bounds__(256) fingerprint_pack_kernel(const uint8_t *__restrict__ fq,
                                                               const uint64_t *__restrict__ seq_start,
                                                               const uint32_t *__restrict__ rec_of, uint64_t n,
                                                               int L, const HashTables *__restrict__ tables,
                                                               uint64_t *__restrict__ keys,
                                                               uint32_t *__restrict__ cols, uint64_t wpc,
                                                               uint32_t *__restrict__ seq2, int wpr) {
    constexpr int kReads = 128;
    __shared__ uint32_t s_pow1[kMaxReadLen + 1], s_pow2[kMaxReadLen + 1];
    __shared__ uint32_t s_colw[8][kMaxReadLen];  // [warp][column]: the warp's 16-read column words
    for (int i = threadIdx.x; i <= kMaxReadLen; i += blockDim.x) {
        s_pow1[i] = tables->pow1[i];
        s_pow2[i] = tables->pow2[i];
    }
    __syncthreads();
    const uint64_t i0 = (uint64_t)blockIdx.x * kReads;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int half = TWO ? lane >> 4 : 0;
    const int j = TWO ? lane & 15 : lane;  // the lane's chunk
    const int nch = (L + 15) >> 4;
    const bool act = j < nch;
    const int vb = act ? min(16, L - 16 * j) : 0;  // bases of the chunk
    const int q = min(16 * (j + 1), L);
    const uint32_t pf1 = s_pow1[act ? L - q : 0], pf2 = s_pow2[act ? L - q : 0];
    const uint32_t pr1 = s_pow1[act ? 16 * j : 0], pr2 = s_pow2[act ? 16 * j : 0];
    // sequence starts of the warp's 16 reads (lane m holds read m's)
    const uint64_t r0 = i0 + (uint64_t)warp * 16;
    uint64_t my_start = 0;
    if (lane < 16 && r0 + lane < n) my_start = seq_start[rec_of[r0 + lane]];
    uint32_t colw[16];
#pragma unroll
    for (int t = 0; t < 16; ++t) colw[t] = 0;
    constexpr int kStep = TWO ? 2 : 1;
    const bool last = TWO ? j == 15 : lane == 31;
    uint32_t w[4];  // the chunk of read m; the next read's is loaded while m is hashed
    {
        const uint64_t a = __shfl_sync(0xffffffffu, my_start, half);
        load16(fq, a + 16 * (uint64_t)j, r0 + half < n ? a + (uint64_t)L : 0, last, w);
    }
    for (int m0 = 0; m0 < 16; m0 += kStep) {
        const int m = m0 + half;
        const uint64_t i = r0 + m;
        const bool live = i < n;
        if (!__any_sync(0xffffffffu, live)) break;
        uint32_t wn[4] = {0, 0, 0, 0};
        if (m0 + kStep < 16) {
            const int mn = m + kStep;
            const uint64_t an = __shfl_sync(0xffffffffu, my_start, mn);
            load16(fq, an + 16 * (uint64_t)j, r0 + mn < n ? an + (uint64_t)L : 0, last, wn);
        }
        static_assert(kR1 == 5u && kR2 == 7u, "powers of the radices below");
        // four bases per step: the 4-base Horner value needs no reduction
        // (at most 4 (R^3 + R^2 + R + 1) = 1600), one fold per step
        uint32_t hf1 = 0, hf2 = 0, hr1 = 0, hr2 = 0, word = 0;
        const int vbl = live ? vb : 0;
        uint32_t cw[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) cw[k] = (w[k] >> 1) & 0x03030303u;  // base codes, one per byte
#pragma unroll
        for (int k = 0; k < 4; ++k) {  // forward, first base most significant
            const int nk = min(max(vbl - 4 * k, 0), 4);
            const uint32_t e = cw[k] + 0x01010101u;
            const uint32_t e0 = e & 0xffu, e1 = (e >> 8) & 0xffu, e2 = (e >> 16) & 0xffu, e3 = e >> 24;
            if (nk == 4) {
                hf1 = mod1((uint64_t)hf1 * 625u + (e0 * 125u + e1 * 25u + e2 * 5u + e3));
                hf2 = mod2((uint64_t)hf2 * 2401u + (e0 * 343u + e1 * 49u + e2 * 7u + e3));
            } else if (nk > 0) {  // the read's last bases
                uint32_t a1 = e0, a2 = e0, p1 = 5u, p2 = 7u;
                if (nk > 1) a1 = a1 * 5u + e1, a2 = a2 * 7u + e1, p1 = 25u, p2 = 49u;
                if (nk > 2) a1 = a1 * 5u + e2, a2 = a2 * 7u + e2, p1 = 125u, p2 = 343u;
                hf1 = mod1((uint64_t)hf1 * p1 + a1);
                hf2 = mod2((uint64_t)hf2 * p2 + a2);
            }
            uint32_t y = (cw[k] | (cw[k] >> 6)) & 0x000f000fu;  // four 2-bit codes -> 8 bits
            word |= ((y & 0xfu) | ((y >> 12) & 0xf0u)) << (8 * k);
        }
#pragma unroll
        for (int k = 3; k >= 0; --k) {  // reverse complement: sum of e'_t R^t, highest t first
            const int nk = min(max(vbl - 4 * k, 0), 4);
            const uint32_t e = (cw[k] ^ 0x02020202u) + 0x01010101u;  // complement
            const uint32_t e0 = e & 0xffu, e1 = (e >> 8) & 0xffu, e2 = (e >> 16) & 0xffu, e3 = e >> 24;
            if (nk > 0) {
                uint32_t g1 = e0, g2 = e0;
                if (nk > 1) g1 += e1 * 5u, g2 += e1 * 7u;
                if (nk > 2) g1 += e2 * 25u, g2 += e2 * 49u;
                if (nk > 3) g1 += e3 * 125u, g2 += e3 * 343u;
                hr1 = mod1((uint64_t)hr1 * 625u + g1);  // words below the top one are full
                hr2 = mod2((uint64_t)hr2 * 2401u + g2);
            }
        }
        word &= vbl >= 16 ? 0xffffffffu : (1u << (2 * vbl)) - 1u;
        uint64_t f1 = 0, f2 = 0, g1 = 0, g2 = 0;
        if (live && act) {
            f1 = mod1((uint64_t)hf1 * pf1);
            f2 = mod2((uint64_t)hf2 * pf2);
            g1 = mod1((uint64_t)hr1 * pr1);
            g2 = mod2((uint64_t)hr2 * pr2);
        }
#pragma unroll
        for (int o = TWO ? 8 : 16; o; o >>= 1) {
            f1 += __shfl_xor_sync(0xffffffffu, f1, o);
            f2 += __shfl_xor_sync(0xffffffffu, f2, o);
            g1 += __shfl_xor_sync(0xffffffffu, g1, o);
            g2 += __shfl_xor_sync(0xffffffffu, g2, o);
        }
        if (live && j == 0) {
            ulonglong2 kv;
            kv.x = ((uint64_t)mod1(f1) << 32) | mod2(f2);
            kv.y = ((uint64_t)mod1(g1) << 32) | mod2(g2);
            *reinterpret_cast<ulonglong2 *>(keys + 2 * i) = kv;
        }
        if (live && act && seq2) seq2[i * wpr + j] = word;
        if (cols) {
#pragma unroll
            for (int t = 0; t < 16; ++t) colw[t] |= ((word >> (2 * t)) & 3u) << (2 * m);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) w[k] = wn[k];
    }
    if (!cols) return;  // no column store wanted (every round runs in the bucket kernel)
    if (TWO) {  // the half-warps hold the even and odd reads' bits
#pragma unroll
        for (int t = 0; t < 16; ++t) colw[t] |= __shfl_xor_sync(0xffffffffu, colw[t], 16);
    }
    if (act && half == 0) {
#pragma unroll
        for (int t = 0; t < 16; ++t)
            if (16 * j + t < L) s_colw[warp][16 * j + t] = colw[t];
    }
    __syncthreads();
    const uint64_t w0 = i0 >> 4;
    for (int p = threadIdx.x; p < L * 8; p += blockDim.x) {
        const int col = p >> 3, qq = p & 7;
        if (w0 + qq < wpc) cols[(uint64_t)col * wpc + w0 + qq] = s_colw[qq][col];
    }
}

static unsigned grid_for(uint64_t work, unsigned per_block, unsigned cap) {
    uint64_t g = (work + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

void launch_nl_count(const uint8_t *fq, uint64_t F, uint32_t *tile_counts, cudaStream_t s) {
    if (!F) return;
    count_launch();
    nl_count_kernel<<<(unsigned)parse_tiles(F), 256, 0, s>>>(fq, F, tile_counts);
}

void launch_nl_locate(const uint8_t *fq, uint64_t F, const uint64_t *tile_excl, uint64_t *seq_start,
                      uint64_t *seq_end, cudaStream_t s) {
    if (!F) return;
    count_launch();
    nl_locate_kernel<<<(unsigned)parse_tiles(F), 256, 0, s>>>(fq, F, tile_excl, seq_start, seq_end);
}

void launch_classify(const uint8_t *fq, const uint64_t *seq_start, const uint64_t *seq_end, uint64_t n_rec,
                     uint32_t *hq, uint32_t *len_minmax, uint32_t *err, cudaStream_t s) {
    if (!n_rec) return;
    count_launch();
    classify_kernel<<<grid_for((n_rec + 31) / 32, 8, 148 * 16), 256, 0, s>>>(fq, seq_start, seq_end, n_rec, hq,
                                                                               len_minmax, err);
}

void launch_scatter_hq(const uint32_t *hq, const uint32_t *idx, uint64_t n_rec, uint32_t *rec_of, cudaStream_t s) {
    if (!n_rec) return;
    count_launch();
    scatter_hq_kernel<<<grid_for(n_rec, 256, 148 * 16), 256, 0, s>>>(hq, idx, n_rec, rec_of);
}

void launch_fingerprint_pack(const uint8_t *fq, const uint64_t *seq_start, const uint32_t *rec_of, uint64_t n,
                             int L, const HashTables *tables, uint64_t *keys, uint32_t *cols, uint64_t wpc,
                             uint32_t *seq2, int wpr, cudaStream_t s) {
    if (!n) return;
    count_launch();
    static_assert(kMaxReadLen <= 512, "32 lanes x 16 bases");
    const unsigned blocks = (unsigned)((n + 127) / 128);
    if (L <= 256)
        fingerprint_pack_kernel<true><<<blocks, 256, 0, s>>>(fq, seq_start, rec_of, n, L, tables, keys, cols, wpc, seq2,
                                                              wpr);
    else
        fingerprint_pack_kernel<false><<<blocks, 256, 0, s>>>(fq, seq_start, rec_of, n, L, tables, keys, cols, wpc,
                                                               seq2, wpr);
}

}  // namespace emp
