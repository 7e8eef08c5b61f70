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
//   classify      one warp per record: N filter, ACGT check, length
//   scatter_hq    kept read i -> record index
//   fingerprint_pack
//                 one warp per read: lane-chunk Horner hashes of the read and
//                 of its reverse complement, combined with R^k from shared
//                 memory; the CTA then writes 128 reads x L columns of 2-bit
//                 codes as whole 32-byte column segments.
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
// newline 4k and ends at newline 4k+1.
__global__ void __launch_bounds__(256) nl_locate_kernel(const uint8_t *__restrict__ fq, uint64_t F,
                                                        const uint64_t *__restrict__ tile_excl,
                                                        uint64_t *__restrict__ seq_start,
                                                        uint64_t *__restrict__ seq_end) {
    __shared__ uint32_t s_warp[8];
    const uint64_t base = (uint64_t)blockIdx.x * kParseTile;
    uint64_t g = tile_excl[blockIdx.x];
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
        const uint64_t off = base + ((uint64_t)k * 256 + threadIdx.x) * 16;
        uint32_t w[4] = {0, 0, 0, 0};
        if (off + 16 <= F) {
            uint4 v = *reinterpret_cast<const uint4 *>(fq + off);
            w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
        } else {
            for (int b = 0; b < 16; ++b)
                if (off + b < F) w[b >> 2] |= (uint32_t)fq[off + b] << (8 * (b & 3));
        }
        uint32_t cnt = nl_in_word(w[0]) + nl_in_word(w[1]) + nl_in_word(w[2]) + nl_in_word(w[3]);
        uint32_t tot;
        uint64_t my = g + block_exclusive_scan<256, uint32_t>(cnt, s_warp, &tot);
        if (cnt) {
#pragma unroll
            for (int b = 0; b < 16; ++b) {
                if (((w[b >> 2] >> (8 * (b & 3))) & 0xffu) == '\n') {
                    const uint64_t pos = off + b;
                    const uint32_t r = (uint32_t)(my & 3u);
                    if (r == 0) seq_start[my >> 2] = pos + 1;
                    else if (r == 1) seq_end[my >> 2] = pos;
                    ++my;
                }
            }
        }
        g += tot;
    }
}

__global__ void __launch_bounds__(256) classify_kernel(const uint8_t *__restrict__ fq,
                                                       const uint64_t *__restrict__ seq_start,
                                                       const uint64_t *__restrict__ seq_end, uint64_t n_rec,
                                                       uint32_t *__restrict__ hq, uint32_t *len_minmax,
                                                       uint32_t *err) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t lmin = 0xffffffffu, lmax = 0, bad_any = 0;
    for (uint64_t k = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < n_rec; k += warps) {
        const uint64_t a = seq_start[k], b = seq_end[k];
        const uint64_t len = b > a ? b - a : 0;
        bool has_n = false, bad = false;
        for (uint64_t o = a + lane; o < b; o += 32) {
            const uint8_t c = fq[o];
            has_n |= is_n_class(c);
            bad |= !is_acgt(c);
        }
        has_n = __any_sync(0xffffffffu, has_n);
        bad = __any_sync(0xffffffffu, bad);
        const bool keep = !has_n && len > 0;
        if (lane == 0) hq[k] = keep ? 1u : 0u;
        if (keep) {
            const uint32_t l32 = len > 0xffffffffull ? 0xffffffffu : (uint32_t)len;
            lmin = min(lmin, l32);
            lmax = max(lmax, l32);
            bad_any |= bad ? 1u : 0u;
        }
    }
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

// PER: bases per lane at most (L <= 32 PER); READS reads per CTA (8 warps,
// READS / 8 reads each), their 2-bit codes staged in a READS x 32 PER tile.
template <int PER, int READS>
__global__ void __launch_bounds__(256) fingerprint_pack_kernel(const uint8_t *__restrict__ fq,
                                                               const uint64_t *__restrict__ seq_start,
                                                               const uint32_t *__restrict__ rec_of, uint64_t n,
                                                               int L, const HashTables *__restrict__ tables,
                                                               uint64_t *__restrict__ keys,
                                                               uint32_t *__restrict__ cols, uint64_t wpc,
                                                               uint32_t *__restrict__ seq2, int wpr) {
    __shared__ uint32_t s_pow1[kMaxReadLen + 1], s_pow2[kMaxReadLen + 1];
    constexpr int kFpRow = 32 * PER, kRowsPerWarp = READS / 8, kGroups = READS / 16;
    __shared__ uint8_t s_codes[READS * kFpRow];
    for (int i = threadIdx.x; i <= kMaxReadLen; i += blockDim.x) {
        s_pow1[i] = tables->pow1[i];
        s_pow2[i] = tables->pow2[i];
    }
    __syncthreads();
    const uint64_t i0 = (uint64_t)blockIdx.x * READS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = (L + 31) >> 5;  // bases per lane, <= PER
    const int a = min(lane * per, L), b = min(a + per, L);
    for (int m = 0; m < kRowsPerWarp; ++m) {
        const int row = warp * kRowsPerWarp + m;
        const uint64_t i = i0 + row;
        if (i >= n) break;
        const uint8_t *s = fq + seq_start[rec_of[i]];
        uint32_t cod[PER];
        uint32_t hf1 = 0, hf2 = 0, hr1 = 0, hr2 = 0;
#pragma unroll
        for (int jj = 0; jj < PER; ++jj) {
            const int j = a + jj;
            cod[jj] = 0;
            if (j < b) {
                const uint32_t v = base_code(s[j]);
                cod[jj] = v;
                s_codes[row * kFpRow + j] = (uint8_t)v;
                hf1 = horner1(hf1, v + 1);
                hf2 = horner2(hf2, v + 1);
            }
        }
#pragma unroll
        for (int jj = PER - 1; jj >= 0; --jj) {
            if (a + jj < b) {
                const uint32_t e = (cod[jj] ^ 2u) + 1u;  // complement
                hr1 = horner1(hr1, e);
                hr2 = horner2(hr2, e);
            }
        }
        uint64_t f1 = 0, f2 = 0, r1 = 0, r2 = 0;
        if (a < b) {
            f1 = mod1((uint64_t)hf1 * s_pow1[L - b]);
            f2 = mod2((uint64_t)hf2 * s_pow2[L - b]);
            r1 = mod1((uint64_t)hr1 * s_pow1[a]);
            r2 = mod2((uint64_t)hr2 * s_pow2[a]);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            f1 += __shfl_xor_sync(0xffffffffu, f1, o);
            f2 += __shfl_xor_sync(0xffffffffu, f2, o);
            r1 += __shfl_xor_sync(0xffffffffu, r1, o);
            r2 += __shfl_xor_sync(0xffffffffu, r2, o);
        }
        if (lane == 0) {
            ulonglong2 kv;
            kv.x = ((uint64_t)mod1(f1) << 32) | mod2(f2);
            kv.y = ((uint64_t)mod1(r1) << 32) | mod2(r2);
            *reinterpret_cast<ulonglong2 *>(keys + 2 * i) = kv;
        }
    }
    __syncthreads();
    const uint64_t w0 = i0 >> 4;
    for (int p = threadIdx.x; p < L * kGroups; p += blockDim.x) {
        const int col = p / kGroups, q = p % kGroups;
        if (w0 + q >= wpc) continue;
        uint32_t word = 0;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int row = q * 16 + m;
            if (i0 + row < n) word |= (uint32_t)s_codes[row * kFpRow + col] << (2 * m);
        }
        cols[(uint64_t)col * wpc + w0 + q] = word;
    }
    if (!seq2) return;
    // read-major copy: word w of read i holds positions 16w .. 16w+15
    for (int p = threadIdx.x; p < READS * wpr; p += blockDim.x) {
        const int row = p / wpr, w = p - row * wpr;
        if (i0 + row >= n) break;
        uint32_t word = 0;
        for (int m = 0; m < 16 && 16 * w + m < L; ++m)
            word |= (uint32_t)s_codes[row * kFpRow + 16 * w + m] << (2 * m);
        seq2[(i0 + row) * wpr + w] = word;
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
    classify_kernel<<<grid_for(n_rec, 8, 148 * 16), 256, 0, s>>>(fq, seq_start, seq_end, n_rec, hq, len_minmax,
                                                                   err);
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
    if (L <= 256) {
        fingerprint_pack_kernel<8, 128><<<(unsigned)((n + 127) / 128), 256, 0, s>>>(fq, seq_start, rec_of, n, L, tables,
                                                                                 keys, cols, wpc, seq2, wpr);
    } else {
        static_assert(kMaxReadLen <= 512, "16 bases per lane");
        fingerprint_pack_kernel<16, 64><<<(unsigned)((n + 63) / 64), 256, 0, s>>>(fq, seq_start, rec_of, n, L, tables,
                                                                               keys, cols, wpc, seq2, wpr);
    }
}

}  // namespace emp
