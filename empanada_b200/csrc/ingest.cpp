// ingest.cpp -- FASTQ input from files, produced chunk by chunk into the
// caller's (pinned) buffers: plain files (slices read by several threads at
// once), gzip (one or more members) and BGZF (blocked gzip, the blocks
// inflated in parallel on the host cores);
// several files are read in order as one FASTQ, with a newline added after a
// file that does not end with one when another file follows.
//
// The reference reads one plain file (read_block, preprocess.cu:195-237); a
// missing file reads as empty there (its ifstream), and so it does here.
#include "ingest.h"

#include <sys/stat.h>
#include <sys/types.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstring>
#include <memory>
#include <new>
#include <thread>
#include <vector>

namespace emp {

namespace {

constexpr size_t kInChunk = 4u << 20;  // compressed bytes read at a time (gzip streams)

// A BGZF block header: the gzip header with FEXTRA holding the 'BC' subfield
// (BSIZE = total block size - 1).  Returns the block size, 0 when h is not one.
size_t bgzf_block_size(const uint8_t *h, size_t n) {
    if (n < 18 || h[0] != 0x1f || h[1] != 0x8b || h[2] != 8 || !(h[3] & 4)) return 0;
    const size_t xlen = h[10] | (size_t)h[11] << 8;
    if (12 + xlen > n) return 0;
    for (size_t o = 12; o + 4 <= 12 + xlen;) {
        const size_t slen = h[o + 2] | (size_t)h[o + 3] << 8;
        if (h[o] == 66 && h[o + 1] == 67 && slen == 2 && o + 6 <= n) return (h[o + 4] | (size_t)h[o + 5] << 8) + 1;
        o += 4 + slen;
    }
    return 0;
}

uint32_t le32(const uint8_t *p) { return p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }

// n bytes of fd from offset off into dst, in slices of at least min_slice
// read by up to `threads` threads at once (from the page cache several
// threads copy 4-5x as fast as one).  *got: the bytes read in one piece from
// the start; fewer than n only where the file ends sooner.
emp_status pread_slices(int fd, uint8_t *dst, size_t n, uint64_t off, int threads, size_t min_slice, size_t *got) {
    *got = 0;
    if (!n) return EMP_OK;
    const int nt = (int)std::max<size_t>(1, std::min<size_t>((size_t)std::max(threads, 1), n / min_slice));
    const size_t per = ((n + nt - 1) / nt + 4095) & ~(size_t)4095;
    std::vector<size_t> done(nt, 0);
    std::atomic<bool> bad{false};
    auto slice = [&](int t) {
        const size_t a = std::min(n, (size_t)t * per), b = std::min(n, a + per);
        size_t p = a;
        while (p < b) {
            const ssize_t r = ::pread(fd, dst + p, b - p, (off_t)(off + p));
            if (r < 0 && errno == EINTR) continue;
            if (r < 0) {
                bad = true;
                break;
            }
            if (r == 0) break;  // the file ends here
            p += (size_t)r;
        }
        done[t] = p - a;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(slice, t);
    slice(0);
    for (std::thread &t : pool) t.join();
    if (bad) return EMP_E_IO;
    size_t total = 0;
    for (int t = 0; t < nt; ++t) {
        total += done[t];
        const size_t a = std::min(n, (size_t)t * per), b = std::min(n, a + per);
        if (done[t] < b - a) break;
    }
    *got = total;
    return EMP_OK;
}

}  // namespace

struct FastqReader::File {
    FILE *f = nullptr;
    int kind = 0;  // 0 plain, 1 gzip, 2 BGZF
    // plain and BGZF: the next file offset to read and the size at open (pread)
    uint64_t off = 0, size = 0;
    // gzip
    z_stream z{};
    bool z_init = false, z_end = false;
    std::vector<uint8_t> in;
    // BGZF: compressed bytes [lo, hi) of buf not yet inflated; `off` is the
    // file offset of buf's end (buf is not zeroed when it grows)
    std::unique_ptr<uint8_t[]> buf;
    size_t buf_cap = 0, lo = 0, hi = 0;
    bool grow(size_t need) {
        if (need <= buf_cap) return true;
        const size_t c = std::max(need, 2 * buf_cap);
        std::unique_ptr<uint8_t[]> nb(new (std::nothrow) uint8_t[c]);
        if (!nb) return false;
        if (hi) std::memcpy(nb.get(), buf.get(), hi);
        buf = std::move(nb);
        buf_cap = c;
        return true;
    }
    ~File() {
        if (z_init) inflateEnd(&z);
        if (f) std::fclose(f);
    }
};

FastqReader::FastqReader() = default;
FastqReader::~FastqReader() { close(); }

void FastqReader::close() {
    delete cur_;
    cur_ = nullptr;
    paths_.clear();
    next_ = 0;
}

emp_status FastqReader::open(const char *const *paths, int n, int threads) {
    close();
    if (n < 0 || (n && !paths)) return EMP_E_INVAL;
    for (int i = 0; i < n; ++i) {
        if (!paths[i]) return EMP_E_INVAL;
        struct stat sb;
        if (::stat(paths[i], &sb) != 0) {
            if (errno != ENOENT) return EMP_E_IO;
            continue;  // missing: reads as empty
        }
        if (!S_ISREG(sb.st_mode)) return EMP_E_IO;
        paths_.emplace_back(paths[i]);
    }
    threads_ = threads > 0 ? threads : (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    size_hint_ = 0;
    bool known = true;
    for (const std::string &p : paths_) {  // total decompressed size when every file tells it cheaply
        uint64_t s = 0;
        if (!measure(p, &s)) known = false;
        size_hint_ += s;
    }
    if (!known) size_hint_ = 0;
    else if (paths_.size() > 1) size_hint_ += paths_.size() - 1;  // room for the added newlines
    last_byte_ = '\n';
    emitted_ = 0;
    pending_nl_ = false;
    return EMP_OK;
}

// Decompressed size of a plain or BGZF file (block headers and ISIZE fields
// only); false for a gzip stream, whose size is not written anywhere whole.
bool FastqReader::measure(const std::string &path, uint64_t *size) {
    *size = 0;
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    uint8_t h[64];
    size_t n = std::fread(h, 1, sizeof h, f);
    bool ok = true;
    if (n < 2 || h[0] != 0x1f || h[1] != 0x8b) {
        struct stat sb;
        ok = ::stat(path.c_str(), &sb) == 0;
        *size = ok ? (uint64_t)sb.st_size : 0;
    } else {
        uint64_t off = 0;
        for (;;) {
            if (std::fseek(f, (long)off, SEEK_SET) != 0) { ok = false; break; }
            n = std::fread(h, 1, sizeof h, f);
            if (n == 0) break;
            const size_t bs = bgzf_block_size(h, n);
            if (!bs) { ok = false; break; }
            uint8_t t[4];
            if (std::fseek(f, (long)(off + bs - 4), SEEK_SET) != 0 || std::fread(t, 1, 4, f) != 4) { ok = false; break; }
            *size += le32(t);
            off += bs;
        }
    }
    std::fclose(f);
    return ok;
}

emp_status FastqReader::open_next() {
    delete cur_;
    cur_ = nullptr;
    if (next_ >= paths_.size()) return EMP_OK;
    File *fl = new File();
    cur_ = fl;
    fl->f = std::fopen(paths_[next_++].c_str(), "rb");
    if (!fl->f) return EMP_E_IO;
    uint8_t h[64];
    const size_t n = std::fread(h, 1, sizeof h, fl->f);
    if (std::fseek(fl->f, 0, SEEK_SET) != 0) return EMP_E_IO;
    struct stat sb;
    if (::fstat(fileno(fl->f), &sb) != 0) return EMP_E_IO;
    fl->size = (uint64_t)sb.st_size;  // plain and BGZF files are read with pread up to this size
    if (n >= 2 && h[0] == 0x1f && h[1] == 0x8b) {
        fl->kind = bgzf_block_size(h, n) ? 2 : 1;
        if (fl->kind == 1) {
            if (inflateInit2(&fl->z, 16 + MAX_WBITS) != Z_OK) return EMP_E_NOMEM;
            fl->z_init = true;
            fl->in.resize(kInChunk);
        }
    }
    return EMP_OK;
}

// Up to cap bytes of the current file into dst.
emp_status FastqReader::read_file(uint8_t *dst, size_t cap, size_t *got) {
    File &fl = *cur_;
    *got = 0;
    if (fl.kind == 0) {  // slices of at least 16 MiB read side by side
        const size_t n = (size_t)std::min<uint64_t>(cap, fl.size > fl.off ? fl.size - fl.off : 0);
        size_t total = 0;
        EMP_TRY_ING(pread_slices(fileno(fl.f), dst, n, fl.off, threads_, 16u << 20, &total));
        if (total < n) fl.size = fl.off + total;  // the file got shorter since it was opened
        fl.off += total;
        *got = total;
        return EMP_OK;
    }
    if (fl.kind == 1) {  // a gzip stream: members one after another
        z_stream &z = fl.z;
        z.next_out = dst;
        z.avail_out = (uInt)std::min<size_t>(cap, 1u << 30);
        while (z.avail_out && !fl.z_end) {
            if (z.avail_in == 0) {
                const size_t r = std::fread(fl.in.data(), 1, fl.in.size(), fl.f);
                if (r == 0) {
                    if (std::ferror(fl.f)) return EMP_E_IO;
                    return EMP_E_FORMAT;  // the stream stopped inside a member
                }
                z.next_in = fl.in.data();
                z.avail_in = (uInt)r;
            }
            const int rc = inflate(&z, Z_NO_FLUSH);
            if (rc == Z_STREAM_END) {  // another member follows, or the file ends
                if (z.avail_in == 0) {
                    const int c = std::fgetc(fl.f);
                    if (c == EOF) {
                        fl.z_end = true;
                        break;
                    }
                    std::ungetc(c, fl.f);
                }
                if (inflateReset(&z) != Z_OK) return EMP_E_FORMAT;
            } else if (rc != Z_OK && rc != Z_BUF_ERROR) {
                return EMP_E_FORMAT;
            }
        }
        *got = (size_t)(z.next_out - dst);
        return EMP_OK;
    }
    // BGZF: whole blocks whose inflated sizes fit cap, inflated in parallel.
    // Compressed bytes come in 32 MiB at a time (read in slices side by
    // side); block bounds are parsed in memory (a block is at most 64 KiB).
    constexpr size_t kMaxBlock = 65536, kRefill = 32u << 20, kMaxIn = 256u << 20;
    std::vector<size_t> boff, bsz, ooff;
    size_t total_out = 0;
    const int fd = fileno(fl.f);
    if (fl.lo) {  // drop what the last call inflated (the rest is under one refill)
        std::memmove(fl.buf.get(), fl.buf.get() + fl.lo, fl.hi - fl.lo);
        fl.hi -= fl.lo;
        fl.lo = 0;
    }
    for (;;) {
        if (fl.hi - fl.lo < kMaxBlock && fl.off < fl.size) {  // room for one whole block, unless the file ends
            const size_t want = (size_t)std::min<uint64_t>(kRefill, fl.size - fl.off);
            if (!fl.grow(fl.hi + want)) return EMP_E_NOMEM;
            size_t p = 0;
            EMP_TRY_ING(pread_slices(fd, fl.buf.get() + fl.hi, want, fl.off, threads_, 4u << 20, &p));
            fl.hi += p;
            fl.off += p;
            if (p < want) fl.size = fl.off;
        }
        const size_t avail = fl.hi - fl.lo;
        if (avail == 0) break;  // the end of the file
        const uint8_t *h = fl.buf.get() + fl.lo;
        const size_t bs = bgzf_block_size(h, avail);
        if (!bs || bs < 26 || bs > avail) return EMP_E_FORMAT;  // not a block, or a block cut short
        const uint32_t isize = le32(h + bs - 4);
        if (total_out + isize > cap) {
            if (boff.empty()) return EMP_E_FORMAT;  // a block larger than BGZF allows (64 KiB)
            break;                                  // for the next call
        }
        boff.push_back(fl.lo);
        bsz.push_back(bs);
        ooff.push_back(total_out);
        total_out += isize;
        fl.lo += bs;
        if (fl.lo - boff.front() > kMaxIn) break;
    }
    std::atomic<size_t> next{0};
    std::atomic<bool> bad{false};
    auto work = [&] {  // one zlib stream per thread, reset for each block
        z_stream z{};
        if (inflateInit2(&z, 16 + MAX_WBITS) != Z_OK) {
            bad = true;
            return;
        }
        for (size_t b; (b = next.fetch_add(1)) < boff.size();) {
            const size_t isize = (b + 1 < boff.size() ? ooff[b + 1] : total_out) - ooff[b];
            if (inflateReset(&z) != Z_OK) {
                bad = true;
                break;
            }
            z.next_in = const_cast<Bytef *>(fl.buf.get() + boff[b]);
            z.avail_in = (uInt)bsz[b];
            z.next_out = dst + ooff[b];
            z.avail_out = (uInt)isize;
            const int rc = inflate(&z, Z_FINISH);
            if (rc != Z_STREAM_END || z.avail_out != 0 || z.avail_in != 0) bad = true;
        }
        inflateEnd(&z);
    };
    const int nt = (int)std::min<size_t>(threads_, (boff.size() + 7) / 8);
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (std::thread &t : pool) t.join();
    if (bad) return EMP_E_FORMAT;
    *got = total_out;
    return EMP_OK;
}

emp_status FastqReader::read(void *dst_v, size_t cap, size_t *got) {
    uint8_t *dst = static_cast<uint8_t *>(dst_v);
    *got = 0;
    if (!dst || cap < kMinChunk) return EMP_E_INVAL;
    while (*got < cap / 2) {  // fill at least half of the buffer unless the input ends
        if (!cur_) {
            if (next_ >= paths_.size()) break;
            EMP_TRY_ING(open_next());
            if (last_byte_ != '\n' && emitted_) pending_nl_ = true;  // the file before ended inside a line
        }
        if (pending_nl_) {  // the newline goes in only if this file (or a later one) has bytes
            size_t g = 0;
            EMP_TRY_ING(read_file(dst + *got + 1, cap - *got - 1, &g));
            if (g == 0) {
                delete cur_;
                cur_ = nullptr;
                continue;
            }
            dst[*got] = '\n';
            pending_nl_ = false;
            *got += g + 1;
            emitted_ += g + 1;
            last_byte_ = dst[*got - 1];
            continue;
        }
        size_t g = 0;
        EMP_TRY_ING(read_file(dst + *got, cap - *got, &g));
        if (g == 0) {
            delete cur_;
            cur_ = nullptr;
            continue;
        }
        *got += g;
        emitted_ += g;
        last_byte_ = dst[*got - 1];
    }
    return EMP_OK;
}

}  // namespace emp
