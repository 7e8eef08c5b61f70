// ingest.h -- FASTQ input from files (plain, gzip, BGZF; several files in
// order), read chunk by chunk into caller buffers.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "empanada.h"

#define EMP_TRY_ING(x)                   \
    do {                                 \
        emp_status _s = (x);             \
        if (_s != EMP_OK) return _s;     \
    } while (0)

namespace emp {

class FastqReader {
  public:
    static constexpr size_t kMinChunk = 256u << 10;  // smallest buffer read() takes
    FastqReader();
    ~FastqReader();
    FastqReader(const FastqReader &) = delete;
    FastqReader &operator=(const FastqReader &) = delete;
    // The files in order.  A missing file reads as empty; a path that exists
    // but is not a regular file is EMP_E_IO; a plain file is read up to its
    // size at the time it is opened.  threads: host threads that read slices
    // of a plain file or inflate BGZF blocks (0: the machine's, at most 32).
    emp_status open(const char *const *paths, int n, int threads = 0);
    // The next bytes of the FASTQ into dst (cap >= kMinChunk): at least cap/2
    // of them unless the input ends; *got = 0 at the end.  EMP_E_FORMAT for a
    // damaged gzip stream or BGZF block, EMP_E_IO for a read error.
    emp_status read(void *dst, size_t cap, size_t *got);
    // The whole FASTQ's size when every file tells it without inflating (plain
    // files, BGZF), else 0.
    uint64_t size_hint() const { return size_hint_; }
    void close();

  private:
    struct File;
    emp_status open_next();
    emp_status read_file(uint8_t *dst, size_t cap, size_t *got);
    static bool measure(const std::string &path, uint64_t *size);
    std::vector<std::string> paths_;
    size_t next_ = 0;
    File *cur_ = nullptr;
    int threads_ = 1;
    uint64_t size_hint_ = 0, emitted_ = 0;
    uint8_t last_byte_ = '\n';
    bool pending_nl_ = false;
};

}  // namespace emp
