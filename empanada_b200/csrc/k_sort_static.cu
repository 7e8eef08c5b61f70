// k_sort_static.cu -- emp_sort_pairs_static: the stable onesweep sort of
// k_sort.cu with its whole working set in one statically sized device array,
// so a call allocates nothing (no cudaMalloc / cudaFree, no allocating
// library routine).
//
// The array holds, for at most kStaticMaxPairs pairs:
//   [alternate keys 8 B/pair][alternate values 4 B/pair][error word, n]
//   [SortScratch header][look-back words, one per (4096-pair tile, digit)]
// Each call clears the error word, the header and the look-back words of its
// own tiles before the sort reads them.  Every call on a device uses the
// same array: calls whose GPU work overlaps (other streams, other host
// threads) race on it and give wrong results.
#include <mutex>

#include "../../include/empanada.h"
#include "kernels.h"

namespace emp {
namespace {

constexpr uint64_t kStaticMaxPairs = EMP_SORT_STATIC_MAX_PAIRS;
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kOffK1 = 0;
constexpr size_t kOffV1 = align_up(kOffK1 + kStaticMaxPairs * sizeof(uint64_t));
constexpr size_t kOffWord = align_up(kOffV1 + kStaticMaxPairs * sizeof(uint32_t));  // u32 error, u64 n at +8
constexpr size_t kOffScr = align_up(kOffWord + 16);
constexpr size_t kMaxTiles = (kStaticMaxPairs + kSortTile - 1) / kSortTile;
constexpr size_t kScrBytes = sizeof(SortScratch) + kMaxTiles * kSortRadix * sizeof(uint64_t);
constexpr size_t kStaticBytes = align_up(kOffScr + kScrBytes);  // 12.6 MB at 2^20 pairs

static __device__ __align__(256) uint8_t g_sort_static[kStaticBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint8_t *g_ptr[kMaxDevices] = {};

// Device address of g_sort_static on the current device (looked up once).
emp_status static_scratch(uint8_t **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return EMP_E_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return EMP_E_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ptr[dev]) {
        uint8_t *p = nullptr;
        if (cudaGetSymbolAddress((void **)&p, g_sort_static) != cudaSuccess || !p) {
            cudaGetLastError();
            return EMP_E_CUDA;
        }
        g_ptr[dev] = p;
    }
    *out = g_ptr[dev];
    return EMP_OK;
}

}  // namespace
}  // namespace emp

extern "C" emp_status emp_sort_pairs_static(uint64_t *d_keys, uint32_t *d_vals, uint64_t n, void *stream) {
    using namespace emp;
    if (n > kStaticMaxPairs) return EMP_E_INVAL;
    if (n && (!d_keys || !d_vals)) return EMP_E_INVAL;  // the argument check of emp_sort_pairs
    if (n < 2) return EMP_OK;
    uint8_t *base = nullptr;
    const emp_status rc = static_scratch(&base);
    if (rc != EMP_OK) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t *err = reinterpret_cast<uint32_t *>(base + kOffWord);
    uint64_t *n_dev = reinterpret_cast<uint64_t *>(base + kOffWord + 8);
    const size_t scr_bytes = sort_scratch_bytes(n);  // header + look-back words of n's tiles
    if (cudaMemsetAsync(err, 0, sizeof(uint32_t), s) != cudaSuccess ||
        cudaMemsetAsync(base + kOffScr, 0, scr_bytes, s) != cudaSuccess) {
        cudaGetLastError();
        return EMP_E_CUDA;
    }
    sort_pairs(d_keys, d_vals, reinterpret_cast<uint64_t *>(base + kOffK1), reinterpret_cast<uint32_t *>(base + kOffV1),
               n, base + kOffScr, n_dev, err, s, nullptr);
    if (cudaGetLastError() != cudaSuccess) return EMP_E_CUDA;
    uint32_t herr = 0;
    if (cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return EMP_E_CUDA;
    }
    if (herr & kErrSpin) return EMP_E_TIMEOUT;
    return EMP_OK;
}
