// pfs_sort_static.cu — the cell-key sort for callers that cannot allocate
// device memory.
//
// Some hosts of this library own the whole device heap themselves: a game
// engine or renderer that sub-allocates every buffer from its own pools, or a
// frame loop with a fixed memory plan, where a cudaMalloc from a library
// would either fail or stall the device (cudaMalloc/cudaFree synchronise).
// pfs_sort_keys_static serves them: it runs the same stable radix sort the
// world step uses (sort_pairs in pfs_sort.cu, unchanged) with its scratch
// buffers carved from one array that lives in this library's static device
// memory, so the call itself allocates nothing.  The caller still provides
// the input keys and the two output arrays.
//
// Limits and sharing:
//  - at most PFS_STATIC_SORT_MAX_KEYS keys per call (larger n is refused with
//    PFS_ERANGE); the array costs about 8.3 MiB of device memory on every GPU
//    that loads the library, held until the process exits;
//  - every call on a device uses the same array and it keeps whatever the
//    previous call left in it (each call overwrites or clears everything the
//    sort reads before reading it), so two calls whose work overlaps on the
//    GPU — on different streams, or from different host threads — race on
//    that scratch and must be serialised by the caller;
//  - the first call on a device looks up the array's device address (host
//    code may not use the symbol itself: on the host it names a stand-in, not
//    device memory) and caches it per device; make that first call before any
//    stream capture is in progress.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/pfs.h"
#include "pfs_sort.cuh"
#include "pfs_world_impl.cuh"

namespace {

constexpr uint32_t kMaxKeys = PFS_STATIC_SORT_MAX_KEYS;
constexpr uint32_t kTileKeys = 4096;  // keys per radix tile (pfs_sort.cu)
constexpr uint32_t kMaxTiles = (kMaxKeys + kTileKeys - 1) / kTileKeys;
// keys_tmp + vals_tmp + per-tile histograms + digit totals + error word
constexpr size_t kWords = 2 * (size_t)kMaxKeys + 256 * (size_t)kMaxTiles + 256 + 64;

static __device__ __align__(256) uint32_t g_sort_scratch[kWords];

constexpr int kMaxDevices = 64;
uint32_t* g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_lock;

int scratch_for_current_device(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return pfs::status_from_cuda(e);
    if (dev < 0 || dev >= kMaxDevices) return PFS_ENODEV;
    std::lock_guard<std::mutex> g(g_setup_lock);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) return pfs::status_from_cuda(e);
        g_scratch_addr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_scratch_addr[dev];
    return PFS_OK;
}

}  // namespace

extern "C" int pfs_sort_keys_static(const uint32_t* keys_dev, uint32_t n, uint32_t key_bits,
                                    uint32_t* sorted_keys_dev, uint32_t* perm_dev,
                                    void* stream) {
    if (n > kMaxKeys) return PFS_ERANGE;
    if (key_bits > 32) return PFS_EINVAL;
    if (n == 0) return PFS_OK;
    if (!keys_dev || !sorted_keys_dev || !perm_dev) return PFS_EINVAL;
    uint32_t* base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc) return rc;
    const int bits = key_bits ? (int)key_bits : pfs::sort_key_bits(n);
    uint32_t* keys_tmp = base;
    uint32_t* vals_tmp = base + kMaxKeys;
    uint32_t* hist = vals_tmp + kMaxKeys;
    uint32_t* digit_total = hist + 256 * (size_t)kMaxTiles;
    uint32_t* err = digit_total + 256;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return pfs::status_from_cuda(e);
    e = pfs::sort_pairs(keys_dev, n, bits, sorted_keys_dev, perm_dev, keys_tmp, vals_tmp, hist,
                        digit_total, err, s);
    return pfs::status_from_cuda(e);
}
