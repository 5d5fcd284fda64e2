// pfs_sort_static.cu — the cell-key sort for callers that cannot allocate
// device memory.
//
// Some hosts of this library own the whole device heap themselves: a game
// engine or renderer that sub-allocates every buffer from its own pools, or a
// frame loop with a fixed memory plan, where a cudaMalloc from a library
// would either fail or stall the device (cudaMalloc/cudaFree synchronise).
// pfs_sort_keys_static serves them: it runs the same stable radix sort the
// world step uses (sort_pairs in pfs_sort.cu) with its scratch
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
//    device memory) and caches it per device and context; make that first
//    call before any stream capture is in progress.  A device reset makes a
//    new context, and the next call looks the address up again;
//  - the kernels' own range checks and bounded waits set an error word in
//    the array; pfs_sort_static_status reads it for the last call.
#include <cstdint>
#include <mutex>

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/pfs.h"
#include "pfs_sort.cuh"
#include "pfs_world_impl.cuh"

namespace {

constexpr uint32_t kMaxKeys = PFS_STATIC_SORT_MAX_KEYS;
constexpr int kMaxKeyBits = 32;
// keys_tmp + vals_tmp + the sort's histograms and look-back words + the
// error word (its own 256-byte line at the end)
constexpr size_t kSortWords = 2 * (size_t)kMaxKeys;
constexpr size_t kWordsUpper = kSortWords + 4 * 256 + 64 + 4 * 256 * (size_t)((kMaxKeys + 4095) / 4096) + 64;

static __device__ __align__(256) uint32_t g_sort_scratch[kWordsUpper];

constexpr int kMaxDevices = 64;
struct ScratchAddr {
    uint32_t* addr = nullptr;
    CUcontext ctx = nullptr;  // the context the address belongs to
};
ScratchAddr g_scratch[kMaxDevices];
std::mutex g_setup_lock;

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

// The current context (the runtime API names devices, not contexts; a reset
// replaces the context and may move the module's static array).
CUcontext current_context() {
    static CtxGetCurrentFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (CtxGetCurrentFn) nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    CUcontext c = nullptr;
    if (fn) fn(&c);
    return c;
}

int scratch_for_current_device(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return pfs::status_from_cuda(e);
    if (dev < 0 || dev >= kMaxDevices) return PFS_ENODEV;
    std::lock_guard<std::mutex> g(g_setup_lock);
    // look the address up again whenever the current context is not the
    // one it was found in (or none is current yet: the lookup makes the
    // device's primary context current)
    ScratchAddr& s = g_scratch[dev];
    const CUcontext ctx = current_context();
    if (!s.addr || !ctx || ctx != s.ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) return pfs::status_from_cuda(e);
        s.addr = static_cast<uint32_t*>(p);
        s.ctx = current_context();
    }
    *out = s.addr;
    return PFS_OK;
}

bool overlaps(const uint32_t* a, const uint32_t* b, uint32_t n) {
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    const uintptr_t len = (uintptr_t)n * sizeof(uint32_t);
    return x < y + len && y < x + len;
}

}  // namespace

extern "C" int pfs_sort_keys_static(const uint32_t* keys_dev, uint32_t n, uint32_t key_bits,
                                    uint32_t* sorted_keys_dev, uint32_t* perm_dev,
                                    void* stream) {
    if (n > kMaxKeys) return PFS_ERANGE;
    if (key_bits > (uint32_t)kMaxKeyBits) return PFS_EINVAL;
    if (n == 0) return PFS_OK;
    if (!keys_dev || !sorted_keys_dev || !perm_dev) return PFS_EINVAL;
    // the first pass may scatter straight into the outputs while other tiles
    // still read the keys, so no two of the three arrays may share memory
    if (overlaps(keys_dev, sorted_keys_dev, n) || overlaps(keys_dev, perm_dev, n) ||
        overlaps(sorted_keys_dev, perm_dev, n))
        return PFS_EINVAL;
    uint32_t* base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc) return rc;
    const int bits = key_bits ? (int)key_bits : pfs::sort_key_bits(n);
    uint32_t* keys_tmp = base;
    uint32_t* vals_tmp = base + kMaxKeys;
    uint32_t* sort_scratch = base + kSortWords;
    uint32_t* err = base + kWordsUpper - 64;
    if (kSortWords + pfs::sort_scratch_words(kMaxKeys, kMaxKeyBits) + 64 > kWordsUpper) return PFS_ERANGE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return pfs::status_from_cuda(e);
    e = pfs::sort_pairs(keys_dev, n, bits, sorted_keys_dev, perm_dev, keys_tmp, vals_tmp,
                        sort_scratch, err, s);
    return pfs::status_from_cuda(e);
}

extern "C" int pfs_sort_static_status(void* stream) {
    uint32_t* base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc) return rc;
    uint32_t word = 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(&word, base + kWordsUpper - 64, sizeof(word),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return pfs::status_from_cuda(e);
    return word ? PFS_EDEVICE : PFS_OK;
}
