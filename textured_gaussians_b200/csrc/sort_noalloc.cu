// tg_sort_pairs_noalloc: the onesweep pair sort for callers that cannot
// allocate device memory.
//
// Some callers of this library have no way to get device scratch memory: a
// renderer or game-engine plugin that hands us only the buffers it owns, a
// real-time loop that must not call cudaMalloc (which may synchronise the
// device) or a host without a caching allocator that cannot afford a
// cudaMalloc/cudaFree pair per call.  For them this entry point keeps the
// sort's scratch (digit histograms, digit offsets, tile counters, the
// look-back status words and the wait-timeout flag) in a file-scope static
// device array of fixed size, so the caller passes only the keys, values and
// their ping-pong buffers.
//
// Costs and limits:
//  * every GPU that loads this library holds kNoAllocScratchBytes (8 MiB + 16 KiB)
//    of device memory for this array until the process exits;
//  * at most kNoAllocMaxPairs (4,194,304) pairs per call; larger sizes are
//    rejected with TG_ERR_INVALID_ARG before anything is launched;
//  * all calls share the one array: the sort clears the part that must start
//    at zero at the start of every call, but calls whose work overlaps on the
//    GPU (different streams, or different host threads, on the same device)
//    race on it and must be serialised by the caller;
//  * the first call on a device looks up the array's device address (with that
//    device current) and caches it; make that first call before any stream
//    capture, since the lookup may load the module.
#include <mutex>

#include "tg_common.cuh"

namespace tg {
int fail_with(int code, const char* msg);  // sets the per-thread tg_last_error() message
size_t sort_workspace_bytes(int64_t n, int end_bit);
int sort_pairs(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, int64_t n, int end_bit,
               void* workspace, size_t ws_bytes, int32_t* result_in_alt, cudaStream_t s, cudaError_t& cerr);
}  // namespace tg

namespace {

constexpr int64_t kNoAllocMaxPairs = int64_t(1) << 22;
constexpr size_t kAlign = 256;
constexpr size_t al(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }
// Same layout the sort carves from any workspace: histograms and digit
// offsets for 8 passes, 8 tile counters, an error flag, then one status word
// per (pass, 4096-key tile, digit).
constexpr size_t kNoAllocScratchBytes = al(4 * 8 * 256) + al(4 * 8 * 256) + al(4 * 8) + al(4) +
                                        al(size_t(4) * 8 * (kNoAllocMaxPairs / 4096) * 256);

static __device__ __align__(256) unsigned char g_sort_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Device address of the scratch array on the current device, looked up once per device.
cudaError_t scratch_on_current_device(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_ptr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

}  // namespace

static_assert(kNoAllocMaxPairs == TG_SORT_NOALLOC_MAX_PAIRS, "header and library disagree on the limit");

extern "C" int tg_sort_pairs_noalloc(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, int64_t n,
                                     int32_t end_bit, int32_t* result_in_alt, tg_stream_t stream) {
    if (result_in_alt == nullptr) return tg::fail_with(TG_ERR_INVALID_ARG, "tg_sort_pairs_noalloc: null result_in_alt");
    *result_in_alt = 0;
    if (n < 0 || n > kNoAllocMaxPairs)
        return tg::fail_with(TG_ERR_INVALID_ARG,
                             "tg_sort_pairs_noalloc: n is outside [0, 4194304], the capacity of its static scratch "
                             "(use tg_sort_pairs with a caller workspace for larger sorts)");
    if (end_bit < 0 || end_bit > 64) return tg::fail_with(TG_ERR_INVALID_ARG, "tg_sort_pairs_noalloc: bad end_bit");
    if (n <= 1) return TG_OK;
    if (!keys || !vals || !keys_alt || !vals_alt)
        return tg::fail_with(TG_ERR_INVALID_ARG, "tg_sort_pairs_noalloc: null pointer");
    if (tg::sort_workspace_bytes(n, end_bit) > kNoAllocScratchBytes)
        return tg::fail_with(TG_ERR_WORKSPACE, "tg_sort_pairs_noalloc: static scratch too small");
    void* scratch = nullptr;
    if (scratch_on_current_device(&scratch) != cudaSuccess)
        return tg::fail_with(TG_ERR_CUDA, "tg_sort_pairs_noalloc: cudaGetSymbolAddress failed on this device");
    cudaError_t cerr;
    const int rc = tg::sort_pairs(keys, vals, keys_alt, vals_alt, n, end_bit, scratch, kNoAllocScratchBytes,
                                  result_in_alt, stream, cerr);
    if (rc == TG_ERR_CUDA) return tg::fail_with(rc, cudaGetErrorString(cerr));
    return rc;
}
