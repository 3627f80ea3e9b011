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
//    device current) and caches it together with the id of the current context;
//    make that first call before any stream capture, since the lookup may load
//    the module.  If the context changes afterwards (cudaDeviceReset, which
//    unloads the module, then a new primary context), the next call sees the
//    different context and looks the address up again instead of using a stale
//    one;
//  * the sort's look-back waits are bounded: a wait that gives up raises an
//    error flag inside the static array, which tg_sort_noalloc_status reads
//    (the flag is cleared at the start of every call).
#include <cuda.h>

#include <mutex>

#include "tg_common.cuh"

namespace tg {
int fail_with(int code, const char* msg);  // sets the per-thread tg_last_error() message
size_t sort_workspace_bytes(int64_t n, int end_bit);
uint32_t* sort_error_flag(void* workspace, int64_t n, int end_bit);
int sort_lookback_selftest(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, void* workspace,
                           size_t ws_bytes, cudaStream_t s, cudaError_t& cerr);
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
struct ScratchCache {
    void* ptr;
    unsigned long long ctx_id;  // unique id of the context the address was looked up in (never reused)
};
ScratchCache g_scratch[kMaxDevices] = {};
std::mutex g_setup_mutex;

// cuCtxGetCurrent and cuCtxGetId, reached through the runtime (the library does not link the driver library).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
template <class Fn>
Fn driver_fn(const char* name) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion(name, &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
        p = nullptr;
    return reinterpret_cast<Fn>(p);
}

// Id of the calling thread's current context (0 when none is current or the lookup fails).
unsigned long long current_ctx_id() {
    static const CtxGetCurrentFn get = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
    static const CtxGetIdFn get_id = driver_fn<CtxGetIdFn>("cuCtxGetId");
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get == nullptr || get_id == nullptr || get(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the scratch array on the current device: looked up once per device and context.
cudaError_t scratch_on_current_device(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    unsigned long long id = current_ctx_id();
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (id == 0 || g_scratch[dev].ptr == nullptr || g_scratch[dev].ctx_id != id) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);  // initialises the primary context if none is current
        if (e != cudaSuccess) return e;
        if ((id = current_ctx_id()) == 0) return cudaErrorInitializationError;
        g_scratch[dev] = ScratchCache{p, id};
    }
    *out = g_scratch[dev].ptr;
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

// Waits for `stream`, then reads the static scratch's look-back error flag: TG_ERR_TIMEOUT if a bounded wait of
// the last allocation-free sort (or self-test) on this device gave up.
extern "C" int tg_sort_noalloc_status(tg_stream_t stream) {
    void* scratch = nullptr;
    if (scratch_on_current_device(&scratch) != cudaSuccess)
        return tg::fail_with(TG_ERR_CUDA, "tg_sort_noalloc_status: cudaGetSymbolAddress failed on this device");
    // the flag sits at the same offset for every size (it precedes the per-tile status words)
    const uint32_t* flag = tg::sort_error_flag(scratch, kNoAllocMaxPairs, 64);
    uint32_t h = 0;
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = cudaMemcpy(&h, flag, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return tg::fail_with(TG_ERR_CUDA, cudaGetErrorString(e));
    if (h) return tg::fail_with(TG_ERR_TIMEOUT, "tg_sort_noalloc_status: a look-back wait of the sort gave up");
    return TG_OK;
}

// tg_sort_lookback_selftest on the static scratch: one CTA waits for a predecessor that never publishes, its
// bounded wait gives up and raises the flag in the static array; returns TG_ERR_TIMEOUT (the expected outcome),
// after which tg_sort_noalloc_status reports the timeout too.
extern "C" int tg_sort_noalloc_lookback_selftest(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt,
                                                 tg_stream_t stream) {
    if (!keys || !vals || !keys_alt || !vals_alt)
        return tg::fail_with(TG_ERR_INVALID_ARG, "tg_sort_noalloc_lookback_selftest: null pointer");
    void* scratch = nullptr;
    if (scratch_on_current_device(&scratch) != cudaSuccess)
        return tg::fail_with(TG_ERR_CUDA, "tg_sort_noalloc_lookback_selftest: cudaGetSymbolAddress failed");
    cudaError_t cerr;
    const int rc = tg::sort_lookback_selftest(keys, vals, keys_alt, vals_alt, scratch, kNoAllocScratchBytes, stream,
                                              cerr);
    if (rc == TG_ERR_CUDA) return tg::fail_with(rc, cudaGetErrorString(cerr));
    if (rc == TG_ERR_TIMEOUT)
        return tg::fail_with(rc, "look-back wait gave up (the expected outcome of this self-test)");
    return rc;
}
