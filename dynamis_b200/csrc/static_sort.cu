// static_sort.cu - the radix sort for callers that cannot allocate device memory.
//
// dyn_radix_sort_static runs the same stable LSD sort as dyn_radix_sort (sort.cuh), but every
// scratch buffer it needs lives in one file-scope __device__ array: it never calls cudaMalloc,
// cudaFree or any allocating library routine. It serves callers that own all device memory
// through their own pool and forbid allocations outside it, and callers on paths where
// cudaMalloc / cudaFree would synchronise the device.
//
// Limits and sharing:
//   * at most DYN_STATIC_SORT_MAX_KEYS keys per call (larger n is refused with DYN_ERR_CAPACITY);
//   * the array is shared by every call on a device and keeps the last call's contents; each call
//     clears the parts that must start at zero (digit histograms, tile tickets, look-back words,
//     status) on its stream before its kernels run;
//   * calls whose work overlaps on the GPU (different streams, or concurrent host threads) race
//     on the array and must be serialised by the caller;
//   * the array is held by every GPU that loads the library, until the process exits.
// The first call on a device, with that device current, looks up the array's device address
// (cudaGetSymbolAddress) and keeps it; make that first call before any stream capture. The address
// is kept per device and per CUDA context: after cudaDeviceReset (a new primary context, into which
// the module is loaded again, possibly elsewhere) the next call looks it up again.
//
// A look-back wait that runs out (DYN_STATUS_LOOKBACK_TIMEOUT) leaves the output unsorted. The
// status word of the latest call stays in the array until the next call clears it:
// dyn_radix_sort_static_status reads it after the stream's work.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "dynamis_cuda.h"
#include "sort.cuh"
#include "world.h"

namespace {

using namespace dyn;

constexpr uint32_t kMaxKeys = DYN_STATIC_SORT_MAX_KEYS;
constexpr uint32_t kMaxPasses = 8;
constexpr uint32_t kMaxTiles = (kMaxKeys + kSortTile - 1) / kSortTile;
// word offsets inside the scratch array
constexpr size_t kAltMajor = 0;
constexpr size_t kAltMinor = kAltMajor + kMaxKeys;
constexpr size_t kAltPayload = kAltMinor + kMaxKeys;
constexpr size_t kHist = kAltPayload + kMaxKeys;
constexpr size_t kTickets = kHist + kMaxPasses * 256;
constexpr size_t kStatus = kTickets + 16;
constexpr size_t kLookback = kStatus + 16;
constexpr size_t kWords = kLookback + (size_t)kMaxPasses * kMaxTiles * 256;

// Host code may not dereference this name: on the host it is only a stand-in for the symbol.
static __device__ __align__(256) uint32_t g_sort_scratch[kWords];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
uint32_t* g_device_scratch[kMaxDevices] = {};
CUcontext g_device_context[kMaxDevices] = {};
// test hook (dyn_debug_sort_fault with no world): the next call's tile tickets and poll limit
bool g_fault_armed = false;
uint32_t g_fault_skip = 0;
uint32_t g_fault_limit = kLookbackSpinLimit;

using CtxGetCurrent = CUresult (*)(CUcontext*);

// The driver's current context, through the runtime's entry-point table (no link against libcuda).
CUcontext current_context() {
    static CtxGetCurrent fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult found;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &found) != cudaSuccess ||
            found != cudaDriverEntryPointSuccess)
            return static_cast<CtxGetCurrent>(nullptr);
        return reinterpret_cast<CtxGetCurrent>(p);
    }();
    CUcontext ctx = nullptr;
    if (fn) fn(&ctx);
    return ctx;
}

// The array's device address on the current device, looked up once per device and context.
cudaError_t scratch_for_current_device(uint32_t** out) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    const CUcontext ctx = current_context();
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_device_scratch[device] || g_device_context[device] != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) return e;
        g_device_scratch[device] = static_cast<uint32_t*>(p);
        g_device_context[device] = ctx;
    }
    *out = g_device_scratch[device];
    return cudaSuccess;
}

inline uint32_t div_up(uint32_t a, uint32_t b) { return (a + b - 1) / b; }
inline uint32_t* tickets_word(uint32_t* scratch) { return scratch + kTickets; }

}  // namespace

extern "C" DYN_API dyn_status dyn_radix_sort_static(uint32_t* major, uint32_t* minor, uint32_t* payload, uint32_t n,
                                                    uint32_t major_digits, uint32_t minor_digits, void* cuda_stream) {
    if (!major || major_digits > 4 || minor_digits > 4 || (minor_digits && !minor)) return DYN_ERR_INVALID;
    if (n > kMaxKeys) return DYN_ERR_CAPACITY;
    uint32_t passes = major_digits + minor_digits;
    if (n == 0 || passes == 0) return DYN_OK;
    // an error left by earlier work stays for its owner to see; the sort does not run over it
    if (cudaPeekAtLastError() != cudaSuccess) return DYN_ERR_CUDA;
    uint32_t* scratch = nullptr;
    if (scratch_for_current_device(&scratch) != cudaSuccess) return DYN_ERR_CUDA;
    uint32_t limit = kLookbackSpinLimit, first_ticket = 0;
    {
        std::lock_guard<std::mutex> guard(g_lock);
        if (g_fault_armed) {
            limit = g_fault_limit;
            first_ticket = g_fault_skip;
            g_fault_armed = false;
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    uint32_t tiles = div_up(n, kSortTile);
    uint32_t* hist = scratch + kHist;
    uint32_t* tickets = scratch + kTickets;
    uint32_t* status = scratch + kStatus;
    uint32_t* lookback = scratch + kLookback;
    // what must start at zero for this call; the rest is overwritten before it is read
    if (cudaMemsetAsync(hist, 0, passes * 256 * sizeof(uint32_t), s) != cudaSuccess) return DYN_ERR_CUDA;
    // the 16 tile-ticket words and the 16 status words that follow them
    if (cudaMemsetAsync(tickets, 0, 32 * sizeof(uint32_t), s) != cudaSuccess) return DYN_ERR_CUDA;
    if (cudaMemsetAsync(lookback, 0, (size_t)passes * tiles * 256 * sizeof(uint32_t), s) != cudaSuccess) return DYN_ERR_CUDA;
    if (first_ticket) {
        // test hook only: the digit passes' tickets start above tile 0 (see dyn_debug_sort_fault)
        static const uint32_t tickets[kMaxPasses] = {1, 1, 1, 1, 1, 1, 1, 1};
        if (cudaMemcpyAsync(tickets_word(scratch), tickets, sizeof(tickets), cudaMemcpyHostToDevice, s) != cudaSuccess)
            return DYN_ERR_CUDA;
    }
    k_sort_histogram<<<div_up(n, 256) < 592u ? div_up(n, 256) : 592u, 256, 0, s>>>(major, minor, nullptr, n, n,
                                                                                     (int)major_digits, (int)minor_digits, hist);
    if (cudaGetLastError() != cudaSuccess) return DYN_ERR_CUDA;
    k_sort_offsets<<<1, 256, 0, s>>>(hist, (int)passes);
    if (cudaGetLastError() != cudaSuccess) return DYN_ERR_CUDA;
    uint32_t* src_major = major;
    uint32_t* src_minor = minor;
    uint32_t* src_val = payload;
    uint32_t* dst_major = scratch + kAltMajor;
    uint32_t* dst_minor = minor ? scratch + kAltMinor : nullptr;
    uint32_t* dst_val = payload ? scratch + kAltPayload : nullptr;
    bool two = minor != nullptr;
    for (uint32_t p = 0; p < passes; ++p) {
        bool on_minor = p < minor_digits;
        int shift = 8 * (int)(on_minor ? p : p - minor_digits);
        uint32_t* key_in = on_minor ? src_minor : src_major;
        uint32_t* key_out = on_minor ? dst_minor : dst_major;
        uint32_t* oth_in = on_minor ? src_major : src_minor;
        uint32_t* oth_out = on_minor ? dst_major : dst_minor;
        uint32_t* lb = lookback + (size_t)p * tiles * 256;
        if (two && payload) {
            k_onesweep<true, true><<<tiles, kSortThreads, 0, s>>>(key_in, oth_in, src_val, key_out, oth_out, dst_val, nullptr, n,
                                                                   n, shift, hist + p * 256, lb, tickets + p, status, limit);
        } else if (two) {
            k_onesweep<true, false><<<tiles, kSortThreads, 0, s>>>(key_in, oth_in, nullptr, key_out, oth_out, nullptr, nullptr,
                                                                    n, n, shift, hist + p * 256, lb, tickets + p, status, limit);
        } else if (payload) {
            k_onesweep<false, true><<<tiles, kSortThreads, 0, s>>>(key_in, nullptr, src_val, key_out, nullptr, dst_val, nullptr,
                                                                    n, n, shift, hist + p * 256, lb, tickets + p, status, limit);
        } else {
            k_onesweep<false, false><<<tiles, kSortThreads, 0, s>>>(key_in, nullptr, nullptr, key_out, nullptr, nullptr, nullptr,
                                                                     n, n, shift, hist + p * 256, lb, tickets + p, status, limit);
        }
        if (cudaGetLastError() != cudaSuccess) return DYN_ERR_CUDA;
        uint32_t* t;
        t = src_major; src_major = dst_major; dst_major = t;
        t = src_minor; src_minor = dst_minor; dst_minor = t;
        t = src_val; src_val = dst_val; dst_val = t;
    }
    if (passes % 2 == 1) {
        size_t bytes = (size_t)n * sizeof(uint32_t);
        if (cudaMemcpyAsync(major, src_major, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return DYN_ERR_CUDA;
        if (two && cudaMemcpyAsync(minor, src_minor, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return DYN_ERR_CUDA;
        if (payload && cudaMemcpyAsync(payload, src_val, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return DYN_ERR_CUDA;
    }
    return DYN_OK;
}

extern "C" DYN_API dyn_status dyn_radix_sort_static_status(void* cuda_stream, uint32_t* out) {
    if (!out) return DYN_ERR_INVALID;
    *out = 0u;
    uint32_t* scratch = nullptr;
    if (scratch_for_current_device(&scratch) != cudaSuccess) return DYN_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    uint32_t word = 0u;
    if (cudaMemcpyAsync(&word, scratch + kStatus, sizeof(word), cudaMemcpyDeviceToHost, s) != cudaSuccess) return DYN_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return DYN_ERR_CUDA;
    *out = word;
    return word ? DYN_ERR_DEVICE_STATUS : DYN_OK;
}

// The no-world branch of dyn_debug_sort_fault (world.cu): arms the next dyn_radix_sort_static call.
dyn_status dyn::static_sort_fault(uint32_t skipped_tiles, uint32_t spin_limit) {
    if (spin_limit == 0u || skipped_tiles > 1u) return DYN_ERR_INVALID;
    std::lock_guard<std::mutex> guard(g_lock);
    g_fault_armed = true;
    g_fault_skip = skipped_tiles;
    g_fault_limit = spin_limit;
    return DYN_OK;
}
