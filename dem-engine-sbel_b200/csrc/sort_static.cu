// sort_static.cu -- deme_radix_sort_pairs_static: the onesweep radix sort of primitives.cu for callers that cannot
// allocate device memory.  Two kinds of caller are meant: code embedded in a host application that has already
// reserved the GPU's memory for its own pool (a coupled fluid solver driving the DEM step, or a framework whose
// caching allocator owns the HBM), where a cudaMalloc fails or splits that pool; and per-step code that must not
// call cudaMalloc/cudaFree because they synchronise the device and stall the work queued on other streams.
// Its scratch (histograms, tile look-back flags, alternate key/value buffers, error word) is one file-scope
// __device__ array, so every device that loads this library holds kStaticSortScratchBytes until the process
// exits.  Host code cannot use the array's name as a device pointer (on the host it names a stand-in object), so
// its device address is looked up with cudaGetSymbolAddress once per device, on the first call made with that
// device current, and passed to the kernels.  That address is kept for the life of the process, so calls after a
// cudaDeviceReset of that device are not supported.  Nothing here calls cudaMalloc/cudaFree or any allocating
// library routine.
//
// deme_radix_sort_status reads back the error word of a sort (this one's, or the allocating sort's in its caller's
// scratch): a look-back wait of the sort that ran out of its iteration limit leaves the output unordered, and only
// the word tells.
#include <mutex>

#include "../../include/deme_b200.h"
#include "primitives.cuh"

namespace {

constexpr size_t kStaticSortScratchBytes = (size_t)17 << 19;  // 8.5 MiB
constexpr size_t kErrOffset = kStaticSortScratchBytes - 256;   // error word, own 256-byte line at the end
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint8_t g_sort_scratch[kStaticSortScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_sort_scratch on the current device; looked up on the first call per device.
int32_t static_scratch(cudaStream_t st, uint8_t** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return DEME_ERR_NO_DEVICE;
    if (dev >= kMaxDevices) return DEME_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        // Set-up may load this library's device code; refuse it inside a stream capture.
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) return DEME_ERR_CUDA;
        if (cap != cudaStreamCaptureStatusNone) return DEME_ERR_STATE;
        if (deme_b200::radix_sort_scratch_bytes(DEME_SORT_STATIC_MAX_N) > kErrOffset) return DEME_ERR_INVALID;
        void* p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (rc != cudaSuccess || p == nullptr) return DEME_ERR_CUDA;
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<uint8_t*>(g_scratch_ptr[dev]);
    return DEME_OK;
}

}  // namespace

extern "C" int32_t deme_radix_sort_pairs_static(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                                uint32_t* vals_out, uint32_t n, int32_t key_bits, void* stream) {
    if (n > DEME_SORT_STATIC_MAX_N) return DEME_ERR_TOO_LARGE;
    if (key_bits < 0 || key_bits > 32) return DEME_ERR_INVALID;
    if (n > 0 && (!keys_in || !vals_in || !keys_out || !vals_out)) return DEME_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    uint8_t* scratch = nullptr;
    const int32_t rc = static_scratch(st, &scratch);
    if (rc != DEME_OK) return rc;
    if (n == 0) return DEME_OK;
    // The histograms, tile flags, tile counter and error word must start at zero; radix_sort_pairs clears the
    // first three on `st` before its kernels read them, the error word is cleared here.
    uint32_t* err = reinterpret_cast<uint32_t*>(scratch + kErrOffset);
    if (cudaMemsetAsync(err, 0, sizeof(uint32_t), st) != cudaSuccess) return DEME_ERR_CUDA;
    deme_b200::radix_sort_pairs(keys_in, vals_in, keys_out, vals_out, n, key_bits, scratch, err, st);
    return cudaGetLastError() == cudaSuccess ? DEME_OK : DEME_ERR_CUDA;
}

extern "C" int32_t deme_radix_sort_status(const void* scratch, uint32_t n, void* stream, uint32_t* word) {
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t* err = nullptr;
    if (scratch) {
        // deme_radix_sort_pairs_device: the word follows the sort's own scratch in the caller's buffer
        err = reinterpret_cast<const uint32_t*>(static_cast<const uint8_t*>(scratch) +
                                                deme_b200::radix_sort_scratch_bytes(n));
    } else {
        uint8_t* base = nullptr;
        const int32_t rc = static_scratch(st, &base);
        if (rc != DEME_OK) return rc;
        err = reinterpret_cast<const uint32_t*>(base + kErrOffset);
    }
    uint32_t w = 0;
    if (cudaMemcpyAsync(&w, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess) return DEME_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return DEME_ERR_CUDA;
    if (word) *word = w;
    return w == 0u ? DEME_OK : DEME_ERR_TIMEOUT;
}
