// primitives.cu -- device-wide primitives written for this project: exclusive scan and a stable onesweep LSD
// radix sort of (uint32 key, uint32 value) pairs.  They replace the CUB calls of the reference
// (cub::DeviceScan::ExclusiveScan, cub::DeviceRadixSort::SortPairs: src/algorithms/DEMCubWrappers.cu:26-59), and
// unlike those wrappers they never synchronise the host.
//
// Onesweep (one pass per 8-bit digit, Adinets & Merrill 2022): one kernel histograms every digit position at once;
// each pass then ranks a tile of keys in shared memory (warp-level multi-split with __match_any_sync, which keeps
// the sort stable), publishes its per-digit counts with a status flag and resolves its global offsets by decoupled
// look-back over the preceding tiles.  Tiles are numbered by an atomic counter at block start, so every tile a
// block waits for is already resident; each wait is still bounded and reports a timeout bit instead of hanging.
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "primitives.cuh"
#include "profiler.cuh"

namespace deme_b200 {

// ------------------------------------------------------------------ scan ----
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sh_warp, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (kScanThreads / 32) ? sh_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < (kScanThreads / 32)) sh_warp[lane] = w;
    }
    __syncthreads();
    uint32_t warp_prefix = warp > 0 ? sh_warp[warp - 1] : 0u;
    total = sh_warp[kScanThreads / 32 - 1];
    return warp_prefix + x - v;
}

// Loads kScanItems consecutive values of one thread; full u32 tiles use 16-byte vector loads.
template <typename T>
__device__ __forceinline__ void load_items(const T* in, uint32_t n, size_t base, uint32_t (&v)[kScanItems]) {
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        size_t idx = base + i;
        v[i] = idx < n ? (uint32_t)in[idx] : 0u;
    }
}
template <>
__device__ __forceinline__ void load_items<uint32_t>(const uint32_t* in, uint32_t n, size_t base,
                                                     uint32_t (&v)[kScanItems]) {
    if (base + kScanItems <= n && ((reinterpret_cast<uintptr_t>(in + base) & 15u) == 0)) {
        const uint4* p = reinterpret_cast<const uint4*>(in + base);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; q++) {
            const uint4 t = __ldg(p + q);
            v[4 * q] = t.x;
            v[4 * q + 1] = t.y;
            v[4 * q + 2] = t.z;
            v[4 * q + 3] = t.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; i++) {
            size_t idx = base + i;
            v[i] = idx < n ? in[idx] : 0u;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const T* in, uint32_t n, uint32_t* block_sums) {
    __shared__ uint32_t sh[kScanThreads / 32];
    const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    load_items<T>(in, n, base, v);
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) s += v[i];
    uint32_t total;
    block_exclusive_scan<T>(s, sh, total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_down_kernel(const T* in, uint32_t n, const uint32_t* block_offsets,
                                                                 uint32_t* out, uint32_t* total_out) {
    __shared__ uint32_t sh[kScanThreads / 32];
    const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    load_items<T>(in, n, base, v);
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) s += v[i];
    uint32_t total;
    uint32_t run = block_exclusive_scan<T>(s, sh, total) + (block_offsets ? block_offsets[blockIdx.x] : 0u);
    if (base + kScanItems <= n && ((reinterpret_cast<uintptr_t>(out + base) & 15u) == 0)) {
        uint4* p = reinterpret_cast<uint4*>(out + base);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; q++) {
            uint4 t;
            t.x = run;
            run += v[4 * q];
            t.y = run;
            run += v[4 * q + 1];
            t.z = run;
            run += v[4 * q + 2];
            t.w = run;
            run += v[4 * q + 3];
            p[q] = t;
        }
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; i++) {
            size_t idx = base + i;
            if (idx < n) out[idx] = run;
            run += v[i];
        }
    }
    // the last tile writes out[n] (total) when asked
    if (total_out && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) *total_out = run;
}

size_t scan_scratch_bytes(uint32_t n) {
    size_t bytes = 0;
    uint32_t m = n;
    do {
        m = (m + kScanTile - 1) / kScanTile;
        bytes += (((size_t)m + 63) / 64) * 64 * sizeof(uint32_t) * 2 + 256;
    } while (m > 1);
    return bytes + 1024;
}

// Exclusive scan of n values into out[0..n) and, if total != nullptr, the sum into *total (device pointer).
template <typename T>
static void exclusive_scan_impl(const T* in, uint32_t n, uint32_t* out, uint32_t* total, uint8_t* scratch,
                                cudaStream_t st) {
    if (n == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), st);
        return;
    }
    const uint32_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 1) {
        ProfScope prof_(KID_SCAN, st);
        scan_down_kernel<T><<<1, kScanThreads, 0, st>>>(in, n, nullptr, out, total);
        return;
    }
    uint32_t* sums = reinterpret_cast<uint32_t*>(scratch);
    uint32_t* offs = sums + ((nb + 63) / 64) * 64;
    uint8_t* next = reinterpret_cast<uint8_t*>(offs + ((nb + 63) / 64) * 64);
    {
        ProfScope prof_(KID_SCAN, st);
        scan_reduce_kernel<T><<<nb, kScanThreads, 0, st>>>(in, n, sums);
    }
    exclusive_scan_impl<uint32_t>(sums, nb, offs, nullptr, next, st);
    {
        ProfScope prof_(KID_SCAN, st);
        scan_down_kernel<T><<<nb, kScanThreads, 0, st>>>(in, n, offs, out, total);
    }
}

void exclusive_scan_u32(const uint32_t* in, uint32_t n, uint32_t* out, uint32_t* total, void* scratch, cudaStream_t st) {
    exclusive_scan_impl<uint32_t>(in, n, out, total, static_cast<uint8_t*>(scratch), st);
}
// ---------------------------------------------------------- single-pass scan ----
// Exclusive scan of uint32 in one pass over the data: tiles take ids in launch order from a ticket, publish their
// sum, and look back at their predecessors' published sums (a warp reads 32 at a time) until one carries its
// inclusive prefix, then publish their own inclusive prefix and write their outputs.  Reads the input once and
// writes the output once.  Each status word is (flag << 32) | value, flag 1 = tile sum, 2 = inclusive prefix; a
// wait that outlasts kScanSpinLimit polls sets ERR_SCAN_LOOKBACK_TIMEOUT and ends (the results are then void).
constexpr uint32_t kScanSpinLimit = 1u << 24;

__device__ __forceinline__ void scan_publish(unsigned long long* w, uint32_t flag, uint32_t v) {
    atomicExch(w, ((unsigned long long)flag << 32) | v);
}

__global__ void __launch_bounds__(kScanThreads) scan_onepass_kernel(const uint32_t* in, uint32_t n, uint32_t* out,
                                                                    uint32_t* total_out, unsigned long long* status,
                                                                    uint32_t* ticket, uint32_t nTiles, uint32_t* err) {
    __shared__ uint32_t sh[kScanThreads / 32];
    __shared__ uint32_t s_tile, s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t base = (size_t)tile * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    load_items<uint32_t>(in, n, base, v);
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) s += v[i];
    uint32_t total;
    const uint32_t excl = block_exclusive_scan<uint32_t>(s, sh, total);
    if (threadIdx.x < 32) {
        const uint32_t lane = threadIdx.x;
        uint32_t prefix = 0;
        if (tile > 0) {
            if (lane == 0) scan_publish(status + tile, 1u, total);
            int64_t pos = (int64_t)tile - 1;  // lane l reads tile pos - l
            uint32_t spins = 0;
            while (true) {
                const int64_t j = pos - (int64_t)lane;
                const unsigned long long w =
                    j >= 0 ? *reinterpret_cast<volatile unsigned long long*>(status + j) : (2ull << 32);
                const uint32_t flag = (uint32_t)(w >> 32);
                const uint32_t incl = __ballot_sync(0xffffffffu, flag == 2u);
                const uint32_t zero = __ballot_sync(0xffffffffu, flag == 0u);
                const int first = incl ? __ffs(incl) - 1 : 32;  // nearest predecessor with its inclusive prefix
                const uint32_t need = first == 32 ? 0xffffffffu : (first == 31 ? 0xffffffffu : ((2u << first) - 1u));
                if (zero & need) {
                    if (++spins > kScanSpinLimit) {
                        if (lane == 0) atomicOr(err, ERR_SCAN_LOOKBACK_TIMEOUT);
                        break;
                    }
                    continue;
                }
                uint32_t c = (int)lane <= first ? (uint32_t)w : 0u;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
                prefix += c;
                if (first < 32) break;
                pos -= 32;
            }
        }
        if (lane == 0) {
            scan_publish(status + tile, 2u, prefix + total);
            s_prefix = prefix;
        }
    }
    __syncthreads();
    uint32_t run = s_prefix + excl;
    if (base + kScanItems <= n && ((reinterpret_cast<uintptr_t>(out + base) & 15u) == 0)) {
        uint4* p = reinterpret_cast<uint4*>(out + base);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; q++) {
            uint4 t;
            t.x = run;
            run += v[4 * q];
            t.y = run;
            run += v[4 * q + 1];
            t.z = run;
            run += v[4 * q + 2];
            t.w = run;
            run += v[4 * q + 3];
            p[q] = t;
        }
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; i++) {
            const size_t idx = base + i;
            if (idx < n) out[idx] = run;
            run += v[i];
        }
    }
    if (total_out && tile == nTiles - 1 && threadIdx.x == kScanThreads - 1) *total_out = run;
}

size_t scan_onepass_scratch_bytes(uint32_t n) {
    const size_t tiles = ((size_t)n + kScanTile - 1) / kScanTile;
    return (tiles + 2) * sizeof(unsigned long long) + 256;
}

void exclusive_scan_u32_onepass(const uint32_t* in, uint32_t n, uint32_t* out, uint32_t* total, void* scratch,
                                uint32_t* err, cudaStream_t st) {
    if (n == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), st);
        return;
    }
    const uint32_t nTiles = (n + kScanTile - 1) / kScanTile;
    unsigned long long* status = static_cast<unsigned long long*>(scratch);
    uint32_t* ticket = reinterpret_cast<uint32_t*>(status + nTiles);
    cudaMemsetAsync(status, 0, ((size_t)nTiles + 1) * sizeof(unsigned long long), st);
    ProfScope prof_(KID_SCAN, st);
    scan_onepass_kernel<<<nTiles, kScanThreads, 0, st>>>(in, n, out, total, status, ticket, nTiles, err);
}

void exclusive_scan_u16(const uint16_t* in, uint32_t n, uint32_t* out, uint32_t* total, void* scratch, cudaStream_t st) {
    exclusive_scan_impl<uint16_t>(in, n, out, total, static_cast<uint8_t*>(scratch), st);
}
void exclusive_scan_u8(const uint8_t* in, uint32_t n, uint32_t* out, uint32_t* total, void* scratch, cudaStream_t st) {
    exclusive_scan_impl<uint8_t>(in, n, out, total, static_cast<uint8_t*>(scratch), st);
}

// ------------------------------------------------------------ radix sort ----
constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsItems = 15;
constexpr int kRsTile = kRsThreads * kRsItems;
constexpr int kRsRadix = 256;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1u;
constexpr uint32_t kLookbackSpinLimit = 1u << 24;

__global__ void __launch_bounds__(kRsThreads) rs_histogram_kernel(const uint32_t* __restrict__ keys, uint32_t n,
                                                                  int passes, uint32_t* hist) {
    __shared__ uint32_t sh[4 * kRsRadix];
    for (int i = threadIdx.x; i < 4 * kRsRadix; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        const uint32_t k = keys[idx];
        for (int p = 0; p < passes; p++) atomicAdd(&sh[p * kRsRadix + ((k >> (8 * p)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRsRadix; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

__global__ void __launch_bounds__(kRsRadix) rs_scan_hist_kernel(uint32_t* hist) {
    // one block per pass: exclusive scan of its 256 bins in place
    __shared__ uint32_t sh[kRsRadix / 32];
    uint32_t* h = hist + blockIdx.x * kRsRadix;
    const uint32_t v = h[threadIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    uint32_t pre = 0;
    for (int w = 0; w < warp; w++) pre += sh[w];
    h[threadIdx.x] = pre + x - v;
}

__global__ void __launch_bounds__(kRsThreads) rs_onesweep_kernel(const uint32_t* __restrict__ keys_in,
                                                                 const uint32_t* __restrict__ vals_in,
                                                                 uint32_t* __restrict__ keys_out,
                                                                 uint32_t* __restrict__ vals_out, uint32_t n, int shift,
                                                                 const uint32_t* __restrict__ digit_offset,
                                                                 uint32_t* tile_status, uint32_t* tile_counter,
                                                                 uint32_t* err) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp_hist[kRsWarps][kRsRadix];
    __shared__ uint32_t s_prefix[kRsRadix];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < kRsWarps * kRsRadix; i += kRsThreads) (&s_warp_hist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t base = (size_t)tile * kRsTile + (size_t)warp * 32 * kRsItems;

    uint32_t key[kRsItems], val[kRsItems], rank[kRsItems];
#pragma unroll
    for (int i = 0; i < kRsItems; i++) {
        const size_t idx = base + (size_t)i * 32 + lane;
        const bool ok = idx < n;
        key[i] = ok ? keys_in[idx] : 0xFFFFFFFFu;
        val[i] = ok ? vals_in[idx] : 0u;
    }
    // warp-level stable ranking, item-major then lane order (= input order within the warp's sub-tile)
    const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int i = 0; i < kRsItems; i++) {
        const uint32_t d = (key[i] >> shift) & 255u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = s_warp_hist[warp][d];
        rank[i] = before + __popc(peers & lt_mask);
        __syncwarp();
        if (lane == __ffs(peers) - 1) s_warp_hist[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // thread t owns digit t: exclusive prefix over warps, tile count, look-back
    {
        const uint32_t d = threadIdx.x;
        uint32_t sum = 0;
#pragma unroll
        for (int w = 0; w < kRsWarps; w++) {
            const uint32_t c = s_warp_hist[w][d];
            s_warp_hist[w][d] = sum;
            sum += c;
        }
        volatile uint32_t* status = tile_status;
        uint32_t exclusive = 0;
        if (tile == 0) {
            status[d] = kFlagPrefix | sum;
        } else {
            status[(size_t)tile * kRsRadix + d] = kFlagAgg | sum;
            uint32_t j = tile - 1;
            uint32_t spins = 0;
            while (true) {
                const uint32_t s = status[(size_t)j * kRsRadix + d];
                const uint32_t flag = s & ~kValueMask;
                if (flag == 0u) {
                    if (++spins > kLookbackSpinLimit) {
                        atomicOr(err, ERR_SORT_LOOKBACK_TIMEOUT);
                        break;
                    }
                    continue;
                }
                exclusive += s & kValueMask;
                if (flag == kFlagPrefix || j == 0) break;
                j--;
            }
            status[(size_t)tile * kRsRadix + d] = kFlagPrefix | ((exclusive + sum) & kValueMask);
        }
        s_prefix[d] = digit_offset[d] + exclusive;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kRsItems; i++) {
        const size_t idx = base + (size_t)i * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[i] >> shift) & 255u;
            const uint32_t pos = s_prefix[d] + s_warp_hist[warp][d] + rank[i];
            keys_out[pos] = key[i];
            vals_out[pos] = val[i];
        }
    }
}

size_t radix_sort_scratch_bytes(uint32_t n) {
    const size_t tiles = ((size_t)n + kRsTile - 1) / kRsTile;
    size_t b = 4 * kRsRadix * sizeof(uint32_t);                 // histograms
    b += (tiles * kRsRadix + 64) * sizeof(uint32_t);             // tile status + counter
    b += 2 * ((size_t)n + 64) * sizeof(uint32_t);                // alternate key/value buffers
    return b + 4096;
}

void radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                      uint32_t n, int key_bits, void* scratch, uint32_t* err, cudaStream_t st) {
    const int passes = key_bits <= 0 ? 0 : (key_bits + 7) / 8;
    if (n == 0) return;
    if (passes == 0) {
        cudaMemcpyAsync(keys_out, keys_in, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vals_out, vals_in, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
        return;
    }
    const uint32_t tiles = (n + kRsTile - 1) / kRsTile;
    uint32_t* hist = static_cast<uint32_t*>(scratch);
    uint32_t* status = hist + 4 * kRsRadix;
    uint32_t* counter = status + (size_t)tiles * kRsRadix;
    uint32_t* alt_k = counter + 64;
    uint32_t* alt_v = alt_k + n + 64;
    cudaMemsetAsync(hist, 0, 4 * kRsRadix * sizeof(uint32_t), st);
    const int hb = (int)std::min<uint32_t>((n + 1023) / 1024, 1184u);
    {
        ProfScope prof_(KID_SORT_HIST, st);
        rs_histogram_kernel<<<hb, kRsThreads, 0, st>>>(keys_in, n, passes, hist);
    }
    {
        ProfScope prof_(KID_SORT_HIST, st);
        rs_scan_hist_kernel<<<passes, kRsRadix, 0, st>>>(hist);
    }
    const uint32_t* src_k = keys_in;
    const uint32_t* src_v = vals_in;
    for (int p = 0; p < passes; p++) {
        const bool to_out = ((passes - 1 - p) % 2) == 0;
        uint32_t* dk = to_out ? keys_out : alt_k;
        uint32_t* dv = to_out ? vals_out : alt_v;
        cudaMemsetAsync(status, 0, ((size_t)tiles * kRsRadix + 64) * sizeof(uint32_t), st);
        {
            ProfScope prof_(KID_SORT_PASS, st);
            rs_onesweep_kernel<<<tiles, kRsThreads, 0, st>>>(src_k, src_v, dk, dv, n, 8 * p, hist + p * kRsRadix,
                                                             status, counter, err);
        }
        src_k = dk;
        src_v = dv;
    }
}

}  // namespace deme_b200
