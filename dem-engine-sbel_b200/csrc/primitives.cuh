// primitives.cuh -- device-wide scan and radix sort written for this project (see primitives.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace deme_b200 {

size_t scan_scratch_bytes(uint32_t n);
// Exclusive scans into out[0..n); *total (device pointer, optional) receives the sum.
void exclusive_scan_u32(const uint32_t* in, uint32_t n, uint32_t* out, uint32_t* total, void* scratch, cudaStream_t st);
void exclusive_scan_u16(const uint16_t* in, uint32_t n, uint32_t* out, uint32_t* total, void* scratch, cudaStream_t st);
void exclusive_scan_u8(const uint8_t* in, uint32_t n, uint32_t* out, uint32_t* total, void* scratch, cudaStream_t st);
// The same for uint32 in one pass over the data (decoupled look-back); a timed-out wait sets bits in *err.
size_t scan_onepass_scratch_bytes(uint32_t n);
void exclusive_scan_u32_onepass(const uint32_t* in, uint32_t n, uint32_t* out, uint32_t* total, void* scratch,
                                uint32_t* err, cudaStream_t st);

size_t radix_sort_scratch_bytes(uint32_t n);
// Stable sort of (key, value) pairs on key bits [0, key_bits).  Inputs are not modified; outputs must not alias
// inputs.  Timeouts of the bounded look-back wait set bits in *err (device pointer).
void radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                      uint32_t n, int key_bits, void* scratch, uint32_t* err, cudaStream_t st);

}  // namespace deme_b200
