// dcb_sort.cuh — device-wide sort, scan and selection (dcb_sort.cu) of the mesh post-pass and
// the vertex refinement. Inputs are not modified; `temp` is caller-provided scratch of at least
// the matching *_temp_bytes size; n < 2^31.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace dcb {

// stable LSD radix sort of keys [begin_bit, end_bit) with 32-bit values carried along
size_t radix_sort_temp_bytes(long long n, int key_bytes, bool pairs);
cudaError_t radix_sort_pairs(void* temp, size_t temp_bytes, const unsigned long long* kin, unsigned long long* kout,
                             const uint32_t* vin, uint32_t* vout, long long n, int begin_bit, int end_bit, cudaStream_t s);
cudaError_t radix_sort_pairs(void* temp, size_t temp_bytes, const uint32_t* kin, uint32_t* kout, const uint32_t* vin,
                             uint32_t* vout, long long n, int begin_bit, int end_bit, cudaStream_t s);
cudaError_t radix_sort_keys(void* temp, size_t temp_bytes, const unsigned long long* kin, unsigned long long* kout,
                            long long n, int begin_bit, int end_bit, cudaStream_t s);

// prefix sums
size_t scan_temp_bytes(long long n);
cudaError_t exclusive_sum(void* temp, size_t temp_bytes, const uint32_t* in, uint32_t* out, long long n, cudaStream_t s);
cudaError_t exclusive_sum(void* temp, size_t temp_bytes, const unsigned long long* in, unsigned long long* out, long long n,
                          cudaStream_t s);
cudaError_t inclusive_sum(void* temp, size_t temp_bytes, const uint32_t* in, uint32_t* out, long long n, cudaStream_t s);

// the flagged items (or their indices) in order, and their count
size_t select_temp_bytes(long long n);
cudaError_t select_flagged(void* temp, size_t temp_bytes, const int4* in, const uint8_t* flags, int4* out,
                           unsigned long long* count, long long n, cudaStream_t s);
cudaError_t select_flagged_index(void* temp, size_t temp_bytes, const uint8_t* flags, int* out, unsigned long long* count,
                                 long long n, cudaStream_t s);

}  // namespace dcb
