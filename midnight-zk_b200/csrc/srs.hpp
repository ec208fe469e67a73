// srs.hpp — KZG test setup on the device (srs.cu)
#pragma once
#include <cstdint>

#include "ntt.hpp"
#include "runtime.hpp"

namespace mzk {

// params.rs:160-209 (G1 part); any output may be null
Status srs_setup_device(Context* ctx, const Domain* d, const uint64_t s[4], void* g, void* lag, void* delta,
                        void* ddelta, cudaStream_t st);
// G1Affine::from_compressed of n 48-byte encodings (status per point: 0 ok,
// 1 bad encoding, 2 not on the curve, 3 not in G1; invalid = their count)
Status g1_decompress_device(Context* ctx, const void* in, uint64_t n, int check_subgroup, void* out,
                            uint8_t* status, uint64_t* invalid, cudaStream_t st);
// ParamsKZG::read_custom, SerdeFormat::Processed (params.rs:283-350), G1 part
// G1Affine::to_compressed of n device points into n x 48 device bytes
Status g1_compress_device(Context* ctx, const void* in, uint64_t n, void* out, cudaStream_t st);
// write_custom (Processed), G1 part, into a host buffer of 4 + 96 n bytes
Status srs_write_processed(Context* ctx, const void* g, const void* lag, uint64_t n, uint8_t* out, size_t out_len,
                           cudaStream_t st);
Status srs_read_processed(Context* ctx, const uint8_t* bytes, size_t len, uint64_t capacity, uint32_t* k_out,
                          void* g, void* lag, void* delta, void* ddelta, cudaStream_t st);
// g_to_lagrange (utils/arithmetic.rs:34-54): out = inverse FFT of the n = 2^k
// points g over the domain, scaled by 1/n, affine
Status g1_to_lagrange_device(Context* ctx, const Domain* d, const void* g, void* out, cudaStream_t st);
// ParamsKZG::downsize (params.rs:96-107): Lagrange and delta bases of a
// smaller domain from the first 2^k points of g
Status srs_downsize_device(Context* ctx, const Domain* d, const void* g, void* lag, void* delta, void* ddelta,
                           cudaStream_t st);
// params.rs:47-57: out[i] = sum_{j >= i} in[j] (affine, n points)
Status g1_suffix_sum_device(Context* ctx, const void* in, uint64_t n, void* out, cudaStream_t st);

}  // namespace mzk
