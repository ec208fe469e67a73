// srs.hpp — KZG test setup on the device (srs.cu)
#pragma once
#include <cstdint>

#include "ntt.hpp"
#include "runtime.hpp"

namespace mzk {

// params.rs:160-209 (G1 part); any output may be null
Status srs_setup_device(Context* ctx, const Domain* d, const uint64_t s[4], void* g, void* lag, void* delta,
                        void* ddelta, cudaStream_t st);
// params.rs:47-57: out[i] = sum_{j >= i} in[j] (affine, n points)
Status g1_suffix_sum_device(Context* ctx, const void* in, uint64_t n, void* out, cudaStream_t st);

}  // namespace mzk
