// grand.hpp — column scans of the prover (grand.cu)
#pragma once
#include <cstdint>

#include "../../include/mzk.h"
#include "ntt.hpp"
#include "runtime.hpp"

namespace mzk {

// out[i] = s^i, i < n
Status fr_powers_device(Context* ctx, const uint64_t s[4], uint64_t n, void* out, cudaStream_t st);
// ff BatchInvert on n device Fr values in place (zeros stay zero)
Status batch_invert_device(Context* ctx, void* a, uint64_t n, cudaStream_t st);
// sum_i poly[i] point^i (utils/arithmetic.rs:59-87), result on the host
Status eval_polynomial_device(Context* ctx, const void* poly, uint64_t n, const uint64_t point[4], uint64_t out[4],
                              cudaStream_t st);
// q (n - 1) = a (n) / (X - b) (utils/arithmetic.rs:106-125)
Status kate_division_device(Context* ctx, const void* a, uint64_t n, const uint64_t b[4], void* q, cudaStream_t st);
// the same for T polynomials of one length n: q[j] = a[j] / (X - b[j]), their
// recurrences launched together (a, q: device pointers; b: host)
Status kate_division_batch(Context* ctx, const void* const* a, void* const* q, const host::Fr4* b, uint32_t T,
                           uint64_t n, cudaStream_t st);
// kzg/mod.rs:125-147 poly_inner_product over m device polynomials (host
// tables of pointers, lengths and scalars)
Status poly_inner_product_device(Context* ctx, const uint64_t* const* polys, const uint64_t* lens, uint32_t m,
                                 const uint64_t* scalars, void* out, uint64_t out_len, cudaStream_t st);
// permutation/prover.rs:81-255
Status permutation_z_device(Context* ctx, const Domain* d, const mzk_permutation_desc* desc, cudaStream_t st);
// logup/prover.rs:195-300
Status logup_device(Context* ctx, const Domain* d, const mzk_logup_desc* desc, cudaStream_t st);

}  // namespace mzk
