// ntt.cuh -- number-theoretic transforms over Fr on sm_100a and the QAP H step.
//
// Transform: X_k = sum_j x_j w^(jk) in natural order (the reference's ntt_h / intt_h,
// src/cuda/ntt.cpp:453 / :583: bit-reverse, then radix-2 decimation in time).  A
// transform of 2^L points runs as ceil(L/S) passes of S <= 11 radix-2 stages; each pass
// stages 2^S elements of one sub-transform in shared memory, the first pass gathers in
// bit-reversed order and the last pass can multiply every output by a per-element
// table or one scalar (used for 1/n scaling, coset shifts and leaving Montgomery form).
//
// Twiddles: W[j] = w^j (Montgomery), j < n_tab/2, for a table built for 2^L_tab points;
// a transform of 2^L <= 2^L_tab points reads W with stride 2^(L_tab - L).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace csb {

struct NttArgs {
  const uint32_t* in = nullptr;     // logical input (natural order)
  const uint32_t* in_odd = nullptr; // if set: logical input is interleave(in, in_odd)
  uint32_t* out = nullptr;          // natural-order output (may equal in only if L <= S)
  uint32_t* tmp = nullptr;          // scratch of 2^L elements when out aliases in
  uint32_t log_n = 0;
  const uint32_t* W = nullptr;      // twiddles for direction of this transform
  uint32_t log_tab = 0;             // W is a table for 2^log_tab points
  const uint32_t* post_tab = nullptr;     // out[i] *= post_tab[i] (Montgomery product)
  const uint32_t* post_scalar = nullptr;  // out[i] *= *post_scalar (Montgomery product)
  // batch instances of the transform: instance y reads and writes in, in_odd, out and tmp
  // offset by y * stride words (W, post_tab and post_scalar are shared)
  uint32_t batch = 1;
  size_t stride = 0;
};

cudaError_t ntt_run(const NttArgs& a, cudaStream_t st);

// W[j] = root^j for j < count (root: one Montgomery element in device memory).
cudaError_t ntt_powers(uint32_t* d_out, const uint32_t* d_root, uint32_t count, cudaStream_t st);
// d_out[j] = table[(stride * idx(j)) mod (stride * n)] with idx(j) = j (dir +1) or
// (n - j) mod n (dir -1), j < count: the reference's root indexing for one direction.
cudaError_t ntt_gather_roots(uint32_t* d_out, const uint32_t* d_table, uint64_t stride, uint32_t n,
                             int dir, uint32_t count, cudaStream_t st);

// Elementwise helpers on Fr arrays (Montgomery products)
cudaError_t fr_mul(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n, cudaStream_t st);
// batch instances of fr_mul, instance y at a, b and out offset by y * stride words
cudaError_t fr_mul_batch(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n, uint32_t batch,
                         size_t stride, cudaStream_t st);
// out = (a*b - c) * s  (s one element)
cudaError_t fr_mul_sub_scale(const uint32_t* a, const uint32_t* b, const uint32_t* c,
                             const uint32_t* s, uint32_t* out, uint32_t n, cudaStream_t st);
// out[i] = a[i] * tab[i]
cudaError_t fr_mul_tab(const uint32_t* a, const uint32_t* tab, uint32_t* out, uint32_t n, cudaStream_t st);

}  // namespace csb
