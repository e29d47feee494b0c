// ecops.cuh -- batched per-point scalar multiplication k_i * P_i (the reference's
// ec_jacscmul_h, src/cuda/ec.cpp:833, and its fixed-base GPU kernel sc1mulecjac_kernel,
// src/cuda/ecbn128_device.cu:326, used to build proving keys), affine Montgomery out.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace csb {

// d_points holds one affine point per term with a stride of point_stride_words
// (0 = every term uses the same base point).  Scalars are normal form, any 256-bit value.
cudaError_t scmul_g1(const uint32_t* d_scalars, const uint32_t* d_points,
                     uint32_t point_stride_words, uint32_t n, uint32_t* d_out, cudaStream_t st);
cudaError_t scmul_g2(const uint32_t* d_scalars, const uint32_t* d_points,
                     uint32_t point_stride_words, uint32_t n, uint32_t* d_out, cudaStream_t st);

}  // namespace csb
