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

// Point utilities behind the reference's ec_jac2aff_h / ec_jacaddreduce_h / ec_isoncurve_h
// (src/cuda/ec.cpp:963, :1266, :1064): Jacobian rows (3 coordinates) <-> affine rows (2),
// the sum of n rows (dims 2 or 3) as one affine point, and a curve check (2 infinity,
// 1 on the curve, 0 not).
cudaError_t jac_to_affine_g1(const uint32_t* jac, uint32_t n, uint32_t* aff, cudaStream_t st);
cudaError_t jac_to_affine_g2(const uint32_t* jac, uint32_t n, uint32_t* aff, cudaStream_t st);
cudaError_t affine_to_jac_g1(const uint32_t* aff, uint32_t n, uint32_t* jac, cudaStream_t st);
cudaError_t affine_to_jac_g2(const uint32_t* aff, uint32_t n, uint32_t* jac, cudaStream_t st);
cudaError_t point_sum_g1(const uint32_t* pts, uint32_t n, int dims, uint32_t* out, cudaStream_t st);
cudaError_t point_sum_g2(const uint32_t* pts, uint32_t n, int dims, uint32_t* out, cudaStream_t st);
cudaError_t on_curve_g1(const uint32_t* p, int jac, uint32_t* flag, cudaStream_t st);
// Subset-sum tables (the reference's ec_inittable_h): ceil(n / order) tables of 2^order affine
// entries, entry j of table t = sum of points t*order + b over the set bits b of j.
cudaError_t subset_table_g1(const uint32_t* aff, uint32_t n, uint32_t order, uint32_t* out, cudaStream_t st);
cudaError_t subset_table_g2(const uint32_t* aff, uint32_t n, uint32_t order, uint32_t* out, cudaStream_t st);
cudaError_t on_curve_g2(const uint32_t* p, int jac, uint32_t* flag, cudaStream_t st);

}  // namespace csb
