// msm_g1.cu -- G1 (Fq) instantiation of the MSM pipeline.
// Montgomery products out of line: the accumulation loop body (one XYZZ + affine
// addition, 10 products) then fits the instruction cache; measured faster at 2^20.
#define CSB_MUL_NOINLINE
#include "msm_impl.cuh"

namespace csb {

cudaError_t msm_g1(const uint32_t* s, const uint32_t* p, uint32_t n, uint32_t* out, void* w,
                   size_t wb, const MsmConfig& cfg, cudaStream_t st) {
  return msm_detail::msm_impl<Fq, false>(s, p, n, out, w, wb, cfg, st);
}

cudaError_t msm_fixed_g1(const uint32_t* s, const uint32_t* table, uint32_t n, uint32_t* out, void* w,
                         size_t wb, const MsmConfig& cfg, cudaStream_t st) {
  return msm_detail::msm_impl<Fq, true>(s, table, n, out, w, wb, cfg, st);
}

cudaError_t msm_fixed_table_g1(const uint32_t* points, uint32_t n, int c, uint32_t* table, void* w,
                               size_t wb, cudaStream_t st) {
  return msm_detail::fixed_table_impl<Fq>(points, n, c, table, w, wb, st);
}
}  // namespace csb
