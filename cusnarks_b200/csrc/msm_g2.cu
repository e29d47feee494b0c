// msm_g2.cu -- G2 (Fq2) instantiation of the MSM pipeline.
// Montgomery products out of line: the accumulation loop body (one XYZZ + affine
// addition, 10 products) then fits the instruction cache; measured faster at 2^20.
#define CSB_MUL_NOINLINE
// Fq products stay 32-bit CIOS here: the FP64-pipe product needs more registers than
// the 168 the Fq2 kernels run at (G2 fixed-base MSM 13.1 -> 13.9 ms with it).  With the
// accumulation uncapped and the batch-affine rounds kept at 168 registers the G2 MSM alone
// gains a little (fixed-base 13.21 -> 13.02 ms), but a 2^20 proof loses (26.1 -> 26.3-26.6 ms):
// its G1 MSMs already fill the FP64 pipe, and G2 on the integer pipes runs beside them.
#ifndef CSB_DP52
#define CSB_DP52 0
#endif
#include "msm_impl.cuh"

namespace csb {

cudaError_t msm_g2(const uint32_t* s, const uint32_t* p, uint32_t n, uint32_t* out, void* w,
                   size_t wb, const MsmConfig& cfg, cudaStream_t st) {
  return msm_detail::msm_impl<Fq2, false>(s, p, n, out, w, wb, cfg, st);
}

cudaError_t msm_fixed_g2(const uint32_t* s, const uint32_t* table, uint32_t n, uint32_t* out, void* w,
                         size_t wb, const MsmConfig& cfg, cudaStream_t st) {
  return msm_detail::msm_impl<Fq2, true>(s, table, n, out, w, wb, cfg, st);
}

cudaError_t msm_fixed_table_g2(const uint32_t* points, uint32_t n, int c, uint32_t* table, void* w,
                               size_t wb, cudaStream_t st) {
  return msm_detail::fixed_table_impl<Fq2>(points, n, c, table, w, wb, st);
}

}  // namespace csb
