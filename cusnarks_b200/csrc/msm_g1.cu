// msm_g1.cu -- G1 (Fq) instantiation of the MSM pipeline.
#include "msm_impl.cuh"

namespace csb {

cudaError_t msm_g1(const uint32_t* s, const uint32_t* p, uint32_t n, uint32_t* out, void* w,
                   size_t wb, const MsmConfig& cfg, cudaStream_t st) {
  return msm_detail::msm_impl<Fq>(s, p, n, out, w, wb, cfg, st);
}
}  // namespace csb
