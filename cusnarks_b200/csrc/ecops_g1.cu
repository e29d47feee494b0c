// ecops_g1.cu -- G1 instantiation of the batched scalar multiplication.
#include "ecops_impl.cuh"

namespace csb {
cudaError_t scmul_g1(const uint32_t* s, const uint32_t* p, uint32_t stride, uint32_t n, uint32_t* out,
                     cudaStream_t st) {
  return ecops_detail::scmul<Fq>(s, p, stride, n, out, st);
}
}  // namespace csb
