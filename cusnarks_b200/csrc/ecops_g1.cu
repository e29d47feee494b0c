// ecops_g1.cu -- G1 instantiation of the batched scalar multiplication.
#include "ecops_impl.cuh"

namespace csb {
cudaError_t scmul_g1(const uint32_t* s, const uint32_t* p, uint32_t stride, uint32_t n, uint32_t* out,
                     cudaStream_t st) {
  return ecops_detail::scmul<Fq>(s, p, stride, n, out, st);
}
cudaError_t jac_to_affine_g1(const uint32_t* jac, uint32_t n, uint32_t* aff, cudaStream_t st) {
  return ecops_detail::jac_to_affine<Fq>(jac, n, aff, st);
}
cudaError_t affine_to_jac_g1(const uint32_t* aff, uint32_t n, uint32_t* jac, cudaStream_t st) {
  return ecops_detail::affine_to_jac<Fq>(aff, n, jac, st);
}
cudaError_t point_sum_g1(const uint32_t* pts, uint32_t n, int dims, uint32_t* out, cudaStream_t st) {
  return ecops_detail::point_sum<Fq>(pts, n, dims, out, st);
}
cudaError_t on_curve_g1(const uint32_t* p, int jac, uint32_t* flag, cudaStream_t st) {
  return ecops_detail::on_curve<Fq>(p, jac, flag, st);
}
cudaError_t subset_table_g1(const uint32_t* aff, uint32_t n, uint32_t order, uint32_t* out, cudaStream_t st) {
  return ecops_detail::subset_table<Fq>(aff, n, order, out, st);
}
}  // namespace csb
