// ecops_impl.cuh -- kernels behind ecops.cuh (instantiated in ecops_g1.cu / ecops_g2.cu).
#pragma once
#include "curve.cuh"
#include "ecops.cuh"
#include "runtime.cuh"

namespace csb {
namespace ecops_detail {

// Left-to-right double-and-add over all 256 scalar bits with an XYZZ accumulator and
// mixed additions of the affine base; one inversion per point for the affine result.
template <class F>
__global__ void __launch_bounds__(128) k_scmul(const uint32_t* __restrict__ scalars,
                                               const uint32_t* __restrict__ points,
                                               uint32_t stride, uint32_t n,
                                               uint32_t* __restrict__ out) {
  constexpr int PW = 2 * FieldWords<F>::value;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k[8];
  ld_limbs8(k, scalars + (size_t)i * 8);
  const uint32_t* pp = points + (size_t)i * stride;
  Affine<F> P = ld_affine<F>(pp);
  XYZZ<F> acc = XYZZ<F>::inf();
  bool inf_in = P.x.is_zero() && P.y == F::one();
  if (!inf_in) {
    int top = 255;
    while (top >= 0 && ((k[top >> 5] >> (top & 31)) & 1u) == 0) top--;
#pragma unroll 1
    for (int b = top; b >= 0; b--) {
      acc = xyzz_dbl(acc);
      if ((k[b >> 5] >> (b & 31)) & 1u) acc = xyzz_madd(acc, P);
    }
  }
  st_affine<F>(out + (size_t)i * PW, xyzz_to_affine(acc));
}

template <class F>
cudaError_t scmul(const uint32_t* s, const uint32_t* p, uint32_t stride, uint32_t n, uint32_t* out,
                  cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_scmul<F><<<(n + 127) / 128, 128, 0, st>>>(s, p, stride, n, out);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ecops_detail
}  // namespace csb
