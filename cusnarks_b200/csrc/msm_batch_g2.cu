// msm_batch_g2.cu -- G2 (Fq2) instantiation of the batched MSM (msm_batch.cuh).
// Montgomery products out of line, as in the single MSM (instruction-cache fit).
#define CSB_MUL_NOINLINE
// Fq products stay 32-bit CIOS here: the FP64-pipe product needs more registers than
// the 168 the Fq2 kernels run at (G2 fixed-base MSM 13.1 -> 13.9 ms with it).
#ifndef CSB_DP52
#define CSB_DP52 0
#endif
#include "msm_batch.cuh"

namespace csb {

cudaError_t msm_batch_g2(const MsmBatch& b, void* w, size_t wb, cudaStream_t st) {
  return msm_detail::batch_impl<Fq2>(b, w, wb, st);
}

}  // namespace csb
