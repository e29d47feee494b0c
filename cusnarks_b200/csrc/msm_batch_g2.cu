// msm_batch_g2.cu -- G2 (Fq2) instantiation of the batched MSM (msm_batch.cuh).
// Montgomery products out of line, as in the single MSM (instruction-cache fit).
#define CSB_MUL_NOINLINE
#include "msm_batch.cuh"

namespace csb {

cudaError_t msm_batch_g2(const MsmBatch& b, void* w, size_t wb, cudaStream_t st) {
  return msm_detail::batch_impl<Fq2>(b, w, wb, st);
}

}  // namespace csb
