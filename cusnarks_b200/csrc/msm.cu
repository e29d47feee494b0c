// msm.cu -- MSM window choice and workspace sizing (kernels: msm_impl.cuh).
#include "msm_batch.cuh"

namespace csb {

int msm_default_window(uint32_t n, bool ec2) { return msm_window_model(n, !ec2); }

int msm_window_model(uint32_t n, bool glv) {
  // minimise W * (terms * madd + 2 * 2^(c-1) * add) + Horner with madd ~ 10, add ~ 14 field
  // products; GLV sorts 2n half-scalars (128 bits), otherwise n full scalars
  const double terms = glv ? 2.0 * n : (double)n;
  int best = 8;
  double best_cost = 1e300;
  for (int c = 6; c <= 20; c++) {
    const double W = msm_detail::msm_windows(c, glv);
    const double cost = W * (terms * 10.0 + 2.0 * (double)(1u << (c - 1)) * 14.0) + 9.0 * (glv ? 128 : 256);
    if (cost < best_cost) { best_cost = cost; best = c; }
  }
  return best;
}

size_t msm_workspace_bytes(uint32_t n, int c, bool ec2, int affine_mode, int glv_mode, int min_task) {
  if (c <= 0) c = msm_default_window(n, ec2);
  const int xb = ec2 ? 256 : 128;
  const bool glv = msm_detail::use_glv(ec2, false, glv_mode, affine_mode, n);
  return msm_detail::make_layout(n, c, xb, min_task > 0 ? (uint32_t)min_task : 0u, false,
                                 msm_detail::layout_affine(ec2, affine_mode, n, c, false, glv), glv).total;
}

int msm_fixed_window(uint32_t n, bool ec2) {
  // one bucket set: W * n * madd + 2 * 2^(c-1) * add
  int best = 8;
  double best_cost = 1e300;
  for (int c = 6; c <= 22; c++) {
    const double W = msm_detail::num_windows(c);
    const double cost = W * (double)n * 10.0 + 2.0 * (double)(1u << (c - 1)) * 14.0;
    if (cost < best_cost) { best_cost = cost; best = c; }
  }
  (void)ec2;
  return best;
}

size_t msm_batch_workspace_bytes(const MsmBatch& b, bool ec2) {
  return msm_detail::batch_layout(b, ec2 ? 256 : 128).total;
}

size_t msm_fixed_table_points(uint32_t n, int c) { return (size_t)msm_detail::num_windows(c) * n; }

size_t msm_fixed_table_work_bytes(uint32_t n, bool ec2) {
  return msm_detail::fixed_table_work_bytes(n, ec2 ? 256 : 128, ec2 ? 64 : 32);
}

size_t msm_fixed_workspace_bytes(uint32_t n, int c, bool ec2, int affine_mode) {
  if (c <= 0) c = msm_fixed_window(n, ec2);
  return msm_detail::make_layout(n, c, ec2 ? 256 : 128, 0u, true,
                                 msm_detail::layout_affine(ec2, affine_mode, n, c, true)).total;
}

}  // namespace csb
