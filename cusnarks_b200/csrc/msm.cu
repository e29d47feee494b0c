// msm.cu -- MSM window choice and workspace sizing (kernels: msm_impl.cuh).
#include "msm_impl.cuh"

namespace csb {

int msm_default_window(uint32_t n, bool ec2) {
  // minimise W * (n * madd + 2 * 2^(c-1) * add) with madd ~ 10, add ~ 14 field products
  int best = 8;
  double best_cost = 1e300;
  for (int c = 6; c <= 20; c++) {
    const double W = msm_detail::num_windows(c);
    const double cost = W * ((double)n * 10.0 + 2.0 * (double)(1u << (c - 1)) * 14.0) + 9.0 * 256;
    if (cost < best_cost) { best_cost = cost; best = c; }
  }
  (void)ec2;
  return best;
}

size_t msm_workspace_bytes(uint32_t n, int c, bool ec2) {
  if (c <= 0) c = msm_default_window(n, ec2);
  const int xb = ec2 ? 256 : 128;
  return msm_detail::make_layout(n, c, xb, msm_detail::kMinTask).total;
}

}  // namespace csb
