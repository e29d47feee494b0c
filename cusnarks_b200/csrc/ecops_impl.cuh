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

// Jacobian (X, Y, Z) points (x = X/Z^2, y = Y/Z^3) -> affine; Z = 0 -> (0, 1).
template <class F>
__global__ void k_jac_to_affine(const uint32_t* __restrict__ jac, uint32_t n, uint32_t* __restrict__ aff) {
  constexpr int FW = FieldWords<F>::value;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* p = jac + (size_t)i * 3 * FW;
  F X, Y, Z;
  ld_field(X, p);
  ld_field(Y, p + FW);
  ld_field(Z, p + 2 * FW);
  Affine<F> r{F::zero(), F::one()};
  if (!Z.is_zero()) {
    const F zi = Z.inv();
    const F zi2 = zi.sqr();
    r.x = X * zi2;
    r.y = Y * (zi2 * zi);
  }
  st_affine<F>(aff + (size_t)i * 2 * FW, r);
}

// Affine points (2 coordinates) -> 3-coordinate rows (x, y, 1); infinity (0, 1) -> the
// reference's Jacobian infinity (0, 1, 0).
template <class F>
__global__ void k_affine_to_jac(const uint32_t* __restrict__ aff, uint32_t n, uint32_t* __restrict__ jac) {
  constexpr int FW = FieldWords<F>::value;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Affine<F> a = ld_affine<F>(aff + (size_t)i * 2 * FW);
  uint32_t* o = jac + (size_t)i * 3 * FW;
  st_field(o, a.x);
  st_field(o + FW, a.y);
  st_field(o + 2 * FW, affine_is_inf(a) ? F::zero() : F::one());
}

// Sum of n points (affine rows of 2 coordinates, or Jacobian rows of 3) in one block:
// strided XYZZ partial sums, then a shared-memory tree; the affine result to out.
template <class F>
__global__ void __launch_bounds__(128) k_point_sum(const uint32_t* __restrict__ pts, uint32_t n, int dims,
                                                   uint32_t* __restrict__ out) {
  constexpr int FW = FieldWords<F>::value;
  constexpr int XW = 4 * FW;
  __shared__ uint32_t red[128][XW];
  XYZZ<F> acc = XYZZ<F>::inf();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t* p = pts + (size_t)i * dims * FW;
    XYZZ<F> q;
    ld_field(q.X, p);
    ld_field(q.Y, p + FW);
    if (dims == 3) {  // Jacobian: ZZ = Z^2, ZZZ = Z^3 (Z = 0: infinity)
      F Z;
      ld_field(Z, p + 2 * FW);
      q.ZZ = Z.sqr();
      q.ZZZ = q.ZZ * Z;
      if (Z.is_zero()) q = XYZZ<F>::inf();
    } else {
      const Affine<F> a{q.X, q.Y};
      q = affine_is_inf(a) ? XYZZ<F>::inf() : XYZZ<F>::from_affine(a);
    }
    acc = xyzz_add_cold(acc, q);
  }
  {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(&acc);
    for (int k = 0; k < XW; k++) red[threadIdx.x][k] = w[k];
  }
  __syncthreads();
  for (int d = blockDim.x / 2; d > 0; d >>= 1) {
    if ((int)threadIdx.x < d) {
      XYZZ<F> a, b;
      uint32_t* wa = reinterpret_cast<uint32_t*>(&a);
      uint32_t* wb = reinterpret_cast<uint32_t*>(&b);
      for (int k = 0; k < XW; k++) { wa[k] = red[threadIdx.x][k]; wb[k] = red[threadIdx.x + d][k]; }
      a = xyzz_add_cold(a, b);
      for (int k = 0; k < XW; k++) red[threadIdx.x][k] = wa[k];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    XYZZ<F> a;
    uint32_t* wa = reinterpret_cast<uint32_t*>(&a);
    for (int k = 0; k < XW; k++) wa[k] = red[0][k];
    st_affine<F>(out, xyzz_to_affine(a));
  }
}

// Curve check of one point (affine, or Jacobian when jac): 2 = the infinity encoding,
// 1 = on y^2 = x^3 + b, 0 = not on the curve.
template <class F>
CSB_DEV F curve_b();
template <>
CSB_DEV Fq curve_b<Fq>() {
  return Fq{{0x50ad28d7u, 0x7a17caa9u, 0xe15521b9u, 0x1f6ac17au, 0x696bd284u, 0x334bea4eu, 0xce179d8eu, 0x2a1f6744u}};
}
template <>
CSB_DEV Fq2 curve_b<Fq2>() {  // 3 / (9 + u), Montgomery
  return Fq2{Fq{{0x77b802a8u, 0x3bf938e3u, 0x3633535du, 0x020b1b27u, 0x49755260u, 0x26b7edf0u, 0x4384a86du, 0x2514c632u}},
             Fq{{0xd1dcff67u, 0x38e7ecccu, 0x93ce0d3eu, 0x65f0b37du, 0x22ac00aau, 0xd749d0ddu, 0x4a688d4du, 0x0141b9ceu}}};
}

template <class F>
__global__ void k_on_curve(const uint32_t* __restrict__ p, int jac, uint32_t* __restrict__ flag) {
  constexpr int FW = FieldWords<F>::value;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  F X, Y, Z = F::one();
  ld_field(X, p);
  ld_field(Y, p + FW);
  if (jac) ld_field(Z, p + 2 * FW);
  if (X.is_zero() && Y == F::one()) { *flag = 2u; return; }  // as ec_iseq_h: X and Y only
  // Y^2 = X^3 + b Z^6
  const F z2 = Z.sqr();
  const F z6 = z2.sqr() * z2;
  *flag = (Y.sqr() == X.sqr() * X + curve_b<F>() * z6) ? 1u : 0u;
}

// Subset-sum tables of groups of `order` affine points (the reference's ec_inittable_h,
// src/cuda/ec.cpp:574): entry j of table t is the sum of the points t*order + b over the set
// bits b of j (points past n count as infinity); affine out, infinity (0, 1).
template <class F>
__global__ void __launch_bounds__(128) k_subset_table(const uint32_t* __restrict__ aff, uint32_t n, uint32_t order,
                                                      uint64_t entries, uint32_t* __restrict__ out) {
  constexpr int PW = 2 * FieldWords<F>::value;
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= entries) return;
  const uint64_t t = g >> order;
  const uint32_t j = (uint32_t)(g & ((1ull << order) - 1));
  XYZZ<F> acc = XYZZ<F>::inf();
#pragma unroll 1
  for (uint32_t b = 0; b < order; b++) {
    const uint64_t idx = t * order + b;
    if (((j >> b) & 1u) && idx < n) {
      const Affine<F> a = ld_affine<F>(aff + idx * PW);
      if (!affine_is_inf(a)) acc = xyzz_madd(acc, a);
    }
  }
  st_affine<F>(out + g * PW, xyzz_to_affine(acc));
}

template <class F>
cudaError_t subset_table(const uint32_t* aff, uint32_t n, uint32_t order, uint32_t* out, cudaStream_t st) {
  if (n == 0 || order == 0 || order > 16) return n == 0 ? cudaSuccess : cudaErrorInvalidValue;
  const uint64_t tables = ((uint64_t)n + order - 1) / order;
  const uint64_t entries = tables << order;
  k_subset_table<F><<<(unsigned)((entries + 127) / 128), 128, 0, st>>>(aff, n, order, entries, out);
  note_launch();
  return cudaGetLastError();
}

template <class F>
cudaError_t scmul(const uint32_t* s, const uint32_t* p, uint32_t stride, uint32_t n, uint32_t* out,
                  cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_scmul<F><<<(n + 127) / 128, 128, 0, st>>>(s, p, stride, n, out);
  note_launch();
  return cudaGetLastError();
}

template <class F>
cudaError_t jac_to_affine(const uint32_t* jac, uint32_t n, uint32_t* aff, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_jac_to_affine<F><<<(n + 127) / 128, 128, 0, st>>>(jac, n, aff);
  note_launch();
  return cudaGetLastError();
}

template <class F>
cudaError_t affine_to_jac(const uint32_t* aff, uint32_t n, uint32_t* jac, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_affine_to_jac<F><<<(n + 127) / 128, 128, 0, st>>>(aff, n, jac);
  note_launch();
  return cudaGetLastError();
}

template <class F>
cudaError_t point_sum(const uint32_t* pts, uint32_t n, int dims, uint32_t* out, cudaStream_t st) {
  k_point_sum<F><<<1, 128, 0, st>>>(pts, n, dims, out);
  note_launch();
  return cudaGetLastError();
}

template <class F>
cudaError_t on_curve(const uint32_t* p, int jac, uint32_t* flag, cudaStream_t st) {
  k_on_curve<F><<<1, 32, 0, st>>>(p, jac, flag);
  note_launch();
  return cudaGetLastError();
}

}  // namespace ecops_detail
}  // namespace csb
