// setup.cu -- GPU proving-key generation and synthetic-circuit witness evaluation.
//
// The reference builds proving keys in src/python/groth_setup.py (calculateValuesAtT :771,
// calculateEncryptedValuesAtT :488): Lagrange basis values at the toxic point t, the wire
// polynomials u_i(t), v_i(t), w_i(t) from the QAP matrices, the C scalars
// (beta u_i + alpha v_i + w_i)/delta and the hExps scalars t^j Z(t)/delta, then fixed-base
// scalar multiplications (its sc1mulecjac kernel).  These kernels compute the same
// quantities on the device so proving keys for 2^20-constraint circuits are built in
// seconds; the point multiplications use cs_scmul_device.
#include <cstdint>
#include <mutex>

#include "../../include/cusnarks_b200.h"
#include "curve.cuh"
#include "runtime.cuh"

namespace csb {
struct Domain;
cudaError_t domain_get(cs_ctx* ctx, uint32_t L, Domain** out);
const uint32_t* domain_wf(const Domain* d);
const uint32_t* domain_consts(const Domain* d);
}  // namespace csb

using namespace csb;

namespace {

// zm = (t^m - 1) / m (Montgomery)
__global__ void k_lagrange_prefix(const uint32_t* __restrict__ t, uint32_t L, const uint32_t* __restrict__ dom_consts,
                                  uint32_t* __restrict__ zm) {
  if (threadIdx.x != 0) return;
  Fr tm = ld_fp<ModR>(t);
  for (uint32_t k = 0; k < L; k++) tm = tm.sqr();
  st_fp<ModR>(zm, (tm - Fr::one()) * ld_fp<ModR>(dom_consts + 16));  // consts[2] = m^-1 R
}

// L_c(t) = w^c (t^m - 1) / (m (t - w^c)), c < m; Wf: w^j for j < m/2 (w^(j+m/2) = -w^j)
__global__ void k_lagrange(const uint32_t* __restrict__ t, const uint32_t* __restrict__ Wf, uint32_t m,
                           const uint32_t* __restrict__ zm, uint32_t* __restrict__ out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m) return;
  const uint32_t h = m >> 1;
  Fr wc = ld_fp<ModR>(Wf + (size_t)(c < h ? c : c - h) * 8);
  if (c >= h) wc = wc.neg();
  const Fr den = ld_fp<ModR>(t) - wc;
  st_fp<ModR>(out + (size_t)c * 8, ld_fp<ModR>(zm) * wc * den.inv());
}

// u_i = sum over wire i's (c, coeff) of coeff * L_c (reference mpoly layout, Montgomery)
__global__ void k_wire_eval(const uint32_t* __restrict__ mpoly, const uint32_t* __restrict__ start,
                            uint32_t n_wires, const uint32_t* __restrict__ Lc, uint32_t n_rows,
                            uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_wires) return;
  const uint32_t nc = mpoly[1 + i];
  const uint64_t block = 1ull + n_wires + 9ull * start[i];
  Fr acc = Fr::zero();
  for (uint32_t k = 0; k < nc; k++) {
    const uint32_t c = mpoly[block + k];
    if (c >= n_rows) continue;
    Fr v;
    const uint32_t* src = mpoly + block + nc + 8ull * k;
    for (int w = 0; w < 8; w++) v.v[w] = src[w];
    acc = acc + v * ld_fp<ModR>(Lc + (size_t)c * 8);
  }
  st_fp<ModR>(out + (size_t)i * 8, acc);
}

// out_i (normal form) = (beta u_i + alpha v_i + w_i) * k (all Montgomery in)
__global__ void k_c_scalars(const uint32_t* __restrict__ u, const uint32_t* __restrict__ v,
                            const uint32_t* __restrict__ w, const uint32_t* __restrict__ alpha,
                            const uint32_t* __restrict__ beta, const uint32_t* __restrict__ k, uint32_t n,
                            uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Fr x = ld_fp<ModR>(beta) * ld_fp<ModR>(u + (size_t)i * 8) + ld_fp<ModR>(alpha) * ld_fp<ModR>(v + (size_t)i * 8) +
               ld_fp<ModR>(w + (size_t)i * 8);
  st_fp<ModR>(out + (size_t)i * 8, (x * ld_fp<ModR>(k)).from_mont());
}

// out_j (normal form) = t^j * k, j < n (k Montgomery)
__global__ void k_pow_scalars(const uint32_t* __restrict__ t, const uint32_t* __restrict__ k, uint32_t n,
                              uint32_t per, uint32_t* __restrict__ out) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t first = (uint64_t)g * per;
  if (first >= n) return;
  const Fr tt = ld_fp<ModR>(t);
  Fr acc = ld_fp<ModR>(k), base = tt;
  uint64_t e = first;
  while (e) {
    if (e & 1) acc = acc * base;
    base = base.sqr();
    e >>= 1;
  }
  for (uint32_t j = 0; j < per && first + j < n; j++) {
    st_fp<ModR>(out + (first + j) * 8, acc.from_mont());
    acc = acc * tt;
  }
}

// Synthetic R1CS layer: out_c = (A_c . w)(B_c . w), normal form; rows in CSR with Montgomery
// coefficients, witness normal form.
__global__ void k_layer_eval(const uint32_t* __restrict__ a_off, const uint32_t* __restrict__ a_wire,
                             const uint32_t* __restrict__ a_coeff, const uint32_t* __restrict__ b_off,
                             const uint32_t* __restrict__ b_wire, const uint32_t* __restrict__ b_coeff,
                             uint32_t n_rows, const uint32_t* __restrict__ w, uint32_t* __restrict__ out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_rows) return;
  Fr sa = Fr::zero(), sb = Fr::zero();  // Montgomery product of Mont coeff and normal w = normal
  for (uint32_t k = a_off[c]; k < a_off[c + 1]; k++)
    sa = sa + ld_fp<ModR>(a_coeff + (size_t)k * 8) * ld_fp<ModR>(w + (size_t)a_wire[k] * 8);
  for (uint32_t k = b_off[c]; k < b_off[c + 1]; k++)
    sb = sb + ld_fp<ModR>(b_coeff + (size_t)k * 8) * ld_fp<ModR>(w + (size_t)b_wire[k] * 8);
  st_fp<ModR>(out + (size_t)c * 8, (sa * sb) * Fr::r2());  // (sa sb R^-1) R^2 R^-1 = sa sb
}

__global__ void k_wire_counts2(const uint32_t* __restrict__ mpoly, uint32_t n_wires, uint32_t* __restrict__ cnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_wires) cnt[i] = mpoly[1 + i];
  if (i == n_wires) cnt[i] = 0;
}

}  // namespace

namespace csb {
cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, void* tmp, cudaStream_t stream);
size_t scan_workspace_bytes(size_t n);
}  // namespace csb

extern "C" {

int cs_setup_lagrange(cs_ctx* ctx, uint32_t log_m, const uint32_t* d_t, uint32_t* d_out) {
  if (!ctx || !d_t || !d_out || log_m < 1 || log_m > 26) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  Domain* dom = nullptr;
  cudaError_t e = domain_get(ctx, log_m, &dom);
  if (e != cudaSuccess) return fail(ctx, e, "lagrange tables");
  if ((e = ctx->out.reserve(256, ctx->stream)) != cudaSuccess) return fail(ctx, e, "lagrange buffer");
  uint32_t* zm = static_cast<uint32_t*>(ctx->out.ptr);
  const uint32_t m = 1u << log_m;
  k_lagrange_prefix<<<1, 32, 0, ctx->stream>>>(d_t, log_m, domain_consts(dom), zm);
  k_lagrange<<<(m + 127) / 128, 128, 0, ctx->stream>>>(d_t, domain_wf(dom), m, zm, d_out);
  note_launch(2);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(ctx, e, "lagrange launch");
  return CS_OK;
}

int cs_setup_wire_eval(cs_ctx* ctx, const uint32_t* d_mpoly, uint32_t n_wires, const uint32_t* d_L, uint32_t n_rows,
                       uint32_t* d_out) {
  if (!ctx || !d_mpoly || !d_L || !d_out) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  const size_t cb = (((size_t)n_wires + 1) * 4 + 255) & ~size_t(255);
  cudaError_t e = ctx->work.reserve(2 * cb + scan_workspace_bytes((size_t)n_wires + 1), ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "wire eval scratch");
  uint32_t* cnt = static_cast<uint32_t*>(ctx->work.ptr);
  uint32_t* start = reinterpret_cast<uint32_t*>(static_cast<char*>(ctx->work.ptr) + cb);
  void* tmp = static_cast<char*>(ctx->work.ptr) + 2 * cb;
  k_wire_counts2<<<(n_wires + 256) / 256, 256, 0, ctx->stream>>>(d_mpoly, n_wires, cnt);
  note_launch();
  if ((e = scan_exclusive_u32(cnt, start, (size_t)n_wires + 1, tmp, ctx->stream)) != cudaSuccess)
    return fail(ctx, e, "wire eval scan");
  k_wire_eval<<<(n_wires + 127) / 128, 128, 0, ctx->stream>>>(d_mpoly, start, n_wires, d_L, n_rows, d_out);
  note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(ctx, e, "wire eval launch");
  return CS_OK;
}

int cs_setup_c_scalars(cs_ctx* ctx, const uint32_t* d_u, const uint32_t* d_v, const uint32_t* d_w, const uint32_t* d_alpha,
                       const uint32_t* d_beta, const uint32_t* d_k, uint32_t n, uint32_t* d_out) {
  if (!ctx || !d_u || !d_v || !d_w || !d_alpha || !d_beta || !d_k || !d_out) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  if (n) {
    k_c_scalars<<<(n + 255) / 256, 256, 0, ctx->stream>>>(d_u, d_v, d_w, d_alpha, d_beta, d_k, n, d_out);
    note_launch();
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CS_OK : fail(ctx, e, "c scalars");
}

int cs_setup_pow_scalars(cs_ctx* ctx, const uint32_t* d_t, const uint32_t* d_k, uint32_t n, uint32_t* d_out) {
  if (!ctx || !d_t || !d_k || !d_out) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  const uint32_t per = 64, threads = (n + per - 1) / per;
  if (n) {
    k_pow_scalars<<<(threads + 127) / 128, 128, 0, ctx->stream>>>(d_t, d_k, n, per, d_out);
    note_launch();
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CS_OK : fail(ctx, e, "pow scalars");
}

int cs_r1cs_layer_eval(cs_ctx* ctx, const uint32_t* a_off, const uint32_t* a_wire, const uint32_t* a_coeff,
                       const uint32_t* b_off, const uint32_t* b_wire, const uint32_t* b_coeff, uint32_t n_rows,
                       const uint32_t* d_w, uint32_t* d_out) {
  if (!ctx || !a_off || !b_off || !d_w || !d_out) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  if (n_rows) {
    k_layer_eval<<<(n_rows + 127) / 128, 128, 0, ctx->stream>>>(a_off, a_wire, a_coeff, b_off, b_wire, b_coeff,
                                                                 n_rows, d_w, d_out);
    note_launch();
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CS_OK : fail(ctx, e, "layer eval");
}

}  // extern "C"
