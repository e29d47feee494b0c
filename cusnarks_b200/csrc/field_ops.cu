// field_ops.cu -- elementwise field arithmetic on device arrays, and the reference's
// host field entry points (src/cuda/ff.cpp, bound at src/cython/_utils_host.pxd:41-65)
// running through the same kernels.
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/cusnarks_b200.h"
#include "curve.cuh"
#include "runtime.cuh"

namespace {

using namespace csb;

template <class M>
__global__ void k_field_op(int op, const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                           uint32_t* __restrict__ out, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  using F = Fp<M>;
  F x = ld_fp<M>(a + (size_t)i * 8);
  F y = F::zero();
  if (op == CS_FOP_MUL || op == CS_FOP_ADD || op == CS_FOP_SUB || op == CS_FOP_MUL_DP52)
    y = ld_fp<M>(b + (size_t)i * 8);
  F r;
  switch (op) {
    case CS_FOP_MUL: r = x * y; break;
    case CS_FOP_ADD: r = x + y; break;
    case CS_FOP_SUB: r = x - y; break;
    case CS_FOP_SQR: r = x.sqr(); break;
    case CS_FOP_INV: r = x.inv(); break;
    case CS_FOP_TO_MONT: r = x.to_mont(); break;
    case CS_FOP_FROM_MONT: r = x.from_mont(); break;
    default: dp52::mont<M>(x.v, y.v, r.v); r = r.canon(); break;  // CS_FOP_MUL_DP52
  }
  st_fp<M>(out + (size_t)i * 8, r);
}

__global__ void k_fq2_mul(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                          uint32_t* __restrict__ out, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Fq2 x, y;
  ld_field(x, a + (size_t)i * 16);
  ld_field(y, b + (size_t)i * 16);
  st_field(out + (size_t)i * 16, x * y);
}

cudaError_t launch_field_op(int op, int pidx, const uint32_t* a, const uint32_t* b, uint32_t* out,
                            uint32_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int T = 256;
  if (op == CS_FOP_FQ2_MUL)
    k_fq2_mul<<<(n + T - 1) / T, T, 0, st>>>(a, b, out, n);
  else if (pidx == 0)
    k_field_op<ModQ><<<(n + T - 1) / T, T, 0, st>>>(op, a, b, out, n);
  else
    k_field_op<ModR><<<(n + T - 1) / T, T, 0, st>>>(op, a, b, out, n);
  note_launch();
  return cudaGetLastError();
}

thread_local int t_field_status = CS_OK;

// Host-pointer helper for the drop-in entry points: copy in, run, copy out, on the
// calling thread's default context.
int host_field_op(int op, int pidx, const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n) {
  cs_ctx* ctx = nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return CS_ERR_NODEVICE; }
  static std::mutex mu;
  static cs_ctx* ctxs[64] = {nullptr};
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64) return CS_ERR_NODEVICE;
    if (!ctxs[dev] && cs_ctx_create(dev, &ctxs[dev]) != CS_OK) return CS_ERR_NODEVICE;
    ctx = ctxs[dev];
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  const size_t w = (op == CS_FOP_FQ2_MUL) ? 16 : 8;
  const size_t bytes = (size_t)n * w * 4, al = (bytes + 255) & ~size_t(255);
  cudaError_t e = ctx->in.reserve(3 * al + 256, ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "field op buffer");
  uint32_t* da = static_cast<uint32_t*>(ctx->in.ptr);
  uint32_t* db = reinterpret_cast<uint32_t*>(static_cast<char*>(ctx->in.ptr) + al);
  uint32_t* dout = reinterpret_cast<uint32_t*>(static_cast<char*>(ctx->in.ptr) + 2 * al);
  if (n) {
    if ((e = cudaMemcpyAsync(da, a, bytes, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return fail(ctx, e, "field op H2D");
    if (b && (e = cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return fail(ctx, e, "field op H2D");
  }
  if ((e = launch_field_op(op, pidx, da, b ? db : da, dout, n, ctx->stream)) != cudaSuccess)
    return fail(ctx, e, "field op launch");
  if (n && (e = cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
    return fail(ctx, e, "field op D2H");
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(ctx, e, "field op sync");
  return CS_OK;
}

}  // namespace

extern "C" {

int cs_field_op_device(cs_ctx* ctx, int op, int pidx, const uint32_t* d_a, const uint32_t* d_b,
                       uint32_t* d_out, uint32_t n) {
  if (!ctx || op < 0 || op > CS_FOP_MUL_DP52 || op == 7 || (pidx != 0 && pidx != 1)) return CS_ERR_ARG;
  if (n && (!d_a || !d_out)) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaEventRecord(ctx->ev_start, ctx->stream);
  cudaError_t e = launch_field_op(op, pidx, d_a, d_b ? d_b : d_a, d_out, n, ctx->stream);
  cudaEventRecord(ctx->ev_stop, ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "field op launch");
  return CS_OK;
}

int cs_field_last_status(void) { return t_field_status; }

void montmult_h(uint32_t* U, const uint32_t* A, const uint32_t* B, uint32_t pidx) {
  t_field_status = (pidx > 1) ? CS_ERR_ARG : host_field_op(CS_FOP_MUL, (int)pidx, A, B, U, 1);
}
void montsquare_h(uint32_t* U, const uint32_t* A, uint32_t pidx) {
  t_field_status = (pidx > 1) ? CS_ERR_ARG : host_field_op(CS_FOP_SQR, (int)pidx, A, nullptr, U, 1);
}
void addm_h(uint32_t* U, const uint32_t* A, const uint32_t* B, uint32_t pidx) {
  t_field_status = (pidx > 1) ? CS_ERR_ARG : host_field_op(CS_FOP_ADD, (int)pidx, A, B, U, 1);
}
void subm_h(uint32_t* U, const uint32_t* A, const uint32_t* B, uint32_t pidx) {
  t_field_status = (pidx > 1) ? CS_ERR_ARG : host_field_op(CS_FOP_SUB, (int)pidx, A, B, U, 1);
}
void montinv_h(uint32_t* y, uint32_t* x, uint32_t pidx) {
  t_field_status = (pidx > 1) ? CS_ERR_ARG : host_field_op(CS_FOP_INV, (int)pidx, x, nullptr, y, 1);
}
void to_montgomeryN_h(uint32_t* z, const uint32_t* x, uint32_t n, uint32_t pidx) {
  t_field_status = (pidx > 1) ? CS_ERR_ARG : host_field_op(CS_FOP_TO_MONT, (int)pidx, x, nullptr, z, n);
}
void from_montgomeryN_h(uint32_t* z, const uint32_t* x, uint32_t n, uint32_t pidx, uint32_t strip_last) {
  if (pidx > 1 || strip_last != 0) {
    t_field_status = pidx > 1 ? CS_ERR_ARG : CS_ERR_UNSUPPORTED;
    return;
  }
  t_field_status = host_field_op(CS_FOP_FROM_MONT, (int)pidx, x, nullptr, z, n);
}

}  // extern "C"
