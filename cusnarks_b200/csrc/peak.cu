// peak.cu -- integer-pipe ceiling used as the roofline denominator for the integer-bound
// kernels (MSM, NTT): sustained 32-bit multiply-add instruction rate of the device,
// measured with independent mad.lo / mad.hi chains (the instruction mix of a CIOS
// Montgomery product) on every SM.
#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/cusnarks_b200.h"
#include "runtime.cuh"
#include "field.cuh"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) k_imad_peak(uint32_t seed, uint32_t* sink) {
  uint32_t a[kChains];
#pragma unroll
  for (int i = 0; i < kChains; i++) a[i] = seed + threadIdx.x * 7u + i;
  const uint32_t b = seed * 3u + 1u;
#pragma unroll 1
  for (int it = 0; it < kIters; it++) {
#pragma unroll
    for (int i = 0; i < kChains; i += 2) {
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[i]) : "r"(b), "r"(a[i + 1]));
      asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(a[i + 1]) : "r"(b), "r"(a[i]));
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int i = 0; i < kChains; i++) x ^= a[i];
  if (x == 0x9e3779b9u) sink[0] = x;  // keeps the chains live
}

// Pipe-rate probes: mode 1 mad.lo only, 2 mad.hi only, 3 mad.wide.u32 (64-bit
// accumulate), 4 fma.rn.f64, 5 CIOS-like carry chains (mad.lo.cc / madc.hi.cc).
template <int MODE>
__global__ void __launch_bounds__(256) k_pipe(uint32_t seed, uint32_t* sink) {
  uint32_t a[kChains];
  uint64_t w[kChains];
  double d[kChains];
#pragma unroll
  for (int i = 0; i < kChains; i++) {
    a[i] = seed + threadIdx.x * 7u + i;
    w[i] = a[i];
    d[i] = (double)a[i] * 1e-9;
  }
  const uint32_t b = seed * 3u + 1u;
  #pragma unroll 1
  for (int it = 0; it < kIters; it++) {
#pragma unroll
    for (int i = 0; i < kChains; i++) {
      if (MODE == 1) asm volatile("mad.lo.u32 %0, %0, %1, %0;" : "+r"(a[i]) : "r"(b));
      if (MODE == 2) asm volatile("mad.hi.u32 %0, %0, %1, %0;" : "+r"(a[i]) : "r"(b));
      if (MODE == 3)
        asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(w[i]) : "r"((uint32_t)w[(i + 1) % kChains]), "r"(b));
      if (MODE == 4) asm volatile("fma.rn.f64 %0, %0, %1, %0;" : "+d"(d[i]) : "d"(d[(i + 1) % kChains]));
    }
    if (MODE == 5) {
      asm volatile("mad.lo.cc.u32 %0, %0, %1, %0;" : "+r"(a[0]) : "r"(b));
#pragma unroll
      for (int i = 1; i < kChains; i++) asm volatile("madc.lo.cc.u32 %0, %0, %1, %0;" : "+r"(a[i]) : "r"(b));
      asm volatile("mad.hi.cc.u32 %0, %0, %1, %0;" : "+r"(a[0]) : "r"(b));
#pragma unroll
      for (int i = 1; i < kChains; i++) asm volatile("madc.hi.cc.u32 %0, %0, %1, %0;" : "+r"(a[i]) : "r"(b));
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int i = 0; i < kChains; i++) x ^= a[i] ^ (uint32_t)w[i] ^ (uint32_t)(d[i] > 3.0);
  if (x == 0x9e3779b9u) sink[0] = x;
}

// Montgomery-product throughput: 4 independent dependent chains x <- x * y per thread.
template <int VARIANT>
__global__ void __launch_bounds__(256) k_mulmod(const uint32_t* __restrict__ seed, uint32_t* sink, int iters) {
  using csb::Fq;
  Fq x[4], y;
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int i = 0; i < 8; i++) x[k].v[i] = seed[i] ^ (threadIdx.x * 13u + k * 7u + i);
#pragma unroll
  for (int i = 0; i < 8; i++) y.v[i] = seed[8 + i];
  x[0].v[7] &= 0x0fffffffu; x[1].v[7] &= 0x0fffffffu; x[2].v[7] &= 0x0fffffffu; x[3].v[7] &= 0x0fffffffu;
  y.v[7] &= 0x0fffffffu;
#pragma unroll 1
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 4; k++) x[k] = VARIANT == 0 ? Fq::mul_lohi(x[k], y) : Fq::mul_wide(x[k], y);
  }
  uint32_t h = 0;
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int i = 0; i < 8; i++) h ^= x[k].v[i];
  if (h == 0x12345u) sink[0] = h;
}

// ALU probe: 8-limb add.cc / addc.cc chains
__global__ void __launch_bounds__(256) k_alu(uint32_t seed, uint32_t* sink) {
  uint32_t a[8], b[8];
#pragma unroll
  for (int i = 0; i < 8; i++) { a[i] = seed + threadIdx.x + i; b[i] = seed * 5u + i; }
#pragma unroll 1
  for (int it = 0; it < kIters; it++) {
    asm volatile("add.cc.u32 %0, %0, %8;\n\taddc.cc.u32 %1, %1, %9;\n\taddc.cc.u32 %2, %2, %10;\n\t"
                 "addc.cc.u32 %3, %3, %11;\n\taddc.cc.u32 %4, %4, %12;\n\taddc.cc.u32 %5, %5, %13;\n\t"
                 "addc.cc.u32 %6, %6, %14;\n\taddc.u32 %7, %7, %15;"
                 : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7])
                 : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
    asm volatile("add.cc.u32 %0, %0, %8;\n\taddc.cc.u32 %1, %1, %9;\n\taddc.cc.u32 %2, %2, %10;\n\t"
                 "addc.cc.u32 %3, %3, %11;\n\taddc.cc.u32 %4, %4, %12;\n\taddc.cc.u32 %5, %5, %13;\n\t"
                 "addc.cc.u32 %6, %6, %14;\n\taddc.u32 %7, %7, %15;"
                 : "+r"(b[0]), "+r"(b[1]), "+r"(b[2]), "+r"(b[3]), "+r"(b[4]), "+r"(b[5]), "+r"(b[6]), "+r"(b[7])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]));
  }
  uint32_t x = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) x ^= a[i] ^ b[i];
  if (x == 0x9e3779b9u) sink[0] = x;
}

// Latency probe: one thread runs CHAINS independent dependent chains x <- x * y, with
// the flag-carry CIOS (VARIANT 0), the wide-product CIOS (1) or the carry-flag-free
// 64-bit CIOS (2); or XYZZ point additions acc <- acc + p (VARIANT 3: wide, 4: c64).
template <int VARIANT, int CHAINS>
__global__ void k_mul_latency(const uint32_t* __restrict__ seed, uint32_t* sink, int iters) {
  using csb::Fq;
  Fq x[CHAINS], y;
#pragma unroll
  for (int k = 0; k < CHAINS; k++)
#pragma unroll
    for (int i = 0; i < 8; i++) x[k].v[i] = (seed[i] ^ (k * 977u)) & (i == 7 ? 0x0fffffffu : 0xffffffffu);
#pragma unroll
  for (int i = 0; i < 8; i++) y.v[i] = seed[8 + i] & (i == 7 ? 0x0fffffffu : 0xffffffffu);
#pragma unroll 1
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < CHAINS; k++)
      x[k] = VARIANT == 0 ? Fq::mul_lohi(x[k], y) : VARIANT == 1 ? Fq::mul_wide(x[k], y) : Fq::mul_c64(x[k], y);
  }
  uint32_t h = 0;
#pragma unroll
  for (int k = 0; k < CHAINS; k++)
#pragma unroll
    for (int i = 0; i < 8; i++) h ^= x[k].v[i];
  if (h == 0x12345u) sink[0] = h;
}

}  // namespace

// Nanoseconds per Montgomery product for one thread running `chains` (1 or 4) independent
// chains; variant 0 flag-carry, 1 wide-product, 2 carry-flag-free 64-bit CIOS.
extern "C" int cs_bench_mul_latency(cs_ctx* ctx, int variant, int chains, double* ns_per_mul) {
  if (!ctx || !ns_per_mul || variant < 0 || variant > 2 || (chains != 1 && chains != 4)) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaError_t e = ctx->out.reserve(256, ctx->stream);
  if (e != cudaSuccess) return csb::fail(ctx, e, "latency probe buffer");
  uint32_t* buf = static_cast<uint32_t*>(ctx->out.ptr);
  if ((e = cudaMemsetAsync(buf, 0x5a, 256, ctx->stream)) != cudaSuccess) return csb::fail(ctx, e, "latency probe init");
  const int iters = 2000;
  float best = 1e30f;
  for (int rep = 0; rep < 3; rep++) {
    cudaEventRecord(ctx->ev_start, ctx->stream);
    if (chains == 1) {
      if (variant == 0) k_mul_latency<0, 1><<<1, 1, 0, ctx->stream>>>(buf, buf + 32, iters);
      else if (variant == 1) k_mul_latency<1, 1><<<1, 1, 0, ctx->stream>>>(buf, buf + 32, iters);
      else k_mul_latency<2, 1><<<1, 1, 0, ctx->stream>>>(buf, buf + 32, iters);
    } else {
      if (variant == 0) k_mul_latency<0, 4><<<1, 1, 0, ctx->stream>>>(buf, buf + 32, iters);
      else if (variant == 1) k_mul_latency<1, 4><<<1, 1, 0, ctx->stream>>>(buf, buf + 32, iters);
      else k_mul_latency<2, 4><<<1, 1, 0, ctx->stream>>>(buf, buf + 32, iters);
    }
    csb::note_launch();
    cudaEventRecord(ctx->ev_stop, ctx->stream);
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return csb::fail(ctx, e, "latency probe kernel");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
    if (rep > 0 && ms < best) best = ms;
  }
  *ns_per_mul = (double)best * 1e6 / ((double)iters * chains);
  return CS_OK;
}

extern "C" int cs_bench_mulmod(cs_ctx* ctx, int variant, double* mulmods_per_s) {
  if (!ctx || !mulmods_per_s || variant < 0 || variant > 2) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  cudaError_t e = ctx->out.reserve(256, ctx->stream);
  if (e != cudaSuccess) return csb::fail(ctx, e, "mulmod probe buffer");
  uint32_t* buf = static_cast<uint32_t*>(ctx->out.ptr);
  cudaMemsetAsync(buf, 0x5a, 256, ctx->stream);
  const int threads = 256, blocks = sms * 4, iters = 256;
  float best = 1e30f;
  for (int rep = 0; rep < 3; rep++) {
    cudaEventRecord(ctx->ev_start, ctx->stream);
    if (variant == 0) k_mulmod<0><<<blocks, threads, 0, ctx->stream>>>(buf, buf + 32, iters);
    else if (variant == 1) k_mulmod<1><<<blocks, threads, 0, ctx->stream>>>(buf, buf + 32, iters);
    else k_alu<<<sms * 8, 256, 0, ctx->stream>>>(3u + rep, buf + 32);
    csb::note_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) return csb::fail(ctx, e, "mulmod probe launch");
    cudaEventRecord(ctx->ev_stop, ctx->stream);
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return csb::fail(ctx, e, "mulmod probe kernel");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
    if (rep > 0 && ms < best) best = ms;
  }
  const double ops = variant < 2 ? (double)blocks * threads * iters * 4 : (double)sms * 8 * 256 * kIters * 16;
  *mulmods_per_s = ops / (best * 1e-3);
  return CS_OK;
}

extern "C" int cs_bench_pipe(cs_ctx* ctx, int mode, double* ops_per_s) {
  if (!ctx || !ops_per_s || mode < 1 || mode > 5) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  cudaError_t e = ctx->out.reserve(256, ctx->stream);
  if (e != cudaSuccess) return csb::fail(ctx, e, "pipe probe buffer");
  const int blocks = sms * 8, threads = 256;
  uint32_t* sink = static_cast<uint32_t*>(ctx->out.ptr);
  float best = 1e30f;
  for (int rep = 0; rep < 3; rep++) {
    cudaEventRecord(ctx->ev_start, ctx->stream);
    switch (mode) {
      case 1: k_pipe<1><<<blocks, threads, 0, ctx->stream>>>(7u + rep, sink); break;
      case 2: k_pipe<2><<<blocks, threads, 0, ctx->stream>>>(7u + rep, sink); break;
      case 3: k_pipe<3><<<blocks, threads, 0, ctx->stream>>>(7u + rep, sink); break;
      case 4: k_pipe<4><<<blocks, threads, 0, ctx->stream>>>(7u + rep, sink); break;
      default: k_pipe<5><<<blocks, threads, 0, ctx->stream>>>(7u + rep, sink); break;
    }
    csb::note_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) return csb::fail(ctx, e, "pipe probe launch");
    cudaEventRecord(ctx->ev_stop, ctx->stream);
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return csb::fail(ctx, e, "pipe probe kernel");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
    if (rep > 0 && ms < best) best = ms;
  }
  const double per_iter = (mode == 5) ? 2.0 * kChains : (double)kChains;
  *ops_per_s = (double)blocks * threads * kIters * per_iter / (best * 1e-3);
  return CS_OK;
}

extern "C" int cs_bench_imad_peak(cs_ctx* ctx, double* imad_per_s) {
  if (!ctx || !imad_per_s) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  cudaError_t e = ctx->out.reserve(256, ctx->stream);
  if (e != cudaSuccess) return csb::fail(ctx, e, "imad peak buffer");
  const int blocks = sms * 8, threads = 256;
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(ctx->ev_start, ctx->stream);
    k_imad_peak<<<blocks, threads, 0, ctx->stream>>>(12345u + rep, static_cast<uint32_t*>(ctx->out.ptr));
    csb::note_launch();
    cudaEventRecord(ctx->ev_stop, ctx->stream);
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return csb::fail(ctx, e, "imad peak kernel");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
    if (rep > 0 && ms < best) best = ms;
  }
  const double ops = (double)blocks * threads * kIters * kChains;
  *imad_per_s = ops / (best * 1e-3);
  return CS_OK;
}
