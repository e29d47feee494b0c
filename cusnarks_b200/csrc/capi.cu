// capi.cu -- extern "C" entry points (include/cusnarks_b200.h).
#include <atomic>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/cusnarks_b200.h"
#include "ecops.cuh"
#include "msm.cuh"
#include "runtime.cuh"

namespace csb {

void domain_release(cs_ctx* ctx);  // hstep.cu
static std::atomic<unsigned long long> g_launches{0};
thread_local unsigned long long t_launches = 0;
void note_launch(unsigned n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  t_launches += n;
}
unsigned long long thread_launches() { return t_launches; }


// Auxiliary streams of the prove pipeline: aux[0..3] carry the A, B1, B2 (G2) and C MSMs,
// aux_h the QAP -> H step -> H MSM chain.  Priorities (lower number = higher priority)
// decide which MSM's blocks the SMs take first when several are ready.
cudaError_t ctx_aux_init(cs_ctx* ctx) {
  if (ctx->aux_ready) return cudaSuccess;
  int least = 0, greatest = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  // the G2 MSM and the QAP / H chain first (measured 32.0 -> 31.6 ms per 2^20 proof)
  int prio[4] = {least, least, greatest, least}, prio_h = greatest;
  for (int i = 0; i < 4 && e == cudaSuccess; i++)
    if (!ctx->aux[i]) e = cudaStreamCreateWithPriority(&ctx->aux[i], cudaStreamNonBlocking, prio[i]);
  if (e == cudaSuccess && !ctx->aux_h) e = cudaStreamCreateWithPriority(&ctx->aux_h, cudaStreamNonBlocking, prio_h);
  for (int i = 0; i < cs_ctx::kAuxEvents && e == cudaSuccess; i++)
    if (!ctx->aux_ev[i]) e = cudaEventCreate(&ctx->aux_ev[i]);  // timed: prove stage times
  if (e == cudaSuccess) ctx->aux_ready = true;
  return e;
}

int fail(cs_ctx* ctx, cudaError_t e, const char* where) {
  if (ctx) ctx->err = std::string(where) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear the sticky-free error state
  return e == cudaErrorMemoryAllocation ? CS_ERR_NOMEM : CS_ERR_CUDA;
}
int fail_msg(cs_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

}  // namespace csb

using csb::fail;
using csb::fail_msg;

namespace {

thread_local int t_status = CS_OK;
thread_local std::string t_error;

std::mutex g_default_mu;
cs_ctx* g_default[64] = {nullptr};

int set_thread_status(int st, cs_ctx* ctx) {
  t_status = st;
  t_error = (st == CS_OK || ctx == nullptr) ? std::string() : ctx->err;
  return st;
}

// Process-wide context of the calling thread's current device, for the drop-in calls.
cs_ctx* default_ctx(int* status) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    *status = CS_ERR_NODEVICE;
    t_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (!g_default[dev]) {
    cs_ctx* c = nullptr;
    int st = cs_ctx_create(dev, &c);
    if (st != CS_OK) {
      *status = st;
      t_error = "context creation failed";
      return nullptr;
    }
    g_default[dev] = c;
  }
  *status = CS_OK;
  return g_default[dev];
}

struct EventScope {
  cs_ctx* ctx;
  explicit EventScope(cs_ctx* c) : ctx(c) { cudaEventRecord(ctx->ev_start, ctx->stream); }
  void stop() { cudaEventRecord(ctx->ev_stop, ctx->stream); }
};

int msm_device_locked(cs_ctx* ctx, int ec2, const uint32_t* s, const uint32_t* p, uint32_t n,
                      uint32_t* out, int window) {
  csb::NvtxRange nvtx(ec2 ? "msm_g2" : "msm_g1");
  const size_t need = csb::msm_workspace_bytes(n, window, ec2 != 0, ctx->msm_affine);
  cudaError_t e = ctx->work.reserve(need, ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "msm workspace");
  csb::MsmConfig cfg;
  cfg.c = window;
  cfg.affine = ctx->msm_affine;
  cfg.acc_start = ctx->ev_phase0;
  cfg.acc_stop = ctx->ev_phase1;
  ctx->phase_valid = true;
  EventScope ev(ctx);
  e = ec2 ? csb::msm_g2(s, p, n, out, ctx->work.ptr, ctx->work.bytes, cfg, ctx->stream)
          : csb::msm_g1(s, p, n, out, ctx->work.ptr, ctx->work.bytes, cfg, ctx->stream);
  ev.stop();
  if (e != cudaSuccess) return fail(ctx, e, "msm launch");
  return CS_OK;
}

}  // namespace

namespace csb {
std::atomic<int> g_fail_allocs{0};
bool debug_take_alloc_failure() {
  int v = g_fail_allocs.load();
  while (v > 0) {
    if (g_fail_allocs.compare_exchange_weak(v, v - 1)) return true;
  }
  return false;
}
// Default context of the current device for the drop-in entry points (created on first use);
// *status and the thread's cs_last_error describe a failure.
cs_ctx* dropin_ctx(int* status) { return default_ctx(status); }
void dropin_status(int st, const char* msg) {
  t_status = st;
  if (msg) t_error = msg;
}
}  // namespace csb

extern "C" {

int cs_ctx_create(int device, cs_ctx** out) {
  if (!out) return CS_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return CS_ERR_NODEVICE;
  }
  if (device < 0 || device >= ndev) return CS_ERR_ARG;
  std::unique_ptr<cs_ctx> c(new cs_ctx());
  c->device = device;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev_start);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev_stop);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev_phase0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev_phase1);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return CS_ERR_CUDA;
  }
  c->own_stream = true;
  *out = c.release();
  return CS_OK;
}

void cs_ctx_destroy(cs_ctx* ctx) {
  if (!ctx) return;
  cudaStreamSynchronize(ctx->stream);
  csb::prove_graphs_release(ctx);
  csb::domain_release(ctx);
  ctx->work.release();
  ctx->in.release();
  ctx->out.release();
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
  if (ctx->ev_phase0) cudaEventDestroy(ctx->ev_phase0);
  if (ctx->ev_phase1) cudaEventDestroy(ctx->ev_phase1);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  for (int i = 0; i < 4; i++)
    if (ctx->aux[i]) { cudaStreamSynchronize(ctx->aux[i]); cudaStreamDestroy(ctx->aux[i]); }
  if (ctx->aux_h) { cudaStreamSynchronize(ctx->aux_h); cudaStreamDestroy(ctx->aux_h); }
  for (int i = 0; i < cs_ctx::kAuxEvents; i++)
    if (ctx->aux_ev[i]) cudaEventDestroy(ctx->aux_ev[i]);
  delete ctx;
}

int cs_ctx_set_prove_graphs(cs_ctx* ctx, int enable) {
  if (!ctx) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  ctx->use_prove_graphs = enable != 0;
  if (!enable) {
    cudaStreamSynchronize(ctx->stream);
    csb::prove_graphs_release(ctx);
  }
  return CS_OK;
}

int cs_ctx_set_stream(cs_ctx* ctx, void* stream) {
  if (!ctx) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (ctx->own_stream && ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  ctx->stream = static_cast<cudaStream_t>(stream);
  ctx->own_stream = false;
  return CS_OK;
}

void* cs_ctx_stream(cs_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int cs_ctx_sync(cs_ctx* ctx) {
  if (!ctx) return CS_ERR_ARG;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "stream sync");
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop) == cudaSuccess) ctx->last_ms = ms;
  if (ctx->phase_valid && cudaEventElapsedTime(&ms, ctx->ev_phase0, ctx->ev_phase1) == cudaSuccess)
    ctx->last_phase_ms = ms;
  ctx->phase_valid = false;
  cudaGetLastError();
  return CS_OK;
}

void cs_debug_fail_allocs(int count) { csb::g_fail_allocs.store(count > 0 ? count : 0); }

int cs_ctx_set_msm_affine_rounds(cs_ctx* ctx, int rounds) {
  if (!ctx || rounds < -1 || rounds > 6) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->msm_affine = rounds;
  return CS_OK;
}

int cs_ctx_prove_stages(cs_ctx* ctx, float* ms, int n) {
  if (!ctx || !ms || n < 1) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->aux_ready) return CS_ERR_ARG;
  if (!ctx->stages_valid)
    return csb::fail_msg(ctx, CS_ERR_UNSUPPORTED,
                         "stage times: the last proof was a graph replay (cs_ctx_set_prove_graphs(ctx, 0) times stages)");
  // completion of: A, B1, B2, C MSM chains, the H step, the H MSM, the whole proof
  cudaEvent_t evs[7] = {ctx->aux_ev[1], ctx->aux_ev[2], ctx->aux_ev[3], ctx->aux_ev[4], ctx->aux_ev[6],
                        ctx->aux_ev[5], ctx->ev_stop};
  for (int i = 0; i < n && i < 7; i++) {
    float t = -1.f;
    if (cudaEventElapsedTime(&t, ctx->ev_start, evs[i]) != cudaSuccess) {
      cudaGetLastError();
      t = -1.f;
    }
    ms[i] = t;
  }
  return CS_OK;
}

const char* cs_ctx_error(cs_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }
float cs_ctx_last_ms(cs_ctx* ctx) { return ctx ? ctx->last_ms : 0.f; }
float cs_ctx_last_phase_ms(cs_ctx* ctx) { return ctx ? ctx->last_phase_ms : 0.f; }

size_t cs_msm_workspace_bytes(uint32_t n, int ec2, int window) {
  return csb::msm_workspace_bytes(n, window, ec2 != 0);
}

int cs_msm_default_window(uint32_t n, int ec2) { return csb::msm_default_window(n, ec2 != 0); }
int cs_msm_num_windows(int window) { return window > 0 ? 254 / window + 1 : 0; }

int cs_msm_device(cs_ctx* ctx, int ec2, const uint32_t* d_scalars, const uint32_t* d_points,
                  uint32_t n, uint32_t* d_out, int window) {
  if (!ctx || (!d_out) || (n && (!d_scalars || !d_points))) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  return msm_device_locked(ctx, ec2, d_scalars, d_points, n, d_out, window);
}

int cs_msm(cs_ctx* ctx, int ec2, const uint32_t* scalars, const uint32_t* points, uint32_t n,
           uint32_t* out_affine, int window) {
  if (!ctx || !out_affine || (n && (!scalars || !points))) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  const size_t pw = ec2 ? 32 : 16;
  const size_t sbytes = (size_t)n * 8 * 4, pbytes = (size_t)n * pw * 4;
  const size_t sb_al = (sbytes + 255) & ~size_t(255);
  cudaError_t e = ctx->in.reserve(sb_al + pbytes + 256, ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "msm input buffer");
  e = ctx->out.reserve(256, ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "msm output buffer");
  uint32_t* ds = static_cast<uint32_t*>(ctx->in.ptr);
  uint32_t* dp = reinterpret_cast<uint32_t*>(static_cast<char*>(ctx->in.ptr) + sb_al);
  uint32_t* dout = static_cast<uint32_t*>(ctx->out.ptr);
  if (n) {
    if ((e = cudaMemcpyAsync(ds, scalars, sbytes, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return fail(ctx, e, "msm H2D scalars");
    if ((e = cudaMemcpyAsync(dp, points, pbytes, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return fail(ctx, e, "msm H2D points");
  }
  int st = msm_device_locked(ctx, ec2, ds, dp, n, dout, window);
  if (st != CS_OK) return st;
  if ((e = cudaMemcpyAsync(out_affine, dout, pw * 4, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
    return fail(ctx, e, "msm D2H");
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(ctx, e, "msm sync");
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop) == cudaSuccess) ctx->last_ms = ms;
  if (cudaEventElapsedTime(&ms, ctx->ev_phase0, ctx->ev_phase1) == cudaSuccess) ctx->last_phase_ms = ms;
  ctx->phase_valid = false;
  return CS_OK;
}

int cs_msm_fixed_window(uint32_t n, int ec2) { return csb::msm_fixed_window(n, ec2 != 0); }

size_t cs_msm_fixed_table_points(uint32_t n, int window) {
  return window >= 4 && window <= 24 ? csb::msm_fixed_table_points(n, window) : 0;
}

size_t cs_msm_fixed_workspace_bytes(uint32_t n, int ec2, int window) {
  return csb::msm_fixed_workspace_bytes(n, window, ec2 != 0);
}

int cs_msm_fixed_table_device(cs_ctx* ctx, int ec2, const uint32_t* d_points, uint32_t n, int window,
                              uint32_t* d_table) {
  if (!ctx || window < 4 || window > 24 || (n && (!d_points || !d_table))) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaError_t e = ctx->work.reserve(csb::msm_fixed_table_work_bytes(n, ec2 != 0), ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "fixed-base table scratch");
  EventScope ev(ctx);
  e = ec2 ? csb::msm_fixed_table_g2(d_points, n, window, d_table, ctx->work.ptr, ctx->work.bytes, ctx->stream)
          : csb::msm_fixed_table_g1(d_points, n, window, d_table, ctx->work.ptr, ctx->work.bytes, ctx->stream);
  ev.stop();
  if (e != cudaSuccess) return fail(ctx, e, "fixed-base table launch");
  return CS_OK;
}

int cs_msm_fixed_device(cs_ctx* ctx, int ec2, const uint32_t* d_scalars, const uint32_t* d_table, uint32_t n,
                        int window, uint32_t* d_out) {
  if (!ctx || !d_out || window < 4 || window > 24 || (n && (!d_scalars || !d_table))) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaError_t e = ctx->work.reserve(csb::msm_fixed_workspace_bytes(n, window, ec2 != 0, ctx->msm_affine), ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "fixed-base msm workspace");
  csb::MsmConfig cfg;
  cfg.c = window;
  cfg.affine = ctx->msm_affine;
  cfg.acc_start = ctx->ev_phase0;
  cfg.acc_stop = ctx->ev_phase1;
  ctx->phase_valid = true;
  EventScope ev(ctx);
  e = ec2 ? csb::msm_fixed_g2(d_scalars, d_table, n, d_out, ctx->work.ptr, ctx->work.bytes, cfg, ctx->stream)
          : csb::msm_fixed_g1(d_scalars, d_table, n, d_out, ctx->work.ptr, ctx->work.bytes, cfg, ctx->stream);
  ev.stop();
  if (e != cudaSuccess) return fail(ctx, e, "fixed-base msm launch");
  return CS_OK;
}

int cs_scmul_device(cs_ctx* ctx, int ec2, const uint32_t* d_scalars, const uint32_t* d_points,
                    uint32_t stride, uint32_t n, uint32_t* d_out) {
  if (!ctx || (n && (!d_scalars || !d_points || !d_out))) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  EventScope ev(ctx);
  cudaError_t e = ec2 ? csb::scmul_g2(d_scalars, d_points, stride, n, d_out, ctx->stream)
                      : csb::scmul_g1(d_scalars, d_points, stride, n, d_out, ctx->stream);
  ev.stop();
  if (e != cudaSuccess) return fail(ctx, e, "scmul launch");
  return CS_OK;
}

int cs_point_sum_device(cs_ctx* ctx, int ec2, const uint32_t* d_points, uint32_t n, int dims,
                        uint32_t* d_out) {
  if (!ctx || !d_out || (n && !d_points) || (dims != 2 && dims != 3)) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  EventScope ev(ctx);
  cudaError_t e = ec2 ? csb::point_sum_g2(d_points, n, dims, d_out, ctx->stream)
                      : csb::point_sum_g1(d_points, n, dims, d_out, ctx->stream);
  ev.stop();
  if (e != cudaSuccess) return fail(ctx, e, "point sum launch");
  return CS_OK;
}

// ------------------------------------------------------------ drop-in entry points ---
int cs_last_status(void) { return t_status; }
unsigned long long cs_kernel_launches(void) { return csb::g_launches.load(); }
const char* cs_last_error(void) { return t_error.c_str(); }

void ec_jacreduce_server_h(jacadd_reduced_t* args) {
  if (!args || !args->out_ep) {
    t_status = CS_ERR_ARG;
    t_error = "ec_jacreduce_server_h: null arguments";
    return;
  }
  if (args->filename != nullptr) {
    t_status = CS_ERR_UNSUPPORTED;
    t_error = "ec_jacreduce_server_h: precomputed table files are not supported";
    return;
  }
  if (args->pidx != 0) {
    t_status = CS_ERR_ARG;
    t_error = "ec_jacreduce_server_h: curve coordinates live in MOD_GROUP (pidx 0)";
    return;
  }
  if (args->n && (!args->scl || !args->x)) {
    t_status = CS_ERR_ARG;
    t_error = "ec_jacreduce_server_h: null scalar or point array";
    return;
  }
  int st = CS_OK;
  cs_ctx* ctx = default_ctx(&st);
  if (!ctx) {
    t_status = st;
    return;
  }
  st = cs_msm(ctx, args->ec2 ? 1 : 0, args->scl, args->x, args->n, args->out_ep, 0);
  set_thread_status(st, ctx);
}

void ec2_jacreduce_server_h(jacadd_reduced_t* args) { ec_jacreduce_server_h(args); }

}  // extern "C"
