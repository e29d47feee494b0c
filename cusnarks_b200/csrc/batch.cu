// batch.cu -- C ABI of the batched MSM (kernels: msm_batch.cuh) and the window autotuner.
//
// A batch plan fixes the instances (device pointers and sizes), picks each instance's
// window, orders instances by window so every window group is a contiguous bucket range,
// and owns the scratch.  cs_msm_batch_run enqueues the whole batch on the context stream;
// with use_graph the sequence is captured into a CUDA graph on the first run and replayed
// afterwards (one graph launch per batch).
#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

#include "../../include/cusnarks_b200.h"
#include "msm.cuh"
#include "runtime.cuh"

namespace {

constexpr int kMaxDev = 64, kMaxLog = 32;
std::mutex g_tune_mu;
int g_tuned[kMaxDev][2][kMaxLog] = {};  // [device][ec2][ceil(log2 n)] -> window, 0 = not tuned

uint32_t ceil_log2(uint32_t n) {
  uint32_t l = 0;
  while (l < 31 && (1u << l) < n) l++;
  return l;
}

int pick_window(int dev, int ec2, uint32_t n) {
  if (dev >= 0 && dev < kMaxDev) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const int w = g_tuned[dev][ec2 ? 1 : 0][ceil_log2(n < 1 ? 1 : n)];
    if (w) return w;
  }
  return csb::msm_window_model(n ? n : 1, false);  // batch instances sort full scalars
}

// Pseudo-random limbs for timing runs (splitmix-style hash); top limb masked below 2^253 so
// scalars are below r.  Coordinates need not be on the curve: the addition formulas run the
// same instructions either way.
__global__ void k_fill_random(uint32_t* p, size_t elems, uint32_t seed) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= elems) return;
  uint64_t x = (uint64_t)i * 0x9e3779b97f4a7c15ull + seed;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    x += 0x9e3779b97f4a7c15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    p[i * 8 + k] = (uint32_t)(k == 7 ? (z & 0x0fffffffu) : z);
  }
}

}  // namespace

struct cs_msm_batch {
  int device = 0;
  int ec2 = 0;
  std::vector<csb::BatchJob> jobs;   // ordered by window
  std::vector<uint32_t> order;       // order[k] = caller index of jobs[k]
  std::vector<csb::BatchGroup> groups;
  csb::MsmBatch plan;
  csb::BatchJob* d_jobs = nullptr;
  void* d_work = nullptr;
  size_t work_bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long launches_per_run = 0;
  ~cs_msm_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (d_work) cudaFree(d_work);
    if (d_jobs) cudaFree(d_jobs);
  }
};

namespace csb {

// Builds a batch plan from instance descriptions (the caller holds ctx->mu): windows (given, or
// tuned / by the cost model for generic instances; a fixed-base instance must give the window
// its table was built with), instances ordered by window, the device job table and the scratch.
int batch_build(cs_ctx* ctx, int ec2, const BatchSpec* jobs, uint32_t njobs, int task, cs_msm_batch** out) {
  *out = nullptr;
  std::unique_ptr<cs_msm_batch> b(new cs_msm_batch());
  b->device = ctx->device;
  b->ec2 = ec2 ? 1 : 0;
  std::vector<int> win(njobs);
  for (uint32_t i = 0; i < njobs; i++) {
    if (!jobs[i].out || (jobs[i].n && (!jobs[i].scalars || !jobs[i].points)))
      return fail_msg(ctx, CS_ERR_ARG, "cs_msm_batch_create: job " + std::to_string(i) + " has a null pointer");
    if (jobs[i].fixed && !jobs[i].window)
      return fail_msg(ctx, CS_ERR_ARG, "batch: a fixed-base instance needs its table's window");
    if (jobs[i].window && (jobs[i].window < 4 || jobs[i].window > (jobs[i].fixed ? 24 : 22)))
      return fail_msg(ctx, CS_ERR_ARG, "cs_msm_batch_create: window must be 0 or 4..22");
    win[i] = jobs[i].window ? jobs[i].window : pick_window(ctx->device, ec2, jobs[i].n);
  }
  b->order.resize(njobs);
  std::iota(b->order.begin(), b->order.end(), 0u);
  std::stable_sort(b->order.begin(), b->order.end(), [&](uint32_t x, uint32_t y) { return win[x] < win[y]; });
  uint64_t terms = 0, buckets = 0, entries = 0, windows = 0;
  uint64_t lv = 0, lv2 = 0;
  for (uint32_t k = 0; k < njobs; k++) {
    const BatchSpec& j = jobs[b->order[k]];
    const int c = win[b->order[k]];
    const uint32_t W = 254 / c + 1;
    const uint32_t sets = j.fixed ? 1u : W;
    BatchJob bj{};
    bj.scalars = j.scalars;
    bj.points = j.points;
    bj.out = j.out;
    bj.n = j.n;
    bj.c = (uint32_t)c;
    bj.W = W;
    bj.fixed = j.fixed ? 1u : 0u;
    bj.sets = sets;
    bj.term0 = (uint32_t)terms;
    bj.bucket0 = (uint32_t)buckets;
    bj.window0 = (uint32_t)windows;
    if (b->groups.empty() || b->groups.back().c != c)
      b->groups.push_back(BatchGroup{c, (uint32_t)buckets, 0u, (uint32_t)windows});
    b->groups.back().windows += sets;
    terms += j.n;
    buckets += (uint64_t)sets << (c - 1);
    entries += (uint64_t)j.n * W;
    windows += sets;
    b->jobs.push_back(bj);
  }
  for (const auto& g : b->groups) {
    const uint64_t n1 = ((uint64_t)1 << (g.c - 1)) / 8 + 1;
    lv = std::max(lv, (uint64_t)g.windows * n1);
    lv2 = std::max(lv2, (uint64_t)g.windows * (n1 / 8 + 1));
  }
  if (terms >= 0xffffffffull || buckets >= 0xffffffffull || entries >= 0x7fffffffull)
    return fail_msg(ctx, CS_ERR_ARG, "cs_msm_batch_create: batch too large (terms x windows must stay below 2^31)");
  MsmBatch& P = b->plan;
  P.njobs = njobs;
  P.terms = (uint32_t)terms;
  P.nbuckets = (uint32_t)buckets;
  P.nentries = entries;
  P.nwindows = (uint32_t)windows;
  P.lv_points = lv;
  P.lv2_points = lv2;
  P.groups = b->groups.data();
  P.ngroups = (uint32_t)b->groups.size();
  if (task <= 0) {
    // about one task per resident accumulation thread (3 blocks of 128 per SM): a batch of
    // small instances splits its buckets so the accumulation keeps every thread busy.
    // Measured per batch of proofs (ms; tile 64 / one task per thread / three): 16 x 2^12
    // 4.03 / 3.53 / 4.29, 4 x 2^14 - / 3.53 / 3.80, 4 x 2^16 - / 9.04 / 9.26.
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const uint64_t per = entries / ((uint64_t)sms * 384);
    task = (int)std::min<uint64_t>(64, std::max<uint64_t>(kBatchMinTask, per));
  }
  P.task = std::min(64, std::max(kBatchMinTask, task));
  cudaError_t e = cudaSuccess;
  if (njobs) {
    e = cudaMalloc(&b->d_jobs, sizeof(BatchJob) * njobs);
    if (e == cudaSuccess)
      e = cudaMemcpy(b->d_jobs, b->jobs.data(), sizeof(BatchJob) * njobs, cudaMemcpyHostToDevice);
    P.d_jobs = b->d_jobs;
    b->work_bytes = msm_batch_workspace_bytes(P, ec2 != 0);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_work, b->work_bytes);
  }
  if (e != cudaSuccess) return fail(ctx, e, "cs_msm_batch_create: device buffers");
  *out = b.release();
  return CS_OK;
}

// Enqueues a batch plan's launches on a stream (no graph of its own).
cudaError_t batch_enqueue(cs_msm_batch* b, cudaStream_t st) {
  if (b->plan.njobs == 0) return cudaSuccess;
  return b->ec2 ? msm_batch_g2(b->plan, b->d_work, b->work_bytes, st)
                : msm_batch_g1(b->plan, b->d_work, b->work_bytes, st);
}

}  // namespace csb

extern "C" {

int cs_msm_batch_create(cs_ctx* ctx, int ec2, const cs_msm_job* jobs, uint32_t njobs, int task,
                        cs_msm_batch** out) {
  if (!ctx || !out || (njobs && !jobs)) return CS_ERR_ARG;
  std::vector<csb::BatchSpec> specs(njobs);
  for (uint32_t i = 0; i < njobs; i++)
    specs[i] = csb::BatchSpec{jobs[i].scalars, jobs[i].points, jobs[i].out, jobs[i].n, jobs[i].window, false};
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  return csb::batch_build(ctx, ec2, specs.data(), njobs, task, out);
}

void cs_msm_batch_destroy(cs_msm_batch* b) { delete b; }

size_t cs_msm_batch_workspace_bytes(const cs_msm_batch* b) { return b ? b->work_bytes : 0; }

int cs_msm_batch_window(const cs_msm_batch* b, uint32_t i) {
  if (!b || i >= b->order.size()) return 0;
  for (size_t k = 0; k < b->order.size(); k++)
    if (b->order[k] == i) return (int)b->jobs[k].c;
  return 0;
}

int cs_msm_batch_run(cs_ctx* ctx, cs_msm_batch* b, int use_graph) {
  if (!ctx || !b) return CS_ERR_ARG;
  csb::NvtxRange nvtx(use_graph ? "msm_batch_graph" : "msm_batch");
  if (b->device != ctx->device) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  if (b->plan.njobs == 0) return CS_OK;
  auto enqueue = [&](cudaStream_t st) {
    return b->ec2 ? csb::msm_batch_g2(b->plan, b->d_work, b->work_bytes, st)
                  : csb::msm_batch_g1(b->plan, b->d_work, b->work_bytes, st);
  };
  cudaError_t e;
  cudaEventRecord(ctx->ev_start, ctx->stream);
  if (!use_graph) {
    e = enqueue(ctx->stream);
  } else {
    if (!b->exec) {
      const unsigned long long before = cs_kernel_launches();
      e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return csb::fail(ctx, e, "batch graph capture begin");
      cudaError_t ee = enqueue(ctx->stream);
      cudaGraph_t g = nullptr;
      e = cudaStreamEndCapture(ctx->stream, &g);
      if (ee != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return csb::fail(ctx, ee, "batch graph capture");
      }
      if (e != cudaSuccess) return csb::fail(ctx, e, "batch graph capture end");
      b->graph = g;
      e = cudaGraphInstantiate(&b->exec, g, 0);
      if (e != cudaSuccess) return csb::fail(ctx, e, "batch graph instantiate");
      // kernels recorded into the graph run on every replay: count them per replay
      b->launches_per_run = cs_kernel_launches() - before;
    }
    e = cudaGraphLaunch(b->exec, ctx->stream);
    if (e == cudaSuccess) csb::note_launch((unsigned)b->launches_per_run);
  }
  cudaEventRecord(ctx->ev_stop, ctx->stream);
  if (e != cudaSuccess) return csb::fail(ctx, e, "batch launch");
  return CS_OK;
}

int cs_msm_autotune(cs_ctx* ctx, int ec2, uint32_t log_min, uint32_t log_max, int* windows_out) {
  if (!ctx || log_min < 1 || log_max > 24 || log_min > log_max) return CS_ERR_ARG;
  std::vector<int> best_w;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    const uint32_t nmax = 1u << log_max;
    const size_t pw = ec2 ? 32 : 16;
    uint32_t *d_s = nullptr, *d_p = nullptr, *d_o = nullptr;
    cudaError_t e = cudaMalloc(&d_s, (size_t)nmax * 32);
    if (e == cudaSuccess) e = cudaMalloc(&d_p, (size_t)nmax * pw * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_o, 256);
    if (e == cudaSuccess) {
      k_fill_random<<<(nmax + 255) / 256, 256, 0, ctx->stream>>>(d_s, nmax, 17u);
      k_fill_random<<<(unsigned)((nmax * pw / 8 + 255) / 256), 256, 0, ctx->stream>>>(d_p, (size_t)nmax * pw / 8, 91u);
      csb::note_launch(2);
      e = cudaGetLastError();
    }
    cudaEvent_t a = nullptr, z = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&z);
    for (uint32_t L = log_min; L <= log_max && e == cudaSuccess; L++) {
      const uint32_t n = 1u << L;
      // the form a batch instance runs: full scalars (single G1 MSMs split them by GLV and
      // keep the cost model's window)
      const int c0 = csb::msm_window_model(n, false);
      float best = 1e30f;
      int bw = c0;
      for (int c = std::max(4, c0 - 2); c <= std::min(22, c0 + 2) && e == cudaSuccess; c++) {
        e = ctx->work.reserve(csb::msm_workspace_bytes(n, c, ec2 != 0, -1, 0), ctx->stream);
        if (e != cudaSuccess) break;
        csb::MsmConfig cfg;
        cfg.c = c;
        cfg.glv = 0;
        float t_best = 1e30f;
        for (int rep = 0; rep < 3 && e == cudaSuccess; rep++) {
          cudaEventRecord(a, ctx->stream);
          e = ec2 ? csb::msm_g2(d_s, d_p, n, d_o, ctx->work.ptr, ctx->work.bytes, cfg, ctx->stream)
                  : csb::msm_g1(d_s, d_p, n, d_o, ctx->work.ptr, ctx->work.bytes, cfg, ctx->stream);
          cudaEventRecord(z, ctx->stream);
          if (e == cudaSuccess) e = cudaEventSynchronize(z);
          float ms = 0.f;
          cudaEventElapsedTime(&ms, a, z);
          if (rep > 0 && ms < t_best) t_best = ms;  // first run warms up
        }
        if (t_best < best) {
          best = t_best;
          bw = c;
        }
      }
      best_w.push_back(bw);
    }
    if (a) cudaEventDestroy(a);
    if (z) cudaEventDestroy(z);
    cudaFree(d_s);
    cudaFree(d_p);
    cudaFree(d_o);
    if (e != cudaSuccess) return csb::fail(ctx, e, "autotune");
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (uint32_t L = log_min; L <= log_max; L++) {
    const int w = best_w[L - log_min];
    if (ctx->device < kMaxDev) g_tuned[ctx->device][ec2 ? 1 : 0][L] = w;
    if (windows_out) windows_out[L - log_min] = w;
  }
  return CS_OK;
}

int cs_msm_tuned_window(cs_ctx* ctx, int ec2, uint32_t n) {
  return ctx ? pick_window(ctx->device, ec2, n) : 0;
}

}  // extern "C"
