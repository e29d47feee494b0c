// msm_batch.cuh -- many MSM instances of uneven size in one pass (instantiated for G1 in
// msm_batch_g1.cu and for G2 in msm_batch_g2.cu).
//
// The reference runs one GPU multi-exp call per instance (src/python/cuda_wrapper.py:216
// ec_mad_cuda2, batches dispatched one by one by groth_prover.py:1563).  Here all instances of
// one group share one digit sort and ONE accumulation launch:
//   * k_bcount / k_bscatter: one thread per term of any instance (binary search of the
//     instance's first term), digits with the instance's own window, buckets in one bucket
//     space (instance after instance, ordered by window);
//   * the task pipeline of the single MSM over all buckets, each task tagged with its
//     instance, and one persistent k_accumulate over the union of tasks, longest first --
//     the work is split by bucket size, not by instance, so a 2^10 instance next to a 2^20
//     one costs its share and no launch;
//   * reduction per window group (instances with equal c are contiguous: one level chain and
//     one k_window_sum launch per distinct c), and k_bfinish: one warp per instance for the
//     window Horner and the affine result.
// Fixed-base instances (resident tables T[j n + i] = 2^(c j) P_i, the proof's MSMs) put every
// digit into one bucket set and need no window Horner.
// The sequence contains no allocation and no host synchronisation, so it can be captured in a
// CUDA graph once and replayed (cs_msm_batch_run).
#pragma once
#include "msm_impl.cuh"

namespace csb {
namespace msm_detail {

// Index of the job whose term range holds global term t (term0 ascending; empty jobs share
// their successor's term0 and are skipped by taking the last job with term0 <= t).
CSB_DEV uint32_t job_of_term(const BatchJob* jobs, uint32_t njobs, uint32_t t) {
  uint32_t lo = 0, hi = njobs;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (jobs[mid].term0 <= t) lo = mid; else hi = mid;
  }
  return lo;
}

template <class F>
__global__ void k_bcount(const BatchJob* __restrict__ jobs, uint32_t njobs, uint32_t terms,
                         uint32_t* __restrict__ counts) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= terms) return;
  const BatchJob jb = jobs[job_of_term(jobs, njobs, t)];
  const uint32_t i = t - jb.term0;
  uint32_t k[8];
  if (!load_scalar<F>(jb.scalars, jb.points, i, k)) return;
  const uint32_t B = 1u << (jb.c - 1);
  for_each_digit(k, (int)jb.c, (int)jb.W, [&](int j, uint32_t mag, bool) {
    atomicAdd(&counts[jb.bucket0 + (jb.fixed ? 0 : (size_t)j * B) + (mag - 1)], 1u);
  });
}

template <class F>
__global__ void k_bscatter(const BatchJob* __restrict__ jobs, uint32_t njobs, uint32_t terms,
                           uint32_t* __restrict__ cursor, uint32_t* __restrict__ entries) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= terms) return;
  const BatchJob jb = jobs[job_of_term(jobs, njobs, t)];
  const uint32_t i = t - jb.term0;
  uint32_t k[8];
  if (!load_scalar<F>(jb.scalars, jb.points, i, k)) return;
  const uint32_t B = 1u << (jb.c - 1);
  for_each_digit(k, (int)jb.c, (int)jb.W, [&](int j, uint32_t mag, bool neg) {
    const uint32_t pos = atomicAdd(&cursor[jb.bucket0 + (jb.fixed ? 0 : (size_t)j * B) + (mag - 1)], 1u);
    entries[pos] = (jb.fixed ? (uint32_t)j * jb.n + i : i) | (neg ? NEG_BIT : 0u);
  });
}

// One warp per instance (quad point operations; the warp's 8 quads compute the same):
// sum_j 2^(c j) S_j over its bucket sets (a fixed-base instance has one), affine result.
template <class F>
__global__ void k_bfinish(const BatchJob* __restrict__ jobs, uint32_t njobs, const uint32_t* __restrict__ wsum) {
  constexpr int XW = 4 * FieldWords<F>::value;
  const uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (q >= njobs) return;  // whole warps leave together
  const BatchJob jb = jobs[q];
  const uint32_t* w = wsum + (size_t)jb.window0 * XW;
  XYZZ<F> r = ld_xyzz<F>(w + (size_t)(jb.sets - 1) * XW);
#pragma unroll 1
  for (int j = (int)jb.sets - 2; j >= 0; j--) {
#pragma unroll 1
    for (uint32_t d = 0; d < jb.c; d++) r = xyzz_dbl_quad(r);
    r = xyzz_add_quad(r, ld_xyzz<F>(w + (size_t)j * XW));
  }
  if ((threadIdx.x & 31) == 0) st_affine<F>(jb.out, xyzz_to_affine(r));
}

struct BatchLayout {
  size_t counters, counts, offsets, entries, tasks, multi, partials, buckets, lv_y, lv_z, lv_y2, lv_z2, wsum,
      scan, total;
};

inline BatchLayout batch_layout(const MsmBatch& b, int xyzz_bytes) {
  const size_t nb = b.nbuckets, ne = b.nentries;
  const size_t tl = (size_t)std::max(kBatchMinTask, std::min(b.task, kMaxTask));
  const size_t lv = b.lv_points, lv2 = b.lv2_points;
  BatchLayout L{};
  size_t o = 0;
  L.counters = o; o = align256(o + kCtrWords * sizeof(uint32_t));
  L.counts = o;   o = align256(o + (nb + 1) * sizeof(uint32_t));
  L.offsets = o;  o = align256(o + (nb + 1) * sizeof(uint32_t));
  L.entries = o;  o = align256(o + ne * sizeof(uint32_t));
  L.tasks = o;    o = align256(o + (nb + ne / tl + 1) * sizeof(Task));
  L.multi = o;    o = align256(o + (ne / (tl + 1) + 1) * sizeof(Multi));
  L.partials = o; o = align256(o + (2 * (ne / tl) + 1) * (size_t)xyzz_bytes);
  L.buckets = o;  o = align256(o + nb * (size_t)xyzz_bytes);
  L.lv_y = o;     o = align256(o + lv * xyzz_bytes);
  L.lv_z = o;     o = align256(o + lv * xyzz_bytes);
  L.lv_y2 = o;    o = align256(o + lv2 * xyzz_bytes);
  L.lv_z2 = o;    o = align256(o + lv2 * xyzz_bytes);
  L.wsum = o;     o = align256(o + (size_t)b.nwindows * xyzz_bytes);
  L.scan = o;
  L.total = o + scan_workspace_bytes(nb + 1);
  return L;
}

template <class F>
cudaError_t batch_impl(const MsmBatch& b, void* d_work, size_t work_bytes, cudaStream_t st) {
  constexpr int XB = 4 * FieldWords<F>::value * 4;
  constexpr int XWD = XB / 4;
  if (b.njobs == 0) return cudaSuccess;
  const BatchLayout L = batch_layout(b, XB);
  if (!d_work || work_bytes < L.total || b.nentries >= (uint64_t)0xffffffffu) return cudaErrorInvalidValue;
  char* base = static_cast<char*>(d_work);
  auto at = [&](size_t off) { return reinterpret_cast<uint32_t*>(base + off); };
  uint32_t *counters = at(L.counters), *counts = at(L.counts), *offsets = at(L.offsets);
  uint32_t *entries = at(L.entries), *partials = at(L.partials), *buckets = at(L.buckets);
  uint32_t *lv_y = at(L.lv_y), *lv_z = at(L.lv_z), *lv_y2 = at(L.lv_y2), *lv_z2 = at(L.lv_z2), *wsum = at(L.wsum);
  Task* tasks = reinterpret_cast<Task*>(base + L.tasks);
  Multi* multi = reinterpret_cast<Multi*>(base + L.multi);
  const uint32_t nb = b.nbuckets;
  const uint32_t task_len = (uint32_t)std::max(kBatchMinTask, std::min(b.task, kMaxTask));  // as the layout
  cudaError_t e;
  if ((e = cudaMemsetAsync(counters, 0, kCtrWords * sizeof(uint32_t), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(counts, 0, ((size_t)nb + 1) * sizeof(uint32_t), st)) != cudaSuccess) return e;
  const int T = 256;
  if (b.terms) {
    k_bcount<F><<<(b.terms + T - 1) / T, T, 0, st>>>(b.d_jobs, b.njobs, b.terms, counts);
    note_launch();
  }
  if ((e = scan_exclusive_u32(counts, offsets, (size_t)nb + 1, base + L.scan, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(counts, offsets, (size_t)nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st)) !=
      cudaSuccess)
    return e;
  if (b.terms) {
    k_bscatter<F><<<(b.terms + T - 1) / T, T, 0, st>>>(b.d_jobs, b.njobs, b.terms, counts, entries);
    note_launch();
  }
  k_task_hist<F><<<(nb + T - 1) / T, T, 0, st>>>(offsets, nb, task_len, counters + kCtrHist, buckets);
  k_task_bins<<<1, 32, 0, st>>>(counters + kCtrHist, task_len, counters + kCtrCursor, counters);
  k_task_emit<F><<<(nb + T - 1) / T, T, 0, st>>>(offsets, nb, task_len, counters + kCtrCursor, tasks, counters,
                                                  multi, b.d_jobs, b.njobs);
  note_launch(3);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // Latency form (one quad per task) when the tasks fill the quads at most four times over:
  // four proofs of 2^12 constraints 2.96 -> 2.62 ms a batch; at eight or sixteen times over the
  // thread form wins (sixteen proofs of 2^12: 4.03 vs 4.76 ms).
  const uint64_t resident_threads = (uint64_t)accumulate_grid<F>(dev, sms) * 128;
  const bool latency_mode = ((uint64_t)nb + b.nentries / task_len + 1) * 4 <= resident_threads * 4;
  if (latency_mode)
    k_accumulate_quad<F><<<accumulate_grid<F>(dev, sms), 128, 0, st>>>(tasks, counters, entries, nullptr, nb, buckets,
                                                                  partials, b.d_jobs);
  else
    k_accumulate<F><<<accumulate_grid<F>(dev, sms), 128, 0, st>>>(tasks, counters, entries, nullptr, nb, buckets,
                                                             partials, b.d_jobs);
  k_combine_small<F><<<sms * 4, 128, 0, st>>>(multi, counters, partials, buckets);
  k_combine<F><<<sms * 4, 128, 0, st>>>(multi, counters, partials, buckets);
  note_launch(3);
  const uint64_t resident = (uint64_t)accumulate_grid<F>(dev, sms) * 128;
  // reduction per window group
  for (uint32_t g = 0; g < b.ngroups; g++) {
    const BatchGroup& G = b.groups[g];
    const uint32_t B = 1u << (G.c - 1);
    const uint32_t WR = G.windows;
    uint32_t nseg = (B + 7) / 8;
    reduce_level<F>(buckets + (size_t)G.bucket0 * XWD, nullptr, B, nseg, (int)WR, 0, lv_y, lv_z, resident, st);
    int levels = 1;
    uint32_t *y = lv_y, *z = lv_z, *y2 = lv_y2, *z2 = lv_z2;
    while (nseg > kTopSegments) {
      const uint32_t nnext = (nseg + 7) / 8;
      reduce_level<F>(y, z, nseg, nnext, (int)WR, levels, y2, z2, resident, st);
      uint32_t* ty = y; y = y2; y2 = ty;
      uint32_t* tz = z; z = z2; z2 = tz;
      nseg = nnext;
      levels++;
    }
    constexpr int WT = WsumThreads<F>::batch;
    k_window_sum<F, WT><<<WR, WT, 0, st>>>(y, z, nseg, 3 * levels, wsum + (size_t)G.window0 * XWD);
    note_launch();
  }
  k_bfinish<F><<<(32 * b.njobs + 127) / 128, 128, 0, st>>>(b.d_jobs, b.njobs, wsum);
  note_launch();
  return cudaGetLastError();
}

}  // namespace msm_detail
}  // namespace csb
