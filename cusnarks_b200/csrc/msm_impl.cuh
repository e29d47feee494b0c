// msm_impl.cuh -- kernels and launch sequence of the Pippenger MSM (pipeline in msm.cuh),
// instantiated for G1 in msm_g1.cu and for G2 in msm_g2.cu.
#pragma once
#include <algorithm>
#include <atomic>
#include "msm.cuh"
#include "curve.cuh"
#include "glv.cuh"
#include "scan.cuh"
#include "runtime.cuh"

namespace csb {
namespace msm_detail {

constexpr int SCALAR_BITS = 254;  // scalars are reduced below r < 2^254 first
constexpr uint32_t NEG_BIT = 0x80000000u;
// Generic G1 MSMs with the GLV split: an entry of the k2 half reads phi(P_i) = (beta x_i, y_i)
// (terms below 2^30).
constexpr uint32_t PHI_BIT = 0x40000000u;
constexpr uint32_t kMinTask = 32;  // workspace bounds assume tasks of at least this size
// ... except for smaller MSMs: their bounds assume tasks of layout_min_task(entries), down to 8
// entries, so the bound stays near 65,536 tasks.  The latency form splits buckets of MSMs of
// at most kSmallEntries entries in tasks of 16 (2^12 fixed-base G1 MSM 0.469 -> 0.445 ms, 2^12
// proof 1.586 -> 1.533 ms against 32; 8 is slower: more partial sums).
constexpr size_t kSmallEntries = 1u << 19;
constexpr uint32_t kLatMinTask = 16;
inline uint32_t layout_min_task(uint64_t entries) {
  return (uint32_t)std::min<uint64_t>(kMinTask, std::max<uint64_t>(8, entries / 65536));
}

__host__ __device__ inline int num_windows(int c) { return SCALAR_BITS / c + 1; }
// Windows of a GLV half-scalar (|k1|, |k2| < 2^127): c W >= 128 leaves the top digit at most
// 2^(c-1) after the signed recoding's carry, so no further window is needed.
__host__ __device__ inline int glv_windows(int c) { return (128 + c - 1) / c; }
// Window count of an MSM: generic G1 MSMs split their scalars by the endomorphism (glv).
__host__ __device__ inline int msm_windows(int c, bool glv) { return glv ? glv_windows(c) : num_windows(c); }

// k <- k mod r for any 256-bit k (at most 5 subtractions since 2^256 / r < 6)
CSB_DEV void scalar_reduce(uint32_t (&k)[8]) {
#pragma unroll 1
  for (int it = 0; it < 6; it++) {
    uint32_t u[8], br;
    SUB_CC(u[0], k[0], ModR::P0); SUBC_CC(u[1], k[1], ModR::P1); SUBC_CC(u[2], k[2], ModR::P2);
    SUBC_CC(u[3], k[3], ModR::P3); SUBC_CC(u[4], k[4], ModR::P4); SUBC_CC(u[5], k[5], ModR::P5);
    SUBC_CC(u[6], k[6], ModR::P6); SUBC_CC(u[7], k[7], ModR::P7); SUBC(br, 0u, 0u);
    if (br) break;
#pragma unroll
    for (int i = 0; i < 8; i++) k[i] = u[i];
  }
}

CSB_DEV uint32_t scalar_bits(const uint32_t (&k)[8], int off, int c) {
  const int w = off >> 5, sh = off & 31;
  if (w >= 8) return 0;
  uint32_t v = k[w] >> sh;
  if (sh + c > 32 && w + 1 < 8) v |= k[w + 1] << (32 - sh);
  return v & ((1u << c) - 1u);
}

// Signed recoding: digit j in (-2^(c-1), 2^(c-1)].  Calls f(j, |d|, negative) for
// every nonzero digit.
template <class Fn>
CSB_DEV void for_each_digit(const uint32_t (&k)[8], int c, int W, Fn f) {
  const uint32_t half = 1u << (c - 1);
  const uint32_t full = 1u << c;
  uint32_t carry = 0;
  for (int j = 0; j < W; j++) {
    const uint32_t raw = scalar_bits(k, j * c, c) + carry;
    if (raw > half) {
      carry = 1;
      const uint32_t mag = full - raw;
      if (mag) f(j, mag, true);
    } else {
      carry = 0;
      if (raw) f(j, raw, false);
    }
  }
}

template <class F>
CSB_DEV bool point_is_inf(const uint32_t* p) {
  constexpr int W = FieldWords<F>::value;
  // reference encoding: X == 0 and Y == 1_mont (Y.c1 == 0 for G2)
  for (int i = 0; i < W; i++)
    if (p[i]) return false;
  const Fq one = Fq::one();
  for (int i = 0; i < 8; i++)
    if (p[W + i] != one.v[i]) return false;
  for (int i = 8; i < W; i++)
    if (p[W + i]) return false;
  return true;
}

template <class F>
CSB_DEV bool load_scalar(const uint32_t* scalars, const uint32_t* points, uint32_t i,
                         uint32_t (&k)[8]) {
  ld_limbs8(k, scalars + (size_t)i * 8);
  scalar_reduce(k);
  if ((k[0] | k[1] | k[2] | k[3] | k[4] | k[5] | k[6] | k[7]) == 0) return false;
  constexpr int PW = 2 * FieldWords<F>::value;
  return !point_is_inf<F>(points + (size_t)i * PW);
}

// Entry placement.  Generic: bucket (window j, |d|-1) of W*B, entry = point index i.
// Fixed-base (tables T[j*n + i] = 2^(c j) P_i): one set of B buckets, bucket |d|-1,
// entry = table index j*n + i, so no per-window sums and no Horner step remain.
template <class F, bool FIXED>
__global__ void k_count(const uint32_t* __restrict__ scalars, const uint32_t* __restrict__ points,
                        uint32_t n, int c, int W, uint32_t* __restrict__ counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k[8];
  if (!load_scalar<F>(scalars, points, i, k)) return;
  const uint32_t B = 1u << (c - 1);
  for_each_digit(k, c, W, [&](int j, uint32_t mag, bool) {
    atomicAdd(&counts[(FIXED ? 0 : (size_t)j * B) + (mag - 1)], 1u);
  });
}

template <class F, bool FIXED>
__global__ void k_scatter(const uint32_t* __restrict__ scalars, const uint32_t* __restrict__ points,
                          uint32_t n, int c, int W, uint32_t* __restrict__ cursor,
                          uint32_t* __restrict__ entries) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k[8];
  if (!load_scalar<F>(scalars, points, i, k)) return;
  const uint32_t B = 1u << (c - 1);
  for_each_digit(k, c, W, [&](int j, uint32_t mag, bool neg) {
    const uint32_t pos = atomicAdd(&cursor[(FIXED ? 0 : (size_t)j * B) + (mag - 1)], 1u);
    entries[pos] = (FIXED ? (uint32_t)j * n + i : i) | (neg ? NEG_BIT : 0u);
  });
}

// GLV split of a generic G1 MSM: k_i P_i = k1 P_i + k2 phi(P_i) with k_i = k1 + k2 lambda
// (mod r), |k1|, |k2| < 2^127, so the pipeline sorts 2n half-size scalars: half the windows,
// half the bucket sets to reduce and half the window Horner.  k_glv_prep writes, per term,
// s2[i] = |k1| (words 0-3) and |k2| (words 4-7) with each half's sign in bit 31 of its top
// word (zero halves for a zero scalar or a point at infinity), and phix[i] = beta x_i.  The
// points themselves are not copied: an entry of the k2 half carries PHI_BIT and reads x from
// phix and y from P_i, so the gathered set stays the n input points plus n x-coordinates.
template <class F>
__global__ void k_glv_prep(const uint32_t* __restrict__ scalars, const uint32_t* __restrict__ points, uint32_t n,
                           uint32_t* __restrict__ s2, uint32_t* __restrict__ phix) {
  constexpr int PW = 2 * FieldWords<F>::value;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k[8];
  ld_limbs8(k, scalars + (size_t)i * 8);
  scalar_reduce(k);
  const uint32_t* P = points + (size_t)i * PW;
  uint32_t k1[4] = {0, 0, 0, 0}, k2[4] = {0, 0, 0, 0}, neg1 = 0, neg2 = 0;
  const bool zero = (k[0] | k[1] | k[2] | k[3] | k[4] | k[5] | k[6] | k[7]) == 0;
  if (!zero && !point_is_inf<F>(P)) {
    const uint64_t kk[4] = {k[0] | (uint64_t)k[1] << 32, k[2] | (uint64_t)k[3] << 32, k[4] | (uint64_t)k[5] << 32,
                            k[6] | (uint64_t)k[7] << 32};
    glv::split_reduced(kk, k1, &neg1, k2, &neg2);
  }
  uint4* o = reinterpret_cast<uint4*>(s2 + (size_t)i * 8);
  o[0] = make_uint4(k1[0], k1[1], k1[2], k1[3] | (neg1 << 31));
  o[1] = make_uint4(k2[0], k2[1], k2[2], k2[3] | (neg2 << 31));
  F x, beta;
  ld_field(x, P);
  glv::beta_mont(beta.v);
  st_field(phix + (size_t)i * 8, x * beta);
}

// Digits of both halves of a split term: f(half, window, |d|, negative), the half's sign
// folded into the digit's.
template <class Fn>
CSB_DEV void for_each_glv_digit(const uint32_t (&t)[8], int c, int W, Fn f) {
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const uint32_t k[8] = {t[4 * h], t[4 * h + 1], t[4 * h + 2], t[4 * h + 3] & 0x7fffffffu, 0u, 0u, 0u, 0u};
    const bool sgn = (t[4 * h + 3] >> 31) != 0;
    for_each_digit(k, c, W, [&](int j, uint32_t mag, bool neg) { f(h, j, mag, neg != sgn); });
  }
}

template <class F>
__global__ void k_count_glv(const uint32_t* __restrict__ s2, uint32_t n, int c, int W, uint32_t* __restrict__ counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t t[8];
  ld_limbs8(t, s2 + (size_t)i * 8);
  const uint32_t B = 1u << (c - 1);
  for_each_glv_digit(t, c, W, [&](int, int j, uint32_t mag, bool) { atomicAdd(&counts[(size_t)j * B + (mag - 1)], 1u); });
}

template <class F>
__global__ void k_scatter_glv(const uint32_t* __restrict__ s2, uint32_t n, int c, int W, uint32_t* __restrict__ cursor,
                              uint32_t* __restrict__ entries) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t t[8];
  ld_limbs8(t, s2 + (size_t)i * 8);
  const uint32_t B = 1u << (c - 1);
  for_each_glv_digit(t, c, W, [&](int h, int j, uint32_t mag, bool neg) {
    const uint32_t pos = atomicAdd(&cursor[(size_t)j * B + (mag - 1)], 1u);
    entries[pos] = i | (h ? PHI_BIT : 0u) | (neg ? NEG_BIT : 0u);
  });
}

// The base of an entry: P_i, or phi(P_i) = (phix[i], y_i) for a GLV k2 entry (phix given).
// One load path either way (the x address is selected), so lanes of a warp that read P and
// phi(P) do not diverge.
template <class F>
CSB_DEV Affine<F> ld_entry_point(const uint32_t* base, const uint32_t* phix, uint32_t ent) {
  constexpr int FW = FieldWords<F>::value;
  constexpr int PW = 2 * FW;
  if constexpr (FW == 8) {
    const bool phi = phix != nullptr && (ent & PHI_BIT) != 0;
    const uint32_t i = ent & ~(NEG_BIT | (phix ? PHI_BIT : 0u));
    const uint32_t* xp = phi ? phix + (size_t)i * 8 : base + (size_t)i * PW;
    Affine<F> p;
    ld_field(p.x, xp);
    ld_field(p.y, base + (size_t)i * PW + FW);
    return p;
  } else {
    return ld_affine<F>(base + (size_t)(ent & ~NEG_BIT) * PW);
  }
}

// Task record: entries [start, start+len) summed into dst.  dst < nb: bucket index;
// dst >= nb: partial slot (dst - nb).  job: the instance whose bases the entries index (a
// batch of MSMs shares one task list; 0 for a single MSM).
struct Task {
  uint32_t start, len, dst, job;
};

// Index of the job whose bucket range holds bucket b (bucket0 ascending, bucket0[0] = 0).
CSB_DEV uint32_t job_of_bucket(const BatchJob* jobs, uint32_t njobs, uint32_t b) {
  uint32_t lo = 0, hi = njobs;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (jobs[mid].bucket0 <= b) lo = mid; else hi = mid;
  }
  return lo;
}
struct Multi {
  uint32_t bucket, pbase, count, pad;
};

// Task lengths are in [1, TASK]; tasks are emitted in descending length (a counting sort
// over TASK+1 bins) so the 32 lanes of a warp walk buckets of nearly equal size.
constexpr int kMaxTask = 96;

// Pass 1: per bucket, histogram of its task lengths; empty buckets become infinity.
template <class F>
__global__ void k_task_hist(const uint32_t* __restrict__ offsets, uint32_t nb, uint32_t task_len,
                            uint32_t* __restrict__ hist, uint32_t* __restrict__ buckets) {
  __shared__ uint32_t sh[kMaxTask + 1];
  for (int i = threadIdx.x; i <= kMaxTask; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nb) {
    const uint32_t cnt = offsets[b + 1] - offsets[b];
    if (cnt == 0) {
      constexpr int XW = 4 * FieldWords<F>::value;
      st_xyzz<F>(buckets + (size_t)b * XW, XYZZ<F>::inf());
    } else {
      const uint32_t nfull = (cnt - 1) / task_len;
      if (nfull) atomicAdd(&sh[task_len], nfull);
      atomicAdd(&sh[cnt - nfull * task_len], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= kMaxTask; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Bin cursors in descending length order; counters[0] = number of tasks.
static __global__ void k_task_bins(const uint32_t* __restrict__ hist, uint32_t task_len,
                            uint32_t* __restrict__ cursor, uint32_t* __restrict__ counters) {
  if (threadIdx.x != 0) return;
  uint32_t run = 0;
  for (int l = (int)task_len; l >= 1; l--) {
    cursor[l] = run;
    run += hist[l];
  }
  counters[0] = run;
}

// Pass 2: emit task records at their sorted positions.  Each block reserves a range per
// length bin with one global atomic, then ranks its tasks inside it.
template <class F>
__global__ void k_task_emit(const uint32_t* __restrict__ offsets, uint32_t nb, uint32_t task_len,
                            uint32_t* __restrict__ cursor, Task* __restrict__ tasks,
                            uint32_t* __restrict__ counters, Multi* __restrict__ multi,
                            const BatchJob* __restrict__ jobs = nullptr, uint32_t njobs = 0) {
  __shared__ uint32_t cnt_s[kMaxTask + 1], base_s[kMaxTask + 1];
  for (int i = threadIdx.x; i <= kMaxTask; i += blockDim.x) cnt_s[i] = 0;
  __syncthreads();
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t start = 0, cnt = 0, nfull = 0, last = 0;
  if (b < nb) {
    start = offsets[b];
    cnt = offsets[b + 1] - start;
    if (cnt) {
      nfull = (cnt - 1) / task_len;
      last = cnt - nfull * task_len;
      if (nfull) atomicAdd(&cnt_s[task_len], nfull);
      atomicAdd(&cnt_s[last], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= kMaxTask; i += blockDim.x)
    base_s[i] = cnt_s[i] ? atomicAdd(&cursor[i], cnt_s[i]) : 0u;
  __syncthreads();
  for (int i = threadIdx.x; i <= kMaxTask; i += blockDim.x) cnt_s[i] = 0;
  __syncthreads();
  if (cnt == 0) return;
  const uint32_t nt = nfull + 1;
  const uint32_t job = jobs ? job_of_bucket(jobs, njobs, b) : 0u;
  uint32_t pbase = 0;
  if (nt > 1) {
    pbase = atomicAdd(&counters[1], nt);
    const uint32_t mslot = atomicAdd(&counters[2], 1u);
    multi[mslot] = {b, pbase, nt, 0u};
  }
#pragma unroll 1
  for (uint32_t t = 0; t < nt; t++) {
    const uint32_t len = t < nfull ? task_len : last;
    const uint32_t slot = base_s[len] + atomicAdd(&cnt_s[len], 1u);
    tasks[slot] = {start + t * task_len, len, nt == 1 ? b : nb + pbase + t, job};
  }
}

// Minimum resident blocks per SM asked of the compiler for the accumulation kernel (0 = no
// register cap): G2 at 3 (168 registers: 12 warps per SM instead of 8, measured faster), G1
// uncapped (caps spilled and measured slower).
template <class F> struct AccMinBlocks { static constexpr int value = 0; };
template <> struct AccMinBlocks<Fq2> { static constexpr int value = 3; };

// The accumulation's mixed addition: over Fq with lazily reduced coordinates (no final
// conditional subtraction per product; the bucket is canonicalised when stored), over Fq2
// the canonical one.
CSB_DEV XYZZ<Fq> madd_acc(const XYZZ<Fq>& acc, const Affine<Fq>& p) { return xyzz_madd_lazy(acc, p); }
CSB_DEV XYZZ<Fq2> madd_acc(const XYZZ<Fq2>& acc, const Affine<Fq2>& p) { return xyzz_madd(acc, p); }
CSB_DEV XYZZ<Fq> canon_acc(const XYZZ<Fq>& a) { return xyzz_canon(a); }
CSB_DEV XYZZ<Fq2> canon_acc(const XYZZ<Fq2>& a) { return a; }

template <class F>
__global__ void __launch_bounds__(128, AccMinBlocks<F>::value) k_accumulate(const Task* __restrict__ tasks,
                                                    const uint32_t* __restrict__ counters,
                                                    const uint32_t* __restrict__ entries,
                                                    const uint32_t* __restrict__ points, uint32_t nb,
                                                    uint32_t* __restrict__ buckets,
                                                    uint32_t* __restrict__ partials,
                                                    const BatchJob* __restrict__ jobs = nullptr,
                                                    const uint32_t* __restrict__ phix = nullptr) {
  constexpr int PW = 2 * FieldWords<F>::value;
  constexpr int XW = 4 * FieldWords<F>::value;
  const uint32_t ntasks = counters[0];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += gridDim.x * blockDim.x) {
    const Task tk = tasks[t];
    const uint32_t* base = jobs ? jobs[tk.job].points : points;
    XYZZ<F> acc = XYZZ<F>::inf();
    if (entries) {
#pragma unroll 1
      for (uint32_t e = 0; e < tk.len; e++) {
        const uint32_t ent = entries[tk.start + e];
        Affine<F> p = ld_entry_point<F>(base, phix, ent);
        if (ent & NEG_BIT) p.y = p.y.neg();
        acc = madd_acc(acc, p);
      }
    } else {  // after batch-affine rounds: points in bucket order, (0, 0) = infinity
#pragma unroll 1
      for (uint32_t e = 0; e < tk.len; e++) {
        const Affine<F> p = ld_affine<F>(base + (size_t)(tk.start + e) * PW);
        if (!(p.x.is_zero() && p.y.is_zero())) acc = madd_acc(acc, p);
      }
    }
    uint32_t* dst = tk.dst < nb ? buckets + (size_t)tk.dst * XW : partials + (size_t)(tk.dst - nb) * XW;
    st_xyzz<F>(dst, canon_acc(acc));
  }
}

// Latency form of k_accumulate for an MSM too small to fill the GPU: one quad per task, each
// lane computing one product of each level of the mixed addition (4 product latencies per
// addition instead of 10).  Same tasks, same results.  The quad operations shuffle across
// the whole warp, so the 8 quads of a warp step together: each walks the longest of the
// warp's 8 tasks and keeps its accumulator past its own task's end (tasks are emitted
// longest first, so neighbours are about as long).
template <class F>
__global__ void __launch_bounds__(128, AccMinBlocks<F>::value) k_accumulate_quad(
    const Task* __restrict__ tasks, const uint32_t* __restrict__ counters, const uint32_t* __restrict__ entries,
    const uint32_t* __restrict__ points, uint32_t nb, uint32_t* __restrict__ buckets,
    uint32_t* __restrict__ partials, const BatchJob* __restrict__ jobs = nullptr,
    const uint32_t* __restrict__ phix = nullptr) {
  constexpr int PW = 2 * FieldWords<F>::value;
  constexpr int XW = 4 * FieldWords<F>::value;
  constexpr uint32_t G = GroupLanes<F>::value, QPW = 32 / G;  // lanes per group, groups per warp
  const uint32_t ntasks = counters[0];
  const uint32_t warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t qw = (threadIdx.x & 31) / G;  // group within the warp
  for (uint32_t base = warp0 * QPW; base < ntasks; base += nwarps * QPW) {  // warp-uniform
    const uint32_t t = base + qw;
    const bool valid = t < ntasks;
    const Task tk = valid ? tasks[t] : Task{0, 0, 0, 0};
    const uint32_t* pts = jobs && valid ? jobs[tk.job].points : points;  // read only where live
    const uint32_t steps = __reduce_max_sync(0xffffffffu, tk.len);
    XYZZ<F> acc = XYZZ<F>::inf();
#pragma unroll 1
    for (uint32_t e = 0; e < steps; e++) {
      const bool live = e < tk.len;
      Affine<F> p{F::zero(), F::zero()};  // past the task's end: not taken
      if (live) {
        if (entries) {
          const uint32_t ent = entries[tk.start + e];
          p = ld_entry_point<F>(pts, phix, ent);
          if (ent & NEG_BIT) p.y = p.y.neg();
        } else {
          p = ld_affine<F>(pts + (size_t)(tk.start + e) * PW);
        }
      }
      const XYZZ<F> nxt = xyzz_madd_quad(acc, p);
      const bool take = live && (entries || !(p.x.is_zero() && p.y.is_zero()));
      acc = xyzz_select(take, nxt, acc);
    }
    if (valid && (threadIdx.x & (G - 1)) == 0) {
      uint32_t* dst = tk.dst < nb ? buckets + (size_t)tk.dst * XW : partials + (size_t)(tk.dst - nb) * XW;
      st_xyzz<F>(dst, acc);
    }
  }
}

// buckets[b] += add[b] (XYZZ, canonical): folds another fixed-base MSM's buckets (same window)
// into this one's before the reduction.
template <class F>
__global__ void __launch_bounds__(128) k_add_buckets(uint32_t* __restrict__ buckets, const uint32_t* __restrict__ add,
                                                     uint32_t nb) {
  constexpr int XW = 4 * FieldWords<F>::value;
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const XYZZ<F> x = ld_xyzz<F>(buckets + (size_t)b * XW), y = ld_xyzz<F>(add + (size_t)b * XW);
  st_xyzz<F>(buckets + (size_t)b * XW, xyzz_add(x, y));
}

// Split buckets with at most kCombineSerial partials: one thread each, a serial sum.
// (The top window of a scalar has fewer bits, so its digits crowd into fewer buckets and
// many of those split into two or three tasks.)
constexpr uint32_t kCombineSerial = 8;

template <class F>
__global__ void __launch_bounds__(128) k_combine_small(const Multi* __restrict__ multi,
                                                       const uint32_t* __restrict__ counters,
                                                       const uint32_t* __restrict__ partials,
                                                       uint32_t* __restrict__ buckets) {
  constexpr int XW = 4 * FieldWords<F>::value;
  const uint32_t nm = counters[2];
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < nm; m += gridDim.x * blockDim.x) {
    const Multi mu = multi[m];
    if (mu.count > kCombineSerial) continue;
    XYZZ<F> acc = ld_xyzz<F>(partials + (size_t)mu.pbase * XW);
#pragma unroll 1
    for (uint32_t i = 1; i < mu.count; i++) acc = xyzz_add(acc, ld_xyzz<F>(partials + (size_t)(mu.pbase + i) * XW));
    st_xyzz<F>(buckets + (size_t)mu.bucket * XW, acc);
  }
}

// Split buckets with more partials: one block each, tree sum.
template <class F>
__global__ void __launch_bounds__(128) k_combine(const Multi* __restrict__ multi,
                                                 const uint32_t* __restrict__ counters,
                                                 const uint32_t* __restrict__ partials,
                                                 uint32_t* __restrict__ buckets) {
  constexpr int XW = 4 * FieldWords<F>::value;
  __shared__ uint32_t red[4][XW];
  const uint32_t nm = counters[2];
  for (uint32_t m = blockIdx.x; m < nm; m += gridDim.x) {
    const Multi mu = multi[m];
    if (mu.count <= kCombineSerial) continue;  // k_combine_small
    XYZZ<F> acc = XYZZ<F>::inf();
#pragma unroll 1
    for (uint32_t i = threadIdx.x; i < mu.count; i += blockDim.x)
      acc = xyzz_add_cold(acc, ld_xyzz<F>(partials + (size_t)(mu.pbase + i) * XW));
    // warp tree
#pragma unroll 1
    for (int d = 16; d > 0; d >>= 1) {
      XYZZ<F> o;
      uint32_t* ow = reinterpret_cast<uint32_t*>(&o);
      const uint32_t* aw = reinterpret_cast<const uint32_t*>(&acc);
#pragma unroll
      for (int w = 0; w < XW; w++) ow[w] = __shfl_down_sync(0xffffffffu, aw[w], d);
      acc = xyzz_add_cold(acc, o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
      const uint32_t* aw = reinterpret_cast<const uint32_t*>(&acc);
      for (int w = 0; w < XW; w++) red[warp][w] = aw[w];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      XYZZ<F> s = XYZZ<F>::inf();
#pragma unroll 1
      for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
        XYZZ<F> o;
        uint32_t* ow = reinterpret_cast<uint32_t*>(&o);
        for (int w = 0; w < XW; w++) ow[w] = red[k][w];
        s = xyzz_add_cold(s, o);
      }
      st_xyzz<F>(buckets + (size_t)mu.bucket * XW, s);
    }
    __syncthreads();
  }
}

// Level k of the bucket reduction.  y: W sequences of n XYZZ points (stride n); z: the
// weighted carry from the previous level (null at level 0).  Thread (j, t) handles
// y[j][8t .. 8t+8):
//   acc = sum_i y_i,  s = sum_i i*y_i,  z'[j][t] = sum_i z[j][8t+i] + 8^k * s,
//   y'[j][t] = acc.
template <class F>
__global__ void __launch_bounds__(128) k_reduce_level(const uint32_t* __restrict__ y,
                                                      const uint32_t* __restrict__ z, uint32_t n,
                                                      uint32_t nout, int W, int level,
                                                      uint32_t* __restrict__ yout,
                                                      uint32_t* __restrict__ zout) {
  constexpr int XW = 4 * FieldWords<F>::value;
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (uint32_t)W * nout) return;
  const uint32_t j = g / nout, t = g % nout;
  const uint32_t* yj = y + (size_t)j * n * XW;
  XYZZ<F> acc = XYZZ<F>::inf(), s = XYZZ<F>::inf();
#pragma unroll 1
  for (int i = 7; i >= 1; i--) {
    const uint32_t idx = 8 * t + i;
    if (idx < n) acc = xyzz_add(acc, ld_xyzz<F>(yj + (size_t)idx * XW));
    s = xyzz_add(s, acc);
  }
  if (8 * t < n) acc = xyzz_add(acc, ld_xyzz<F>(yj + (size_t)(8 * t) * XW));
#pragma unroll 1
  for (int d = 0; d < 3 * level; d++) s = xyzz_dbl(s);
  if (z) {
    const uint32_t* zj = z + (size_t)j * n * XW;
#pragma unroll 1
    for (int i = 0; i < 8; i++) {
      const uint32_t idx = 8 * t + i;
      if (idx < n) s = xyzz_add(s, ld_xyzz<F>(zj + (size_t)idx * XW));
    }
  }
  st_xyzz<F>(yout + ((size_t)j * nout + t) * XW, acc);
  st_xyzz<F>(zout + ((size_t)j * nout + t) * XW, s);
}


// k_reduce_level with one quad per output segment (quad point operations): the latency form
// for levels too small to fill the GPU.  Every lane of a launched warp runs the operations
// (quads past the end work on points at infinity and store nothing).
template <class F>
__global__ void __launch_bounds__(128) k_reduce_level_quad(const uint32_t* __restrict__ y,
                                                           const uint32_t* __restrict__ z, uint32_t n,
                                                           uint32_t nout, int W, int level,
                                                           uint32_t* __restrict__ yout,
                                                           uint32_t* __restrict__ zout) {
  constexpr int XW = 4 * FieldWords<F>::value;
  constexpr uint32_t G = GroupLanes<F>::value;
  const uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool valid = g < (uint32_t)W * nout;
  const uint32_t j = valid ? g / nout : 0u, t = valid ? g % nout : 0u;
  const uint32_t* yj = y + (size_t)j * n * XW;
  // running sum acc and sum of running sums s over the segment's buckets 7..1, starting at
  // bucket 7 (no additions to infinity)
  XYZZ<F> acc = valid && 8 * t + 7 < n ? ld_xyzz<F>(yj + (size_t)(8 * t + 7) * XW) : XYZZ<F>::inf();
  XYZZ<F> s = acc;
#pragma unroll 1
  for (int i = 6; i >= 1; i--) {
    const uint32_t idx = 8 * t + i;
    const XYZZ<F> v = valid && idx < n ? ld_xyzz<F>(yj + (size_t)idx * XW) : XYZZ<F>::inf();
    acc = add_q(acc, v);
    s = add_q(s, acc);
  }
  {
    const XYZZ<F> v = valid && 8 * t < n ? ld_xyzz<F>(yj + (size_t)(8 * t) * XW) : XYZZ<F>::inf();
    acc = add_q(acc, v);
  }
#pragma unroll 1
  for (int d = 0; d < 3 * level; d++) s = dbl_q(s);
  if (z) {  // uniform: a kernel argument
    const uint32_t* zj = z + (size_t)j * n * XW;
#pragma unroll 1
    for (int i = 0; i < 8; i++) {
      const uint32_t idx = 8 * t + i;
      const XYZZ<F> v = valid && idx < n ? ld_xyzz<F>(zj + (size_t)idx * XW) : XYZZ<F>::inf();
      s = add_q(s, v);
    }
  }
  if (valid && (threadIdx.x & (G - 1)) == 0) {
    st_xyzz<F>(yout + ((size_t)j * nout + t) * XW, acc);
    st_xyzz<F>(zout + ((size_t)j * nout + t) * XW, s);
  }
}

template <class F>
CSB_DEV XYZZ<F> shfl_down_xyzz(const XYZZ<F>& v, int d) {
  constexpr int XW = 4 * FieldWords<F>::value;
  XYZZ<F> o;
  uint32_t* ow = reinterpret_cast<uint32_t*>(&o);
  const uint32_t* vw = reinterpret_cast<const uint32_t*>(&v);
#pragma unroll
  for (int w = 0; w < XW; w++) ow[w] = __shfl_down_sync(0xffffffffu, vw[w], d);
  return o;
}

// k_reduce_level_quad for the levels that carry weighted sums z (levels >= 1): two quads per
// output segment, side by side in one warp.  The even quad runs the running sums of the segment
// totals y and then the doublings; the odd quad sums the segment's eight z values meanwhile (each
// step is the same point addition on operands picked by role, so the warp does not diverge), and
// one shuffle and one addition join them: 13 + 3L + 1 dependent point operations instead of
// 13 + 3L + 8.  Same sums as k_reduce_level_quad.
template <class F>
__global__ void __launch_bounds__(128) k_reduce_level_quad2(const uint32_t* __restrict__ y,
                                                            const uint32_t* __restrict__ z, uint32_t n,
                                                            uint32_t nout, int W, int level,
                                                            uint32_t* __restrict__ yout,
                                                            uint32_t* __restrict__ zout) {
  constexpr int XW = 4 * FieldWords<F>::value;
  constexpr uint32_t G = GroupLanes<F>::value;
  const uint32_t gq = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const uint32_t g = gq >> 1;
  const bool zq = (gq & 1) != 0;  // the odd quad of the pair sums the z values
  const bool valid = g < (uint32_t)W * nout;
  const uint32_t j = valid ? g / nout : 0u, t = valid ? g % nout : 0u;
  const uint32_t* yj = y + (size_t)j * n * XW;
  const uint32_t* zj = z + (size_t)j * n * XW;
  auto ld = [&](const uint32_t* base, uint32_t i) {
    const uint32_t idx = 8 * t + i;
    return valid && idx < n ? ld_xyzz<F>(base + (size_t)idx * XW) : XYZZ<F>::inf();
  };
  // even quad: a = running sum from bucket 7 down, s = sum of the running sums 7..1;
  // odd quad: a = z_0 + ... + z_7
  XYZZ<F> a = zq ? ld(zj, 0) : ld(yj, 7);
  XYZZ<F> s = a;
#pragma unroll 1
  for (int step = 0; step < 13; step++) {
    // even quad: even steps a += y_i (i = 6..0), odd steps s += a; odd quad: a += z_{step+1}
    const bool even_step = (step & 1) == 0;
    XYZZ<F> p, q;
    if (zq) {
      p = a;
      q = step < 7 ? ld(zj, step + 1) : XYZZ<F>::inf();
    } else if (even_step) {
      p = a;
      q = ld(yj, 6 - (step >> 1));
    } else {
      p = s;
      q = a;
    }
    const XYZZ<F> r = add_q(p, q);  // every lane of the warp, every step
    if (zq || even_step) a = r; else s = r;
  }
  // the odd quads double their own s too and drop it: the quad operations shuffle across
  // the whole warp, so every lane takes part in the same steps (no extra latency)
#pragma unroll 1
  for (int d = 0; d < 3 * level; d++) s = dbl_q(s);
  s = add_q(s, shfl_down_xyzz(a, G));  // even groups: + the odd neighbour's z sum
  if (valid && !zq && (threadIdx.x & (G - 1)) == 0) {
    st_xyzz<F>(yout + ((size_t)j * nout + t) * XW, a);
    st_xyzz<F>(zout + ((size_t)j * nout + t) * XW, s);
  }
}

// Per-window sum after levels 0..L-1.  With y_t the segment totals and z_t the weighted
// carries of the last level, S_j = sum_t (y_t + z_t) + G * sum_t t * y_t with G = 8^L =
// 2^shift.  One block per window, E consecutive segments per virtual thread u:
//   V_u = Y_u + Z_u + G * sum_i i*y_{uE+i}      (Y_u, Z_u: the thread's totals)
//   sum_t t*y_t = sum_u [sum_i i*y_{uE+i}] + E * sum_{u>=1} Suf(u),  Suf(u) = sum_{v>=u} Y_v
// so S_j = sum_u (Y_u + Z_u + G (W_u + E Suf(u) [u >= 1])) with W_u = sum_i i*y_{uE+i}: a suffix
// scan and a reduction over the block's virtual threads, about 3E + 2 log2(VT) + shift
// dependent point operations instead of a serial pass over the segments.
// Threads of the per-window sum (one block per window).  128 (4 warps, one per SM
// sub-partition) shortens each dependent point operation enough to pay for the longer chains
// of 32 virtual threads: 2^12 proof 2.00 -> 1.91 ms, G2 2^12 fixed-base MSM 1.68 -> 1.58 ms.
// Over Fq2 (16-lane groups) 256 threads, 16 virtual threads, for the single MSM and batches
// (128: G2 fixed-base 2^20 13.5 ms, 256: 13.0; 512 slower at every size).
constexpr int kWsumThreads = 128;
template <class F> struct WsumThreads { static constexpr int single = kWsumThreads, batch = 256; };
template <> struct WsumThreads<Fq2> { static constexpr int single = 256, batch = 256; };
template <class F, int THREADS>
__global__ void __launch_bounds__(THREADS) k_window_sum(const uint32_t* __restrict__ y,
                                                        const uint32_t* __restrict__ z, uint32_t n1,
                                                        int shift, uint32_t* __restrict__ wsum) {
  // Group form: each group of G lanes is one virtual thread u running group point operations,
  // so the block has VT = THREADS / G virtual threads.  The scan and the reduction across them
  // go through shared memory (double-buffered Hillis-Steele steps); the group's first lane
  // writes, every lane reads.
  constexpr int XW = 4 * FieldWords<F>::value;
  constexpr uint32_t G = GroupLanes<F>::value;
  constexpr uint32_t VT = THREADS / G;
  static_assert(VT >= 1 && (VT & (VT - 1)) == 0, "virtual threads: a power of two");
  __shared__ uint32_t sh[2][VT][XW];
  const int j = blockIdx.x;
  const uint32_t* yj = y + (size_t)j * n1 * XW;
  const uint32_t* zj = z + (size_t)j * n1 * XW;
  const uint32_t E = (n1 + VT - 1) / VT;  // n1 is a power of two
  const uint32_t u = threadIdx.x / G;
  const bool lead = (threadIdx.x & (G - 1)) == 0;
  auto put = [&](int b, uint32_t slot, const XYZZ<F>& v) {
    if (lead) {
      const uint32_t* w = reinterpret_cast<const uint32_t*>(&v);
      for (int k = 0; k < XW; k++) sh[b][slot][k] = w[k];
    }
  };
  auto get = [&](int b, uint32_t slot) {
    XYZZ<F> v;
    uint32_t* w = reinterpret_cast<uint32_t*>(&v);
    for (int k = 0; k < XW; k++) w[k] = sh[b][slot][k];
    return v;
  };
  // the sums start at the thread's last segment (no additions to infinity)
  XYZZ<F> acc, zs, ws = XYZZ<F>::inf();
  {
    const uint32_t idx = u * E + (E - 1);
    const bool in = idx < n1;
    acc = in ? ld_xyzz<F>(yj + (size_t)idx * XW) : XYZZ<F>::inf();
    zs = in ? ld_xyzz<F>(zj + (size_t)idx * XW) : XYZZ<F>::inf();
  }
#pragma unroll 1
  for (int i = (int)E - 2; i >= 0; i--) {  // uniform trip count; past n1 the terms are infinity
    const uint32_t idx = u * E + i;
    const bool in = idx < n1;
    ws = add_q(ws, acc);  // acc = sum of the thread's segments above i
    acc = add_q(acc, in ? ld_xyzz<F>(yj + (size_t)idx * XW) : XYZZ<F>::inf());
    zs = add_q(zs, in ? ld_xyzz<F>(zj + (size_t)idx * XW) : XYZZ<F>::inf());
  }
  // V_u = acc + zs + 2^shift (ws + E Suf(u) [u >= 1]): one chain of shift doublings for both
  // terms (ws is infinity with one segment per thread)
  XYZZ<F> V = add_q(acc, zs);
  // inclusive suffix scan of acc over the virtual threads: Suf(u)
  XYZZ<F> suf = acc;
  int cur = 0;
  put(cur, u, suf);
  __syncthreads();
#pragma unroll 1
  for (uint32_t d = 1; d < VT; d <<= 1) {
    const bool has = u + d < VT;
    const XYZZ<F> o = has ? get(cur, u + d) : XYZZ<F>::inf();
    suf = xyzz_select(has, add_q(suf, o), suf);
    cur ^= 1;
    put(cur, u, suf);
    __syncthreads();
  }
  {  // computed by every group (uniform); E Suf(u) kept where u >= 1 and u E < n1
#pragma unroll 1
    for (uint32_t m = E; m > 1; m >>= 1) suf = dbl_q(suf);  // E is a power of two
    XYZZ<F> T = xyzz_select(u >= 1 && u * E < n1, add_q(ws, suf), ws);
#pragma unroll 1
    for (int d = 0; d < shift; d++) T = dbl_q(T);
    V = add_q(V, T);
  }
  // reduction of V over the virtual threads
  cur ^= 1;  // the buffer no step reads any more
  put(cur, u, V);
  __syncthreads();
#pragma unroll 1
  for (uint32_t d = VT / 2; d >= 1; d >>= 1) {
    const bool has = u < d;
    const XYZZ<F> o = has ? get(cur, u + d) : XYZZ<F>::inf();
    V = xyzz_select(has, add_q(V, o), V);
    cur ^= 1;
    put(cur, u, V);
    __syncthreads();
  }
  if (u == 0 && lead) st_xyzz<F>(wsum + (size_t)j * XW, V);
}

// sum_j 2^(c j) S_j (Horner over the windows) and the affine result.
template <class F>
__global__ void k_finish(const uint32_t* __restrict__ wsum, int W, int c, uint32_t* __restrict__ out) {
  constexpr int XW = 4 * FieldWords<F>::value;
  if (blockIdx.x != 0) return;
  // one warp (launched with 32 threads; its 8 quads compute the same): the independent
  // products of each doubling and addition run on the lanes of a quad
  XYZZ<F> r = ld_xyzz<F>(wsum + (size_t)(W - 1) * XW);
#pragma unroll 1
  for (int j = W - 2; j >= 0; j--) {
#pragma unroll 1
    for (int d = 0; d < c; d++) r = xyzz_dbl_quad(r);
    r = xyzz_add_quad(r, ld_xyzz<F>(wsum + (size_t)j * XW));
  }
  if (threadIdx.x == 0) st_affine<F>(out, xyzz_to_affine(r));
}

template <class F>
__global__ void k_store_inf(uint32_t* out) {
  if (threadIdx.x == 0) st_affine<F>(out, Affine<F>{F::zero(), F::one()});
}

// ---------------------------------------------------------- batch-affine rounds ----
// Before the XYZZ accumulation, buckets are halved R times by adding their points in pairs
// in affine coordinates: lambda = (y2 - y1) / (x2 - x1) (or 3 x^2 / 2y for equal points),
// x3 = lambda^2 - x1 - x2, y3 = lambda (x1 - x3) - y1.  The divisions of kAffK consecutive
// pairs share one inversion (Montgomery's simultaneous inversion: prefix products, one
// inverse, back substitution), so an addition costs about 6 products instead of the
// 10 of an XYZZ + affine addition.  Round r maps bucket b's c_b points at in_off[b] to
// ceil(c_b / 2) points at out_off[b]; an odd last point is copied.  Points at infinity
// inside the rounds are (0, 0), which is on neither curve.
constexpr uint32_t kAffK = 64;  // 32 and 128 measured slower (G2 fixed-base 2^20)

template <class F>
CSB_DEV bool aff_zero(const Affine<F>& a) { return a.x.is_zero() && a.y.is_zero(); }

// Pair of round-r inputs for output slot s of bucket b.  FIRST: round 0 reads the bases
// through the sorted entries (sign bit -> negated y); later rounds read the previous round.
template <class F, bool FIRST>
CSB_DEV void aff_pair(const uint32_t* in_off, const uint32_t* out_off, uint32_t b, uint32_t s,
                      const uint32_t* entries, const uint32_t* src, Affine<F>& p, Affine<F>& q, bool& has_q) {
  constexpr int PW = 2 * FieldWords<F>::value;
  const uint32_t j = s - out_off[b];
  const uint32_t i0 = in_off[b] + 2 * j;
  has_q = i0 + 1 < in_off[b + 1];
  if (FIRST) {
    const uint32_t e0 = entries[i0];
    p = ld_affine<F>(src + (size_t)(e0 & ~NEG_BIT) * PW);
    if (e0 & NEG_BIT) p.y = p.y.neg();
    if (has_q) {
      const uint32_t e1 = entries[i0 + 1];
      q = ld_affine<F>(src + (size_t)(e1 & ~NEG_BIT) * PW);
      if (e1 & NEG_BIT) q.y = q.y.neg();
    }
  } else {
    p = ld_affine<F>(src + (size_t)i0 * PW);
    if (has_q) q = ld_affine<F>(src + (size_t)(i0 + 1) * PW);
  }
}

// Denominator of a pair and its kind: 0 add, 1 double, 2 result p, 3 result q, 4 infinity.
template <class F>
CSB_DEV int aff_kind(const Affine<F>& p, const Affine<F>& q, bool has_q, F& d) {
  d = F::one();
  if (!has_q || aff_zero(q)) return 2;
  if (aff_zero(p)) return 3;
  if (!(p.x == q.x)) {
    d = q.x - p.x;
    return 0;
  }
  if (p.y == q.y) {
    d = p.y.dbl();
    return 1;
  }
  return 4;
}

// The denominator of slot s from the two x coordinates alone (half the bytes of the pair);
// the y coordinates are read only where the kind depends on them (a zero x: a point at
// infinity or x = 0; equal x: doubling or opposite points).
template <class F, bool FIRST>
CSB_DEV F aff_denominator(const uint32_t* in_off, const uint32_t* out_off, uint32_t b, uint32_t s,
                          const uint32_t* entries, const uint32_t* src) {
  constexpr int PW = 2 * FieldWords<F>::value;
  const uint32_t i0 = in_off[b] + 2 * (s - out_off[b]);
  if (i0 + 1 >= in_off[b + 1]) return F::one();  // odd last point: copied
  const uint32_t a0 = FIRST ? (entries[i0] & ~NEG_BIT) : i0;
  const uint32_t a1 = FIRST ? (entries[i0 + 1] & ~NEG_BIT) : i0 + 1;
  F px, qx;
  ld_field(px, src + (size_t)a0 * PW);
  ld_field(qx, src + (size_t)a1 * PW);
  if (!px.is_zero() && !qx.is_zero() && !(px == qx)) return qx - px;
  Affine<F> p, q;
  bool has_q;
  aff_pair<F, FIRST>(in_off, out_off, b, s, entries, src, p, q, has_q);
  F d;
  aff_kind(p, q, has_q, d);
  return d;
}

template <class F>
CSB_DEV uint32_t bucket_of_slot(const uint32_t* off, uint32_t nb, uint32_t s) {
  uint32_t lo = 0, hi = nb;  // largest b with off[b] <= s (empty buckets share offsets)
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= s) lo = mid; else hi = mid;
  }
  return lo;
}

template <class F, bool FIRST>
__global__ void __launch_bounds__(128) k_affine_round(const uint32_t* __restrict__ in_off,
                                                      const uint32_t* __restrict__ out_off, uint32_t nb,
                                                      const uint32_t* __restrict__ entries,
                                                      const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                                      uint32_t* __restrict__ pref) {
  constexpr int FW = FieldWords<F>::value;
  constexpr int PW = 2 * FW;
  const uint32_t total = out_off[nb];
  const uint32_t s0 = (blockIdx.x * blockDim.x + threadIdx.x) * kAffK;
  if (s0 >= total) return;
  const uint32_t s1 = min(total, s0 + kAffK);
  const uint32_t b0 = bucket_of_slot<F>(out_off, nb, s0);
  // phase 1: prefix products of the denominators
  F acc = F::one();
  uint32_t b = b0;
  for (uint32_t s = s0; s < s1; s++) {
    while (out_off[b + 1] <= s) b++;
    acc = acc * aff_denominator<F, FIRST>(in_off, out_off, b, s, entries, src);
    st_field(pref + (size_t)s * FW, acc);
  }
  F inv = acc.inv();
  // phase 2: back substitution and the additions, last slot first
  for (uint32_t s = s1; s-- > s0;) {
    while (out_off[b] > s) b--;
    Affine<F> p, q;
    bool has_q;
    aff_pair<F, FIRST>(in_off, out_off, b, s, entries, src, p, q, has_q);
    F d;
    const int kind = aff_kind(p, q, has_q, d);
    F before = F::one();
    if (s > s0) {  // written above by this thread: a plain (coherent) load, not __ldg
      uint32_t* bw = reinterpret_cast<uint32_t*>(&before);
      const uint4* pv = reinterpret_cast<const uint4*>(pref + (size_t)(s - 1) * FW);
#pragma unroll
      for (int k = 0; k < FW / 4; k++) {
        const uint4 v = pv[k];
        bw[4 * k] = v.x; bw[4 * k + 1] = v.y; bw[4 * k + 2] = v.z; bw[4 * k + 3] = v.w;
      }
    }
    const F id = inv * before;  // 1 / d
    inv = inv * d;
    Affine<F> r;
    if (kind == 0 || kind == 1) {
      const F lam = kind == 0 ? (q.y - p.y) * id : (p.x.sqr() * (F::one() + F::one() + F::one())) * id;
      const F x3 = lam.sqr() - p.x - q.x;
      r.x = x3;
      r.y = lam * (p.x - x3) - p.y;
    } else if (kind == 2) {
      r = p;
    } else if (kind == 3) {
      r = q;
    } else {
      r.x = F::zero();
      r.y = F::zero();
    }
    st_affine<F>(dst + (size_t)s * PW, r);
  }
}

// out[b] = ceil(in[b] / 2) for the next round's counts (written into a count array that the
// scan turns into offsets; out[nb] = 0 so the scan's last element is the total).
static __global__ void k_half_counts(const uint32_t* __restrict__ off, uint32_t nb, uint32_t* __restrict__ out) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nb) out[b] = (off[b + 1] - off[b] + 1) >> 1;
  if (b == nb) out[b] = 0;
}

// --------------------------------------------------------------- workspace layout ----
// counters block: [0] tasks, [1] partial slots, [2] split buckets; hist at +16 and
// bin cursors at +128 (kMaxTask + 1 words each).
constexpr int kCtrHist = 16, kCtrCursor = 128, kCtrWords = 256;
static_assert(kCtrHist + kMaxTask + 1 <= kCtrCursor && kCtrCursor + kMaxTask + 1 <= kCtrWords,
              "task-length bins must not overlap");
// the reduction adds levels until a window has at most this many segments
constexpr uint32_t kTopSegments = 256;

struct Layout {
  size_t counts, offsets, entries, tasks, multi, partials, buckets, lv_y, lv_z, lv_y2, lv_z2, wsum,
      counters, off2, pa, pb, pref, glv_s, glv_p, total;
  bool affine, glv;
};

static inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// task_len: the shortest task the MSM will run (0: automatic, layout_min_task of its entries).
inline Layout make_layout(uint32_t n, int c, int xyzz_bytes, uint32_t task_len, bool fixed = false,
                          bool affine = true, bool glv = false) {
  const int W = msm_windows(c, glv);
  const size_t nt = glv ? 2 * (size_t)n : n;  // terms the pipeline sorts (GLV: k1 P_i and k2 phi(P_i))
  const size_t nb = fixed ? ((size_t)1 << (c - 1)) : (size_t)W << (c - 1);
  const int WR = fixed ? 1 : W;  // bucket sets reduced
  const size_t ne = nt * W;
  if (task_len == 0) task_len = layout_min_task(ne);
  const size_t max_tasks = nb + ne / task_len + 1;
  const size_t max_partials = 2 * (ne / task_len) + 1;
  const size_t n1 = ((size_t)1 << (c - 1)) / 8 + 1;
  const size_t n2 = (size_t)WR * (n1 / 8 + 1);
  Layout L{};
  size_t o = 0;
  L.counters = o; o = align256(o + kCtrWords * sizeof(uint32_t));
  L.counts = o;   o = align256(o + (nb + 1) * sizeof(uint32_t));
  L.offsets = o;  o = align256(o + (nb + 1) * sizeof(uint32_t));
  L.entries = o;  o = align256(o + ne * sizeof(uint32_t));
  L.tasks = o;    o = align256(o + max_tasks * sizeof(Task));
  L.multi = o;    o = align256(o + (ne / (task_len + 1) + 1) * sizeof(Multi));
  L.partials = o; o = align256(o + max_partials * (size_t)xyzz_bytes);
  L.buckets = o;  o = align256(o + nb * (size_t)xyzz_bytes);
  L.lv_y = o;     o = align256(o + (size_t)WR * n1 * xyzz_bytes);
  L.lv_z = o;     o = align256(o + (size_t)WR * n1 * xyzz_bytes);
  L.lv_y2 = o;    o = align256(o + n2 * xyzz_bytes);
  L.lv_z2 = o;    o = align256(o + n2 * xyzz_bytes);
  L.wsum = o;     o = align256(o + (size_t)WR * xyzz_bytes);
  L.glv = glv;
  if (glv) {  // per term: both split halves (8 words) and beta x_i (8 words)
    L.glv_s = o;  o = align256(o + (size_t)n * 32);
    L.glv_p = o;  o = align256(o + (size_t)n * 32);
  }
  L.affine = affine;
  if (affine) {  // batch-affine rounds: offsets ping-pong, two point arrays, prefix products
    const size_t pb = (size_t)xyzz_bytes / 2, fb = (size_t)xyzz_bytes / 4;
    L.off2 = o;   o = align256(o + (nb + 1) * sizeof(uint32_t));
    L.pa = o;     o = align256(o + (ne / 2 + 2 * nb + 1) * pb);
    L.pb = o;     o = align256(o + (ne / 4 + 2 * nb + 1) * pb);
    L.pref = o;   o = align256(o + (ne / 2 + 2 * nb + 1) * fb);
  }
  L.total = o + scan_workspace_bytes(nb + 1);
  return L;
}

// Batch-affine rounds before the XYZZ accumulation (the expected bucket size is N W /
// buckets; a round needs about 8 points per bucket to pay).  Measured at 2^20: G1 is
// fastest without rounds (its XYZZ addition costs 10 products of 136 wide multiplies and
// already outruns the gather-bound affine round), G2 with two (Fq2 products are 3 Fq
// products, so the 6-vs-10 product saving outweighs the extra traffic).
inline int auto_affine_rounds_rt(bool ec2, uint32_t n, int W, size_t nb) {
  // a round runs kAffK pairs per thread in sequence around one inversion: it needs enough
  // pairs (>= 2^22, i.e. N W >= 2^23 entries) to fill the GPU, or its chain sets the latency
  // (2 rounds cost 2.5 ms in a 2^12-term G2 MSM)
  if ((uint64_t)n * W < (1ull << 23)) return 0;
  // G1 rounds measured slower, alone and inside proofs (2^20 proof 29.1 -> 30.2 ms with one
  // round, 30.7 ms with two; with the FP64-pipe products 26.5 -> 29.1 ms with one round, the
  // 2^20 fixed-base MSM 4.28 -> 5.20 ms): its mixed addition is cheap enough that the extra
  // passes lose.  L2 prefetching the round's gathers a few slots ahead did not help either
  // (G2 fixed-base 13.10 ms without, 13.27 / 13.31 / 13.40 ms 2 / 4 / 8 slots ahead).
  const int cap = ec2 ? 2 : 0;
  const double avg = (double)n * W / (double)nb;
  int r = 0;
  while (r < cap && avg >= (double)(8u << r)) r++;
  return r;
}
template <class F>
inline int auto_affine_rounds(uint32_t n, int W, size_t nb) {
  return auto_affine_rounds_rt(FieldWords<F>::value == 16, n, W, nb);
}
// Whether an MSM reserves the round buffers: affine_mode -1 auto, 0 never, > 0 that many rounds.
inline bool layout_affine(bool ec2, int affine_mode, uint32_t n, int c, bool fixed, bool glv = false) {
  if (affine_mode >= 0) return affine_mode > 0;
  const int W = msm_windows(c, glv);
  const size_t nb = fixed ? ((size_t)1 << (c - 1)) : (size_t)W << (c - 1);
  return auto_affine_rounds_rt(ec2, glv ? 2 * n : n, W, nb) > 0;
}
// Whether an MSM splits its scalars by the GLV endomorphism: generic G1 MSMs unless turned off.
// Batch-affine rounds (asked for explicitly; G1 runs none by default) read plain point indices,
// so they turn the split off.
inline bool use_glv(bool ec2, bool fixed, int glv_mode, int affine_mode, uint32_t n) {
  return !ec2 && !fixed && glv_mode != 0 && affine_mode <= 0 && n < PHI_BIT;
}

// Resident blocks of k_accumulate per SM, cached per device (callers on several threads and
// devices: server slots, the allocation-free entry point).
template <class F>
int accumulate_grid(int dev, int sms) {
  static std::atomic<int> blocks_per_sm[64];
  const int slot = dev >= 0 && dev < 64 ? dev : 0;
  int b = blocks_per_sm[slot].load(std::memory_order_relaxed);
  if (b == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_accumulate<F>, 128, 0) != cudaSuccess || b < 1)
      b = 1;
    blocks_per_sm[slot].store(b, std::memory_order_relaxed);
  }
  return b * sms;
}

// One level of the bucket reduction (level 0: y = the buckets, z = null): one thread per
// output segment while the level's groups would not fit the resident threads (least work,
// for full GPUs), else one group per segment (group point operations: a fraction of the
// chain's latency for a little more work).
template <class F>
void reduce_level(const uint32_t* y, const uint32_t* z, uint32_t n, uint32_t nout, int W, int level,
                  uint32_t* yout, uint32_t* zout, uint64_t resident, cudaStream_t st) {
  const uint64_t outs = (uint64_t)W * nout;
  // group forms while their lanes fit the resident threads once (G lanes per point
  // operation: 4 over Fq, 16 over Fq2); letting 16-lane groups run up to four times over
  // slowed a 2^20 proof 26.0 -> 26.8 ms and a batch of 16 proofs of 2^12 3.57 -> 3.94 ms
  constexpr uint64_t G = GroupLanes<F>::value;
  if (z && outs * 2 * G <= resident)
    k_reduce_level_quad2<F><<<(uint32_t)((outs * 2 * G + 127) / 128), 128, 0, st>>>(y, z, n, nout, W, level, yout,
                                                                                   zout);
  else if (outs * G <= resident)
    k_reduce_level_quad<F><<<(uint32_t)((outs * G + 127) / 128), 128, 0, st>>>(y, z, n, nout, W, level, yout, zout);
  else
    k_reduce_level<F><<<(uint32_t)((outs + 127) / 128), 128, 0, st>>>(y, z, n, nout, W, level, yout, zout);
  note_launch();
}

// One MSM.  Generic: d_points holds n points.  FIXED: d_points is a table of W*n points,
// T[j*n + i] = 2^(c j) P_i, built with the same c (fixed_table_impl).
template <class F, bool FIXED>
cudaError_t msm_impl(const uint32_t* d_scalars, const uint32_t* d_points, uint32_t n_in,
                     uint32_t* d_out, void* d_work, size_t work_bytes, const MsmConfig& cfg,
                     cudaStream_t st) {
  constexpr bool EC2 = FieldWords<F>::value == 16;
  constexpr int XB = 4 * FieldWords<F>::value * 4;  // bytes per XYZZ point
  // shared buckets: fixed-base MSMs (one bucket set) with terms (the accumulation is what
  // writes every bucket of the array)
  if ((cfg.bucket_out || cfg.bucket_add) && (!FIXED || n_in == 0)) return cudaErrorInvalidValue;
  if (cfg.bucket_out && cfg.bucket_add) return cudaErrorInvalidValue;
  if (n_in == 0) {
    k_store_inf<F><<<1, 32, 0, st>>>(d_out);
    note_launch();
    return cudaGetLastError();
  }
  if (FIXED && cfg.c <= 0) return cudaErrorInvalidValue;  // the table fixes the window
  const int c = cfg.c > 0 ? cfg.c : msm_default_window(n_in, EC2);
  if (c < 4 || c > 24) return cudaErrorInvalidValue;
  const bool glv = use_glv(EC2, FIXED, cfg.glv, cfg.affine, n_in);
  const int W = msm_windows(c, glv);
  // entry positions are uint32 and fixed-base entries carry a table index below the sign bit
  if ((uint64_t)W * n_in * (glv ? 2 : 1) >= (uint64_t)NEG_BIT) return cudaErrorInvalidValue;
  const uint32_t n = glv ? 2 * n_in : n_in;  // terms sorted into buckets
  const uint32_t nb = FIXED ? (1u << (c - 1)) : (uint32_t)W << (c - 1);
  const int rounds_req = cfg.affine < 0 ? auto_affine_rounds<F>(n, W, nb) : cfg.affine;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // threads the accumulation keeps resident: an MSM whose tasks (at the shortest length) fit
  // four times over runs in latency form (one quad per task, shortest tasks)
  const uint64_t resident = (uint64_t)accumulate_grid<F>(dev, sms) * 128;
  const bool latency_mode = rounds_req == 0 && ((uint64_t)nb + (uint64_t)n * W / kMinTask + 1) * 4 <= resident;
  // Automatic tile: about one task per resident thread, so a mid-size MSM (too many tasks for
  // the latency form, too few to fill the GPU at 64 entries a task) still keeps every thread
  // busy; 64 entries at most, or 96 where buckets average 48 or more (a GLV-split 2^20 MSM
  // averages 64: tiles of 64 split half its buckets and the partial sums cost a combine pass;
  // 2^20 5.16 -> 5.07 ms, 2^22 17.8 -> 17.3 ms); the latency form the shortest.
  const uint64_t ne = (uint64_t)n * W;
  const uint32_t tmin = cfg.min_task > 0 ? (uint32_t)cfg.min_task : layout_min_task(ne);  // the layout's bound
  uint32_t task_len;
  if (cfg.task > 0) {
    task_len = (uint32_t)cfg.task;
  } else {
    const uint64_t room = resident > nb / 2 + 1024 ? resident - nb / 2 : resident / 2;  // split buckets
    task_len = (uint32_t)std::min<uint64_t>(64, (ne + room - 1) / room);
    if (task_len == 64 && ne >= 48ull * nb) task_len = 96;
  }
  if (latency_mode) task_len = ne <= kSmallEntries ? kLatMinTask : kMinTask;
  task_len = std::max(task_len, tmin);  // the workspace is sized for tasks of at least tmin entries
  if (task_len > (uint32_t)kMaxTask) task_len = kMaxTask;
  const Layout L = make_layout(n_in, c, XB, cfg.min_task > 0 ? (uint32_t)cfg.min_task : 0u, FIXED,
                               layout_affine(EC2, cfg.affine, n_in, c, FIXED, glv), glv);
  if (work_bytes < L.total || d_work == nullptr) return cudaErrorInvalidValue;
  char* base = static_cast<char*>(d_work);
  uint32_t* counters = reinterpret_cast<uint32_t*>(base + L.counters);
  uint32_t* counts = reinterpret_cast<uint32_t*>(base + L.counts);
  uint32_t* offsets = reinterpret_cast<uint32_t*>(base + L.offsets);
  uint32_t* entries = reinterpret_cast<uint32_t*>(base + L.entries);
  Task* tasks = reinterpret_cast<Task*>(base + L.tasks);
  Multi* multi = reinterpret_cast<Multi*>(base + L.multi);
  uint32_t* partials = reinterpret_cast<uint32_t*>(base + L.partials);
  uint32_t* buckets = cfg.bucket_out ? cfg.bucket_out : reinterpret_cast<uint32_t*>(base + L.buckets);
  uint32_t* lv_y = reinterpret_cast<uint32_t*>(base + L.lv_y);
  uint32_t* lv_z = reinterpret_cast<uint32_t*>(base + L.lv_z);
  uint32_t* lv_y2 = reinterpret_cast<uint32_t*>(base + L.lv_y2);
  uint32_t* lv_z2 = reinterpret_cast<uint32_t*>(base + L.lv_z2);
  uint32_t* wsum = reinterpret_cast<uint32_t*>(base + L.wsum);
  void* scan_tmp = base + (L.total - scan_workspace_bytes(nb + 1));

  cudaError_t e;
  const int T = 256;
  uint32_t* glv_s = glv ? reinterpret_cast<uint32_t*>(base + L.glv_s) : nullptr;
  const uint32_t* phix = glv ? reinterpret_cast<uint32_t*>(base + L.glv_p) : nullptr;
  if constexpr (!EC2 && !FIXED) {
    if (glv) {
      k_glv_prep<F><<<(n_in + T - 1) / T, T, 0, st>>>(d_scalars, d_points, n_in, glv_s, const_cast<uint32_t*>(phix));
      note_launch();
    }
  }
  if ((e = cudaMemsetAsync(counters, 0, kCtrWords * sizeof(uint32_t), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(counts, 0, (nb + 1) * sizeof(uint32_t), st)) != cudaSuccess) return e;
  if (glv)
    k_count_glv<F><<<(n_in + T - 1) / T, T, 0, st>>>(glv_s, n_in, c, W, counts);
  else
    k_count<F, FIXED><<<(n + T - 1) / T, T, 0, st>>>(d_scalars, d_points, n, c, W, counts);
  note_launch();
  if ((e = scan_exclusive_u32(counts, offsets, nb + 1, scan_tmp, st)) != cudaSuccess) return e;
  // counts is reused as the scatter cursor
  if ((e = cudaMemcpyAsync(counts, offsets, nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
    return e;
  if (glv)
    k_scatter_glv<F><<<(n_in + T - 1) / T, T, 0, st>>>(glv_s, n_in, c, W, counts, entries);
  else
    k_scatter<F, FIXED><<<(n + T - 1) / T, T, 0, st>>>(d_scalars, d_points, n, c, W, counts, entries);
  note_launch();
  // batch-affine halving rounds (counts is free again and holds the halved counts)
  const uint32_t* acc_entries = entries;
  const uint32_t* acc_points = d_points;
  uint32_t* acc_off = offsets;
  const int rounds = L.affine ? std::min(rounds_req, 6) : 0;
  if (rounds > 0) {
    uint32_t* off_in = offsets;
    uint32_t* off_out = reinterpret_cast<uint32_t*>(base + L.off2);
    uint32_t* pa = reinterpret_cast<uint32_t*>(base + L.pa);
    uint32_t* pb = reinterpret_cast<uint32_t*>(base + L.pb);
    uint32_t* pref = reinterpret_cast<uint32_t*>(base + L.pref);
    const uint32_t* src = d_points;
    uint32_t* dst = pa;
    size_t max_slots = (size_t)n * W / 2 + 2 * (size_t)nb + 1;
    for (int r = 0; r < rounds; r++) {
      k_half_counts<<<(nb + 1 + T - 1) / T, T, 0, st>>>(off_in, nb, counts);
      if ((e = scan_exclusive_u32(counts, off_out, nb + 1, scan_tmp, st)) != cudaSuccess) return e;
      const size_t threads = (max_slots + kAffK - 1) / kAffK;
      const unsigned blocks = (unsigned)((threads + 127) / 128);
      if (r == 0)
        k_affine_round<F, true><<<blocks, 128, 0, st>>>(off_in, off_out, nb, entries, d_points, dst, pref);
      else
        k_affine_round<F, false><<<blocks, 128, 0, st>>>(off_in, off_out, nb, nullptr, src, dst, pref);
      note_launch(2);
      src = dst;
      dst = dst == pa ? pb : pa;
      uint32_t* t = off_in; off_in = off_out; off_out = t;
      max_slots = max_slots / 2 + 2 * (size_t)nb + 1;
    }
    acc_entries = nullptr;
    acc_points = src;
    acc_off = off_in;
  }
  k_task_hist<F><<<(nb + T - 1) / T, T, 0, st>>>(acc_off, nb, task_len, counters + kCtrHist, buckets);
  note_launch();
  k_task_bins<<<1, 32, 0, st>>>(counters + kCtrHist, task_len, counters + kCtrCursor, counters);
  note_launch();
  k_task_emit<F><<<(nb + T - 1) / T, T, 0, st>>>(acc_off, nb, task_len, counters + kCtrCursor, tasks,
                                                  counters, multi);
  note_launch();
  if (cfg.acc_start) cudaEventRecord(cfg.acc_start, st);
  if (latency_mode)
    k_accumulate_quad<F><<<accumulate_grid<F>(dev, sms), 128, 0, st>>>(tasks, counters, acc_entries, acc_points, nb,
                                                                  buckets, partials, nullptr, phix);
  else
    k_accumulate<F><<<accumulate_grid<F>(dev, sms), 128, 0, st>>>(tasks, counters, acc_entries, acc_points, nb,
                                                             buckets, partials, nullptr, phix);
  note_launch();
  k_combine_small<F><<<sms * 4, 128, 0, st>>>(multi, counters, partials, buckets);
  k_combine<F><<<sms * 4, 128, 0, st>>>(multi, counters, partials, buckets);
  note_launch(2);
  if (cfg.acc_stop) cudaEventRecord(cfg.acc_stop, st);
  const int WR = FIXED ? 1 : W;
  const uint32_t B = 1u << (c - 1);
  if (cfg.bucket_out) {  // buckets handed on: this MSM's own result is the point at infinity
    k_store_inf<F><<<1, 32, 0, st>>>(d_out);
    note_launch();
    return cudaGetLastError();
  }
  if (cfg.bucket_add) {
    if (cfg.bucket_ready) cudaStreamWaitEvent(st, cfg.bucket_ready, 0);
    k_add_buckets<F><<<(B + 127) / 128, 128, 0, st>>>(buckets, cfg.bucket_add, B);
    note_launch();
  }
  // level 0: segments of 8 buckets -> totals y and in-segment weighted sums z
  uint32_t nseg = (B + 7) / 8;
  reduce_level<F>(buckets, nullptr, B, nseg, WR, 0, lv_y, lv_z, resident, st);
  int levels = 1;
  uint32_t *y = lv_y, *z = lv_z, *y2 = lv_y2, *z2 = lv_z2;
  // more levels until the top block's chain is short
  while (nseg > kTopSegments) {
    const uint32_t nnext = (nseg + 7) / 8;
    reduce_level<F>(y, z, nseg, nnext, WR, levels, y2, z2, resident, st);
    uint32_t* ty = y; y = y2; y2 = ty;
    uint32_t* tz = z; z = z2; z2 = tz;
    nseg = nnext;
    levels++;
  }
  constexpr int WT = WsumThreads<F>::single;
  k_window_sum<F, WT><<<WR, WT, 0, st>>>(y, z, nseg, 3 * levels, wsum);
  note_launch();
  k_finish<F><<<1, 32, 0, st>>>(wsum, WR, c, d_out);
  note_launch();
  return cudaGetLastError();
}

// Fixed-base tables.  table[0..n) = points; table[j n + i] = 2^c table[(j-1) n + i],
// computed in XYZZ and brought back to affine with one inversion per run of kAffRun
// points (Montgomery's simultaneous inversion).  Points at infinity stay infinity.
constexpr int kAffRun = 16;

template <class F>
__global__ void __launch_bounds__(128) k_table_double(const uint32_t* __restrict__ src, uint32_t n, int c,
                                                      uint32_t* __restrict__ xyzz) {
  constexpr int XW = 4 * FieldWords<F>::value;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Affine<F> p = ld_affine<F>(src + (size_t)i * 2 * FieldWords<F>::value);
  XYZZ<F> r = XYZZ<F>::inf();
  if (!affine_is_inf(p)) {
    r = xyzz_mdbl(p);
#pragma unroll 1
    for (int d = 1; d < c; d++) r = xyzz_dbl(r);
  }
  st_xyzz<F>(xyzz + (size_t)i * XW, r);
}

// Thread t converts points [t R, t R + R): prefix products of ZZ*ZZZ, one inverse, and
// the back substitution; `pref` holds the prefix products (n field elements).
template <class F>
__global__ void __launch_bounds__(128) k_batch_affine(const uint32_t* __restrict__ xyzz, uint32_t n,
                                                      uint32_t* __restrict__ pref, uint32_t* __restrict__ dst) {
  constexpr int FW = FieldWords<F>::value;
  constexpr int XW = 4 * FW;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lo = t * kAffRun;
  if (lo >= n) return;
  const uint32_t hi = min(n, lo + kAffRun);
  F acc = F::one();
  for (uint32_t i = lo; i < hi; i++) {
    const XYZZ<F> p = ld_xyzz<F>(xyzz + (size_t)i * XW);
    if (!p.is_inf()) acc = acc * (p.ZZ * p.ZZZ);
    st_field(pref + (size_t)i * FW, acc);
  }
  F inv = acc.inv();
  for (uint32_t i = hi; i-- > lo;) {
    const XYZZ<F> p = ld_xyzz<F>(xyzz + (size_t)i * XW);
    uint32_t* o = dst + (size_t)i * 2 * FW;
    if (p.is_inf()) {
      st_affine<F>(o, Affine<F>{F::zero(), F::one()});
      continue;
    }
    F before = F::one();
    if (i > lo) {  // written above by this thread: a plain (coherent) load, not __ldg
      uint32_t* bw = reinterpret_cast<uint32_t*>(&before);
      const uint4* src = reinterpret_cast<const uint4*>(pref + (size_t)(i - 1) * FW);
#pragma unroll
      for (int q = 0; q < FW / 4; q++) {
        const uint4 v = src[q];
        bw[4 * q] = v.x; bw[4 * q + 1] = v.y; bw[4 * q + 2] = v.z; bw[4 * q + 3] = v.w;
      }
    }
    const F ip = inv * before;          // 1 / (ZZ ZZZ)
    inv = inv * (p.ZZ * p.ZZZ);
    st_affine<F>(o, Affine<F>{p.X * (p.ZZZ * ip), p.Y * (p.ZZ * ip)});
  }
}

inline size_t fixed_table_work_bytes(uint32_t n, int xyzz_bytes, int field_bytes) {
  return align256((size_t)n * xyzz_bytes) + align256((size_t)n * field_bytes);
}

template <class F>
cudaError_t fixed_table_impl(const uint32_t* d_points, uint32_t n, int c, uint32_t* d_table, void* d_work,
                             size_t work_bytes, cudaStream_t st) {
  constexpr int FW = FieldWords<F>::value;
  constexpr int XB = 16 * FW, PB = 8 * FW;
  if (c < 4 || c > 24) return cudaErrorInvalidValue;
  if (n == 0) return cudaSuccess;
  if (!d_work || work_bytes < fixed_table_work_bytes(n, XB, 4 * FW)) return cudaErrorInvalidValue;
  uint32_t* xyzz = static_cast<uint32_t*>(d_work);
  uint32_t* pref = reinterpret_cast<uint32_t*>(static_cast<char*>(d_work) + align256((size_t)n * XB));
  const int W = num_windows(c);
  cudaError_t e = cudaMemcpyAsync(d_table, d_points, (size_t)n * PB, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return e;
  const uint32_t runs = (n + kAffRun - 1) / kAffRun;
  for (int j = 1; j < W; j++) {
    const uint32_t* src = d_table + (size_t)(j - 1) * n * 2 * FW;
    uint32_t* dst = d_table + (size_t)j * n * 2 * FW;
    k_table_double<F><<<(n + 127) / 128, 128, 0, st>>>(src, n, c, xyzz);
    k_batch_affine<F><<<(runs + 127) / 128, 128, 0, st>>>(xyzz, n, pref, dst);
    note_launch(2);
  }
  return cudaGetLastError();
}

}  // namespace msm_detail
}  // namespace csb
