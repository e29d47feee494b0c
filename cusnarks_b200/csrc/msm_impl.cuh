// msm_impl.cuh -- kernels and launch sequence of the Pippenger MSM (pipeline in msm.cuh),
// instantiated for G1 in msm_g1.cu and for G2 in msm_g2.cu.
#pragma once
#include "msm.cuh"
#include "curve.cuh"
#include "scan.cuh"

namespace csb {
namespace msm_detail {

constexpr int SCALAR_BITS = 254;  // scalars are reduced below r < 2^254 first
constexpr uint32_t NEG_BIT = 0x80000000u;
constexpr uint32_t kMinTask = 32;  // workspace bounds assume tasks of at least this size

__host__ __device__ inline int num_windows(int c) { return SCALAR_BITS / c + 1; }

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

template <class F>
__global__ void k_count(const uint32_t* __restrict__ scalars, const uint32_t* __restrict__ points,
                        uint32_t n, int c, int W, uint32_t* __restrict__ counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k[8];
  if (!load_scalar<F>(scalars, points, i, k)) return;
  const uint32_t B = 1u << (c - 1);
  for_each_digit(k, c, W, [&](int j, uint32_t mag, bool) {
    atomicAdd(&counts[(size_t)j * B + (mag - 1)], 1u);
  });
}

template <class F>
__global__ void k_scatter(const uint32_t* __restrict__ scalars, const uint32_t* __restrict__ points,
                          uint32_t n, int c, int W, uint32_t* __restrict__ cursor,
                          uint32_t* __restrict__ entries) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k[8];
  if (!load_scalar<F>(scalars, points, i, k)) return;
  const uint32_t B = 1u << (c - 1);
  for_each_digit(k, c, W, [&](int j, uint32_t mag, bool neg) {
    const uint32_t pos = atomicAdd(&cursor[(size_t)j * B + (mag - 1)], 1u);
    entries[pos] = i | (neg ? NEG_BIT : 0u);
  });
}

// Task record: entries [start, start+len) summed into dst.  dst < nb: bucket index;
// dst >= nb: partial slot (dst - nb).
struct Task {
  uint32_t start, len, dst, pad;
};
struct Multi {
  uint32_t bucket, pbase, count, pad;
};

// One thread per bucket: emit its tasks; empty buckets are set to infinity here.
template <class F>
__global__ void k_tasks(const uint32_t* __restrict__ offsets, uint32_t nb, uint32_t task_len,
                        Task* __restrict__ tasks, uint32_t* __restrict__ counters,
                        Multi* __restrict__ multi, uint32_t* __restrict__ buckets) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  uint32_t start = 0, cnt = 0, nt = 0;
  if (b < nb) {
    start = offsets[b];
    cnt = offsets[b + 1] - start;
    nt = (cnt + task_len - 1) / task_len;
  }
  // warp-aggregated slot allocation for tasks
  uint32_t incl = nt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= (uint32_t)d) incl += v;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  uint32_t base = 0;
  if (lane == 31 && total) base = atomicAdd(&counters[0], total);
  base = __shfl_sync(0xffffffffu, base, 31);
  if (b >= nb) return;
  uint32_t slot = base + incl - nt;
  if (nt == 0) {
    constexpr int PW = 4 * FieldWords<F>::value;
    st_xyzz<F>(buckets + (size_t)b * PW, XYZZ<F>::inf());
    return;
  }
  if (nt == 1) {
    tasks[slot] = {start, cnt, b, 0u};
    return;
  }
  const uint32_t pbase = atomicAdd(&counters[1], nt);
  const uint32_t mslot = atomicAdd(&counters[2], 1u);
  multi[mslot] = {b, pbase, nt, 0u};
  for (uint32_t t = 0; t < nt; t++) {
    const uint32_t s = start + t * task_len;
    const uint32_t l = min(task_len, cnt - t * task_len);
    tasks[slot + t] = {s, l, nb + pbase + t, 0u};
  }
}

template <class F>
__global__ void __launch_bounds__(128) k_accumulate(const Task* __restrict__ tasks,
                                                    const uint32_t* __restrict__ counters,
                                                    const uint32_t* __restrict__ entries,
                                                    const uint32_t* __restrict__ points, uint32_t nb,
                                                    uint32_t* __restrict__ buckets,
                                                    uint32_t* __restrict__ partials) {
  constexpr int PW = 2 * FieldWords<F>::value;
  constexpr int XW = 4 * FieldWords<F>::value;
  const uint32_t ntasks = counters[0];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += gridDim.x * blockDim.x) {
    const Task tk = tasks[t];
    XYZZ<F> acc = XYZZ<F>::inf();
#pragma unroll 1
    for (uint32_t e = 0; e < tk.len; e++) {
      const uint32_t ent = entries[tk.start + e];
      Affine<F> p = ld_affine<F>(points + (size_t)(ent & ~NEG_BIT) * PW);
      if (ent & NEG_BIT) p.y = p.y.neg();
      acc = xyzz_madd(acc, p);
    }
    uint32_t* dst = tk.dst < nb ? buckets + (size_t)tk.dst * XW : partials + (size_t)(tk.dst - nb) * XW;
    st_xyzz<F>(dst, acc);
  }
}

// One block per split bucket: tree-sum its partials.
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
    XYZZ<F> acc = XYZZ<F>::inf();
#pragma unroll 1
    for (uint32_t i = threadIdx.x; i < mu.count; i += blockDim.x)
      acc = xyzz_add(acc, ld_xyzz<F>(partials + (size_t)(mu.pbase + i) * XW));
    // warp tree
#pragma unroll 1
    for (int d = 16; d > 0; d >>= 1) {
      XYZZ<F> o;
      uint32_t* ow = reinterpret_cast<uint32_t*>(&o);
      const uint32_t* aw = reinterpret_cast<const uint32_t*>(&acc);
#pragma unroll
      for (int w = 0; w < XW; w++) ow[w] = __shfl_down_sync(0xffffffffu, aw[w], d);
      acc = xyzz_add(acc, o);
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
        s = xyzz_add(s, o);
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

// Window sums S_j = y_j + z_j, then sum_j 2^(c j) S_j and the affine result.
template <class F>
__global__ void k_finish(const uint32_t* __restrict__ y, const uint32_t* __restrict__ z, int W,
                         int c, uint32_t* __restrict__ out) {
  constexpr int XW = 4 * FieldWords<F>::value;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  XYZZ<F> r = XYZZ<F>::inf();
#pragma unroll 1
  for (int j = W - 1; j >= 0; j--) {
#pragma unroll 1
    for (int d = 0; d < c && j != W - 1; d++) r = xyzz_dbl(r);
    r = xyzz_add(r, ld_xyzz<F>(y + (size_t)j * XW));
    r = xyzz_add(r, ld_xyzz<F>(z + (size_t)j * XW));
  }
  st_affine<F>(out, xyzz_to_affine(r));
}

template <class F>
__global__ void k_store_inf(uint32_t* out) {
  if (threadIdx.x == 0) st_affine<F>(out, Affine<F>{F::zero(), F::one()});
}

// --------------------------------------------------------------- workspace layout ----
struct Layout {
  size_t counts, offsets, entries, tasks, multi, partials, buckets, lv_a, lv_b, counters, total;
};

static inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

inline Layout make_layout(uint32_t n, int c, int xyzz_bytes, uint32_t task_len) {
  const int W = num_windows(c);
  const size_t nb = (size_t)W << (c - 1);
  const size_t ne = (size_t)n * W;
  const size_t max_tasks = nb + ne / task_len + 1;
  const size_t max_partials = 2 * (ne / task_len) + 1;
  Layout L{};
  size_t o = 0;
  L.counters = o; o = align256(o + 4 * sizeof(uint32_t));
  L.counts = o;   o = align256(o + (nb + 1) * sizeof(uint32_t));
  L.offsets = o;  o = align256(o + (nb + 1) * sizeof(uint32_t));
  L.entries = o;  o = align256(o + ne * sizeof(uint32_t));
  L.tasks = o;    o = align256(o + max_tasks * sizeof(Task));
  L.multi = o;    o = align256(o + (ne / (task_len + 1) + 1) * sizeof(Multi));
  L.partials = o; o = align256(o + max_partials * (size_t)xyzz_bytes);
  L.buckets = o;  o = align256(o + nb * (size_t)xyzz_bytes);
  const size_t lv = ((nb / 8) + W) * (size_t)xyzz_bytes;
  L.lv_a = o;     o = align256(o + 2 * lv);
  L.lv_b = o;     o = align256(o + 2 * lv);
  L.total = o + scan_workspace_bytes(nb + 1);
  return L;
}

template <class F>
cudaError_t msm_impl(const uint32_t* d_scalars, const uint32_t* d_points, uint32_t n,
                     uint32_t* d_out, void* d_work, size_t work_bytes, const MsmConfig& cfg,
                     cudaStream_t st) {
  constexpr bool EC2 = FieldWords<F>::value == 16;
  constexpr int XB = 4 * FieldWords<F>::value * 4;  // bytes per XYZZ point
  if (n == 0) {
    k_store_inf<F><<<1, 32, 0, st>>>(d_out);
    return cudaGetLastError();
  }
  const int c = cfg.c > 0 ? cfg.c : msm_default_window(n, EC2);
  if (c < 4 || c > 24) return cudaErrorInvalidValue;
  const uint32_t task_len = cfg.task >= (int)kMinTask ? (uint32_t)cfg.task : 64u;
  const int W = num_windows(c);
  const uint32_t nb = (uint32_t)W << (c - 1);
  const Layout L = make_layout(n, c, XB, kMinTask);
  if (work_bytes < L.total || d_work == nullptr) return cudaErrorInvalidValue;
  char* base = static_cast<char*>(d_work);
  uint32_t* counters = reinterpret_cast<uint32_t*>(base + L.counters);
  uint32_t* counts = reinterpret_cast<uint32_t*>(base + L.counts);
  uint32_t* offsets = reinterpret_cast<uint32_t*>(base + L.offsets);
  uint32_t* entries = reinterpret_cast<uint32_t*>(base + L.entries);
  Task* tasks = reinterpret_cast<Task*>(base + L.tasks);
  Multi* multi = reinterpret_cast<Multi*>(base + L.multi);
  uint32_t* partials = reinterpret_cast<uint32_t*>(base + L.partials);
  uint32_t* buckets = reinterpret_cast<uint32_t*>(base + L.buckets);
  uint32_t* lva = reinterpret_cast<uint32_t*>(base + L.lv_a);
  uint32_t* lvb = reinterpret_cast<uint32_t*>(base + L.lv_b);
  void* scan_tmp = base + (L.total - scan_workspace_bytes(nb + 1));

  cudaError_t e;
  if ((e = cudaMemsetAsync(counters, 0, 4 * sizeof(uint32_t), st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(counts, 0, (nb + 1) * sizeof(uint32_t), st)) != cudaSuccess) return e;
  const int T = 256;
  k_count<F><<<(n + T - 1) / T, T, 0, st>>>(d_scalars, d_points, n, c, W, counts);
  if ((e = scan_exclusive_u32(counts, offsets, nb + 1, scan_tmp, st)) != cudaSuccess) return e;
  // counts is reused as the scatter cursor
  if ((e = cudaMemcpyAsync(counts, offsets, nb * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
    return e;
  k_scatter<F><<<(n + T - 1) / T, T, 0, st>>>(d_scalars, d_points, n, c, W, counts, entries);
  k_tasks<F><<<(nb + T - 1) / T, T, 0, st>>>(offsets, nb, task_len, tasks, counters, multi, buckets);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_accumulate<F><<<sms * 8, 128, 0, st>>>(tasks, counters, entries, d_points, nb, buckets, partials);
  k_combine<F><<<sms * 4, 128, 0, st>>>(multi, counters, partials, buckets);
  // hierarchical bucket reduction
  const uint32_t* y = buckets;
  const uint32_t* z = nullptr;
  uint32_t len = 1u << (c - 1);
  uint32_t* bufs[2][2] = {{lva, lva + ((size_t)(nb / 8) + W) * (XB / 4)},
                          {lvb, lvb + ((size_t)(nb / 8) + W) * (XB / 4)}};
  int level = 0, pp = 0;
  while (len > 1) {
    const uint32_t nout = (len + 7) / 8;
    uint32_t* yo = bufs[pp][0];
    uint32_t* zo = bufs[pp][1];
    const uint32_t threads = (uint32_t)W * nout;
    k_reduce_level<F><<<(threads + 127) / 128, 128, 0, st>>>(y, z, len, nout, W, level, yo, zo);
    y = yo; z = zo; len = nout; level++; pp ^= 1;
  }
  if (z == nullptr) {
    // c == 1 is excluded above, so at least one level always runs
    return cudaErrorInvalidValue;
  }
  k_finish<F><<<1, 32, 0, st>>>(y, z, W, c, d_out);
  return cudaGetLastError();
}

}  // namespace msm_detail
}  // namespace csb
