// ntt.cu -- radix-2 NTT passes in shared memory and Fr elementwise helpers (ntt.cuh).
#include "ntt.cuh"
#include "curve.cuh"
#include "runtime.cuh"

namespace csb {

namespace {

constexpr int kMaxStages = 11;  // 2^11 elements x 32 B = 64 KB of shared memory per block
constexpr int kThreads = 256;

CSB_DEV void lds_fr(Fr& x, const uint4* s, uint32_t i) {
  const uint4 a = s[2 * i], b = s[2 * i + 1];
  x.v[0] = a.x; x.v[1] = a.y; x.v[2] = a.z; x.v[3] = a.w;
  x.v[4] = b.x; x.v[5] = b.y; x.v[6] = b.z; x.v[7] = b.w;
}
CSB_DEV void sts_fr(uint4* s, uint32_t i, const Fr& x) {
  s[2 * i] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
  s[2 * i + 1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

// One pass: stages s0 .. s0+S-1 of a radix-2 DIT transform of 2^L points.  Block q owns
// the 2^S elements base + (i << s0), base = ((q >> s0) << (s0 + S)) + (q & (2^s0 - 1)).
// blockIdx.y: the instance of a batch, its arrays `stride` words after the previous one's.
__global__ void __launch_bounds__(kThreads) k_ntt_pass(
    const uint32_t* __restrict__ in, const uint32_t* __restrict__ in_odd, uint32_t* out,
    uint32_t L, uint32_t s0, uint32_t S, int bitrev, const uint32_t* __restrict__ W,
    uint32_t wshift, const uint32_t* __restrict__ post_tab, const uint32_t* __restrict__ post_scalar,
    size_t stride) {
  extern __shared__ uint4 sm[];
  const size_t inst = (size_t)blockIdx.y * stride;
  in += inst;
  if (in_odd) in_odd += inst;
  out += inst;
  const uint32_t q = blockIdx.x;
  const uint32_t rmask = (1u << s0) - 1u;
  const uint64_t base = ((uint64_t)(q >> s0) << (s0 + S)) + (q & rmask);
  const uint32_t cnt = 1u << S;
  for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
    const uint64_t g = base + ((uint64_t)i << s0);
    uint64_t src = g;
    if (bitrev) src = __brev((uint32_t)g) >> (32 - L);
    const uint32_t* p = in_odd ? ((src & 1) ? in_odd : in) + (src >> 1) * 8 : in + src * 8;
    Fr x = ld_fp<ModR>(p);
    sts_fr(sm, i, x);
  }
  __syncthreads();
  const uint32_t r = q & rmask;
  for (uint32_t t = 0; t < S; t++) {
    const uint32_t s = s0 + t;
    const uint32_t tmask = (1u << t) - 1u;
    const uint32_t tw_shift = L - s - 1 + wshift;
    for (uint32_t b = threadIdx.x; b < cnt / 2; b += blockDim.x) {
      const uint32_t lo = ((b >> t) << (t + 1)) | (b & tmask);
      const uint32_t hi = lo + (1u << t);
      const uint64_t k = (uint64_t)r + ((uint64_t)(lo & tmask) << s0);
      Fr x, y;
      lds_fr(x, sm, lo);
      lds_fr(y, sm, hi);
      if (k != 0) y = y * ld_fp<ModR>(W + (k << tw_shift) * 8);
      sts_fr(sm, lo, x + y);
      sts_fr(sm, hi, x - y);
    }
    __syncthreads();
  }
  Fr sc;
  if (post_scalar) sc = ld_fp<ModR>(post_scalar);
  for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
    const uint64_t g = base + ((uint64_t)i << s0);
    Fr x;
    lds_fr(x, sm, i);
    if (post_scalar) x = x * sc;
    if (post_tab) x = x * ld_fp<ModR>(post_tab + g * 8);
    st_fp<ModR>(out + g * 8, x);
  }
}

// W[j] = root^j: each thread raises root to its first index, then steps.
__global__ void k_powers(uint32_t* __restrict__ out, const uint32_t* __restrict__ root, uint32_t count,
                         uint32_t per_thread) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t first = (uint64_t)t * per_thread;
  if (first >= count) return;
  const Fr w = ld_fp<ModR>(root);
  Fr acc = Fr::one(), base = w;
  uint64_t e = first;
  while (e) {
    if (e & 1) acc = acc * base;
    base = base.sqr();
    e >>= 1;
  }
  for (uint32_t j = 0; j < per_thread && first + j < count; j++) {
    st_fp<ModR>(out + (first + j) * 8, acc);
    acc = acc * w;
  }
}

__global__ void k_gather_roots(uint32_t* __restrict__ out, const uint32_t* __restrict__ table,
                               uint64_t stride, uint32_t n, int dir, uint32_t count) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const uint64_t idx = dir > 0 ? j : (uint64_t)((n - j) & (n - 1));
  const uint64_t src = (stride * idx) & (stride * (uint64_t)n - 1);
  const uint4* s = reinterpret_cast<const uint4*>(table + src * 8);
  uint4* d = reinterpret_cast<uint4*>(out + (uint64_t)j * 8);
  d[0] = s[0];
  d[1] = s[1];
}

__global__ void k_fr_mul(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                         uint32_t* __restrict__ out, uint32_t n, size_t stride) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t o = (size_t)blockIdx.y * stride + (size_t)i * 8;
  st_fp<ModR>(out + o, ld_fp<ModR>(a + o) * ld_fp<ModR>(b + o));
}

__global__ void k_fr_mul_sub_scale(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                                   const uint32_t* __restrict__ c, const uint32_t* __restrict__ s,
                                   uint32_t* __restrict__ out, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Fr v = ld_fp<ModR>(a + (size_t)i * 8) * ld_fp<ModR>(b + (size_t)i * 8) - ld_fp<ModR>(c + (size_t)i * 8);
  st_fp<ModR>(out + (size_t)i * 8, v * ld_fp<ModR>(s));
}

void plan_passes(uint32_t L, uint32_t* sizes, int* np) {
  const int n = (int)((L + kMaxStages - 1) / kMaxStages);
  int k = 0;
  uint32_t left = L;
  for (int p = 0; p < n; p++) {
    const uint32_t sz = (left + (n - p) - 1) / (n - p);  // even split, larger first
    sizes[k++] = sz;
    left -= sz;
  }
  *np = k;
}

}  // namespace

cudaError_t ntt_run(const NttArgs& a, cudaStream_t st) {
  const uint32_t L = a.log_n;
  if (L == 0 || L > 28 || a.log_tab < L || !a.W || !a.in || !a.out || a.batch == 0 || a.batch > 65535)
    return cudaErrorInvalidValue;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_ntt_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (1 << kMaxStages) * 32);
    attr_set = true;
  }
  uint32_t sizes[8];
  int np = 0;
  plan_passes(L, sizes, &np);
  const bool alias = (a.in == a.out) || (a.in_odd == a.out);
  uint32_t* work = a.out;
  if (alias && np > 1) {
    if (!a.tmp) return cudaErrorInvalidValue;
    work = a.tmp;
  }
  uint32_t s0 = 0;
  for (int p = 0; p < np; p++) {
    const uint32_t S = sizes[p];
    const bool first = (p == 0), last = (p == np - 1);
    const uint32_t* src = first ? a.in : work;
    const uint32_t* src_odd = first ? a.in_odd : nullptr;
    uint32_t* dst = last ? a.out : work;
    const unsigned blocks = 1u << (L - S);
    const unsigned threads = (1u << (S - 1)) < (unsigned)kThreads ? (1u << (S - 1)) : (unsigned)kThreads;
    k_ntt_pass<<<dim3(blocks, a.batch), threads > 0 ? threads : 1, (1u << S) * 32, st>>>(
        src, src_odd, dst, L, s0, S, first ? 1 : 0, a.W, a.log_tab - L,
        last ? a.post_tab : nullptr, last ? a.post_scalar : nullptr, a.stride);
    note_launch();
    s0 += S;
  }
  return cudaGetLastError();
}

cudaError_t ntt_powers(uint32_t* d_out, const uint32_t* d_root, uint32_t count, cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  const uint32_t per = 64;
  const uint32_t threads = (count + per - 1) / per;
  k_powers<<<(threads + 127) / 128, 128, 0, st>>>(d_out, d_root, count, per);
  note_launch();
  return cudaGetLastError();
}

cudaError_t ntt_gather_roots(uint32_t* d_out, const uint32_t* d_table, uint64_t stride, uint32_t n,
                             int dir, uint32_t count, cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  k_gather_roots<<<(count + 255) / 256, 256, 0, st>>>(d_out, d_table, stride, n, dir, count);
  note_launch();
  return cudaGetLastError();
}

cudaError_t fr_mul(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n, cudaStream_t st) {
  return fr_mul_batch(a, b, out, n, 1, 0, st);
}

cudaError_t fr_mul_batch(const uint32_t* a, const uint32_t* b, uint32_t* out, uint32_t n, uint32_t batch,
                         size_t stride, cudaStream_t st) {
  if (n == 0 || batch == 0) return cudaSuccess;
  if (batch > 65535) return cudaErrorInvalidValue;
  k_fr_mul<<<dim3((n + 255) / 256, batch), 256, 0, st>>>(a, b, out, n, stride);
  note_launch();
  return cudaGetLastError();
}

cudaError_t fr_mul_tab(const uint32_t* a, const uint32_t* tab, uint32_t* out, uint32_t n, cudaStream_t st) {
  return fr_mul(a, tab, out, n, st);
}

cudaError_t fr_mul_sub_scale(const uint32_t* a, const uint32_t* b, const uint32_t* c, const uint32_t* s,
                             uint32_t* out, uint32_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_fr_mul_sub_scale<<<(n + 255) / 256, 256, 0, st>>>(a, b, c, s, out, n);
  note_launch();
  return cudaGetLastError();
}

}  // namespace csb
