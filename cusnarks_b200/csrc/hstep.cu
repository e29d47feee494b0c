// hstep.cu -- NTT / INTT / H-step entry points: the reference's host functions on this
// path (ntt_h, intt_h, find_roots_h, ntt_interpolandmul_server_h) and the context API with
// device pointers and HBM-resident twiddle tables.
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/cusnarks_b200.h"
#include "curve.cuh"
#include "ntt.cuh"
#include "runtime.cuh"

namespace csb {

// Primitive 2^28-th root of unity of Fr, 5^((r-1)/2^28), Montgomery form; the 2^k-th
// roots are its 2^(28-k)-th powers (the same chain as the reference's proots_field table,
// src/cuda/constants.cpp:323, which tabulates 5^((r-1)/2^k)).
__constant__ uint32_t c_w28[8] = {0x80d13d9cu, 0x636e7355u, 0x2445ffd6u, 0xa22bf374u,
                                  0x1eb203d8u, 0x56452ac0u, 0x2963f9e7u, 0x1860ef94u};
// Multiplicative generator g = 5 of Fr^*, Montgomery form (coset shift of the H step).
__constant__ uint32_t c_gen[8] = {0x9fffffe6u, 0x1b0d0ef9u, 0xa32a913fu, 0xeaba68a3u,
                                  0xd8dd0689u, 0x47d8eb76u, 0x20f5bbc3u, 0x15d00855u};

namespace {

constexpr int kMaxLog = 27;

// consts layout (Fr elements): 0 w_n, 1 w_n^-1, 2 n^-1 R (Montgomery), 3 n^-1 (normal),
// 4 (n/2)^-1 R, 5 g, 6 g^-1, 7 (g^(n/2) - 1)^-1, 8 (n/2)^-1 (normal)
__global__ void k_domain_consts(uint32_t L, uint32_t* out) {
  if (threadIdx.x != 0) return;
  Fr w;
  for (int i = 0; i < 8; i++) w.v[i] = c_w28[i];
  for (uint32_t k = L; k < 28; k++) w = w.sqr();
  st_fp<ModR>(out + 0, w);
  st_fp<ModR>(out + 8, w.inv());
  Fr nn = Fr::zero();
  nn.v[L >> 5] = 1u << (L & 31);
  const Fr ninv = nn.to_mont().inv();
  st_fp<ModR>(out + 16, ninv);
  st_fp<ModR>(out + 24, ninv.from_mont());
  Fr hh = Fr::zero();
  if (L >= 1) hh.v[(L - 1) >> 5] = 1u << ((L - 1) & 31);
  const Fr hinv = L >= 1 ? hh.to_mont().inv() : Fr::one();
  st_fp<ModR>(out + 32, hinv);
  Fr g;
  for (int i = 0; i < 8; i++) g.v[i] = c_gen[i];
  st_fp<ModR>(out + 40, g);
  st_fp<ModR>(out + 48, g.inv());
  Fr gm = g;
  for (uint32_t k = 1; k < L; k++) gm = gm.sqr();  // g^(n/2)
  st_fp<ModR>(out + 56, (gm - Fr::one()).inv());
  st_fp<ModR>(out + 64, hinv.from_mont());
}

// T[i] = s * g^-i as a normal-form value: a Montgomery product x*T[i] then yields
// x * s * g^-i in normal form (unshift, scale and leave Montgomery form at once).
__global__ void k_scaled_normal(const uint32_t* __restrict__ pw, const uint32_t* __restrict__ s,
                                uint32_t* __restrict__ out, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  st_fp<ModR>(out + (size_t)i * 8, (ld_fp<ModR>(pw + (size_t)i * 8) * ld_fp<ModR>(s)).from_mont());
}

}  // namespace

// Twiddle and coset tables for transforms of 2^L points, resident in HBM per context.
struct Domain {
  uint32_t L = 0;
  uint32_t* consts = nullptr;  // 9 elements (see k_domain_consts)
  uint32_t* Wf = nullptr;      // w^j, j < 2^(L-1)
  uint32_t* Wi = nullptr;      // w^-j
  uint32_t* G = nullptr;       // g^i, i < 2^(L-1)      (coset of the half-size domain)
  uint32_t* Tinv = nullptr;    // (2^(L-1))^-1 g^-i, normal form, i < 2^(L-1)
  ~Domain() {
    cudaFree(consts); cudaFree(Wf); cudaFree(Wi); cudaFree(G); cudaFree(Tinv);
  }
};

struct DomainCache {
  std::mutex mu;
  std::map<uint32_t, std::unique_ptr<Domain>> by_log;
};

static std::mutex g_dom_mu;
static std::map<cs_ctx*, std::unique_ptr<DomainCache>> g_dom;

void domain_release(cs_ctx* ctx) {
  std::lock_guard<std::mutex> lk(g_dom_mu);
  g_dom.erase(ctx);
}

// Tables for a 2^L-point domain (built once per context and size).
cudaError_t domain_get(cs_ctx* ctx, uint32_t L, Domain** out) {
  DomainCache* dc;
  {
    std::lock_guard<std::mutex> lk(g_dom_mu);
    auto& p = g_dom[ctx];
    if (!p) p.reset(new DomainCache());
    dc = p.get();
  }
  std::lock_guard<std::mutex> lk(dc->mu);
  auto it = dc->by_log.find(L);
  if (it != dc->by_log.end()) { *out = it->second.get(); return cudaSuccess; }
  if (L < 1 || L > kMaxLog) return cudaErrorInvalidValue;
  std::unique_ptr<Domain> d(new Domain());
  d->L = L;
  const size_t half = (size_t)1 << (L - 1);
  cudaError_t e;
  if ((e = cudaMalloc(&d->consts, 9 * 32)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&d->Wf, half * 32)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&d->Wi, half * 32)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&d->G, half * 32)) != cudaSuccess) return e;
  if ((e = cudaMalloc(&d->Tinv, half * 32)) != cudaSuccess) return e;
  cudaStream_t st = ctx->stream;
  k_domain_consts<<<1, 32, 0, st>>>(L, d->consts);
  note_launch();
  if ((e = ntt_powers(d->Wf, d->consts + 0, (uint32_t)half, st)) != cudaSuccess) return e;
  if ((e = ntt_powers(d->Wi, d->consts + 8, (uint32_t)half, st)) != cudaSuccess) return e;
  if ((e = ntt_powers(d->G, d->consts + 40, (uint32_t)half, st)) != cudaSuccess) return e;
  // Tinv[i] = (n/2)^-1 g^-i (normal form): powers of g^-1 into Tinv, then scale in place
  if ((e = ntt_powers(d->Tinv, d->consts + 48, (uint32_t)half, st)) != cudaSuccess) return e;
  k_scaled_normal<<<(unsigned)((half + 255) / 256), 256, 0, st>>>(d->Tinv, d->consts + 32, d->Tinv,
                                                                    (uint32_t)half);
  note_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  *out = d.get();
  dc->by_log[L] = std::move(d);
  return cudaSuccess;
}

const uint32_t* domain_wf(const Domain* d) { return d->Wf; }
const uint32_t* domain_wi(const Domain* d) { return d->Wi; }
const uint32_t* domain_consts(const Domain* d) { return d->consts; }

// ----------------------------------------------------------------- H step cores -----
// Reference semantics (src/cuda/ntt.cpp:778 interpol_and_mul_h): A, B evaluations on the
// m-th roots (Montgomery) -> the 2m coefficients of A(x)B(x) in normal form.
//   tabs: Wf2/Wi2 twiddles of the 2m-point domain, shift[i] (i < m) the odd-coset shift,
//   minv_R = m^-1 (Montgomery), m2inv = (2m)^-1 (normal form).
// Scratch: 4 m elements.  A and B are not modified.  batch instances: instance y's A, B,
// out and scratch lie y * stride words after instance 0's (the tables are shared).
cudaError_t hstep_reference_core(const uint32_t* A, const uint32_t* B, uint32_t L, const uint32_t* Wf2,
                                 const uint32_t* Wi2, const uint32_t* shift, const uint32_t* minv_R,
                                 const uint32_t* m2inv, uint32_t* out, uint32_t* scratch, cudaStream_t st,
                                 uint32_t batch = 1, size_t stride = 0) {
  const size_t m = (size_t)1 << L;
  uint32_t* E = scratch;
  uint32_t* O = scratch + m * 8;
  uint32_t* a = scratch + 2 * m * 8;
  uint32_t* b = scratch + 3 * m * 8;
  cudaError_t e;
  if ((e = fr_mul_batch(A, B, E, (uint32_t)m, batch, stride, st)) != cudaSuccess) return e;
  NttArgs t;
  t.batch = batch; t.stride = stride;
  t.log_n = L; t.log_tab = L + 1;
  // a = shift * INTT_m(A), b likewise
  t.in = A; t.out = a; t.W = Wi2; t.post_scalar = minv_R; t.post_tab = shift;
  if ((e = ntt_run(t, st)) != cudaSuccess) return e;
  t.in = B; t.out = b;
  if ((e = ntt_run(t, st)) != cudaSuccess) return e;
  // odd-coset evaluations, in place
  t.post_scalar = nullptr; t.post_tab = nullptr; t.W = Wf2;
  t.in = a; t.out = a; t.tmp = O;
  if ((e = ntt_run(t, st)) != cudaSuccess) return e;
  t.in = b; t.out = b; t.tmp = O;
  if ((e = ntt_run(t, st)) != cudaSuccess) return e;
  if ((e = fr_mul_batch(a, b, O, (uint32_t)m, batch, stride, st)) != cudaSuccess) return e;
  // 2m coefficients, normal form
  NttArgs u;
  u.batch = batch; u.stride = stride;
  u.log_n = L + 1; u.log_tab = L + 1;
  u.in = E; u.in_odd = O; u.out = out; u.W = Wi2; u.post_scalar = m2inv;
  return ntt_run(u, st);
}

// Coset variant: H (m coefficients, normal form) of (A B - C) / (x^m - 1) evaluated on
// g*<w>.  dom: the 2m-point domain (its G / Tinv cover m entries, w_m = Wf2 stride 2).
cudaError_t hstep_coset_core(const uint32_t* A, const uint32_t* B, const uint32_t* C, uint32_t L,
                             const Domain* dom, uint32_t* out, uint32_t* scratch, cudaStream_t st) {
  const size_t m = (size_t)1 << L;
  uint32_t* a = scratch;
  uint32_t* b = scratch + m * 8;
  uint32_t* c = scratch + 2 * m * 8;
  uint32_t* tmp = scratch + 3 * m * 8;
  const uint32_t* src[3] = {A, B, C};
  uint32_t* dst[3] = {a, b, c};
  cudaError_t e;
  for (int k = 0; k < 3; k++) {
    NttArgs t;
    t.log_n = L; t.log_tab = L + 1; t.W = dom->Wi;
    t.in = src[k]; t.out = dst[k]; t.post_scalar = dom->consts + 32; t.post_tab = dom->G;
    if ((e = ntt_run(t, st)) != cudaSuccess) return e;
    NttArgs f;
    f.log_n = L; f.log_tab = L + 1; f.W = dom->Wf;
    f.in = dst[k]; f.out = dst[k]; f.tmp = tmp;
    if ((e = ntt_run(f, st)) != cudaSuccess) return e;
  }
  if ((e = fr_mul_sub_scale(a, b, c, dom->consts + 56, a, (uint32_t)m, st)) != cudaSuccess) return e;
  NttArgs h;
  h.log_n = L; h.log_tab = L + 1; h.W = dom->Wi;
  h.in = a; h.out = out; h.tmp = tmp; h.post_tab = dom->Tinv;
  return ntt_run(h, st);
}

}  // namespace csb

using namespace csb;

namespace {

thread_local int t_ntt_status = CS_OK;
thread_local std::string t_ntt_error;

cs_ctx* ntt_default_ctx() {
  static std::mutex mu;
  static cs_ctx* ctxs[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { cudaGetLastError(); return nullptr; }
  std::lock_guard<std::mutex> lk(mu);
  if (!ctxs[dev] && cs_ctx_create(dev, &ctxs[dev]) != CS_OK) return nullptr;
  return ctxs[dev];
}

void set_status(int st, cs_ctx* ctx) {
  t_ntt_status = st;
  t_ntt_error = (st == CS_OK || !ctx) ? std::string() : ctx->err;
}

// Device layout helper for host-pointer calls: carve the ctx input arena.
struct Carve {
  char* p;
  explicit Carve(void* base) : p(static_cast<char*>(base)) {}
  uint32_t* take(size_t bytes) {
    uint32_t* r = reinterpret_cast<uint32_t*>(p);
    p += (bytes + 255) & ~size_t(255);
    return r;
  }
};

// Reference ntt_h / intt_h on host data.  scale_fmat < 0: no scaling (ntt_h).
int host_ntt(cs_ctx* ctx, uint32_t* A, const uint32_t* roots, uint32_t L, uint64_t astride,
             uint64_t rstride, int dir, int scale_fmat) {
  if (L == 0) return CS_OK;
  if (L > 27) return fail_msg(ctx, CS_ERR_ARG, "transform too large");
  const size_t n = (size_t)1 << L, half = n / 2;
  // twiddles for this direction, gathered from the caller's table exactly as the
  // reference indexes it: roots[(rstride * k) mod (rstride * n)], k = +-j
  std::vector<uint32_t> W(half * 8);
  for (size_t j = 0; j < half; j++) {
    const uint64_t idx = dir > 0 ? j : ((n - j) & (n - 1));
    const uint64_t src = (rstride * idx) & (rstride * (uint64_t)n - 1);
    std::memcpy(&W[j * 8], roots + src * 8, 32);
  }
  std::vector<uint32_t> hostA;
  const uint32_t* src_host = A;
  if (astride != 1) {
    hostA.resize(n * 8);
    for (size_t i = 0; i < n; i++) std::memcpy(&hostA[i * 8], A + astride * i * 8, 32);
    src_host = hostA.data();
  }
  const size_t bytes = n * 32;
  cudaError_t e = ctx->in.reserve(3 * ((bytes + 255) & ~size_t(255)) + half * 32 + 2048, ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "ntt buffers");
  Carve cv(ctx->in.ptr);
  uint32_t* dA = cv.take(bytes);
  uint32_t* dOut = cv.take(bytes);
  uint32_t* dW = cv.take(half * 32);
  uint32_t* dC = cv.take(9 * 32);
  if ((e = cudaMemcpyAsync(dA, src_host, bytes, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
    return fail(ctx, e, "ntt H2D");
  if (half && (e = cudaMemcpyAsync(dW, W.data(), half * 32, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
    return fail(ctx, e, "ntt H2D roots");
  NttArgs t;
  t.in = dA; t.out = dOut; t.log_n = L; t.log_tab = L; t.W = dW;
  if (scale_fmat >= 0) {
    k_domain_consts<<<1, 32, 0, ctx->stream>>>(L, dC);
    note_launch();
    t.post_scalar = dC + (scale_fmat ? 16 : 24);
  }
  if (L == 1) {
    // a 2-point transform needs W[0] = roots[0] only; handled by the same kernel
  }
  cudaEventRecord(ctx->ev_start, ctx->stream);
  if ((e = ntt_run(t, ctx->stream)) != cudaSuccess) return fail(ctx, e, "ntt launch");
  cudaEventRecord(ctx->ev_stop, ctx->stream);
  std::vector<uint32_t> outv;
  uint32_t* dst_host = A;
  if (astride != 1) { outv.resize(n * 8); dst_host = outv.data(); }
  if ((e = cudaMemcpyAsync(dst_host, dOut, bytes, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
    return fail(ctx, e, "ntt D2H");
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(ctx, e, "ntt sync");
  if (astride != 1)
    for (size_t i = 0; i < n; i++) std::memcpy(A + astride * i * 8, &outv[i * 8], 32);
  return CS_OK;
}

std::vector<uint32_t>& interp_result() {
  static std::vector<uint32_t> buf;
  return buf;
}
// the last H step's (Nrows, Ncols) and its result in the reference's pre-transpose layout
uint32_t g_interp_rows = 0, g_interp_cols = 0;
std::vector<uint32_t>& interp_mmul() {
  static std::vector<uint32_t> buf;
  return buf;
}

}  // namespace

extern "C" {

int cs_ntt_last_status(void) { return t_ntt_status; }

void ntt_h(uint32_t* A, const uint32_t* roots, uint32_t levels, unsigned long long astride,
           unsigned long long rstride, int32_t direction, uint32_t pidx) {
  cs_ctx* ctx = ntt_default_ctx();
  if (!ctx) { t_ntt_status = CS_ERR_NODEVICE; return; }
  if (pidx != 1 || !A || !roots || astride == 0 || rstride == 0) { t_ntt_status = CS_ERR_ARG; return; }
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  set_status(host_ntt(ctx, A, roots, levels, astride, rstride, direction >= 0 ? 1 : -1, -1), ctx);
}

void intt_h(uint32_t* A, const uint32_t* roots, uint32_t fmat, uint32_t levels, unsigned long long rstride,
            uint32_t pidx) {
  cs_ctx* ctx = ntt_default_ctx();
  if (!ctx) { t_ntt_status = CS_ERR_NODEVICE; return; }
  if (pidx != 1 || !A || !roots || rstride == 0) { t_ntt_status = CS_ERR_ARG; return; }
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  set_status(host_ntt(ctx, A, roots, levels, 1, rstride, -1, fmat ? 1 : 0), ctx);
}

void find_roots_h(uint32_t* roots, uint32_t* primitive_root, uint32_t nroots, uint32_t pidx) {
  cs_ctx* ctx = ntt_default_ctx();
  if (!ctx) { t_ntt_status = CS_ERR_NODEVICE; return; }
  if (pidx != 1 || !roots || !primitive_root) { t_ntt_status = CS_ERR_ARG; return; }
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaError_t e = ctx->in.reserve((size_t)nroots * 32 + 512, ctx->stream);
  if (e != cudaSuccess) { set_status(fail(ctx, e, "find_roots buffer"), ctx); return; }
  uint32_t* d = static_cast<uint32_t*>(ctx->in.ptr);
  uint32_t* droot = d + (size_t)nroots * 8;
  if ((e = cudaMemcpyAsync(droot, primitive_root, 32, cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess &&
      (e = ntt_powers(d, droot, nroots, ctx->stream)) == cudaSuccess &&
      (e = cudaMemcpyAsync(roots, d, (size_t)nroots * 32, cudaMemcpyDeviceToHost, ctx->stream)) == cudaSuccess)
    e = cudaStreamSynchronize(ctx->stream);
  set_status(e == cudaSuccess ? CS_OK : fail(ctx, e, "find_roots"), ctx);
}

uint32_t* ntt_interpolandmul_server_h(ntt_interpolandmul_t* args) {
  cs_ctx* ctx = ntt_default_ctx();
  if (!ctx) { t_ntt_status = CS_ERR_NODEVICE; return nullptr; }
  if (!args || !args->A || !args->B || !args->roots || args->pidx != 1 || args->rstride < 2) {
    t_ntt_status = CS_ERR_ARG;
    return nullptr;
  }
  const uint32_t L = args->Nrows + args->Ncols;
  if (L < 1 || L > 26) { t_ntt_status = CS_ERR_ARG; return nullptr; }
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  const size_t m = (size_t)1 << L, mb = m * 32;
  const uint64_t s2 = args->rstride >> 1;  // stride of the 2m-point transform
  std::vector<uint32_t> Wf(m * 8), Wi(m * 8);
  for (size_t j = 0; j < m; j++) {
    const uint64_t fi = (s2 * j) & (s2 * 2 * m - 1);
    const uint64_t ii = (s2 * ((2 * m - j) & (2 * m - 1))) & (s2 * 2 * m - 1);
    std::memcpy(&Wf[j * 8], args->roots + fi * 8, 32);
    std::memcpy(&Wi[j * 8], args->roots + ii * 8, 32);
  }
  cudaError_t e = ctx->in.reserve(12 * mb + 16 * 256 + 1024, ctx->stream);
  if (e != cudaSuccess) { set_status(fail(ctx, e, "interpolandmul buffers"), ctx); return nullptr; }
  Carve cv(ctx->in.ptr);
  uint32_t* dA = cv.take(mb);
  uint32_t* dB = cv.take(mb);
  uint32_t* dWf = cv.take(mb);
  uint32_t* dWi = cv.take(mb);
  uint32_t* dS = cv.take(mb);
  uint32_t* dOut = cv.take(2 * mb);
  uint32_t* dScr = cv.take(4 * mb);
  uint32_t* dCm = cv.take(9 * 32);   // m-point constants: [2] m^-1 R
  uint32_t* dC2 = cv.take(9 * 32);   // 2m-point constants: [3] (2m)^-1 normal
  std::vector<uint32_t>& res = interp_result();
  res.assign(2 * m * 8, 0u);
  bool ok = (e = cudaMemcpyAsync(dA, args->A, mb, cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess &&
            (e = cudaMemcpyAsync(dB, args->B, mb, cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess &&
            (e = cudaMemcpyAsync(dWf, Wf.data(), mb, cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess &&
            (e = cudaMemcpyAsync(dWi, Wi.data(), mb, cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess &&
            (e = cudaMemcpyAsync(dS, args->roots, mb, cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess;
  if (ok) {
    k_domain_consts<<<1, 32, 0, ctx->stream>>>(L, dCm);
    k_domain_consts<<<1, 32, 0, ctx->stream>>>(L + 1, dC2);
    note_launch(2);
    cudaEventRecord(ctx->ev_start, ctx->stream);
    e = hstep_reference_core(dA, dB, L, dWf, dWi, dS, dCm + 16, dC2 + 24, dOut, dScr, ctx->stream);
    cudaEventRecord(ctx->ev_stop, ctx->stream);
    ok = e == cudaSuccess &&
         (e = cudaMemcpyAsync(res.data(), dOut, 2 * mb, cudaMemcpyDeviceToHost, ctx->stream)) == cudaSuccess &&
         (e = cudaStreamSynchronize(ctx->stream)) == cudaSuccess;
  }
  if (!ok) { set_status(fail(ctx, e, "interpolandmul"), ctx); return nullptr; }
  g_interp_rows = args->Nrows;
  g_interp_cols = args->Ncols;
  interp_mmul().clear();
  set_status(CS_OK, ctx);
  return res.data();
}

uint32_t* get_Mtranspose_h(void) { return interp_result().empty() ? nullptr : interp_result().data(); }

// The reference keeps the H step's coefficients in M_mul as a 2^mr x 2^mc matrix before its
// last transpose into M_transpose (ntt.cpp:1066, split from ntt.cpp:767).
uint32_t* get_Mmul_h(void) {
  std::vector<uint32_t>& res = interp_result();
  if (res.empty()) return nullptr;
  std::vector<uint32_t>& mm = interp_mmul();
  if (mm.empty()) {
    const uint32_t mr = g_interp_rows < g_interp_cols ? g_interp_rows + 1 : g_interp_rows;
    const uint32_t mc = g_interp_rows < g_interp_cols ? g_interp_cols : g_interp_cols + 1;
    const size_t R = (size_t)1 << mr, C = (size_t)1 << mc;
    if (R * C * 8 != res.size()) return nullptr;
    mm.resize(res.size());
    for (size_t r = 0; r < R; r++)
      for (size_t c = 0; c < C; c++) std::memcpy(&mm[(r * C + c) * 8], &res[(c * R + r) * 8], 32);
  }
  return mm.data();
}

// Four-step transforms of the reference (ntt.cpp:274, :199): their result is the
// natural-order transform of 2^(Nrows+Ncols) points, computed here in one pass.
void ntt_parallel_h(uint32_t* A, const uint32_t* roots, uint32_t Nrows, uint32_t Ncols,
                    unsigned long long rstride, int32_t direction, fft_mode_t fft_mode, uint32_t pidx) {
  cs_ctx* ctx = ntt_default_ctx();
  if (!ctx) { t_ntt_status = CS_ERR_NODEVICE; return; }
  if (pidx != 1 || !A || !roots || rstride == 0 || (int)fft_mode < 0 || fft_mode >= FFT_T_MODE_N) {
    t_ntt_status = CS_ERR_ARG;
    return;
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  set_status(host_ntt(ctx, A, roots, Nrows + Ncols, 1, rstride, direction >= 0 ? 1 : -1, -1), ctx);
}

void ntt_parallel2D_h(uint32_t* A, const uint32_t* roots, uint32_t Nrows, uint32_t fft_Nyx, uint32_t Ncols,
                      uint32_t fft_Nxx, unsigned long long rstride, int32_t direction, uint32_t pidx) {
  cs_ctx* ctx = ntt_default_ctx();
  if (!ctx) { t_ntt_status = CS_ERR_NODEVICE; return; }
  if (pidx != 1 || !A || !roots || rstride == 0 || direction != 1 || fft_Nyx > Nrows || fft_Nxx > Ncols) {
    t_ntt_status = CS_ERR_ARG;
    return;
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  set_status(host_ntt(ctx, A, roots, Nrows + Ncols, 1, rstride, 1, -1), ctx);
}

// ------------------------------------------------------------ context API ------------
int cs_ntt_device(cs_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t log_n, int direction,
                  int fmat) {
  if (!ctx || !d_in || !d_out || log_n < 1 || log_n > 27) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  Domain* dom = nullptr;
  cudaError_t e = domain_get(ctx, log_n, &dom);
  if (e != cudaSuccess) return fail(ctx, e, "ntt domain");
  const size_t bytes = ((size_t)32 << log_n);
  if (d_in == d_out) {
    if ((e = ctx->work.reserve(bytes, ctx->stream)) != cudaSuccess) return fail(ctx, e, "ntt scratch");
  }
  NttArgs t;
  t.in = d_in; t.out = d_out; t.tmp = static_cast<uint32_t*>(ctx->work.ptr);
  t.log_n = log_n; t.log_tab = log_n;
  t.W = direction >= 0 ? dom->Wf : dom->Wi;
  if (direction < 0) t.post_scalar = dom->consts + (fmat ? 16 : 24);
  cudaEventRecord(ctx->ev_start, ctx->stream);
  e = ntt_run(t, ctx->stream);
  cudaEventRecord(ctx->ev_stop, ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "ntt launch");
  return CS_OK;
}

int cs_hstep_device(cs_ctx* ctx, int variant, const uint32_t* d_A, const uint32_t* d_B, const uint32_t* d_C,
                    uint32_t log_m, uint32_t* d_out) {
  if (!ctx || !d_A || !d_B || !d_out || log_m < 1 || log_m > 26) return CS_ERR_ARG;
  if (variant == CS_HSTEP_COSET && !d_C) return CS_ERR_ARG;
  if (variant != CS_HSTEP_REFERENCE && variant != CS_HSTEP_COSET) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  Domain *dom2 = nullptr, *dom1 = nullptr;
  cudaError_t e = domain_get(ctx, log_m + 1, &dom2);
  if (e == cudaSuccess) e = domain_get(ctx, log_m, &dom1);
  if (e != cudaSuccess) return fail(ctx, e, "hstep domain");
  const size_t mb = (size_t)32 << log_m;
  if ((e = ctx->work.reserve(4 * mb, ctx->stream)) != cudaSuccess) return fail(ctx, e, "hstep scratch");
  uint32_t* scr = static_cast<uint32_t*>(ctx->work.ptr);
  cudaEventRecord(ctx->ev_start, ctx->stream);
  if (variant == CS_HSTEP_REFERENCE)
    e = hstep_reference_core(d_A, d_B, log_m, dom2->Wf, dom2->Wi, dom2->Wf, dom1->consts + 16,
                             dom2->consts + 24, d_out, scr, ctx->stream);
  else
    e = hstep_coset_core(d_A, d_B, d_C, log_m, dom2, d_out, scr, ctx->stream);
  cudaEventRecord(ctx->ev_stop, ctx->stream);
  if (e != cudaSuccess) return fail(ctx, e, "hstep launch");
  return CS_OK;
}

}  // extern "C"
