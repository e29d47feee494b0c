// prove.cu -- device-resident proving key and the Groth16 prove pipeline.
//
// Follows the reference's CPU proving sequence (src/python/groth_prover.py:575-790
// pysnarkP_CPU and :1414-1453 in gen_proof):
//   pA = A.w, pB = B.w on the domain (mpoly_eval)       -> QAP rows (qap.cu)
//   M  = coefficients of A(x)B(x)                       -> H step, reference variant
//   polH = M[m .. 2m-2]
//   pi_A  = MSM(w ++ [1, r], A ++ [alpha_1, delta_1])   (G1)
//   pi_B  = MSM(w ++ [1, s], B2 ++ [beta_2, delta_2])   (G2)
//   pi_B1 = MSM(w ++ [1, s], B1 ++ [beta_1, delta_1])   (G1)
//   pi_C  = MSM(w[nPub+1 : nVars], C[nPub+1 : nVars])   (G1)
//   pi_C2 = MSM(polH ++ [-r s], hExps[0 .. m-2] ++ [delta_1])
//   pi_C <- pi_C2 + pi_C + s pi_A + r pi_B1
// The four witness MSMs run on separate streams and overlap the QAP/H-step chain; the
// scalings s pi_A and r pi_B1 start as soon as their MSM finishes.  With fixed-base tables
// of one window for C and H, the C MSM accumulates its buckets early (beside the H step) and
// hands them to the H MSM, which adds them to its own before its reduction: pi_C + pi_C2 from
// one bucket reduction instead of two (the same group element, so the same affine proof).
#include <atomic>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <algorithm>
#include <vector>

#include "../../include/cusnarks_b200.h"
#include "curve.cuh"
#include "msm.cuh"
#include "ntt.cuh"
#include "glv.cuh"
#include "qap.cuh"
#include "runtime.cuh"

namespace csb {
struct Domain;
int batch_build(cs_ctx* ctx, int ec2, const BatchSpec* jobs, uint32_t njobs, int task, cs_msm_batch** out);
cudaError_t batch_enqueue(cs_msm_batch* b, cudaStream_t st);
cudaError_t domain_get(cs_ctx* ctx, uint32_t L, Domain** out);
cudaError_t hstep_reference_core(const uint32_t* A, const uint32_t* B, uint32_t L, const uint32_t* Wf2,
                                 const uint32_t* Wi2, const uint32_t* shift, const uint32_t* minv_R,
                                 const uint32_t* m2inv, uint32_t* out, uint32_t* scratch, cudaStream_t st,
                                 uint32_t batch = 1, size_t stride = 0);
// accessors into the opaque Domain (hstep.cu)
const uint32_t* domain_wf(const Domain* d);
const uint32_t* domain_wi(const Domain* d);
const uint32_t* domain_consts(const Domain* d);
}  // namespace csb

using namespace csb;

struct cs_pk {
  uint64_t id = 0;  // unique per key and per fixed-base table build: names the key in graph caches
  int device = 0;
  uint32_t n_vars = 0, n_public = 0, m = 0, log_m = 0;
  QapRows rows_a, rows_b;
  uint32_t* a_ext = nullptr;   // nVars+2 G1
  uint32_t* b1_ext = nullptr;  // nVars+2 G1
  uint32_t* b2_ext = nullptr;  // nVars+2 G2
  uint32_t* c = nullptr;       // nVars G1
  uint32_t* h_ext = nullptr;   // m G1: hExps[0..m-2] ++ delta_1
  // Fixed-base tables of the five MSMs (msm.cuh), in one allocation; c == 0: none.
  struct Fixed {
    uint32_t* table = nullptr;
    uint32_t n = 0;
    int c = 0;
  };
  Fixed fa, fb1, fb2, fc, fh;
  void* fixed_block = nullptr;
  size_t fixed_bytes = 0, base_bytes = 0;
  std::vector<void*> owned;
  bool has_fixed() const { return fixed_block != nullptr; }
  void drop_fixed() {
    if (fixed_block) cudaFree(fixed_block);
    fixed_block = nullptr;
    fixed_bytes = 0;
    fa = fb1 = fb2 = fc = fh = Fixed{};
  }
  ~cs_pk() {
    drop_fixed();
    for (void* p : owned) cudaFree(p);
  }
  cudaError_t alloc(void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 256);
    if (e == cudaSuccess) {
      owned.push_back(*p);
      base_bytes += bytes ? bytes : 256;
    }
    return e;
  }
};

namespace {

std::atomic<uint64_t> g_pk_ids{1};

inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// scalars[n] = 1, scalars[n+1] = x (normal form)
__global__ void k_set_tail(uint32_t* __restrict__ scalars, uint32_t n, const uint32_t* __restrict__ x) {
  const int t = threadIdx.x;
  if (t < 8) {
    scalars[(size_t)n * 8 + t] = t == 0 ? 1u : 0u;
    scalars[(size_t)(n + 1) * 8 + t] = x[t];
  }
}

// dst = -(r s) mod r_field, normal form (the reference's montmult_neg_h(r_mont, s))
__global__ void k_neg_rs(const uint32_t* __restrict__ r, const uint32_t* __restrict__ s, uint32_t* __restrict__ dst) {
  if (threadIdx.x != 0) return;
  const Fr rm = ld_fp<ModR>(r).to_mont();
  st_fp<ModR>(dst, Fr::zero() - rm * ld_fp<ModR>(s));
}

// ---- k * P through the GLV endomorphism of BN254 G1 (glv.cuh): k = k1 + k2 lambda (mod r),
// |k1|, |k2| < 2^127, and k P = k1 P + k2 phi(P): 127 joint doublings instead of 254.
struct GlvSplit {
  uint32_t k1[4], k2[4];  // magnitudes, little-endian
  uint32_t neg1, neg2, pad[6];
};

namespace glv_host {
using namespace csb::glv;
// k mod r for any 256-bit k (at most 5 subtractions)
inline void reduce_r(uint64_t* k) {
  static constexpr uint64_t R[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull,
                                    0x30644e72e131a029ull};
  for (int it = 0; it < 6; it++) {
    bool ge = true;
    for (int i = 3; i >= 0; i--) {
      if (k[i] != R[i]) { ge = k[i] > R[i]; break; }
    }
    if (!ge) return;
    addsub(k, R, 4, true);
  }
}

inline GlvSplit split(const uint32_t* k32) {
  uint64_t k[4];
  for (int i = 0; i < 4; i++) k[i] = (uint64_t)k32[2 * i] | ((uint64_t)k32[2 * i + 1] << 32);
  reduce_r(k);
  GlvSplit g{};
  split_reduced(k, g.k1, &g.neg1, g.k2, &g.neg2);
  return g;
}
}  // namespace glv_host

// out (XYZZ) = k * P for P affine (G1), k given as its GLV split.
// One warp (launched with 32 threads; its 8 quads compute the same): the independent
// products of each doubling and addition run on the lanes of a quad; lane 0 stores.
__device__ void scale_point_glv(const uint32_t* __restrict__ P, const GlvSplit* __restrict__ gs,
                                uint32_t* __restrict__ out) {
  Fq beta;
  glv::beta_mont(beta.v);
  const GlvSplit g = *gs;
  Affine<Fq> p = ld_affine<Fq>(P);
  XYZZ<Fq> acc = XYZZ<Fq>::inf();
  if (!affine_is_inf(p)) {
    Affine<Fq> q{p.x * beta, p.y};  // phi(P) = lambda P
    if (g.neg1) p.y = p.y.neg();
    if (g.neg2) q.y = q.y.neg();
    const XYZZ<Fq> pq = xyzz_madd(XYZZ<Fq>::from_affine(p), q);  // P + phi(P) (never infinity)
    for (int b = 127; b >= 0; b--) {
      acc = xyzz_dbl_quad(acc);
      const uint32_t e1 = (g.k1[b >> 5] >> (b & 31)) & 1u, e2 = (g.k2[b >> 5] >> (b & 31)) & 1u;
      if (e1 && e2) acc = xyzz_add_quad(acc, pq);
      else if (e1) acc = xyzz_add_quad(acc, XYZZ<Fq>::from_affine(p));
      else if (e2) acc = xyzz_add_quad(acc, XYZZ<Fq>::from_affine(q));
    }
  }
  if (threadIdx.x == 0) st_xyzz<Fq>(out, acc);
}
__global__ void k_scale_point_glv(const uint32_t* __restrict__ P, const GlvSplit* __restrict__ gs,
                                  uint32_t* __restrict__ out) {
  scale_point_glv(P, gs, out);
}

// pi_C = C2 + C + sA + rB1 (C2, C affine; sA, rB1 XYZZ) -> affine
__device__ void final_c(const uint32_t* __restrict__ c2, const uint32_t* __restrict__ c,
                        const uint32_t* __restrict__ sa, const uint32_t* __restrict__ rb1,
                        uint32_t* __restrict__ out) {
  XYZZ<Fq> acc = XYZZ<Fq>::inf();
  const Affine<Fq> a = ld_affine<Fq>(c2), b = ld_affine<Fq>(c);
  if (!affine_is_inf(a)) acc = xyzz_madd(acc, a);
  if (!affine_is_inf(b)) acc = xyzz_madd(acc, b);
  acc = xyzz_add(acc, ld_xyzz<Fq>(sa));
  acc = xyzz_add(acc, ld_xyzz<Fq>(rb1));
  st_affine<Fq>(out, xyzz_to_affine(acc));
}
__global__ void k_final_c(const uint32_t* __restrict__ c2, const uint32_t* __restrict__ c,
                          const uint32_t* __restrict__ sa, const uint32_t* __restrict__ rb1,
                          uint32_t* __restrict__ out) {
  if (threadIdx.x == 0) final_c(c2, c, sa, rb1, out);
}

cudaError_t copy_in(void* dst, const void* src, size_t bytes, int on_device, cudaStream_t st) {
  if (!bytes) return cudaSuccess;
  return cudaMemcpyAsync(dst, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
}

uint32_t ilog2_exact(uint32_t m) {
  uint32_t l = 0;
  while ((1u << l) < m) l++;
  return (1u << l) == m ? l : 0xffffffffu;
}

// Layout of the per-call prove scratch.
struct ProvePlan {
  size_t wA, wB, pA, pB, M, hscr, ms_a, ms_b1, ms_b2, ms_c, ms_h, pts, rs, cbk, total;
  size_t bytes_a, bytes_b1, bytes_b2, bytes_c, bytes_h;
  // C and H share one bucket reduction: both fixed-base with the same window, C's buckets
  // (cbk) folded into H's before H reduces (pi_C only needs their sum)
  bool share_ch;
};

ProvePlan plan_prove(const cs_pk* pk) {
  ProvePlan P{};
  const size_t nv = pk->n_vars, m = pk->m;
  const uint32_t nc = pk->n_vars - pk->n_public - 1;
  if (pk->has_fixed()) {
    P.bytes_a = msm_fixed_workspace_bytes(pk->fa.n, pk->fa.c, false);
    P.bytes_b1 = msm_fixed_workspace_bytes(pk->fb1.n, pk->fb1.c, false);
    P.bytes_b2 = msm_fixed_workspace_bytes(pk->fb2.n, pk->fb2.c, true);
    P.bytes_c = msm_fixed_workspace_bytes(pk->fc.n, pk->fc.c, false);
    P.bytes_h = msm_fixed_workspace_bytes(pk->fh.n, pk->fh.c, false);
  } else {
    P.bytes_a = msm_workspace_bytes(pk->n_vars + 2, 0, false);
    P.bytes_b1 = P.bytes_a;
    P.bytes_b2 = msm_workspace_bytes(pk->n_vars + 2, 0, true);
    P.bytes_c = msm_workspace_bytes(nc, 0, false);
    P.bytes_h = msm_workspace_bytes(pk->m, 0, false);
  }
  size_t o = 0;
  P.wA = o; o += al256((nv + 2) * 32);
  P.wB = o; o += al256((nv + 2) * 32);
  P.pA = o; o += al256(m * 32);
  P.pB = o; o += al256(m * 32);
  P.M = o; o += al256(2 * m * 32);
  P.hscr = o; o += al256(4 * m * 32);
  P.ms_a = o; o += al256(P.bytes_a);
  P.ms_b1 = o; o += al256(P.bytes_b1);
  P.ms_b2 = o; o += al256(P.bytes_b2);
  P.ms_c = o; o += al256(P.bytes_c);
  P.ms_h = o; o += al256(P.bytes_h);
  P.pts = o; o += 2048;   // outA 64, outB1 64, outB2 128, outC 64, outH 64, sA 128, rB1 128, piC 64
  P.rs = o; o += 256;     // r, s, -rs, then the GLV splits of s and r (2 x 64 B)
  P.share_ch = pk->has_fixed() && pk->fc.c > 0 && pk->fc.c == pk->fh.c && pk->fc.n > 0 && pk->fh.n > 0;
  P.cbk = o;
  if (P.share_ch) o += al256(((size_t)1 << (pk->fc.c - 1)) * 128);  // G1 XYZZ buckets
  P.total = o;
  return P;
}

// The proof's launch sequence after the scalar uploads (which cs_prove_device makes): the
// witness scalars with their extensions, the four witness MSMs on the auxiliary streams with
// the GLV scalings, QAP -> H step -> H MSM on the H stream, the join and the final pi_C.
// Results land in the scratch's point area.  Sets *where on failure.
cudaError_t prove_body(cs_ctx* ctx, cs_pk* pk, const ProvePlan& P, const uint32_t* d_w, Domain* dom1,
                       Domain* dom2, const char** where) {
  char* base = static_cast<char*>(ctx->work.ptr);
  auto at = [&](size_t off) { return reinterpret_cast<uint32_t*>(base + off); };
  uint32_t *wA = at(P.wA), *wB = at(P.wB), *pA = at(P.pA), *pB = at(P.pB), *M = at(P.M), *hscr = at(P.hscr);
  uint32_t* pts = at(P.pts);
  uint32_t *outA = pts, *outB1 = pts + 16, *outB2 = pts + 32, *outC = pts + 64, *outH = pts + 80;
  uint32_t *sA = pts + 96, *rB1 = pts + 128, *piC = pts + 160;
  uint32_t* rs = at(P.rs);
  const uint32_t nv = pk->n_vars, m = pk->m, np1 = pk->n_public + 1;
  cudaStream_t s0 = ctx->stream;
  cudaEvent_t ev_w = ctx->aux_ev[0];
  MsmConfig cfg;
  cudaError_t e;
  // scalars: w ++ [1, r] and w ++ [1, s]; -rs
  bool ok = (e = cudaMemcpyAsync(wA, d_w, (size_t)nv * 32, cudaMemcpyDeviceToDevice, s0)) == cudaSuccess &&
            (e = cudaMemcpyAsync(wB, d_w, (size_t)nv * 32, cudaMemcpyDeviceToDevice, s0)) == cudaSuccess;
  if (!ok) { *where = "prove inputs"; return e; }
  k_set_tail<<<1, 32, 0, s0>>>(wA, nv, rs);
  k_set_tail<<<1, 32, 0, s0>>>(wB, nv, rs + 8);
  k_neg_rs<<<1, 32, 0, s0>>>(rs, rs + 8, rs + 16);
  note_launch(3);
  cudaEventRecord(ev_w, s0);
  // witness MSMs on the auxiliary streams
  cudaStream_t sa = ctx->aux[0], sb1 = ctx->aux[1], sb2 = ctx->aux[2], sc = ctx->aux[3];
  for (int i = 0; i < 4; i++) cudaStreamWaitEvent(ctx->aux[i], ev_w, 0);
  // resident fixed-base tables when the key has them, else the generic MSM over the points
  auto run_msm = [&](bool ec2, const uint32_t* sc, const uint32_t* pts, const cs_pk::Fixed& f, uint32_t n,
                     uint32_t* out, size_t off, size_t bytes, cudaStream_t st, const MsmConfig* share = nullptr) {
    if (pk->has_fixed()) {
      MsmConfig fcfg = share ? *share : MsmConfig{};
      fcfg.c = f.c;
      return ec2 ? msm_fixed_g2(sc, f.table, n, out, at(off), bytes, fcfg, st)
                 : msm_fixed_g1(sc, f.table, n, out, at(off), bytes, fcfg, st);
    }
    return ec2 ? msm_g2(sc, pts, n, out, at(off), bytes, cfg, st) : msm_g1(sc, pts, n, out, at(off), bytes, cfg, st);
  };
  // C hands its buckets to H (outC is then the point at infinity, and outH the sum of both)
  MsmConfig share_c, share_h;
  if (P.share_ch) {
    share_c.bucket_out = at(P.cbk);
    share_h.bucket_add = at(P.cbk);
    share_h.bucket_ready = ctx->aux_ev[7];
  }
  ok = (e = run_msm(false, wA, pk->a_ext, pk->fa, nv + 2, outA, P.ms_a, P.bytes_a, sa)) == cudaSuccess &&
       (e = run_msm(false, wB, pk->b1_ext, pk->fb1, nv + 2, outB1, P.ms_b1, P.bytes_b1, sb1)) == cudaSuccess &&
       (e = run_msm(true, wB, pk->b2_ext, pk->fb2, nv + 2, outB2, P.ms_b2, P.bytes_b2, sb2)) == cudaSuccess &&
       (e = run_msm(false, wA + (size_t)np1 * 8, pk->c + (size_t)np1 * 16, pk->fc, nv - np1, outC, P.ms_c, P.bytes_c,
                    sc, &share_c)) == cudaSuccess;
  if (!ok) { *where = "prove witness MSMs"; return e; }
  if (P.share_ch && (e = cudaEventRecord(ctx->aux_ev[7], sc)) != cudaSuccess) { *where = "prove C buckets"; return e; }
  {
    const GlvSplit* gsp = reinterpret_cast<const GlvSplit*>(rs + 32);
    k_scale_point_glv<<<1, 32, 0, sa>>>(outA, gsp, sA);        // s * pi_A
    k_scale_point_glv<<<1, 32, 0, sb1>>>(outB1, gsp + 1, rB1);  // r * pi_B1
  }
  note_launch(2);
  // QAP evaluation, H step and H MSM on their own stream
  cudaStream_t sh = ctx->aux_h;
  cudaStreamWaitEvent(sh, ev_w, 0);
  ok = (e = qap_eval(pk->rows_a, d_w, pA, 0, sh)) == cudaSuccess &&
       (e = qap_eval(pk->rows_b, d_w, pB, 0, sh)) == cudaSuccess &&
       (e = hstep_reference_core(pA, pB, pk->log_m, domain_wf(dom2), domain_wi(dom2), domain_wf(dom2),
                                 domain_consts(dom1) + 16, domain_consts(dom2) + 24, M, hscr, sh)) == cudaSuccess &&
       (e = cudaEventRecord(ctx->aux_ev[6], sh)) == cudaSuccess &&  // H step done (stage times)
       // polH = M[m .. 2m-2]; M[2m-1] (always zero) becomes the -rs term for delta_1
       (e = cudaMemcpyAsync(M + (size_t)(2 * m - 1) * 8, rs + 16, 32, cudaMemcpyDeviceToDevice, sh)) == cudaSuccess &&
       (e = run_msm(false, M + (size_t)m * 8, pk->h_ext, pk->fh, m, outH, P.ms_h, P.bytes_h, sh, &share_h)) == cudaSuccess;
  if (!ok) { *where = "prove QAP/H"; return e; }
  // pi_C needs the A, B1, C and H chains but not the G2 MSM: it runs on the H stream while
  // B2 may still be running, and the context stream joins both (2^12 proof: the G2 chain ends
  // last, so pi_C's affine conversion no longer follows it)
  cudaEventRecord(ctx->aux_ev[5], sh);  // H MSM done (stage times)
  for (int i : {0, 1, 3}) {
    cudaEventRecord(ctx->aux_ev[1 + i], ctx->aux[i]);
    cudaStreamWaitEvent(sh, ctx->aux_ev[1 + i], 0);
  }
  k_final_c<<<1, 32, 0, sh>>>(outH, outC, sA, rB1, piC);
  note_launch();
  cudaEventRecord(ctx->aux_ev[3], ctx->aux[2]);  // B2 done
  cudaEventRecord(ctx->aux_ev[8], sh);           // pi_C done
  cudaStreamWaitEvent(s0, ctx->aux_ev[3], 0);
  cudaStreamWaitEvent(s0, ctx->aux_ev[8], 0);
  return cudaGetLastError();
}

// Captures prove_body on the context stream as a CUDA graph, keeps it for the key, witness
// buffer and scratch, and launches it.  Capture is thread-local, so other threads
// (other server slots) keep launching meanwhile.  If the capture or its instantiation fails, the
// entry records that and the sequence runs launch by launch, now and on later calls.
cudaError_t prove_capture(cs_ctx* ctx, cs_pk* pk, const ProvePlan& P, const uint32_t* d_w, Domain* dom1,
                          Domain* dom2, const char** where) {
  // a served context sees every key of its server: room for that many, the oldest goes first
  // (a graph destroyed while a launch of it runs is freed when the launch completes)
  constexpr size_t kMaxGraphs = 32;
  cudaStream_t s0 = ctx->stream;
  // entries made with an earlier scratch arena can never match again
  for (size_t i = 0; i < ctx->prove_graphs.size();) {
    auto& x = ctx->prove_graphs[i];
    if (x.work != ctx->work.ptr || x.work_bytes != ctx->work.bytes) {
      if (x.exec) cudaGraphExecDestroy(x.exec);
      ctx->prove_graphs.erase(ctx->prove_graphs.begin() + i);
    } else {
      i++;
    }
  }
  if (ctx->prove_graphs.size() >= kMaxGraphs) {
    if (ctx->prove_graphs.front().exec) cudaGraphExecDestroy(ctx->prove_graphs.front().exec);
    ctx->prove_graphs.erase(ctx->prove_graphs.begin());
  }
  cs_ctx::ProveGraph g;
  g.pk_id = pk->id;
  g.d_w = d_w;
  g.work = ctx->work.ptr;
  g.work_bytes = ctx->work.bytes;
  const unsigned long long l0 = thread_launches();
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const cudaError_t eb = prove_body(ctx, pk, P, d_w, dom1, dom2, where);
    e = cudaStreamEndCapture(s0, &graph);
    if (eb != cudaSuccess) e = eb;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g.exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e == cudaSuccess) {
    g.launches = thread_launches() - l0;
    ctx->prove_graphs.push_back(g);
    *where = "prove graph launch";
    return cudaGraphLaunch(g.exec, s0);
  }
  // capture failed: clear the error, remember not to capture this combination again and run
  // the launches directly
  cudaGetLastError();
  g.exec = nullptr;
  ctx->prove_graphs.push_back(g);
  *where = "prove launch";
  return prove_body(ctx, pk, P, d_w, dom1, dom2, where);
}

// ------------------------------------------------------------------ proof batches ----
// Several proofs with one key in one pass: their MSMs run as three batched launch sequences
// (the A, B1 and C MSMs of every proof in one G1 batch, the B2 MSMs in one G2 batch, the H
// MSMs in one G1 batch after the H steps), each a single sort and a single accumulation over
// all instances' buckets with the resident fixed-base tables; the QAP and H steps, the GLV
// scalings and the final combinations run per proof inside the same captured sequence.

// One proof's call inputs, uploaded in one copy per batch.
struct BatchCall {
  uint32_t r[8], s[8];
  GlvSplit glv[2];  // s (for s pi_A), r (for r pi_B1)
  const uint32_t* d_w;
  uint32_t* d_proof;
  uint32_t pad[12];
};
static_assert(sizeof(BatchCall) == 256, "BatchCall layout");

struct ProveBatch {
  uint64_t pk_id = 0;
  uint32_t k = 0;
  void* buf = nullptr;
  size_t per = 0, calls_off = 0, bytes = 0;
  size_t o_wA = 0, o_wB = 0, o_pA = 0, o_pB = 0, o_M = 0, o_hscr = 0, o_pts = 0, o_rs = 0;
  PinnedBuffer host;
  cudaEvent_t uploaded = nullptr;
  cs_msm_batch *g1abc = nullptr, *g2 = nullptr, *g1h = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long launches = 0;
  bool no_graph = false;
  ~ProveBatch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (g1abc) cs_msm_batch_destroy(g1abc);
    if (g2) cs_msm_batch_destroy(g2);
    if (g1h) cs_msm_batch_destroy(g1h);
    if (uploaded) cudaEventDestroy(uploaded);
    host.release();
    if (buf) cudaFree(buf);
  }
  uint32_t* at(uint32_t i, size_t off) const {
    return reinterpret_cast<uint32_t*>(static_cast<char*>(buf) + (size_t)i * per + off);
  }
  BatchCall* calls() const { return reinterpret_cast<BatchCall*>(static_cast<char*>(buf) + calls_off); }
};

// wA = w ++ [1, r], wB = w ++ [1, s] per proof (grid.y = proof); thread 0 of each proof also
// writes r, s, -r s and the GLV splits into the proof's rs area.
__global__ void k_batch_prep(const BatchCall* __restrict__ calls, uint32_t nv, char* __restrict__ base, size_t per,
                             size_t o_wA, size_t o_wB, size_t o_rs) {
  const uint32_t k = blockIdx.y;
  const BatchCall* c = calls + k;
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t* wA = reinterpret_cast<uint32_t*>(base + (size_t)k * per + o_wA);
  uint32_t* wB = reinterpret_cast<uint32_t*>(base + (size_t)k * per + o_wB);
  if (e < nv) {
    uint32_t v[8];
    ld_limbs8(v, c->d_w + (size_t)e * 8);
    st_limbs8(wA + (size_t)e * 8, v);
    st_limbs8(wB + (size_t)e * 8, v);
  } else if (e < nv + 2) {
    for (int t = 0; t < 8; t++) {
      const uint32_t one = t == 0 ? 1u : 0u;
      wA[(size_t)e * 8 + t] = e == nv ? one : c->r[t];
      wB[(size_t)e * 8 + t] = e == nv ? one : c->s[t];
    }
  }
  if (e == 0) {
    uint32_t* rs = reinterpret_cast<uint32_t*>(base + (size_t)k * per + o_rs);
    for (int t = 0; t < 8; t++) { rs[t] = c->r[t]; rs[8 + t] = c->s[t]; }
    Fr rr, ss;
    for (int t = 0; t < 8; t++) { rr.v[t] = c->r[t]; ss.v[t] = c->s[t]; }
    const Fr neg = Fr::zero() - rr.to_mont() * ss;  // -(r s), normal form
    for (int t = 0; t < 8; t++) rs[16 + t] = neg.v[t];
    const uint32_t* g = reinterpret_cast<const uint32_t*>(c->glv);
    for (int t = 0; t < 32; t++) rs[32 + t] = g[t];
  }
}

// s pi_A and r pi_B1 of every proof: block 2k + which, one warp each.
__global__ void k_batch_scale(char* __restrict__ base, size_t per, size_t o_pts, size_t o_rs) {
  const uint32_t k = blockIdx.x >> 1, which = blockIdx.x & 1;
  uint32_t* pts = reinterpret_cast<uint32_t*>(base + (size_t)k * per + o_pts);
  const GlvSplit* gs = reinterpret_cast<const GlvSplit*>(base + (size_t)k * per + o_rs + 32 * 4) + which;
  scale_point_glv(which ? pts + 16 : pts, gs, which ? pts + 128 : pts + 96);
}

// Proof k's H coefficient 2m-1 (always zero) becomes its -r s (block k), the scalar of the
// delta_1 point that ends the H MSM's bases, as in the single-proof path.
__global__ void k_batch_rs(char* __restrict__ base, size_t per, size_t o_rs, size_t o_M, size_t m) {
  const uint32_t* rs = reinterpret_cast<const uint32_t*>(base + blockIdx.x * per + o_rs) + 16;
  uint32_t* M = reinterpret_cast<uint32_t*>(base + blockIdx.x * per + o_M) + (2 * m - 1) * 8;
  M[threadIdx.x] = rs[threadIdx.x];
}

// pi_C of every proof (block k): needs the G1 MSMs, their scalings and the H MSMs, not G2.
__global__ void k_batch_pic(char* __restrict__ base, size_t per, size_t o_pts) {
  uint32_t* pts = reinterpret_cast<uint32_t*>(base + (size_t)blockIdx.x * per + o_pts);
  if (threadIdx.x == 0) final_c(pts + 80, pts + 64, pts + 96, pts + 128, pts + 160);
}

// The proof words of every proof (block k) to the caller's buffer.
__global__ void k_batch_final(const BatchCall* __restrict__ calls, char* __restrict__ base, size_t per,
                              size_t o_pts) {
  const uint32_t k = blockIdx.x;
  const uint32_t* pts = reinterpret_cast<const uint32_t*>(base + (size_t)k * per + o_pts);
  const uint32_t t = threadIdx.x;  // 64 threads: pi_A (16) | pi_B (32) | pi_C (16)
  if (t < 64) {
    const uint32_t v = t < 16 ? pts[t] : t < 48 ? pts[32 + (t - 16)] : pts[160 + (t - 48)];
    calls[k].d_proof[t] = v;
  }
}

// The batch's launch sequence after the call upload.
cudaError_t prove_batch_body(cs_ctx* ctx, cs_pk* pk, ProveBatch& B, Domain* dom1, Domain* dom2, const char** where) {
  const uint32_t nv = pk->n_vars, m = pk->m, K = B.k;
  char* base = static_cast<char*>(B.buf);
  cudaStream_t s0 = ctx->stream, sa = ctx->aux[0], sb = ctx->aux[1], sh = ctx->aux_h;
  cudaError_t e;
  k_batch_prep<<<dim3((nv + 2 + 127) / 128, K), 128, 0, s0>>>(B.calls(), nv, base, B.per, B.o_wA, B.o_wB, B.o_rs);
  note_launch();
  cudaEventRecord(ctx->aux_ev[0], s0);
  for (cudaStream_t st : {sa, sb, sh}) cudaStreamWaitEvent(st, ctx->aux_ev[0], 0);
  // A, B1, C of every proof; then the GLV scalings (they read pi_A, pi_B1)
  if ((e = batch_enqueue(B.g1abc, sa)) != cudaSuccess) { *where = "prove batch G1 MSMs"; return e; }
  k_batch_scale<<<2 * K, 32, 0, sa>>>(base, B.per, B.o_pts, B.o_rs);
  note_launch();
  if ((e = batch_enqueue(B.g2, sb)) != cudaSuccess) { *where = "prove batch G2 MSMs"; return e; }
  {  // the K QAP evaluations and H steps as batched launches (per-proof arrays B.per bytes apart)
    const size_t stride = B.per / sizeof(uint32_t);
    const bool ok =
        (e = qap_eval(pk->rows_a, B.at(0, B.o_wA), B.at(0, B.o_pA), 0, sh, K, stride)) == cudaSuccess &&
        (e = qap_eval(pk->rows_b, B.at(0, B.o_wA), B.at(0, B.o_pB), 0, sh, K, stride)) == cudaSuccess &&
        (e = hstep_reference_core(B.at(0, B.o_pA), B.at(0, B.o_pB), pk->log_m, domain_wf(dom2), domain_wi(dom2),
                                  domain_wf(dom2), domain_consts(dom1) + 16, domain_consts(dom2) + 24,
                                  B.at(0, B.o_M), B.at(0, B.o_hscr), sh, K, stride)) == cudaSuccess;
    if (!ok) { *where = "prove batch QAP/H"; return e; }
    k_batch_rs<<<K, 8, 0, sh>>>(base, B.per, B.o_rs, B.o_M, m);
    note_launch();
  }
  if ((e = batch_enqueue(B.g1h, sh)) != cudaSuccess) { *where = "prove batch H MSMs"; return e; }
  // pi_C beside the G2 batch (on the H stream once the G1 side is done), then the proof words
  cudaEventRecord(ctx->aux_ev[1], sa);
  cudaStreamWaitEvent(sh, ctx->aux_ev[1], 0);
  k_batch_pic<<<K, 32, 0, sh>>>(base, B.per, B.o_pts);
  cudaEventRecord(ctx->aux_ev[2], sb);
  cudaEventRecord(ctx->aux_ev[5], sh);
  for (int i : {2, 5}) cudaStreamWaitEvent(s0, ctx->aux_ev[i], 0);
  k_batch_final<<<K, 64, 0, s0>>>(B.calls(), base, B.per, B.o_pts);
  note_launch(2);
  return cudaGetLastError();
}

// The context's plan for (key, batch size), made on first use: per-proof scratch, the three
// MSM batch plans over it, the pinned call staging.  At most 16 plans per context (a server
// slot meets a few small keys at a few batch sizes); the least recently used one goes.
int prove_batch_plan(cs_ctx* ctx, cs_pk* pk, uint32_t K, ProveBatch** out) {
  auto& plans = ctx->prove_batches;
  for (size_t i = 0; i < plans.size(); i++) {
    ProveBatch* b = static_cast<ProveBatch*>(plans[i].get());
    if (b->pk_id == pk->id && b->k == K) {
      std::rotate(plans.begin() + i, plans.begin() + i + 1, plans.end());  // most recent last
      *out = b;
      return CS_OK;
    }
  }
  constexpr size_t kMaxPlans = 16;
  if (ctx->prove_batches.size() >= kMaxPlans) {  // the least recent goes, once nothing of it runs
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail(ctx, e, "prove batch plan cache");
    ctx->prove_batches.erase(ctx->prove_batches.begin());
  }
  std::shared_ptr<ProveBatch> B(new ProveBatch());
  B->pk_id = pk->id;
  B->k = K;
  const size_t nv = pk->n_vars, m = pk->m;
  size_t o = 0;
  B->o_wA = o; o += al256((nv + 2) * 32);
  B->o_wB = o; o += al256((nv + 2) * 32);
  B->o_pA = o; o += al256(m * 32);
  B->o_pB = o; o += al256(m * 32);
  B->o_M = o; o += al256(2 * m * 32);
  B->o_hscr = o; o += al256(4 * m * 32);
  B->o_pts = o; o += 2048;
  B->o_rs = o; o += 256;
  B->per = al256(o);
  B->calls_off = B->per * K;
  B->bytes = B->calls_off + sizeof(BatchCall) * K;
  cudaError_t e = cudaMalloc(&B->buf, B->bytes);
  if (e == cudaSuccess) e = B->host.reserve(sizeof(BatchCall) * K);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->uploaded, cudaEventDisableTiming);
  if (e != cudaSuccess) return fail(ctx, e, "prove batch buffers");
  const uint32_t np1 = pk->n_public + 1;
  std::vector<BatchSpec> abc, b2, h;
  for (uint32_t i = 0; i < K; i++) {
    uint32_t* pts = B->at(i, B->o_pts);
    abc.push_back(BatchSpec{B->at(i, B->o_wA), pk->fa.table, pts, pk->fa.n, pk->fa.c, true});
    abc.push_back(BatchSpec{B->at(i, B->o_wB), pk->fb1.table, pts + 16, pk->fb1.n, pk->fb1.c, true});
    abc.push_back(BatchSpec{B->at(i, B->o_wA) + (size_t)np1 * 8, pk->fc.table, pts + 64, pk->fc.n, pk->fc.c, true});
    b2.push_back(BatchSpec{B->at(i, B->o_wB), pk->fb2.table, pts + 32, pk->fb2.n, pk->fb2.c, true});
    h.push_back(BatchSpec{B->at(i, B->o_M) + (size_t)m * 8, pk->fh.table, pts + 80, pk->fh.n, pk->fh.c, true});
  }
  int st = batch_build(ctx, 0, abc.data(), (uint32_t)abc.size(), 0, &B->g1abc);
  if (st == CS_OK) st = batch_build(ctx, 1, b2.data(), (uint32_t)b2.size(), 0, &B->g2);
  if (st == CS_OK) st = batch_build(ctx, 0, h.data(), (uint32_t)h.size(), 0, &B->g1h);
  if (st != CS_OK) return st;
  ctx->prove_batches.push_back(B);
  *out = B.get();
  return CS_OK;
}

}  // namespace

namespace csb {
void prove_graphs_release(cs_ctx* ctx) {
  for (auto& g : ctx->prove_graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  ctx->prove_graphs.clear();
  ctx->prove_batches.clear();
}
size_t prove_workspace_bytes(const cs_pk* pk) { return plan_prove(pk).total; }
uint32_t pk_domain(const cs_pk* pk) { return pk->m; }
bool pk_has_fixed(const cs_pk* pk) { return pk->has_fixed(); }
// Whether the context already holds the batch plan for (key, k): a batch then allocates nothing.
bool prove_batch_ready(cs_ctx* ctx, const cs_pk* pk, uint32_t k) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  for (auto& p : ctx->prove_batches) {
    const ProveBatch* b = static_cast<const ProveBatch*>(p.get());
    if (b->pk_id == pk->id && b->k == k) return true;
  }
  return false;
}
uint32_t pk_n_vars(const cs_pk* pk) { return pk->n_vars; }
// Grows the context's arenas to what a proof with this key needs (cs_prove would grow them
// on its first call): lets the server allocate a slot's scratch right after admission.
// Grows the context's scratch arena and witness buffer to at least these sizes.
cudaError_t ctx_reserve(cs_ctx* ctx, size_t work_bytes, size_t in_bytes) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaError_t e = ctx->work.reserve(work_bytes, ctx->stream);
  if (e == cudaSuccess) e = ctx->in.reserve(in_bytes, ctx->stream);
  return e;
}
}  // namespace csb

extern "C" {

int cs_pk_create(cs_ctx* ctx, const cs_pk_desc* d, int on_device, cs_pk** out) {
  if (!ctx || !d || !out) return CS_ERR_ARG;
  *out = nullptr;
  if (d->n_vars < d->n_public + 2 || !d->polsA || !d->polsB || !d->A || !d->B1 || !d->B2 || !d->C ||
      !d->hExps || !d->delta_1)
    return fail_msg(ctx, CS_ERR_ARG, "cs_pk_create: incomplete proving key description");
  const uint32_t L = ilog2_exact(d->domain_size);
  if (L == 0xffffffffu || L < 2 || L > 26) return fail_msg(ctx, CS_ERR_ARG, "cs_pk_create: domain size must be 2^k, 4 <= 2^k <= 2^26");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  std::unique_ptr<cs_pk> pk(new cs_pk());
  pk->id = g_pk_ids.fetch_add(1);
  pk->device = ctx->device;
  pk->n_vars = d->n_vars;
  pk->n_public = d->n_public;
  pk->m = d->domain_size;
  pk->log_m = L;
  const size_t nv = d->n_vars, m = d->domain_size;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  // points
  if ((e = pk->alloc((void**)&pk->a_ext, (nv + 2) * 64)) != cudaSuccess ||
      (e = pk->alloc((void**)&pk->b1_ext, (nv + 2) * 64)) != cudaSuccess ||
      (e = pk->alloc((void**)&pk->b2_ext, (nv + 2) * 128)) != cudaSuccess ||
      (e = pk->alloc((void**)&pk->c, nv * 64)) != cudaSuccess ||
      (e = pk->alloc((void**)&pk->h_ext, m * 64)) != cudaSuccess)
    return fail(ctx, e, "cs_pk_create: point buffers");
  if ((e = copy_in(pk->a_ext, d->A, (nv + 2) * 64, on_device, st)) != cudaSuccess ||
      (e = copy_in(pk->b1_ext, d->B1, (nv + 2) * 64, on_device, st)) != cudaSuccess ||
      (e = copy_in(pk->b2_ext, d->B2, (nv + 2) * 128, on_device, st)) != cudaSuccess ||
      (e = copy_in(pk->c, d->C, nv * 64, on_device, st)) != cudaSuccess ||
      (e = copy_in(pk->h_ext, d->hExps, (m - 1) * 64, on_device, st)) != cudaSuccess ||
      (e = copy_in(pk->h_ext + (m - 1) * 16, d->delta_1, 64, on_device, st)) != cudaSuccess)
    return fail(ctx, e, "cs_pk_create: point upload");
  // QAP matrices: reference mpoly layout -> constraint rows
  for (int which = 0; which < 2; which++) {
    const uint32_t* pm = which == 0 ? d->polsA : d->polsB;
    const size_t words = which == 0 ? d->polsA_words : d->polsB_words;
    const uint32_t n_entries = which == 0 ? d->polsA_entries : d->polsB_entries;
    QapRows& R = which == 0 ? pk->rows_a : pk->rows_b;
    uint32_t* dm = nullptr;
    if ((e = cudaMalloc(&dm, words * 4)) != cudaSuccess) return fail(ctx, e, "cs_pk_create: mpoly");
    e = copy_in(dm, pm, words * 4, on_device, st);
    if (e == cudaSuccess) e = pk->alloc((void**)&R.row_off, (m + 1) * 4);
    if (e == cudaSuccess) e = pk->alloc((void**)&R.wire, (size_t)n_entries * 4);
    if (e == cudaSuccess) e = pk->alloc((void**)&R.coeff, (size_t)n_entries * 32);
    void* scratch = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&scratch, qap_transpose_scratch_bytes(d->n_vars, (uint32_t)m, n_entries));
    if (e == cudaSuccess) e = qap_transpose(dm, d->n_vars, n_entries, 0, d->n_vars, (uint32_t)m, R, scratch, st);
    R.n_entries = n_entries;
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(scratch);
    cudaFree(dm);
    if (e != cudaSuccess) return fail(ctx, e, "cs_pk_create: QAP transpose");
  }
  Domain* dom = nullptr;
  if ((e = domain_get(ctx, L + 1, &dom)) != cudaSuccess) return fail(ctx, e, "cs_pk_create: NTT tables");
  if ((e = domain_get(ctx, L, &dom)) != cudaSuccess) return fail(ctx, e, "cs_pk_create: NTT tables");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(ctx, e, "cs_pk_create: sync");
  *out = pk.release();
  return CS_OK;
}

void cs_pk_destroy(cs_pk* pk) { delete pk; }

int cs_pk_fixed_base(cs_ctx* ctx, cs_pk* pk, int window) {
  if (!ctx || !pk || window > 24 || (window > 0 && window < 4)) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  // tables may be read by proofs still in flight on this context
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  for (int i = 0; i < 4 && e == cudaSuccess; i++)
    if (ctx->aux[i]) e = cudaStreamSynchronize(ctx->aux[i]);
  if (e != cudaSuccess) return fail(ctx, e, "cs_pk_fixed_base: sync");
  pk->drop_fixed();
  pk->id = g_pk_ids.fetch_add(1);  // the tables move: graphs captured with the old ones are stale
  if (window < 0) return CS_OK;
  const uint32_t nv = pk->n_vars, np1 = pk->n_public + 1;
  struct Job {
    cs_pk::Fixed* f;
    const uint32_t* pts;
    uint32_t n;
    bool ec2;
  } jobs[5] = {{&pk->fa, pk->a_ext, nv + 2, false},
               {&pk->fb1, pk->b1_ext, nv + 2, false},
               {&pk->fb2, pk->b2_ext, nv + 2, true},
               {&pk->fc, pk->c + (size_t)np1 * 16, nv - np1, false},
               {&pk->fh, pk->h_ext, pk->m, false}};
  size_t total = 0, scratch = 0;
  size_t offs[5];
  for (int k = 0; k < 5; k++) {
    Job& j = jobs[k];
    const int c = window > 0 ? window : msm_fixed_window(j.n, j.ec2);
    offs[k] = total;
    total += al256(msm_fixed_table_points(j.n, c) * (j.ec2 ? 128 : 64));
    const size_t sb = msm_fixed_table_work_bytes(j.n, j.ec2);
    if (sb > scratch) scratch = sb;
    j.f->n = j.n;
    j.f->c = c;
  }
  if ((e = ctx->work.reserve(scratch, ctx->stream)) != cudaSuccess) {
    pk->fa = pk->fb1 = pk->fb2 = pk->fc = pk->fh = cs_pk::Fixed{};
    return fail(ctx, e, "cs_pk_fixed_base: table scratch");
  }
  void* block = nullptr;
  if ((e = cudaMalloc(&block, total)) != cudaSuccess) {
    pk->fa = pk->fb1 = pk->fb2 = pk->fc = pk->fh = cs_pk::Fixed{};
    return fail(ctx, e, "cs_pk_fixed_base: tables");
  }
  pk->fixed_block = block;
  pk->fixed_bytes = total;
  for (int k = 0; k < 5 && e == cudaSuccess; k++) {
    Job& j = jobs[k];
    j.f->table = reinterpret_cast<uint32_t*>(static_cast<char*>(block) + offs[k]);
    e = j.ec2 ? msm_fixed_table_g2(j.pts, j.n, j.f->c, j.f->table, ctx->work.ptr, ctx->work.bytes, ctx->stream)
              : msm_fixed_table_g1(j.pts, j.n, j.f->c, j.f->table, ctx->work.ptr, ctx->work.bytes, ctx->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    pk->drop_fixed();
    return fail(ctx, e, "cs_pk_fixed_base: table build");
  }
  return CS_OK;
}

size_t cs_pk_device_bytes(const cs_pk* pk) { return pk ? pk->base_bytes + pk->fixed_bytes : 0; }

int cs_pk_fixed_window(const cs_pk* pk, int which) {
  if (!pk || !pk->has_fixed() || which < 0 || which > 4) return 0;
  const cs_pk::Fixed* f[5] = {&pk->fa, &pk->fb1, &pk->fb2, &pk->fc, &pk->fh};
  return f[which]->c;
}

size_t cs_prove_workspace_bytes(const cs_pk* pk) { return pk ? plan_prove(pk).total : 0; }

int cs_prove_device(cs_ctx* ctx, cs_pk* pk, const uint32_t* d_w, const uint32_t* r, const uint32_t* s,
                    uint32_t* d_proof) {
  if (!ctx || !pk || !d_w || !r || !s || !d_proof) return CS_ERR_ARG;
  NvtxRange nvtx("cs_prove");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaError_t e = ctx_aux_init(ctx);
  if (e != cudaSuccess) return fail(ctx, e, "prove streams");
  const ProvePlan P = plan_prove(pk);
  if ((e = ctx->work.reserve(P.total, ctx->stream)) != cudaSuccess) return fail(ctx, e, "prove workspace");
  Domain *dom2 = nullptr, *dom1 = nullptr;
  if ((e = domain_get(ctx, pk->log_m + 1, &dom2)) != cudaSuccess || (e = domain_get(ctx, pk->log_m, &dom1)) != cudaSuccess)
    return fail(ctx, e, "prove tables");
  char* base = static_cast<char*>(ctx->work.ptr);
  uint32_t* pts = reinterpret_cast<uint32_t*>(base + P.pts);
  uint32_t *outA = pts, *outB2 = pts + 32, *piC = pts + 160;
  uint32_t* rs = reinterpret_cast<uint32_t*>(base + P.rs);
  cudaStream_t s0 = ctx->stream;
  const GlvSplit glv_rs[2] = {glv_host::split(s), glv_host::split(r)};  // s * pi_A, r * pi_B1
  cudaEventRecord(ctx->ev_start, s0);
  // the call's scalars r, s and their GLV splits go to the device first; everything after
  // them depends only on the key, the witness buffer and the scratch layout
  bool ok = (e = cudaMemcpyAsync(rs, r, 32, cudaMemcpyHostToDevice, s0)) == cudaSuccess &&
            (e = cudaMemcpyAsync(rs + 8, s, 32, cudaMemcpyHostToDevice, s0)) == cudaSuccess &&
            (e = cudaMemcpyAsync(rs + 32, glv_rs, sizeof(glv_rs), cudaMemcpyHostToDevice, s0)) == cudaSuccess;
  if (!ok) return fail(ctx, e, "prove inputs");
  const char* where = "prove launch";
  // Graphs pay where launching is a visible part of a proof (small domains: a 2^12 proof
  // served ~1.45x faster); for large domains they change nothing alone and slowed a served
  // mix of sizes, so those proofs launch directly.
  constexpr uint32_t kGraphMaxDomain = 1u << 17;
  if (!ctx->use_prove_graphs || pk->m > kGraphMaxDomain) {
    e = prove_body(ctx, pk, P, d_w, dom1, dom2, &where);
    ctx->stages_valid = true;
  } else {
    cs_ctx::ProveGraph* g = nullptr;
    for (auto& x : ctx->prove_graphs)
      if (x.pk_id == pk->id && x.d_w == d_w && x.work == ctx->work.ptr && x.work_bytes == ctx->work.bytes)
        g = &x;
    if (g && g->exec) {
      e = cudaGraphLaunch(g->exec, s0);
      note_launch((unsigned)g->launches);
      where = "prove graph launch";
      ctx->stages_valid = false;
    } else if (g) {
      e = prove_body(ctx, pk, P, d_w, dom1, dom2, &where);
      ctx->stages_valid = true;
    } else {
      e = prove_capture(ctx, pk, P, d_w, dom1, dom2, &where);
      ctx->stages_valid = false;
    }
  }
  if (e != cudaSuccess) return fail(ctx, e, where);
  // proof = pi_A (16) | pi_B (32) | pi_C (16), affine Montgomery
  ok = (e = cudaMemcpyAsync(d_proof, outA, 64, cudaMemcpyDeviceToDevice, s0)) == cudaSuccess &&
       (e = cudaMemcpyAsync(d_proof + 16, outB2, 128, cudaMemcpyDeviceToDevice, s0)) == cudaSuccess &&
       (e = cudaMemcpyAsync(d_proof + 48, piC, 64, cudaMemcpyDeviceToDevice, s0)) == cudaSuccess;
  cudaEventRecord(ctx->ev_stop, s0);
  if (!ok) return fail(ctx, e, "prove output");
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(ctx, e, "prove launch");
  return CS_OK;
}

int cs_prove_batch_device(cs_ctx* ctx, cs_pk* pk, uint32_t k, const uint32_t* const* d_w, const uint32_t* r,
                          const uint32_t* s, uint32_t* const* d_proof) {
  if (!ctx || !pk || !d_w || !r || !s || !d_proof || k == 0 || k > 64) return CS_ERR_ARG;
  for (uint32_t i = 0; i < k; i++)
    if (!d_w[i] || !d_proof[i]) return CS_ERR_ARG;
  if (k == 1 || !pk->has_fixed()) {  // nothing to merge: the single-proof path, one by one
    for (uint32_t i = 0; i < k; i++) {
      const int st = cs_prove_device(ctx, pk, d_w[i], r + 8 * (size_t)i, s + 8 * (size_t)i, d_proof[i]);
      if (st != CS_OK) return st;
    }
    return CS_OK;
  }
  NvtxRange nvtx("cs_prove_batch");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaError_t e = ctx_aux_init(ctx);
  if (e != cudaSuccess) return fail(ctx, e, "prove streams");
  Domain *dom2 = nullptr, *dom1 = nullptr;
  if ((e = domain_get(ctx, pk->log_m + 1, &dom2)) != cudaSuccess || (e = domain_get(ctx, pk->log_m, &dom1)) != cudaSuccess)
    return fail(ctx, e, "prove tables");
  ProveBatch* B = nullptr;
  int st = prove_batch_plan(ctx, pk, k, &B);
  if (st != CS_OK) return st;
  // the staging area may still feed the previous batch's upload
  if ((e = cudaEventSynchronize(B->uploaded)) != cudaSuccess) return fail(ctx, e, "prove batch staging");
  BatchCall* hc = static_cast<BatchCall*>(B->host.ptr);
  for (uint32_t i = 0; i < k; i++) {
    BatchCall c{};
    std::memcpy(c.r, r + 8 * (size_t)i, 32);
    std::memcpy(c.s, s + 8 * (size_t)i, 32);
    c.glv[0] = glv_host::split(c.s);
    c.glv[1] = glv_host::split(c.r);
    c.d_w = d_w[i];
    c.d_proof = d_proof[i];
    hc[i] = c;
  }
  cudaStream_t s0 = ctx->stream;
  cudaEventRecord(ctx->ev_start, s0);
  if ((e = cudaMemcpyAsync(B->calls(), hc, sizeof(BatchCall) * k, cudaMemcpyHostToDevice, s0)) != cudaSuccess)
    return fail(ctx, e, "prove batch inputs");
  cudaEventRecord(B->uploaded, s0);
  const char* where = "prove batch launch";
  if (B->exec) {
    e = cudaGraphLaunch(B->exec, s0);
    note_launch((unsigned)B->launches);
  } else if (B->no_graph || !ctx->use_prove_graphs) {
    e = prove_batch_body(ctx, pk, *B, dom1, dom2, &where);
  } else {  // capture the sequence once for this plan and launch it
    const unsigned long long l0 = thread_launches();
    cudaGraph_t graph = nullptr;
    e = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const cudaError_t eb = prove_batch_body(ctx, pk, *B, dom1, dom2, &where);
      e = cudaStreamEndCapture(s0, &graph);
      if (eb != cudaSuccess) e = eb;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&B->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e == cudaSuccess) {
      B->launches = thread_launches() - l0;
      e = cudaGraphLaunch(B->exec, s0);
    } else {
      cudaGetLastError();
      B->exec = nullptr;
      B->no_graph = true;
      e = prove_batch_body(ctx, pk, *B, dom1, dom2, &where);
    }
  }
  ctx->stages_valid = false;
  cudaEventRecord(ctx->ev_stop, s0);
  if (e != cudaSuccess) return fail(ctx, e, where);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(ctx, e, "prove batch launch");
  return CS_OK;
}

int cs_prove(cs_ctx* ctx, cs_pk* pk, const uint32_t* w, const uint32_t* r, const uint32_t* s, uint32_t* proof) {
  if (!ctx || !pk || !w || !proof) return CS_ERR_ARG;
  cudaError_t e;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if ((e = ctx->in.reserve((size_t)pk->n_vars * 32 + 512, ctx->stream)) != cudaSuccess)
      return fail(ctx, e, "prove witness buffer");
    if ((e = cudaMemcpyAsync(ctx->in.ptr, w, (size_t)pk->n_vars * 32, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return fail(ctx, e, "prove witness upload");
  }
  uint32_t* d_w = static_cast<uint32_t*>(ctx->in.ptr);
  uint32_t* d_proof = d_w + (size_t)pk->n_vars * 8;
  int st = cs_prove_device(ctx, pk, d_w, r, s, d_proof);
  if (st != CS_OK) return st;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if ((e = cudaMemcpyAsync(proof, d_proof, 64 * 4, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
    return fail(ctx, e, "prove download");
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail(ctx, e, "prove sync");
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop) == cudaSuccess) ctx->last_ms = ms;
  return CS_OK;
}

}  // extern "C"
