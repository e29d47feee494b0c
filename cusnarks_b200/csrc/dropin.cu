// dropin.cu -- the rest of the reference's host functions the Cython layer binds
// (src/cython/_utils_host.pxd): point utilities of src/cuda/ec.cpp on the GPU, and the
// bookkeeping / file routines of bigint.cpp, ntt.cpp, init.cpp, utils_host.cpp and
// file_utils.cpp on the host.  Same names, arguments and layouts; like the other drop-ins,
// failures are reported by cs_last_status() / cs_last_error() instead of exit().
//
// Point rows: G1 Jacobian 3 x 8 words (X, Y, Z), affine 2 x 8; G2 Jacobian 3 x 16, affine
// 2 x 16; Montgomery form; infinity (0, 1, 0) / (0, 1).  Jacobian results are returned
// normalised (Z = 1), which is the same point as the reference's (x = X/Z^2, y = Y/Z^3).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sys/ipc.h>
#include <sys/shm.h>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cusnarks_b200.h"
#include "ecops.cuh"
#include "runtime.cuh"

namespace csb {
cs_ctx* dropin_ctx(int* status);
void dropin_status(int st, const char* msg);
}  // namespace csb

namespace {

using namespace csb;

// Stages host rows into the context's input arena, runs fn(d_in, d_out) on its stream and
// copies out_words back.  Returns a cs status.
// d_scr: scratch_words of device scratch that overlaps neither input nor output.
template <class Fn>
int run_on_device(const char* what, const uint32_t* in, size_t in_words, uint32_t* out, size_t out_words,
                  size_t scratch_words, Fn fn) {
  int st = CS_OK;
  cs_ctx* ctx = dropin_ctx(&st);
  if (!ctx) return st;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  auto al = [](size_t w) { return (w * 4 + 255) & ~size_t(255); };
  const size_t in_b = al(in_words), out_b = al(out_words);
  cudaError_t e = ctx->in.reserve(in_b + out_b + al(scratch_words), ctx->stream);
  if (e != cudaSuccess) { dropin_status(CS_ERR_NOMEM, what); return CS_ERR_NOMEM; }
  char* base = static_cast<char*>(ctx->in.ptr);
  uint32_t* d_in = reinterpret_cast<uint32_t*>(base);
  uint32_t* d_out = reinterpret_cast<uint32_t*>(base + in_b);
  uint32_t* d_scr = reinterpret_cast<uint32_t*>(base + in_b + out_b);
  if (in_words) e = cudaMemcpyAsync(d_in, in, in_words * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = fn(d_in, d_out, d_scr, ctx->stream);
  if (e == cudaSuccess && out_words) e = cudaMemcpyAsync(out, d_out, out_words * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    const std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    dropin_status(CS_ERR_CUDA, m.c_str());
    return CS_ERR_CUDA;
  }
  dropin_status(CS_OK, "");
  return CS_OK;
}

bool bad_pidx(uint32_t pidx, const char* what) {
  if (pidx == 0) return false;
  dropin_status(CS_ERR_ARG, (std::string(what) + ": points live in MOD_GROUP (pidx 0)").c_str());
  return true;
}

// y (rows of 2 or 3 coordinates) from affine rows in d_aff.
cudaError_t emit_rows(bool ec2, const uint32_t* d_aff, uint32_t n, uint32_t* d_out, bool strip, cudaStream_t st) {
  const size_t fw = ec2 ? 16 : 8;
  if (strip)
    return cudaMemcpyAsync(d_out, d_aff, (size_t)n * 2 * fw * 4, cudaMemcpyDeviceToDevice, st);
  return ec2 ? affine_to_jac_g2(d_aff, n, d_out, st) : affine_to_jac_g1(d_aff, n, d_out, st);
}

void jac2aff(bool ec2, uint32_t* y, const uint32_t* x, uint32_t n, uint32_t pidx, uint32_t strip) {
  if (bad_pidx(pidx, "ec_jac2aff_h")) return;
  const size_t fw = ec2 ? 16 : 8;
  run_on_device("ec_jac2aff_h", x, (size_t)n * 3 * fw, y, (size_t)n * (strip ? 2 : 3) * fw, (size_t)n * 2 * fw,
                [&](uint32_t* d_in, uint32_t* d_out, uint32_t* d_scr, cudaStream_t st) {
                  uint32_t* d_aff = strip ? d_out : d_scr;
                  cudaError_t e = ec2 ? jac_to_affine_g2(d_in, n, d_aff, st) : jac_to_affine_g1(d_in, n, d_aff, st);
                  if (e != cudaSuccess || strip) return e;
                  return emit_rows(ec2, d_aff, n, d_out, false, st);
                });
}

void jacaddreduce(bool ec2, uint32_t* z, const uint32_t* x, uint32_t n, uint32_t pidx, uint32_t to_aff,
                  uint32_t add_in, uint32_t strip) {
  if (bad_pidx(pidx, "ec_jacaddreduce_h")) return;
  (void)to_aff;  // affine and Z = 1 Jacobian rows coincide
  const size_t fw = ec2 ? 16 : 8;
  const int dims = add_in ? 2 : 3;
  run_on_device("ec_jacaddreduce_h", x, (size_t)n * dims * fw, z, (strip ? 2 : 3) * fw, 2 * fw,
                [&](uint32_t* d_in, uint32_t* d_out, uint32_t* d_aff, cudaStream_t st) {
                  cudaError_t e = ec2 ? point_sum_g2(d_in, n, dims, d_aff, st) : point_sum_g1(d_in, n, dims, d_aff, st);
                  if (e != cudaSuccess) return e;
                  return emit_rows(ec2, d_aff, 1, d_out, strip != 0, st);
                });
}

// z[i] = scl[i] * P_i: P_i rows of 3 (Jacobian) or 2 (add_last: affine) coordinates,
// stride 0 = one shared point (the sc1mul form).
void jacscmul(bool ec2, uint32_t* z, const uint32_t* scl, const uint32_t* x, uint32_t n, uint32_t add_last,
              bool shared_point) {
  const size_t fw = ec2 ? 16 : 8;
  const uint32_t dims = add_last ? 2 : 3;
  const uint32_t npts = shared_point ? 1u : n;
  // input: scalars (n x 8) then points (npts x dims x fw)
  std::vector<uint32_t> in((size_t)n * 8 + (size_t)npts * dims * fw);
  std::memcpy(in.data(), scl, (size_t)n * 32);
  std::memcpy(in.data() + (size_t)n * 8, x, (size_t)npts * dims * fw * 4);
  // scratch: npts affine bases, then n affine products
  run_on_device("ec_jacscmul_h", in.data(), in.size(), z, (size_t)n * 3 * fw, ((size_t)npts + n) * 2 * fw,
                [&](uint32_t* d_in, uint32_t* d_out, uint32_t* d_scr, cudaStream_t st) {
                  const uint32_t* d_s = d_in;
                  uint32_t* d_p = d_in + (size_t)n * 8;
                  uint32_t* d_base = d_p;
                  cudaError_t e = cudaSuccess;
                  if (!add_last) {  // Jacobian bases -> affine
                    d_base = d_scr;
                    e = ec2 ? jac_to_affine_g2(d_p, npts, d_base, st) : jac_to_affine_g1(d_p, npts, d_base, st);
                  }
                  if (e != cudaSuccess) return e;
                  uint32_t* d_aff = d_scr + (size_t)npts * 2 * fw;
                  const uint32_t stride = shared_point ? 0u : (uint32_t)(2 * fw);
                  e = ec2 ? scmul_g2(d_s, d_base, stride, n, d_aff, st) : scmul_g1(d_s, d_base, stride, n, d_aff, st);
                  if (e != cudaSuccess) return e;
                  return ec2 ? affine_to_jac_g2(d_aff, n, d_out, st) : affine_to_jac_g1(d_aff, n, d_out, st);
                });
}

// ectable <- ceil(n / order) subset-sum tables of 2^order Jacobian rows (Z = 1; infinity
// (0, 1, 0)): rows of x are affine (add_last) or Jacobian points.
void inittable(bool ec2, const uint32_t* x, uint32_t* ectable, uint32_t n, uint32_t order, uint32_t pidx,
               uint32_t add_last) {
  const char* what = ec2 ? "ec2_inittable_h" : "ec_inittable_h";
  if (bad_pidx(pidx, what)) return;
  if (order == 0 || order > 16) {
    dropin_status(CS_ERR_ARG, (std::string(what) + ": table_order must be 1..16").c_str());
    return;
  }
  const size_t fw = ec2 ? 16 : 8;
  const uint32_t dims = add_last ? 2 : 3;
  const size_t entries = (((size_t)n + order - 1) / order) << order;
  // scratch: n affine points, then the affine table
  run_on_device(what, x, (size_t)n * dims * fw, ectable, entries * 3 * fw, ((size_t)n + entries) * 2 * fw,
                [&](uint32_t* d_in, uint32_t* d_out, uint32_t* d_scr, cudaStream_t st) {
                  const uint32_t* d_aff = d_in;
                  cudaError_t e = cudaSuccess;
                  if (!add_last) {
                    e = ec2 ? jac_to_affine_g2(d_in, n, d_scr, st) : jac_to_affine_g1(d_in, n, d_scr, st);
                    d_aff = d_scr;
                  }
                  if (e != cudaSuccess) return e;
                  uint32_t* d_tab = d_scr + (size_t)n * 2 * fw;
                  e = ec2 ? subset_table_g2(d_aff, n, order, d_tab, st) : subset_table_g1(d_aff, n, order, d_tab, st);
                  if (e != cudaSuccess) return e;
                  return ec2 ? affine_to_jac_g2(d_tab, (uint32_t)entries, d_out, st)
                             : affine_to_jac_g1(d_tab, (uint32_t)entries, d_out, st);
                });
}

uint32_t isoncurve(bool ec2, const uint32_t* x, uint32_t is_affine, uint32_t pidx) {
  if (bad_pidx(pidx, "ec_isoncurve_h")) return 0;
  const size_t fw = ec2 ? 16 : 8;
  uint32_t flag = 0;
  run_on_device("ec_isoncurve_h", x, (is_affine ? 2 : 3) * fw, &flag, 1, 0,
                [&](uint32_t* d_in, uint32_t* d_out, uint32_t*, cudaStream_t st) {
                  return ec2 ? on_curve_g2(d_in, is_affine ? 0 : 1, d_out, st)
                             : on_curve_g1(d_in, is_affine ? 0 : 1, d_out, st);
                });
  return flag;
}

}  // namespace

extern "C" {

void ec_jac2aff_h(uint32_t* y, uint32_t* x, uint32_t n, uint32_t pidx, uint32_t strip_last) {
  jac2aff(false, y, x, n, pidx, strip_last);
}
void ec2_jac2aff_h(uint32_t* y, uint32_t* x, uint32_t n, uint32_t pidx, uint32_t strip_last) {
  jac2aff(true, y, x, n, pidx, strip_last);
}
void ec_jacaddreduce_h(uint32_t* z, uint32_t* x, uint32_t n, uint32_t pidx, uint32_t to_aff, uint32_t add_in,
                       uint32_t strip_last) {
  jacaddreduce(false, z, x, n, pidx, to_aff, add_in, strip_last);
}
void ec2_jacaddreduce_h(uint32_t* z, uint32_t* x, uint32_t n, uint32_t pidx, uint32_t to_aff, uint32_t add_in,
                        uint32_t strip_last) {
  jacaddreduce(true, z, x, n, pidx, to_aff, add_in, strip_last);
}
void ec_jacscmul_h(uint32_t* z, uint32_t* scl, uint32_t* x, uint32_t n, uint32_t pidx, uint32_t add_last) {
  if (bad_pidx(pidx, "ec_jacscmul_h")) return;
  jacscmul(false, z, scl, x, n, add_last, false);
}
void ec2_jacscmul_h(uint32_t* z, uint32_t* scl, uint32_t* x, uint32_t n, uint32_t pidx, uint32_t add_last) {
  if (bad_pidx(pidx, "ec2_jacscmul_h")) return;
  jacscmul(true, z, scl, x, n, add_last, false);
}
// x = n scalars followed by one base point (ec.cpp:819)
void ec_jacsc1mul_h(uint32_t* z, uint32_t* x, uint32_t n, uint32_t pidx, uint32_t add_last) {
  if (bad_pidx(pidx, "ec_jacsc1mul_h")) return;
  jacscmul(false, z, x, x + (size_t)n * 8, n, add_last, true);
}
void ec2_jacsc1mul_h(uint32_t* z, uint32_t* x, uint32_t n, uint32_t pidx, uint32_t add_last) {
  if (bad_pidx(pidx, "ec2_jacsc1mul_h")) return;
  jacscmul(true, z, x, x + (size_t)n * 8, n, add_last, true);
}
uint32_t ec_isoncurve_h(uint32_t* x, uint32_t is_affine, uint32_t pidx) { return isoncurve(false, x, is_affine, pidx); }
uint32_t ec2_isoncurve_h(uint32_t* x, uint32_t is_affine, uint32_t pidx) { return isoncurve(true, x, is_affine, pidx); }
// ec.cpp:131 / :462 (and the G2 forms): one Jacobian addition / doubling, the result
// normalised (Z = 1; infinity (0, 1, 0)) -- the same point as the reference's.
static void jacadd2(bool ec2, uint32_t* z, const uint32_t* x, const uint32_t* y, uint32_t pidx, const char* what) {
  if (bad_pidx(pidx, what)) return;
  const size_t fw = ec2 ? 16 : 8;
  std::vector<uint32_t> in(6 * fw);
  std::memcpy(in.data(), x, 3 * fw * 4);
  std::memcpy(in.data() + 3 * fw, y, 3 * fw * 4);
  run_on_device(what, in.data(), in.size(), z, 3 * fw, 2 * fw,
                [&](uint32_t* d_in, uint32_t* d_out, uint32_t* d_aff, cudaStream_t st) {
                  cudaError_t e = ec2 ? point_sum_g2(d_in, 2, 3, d_aff, st) : point_sum_g1(d_in, 2, 3, d_aff, st);
                  if (e != cudaSuccess) return e;
                  return emit_rows(ec2, d_aff, 1, d_out, false, st);
                });
}
void ec_jacadd_h(uint32_t* z, uint32_t* x, uint32_t* y, uint32_t pidx) { jacadd2(false, z, x, y, pidx, "ec_jacadd_h"); }
void ec2_jacadd_h(uint32_t* z, uint32_t* x, uint32_t* y, uint32_t pidx) { jacadd2(true, z, x, y, pidx, "ec2_jacadd_h"); }
void ec_jacdouble_h(uint32_t* z, uint32_t* x, uint32_t pidx) { jacadd2(false, z, x, x, pidx, "ec_jacdouble_h"); }
void ec2_jacdouble_h(uint32_t* z, uint32_t* x, uint32_t pidx) { jacadd2(true, z, x, x, pidx, "ec2_jacdouble_h"); }

// mpoly.cpp:266 / :278: the coefficient values of an mpoly (layout mpoly.cpp:195) to or from
// Montgomery form, in place: gathered into one array, converted on the GPU, scattered back.
static void mpoly_convert(uint32_t* x, uint32_t pidx, bool to_mont) {
  std::vector<size_t> blocks;  // (offset, count) pairs
  size_t total = 0;
  size_t off = 1 + (size_t)x[0];
  for (uint32_t i = 0; i < x[0]; i++) {
    const uint32_t c = x[i + 1];
    off += c;  // the constraint indices
    blocks.push_back(off);
    blocks.push_back(c);
    total += c;
    off += (size_t)c * 8;
  }
  std::vector<uint32_t> vals(total * 8);
  size_t k = 0;
  for (size_t b = 0; b < blocks.size(); b += 2) {
    std::memcpy(&vals[k * 8], x + blocks[b], blocks[b + 1] * 32);
    k += blocks[b + 1];
  }
  if (total) {
    if (to_mont) to_montgomeryN_h(vals.data(), vals.data(), (uint32_t)total, pidx);
    else from_montgomeryN_h(vals.data(), vals.data(), (uint32_t)total, pidx, 0);
    if (cs_field_last_status() != CS_OK) {
      dropin_status(cs_field_last_status(), to_mont ? "mpoly_to_montgomery_h" : "mpoly_from_montgomery_h");
      return;
    }
  }
  k = 0;
  for (size_t b = 0; b < blocks.size(); b += 2) {
    std::memcpy(x + blocks[b], &vals[k * 8], blocks[b + 1] * 32);
    k += blocks[b + 1];
  }
  dropin_status(CS_OK, "");
}
void mpoly_to_montgomery_h(uint32_t* x, uint32_t pidx) { mpoly_convert(x, pidx, true); }
void mpoly_from_montgomery_h(uint32_t* x, uint32_t pidx) { mpoly_convert(x, pidx, false); }

// bigint.cpp / ff.cpp:626: U = A + B mod 2^256; samples[i] = start + i inc, reduced below mod
// (when given) by repeated subtraction, as the reference does.
void addu256_h(uint32_t* U, const uint32_t* A, const uint32_t* B) {
  uint64_t c = 0;
  for (int i = 0; i < 8; i++) {
    c += (uint64_t)A[i] + B[i];
    U[i] = (uint32_t)c;
    c >>= 32;
  }
}
static bool geq256(const uint32_t* a, const uint32_t* b) {
  for (int i = 7; i >= 0; i--)
    if (a[i] != b[i]) return a[i] > b[i];
  return true;
}
void rangeu256_h(uint32_t* samples, uint32_t nsamples, const uint32_t* start, uint32_t inc, const uint32_t* mod) {
  if (nsamples == 0) return;
  const uint32_t step[8] = {inc, 0, 0, 0, 0, 0, 0, 0};
  std::memcpy(samples, start, 32);
  for (uint32_t i = 1; i < nsamples; i++) {
    uint32_t* s = samples + (size_t)i * 8;
    addu256_h(s, samples + (size_t)(i - 1) * 8, step);
    while (mod && geq256(s, mod)) {
      int64_t br = 0;
      for (int k = 0; k < 8; k++) {
        br += (int64_t)s[k] - mod[k];
        s[k] = (uint32_t)br;
        br >>= 32;
      }
    }
  }
}

void ec_inittable_h(uint32_t* x, uint32_t* ectable, uint32_t n, uint32_t table_order, uint32_t pidx,
                    uint32_t add_last) {
  inittable(false, x, ectable, n, table_order, pidx, add_last);
}
void ec2_inittable_h(uint32_t* x, uint32_t* ectable, uint32_t n, uint32_t table_order, uint32_t pidx,
                     uint32_t add_last) {
  inittable(true, x, ectable, n, table_order, pidx, add_last);
}

// ec.cpp:1153 / :1164, as the reference computes them: z[j] is the infinity test (first two
// coordinates equal to the affine infinity's, (0, 1_mont) in G1 with the Montgomery one of
// modulus pidx, X = 0 in G2) of the rows the reference reads, which start 2 j words into x
// in G1 (it steps by the coordinate count) and 4 words into x for every j in G2.
void ec_isinf(uint32_t* z, const uint32_t* x, const uint32_t n, const uint32_t pidx) {
  // the Montgomery one of the modulus pidx selects (constants.cpp:264-292)
  static const uint32_t ones[2][8] = {{0xc58f0d9du, 0xd35d438du, 0xf5c70b3du, 0x0a78eb28u,
                                       0x7879462cu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u},
                                      {0x4ffffffbu, 0xac96341cu, 0x9f60cd29u, 0x36fc7695u,
                                       0x7879462eu, 0x666ea36fu, 0x9a07df2fu, 0x0e0a77c1u}};
  if (pidx > 1) {
    dropin_status(CS_ERR_ARG, "ec_isinf: pidx must be 0 or 1");
    return;
  }
  const uint32_t* one = ones[pidx];
  for (uint32_t j = 0; j < n; j++) {
    const uint32_t* r = x + (size_t)j * 2;
    bool inf = true;
    for (int k = 0; k < 8; k++) inf = inf && r[k] == 0 && r[8 + k] == one[k];
    z[j] = inf ? 1u : 0u;
  }
  dropin_status(CS_OK, "");
}
void ec2_isinf(uint32_t* z, const uint32_t* x, const uint32_t n, const uint32_t pidx) {
  if (pidx > 1) {
    dropin_status(CS_ERR_ARG, "ec2_isinf: pidx must be 0 or 1");
    return;
  }
  bool inf = true;
  for (int k = 0; k < 16; k++) inf = inf && x[4 + k] == 0;
  for (uint32_t j = 0; j < n; j++) z[j] = inf ? 1u : 0u;
  dropin_status(CS_OK, "");
}

// ------------------------------------------------------------------ host routines ----
// bigint.cpp:72: idx = 0..len-1, sorted (std::sort, unstable) by the most significant word
// of v[idx] when sort_en.
void sortu256_idx_h(uint32_t* idx, const uint32_t* v, uint32_t len, uint32_t sort_en) {
  for (uint32_t i = 0; i < len; i++) idx[i] = i;
  if (sort_en)
    std::sort(idx, idx + len, [v](uint32_t a, uint32_t b) { return v[(size_t)a * 8 + 7] < v[(size_t)b * 8 + 7]; });
}

// ntt.cpp:1116: transform decomposition parameters for nsamples (the prover reads levels
// and fft_N to size its roots tables).
void ntt_build_h(fft_params_t* p, uint32_t nsamples) {
  const uint32_t min_samples = 1u << 6;
  const uint32_t ns = std::max(nsamples, min_samples);
  uint32_t levels = (uint32_t)std::ceil(std::log2((double)ns));
  std::memset(p, 0, sizeof(fft_params_t));
  p->padding = (1u << levels) - nsamples;
  p->levels = levels;
  if (ns <= 32) {
    p->fft_type = FFT_T_1D;
    p->fft_N[0] = levels;
  } else if (ns <= (1u << 20)) {
    p->fft_type = FFT_T_3D;
    p->fft_N[3] = levels / 2;
    p->fft_N[2] = levels - levels / 2;
    p->fft_N[1] = levels / 4;
    p->fft_N[0] = (levels - levels / 2) / 2;
  } else {
    p->fft_type = FFT_T_4D;
    p->fft_N[7] = levels / 2;
    p->fft_N[6] = levels - levels / 2;
    p->fft_N[5] = levels / 4;
    p->fft_N[4] = (levels - levels / 2) / 2;
    levels = p->fft_N[7];
    p->fft_N[3] = levels / 2;
    p->fft_N[2] = levels - levels / 2;
    p->fft_N[1] = levels / 4;
    p->fft_N[0] = (levels - levels / 2) / 2;
  }
}

uint32_t get_nprocs_h(void) {
  const unsigned n = std::thread::hardware_concurrency();
  return n ? n : 1;
}

// init.cpp:44 / :54.  Nothing to load here (no roots files: twiddles are computed on the
// device when first needed); init_h creates the current device's default context early,
// release_h synchronises it.
void init_h(void) {
  int st = CS_OK;
  dropin_ctx(&st);
}
void release_h(void) {
  int st = CS_OK;
  cs_ctx* ctx = dropin_ctx(&st);
  if (ctx) cs_ctx_sync(ctx);
}

// file_utils.cpp routines (raw little-endian uint32 words).
void readU256CircuitFile_h(uint32_t* samples, const char* filename, unsigned long long nwords) {
  FILE* f = std::fopen(filename, "rb");
  if (!f) { dropin_status(CS_ERR_ARG, "readU256CircuitFile_h: cannot open file"); return; }
  if (nwords) {
    if (std::fread(samples, 4, nwords, f) != nwords) dropin_status(CS_ERR_ARG, "readU256CircuitFile_h: short file");
  } else {
    size_t i = 0;
    while (std::fread(&samples[i], 4, 1, f) == 1) i++;
  }
  std::fclose(f);
}
// file_utils.cpp:49 / :447: the first header words of a circuit / proving-key file (the
// proving-key reader takes the nine leading words in order, so its domainSize field holds
// the file's domainBits word, as the reference's does).
void readU256CircuitFileHeader_h(cirbin_hfile_t* h, const char* filename) {
  FILE* f = std::fopen(filename, "rb");
  if (!f) { dropin_status(CS_ERR_ARG, "readU256CircuitFileHeader_h: cannot open file"); return; }
  unsigned long long w[9] = {0};
  const size_t got = std::fread(w, sizeof(unsigned long long), 9, f);
  std::fclose(f);
  h->nWords = w[0]; h->nPubInputs = w[1]; h->nOutputs = w[2]; h->nVars = w[3]; h->nConstraints = w[4];
  h->cirformat = w[5]; h->R1CSA_nWords = w[6]; h->R1CSB_nWords = w[7]; h->R1CSC_nWords = w[8];
  dropin_status(got == 9 ? CS_OK : CS_ERR_ARG, got == 9 ? "" : "readU256CircuitFileHeader_h: short file");
}
void readU256PKFileHeader_h(pkbin_hfile_t* h, const char* filename) {
  FILE* f = std::fopen(filename, "rb");
  if (!f) { dropin_status(CS_ERR_ARG, "readU256PKFileHeader_h: cannot open file"); return; }
  uint32_t w[9] = {0};
  const size_t got = std::fread(w, 4, 9, f);
  std::fclose(f);
  h->nWords = w[0]; h->ftype = w[1]; h->protocol = w[2]; h->Rbitlen = w[3]; h->k_binformat = w[4];
  h->k_ecformat = w[5]; h->nVars = w[6]; h->nPublic = w[7]; h->domainSize = w[8];
  dropin_status(got == 9 ? CS_OK : CS_ERR_ARG, got == 9 ? "" : "readU256PKFileHeader_h: short file");
}
void readU256PKFile_h(uint32_t* samples, const char* filename, unsigned long long nwords) {
  readU256CircuitFile_h(samples, filename, nwords);
}
// insize 256-bit elements in the file; every (insize/outsize)-th is kept
void readU256DataFile_h(uint32_t* samples, const char* filename, uint32_t insize, uint32_t outsize) {
  FILE* f = std::fopen(filename, "rb");
  if (!f) { dropin_status(CS_ERR_ARG, "readU256DataFile_h: cannot open file"); return; }
  const uint32_t count = outsize ? insize / outsize : 1;
  if (count != 1) {
    uint32_t r[8];
    uint32_t k = 0;
    for (uint32_t i = 0; i < insize; i++) {
      if (std::fread(r, 4, 8, f) != 8) break;
      if (i % count == 0) std::memcpy(&samples[(size_t)k++ * 8], r, 32);
    }
  } else if (std::fread(samples, 32, outsize, f) != outsize) {
    dropin_status(CS_ERR_ARG, "readU256DataFile_h: short file");
  }
  std::fclose(f);
}
void readU256DataFileFromOffset_h(uint32_t* samples, const char* filename, unsigned long long woffset,
                                  unsigned long long nwords) {
  FILE* f = std::fopen(filename, "rb");
  if (!f) { dropin_status(CS_ERR_ARG, "readU256DataFileFromOffset_h: cannot open file"); return; }
  if (std::fseek(f, (long)(woffset * 4), SEEK_SET) != 0 || std::fread(samples, 4, nwords, f) != nwords)
    dropin_status(CS_ERR_ARG, "readU256DataFileFromOffset_h: short file");
  std::fclose(f);
}
void writeU256DataFile_h(uint32_t* samples, const char* filename, unsigned long long nwords) {
  FILE* f = std::fopen(filename, "wb");
  if (!f) { dropin_status(CS_ERR_ARG, "writeU256DataFile_h: cannot open file"); return; }
  std::fwrite(samples, 4, nwords, f);
  std::fclose(f);
}
void appendU256DataFile_h(uint32_t* samples, const char* filename, unsigned long long nwords) {
  FILE* f = std::fopen(filename, "ab");
  if (!f) { dropin_status(CS_ERR_ARG, "appendU256DataFile_h: cannot open file"); return; }
  std::fwrite(samples, 4, nwords, f);
  std::fclose(f);
}
// witness .bin (fmt 1: values after the 4-word header) / .dat (fmt 0: values from byte 32)
void readWitnessFile_h(uint32_t* samples, const char* filename, uint32_t fmt, unsigned long long inlen) {
  FILE* f = std::fopen(filename, "rb");
  if (!f) { dropin_status(CS_ERR_ARG, "readWitnessFile_h: cannot open file"); return; }
  if (std::fseek(f, fmt ? 16 : 32, SEEK_SET) != 0 || std::fread(samples, 32, inlen, f) != inlen)
    dropin_status(CS_ERR_ARG, "readWitnessFile_h: short file");
  std::fclose(f);
}
void writeWitnessFile_h(uint32_t* samples, const char* filename, unsigned long long nwords) {
  FILE* f = std::fopen(filename, "wb");
  if (!f) { dropin_status(CS_ERR_ARG, "writeWitnessFile_h: cannot open file"); return; }
  const uint64_t n = nwords;
  const uint32_t wsize = 8, wmore = 0;
  std::fwrite(&n, 8, 1, f);
  std::fwrite(&wsize, 4, 1, f);
  std::fwrite(&wmore, 4, 1, f);
  std::fwrite(samples, 32, nwords, f);
  std::fclose(f);
}

// System V shared memory for the witness, as the reference's processes share it
// (utils_host.cpp:156 / :180: key 123456, created if absent, mode 0666).
int shared_new_h(void** shmem, unsigned long long size) {
  if (!shmem) return -1;
  const int shmid = shmget((key_t)123456, (size_t)size, IPC_CREAT | 0666);
  if (shmid < 0) return -1;
  void* p = shmat(shmid, nullptr, 0);
  if (p == (void*)-1) return -1;
  *shmem = p;
  return shmid;
}

void shared_free_h(void* shmem, int shmid) {
  if (shmem) shmdt(shmem);
  shmctl(shmid, IPC_RMID, nullptr);
}

// Circuit compilation and EC table files: bound by the reference's Cython layer, not on this
// library's path.  Outputs are zeroed; the status says why.
void readR1CSFileHeader_h(r1csv1_t* r1cs_hdr, const char* filename) {
  if (r1cs_hdr) memset(r1cs_hdr, 0, sizeof(*r1cs_hdr));
  dropin_status(CS_ERR_UNSUPPORTED, "readR1CSFileHeader_h: R1CS files are compiled before proving (not on this path)");
}
void readR1CSFile_h(uint32_t*, const char*, r1csv1_t*, r1cs_idx_t) {
  dropin_status(CS_ERR_UNSUPPORTED, "readR1CSFile_h: R1CS files are compiled before proving (not on this path)");
}
void r1cs_to_mpoly_len_h(uint32_t*, uint32_t*, cirbin_hfile_t*, uint32_t) {
  dropin_status(CS_ERR_UNSUPPORTED, "r1cs_to_mpoly_len_h: circuit compilation is not on this path");
}
void r1cs_to_mpoly_h(uint32_t*, uint32_t*, cirbin_hfile_t*, uint32_t, uint32_t, uint32_t) {
  dropin_status(CS_ERR_UNSUPPORTED, "r1cs_to_mpoly_h: circuit compilation is not on this path");
}
void readECTablesNElementsFile_h(ec_table_offset_t* t, const char*) {
  if (t) memset(t, 0, sizeof(*t));
  dropin_status(CS_ERR_UNSUPPORTED, "readECTablesNElementsFile_h: precomputed EC table files are not supported");
}

}  // extern "C"
