// qap.cu -- transpose of the reference mpoly layout into constraint rows, and the
// row-parallel QAP evaluation (qap.cuh); drop-in mpoly_eval_server_h / mpoly_eval_h.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cusnarks_b200.h"
#include "curve.cuh"
#include "qap.cuh"
#include "runtime.cuh"
#include "scan.cuh"

namespace csb {

namespace {

inline size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

__global__ void k_wire_counts(const uint32_t* __restrict__ mpoly, uint32_t n_wires, uint32_t* __restrict__ cnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_wires) cnt[i] = mpoly[1 + i];
  if (i == n_wires) cnt[i] = 0;
}

// entry e -> (wire, k): binary search in the exclusive scan of per-wire counts
CSB_DEV uint32_t find_wire(const uint32_t* __restrict__ start, uint32_t n_wires, uint32_t e) {
  uint32_t lo = 0, hi = n_wires;  // start[lo] <= e < start[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (start[mid] <= e) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void k_row_counts(const uint32_t* __restrict__ mpoly, uint32_t n_wires, const uint32_t* __restrict__ start,
                             uint32_t n_entries, uint32_t wire_lo, uint32_t wire_hi, uint32_t n_rows,
                             uint32_t* __restrict__ row_cnt) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_entries) return;
  const uint32_t i = find_wire(start, n_wires, e);
  if (i < wire_lo || i >= wire_hi) return;
  const uint32_t k = e - start[i];
  const uint64_t block = 1ull + n_wires + 9ull * start[i];
  const uint32_t c = mpoly[block + k];
  if (c < n_rows) atomicAdd(&row_cnt[c], 1u);
}

__global__ void k_row_scatter(const uint32_t* __restrict__ mpoly, uint32_t n_wires, const uint32_t* __restrict__ start,
                              uint32_t n_entries, uint32_t wire_lo, uint32_t wire_hi, uint32_t n_rows,
                              uint32_t* __restrict__ cursor, uint32_t* __restrict__ wire_out,
                              uint32_t* __restrict__ coeff_out) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_entries) return;
  const uint32_t i = find_wire(start, n_wires, e);
  if (i < wire_lo || i >= wire_hi) return;
  const uint32_t k = e - start[i];
  const uint32_t nc = start[i + 1] - start[i];
  const uint64_t block = 1ull + n_wires + 9ull * start[i];
  const uint32_t c = mpoly[block + k];
  if (c >= n_rows) return;
  const uint32_t pos = atomicAdd(&cursor[c], 1u);
  wire_out[pos] = i;
  // coefficient words are 4-byte aligned only: scalar loads
  Fr v;
  const uint32_t* src = mpoly + block + nc + 8ull * k;
#pragma unroll
  for (int w = 0; w < 8; w++) v.v[w] = src[w];
  st_fp<ModR>(coeff_out + (size_t)pos * 8, v * Fr::r2());
}

__global__ void k_qap_eval(const uint32_t* __restrict__ row_off, const uint32_t* __restrict__ wire,
                           const uint32_t* __restrict__ coeff, const uint32_t* __restrict__ w, uint32_t n_rows,
                           int accumulate, uint32_t* __restrict__ out, size_t stride) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_rows) return;
  w += (size_t)blockIdx.y * stride;  // instance y of a batch
  out += (size_t)blockIdx.y * stride;
  Fr acc = accumulate ? ld_fp<ModR>(out + (size_t)c * 8) : Fr::zero();
  const uint32_t b = row_off[c], e = row_off[c + 1];
  for (uint32_t k = b; k < e; k++) acc = acc + ld_fp<ModR>(coeff + (size_t)k * 8) * ld_fp<ModR>(w + (size_t)wire[k] * 8);
  st_fp<ModR>(out + (size_t)c * 8, acc);
}

}  // namespace

size_t qap_transpose_scratch_bytes(uint32_t n_wires, uint32_t n_rows, uint32_t n_entries) {
  (void)n_entries;
  return al256((size_t)(n_wires + 1) * 4) * 2 + al256((size_t)(n_rows + 1) * 4) * 2 +
         scan_workspace_bytes((size_t)(n_wires > n_rows ? n_wires : n_rows) + 1) + 256;
}

cudaError_t qap_transpose(const uint32_t* d_mpoly, uint32_t n_wires, uint32_t n_entries, uint32_t wire_lo,
                          uint32_t wire_hi, uint32_t n_rows, QapRows& rows, void* scratch, cudaStream_t st) {
  char* p = static_cast<char*>(scratch);
  uint32_t* wcnt = reinterpret_cast<uint32_t*>(p);  p += al256((size_t)(n_wires + 1) * 4);
  uint32_t* wstart = reinterpret_cast<uint32_t*>(p); p += al256((size_t)(n_wires + 1) * 4);
  uint32_t* rcnt = reinterpret_cast<uint32_t*>(p);  p += al256((size_t)(n_rows + 1) * 4);
  uint32_t* cursor = reinterpret_cast<uint32_t*>(p); p += al256((size_t)(n_rows + 1) * 4);
  void* scan_tmp = p;
  cudaError_t e;
  k_wire_counts<<<(n_wires + 256) / 256, 256, 0, st>>>(d_mpoly, n_wires, wcnt);
  note_launch();
  if ((e = scan_exclusive_u32(wcnt, wstart, (size_t)n_wires + 1, scan_tmp, st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(rcnt, 0, (size_t)(n_rows + 1) * 4, st)) != cudaSuccess) return e;
  if (n_entries) {
    k_row_counts<<<(n_entries + 255) / 256, 256, 0, st>>>(d_mpoly, n_wires, wstart, n_entries, wire_lo, wire_hi,
                                                            n_rows, rcnt);
    note_launch();
  }
  if ((e = scan_exclusive_u32(rcnt, rows.row_off, (size_t)n_rows + 1, scan_tmp, st)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(cursor, rows.row_off, (size_t)n_rows * 4, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
    return e;
  if (n_entries) {
    k_row_scatter<<<(n_entries + 255) / 256, 256, 0, st>>>(d_mpoly, n_wires, wstart, n_entries, wire_lo, wire_hi,
                                                             n_rows, cursor, rows.wire, rows.coeff);
    note_launch();
  }
  rows.n_rows = n_rows;
  return cudaGetLastError();
}

cudaError_t qap_eval(const QapRows& rows, const uint32_t* d_w, uint32_t* d_out, int accumulate, cudaStream_t st,
                     uint32_t batch, size_t stride) {
  if (rows.n_rows == 0 || batch == 0) return cudaSuccess;
  if (batch > 65535) return cudaErrorInvalidValue;
  k_qap_eval<<<dim3((rows.n_rows + 255) / 256, batch), 256, 0, st>>>(rows.row_off, rows.wire, rows.coeff, d_w,
                                                                      rows.n_rows, accumulate, d_out, stride);
  note_launch();
  return cudaGetLastError();
}

}  // namespace csb

using namespace csb;

namespace {
thread_local int t_qap_status = CS_OK;

cs_ctx* qap_default_ctx() {
  static std::mutex mu;
  static cs_ctx* ctxs[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { cudaGetLastError(); return nullptr; }
  std::lock_guard<std::mutex> lk(mu);
  if (!ctxs[dev] && cs_ctx_create(dev, &ctxs[dev]) != CS_OK) return nullptr;
  return ctxs[dev];
}

// Words of a reference mpoly, read from its header counts.
size_t mpoly_words(const uint32_t* pin, uint32_t* n_entries) {
  const uint32_t n = pin[0];
  uint64_t e = 0;
  for (uint32_t i = 0; i < n; i++) e += pin[1 + i];
  *n_entries = (uint32_t)e;
  return 1 + (size_t)n + 9 * (size_t)e;
}
}  // namespace

extern "C" {

int cs_qap_last_status(void) { return t_qap_status; }

// pout has ncoeff = n_rows rows; the reference's caller sizes it by the domain.  The
// reference does not pass that size, so the rows touched are bounded by the largest
// constraint index present (scanned on the host from the mpoly's index words).
void mpoly_eval_server_h(mpoly_eval_t* args) {
  if (!args || !args->pout || !args->scalar || !args->pin || args->pidx != 1) {
    t_qap_status = CS_ERR_ARG;
    return;
  }
  cs_ctx* ctx = qap_default_ctx();
  if (!ctx) { t_qap_status = CS_ERR_NODEVICE; return; }
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  const uint32_t* pin = args->pin;
  const uint32_t n_wires = pin[0];
  uint32_t n_entries = 0;
  const size_t words = mpoly_words(pin, &n_entries);
  // highest constraint index referenced -> rows of pout in use
  uint32_t n_rows = 0;
  {
    uint64_t off = 1 + (uint64_t)n_wires;
    for (uint32_t i = 0; i < n_wires; i++) {
      const uint32_t nc = pin[1 + i];
      if (i >= args->start_idx && i < args->last_idx)
        for (uint32_t k = 0; k < nc; k++) n_rows = pin[off + k] + 1 > n_rows ? pin[off + k] + 1 : n_rows;
      off += 9ull * nc;
    }
  }
  const uint32_t lo = args->start_idx, hi = args->last_idx > n_wires ? n_wires : args->last_idx;
  const size_t wbytes = (size_t)n_wires * 32, mbytes = words * 4, obytes = (size_t)n_rows * 32;
  const size_t need = al256(mbytes) + al256(wbytes) + al256(obytes) + al256((size_t)(n_rows + 1) * 4) +
                      al256((size_t)n_entries * 4) + al256((size_t)n_entries * 32) +
                      qap_transpose_scratch_bytes(n_wires, n_rows, n_entries) + 1024;
  cudaError_t e = ctx->in.reserve(need, ctx->stream);
  if (e != cudaSuccess) { t_qap_status = fail(ctx, e, "mpoly buffers"); return; }
  char* p = static_cast<char*>(ctx->in.ptr);
  uint32_t* dm = reinterpret_cast<uint32_t*>(p); p += al256(mbytes);
  uint32_t* dw = reinterpret_cast<uint32_t*>(p); p += al256(wbytes);
  uint32_t* dout = reinterpret_cast<uint32_t*>(p); p += al256(obytes);
  QapRows rows;
  rows.row_off = reinterpret_cast<uint32_t*>(p); p += al256((size_t)(n_rows + 1) * 4);
  rows.wire = reinterpret_cast<uint32_t*>(p); p += al256((size_t)n_entries * 4);
  rows.coeff = reinterpret_cast<uint32_t*>(p); p += al256((size_t)n_entries * 32);
  void* scratch = p;
  bool ok = (e = cudaMemcpyAsync(dm, pin, mbytes, cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess &&
            (e = cudaMemcpyAsync(dw, args->scalar, wbytes, cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess &&
            (!obytes || (e = cudaMemcpyAsync(dout, args->pout, obytes, cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess) &&
            (e = qap_transpose(dm, n_wires, n_entries, lo, hi, n_rows, rows, scratch, ctx->stream)) == cudaSuccess &&
            (e = qap_eval(rows, dw, dout, 1, ctx->stream)) == cudaSuccess &&
            (!obytes || (e = cudaMemcpyAsync(args->pout, dout, obytes, cudaMemcpyDeviceToHost, ctx->stream)) == cudaSuccess) &&
            (e = cudaStreamSynchronize(ctx->stream)) == cudaSuccess;
  t_qap_status = ok ? CS_OK : fail(ctx, e, "mpoly_eval");
}

void* mpoly_eval_h(void* vargs) {
  mpoly_eval_server_h(static_cast<mpoly_eval_t*>(vargs));
  return nullptr;
}

}  // extern "C"
