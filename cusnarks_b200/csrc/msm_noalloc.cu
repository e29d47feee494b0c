// msm_noalloc.cu -- a G1 multi-exponentiation entry point that allocates no memory.
//
// Who needs it: code that runs inside a host application which owns every device
// allocation through its own pool (and forbids or cannot afford a direct cudaMalloc, whose
// implicit device synchronisation also stalls latency-critical paths).  Such callers pass
// inputs and outputs they already hold; the MSM's scratch (bucket counts, sorted entries,
// tasks and bucket sums) comes from the fixed array below instead of the heap.
//
// The array is a file-scope __device__ object, so every GPU on which this library's
// module is loaded keeps these bytes reserved until the process exits.  All calls on a
// device share it and it keeps the previous call's contents; the MSM clears what must
// start at zero (its counters and bucket counts) itself on every call.  Two calls whose
// work overlaps on the GPU (different streams, no ordering between them) race on the
// array and give wrong results: order them on one stream or serialise them.
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/cusnarks_b200.h"
#include "msm.cuh"

namespace {

constexpr size_t kScratchBytes = 32ull << 20;  // 32 MiB: G1 MSMs of up to 2^16 terms
constexpr int kTask = 32;  // shortest accumulation task: the array's size is fixed on it
static __device__ __align__(256) unsigned char g_msm_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_addr[64] = {nullptr};
thread_local std::string t_noalloc_err;

}  // namespace

extern "C" {

size_t cs_msm_noalloc_scratch_bytes(void) { return kScratchBytes; }

uint32_t cs_msm_g1_noalloc_max_terms(void) {
  uint32_t lo = 0, hi = 1u << 24;
  while (lo < hi) {  // largest n whose automatic-window workspace fits the array
    const uint32_t mid = lo + (hi - lo + 1) / 2;
    if (csb::msm_workspace_bytes(mid, 0, false, 0, 0, kTask) <= kScratchBytes) lo = mid; else hi = mid - 1;
  }
  return lo;
}

const char* cs_msm_g1_noalloc_error(void) { return t_noalloc_err.c_str(); }

int cs_msm_g1_noalloc(const uint32_t* d_scalars, const uint32_t* d_points, uint32_t n,
                      uint32_t* d_out_affine, void* stream) {
  t_noalloc_err.clear();
  if (!d_out_affine || (n && (!d_scalars || !d_points))) {
    t_noalloc_err = "cs_msm_g1_noalloc: null pointer argument";
    return CS_ERR_ARG;
  }
  const size_t need = csb::msm_workspace_bytes(n, 0, false, 0, 0, kTask);
  if (need > kScratchBytes) {
    t_noalloc_err = "cs_msm_g1_noalloc: " + std::to_string(n) + " terms need " + std::to_string(need) +
                    " bytes of scratch, above the fixed " + std::to_string(kScratchBytes) +
                    "-byte array (at most " + std::to_string(cs_msm_g1_noalloc_max_terms()) + " terms)";
    return CS_ERR_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    t_noalloc_err = std::string("cs_msm_g1_noalloc: no current device: ") + cudaGetErrorString(e);
    cudaGetLastError();
    return CS_ERR_NODEVICE;
  }
  void* scratch = nullptr;
  {
    // Once per device, with that device current: the host-side name g_msm_scratch is only
    // a stand-in; the device address of the array comes from cudaGetSymbolAddress.
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_msm_scratch);
      if (e != cudaSuccess || p == nullptr) {
        t_noalloc_err = std::string("cs_msm_g1_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
        cudaGetLastError();
        return CS_ERR_CUDA;
      }
      g_scratch_addr[dev] = p;
    }
    scratch = g_scratch_addr[dev];
  }
  csb::MsmConfig cfg;  // automatic window, no timing events
  cfg.affine = 0;      // XYZZ accumulation only: the fixed array is sized without round buffers
  cfg.glv = 0;         // nor the GLV split's buffers (2n scalars and points)
  cfg.min_task = kTask;  // and for tasks of at least 32 entries
  e = csb::msm_g1(d_scalars, d_points, n, d_out_affine, scratch, kScratchBytes, cfg,
                  static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    t_noalloc_err = std::string("cs_msm_g1_noalloc: ") + cudaGetErrorString(e);
    cudaGetLastError();
    return CS_ERR_CUDA;
  }
  return CS_OK;
}

}  // extern "C"
