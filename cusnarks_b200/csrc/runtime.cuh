// runtime.cuh -- per-context device state for the C ABI: stream, scratch arena, staging
// buffers, timing events and the last error message.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <cstdio>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>  // header-only; ranges cost nothing unless a profiler is attached

namespace csb {

// Named host range around the enqueueing of a library call (nsys / ncu --nvtx).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Test hook (cs_debug_fail_allocs): while positive, arena growth fails as if the device
// were out of memory, one failure per call.
bool debug_take_alloc_failure();

// Grow-only device buffer (256-byte aligned).  Growing synchronises the owning stream
// first so no in-flight kernel still uses the old block.
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaError_t reserve(size_t need, cudaStream_t st) {
    if (need <= bytes) return cudaSuccess;
    if (ptr) {
      cudaError_t e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return e;
      cudaFree(ptr);
      ptr = nullptr;
      bytes = 0;
    }
    size_t sz = need + need / 8;  // headroom for slightly larger calls
    if (debug_take_alloc_failure()) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(&ptr, sz);
    if (e != cudaSuccess) { ptr = nullptr; return e; }
    bytes = sz;
    return cudaSuccess;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
};

struct PinnedBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaError_t reserve(size_t need) {
    if (need <= bytes) return cudaSuccess;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
    cudaError_t e = cudaMallocHost(&ptr, need);
    if (e != cudaSuccess) { ptr = nullptr; return e; }
    bytes = need;
    return cudaSuccess;
  }
  void release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
  }
};

}  // namespace csb

// The opaque context behind cs_ctx_t in the C header.
struct cs_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  csb::DeviceBuffer work;      // kernel scratch
  csb::DeviceBuffer in;        // device copies of host inputs
  csb::DeviceBuffer out;       // device results
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  cudaEvent_t ev_phase0 = nullptr, ev_phase1 = nullptr;  // bucket accumulation of the last MSM
  float last_ms = 0.f;
  float last_phase_ms = 0.f;
  bool phase_valid = false;
  int msm_affine = -1;         // batch-affine rounds of MSMs on this context: -1 auto, 0 off
  std::string err;
  std::mutex mu;               // one call at a time per context
  // auxiliary streams / events for fork-join pipelines (prove), created on first use
  cudaStream_t aux[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaStream_t aux_h = nullptr;  // QAP -> H step -> H MSM chain of a proof
  static constexpr int kAuxEvents = 9;
  cudaEvent_t aux_ev[kAuxEvents] = {nullptr};
  bool aux_ready = false;
  // Proof launch sequences captured as CUDA graphs (prove.cu): one per key, witness buffer
  // and scratch arena, replayed while all three are those of the capture.
  struct ProveGraph {
    uint64_t pk_id = 0;
    const void* d_w = nullptr;
    void* work = nullptr;
    size_t work_bytes = 0;
    cudaGraphExec_t exec = nullptr;  // null: the capture failed, the sequence runs launch by launch
    unsigned long long launches = 0; // kernels in the graph
  };
  std::vector<ProveGraph> prove_graphs;
  bool use_prove_graphs = true;
  std::vector<std::shared_ptr<void>> prove_batches;  // plans of cs_prove_batch_device (prove.cu)
  bool stages_valid = false;  // the stage events hold the last proof's times (not a graph replay)
};

namespace csb {
// Creates the context's auxiliary streams and events (idempotent).
cudaError_t ctx_aux_init(cs_ctx* ctx);
// Counts kernel launches made by this library (cs_kernel_launches()).
void note_launch(unsigned n = 1);
// Kernel launches counted by the calling thread so far.
unsigned long long thread_launches();
// Destroys the context's captured proof graphs and proof-batch plans (the stream must be idle).
void prove_graphs_release(cs_ctx* ctx);
// Records a CUDA error on the context and maps it to the C ABI status code.
int fail(cs_ctx* ctx, cudaError_t e, const char* where);
int fail_msg(cs_ctx* ctx, int code, const std::string& msg);
}  // namespace csb
