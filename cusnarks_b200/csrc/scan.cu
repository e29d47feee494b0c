// scan.cu -- multi-level exclusive scan: every block scans 4096 elements (1024 threads x
// 4), block totals are scanned recursively, then added back.
#include "scan.cuh"
#include "runtime.cuh"

namespace csb {

namespace {
constexpr int kThreads = 1024;
constexpr int kPer = 4;
constexpr size_t kTile = (size_t)kThreads * kPer;

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

__global__ void __launch_bounds__(kThreads) k_scan_tile(const uint32_t* __restrict__ in,
                                                        uint32_t* __restrict__ out, size_t n,
                                                        uint32_t* __restrict__ tile_sums) {
  __shared__ uint32_t warp_tot[32];
  const size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kPer;
  uint32_t v[kPer];
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kPer; i++) {
    v[i] = (base + i < n) ? in[base + i] : 0u;
    s += v[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = s;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += t;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = warp_tot[lane];
    uint32_t wi = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, wi, d);
      if (lane >= d) wi += t;
    }
    warp_tot[lane] = wi - w;  // exclusive warp offsets
    if (lane == 31 && tile_sums) tile_sums[blockIdx.x] = wi;
  }
  __syncthreads();
  uint32_t run = warp_tot[warp] + incl - s;
#pragma unroll
  for (int i = 0; i < kPer; i++) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
}

__global__ void k_add_tile_offsets(uint32_t* __restrict__ out, size_t n,
                                   const uint32_t* __restrict__ tile_off) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += tile_off[i / kTile];
}

}  // namespace

size_t scan_workspace_bytes(size_t n) {
  size_t total = 0;
  while (n > kTile) {
    const size_t tiles = (n + kTile - 1) / kTile;
    total += 2 * align256(tiles * sizeof(uint32_t));
    n = tiles;
  }
  return total + 256;
}

cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, void* tmp,
                               cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  if (n <= kTile) {
    k_scan_tile<<<1, kThreads, 0, st>>>(in, out, n, nullptr);
    note_launch();
    return cudaGetLastError();
  }
  const size_t tiles = (n + kTile - 1) / kTile;
  uint32_t* sums = static_cast<uint32_t*>(tmp);
  uint32_t* sums_scan = reinterpret_cast<uint32_t*>(static_cast<char*>(tmp) + align256(tiles * 4));
  void* rest = static_cast<char*>(tmp) + 2 * align256(tiles * 4);
  k_scan_tile<<<(unsigned)tiles, kThreads, 0, st>>>(in, out, n, sums);
  note_launch();
  cudaError_t e = scan_exclusive_u32(sums, sums_scan, tiles, rest, st);
  if (e != cudaSuccess) return e;
  k_add_tile_offsets<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n, sums_scan);
  note_launch();
  return cudaGetLastError();
}

}  // namespace csb
