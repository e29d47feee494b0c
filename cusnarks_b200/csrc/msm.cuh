// msm.cuh -- Pippenger multi-scalar multiplication for BN254 G1/G2 on sm_100a.
//
// Replaces the reference's GPU multi-exp (src/cuda/ecbn128_device.cu:508
// madecjac_shfl_kernel + :567 redecjac_kernel, per-thread Shamir tables and a shuffle
// tree) and produces the value of its CPU multi-exp ec_jacreduce_server_h
// (src/cuda/ec.cpp:1536): sum_i k_i * P_i as an affine Montgomery point.
//
// Pipeline for one instance of N terms, window width c, W = floor(254/c) + 1 windows,
// B = 2^(c-1) buckets per window:
//   1. digits:   each scalar (any 256-bit value) is reduced mod r and recoded into W
//                signed c-bit digits d in (-2^(c-1), 2^(c-1)]; every nonzero digit adds
//                one to the count of bucket (window, |d|-1).  Zero scalars and points at
//                infinity produce no entries.
//   2. scan:     exclusive prefix sum of the W*B counts -> bucket offsets.
//   3. scatter:  digits are recomputed and (point index | sign) is written into the slot
//                of its bucket: a counting sort of the N*W (bucket, point) pairs.
//   4. accumulate: buckets are summed with mixed XYZZ + affine additions.  Buckets are
//                split into tasks of at most TASK points; tasks run longest first so
//                warps see similar trip counts.  Partial sums of split buckets are added
//                back together by a second pass.
//   5. reduce:   per window, sum_b (b+1) * bucket_b by hierarchical running sums over
//                segments of 8 buckets (level k leaves sum_i i*y_i with weight 8^k and
//                the segment total for the next level).
//   6. finish:   level results are combined with 3-bit Horner steps, windows with c-bit
//                Horner steps, and the result is converted to affine.
//
// Fixed-base variant, for bases that stay resident (a proving key): a table
// T[j*N + i] = 2^(c j) P_i of W*N affine points is built once, every digit of every
// scalar goes into ONE set of 2^(c-1) buckets, and steps 5-6 reduce a single window
// (more 8-bucket levels, no window Horner).  With the per-window tail gone a wider
// window (c ~ 20 at N = 2^20: 13 instead of 16 windows) also cuts the accumulation.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

namespace csb {

// Instance of a batch of MSMs: device pointers, size, window, and its first term, bucket
// and window in the batch (instances are ordered by window so each window group occupies a
// contiguous bucket range).
// A batch instance.  fixed = 0: points holds n points, W bucket sets (one per window).
// fixed = 1: points is a fixed-base table T[j n + i] = 2^(c j) P_i of W windows, one bucket set
// (entries are table indices), no window Horner.  sets: bucket sets (W or 1).
struct BatchJob {
  const uint32_t* scalars;
  const uint32_t* points;
  uint32_t* out;
  uint32_t n, c, W, bucket0, window0, term0, fixed, sets;
};

// A group of batch instances sharing one window c: buckets [bucket0, bucket0 + windows * B),
// window sums [window0, window0 + windows).
struct BatchGroup {
  int c;
  uint32_t bucket0, windows, window0;
};

// A batch plan: the job table (device), totals and the groups, scratch of
// msm_batch_workspace_bytes() bytes.
struct MsmBatch {
  const BatchJob* d_jobs = nullptr;
  uint32_t njobs = 0;
  uint32_t terms = 0;      // sum of n
  uint32_t nbuckets = 0;   // sum of W * 2^(c-1)
  uint64_t nentries = 0;   // sum of n * W (upper bound of bucket entries)
  uint32_t nwindows = 0;   // sum of W
  uint64_t lv_points = 0, lv2_points = 0;  // max over groups of W*(2^(c-1)/8+1), W*(.../64+1)
  const BatchGroup* groups = nullptr;  // host array
  uint32_t ngroups = 0;
  int task = 64;           // entries per accumulation task, kBatchMinTask..64 (set by the builder)
};
constexpr int kBatchMinTask = 8;
size_t msm_batch_workspace_bytes(const MsmBatch& b, bool ec2);
// An instance as a caller describes it (batch.cu builds the plan): fixed = a fixed-base table
// built with `window`, which is then required.
struct BatchSpec {
  const uint32_t* scalars;
  const uint32_t* points;
  uint32_t* out;
  uint32_t n;
  int window;
  bool fixed;
};
cudaError_t msm_batch_g1(const MsmBatch& b, void* d_work, size_t work_bytes, cudaStream_t stream);
cudaError_t msm_batch_g2(const MsmBatch& b, void* d_work, size_t work_bytes, cudaStream_t stream);

struct MsmConfig {
  int c = 0;          // window bits; 0 = pick from N
  int task = 0;       // points per accumulation task, 8..96 (0: automatic)
  int min_task = 0;   // shortest task the workspace is sized for (0: automatic, by the MSM's
                      // entries; msm_workspace_bytes takes the same value)
  int affine = -1;    // batch-affine halving rounds before the XYZZ accumulation: -1 auto, 0 off
  int glv = -1;       // generic G1 MSMs: split the scalars by the GLV endomorphism (-1 auto = on, 0 off)
  // optional events recorded around the bucket-accumulation kernels (phase timing)
  cudaEvent_t acc_start = nullptr, acc_stop = nullptr;
  // Two fixed-base MSMs with the same window whose sums are added (a proof's C and H terms)
  // share one bucket reduction.  bucket_out: the MSM accumulates into that array (2^(c-1)
  // XYZZ buckets), skips the reduction and returns the point at infinity.  bucket_add: after
  // its own accumulation (and after waiting for bucket_ready when given) the MSM adds that
  // array into its buckets, so its result is the sum of both MSMs.
  uint32_t* bucket_out = nullptr;
  const uint32_t* bucket_add = nullptr;
  cudaEvent_t bucket_ready = nullptr;
};

// Bytes of device scratch one MSM of n terms needs (G2 when ec2).
// affine_mode: batch-affine rounds the MSM will run (-1 automatic, 0 none, > 0 that many).
// glv_mode: as MsmConfig::glv (G1 only).
// min_task: the MsmConfig::min_task the call will use (0 automatic).
size_t msm_workspace_bytes(uint32_t n, int c, bool ec2, int affine_mode = -1, int glv_mode = -1, int min_task = 0);
// Window for n terms: G1 for the GLV split (2n terms of 128 bits), G2 for n of 254 bits.
int msm_default_window(uint32_t n, bool ec2);
// The cost model's window for n terms with (glv) or without the GLV split.
int msm_window_model(uint32_t n, bool glv);

// d_scalars: n x 8 words (normal form), d_points: n affine points (16 or 32 words),
// d_out: one affine point (16 or 32 words), d_work: msm_workspace_bytes() bytes,
// 256-byte aligned.  Everything runs on `stream`; nothing is allocated.
cudaError_t msm_g1(const uint32_t* d_scalars, const uint32_t* d_points, uint32_t n,
                   uint32_t* d_out, void* d_work, size_t work_bytes, const MsmConfig& cfg,
                   cudaStream_t stream);
cudaError_t msm_g2(const uint32_t* d_scalars, const uint32_t* d_points, uint32_t n,
                   uint32_t* d_out, void* d_work, size_t work_bytes, const MsmConfig& cfg,
                   cudaStream_t stream);

// Fixed-base MSM.  Window for a table of n bases; table points (W*n); scratch bytes to
// build a table (table_work) and to run one MSM (workspace).  cfg.c must equal the c the
// table was built with.
int msm_fixed_window(uint32_t n, bool ec2);
size_t msm_fixed_table_points(uint32_t n, int c);
size_t msm_fixed_table_work_bytes(uint32_t n, bool ec2);
size_t msm_fixed_workspace_bytes(uint32_t n, int c, bool ec2, int affine_mode = -1);
cudaError_t msm_fixed_table_g1(const uint32_t* d_points, uint32_t n, int c, uint32_t* d_table, void* d_work,
                               size_t work_bytes, cudaStream_t stream);
cudaError_t msm_fixed_table_g2(const uint32_t* d_points, uint32_t n, int c, uint32_t* d_table, void* d_work,
                               size_t work_bytes, cudaStream_t stream);
cudaError_t msm_fixed_g1(const uint32_t* d_scalars, const uint32_t* d_table, uint32_t n, uint32_t* d_out,
                         void* d_work, size_t work_bytes, const MsmConfig& cfg, cudaStream_t stream);
cudaError_t msm_fixed_g2(const uint32_t* d_scalars, const uint32_t* d_table, uint32_t n, uint32_t* d_out,
                         void* d_work, size_t work_bytes, const MsmConfig& cfg, cudaStream_t stream);

}  // namespace csb
