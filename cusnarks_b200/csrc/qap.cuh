// qap.cuh -- sparse QAP evaluation (the reference's mpoly_eval_h, src/cuda/mpoly.cpp:125).
//
// The reference stores each QAP polynomial matrix "by wire" (r1cs_to_mpoly_h, mpoly.cpp:195):
//   [N][ncoeff_0 .. ncoeff_{N-1}] then, per wire i, ncoeff_i constraint indices followed by
//   ncoeff_i 8-word Montgomery coefficients,
// and evaluates out[c] += w_i * coeff (Montgomery) by scattering per wire, which races when
// threaded (mpoly.cpp:67-168).  Here the matrix is transposed once on the device into rows
// by constraint (CSR); each output element is then a short gather-and-sum owned by one
// thread: deterministic, and exact field sums make the order irrelevant.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

namespace csb {

struct QapRows {
  uint32_t n_rows = 0;       // constraints (domain points) covered
  uint32_t n_entries = 0;
  uint32_t* row_off = nullptr;   // n_rows + 1
  uint32_t* wire = nullptr;      // n_entries
  uint32_t* coeff = nullptr;     // n_entries x 8: coefficient x R (Montgomery of the Montgomery
                                 // value), so a Montgomery product with a normal-form witness
                                 // value gives the Montgomery-form term directly
};

// Scratch bytes and entry counts needed to transpose an mpoly with n_wires wires, n_entries
// coefficients into n_rows rows.
size_t qap_transpose_scratch_bytes(uint32_t n_wires, uint32_t n_rows, uint32_t n_entries);

// d_mpoly: the reference layout on the device (words); wires [wire_lo, wire_hi) are kept.
// rows: caller-allocated arrays sized for n_rows / n_entries.  scratch: see above.
cudaError_t qap_transpose(const uint32_t* d_mpoly, uint32_t n_wires, uint32_t n_total_entries,
                          uint32_t wire_lo, uint32_t wire_hi, uint32_t n_rows, QapRows& rows,
                          void* scratch, cudaStream_t st);

// out[c] (+)= sum over row c of coeff * w[wire]; accumulate != 0 adds into out.  batch
// instances: instance y reads w and writes out y * stride words further on.
cudaError_t qap_eval(const QapRows& rows, const uint32_t* d_w, uint32_t* d_out, int accumulate,
                     cudaStream_t st, uint32_t batch = 1, size_t stride = 0);

}  // namespace csb
