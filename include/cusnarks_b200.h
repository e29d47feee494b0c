/*
 * cusnarks_b200.h -- C ABI of the B200 (sm_100a) Groth16/BN128 prover hot path.
 *
 * Two layers:
 *
 *  1. Drop-in entry points with the names, argument structs and data layouts of the
 *     reference's host functions that its Cython layer (src/cython/_utils_host.pxd)
 *     binds.  Each declaration cites the reference function it replaces.  They take host
 *     pointers, run on the GPU and return when the result is in host memory.  Unlike the
 *     reference they never exit() the process: a failure leaves the output untouched and
 *     is reported by cs_last_error() / cs_last_status().
 *
 *  2. A context API (cs_*) with explicit status codes, device-pointer variants that run
 *     asynchronously on the context's stream, and timing.
 *
 * Data conventions (reference src/cuda/types.h): field elements are 8 little-endian
 * uint32 limbs; pidx 0 = base field q (MOD_GROUP), 1 = scalar field r (MOD_FIELD);
 * points are affine Montgomery, G1 = X|Y (16 words), G2 = X.c0|X.c1|Y.c0|Y.c1 (32 words);
 * infinity is (0, 1_mont) in G1 and (0, 0, 1_mont, 0) in G2; MSM scalars are normal form
 * and may take any 256-bit value.
 */
#ifndef CUSNARKS_B200_H
#define CUSNARKS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes --- */
#define CS_OK 0
#define CS_ERR_CUDA 1        /* a CUDA call failed (message in cs_last_error) */
#define CS_ERR_ARG 2         /* invalid argument */
#define CS_ERR_NOMEM 3       /* device or pinned allocation failed */
#define CS_ERR_UNSUPPORTED 4 /* option the GPU path does not implement */
#define CS_ERR_NODEVICE 5    /* no CUDA device */

/* ------------------------------------------- reference argument structs (layouts) --- */
/* jacadd_reduced_t, reference src/cuda/types.h:548-567 (same member order and types). */
typedef struct {
  uint32_t *out_ep;
  uint32_t *scl;
  uint32_t *x;
  uint32_t n;
  uint32_t ec2;
  uint32_t compute_table;
  uint32_t *ec_table;
  uint32_t pidx;
  uint32_t max_threads;
  uint32_t start_idx;
  uint32_t last_idx;
  uint32_t thread_id;
  uint32_t pippen;
  unsigned long long offset;
  unsigned long long total_words;
  uint32_t order;
  char *filename;
} jacadd_reduced_t;

/* ------------------------------------------------ drop-in reference entry points --- */
/* Replaces ec_jacreduce_server_h, reference src/cuda/ec.cpp:1536 (bound at
 * src/cython/_utils_host.pxd:139).  out_ep <- sum_i scl[i] * x[i] as affine Montgomery
 * (X, Y) for G1 or (X.c0, X.c1, Y.c0, Y.c1) for G2 (ec2 != 0), the reference's
 * strip_last output.  order, pippen, max_threads and compute_table only tune the
 * reference's CPU algorithm and are ignored; a non-NULL filename (precomputed table file)
 * is not supported and fails with CS_ERR_UNSUPPORTED. */
void ec_jacreduce_server_h(jacadd_reduced_t *args);
/* Replaces ec2_jacreduce_server_h, reference src/cuda/ec.cpp:1530 (same as above). */
void ec2_jacreduce_server_h(jacadd_reduced_t *args);

/* Status of the last drop-in call made by this thread, and its message. */
int cs_last_status(void);
const char *cs_last_error(void);

/* -------------------------------------------------------------- context API --------- */
typedef struct cs_ctx cs_ctx;

/* Creates a context on `device` with its own non-blocking stream. */
int cs_ctx_create(int device, cs_ctx **out);
void cs_ctx_destroy(cs_ctx *ctx);
/* Run subsequent device-pointer calls on `stream` (a cudaStream_t; NULL = legacy). */
int cs_ctx_set_stream(cs_ctx *ctx, void *stream);
void *cs_ctx_stream(cs_ctx *ctx);
int cs_ctx_sync(cs_ctx *ctx);
const char *cs_ctx_error(cs_ctx *ctx);
/* Device time in milliseconds of the kernels of the last cs_* call (CUDA events). */
float cs_ctx_last_ms(cs_ctx *ctx);

/* Multi-exponentiation with host pointers: copies in, computes, copies the affine result
 * out, synchronises.  ec2 selects G2.  window = Pippenger window bits (0 = automatic). */
int cs_msm(cs_ctx *ctx, int ec2, const uint32_t *scalars, const uint32_t *points, uint32_t n,
           uint32_t *out_affine, int window);
/* Same with device pointers, asynchronous on the context stream.  Scratch comes from the
 * context's device arena (grown on demand; growing synchronises the stream). */
int cs_msm_device(cs_ctx *ctx, int ec2, const uint32_t *d_scalars, const uint32_t *d_points,
                  uint32_t n, uint32_t *d_out_affine, int window);
/* Scratch bytes one MSM of n terms needs (window 0 = automatic). */
size_t cs_msm_workspace_bytes(uint32_t n, int ec2, int window);

#ifdef __cplusplus
}
#endif

#endif /* CUSNARKS_B200_H */
