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
#define CS_ERR_TIMEOUT 6     /* a wait ran out of time (the request is still pending) */
#define CS_ERR_CANCELLED 7   /* the request was cancelled before it ran */

/* ------------------------------------------- reference argument structs (layouts) --- */
/* The structs and enums below repeat the reference's src/cuda/types.h layouts.  A
 * translation unit that includes the reference's own types.h as well (the reference's
 * Cython module built against this library) defines CS_REFERENCE_TYPES first, and the
 * declarations then use the reference's definitions. */
#ifndef CS_REFERENCE_TYPES
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

/* ntt_interpolandmul_t, reference src/cuda/types.h:530-546. */
typedef struct {
  uint32_t *A;
  uint32_t *B;
  uint32_t *roots;
  uint32_t Nrows;
  uint32_t Ncols;
  uint32_t mNrows;
  uint32_t mNcols;
  uint32_t nroots;
  uint32_t rstride;
  uint32_t pidx;
  uint32_t max_threads;
  uint32_t start_idx;
  uint32_t last_idx;
  uint32_t thread_id;
} ntt_interpolandmul_t;

/* mpoly_eval_t, reference src/cuda/types.h:516-528. */
typedef struct {
  uint32_t *pout;
  const uint32_t *scalar;
  uint32_t *pin;
  uint32_t reduce_coeff;
  uint32_t start_idx;
  uint32_t last_idx;
  uint32_t max_threads;
  uint32_t thread_id;
  uint32_t pidx;
} mpoly_eval_t;
#endif /* CS_REFERENCE_TYPES */

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

/* Field arithmetic, reference src/cuda/ff.cpp (bound at src/cython/_utils_host.pxd:41-65):
 * single-element Montgomery product, square, modular add/sub and Montgomery inverse
 * (replacing montmult_h ff.cpp:225, montsquare_h :423, addm_h :679, subm_h :713,
 * montinv_h :745), and the batched conversions to_montgomeryN_h :658 and
 * from_montgomeryN_h :503 (strip_last 0 only; other values report CS_ERR_UNSUPPORTED).
 * Results go to host memory; status in cs_field_last_status(). */
void montmult_h(uint32_t *U, const uint32_t *A, const uint32_t *B, uint32_t pidx);
void montsquare_h(uint32_t *U, const uint32_t *A, uint32_t pidx);
void addm_h(uint32_t *U, const uint32_t *A, const uint32_t *B, uint32_t pidx);
void subm_h(uint32_t *U, const uint32_t *A, const uint32_t *B, uint32_t pidx);
void montinv_h(uint32_t *y, uint32_t *x, uint32_t pidx);
void to_montgomeryN_h(uint32_t *z, const uint32_t *x, uint32_t n, uint32_t pidx);
void from_montgomeryN_h(uint32_t *z, const uint32_t *x, uint32_t n, uint32_t pidx, uint32_t strip_last);
int cs_field_last_status(void);

/* Number-theoretic transforms over Fr (pidx must be 1, MOD_FIELD).
 * Replaces ntt_h, reference src/cuda/ntt.cpp:453 (bound at _utils_host.pxd:70):
 *   A[k*astride] <- sum_j A[j*astride] roots[(rstride*j*k*direction) mod (rstride*2^levels)],
 *   natural order, in place.
 * Replaces intt_h, reference src/cuda/ntt.cpp:583 (_utils_host.pxd:72): the inverse
 *   transform (direction -1 on the same table) scaled by 2^-levels, output Montgomery
 *   (fmat 1) or normal form (fmat 0).
 * Replaces find_roots_h, reference src/cuda/ntt.cpp:1164: roots[i] = primitive_root^i.
 * Status in cs_ntt_last_status(). */
void ntt_h(uint32_t *A, const uint32_t *roots, uint32_t levels, unsigned long long astride,
           unsigned long long rstride, int32_t direction, uint32_t pidx);
void intt_h(uint32_t *A, const uint32_t *roots, uint32_t fmat, uint32_t levels,
            unsigned long long rstride, uint32_t pidx);
void find_roots_h(uint32_t *roots, uint32_t *primitive_root, uint32_t nroots, uint32_t pidx);
/* Replaces ntt_interpolandmul_server_h, reference src/cuda/ntt.cpp:672 (_utils_host.pxd:89):
 * A, B = evaluations (Montgomery) on the m = 2^(Nrows+Ncols) roots; returns a pointer to
 * the 2m coefficients of A(x)B(x) in normal form, held in a library buffer that stays
 * valid until the next call (the reference returns its global M_transpose the same way).
 * roots is the caller's concatenated table whose first 2m entries are powers of the 2m-th
 * root; rstride as in the reference (2).  A and B are left unmodified.  NULL on error. */
uint32_t *ntt_interpolandmul_server_h(ntt_interpolandmul_t *args);
/* Replaces get_Mtranspose_h, reference src/cuda/ntt.cpp:659: the last H-step result. */
uint32_t *get_Mtranspose_h(void);
/* Replaces get_Mmul_h, reference src/cuda/ntt.cpp:650 (_utils_host.pxd:91): the last H-step
 * result before the reference's final transpose, i.e. the 2m coefficients as a
 * 2^mNrows x 2^mNcols matrix M with M[r][c] = coefficient c*2^mNrows + r, where
 * (mNrows, mNcols) = (Nrows+1, Ncols) if Nrows < Ncols else (Nrows, Ncols+1)
 * (ntt.cpp:767).  Valid until the next H-step call; NULL before the first. */
uint32_t *get_Mmul_h(void);
#ifndef CS_REFERENCE_TYPES
/* fft_mode_t, reference src/cuda/types.h:235 */
typedef enum { FFT_T_DIT = 0, FFT_T_DIF, FFT_T_MODE_N } fft_mode_t;
#endif
/* Replaces ntt_parallel_h, reference src/cuda/ntt.cpp:274 (_utils_host.pxd:78): the reference
 * computes the 2^(Nrows+Ncols)-point transform by four steps (column transforms, twiddles,
 * row transforms, transpose); its result is the natural-order transform of ntt_h with
 * levels = Nrows + Ncols, astride 1, for both fft_mode values, which is what this returns. */
void ntt_parallel_h(uint32_t *A, const uint32_t *roots, uint32_t Nrows, uint32_t Ncols,
                    unsigned long long rstride, int32_t direction, fft_mode_t fft_mode, uint32_t pidx);
/* Replaces ntt_parallel2D_h, reference src/cuda/ntt.cpp:199 (_utils_host.pxd:82): with
 * direction 1 (the reference's only use: intt_parallel2D_h and its tests pass inverse roots
 * with direction 1) the same natural-order 2^(Nrows+Ncols)-point transform.  The reference's
 * twiddle step ignores direction, so direction -1 is not a transform there; it is refused
 * here (status CS_ERR_ARG).  fft_Nyx / fft_Nxx only choose the reference's inner split. */
void ntt_parallel2D_h(uint32_t *A, const uint32_t *roots, uint32_t Nrows, uint32_t fft_Nyx, uint32_t Ncols,
                      uint32_t fft_Nxx, unsigned long long rstride, int32_t direction, uint32_t pidx);
int cs_ntt_last_status(void);

/* QAP evaluation.  Replaces mpoly_eval_server_h, reference src/cuda/mpoly.cpp:67
 * (_utils_host.pxd:207), and mpoly_eval_h, mpoly.cpp:125: pout[c] += toMont(scalar[i]) *
 * coeff for every (c, coeff) of the polynomials i in [start_idx, last_idx) of the
 * reference mpoly layout pin (mpoly.cpp:195).  Deterministic (no racing threads); pidx
 * must be 1.  Status in cs_qap_last_status(). */
void mpoly_eval_server_h(mpoly_eval_t *args);
void *mpoly_eval_h(void *args);
int cs_qap_last_status(void);

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
/* Device time in milliseconds of the bucket-accumulation kernels of the last MSM. */
float cs_ctx_last_phase_ms(cs_ctx *ctx);
/* Batch-affine halving rounds run before the XYZZ bucket accumulation by this context's
 * cs_msm / cs_msm_device / cs_msm_fixed_device calls: -1 automatic (default), 0 none, 1..6.
 * Results do not depend on it. */
int cs_ctx_set_msm_affine_rounds(cs_ctx *ctx, int rounds);
/* Test hook: the next `count` growths of any context's device arenas fail as if the device
 * were out of memory (the call reports CS_ERR_NOMEM and the context stays usable). */
void cs_debug_fail_allocs(int count);

/* Multi-exponentiation with host pointers: copies in, computes, copies the affine result
 * out, synchronises.  ec2 selects G2.  window = Pippenger window bits (0 = automatic).
 * G1 splits every scalar by the GLV endomorphism of BN254 (k = k1 + k2 lambda mod r with
 * |k1|, |k2| < 2^127; k P = k1 P + k2 phi(P), phi(x, y) = (beta x, y)) and sorts the 2n
 * half-scalars: ceil(128 / window) windows, half the bucket sets and half the window Horner
 * of the full scalars' 254 / window + 1.  The result is the same point. */
int cs_msm(cs_ctx *ctx, int ec2, const uint32_t *scalars, const uint32_t *points, uint32_t n,
           uint32_t *out_affine, int window);
/* Same with device pointers, asynchronous on the context stream.  Scratch comes from the
 * context's device arena (grown on demand; growing synchronises the stream). */
int cs_msm_device(cs_ctx *ctx, int ec2, const uint32_t *d_scalars, const uint32_t *d_points,
                  uint32_t n, uint32_t *d_out_affine, int window);
/* Scratch bytes one MSM of n terms needs (window 0 = automatic). */
size_t cs_msm_workspace_bytes(uint32_t n, int ec2, int window);
/* Window bits the automatic choice uses for n terms (G1: for the GLV split), and the window
 * count of a full scalar (254 / window + 1: G2, fixed-base tables, batch instances). */
int cs_msm_default_window(uint32_t n, int ec2);
int cs_msm_num_windows(int window);

/* Fixed-base multi-exponentiation for bases that stay resident in HBM (a proving key).
 * The reference re-sends the proving-key points with every proof (groth_prover.py:1563
 * findECPointsDispatch); here a table of cs_msm_fixed_table_points(n, window) affine points
 * T[j*n + i] = 2^(window*j) P_i is built once by cs_msm_fixed_table_device, and every
 * cs_msm_fixed_device call over those bases sums all windows in one bucket set (no
 * per-window reduction, no window Horner step).  Same result as cs_msm_device on the
 * original points.  window in [4, 24]; cs_msm_fixed_window picks one for n bases. */
int cs_msm_fixed_window(uint32_t n, int ec2);
size_t cs_msm_fixed_table_points(uint32_t n, int window);
size_t cs_msm_fixed_workspace_bytes(uint32_t n, int ec2, int window);
int cs_msm_fixed_table_device(cs_ctx *ctx, int ec2, const uint32_t *d_points, uint32_t n, int window,
                              uint32_t *d_table);
int cs_msm_fixed_device(cs_ctx *ctx, int ec2, const uint32_t *d_scalars, const uint32_t *d_table,
                        uint32_t n, int window, uint32_t *d_out_affine);

/* Batched multi-exponentiation: many instances of uneven size (device pointers) summed in one
 * pass -- one digit sort and ONE bucket-accumulation launch over the union of their buckets,
 * split by bucket size, then one reduction per distinct window.  Replaces one GPU multi-exp
 * call per instance (cuda_wrapper.py:216 ec_mad_cuda2 driven by groth_prover.py:1563).
 * window 0 = the autotuned window for the instance's size (cs_msm_autotune) or, untuned, the
 * cost-model default.  cs_msm_batch_run is asynchronous on the context stream; use_graph != 0
 * captures the sequence into a CUDA graph on the first run and replays it afterwards (the
 * plan's pointers are baked in: change inputs in place).  task = bucket tile (max entries
 * per accumulation task, 8..64; 0 = by the batch's size: about one task per resident
 * accumulation thread, 8..64).  Each result equals cs_msm_device's. */
typedef struct {
  const uint32_t *scalars, *points;
  uint32_t *out;
  uint32_t n;
  int window;
} cs_msm_job;
typedef struct cs_msm_batch cs_msm_batch;
int cs_msm_batch_create(cs_ctx *ctx, int ec2, const cs_msm_job *jobs, uint32_t njobs, int task,
                        cs_msm_batch **out);
int cs_msm_batch_run(cs_ctx *ctx, cs_msm_batch *batch, int use_graph);
void cs_msm_batch_destroy(cs_msm_batch *batch);
size_t cs_msm_batch_workspace_bytes(const cs_msm_batch *batch);
int cs_msm_batch_window(const cs_msm_batch *batch, uint32_t job);
/* Window autotuner for batched MSMs: times the MSM of full scalars (the form a batch instance
 * runs) at each size 2^log_min..2^log_max for windows around the cost-model choice and keeps
 * the fastest per size (per device, process-wide); windows_out (optional) receives them.
 * Synchronous. */
int cs_msm_autotune(cs_ctx *ctx, int ec2, uint32_t log_min, uint32_t log_max, int *windows_out);
int cs_msm_tuned_window(cs_ctx *ctx, int ec2, uint32_t n);

/* Elementwise field operation on n elements of device arrays (8 words each; 16 for
 * CS_FOP_FQ2_MUL, which multiplies in Fq2 = Fq[u]/(u^2+1) regardless of pidx).
 * d_b is ignored by the unary operations.  Asynchronous on the context stream. */
#define CS_FOP_MUL 0       /* Montgomery product a*b*R^-1 */
#define CS_FOP_ADD 1
#define CS_FOP_SUB 2
#define CS_FOP_SQR 3
#define CS_FOP_INV 4       /* Montgomery inverse (aR)^-1 R, 0 -> 0 */
#define CS_FOP_TO_MONT 5   /* a -> aR */
#define CS_FOP_FROM_MONT 6 /* aR -> a */
#define CS_FOP_FQ2_MUL 8
#define CS_FOP_MUL_DP52 9  /* Montgomery product, radix-2^52 FP64-pipe variant (cross-check) */
int cs_field_op_device(cs_ctx *ctx, int op, int pidx, const uint32_t *d_a, const uint32_t *d_b,
                       uint32_t *d_out, uint32_t n);

/* Batched scalar multiplication out[i] = scalars[i] * points[i] (affine Montgomery in and
 * out, like the reference's ec_jacscmul_h + ec_jac2aff_h, src/cuda/ec.cpp:833, :963).
 * point_stride_words = words between consecutive base points; 0 = one shared base
 * (fixed-base, as the reference's proving-key generation kernel sc1mulecjac_kernel,
 * src/cuda/ecbn128_device.cu:326).  Device pointers, asynchronous on the context stream. */
int cs_scmul_device(cs_ctx *ctx, int ec2, const uint32_t *d_scalars, const uint32_t *d_points,
                    uint32_t point_stride_words, uint32_t n, uint32_t *d_out_affine);

/* Sum of n points as one affine point (Montgomery, the reference's infinity encoding):
 * rows of dims = 2 (affine) or 3 (Jacobian) coordinates, as the reference's
 * ec_jacaddreduce_h (src/cuda/ec.cpp:1266) on device data.  It combines the per-shard
 * results of an MSM split across GPUs.  Device pointers, asynchronous on the context stream. */
int cs_point_sum_device(cs_ctx *ctx, int ec2, const uint32_t *d_points, uint32_t n, int dims,
                        uint32_t *d_out_affine);

/* Transform of 2^log_n Fr elements (Montgomery) with the context's resident twiddles
 * (primitive roots 5^((r-1)/2^k), the reference's proots_field chain).  direction >= 0:
 * forward; < 0: inverse scaled by 2^-log_n, Montgomery (fmat 1) or normal (fmat 0) out.
 * d_in may equal d_out.  Asynchronous on the context stream. */
int cs_ntt_device(cs_ctx *ctx, const uint32_t *d_in, uint32_t *d_out, uint32_t log_n, int direction,
                  int fmat);
/* H step on device arrays of m = 2^log_m evaluations (Montgomery):
 *   CS_HSTEP_REFERENCE: d_out (2m) = coefficients of A(x)B(x), normal form (d_C unused),
 *                       as ntt_interpolandmul_server_h;
 *   CS_HSTEP_COSET:     d_out (m) = coefficients of (A B - C)/(x^m - 1) evaluated on the
 *                       coset 5*<w>, normal form.
 * Both give the Groth16 quotient H in d_out[m .. 2m-2] / d_out[0 .. m-2] when A B - C
 * vanishes on the domain. */
#define CS_HSTEP_REFERENCE 0
#define CS_HSTEP_COSET 1
int cs_hstep_device(cs_ctx *ctx, int variant, const uint32_t *d_A, const uint32_t *d_B,
                    const uint32_t *d_C, uint32_t log_m, uint32_t *d_out);

/* ----------------------------------------- remaining host functions of the binding --- */
/* The rest of the reference's host functions that src/cython/_utils_host.pxd binds and
 * the prover calls.  Point rows: Montgomery, G1 Jacobian 3 x 8 words / affine 2 x 8, G2
 * 3 x 16 / 2 x 16, infinity (0, 1, 0) / (0, 1); pidx must be 0 (MOD_GROUP).  The point
 * routines run on the GPU (default context of the current device); Jacobian results come
 * back normalised (Z = 1): the same points as the reference's.  Status: cs_last_status(). */
/* ec.cpp:963 -- Jacobian -> affine rows (strip_last: 2 coordinates, else x, y, 1). */
void ec_jac2aff_h(uint32_t *y, uint32_t *x, uint32_t n, uint32_t pidx, uint32_t strip_last);
void ec2_jac2aff_h(uint32_t *y, uint32_t *x, uint32_t n, uint32_t pidx, uint32_t strip_last);
/* ec.cpp:1266 -- sum of n rows (add_in: affine rows of 2, else Jacobian rows of 3). */
void ec_jacaddreduce_h(uint32_t *z, uint32_t *x, uint32_t n, uint32_t pidx, uint32_t to_aff, uint32_t add_in,
                       uint32_t strip_last);
void ec2_jacaddreduce_h(uint32_t *z, uint32_t *x, uint32_t n, uint32_t pidx, uint32_t to_aff, uint32_t add_in,
                        uint32_t strip_last);
/* ec.cpp:833 / :819 -- z[i] = scl[i] * P_i (bases Jacobian, or affine with add_last);
 * sc1mul: x = n scalars followed by one base.  Jacobian rows out. */
void ec_jacscmul_h(uint32_t *z, uint32_t *scl, uint32_t *x, uint32_t n, uint32_t pidx, uint32_t add_last);
void ec2_jacscmul_h(uint32_t *z, uint32_t *scl, uint32_t *x, uint32_t n, uint32_t pidx, uint32_t add_last);
void ec_jacsc1mul_h(uint32_t *z, uint32_t *x, uint32_t n, uint32_t pidx, uint32_t add_last);
void ec2_jacsc1mul_h(uint32_t *z, uint32_t *x, uint32_t n, uint32_t pidx, uint32_t add_last);
/* ec.cpp:1064 -- 2: the infinity encoding (X = 0, Y = 1), 1: on the curve, 0: not. */
uint32_t ec_isoncurve_h(uint32_t *x, uint32_t is_affine, uint32_t pidx);
uint32_t ec2_isoncurve_h(uint32_t *x, uint32_t is_affine, uint32_t pidx);
/* ec.cpp:574 / ec2_inittable_h -- subset-sum tables: ectable <- ceil(n / table_order) tables
 * of 2^table_order Jacobian rows, entry j of table t = sum of points t*table_order + b over the
 * set bits b of j (points past n are infinity); x rows affine (add_last) or Jacobian.  Rows
 * are returned normalised (Z = 1; infinity (0, 1, 0)): the same points as the reference's. */
void ec_inittable_h(uint32_t *x, uint32_t *ectable, uint32_t n, uint32_t table_order, uint32_t pidx,
                    uint32_t add_last);
void ec2_inittable_h(uint32_t *x, uint32_t *ectable, uint32_t n, uint32_t table_order, uint32_t pidx,
                     uint32_t add_last);
/* ec.cpp:131 / :462 (and ec2_jacadd_h / ec2_jacdouble_h) -- one Jacobian addition / doubling;
 * the result is returned normalised (Z = 1; infinity (0, 1, 0)): the reference's point. */
void ec_jacadd_h(uint32_t *z, uint32_t *x, uint32_t *y, uint32_t pidx);
void ec2_jacadd_h(uint32_t *z, uint32_t *x, uint32_t *y, uint32_t pidx);
void ec_jacdouble_h(uint32_t *z, uint32_t *x, uint32_t pidx);
void ec2_jacdouble_h(uint32_t *z, uint32_t *x, uint32_t pidx);
/* mpoly.cpp:266 / :278 -- the mpoly's coefficient values (layout mpoly.cpp:195) from / to
 * Montgomery form in place (converted on the GPU). */
void mpoly_from_montgomery_h(uint32_t *x, uint32_t pidx);
void mpoly_to_montgomery_h(uint32_t *x, uint32_t pidx);
/* U = A + B mod 2^256 (the reference's addu256_h); ff.cpp:626 rangeu256_h: samples[i] =
 * start + i inc, reduced below mod (if not NULL) by repeated subtraction. */
void addu256_h(uint32_t *U, const uint32_t *A, const uint32_t *B);
void rangeu256_h(uint32_t *samples, uint32_t nsamples, const uint32_t *start, uint32_t inc, const uint32_t *mod);
/* ec.cpp:1153 / :1164 -- infinity flags with the reference's row addressing (G1: rows start
 * 2 j words into x; G2: every flag tests the row at word 4). */
void ec_isinf(uint32_t *z, const uint32_t *x, const uint32_t n, const uint32_t pidx);
void ec2_isinf(uint32_t *z, const uint32_t *x, const uint32_t n, const uint32_t pidx);
/* bigint.cpp:72 -- indices 0..len-1, sorted (std::sort) by the top word of v[i] if sort_en. */
void sortu256_idx_h(uint32_t *idx, const uint32_t *v, uint32_t len, uint32_t sort_en);
/* ntt.cpp:1116 -- transform decomposition of nsamples (types.h fft_params_t layout). */
#ifndef CS_REFERENCE_TYPES
typedef enum { FFT_T_1D = 0, FFT_T_2D, FFT_T_3D, FFT_T_4D, FFT_T_N } fft_t;
typedef struct {
  fft_t fft_type;
  uint32_t fft_N[1 << (FFT_T_N - 1)];
  uint32_t padding;
  uint32_t levels;
} fft_params_t;
#endif
void ntt_build_h(fft_params_t *ntt_params, uint32_t nsamples);
/* init.cpp:44 / :54 (no roots files are read: twiddles are made on the device), and
 * utils_host get_nprocs_h. */
void init_h(void);
void release_h(void);
uint32_t get_nprocs_h(void);
/* file_utils.cpp: raw little-endian words; witness .bin values after a 4-word header
 * (fmt 1), .dat values from byte 32 (fmt 0). */
void readU256CircuitFile_h(uint32_t *samples, const char *filename, unsigned long long nwords);
void readU256PKFile_h(uint32_t *samples, const char *filename, unsigned long long nwords);
/* types.h cirbin_hfile_t / pkbin_hfile_t and file_utils.cpp:49 / :447: the leading header
 * words of a circuit file (9 x uint64) and of a proving-key file (9 x uint32, read in order,
 * so domainSize receives the file's domainBits word, as in the reference). */
#ifndef CS_REFERENCE_TYPES
typedef struct {
  unsigned long long nWords, nPubInputs, nOutputs, nVars, nConstraints, cirformat, R1CSA_nWords,
      R1CSB_nWords, R1CSC_nWords;
} cirbin_hfile_t;
typedef struct {
  uint32_t nWords, ftype, protocol, Rbitlen, k_binformat, k_ecformat, nVars, nPublic, domainSize;
} pkbin_hfile_t;
#endif
void readU256CircuitFileHeader_h(cirbin_hfile_t *hfile, const char *filename);
void readU256PKFileHeader_h(pkbin_hfile_t *hfile, const char *filename);
void readU256DataFile_h(uint32_t *samples, const char *filename, uint32_t insize, uint32_t outsize);
void readU256DataFileFromOffset_h(uint32_t *samples, const char *filename, unsigned long long woffset,
                                  unsigned long long nwords);
void writeU256DataFile_h(uint32_t *samples, const char *filename, unsigned long long nwords);
void appendU256DataFile_h(uint32_t *samples, const char *filename, unsigned long long nwords);
void readWitnessFile_h(uint32_t *samples, const char *filename, uint32_t fmt, unsigned long long inlen);
void writeWitnessFile_h(uint32_t *samples, const char *filename, unsigned long long nwords);

/* The rest of what the reference's Cython layer binds (src/cython/_utils_host.pxd), exported
 * so that its module links against this library unchanged.
 *   shared_new_h / shared_free_h (utils_host.cpp:156 / :180): the System V shared-memory
 *     witness buffer (key 123456) the reference's processes exchange; same behaviour.
 *   readR1CSFileHeader_h / readR1CSFile_h (file_utils.cpp), r1cs_to_mpoly_len_h /
 *     r1cs_to_mpoly_h (mpoly.cpp:201): circuit compilation, before proving -- not on this
 *     library's path (it reads compiled proving keys); they zero their outputs and report
 *     CS_ERR_UNSUPPORTED in cs_last_status().
 *   readECTablesNElementsFile_h: precomputed EC table files, refused like the table-file
 *     option of ec_jacreduce_server_h (CS_ERR_UNSUPPORTED). */
#ifndef CS_REFERENCE_TYPES
/* r1csv1_t, r1cs_idx_t, ec_table_offset_t: reference src/cuda/types.h:581-626 */
typedef struct {
  uint32_t magic_number, version, nsections, word_width_bytes, nVars, nPubOutputs, nPubInputs, nPrivInputs;
  unsigned long long nLabels;
  uint32_t nConstraints, R1CSA_nCoeff, R1CSB_nCoeff, R1CSC_nCoeff, constraintOffset;
  long long constraintLen;
} r1csv1_t;
typedef enum { R1CSA_IDX = 0, R1CSB_IDX = 1, R1CSC_IDX = 2, R1CS_N_IDX = 3 } r1cs_idx_t;
typedef struct {
  uint32_t table_order;
  unsigned long long woffset_A, woffset_B2, woffset_B1, woffset_C, woffset_hExps, nwords_tdata;
} ec_table_offset_t;
#endif
int shared_new_h(void **shmem, unsigned long long size);
void shared_free_h(void *shmem, int shmid);
void readR1CSFileHeader_h(r1csv1_t *r1cs_hdr, const char *filename);
void readR1CSFile_h(uint32_t *samples, const char *filename, r1csv1_t *r1cs, r1cs_idx_t r1cs_idx);
void r1cs_to_mpoly_len_h(uint32_t *plen_out, uint32_t *cin, cirbin_hfile_t *header, uint32_t extend);
void r1cs_to_mpoly_h(uint32_t *pout, uint32_t *cin, cirbin_hfile_t *header, uint32_t to_mont, uint32_t pidx,
                     uint32_t extend);
void readECTablesNElementsFile_h(ec_table_offset_t *table_offset, const char *filename);

/* G1 multi-exponentiation that allocates nothing (no counterpart in the reference).
 * For callers whose device memory is owned by a host framework's pool and who may not
 * call cudaMalloc themselves, or cannot afford its implicit synchronisation on a
 * latency-critical path.  Inputs and output are the caller's device pointers (same
 * layout as cs_msm_device, automatic window); scratch is a fixed file-scope device array
 * of cs_msm_noalloc_scratch_bytes() bytes (32 MiB) that every GPU loading this library
 * keeps reserved until exit, which bounds n to cs_msm_g1_noalloc_max_terms() (at least
 * 2^16; query the function rather than hard-coding a figure: 69,843 with the current
 * automatic window); larger n is rejected with CS_ERR_ARG and a message in
 * cs_msm_g1_noalloc_error().
 * Runs asynchronously on `stream` (a cudaStream_t, NULL = legacy default stream).  The
 * first call on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture.  Every call shares
 * the array: calls that overlap on the GPU race, so order them on one stream. */
int cs_msm_g1_noalloc(const uint32_t *d_scalars, const uint32_t *d_points, uint32_t n,
                      uint32_t *d_out_affine, void *stream);
size_t cs_msm_noalloc_scratch_bytes(void);
uint32_t cs_msm_g1_noalloc_max_terms(void);
const char *cs_msm_g1_noalloc_error(void);

/* --------------------------------------------------------------- Groth16 prove ----- */
/* Proving key as the reference stores it (src/python/pysnarks_utils.py pkvars_to_bin with
 * the extension of :653-657), Montgomery affine points:
 *   A, B1: n_vars + 2 G1 points (A ++ alpha_1 ++ delta_1, B1 ++ beta_1 ++ delta_1),
 *   B2: n_vars + 2 G2 points (B2 ++ beta_2 ++ delta_2), C: n_vars G1 points (entries below
 *   n_public + 1 unused), hExps: domain_size - 1 G1 points, delta_1: one G1 point,
 *   polsA / polsB: QAP matrices in the mpoly layout (polsA extended with the public rows). */
typedef struct {
  uint32_t n_vars, n_public, domain_size;
  const uint32_t *polsA; size_t polsA_words; uint32_t polsA_entries;
  const uint32_t *polsB; size_t polsB_words; uint32_t polsB_entries;
  const uint32_t *A, *B1, *B2, *C, *hExps, *delta_1;
} cs_pk_desc;
typedef struct cs_pk cs_pk;

/* Uploads (on_device = 0: host pointers) or copies (1: device pointers) the key into HBM,
 * transposes the QAP matrices into constraint rows and builds the NTT tables; the key
 * then serves any number of proofs. */
int cs_pk_create(cs_ctx *ctx, const cs_pk_desc *desc, int on_device, cs_pk **out);
void cs_pk_destroy(cs_pk *pk);
size_t cs_prove_workspace_bytes(const cs_pk *pk);
/* Builds fixed-base tables (cs_msm_fixed_*) for the key's five MSMs (window > 0: that
 * window for all; 0: chosen per MSM) or drops them (window < 0); cs_prove uses the tables
 * whenever the key has them.  About 13 x the G1/G2 point bytes at 2^20 (~5 GiB).
 * Synchronises the context's streams first.  cs_pk_device_bytes: HBM the key holds;
 * cs_pk_fixed_window: window of table `which` (0 A, 1 B1, 2 B2, 3 C, 4 H; 0 = none). */
int cs_pk_fixed_base(cs_ctx *ctx, cs_pk *pk, int window);
size_t cs_pk_device_bytes(const cs_pk *pk);
int cs_pk_fixed_window(const cs_pk *pk, int which);
/* Groth16 proof for witness w (n_vars normal-form elements, w[0] = 1), blinding r and s
 * (normal form, host pointers): proof = pi_A (16 words) | pi_B (32) | pi_C (16), affine
 * Montgomery, the reference prover's pi_a_eccf1 / pi_b_eccf2 / pi_c_eccf1
 * (groth_prover.py:1245 gen_proof; CPU sequence :575-790 and :1414-1453).
 * cs_prove: host witness and proof, synchronous.  cs_prove_device: device witness and
 * proof buffers, asynchronous on the context stream (r and s are read at call time).
 * The launch sequence after the scalar uploads is captured as a CUDA graph on the first
 * proof with a given key, witness buffer and scratch arena on a context, and replayed by
 * later proofs with the same three (one graph launch instead of ~150 API calls per proof). */
int cs_prove(cs_ctx *ctx, cs_pk *pk, const uint32_t *w, const uint32_t *r, const uint32_t *s,
             uint32_t *proof);
int cs_prove_device(cs_ctx *ctx, cs_pk *pk, const uint32_t *d_w, const uint32_t *r, const uint32_t *s,
                    uint32_t *d_proof);
/* k proofs with one key in one pass (no counterpart in the reference, which proves one at a
 * time): the A, B1 and C MSMs of all k proofs run as one batched G1 multi-exponentiation (one
 * sort, one accumulation over every instance's buckets, the key's fixed-base tables), the B2
 * MSMs as one G2 batch and the H MSMs as one G1 batch after the per-proof QAP and H steps;
 * the sequence is captured as a CUDA graph per context, key and k.  d_w, d_proof: host arrays
 * of k device pointers (witnesses, 64-word proofs); r, s: k x 8 words each, host.  Same proof
 * bytes as k calls of cs_prove_device.  1 <= k <= 64; a key without fixed-base tables, or
 * k = 1, proves one by one.  Asynchronous on the context stream. */
int cs_prove_batch_device(cs_ctx *ctx, cs_pk *pk, uint32_t k, const uint32_t *const *d_w, const uint32_t *r,
                          const uint32_t *s, uint32_t *const *d_proof);
/* Stage completion times (ms after the start) of the context's last finished proof: A, B1,
 * B2 (G2), C MSM chains, H step, H MSM, whole proof (up to n of them; the reference prover's
 * t_GP phase dict).  Call after the proof has completed (cs_prove, or cs_ctx_sync).  Graph
 * replays carry no stage events: CS_ERR_UNSUPPORTED after one (turn graphs off to time stages). */
int cs_ctx_prove_stages(cs_ctx *ctx, float *ms, int n);
/* Proof graphs on this context on (default) or off (off also frees the captured graphs). */
int cs_ctx_set_prove_graphs(cs_ctx *ctx, int enable);

/* ----------------------------------------------- served proving (continuous batching) */
/* Replaces the reference's one-proof-at-a-time server loop (groth_prover.py:808-891
 * startServer, which drops requests that arrive while a proof runs and re-copies the
 * proving key per proof).  `slots` worker threads each own a context (streams, scratch
 * arena, twiddles); requests queue FIFO and start as soon as a slot is free and free
 * device memory minus the bytes promised to admitted requests covers the slot's scratch
 * growth plus reserve_bytes.  Admitted proofs run concurrently on the device.  A request
 * whose scratch can never fit (no proof running) fails with CS_ERR_NOMEM.
 * Keys (cs_pk, created on the same device) must outlive the server.  w and proof
 * (host memory, as cs_prove) must stay valid until cs_server_wait returns for the ticket.
 * cs_server_wait: timeout_s < 0 waits for good; returns the proof's status, or
 * CS_ERR_TIMEOUT with the request still pending (wait again). */
typedef struct cs_server cs_server;
typedef struct {
  int status;
  double queue_ms;    /* submit -> start on a slot */
  double latency_ms;  /* submit -> proof in host memory */
  float device_ms;    /* device time of the prove kernels (CUDA events) */
} cs_server_result;
typedef struct {
  uint64_t completed, failed, rejected, cancelled;
  uint64_t queued;
  uint32_t running, max_concurrent;
  size_t promised_bytes;
  double p50_ms, p99_ms;            /* latency (submit -> done) over the last 1024 proofs */
  size_t hbm_free_bytes, hbm_total_bytes;
  uint64_t batched;         /* proofs that ran in a same-key batch of two or more */
  uint64_t batches;         /* such batches */
  uint32_t max_batch_seen;  /* largest batch so far */
} cs_server_counters;
int cs_server_create(int device, int slots, size_t reserve_bytes, cs_server **out);
void cs_server_destroy(cs_server *srv);
int cs_server_add_key(cs_server *srv, cs_pk *pk, int *key_id);
int cs_server_submit(cs_server *srv, int key_id, const uint32_t *w, const uint32_t *r, const uint32_t *s,
                     uint32_t *proof, uint64_t *ticket);
int cs_server_wait(cs_server *srv, uint64_t ticket, double timeout_s, cs_server_result *res);
int cs_server_stats(cs_server *srv, cs_server_counters *st);
/* Same-key batching: a slot that takes a request whose key has at most 2^16 constraints (and
 * fixed-base tables) takes up to k - 1 more queued requests with that key along and proves
 * them in one cs_prove_batch_device pass (k the largest power of two <= max_batch that the
 * queue fills, at least 4; fewer run one by one).  Proof bytes are those of lone proofs.
 * Default 16; below 4 turns batching off; 1 <= max_batch <= 64. */
int cs_server_set_max_batch(cs_server *srv, int max_batch);
/* Removes a request that is still queued (its wait returns CS_ERR_CANCELLED); CS_ERR_ARG when
 * the request is unknown, already running or finished. */
int cs_server_cancel(cs_server *srv, uint64_t ticket);
const char *cs_server_error(cs_server *srv);

/* ------------------------------------------- proving-key generation (setup) -------- */
/* Device kernels for building proving keys (the quantities of the reference's
 * groth_setup.py calculateValuesAtT :771 / calculateEncryptedValuesAtT :488); all Fr
 * values Montgomery unless noted, device pointers, asynchronous on the context stream.
 *   cs_setup_lagrange:   out[c] = L_c(t) = w^c (t^m - 1) / (m (t - w^c)), c < m = 2^log_m.
 *   cs_setup_wire_eval:  out[i] = sum_c M[i][c] L[c] for the mpoly-layout matrix M (rows of
 *                        index >= n_rows ignored), i.e. u_i(t) / v_i(t) / w_i(t).
 *   cs_setup_c_scalars:  out[i] = (beta u_i + alpha v_i + w_i) k, normal form (k = 1/delta
 *                        for C, 1/gamma for the verifying key's IC).
 *   cs_setup_pow_scalars: out[j] = t^j k, j < n, normal form (k = Z(t)/delta: hExps).
 *   cs_r1cs_layer_eval:  out[c] = (A_c . w)(B_c . w), normal form, for CSR rows with
 *                        Montgomery coefficients and a normal-form witness (evaluates the
 *                        outputs of one layer of a synthetic circuit). */
int cs_setup_lagrange(cs_ctx *ctx, uint32_t log_m, const uint32_t *d_t, uint32_t *d_out);
int cs_setup_wire_eval(cs_ctx *ctx, const uint32_t *d_mpoly, uint32_t n_wires, const uint32_t *d_L,
                       uint32_t n_rows, uint32_t *d_out);
int cs_setup_c_scalars(cs_ctx *ctx, const uint32_t *d_u, const uint32_t *d_v, const uint32_t *d_w,
                       const uint32_t *d_alpha, const uint32_t *d_beta, const uint32_t *d_k, uint32_t n,
                       uint32_t *d_out);
int cs_setup_pow_scalars(cs_ctx *ctx, const uint32_t *d_t, const uint32_t *d_k, uint32_t n, uint32_t *d_out);
int cs_r1cs_layer_eval(cs_ctx *ctx, const uint32_t *a_off, const uint32_t *a_wire, const uint32_t *a_coeff,
                       const uint32_t *b_off, const uint32_t *b_wire, const uint32_t *b_coeff, uint32_t n_rows,
                       const uint32_t *d_w, uint32_t *d_out);

/* ------------------------------------------------------------ measurement ----------- */
/* Instruction-rate probes (ops per second, all SMs): mode 1 mad.lo.u32, 2 mad.hi.u32,
 * 3 mad.wide.u32, 4 fma.rn.f64, 5 carry-chained mad.lo.cc/madc.hi.cc. */
int cs_bench_pipe(cs_ctx *ctx, int mode, double *ops_per_s);
/* Number of kernels this library has launched in the process so far. */
unsigned long long cs_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* CUSNARKS_B200_H */
