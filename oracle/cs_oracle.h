/*
 * cs_oracle.h -- CPU restatement of the reference (druiz0992/cusnarks) Groth16/BN128
 * prover hot path.  TEST INFRASTRUCTURE ONLY: it is the checker that tests/, the smoke
 * check and bench.py's CPU baseline leg compare the CUDA library against.  Nothing in
 * the product library links, loads or calls it.
 *
 * Conventions (same as the reference, src/cuda/types.h):
 *   - a field element is 8 little-endian uint32 limbs (NWORDS_256BIT = 8);
 *   - pidx 0 = BN254 base field q (MOD_GROUP), pidx 1 = scalar field r (MOD_FIELD);
 *   - "Montgomery" means x * 2^256 mod p;
 *   - G1 affine = (X, Y) 16 words, G1 Jacobian = (X, Y, Z) 24 words;
 *   - G2 affine = (X.c0, X.c1, Y.c0, Y.c1) 32 words, G2 Jacobian 48 words;
 *   - the point at infinity is (0, 1_mont) for G1 and (0, 0, 1_mont, 0) for G2
 *     (src/cuda/constants.cpp:264-292), Jacobian infinity has X = 0, Y = 1_mont.
 */
#ifndef CS_ORACLE_H
#define CS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* field, pidx selects the modulus */
void or_montmult(uint32_t *z, const uint32_t *a, const uint32_t *b, uint32_t pidx);
void or_addm(uint32_t *z, const uint32_t *a, const uint32_t *b, uint32_t pidx);
void or_subm(uint32_t *z, const uint32_t *a, const uint32_t *b, uint32_t pidx);
void or_to_mont(uint32_t *z, const uint32_t *a, uint32_t n, uint32_t pidx);
void or_from_mont(uint32_t *z, const uint32_t *a, uint32_t n, uint32_t pidx);
void or_montinv(uint32_t *z, const uint32_t *a, uint32_t pidx);
void or_montmult_ext(uint32_t *z, const uint32_t *a, const uint32_t *b, uint32_t pidx);
void or_get_const(uint32_t *one_mont, uint32_t *r2, uint32_t pidx);

/* curve */
void or_ec_jacadd(uint32_t *z, const uint32_t *x, const uint32_t *y, uint32_t ec2);
void or_ec_jacdouble(uint32_t *z, const uint32_t *x, uint32_t ec2);
void or_ec_jacaddmixed(uint32_t *z, const uint32_t *x_aff, const uint32_t *y_jac, uint32_t ec2);
void or_ec_jac2aff(uint32_t *y, const uint32_t *x, uint32_t n, uint32_t ec2);
void or_ec_scmul(uint32_t *z_aff, const uint32_t *scl, const uint32_t *x_aff, uint32_t n, uint32_t ec2);
uint32_t or_ec_isoncurve_aff(const uint32_t *x_aff, uint32_t ec2);

/* multi-exponentiation: out_aff = sum scl[i] * x[i] (scalars normal form, any 256-bit
 * value; points affine Montgomery).  order = subset-sum table width (reference default 6). */
void or_msm(uint32_t *out_aff, const uint32_t *scl, const uint32_t *x_aff, uint32_t n,
            uint32_t ec2, uint32_t order, uint32_t nthreads);

/* number-theoretic transforms over pidx with a caller-provided roots table */
void or_ntt(uint32_t *A, const uint32_t *roots, uint32_t levels, uint64_t astride,
            uint64_t rstride, int32_t direction, uint32_t pidx);
void or_intt(uint32_t *A, const uint32_t *roots, uint32_t fmat, uint32_t levels,
             uint64_t rstride, uint32_t pidx);
void or_find_roots(uint32_t *roots, uint32_t levels);
void or_root_powers(uint32_t *roots, const uint32_t *proot, uint64_t n);
void or_primitive_root(uint32_t *root_mont, uint32_t levels);

/* H step, reference semantics: M (2m words*8, normal form) = coefficients of A(x)*B(x) */
void or_interpolandmul(uint32_t *M, const uint32_t *A, const uint32_t *B,
                       const uint32_t *roots, uint32_t levels, uint64_t rstride);
/* H step, coset variant: H (m coefficients, normal form) of (A*B - C)/(x^m - 1)
 * evaluated on the coset g*<w>, g = multiplicative generator 5 of Fr. */
void or_hstep_coset(uint32_t *H, const uint32_t *A, const uint32_t *B, const uint32_t *C,
                    uint32_t levels);

/* sparse QAP evaluation, reference mpoly layout */
void or_mpoly_eval(uint32_t *pout, const uint32_t *scalar, const uint32_t *pin,
                   uint32_t start_idx, uint32_t last_idx, uint32_t pidx);

/* batched Montgomery products of any 256-bit operands (reduced mod p first) */
void or_montmult_batch(uint32_t *z, const uint32_t *a, const uint32_t *b, uint64_t n, uint32_t pidx);

/* the benchmark circuit's witness and proving key without a GPU */
void or_r1cs_eval(uint32_t *w, uint64_t first_out, uint64_t nc, uint32_t per_row,
                  const uint32_t *a_wire, const uint32_t *a_coeff,
                  const uint32_t *b_wire, const uint32_t *b_coeff);
void or_lagrange_at(uint32_t *out, uint32_t levels, const uint32_t *t_mont);
void or_wire_eval(uint32_t *out, const uint32_t *mpoly, const uint32_t *Lc, uint32_t n_rows);
void or_c_scalars(uint32_t *out, const uint32_t *u, const uint32_t *v, const uint32_t *w,
                  const uint32_t *alpha, const uint32_t *beta, const uint32_t *k, uint64_t n);
void or_pow_scalars(uint32_t *out, const uint32_t *t_mont, const uint32_t *k, uint64_t n);
void or_fixed_base_mul(uint32_t *out_aff, const uint32_t *scl, uint64_t n, const uint32_t *base_aff,
                       uint32_t ec2);

#ifdef __cplusplus
}
#endif
#endif
