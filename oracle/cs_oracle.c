/*
 * cs_oracle.c -- CPU restatement of the reference (druiz0992/cusnarks) Groth16/BN128
 * prover hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: tests/, the smoke check and the
 * CPU baseline leg of bench.py use it to check (and to time beside) the CUDA library.
 * The product library never links, loads or calls it.
 *
 * Each function names the reference routine it restates (paths inside the reference
 * project).  Arithmetic is written independently: 4x64-bit CIOS Montgomery products
 * with a final conditional subtraction, so every field result is the unique value in
 * [0, p) -- the same words the reference's FIOS C code or its ADX assembly return.
 */
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "cs_oracle.h"

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------------------
 * Moduli.  pidx 0 = q (MOD_GROUP, base field of BN254), pidx 1 = r (MOD_FIELD, scalar
 * field).  Values: src/cuda/ff.cpp:487-490 (decimal there); the Montgomery constants
 * (n0', R mod p, R^2 mod p) are derived here at first use instead of being tabulated.
 * ---------------------------------------------------------------------------------- */
typedef struct {
  uint64_t p[4];
  uint64_t one[4];   /* R mod p  (Montgomery 1) */
  uint64_t r2[4];    /* R^2 mod p */
  uint64_t n0;       /* -p^{-1} mod 2^64 */
} modctx_t;

static modctx_t MODS[2] = {
  {{0x3c208c16d87cfd47ull, 0x97816a916871ca8dull, 0xb85045b68181585dull, 0x30644e72e131a029ull}, {0}, {0}, 0},
  {{0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull, 0x30644e72e131a029ull}, {0}, {0}, 0},
};
static int g_inited = 0;

static int geq4(const uint64_t *a, const uint64_t *b) {
  for (int i = 3; i >= 0; i--) {
    if (a[i] > b[i]) return 1;
    if (a[i] < b[i]) return 0;
  }
  return 1;
}
static uint64_t sub4(uint64_t *z, const uint64_t *a, const uint64_t *b) {
  uint64_t br = 0;
  for (int i = 0; i < 4; i++) {
    u128 d = (u128)a[i] - b[i] - br;
    z[i] = (uint64_t)d;
    br = (uint64_t)(d >> 64) & 1;
  }
  return br;
}
static uint64_t add4(uint64_t *z, const uint64_t *a, const uint64_t *b) {
  uint64_t c = 0;
  for (int i = 0; i < 4; i++) {
    u128 s = (u128)a[i] + b[i] + c;
    z[i] = (uint64_t)s;
    c = (uint64_t)(s >> 64);
  }
  return c;
}
static void fadd(uint64_t *z, const uint64_t *a, const uint64_t *b, const modctx_t *m) {
  uint64_t t[4];
  uint64_t c = add4(t, a, b);
  if (c || geq4(t, m->p)) sub4(t, t, m->p);
  memcpy(z, t, 32);
}
static void fsub(uint64_t *z, const uint64_t *a, const uint64_t *b, const modctx_t *m) {
  uint64_t t[4];
  if (sub4(t, a, b)) add4(t, t, m->p);
  memcpy(z, t, 32);
}
/* CIOS Montgomery product a*b*2^-256 mod p, inputs < p, output in [0, p). */
static void fmul(uint64_t *z, const uint64_t *a, const uint64_t *b, const modctx_t *m) {
  uint64_t t[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++) {
    u128 c = 0;
    for (int j = 0; j < 4; j++) {
      c += (u128)a[j] * b[i] + t[j];
      t[j] = (uint64_t)c;
      c >>= 64;
    }
    c += t[4];
    t[4] = (uint64_t)c;
    t[5] = (uint64_t)(c >> 64);
    uint64_t q = t[0] * m->n0;
    c = ((u128)q * m->p[0] + t[0]) >> 64;
    for (int j = 1; j < 4; j++) {
      c += (u128)q * m->p[j] + t[j];
      t[j - 1] = (uint64_t)c;
      c >>= 64;
    }
    c += t[4];
    t[3] = (uint64_t)c;
    t[4] = t[5] + (uint64_t)(c >> 64);
  }
  if (t[4] || geq4(t, m->p)) sub4(t, t, m->p);
  memcpy(z, t, 32);
}

static void init_mods(void) {
  if (g_inited) return;
  for (int k = 0; k < 2; k++) {
    modctx_t *m = &MODS[k];
    uint64_t inv = 1;
    for (int i = 0; i < 7; i++) inv *= 2 - m->p[0] * inv;  /* Newton: p*inv = 1 mod 2^64 */
    m->n0 = (uint64_t)0 - inv;
    uint64_t x[4] = {1, 0, 0, 0};
    for (int i = 0; i < 512; i++) {
      fadd(x, x, x, m);
      if (i == 255) memcpy(m->one, x, 32);
    }
    memcpy(m->r2, x, 32);
  }
  g_inited = 1;
}

static void fpow(uint64_t *z, const uint64_t *a_mont, const uint64_t *e, const modctx_t *m) {
  uint64_t acc[4];
  memcpy(acc, m->one, 32);
  for (int i = 255; i >= 0; i--) {
    fmul(acc, acc, acc, m);
    if ((e[i >> 6] >> (i & 63)) & 1) fmul(acc, acc, a_mont, m);
  }
  memcpy(z, acc, 32);
}
static void finv(uint64_t *z, const uint64_t *a_mont, const modctx_t *m) {
  uint64_t e[4], two[4] = {2, 0, 0, 0};
  sub4(e, m->p, two);
  fpow(z, a_mont, e, m);
}

/* ---------------------------------------- public field API (src/cuda/ff.cpp) ------ */
void or_montmult(uint32_t *z, const uint32_t *a, const uint32_t *b, uint32_t pidx) {
  init_mods();
  uint64_t x[4], y[4], t[4];
  memcpy(x, a, 32); memcpy(y, b, 32);
  fmul(t, x, y, &MODS[pidx]);
  memcpy(z, t, 32);
}
void or_addm(uint32_t *z, const uint32_t *a, const uint32_t *b, uint32_t pidx) {
  init_mods();
  uint64_t x[4], y[4], t[4];
  memcpy(x, a, 32); memcpy(y, b, 32);
  fadd(t, x, y, &MODS[pidx]);
  memcpy(z, t, 32);
}
void or_subm(uint32_t *z, const uint32_t *a, const uint32_t *b, uint32_t pidx) {
  init_mods();
  uint64_t x[4], y[4], t[4];
  memcpy(x, a, 32); memcpy(y, b, 32);
  fsub(t, x, y, &MODS[pidx]);
  memcpy(z, t, 32);
}
/* to_montgomeryN_h (ff.cpp): z = a * R mod p.  Inputs >= p are reduced first, as the
 * reference's Montgomery product by R^2 does for any a < 2^256. */
void or_to_mont(uint32_t *z, const uint32_t *a, uint32_t n, uint32_t pidx) {
  init_mods();
  const modctx_t *m = &MODS[pidx];
  for (uint32_t i = 0; i < n; i++) {
    uint64_t x[4], t[4];
    memcpy(x, a + 8 * i, 32);
    fmul(t, x, m->r2, m);
    memcpy(z + 8 * i, t, 32);
  }
}
void or_from_mont(uint32_t *z, const uint32_t *a, uint32_t n, uint32_t pidx) {
  init_mods();
  const modctx_t *m = &MODS[pidx];
  uint64_t one[4] = {1, 0, 0, 0};
  for (uint32_t i = 0; i < n; i++) {
    uint64_t x[4], t[4];
    memcpy(x, a + 8 * i, 32);
    fmul(t, x, one, m);
    memcpy(z + 8 * i, t, 32);
  }
}
/* montinv_h (ff.cpp:745): Montgomery inverse, (aR)^-1 R.  Fermat exponentiation here;
 * the inverse is unique so the reference's almost-inverse gives the same words. */
void or_montinv(uint32_t *z, const uint32_t *a, uint32_t pidx) {
  init_mods();
  uint64_t x[4], t[4];
  memcpy(x, a, 32);
  finv(t, x, &MODS[pidx]);
  memcpy(z, t, 32);
}
void or_get_const(uint32_t *one_mont, uint32_t *r2, uint32_t pidx) {
  init_mods();
  if (one_mont) memcpy(one_mont, MODS[pidx].one, 32);
  if (r2) memcpy(r2, MODS[pidx].r2, 32);
}

/* ------------------------------------------------------- Fp2 = Fq[u]/(u^2 + 1) --- */
/* montmult_ext_h (ff.cpp:389): 3-multiplication Karatsuba, non-residue -1. */
static void f2mul(uint64_t *z, const uint64_t *a, const uint64_t *b, const modctx_t *m) {
  uint64_t v0[4], v1[4], sa[4], sb[4], t[4];
  fmul(v0, a, b, m);
  fmul(v1, a + 4, b + 4, m);
  fadd(sa, a, a + 4, m);
  fadd(sb, b, b + 4, m);
  fmul(t, sa, sb, m);
  fsub(t, t, v0, m);
  fsub(z + 4, t, v1, m);
  fsub(z, v0, v1, m);
}
static void f2add(uint64_t *z, const uint64_t *a, const uint64_t *b, const modctx_t *m) {
  fadd(z, a, b, m); fadd(z + 4, a + 4, b + 4, m);
}
static void f2sub(uint64_t *z, const uint64_t *a, const uint64_t *b, const modctx_t *m) {
  fsub(z, a, b, m); fsub(z + 4, a + 4, b + 4, m);
}
static void f2inv(uint64_t *z, const uint64_t *a, const modctx_t *m) {
  uint64_t n0[4], n1[4], d[4], di[4], zero[4] = {0, 0, 0, 0};
  fmul(n0, a, a, m);
  fmul(n1, a + 4, a + 4, m);
  fadd(d, n0, n1, m);
  finv(di, d, m);
  fmul(z, a, di, m);
  fmul(n1, a + 4, di, m);
  fsub(z + 4, zero, n1, m);
}
void or_montmult_ext(uint32_t *z, const uint32_t *a, const uint32_t *b, uint32_t pidx) {
  init_mods();
  uint64_t x[8], y[8], t[8];
  memcpy(x, a, 64); memcpy(y, b, 64);
  f2mul(t, x, y, &MODS[pidx]);
  memcpy(z, t, 64);
}

/* ------------------------------------------------------------------------ curve --- */
/* Generic over Fq (w = 4 words of 64 bits) and Fq2 (w = 8). */
typedef struct {
  int w;
  void (*mul)(uint64_t *, const uint64_t *, const uint64_t *, const modctx_t *);
  void (*add)(uint64_t *, const uint64_t *, const uint64_t *, const modctx_t *);
  void (*sub)(uint64_t *, const uint64_t *, const uint64_t *, const modctx_t *);
} fops_t;
static const fops_t FOPS[2] = {{4, fmul, fadd, fsub}, {8, f2mul, f2add, f2sub}};
#define MAXW 8

static int e_iszero(const uint64_t *a, int w) {
  for (int i = 0; i < w; i++) if (a[i]) return 0;
  return 1;
}
static void e_one(uint64_t *a, int w) {
  memset(a, 0, 8 * w);
  memcpy(a, MODS[0].one, 32);
}
/* Jacobian point: X | Y | Z, each w words */
static void pt_inf(uint64_t *P, int w) {
  memset(P, 0, 3 * 8 * w);
  e_one(P + w, w);
}
static int pt_isinf(const uint64_t *P, int w) { return e_iszero(P + 2 * w, w); }

/* ec_jacdouble_h (src/cuda/ec.cpp:462): S = 4XY^2, M = 3X^2, X' = M^2 - 2S,
 * Y' = M(S - X') - 8Y^4, Z' = 2YZ. */
static void pt_double(uint64_t *R, const uint64_t *P, const fops_t *f) {
  const modctx_t *m = &MODS[0];
  int w = f->w;
  if (pt_isinf(P, w)) { memmove(R, P, 3 * 8 * w); return; }
  uint64_t X[MAXW], Y[MAXW], Z[MAXW], ysq[MAXW], y4[MAXW], S[MAXW], M[MAXW], t[MAXW];
  memcpy(X, P, 8 * w); memcpy(Y, P + w, 8 * w); memcpy(Z, P + 2 * w, 8 * w);
  f->mul(ysq, Y, Y, m);
  f->mul(y4, ysq, ysq, m);
  f->mul(S, X, ysq, m);
  f->add(S, S, S, m); f->add(S, S, S, m);
  f->mul(M, X, X, m);
  f->add(t, M, M, m); f->add(M, t, M, m);
  f->mul(R, M, M, m);
  f->sub(R, R, S, m); f->sub(R, R, S, m);
  f->mul(R + 2 * w, Y, Z, m);
  f->add(R + 2 * w, R + 2 * w, R + 2 * w, m);
  f->add(t, y4, y4, m); f->add(t, t, t, m); f->add(t, t, t, m);
  f->sub(S, S, R, m);
  f->mul(S, M, S, m);
  f->sub(R + w, S, t, m);
}

/* ec_jacadd_h (src/cuda/ec.cpp:131): U1 = X1 Z2^2, U2 = X2 Z1^2, S1 = Y1 Z2^3,
 * S2 = Y2 Z1^3; equal U with equal S doubles, opposite S gives infinity. */
static void pt_add(uint64_t *R, const uint64_t *P, const uint64_t *Q, const fops_t *f) {
  const modctx_t *m = &MODS[0];
  int w = f->w;
  if (pt_isinf(P, w)) { memmove(R, Q, 3 * 8 * w); return; }
  if (pt_isinf(Q, w)) { memmove(R, P, 3 * 8 * w); return; }
  uint64_t z1s[MAXW], z1c[MAXW], z2s[MAXW], z2c[MAXW], U1[MAXW], U2[MAXW], S1[MAXW], S2[MAXW];
  uint64_t H[MAXW], Rr[MAXW], H2[MAXW], H3[MAXW], X3[MAXW], Y3[MAXW], Z3[MAXW], t[MAXW];
  f->mul(z1s, P + 2 * w, P + 2 * w, m);
  f->mul(z1c, z1s, P + 2 * w, m);
  f->mul(z2s, Q + 2 * w, Q + 2 * w, m);
  f->mul(z2c, z2s, Q + 2 * w, m);
  f->mul(U1, P, z2s, m);
  f->mul(U2, Q, z1s, m);
  f->mul(S1, P + w, z2c, m);
  f->mul(S2, Q + w, z1c, m);
  if (memcmp(U1, U2, 8 * w) == 0) {
    if (memcmp(S1, S2, 8 * w) != 0) { pt_inf(R, w); return; }
    uint64_t tmp[3 * MAXW];
    memcpy(tmp, P, 3 * 8 * w);
    pt_double(R, tmp, f);
    return;
  }
  f->sub(H, U2, U1, m);
  f->sub(Rr, S2, S1, m);
  f->mul(H2, H, H, m);
  f->mul(H3, H, H2, m);
  f->mul(X3, Rr, Rr, m);
  f->sub(X3, X3, H3, m);
  f->mul(U1, U1, H2, m);
  f->sub(X3, X3, U1, m);
  f->sub(X3, X3, U1, m);
  f->mul(S1, S1, H3, m);
  f->sub(t, U1, X3, m);
  f->mul(Y3, Rr, t, m);
  f->sub(Y3, Y3, S1, m);
  f->mul(Z3, P + 2 * w, Q + 2 * w, m);
  f->mul(Z3, Z3, H, m);
  memcpy(R, X3, 8 * w); memcpy(R + w, Y3, 8 * w); memcpy(R + 2 * w, Z3, 8 * w);
}

/* affine (X, Y) with the reference's infinity encoding (0, 1_mont) -> Jacobian */
static int aff_isinf(const uint64_t *A, int w) {
  uint64_t one[MAXW];
  e_one(one, w);
  return e_iszero(A, w) && memcmp(A + w, one, 8 * w) == 0;
}
static void aff_to_jac(uint64_t *P, const uint64_t *A, int w) {
  if (aff_isinf(A, w)) { pt_inf(P, w); return; }
  memcpy(P, A, 2 * 8 * w);
  e_one(P + 2 * w, w);
}
/* ec_jac2aff_h (src/cuda/ec.cpp:963): (X/Z^2, Y/Z^3); Z = 0 -> (0, 1_mont). */
static void jac_to_aff(uint64_t *A, const uint64_t *P, const fops_t *f) {
  const modctx_t *m = &MODS[0];
  int w = f->w;
  if (pt_isinf(P, w)) {
    memset(A, 0, 2 * 8 * w);
    e_one(A + w, w);
    return;
  }
  uint64_t zi[MAXW], zi2[MAXW], zi3[MAXW];
  if (w == 4) finv(zi, P + 2 * w, m); else f2inv(zi, P + 2 * w, m);
  f->mul(zi2, zi, zi, m);
  f->mul(zi3, zi2, zi, m);
  f->mul(A, P, zi2, m);
  f->mul(A + w, P + w, zi3, m);
}

void or_ec_jacadd(uint32_t *z, const uint32_t *x, const uint32_t *y, uint32_t ec2) {
  init_mods();
  const fops_t *f = &FOPS[ec2 ? 1 : 0];
  uint64_t P[3 * MAXW], Q[3 * MAXW], R[3 * MAXW];
  memcpy(P, x, 3 * 8 * f->w); memcpy(Q, y, 3 * 8 * f->w);
  pt_add(R, P, Q, f);
  memcpy(z, R, 3 * 8 * f->w);
}
void or_ec_jacdouble(uint32_t *z, const uint32_t *x, uint32_t ec2) {
  init_mods();
  const fops_t *f = &FOPS[ec2 ? 1 : 0];
  uint64_t P[3 * MAXW], R[3 * MAXW];
  memcpy(P, x, 3 * 8 * f->w);
  pt_double(R, P, f);
  memcpy(z, R, 3 * 8 * f->w);
}
/* ec_jacaddmixed_h (src/cuda/ec.cpp:216): affine x plus Jacobian y. */
void or_ec_jacaddmixed(uint32_t *z, const uint32_t *x_aff, const uint32_t *y_jac, uint32_t ec2) {
  init_mods();
  const fops_t *f = &FOPS[ec2 ? 1 : 0];
  uint64_t A[2 * MAXW], P[3 * MAXW], Q[3 * MAXW], R[3 * MAXW];
  memcpy(A, x_aff, 2 * 8 * f->w);
  memcpy(Q, y_jac, 3 * 8 * f->w);
  aff_to_jac(P, A, f->w);
  pt_add(R, P, Q, f);
  memcpy(z, R, 3 * 8 * f->w);
}
void or_ec_jac2aff(uint32_t *y, const uint32_t *x, uint32_t n, uint32_t ec2) {
  init_mods();
  const fops_t *f = &FOPS[ec2 ? 1 : 0];
  for (uint32_t i = 0; i < n; i++) {
    uint64_t P[3 * MAXW], A[2 * MAXW];
    memcpy(P, x + (size_t)i * 6 * f->w, 3 * 8 * f->w);
    jac_to_aff(A, P, f);
    memcpy(y + (size_t)i * 4 * f->w, A, 2 * 8 * f->w);
  }
}
/* ec_isoncurve_h: y^2 == x^3 + b, b = 3 (G1) or 3/(9+u) (G2), Montgomery domain. */
uint32_t or_ec_isoncurve_aff(const uint32_t *x_aff, uint32_t ec2) {
  init_mods();
  const fops_t *f = &FOPS[ec2 ? 1 : 0];
  const modctx_t *m = &MODS[0];
  int w = f->w;
  uint64_t A[2 * MAXW], lhs[MAXW], rhs[MAXW], b[MAXW];
  memcpy(A, x_aff, 2 * 8 * w);
  if (aff_isinf(A, w)) return 1;
  f->mul(lhs, A + w, A + w, m);
  f->mul(rhs, A, A, m);
  f->mul(rhs, rhs, A, m);
  memset(b, 0, sizeof(b));
  uint64_t three[4] = {3, 0, 0, 0};
  fmul(b, three, m->r2, m);
  if (w == 8) {  /* b' = 3 / (9 + u) */
    uint64_t nine[4] = {9, 0, 0, 0}, d[8], di[8];
    fmul(d, nine, m->r2, m);
    memcpy(d + 4, m->one, 32);
    f2inv(di, d, m);
    uint64_t b3[8] = {0};
    memcpy(b3, b, 32);
    f2mul(b, b3, di, m);
  }
  f->add(rhs, rhs, b, m);
  return memcmp(lhs, rhs, 8 * w) == 0;
}

/* ec_jacscmul_h (src/cuda/ec.cpp:833): per-point scalar multiplication, here
 * left-to-right double-and-add with affine output. */
void or_ec_scmul(uint32_t *z_aff, const uint32_t *scl, const uint32_t *x_aff, uint32_t n, uint32_t ec2) {
  init_mods();
  const fops_t *f = &FOPS[ec2 ? 1 : 0];
  int w = f->w;
#pragma omp parallel for schedule(dynamic, 16)
  for (long i = 0; i < (long)n; i++) {
    uint64_t A[2 * MAXW], B[3 * MAXW], acc[3 * MAXW], out[2 * MAXW];
    memcpy(A, x_aff + (size_t)i * 4 * w, 2 * 8 * w);
    aff_to_jac(B, A, w);
    pt_inf(acc, w);
    const uint32_t *k = scl + (size_t)i * 8;
    for (int b = 255; b >= 0; b--) {
      pt_double(acc, acc, f);
      if ((k[b >> 5] >> (b & 31)) & 1) pt_add(acc, acc, B, f);
    }
    jac_to_aff(out, acc, f);
    memcpy(z_aff + (size_t)i * 4 * w, out, 2 * 8 * w);
  }
}

/* ---------------------------------------------------------------- multi-exp ------ */
/* ec_jacreduce_server_h -> ec_jacreduce_batch_h -> ec_jacscmul_opt_h ->
 * ec_inittable_h -> ec_jacdouble_finish_h -> ec_jacaddreduce_finish_h
 * (src/cuda/ec.cpp:1536, :1706, :699, :574, :2004, :1175).
 * Points are cut into groups of `order`; each group gets a 2^order subset-sum table
 * (entry b = sum of the group's points whose bit is set in b).  For every bit position
 * j (255..0) the group's j-th scalar bits select one table entry, which is added into the
 * accumulator EP[j].  Finally P = sum_j 2^j EP[j] by double-and-add, per thread, and the
 * thread partials are summed and converted to affine. */
void or_msm(uint32_t *out_aff, const uint32_t *scl, const uint32_t *x_aff, uint32_t n,
            uint32_t ec2, uint32_t order, uint32_t nthreads) {
  init_mods();
  const fops_t *f = &FOPS[ec2 ? 1 : 0];
  const int w = f->w;
  const size_t PJ = 3 * (size_t)w;  /* uint64 words per Jacobian point */
  if (order < 1) order = 1;
  if (order > 12) order = 12;
  int nt = (int)nthreads;
#ifdef _OPENMP
  if (nt <= 0) nt = omp_get_max_threads();
#else
  nt = 1;
#endif
  uint32_t ngroups = (n + order - 1) / order;
  if ((uint32_t)nt > ngroups && ngroups > 0) nt = (int)ngroups;
  if (nt < 1) nt = 1;
  uint64_t *EPall = (uint64_t *)malloc(sizeof(uint64_t) * PJ * 256 * nt);
  uint64_t *partial = (uint64_t *)malloc(sizeof(uint64_t) * PJ * nt);
#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    uint64_t *EP = EPall + (size_t)tid * PJ * 256;
    uint64_t *table = (uint64_t *)malloc(sizeof(uint64_t) * PJ * ((size_t)1 << order));
    for (int j = 0; j < 256; j++) pt_inf(EP + j * PJ, w);
#pragma omp for schedule(static)
    for (long g = 0; g < (long)ngroups; g++) {
      uint32_t base = (uint32_t)g * order;
      uint32_t cnt = (n - base < order) ? (n - base) : order;
      uint32_t tsize = 1u << order, lastpow2 = 1;
      pt_inf(table, w);
      for (uint32_t j = 1; j < tsize; j++) {
        if ((j & (j - 1)) == 0) {
          uint32_t k = __builtin_ctz(j);
          lastpow2 = j;
          if (k < cnt) {
            uint64_t A[2 * MAXW];
            memcpy(A, x_aff + (size_t)(base + k) * 4 * w, 2 * 8 * w);
            aff_to_jac(table + j * PJ, A, w);
          } else {
            pt_inf(table + j * PJ, w);
          }
        } else {
          pt_add(table + j * PJ, table + lastpow2 * PJ, table + (j - lastpow2) * PJ, f);
        }
      }
      for (int bit = 255; bit >= 0; bit--) {
        uint32_t b = 0;
        for (uint32_t k = 0; k < cnt; k++)
          b |= ((scl[(size_t)(base + k) * 8 + (bit >> 5)] >> (bit & 31)) & 1u) << k;
        if (b) pt_add(EP + bit * PJ, table + b * PJ, EP + bit * PJ, f);
      }
    }
    uint64_t *P = partial + (size_t)tid * PJ;
    memcpy(P, EP + 255 * PJ, 8 * PJ);
    for (int j = 254; j >= 0; j--) {
      pt_double(P, P, f);
      pt_add(P, P, EP + j * PJ, f);
    }
    free(table);
  }
  uint64_t acc[3 * MAXW], A[2 * MAXW];
  pt_inf(acc, w);
  for (int t = 0; t < nt; t++) pt_add(acc, acc, partial + (size_t)t * PJ, f);
  jac_to_aff(A, acc, f);
  memcpy(out_aff, A, 2 * 8 * w);
  free(EPall);
  free(partial);
}

/* --------------------------------------------------------------------- NTT ------- */
static uint32_t bitrev(uint32_t x, uint32_t levels) {
  uint32_t r = 0;
  for (uint32_t i = 0; i < levels; i++) { r = (r << 1) | (x & 1); x >>= 1; }
  return r;
}
/* ntt_reorder_h (src/cuda/ntt.cpp:490) */
static void reorder(uint64_t *A, uint32_t levels, uint64_t astride) {
  uint32_t n = 1u << levels;
  for (uint32_t i = 0; i < n; i++) {
    uint32_t j = bitrev(i, levels);
    if (j > i) {
      uint64_t t[4];
      memcpy(t, A + astride * i * 4, 32);
      memcpy(A + astride * i * 4, A + astride * j * 4, 32);
      memcpy(A + astride * j * 4, t, 32);
    }
  }
}
/* _ntt_h (src/cuda/ntt.cpp:392): iterative radix-2 DIT on bit-reversed data;
 * the twiddle for butterfly k of a size-s stage is roots[(rstride*k*dir*n/s) mod rstride*n]. */
static void ntt_core(uint64_t *A, const uint64_t *roots, uint32_t levels, uint64_t astride,
                     uint64_t rstride, int32_t direction, const modctx_t *m) {
  int64_t n = (int64_t)1 << levels;
  uint64_t mask = rstride * (uint64_t)n - 1;
  for (int64_t size = 2; size <= n; size *= 2) {
    int64_t half = size >> 1;
    int64_t step = (int64_t)direction * (n / size);
    for (int64_t i = 0; i < n; i += size) {
      int64_t k = 0;
      for (int64_t j = i; j < i + half; j++) {
        uint64_t ridx = ((uint64_t)k * rstride) & mask;
        uint64_t *lo = A + (uint64_t)j * astride * 4, *hi = A + (uint64_t)(j + half) * astride * 4;
        uint64_t right[4];
        fmul(right, hi, roots + ridx * 4, m);
        fsub(hi, lo, right, m);
        fadd(lo, lo, right, m);
        k += step;
      }
    }
  }
}
/* ntt_h (src/cuda/ntt.cpp:453) */
void or_ntt(uint32_t *A, const uint32_t *roots, uint32_t levels, uint64_t astride,
            uint64_t rstride, int32_t direction, uint32_t pidx) {
  init_mods();
  reorder((uint64_t *)A, levels, astride);
  ntt_core((uint64_t *)A, (const uint64_t *)roots, levels, astride, rstride, direction, &MODS[pidx]);
}
/* scalers 1/2^levels of r in normal (fmat 0) or Montgomery (fmat 1) form, as
 * CusnarksIScalerGet (src/cuda/constants.cpp:399) returns them. */
static void iscaler(uint64_t *s, uint32_t fmat, uint32_t levels) {
  const modctx_t *m = &MODS[1];
  uint64_t nn[4] = {0, 0, 0, 0}, nm[4];
  nn[levels >> 6] = 1ull << (levels & 63);
  fmul(nm, nn, m->r2, m);   /* n in Montgomery */
  finv(nm, nm, m);          /* n^-1 in Montgomery */
  if (fmat) { memcpy(s, nm, 32); return; }
  uint64_t one[4] = {1, 0, 0, 0};
  fmul(s, nm, one, m);
}
/* intt_h (src/cuda/ntt.cpp:583): reorder, DIT with direction -1, scale by 1/n. */
void or_intt(uint32_t *A, const uint32_t *roots, uint32_t fmat, uint32_t levels,
             uint64_t rstride, uint32_t pidx) {
  init_mods();
  uint64_t *a = (uint64_t *)A;
  reorder(a, levels, 1);
  ntt_core(a, (const uint64_t *)roots, levels, 1, rstride, -1, &MODS[pidx]);
  uint64_t s[4];
  iscaler(s, fmat, levels);
  for (uint64_t i = 0; i < (1ull << levels); i++) fmul(a + 4 * i, a + 4 * i, s, &MODS[pidx]);
}
/* primitive 2^levels-th root of unity of Fr, Montgomery form: 5^((r-1)/2^levels), the
 * same chain as proots_field (src/cuda/constants.cpp:323). */
void or_primitive_root(uint32_t *root_mont, uint32_t levels) {
  init_mods();
  const modctx_t *m = &MODS[1];
  uint64_t e[4], one[4] = {1, 0, 0, 0}, g[4], five[4] = {5, 0, 0, 0};
  sub4(e, m->p, one);
  for (uint32_t i = 0; i < levels; i++) {  /* e >>= 1 */
    for (int k = 0; k < 4; k++) e[k] = (e[k] >> 1) | (k < 3 ? (e[k + 1] << 63) : 0);
  }
  fmul(g, five, m->r2, m);
  uint64_t w[4];
  fpow(w, g, e, m);
  memcpy(root_mont, w, 32);
}
/* find_roots_h (src/cuda/ntt.cpp:1164): roots[i] = proot^i, i < n, Montgomery. */
void or_root_powers(uint32_t *roots, const uint32_t *proot, uint64_t n) {
  init_mods();
  const modctx_t *m = &MODS[1];
  uint64_t w[4], acc[4];
  memcpy(w, proot, 32);
  memcpy(acc, m->one, 32);
  for (uint64_t i = 0; i < n; i++) {
    memcpy(roots + 8 * i, acc, 32);
    fmul(acc, acc, w, m);
  }
}
/* computeRoots_h (src/cuda/ntt.cpp:1181): the roots file, powers of proots_field[levels]. */
void or_find_roots(uint32_t *roots, uint32_t levels) {
  uint32_t w[8];
  or_primitive_root(w, levels);
  or_root_powers(roots, w, 1ull << levels);
}

/* ntt_interpolandmul_server_h -> interpol_and_mul_h (src/cuda/ntt.cpp:672, :778),
 * restated without the 4-step decomposition (which only reorganises the same
 * transforms):
 *   1. Me[i] = A[i]*B[i]                       even evaluations of A*B on the 2m-th roots
 *   2. a = INTT_m(A), b = INTT_m(B)            Montgomery, twiddles roots[rstride*k]
 *   3. a[i] *= roots[i], b[i] *= roots[i]      shift to the odd 2m-th roots
 *   4. A' = NTT_m(a), B' = NTT_m(b);  Mo[i] = A'[i]*B'[i]
 *   5. M = INTT_2m(interleave(Me, Mo)) with twiddles roots[(rstride/2)*k], scaled to
 *      normal form (scaler_ext).
 * `roots` is the first (2m-entry) part of the caller's table, levels = log2(m). */
void or_interpolandmul(uint32_t *M, const uint32_t *A, const uint32_t *B,
                       const uint32_t *roots, uint32_t levels, uint64_t rstride) {
  init_mods();
  const modctx_t *m = &MODS[1];
  uint64_t n = 1ull << levels;
  uint64_t *a = (uint64_t *)malloc(32 * n), *b = (uint64_t *)malloc(32 * n);
  uint64_t *Mw = (uint64_t *)M;
  const uint64_t *rt = (const uint64_t *)roots;
  memcpy(a, A, 32 * n); memcpy(b, B, 32 * n);
  for (uint64_t i = 0; i < n; i++) fmul(Mw + 8 * i, a + 4 * i, b + 4 * i, m);
  or_intt((uint32_t *)a, roots, 1, levels, rstride, 1);
  or_intt((uint32_t *)b, roots, 1, levels, rstride, 1);
  for (uint64_t i = 0; i < n; i++) {
    fmul(a + 4 * i, a + 4 * i, rt + 4 * i, m);
    fmul(b + 4 * i, b + 4 * i, rt + 4 * i, m);
  }
  or_ntt((uint32_t *)a, roots, levels, 1, rstride, 1, 1);
  or_ntt((uint32_t *)b, roots, levels, 1, rstride, 1, 1);
  for (uint64_t i = 0; i < n; i++) fmul(Mw + 8 * i + 4, a + 4 * i, b + 4 * i, m);
  or_intt(M, roots, 0, levels + 1, rstride / 2, 1);
  free(a); free(b);
}

/* Coset H step (not in the reference; stated from the Groth16 quotient):
 *   a,b,c = INTT_m(A,B,C); scale coefficient i by g^i; evaluate with NTT_m on g*<w>;
 *   H'(i) = (A'B' - C') / (g^m - 1); h = INTT_m(H'); unscale coefficient i by g^-i;
 *   output normal form.  g = 5, w = primitive m-th root (same chain as or_find_roots). */
void or_hstep_coset(uint32_t *H, const uint32_t *A, const uint32_t *B, const uint32_t *C,
                    uint32_t levels) {
  init_mods();
  const modctx_t *m = &MODS[1];
  uint64_t n = 1ull << levels;
  uint64_t *roots = (uint64_t *)malloc(32 * n);
  or_find_roots((uint32_t *)roots, levels);
  uint64_t *v[3];
  const uint32_t *src[3] = {A, B, C};
  uint64_t five[4] = {5, 0, 0, 0}, g[4], gi[4], gp[4];
  fmul(g, five, m->r2, m);
  finv(gi, g, m);
  for (int k = 0; k < 3; k++) {
    v[k] = (uint64_t *)malloc(32 * n);
    memcpy(v[k], src[k], 32 * n);
    or_intt((uint32_t *)v[k], (uint32_t *)roots, 1, levels, 1, 1);
    memcpy(gp, m->one, 32);
    for (uint64_t i = 0; i < n; i++) { fmul(v[k] + 4 * i, v[k] + 4 * i, gp, m); fmul(gp, gp, g, m); }
    or_ntt((uint32_t *)v[k], (uint32_t *)roots, levels, 1, 1, 1, 1);
  }
  /* (g^m - 1)^-1 */
  uint64_t gm[4], zinv[4];
  memcpy(gm, m->one, 32);
  for (uint64_t i = 0; i < n; i++) fmul(gm, gm, g, m);
  fsub(gm, gm, m->one, m);
  finv(zinv, gm, m);
  for (uint64_t i = 0; i < n; i++) {
    uint64_t t[4];
    fmul(t, v[0] + 4 * i, v[1] + 4 * i, m);
    fsub(t, t, v[2] + 4 * i, m);
    fmul(v[0] + 4 * i, t, zinv, m);
  }
  or_intt((uint32_t *)v[0], (uint32_t *)roots, 1, levels, 1, 1);
  memcpy(gp, m->one, 32);
  uint64_t one[4] = {1, 0, 0, 0};
  for (uint64_t i = 0; i < n; i++) {
    uint64_t t[4];
    fmul(t, v[0] + 4 * i, gp, m);
    fmul(t, t, one, m);  /* leave Montgomery form */
    memcpy(H + 8 * i, t, 32);
    fmul(gp, gp, gi, m);
  }
  for (int k = 0; k < 3; k++) free(v[k]);
  free(roots);
}

/* ------------------------------------------------------------------ QAP ---------- */
/* mpoly_eval_h (src/cuda/mpoly.cpp:125).  pin layout (r1cs_to_mpoly_h, mpoly.cpp:195):
 *   pin[0] = number of polynomials (variables) N
 *   pin[1 .. N] = number of coefficients of each polynomial
 *   then per polynomial i: ncoeff_i constraint indices, followed by ncoeff_i
 *   8-word Montgomery values.
 * pout[c] += toMont(scalar[i]) * value, for every (c, value) of polynomial i. */
void or_mpoly_eval(uint32_t *pout, const uint32_t *scalar, const uint32_t *pin,
                   uint32_t start_idx, uint32_t last_idx, uint32_t pidx) {
  init_mods();
  const modctx_t *m = &MODS[pidx];
  uint64_t npoly = pin[0];
  uint64_t acc = 0;
  for (uint64_t i = 0; i < start_idx; i++) acc += pin[i + 1];
  uint64_t doff = acc * 9 + 1 + npoly;
  for (uint64_t i = start_idx; i < last_idx; i++) {
    uint64_t s[4], sm[4];
    memcpy(s, scalar + 8 * i, 32);
    fmul(sm, s, m->r2, m);
    uint64_t nc = pin[1 + i];
    uint64_t voff = doff + nc;
    for (uint64_t j = 0; j < nc; j++) {
      uint64_t c = pin[doff + j];
      uint64_t v[4], prod[4], o[4];
      memcpy(v, pin + voff + 8 * j, 32);
      fmul(prod, v, sm, m);
      memcpy(o, pout + 8 * c, 32);
      fadd(o, o, prod, m);
      memcpy(pout + 8 * c, o, 32);
    }
    acc += nc;
    doff = acc * 9 + 1 + npoly;
  }
}

/* ----------------------------------------------------- batched products ----------- */
/* z[i] = a[i] * b[i] * 2^-256 mod p for n pairs (OpenMP).  Operands may be any 256-bit
 * values: they are reduced mod p first, so lazily reduced inputs in [p, 2^256) give the
 * product of their residues (montmult_h, src/cuda/ff.cpp:225, on reduced operands). */
static void reduce4(uint64_t *x, const modctx_t *m) {
  while (geq4(x, m->p)) sub4(x, x, m->p);
}
void or_montmult_batch(uint32_t *z, const uint32_t *a, const uint32_t *b, uint64_t n, uint32_t pidx) {
  init_mods();
  const modctx_t *m = &MODS[pidx];
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; i++) {
    uint64_t x[4], y[4], t[4];
    memcpy(x, a + 8 * (size_t)i, 32);
    memcpy(y, b + 8 * (size_t)i, 32);
    reduce4(x, m);
    reduce4(y, m);
    fmul(t, x, y, m);
    memcpy(z + 8 * (size_t)i, t, 32);
  }
}

/* ------------------------------------ benchmark circuit and proving key on the CPU --- */
/* The benchmark's synthetic circuit and its proving key, built without a GPU (for a
 * process that must not load the CUDA library).  The quantities are those of Groth16
 * setup as the reference computes them (src/python/groth_setup.py: calculateValuesAtT
 * :771, calculateEncryptedValuesAtT :488): Lagrange basis at t, wire polynomials at t,
 * the C scalars (beta u + alpha v + w)/delta, t^j Z(t)/delta, and fixed-base scalar
 * multiplications of the generators. */

/* Witness of the synthetic circuit, constraints in order: w[first_out + c] =
 * (sum_k a_coeff * w[a_wire]) * (sum_k b_coeff * w[b_wire]), `per_row` terms each side,
 * coefficients Montgomery, witness normal form.  A constraint reads only wires defined
 * before its layer, so one pass in order computes every output. */
void or_r1cs_eval(uint32_t *w, uint64_t first_out, uint64_t nc, uint32_t per_row,
                  const uint32_t *a_wire, const uint32_t *a_coeff,
                  const uint32_t *b_wire, const uint32_t *b_coeff) {
  init_mods();
  const modctx_t *m = &MODS[1];
  for (uint64_t c = 0; c < nc; c++) {
    uint64_t sa[4] = {0, 0, 0, 0}, sb[4] = {0, 0, 0, 0}, t[4], v[4], x[4];
    for (uint32_t k = 0; k < per_row; k++) {
      const uint64_t e = c * per_row + k;
      memcpy(v, a_coeff + 8 * e, 32);
      memcpy(x, w + 8 * (size_t)a_wire[e], 32);
      fmul(t, v, x, m);           /* Montgomery coefficient times normal value = normal */
      fadd(sa, sa, t, m);
      memcpy(v, b_coeff + 8 * e, 32);
      memcpy(x, w + 8 * (size_t)b_wire[e], 32);
      fmul(t, v, x, m);
      fadd(sb, sb, t, m);
    }
    fmul(t, sa, sb, m);           /* sa sb / R */
    fmul(t, t, m->r2, m);         /* sa sb */
    memcpy(w + 8 * (first_out + c), t, 32);
  }
}

/* out[i] = 1 / in[i] for n nonzero Montgomery elements of Fr (one inversion). */
static void batch_inv_fr(uint64_t *out, const uint64_t *in, uint64_t n) {
  const modctx_t *m = &MODS[1];
  if (n == 0) return;
  uint64_t *pre = (uint64_t *)malloc(32 * n), acc[4], inv[4], t[4];
  memcpy(acc, m->one, 32);
  for (uint64_t i = 0; i < n; i++) {
    fmul(acc, acc, in + 4 * i, m);
    memcpy(pre + 4 * i, acc, 32);
  }
  finv(inv, acc, m);
  for (uint64_t i = n; i-- > 0;) {
    if (i) fmul(t, inv, pre + 4 * (i - 1), m); else memcpy(t, inv, 32);
    fmul(inv, inv, in + 4 * i, m);
    memcpy(out + 4 * i, t, 32);
  }
  free(pre);
}

/* Lagrange basis of the domain <w> (m = 2^levels, w the reference's primitive root) at
 * t: L_c(t) = w^c (t^m - 1) / (m (t - w^c)), Montgomery in and out. */
void or_lagrange_at(uint32_t *out, uint32_t levels, const uint32_t *t_mont) {
  init_mods();
  const modctx_t *m = &MODS[1];
  const uint64_t n = 1ull << levels;
  uint64_t t[4], tm[4], zm[4], nn[4] = {0, 0, 0, 0}, ninv[4];
  memcpy(t, t_mont, 32);
  memcpy(tm, t, 32);
  for (uint32_t k = 0; k < levels; k++) fmul(tm, tm, tm, m);
  fsub(zm, tm, m->one, m);
  nn[levels >> 6] = 1ull << (levels & 63);
  fmul(ninv, nn, m->r2, m);
  finv(ninv, ninv, m);
  fmul(zm, zm, ninv, m);           /* (t^m - 1) / m */
  uint64_t *wp = (uint64_t *)malloc(32 * n), *den = (uint64_t *)malloc(32 * n);
  or_find_roots((uint32_t *)wp, levels);
  for (uint64_t c = 0; c < n; c++) fsub(den + 4 * c, t, wp + 4 * c, m);
  batch_inv_fr(den, den, n);
  for (uint64_t c = 0; c < n; c++) {
    uint64_t v[4];
    fmul(v, zm, wp + 4 * c, m);
    fmul(v, v, den + 4 * c, m);
    memcpy(out + 8 * c, v, 32);
  }
  free(wp);
  free(den);
}

/* Wire polynomials at t: out[i] = sum over wire i's (c, coeff) of coeff * L[c] for
 * c < n_rows, reference mpoly layout (src/cuda/mpoly.cpp:195), Montgomery. */
void or_wire_eval(uint32_t *out, const uint32_t *mpoly, const uint32_t *Lc, uint32_t n_rows) {
  init_mods();
  const modctx_t *m = &MODS[1];
  const uint64_t nw = mpoly[0];
  uint64_t *start = (uint64_t *)malloc(8 * (nw + 1));
  start[0] = 0;
  for (uint64_t i = 0; i < nw; i++) start[i + 1] = start[i] + mpoly[1 + i];
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)nw; i++) {
    const uint64_t nc = mpoly[1 + i];
    const uint64_t blk = 1 + nw + 9 * start[i];
    uint64_t acc[4] = {0, 0, 0, 0}, v[4], l[4], t[4];
    for (uint64_t k = 0; k < nc; k++) {
      const uint32_t c = mpoly[blk + k];
      if (c >= n_rows) continue;
      memcpy(v, mpoly + blk + nc + 8 * k, 32);
      memcpy(l, Lc + 8 * (size_t)c, 32);
      fmul(t, v, l, m);
      fadd(acc, acc, t, m);
    }
    memcpy(out + 8 * (size_t)i, acc, 32);
  }
  free(start);
}

/* out[i] (normal form) = (beta u_i + alpha v_i + w_i) k, inputs Montgomery. */
void or_c_scalars(uint32_t *out, const uint32_t *u, const uint32_t *v, const uint32_t *w,
                  const uint32_t *alpha, const uint32_t *beta, const uint32_t *k, uint64_t n) {
  init_mods();
  const modctx_t *m = &MODS[1];
  uint64_t al[4], be[4], kk[4], one[4] = {1, 0, 0, 0};
  memcpy(al, alpha, 32); memcpy(be, beta, 32); memcpy(kk, k, 32);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; i++) {
    uint64_t x[4], y[4], t[4];
    memcpy(t, u + 8 * (size_t)i, 32);
    fmul(x, be, t, m);
    memcpy(t, v + 8 * (size_t)i, 32);
    fmul(y, al, t, m);
    fadd(x, x, y, m);
    memcpy(t, w + 8 * (size_t)i, 32);
    fadd(x, x, t, m);
    fmul(x, x, kk, m);
    fmul(x, x, one, m);
    memcpy(out + 8 * (size_t)i, x, 32);
  }
}

/* out[j] (normal form) = t^j k for j < n, t and k Montgomery. */
void or_pow_scalars(uint32_t *out, const uint32_t *t_mont, const uint32_t *k, uint64_t n) {
  init_mods();
  const modctx_t *m = &MODS[1];
  uint64_t t[4], acc[4], one[4] = {1, 0, 0, 0}, x[4];
  memcpy(t, t_mont, 32);
  memcpy(acc, k, 32);
  for (uint64_t j = 0; j < n; j++) {
    fmul(x, acc, one, m);
    memcpy(out + 8 * j, x, 32);
    fmul(acc, acc, t, m);
  }
}

/* Jacobian P plus affine A (not infinity), the formulas of ec_jacaddmixed_h
 * (src/cuda/ec.cpp:216) with Z2 = 1; equal points double, opposite ones give infinity. */
static void pt_madd(uint64_t *R, const uint64_t *P, const uint64_t *A, const fops_t *f) {
  const modctx_t *m = &MODS[0];
  const int w = f->w;
  if (pt_isinf(P, w)) {
    memcpy(R, A, 2 * 8 * w);
    e_one(R + 2 * w, w);
    return;
  }
  uint64_t z1s[MAXW], z1c[MAXW], U2[MAXW], S2[MAXW], H[MAXW], Rr[MAXW], HH[MAXW], HHH[MAXW];
  uint64_t V[MAXW], X3[MAXW], Y3[MAXW], Z3[MAXW], t[MAXW];
  f->mul(z1s, P + 2 * w, P + 2 * w, m);
  f->mul(z1c, z1s, P + 2 * w, m);
  f->mul(U2, A, z1s, m);
  f->mul(S2, A + w, z1c, m);
  if (memcmp(U2, P, 8 * w) == 0) {
    if (memcmp(S2, P + w, 8 * w) != 0) { pt_inf(R, w); return; }
    uint64_t tmp[3 * MAXW];
    memcpy(tmp, P, 3 * 8 * w);
    pt_double(R, tmp, f);
    return;
  }
  f->sub(H, U2, P, m);
  f->sub(Rr, S2, P + w, m);
  f->mul(HH, H, H, m);
  f->mul(HHH, H, HH, m);
  f->mul(V, P, HH, m);
  f->mul(X3, Rr, Rr, m);
  f->sub(X3, X3, HHH, m);
  f->sub(X3, X3, V, m);
  f->sub(X3, X3, V, m);
  f->sub(t, V, X3, m);
  f->mul(Y3, Rr, t, m);
  f->mul(t, P + w, HHH, m);
  f->sub(Y3, Y3, t, m);
  f->mul(Z3, P + 2 * w, H, m);
  memcpy(R, X3, 8 * w); memcpy(R + w, Y3, 8 * w); memcpy(R + 2 * w, Z3, 8 * w);
}

/* Jacobian -> affine for n points with one inversion (Montgomery's simultaneous
 * inversion over the nonzero Z); infinity -> (0, 1_mont). */
static void jac_to_aff_batch(uint64_t *A, const uint64_t *P, uint64_t n, const fops_t *f) {
  const modctx_t *m = &MODS[0];
  const int w = f->w;
  const size_t PJ = 3 * (size_t)w, PA = 2 * (size_t)w;
  uint64_t *pre = (uint64_t *)malloc(8 * (size_t)w * (n + 1));
  uint64_t acc[MAXW], inv[MAXW], zi[MAXW], zi2[MAXW], zi3[MAXW];
  e_one(acc, w);
  for (uint64_t i = 0; i < n; i++) {
    if (!pt_isinf(P + i * PJ, w)) f->mul(acc, acc, P + i * PJ + 2 * w, m);
    memcpy(pre + (size_t)w * i, acc, 8 * w);
  }
  if (w == 4) finv(inv, acc, m); else f2inv(inv, acc, m);
  for (uint64_t i = n; i-- > 0;) {
    const uint64_t *Q = P + i * PJ;
    if (pt_isinf(Q, w)) {
      memset(A + i * PA, 0, 8 * PA);
      e_one(A + i * PA + w, w);
      continue;
    }
    if (i) f->mul(zi, inv, pre + (size_t)w * (i - 1), m); else memcpy(zi, inv, 8 * w);
    f->mul(inv, inv, Q + 2 * w, m);
    f->mul(zi2, zi, zi, m);
    f->mul(zi3, zi2, zi, m);
    f->mul(A + i * PA, Q, zi2, m);
    f->mul(A + i * PA + w, Q + w, zi3, m);
  }
  free(pre);
}

/* out[i] = scl[i] * G for one base G (affine Montgomery, not infinity); scalars normal
 * form below 2^256; affine Montgomery out.  Comb over 8-bit windows: table
 * T[j][d] = d 2^(8j) G, then 32 mixed additions per scalar, affine conversion with one
 * inversion per run of 256 points (the fixed-base multiplication of the reference's
 * sc1mulecjac kernel, src/cuda/ecbn128_device.cu:326, in another schedule). */
void or_fixed_base_mul(uint32_t *out_aff, const uint32_t *scl, uint64_t n, const uint32_t *base_aff,
                       uint32_t ec2) {
  init_mods();
  const fops_t *f = &FOPS[ec2 ? 1 : 0];
  const int w = f->w;
  const size_t PJ = 3 * (size_t)w, PA = 2 * (size_t)w;
  uint64_t *tab = (uint64_t *)malloc(8 * PA * 32 * 256);
  {
    uint64_t B[3 * MAXW], A[2 * MAXW];
    memcpy(A, base_aff, 8 * PA);
    aff_to_jac(B, A, w);
    uint64_t *jt = (uint64_t *)malloc(8 * PJ * 32 * 256);
    for (int j = 0; j < 32; j++) {
      uint64_t *row = jt + (size_t)j * 256 * PJ;
      pt_inf(row, w);
      for (int d = 1; d < 256; d++) pt_add(row + d * PJ, row + (d - 1) * PJ, B, f);
      for (int k = 0; k < 8; k++) pt_double(B, B, f);
    }
    jac_to_aff_batch(tab, jt, 32 * 256, f);
    free(jt);
  }
  const uint64_t RUN = 256;
  const uint64_t nruns = (n + RUN - 1) / RUN;
#pragma omp parallel
  {
    uint64_t *jac = (uint64_t *)malloc(8 * PJ * RUN), *aff = (uint64_t *)malloc(8 * PA * RUN);
#pragma omp for schedule(dynamic, 4)
    for (long r = 0; r < (long)nruns; r++) {
      const uint64_t lo = (uint64_t)r * RUN, hi = lo + RUN < n ? lo + RUN : n;
      for (uint64_t i = lo; i < hi; i++) {
        uint64_t *acc = jac + (i - lo) * PJ;
        pt_inf(acc, w);
        const uint8_t *k = (const uint8_t *)(scl + 8 * i);
        for (int j = 0; j < 32; j++)
          if (k[j]) pt_madd(acc, acc, tab + ((size_t)j * 256 + k[j]) * PA, f);
      }
      jac_to_aff_batch(aff, jac, hi - lo, f);
      memcpy(out_aff + 4 * (size_t)w * lo, aff, 8 * PA * (hi - lo));
    }
    free(jac);
    free(aff);
  }
  free(tab);
}
