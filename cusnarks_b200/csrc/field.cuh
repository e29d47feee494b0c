// field.cuh -- 256-bit Montgomery arithmetic for BN254 on sm_100a.
//
// Elements are 8 little-endian 32-bit limbs held in registers, Montgomery form
// x * 2^256 mod p, always fully reduced to [0, p) at the boundary of every operation, so
// results are word-for-word the values the reference's host code produces
// (src/cuda/ff.cpp montmult_h / addm_h / subm_h, same layout as src/cuda/types.h
// NWORDS_256BIT).  Products are CIOS Montgomery multiplications on 32x32->64 wide
// products folded by add-with-carry chains; BN254 moduli are below 2^254, so the CIOS
// accumulator never needs a tenth limb and a single conditional subtraction finishes
// every product.  Units that call products out of line (the G1 MSM) compute the same
// Montgomery product in radix 2^52 on the FP64 pipe instead (namespace dp52).
#pragma once
#include <cstdint>

namespace csb {

#define CSB_DEV __device__ __forceinline__

// ---------------------------------------------------------------- moduli ------------
struct ModQ {  // base field q (the reference's MOD_GROUP, pidx 0)
  static constexpr uint32_t P0 = 0xd87cfd47u, P1 = 0x3c208c16u, P2 = 0x6871ca8du, P3 = 0x97816a91u,
                            P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
  static constexpr uint32_t NP0 = 0xe4866389u;  // -q^-1 mod 2^32
  static constexpr uint32_t ONE0 = 0xc58f0d9du, ONE1 = 0xd35d438du, ONE2 = 0xf5c70b3du, ONE3 = 0x0a78eb28u,
                            ONE4 = 0x7879462cu, ONE5 = 0x666ea36fu, ONE6 = 0x9a07df2fu, ONE7 = 0x0e0a77c1u;
  static constexpr uint32_t R20 = 0x538afa89u, R21 = 0xf32cfc5bu, R22 = 0xd44501fbu, R23 = 0xb5e71911u,
                            R24 = 0x0a417ff6u, R25 = 0x47ab1effu, R26 = 0xcab8351fu, R27 = 0x06d89f71u;
  static constexpr uint32_t R30 = 0xda1530dfu, R31 = 0xb1cd6dafu, R32 = 0xa7283db6u, R33 = 0x62f210e6u,
                            R34 = 0x0ada0afbu, R35 = 0xef7f0b0cu, R36 = 0x2d592544u, R37 = 0x20fd6e90u;
  // q in radix 2^52 and -q^-1 mod 2^52 (FP64-pipe product)
  static CSB_DEV double L52(int i) {
    return i == 0 ? 154029749239111.0 : i == 1 ? 2558044347618242.0 : i == 2 ? 423691504025962.0
         : i == 3 ? 2817616741948264.0 : 53207371014449.0;
  }
  static constexpr double NP52 = 571208714576777.0;
};
struct ModR {  // scalar field r (the reference's MOD_FIELD, pidx 1)
  static constexpr uint32_t P0 = 0xf0000001u, P1 = 0x43e1f593u, P2 = 0x79b97091u, P3 = 0x2833e848u,
                            P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
  static constexpr uint32_t NP0 = 0xefffffffu;  // -r^-1 mod 2^32
  static constexpr uint32_t ONE0 = 0x4ffffffbu, ONE1 = 0xac96341cu, ONE2 = 0x9f60cd29u, ONE3 = 0x36fc7695u,
                            ONE4 = 0x7879462eu, ONE5 = 0x666ea36fu, ONE6 = 0x9a07df2fu, ONE7 = 0x0e0a77c1u;
  static constexpr uint32_t R20 = 0xae216da7u, R21 = 0x1bb8e645u, R22 = 0xe35c59e3u, R23 = 0x53fe3ab1u,
                            R24 = 0x53bb8085u, R25 = 0x8c49833du, R26 = 0x7f4e44a5u, R27 = 0x0216d0b1u;
  static constexpr uint32_t R30 = 0xb4bf0040u, R31 = 0x5e94d8e1u, R32 = 0x1cfbb6b8u, R33 = 0x2a489cbeu,
                            R34 = 0xa19fcfedu, R35 = 0x893cc664u, R36 = 0x7fcc657cu, R37 = 0x0cf8594bu;
  static CSB_DEV double L52(int i) {
    return i == 0 ? 551490712240129.0 : i == 1 ? 1275002230477886.0 : i == 2 ? 423691496731624.0
         : i == 3 ? 2817616741948264.0 : 53207371014449.0;
  }
  static constexpr double NP52 = 551490712240127.0;
};

// ------------------------------------------------- products on the FP64 pipe ----------
// Montgomery product in radix 2^52 (Emmart, Zheng and Weems, "Faster modular
// exponentiation using double precision floating point arithmetic on the GPU", ARITH
// 2018): limbs are exact integers held in doubles; a 52x52-bit product x*y < 2^104 splits
// exactly into its high and low 52 bits with two round-toward-zero FMAs,
//   h = fma_rz(x, y, 2^104)            = 2^104 + H 2^52   (bits of h: exponent | H)
//   l = fma_rz(x, y, 2^104 + 2^52 - h) = 2^52 + L         (bits of l: exponent | L),
// and the raw bit patterns are summed per column in 64-bit integers, the exponent bits
// taken off in bulk by the column's starting value.  The multiplies run on the FP64 pipe
// and the column sums on the integer ALU, which a 32-bit CIOS leaves saturated by its
// add-with-carry chains (B200: 56 vs 46 G lazy products/s).
// The 8x32-bit operands are re-cut into five 52-bit limbs, one of them shifted left by 4:
// REDC in radix 2^52 divides by 2^260, so the result is a*b*2^-256 mod p, the same
// Montgomery product as the 32-bit CIOS.  For a, b < 2p it is below
// 16 a b / 2^260 + p < 2p (BN254: 64 p / 2^260 < 0.77), a lazily reduced value.
#ifndef CSB_DP52
#define CSB_DP52 1
#endif
namespace dp52 {
constexpr uint64_t kMask = 0x000FFFFFFFFFFFFFull;
constexpr uint64_t kBitsLo = 0x4330000000000000ull;  // bits of 2^52
constexpr uint64_t kBitsHi = 0x4670000000000000ull;  // bits of 2^104
// x*y into the column pair (lo: bits 0..51 of the product, hi: bits 52..103)
CSB_DEV void acc_prod(double x, double y, uint64_t& lo, uint64_t& hi) {
  const double h = __fma_rz(x, y, 0x1p104);
  const double l = __fma_rz(x, y, 0x1.0000000000001p104 - h);
  lo += (uint64_t)__double_as_longlong(l);
  hi += (uint64_t)__double_as_longlong(h);
}
// products landing in column k of a 5x5 schoolbook product
__host__ __device__ constexpr int terms(int k) { return (k < 0 || k > 8) ? 0 : (k < 4 ? k + 1 : 9 - k); }
// column k starts at minus the exponent bits of its terms: a*b and m*p each put terms(k)
// low halves and terms(k-1) high halves into it
__host__ __device__ constexpr uint64_t col_start(int k) {
  return (uint64_t)0 - (uint64_t)(2 * terms(k)) * kBitsLo - (uint64_t)(2 * terms(k - 1)) * kBitsHi;
}
// integer v < 2^52 as a double
CSB_DEV double to_dbl(uint64_t v) { return __longlong_as_double((long long)(v | kBitsLo)) - 0x1p52; }
CSB_DEV void words(const uint32_t (&x)[8], uint64_t (&w)[4]) {
#pragma unroll
  for (int i = 0; i < 4; i++) w[i] = x[2 * i] | (uint64_t)x[2 * i + 1] << 32;
}
// x = sum l_i 2^(52 i)
CSB_DEV void cut(const uint32_t (&x)[8], double (&l)[5]) {
  uint64_t w[4];
  words(x, w);
  l[0] = to_dbl(w[0] & kMask);
  l[1] = to_dbl(((w[0] >> 52) | (w[1] << 12)) & kMask);
  l[2] = to_dbl(((w[1] >> 40) | (w[2] << 24)) & kMask);
  l[3] = to_dbl(((w[2] >> 28) | (w[3] << 36)) & kMask);
  l[4] = to_dbl(w[3] >> 16);
}
// 16 x = sum l_i 2^(52 i)
CSB_DEV void cut16(const uint32_t (&x)[8], double (&l)[5]) {
  uint64_t w[4];
  words(x, w);
  l[0] = to_dbl((w[0] << 4) & kMask);
  l[1] = to_dbl(((w[0] >> 48) | (w[1] << 16)) & kMask);
  l[2] = to_dbl(((w[1] >> 36) | (w[2] << 28)) & kMask);
  l[3] = to_dbl(((w[2] >> 24) | (w[3] << 40)) & kMask);
  l[4] = to_dbl(w[3] >> 12);
}
// a*b*2^-256 mod p, lazily reduced (< 2p for a, b < 2p)
template <class M>
CSB_DEV void mont(const uint32_t (&x)[8], const uint32_t (&y)[8], uint32_t (&out)[8]) {
  double a[5], b[5];
  cut16(x, a);
  cut(y, b);
  uint64_t c[10];
#pragma unroll
  for (int k = 0; k < 10; k++) c[k] = col_start(k);
#pragma unroll
  for (int i = 0; i < 5; i++)
#pragma unroll
    for (int j = 0; j < 5; j++) acc_prod(a[i], b[j], c[i + j], c[i + j + 1]);
#pragma unroll
  for (int k = 0; k < 5; k++) {
    if (k > 0) c[k] += c[k - 1] >> 52;  // column k-1 is complete (and 0 mod 2^52)
    // m = (c_k mod 2^52) * (-p^-1) mod 2^52: the low half of one more split product
    const double t = to_dbl(c[k] & kMask);
    const double h = __fma_rz(t, M::NP52, 0x1p104);
    const double m = __fma_rz(t, M::NP52, 0x1.0000000000001p104 - h) - 0x1p52;
#pragma unroll
    for (int j = 0; j < 5; j++) acc_prod(m, M::L52(j), c[k + j], c[k + j + 1]);
  }
  uint64_t r[5];
  uint64_t carry = c[4] >> 52;
#pragma unroll
  for (int j = 0; j < 5; j++) {
    const uint64_t v = c[5 + j] + carry;
    carry = v >> 52;
    r[j] = j < 4 ? (v & kMask) : v;
  }
  const uint64_t w0 = r[0] | (r[1] << 52), w1 = (r[1] >> 12) | (r[2] << 40);
  const uint64_t w2 = (r[2] >> 24) | (r[3] << 28), w3 = (r[3] >> 36) | (r[4] << 16);
  out[0] = (uint32_t)w0; out[1] = (uint32_t)(w0 >> 32);
  out[2] = (uint32_t)w1; out[3] = (uint32_t)(w1 >> 32);
  out[4] = (uint32_t)w2; out[5] = (uint32_t)(w2 >> 32);
  out[6] = (uint32_t)w3; out[7] = (uint32_t)(w3 >> 32);
}
}  // namespace dp52

// ------------------------------------------------------------ carry-chain helpers ----
// Each helper is one PTX instruction; `volatile` keeps the carry flag sequence in
// program order.
#define ADD_CC(d, a, b)     asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define ADDC_CC(d, a, b)    asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define ADDC(d, a, b)       asm volatile("addc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define SUB_CC(d, a, b)     asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define SUBC_CC(d, a, b)    asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define SUBC(d, a, b)       asm volatile("subc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))

// t[0..8] += a[0..7] * b using 32x32->64 wide products (IMAD.WIDE): the even-index
// products a0b, a2b, a4b, a6b tile limbs 0..7 without overlap and the odd ones tile
// limbs 1..8, so each half is a ready 8-limb addend; two add.cc chains fold them in.
// Requires the true sum to fit in 9 limbs.
CSB_DEV void row_mad_wide(uint32_t (&t)[9], const uint32_t (&a)[8], uint32_t b) {
  asm volatile(
      "{\n\t.reg .b64 p;\n\t.reg .u32 lo, hi;\n\t"
      // even products: limbs 0..7, carry into t8
      "mul.wide.u32 p, %9, %17;\n\tmov.b64 {lo, hi}, p;\n\t"
      "add.cc.u32 %0, %0, lo;\n\taddc.cc.u32 %1, %1, hi;\n\t"
      "mul.wide.u32 p, %11, %17;\n\tmov.b64 {lo, hi}, p;\n\t"
      "addc.cc.u32 %2, %2, lo;\n\taddc.cc.u32 %3, %3, hi;\n\t"
      "mul.wide.u32 p, %13, %17;\n\tmov.b64 {lo, hi}, p;\n\t"
      "addc.cc.u32 %4, %4, lo;\n\taddc.cc.u32 %5, %5, hi;\n\t"
      "mul.wide.u32 p, %15, %17;\n\tmov.b64 {lo, hi}, p;\n\t"
      "addc.cc.u32 %6, %6, lo;\n\taddc.cc.u32 %7, %7, hi;\n\t"
      "addc.u32 %8, %8, 0;\n\t"
      // odd products: limbs 1..8
      "mul.wide.u32 p, %10, %17;\n\tmov.b64 {lo, hi}, p;\n\t"
      "add.cc.u32 %1, %1, lo;\n\taddc.cc.u32 %2, %2, hi;\n\t"
      "mul.wide.u32 p, %12, %17;\n\tmov.b64 {lo, hi}, p;\n\t"
      "addc.cc.u32 %3, %3, lo;\n\taddc.cc.u32 %4, %4, hi;\n\t"
      "mul.wide.u32 p, %14, %17;\n\tmov.b64 {lo, hi}, p;\n\t"
      "addc.cc.u32 %5, %5, lo;\n\taddc.cc.u32 %6, %6, hi;\n\t"
      "mul.wide.u32 p, %16, %17;\n\tmov.b64 {lo, hi}, p;\n\t"
      "addc.cc.u32 %7, %7, lo;\n\taddc.u32 %8, %8, hi;\n\t}"
      : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]),
        "+r"(t[7]), "+r"(t[8])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
        "r"(b));
}

template <class M>
struct Fp;
// Out-of-line Montgomery product (arguments and result in registers): keeps loop bodies
// that chain many products small enough for the instruction cache.
template <class M>
__device__ __noinline__ Fp<M> fp_mul_call(Fp<M> a, Fp<M> b);

template <class M>
struct Fp {
  uint32_t v[8];

  static CSB_DEV Fp zero() { Fp r; for (int i = 0; i < 8; i++) r.v[i] = 0; return r; }
  static CSB_DEV Fp one() {
    return Fp{{M::ONE0, M::ONE1, M::ONE2, M::ONE3, M::ONE4, M::ONE5, M::ONE6, M::ONE7}};
  }
  static CSB_DEV Fp r2() { return Fp{{M::R20, M::R21, M::R22, M::R23, M::R24, M::R25, M::R26, M::R27}}; }
  static CSB_DEV Fp r3() { return Fp{{M::R30, M::R31, M::R32, M::R33, M::R34, M::R35, M::R36, M::R37}}; }

  CSB_DEV bool is_zero() const {
    return (v[0] | v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7]) == 0;
  }
  CSB_DEV bool operator==(const Fp& o) const {
    return ((v[0] ^ o.v[0]) | (v[1] ^ o.v[1]) | (v[2] ^ o.v[2]) | (v[3] ^ o.v[3]) |
            (v[4] ^ o.v[4]) | (v[5] ^ o.v[5]) | (v[6] ^ o.v[6]) | (v[7] ^ o.v[7])) == 0;
  }
  CSB_DEV bool is_one() const { return *this == one(); }

  // r = t - p if t >= p else t, for t < 2p (t given in 8 limbs).
  static CSB_DEV void reduce_once(uint32_t (&t)[8]) {
    uint32_t u[8], br;
    SUB_CC(u[0], t[0], M::P0); SUBC_CC(u[1], t[1], M::P1); SUBC_CC(u[2], t[2], M::P2);
    SUBC_CC(u[3], t[3], M::P3); SUBC_CC(u[4], t[4], M::P4); SUBC_CC(u[5], t[5], M::P5);
    SUBC_CC(u[6], t[6], M::P6); SUBC_CC(u[7], t[7], M::P7); SUBC(br, 0u, 0u);
    // br = 0xffffffff if t < p (borrow), 0 otherwise
#pragma unroll
    for (int i = 0; i < 8; i++) t[i] = (t[i] & br) | (u[i] & ~br);
  }

  friend CSB_DEV Fp operator+(const Fp& a, const Fp& b) {
    uint32_t t[8];
    ADD_CC(t[0], a.v[0], b.v[0]);  ADDC_CC(t[1], a.v[1], b.v[1]); ADDC_CC(t[2], a.v[2], b.v[2]);
    ADDC_CC(t[3], a.v[3], b.v[3]); ADDC_CC(t[4], a.v[4], b.v[4]); ADDC_CC(t[5], a.v[5], b.v[5]);
    ADDC_CC(t[6], a.v[6], b.v[6]); ADDC(t[7], a.v[7], b.v[7]);
    reduce_once(t);
    Fp r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = t[i];
    return r;
  }
  friend CSB_DEV Fp operator-(const Fp& a, const Fp& b) {
    uint32_t t[8], br;
    SUB_CC(t[0], a.v[0], b.v[0]);  SUBC_CC(t[1], a.v[1], b.v[1]); SUBC_CC(t[2], a.v[2], b.v[2]);
    SUBC_CC(t[3], a.v[3], b.v[3]); SUBC_CC(t[4], a.v[4], b.v[4]); SUBC_CC(t[5], a.v[5], b.v[5]);
    SUBC_CC(t[6], a.v[6], b.v[6]); SUBC_CC(t[7], a.v[7], b.v[7]); SUBC(br, 0u, 0u);
    // add p back if the subtraction borrowed
    const uint32_t p0 = M::P0 & br, p1 = M::P1 & br, p2 = M::P2 & br, p3 = M::P3 & br;
    const uint32_t p4 = M::P4 & br, p5 = M::P5 & br, p6 = M::P6 & br, p7 = M::P7 & br;
    Fp r;
    ADD_CC(r.v[0], t[0], p0);  ADDC_CC(r.v[1], t[1], p1); ADDC_CC(r.v[2], t[2], p2);
    ADDC_CC(r.v[3], t[3], p3); ADDC_CC(r.v[4], t[4], p4); ADDC_CC(r.v[5], t[5], p5);
    ADDC_CC(r.v[6], t[6], p6); ADDC(r.v[7], t[7], p7);
    return r;
  }
  CSB_DEV Fp neg() const { return zero() - *this; }
  CSB_DEV Fp dbl() const { return *this + *this; }

  // CIOS Montgomery product with wide (IMAD.WIDE) row products.
  static CSB_DEV Fp mul_wide(const Fp& a, const Fp& b) {
    const uint32_t (&A)[8] = a.v;
    const uint32_t P[8] = {M::P0, M::P1, M::P2, M::P3, M::P4, M::P5, M::P6, M::P7};
    uint32_t t[9];
#pragma unroll
    for (int i = 0; i < 9; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      row_mad_wide(t, A, b.v[i]);
      const uint32_t m = t[0] * M::NP0;
      row_mad_wide(t, P, m);
#pragma unroll
      for (int j = 0; j < 8; j++) t[j] = t[j + 1];
      t[8] = 0;
    }
    uint32_t r8[8];
#pragma unroll
    for (int i = 0; i < 8; i++) r8[i] = t[i];
    reduce_once(r8);
    Fp r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = r8[i];
    return r;
  }

  // ---- lazily reduced values in [0, 2p) (BN254: 4p < 2^256) --------------------------
  // CIOS without the final conditional subtraction: for a, b < 2p the result is below
  // (a b + m p) / 2^256 < (4p^2 + 2^256 p) / 2^256 < 2p.
  static CSB_DEV Fp mul_wide_lazy(const Fp& a, const Fp& b) {
    const uint32_t P[8] = {M::P0, M::P1, M::P2, M::P3, M::P4, M::P5, M::P6, M::P7};
    uint32_t t[9];
#pragma unroll
    for (int i = 0; i < 9; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      row_mad_wide(t, a.v, b.v[i]);
      const uint32_t m = t[0] * M::NP0;
      row_mad_wide(t, P, m);
#pragma unroll
      for (int j = 0; j < 8; j++) t[j] = t[j + 1];
      t[8] = 0;
    }
    Fp r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = t[i];
    return r;
  }
  static CSB_DEV Fp mul_lazy(const Fp& a, const Fp& b);
  // 2p, limb i
  static CSB_DEV uint32_t p2(int i) {
    const uint32_t P[8] = {M::P0, M::P1, M::P2, M::P3, M::P4, M::P5, M::P6, M::P7};
    return (P[i] << 1) | (i > 0 ? P[i - 1] >> 31 : 0u);
  }
  // a + b for a, b < 2p, result < 2p
  static CSB_DEV Fp add_lazy(const Fp& a, const Fp& b) {
    uint32_t t[8], u[8], br;
    ADD_CC(t[0], a.v[0], b.v[0]);  ADDC_CC(t[1], a.v[1], b.v[1]); ADDC_CC(t[2], a.v[2], b.v[2]);
    ADDC_CC(t[3], a.v[3], b.v[3]); ADDC_CC(t[4], a.v[4], b.v[4]); ADDC_CC(t[5], a.v[5], b.v[5]);
    ADDC_CC(t[6], a.v[6], b.v[6]); ADDC(t[7], a.v[7], b.v[7]);
    SUB_CC(u[0], t[0], p2(0)); SUBC_CC(u[1], t[1], p2(1)); SUBC_CC(u[2], t[2], p2(2));
    SUBC_CC(u[3], t[3], p2(3)); SUBC_CC(u[4], t[4], p2(4)); SUBC_CC(u[5], t[5], p2(5));
    SUBC_CC(u[6], t[6], p2(6)); SUBC_CC(u[7], t[7], p2(7)); SUBC(br, 0u, 0u);
    Fp r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = (t[i] & br) | (u[i] & ~br);
    return r;
  }
  // a - b for a, b < 2p, result < 2p
  static CSB_DEV Fp sub_lazy(const Fp& a, const Fp& b) {
    uint32_t t[8], br;
    SUB_CC(t[0], a.v[0], b.v[0]);  SUBC_CC(t[1], a.v[1], b.v[1]); SUBC_CC(t[2], a.v[2], b.v[2]);
    SUBC_CC(t[3], a.v[3], b.v[3]); SUBC_CC(t[4], a.v[4], b.v[4]); SUBC_CC(t[5], a.v[5], b.v[5]);
    SUBC_CC(t[6], a.v[6], b.v[6]); SUBC_CC(t[7], a.v[7], b.v[7]); SUBC(br, 0u, 0u);
    Fp r;
    ADD_CC(r.v[0], t[0], p2(0) & br);  ADDC_CC(r.v[1], t[1], p2(1) & br); ADDC_CC(r.v[2], t[2], p2(2) & br);
    ADDC_CC(r.v[3], t[3], p2(3) & br); ADDC_CC(r.v[4], t[4], p2(4) & br); ADDC_CC(r.v[5], t[5], p2(5) & br);
    ADDC_CC(r.v[6], t[6], p2(6) & br); ADDC(r.v[7], t[7], p2(7) & br);
    return r;
  }
  // zero mod p for a value < 2p: 0 or p
  CSB_DEV bool is_zero_lazy() const {
    const uint32_t z = v[0] | v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7];
    const uint32_t e = (v[0] ^ M::P0) | (v[1] ^ M::P1) | (v[2] ^ M::P2) | (v[3] ^ M::P3) | (v[4] ^ M::P4) |
                       (v[5] ^ M::P5) | (v[6] ^ M::P6) | (v[7] ^ M::P7);
    return z == 0 || e == 0;
  }
  // the canonical representative in [0, p) of a value < 2p
  CSB_DEV Fp canon() const {
    uint32_t t[8];
#pragma unroll
    for (int i = 0; i < 8; i++) t[i] = v[i];
    reduce_once(t);
    Fp r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = t[i];
    return r;
  }

  friend CSB_DEV Fp operator*(const Fp& a, const Fp& b) {
#if defined(CSB_MUL_NOINLINE)
    return fp_mul_call<M>(a, b);
#else
    return mul_wide(a, b);
#endif
  }

  CSB_DEV Fp sqr() const { return (*this) * (*this); }

  // x -> x * R mod p (normal form to Montgomery); any 256-bit x < 2^256 is accepted
  // because the CIOS bound only needs a*b < p * 2^256.
  CSB_DEV Fp to_mont() const { return (*this) * r2(); }
  CSB_DEV Fp from_mont() const {
    Fp o = zero();
    o.v[0] = 1;
    return (*this) * o;
  }

  // Montgomery inverse (aR -> a^-1 R; 0 -> 0).  Binary extended Euclid on the integer
  // x = aR gives x^-1 = a^-1 R^-1; one Montgomery product by R^3 restores a^-1 R.  Used
  // for the few final affine conversions, where a single thread's latency is what counts.
  CSB_DEV Fp inv() const {
    if (is_zero()) return zero();
    const uint32_t P[8] = {M::P0, M::P1, M::P2, M::P3, M::P4, M::P5, M::P6, M::P7};
    uint32_t u[8], v[8], x1[8], x2[8];
#pragma unroll
    for (int i = 0; i < 8; i++) { u[i] = this->v[i]; v[i] = P[i]; x1[i] = 0; x2[i] = 0; }
    x1[0] = 1;
#pragma unroll 1
    for (int guard = 0; guard < 2048; guard++) {
      const bool u1 = (u[0] == 1) && ((u[1] | u[2] | u[3] | u[4] | u[5] | u[6] | u[7]) == 0);
      const bool v1 = (v[0] == 1) && ((v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7]) == 0);
      if (u1 || v1) break;
      // (a zero u or v only arises from an unreduced input; the bounded loops end anyway)
#pragma unroll 1
      for (int k = 0; k < 256 && (u[0] & 1u) == 0; k++) { shr1(u); half_mod(x1, P); }
#pragma unroll 1
      for (int k = 0; k < 256 && (v[0] & 1u) == 0; k++) { shr1(v); half_mod(x2, P); }
      if (geq(u, v)) { sub8(u, v); sub_mod(x1, x2, P); }
      else { sub8(v, u); sub_mod(x2, x1, P); }
    }
    const bool u1 = (u[0] == 1) && ((u[1] | u[2] | u[3] | u[4] | u[5] | u[6] | u[7]) == 0);
    Fp r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = u1 ? x1[i] : x2[i];
    return r * r3();
  }

 private:
  static CSB_DEV void shr1(uint32_t (&a)[8]) {
#pragma unroll
    for (int i = 0; i < 7; i++) a[i] = (a[i] >> 1) | (a[i + 1] << 31);
    a[7] >>= 1;
  }
  static CSB_DEV bool geq(const uint32_t (&a)[8], const uint32_t (&b)[8]) {
#pragma unroll
    for (int i = 7; i >= 0; i--) {
      if (a[i] != b[i]) return a[i] > b[i];
    }
    return true;
  }
  static CSB_DEV void sub8(uint32_t (&a)[8], const uint32_t (&b)[8]) {
    SUB_CC(a[0], a[0], b[0]); SUBC_CC(a[1], a[1], b[1]); SUBC_CC(a[2], a[2], b[2]);
    SUBC_CC(a[3], a[3], b[3]); SUBC_CC(a[4], a[4], b[4]); SUBC_CC(a[5], a[5], b[5]);
    SUBC_CC(a[6], a[6], b[6]); SUBC(a[7], a[7], b[7]);
  }
  // x <- x/2 mod p for x < p
  static CSB_DEV void half_mod(uint32_t (&x)[8], const uint32_t (&P)[8]) {
    if (x[0] & 1u) {
      uint32_t c;
      ADD_CC(x[0], x[0], P[0]); ADDC_CC(x[1], x[1], P[1]); ADDC_CC(x[2], x[2], P[2]);
      ADDC_CC(x[3], x[3], P[3]); ADDC_CC(x[4], x[4], P[4]); ADDC_CC(x[5], x[5], P[5]);
      ADDC_CC(x[6], x[6], P[6]); ADDC_CC(x[7], x[7], P[7]); ADDC(c, 0u, 0u);
      shr1(x);
      x[7] |= c << 31;
    } else {
      shr1(x);
    }
  }
  // x <- x - y mod p for x, y < p
  static CSB_DEV void sub_mod(uint32_t (&x)[8], const uint32_t (&y)[8], const uint32_t (&P)[8]) {
    uint32_t br;
    SUB_CC(x[0], x[0], y[0]); SUBC_CC(x[1], x[1], y[1]); SUBC_CC(x[2], x[2], y[2]);
    SUBC_CC(x[3], x[3], y[3]); SUBC_CC(x[4], x[4], y[4]); SUBC_CC(x[5], x[5], y[5]);
    SUBC_CC(x[6], x[6], y[6]); SUBC_CC(x[7], x[7], y[7]); SUBC(br, 0u, 0u);
    if (br) {
      ADD_CC(x[0], x[0], P[0]); ADDC_CC(x[1], x[1], P[1]); ADDC_CC(x[2], x[2], P[2]);
      ADDC_CC(x[3], x[3], P[3]); ADDC_CC(x[4], x[4], P[4]); ADDC_CC(x[5], x[5], P[5]);
      ADDC_CC(x[6], x[6], P[6]); ADDC(x[7], x[7], P[7]);
    }
  }

 public:
};

using Fq = Fp<ModQ>;
using Fr = Fp<ModR>;

// ------------------------------------------------------------ Fq2 = Fq[u]/(u^2+1) ----
template <class M>
__device__ __noinline__ Fp<M> fp_mul_call(Fp<M> a, Fp<M> b) {
#if CSB_DP52
  Fp<M> r;
  dp52::mont<M>(a.v, b.v, r.v);
  return r.canon();
#else
  return Fp<M>::mul_wide(a, b);
#endif
}

template <class M>
__device__ __noinline__ Fp<M> fp_mul_lazy_call(Fp<M> a, Fp<M> b) {
#if CSB_DP52
  Fp<M> r;
  dp52::mont<M>(a.v, b.v, r.v);
  return r;
#else
  return Fp<M>::mul_wide_lazy(a, b);
#endif
}

template <class M>
CSB_DEV Fp<M> Fp<M>::mul_lazy(const Fp<M>& a, const Fp<M>& b) {
#if defined(CSB_MUL_NOINLINE)
  return fp_mul_lazy_call<M>(a, b);
#else
  return mul_wide_lazy(a, b);
#endif
}

struct Fq2 {
  Fq c0, c1;
  static CSB_DEV Fq2 zero() { return {Fq::zero(), Fq::zero()}; }
  static CSB_DEV Fq2 one() { return {Fq::one(), Fq::zero()}; }
  CSB_DEV bool is_zero() const { return c0.is_zero() && c1.is_zero(); }
  CSB_DEV bool operator==(const Fq2& o) const { return c0 == o.c0 && c1 == o.c1; }
  friend CSB_DEV Fq2 operator+(const Fq2& a, const Fq2& b) { return {a.c0 + b.c0, a.c1 + b.c1}; }
  friend CSB_DEV Fq2 operator-(const Fq2& a, const Fq2& b) { return {a.c0 - b.c0, a.c1 - b.c1}; }
  // Karatsuba, 3 products (src/cuda/ff.cpp montmult_ext_h: same non-residue -1)
  friend CSB_DEV Fq2 operator*(const Fq2& a, const Fq2& b) {
    const Fq v0 = a.c0 * b.c0;
    const Fq v1 = a.c1 * b.c1;
    const Fq s = (a.c0 + a.c1) * (b.c0 + b.c1);
    return {v0 - v1, s - v0 - v1};
  }
  // (a0 + a1 u)^2 = (a0 + a1)(a0 - a1) + 2 a0 a1 u
  CSB_DEV Fq2 sqr() const {
    const Fq p = c0 * c1;
    return {(c0 + c1) * (c0 - c1), p + p};
  }
  CSB_DEV Fq2 neg() const { return {c0.neg(), c1.neg()}; }
  CSB_DEV Fq2 dbl() const { return {c0.dbl(), c1.dbl()}; }
  CSB_DEV Fq2 inv() const {
    const Fq d = (c0.sqr() + c1.sqr()).inv();
    return {c0 * d, (c1 * d).neg()};
  }
};

}  // namespace csb
