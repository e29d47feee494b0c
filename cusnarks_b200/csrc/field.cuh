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
#ifndef CSB_FQ2_MODE
#define CSB_FQ2_MODE 0  // Fq2 product: 0 CIOS x3, 1 carry-flag-free CIOS x3, 2 lazy reduction
#endif

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
  // q^2, 16 limbs (lazy-reduction offset)
  static CSB_DEV uint32_t P2_LIMB(int i) {
    constexpr uint32_t k[16] = {0x275d69b1u, 0x3b5458a2u, 0x09eac101u, 0xa602072du,
                                0x6d96cadcu, 0x4a50189cu, 0x7a1242c8u, 0x04689e95u,
                                0x34c6b38du, 0x26edfa5cu, 0x16375606u, 0xb00b8551u,
                                0x0348d21cu, 0x599a6f7cu, 0x763cbf9cu, 0x0925c4b8u};
    return k[i];
  }
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

// Paired products (CSB_PAIR, opt-in; only with out-of-line products): Fp::mul2 computes two
// independent products in one call with their rows interleaved.  Measured at 2^20: the G1
// MSM alone 3 % faster (accumulation capped at 128 registers), a whole proof 2.7 % slower
// (its five MSMs share the SMs and the paired body doubles the multiply's code), so off.
#if defined(CSB_PAIR) && defined(CSB_MUL_NOINLINE) && !defined(CSB_MUL_LOHI)
#define CSB_PAIRED 1
#else
#define CSB_PAIRED 0
#endif

// ------------------------------------------------------------ carry-chain helpers ----
// Each helper is one PTX instruction; `volatile` keeps the carry flag sequence in
// program order.
#define MAD_LO_CC(d, a, b)  asm volatile("mad.lo.cc.u32 %0, %1, %2, %0;" : "+r"(d) : "r"(a), "r"(b))
#define MADC_LO_CC(d, a, b) asm volatile("madc.lo.cc.u32 %0, %1, %2, %0;" : "+r"(d) : "r"(a), "r"(b))
#define MAD_HI_CC(d, a, b)  asm volatile("mad.hi.cc.u32 %0, %1, %2, %0;" : "+r"(d) : "r"(a), "r"(b))
#define MADC_HI_CC(d, a, b) asm volatile("madc.hi.cc.u32 %0, %1, %2, %0;" : "+r"(d) : "r"(a), "r"(b))
#define MADC_HI(d, a, b)    asm volatile("madc.hi.u32 %0, %1, %2, %0;" : "+r"(d) : "r"(a), "r"(b))
#define ADDC_Z(d)           asm volatile("addc.u32 %0, 0, 0;" : "=r"(d))
#define ADD_CC(d, a, b)     asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define ADDC_CC(d, a, b)    asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define ADDC(d, a, b)       asm volatile("addc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define SUB_CC(d, a, b)     asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define SUBC_CC(d, a, b)    asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define SUBC(d, a, b)       asm volatile("subc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))

// t[0..8] += a[0..7] * b.  Requires the true sum to fit in 9 limbs.
CSB_DEV void row_mad(uint32_t (&t)[9], const uint32_t (&a)[8], uint32_t b) {
  MAD_LO_CC(t[0], a[0], b);  MADC_LO_CC(t[1], a[1], b); MADC_LO_CC(t[2], a[2], b);
  MADC_LO_CC(t[3], a[3], b); MADC_LO_CC(t[4], a[4], b); MADC_LO_CC(t[5], a[5], b);
  MADC_LO_CC(t[6], a[6], b); MADC_LO_CC(t[7], a[7], b);
  uint32_t c; ADDC_Z(c); t[8] += c;
  MAD_HI_CC(t[1], a[0], b);  MADC_HI_CC(t[2], a[1], b); MADC_HI_CC(t[3], a[2], b);
  MADC_HI_CC(t[4], a[3], b); MADC_HI_CC(t[5], a[4], b); MADC_HI_CC(t[6], a[5], b);
  MADC_HI_CC(t[7], a[6], b); MADC_HI(t[8], a[7], b);
}

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
template <class M>
struct FpPair;
// Out-of-line Montgomery product (arguments and result in registers): keeps loop bodies
// that chain many products small enough for the instruction cache.
template <class M>
__device__ __noinline__ Fp<M> fp_mul_call(Fp<M> a, Fp<M> b);
// Out-of-line pair of independent products (a*b, c*d) with interleaved rows.
template <class M>
__device__ __noinline__ FpPair<M> fp_mul2_call(Fp<M> a, Fp<M> b, Fp<M> c, Fp<M> d);

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

  // Two independent CIOS products x = a*b, y = c*d with their rows interleaved: the carry
  // chains of one product fill the fixed-latency dependency stalls of the other, which a
  // single product (one long serial chain) cannot.
  static CSB_DEV void mul_wide2(const Fp& a, const Fp& b, const Fp& c, const Fp& d, Fp& x, Fp& y) {
    const uint32_t P[8] = {M::P0, M::P1, M::P2, M::P3, M::P4, M::P5, M::P6, M::P7};
    uint32_t t[9], u[9];
#pragma unroll
    for (int i = 0; i < 9; i++) { t[i] = 0; u[i] = 0; }
#pragma unroll
    for (int i = 0; i < 8; i++) {
      row_mad_wide(t, a.v, b.v[i]);
      row_mad_wide(u, c.v, d.v[i]);
      const uint32_t mt = t[0] * M::NP0;
      const uint32_t mu = u[0] * M::NP0;
      row_mad_wide(t, P, mt);
      row_mad_wide(u, P, mu);
#pragma unroll
      for (int j = 0; j < 8; j++) { t[j] = t[j + 1]; u[j] = u[j + 1]; }
      t[8] = 0;
      u[8] = 0;
    }
    uint32_t r8[8], s8[8];
#pragma unroll
    for (int i = 0; i < 8; i++) { r8[i] = t[i]; s8[i] = u[i]; }
    reduce_once(r8);
    reduce_once(s8);
#pragma unroll
    for (int i = 0; i < 8; i++) { x.v[i] = r8[i]; y.v[i] = s8[i]; }
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

  // x = a*b, y = c*d in one out-of-line call with interleaved rows (any unit): about the
  // latency of one product for two, where a single thread's chain is the cost.
  static CSB_DEV void mul2_ool(const Fp& a, const Fp& b, const Fp& c, const Fp& d, Fp& x, Fp& y) {
    const FpPair<M> r = fp_mul2_call<M>(a, b, c, d);
    x = r.x;
    y = r.y;
  }
  static CSB_DEV void sqr2_ool(const Fp& a, const Fp& c, Fp& x, Fp& y) { mul2_ool(a, a, c, c, x, y); }

  // x = a*b, y = c*d.  With CSB_PAIR one out-of-line call computes both with interleaved
  // rows; otherwise two products (inlined ones are scheduled together anyway).
  static CSB_DEV void mul2(const Fp& a, const Fp& b, const Fp& c, const Fp& d, Fp& x, Fp& y) {
#if CSB_PAIRED
    mul2_ool(a, b, c, d, x, y);
#else
    const Fp xx = a * b;
    y = c * d;
    x = xx;
#endif
  }
  // x = a^2, y = c^2
  static CSB_DEV void sqr2(const Fp& a, const Fp& c, Fp& x, Fp& y) { mul2(a, a, c, c, x, y); }

  // CIOS Montgomery product in plain 64-bit C++ arithmetic (no carry flag): independent
  // products can be interleaved by the compiler.
  static CSB_DEV Fp mul_c64(const Fp& a, const Fp& b) {
    const uint32_t P[8] = {M::P0, M::P1, M::P2, M::P3, M::P4, M::P5, M::P6, M::P7};
    uint32_t t[10];
#pragma unroll
    for (int i = 0; i < 10; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      uint64_t c = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const uint64_t s = (uint64_t)a.v[j] * b.v[i] + t[j] + c;
        t[j] = (uint32_t)s;
        c = s >> 32;
      }
      const uint64_t s8 = (uint64_t)t[8] + c;
      t[8] = (uint32_t)s8;
      t[9] = (uint32_t)(s8 >> 32);
      const uint32_t m = t[0] * M::NP0;
      uint64_t c2 = ((uint64_t)m * P[0] + t[0]) >> 32;
#pragma unroll
      for (int j = 1; j < 8; j++) {
        const uint64_t s = (uint64_t)m * P[j] + t[j] + c2;
        t[j - 1] = (uint32_t)s;
        c2 = s >> 32;
      }
      const uint64_t s7 = (uint64_t)t[8] + c2;
      t[7] = (uint32_t)s7;
      t[8] = t[9] + (uint32_t)(s7 >> 32);
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

  // Full 512-bit product a*b (16 limbs), 64-bit C++ arithmetic.
  static CSB_DEV void mul_full(uint32_t (&t)[16], const Fp& a, const Fp& b) {
#pragma unroll
    for (int i = 0; i < 16; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      uint64_t c = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const uint64_t s = (uint64_t)a.v[j] * b.v[i] + t[i + j] + c;
        t[i + j] = (uint32_t)s;
        c = s >> 32;
      }
      t[i + 8] = (uint32_t)c;
    }
  }

  // Montgomery reduction T * 2^-256 mod p for T < p * 2^256 (16 limbs, consumed).
  static CSB_DEV Fp redc(uint32_t (&t)[16]) {
    const uint32_t P[8] = {M::P0, M::P1, M::P2, M::P3, M::P4, M::P5, M::P6, M::P7};
    uint32_t hi = 0;  // overflow of limb i+8, owed to limb i+9
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const uint32_t m = t[i] * M::NP0;
      uint64_t c = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const uint64_t s = (uint64_t)m * P[j] + t[i + j] + c;
        t[i + j] = (uint32_t)s;
        c = s >> 32;
      }
      // row carry into limb i+8; its own overflow goes to limb i+9 with the next row
      const uint64_t s8 = (uint64_t)t[i + 8] + c + hi;
      t[i + 8] = (uint32_t)s8;
      hi = (uint32_t)(s8 >> 32);
    }
    // T < p 2^256 keeps the result below 2p < 2^256: hi is 0 here
    uint32_t r8[8];
#pragma unroll
    for (int i = 0; i < 8; i++) r8[i] = t[8 + i];
    reduce_once(r8);
    Fp r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = r8[i];
    return r;
  }

  friend CSB_DEV Fp operator*(const Fp& a, const Fp& b) {
#if defined(CSB_MUL_LOHI)
    return mul_lohi(a, b);
#elif defined(CSB_MUL_NOINLINE)
    return fp_mul_call<M>(a, b);
#else
    return mul_wide(a, b);
#endif
  }

  // CIOS Montgomery product with mad.lo / mad.hi carry chains.
  static CSB_DEV Fp mul_lohi(const Fp& a, const Fp& b) {
    const uint32_t (&A)[8] = a.v;
    const uint32_t P[8] = {M::P0, M::P1, M::P2, M::P3, M::P4, M::P5, M::P6, M::P7};
    uint32_t t[9];
#pragma unroll
    for (int i = 0; i < 9; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      row_mad(t, A, b.v[i]);
      const uint32_t m = t[0] * M::NP0;
      row_mad(t, P, m);
      // t[0] is now zero: shift one limb down
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
#if defined(CSB_MUL_CALL_LOHI)
  return Fp<M>::mul_lohi(a, b);
#elif CSB_DP52
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

template <class M>
struct FpPair {
  Fp<M> x, y;
};

template <class M>
__device__ __noinline__ FpPair<M> fp_mul2_call(Fp<M> a, Fp<M> b, Fp<M> c, Fp<M> d) {
  FpPair<M> r;
  Fp<M>::mul_wide2(a, b, c, d, r.x, r.y);
  return r;
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
#if CSB_FQ2_MODE == 1
    const Fq v0 = Fq::mul_c64(a.c0, b.c0);
    const Fq v1 = Fq::mul_c64(a.c1, b.c1);
    const Fq s = Fq::mul_c64(a.c0 + a.c1, b.c0 + b.c1);
    return {v0 - v1, s - v0 - v1};
#elif CSB_FQ2_MODE == 2
    return mul_lazy(a, b);
#elif CSB_PAIRED
    Fq v0, v1;
    Fq::mul2(a.c0, b.c0, a.c1, b.c1, v0, v1);
    const Fq s = (a.c0 + a.c1) * (b.c0 + b.c1);
    return {v0 - v1, s - v0 - v1};
#else
    const Fq v0 = a.c0 * b.c0;
    const Fq v1 = a.c1 * b.c1;
    const Fq s = (a.c0 + a.c1) * (b.c0 + b.c1);
    return {v0 - v1, s - v0 - v1};
#endif
  }
  // x = a*b, y = c*d: six Fq products as three interleaved out-of-line pairs
  static CSB_DEV void mul2_ool(const Fq2& a, const Fq2& b, const Fq2& c, const Fq2& d, Fq2& x, Fq2& y) {
    Fq a0, a1, c0, c1, sa, sc;
    Fq::mul2_ool(a.c0, b.c0, a.c1, b.c1, a0, a1);
    Fq::mul2_ool(c.c0, d.c0, c.c1, d.c1, c0, c1);
    Fq::mul2_ool(a.c0 + a.c1, b.c0 + b.c1, c.c0 + c.c1, d.c0 + d.c1, sa, sc);
    x = {a0 - a1, sa - a0 - a1};
    y = {c0 - c1, sc - c0 - c1};
  }
  // x = a^2, y = c^2: four Fq products as two out-of-line pairs
  static CSB_DEV void sqr2_ool(const Fq2& a, const Fq2& c, Fq2& x, Fq2& y) {
    Fq pa, pc, qa, qc;
    Fq::mul2_ool(a.c0, a.c1, c.c0, c.c1, pa, pc);
    Fq::mul2_ool(a.c0 + a.c1, a.c0 - a.c1, c.c0 + c.c1, c.c0 - c.c1, qa, qc);
    x = {qa, pa + pa};
    y = {qc, pc + pc};
  }
  static CSB_DEV void mul2(const Fq2& a, const Fq2& b, const Fq2& c, const Fq2& d, Fq2& x, Fq2& y) {
#if CSB_PAIRED
    mul2_ool(a, b, c, d, x, y);
#else
    const Fq2 xx = a * b;
    y = c * d;
    x = xx;
#endif
  }
  static CSB_DEV void sqr2(const Fq2& a, const Fq2& c, Fq2& x, Fq2& y) {
#if CSB_PAIRED
    sqr2_ool(a, c, x, y);
#else
    const Fq2 xx = a.sqr();
    y = c.sqr();
    x = xx;
#endif
  }
  // Karatsuba with lazy reduction: three 512-bit products, two Montgomery reductions.
  //   c0 = a0 b0 - a1 b1 + p^2 (in [0, 2p^2)),  c1 = (a0+a1)(b0+b1) - a0 b0 - a1 b1 (< 2p^2)
  // with the sums a0+a1, b0+b1 unreduced (< 2^255); both stay below p 2^256.
  static CSB_DEV Fq2 mul_lazy(const Fq2& a, const Fq2& b) {
    uint32_t v0[16], v1[16], s[16];
    Fq::mul_full(v0, a.c0, b.c0);
    Fq::mul_full(v1, a.c1, b.c1);
    Fq sa, sb;
    {
      uint64_t ca = 0, cb = 0;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        ca += (uint64_t)a.c0.v[i] + a.c1.v[i];
        cb += (uint64_t)b.c0.v[i] + b.c1.v[i];
        sa.v[i] = (uint32_t)ca;
        sb.v[i] = (uint32_t)cb;
        ca >>= 32;
        cb >>= 32;
      }
    }
    Fq::mul_full(s, sa, sb);
    // s <- s - v0 - v1 ; v0 <- v0 - v1 + p^2
    int64_t bs = 0, b0 = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) {
      bs += (int64_t)s[i] - v0[i] - v1[i];
      b0 += (int64_t)v0[i] - v1[i] + ModQ::P2_LIMB(i);
      s[i] = (uint32_t)bs;
      v0[i] = (uint32_t)b0;
      bs >>= 32;  // arithmetic shift: borrow in -2..0
      b0 >>= 32;
    }
    return {Fq::redc(v0), Fq::redc(s)};
  }
  // (a0 + a1 u)^2 = (a0 + a1)(a0 - a1) + 2 a0 a1 u
  CSB_DEV Fq2 sqr() const {
#if CSB_PAIRED
    Fq p, q;
    Fq::mul2(c0, c1, c0 + c1, c0 - c1, p, q);
    return {q, p + p};
#else
    const Fq p = c0 * c1;
    return {(c0 + c1) * (c0 - c1), p + p};
#endif
  }
  CSB_DEV Fq2 neg() const { return {c0.neg(), c1.neg()}; }
  CSB_DEV Fq2 dbl() const { return {c0.dbl(), c1.dbl()}; }
  CSB_DEV Fq2 inv() const {
    const Fq d = (c0.sqr() + c1.sqr()).inv();
    return {c0 * d, (c1 * d).neg()};
  }
};

}  // namespace csb
