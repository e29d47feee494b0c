// glv.cuh -- scalar decomposition for the GLV endomorphism of BN254 G1, host and device.
//
// phi(x, y) = (beta x, y) = lambda P with beta^3 = 1 in Fq and lambda^2 + lambda + 1 = 0 in Fr.
// A scalar k < r splits as k = k1 + k2 lambda (mod r) with |k1|, |k2| < 2^127, from the short
// lattice basis (a1, b1), (a2, b2) of {(x, y) : x + y lambda = 0 mod r} (extended Euclid on
// (r, lambda); b2 = a1, b1 < 0):
//   c1 = round(b2 k / r), c2 = round(-b1 k / r)   (as (k g1) >> 256 and (k g2) >> 256),
//   k1 = k - c1 a1 - c2 a2,  k2 = c1 |b1| - c2 b2.
// Used by the proof's r, s scalings (one scalar each, on the host) and by the generic G1 MSM
// (every scalar, on the device): k P = k1 P + k2 phi(P) needs 127 doublings, not 254.
#pragma once
#include <cstdint>

namespace csb {
namespace glv {

constexpr uint64_t G1C[2] = {0xd91d232ec7e0b3d7ull, 0x2ull};
constexpr uint64_t G2C[3] = {0x7a7bd9d4391eb18eull, 0x4ccef014a773d2cfull, 0x2ull};
constexpr uint64_t A1 = 0x89d3256894d213e3ull;  // = b2
constexpr uint64_t A2[2] = {0x0be4e1541221250bull, 0x6f4d8248eeb859fdull};
constexpr uint64_t B1ABS[2] = {0x8211bbeb7d4f1128ull, 0x6f4d8248eeb859fcull};
// beta in Montgomery form (Fq), 8 little-endian words (written as immediates: device code
// cannot index a host constant array)
__host__ __device__ inline void beta_mont(uint32_t* b) {
  b[0] = 0xd782e155u; b[1] = 0x71930c11u; b[2] = 0xffbe3323u; b[3] = 0xa6bb947cu;
  b[4] = 0xd4741444u; b[5] = 0xaa303344u; b[6] = 0x26594943u; b[7] = 0x2c3b3f0du;
}

__host__ __device__ inline uint64_t mul64(uint64_t a, uint64_t b, uint64_t& hi) {
#ifdef __CUDA_ARCH__
  hi = __umul64hi(a, b);
  return a * b;
#else
  const unsigned __int128 p = (unsigned __int128)a * b;
  hi = (uint64_t)(p >> 64);
  return (uint64_t)p;
#endif
}

// r[0 .. na+nb) = a * b (little-endian 64-bit limbs)
__host__ __device__ inline void mulv(const uint64_t* a, int na, const uint64_t* b, int nb, uint64_t* r) {
  for (int i = 0; i < na + nb; i++) r[i] = 0;
  for (int i = 0; i < na; i++) {
    uint64_t carry = 0;
    for (int j = 0; j < nb; j++) {
      uint64_t hi;
      const uint64_t lo = mul64(a[i], b[j], hi);
      uint64_t s = r[i + j] + lo;
      uint64_t c = s < lo;
      s += carry;
      c += s < carry;
      r[i + j] = s;
      carry = hi + c;  // hi <= 2^64 - 2: no overflow
    }
    r[i + nb] = carry;
  }
}

// acc (4 limbs, mod 2^256) += v or -= v (v up to 4 limbs)
__host__ __device__ inline void addsub(uint64_t* acc, const uint64_t* v, int nv, bool sub) {
  uint64_t carry = sub ? 1 : 0;  // two's complement: acc + ~v + 1
  for (int i = 0; i < 4; i++) {
    const uint64_t w = i < nv ? v[i] : 0;
    const uint64_t x = sub ? ~w : w;
    uint64_t s = acc[i] + x;
    uint64_t c = s < x;
    s += carry;
    c += s < carry;
    acc[i] = s;
    carry = c;
  }
}

// |v| (below 2^127) as four 32-bit words, and the sign of the two's complement value v
__host__ __device__ inline void to_mag(const uint64_t* v, uint32_t* mag, uint32_t* neg) {
  uint64_t t[4] = {v[0], v[1], v[2], v[3]};
  *neg = (t[3] >> 63) ? 1u : 0u;
  if (*neg) {
    uint64_t carry = 1;
    for (int i = 0; i < 4; i++) {
      const uint64_t s = ~t[i] + carry;
      carry = (carry && s == 0) ? 1 : 0;
      t[i] = s;
    }
  }
  for (int i = 0; i < 2; i++) {
    mag[2 * i] = (uint32_t)t[i];
    mag[2 * i + 1] = (uint32_t)(t[i] >> 32);
  }
}

// k (< r, four 64-bit limbs) -> |k1|, |k2| (four 32-bit words each) and their signs
__host__ __device__ inline void split_reduced(const uint64_t* k, uint32_t* k1m, uint32_t* neg1, uint32_t* k2m,
                                              uint32_t* neg2) {
  // local copies: device code reads the constants as immediates
  const uint64_t g1c[2] = {G1C[0], G1C[1]}, g2c[3] = {G2C[0], G2C[1], G2C[2]};
  const uint64_t a1[1] = {A1}, a2[2] = {A2[0], A2[1]}, b1[2] = {B1ABS[0], B1ABS[1]};
  uint64_t p1[6], p2[7];
  mulv(k, 4, g1c, 2, p1);
  mulv(k, 4, g2c, 3, p2);
  const uint64_t c1[1] = {p1[4]};         // < 2^64
  const uint64_t c2[2] = {p2[4], p2[5]};  // < 2^128
  uint64_t t[4];
  uint64_t k1[4] = {k[0], k[1], k[2], k[3]}, k2[4] = {0, 0, 0, 0};
  mulv(c1, 1, a1, 1, t);  // c1 a1 (2 limbs)
  addsub(k1, t, 2, true);
  uint64_t t4[4];
  mulv(c2, 2, a2, 2, t4);  // c2 a2
  addsub(k1, t4, 4, true);
  mulv(c1, 1, b1, 2, t);  // c1 |b1| (3 limbs)
  addsub(k2, t, 3, false);
  mulv(c2, 2, a1, 1, t);  // c2 b2, b2 = a1 (3 limbs)
  addsub(k2, t, 3, true);
  to_mag(k1, k1m, neg1);
  to_mag(k2, k2m, neg2);
}

}  // namespace glv
}  // namespace csb
