// curve.cuh -- BN254 G1 (over Fq) and G2 (over Fq2) point arithmetic on sm_100a.
//
// Accumulators use extended Jacobian "XYZZ" coordinates (x = X/ZZ, y = Y/ZZZ,
// ZZ^3 = ZZZ^2): a mixed addition costs 8M + 2S and needs no inversion, a full addition
// 12M + 2S, a doubling 6M + 3S (formulas from the Explicit-Formulas Database,
// add-2008-s / madd-2008-s / dbl-2008-s-1 for a = 0).  Infinity is ZZ = 0.
//
// Affine points in memory follow the reference layout (src/cuda/types.h ECP_JAC_INDIMS):
// G1 = X | Y (16 words), G2 = X.c0 | X.c1 | Y.c0 | Y.c1 (32 words), Montgomery form, with
// the reference's infinity encoding (0, 1_mont) (src/cuda/constants.cpp:264-292).
#pragma once
#include "field.cuh"

namespace csb {

template <class F>
struct Affine {
  F x, y;
};

template <class F>
struct XYZZ {
  F X, Y, ZZ, ZZZ;

  static CSB_DEV XYZZ inf() { return {F::zero(), F::one(), F::zero(), F::zero()}; }
  CSB_DEV bool is_inf() const { return ZZ.is_zero(); }
  static CSB_DEV XYZZ from_affine(const Affine<F>& a) { return {a.x, a.y, F::one(), F::one()}; }
};

// the reference's affine infinity: X == 0 and Y == 1 (Montgomery)
template <class F>
CSB_DEV bool affine_is_inf(const Affine<F>& a) {
  return a.x.is_zero() && a.y == F::one();
}

// dbl-2008-s-1 (a = 0)
template <class F>
CSB_DEV XYZZ<F> xyzz_dbl(const XYZZ<F>& p) {
  if (p.is_inf()) return p;
  {
    const F U = p.Y.dbl();
    const F V = U.sqr();
    const F W = U * V;
    const F S = p.X * V;
    const F X2 = p.X.sqr();
    const F M = X2.dbl() + X2;
    XYZZ<F> r;
    r.X = M.sqr() - S.dbl();
    r.Y = M * (S - r.X) - W * p.Y;
    r.ZZ = V * p.ZZ;
    r.ZZZ = W * p.ZZZ;
    return r;
  }
}

// mdbl-2008-s-1: double an affine point
template <class F>
CSB_DEV XYZZ<F> xyzz_mdbl(const Affine<F>& p) {
  const F U = p.y.dbl();
  const F V = U.sqr();
  const F W = U * V;
  const F S = p.x * V;
  const F X2 = p.x.sqr();
  const F M = X2.dbl() + X2;
  XYZZ<F> r;
  r.X = M.sqr() - S.dbl();
  r.Y = M * (S - r.X) - W * p.y;
  r.ZZ = V;
  r.ZZZ = W;
  return r;
}

// madd-2008-s: p (XYZZ) + q (affine, not infinity)
template <class F>
CSB_DEV XYZZ<F> xyzz_madd(const XYZZ<F>& p, const Affine<F>& q) {
  if (p.is_inf()) return XYZZ<F>::from_affine(q);
  {
    const F U2 = q.x * p.ZZ;
    const F S2 = q.y * p.ZZZ;
    const F P = U2 - p.X;
    const F R = S2 - p.Y;
    if (P.is_zero()) {
      if (R.is_zero()) return xyzz_mdbl(q);
      return XYZZ<F>::inf();
    }
    const F PP = P.sqr();
    const F PPP = P * PP;
    const F Q = p.X * PP;
    XYZZ<F> r;
    r.X = R.sqr() - PPP - Q.dbl();
    r.Y = R * (Q - r.X) - p.Y * PPP;
    r.ZZ = p.ZZ * PP;
    r.ZZZ = p.ZZZ * PPP;
    return r;
  }
}

// madd-2008-s over Fq with lazily reduced coordinates (values in [0, 2p), products without
// the final conditional subtraction): the G1 bucket accumulation's addition.  Inputs may be
// lazy; q canonical; callers canonicalise before storing (xyzz_canon).
CSB_DEV XYZZ<Fq> xyzz_madd_lazy(const XYZZ<Fq>& p, const Affine<Fq>& q) {
  if (p.ZZ.is_zero_lazy()) return XYZZ<Fq>::from_affine(q);
  const Fq U2 = Fq::mul_lazy(q.x, p.ZZ);
  const Fq S2 = Fq::mul_lazy(q.y, p.ZZZ);
  const Fq P = Fq::sub_lazy(U2, p.X);
  const Fq R = Fq::sub_lazy(S2, p.Y);
  if (P.is_zero_lazy()) {
    if (R.is_zero_lazy()) return xyzz_mdbl(q);
    return XYZZ<Fq>::inf();
  }
  const Fq PP = Fq::mul_lazy(P, P);
  const Fq PPP = Fq::mul_lazy(P, PP);
  const Fq Q = Fq::mul_lazy(p.X, PP);
  XYZZ<Fq> r;
  r.X = Fq::sub_lazy(Fq::sub_lazy(Fq::mul_lazy(R, R), PPP), Fq::add_lazy(Q, Q));
  r.Y = Fq::sub_lazy(Fq::mul_lazy(R, Fq::sub_lazy(Q, r.X)), Fq::mul_lazy(p.Y, PPP));
  r.ZZ = Fq::mul_lazy(p.ZZ, PP);
  r.ZZZ = Fq::mul_lazy(p.ZZZ, PPP);
  return r;
}
CSB_DEV XYZZ<Fq> xyzz_canon(const XYZZ<Fq>& p) { return {p.X.canon(), p.Y.canon(), p.ZZ.canon(), p.ZZZ.canon()}; }

// add-2008-s: p + q, both XYZZ
template <class F>
CSB_DEV XYZZ<F> xyzz_add(const XYZZ<F>& p, const XYZZ<F>& q) {
  if (p.is_inf()) return q;
  if (q.is_inf()) return p;
  {
    const F U1 = p.X * q.ZZ;
    const F U2 = q.X * p.ZZ;
    const F S1 = p.Y * q.ZZZ;
    const F S2 = q.Y * p.ZZZ;
    const F P = U2 - U1;
    const F R = S2 - S1;
    if (P.is_zero()) {
      if (R.is_zero()) return xyzz_dbl(p);
      return XYZZ<F>::inf();
    }
    const F PP = P.sqr();
    const F PPP = P * PP;
    const F Q = U1 * PP;
    XYZZ<F> r;
    r.X = R.sqr() - PPP - Q.dbl();
    r.Y = R * (Q - r.X) - S1 * PPP;
    r.ZZ = p.ZZ * q.ZZ * PP;
    r.ZZZ = p.ZZZ * q.ZZZ * PPP;
    return r;
  }
}

// Out-of-line copies for kernels whose cost is latency, not throughput (bucket-sum
// scans, window combination): one body per kernel instead of one per call site keeps
// code size and compile time in check, notably over Fq2.
template <class F>
__device__ __noinline__ XYZZ<F> xyzz_add_cold(const XYZZ<F> p, const XYZZ<F> q) { return xyzz_add(p, q); }
template <class F>
__device__ __noinline__ XYZZ<F> xyzz_dbl_cold(const XYZZ<F> p) { return xyzz_dbl(p); }

// ------------------------------------------------ quad-parallel point operations -----
// For chains that a point runs through alone (window Horner, scalar multiplication, the
// buckets of a small MSM): the lanes of an aligned group hold the same point and each
// computes part of the independent products of a dependency level, so a doubling costs 3
// product latencies instead of 9, an addition 4 instead of 14 and a mixed addition 4
// instead of 10.  A group is 4 lanes over Fq (a "quad": one product each) and 16 lanes over
// Fq2 (twelve of them one Fq product each of the level's four Karatsuba products).  The
// shuffles use the full warp mask, so every lane of the warp must call these together (the
// warp's groups may hold different points: the special cases -- infinity, equal or opposite
// points -- are selected after the general formula, never branched around it); every lane of
// a group returns the same result.  The names keep "quad" for the group.
template <class F> struct GroupLanes { static constexpr int value = 4; };
template <> struct GroupLanes<Fq2> { static constexpr int value = 16; };

template <int G, class T>
CSB_DEV T grp_bcast(const T& v, int src) {
  constexpr int TW = sizeof(T) / 4;
  T o;
  uint32_t* ow = reinterpret_cast<uint32_t*>(&o);
  const uint32_t* vw = reinterpret_cast<const uint32_t*>(&v);
#pragma unroll
  for (int w = 0; w < TW; w++) ow[w] = __shfl_sync(0xffffffffu, vw[w], src, G);
  return o;
}
template <class F>
CSB_DEV F quad_bcast(const F& v, int src) { return grp_bcast<4>(v, src); }

template <class F>
CSB_DEV F pick4(int k, const F& v0, const F& v1, const F& v2, const F& v3) {
  return k == 0 ? v0 : k == 1 ? v1 : k == 2 ? v2 : v3;
}

template <class F>
CSB_DEV XYZZ<F> xyzz_select(bool c, const XYZZ<F>& a, const XYZZ<F>& b) { return c ? a : b; }

// quad lane k computes a_k * b_k; every lane gets the four products
template <class F>
CSB_DEV void quad_mul4(const F& a0, const F& b0, const F& a1, const F& b1, const F& a2, const F& b2,
                       const F& a3, const F& b3, F& r0, F& r1, F& r2, F& r3) {
  const int k = threadIdx.x & 3;
  const F r = pick4(k, a0, a1, a2, a3) * pick4(k, b0, b1, b2, b3);
  r0 = quad_bcast(r, 0);
  r1 = quad_bcast(r, 1);
  r2 = quad_bcast(r, 2);
  r3 = quad_bcast(r, 3);
}
// Over Fq2, in groups of 16 lanes: lane l < 12 computes part l mod 3 of Karatsuba product
// l / 3 (a0 b0, a1 b1 or (a0 + a1)(b0 + b1), the Fq products Fq2's operator* forms), every lane
// gathers the twelve and forms the four products as operator* does: the same bits, one Fq
// product latency per level instead of three.
template <>
CSB_DEV void quad_mul4<Fq2>(const Fq2& a0, const Fq2& b0, const Fq2& a1, const Fq2& b1, const Fq2& a2,
                            const Fq2& b2, const Fq2& a3, const Fq2& b3, Fq2& r0, Fq2& r1, Fq2& r2, Fq2& r3) {
  const int l = threadIdx.x & 15;
  const int j = l < 12 ? l / 3 : 0, part = l < 12 ? l - 3 * j : 0;
  const Fq2 a = pick4(j, a0, a1, a2, a3), b = pick4(j, b0, b1, b2, b3);
  const Fq x = part == 0 ? a.c0 : (part == 1 ? a.c1 : a.c0 + a.c1);
  const Fq y = part == 0 ? b.c0 : (part == 1 ? b.c1 : b.c0 + b.c1);
  const Fq p = x * y;
  Fq2 r[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const Fq v0 = grp_bcast<16>(p, 3 * k), v1 = grp_bcast<16>(p, 3 * k + 1), s = grp_bcast<16>(p, 3 * k + 2);
    r[k] = Fq2{v0 - v1, s - v0 - v1};
  }
  r0 = r[0];
  r1 = r[1];
  r2 = r[2];
  r3 = r[3];
}

// dbl-2008-s-1, three levels of products
template <class F>
CSB_DEV XYZZ<F> xyzz_dbl_quad(const XYZZ<F>& p) {
  const F U = p.Y.dbl();
  F V, X2, W, S, MM, ZZ3, T1, T2, ZZZ3, unused;
  quad_mul4(U, U, p.X, p.X, U, U, p.X, p.X, V, X2, unused, unused);
  const F M = X2.dbl() + X2;
  quad_mul4(U, V, p.X, V, M, M, V, p.ZZ, W, S, MM, ZZ3);
  XYZZ<F> r;
  r.X = MM - S.dbl();
  quad_mul4(M, S - r.X, W, p.Y, W, p.ZZZ, W, p.ZZZ, T1, T2, ZZZ3, unused);
  r.Y = T1 - T2;
  r.ZZ = ZZ3;
  r.ZZZ = ZZZ3;
  return xyzz_select(p.is_inf(), p, r);
}

// add-2008-s, four levels of products
template <class F>
CSB_DEV XYZZ<F> xyzz_add_quad(const XYZZ<F>& p, const XYZZ<F>& q) {
  F U1, U2, S1, S2;
  quad_mul4(p.X, q.ZZ, q.X, p.ZZ, p.Y, q.ZZZ, q.Y, p.ZZZ, U1, U2, S1, S2);
  const F P = U2 - U1;
  const F R = S2 - S1;
  F PP, RR, Z2, Z3, PPP, Q, ZZ3, ZZZ3, T1, T2, unused;
  quad_mul4(P, P, R, R, p.ZZ, q.ZZ, p.ZZZ, q.ZZZ, PP, RR, Z2, Z3);
  quad_mul4(P, PP, U1, PP, Z2, PP, Z3, P, PPP, Q, ZZ3, unused);
  XYZZ<F> r;
  r.X = RR - PPP - Q.dbl();
  quad_mul4(R, Q - r.X, S1, PPP, Z3, PPP, Z3, PPP, T1, T2, ZZZ3, unused);
  r.Y = T1 - T2;
  r.ZZ = ZZ3;
  r.ZZZ = ZZZ3;
  if (P.is_zero() && !p.is_inf() && !q.is_inf())  // equal or opposite points (rare): no shuffles
    r = R.is_zero() ? xyzz_dbl(p) : XYZZ<F>::inf();
  return p.is_inf() ? q : (q.is_inf() ? p : r);
}

// madd-2008-s, four levels of products
template <class F>
CSB_DEV XYZZ<F> xyzz_madd_quad(const XYZZ<F>& p, const Affine<F>& q) {
  F U2, S2, PP, RR, PPP, Q, ZZ3, T1, T2, ZZZ3, unused;
  quad_mul4(q.x, p.ZZ, q.y, p.ZZZ, q.x, p.ZZ, q.y, p.ZZZ, U2, S2, unused, unused);
  const F P = U2 - p.X;
  const F R = S2 - p.Y;
  quad_mul4(P, P, R, R, P, P, R, R, PP, RR, unused, unused);
  quad_mul4(P, PP, p.X, PP, p.ZZ, PP, p.ZZ, PP, PPP, Q, ZZ3, unused);
  XYZZ<F> r;
  r.X = RR - PPP - Q.dbl();
  quad_mul4(R, Q - r.X, p.Y, PPP, p.ZZZ, PPP, p.ZZZ, PPP, T1, T2, ZZZ3, unused);
  r.Y = T1 - T2;
  r.ZZ = ZZ3;
  r.ZZZ = ZZZ3;
  if (P.is_zero() && !p.is_inf())  // equal or opposite points (rare): no shuffles
    r = R.is_zero() ? xyzz_mdbl(q) : XYZZ<F>::inf();
  return p.is_inf() ? XYZZ<F>::from_affine(q) : r;
}

template <class F>
CSB_DEV XYZZ<F> xyzz_neg(const XYZZ<F>& p) {
  XYZZ<F> r = p;
  r.Y = p.Y.neg();
  return r;
}

// XYZZ -> affine with the reference infinity encoding
template <class F>
CSB_DEV Affine<F> xyzz_to_affine(const XYZZ<F>& p) {
  if (p.is_inf()) return {F::zero(), F::one()};
  const F t = (p.ZZ * p.ZZZ).inv();   // 1 / (ZZ ZZZ)
  const F izz = t * p.ZZZ;            // 1 / ZZ
  const F izzz = t * p.ZZ;            // 1 / ZZZ
  return {p.X * izz, p.Y * izzz};
}

// ------------------------------------------------------------------ memory I/O -------
// 128-bit loads/stores of limbs; pointers must be 16-byte aligned.
CSB_DEV void ld_limbs8(uint32_t (&v)[8], const uint32_t* p) {
  const uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
  const uint4 b = __ldg(reinterpret_cast<const uint4*>(p) + 1);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
CSB_DEV void st_limbs8(uint32_t* p, const uint32_t (&v)[8]) {
  reinterpret_cast<uint4*>(p)[0] = make_uint4(v[0], v[1], v[2], v[3]);
  reinterpret_cast<uint4*>(p)[1] = make_uint4(v[4], v[5], v[6], v[7]);
}
template <class M>
CSB_DEV Fp<M> ld_fp(const uint32_t* p) { Fp<M> r; ld_limbs8(r.v, p); return r; }
template <class M>
CSB_DEV void st_fp(uint32_t* p, const Fp<M>& a) { st_limbs8(p, a.v); }

// number of 32-bit words of one coordinate
template <class F> struct FieldWords;
template <> struct FieldWords<Fq> { static constexpr int value = 8; };
template <> struct FieldWords<Fq2> { static constexpr int value = 16; };

CSB_DEV void ld_field(Fq& a, const uint32_t* p) { ld_limbs8(a.v, p); }
CSB_DEV void ld_field(Fq2& a, const uint32_t* p) { ld_limbs8(a.c0.v, p); ld_limbs8(a.c1.v, p + 8); }
CSB_DEV void st_field(uint32_t* p, const Fq& a) { st_limbs8(p, a.v); }
CSB_DEV void st_field(uint32_t* p, const Fq2& a) { st_limbs8(p, a.c0.v); st_limbs8(p + 8, a.c1.v); }

template <class F>
CSB_DEV Affine<F> ld_affine(const uint32_t* p) {
  constexpr int W = FieldWords<F>::value;
  Affine<F> a;
  ld_field(a.x, p);
  ld_field(a.y, p + W);
  return a;
}
template <class F>
CSB_DEV void st_affine(uint32_t* p, const Affine<F>& a) {
  constexpr int W = FieldWords<F>::value;
  st_field(p, a.x);
  st_field(p + W, a.y);
}
template <class F>
CSB_DEV XYZZ<F> ld_xyzz(const uint32_t* p) {
  constexpr int W = FieldWords<F>::value;
  XYZZ<F> a;
  ld_field(a.X, p); ld_field(a.Y, p + W); ld_field(a.ZZ, p + 2 * W); ld_field(a.ZZZ, p + 3 * W);
  return a;
}
template <class F>
CSB_DEV void st_xyzz(uint32_t* p, const XYZZ<F>& a) {
  constexpr int W = FieldWords<F>::value;
  st_field(p, a.X); st_field(p + W, a.Y); st_field(p + 2 * W, a.ZZ); st_field(p + 3 * W, a.ZZZ);
}

// Quad operations as calls over Fq2: one body per kernel instead of one per use, for kernels
// that chain many of them, whose inlined copies overflow the register file.
template <class F>
__device__ __noinline__ XYZZ<F> xyzz_add_quad_call(const XYZZ<F> p, const XYZZ<F> q) { return xyzz_add_quad(p, q); }
template <class F>
__device__ __noinline__ XYZZ<F> xyzz_dbl_quad_call(const XYZZ<F> p) { return xyzz_dbl_quad(p); }
template <class F>
CSB_DEV XYZZ<F> add_q(const XYZZ<F>& p, const XYZZ<F>& q) {
  if constexpr (FieldWords<F>::value == 16) return xyzz_add_quad_call(p, q);
  else return xyzz_add_quad(p, q);
}
template <class F>
CSB_DEV XYZZ<F> dbl_q(const XYZZ<F>& p) {
  if constexpr (FieldWords<F>::value == 16) return xyzz_dbl_quad_call(p);
  else return xyzz_dbl_quad(p);
}

}  // namespace csb
