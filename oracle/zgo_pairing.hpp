// ORACLE — test infrastructure only (see zgo_field.hpp).
// A bilinear, non-degenerate pairing on BN254 G1 x G2 for the verifier's
// equality checks e(a,b) == e(c,d) (crates/amt/src/verify_params.rs:198-211
// via ark-ec's Bn254 pairing). ark uses the optimal ate pairing; every
// non-degenerate pairing on these groups is a fixed power (coprime to r) of
// it, so equality tests give identical answers. The reduced Tate pairing is
// used here because it needs no twist Frobenius constants:
//   e(P, Q) = f_{r,P}(psi(Q))^((q^12 - 1) / r),  psi(x, y) = (x v, y v w)
// with Fq12 = Fq6[w]/(w^2 - v), Fq6 = Fq2[v]/(v^3 - (9+u)).
#pragma once
#include "zgo_curve.hpp"

namespace zgo {

static const u64 PAIRING_R[4] = {FrCfg::P[0], FrCfg::P[1], FrCfg::P[2], FrCfg::P[3]};
static const std::vector<u64> PAIRING_Q2 = {
    0x3b5458a2275d69b1ULL, 0xa602072d09eac101ULL, 0x4a50189c6d96cadcULL, 0x04689e957a1242c8ULL,
    0x26edfa5c34c6b38dULL, 0xb00b855116375606ULL, 0x599a6f7c0348d21cULL, 0x0925c4b8763cbf9cULL};
// (q^4 - q^2 + 1) / r
static const std::vector<u64> PAIRING_HARD = {
    0xe81bb482ccdf42b1ULL, 0x5abf5cc4f49c36d4ULL, 0xf1154e7e1da014fdULL, 0xdcc7b44c87cdbacfULL,
    0xaaa441e3954bcf8aULL, 0x6b887d56d5095f23ULL, 0x79581e16f3fd90c6ULL, 0x3b1b1355d189227dULL,
    0x4e529a5861876f6bULL, 0x6c0eb522d5b12278ULL, 0x331ec15183177fafULL, 0x01baaa710b0759adULL};

// line value c00 + c01 v + c11 v w
static inline Fq12 line_elem(const Fq& c00, const Fq2& c01, const Fq2& c11) {
  Fq12 l;
  l.c0 = {Fq2{c00, Fq::zero()}, c01, Fq2::zero()};
  l.c1 = {Fq2::zero(), c11, Fq2::zero()};
  return l;
}

static inline Fq12 miller_tate(const G1A& P, const G2A& Q) {
  if (P.inf || Q.inf) return Fq12::one();
  G1J T = G1J::from_affine(P);
  Fq12 f = Fq12::one();
  for (int i = 252; i >= 0; --i) {
    // tangent at T, scaled by 2 Y Z^3 (an Fq factor, removed by the final exponentiation)
    {
      const Fq &X = T.X, &Y = T.Y, &Z = T.Z;
      Fq X2 = X.sqr(), Z2 = Z.sqr();
      Fq c00 = X2 * X * Fq::from_u64(3) - Y.sqr().dbl();
      Fq2 c01 = Q.x * (-(X2 * Z2 * Fq::from_u64(3)));
      Fq2 c11 = Q.y * ((Y * Z2 * Z).dbl());
      f = f.sqr() * line_elem(c00, c01, c11);
      T = T.dbl();
    }
    if ((PAIRING_R[i / 64] >> (i % 64)) & 1) {
      const Fq &X = T.X, &Y = T.Y, &Z = T.Z;
      Fq Z2 = Z.sqr();
      Fq H = P.x * Z2 - X;
      Fq N = P.y * Z2 * Z - Y;
      if (H.is_zero()) {
        // vertical line (T = -P): its value lies in Fq6 and is killed by the
        // final exponentiation; T becomes infinity (only at the last bit).
        T = T.add_affine(P);
        continue;
      }
      Fq ZH = Z * H;
      Fq c00 = N * P.x - ZH * P.y;
      Fq2 c01 = Q.x * (-N);
      Fq2 c11 = Q.y * ZH;
      f = f * line_elem(c00, c01, c11);
      T = T.add_affine(P);
    }
  }
  return f;
}

static inline Fq12 final_exp(const Fq12& f) {
  Fq12 f1 = f.conj() * f.inverse();          // f^(q^6 - 1)
  Fq12 f2 = f1.pow_big(PAIRING_Q2) * f1;     // ^(q^2 + 1)
  return f2.pow_big(PAIRING_HARD);           // ^((q^4 - q^2 + 1)/r)
}

static inline Fq12 pairing(const G1A& P, const G2A& Q) { return final_exp(miller_tate(P, Q)); }

// e(a, b) == e(c, d)  <=>  e(a, b) * e(-c, d) == 1
static inline bool pairing_eq(const G1A& a, const G2A& b, const G1A& c, const G2A& d) {
  Fq12 m = miller_tate(a, b) * miller_tate(affine_neg(c), d);
  return final_exp(m) == Fq12::one();
}

}  // namespace zgo
