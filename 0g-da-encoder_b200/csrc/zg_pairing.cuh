// BN254 pairing arithmetic for batched slice verification (host and device).
//
// The reference verifies AMT proofs with pairing equalities
// e(a, b) == e(c, d) (crates/amt/src/verify_params.rs:136-211), batched by
// its DeferredVerifier into random linear combinations
// (crates/amt/src/deferred_verification.rs:67-146). Only the answer of such
// an equality test matters, and every non-degenerate bilinear pairing on
// G1 x G2 is a fixed power (coprime to r) of ark's optimal ate pairing, so it
// gives the same answers. This file uses the reduced Tate pairing
//   e(P, Q) = f_{r,P}(psi(Q))^((q^12 - 1) / r)
// because its Miller loop iterates a G1 point (cheap Fq arithmetic, one
// independent loop per GPU thread) and needs no twist Frobenius constants.
// Tower: Fq2 = Fq[u]/(u^2 + 1), Fq6 = Fq2[v]/(v^3 - xi) with xi = 9 + u,
// Fq12 = Fq6[w]/(w^2 - v). G2 lives on the D-type twist y^2 = x^3 + 3/xi
// over Fq2 and psi(x, y) = (x v, y v w) maps it into E(Fq12).
// Line values carry factors in Fq (and a vertical line a factor in Fq6); the
// final exponentiation sends both to 1.
#pragma once
#include "zg_curve.cuh"

namespace zg {

// Fq products of the tower go through the out-of-line device product: the
// Miller loop then stays a few thousand instructions long (inlined, a 253-step
// loop over Fq12 arithmetic is hundreds of thousands of instructions).
ZG_HD Fq zp_mul(const Fq& a, const Fq& b) {
#if defined(__CUDA_ARCH__) && !defined(ZG_INLINE_FMUL)
  return fq_mul_ool(a, b);
#else
  return Fq::mul(a, b);
#endif
}

struct Fq2 {
  Fq c0, c1;
  ZG_HD static Fq2 zero() { return Fq2{Fq::zero(), Fq::zero()}; }
  ZG_HD static Fq2 one() { return Fq2{Fq::one(), Fq::zero()}; }
  ZG_HD bool is_zero() const { return c0.is_zero() && c1.is_zero(); }
  ZG_HD bool operator==(const Fq2& o) const { return c0 == o.c0 && c1 == o.c1; }
  ZG_HD Fq2 operator+(const Fq2& o) const { return Fq2{c0 + o.c0, c1 + o.c1}; }
  ZG_HD Fq2 operator-(const Fq2& o) const { return Fq2{c0 - o.c0, c1 - o.c1}; }
  ZG_HD Fq2 operator-() const { return Fq2{-c0, -c1}; }
  ZG_HD Fq2 dbl() const { return Fq2{c0 + c0, c1 + c1}; }
  // (a0 + a1 u)(b0 + b1 u), three products
  ZG_HD Fq2 operator*(const Fq2& o) const {
    const Fq a = zp_mul(c0, o.c0), b = zp_mul(c1, o.c1);
    const Fq s = zp_mul(c0 + c1, o.c0 + o.c1);
    return Fq2{a - b, s - a - b};
  }
  ZG_HD Fq2 mul_fq(const Fq& k) const { return Fq2{zp_mul(c0, k), zp_mul(c1, k)}; }
  ZG_HD Fq2 sqr() const {
    const Fq m = zp_mul(c0, c1);
    return Fq2{zp_mul(c0 + c1, c0 - c1), m + m};
  }
  // (9 + u)(a0 + a1 u) = (9 a0 - a1) + (a0 + 9 a1) u, by additions
  ZG_HD Fq2 mul_xi() const {
    Fq e0 = c0 + c0, e1 = c1 + c1;
    e0 = e0 + e0;
    e1 = e1 + e1;
    e0 = e0 + e0 + c0;  // 9 a0
    e1 = e1 + e1 + c1;  // 9 a1
    return Fq2{e0 - c1, c0 + e1};
  }
  ZG_HD Fq2 inverse() const {
    const Fq n = zp_mul(c0, c0) + zp_mul(c1, c1);
    const Fq ni = n.inverse();
    return Fq2{zp_mul(c0, ni), -zp_mul(c1, ni)};
  }
};

struct Fq6 {
  Fq2 c0, c1, c2;
  ZG_HD static Fq6 zero() { return Fq6{Fq2::zero(), Fq2::zero(), Fq2::zero()}; }
  ZG_HD static Fq6 one() { return Fq6{Fq2::one(), Fq2::zero(), Fq2::zero()}; }
  ZG_HD bool operator==(const Fq6& o) const { return c0 == o.c0 && c1 == o.c1 && c2 == o.c2; }
  ZG_HD Fq6 operator+(const Fq6& o) const { return Fq6{c0 + o.c0, c1 + o.c1, c2 + o.c2}; }
  ZG_HD Fq6 operator-(const Fq6& o) const { return Fq6{c0 - o.c0, c1 - o.c1, c2 - o.c2}; }
  ZG_HD Fq6 operator-() const { return Fq6{-c0, -c1, -c2}; }
  // Karatsuba over Fq2: six products
  ZG_HD Fq6 operator*(const Fq6& o) const {
    const Fq2 a = c0 * o.c0, b = c1 * o.c1, c = c2 * o.c2;
    const Fq2 t0 = ((c1 + c2) * (o.c1 + o.c2) - b - c).mul_xi() + a;
    const Fq2 t1 = (c0 + c1) * (o.c0 + o.c1) - a - b + c.mul_xi();
    const Fq2 t2 = (c0 + c2) * (o.c0 + o.c2) - a - c + b;
    return Fq6{t0, t1, t2};
  }
  // v * (c0 + c1 v + c2 v^2) = xi c2 + c0 v + c1 v^2
  ZG_HD Fq6 mul_v() const { return Fq6{c2.mul_xi(), c0, c1}; }
  // times (a + b v), a in Fq, b in Fq2
  ZG_HD Fq6 mul_ab(const Fq& a, const Fq2& b) const {
    return Fq6{c0.mul_fq(a) + (c2 * b).mul_xi(), c0 * b + c1.mul_fq(a), c1 * b + c2.mul_fq(a)};
  }
  // times (b v), b in Fq2
  ZG_HD Fq6 mul_bv(const Fq2& b) const { return Fq6{(c2 * b).mul_xi(), c0 * b, c1 * b}; }
  ZG_HD Fq6 inverse() const {
    const Fq2 A = c0.sqr() - (c1 * c2).mul_xi();
    const Fq2 B = c2.sqr().mul_xi() - c0 * c1;
    const Fq2 C = c1.sqr() - c0 * c2;
    const Fq2 F = (c2 * B + c1 * C).mul_xi() + c0 * A;
    const Fq2 Fi = F.inverse();
    return Fq6{A * Fi, B * Fi, C * Fi};
  }
};

struct Fq12 {
  Fq6 c0, c1;
  ZG_HD static Fq12 one() { return Fq12{Fq6::one(), Fq6::zero()}; }
  ZG_HD bool operator==(const Fq12& o) const { return c0 == o.c0 && c1 == o.c1; }
  ZG_HD bool is_one() const { return *this == one(); }
  ZG_HD Fq12 operator*(const Fq12& o) const;
  ZG_HD Fq12 sqr() const;
  ZG_HD Fq12 conj() const { return Fq12{c0, -c1}; }
  ZG_HD Fq12 inverse() const {
    const Fq6 t = (c0 * c0 - (c1 * c1).mul_v()).inverse();
    return Fq12{c0 * t, -(c1 * t)};
  }
  ZG_HD Fq12 mul_line(const Fq& c00, const Fq2& c01, const Fq2& c11) const;
  // this^e, e little-endian 32-bit words
  ZG_HD Fq12 pow_words(const uint32_t* e, int n) const {
    Fq12 r = one();
    bool started = false;
    for (int i = n - 1; i >= 0; --i)
      for (int k = 31; k >= 0; --k) {
        if (started) r = r.sqr();
        if ((e[i] >> k) & 1) {
          r = started ? r * (*this) : *this;
          started = true;
        }
      }
    return r;
  }
};

// Fq12 product, square and sparse line product, out of line
__host__ __device__ __noinline__ Fq12 fq12_mul(const Fq12 x, const Fq12 o) {
  const Fq6 a = x.c0 * o.c0, b = x.c1 * o.c1;
  const Fq6 s = (x.c0 + x.c1) * (o.c0 + o.c1);
  return Fq12{a + b.mul_v(), s - a - b};
}
// (c0 + c1 w)^2 = (c0^2 + v c1^2) + 2 c0 c1 w, with two Fq6 products:
// c0^2 + v c1^2 = (c0 + c1)(c0 + v c1) - c0 c1 - v c0 c1
__host__ __device__ __noinline__ Fq12 fq12_sqr(const Fq12 x) {
  const Fq6 m = x.c0 * x.c1;
  const Fq6 s = (x.c0 + x.c1) * (x.c0 + x.c1.mul_v());
  return Fq12{s - m - m.mul_v(), m + m};
}
// times the line value c00 + c01 v + c11 v w (c00 in Fq; c01, c11 in Fq2):
// (f0 + f1 w)(L0 + L1 w) with L0 = c00 + c01 v, L1 = c11 v, w^2 = v
__host__ __device__ __noinline__ Fq12 fq12_mul_line(const Fq12 x, const Fq c00, const Fq2 c01, const Fq2 c11) {
  const Fq6 a = x.c0.mul_ab(c00, c01), b = x.c1.mul_bv(c11);
  const Fq6 e = x.c0.mul_bv(c11) + x.c1.mul_ab(c00, c01);
  return Fq12{a + b.mul_v(), e};
}
ZG_HD Fq12 Fq12::operator*(const Fq12& o) const { return fq12_mul(*this, o); }
ZG_HD Fq12 Fq12::sqr() const { return fq12_sqr(*this); }
ZG_HD Fq12 Fq12::mul_line(const Fq& c00, const Fq2& c01, const Fq2& c11) const {
  return fq12_mul_line(*this, c00, c01, c11);
}

struct G2Aff {
  Fq2 x, y;
  uint32_t inf;
};

// Jacobian G2 point on the twist (x = X/Z^2, y = Y/Z^3), a = 0
struct G2Jac {
  Fq2 X, Y, Z;
  ZG_HD static G2Jac inf() { return G2Jac{Fq2::one(), Fq2::one(), Fq2::zero()}; }
  ZG_HD bool is_inf() const { return Z.is_zero(); }
  ZG_HD G2Jac dbl() const {
    if (is_inf()) return *this;
    const Fq2 A = X.sqr(), B = Y.sqr(), C = B.sqr();
    const Fq2 D = ((X + B).sqr() - A - C).dbl();
    const Fq2 E = A.dbl() + A, F = E.sqr();
    G2Jac r;
    r.X = F - D.dbl();
    const Fq2 C8 = C.dbl().dbl().dbl();
    r.Y = E * (D - r.X) - C8;
    r.Z = (Y * Z).dbl();
    return r;
  }
  // this + (x, y), affine operand not at infinity
  ZG_HD G2Jac add_affine(const Fq2& x, const Fq2& y) const {
    if (is_inf()) return G2Jac{x, y, Fq2::one()};
    const Fq2 Z1Z1 = Z.sqr();
    const Fq2 U2 = x * Z1Z1, S2 = y * Z * Z1Z1;
    const Fq2 H = U2 - X, Rr = S2 - Y;
    if (H.is_zero()) {
      if (Rr.is_zero()) return dbl();
      return inf();
    }
    const Fq2 HH = H.sqr(), HHH = H * HH, V = X * HH;
    G2Jac r;
    r.X = Rr.sqr() - HHH - V.dbl();
    r.Y = Rr * (V - r.X) - Y * HHH;
    r.Z = Z * H;
    return r;
  }
  ZG_HD G2Aff to_affine() const {
    G2Aff a;
    if (is_inf()) {
      a.x = Fq2::zero();
      a.y = Fq2::zero();
      a.inf = 1;
      return a;
    }
    const Fq2 zi = Z.inverse(), zi2 = zi.sqr();
    a.x = X * zi2;
    a.y = Y * zi2 * zi;
    a.inf = 0;
    return a;
  }
};

// the standard BN254 G2 generator (Montgomery form), the `g2` of every
// reference param file
ZG_HD G2Aff g2_generator() {
  // x.c0, x.c1, y.c0, y.c1 of the generator times 2^256 mod q
  const uint32_t w[4][8] = {
      {0x02bc2026u, 0x8e83b5d1u, 0x497b0172u, 0xdceb1935u, 0x97811adfu, 0xfbb82647u, 0xaf96503bu, 0x19573841u},
      {0xa84c6140u, 0xafb4737du, 0x5802d8c4u, 0x6043dd5au, 0x52a02f86u, 0x09e950fcu, 0x3aea7b6bu, 0x14fef083u},
      {0x886be9f6u, 0x619dfa9du, 0xf59e9b78u, 0xfe7fd297u, 0x231b7dfeu, 0xff9e1a62u, 0xae9e4206u, 0x28fd7eebu},
      {0xc71856eeu, 0x64095b56u, 0x327d3cbbu, 0xdc57f922u, 0x33351076u, 0x55f935beu, 0x93fd6482u, 0x0da4a0e6u}};
  G2Aff g;
  Fq t[4];
  for (int k = 0; k < 4; ++k) {
    for (int i = 0; i < 8; ++i) t[k].v[i] = w[k][i];
  }
  g.x = Fq2{t[0], t[1]};
  g.y = Fq2{t[2], t[3]};
  g.inf = 0;
  return g;
}

// Miller function f_{r,P}(psi(Q)) (up to factors the final exponentiation
// removes); P in G1 affine (Montgomery), Q on the twist.
ZG_HD Fq12 miller_tate(const G1Aff& P, bool p_inf, const G2Aff& Q) {
  Fq12 f = Fq12::one();
  if (p_inf || Q.inf) return f;
  // r = FrCfg modulus; bits 252..0 after the leading one
  const uint32_t r[8] = {FrCfg::p0, FrCfg::p1, FrCfg::p2, FrCfg::p3, FrCfg::p4, FrCfg::p5, FrCfg::p6, FrCfg::p7};
  Fq X = P.x, Y = P.y, Z = Fq::one();
  bool t_inf = false;
  for (int i = 252; i >= 0; --i) {
    // tangent at T, times 2 Y Z^3: (3X^3 - 2Y^2) - 3X^2 Z^2 x' v + 2Y Z^3 y' v w
    {
      const Fq A = zp_mul(X, X), B = zp_mul(Y, Y), C = zp_mul(B, B), Z2 = zp_mul(Z, Z);
      const Fq E = A + A + A;
      const Fq c00 = zp_mul(X, E) - (B + B);
      const Fq2 c01 = Q.x.mul_fq(-zp_mul(E, Z2));
      const Fq YZ = zp_mul(Y, Z);
      const Fq Z3 = YZ + YZ;
      const Fq2 c11 = Q.y.mul_fq(zp_mul(Z3, Z2));
      f = f.sqr().mul_line(c00, c01, c11);
      const Fq XB = X + B;
      const Fq D0 = zp_mul(XB, XB) - A - C;
      const Fq D = D0 + D0;
      const Fq F = zp_mul(E, E);
      const Fq X3 = F - (D + D);
      Fq C8 = C + C;
      C8 = C8 + C8;
      C8 = C8 + C8;
      Y = zp_mul(E, D - X3) - C8;
      X = X3;
      Z = Z3;
    }
    if ((r[i >> 5] >> (i & 31)) & 1) {
      // chord through T and P, times Z H: (N xP - Z H yP) - N x' v + Z H y' v w
      const Fq Z2 = zp_mul(Z, Z);
      const Fq H = zp_mul(P.x, Z2) - X;
      const Fq N = zp_mul(zp_mul(P.y, Z2), Z) - Y;
      if (H.is_zero()) {
        // T = -P (only at the last bit): the vertical line lies in Fq6
        t_inf = true;
        continue;
      }
      const Fq ZH = zp_mul(Z, H);
      f = f.mul_line(zp_mul(N, P.x) - zp_mul(ZH, P.y), Q.x.mul_fq(-N), Q.y.mul_fq(ZH));
      const Fq HH = zp_mul(H, H), HHH = zp_mul(H, HH), V = zp_mul(X, HH);
      const Fq X3 = zp_mul(N, N) - HHH - (V + V);
      Y = zp_mul(N, V - X3) - zp_mul(Y, HHH);
      X = X3;
      Z = ZH;
    }
  }
  (void)t_inf;
  return f;
}

// f^((q^12 - 1) / r) = ((f^(q^6 - 1))^(q^2 + 1))^((q^4 - q^2 + 1) / r)
ZG_HD Fq12 final_exp(const Fq12& f) {
  const uint32_t q2[16] = {0x275d69b1u, 0x3b5458a2u, 0x09eac101u, 0xa602072du, 0x6d96cadcu, 0x4a50189cu,
                           0x7a1242c8u, 0x04689e95u, 0x34c6b38du, 0x26edfa5cu, 0x16375606u, 0xb00b8551u,
                           0x0348d21cu, 0x599a6f7cu, 0x763cbf9cu, 0x0925c4b8u};
  const uint32_t hard[24] = {0xccdf42b1u, 0xe81bb482u, 0xf49c36d4u, 0x5abf5cc4u, 0x1da014fdu, 0xf1154e7eu,
                             0x87cdbacfu, 0xdcc7b44cu, 0x954bcf8au, 0xaaa441e3u, 0xd5095f23u, 0x6b887d56u,
                             0xf3fd90c6u, 0x79581e16u, 0xd189227du, 0x3b1b1355u, 0x61876f6bu, 0x4e529a58u,
                             0xd5b12278u, 0x6c0eb522u, 0x83177fafu, 0x331ec151u, 0x0b0759adu, 0x01baaa71u};
  const Fq12 f1 = f.conj() * f.inverse();
  const Fq12 f2 = f1.pow_words(q2, 16) * f1;
  return f2.pow_words(hard, 24);
}

}  // namespace zg
