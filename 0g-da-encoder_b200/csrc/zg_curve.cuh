// BN254 G1 (y^2 = x^3 + 3 over Fq) for the MSM buckets.
// Accumulators use extended Jacobian "XYZZ" coordinates (x = X/ZZ, y = Y/ZZZ,
// ZZ^3 = ZZZ^2): mixed addition costs 8M + 2S, XYZZ + XYZZ 12M + 2S.
// Formulas: madd-2008-s, mdbl-2008-s, add-2008-s, dbl-2008-s-1 of the
// Explicit-Formulas Database (Bernstein-Lange), with the equal / opposite
// point cases routed to doubling / infinity. Infinity is ZZ == 0.
#pragma once
#include "zg_field.cuh"

namespace zg {

struct G1Aff {
  Fq x, y;
};

struct XYZZ {
  Fq X, Y, ZZ, ZZZ;

  ZG_HD static XYZZ inf() {
    XYZZ r;
    r.X = Fq::one(); r.Y = Fq::one(); r.ZZ = Fq::zero(); r.ZZZ = Fq::zero();
    return r;
  }
  ZG_HD bool is_inf() const { return ZZ.is_zero(); }
  ZG_HD static XYZZ from_affine(const G1Aff& a) {
    XYZZ r;
    r.X = a.x; r.Y = a.y; r.ZZ = Fq::one(); r.ZZZ = Fq::one();
    return r;
  }

  // 2 * (x, y) for an affine point (mdbl-2008-s)
  ZG_HD static XYZZ dbl_affine(const Fq& x, const Fq& y) {
    Fq U = y + y;
    Fq V = U.sqr();
    Fq W = U * V;
    Fq S = x * V;
    Fq xx = x.sqr();
    Fq M = xx + xx + xx;
    XYZZ r;
    r.X = M.sqr() - (S + S);
    r.Y = M * (S - r.X) - W * y;
    r.ZZ = V;
    r.ZZZ = W;
    return r;
  }

  // dbl-2008-s-1 (a = 0)
  ZG_HD XYZZ dbl() const {
    if (is_inf()) return *this;
    Fq U = Y + Y;
    Fq V = U.sqr();
    Fq W = U * V;
    Fq S = X * V;
    Fq xx = X.sqr();
    Fq M = xx + xx + xx;
    XYZZ r;
    r.X = M.sqr() - (S + S);
    r.Y = M * (S - r.X) - W * Y;
    r.ZZ = V * ZZ;
    r.ZZZ = W * ZZZ;
    return r;
  }

  // this + (x2, y2) (madd-2008-s)
  ZG_HD void add_affine(const Fq& x2, const Fq& y2) {
    if (is_inf()) {
      X = x2; Y = y2; ZZ = Fq::one(); ZZZ = Fq::one();
      return;
    }
    Fq U2 = x2 * ZZ;
    Fq S2 = y2 * ZZZ;
    Fq P = U2 - X;
    Fq R = S2 - Y;
    if (P.is_zero()) {
      if (R.is_zero()) *this = dbl_affine(x2, y2);
      else *this = inf();
      return;
    }
    Fq PP = P.sqr();
    Fq PPP = P * PP;
    Fq Q = X * PP;
    Fq X3 = R.sqr() - PPP - (Q + Q);
    Fq Y3 = R * (Q - X3) - Y * PPP;
    ZZ = ZZ * PP;
    ZZZ = ZZZ * PPP;
    X = X3;
    Y = Y3;
  }

  // this + o (add-2008-s)
  ZG_HD void add(const XYZZ& o) {
    if (o.is_inf()) return;
    if (is_inf()) { *this = o; return; }
    Fq U1 = X * o.ZZ;
    Fq U2 = o.X * ZZ;
    Fq S1 = Y * o.ZZZ;
    Fq S2 = o.Y * ZZZ;
    Fq P = U2 - U1;
    Fq R = S2 - S1;
    if (P.is_zero()) {
      if (R.is_zero()) *this = dbl();
      else *this = inf();
      return;
    }
    Fq PP = P.sqr();
    Fq PPP = P * PP;
    Fq Q = U1 * PP;
    Fq X3 = R.sqr() - PPP - (Q + Q);
    Fq Y3 = R * (Q - X3) - S1 * PPP;
    ZZ = ZZ * o.ZZ * PP;
    ZZZ = ZZZ * o.ZZZ * PPP;
    X = X3;
    Y = Y3;
  }

  ZG_HD XYZZ neg() const {
    XYZZ r = *this;
    r.Y = -Y;
    return r;
  }

  // affine coordinates (Montgomery form); returns false for infinity
  ZG_HD bool to_affine(G1Aff& out) const {
    if (is_inf()) return false;
    Fq izzz = ZZZ.inverse();
    Fq izz = ZZ.sqr() * izzz.sqr();  // ZZ^2 / ZZZ^2 = 1 / ZZ
    out.x = X * izz;
    out.y = Y * izzz;
    return true;
  }
};

// ark-serialize 0.4 uncompressed G1 (x || y canonical little-endian, y's top
// byte carries SWFlags: bit 7 = y > -y, bit 6 = infinity), the layout of
// every G1 field of the reference's EncodedSlice
// (crates/encoder/src/encoder/slice.rs:15-20, derive(CanonicalSerialize)).
ZG_HD void g1_serialize(const XYZZ& p, uint8_t out[64]) {
  G1Aff a;
  if (!p.to_affine(a)) {
    for (int i = 0; i < 64; ++i) out[i] = 0;
    out[63] = 0x40;
    return;
  }
  Fq x = a.x.to_canonical(), y = a.y.to_canonical();
  for (int i = 0; i < 8; ++i) {
    for (int k = 0; k < 4; ++k) {
      out[4 * i + k] = (uint8_t)(x.v[i] >> (8 * k));
      out[32 + 4 * i + k] = (uint8_t)(y.v[i] >> (8 * k));
    }
  }
  if (a.y.canonical_is_negative()) out[63] |= 0x80;
}

}  // namespace zg
