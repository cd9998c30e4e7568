// BN254 G1 (y^2 = x^3 + 3 over Fq) for the MSM buckets.
// Accumulators use extended Jacobian "XYZZ" coordinates (x = X/ZZ, y = Y/ZZZ,
// ZZ^3 = ZZZ^2): mixed addition costs 8M + 2S, XYZZ + XYZZ 12M + 2S.
// Formulas: madd-2008-s, mdbl-2008-s, add-2008-s, dbl-2008-s-1 of the
// Explicit-Formulas Database (Bernstein-Lange), with the equal / opposite
// point cases routed to doubling / infinity. Infinity is ZZ == 0.
#pragma once
#include "zg_field.cuh"
#include "zg_field_f64.cuh"
#include "zg_field_w28.cuh"

namespace zg {

// Field products of the curve formulas go through out-of-line device
// functions: the formulas then compile to a few hundred instructions that stay
// in the instruction cache, instead of ten inlined ~300-instruction products
// per point addition (host builds inline them). Independent products are
// issued in pairs. Five interchangeable product kinds (same values):
//   MulImad   both products of a pair on the integer multiply-add pipe
//             (Fq::mul2, the two CIOS carry chains interleaved);
//   MulHybrid the first on the integer pipe (Fq::mul), the second on the FP64
//             pipe (f52::mont_mul): the MSM bucket loop saturates the integer
//             pipe with carry-chain IMADs, so this pair keeps both pipes busy;
//   MulF64    both on the FP64 pipe;
//   MulW28    both as 28-bit-limb products with 64-bit column sums
//             (w28::mont_mul: wide multiply-adds without carry flags, the
//             columns independent chains);
//   MulW28Hybrid the first as a 28-bit-limb product, the second on the FP64
//             pipe.
// The curve formulas are templates over the kind; one kernel uses one kind
// only (two product functions in one hot loop overflow the instruction
// cache). MulHybrid is the default; the MSM kernel comes in all three and the
// context's tuning picks one (on the B200 the hybrid pair is fastest).
struct FqPair {
  Fq a, b;
};
#if defined(__CUDA_ARCH__) && !defined(ZG_INLINE_FMUL)
static __device__ __noinline__ Fq fq_mul_ool(const Fq a, const Fq b) { return Fq::mul(a, b); }
static __device__ __noinline__ FqPair fq_mul2_imad_ool(const Fq a, const Fq b, const Fq c, const Fq d) {
  FqPair r;
  Fq::mul2(a, b, c, d, r.a, r.b);
  return r;
}
static __device__ __noinline__ FqPair fq_mul2_hybrid_ool(const Fq a, const Fq b, const Fq c, const Fq d) {
  FqPair r;
  r.a = Fq::mul(a, b);
  r.b = f52::mont_mul(c, d);
  return r;
}
static __device__ __noinline__ Fq fq_mul_f64_ool(const Fq a, const Fq b) { return f52::mont_mul(a, b); }
static __device__ __noinline__ Fq fq_mul_w28_ool(const Fq a, const Fq b) { return w28::mont_mul(a, b); }
static __device__ __noinline__ FqPair fq_mul2_w28_ool(const Fq a, const Fq b, const Fq c, const Fq d) {
  FqPair r;
  r.a = w28::mont_mul(a, b);
  r.b = w28::mont_mul(c, d);
  return r;
}
static __device__ __noinline__ FqPair fq_mul2_w28f64_ool(const Fq a, const Fq b, const Fq c, const Fq d) {
  FqPair r;
  r.a = w28::mont_mul(a, b);
  r.b = f52::mont_mul(c, d);
  return r;
}
static __device__ __noinline__ FqPair fq_mul2_f64_ool(const Fq a, const Fq b, const Fq c, const Fq d) {
  FqPair r;
  r.a = f52::mont_mul(a, b);
  r.b = f52::mont_mul(c, d);
  return r;
}
struct MulImad {
  static __device__ __forceinline__ Fq mul(const Fq& a, const Fq& b) { return fq_mul_ool(a, b); }
  static __device__ __forceinline__ FqPair mul2(const Fq& a, const Fq& b, const Fq& c, const Fq& d) {
    return fq_mul2_imad_ool(a, b, c, d);
  }
};
struct MulHybrid {
  static __device__ __forceinline__ Fq mul(const Fq& a, const Fq& b) { return fq_mul_ool(a, b); }
  static __device__ __forceinline__ FqPair mul2(const Fq& a, const Fq& b, const Fq& c, const Fq& d) {
    return fq_mul2_hybrid_ool(a, b, c, d);
  }
};
struct MulF64 {
  static __device__ __forceinline__ Fq mul(const Fq& a, const Fq& b) { return fq_mul_f64_ool(a, b); }
  static __device__ __forceinline__ FqPair mul2(const Fq& a, const Fq& b, const Fq& c, const Fq& d) {
    return fq_mul2_f64_ool(a, b, c, d);
  }
};
struct MulW28 {
  static __device__ __forceinline__ Fq mul(const Fq& a, const Fq& b) { return fq_mul_w28_ool(a, b); }
  static __device__ __forceinline__ FqPair mul2(const Fq& a, const Fq& b, const Fq& c, const Fq& d) {
    return fq_mul2_w28_ool(a, b, c, d);
  }
};
struct MulW28Hybrid {
  static __device__ __forceinline__ Fq mul(const Fq& a, const Fq& b) { return fq_mul_w28_ool(a, b); }
  static __device__ __forceinline__ FqPair mul2(const Fq& a, const Fq& b, const Fq& c, const Fq& d) {
    return fq_mul2_w28f64_ool(a, b, c, d);
  }
};
#else
// host builds: the same values through Fq::mul; three distinct types so that
// kernel templates keep one instance per kind in both compilation passes
struct MulHost {
  static ZG_HD Fq mul(const Fq& a, const Fq& b) { return Fq::mul(a, b); }
  static ZG_HD FqPair mul2(const Fq& a, const Fq& b, const Fq& c, const Fq& d) {
    FqPair r;
    Fq::mul2(a, b, c, d, r.a, r.b);
    return r;
  }
};
struct MulImad : MulHost {};
struct MulHybrid : MulHost {};
struct MulF64 : MulHost {};
struct MulW28 : MulHost {};
struct MulW28Hybrid : MulHost {};
#endif

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
  template <class M = MulHybrid>
  ZG_HD static XYZZ dbl_affine(const Fq& x, const Fq& y) {
    Fq U = y + y;
    FqPair vx = M::mul2(U, U, x, x);        // V = U^2, xx = x^2
    Fq Mv = vx.b + vx.b + vx.b;
    FqPair ws = M::mul2(U, vx.a, x, vx.a);  // W = U V, S = x V
    XYZZ r;
    r.X = M::mul(Mv, Mv) - (ws.b + ws.b);
    FqPair y3 = M::mul2(Mv, ws.b - r.X, ws.a, y);
    r.Y = y3.a - y3.b;
    r.ZZ = vx.a;
    r.ZZZ = ws.a;
    return r;
  }

  // dbl-2008-s-1 (a = 0)
  template <class M = MulHybrid>
  ZG_HD XYZZ dbl() const {
    if (is_inf()) return *this;
    Fq U = Y + Y;
    FqPair vx = M::mul2(U, U, X, X);        // V, XX
    Fq Mv = vx.b + vx.b + vx.b;
    FqPair ws = M::mul2(U, vx.a, X, vx.a);  // W, S
    FqPair mz = M::mul2(Mv, Mv, vx.a, ZZ);  // M^2, V ZZ
    XYZZ r;
    r.X = mz.a - (ws.b + ws.b);
    FqPair y3 = M::mul2(Mv, ws.b - r.X, ws.a, Y);
    r.Y = y3.a - y3.b;
    r.ZZ = mz.b;
    r.ZZZ = M::mul(ws.a, ZZZ);
    return r;
  }

  // this + (x2, y2) (madd-2008-s)
  template <class M = MulHybrid>
  ZG_HD void add_affine(const Fq& x2, const Fq& y2) {
    if (is_inf()) {
      X = x2; Y = y2; ZZ = Fq::one(); ZZZ = Fq::one();
      return;
    }
    FqPair us = M::mul2(x2, ZZ, y2, ZZZ);   // U2, S2
    Fq P = us.a - X;
    Fq R = us.b - Y;
    if (P.is_zero()) {
      if (R.is_zero()) *this = dbl_affine<M>(x2, y2);
      else *this = inf();
      return;
    }
    FqPair pr = M::mul2(P, P, R, R);        // PP, R^2
    FqPair pq = M::mul2(P, pr.a, X, pr.a);  // PPP, Q
    FqPair zz = M::mul2(ZZ, pr.a, ZZZ, pq.a);
    Fq X3 = pr.b - pq.a - (pq.b + pq.b);
    FqPair y3 = M::mul2(R, pq.b - X3, Y, pq.a);
    X = X3;
    Y = y3.a - y3.b;
    ZZ = zz.a;
    ZZZ = zz.b;
  }

  // this + o (add-2008-s)
  template <class M = MulHybrid>
  ZG_HD void add(const XYZZ& o) {
    if (o.is_inf()) return;
    if (is_inf()) { *this = o; return; }
    FqPair u = M::mul2(X, o.ZZ, o.X, ZZ);     // U1, U2
    FqPair sv = M::mul2(Y, o.ZZZ, o.Y, ZZZ);  // S1, S2
    Fq P = u.b - u.a;
    Fq R = sv.b - sv.a;
    if (P.is_zero()) {
      if (R.is_zero()) *this = dbl<M>();
      else *this = inf();
      return;
    }
    FqPair pr = M::mul2(P, P, R, R);          // PP, R^2
    FqPair pq = M::mul2(P, pr.a, u.a, pr.a);  // PPP, Q
    FqPair zt = M::mul2(ZZ, o.ZZ, ZZZ, o.ZZZ);
    Fq X3 = pr.b - pq.a - (pq.b + pq.b);
    FqPair y3 = M::mul2(R, pq.b - X3, sv.a, pq.a);
    FqPair zz = M::mul2(zt.a, pr.a, zt.b, pq.a);
    X = X3;
    Y = y3.a - y3.b;
    ZZ = zz.a;
    ZZZ = zz.b;
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
