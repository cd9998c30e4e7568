// ORACLE — test infrastructure only (see zgo_field.hpp).
// BN254 G1 (over Fq, y^2 = x^3 + 3) and G2 (over Fq2, y^2 = x^3 + 3/(9+u)),
// the groups of ark-bn254 0.4.0 (Cargo.lock:170) used by the reference for
// commitments/proofs (crates/amt/src/ec_algebra.rs:25-33).
#pragma once
#include "zgo_field.hpp"

namespace zgo {

template <class F>
struct Affine {
  F x, y;
  bool inf;
  bool operator==(const Affine& o) const {
    if (inf || o.inf) return inf == o.inf;
    return x == o.x && y == o.y;
  }
  bool operator!=(const Affine& o) const { return !(*this == o); }
};

template <class F>
struct Jac {  // (X/Z^2, Y/Z^3); Z == 0 is infinity
  F X, Y, Z;
  static Jac inf() { return {F::one(), F::one(), F::zero()}; }
  bool is_inf() const { return Z.is_zero(); }
  static Jac from_affine(const Affine<F>& a) {
    if (a.inf) return inf();
    return {a.x, a.y, F::one()};
  }
  Jac dbl() const {  // a = 0 (dbl-2009-l)
    if (is_inf()) return *this;
    F A = X.sqr(), B = Y.sqr(), C = B.sqr();
    F D = ((X + B).sqr() - A - C).dbl();
    F E = A.dbl() + A;
    F Fv = E.sqr();
    F X3 = Fv - D.dbl();
    F C8 = C.dbl().dbl().dbl();
    F Y3 = E * (D - X3) - C8;
    F Z3 = (Y * Z).dbl();
    return {X3, Y3, Z3};
  }
  Jac add(const Jac& o) const {  // add-2007-bl with explicit special cases
    if (is_inf()) return o;
    if (o.is_inf()) return *this;
    F Z1Z1 = Z.sqr(), Z2Z2 = o.Z.sqr();
    F U1 = X * Z2Z2, U2 = o.X * Z1Z1;
    F S1 = Y * o.Z * Z2Z2, S2 = o.Y * Z * Z1Z1;
    if (U1 == U2) {
      if (S1 == S2) return dbl();
      return inf();
    }
    F H = U2 - U1;
    F I = H.dbl().sqr();
    F J = H * I;
    F r = (S2 - S1).dbl();
    F V = U1 * I;
    F X3 = r.sqr() - J - V.dbl();
    F Y3 = r * (V - X3) - (S1 * J).dbl();
    F Z3 = ((Z + o.Z).sqr() - Z1Z1 - Z2Z2) * H;
    return {X3, Y3, Z3};
  }
  Jac add_affine(const Affine<F>& a) const { return add(from_affine(a)); }
  Jac neg() const { return {X, -Y, Z}; }
  Affine<F> to_affine() const {
    if (is_inf()) return {F::zero(), F::zero(), true};
    F zi = Z.inverse();
    F zi2 = zi.sqr();
    return {X * zi2, Y * zi2 * zi, false};
  }
  bool eq(const Jac& o) const {
    if (is_inf() || o.is_inf()) return is_inf() == o.is_inf();
    F Z1Z1 = Z.sqr(), Z2Z2 = o.Z.sqr();
    return X * Z2Z2 == o.X * Z1Z1 && Y * o.Z * Z2Z2 == o.Y * Z * Z1Z1;
  }
  // scalar multiplication by a canonical 256-bit integer
  Jac mul(const BigInt& k) const {
    Jac r = inf();
    for (int i = 255; i >= 0; --i) {
      r = r.dbl();
      if ((k.v[i / 64] >> (i % 64)) & 1) r = r.add(*this);
    }
    return r;
  }
};

template <class F>
static inline Affine<F> affine_neg(const Affine<F>& a) {
  if (a.inf) return a;
  return {a.x, -a.y, false};
}

// batch normalization (CurveGroup::normalize_batch) via Montgomery's trick
template <class F>
static void normalize_batch(const Jac<F>* in, Affine<F>* out, size_t n) {
  std::vector<F> prod(n);
  F acc = F::one();
  for (size_t i = 0; i < n; ++i) {
    prod[i] = acc;
    if (!in[i].is_inf()) acc = acc * in[i].Z;
  }
  F inv = acc.inverse();
  for (size_t i = n; i-- > 0;) {
    if (in[i].is_inf()) { out[i] = {F::zero(), F::zero(), true}; continue; }
    F zi = inv * prod[i];
    inv = inv * in[i].Z;
    F zi2 = zi.sqr();
    out[i] = {in[i].X * zi2, in[i].Y * zi2 * zi, false};
  }
}

typedef Affine<Fq> G1A;
typedef Jac<Fq> G1J;
typedef Affine<Fq2> G2A;
typedef Jac<Fq2> G2J;

static inline G1A g1_generator() {
  return {Fq::from_u64(1), Fq::from_u64(2), false};
}
static inline G2A g2_generator() {
  // ark-bn254 0.4.0 g2::G2_GENERATOR_X / _Y (the EIP-197 generator)
  static const BigInt xc0 = {{0x46debd5cd992f6edULL, 0x674322d4f75edaddULL,
                              0x426a00665e5c4479ULL, 0x1800deef121f1e76ULL}};
  static const BigInt xc1 = {{0x97e485b7aef312c2ULL, 0xf1aa493335a9e712ULL,
                              0x7260bfb731fb5d25ULL, 0x198e9393920d483aULL}};
  static const BigInt yc0 = {{0x4ce6cc0166fa7daaULL, 0xe3d1e7690c43d37bULL,
                              0x4aab71808dcb408fULL, 0x12c85ea5db8c6debULL}};
  static const BigInt yc1 = {{0x55acdadcd122975bULL, 0xbc4b313370b38ef3ULL,
                              0xec9e99ad690c3395ULL, 0x090689d0585ff075ULL}};
  return {{Fq::from_bigint(xc0), Fq::from_bigint(xc1)},
          {Fq::from_bigint(yc0), Fq::from_bigint(yc1)}, false};
}

static inline bool g1_on_curve(const G1A& p) {
  if (p.inf) return true;
  return p.y.sqr() == p.x.sqr() * p.x + Fq::from_u64(3);
}
static inline Fq2 g2_coeff_b() {
  Fq2 xi = {Fq::from_u64(9), Fq::from_u64(1)};
  return Fq2{Fq::from_u64(3), Fq::zero()} * xi.inverse();
}
static inline bool g2_on_curve(const G2A& p) {
  if (p.inf) return true;
  return p.y.sqr() == p.x.sqr() * p.x + g2_coeff_b();
}

// ---------------------------------------------------------------------------
// Multi-scalar multiplication (the reference calls ark-ec VariableBaseMSM::msm,
// crates/amt/src/prove_params/prove.rs:17,31,55,77). Pippenger with unsigned
// windows; the result is a group element, unique whatever the algorithm.
template <class F>
static Jac<F> msm(const Affine<F>* bases, const BigInt* scalars, size_t n) {
  if (n == 0) return Jac<F>::inf();
  int c = 1;
  while ((size_t(1) << (c + 2)) < n && c < 16) ++c;
  if (n < 8) {
    Jac<F> acc = Jac<F>::inf();
    for (size_t i = 0; i < n; ++i) acc = acc.add(Jac<F>::from_affine(bases[i]).mul(scalars[i]));
    return acc;
  }
  int windows = (256 + c - 1) / c;
  std::vector<Jac<F>> buckets(size_t(1) << c);
  Jac<F> total = Jac<F>::inf();
  for (int w = windows - 1; w >= 0; --w) {
    for (int k = 0; k < c; ++k) total = total.dbl();
    for (auto& b : buckets) b = Jac<F>::inf();
    for (size_t i = 0; i < n; ++i) {
      int bit = w * c;
      u64 d = 0;
      for (int k = 0; k < c && bit + k < 256; ++k)
        d |= ((scalars[i].v[(bit + k) / 64] >> ((bit + k) % 64)) & 1) << k;
      if (d) buckets[d] = buckets[d].add_affine(bases[i]);
    }
    Jac<F> run = Jac<F>::inf(), sum = Jac<F>::inf();
    for (size_t b = buckets.size() - 1; b >= 1; --b) {
      run = run.add(buckets[b]);
      sum = sum.add(run);
    }
    total = total.add(sum);
  }
  return total;
}

}  // namespace zgo
