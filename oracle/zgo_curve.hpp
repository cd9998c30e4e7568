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
  // this + affine point (madd-2007-bl: 7M + 4S, the mixed addition ark-ec 0.4
  // uses for `Projective += &Affine`), with the equal / opposite cases
  Jac add_affine(const Affine<F>& a) const {
    if (a.inf) return *this;
    if (is_inf()) return from_affine(a);
    F Z1Z1 = Z.sqr();
    F U2 = a.x * Z1Z1;
    F S2 = a.y * Z * Z1Z1;
    if (U2 == X) {
      if (S2 == Y) return dbl();
      return inf();
    }
    F H = U2 - X;
    F HH = H.sqr();
    F I = HH.dbl().dbl();
    F J = H * I;
    F r = (S2 - Y).dbl();
    F V = X * I;
    F X3 = r.sqr() - J - V.dbl();
    F Y3 = r * (V - X3) - (Y * J).dbl();
    F Z3 = (Z + H).sqr() - Z1Z1 - HH;
    return {X3, Y3, Z3};
  }
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
// Multi-scalar multiplication: a restatement of the algorithm behind the
// reference's MSM calls (VariableBaseMSM::msm, crates/amt/src/prove_params/
// prove.rs:17,31,55,77), ark-ec 0.4.2's signed-digit bucket method for curves
// with cheap negation (msm_bigint_wnaf; ark-ec is a third-party dependency,
// Cargo.lock:180, not present here, so this follows its published algorithm):
//  * window width c = 3 below 32 points, else floor(ceil_log2(n) * 69 / 100) + 2
//    (ark's ln_without_floats(n) + 2);
//  * every scalar is cut into ceil(254 / c) signed digits in
//    [-2^(c-1), 2^(c-1)) read word-wise from its 64-bit limbs, the carry of
//    the last window folded into the last digit (ark's make_digits);
//  * per window (in parallel over windows, as ark's `parallel` feature runs
//    them): 2^c Jacobian buckets, bucket |d| - 1 += +-base with a mixed
//    addition, then the running-sum reduction from the top bucket down;
//  * the window sums are folded from the top window with c doublings each.
// The result is a group element, the same whatever the algorithm.
static inline int ark_msm_window(size_t n) {
  if (n < 32) return 3;
  int l = 0;
  while ((size_t(1) << l) < n) ++l;
  return l * 69 / 100 + 2;
}
static inline void signed_digits(const BigInt& s, int c, int count, int32_t* out) {
  const u64 radix = u64(1) << c, mask = radix - 1;
  u64 carry = 0;
  for (int i = 0; i < count; ++i) {
    const int off = i * c, li = off / 64, sh = off % 64;
    u64 bits = s.v[li] >> sh;
    if (sh + c > 64 && li + 1 < 4) bits |= s.v[li + 1] << (64 - sh);
    const u64 coef = carry + (bits & mask);
    carry = (coef + radix / 2) >> c;
    out[i] = (int32_t)((int64_t)coef - (int64_t)(carry << c));
  }
  out[count - 1] += (int32_t)(carry << c);
}
template <class F>
static Jac<F> msm(const Affine<F>* bases, const BigInt* scalars, size_t n) {
  if (n == 0) return Jac<F>::inf();
  const int c = ark_msm_window(n);
  const int count = (254 + c - 1) / c;
  std::vector<int32_t> dig(n * count);
#pragma omp parallel for schedule(static) if (n >= 4096)
  for (size_t i = 0; i < n; ++i) signed_digits(scalars[i], c, count, &dig[i * count]);
  std::vector<Jac<F>> wsum(count);
#pragma omp parallel for schedule(dynamic, 1) if (n >= 256)
  for (int w = 0; w < count; ++w) {
    std::vector<Jac<F>> buckets(size_t(1) << c, Jac<F>::inf());
    for (size_t i = 0; i < n; ++i) {
      const int32_t d = dig[i * count + w];
      if (d > 0) buckets[d - 1] = buckets[d - 1].add_affine(bases[i]);
      else if (d < 0) buckets[-d - 1] = buckets[-d - 1].add_affine(affine_neg(bases[i]));
    }
    Jac<F> run = Jac<F>::inf(), acc = Jac<F>::inf();
    for (size_t b = buckets.size(); b-- > 0;) {
      run = run.add(buckets[b]);
      acc = acc.add(run);
    }
    wsum[w] = acc;
  }
  Jac<F> total = Jac<F>::inf();
  for (int w = count - 1; w >= 1; --w) {
    total = total.add(wsum[w]);
    for (int k = 0; k < c; ++k) total = total.dbl();
  }
  return total.add(wsum[0]);
}

}  // namespace zgo
