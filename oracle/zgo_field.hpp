// ORACLE — test infrastructure only. CPU restatement of the 0G DA encoder's
// arithmetic (BN254 Fr/Fq, Fq2/Fq6/Fq12). Never linked into the product
// library; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
// load it, as the checker.
//
// Representation follows ark-ff 0.4.2 (third-party dependency of the
// reference, Cargo.lock:199): Montgomery form with R = 2^256, four 64-bit
// little-endian limbs. The reference's mont file format
// (crates/amt/src/prove_params/fast_serde_bn254.rs:139-187) stores exactly
// these limbs.
#pragma once
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace zgo {

typedef unsigned __int128 u128;
typedef uint64_t u64;

struct BigInt {
  u64 v[4];
};

static inline bool big_geq(const u64 a[4], const u64 b[4]) {
  for (int i = 3; i >= 0; --i) {
    if (a[i] != b[i]) return a[i] > b[i];
  }
  return true;
}
static inline u64 big_sub(u64 r[4], const u64 a[4], const u64 b[4]) {
  u64 borrow = 0;
  for (int i = 0; i < 4; ++i) {
    u128 t = (u128)a[i] - b[i] - borrow;
    r[i] = (u64)t;
    borrow = (u64)(t >> 64) & 1;
  }
  return borrow;
}
static inline u64 big_add(u64 r[4], const u64 a[4], const u64 b[4]) {
  u64 carry = 0;
  for (int i = 0; i < 4; ++i) {
    u128 t = (u128)a[i] + b[i] + carry;
    r[i] = (u64)t;
    carry = (u64)(t >> 64);
  }
  return carry;
}

// Field configuration: modulus P, R^2 mod P, INV = -P^{-1} mod 2^64.
struct FrCfg {
  static constexpr u64 P[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL,
                               0xb85045b68181585dULL, 0x30644e72e131a029ULL};
  static constexpr u64 R2[4] = {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL,
                                0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL};
  static constexpr u64 INV = 0xc2e1f593efffffffULL;
};
struct FqCfg {
  static constexpr u64 P[4] = {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL,
                               0xb85045b68181585dULL, 0x30644e72e131a029ULL};
  static constexpr u64 R2[4] = {0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL,
                                0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL};
  static constexpr u64 INV = 0x87d20782e4866389ULL;
};

template <class C>
struct Fp {
  u64 v[4];  // Montgomery form

  static Fp zero() { Fp r; memset(r.v, 0, 32); return r; }
  static Fp one() { return from_u64(1); }
  static Fp from_u64(u64 x) {
    BigInt b = {{x, 0, 0, 0}};
    return from_bigint(b);
  }
  // canonical integer (< P) -> Montgomery (x * R mod P).
  static Fp from_bigint(const BigInt& b) {
    Fp t; memcpy(t.v, b.v, 32);
    Fp r2; memcpy(r2.v, C::R2, 32);
    return t * r2;
  }
  static Fp from_raw_mont(const u64 m[4]) { Fp r; memcpy(r.v, m, 32); return r; }
  BigInt to_bigint() const {
    Fp one_raw = zero(); one_raw.v[0] = 1;
    Fp t = (*this) * one_raw;
    BigInt b; memcpy(b.v, t.v, 32);
    return b;
  }
  bool is_zero() const { return (v[0] | v[1] | v[2] | v[3]) == 0; }
  bool operator==(const Fp& o) const { return memcmp(v, o.v, 32) == 0; }
  bool operator!=(const Fp& o) const { return !(*this == o); }

  // add / sub / mul: unrolled four-limb code with u128 carries and a final
  // conditional subtraction chosen by mask (same values as the textbook
  // forms; both moduli are below 2^254, so a + b < 2^255 never carries out)
  static inline void sub_p_if_geq(u64 r[4]) {
    u128 t = (u128)r[0] - C::P[0];
    const u64 d0 = (u64)t;
    t = (u128)r[1] - C::P[1] - (u64)((t >> 64) & 1);
    const u64 d1 = (u64)t;
    t = (u128)r[2] - C::P[2] - (u64)((t >> 64) & 1);
    const u64 d2 = (u64)t;
    t = (u128)r[3] - C::P[3] - (u64)((t >> 64) & 1);
    const u64 d3 = (u64)t;
    const u64 keep = (u64)0 - (u64)((t >> 64) & 1);  // all ones when r < P
    r[0] = (r[0] & keep) | (d0 & ~keep);
    r[1] = (r[1] & keep) | (d1 & ~keep);
    r[2] = (r[2] & keep) | (d2 & ~keep);
    r[3] = (r[3] & keep) | (d3 & ~keep);
  }
  Fp operator+(const Fp& o) const {
    Fp r;
    u128 t = (u128)v[0] + o.v[0];
    r.v[0] = (u64)t;
    t = (u128)v[1] + o.v[1] + (u64)(t >> 64);
    r.v[1] = (u64)t;
    t = (u128)v[2] + o.v[2] + (u64)(t >> 64);
    r.v[2] = (u64)t;
    r.v[3] = v[3] + o.v[3] + (u64)(t >> 64);
    sub_p_if_geq(r.v);
    return r;
  }
  Fp operator-(const Fp& o) const {
    Fp r;
    u128 t = (u128)v[0] - o.v[0];
    r.v[0] = (u64)t;
    t = (u128)v[1] - o.v[1] - (u64)((t >> 64) & 1);
    r.v[1] = (u64)t;
    t = (u128)v[2] - o.v[2] - (u64)((t >> 64) & 1);
    r.v[2] = (u64)t;
    t = (u128)v[3] - o.v[3] - (u64)((t >> 64) & 1);
    r.v[3] = (u64)t;
    const u64 m = (u64)0 - (u64)((t >> 64) & 1);  // all ones on borrow: add P back
    t = (u128)r.v[0] + (C::P[0] & m);
    r.v[0] = (u64)t;
    t = (u128)r.v[1] + (C::P[1] & m) + (u64)(t >> 64);
    r.v[1] = (u64)t;
    t = (u128)r.v[2] + (C::P[2] & m) + (u64)(t >> 64);
    r.v[2] = (u64)t;
    r.v[3] = r.v[3] + (C::P[3] & m) + (u64)(t >> 64);
    return r;
  }
  Fp operator-() const {
    if (is_zero()) return *this;
    Fp r; big_sub(r.v, C::P, v); return r;
  }
  // CIOS Montgomery multiplication, rows unrolled. The top limb of both
  // moduli is below 2^62, so the running value never needs a fifth limb
  // beyond one carry word (the "no-carry" form of CIOS).
  Fp operator*(const Fp& o) const {
    u64 t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    for (int i = 0; i < 4; ++i) {
      const u64 bi = o.v[i];
      u128 x = (u128)v[0] * bi + t0;
      const u64 a0 = (u64)x;
      u64 A = (u64)(x >> 64);
      const u64 m = a0 * C::INV;
      u128 y = (u128)m * C::P[0] + a0;
      u64 Cc = (u64)(y >> 64);
      x = (u128)v[1] * bi + t1 + A;
      A = (u64)(x >> 64);
      y = (u128)m * C::P[1] + (u64)x + Cc;
      Cc = (u64)(y >> 64);
      t0 = (u64)y;
      x = (u128)v[2] * bi + t2 + A;
      A = (u64)(x >> 64);
      y = (u128)m * C::P[2] + (u64)x + Cc;
      Cc = (u64)(y >> 64);
      t1 = (u64)y;
      x = (u128)v[3] * bi + t3 + A;
      A = (u64)(x >> 64);
      y = (u128)m * C::P[3] + (u64)x + Cc;
      Cc = (u64)(y >> 64);
      t2 = (u64)y;
      t3 = Cc + A;
    }
    Fp r;
    r.v[0] = t0; r.v[1] = t1; r.v[2] = t2; r.v[3] = t3;
    sub_p_if_geq(r.v);
    return r;
  }
  Fp& operator+=(const Fp& o) { *this = *this + o; return *this; }
  Fp& operator-=(const Fp& o) { *this = *this - o; return *this; }
  Fp& operator*=(const Fp& o) { *this = *this * o; return *this; }
  Fp sqr() const { return (*this) * (*this); }
  Fp dbl() const { return *this + *this; }
  Fp pow(const u64* e, int nlimbs) const {
    Fp r = one(), b = *this;
    for (int i = 0; i < nlimbs; ++i) {
      u64 w = e[i];
      for (int k = 0; k < 64; ++k) {
        if (w & 1) r *= b;
        b = b.sqr();
        w >>= 1;
      }
    }
    return r;
  }
  Fp pow_u64(u64 e) const { return pow(&e, 1); }
  Fp inverse() const {  // Fermat; inverse(0) = 0 (callers check)
    u64 e[4]; u64 two[4] = {2, 0, 0, 0};
    big_sub(e, C::P, two);
    return pow(e, 4);
  }
  // canonical ordering, as ark-ff compares field elements (into_bigint order)
  bool canon_gt(const Fp& o) const {
    BigInt a = to_bigint(), b = o.to_bigint();
    for (int i = 3; i >= 0; --i)
      if (a.v[i] != b.v[i]) return a.v[i] > b.v[i];
    return false;
  }
  void to_le_bytes(uint8_t out[32]) const {
    BigInt b = to_bigint();
    memcpy(out, b.v, 32);
  }
  static bool from_le_bytes(const uint8_t in[32], Fp* out) {
    BigInt b; memcpy(b.v, in, 32);
    if (big_geq(b.v, C::P)) return false;
    *out = from_bigint(b);
    return true;
  }
};

typedef Fp<FrCfg> Fr;
typedef Fp<FqCfg> Fq;

// Fq2 = Fq[u]/(u^2 + 1)
struct Fq2 {
  Fq c0, c1;
  static Fq2 zero() { return {Fq::zero(), Fq::zero()}; }
  static Fq2 one() { return {Fq::one(), Fq::zero()}; }
  bool is_zero() const { return c0.is_zero() && c1.is_zero(); }
  bool operator==(const Fq2& o) const { return c0 == o.c0 && c1 == o.c1; }
  bool operator!=(const Fq2& o) const { return !(*this == o); }
  Fq2 operator+(const Fq2& o) const { return {c0 + o.c0, c1 + o.c1}; }
  Fq2 operator-(const Fq2& o) const { return {c0 - o.c0, c1 - o.c1}; }
  Fq2 operator-() const { return {-c0, -c1}; }
  Fq2 operator*(const Fq2& o) const {
    Fq a = c0 * o.c0, b = c1 * o.c1;
    Fq s = (c0 + c1) * (o.c0 + o.c1);
    return {a - b, s - a - b};
  }
  Fq2 operator*(const Fq& k) const { return {c0 * k, c1 * k}; }
  Fq2& operator+=(const Fq2& o) { *this = *this + o; return *this; }
  Fq2& operator-=(const Fq2& o) { *this = *this - o; return *this; }
  Fq2& operator*=(const Fq2& o) { *this = *this * o; return *this; }
  Fq2 sqr() const { return (*this) * (*this); }
  Fq2 dbl() const { return *this + *this; }
  Fq2 conj() const { return {c0, -c1}; }
  Fq2 inverse() const {
    Fq n = c0.sqr() + c1.sqr();
    Fq ni = n.inverse();
    return {c0 * ni, -(c1 * ni)};
  }
  // multiply by the non-residue xi = 9 + u used for Fq6
  Fq2 mul_xi() const {
    Fq nine = Fq::from_u64(9);
    return {c0 * nine - c1, c0 + c1 * nine};
  }
  Fq2 pow(const u64* e, int n) const {
    Fq2 r = one(), b = *this;
    for (int i = 0; i < n; ++i) {
      u64 w = e[i];
      for (int k = 0; k < 64; ++k) { if (w & 1) r *= b; b = b.sqr(); w >>= 1; }
    }
    return r;
  }
  // ark-ff QuadExtField ordering: c1 first, then c0
  bool canon_gt(const Fq2& o) const {
    if (c1 != o.c1) return c1.canon_gt(o.c1);
    return c0.canon_gt(o.c0);
  }
};

// Fq6 = Fq2[v]/(v^3 - xi)
struct Fq6 {
  Fq2 c0, c1, c2;
  static Fq6 zero() { return {Fq2::zero(), Fq2::zero(), Fq2::zero()}; }
  static Fq6 one() { return {Fq2::one(), Fq2::zero(), Fq2::zero()}; }
  bool operator==(const Fq6& o) const { return c0 == o.c0 && c1 == o.c1 && c2 == o.c2; }
  Fq6 operator+(const Fq6& o) const { return {c0 + o.c0, c1 + o.c1, c2 + o.c2}; }
  Fq6 operator-(const Fq6& o) const { return {c0 - o.c0, c1 - o.c1, c2 - o.c2}; }
  Fq6 operator-() const { return {-c0, -c1, -c2}; }
  Fq6 operator*(const Fq6& o) const {
    Fq2 a = c0 * o.c0, b = c1 * o.c1, c = c2 * o.c2;
    Fq2 t0 = ((c1 + c2) * (o.c1 + o.c2) - b - c).mul_xi() + a;
    Fq2 t1 = (c0 + c1) * (o.c0 + o.c1) - a - b + c.mul_xi();
    Fq2 t2 = (c0 + c2) * (o.c0 + o.c2) - a - c + b;
    return {t0, t1, t2};
  }
  Fq6 mul_v() const { return {c2.mul_xi(), c0, c1}; }
  Fq6 inverse() const {
    Fq2 A = c0.sqr() - (c1 * c2).mul_xi();
    Fq2 B = c2.sqr().mul_xi() - c0 * c1;
    Fq2 C = c1.sqr() - c0 * c2;
    Fq2 F = (c2 * B + c1 * C).mul_xi() + c0 * A;
    Fq2 Fi = F.inverse();
    return {A * Fi, B * Fi, C * Fi};
  }
};

// Fq12 = Fq6[w]/(w^2 - v)
struct Fq12 {
  Fq6 c0, c1;
  static Fq12 one() { return {Fq6::one(), Fq6::zero()}; }
  bool operator==(const Fq12& o) const { return c0 == o.c0 && c1 == o.c1; }
  bool operator!=(const Fq12& o) const { return !(*this == o); }
  Fq12 operator*(const Fq12& o) const {
    Fq6 a = c0 * o.c0, b = c1 * o.c1;
    Fq6 s = (c0 + c1) * (o.c0 + o.c1);
    return {a + b.mul_v(), s - a - b};
  }
  Fq12 sqr() const { return (*this) * (*this); }
  Fq12 conj() const { return {c0, -c1}; }
  Fq12 inverse() const {
    Fq6 t = (c0 * c0 - (c1 * c1).mul_v()).inverse();
    return {c0 * t, -(c1 * t)};
  }
  Fq12 pow_big(const std::vector<u64>& e) const {
    Fq12 r = one(), b = *this;
    for (size_t i = 0; i < e.size(); ++i) {
      u64 w = e[i];
      for (int k = 0; k < 64; ++k) { if (w & 1) r = r * b; b = b.sqr(); w >>= 1; }
    }
    return r;
  }
};

// Fr two-adic root of unity: generator 5 raised to (r-1)/2^28 (ark-bn254 FrConfig
// declares generator = 5; ark-ff derives TWO_ADIC_ROOT_OF_UNITY = g^t).
static inline Fr fr_two_adic_root() {
  static const BigInt W = {{0x9bd61b6e725b19f0ULL, 0x402d111e41112ed4ULL,
                            0x00e0a7eb8ef62abcULL, 0x2a3c09f0a58a7e85ULL}};
  return Fr::from_bigint(W);
}
static const int FR_TWO_ADICITY = 28;

// Radix2EvaluationDomain::new(2^log_n).group_gen
static inline Fr fr_root_of_unity(int log_n) {
  Fr w = fr_two_adic_root();
  for (int i = log_n; i < FR_TWO_ADICITY; ++i) w = w.sqr();
  return w;
}

}  // namespace zgo
