// BN254 Montgomery product (Fq or Fr) with 28-bit limbs and 64-bit column sums.
//
// Fq::mul runs the 8 x 32-bit CIOS rows as carry chains (mad.lo.cc /
// madc.hi.cc): every step waits on the previous one's carry flag, and on
// sm_100a the carrying multiply-adds take twice the pipe time of plain ones.
// This product computes the same value (a * b / 2^256 mod p, inputs and
// output in [0, p), 8 x 32-bit words) without carry flags:
//
//  * both operands are cut into 10 limbs of 28 bits (the last one 4 bits);
//  * the 100 limb products (< 2^56 each) are summed per column in 64-bit
//    words by 32 x 32 -> 64 multiply-adds (a column never holds more than 20
//    terms below 2^56 plus a carry, < 2^61), so the columns are independent
//    chains, not one carry chain;
//  * Montgomery reduction removes 9 x 28 + 4 = 256 bits (R = 2^256, the
//    representation of Fq::mul and of the param files): per step
//    m = t_i * (-p^-1) mod 2^28 (the last step mod 2^4), t += m * p at that
//    column, and t_i's upper bits move to t_(i+1);
//  * the columns from bit 252 up are normalised into 28-bit limbs, shifted
//    right by 4 bits and repacked into 32-bit words (< 2p), then reduced once.
// Host and device share the code (plain 64-bit arithmetic); the device
// compiles each (uint64_t)x * y + t to one wide multiply-add.
#pragma once
#include "zg_field.cuh"

namespace zg {
namespace w28 {

constexpr uint32_t M28 = (1u << 28) - 1;

// 28-bit limbs of the moduli and -p^-1 mod 2^28 / mod 2^4
struct FqLimbs {
  static constexpr uint32_t PINV28 = 0x4866389u, PINV4 = 0x9u;
  static ZG_HD constexpr uint32_t P(int j) {
    return j == 0 ? 0x87cfd47u : j == 1 ? 0x208c16du : j == 2 ? 0x1ca8d3cu : j == 3 ? 0x6a91687u
         : j == 4 ? 0x85d9781u : j == 5 ? 0xb681815u : j == 6 ? 0x9b85045u : j == 7 ? 0xe131a02u
         : j == 8 ? 0x644e72u : 0x3u;
  }
};
struct FrLimbs {
  static constexpr uint32_t PINV28 = 0xfffffffu, PINV4 = 0xfu;
  static ZG_HD constexpr uint32_t P(int j) {
    return j == 0 ? 0x1u : j == 1 ? 0xe1f593fu : j == 2 ? 0x9709143u : j == 3 ? 0xe84879bu
         : j == 4 ? 0x85d2833u : j == 5 ? 0xb681815u : j == 6 ? 0x9b85045u : j == 7 ? 0xe131a02u
         : j == 8 ? 0x644e72u : 0x3u;
  }
};
template <class C> struct Limbs;
template <> struct Limbs<FqCfg> : FqLimbs {};
template <> struct Limbs<FrCfg> : FrLimbs {};

template <class C>
ZG_HD void split(const Fp<C>& a, uint32_t x[10]) {
  const uint32_t* v = a.v;
  x[0] = v[0] & M28;
  x[1] = ((v[0] >> 28) | (v[1] << 4)) & M28;
  x[2] = ((v[1] >> 24) | (v[2] << 8)) & M28;
  x[3] = ((v[2] >> 20) | (v[3] << 12)) & M28;
  x[4] = ((v[3] >> 16) | (v[4] << 16)) & M28;
  x[5] = ((v[4] >> 12) | (v[5] << 20)) & M28;
  x[6] = ((v[5] >> 8) | (v[6] << 24)) & M28;
  x[7] = (v[6] >> 4) & M28;
  x[8] = v[7] & M28;
  x[9] = v[7] >> 28;
}

// a * b / 2^256 mod p for a, b < p; result < p (p the modulus of C: Fq or Fr)
template <class C>
ZG_HD Fp<C> mont_mul(const Fp<C>& a, const Fp<C>& b) {
  typedef Limbs<C> L;
  uint32_t x[10], y[10];
  split(a, x);
  split(b, y);
  uint64_t t[20];
#pragma unroll
  for (int k = 0; k < 20; ++k) t[k] = 0;
#pragma unroll
  for (int i = 0; i < 10; ++i)
#pragma unroll
    for (int j = 0; j < 10; ++j) t[i + j] += (uint64_t)x[i] * y[j];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const uint32_t m = ((uint32_t)t[i] * L::PINV28) & M28;
#pragma unroll
    for (int j = 0; j < 10; ++j) t[i + j] += (uint64_t)m * L::P(j);
    t[i + 1] += t[i] >> 28;
  }
  {
    const uint32_t m = ((uint32_t)t[9] * L::PINV4) & 15u;
#pragma unroll
    for (int j = 0; j < 10; ++j) t[9 + j] += (uint64_t)m * L::P(j);
  }
  // columns 9.. into 28-bit limbs r[0..9] (value r * 2^252, r[0] % 16 == 0)
  uint32_t r[10];
  uint64_t c = 0;
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    c += t[9 + k];
    r[k] = (uint32_t)c & M28;
    c >>= 28;
  }
  // drop the 4 low bits: bit 28 k - 4 of the result is bit 0 of r[k]
  Fp<C> o;
  o.v[0] = (r[0] >> 4) | (r[1] << 24);
  o.v[1] = (r[1] >> 8) | (r[2] << 20);
  o.v[2] = (r[2] >> 12) | (r[3] << 16);
  o.v[3] = (r[3] >> 16) | (r[4] << 12);
  o.v[4] = (r[4] >> 20) | (r[5] << 8);
  o.v[5] = (r[5] >> 24) | (r[6] << 4);
  o.v[6] = r[7] | (r[8] << 28);
  o.v[7] = (r[8] >> 4) | (r[9] << 24);
  Fp<C> s;
  const uint32_t borrow = Fp<C>::sub_raw(s, o, Fp<C>::modulus());
  return borrow ? o : s;
}

}  // namespace w28
}  // namespace zg
