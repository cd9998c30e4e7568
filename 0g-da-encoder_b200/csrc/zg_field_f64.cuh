// BN254 Montgomery product (Fq, and Fr for the NTTs) on the FP64 pipe (device only).
//
// The MSM bucket loop saturates the integer multiply-add pipe, while the
// FP64 pipe of the SM (DFMA at the same rate as IMAD on sm_100a) is idle. This
// product computes the same value as Fq::mul (a * b / 2^256 mod p, inputs and
// output in [0, p), 8 x 32-bit words) with 52-bit limbs held in doubles:
//
//  * operands are split into 5 limbs of 52 bits (the last one 48 bits), each
//    an exact double;
//  * a limb product a*b (< 2^104) is split exactly into hi = floor(ab / 2^52)
//    and lo = ab mod 2^52 by two FMAs: h = fma_rz(a, b, 2^104) holds hi in its
//    mantissa, and l = fma(a, b, 2^104 + 2^52 - h) = 2^52 + lo is exact (the
//    addend is an exact multiple of 2^52 below 2^104);
//  * the bit patterns of h and l (integers offset by the patterns of 2^104 and
//    2^52) are summed in 64-bit integer column accumulators whose initial
//    values cancel the offsets; the offsets are multiples of 2^52, so the low
//    52 bits of a column are exact at any time;
//  * Montgomery reduction runs limb by limb (CIOS order): 4 steps of 52 bits
//    and one of 48 bits remove 256 bits, m = t_i * (-p^-1) mod 2^52 (2^48) by
//    the same split;
//  * the result (< 2p) is repacked into 32-bit words and reduced once.
// Column sums stay below 2^58 (at most 20 terms below 2^52 plus a carry).
#pragma once
#include "zg_field.cuh"

namespace zg {
namespace f52 {

constexpr uint64_t KL = 0x4330000000000000ull;  // bit pattern of 2^52
constexpr uint64_t KH = 0x4670000000000000ull;  // bit pattern of 2^104
constexpr uint64_t M52 = (1ull << 52) - 1;

// products a_i * b_j with i + j = c (5 x 5 limbs)
__host__ __device__ constexpr int nprod(int c) { return (c < 0 || c > 8) ? 0 : (c <= 4 ? c + 1 : 9 - c); }
// column c receives 2 * nprod(c) low halves and 2 * nprod(c - 1) high halves
// (operand products and reduction products)
__host__ __device__ constexpr uint64_t col_init(int c) {
  return (uint64_t)0 - (uint64_t)(2 * nprod(c)) * KL - (uint64_t)(2 * nprod(c - 1)) * KH;
}

// 52-bit limbs of the modulus, -p^-1 mod 2^52 and mod 2^48 (Fq and Fr)
template <class C> struct Limbs52;
template <> struct Limbs52<FqCfg> {
  static __device__ __forceinline__ double P(int j) {
    return j == 0 ? (double)0x8c16d87cfd47ull
         : j == 1 ? (double)0x916871ca8d3c2ull
         : j == 2 ? (double)0x181585d97816aull
         : j == 3 ? (double)0xa029b85045b68ull
                  : (double)0x30644e72e131ull;
  }
  static constexpr double PINV52 = (double)0x20782e4866389ull;
  static constexpr double PINV48 = (double)0x782e4866389ull;
};
template <> struct Limbs52<FrCfg> {
  static __device__ __forceinline__ double P(int j) {
    return j == 0 ? (double)0x1f593f0000001ull
         : j == 1 ? (double)0x4879b9709143eull
         : j == 2 ? (double)0x181585d2833e8ull
         : j == 3 ? (double)0xa029b85045b68ull
                  : (double)0x30644e72e131ull;
  }
  static constexpr double PINV52 = (double)0x1f593efffffffull;
  static constexpr double PINV48 = (double)0xf593efffffffull;
};

// exact double of the 52-bit integer hi20:lo (hi20 < 2^20)
__device__ __forceinline__ double u52(uint32_t lo, uint32_t hi20) {
  return __dsub_rn(__hiloint2double((int)(hi20 | 0x43300000u), (int)lo), 0x1p52);
}

template <class C>
__device__ __forceinline__ void split(const Fp<C>& a, double* x) {
  const uint32_t* w = a.v;
  x[0] = u52(w[0], w[1] & 0xfffffu);
  x[1] = u52(__funnelshift_r(w[1], w[2], 20), __funnelshift_r(w[2], w[3], 20) & 0xfffffu);
  x[2] = u52(__funnelshift_r(w[3], w[4], 8), (w[4] >> 8) & 0xfffffu);
  x[3] = u52(__funnelshift_r(w[4], w[5], 28), __funnelshift_r(w[5], w[6], 28) & 0xfffffu);
  x[4] = u52(__funnelshift_r(w[6], w[7], 16), w[7] >> 16);
}

// lo += bits(2^52 + (ab mod 2^52)), hi += bits(2^104 + floor(ab / 2^52) 2^52)
__device__ __forceinline__ void prod(double a, double b, uint64_t& lo, uint64_t& hi) {
  const double h = __fma_rz(a, b, 0x1p104);
  const double d = __dsub_rn(0x1p104 + 0x1p52, h);
  const double l = __fma_rn(a, b, d);
  lo += (uint64_t)__double_as_longlong(l);
  hi += (uint64_t)__double_as_longlong(h);
}

// a * b / 2^256 mod p for a, b < p; result < p (p the modulus of C: Fq or Fr)
template <class C>
__device__ __forceinline__ Fp<C> mont_mul(const Fp<C>& a, const Fp<C>& b) {
  typedef Limbs52<C> L;
  double A[5], B[5];
  split(a, A);
  split(b, B);
  uint64_t t[10];
#pragma unroll
  for (int c = 0; c < 10; ++c) t[c] = col_init(c);
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int j = 0; j < 5; ++j) prod(A[i], B[j], t[i + j], t[i + j + 1]);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double ti = u52((uint32_t)t[i], (uint32_t)(t[i] >> 32) & 0xfffffu);
    const double h = __fma_rz(ti, L::PINV52, 0x1p104);
    const double d = __dsub_rn(0x1p104 + 0x1p52, h);
    const double m = __dsub_rn(__fma_rn(ti, L::PINV52, d), 0x1p52);
#pragma unroll
    for (int j = 0; j < 5; ++j) prod(m, L::P(j), t[i + j], t[i + j + 1]);
    t[i + 1] += t[i] >> 52;
  }
  {
    const double t4 = u52((uint32_t)t[4], (uint32_t)(t[4] >> 32) & 0xffffu);  // low 48 bits
    const double h = __fma_rz(t4, L::PINV48, 0x1p100);
    const double d = __dsub_rn(0x1p100 + 0x1p48, h);
    const double m = __dsub_rn(__fma_rn(t4, L::PINV48, d), 0x1p48);
#pragma unroll
    for (int j = 0; j < 5; ++j) prod(m, L::P(j), t[4 + j], t[5 + j]);
  }
  // normalise columns 4..9; the value is t / 2^256 = bits 256.. of sum t_c 2^(52c)
  const uint32_t top = (uint32_t)(t[4] >> 48) & 15u;
  t[5] += t[4] >> 52;
  t[6] += t[5] >> 52;
  t[7] += t[6] >> 52;
  t[8] += t[7] >> 52;
  t[9] += t[8] >> 52;
  const uint64_t n5 = t[5] & M52, n6 = t[6] & M52, n7 = t[7] & M52, n8 = t[8] & M52, n9 = t[9];
  Fp<C> r;
  r.v[0] = top | (uint32_t)(n5 << 4);
  r.v[1] = (uint32_t)(n5 >> 28) | (uint32_t)(n6 << 24);
  r.v[2] = (uint32_t)(n6 >> 8);
  r.v[3] = (uint32_t)(n6 >> 40) | (uint32_t)(n7 << 12);
  r.v[4] = (uint32_t)(n7 >> 20);
  r.v[5] = (uint32_t)n8;
  r.v[6] = (uint32_t)(n8 >> 32) | (uint32_t)(n9 << 20);
  r.v[7] = (uint32_t)(n9 >> 12);
  Fp<C> s;
  const uint32_t borrow = Fp<C>::sub_raw(s, r, Fp<C>::modulus());
  return borrow ? r : s;
}

}  // namespace f52
}  // namespace zg
