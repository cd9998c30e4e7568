// BN254 prime-field arithmetic for sm_100a: eight 32-bit limbs, Montgomery
// form with R = 2^256 (the same representation as ark-ff's four 64-bit limbs,
// so device buffers and the reference's mont param files share bytes,
// crates/amt/src/prove_params/fast_serde_bn254.rs:139-187).
//
// Multiplication is CIOS Montgomery: per limb b_i one multiply-accumulate row
// t += a * b_i and one reduction row t += m * p, each row split in an
// even-limb and an odd-limb carry chain (mad.lo.cc / madc.hi.cc) so every
// product half lands on its own limb without a second pass. Outputs that are
// written before every input of an asm block has been read are early-clobber
// ("=&r"), so the compiler never assigns them an input's register. Host builds
// use a portable 64-bit path with identical results.
#pragma once
#include <stdint.h>

#ifndef ZG_HD
#define ZG_HD __host__ __device__ __forceinline__
#endif

namespace zg {

struct FqCfg {
  static constexpr uint32_t p0 = 0xd87cfd47u, p1 = 0x3c208c16u, p2 = 0x6871ca8du, p3 = 0x97816a91u,
                            p4 = 0x8181585du, p5 = 0xb85045b6u, p6 = 0xe131a029u, p7 = 0x30644e72u;
  static constexpr uint32_t inv = 0xe4866389u;
  static constexpr uint32_t r2_0 = 0x538afa89u, r2_1 = 0xf32cfc5bu, r2_2 = 0xd44501fbu, r2_3 = 0xb5e71911u,
                            r2_4 = 0x0a417ff6u, r2_5 = 0x47ab1effu, r2_6 = 0xcab8351fu, r2_7 = 0x06d89f71u;
  static constexpr uint32_t one0 = 0xc58f0d9du, one1 = 0xd35d438du, one2 = 0xf5c70b3du, one3 = 0x0a78eb28u,
                            one4 = 0x7879462cu, one5 = 0x666ea36fu, one6 = 0x9a07df2fu, one7 = 0x0e0a77c1u;
};
struct FrCfg {
  static constexpr uint32_t p0 = 0xf0000001u, p1 = 0x43e1f593u, p2 = 0x79b97091u, p3 = 0x2833e848u,
                            p4 = 0x8181585du, p5 = 0xb85045b6u, p6 = 0xe131a029u, p7 = 0x30644e72u;
  static constexpr uint32_t inv = 0xefffffffu;
  static constexpr uint32_t r2_0 = 0xae216da7u, r2_1 = 0x1bb8e645u, r2_2 = 0xe35c59e3u, r2_3 = 0x53fe3ab1u,
                            r2_4 = 0x53bb8085u, r2_5 = 0x8c49833du, r2_6 = 0x7f4e44a5u, r2_7 = 0x0216d0b1u;
  static constexpr uint32_t one0 = 0x4ffffffbu, one1 = 0xac96341cu, one2 = 0x9f60cd29u, one3 = 0x36fc7695u,
                            one4 = 0x7879462eu, one5 = 0x666ea36fu, one6 = 0x9a07df2fu, one7 = 0x0e0a77c1u;
};

template <class C>
struct Fp {
  uint32_t v[8];

  ZG_HD static Fp zero() {
    Fp r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = 0;
    return r;
  }
  ZG_HD static Fp modulus() {
    Fp r;
    r.v[0] = C::p0; r.v[1] = C::p1; r.v[2] = C::p2; r.v[3] = C::p3;
    r.v[4] = C::p4; r.v[5] = C::p5; r.v[6] = C::p6; r.v[7] = C::p7;
    return r;
  }
  ZG_HD static Fp one() {
    Fp r;
    r.v[0] = C::one0; r.v[1] = C::one1; r.v[2] = C::one2; r.v[3] = C::one3;
    r.v[4] = C::one4; r.v[5] = C::one5; r.v[6] = C::one6; r.v[7] = C::one7;
    return r;
  }
  ZG_HD static Fp r2() {
    Fp r;
    r.v[0] = C::r2_0; r.v[1] = C::r2_1; r.v[2] = C::r2_2; r.v[3] = C::r2_3;
    r.v[4] = C::r2_4; r.v[5] = C::r2_5; r.v[6] = C::r2_6; r.v[7] = C::r2_7;
    return r;
  }
  ZG_HD bool is_zero() const {
    uint32_t o = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) o |= v[i];
    return o == 0;
  }
  ZG_HD bool operator==(const Fp& o) const {
    uint32_t d = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) d |= v[i] ^ o.v[i];
    return d == 0;
  }
  ZG_HD bool operator!=(const Fp& o) const { return !(*this == o); }

  // ---- add / sub (inputs and outputs fully reduced, in [0, p))
  ZG_HD static Fp add(const Fp& a, const Fp& b) {
    Fp s, t;
    uint32_t carry = add_raw(s, a, b);
    uint32_t borrow = sub_raw(t, s, modulus());
    // keep s when (no carry and borrow) i.e. s < p
    bool keep = (carry == 0) && (borrow != 0);
    return keep ? s : t;
  }
  ZG_HD static Fp sub(const Fp& a, const Fp& b) {
    Fp d, e;
    uint32_t borrow = sub_raw(d, a, b);
    add_raw(e, d, modulus());
    return borrow ? e : d;
  }
  ZG_HD static Fp neg(const Fp& a) {
    if (a.is_zero()) return a;
    Fp r;
    sub_raw(r, modulus(), a);
    return r;
  }
  ZG_HD static Fp dbl(const Fp& a) { return add(a, a); }

  ZG_HD Fp operator+(const Fp& o) const { return add(*this, o); }
  ZG_HD Fp operator-(const Fp& o) const { return sub(*this, o); }
  ZG_HD Fp operator-() const { return neg(*this); }
  ZG_HD Fp operator*(const Fp& o) const { return mul(*this, o); }
  ZG_HD Fp& operator+=(const Fp& o) { *this = add(*this, o); return *this; }
  ZG_HD Fp& operator-=(const Fp& o) { *this = sub(*this, o); return *this; }
  ZG_HD Fp& operator*=(const Fp& o) { *this = mul(*this, o); return *this; }
  ZG_HD Fp sqr() const { return mul(*this, *this); }

  ZG_HD static uint32_t add_raw(Fp& r, const Fp& a, const Fp& b) {
#ifdef __CUDA_ARCH__
    uint32_t c;
    asm("add.cc.u32 %0, %9, %17;\n\t"
        "addc.cc.u32 %1, %10, %18;\n\t"
        "addc.cc.u32 %2, %11, %19;\n\t"
        "addc.cc.u32 %3, %12, %20;\n\t"
        "addc.cc.u32 %4, %13, %21;\n\t"
        "addc.cc.u32 %5, %14, %22;\n\t"
        "addc.cc.u32 %6, %15, %23;\n\t"
        "addc.cc.u32 %7, %16, %24;\n\t"
        "addc.u32 %8, 0, 0;"
        : "=&r"(r.v[0]), "=&r"(r.v[1]), "=&r"(r.v[2]), "=&r"(r.v[3]), "=&r"(r.v[4]), "=&r"(r.v[5]),
          "=&r"(r.v[6]), "=&r"(r.v[7]), "=&r"(c)
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
          "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]),
          "r"(b.v[6]), "r"(b.v[7]));
    return c;
#else
    uint64_t c = 0;
    for (int i = 0; i < 8; ++i) {
      uint64_t s = (uint64_t)a.v[i] + b.v[i] + c;
      r.v[i] = (uint32_t)s;
      c = s >> 32;
    }
    return (uint32_t)c;
#endif
  }
  // returns 1 on borrow
  ZG_HD static uint32_t sub_raw(Fp& r, const Fp& a, const Fp& b) {
#ifdef __CUDA_ARCH__
    uint32_t c;
    asm("sub.cc.u32 %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32 %8, 0, 0;"
        : "=&r"(r.v[0]), "=&r"(r.v[1]), "=&r"(r.v[2]), "=&r"(r.v[3]), "=&r"(r.v[4]), "=&r"(r.v[5]),
          "=&r"(r.v[6]), "=&r"(r.v[7]), "=&r"(c)
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
          "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]), "r"(b.v[4]), "r"(b.v[5]),
          "r"(b.v[6]), "r"(b.v[7]));
    return c & 1;
#else
    int64_t br = 0;
    for (int i = 0; i < 8; ++i) {
      int64_t s = (int64_t)a.v[i] - b.v[i] - br;
      br = s < 0 ? 1 : 0;
      r.v[i] = (uint32_t)s;
    }
    return (uint32_t)br;
#endif
  }

  // ---- Montgomery multiplication: a * b / R mod p, inputs in [0, p)
  ZG_HD static Fp mul(const Fp& a, const Fp& b) {
#ifdef __CUDA_ARCH__
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0, t8;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint32_t bi = b.v[i];
      // t[0..8] = t[0..7] + a * bi   (even limbs chain, then odd limbs chain)
      asm("mad.lo.cc.u32 %0, %9, %17, %0;\n\t"
          "madc.hi.cc.u32 %1, %9, %17, %1;\n\t"
          "madc.lo.cc.u32 %2, %11, %17, %2;\n\t"
          "madc.hi.cc.u32 %3, %11, %17, %3;\n\t"
          "madc.lo.cc.u32 %4, %13, %17, %4;\n\t"
          "madc.hi.cc.u32 %5, %13, %17, %5;\n\t"
          "madc.lo.cc.u32 %6, %15, %17, %6;\n\t"
          "madc.hi.cc.u32 %7, %15, %17, %7;\n\t"
          "addc.u32 %8, 0, 0;\n\t"
          "mad.lo.cc.u32 %1, %10, %17, %1;\n\t"
          "madc.hi.cc.u32 %2, %10, %17, %2;\n\t"
          "madc.lo.cc.u32 %3, %12, %17, %3;\n\t"
          "madc.hi.cc.u32 %4, %12, %17, %4;\n\t"
          "madc.lo.cc.u32 %5, %14, %17, %5;\n\t"
          "madc.hi.cc.u32 %6, %14, %17, %6;\n\t"
          "madc.lo.cc.u32 %7, %16, %17, %7;\n\t"
          "madc.hi.u32 %8, %16, %17, %8;"
          : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "=&r"(t8)
          : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
            "r"(a.v[7]), "r"(bi));
      const uint32_t m = t0 * C::inv;
      // t[0..8] += m * p ; t0 becomes 0 and is dropped by the shift below
      asm("mad.lo.cc.u32 %0, %9, %10, %0;\n\t"
          "madc.hi.cc.u32 %1, %9, %10, %1;\n\t"
          "madc.lo.cc.u32 %2, %9, %12, %2;\n\t"
          "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"
          "madc.lo.cc.u32 %4, %9, %14, %4;\n\t"
          "madc.hi.cc.u32 %5, %9, %14, %5;\n\t"
          "madc.lo.cc.u32 %6, %9, %16, %6;\n\t"
          "madc.hi.cc.u32 %7, %9, %16, %7;\n\t"
          "addc.u32 %8, %8, 0;\n\t"
          "mad.lo.cc.u32 %1, %9, %11, %1;\n\t"
          "madc.hi.cc.u32 %2, %9, %11, %2;\n\t"
          "madc.lo.cc.u32 %3, %9, %13, %3;\n\t"
          "madc.hi.cc.u32 %4, %9, %13, %4;\n\t"
          "madc.lo.cc.u32 %5, %9, %15, %5;\n\t"
          "madc.hi.cc.u32 %6, %9, %15, %6;\n\t"
          "madc.lo.cc.u32 %7, %9, %17, %7;\n\t"
          "madc.hi.u32 %8, %9, %17, %8;"
          : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8)
          : "r"(m), "r"(C::p0), "r"(C::p1), "r"(C::p2), "r"(C::p3), "r"(C::p4), "r"(C::p5), "r"(C::p6),
            "r"(C::p7));
      t0 = t1; t1 = t2; t2 = t3; t3 = t4; t4 = t5; t5 = t6; t6 = t7; t7 = t8;
    }
    Fp r;
    r.v[0] = t0; r.v[1] = t1; r.v[2] = t2; r.v[3] = t3;
    r.v[4] = t4; r.v[5] = t5; r.v[6] = t6; r.v[7] = t7;
    Fp s;
    uint32_t borrow = sub_raw(s, r, modulus());
    return borrow ? r : s;
#else
    return mul_host(a, b);
#endif
  }

#ifndef __CUDA_ARCH__
  // the host product, out of line: inlined into every host use of the
  // extension-field and curve formulas it makes the host object huge and slow
  // to compile, for no speed that matters on the host
  __host__ __attribute__((noinline)) static Fp mul_host(const Fp& a, const Fp& b) {
    uint32_t t[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const Fp p = modulus();
    for (int i = 0; i < 8; ++i) {
      uint64_t c = 0;
      for (int j = 0; j < 8; ++j) {
        uint64_t s = (uint64_t)a.v[j] * b.v[i] + t[j] + c;
        t[j] = (uint32_t)s;
        c = s >> 32;
      }
      uint64_t s = (uint64_t)t[8] + c;
      t[8] = (uint32_t)s;
      t[9] = (uint32_t)(s >> 32);
      uint32_t m = t[0] * C::inv;
      s = (uint64_t)m * p.v[0] + t[0];
      c = s >> 32;
      for (int j = 1; j < 8; ++j) {
        s = (uint64_t)m * p.v[j] + t[j] + c;
        t[j - 1] = (uint32_t)s;
        c = s >> 32;
      }
      s = (uint64_t)t[8] + c;
      t[7] = (uint32_t)s;
      t[8] = t[9] + (uint32_t)(s >> 32);
    }
    Fp r;
    for (int i = 0; i < 8; ++i) r.v[i] = t[i];
    Fp d;
    uint32_t borrow = sub_raw(d, r, p);
    return (t[8] == 0 && borrow) ? r : d;
  }
#endif

  // two independent products r1 = a*b, r2 = c*d with their CIOS rows
  // interleaved: the two carry chains have no data dependence, so either
  // fills the other's multiply latency.
  ZG_HD static void mul2(const Fp& a, const Fp& b, const Fp& c, const Fp& d, Fp& r1, Fp& r2) {
#ifdef __CUDA_ARCH__
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0, t8 = 0;
    uint32_t u0 = 0, u1 = 0, u2 = 0, u3 = 0, u4 = 0, u5 = 0, u6 = 0, u7 = 0, u8 = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      row_mac(t0, t1, t2, t3, t4, t5, t6, t7, t8, a, b.v[i]);
      row_mac(u0, u1, u2, u3, u4, u5, u6, u7, u8, c, d.v[i]);
      const uint32_t m = t0 * C::inv;
      const uint32_t n = u0 * C::inv;
      row_red(t0, t1, t2, t3, t4, t5, t6, t7, t8, m);
      row_red(u0, u1, u2, u3, u4, u5, u6, u7, u8, n);
      t0 = t1; t1 = t2; t2 = t3; t3 = t4; t4 = t5; t5 = t6; t6 = t7; t7 = t8;
      u0 = u1; u1 = u2; u2 = u3; u3 = u4; u4 = u5; u5 = u6; u6 = u7; u7 = u8;
    }
    Fp x, y;
    x.v[0] = t0; x.v[1] = t1; x.v[2] = t2; x.v[3] = t3; x.v[4] = t4; x.v[5] = t5; x.v[6] = t6; x.v[7] = t7;
    y.v[0] = u0; y.v[1] = u1; y.v[2] = u2; y.v[3] = u3; y.v[4] = u4; y.v[5] = u5; y.v[6] = u6; y.v[7] = u7;
    Fp xs, ys;
    uint32_t bx = sub_raw(xs, x, modulus());
    uint32_t by = sub_raw(ys, y, modulus());
    r1 = bx ? x : xs;
    r2 = by ? y : ys;
#else
    Fp x = mul(a, b), y = mul(c, d);
    r1 = x;
    r2 = y;
#endif
  }

#ifdef __CUDA_ARCH__
  // t[0..8] = t[0..7] + a * bi (even limbs chain, then odd limbs chain)
  __device__ __forceinline__ static void row_mac(uint32_t& t0, uint32_t& t1, uint32_t& t2, uint32_t& t3,
                                                 uint32_t& t4, uint32_t& t5, uint32_t& t6, uint32_t& t7,
                                                 uint32_t& t8, const Fp& a, uint32_t bi) {
    asm("mad.lo.cc.u32 %0, %9, %17, %0;\n\t"
        "madc.hi.cc.u32 %1, %9, %17, %1;\n\t"
        "madc.lo.cc.u32 %2, %11, %17, %2;\n\t"
        "madc.hi.cc.u32 %3, %11, %17, %3;\n\t"
        "madc.lo.cc.u32 %4, %13, %17, %4;\n\t"
        "madc.hi.cc.u32 %5, %13, %17, %5;\n\t"
        "madc.lo.cc.u32 %6, %15, %17, %6;\n\t"
        "madc.hi.cc.u32 %7, %15, %17, %7;\n\t"
        "addc.u32 %8, 0, 0;\n\t"
        "mad.lo.cc.u32 %1, %10, %17, %1;\n\t"
        "madc.hi.cc.u32 %2, %10, %17, %2;\n\t"
        "madc.lo.cc.u32 %3, %12, %17, %3;\n\t"
        "madc.hi.cc.u32 %4, %12, %17, %4;\n\t"
        "madc.lo.cc.u32 %5, %14, %17, %5;\n\t"
        "madc.hi.cc.u32 %6, %14, %17, %6;\n\t"
        "madc.lo.cc.u32 %7, %16, %17, %7;\n\t"
        "madc.hi.u32 %8, %16, %17, %8;"
        : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8)
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]), "r"(a.v[6]),
          "r"(a.v[7]), "r"(bi));
  }
  // t[0..8] += m * p
  __device__ __forceinline__ static void row_red(uint32_t& t0, uint32_t& t1, uint32_t& t2, uint32_t& t3,
                                                 uint32_t& t4, uint32_t& t5, uint32_t& t6, uint32_t& t7,
                                                 uint32_t& t8, uint32_t m) {
    asm("mad.lo.cc.u32 %0, %9, %10, %0;\n\t"
        "madc.hi.cc.u32 %1, %9, %10, %1;\n\t"
        "madc.lo.cc.u32 %2, %9, %12, %2;\n\t"
        "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"
        "madc.lo.cc.u32 %4, %9, %14, %4;\n\t"
        "madc.hi.cc.u32 %5, %9, %14, %5;\n\t"
        "madc.lo.cc.u32 %6, %9, %16, %6;\n\t"
        "madc.hi.cc.u32 %7, %9, %16, %7;\n\t"
        "addc.u32 %8, %8, 0;\n\t"
        "mad.lo.cc.u32 %1, %9, %11, %1;\n\t"
        "madc.hi.cc.u32 %2, %9, %11, %2;\n\t"
        "madc.lo.cc.u32 %3, %9, %13, %3;\n\t"
        "madc.hi.cc.u32 %4, %9, %13, %4;\n\t"
        "madc.lo.cc.u32 %5, %9, %15, %5;\n\t"
        "madc.hi.cc.u32 %6, %9, %15, %6;\n\t"
        "madc.lo.cc.u32 %7, %9, %17, %7;\n\t"
        "madc.hi.u32 %8, %9, %17, %8;"
        : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7), "+r"(t8)
        : "r"(m), "r"(C::p0), "r"(C::p1), "r"(C::p2), "r"(C::p3), "r"(C::p4), "r"(C::p5), "r"(C::p6),
          "r"(C::p7));
  }
#endif

  // canonical (< p) -> Montgomery
  ZG_HD static Fp from_canonical(const Fp& a) { return mul(a, r2()); }
  // Montgomery -> canonical
  ZG_HD Fp to_canonical() const {
    Fp one_raw = zero();
    one_raw.v[0] = 1;
    return mul(*this, one_raw);
  }
  ZG_HD static Fp from_u32(uint32_t x) {
    Fp a = zero();
    a.v[0] = x;
    return from_canonical(a);
  }
  // a^e for a little-endian exponent of n 32-bit words
  ZG_HD Fp pow(const uint32_t* e, int n) const {
    Fp r = one(), b = *this;
    for (int i = 0; i < n; ++i) {
      uint32_t w = e[i];
      for (int k = 0; k < 32; ++k) {
        if (w & 1) r = mul(r, b);
        b = mul(b, b);
        w >>= 1;
      }
    }
    return r;
  }
  ZG_HD Fp pow_u64(uint64_t e) const {
    uint32_t w[2] = {(uint32_t)e, (uint32_t)(e >> 32)};
    return pow(w, 2);
  }
  // Fermat inverse; inverse(0) = 0
  ZG_HD Fp inverse() const {
    uint32_t e[8] = {C::p0 - 2, C::p1, C::p2, C::p3, C::p4, C::p5, C::p6, C::p7};
    return pow(e, 8);
  }
  // canonical value > (p-1)/2, i.e. ark's "y > -y" (SWFlags::YIsNegative)
  ZG_HD bool canonical_is_negative() const {
    Fp c = to_canonical();
    Fp d = neg(c);  // canonical of -y as integer
    // compare c > d as integers
    for (int i = 7; i >= 0; --i)
      if (c.v[i] != d.v[i]) return c.v[i] > d.v[i];
    return false;
  }
};

typedef Fp<FqCfg> Fq;
typedef Fp<FrCfg> Fr;

}  // namespace zg
