// ORACLE — test infrastructure only (see zgo_field.hpp / zgo_encoder.hpp).
#include "zgo_encoder.hpp"

#include <algorithm>
#include <cassert>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace zgo {

// ---------------------------------------------------------------------------
// crates/amt/src/utils.rs:54-64
size_t bitreverse(size_t n, int l) {
  size_t r = 0;
  for (int i = 0; i < l; ++i) r = (r << 1) | ((n >> i) & 1);
  return r;
}
size_t swap_bits(size_t n, int lo, int hi) {
  size_t lowest = n & ((size_t(1) << lo) - 1);
  size_t next = (n >> lo) & ((size_t(1) << hi) - 1);
  return (lowest << hi) | next;
}

static int log2_exact(size_t n) {
  int l = 0;
  while ((size_t(1) << l) < n) ++l;
  return l;
}

// ---------------------------------------------------------------------------
// Radix-2 DFT over Fr: out[k] = sum_j in[j] omega^{jk} (ark-poly
// Radix2EvaluationDomain::fft / ifft semantics, inputs zero-padded to the
// domain size).
void fr_ntt_omega(std::vector<Fr>& a, const Fr& omega) {
  size_t n = a.size();
  int l = log2_exact(n);
  for (size_t i = 0; i < n; ++i) {
    size_t j = bitreverse(i, l);
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    Fr wl = omega;
    for (size_t k = len; k < n; k <<= 1) wl = wl.sqr();
    size_t half = len / 2;
    std::vector<Fr> tw(half);
    tw[0] = Fr::one();
    for (size_t k = 1; k < half; ++k) tw[k] = tw[k - 1] * wl;
#pragma omp parallel for schedule(static) if (n >= 4096)
    for (size_t i = 0; i < n; i += len) {
      for (size_t k = 0; k < half; ++k) {
        Fr u = a[i + k], v = a[i + k + half] * tw[k];
        a[i + k] = u + v;
        a[i + k + half] = u - v;
      }
    }
  }
}
static size_t next_pow2(size_t n) {
  size_t p = 1;
  while (p < n) p <<= 1;
  return p;
}
void fr_fft(std::vector<Fr>& a) {
  size_t n = next_pow2(std::max<size_t>(a.size(), 1));
  a.resize(n, Fr::zero());
  fr_ntt_omega(a, fr_root_of_unity(log2_exact(n)));
}
void fr_ifft(std::vector<Fr>& a) {
  size_t n = next_pow2(std::max<size_t>(a.size(), 1));
  a.resize(n, Fr::zero());
  fr_ntt_omega(a, fr_root_of_unity(log2_exact(n)).inverse());
  Fr ninv = Fr::from_u64(n).inverse();
  for (auto& x : a) x *= ninv;
}

// crates/amt/src/prove_params/generate.rs:128-137
Fr coset_factor(size_t length, size_t idx) {
  int depth = log2_exact(length);
  int rest = FR_TWO_ADICITY - depth;
  u64 pow = bitreverse(idx, rest);
  return fr_two_adic_root().pow_u64(pow);
}

// group NTT used by the EC-domain param restatement (generate.rs:197-263)
template <class F>
static void group_ntt(std::vector<Jac<F>>& a, const Fr& omega) {
  size_t n = a.size();
  int l = log2_exact(n);
  for (size_t i = 0; i < n; ++i) {
    size_t j = bitreverse(i, l);
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    Fr wl = omega;
    for (size_t k = len; k < n; k <<= 1) wl = wl.sqr();
    size_t half = len / 2;
    std::vector<BigInt> tw(half);
    Fr t = Fr::one();
    for (size_t k = 0; k < half; ++k) { tw[k] = t.to_bigint(); t *= wl; }
#pragma omp parallel for schedule(dynamic)
    for (size_t idx = 0; idx < n / 2; ++idx) {
      size_t i = (idx / half) * len, k = idx % half;
      Jac<F> u = a[i + k], v = a[i + k + half].mul(tw[k]);
      a[i + k] = u.add(v);
      a[i + k + half] = u.add(v.neg());
    }
  }
}
template <class F>
static void group_scale(std::vector<Jac<F>>& a, const Fr& s) {
  BigInt b = s.to_bigint();
#pragma omp parallel for schedule(dynamic)
  for (size_t i = 0; i < a.size(); ++i) a[i] = a[i].mul(b);
}

template <class F>
static std::vector<Affine<F>> enact(std::vector<Jac<F>>& in) {
  std::vector<Affine<F>> out(in.size());
  normalize_batch(in.data(), out.data(), in.size());
  index_reverse(out);
  return out;
}

// ---------------------------------------------------------------------------
// Seeded tau: the reference draws tau from thread_rng (power_tau.rs:58); this
// build fixes tau = (w0 + w1 2^64 + ... + w7 2^448) mod r, w_i the SplitMix64
// stream started at `seed`.
static uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
Fr tau_from_seed(uint64_t seed) {
  uint64_t s = seed;
  uint64_t w[8];
  for (int i = 0; i < 8; ++i) w[i] = splitmix64(s);
  // value = lo + hi * 2^256 (mod r); each 256-bit half reduced by subtraction
  auto reduce = [](const uint64_t* x) {
    u64 t[4];
    memcpy(t, x, 32);
    while (big_geq(t, FrCfg::P)) big_sub(t, t, FrCfg::P);
    BigInt b; memcpy(b.v, t, 32);
    return Fr::from_bigint(b);
  };
  Fr lo = reduce(w), hi = reduce(w + 4);
  // 2^256 mod r: its canonical integer equals the Montgomery limbs of one
  BigInt rb;
  memcpy(rb.v, Fr::one().v, 32);
  Fr two256 = Fr::from_bigint(rb);
  return lo + hi * two256;
}

// crates/amt/src/power_tau.rs:28-80
PowerTau power_tau_setup(const Fr& tau, int depth) {
  size_t n = size_t(1) << depth;
  size_t high_start = (size_t(1) << (depth + 2)) - n;
  FixedBase<Fq> fb1(g1_generator());
  FixedBase<Fq2> fb2(g2_generator());
  std::vector<Fr> pw(n);
  pw[0] = Fr::one();
  for (size_t i = 1; i < n; ++i) pw[i] = pw[i - 1] * tau;
  Fr ths = tau.pow_u64(high_start);
  std::vector<G1J> g1(n), hg1(n);
  std::vector<G2J> g2(n);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) {
    g1[i] = fb1.mul(pw[i]);
    hg1[i] = fb1.mul(pw[i] * ths);
    g2[i] = fb2.mul(pw[i]);
  }
  PowerTau pp;
  pp.g1pp.resize(n); pp.high_g1pp.resize(n); pp.g2pp.resize(n);
  normalize_batch(g1.data(), pp.g1pp.data(), n);
  normalize_batch(hg1.data(), pp.high_g1pp.data(), n);
  normalize_batch(g2.data(), pp.g2pp.data(), n);
  pp.high_g2 = fb2.mul(ths).to_affine();
  return pp;
}

// crates/amt/src/prove_params/generate.rs:139-263, EC domain (G1/G2 FFTs).
AMTParams amt_from_pp_ec(const PowerTau& pp, int prove_depth, int coset) {
  size_t length = pp.g1pp.size();
  int depth = log2_exact(length);
  std::vector<G1J> g1pp(length), hg1pp(length);
  std::vector<G2J> g2pp(length);
  for (size_t i = 0; i < length; ++i) {
    g1pp[i] = G1J::from_affine(pp.g1pp[i]);
    hg1pp[i] = G1J::from_affine(pp.high_g1pp[i]);
    g2pp[i] = G2J::from_affine(pp.g2pp[i]);
  }
  G2J hg2 = G2J::from_affine(pp.high_g2);
  if (coset > 0) {
    Fr w = coset_factor(length, coset).inverse();
#pragma omp parallel for schedule(dynamic)
    for (size_t i = 0; i < length; ++i) {
      BigInt e = w.pow_u64(i).to_bigint();
      g1pp[i] = g1pp[i].mul(e);
      g2pp[i] = g2pp[i].mul(e);
      hg1pp[i] = hg1pp[i].mul(e);
    }
  }
  Fr omega = fr_root_of_unity(depth);
  Fr size_inv = Fr::from_u64(length).inverse();
  AMTParams p;
  p.depth = depth;
  p.prove_depth = prove_depth;
  // basis = ifft(g1pp)
  {
    std::vector<G1J> b = g1pp;
    group_ntt(b, omega.inverse());
    group_scale(b, size_inv);
    p.basis = enact(b);
  }
  for (int d = 1; d <= prove_depth; ++d) {
    size_t max_coeff = size_t(1) << (depth - d);
    std::vector<G1J> coeff(length, G1J::inf());
    for (size_t i = 1; i <= max_coeff; ++i) coeff[i] = g1pp[max_coeff - i];
    group_ntt(coeff, omega);
    group_scale(coeff, size_inv);
    p.quotients.push_back(enact(coeff));
  }
  for (int d = 1; d <= prove_depth; ++d) {
    size_t step = size_t(1) << (depth - d);
    size_t sz = size_t(1) << d;
    std::vector<G2J> coeff(sz, G2J::inf());
    coeff[0] = g2pp[length - step];
    for (size_t i = 1; i < length / step; ++i) coeff[i] = g2pp[(i - 1) * step];
    group_ntt(coeff, fr_root_of_unity(d).inverse());  // group_gen <-> group_gen_inv
    p.vanishes.push_back(enact(coeff));
  }
  {
    std::vector<G1J> b = hg1pp;
    group_ntt(b, omega.inverse());
    group_scale(b, size_inv);
    p.high_basis = enact(b);
  }
  p.g2 = g2pp[0].to_affine();
  p.high_g2 = hg2.to_affine();
  return p;
}

// Scalar-domain twin of amt_from_pp_ec: with tau known, every param point is
// s * G; the scalars follow the same FFT formulas over Fr.
AMTScalars amt_scalars(const Fr& tau, int depth, int prove_depth, int coset) {
  size_t length = size_t(1) << depth;
  size_t high_start = (size_t(1) << (depth + 2)) - length;
  Fr w = coset > 0 ? coset_factor(length, coset).inverse() : Fr::one();
  Fr tp = tau * w;
  std::vector<Fr> pw(length);
  pw[0] = Fr::one();
  for (size_t i = 1; i < length; ++i) pw[i] = pw[i - 1] * tp;
  Fr ths = tau.pow_u64(high_start);
  AMTScalars s;
  s.basis = pw;
  fr_ifft(s.basis);
  s.high_basis.resize(length);
  for (size_t i = 0; i < length; ++i) s.high_basis[i] = s.basis[i] * ths;
  index_reverse(s.basis);
  index_reverse(s.high_basis);
  Fr size_inv = Fr::from_u64(length).inverse();
  s.quotients.resize(prove_depth);
#pragma omp parallel for schedule(dynamic)
  for (int d = 1; d <= prove_depth; ++d) {
    size_t max_coeff = size_t(1) << (depth - d);
    std::vector<Fr> coeff(length, Fr::zero());
    for (size_t i = 1; i <= max_coeff; ++i) coeff[i] = pw[max_coeff - i];
    fr_ntt_omega(coeff, fr_root_of_unity(depth));
    for (auto& x : coeff) x *= size_inv;
    index_reverse(coeff);
    s.quotients[d - 1] = coeff;
  }
  for (int d = 1; d <= prove_depth; ++d) {
    size_t step = size_t(1) << (depth - d);
    size_t sz = size_t(1) << d;
    std::vector<Fr> coeff(sz, Fr::zero());
    coeff[0] = pw[length - step];
    for (size_t i = 1; i < length / step; ++i) coeff[i] = pw[(i - 1) * step];
    fr_ntt_omega(coeff, fr_root_of_unity(d).inverse());
    index_reverse(coeff);
    s.vanishes.push_back(coeff);
  }
  s.high_g2 = ths;
  return s;
}

AMTParams amt_from_scalars(const AMTScalars& s, int depth, int prove_depth) {
  static FixedBase<Fq>* fb1 = nullptr;
  static FixedBase<Fq2>* fb2 = nullptr;
#pragma omp critical(zgo_fixed_base)
  {
    if (!fb1) fb1 = new FixedBase<Fq>(g1_generator());
    if (!fb2) fb2 = new FixedBase<Fq2>(g2_generator());
  }
  auto g1line = [&](const std::vector<Fr>& sc) {
    std::vector<G1J> j(sc.size());
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < sc.size(); ++i) j[i] = fb1->mul(sc[i]);
    std::vector<G1A> a(sc.size());
    normalize_batch(j.data(), a.data(), j.size());
    return a;
  };
  auto g2line = [&](const std::vector<Fr>& sc) {
    std::vector<G2J> j(sc.size());
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < sc.size(); ++i) j[i] = fb2->mul(sc[i]);
    std::vector<G2A> a(sc.size());
    normalize_batch(j.data(), a.data(), j.size());
    return a;
  };
  AMTParams p;
  p.depth = depth;
  p.prove_depth = prove_depth;
  p.basis = g1line(s.basis);
  for (auto& q : s.quotients) p.quotients.push_back(g1line(q));
  for (auto& v : s.vanishes) p.vanishes.push_back(g2line(v));
  p.high_basis = g1line(s.high_basis);
  p.g2 = g2_generator();
  p.high_g2 = fb2->mul(s.high_g2).to_affine();
  return p;
}

// ---------------------------------------------------------------------------
// mont file format, crates/amt/src/prove_params/fast_serde_bn254.rs:20-88
static void put_raw(const u64 v[4], std::vector<uint8_t>& out) {
  const uint8_t* b = reinterpret_cast<const uint8_t*>(v);
  out.insert(out.end(), b, b + 32);
}
void ser_g1(const G1A& p, std::vector<uint8_t>& out) {
  uint8_t buf[64];
  if (p.inf) {
    memset(buf, 0, 64);
    buf[63] |= 0x40;
  } else {
    p.x.to_le_bytes(buf);
    p.y.to_le_bytes(buf + 32);
    if ((-p.y).canon_gt(p.y) || p.y == -p.y) {
      // YIsPositive: y <= -y
    } else {
      buf[63] |= 0x80;
    }
  }
  out.insert(out.end(), buf, buf + 64);
}
void ser_g2(const G2A& p, std::vector<uint8_t>& out) {
  uint8_t buf[128];
  if (p.inf) {
    memset(buf, 0, 128);
    buf[127] |= 0x40;
  } else {
    p.x.c0.to_le_bytes(buf);
    p.x.c1.to_le_bytes(buf + 32);
    p.y.c0.to_le_bytes(buf + 64);
    p.y.c1.to_le_bytes(buf + 96);
    Fq2 ny = -p.y;
    if (!(ny.canon_gt(p.y) || ny == p.y)) buf[127] |= 0x80;
  }
  out.insert(out.end(), buf, buf + 128);
}
void write_amt_params_mont(const AMTParams& p, std::vector<uint8_t>& out) {
  out.clear();
  out.insert(out.end(), {'b', 'a', 'm', 't'});
  out.push_back((uint8_t)log2_exact(p.basis.size()));
  out.push_back((uint8_t)p.quotients.size());
  ser_g2(p.g2, out);
  ser_g2(p.high_g2, out);
  auto g1raw = [&](const G1A& a) { put_raw(a.x.v, out); put_raw(a.y.v, out); };
  auto g2raw = [&](const G2A& a) {
    put_raw(a.x.c0.v, out); put_raw(a.x.c1.v, out);
    put_raw(a.y.c0.v, out); put_raw(a.y.c1.v, out);
  };
  for (auto& b : p.basis) g1raw(b);
  for (auto& l : p.quotients) for (auto& b : l) g1raw(b);
  for (auto& l : p.vanishes) for (auto& b : l) g2raw(b);
  for (auto& b : p.high_basis) g1raw(b);
}
static bool de_fq(const uint8_t*& p, const uint8_t* end, Fq* out, uint8_t* flags) {
  if (end - p < 32) return false;
  uint8_t b[32];
  memcpy(b, p, 32);
  p += 32;
  if (flags) {
    *flags = b[31] >> 6;
    b[31] &= 0x3f;
  }
  return Fq::from_le_bytes(b, out);
}
static bool de_g2(const uint8_t*& p, const uint8_t* end, G2A* out) {
  Fq x0, x1, y0, y1;
  uint8_t fl;
  if (!de_fq(p, end, &x0, nullptr) || !de_fq(p, end, &x1, nullptr) ||
      !de_fq(p, end, &y0, nullptr) || !de_fq(p, end, &y1, &fl))
    return false;
  if (fl == 3) return false;
  if (fl == 1) { *out = {Fq2::zero(), Fq2::zero(), true}; return true; }
  *out = {{x0, x1}, {y0, y1}, false};
  return g2_on_curve(*out);
}
bool de_g1(const uint8_t*& p, const uint8_t* end, G1A* out) {
  Fq x, y;
  uint8_t fl;
  if (!de_fq(p, end, &x, nullptr) || !de_fq(p, end, &y, &fl)) return false;
  if (fl == 3) return false;
  if (fl == 1) { *out = {Fq::zero(), Fq::zero(), true}; return true; }
  *out = {x, y, false};
  return g1_on_curve(*out);
}
bool read_amt_params_mont(const uint8_t* in, size_t len, AMTParams* out) {
  const uint8_t* p = in;
  const uint8_t* end = in + len;
  if (len < 6 || memcmp(p, "bamt", 4) != 0) return false;
  p += 4;
  int degree = *p++;
  int sub = *p++;
  if (!de_g2(p, end, &out->g2) || !de_g2(p, end, &out->high_g2)) return false;
  size_t n = size_t(1) << degree;
  auto g1line = [&](std::vector<G1A>& v, size_t cnt) {
    if ((size_t)(end - p) < cnt * 64) return false;
    v.resize(cnt);
    for (size_t i = 0; i < cnt; ++i) {
      u64 x[4], y[4];
      memcpy(x, p, 32); memcpy(y, p + 32, 32);
      p += 64;
      v[i] = {Fq::from_raw_mont(x), Fq::from_raw_mont(y), false};
    }
    return true;
  };
  if (!g1line(out->basis, n)) return false;
  out->quotients.assign(sub, {});
  for (int d = 0; d < sub; ++d) if (!g1line(out->quotients[d], n)) return false;
  out->vanishes.assign(sub, {});
  for (int d = 0; d < sub; ++d) {
    size_t cnt = size_t(1) << (d + 1);
    if ((size_t)(end - p) < cnt * 128) return false;
    out->vanishes[d].resize(cnt);
    for (size_t i = 0; i < cnt; ++i) {
      u64 a[4], b[4], c[4], e[4];
      memcpy(a, p, 32); memcpy(b, p + 32, 32); memcpy(c, p + 64, 32); memcpy(e, p + 96, 32);
      p += 128;
      out->vanishes[d][i] = {{Fq::from_raw_mont(a), Fq::from_raw_mont(b)},
                             {Fq::from_raw_mont(c), Fq::from_raw_mont(e)}, false};
    }
  }
  if (!g1line(out->high_basis, n)) return false;
  out->depth = degree;
  out->prove_depth = sub;
  return true;
}

// ---------------------------------------------------------------------------
// crates/encoder/src/raw_data.rs:55-73
bool raw_data_from_bytes(const Dims& d, const uint8_t* in, size_t len, std::vector<uint8_t>* out) {
  if (len > d.max_raw()) return false;
  out->assign(d.max_blob(), 0);
  if (len) memcpy(out->data(), in, len);
  uint32_t l32 = (uint32_t)len;
  memcpy(out->data() + d.max_raw(), &l32, 4);
  return true;
}
// crates/encoder/src/raw_blob.rs:33-40 + utils.rs:10-15
std::vector<Fr> raw_blob_from_raw_data(const Dims& d, const std::vector<uint8_t>& raw) {
  std::vector<Fr> out(d.n());
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < d.n(); ++i) {
    BigInt b = {{0, 0, 0, 0}};
    memcpy(b.v, raw.data() + RAW_UNIT * i, RAW_UNIT);
    out[i] = Fr::from_bigint(b);
  }
  return out;
}
H256 scalar_to_h256(const Fr& x) {
  H256 h;
  x.to_le_bytes(h.data());
  return h;
}

// crates/amt/src/blob/encode.rs:135-158
std::vector<Fr> to_coset_blob(const std::vector<Fr>& data, size_t coset) {
  if (coset == 0) return data;
  Fr g = coset_factor(data.size(), coset);
  std::vector<Fr> coeff = data;
  fr_ifft(coeff);
  Fr base = Fr::one();
  for (auto& x : coeff) { x *= base; base *= g; }
  fr_fft(coeff);
  return coeff;
}

std::vector<BigInt> to_bigints(const Fr* s, size_t n) {
  std::vector<BigInt> out(n);
  for (size_t i = 0; i < n; ++i) out[i] = s[i].to_bigint();
  return out;
}

// crates/amt/src/prove_params/prove.rs:20-102 (the CPU plugin of AMTProofs).
// The reference maps over a layer's MSMs one after the other and each MSM
// runs its windows in parallel (ark-ec's `parallel` feature); so does this
// restatement, except that MSMs of fewer than 256 points (test shapes only:
// a layer's MSMs hold at least 1024 points at the production shape) run side
// by side instead, since their windows are too small to split.
AllProofs gen_all_proofs(const AMTParams& amt, const std::vector<Fr>& ri, G1J* commitment) {
  size_t len = amt.len();
  size_t batch = len / (size_t(1) << amt.quotients.size());
  std::vector<BigInt> sc = to_bigints(ri.data(), ri.size());
  AllProofs ap;
  ap.input_len = len;
  ap.batch_size = batch;
  int last_depth = log2_exact(len / batch);
  for (int depth = 1; depth <= last_depth; ++depth) {
    size_t items = size_t(1) << depth;
    size_t chunk = len / items;
    std::vector<G1J> q(items);
#pragma omp parallel for schedule(dynamic) if (chunk < 256)
    for (size_t k = 0; k < items; ++k)
      q[k] = msm(amt.quotients[depth - 1].data() + k * chunk, sc.data() + k * chunk, chunk);
    std::vector<G1A> qa(items);
    normalize_batch(q.data(), qa.data(), items);
    ap.proofs.push_back(qa);
  }
  // gen_commitment_tree + build_commitment_tree
  size_t nb = len / batch;
  std::vector<G1J> last(nb);
#pragma omp parallel for schedule(dynamic) if (batch < 256)
  for (size_t k = 0; k < nb; ++k) last[k] = msm(amt.basis.data() + k * batch, sc.data() + k * batch, batch);
  std::vector<G1A> layer(nb);
  normalize_batch(last.data(), layer.data(), nb);
  std::vector<std::vector<G1A>> rev;
  while (layer.size() > 1) {
    std::vector<G1J> next(layer.size() / 2);
    for (size_t i = 0; i < next.size(); ++i)
      next[i] = G1J::from_affine(layer[2 * i]).add_affine(layer[2 * i + 1]);
    std::vector<G1A> na(next.size());
    normalize_batch(next.data(), na.data(), next.size());
    rev.push_back(layer);
    layer = na;
  }
  *commitment = G1J::from_affine(layer[0]);
  ap.commitments.assign(rev.rbegin(), rev.rend());
  G1J high = msm(amt.high_basis.data(), sc.data(), len);
  ap.high_commitment = high.to_affine();
  return ap;
}

// crates/amt/src/blob/encode.rs:171-183
HalfBlob half_blob_generate(const Dims& d, std::vector<Fr> points, const AMTParams& amt) {
  index_reverse(points);
  G1J c;
  HalfBlob hb;
  hb.proofs = gen_all_proofs(amt, points, &c);
  index_reverse(points);
  change_matrix_direction(points, d.log_row, d.log_col);
  hb.blob = points;
  hb.commitment = c.to_affine();
  return hb;
}

static void keccak_chunked(const std::vector<H256>& in, size_t chunk, std::vector<H256>& out) {
  out.resize(in.size() / chunk);
#pragma omp parallel for schedule(static) if (in.size() > 4096)
  for (size_t i = 0; i < out.size(); ++i)
    keccak256(in[i * chunk].data(), 32 * chunk, out[i].data());
}

// crates/encoder/src/merkle/blob.rs:15-34
Merkle merkle_build(const Dims& d, std::vector<H256> data) {
  Merkle m;
  std::vector<H256> last;
  keccak_chunked(data, 8, last);
  std::vector<std::vector<H256>> rev;
  while (last.size() > (size_t)COSET_N) {
    std::vector<H256> next;
    keccak_chunked(last, 2, next);
    rev.push_back(last);
    last = next;
  }
  rev.push_back(last);
  m.tree.assign(rev.rbegin(), rev.rend());
  m.data = std::move(data);
  (void)d;
  return m;
}

H256 compute_file_root(const H256 roots[COSET_N]) {
  uint8_t buf[64];
  H256 t, r;
  memcpy(buf, roots[0].data(), 32);
  memcpy(buf + 32, roots[1].data(), 32);
  keccak256(buf, 64, t.data());
  memcpy(buf, t.data(), 32);
  memcpy(buf + 32, roots[2].data(), 32);
  keccak256(buf, 64, r.data());
  return r;
}

// crates/encoder/src/encoder/blob.rs:32-42, amt/blob.rs:19-27, encode.rs:91-108
void encoded_blob_build(const Dims& d, const std::vector<Fr>& raw_blob, const AMTParams* amt,
                        EncodedBlob* out) {
  out->dims = d;
  std::vector<Fr> points = raw_blob;
  change_matrix_direction(points, d.log_col, d.log_row);
  for (int c = 0; c < COSET_N; ++c)
    out->halves[c] = half_blob_generate(d, to_coset_blob(points, c), amt[c]);
  for (int c = 1; c < COSET_N; ++c)
    if (out->halves[c].commitment != out->halves[0].commitment) abort();  // assert_commitment_consistent
  std::vector<H256> data(COSET_N * d.n());
  for (int c = 0; c < COSET_N; ++c)
    for (size_t i = 0; i < d.n(); ++i) data[c * d.n() + i] = scalar_to_h256(out->halves[c].blob[i]);
  out->merkle = merkle_build(d, std::move(data));
}

// encoder/blob.rs:44-49 -> amt/blob.rs:49-57, encode.rs:185-200, proofs.rs:17-30,
// merkle/blob.rs:44-57
EncodedSlice encoded_blob_get_row(const EncodedBlob& b, size_t index) {
  const Dims& d = b.dims;
  EncodedSlice s;
  s.index = index;
  size_t coset = index / d.rows(), local = index % d.rows();
  const HalfBlob& hb = b.halves[coset];
  s.amt.index = index;
  s.amt.commitment = hb.commitment;
  s.amt.row.index = local;
  s.amt.row.row.assign(hb.blob.begin() + local * d.cols(), hb.blob.begin() + (local + 1) * d.cols());
  size_t rev = bitreverse(local, d.log_row);
  int bits = (int)hb.proofs.commitments.size();
  for (int dd = 0; dd < bits; ++dd) {
    size_t lv = rev >> (bits - 1 - dd);
    s.amt.row.proof.v.push_back({hb.proofs.commitments[dd][lv ^ 1], hb.proofs.proofs[dd][lv ^ 1]});
  }
  s.amt.row.high_commitment = hb.proofs.high_commitment;
  for (int c = 0; c < COSET_N; ++c) s.merkle.root[c] = b.merkle.tree[0][c];
  for (int dd = d.log_row; dd >= 1; --dd) {
    size_t height = d.log_row - dd;
    size_t idx = index >> height;
    s.merkle.proof.push_back(b.merkle.tree[dd][idx ^ 1]);
  }
  s.merkle.leaf_index = index;
  s.merkle.leaf = b.merkle.tree[d.log_row][index];
  return s;
}

// ---------------------------------------------------------------------------
// ark-serialize 0.4 derive(CanonicalSerialize), uncompressed
static void put_u64(uint64_t v, std::vector<uint8_t>& out) {
  const uint8_t* b = reinterpret_cast<const uint8_t*>(&v);
  out.insert(out.end(), b, b + 8);
}
void serialize_slice(const EncodedSlice& s, std::vector<uint8_t>& out) {
  out.clear();
  put_u64(s.index, out);
  put_u64(s.amt.index, out);
  ser_g1(s.amt.commitment, out);
  put_u64(s.amt.row.index, out);
  put_u64(s.amt.row.row.size(), out);
  for (auto& x : s.amt.row.row) {
    uint8_t b[32];
    x.to_le_bytes(b);
    out.insert(out.end(), b, b + 32);
  }
  put_u64(s.amt.row.proof.v.size(), out);
  for (auto& pr : s.amt.row.proof.v) { ser_g1(pr.first, out); ser_g1(pr.second, out); }
  ser_g1(s.amt.row.high_commitment, out);
  for (int c = 0; c < COSET_N; ++c) out.insert(out.end(), s.merkle.root[c].begin(), s.merkle.root[c].end());
  put_u64(s.merkle.proof.size(), out);
  for (auto& h : s.merkle.proof) out.insert(out.end(), h.begin(), h.end());
  put_u64(s.merkle.leaf_index, out);
  out.insert(out.end(), s.merkle.leaf.begin(), s.merkle.leaf.end());
}
static bool get_u64(const uint8_t*& p, const uint8_t* end, uint64_t* v) {
  if (end - p < 8) return false;
  memcpy(v, p, 8);
  p += 8;
  return true;
}
static bool get_h256(const uint8_t*& p, const uint8_t* end, H256* h) {
  if (end - p < 32) return false;
  memcpy(h->data(), p, 32);
  p += 32;
  return true;
}
bool deserialize_slice(const uint8_t* in, size_t len, EncodedSlice* s) {
  const uint8_t* p = in;
  const uint8_t* end = in + len;
  uint64_t n;
  if (!get_u64(p, end, &s->index) || !get_u64(p, end, &s->amt.index) || !de_g1(p, end, &s->amt.commitment) ||
      !get_u64(p, end, &s->amt.row.index) || !get_u64(p, end, &n))
    return false;
  if (n > (uint64_t)(end - p) / 32) return false;
  s->amt.row.row.resize(n);
  for (uint64_t i = 0; i < n; ++i) {
    if (!Fr::from_le_bytes(p, &s->amt.row.row[i])) return false;
    p += 32;
  }
  if (!get_u64(p, end, &n) || n > (uint64_t)(end - p) / 128) return false;
  s->amt.row.proof.v.resize(n);
  for (uint64_t i = 0; i < n; ++i)
    if (!de_g1(p, end, &s->amt.row.proof.v[i].first) || !de_g1(p, end, &s->amt.row.proof.v[i].second)) return false;
  if (!de_g1(p, end, &s->amt.row.high_commitment)) return false;
  for (int c = 0; c < COSET_N; ++c)
    if (!get_h256(p, end, &s->merkle.root[c])) return false;
  if (!get_u64(p, end, &n) || n > (uint64_t)(end - p) / 32) return false;
  s->merkle.proof.resize(n);
  for (uint64_t i = 0; i < n; ++i) get_h256(p, end, &s->merkle.proof[i]);
  if (!get_u64(p, end, &s->merkle.leaf_index) || !get_h256(p, end, &s->merkle.leaf)) return false;
  return p == end;
}

// ---------------------------------------------------------------------------
// Verification: encoder/slice.rs:73-95, amt/slice.rs:53-103, encode.rs:225-241,
// verify_params.rs:136-211, merkle/slice.rs:50-104.
enum {
  V_OK = 0,
  V_UNMATCHED_AMT_INDEX = 1,
  V_UNMATCHED_MERKLE_INDEX = 2,
  V_AMT_INCORRECT_COMMITMENT = 10,
  V_AMT_INCORRECT_ROW_SIZE = 11,
  V_AMT_ROW_INDEX_OVERFLOW = 12,
  V_AMT_UNMATCHED_COSET_INDEX = 13,
  V_AMT_INCORRECT_PROOF = 14,
  V_MERKLE_INCORRECT_ROOT = 20,
  V_MERKLE_INCORRECT_SIZE = 21,
  V_MERKLE_ROW_INDEX_OVERFLOW = 22,
  V_MERKLE_INCORRECT_LOCAL_ROOT = 23,
  V_MERKLE_INCORRECT_PROOF = 24,
};
enum { P_UNEXPECTED_DATA_LENGTH = 0, P_INCORRECT_POSITION = 1, P_KZG = 2, P_INCONSISTENT = 3, P_LDT = 4 };

static int verify_amt_proof(const AMTParams& amt, const std::vector<Fr>& data, size_t batch_index,
                            const Proof& proof, const G1A& commitment, const G1A& high, int64_t* kzg_d) {
  size_t depth = proof.v.size();
  if (depth >= 63) return P_UNEXPECTED_DATA_LENGTH;
  size_t num_batch = size_t(1) << depth;
  size_t batch = amt.basis.size() / num_batch;
  if (batch != data.size()) return P_UNEXPECTED_DATA_LENGTH;
  if (batch_index >= num_batch) return P_INCORRECT_POSITION;
  G1J acc = G1J::inf();
  for (size_t dd = depth; dd-- > 0;) {
    size_t vi = batch_index >> (depth - 1 - dd);
    const G2A& vanish = amt.vanishes[dd][vi ^ 1];
    if (!pairing_eq(proof.v[dd].first, amt.g2, proof.v[dd].second, vanish)) {
      *kzg_d = (int64_t)dd;
      return P_KZG;
    }
    acc = acc.add_affine(proof.v[dd].first);
  }
  std::vector<BigInt> sc = to_bigints(data.data(), data.size());
  G1J self = msm(amt.basis.data() + batch_index * batch, sc.data(), batch);
  if (!acc.add(self).eq(G1J::from_affine(commitment))) return P_INCONSISTENT;
  if (!pairing_eq(high, amt.g2, commitment, amt.high_g2)) return P_LDT;
  return -1;
}

VerifyResult slice_verify(const Dims& d, const AMTParams* amt, const EncodedSlice& s,
                          const G1A& auth_commitment, const H256& auth_root) {
  VerifyResult r;
  if (s.index != s.amt.index) {
    r.code = V_UNMATCHED_AMT_INDEX; r.a = s.index; r.b = s.amt.index; return r;
  }
  if (s.index != s.merkle.leaf_index) {
    r.code = V_UNMATCHED_MERKLE_INDEX; r.a = s.index; r.b = s.merkle.leaf_index; return r;
  }
  // amt
  if (s.amt.commitment != auth_commitment) { r.code = V_AMT_INCORRECT_COMMITMENT; return r; }
  if (s.amt.row.row.size() != d.cols()) {
    r.code = V_AMT_INCORRECT_ROW_SIZE; r.a = s.amt.row.row.size(); r.b = d.cols(); return r;
  }
  if (s.amt.index >= d.rows_encoded()) {
    r.code = V_AMT_ROW_INDEX_OVERFLOW; r.a = s.amt.index; r.b = d.rows_encoded(); return r;
  }
  size_t coset = s.amt.index / d.rows(), local = s.amt.index % d.rows();
  if (local != s.amt.row.index) {
    r.code = V_AMT_UNMATCHED_COSET_INDEX; r.a = coset; r.b = local; r.c = s.amt.row.index; return r;
  }
  {
    std::vector<Fr> data = s.amt.row.row;
    index_reverse(data);
    size_t bi = bitreverse(s.amt.row.index, d.log_row);
    int64_t kd = 0;
    int e = verify_amt_proof(amt[coset], data, bi, s.amt.row.proof, s.amt.commitment,
                             s.amt.row.high_commitment, &kd);
    if (e >= 0) {
      r.code = V_AMT_INCORRECT_PROOF; r.a = coset; r.b = s.amt.row.index;
      r.sub = e; r.c = (e == P_KZG) ? kd : 0;
      return r;
    }
  }
  // merkle
  const SliceMerkle& m = s.merkle;
  if (compute_file_root(m.root) != auth_root) { r.code = V_MERKLE_INCORRECT_ROOT; return r; }
  std::vector<H256> row(s.amt.row.row.size());
  for (size_t i = 0; i < row.size(); ++i) row[i] = scalar_to_h256(s.amt.row.row[i]);
  if (row.size() != d.cols()) { r.code = V_MERKLE_INCORRECT_SIZE; r.a = row.size(); r.b = d.cols(); return r; }
  if (m.leaf_index >= d.rows_encoded()) {
    r.code = V_MERKLE_ROW_INDEX_OVERFLOW; r.a = m.leaf_index; r.b = d.rows_encoded(); return r;
  }
  std::vector<H256> layer;
  keccak_chunked(row, 8, layer);
  while (layer.size() > 1) {
    std::vector<H256> next;
    keccak_chunked(layer, 2, next);
    layer = next;
  }
  if (layer[0] != m.leaf) { r.code = V_MERKLE_INCORRECT_LOCAL_ROOT; r.a = m.leaf_index; return r; }
  size_t position = m.leaf_index % d.n();
  H256 acc = m.leaf;
  for (auto& b : m.proof) {
    uint8_t buf[64];
    if (position % 2 == 1) { memcpy(buf, b.data(), 32); memcpy(buf + 32, acc.data(), 32); }
    else { memcpy(buf, acc.data(), 32); memcpy(buf + 32, b.data(), 32); }
    position >>= 1;
    keccak256(buf, 64, acc.data());
  }
  if (acc != m.root[m.leaf_index / d.rows()]) { r.code = V_MERKLE_INCORRECT_PROOF; r.a = m.leaf_index; return r; }
  return r;
}

// ---------------------------------------------------------------------------
// Recovery: crates/recovery/src/{lib,data_poly,zpoly,data_times_zpoly,utils,poly}.rs
static const int COSET_MORE = 4;

static std::vector<Fr> fx_to_fkx(const std::vector<Fr>& c, const Fr& k) {  // utils.rs:62-74
  std::vector<Fr> out = c;
  Fr base = Fr::one();
  for (auto& x : out) { x *= base; base *= k; }
  return out;
}
static std::vector<Fr> coeffs_to_evals_coset(const Dims& d, const std::vector<Fr>& coeffs, size_t c) {
  std::vector<Fr> cf = c ? fx_to_fkx(coeffs, coset_factor(d.n(), c)) : coeffs;
  size_t deg = std::max(next_pow2(cf.size()), d.n());
  cf.resize(deg, Fr::zero());
  fr_fft(cf);
  std::vector<Fr> ev(d.n());
  size_t step = deg / d.n();
  for (size_t i = 0; i < d.n(); ++i) ev[i] = cf[i * step];
  change_matrix_direction(ev, d.log_row, d.log_col);
  return ev;
}
static std::vector<Fr> coeffs_to_evals_larger(const Dims& d, const std::vector<Fr>& coeffs) {
  std::vector<Fr> out;
  out.reserve(COSET_MORE * d.n());
  for (int c = 0; c < COSET_MORE; ++c) {
    auto e = coeffs_to_evals_coset(d, coeffs, c);
    out.insert(out.end(), e.begin(), e.end());
  }
  return out;
}
static std::vector<Fr> trim(std::vector<Fr> v) {  // Poly::from_vec + to_vec
  while (v.size() > 1 && v.back().is_zero()) v.pop_back();
  if (v.empty()) v.push_back(Fr::zero());
  return v;
}
static std::vector<Fr> evals_to_poly(const Dims& d, const std::vector<Fr>& evals) {  // utils.rs:112-143
  std::vector<std::vector<Fr>> chunks(COSET_MORE);
  for (int c = 0; c < COSET_MORE; ++c) {
    chunks[c].assign(evals.begin() + c * d.n(), evals.begin() + (c + 1) * d.n());
    change_matrix_direction(chunks[c], d.log_col, d.log_row);
  }
  std::vector<Fr> t;
  for (int c = 0; c < COSET_MORE; ++c) {
    auto& ch = chunks[bitreverse(c, 2)];
    t.insert(t.end(), ch.begin(), ch.end());
  }
  change_matrix_direction(t, d.log_row + d.log_col, 2);
  fr_ifft(t);
  return trim(t);
}
static std::vector<Fr> poly_mul(const std::vector<Fr>& a, const std::vector<Fr>& b) {
  size_t rl = a.size() + b.size() - 1;
  if (a.size() * b.size() < 4096) {
    std::vector<Fr> r(rl, Fr::zero());
    for (size_t i = 0; i < a.size(); ++i)
      if (!a[i].is_zero())
        for (size_t j = 0; j < b.size(); ++j) r[i + j] += a[i] * b[j];
    return r;
  }
  size_t n = next_pow2(rl);
  std::vector<Fr> x = a, y = b;
  x.resize(n, Fr::zero()); y.resize(n, Fr::zero());
  fr_fft(x); fr_fft(y);
  for (size_t i = 0; i < n; ++i) x[i] *= y[i];
  fr_ifft(x);
  x.resize(rl);
  return x;
}
// zpoly.rs:60-78: prod over erased rows of (x^COL - c_row)
static std::vector<Fr> zpoly(const Dims& d, const std::set<size_t>& erased) {
  Fr wpow = fr_root_of_unity(d.log_row + d.log_col).pow_u64(d.cols());
  std::vector<std::vector<Fr>> polys;
  for (size_t id : erased) {
    size_t c = id / d.rows(), local = id % d.rows();
    Fr m0 = c == 0 ? -Fr::one() : -(coset_factor(d.n(), c).pow_u64(d.cols()));
    Fr z0 = m0 * wpow.pow_u64(local);
    std::vector<Fr> p(d.cols() + 1, Fr::zero());
    p[0] = z0;
    p[d.cols()] = Fr::one();
    polys.push_back(p);
  }
  if (polys.empty()) return {Fr::one()};
  while (polys.size() > 1) {
    std::vector<std::vector<Fr>> next((polys.size() + 1) / 2);
#pragma omp parallel for schedule(dynamic)
    for (size_t i = 0; i < next.size(); ++i)
      next[i] = (2 * i + 1 < polys.size()) ? poly_mul(polys[2 * i], polys[2 * i + 1]) : polys[2 * i];
    polys.swap(next);
  }
  return polys[0];
}

int recover_from_da_slice(const Dims& d, const std::map<size_t, std::vector<uint8_t>>& slices,
                          std::vector<uint8_t>* out, std::string* msg) {
  std::map<size_t, std::vector<Fr>> lines;
  for (auto& kv : slices) {
    if (kv.second.size() != BLOB_UNIT * d.cols()) continue;  // raw_slice_to_line Err -> dropped
    std::vector<Fr> line(d.cols());
    for (size_t i = 0; i < d.cols(); ++i)
      if (!Fr::from_le_bytes(kv.second.data() + 32 * i, &line[i])) {
        *msg = "Non-canonical field element in slice";
        return 7;
      }
    lines[kv.first] = line;
  }
  if (lines.size() < d.rows()) { *msg = "Not enough valid lines"; return 1; }
  // data_poly.rs:36-56 check_input
  if (lines.rbegin()->first >= d.rows_encoded()) { *msg = "Cannot recover data: RowIdOverflow"; return 2; }
  std::set<size_t> erased;
  for (size_t i = 0; i < COSET_MORE * d.rows(); ++i)
    if (!lines.count(i)) erased.insert(i);
  std::vector<Fr> data(COSET_MORE * d.n(), Fr::zero());
  for (auto& kv : lines)
    for (size_t e = 0; e < d.cols(); ++e) data[kv.first * d.cols() + e] = kv.second[e];
  std::vector<Fr> z = zpoly(d, erased);
  std::vector<Fr> ze = coeffs_to_evals_larger(d, z);
  for (size_t i = 0; i < data.size(); ++i) data[i] *= ze[i];
  std::vector<Fr> dz = evals_to_poly(d, data);
  uint64_t s = 0x5eed5eed5eedULL;
  for (int tries = 0; tries < 100; ++tries) {
    BigInt kb = {{splitmix64(s), splitmix64(s), splitmix64(s), splitmix64(s) & 0x0fffffffffffffffULL}};
    Fr k = Fr::from_bigint(kb);
    if (k.is_zero() || k == Fr::one()) continue;
    std::vector<Fr> zk = coeffs_to_evals_larger(d, fx_to_fkx(z, k));
    bool ok = true;
    for (auto& x : zk) if (x.is_zero()) { ok = false; break; }
    if (!ok) continue;
    std::vector<Fr> dzk = coeffs_to_evals_larger(d, fx_to_fkx(dz, k));
    for (size_t i = 0; i < dzk.size(); ++i) dzk[i] *= zk[i].inverse();
    std::vector<Fr> dk = evals_to_poly(d, dzk);
    std::vector<Fr> dc = fx_to_fkx(dk, k.inverse());
    if (dc.size() > d.n() + 1) { *msg = "Inconsistent rows (degree check)"; return 8; }
    std::vector<Fr> blob = coeffs_to_evals_coset(d, dc, 0);
    // raw_blob.rs:42-58, raw_data.rs:25-38
    std::vector<uint8_t> raw;
    raw.reserve(d.max_blob());
    for (auto& x : blob) {
      H256 h = scalar_to_h256(x);
      if (h[31] != 0) { *msg = "Incorrect scalar"; return 3; }
      raw.insert(raw.end(), h.begin(), h.begin() + 31);
    }
    uint32_t l32;
    memcpy(&l32, raw.data() + d.max_raw(), 4);
    if (l32 > d.max_raw()) { *msg = "Incorrect length field"; return 4; }
    for (size_t i = l32; i < d.max_raw(); ++i)
      if (raw[i]) { *msg = "Non zero in padding range"; return 5; }
    out->assign(raw.begin(), raw.begin() + l32);
    return 0;
  }
  *msg = "Cannot recover data: ExtaustiveK";
  return 6;
}

}  // namespace zgo
