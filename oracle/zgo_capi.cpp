// ORACLE — test infrastructure only (see zgo_field.hpp).
// extern "C" surface of the oracle for the Python test harness (ctypes).
//
// Verifier result codes (VerifierError / AmtError / MerkleError of
// crates/encoder/src/encoder/error.rs:8-22, amt/error.rs:3-26,
// merkle/error.rs:1-8; AmtProofError of crates/amt/src/proofs.rs:49-56):
//   0 Ok
//   1 UnmatchedAMTIndex{row_index=a, amt_index=b}
//   2 UnmatchedMerkleIndex{row_index=a, merkle_index=b}
//  10 AMT(IncorrectCommitment)
//  11 AMT(IncorrectRowSize{actual=a, expected=b})
//  12 AMT(RowIndexOverflow{actual=a, expected_max=b})
//  13 AMT(UnmatchedCosetIndex{coset_index=a, local_index=b, amt_index=c})
//  14 AMT(IncorrectProof{coset_index=a, amt_index=b, error=sub})
//       sub: 0 UnexpectedDataLength, 1 IncorrectPosition, 2 KzgError(c),
//            3 InconsistentCommitment, 4 FailedLowDegreeTest
//  20 Merkle(IncorrectRoot)
//  21 Merkle(IncorrectSize{actual=a, expected=b})
//  22 Merkle(RowIndexOverflow{actual=a, expected_max=b})
//  23 Merkle(IncorrectLocalRoot{row_index=a})
//  24 Merkle(IncorrectProof{row_index=a})
//  30 the slice bytes do not deserialize
#include <cstdio>

#include "zgo_encoder.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace zgo;

namespace {
struct ParamsHandle {
  Dims d;
  Fr tau;
  bool has_tau = false;
  AMTParams amt[COSET_N];
};
struct BlobHandle {
  EncodedBlob blob;
};
void g1_reply_bytes(const G1A& p, uint8_t out[64]) {  // grpc/src/service.rs:77-83
  if (p.inf) { memset(out, 0, 64); return; }
  p.x.to_le_bytes(out);
  p.y.to_le_bytes(out + 32);
}
bool g1_from_reply(const uint8_t in[64], G1A* p) {
  bool zero = true;
  for (int i = 0; i < 64; ++i) zero &= in[i] == 0;
  if (zero) { *p = {Fq::zero(), Fq::zero(), true}; return true; }
  if (!Fq::from_le_bytes(in, &p->x) || !Fq::from_le_bytes(in + 32, &p->y)) return false;
  p->inf = false;
  return true;
}
}  // namespace

extern "C" {

int zgo_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void zgo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// ---- primitives --------------------------------------------------------------
void zgo_keccak256(const uint8_t* in, size_t len, uint8_t out[32], uint8_t pad) {
  keccak256_pad(in, len, out, pad);
}
// in-place DFT on canonical LE 32-byte Fr elements; returns 0 or -1 on a
// non-canonical input
int zgo_fr_ntt(uint8_t* data, size_t n, int inverse, size_t coset_idx, size_t coset_len) {
  std::vector<Fr> v(n);
  for (size_t i = 0; i < n; ++i)
    if (!Fr::from_le_bytes(data + 32 * i, &v[i])) return -1;
  if (coset_idx && !inverse) {
    // coefficients * g^i then forward transform (to_coset_blob's inner step)
    Fr g = coset_factor(coset_len, coset_idx), b = Fr::one();
    for (auto& x : v) { x *= b; b *= g; }
  }
  if (inverse) fr_ifft(v); else fr_fft(v);
  for (size_t i = 0; i < n; ++i) v[i].to_le_bytes(data + 32 * i);
  return 0;
}
void zgo_fr_root_of_unity(int log_n, uint8_t out[32]) { fr_root_of_unity(log_n).to_le_bytes(out); }
void zgo_fr_coset_factor(size_t length, size_t idx, uint8_t out[32]) { coset_factor(length, idx).to_le_bytes(out); }
void zgo_tau_from_seed(uint64_t seed, uint8_t out[32]) { tau_from_seed(seed).to_le_bytes(out); }
// Fr product of two canonical elements (used to pin against Python big ints)
void zgo_fr_mul(const uint8_t a[32], const uint8_t b[32], uint8_t out[32]) {
  Fr x, y;
  Fr::from_le_bytes(a, &x);
  Fr::from_le_bytes(b, &y);
  (x * y).to_le_bytes(out);
}
// k * G1 as ark uncompressed bytes
void zgo_g1_mul_gen(const uint8_t k[32], uint8_t out[64]) {
  BigInt b; memcpy(b.v, k, 32);
  std::vector<uint8_t> v;
  ser_g1(G1J::from_affine(g1_generator()).mul(b).to_affine(), v);
  memcpy(out, v.data(), 64);
}
// MSM over affine bases in mont format (x||y raw Montgomery limbs, 64 B each)
// and canonical LE scalars; result as ark uncompressed bytes.
void zgo_msm_g1(const uint8_t* bases_mont, const uint8_t* scalars, size_t n, uint8_t out[64]) {
  std::vector<G1A> b(n);
  std::vector<BigInt> s(n);
  for (size_t i = 0; i < n; ++i) {
    u64 x[4], y[4];
    memcpy(x, bases_mont + 64 * i, 32);
    memcpy(y, bases_mont + 64 * i + 32, 32);
    b[i] = {Fq::from_raw_mont(x), Fq::from_raw_mont(y), false};
    memcpy(s[i].v, scalars + 32 * i, 32);
  }
  std::vector<uint8_t> v;
  ser_g1(msm(b.data(), s.data(), n).to_affine(), v);
  memcpy(out, v.data(), 64);
}
// bilinearity and non-degeneracy of the oracle pairing for scalars derived from seed
int zgo_pairing_selftest(uint64_t seed) {
  Fr a = tau_from_seed(seed), b = tau_from_seed(seed + 1);
  G1A P = g1_generator();
  G2A Q = g2_generator();
  G1A aP = G1J::from_affine(P).mul(a.to_bigint()).to_affine();
  G2A bQ = G2J::from_affine(Q).mul(b.to_bigint()).to_affine();
  G1A abP = G1J::from_affine(P).mul((a * b).to_bigint()).to_affine();
  Fq12 e1 = pairing(aP, bQ), e2 = pairing(abP, Q), e0 = pairing(P, Q);
  if (e0 == Fq12::one()) return 0;
  if (e1 != e2) return 0;
  if (!pairing_eq(aP, bQ, abP, Q)) return 0;
  if (pairing_eq(aP, bQ, P, Q)) return 0;
  BigInt rb = {{FrCfg::P[0], FrCfg::P[1], FrCfg::P[2], FrCfg::P[3]}};
  if (!G1J::from_affine(P).mul(rb).is_inf()) return 0;
  if (!G2J::from_affine(Q).mul(rb).is_inf()) return 0;
  return 1;
}

// ---- params -------------------------------------------------------------------
// mode 0: scalar-domain builder; mode 1: EC-domain restatement of
// AMTParams::from_pp (slow, small depths only)
void* zgo_params_new(int log_row, int log_col, uint64_t seed, int mode) {
  auto* h = new ParamsHandle();
  h->d = {log_row, log_col};
  h->tau = tau_from_seed(seed);
  h->has_tau = true;
  int depth = log_row + log_col;
  if (mode == 1) {
    PowerTau pp = power_tau_setup(h->tau, depth);
    for (int c = 0; c < COSET_N; ++c) h->amt[c] = amt_from_pp_ec(pp, log_row, c);
  } else {
    for (int c = 0; c < COSET_N; ++c)
      h->amt[c] = amt_from_scalars(amt_scalars(h->tau, depth, log_row, c), depth, log_row);
  }
  return h;
}
void* zgo_params_from_mont(int log_row, int log_col, const uint8_t* const* files, const size_t* lens) {
  auto* h = new ParamsHandle();
  h->d = {log_row, log_col};
  for (int c = 0; c < COSET_N; ++c)
    if (!read_amt_params_mont(files[c], lens[c], &h->amt[c])) { delete h; return nullptr; }
  return h;
}
void zgo_params_free(void* p) { delete static_cast<ParamsHandle*>(p); }
size_t zgo_params_mont(void* p, int coset, uint8_t* out, size_t cap) {
  std::vector<uint8_t> v;
  write_amt_params_mont(static_cast<ParamsHandle*>(p)->amt[coset], v);
  if (out && cap >= v.size()) memcpy(out, v.data(), v.size());
  return v.size();
}
// Selected param points of one line at any depth, from the scalar domain.
// line: 0..prove_depth-1 quotients, prove_depth basis, prove_depth+1 high_basis.
// Output: 64-byte mont (x||y raw limbs) per requested index.
int zgo_param_points(int log_row, int log_col, uint64_t seed, int coset, int line, const uint64_t* idx, size_t n,
                     uint8_t* out) {
  int depth = log_row + log_col;
  Fr tau = tau_from_seed(seed);
  size_t length = size_t(1) << depth;
  size_t high_start = (size_t(1) << (depth + 2)) - length;
  Fr w = coset > 0 ? coset_factor(length, coset).inverse() : Fr::one();
  Fr tp = tau * w;
  std::vector<Fr> pw(length);
  pw[0] = Fr::one();
  for (size_t i = 1; i < length; ++i) pw[i] = pw[i - 1] * tp;
  std::vector<Fr> sc;
  if (line >= log_row) {
    sc = pw;
    fr_ifft(sc);
    if (line == log_row + 1) {
      Fr ths = tau.pow_u64(high_start);
      for (auto& x : sc) x *= ths;
    }
  } else {
    int d = line + 1;
    size_t max_coeff = size_t(1) << (depth - d);
    sc.assign(length, Fr::zero());
    for (size_t i = 1; i <= max_coeff; ++i) sc[i] = pw[max_coeff - i];
    fr_ntt_omega(sc, fr_root_of_unity(depth));
    Fr si = Fr::from_u64(length).inverse();
    for (auto& x : sc) x *= si;
  }
  G1J g = G1J::from_affine(g1_generator());
  std::vector<G1J> pts(n);
#pragma omp parallel for schedule(dynamic)
  for (size_t i = 0; i < n; ++i) {
    size_t pos = bitreverse(idx[i], depth);  // enact() bit-reverses the line
    pts[i] = g.mul(sc[pos].to_bigint());
  }
  std::vector<G1A> a(n);
  normalize_batch(pts.data(), a.data(), n);
  for (size_t i = 0; i < n; ++i) {
    memcpy(out + 64 * i, a[i].x.v, 32);
    memcpy(out + 64 * i + 32, a[i].y.v, 32);
  }
  return 0;
}


// Merkle roots (merkle/blob.rs:15-34) of n_items 32-byte items; writes 3 x 32 B
void zgo_merkle_roots(int log_row, int log_col, const uint8_t* items, uint8_t out[96]) {
  Dims d = {log_row, log_col};
  std::vector<H256> data(COSET_N * d.n());
  for (size_t i = 0; i < data.size(); ++i) memcpy(data[i].data(), items + 32 * i, 32);
  Merkle m = merkle_build(d, std::move(data));
  for (int c = 0; c < COSET_N; ++c) memcpy(out + 32 * c, m.tree[0][c].data(), 32);
}

// Verifier params (AMTVerifyParams: basis, vanishes, g2, high_g2;
// crates/amt/src/verify_params.rs:22-28) with the basis lines supplied by the
// caller (3 x N points, 64 B mont each) and the G2 parts from the scalar
// domain of the seeded tau.
void* zgo_verify_params_new(int log_row, int log_col, uint64_t seed, const uint8_t* basis_lines) {
  auto* h = new ParamsHandle();
  h->d = {log_row, log_col};
  h->tau = tau_from_seed(seed);
  h->has_tau = true;
  int depth = log_row + log_col;
  size_t n = h->d.n();
  for (int c = 0; c < COSET_N; ++c) {
    AMTScalars s;
    {
      // only the G2 part of the scalar-domain builder is needed
      size_t length = n;
      size_t high_start = (size_t(1) << (depth + 2)) - length;
      Fr w = c > 0 ? coset_factor(length, c).inverse() : Fr::one();
      Fr tp = h->tau * w;
      std::vector<Fr> pw(length);
      pw[0] = Fr::one();
      for (size_t i = 1; i < length; ++i) pw[i] = pw[i - 1] * tp;
      for (int dd = 1; dd <= log_row; ++dd) {
        size_t step = size_t(1) << (depth - dd);
        size_t sz = size_t(1) << dd;
        std::vector<Fr> coeff(sz, Fr::zero());
        coeff[0] = pw[length - step];
        for (size_t i = 1; i < length / step; ++i) coeff[i] = pw[(i - 1) * step];
        fr_ntt_omega(coeff, fr_root_of_unity(dd).inverse());
        index_reverse(coeff);
        s.vanishes.push_back(coeff);
      }
      s.high_g2 = h->tau.pow_u64(high_start);
    }
    AMTParams p = amt_from_scalars(s, depth, log_row);
    p.basis.resize(n);
    for (size_t i = 0; i < n; ++i) {
      u64 x[4], y[4];
      memcpy(x, basis_lines + (c * n + i) * 64, 32);
      memcpy(y, basis_lines + (c * n + i) * 64 + 32, 32);
      p.basis[i] = {Fq::from_raw_mont(x), Fq::from_raw_mont(y), false};
    }
    h->amt[c] = p;
  }
  return h;
}

// ---- encode -------------------------------------------------------------------
// returns nullptr and *err = 1 for TooLargeBlob
void* zgo_encode(void* params, const uint8_t* data, size_t len, int* err) {
  auto* ph = static_cast<ParamsHandle*>(params);
  std::vector<uint8_t> raw;
  if (!raw_data_from_bytes(ph->d, data, len, &raw)) { *err = 1; return nullptr; }
  *err = 0;
  auto* bh = new BlobHandle();
  encoded_blob_build(ph->d, raw_blob_from_raw_data(ph->d, raw), ph->amt, &bh->blob);
  return bh;
}
void zgo_blob_free(void* b) { delete static_cast<BlobHandle*>(b); }
void zgo_blob_commitment(void* b, uint8_t out[64]) {
  g1_reply_bytes(static_cast<BlobHandle*>(b)->blob.halves[0].commitment, out);
}
void zgo_blob_roots(void* b, uint8_t out[96]) {
  auto& m = static_cast<BlobHandle*>(b)->blob.merkle;
  for (int c = 0; c < COSET_N; ++c) memcpy(out + 32 * c, m.tree[0][c].data(), 32);
}
void zgo_blob_file_root(void* b, uint8_t out[32]) {
  auto& m = static_cast<BlobHandle*>(b)->blob.merkle;
  H256 roots[COSET_N] = {m.tree[0][0], m.tree[0][1], m.tree[0][2]};
  H256 r = compute_file_root(roots);
  memcpy(out, r.data(), 32);
}
void zgo_blob_data(void* b, uint8_t* out) {
  auto& m = static_cast<BlobHandle*>(b)->blob.merkle;
  for (size_t i = 0; i < m.data.size(); ++i) memcpy(out + 32 * i, m.data[i].data(), 32);
}
size_t zgo_blob_slice(void* b, size_t index, uint8_t* out, size_t cap) {
  auto& blob = static_cast<BlobHandle*>(b)->blob;
  std::vector<uint8_t> v;
  serialize_slice(encoded_blob_get_row(blob, index), v);
  if (out && cap >= v.size()) memcpy(out, v.data(), v.size());
  return v.size();
}
// AMT outputs of one coset as ark uncompressed G1 bytes, in the order
// [commitment][commitments[0..LR) concatenated][proofs[0..LR) concatenated][high]
size_t zgo_blob_amt_outputs(void* b, int coset, uint8_t* out) {
  auto& hb = static_cast<BlobHandle*>(b)->blob.halves[coset];
  std::vector<uint8_t> v;
  ser_g1(hb.commitment, v);
  for (auto& l : hb.proofs.commitments) for (auto& p : l) ser_g1(p, v);
  for (auto& l : hb.proofs.proofs) for (auto& p : l) ser_g1(p, v);
  ser_g1(hb.proofs.high_commitment, v);
  if (out) memcpy(out, v.data(), v.size());
  return v.size() / 64;
}

// Expected AMT outputs of one coset from the scalar domain (tau known):
// every param point is s*G, so each MSM equals (sum_t scalar_t * s_t) * G.
// `coset_rows` = encoded coset values, row-major canonical LE 32 B.
// Output layout as zgo_blob_amt_outputs.
int zgo_amt_scalar_domain(int log_row, int log_col, uint64_t seed, int coset, const uint8_t* coset_rows,
                          uint8_t* out) {
  Dims d = {log_row, log_col};
  int depth = log_row + log_col;
  size_t n = d.n();
  std::vector<Fr> blob(n);
  for (size_t i = 0; i < n; ++i)
    if (!Fr::from_le_bytes(coset_rows + 32 * i, &blob[i])) return -1;
  // blob row-major -> points (column-major) -> ri (bit-reversed)
  change_matrix_direction(blob, log_row, log_col);
  index_reverse(blob);
  AMTScalars s = amt_scalars(tau_from_seed(seed), depth, log_row, coset);
  size_t batch = n >> log_row;
  auto dot = [&](const std::vector<Fr>& line, size_t lo, size_t cnt) {
    Fr acc = Fr::zero();
    for (size_t i = lo; i < lo + cnt; ++i) acc += line[i] * blob[i];
    return acc;
  };
  // commitment tree leaves
  size_t nb = n / batch;
  std::vector<Fr> layer(nb);
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < nb; ++k) layer[k] = dot(s.basis, k * batch, batch);
  std::vector<std::vector<Fr>> levels;  // levels[0] = 2 nodes ... levels[LR-1] = nb nodes
  std::vector<Fr> cur = layer;
  std::vector<std::vector<Fr>> rev;
  while (cur.size() > 1) {
    rev.push_back(cur);
    std::vector<Fr> nx(cur.size() / 2);
    for (size_t i = 0; i < nx.size(); ++i) nx[i] = cur[2 * i] + cur[2 * i + 1];
    cur = nx;
  }
  levels.assign(rev.rbegin(), rev.rend());
  std::vector<Fr> all;
  all.push_back(cur[0]);
  for (auto& l : levels) all.insert(all.end(), l.begin(), l.end());
  for (int dd = 1; dd <= log_row; ++dd) {
    size_t items = size_t(1) << dd, chunk = n / items;
    std::vector<Fr> q(items);
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < items; ++k) q[k] = dot(s.quotients[dd - 1], k * chunk, chunk);
    all.insert(all.end(), q.begin(), q.end());
  }
  all.push_back(dot(s.high_basis, 0, n));
  G1J g = G1J::from_affine(g1_generator());
  std::vector<G1J> pts(all.size());
#pragma omp parallel for schedule(dynamic)
  for (size_t i = 0; i < all.size(); ++i) pts[i] = g.mul(all[i].to_bigint());
  std::vector<G1A> a(all.size());
  normalize_batch(pts.data(), a.data(), a.size());
  std::vector<uint8_t> v;
  for (auto& p : a) ser_g1(p, v);
  memcpy(out, v.data(), v.size());
  return (int)a.size();
}

// ---- verify -------------------------------------------------------------------
int zgo_slice_verify(void* params, const uint8_t* slice, size_t len, const uint8_t commitment[64],
                     const uint8_t root[32], int64_t detail[4]) {
  auto* ph = static_cast<ParamsHandle*>(params);
  EncodedSlice s;
  detail[0] = detail[1] = detail[2] = detail[3] = 0;
  if (!deserialize_slice(slice, len, &s)) return 30;
  G1A c;
  if (!g1_from_reply(commitment, &c)) return 30;
  H256 r;
  memcpy(r.data(), root, 32);
  VerifyResult v = slice_verify(ph->d, ph->amt, s, c, r);
  detail[0] = v.sub; detail[1] = v.a; detail[2] = v.b; detail[3] = v.c;
  return v.code;
}



// n pseudo-random G1 points k_i * G (k_i from the SplitMix64 stream at seed),
// 64 B mont x||y each: stand-in bases for timing samples, where the MSM cost
// does not depend on which points are summed
void zgo_random_points(uint64_t seed, size_t n, uint8_t* out) {
  static FixedBaseG1* fb = nullptr;
#pragma omp critical(zgo_rand_fb)
  {
    if (!fb) fb = new FixedBaseG1(g1_generator());
  }
  std::vector<G1J> j(n);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) j[i] = fb->mul(tau_from_seed(seed + i));
  std::vector<G1A> a(n);
  normalize_batch(j.data(), a.data(), n);
  for (size_t i = 0; i < n; ++i) {
    memcpy(out + 64 * i, a[i].x.v, 32);
    memcpy(out + 64 * i + 32, a[i].y.v, 32);
  }
}

// ---- CPU baseline ---------------------------------------------------------------
// The restated CPU path of EncoderService::process_data (grpc/src/service.rs:
// 69-105) on full blobs, cut into steps of one coset each so that a timing
// run can stop at any step without extrapolating: three consecutive steps
// are exactly one blob.
//   coset 0: RawData::try_from + RawBlob::from (raw_data.rs:55-72,
//            raw_blob.rs:33-40), change_matrix_direction, then coset 0's
//            half blob (encode.rs:91-108, 171-183: to_coset_blob, index_reverse,
//            gen_all_proofs with the prove.rs:58-102 decomposition, every MSM
//            the ark-style bucket method of zgo_curve.hpp);
//   coset 1: coset 1's half blob;
//   coset 2: coset 2's half blob, assert_commitment_consistent, the keccak
//            Merkle tree (merkle/blob.rs:15-34), the file root and the 3072
//            ark-serialized slices of the reply (service.rs:85-95).
struct CpuJob {
  ParamsHandle* ph = nullptr;
  std::vector<uint8_t> payload;
  std::vector<Fr> points;  // column-major blob of the current blob
  EncodedBlob blob;
  int next = 0;            // coset of the next step
  uint8_t file_root[32] = {0};
  size_t reply_bytes = 0;
};
void* zgo_cpu_job_new(void* params, const uint8_t* data, size_t len) {
  auto* j = new CpuJob();
  j->ph = static_cast<ParamsHandle*>(params);
  j->payload.assign(data, data + len);
  return j;
}
void zgo_cpu_job_free(void* job) { delete static_cast<CpuJob*>(job); }
// Runs the job's next step; returns the coset it covered (0, 1, 2) or -1 when
// the payload is too large. After a coset-2 step file_root (32 B) and
// reply_bytes (total serialized slice bytes) describe the finished blob.
int zgo_cpu_job_step(void* job, uint8_t* file_root, size_t* reply_bytes) {
  auto* j = static_cast<CpuJob*>(job);
  const Dims& d = j->ph->d;
  const int c = j->next;
  if (c == 0) {
    std::vector<uint8_t> raw;
    if (!raw_data_from_bytes(d, j->payload.data(), j->payload.size(), &raw)) return -1;
    j->points = raw_blob_from_raw_data(d, raw);
    change_matrix_direction(j->points, d.log_col, d.log_row);
    j->blob = EncodedBlob();
    j->blob.dims = d;
  }
  j->blob.halves[c] = half_blob_generate(d, to_coset_blob(j->points, c), j->ph->amt[c]);
  if (c == COSET_N - 1) {
    for (int k = 1; k < COSET_N; ++k)
      if (j->blob.halves[k].commitment != j->blob.halves[0].commitment) abort();
    const size_t n = d.n();
    std::vector<H256> data(COSET_N * n);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < COSET_N * n; ++i) data[i] = scalar_to_h256(j->blob.halves[i / n].blob[i % n]);
    j->blob.merkle = merkle_build(d, std::move(data));
    H256 roots[COSET_N] = {j->blob.merkle.tree[0][0], j->blob.merkle.tree[0][1], j->blob.merkle.tree[0][2]};
    H256 fr = compute_file_root(roots);
    memcpy(j->file_root, fr.data(), 32);
    const size_t ns = COSET_N * d.rows();
    std::vector<size_t> sizes(ns);
#pragma omp parallel for schedule(dynamic, 16)
    for (size_t i = 0; i < ns; ++i) {
      std::vector<uint8_t> v;
      serialize_slice(encoded_blob_get_row(j->blob, i), v);
      sizes[i] = v.size();
    }
    j->reply_bytes = 0;
    for (size_t x : sizes) j->reply_bytes += x;
  }
  j->next = (c + 1) % COSET_N;
  if (file_root) memcpy(file_root, j->file_root, 32);
  if (reply_bytes) *reply_bytes = j->reply_bytes;
  return c;
}

// All slices of an oracle blob back to back (3R x slice size), serialized in
// parallel: the full-blob comparison of the production tests.
size_t zgo_blob_all_slices(void* b, uint8_t* out, size_t cap) {
  auto& blob = static_cast<BlobHandle*>(b)->blob;
  const size_t ns = COSET_N * blob.dims.rows();
  std::vector<uint8_t> first;
  serialize_slice(encoded_blob_get_row(blob, 0), first);
  const size_t sz = first.size();
  if (!out) return ns * sz;
  if (cap < ns * sz) return 0;
  bool ok = true;
#pragma omp parallel for schedule(dynamic, 16) reduction(&& : ok)
  for (size_t i = 0; i < ns; ++i) {
    std::vector<uint8_t> v;
    serialize_slice(encoded_blob_get_row(blob, i), v);
    if (v.size() != sz) { ok = false; continue; }
    memcpy(out + i * sz, v.data(), sz);
  }
  return ok ? ns * sz : 0;
}

// ---- recovery -----------------------------------------------------------------
int zgo_recover(int log_row, int log_col, const uint64_t* ids, const uint8_t* const* rows, const size_t* lens,
                size_t n, uint8_t* out, size_t* out_len, char* msg, size_t msgcap) {
  Dims d = {log_row, log_col};
  std::map<size_t, std::vector<uint8_t>> m;
  for (size_t i = 0; i < n; ++i) m[ids[i]] = std::vector<uint8_t>(rows[i], rows[i] + lens[i]);
  std::vector<uint8_t> o;
  std::string s;
  int rc = recover_from_da_slice(d, m, &o, &s);
  if (msg && msgcap) snprintf(msg, msgcap, "%s", s.c_str());
  if (rc == 0) {
    memcpy(out, o.data(), o.size());
    *out_len = o.size();
  }
  return rc;
}

}  // extern "C"
