// ORACLE — test infrastructure only (see zgo_field.hpp).
// CPU restatement of the reference's encode path:
//   crates/encoder/src/{raw_data,raw_blob,utils}.rs, encoder/{blob,slice}.rs,
//   amt/{blob,slice}.rs, merkle/{blob,slice}.rs,
//   crates/amt/src/{utils,proofs,power_tau,verify_params}.rs, blob/encode.rs,
//   prove_params/{generate,prove,fast_serde_bn254}.rs,
//   crates/recovery/src/*.rs, grpc/src/service.rs:69-105.
// Sizes are runtime parameters (LOG_ROW, LOG_COL), COSET_N = 3, as the
// reference's const generics <COSET_N, LOG_COL, LOG_ROW>
// (crates/amt/src/blob/encode.rs:21-28).
#pragma once
#include <array>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "zgo_curve.hpp"
#include "zgo_keccak.hpp"
#include "zgo_pairing.hpp"

namespace zgo {

typedef std::array<uint8_t, 32> H256;
static const int COSET_N = 3;
static const int RAW_UNIT = 31;
static const int BLOB_UNIT = 32;

struct Dims {
  int log_row, log_col;
  size_t rows() const { return size_t(1) << log_row; }
  size_t cols() const { return size_t(1) << log_col; }
  size_t n() const { return size_t(1) << (log_row + log_col); }        // RAW_BLOB_SIZE
  size_t rows_encoded() const { return rows() * COSET_N; }             // BLOB_ROW_ENCODED
  size_t max_blob() const { return RAW_UNIT * n(); }                   // MAX_BLOB_SIZE
  size_t max_raw() const { return max_blob() - 4; }                    // MAX_RAW_DATA_SIZE
};

// ---- index helpers: crates/amt/src/utils.rs:54-116
size_t bitreverse(size_t n, int l);
size_t swap_bits(size_t n, int lo, int hi);
template <class T>
void index_reverse(std::vector<T>& a) {
  size_t n = a.size();
  int depth = 0;
  while ((size_t(1) << depth) < n) ++depth;
  for (size_t i = 0; i < n; ++i) {
    size_t ri = bitreverse(i, depth);
    if (i < ri) std::swap(a[i], a[ri]);
  }
}
template <class T>
void change_matrix_direction(std::vector<T>& a, int log_current, int log_next) {
  std::vector<T> out(a.size());
  for (size_t i = 0; i < a.size(); ++i) out[swap_bits(i, log_current, log_next)] = a[i];
  a.swap(out);
}

// ---- NTT with ark-poly Radix2EvaluationDomain semantics
void fr_fft(std::vector<Fr>& a);   // a[k] <- sum_j a[j] w^{jk}; pads to pow2
void fr_ifft(std::vector<Fr>& a);  // inverse, scaled by 1/n
void fr_ntt_omega(std::vector<Fr>& a, const Fr& omega);
Fr coset_factor(size_t length, size_t idx);  // prove_params/generate.rs:128-137

// fixed-base multiplication table: entry [w][d-1] = d * 2^{8w} * G
template <class F>
struct FixedBase {
  std::vector<Affine<F>> tab;
  explicit FixedBase(const Affine<F>& g) {
    std::vector<Jac<F>> j(32 * 255);
    Jac<F> base = Jac<F>::from_affine(g);
    for (int w = 0; w < 32; ++w) {
      Jac<F> acc = base;
      for (int d = 1; d <= 255; ++d) {
        j[w * 255 + d - 1] = acc;
        acc = acc.add(base);
      }
      base = acc;  // 256 * base
    }
    tab.resize(j.size());
    normalize_batch(j.data(), tab.data(), j.size());
  }
  Jac<F> mul(const Fr& s) const {
    BigInt k = s.to_bigint();
    Jac<F> acc = Jac<F>::inf();
    for (int w = 0; w < 32; ++w) {
      unsigned d = (k.v[w / 8] >> (8 * (w % 8))) & 0xff;
      if (d) acc = acc.add_affine(tab[w * 255 + d - 1]);
    }
    return acc;
  }
};

typedef FixedBase<Fq> FixedBaseG1;

// ---- params
struct PowerTau {
  std::vector<G1A> g1pp, high_g1pp;
  std::vector<G2A> g2pp;
  G2A high_g2;
};
struct AMTParams {
  int depth = 0, prove_depth = 0;
  std::vector<G1A> basis;
  std::vector<std::vector<G1A>> quotients;
  std::vector<std::vector<G2A>> vanishes;
  G2A g2, high_g2;
  std::vector<G1A> high_basis;
  size_t len() const { return basis.size(); }
};
// scalar of every param point for a known tau (test fixture only)
struct AMTScalars {
  std::vector<Fr> basis, high_basis;
  std::vector<std::vector<Fr>> quotients, vanishes;
  Fr high_g2;
};
Fr tau_from_seed(uint64_t seed);
PowerTau power_tau_setup(const Fr& tau, int depth);                 // power_tau.rs:54-80
AMTParams amt_from_pp_ec(const PowerTau& pp, int prove_depth, int coset);  // generate.rs:139-263
AMTScalars amt_scalars(const Fr& tau, int depth, int prove_depth, int coset);
AMTParams amt_from_scalars(const AMTScalars& s, int depth, int prove_depth);
void write_amt_params_mont(const AMTParams& p, std::vector<uint8_t>& out);  // fast_serde_bn254.rs:20-53
bool read_amt_params_mont(const uint8_t* in, size_t len, AMTParams* out);   // fast_serde_bn254.rs:55-88

// ---- encode
struct AllProofs {
  std::vector<std::vector<G1A>> commitments, proofs;
  size_t input_len = 0, batch_size = 0;
  G1A high_commitment;
};
struct HalfBlob {
  std::vector<Fr> blob;
  G1A commitment;
  AllProofs proofs;
};
struct Proof {
  std::vector<std::pair<G1A, G1A>> v;
};
struct BlobRow {
  uint64_t index;
  std::vector<Fr> row;
  Proof proof;
  G1A high_commitment;
};
struct SliceAMT {
  uint64_t index;
  G1A commitment;
  BlobRow row;
};
struct SliceMerkle {
  H256 root[COSET_N];
  std::vector<H256> proof;
  uint64_t leaf_index;
  H256 leaf;
};
struct EncodedSlice {
  uint64_t index;
  SliceAMT amt;
  SliceMerkle merkle;
};
struct Merkle {
  std::vector<H256> data;
  std::vector<std::vector<H256>> tree;
};
struct EncodedBlob {
  Dims dims;
  HalfBlob halves[COSET_N];
  Merkle merkle;
};

bool raw_data_from_bytes(const Dims& d, const uint8_t* in, size_t len, std::vector<uint8_t>* out);
std::vector<Fr> raw_blob_from_raw_data(const Dims& d, const std::vector<uint8_t>& raw);
std::vector<Fr> to_coset_blob(const std::vector<Fr>& data, size_t coset);
std::vector<BigInt> to_bigints(const Fr* s, size_t n);
AllProofs gen_all_proofs(const AMTParams& amt, const std::vector<Fr>& ri_data, G1J* commitment);
HalfBlob half_blob_generate(const Dims& d, std::vector<Fr> points, const AMTParams& amt);
Merkle merkle_build(const Dims& d, std::vector<H256> data);
void encoded_blob_build(const Dims& d, const std::vector<Fr>& raw_blob, const AMTParams* amt,
                        EncodedBlob* out);
H256 compute_file_root(const H256 roots[COSET_N]);
EncodedSlice encoded_blob_get_row(const EncodedBlob& b, size_t index);
H256 scalar_to_h256(const Fr& x);

// ---- ark-serialize 0.4 (uncompressed)
void ser_g1(const G1A& p, std::vector<uint8_t>& out);
bool de_g1(const uint8_t*& p, const uint8_t* end, G1A* out);
void ser_g2(const G2A& p, std::vector<uint8_t>& out);
void serialize_slice(const EncodedSlice& s, std::vector<uint8_t>& out);
bool deserialize_slice(const uint8_t* in, size_t len, EncodedSlice* out);

// ---- verify (codes documented in oracle/zgo_capi.cpp)
struct VerifyResult {
  int32_t code = 0, sub = 0;
  int64_t a = 0, b = 0, c = 0;
};
VerifyResult slice_verify(const Dims& d, const AMTParams* amt, const EncodedSlice& s,
                          const G1A& authoritative_commitment, const H256& authoritative_root);

// ---- recovery (crates/recovery/src/lib.rs:15-43)
// returns 0 on success, else an error code; msg receives the reference's text
int recover_from_da_slice(const Dims& d, const std::map<size_t, std::vector<uint8_t>>& slices,
                          std::vector<uint8_t>* out, std::string* msg);

}  // namespace zgo
