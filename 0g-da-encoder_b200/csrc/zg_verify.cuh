// Device kernels of batched slice verification (zg_verify_slices).
//
// The reference checks one EncodedSlice at a time (EncodedSlice::verify,
// crates/encoder/src/encoder/slice.rs:73-95): a Merkle path
// (merkle/slice.rs:50-104) and an AMT proof of 10 KZG pairing equalities, one
// MSM consistency check and one low-degree pairing test
// (crates/amt/src/verify_params.rs:136-211); its DeferredVerifier
// (deferred_verification.rs:67-146) folds many such checks into random linear
// combinations. Here a whole batch of slices is checked at once:
//  * Merkle paths: one CTA per slice (k_verify_merkle);
//  * MSM checks: sum_i alpha_i (sum_t basis[bi C + t] data_i[t]) over all
//    slices of a coset is ONE MSM over the coset's basis line (scalars
//    alpha_i data_i[t] scattered by k_verify_scalars), run on the context's
//    fixed-base tables;
//  * pairing checks: e(L, g2) prod_g e(-G_g, V_g) prod_c e(-H_c, high_g2_c) = 1
//    with L, G_g, H_c random-weighted G1 sums (k_g1_mul_words + segment
//    sums), one Miller loop per distinct G2 point (k_miller) and one final
//    exponentiation on the host.
#pragma once
#include "zg_pairing.cuh"

namespace zg {

// out[i] = s_i * P_i for affine P_i (inf[i] != 0: the point at infinity) and
// little-endian scalars of `nw` 32-bit words (s_i at sc + i * nw)
__global__ void __launch_bounds__(128) k_g1_mul_words(const G1Aff* __restrict__ pts, const uint8_t* __restrict__ inf,
                                                      const uint32_t* __restrict__ sc, int nw, XYZZ* __restrict__ out,
                                                      uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  XYZZ acc = XYZZ::inf();
  if (!inf[i]) {
    const G1Aff p = pts[i];
    const uint32_t* s = sc + (size_t)i * nw;
    bool started = false;
    for (int w = nw - 1; w >= 0; --w) {
      const uint32_t word = s[w];
#pragma unroll 1
      for (int b = 31; b >= 0; --b) {
        if (started) acc = acc.dbl();
        if ((word >> b) & 1) {
          acc.add_affine(p.x, p.y);
          started = true;
        }
      }
    }
  }
  store_xyzz(out + i, acc);
}

// out[g] = sum of terms[k] for k in [off[g], off[g + 1])
__global__ void __launch_bounds__(128) k_seg_sum(const XYZZ* __restrict__ terms, const uint32_t* __restrict__ off,
                                                 XYZZ* __restrict__ out, uint32_t nseg) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nseg) return;
  XYZZ acc = XYZZ::inf();
  for (uint32_t k = off[g]; k < off[g + 1]; ++k) acc.add(load_xyzz(terms + k));
  store_xyzz(out + g, acc);
}

// Miller inputs: affine (negated when neg[j]) G1 points with infinity flags
__global__ void __launch_bounds__(128) k_pairing_inputs(const XYZZ* __restrict__ in, const uint8_t* __restrict__ neg,
                                                        G1Aff* __restrict__ out, uint8_t* __restrict__ inf, uint32_t n) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  G1Aff a;
  const bool ok = in[j].to_affine(a);
  if (ok && neg[j]) a.y = -a.y;
  if (!ok) { a.x = Fq::zero(); a.y = Fq::zero(); }
  out[j] = a;
  inf[j] = ok ? 0 : 1;
}

// f[j] = Miller function of (P_j, Q_j), one loop per thread
__global__ void __launch_bounds__(64) k_miller(const G1Aff* __restrict__ P, const uint8_t* __restrict__ pinf,
                                               const G2Aff* __restrict__ Q, Fq12* __restrict__ f, uint32_t n) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  f[j] = miller_tate(P[j], pinf[j] != 0, Q[j]);
}

// part[t] = product of f[k] for k = t, t + T, t + 2T, ... (one CTA of T threads)
__global__ void __launch_bounds__(128) k_fq12_partial(const Fq12* __restrict__ f, uint32_t n, Fq12* __restrict__ part) {
  Fq12 acc = Fq12::one();
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) acc = acc * f[k];
  part[threadIdx.x] = acc;
}

// out[i] = s_i * g2 for canonical Fr scalars (32 B little-endian each)
__global__ void __launch_bounds__(64) k_g2_mul(const uint8_t* __restrict__ sc, G2Aff g2, G2Aff* __restrict__ out,
                                               uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* s = reinterpret_cast<const uint32_t*>(sc + (size_t)i * 32);
  G2Jac acc = G2Jac::inf();
  for (int w = 7; w >= 0; --w) {
    const uint32_t word = s[w];
#pragma unroll 1
    for (int b = 31; b >= 0; --b) {
      acc = acc.dbl();
      if ((word >> b) & 1) acc = acc.add_affine(g2.x, g2.y);
    }
  }
  out[i] = acc.to_affine();
}

// Byte offsets inside one serialized EncodedSlice (the layout k_slices writes):
//   0 index | 8 amt.index | 16 commitment | 80 row.index | 88 row len | 96 row
//   | proof len | LR x (commitment_d, quotient_d) | high | roots[3] | proof len
//   | LR x sibling | leaf_index | leaf
struct SliceOffsets {
  uint32_t row, proof, high, roots, mproof, leaf_index, leaf, size;
  __host__ __device__ SliceOffsets(int lr, int lc) {
    row = 96;
    proof = row + (32u << lc) + 8;
    high = proof + 128u * lr;
    roots = high + 64;
    mproof = roots + 96 + 8;
    leaf_index = mproof + 32u * lr;
    leaf = leaf_index + 8;
    size = leaf + 32;
  }
};

__device__ __forceinline__ void keccak_pair(const uint8_t* a, const uint8_t* b, uint8_t* out) {
  uint64_t in[8], h[4];
  for (int k = 0; k < 4; ++k) {
    uint64_t x = 0, y = 0;
    for (int t = 0; t < 8; ++t) {
      x |= (uint64_t)a[8 * k + t] << (8 * t);
      y |= (uint64_t)b[8 * k + t] << (8 * t);
    }
    in[k] = x;
    in[4 + k] = y;
  }
  keccak256_64(in, h);
  for (int k = 0; k < 4; ++k)
    for (int t = 0; t < 8; ++t) out[8 * k + t] = (uint8_t)(h[k] >> (8 * t));
}

// Merkle part of EncodedSlice::verify (merkle/slice.rs:50-104) in the
// reference's order: file root of the slice's roots, leaf index range, the
// row's local root against the leaf, the sibling path against
// roots[leaf_index / R]. Slice j of the batch starts at slices + j * stride
// (16-byte aligned) with the standard layout up to its Merkle proof, whose
// length is nproof[j]. One CTA of 128 threads per slice.
__global__ void __launch_bounds__(128) k_verify_merkle(const uint8_t* __restrict__ slices, uint64_t stride, int lr,
                                                       int lc, const uint32_t* __restrict__ nproof,
                                                       const uint8_t* __restrict__ auth_root,
                                                       int32_t* __restrict__ code) {
  __shared__ __align__(16) uint8_t nodes[2][128 * 32];
  __shared__ int bad_root;
  const SliceOffsets L(lr, lc);
  const uint8_t* s = slices + (uint64_t)blockIdx.x * stride;
  const uint32_t np = nproof[blockIdx.x];  // sibling count (LR in a well-formed slice)
  const uint32_t li_off = L.mproof + 32 * np;
  const uint32_t C = 1u << lc, R = 1u << lr;
  const uint32_t nleaf = C / 8;  // <= 128
  if (threadIdx.x == 0) {
    uint8_t h01[32], fr[32];
    keccak_pair(s + L.roots, s + L.roots + 32, h01);
    keccak_pair(h01, s + L.roots + 64, fr);
    int bad = 0;
    for (int k = 0; k < 32; ++k) bad |= fr[k] != auth_root[k];
    bad_root = bad;
  }
  // leaves: keccak256 of 8 consecutive 32-byte items of the row
  for (uint32_t j = threadIdx.x; j < nleaf; j += blockDim.x) {
    const uint64_t* src = reinterpret_cast<const uint64_t*>(s + L.row + (size_t)j * 256);
    uint64_t in[32], h[4];
    for (int k = 0; k < 32; ++k) in[k] = src[k];
    keccak256_256(in, h);
    uint64_t* d = reinterpret_cast<uint64_t*>(nodes[0] + 32 * j);
    for (int k = 0; k < 4; ++k) d[k] = h[k];
  }
  __syncthreads();
  int cur = 0;
  for (uint32_t cnt = nleaf; cnt > 1; cnt >>= 1) {
    for (uint32_t j = threadIdx.x; j < cnt / 2; j += blockDim.x)
      keccak_pair(nodes[cur] + 64 * j, nodes[cur] + 64 * j + 32, nodes[cur ^ 1] + 32 * j);
    __syncthreads();
    cur ^= 1;
  }
  if (threadIdx.x != 0) return;
  int32_t c = 0;
  uint64_t li = 0;
  for (int t = 0; t < 8; ++t) li |= (uint64_t)s[li_off + t] << (8 * t);
  if (bad_root) c = 20;
  else if (li >= 3ull * R) c = 22;
  else {
    int diff = 0;
    for (int k = 0; k < 32; ++k) diff |= nodes[cur][k] != s[li_off + 8 + k];
    if (diff) c = 23;
    else {
      uint8_t acc[32];
      for (int k = 0; k < 32; ++k) acc[k] = s[li_off + 8 + k];
      uint64_t pos = li % R;
      for (uint32_t d = 0; d < np; ++d) {
        const uint8_t* sib = s + L.mproof + 32 * d;
        uint8_t nxt[32];
        if (pos & 1) keccak_pair(sib, acc, nxt);
        else keccak_pair(acc, sib, nxt);
        for (int k = 0; k < 32; ++k) acc[k] = nxt[k];
        pos >>= 1;
      }
      const uint8_t* root = s + L.roots + 32 * (li / R);
      int pd = 0;
      for (int k = 0; k < 32; ++k) pd |= acc[k] != root[k];
      if (pd) c = 24;
    }
  }
  code[blockIdx.x] = c;
}

// scal[coset(j)][bi(j) C + t] = alpha_j * row_j[bitrev(t)] (canonical), row_j
// the row of the slice at position pos[j] of the batch buffer: the
// scalars of the batch's MSM checks (the row is index_reverse'd, encode.rs:225-241).
// alpha in Montgomery form, so one product gives the canonical result.
__global__ void __launch_bounds__(256) k_verify_scalars(const uint8_t* __restrict__ slices, uint64_t stride,
                                                        const uint32_t* __restrict__ pos, int lc,
                                                        const uint32_t* __restrict__ coset,
                                                        const uint32_t* __restrict__ bi, const Fr* __restrict__ alpha,
                                                        uint8_t* __restrict__ scal, uint64_t coset_stride) {
  const uint32_t j = blockIdx.x;
  const uint32_t C = 1u << lc;
  const Fr* row = reinterpret_cast<const Fr*>(slices + (uint64_t)pos[j] * stride + 96);
  const Fr a = alpha[j];
  Fr* dst = reinterpret_cast<Fr*>(scal + coset[j] * coset_stride) + (size_t)bi[j] * C;
  for (uint32_t t = threadIdx.x; t < C; t += blockDim.x) dst[t] = load_fr(row + brev_bits(t, lc)) * a;
}

}  // namespace zg
