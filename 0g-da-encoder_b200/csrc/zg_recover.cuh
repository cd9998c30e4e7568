// Erasure recovery of the original blob from any >= R encoded rows
// (crates/recovery/src/lib.rs:15-43, data_poly.rs:72-118).
//
// The reference decodes over the full 4N-point domain (4 cosets, the fourth
// virtual and always erased): Z = prod over erased rows of (x^C - c_row),
// D*Z interpolated, D = (D*Z)/Z on a shifted coset, then D on coset 0. The
// result is the unique data polynomial, so it is computed here in factored
// form. Write D(x) = sum_{s<C} x^s P_s(x^C) with deg P_s < R. Encoded row r of
// coset c holds D at g_c w^r v^j (v = w^R), so a C-point inverse NTT of the
// row gives (g_c w^r)^s P_s(y) at y = (g_c w^r)^C = W^(4r + pi(c)), W the
// 4R-th root of unity, pi = (0, 2, 1) for cosets 0, 1, 2 (and 3 for the
// virtual coset, whose rows are always erased). Each column s is then an
// erasure decode of a degree < R polynomial over the 4R-point domain with the
// same erased set for every s:
//   Z(y) = prod_{e erased} (y - W^e);  G = P_s Z is known on all 4R points
//   (zero where Z vanishes) and has degree < R + #erased <= 4R;
//   P_s = G / Z evaluated on k W^i (k = 5, no zero of Z there), interpolated,
//   then evaluated at the R points W^{4r} of coset 0.
// Finally row r of the data is the C-point NTT of w^{rs} P_s(W^{4r}).
#pragma once
#include "zg_kernels.cuh"

namespace zg {

// domain index of encoded row `id` (coset c = id / R, row r = id % R)
__device__ __forceinline__ uint32_t rec_domain_index(uint32_t id, int lr) {
  const uint32_t c = id >> lr, r = id & ((1u << lr) - 1);
  const uint32_t pi = (c == 1) ? 2u : (c == 2 ? 1u : c);
  return 4 * r + pi;
}

// Per received row: canonical check, inverse C-point NTT, times g_c^{-s} / C
// and w^{-r s}; writes V[s][4r + pi(c)] (Montgomery). err bit 0: a value >= r.
__global__ void __launch_bounds__(256) k_rec_rows(const uint8_t* __restrict__ rows, const uint32_t* __restrict__ ids,
                                                  Fr* __restrict__ V, int lr, int lc,
                                                  const Fr* __restrict__ twi_c, const Fr* __restrict__ ginv,
                                                  const Fr* __restrict__ wni_lo, const Fr* __restrict__ wni_hi,
                                                  uint32_t* __restrict__ err) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int C = 1 << lc;
  const uint32_t M = 4u << lr;
  Fr* s = reinterpret_cast<Fr*>(smem);
  const uint32_t id = ids[blockIdx.x];
  const uint32_t c = id >> lr, r = id & ((1u << lr) - 1);
  const Fr* src = reinterpret_cast<const Fr*>(rows) + (size_t)blockIdx.x * C;
  auto get = [&](int j) {
    Fr x = load_fr(src + j);
    Fr d;
    if (!Fr::sub_raw(d, x, Fr::modulus())) {  // x >= r
      atomicOr(err, 1u);
      x = Fr::zero();
    }
    return Fr::from_canonical(x);
  };
  const uint32_t di = rec_domain_index(id, lr);
  const uint32_t nmask = (1u << (lr + lc)) - 1;
  ntt_block(s, lc, twi_c, get, [&](int k, const Fr& x) {
    V[(size_t)k * M + di] = x * ginv[(size_t)c * C + k] * pow_split(wni_lo, wni_hi, (uint32_t)k * r, lc, nmask);
  });
}

// zw[i] = Z(W^i) (zero at the erased points) and zinv[i] = 1 / Z(k W^i),
// Z(y) = prod_{e in erased} (y - W^e)
__global__ void k_rec_zinv(const uint16_t* __restrict__ erased, uint32_t ne, const Fr* __restrict__ wpow,
                           Fr k, Fr* __restrict__ zw, Fr* __restrict__ zinv, uint32_t M) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const Fr x = wpow[i], y = k * x;
  Fr z = Fr::one(), zx = Fr::one();
  for (uint32_t e = 0; e < ne; ++e) {
    const Fr we = wpow[erased[e]];
    z = z * (y - we);
    zx = zx * (x - we);
  }
  zw[i] = zx;
  zinv[i] = z.inverse();
}

// Per column s: decode P_s from its 4R samples (zeros at erased points), then
// W_out[r][s] = w^{r s} P_s(W^{4r}). err bit 1: a coefficient >= R is nonzero
// (the rows are not one codeword).
__global__ void __launch_bounds__(256) k_rec_cols(const Fr* __restrict__ V, Fr* __restrict__ Wout, int lr, int lc,
                                                  const Fr* __restrict__ twf_m, const Fr* __restrict__ twi_m,
                                                  const Fr* __restrict__ kpow, const Fr* __restrict__ kinv,
                                                  const Fr* __restrict__ zw, const Fr* __restrict__ zinv, const Fr* __restrict__ twf_r,
                                                  const Fr* __restrict__ wn_lo, const Fr* __restrict__ wn_hi,
                                                  uint32_t* __restrict__ err) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int lm = lr + 2;
  const uint32_t M = 1u << lm, R = 1u << lr, C = 1u << lc;
  Fr* a = reinterpret_cast<Fr*>(smem);
  const uint32_t col = blockIdx.x;
  const Fr* src = V + (size_t)col * M;
  // G = P_s Z on W^i (zero at the erased points, where Z vanishes) -> coefficients
  // then evaluate G(k W^i): coefficient j times k^j / M (the inverse
  // transform's 1/M), in place (the last pass writes where it read)
  ntt_block(a, lm, twi_m, [&](int i) { return load_fr(src + i) * zw[i]; },
            [&](int j, const Fr& x) { a[j] = x * kpow[j]; });
  // bit-reverse permute in place for the next DIT pass
  for (uint32_t j = threadIdx.x; j < M; j += blockDim.x) {
    uint32_t rj = brev_bits(j, lm);
    if (j < rj) {
      Fr t = a[j];
      a[j] = a[rj];
      a[rj] = t;
    }
  }
  __syncthreads();
  ntt_smem(a, lm, twf_m);
  // P_s(k W^i) = G(k W^i) / Z(k W^i)
  for (uint32_t i = threadIdx.x; i < M; i += blockDim.x) a[i] = a[i] * zinv[i];
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < M; j += blockDim.x) {
    uint32_t rj = brev_bits(j, lm);
    if (j < rj) {
      Fr t = a[j];
      a[j] = a[rj];
      a[rj] = t;
    }
  }
  __syncthreads();
  ntt_smem(a, lm, twi_m);
  // coefficients of P_s(k x), times k^{-j} / M -> coefficients of P_s.
  // Coefficient j of P_s is the x^(s + C j) term of D. The reference accepts
  // deg D <= N (data_poly.rs:111) and evaluates on coset 0, where x^N = 1;
  // any higher term means the rows are not one codeword.
  for (uint32_t j = threadIdx.x; j < M; j += blockDim.x) {
    Fr v = a[j] * kinv[j];
    if ((j > R || (j == R && col > 0)) && !v.is_zero()) atomicOr(err, 2u);
    a[j] = v;
  }
  __syncthreads();
  // P_s at W^{4r} = w_R^r for r < R: R-point forward transform of the first R
  // coefficients (the x^N term of column 0 folds onto x^0)
  Fr* b = a + M;  // second buffer of R entries
  const uint32_t nmask = (1u << (lr + lc)) - 1;
  ntt_block(b, lr, twf_r, [&](int j) { return (j == 0 && col == 0) ? a[0] + a[R] : a[j]; },
            [&](int r, const Fr& x) {
              Wout[(size_t)r * C + col] = x * pow_split(wn_lo, wn_hi, col * (uint32_t)r, lc, nmask);
            });
}

// Row r of the data: C-point NTT of Wout[r][*], canonical, packed into the
// 31-byte chunks of RawData. err bit 2: an element's byte 31 is nonzero
// ("Incorrect scalar", raw_blob.rs:46-50).
__global__ void __launch_bounds__(256) k_rec_out(const Fr* __restrict__ Win, uint8_t* __restrict__ raw, int lc,
                                                 const Fr* __restrict__ twf_c, uint32_t* __restrict__ err) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int C = 1 << lc;
  Fr* s = reinterpret_cast<Fr*>(smem);
  const uint32_t r = blockIdx.x;
  ntt_block(s, lc, twf_c, [&](int k) { return load_fr(Win + (size_t)r * C + k); }, [&](int j, const Fr& v) {
    Fr x = v.to_canonical();
    if (x.v[7] >> 24) atomicOr(err, 4u);
    uint8_t* dst = raw + 31 * ((size_t)r * C + j);
#pragma unroll
    for (int t = 0; t < 31; ++t) dst[t] = (uint8_t)(x.v[t >> 2] >> (8 * (t & 3)));
  });
}

}  // namespace zg
