// Device kernels of the blob-encoding path.
//
// Layout in HBM for one blob of R = 2^LR rows and C = 2^LC columns
// (N = R*C scalars; production R = C = 1024):
//   enc   [3][R][C] x 32 B   encoded rows, canonical little-endian Fr, coset-
//                             major then row-major: the reference's
//                             EncodedBlob::get_data() order (amt/blob.rs:29-40)
//   T1    [R][C]   Fr(mont)  row-iNTT output of the original rows
//   Bc    [2][R][C] Fr(mont) column pass output for cosets 1, 2 (transposed)
//   bases [3][L][N] G1 affine (Montgomery x||y, 64 B), L = LR + 2 lines in the
//                             order quotients[0..LR), basis, high_basis (the
//                             upload order of prove_gpu.rs:42-47)
//   win   [3][L][R][32] XYZZ  per-chunk MSM window sums
//   amt   [3][4R-2] 64 B     AMT outputs, ark uncompressed G1
//   tree  levels of the Merkle tree (level d holds 3*2^d nodes)
#pragma once
#include <stdint.h>

#include "zg_curve.cuh"
#include "zg_keccak.cuh"

namespace zg {

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, int bits) {
  return bits == 0 ? 0u : (__brev(x) >> (32 - bits));
}

// ---------------------------------------------------------------------------
// Shared-memory DIT NTT in radix-4 passes; s[] holds the input in
// bit-reversed order. Result in natural order. Stage st pairs elements
// half = 2^(st-1) apart with twiddle w^((n >> st) * (i mod half)), w the
// n-th root in use. The twiddles are stored stage by stage: tw[half + i] =
// w^((n >> st) * i) for i < half (tw[0] = 1, n entries in all), so the
// threads of a warp read consecutive entries at every stage instead of
// entries n >> st apart. A pass runs two stages st, st + 1 in
// registers: each thread takes the four elements base + j h (h = 2^(st-1),
// base with bits st-1 and st clear), so the pass reads and writes shared
// memory once instead of twice and needs one barrier instead of two; n / 4
// groups keep a 256-thread CTA busy on a 1024-point transform. An odd last
// stage runs as a radix-2 pass. (Radix-2^3 passes, eight elements per
// thread, measured slower: 1.56 against 1.32 ms for the RS extension, with
// half the threads of a 1024-point transform idle and registers spilled.)
template <class F>
__device__ __forceinline__ void ntt_bfly(F& a, F& b, const F& w) {
  const F v = b * w;
  b = a - v;
  a = a + v;
}

// one radix-4 pass over stages st and st + 1 of the transform in s;
// out(i, x) receives element i of the pass's result
template <class F, class Out>
__device__ __forceinline__ void ntt_r4_pass(const F* s, int logn, int st, const F* __restrict__ tw, Out out) {
  const int n = 1 << logn;
  const int h = 1 << (st - 1);
  for (int g = threadIdx.x; g < (n >> 2); g += blockDim.x) {
    const int k0 = g & (h - 1);
    const int base = ((g >> (st - 1)) << (st + 1)) + k0;
    F x0 = s[base], x1 = s[base + h], x2 = s[base + 2 * h], x3 = s[base + 3 * h];
    // each stage's two twiddle products are independent: one interleaved
    // pair of carry chains (F::mul2) instead of two products in a row
    // (a pair with one product on the FP64 pipe measured slower here: 108
    // registers against 64 halve the resident CTAs)
    const F w1 = tw[h + k0];
    F v, u;
    F::mul2(x1, w1, x3, w1, v, u);
    x1 = x0 - v;
    x0 = x0 + v;
    x3 = x2 - u;
    x2 = x2 + u;
    F::mul2(x2, tw[2 * h + k0], x3, tw[3 * h + k0], v, u);
    out(base, x0 + v);
    out(base + h, x1 + u);
    out(base + 2 * h, x0 - v);
    out(base + 3 * h, x1 - u);
  }
  __syncthreads();
}

// the last stage alone (odd logn): radix-2
template <class F, class Out>
__device__ __forceinline__ void ntt_r2_pass(const F* s, int logn, const F* __restrict__ tw, Out out) {
  const int h = 1 << (logn - 1);
  for (int g = threadIdx.x; g < h; g += blockDim.x) {
    F a = s[g], b = s[g + h];
    ntt_bfly(a, b, tw[h + g]);
    out(g, a);
    out(g + h, b);
  }
  __syncthreads();
}

// In-place transform of s[] (input in bit-reversed order).
template <class F>
__device__ __forceinline__ void ntt_smem(F* s, int logn, const F* __restrict__ tw) {
  auto to_s = [s](int i, const F& x) { s[i] = x; };
  int st = 1;
  for (; st + 1 <= logn; st += 2) ntt_r4_pass(s, logn, st, tw, to_s);
  if (st == logn) ntt_r2_pass(s, logn, tw, to_s);
}

// Transform of n = 2^logn elements with its input and output fused into the
// first and last passes: element i of the natural-order input is get(i)
// (called once per element), element k of the result goes to put(k, x)
// (once per element); s[] is n elements of scratch that neither get nor put
// may touch. The first pass reads its four inputs straight from get: the
// group at bit-reversed positions 4g .. 4g+3 holds the natural elements
// t, t + n/2, t + n/4, t + 3n/4 for g = bitrev(t), so thread t loads them
// (coalesced across threads) and runs stages 1 and 2 in registers, whose
// twiddles are 1 except w^(n/4): one product instead of four, and no pass of
// its own over shared memory. The last pass writes its results to put instead
// of back to s. Ends with a barrier.
template <class F, class Get, class Put>
__device__ __forceinline__ void ntt_block(F* s, int logn, const F* __restrict__ tw, Get get, Put put) {
  if (logn < 2) {
    if (threadIdx.x == 0) {
      F a = get(0);
      if (logn == 1) {
        F b = get(1);
        ntt_bfly(a, b, tw[1]);
        put(1, b);
      }
      put(0, a);
    }
    __syncthreads();
    return;
  }
  const int q = 1 << (logn - 2);
  const F wq = tw[3];  // w^(n/4), stage 2's second twiddle
  for (int t = threadIdx.x; t < q; t += blockDim.x) {
    const F x0 = get(t), x1 = get(t + 2 * q), x2 = get(t + q), x3 = get(t + 3 * q);
    const F y0 = x0 + x1, y1 = x0 - x1, y2 = x2 + x3;
    const F u = (x2 - x3) * wq;
    if (logn == 2) {
      put(0, y0 + y2);
      put(1, y1 + u);
      put(2, y0 - y2);
      put(3, y1 - u);
    } else {
      const int b = (int)brev_bits(t, logn - 2) << 2;
      s[b] = y0 + y2;
      s[b + 1] = y1 + u;
      s[b + 2] = y0 - y2;
      s[b + 3] = y1 - u;
    }
  }
  __syncthreads();
  if (logn == 2) return;
  auto to_s = [s](int i, const F& x) { s[i] = x; };
  int st = 3;
  for (; st + 2 <= logn; st += 2) ntt_r4_pass(s, logn, st, tw, to_s);
  if (st + 1 == logn)
    ntt_r4_pass(s, logn, st, tw, put);
  else
    ntt_r2_pass(s, logn, tw, put);
}

__device__ __forceinline__ Fr load_fr(const Fr* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  uint4 a = q[0], b = q[1];
  Fr r;
  r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
  r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
  return r;
}
__device__ __forceinline__ void store_fr(Fr* p, const Fr& x) {
  uint4* q = reinterpret_cast<uint4*>(p);
  q[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
  q[1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

// w_N^e from the split tables lo[e & (C-1)] * hi[e >> LC]
__device__ __forceinline__ Fr pow_split(const Fr* lo, const Fr* hi, uint32_t e, int lc, uint32_t nmask) {
  e &= nmask;
  return lo[e & ((1u << lc) - 1)] * hi[e >> lc];
}

// The three passes work on canonical values without converting them to
// Montgomery form and back: every step is linear in the data and multiplies
// only by constants stored in Montgomery form (twiddles, coset powers, 1/N),
// and a Montgomery product of a canonical x with c R is the canonical x c;
// so canonical data in gives the canonical extension out (the products a
// conversion would cost, 3 per element of a coset, are saved).
//
// Pass 1: original row r -> canonical enc[0][r][*], and
// T1[r][s] = w_N^{-s r} * sum_j v_C^{-s j} D[r][j].
// D[r][j] is the Fr of the 31-byte chunk r*C + j of the zero-padded RawData
// whose last four bytes hold the payload length (raw_data.rs:55-73,
// raw_blob.rs:33-40).
// The payload length is `len`, or *d_len when d_len is set (graph launches,
// whose parameters are fixed at capture).
//
// 80 registers per thread (a few bytes spilled): three 256-thread CTAs per
// SM, as the shared memory allows (96 registers unbounded: two, and 5 %
// slower).
__global__ void __maxnreg__(80) k_rows_from_raw(const uint8_t* __restrict__ raw, uint64_t len,
                                                       const uint64_t* __restrict__ d_len, uint64_t max_raw, int lr,
                                                       int lc, uint8_t* __restrict__ enc0, Fr* __restrict__ T1,
                                                       const Fr* __restrict__ twi_c, const Fr* __restrict__ wni_lo,
                                                       const Fr* __restrict__ wni_hi) {
  extern __shared__ __align__(16) uint8_t smem[];
  if (d_len) len = *d_len;
  const int C = 1 << lc;
  const uint32_t r = blockIdx.x;
  Fr* s = reinterpret_cast<Fr*>(smem);
  uint8_t* bytes = smem + (size_t)C * sizeof(Fr);
  const uint64_t base = (uint64_t)31 * r * C;
  const uint32_t nbytes = 31u * C;
  // the row's bytes: whole 16-byte words straight from raw while they lie
  // inside the payload (raw and the row start 16-byte aligned), the rest
  // (payload end, zero padding, length trailer) byte by byte
  uint32_t done = 0;
  if (((reinterpret_cast<uintptr_t>(raw) | base) & 15) == 0 && len > base) {
    const uint32_t nv = (uint32_t)(min(len - base, (uint64_t)nbytes) >> 4);
    const uint4* src = reinterpret_cast<const uint4*>(raw + base);
    uint4* dst = reinterpret_cast<uint4*>(bytes);
#pragma unroll 4
    for (uint32_t i = threadIdx.x; i < nv; i += blockDim.x) dst[i] = src[i];
    done = nv << 4;
  }
  for (uint32_t i = done + threadIdx.x; i < nbytes; i += blockDim.x) {
    uint64_t o = base + i;
    uint8_t v = 0;
    if (o < len) v = raw[o];
    else if (o >= max_raw) v = (uint8_t)(len >> (8 * (o - max_raw)));
    bytes[i] = v;
  }
  __syncthreads();
  // element j: bytes 31 j .. 31 j + 30 as eight little-endian words, cut
  // from the nine aligned words that hold them (the buffer has 16 bytes of
  // slack behind the last element); unpacked once, stored to enc0
  // (canonical: the passes are linear, see above) and handed to the transform
  auto get = [&](int j) {
    // one element's loads at a time (hoisting all four elements' 36 word
    // loads ahead would cost a resident CTA per SM in registers)
    asm volatile("" ::: "memory");
    const uint32_t off = 31u * (uint32_t)j;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(bytes) + (off >> 2);
    const uint32_t sh = (off & 3) * 8;
    Fr x;
#pragma unroll
    for (int k = 0; k < 8; ++k) x.v[k] = __funnelshift_r(w[k], w[k + 1], sh);
    x.v[7] &= 0x00ffffffu;
    store_fr(reinterpret_cast<Fr*>(enc0) + ((size_t)r * C + j), x);
    return x;
  };
  // the result stays in s and takes its twiddles in a loop of its own (in
  // the last pass the table loads and two products per element raise the
  // registers past three resident CTAs)
  ntt_block(s, lc, twi_c, get, [&](int k, const Fr& x) { s[k] = x; });
  const uint32_t nmask = (1u << (lr + lc)) - 1;
  for (int k = threadIdx.x; k < C; k += blockDim.x)
    store_fr(T1 + (size_t)r * C + k, s[k] * pow_split(wni_lo, wni_hi, (uint32_t)k * r, lc, nmask));
}

// Pass 2: per column s, iNTT over rows (size R), then per extension coset
// c in {1, 2}: scale coefficient m = s + C q by g_c^m / N, forward NTT over q,
// multiply by w_N^{s r}; store Bc[c-1][r][s].
// One CTA handles `cpb` consecutive columns one after the other (a tuning
// knob: fewer, longer CTAs against more, shorter ones).
// 80 registers per thread: three 256-thread CTAs per SM (107 unbounded: two,
// and 4 % slower).
__global__ void __maxnreg__(80) k_cols(const Fr* __restrict__ T1, Fr* __restrict__ Bc, int lr, int lc,
                       const Fr* __restrict__ twi_r, const Fr* __restrict__ twf_r,
                       const Fr* __restrict__ gs_lo, const Fr* __restrict__ gs_hi,
                       const Fr* __restrict__ wn_lo, const Fr* __restrict__ wn_hi, int cpb) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int R = 1 << lr, C = 1 << lc;
  Fr* coef = reinterpret_cast<Fr*>(smem);
  Fr* work = coef + (size_t)R;
  const uint32_t nmask = (1u << (lr + lc)) - 1;
  for (int cc = 0; cc < cpb; ++cc) {
    const uint32_t s = blockIdx.x * cpb + cc;
    if (s >= (uint32_t)C) break;
    // coefficients of column s (in place in coef, its own scratch: the last
    // pass writes each element where it read it)
    ntt_block(coef, lr, twi_r, [&](int r) { return load_fr(T1 + (size_t)r * C + s); },
              [&](int k, const Fr& x) { coef[k] = x; });
    for (int c = 0; c < 2; ++c) {
      const Fr glo = gs_lo[c * C + s];
      ntt_block(work, lr, twf_r, [&](int q) { return coef[q] * glo * gs_hi[c * R + q]; },
                [&](int r, const Fr& x) { work[r] = x; });
      for (int r = threadIdx.x; r < R; r += blockDim.x)
        store_fr(Bc + ((size_t)c * R + r) * C + s, work[r] * pow_split(wn_lo, wn_hi, s * (uint32_t)r, lc, nmask));
      __syncthreads();
    }
  }
}

// Pass 3: per coset c in {1,2} and row r, forward NTT over s (size C):
// enc[c][r][j] = canonical( sum_s v_C^{s j} Bc[c-1][r][s] ).
__global__ void __launch_bounds__(512) k_rows_ntt(const Fr* __restrict__ Bc, uint8_t* __restrict__ enc, int lr, int lc,
                           const Fr* __restrict__ twf_c) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int R = 1 << lr, C = 1 << lc;
  const uint32_t r = blockIdx.x, c = blockIdx.y;
  Fr* s = reinterpret_cast<Fr*>(smem);
  const Fr* src = Bc + ((size_t)c * R + r) * C;
  Fr* dst = reinterpret_cast<Fr*>(enc) + ((size_t)(c + 1) * R + r) * C;
  ntt_block(s, lc, twf_c, [&](int k) { return load_fr(src + k); }, [&](int j, const Fr& x) { store_fr(dst + j, x); });
}

// ---------------------------------------------------------------------------
// MSM over per-row chunks (the decomposition of prove_gpu.rs:55-87: for every
// line l and chunk b, the MSM of the C scalars of chunk b against
// bases[l][b*C .. (b+1)*C)). Chunk b of the bit-reversed coset vector is
// encoded row bitrev(b), element t is column bitrev(t)
// (HalfBlob::generate, crates/amt/src/blob/encode.rs:171-183).
//
// Signed 8-bit windows: 32 windows, digits in [-128, 127], buckets 1..128.
// One CTA per (chunk, coset): the digits of the chunk's C scalars are
// counting-sorted into per-window bucket lists once and reused for all L
// lines. Thread (line li, window w, segment g) owns buckets 64g+1..64g+64 of
// one window: it sums each bucket from the affine bases and folds it into
// running sums, so no bucket array is materialised; the two segments of a
// window meet through a warp shuffle.
constexpr int MSM_WINDOWS = 32;
constexpr int MSM_THREADS = 256;
constexpr int MSM_LINES_PER_PASS = MSM_THREADS / (MSM_WINDOWS * 2);

__device__ __forceinline__ XYZZ shfl_down_xyzz(const XYZZ& p, int delta) {
  XYZZ r;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    r.X.v[i] = __shfl_down_sync(0xffffffffu, p.X.v[i], delta);
    r.Y.v[i] = __shfl_down_sync(0xffffffffu, p.Y.v[i], delta);
    r.ZZ.v[i] = __shfl_down_sync(0xffffffffu, p.ZZ.v[i], delta);
    r.ZZZ.v[i] = __shfl_down_sync(0xffffffffu, p.ZZZ.v[i], delta);
  }
  return r;
}

__device__ __forceinline__ G1Aff load_aff(const G1Aff* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  uint4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
  G1Aff r;
  r.x.v[0] = a.x; r.x.v[1] = a.y; r.x.v[2] = a.z; r.x.v[3] = a.w;
  r.x.v[4] = b.x; r.x.v[5] = b.y; r.x.v[6] = b.z; r.x.v[7] = b.w;
  r.y.v[0] = c.x; r.y.v[1] = c.y; r.y.v[2] = c.z; r.y.v[3] = c.w;
  r.y.v[4] = d.x; r.y.v[5] = d.y; r.y.v[6] = d.z; r.y.v[7] = d.w;
  return r;
}

__device__ __forceinline__ void store_xyzz(XYZZ* p, const XYZZ& x) {
  store_fr(reinterpret_cast<Fr*>(&p->X), *reinterpret_cast<const Fr*>(&x.X));
  store_fr(reinterpret_cast<Fr*>(&p->Y), *reinterpret_cast<const Fr*>(&x.Y));
  store_fr(reinterpret_cast<Fr*>(&p->ZZ), *reinterpret_cast<const Fr*>(&x.ZZ));
  store_fr(reinterpret_cast<Fr*>(&p->ZZZ), *reinterpret_cast<const Fr*>(&x.ZZZ));
}
__device__ __forceinline__ XYZZ load_xyzz(const XYZZ* p) {
  XYZZ r;
  Fr a = load_fr(reinterpret_cast<const Fr*>(&p->X));
  Fr b = load_fr(reinterpret_cast<const Fr*>(&p->Y));
  Fr c = load_fr(reinterpret_cast<const Fr*>(&p->ZZ));
  Fr d = load_fr(reinterpret_cast<const Fr*>(&p->ZZZ));
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    r.X.v[i] = a.v[i]; r.Y.v[i] = b.v[i]; r.ZZ.v[i] = c.v[i]; r.ZZZ.v[i] = d.v[i];
  }
  return r;
}

struct MsmChunkArgs {
  const uint8_t* scalars;  // canonical 32 B scalars
  const G1Aff* bases;      // [cosets][L][N]
  XYZZ* win;               // [cosets][L][nchunks][32]
  int lr, lc;              // nchunks = 2^lr, chunk = 2^lc
  int lines;               // L
  int bitrev_rows;         // 1: chunk b reads encoded row bitrev(b), column bitrev(t)
  uint64_t scalar_coset_stride;  // scalars between cosets (elements)
  uint64_t base_coset_stride;    // bases between cosets (points)
  uint64_t base_line_stride;     // bases between lines (points)
};

__global__ void __launch_bounds__(MSM_THREADS, 1) k_msm_chunks(MsmChunkArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int C = 1 << a.lc;
  const uint32_t b = blockIdx.x, coset = blockIdx.y;
  // smem: scalars [C][8] u32 | lists [32][C] u16 | offs [32][129] u16 | cnt [129] u32
  uint32_t* scal = reinterpret_cast<uint32_t*>(smem);
  uint16_t* lists = reinterpret_cast<uint16_t*>(scal + (size_t)C * 8);
  uint16_t* offs = lists + (size_t)MSM_WINDOWS * C;
  uint32_t* cnt = reinterpret_cast<uint32_t*>(offs + MSM_WINDOWS * 129 + (MSM_WINDOWS * 129) % 2);

  const uint32_t row = a.bitrev_rows ? brev_bits(b, a.lr) : b;
  const uint8_t* src = a.scalars + (a.scalar_coset_stride * coset + (uint64_t)row * C) * 32;
  for (int t = threadIdx.x; t < C; t += blockDim.x) {
    uint32_t col = a.bitrev_rows ? brev_bits(t, a.lc) : t;
    const uint4* q = reinterpret_cast<const uint4*>(src + (size_t)col * 32);
    uint4 x = q[0], y = q[1];
    uint32_t* d = scal + (size_t)t * 8;
    d[0] = x.x; d[1] = x.y; d[2] = x.z; d[3] = x.w; d[4] = y.x; d[5] = y.y; d[6] = y.z; d[7] = y.w;
  }
  __syncthreads();

  // signed-digit decomposition + per-window counting sort
  constexpr int MAXPER = 8;  // supports C <= 2048
  uint32_t carry_bits = 0;   // bit i: carry of this thread's i-th scalar
  for (int w = 0; w < MSM_WINDOWS; ++w) {
    for (int k = threadIdx.x; k <= 128; k += blockDim.x) cnt[k] = 0;
    __syncthreads();
    int digs[MAXPER];
#pragma unroll
    for (int i = 0; i < MAXPER; ++i) {
      int t = threadIdx.x + i * blockDim.x;
      digs[i] = 0;
      if (t < C) {
        uint32_t byte = (scal[(size_t)t * 8 + (w >> 2)] >> (8 * (w & 3))) & 0xff;
        uint32_t v = byte + ((carry_bits >> i) & 1);
        int d;
        if (v >= 128) { d = (int)v - 256; carry_bits |= 1u << i; }
        else { d = (int)v; carry_bits &= ~(1u << i); }
        digs[i] = d;
        if (d) atomicAdd(&cnt[d < 0 ? -d : d], 1u);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t acc = 0;
      for (int k = 1; k <= 128; ++k) {
        offs[w * 129 + k - 1] = (uint16_t)acc;
        uint32_t c = cnt[k];
        cnt[k] = acc;
        acc += c;
      }
      offs[w * 129 + 128] = (uint16_t)acc;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < MAXPER; ++i) {
      int t = threadIdx.x + i * blockDim.x;
      int d = digs[i];
      if (t < C && d) {
        uint32_t k = d < 0 ? -d : d;
        uint32_t pos = atomicAdd(&cnt[k], 1u);
        lists[(size_t)w * C + pos] = (uint16_t)(t | (d < 0 ? 0x8000 : 0));
      }
    }
    __syncthreads();
  }

  // bucket accumulation + window reduction
  const int li = threadIdx.x / (MSM_WINDOWS * 2);
  const int w = (threadIdx.x / 2) % MSM_WINDOWS;
  const int g = threadIdx.x & 1;
  const int nchunks = 1 << a.lr;
  for (int l0 = 0; l0 < a.lines; l0 += MSM_LINES_PER_PASS) {
    const int l = l0 + li;
    const bool active = l < a.lines;
    const G1Aff* bl = a.bases + a.base_coset_stride * coset + (size_t)(active ? l : 0) * a.base_line_stride +
                      (size_t)b * C;
    XYZZ run = XYZZ::inf(), acc = XYZZ::inf();
    if (active) {
      for (int k = 64 * g + 64; k > 64 * g; --k) {
        XYZZ bucket = XYZZ::inf();
        const int beg = offs[w * 129 + k - 1], end = offs[w * 129 + k];
        for (int e = beg; e < end; ++e) {
          uint32_t ent = lists[(size_t)w * C + e];
          G1Aff p = load_aff(bl + (ent & 0x7fff));
          if (ent & 0x8000) p.y = -p.y;
          bucket.add_affine(p.x, p.y);
        }
        run.add(bucket);
        acc.add(run);
      }
    }
    // window = acc0 + acc1 + 64 * run1   (segment 1 holds buckets 65..128)
    XYZZ acc1 = shfl_down_xyzz(acc, 1);
    XYZZ run1 = shfl_down_xyzz(run, 1);
    if (active && g == 0) {
#pragma unroll 1
      for (int i = 0; i < 6; ++i) run1 = run1.dbl();
      acc.add(acc1);
      acc.add(run1);
      store_xyzz(a.win + (((size_t)coset * a.lines + l) * nchunks + b) * MSM_WINDOWS + w, acc);
    }
  }
}


// ---------------------------------------------------------------------------
// MSM with fixed-base windows. The params never change, so every base P is
// stored with its window multiples T_w = 2^{11 w} P (w < 24): a chunk MSM
//   sum_t s_t P_t = sum_t sum_w d_{t,w} T_w[t]
// over the signed 11-bit digits d of the scalars is one bucket accumulation
// (buckets |d| = 1..1024) with no doublings. Per chunk: ~24 x 1024 mixed adds
// plus 2 x 1024 bucket-reduction adds, against 32 x (1024 + 256) for 8-bit
// windows with doublings.
constexpr int FB_BITS = 11;
constexpr int FB_WINDOWS = 24;                    // ceil((254 + 1) / 11)
constexpr int FB_BUCKETS = 1 << (FB_BITS - 1);    // 1024
constexpr int FB_ACC_THREADS = 128;
constexpr int FB_PER_THREAD = FB_BUCKETS / FB_ACC_THREADS;  // 8 buckets per thread
__host__ __device__ constexpr int fb_log2(int x) { return x <= 1 ? 0 : 1 + fb_log2(x / 2); }
constexpr int FB_PER_THREAD_LOG = fb_log2(FB_PER_THREAD);
constexpr int FB_ACC_MIN_CTAS = 512 / FB_ACC_THREADS;  // resident CTAs per SM at 128 registers

// Wide windows for the AMT lines whose nodes are MSMs over more than 1024
// points. Such a line's nodes are cut into sort units of U = 2^ulog points
// (11 <= ulog <= 15, U <= the node size) that share U buckets of signed
// (ulog + 1)-bit digits: W = floor(254 / c) + 1 windows of c = ulog + 1 bits,
// i.e. 16 bucket additions per point at U = 2^15 instead of 24, and the bucket
// reduction paid per unit instead of per 1024-point chunk. A unit's buckets
// are cut into U / 1024 blocks of FB_BUCKETS, each block one work item of
// k_fb_accum: with 1024 columns a (coset, line) still has exactly R items,
// item u * (U / 1024) + blk = block blk of unit u, and a node's items are
// contiguous, so the AMT tree kernel sums them like chunk results.
constexpr int WD_MIN_LOG = 11;
constexpr int WD_MAX_LOG = 15;
__host__ __device__ constexpr int wd_windows(int ulog) { return 254 / (ulog + 1) + 1; }
// The top digit of a scalar < r never carries out: (r - 1) >> ((W - 1) c) + 1
// < 2^(c - 1) for every c = 12 .. 16 (top values 3, 96, 3, 12388, 12388).
static_assert(wd_windows(15) == 16 && wd_windows(14) == 17 && wd_windows(13) == 19 && wd_windows(12) == 20 &&
                  wd_windows(11) == 22,
              "window counts");
__host__ __device__ constexpr uint64_t wd_unit_ents(int ulog) { return (uint64_t)wd_windows(ulog) << ulog; }

// col[(w + 1) * N] = 2^(BITS (w + 1)) * col[0] for w < WIN - 1: BITS
// doublings per window, then one batch inversion for the affine conversions.
template <int BITS, int WIN>
__device__ void fb_fill_windows(G1Aff* col, uint64_t N) {
  XYZZ pts[WIN - 1];
  XYZZ acc = XYZZ::from_affine(col[0]);
  for (int w = 1; w < WIN; ++w) {
#pragma unroll 1
    for (int k = 0; k < BITS; ++k) acc = acc.dbl();
    pts[w - 1] = acc;
  }
  // batch inversion of the ZZZ coordinates (bases are never infinity)
  Fq pre[WIN - 1];
  Fq run = Fq::one();
  for (int w = 0; w < WIN - 1; ++w) {
    pre[w] = run;
    run = MulHybrid::mul(run, pts[w].ZZZ);
  }
  Fq inv = run.inverse();
  for (int w = WIN - 2; w >= 0; --w) {
    Fq izzz = MulHybrid::mul(inv, pre[w]);
    inv = MulHybrid::mul(inv, pts[w].ZZZ);
    Fq izz = MulHybrid::mul(MulHybrid::mul(pts[w].ZZ, pts[w].ZZ), MulHybrid::mul(izzz, izzz));
    G1Aff a;
    a.x = MulHybrid::mul(pts[w].X, izz);
    a.y = MulHybrid::mul(pts[w].Y, izzz);
    col[(uint64_t)(w + 1) * N] = a;
  }
}

// window w's multiples: tab[(line * W + w) * N + p]; window 0 already holds the
// bases. One thread per (line, point).
__global__ void __launch_bounds__(128) k_fb_tables(G1Aff* tab, uint64_t N, uint64_t nlines) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nlines * N) return;
  const uint64_t line = i / N, p = i % N;
  fb_fill_windows<FB_BITS, FB_WINDOWS>(tab + line * FB_WINDOWS * N + p, N);
}

// Wide-window tables of a class of nl lines of unit 2^ULOG:
// wtab[((cs * nl + wl) * W + w) * N + p] = 2^(c w) P, P = point p of AMT line
// (hi_last && wl == nl - 1 ? L - 1 : l0 + wl) of coset cs, read from window 0
// of the 11-bit table tab[cs][line][FB_WINDOWS][N].
template <int ULOG>
__global__ void __launch_bounds__(128) k_wd_tables(G1Aff* wtab, const G1Aff* __restrict__ tab, uint64_t N, int L,
                                                   int l0, int nl, int hi_last) {
  constexpr int W = wd_windows(ULOG);
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3ull * nl * N) return;
  const uint64_t p = i % N, cl = i / N;  // cl = cs * nl + wl
  const int wl = (int)(cl % nl), cs = (int)(cl / nl);
  const int line = (hi_last && wl == nl - 1) ? L - 1 : l0 + wl;
  G1Aff* col = wtab + cl * W * N + p;
  col[0] = tab[((uint64_t)cs * L + line) * FB_WINDOWS * N + p];
  fb_fill_windows<ULOG + 1, W>(col, N);
}

// signed 11-bit digit w of a scalar given as 8 little-endian u32 limbs
__device__ __forceinline__ uint32_t fb_window_bits(const uint32_t* s, int w) {
  const int o = FB_BITS * w;
  const int li = o >> 5, sh = o & 31;
  uint32_t v = s[li] >> sh;
  if (sh > 32 - FB_BITS && li + 1 < 8) v |= s[li + 1] << (32 - sh);
  return v & ((1u << FB_BITS) - 1);
}

// Per chunk: counting sort of the (point, window) pairs by |digit|.
//   offs[g][k-1] .. offs[g][k]  = entries of bucket k (k = 1..1024)
//   ents[g][e] = t | w << 10 | sign << 15
// g = coset * nchunks + chunk. Chunk b reads encoded row bitrev(b), element t
// = column bitrev(t) when bitrev_rows is set (HalfBlob::generate's index_reverse).
__global__ void __launch_bounds__(256) k_fb_sort(const uint8_t* __restrict__ scalars, uint32_t* __restrict__ offs,
                                                 uint16_t* __restrict__ ents, int lr, int lc, int bitrev_rows,
                                                 uint64_t scalar_coset_stride) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int C = 1 << lc;
  const uint32_t b = blockIdx.x, coset = blockIdx.y;
  const uint32_t g = coset * (1u << lr) + b;
  uint32_t* scal = reinterpret_cast<uint32_t*>(smem);            // [C][8]
  uint32_t* cnt = scal + (size_t)C * 8;                           // [FB_BUCKETS + 1]
  uint32_t* part = cnt + FB_BUCKETS + 1;                          // [256]
  uint16_t* lst = reinterpret_cast<uint16_t*>(part + 256);        // [W * C]
  const uint32_t row = bitrev_rows ? brev_bits(b, lr) : b;
  const uint8_t* src = scalars + (scalar_coset_stride * coset + (uint64_t)row * C) * 32;
  for (int t = threadIdx.x; t < C; t += blockDim.x) {
    uint32_t col = bitrev_rows ? brev_bits(t, lc) : t;
    const uint4* q = reinterpret_cast<const uint4*>(src + (size_t)col * 32);
    uint4 x = q[0], y = q[1];
    uint32_t* d = scal + (size_t)t * 8;
    d[0] = x.x; d[1] = x.y; d[2] = x.z; d[3] = x.w; d[4] = y.x; d[5] = y.y; d[6] = y.z; d[7] = y.w;
  }
  for (int k = threadIdx.x; k <= FB_BUCKETS; k += blockDim.x) cnt[k] = 0;
  __syncthreads();
  // pass 1: counts
  for (int t = threadIdx.x; t < C; t += blockDim.x) {
    const uint32_t* s = scal + (size_t)t * 8;
    uint32_t carry = 0;
    for (int w = 0; w < FB_WINDOWS; ++w) {
      uint32_t v = fb_window_bits(s, w) + carry;
      int d;
      if (v >= (uint32_t)FB_BUCKETS) { d = (int)v - (1 << FB_BITS); carry = 1; }
      else { d = (int)v; carry = 0; }
      if (d) atomicAdd(&cnt[d < 0 ? -d : d], 1u);
    }
  }
  __syncthreads();
  // exclusive scan of cnt[1..1024] in 256 blocks of 4
  {
    const int k0 = 1 + 4 * threadIdx.x;
    uint32_t s4 = 0;
    for (int k = k0; k < k0 + 4; ++k) s4 += cnt[k];
    part[threadIdx.x] = s4;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t acc = 0;
      for (int i = 0; i < 256; ++i) { uint32_t v = part[i]; part[i] = acc; acc += v; }
    }
    __syncthreads();
    uint32_t acc = part[threadIdx.x];
    for (int k = k0; k < k0 + 4; ++k) {
      uint32_t v = cnt[k];
      cnt[k] = acc;            // becomes the fill pointer of bucket k
      offs[(size_t)g * (FB_BUCKETS + 1) + k - 1] = acc;
      acc += v;
    }
    if (threadIdx.x == blockDim.x - 1) offs[(size_t)g * (FB_BUCKETS + 1) + FB_BUCKETS] = acc;
  }
  __syncthreads();
  // pass 2: scatter
  for (int t = threadIdx.x; t < C; t += blockDim.x) {
    const uint32_t* s = scal + (size_t)t * 8;
    uint32_t carry = 0;
    for (int w = 0; w < FB_WINDOWS; ++w) {
      uint32_t v = fb_window_bits(s, w) + carry;
      int d;
      if (v >= (uint32_t)FB_BUCKETS) { d = (int)v - (1 << FB_BITS); carry = 1; }
      else { d = (int)v; carry = 0; }
      if (d) {
        uint32_t pos = atomicAdd(&cnt[d < 0 ? -d : d], 1u);
        lst[pos] = (uint16_t)(t | (w << 10) | (d < 0 ? 0x8000 : 0));
      }
    }
  }
  __syncthreads();
  const uint32_t total = offs[(size_t)g * (FB_BUCKETS + 1) + FB_BUCKETS];
  uint16_t* dst = ents + (size_t)g * FB_WINDOWS * C;
  for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) dst[e] = lst[e];
}

constexpr int WD_SORT_THREADS = 1024;
inline size_t wd_sort_smem_bytes(int ulog) { return (size_t)((1u << ulog) + 1 + 32) * sizeof(uint32_t); }

// Per sort unit of U = 2^ULOG consecutive points of a coset (chunks
// u U / 1024 .. (u + 1) U / 1024 - 1 of 1024 columns): counting sort of the
// (point, window) pairs by |digit| of the signed c = ULOG + 1 bit digits.
//   offs[cs][u][k] .. offs[cs][u][k + 1] = entries of bucket k (|digit| = k + 1)
//   ents[cs][u][e] = p | w << ULOG | sign << 31, p the point within the unit
// Point p of unit u is chunk b = (u U + p) >> lc, element t = (u U + p) &
// (2^lc - 1), read like k_fb_sort reads it. Pass 1 counts, a block scan turns
// the counts into fill pointers, pass 2 scatters (the scalars are read twice).
template <int C>
__device__ __forceinline__ uint32_t wd_window_bits(const uint32_t* s, int w) {
  const int o = C * w;
  const int li = o >> 5, sh = o & 31;
  uint32_t v = s[li] >> sh;
  if (sh > 32 - C && li + 1 < 8) v |= s[li + 1] << (32 - sh);
  return v & ((1u << C) - 1);
}

template <int ULOG>
__global__ void __launch_bounds__(WD_SORT_THREADS) k_wd_sort(const uint8_t* __restrict__ scalars,
                                                             uint32_t* __restrict__ offs, uint32_t* __restrict__ ents,
                                                             int lr, int lc, int bitrev_rows,
                                                             uint64_t scalar_coset_stride) {
  constexpr int C = ULOG + 1, W = wd_windows(ULOG);
  constexpr uint32_t U = 1u << ULOG, NB = U;           // buckets = 2^(c - 1) = U
  constexpr int PER = (int)NB / WD_SORT_THREADS;       // counters per thread in the scan
  static_assert(PER >= 1, "at least 1024 buckets");
  extern __shared__ __align__(16) uint32_t wcnt[];     // [NB + 1], then [32] warp sums
  uint32_t* wsum = wcnt + NB + 1;
  const uint32_t unit = blockIdx.x, coset = blockIdx.y, nunits = gridDim.x;
  const uint32_t Cn = 1u << lc;
  const uint8_t* src = scalars + scalar_coset_stride * coset * 32;
  uint32_t* o = offs + ((size_t)coset * nunits + unit) * (NB + 1);
  uint32_t* e = ents + ((size_t)coset * nunits + unit) * wd_unit_ents(ULOG);
  for (uint32_t k = threadIdx.x; k <= NB; k += blockDim.x) wcnt[k] = 0;
  __syncthreads();
  for (int pass = 0; pass < 2; ++pass) {
    for (uint32_t p = threadIdx.x; p < U; p += blockDim.x) {
      const uint32_t gp = (unit << ULOG) + p;
      const uint32_t b = gp >> lc, t = gp & (Cn - 1);
      const uint32_t row = bitrev_rows ? brev_bits(b, lr) : b;
      const uint32_t col = bitrev_rows ? brev_bits(t, lc) : t;
      const uint4* q = reinterpret_cast<const uint4*>(src + ((uint64_t)row * Cn + col) * 32);
      const uint4 x = q[0], y = q[1];
      const uint32_t s[8] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
      uint32_t carry = 0;
#pragma unroll
      for (int w = 0; w < W; ++w) {
        const uint32_t v = wd_window_bits<C>(s, w) + carry;
        uint32_t mag, neg;
        if (v >= NB) { mag = (1u << C) - v; neg = 1; carry = 1; }
        else { mag = v; neg = 0; carry = 0; }
        if (mag) {
          const uint32_t pos = atomicAdd(&wcnt[mag - 1], 1u);
          if (pass) e[pos] = p | (uint32_t)w << ULOG | neg << 31;
        }
      }
    }
    __syncthreads();
    if (pass == 0) {
      // exclusive scan of the NB counts: PER per thread, warp scans, warp sums
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      const int k0 = threadIdx.x * PER;
      uint32_t sum = 0;
      for (int i = 0; i < PER; ++i) sum += wcnt[k0 + i];
      uint32_t incl = sum;
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
      }
      if (lane == 31) wsum[warp] = incl;
      __syncthreads();
      if (warp == 0) {
        const uint32_t ws = wsum[lane];
        uint32_t wi = ws;
        for (int d = 1; d < 32; d <<= 1) {
          const uint32_t v = __shfl_up_sync(0xffffffffu, wi, d);
          if (lane >= d) wi += v;
        }
        wsum[lane] = wi - ws;
      }
      __syncthreads();
      uint32_t acc = wsum[warp] + incl - sum;
      for (int i = 0; i < PER; ++i) {
        const uint32_t v = wcnt[k0 + i];
        wcnt[k0 + i] = acc;
        o[k0 + i] = acc;
        acc += v;
      }
      if (threadIdx.x == blockDim.x - 1) o[NB] = acc;
      __syncthreads();
    }
  }
}

struct FbAccArgs {
  const G1Aff* tab = nullptr;      // [cosets][Ltot][W][tabN]
  const uint32_t* offs = nullptr;
  const uint16_t* ents = nullptr;    // chunk items
  const uint32_t* ents32 = nullptr;  // wide items (k_wd_sort's lists)
  XYZZ* outT = nullptr;            // [cosets * nchunks * lines][FB_ACC_THREADS]
  XYZZ* outS = nullptr;
  int lr = 0, lc = 0, lines = 1;   // 2^lr items of each of `lines` lines per coset
  int l0 = 0, Ltot = 1;            // item line l reads table line l0 + l of Ltot per coset
  int ulog = 10;                   // wide items: sort units of 2^ulog points
  int mlog = 0;                    // wide items: 2^mlog consecutive sort units share buckets
  int W = FB_WINDOWS;              // windows per table line (wd_windows(ulog) for wide items)
  uint64_t tabN = 0;               // points per window table (the param line length)
};

// Persistent CTAs over the (chunk, line) work items. Per item:
//  1. every bucket is cut into tasks of at most tsz entries (the top
//     window's digits are tiny, so buckets 1 and 2 hold ~10x the average);
//     tsz = task unless the item holds more than (FB_MAX_TASKS -
//     FB_BUCKETS) * task entries (wide items of skewed scalars), so an
//     item never has more than FB_MAX_TASKS tasks;
//  2. tasks are counting-sorted by size and round r gives thread i the task at
//     sorted position 128 r + i: the 32 lanes of a warp run tasks of nearly
//     equal length;
//  3. task partial sums go to this CTA's scratch (gpart, L2-resident);
//  4. thread i merges the partials of buckets 8i+1 .. 8i+8 and folds them
//     into running sums S_i = sum B_k, T_i = sum (k - 8i) B_k.
// Wide items (ents32 set) are 1024-bucket blocks of a wide unit of 2^(ulog +
// mlog) points whose buckets are those of its 2^mlog sort units of 2^ulog
// points (k_wd_sort; mlog <= 1): item g of a coset is block g & (2^(ulog -
// 10) - 1) of unit g >> (ulog - 10); bucket k's entries are those of sort
// unit 0 followed by those of sort unit 1, indexing the points of the
// merged unit and the W windows of the wide table. A merged unit pays one
// bucket reduction for twice the points.
// One launch covers up to FB_MAX_SETS item sets (a blob's chunk items and its
// wide classes, for up to FB_MAX_BLOBS blobs whose MSMs share the launch):
// set k holds items start[k] .. start[k + 1] - 1, described by a[k] with
// local item index u - start[k]. One launch keeps the persistent CTAs busy to
// the end of the whole MSM instead of leaving a partial last round per set. A CTA takes its next item from the counter *next (zero at
// launch): items differ in size (a wide unit's block 0 holds the top
// window's digits), and a fixed item-to-CTA map would give some CTAs every
// heavy item.
constexpr int FB_MAX_BLOBS = 2;  // blobs per fused MSM launch
constexpr int FB_MAX_SETS = 8 * FB_MAX_BLOBS;
struct FbAccPlan {
  int n = 0;
  uint32_t start[FB_MAX_SETS + 1] = {};
  FbAccArgs a[FB_MAX_SETS];
};
// Bucket task size (entries per task, a tuning choice within [FB_TASK_MIN,
// FB_TASK_MAX]); the task arrays are sized for the smallest.
constexpr int FB_TASK_MIN = 32;
constexpr int FB_TASK_MAX = 96;
constexpr int FB_TASK_DEFAULT = 64;
constexpr int FB_MAX_TASKS = FB_BUCKETS + FB_WINDOWS * 1024 / FB_TASK_MIN;  // chunk <= 1024 points
// M is the product kind of the point additions (MulImad / MulHybrid / MulF64,
// chosen by the context's tuning; identical results).
template <class M>
__global__ void __launch_bounds__(FB_ACC_THREADS, FB_ACC_MIN_CTAS) k_fb_accum(const FbAccPlan plan, XYZZ* __restrict__ gpart_all,
                                                                uint32_t* __restrict__ next, uint32_t task) {
  __shared__ uint32_t soffs[FB_BUCKETS + 1];
  __shared__ uint32_t soffs2[FB_BUCKETS + 1];  // the second sort unit of a merged wide item
  __shared__ uint16_t tstart[FB_BUCKETS + 1];
  __shared__ uint16_t order[FB_MAX_TASKS];
  __shared__ uint16_t tbucket[FB_MAX_TASKS];
  __shared__ uint32_t bins[FB_TASK_MAX + 1];
  task = min(max(task, (uint32_t)FB_TASK_MIN), (uint32_t)FB_TASK_MAX);
  __shared__ uint32_t item;
  XYZZ* gpart = gpart_all + (size_t)blockIdx.x * FB_MAX_TASKS;
  const uint32_t units = plan.start[plan.n];
  for (;;) {
    __syncthreads();  // every thread has read the previous item number
    if (threadIdx.x == 0) item = atomicAdd(next, 1u);
    __syncthreads();
    const uint32_t gu = item;
    if (gu >= units) break;
    int set = 0;
    while (set + 1 < plan.n && gu >= plan.start[set + 1]) ++set;
    const FbAccArgs& a = plan.a[set];
    const uint32_t u = gu - plan.start[set];
    const uint32_t nch = 1u << a.lr;
    const uint64_t N = a.tabN;
    const uint32_t l = u % a.lines, g = u / a.lines;
    const uint32_t coset = g / nch, b = g % nch;
    const uint32_t* offs;
    const uint32_t* offs2 = nullptr;
    const uint16_t* ents = nullptr;
    const uint32_t* ents32 = a.ents32;
    const uint32_t* ents32b = nullptr;
    const bool wide = ents32 != nullptr;
    const uint32_t ulog = (uint32_t)a.ulog;
    const G1Aff* tabl;
    if (wide) {
      const int bl = a.ulog - 10, ml = a.mlog;
      const uint32_t unit = b >> bl, blk = b & ((1u << bl) - 1);
      const size_t cu = (size_t)coset * ((size_t)(nch >> bl) << ml) + ((size_t)unit << ml);  // first sort unit
      offs = a.offs + cu * ((1u << a.ulog) + 1) + (size_t)blk * FB_BUCKETS;
      ents32 += cu * wd_unit_ents(a.ulog);
      if (ml) {
        offs2 = offs + ((1u << a.ulog) + 1);
        ents32b = ents32 + wd_unit_ents(a.ulog);
      }
      tabl = a.tab + ((uint64_t)coset * a.Ltot + a.l0 + l) * a.W * N + ((uint64_t)unit << (a.ulog + ml));
    } else {
      offs = a.offs + (size_t)g * (FB_BUCKETS + 1);
      ents = a.ents + (size_t)g * FB_WINDOWS * (1u << a.lc);
      tabl = a.tab + ((uint64_t)coset * a.Ltot + a.l0 + l) * FB_WINDOWS * N + ((uint64_t)b << a.lc);
    }
    __syncthreads();  // the previous item is finished with the shared arrays and gpart
    for (int k = threadIdx.x; k <= FB_BUCKETS; k += blockDim.x) {
      soffs[k] = offs[k];
      soffs2[k] = offs2 ? offs2[k] : 0u;
    }
    for (int k = threadIdx.x; k <= FB_TASK_MAX; k += blockDim.x) bins[k] = 0;
    __syncthreads();
    // entries of bucket k (0-based): its range in the first sort unit's list,
    // then (merged items) its range in the second's
    auto bcount = [&](int k) { return (soffs[k + 1] - soffs[k]) + (soffs2[k + 1] - soffs2[k]); };
    const uint32_t nent = (soffs[FB_BUCKETS] - soffs[0]) + (soffs2[FB_BUCKETS] - soffs2[0]);
    const uint32_t cap = (uint32_t)(FB_MAX_TASKS - FB_BUCKETS);
    const uint32_t tsz = max(task, (nent + cap - 1) / cap);
    // tasks per bucket, exclusive scan -> tstart (bucket k = 0-based index)
    if (threadIdx.x < 32) {
      // warp-level scan over 1024 buckets, 32 per lane
      const int lane = threadIdx.x;
      uint32_t loc[32];
      uint32_t sum = 0;
      for (int i = 0; i < 32; ++i) {
        const int k = lane * 32 + i;
        const uint32_t c = bcount(k);
        loc[i] = (c + tsz - 1) / tsz;
        sum += loc[i];
      }
      uint32_t incl = sum;
      for (int d = 1; d < 32; d <<= 1) {
        uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
      }
      uint32_t acc = incl - sum;
      for (int i = 0; i < 32; ++i) {
        tstart[lane * 32 + i] = (uint16_t)acc;
        acc += loc[i];
      }
      if (lane == 31) tstart[FB_BUCKETS] = (uint16_t)acc;
    }
    __syncthreads();
    const uint32_t ntasks = tstart[FB_BUCKETS];
    // size of task j of bucket k: tsz except the bucket's last task; bin
    // task - size * task / tsz (task - size when tsz = task): larger tasks
    // first
    for (int k = threadIdx.x; k < FB_BUCKETS; k += blockDim.x) {
      const uint32_t c = bcount(k);
      for (uint32_t t = tstart[k]; t < tstart[k + 1]; ++t) {
        tbucket[t] = (uint16_t)k;
        const uint32_t j = t - tstart[k];
        const uint32_t sz = min(tsz, c - j * tsz);
        atomicAdd(&bins[task - sz * task / tsz], 1u);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t acc = 0;
      for (uint32_t i = 0; i <= task; ++i) { uint32_t v = bins[i]; bins[i] = acc; acc += v; }
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < ntasks; t += blockDim.x) {
      const uint32_t k = tbucket[t];
      const uint32_t c = bcount(k);
      const uint32_t j = t - tstart[k];
      const uint32_t sz = min(tsz, c - j * tsz);
      order[atomicAdd(&bins[task - sz * task / tsz], 1u)] = (uint16_t)t;
    }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < ntasks; r += blockDim.x) {
      const uint32_t t = order[r];
      const uint32_t k = tbucket[t];
      // positions q0 .. q1 - 1 of the bucket's entries (first sort unit's
      // c0, then the second's)
      const uint32_t c0 = soffs[k + 1] - soffs[k];
      const uint32_t q0 = (t - tstart[k]) * tsz;
      const uint32_t q1 = min(q0 + tsz, bcount(k));
      XYZZ B = XYZZ::inf();
      for (uint32_t q = q0; q < q1; ++q) {
        uint32_t idx, w, neg;
        if (wide) {
          const bool second = q >= c0;
          const uint32_t v = second ? ents32b[soffs2[k] + (q - c0)] : ents32[soffs[k] + q];
          idx = (v & ((1u << ulog) - 1)) + (second ? (1u << ulog) : 0u);
          w = (v >> ulog) & 31;
          neg = v >> 31;
        } else {
          const uint32_t v = ents[soffs[k] + q];
          idx = v & 0x3ff;
          w = (v >> 10) & 31;
          neg = v >> 15;
        }
        G1Aff p = load_aff(tabl + (uint64_t)w * N + idx);
        if (neg) p.y = -p.y;
        B.template add_affine<M>(p.x, p.y);
      }
      store_xyzz(gpart + t, B);
    }
    __syncthreads();
    const int k0 = threadIdx.x * FB_PER_THREAD;  // 0-based buckets k0 .. k0+7
    XYZZ S = XYZZ::inf(), T = XYZZ::inf();
    for (int k = k0 + FB_PER_THREAD - 1; k >= k0; --k) {
      for (uint32_t t = tstart[k]; t < tstart[k + 1]; ++t) S.template add<M>(load_xyzz(gpart + t));
      T.template add<M>(S);
    }
    store_xyzz(a.outT + (size_t)u * FB_ACC_THREADS + threadIdx.x, T);
    store_xyzz(a.outS + (size_t)u * FB_ACC_THREADS + threadIdx.x, S);
  }
}

// Where a combine launch's items go. The launch covers up to FB_MAX_SETS item
// sets (the chunk items, then one set per wide unit size); set k holds items
// start[k] .. start[k + 1] - 1, whose (T, S) partials sit at the same
// positions. Local item v = u - start[k] of line l = v % lines (g = v / lines,
// coset g >> lr, b = g & (2^lr - 1)) is written to part[(coset * L + line) *
// 2^lr + b], line = L - 1 for the set's last line when hi_last, else l0 + l.
// Wide items (block blk = b & (2^bpu_log - 1) of a unit) add 1024 blk *
// sum_k B_k: their buckets hold digits 1024 blk + k + 1 (bpu_log = 0 for
// chunk items). part_off places a fused launch's blob in its own part block.
// lr: log2 of the set's items per (coset, line); a wide set's items are
// blocks of 2^bpu_log per unit, and a merged unit (mlog = 1) spans 2^(bpu_log
// + mlog) part slots (one per 1024 points): its items fill the first 2^bpu_log
// and the identity the rest, so the AMT trees sum every line's R slots alike.
struct FbCombineMap {
  int lr, lines, l0, L, hi_last, bpu_log, mlog;
  uint64_t part_off;
};
struct FbCombinePlan {
  int n = 0;
  uint32_t start[FB_MAX_SETS + 1] = {};
  FbCombineMap m[FB_MAX_SETS] = {};
};

// the set of item u, its map and its local index
__device__ __forceinline__ const FbCombineMap& fb_plan_item(const FbCombinePlan& p, uint32_t u, uint32_t* v) {
  int k = 0;
  while (k + 1 < p.n && u >= p.start[k + 1]) ++k;
  *v = u - p.start[k];
  return p.m[k];
}

__device__ __forceinline__ size_t fb_part_index(const FbCombineMap& m, uint32_t v) {
  const uint32_t l = v % m.lines, g = v / m.lines;
  const uint32_t nch = 1u << m.lr;
  const uint32_t line = (m.hi_last && l == (uint32_t)m.lines - 1) ? (uint32_t)m.L - 1 : (uint32_t)m.l0 + l;
  const uint32_t b = g % nch, bmask = (1u << m.bpu_log) - 1;
  const uint32_t slot = ((b >> m.bpu_log) << (m.bpu_log + m.mlog)) | (b & bmask);
  return ((size_t)(g / nch) * m.L + line) * ((size_t)nch << m.mlog) + slot;
}

// the identity in the part slots of a merged unit that no item fills
__device__ __forceinline__ void fb_fill_unused_slots(const FbCombineMap& m, XYZZ* slot0) {
  for (uint32_t t = 1; t < (1u << m.mlog); ++t) store_xyzz(slot0 + ((size_t)t << m.bpu_log), XYZZ::inf());
}

__device__ __forceinline__ uint32_t fb_item_block(const FbCombineMap& m, uint32_t v) {
  return (v / m.lines) & ((1u << m.bpu_log) - 1);
}

// (1024 blk) * P for blk < 32
__device__ XYZZ fb_block_term(const XYZZ& P, uint32_t blk) {
  XYZZ r = XYZZ::inf();
#pragma unroll 1
  for (int bit = 4; bit >= 0; --bit) {
    r = r.dbl();
    if ((blk >> bit) & 1) r.add(P);
  }
#pragma unroll 1
  for (int k = 0; k < 10; ++k) r = r.dbl();
  return r;
}

// Per item: P = sum_i T_i + 8 * sum_i i S_i (+ the wide block term); written
// to part for the AMT trees.
__global__ void __launch_bounds__(64) k_fb_combine(const XYZZ* __restrict__ T, const XYZZ* __restrict__ S,
                                                   XYZZ* __restrict__ part, FbCombinePlan plan) {
  const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= plan.start[plan.n]) return;
  uint32_t v;
  const FbCombineMap& m = fb_plan_item(plan, u, &v);
  const XYZZ* t = T + (size_t)u * FB_ACC_THREADS;
  const XYZZ* s = S + (size_t)u * FB_ACC_THREADS;
  XYZZ tot = XYZZ::inf(), run = XYZZ::inf(), wsum = XYZZ::inf();
  for (int i = FB_ACC_THREADS - 1; i >= 1; --i) {
    run.add(load_xyzz(s + i));
    wsum.add(run);
  }
  for (int i = 0; i < FB_ACC_THREADS; ++i) tot.add(load_xyzz(t + i));
#pragma unroll 1
  for (int k = 0; k < FB_PER_THREAD_LOG; ++k) wsum = wsum.dbl();  // x FB_PER_THREAD
  tot.add(wsum);
  const uint32_t blk = fb_item_block(m, v);
  if (blk) {
    run.add(load_xyzz(s));  // sum of all the item's buckets
    tot.add(fb_block_term(run, blk));
  }
  XYZZ* dst = part + m.part_off + fb_part_index(m, v);
  store_xyzz(dst, tot);
  fb_fill_unused_slots(m, dst);
}

__device__ __forceinline__ XYZZ shfl_xor_xyzz(const XYZZ& p, int m) {
  XYZZ r;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    r.X.v[i] = __shfl_xor_sync(0xffffffffu, p.X.v[i], m);
    r.Y.v[i] = __shfl_xor_sync(0xffffffffu, p.Y.v[i], m);
    r.ZZ.v[i] = __shfl_xor_sync(0xffffffffu, p.ZZ.v[i], m);
    r.ZZZ.v[i] = __shfl_xor_sync(0xffffffffu, p.ZZZ.v[i], m);
  }
  return r;
}

// k_fb_combine with one warp per item, for launches with few items (the
// single MSMs of zg_ctx_msm and of slice verification: 1024 items leave
// k_fb_combine's one thread per item on a handful of SMs). With P =
// FB_ACC_THREADS / 32 partials per lane, lane l folds partials P l .. P l +
// P - 1 into t_l, s_l and w_l = sum_k k S_{Pl+k}; then
// sum_i i S_i = P sum_l l s_l + sum_l w_l, sum_l l s_l being the sum over
// lanes l >= 1 of the suffix sums U_l = sum_{m >= l} s_m (a warp scan). About
// three times the additions of k_fb_combine, so blob encodes keep that one.
__global__ void __launch_bounds__(128) k_fb_combine_warp(const XYZZ* __restrict__ T, const XYZZ* __restrict__ S,
                                                         XYZZ* __restrict__ part, FbCombinePlan plan) {
  constexpr int P = FB_ACC_THREADS / 32;  // partials per lane
  static_assert(P >= 1 && (P & (P - 1)) == 0, "a power of two of partials per lane");
  const uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (u >= plan.start[plan.n]) return;  // uniform per warp
  uint32_t v;
  const FbCombineMap& m = fb_plan_item(plan, u, &v);
  const XYZZ* t = T + (size_t)u * FB_ACC_THREADS + P * lane;
  const XYZZ* s = S + (size_t)u * FB_ACC_THREADS + P * lane;
  XYZZ tl = load_xyzz(t);
  for (int k = 1; k < P; ++k) tl.add(load_xyzz(t + k));
  XYZZ run = XYZZ::inf(), w = XYZZ::inf();
  for (int k = P - 1; k >= 1; --k) {
    run.add(load_xyzz(s + k));
    w.add(run);
  }
  run.add(load_xyzz(s));
  XYZZ U = run;
  for (int d = 1; d < 32; d <<= 1) {
    const XYZZ v = shfl_down_xyzz(U, d);
    if (lane + d < 32) U.add(v);
  }
  XYZZ a = lane >= 1 ? U : XYZZ::inf();
  for (int mk = 16; mk >= 1; mk >>= 1) {
    tl.add(shfl_xor_xyzz(tl, mk));
    w.add(shfl_xor_xyzz(w, mk));
    a.add(shfl_xor_xyzz(a, mk));
  }
  if (lane == 0) {
#pragma unroll 1
    for (int k = 0; k < fb_log2(P); ++k) a = a.dbl();  // P sum_l l s_l
    a.add(w);                                           // sum_i i S_i
#pragma unroll 1
    for (int k = 0; k < FB_PER_THREAD_LOG; ++k) a = a.dbl();  // x FB_PER_THREAD
    tl.add(a);
    const uint32_t blk = fb_item_block(m, v);
    if (blk) tl.add(fb_block_term(U, blk));  // U at lane 0 = sum of all the item's buckets
    XYZZ* dst = part + m.part_off + fb_part_index(m, v);
    store_xyzz(dst, tl);
    fb_fill_unused_slots(m, dst);
  }
}

// out = sum of the n points of `in` (one CTA of 256 threads)
__global__ void __launch_bounds__(256) k_sum_points(const XYZZ* __restrict__ in, uint32_t n, XYZZ* __restrict__ out) {
  __shared__ XYZZ sh[256];
  XYZZ acc = XYZZ::inf();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) acc.add(load_xyzz(in + i));
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      XYZZ t = sh[threadIdx.x];
      t.add(sh[threadIdx.x + w]);
      sh[threadIdx.x] = t;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) store_xyzz(out, sh[0]);
}

// sum_w 2^{8w} win[w] for each (coset, line, chunk)
__global__ void __launch_bounds__(64) k_msm_combine(const XYZZ* __restrict__ win, XYZZ* __restrict__ out, uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const XYZZ* w = win + (size_t)i * MSM_WINDOWS;
  XYZZ acc = load_xyzz(w + MSM_WINDOWS - 1);
  for (int k = MSM_WINDOWS - 2; k >= 0; --k) {
#pragma unroll 1
    for (int d = 0; d < 8; ++d) acc = acc.dbl();
    acc.add(load_xyzz(w + k));
  }
  store_xyzz(out + i, acc);
}

// ---------------------------------------------------------------------------
// AMT aggregation (prove.rs:20-52 build_commitment_tree, prove_gpu.rs:89-123
// aggregate_line / high commitment). part[c][l][b] are the per-chunk MSMs.
// One CTA per (line, coset). Output nodes per coset, XYZZ, in the order
//   [root][commitments[0] (2) .. commitments[LR-1] (R)][proofs[0] .. proofs[LR-1]][high]
__device__ __forceinline__ uint32_t amt_commit_off(int d) { return 1 + ((2u << d) - 2); }
__device__ __forceinline__ uint32_t amt_proof_off(int d, int lr) { return (2u << lr) - 1 + ((2u << d) - 2); }

__global__ void __launch_bounds__(256) k_amt_tree(XYZZ* __restrict__ part, XYZZ* __restrict__ nodes, int lr, int lines) {
  const int l = blockIdx.x, c = blockIdx.y;
  const int R = 1 << lr;
  const uint32_t per_coset = 4u * R - 2;
  XYZZ* p = part + ((size_t)c * lines + l) * R;
  XYZZ* o = nodes + (size_t)c * per_coset;
  // levels to reduce: quotient layer d = l + 1 keeps 2^d nodes; basis keeps all
  // levels; high keeps 1
  int keep_log = (l < lr) ? (l + 1) : 0;
  const bool is_basis = (l == lr);
  if (is_basis) {
    for (int i = threadIdx.x; i < R; i += blockDim.x) o[amt_commit_off(lr - 1) + i] = p[i];
  }
  int cur = R;
  int lvl = lr;  // current array holds 2^lvl nodes
  while (lvl > keep_log) {
    int half = cur >> 1;
    __syncthreads();
    // read pairs then write, two phases to allow in-place reduction
    for (int base = 0; base < half; base += blockDim.x) {
      int i = base + threadIdx.x;
      XYZZ s;
      if (i < half) {
        s = p[2 * i];
        s.add(p[2 * i + 1]);
      }
      __syncthreads();
      if (i < half) p[i] = s;
      __syncthreads();
    }
    cur = half;
    --lvl;
    if (is_basis) {
      if (lvl >= 1) {
        for (int i = threadIdx.x; i < cur; i += blockDim.x) o[amt_commit_off(lvl - 1) + i] = p[i];
      } else if (threadIdx.x == 0) {
        o[0] = p[0];
      }
    }
  }
  __syncthreads();
  if (l < lr) {
    for (int i = threadIdx.x; i < cur; i += blockDim.x) o[amt_proof_off(l, lr) + i] = p[i];
  } else if (l == lr + 1) {
    if (threadIdx.x == 0) o[per_coset - 1] = p[0];
  }
}

// XYZZ node -> 64-byte ark G1
__global__ void __launch_bounds__(128) k_serialize_nodes(const XYZZ* __restrict__ nodes, uint8_t* __restrict__ out, uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint8_t buf[64];
  g1_serialize(nodes[i], buf);
  uint4* d = reinterpret_cast<uint4*>(out + (size_t)i * 64);
  const uint32_t* w = reinterpret_cast<const uint32_t*>(buf);
  d[0] = make_uint4(w[0], w[1], w[2], w[3]);
  d[1] = make_uint4(w[4], w[5], w[6], w[7]);
  d[2] = make_uint4(w[8], w[9], w[10], w[11]);
  d[3] = make_uint4(w[12], w[13], w[14], w[15]);
}

// ---------------------------------------------------------------------------
// Merkle tree (merkle/blob.rs:15-34): leaves = keccak(8 x 32 B), parents =
// keccak(left || right) until 3 coset roots remain.
__global__ void __launch_bounds__(128) k_merkle_leaves(const uint8_t* __restrict__ data, uint8_t* __restrict__ leaves, uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint64_t* src = reinterpret_cast<const uint64_t*>(data + (size_t)i * 256);
  uint64_t in[32];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    ulonglong2 v = reinterpret_cast<const ulonglong2*>(src)[k];
    in[2 * k] = v.x;
    in[2 * k + 1] = v.y;
  }
  uint64_t out[4];
  keccak256_256(in, out);
  ulonglong2* d = reinterpret_cast<ulonglong2*>(leaves + (size_t)i * 32);
  d[0] = make_ulonglong2(out[0], out[1]);
  d[1] = make_ulonglong2(out[2], out[3]);
}
__global__ void __launch_bounds__(128) k_merkle_parents(const uint8_t* __restrict__ child, uint8_t* __restrict__ parent, uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const ulonglong2* src = reinterpret_cast<const ulonglong2*>(child + (size_t)i * 64);
  uint64_t in[8];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    ulonglong2 v = src[k];
    in[2 * k] = v.x;
    in[2 * k + 1] = v.y;
  }
  uint64_t out[4];
  keccak256_64(in, out);
  ulonglong2* d = reinterpret_cast<ulonglong2*>(parent + (size_t)i * 32);
  d[0] = make_ulonglong2(out[0], out[1]);
  d[1] = make_ulonglong2(out[2], out[3]);
}
// The upper levels of the Merkle tree in one launch: levels top - 1 .. 0
// from level top (at most 1024 nodes per coset), one CTA per coset subtree,
// each level hashed from the previous one in shared memory and written out.
// Level d holds 3 * 2^d nodes (coset c's at c 2^d ..), at byte offset
// 96 (2^d - 1) of the tree buffer. Block size max(1, 2^(top - 1)).
constexpr int MERKLE_TOP_MAX = 10;
__global__ void __launch_bounds__(512) k_merkle_top(uint8_t* __restrict__ tree, int top) {
  __shared__ uint64_t sn[(1 << MERKLE_TOP_MAX) * 4];
  const uint32_t c = blockIdx.x, n = 1u << top;
  const uint64_t* src = reinterpret_cast<const uint64_t*>(tree + 96 * ((1ull << top) - 1) + (size_t)c * n * 32);
  for (uint32_t i = threadIdx.x; i < 4 * n; i += blockDim.x) sn[i] = src[i];
  __syncthreads();
  for (int d = top - 1; d >= 0; --d) {
    const uint32_t cnt = 1u << d, i = threadIdx.x;
    uint64_t out[4];
    if (i < cnt) {
      uint64_t in[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) in[k] = sn[8 * i + k];
      keccak256_64(in, out);
    }
    __syncthreads();
    if (i < cnt) {
      uint64_t* dst = reinterpret_cast<uint64_t*>(tree + 96 * ((1ull << d) - 1) + ((size_t)c * cnt + i) * 32);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        sn[4 * i + k] = out[k];
        dst[k] = out[k];
      }
    }
    __syncthreads();
  }
}

// keccak(keccak(r0 || r1) || r2)  (encoder/blob.rs:64-72)
__global__ void k_file_root(const uint8_t* __restrict__ roots, uint8_t* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const uint64_t* r = reinterpret_cast<const uint64_t*>(roots);
  uint64_t in[8], t[4];
  for (int k = 0; k < 8; ++k) in[k] = r[k];
  keccak256_64(in, t);
  for (int k = 0; k < 4; ++k) { in[k] = t[k]; in[4 + k] = r[8 + k]; }
  keccak256_64(in, t);
  uint64_t* o = reinterpret_cast<uint64_t*>(out);
  for (int k = 0; k < 4; ++k) o[k] = t[k];
}

// ---------------------------------------------------------------------------
// EncodedSlice serialisation (ark-serialize 0.4 derive, uncompressed):
//   index | amt{index | commitment | row{index | len,row | len,proof | high}}
//   | merkle{roots[3] | len,proof | leaf_index | leaf}
// (encoder/slice.rs:15-20, amt/slice.rs:13-18, blob/encode.rs:202-209,
//  proofs.rs:34-35, merkle/slice.rs:12-19). One CTA per slice.
struct SliceArgs {
  const uint8_t* enc;    // [3][R][C] x 32
  const uint8_t* amt;    // [3][4R-2] x 64
  const uint8_t* tree;   // Merkle levels, level d at tree_off[d]
  const uint64_t* tree_off;
  uint8_t* out;          // [3R][slice_size]
  int lr, lc;
  uint64_t slice_size;
};
__device__ __forceinline__ void put_u64(uint8_t* p, uint64_t v) {
#pragma unroll
  for (int i = 0; i < 8; ++i) p[i] = (uint8_t)(v >> (8 * i));
}
__global__ void __launch_bounds__(256) k_slices(SliceArgs a) {
  const int R = 1 << a.lr, C = 1 << a.lc;
  const uint32_t index = blockIdx.x;
  const uint32_t coset = index / R, local = index % R;
  uint8_t* o = a.out + (uint64_t)index * a.slice_size;
  const uint8_t* amt = a.amt + (size_t)coset * (4 * R - 2) * 64;
  // row data, 16-byte vectors (offset 96 is 16-byte aligned when slice_size is)
  const uint4* row = reinterpret_cast<const uint4*>(a.enc + ((size_t)coset * R + local) * C * 32);
  uint8_t* rowdst = o + 96;
  for (int k = threadIdx.x; k < C * 2; k += blockDim.x) {
    uint4 v = row[k];
    uint8_t* d = rowdst + 16 * k;
    const uint8_t* s = reinterpret_cast<const uint8_t*>(&v);
#pragma unroll
    for (int i = 0; i < 16; ++i) d[i] = s[i];
  }
  const uint32_t rev = brev_bits(local, a.lr);
  uint8_t* after = o + 96 + (size_t)32 * C;
  // proof pairs: 8 + 128 LR bytes
  if (threadIdx.x == 0) {
    put_u64(o, index);
    put_u64(o + 8, index);
    put_u64(o + 80, local);
    put_u64(o + 88, (uint64_t)C);
    put_u64(after, (uint64_t)a.lr);
  }
  for (int k = threadIdx.x; k < 64; k += blockDim.x) o[16 + k] = amt[k];  // commitment (root)
  for (int e = threadIdx.x; e < a.lr * 128; e += blockDim.x) {
    int dd = e / 128, off = e % 128;
    uint32_t lv = rev >> (a.lr - 1 - dd);
    uint32_t node = lv ^ 1;
    const uint8_t* src = (off < 64) ? amt + (size_t)(1 + (2u << dd) - 2 + node) * 64 + off
                                    : amt + (size_t)((2u << a.lr) - 1 + (2u << dd) - 2 + node) * 64 + (off - 64);
    after[8 + e] = *src;
  }
  uint8_t* high = after + 8 + 128 * a.lr;
  for (int k = threadIdx.x; k < 64; k += blockDim.x) high[k] = amt[(size_t)(4 * R - 3) * 64 + k];
  uint8_t* mk = high + 64;
  const uint8_t* roots = a.tree + a.tree_off[0];
  for (int k = threadIdx.x; k < 96; k += blockDim.x) mk[k] = roots[k];
  if (threadIdx.x == 0) put_u64(mk + 96, (uint64_t)a.lr);
  for (int e = threadIdx.x; e < a.lr * 32; e += blockDim.x) {
    int i = e / 32, off = e % 32;
    int d = a.lr - i;  // d = LR .. 1
    uint32_t idx = index >> (a.lr - d);
    mk[104 + e] = a.tree[a.tree_off[d] + (size_t)(idx ^ 1) * 32 + off];
  }
  uint8_t* tail = mk + 104 + 32 * a.lr;
  if (threadIdx.x == 0) put_u64(tail, index);
  for (int k = threadIdx.x; k < 32; k += blockDim.x) tail[8 + k] = a.tree[a.tree_off[a.lr] + (size_t)index * 32 + k];
}

// ---------------------------------------------------------------------------
// parameter building (seeded tau; scalar domain then fixed-base multiply)

// out[i] = x^i (Montgomery) for i < n
__global__ void k_powers(Fr x, Fr* out, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = x.pow_u64(i);
}
__global__ void k_scale(Fr* v, Fr s, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = v[i] * s;
}
// quotient coefficient vector of layer d: c[i] = pw[M - i] for 1 <= i <= M, else 0
__global__ void k_quot_coeff(const Fr* pw, Fr* c, uint32_t M, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  c[i] = (i >= 1 && i <= M) ? pw[M - i] : Fr::zero();
}

// generic four-step NTT pass A: for each column s (C of them) of x viewed as
// [R][C] row-major: R-point transform over q, times w_N^{s r}; writes Y[r][s].
// blockIdx.y selects the vector of a batch (vectors of R C elements back to back).
// With cs_lo set, element i of x is first multiplied by
// cs_lo[i mod 2^cs_h] * cs_hi[i >> cs_h] (the coset shift).
__global__ void __launch_bounds__(256) k_ntt4_colpass(const Fr* __restrict__ x, Fr* __restrict__ y, int lr, int lc,
                               const Fr* __restrict__ tw_r, const Fr* __restrict__ w_lo,
                               const Fr* __restrict__ w_hi, const Fr* __restrict__ cs_lo,
                               const Fr* __restrict__ cs_hi, int cs_h) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int C = 1 << lc;
  Fr* s = reinterpret_cast<Fr*>(smem);
  const uint32_t col = blockIdx.x;
  x += (size_t)blockIdx.y << (lr + lc);
  y += (size_t)blockIdx.y << (lr + lc);
  const uint32_t nmask = (1u << (lr + lc)) - 1;
  auto get = [&](int q) {
    const uint32_t i = (uint32_t)q * C + col;
    const Fr e = load_fr(x + i);
    return cs_lo ? e * (cs_lo[i & ((1u << cs_h) - 1)] * cs_hi[i >> cs_h]) : e;
  };
  ntt_block(s, lr, tw_r, get, [&](int r, const Fr& v) { s[r] = v; });
  for (int r = threadIdx.x; r < (1 << lr); r += blockDim.x)
    store_fr(y + (size_t)r * C + col, s[r] * pow_split(w_lo, w_hi, col * (uint32_t)r, lc, nmask));
}
// pass B: for each r, C-point transform over s of Y[r][*]; out[j R + r]
// (times scale when do_scale)
__global__ void __launch_bounds__(256) k_ntt4_rowpass(const Fr* __restrict__ y, Fr* __restrict__ out, int lr, int lc,
                               const Fr* __restrict__ tw_c, int do_scale, Fr scale) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int R = 1 << lr, C = 1 << lc;
  Fr* s = reinterpret_cast<Fr*>(smem);
  const uint32_t r = blockIdx.x;
  y += (size_t)blockIdx.y << (lr + lc);
  out += (size_t)blockIdx.y << (lr + lc);
  ntt_block(s, lc, tw_c, [&](int k) { return load_fr(y + (size_t)r * C + k); },
            [&](int j, const Fr& v) { store_fr(out + (size_t)j * R + r, do_scale ? v * scale : v); });
}

// fixed-base table of G: tab[w*255 + d - 1] = d * 2^{8w} * G (XYZZ)
__global__ void __launch_bounds__(32) k_fixed_table(XYZZ* tab, G1Aff g) {
  int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= 32) return;
  XYZZ base = XYZZ::from_affine(g);
  for (int i = 0; i < 8 * w; ++i) base = base.dbl();
  XYZZ acc = base;
  for (int d = 1; d <= 255; ++d) {
    tab[w * 255 + d - 1] = acc;
    acc.add(base);
  }
}
__global__ void __launch_bounds__(256) k_xyzz_to_affine(const XYZZ* in, G1Aff* out, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  G1Aff a;
  if (!in[i].to_affine(a)) { a.x = Fq::zero(); a.y = Fq::zero(); }
  out[i] = a;
}
// out[p] = s[bitrev(p)] * G (enact: normalize + index_reverse, generate.rs:122-126)
__global__ void __launch_bounds__(256) k_fixed_mul(const G1Aff* __restrict__ tab, const Fr* __restrict__ sc, G1Aff* __restrict__ out,
                            uint32_t n, int logn) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  Fr s = sc[brev_bits(p, logn)].to_canonical();
  XYZZ acc = XYZZ::inf();
#pragma unroll 1
  for (int w = 0; w < 32; ++w) {
    uint32_t d = (s.v[w >> 2] >> (8 * (w & 3))) & 0xff;
    if (d) {
      G1Aff t = tab[w * 255 + d - 1];
      acc.add_affine(t.x, t.y);
    }
  }
  G1Aff a;
  if (!acc.to_affine(a)) { a.x = Fq::zero(); a.y = Fq::zero(); }
  out[p] = a;
}

}  // namespace zg
