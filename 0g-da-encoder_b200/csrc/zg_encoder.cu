// Host orchestration and C ABI of the B200 blob encoder (include/zg_encoder.h).
//
// One zg_ctx owns one device's params (3 cosets x (LR+2) G1 lines, resident
// in HBM for the context's lifetime, the role of AMTParams' lazily uploaded
// MsmBasisOnDevice in crates/amt/src/prove_params/prove_gpu.rs:30-53), the
// twiddle tables and the per-blob scratch. Encodes on one context are
// serialised by a mutex; use one context per stream of work for overlap.
#include <cuda_runtime.h>
#include <dirent.h>
#include <errno.h>
#include <sys/random.h>

#include <atomic>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <tuple>
#include <mutex>
#include <thread>
#include <deque>
#include <functional>
#include <random>
#include <string>
#include <vector>

#include "../../include/zg_encoder.h"
#include "zg_kernels.cuh"
#include "zg_recover.cuh"
#include "zg_verify.cuh"

using namespace zg;

namespace {

thread_local std::string g_err;
int fail(int code, const std::string& m) {
  g_err = m;
  return code;
}
#define ZG_CK(x)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (x);                                                                \
    if (e_ != cudaSuccess) return fail(ZG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

uint32_t host_brev(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; ++i) r = (r << 1) | ((x >> i) & 1);
  return r;
}

// Fr two-adic root of unity 5^((r-1)/2^28) (ark-bn254 FrConfig generator 5)
Fr fr_two_adic_root() {
  Fr c;
  const uint32_t w[8] = {0x725b19f0u, 0x9bd61b6eu, 0x41112ed4u, 0x402d111eu,
                         0x8ef62abcu, 0x00e0a7ebu, 0xa58a7e85u, 0x2a3c09f0u};
  for (int i = 0; i < 8; ++i) c.v[i] = w[i];
  return Fr::from_canonical(c);
}
Fr fr_root(int log_n) {
  Fr w = fr_two_adic_root();
  for (int i = log_n; i < 28; ++i) w = w.sqr();
  return w;
}
// AMTParams::coset_factor (crates/amt/src/prove_params/generate.rs:128-137)
Fr coset_factor(int log_len, uint32_t idx) {
  uint32_t pow = host_brev(idx, 28 - log_len);
  return fr_two_adic_root().pow_u64(pow);
}

uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
// tau = (w0 + w1 2^64 + ... + w7 2^448) mod r, w_i the SplitMix64 stream at `seed`
Fr tau_from_seed(uint64_t seed) {
  uint64_t s = seed, w[8];
  for (int i = 0; i < 8; ++i) w[i] = splitmix64(s);
  auto reduce = [](const uint64_t* x) {
    Fr a;
    for (int i = 0; i < 4; ++i) {
      a.v[2 * i] = (uint32_t)x[i];
      a.v[2 * i + 1] = (uint32_t)(x[i] >> 32);
    }
    for (;;) {
      Fr d;
      if (Fr::sub_raw(d, a, Fr::modulus())) break;
      a = d;
    }
    return Fr::from_canonical(a);
  };
  Fr lo = reduce(w), hi = reduce(w + 4);
  Fr two256 = Fr::from_canonical(Fr::one());  // 2^256 mod r as a field element
  return lo + hi * two256;
}

Fr host_fr_from_u32(uint32_t x) { return Fr::from_u32(x); }

// twiddle tables for an N = R * C transform
struct Twiddles {
  int lr = 0, lc = 0;
  Fr *twf_c = nullptr, *twi_c = nullptr, *twf_r = nullptr, *twi_r = nullptr;
  Fr *wn_lo = nullptr, *wn_hi = nullptr, *wni_lo = nullptr, *wni_hi = nullptr;
  Fr *gs_lo = nullptr, *gs_hi = nullptr;  // coset scale tables (cosets 1, 2)
};

template <class T>
int upload(T** dst, const std::vector<T>& v) {
  ZG_CK(cudaMalloc(dst, sizeof(T) * std::max<size_t>(v.size(), 1)));
  ZG_CK(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return 0;
}
std::vector<Fr> pow_table(const Fr& x, size_t n) {
  std::vector<Fr> t(n);
  Fr a = Fr::one();
  for (size_t i = 0; i < n; ++i) { t[i] = a; a = a * x; }
  return t;
}
// The transform core's twiddles of the n-point transform with root w, stage
// by stage: t[h + i] = w^(i n / (2h)) for h = 1, 2, 4, .. n/2 and i < h (the
// twiddles of the stage whose butterflies span h), t[0] = 1.
std::vector<Fr> stage_table(const Fr& w, size_t n) {
  std::vector<Fr> t(std::max<size_t>(n, 1));
  t[0] = Fr::one();
  const std::vector<Fr> p = pow_table(w, std::max<size_t>(n / 2, 1));
  for (size_t h = 1; h < n; h <<= 1)
    for (size_t i = 0; i < h; ++i) t[h + i] = p[i * (n / (2 * h))];
  return t;
}
int make_twiddles(int lr, int lc, Twiddles* tw) {
  tw->lr = lr;
  tw->lc = lc;
  const size_t R = size_t(1) << lr, C = size_t(1) << lc, N = R * C;
  Fr wc = fr_root(lc), wr = fr_root(lr), wn = fr_root(lr + lc);
  int rc = 0;
  if ((rc = upload(&tw->twf_c, stage_table(wc, C)))) return rc;
  if ((rc = upload(&tw->twi_c, stage_table(wc.inverse(), C)))) return rc;
  if ((rc = upload(&tw->twf_r, stage_table(wr, R)))) return rc;
  if ((rc = upload(&tw->twi_r, stage_table(wr.inverse(), R)))) return rc;
  if ((rc = upload(&tw->wn_lo, pow_table(wn, C)))) return rc;
  if ((rc = upload(&tw->wn_hi, pow_table(wn.pow_u64(C), R)))) return rc;
  Fr wni = wn.inverse();
  if ((rc = upload(&tw->wni_lo, pow_table(wni, C)))) return rc;
  if ((rc = upload(&tw->wni_hi, pow_table(wni.pow_u64(C), R)))) return rc;
  Fr ninv = host_fr_from_u32((uint32_t)N).inverse();
  std::vector<Fr> lo, hi;
  for (int c = 1; c <= 2; ++c) {
    Fr g = coset_factor(lr + lc, c);
    std::vector<Fr> a = pow_table(g, C);
    for (auto& x : a) x = x * ninv;
    lo.insert(lo.end(), a.begin(), a.end());
    std::vector<Fr> b = pow_table(g.pow_u64(C), R);
    hi.insert(hi.end(), b.begin(), b.end());
  }
  if ((rc = upload(&tw->gs_lo, lo))) return rc;
  if ((rc = upload(&tw->gs_hi, hi))) return rc;
  return 0;
}
void free_twiddles(Twiddles* tw) {
  Fr* ps[] = {tw->twf_c, tw->twi_c, tw->twf_r, tw->twi_r, tw->wn_lo, tw->wn_hi,
              tw->wni_lo, tw->wni_hi, tw->gs_lo, tw->gs_hi};
  for (Fr* p : ps) if (p) cudaFree(p);
  *tw = Twiddles();
}

size_t fb_sort_smem_bytes(int lc) {
  size_t C = size_t(1) << lc;
  return C * 32 + (FB_BUCKETS + 1) * 4 + 256 * 4 + (size_t)FB_WINDOWS * C * 2 + 16;
}

size_t msm_smem_bytes(int lc) {
  size_t C = size_t(1) << lc;
  return C * 32 + (size_t)MSM_WINDOWS * C * 2 + MSM_WINDOWS * 129 * 2 + 129 * 4 + 16;
}

// The dynamic shared-memory limit is a per-device attribute of each kernel,
// so it is raised once for every device a call runs on (the device current at
// the call).
int set_smem_limits() {
  static std::set<int> done;
  static std::mutex m;
  std::lock_guard<std::mutex> g(m);
  int dev = 0;
  ZG_CK(cudaGetDevice(&dev));
  if (done.count(dev)) return 0;
  const int big = 227 * 1024;
  ZG_CK(cudaFuncSetAttribute(k_rows_from_raw, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_rows_ntt, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_msm_chunks, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_fb_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_wd_sort<15>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_wd_sort<14>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_wd_sort<13>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_wd_sort<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_wd_sort<11>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_ntt4_colpass, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  ZG_CK(cudaFuncSetAttribute(k_ntt4_rowpass, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  done.insert(dev);
  return 0;
}

inline unsigned nblk(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// threads of a CTA that runs one 2^logn-point transform: one per radix-4
// group of the shared-memory passes (2^(logn - 2)), within [32, 256]
unsigned ntt_threads(int logn) { return (unsigned)std::min(256, std::max(32, 1 << std::max(0, logn - 2))); }

// natural-order N-point transform out = DFT(x) (or inverse without 1/N), via
// the column / row passes; tmp has N elements
// (batch vectors back to back in x, tmp and out; batch <= 65535). With cs_lo
// set, input i is first multiplied by g^i = cs_lo[i mod 2^cs_h] cs_hi[i >> cs_h]
// (coset shift); with scale set, every output by *scale.
void ntt4(const Twiddles& tw, const Fr* x, Fr* tmp, Fr* out, bool inverse, cudaStream_t s, uint32_t batch = 1,
          const Fr* cs_lo = nullptr, const Fr* cs_hi = nullptr, int cs_h = 0, const Fr* scale = nullptr) {
  const int lr = tw.lr, lc = tw.lc;
  const size_t R = size_t(1) << lr, C = size_t(1) << lc;
  k_ntt4_colpass<<<dim3((unsigned)C, batch), ntt_threads(lr), R * sizeof(Fr), s>>>(
      x, tmp, lr, lc, inverse ? tw.twi_r : tw.twf_r, inverse ? tw.wni_lo : tw.wn_lo, inverse ? tw.wni_hi : tw.wn_hi,
      cs_lo, cs_hi, cs_h);
  k_ntt4_rowpass<<<dim3((unsigned)R, batch), ntt_threads(lc), C * sizeof(Fr), s>>>(
      tmp, out, lr, lc, inverse ? tw.twi_c : tw.twf_c, scale != nullptr, scale ? *scale : Fr::zero());
}

}  // namespace

// Scratch of zg_msm_chunks_noalloc: window sums and per-MSM results of at
// most ZG_NOALLOC_MAX_MSMS chunk MSMs (lines x chunks). It lives in the
// module's static device memory, so every GPU that loads this library holds
// these ~4.3 MB until the process exits.
constexpr uint32_t ZG_NOALLOC_MAX_MSMS = 1024;
static __device__ __align__(256) uint8_t g_noalloc_scratch[(size_t)ZG_NOALLOC_MAX_MSMS * (MSM_WINDOWS + 1) *
                                                           sizeof(XYZZ)];

namespace {
struct Engine;
void engine_shutdown(Engine* e);
}  // namespace

// Device scratch of the encodes issued on one stream: the RS intermediates
// (shared by the lane's blobs, whose passes run one after another) and, per
// blob slot, the MSM's digit-sort output, per-item partial sums, per-chunk
// results and AMT nodes. The context owns a lane of one slot (plain and
// device encodes, verification, zg_ctx_msm); each unit of the request
// pipeline owns a lane of up to FB_MAX_BLOBS slots, whose blobs share one
// bucket-accumulation launch.
struct Lane {
  int cap = 0;                  // blob slots
  Fr* T1 = nullptr;             // [R][C] row-iNTT output
  Fr* Bc = nullptr;             // [2][R][C] column-pass output
  uint32_t* fb_offs = nullptr;  // [cap][3R][FB_BUCKETS + 1]
  uint16_t* fb_ents = nullptr;  // [cap][3R][FB_WINDOWS C]
  struct Wd {
    uint32_t* offs = nullptr;   // [cap][3][units][2^ulog + 1]
    uint32_t* ents = nullptr;   // [cap][3][units][W 2^ulog]
  };
  std::vector<Wd> wd;           // per wide class of the context
  XYZZ* fb_T = nullptr;         // [cap][items][FB_ACC_THREADS]
  XYZZ* fb_S = nullptr;
  XYZZ* fb_gbuf = nullptr;      // per persistent CTA task partial sums
  uint32_t* fb_next = nullptr;  // k_fb_accum's item counter
  XYZZ* win = nullptr;          // 8-bit path: [3][L][R][MSM_WINDOWS] (cap 1)
  XYZZ* part = nullptr;         // [cap][3][L][R] per-item MSM results
  XYZZ* nodes = nullptr;        // [cap][3][4R - 2] AMT nodes
};

struct zg_ctx {
  int device = 0;
  int lr = 0, lc = 0, L = 0;
  size_t R = 0, C = 0, N = 0;
  size_t max_blob = 0, max_raw = 0;
  cudaStream_t stream = nullptr;
  Twiddles tw;
  // params with their fixed-base window multiples: tab[c][l][w][p] (W windows
  // per line, window 0 = the param points themselves)
  bool fb = false;
  int W = 1;
  G1Aff* tab = nullptr;
  G1Aff* line_ptr(int c, int l) const { return tab + ((size_t)c * L + l) * W * N; }
  Lane lane;                        // the context's own scratch (one blob slot)
  unsigned fb_ctas[ZG_MSM_PRODUCTS] = {};  // resident CTAs of k_fb_accum per product kind
  unsigned fb_ctas_max() const {
    unsigned m = 1;
    for (unsigned x : fb_ctas) m = std::max(m, x);
    return m;
  }
  // Wide-window classes (k_wd_sort): class k sorts units of 2^ulog points
  // into 2^ulog buckets of (ulog + 1)-bit digits, for AMT lines l0 .. l0 +
  // nl - 1 (the last one the high line L - 1 when hi_last); tab[c][wl][W][N]
  // holds their window multiples (each lane holds the sort output). With
  // mlog = 1 its items merge pairs of sort units (units of 2^(ulog + 1)
  // points sharing 2^ulog buckets), and the class reads the sort output of
  // class sort_of (the first class of the same ulog, which runs the sort).
  // The 11-bit chunk items cover the other lines, n_l0 .. n_l0 + n_lines - 1.
  struct WdClass {
    int ulog = 0, mlog = 0, sort_of = 0, W = 0, l0 = 0, nl = 0, hi_last = 0;
    G1Aff* tab = nullptr;
  };
  std::vector<WdClass> wd;
  int n_l0 = 0, n_lines = 0;
  int wd_on = 0;  // wide classes in use (a prefix of wd, a tuning choice)
  int wide_lines() const {
    int n = 0;
    for (int k = 0; k < wd_on; ++k) n += wd[k].nl;
    return n;
  }
  // free choices of the kernels (zg_ctx_autotune / zg_ctx_set_tuning); the
  // defaults are the fastest on the B200. tuning_gen counts changes, so the
  // request pipeline re-captures its CUDA graphs.
  uint32_t msm_product = ZG_MSM_PRODUCT_HYBRID;
  uint32_t msm_task = FB_TASK_DEFAULT;
  uint32_t ntt_cpb = 2, ntt_threads = 256;
  uint64_t tuning_gen = 0;
  uint8_t* raw = nullptr;
  uint8_t* enc = nullptr;
  uint8_t* amt = nullptr;
  uint8_t* tree = nullptr;
  uint64_t* tree_off_d = nullptr;
  std::vector<uint64_t> tree_off;
  int tree_depth = 0;  // leaves live at level tree_depth
  size_t tree_bytes = 0;
  uint8_t* slices = nullptr;
  size_t slice_size = 0;
  uint8_t* file_root = nullptr;
  uint8_t* h_in = nullptr;  // pinned staging for payloads
  // recovery buffers and tables, allocated on the first zg_recover call
  bool rec_ready = false;
  Fr *rec_ginv = nullptr, *rec_kpow = nullptr, *rec_kinv = nullptr, *rec_wpow = nullptr, *rec_zinv = nullptr,
     *rec_zw = nullptr;
  Fr *rec_V = nullptr, *rec_W = nullptr;
  uint8_t* rec_rows = nullptr;   // device copy of the received rows
  uint8_t* rec_raw = nullptr;    // device RawData
  uint32_t* rec_ids = nullptr;
  uint16_t* rec_erased = nullptr;
  uint32_t* rec_err = nullptr;
  uint8_t* h_rec = nullptr;      // pinned staging (rows in, RawData out)
  // G2 side of the params, for slice verification: g2 (the generator) and per
  // coset high_g2 and the vanishing points (level d holds 2^(d+1) points at
  // offset 2^(d+1) - 2). Read from the params files, or built from the seeded
  // tau on the first verification.
  bool g2_ready = false;
  bool seeded = false;
  uint64_t tau_seed = 0;
  std::vector<G2Aff> vanish[3];
  G2Aff high_g2[3];
  // measurement: optional per-phase events and a count of kernel launches
  bool profiling = false;
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  // completion of the last encode; every encode's stream waits on it first, so
  // encodes issued on different streams never overlap on the shared scratch
  cudaEvent_t done = nullptr;
  std::atomic<uint64_t> launches{0};
  std::mutex mu;
  // request pipeline (zg_submit / zg_wait / zg_encode_batch), started on
  // first use with the settings of zg_ctx_set_pipeline
  Engine* eng = nullptr;
  std::mutex eng_mu;
  zg_pipeline_config pipe_cfg{0, 0, 0};
  zg_pipeline_stats pipe_stats{};
  // recovery runs on its own stream and buffers, beside the encodes
  cudaStream_t rec_stream = nullptr;
  std::mutex rec_mu;
};

// Process-wide pool of page-locked reply buffers: pinning ~200 MB per reply
// costs far more than the copies themselves, so freed buffers are kept, up
// to 16 GiB in all (a batch of 32 full replies with encoded data is 6.6 GB;
// with a cap of eight buffers per size, a batch that returns its replies
// together re-pinned most of them and ran slower than one blob at a time),
// for the next reply.
namespace {
std::mutex g_pin_mu;
std::multimap<size_t, void*> g_pin_pool;
size_t g_pin_bytes = 0;  // bytes held by the pool
constexpr size_t kPinPoolMax = 16ull << 30;
void* pinned_get(size_t bytes) {
  {
    std::lock_guard<std::mutex> g(g_pin_mu);
    auto it = g_pin_pool.find(bytes);
    if (it != g_pin_pool.end()) {
      void* p = it->second;
      g_pin_pool.erase(it);
      g_pin_bytes -= bytes;
      return p;
    }
  }
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
  return p;
}
void pinned_put(void* p, size_t bytes) {
  if (!p) return;
  std::lock_guard<std::mutex> g(g_pin_mu);
  if (g_pin_bytes + bytes <= kPinPoolMax) {
    g_pin_pool.emplace(bytes, p);
    g_pin_bytes += bytes;
  } else {
    cudaFreeHost(p);
  }
}
}  // namespace

struct zg_reply {
  uint32_t version = 0;
  uint8_t commitment[64];
  uint8_t storage_root[32];
  uint8_t roots[96];
  uint8_t* data = nullptr;  // pinned
  size_t data_len = 0;
  uint8_t* slices = nullptr;  // pinned
  size_t slice_size = 0, nslices = 0;
  std::vector<uint8_t> payload;  // recovered bytes (recovery requests)
};

namespace {

// Wide-window classes of a context with 1024 columns: quotient line l's nodes
// hold 2^(lr + 9 - l) points and the high line's 2^(lr + 10), so a line takes
// units of 2^min(16, log2 node) points when its nodes hold more than 1024
// (units of 2^16 points: pairs of 2^15-point sort units sharing their
// buckets). A class per unit size, largest first; each class's tables are
// allocated only with 8 GiB left over for the blob buffers and the request
// pipeline's slots, and the first class that does not fit ends the list, so
// the chunk lines stay one contiguous range n_l0 .. n_l0 + n_lines - 1 (the
// high line last when it has no class).
constexpr int WD_MERGED_LOG = WD_MAX_LOG + 1;  // largest unit: two sort units
void plan_wide_classes(zg_ctx* c) {
  const int lr = c->lr;
  int next = 0;  // first quotient line without a class
  bool high = false;
  for (int u = WD_MERGED_LOG; u >= WD_MIN_LOG; --u) {
    zg_ctx::WdClass k;
    k.ulog = std::min(u, WD_MAX_LOG);
    k.mlog = u - k.ulog;
    k.sort_of = (int)c->wd.size();
    for (int j = 0; j < (int)c->wd.size(); ++j)
      if (c->wd[j].ulog == k.ulog) {
        k.sort_of = j;
        break;
      }
    k.W = wd_windows(k.ulog);
    k.l0 = next;
    int nq = 0;
    while (next + nq < lr && std::min(WD_MERGED_LOG, lr + 9 - (next + nq)) == u) ++nq;
    const bool hi = std::min(WD_MERGED_LOG, lr + 10) == u;
    if (!nq && !hi) continue;
    k.nl = nq + (hi ? 1 : 0);
    k.hi_last = hi ? 1 : 0;
    const size_t bytes = (size_t)3 * k.nl * k.W * c->N * sizeof(G1Aff);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b < bytes + (8ull << 30) ||
        cudaMalloc(&k.tab, bytes) != cudaSuccess) {
      cudaGetLastError();
      break;
    }
    next += nq;
    high = high || hi;
    c->wd.push_back(k);
  }
  c->n_l0 = next;
  c->n_lines = lr + 1 - next + (high ? 0 : 1);
  c->wd_on = (int)c->wd.size();
}

// Uses the first `on` wide classes (largest unit first); the lines of the
// others run 11-bit chunk items, which stay one contiguous line range.
void apply_wide_classes(zg_ctx* c, int on) {
  int next = 0;
  bool high = false;
  for (int k = 0; k < on; ++k) {
    next += c->wd[k].nl - c->wd[k].hi_last;
    high = high || c->wd[k].hi_last;
  }
  c->wd_on = on;
  c->n_l0 = next;
  c->n_lines = c->lr + 1 - next + (high ? 0 : 1);
}

// work items of one blob's MSM: every (coset, chunk or unit block, line),
// the chunk lines first, then each wide class in use (a merged class has half
// the items per line); blob_items_max bounds it for every choice of classes
uint32_t blob_items_max(const zg_ctx* c) { return (uint32_t)(3 * c->R * c->L); }
uint32_t blob_items(const zg_ctx* c) {
  uint32_t u = (uint32_t)(3 * c->R * c->n_lines);
  for (int j = 0; j < c->wd_on; ++j) u += (uint32_t)(3 * (c->R >> c->wd[j].mlog) * c->wd[j].nl);
  return u;
}

// device bytes of a lane of `cap` blob slots (the request pipeline's
// admission compares this with the free HBM)
size_t lane_bytes(const zg_ctx* c, int cap) {
  const size_t N = c->N, R = c->R;
  size_t b = 3 * N * sizeof(Fr);
  size_t per = 3 * (size_t)c->L * R * sizeof(XYZZ) + 3 * (4 * R - 2) * sizeof(XYZZ);
  if (c->fb) {
    per += 3 * R * (FB_BUCKETS + 1) * 4 + 3 * R * FB_WINDOWS * c->C * 2 +
           2 * (size_t)blob_items_max(c) * FB_ACC_THREADS * sizeof(XYZZ);
    for (size_t j = 0; j < c->wd.size(); ++j) {
      const zg_ctx::WdClass& k = c->wd[j];
      if (k.sort_of == (int)j)
        per += 3 * (N >> k.ulog) * (((size_t)1 << k.ulog) + 1) * 4 + 3 * (N >> k.ulog) * wd_unit_ents(k.ulog) * 4;
    }
    b += (size_t)c->fb_ctas_max() * FB_MAX_TASKS * sizeof(XYZZ);
  } else {
    per += 3 * (size_t)c->L * R * MSM_WINDOWS * sizeof(XYZZ);
  }
  return b + per * (size_t)cap;
}

void free_lane(Lane* ln) {
  void* ps[] = {ln->T1, ln->Bc, ln->fb_offs, ln->fb_ents, ln->fb_T, ln->fb_S, ln->fb_gbuf, ln->fb_next,
                ln->win, ln->part, ln->nodes};
  for (void* p : ps) if (p) cudaFree(p);
  for (Lane::Wd& w : ln->wd) {
    if (w.offs) cudaFree(w.offs);
    if (w.ents) cudaFree(w.ents);
  }
  *ln = Lane();
}

int alloc_lane(zg_ctx* c, Lane* ln, int cap) {
  const size_t N = c->N, R = c->R;
  if (cap < 1 || cap > FB_MAX_BLOBS || (!c->fb && cap > 1)) return fail(ZG_ERR_INVALID_ARG, "lane capacity");
  ln->cap = cap;
  const size_t k = (size_t)cap;
  ZG_CK(cudaMalloc(&ln->T1, N * sizeof(Fr)));
  ZG_CK(cudaMalloc(&ln->Bc, 2 * N * sizeof(Fr)));
  if (c->fb) {
    ZG_CK(cudaMalloc(&ln->fb_offs, k * 3 * R * (FB_BUCKETS + 1) * sizeof(uint32_t)));
    ZG_CK(cudaMalloc(&ln->fb_ents, k * 3 * R * FB_WINDOWS * c->C * sizeof(uint16_t)));
    ZG_CK(cudaMalloc(&ln->fb_T, k * blob_items_max(c) * FB_ACC_THREADS * sizeof(XYZZ)));
    ZG_CK(cudaMalloc(&ln->fb_S, k * blob_items_max(c) * FB_ACC_THREADS * sizeof(XYZZ)));
    ln->wd.resize(c->wd.size());
    for (size_t j = 0; j < c->wd.size(); ++j) {
      if (c->wd[j].sort_of != (int)j) continue;  // reads another class's sort output
      const size_t units = N >> c->wd[j].ulog;
      ZG_CK(cudaMalloc(&ln->wd[j].offs, k * 3 * units * (((size_t)1 << c->wd[j].ulog) + 1) * sizeof(uint32_t)));
      ZG_CK(cudaMalloc(&ln->wd[j].ents, k * 3 * units * wd_unit_ents(c->wd[j].ulog) * sizeof(uint32_t)));
    }
    ZG_CK(cudaMalloc(&ln->fb_gbuf, (size_t)c->fb_ctas_max() * FB_MAX_TASKS * sizeof(XYZZ)));
    ZG_CK(cudaMalloc(&ln->fb_next, sizeof(uint32_t)));
  } else {
    ZG_CK(cudaMalloc(&ln->win, 3 * (size_t)c->L * R * MSM_WINDOWS * sizeof(XYZZ)));
  }
  ZG_CK(cudaMalloc(&ln->part, k * 3 * (size_t)c->L * R * sizeof(XYZZ)));
  ZG_CK(cudaMalloc(&ln->nodes, k * 3 * (4 * R - 2) * sizeof(XYZZ)));
  return 0;
}

int alloc_blob_buffers(zg_ctx* c) {
  if (c->fb) {
    int sms = 0, per_sm[ZG_MSM_PRODUCTS] = {};
    ZG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    ZG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0], k_fb_accum<MulImad>, FB_ACC_THREADS, 0));
    ZG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1], k_fb_accum<MulHybrid>, FB_ACC_THREADS, 0));
    ZG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[2], k_fb_accum<MulF64>, FB_ACC_THREADS, 0));
    ZG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[3], k_fb_accum<MulW28>, FB_ACC_THREADS, 0));
    ZG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[4], k_fb_accum<MulW28Hybrid>, FB_ACC_THREADS, 0));
    for (int k = 0; k < ZG_MSM_PRODUCTS; ++k) c->fb_ctas[k] = (unsigned)std::max(1, sms * std::max(1, per_sm[k]));
  }
  int rc = alloc_lane(c, &c->lane, 1);
  if (rc) return rc;
  const size_t N = c->N, R = c->R;
  ZG_CK(cudaMalloc(&c->raw, c->max_blob + 16));
  ZG_CK(cudaMalloc(&c->enc, 3 * N * 32));
  ZG_CK(cudaMalloc(&c->amt, 3 * (4 * R - 2) * 64));
  // Merkle levels: level d holds 3 * 2^d nodes; leaves at depth LR + LC - 3
  c->tree_depth = c->lr + c->lc - 3;
  c->tree_off.assign(c->tree_depth + 1, 0);
  size_t off = 0;
  for (int d = 0; d <= c->tree_depth; ++d) {
    c->tree_off[d] = off;
    off += (size_t)3 * ((size_t)1 << d) * 32;
  }
  c->tree_bytes = off;
  ZG_CK(cudaMalloc(&c->tree, off));
  ZG_CK(cudaMalloc(&c->tree_off_d, c->tree_off.size() * sizeof(uint64_t)));
  ZG_CK(cudaMemcpy(c->tree_off_d, c->tree_off.data(), c->tree_off.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
  c->slice_size = 312 + 32 * c->C + 160 * (size_t)c->lr;
  ZG_CK(cudaMalloc(&c->slices, 3 * R * c->slice_size));
  ZG_CK(cudaMalloc(&c->file_root, 32));
  ZG_CK(cudaMallocHost(&c->h_in, c->max_blob + 16));
  return 0;
}

// Seeded params on the device: with tau known every param point is s * G1 for
// a scalar s given by the Fr versions of the EC FFT formulas of
// AMTParams::from_pp (generate.rs:139-232):
//   basis      = enact(ifft(tau'^i))
//   quotient_d = enact(fft(c_d) / N),  c_d[i] = tau'^(M-i) for 1 <= i <= M = N >> d
//   high_basis = enact(tau^(3N) * ifft(tau'^i))
// with tau' = tau / coset_factor(N, c) (generate.rs:152-170) and enact =
// normalize + index_reverse (generate.rs:122-126).
int build_seeded_params(zg_ctx* c, uint64_t seed) {
  const size_t N = c->N;
  const int ln = c->lr + c->lc;
  cudaStream_t s = c->stream;
  Fr tau = tau_from_seed(seed);
  Fr* pw = nullptr;
  Fr* sc = nullptr;
  Fr* tmp = nullptr;
  Fr* coeff = nullptr;
  XYZZ* tabx = nullptr;
  G1Aff* tab = nullptr;
  ZG_CK(cudaMalloc(&pw, N * sizeof(Fr)));
  ZG_CK(cudaMalloc(&sc, N * sizeof(Fr)));
  ZG_CK(cudaMalloc(&tmp, N * sizeof(Fr)));
  ZG_CK(cudaMalloc(&coeff, N * sizeof(Fr)));
  ZG_CK(cudaMalloc(&tabx, 32 * 255 * sizeof(XYZZ)));
  ZG_CK(cudaMalloc(&tab, 32 * 255 * sizeof(G1Aff)));
  G1Aff g;
  g.x = Fq::from_u32(1);
  g.y = Fq::from_u32(2);
  k_fixed_table<<<1, 32, 0, s>>>(tabx, g);
  k_xyzz_to_affine<<<nblk(32 * 255, 256), 256, 0, s>>>(tabx, tab, 32 * 255);
  Fr ninv = host_fr_from_u32((uint32_t)N).inverse();
  Fr tau_hs = tau.pow_u64((uint64_t)3 * N);  // high_start = 2^(depth+2) - 2^depth
  const unsigned T = 256;
  for (int cs = 0; cs < 3; ++cs) {
    Fr tp = cs ? tau * coset_factor(ln, cs).inverse() : tau;
    k_powers<<<nblk(N, T), T, 0, s>>>(tp, pw, (uint32_t)N);
    ntt4(c->tw, pw, tmp, sc, true, s);
    k_scale<<<nblk(N, T), T, 0, s>>>(sc, ninv, (uint32_t)N);
    k_fixed_mul<<<nblk(N, T), T, 0, s>>>(tab, sc, c->line_ptr(cs, c->lr), (uint32_t)N, ln);
    k_scale<<<nblk(N, T), T, 0, s>>>(sc, tau_hs, (uint32_t)N);
    k_fixed_mul<<<nblk(N, T), T, 0, s>>>(tab, sc, c->line_ptr(cs, c->lr + 1), (uint32_t)N, ln);
    for (int d = 1; d <= c->lr; ++d) {
      k_quot_coeff<<<nblk(N, T), T, 0, s>>>(pw, coeff, (uint32_t)(N >> d), (uint32_t)N);
      ntt4(c->tw, coeff, tmp, sc, false, s);
      k_scale<<<nblk(N, T), T, 0, s>>>(sc, ninv, (uint32_t)N);
      k_fixed_mul<<<nblk(N, T), T, 0, s>>>(tab, sc, c->line_ptr(cs, d - 1), (uint32_t)N, ln);
    }
  }
  ZG_CK(cudaStreamSynchronize(s));
  ZG_CK(cudaGetLastError());
  cudaFree(pw); cudaFree(sc); cudaFree(tmp); cudaFree(coeff); cudaFree(tabx); cudaFree(tab);
  return 0;
}

// reference mont files: amt-prove-coset{c}-mont-{hash}-{LR:02}-{LN:02}.bin
// (crates/amt/src/utils.rs:20-45; format fast_serde_bn254.rs:20-88)
// canonical little-endian field element (top `flag_bits` bits of the last
// byte masked off) below the modulus
template <class F>
bool field_from_le(const uint8_t* b, F* out, uint8_t* flags = nullptr) {
  F x;
  for (int i = 0; i < 8; ++i)
    x.v[i] = (uint32_t)b[4 * i] | (uint32_t)b[4 * i + 1] << 8 | (uint32_t)b[4 * i + 2] << 16 |
             (uint32_t)b[4 * i + 3] << 24;
  if (flags) {
    *flags = (uint8_t)(x.v[7] >> 30);
    x.v[7] &= 0x3fffffffu;
  }
  F d;
  if (!F::sub_raw(d, x, F::modulus())) return false;  // x >= modulus
  *out = F::from_canonical(x);
  return true;
}

// ark-serialize uncompressed G2 (x.c0 | x.c1 | y.c0 | y.c1, flags in the top
// bits of the last byte)
bool g2_from_ark(const uint8_t* b, G2Aff* out) {
  uint8_t fl = 0;
  Fq t[4];
  for (int k = 0; k < 4; ++k)
    if (!field_from_le(b + 32 * k, &t[k], k == 3 ? &fl : nullptr)) return false;
  if (fl == 3) return false;
  out->inf = fl == 1;
  out->x = Fq2{t[0], t[1]};
  out->y = Fq2{t[2], t[3]};
  return true;
}

int load_mont_params(zg_ctx* c, const char* dir) {
  const int ln = c->lr + c->lc;
  std::vector<uint8_t> hostline(c->N * 64);
  for (int cs = 0; cs < 3; ++cs) {
    char prefix[64], suffix[32];
    snprintf(prefix, sizeof(prefix), "amt-prove-coset%d-mont-", cs);
    snprintf(suffix, sizeof(suffix), "-%02d-%02d.bin", c->lr, ln);
    std::string found;
    DIR* dp = opendir(dir);
    if (!dp) return fail(ZG_ERR_PARAMS, std::string("cannot open params dir ") + dir);
    while (dirent* e = readdir(dp)) {
      std::string n = e->d_name;
      if (n.rfind(prefix, 0) == 0 && n.size() > strlen(suffix) &&
          n.compare(n.size() - strlen(suffix), strlen(suffix), suffix) == 0) {
        found = std::string(dir) + "/" + n;
        break;
      }
    }
    closedir(dp);
    if (found.empty()) return fail(ZG_ERR_PARAMS, std::string("no ") + prefix + "*" + suffix + " in " + dir);
    FILE* f = fopen(found.c_str(), "rb");
    if (!f) return fail(ZG_ERR_PARAMS, "cannot open " + found);
    uint8_t hdr[6];
    bool ok = fread(hdr, 1, 6, f) == 6 && memcmp(hdr, "bamt", 4) == 0 && hdr[4] == ln && hdr[5] == c->lr;
    uint8_t g2b[256];
    ok = ok && fread(g2b, 1, 256, f) == 256;  // g2, high_g2 (uncompressed G2, 128 B each)
    ok = ok && g2_from_ark(g2b + 128, &c->high_g2[cs]);
    auto read_line = [&](G1Aff* dst) {
      if (fread(hostline.data(), 1, hostline.size(), f) != hostline.size()) return false;
      return cudaMemcpy(dst, hostline.data(), hostline.size(), cudaMemcpyHostToDevice) == cudaSuccess;
    };
    ok = ok && read_line(c->line_ptr(cs, c->lr));  // basis
    for (int d = 0; ok && d < c->lr; ++d) ok = read_line(c->line_ptr(cs, d));
    // vanishing points: raw Montgomery x.c0 | x.c1 | y.c0 | y.c1 (fast_serde_bn254.rs:139-160)
    c->vanish[cs].assign((size_t)2 * c->R - 2, G2Aff{});
    for (size_t k = 0; ok && k < c->vanish[cs].size(); ++k) {
      uint32_t w[32];
      ok = fread(w, 1, 128, f) == 128;
      G2Aff& g = c->vanish[cs][k];
      for (int i = 0; i < 8; ++i) {
        g.x.c0.v[i] = w[i];
        g.x.c1.v[i] = w[8 + i];
        g.y.c0.v[i] = w[16 + i];
        g.y.c1.v[i] = w[24 + i];
      }
      g.inf = 0;
    }
    ok = ok && read_line(c->line_ptr(cs, c->lr + 1));  // high_basis
    fclose(f);
    if (!ok) return fail(ZG_ERR_PARAMS, "malformed params file " + found);
  }
  c->g2_ready = true;
  return 0;
}

int check_launch() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ZG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return 0;
}

// Leaves, then one launch per level down to MERKLE_TOP_MAX, then the levels
// above in one k_merkle_top launch (off[d] = 96 (2^d - 1), the layout it
// assumes).
int merkle_levels(const uint8_t* items, size_t n_items, uint8_t* tree, const std::vector<uint64_t>& off,
                  int depth, cudaStream_t s) {
  const unsigned T = 128;
  size_t leaves = n_items / 8;
  k_merkle_leaves<<<nblk(leaves, T), T, 0, s>>>(items, tree + off[depth], (uint32_t)leaves);
  const int top = std::min(depth, MERKLE_TOP_MAX);
  for (int d = depth - 1; d >= top; --d) {
    size_t cnt = (size_t)3 << d;
    k_merkle_parents<<<nblk(cnt, T), T, 0, s>>>(tree + off[d + 1], tree + off[d], (uint32_t)cnt);
  }
  if (top > 0) k_merkle_top<<<3, std::max(1, 1 << (top - 1)), 0, s>>>(tree, top);
  return check_launch();
}

// Per-blob inputs and outputs: the payload, the encoded data, the Merkle
// tree, the serialized AMT nodes, the slices and the file root. The context
// owns one set (the plain path); every slot of the request pipeline owns
// one, so one blob's copies overlap another's compute.
struct BlobBufs {
  uint8_t* raw = nullptr;
  uint64_t* d_len = nullptr;  // payload length, for graph launches
  uint8_t* enc = nullptr;
  uint8_t* tree = nullptr;
  uint8_t* amt = nullptr;
  uint8_t* slices = nullptr;
  uint8_t* file_root = nullptr;
};

BlobBufs ctx_bufs(zg_ctx* c) {
  BlobBufs b;
  b.raw = c->raw;
  b.enc = c->enc;
  b.tree = c->tree;
  b.amt = c->amt;
  b.slices = c->slices;
  b.file_root = c->file_root;
  return b;
}

// Kernel launches of an encode of nb blobs on one lane: per blob 3 RS passes,
// the Merkle leaves, lower parent levels and top levels, file root, the
// digit sorts, trees,
// serialisation and slices; once for all of them the bucket accumulation
// (and its counter reset) and the combine (the 8-bit path: chunks + combine
// per blob).
uint64_t launches_per_encode(const zg_ctx* c, int nb = 1) {
  const int top = std::min(c->tree_depth, MERKLE_TOP_MAX);
  const uint64_t merkle = 1 + (uint64_t)(c->tree_depth - top) + (top > 0 ? 1 : 0);
  uint64_t sorts = 0;  // the wide classes in use that run their own digit sort
  for (int k = 0; k < c->wd_on; ++k) sorts += c->wd[k].sort_of == k ? 1 : 0;
  const uint64_t per = 3 + merkle + 1 + (c->fb ? 1 + sorts : 2) + 1 + 1 + 1;
  return per * (uint64_t)nb + (c->fb ? 2 : 0);
}

// blob slot b's chunk work items: (coset, chunk, line) over the 11-bit tables,
// for the lines without wide windows (n_l0 .. n_l0 + n_lines - 1)
FbAccArgs blob_fb_args(const zg_ctx* c, const Lane& ln, int b = 0) {
  const size_t R = c->R;
  FbAccArgs fa;
  fa.tab = c->tab;
  fa.offs = ln.fb_offs + (size_t)b * 3 * R * (FB_BUCKETS + 1);
  fa.ents = ln.fb_ents + (size_t)b * 3 * R * FB_WINDOWS * c->C;
  fa.outT = ln.fb_T + (size_t)b * blob_items(c) * FB_ACC_THREADS;
  fa.outS = ln.fb_S + (size_t)b * blob_items(c) * FB_ACC_THREADS;
  fa.lr = c->lr;
  fa.lc = c->lc;
  fa.lines = c->n_lines;
  fa.l0 = c->n_l0;
  fa.Ltot = c->L;
  fa.W = FB_WINDOWS;
  fa.tabN = c->N;
  return fa;
}

// first item of wide class k in a blob's item order (chunk items, then the
// classes); the (T, S) partials of item u sit at fb_T / fb_S + 128 u
uint32_t blob_wd_first_item(const zg_ctx* c, size_t k) {
  uint32_t u = (uint32_t)(3 * c->R * c->n_lines);
  for (size_t j = 0; j < k; ++j) u += (uint32_t)(3 * (c->R >> c->wd[j].mlog) * c->wd[j].nl);
  return u;
}

// the sort output of wide class k for blob slot b
uint32_t* lane_wd_offs(const zg_ctx* c, const Lane& ln, size_t k, int b) {
  const size_t units = c->N >> c->wd[k].ulog;
  return ln.wd[c->wd[k].sort_of].offs + (size_t)b * 3 * units * (((size_t)1 << c->wd[k].ulog) + 1);
}
uint32_t* lane_wd_ents(const zg_ctx* c, const Lane& ln, size_t k, int b) {
  return ln.wd[c->wd[k].sort_of].ents + (size_t)b * 3 * c->N * wd_windows(c->wd[k].ulog);
}

// blob slot b's work items of wide class k: (coset, unit block, line)
FbAccArgs blob_wd_args(const zg_ctx* c, const Lane& ln, size_t k, int b = 0) {
  const zg_ctx::WdClass& w = c->wd[k];
  const size_t first = ((size_t)b * blob_items(c) + blob_wd_first_item(c, k)) * FB_ACC_THREADS;
  FbAccArgs fa;
  fa.tab = w.tab;
  fa.offs = lane_wd_offs(c, ln, k, b);
  fa.ents32 = lane_wd_ents(c, ln, k, b);
  fa.outT = ln.fb_T + first;
  fa.outS = ln.fb_S + first;
  fa.lr = c->lr - w.mlog;  // 2^lr items per (coset, line)
  fa.lc = c->lc;
  fa.lines = w.nl;
  fa.l0 = 0;
  fa.Ltot = w.nl;
  fa.ulog = w.ulog;
  fa.mlog = w.mlog;
  fa.W = w.W;
  fa.tabN = c->N;
  return fa;
}

// the combine plan of nb blobs on a lane: per blob the chunk items, then
// every wide class; blob b's items follow blob b - 1's, its results go to
// part block b
FbCombinePlan blob_fb_plan(const zg_ctx* c, int nb = 1) {
  FbCombinePlan p;
  const int per = 1 + c->wd_on;
  const uint64_t part_blk = 3 * (uint64_t)c->L * c->R;
  p.n = per * nb;
  for (int b = 0; b < nb; ++b) {
    const uint32_t base = (uint32_t)b * blob_items(c);
    p.start[per * b] = base;
    p.m[per * b] = FbCombineMap{c->lr, c->n_lines, c->n_l0, c->L, 0, 0, 0, part_blk * b};
    for (size_t k = 0; k < (size_t)c->wd_on; ++k) {
      const zg_ctx::WdClass& w = c->wd[k];
      p.start[per * b + 1 + k] = base + blob_wd_first_item(c, k);
      p.m[per * b + 1 + k] =
          FbCombineMap{c->lr - w.mlog, w.nl, w.l0, c->L, w.hi_last, w.ulog - 10, w.mlog, part_blk * b};
    }
  }
  p.start[p.n] = (uint32_t)nb * blob_items(c);
  return p;
}

// the items of a single MSM over one table line (lines = 1)
FbCombinePlan single_fb_plan(int lr) {
  FbCombinePlan p;
  p.n = 1;
  p.start[0] = 0;
  p.start[1] = 1u << lr;
  p.m[0] = FbCombineMap{lr, 1, 0, 1, 0, 0, 0, 0};
  return p;
}

// seeded pseudo-random payload bytes (the autotuner's synthetic blob)
__global__ void k_fill_payload(uint8_t* p, uint64_t n, uint64_t seed) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t z = (i >> 3) * 0x9e3779b97f4a7c15ull + seed;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    p[i] = (uint8_t)(z >> (8 * (i & 7)));
  }
}

// k_fb_accum over the item sets of `p` with product kind `kind`, on a lane's
// counter and task scratch
void launch_fb_accum(const zg_ctx* c, const Lane& ln, uint32_t kind, const FbAccPlan& p, cudaStream_t s) {
  const uint32_t units = p.start[p.n];
  const unsigned grid = std::min<unsigned>(c->fb_ctas[kind], units);
  cudaMemsetAsync(ln.fb_next, 0, sizeof(uint32_t), s);
  const uint32_t task = c->msm_task;
  switch (kind) {
    case ZG_MSM_PRODUCT_IMAD: k_fb_accum<MulImad><<<grid, FB_ACC_THREADS, 0, s>>>(p, ln.fb_gbuf, ln.fb_next, task); break;
    case ZG_MSM_PRODUCT_FP64: k_fb_accum<MulF64><<<grid, FB_ACC_THREADS, 0, s>>>(p, ln.fb_gbuf, ln.fb_next, task); break;
    case ZG_MSM_PRODUCT_W28: k_fb_accum<MulW28><<<grid, FB_ACC_THREADS, 0, s>>>(p, ln.fb_gbuf, ln.fb_next, task); break;
    case ZG_MSM_PRODUCT_W28_HYBRID:
      k_fb_accum<MulW28Hybrid><<<grid, FB_ACC_THREADS, 0, s>>>(p, ln.fb_gbuf, ln.fb_next, task);
      break;
    default: k_fb_accum<MulHybrid><<<grid, FB_ACC_THREADS, 0, s>>>(p, ln.fb_gbuf, ln.fb_next, task); break;
  }
}

// a plan of one item set: the first `units` items of `fa`
FbAccPlan single_acc_plan(const FbAccArgs& fa, uint32_t units) {
  FbAccPlan p;
  p.n = 1;
  p.start[0] = 0;
  p.start[1] = units;
  p.a[0] = fa;
  return p;
}

// The MSM items of nb blobs on a lane in one plan. The sets run in order of
// decreasing entries per item (the wide items of 2^16-point units, the chunk
// items, then the other wide classes from 2^11-point units, 22 windows, to
// 2^15, 16 windows), blob by blob within a kind, so that the persistent
// kernel ends on its shortest items; each set's results still go to its
// place in the combine's item order (blob_fb_plan).
FbAccPlan blob_acc_plan(const zg_ctx* c, const Lane& ln, int nb = 1) {
  struct Kind {
    int k;  // wide class, or -1 for the chunk items
    uint32_t ents;  // entries per item (windows x 1024 points)
  };
  std::vector<Kind> kinds{{-1, (uint32_t)FB_WINDOWS * 1024u}};
  for (int k = 0; k < c->wd_on; ++k)
    kinds.push_back({k, ((uint32_t)wd_windows(c->wd[k].ulog) * 1024u) << c->wd[k].mlog});
  std::stable_sort(kinds.begin(), kinds.end(), [](const Kind& x, const Kind& y) { return x.ents > y.ents; });
  FbAccPlan p;
  uint32_t at = 0;
  for (const Kind& kd : kinds)
    for (int b = 0; b < nb; ++b) {
      p.start[p.n] = at;
      if (kd.k < 0) {
        p.a[p.n] = blob_fb_args(c, ln, b);
        at += (uint32_t)(3 * c->R * c->n_lines);
      } else {
        const zg_ctx::WdClass& w = c->wd[kd.k];
        p.a[p.n] = blob_wd_args(c, ln, (size_t)kd.k, b);
        at += (uint32_t)(3 * (c->R >> w.mlog) * w.nl);
      }
      ++p.n;
    }
  p.start[p.n] = at;
  return p;
}

// P = sum_i T_i + 8 sum_i i S_i per item: one thread per item for a blob's
// items (fewest additions), one warp per item below 16 384 items
void launch_fb_combine(const Lane& ln, const FbCombinePlan& p, cudaStream_t s) {
  const uint32_t units = p.start[p.n];
  if (units >= 16384) k_fb_combine<<<nblk(units, 64), 64, 0, s>>>(ln.fb_T, ln.fb_S, ln.part, p);
  else k_fb_combine_warp<<<nblk((size_t)units * 32, 128), 128, 0, s>>>(ln.fb_T, ln.fb_S, ln.part, p);
}

// k_wd_sort / k_wd_tables for a class's unit size
void launch_wd_sort(int ulog, const uint8_t* enc, uint32_t* offs, uint32_t* ents, int lr, int lc, size_t N,
                    cudaStream_t s) {
  const dim3 grid((unsigned)(N >> ulog), 3);
  const size_t sm = wd_sort_smem_bytes(ulog);
  switch (ulog) {
    case 15: k_wd_sort<15><<<grid, WD_SORT_THREADS, sm, s>>>(enc, offs, ents, lr, lc, 1, N); break;
    case 14: k_wd_sort<14><<<grid, WD_SORT_THREADS, sm, s>>>(enc, offs, ents, lr, lc, 1, N); break;
    case 13: k_wd_sort<13><<<grid, WD_SORT_THREADS, sm, s>>>(enc, offs, ents, lr, lc, 1, N); break;
    case 12: k_wd_sort<12><<<grid, WD_SORT_THREADS, sm, s>>>(enc, offs, ents, lr, lc, 1, N); break;
    default: k_wd_sort<11><<<grid, WD_SORT_THREADS, sm, s>>>(enc, offs, ents, lr, lc, 1, N); break;
  }
}
void launch_wd_tables(const zg_ctx* c, const zg_ctx::WdClass& k, cudaStream_t s) {
  const unsigned g = nblk((uint64_t)3 * k.nl * c->N, 128);
  switch (k.ulog) {
    case 15: k_wd_tables<15><<<g, 128, 0, s>>>(k.tab, c->tab, c->N, c->L, k.l0, k.nl, k.hi_last); break;
    case 14: k_wd_tables<14><<<g, 128, 0, s>>>(k.tab, c->tab, c->N, c->L, k.l0, k.nl, k.hi_last); break;
    case 13: k_wd_tables<13><<<g, 128, 0, s>>>(k.tab, c->tab, c->N, c->L, k.l0, k.nl, k.hi_last); break;
    case 12: k_wd_tables<12><<<g, 128, 0, s>>>(k.tab, c->tab, c->N, c->L, k.l0, k.nl, k.hi_last); break;
    default: k_wd_tables<11><<<g, 128, 0, s>>>(k.tab, c->tab, c->N, c->L, k.l0, k.nl, k.hi_last); break;
  }
}

// the three RS-extension passes with a given column tile and block size
void launch_rs(const zg_ctx* c, const Lane& ln, const uint8_t* raw, size_t len, const uint64_t* d_len, uint8_t* enc,
               uint32_t cpb, uint32_t threads, cudaStream_t s) {
  const int lr = c->lr, lc = c->lc;
  const size_t R = c->R, C = c->C;
  k_rows_from_raw<<<(unsigned)R, threads, C * sizeof(Fr) + 31 * C + 16, s>>>(raw, len, d_len, c->max_raw, lr, lc, enc,
                                                                        ln.T1, c->tw.twi_c, c->tw.wni_lo,
                                                                        c->tw.wni_hi);
  k_cols<<<nblk(C, cpb), threads, 2 * R * sizeof(Fr), s>>>(ln.T1, ln.Bc, lr, lc, c->tw.twi_r, c->tw.twf_r,
                                                            c->tw.gs_lo, c->tw.gs_hi, c->tw.wn_lo, c->tw.wn_hi,
                                                            (int)cpb);
  k_rows_ntt<<<dim3((unsigned)R, 2), threads, C * sizeof(Fr), s>>>(ln.Bc, enc, lr, lc, c->tw.twf_c);
}

// The pipeline of nb blobs on one lane, launches only, in three phases:
// PHASE_PRE every blob's RS extension, Merkle tree and digit sorts;
// PHASE_ACC ONE bucket accumulation over all their MSM items; PHASE_POST ONE
// combine, then every blob's AMT trees, serialisation and slices. Blob i's
// payload is `lens[i]` bytes at b[i].raw, or *b[i].d_len bytes when
// `by_device_len` (graph capture).
constexpr int PHASE_PRE = 1, PHASE_ACC = 2, PHASE_POST = 4, PHASE_ALL = 7;
int encode_launches(zg_ctx* c, const Lane& ln, const BlobBufs* b, int nb, const size_t* lens, bool by_device_len,
                    cudaStream_t s, bool marks, int phases = PHASE_ALL) {
  const int lr = c->lr, lc = c->lc;
  const size_t R = c->R, N = c->N;
  if (nb < 1 || nb > ln.cap) return fail(ZG_ERR_INTERNAL, "lane capacity exceeded");
  auto mark = [&](int k) {
    if (marks && c->profiling) cudaEventRecord(c->ev[k], s);
  };
  int rc = 0;
  if (phases & PHASE_PRE) {
  mark(0);
  // RS extension: rows iNTT, column passes, rows NTT
  for (int i = 0; i < nb; ++i)
    launch_rs(c, ln, b[i].raw, by_device_len ? 0 : lens[i], by_device_len ? b[i].d_len : nullptr, b[i].enc,
              c->ntt_cpb, c->ntt_threads, s);
  rc = check_launch();
  if (rc) return rc;
  mark(1);
  // Merkle tree over the encoded data and the file root
  for (int i = 0; i < nb; ++i) {
    if ((rc = merkle_levels(b[i].enc, 3 * N, b[i].tree, c->tree_off, c->tree_depth, s))) return rc;
    k_file_root<<<1, 32, 0, s>>>(b[i].tree + c->tree_off[0], b[i].file_root);
  }
  mark(2);
  // AMT: MSM items of every blob, trees, serialisation
  if (c->fb) {
    for (int i = 0; i < nb; ++i) {
      const FbAccArgs fa = blob_fb_args(c, ln, i);
      k_fb_sort<<<dim3((unsigned)R, 3), 256, fb_sort_smem_bytes(lc), s>>>(b[i].enc, const_cast<uint32_t*>(fa.offs),
                                                                           const_cast<uint16_t*>(fa.ents), lr, lc, 1, N);
      for (size_t k = 0; k < (size_t)c->wd_on; ++k)
        if (c->wd[k].sort_of == (int)k)
          launch_wd_sort(c->wd[k].ulog, b[i].enc, lane_wd_offs(c, ln, k, i), lane_wd_ents(c, ln, k, i), lr, lc, N, s);
    }
  }
  }  // PHASE_PRE
  if (c->fb) {
    if (phases & PHASE_ACC) launch_fb_accum(c, ln, c->msm_product, blob_acc_plan(c, ln, nb), s);
    if (phases & PHASE_POST) {
      mark(3);
      launch_fb_combine(ln, blob_fb_plan(c, nb), s);
    }
  } else {
    MsmChunkArgs a;
    a.scalars = b[0].enc;
    a.bases = c->tab;
    a.win = ln.win;
    a.lr = lr;
    a.lc = lc;
    a.lines = c->L;
    a.bitrev_rows = 1;
    a.scalar_coset_stride = N;
    a.base_coset_stride = (uint64_t)c->L * c->W * N;
    a.base_line_stride = (uint64_t)c->W * N;
    if (phases & PHASE_ACC) k_msm_chunks<<<dim3((unsigned)R, 3), MSM_THREADS, msm_smem_bytes(lc), s>>>(a);
    if (phases & PHASE_POST) {
      mark(3);
      const uint32_t nmsm = (uint32_t)(3 * c->L * R);
      k_msm_combine<<<nblk(nmsm, 64), 64, 0, s>>>(ln.win, ln.part, nmsm);
    }
  }
  if (!(phases & PHASE_POST)) return check_launch();
  const uint32_t nn = (uint32_t)(3 * (4 * R - 2));
  for (int i = 0; i < nb; ++i) {
    XYZZ* part = ln.part + (size_t)i * 3 * c->L * R;
    XYZZ* nodes = ln.nodes + (size_t)i * nn;
    k_amt_tree<<<dim3((unsigned)c->L, 3), 256, 0, s>>>(part, nodes, lr, c->L);
    k_serialize_nodes<<<nblk(nn, 128), 128, 0, s>>>(nodes, b[i].amt, nn);
  }
  mark(4);
  for (int i = 0; i < nb; ++i) {
    SliceArgs sa;
    sa.enc = b[i].enc;
    sa.amt = b[i].amt;
    sa.tree = b[i].tree;
    sa.tree_off = c->tree_off_d;
    sa.out = b[i].slices;
    sa.lr = lr;
    sa.lc = lc;
    sa.slice_size = c->slice_size;
    k_slices<<<(unsigned)(3 * R), 256, 0, s>>>(sa);
  }
  mark(5);
  return check_launch();
}

// the full per-blob pipeline on the context's own lane and buffers; d_data
// holds `len` payload bytes
int encode_device_locked(zg_ctx* c, const uint8_t* d_data, size_t len, cudaStream_t s) {
  if (cudaStreamWaitEvent(s, c->done, 0) != cudaSuccess) return fail(ZG_ERR_CUDA, "stream wait failed");
  BlobBufs b = ctx_bufs(c);
  b.raw = const_cast<uint8_t*>(d_data);
  int rc = encode_launches(c, c->lane, &b, 1, &len, false, s, true);
  if (rc) return rc;
  c->launches += launches_per_encode(c);
  if (cudaEventRecord(c->done, s) != cudaSuccess) return fail(ZG_ERR_CUDA, "event record failed");
  return 0;
}

std::mutex g_ntt_mu;
// twiddle tables of the standalone entry points, per (device, lr, lc): device
// memory of the device current at the call
std::map<std::tuple<int, int, int>, Twiddles> g_ntt_tw;

int current_device() {
  int dev = 0;
  cudaGetDevice(&dev);
  return dev;
}

const Twiddles* cached_twiddles(int lr, int lc) {
  std::lock_guard<std::mutex> g(g_ntt_mu);
  auto key = std::make_tuple(current_device(), lr, lc);
  auto it = g_ntt_tw.find(key);
  if (it != g_ntt_tw.end()) return &it->second;
  Twiddles t;
  if (make_twiddles(lr, lc, &t)) return nullptr;
  return &(g_ntt_tw[key] = t);
}

// g^e for e < 2^logn as lo[e & (2^h - 1)] * hi[e >> h], h = (logn + 1) / 2
// (Montgomery form), for the coset shift of zg_ntt; one pair per (device, logn,
// coset)
// g^e = lo[e mod 2^h] * hi[e >> h] for e < 2^logn (h = logn: lo alone)
struct CosetPows {
  Fr* lo = nullptr;
  Fr* hi = nullptr;
  int h = 0;
};
std::map<std::tuple<int, int, uint32_t>, CosetPows> g_coset_pows;  // per device; guarded by g_ntt_mu

const CosetPows* cached_coset_pows(int logn, uint32_t coset) {
  std::lock_guard<std::mutex> g(g_ntt_mu);
  auto key = std::make_tuple(current_device(), logn, coset);
  auto it = g_coset_pows.find(key);
  if (it != g_coset_pows.end()) return &it->second;
  CosetPows p;
  // one full table up to the single-CTA transform's size, else split in two
  p.h = logn <= 11 ? logn : (logn + 1) / 2;
  const size_t nlo = size_t(1) << p.h, nhi = size_t(1) << (logn - p.h);
  const Fr gen = coset_factor(logn, coset);
  std::vector<Fr> lo(nlo), hi(nhi);
  lo[0] = Fr::one();
  for (size_t j = 1; j < nlo; ++j) lo[j] = lo[j - 1] * gen;
  const Fr gh = lo[nlo - 1] * gen;  // g^(2^h)
  hi[0] = Fr::one();
  for (size_t j = 1; j < nhi; ++j) hi[j] = hi[j - 1] * gh;
  if (cudaMalloc(&p.lo, nlo * sizeof(Fr)) != cudaSuccess || cudaMalloc(&p.hi, nhi * sizeof(Fr)) != cudaSuccess ||
      cudaMemcpy(p.lo, lo.data(), nlo * sizeof(Fr), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p.hi, hi.data(), nhi * sizeof(Fr), cudaMemcpyHostToDevice) != cudaSuccess) {
    if (p.lo) cudaFree(p.lo);
    if (p.hi) cudaFree(p.hi);
    return nullptr;
  }
  return &(g_coset_pows[key] = p);
}

// The stream-ordered pool of the current device keeps freed memory instead of
// returning it at every synchronisation, so zg_ntt's per-call scratch
// (cudaMallocAsync / cudaFreeAsync) is mapped once, not once per call. The
// pool then holds the largest scratch used so far (one transform batch).
void keep_pool_memory() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  static std::set<int> done;  // guarded by g_ntt_mu
  std::lock_guard<std::mutex> g(g_ntt_mu);
  if (!done.insert(dev).second) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
}

// single-CTA transform of each contiguous vector (n <= 2048). The coset
// shift (input i times g^i, from the full table cs_lo when cs_lo is set) and
// the inverse's 1/n (output times scale, when do_scale) are products of the
// transform's own loads and stores: Montgomery products with Montgomery
// constants, so canonical values stay canonical.
__global__ void __launch_bounds__(256) k_ntt_small(Fr* v, int logn, const Fr* tw, const Fr* __restrict__ cs_lo,
                                                   int do_scale, Fr scale) {
  extern __shared__ __align__(16) uint8_t smem[];
  Fr* s = reinterpret_cast<Fr*>(smem);
  const int n = 1 << logn;
  Fr* p = v + (size_t)blockIdx.x * n;
  ntt_block(s, logn, tw, [&](int i) { return cs_lo ? p[i] * cs_lo[i] : p[i]; },
            [&](int i, const Fr& x) { p[i] = do_scale ? x * scale : x; });
}


// device-vs-host arithmetic self test: out[k] counts mismatches of op k over
// n input pairs (0 Fq mul, 1 Fq mul with immediate modulus, 2 Fq add, 3 Fq sub,
// 4 Fr mul, 5 Fr canonical round trip, 6 XYZZ add vs doubling, 7 Fq mul with
// 28-bit limbs, 8 Fr mul on the FP64 pipe)
constexpr int SELFTEST_OPS = 9;
__global__ void k_selftest(const Fq* a, const Fq* b, Fq* res, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Fq x = a[i], y = b[i];
  res[SELFTEST_OPS * i + 0] = Fq::mul(x, y);
  res[SELFTEST_OPS * i + 1] = f52::mont_mul(x, y);
  res[SELFTEST_OPS * i + 2] = Fq::add(x, y);
  res[SELFTEST_OPS * i + 3] = Fq::sub(x, y);
  Fr xr = *reinterpret_cast<const Fr*>(&x), yr = *reinterpret_cast<const Fr*>(&y);
  Fr m = Fr::mul(xr, yr);
  res[SELFTEST_OPS * i + 4] = *reinterpret_cast<Fq*>(&m);
  Fr rt = Fr::from_canonical(xr).to_canonical();
  res[SELFTEST_OPS * i + 5] = *reinterpret_cast<Fq*>(&rt);
  // P + P via add() must equal dbl(); P = (x, y) is not on the curve, the
  // formulas are still polynomial identities in the coordinates
  XYZZ p1 = XYZZ::from_affine(G1Aff{x, y});
  XYZZ d1 = p1.dbl();
  XYZZ s1 = p1;
  s1.add(p1);
  res[SELFTEST_OPS * i + 6] = (d1.X == s1.X && d1.Y == s1.Y && d1.ZZ == s1.ZZ && d1.ZZZ == s1.ZZZ) ? Fq::one() : Fq::zero();
  res[SELFTEST_OPS * i + 7] = w28::mont_mul(x, y);
  Fr mf = f52::mont_mul(xr, yr);
  res[SELFTEST_OPS * i + 8] = *reinterpret_cast<Fq*>(&mf);
}




// independent 32-bit multiply-add chains: the integer multiply throughput the
// Montgomery products are built from
__global__ void k_imad_probe(uint32_t* sink, uint32_t iters, uint32_t seed) {
  uint32_t a0 = seed + threadIdx.x, a1 = a0 ^ 0x9e3779b9u, a2 = a0 + 0x7f4a7c15u, a3 = a0 * 3u,
           a4 = a0 ^ 0x85ebca6bu, a5 = a0 + 0xc2b2ae35u, a6 = a0 * 5u, a7 = a0 ^ 0x27d4eb2fu;
  const uint32_t m = seed | 1u, k = seed ^ 0x5bd1e995u;
  for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a0) : "r"(m), "r"(k));
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a1) : "r"(m), "r"(k));
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a2) : "r"(m), "r"(k));
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a3) : "r"(m), "r"(k));
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a4) : "r"(m), "r"(k));
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a5) : "r"(m), "r"(k));
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a6) : "r"(m), "r"(k));
      asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a7) : "r"(m), "r"(k));
    }
  }
  uint32_t x = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
  if (x == 0x12345678u) sink[0] = x;
}

// Recovery set-up: tables for the factored decode (see zg_recover.cuh) and
// buffers sized for 3R received rows.
int rec_setup(zg_ctx* c) {
  if (c->rec_ready) return 0;
  const int lr = c->lr, lc = c->lc, lm = c->lr + 2;
  const size_t R = c->R, C = c->C, M = size_t(1) << lm;
  if (lr > 10) return fail(ZG_ERR_INVALID_ARG, "recovery supports log_row <= 10");
  std::vector<Fr> ginv;
  Fr cinv = host_fr_from_u32((uint32_t)C).inverse();
  for (int cs = 0; cs < 3; ++cs) {
    Fr g = cs ? coset_factor(lr + lc, cs).inverse() : Fr::one();
    std::vector<Fr> t = pow_table(g, C);
    for (auto& x : t) x = x * cinv;
    ginv.insert(ginv.end(), t.begin(), t.end());
  }
  Fr k = host_fr_from_u32(5);  // generator of Fr*: never a root of unity of the domain
  Fr minv = host_fr_from_u32((uint32_t)M).inverse();
  std::vector<Fr> kp = pow_table(k, M), ki = pow_table(k.inverse(), M);
  for (auto& x : kp) x = x * minv;
  for (auto& x : ki) x = x * minv;
  int rc = 0;
  if ((rc = upload(&c->rec_ginv, ginv)) || (rc = upload(&c->rec_kpow, kp)) || (rc = upload(&c->rec_kinv, ki)) ||
      (rc = upload(&c->rec_wpow, pow_table(fr_root(lm), M))))
    return rc;
  ZG_CK(cudaMalloc(&c->rec_zinv, M * sizeof(Fr)));
  ZG_CK(cudaMalloc(&c->rec_zw, M * sizeof(Fr)));
  ZG_CK(cudaMalloc(&c->rec_V, M * C * sizeof(Fr)));
  ZG_CK(cudaMalloc(&c->rec_W, R * C * sizeof(Fr)));
  ZG_CK(cudaMalloc(&c->rec_rows, 3 * R * C * 32));
  ZG_CK(cudaMalloc(&c->rec_raw, c->max_blob + 16));
  ZG_CK(cudaMalloc(&c->rec_ids, 3 * R * sizeof(uint32_t)));
  ZG_CK(cudaMalloc(&c->rec_erased, M * sizeof(uint16_t)));
  ZG_CK(cudaMalloc(&c->rec_err, sizeof(uint32_t)));
  ZG_CK(cudaMallocHost(&c->h_rec, std::max(3 * R * C * 32, c->max_blob + 16)));
  ZG_CK(cudaStreamCreateWithFlags(&c->rec_stream, cudaStreamNonBlocking));
  ZG_CK(cudaFuncSetAttribute(k_rec_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  ZG_CK(cudaFuncSetAttribute(k_rec_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  ZG_CK(cudaFuncSetAttribute(k_rec_out, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  c->rec_ready = true;
  return 0;
}

// ---------------------------------------------------------------------------
// Request pipeline (zg_submit / zg_wait / zg_encode_batch): continuous
// batching over units. A unit is a lane of up to FB_MAX_BLOBS blob slots,
// with its own stream, per-blob buffers and pinned staging. The issuer
// thread hands the waiting encode requests, in submission order, to a free
// unit, up to `fuse` at a time; the unit copies the payloads in, replays the
// CUDA graph of its fill level (every blob's RS extension, Merkle tree and
// digit sorts, one bucket accumulation and one combine over all their MSM
// items, every blob's trees and slices; the payload lengths are read from
// device memory) and copies the replies out, all on its stream. When every
// unit is busy and requests wait, the issuer creates another unit if the
// device's free memory covers it plus the reserve, up to max_units; else
// the request waits for a unit. The units' computes run one after another
// in issue order (each fills the GPU: 16 blobs computing side by side on 8
// units encoded 32 uneven blobs at 5.85 blobs/s against 6.29 for one blob
// at a time), and each unit's copies overlap the others' compute. Each unit
// has a completion thread that finishes its replies once its copies are
// done. Recovery requests go to a
// worker thread that runs zg_recover on the context's recovery stream,
// beside the encodes.
static_assert(ZG_MAX_FUSED_BLOBS == FB_MAX_BLOBS, "header and kernels agree on the fused blob count");

struct Request {
  zg_request req{};
  zg_reply* reply = nullptr;
  int status = 0;
  std::string error;
  bool done = false;
};

struct Unit {
  Lane lane;
  BlobBufs b[FB_MAX_BLOBS];
  uint8_t* h_stage[FB_MAX_BLOBS] = {};  // pinned payload staging for pageable callers
  uint8_t* h_small[FB_MAX_BLOBS] = {};  // pinned: [0,8) length, [8,200) coset commitments,
                                        // [200,296) roots, [296,328) file root
  cudaStream_t s = nullptr;
  cudaEvent_t ev_comp = nullptr;  // end of the unit's compute (the next unit's compute waits on it)
  cudaEvent_t ev_out = nullptr;
  // per fill level k + 1, the three phases of the encode (pre, accumulation,
  // post) as CUDA graphs
  cudaGraphExec_t graph[FB_MAX_BLOBS][3] = {};
  uint64_t gen[FB_MAX_BLOBS] = {};           // the context's tuning_gen at each capture
  std::vector<Request*> reqs;                // in flight (empty: free)
  bool issued = false;                       // its copies and launches are queued
  std::thread completer;
};

struct Engine {
  zg_ctx* c = nullptr;
  std::vector<std::unique_ptr<Unit>> units;
  std::mutex mu;  // queues, units' request lists, tickets
  std::condition_variable cv;
  std::deque<Request*> queue;   // encodes
  std::deque<Request*> rqueue;  // recoveries
  std::map<uint64_t, Request*> tickets;
  uint64_t next_ticket = 1;
  uint64_t in_flight = 0;
  bool stop = false, stop_units = false;
  bool use_graph = true;
  int fuse = FB_MAX_BLOBS;
  size_t max_units = 3, reserve = 4ull << 30;
  cudaEvent_t last_comp = nullptr;  // compute of the unit issued last (issuer thread only)
  std::thread issuer, recoverer;
};

void complete(Engine* e, Request* q, int status, const std::string& err) {
  std::lock_guard<std::mutex> g(e->mu);
  q->status = status;
  q->error = err;
  q->done = true;
  e->cv.notify_all();
}

void free_unit(Unit* u) {
  if (u->ev_out) cudaEventSynchronize(u->ev_out);
  for (auto& gk : u->graph)
    for (cudaGraphExec_t& g : gk)
      if (g) cudaGraphExecDestroy(g);
  for (int i = 0; i < FB_MAX_BLOBS; ++i) {
    BlobBufs& b = u->b[i];
    void* d[] = {b.raw, b.d_len, b.enc, b.tree, b.amt, b.slices, b.file_root};
    for (void* p : d) if (p) cudaFree(p);
    if (u->h_stage[i]) cudaFreeHost(u->h_stage[i]);
    if (u->h_small[i]) cudaFreeHost(u->h_small[i]);
  }
  free_lane(&u->lane);
  if (u->ev_comp) cudaEventDestroy(u->ev_comp);
  if (u->ev_out) cudaEventDestroy(u->ev_out);
  if (u->s) cudaStreamDestroy(u->s);
}

// device bytes of one unit: its lane plus the per-blob buffers
size_t unit_bytes(const zg_ctx* c, int cap) {
  const size_t per = (c->max_blob + 16) + 8 + 3 * c->N * 32 + c->tree_bytes + 3 * (4 * c->R - 2) * 64 +
                     3 * c->R * c->slice_size + 32;
  return lane_bytes(c, cap) + per * (size_t)cap;
}

// a new unit, when the free device memory covers it plus the reserve
Unit* make_unit(Engine* e) {
  zg_ctx* c = e->c;
  const int cap = c->fb ? e->fuse : 1;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b < unit_bytes(c, cap) + e->reserve) {
    cudaGetLastError();
    return nullptr;
  }
  std::unique_ptr<Unit> u(new Unit());
  const size_t N = c->N, R = c->R;
  bool ok = alloc_lane(c, &u->lane, cap) == 0;
  for (int i = 0; ok && i < cap; ++i) {
    BlobBufs& b = u->b[i];
    ok = cudaMalloc(&b.raw, c->max_blob + 16) == cudaSuccess && cudaMalloc(&b.d_len, 8) == cudaSuccess &&
         cudaMalloc(&b.enc, 3 * N * 32) == cudaSuccess && cudaMalloc(&b.tree, c->tree_bytes) == cudaSuccess &&
         cudaMalloc(&b.amt, 3 * (4 * R - 2) * 64) == cudaSuccess &&
         cudaMalloc(&b.slices, 3 * R * c->slice_size) == cudaSuccess && cudaMalloc(&b.file_root, 32) == cudaSuccess &&
         cudaMallocHost(&u->h_stage[i], c->max_blob + 16) == cudaSuccess &&
         cudaMallocHost(&u->h_small[i], 512) == cudaSuccess;
  }
  ok = ok && cudaStreamCreateWithFlags(&u->s, cudaStreamNonBlocking) == cudaSuccess &&
       cudaEventCreateWithFlags(&u->ev_comp, cudaEventDisableTiming) == cudaSuccess &&
       cudaEventCreateWithFlags(&u->ev_out, cudaEventDisableTiming | cudaEventBlockingSync) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    free_unit(u.get());
    return nullptr;
  }
  return u.release();
}

// the CUDA graphs of a unit filled with k blobs, one per phase (captured on
// first use and after a tuning change)
int unit_graph(Engine* e, Unit* u, int k) {
  zg_ctx* c = e->c;
  cudaGraphExec_t* gx = u->graph[k - 1];
  if (gx[0] && u->gen[k - 1] != c->tuning_gen) {
    for (int ph = 0; ph < 3; ++ph) {
      if (gx[ph]) cudaGraphExecDestroy(gx[ph]);
      gx[ph] = nullptr;
    }
  }
  if (gx[0] || !e->use_graph) return 0;
  cudaStream_t cs = nullptr;
  ZG_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  bool ok = true;
  for (int ph = 0; ph < 3 && ok; ++ph) {
    cudaGraph_t g = nullptr;
    cudaError_t err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    int rc = 0;
    if (err == cudaSuccess) {
      rc = encode_launches(c, u->lane, u->b, k, nullptr, true, cs, false, 1 << ph);
      err = cudaStreamEndCapture(cs, &g);
    }
    if (err == cudaSuccess && rc == 0) err = cudaGraphInstantiate(&gx[ph], g, 0);
    if (g) cudaGraphDestroy(g);
    ok = err == cudaSuccess && rc == 0;
  }
  u->gen[k - 1] = c->tuning_gen;
  cudaStreamDestroy(cs);
  if (!ok) {  // launch the kernels one by one instead
    cudaGetLastError();
    for (int ph = 0; ph < 3; ++ph) {
      if (gx[ph]) cudaGraphExecDestroy(gx[ph]);
      gx[ph] = nullptr;
    }
    e->use_graph = false;
  }
  return 0;
}

// copies in, the fused encode of the unit's requests, copies out; all on the
// unit's stream
int issue_unit(Engine* e, Unit* u) {
  zg_ctx* c = e->c;
  const int k = (int)u->reqs.size();
  size_t lens[FB_MAX_BLOBS] = {};
  const uint8_t* src[FB_MAX_BLOBS] = {};
  for (int i = 0; i < k; ++i) {
    Request* q = u->reqs[i];
    zg_reply* r = new zg_reply();
    q->reply = r;
    r->slice_size = c->slice_size;
    r->nslices = 3 * c->R;
    if (!(r->slices = (uint8_t*)pinned_get(r->nslices * r->slice_size)))
      return fail(ZG_ERR_CUDA, "cannot allocate pinned reply");
    if (q->req.require_data) {
      r->data_len = 3 * c->N * 32;
      if (!(r->data = (uint8_t*)pinned_get(r->data_len))) return fail(ZG_ERR_CUDA, "cannot allocate pinned reply");
    }
    lens[i] = q->req.len;
    src[i] = q->req.data;
    cudaPointerAttributes pa;
    if (lens[i] && (cudaPointerGetAttributes(&pa, src[i]) != cudaSuccess || pa.type != cudaMemoryTypeHost)) {
      cudaGetLastError();
      memcpy(u->h_stage[i], src[i], lens[i]);
      src[i] = u->h_stage[i];
    }
    const uint64_t len64 = lens[i];
    memcpy(u->h_small[i], &len64, 8);
  }
  ZG_CK(cudaSetDevice(c->device));
  int rc = 0;
  {
    std::lock_guard<std::mutex> g(c->mu);  // the tuning the graph captures
    rc = unit_graph(e, u, k);
  }
  if (rc) return rc;
  cudaStream_t s = u->s;
  for (int i = 0; i < k; ++i) {
    ZG_CK(cudaMemcpyAsync(u->b[i].d_len, u->h_small[i], 8, cudaMemcpyHostToDevice, s));
    if (lens[i]) ZG_CK(cudaMemcpyAsync(u->b[i].raw, src[i], lens[i], cudaMemcpyHostToDevice, s));
  }
  // The units' computes run one after another in issue order: each fills
  // the GPU, and side by side they only contend for SMs and L2. A unit's
  // copies overlap the others' compute. (Ordering only the accumulations and
  // letting the pre and post phases overlap other units gained 1 % on the
  // 32-blob batch and doubled the p99 latency at 3 and 6 requests/s.)
  if (e->last_comp) ZG_CK(cudaStreamWaitEvent(s, e->last_comp, 0));
  for (int ph = 0; ph < 3; ++ph) {
    if (u->graph[k - 1][ph]) {
      ZG_CK(cudaGraphLaunch(u->graph[k - 1][ph], s));
    } else {
      std::lock_guard<std::mutex> g(c->mu);
      if ((rc = encode_launches(c, u->lane, u->b, k, lens, false, s, false, 1 << ph))) return rc;
    }
  }
  ZG_CK(cudaEventRecord(u->ev_comp, s));
  e->last_comp = u->ev_comp;
  c->launches += launches_per_encode(c, k);
  for (int i = 0; i < k; ++i) {
    const BlobBufs& b = u->b[i];
    zg_reply* r = u->reqs[i]->reply;
    for (int cs = 0; cs < 3; ++cs)
      ZG_CK(cudaMemcpyAsync(u->h_small[i] + 8 + 64 * cs, b.amt + (size_t)cs * (4 * c->R - 2) * 64, 64,
                            cudaMemcpyDeviceToHost, s));
    ZG_CK(cudaMemcpyAsync(u->h_small[i] + 200, b.tree + c->tree_off[0], 96, cudaMemcpyDeviceToHost, s));
    ZG_CK(cudaMemcpyAsync(u->h_small[i] + 296, b.file_root, 32, cudaMemcpyDeviceToHost, s));
    ZG_CK(cudaMemcpyAsync(r->slices, b.slices, r->nslices * r->slice_size, cudaMemcpyDeviceToHost, s));
    if (r->data) ZG_CK(cudaMemcpyAsync(r->data, b.enc, r->data_len, cudaMemcpyDeviceToHost, s));
  }
  ZG_CK(cudaEventRecord(u->ev_out, s));
  return 0;
}

// after the unit's copy-out: the reply fields zg_encode fills
int finish_encode(Unit* u, int i) {
  zg_reply* r = u->reqs[i]->reply;
  const uint8_t* amt = u->h_small[i] + 8;
  if (memcmp(amt, amt + 64, 64) || memcmp(amt, amt + 128, 64))
    return fail(ZG_ERR_INTERNAL, "coset commitments differ");
  if (amt[63] & 0x40) {
    memset(r->commitment, 0, 64);
  } else {
    memcpy(r->commitment, amt, 64);
    r->commitment[63] &= 0x3f;
  }
  memcpy(r->roots, u->h_small[i] + 200, 96);
  memcpy(r->storage_root, u->h_small[i] + 296, 32);
  return 0;
}

void unit_completer(Engine* e, Unit* u) {
  cudaSetDevice(e->c->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(e->mu);
      e->cv.wait(lk, [&] { return e->stop_units || u->issued; });
      if (!u->issued) break;
    }
    const cudaError_t err = cudaEventSynchronize(u->ev_out);
    std::vector<Request*> reqs = u->reqs;
    std::vector<int> rcs(reqs.size(), 0);
    std::vector<std::string> msgs(reqs.size());
    for (size_t i = 0; i < reqs.size(); ++i) {
      rcs[i] = err != cudaSuccess ? fail(ZG_ERR_CUDA, std::string("encode: ") + cudaGetErrorString(err))
                                  : finish_encode(u, (int)i);
      if (rcs[i]) msgs[i] = g_err;
    }
    {
      std::lock_guard<std::mutex> g(e->mu);
      u->reqs.clear();
      u->issued = false;
      e->in_flight -= reqs.size();
    }
    for (size_t i = 0; i < reqs.size(); ++i) complete(e, reqs[i], rcs[i], msgs[i]);
  }
}

void issuer_loop(Engine* e) {
  zg_ctx* c = e->c;
  cudaSetDevice(c->device);
  for (;;) {
    Unit* u = nullptr;
    {
      std::unique_lock<std::mutex> lk(e->mu);
      e->cv.wait(lk, [&] { return e->stop || !e->queue.empty(); });
      if (e->queue.empty()) break;
      auto free_unit_of = [&]() -> Unit* {
        for (auto& x : e->units)
          if (x->reqs.empty()) return x.get();
        return nullptr;
      };
      u = free_unit_of();
      if (!u && e->units.size() < e->max_units) {
        lk.unlock();
        Unit* nu = make_unit(e);
        lk.lock();
        if (nu) {
          e->units.emplace_back(nu);
          e->c->pipe_stats.units++;
          nu->completer = std::thread(unit_completer, e, nu);
          u = nu;
        }
      }
      if (!u) {
        if (e->units.empty()) {  // not even one unit fits: fail the request
          Request* q = e->queue.front();
          e->queue.pop_front();
          lk.unlock();
          complete(e, q, fail(ZG_ERR_CUDA, "request pipeline: no device memory for a unit"), g_err);
          continue;
        }
        e->cv.wait(lk, [&] { return (u = free_unit_of()) != nullptr; });
      }
      const size_t k = std::min<size_t>((size_t)u->lane.cap, e->queue.size());
      for (size_t i = 0; i < k; ++i) {
        u->reqs.push_back(e->queue.front());
        e->queue.pop_front();
      }
      e->in_flight += k;
      c->pipe_stats.launches[k - 1]++;
      c->pipe_stats.max_in_flight = std::max<uint64_t>(c->pipe_stats.max_in_flight, e->in_flight);
    }
    const int rc = issue_unit(e, u);
    if (rc) {
      // whatever was queued for the unit must end before it is reused
      cudaStreamSynchronize(u->s);
      const std::string m = g_err;
      std::vector<Request*> reqs;
      {
        std::lock_guard<std::mutex> g(e->mu);
        reqs.swap(u->reqs);
        e->in_flight -= reqs.size();
      }
      for (Request* q : reqs) complete(e, q, rc, m);
    } else {
      std::lock_guard<std::mutex> g(e->mu);
      u->issued = true;
      e->cv.notify_all();
    }
  }
}

void recovery_loop(Engine* e) {
  zg_ctx* c = e->c;
  cudaSetDevice(c->device);
  for (;;) {
    Request* q = nullptr;
    {
      std::unique_lock<std::mutex> lk(e->mu);
      e->cv.wait(lk, [&] { return e->stop || !e->rqueue.empty(); });
      if (e->rqueue.empty()) break;
      q = e->rqueue.front();
      e->rqueue.pop_front();
    }
    zg_reply* r = new zg_reply();
    q->reply = r;
    r->payload.resize(c->max_raw);
    size_t out_len = 0;
    const int rc = zg_recover(c, q->req.row_ids, q->req.rows, q->req.row_lens, q->req.n_rows, r->payload.data(),
                              r->payload.size(), &out_len);
    if (rc == ZG_OK) r->payload.resize(out_len);
    {
      std::lock_guard<std::mutex> g(e->mu);
      c->pipe_stats.recoveries++;
    }
    complete(e, q, rc, rc ? g_err : std::string());
  }
}

int engine_start(zg_ctx* c) {
  std::lock_guard<std::mutex> g(c->eng_mu);
  if (c->eng) return 0;
  ZG_CK(cudaSetDevice(c->device));
  Engine* e = new Engine();
  e->c = c;
  const zg_pipeline_config& pc = c->pipe_cfg;
  e->fuse = pc.blobs_per_launch ? (int)std::min<uint32_t>(pc.blobs_per_launch, FB_MAX_BLOBS) : FB_MAX_BLOBS;
  e->max_units = pc.max_units ? std::min<size_t>(pc.max_units, 8) : 3;
  e->reserve = (pc.reserve_mib ? (size_t)pc.reserve_mib : 4096) << 20;
  c->pipe_stats.unit_bytes = unit_bytes(c, c->fb ? e->fuse : 1);
  e->issuer = std::thread(issuer_loop, e);
  e->recoverer = std::thread(recovery_loop, e);
  c->eng = e;
  return 0;
}

// Drains the queues and the units, then frees the pipeline. Requests nobody
// waited for are freed with their replies.
void engine_shutdown(Engine* e) {
  {
    std::lock_guard<std::mutex> g(e->mu);
    e->stop = true;
    e->cv.notify_all();
  }
  if (e->issuer.joinable()) e->issuer.join();
  if (e->recoverer.joinable()) e->recoverer.join();
  {
    std::unique_lock<std::mutex> lk(e->mu);
    e->cv.wait(lk, [&] { return e->in_flight == 0; });
    e->stop_units = true;
    e->cv.notify_all();
  }
  for (auto& u : e->units)
    if (u->completer.joinable()) u->completer.join();
  cudaSetDevice(e->c->device);
  for (auto& kv : e->tickets) {
    zg_reply_free(kv.second->reply);
    delete kv.second;
  }
  for (auto& u : e->units) free_unit(u.get());
  e->units.clear();
  e->c->eng = nullptr;
  delete e;
}

}  // namespace

namespace {
// ---------------------------------------------------------------------------
// Batched slice verification (zg_verify_slices): host side.

// G2 side of seeded params, built on first use: vanishes[d-1][k] =
// DFT_{w^-1}(coeff)[bitrev_d(k)] * G2 with coeff[0] = tau_c^(N - step), coeff[i] =
// tau_c^((i-1) step), step = N / 2^d (AMTParams::gen_vanishes,
// crates/amt/src/prove_params/generate.rs:234-263, on the coset-adjusted
// powers of from_pp :139-176); high_g2 = tau^(3N) * G2 (high_g2pp has one
// element, so the coset adjustment multiplies it by w^0).
void host_dft(std::vector<Fr>& a, const Fr& root) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; ++i) {  // bit reversal, then iterative DIT
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    Fr w = root;
    for (size_t k = len; k < n; k <<= 1) w = w.sqr();
    for (size_t i = 0; i < n; i += len) {
      Fr t = Fr::one();
      for (size_t k = 0; k < len / 2; ++k) {
        const Fr u = a[i + k], v = a[i + k + len / 2] * t;
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
        t = t * w;
      }
    }
  }
}

int ensure_g2(zg_ctx* c) {
  if (c->g2_ready) return 0;
  if (!c->seeded) return fail(ZG_ERR_PARAMS, "the context has no G2 params");
  const int ln = c->lr + c->lc;
  const size_t N = c->N;
  const Fr tau = tau_from_seed(c->tau_seed);
  std::vector<Fr> sc;  // canonical scalars: per coset the vanishes, then high_g2
  for (int cs = 0; cs < 3; ++cs) {
    const Fr tp = cs ? tau * coset_factor(ln, cs).inverse() : tau;
    for (int d = 1; d <= c->lr; ++d) {
      const size_t step = N >> d, sz = (size_t)1 << d;
      const Fr ts = tp.pow_u64(step);
      std::vector<Fr> coeff(sz);
      coeff[0] = tp.pow_u64(N - step);
      Fr x = Fr::one();
      for (size_t i = 1; i < sz; ++i) {
        coeff[i] = x;
        x = x * ts;
      }
      host_dft(coeff, fr_root(d).inverse());
      // enact = normalize + index_reverse (generate.rs:122-126)
      for (size_t k = 0; k < sz; ++k) sc.push_back(coeff[host_brev((uint32_t)k, d)].to_canonical());
    }
  }
  sc.push_back(tau.pow_u64((uint64_t)3 * N).to_canonical());
  const size_t n = sc.size();
  uint8_t* d_sc = nullptr;
  G2Aff* d_out = nullptr;
  ZG_CK(cudaMalloc(&d_sc, n * 32));
  ZG_CK(cudaMalloc(&d_out, n * sizeof(G2Aff)));
  ZG_CK(cudaMemcpy(d_sc, sc.data(), n * 32, cudaMemcpyHostToDevice));
  k_g2_mul<<<nblk(n, 64), 64, 0, c->stream>>>(d_sc, g2_generator(), d_out, (uint32_t)n);
  std::vector<G2Aff> out(n);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaMemcpy(out.data(), d_out, n * sizeof(G2Aff), cudaMemcpyDeviceToHost);
  cudaFree(d_sc);
  cudaFree(d_out);
  if (e != cudaSuccess) return fail(ZG_ERR_CUDA, std::string("G2 params: ") + cudaGetErrorString(e));
  const size_t per = 2 * c->R - 2;
  for (int cs = 0; cs < 3; ++cs) {
    c->vanish[cs].assign(out.begin() + cs * per, out.begin() + (cs + 1) * per);
    c->high_g2[cs] = out[n - 1];
  }
  c->g2_ready = true;
  return 0;
}

struct G1Pt {
  G1Aff p;
  uint8_t inf = 1;
};

// ark-serialize uncompressed G1 with validation (the point must be on
// y^2 = x^3 + 3; G1 has cofactor 1)
bool g1_from_ark(const uint8_t* b, G1Pt* out) {
  uint8_t fl = 0;
  Fq x, y;
  if (!field_from_le(b, &x) || !field_from_le(b + 32, &y, &fl)) return false;
  if (fl == 3) return false;
  if (fl == 1) {
    out->inf = 1;
    out->p.x = Fq::zero();
    out->p.y = Fq::zero();
    return true;
  }
  if (!(y * y == x * x * x + Fq::from_u32(3))) return false;
  out->inf = 0;
  out->p.x = x;
  out->p.y = y;
  return true;
}
// EncodeBlobReply.erasure_commitment: x || y as canonical field elements, the
// affine point at infinity as (0, 0) (grpc/src/service.rs:77-83)
bool g1_from_reply(const uint8_t* b, G1Pt* out) {
  bool zero = true;
  for (int i = 0; i < 64; ++i) zero &= b[i] == 0;
  out->inf = zero ? 1 : 0;
  out->p.x = Fq::zero();
  out->p.y = Fq::zero();
  return zero || (field_from_le(b, &out->p.x) && field_from_le(b + 32, &out->p.y));
}
bool g1_eq(const G1Pt& a, const G1Pt& b) { return a.inf == b.inf && (a.inf || (a.p.x == b.p.x && a.p.y == b.p.y)); }

uint64_t le_u64(const uint8_t* p) {
  uint64_t v = 0;
  for (int i = 0; i < 8; ++i) v |= (uint64_t)p[i] << (8 * i);
  return v;
}

// 32 little-endian bytes below r (a canonical Fr), without conversion
bool fr_canonical(const uint8_t* b) {
  const uint32_t r[8] = {FrCfg::p0, FrCfg::p1, FrCfg::p2, FrCfg::p3, FrCfg::p4, FrCfg::p5, FrCfg::p6, FrCfg::p7};
  for (int i = 7; i >= 0; --i) {
    const uint32_t w = (uint32_t)b[4 * i] | (uint32_t)b[4 * i + 1] << 8 | (uint32_t)b[4 * i + 2] << 16 |
                       (uint32_t)b[4 * i + 3] << 24;
    if (w != r[i]) return w < r[i];
  }
  return false;
}

// one deserialized EncodedSlice (the fields the checks read)
struct PSlice {
  const uint8_t* bytes = nullptr;
  size_t len = 0;
  uint64_t index = 0, amt_index = 0, row_index = 0, row_len = 0, leaf_index = 0, nmerkle = 0;
  G1Pt commitment, high;
  std::vector<G1Pt> comm, quot;
};

// CanonicalDeserialize of EncodedSlice (derive order, encoder/slice.rs:15-20):
// every length prefix bounded by the remaining bytes, field elements
// canonical, points on the curve, no trailing bytes.
bool parse_slice(const uint8_t* in, size_t len, PSlice* s) {
  const uint8_t* p = in;
  const uint8_t* end = in + len;
  auto left = [&]() { return (size_t)(end - p); };
  s->bytes = in;
  s->len = len;
  if (left() < 16 + 64 + 16) return false;
  s->index = le_u64(p);
  s->amt_index = le_u64(p + 8);
  if (!g1_from_ark(p + 16, &s->commitment)) return false;
  s->row_index = le_u64(p + 80);
  s->row_len = le_u64(p + 88);
  p += 96;
  if (s->row_len > left() / 32) return false;
  for (uint64_t i = 0; i < s->row_len; ++i, p += 32)
    if (!fr_canonical(p)) return false;
  if (left() < 8) return false;
  const uint64_t np = le_u64(p);
  p += 8;
  if (np > left() / 128) return false;
  s->comm.resize(np);
  s->quot.resize(np);
  for (uint64_t i = 0; i < np; ++i, p += 128)
    if (!g1_from_ark(p, &s->comm[i]) || !g1_from_ark(p + 64, &s->quot[i])) return false;
  if (left() < 64 + 96 + 8 || !g1_from_ark(p, &s->high)) return false;
  p += 64 + 96;
  const uint64_t nm = le_u64(p);
  p += 8;
  if (nm > left() / 32) return false;
  s->nmerkle = nm;
  p += 32 * nm;
  if (left() < 40) return false;
  s->leaf_index = le_u64(p);
  p += 40;
  return p == end;
}

// 128-bit coefficients (below r) of the random linear combinations. With
// os set, every coefficient is drawn from the kernel's CSPRNG (getrandom), so
// a batch that fails the checks passes a combination with probability at
// most 2^-128 (a nonzero degree-1 polynomial in a uniform 128-bit
// coefficient vanishes for at most one value of it). Otherwise they come from
// a SplitMix64 stream at a caller-given seed: reproducible, for tests, and
// not safe against slices built by someone who knows the seed.
struct Coeffs {
  uint64_t s = 0;
  bool os = false;
  bool failed = false;  // the OS generator did not answer
  void next(uint32_t w[4]) {
    if (os) {
      uint8_t* p = reinterpret_cast<uint8_t*>(w);
      size_t got = 0;
      while (got < 16) {
        const ssize_t k = getrandom(p + got, 16 - got, 0);
        if (k < 0) {
          if (errno == EINTR) continue;
          failed = true;
          memset(w, 0, 16);
          return;
        }
        got += (size_t)k;
      }
      return;
    }
    for (int k = 0; k < 2; ++k) {
      const uint64_t x = splitmix64(s);
      w[2 * k] = (uint32_t)x;
      w[2 * k + 1] = (uint32_t)(x >> 32);
    }
  }
};
Fr fr_of_words(const uint32_t w[4]) {
  Fr x = Fr::zero();
  for (int i = 0; i < 4; ++i) x.v[i] = w[i];
  return Fr::from_canonical(x);
}

// device scratch of one zg_verify_slices call
struct VerifyRun {
  zg_ctx* c = nullptr;
  cudaStream_t s = nullptr;
  const std::vector<PSlice>* sl = nullptr;
  G1Pt auth;
  uint8_t* d_slices = nullptr;  // slices of the batch, stride bytes apart
  uint64_t stride = 0;
  std::vector<uint32_t> dpos;   // slice index -> position in d_slices
  uint8_t* d_scal = nullptr;    // [3][N] canonical scalars of the MSM checks
  Coeffs rng{0};
  std::vector<void*> owned;
  template <class T>
  T* dev(size_t n) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, std::max<size_t>(n, 1) * sizeof(T), s) != cudaSuccess) return nullptr;
    owned.push_back(p);
    return static_cast<T*>(p);
  }
  void release() {
    for (void* p : owned) cudaFreeAsync(p, s);
    owned.clear();
  }
};

uint32_t slice_coset(const zg_ctx* c, const PSlice& p) { return (uint32_t)(p.amt_index / c->R); }
uint32_t slice_bi(const zg_ctx* c, const PSlice& p) { return host_brev((uint32_t)(p.row_index), c->lr); }

// MSM over every coset's basis line with the scalars in d_scal (cosets with
// present[c]); out[c] on the device
int verify_msms(VerifyRun& v, const bool present[3], XYZZ* out) {
  zg_ctx* c = v.c;
  const uint32_t R = (uint32_t)c->R;
  for (int cs = 0; cs < 3; ++cs) {
    if (!present[cs]) continue;
    k_fb_sort<<<dim3(R, 1), 256, fb_sort_smem_bytes(c->lc), v.s>>>(v.d_scal + (size_t)cs * c->N * 32, c->lane.fb_offs,
                                                                   c->lane.fb_ents, c->lr, c->lc, 0, 0);
    FbAccArgs fa;
    fa.tab = c->line_ptr(cs, c->lr);
    fa.offs = c->lane.fb_offs;
    fa.ents = c->lane.fb_ents;
    fa.outT = c->lane.fb_T;
    fa.outS = c->lane.fb_S;
    fa.ents32 = nullptr;
    fa.lr = c->lr;
    fa.lc = c->lc;
    fa.lines = 1;
    fa.l0 = 0;
    fa.Ltot = 1;
    fa.tabN = c->N;
    launch_fb_accum(c, c->lane, c->msm_product, single_acc_plan(fa, R), v.s);
    launch_fb_combine(c->lane, single_fb_plan(c->lr), v.s);
    k_sum_points<<<1, 256, 0, v.s>>>(c->lane.part, R, out + cs);
  }
  return check_launch();
}

// host side: a == b for XYZZ points
bool xyzz_eq(const XYZZ& a, const XYZZ& b) {
  XYZZ d = a;
  d.add(b.neg());
  return d.is_inf();
}

// One random linear combination over the AMT checks of `ids` (verify_params.rs:136-211):
// ok_msm: sum_i a_i (MSM_i + sum_d comm_id - commitment) == O;
// ok_pair: e(L, g2) prod e(-G, V) prod e(-H_c, high_g2_c) == 1.
int amt_batch(VerifyRun& v, const std::vector<uint32_t>& ids, bool* ok) {
  zg_ctx* c = v.c;
  const std::vector<PSlice>& sl = *v.sl;
  const int LR = c->lr;
  const size_t n = ids.size();
  const uint32_t per = (uint32_t)(2 * c->R - 2);
  // coefficients
  std::vector<uint32_t> alpha_w(4 * n), beta_w(4 * n * LR), gamma_w(4 * n);
  for (size_t j = 0; j < n; ++j) {
    v.rng.next(&alpha_w[4 * j]);
    for (int d = 0; d < LR; ++d) v.rng.next(&beta_w[4 * (j * LR + d)]);
    v.rng.next(&gamma_w[4 * j]);
  }
  if (v.rng.failed) return fail(ZG_ERR_INTERNAL, "getrandom failed: no coefficients for the batch checks");
  // MSM check scalars
  bool present[3] = {false, false, false};
  std::vector<uint32_t> h_pos(n), h_cos(n), h_bi(n);
  std::vector<Fr> h_alpha(n);
  Fr asum[3] = {Fr::zero(), Fr::zero(), Fr::zero()}, gsum[3] = {Fr::zero(), Fr::zero(), Fr::zero()};
  for (size_t j = 0; j < n; ++j) {
    const PSlice& p = sl[ids[j]];
    h_pos[j] = v.dpos[ids[j]];
    h_cos[j] = slice_coset(c, p);
    h_bi[j] = slice_bi(c, p);
    h_alpha[j] = fr_of_words(&alpha_w[4 * j]);
    present[h_cos[j]] = true;
    asum[h_cos[j]] = asum[h_cos[j]] + h_alpha[j];
    gsum[h_cos[j]] = gsum[h_cos[j]] + fr_of_words(&gamma_w[4 * j]);
  }
  uint32_t* d_pos = v.dev<uint32_t>(n);
  uint32_t* d_cos = v.dev<uint32_t>(n);
  uint32_t* d_bi = v.dev<uint32_t>(n);
  Fr* d_alpha = v.dev<Fr>(n);
  if (!d_pos || !d_cos || !d_bi || !d_alpha) return fail(ZG_ERR_CUDA, "verify: device allocation failed");
  ZG_CK(cudaMemcpyAsync(d_pos, h_pos.data(), 4 * n, cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_cos, h_cos.data(), 4 * n, cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_bi, h_bi.data(), 4 * n, cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_alpha, h_alpha.data(), n * sizeof(Fr), cudaMemcpyHostToDevice, v.s));
  for (int cs = 0; cs < 3; ++cs)
    if (present[cs]) ZG_CK(cudaMemsetAsync(v.d_scal + (size_t)cs * c->N * 32, 0, c->N * 32, v.s));
  k_verify_scalars<<<(unsigned)n, 256, 0, v.s>>>(v.d_slices, v.stride, d_pos, c->lc, d_cos, d_bi, d_alpha, v.d_scal,
                                                 c->N * 32);
  XYZZ* d_msm = v.dev<XYZZ>(3);
  if (!d_msm) return fail(ZG_ERR_CUDA, "verify: device allocation failed");
  int rc = verify_msms(v, present, d_msm);
  if (rc) return rc;
  // weighted G1 terms: [L: comm (beta), high (gamma)] [G: quot (beta), by group] [D: comm (alpha)]
  std::vector<uint32_t> gkey(n * LR);
  std::vector<uint32_t> gcount((size_t)3 * per, 0);
  for (size_t j = 0; j < n; ++j)
    for (int d = 0; d < LR; ++d) {
      const uint32_t vi = (h_bi[j] >> (LR - 1 - d)) ^ 1u;
      gkey[j * LR + d] = h_cos[j] * per + ((2u << d) - 2) + vi;
      ++gcount[gkey[j * LR + d]];
    }
  std::vector<uint32_t> gid((size_t)3 * per, UINT32_MAX), goff(1, 0);
  for (size_t k = 0; k < gid.size(); ++k)
    if (gcount[k]) {
      gid[k] = (uint32_t)goff.size() - 1;
      goff.push_back(goff.back() + gcount[k]);
    }
  const uint32_t ng = (uint32_t)goff.size() - 1;
  const size_t nL = n * (LR + 1), nG = n * LR, nD = n * LR, nt = nL + nG + nD;
  std::vector<G1Aff> tp(nt);
  std::vector<uint8_t> tinf(nt);
  std::vector<uint32_t> tsc(4 * nt);
  std::vector<uint32_t> fill(goff.begin(), goff.end() - 1);
  auto put = [&](size_t t, const G1Pt& q, const uint32_t* w) {
    tp[t] = q.p;
    tinf[t] = q.inf;
    for (int k = 0; k < 4; ++k) tsc[4 * t + k] = w[k];
  };
  for (size_t j = 0; j < n; ++j) {
    const PSlice& p = sl[ids[j]];
    for (int d = 0; d < LR; ++d) {
      put(j * (LR + 1) + d, p.comm[d], &beta_w[4 * (j * LR + d)]);
      put(nL + fill[gid[gkey[j * LR + d]]]++, p.quot[d], &beta_w[4 * (j * LR + d)]);
      put(nL + nG + j * LR + d, p.comm[d], &alpha_w[4 * j]);
    }
    put(j * (LR + 1) + LR, p.high, &gamma_w[4 * j]);
  }
  G1Aff* d_tp = v.dev<G1Aff>(nt);
  uint8_t* d_tinf = v.dev<uint8_t>(nt);
  uint32_t* d_tsc = v.dev<uint32_t>(4 * nt);
  XYZZ* d_terms = v.dev<XYZZ>(nt);
  uint32_t* d_goff = v.dev<uint32_t>(goff.size());
  // pairing inputs: [0] L, [1..ng] G_g, then H_c per present coset; extra: D sum, A, H scalars
  const uint32_t npair = 1 + ng + (present[0] + present[1] + present[2]);
  XYZZ* d_pin = v.dev<XYZZ>(npair + 2);  // + D sum, A = (sum alpha) commitment
  if (!d_tp || !d_tinf || !d_tsc || !d_terms || !d_goff || !d_pin) return fail(ZG_ERR_CUDA, "verify: allocation");
  ZG_CK(cudaMemcpyAsync(d_tp, tp.data(), nt * sizeof(G1Aff), cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_tinf, tinf.data(), nt, cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_tsc, tsc.data(), 16 * nt, cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_goff, goff.data(), 4 * goff.size(), cudaMemcpyHostToDevice, v.s));
  k_g1_mul_words<<<nblk(nt, 128), 128, 0, v.s>>>(d_tp, d_tinf, d_tsc, 4, d_terms, (uint32_t)nt);
  k_sum_points<<<1, 256, 0, v.s>>>(d_terms, (uint32_t)nL, d_pin);
  k_seg_sum<<<nblk(ng, 128), 128, 0, v.s>>>(d_terms + nL, d_goff, d_pin + 1, ng);
  k_sum_points<<<1, 256, 0, v.s>>>(d_terms + nL + nG, (uint32_t)nD, d_pin + npair);
  // full-size multiples of the commitment: H_c = (sum gamma over c) C, A = (sum alpha) C
  std::vector<uint32_t> big;
  std::vector<G1Aff> bigp;
  Fr atot = asum[0] + asum[1] + asum[2];
  for (int cs = 0; cs < 4; ++cs) {
    if (cs < 3 && !present[cs]) continue;
    const Fr k = (cs < 3 ? gsum[cs] : atot).to_canonical();
    big.insert(big.end(), k.v, k.v + 8);
    bigp.push_back(v.auth.p);
  }
  const uint32_t nb = (uint32_t)bigp.size();
  G1Aff* d_bp = v.dev<G1Aff>(nb);
  uint8_t* d_binf = v.dev<uint8_t>(nb);
  uint32_t* d_bsc = v.dev<uint32_t>(8 * nb);
  if (!d_bp || !d_binf || !d_bsc) return fail(ZG_ERR_CUDA, "verify: allocation");
  std::vector<uint8_t> binf(nb, v.auth.inf);
  ZG_CK(cudaMemcpyAsync(d_bp, bigp.data(), nb * sizeof(G1Aff), cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_binf, binf.data(), nb, cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_bsc, big.data(), 32 * nb, cudaMemcpyHostToDevice, v.s));
  // H_c land after the groups, A after the D sum
  k_g1_mul_words<<<1, 128, 0, v.s>>>(d_bp, d_binf, d_bsc, 8, d_pin + 1 + ng, nb - 1);
  k_g1_mul_words<<<1, 128, 0, v.s>>>(d_bp + nb - 1, d_binf + nb - 1, d_bsc + 8 * (nb - 1), 8, d_pin + npair + 1, 1);
  // MSM check on the host
  XYZZ hm[3], hd[2];
  ZG_CK(cudaMemcpyAsync(hm, d_msm, sizeof(hm), cudaMemcpyDeviceToHost, v.s));
  ZG_CK(cudaMemcpyAsync(hd, d_pin + npair, sizeof(hd), cudaMemcpyDeviceToHost, v.s));
  // pairing: Miller loops on the device
  std::vector<G2Aff> q(npair);
  std::vector<uint8_t> neg(npair, 1);
  q[0] = g2_generator();
  neg[0] = 0;
  for (size_t k = 0; k < gid.size(); ++k)
    if (gid[k] != UINT32_MAX) q[1 + gid[k]] = c->vanish[k / per][k % per];
  for (int cs = 0, h = 0; cs < 3; ++cs)
    if (present[cs]) q[1 + ng + h++] = c->high_g2[cs];
  G2Aff* d_q = v.dev<G2Aff>(npair);
  uint8_t* d_neg = v.dev<uint8_t>(npair);
  G1Aff* d_pa = v.dev<G1Aff>(npair);
  uint8_t* d_pinf = v.dev<uint8_t>(npair);
  Fq12* d_f = v.dev<Fq12>(npair);
  Fq12* d_part = v.dev<Fq12>(128);
  if (!d_q || !d_neg || !d_pa || !d_pinf || !d_f || !d_part) return fail(ZG_ERR_CUDA, "verify: allocation");
  ZG_CK(cudaMemcpyAsync(d_q, q.data(), npair * sizeof(G2Aff), cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_neg, neg.data(), npair, cudaMemcpyHostToDevice, v.s));
  k_pairing_inputs<<<nblk(npair, 128), 128, 0, v.s>>>(d_pin, d_neg, d_pa, d_pinf, npair);
  k_miller<<<nblk(npair, 64), 64, 0, v.s>>>(d_pa, d_pinf, d_q, d_f, npair);
  k_fq12_partial<<<1, 128, 0, v.s>>>(d_f, npair, d_part);
  std::vector<Fq12> part(128);
  ZG_CK(cudaMemcpyAsync(part.data(), d_part, 128 * sizeof(Fq12), cudaMemcpyDeviceToHost, v.s));
  if ((rc = check_launch())) return rc;
  ZG_CK(cudaStreamSynchronize(v.s));
  XYZZ left = XYZZ::inf();
  for (int cs = 0; cs < 3; ++cs)
    if (present[cs]) left.add(hm[cs]);
  left.add(hd[0]);
  const bool ok_msm = xyzz_eq(left, hd[1]);
  Fq12 f = Fq12::one();
  for (auto& x : part) f = f * x;
  const bool ok_pair = final_exp(f).is_one();
  *ok = ok_msm && ok_pair;
  return 0;
}

// host pairing equality e(a, b) == e(c, d)
bool host_pairing_eq(const G1Pt& a, const G2Aff& b, const G1Pt& cc, const G2Aff& d) {
  G1Aff cn = cc.p;
  cn.y = -cn.y;
  return final_exp(miller_tate(a.p, a.inf != 0, b) * miller_tate(cn, cc.inf != 0, d)).is_one();
}

// verify_amt_proof for one slice in the reference's order (KZG from the
// deepest layer, MSM consistency, low-degree test); sub / kzg d as the
// reference's AmtProofError
int amt_single(VerifyRun& v, uint32_t id, int* sub, int64_t* kzg_d) {
  zg_ctx* c = v.c;
  const PSlice& p = (*v.sl)[id];
  const uint32_t cs = slice_coset(c, p), bi = slice_bi(c, p);
  const int LR = c->lr;
  const uint32_t per = (uint32_t)(2 * c->R - 2);
  (void)per;
  for (int d = LR - 1; d >= 0; --d) {
    const uint32_t vi = (bi >> (LR - 1 - d)) ^ 1u;
    const G2Aff& V = c->vanish[cs][((2u << d) - 2) + vi];
    if (!host_pairing_eq(p.comm[d], g2_generator(), p.quot[d], V)) {
      *sub = 2;
      *kzg_d = d;
      return 0;
    }
  }
  // MSM consistency: sum_d comm_d + MSM(basis[bi C ..], data) == commitment
  bool present[3] = {false, false, false};
  present[cs] = true;
  uint32_t* d_pos = v.dev<uint32_t>(1);
  uint32_t* d_cos = v.dev<uint32_t>(1);
  uint32_t* d_bi = v.dev<uint32_t>(1);
  Fr* d_alpha = v.dev<Fr>(1);
  XYZZ* d_msm = v.dev<XYZZ>(3);
  if (!d_pos || !d_cos || !d_bi || !d_alpha || !d_msm) return fail(ZG_ERR_CUDA, "verify: allocation");
  const Fr one = Fr::one();
  ZG_CK(cudaMemcpyAsync(d_pos, &v.dpos[id], 4, cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_cos, &cs, 4, cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_bi, &bi, 4, cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemcpyAsync(d_alpha, &one, sizeof(Fr), cudaMemcpyHostToDevice, v.s));
  ZG_CK(cudaMemsetAsync(v.d_scal + (size_t)cs * c->N * 32, 0, c->N * 32, v.s));
  k_verify_scalars<<<1, 256, 0, v.s>>>(v.d_slices, v.stride, d_pos, c->lc, d_cos, d_bi, d_alpha, v.d_scal, c->N * 32);
  int rc = verify_msms(v, present, d_msm);
  if (rc) return rc;
  XYZZ m;
  ZG_CK(cudaMemcpyAsync(&m, d_msm + cs, sizeof(XYZZ), cudaMemcpyDeviceToHost, v.s));
  ZG_CK(cudaStreamSynchronize(v.s));
  for (int d = 0; d < LR; ++d)
    if (!p.comm[d].inf) m.add_affine(p.comm[d].p.x, p.comm[d].p.y);
  XYZZ com = XYZZ::inf();
  if (!v.auth.inf) com.add_affine(v.auth.p.x, v.auth.p.y);
  if (!xyzz_eq(m, com)) {
    *sub = 3;
    return 0;
  }
  if (!host_pairing_eq(p.high, g2_generator(), v.auth, c->high_g2[cs])) {
    *sub = 4;
    return 0;
  }
  *sub = -1;
  return 0;
}

// bisect a failing batch down to its failing slices
int amt_resolve(VerifyRun& v, const std::vector<uint32_t>& ids, std::vector<int>& sub, std::vector<int64_t>& kd) {
  if (ids.empty()) return 0;
  if (ids.size() == 1) {
    int s = -1;
    int64_t d = 0;
    int rc = amt_single(v, ids[0], &s, &d);
    sub[ids[0]] = s;
    kd[ids[0]] = d;
    return rc;
  }
  bool ok = false;
  int rc = amt_batch(v, ids, &ok);
  if (rc || ok) return rc;
  std::vector<uint32_t> a(ids.begin(), ids.begin() + ids.size() / 2), b(ids.begin() + ids.size() / 2, ids.end());
  if ((rc = amt_resolve(v, a, sub, kd))) return rc;
  return amt_resolve(v, b, sub, kd);
}

}  // namespace

extern "C" {

const char* zg_last_error(void) { return g_err.c_str(); }

int zg_ctx_create(const zg_config* cfg, zg_ctx** out) {
  if (!cfg || !out) return fail(ZG_ERR_INVALID_ARG, "null argument");
  if (cfg->log_row < 1 || cfg->log_col < 3 || cfg->log_row > 11 || cfg->log_col > 11)
    return fail(ZG_ERR_INVALID_ARG, "log_row must be in [1, 11] and log_col in [3, 11]");
  zg_ctx* c = new zg_ctx();
  *out = nullptr;
  c->device = cfg->device;
  c->lr = (int)cfg->log_row;
  c->lc = (int)cfg->log_col;
  c->L = c->lr + 2;
  c->R = size_t(1) << c->lr;
  c->C = size_t(1) << c->lc;
  c->N = c->R * c->C;
  c->max_blob = 31 * c->N;
  c->max_raw = c->max_blob - 4;
  int rc = 0;
  auto bail = [&](int code) {
    zg_ctx_destroy(c);
    return code;
  };
  if (cudaSetDevice(c->device) != cudaSuccess) return bail(fail(ZG_ERR_CUDA, "cudaSetDevice failed"));
  if ((rc = set_smem_limits())) return bail(rc);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(ZG_ERR_CUDA, "stream create failed"));
  if (cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventRecord(c->done, c->stream) != cudaSuccess)
    return bail(fail(ZG_ERR_CUDA, "event create failed"));
  if ((rc = make_twiddles(c->lr, c->lc, &c->tw))) return bail(rc);
  // MSM variant: fixed-base windows (tables of 24 multiples per param point)
  // unless 8-bit windows are requested or the tables do not fit
  const uint32_t wb = cfg->msm_window_bits;
  if (wb != 0 && wb != 8 && wb != (uint32_t)FB_BITS)
    return bail(fail(ZG_ERR_INVALID_ARG, "msm_window_bits must be 0, 8 or 11"));
  c->fb = (wb == 0 || wb == (uint32_t)FB_BITS) && c->lc <= 10;
  c->W = c->fb ? FB_WINDOWS : 1;
  if (c->fb && cudaMalloc(&c->tab, (size_t)3 * c->L * c->W * c->N * sizeof(G1Aff)) != cudaSuccess) {
    cudaGetLastError();
    if (wb == (uint32_t)FB_BITS) return bail(fail(ZG_ERR_CUDA, "cannot allocate fixed-base tables"));
    c->fb = false;
    c->W = 1;
    c->tab = nullptr;
  }
  if (!c->tab && cudaMalloc(&c->tab, (size_t)3 * c->L * c->N * sizeof(G1Aff)) != cudaSuccess)
    return bail(fail(ZG_ERR_CUDA, "cannot allocate params"));
  c->n_l0 = 0;
  c->n_lines = c->L;
  if (c->fb && wb == 0 && c->lc == 10) plan_wide_classes(c);
  if ((rc = alloc_blob_buffers(c))) return bail(rc);
  if (cfg->params_dir && cfg->params_dir[0]) rc = load_mont_params(c, cfg->params_dir);
  else {
    rc = build_seeded_params(c, cfg->tau_seed);
    c->seeded = true;
    c->tau_seed = cfg->tau_seed;
  }
  if (rc) return bail(rc);
  if (c->fb) {
    const uint64_t nl = (uint64_t)3 * c->L;
    k_fb_tables<<<nblk(nl * c->N, 128), 128, 0, c->stream>>>(c->tab, c->N, nl);
    for (const zg_ctx::WdClass& k : c->wd) launch_wd_tables(c, k, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
      return bail(fail(ZG_ERR_CUDA, "fixed-base table build failed"));
  }
  *out = c;
  return ZG_OK;
}

void zg_ctx_destroy(zg_ctx* c) {
  if (!c) return;
  if (c->eng) engine_shutdown(c->eng);
  cudaSetDevice(c->device);
  if (c->done) cudaEventSynchronize(c->done);  // work queued on caller streams
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_twiddles(&c->tw);
  void* rp[] = {c->rec_zw, c->rec_ginv, c->rec_kpow, c->rec_kinv, c->rec_wpow, c->rec_zinv, c->rec_V, c->rec_W,
                c->rec_rows, c->rec_raw, c->rec_ids, c->rec_erased, c->rec_err};
  for (void* p : rp) if (p) cudaFree(p);
  if (c->h_rec) cudaFreeHost(c->h_rec);
  if (c->rec_stream) cudaStreamDestroy(c->rec_stream);
  free_lane(&c->lane);
  void* ps[] = {c->tab, c->raw, c->enc, c->amt, c->tree, c->tree_off_d, c->slices, c->file_root};
  for (void* p : ps) if (p) cudaFree(p);
  for (zg_ctx::WdClass& k : c->wd)
    if (k.tab) cudaFree(k.tab);
  if (c->h_in) cudaFreeHost(c->h_in);
  for (cudaEvent_t e : c->ev) if (e) cudaEventDestroy(e);
  if (c->done) cudaEventDestroy(c->done);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int zg_encode_device(zg_ctx* c, const void* d_data, size_t len, void* stream, zg_device_blob* out) {
  if (!c || !out || (!d_data && len)) return fail(ZG_ERR_INVALID_ARG, "null argument");
  if (len > c->max_raw) {
    char m[128];
    snprintf(m, sizeof(m), "TooLargeBlob { actual: %zu, expected_max: %zu }", len, c->max_raw);
    return fail(ZG_ERR_TOO_LARGE_BLOB, m);
  }
  std::lock_guard<std::mutex> g(c->mu);
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(ZG_ERR_CUDA, "cudaSetDevice failed");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  int rc = encode_device_locked(c, (const uint8_t*)d_data, len, s);
  if (rc) return rc;
  out->encoded_data = c->enc;
  out->slices = c->slices;
  out->slice_size = c->slice_size;
  out->amt_outputs = c->amt;
  out->roots = c->tree + c->tree_off[0];
  out->file_root = c->file_root;
  return ZG_OK;
}

int zg_encode(zg_ctx* c, const uint8_t* data, size_t len, int require_data, zg_reply** out) {
  if (!c || !out || (!data && len)) return fail(ZG_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (len > c->max_raw) {  // RawData::try_from (crates/encoder/src/raw_data.rs:55-72)
    char m[128];
    snprintf(m, sizeof(m), "TooLargeBlob { actual: %zu, expected_max: %zu }", len, c->max_raw);
    return fail(ZG_ERR_TOO_LARGE_BLOB, m);
  }
  std::lock_guard<std::mutex> g(c->mu);
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(ZG_ERR_CUDA, "cudaSetDevice failed");
  cudaStream_t s = c->stream;
  zg_reply* r = new zg_reply();
  auto bail = [&](int code) {
    zg_reply_free(r);
    return code;
  };
  r->slice_size = c->slice_size;
  r->nslices = 3 * c->R;
  if (!(r->slices = (uint8_t*)pinned_get(r->nslices * r->slice_size)))
    return bail(fail(ZG_ERR_CUDA, "cannot allocate pinned reply"));
  if (require_data) {
    r->data_len = 3 * c->N * 32;
    if (!(r->data = (uint8_t*)pinned_get(r->data_len)))
      return bail(fail(ZG_ERR_CUDA, "cannot allocate pinned reply"));
  }
  // page-locked caller buffers are copied by DMA directly; pageable ones go
  // through the context's pinned staging buffer
  const uint8_t* src = data;
  cudaPointerAttributes pa;
  if (len && (cudaPointerGetAttributes(&pa, data) != cudaSuccess || pa.type != cudaMemoryTypeHost)) {
    cudaGetLastError();
    memcpy(c->h_in, data, len);
    src = c->h_in;
  }
  if (len && cudaMemcpyAsync(c->raw, src, len, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return bail(fail(ZG_ERR_CUDA, "H2D copy failed"));
  int rc = encode_device_locked(c, c->raw, len, s);
  if (rc) return bail(rc);
  uint8_t amt_roots[3][64];
  bool ok = true;
  for (int cs = 0; cs < 3 && ok; ++cs)
    ok = cudaMemcpyAsync(amt_roots[cs], c->amt + (size_t)cs * (4 * c->R - 2) * 64, 64, cudaMemcpyDeviceToHost, s) ==
         cudaSuccess;
  ok = ok && cudaMemcpyAsync(r->roots, c->tree + c->tree_off[0], 96, cudaMemcpyDeviceToHost, s) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(r->storage_root, c->file_root, 32, cudaMemcpyDeviceToHost, s) == cudaSuccess;
  ok = ok && cudaMemcpyAsync(r->slices, c->slices, r->nslices * r->slice_size, cudaMemcpyDeviceToHost, s) ==
             cudaSuccess;
  if (require_data)
    ok = ok && cudaMemcpyAsync(r->data, c->enc, r->data_len, cudaMemcpyDeviceToHost, s) == cudaSuccess;
  if (!ok) return bail(fail(ZG_ERR_CUDA, "D2H copy failed"));
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return bail(fail(ZG_ERR_CUDA, std::string("encode: ") + cudaGetErrorString(e)));
  // EncodedBlobAMT::assert_commitment_consistent (crates/encoder/src/amt/blob.rs:42-47)
  if (memcmp(amt_roots[0], amt_roots[1], 64) || memcmp(amt_roots[0], amt_roots[2], 64))
    return bail(fail(ZG_ERR_INTERNAL, "coset commitments differ"));
  // erasure_commitment = x || y canonical without flags (grpc/src/service.rs:77-83)
  if (amt_roots[0][63] & 0x40) {
    memset(r->commitment, 0, 64);
  } else {
    memcpy(r->commitment, amt_roots[0], 64);
    r->commitment[63] &= 0x3f;
  }
  *out = r;
  return ZG_OK;
}

int zg_submit(zg_ctx* c, const zg_request* req, uint64_t* ticket) {
  if (!c || !req || !ticket) return fail(ZG_ERR_INVALID_ARG, "null argument");
  if (req->kind == ZG_REQ_ENCODE) {
    if (!req->data && req->len) return fail(ZG_ERR_INVALID_ARG, "null payload");
    if (req->len > c->max_raw) {  // RawData::try_from (crates/encoder/src/raw_data.rs:55-72)
      char m[128];
      snprintf(m, sizeof(m), "TooLargeBlob { actual: %zu, expected_max: %zu }", req->len, c->max_raw);
      return fail(ZG_ERR_TOO_LARGE_BLOB, m);
    }
  } else if (req->kind == ZG_REQ_RECOVER) {
    if (req->n_rows && (!req->row_ids || !req->rows || !req->row_lens)) return fail(ZG_ERR_INVALID_ARG, "null rows");
  } else {
    return fail(ZG_ERR_INVALID_ARG, "unknown request kind");
  }
  int rc = engine_start(c);
  if (rc) return rc;
  Engine* e = c->eng;
  Request* q = new Request();
  q->req = *req;
  std::lock_guard<std::mutex> g(e->mu);
  *ticket = e->next_ticket++;
  e->tickets[*ticket] = q;
  (req->kind == ZG_REQ_RECOVER ? e->rqueue : e->queue).push_back(q);
  e->cv.notify_all();
  return ZG_OK;
}

int zg_ctx_set_pipeline(zg_ctx* c, const zg_pipeline_config* cfg) {
  if (!c || !cfg) return fail(ZG_ERR_INVALID_ARG, "null argument");
  if (cfg->blobs_per_launch > FB_MAX_BLOBS || cfg->max_units > 8)
    return fail(ZG_ERR_INVALID_ARG, "pipeline: blobs_per_launch <= ZG_MAX_FUSED_BLOBS, max_units <= 8");
  std::lock_guard<std::mutex> g(c->eng_mu);
  if (c->eng) engine_shutdown(c->eng);
  c->pipe_cfg = *cfg;
  return ZG_OK;
}

int zg_ctx_pipeline_stats(zg_ctx* c, zg_pipeline_stats* out) {
  if (!c || !out) return fail(ZG_ERR_INVALID_ARG, "null argument");
  Engine* e = c->eng;
  if (e) {
    std::lock_guard<std::mutex> g(e->mu);
    *out = c->pipe_stats;
  } else {
    *out = c->pipe_stats;
  }
  return ZG_OK;
}

int zg_wait(zg_ctx* c, uint64_t ticket, int64_t timeout_ms, zg_reply** out) {
  if (!c || !out) return fail(ZG_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  Engine* e = c->eng;
  if (!e) return fail(ZG_ERR_INVALID_ARG, "unknown ticket");
  std::unique_lock<std::mutex> lk(e->mu);
  auto it = e->tickets.find(ticket);
  if (it == e->tickets.end()) return fail(ZG_ERR_INVALID_ARG, "unknown ticket");
  Request* q = it->second;
  auto ready = [&] { return q->done; };
  if (timeout_ms < 0) {
    e->cv.wait(lk, ready);
  } else if (!e->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return fail(ZG_ERR_TIMEOUT, "request not finished");
  }
  e->tickets.erase(it);
  lk.unlock();
  const int status = q->status;
  if (status == ZG_OK) {
    *out = q->reply;
  } else {
    zg_reply_free(q->reply);
    fail(status, q->error);
  }
  delete q;
  return status;
}

int zg_encode_batch(zg_ctx* c, size_t n, const uint8_t* const* data, const size_t* lens, int require_data,
                    zg_reply** out) {
  if (!c || (n && (!data || !lens || !out))) return fail(ZG_ERR_INVALID_ARG, "null argument");
  for (size_t i = 0; i < n; ++i) {
    out[i] = nullptr;
    if (!data[i] && lens[i]) return fail(ZG_ERR_INVALID_ARG, "null payload");
    if (lens[i] > c->max_raw) {
      char m[160];
      snprintf(m, sizeof(m), "TooLargeBlob { actual: %zu, expected_max: %zu }", lens[i], c->max_raw);
      return fail(ZG_ERR_TOO_LARGE_BLOB, m);
    }
  }
  // all n requests enter the queue at once, so the pipeline sees them
  // together and fuses them into full units
  int first = engine_start(c);
  if (first) return first;
  std::string first_msg;
  std::vector<uint64_t> t(n);
  const size_t issued = n;
  {
    Engine* e = c->eng;
    std::lock_guard<std::mutex> g(e->mu);
    for (size_t i = 0; i < n; ++i) {
      Request* q = new Request();
      q->req.kind = ZG_REQ_ENCODE;
      q->req.data = data[i];
      q->req.len = lens[i];
      q->req.require_data = require_data;
      t[i] = e->next_ticket++;
      e->tickets[t[i]] = q;
      e->queue.push_back(q);
    }
    e->cv.notify_all();
  }
  for (size_t i = 0; i < issued; ++i) {
    int rc = zg_wait(c, t[i], -1, &out[i]);
    if (rc && first == ZG_OK) {
      first = rc;
      first_msg = g_err;
    }
  }
  if (first != ZG_OK) {
    for (size_t i = 0; i < n; ++i) {
      zg_reply_free(out[i]);
      out[i] = nullptr;
    }
    return fail(first, first_msg);
  }
  return ZG_OK;
}

const uint8_t* zg_reply_payload(const zg_reply* r, size_t* len) {
  if (len) *len = r ? r->payload.size() : 0;
  return r && !r->payload.empty() ? r->payload.data() : nullptr;
}

int zg_ctx_warmup(zg_ctx* c) {
  zg_reply* r = nullptr;
  int rc = zg_encode(c, nullptr, 0, 1, &r);
  zg_reply_free(r);
  return rc;
}

void zg_reply_free(zg_reply* r) {
  if (!r) return;
  pinned_put(r->slices, r->nslices * r->slice_size);
  pinned_put(r->data, r->data_len);
  delete r;
}
uint32_t zg_reply_version(const zg_reply* r) { return r->version; }
const uint8_t* zg_reply_erasure_commitment(const zg_reply* r, size_t* len) {
  if (len) *len = 64;
  return r->commitment;
}
const uint8_t* zg_reply_storage_root(const zg_reply* r, size_t* len) {
  if (len) *len = 32;
  return r->storage_root;
}
const uint8_t* zg_reply_encoded_data(const zg_reply* r, size_t* len) {
  if (len) *len = r->data_len;
  return r->data;
}
size_t zg_reply_num_slices(const zg_reply* r) { return r->nslices; }
const uint8_t* zg_reply_slice(const zg_reply* r, size_t index, size_t* len) {
  if (index >= r->nslices) {
    if (len) *len = 0;
    return nullptr;
  }
  if (len) *len = r->slice_size;
  return r->slices + index * r->slice_size;
}
const uint8_t* zg_reply_roots(const zg_reply* r, size_t* len) {
  if (len) *len = 96;
  return r->roots;
}

int zg_ctx_param_points(zg_ctx* c, int coset, int line, size_t first, size_t count, uint8_t* host_out,
                        size_t cap) {
  if (!c || coset < 0 || coset > 2 || line < 0 || line >= c->L || first > c->N || count > c->N - first)
    return fail(ZG_ERR_INVALID_ARG, "bad param range");
  size_t bytes = count * sizeof(G1Aff);
  if (cap < bytes) return fail(ZG_ERR_INVALID_ARG, "buffer too small");
  std::lock_guard<std::mutex> g(c->mu);
  ZG_CK(cudaSetDevice(c->device));
  ZG_CK(cudaMemcpy(host_out, c->line_ptr(coset, line) + first, bytes, cudaMemcpyDeviceToHost));
  return ZG_OK;
}

int zg_verify_slices(zg_ctx* c, const uint8_t* const* slices, const size_t* lens, size_t n, const uint8_t* commitment,
                     const uint8_t* storage_root, uint64_t seed, int32_t* codes, int64_t* details) {
  if (!c || !commitment || !storage_root || (n && (!slices || !lens || !codes)))
    return fail(ZG_ERR_INVALID_ARG, "null argument");
  if (!c->fb) return fail(ZG_ERR_INVALID_ARG, "zg_verify_slices needs the fixed-base tables (msm_window_bits 0 or 11)");
  std::lock_guard<std::mutex> g(c->mu);
  ZG_CK(cudaSetDevice(c->device));
  keep_pool_memory();
  int rc = ensure_g2(c);
  if (rc) return rc;
  const uint64_t R = c->R, C = c->C;
  std::vector<PSlice> sl(n);
  std::vector<int64_t> det(4 * n, 0);
  for (size_t i = 0; i < n; ++i) codes[i] = 0;
  VerifyRun v;
  v.c = c;
  v.s = c->stream;
  v.sl = &sl;
  v.rng.s = seed;
  v.rng.os = seed == 0;
  const bool auth_ok = g1_from_reply(commitment, &v.auth);
  // deserialization and the structural checks, in the reference's order
  // (EncodedSlice::verify, encoder/slice.rs:73-95; EncodedSliceAMT::verify,
  // amt/slice.rs:53-103; verify_amt_proof's length checks, verify_params.rs:147-160)
  std::vector<uint32_t> batch;
  size_t maxlen = 0;
  for (size_t i = 0; i < n; ++i) {
    int64_t* d = &det[4 * i];
    PSlice& p = sl[i];
    if (!auth_ok || !slices[i] || !parse_slice(slices[i], lens[i], &p)) { codes[i] = 30; continue; }
    const uint64_t coset = p.amt_index / R, local = p.amt_index % R;
    if (p.index != p.amt_index) { codes[i] = 1; d[1] = (int64_t)p.index; d[2] = (int64_t)p.amt_index; }
    else if (p.index != p.leaf_index) { codes[i] = 2; d[1] = (int64_t)p.index; d[2] = (int64_t)p.leaf_index; }
    else if (!g1_eq(p.commitment, v.auth)) codes[i] = 10;
    else if (p.row_len != C) { codes[i] = 11; d[1] = (int64_t)p.row_len; d[2] = (int64_t)C; }
    else if (p.amt_index >= 3 * R) { codes[i] = 12; d[1] = (int64_t)p.amt_index; d[2] = (int64_t)(3 * R); }
    else if (local != p.row_index) { codes[i] = 13; d[1] = (int64_t)coset; d[2] = (int64_t)local; d[3] = (int64_t)p.row_index; }
    else if (p.comm.size() != (size_t)c->lr) {
      // proof depth: batch = N >> depth must equal the row length
      codes[i] = 14;
      d[1] = (int64_t)coset;
      d[2] = (int64_t)p.row_index;
      const size_t depth = p.comm.size();
      d[0] = (depth >= 63 || (c->N >> depth) != C) ? 0 : 1;
    } else {
      batch.push_back((uint32_t)i);
      maxlen = std::max(maxlen, lens[i]);
    }
  }
  if (!batch.empty()) {
    const size_t nb = batch.size();
    v.stride = (maxlen + 15) & ~(size_t)15;
    v.dpos.assign(n, 0);
    uint8_t* stage = (uint8_t*)pinned_get(nb * v.stride);
    if (!stage) return fail(ZG_ERR_CUDA, "cannot allocate pinned staging");
    std::vector<uint32_t> nproof(nb);
    for (size_t j = 0; j < nb; ++j) {
      const uint32_t i = batch[j];
      v.dpos[i] = (uint32_t)j;
      memcpy(stage + j * v.stride, slices[i], lens[i]);
      nproof[j] = (uint32_t)sl[i].nmerkle;
    }
    v.d_slices = v.dev<uint8_t>(nb * v.stride);
    v.d_scal = v.dev<uint8_t>(3 * c->N * 32);
    uint32_t* d_np = v.dev<uint32_t>(nb);
    uint8_t* d_root = v.dev<uint8_t>(32);
    int32_t* d_mcode = v.dev<int32_t>(nb);
    rc = (!v.d_slices || !v.d_scal || !d_np || !d_root || !d_mcode) ? fail(ZG_ERR_CUDA, "verify: allocation") : 0;
    std::vector<int32_t> mcode(nb, 0);
    std::vector<int> sub(n, -1);
    std::vector<int64_t> kd(n, 0);
    if (!rc) {
      cudaStreamWaitEvent(v.s, c->done, 0);
      cudaMemcpyAsync(v.d_slices, stage, nb * v.stride, cudaMemcpyHostToDevice, v.s);
      cudaMemcpyAsync(d_np, nproof.data(), 4 * nb, cudaMemcpyHostToDevice, v.s);
      cudaMemcpyAsync(d_root, storage_root, 32, cudaMemcpyHostToDevice, v.s);
      k_verify_merkle<<<(unsigned)nb, 128, 0, v.s>>>(v.d_slices, v.stride, c->lr, c->lc, d_np, d_root, d_mcode);
      cudaMemcpyAsync(mcode.data(), d_mcode, 4 * nb, cudaMemcpyDeviceToHost, v.s);
      rc = check_launch();
    }
    // the AMT checks: one random linear combination per round, bisected down
    // to the failing slices when it fails. Slices naming the same (coset, row)
    // go to different rounds: their MSM scalars share one place of the
    // coset's scalar vector.
    std::vector<std::vector<uint32_t>> rounds;
    {
      std::map<uint64_t, uint32_t> seen;
      for (uint32_t i : batch) {
        const uint32_t k = seen[sl[i].amt_index]++;
        if (k >= rounds.size()) rounds.emplace_back();
        rounds[k].push_back(i);
      }
    }
    for (size_t r = 0; !rc && r < rounds.size(); ++r) {
      const std::vector<uint32_t>& ids = rounds[r];
      bool ok = false;
      rc = amt_batch(v, ids, &ok);
      if (!rc && !ok) {
        const size_t h = ids.size() / 2;
        std::vector<uint32_t> a(ids.begin(), ids.begin() + h), b(ids.begin() + h, ids.end());
        if (ids.size() == 1) rc = amt_resolve(v, ids, sub, kd);
        else if (!(rc = amt_resolve(v, a, sub, kd))) rc = amt_resolve(v, b, sub, kd);
      }
    }
    if (!rc) rc = cudaStreamSynchronize(v.s) == cudaSuccess ? 0 : fail(ZG_ERR_CUDA, "verify: stream failed");
    if (!rc) cudaEventRecord(c->done, v.s);
    v.release();
    cudaStreamSynchronize(v.s);
    pinned_put(stage, nb * v.stride);
    if (rc) return rc;
    for (size_t j = 0; j < nb; ++j) {
      const uint32_t i = batch[j];
      int64_t* d = &det[4 * i];
      if (sub[i] >= 0) {
        codes[i] = 14;
        d[0] = sub[i];
        d[1] = (int64_t)(sl[i].amt_index / R);
        d[2] = (int64_t)sl[i].row_index;
        d[3] = sub[i] == 2 ? kd[i] : 0;
      } else if (mcode[j]) {
        codes[i] = mcode[j];
        if (mcode[j] == 22) { d[1] = (int64_t)sl[i].leaf_index; d[2] = (int64_t)(3 * R); }
        if (mcode[j] == 23 || mcode[j] == 24) d[1] = (int64_t)sl[i].leaf_index;
      }
    }
  }
  if (details) memcpy(details, det.data(), det.size() * sizeof(int64_t));
  return ZG_OK;
}

int zg_ctx_get_tuning(zg_ctx* c, zg_tuning* out) {
  if (!c || !out) return fail(ZG_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> g(c->mu);
  memset(out, 0, sizeof(*out));
  out->msm_product = c->msm_product;
  out->msm_task = c->msm_task;
  out->msm_wide_classes = (uint32_t)c->wd_on;
  out->ntt_cols_per_cta = c->ntt_cpb;
  out->ntt_threads = c->ntt_threads;
  out->msm_wide_lines = (uint32_t)c->wide_lines();
  out->msm_wide_avail = (uint32_t)c->wd.size();
  return ZG_OK;
}

namespace {
const uint32_t kTaskSizes[ZG_MSM_TASK_SIZES] = {32, 48, 64, 96};
bool tuning_valid(const zg_ctx* c, const zg_tuning* t) {
  const uint32_t cpb = t->ntt_cols_per_cta, th = t->ntt_threads;
  bool task_ok = false;
  for (uint32_t x : kTaskSizes) task_ok = task_ok || t->msm_task == x;
  return t->msm_product < ZG_MSM_PRODUCTS && task_ok && t->msm_wide_classes <= c->wd.size() &&
         (cpb == 1 || cpb == 2 || cpb == 4) && (th == 128 || th == 256 || th == 512);
}
}  // namespace

int zg_ctx_set_tuning(zg_ctx* c, const zg_tuning* t) {
  if (!c || !t) return fail(ZG_ERR_INVALID_ARG, "null argument");
  if (!tuning_valid(c, t))
    return fail(ZG_ERR_INVALID_ARG,
                "tuning: msm_product < ZG_MSM_PRODUCTS, msm_task 32/48/64/96, msm_wide_classes <= msm_wide_avail, "
                "ntt_cols_per_cta 1/2/4, ntt_threads 128/256/512");
  std::lock_guard<std::mutex> g(c->mu);
  ZG_CK(cudaSetDevice(c->device));
  ZG_CK(cudaEventSynchronize(c->done));  // no launch with the old choices is in flight
  c->msm_product = t->msm_product;
  c->msm_task = t->msm_task;
  apply_wide_classes(c, (int)t->msm_wide_classes);
  c->ntt_cpb = t->ntt_cols_per_cta;
  c->ntt_threads = t->ntt_threads;
  ++c->tuning_gen;
  return ZG_OK;
}

int zg_ctx_autotune(zg_ctx* c, zg_tuning* out) {
  if (!c) return fail(ZG_ERR_INVALID_ARG, "null context");
  std::lock_guard<std::mutex> g(c->mu);
  ZG_CK(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  ZG_CK(cudaStreamWaitEvent(s, c->done, 0));
  zg_tuning t;
  memset(&t, 0, sizeof(t));
  for (float& x : t.wide_ms) x = -1.f;
  const uint32_t old_task = c->msm_task;
  const int old_wd = c->wd_on;
  // a full-size synthetic blob on the context's own buffers, with every wide
  // class in use: its encode leaves every digit sort in place for the
  // kernel samples below
  apply_wide_classes(c, (int)c->wd.size());
  const size_t len = c->max_raw;
  k_fill_payload<<<(unsigned)std::min<size_t>(nblk(len, 256), 4096), 256, 0, s>>>(c->raw, len, 0x5eedull);
  const BlobBufs cb = ctx_bufs(c);
  int rc = encode_launches(c, c->lane, &cb, 1, &len, false, s, false);
  if (rc) return rc;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ZG_CK(cudaEventCreate(&e0));
  ZG_CK(cudaEventCreate(&e1));
  auto timed = [&](const std::function<void()>& fn) -> float {
    fn();  // warm-up
    cudaEventRecord(e0, s);
    fn();
    cudaEventRecord(e1, s);
    float ms = -1.f;
    if (cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    return ms;
  };
  auto argmin = [](const float* v, int n, int dflt) {
    int b = dflt;
    for (int i = 0; i < n; ++i)
      if (v[i] > 0 && (v[b] <= 0 || v[i] < v[b])) b = i;
    return b;
  };
  // the default choice stays unless another is faster by more than 1 %
  // (the kinds and task sizes differ by a few percent, timing noise by less)
  auto pick = [&](const float* v, int n, int dflt) {
    const int b = argmin(v, n, dflt);
    return (v[dflt] > 0 && !(v[b] < 0.99f * v[dflt])) ? dflt : b;
  };
  uint32_t best_msm = c->msm_product, best_task = old_task;
  int best_wd = old_wd;
  if (c->fb) {
    // the whole blob MSM (digit sorts, bucket accumulation, combine) with the
    // first j wide classes, product kind `kind`
    auto full_msm = [&](uint32_t kind, int j) {
      const FbAccArgs f0 = blob_fb_args(c, c->lane);
      k_fb_sort<<<dim3((unsigned)c->R, 3), 256, fb_sort_smem_bytes(c->lc), s>>>(
          c->enc, const_cast<uint32_t*>(f0.offs), const_cast<uint16_t*>(f0.ents), c->lr, c->lc, 1, c->N);
      for (int k = 0; k < j; ++k)
        if (c->wd[k].sort_of == k)
          launch_wd_sort(c->wd[k].ulog, c->enc, lane_wd_offs(c, c->lane, k, 0), lane_wd_ents(c, c->lane, k, 0), c->lr,
                         c->lc, c->N, s);
      launch_fb_accum(c, c->lane, kind, blob_acc_plan(c, c->lane, 1), s);
      launch_fb_combine(c->lane, blob_fb_plan(c, 1), s);
    };
    const int all_wd = (int)c->wd.size();
    // 1. product kind and 2. task size: the whole MSM with every wide class,
    // each choice timed twice in round-robin order, the faster time kept
    // (a sample of items ranked the kinds within its noise: a kind 3 % slower
    // on the whole blob could win on the sample)
    c->msm_task = FB_TASK_DEFAULT;
    for (uint32_t k = 0; k < ZG_MSM_PRODUCTS; ++k) full_msm(k, all_wd);  // first launches (module loading)
    for (float& x : t.msm_ms) x = -1.f;
    for (int round = 0; round < 2; ++round)
      for (uint32_t k = 0; k < ZG_MSM_PRODUCTS; ++k) {
        const float ms = timed([&] { full_msm(k, all_wd); });
        if (ms > 0 && (t.msm_ms[k] <= 0 || ms < t.msm_ms[k])) t.msm_ms[k] = ms;
      }
    best_msm = (uint32_t)pick(t.msm_ms, ZG_MSM_PRODUCTS, ZG_MSM_PRODUCT_HYBRID);
    for (float& x : t.task_ms) x = -1.f;
    for (int round = 0; round < 2; ++round)
      for (int k = 0; k < ZG_MSM_TASK_SIZES; ++k) {
        c->msm_task = kTaskSizes[k];
        const float ms = timed([&] { full_msm(best_msm, all_wd); });
        if (ms > 0 && (t.task_ms[k] <= 0 || ms < t.task_ms[k])) t.task_ms[k] = ms;
      }
    best_task = kTaskSizes[pick(t.task_ms, ZG_MSM_TASK_SIZES, 2)];
    c->msm_task = best_task;
    // 3. window width per line: the first j wide classes, j = 0 .. all
    for (int j = 0; j <= all_wd; ++j) {
      apply_wide_classes(c, j);
      t.wide_ms[j] = timed([&] { full_msm(best_msm, j); });
    }
    best_wd = pick(t.wide_ms, all_wd + 1, all_wd);
  }
  apply_wide_classes(c, best_wd);
  const uint32_t cpbs[3] = {1, 2, 4}, ths[3] = {128, 256, 512};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      t.ntt_ms[3 * i + j] = timed([&] { launch_rs(c, c->lane, c->raw, len, nullptr, c->enc, cpbs[i], ths[j], s); });
  const int bn = argmin(t.ntt_ms, 9, 4);
  rc = check_launch();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    c->msm_task = old_task;
    apply_wide_classes(c, old_wd);
    return rc;
  }
  ZG_CK(cudaEventRecord(c->done, s));
  ZG_CK(cudaStreamSynchronize(s));
  c->msm_product = best_msm;
  c->msm_task = best_task;
  c->ntt_cpb = cpbs[bn / 3];
  c->ntt_threads = ths[bn % 3];
  ++c->tuning_gen;
  t.msm_product = best_msm;
  t.msm_task = best_task;
  t.msm_wide_classes = (uint32_t)c->wd_on;
  t.ntt_cols_per_cta = c->ntt_cpb;
  t.ntt_threads = c->ntt_threads;
  t.msm_wide_lines = (uint32_t)c->wide_lines();
  t.msm_wide_avail = (uint32_t)c->wd.size();
  if (out) *out = t;
  return ZG_OK;
}

int zg_ctx_set_profiling(zg_ctx* c, int enable) {
  if (!c) return fail(ZG_ERR_INVALID_ARG, "null context");
  std::lock_guard<std::mutex> g(c->mu);
  ZG_CK(cudaSetDevice(c->device));
  if (enable && !c->ev[0])
    for (cudaEvent_t& e : c->ev) ZG_CK(cudaEventCreate(&e));
  c->profiling = enable != 0;
  return ZG_OK;
}

int zg_ctx_phase_times(zg_ctx* c, float* ms, int n) {
  if (!c || !ms || !c->ev[0]) return fail(ZG_ERR_INVALID_ARG, "profiling not enabled");
  std::lock_guard<std::mutex> g(c->mu);
  ZG_CK(cudaSetDevice(c->device));
  ZG_CK(cudaEventSynchronize(c->ev[5]));
  for (int k = 0; k < 5 && k < n; ++k) ZG_CK(cudaEventElapsedTime(&ms[k], c->ev[k], c->ev[k + 1]));
  return ZG_OK;
}

uint64_t zg_ctx_launches(const zg_ctx* c) { return c ? c->launches.load() : 0; }

int zg_msm_chunks(const void* d_bases, const void* d_scalars, uint32_t lines, uint32_t log_nchunks,
                  uint32_t log_chunk, void* d_out, void* stream) {
  if (!d_bases || !d_scalars || !d_out || lines == 0 || log_chunk > 10 || log_nchunks > 20)
    return fail(ZG_ERR_INVALID_ARG, "bad msm arguments");
  int rc = set_smem_limits();
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t nch = size_t(1) << log_nchunks;
  const size_t count = (size_t)lines * nch;
  XYZZ *win = nullptr, *part = nullptr;
  keep_pool_memory();
  ZG_CK(cudaMallocAsync(&win, count * MSM_WINDOWS * sizeof(XYZZ), s));
  ZG_CK(cudaMallocAsync(&part, count * sizeof(XYZZ), s));
  MsmChunkArgs a;
  a.scalars = (const uint8_t*)d_scalars;
  a.bases = (const G1Aff*)d_bases;
  a.win = win;
  a.lr = (int)log_nchunks;
  a.lc = (int)log_chunk;
  a.lines = (int)lines;
  a.bitrev_rows = 0;
  a.scalar_coset_stride = 0;
  a.base_coset_stride = 0;
  a.base_line_stride = (uint64_t)nch << log_chunk;
  k_msm_chunks<<<dim3((unsigned)nch, 1), MSM_THREADS, msm_smem_bytes((int)log_chunk), s>>>(a);
  k_msm_combine<<<nblk(count, 64), 64, 0, s>>>(win, part, (uint32_t)count);
  k_serialize_nodes<<<nblk(count, 128), 128, 0, s>>>(part, (uint8_t*)d_out, (uint32_t)count);
  rc = check_launch();
  cudaFreeAsync(win, s);
  cudaFreeAsync(part, s);
  return rc;
}

// Allocation-free twin of zg_msm_chunks: same kernels, with the scratch in
// g_noalloc_scratch. Host code must not hand the array's name to a kernel (on
// the host it names a stand-in, not device memory), so its device address is
// looked up with cudaGetSymbolAddress, with the call's device current, on
// every call: the lookup is cheap once the module is loaded, and an address
// cached across a cudaDeviceReset would point into the freed old module. The
// first call on a device loads the module there and should come before any
// stream capture.
int zg_msm_chunks_noalloc(const void* d_bases, const void* d_scalars, uint32_t lines, uint32_t log_nchunks,
                          uint32_t log_chunk, void* d_out, void* stream) {
  if (!d_bases || !d_scalars || !d_out || lines == 0 || log_chunk > 10 || log_nchunks > 20)
    return fail(ZG_ERR_INVALID_ARG, "bad msm arguments");
  const uint64_t count = (uint64_t)lines << log_nchunks;
  if (count > ZG_NOALLOC_MAX_MSMS) {
    char m[160];
    snprintf(m, sizeof(m), "zg_msm_chunks_noalloc: lines * 2^log_nchunks = %llu exceeds the static scratch limit %u",
             (unsigned long long)count, ZG_NOALLOC_MAX_MSMS);
    return fail(ZG_ERR_INVALID_ARG, m);
  }
  void* scratch = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
  if (e != cudaSuccess || !scratch)
    return fail(ZG_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
  int rc = set_smem_limits();
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  XYZZ* win = reinterpret_cast<XYZZ*>(scratch);
  XYZZ* part = win + count * MSM_WINDOWS;
  MsmChunkArgs a;
  a.scalars = (const uint8_t*)d_scalars;
  a.bases = (const G1Aff*)d_bases;
  a.win = win;
  a.lr = (int)log_nchunks;
  a.lc = (int)log_chunk;
  a.lines = (int)lines;
  a.bitrev_rows = 0;
  a.scalar_coset_stride = 0;
  a.base_coset_stride = 0;
  a.base_line_stride = (uint64_t)1 << (log_nchunks + log_chunk);
  k_msm_chunks<<<dim3(1u << log_nchunks, 1), MSM_THREADS, msm_smem_bytes((int)log_chunk), s>>>(a);
  k_msm_combine<<<nblk(count, 64), 64, 0, s>>>(win, part, (uint32_t)count);
  k_serialize_nodes<<<nblk(count, 128), 128, 0, s>>>(part, (uint8_t*)d_out, (uint32_t)count);
  return check_launch();
}

int zg_recover(zg_ctx* c, const uint64_t* row_ids, const uint8_t* const* rows, const size_t* row_lens, size_t n,
               uint8_t* out, size_t out_cap, size_t* out_len) {
  if (!c || (n && (!row_ids || !rows || !row_lens)) || !out_len) return fail(ZG_ERR_INVALID_ARG, "null argument");
  const size_t R = c->R, C = c->C, M = 4 * R;
  const int lr = c->lr, lc = c->lc, lm = lr + 2;
  // raw_slice_to_line drops rows of the wrong length; a map keeps one row per id
  std::map<uint64_t, const uint8_t*> valid;
  for (size_t i = 0; i < n; ++i)
    if (row_lens[i] == 32 * C) valid[row_ids[i]] = rows[i];
  // The reference converts every row (and panics on a value >= r) before it
  // counts them, so a non-canonical row outranks the two input errors. On the
  // good path the rows are checked on the device.
  auto any_noncanonical = [&]() {
    for (auto& kv : valid)
      for (size_t j = 0; j < C; ++j) {
        Fr x, d;
        memcpy(x.v, kv.second + 32 * j, 32);
        if (!Fr::sub_raw(d, x, Fr::modulus())) return true;
      }
    return false;
  };
  const char* input_err = nullptr;
  if (valid.size() < R)
    input_err = "Not enough valid lines";
  else if (valid.rbegin()->first >= 3 * R)
    input_err = "Cannot recover data: RowIdOverflow";
  if (input_err) {
    if (any_noncanonical()) return fail(ZG_ERR_RECOVERY, "Non-canonical field element in slice");
    return fail(ZG_ERR_RECOVERY, input_err);
  }
  // recovery has its own buffers and stream: it runs beside encodes
  std::lock_guard<std::mutex> g(c->rec_mu);
  ZG_CK(cudaSetDevice(c->device));
  int rc = rec_setup(c);
  if (rc) return rc;
  cudaStream_t s = c->rec_stream;
  // received rows -> pinned staging -> device; erased domain points (incl. the virtual coset)
  std::vector<uint32_t> ids;
  std::vector<uint8_t> known(M, 0);
  size_t k = 0;
  for (auto& kv : valid) {
    memcpy(c->h_rec + k * 32 * C, kv.second, 32 * C);
    ids.push_back((uint32_t)kv.first);
    const uint32_t cs = (uint32_t)(kv.first >> lr), r = (uint32_t)(kv.first & (R - 1));
    known[4 * r + (cs == 1 ? 2 : (cs == 2 ? 1 : cs))] = 1;
    ++k;
  }
  std::vector<uint16_t> erased;
  for (size_t i = 0; i < M; ++i)
    if (!known[i]) erased.push_back((uint16_t)i);
  ZG_CK(cudaMemcpyAsync(c->rec_rows, c->h_rec, k * 32 * C, cudaMemcpyHostToDevice, s));
  ZG_CK(cudaMemcpyAsync(c->rec_ids, ids.data(), k * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  ZG_CK(cudaMemcpyAsync(c->rec_erased, erased.data(), erased.size() * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
  ZG_CK(cudaMemsetAsync(c->rec_V, 0, M * C * sizeof(Fr), s));
  ZG_CK(cudaMemsetAsync(c->rec_err, 0, sizeof(uint32_t), s));
  const Twiddles* tm = cached_twiddles(0, lm);
  if (!tm) return ZG_ERR_CUDA;
  k_rec_rows<<<(unsigned)k, 256, C * sizeof(Fr), s>>>(c->rec_rows, c->rec_ids, c->rec_V, lr, lc, c->tw.twi_c,
                                                       c->rec_ginv, c->tw.wni_lo, c->tw.wni_hi, c->rec_err);
  k_rec_zinv<<<nblk(M, 128), 128, 0, s>>>(c->rec_erased, (uint32_t)erased.size(), c->rec_wpow, host_fr_from_u32(5),
                                          c->rec_zw, c->rec_zinv, (uint32_t)M);
  k_rec_cols<<<(unsigned)C, 256, (M + R) * sizeof(Fr), s>>>(c->rec_V, c->rec_W, lr, lc, tm->twf_c, tm->twi_c,
                                                             c->rec_kpow, c->rec_kinv, c->rec_zw, c->rec_zinv, c->tw.twf_r,
                                                             c->tw.wn_lo, c->tw.wn_hi, c->rec_err);
  k_rec_out<<<(unsigned)R, 256, C * sizeof(Fr), s>>>(c->rec_W, c->rec_raw, lc, c->tw.twf_c, c->rec_err);
  if ((rc = check_launch())) return rc;
  uint32_t err = 0;
  ZG_CK(cudaMemcpyAsync(&err, c->rec_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  ZG_CK(cudaMemcpyAsync(c->h_rec, c->rec_raw, c->max_blob, cudaMemcpyDeviceToHost, s));
  ZG_CK(cudaStreamSynchronize(s));
  // the reference panics on these two (from_bigint(...).unwrap(), the degree assert)
  if (err & 1) return fail(ZG_ERR_RECOVERY, "Non-canonical field element in slice");
  if (err & 2) return fail(ZG_ERR_RECOVERY, "Inconsistent rows (degree check)");
  // RawBlob -> RawData (crates/encoder/src/raw_blob.rs:42-58, raw_data.rs:25-38)
  if (err & 4) return fail(ZG_ERR_RECOVERY, "Incorrect scalar");
  uint32_t l32;
  memcpy(&l32, c->h_rec + c->max_raw, 4);
  if (l32 > c->max_raw) return fail(ZG_ERR_RECOVERY, "Incorrect length field");
  for (size_t i = l32; i < c->max_raw; ++i)
    if (c->h_rec[i]) return fail(ZG_ERR_RECOVERY, "Non zero in padding range");
  if (out_cap < l32) return fail(ZG_ERR_INVALID_ARG, "output buffer too small");
  memcpy(out, c->h_rec, l32);
  *out_len = l32;
  return ZG_OK;
}

int zg_ctx_msm(zg_ctx* c, uint32_t coset, uint32_t line, const void* d_scalars, size_t n, void* d_out, void* stream) {
  if (!c || !d_scalars || !d_out) return fail(ZG_ERR_INVALID_ARG, "null argument");
  if (!c->fb) return fail(ZG_ERR_INVALID_ARG, "zg_ctx_msm needs the fixed-base tables (msm_window_bits 0 or 11)");
  if (coset >= 3 || line >= (uint32_t)c->L) return fail(ZG_ERR_INVALID_ARG, "coset or line out of range");
  if (n < c->C || n > c->N || (n & (n - 1))) return fail(ZG_ERR_INVALID_ARG, "n must be a power of two in [2^log_col, N]");
  // work items = chunks of 2^lcs points: 1024-point chunks leave most SMs
  // idle below 2^19 points (one CTA per item), so chunks shrink down to 128
  // points until there are 512 items, as far as the context's chunk buffers
  // (3 R chunks) allow; the tables are per point, so any chunking reads them
  int logn = 0;
  while (((size_t)1 << logn) < n) ++logn;
  int lcs = c->lc;
  while (lcs > 7 && (n >> lcs) < 512 && (n >> (lcs - 1)) <= 3 * c->R) --lcs;
  const int lrn = logn - lcs;
  const uint32_t nch = 1u << lrn;
  std::lock_guard<std::mutex> g(c->mu);
  ZG_CK(cudaSetDevice(c->device));
  cudaStream_t s = (cudaStream_t)stream;
  ZG_CK(cudaStreamWaitEvent(s, c->done, 0));
  k_fb_sort<<<dim3(nch, 1), 256, fb_sort_smem_bytes(lcs), s>>>((const uint8_t*)d_scalars, c->lane.fb_offs, c->lane.fb_ents,
                                                                lrn, lcs, 0, 0);
  FbAccArgs fa;
  fa.tab = c->line_ptr((int)coset, (int)line);
  fa.offs = c->lane.fb_offs;
  fa.ents = c->lane.fb_ents;
  fa.outT = c->lane.fb_T;
  fa.outS = c->lane.fb_S;
  fa.ents32 = nullptr;
  fa.lr = lrn;
  fa.lc = lcs;
  fa.lines = 1;
  fa.l0 = 0;
  fa.Ltot = 1;
  fa.tabN = c->N;
  launch_fb_accum(c, c->lane, c->msm_product, single_acc_plan(fa, nch), s);
  launch_fb_combine(c->lane, single_fb_plan(lrn), s);
  k_sum_points<<<1, 256, 0, s>>>(c->lane.part, nch, c->lane.nodes);
  k_serialize_nodes<<<1, 128, 0, s>>>(c->lane.nodes, (uint8_t*)d_out, 1);
  c->launches += 5;
  ZG_CK(cudaEventRecord(c->done, s));
  return check_launch();
}

// ---- LightEncodedSlice (crates/encoder/src/encoder/light_slice.rs:11-79):
// the ark-serialized slice without its row. Both layouts are fixed-offset:
//   EncodedSlice: index | amt.index | commitment | row.index | (len, row) |
//                 (len, proof pairs) | high | roots | (len, path) | merkle.index | leaf
//   Light:        index | commitment | (len, proof pairs) | high | roots | (len, path) | leaf
namespace {
struct SliceLayout {
  size_t C, lr, row, proof, high, roots, path, midx, leaf, size, light_size;
  SliceLayout(uint32_t log_row, uint32_t log_col) {
    C = size_t(1) << log_col;
    lr = log_row;
    row = 88;
    proof = 96 + 32 * C;
    high = proof + 8 + 128 * lr;
    roots = high + 64;
    path = roots + 96;
    midx = path + 8 + 32 * lr;
    leaf = midx + 8;
    size = leaf + 32;
    light_size = 8 + 64 + (8 + 128 * lr) + 64 + 96 + (8 + 32 * lr) + 32;
  }
};
uint64_t get_u64(const uint8_t* p) {
  uint64_t v;
  memcpy(&v, p, 8);
  return v;
}
}  // namespace

int zg_light_slice_from_slice(const uint8_t* slice, size_t len, uint32_t log_row, uint32_t log_col, uint8_t* out,
                              size_t cap, size_t* out_len) {
  if (!slice || !out || !out_len || log_row < 1 || log_row > 20 || log_col > 20)
    return fail(ZG_ERR_INVALID_ARG, "bad arguments");
  const SliceLayout L(log_row, log_col);
  if (len != L.size) return fail(ZG_ERR_INVALID_ARG, "slice length does not match the blob shape");
  if (get_u64(slice + L.row) != L.C || get_u64(slice + L.proof) != L.lr || get_u64(slice + L.path) != L.lr)
    return fail(ZG_ERR_INVALID_ARG, "slice vector lengths do not match the blob shape");
  const uint64_t index = get_u64(slice);
  char m[160];
  // EncodedSlice::check_amt_idx / check_merkle_idx (slice.rs:41-71), unwrapped by from_slice
  if (get_u64(slice + 8) != index) {
    snprintf(m, sizeof(m), "UnmatchedAMTIndex { row_index: %llu, amt_index: %llu }", (unsigned long long)index,
             (unsigned long long)get_u64(slice + 8));
    return fail(ZG_ERR_INVALID_ARG, m);
  }
  if (get_u64(slice + L.midx) != index) {
    snprintf(m, sizeof(m), "UnmatchedMerkleIndex { row_index: %llu, merkle_index: %llu }",
             (unsigned long long)index, (unsigned long long)get_u64(slice + L.midx));
    return fail(ZG_ERR_INVALID_ARG, m);
  }
  if (cap < L.light_size) return fail(ZG_ERR_INVALID_ARG, "output buffer too small");
  uint8_t* o = out;
  memcpy(o, slice, 8), o += 8;
  memcpy(o, slice + 16, 64), o += 64;
  memcpy(o, slice + L.proof, L.roots - L.proof), o += L.roots - L.proof;  // proof pairs, high
  memcpy(o, slice + L.roots, L.midx - L.roots), o += L.midx - L.roots;    // roots, path
  memcpy(o, slice + L.leaf, 32), o += 32;
  *out_len = L.light_size;
  return ZG_OK;
}

int zg_light_slice_into_slice(const uint8_t* light, size_t len, const uint8_t* row, size_t row_len,
                              uint32_t log_row, uint32_t log_col, uint8_t* out, size_t cap, size_t* out_len) {
  if (!light || !row || !out || !out_len || log_row < 1 || log_row > 20 || log_col > 20)
    return fail(ZG_ERR_INVALID_ARG, "bad arguments");
  const SliceLayout L(log_row, log_col);
  if (len != L.light_size) return fail(ZG_ERR_INVALID_ARG, "light slice length does not match the blob shape");
  if (row_len != 32 * L.C) return fail(ZG_ERR_INVALID_ARG, "row length does not match the blob shape");
  if (cap < L.size) return fail(ZG_ERR_INVALID_ARG, "output buffer too small");
  const uint64_t index = get_u64(light);
  const uint64_t R = uint64_t(1) << log_row;
  const uint8_t* proof = light + 72;
  const size_t proof_bytes = L.roots - L.proof;  // (len, pairs) and high
  const uint8_t* roots = proof + proof_bytes;
  const size_t roots_bytes = L.midx - L.roots;   // roots and (len, path)
  const uint8_t* leaf = roots + roots_bytes;
  uint8_t* o = out;
  auto put = [&](uint64_t v) { memcpy(o, &v, 8), o += 8; };
  put(index);
  put(index);                   // EncodedSliceAMT::new(self.index, ...)
  memcpy(o, light + 8, 64), o += 64;
  put(index % R);               // BlobRow.index
  put(L.C);
  memcpy(o, row, 32 * L.C), o += 32 * L.C;
  memcpy(o, proof, proof_bytes), o += proof_bytes;
  memcpy(o, roots, roots_bytes), o += roots_bytes;
  put(index);                   // EncodedSliceMerkle::new(..., self.index, ...)
  memcpy(o, leaf, 32), o += 32;
  *out_len = L.size;
  return ZG_OK;
}

int zg_ntt(void* d_data, uint32_t log_n, uint32_t batch, int inverse, uint32_t coset_idx, void* stream) {
  if (!d_data || log_n < 1 || log_n > 22 || batch == 0) return fail(ZG_ERR_INVALID_ARG, "bad ntt arguments");
  if (coset_idx && inverse) return fail(ZG_ERR_INVALID_ARG, "coset shift is forward-only");
  int rc = set_smem_limits();
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  ZG_CK(cudaFuncSetAttribute(k_ntt_small, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  const size_t n = size_t(1) << log_n;
  Fr* v = (Fr*)d_data;
  const CosetPows* cp = nullptr;
  if (coset_idx && !(cp = cached_coset_pows((int)log_n, coset_idx))) return fail(ZG_ERR_CUDA, "coset table alloc failed");
  const Fr ninv = host_fr_from_u32((uint32_t)n).inverse();
  // the transforms run on the canonical values directly (linear passes with
  // Montgomery-form twiddles keep canonical values canonical); the coset
  // shift and the inverse's 1/n are products in the transforms' first loads
  // and last stores
  if (log_n <= 11) {
    const Twiddles* tw = cached_twiddles(0, (int)log_n);
    if (!tw) return ZG_ERR_CUDA;
    for (uint32_t b0 = 0; b0 < batch;) {
      uint32_t nb = std::min<uint32_t>(batch - b0, 65535);
      k_ntt_small<<<nb, ntt_threads((int)log_n), n * sizeof(Fr), s>>>(
          v + (size_t)b0 * n, (int)log_n, inverse ? tw->twi_c : tw->twf_c, cp ? cp->lo : nullptr, inverse, ninv);
      b0 += nb;
    }
  } else {
    const int lc = (int)(log_n + 1) / 2, lr = (int)log_n - lc;
    const Twiddles* tw = cached_twiddles(lr, lc);
    if (!tw) return ZG_ERR_CUDA;
    const uint32_t per = std::min<uint32_t>(batch, 65535);
    keep_pool_memory();
    Fr* tmp = nullptr;
    ZG_CK(cudaMallocAsync(&tmp, (size_t)per * n * sizeof(Fr), s));
    for (uint32_t b0 = 0; b0 < batch; b0 += per) {
      const uint32_t nb = std::min<uint32_t>(batch - b0, per);
      ntt4(*tw, v + (size_t)b0 * n, tmp, v + (size_t)b0 * n, inverse != 0, s, nb, cp ? cp->lo : nullptr,
           cp ? cp->hi : nullptr, cp ? cp->h : 0, inverse ? &ninv : nullptr);
    }
    cudaFreeAsync(tmp, s);
  }
  return check_launch();
}


int zg_selftest(int* fails, int nops) {
  const uint32_t n = 1024;
  std::vector<Fq> a(n), b(n);
  uint64_t st = 0x1234;
  for (uint32_t i = 0; i < n; ++i) {
    for (int k = 0; k < 8; ++k) {
      a[i].v[k] = (uint32_t)splitmix64(st);
      b[i].v[k] = (uint32_t)splitmix64(st);
    }
    // full-range operands below the Fr modulus (so they are valid for both fields)
    a[i].v[7] &= 0x3fffffffu;
    b[i].v[7] &= 0x3fffffffu;
    if (i & 1) { a[i].v[7] &= 0x0fffffffu; b[i].v[7] &= 0x0fffffffu; }
    for (Fq* x : {&a[i], &b[i]}) {
      Fr t = *reinterpret_cast<Fr*>(x);
      for (;;) {
        Fr d;
        if (Fr::sub_raw(d, t, Fr::modulus())) break;
        t = d;
      }
      *x = *reinterpret_cast<Fq*>(&t);
    }
  }
  Fq *da = nullptr, *db = nullptr, *dr = nullptr;
  ZG_CK(cudaMalloc(&da, n * sizeof(Fq)));
  ZG_CK(cudaMalloc(&db, n * sizeof(Fq)));
  ZG_CK(cudaMalloc(&dr, SELFTEST_OPS * n * sizeof(Fq)));
  ZG_CK(cudaMemcpy(da, a.data(), n * sizeof(Fq), cudaMemcpyHostToDevice));
  ZG_CK(cudaMemcpy(db, b.data(), n * sizeof(Fq), cudaMemcpyHostToDevice));
  k_selftest<<<n / 128, 128>>>(da, db, dr, n);
  ZG_CK(cudaDeviceSynchronize());
  std::vector<Fq> r(SELFTEST_OPS * n);
  ZG_CK(cudaMemcpy(r.data(), dr, SELFTEST_OPS * n * sizeof(Fq), cudaMemcpyDeviceToHost));
  cudaFree(da); cudaFree(db); cudaFree(dr);
  int cnt[SELFTEST_OPS] = {};
  for (uint32_t i = 0; i < n; ++i) {
    Fq x = a[i], y = b[i];
    Fq e[SELFTEST_OPS];
    e[0] = Fq::mul(x, y);
    e[1] = e[0];
    e[2] = Fq::add(x, y);
    e[3] = Fq::sub(x, y);
    Fr xr = *reinterpret_cast<const Fr*>(&x), yr = *reinterpret_cast<const Fr*>(&y);
    Fr m = Fr::mul(xr, yr);
    e[4] = *reinterpret_cast<Fq*>(&m);
    e[5] = *reinterpret_cast<Fq*>(&xr);
    e[6] = Fq::one();
    e[7] = e[0];
    e[8] = e[4];
    for (int k = 0; k < SELFTEST_OPS; ++k) cnt[k] += (r[SELFTEST_OPS * i + k] != e[k]);
  }
  for (int k = 0; k < nops && k < SELFTEST_OPS; ++k) fails[k] = cnt[k];
  return ZG_OK;
}




int zg_probe_imad(int device, double* gimad_per_s) {
  if (!gimad_per_s) return fail(ZG_ERR_INVALID_ARG, "null output");
  ZG_CK(cudaSetDevice(device));
  int sms = 0;
  ZG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  uint32_t* sink = nullptr;
  ZG_CK(cudaMalloc(&sink, 4));
  cudaEvent_t e0, e1;
  ZG_CK(cudaEventCreate(&e0));
  ZG_CK(cudaEventCreate(&e1));
  const unsigned blocks = (unsigned)sms * 8, threads = 256;
  const uint32_t iters = 4096;
  k_imad_probe<<<blocks, threads>>>(sink, 64, 7);  // warm-up
  ZG_CK(cudaEventRecord(e0));
  k_imad_probe<<<blocks, threads>>>(sink, iters, 7);
  ZG_CK(cudaEventRecord(e1));
  ZG_CK(cudaEventSynchronize(e1));
  float ms = 0;
  ZG_CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  double ops = (double)blocks * threads * iters * 16 * 8;
  *gimad_per_s = ops / (ms * 1e-3) / 1e9;
  return ZG_OK;
}

}  // extern "C"

namespace {
// Fq products of one kind issued as the point additions issue them: each
// thread runs one dependent chain of product pairs (M::mul2, the out-of-line
// pair function of the bucket loop), launched with the bucket kernel's shape
// (FB_ACC_THREADS threads, FB_ACC_MIN_CTAS CTAs per SM).
template <class M>
__global__ void __launch_bounds__(FB_ACC_THREADS, FB_ACC_MIN_CTAS) k_product_probe(Fq* sink, uint32_t iters) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  Fq a, b, c, d;
  for (int i = 0; i < 8; ++i) {
    a.v[i] = tid * 0x9e3779b9u + i;
    b.v[i] = tid ^ (0x7f4a7c15u * (i + 1));
    c.v[i] = a.v[i] ^ 0x5bd1e995u;
    d.v[i] = b.v[i] + 0x1234567u;
  }
  a.v[7] &= 0x0fffffffu; b.v[7] &= 0x0fffffffu; c.v[7] &= 0x0fffffffu; d.v[7] &= 0x0fffffffu;
  for (uint32_t it = 0; it < iters; ++it) {
    const FqPair r = M::mul2(a, b, c, d);
    a = r.a;
    c = r.b;
  }
  sink[2 * tid] = a;
  sink[2 * tid + 1] = c;
}

template <class M>
int product_probe(int sms, double* out) {
  const unsigned blocks = (unsigned)sms * FB_ACC_MIN_CTAS, threads = FB_ACC_THREADS;
  Fq* sink = nullptr;
  ZG_CK(cudaMalloc(&sink, sizeof(Fq) * 2 * blocks * threads));
  cudaEvent_t e0, e1;
  ZG_CK(cudaEventCreate(&e0));
  ZG_CK(cudaEventCreate(&e1));
  const uint32_t iters = 2048;
  k_product_probe<M><<<blocks, threads>>>(sink, 16);  // warm-up
  ZG_CK(cudaEventRecord(e0));
  k_product_probe<M><<<blocks, threads>>>(sink, iters);
  ZG_CK(cudaEventRecord(e1));
  ZG_CK(cudaEventSynchronize(e1));
  float ms = 0;
  ZG_CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  *out = 2.0 * blocks * threads * iters / (ms * 1e-3) / 1e9;
  return ZG_OK;
}
}  // namespace

extern "C" {

int zg_probe_products(int device, uint32_t kind, double* gprod_per_s) {
  if (!gprod_per_s || kind >= ZG_MSM_PRODUCTS) return fail(ZG_ERR_INVALID_ARG, "bad product probe arguments");
  ZG_CK(cudaSetDevice(device));
  int sms = 0;
  ZG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  switch (kind) {
    case ZG_MSM_PRODUCT_IMAD: return product_probe<MulImad>(sms, gprod_per_s);
    case ZG_MSM_PRODUCT_FP64: return product_probe<MulF64>(sms, gprod_per_s);
    case ZG_MSM_PRODUCT_W28: return product_probe<MulW28>(sms, gprod_per_s);
    case ZG_MSM_PRODUCT_W28_HYBRID: return product_probe<MulW28Hybrid>(sms, gprod_per_s);
    default: return product_probe<MulHybrid>(sms, gprod_per_s);
  }
}

int zg_merkle_roots(const void* d_items, size_t n_items, void* d_roots, void* stream) {
  if (!d_items || !d_roots || n_items < 24 || n_items % 24) return fail(ZG_ERR_INVALID_ARG, "n_items must be 3*8*2^k");
  size_t leaves = n_items / 8;
  size_t per = leaves / 3;
  if (per & (per - 1)) return fail(ZG_ERR_INVALID_ARG, "n_items must be 3*8*2^k");
  int depth = 0;
  while (((size_t)3 << depth) < leaves) ++depth;
  std::vector<uint64_t> off(depth + 1);
  size_t o = 0;
  for (int d = 0; d <= depth; ++d) {
    off[d] = o;
    o += ((size_t)3 << d) * 32;
  }
  cudaStream_t s = (cudaStream_t)stream;
  uint8_t* tree = nullptr;
  keep_pool_memory();
  ZG_CK(cudaMallocAsync(&tree, o, s));
  int rc = merkle_levels((const uint8_t*)d_items, n_items, tree, off, depth, s);
  if (!rc) ZG_CK(cudaMemcpyAsync(d_roots, tree, 96, cudaMemcpyDeviceToDevice, s));
  cudaFreeAsync(tree, s);
  return rc;
}

}  // extern "C"
