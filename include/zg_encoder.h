/*
 * zg_encoder.h — C ABI of the B200 blob encoder for the 0G DA encoder path.
 *
 * The reference (0glabs/0g-da-encoder, Rust) exposes this path as
 *   - the gRPC service Encoder.EncodeBlob            grpc/proto/encoder.proto:5-21
 *   - EncoderService::process_data(&[u8], bool)        grpc/src/service.rs:67-105
 *   - EncodedBlob::build / get_row / get_commitment /
 *     get_roots / get_file_root / get_data             crates/encoder/src/encoder/blob.rs:32-62
 *   - RawData::try_from(&[u8]) -> TooLargeBlob         crates/encoder/src/raw_data.rs:55-72
 *   - ZgEncoderParams::from_dir_mont(dir, .., None)    crates/amt/src/blob/encode.rs:114-132
 *   - AMTProofs::gen_amt_proofs (plugin point)         crates/amt/src/prove_params/interfaces.rs:7-15
 * Every entry point below names the reference item it replaces. Plain
 * pointers and sizes only; no exceptions or panics cross this boundary.
 *
 * Status codes: ZG_OK (0); ZG_ERR_TOO_LARGE_BLOB (1) is the reference's only
 * recoverable encoder error (EncoderError::TooLargeBlob); negative values are
 * configuration / device errors. zg_last_error() returns the message of the
 * calling thread's last failure; for ZG_ERR_TOO_LARGE_BLOB it is the
 * reference's Debug text "TooLargeBlob { actual: A, expected_max: M }" that
 * the gRPC layer returns as Status::Unknown (grpc/src/service.rs:61).
 */
#ifndef ZG_ENCODER_H
#define ZG_ENCODER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZG_OK 0
#define ZG_ERR_TOO_LARGE_BLOB 1
#define ZG_ERR_RECOVERY 2
#define ZG_ERR_TIMEOUT 3
#define ZG_ERR_INVALID_ARG (-1)
#define ZG_ERR_CUDA (-2)
#define ZG_ERR_PARAMS (-3)
#define ZG_ERR_INTERNAL (-4)

typedef struct zg_ctx zg_ctx;
typedef struct zg_reply zg_reply;

typedef struct zg_config {
  uint32_t log_row;        /* BLOB_ROW_LOG (crates/encoder/src/constants.rs:14), 10 in production */
  uint32_t log_col;        /* BLOB_COL_LOG (constants.rs:15), 10 in production */
  uint64_t tau_seed;       /* params from a seeded tau when params_dir is NULL */
  const char* params_dir;  /* else: amt-prove-coset{0,1,2}-mont-*-{LR:02}-{LR+LC:02}.bin */
  int device;              /* CUDA device ordinal */
  uint32_t msm_window_bits;/* 0 = auto: 11-bit fixed-base windows when the window
                              tables fit in HBM (else 8-bit), and with 1024
                              columns wider fixed-base windows (12 to 16 bits,
                              one width per AMT line by its node size) for the
                              lines whose nodes hold more than 1024 points, as
                              far as those tables fit with 8 GiB to spare;
                              11 = 11-bit tables only; 8 */
} zg_config;

/* Builds the device-resident encoder params (3 cosets x (LR + 2) G1 lines).
 * Replaces ZgEncoderParams::from_dir_mont (crates/amt/src/blob/encode.rs:114-132)
 * and, for the seeded case, PowerTau::setup_inner + AMTParams::from_pp
 * (crates/amt/src/power_tau.rs:54-80, prove_params/generate.rs:139-263). */
int zg_ctx_create(const zg_config* cfg, zg_ctx** out);
void zg_ctx_destroy(zg_ctx* ctx);
/* ZgEncoderParams::warmup (crates/amt/src/blob/encode.rs:85-89): runs one
 * encode of an empty payload so later calls see warm caches. */
int zg_ctx_warmup(zg_ctx* ctx);

/* EncoderService::process_data (grpc/src/service.rs:67-105): payload bytes ->
 * EncodeBlobReply. `data` is host memory. On ZG_OK *out owns the reply. */
int zg_encode(zg_ctx* ctx, const uint8_t* data, size_t len, int require_data, zg_reply** out);
void zg_reply_free(zg_reply* r);
uint32_t zg_reply_version(const zg_reply* r);                              /* service.rs:98 */
const uint8_t* zg_reply_erasure_commitment(const zg_reply* r, size_t* len); /* service.rs:77-83, 64 B */
const uint8_t* zg_reply_storage_root(const zg_reply* r, size_t* len);       /* get_file_root, 32 B */
const uint8_t* zg_reply_encoded_data(const zg_reply* r, size_t* len);       /* get_data, service.rs:85-91 */
size_t zg_reply_num_slices(const zg_reply* r);                              /* BLOB_ROW_ENCODED */
const uint8_t* zg_reply_slice(const zg_reply* r, size_t index, size_t* len);/* get_row(i) serialized */
const uint8_t* zg_reply_roots(const zg_reply* r, size_t* len);              /* EncodedBlob::get_roots, 96 B */

/* Device-resident variant of zg_encode: `d_data` is device memory, results
 * stay in context-owned device buffers (valid until the next encode on the
 * same context) and the call returns after queuing work on `stream`
 * (cudaStream_t, NULL = the context stream). Same math as zg_encode. */
typedef struct zg_device_blob {
  const uint8_t* encoded_data;  /* [3][R][C] x 32 B, canonical */
  const uint8_t* slices;        /* [3R] x slice_size, serialized EncodedSlice */
  size_t slice_size;
  const uint8_t* amt_outputs;   /* [3][4R-2] x 64 B ark G1: root, commitment tree, proof layers, high */
  const uint8_t* roots;         /* 3 x 32 B */
  const uint8_t* file_root;     /* 32 B */
} zg_device_blob;
int zg_encode_device(zg_ctx* ctx, const void* d_data, size_t len, void* stream, zg_device_blob* out);

/* Copy of points [first, first + count) of one device param line (64 B mont
 * x||y each), the layout of the reference's mont files
 * (fast_serde_bn254.rs:139-160). line < LR: quotients[line]; LR: basis;
 * LR+1: high_basis. */
int zg_ctx_param_points(zg_ctx* ctx, int coset, int line, size_t first, size_t count, uint8_t* host_out,
                        size_t cap);

/* Tuning of the kernels' free choices (no reference counterpart: the
 * reference's GPU plugin fixes its window width and launch shapes inside
 * ag-cuda-ec, prove_gpu.rs:16-17,77). Every choice gives identical results.
 *   msm_product      field products of the MSM point additions:
 *                    ZG_MSM_PRODUCT_IMAD both products of each independent pair
 *                    as 32-bit carry-chain CIOS on the integer multiply-add
 *                    pipe, ZG_MSM_PRODUCT_HYBRID one there and one on the FP64
 *                    pipe, ZG_MSM_PRODUCT_FP64 both on the FP64 pipe,
 *                    ZG_MSM_PRODUCT_W28 both as 28-bit-limb products with 64-bit
 *                    column sums (wide multiply-adds, no carry flags),
 *                    ZG_MSM_PRODUCT_W28_HYBRID one of those and one on the FP64
 *                    pipe;
 *   msm_task         bucket layout: entries per bucket-accumulation task, 32,
 *                    48, 64 (default) or 96 (buckets are cut into tasks of at
 *                    most this many points, scheduled by size);
 *   msm_wide_classes MSM window width per AMT line: how many of the context's
 *                    wide-window classes are in use, largest unit first (class
 *                    u gives the lines whose nodes hold >= 2^u points units of
 *                    2^u points: (u + 1)-bit windows for u <= 15; u = 16 uses
 *                    16-bit windows, pairs of 2^15-point sort units sharing
 *                    their buckets; the lines of the classes not in use run
 *                    11-bit windows per 1024-point chunk); at most
 *                    msm_wide_avail;
 *   ntt_cols_per_cta columns per CTA of the RS column pass: 1, 2 (default), 4;
 *   ntt_threads      threads per CTA of the three RS passes: 128, 256 (default), 512.
 * zg_ctx_autotune encodes a synthetic full-size blob on the context and
 * times the whole blob MSM (digit sorts, bucket accumulation, combine) with
 * each product kind and every wide class (msm_ms), with each task size and
 * the chosen kind (task_ms, sizes {32, 48, 64, 96}); each of these twice in
 * round-robin order, the faster time kept. Then the MSM with 0 ..
 * msm_wide_avail wide classes (wide_ms; -1 where the context has no such
 * class) and each NTT shape on the full RS extension (ntt_ms[3 * i + j] for
 * cols_per_cta {1, 2, 4}[i] and threads {128, 256, 512}[j]). For the MSM
 * choices the default (hybrid kind, task 64, every wide class) stays unless
 * another is more than 1 % faster; for the NTT shape the fastest wins. It
 * returns the choice with the times (ms), runs after the context's queued
 * work and takes several seconds at production size; the request pipeline
 * re-captures its CUDA graphs for the new choice. */
#define ZG_MSM_PRODUCT_IMAD 0
#define ZG_MSM_PRODUCT_HYBRID 1
#define ZG_MSM_PRODUCT_FP64 2
#define ZG_MSM_PRODUCT_W28 3
#define ZG_MSM_PRODUCT_W28_HYBRID 4
#define ZG_MSM_PRODUCTS 5
#define ZG_MSM_TASK_SIZES 4
#define ZG_MSM_WIDE_MAX 6
typedef struct zg_tuning {
  uint32_t msm_product;
  uint32_t msm_task;
  uint32_t msm_wide_classes;
  uint32_t ntt_cols_per_cta;
  uint32_t ntt_threads;
  float msm_ms[ZG_MSM_PRODUCTS];
  float task_ms[ZG_MSM_TASK_SIZES];
  float wide_ms[ZG_MSM_WIDE_MAX + 1];
  float ntt_ms[9];
  uint32_t msm_wide_lines; /* read-only: AMT lines on wide windows with the chosen classes */
  uint32_t msm_wide_avail; /* read-only: wide-window classes whose tables the context holds */
} zg_tuning;
int zg_ctx_autotune(zg_ctx* ctx, zg_tuning* out);
int zg_ctx_get_tuning(zg_ctx* ctx, zg_tuning* out);
int zg_ctx_set_tuning(zg_ctx* ctx, const zg_tuning* t);

/* Measurement hooks (no reference counterpart; the reference logs tracing
 * spans, grpc/src/service.rs:68). With profiling on, every encode records CUDA
 * events between its phases; zg_ctx_phase_times returns the last encode's
 * phase durations in ms: [RS extension, Merkle, MSM, AMT aggregation,
 * slice assembly]. zg_ctx_launches counts kernels this context launched. */
int zg_ctx_set_profiling(zg_ctx* ctx, int enable);
int zg_ctx_phase_times(zg_ctx* ctx, float* ms, int n);
uint64_t zg_ctx_launches(const zg_ctx* ctx);
/* Integer multiply-add rate of the device (independent mad.lo.u32 chains),
 * in 1e9 per second: the denominator of the MSM roofline. */
int zg_probe_imad(int device, double* gimad_per_s);
/* Fq Montgomery products per second (1e9) of one product kind, issued as the
 * MSM bucket loop issues them (one dependent chain of independent product
 * pairs per thread, the bucket kernel's launch shape): the ceiling of the
 * bucket accumulation's executed work. */
int zg_probe_products(int device, uint32_t kind, double* gprod_per_s);

/* recover_from_da_slice (crates/recovery/src/lib.rs:15-43): original payload
 * bytes from any >= R encoded rows. rows[i] (host memory, row_lens[i] bytes)
 * is encoded row row_ids[i] (0 <= id < 3R) as 32-byte canonical elements, the
 * EncodedSlice::merkle_row() bytes. Rows of the wrong length are dropped and
 * one row is kept per id, as the reference's BTreeMap input does. Returns
 * ZG_OK with the payload in out[0..*out_len), or ZG_ERR_RECOVERY with the
 * reference's error text in zg_last_error(): "Not enough valid lines",
 * "Cannot recover data: RowIdOverflow", "Incorrect scalar", "Incorrect length
 * field", "Non zero in padding range"; rows that are not one codeword or hold
 * a value >= r (the reference panics) give their own messages. */
int zg_recover(zg_ctx* ctx, const uint64_t* row_ids, const uint8_t* const* rows, const size_t* row_lens, size_t n,
               uint8_t* out, size_t out_cap, size_t* out_len);

/* Request pipeline, the serving path (the reference serves EncodeBlob on
 * tokio workers, grpc/src/service.rs:49-65; recovery is
 * recover_from_da_slice). zg_submit queues a request and returns at once;
 * zg_wait blocks for its result (timeout_ms < 0: no limit; ZG_ERR_TIMEOUT
 * leaves it queued). Continuous batching: encode requests are taken in
 * submission order by units, each a stream with its own device buffers for
 * up to ZG_MAX_FUSED_BLOBS blobs; a unit takes every waiting request up to
 * that count and encodes them as one launch sequence whose bucket
 * accumulation spans all their MSMs, replayed from a CUDA graph. A new unit
 * is created when every unit is busy, requests are waiting and the device's
 * free memory covers one more unit plus the reserve, so admission follows
 * free HBM; the units' encodes run on the device one after another in issue
 * order while each unit's copies overlap the others' compute. Recovery
 * requests run beside the encodes on their own stream. The caller keeps the request's input buffers
 * valid until zg_wait has returned its result. Encode replies are
 * zg_encode's, bit for bit; recovery replies hold the payload
 * (zg_reply_payload). A failed request's status comes back from zg_wait with
 * its message in zg_last_error(). TooLargeBlob is reported by zg_submit. */
#define ZG_REQ_ENCODE 0
#define ZG_REQ_RECOVER 1
typedef struct zg_request {
  int kind;
  const uint8_t* data; /* encode */
  size_t len;
  int require_data;
  const uint64_t* row_ids; /* recover: as zg_recover */
  const uint8_t* const* rows;
  const size_t* row_lens;
  size_t n_rows;
} zg_request;
int zg_submit(zg_ctx* ctx, const zg_request* req, uint64_t* ticket);
int zg_wait(zg_ctx* ctx, uint64_t ticket, int64_t timeout_ms, zg_reply** out);
const uint8_t* zg_reply_payload(const zg_reply* r, size_t* len);
/* n encodes through the pipeline (uneven payloads welcome); out[i] as
 * zg_encode's reply for data[i], bit-identical to it. On any error no reply
 * is returned. */
int zg_encode_batch(zg_ctx* ctx, size_t n, const uint8_t* const* data, const size_t* lens, int require_data,
                    zg_reply** out);
/* Pipeline settings (no reference counterpart): max_units caps the units
 * (0 = 3, as far as the free HBM allows; at most 8), blobs_per_launch the
 * blobs a unit fuses into one launch sequence (0 = ZG_MAX_FUSED_BLOBS, 1 =
 * no fusing), reserve_mib the device memory admission leaves free (0 = 4096).
 * Takes effect for the next request: a running pipeline is drained and
 * restarted. zg_ctx_pipeline_stats reports what the pipeline did since the
 * context was created. */
#define ZG_MAX_FUSED_BLOBS 2
typedef struct zg_pipeline_config {
  uint32_t max_units;
  uint32_t blobs_per_launch;
  uint32_t reserve_mib;
} zg_pipeline_config;
typedef struct zg_pipeline_stats {
  uint64_t units;             /* units created */
  uint64_t launches[ZG_MAX_FUSED_BLOBS]; /* unit launches of k + 1 blobs */
  uint64_t max_in_flight;     /* most encode requests on the device at once */
  uint64_t recoveries;        /* recovery requests run */
  uint64_t unit_bytes;        /* device bytes of one unit */
} zg_pipeline_stats;
int zg_ctx_set_pipeline(zg_ctx* ctx, const zg_pipeline_config* cfg);
int zg_ctx_pipeline_stats(zg_ctx* ctx, zg_pipeline_stats* out);

/* One MSM over the first n points of a param line with the context's
 * fixed-base tables: out = sum_i scalars[i] * line[i], written as a 64-byte
 * ark G1 (the shape of VariableBaseMSM::msm in prove.rs:17-31 against
 * `basis`, line log_row, or another line). scalars: n canonical 32-byte Fr
 * in device memory; n a power of two in [2^log_col, 2^(log_row+log_col)].
 * Stream-ordered on `stream`, after any earlier encode of the context. */
int zg_ctx_msm(zg_ctx* ctx, uint32_t coset, uint32_t line, const void* d_scalars, size_t n, void* d_out,
               void* stream);

/* Batched EncodedSlice::verify (crates/encoder/src/encoder/slice.rs:73-95) on
 * the GPU. slices[i] (host memory, lens[i] bytes) is one ark-serialized
 * EncodedSlice of a blob, checked against the blob's erasure commitment (the
 * 64 bytes of zg_reply_erasure_commitment: x || y canonical little-endian,
 * all zero for the point at infinity) and storage root (32 B).
 * codes[i] receives the verdict in the reference's check order:
 *   ZG_V_OK, ZG_V_UNMATCHED_AMT_INDEX, ZG_V_UNMATCHED_MERKLE_INDEX (VerifierError),
 *   ZG_V_AMT_INCORRECT_COMMITMENT .. ZG_V_AMT_INCORRECT_PROOF (AmtSignerError),
 *   ZG_V_MERKLE_INCORRECT_ROOT .. ZG_V_MERKLE_INCORRECT_PROOF (MerkleSignerError),
 *   ZG_V_DESERIALIZE (the bytes are not a valid EncodedSlice);
 * details (4 int64 per slice, may be NULL) the variant's fields: [0] the
 * AmtProofError of ZG_V_AMT_INCORRECT_PROOF (0 UnexpectedDataLength,
 * 1 IncorrectPosition, 2 KzgError(d), 3 InconsistentCommitment,
 * 4 FailedLowDegreeTest), [1..3] the variant's integers (indices and sizes,
 * d of KzgError in [3]). The AMT pairing and MSM checks of all slices are
 * folded into random linear combinations (the reference's DeferredVerifier,
 * crates/amt/src/deferred_verification.rs:67-146) with 128-bit coefficients,
 * and bisected down to single slices when a combination fails, so every code
 * is the one EncodedSlice::verify returns. With seed == 0 every coefficient
 * is drawn from the operating system's CSPRNG (getrandom, like the
 * reference's OsRng draws), and a combination accepts a failing batch with
 * probability at most 2^-128. A nonzero seed makes the coefficients a
 * SplitMix64 stream at that seed: reproducible, for tests only, and NOT safe
 * against slices crafted by anyone who knows the seed. Needs the fixed-base
 * tables.
 * Returns ZG_OK once every slice has its verdict. */
#define ZG_V_OK 0
#define ZG_V_UNMATCHED_AMT_INDEX 1
#define ZG_V_UNMATCHED_MERKLE_INDEX 2
#define ZG_V_AMT_INCORRECT_COMMITMENT 10
#define ZG_V_AMT_INCORRECT_ROW_SIZE 11
#define ZG_V_AMT_ROW_INDEX_OVERFLOW 12
#define ZG_V_AMT_UNMATCHED_COSET_INDEX 13
#define ZG_V_AMT_INCORRECT_PROOF 14
#define ZG_V_MERKLE_INCORRECT_ROOT 20
#define ZG_V_MERKLE_INCORRECT_SIZE 21
#define ZG_V_MERKLE_ROW_INDEX_OVERFLOW 22
#define ZG_V_MERKLE_INCORRECT_LOCAL_ROOT 23
#define ZG_V_MERKLE_INCORRECT_PROOF 24
#define ZG_V_DESERIALIZE 30
int zg_verify_slices(zg_ctx* ctx, const uint8_t* const* slices, const size_t* lens, size_t n,
                     const uint8_t* commitment, const uint8_t* storage_root, uint64_t seed, int32_t* codes,
                     int64_t* details);

/* LightEncodedSlice (crates/encoder/src/encoder/light_slice.rs:11-79), host
 * byte conversions of the ark-serialized layouts (no device work).
 * from_slice: LightEncodedSlice::from_slice / EncodedSlice::into_light_slice;
 * the reference unwraps check_amt_idx / check_merkle_idx, here those come
 * back as ZG_ERR_INVALID_ARG with the VerifierError text. into_slice:
 * LightEncodedSlice::into_slice(row), row = C canonical 32-byte scalars. */
int zg_light_slice_from_slice(const uint8_t* slice, size_t len, uint32_t log_row, uint32_t log_col, uint8_t* out,
                              size_t cap, size_t* out_len);
int zg_light_slice_into_slice(const uint8_t* light, size_t len, const uint8_t* row, size_t row_len,
                              uint32_t log_row, uint32_t log_col, uint8_t* out, size_t cap, size_t* out_len);

/* Kernel-level entry points (device pointers, stream-ordered on `stream`).
 * zg_msm_chunks: the AMT plugin's MSM decomposition (prove_gpu.rs:55-87):
 * for every line l < lines and chunk b < nchunks,
 *   out[l][b] = sum_t scalars[b*chunk + t] * bases[l][b*chunk + t]
 * written as 64-byte ark G1. scalars: canonical 32 B; bases: mont x||y.
 * nchunks and chunk are powers of two, chunk <= 1024. */
int zg_msm_chunks(const void* d_bases, const void* d_scalars, uint32_t lines, uint32_t log_nchunks,
                  uint32_t log_chunk, void* d_out, void* stream);
/* Allocation-free variant of zg_msm_chunks (no counterpart in the reference).
 * Same arguments and results, but it calls no cudaMalloc / cudaFree and no
 * allocating library routine: its scratch is a static device array sized for
 * at most 1024 chunk MSMs (lines * 2^log_nchunks <= 1024; larger requests
 * fail with ZG_ERR_INVALID_ARG). It is meant for callers that cannot
 * allocate device memory per call, such as a process that has handed all
 * free HBM to another allocator at start-up, or a loop that must never block
 * on cudaMalloc (which can synchronize the device).
 * Every call looks the array's device address up (cudaGetSymbolAddress)
 * with the call's device current; the first call on a device also loads the
 * module there, so make that first call before any stream capture. The
 * array is the module's, so it does not survive cudaDeviceReset; the next
 * call after a reset finds the reloaded module's array. Every call on a
 * device shares the one array
 * (it keeps the last call's contents; every element is written before it is
 * read, so nothing needs clearing), so calls that overlap on the GPU, e.g. on
 * two streams at once, race: order them on one stream or with events. */
int zg_msm_chunks_noalloc(const void* d_bases, const void* d_scalars, uint32_t lines, uint32_t log_nchunks,
                          uint32_t log_chunk, void* d_out, void* stream);
/* Batched radix-2 NTT over Fr with ark-poly Radix2EvaluationDomain semantics
 * (crates/amt/src/blob/encode.rs:142-157): `batch` contiguous vectors of
 * 2^log_n canonical 32-byte elements, transformed in place. inverse != 0
 * applies the 1/n scaled inverse. coset_idx > 0 (forward only) multiplies
 * coefficient i by coset_factor(2^log_n, coset_idx)^i first (to_coset_blob). */
int zg_ntt(void* d_data, uint32_t log_n, uint32_t batch, int inverse, uint32_t coset_idx, void* stream);
/* Keccak-256 Merkle levels (crates/encoder/src/merkle/blob.rs:15-34) over
 * n_items 32-byte items: leaves = keccak(8 items), then pairwise parents
 * until <= 3 nodes; writes the 3 roots (or fewer) to d_roots. */
int zg_merkle_roots(const void* d_items, size_t n_items, void* d_roots, void* stream);

/* Device arithmetic self test (no reference counterpart): compares the device
 * field and curve routines against the host build of the same code on fixed
 * pseudo-random inputs; fails[k] receives the mismatch count of check k
 * (0 Fq mul, 1 Fq mul on the FP64 pipe, 2 Fq add, 3 Fq sub, 4 Fr mul,
 * 5 Fr Montgomery round trip, 6 XYZZ add(P, P) == dbl(P), 7 Fq mul with
 * 28-bit limbs, 8 Fr mul on the FP64 pipe). */
int zg_selftest(int* fails, int nops);

const char* zg_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* ZG_ENCODER_H */
