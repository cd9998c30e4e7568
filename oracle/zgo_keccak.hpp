// ORACLE — test infrastructure only (see zgo_field.hpp).
// Keccak-256 as computed by tiny-keccak 2.0.2 `Keccak::v256` and keccak-hash
// 0.10.0 `keccak` (Cargo.lock:2723,1539), called at
// crates/encoder/src/utils.rs:45-66 and crates/encoder/src/merkle/slice.rs:95.
// Published algorithm: Keccak-f[1600], rate 1088 bits, original padding
// (0x01 ... 0x80), 32-byte output.
#pragma once
#include <cstdint>
#include <cstring>

namespace zgo {

static const uint64_t KECCAK_RC[24] = {
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808aULL, 0x8000000080008000ULL,
    0x000000000000808bULL, 0x0000000080000001ULL, 0x8000000080008081ULL, 0x8000000000008009ULL,
    0x000000000000008aULL, 0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000aULL,
    0x000000008000808bULL, 0x800000000000008bULL, 0x8000000000008089ULL, 0x8000000000008003ULL,
    0x8000000000008002ULL, 0x8000000000000080ULL, 0x000000000000800aULL, 0x800000008000000aULL,
    0x8000000080008081ULL, 0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};

static inline uint64_t rotl64(uint64_t x, int s) { return s ? (x << s) | (x >> (64 - s)) : x; }

// rotation offsets r[x][y] of the rho step, indexed [x + 5 y]
static const int KECCAK_ROT[25] = {0,  1,  62, 28, 27, 36, 44, 6,  55, 20, 3,  10, 43,
                                   25, 39, 41, 45, 15, 21, 8,  18, 2,  61, 56, 14};

static inline void keccak_f(uint64_t A[25]) {
  for (int round = 0; round < 24; ++round) {
    uint64_t C[5], D[5], B[25];
    for (int x = 0; x < 5; ++x) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
    for (int x = 0; x < 5; ++x) D[x] = C[(x + 4) % 5] ^ rotl64(C[(x + 1) % 5], 1);
    for (int i = 0; i < 25; ++i) A[i] ^= D[i % 5];
    // rho + pi: B[y, 2x+3y] = rot(A[x, y], r[x, y])
    for (int x = 0; x < 5; ++x)
      for (int y = 0; y < 5; ++y) B[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(A[x + 5 * y], KECCAK_ROT[x + 5 * y]);
    // chi
    for (int x = 0; x < 5; ++x)
      for (int y = 0; y < 5; ++y)
        A[x + 5 * y] = B[x + 5 * y] ^ ((~B[(x + 1) % 5 + 5 * y]) & B[(x + 2) % 5 + 5 * y]);
    A[0] ^= KECCAK_RC[round];
  }
}

// generic sponge; pad = 0x01 for Keccak-256, 0x06 for SHA3-256 (same permutation)
static inline void keccak256_pad(const uint8_t* in, size_t len, uint8_t out[32], uint8_t pad) {
  const size_t rate = 136;
  uint64_t A[25];
  memset(A, 0, sizeof(A));
  while (len >= rate) {
    for (size_t i = 0; i < rate / 8; ++i) {
      uint64_t w; memcpy(&w, in + 8 * i, 8); A[i] ^= w;
    }
    keccak_f(A);
    in += rate; len -= rate;
  }
  uint8_t block[136];
  memset(block, 0, rate);
  memcpy(block, in, len);
  block[len] ^= pad;
  block[rate - 1] ^= 0x80;
  for (size_t i = 0; i < rate / 8; ++i) {
    uint64_t w; memcpy(&w, block + 8 * i, 8); A[i] ^= w;
  }
  keccak_f(A);
  memcpy(out, A, 32);
}

static inline void keccak256(const uint8_t* in, size_t len, uint8_t out[32]) {
  keccak256_pad(in, len, out, 0x01);
}

}  // namespace zgo
