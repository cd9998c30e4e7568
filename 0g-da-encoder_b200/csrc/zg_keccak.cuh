// Keccak-256 (Keccak-f[1600], rate 136 bytes, original 0x01 padding) as used
// by the reference's Merkle tree (tiny-keccak 2.0.2 `Keccak::v256`,
// crates/encoder/src/utils.rs:45-66; keccak-hash 0.10 `keccak`,
// crates/encoder/src/merkle/slice.rs:95). State lives in 25 64-bit
// registers; the rho/pi/chi steps are fully unrolled.
#pragma once
#include <stdint.h>

namespace zg {

__device__ __constant__ uint64_t KECCAK_RC_DEV[24] = {
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808aULL, 0x8000000080008000ULL,
    0x000000000000808bULL, 0x0000000080000001ULL, 0x8000000080008081ULL, 0x8000000000008009ULL,
    0x000000000000008aULL, 0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000aULL,
    0x000000008000808bULL, 0x800000000000008bULL, 0x8000000000008089ULL, 0x8000000000008003ULL,
    0x8000000000008002ULL, 0x8000000000000080ULL, 0x000000000000800aULL, 0x800000008000000aULL,
    0x8000000080008081ULL, 0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};

__device__ __forceinline__ uint64_t k_rotl(uint64_t x, int s) { return (x << s) | (x >> (64 - s)); }

__device__ __forceinline__ void keccak_f1600(uint64_t a[25]) {
#pragma unroll 1
  for (int round = 0; round < 24; ++round) {
    uint64_t c0 = a[0] ^ a[5] ^ a[10] ^ a[15] ^ a[20];
    uint64_t c1 = a[1] ^ a[6] ^ a[11] ^ a[16] ^ a[21];
    uint64_t c2 = a[2] ^ a[7] ^ a[12] ^ a[17] ^ a[22];
    uint64_t c3 = a[3] ^ a[8] ^ a[13] ^ a[18] ^ a[23];
    uint64_t c4 = a[4] ^ a[9] ^ a[14] ^ a[19] ^ a[24];
    uint64_t d0 = c4 ^ k_rotl(c1, 1), d1 = c0 ^ k_rotl(c2, 1), d2 = c1 ^ k_rotl(c3, 1),
             d3 = c2 ^ k_rotl(c4, 1), d4 = c3 ^ k_rotl(c0, 1);
    a[0] ^= d0; a[5] ^= d0; a[10] ^= d0; a[15] ^= d0; a[20] ^= d0;
    a[1] ^= d1; a[6] ^= d1; a[11] ^= d1; a[16] ^= d1; a[21] ^= d1;
    a[2] ^= d2; a[7] ^= d2; a[12] ^= d2; a[17] ^= d2; a[22] ^= d2;
    a[3] ^= d3; a[8] ^= d3; a[13] ^= d3; a[18] ^= d3; a[23] ^= d3;
    a[4] ^= d4; a[9] ^= d4; a[14] ^= d4; a[19] ^= d4; a[24] ^= d4;
    // rho + pi: b[y + 5((2x + 3y) % 5)] = rotl(a[x + 5y], r[x][y])
    uint64_t b[25];
    b[0] = a[0];
    b[10] = k_rotl(a[1], 1);
    b[20] = k_rotl(a[2], 62);
    b[5] = k_rotl(a[3], 28);
    b[15] = k_rotl(a[4], 27);
    b[16] = k_rotl(a[5], 36);
    b[1] = k_rotl(a[6], 44);
    b[11] = k_rotl(a[7], 6);
    b[21] = k_rotl(a[8], 55);
    b[6] = k_rotl(a[9], 20);
    b[7] = k_rotl(a[10], 3);
    b[17] = k_rotl(a[11], 10);
    b[2] = k_rotl(a[12], 43);
    b[12] = k_rotl(a[13], 25);
    b[22] = k_rotl(a[14], 39);
    b[23] = k_rotl(a[15], 41);
    b[8] = k_rotl(a[16], 45);
    b[18] = k_rotl(a[17], 15);
    b[3] = k_rotl(a[18], 21);
    b[13] = k_rotl(a[19], 8);
    b[14] = k_rotl(a[20], 18);
    b[24] = k_rotl(a[21], 2);
    b[9] = k_rotl(a[22], 61);
    b[19] = k_rotl(a[23], 56);
    b[4] = k_rotl(a[24], 14);
#pragma unroll
    for (int y = 0; y < 5; ++y) {
      uint64_t t0 = b[5 * y], t1 = b[5 * y + 1], t2 = b[5 * y + 2], t3 = b[5 * y + 3], t4 = b[5 * y + 4];
      a[5 * y] = t0 ^ (~t1 & t2);
      a[5 * y + 1] = t1 ^ (~t2 & t3);
      a[5 * y + 2] = t2 ^ (~t3 & t4);
      a[5 * y + 3] = t3 ^ (~t4 & t0);
      a[5 * y + 4] = t4 ^ (~t0 & t1);
    }
    a[0] ^= KECCAK_RC_DEV[round];
  }
}

// keccak256 of exactly 64 bytes given as 8 little-endian words
__device__ __forceinline__ void keccak256_64(const uint64_t in[8], uint64_t out[4]) {
  uint64_t a[25];
#pragma unroll
  for (int i = 0; i < 25; ++i) a[i] = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = in[i];
  a[8] = 0x01;                      // padding byte at offset 64
  a[16] = 0x8000000000000000ULL;    // final bit at offset 135
  keccak_f1600(a);
#pragma unroll
  for (int i = 0; i < 4; ++i) out[i] = a[i];
}

// keccak256 of exactly 256 bytes given as 32 little-endian words
__device__ __forceinline__ void keccak256_256(const uint64_t in[32], uint64_t out[4]) {
  uint64_t a[25];
#pragma unroll
  for (int i = 0; i < 25; ++i) a[i] = 0;
#pragma unroll
  for (int i = 0; i < 17; ++i) a[i] = in[i];
  keccak_f1600(a);
#pragma unroll
  for (int i = 0; i < 15; ++i) a[i] ^= in[17 + i];
  a[15] ^= 0x01;                    // offset 120 of the second block
  a[16] ^= 0x8000000000000000ULL;
  keccak_f1600(a);
#pragma unroll
  for (int i = 0; i < 4; ++i) out[i] = a[i];
}

}  // namespace zg
