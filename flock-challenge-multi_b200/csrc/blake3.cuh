// Device BLAKE3 compression (published BLAKE3 specification; the reference
// reaches it through the `blake3` crate 1.8.6 and restates it in
// crates/flock-prover/src/r1cs_hashes/blake3.rs:266-350).  Returns the first
// eight output words (chaining value / first 32 bytes of a root output).
#pragma once
#include <cstdint>

namespace b3d {
__constant__ __device__ static const uint32_t kIV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                                      0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
enum : uint32_t { CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8 };

__device__ __forceinline__ uint32_t rotr(uint32_t x, int n) { return __funnelshift_r(x, x, n); }

#define B3G(a, b, c, d, x, y)      \
  a = a + b + (x); d = rotr(d ^ a, 16); \
  c = c + d;       b = rotr(b ^ c, 12); \
  a = a + b + (y); d = rotr(d ^ a, 8);  \
  c = c + d;       b = rotr(b ^ c, 7);

// message schedule: word index used by round r at slot i = PERM^r(i)
__device__ __forceinline__ void compress(const uint32_t cv[8], const uint32_t m[16], uint64_t counter,
                                         uint32_t block_len, uint32_t flags, uint32_t out[8]) {
  uint32_t s0 = cv[0], s1 = cv[1], s2 = cv[2], s3 = cv[3], s4 = cv[4], s5 = cv[5], s6 = cv[6], s7 = cv[7];
  uint32_t s8 = kIV[0], s9 = kIV[1], s10 = kIV[2], s11 = kIV[3];
  uint32_t s12 = (uint32_t)counter, s13 = (uint32_t)(counter >> 32), s14 = block_len, s15 = flags;
  uint32_t w[16];
#pragma unroll
  for (int i = 0; i < 16; i++) w[i] = m[i];
#pragma unroll
  for (int r = 0; r < 7; r++) {
    B3G(s0, s4, s8, s12, w[0], w[1]);
    B3G(s1, s5, s9, s13, w[2], w[3]);
    B3G(s2, s6, s10, s14, w[4], w[5]);
    B3G(s3, s7, s11, s15, w[6], w[7]);
    B3G(s0, s5, s10, s15, w[8], w[9]);
    B3G(s1, s6, s11, s12, w[10], w[11]);
    B3G(s2, s7, s8, s13, w[12], w[13]);
    B3G(s3, s4, s9, s14, w[14], w[15]);
    if (r < 6) {
      uint32_t t[16] = {w[2], w[6], w[3], w[10], w[7], w[0], w[4], w[13],
                        w[1], w[11], w[12], w[5], w[9], w[14], w[15], w[8]};
#pragma unroll
      for (int i = 0; i < 16; i++) w[i] = t[i];
    }
  }
  out[0] = s0 ^ s8; out[1] = s1 ^ s9; out[2] = s2 ^ s10; out[3] = s3 ^ s11;
  out[4] = s4 ^ s12; out[5] = s5 ^ s13; out[6] = s6 ^ s14; out[7] = s7 ^ s15;
}
#undef B3G
}  // namespace b3d
