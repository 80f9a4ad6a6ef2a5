// K0: input generation + BLAKE3-compression R1CS witness, device side.
//
// One thread per compression.  The thread regenerates its inputs from the
// seed with the counter-based form of the benchmark SplitMix64 stream
// (benchmark-tools/common/src/lib.rs:25-37; state of draw j of compression i
// is init + (25 i + j + 1) * gamma, crates/flock-prover/src/seed_pipe.rs:
// 114-146), runs the compression and streams the three packed row-witness
// bit vectors of its 2^14-bit block:
//   z = the witness, a = A_0 z, b = B_0 z
// with the row semantics of crates/flock-prover/src/r1cs_hashes/blake3.rs:
// constant row (1,1,1); input and lin-id rows (v, v, 1); carry rows
// (carry_aux, X ^ cin, Y ^ cin); padding rows 0 (:1890-1905), in the
// I/O-aligned layout of :198-222.  Bits [512, 15409) are produced in address
// order by a 64-bit streaming writer; the 512-bit cv/out_lo prefix and the
// zero tail are written at the end.  c = C z = z is not materialised.
#include "kernels.cuh"

namespace {
constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;

__device__ __forceinline__ uint32_t splitmix(uint64_t state) {
  uint64_t z = state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return (uint32_t)(z ^ (z >> 31));
}

struct RowStream {
  uint64_t* z;
  uint64_t* a;
  uint64_t* b;
  uint64_t zw = 0, aw = 0, bw = 0;
  int fill = 0;  // bits pending in the accumulators
  int word = 8;  // next u64 index to write (bit 512 starts word 8)
  __device__ __forceinline__ void put(int n, uint32_t zv, uint32_t av, uint32_t bv) {
    zw |= (uint64_t)zv << fill;
    aw |= (uint64_t)av << fill;
    bw |= (uint64_t)bv << fill;
    int nf = fill + n;
    if (nf >= 64) {
      z[word] = zw;
      a[word] = aw;
      b[word] = bw;
      word++;
      int used = 64 - fill;  // bits of this field already consumed
      zw = used < 32 ? (uint64_t)(zv >> used) : 0;
      aw = used < 32 ? (uint64_t)(av >> used) : 0;
      bw = used < 32 ? (uint64_t)(bv >> used) : 0;
      nf -= 64;
    }
    fill = nf;
  }
  __device__ __forceinline__ void ident(uint32_t v) { put(32, v, v, 0xFFFFFFFFu); }
  __device__ __forceinline__ uint32_t add(uint32_t x, uint32_t y) {
    uint32_t s = x + y, cin = s ^ x ^ y;
    uint32_t l = (x ^ cin) & 0x7FFFFFFFu, r = (y ^ cin) & 0x7FFFFFFFu;
    put(31, l & r, l, r);
    return s;
  }
};

__device__ __forceinline__ uint32_t rr(uint32_t x, int n) { return __funnelshift_r(x, x, n); }

__device__ void compression_witness(const uint32_t cv[8], const uint32_t m_in[16], uint32_t tlo, uint32_t thi,
                                    uint32_t blen, uint32_t flags, uint64_t* z, uint64_t* a, uint64_t* b) {
  RowStream s{z, a, b};
  s.put(1, 1, 1, 1);  // constant wire at bit 512
  uint32_t m[16];
#pragma unroll
  for (int i = 0; i < 16; i++) { m[i] = m_in[i]; s.ident(m[i]); }
  s.ident(tlo);
  s.ident(thi);
  s.ident(blen);
  s.ident(flags);
  uint32_t v[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                    b3d::kIV[0], b3d::kIV[1], b3d::kIV[2], b3d::kIV[3], tlo, thi, blen, flags};
#define WG(A, B, C, D, X, Y)                                   \
  {                                                            \
    uint32_t a1 = s.add(s.add(v[A], v[B]), (X));               \
    uint32_t d1 = rr(v[D] ^ a1, 16);                           \
    uint32_t c1 = s.add(v[C], d1);                             \
    uint32_t b1 = rr(v[B] ^ c1, 12);                           \
    uint32_t a2 = s.add(s.add(a1, b1), (Y));                   \
    uint32_t d2 = rr(d1 ^ a2, 8);                              \
    uint32_t c2 = s.add(c1, d2);                               \
    uint32_t bn = rr(b1 ^ c2, 7);                              \
    s.ident(bn);                                               \
    s.ident(d2);                                               \
    v[A] = a2; v[B] = bn; v[C] = c2; v[D] = d2;                \
  }
#pragma unroll 1
  for (int r = 0; r < 7; r++) {
    WG(0, 4, 8, 12, m[0], m[1]);
    WG(1, 5, 9, 13, m[2], m[3]);
    WG(2, 6, 10, 14, m[4], m[5]);
    WG(3, 7, 11, 15, m[6], m[7]);
    WG(0, 5, 10, 15, m[8], m[9]);
    WG(1, 6, 11, 12, m[10], m[11]);
    WG(2, 7, 8, 13, m[12], m[13]);
    WG(3, 4, 9, 14, m[14], m[15]);
    uint32_t t[16] = {m[2], m[6], m[3], m[10], m[7], m[0], m[4], m[13],
                      m[1], m[11], m[12], m[5], m[9], m[14], m[15], m[8]};
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = t[i];
  }
#undef WG
  uint32_t lo[8];
#pragma unroll
  for (int w = 0; w < 8; w++) {
    lo[w] = v[w] ^ v[w + 8];
    s.ident(v[w + 8] ^ cv[w]);  // out_hi at 15153 + 32 w
  }
  // bit 15409 reached: flush the partial word, then zero padding to 16384
  s.put(0, 0, 0, 0);
  z[s.word] = s.zw; a[s.word] = s.aw; b[s.word] = s.bw;
  for (int w = s.word + 1; w < 256; w++) { z[w] = 0; a[w] = 0; b[w] = 0; }
  // prefix: cv (bits 0..255) and out_lo (256..511), rows (v, v, 1)
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint64_t c = (uint64_t)cv[2 * k] | ((uint64_t)cv[2 * k + 1] << 32);
    uint64_t o = (uint64_t)lo[2 * k] | ((uint64_t)lo[2 * k + 1] << 32);
    z[k] = c; a[k] = c; b[k] = ~0ull;
    z[4 + k] = o; a[4 + k] = o; b[4 + k] = ~0ull;
  }
}
}  // namespace

__global__ void k_witness_seed(uint64_t seed, uint32_t log2, uint32_t n_blocks, uint32_t n_slots,
                               f128* __restrict__ z, f128* __restrict__ a, f128* __restrict__ b) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_slots) return;
  uint32_t cv[8], m[16], ctr = 0, blen = 0, flags = 0;
  if (i < n_blocks) {
    uint64_t init = seed ^ (((uint64_t)log2 << 29) | ((uint64_t)log2 >> 35));
    uint64_t st = init + (uint64_t)(25ull * i) * kGamma;
#pragma unroll
    for (int w = 0; w < 8; w++) { st += kGamma; cv[w] = splitmix(st); }
#pragma unroll
    for (int w = 0; w < 16; w++) { st += kGamma; m[w] = splitmix(st); }
    st += kGamma;
    ctr = splitmix(st);
    blen = 64;
    flags = 11;
  } else {  // padding slot: the all-zero compression (blake3.rs:4631-4636)
#pragma unroll
    for (int w = 0; w < 8; w++) cv[w] = 0;
#pragma unroll
    for (int w = 0; w < 16; w++) m[w] = 0;
  }
  size_t off = (size_t)i * 256;
  compression_witness(cv, m, ctr, 0, blen, flags, reinterpret_cast<uint64_t*>(z) + off,
                      reinterpret_cast<uint64_t*>(a) + off, reinterpret_cast<uint64_t*>(b) + off);
}

// blocks: 25 u32 per compression (cv[8], m[16], counter_lo); counter_hi = 0,
// block_len = 64, flags = 11 as in the benchmark generator.
__global__ void k_witness_blocks(const uint32_t* __restrict__ blocks, uint32_t n_blocks, uint32_t n_slots,
                                 f128* __restrict__ z, f128* __restrict__ a, f128* __restrict__ b) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_slots) return;
  uint32_t cv[8] = {0}, m[16] = {0}, ctr = 0, blen = 0, flags = 0;
  if (i < n_blocks) {
    const uint32_t* p = blocks + (size_t)25 * i;
#pragma unroll
    for (int w = 0; w < 8; w++) cv[w] = p[w];
#pragma unroll
    for (int w = 0; w < 16; w++) m[w] = p[8 + w];
    ctr = p[24];
    blen = 64;
    flags = 11;
  }
  size_t off = (size_t)i * 256;
  compression_witness(cv, m, ctr, 0, blen, flags, reinterpret_cast<uint64_t*>(z) + off,
                      reinterpret_cast<uint64_t*>(a) + off, reinterpret_cast<uint64_t*>(b) + off);
}

void launch_witness_seed(uint64_t seed, uint32_t log2, uint32_t n_blocks, uint32_t n_slots, f128* z, f128* a,
                         f128* b, cudaStream_t s) {
  count_launch(); k_witness_seed<<<(n_slots + 127) / 128, 128, 0, s>>>(seed, log2, n_blocks, n_slots, z, a, b);
}
void launch_witness_blocks(const uint32_t* blocks, uint32_t n_blocks, uint32_t n_slots, f128* z, f128* a, f128* b,
                           cudaStream_t s) {
  count_launch(); k_witness_blocks<<<(n_slots + 127) / 128, 128, 0, s>>>(blocks, n_blocks, n_slots, z, a, b);
}
