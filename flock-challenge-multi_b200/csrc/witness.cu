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

// Words are staged per thread in shared memory, 16 per stream, and written
// out by the whole warp once every lane has filled a 16-word block: the
// layout of the 2^14-bit block is data-independent, so all lanes reach the
// same word at the same time, and the warp stores each thread's 128-byte
// run with 16 consecutive lanes (two full lines per store instruction).
constexpr int kWThreads = 128;
constexpr int kStride = 17;  // words per staged thread row (16 + 1 pad)
constexpr size_t kWitnessSmem = (size_t)3 * kWThreads * kStride * sizeof(uint64_t);

struct Stage {
  uint64_t* sm;      // [stream][thread][kStride] for this CTA
  uint64_t* out[3];  // z, a, b of compression i0 (the warp's first)
  int lane, warp;
  uint32_t valid;    // lanes whose compression slot exists
};

// store words [lo, hi) of block blk of the warp's 32 compressions
__device__ __forceinline__ void flush(const Stage& S, int blk, int lo, int hi) {
  __syncwarp();
#pragma unroll
  for (int st = 0; st < 3; st++) {
    const uint64_t* src = S.sm + ((size_t)st * kWThreads + S.warp * 32) * kStride;
    for (int idx = S.lane; idx < 32 * 16; idx += 32) {
      const int t = idx >> 4, w = idx & 15;
      if (w >= lo && w < hi && ((S.valid >> t) & 1))
        S.out[st][(size_t)t * 256 + blk * 16 + w] = src[t * kStride + w];
    }
  }
  __syncwarp();
}

struct RowStream {
  const Stage& S;
  uint64_t* z;  // this thread's staged rows (stride kWThreads * kStride between streams)
  uint64_t zw = 0, aw = 0, bw = 0;
  int fill = 0;  // bits pending in the accumulators
  int word = 8;  // next u64 index to write (bit 512 starts word 8)
  __device__ __forceinline__ void emit(uint64_t zv, uint64_t av, uint64_t bv) {
    const int w = word & 15;
    z[w] = zv;
    z[kWThreads * kStride + w] = av;
    z[2 * kWThreads * kStride + w] = bv;
    if (w == 15) flush(S, word >> 4, word < 16 ? 8 : 0, 16);
    word++;
  }
  __device__ __forceinline__ void put(int n, uint32_t zv, uint32_t av, uint32_t bv) {
    zw |= (uint64_t)zv << fill;
    aw |= (uint64_t)av << fill;
    bw |= (uint64_t)bv << fill;
    int nf = fill + n;
    if (nf >= 64) {
      emit(zw, aw, bw);
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
                                    uint32_t blen, uint32_t flags, const Stage& S) {
  uint64_t* row = S.sm + (size_t)threadIdx.x * kStride;
  RowStream s{S, row};
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
  // bit 15409 reached: the partial word, then zero padding to 16384
  s.put(0, 0, 0, 0);
  s.emit(s.zw, s.aw, s.bw);
  while (s.word < 256) s.emit(0, 0, 0);
  // prefix: cv (bits 0..255) and out_lo (256..511), rows (v, v, 1)
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint64_t c = (uint64_t)cv[2 * k] | ((uint64_t)cv[2 * k + 1] << 32);
    uint64_t o = (uint64_t)lo[2 * k] | ((uint64_t)lo[2 * k + 1] << 32);
    row[k] = c; row[kWThreads * kStride + k] = c; row[2 * kWThreads * kStride + k] = ~0ull;
    row[4 + k] = o; row[kWThreads * kStride + 4 + k] = o; row[2 * kWThreads * kStride + 4 + k] = ~0ull;
  }
  flush(S, 0, 0, 8);
}

__device__ __forceinline__ Stage make_stage(uint64_t* sm, f128* z, f128* a, f128* b, uint32_t n_slots, uint32_t cta) {
  Stage S;
  S.sm = sm;
  S.lane = threadIdx.x & 31;
  S.warp = threadIdx.x >> 5;
  const uint32_t i0 = cta * kWThreads + S.warp * 32;
  S.out[0] = reinterpret_cast<uint64_t*>(z) + (size_t)i0 * 256;
  S.out[1] = reinterpret_cast<uint64_t*>(a) + (size_t)i0 * 256;
  S.out[2] = reinterpret_cast<uint64_t*>(b) + (size_t)i0 * 256;
  S.valid = i0 >= n_slots ? 0u : (n_slots - i0 >= 32 ? 0xffffffffu : (1u << (n_slots - i0)) - 1u);
  return S;
}
}  // namespace

// CTA `cta` of the witness of 2^log2 seeded compressions (n_slots >= n_blocks
// slots; padding slots hold the all-zero compression, blake3.rs:4631-4636)
__device__ __forceinline__ void witness_seed_cta(uint64_t* sm, uint64_t seed, uint32_t log2, uint32_t n_blocks,
                                                 uint32_t n_slots, f128* z, f128* a, f128* b, uint32_t cta) {
  const Stage S = make_stage(sm, z, a, b, n_slots, cta);
  uint32_t i = cta * kWThreads + threadIdx.x;
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
  } else {
#pragma unroll
    for (int w = 0; w < 8; w++) cv[w] = 0;
#pragma unroll
    for (int w = 0; w < 16; w++) m[w] = 0;
  }
  compression_witness(cv, m, ctr, 0, blen, flags, S);
}

__global__ void __launch_bounds__(kWThreads, 4) k_witness_seed(uint64_t seed, uint32_t log2, uint32_t n_blocks,
                                                           uint32_t n_slots, f128* __restrict__ z,
                                                           f128* __restrict__ a, f128* __restrict__ b) {
  extern __shared__ uint64_t wsm[];
  witness_seed_cta(wsm, seed, log2, n_blocks, n_slots, z, a, b, blockIdx.x);
}

// The witnesses of a batch of proofs in one launch: CTA c belongs to the job
// j with jobs[j].wcta0 <= c < jobs[j + 1].wcta0.
__global__ void __launch_bounds__(kWThreads, 4) k_witness_seed_batch(const BatchJob* __restrict__ jobs, int n_jobs) {
  extern __shared__ uint64_t wsm[];
  const uint32_t c = blockIdx.x;
  int lo = 0, hi = n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].wcta0 <= c) lo = mid;
    else hi = mid - 1;
  }
  const BatchJob& J = jobs[lo];
  witness_seed_cta(wsm, J.seed, J.log2, J.n_blocks, J.n_slots, J.z, J.a, J.b, c - (uint32_t)J.wcta0);
}

// blocks: REC u32 per compression.  REC = 25: cv[8], m[16], counter_lo, with
// counter_hi = 0, block_len = 64, flags = 11 as in the benchmark generator.
// REC = 28: the full record cv[8], m[16], counter (u64), block_len, flags
// (Compression, blake3.rs:1861).
template <int REC>
__global__ void __launch_bounds__(kWThreads, 4) k_witness_blocks(const uint32_t* __restrict__ blocks, uint32_t n_blocks,
                                                             uint32_t n_slots, f128* __restrict__ z,
                                                             f128* __restrict__ a, f128* __restrict__ b) {
  extern __shared__ uint64_t wsm[];
  const Stage S = make_stage(wsm, z, a, b, n_slots, blockIdx.x);
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t cv[8] = {0}, m[16] = {0}, ctr = 0, ctr_hi = 0, blen = 0, flags = 0;
  if (i < n_blocks) {
    const uint32_t* p = blocks + (size_t)REC * i;
#pragma unroll
    for (int w = 0; w < 8; w++) cv[w] = p[w];
#pragma unroll
    for (int w = 0; w < 16; w++) m[w] = p[8 + w];
    ctr = p[24];
    if (REC == 28) {
      ctr_hi = p[25];
      blen = p[26];
      flags = p[27];
    } else {
      blen = 64;
      flags = 11;
    }
  }
  compression_witness(cv, m, ctr, ctr_hi, blen, flags, S);
}

void launch_witness_seed(uint64_t seed, uint32_t log2, uint32_t n_blocks, uint32_t n_slots, f128* z, f128* a,
                         f128* b, cudaStream_t s) {
  CK(cudaFuncSetAttribute(k_witness_seed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWitnessSmem));
  count_launch();
  k_witness_seed<<<(n_slots + kWThreads - 1) / kWThreads, kWThreads, kWitnessSmem, s>>>(seed, log2, n_blocks, n_slots,
                                                                                     z, a, b);
}
void launch_witness_blocks(const uint32_t* blocks, uint32_t n_blocks, uint32_t n_slots, f128* z, f128* a, f128* b,
                           cudaStream_t s, bool records) {
  auto kern = records ? k_witness_blocks<28> : k_witness_blocks<25>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWitnessSmem));
  count_launch();
  kern<<<(n_slots + kWThreads - 1) / kWThreads, kWThreads, kWitnessSmem, s>>>(blocks, n_blocks, n_slots, z, a, b);
}

uint32_t witness_ctas(uint32_t n_slots) { return (n_slots + kWThreads - 1) / kWThreads; }
void launch_witness_seed_batch(const BatchJob* jobs, int n_jobs, uint32_t total_ctas, cudaStream_t s) {
  CK(cudaFuncSetAttribute(k_witness_seed_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWitnessSmem));
  count_launch();
  k_witness_seed_batch<<<total_ctas, kWThreads, kWitnessSmem, s>>>(jobs, n_jobs);
}
