// K0 for the SHA-256 compression statement: input generation + the packed
// row witness of one compression per 2^15-bit block, device side.
//
// One thread per compression.  The thread streams the three bit vectors of
// its block, z (the witness), a = A_0 z and b = B_0 z, with the row
// semantics of crates/flock-prover/src/r1cs_hashes/sha2.rs:332-520:
//   input rows H_in, M and materialised sums (W[t], T1, E_NEW, A_NEW, H_out):
//     (v, v, 1)
//   Ch rows   (e & (f ^ g), e, f ^ g);  Maj rows ((a ^ b) & (a ^ c), a ^ b, a ^ c)
//   carry rows of an ADD x + y: (carry_aux, x ^ cin, y ^ cin), 31 per ADD
//   the constant row (1, 1, 1) at bit 31400; zero rows after it.
// The layout (:56-121) is region-major (all Ch rows, then all Maj rows, then
// the round carries, ...), not in the order the compression produces them,
// so the thread replays the 64 rounds once per region and writes every bit
// in address order through a 64-bit streaming writer; a replay costs about
// 3 K integer operations, far less than the 12 KiB the thread writes.  The
// message schedule W[0..63] is kept per thread in shared memory.
//
// Inputs: records of 24 u32 (h_in[8], m[16]) and the slots from n on hold
// the compression of the all-zero (h_in, m) (sha2.rs:1185-1209); or the
// benchmark generator of crates/flock-prover/benches/sha2_proof.rs:56-71, one
// SplitMix64 stream from `seed` with 24 draws per compression (h then m), in
// counter form: draw j of compression i uses state seed + (24 i + j + 1) gamma.
#include "kernels.cuh"

namespace {
constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;
constexpr int kThreads = 128;
constexpr int kStride = 17;         // staged u64 words per thread row (16 + 1 pad)
constexpr int kBlockWords = 512;    // u64 words of a 2^15-bit block
constexpr size_t kStageWords = (size_t)3 * kThreads * kStride;
constexpr size_t kSmem = kStageWords * sizeof(uint64_t) + (size_t)64 * kThreads * sizeof(uint32_t);

__constant__ uint32_t kShaK[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

__device__ __forceinline__ uint32_t splitmix(uint64_t state) {
  uint64_t z = state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return (uint32_t)(z ^ (z >> 31));
}
__device__ __forceinline__ uint32_t rr(uint32_t x, int n) { return __funnelshift_r(x, x, n); }

// The warp's 32 compressions are written together: the layout does not
// depend on the data, so every lane fills word w of its staged row at the
// same time, and once 16 words are staged the warp stores each lane's
// 128-byte run with 16 consecutive lanes (two full lines per store).
struct Writer {
  uint64_t* row;      // this thread's staged row of stream 0 (streams kThreads * kStride apart)
  uint64_t* warp_sm;  // the warp's first staged row of stream 0
  uint64_t* out[3];   // z, a, b of the warp's first compression
  uint32_t valid;     // lanes whose slot exists
  int lane;
  uint64_t zw = 0, aw = 0, bw = 0;
  int fill = 0, word = 0;

  __device__ __forceinline__ void flush(int blk) {
    __syncwarp();
#pragma unroll
    for (int st = 0; st < 3; st++) {
      const uint64_t* src = warp_sm + (size_t)st * kThreads * kStride;
      for (int idx = lane; idx < 32 * 16; idx += 32) {
        const int t = idx >> 4, w = idx & 15;
        if ((valid >> t) & 1) out[st][(size_t)t * kBlockWords + blk * 16 + w] = src[t * kStride + w];
      }
    }
    __syncwarp();
  }
  __device__ __forceinline__ void emit(uint64_t zv, uint64_t av, uint64_t bv) {
    const int w = word & 15;
    row[w] = zv;
    row[kThreads * kStride + w] = av;
    row[2 * kThreads * kStride + w] = bv;
    if (w == 15) flush(word >> 4);
    word++;
  }
  // the next n <= 32 rows
  __device__ __forceinline__ void put(int n, uint32_t zv, uint32_t av, uint32_t bv) {
    zw |= (uint64_t)zv << fill;
    aw |= (uint64_t)av << fill;
    bw |= (uint64_t)bv << fill;
    int nf = fill + n;
    if (nf >= 64) {
      emit(zw, aw, bw);
      const int used = 64 - fill;
      zw = used < 32 ? (uint64_t)(zv >> used) : 0;
      aw = used < 32 ? (uint64_t)(av >> used) : 0;
      bw = used < 32 ? (uint64_t)(bv >> used) : 0;
      nf -= 64;
    }
    fill = nf;
  }
  __device__ __forceinline__ void ident(uint32_t v) { put(32, v, v, 0xFFFFFFFFu); }
  // x + y: its 31 carry rows; returns the sum
  __device__ __forceinline__ uint32_t add(uint32_t x, uint32_t y) {
    const uint32_t s = x + y, cin = s ^ x ^ y;
    const uint32_t l = (x ^ cin) & 0x7FFFFFFFu, r = (y ^ cin) & 0x7FFFFFFFu;
    put(31, l & r, l, r);
    return s;
  }
};

// What a replay of the rounds writes.
enum Region { kNone, kCh, kMaj, kCarries, kT1, kENew, kANew };

// The 64 rounds from h_in over the schedule W (shared memory, word t of this
// thread at W[t * kThreads]); writes the rows of `region`, returns the final
// state in s.
template <int R>
__device__ __forceinline__ void rounds(const uint32_t h_in[8], const uint32_t* W, Writer& wr, uint32_t s[8]) {
#pragma unroll
  for (int i = 0; i < 8; i++) s[i] = h_in[i];
#pragma unroll 1
  for (int r = 0; r < 64; r++) {
    const uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
    const uint32_t fg = f ^ g, ab = a ^ b, ac = a ^ c;
    const uint32_t ch = e & fg, maj = ab & ac;
    if (R == kCh) wr.put(32, ch, e, fg);
    if (R == kMaj) wr.put(32, maj, ab, ac);
    const uint32_t S1 = rr(e, 6) ^ rr(e, 11) ^ rr(e, 25), S0 = rr(a, 2) ^ rr(a, 13) ^ rr(a, 22);
    uint32_t t1, t2, e_new, a_new;
    if (R == kCarries) {
      t1 = wr.add(wr.add(wr.add(wr.add(h, S1), ch ^ g), kShaK[r]), W[r * kThreads]);
      t2 = wr.add(S0, maj ^ a);
      e_new = wr.add(d, t1);
      a_new = wr.add(t1, t2);
    } else {
      t1 = h + S1 + (ch ^ g) + kShaK[r] + W[r * kThreads];
      t2 = S0 + (maj ^ a);
      e_new = d + t1;
      a_new = t1 + t2;
    }
    if (R == kT1) wr.ident(t1);
    if (R == kENew) wr.ident(e_new);
    if (R == kANew) wr.ident(a_new);
    s[7] = g; s[6] = f; s[5] = e; s[4] = e_new; s[3] = c; s[2] = b; s[1] = a; s[0] = a_new;
  }
}

__device__ void sha_witness(const uint32_t h_in[8], const uint32_t m[16], uint32_t* W, Writer& wr) {
  // schedule (values only; its rows are written in their region below)
#pragma unroll
  for (int t = 0; t < 16; t++) W[t * kThreads] = m[t];
#pragma unroll 1
  for (int t = 16; t < 64; t++) {
    const uint32_t w2 = W[(t - 2) * kThreads], w15 = W[(t - 15) * kThreads];
    const uint32_t s1 = rr(w2, 17) ^ rr(w2, 19) ^ (w2 >> 10), s0 = rr(w15, 7) ^ rr(w15, 18) ^ (w15 >> 3);
    W[t * kThreads] = s1 + W[(t - 7) * kThreads] + s0 + W[(t - 16) * kThreads];
  }
  uint32_t s[8];
  rounds<kNone>(h_in, W, wr, s);
  // bits 0..1023: H_in, H_out, M
#pragma unroll
  for (int i = 0; i < 8; i++) wr.ident(h_in[i]);
#pragma unroll
  for (int i = 0; i < 8; i++) wr.ident(s[i] + h_in[i]);
#pragma unroll
  for (int i = 0; i < 16; i++) wr.ident(m[i]);
  rounds<kCh>(h_in, W, wr, s);       // 1024..3071
  rounds<kMaj>(h_in, W, wr, s);      // 3072..5119
  rounds<kCarries>(h_in, W, wr, s);  // 5120..19007
#pragma unroll 1
  for (int t = 16; t < 64; t++) wr.ident(W[t * kThreads]);  // 19008..20543
#pragma unroll 1
  for (int t = 16; t < 64; t++) {  // 20544..25007
    const uint32_t w2 = W[(t - 2) * kThreads], w15 = W[(t - 15) * kThreads];
    const uint32_t s1 = rr(w2, 17) ^ rr(w2, 19) ^ (w2 >> 10), s0 = rr(w15, 7) ^ rr(w15, 18) ^ (w15 >> 3);
    wr.add(wr.add(wr.add(s1, W[(t - 7) * kThreads]), s0), W[(t - 16) * kThreads]);
  }
  rounds<kT1>(h_in, W, wr, s);    // 25008..27055
  rounds<kENew>(h_in, W, wr, s);  // 27056..29103
  rounds<kANew>(h_in, W, wr, s);  // 29104..31151
#pragma unroll
  for (int i = 0; i < 8; i++) wr.add(s[i], h_in[i]);  // 31152..31399
  wr.put(1, 1, 1, 1);                                 // the constant wire, 31400
  wr.put(0, 0, 0, 0);
  wr.emit(wr.zw, wr.aw, wr.bw);
  while (wr.word < kBlockWords) wr.emit(0, 0, 0);
}

__device__ __forceinline__ Writer make_writer(uint64_t* sm, f128* z, f128* a, f128* b, uint32_t n_slots) {
  Writer wr;
  wr.lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  wr.row = sm + (size_t)threadIdx.x * kStride;
  wr.warp_sm = sm + (size_t)warp * 32 * kStride;
  const uint32_t i0 = blockIdx.x * kThreads + warp * 32;
  wr.out[0] = reinterpret_cast<uint64_t*>(z) + (size_t)i0 * kBlockWords;
  wr.out[1] = reinterpret_cast<uint64_t*>(a) + (size_t)i0 * kBlockWords;
  wr.out[2] = reinterpret_cast<uint64_t*>(b) + (size_t)i0 * kBlockWords;
  wr.valid = i0 >= n_slots ? 0u : (n_slots - i0 >= 32 ? 0xffffffffu : (1u << (n_slots - i0)) - 1u);
  return wr;
}

// records: n_blocks x 24 u32 (h_in, m), or nullptr for the benchmark
// generator from `seed`; slots n_blocks.. hold the all-zero compression
__global__ void __launch_bounds__(kThreads) k_witness_sha(const uint32_t* __restrict__ records, uint64_t seed,
                                                          uint32_t n_blocks, uint32_t n_slots, f128* z, f128* a,
                                                          f128* b) {
  extern __shared__ __align__(16) uint64_t sm[];
  uint32_t* W = reinterpret_cast<uint32_t*>(sm + kStageWords) + threadIdx.x;
  Writer wr = make_writer(sm, z, a, b, n_slots);
  const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
  uint32_t h[8], m[16];
  if (i < n_blocks && records) {
    const uint32_t* r = records + (size_t)i * 24;
#pragma unroll
    for (int k = 0; k < 8; k++) h[k] = r[k];
#pragma unroll
    for (int k = 0; k < 16; k++) m[k] = r[8 + k];
  } else if (i < n_blocks) {
    uint64_t st = seed + (uint64_t)(24ull * i) * kGamma;
#pragma unroll
    for (int k = 0; k < 8; k++) { st += kGamma; h[k] = splitmix(st); }
#pragma unroll
    for (int k = 0; k < 16; k++) { st += kGamma; m[k] = splitmix(st); }
  } else {
#pragma unroll
    for (int k = 0; k < 8; k++) h[k] = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) m[k] = 0;
  }
  sha_witness(h, m, W, wr);
}
}  // namespace

void launch_witness_sha(const uint32_t* records, uint64_t seed, uint32_t n_blocks, uint32_t n_slots, f128* z, f128* a,
                        f128* b, cudaStream_t s) {
  CK(cudaFuncSetAttribute(k_witness_sha, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
  count_launch();
  k_witness_sha<<<(n_slots + kThreads - 1) / kThreads, kThreads, kSmem, s>>>(records, seed, n_blocks, n_slots, z, a,
                                                                             b);
}
