// The Keccak-f[1600] statement on the device
// (crates/flock-prover/src/r1cs_hashes/keccak.rs, the monolithic encoder at
// K_LOG = 16): the packed row witness (K0) and the lincheck's matrix
// combination (K6), whose matrices are implicit.
//
// Block layout (keccak.rs:437-505), u64 words of one 2^16-bit block: state_0
// lanes at words 0..24, state_24 at 32..56, the constant 1 at word 64, t_r
// (the chi AND rows of round r) at words 65 + 25 r .. 89 + 25 r; bit z of
// word (base + x + 5y) is state bit (x, y, z).  Rows (keccak.rs:566-644):
//   state_0 / state_24:  z = a = lane value, b = 1
//   constant:            z = a = b = 1
//   t_r (chi):           z = ~B[x+1] & B[x+2], a = ~B[x+1], b = B[x+2],
//                        B = pi(rho(theta(state_r)))
// every other bit 0.  Padding slots hold keccak_f of the zero state
// (keccak.rs:646-660).
//
// Witness: one warp per permutation, lane l < 25 holding lane l of the state.
// theta's column parities, rho-pi's lane permutation and chi's neighbours are
// warp shuffles; every round the warp stores 25 consecutive u64 of t, a and b,
// so a permutation's three 8 KiB blocks are written front to back by one warp.
//
// Matrix combination comb = alpha A^T e + B^T e (+ beta at the constant),
// the walker of keccak.rs:681-848 (KeccakLincheckCircuit::fold_alpha_batched).
// state_r is a linear function of state_0 and t_0..t_{r-1} (state_{r+1} =
// phi(state_r) + t_r + RC_r, phi = pi rho theta), so A^T and B^T are applied
// by the transposed recurrence, A and B sides merged by linearity:
//   K_24 = alpha pin,  K_r = phi^T(K_{r+1} + W_r),
//   W_r(x, y, z) = alpha E_r(x - 1, y, z) + E_r(x - 2, y, z)
// with E_r = e over t_r's rows and pin = e over state_24's rows; K_r lands on
// t_{r-1}'s columns (K_0 on state_0's, plus alpha e there), alpha pin on
// t_23's.  The constant column collects every row's constant part, the round
// constants' share included: sum_r <phi(c_r), W_r> + <c_24, alpha pin> with
// c_0 = 0, c_{r+1} = phi(c_r) + RC_r (the state reached from state_0 = 0 and
// t = 0).  phi^T = theta^T P^T: a gather through the rho-pi permutation, then
// theta^T(u)(x, y, z) = u(x, y, z) + sum_y' u(x + 1, y', z) + sum_y' u(x - 1, y', z + 1).
// Vectors over a state are indexed lane-major, p = 64 (x + 5y) + z, which is
// also the offset of bit (x, y, z) inside a state's or t_r's region.
//
// The 3-wide encoder (keccak3.rs, K_LOG = 17) packs three independent
// permutations per block: sub-keccak i has state_0 in slot 2i (words 64 i..),
// state_24 in slot 2i + 1, the constant is shared at word 192 (bit 12288) and
// t[i, r] is tight from word 193 in the order i * 24 + r.  Its walker is three
// copies of the recurrence (one CTA each) into one comb, the constant column
// collected atomically.  A Shape names the layout.
#include "kernels.cuh"

#include <map>
#include <mutex>

namespace {
constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;
constexpr int kWarps = 8;           // permutations per CTA of the witness kernel
constexpr int kState = 1600;
constexpr int kWRows = 26;          // per permutation: W_0..W_23, alpha pin, alpha e over state_0

// block layout: `width` permutations per block of `words` u64 words
struct Shape {
  int width, words;
  int const_word;  // the constant wire (bit 0 of this word)
  int t_word;      // first word of t[0, 0]
  __host__ __device__ int s0_word(int i) const { return 64 * i; }
  __host__ __device__ int s24_word(int i) const { return 64 * i + 32; }
  __host__ __device__ int t_first(int i) const { return t_word + 25 * 24 * i; }  // t[i, 0]
};
Shape shape_of(int width) {
  return width == 3 ? Shape{3, 2048, 192, 193} : Shape{1, 1024, 64, 65};
}

// rotation offsets r[x][y] of rho (FIPS 202 3.2.2), index 5 x + y
__constant__ uint8_t kRho[25] = {0,  36, 3,  41, 18, 1,  44, 10, 45, 2,  62, 6, 43,
                                 15, 61, 28, 55, 25, 21, 56, 27, 20, 39, 8,  14};
const uint8_t kRhoHost[25] = {0,  36, 3,  41, 18, 1,  44, 10, 45, 2,  62, 6, 43,
                              15, 61, 28, 55, 25, 21, 56, 27, 20, 39, 8,  14};
// iota's round constants (FIPS 202 3.2.5)
__constant__ uint64_t kRc[24] = {
    0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808Aull, 0x8000000080008000ull,
    0x000000000000808Bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
    0x000000000000008Aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000Aull,
    0x000000008000808Bull, 0x800000000000008Bull, 0x8000000000008089ull, 0x8000000000008003ull,
    0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800Aull, 0x800000008000000Aull,
    0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};
const uint64_t kRcHost[24] = {
    0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808Aull, 0x8000000080008000ull,
    0x000000000000808Bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
    0x000000000000008Aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000Aull,
    0x000000008000808Bull, 0x800000000000008Bull, 0x8000000000008089ull, 0x8000000000008003ull,
    0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800Aull, 0x800000008000000Aull,
    0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};

__host__ __device__ __forceinline__ uint64_t rotl64(uint64_t v, int n) {
  return n ? (v << n) | (v >> (64 - n)) : v;
}
__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // SplitMix64's output function
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// states: n_perm x 25 u64 lanes, or nullptr for the benchmark generator
// (benches/keccak3_proof.rs:66-93: 25 SplitMix64 draws per state, state bit
// i = x + 5y + 25z is bit i mod 64 of draw i / 64; draw k of the stream uses
// state seed + (k + 1) gamma).  Permutation i of block o is input o * width +
// i; inputs n_perm.. (and padding blocks) are the zero state.
__global__ void __launch_bounds__(32 * kWarps) k_witness_keccak(const uint64_t* __restrict__ states, uint64_t seed,
                                                                uint32_t n_perm, uint32_t n_slots, Shape S,
                                                                uint64_t* __restrict__ z, uint64_t* __restrict__ a,
                                                                uint64_t* __restrict__ b) {
  const int lane = threadIdx.x & 31;
  const uint32_t wid = blockIdx.x * kWarps + (threadIdx.x >> 5);
  const uint32_t o = wid / S.width;  // block
  const int sub = (int)(wid % S.width);
  if (o >= n_slots) return;  // warp-uniform
  const uint32_t perm = o * S.width + sub;
  const bool on = lane < 25;
  const int x = lane % 5, y = lane / 5;
  uint64_t s = 0;
  if (perm < n_perm) {
    if (states) {
      s = on ? states[(size_t)perm * 25 + lane] : 0;
    } else {
      const uint64_t d = mix64(seed + (uint64_t)(25ull * perm + lane + 1) * kGamma);
#pragma unroll 8
      for (int zz = 0; zz < 64; zz++) {
        const int i = lane + 25 * zz;
        const uint64_t v = __shfl_sync(0xffffffffu, d, (i >> 6) & 31);
        s |= ((v >> (i & 63)) & 1ull) << zz;
      }
      if (!on) s = 0;
    }
  }
  // rho-pi pulls lane (x, y) from lane (a, b) = ((x + 3y) mod 5, x), rotated by r[a][b]
  const int pa = (x + 3 * y) % 5, pb = x;
  const int src = pa + 5 * pb, rot = on ? kRho[5 * pa + pb] : 0;
  const int n1 = (x + 1) % 5 + 5 * y, n2 = (x + 2) % 5 + 5 * y;
  const int cm = (x + 4) % 5, cp = (x + 1) % 5;
  uint64_t* zb = z + (size_t)o * S.words;
  uint64_t* ab = a + (size_t)o * S.words;
  uint64_t* bb = b + (size_t)o * S.words;
  const int w0 = S.s0_word(sub);
  zb[w0 + lane] = s;  // lanes 25..31 write the slot's zero words 25..31
  ab[w0 + lane] = s;
  bb[w0 + lane] = on ? ~0ull : 0ull;
  const int tw = S.t_first(sub);
  for (int r = 0; r < 24; r++) {
    uint64_t c = 0;
#pragma unroll
    for (int k = 0; k < 5; k++) c ^= __shfl_sync(0xffffffffu, s, x + 5 * k);
    const uint64_t d = __shfl_sync(0xffffffffu, c, cm) ^ rotl64(__shfl_sync(0xffffffffu, c, cp), 1);
    const uint64_t bv = rotl64(__shfl_sync(0xffffffffu, s ^ d, src), rot);
    const uint64_t b1 = __shfl_sync(0xffffffffu, bv, n1 & 31), b2 = __shfl_sync(0xffffffffu, bv, n2 & 31);
    const uint64_t t = ~b1 & b2;
    if (on) {
      const int w = tw + 25 * r + lane;
      zb[w] = t;
      ab[w] = ~b1;
      bb[w] = b2;
    }
    s = bv ^ t;
    if (lane == 0) s ^= kRc[r];
  }
  const int w24 = S.s24_word(sub);
  zb[w24 + lane] = on ? s : 0;
  ab[w24 + lane] = on ? s : 0;
  bb[w24 + lane] = on ? ~0ull : 0ull;
  if (sub == 0 && lane == 0) zb[S.const_word] = ab[S.const_word] = bb[S.const_word] = 1;
  if (sub == S.width - 1)  // the block's zero tail after the last t row
    for (int w = S.t_first(S.width) + lane; w < S.words; w += 32) zb[w] = ab[w] = bb[w] = 0;
}

// W rows (see the file comment) and the zero columns of comb (the constant
// column too: the walkers XOR their parts into it).
// W[i][r][p], r < 24: alpha E_r(x - 1, y, z) + E_r(x - 2, y, z); W[i][24] =
// alpha pin; W[i][25] = alpha e over state_0 (permutation i of the block).
__global__ void __launch_bounds__(256) k_keccak_w(const f128* __restrict__ e, f128 alpha, Shape S,
                                                  f128* __restrict__ W, f128* __restrict__ comb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < S.width * kWRows * kState) {
    const int sub = i / (kWRows * kState), r = i / kState % kWRows, p = i % kState;
    f128 v;
    if (r < 24) {
      const int l = p >> 6, zz = p & 63, x = l % 5, y5 = l - x;
      const f128* E = e + 64 * S.t_first(sub) + kState * r;
      v = fx(fmul(alpha, ldg(E + 64 * ((x + 4) % 5 + y5) + zz)), ldg(E + 64 * ((x + 3) % 5 + y5) + zz));
    } else {
      v = fmul(alpha, ldg(e + 64 * (r == 24 ? S.s24_word(sub) : S.s0_word(sub)) + p));
    }
    st(W + i, v);
  }
  // comb is written by the walkers on state_0 and t of every permutation
  const int t0 = 64 * S.t_word, t1 = 64 * S.t_first(S.width);
  for (int c = i; c < 64 * S.words; c += gridDim.x * blockDim.x) {
    const bool walked = (c < 64 * S.const_word && (c & 4095) < kState) || (c >= t0 && c < t1);
    if (!walked) st(comb + c, mk(0, 0));
  }
}

// One CTA: the transposed recurrence over 24 rounds (3 barriers a round).
// masks: 25 x 25 u64, masks[r] = phi(c_r) (r < 24), masks[24] = c_24.
// CTA i walks permutation i of the block.
constexpr int kWalkThreads = 800;  // two state positions per thread
__global__ void __launch_bounds__(kWalkThreads) k_keccak_walk(const f128* __restrict__ e, const f128* __restrict__ Wg,
                                                              const uint64_t* __restrict__ masks, f128 alpha,
                                                              f128 beta, Shape S, f128* __restrict__ comb) {
  extern __shared__ __align__(16) uint8_t wsm[];
  f128* K = reinterpret_cast<f128*>(wsm);  // [1600] the running K
  f128* U = K + kState;                    // [1600] K pulled back through rho-pi
  f128* D = U + kState;                    // [5][64] column sums of U
  __shared__ uint16_t dst[kState];         // rho-pi destination of each source position
  __shared__ f128 red[3][32];
  const int tid = threadIdx.x, sub = blockIdx.x;
  const f128* W = Wg + (size_t)sub * kWRows * kState;
  const int tb = 64 * S.t_first(sub), b0 = 64 * S.s0_word(sub), b24 = 64 * S.s24_word(sub);
  for (int q = tid; q < kState; q += kWalkThreads) {
    const int l = q >> 6, zz = q & 63, pa = l % 5, pb = l / 5;  // source (pa, pb, zz)
    const int dx = pb, dy = (2 * pa + 3 * pb) % 5, dz = (zz + kRho[5 * pa + pb]) & 63;
    dst[q] = (uint16_t)(64 * (dx + 5 * dy) + dz);
  }
  f128 acc = mk(0, 0), acc_row = mk(0, 0), acc_t = mk(0, 0);
  for (int p = tid; p < kState; p += kWalkThreads) {
    const f128 k = ldg(W + 24 * kState + p);
    K[p] = k;
    st(comb + tb + 23 * kState + p, k);
    if ((masks[24 * 25 + (p >> 6)] >> (p & 63)) & 1) acc = fx(acc, k);
    acc_row = fx(acc_row, fx(ldg(e + b0 + p), ldg(e + b24 + p)));  // state_0 and state_24 rows' B = [const]
  }
  for (int r = 23; r >= 0; r--) {
    for (int p = tid; p < kState; p += kWalkThreads) {
      const f128 w = ldg(W + r * kState + p);
      if ((masks[r * 25 + (p >> 6)] >> (p & 63)) & 1) acc = fx(acc, w);
      acc_t = fx(acc_t, ldg(e + tb + r * kState + p));
      K[p] = fx(K[p], w);
    }
    __syncthreads();
    for (int q = tid; q < kState; q += kWalkThreads) U[q] = K[dst[q]];
    __syncthreads();
    if (tid < 320) {
      const int x = tid >> 6, zz = tid & 63;
      f128 s = mk(0, 0);
#pragma unroll
      for (int y = 0; y < 5; y++) s = fx(s, U[64 * (x + 5 * y) + zz]);
      D[tid] = s;
    }
    __syncthreads();
    for (int k = tid; k < kState; k += kWalkThreads) {
      const int l = k >> 6, zz = k & 63, x = l % 5;
      const f128 v = fx(U[k], fx(D[64 * ((x + 1) % 5) + zz], D[64 * ((x + 4) % 5) + ((zz + 1) & 63)]));
      K[k] = v;
      if (r > 0) st(comb + tb + (r - 1) * kState + k, v);
      else st(comb + b0 + k, fx(v, ldg(W + 25 * kState + k)));
    }
    // the next round's update touches only this thread's own K entries; the
    // barrier after it orders them before the gather
  }
  acc = warp_xor(acc);
  acc_row = warp_xor(acc_row);
  acc_t = warp_xor(acc_t);
  if ((tid & 31) == 0) {
    red[0][tid >> 5] = acc;
    red[1][tid >> 5] = acc_row;
    red[2][tid >> 5] = acc_t;
  }
  __syncthreads();
  if (tid == 0) {
    f128 s0 = mk(0, 0), s1 = mk(0, 0), s2 = mk(0, 0);
    for (int w = 0; w < kWalkThreads / 32; w++) {
      s0 = fx(s0, red[0][w]);
      s1 = fx(s1, red[1][w]);
      s2 = fx(s2, red[2][w]);
    }
    // chi rows' A = 1 + B[x+1]: alpha sum E; the rows' B = [const] and the
    // round constants; once per block: the constant row (1, 1, 1),
    // (alpha + 1) e[const], and the pin beta
    f128 v = fx(fx(s0, s1), fmul(alpha, s2));
    if (sub == 0) {
      const f128 ec = ldg(e + 64 * S.const_word);
      v = fx(v, fx(fx(fmul(alpha, ec), ec), beta));
    }
    atomic_xor128(comb + 64 * S.const_word, v);
  }
}
constexpr size_t kWalkSmem = (2 * kState + 320) * sizeof(f128);

// masks[r] = phi(c_r) for r < 24 and masks[24] = c_24 (lanes), computed with
// the lane form of theta and rho-pi
std::vector<uint64_t> round_constant_masks() {
  std::vector<uint64_t> m(25 * 25, 0);
  uint64_t c[25] = {};
  for (int r = 0; r < 24; r++) {
    uint64_t col[5], th[25], out[25];
    for (int x = 0; x < 5; x++) col[x] = c[x] ^ c[x + 5] ^ c[x + 10] ^ c[x + 15] ^ c[x + 20];
    for (int l = 0; l < 25; l++) th[l] = c[l] ^ col[(l % 5 + 4) % 5] ^ rotl64(col[(l % 5 + 1) % 5], 1);
    for (int l = 0; l < 25; l++) {
      const int x = l % 5, y = l / 5, pa = (x + 3 * y) % 5, pb = x;
      out[l] = rotl64(th[pa + 5 * pb], kRhoHost[5 * pa + pb]);
    }
    for (int l = 0; l < 25; l++) m[r * 25 + l] = out[l];
    for (int l = 0; l < 25; l++) c[l] = out[l];
    c[0] ^= kRcHost[r];
  }
  for (int l = 0; l < 25; l++) m[24 * 25 + l] = c[l];
  return m;
}
}  // namespace

void launch_witness_keccak(const uint64_t* states, uint64_t seed, uint32_t n_perm, uint32_t n_slots, f128* z, f128* a,
                           f128* b, cudaStream_t s, int width) {
  const Shape S = shape_of(width);
  const uint64_t warps = (uint64_t)n_slots * S.width;
  count_launch();
  k_witness_keccak<<<(unsigned)((warps + kWarps - 1) / kWarps), 32 * kWarps, 0, s>>>(
      states, seed, n_perm, n_slots, S, reinterpret_cast<uint64_t*>(z), reinterpret_cast<uint64_t*>(a),
      reinterpret_cast<uint64_t*>(b));
}

const uint64_t* keccak_masks(int device) {
  static std::mutex mu;
  static std::map<int, uint64_t*> per_device;
  std::lock_guard<std::mutex> lk(mu);
  auto it = per_device.find(device);
  if (it != per_device.end()) return it->second;
  const std::vector<uint64_t> m = round_constant_masks();
  DeviceScope on(device);
  uint64_t* p = nullptr;
  CK(cudaMalloc(&p, m.size() * sizeof(uint64_t)));
  CK(cudaMemcpy(p, m.data(), m.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
  per_device[device] = p;
  return p;
}

size_t keccak_comb_scratch(int width) { return (size_t)shape_of(width).width * kWRows * kState; }

void keccak_comb(const f128* e, f128 alpha, f128 beta, const uint64_t* masks, f128* W, f128* comb, cudaStream_t s,
                 int width) {
  const Shape S = shape_of(width);
  count_launch(2);
  k_keccak_w<<<(S.width * kWRows * kState + 255) / 256, 256, 0, s>>>(e, alpha, S, W, comb);
  CK(cudaFuncSetAttribute(k_keccak_walk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWalkSmem));
  k_keccak_walk<<<S.width, kWalkThreads, kWalkSmem, s>>>(e, W, masks, alpha, beta, S, comb);
}
