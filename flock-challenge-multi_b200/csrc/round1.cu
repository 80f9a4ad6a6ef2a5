// K4: zerocheck round 1 (univariate skip over the 6 low row bits, extract-c
// form) — crates/flock-core/src/zerocheck/univariate_skip.rs:90-160 semantics:
//   P_AB(l) = sum_x eq(r_rest, x) phi8(a^_l(x) * b^_l(x))       l in Lambda
//   P_C(l)  = sum_s phi8(M[l][s]) * S_s,  S_s = sum_x eq(r_rest, x) c_s(x)
// where row x holds the 64 bits s of the skip block, a^_l = sum_s M[l][s] a_s
// is the GF(2^8) extension S -> Lambda, and C = I so c = z.
//
// B200 mapping.  A thread owns 8 consecutive rows (one value of the three
// "small" rest bits xs) of one 128-row block (xm = its 4 "medium" bits):
//  * the extension is a byte-window table lookup that returns the result
//    bit-sliced over l: 8 planes x 64 bits (plane i bit l = bit i of a^_l);
//  * a^ * b^ for all 64 l at once is a bit-sliced GF(2^8) product
//    (64 AND + 64 XOR, then the x^8 = x^4 + x^3 + x + 1 fold);
//  * eq over the three small bits is phi8(g(xs)) (fixed subfield constants,
//    univariate_skip_optimized.rs:136-215), so sum_xs g(xs) * v is formed in
//    GF(2^8) by compile-time XOR networks;
//  * eq over the four medium bits is C * x^xm: the 16 threads of a block
//    exchange their planes with warp ballots, giving per (l, plane k) a
//    16-bit polynomial W, and sum_xm x^xm phi8(u) = sum_k phi8(e_k) * W_k(x),
//    read from 8 x 256-entry tables of phi8(e_k) * v(x);
//  * one product by C * eq(r_hi, block) per (l, block) finishes the sum.
// The C column needs no extension: its eq-weighted bit sums are formed the
// same way (planes over s), kept apart by row bit 6 so that they are the
// c-claim's ring-switch statistic s_hat_v (pcs/ring_switch.rs:1594-1640 at
// the suffix r[7..m]), and extended once on the host.
#include "kernels.cuh"

namespace {
constexpr uint8_t gf8c(uint8_t a, uint8_t b) {
  uint32_t acc = 0;
  for (int i = 0; i < 8; i++)
    if ((a >> i) & 1) acc ^= (uint32_t)b << i;
  for (int i = 14; i >= 8; i--)
    if ((acc >> i) & 1) acc ^= 0x11Bu << (i - 8);
  return (uint8_t)acc;
}
constexpr uint8_t small_g(int xs) {  // eq(r[6..9], xs) = phi8(g(xs))
  const uint8_t s[3] = {0xF7, 0x53, 0xB5};
  uint8_t g = 1;
  for (int i = 0; i < 3; i++) g = gf8c(g, ((xs >> i) & 1) ? s[i] : (uint8_t)(1 ^ s[i]));
  return g;
}
// column j of the bit matrix of multiplication by g(xs): g(xs) * x^j
constexpr uint8_t gcol(int xs, int j) { return gf8c(small_g(xs), (uint8_t)(1u << j)); }

struct Round1Tables {
  uint64_t lde[8][256][8];  // [byte position][byte value][plane] bit l
  f128 tk[8][256];           // phi8(e_k) * v(x) for 8-bit polynomials v
};

__device__ __forceinline__ void lde(const Round1Tables* T, uint64_t row, uint64_t out[8]) {
#pragma unroll
  for (int i = 0; i < 8; i++) out[i] = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(T->lde[k][(row >> (8 * k)) & 0xFF]);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      ulonglong2 v = p[q];
      out[2 * q] ^= v.x;
      out[2 * q + 1] ^= v.y;
    }
  }
}

// bit-sliced GF(2^8) product of 64 element pairs
__device__ __forceinline__ void gf8_mul_sliced(const uint64_t A[8], const uint64_t B[8], uint64_t P[8]) {
  uint64_t c[15];
#pragma unroll
  for (int i = 0; i < 15; i++) c[i] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) c[i + j] ^= A[i] & B[j];
#pragma unroll
  for (int d = 14; d >= 8; d--) {
    c[d - 8] ^= c[d];
    c[d - 7] ^= c[d];
    c[d - 5] ^= c[d];
    c[d - 4] ^= c[d];
  }
#pragma unroll
  for (int i = 0; i < 8; i++) P[i] = c[i];
}

template <int XS>
__device__ __forceinline__ void gmul_acc(const uint64_t P[8], uint64_t U[8]) {
#pragma unroll
  for (int j = 0; j < 8; j++)
#pragma unroll
    for (int i = 0; i < 8; i++)
      if ((gcol(XS, j) >> i) & 1) U[i] ^= P[j];
}
// eq(r[7..9], xs >> 1) = phi8(g2(xs >> 1)): the C sums keep row bit 6 (xs & 1)
// apart, which makes them the ring-switch statistic s_hat_v of the c-claim
constexpr uint8_t small_g2(int xs2) {
  const uint8_t s[2] = {0x53, 0xB5};
  uint8_t g = 1;
  for (int i = 0; i < 2; i++) g = gf8c(g, ((xs2 >> i) & 1) ? s[i] : (uint8_t)(1 ^ s[i]));
  return g;
}
template <int XS>
__device__ __forceinline__ void cacc(uint64_t c, uint64_t Y0[8], uint64_t Y1[8]) {
#pragma unroll
  for (int k = 0; k < 8; k++)
    if ((small_g2(XS >> 1) >> k) & 1) {
      if (XS & 1) Y1[k] ^= c;
      else Y0[k] ^= c;
    }
}

template <int XS>
__device__ __forceinline__ void row_step(const Round1Tables* T, const uint64_t* __restrict__ a,
                                         const uint64_t* __restrict__ b, const uint64_t* __restrict__ c,
                                         size_t row0, uint64_t U[8], uint64_t Y0[8], uint64_t Y1[8]) {
  uint64_t A[8], B[8], P[8];
  lde(T, __ldg(a + row0 + XS), A);
  lde(T, __ldg(b + row0 + XS), B);
  gf8_mul_sliced(A, B, P);
  gmul_acc<XS>(P, U);
  cacc<XS>(__ldg(c + row0 + XS), Y0, Y1);
}

// ballot transpose of 8 planes: w[k] (for l = lane + 32 * hi) holds, in bits
// 0..15, block 2 warp's 16-bit polynomial and in bits 16..31 block 2 warp + 1's
__device__ __forceinline__ void transpose_planes(const uint64_t V[8], int lane, int hi, uint32_t w[8]) {
#pragma unroll
  for (int k = 0; k < 8; k++) {
    uint32_t keep = 0;
#pragma unroll
    for (int l = 0; l < 32; l++) {
      uint32_t m = __ballot_sync(0xffffffffu, (V[k] >> (l + 32 * hi)) & 1);
      keep = lane == l ? m : keep;
    }
    w[k] = keep;
  }
}

// W planes -> sum_k phi8(e_k) W_k(x), W_k = 16-bit polynomial (lo | hi << 8)
__device__ __forceinline__ f128 fold_w(const Round1Tables* T, const uint32_t w[8], int shift) {
  f128 lo = mk(0, 0), hi = mk(0, 0);
#pragma unroll
  for (int k = 0; k < 8; k++) {
    uint32_t v = (w[k] >> shift) & 0xFFFF;
    lo = fx(lo, ld(&T->tk[k][v & 0xFF]));
    hi = fx(hi, ld(&T->tk[k][v >> 8]));
  }
  return fx(lo, mul_xk(hi, 8));
}
}  // namespace

size_t round1_tables_size() { return sizeof(Round1Tables); }

// out[0..64) += P_AB; out[64 + 64 h + s] += sum_i eq(r[7..m], i) bit_(s+64h)(z_i)
// (the c-claim ring-switch statistic; C is extended from it on the host)
__global__ void __launch_bounds__(256) k_zc_round1(const uint64_t* __restrict__ a, const uint64_t* __restrict__ b,
                                                   const uint64_t* __restrict__ c, const Round1Tables* __restrict__ tabs,
                                                   const f128* __restrict__ eqc, size_t n_blocks, f128* __restrict__ out) {
  extern __shared__ __align__(16) uint8_t sm[];
  Round1Tables* T = reinterpret_cast<Round1Tables*>(sm);
  {
    const uint4* src = reinterpret_cast<const uint4*>(tabs);
    uint4* dst = reinterpret_cast<uint4*>(sm);
    for (int i = threadIdx.x; i < (int)(sizeof(Round1Tables) / 16); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u256 acc[6];
#pragma unroll
  for (int q = 0; q < 6; q++) acc[q] = zero256();
  for (size_t blk16 = blockIdx.x; blk16 * 16 < n_blocks; blk16 += gridDim.x) {
    const size_t blk = blk16 * 16 + 2 * warp + (lane >> 4);
    const int xm = lane & 15;
    const size_t row0 = blk * 128 + (size_t)xm * 8;
    uint64_t U[8], Y0[8], Y1[8];
#pragma unroll
    for (int i = 0; i < 8; i++) { U[i] = 0; Y0[i] = 0; Y1[i] = 0; }
    row_step<0>(T, a, b, c, row0, U, Y0, Y1);
    row_step<1>(T, a, b, c, row0, U, Y0, Y1);
    row_step<2>(T, a, b, c, row0, U, Y0, Y1);
    row_step<3>(T, a, b, c, row0, U, Y0, Y1);
    row_step<4>(T, a, b, c, row0, U, Y0, Y1);
    row_step<5>(T, a, b, c, row0, U, Y0, Y1);
    row_step<6>(T, a, b, c, row0, U, Y0, Y1);
    row_step<7>(T, a, b, c, row0, U, Y0, Y1);
    const size_t bA = blk16 * 16 + 2 * warp;
    const f128 eA = ldg(eqc + bA), eB = ldg(eqc + bA + 1);
    uint32_t w[8];
    transpose_planes(U, lane, 0, w);
    acc_wide(acc[0], mul_wide(fold_w(T, w, 0), eA));
    acc_wide(acc[0], mul_wide(fold_w(T, w, 16), eB));
    transpose_planes(U, lane, 1, w);
    acc_wide(acc[1], mul_wide(fold_w(T, w, 0), eA));
    acc_wide(acc[1], mul_wide(fold_w(T, w, 16), eB));
    transpose_planes(Y0, lane, 0, w);
    acc_wide(acc[2], mul_wide(fold_w(T, w, 0), eA));
    acc_wide(acc[2], mul_wide(fold_w(T, w, 16), eB));
    transpose_planes(Y0, lane, 1, w);
    acc_wide(acc[3], mul_wide(fold_w(T, w, 0), eA));
    acc_wide(acc[3], mul_wide(fold_w(T, w, 16), eB));
    transpose_planes(Y1, lane, 0, w);
    acc_wide(acc[4], mul_wide(fold_w(T, w, 0), eA));
    acc_wide(acc[4], mul_wide(fold_w(T, w, 16), eB));
    transpose_planes(Y1, lane, 1, w);
    acc_wide(acc[5], mul_wide(fold_w(T, w, 0), eA));
    acc_wide(acc[5], mul_wide(fold_w(T, w, 16), eB));
  }
#pragma unroll
  for (int q = 0; q < 6; q++) atomic_xor128(out + 32 * q + lane, reduce(acc[q]));
}

void zc_round1(const f128* a, const f128* b, const f128* c, const void* tabs, const f128* eqc, size_t n_blocks,
               f128* out, int grid, cudaStream_t s) {
  size_t smem = sizeof(Round1Tables);
  CK(cudaFuncSetAttribute(k_zc_round1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  count_launch();
  k_zc_round1<<<grid, 256, smem, s>>>((const uint64_t*)a, (const uint64_t*)b, (const uint64_t*)c,
                                      (const Round1Tables*)tabs, eqc, n_blocks, out);
}

// Host construction of the tables from the S -> Lambda matrix M[l][s] and phi8.
void build_round1_tables_host(const uint8_t M[64][64], const f128* phi8, void* dst) {
  Round1Tables* T = reinterpret_cast<Round1Tables*>(dst);
  memset(T, 0, sizeof(Round1Tables));
  for (int k = 0; k < 8; k++)
    for (int v = 0; v < 256; v++)
      for (int l = 0; l < 64; l++) {
        uint8_t e = 0;
        for (int j = 0; j < 8; j++)
          if ((v >> j) & 1) e ^= M[l][8 * k + j];
        for (int i = 0; i < 8; i++)
          if ((e >> i) & 1) T->lde[k][v][i] |= 1ull << l;
      }
  for (int k = 0; k < 8; k++)
    for (int v = 0; v < 256; v++) {
      // phi8(e_k) * v(x): shift-and-add of the 8 coefficients of v
      f128 base = phi8[1 << k], acc = mk(0, 0);
      for (int j = 0; j < 8; j++)
        if ((v >> j) & 1) acc = fx(acc, mul_xk(base, j));
      T->tk[k][v] = acc;
    }
}
