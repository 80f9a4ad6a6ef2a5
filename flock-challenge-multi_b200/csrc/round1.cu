// K4: zerocheck round 1 (univariate skip over the 6 low row bits, extract-c
// form) — crates/flock-core/src/zerocheck/univariate_skip.rs:90-160 semantics:
//   P_AB(l) = sum_x eq(r_rest, x) phi8(a^_l(x) * b^_l(x))       l in Lambda
//   P_C(l)  = sum_s phi8(M[l][s]) * S_s,  S_s = sum_x eq(r_rest, x) c_s(x)
// where row x holds the 64 bits s of the skip block, a^_l = sum_s M[l][s] a_s
// is the GF(2^8) extension S -> Lambda, and C = I so c = z.
//
// B200 mapping.  A thread owns one row group g = (128-row block, xm = the 4
// "medium" row bits): 8 consecutive rows, one per value of the 3 "small" bits
// xs.  The eq weight of row (g, xs) factors as E(g) * phi8(gs(xs)) with
// E(g) = C * eq(r_hi, block) * x^xm (the medium challenges make eq over xm
// equal to C * x^xm) and gs(xs) a fixed GF(2^8) constant
// (univariate_skip_optimized.rs:136-215).
//  * The extension is a byte-window table lookup that returns a^_l for all 64
//    l bit-sliced (8 planes x 64 bits).  Windows are 7 bits wide (the last 8)
//    and every 64-byte entry is stored twice in a 128-byte slot row; lane L
//    reads its four 16-byte chunks in the order rotated by L mod 4 from the
//    copy picked by bit 2 of L, so the 8 lanes of every quarter warp hit 8
//    distinct 16-byte bank groups whatever the data: no bank conflicts.
//  * a^ * b^ for all 64 l is a bit-sliced GF(2^8) product and
//    U = sum_xs gs(xs) * P(xs) a compile-time XOR network.
//  * phi8 is GF(2)-linear, so
//      P_AB(l) = sum_k phi8(e_k) H(l, k),  H(l, k) = XOR_g bit_k(U_l(g)) E(g):
//    a warp transposes its planes (shuffle butterflies) so lane l' holds, per
//    plane k, the 32 bits of l = l' (+32) over the warp's 32 row groups, and
//    XORs E(g) in through 4-bit subset-sum tables of the group's E values.
//    No GF(2^128) product is formed per row group; the 8 x 64 products by
//    phi8(e_k) are done once on the host.
// The C column needs no extension: with gs2 the 2-bit weights of xs >> 1,
//    S_(s + 64 h) = sum_j phi8(gs2(j)) H_C(s, h, j),
//    H_C(s, h, j) = XOR_g bit_s(c(g, 2 j + h)) E(g),
// which keeps row bit 6 (h) apart: these are the c-claim's ring-switch
// statistic s_hat_v (pcs/ring_switch.rs:1594-1640 at the suffix r[7..m]).
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

// extension tables: windows 0..7 cover row bits [7p, 7p + 7), window 8 bits
// [56, 64); entry = 8 slots of 16 bytes, slots c and c + 4 hold chunk c
// (planes 2c, 2c + 1 of a^ for the window's bits)
constexpr int kWin7 = 128 * 128;               // bytes per 7-bit window
constexpr int kLdeBytes = 8 * kWin7 + 256 * 128;  // 160 KiB
constexpr int kSubsetBytes = 8 * 16 * 16;      // per warp: 8 groups x 16 subset sums
constexpr int kWarps = 8;

struct Lanes {
  uint32_t off[4];  // byte offset of the slot holding the chunk read at step q
  uint32_t keep[5], sh[5];  // butterfly transpose masks and rotate amounts
  bool r1, r2;
};

__device__ __forceinline__ Lanes lanes_of(int lane) {
  Lanes L;
  const int r = lane & 3, half = (lane >> 2) & 1;
#pragma unroll
  for (int q = 0; q < 4; q++) L.off[q] = (uint32_t)((((q + r) & 3) + 4 * half) * 16);
  const uint32_t M[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int t = 0; t < 5; t++) {
    const int j = 16 >> t;
    L.keep[t] = (lane & j) ? ~M[t] : M[t];
    L.sh[t] = (lane & j) ? j : 32 - j;
  }
  L.r1 = lane & 1;
  L.r2 = lane & 2;
  return L;
}

// 32 x 32 bit transpose across the warp: lane c receives bit L of its result
// from bit c of lane L's x
__device__ __forceinline__ uint32_t transpose32(uint32_t x, const Lanes& L) {
#pragma unroll
  for (int t = 0; t < 5; t++) {
    const int j = 16 >> t;
    uint32_t s = x & ~L.keep[t];
    s = __funnelshift_l(s, s, L.sh[t]);
    x = (x & L.keep[t]) | __shfl_xor_sync(0xffffffffu, s, j);
  }
  return x;
}

__device__ __forceinline__ void lde(const uint8_t* sm, const Lanes& L, uint64_t row, uint64_t out[8]) {
  ulonglong2 acc[4];
#pragma unroll
  for (int q = 0; q < 4; q++) acc[q] = make_ulonglong2(0, 0);
#pragma unroll
  for (int p = 0; p < 9; p++) {
    const uint32_t v = p < 8 ? (uint32_t)(row >> (7 * p)) & 127u : (uint32_t)(row >> 56);
    const uint8_t* base = sm + (p < 8 ? p * kWin7 : 8 * kWin7) + v * 128u;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      ulonglong2 t = *reinterpret_cast<const ulonglong2*>(base + L.off[q]);
      acc[q].x ^= t.x;
      acc[q].y ^= t.y;
    }
  }
  // acc[q] holds chunk (q + lane) mod 4: undo the rotation
  ulonglong2 t0 = L.r1 ? acc[3] : acc[0], t1 = L.r1 ? acc[0] : acc[1];
  ulonglong2 t2 = L.r1 ? acc[1] : acc[2], t3 = L.r1 ? acc[2] : acc[3];
  ulonglong2 u0 = L.r2 ? t2 : t0, u1 = L.r2 ? t3 : t1, u2 = L.r2 ? t0 : t2, u3 = L.r2 ? t1 : t3;
  out[0] = u0.x; out[1] = u0.y; out[2] = u1.x; out[3] = u1.y;
  out[4] = u2.x; out[5] = u2.y; out[6] = u3.x; out[7] = u3.y;
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

template <int XS>
__device__ __forceinline__ void row_step(const uint8_t* sm, const Lanes& L, uint64_t a, uint64_t b, uint64_t U[8]) {
  uint64_t A[8], B[8], P[8];
  lde(sm, L, a, A);
  lde(sm, L, b, B);
  gf8_mul_sliced(A, B, P);
  gmul_acc<XS>(P, U);
}

// E(g) of this lane's row group into the warp's 4-bit subset-sum tables:
// table n (lanes 4n..4n+3), entry v = XOR of E(4n + i) over the set bits i of v
__device__ __forceinline__ void build_subsets(f128 E, int lane, f128* T) {
  const int n = lane >> 2, i = lane & 3;
  f128 e[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    e[j].lo = __shfl_sync(0xffffffffu, E.lo, 4 * n + j);
    e[j].hi = __shfl_sync(0xffffffffu, E.hi, 4 * n + j);
  }
  f128 base = mk(0, 0);
  if (i & 1) base = fx(base, e[2]);
  if (i & 2) base = fx(base, e[3]);
  f128* t = T + n * 16 + 4 * i;
  st(t + 0, base);
  st(t + 1, fx(base, e[0]));
  st(t + 2, fx(base, e[1]));
  st(t + 3, fx(fx(base, e[0]), e[1]));
}

// acc ^= XOR of E(g) over the lanes g whose bit is set in w
__device__ __forceinline__ void accumulate(const uint8_t* T, uint32_t w, f128& acc) {
#pragma unroll
  for (int n = 0; n < 8; n++) {
    const f128 v = ld(reinterpret_cast<const f128*>(T + n * 256 + ((w >> (4 * n)) & 15u) * 16));
    acc = fx(acc, v);
  }
}

__device__ __forceinline__ f128 group_weight(const f128* __restrict__ eqc, size_t blk, int xm) {
  return mul_xk(ldg(eqc + blk), xm);
}

// per-CTA XOR of the 8 warps' accumulators (through the table area), then one
// atomic per output word: out[idx(lane, hi, t)] for t < NT
template <int NT>
__device__ __forceinline__ void flush(uint8_t* sm, const f128 (&H)[NT][2], int warp, int lane, f128* out) {
  __syncthreads();
  f128* R = reinterpret_cast<f128*>(sm);  // [warp][t][hi][lane]
#pragma unroll
  for (int t = 0; t < NT; t++)
#pragma unroll
    for (int hi = 0; hi < 2; hi++) st(R + ((warp * NT + t) * 2 + hi) * 32 + lane, H[t][hi]);
  __syncthreads();
  for (int i = threadIdx.x; i < NT * 64; i += blockDim.x) {
    f128 v = mk(0, 0);
    for (int w = 0; w < kWarps; w++) v = fx(v, ld(R + w * NT * 64 + i));
    const int t = i / 64, hi = (i / 32) & 1, ln = i & 31;
    atomic_xor128(out + (size_t)(ln + 32 * hi) * NT + t, v);
  }
}
}  // namespace

size_t round1_tables_size() { return kLdeBytes; }

// out[l * 8 + k] ^= H(l, k) for this kernel's row groups
__global__ void __launch_bounds__(256, 1) k_zc_round1_ab(const uint64_t* __restrict__ a,
                                                         const uint64_t* __restrict__ b,
                                                         const uint8_t* __restrict__ tabs,
                                                         const f128* __restrict__ eqc, size_t n_blocks,
                                                         f128* __restrict__ out) {
  extern __shared__ __align__(128) uint8_t sm[];
  {
    const uint4* src = reinterpret_cast<const uint4*>(tabs);
    uint4* dst = reinterpret_cast<uint4*>(sm);
    for (int i = threadIdx.x; i < kLdeBytes / 16; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const Lanes L = lanes_of(lane);
  f128* T = reinterpret_cast<f128*>(sm + kLdeBytes + warp * kSubsetBytes);
  f128 H[8][2];
#pragma unroll
  for (int k = 0; k < 8; k++) H[k][0] = H[k][1] = mk(0, 0);
  for (size_t blk16 = blockIdx.x; blk16 * 16 < n_blocks; blk16 += gridDim.x) {
    const size_t blk = blk16 * 16 + 2 * warp + (lane >> 4);
    const int xm = lane & 15;
    const ulonglong2* pa = reinterpret_cast<const ulonglong2*>(a + blk * 128 + (size_t)xm * 8);
    const ulonglong2* pb = reinterpret_cast<const ulonglong2*>(b + blk * 128 + (size_t)xm * 8);
    uint64_t U[8];
#pragma unroll
    for (int i = 0; i < 8; i++) U[i] = 0;
    {
      ulonglong2 ra = __ldg(pa), rb = __ldg(pb);
      row_step<0>(sm, L, ra.x, rb.x, U);
      row_step<1>(sm, L, ra.y, rb.y, U);
      ra = __ldg(pa + 1); rb = __ldg(pb + 1);
      row_step<2>(sm, L, ra.x, rb.x, U);
      row_step<3>(sm, L, ra.y, rb.y, U);
      ra = __ldg(pa + 2); rb = __ldg(pb + 2);
      row_step<4>(sm, L, ra.x, rb.x, U);
      row_step<5>(sm, L, ra.y, rb.y, U);
      ra = __ldg(pa + 3); rb = __ldg(pb + 3);
      row_step<6>(sm, L, ra.x, rb.x, U);
      row_step<7>(sm, L, ra.y, rb.y, U);
    }
    __syncwarp();  // the previous iteration's subset tables are no longer read
    build_subsets(group_weight(eqc, blk, xm), lane, T);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 8; k++)
#pragma unroll
      for (int hi = 0; hi < 2; hi++)
        accumulate(reinterpret_cast<const uint8_t*>(T), transpose32((uint32_t)(U[k] >> (32 * hi)), L), H[k][hi]);
  }
  flush<8>(sm, H, warp, lane, out);
}

// out[s * 8 + 4 h + j] ^= H_C(s, h, j) for this kernel's row groups
__global__ void __launch_bounds__(256) k_zc_round1_c(const uint64_t* __restrict__ c, const f128* __restrict__ eqc,
                                                     size_t n_blocks, f128* __restrict__ out) {
  extern __shared__ __align__(128) uint8_t sm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const Lanes L = lanes_of(lane);
  f128* T = reinterpret_cast<f128*>(sm + warp * kSubsetBytes);
  f128 H[8][2];
#pragma unroll
  for (int k = 0; k < 8; k++) H[k][0] = H[k][1] = mk(0, 0);
  for (size_t blk16 = blockIdx.x; blk16 * 16 < n_blocks; blk16 += gridDim.x) {
    const size_t blk = blk16 * 16 + 2 * warp + (lane >> 4);
    const int xm = lane & 15;
    const ulonglong2* pc = reinterpret_cast<const ulonglong2*>(c + blk * 128 + (size_t)xm * 8);
    uint64_t r[8];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      ulonglong2 v = __ldg(pc + i);
      r[2 * i] = v.x;
      r[2 * i + 1] = v.y;
    }
    __syncwarp();
    build_subsets(group_weight(eqc, blk, xm), lane, T);
    __syncwarp();
    // slot t = 4 h + j holds row xs = 2 j + h
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int hi = 0; hi < 2; hi++)
          accumulate(reinterpret_cast<const uint8_t*>(T), transpose32((uint32_t)(r[2 * j + h] >> (32 * hi)), L),
                     H[4 * h + j][hi]);
  }
  flush<8>(sm, H, warp, lane, out);
}

void zc_round1(const f128* a, const f128* b, const f128* c, const void* tabs, const f128* eqc, size_t n_blocks,
               f128* out, int grid, cudaStream_t s) {
  if (n_blocks % 16) throw CudaError("zc_round1: block count not a multiple of 16");
  const int smem_ab = kLdeBytes + kWarps * kSubsetBytes;
  const int smem_c = 8 * 2 * 32 * 16 * kWarps > kWarps * kSubsetBytes ? 8 * 2 * 32 * 16 * kWarps
                                                                        : kWarps * kSubsetBytes;
  CK(cudaFuncSetAttribute(k_zc_round1_ab, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_ab));
  CK(cudaFuncSetAttribute(k_zc_round1_c, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_c));
  count_launch();
  k_zc_round1_ab<<<grid, 256, smem_ab, s>>>((const uint64_t*)a, (const uint64_t*)b, (const uint8_t*)tabs, eqc,
                                            n_blocks, out);
  count_launch();
  k_zc_round1_c<<<2 * grid, 256, smem_c, s>>>((const uint64_t*)c, eqc, n_blocks, out + 512);
}

// Host construction of the extension tables from the S -> Lambda matrix M[l][s].
void build_round1_tables_host(const uint8_t M[64][64], const f128* phi8, void* dst) {
  (void)phi8;
  uint8_t* T = reinterpret_cast<uint8_t*>(dst);
  memset(T, 0, kLdeBytes);
  for (int p = 0; p < 9; p++) {
    const int bits = p < 8 ? 7 : 8, s0 = 7 * p;
    uint8_t* W = T + (p < 8 ? p * kWin7 : 8 * kWin7);
    for (int v = 0; v < (1 << bits); v++) {
      uint64_t planes[8] = {};
      for (int l = 0; l < 64; l++) {
        uint8_t e = 0;
        for (int j = 0; j < bits; j++)
          if ((v >> j) & 1) e ^= M[l][s0 + j];
        for (int i = 0; i < 8; i++)
          if ((e >> i) & 1) planes[i] |= 1ull << l;
      }
      for (int c = 0; c < 4; c++) {
        memcpy(W + v * 128 + c * 16, &planes[2 * c], 16);
        memcpy(W + v * 128 + (c + 4) * 16, &planes[2 * c], 16);
      }
    }
  }
}
