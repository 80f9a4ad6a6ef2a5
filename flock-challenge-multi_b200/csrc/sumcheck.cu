// K3-K8: the sumcheck-family kernels of the prover.
//
//  K3 eq tables:        eq(r, x) = prod_i (x_i ? r_i : 1 + r_i), bit i of x <-> r_i
//                       (zerocheck/univariate_skip.rs:31-87, lincheck.rs:2080-2125);
//                       materialised as lo[x & mask] * hi[x >> s].
//  K4 zerocheck round 1 (univariate skip over the 6 low bits, extract-c form):
//                       P_AB(l) = sum_x eq(r_rest, x) phi8(a^_l(x) b^_l(x)),
//                       P_C(l)  = sum_x eq(r_rest, x) phi8(c^_l(x)), l in Lambda
//                       (univariate_skip.rs:90-160).  The first seven rest
//                       variables carry the fixed inner challenges
//                       (univariate_skip_optimized.rs:136-233): three phi8
//                       subfield constants and four gamma^(2^i)/(1+gamma^(2^i)),
//                       so eq on a 128-row block is phi8(g(xs)) * C * gamma^xm:
//                       the small part is folded in GF(2^8), the medium part is a
//                       shift by xm bits, one general product per block and l.
//  K5 zerocheck multilinear rounds: message (G(1), G(inf)) of
//                       G(X) = sum eq(.) a^(X,.) b^(X,.), LSB binding, fused with
//                       the fold of the previous round (zerocheck.rs:1735-1795,
//                       multilinear.rs:575-657,3194-3330).
//  K6 lincheck:         comb = alpha A^T eq + B^T eq (CSC gather; lincheck.rs:175-200),
//                       z_vec[c] = sum_o eq(x_outer, o) z[c + 2^14 o],
//                       8 top-binding product-sumcheck rounds (lincheck.rs:4968-4990,5880-6050).
//  K7 ring switch:      s_hat_v[r] = sum_i eq(i) bit_r(z_i) (ring_switch.rs:1594-1640);
//                       b_combined[i] = sum_k gamma_k sum_b bit_b(eq_k(i)) eq''_k[b]
//                       (ring_switch.rs:1952-2130, pcs.rs:778-1290).
//  K8 Ligerito:         round messages u0 = sum f0 b0, u2 = sum (f0+f1)(b0+b1) and
//                       LSB folds (pcs/ligerito.rs:4923-5020, 8894-9100).
#include "kernels.cuh"
#include <algorithm>

namespace {
}  // namespace

// ------------------------------------------------------------------ K3 --
__global__ void k_eq_split(const f128* __restrict__ lo, const f128* __restrict__ hi, int s, size_t n,
                           f128* __restrict__ out) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  st(out + i, fmul(ldg(lo + (i & ((1ull << s) - 1))), ldg(hi + (i >> s))));
}

// eq tables built on the device: out[i] = scale * prod_j (bit j of i ? r_j : 1 + r_j)
// (the same values as the doubling construction of eq(r, .), field products
// being exact)
struct EqVec {
  f128 r[24];
  f128 scale;
  int n;
};
__global__ void k_eq_build(EqVec E, f128* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ((size_t)1 << E.n)) return;
  f128 v = E.scale;
  for (int j = 0; j < E.n; j++) v = fmul(v, ((i >> j) & 1) ? E.r[j] : fx(E.r[j], mk(1, 0)));
  st(out + i, v);
}

// out[s + 64 k] = L[s] * e[k]
struct Vec64 {
  f128 v[64];
};
__global__ void k_outer64(Vec64 L, const f128* __restrict__ e, size_t n_e, f128* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 64 * n_e) return;
  st(out + i, fmul(L.v[i & 63], ldg(e + (i >> 6))));
}

// out[i] += beta * x[i]
__global__ void k_axpy(f128* __restrict__ out, const f128* __restrict__ x, f128 beta, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  st(out + i, fx(ld(out + i), fmul(ld(x + i), beta)));
}

// out[0] ^= sum_i f[i] g[i]
__global__ void k_inner(const f128* __restrict__ f, const f128* __restrict__ g, size_t n, f128* out) {
  u256 acc = zero256();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    acc_wide(acc, mul_wide(ld(f + i), ld(g + i)));
  block_xor_out(reduce(acc), out);
}

// ------------------------------------------------------------------ K5 --
// last fold: 2 -> 1 values per vector
__global__ void k_fold_pair_final(const f128* a_in, const f128* b_in, f128 rho, f128* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    f128 a0 = a_in[0], a1 = a_in[1], b0 = b_in[0], b1 = b_in[1];
    out[0] = fx(a0, fmul(rho, fx(a0, a1)));
    out[1] = fx(b0, fmul(rho, fx(b0, b1)));
  }
}

void fold_pair_final(const f128* a_in, const f128* b_in, f128 rho, f128* out, cudaStream_t s) {
  count_launch(); k_fold_pair_final<<<1, 32, 0, s>>>(a_in, b_in, rho, out);
}

// ------------------------------------------------------------------ K6 --
// comb[c] = alpha * (A^T eq)[c] + (B^T eq)[c] (+ beta at the pinned column):
// one warp per column, its lanes striding over the column's nonzeros
// (CSC row indices) and XOR-reducing by shuffles.
__global__ void __launch_bounds__(256) k_lc_comb(const uint32_t* __restrict__ at_ptr,
                                                 const uint16_t* __restrict__ at_row,
                                                 const uint32_t* __restrict__ bt_ptr,
                                                 const uint16_t* __restrict__ bt_row, const f128* __restrict__ eq,
                                                 f128 alpha, f128 beta, int pin, int k, f128* __restrict__ comb) {
  const int c = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= k) return;
  f128 sa = mk(0, 0), sb = mk(0, 0);
  for (uint32_t j = at_ptr[c] + lane; j < at_ptr[c + 1]; j += 32) sa = fx(sa, ldg(eq + at_row[j]));
  for (uint32_t j = bt_ptr[c] + lane; j < bt_ptr[c + 1]; j += 32) sb = fx(sb, ldg(eq + bt_row[j]));
  sa = warp_xor(sa);
  sb = warp_xor(sb);
  if (lane == 0) {
    f128 v = fx(fmul(alpha, sa), sb);
    if (c == pin) v = fx(v, beta);
    st(comb + c, v);
  }
}

// z_vec[i] = XOR over compressions o of eq(x_outer, o) where bit i of o's
// 2^k_log-bit block is set (lincheck.rs:2423 partial_fold_packed_z_block_major).
// A CTA owns 4096 bit positions (a quarter of a 2^14-bit block, an eighth of
// a 2^15-bit one) and a run of compressions; a thread owns 16 positions (one
// u16 of each block).  For
// every 8 compressions the CTA builds the 256 subset sums of their eq
// weights; a thread transposes its 8 u16 words into 16 bytes (bit k of byte
// p = bit p of compression k) and XORs in one table entry per position.
namespace {
constexpr int kZvGroups = 8;  // 8-compression tables built per barrier pair

__device__ __forceinline__ uint64_t transpose8x8(uint64_t x) {
  uint64_t t;
  t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
  x = x ^ t ^ (t << 7);
  t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
  x = x ^ t ^ (t << 14);
  t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
  x = x ^ t ^ (t << 28);
  return x;
}
}  // namespace

__global__ void __launch_bounds__(256) k_lc_zvec(const uint16_t* __restrict__ z, const f128* __restrict__ eqo,
                                                 size_t n_outer, int chunk, int bw, f128* __restrict__ zv) {
  __shared__ __align__(16) f128 T[kZvGroups][256];
  const int col = blockIdx.x;  // 4096-bit column of the block (bw u16 per block)
  const int t = threadIdx.x;
  const size_t o0 = (size_t)blockIdx.y * chunk;
  const size_t o1 = o0 + chunk < n_outer ? o0 + chunk : n_outer;
  f128 acc[16];
#pragma unroll
  for (int p = 0; p < 16; p++) acc[p] = mk(0, 0);
  for (size_t ob = o0; ob < o1; ob += 8 * kZvGroups) {
    __syncthreads();
    // entry v of table g: XOR of eq(o) over the set bits k of v, o = ob + 8g + k
#pragma unroll 1
    for (int g = 0; g < kZvGroups; g++) {
      f128 v = mk(0, 0);
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const size_t o = ob + 8 * g + k;
        if (((t >> k) & 1) && o < o1) v = fx(v, ldg(eqo + o));
      }
      st(&T[g][t], v);
    }
    __syncthreads();
    // the next group's words are loaded while the current one is folded in
    uint32_t r[8], rn[8];
#pragma unroll
    for (int k = 0; k < 8; k++) r[k] = ob + k < o1 ? z[(ob + k) * bw + col * 256 + t] : 0u;
#pragma unroll 1
    for (int g = 0; g < kZvGroups; g++) {
      const size_t og = ob + 8 * g;
      if (og >= o1) break;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const size_t o = og + 8 + k;
        rn[k] = (g + 1 < kZvGroups && o < o1) ? z[o * bw + col * 256 + t] : 0u;
      }
      const uint32_t t01 = __byte_perm(r[0], r[1], 0x5140), t23 = __byte_perm(r[2], r[3], 0x5140);
      const uint32_t t45 = __byte_perm(r[4], r[5], 0x5140), t67 = __byte_perm(r[6], r[7], 0x5140);
      const uint64_t lo = transpose8x8((uint64_t)__byte_perm(t01, t23, 0x5410) |
                                       ((uint64_t)__byte_perm(t45, t67, 0x5410) << 32));
      const uint64_t hi = transpose8x8((uint64_t)__byte_perm(t01, t23, 0x7632) |
                                       ((uint64_t)__byte_perm(t45, t67, 0x7632) << 32));
#pragma unroll
      for (int p = 0; p < 8; p++) {
        acc[p] = fx(acc[p], ld(&T[g][(lo >> (8 * p)) & 0xFF]));
        acc[8 + p] = fx(acc[8 + p], ld(&T[g][(hi >> (8 * p)) & 0xFF]));
      }
#pragma unroll
      for (int k = 0; k < 8; k++) r[k] = rn[k];
    }
  }
#pragma unroll
  for (int p = 0; p < 16; p++) atomic_xor128(zv + col * 4096 + 16 * t + p, acc[p]);
}

// One lincheck round (top binding): with do_fold, fold comb and zv (2 len
// values each) at r into their first len values; with emit, add the
// message over the (folded) pairs (i, i + len/2) into out[0..2):
// q1 = sum c1 z1, qinf = sum (c0 + c1)(z0 + z1).  Thread i < len/2 owns
// outputs i and i + len/2 and reads exactly the four inputs that fold into
// them, so the grid needs no synchronisation; the message is XOR-reduced per
// CTA and added atomically (out must be zero).
__global__ void __launch_bounds__(256) k_lc_round(f128* comb, f128* zv, int len, int do_fold, f128 r, int emit,
                                                  f128* out) {
  const int h = len >> 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  f128 q1 = mk(0, 0), qi = mk(0, 0);
  if (i < h) {
    f128 c0 = comb[i], c1 = comb[i + h], z0 = zv[i], z1 = zv[i + h];
    if (do_fold) {
      const f128 c0h = comb[i + len], c1h = comb[i + h + len], z0h = zv[i + len], z1h = zv[i + h + len];
      c0 = fx(c0, fmul(r, fx(c0h, c0)));
      c1 = fx(c1, fmul(r, fx(c1h, c1)));
      z0 = fx(z0, fmul(r, fx(z0h, z0)));
      z1 = fx(z1, fmul(r, fx(z1h, z1)));
      comb[i] = c0;
      comb[i + h] = c1;
      zv[i] = z0;
      zv[i + h] = z1;
    }
    if (emit) {
      q1 = fmul(c1, z1);
      qi = fmul(fx(c0, c1), fx(z0, z1));
    }
  }
  if (!emit) return;
  block_xor_out(q1, out);
  block_xor_out(qi, out + 1);
}

void lc_comb(const uint32_t* at_ptr, const uint16_t* at_row, const uint32_t* bt_ptr, const uint16_t* bt_row,
             const f128* eq, f128 alpha, f128 beta, int pin, int k, f128* comb, cudaStream_t s) {
  count_launch();
  k_lc_comb<<<k * 32 / 256, 256, 0, s>>>(at_ptr, at_row, bt_ptr, bt_row, eq, alpha, beta, pin, k, comb);
}
void lc_zvec(const f128* z, const f128* eqo, size_t n_outer, int k_log, f128* zv, int sms, cudaStream_t s) {
  // compressions per CTA (a multiple of 64), sized so that the columns x
  // chunks fill one wave of resident CTAs
  const size_t cols = (size_t)1 << (k_log - 12);
  const size_t slots = (size_t)resident_grid((const void*)k_lc_zvec, 256, 0, sms);
  const size_t rows = std::max<size_t>(1, slots / cols);
  const size_t chunk = std::max<size_t>(64, ((n_outer + rows - 1) / rows + 63) / 64 * 64);
  dim3 grid((unsigned)cols, (unsigned)((n_outer + chunk - 1) / chunk));
  count_launch();
  k_lc_zvec<<<grid, 256, 0, s>>>((const uint16_t*)z, eqo, n_outer, (int)chunk, 1 << (k_log - 4), zv);
}
void lc_round(f128* comb, f128* zv, int len, bool fold, f128 r, bool emit, f128* out, cudaStream_t s) {
  const int threads = std::max(1, len / 2);
  count_launch();
  k_lc_round<<<(threads + 255) / 256, 256, 0, s>>>(comb, zv, len, fold, r, emit, out);
}

// ------------------------------------------------------------------ K7 --
// ------------------------------------------------------------------ K8 --
__global__ void __launch_bounds__(256) k_lig_msg(const f128* __restrict__ f, const f128* __restrict__ b,
                                                 size_t n_pairs, f128* __restrict__ out) {
  u256 u0 = zero256(), u2 = zero256();
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_pairs; j += (size_t)gridDim.x * blockDim.x) {
    f128 f0 = ld(f + 2 * j), f1 = ld(f + 2 * j + 1), b0 = ld(b + 2 * j), b1 = ld(b + 2 * j + 1);
    acc_wide(u0, mul_wide(f0, b0));
    acc_wide(u2, mul_wide(fx(f0, f1), fx(b0, b1)));
  }
  block_xor_out(reduce(u0), out);
  block_xor_out(reduce(u2), out + 1);
}

// fold f and b at r (LSB binding), then emit the next message on the folded
// pair; TAB: products by r go through a CTA-resident 8-bit window table
template <bool TAB>
__global__ void __launch_bounds__(256) k_lig_fold_msg(const f128* __restrict__ f, const f128* __restrict__ b,
                                                      f128* __restrict__ fo, f128* __restrict__ bo, f128 r,
                                                      size_t n_pairs_out, int emit, f128* __restrict__ out) {
  extern __shared__ __align__(16) uint8_t sm[];
  MulTab8* rt = reinterpret_cast<MulTab8*>(sm);
  if (TAB) multab_build(rt, r);
  auto mr = [&](f128 v) { return TAB ? multab_mul(rt, v) : fmul(r, v); };
  u256 u0 = zero256(), u2 = zero256();
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_pairs_out; j += (size_t)gridDim.x * blockDim.x) {
    f128 fv[4], bv[4];
#pragma unroll
    for (int k = 0; k < 4; k++) { fv[k] = ld(f + 4 * j + k); bv[k] = ld(b + 4 * j + k); }
    f128 f0 = fx(fv[0], mr(fx(fv[0], fv[1]))), f1 = fx(fv[2], mr(fx(fv[2], fv[3])));
    f128 b0 = fx(bv[0], mr(fx(bv[0], bv[1]))), b1 = fx(bv[2], mr(fx(bv[2], bv[3])));
    st(fo + 2 * j, f0); st(fo + 2 * j + 1, f1);
    st(bo + 2 * j, b0); st(bo + 2 * j + 1, b1);
    if (emit) {
      acc_wide(u0, mul_wide(f0, b0));
      acc_wide(u2, mul_wide(fx(f0, f1), fx(b0, b1)));
    }
  }
  if (emit) {
    block_xor_out(reduce(u0), out);
    block_xor_out(reduce(u2), out + 1);
  }
}

// Degree-3 sumcheck round over plain F128 vectors (the zerocheck round of
// zerocheck/multilinear.rs:616-657 in its unstructured form): for the pairs
// (a0, a1) = (a[2j], a[2j+1]), (b0, b1) likewise and eq weight e[j],
//   G(1) = sum_j e[j] a1 b1,  G(inf) = sum_j e[j] (a0 + a1)(b0 + b1),
// optionally after folding the previous round's pairs at rho (LSB binding,
// a' = a0 + rho (a0 + a1); multilinear.rs:3194-3219).  The eq product is
// accumulated unreduced; rho's operand split is built once per thread.
template <bool FOLD>
__global__ void __launch_bounds__(256) k_sc3_round(const f128* __restrict__ a, const f128* __restrict__ b,
                                                   const f128* __restrict__ e, f128* __restrict__ ao,
                                                   f128* __restrict__ bo, f128 rho, size_t n_pairs,
                                                   f128* __restrict__ out) {
  const MulConst R = mulconst(rho);
  u256 g1 = zero256(), gi = zero256();
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_pairs; j += (size_t)gridDim.x * blockDim.x) {
    f128 a0, a1, b0, b1;
    if (FOLD) {
      f128 av[4], bv[4];
#pragma unroll
      for (int k = 0; k < 4; k++) { av[k] = ld(a + 4 * j + k); bv[k] = ld(b + 4 * j + k); }
      a0 = fx(av[0], fmul_c(fx(av[0], av[1]), R));
      a1 = fx(av[2], fmul_c(fx(av[2], av[3]), R));
      b0 = fx(bv[0], fmul_c(fx(bv[0], bv[1]), R));
      b1 = fx(bv[2], fmul_c(fx(bv[2], bv[3]), R));
      st(ao + 2 * j, a0); st(ao + 2 * j + 1, a1);
      st(bo + 2 * j, b0); st(bo + 2 * j + 1, b1);
    } else {
      a0 = ld(a + 2 * j); a1 = ld(a + 2 * j + 1);
      b0 = ld(b + 2 * j); b1 = ld(b + 2 * j + 1);
    }
    const f128 w = ld(e + j);
    acc_wide(g1, mul_wide(w, fmul(a1, b1)));
    acc_wide(gi, mul_wide(w, fmul(fx(a0, a1), fx(b0, b1))));
  }
  block_xor_out(reduce(g1), out);
  block_xor_out(reduce(gi), out + 1);
}

void sc3_round(const f128* a, const f128* b, const f128* e, f128* ao, f128* bo, const f128* rho, size_t n_pairs,
               f128* out, int grid, cudaStream_t s) {
  count_launch();
  if (rho)
    k_sc3_round<true><<<grid, 256, 0, s>>>(a, b, e, ao, bo, *rho, n_pairs, out);
  else
    k_sc3_round<false><<<grid, 256, 0, s>>>(a, b, e, ao, bo, mk(0, 0), n_pairs, out);
}

// sms: the SMs the launch may fill (one wave of resident CTAs on them)
void lig_msg(const f128* f, const f128* b, size_t n_pairs, f128* out, int sms, cudaStream_t s) {
  const int grid = resident_grid((const void*)k_lig_msg, 256, 0, sms);
  count_launch(); k_lig_msg<<<grid, 256, 0, s>>>(f, b, n_pairs, out);
}
void lig_fold_msg(const f128* f, const f128* b, f128* fo, f128* bo, f128 r, size_t n_pairs_out, bool emit, f128* out,
                  int sms, cudaStream_t s) {
  count_launch();
  if (n_pairs_out >= (1u << 14)) {
    size_t smem = sizeof(MulTab8);
    CK(cudaFuncSetAttribute(k_lig_fold_msg<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = resident_grid((const void*)k_lig_fold_msg<true>, 256, smem, sms);
    k_lig_fold_msg<true><<<grid, 256, smem, s>>>(f, b, fo, bo, r, n_pairs_out, emit, out);
  } else {
    const int grid = resident_grid((const void*)k_lig_fold_msg<false>, 256, 0, sms);
    k_lig_fold_msg<false><<<grid, 256, 0, s>>>(f, b, fo, bo, r, n_pairs_out, emit, out);
  }
}
void eq_split(const f128* lo, const f128* hi, int s_bits, size_t n, f128* out, cudaStream_t s) {
  count_launch(); k_eq_split<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(lo, hi, s_bits, n, out);
}
void eq_build(const f128* r, int n, f128 scale, f128* out, cudaStream_t s) {
  if (n < 0 || n > 24) throw CudaError("eq_build: at most 24 variables");
  EqVec E;
  for (int j = 0; j < n; j++) E.r[j] = r[j];
  E.scale = scale;
  E.n = n;
  const size_t len = (size_t)1 << n;
  count_launch();
  k_eq_build<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(E, out);
}
void outer64(const f128* L, const f128* e, size_t n_e, f128* out, cudaStream_t s) {
  Vec64 V;
  for (int j = 0; j < 64; j++) V.v[j] = L[j];
  count_launch();
  k_outer64<<<(unsigned)((64 * n_e + 255) / 256), 256, 0, s>>>(V, e, n_e, out);
}
void axpy(f128* out, const f128* x, f128 beta, size_t n, cudaStream_t s) {
  count_launch(); k_axpy<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, x, beta, n);
}
void inner(const f128* f, const f128* g, size_t n, f128* out, int grid, cudaStream_t s) {
  count_launch(); k_inner<<<grid, 256, 0, s>>>(f, g, n, out);
}
