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

namespace {
__device__ __forceinline__ void block_xor_out(f128 v, f128* out) {
  __shared__ f128 red[32];
  v = warp_xor(v);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    int nw = (blockDim.x + 31) >> 5;
    f128 x = l < nw ? red[l] : mk(0, 0);
    x = warp_xor(x);
    if (l == 0) atomic_xor128(out, x);
  }
  __syncthreads();
}
}  // namespace

// ------------------------------------------------------------------ K3 --
__global__ void k_eq_split(const f128* __restrict__ lo, const f128* __restrict__ hi, int s, size_t n,
                           f128* __restrict__ out) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  st(out + i, fmul(ldg(lo + (i & ((1ull << s) - 1))), ldg(hi + (i >> s))));
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

// ------------------------------------------------------------------ K4 --
struct Round1Tables {
  uint8_t lde[8][256][64];  // byte-window tables of the S -> Lambda extension
  uint8_t exp_[512], log_[256];
  f128 phi[256];
  uint8_t g_log[8];          // log of the small-eq GF(2^8) weights (0xFF = zero)
};

__global__ void __launch_bounds__(256) k_zc_round1(const uint64_t* __restrict__ a, const uint64_t* __restrict__ b,
                                                   const uint64_t* __restrict__ c, const Round1Tables* __restrict__ tabs,
                                                   const f128* __restrict__ eqc, size_t n_blocks, f128* __restrict__ out) {
  extern __shared__ __align__(16) uint8_t sm[];
  Round1Tables* T = reinterpret_cast<Round1Tables*>(sm);
  uint8_t* tile = sm + sizeof(Round1Tables);  // [2 kinds][256 rows][64]
  {
    const uint4* src = reinterpret_cast<const uint4*>(tabs);
    uint4* dst = reinterpret_cast<uint4*>(sm);
    for (int i = threadIdx.x; i < (int)(sizeof(Round1Tables) / 16); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int t = threadIdx.x;
  const int lam = t & 63, kind = (t >> 6) & 1, half = t >> 7;  // phase-2 role
  u256 acc = zero256();
  for (size_t blk2 = blockIdx.x; blk2 * 2 < n_blocks; blk2 += gridDim.x) {
    // phase 1: thread t extends row (256 * blk2 + t) of a, b, c
    size_t row = blk2 * 256 + t;
    uint64_t ra = a[row], rb = b[row], rc = c[row];
    uint4 ea[4], eb[4], ec[4];
#pragma unroll
    for (int q = 0; q < 4; q++) { ea[q] = make_uint4(0, 0, 0, 0); eb[q] = ea[q]; ec[q] = ea[q]; }
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const uint4* pa = reinterpret_cast<const uint4*>(T->lde[k][(ra >> (8 * k)) & 0xFF]);
      const uint4* pb = reinterpret_cast<const uint4*>(T->lde[k][(rb >> (8 * k)) & 0xFF]);
      const uint4* pc = reinterpret_cast<const uint4*>(T->lde[k][(rc >> (8 * k)) & 0xFF]);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        uint4 x = pa[q], y = pb[q], z = pc[q];
        ea[q].x ^= x.x; ea[q].y ^= x.y; ea[q].z ^= x.z; ea[q].w ^= x.w;
        eb[q].x ^= y.x; eb[q].y ^= y.y; eb[q].z ^= y.z; eb[q].w ^= y.w;
        ec[q].x ^= z.x; ec[q].y ^= z.y; ec[q].z ^= z.z; ec[q].w ^= z.w;
      }
    }
    const uint8_t* A = reinterpret_cast<const uint8_t*>(ea);
    const uint8_t* B = reinterpret_cast<const uint8_t*>(eb);
    uint8_t prod[64];
#pragma unroll
    for (int l = 0; l < 64; l++) {
      uint8_t x = A[l], y = B[l];
      prod[l] = (x && y) ? T->exp_[T->log_[x] + T->log_[y]] : 0;
    }
    uint4* dab = reinterpret_cast<uint4*>(tile + (size_t)t * 64);
    uint4* dc = reinterpret_cast<uint4*>(tile + 256 * 64 + (size_t)t * 64);
#pragma unroll
    for (int q = 0; q < 4; q++) { dab[q] = reinterpret_cast<const uint4*>(prod)[q]; dc[q] = ec[q]; }
    __syncthreads();
    // phase 2: thread (half, kind, lam) folds the 128 rows of block 2*blk2+half
    const uint8_t* src = tile + (size_t)kind * 256 * 64 + (size_t)half * 128 * 64;
    uint64_t w0 = 0, w1 = 0, w2 = 0;  // 144-bit accumulator of sum_xm gamma^xm phi8(u)
    for (int xm = 0; xm < 16; xm++) {
      uint8_t u = 0;
#pragma unroll
      for (int xs = 0; xs < 8; xs++) {
        uint8_t v = src[(xm * 8 + xs) * 64 + lam];
        uint8_t gl = T->g_log[xs];
        if (v && gl != 0xFF) u ^= T->exp_[T->log_[v] + gl];
      }
      f128 p = T->phi[u];
      if (xm == 0) { w0 ^= p.lo; w1 ^= p.hi; }
      else { w0 ^= p.lo << xm; w1 ^= (p.hi << xm) | (p.lo >> (64 - xm)); w2 ^= p.hi >> (64 - xm); }
    }
    f128 v = reduce256(w0, w1, w2, 0);
    size_t blk = blk2 * 2 + half;
    acc_wide(acc, mul_wide(v, ldg(eqc + blk)));
    __syncthreads();
  }
  f128 r = reduce(acc);
  // threads (half 0, half 1) with the same (kind, lam) hit the same output
  atomic_xor128(out + kind * 64 + lam, r);
}

void zc_round1(const f128* a, const f128* b, const f128* c, const void* tabs, const f128* eqc, size_t n_blocks,
               f128* out, int grid, cudaStream_t s) {
  size_t smem = sizeof(Round1Tables) + 2 * 256 * 64;
  CK(cudaFuncSetAttribute(k_zc_round1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  count_launch(); k_zc_round1<<<grid, 256, smem, s>>>((const uint64_t*)a, (const uint64_t*)b, (const uint64_t*)c,
                                      (const Round1Tables*)tabs, eqc, n_blocks, out);
}
size_t round1_tables_size() { return sizeof(Round1Tables); }

// ------------------------------------------------------------------ K5 --
// Lagrange byte tables: lag[k][v] = sum_{bit j of v} L_{8k+j}(z)
__device__ __forceinline__ f128 lag_lookup(const f128* lag, uint64_t row) {
  f128 s = mk(0, 0);
#pragma unroll
  for (int k = 0; k < 8; k++) s = fx(s, lag[k * 256 + ((row >> (8 * k)) & 0xFF)]);
  return s;
}

// Round-0 message from the packed rows: pair j = (row 2j, row 2j+1) = (lo, hi) of word j.
__global__ void __launch_bounds__(256) k_zc_msg0(const f128* __restrict__ a, const f128* __restrict__ b,
                                                 const f128* __restrict__ lag_g, const f128* __restrict__ elo,
                                                 const f128* __restrict__ ehi, int es, size_t n_pairs,
                                                 f128* __restrict__ out) {
  __shared__ f128 lag[8 * 256];
  for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) lag[i] = lag_g[i];
  __syncthreads();
  u256 g1 = zero256(), gi = zero256();
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_pairs; j += (size_t)gridDim.x * blockDim.x) {
    f128 wa = ld(a + j), wb = ld(b + j);
    f128 a0 = lag_lookup(lag, wa.lo), a1 = lag_lookup(lag, wa.hi);
    f128 b0 = lag_lookup(lag, wb.lo), b1 = lag_lookup(lag, wb.hi);
    f128 e = fmul(ldg(elo + (j & ((1ull << es) - 1))), ldg(ehi + (j >> es)));
    acc_wide(g1, mul_wide(e, fmul(a1, b1)));
    acc_wide(gi, mul_wide(e, fmul(fx(a0, a1), fx(b0, b1))));
  }
  block_xor_out(reduce(g1), out);
  block_xor_out(reduce(gi), out + 1);
}

// Fold round i (challenge rho) and emit the message of round i + 1.
// FROM_PACKED: round i = 0, values a^_0 come from the packed rows.
template <bool FROM_PACKED>
__global__ void __launch_bounds__(256) k_zc_fold_msg(const f128* __restrict__ a_in, const f128* __restrict__ b_in,
                                                     f128* __restrict__ a_out, f128* __restrict__ b_out,
                                                     const f128* __restrict__ lag_g, f128 rho,
                                                     const f128* __restrict__ elo, const f128* __restrict__ ehi, int es,
                                                     size_t n_pairs_out, int emit, f128* __restrict__ out) {
  __shared__ f128 lag[FROM_PACKED ? 8 * 256 : 1];
  if (FROM_PACKED) {
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) lag[i] = lag_g[i];
    __syncthreads();
  }
  u256 g1 = zero256(), gi = zero256();
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_pairs_out; j += (size_t)gridDim.x * blockDim.x) {
    f128 av[4], bv[4];
    if (FROM_PACKED) {
      f128 w0 = ld(a_in + 2 * j), w1 = ld(a_in + 2 * j + 1), v0 = ld(b_in + 2 * j), v1 = ld(b_in + 2 * j + 1);
      av[0] = lag_lookup(lag, w0.lo); av[1] = lag_lookup(lag, w0.hi);
      av[2] = lag_lookup(lag, w1.lo); av[3] = lag_lookup(lag, w1.hi);
      bv[0] = lag_lookup(lag, v0.lo); bv[1] = lag_lookup(lag, v0.hi);
      bv[2] = lag_lookup(lag, v1.lo); bv[3] = lag_lookup(lag, v1.hi);
    } else {
#pragma unroll
      for (int k = 0; k < 4; k++) { av[k] = ld(a_in + 4 * j + k); bv[k] = ld(b_in + 4 * j + k); }
    }
    f128 a0 = fx(av[0], fmul(rho, fx(av[0], av[1]))), a1 = fx(av[2], fmul(rho, fx(av[2], av[3])));
    f128 b0 = fx(bv[0], fmul(rho, fx(bv[0], bv[1]))), b1 = fx(bv[2], fmul(rho, fx(bv[2], bv[3])));
    st(a_out + 2 * j, a0); st(a_out + 2 * j + 1, a1);
    st(b_out + 2 * j, b0); st(b_out + 2 * j + 1, b1);
    if (emit) {
      f128 e = fmul(ldg(elo + (j & ((1ull << es) - 1))), ldg(ehi + (j >> es)));
      acc_wide(g1, mul_wide(e, fmul(a1, b1)));
      acc_wide(gi, mul_wide(e, fmul(fx(a0, a1), fx(b0, b1))));
    }
  }
  if (emit) {
    block_xor_out(reduce(g1), out);
    block_xor_out(reduce(gi), out + 1);
  }
}

// last fold: 2 -> 1 values per vector
__global__ void k_fold_pair_final(const f128* a_in, const f128* b_in, f128 rho, f128* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    f128 a0 = a_in[0], a1 = a_in[1], b0 = b_in[0], b1 = b_in[1];
    out[0] = fx(a0, fmul(rho, fx(a0, a1)));
    out[1] = fx(b0, fmul(rho, fx(b0, b1)));
  }
}

void zc_msg0(const f128* a, const f128* b, const f128* lag, const f128* elo, const f128* ehi, int es, size_t n_pairs,
             f128* out, int grid, cudaStream_t s) {
  count_launch(); k_zc_msg0<<<grid, 256, 0, s>>>(a, b, lag, elo, ehi, es, n_pairs, out);
}
void zc_fold_msg(bool from_packed, const f128* a_in, const f128* b_in, f128* a_out, f128* b_out, const f128* lag,
                 f128 rho, const f128* elo, const f128* ehi, int es, size_t n_pairs_out, bool emit, f128* out,
                 int grid, cudaStream_t s) {
  count_launch();
  if (from_packed)
    k_zc_fold_msg<true><<<grid, 256, 0, s>>>(a_in, b_in, a_out, b_out, lag, rho, elo, ehi, es, n_pairs_out, emit, out);
  else
    k_zc_fold_msg<false><<<grid, 256, 0, s>>>(a_in, b_in, a_out, b_out, lag, rho, elo, ehi, es, n_pairs_out, emit, out);
}
void fold_pair_final(const f128* a_in, const f128* b_in, f128 rho, f128* out, cudaStream_t s) {
  count_launch(); k_fold_pair_final<<<1, 32, 0, s>>>(a_in, b_in, rho, out);
}

// ------------------------------------------------------------------ K6 --
__global__ void k_lc_comb(const uint32_t* __restrict__ at_ptr, const uint16_t* __restrict__ at_row,
                          const uint32_t* __restrict__ bt_ptr, const uint16_t* __restrict__ bt_row,
                          const f128* __restrict__ eq, f128 alpha, f128 beta, int pin, f128* __restrict__ comb) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= kK_) return;
  f128 sa = mk(0, 0), sb = mk(0, 0);
  for (uint32_t j = at_ptr[c]; j < at_ptr[c + 1]; j++) sa = fx(sa, ldg(eq + at_row[j]));
  for (uint32_t j = bt_ptr[c]; j < bt_ptr[c + 1]; j++) sb = fx(sb, ldg(eq + bt_row[j]));
  f128 v = fx(fmul(alpha, sa), sb);
  if (c == pin) v = fx(v, beta);
  st(comb + c, v);
}

// z_vec: thread (byte position cb, o-chunk) accumulates 8 columns
__global__ void __launch_bounds__(128) k_lc_zvec(const uint8_t* __restrict__ z, const f128* __restrict__ eqo,
                                                 size_t n_outer, int chunk, f128* __restrict__ zv) {
  int cb = blockIdx.x * blockDim.x + threadIdx.x;  // 0..2047
  size_t o0 = (size_t)blockIdx.y * chunk, o1 = o0 + chunk < n_outer ? o0 + chunk : n_outer;
  f128 acc[8];
#pragma unroll
  for (int k = 0; k < 8; k++) acc[k] = mk(0, 0);
  for (size_t o = o0; o < o1; o++) {
    uint32_t byte = z[o * 2048 + cb];
    if (!byte) continue;
    f128 e = ldg(eqo + o);
#pragma unroll
    for (int k = 0; k < 8; k++)
      if ((byte >> k) & 1) acc[k] = fx(acc[k], e);
  }
#pragma unroll
  for (int k = 0; k < 8; k++) atomic_xor128(zv + 8 * cb + k, acc[k]);
}

// One CTA: optionally bind the top variable at r (fold), then emit (q(1), q(inf)).
__global__ void __launch_bounds__(512) k_lc_round(f128* comb, f128* zv, int len, int do_fold, f128 r, int emit,
                                                   f128* out) {
  int t = threadIdx.x;
  if (do_fold) {
    int half = len;  // len is the length after folding
    for (int i = t; i < half; i += blockDim.x) {
      f128 c0 = comb[i], c1 = comb[i + half], z0 = zv[i], z1 = zv[i + half];
      comb[i] = fx(c0, fmul(r, fx(c1, c0)));
      zv[i] = fx(z0, fmul(r, fx(z1, z0)));
    }
    __syncthreads();
  }
  if (!emit) return;
  int half = len >> 1;
  u256 q1 = zero256(), qi = zero256();
  for (int i = t; i < half; i += blockDim.x) {
    f128 c0 = comb[i], c1 = comb[i + half], z0 = zv[i], z1 = zv[i + half];
    acc_wide(q1, mul_wide(c1, z1));
    acc_wide(qi, mul_wide(fx(c0, c1), fx(z0, z1)));
  }
  __shared__ f128 red[2][32];
  f128 a = warp_xor(reduce(q1)), bq = warp_xor(reduce(qi));
  if ((t & 31) == 0) { red[0][t >> 5] = a; red[1][t >> 5] = bq; }
  __syncthreads();
  if (t == 0) {
    f128 x = mk(0, 0), y = mk(0, 0);
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) { x = fx(x, red[0][w]); y = fx(y, red[1][w]); }
    out[0] = x;
    out[1] = y;
  }
}

void lc_comb(const uint32_t* at_ptr, const uint16_t* at_row, const uint32_t* bt_ptr, const uint16_t* bt_row,
             const f128* eq, f128 alpha, f128 beta, int pin, f128* comb, cudaStream_t s) {
  count_launch(); k_lc_comb<<<kK_ / 128, 128, 0, s>>>(at_ptr, at_row, bt_ptr, bt_row, eq, alpha, beta, pin, comb);
}
void lc_zvec(const f128* z, const f128* eqo, size_t n_outer, f128* zv, cudaStream_t s) {
  int chunk = 256;
  dim3 grid(2048 / 128, (unsigned)((n_outer + chunk - 1) / chunk));
  count_launch(); k_lc_zvec<<<grid, 128, 0, s>>>((const uint8_t*)z, eqo, n_outer, chunk, zv);
}
void lc_round(f128* comb, f128* zv, int len, bool fold, f128 r, bool emit, f128* out, cudaStream_t s) {
  count_launch(); k_lc_round<<<1, 512, 0, s>>>(comb, zv, len, fold, r, emit, out);
}

// ------------------------------------------------------------------ K7 --
// s_hat_v[r] = sum_i eq(i) bit_r(z_i): lane l of each warp owns r = l + 32 k
__global__ void __launch_bounds__(256) k_shat(const f128* __restrict__ z, const f128* __restrict__ eq, size_t n,
                                              f128* __restrict__ out) {
  int lane = threadIdx.x & 31;
  f128 acc[4];
#pragma unroll
  for (int k = 0; k < 4; k++) acc[k] = mk(0, 0);
  size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t base = warp * 32; base < n; base += nw * 32) {
    size_t i = base + lane;
    f128 zi = i < n ? ld(z + i) : mk(0, 0), ei = i < n ? ld(eq + i) : mk(0, 0);
#pragma unroll 4
    for (int s = 0; s < 32; s++) {
      uint64_t zl = __shfl_sync(0xffffffffu, zi.lo, s), zh = __shfl_sync(0xffffffffu, zi.hi, s);
      uint64_t el = __shfl_sync(0xffffffffu, ei.lo, s), eh = __shfl_sync(0xffffffffu, ei.hi, s);
      uint32_t w0 = (uint32_t)zl, w1 = (uint32_t)(zl >> 32), w2 = (uint32_t)zh, w3 = (uint32_t)(zh >> 32);
      uint64_t m0 = 0ull - ((w0 >> lane) & 1), m1 = 0ull - ((w1 >> lane) & 1);
      uint64_t m2 = 0ull - ((w2 >> lane) & 1), m3 = 0ull - ((w3 >> lane) & 1);
      acc[0].lo ^= el & m0; acc[0].hi ^= eh & m0;
      acc[1].lo ^= el & m1; acc[1].hi ^= eh & m1;
      acc[2].lo ^= el & m2; acc[2].hi ^= eh & m2;
      acc[3].lo ^= el & m3; acc[3].hi ^= eh & m3;
    }
  }
#pragma unroll
  for (int k = 0; k < 4; k++) atomic_xor128(out + 32 * k + lane, acc[k]);
}

// b_combined[i] = T0(eq0[i]) + T1(eq1[i]), Tk = 16 byte tables of gamma_k eq''_k
__global__ void __launch_bounds__(256) k_bcombined(const f128* __restrict__ eq0, const f128* __restrict__ eq1,
                                                   const f128* __restrict__ tabs, size_t n, f128* __restrict__ out) {
  extern __shared__ f128 T[];  // [2][16][256]
  for (int i = threadIdx.x; i < 2 * 16 * 256; i += blockDim.x) T[i] = tabs[i];
  __syncthreads();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    f128 e0 = ld(eq0 + i), e1 = ld(eq1 + i), acc = mk(0, 0);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      acc = fx(acc, T[k * 256 + ((e0.lo >> (8 * k)) & 0xFF)]);
      acc = fx(acc, T[(8 + k) * 256 + ((e0.hi >> (8 * k)) & 0xFF)]);
      acc = fx(acc, T[4096 + k * 256 + ((e1.lo >> (8 * k)) & 0xFF)]);
      acc = fx(acc, T[4096 + (8 + k) * 256 + ((e1.hi >> (8 * k)) & 0xFF)]);
    }
    st(out + i, acc);
  }
}

void ring_shat(const f128* z, const f128* eq, size_t n, f128* out, int grid, cudaStream_t s) {
  count_launch(); k_shat<<<grid, 256, 0, s>>>(z, eq, n, out);
}
void ring_bcombined(const f128* eq0, const f128* eq1, const f128* tabs, size_t n, f128* out, int grid, cudaStream_t s) {
  size_t smem = 2 * 16 * 256 * sizeof(f128);
  CK(cudaFuncSetAttribute(k_bcombined, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  count_launch(); k_bcombined<<<grid, 256, smem, s>>>(eq0, eq1, tabs, n, out);
}

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

// fold f and b at r (LSB binding), then emit the next message on the folded pair
__global__ void __launch_bounds__(256) k_lig_fold_msg(const f128* __restrict__ f, const f128* __restrict__ b,
                                                      f128* __restrict__ fo, f128* __restrict__ bo, f128 r,
                                                      size_t n_pairs_out, int emit, f128* __restrict__ out) {
  u256 u0 = zero256(), u2 = zero256();
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_pairs_out; j += (size_t)gridDim.x * blockDim.x) {
    f128 fv[4], bv[4];
#pragma unroll
    for (int k = 0; k < 4; k++) { fv[k] = ld(f + 4 * j + k); bv[k] = ld(b + 4 * j + k); }
    f128 f0 = fx(fv[0], fmul(r, fx(fv[0], fv[1]))), f1 = fx(fv[2], fmul(r, fx(fv[2], fv[3])));
    f128 b0 = fx(bv[0], fmul(r, fx(bv[0], bv[1]))), b1 = fx(bv[2], fmul(r, fx(bv[2], bv[3])));
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

void lig_msg(const f128* f, const f128* b, size_t n_pairs, f128* out, int grid, cudaStream_t s) {
  count_launch(); k_lig_msg<<<grid, 256, 0, s>>>(f, b, n_pairs, out);
}
void lig_fold_msg(const f128* f, const f128* b, f128* fo, f128* bo, f128 r, size_t n_pairs_out, bool emit, f128* out,
                  int grid, cudaStream_t s) {
  count_launch(); k_lig_fold_msg<<<grid, 256, 0, s>>>(f, b, fo, bo, r, n_pairs_out, emit, out);
}
void eq_split(const f128* lo, const f128* hi, int s_bits, size_t n, f128* out, cudaStream_t s) {
  count_launch(); k_eq_split<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(lo, hi, s_bits, n, out);
}
void axpy(f128* out, const f128* x, f128 beta, size_t n, cudaStream_t s) {
  count_launch(); k_axpy<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, x, beta, n);
}
void inner(const f128* f, const f128* g, size_t n, f128* out, int grid, cudaStream_t s) {
  count_launch(); k_inner<<<grid, 256, 0, s>>>(f, g, n, out);
}
