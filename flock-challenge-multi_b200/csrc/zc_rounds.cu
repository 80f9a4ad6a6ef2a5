// K5: zerocheck multilinear rounds (crates/flock-core/src/zerocheck.rs:
// 1735-1795 verifier order; multilinear.rs:575-657 fold-at-z and
// round_pair_naive, :3194-3330 fused fold + message).
//
// Round k binds rest variable k (the LSB of the current vectors a^, b^) and
// sends G(1) = sum_j e(j) a^(2j+1) b^(2j+1) and
// G(inf) = sum_j e(j) (a^(2j)+a^(2j+1)) (b^(2j)+b^(2j+1)) with
// e(j) = eq(r[7+k..m], j).  Round 0 reads the packed rows directly:
// a^(x) = sum_s L_s(z) a_s(x) through 8 byte-window tables of the Lagrange
// weights.  Every later round first folds at the previous challenge rho:
// a^'(i) = a^(2i) + rho (a^(2i) + a^(2i+1)) — a product by a constant, done
// through a CTA-resident 8-bit window table of rho.
//
// The eq weights exploit the fixed inner challenges of the zerocheck
// (univariate_skip_optimized.rs:136-233): the low `ns` bits of j sit on
// phi8 subfield constants (weight phi8(g(js))) and the next `nm` bits on the
// medium constants (weight C * x^(sum of 2^t over set bits)), so a warp sums
// its 32 pairs with shifts and shuffles, and only one product by phi8(g(js))
// and one by eq(random suffix, group) remain per group of 2^(ns+nm) pairs.
#include "kernels.cuh"

namespace {
struct ZcArgs {
  const f128* a_in;
  const f128* b_in;
  f128* a_out;
  f128* b_out;
  const f128* lag;  // 8 x 256 Lagrange byte table (packed input)
  f128 rho;
  size_t n_pairs;   // pairs of the message round
  int ns, nm;
  int shift[4];
  f128 K[4];        // phi8(g(js)), js < 2^ns
  const f128* elo;  // eq over the random suffix (x C), indexed by group
  const f128* ehi;
  int es;
  f128* out;
};

__device__ __forceinline__ f128 lag_lookup(const f128* lag, uint64_t row) {
  f128 s = mk(0, 0);
#pragma unroll
  for (int k = 0; k < 8; k++) s = fx(s, lag[k * 256 + ((row >> (8 * k)) & 0xFF)]);
  return s;
}

struct W3 {
  uint64_t w0, w1, w2;
};
__device__ __forceinline__ W3 shl144(f128 v, int sh) {
  W3 r;
  if (sh == 0) {
    r.w0 = v.lo; r.w1 = v.hi; r.w2 = 0;
  } else {
    r.w0 = v.lo << sh;
    r.w1 = (v.hi << sh) | (v.lo >> (64 - sh));
    r.w2 = v.hi >> (64 - sh);
  }
  return r;
}
__device__ __forceinline__ void xshfl(W3& v, int m) {
  v.w0 ^= shfl_xor64(v.w0, m);
  v.w1 ^= shfl_xor64(v.w1, m);
  v.w2 ^= shfl_xor64(v.w2, m);
}
__device__ __forceinline__ void xshfl(f128& v, int m) {
  v.lo ^= shfl_xor64(v.lo, m);
  v.hi ^= shfl_xor64(v.hi, m);
}

template <bool PACKED, bool FOLD>
__global__ void __launch_bounds__(256) k_zc_round(ZcArgs A) {
  extern __shared__ __align__(16) uint8_t sm[];
  MulTab8* rt = reinterpret_cast<MulTab8*>(sm);
  f128* lag = reinterpret_cast<f128*>(sm + (FOLD ? sizeof(MulTab8) : 0));
  if (PACKED)
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) lag[i] = A.lag[i];
  if (FOLD) multab_build(rt, A.rho);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int g_bits = A.ns + A.nm;
  const size_t G = (size_t)1 << g_bits;
  const int nsub = g_bits > 5 ? 1 << (g_bits - 5) : 1;   // 32-pair chunks per group
  const int lane_m = (g_bits > 5 ? 5 : g_bits) - A.ns;   // medium bits inside the lane index
  const size_t span = (size_t)32 * nsub;                  // pairs per warp iteration
  const size_t n_warps = ((size_t)gridDim.x * blockDim.x) >> 5;
  u256 acc1 = zero256(), acci = zero256();
  for (size_t base = (((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * span; base < A.n_pairs;
       base += n_warps * span) {
    W3 s1 = {0, 0, 0}, si = {0, 0, 0};
    for (int sub = 0; sub < nsub; sub++) {
      const size_t j = base + (size_t)sub * 32 + lane;
      f128 a0 = mk(0, 0), a1 = a0, b0 = a0, b1 = a0;
      if (j >= A.n_pairs) {
        // lanes past the end of a short final round contribute nothing
      } else if (!FOLD) {  // round 0: pair (2j, 2j+1) = (lo, hi) of packed word j
        f128 wa = ld(A.a_in + j), wb = ld(A.b_in + j);
        a0 = lag_lookup(lag, wa.lo); a1 = lag_lookup(lag, wa.hi);
        b0 = lag_lookup(lag, wb.lo); b1 = lag_lookup(lag, wb.hi);
      } else {
        f128 av[4], bv[4];
        if (PACKED) {
          f128 w0 = ld(A.a_in + 2 * j), w1 = ld(A.a_in + 2 * j + 1);
          f128 v0 = ld(A.b_in + 2 * j), v1 = ld(A.b_in + 2 * j + 1);
          av[0] = lag_lookup(lag, w0.lo); av[1] = lag_lookup(lag, w0.hi);
          av[2] = lag_lookup(lag, w1.lo); av[3] = lag_lookup(lag, w1.hi);
          bv[0] = lag_lookup(lag, v0.lo); bv[1] = lag_lookup(lag, v0.hi);
          bv[2] = lag_lookup(lag, v1.lo); bv[3] = lag_lookup(lag, v1.hi);
        } else {
#pragma unroll
          for (int k = 0; k < 4; k++) { av[k] = ld(A.a_in + 4 * j + k); bv[k] = ld(A.b_in + 4 * j + k); }
        }
        a0 = fx(av[0], multab_mul(rt, fx(av[0], av[1])));
        a1 = fx(av[2], multab_mul(rt, fx(av[2], av[3])));
        b0 = fx(bv[0], multab_mul(rt, fx(bv[0], bv[1])));
        b1 = fx(bv[2], multab_mul(rt, fx(bv[2], bv[3])));
        st(A.a_out + 2 * j, a0); st(A.a_out + 2 * j + 1, a1);
        st(A.b_out + 2 * j, b0); st(A.b_out + 2 * j + 1, b1);
      }
      f128 p1 = fmul(a1, b1), pi = fmul(fx(a0, a1), fx(b0, b1));
      const size_t jm = (j >> A.ns) & ((1ull << A.nm) - 1);
      int sh = 0;
#pragma unroll
      for (int t = 0; t < 4; t++)
        if (t < A.nm && ((jm >> t) & 1)) sh += A.shift[t];
      W3 v1 = shl144(p1, sh), vi = shl144(pi, sh);
      s1.w0 ^= v1.w0; s1.w1 ^= v1.w1; s1.w2 ^= v1.w2;
      si.w0 ^= vi.w0; si.w1 ^= vi.w1; si.w2 ^= vi.w2;
    }
    // sum the medium bits held in the lane index
    for (int t = 0; t < lane_m; t++) {
      xshfl(s1, 1 << (A.ns + t));
      xshfl(si, 1 << (A.ns + t));
    }
    f128 g1 = reduce256(s1.w0, s1.w1, s1.w2, 0), gi = reduce256(si.w0, si.w1, si.w2, 0);
    if (A.ns > 0) {
      f128 k = A.K[lane & ((1 << A.ns) - 1)];
      g1 = fmul(g1, k);
      gi = fmul(gi, k);
      for (int t = 0; t < A.ns; t++) {
        xshfl(g1, 1 << t);
        xshfl(gi, 1 << t);
      }
    }
    const int lane_g = g_bits > 5 ? 5 : g_bits;
    if ((lane & ((1 << lane_g) - 1)) == 0 && base + lane < A.n_pairs) {
      size_t grp = (base + lane) >> g_bits;
      f128 e = fmul(ldg(A.elo + (grp & ((1ull << A.es) - 1))), ldg(A.ehi + (grp >> A.es)));
      acc_wide(acc1, mul_wide(g1, e));
      acc_wide(acci, mul_wide(gi, e));
    }
  }
  // block reduction of both message components
  f128 r1 = warp_xor(reduce(acc1)), ri = warp_xor(reduce(acci));
  __shared__ f128 red[2][8];
  int w = threadIdx.x >> 5;
  if (lane == 0) { red[0][w] = r1; red[1][w] = ri; }
  __syncthreads();
  if (threadIdx.x == 0) {
    f128 x = mk(0, 0), y = mk(0, 0);
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) { x = fx(x, red[0][k]); y = fx(y, red[1][k]); }
    atomic_xor128(A.out, x);
    atomic_xor128(A.out + 1, y);
  }
}
}  // namespace

// One zerocheck round launch.  n_pairs is a multiple of 32 or smaller than it
// only when the whole round fits one group (handled with G = n_pairs lanes).
void zc_round(bool packed, bool fold, const f128* a_in, const f128* b_in, f128* a_out, f128* b_out, const f128* lag,
              f128 rho, size_t n_pairs, int ns, int nm, const int* shift, const f128* K, const f128* elo,
              const f128* ehi, int es, f128* out, int grid, cudaStream_t s) {
  ZcArgs A;
  A.a_in = a_in; A.b_in = b_in; A.a_out = a_out; A.b_out = b_out; A.lag = lag; A.rho = rho;
  A.n_pairs = n_pairs; A.ns = ns; A.nm = nm;
  for (int t = 0; t < 4; t++) { A.shift[t] = shift ? shift[t] : 0; A.K[t] = K ? K[t] : mk(0, 0); }
  A.elo = elo; A.ehi = ehi; A.es = es; A.out = out;
  size_t smem = (fold ? sizeof(MulTab8) : 0) + (packed ? 8 * 256 * sizeof(f128) : 0);
  size_t warps_needed = (n_pairs + 31) / 32;
  int g = (int)std::min<size_t>((size_t)grid, (warps_needed + 7) / 8);
  if (g < 1) g = 1;
  count_launch();
  if (packed && fold) {
    CK(cudaFuncSetAttribute(k_zc_round<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_zc_round<true, true><<<g, 256, smem, s>>>(A);
  } else if (packed) {
    CK(cudaFuncSetAttribute(k_zc_round<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_zc_round<true, false><<<g, 256, smem, s>>>(A);
  } else {
    CK(cudaFuncSetAttribute(k_zc_round<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_zc_round<false, true><<<g, 256, smem, s>>>(A);
  }
}
