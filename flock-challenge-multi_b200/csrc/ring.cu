// K7: ring switch (DP24 with phi8 weights) — crates/flock-core/src/pcs/
// ring_switch.rs.  Per claim k with suffix point x_k[1..] (25 coordinates at
// m = 32):  s_hat_v[r] = sum_i eq(suffix, i) bit_r(z_i)  (:1594-1640), and the
// transparent rs_eq_ind[i] = sum_b bit_b(eq(suffix, i)) eq''[b]  (:1952-2087).
// The open combines them: b_combined = sum_k gamma_k rs_eq_ind_k (pcs.rs:778-1290).
//
//  * s_hat_v of the ab-claim: its suffix is (r_inner_rest[1..8], x_outer), so
//    it is a 128 x 128 contraction of the lincheck's pre-sumcheck z_vec
//    (z_vec[c] = sum_o eq(x_outer, o) z[c + 2^14 o]):
//      s_hat_v[r] = sum_t eq(r_inner_rest[1..], t) z_vec[128 t + r]
//    (the reference's s_hat_v_from_z_vec, ring_switch.rs:1273).  The c-claim's
//    statistic is captured by zerocheck round 1 (round1.cu).
//  * b_combined: with eq(suffix, i) = eq_lo(i_lo) * eq_hi(i_hi), the map
//    u -> gamma_k L_k(u * eq_hi(i_hi)) is GF(2)-linear; per 2^12-element
//    chunk it is tabulated once as a 4-bit window table (the images of the
//    128 basis vectors, then the 16 subset sums of each window) and applied
//    to eq_lo with 32 conflict-free lookups per claim — no general products.
#include "kernels.cuh"

// one CTA per output r, one thread per t; the 128 products are XOR-reduced
// across the CTA (warp shuffles, then the four warp sums)
// a thread per 128-bit word of the block (128 to 1024 words), a CTA per bit r
__global__ void __launch_bounds__(1024) k_shat_from_zvec(const f128* __restrict__ zv, const f128* __restrict__ eqt,
                                                         f128* __restrict__ out) {
  __shared__ f128 red[32];
  const int r = blockIdx.x, t = threadIdx.x;
  f128 v = warp_xor(fmul(ldg(eqt + t), ldg(zv + 128 * t + r)));
  if ((t & 31) == 0) red[t >> 5] = v;
  __syncthreads();
  if (t == 0) {
    f128 s = mk(0, 0);
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s = fx(s, red[w]);
    out[r] = s;
  }
}

namespace {
__device__ __forceinline__ f128 apply_tab(const f128* T, f128 y) {  // T = [16][256] global
  f128 acc = mk(0, 0);
#pragma unroll
  for (int p = 0; p < 8; p++) {
    acc = fx(acc, ldg(T + p * 256 + ((y.lo >> (8 * p)) & 0xFF)));
    acc = fx(acc, ldg(T + (8 + p) * 256 + ((y.hi >> (8 * p)) & 0xFF)));
  }
  return acc;
}
}  // namespace

// out[chunk * 2^lo_bits + i_lo] = gamma0 L0(eq_lo0[i_lo] eq_hi0[chunk]) + gamma1 L1(...)
// Lk: [16][256] byte tables of gamma_k eq''_k (global)
__global__ void __launch_bounds__(512) k_bcombined_ct(const f128* __restrict__ elo0, const f128* __restrict__ ehi0,
                                                      const f128* __restrict__ elo1, const f128* __restrict__ ehi1,
                                                      const f128* __restrict__ L0, const f128* __restrict__ L1,
                                                      int lo_bits, size_t n_chunks, f128* __restrict__ out) {
  extern __shared__ __align__(16) uint8_t sm[];
  Tab4* C = reinterpret_cast<Tab4*>(sm);  // [2]: the chunk's maps of claims 0 and 1
  const size_t chunk_len = (size_t)1 << lo_bits;
  for (size_t ch = blockIdx.x; ch < n_chunks; ch += gridDim.x) {
    if (threadIdx.x < 64) {  // thread (k, w): window w of claim k's map
      const int k = threadIdx.x >> 5, w = threadIdx.x & 31;
      const f128* L = k ? L1 : L0;
      const f128 y = mul_x128(ldg((k ? ehi1 : ehi0) + ch), 4 * w);  // E x^(4w)
      tab4_window(C + k, w, apply_tab(L, y), apply_tab(L, mul_xk(y, 1)), apply_tab(L, mul_xk(y, 2)),
                  apply_tab(L, mul_xk(y, 3)));
    }
    __syncthreads();
    for (size_t i = threadIdx.x; i < chunk_len; i += blockDim.x)
      st(out + ch * chunk_len + i, fx(tab4_mul(C, ldg(elo0 + i)), tab4_mul(C + 1, ldg(elo1 + i))));
    __syncthreads();  // the next chunk's tables replace these
  }
}

// The same b_combined, and with it the first Ligerito message over (f, b)
// (the plain round k_lig_msg computes): msg[0] ^= sum_j f[2j] b[2j],
// msg[1] ^= sum_j (f[2j] + f[2j+1]) (b[2j] + b[2j+1]).  A thread owns the pair
// (2j, 2j+1) of a chunk.  The table lookups load the shared-memory pipe and
// the message's two products per pair the integer multipliers, so one pass
// keeps both busy where the two kernels each left the other pipe idle, and b
// is not read back.
__global__ void __launch_bounds__(256, 3) k_bcombined_msg(const f128* __restrict__ elo0, const f128* __restrict__ ehi0,
                                                          const f128* __restrict__ elo1, const f128* __restrict__ ehi1,
                                                          const f128* __restrict__ L0, const f128* __restrict__ L1,
                                                          int lo_bits, size_t n_chunks, const f128* __restrict__ f,
                                                          f128* __restrict__ out, f128* __restrict__ msg) {
  extern __shared__ __align__(16) uint8_t sm[];
  Tab4* C = reinterpret_cast<Tab4*>(sm);
  const size_t half = (size_t)1 << (lo_bits - 1);
  u256 u0 = zero256(), u2 = zero256();
  for (size_t ch = blockIdx.x; ch < n_chunks; ch += gridDim.x) {
    if (threadIdx.x < 64) {
      const int k = threadIdx.x >> 5, w = threadIdx.x & 31;
      const f128* L = k ? L1 : L0;
      const f128 y = mul_x128(ldg((k ? ehi1 : ehi0) + ch), 4 * w);
      tab4_window(C + k, w, apply_tab(L, y), apply_tab(L, mul_xk(y, 1)), apply_tab(L, mul_xk(y, 2)),
                  apply_tab(L, mul_xk(y, 3)));
    }
    __syncthreads();
    for (size_t j = threadIdx.x; j < half; j += blockDim.x) {
      const size_t i = 2 * j, o = (ch << lo_bits) + i;
      const f128 b0 = fx(tab4_mul(C, ldg(elo0 + i)), tab4_mul(C + 1, ldg(elo1 + i)));
      const f128 b1 = fx(tab4_mul(C, ldg(elo0 + i + 1)), tab4_mul(C + 1, ldg(elo1 + i + 1)));
      st(out + o, b0);
      st(out + o + 1, b1);
      const f128 f0 = ldg(f + o), f1 = ldg(f + o + 1);
      acc_wide(u0, mul_wide(f0, b0));
      acc_wide(u2, mul_wide(fx(f0, f1), fx(b0, b1)));
    }
    __syncthreads();  // the next chunk's tables replace these
  }
  block_xor_out(reduce(u0), msg);
  block_xor_out(reduce(u2), msg + 1);
}

void ring_shat_ab(const f128* zv_pre, const f128* eqt, int k_log, f128* out, cudaStream_t s) {
  count_launch();
  k_shat_from_zvec<<<128, 1 << (k_log - 7), 0, s>>>(zv_pre, eqt, out);
}

void ring_bcombined_ct(const f128* elo0, const f128* ehi0, const f128* elo1, const f128* ehi1, const f128* L0,
                       const f128* L1, int lo_bits, size_t n_chunks, f128* out, int sms, cudaStream_t s,
                       const f128* f, f128* msg) {
  size_t smem = 2 * kTab4Bytes;
  if (f && msg) {
    if (lo_bits < 1) throw CudaError("ring_bcombined_ct: the message needs chunks of at least 2 values");
    CK(cudaFuncSetAttribute(k_bcombined_msg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const size_t grid = (size_t)resident_grid((const void*)k_bcombined_msg, 256, smem, sms);
    count_launch();
    k_bcombined_msg<<<(unsigned)std::min<size_t>(n_chunks, grid), 256, smem, s>>>(elo0, ehi0, elo1, ehi1, L0, L1,
                                                                                 lo_bits, n_chunks, f, out, msg);
    return;
  }
  CK(cudaFuncSetAttribute(k_bcombined_ct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // one wave of resident CTAs: one CTA's table build overlaps the others' lookups
  const size_t grid = (size_t)resident_grid((const void*)k_bcombined_ct, 512, smem, sms);
  count_launch();
  k_bcombined_ct<<<(unsigned)std::min<size_t>(n_chunks, grid), 512, smem, s>>>(elo0, ehi0, elo1, ehi1, L0, L1,
                                                                              lo_bits, n_chunks, out);
}
