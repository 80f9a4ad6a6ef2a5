// Merkle-path kernels (SHA-256 statement, 2^15-bit blocks of 256 packed
// words): the slot fold that collapses each instance's four 256-bit slots
// (H_in, H_out, M_lo, M_hi: packed words 2s, 2s + 1 of its block) to one
// value apiece, the weight tables of the shift sumcheck, its degree-3 rounds
// over seven tables, and the scatter of the packed-direct claim into
// b_combined (the claim point [tau_pos, sel_slot, side, 0^5, instance] is
// nonzero only on words 0..7 of each block).
// crates/flock-prover/src/r1cs_hashes/merkle_path_common.rs:180-225
// (fold_all_slots), :262-282 (claim point); crates/flock-prover/src/
// merkle_path.rs:245-385 (tables, y-rounds); crates/flock-core/src/pcs.rs:
// 1236-1248 (scatter).
#include "kernels.cuh"
#include <algorithm>

namespace {

constexpr int kBlockWords = 256;  // packed words of a 2^15-bit block

__global__ void __launch_bounds__(256) k_mp_fold(const f128* __restrict__ z, size_t n_inst, f128 e0, f128 e1,
                                                 f128* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst) return;
  const f128* w = z + kBlockWords * i;
#pragma unroll
  for (int s = 0; s < 4; s++) out[s * n_inst + i] = fx(fmul(e0, w[2 * s]), fmul(e1, w[2 * s + 1]));
}

// ta[i] = eq_p[i >> pos_log] (i_q == 0 ? alpha : eq_q[i_q - 1]);
// tb[i] = b[i] unless i is the first row of its path (B := 0 there)
__global__ void __launch_bounds__(256) k_mp_tables(const f128* __restrict__ eq_q, const f128* __restrict__ eq_p,
                                                   f128 alpha, int pos_log, size_t n, const uint8_t* __restrict__ b,
                                                   f128* __restrict__ ta, f128* __restrict__ tb) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t iq = i & (((size_t)1 << pos_log) - 1);
  ta[i] = fmul(eq_p[i >> pos_log], iq == 0 ? alpha : eq_q[iq - 1]);
  tb[i] = mk(b[i] && iq != 0 ? 1 : 0, 0);
}

// One y-round: with do_fold, fold every table (2 len values) at r into its
// first len values (top variable); with emit, add the round polynomial at
// X = 1, w, w + 1 over the pairs (i, i + len/2) into out[0..3):
//   q(X) = sum te(X) gz(X) + ta(X) (gxl(X) + tb(X) (gxl(X) + gxr(X))),
// each table T(X) = T_lo + X (T_hi + T_lo), w = x.  Thread i < len/2 owns
// outputs i and i + len/2 of every table, so no grid synchronisation.
__global__ void __launch_bounds__(256) k_mp_round(MpTables T, int len, int do_fold, f128 r, int emit, f128* out) {
  const int h = len >> 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  f128 s1 = mk(0, 0), sw = mk(0, 0), sw1 = mk(0, 0);
  if (i < h) {
    f128 lo[7], hi[7];
#pragma unroll
    for (int t = 0; t < 7; t++) {
      f128* p = T.t[t];
      lo[t] = p[i];
      hi[t] = p[i + h];
      if (do_fold) {
        lo[t] = fx(lo[t], fmul(r, fx(p[i + len], lo[t])));
        hi[t] = fx(hi[t], fmul(r, fx(p[i + h + len], hi[t])));
        p[i] = lo[t];
        p[i + h] = hi[t];
      }
    }
    if (emit) {
      // tables 0..5: ta, te, tb, gz, gxl, gxr (6: g_other, folded only)
      f128 d[6], v1[6], vw[6], vw1[6];
#pragma unroll
      for (int t = 0; t < 6; t++) {
        d[t] = fx(hi[t], lo[t]);
        v1[t] = hi[t];
        vw[t] = fx(lo[t], mul_xk(d[t], 1));
        vw1[t] = fx(vw[t], d[t]);
      }
      auto q = [](const f128* v) {
        return fx(fmul(v[1], v[3]), fmul(v[0], fx(v[4], fmul(v[2], fx(v[4], v[5])))));
      };
      s1 = q(v1);
      sw = q(vw);
      sw1 = q(vw1);
    }
  }
  if (!emit) return;
  block_xor_out(s1, out);
  block_xor_out(sw, out + 1);
  block_xor_out(sw1, out + 2);
}

__global__ void __launch_bounds__(256) k_mp_scatter(f128* __restrict__ bc, const f128* __restrict__ eq_inst,
                                                    size_t n_inst, MpCoeffs c) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst) return;
  const f128 e = eq_inst[i];
  f128* w = bc + kBlockWords * i;
#pragma unroll
  for (int k = 0; k < 8; k++) w[k] = fx(w[k], fmul(c.c[k], e));
}

}  // namespace

void mp_fold(const f128* z, size_t n_inst, f128 e0, f128 e1, f128* out, cudaStream_t s) {
  count_launch();
  k_mp_fold<<<(unsigned)((n_inst + 255) / 256), 256, 0, s>>>(z, n_inst, e0, e1, out);
}
void mp_tables(const f128* eq_q, const f128* eq_p, f128 alpha, int pos_log, size_t n, const uint8_t* b, f128* ta,
               f128* tb, cudaStream_t s) {
  count_launch();
  k_mp_tables<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(eq_q, eq_p, alpha, pos_log, n, b, ta, tb);
}
void mp_round(const MpTables& T, int len, bool fold, f128 r, bool emit, f128* out, cudaStream_t s) {
  const int threads = std::max(1, len / 2);
  count_launch();
  k_mp_round<<<(threads + 255) / 256, 256, 0, s>>>(T, len, fold, r, emit, out);
}
void mp_scatter(f128* bc, const f128* eq_inst, size_t n_inst, const MpCoeffs& c, cudaStream_t s) {
  count_launch();
  k_mp_scatter<<<(unsigned)((n_inst + 255) / 256), 256, 0, s>>>(bc, eq_inst, n_inst, c);
}
