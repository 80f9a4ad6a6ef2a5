// Hash-chain kernels: the per-instance region fold that collapses each
// instance's input cv (packed words 0, 1 of its block of `per` words: 128 for
// BLAKE3, 256 for SHA-256, whose H_in / H_out slots sit at the same bytes) and
// output (words 2, 3) to one value, and the scatter of the chain's
// packed-direct claim gamma * eq(point) into b_combined.  The claim point is
// [tau_pos, sel0, 0^(log2 per - 2), instance], so eq(point) is nonzero only on
// words 0..3 of each block: eq(point)[per i + w] = c[w] / gamma * eq(instance, i).
// crates/flock-prover/src/r1cs_hashes/chain_common.rs:148-199 (fold_in_out),
// :217-239 (claim point); crates/flock-core/src/pcs.rs:1236-1248 (scatter).
// The shift sumcheck itself runs on k_lc_round (the same top-variable
// product rounds; chain.rs:184-212).
#include "kernels.cuh"

namespace {

__global__ void __launch_bounds__(256) k_chain_fold(const f128* __restrict__ z, size_t n_inst, size_t per, f128 e0,
                                                    f128 e1, f128* __restrict__ g) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst) return;
  const f128* w = z + per * i;
  g[i] = fx(fmul(e0, w[0]), fmul(e1, w[1]));
  g[n_inst + i] = fx(fmul(e0, w[2]), fmul(e1, w[3]));
}

__global__ void __launch_bounds__(256) k_chain_scatter(f128* __restrict__ bc, const f128* __restrict__ eq_inst,
                                                       size_t n_inst, size_t per, f128 c0, f128 c1, f128 c2,
                                                       f128 c3) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst) return;
  const f128 e = eq_inst[i];
  f128* w = bc + per * i;
  w[0] = fx(w[0], fmul(c0, e));
  w[1] = fx(w[1], fmul(c1, e));
  w[2] = fx(w[2], fmul(c2, e));
  w[3] = fx(w[3], fmul(c3, e));
}

}  // namespace

void chain_fold(const f128* z, size_t n_inst, size_t per, f128 e0, f128 e1, f128* g, cudaStream_t s) {
  count_launch();
  k_chain_fold<<<(unsigned)((n_inst + 255) / 256), 256, 0, s>>>(z, n_inst, per, e0, e1, g);
}

void chain_scatter(f128* bc, const f128* eq_inst, size_t n_inst, size_t per, const f128 c[4], cudaStream_t s) {
  count_launch();
  k_chain_scatter<<<(unsigned)((n_inst + 255) / 256), 256, 0, s>>>(bc, eq_inst, n_inst, per, c[0], c[1], c[2],
                                                                    c[3]);
}
