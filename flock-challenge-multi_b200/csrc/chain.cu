// Hash-chain kernels: the per-instance region fold that collapses each
// instance's input region (packed words 0..R-1 of its block of `per` words)
// and output region (words out_word..out_word+R-1) to one value apiece, with
// weights eq(tau_pos, w): R = 2 for BLAKE3 and SHA-256 (256-bit slots at
// words 0 and 2), 16 for Keccak (2048-bit slots at words 0 and 16); and the
// scatter of the chain's packed-direct claim gamma * eq(point) into
// b_combined.  The claim point is [tau_pos, sel0, 0^high, instance], so
// eq(point) is nonzero only on words 0..2R-1 of each block:
// eq(point)[per i + w] = c[w] / gamma * eq(instance, i).
// crates/flock-prover/src/r1cs_hashes/chain_common.rs:148-199 (fold_in_out),
// :217-239 (claim point); crates/flock-core/src/pcs.rs:1236-1248 (scatter).
// The shift sumcheck itself runs on k_lc_round (the same top-variable
// product rounds; chain.rs:184-212).
#include "kernels.cuh"

namespace {
struct FoldCoefs {
  f128 e[16];  // eq(tau_pos, w) for the R packed words of a region
  int R, out_word;
};
struct ScatterCoefs {
  f128 c[32];  // gamma eq(point) restricted to the block's first W words
  int W;
};

__global__ void __launch_bounds__(256) k_chain_fold(const f128* __restrict__ z, size_t n_inst, size_t per,
                                                    FoldCoefs F, f128* __restrict__ g) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst) return;
  const f128* w = z + per * i;
  f128 in = mk(0, 0), out = mk(0, 0);
  for (int k = 0; k < F.R; k++) {
    in = fx(in, fmul(F.e[k], ldg(w + k)));
    out = fx(out, fmul(F.e[k], ldg(w + F.out_word + k)));
  }
  g[i] = in;
  g[n_inst + i] = out;
}

__global__ void __launch_bounds__(256) k_chain_scatter(f128* __restrict__ bc, const f128* __restrict__ eq_inst,
                                                       size_t n_inst, size_t per, ScatterCoefs S) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst) return;
  const f128 e = eq_inst[i];
  f128* w = bc + per * i;
  for (int k = 0; k < S.W; k++) w[k] = fx(w[k], fmul(S.c[k], e));
}

}  // namespace

void chain_fold(const f128* z, size_t n_inst, size_t per, const f128* e, int R, int out_word, f128* g,
                cudaStream_t s) {
  if (R < 1 || R > 16) throw CudaError("chain_fold: at most 16 packed words per region");
  FoldCoefs F;
  for (int k = 0; k < R; k++) F.e[k] = e[k];
  F.R = R;
  F.out_word = out_word;
  count_launch();
  k_chain_fold<<<(unsigned)((n_inst + 255) / 256), 256, 0, s>>>(z, n_inst, per, F, g);
}

void chain_scatter(f128* bc, const f128* eq_inst, size_t n_inst, size_t per, const f128* c, int W, cudaStream_t s) {
  if (W < 1 || W > 32) throw CudaError("chain_scatter: at most 32 words");
  ScatterCoefs S;
  for (int k = 0; k < W; k++) S.c[k] = c[k];
  S.W = W;
  count_launch();
  k_chain_scatter<<<(unsigned)((n_inst + 255) / 256), 256, 0, s>>>(bc, eq_inst, n_inst, per, S);
}
