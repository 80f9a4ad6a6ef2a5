// Additive NTTs and Merkle trees of the oracle (test infrastructure; see
// flockref.hpp).
//  * F128 LCH NTT: crates/flock-core/src/ntt/additive_ntt_f128.rs — subspace
//    evals :54-87, breadth-first twiddles :108-131, twiddle(l,b) :2684-2693,
//    scalar interleaved forward :4766-4800; RS encode == zero-pad + full
//    forward (pcs/commit.rs:1838-1877 commit_matches_full_ntt_oracle).
//  * GF(2^8) NTT: crates/flock-core/src/ntt.rs:22-169.
//  * Merkle: crates/flock-core/src/merkle.rs — flat layout :16-21,
//    fill_merkle_tree :777-812, merkle_multi_proof :1020-1058.
#include "flockref.hpp"
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>

namespace flockref {

AdditiveNtt::AdditiveNtt(int d) : dim(d) {
  std::vector<F128> basis(d);
  for (int i = 0; i < d; i++) basis[i] = F128(1ull << i, 0);
  evals.push_back(basis);
  for (int i = 1; i < d; i++) {
    std::vector<F128> row;
    const std::vector<F128>& prev = evals[i - 1];
    for (size_t k = 1; k < prev.size(); k++) row.push_back(prev[k] * (prev[k] + prev[0]));
    evals.push_back(row);
  }
  for (auto& row : evals) {
    F128 inv = f128_inv(row[0]);
    for (auto& v : row) v = v * inv;
  }
  twiddles.clear();
  for (int layer = 0; layer < d; layer++) {
    size_t start = twiddles.size();
    const std::vector<F128>& er = evals[d - layer - 1];
    twiddles.push_back(ZERO);
    for (size_t bit = 0; bit + 1 < er.size(); bit++) {
      size_t half = (size_t)1 << bit;
      for (size_t b = 0; b < half; b++) twiddles.push_back(twiddles[start + b] + er[bit + 1]);
    }
  }
}

void AdditiveNtt::forward_interleaved(std::vector<F128>& data, size_t num_ntts, int start_layer) const {
  size_t n_pos = data.size() / num_ntts;
  int log_d = 0;
  while (((size_t)1 << log_d) < n_pos) log_d++;
  for (int layer = start_layer; layer < log_d; layer++) {
    size_t num_blocks = (size_t)1 << layer;
    size_t half = (size_t)1 << (log_d - layer - 1);
    par_for(num_blocks * half, [&](size_t i0, size_t i1, int) {
      size_t blk_t = ~(size_t)0;
      F128 t;
      for (size_t i = i0; i < i1; i++) {
        const size_t blk = i / half, row = i % half;
        if (blk != blk_t) { t = twiddle(layer, blk); blk_t = blk; }
        size_t start = blk * 2 * half * num_ntts;
        size_t top = start + row * num_ntts, bot = top + half * num_ntts;
        for (size_t lane = 0; lane < num_ntts; lane++) {
          F128 v = data[bot + lane];
          F128 u = data[top + lane] + v * t;
          data[top + lane] = u;
          data[bot + lane] = v + u;
        }
      }
    });
  }
}

const AdditiveNtt& standard_ntt(int dim) {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<AdditiveNtt>> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto& p = cache[dim];
  if (!p) p.reset(new AdditiveNtt(dim));
  return *p;
}

void rs_encode(const std::vector<F128>& msg, size_t lanes, int log_inv_rate, std::vector<F128>& cw) {
  cw.assign(msg.size() << log_inv_rate, ZERO);
  std::copy(msg.begin(), msg.end(), cw.begin());
  size_t n_pos = cw.size() / lanes;
  int log_d = 0;
  while (((size_t)1 << log_d) < n_pos) log_d++;
  standard_ntt(log_d).forward_interleaved(cw, lanes, 0);
}

// ---- GF(2^8) additive NTT (ntt.rs:22-169) ----
static uint8_t next_s8(uint8_t s, uint8_t root) { return gf8_mul(s, s) ^ gf8_mul(root, s); }

Gf8Ntt::Gf8Ntt(int k_, uint8_t beta) : k(k_) {
  size_t n = (size_t)1 << k;
  tw.assign(n - 1, 0);
  size_t len = n >> 1;
  std::vector<uint8_t> layer(len);
  for (size_t i = 0; i < len; i++) layer[i] = beta ^ (uint8_t)(2 * i);
  uint8_t s_at_root = 1;
  size_t write_at = len;
  for (size_t i = 0; i < len; i++) tw[write_at - 1 + i] = layer[i];
  for (int it = 1; it < k; it++) {
    write_at >>= 1;
    uint8_t next_root = next_s8(layer[1] ^ layer[0], s_at_root);
    size_t new_len = write_at;
    for (size_t i = 0; i < new_len; i++) layer[i] = next_s8(layer[2 * i], s_at_root);
    len = new_len;
    s_at_root = next_root;
    uint8_t inv = gf8_inv(s_at_root);
    for (size_t j = 0; j < len; j++) tw[write_at - 1 + j] = gf8_mul(inv, layer[j]);
  }
}

static void fft_rec(uint8_t* v, size_t n, const uint8_t* tw, size_t idx) {
  if (n == 1) return;
  size_t half = n >> 1;
  uint8_t lam = tw[idx - 1];
  for (size_t i = 0; i < half; i++) {
    uint8_t w = v[half + i];
    v[i] ^= gf8_mul(lam, w);
    v[half + i] = w ^ v[i];
  }
  fft_rec(v, half, tw, 2 * idx);
  fft_rec(v + half, half, tw, 2 * idx + 1);
}
static void ifft_rec(uint8_t* v, size_t n, const uint8_t* tw, size_t idx) {
  if (n == 1) return;
  size_t half = n >> 1;
  ifft_rec(v, half, tw, 2 * idx);
  ifft_rec(v + half, half, tw, 2 * idx + 1);
  uint8_t lam = tw[idx - 1];
  for (size_t i = 0; i < half; i++) {
    v[half + i] ^= v[i];
    v[i] ^= gf8_mul(lam, v[half + i]);
  }
}
void Gf8Ntt::forward(uint8_t* v) const { fft_rec(v, (size_t)1 << k, tw.data(), 1); }
void Gf8Ntt::inverse(uint8_t* v) const { ifft_rec(v, (size_t)1 << k, tw.data(), 1); }

// ---- Merkle ----
std::vector<Hash> merkle_tree(const uint8_t* data, size_t n_leaves, size_t leaf_size, int kind) {
  std::vector<Hash> tree(2 * n_leaves - 1);
  par_for(n_leaves, [&](size_t i0, size_t i1, int) {
    for (size_t i = i0; i < i1; i++) {
      if (kind == SHA256) sha::hash(data + i * leaf_size, leaf_size, tree[i].data());
      else b3::leaf_cv(data + i * leaf_size, leaf_size, tree[i].data());
    }
  });
  size_t rs = 0, rl = n_leaves;
  while (rl > 1) {
    size_t nl = rl >> 1;
    par_for(nl, [&](size_t j0, size_t j1, int) {
      for (size_t j = j0; j < j1; j++) {
        if (kind == SHA256) {
          uint8_t lr[64];
          memcpy(lr, tree[rs + 2 * j].data(), 32);
          memcpy(lr + 32, tree[rs + 2 * j + 1].data(), 32);
          sha::hash(lr, 64, tree[rs + rl + j].data());
        } else {
          b3::parent_cv(tree[rs + 2 * j].data(), tree[rs + 2 * j + 1].data(), tree[rs + rl + j].data());
        }
      }
    });
    rs += rl;
    rl = nl;
  }
  return tree;
}

std::vector<Hash> merkle_multi_proof(const std::vector<Hash>& tree, size_t n_leaves, std::vector<size_t> act) {
  std::vector<Hash> proof;
  if (act.empty() || n_leaves == 1) return proof;
  std::sort(act.begin(), act.end());
  act.erase(std::unique(act.begin(), act.end()), act.end());
  size_t ls = 0, ll = n_leaves;
  while (ll > 1) {
    size_t written = 0, i = 0;
    while (i < act.size()) {
      size_t p = act[i];
      bool sib = i + 1 < act.size() && act[i + 1] == (p ^ 1);
      if (sib) i += 2;
      else { proof.push_back(tree[ls + (p ^ 1)]); i += 1; }
      act[written++] = p >> 1;
    }
    act.resize(written);
    ls += ll;
    ll >>= 1;
  }
  return proof;
}

}  // namespace flockref
