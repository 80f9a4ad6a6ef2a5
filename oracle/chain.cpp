// BLAKE3 hash-chain prover of the oracle (test infrastructure; see
// flockref.hpp).  Restates:
//  * the shift argument, crates/flock-prover/src/chain.rs: shift_mle
//    :75-100, prove_chain_shift :155-236 (tau, alpha, weight table over
//    (y, s0) with s0 the high bit, n+1 degree-2 rounds (q(1), q(inf)) that
//    bind the top variable), verify_chain_shift :238-300;
//  * the generic chain glue, r1cs_hashes/chain_common.rs: tau_pos sampled
//    after the core (:318-320), fold_in_out :148-199, the claim point
//    [tau_pos, sel0, 0^high, instance] of the row-major layout :217-239,
//    fold_public_phys :84-118;
//  * BLAKE3's CHAIN_LAYOUT, r1cs_hashes/blake3.rs:5160-5167: input cv at
//    byte 0, out_lo at byte 32, 256-bit slots (region_log 8), so tau_pos has
//    one coordinate and five slot bits are zero;
//  * the CLI's honest chain, bin/flock_chain.rs:178-193 (SplitMix64) and
//    :236-260 (counter 0, block_len 64, flags 0);
//  * the SHA-256 chain, Sha256HybridSetup::prove_chain (r1cs_hashes/sha2.rs:
//    1557-1589) with CHAIN_LAYOUT (:1476-1483): H_in at byte 0, H_out at byte
//    32, the same 256-bit slots, in 2^15-bit blocks; the CLI's SHA-256 chain
//    (bin/flock_chain.rs:279-316: H_0 = the SHA-256 IV, 16 SplitMix64 words
//    per message); the bundle's hash kind Sha2 (proof_io.rs:51-58);
//  * the Keccak chain, KeccakSetup::prove_chain (keccak.rs:1000-1022) with
//    its CHAIN_LAYOUT (:839-846): state_0 and state_24 in 2048-bit slots
//    (region_log 11: tau_pos has 4 coordinates, the claim point 4 zero slot
//    bits), 1600-bit endpoints (state_to_phys_bits :850-857); the CLI's
//    chain of successive permutations from a start state (flock_chain.rs:
//    319-366).
#include "flockref.hpp"
#include <stdexcept>

namespace flockref {

void compress_cv(const Compression& c, uint32_t out[8]) {
  uint32_t st[16];
  b3::compress_words(c.cv, c.m, c.counter, c.block_len, c.flags, st);
  for (int i = 0; i < 8; i++) out[i] = st[i];
}

std::vector<Compression> chain_blocks(uint64_t seed, const uint32_t initial_cv[8], size_t steps) {
  uint64_t s = seed;
  auto nx = [&]() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  std::vector<Compression> out(steps);
  uint32_t cv[8];
  memcpy(cv, initial_cv, 32);
  for (size_t i = 0; i < steps; i++) {
    Compression& c = out[i];
    memcpy(c.cv, cv, 32);
    for (int w = 0; w < 16; w++) c.m[w] = (uint32_t)nx();
    c.counter = 0;
    c.block_len = 64;
    c.flags = 0;
    compress_cv(c, cv);
  }
  return out;
}

F128 eq_eval(const std::vector<F128>& a, const std::vector<F128>& b) {
  F128 acc = ONE;
  for (size_t i = 0; i < a.size(); i++) acc *= ONE + a[i] + b[i];
  return acc;
}

F128 shift_mle(const std::vector<F128>& a, const std::vector<F128>& b) {
  size_t n = a.size();
  std::vector<F128> pre(n + 1, ONE), suf(n + 1, ONE);
  for (size_t j = 0; j < n; j++) pre[j + 1] = pre[j] * (a[j] * (ONE + b[j]));
  for (size_t j = n; j-- > 0;) suf[j] = suf[j + 1] * (ONE + a[j] + b[j]);
  F128 acc = ZERO;
  for (size_t j = 0; j < n; j++) acc += pre[j] * ((ONE + a[j]) * b[j]) * suf[j + 1];
  return acc;
}

ShiftProof shift_prove(const std::vector<F128>& in, const std::vector<F128>& out, Challenger& ch,
                       ChainClaims& claims) {
  const size_t N = in.size();
  if (N == 0 || (N & (N - 1)) || out.size() != N) throw std::runtime_error("shift: sizes");
  size_t n = 0;
  while (((size_t)1 << n) < N) n++;
  std::vector<F128> tau = ch.sample_f128_vec(n);
  F128 alpha = ch.sample_f128();
  std::vector<F128> eqt = build_eq(tau);
  // W(y, 0) = eq(tau, y - 1) (y >= 1) + alpha [y == 0];  W(y, 1) = eq(tau, y)
  std::vector<F128> w(2 * N, ZERO), g(2 * N);
  for (size_t y = 1; y < N; y++) w[y] = eqt[y - 1];
  w[0] += alpha;
  for (size_t y = 0; y < N; y++) w[N + y] = eqt[y];
  for (size_t y = 0; y < N; y++) { g[y] = in[y]; g[N + y] = out[y]; }
  ShiftProof pf;
  std::vector<F128> rs;
  for (size_t d = 0; d <= n; d++) {
    size_t half = g.size() / 2;
    F128 e1 = ZERO, einf = ZERO;
    for (size_t i = 0; i < half; i++) {
      e1 += w[i + half] * g[i + half];
      einf += (w[i + half] + w[i]) * (g[i + half] + g[i]);
    }
    ch.observe_f128(e1);
    ch.observe_f128(einf);
    F128 r = ch.sample_f128();
    for (size_t i = 0; i < half; i++) {
      w[i] += r * (w[i + half] + w[i]);
      g[i] += r * (g[i + half] + g[i]);
    }
    w.resize(half);
    g.resize(half);
    pf.rounds.push_back({e1, einf});
    rs.push_back(r);
  }
  // round k bound variable n - k: full[n - k] = rs[k]; s0 is variable n
  std::vector<F128> full(n + 1);
  for (size_t k = 0; k <= n; k++) full[n - k] = rs[k];
  claims.instance_point.assign(full.begin(), full.begin() + n);
  claims.sel0 = full[n];
  claims.value = g[0];
  pf.g_at_point = g[0];
  return pf;
}

bool shift_verify(const ShiftProof& pf, F128 x0_r, F128 xlast_r, size_t n, Challenger& ch, ChainClaims& claims) {
  if (pf.rounds.size() != n + 1) return false;
  std::vector<F128> tau = ch.sample_f128_vec(n);
  F128 alpha = ch.sample_f128();
  F128 tau_prod = ONE;
  for (const F128& t : tau) tau_prod *= t;
  F128 claim = tau_prod * xlast_r + alpha * x0_r;
  std::vector<F128> rs;
  for (const auto& rd : pf.rounds) {
    ch.observe_f128(rd.first);
    ch.observe_f128(rd.second);
    F128 r = ch.sample_f128();
    // q(X) = einf X^2 + c1 X + e0 through q(0) = claim + e1, q(1) = e1
    F128 e0 = claim + rd.first;
    F128 c1 = e0 + rd.first + rd.second;
    claim = rd.second * r * r + c1 * r + e0;
    rs.push_back(r);
  }
  std::vector<F128> full(n + 1);
  for (size_t k = 0; k <= n; k++) full[n - k] = rs[k];
  std::vector<F128> taup(full.begin(), full.begin() + n);
  F128 s0 = full[n];
  F128 w_final = shift_mle(tau, taup) * (ONE + s0) + eq_eval(tau, taup) * s0 +
                 alpha * eq_eval(taup, std::vector<F128>(n, ZERO)) * (ONE + s0);
  if (claim != w_final * pf.g_at_point) return false;
  claims.instance_point = taup;
  claims.sel0 = s0;
  claims.value = pf.g_at_point;
  return true;
}

// physical bits of a 256-bit value of 8 u32 words (cv_to_phys_bits,
// blake3.rs:5169-5180, sha2.rs:1487-1495): bit 32 w + b = bit b of word w
static std::vector<uint8_t> phys_of_words(const uint32_t cv[8]) {
  std::vector<uint8_t> p(256);
  for (int i = 0; i < 256; i++) p[i] = (uint8_t)((cv[i / 32] >> (i % 32)) & 1);
  return p;
}
// physical bits of a Keccak state: bit z of lane l at 64 l + z (within_lane_contiguous)
static std::vector<uint8_t> phys_of_lanes(const uint64_t lanes[25]) {
  std::vector<uint8_t> p(1600);
  for (int i = 0; i < 1600; i++) p[i] = (uint8_t)((lanes[i / 64] >> (i % 64)) & 1);
  return p;
}

// fold_public_phys (chain_common.rs:84-118): sum over the region's packed
// positions of eq(tau_pos, pos) times the 128 physical bits there
F128 fold_public_phys(const std::vector<uint8_t>& phys, const std::vector<F128>& tau_pos) {
  const std::vector<F128> eq = build_eq(tau_pos);
  F128 acc = ZERO;
  for (size_t pos = 0; pos < eq.size(); pos++) {
    uint64_t lo = 0, hi = 0;
    for (int b = 0; b < 128; b++) {
      const size_t i = pos * 128 + (size_t)b;
      if (i < phys.size() && phys[i]) (b < 64 ? lo : hi) |= 1ull << (b % 64);
    }
    acc += eq[pos] * F128(lo, hi);
  }
  return acc;
}

// The chain glue after the core (prove_chain_ligerito_generic,
// chain_common.rs:271-346): tau_pos over the region's packed words, the
// input region at words 0.. and the output region at words out_word.. of each
// block of `per` packed words; cb's endpoints are set; `shift_ok` gets the
// oracle's own check of the shift argument.
static CoreHook chain_hook(ChainBundle& cb, size_t N, int n_log, size_t per, int region_log, size_t out_word,
                           bool& shift_ok) {
  return [&cb, N, n_log, per, region_log, out_word, &shift_ok](Challenger& ch, const std::vector<F128>& z) {
    const std::vector<F128> tau_pos = ch.sample_f128_vec((size_t)region_log - 7);
    const std::vector<F128> et = build_eq(tau_pos);
    std::vector<F128> in(N), out(N);
    for (size_t i = 0; i < N; i++) {
      F128 a = ZERO, b = ZERO;
      for (size_t w = 0; w < et.size(); w++) {
        a += et[w] * z[per * i + w];
        b += et[w] * z[per * i + out_word + w];
      }
      in[i] = a;
      out[i] = b;
    }
    Challenger vch = ch;  // the verifier's transcript from here on
    ChainClaims cl;
    cb.shift = shift_prove(in, out, ch, cl);
    ChainClaims vcl;
    shift_ok = shift_verify(cb.shift, fold_public_phys(cb.phys0, tau_pos), fold_public_phys(cb.phys_last, tau_pos),
                            (size_t)n_log, vch, vcl) &&
               vcl.value == cl.value && vcl.sel0 == cl.sel0 && vcl.instance_point == cl.instance_point;
    // [tau_pos, sel0, 0^(k_log - region_log - 1), instance] (chain_common.rs:211-231)
    DirectClaim dc;
    dc.point = tau_pos;
    dc.point.push_back(cl.sel0);
    int k_log = 7;
    for (size_t p2 = per; p2 > 1; p2 >>= 1) k_log++;
    for (int i = 0; i < k_log - region_log - 1; i++) dc.point.push_back(ZERO);
    dc.point.insert(dc.point.end(), cl.instance_point.begin(), cl.instance_point.end());
    dc.value = cl.value;
    return std::vector<DirectClaim>{dc};
  };
}

ChainBundle prove_chain(const std::vector<Compression>& blocks, int n_log, const std::string& domain,
                        bool* check, const uint32_t* claimed_cv_last) {
  const size_t N = (size_t)1 << n_log;
  if (blocks.size() != N) throw std::runtime_error("prove_chain: the chain must fill 2^n_log slots");
  ChainBundle cb;
  uint32_t last[8];
  compress_cv(blocks[N - 1], last);
  cb.phys0 = phys_of_words(blocks[0].cv);
  cb.phys_last = phys_of_words(claimed_cv_last ? claimed_cv_last : last);
  bool shift_ok = false;
  cb.core = prove_with(blocks, n_log, domain, chain_hook(cb, N, n_log, 128, 8, 2, shift_ok));
  if (check) *check = shift_ok && last_open_identity_ok();
  return cb;
}

std::vector<sha::Compression> sha256_chain_blocks(uint64_t seed, const uint32_t initial[8], size_t steps) {
  uint64_t s = seed;
  auto nx = [&]() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  std::vector<sha::Compression> out(steps);
  uint32_t h[8];
  memcpy(h, initial, 32);
  for (size_t i = 0; i < steps; i++) {
    memcpy(out[i].h, h, 32);
    for (int w = 0; w < 16; w++) out[i].m[w] = (uint32_t)nx();
    sha::compress(out[i].h, out[i].m, h);
  }
  return out;
}

ChainBundle prove_sha256_chain(const std::vector<sha::Compression>& blocks, int n_log, const std::string& domain,
                               bool* check, const uint32_t* claimed_cv_last) {
  const size_t N = (size_t)1 << n_log;
  if (blocks.size() != N) throw std::runtime_error("prove_chain: the chain must fill 2^n_log slots");
  ChainBundle cb;
  cb.kind = 1;  // HashKind::Sha2
  uint32_t last[8];
  sha::compress(blocks[N - 1].h, blocks[N - 1].m, last);
  cb.phys0 = phys_of_words(blocks[0].h);
  cb.phys_last = phys_of_words(claimed_cv_last ? claimed_cv_last : last);
  bool shift_ok = false;
  std::vector<F128> z, a, b;
  generate_sha256_witness(blocks, n_log, z, a, b);
  cb.core = prove_core(sha256_r1cs(n_log), std::move(z), a, b, domain,
                       chain_hook(cb, N, n_log, (size_t)1 << (15 - 7), 8, 2, shift_ok));
  if (check) *check = shift_ok && last_open_identity_ok();
  return cb;
}

ChainBundle prove_keccak_chain(const std::vector<keccak::State>& states, int n_log, const std::string& domain,
                               bool* check, const uint64_t* claimed_last) {
  const size_t N = (size_t)1 << n_log;
  if (states.size() != N) throw std::runtime_error("prove_chain: the chain must fill 2^n_log slots");
  ChainBundle cb;
  cb.kind = 2;  // HashKind::Keccak
  keccak::State last = states[N - 1];
  keccak::permute(last.lanes);
  cb.phys0 = phys_of_lanes(states[0].lanes);
  cb.phys_last = phys_of_lanes(claimed_last ? claimed_last : last.lanes);
  bool shift_ok = false;
  const keccak::Layout& L = keccak::single_layout();
  std::vector<F128> z, a, b;
  generate_keccak_witness(L, states, n_log, z, a, b);
  cb.core = prove_core(keccak_r1cs(L, n_log), std::move(z), a, b, domain,
                       chain_hook(cb, N, n_log, (size_t)1 << (16 - 7), 11, 16, shift_ok));
  if (check) *check = shift_ok && last_open_identity_ok();
  return cb;
}

}  // namespace flockref
