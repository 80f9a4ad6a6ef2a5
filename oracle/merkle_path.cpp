// SHA-256 Merkle-path prover of the oracle (test infrastructure; see
// flockref.hpp).  Restates:
//  * the Merkle-path shift sumcheck, crates/flock-prover/src/merkle_path.rs:
//    OMEGA and lagrange_eval_degree3 :114-169, slot_indicator :171-183,
//    prove_merkle_path_shift :226-467 (tau, alpha, the factor tables
//    T_shift_alpha / T_eq / T_b with B := 0 on the first row of every path,
//    n degree-3 rounds binding the top instance variable with messages
//    (q(1), q(w), q(w+1)), then two degree-2 rounds over the slot selector
//    (sd first, then ss)), verify_merkle_path_shift :469-590;
//  * the generic glue, r1cs_hashes/merkle_path_common.rs: tau_pos sampled
//    after the core, fold_all_slots :180-225, the row-major claim point
//    [tau_pos, sel_slot, side, 0^high, instance] :262-282, fold_public_phys
//    :124-150, prove/verify_merkle_paths_ligerito_generic :314-537;
//  * SHA-256's MERKLE_LAYOUT, r1cs_hashes/sha2.rs:1634-1645: 256-bit slots
//    at byte 0 (slot 0 H_in, 1 H_out = Z, 2 M_lo = X_L, 3 M_hi = X_R), so
//    tau_pos has one coordinate and 15 - 8 - 2 = 5 slot bits are zero;
//  * the honest path of benches/sha2_merkle_proof.rs:49-76 (every H_in the
//    SHA-256 IV; SplitMix64 draws, low 32 bits) and the replicated paths of
//    the multi-path tests, sha2.rs:2475-2497.
#include "flockref.hpp"
#include <stdexcept>

namespace flockref {

namespace {
const F128 OMEGA(2, 0);

F128 lagrange3(F128 q0, F128 q1, F128 qw, F128 qw1, F128 r) {
  const F128 w = OMEGA, w1 = OMEGA + ONE;
  const F128 l0 = (r + ONE) * (r + w) * (r + w1) * f128_inv(w * w1);
  const F128 l1 = r * (r + w) * (r + w1) * f128_inv((ONE + w) * w);
  const F128 l2 = r * (r + ONE) * (r + w1) * f128_inv(w * w1);
  const F128 l3 = r * (r + ONE) * (r + w) * f128_inv(w1 * w);
  return q0 * l0 + q1 * l1 + qw * l2 + qw1 * l3;
}

F128 slot_ind(int s, F128 ss, F128 sd) {
  return ((s & 1) ? ss : ONE + ss) * (((s >> 1) & 1) ? sd : ONE + sd);
}

// SHA-256 MERKLE_LAYOUT
constexpr int Z_SLOT = 1, XL_SLOT = 2, XR_SLOT = 3, OTHER_SLOT = 0;

F128 fold_hash(const uint32_t h[8], F128 tau_pos) {
  F128 p0((uint64_t)h[0] | (uint64_t)h[1] << 32, (uint64_t)h[2] | (uint64_t)h[3] << 32);
  F128 p1((uint64_t)h[4] | (uint64_t)h[5] << 32, (uint64_t)h[6] | (uint64_t)h[7] << 32);
  return (ONE + tau_pos) * p0 + tau_pos * p1;
}
}  // namespace

MerkleShiftProof mp_shift_prove(int path_log, const std::vector<F128> slot[4], const std::vector<uint8_t>& b_bits,
                                Challenger& ch, MerkleClaims& claims) {
  const size_t N = slot[0].size();
  int n = 0;
  while (((size_t)1 << n) < N) n++;
  if (((size_t)1 << n) != N || b_bits.size() != N || path_log > n) throw std::runtime_error("merkle shift: sizes");
  const int pos_log = n - path_log;
  const size_t n_pos = (size_t)1 << pos_log;
  std::vector<F128> tau = ch.sample_f128_vec(n);
  const F128 alpha = ch.sample_f128();
  std::vector<F128> tq(tau.begin(), tau.begin() + pos_log), tp(tau.begin() + pos_log, tau.end());
  std::vector<F128> eq_tau = build_eq(tau), eq_p = build_eq(tp), eq_q = build_eq(tq);
  std::vector<F128> ta(N), te = eq_tau, tb(N);
  for (size_t i = 0; i < N; i++) {
    const size_t ip = i >> pos_log, iq = i & (n_pos - 1);
    ta[i] = eq_p[ip] * (iq == 0 ? alpha : eq_q[iq - 1]);
    tb[i] = (b_bits[i] && iq != 0) ? ONE : ZERO;
  }
  std::vector<F128> gz = slot[Z_SLOT], gxl = slot[XL_SLOT], gxr = slot[XR_SLOT], go = slot[OTHER_SLOT];
  MerkleShiftProof pf;
  std::vector<F128> rs;
  const F128 pts[3] = {ONE, OMEGA, OMEGA + ONE};
  auto at = [](const std::vector<F128>& t, size_t i, size_t h, F128 x) { return t[i] + x * (t[i + h] + t[i]); };
  for (int round = 0; round < n; round++) {
    const size_t h = ta.size() / 2;
    F128 s[3] = {ZERO, ZERO, ZERO};
    for (int e = 0; e < 3; e++) {
      const F128 x = pts[e];
      F128 acc = ZERO;
      for (size_t i = 0; i < h; i++) {
        const F128 a = at(ta, i, h, x), q = at(te, i, h, x), b = at(tb, i, h, x);
        acc += q * at(gz, i, h, x) + a * (ONE + b) * at(gxl, i, h, x) + a * b * at(gxr, i, h, x);
      }
      s[e] = acc;
    }
    for (int e = 0; e < 3; e++) ch.observe_f128(s[e]);
    const F128 r = ch.sample_f128();
    pf.rounds.push_back({s[0], s[1], s[2]});
    rs.push_back(r);
    for (std::vector<F128>* t : {&ta, &te, &tb, &gz, &gxl, &gxr, &go}) {
      for (size_t i = 0; i < h; i++) (*t)[i] = at(*t, i, h, r);
      t->resize(h);
    }
  }
  F128 w[4] = {ZERO, ZERO, ZERO, ZERO}, g[4];
  w[Z_SLOT] = te[0];
  w[XL_SLOT] = ta[0] * (ONE + tb[0]);
  w[XR_SLOT] = ta[0] * tb[0];
  g[Z_SLOT] = gz[0];
  g[XL_SLOT] = gxl[0];
  g[XR_SLOT] = gxr[0];
  g[OTHER_SLOT] = go[0];
  std::vector<F128> wv(w, w + 4), gv(g, g + 4);
  for (int round = 0; round < 2; round++) {
    const size_t h = wv.size() / 2;
    F128 s[3] = {ZERO, ZERO, ZERO};
    for (int e = 0; e < 3; e++)
      for (size_t i = 0; i < h; i++) s[e] += at(wv, i, h, pts[e]) * at(gv, i, h, pts[e]);
    for (int e = 0; e < 3; e++) ch.observe_f128(s[e]);
    const F128 r = ch.sample_f128();
    pf.rounds.push_back({s[0], s[1], s[2]});
    rs.push_back(r);
    for (size_t i = 0; i < h; i++) { wv[i] = at(wv, i, h, r); gv[i] = at(gv, i, h, r); }
    wv.resize(h);
    gv.resize(h);
  }
  pf.g_at_point = gv[0];
  claims.instance_point.resize(n);
  for (int j = 0; j < n; j++) claims.instance_point[j] = rs[n - 1 - j];
  claims.side = rs[n];
  claims.sel_slot = rs[n + 1];
  claims.value = gv[0];
  return pf;
}

bool mp_shift_verify(int path_log, const MerkleShiftProof& pf, const std::vector<F128>& leaf_evals, F128 root_r,
                     const std::vector<uint8_t>& b_bits, int n, Challenger& ch, MerkleClaims& claims) {
  if (pf.rounds.size() != (size_t)n + 2) return false;
  const int pos_log = n - path_log;
  std::vector<F128> tau = ch.sample_f128_vec(n);
  const F128 alpha = ch.sample_f128();
  std::vector<F128> tq(tau.begin(), tau.begin() + pos_log), tp(tau.begin() + pos_log, tau.end());
  F128 ones = ONE;
  for (const F128& t : tq) ones *= t;
  std::vector<F128> eq_p = build_eq(tp);
  F128 leaf = ZERO;
  for (size_t i = 0; i < eq_p.size(); i++) leaf += eq_p[i] * leaf_evals[i];
  F128 claim = ones * root_r + alpha * leaf;
  std::vector<F128> rs;
  for (const auto& m : pf.rounds) {
    for (const F128& v : m) ch.observe_f128(v);
    const F128 r = ch.sample_f128();
    claim = lagrange3(claim + m[0], m[0], m[1], m[2], r);
    rs.push_back(r);
  }
  std::vector<F128> ip(n);
  for (int j = 0; j < n; j++) ip[j] = rs[n - 1 - j];
  const F128 side = rs[n], sel = rs[n + 1];
  std::vector<F128> yq(ip.begin(), ip.begin() + pos_log), yp(ip.begin() + pos_log, ip.end());
  F128 z0 = ONE;
  for (const F128& t : yq) z0 *= ONE + t;
  const F128 ta = eq_eval(tp, yp) * (shift_mle(tq, yq) + alpha * z0);
  const F128 te = eq_eval(tau, ip);
  std::vector<F128> eq_ip = build_eq(ip);
  F128 tb = ZERO;
  const size_t n_pos = (size_t)1 << pos_log;
  for (size_t i = 0; i < b_bits.size(); i++)
    if (b_bits[i] && (i & (n_pos - 1)) != 0) tb += eq_ip[i];
  const F128 w = slot_ind(Z_SLOT, sel, side) * te + slot_ind(XL_SLOT, sel, side) * ta * (ONE + tb) +
                 slot_ind(XR_SLOT, sel, side) * ta * tb;
  if (claim != w * pf.g_at_point) return false;
  claims.instance_point = ip;
  claims.side = side;
  claims.sel_slot = sel;
  claims.value = pf.g_at_point;
  return true;
}

MerklePathInputs sha256_merkle_paths(int n_log, int path_log, uint64_t seed) {
  const size_t N = (size_t)1 << n_log, L = N >> path_log;
  uint64_t s = seed;
  auto nx = [&]() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return (uint32_t)(z ^ (z >> 31));
  };
  MerklePathInputs in;
  uint32_t leaf[8], cur[8];
  for (int i = 0; i < 8; i++) leaf[i] = nx();
  std::vector<uint8_t> b(L, 0);
  for (size_t i = 1; i < L; i++) b[i] = nx() & 1;
  std::vector<sha::Compression> path(L);
  memcpy(cur, leaf, 32);
  for (size_t i = 0; i < L; i++) {
    uint32_t sib[8];
    for (int k = 0; k < 8; k++) sib[k] = nx();
    sha::Compression& c = path[i];
    memcpy(c.h, sha::IV, 32);
    memcpy(c.m + (b[i] ? 8 : 0), cur, 32);
    memcpy(c.m + (b[i] ? 0 : 8), sib, 32);
    sha::compress(c.h, c.m, cur);
  }
  for (size_t p = 0; p < ((size_t)1 << path_log); p++) {
    in.blocks.insert(in.blocks.end(), path.begin(), path.end());
    in.b_bits.insert(in.b_bits.end(), b.begin(), b.end());
    in.leaves.push_back(std::array<uint32_t, 8>());
    memcpy(in.leaves.back().data(), leaf, 32);
  }
  memcpy(in.root.data(), cur, 32);
  return in;
}

MerkleBundle prove_sha256_merkle(const MerklePathInputs& in, int n_log, int path_log, const std::string& domain,
                                 bool* check) {
  const size_t N = (size_t)1 << n_log;
  if (in.blocks.size() != N || in.b_bits.size() != N || in.leaves.size() != ((size_t)1 << path_log))
    throw std::runtime_error("prove_sha256_merkle: the paths must fill 2^n_log slots");
  MerkleBundle mb;
  bool shift_ok = false;
  CoreHook hook = [&](Challenger& ch, const std::vector<F128>& z) {
    const F128 tp = ch.sample_f128_vec(1)[0];
    // fold_all_slots: slot s of block i is words 2s, 2s + 1 (256 words per block)
    std::vector<F128> slot[4];
    for (int s = 0; s < 4; s++) {
      slot[s].resize(N);
      for (size_t i = 0; i < N; i++) slot[s][i] = (ONE + tp) * z[256 * i + 2 * s] + tp * z[256 * i + 2 * s + 1];
    }
    Challenger vch = ch;  // the verifier's transcript from here on
    MerkleClaims cl, vcl;
    mb.shift = mp_shift_prove(path_log, slot, in.b_bits, ch, cl);
    std::vector<F128> leaf_evals;
    for (const auto& l : in.leaves) leaf_evals.push_back(fold_hash(l.data(), tp));
    shift_ok = mp_shift_verify(path_log, mb.shift, leaf_evals, fold_hash(in.root.data(), tp), in.b_bits, n_log, vch,
                               vcl) &&
               vcl.value == cl.value && vcl.instance_point == cl.instance_point;
    DirectClaim dc;
    dc.point = {tp, cl.sel_slot, cl.side};
    for (int i = 0; i < 5; i++) dc.point.push_back(ZERO);
    dc.point.insert(dc.point.end(), cl.instance_point.begin(), cl.instance_point.end());
    dc.value = cl.value;
    return std::vector<DirectClaim>{dc};
  };
  std::vector<F128> z, a, b;
  generate_sha256_witness(in.blocks, n_log, z, a, b);
  mb.core = prove_core(sha256_r1cs(n_log), std::move(z), a, b, domain, hook);
  if (check) *check = shift_ok && last_open_identity_ok();
  return mb;
}

}  // namespace flockref
