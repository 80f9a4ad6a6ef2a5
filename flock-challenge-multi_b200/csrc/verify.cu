// Verifier of FLOCK v4 bundles for the self-checking prover: the compression
// statement (Blake3Setup::verify -> verifier::verify_ligerito,
// crates/flock-core/src/verifier.rs:95-232) and the hash-chain statement
// (Blake3Setup::verify_chain, r1cs_hashes/blake3.rs:5217-5240 ->
// chain_common.rs:355-420).  It replays the transcript and checks, in the
// reference verifier's order:
//  * the zerocheck rounds and its final product (zerocheck.rs:1642-1797);
//  * the lincheck rounds against the folded matrix combination
//    (lincheck.rs:5876-6050) -- the one O(statement) step, which runs on
//    this setup's device copy of the block matrices with the prover's own
//    comb kernel (k_lc_comb);
//  * for chains, the shift argument from the public endpoints
//    (chain.rs:238-300);
//  * each ring switch's claim (ring_switch.rs:4783-4811), the batched open's
//    target (pcs.rs:1861-1990) and the Ligerito proof
//    (pcs/ligerito.rs:11321-11834): proof-of-work nonces, Merkle
//    multi-proofs of every opened row (merkle.rs:1122-1190), the induced
//    sums, and the final inner product against the residual basis, whose
//    ring-switch part is evaluated in the 128 x 128 tensor algebra
//    (pcs/tensor_algebra.rs, ring_switch.rs:4864-4935).
#include "prover.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

namespace flock {
namespace {

// ---------------------------------------------------------------- decode --
struct Rd {
  const uint8_t* p;
  size_t n, i = 0;
  bool bad = false;
  bool need(size_t k) {
    if (bad || n - i < k) bad = true;
    return !bad;
  }
  uint64_t u64() {
    if (!need(8)) return 0;
    uint64_t v = 0;
    for (int k = 0; k < 8; k++) v |= (uint64_t)p[i + k] << (8 * k);
    i += 8;
    return v;
  }
  uint32_t u32() {
    if (!need(4)) return 0;
    uint32_t v = 0;
    for (int k = 0; k < 4; k++) v |= (uint32_t)p[i + k] << (8 * k);
    i += 4;
    return v;
  }
  f128 f() {
    uint64_t lo = u64(), hi = u64();
    return mk(lo, hi);
  }
  H32 h() {
    H32 v{};
    if (need(32)) { memcpy(v.data(), p + i, 32); i += 32; }
    return v;
  }
  // a length prefix, bounded by what the remaining bytes can hold
  size_t len(size_t elem_bytes) {
    uint64_t v = u64();
    if (bad || v > (n - i) / elem_bytes) { bad = true; return 0; }
    return (size_t)v;
  }
  std::vector<f128> fs() {
    std::vector<f128> v(len(16));
    for (auto& x : v) x = f();
    return v;
  }
  std::vector<H32> hs() {
    std::vector<H32> v(len(32));
    for (auto& x : v) x = h();
    return v;
  }
  std::vector<std::pair<f128, f128>> pairs() {
    std::vector<std::pair<f128, f128>> v(len(32));
    for (auto& x : v) { x.first = f(); x.second = f(); }
    return v;
  }
  std::vector<uint64_t> u64s() {
    std::vector<uint64_t> v(len(8));
    for (auto& x : v) x = u64();
    return v;
  }
  Opening open() {
    Opening o;
    o.rows.resize(len(8));
    for (auto& r : o.rows) r = fs();
    o.proof = hs();
    return o;
  }
  // a Vec<bool> of at most 2048 bits into words (bit b = bit b % 64 of word b / 64)
  bool bools(uint64_t words[32], int& nbits) {
    const uint64_t len = u64();
    if (len > 2048 || !need(len)) return false;
    memset(words, 0, 32 * sizeof(uint64_t));
    for (uint64_t b = 0; b < len; b++) {
      uint8_t v = p[i + b];
      if (v > 1) return false;
      words[b / 64] |= (uint64_t)v << (b % 64);
    }
    i += len;
    nbits = (int)len;
    return true;
  }
};

// FLOCK v4 R1csProofBundleLigerito (flavor 2) or ChainProofBundleLigerito
// (flavor 3), the inverse of encode()
// merkle: the header-less bincode of (Commitment, MerklePathProofLigerito)
bool decode(const uint8_t* bytes, size_t n, Proof& P, std::string& why, bool merkle = false) {
  Rd r{bytes, n};
  if (!merkle) {
    if (n < 7 || memcmp(bytes, "FLOCK", 5) != 0) return why = "bad magic", false;
    if (bytes[5] != 4) return why = "unsupported version", false;
    if (bytes[6] != 2 && bytes[6] != 3) return why = "unknown flavor", false;
    r.i = 7;
  }
  P.merkle = merkle;
  P.chain = !merkle && bytes[6] == 3;
  if (P.chain) {
    P.chain_kind = r.u32();
    if (P.chain_kind > 2) return why = "unknown chain hash kind", false;
  }
  P.root = r.h();
  P.m = r.u64();
  if (r.u64() != 1 || r.u64() != 6 || r.u32() != 0) return why = "PCS parameters are not (rate 1/2, batch 2^6, Fast)", false;
  P.merkle_fn = (int)r.u32();
  if (P.merkle_fn != kFnSha256 && P.merkle_fn != kFnBlake3) return why = "unknown Merkle hash", false;
  P.r1_ab = r.fs();
  P.r1_c = r.fs();
  P.zc_rounds = r.pairs();
  P.fa = r.f();
  P.fb = r.f();
  P.fc = r.f();
  P.lc_rounds = r.pairs();
  P.z_partial = r.fs();
  if (P.chain) {
    P.shift_rounds = r.pairs();
    P.g_at_point = r.f();
  }
  if (P.merkle) {
    P.mp_rounds.resize(r.len(48));
    for (auto& q : P.mp_rounds)
      for (f128& v : q) v = r.f();
    P.g_at_point = r.f();
  }
  P.s_hat_v.resize(r.len(8));
  for (auto& v : P.s_hat_v) v = r.fs();
  P.lig_root = r.h();
  P.initial = r.open();
  P.roots = r.hs();
  P.levels.resize(r.len(16));
  for (auto& l : P.levels) l = r.open();
  P.yr = r.fs();
  P.final_open = r.open();
  P.sc_msgs = r.pairs();
  P.grind_nonces = r.u64s();
  P.ood = r.fs();
  P.fold_nonces = r.u64s();
  int last_bits = 0;
  if (P.chain && (!r.bools(P.end0, P.end_bits) || !r.bools(P.end_last, last_bits) || last_bits != P.end_bits))
    return why = "chain endpoints", false;
  if (r.bad) return why = "truncated", false;
  if (r.i != n) return why = "trailing bytes", false;
  return true;
}

// ----------------------------------------------------------- field utils --
bool feq(f128 a, f128 b) { return a.lo == b.lo && a.hi == b.hi; }
f128 ip(const f128* a, const f128* b, size_t n) {
  f128 s = mk(0, 0);
  for (size_t i = 0; i < n; i++) s = fx(s, hmul(a[i], b[i]));
  return s;
}
f128 eq_eval(const f128* a, const f128* b, size_t n) {
  f128 acc = hone();
  for (size_t i = 0; i < n; i++) acc = hmul(acc, fx(hone(), fx(a[i], b[i])));
  return acc;
}
// eq(pt, y) for a boolean y given by its bits
f128 eq_binary(const f128* pt, size_t n, uint64_t y) {
  f128 acc = hone();
  for (size_t j = 0; j < n; j++) acc = hmul(acc, (y >> j) & 1 ? pt[j] : fx(hone(), pt[j]));
  return acc;
}
// Lagrange interpolation at z from the 64 values on the Lambda nodes, over
// Lambda alone (interpolate_at_z_on_lambda) and over S u Lambda with zeros on
// S (interpolate_at_z_combined), zerocheck/multilinear.rs:410-535
f128 interp_lambda(const std::vector<f128>& v, f128 z) {
  std::vector<f128> w = hlagrange(z, 64);
  return ip(w.data(), v.data(), 64);
}
f128 interp_combined(const std::vector<f128>& v, f128 z) {
  const f128* P = phi8_table();
  // the denominators prod_{j != i} (s_i + s_j) depend only on the nodes
  static const std::vector<f128> inv_den = [P] {
    std::vector<f128> d(64);
    for (int i = 0; i < 64; i++) {
      f128 den = hone();
      for (int j = 0; j < 128; j++)
        if (j != 64 + i) den = hmul(den, fx(P[64 + i], P[j]));
      d[i] = hinv(den);
    }
    return d;
  }();
  // numerators prod_{j != i} (z + s_j) from prefix and suffix products
  f128 pre[129], suf[129];
  pre[0] = suf[128] = hone();
  for (int j = 0; j < 128; j++) pre[j + 1] = hmul(pre[j], fx(z, P[j]));
  for (int j = 128; j-- > 0;) suf[j] = hmul(suf[j + 1], fx(z, P[j]));
  f128 acc = mk(0, 0);
  for (int i = 0; i < 64; i++) {
    const int node = 64 + i;
    acc = fx(acc, hmul(hmul(hmul(pre[node], suf[node + 1]), inv_den[i]), v[i]));
  }
  return acc;
}
// ----------------------------------------------------- tensor algebra --
// An element of F128 (x) F128 as 128 rows; transpose swaps the two factors
// (bit j of row i <-> bit i of row j), pcs/tensor_algebra.rs.
struct TA {
  f128 e[128];
};
void ta_transpose(TA& t) {
  const std::vector<f128> out = transpose128(std::vector<f128>(t.e, t.e + 128));
  for (int j = 0; j < 128; j++) t.e[j] = out[j];
}
void ta_scale(TA& t, f128 s) {
  for (auto& x : t.e) x = hmul(x, s);
}
f128 ta_fold_vertical(TA t, const std::vector<f128>& c) {
  ta_transpose(t);
  return ip(t.e, c.data(), 128);
}
// eval_rs_eq_prefix: start at 1 (vertical); per coordinate
// t += t * z (vertical) + t * q (horizontal)
TA rs_eq_prefix(const f128* zv, const f128* q, size_t n) {
  TA t;
  for (auto& x : t.e) x = mk(0, 0);
  t.e[0] = hone();
  for (size_t i = 0; i < n; i++) {
    TA v = t, h = t;
    ta_scale(v, zv[i]);
    ta_transpose(h);
    ta_scale(h, q[i]);
    ta_transpose(h);
    for (int k = 0; k < 128; k++) t.e[k] = fx(t.e[k], fx(v.e[k], h.e[k]));
  }
  return t;
}

// ------------------------------------------------------- BLAKE3 Merkle --
H32 cv_bytes(const uint32_t w[8]) {
  H32 h;
  for (int i = 0; i < 8; i++)
    for (int k = 0; k < 4; k++) h[4 * i + k] = (uint8_t)(w[i] >> (8 * k));
  return h;
}
// non-root chaining value of a leaf of at most one chunk (merkle.rs:192-197);
// with SHA-256 Merkle hashing, SHA256(leaf) (merkle.rs:205-214)
H32 leaf_cv(const uint8_t* d, size_t len, int fn = kFnBlake3) {
  if (fn == kFnSha256) {
    H32 h;
    sha256_bytes(d, len, h.data());
    return h;
  }
  uint32_t cv[8], out[16], m[16];
  memcpy(cv, kB3IV, 32);
  const size_t nb = std::max<size_t>(1, (len + 63) / 64);
  for (size_t b = 0; b < nb; b++) {
    uint8_t blk[64] = {0};
    const size_t off = 64 * b, bl = std::min<size_t>(64, len - off);
    memcpy(blk, d + off, bl);
    for (int i = 0; i < 16; i++) m[i] = (uint32_t)blk[4 * i] | (uint32_t)blk[4 * i + 1] << 8 |
                                       (uint32_t)blk[4 * i + 2] << 16 | (uint32_t)blk[4 * i + 3] << 24;
    const uint32_t flags = (b == 0 ? 1u : 0u) | (b + 1 == nb ? 2u : 0u);
    b3_compress(cv, m, 0, (uint32_t)bl, flags, out);
    memcpy(cv, out, 32);
  }
  return cv_bytes(cv);
}
H32 parent_cv(const H32& l, const H32& r, int fn = kFnBlake3) {
  if (fn == kFnSha256) {
    uint8_t b[64];
    memcpy(b, l.data(), 32);
    memcpy(b + 32, r.data(), 32);
    H32 h;
    sha256_bytes(b, 64, h.data());
    return h;
  }
  uint32_t m[16], out[16];
  for (int i = 0; i < 8; i++) {
    m[i] = (uint32_t)l[4 * i] | (uint32_t)l[4 * i + 1] << 8 | (uint32_t)l[4 * i + 2] << 16 | (uint32_t)l[4 * i + 3] << 24;
    m[8 + i] = (uint32_t)r[4 * i] | (uint32_t)r[4 * i + 1] << 8 | (uint32_t)r[4 * i + 2] << 16 |
               (uint32_t)r[4 * i + 3] << 24;
  }
  b3_compress(kB3IV, m, 0, 64, 4 /*PARENT*/, out);
  return cv_bytes(out);
}
// verify_merkle_multi_proof (merkle.rs:1122-1190)
bool merkle_multi_verify(const H32& root, size_t n_leaves, const std::vector<size_t>& pos,
                         const std::vector<H32>& leaves, const std::vector<H32>& proof, int fn) {
  if (n_leaves == 0 || (n_leaves & (n_leaves - 1)) || pos.size() != leaves.size()) return false;
  if (pos.empty()) return proof.empty();
  for (size_t i = 0; i < pos.size(); i++)
    if (pos[i] >= n_leaves || (i && pos[i - 1] >= pos[i])) return false;
  if (n_leaves == 1) return proof.empty() && leaves[0] == root;
  std::vector<std::pair<size_t, H32>> act;
  for (size_t i = 0; i < pos.size(); i++) act.push_back({pos[i], leaves[i]});
  size_t pi = 0;
  for (size_t ll = n_leaves; ll > 1; ll >>= 1) {
    std::vector<std::pair<size_t, H32>> nx;
    for (size_t i = 0; i < act.size();) {
      const size_t p = act[i].first;
      H32 l, r;
      if (i + 1 < act.size() && act[i + 1].first == (p ^ 1)) {
        l = act[i].second;
        r = act[i + 1].second;
        i += 2;
      } else {
        if (pi >= proof.size()) return false;
        const H32& sib = proof[pi++];
        if (p & 1) { l = sib; r = act[i].second; }
        else { l = act[i].second; r = sib; }
        i += 1;
      }
      nx.push_back({p >> 1, parent_cv(l, r, fn)});
    }
    act.swap(nx);
  }
  return pi == proof.size() && act.size() == 1 && act[0].second == root;
}
// verify_level_opens (pcs/ligerito.rs:12441-12468): rows of `lanes` values;
// `cvs`, when given, holds the rows' leaf chaining values already hashed
bool level_opens_ok(const H32& root, size_t block_len, const std::vector<size_t>& q, const Opening& o,
                    size_t lanes, const std::vector<H32>* cvs, int fn) {
  if (q.size() != o.rows.size()) return false;
  std::vector<H32> leaves;
  for (size_t i = 0; i < o.rows.size(); i++) {
    const auto& row = o.rows[i];
    if (row.size() != lanes || lanes * 16 > 1024) return false;
    leaves.push_back(cvs ? (*cvs)[i] : leaf_cv(reinterpret_cast<const uint8_t*>(row.data()), lanes * 16, fn));
  }
  return merkle_multi_verify(root, block_len, q, leaves, o.proof, fn);
}

// The leaf chaining values of every opened row, per opening (initial,
// levels, final), through V.leaf_cvs when it is set and the rows are
// uniform within each opening; empty entries are hashed on the host.
std::vector<std::vector<H32>> opened_leaf_cvs(const Proof& P, const VerifyStatement& V) {
  std::vector<const Opening*> ops{&P.initial};
  for (const Opening& o : P.levels) ops.push_back(&o);
  ops.push_back(&P.final_open);
  std::vector<std::vector<H32>> out(ops.size());
  if (!V.leaf_cvs) return out;
  std::vector<uint8_t> data;
  std::vector<size_t> sizes, counts;
  for (const Opening* o : ops) {
    size_t sz = o->rows.empty() ? 0 : o->rows[0].size() * 16;
    bool ok = sz > 0 && sz <= 1024;
    for (const auto& r : o->rows) ok = ok && r.size() * 16 == sz;
    sizes.push_back(ok ? sz : 0);
    counts.push_back(ok ? o->rows.size() : 0);
    if (!ok) continue;
    for (const auto& r : o->rows) {
      const uint8_t* b = reinterpret_cast<const uint8_t*>(r.data());
      data.insert(data.end(), b, b + sz);
    }
  }
  std::vector<H32> all = V.leaf_cvs(data.data(), sizes, counts, P.merkle_fn);
  size_t at = 0;
  for (size_t k = 0; k < ops.size(); k++) {
    if (!counts[k]) continue;
    if (at + counts[k] > all.size()) return std::vector<std::vector<H32>>(ops.size());
    out[k].assign(all.begin() + (long)at, all.begin() + (long)(at + counts[k]));
    at += counts[k];
  }
  return out;
}

// ---------------------------------------------------- transcript checks --
// FsChallenger::verify_pow (challenger.rs:502-545): the BLAKE3 hash of
// state digest || nonce (LE) || 0^24 has `bits` leading zero bits (bits = 0:
// the nonce is 0); the nonce is observed either way
bool pow_ok(Transcript& tr, uint64_t nonce, uint32_t bits) { return tr.verify_pow(nonce, bits); }

// A Ligerito round's quadratic from its message (u0, u2) and running claim
// (pcs/ligerito.rs:4929-4958)
struct Quad {
  f128 c, b, a;
  static Quad from(std::pair<f128, f128> msg, f128 claim) { return {msg.first, fx(claim, msg.second), msg.second}; }
  f128 eval(f128 r) const { return fx(c, fx(hmul(r, b), hmul(hmul(r, r), a))); }
  static Quad fold(const Quad& p, const Quad& q, f128 al) {
    return {fx(p.c, hmul(al, q.c)), fx(p.b, hmul(al, q.b)), fx(p.a, hmul(al, q.a))};
  }
};

// s_{k+1}(x) = s_k(x)^2 + s_k(v_k) s_k(x); the subspace polynomials at the
// basis points (pcs/ligerito.rs:1186-1210)
f128 next_s(f128 s, f128 root) { return fx(hmul(s, s), hmul(root, s)); }
std::vector<f128> eval_sk_at_vks(int log_n) {
  std::vector<f128> sks((size_t)log_n + 1, mk(0, 0));
  sks[0] = hone();
  if (log_n == 0) return sks;
  std::vector<f128> layer;
  for (int i = 1; i <= log_n; i++) layer.push_back(mk(1ull << i, 0));
  int cur = log_n;
  for (int i = 0; i < log_n; i++) {
    for (int j = 0; j < cur; j++) {
      f128 v = next_s(layer[j], sks[i]);
      if (j == 0) sks[i + 1] = v;
      else layer[j - 1] = v;
    }
    cur--;
  }
  return sks;
}
// induce_sumcheck_enforced_sum (pcs/ligerito.rs:1310-1335)
f128 enforced_sum(const Opening& o, const std::vector<f128>& v, const std::vector<size_t>& q,
                  const std::vector<f128>& alpha) {
  std::vector<f128> eq = heq(v), aw = heq(alpha);
  f128 s = mk(0, 0);
  for (size_t i = 0; i < o.rows.size(); i++) s = fx(s, hmul(aw[i], ip(o.rows[i].data(), eq.data(), eq.size())));
  return s;
}
// induce_sumcheck_evaluate_at_residual (pcs/ligerito.rs:1346-1435)
std::vector<f128> induce_residual(int log_msg_cols, const std::vector<size_t>& q, const std::vector<f128>& alpha,
                                  const f128* ris, int prefix_len, int yr_log_n) {
  // s_k(v_k) and their inverses depend only on the level's size: cached
  static std::mutex mu;
  static std::map<int, std::pair<std::vector<f128>, std::vector<f128>>> cache;
  std::vector<f128> sks, inv;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(log_msg_cols);
    if (it == cache.end()) {
      std::vector<f128> s = eval_sk_at_vks(log_msg_cols), iv(s.size());
      for (size_t i = 0; i < s.size(); i++) iv[i] = (s[i].lo | s[i].hi) ? hinv(s[i]) : mk(0, 0);
      it = cache.emplace(log_msg_cols, std::make_pair(s, iv)).first;
    }
    sks = it->second.first;
    inv = it->second.second;
  }
  std::vector<f128> aw = heq(alpha);
  std::vector<f128> out((size_t)1 << yr_log_n, mk(0, 0));
  for (size_t i = 0; i < q.size(); i++) {
    std::vector<f128> sx((size_t)log_msg_cols);
    if (log_msg_cols > 0) {
      sx[0] = mk((uint64_t)q[i], 0);
      for (int k = 1; k < log_msg_cols; k++) sx[k] = next_s(sx[k - 1], sks[k - 1]);
      for (int k = 0; k < log_msg_cols; k++) sx[k] = hmul(sx[k], inv[k]);
    }
    f128 pre = hone();
    for (int k = 0; k < prefix_len; k++) pre = hmul(pre, fx(hone(), hmul(ris[k], fx(hone(), sx[k]))));
    const f128 w = hmul(aw[i], pre);
    for (size_t y = 0; y < out.size(); y++) {
      f128 suf = hone();
      for (int j = 0; j < yr_log_n; j++)
        if ((y >> j) & 1) suf = hmul(suf, sx[(size_t)prefix_len + j]);
      out[y] = fx(out[y], hmul(w, suf));
    }
  }
  return out;
}

// shift_mle (chain.rs:75-100)
f128 shift_mle(const std::vector<f128>& a, const std::vector<f128>& b) {
  const size_t n = a.size();
  std::vector<f128> pre(n + 1, hone()), suf(n + 1, hone());
  for (size_t j = 0; j < n; j++) pre[j + 1] = hmul(pre[j], hmul(a[j], fx(hone(), b[j])));
  for (size_t j = n; j-- > 0;) suf[j] = hmul(suf[j + 1], fx(hone(), fx(a[j], b[j])));
  f128 acc = mk(0, 0);
  for (size_t j = 0; j < n; j++) acc = fx(acc, hmul(hmul(pre[j], hmul(fx(hone(), a[j]), b[j])), suf[j + 1]));
  return acc;
}
// tau_pos-MLE of a public region over its packed positions (fold_public_phys,
// chain_common.rs:84-118): sum_w eq(tau_pos, w) packed word w
f128 fold_region(const uint64_t words[32], const std::vector<f128>& tau_pos) {
  const std::vector<f128> et = heq(tau_pos);
  f128 acc = mk(0, 0);
  for (size_t w = 0; w < et.size(); w++) acc = fx(acc, hmul(et[w], mk(words[2 * w], words[2 * w + 1])));
  return acc;
}
// a 256-bit public value (8 u32 words) over its two packed positions
f128 fold_cv(const uint32_t cv[8], f128 tp) {
  const f128 p0 = mk((uint64_t)cv[0] | (uint64_t)cv[1] << 32, (uint64_t)cv[2] | (uint64_t)cv[3] << 32);
  const f128 p1 = mk((uint64_t)cv[4] | (uint64_t)cv[5] << 32, (uint64_t)cv[6] | (uint64_t)cv[7] << 32);
  return fx(hmul(fx(hone(), tp), p0), hmul(tp, p1));
}

struct RsClaim {
  f128 z_skip, value;
  std::vector<f128> x;  // x_inner_rest ++ x_outer
};

}  // namespace

// ------------------------------------------------------------- verify --
std::string verify_bundle(const uint8_t* bytes, size_t len, const std::string& domain, const VerifyStatement& V) {
  Proof P;
  std::string why;
  if (!decode(bytes, len, P, why, V.merkle != nullptr)) return "malformed bundle: " + why;
  const int m = V.m, n_log = V.m - V.k_log;
  if (P.m != (uint64_t)m) return "bundle is for another statement size";
  const Ladder* lad = ladder_for(m);
  if (!lad) return "no Ligerito configuration for this size";
  const Ladder& Ld = *lad;
  Transcript tr(domain, V.fs_fn);
  tr.label("flock-r1cs-v0");
  tr.bytes(V.digest.data(), 32);
  tr.bytes(P.root.data(), 32);

  // ---- zerocheck
  const int ks = kKSkip, n_mlv = m - kKSkip;
  if (P.r1_ab.size() != 64 || P.r1_c.size() != 64 || P.zc_rounds.size() != (size_t)n_mlv)
    return "zerocheck: malformed";
  tr.label("flock-zerocheck-v0");
  std::vector<f128> r = tr.sample_vec(ks), r_outer = tr.sample_vec((size_t)(m - ks - 7));
  for (f128 v : small_consts()) r.push_back(v);
  for (f128 v : medium_consts()) r.push_back(v);
  r.insert(r.end(), r_outer.begin(), r_outer.end());
  tr.f128s(P.r1_ab.data(), 64);
  tr.f128s(P.r1_c.data(), 64);
  const f128 zz = tr.sample();
  const f128 pc = interp_lambda(P.r1_c, zz);
  if (!feq(pc, P.fc)) return "zerocheck: c evaluation";
  std::vector<f128> comb_l(64);
  for (int i = 0; i < 64; i++) comb_l[i] = fx(P.r1_ab[i], P.r1_c[i]);
  f128 run = fx(interp_combined(comb_l, zz), pc);
  std::vector<f128> rhos;
  for (int i = 0; i < n_mlv; i++) {
    const f128 req = r[(size_t)(ks + i)], g1 = P.zc_rounds[i].first, gi = P.zc_rounds[i].second;
    const f128 g0 = hmul(fx(run, hmul(req, g1)), hinv(fx(hone(), req)));
    tr.f128v(g1);
    tr.f128v(gi);
    const f128 rho = tr.sample();
    rhos.push_back(rho);
    const f128 opr = fx(hone(), rho);
    run = fx(fx(hmul(g0, opr), hmul(g1, rho)), hmul(gi, hmul(rho, opr)));
  }
  if (!feq(run, hmul(P.fa, P.fb))) return "zerocheck: final product";
  tr.f128v(P.fa);
  tr.f128v(P.fb);

  // ---- lincheck: comb = alpha A^T eq + B^T eq (+ beta at the constant
  // column) over the block's 2^k_log columns, built on the device
  const int ir = V.k_log - kKSkip;
  if (P.lc_rounds.size() != (size_t)ir || P.z_partial.size() != 64) return "lincheck: malformed";
  std::vector<f128> x_inner(rhos.begin(), rhos.begin() + ir), x_outer(rhos.begin() + ir, rhos.end());
  tr.label("flock-lincheck-v0");
  const f128 alpha = tr.sample();
  const f128 beta = tr.sample();
  std::vector<f128> cv = V.comb(zz, x_inner, alpha, beta);
  if (cv.size() != (size_t)1 << V.k_log) return "lincheck: matrix combination";
  run = fx(fx(hmul(alpha, P.fa), P.fb), beta);
  std::vector<f128> rr;
  for (const auto& rd : P.lc_rounds) {
    tr.f128v(rd.first);
    tr.f128v(rd.second);
    const f128 rk = tr.sample();
    const f128 e0 = fx(run, rd.first), c1 = fx(fx(e0, rd.first), rd.second);
    run = fx(fx(hmul(rd.second, hmul(rk, rk)), hmul(c1, rk)), e0);
    const size_t h = cv.size() / 2;
    for (size_t i = 0; i < h; i++) cv[i] = fx(cv[i], hmul(rk, fx(cv[i + h], cv[i])));
    cv.resize(h);
    rr.push_back(rk);
  }
  tr.f128s(P.z_partial.data(), 64);
  if (!feq(run, ip(cv.data(), P.z_partial.data(), 64))) return "lincheck: final sum";
  const f128 r_inner_skip = tr.sample();
  std::vector<f128> lam = hlagrange(r_inner_skip, 0);
  const f128 w = ip(lam.data(), P.z_partial.data(), 64);

  RsClaim cl[2];
  cl[0].z_skip = r_inner_skip;
  cl[0].value = w;
  cl[0].x.assign(rr.rbegin(), rr.rend());
  cl[0].x.insert(cl[0].x.end(), x_outer.begin(), x_outer.end());
  cl[1].z_skip = zz;
  cl[1].value = P.fc;
  cl[1].x.assign(r.begin() + ks, r.end());

  // ---- hash chain: tau_pos, the shift argument from the public endpoints
  std::vector<f128> pd_point;
  if (P.chain) {
    const ChainGeom CG = chain_geom(V.hash);
    if (P.chain_kind != (uint32_t)CG.kind) return "chain: hash kind of another statement";
    if (P.end_bits != CG.region_bits) return "chain: endpoint length";
    const std::vector<f128> tpv = tr.sample_vec((size_t)CG.region_log - 7);
    const size_t n = (size_t)n_log;
    if (P.shift_rounds.size() != n + 1) return "chain: malformed shift proof";
    std::vector<f128> tau = tr.sample_vec(n);
    const f128 al = tr.sample();
    f128 tprod = hone();
    for (f128 t : tau) tprod = hmul(tprod, t);
    f128 claim = fx(hmul(tprod, fold_region(P.end_last, tpv)), hmul(al, fold_region(P.end0, tpv)));
    std::vector<f128> rs;
    for (const auto& rd : P.shift_rounds) {
      tr.f128v(rd.first);
      tr.f128v(rd.second);
      const f128 rk = tr.sample();
      const f128 e0 = fx(claim, rd.first), c1 = fx(fx(e0, rd.first), rd.second);
      claim = fx(fx(hmul(rd.second, hmul(rk, rk)), hmul(c1, rk)), e0);
      rs.push_back(rk);
    }
    std::vector<f128> full(n + 1);
    for (size_t k = 0; k <= n; k++) full[n - k] = rs[k];
    std::vector<f128> taup(full.begin(), full.begin() + n), zero(n, mk(0, 0));
    const f128 s0 = full[n], ops0 = fx(hone(), s0);
    const f128 wf = fx(fx(hmul(shift_mle(tau, taup), ops0), hmul(eq_eval(tau.data(), taup.data(), n), s0)),
                       hmul(hmul(al, eq_eval(taup.data(), zero.data(), n)), ops0));
    if (!feq(claim, hmul(wf, P.g_at_point))) return "chain: shift argument";
    // [tau_pos, s0, 0^(k_log - region_log - 1), instance]
    const size_t off = (size_t)V.k_log - 7, tl = tpv.size();
    pd_point.assign(off + n, mk(0, 0));
    for (size_t j = 0; j < tl; j++) pd_point[j] = tpv[j];
    pd_point[tl] = s0;
    for (size_t i = 0; i < n; i++) pd_point[off + i] = taup[i];
  }

  // ---- Merkle paths: tau_pos, the shift sumcheck from the public leaves
  // and root (merkle_path.rs:469-590, merkle_path_common.rs:459-537)
  if (V.merkle) {
    const MerklePublic& M = *V.merkle;
    const f128 tp = tr.sample_vec(1)[0];
    const size_t n = (size_t)n_log;
    if (M.path_log < 0 || (size_t)M.path_log > n || M.b_bits.size() != ((size_t)1 << n) ||
        M.leaves.size() != ((size_t)1 << M.path_log))
      return "merkle: public inputs do not match the statement size";
    if (P.mp_rounds.size() != n + 2) return "merkle: malformed shift proof";
    const size_t pos_log = n - (size_t)M.path_log;
    const std::vector<f128> tau = tr.sample_vec(n);
    const f128 al = tr.sample();
    const std::vector<f128> tq(tau.begin(), tau.begin() + (long)pos_log), tpp(tau.begin() + (long)pos_log, tau.end());
    f128 ones = hone();
    for (f128 t : tq) ones = hmul(ones, t);
    const std::vector<f128> eqp = heq(tpp);
    f128 leaf = mk(0, 0);
    for (size_t i = 0; i < eqp.size(); i++) leaf = fx(leaf, hmul(eqp[i], fold_cv(M.leaves[i].data(), tp)));
    f128 claim = fx(hmul(ones, fold_cv(M.root.data(), tp)), hmul(al, leaf));
    // Lagrange over {0, 1, w, w + 1}, w = x
    const f128 om = mk(2, 0), om1 = fx(om, hone());
    const f128 d0 = hinv(hmul(om, om1)), d1 = hinv(hmul(om1, om));
    std::vector<f128> rs;
    for (const auto& q : P.mp_rounds) {
      for (const f128& v : q) tr.f128v(v);
      const f128 rk = tr.sample();
      const f128 q0 = fx(claim, q[0]);
      const f128 a = fx(rk, hone()), b = fx(rk, om), c = fx(rk, om1);
      claim = fx(fx(hmul(hmul(hmul(a, b), c), hmul(q0, d0)), hmul(hmul(hmul(rk, b), c), hmul(q[0], d1))),
                 fx(hmul(hmul(hmul(rk, a), c), hmul(q[1], d0)), hmul(hmul(hmul(rk, a), b), hmul(q[2], d1))));
      rs.push_back(rk);
    }
    std::vector<f128> ipt(n);
    for (size_t j = 0; j < n; j++) ipt[j] = rs[n - 1 - j];
    const f128 side = rs[n], sel = rs[n + 1];
    const std::vector<f128> yq(ipt.begin(), ipt.begin() + (long)pos_log), yp(ipt.begin() + (long)pos_log, ipt.end());
    f128 z0 = hone();
    for (f128 t : yq) z0 = hmul(z0, fx(hone(), t));
    const f128 tsa = hmul(eq_eval(tpp.data(), yp.data(), yp.size()), fx(shift_mle(tq, yq), hmul(al, z0)));
    const f128 teq = eq_eval(tau.data(), ipt.data(), n);
    const std::vector<f128> eqi = heq(ipt);
    f128 tb = mk(0, 0);
    const size_t mask = ((size_t)1 << pos_log) - 1;
    for (size_t i = 0; i < M.b_bits.size(); i++)
      if (M.b_bits[i] && (i & mask) != 0) tb = fx(tb, eqi[i]);
    // slot indicator of s = ss | sd << 1: Z = 1, X_L = 2, X_R = 3
    auto ind = [&](int s) {
      return hmul((s & 1) ? sel : fx(hone(), sel), (s >> 1) ? side : fx(hone(), side));
    };
    const f128 wf = fx(hmul(ind(1), teq), fx(hmul(hmul(ind(2), tsa), fx(hone(), tb)), hmul(hmul(ind(3), tsa), tb)));
    if (!feq(claim, hmul(wf, P.g_at_point))) return "merkle: shift sumcheck";
    pd_point.assign(8 + n, mk(0, 0));
    pd_point[0] = tp;
    pd_point[1] = sel;
    pd_point[2] = side;
    for (size_t j = 0; j < n; j++) pd_point[8 + j] = ipt[j];
  }

  // ---- batched open: ring switches, the packed-direct claim, the target
  if (P.s_hat_v.size() != 2) return "open: expected two ring-switched claims";
  tr.label("flock-pcs-open-batch-v0");
  std::vector<f128> eqd[2];
  f128 sc[2];
  for (int k = 0; k < 2; k++) {
    const std::vector<f128>& sv = P.s_hat_v[k];
    if (sv.size() != 128) return "ring switch: malformed";
    tr.label("flock-ring-switch-v0");
    tr.f128s(sv.data(), 128);
    // claim weights: L_i(z_skip) eq(x[0], bit 6) (ring_switch.rs:138-160)
    std::vector<f128> L = hlagrange(cl[k].z_skip, 0);
    f128 chk = mk(0, 0);
    for (int i = 0; i < 128; i++)
      chk = fx(chk, hmul(hmul(L[i & 63], (i >> 6) ? cl[k].x[0] : fx(hone(), cl[k].x[0])), sv[i]));
    if (!feq(chk, cl[k].value)) return "ring switch: claim";
    eqd[k] = heq(tr.sample_vec(7));
    TA u;
    for (int i = 0; i < 128; i++) u.e[i] = sv[i];
    ta_transpose(u);
    sc[k] = ip(u.e, eqd[k].data(), 128);
  }
  const f128 gam[2] = {tr.sample(), tr.sample()};
  f128 target = fx(hmul(gam[0], sc[0]), hmul(gam[1], sc[1]));
  f128 gpd = mk(0, 0);
  if (P.chain || P.merkle) {
    tr.label("flock-pcs-packed-direct-v0");
    tr.f128v(P.g_at_point);
    gpd = tr.sample();
    target = fx(target, hmul(gpd, P.g_at_point));
  }

  // ---- Ligerito (recursive_verifier_with_basis_succinct)
  const int log_n = m - 7, ik = Ld.initial_k, rsteps = (int)Ld.ks.size();
  if (!Ld.ood.empty() && Ld.ood[0] != 0) return "ligerito: config";
  if (P.lig_root != P.root) return "ligerito: initial root";
  tr.label("flock-ligerito-basis-v0");
  tr.f128v(target);
  tr.bytes(P.root.data(), 32);
  size_t tx = 0, fi = 0, oi = 0, ni = 0;
  auto next_msg = [&](std::pair<f128, f128>& msg) {
    if (tx >= P.sc_msgs.size()) return false;
    msg = P.sc_msgs[tx++];
    tr.f128v(msg.first);
    tr.f128v(msg.second);
    return true;
  };
  auto ood_n = [&](int lvl) { return lvl < (int)Ld.ood.size() ? Ld.ood[lvl] : 0; };
  auto fold_bits = [&](int lvl, int j) { return lvl < (int)Ld.fold_grind.size() ? std::max(0, Ld.fold_grind[lvl] - j) : 0; };
  f128 t_r = target;
  std::pair<f128, f128> msg;
  if (!next_msg(msg)) return "ligerito: transcript length";
  Quad quad = Quad::from(msg, t_r);
  struct OodCtx { std::vector<f128> z; size_t ris_start; f128 beta; };
  struct LevelCtx { int log_msg_cols; std::vector<size_t> q; std::vector<f128> alpha; size_t ris_start; f128 beta; };
  std::vector<OodCtx> oods;
  std::vector<LevelCtx> lvls;
  std::vector<f128> ris;
  auto fold_rounds = [&](int lvl, int count, std::vector<f128>& out_rs) {
    for (int j = 0; j < count; j++) {
      const int bits = fold_bits(lvl, j);
      if (bits > 0) {
        if (fi >= P.fold_nonces.size() || !pow_ok(tr, P.fold_nonces[fi++], (uint32_t)bits)) return false;
      }
      const f128 ri = tr.sample();
      ris.push_back(ri);
      out_rs.push_back(ri);
      t_r = quad.eval(ri);
      if (!next_msg(msg)) return false;
      quad = Quad::from(msg, t_r);
    }
    return true;
  };
  auto ood_round = [&](int count, int nvars) {
    for (int s = 0; s < count; s++) {
      std::vector<f128> zp = tr.sample_vec((size_t)nvars);
      if (oi >= P.ood.size()) return false;
      const f128 y = P.ood[oi++];
      tr.f128v(y);
      if (!next_msg(msg)) return false;
      const Quad iq = Quad::from(msg, y);
      const f128 be = tr.sample();
      quad = Quad::fold(quad, iq, be);
      t_r = fx(t_r, hmul(be, y));
      oods.push_back({zp, ris.size(), be});
    }
    return true;
  };
  std::vector<f128> lane_rs;
  if (!fold_rounds(0, ik, lane_rs)) return "ligerito: L0 fold rounds";
  if (P.roots.empty()) return "ligerito: roots";
  tr.bytes(P.roots[0].data(), 32);
  // OOD samples of the folded message (ris holds the initial_k lane folds)
  if (!ood_round(ood_n(1), log_n - ik)) return "ligerito: OOD";
  if (ni >= P.grind_nonces.size() || !pow_ok(tr, P.grind_nonces[ni++], (uint32_t)Ld.grind[0]))
    return "ligerito: L0 proof of work";
  const size_t block0 = (size_t)1 << (log_n - ik + Ld.rate[0]);
  std::vector<size_t> q0 = sample_distinct_queries(tr, block0, (size_t)Ld.queries[0]);
  std::vector<f128> a0 = tr.sample_vec(ceil_log2((size_t)Ld.queries[0]));
  const std::vector<std::vector<H32>> lcv = opened_leaf_cvs(P, V);
  auto cvs_of = [&](size_t k) { return lcv[k].empty() ? nullptr : &lcv[k]; };
  if (!level_opens_ok(P.root, block0, q0, P.initial, (size_t)1 << ik, cvs_of(0), P.merkle_fn)) return "ligerito: L0 openings";
  const int n1 = log_n - ik;
  {
    const f128 es = enforced_sum(P.initial, lane_rs, q0, a0);
    if (!next_msg(msg)) return "ligerito: transcript length";
    const Quad iq = Quad::from(msg, es);
    const f128 be = tr.sample();
    quad = Quad::fold(quad, iq, be);
    t_r = fx(t_r, hmul(be, es));
    lvls.push_back({n1, q0, a0, (size_t)ik, be});
  }
  H32 prev_root = P.roots[0];
  if (rsteps < 1) return "ligerito: config";
  int prev_lni = Ld.ks[0], prev_lmc = n1 - Ld.ks[0], prev_rate = Ld.rate[1];
  size_t next_root = 1, rp = 0;
  int n_cur = n1;
  for (int i = 0; i < rsteps; i++) {
    const int k_i = Ld.ks[i];
    if (n_cur < k_i) return "ligerito: config";
    std::vector<f128> level_rs;
    if (!fold_rounds(i + 1, k_i, level_rs)) return "ligerito: fold rounds";
    n_cur -= k_i;
    if (i == rsteps - 1) {
      if (tx != P.sc_msgs.size() || oi != P.ood.size() || fi != P.fold_nonces.size())
        return "ligerito: transcript length";
      if (P.yr.size() != ((size_t)1 << n_cur)) return "ligerito: final message length";
      for (f128 v : P.yr) tr.f128v(v);
      if (ni >= P.grind_nonces.size() || !pow_ok(tr, P.grind_nonces[ni++], (uint32_t)Ld.grind[i + 1]))
        return "ligerito: final proof of work";
      const size_t pbl = (size_t)1 << (prev_lmc + prev_rate);
      std::vector<size_t> ql = sample_distinct_queries(tr, pbl, (size_t)Ld.queries[i + 1]);
      std::vector<f128> al = tr.sample_vec(ceil_log2((size_t)Ld.queries[i + 1]));
      if (!level_opens_ok(prev_root, pbl, ql, P.final_open, (size_t)1 << prev_lni, cvs_of(lcv.size() - 1),
                          P.merkle_fn))
        return "ligerito: final openings";
      const f128 es = enforced_sum(P.final_open, level_rs, ql, al);
      const f128 be = tr.sample();
      t_r = fx(t_r, hmul(be, es));
      lvls.push_back({n_cur, ql, al, ris.size(), be});
      const int yr_log_n = n_cur;
      const size_t yl = P.yr.size();
      std::vector<f128> comb_y(yl, mk(0, 0));
      for (const LevelCtx& c : lvls) {
        std::vector<f128> res = induce_residual(c.log_msg_cols, c.q, c.alpha, ris.data() + c.ris_start,
                                                c.log_msg_cols - yr_log_n, yr_log_n);
        for (size_t y = 0; y < yl; y++) comb_y[y] = fx(comb_y[y], hmul(c.beta, res[y]));
      }
      for (const OodCtx& c : oods) {
        const size_t folded = c.z.size() - (size_t)yr_log_n;
        if (c.z.size() < (size_t)yr_log_n || c.ris_start + folded > ris.size()) return "ligerito: OOD context";
        f128 sca = c.beta;
        for (size_t b = 0; b < folded; b++) sca = hmul(sca, fx(hone(), fx(c.z[b], ris[c.ris_start + b])));
        std::vector<f128> tail = heq(std::vector<f128>(c.z.begin() + (long)folded, c.z.end()));
        for (size_t y = 0; y < yl; y++) comb_y[y] = fx(comb_y[y], hmul(tail[y], sca));
      }
      // the combined basis b at (ris, y): the ring-switched claims in the
      // tensor algebra, the packed-direct claim as an eq evaluation
      const size_t pl = ris.size();
      if (pl + (size_t)yr_log_n != (size_t)log_n) return "ligerito: residual arity";
      for (int k = 0; k < 2; k++) {
        const TA pre = rs_eq_prefix(cl[k].x.data() + 1, ris.data(), pl);
        const f128* suf = cl[k].x.data() + 1 + pl;
        for (size_t y = 0; y < yl; y++) {
          f128 s = hone();
          for (int j = 0; j < yr_log_n; j++) s = hmul(s, (y >> j) & 1 ? suf[j] : fx(hone(), suf[j]));
          TA t = pre;
          ta_scale(t, s);
          comb_y[y] = fx(comb_y[y], hmul(gam[k], ta_fold_vertical(t, eqd[k])));
        }
      }
      if (P.chain || P.merkle) {
        const f128 pre = eq_eval(pd_point.data(), ris.data(), pl);
        for (size_t y = 0; y < yl; y++)
          comb_y[y] = fx(comb_y[y], hmul(hmul(gpd, pre), eq_binary(pd_point.data() + pl, (size_t)yr_log_n, y)));
      }
      const f128 inner = ip(P.yr.data(), comb_y.data(), yl);
      if (!feq(inner, t_r)) return "ligerito: final inner product";
      return "";
    }
    if (next_root >= P.roots.size()) return "ligerito: roots";
    const H32 root_next = P.roots[next_root++];
    tr.bytes(root_next.data(), 32);
    if (!ood_round(ood_n(i + 2), n_cur)) return "ligerito: OOD";
    if (ni >= P.grind_nonces.size() || !pow_ok(tr, P.grind_nonces[ni++], (uint32_t)Ld.grind[i + 1]))
      return "ligerito: level proof of work";
    const size_t pbl = (size_t)1 << (prev_lmc + prev_rate);
    std::vector<size_t> qi = sample_distinct_queries(tr, pbl, (size_t)Ld.queries[i + 1]);
    std::vector<f128> al = tr.sample_vec(ceil_log2((size_t)Ld.queries[i + 1]));
    if (rp >= P.levels.size()) return "ligerito: level openings missing";
    const Opening& o = P.levels[rp++];
    if (!level_opens_ok(prev_root, pbl, qi, o, (size_t)1 << prev_lni, cvs_of(rp), P.merkle_fn)) return "ligerito: level openings";
    const f128 es = enforced_sum(o, level_rs, qi, al);
    if (!next_msg(msg)) return "ligerito: transcript length";
    const Quad iq = Quad::from(msg, es);
    const f128 be = tr.sample();
    quad = Quad::fold(quad, iq, be);
    t_r = fx(t_r, hmul(be, es));
    lvls.push_back({n_cur, qi, al, ris.size(), be});
    prev_root = root_next;
    if (i + 1 >= rsteps || n_cur < Ld.ks[i + 1]) return "ligerito: config";
    prev_lni = Ld.ks[i + 1];
    prev_lmc = n_cur - Ld.ks[i + 1];
    prev_rate = Ld.rate[(size_t)i + 2];
  }
  return "ligerito: config";
}

// The device half of the verifier: the lincheck's matrix combination over
// this setup's CSC copy of the block matrices, with the prover's kernels.
namespace {
// Device scratch of one verification in flight: eq(x_inner) (256 values), the
// lincheck's eq table and matrix combination (2^14 values each), the opened
// rows (1 MiB) and their leaf chaining values (512 KiB).
struct VerifyBufs {
  f128 *eqx, *eqi, *comb;
  f128* kcw;  // the Keccak walker's W rows (Keccak statements only)
  uint8_t* rows;
  uint32_t* cvs;
  size_t rows_cap, cvs_cap;  // bytes
};
// the device half of the verifier over the CSC copy of the block matrices
// given by at_*, bt_* (the Keccak statement's implicit matrices by its
// walker): the matrix combination and the opened rows' leaves
VerifyStatement device_statement(int m, int hash, const std::array<uint8_t, 32>& digest, const uint32_t* at_ptr,
                                 const uint16_t* at_row, const uint32_t* bt_ptr, const uint16_t* bt_row,
                                 const VerifyBufs& B, cudaStream_t st) {
  VerifyStatement V;
  V.m = m;
  V.k_log = hash_k_log(hash);
  V.hash = hash;
  V.digest = digest;
  const int kk = 1 << V.k_log, pin = statement(hash).z_const;
  V.comb = [=](f128 zskip, const std::vector<f128>& x_inner, f128 alpha, f128 beta) {
    std::vector<f128> L = hlagrange(zskip, 0), cv(kk);
    eq_build(x_inner.data(), (int)x_inner.size(), hone(), B.eqx, st);
    outer64(L.data(), B.eqx, (size_t)1 << x_inner.size(), B.eqi, st);
    if (is_keccak(hash)) {
      int dev = 0;
      CK(cudaGetDevice(&dev));
      keccak_comb(B.eqi, alpha, beta, keccak_masks(dev), B.kcw, B.comb, st, keccak_width(hash));
    } else {
      lc_comb(at_ptr, at_row, bt_ptr, bt_row, B.eqi, alpha, beta, pin, kk, B.comb, st);
    }
    CK(cudaMemcpyAsync(cv.data(), B.comb, kk * sizeof(f128), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return cv;
  };
  // every opened row's leaf chaining value in one upload
  V.leaf_cvs = [=](const uint8_t* data, const std::vector<size_t>& sizes, const std::vector<size_t>& counts,
                   int merkle_fn) {
    size_t bytes = 0, n = 0;
    for (size_t k = 0; k < sizes.size(); k++) bytes += sizes[k] * counts[k], n += counts[k];
    std::vector<H32> cvs(n);
    if (n == 0 || bytes > B.rows_cap || n * 32 > B.cvs_cap) return std::vector<H32>();
    CK(cudaMemcpyAsync(B.rows, data, bytes, cudaMemcpyHostToDevice, st));
    size_t off = 0, at = 0;
    for (size_t k = 0; k < sizes.size(); k++) {
      if (!counts[k]) continue;
      merkle_leaves(B.rows + off, counts[k], sizes[k], B.cvs + 8 * at, merkle_fn, st);
      off += sizes[k] * counts[k];
      at += counts[k];
    }
    CK(cudaMemcpyAsync(cvs.data(), B.cvs, n * 32, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return cvs;
  };
  return V;
}

// One device copy of each hash's block matrices (CSC) per device, shared by
// every Verifier on it (they are the same for every statement size).
struct DevCsc {
  uint32_t *at_ptr = nullptr, *bt_ptr = nullptr;
  uint16_t *at_row = nullptr, *bt_row = nullptr;
};
const DevCsc& shared_csc(int device, int hash) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, DevCsc> m;
  std::lock_guard<std::mutex> lk(mu);
  auto it = m.find({device, hash});
  if (it != m.end()) return it->second;
  const Statement& S = statement(hash);
  DevCsc d;
  auto up = [](auto& dst, const auto& src) {
    CK(cudaMalloc(&dst, src.size() * sizeof(src[0])));
    CK(cudaMemcpy(dst, src.data(), src.size() * sizeof(src[0]), cudaMemcpyHostToDevice));
  };
  up(d.at_ptr, S.at_ptr);
  up(d.bt_ptr, S.bt_ptr);
  up(d.at_row, S.at_row);
  up(d.bt_row, S.bt_row);
  return m[{device, hash}] = d;
}
}  // namespace

// The setup's own buffers and stream (flock_verify: the caller owns the setup).
std::string Setup::verify(const uint8_t* bytes, size_t len, const std::string& domain, const MerklePublic* merkle) {
  VerifyBufs B{zv_pre, eq_inner, comb, kc_w, reinterpret_cast<uint8_t*>(gather), reinterpret_cast<uint32_t*>(idx),
               ((size_t)1 << 16) * sizeof(f128), ((size_t)1 << 16) * sizeof(uint64_t)};
  if (merkle && hash != kHashSha256) return "a Merkle path is a SHA-256 statement";
  VerifyStatement V = device_statement(m, hash, digest, at_ptr, at_row, bt_ptr, bt_row, B, st);
  V.merkle = merkle;
  V.fs_fn = fs_fn;
  return verify_bundle(bytes, len, domain, V);
}

Verifier::Verifier(int device) : device_(device) {
  DeviceScope on(device);
  CK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
  CK(cudaMalloc(&eqx_, ((size_t)1 << (kMaxKLog - kKSkip)) * sizeof(f128)));  // eq(x_inner), 2^(k_log - 6)
  CK(cudaMalloc(&eqi_, ((size_t)1 << kMaxKLog) * sizeof(f128)));  // the largest block of the statements
  CK(cudaMalloc(&comb_, ((size_t)1 << kMaxKLog) * sizeof(f128)));
  CK(cudaMalloc(&kcw_, keccak_comb_scratch(3) * sizeof(f128)));
  CK(cudaMalloc(&rows_, kRowsCap));
  CK(cudaMalloc(&cvs_, kCvsCap));
}

Verifier::~Verifier() {
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device_);
  if (st_) cudaStreamSynchronize(st_);
  for (void* p : {(void*)eqx_, (void*)eqi_, (void*)comb_, (void*)kcw_, (void*)rows_, (void*)cvs_}) cudaFree(p);
  if (st_) cudaStreamDestroy(st_);
  if (prev >= 0) cudaSetDevice(prev);
}

std::string Verifier::verify(const uint8_t* bytes, size_t len, const std::string& domain, int hash,
                             const MerklePublic* merkle, int fs_fn) {
  if (len < 7 + 4 + 32 + 8) return "malformed bundle: truncated";
  if (merkle && hash != kHashSha256) return "a Merkle path is a SHA-256 statement";
  // the statement size is the bundle's m (after the header, the optional
  // hash kind and the root; a Merkle-path proof has neither header nor hash
  // kind); verify_bundle checks everything else
  const size_t at = merkle ? 32 : 7 + (bytes[6] == 3 ? 4 : 0) + 32;
  uint64_t mm = 0;
  for (int k = 0; k < 8; k++) mm |= (uint64_t)bytes[at + k] << (8 * k);
  if (!known_hash(hash)) return "unknown statement hash";
  if (hash == kHashKeccak3 && !merkle && bytes[6] != 2) return "the 3-wide Keccak statement has no chains";
  // BLAKE3: 2^8..2^20 compressions; SHA-256: 2^7..2^19; Keccak: 2^6..2^18
  // blocks of one permutation, 2^5..2^17 of three (the same m range)
  if (mm < 22 || mm > 34) return "bundle is for an unsupported statement size";
  // the stream and buffers belong to device_, whichever device the calling
  // thread has current; the caller's device is restored on return
  DeviceScope on(device_);
  const DevCsc& C = shared_csc(device_, hash);
  const VerifyBufs B{eqx_, eqi_, comb_, kcw_, rows_, cvs_, kRowsCap, kCvsCap};
  VerifyStatement V = device_statement((int)mm, hash, statement_digest(hash, (int)mm), C.at_ptr, C.at_row, C.bt_ptr,
                                       C.bt_row, B, st_);
  V.merkle = merkle;
  V.fs_fn = fs_fn;
  return verify_bundle(bytes, len, domain, V);
}

}  // namespace flock
