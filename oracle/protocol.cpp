// Prover sub-protocols of the oracle (test infrastructure; see flockref.hpp).
// Each function restates the reference's naive / verifier-order semantics:
//  * eq tables: zerocheck/univariate_skip.rs:31-87, lincheck.rs:2080-2125
//  * Lagrange over phi_8 nodes: zerocheck/multilinear.rs:283-400, 470-535
//  * fixed inner eq constants: zerocheck/univariate_skip_optimized.rs:136-233
//  * zerocheck: round1_naive univariate_skip.rs:90-160; transcript order and
//    round semantics zerocheck.rs:1642-1797 (verify) / :539-1640 (prove)
//  * lincheck: lincheck.rs:4653-4665 (quirky eq), :4968-4990 (bind top),
//    :5880-6050 (verify order)
//  * ring switch: pcs/ring_switch.rs:138-160, 1594-1640, 1916-1975, 3653-3725
//  * batched open: pcs.rs:130-290, 1861-1990
//  * Ligerito: pcs/ligerito.rs:1162-1176 (partial_eval_lsb), :1186-1210
//    (eval_sk_at_vks), :1257-1300 (scaled basis), :1310-1336 (enforced
//    sum), :1436-1540 (induce_sumcheck_poly), :4750-4868 (ligero_commit),
//    :4923-5020 (messages), :8894-9100 (SumcheckProver), :9665-9719
//    (queries), :11321-11834 (transcript order, mirrored here), config
//    parse :963-1013 and configs/ligerito/m*_fast.toml (embedded as data).
//  * serialization: crates/flock-prover/src/proof_io.rs:40-215 (bincode 1.3
//    fixint: u64 lengths, enums as u32 variant index, structs in field order)
#include "flockref.hpp"
#include <algorithm>
#include <map>
#include <set>
#include <stdexcept>

namespace flockref {

// --------------------------------------------------------------------------
// Helpers
// --------------------------------------------------------------------------
std::vector<F128> build_eq(const std::vector<F128>& r) {
  std::vector<F128> t((size_t)1 << r.size());
  t[0] = ONE;
  for (size_t i = 0; i < r.size(); i++) {
    size_t len = (size_t)1 << i;
    for (size_t x = 0; x < len; x++) {
      F128 hi = t[x] * r[i];
      t[x + len] = hi;
      t[x] += hi;
    }
  }
  return t;
}

std::vector<F128> lagrange_weights(int k_skip, F128 z, int node_base) {
  int ell = 1 << k_skip;
  std::vector<F128> w(ell);
  for (int i = 0; i < ell; i++) {
    F128 si = phi8((uint8_t)(node_base + i)), num = ONE, den = ONE;
    for (int j = 0; j < ell; j++) {
      if (j == i) continue;
      F128 sj = phi8((uint8_t)(node_base + j));
      num = num * (z + sj);
      den = den * (si + sj);
    }
    w[i] = num * f128_inv(den);
  }
  return w;
}

F128 interpolate_on_lambda(const std::vector<F128>& vals, F128 z) {
  std::vector<F128> w = lagrange_weights(K_SKIP, z, 1 << K_SKIP);
  F128 acc = ZERO;
  for (size_t i = 0; i < vals.size(); i++) acc += w[i] * vals[i];
  return acc;
}

F128 interpolate_combined(const std::vector<F128>& vals, F128 z) {
  int ell = 1 << K_SKIP;
  F128 acc = ZERO;
  for (int i = 0; i < ell; i++) {
    int node = ell + i;
    F128 si = phi8((uint8_t)node), num = ONE, den = ONE;
    for (int j = 0; j < 2 * ell; j++) {
      if (j == node) continue;
      F128 sj = phi8((uint8_t)j);
      num = num * (z + sj);
      den = den * (si + sj);
    }
    acc += num * f128_inv(den) * vals[i];
  }
  return acc;
}

std::array<F128, 3> small_challenges() { return {phi8(0xF7), phi8(0x53), phi8(0xB5)}; }

std::array<F128, 4> medium_challenges() {
  std::array<F128, 4> out;
  const int sh[4] = {1, 2, 4, 8};
  for (int i = 0; i < 4; i++) {
    F128 g(1ull << sh[i], 0);
    out[i] = g * f128_inv(ONE + g);
  }
  return out;
}

static F128 next_s(F128 s, F128 root) { return s * s + root * s; }

std::vector<F128> eval_sk_at_vks(int log_n) {
  std::vector<F128> sks(log_n + 1, ZERO);
  sks[0] = ONE;
  if (log_n == 0) return sks;
  std::vector<F128> layer;
  for (int i = 1; i <= log_n; i++) layer.push_back(F128(1ull << i, 0));
  int cur = log_n;
  for (int i = 0; i < log_n; i++) {
    for (int j = 0; j < cur; j++) {
      F128 v = next_s(layer[j], sks[i]);
      if (j == 0) sks[i + 1] = v;
      else layer[j - 1] = v;
    }
    cur--;
  }
  return sks;
}

static inline bool bit_of(const std::vector<F128>& v, size_t g) {
  const F128& w = v[g >> 7];
  unsigned r = g & 127;
  return ((r < 64 ? w.lo >> r : w.hi >> (r - 64)) & 1) != 0;
}

static size_t ceil_log2(size_t n) {
  if (n <= 1) return 0;
  size_t v = n - 1, l = 0;
  while (v) { l++; v >>= 1; }
  return l;
}

// --------------------------------------------------------------------------
// Zerocheck
// --------------------------------------------------------------------------
struct ZcClaim { F128 z; std::vector<F128> mlv, r_rest; F128 a_eval, b_eval, c_eval; };

// 64 x 64 GF(2^8) low-degree-extension matrix S -> Lambda, as 8 byte tables
// (row r of the unit input e_s extended by inv_NTT_S then fwd_NTT_Lambda).
static std::vector<std::array<uint8_t, 64>> lde_byte_tables() {
  Gf8Ntt ns(K_SKIP, 0), nl(K_SKIP, 64);
  std::array<std::array<uint8_t, 64>, 64> col;  // col[s] = extension of e_s
  for (int s = 0; s < 64; s++) {
    uint8_t v[64] = {0};
    v[s] = 1;
    ns.inverse(v);
    nl.forward(v);
    memcpy(col[s].data(), v, 64);
  }
  std::vector<std::array<uint8_t, 64>> t(8 * 256);
  for (int byte = 0; byte < 8; byte++)
    for (int val = 0; val < 256; val++) {
      std::array<uint8_t, 64> acc{};
      for (int bit = 0; bit < 8; bit++)
        if ((val >> bit) & 1)
          for (int l = 0; l < 64; l++) acc[l] ^= col[8 * byte + bit][l];
      t[byte * 256 + val] = acc;
    }
  return t;
}

static void lde_row(const std::vector<std::array<uint8_t, 64>>& t, uint64_t row, uint8_t out[64]) {
  memset(out, 0, 64);
  for (int byte = 0; byte < 8; byte++) {
    const auto& e = t[byte * 256 + ((row >> (8 * byte)) & 0xFF)];
    for (int l = 0; l < 64; l++) out[l] ^= e[l];
  }
}

static ZerocheckProof zerocheck_prove(const std::vector<F128>& a, const std::vector<F128>& b,
                                      const std::vector<F128>& c, int m, Challenger& ch, ZcClaim& claim) {
  ZerocheckProof pf;
  ch.observe_label("flock-zerocheck-v0");
  std::vector<F128> r_skip = ch.sample_f128_vec(K_SKIP);
  std::vector<F128> r_outer = ch.sample_f128_vec(m - K_SKIP - 7);
  std::vector<F128> r(m);
  for (int i = 0; i < K_SKIP; i++) r[i] = r_skip[i];
  auto sm = small_challenges();
  auto md = medium_challenges();
  for (int i = 0; i < 3; i++) r[K_SKIP + i] = sm[i];
  for (int i = 0; i < 4; i++) r[K_SKIP + 3 + i] = md[i];
  for (int i = 0; i < m - 13; i++) r[13 + i] = r_outer[i];

  std::vector<F128> r_rest(r.begin() + K_SKIP, r.end());
  std::vector<F128> eq = build_eq(r_rest);
  size_t n_rows = (size_t)1 << (m - K_SKIP);
  auto tabs = lde_byte_tables();
  // S[l][k] = sum over rows whose extended GF(2^8) value at lambda_l has bit k.
  std::vector<F128> sab(64 * 8, ZERO), sc(64 * 8, ZERO);
  std::vector<std::vector<F128>> plab(par_threads(), std::vector<F128>(512, ZERO)), plc = plab;
  par_for(n_rows, [&](size_t x0, size_t x1, int ti) {
    std::vector<F128>& lab = plab[ti];
    std::vector<F128>& lc = plc[ti];
    for (size_t x = x0; x < x1; x++) {
      const F128& wa = a[x >> 1];
      const F128& wb = b[x >> 1];
      const F128& wc = c[x >> 1];
      uint64_t ra = (x & 1) ? wa.hi : wa.lo, rb = (x & 1) ? wb.hi : wb.lo, rc = (x & 1) ? wc.hi : wc.lo;
      uint8_t ea[64], eb[64], ec[64];
      lde_row(tabs, ra, ea);
      lde_row(tabs, rb, eb);
      lde_row(tabs, rc, ec);
      F128 e = eq[x];
      for (int l = 0; l < 64; l++) {
        uint8_t vab = gf8_mul(ea[l], eb[l]), vc = ec[l];
        for (int k = 0; k < 8; k++) {
          if ((vab >> k) & 1) lab[l * 8 + k] += e;
          if ((vc >> k) & 1) lc[l * 8 + k] += e;
        }
      }
    }
  });
  for (size_t ti = 0; ti < plab.size(); ti++)
    for (int i = 0; i < 512; i++) { sab[i] += plab[ti][i]; sc[i] += plc[ti][i]; }
  pf.round1_ab.assign(64, ZERO);
  pf.round1_c.assign(64, ZERO);
  for (int l = 0; l < 64; l++)
    for (int k = 0; k < 8; k++) {
      pf.round1_ab[l] += phi8((uint8_t)(1 << k)) * sab[l * 8 + k];
      pf.round1_c[l] += phi8((uint8_t)(1 << k)) * sc[l * 8 + k];
    }
  ch.observe_f128_slice(pf.round1_ab);
  ch.observe_f128_slice(pf.round1_c);
  F128 z = ch.sample_f128();

  // fold a, b at z over the skip variables: hat(x) = sum_s L_s(z) bit(s, x)
  std::vector<F128> L = lagrange_weights(K_SKIP, z, 0);
  std::vector<F128> fa(n_rows), fb(n_rows);
  par_for(n_rows, [&](size_t x0, size_t x1, int) {
    for (size_t x = x0; x < x1; x++) {
      const F128& wa = a[x >> 1];
      const F128& wb = b[x >> 1];
      uint64_t ra = (x & 1) ? wa.hi : wa.lo, rb = (x & 1) ? wb.hi : wb.lo;
      F128 sa = ZERO, sb = ZERO;
      for (int s = 0; s < 64; s++) {
        if ((ra >> s) & 1) sa += L[s];
        if ((rb >> s) & 1) sb += L[s];
      }
      fa[x] = sa;
      fb[x] = sb;
    }
  });
  F128 c_eval = interpolate_on_lambda(pf.round1_c, z);

  int n_mlv = m - K_SKIP;
  std::vector<F128> rhos;
  for (int i = 0; i < n_mlv; i++) {
    std::vector<F128> rem(r.begin() + K_SKIP + i + 1, r.end());
    std::vector<F128> e = build_eq(rem);
    size_t half = fa.size() / 2;
    F128 g1 = ZERO, ginf = ZERO;
    std::vector<F128> p1(par_threads(), ZERO), pinf(par_threads(), ZERO);
    par_for(half, [&](size_t j0, size_t j1, int ti) {
      F128 l1 = ZERO, linf = ZERO;
      for (size_t j = j0; j < j1; j++) {
        F128 a0 = fa[2 * j], a1 = fa[2 * j + 1], b0 = fb[2 * j], b1 = fb[2 * j + 1];
        l1 += e[j] * (a1 * b1);
        linf += e[j] * ((a0 + a1) * (b0 + b1));
      }
      p1[ti] = l1;
      pinf[ti] = linf;
    });
    for (size_t ti = 0; ti < p1.size(); ti++) { g1 += p1[ti]; ginf += pinf[ti]; }
    pf.rounds.push_back({g1, ginf});
    ch.observe_f128(g1);
    ch.observe_f128(ginf);
    F128 rho = ch.sample_f128();
    rhos.push_back(rho);
    std::vector<F128> na(half), nb(half);
    par_for(half, [&](size_t j0, size_t j1, int) {
      for (size_t j = j0; j < j1; j++) {
        na[j] = fa[2 * j] + rho * (fa[2 * j] + fa[2 * j + 1]);
        nb[j] = fb[2 * j] + rho * (fb[2 * j] + fb[2 * j + 1]);
      }
    });
    fa.swap(na);
    fb.swap(nb);
  }
  pf.final_a = fa[0];
  pf.final_b = fb[0];
  pf.final_c = c_eval;
  ch.observe_f128(pf.final_a);
  ch.observe_f128(pf.final_b);
  claim.z = z;
  claim.mlv = rhos;
  claim.r_rest = r_rest;
  claim.a_eval = pf.final_a;
  claim.b_eval = pf.final_b;
  claim.c_eval = c_eval;
  return pf;
}

// --------------------------------------------------------------------------
// Lincheck
// --------------------------------------------------------------------------
struct LcClaim { F128 r_inner_skip; std::vector<F128> r_inner_rest; F128 w; };

static LincheckProof lincheck_prove(const std::vector<F128>& zp, int m, const R1cs& rc, F128 z_skip,
                                    const std::vector<F128>& x_inner_rest, const std::vector<F128>& x_outer,
                                    Challenger& ch, LcClaim& claim) {
  LincheckProof pf;
  ch.observe_label("flock-lincheck-v0");
  F128 alpha = ch.sample_f128();
  std::vector<F128> lam = lagrange_weights(K_SKIP, z_skip, 0);
  std::vector<F128> eqr = build_eq(x_inner_rest);
  const int K = 1 << rc.k_log;
  std::vector<F128> eq_inner(K);
  for (int ir = 0; ir < (int)eqr.size(); ir++)
    for (int is = 0; is < 64; is++) eq_inner[is + 64 * ir] = lam[is] * eqr[ir];
  std::vector<F128> comb(K, ZERO);
  if (rc.walker) {
    comb = keccak::lincheck_comb(*rc.keccak, alpha, eq_inner);
  } else {
    for (int row = 0; row < K; row++) {
      F128 ea = alpha * eq_inner[row], e = eq_inner[row];
      for (uint32_t j = rc.a0.ptr[row]; j < rc.a0.ptr[row + 1]; j++) comb[rc.a0.col[j]] += ea;
      for (uint32_t j = rc.b0.ptr[row]; j < rc.b0.ptr[row + 1]; j++) comb[rc.b0.col[j]] += e;
    }
  }
  F128 beta = ch.sample_f128();
  comb[rc.z_const] += beta;

  // z_vec[c] = sum_o eq(x_outer, o) z[c + 2^k_log o]
  std::vector<F128> eqo = build_eq(x_outer);
  std::vector<F128> zv(K, ZERO);
  size_t n_outer = eqo.size();
  par_for(K, [&](size_t c0, size_t c1, int) {
    for (size_t cidx = c0; cidx < c1; cidx++) {
      F128 acc = ZERO;
      for (size_t o = 0; o < n_outer; o++)
        if (bit_of(zp, cidx + (o << rc.k_log))) acc += eqo[o];
      zv[cidx] = acc;
    }
  });
  std::vector<F128> rr;
  for (int round = 0; round < rc.k_log - K_SKIP; round++) {
    size_t half = comb.size() / 2;
    F128 q1 = ZERO, qinf = ZERO;
    for (size_t i = 0; i < half; i++) {
      q1 += comb[i + half] * zv[i + half];
      qinf += (comb[i + half] + comb[i]) * (zv[i + half] + zv[i]);
    }
    pf.rounds.push_back({q1, qinf});
    ch.observe_f128(q1);
    ch.observe_f128(qinf);
    F128 r = ch.sample_f128();
    rr.push_back(r);
    for (size_t i = 0; i < half; i++) {
      comb[i] = comb[i] + r * (comb[i + half] + comb[i]);
      zv[i] = zv[i] + r * (zv[i + half] + zv[i]);
    }
    comb.resize(half);
    zv.resize(half);
  }
  pf.z_partial = zv;
  ch.observe_f128_slice(pf.z_partial);
  F128 ris = ch.sample_f128();
  std::vector<F128> l2 = lagrange_weights(K_SKIP, ris, 0);
  F128 w = ZERO;
  for (int i = 0; i < 64; i++) w += l2[i] * zv[i];
  claim.r_inner_skip = ris;
  claim.r_inner_rest.assign(rr.rbegin(), rr.rend());
  claim.w = w;
  return pf;
}

// --------------------------------------------------------------------------
// Ligerito
// --------------------------------------------------------------------------
static void round_msg(const std::vector<F128>& f, const std::vector<F128>& b, SumcheckMsg& msg) {
  size_t half = f.size() / 2;
  F128 u0 = ZERO, u2 = ZERO;
  std::vector<F128> p0(par_threads(), ZERO), p2(par_threads(), ZERO);
  par_for(half, [&](size_t j0, size_t j1, int ti) {
    F128 l0 = ZERO, l2 = ZERO;
    for (size_t j = j0; j < j1; j++) {
      F128 f0 = f[2 * j], f1 = f[2 * j + 1], b0 = b[2 * j], b1 = b[2 * j + 1];
      l0 += f0 * b0;
      l2 += (f0 + f1) * (b0 + b1);
    }
    p0[ti] = l0;
    p2[ti] = l2;
  });
  for (size_t ti = 0; ti < p0.size(); ti++) { u0 += p0[ti]; u2 += p2[ti]; }
  msg.u0 = u0;
  msg.u2 = u2;
}

static void fold_lsb(std::vector<F128>& v, F128 r) {
  size_t half = v.size() / 2;
  std::vector<F128> n(half);
  par_for(half, [&](size_t j0, size_t j1, int) {
    for (size_t j = j0; j < j1; j++) n[j] = v[2 * j] + r * (v[2 * j] + v[2 * j + 1]);
  });
  v.swap(n);
}

struct LigeroLevel {
  std::vector<F128> cw;
  std::vector<Hash> tree;
  size_t block_len = 0, lanes = 0;
};

HashKinds& hash_kinds() {
  static thread_local HashKinds k;
  return k;
}

static LigeroLevel ligero_commit(const std::vector<F128>& poly, int log_lanes, int log_inv_rate) {
  LigeroLevel lv;
  lv.lanes = (size_t)1 << log_lanes;
  rs_encode(poly, lv.lanes, log_inv_rate, lv.cw);
  lv.block_len = lv.cw.size() / lv.lanes;
  lv.tree = merkle_tree((const uint8_t*)lv.cw.data(), lv.block_len, lv.lanes * 16, hash_kinds().merkle);
  return lv;
}

static std::vector<size_t> sample_queries(Challenger& ch, size_t block_len, size_t count) {
  std::vector<size_t> out;
  std::set<size_t> seen;
  while (out.size() < count) {
    F128 v = ch.sample_f128();
    size_t q = (size_t)(v.lo % block_len);
    if (seen.insert(q).second) out.push_back(q);
  }
  std::sort(out.begin(), out.end());
  return out;
}

// Induced basis over the folded message domain (n = log_msg_cols vars):
// b[j] = sum_i eq(alpha)[i] * prod_{k in bits(j)} S_k(q_i)/S_k(v_k).
static void induce(int log_msg_cols, const std::vector<std::vector<F128>>& rows, const std::vector<F128>& vch,
                   const std::vector<size_t>& queries, const std::vector<F128>& alpha,
                   std::vector<F128>& basis, F128& enforced) {
  size_t n = (size_t)1 << log_msg_cols;
  std::vector<F128> eq = build_eq(vch);
  std::vector<F128> ap = build_eq(alpha);
  std::vector<F128> sks = eval_sk_at_vks(log_msg_cols);
  std::vector<F128> inv(sks.size());
  for (size_t i = 0; i < sks.size(); i++) inv[i] = sks[i].is_zero() ? ZERO : f128_inv(sks[i]);
  basis.assign(n, ZERO);
  enforced = ZERO;
  std::vector<F128> local(n), sx(std::max(log_msg_cols, 1));
  for (size_t i = 0; i < queries.size(); i++) {
    F128 dot = ZERO;
    for (size_t l = 0; l < rows[i].size(); l++) dot += rows[i][l] * eq[l];
    enforced += dot * ap[i];
    F128 x((uint64_t)queries[i], 0);
    if (log_msg_cols > 0) {
      sx[0] = x;
      for (int k = 1; k < log_msg_cols; k++) sx[k] = next_s(sx[k - 1], sks[k - 1]);
      for (int k = 0; k < log_msg_cols; k++) sx[k] = sx[k] * inv[k];
    }
    local[0] = ap[i];
    for (int k = 0; k < log_msg_cols; k++) {
      size_t cur = (size_t)1 << k;
      for (size_t t = 0; t < cur; t++) local[t + cur] = sx[k] * local[t];
    }
    for (size_t j = 0; j < n; j++) basis[j] += local[j];
  }
}

static void open_rows(const LigeroLevel& lv, const std::vector<size_t>& q, RecursiveProof& rp) {
  rp.opened_rows.clear();
  for (size_t p : q)
    rp.opened_rows.emplace_back(lv.cw.begin() + p * lv.lanes, lv.cw.begin() + (p + 1) * lv.lanes);
  rp.merkle_proof = merkle_multi_proof(lv.tree, lv.block_len, q);
}

static LigeritoProof ligerito_prove(const LigeritoConfig& cfg, std::vector<F128> f, std::vector<F128> b,
                                    F128 target, const LigeroLevel& l0, Challenger& ch) {
  LigeritoProof pf;
  pf.initial_root = l0.tree.back();
  ch.observe_label("flock-ligerito-basis-v0");
  ch.observe_f128(target);
  ch.observe_bytes(pf.initial_root.data(), 32);
  auto push_msg = [&](const SumcheckMsg& m) {
    pf.sumcheck_transcript.push_back(m);
    ch.observe_f128(m.u0);
    ch.observe_f128(m.u2);
  };
  SumcheckMsg msg;
  round_msg(f, b, msg);
  push_msg(msg);
  auto fold_round = [&](int bits) -> F128 {
    if (bits > 0) pf.fold_grinding_nonces.push_back(ch.grind_pow((uint32_t)bits));
    F128 r = ch.sample_f128();
    fold_lsb(f, r);
    fold_lsb(b, r);
    SumcheckMsg m;
    round_msg(f, b, m);
    push_msg(m);
    return r;
  };
  auto introduce = [&](const std::vector<F128>& bnew) {
    SumcheckMsg m;
    round_msg(f, bnew, m);
    push_msg(m);
    F128 beta = ch.sample_f128();
    for (size_t j = 0; j < b.size(); j++) b[j] += beta * bnew[j];
  };
  auto do_ood = [&](int count) {
    for (int s = 0; s < count; s++) {
      int n = 0;
      while (((size_t)1 << n) < f.size()) n++;
      std::vector<F128> zpt = ch.sample_f128_vec(n);
      std::vector<F128> e = build_eq(zpt);
      F128 y = ZERO;
      for (size_t j = 0; j < f.size(); j++) y += f[j] * e[j];
      pf.ood_values.push_back(y);
      ch.observe_f128(y);
      introduce(e);
    }
  };
  int r_steps = (int)cfg.recursive_ks.size();
  std::vector<F128> lane_rs;
  for (int j = 0; j < cfg.initial_k; j++) lane_rs.push_back(fold_round(std::max(0, cfg.fold_grinding_bits[0] - j)));

  int n_cur = 0;
  while (((size_t)1 << n_cur) < f.size()) n_cur++;
  LigeroLevel prev = ligero_commit(f, cfg.recursive_ks[0], cfg.log_inv_rates[1]);
  pf.recursive_roots.push_back(prev.tree.back());
  ch.observe_bytes(prev.tree.back().data(), 32);
  do_ood(cfg.ood_samples.size() > 1 ? cfg.ood_samples[1] : 0);
  pf.grinding_nonces.push_back(ch.grind_pow((uint32_t)cfg.grinding_bits[0]));
  std::vector<size_t> q0 = sample_queries(ch, l0.block_len, (size_t)cfg.queries[0]);
  std::vector<F128> alpha0 = ch.sample_f128_vec(ceil_log2((size_t)cfg.queries[0]));
  open_rows(l0, q0, pf.initial_proof);
  {
    std::vector<F128> basis;
    F128 enf;
    induce(n_cur, pf.initial_proof.opened_rows, lane_rs, q0, alpha0, basis, enf);
    introduce(basis);
  }
  for (int i = 0; i < r_steps; i++) {
    int k_i = cfg.recursive_ks[i];
    std::vector<F128> level_rs;
    for (int j = 0; j < k_i; j++) {
      int fb = (i + 1) < (int)cfg.fold_grinding_bits.size() ? cfg.fold_grinding_bits[i + 1] : 0;
      level_rs.push_back(fold_round(std::max(0, fb - j)));
    }
    n_cur -= k_i;
    if (i == r_steps - 1) {
      pf.final_proof.yr = f;
      for (const F128& v : f) ch.observe_f128(v);
      pf.grinding_nonces.push_back(ch.grind_pow((uint32_t)cfg.grinding_bits[i + 1]));
      std::vector<size_t> ql = sample_queries(ch, prev.block_len, (size_t)cfg.queries[i + 1]);
      ch.sample_f128_vec(ceil_log2((size_t)cfg.queries[i + 1]));
      RecursiveProof rp;
      open_rows(prev, ql, rp);
      pf.final_proof.opened_rows = rp.opened_rows;
      pf.final_proof.merkle_proof = rp.merkle_proof;
      ch.sample_f128();  // beta_last (verifier-side; keeps the transcripts in lockstep)
      return pf;
    }
    LigeroLevel next = ligero_commit(f, cfg.recursive_ks[i + 1], cfg.log_inv_rates[i + 2]);
    pf.recursive_roots.push_back(next.tree.back());
    ch.observe_bytes(next.tree.back().data(), 32);
    do_ood((i + 2) < (int)cfg.ood_samples.size() ? cfg.ood_samples[i + 2] : 0);
    pf.grinding_nonces.push_back(ch.grind_pow((uint32_t)cfg.grinding_bits[i + 1]));
    std::vector<size_t> qi = sample_queries(ch, prev.block_len, (size_t)cfg.queries[i + 1]);
    std::vector<F128> alphai = ch.sample_f128_vec(ceil_log2((size_t)cfg.queries[i + 1]));
    RecursiveProof rp;
    open_rows(prev, qi, rp);
    std::vector<F128> basis;
    F128 enf;
    induce(n_cur, rp.opened_rows, level_rs, qi, alphai, basis, enf);
    pf.recursive_proofs.push_back(rp);
    introduce(basis);
    prev = std::move(next);
  }
  throw std::runtime_error("unreachable");
}

// --------------------------------------------------------------------------
// Ring switch + batched open
// --------------------------------------------------------------------------
static void ring_switch(const std::vector<F128>& zp, const std::vector<F128>& x_full, Challenger& ch,
                        std::vector<F128>& s_hat_v, F128& claim, std::vector<F128>& rs_eq_ind) {
  ch.observe_label("flock-ring-switch-v0");
  std::vector<F128> suffix(x_full.begin() + 1, x_full.end());
  std::vector<F128> eqs = build_eq(suffix);
  s_hat_v.assign(128, ZERO);
  std::vector<std::vector<F128>> ploc(par_threads(), std::vector<F128>(128, ZERO));
  par_for(zp.size(), [&](size_t i0, size_t i1, int ti) {
    std::vector<F128>& loc = ploc[ti];
    for (size_t i = i0; i < i1; i++) {
      for (int r = 0; r < 64; r++) {
        if ((zp[i].lo >> r) & 1) loc[r] += eqs[i];
        if ((zp[i].hi >> r) & 1) loc[64 + r] += eqs[i];
      }
    }
  });
  for (auto& loc : ploc)
    for (int r = 0; r < 128; r++) s_hat_v[r] += loc[r];
  ch.observe_f128_slice(s_hat_v);
  std::vector<F128> rdp = ch.sample_f128_vec(7);
  std::vector<F128> eqd = build_eq(rdp);
  // s_hat_u[b] has bit i = bit b of s_hat_v[i]
  std::vector<F128> u(128, ZERO);
  for (int i = 0; i < 128; i++)
    for (int bb = 0; bb < 128; bb++) {
      uint64_t bit = bb < 64 ? (s_hat_v[i].lo >> bb) & 1 : (s_hat_v[i].hi >> (bb - 64)) & 1;
      if (bit) {
        if (i < 64) u[bb].lo |= 1ull << i;
        else u[bb].hi |= 1ull << (i - 64);
      }
    }
  claim = ZERO;
  for (int bb = 0; bb < 128; bb++) claim += u[bb] * eqd[bb];
  rs_eq_ind.assign(eqs.size(), ZERO);
  par_for(eqs.size(), [&](size_t i0, size_t i1, int) {
    for (size_t i = i0; i < i1; i++) {
      F128 acc = ZERO;
      for (int bb = 0; bb < 64; bb++) {
        if ((eqs[i].lo >> bb) & 1) acc += eqd[bb];
        if ((eqs[i].hi >> bb) & 1) acc += eqd[64 + bb];
      }
      rs_eq_ind[i] = acc;
    }
  });
}

// --------------------------------------------------------------------------
// Ligerito configs (configs/ligerito/m{22..34}_fast.toml, carried as data):
// per level {log_inv_rate, k_recursive, queries, grinding_bits,
// fold_grinding_bits, ood_samples}; level 0 has k = initial_k = 6.
// --------------------------------------------------------------------------
struct LevelRow { int rate, k, queries, grind, fold_grind, ood; };
static const std::map<int, std::pair<std::vector<LevelRow>, int>>& config_table() {
  static const std::map<int, std::pair<std::vector<LevelRow>, int>> t = {
#include "ligerito_fast_configs.inc"
  };
  return t;
}

const LigeritoConfig& ligerito_config(int m) {
  static std::map<int, LigeritoConfig> cache;
  auto it = cache.find(m);
  if (it != cache.end()) return it->second;
  auto row = config_table().find(m);
  if (row == config_table().end()) throw std::runtime_error("no Ligerito config for m");
  LigeritoConfig c;
  const auto& lv = row->second.first;
  c.initial_k = lv[0].k;
  for (size_t i = 0; i < lv.size(); i++) {
    c.log_inv_rates.push_back(lv[i].rate);
    if (i > 0) c.recursive_ks.push_back(lv[i].k);
    c.queries.push_back(lv[i].queries);
    c.grinding_bits.push_back(lv[i].grind);
    c.fold_grinding_bits.push_back(lv[i].fold_grind);
    c.ood_samples.push_back(lv[i].ood);
  }
  c.yr_log_n = row->second.second;
  return cache[m] = c;
}

// --------------------------------------------------------------------------
// Serialization (bincode 1.3, fixint, little endian)
// --------------------------------------------------------------------------
namespace {
struct W {
  std::vector<uint8_t> out;
  void u8(uint8_t v) { out.push_back(v); }
  void u32(uint32_t v) { for (int i = 0; i < 4; i++) out.push_back((uint8_t)(v >> (8 * i))); }
  void u64(uint64_t v) { for (int i = 0; i < 8; i++) out.push_back((uint8_t)(v >> (8 * i))); }
  void f(const F128& v) { u64(v.lo); u64(v.hi); }
  void h(const Hash& v) { out.insert(out.end(), v.begin(), v.end()); }
  void fv(const std::vector<F128>& v) { u64(v.size()); for (auto& x : v) f(x); }
  void hv(const std::vector<Hash>& v) { u64(v.size()); for (auto& x : v) h(x); }
  void rows(const std::vector<std::vector<F128>>& r) { u64(r.size()); for (auto& x : r) fv(x); }
  void pairs(const std::vector<std::pair<F128, F128>>& p) { u64(p.size()); for (auto& x : p) { f(x.first); f(x.second); } }
  void u64v(const std::vector<uint64_t>& v) { u64(v.size()); for (auto x : v) u64(x); }
};
}  // namespace

static void put_header(W& w, uint8_t flavor) {
  const char* magic = "FLOCK";
  for (int i = 0; i < 5; i++) w.u8((uint8_t)magic[i]);
  w.u8(4);  // VERSION
  w.u8(flavor);
}

// Commitment, ZerocheckProof, LincheckProof (the fields a compression bundle
// and a chain bundle share, in this order)
static void put_core(W& w, const Bundle& bd) {
  // Commitment { root, params { m, log_inv_rate, log_batch_size, profile, merkle_hash } }
  w.h(bd.root);
  w.u64(bd.m);
  w.u64(bd.log_inv_rate);
  w.u64(bd.log_batch_size);
  w.u32(bd.profile);
  w.u32(bd.merkle_hash);
  // ZerocheckProof
  w.fv(bd.zc.round1_ab);
  w.fv(bd.zc.round1_c);
  w.pairs(bd.zc.rounds);
  w.f(bd.zc.final_a);
  w.f(bd.zc.final_b);
  w.f(bd.zc.final_c);
  // LincheckProof
  w.pairs(bd.lc.rounds);
  w.fv(bd.lc.z_partial);
}

// BatchOpeningProofLigerito { ring_switches: Vec<{s_hat_v}>, ligerito }
static void put_open(W& w, const Bundle& bd) {
  w.u64(bd.s_hat_v.size());
  for (auto& s : bd.s_hat_v) w.fv(s);
  const LigeritoProof& L = bd.lig;
  w.h(L.initial_root);
  w.rows(L.initial_proof.opened_rows);
  w.hv(L.initial_proof.merkle_proof);
  w.hv(L.recursive_roots);
  w.u64(L.recursive_proofs.size());
  for (auto& rp : L.recursive_proofs) { w.rows(rp.opened_rows); w.hv(rp.merkle_proof); }
  w.fv(L.final_proof.yr);
  w.rows(L.final_proof.opened_rows);
  w.hv(L.final_proof.merkle_proof);
  w.u64(L.sumcheck_transcript.size());
  for (auto& m : L.sumcheck_transcript) { w.f(m.u0); w.f(m.u2); }
  w.u64v(L.grinding_nonces);
  w.fv(L.ood_values);
  w.u64v(L.fold_grinding_nonces);
}

std::vector<uint8_t> serialize(const Bundle& bd) {
  W w;
  put_header(w, 2);  // flavor: R1CS Ligerito
  put_core(w, bd);
  put_open(w, bd);
  return w.out;
}

std::vector<uint8_t> serialize_merkle(const MerkleBundle& mb) {
  W w;
  put_core(w, mb.core);
  w.u64(mb.shift.rounds.size());
  for (const auto& r : mb.shift.rounds)
    for (const F128& v : r) w.f(v);
  w.f(mb.shift.g_at_point);
  put_open(w, mb.core);
  return w.out;
}

// ChainProofBundleLigerito { hash_kind, commitment, proof { zerocheck,
// lincheck, shift { rounds, g_at_point }, pcs_open }, cv_0_phys, cv_last_phys }
// (proof_io.rs:144-157, 943-950; chain_common.rs:247-253; chain.rs:103-112);
// Vec<bool> is a u64 length and one byte per bool.
std::vector<uint8_t> serialize_chain(const ChainBundle& cb) {
  W w;
  put_header(w, 3);  // flavor: chain Ligerito
  w.u32(cb.kind);    // HashKind: Blake3 = 0, Sha2 = 1
  put_core(w, cb.core);
  w.pairs(cb.shift.rounds);
  w.f(cb.shift.g_at_point);
  put_open(w, cb.core);
  for (const std::vector<uint8_t>* bits : {&cb.phys0, &cb.phys_last}) {
    w.u64(bits->size());
    for (uint8_t b : *bits) w.u8(b);
  }
  return w.out;
}

// --------------------------------------------------------------------------
// Full prove (prover.rs:373-473).  `after_core` (may be empty) runs between
// the lincheck and the batched open, on the same transcript, and returns the
// packed-direct claims the open batches with the two ring-switched ones
// (pcs.rs:130-290; claim combine pcs.rs:844-872, 1236-1248): each claim's
// value is observed under its label, one gamma is sampled per claim after
// the ring-switch gammas, the target gains gamma * value and b_combined
// gains gamma * eq(point), scattered over the point's nonzero coordinates
// (ring_switch.rs:2600-2617 build_eq_sparse, :2565-2571 scatter_idx).
// --------------------------------------------------------------------------
Bundle prove_with(const std::vector<Compression>& blocks, int n_log, const std::string& domain,
                  const CoreHook& after_core) {
  std::vector<F128> z, a, b;
  generate_witness(blocks, n_log, z, a, b);
  return prove_core(blake3_r1cs(n_log), std::move(z), a, b, domain, after_core);
}

Bundle prove_core(const R1cs& rc, std::vector<F128> z, const std::vector<F128>& a, const std::vector<F128>& b,
                  const std::string& domain, const CoreHook& after_core) {
  int m = rc.m;
  const LigeritoConfig& cfg = ligerito_config(m);

  // commit: RS-encode 64 interleaved lanes at rate 1/2, Merkle over positions
  LigeroLevel l0 = ligero_commit(z, 6, 1);
  Bundle bd;
  bd.root = l0.tree.back();
  bd.m = (uint64_t)m;
  bd.merkle_hash = (uint32_t)hash_kinds().merkle;

  Challenger ch(domain, hash_kinds().transcript);
  ch.observe_label("flock-r1cs-v0");
  ch.observe_bytes(rc.digest.data(), 32);
  ch.observe_bytes(bd.root.data(), 32);

  ZcClaim zc;
  bd.zc = zerocheck_prove(a, b, z, m, ch, zc);
  int ir = rc.k_log - K_SKIP;
  std::vector<F128> x_inner(zc.mlv.begin(), zc.mlv.begin() + ir);
  std::vector<F128> x_outer(zc.mlv.begin() + ir, zc.mlv.end());
  LcClaim lc;
  bd.lc = lincheck_prove(z, m, rc, zc.z, x_inner, x_outer, ch, lc);

  std::vector<DirectClaim> direct;
  if (after_core) direct = after_core(ch, z);

  // claims: ab at (r_inner_skip, r_inner_rest ++ x_outer); c at (z, r_rest)
  std::vector<F128> xab = lc.r_inner_rest;
  xab.insert(xab.end(), x_outer.begin(), x_outer.end());
  std::vector<F128> xc = zc.r_rest;

  ch.observe_label("flock-pcs-open-batch-v0");
  std::vector<F128> s0, s1, rs0, rs1;
  F128 c0, c1;
  ring_switch(z, xab, ch, s0, c0, rs0);
  ring_switch(z, xc, ch, s1, c1, rs1);
  bd.s_hat_v = {s0, s1};
  F128 g0 = ch.sample_f128(), g1 = ch.sample_f128();
  F128 target = g0 * c0 + g1 * c1;
  std::vector<F128> bc(rs0.size());
  par_for(bc.size(), [&](size_t i0, size_t i1, int) {
    for (size_t i = i0; i < i1; i++) bc[i] = g0 * rs0[i] + g1 * rs1[i];
  });
  for (const DirectClaim& d : direct) {
    ch.observe_label("flock-pcs-packed-direct-v0");
    ch.observe_f128(d.value);
  }
  std::vector<F128> gd;
  for (size_t k = 0; k < direct.size(); k++) gd.push_back(ch.sample_f128());
  for (size_t k = 0; k < direct.size(); k++) {
    const DirectClaim& d = direct[k];
    if (d.point.size() != (size_t)(m - 7)) throw std::runtime_error("packed-direct point length");
    target += gd[k] * d.value;
    std::vector<size_t> live;
    std::vector<F128> live_coords;
    for (size_t i = 0; i < d.point.size(); i++)
      if (!d.point[i].is_zero()) { live.push_back(i); live_coords.push_back(d.point[i]); }
    std::vector<F128> t = build_eq(live_coords);
    for (size_t c = 0; c < t.size(); c++) {
      size_t idx = 0;
      for (size_t j = 0; j < live.size(); j++) idx |= ((c >> j) & 1) << live[j];
      bc[idx] += gd[k] * t[c];
    }
  }
  if (after_core) last_open_identity_ok() = open_identity(z, bc, target);
  bd.lig = ligerito_prove(cfg, z, bc, target, l0, ch);
  return bd;
}

Bundle prove(const std::vector<Compression>& blocks, int n_log, const std::string& domain) {
  return prove_with(blocks, n_log, domain, CoreHook());
}

// sum_j b_combined[j] * z_packed[j] == target: the batched open's claim, which
// the Ligerito sumcheck then proves (pcs.rs:130-290)
bool open_identity(const std::vector<F128>& z, const std::vector<F128>& bc, F128 target) {
  std::vector<F128> part(par_threads(), ZERO);
  par_for(z.size(), [&](size_t i0, size_t i1, int ti) {
    F128 acc = ZERO;
    for (size_t i = i0; i < i1; i++) acc += bc[i] * z[i];
    part[ti] = acc;
  });
  F128 s = ZERO;
  for (const F128& p : part) s += p;
  return s == target;
}

bool& last_open_identity_ok() {
  static thread_local bool ok = false;
  return ok;
}

}  // namespace flockref
