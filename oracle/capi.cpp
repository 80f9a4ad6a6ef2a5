// extern "C" surface of the oracle for the Python test harness (ctypes).
// Test infrastructure only (see flockref.hpp): loaded by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline / reference arm.
#include "flockref.hpp"
#include <chrono>
#include <cstdio>

using namespace flockref;

extern "C" {

int flockref_prove(uint32_t log2, uint64_t seed, uint8_t* out, size_t cap, size_t* out_len) {
  try {
    auto blocks = generate_compressions(log2, seed);
    Bundle b = prove(blocks, (int)log2, "flock-bench-v0");
    std::vector<uint8_t> bytes = serialize(b);
    *out_len = bytes.size();
    if (bytes.size() > cap) return 2;
    memcpy(out, bytes.data(), bytes.size());
    return 0;
  } catch (...) {
    return 1;
  }
}

// Hash chains.  A compression record is 28 u32: cv[8], m[16], counter (u64,
// little endian), block_len, flags -- the layout of flockref::Compression.
static_assert(sizeof(Compression) == 112, "compression record");

void flockref_chain_blocks(uint64_t seed, const uint32_t* initial_cv, size_t steps, uint32_t* out28) {
  std::vector<Compression> v = chain_blocks(seed, initial_cv ? initial_cv : b3::IV, steps);
  memcpy(out28, v.data(), v.size() * sizeof(Compression));
}

// prove_fast over any n >= 1 given compressions (Blake3Setup::new(n) +
// prove_fast, blake3.rs:1854-1858, 4706-4780, 4846): the statement has
// 2^n_log slots with n_log = max(3, ceil(log2 n)) (min_n_blocks_log), and
// slots n.. hold the all-zero compression (the `padding` of
// generate_witness_with_ab_packed_and_round1_inner_impl_with_commit,
// blake3.rs:2527, with BlockSource::with_block, seed_pipe.rs:210-226).
int flockref_prove_records(const uint32_t* blocks28, size_t n, const uint8_t* domain, size_t dlen, uint8_t* out,
                           size_t cap, size_t* out_len) {
  try {
    if (n == 0) return 3;
    int n_log = 3;
    while (((size_t)1 << n_log) < n) n_log++;
    std::vector<Compression> blocks(n);
    memcpy(blocks.data(), blocks28, n * sizeof(Compression));
    Bundle b = prove(blocks, n_log, std::string((const char*)domain, dlen));
    std::vector<uint8_t> bytes = serialize(b);
    *out_len = bytes.size();
    if (bytes.size() > cap) return 2;
    memcpy(out, bytes.data(), bytes.size());
    return 0;
  } catch (...) {
    return 1;
  }
}

// prove_chain over 2^log2 given compressions.  `check` receives 1 when the
// shift argument verifies from the bundle's public endpoints and the batched
// open's claim identity holds.  A non-null `cv_last` replaces the public
// output endpoint (written to the bundle and used by that check).
int flockref_prove_chain_blocks(const uint32_t* blocks28, uint32_t log2, const uint8_t* domain, size_t dlen,
                                const uint32_t* cv_last, uint8_t* out, size_t cap, size_t* out_len, int* check) {
  try {
    std::vector<Compression> blocks((size_t)1 << log2);
    memcpy(blocks.data(), blocks28, blocks.size() * sizeof(Compression));
    std::string d((const char*)domain, dlen);
    bool ok = false;
    ChainBundle cb = prove_chain(blocks, (int)log2, d, &ok, cv_last);
    if (check) *check = ok ? 1 : 0;
    std::vector<uint8_t> bytes = serialize_chain(cb);
    *out_len = bytes.size();
    if (bytes.size() > cap) return 2;
    memcpy(out, bytes.data(), bytes.size());
    return 0;
  } catch (...) {
    return 1;
  }
}

// Keccak chains: 2^log2 states (25 u64 lanes each); claimed_last: 25 lanes or null
int flockref_prove_keccak_chain(const uint64_t* states25, uint32_t log2, const uint8_t* domain, size_t dlen,
                                const uint64_t* claimed_last, uint8_t* out, size_t cap, size_t* out_len,
                                int* check) {
  try {
    std::vector<keccak::State> st((size_t)1 << log2);
    memcpy(st.data(), states25, st.size() * sizeof(keccak::State));
    bool ok = false;
    ChainBundle cb = prove_keccak_chain(st, (int)log2, std::string((const char*)domain, dlen), &ok, claimed_last);
    if (check) *check = ok ? 1 : 0;
    std::vector<uint8_t> bytes = serialize_chain(cb);
    *out_len = bytes.size();
    if (bytes.size() > cap) return 2;
    memcpy(out, bytes.data(), bytes.size());
    return 0;
  } catch (const std::exception& e) {
    fprintf(stderr, "flockref_prove_keccak_chain: %s\n", e.what());
    return 1;
  }
}

// SHA-256 chains: records of 24 u32 (h_in, m), 2^log2 of them
void flockref_sha256_chain_blocks(uint64_t seed, const uint32_t* initial, size_t steps, uint32_t* out24) {
  static const uint32_t iv[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  auto v = sha256_chain_blocks(seed, initial ? initial : iv, steps);
  memcpy(out24, v.data(), v.size() * sizeof(sha::Compression));
}
int flockref_prove_sha256_chain(const uint32_t* blocks24, uint32_t log2, const uint8_t* domain, size_t dlen,
                                const uint32_t* cv_last, uint8_t* out, size_t cap, size_t* out_len, int* check) {
  try {
    std::vector<sha::Compression> blocks((size_t)1 << log2);
    memcpy(blocks.data(), blocks24, blocks.size() * sizeof(sha::Compression));
    bool ok = false;
    ChainBundle cb = prove_sha256_chain(blocks, (int)log2, std::string((const char*)domain, dlen), &ok, cv_last);
    if (check) *check = ok ? 1 : 0;
    std::vector<uint8_t> bytes = serialize_chain(cb);
    *out_len = bytes.size();
    if (bytes.size() > cap) return 2;
    memcpy(out, bytes.data(), bytes.size());
    return 0;
  } catch (const std::exception& e) {
    fprintf(stderr, "flockref_prove_sha256_chain: %s\n", e.what());
    return 1;
  }
}

void flockref_f128_mul(const uint64_t* a, const uint64_t* b, uint64_t* out) {
  F128 r = F128(a[0], a[1]) * F128(b[0], b[1]);
  out[0] = r.lo;
  out[1] = r.hi;
}
// element-wise products of n F128 values ({lo, hi} pairs)
void flockref_f128_mul_n(const uint64_t* a, const uint64_t* b, size_t n, uint64_t* out) {
  for (size_t i = 0; i < n; i++) {
    F128 r = F128(a[2 * i], a[2 * i + 1]) * F128(b[2 * i], b[2 * i + 1]);
    out[2 * i] = r.lo;
    out[2 * i + 1] = r.hi;
  }
}
void flockref_f128_inv(const uint64_t* a, uint64_t* out) {
  F128 r = f128_inv(F128(a[0], a[1]));
  out[0] = r.lo;
  out[1] = r.hi;
}
void flockref_phi8_table(uint64_t* out512) {
  const F128* t = phi8_table();
  for (int i = 0; i < 256; i++) { out512[2 * i] = t[i].lo; out512[2 * i + 1] = t[i].hi; }
}
uint8_t flockref_gf8_mul(uint8_t a, uint8_t b) { return gf8_mul(a, b); }

void flockref_blake3_hash(const uint8_t* d, size_t n, uint8_t* out32) { b3::hash(d, n, out32); }
void flockref_blake3_xof(const uint8_t* d, size_t n, uint8_t* out, size_t olen) {
  b3::Hasher h;
  h.update(d, n);
  h.finalize_xof(out, olen);
}
void flockref_blake3_leaf_cv(const uint8_t* d, size_t n, uint8_t* out32) { b3::leaf_cv(d, n, out32); }
void flockref_blake3_parent_cv(const uint8_t* l, const uint8_t* r, uint8_t* out32) { b3::parent_cv(l, r, out32); }

void flockref_generate_compressions(uint32_t log2, uint64_t seed, uint32_t* out25) {
  auto v = generate_compressions(log2, seed);
  for (size_t i = 0; i < v.size(); i++) {
    uint32_t* o = out25 + 25 * i;
    memcpy(o, v[i].cv, 32);
    memcpy(o + 8, v[i].m, 64);
    o[24] = (uint32_t)v[i].counter;
  }
}

// z, a, b: 2^(14 + n_log - 7) F128 each (as u64 pairs)
void flockref_witness(uint32_t log2, uint64_t seed, uint64_t* z, uint64_t* a, uint64_t* b) {
  auto blocks = generate_compressions(log2, seed);
  std::vector<F128> vz, va, vb;
  generate_witness(blocks, (int)log2, vz, va, vb);
  memcpy(z, vz.data(), vz.size() * 16);
  memcpy(a, va.data(), va.size() * 16);
  memcpy(b, vb.data(), vb.size() * 16);
}

// a_out, b_out = A0 z, B0 z for n_blocks blocks of packed z (matrix apply)
void flockref_apply_matrices(const uint64_t* z, int n_blocks, uint64_t* a_out, uint64_t* b_out) {
  const R1cs& rc = blake3_r1cs(3);
  size_t n = (size_t)n_blocks * (K / 128);
  std::vector<F128> vz(n), va, vb;
  memcpy(vz.data(), z, n * 16);
  apply_block_diag(rc.a0, vz, n_blocks, va);
  apply_block_diag(rc.b0, vz, n_blocks, vb);
  memcpy(a_out, va.data(), n * 16);
  memcpy(b_out, vb.data(), n * 16);
}

void flockref_statement_digest(uint32_t n_log, uint8_t* out32) {
  const R1cs& rc = blake3_r1cs((int)n_log);
  memcpy(out32, rc.digest.data(), 32);
}
uint64_t flockref_matrix_nnz(int which) {
  const R1cs& rc = blake3_r1cs(3);
  return which == 0 ? rc.a0.col.size() : rc.b0.col.size();
}
// CSR export of A0 (which=0) / B0 (which=1): ptr[K+1], col[nnz]
void flockref_matrix_csr(int which, uint32_t* ptr, uint16_t* col) {
  const R1cs& rc = blake3_r1cs(3);
  const SparseRows& s = which == 0 ? rc.a0 : rc.b0;
  memcpy(ptr, s.ptr.data(), s.ptr.size() * 4);
  memcpy(col, s.col.data(), s.col.size() * 2);
}

// RS encode: msg has n_pos positions x lanes (position-major); out 2^rate x larger
void flockref_rs_encode(const uint64_t* msg, size_t n_pos, size_t lanes, int log_inv_rate, uint64_t* out) {
  std::vector<F128> m(n_pos * lanes), cw;
  memcpy(m.data(), msg, m.size() * 16);
  rs_encode(m, lanes, log_inv_rate, cw);
  memcpy(out, cw.data(), cw.size() * 16);
}
void flockref_ntt_twiddles(int dim, uint64_t* out) {
  const AdditiveNtt& n = standard_ntt(dim);
  memcpy(out, n.twiddles.data(), n.twiddles.size() * 16);
}

// Merkle: tree of 2n-1 nodes (32 B each)
void flockref_merkle_tree(const uint8_t* data, size_t n_leaves, size_t leaf_size, uint8_t* tree_out) {
  auto t = merkle_tree(data, n_leaves, leaf_size);
  memcpy(tree_out, t.data(), t.size() * 32);
}
size_t flockref_merkle_multi_proof(const uint8_t* tree, size_t n_leaves, const uint64_t* pos, size_t npos,
                                   uint8_t* out, size_t cap_nodes) {
  std::vector<Hash> t(2 * n_leaves - 1);
  memcpy(t.data(), tree, t.size() * 32);
  std::vector<size_t> p(pos, pos + npos);
  auto pr = merkle_multi_proof(t, n_leaves, p);
  if (pr.size() <= cap_nodes) memcpy(out, pr.data(), pr.size() * 32);
  return pr.size();
}

void flockref_build_eq(const uint64_t* r, int n, uint64_t* out) {
  std::vector<F128> v(n);
  memcpy(v.data(), r, n * 16);
  auto e = build_eq(v);
  memcpy(out, e.data(), e.size() * 16);
}
void flockref_lagrange(const uint64_t* z, int node_base, uint64_t* out64) {
  auto w = lagrange_weights(K_SKIP, F128(z[0], z[1]), node_base);
  memcpy(out64, w.data(), 64 * 16);
}

// Challenger script: domain, then ops; used to pin transcript framing.
void* flockref_ch_new(const char* domain) { return new Challenger(domain); }
void flockref_ch_free(void* c) { delete (Challenger*)c; }
void flockref_ch_label(void* c, const char* l) { ((Challenger*)c)->observe_label(l); }
void flockref_ch_observe(void* c, const uint64_t* v) { ((Challenger*)c)->observe_f128(F128(v[0], v[1])); }
void flockref_ch_observe_slice(void* c, const uint64_t* v, size_t n) {
  std::vector<F128> x(n);
  memcpy(x.data(), v, n * 16);
  ((Challenger*)c)->observe_f128_slice(x);
}
void flockref_ch_bytes(void* c, const uint8_t* d, size_t n) { ((Challenger*)c)->observe_bytes(d, n); }
void flockref_ch_sample(void* c, uint64_t* out) {
  F128 v = ((Challenger*)c)->sample_f128();
  out[0] = v.lo;
  out[1] = v.hi;
}
void flockref_ch_sample_vec(void* c, size_t n, uint64_t* out) {
  auto v = ((Challenger*)c)->sample_f128_vec(n);
  memcpy(out, v.data(), n * 16);
}
uint64_t flockref_ch_grind(void* c, uint32_t bits) { return ((Challenger*)c)->grind_pow(bits); }
void flockref_ch_digest(void* c, uint8_t* out32) { ((Challenger*)c)->state_digest(out32); }
int flockref_pow_ok(const uint8_t* digest, uint64_t nonce, uint32_t bits) { return pow_ok(digest, nonce, bits); }

// ---- SHA-256 compressions.  A record is 24 u32: h_in[8], m[16].
static_assert(sizeof(sha::Compression) == 96, "sha-256 record");

void flockref_sha256_compress(const uint32_t* h, const uint32_t* m, uint32_t* out8) { sha::compress(h, m, out8); }
void flockref_sha256_bench_inputs(size_t n, uint64_t seed, uint32_t* out24) {
  auto v = sha::bench_inputs(n, seed);
  memcpy(out24, v.data(), v.size() * sizeof(sha::Compression));
}
int flockref_sha256_min_n_blocks_log(size_t n) { return sha::min_n_blocks_log(n); }
void flockref_sha256_digest(uint32_t n_log, uint8_t* out32) {
  memcpy(out32, sha256_r1cs((int)n_log).digest.data(), 32);
}
uint64_t flockref_sha256_matrix_nnz(int which) {
  const R1cs& rc = sha256_r1cs(3);
  return which == 0 ? rc.a0.col.size() : rc.b0.col.size();
}
// CSR export of A0 (which=0) / B0 (which=1): ptr[2^15 + 1], col[nnz]
void flockref_sha256_matrix_csr(int which, uint32_t* ptr, uint16_t* col) {
  const R1cs& rc = sha256_r1cs(3);
  const SparseRows& s = which == 0 ? rc.a0 : rc.b0;
  memcpy(ptr, s.ptr.data(), s.ptr.size() * 4);
  memcpy(col, s.col.data(), s.col.size() * 2);
}
// z, a, b: 2^(15 + n_log - 7) F128 each, for n records over 2^n_log blocks
void flockref_sha256_witness(const uint32_t* rec24, size_t n, uint32_t n_log, uint64_t* z, uint64_t* a,
                             uint64_t* b) {
  std::vector<sha::Compression> blocks(n);
  memcpy(blocks.data(), rec24, n * sizeof(sha::Compression));
  std::vector<F128> vz, va, vb;
  generate_sha256_witness(blocks, (int)n_log, vz, va, vb);
  memcpy(z, vz.data(), vz.size() * 16);
  memcpy(a, va.data(), va.size() * 16);
  memcpy(b, vb.data(), vb.size() * 16);
}
// Sha256HybridSetup::new(n) + prove_fast over n >= 1 records
int flockref_prove_sha256(const uint32_t* rec24, size_t n, const uint8_t* domain, size_t dlen, uint8_t* out,
                          size_t cap, size_t* out_len) {
  try {
    if (n == 0) return 3;
    std::vector<sha::Compression> blocks(n);
    memcpy(blocks.data(), rec24, n * sizeof(sha::Compression));
    Bundle b = prove_sha256(blocks, sha::min_n_blocks_log(n), std::string((const char*)domain, dlen));
    std::vector<uint8_t> bytes = serialize(b);
    *out_len = bytes.size();
    if (bytes.size() > cap) return 2;
    memcpy(out, bytes.data(), bytes.size());
    return 0;
  } catch (...) {
    return 1;
  }
}

// A proof of the all-zero witness of the SHA-256 statement over 2^n_log
// blocks (it satisfies every row but the constant wire's pin; sha2.rs:2292
// const_pin_all_zero_rejected)
int flockref_prove_sha256_zero(uint32_t n_log, const uint8_t* domain, size_t dlen, uint8_t* out, size_t cap,
                               size_t* out_len) {
  try {
    const size_t words = (size_t)1 << (sha::K_LOG_SHA + n_log - 7);
    std::vector<F128> z(words, ZERO), a(words, ZERO), b(words, ZERO);
    Bundle bd = prove_core(sha256_r1cs((int)n_log), std::move(z), a, b, std::string((const char*)domain, dlen),
                           CoreHook());
    std::vector<uint8_t> bytes = serialize(bd);
    *out_len = bytes.size();
    if (bytes.size() > cap) return 2;
    memcpy(out, bytes.data(), bytes.size());
    return 0;
  } catch (...) {
    return 1;
  }
}

// SHA-256 Merkle paths: the honest inputs (records 24 u32, b bits, leaves
// 8 u32 each, root) and the proof over given inputs; `check` as for chains.
void flockref_sha256_merkle_inputs(uint32_t n_log, uint32_t path_log, uint64_t seed, uint32_t* rec24, uint8_t* b,
                                   uint32_t* leaves, uint32_t* root) {
  MerklePathInputs in = sha256_merkle_paths((int)n_log, (int)path_log, seed);
  memcpy(rec24, in.blocks.data(), in.blocks.size() * 96);
  memcpy(b, in.b_bits.data(), in.b_bits.size());
  for (size_t p = 0; p < in.leaves.size(); p++) memcpy(leaves + 8 * p, in.leaves[p].data(), 32);
  memcpy(root, in.root.data(), 32);
}
int flockref_prove_sha256_merkle(const uint32_t* rec24, const uint8_t* b, const uint32_t* leaves,
                                 const uint32_t* root, uint32_t n_log, uint32_t path_log, const uint8_t* domain,
                                 size_t dlen, uint8_t* out, size_t cap, size_t* out_len, int* check) {
  try {
    const size_t N = (size_t)1 << n_log;
    MerklePathInputs in;
    in.blocks.resize(N);
    memcpy(in.blocks.data(), rec24, N * 96);
    in.b_bits.assign(b, b + N);
    in.leaves.resize((size_t)1 << path_log);
    for (size_t p = 0; p < in.leaves.size(); p++) memcpy(in.leaves[p].data(), leaves + 8 * p, 32);
    memcpy(in.root.data(), root, 32);
    bool ok = false;
    MerkleBundle mb = prove_sha256_merkle(in, (int)n_log, (int)path_log, std::string((const char*)domain, dlen), &ok);
    if (check) *check = ok ? 1 : 0;
    std::vector<uint8_t> bytes = serialize_merkle(mb);
    *out_len = bytes.size();
    if (bytes.size() > cap) return 2;
    memcpy(out, bytes.data(), bytes.size());
    return 0;
  } catch (...) {
    return 1;
  }
}

// The hash kinds (0 SHA-256, 1 BLAKE3) of the proofs this thread makes next:
// the PCS Merkle trees and the transcript (PcsParams::merkle_hash,
// FsChallenger::with_hash).
void flockref_set_hash_kinds(int merkle, int transcript) {
  hash_kinds().merkle = merkle;
  hash_kinds().transcript = transcript;
}
void flockref_sha256(const uint8_t* d, size_t n, uint8_t* out32) { sha::hash(d, n, out32); }
void flockref_merkle_tree_hash(const uint8_t* data, size_t n_leaves, size_t leaf_size, int kind, uint8_t* tree_out) {
  auto t = merkle_tree(data, n_leaves, leaf_size, kind);
  memcpy(tree_out, t.data(), t.size() * 32);
}
void* flockref_ch_new_hash(const char* domain, int kind) { return new Challenger(domain, kind); }

// ---- Keccak-f[1600].  A state is 25 u64 lanes (lane x + 5y, bit z).  width:
// 1 = the single encoder (keccak.rs), 3 = the 3-wide one (keccak3.rs).
static_assert(sizeof(keccak::State) == 200, "keccak state");
static const keccak::Layout& layout_of(int width) {
  return width == 3 ? keccak::wide_layout() : keccak::single_layout();
}
void flockref_keccak_f(uint64_t* lanes25) { keccak::permute(lanes25); }
void flockref_keccak_bench_inputs(size_t n, uint64_t seed, uint64_t* out25) {
  auto v = keccak::bench_inputs(n, seed);
  memcpy(out25, v.data(), v.size() * sizeof(keccak::State));
}
void flockref_keccak_digest(int width, uint32_t n_log, uint8_t* out32) {
  memcpy(out32, keccak_r1cs(layout_of(width), (int)n_log).digest.data(), 32);
}
// z, a, b: 2^(k_log + n_log - 7) F128 each
void flockref_keccak_witness(int width, const uint64_t* states, size_t n, uint32_t n_log, uint64_t* z, uint64_t* a,
                             uint64_t* b) {
  std::vector<keccak::State> s(n);
  memcpy(s.data(), states, n * sizeof(keccak::State));
  std::vector<F128> vz, va, vb;
  generate_keccak_witness(layout_of(width), s, (int)n_log, vz, va, vb);
  memcpy(z, vz.data(), vz.size() * 16);
  memcpy(a, va.data(), va.size() * 16);
  memcpy(b, vb.data(), vb.size() * 16);
}
// the walker's alpha A^T e + B^T e over the block's 2^k_log rows
void flockref_keccak_comb(int width, const uint64_t* alpha, const uint64_t* e, uint64_t* out) {
  const keccak::Layout& L = layout_of(width);
  std::vector<F128> ev((size_t)1 << L.k_log);
  memcpy(ev.data(), e, ev.size() * 16);
  auto c = keccak::lincheck_comb(L, F128(alpha[0], alpha[1]), ev);
  memcpy(out, c.data(), c.size() * 16);
}
int flockref_prove_keccak(int width, const uint64_t* states, size_t n, const uint8_t* domain, size_t dlen,
                          uint8_t* out, size_t cap, size_t* out_len) {
  try {
    if (n == 0) return 3;
    const keccak::Layout& L = layout_of(width);
    std::vector<keccak::State> s(n);
    memcpy(s.data(), states, n * sizeof(keccak::State));
    Bundle b = prove_keccak(L, s, keccak::min_n_blocks_log(L, n), std::string((const char*)domain, dlen));
    std::vector<uint8_t> bytes = serialize(b);
    *out_len = bytes.size();
    if (bytes.size() > cap) return 2;
    memcpy(out, bytes.data(), bytes.size());
    return 0;
  } catch (...) {
    return 1;
  }
}

// round1_deg4_naive over packed rows (2^(m-6) u64 per vector); r: m F128;
// outputs: 192 F128 each
void flockref_round1_deg4(const uint64_t* a, const uint64_t* b, const uint64_t* c, const uint64_t* d,
                          const uint64_t* z, uint32_t m, const uint64_t* r, uint64_t* p_abcd, uint64_t* p_z) {
  std::vector<F128> rv(m);
  memcpy(rv.data(), r, m * 16);
  std::vector<F128> pa, pz;
  round1_deg4(a, b, c, d, z, (int)m, rv, pa, pz);
  memcpy(p_abcd, pa.data(), 192 * 16);
  memcpy(p_z, pz.data(), 192 * 16);
}

// Whether the last proof on this thread that records it (chain, Merkle-path
// and Keccak proofs) had sum_j b_combined[j] z[j] == target.
int flockref_last_open_identity_ok(void) { return last_open_identity_ok() ? 1 : 0; }

// Wall-clock seconds of one full oracle prove at log2 (for the CPU baseline).
double flockref_time_prove(uint32_t log2, uint64_t seed, size_t* proof_len) {
  auto blocks = generate_compressions(log2, seed);
  blake3_r1cs((int)log2);
  auto t0 = std::chrono::steady_clock::now();
  Bundle b = prove(blocks, (int)log2, "flock-bench-v0");
  std::vector<uint8_t> bytes = serialize(b);
  auto t1 = std::chrono::steady_clock::now();
  *proof_len = bytes.size();
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
