// Host-side support of the B200 prover: field ops on small vectors, the
// BLAKE3 Fiat-Shamir transcript, the BLAKE3-compression R1CS statement, the
// Ligerito ladder configs and the FLOCK wire format.  Everything here is
// O(transcript) work between GPU phases; all O(witness) work is on the GPU.
#pragma once
#include <array>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include "gf128.cuh"

namespace flock {

// ---- GF(2^128) on the host (PCLMULQDQ); gf2_128.rs:22-265 semantics ----
f128 hmul(f128 a, f128 b);
f128 hinv(f128 a);
inline f128 hadd(f128 a, f128 b) { return fx(a, b); }
const f128* phi8_table();              // field/phi8.rs:18-1050 (basis-expanded)
inline const f128 hone() { return mk(1, 0); }
std::vector<f128> heq(const std::vector<f128>& r);           // eq table, bit i <-> r[i]
std::vector<f128> hlagrange(f128 z, int node_base);           // 64 weights over phi8 nodes
// 64 x 64 bit transpose in place (row r = a[r], column c = bit c)
void transpose64(uint64_t a[64]);
// 128 x 128 bit transpose: bit i of out[j] = bit j of rows[i] (128 rows)
std::vector<f128> transpose128(const std::vector<f128>& rows);
// out[v] = XOR of v8[j] over the set bits j of v, v < 256
void subset_sums8(const f128* v8, f128* out);
uint8_t hgf8_mul(uint8_t a, uint8_t b);

// ---- BLAKE3 hasher (incremental, root / XOF) ----
class B3 {
 public:
  B3();
  void update(const void* p, size_t n);
  void xof(uint8_t* out, size_t n) const;
  void digest(uint8_t out[32]) const { xof(out, 32); }
 private:
  void chunk_done();
  uint32_t cv_[8];
  uint64_t chunk_ = 0;
  uint8_t buf_[64];
  size_t blen_ = 0;
  int nblk_ = 0;
  std::vector<std::array<uint32_t, 8>> stack_;
};
void b3_compress(const uint32_t cv[8], const uint32_t m[16], uint64_t ctr, uint32_t blen, uint32_t flags, uint32_t out[16]);
extern const uint32_t kB3IV[8];  // the BLAKE3 IV (the SHA-256 initial hash words)

// The hash function behind a Merkle tree or a Fiat-Shamir transcript
// (HashKind, crates/flock-core/src/hash.rs:20-30; these are its serde
// discriminants, and Sha256 is the reference's default).
enum HashFn : int { kFnSha256 = 0, kFnBlake3 = 1 };

// ---- SHA-256 hasher (FIPS 180-4), incremental; copies are snapshots ----
class S256 {
 public:
  S256();
  void update(const void* p, size_t n);
  void digest(uint8_t out[32]) const;
 private:
  uint32_t h_[8];
  uint8_t buf_[64];
  size_t blen_ = 0;
  uint64_t total_ = 0;
};
void sha256_bytes(const void* p, size_t n, uint8_t out[32]);

// ---- Fiat-Shamir transcript (challenger.rs:170-600) ----
class Transcript {
 public:
  // FsChallenger::with_hash(domain, fn) (challenger.rs:227-250)
  explicit Transcript(const std::string& domain, int fn = kFnBlake3);
  void label(const char* s);
  void f128v(f128 v);
  void f128s(const f128* v, size_t n);
  void bytes(const void* p, size_t n);
  f128 sample();
  std::vector<f128> sample_vec(size_t n);
  void state_digest(uint8_t out[32]) const {
    if (fn_ == kFnSha256) s_.digest(out);
    else h_.digest(out);
  }
  int fn() const { return fn_; }
  void nonce(uint64_t n) { uint8_t b[8]; for (int i = 0; i < 8; i++) b[i] = (uint8_t)(n >> (8 * i)); bytes(b, 8); }
  // a label of arbitrary bytes (label() takes a C string)
  void label_bytes(const void* p, size_t n);
  // FsChallenger::verify_pow (challenger.rs:502-545, 580-601): the hash of
  // state digest || nonce (LE) -- BLAKE3 pads the preimage with 0^24, SHA-256
  // does not -- has `bits` leading zero bits (bits = 0: the nonce is 0); the
  // nonce is observed either way
  bool verify_pow(uint64_t nonce, uint32_t bits);
 private:
  void put(const void* p, size_t n) {
    if (fn_ == kFnSha256) s_.update(p, n);
    else h_.update(p, n);
  }
  // squeeze_into (challenger.rs:288-303): the BLAKE3 XOF of the state, or
  // SHA256(state || ctr LE) for ctr = 0, 1, ... (32 bytes each)
  void squeeze(uint8_t* out, size_t n) const;
  int fn_ = kFnBlake3;
  B3 h_;
  S256 s_;
};

// The smallest nonce whose BLAKE3 root hash of (digest || nonce LE || 0^24)
// has `bits` leading zero bits, searched on the host (grind_pow,
// challenger.rs:384-475): for a few bits this is cheaper than a GPU round trip.
uint64_t pow_search_host(const uint8_t digest[32], uint32_t bits, int fn = kFnBlake3);
// the PoW predicate (challenger.rs:580-601)
bool pow_hash_ok(const uint8_t digest[32], uint64_t nonce, uint32_t bits, int fn);
// grinds of at most this many bits run on the host
constexpr uint32_t kHostPowBits = 6;

// Ligerito query positions: `count` distinct values sample().lo % block_len,
// first occurrences kept, sorted (pcs/ligerito.rs:9665-9718)
std::vector<size_t> sample_distinct_queries(Transcript& tr, size_t block_len, size_t count);
size_t ceil_log2(size_t n);
// the zerocheck's fixed inner challenges (univariate_skip_optimized.rs:198-215):
// phi8(0xF7), phi8(0x53), phi8(0xB5) and gamma^(2^i) / (1 + gamma^(2^i)),
// gamma = x, i = 1, 2, 4, 8 as shifts
std::vector<f128> small_consts();
std::vector<f128> medium_consts();

// ---- R1CS statements: one compression per 2^k_log-bit block ----
// The hash a statement encodes.  BLAKE3 (r1cs_hashes/blake3.rs): 2^14-bit
// blocks, constant wire at bit 512.  SHA-256 (r1cs_hashes/sha2.rs): 2^15-bit
// blocks, constant wire at bit 31400.  Keccak-f[1600] (r1cs_hashes/keccak.rs):
// 2^16-bit blocks, constant wire at bit 4096, implicit matrices (the block
// statement is the empty stub of common.rs:120-138; the lincheck applies
// them through keccak_comb).  3-wide Keccak (r1cs_hashes/keccak3.rs): three
// permutations per 2^17-bit block, constant wire at bit 12288.
enum HashKind : int { kHashBlake3 = 0, kHashSha256 = 1, kHashKeccak = 2, kHashKeccak3 = 3 };
constexpr int kKLog = 14, kK = 1 << kKLog, kKSkip = 6, kZConst = 512, kUseful = 15409;
constexpr int kShaKLog = 15, kShaZConst = 31400, kShaUseful = 31401;
constexpr int kKeccakKLog = 16, kKeccakZConst = 4096, kKeccakUseful = 42560;
constexpr int kKeccak3KLog = 17, kKeccak3ZConst = 12288, kKeccak3Useful = 127552;
constexpr int kMaxKLog = kKeccak3KLog;  // the largest block of the statements
struct Statement {
  int k_log = kKLog, z_const = kZConst, useful = kUseful;
  bool implicit = false;                 // matrices applied by a walker, not stored
  std::vector<uint32_t> a_ptr, b_ptr;    // CSR rows
  std::vector<uint16_t> a_col, b_col;
  std::vector<uint32_t> at_ptr, bt_ptr;  // CSC (column -> rows)
  std::vector<uint16_t> at_row, bt_row;
};
const Statement& statement(int hash);    // matrices (built once per process)
inline const Statement& blake3_statement() { return statement(kHashBlake3); }
std::array<uint8_t, 32> statement_digest(int hash, int m);
inline std::array<uint8_t, 32> statement_digest(int m) { return statement_digest(kHashBlake3, m); }
// sha256_compress (r1cs_hashes/sha2.rs:1502-1546): out = h_in + rounds(h_in, m)
void sha256_compress(const uint32_t h_in[8], const uint32_t m[16], uint32_t out[8]);
// keccak_f (keccak.rs:423-428, FIPS 202 Keccak-f[1600]) on 25 lanes (lane
// x + 5y, bit z), in place
void keccak_f(uint64_t lanes[25]);
// block size of a hash's statement (log2 bits)
inline int hash_k_log(int hash) {
  return hash == kHashSha256 ? kShaKLog : hash == kHashKeccak ? kKeccakKLog : hash == kHashKeccak3 ? kKeccak3KLog : kKLog;
}
inline bool known_hash(int hash) { return hash >= kHashBlake3 && hash <= kHashKeccak3; }
inline bool is_keccak(int hash) { return hash == kHashKeccak || hash == kHashKeccak3; }
// A statement's hash-chain geometry (ChainLayout, chain_common.rs:29-63): the
// input and output regions are aligned 2^region_log-bit slots at packed words
// 0 and out_word of each block, holding region_bits real bits
// (blake3.rs:5160-5167, sha2.rs:1476-1483, keccak.rs:839-846).
struct ChainGeom {
  int region_log, out_word, region_bits, kind;  // kind: the bundle's HashKind
};
inline ChainGeom chain_geom(int hash) {
  if (hash == kHashKeccak) return ChainGeom{11, 16, 1600, 2};
  return ChainGeom{8, 2, 256, hash == kHashSha256 ? 1 : 0};
}
// permutations per block of a Keccak statement
inline int keccak_width(int hash) { return hash == kHashKeccak3 ? 3 : 1; }

// ---- Ligerito fast ladder (configs/ligerito/m*_fast.toml) ----
struct Ladder {
  int initial_k = 6, yr_log_n = 0;
  std::vector<int> rate, ks, queries, grind, fold_grind, ood;  // per level
};
const Ladder* ladder_for(int m);

// ---- proof object + FLOCK v4 bincode-fixint writer (proof_io.rs:40-215) ----
using H32 = std::array<uint8_t, 32>;
struct Opening { std::vector<std::vector<f128>> rows; std::vector<H32> proof; };
struct Proof {
  H32 root{};
  uint64_t m = 0;
  std::vector<f128> r1_ab, r1_c;
  std::vector<std::pair<f128, f128>> zc_rounds;
  f128 fa{}, fb{}, fc{};
  std::vector<std::pair<f128, f128>> lc_rounds;
  std::vector<f128> z_partial;
  std::vector<std::vector<f128>> s_hat_v;
  H32 lig_root{};
  Opening initial;
  std::vector<H32> roots;
  std::vector<Opening> levels;
  std::vector<f128> yr;
  Opening final_open;
  std::vector<std::pair<f128, f128>> sc_msgs;
  std::vector<uint64_t> grind_nonces, fold_nonces;
  std::vector<f128> ood;
  // hash-chain bundle (flavor 3): the shift argument and public endpoints
  bool chain = false;
  uint32_t chain_kind = 0;  // the bundle's HashKind (proof_io.rs:51-58): 0 Blake3, 1 Sha2, 2 Keccak
  std::vector<std::pair<f128, f128>> shift_rounds;
  f128 g_at_point{};
  // the public endpoints in the region's physical bit order (bit i of the
  // region = bit i % 64 of word i / 64), end_bits of them
  uint64_t end0[32] = {}, end_last[32] = {};
  int end_bits = 256;
  // SHA-256 Merkle-path proof: the shift sumcheck's (q(1), q(w), q(w+1))
  // rounds (g_at_point above); encoded as bincode of (Commitment,
  // MerklePathProofLigerito), without a FLOCK header
  bool merkle = false;
  std::vector<std::array<f128, 3>> mp_rounds;
  int merkle_fn = kFnBlake3;  // PcsParams::merkle_hash of the commitment
};
std::vector<uint8_t> encode(const Proof& p);

}  // namespace flock
