// flockref — CPU restatement of the Flock BLAKE3-compression prover.
//
// TEST INFRASTRUCTURE ONLY. This directory is the oracle that the CUDA
// product is checked against: only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference arm of bench.py may load or run it, and only as
// the checker. The product library never links, loads or calls it.
//
// Parity pin: proofs produced by this restatement are accepted by the
// reference's own prebuilt trusted verifier
// (benchmark-tools/trusted/flock_benchmark_verifier, run as a program, never
// inspected), which recomputes the pristine witness + commitment root and
// replays the full transcript.  BLAKE3 primitives are pinned by the Python
// `blake3` module (root hashes) and by the verifier's root recompute.
//
// Every function cites the reference file:line it restates (paths relative
// to the reference project root).
#pragma once
#include <cstdint>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>
#include <array>
#include <functional>

namespace flockref {

// Parallel loops: FLOCKREF_THREADS host threads (default 1, the
// single-threaded restatement that the CPU baseline times).  Field sums are
// XORs, so a reduction's result does not depend on how a range is split.
int par_threads();
// f(begin, end, slice) over par_threads() contiguous slices of [0, n)
void par_for(size_t n, const std::function<void(size_t, size_t, int)>& f);

// ---------------------------------------------------------------------------
// GF(2^128), GHASH polynomial x^128 + x^7 + x^2 + x + 1, lo = x^0..63.
// crates/flock-core/src/field/gf2_128.rs:22-265, gf2_128/portable.rs.
// ---------------------------------------------------------------------------
struct F128 {
  uint64_t lo = 0, hi = 0;
  F128() = default;
  constexpr F128(uint64_t l, uint64_t h) : lo(l), hi(h) {}
  bool is_zero() const { return lo == 0 && hi == 0; }
  bool operator==(const F128& o) const { return lo == o.lo && hi == o.hi; }
  bool operator!=(const F128& o) const { return !(*this == o); }
};
static_assert(sizeof(F128) == 16, "F128 layout");
inline F128 operator+(F128 a, F128 b) { return F128(a.lo ^ b.lo, a.hi ^ b.hi); }
inline F128& operator+=(F128& a, F128 b) { a.lo ^= b.lo; a.hi ^= b.hi; return a; }
F128 operator*(F128 a, F128 b);
inline F128& operator*=(F128& a, F128 b) { a = a * b; return a; }
F128 f128_inv(F128 a);
inline const F128 ONE(1, 0);
inline const F128 ZERO(0, 0);

struct U256 { uint64_t r0 = 0, r1 = 0, r2 = 0, r3 = 0; };
U256 mul_unreduced(F128 a, F128 b);
F128 ghash_reduce(uint64_t r0, uint64_t r1, uint64_t r2, uint64_t r3);

// GF(2^8) with the AES polynomial 0x11B.  field/gf2_8.rs:20-140.
uint8_t gf8_mul(uint8_t a, uint8_t b);
uint8_t gf8_inv(uint8_t a);
// phi_8: GF(2^8) -> GF(2^128) field embedding.  field/phi8.rs:18-1050.
F128 phi8(uint8_t v);
const F128* phi8_table();

// ---------------------------------------------------------------------------
// BLAKE3 (spec restatement; crate blake3 1.8.6 semantics).
// ---------------------------------------------------------------------------
namespace b3 {
extern const uint32_t IV[8];
enum : uint32_t { CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8 };
void compress(const uint32_t cv[8], const uint8_t block[64], uint64_t counter,
              uint32_t block_len, uint32_t flags, uint32_t out[16]);
// compress with block given as 16 little-endian words
void compress_words(const uint32_t cv[8], const uint32_t m[16], uint64_t counter,
                    uint32_t block_len, uint32_t flags, uint32_t out[16]);

class Hasher {
 public:
  Hasher();
  void update(const void* data, size_t len);
  void finalize(uint8_t out32[32]) const;                // root hash
  void finalize_xof(uint8_t* out, size_t len) const;     // root XOF
  void finalize_non_root(uint8_t out32[32]) const;       // hazmat finalize_non_root
 private:
  struct Output { uint32_t cv[8]; uint8_t block[64]; uint32_t block_len; uint64_t counter; uint32_t flags; };
  Output final_output() const;
  void push_cv(const uint32_t cv[8], uint64_t total_chunks);
  uint32_t chunk_cv_[8];
  uint64_t chunk_counter_ = 0;
  uint8_t buf_[64];
  size_t buf_len_ = 0;
  uint8_t blocks_compressed_ = 0;
  std::vector<std::array<uint32_t, 8>> stack_;
};
void hash(const void* data, size_t len, uint8_t out32[32]);
// non-root chaining value of a leaf of any length (merkle.rs:192-197)
void leaf_cv(const void* data, size_t len, uint8_t out32[32]);
// parent chaining value (merkle.rs:199-203)
void parent_cv(const uint8_t l[32], const uint8_t r[32], uint8_t out32[32]);
}  // namespace b3

using Hash = std::array<uint8_t, 32>;

// ---------------------------------------------------------------------------
// The hash behind Merkle trees and the transcript: HashKind
// (crates/flock-core/src/hash.rs:20-30; Sha256 = 0 is the default).
// ---------------------------------------------------------------------------
enum HashKind : int { SHA256 = 0, BLAKE3 = 1 };
namespace sha {
// SHA-256 (FIPS 180-4) over bytes, incremental
class Hasher {
 public:
  Hasher();
  void update(const void* data, size_t len);
  void finalize(uint8_t out32[32]) const;
 private:
  uint32_t h_[8];
  uint8_t buf_[64];
  size_t blen_ = 0;
  uint64_t total_ = 0;
};
void hash(const void* data, size_t len, uint8_t out32[32]);
}  // namespace sha
// The hash kinds of the proofs the oracle makes on this thread (Merkle
// trees, transcript); both BLAKE3 unless set (the benchmark's choice).
struct HashKinds { int merkle = BLAKE3, transcript = BLAKE3; };
HashKinds& hash_kinds();

// ---------------------------------------------------------------------------
// Fiat-Shamir challenger over BLAKE3.  crates/flock-core/src/challenger.rs:170-380
// ---------------------------------------------------------------------------
class Challenger {
 public:
  // FsChallenger::with_hash (challenger.rs:227-250)
  explicit Challenger(const std::string& domain, int kind = BLAKE3);
  void observe_label(const std::string& label);
  void observe_f128(F128 v);
  void observe_f128_slice(const std::vector<F128>& v);
  void observe_bytes(const void* data, size_t len);
  F128 sample_f128();
  std::vector<F128> sample_f128_vec(size_t n);
  uint64_t grind_pow(uint32_t bits);           // smallest satisfying nonce
  bool verify_pow(uint64_t nonce, uint32_t bits);
  void state_digest(uint8_t out[32]) const;
  int kind() const { return kind_; }
 private:
  void absorb(const void* p, size_t n) {
    if (kind_ == SHA256) s_.update(p, n);
    else h_.update(p, n);
  }
  // squeeze_into (challenger.rs:288-303)
  void squeeze(uint8_t* out, size_t n) const;
  int kind_ = BLAKE3;
  b3::Hasher h_;
  sha::Hasher s_;
};
// pow_has_leading_zero_bits (challenger.rs:580-601)
bool pow_ok(const uint8_t digest[32], uint64_t nonce, uint32_t bits, int kind = BLAKE3);

// ---------------------------------------------------------------------------
// BLAKE3 compression R1CS.  crates/flock-prover/src/r1cs_hashes/blake3.rs
// ---------------------------------------------------------------------------
constexpr int K_LOG = 14;
constexpr int K = 1 << K_LOG;
constexpr int K_SKIP = 6;
constexpr int Z_CONST_POS = 512;
constexpr int USEFUL_BITS = 15409;

struct Compression { uint32_t cv[8]; uint32_t m[16]; uint64_t counter; uint32_t block_len; uint32_t flags; };

// benchmark-tools/common/src/lib.rs:25-37
std::vector<Compression> generate_compressions(uint32_t log2, uint64_t seed);

struct SparseRows { std::vector<uint32_t> ptr; std::vector<uint16_t> col; };  // CSR, K rows
namespace keccak { struct Layout; }
struct R1cs {
  int m = 0, n_log = 0;
  int k_log = K_LOG, z_const = Z_CONST_POS;  // block size and the pinned constant column
  bool walker = false;  // the lincheck marginal comes from the Keccak walker, not a0 / b0
  const keccak::Layout* keccak = nullptr;  // the walker's block layout
  SparseRows a0, b0;
  std::array<uint8_t, 32> digest{};
};
// crates/flock-core/src/r1cs.rs:334-385: BLAKE3 of the tag, m, k_log,
// k_skip, the row-major layout byte and the length-prefixed A_0, B_0, C_0 = I
std::array<uint8_t, 32> statement_digest(int m, int k_log, int k_skip, const SparseRows& a0, const SparseRows& b0);
const R1cs& blake3_r1cs(int n_log);   // cached per n_log; matrices shared
void build_matrices(SparseRows& a, SparseRows& b);
// packed witness: z, a, b each 2^(m-7) F128 (bit r of word i = bit 128 i + r)
void generate_witness(const std::vector<Compression>& blocks, int n_log,
                      std::vector<F128>& z, std::vector<F128>& a, std::vector<F128>& b);
// out = (I_n (x) M_0) z for blocks of m0's row count (2^k_log) bits
void apply_block_diag(const SparseRows& m0, const std::vector<F128>& z, int n_blocks,
                      std::vector<F128>& out);

// ---------------------------------------------------------------------------
// SHA-256 compression R1CS.  crates/flock-prover/src/r1cs_hashes/sha2.rs
// (one compression per 2^15-bit block, the I/O-aligned layout).
// ---------------------------------------------------------------------------
namespace sha {
constexpr int K_LOG_SHA = 15;
constexpr int K_SHA = 1 << K_LOG_SHA;
constexpr int Z_CONST_POS = 31400;
constexpr int USEFUL_BITS = 31401;
extern const uint32_t IV[8];   // FIPS 180-4 5.3.3
extern const uint32_t RC[64];  // FIPS 180-4 4.2.2
struct Compression { uint32_t h[8]; uint32_t m[16]; };
// sha256_compress (sha2.rs:1502-1546): H_out = H_in + rounds(H_in, M)
void compress(const uint32_t h[8], const uint32_t m[16], uint32_t out[8]);
// benches/sha2_proof.rs:56-71: one SplitMix64 stream from `seed`, h then m
std::vector<Compression> bench_inputs(size_t n, uint64_t seed);
// sha2.rs:1217-1221: log2 of the block slots for n compressions (>= 3)
int min_n_blocks_log(size_t n);
void build_matrices(SparseRows& a, SparseRows& b);
// the 2^15-bit boolean witness of one compression (sha2.rs:545-606), ORed
// into a zeroed 512-word block
void block_witness(const Compression& c, uint64_t* z);
}  // namespace sha
const R1cs& sha256_r1cs(int n_log);

// ---------------------------------------------------------------------------
// Keccak-f[1600] R1CS.  crates/flock-prover/src/r1cs_hashes/keccak.rs (one
// permutation per 2^16-bit block; implicit matrices and a lincheck walker).
// ---------------------------------------------------------------------------
namespace keccak {
constexpr int K_LOG_KECCAK = 16;
constexpr int K_KECCAK = 1 << K_LOG_KECCAK;
constexpr int Z_CONST = 4096;
constexpr int T_BASE = 4160;
constexpr int USEFUL_BITS = T_BASE + 24 * 1600;  // 42,560
// the 3-wide encoder (keccak3.rs:52-100)
constexpr int K_LOG_KECCAK3 = 17;
constexpr int Z_CONST3 = 12288;
constexpr int T_BASE3 = 12352;
// a block layout: n_sub permutations per 2^k_log-bit block
struct Layout { int k_log, n_sub, z_const, t_base; };
const Layout& single_layout();  // keccak.rs
const Layout& wide_layout();    // keccak3.rs
extern const uint64_t RC[24];
struct State { uint64_t lanes[25]; };  // lane x + 5y, bit z
// Keccak-f[1600] (FIPS 202) on lanes, in place
void permute(uint64_t lanes[25]);
// benches/keccak3_proof.rs:80-93: 25 SplitMix64 draws per state, bit i (index
// x + 5y + 25z) = bit i mod 64 of draw i / 64
std::vector<State> bench_inputs(size_t n, uint64_t seed);
// min_n_keccaks_log (keccak.rs:513-518) / min_n_blocks_log (keccak3.rs:144-150)
int min_n_blocks_log(const Layout& L, size_t n);
// one block's z, a, b (zeroed by the caller) from its L.n_sub input states
void block_witness(const Layout& L, const State* in, uint64_t* z, uint64_t* a, uint64_t* b);
// fold_alpha_batched: alpha A^T e + B^T e for e over the block's 2^k_log rows
std::vector<F128> lincheck_comb(const Layout& L, F128 alpha, const std::vector<F128>& e);
}  // namespace keccak
const R1cs& keccak_r1cs(const keccak::Layout& L, int n_log);
void generate_keccak_witness(const keccak::Layout& L, const std::vector<keccak::State>& states, int n_log,
                             std::vector<F128>& z, std::vector<F128>& a, std::vector<F128>& b);
// z by the boolean witness (padding blocks: the all-zero (h_in, m)
// compression), a = A_0 z and b = B_0 z from the matrices
void generate_sha256_witness(const std::vector<sha::Compression>& blocks, int n_log, std::vector<F128>& z,
                             std::vector<F128>& a, std::vector<F128>& b);

// ---------------------------------------------------------------------------
// Additive NTT over F128 (novel basis, neighbours-last) and GF(2^8) NTT.
// ntt/additive_ntt_f128.rs:54-141,2640-2800,4766-4800; ntt.rs:22-169
// ---------------------------------------------------------------------------
struct AdditiveNtt {
  int dim = 0;
  std::vector<std::vector<F128>> evals;
  std::vector<F128> twiddles;  // layer l at offset 2^l - 1
  explicit AdditiveNtt(int dim);
  F128 twiddle(int layer, size_t block) const { return twiddles[((size_t)1 << layer) - 1 + block]; }
  void forward_interleaved(std::vector<F128>& data, size_t num_ntts, int start_layer = 0) const;
};
const AdditiveNtt& standard_ntt(int dim);
// RS encode: msg (n positions x lanes) -> codeword (n * 2^rate positions x lanes)
void rs_encode(const std::vector<F128>& msg, size_t lanes, int log_inv_rate, std::vector<F128>& cw);

struct Gf8Ntt {
  int k; std::vector<uint8_t> tw;
  Gf8Ntt(int k, uint8_t beta);
  void forward(uint8_t* v) const;
  void inverse(uint8_t* v) const;
};

// ---------------------------------------------------------------------------
// Merkle (BLAKE3 leaf/parent CVs, flat 2n-1 layout).  merkle.rs:16-21,192-240,753-1072
// ---------------------------------------------------------------------------
// hash_leaf / hash_pair (merkle.rs:205-230): BLAKE3 non-root chaining
// values, or SHA256(leaf) and SHA256(left || right)
std::vector<Hash> merkle_tree(const uint8_t* data, size_t n_leaves, size_t leaf_size, int kind = BLAKE3);
std::vector<Hash> merkle_multi_proof(const std::vector<Hash>& tree, size_t n_leaves,
                                     std::vector<size_t> positions);

// ---------------------------------------------------------------------------
// Sub-protocol helpers
// ---------------------------------------------------------------------------
std::vector<F128> build_eq(const std::vector<F128>& r);       // index bit i <-> r[i]
std::vector<F128> lagrange_weights(int k_skip, F128 z, int node_base);
F128 interpolate_on_lambda(const std::vector<F128>& vals, F128 z);
F128 interpolate_combined(const std::vector<F128>& vals, F128 z);
std::array<F128, 3> small_challenges();
std::array<F128, 4> medium_challenges();
std::vector<F128> eval_sk_at_vks(int log_n);

// ---------------------------------------------------------------------------
// Proof structures (serde field order) and bincode-fixint serialization.
// crates/flock-prover/src/proof_io.rs:40-232
// ---------------------------------------------------------------------------
struct SumcheckMsg { F128 u0, u2; };
struct RecursiveProof { std::vector<std::vector<F128>> opened_rows; std::vector<Hash> merkle_proof; };
struct FinalProof { std::vector<F128> yr; std::vector<std::vector<F128>> opened_rows; std::vector<Hash> merkle_proof; };
struct LigeritoProof {
  Hash initial_root{};
  RecursiveProof initial_proof;
  std::vector<Hash> recursive_roots;
  std::vector<RecursiveProof> recursive_proofs;
  FinalProof final_proof;
  std::vector<SumcheckMsg> sumcheck_transcript;
  std::vector<uint64_t> grinding_nonces;
  std::vector<F128> ood_values;
  std::vector<uint64_t> fold_grinding_nonces;
};
struct ZerocheckProof {
  std::vector<F128> round1_ab, round1_c;
  std::vector<std::pair<F128, F128>> rounds;
  F128 final_a, final_b, final_c;
};
struct LincheckProof { std::vector<std::pair<F128, F128>> rounds; std::vector<F128> z_partial; };
struct Bundle {
  Hash root{};
  uint64_t m = 0, log_inv_rate = 1, log_batch_size = 6;
  uint32_t profile = 0, merkle_hash = 1;  // Fast, Blake3
  ZerocheckProof zc;
  LincheckProof lc;
  std::vector<std::vector<F128>> s_hat_v;  // one per ring-switched claim
  LigeritoProof lig;
};
std::vector<uint8_t> serialize(const Bundle& b);

struct LigeritoConfig {
  int initial_k = 6;
  std::vector<int> log_inv_rates, recursive_ks, queries, grinding_bits, fold_grinding_bits, ood_samples;
  int yr_log_n = 0;
};
const LigeritoConfig& ligerito_config(int m);

// ---------------------------------------------------------------------------
// Full prover.  crates/flock-prover/src/prover.rs:373-473 (generic path,
// byte-identical to Blake3Setup::prove_fast).
// ---------------------------------------------------------------------------
Bundle prove(const std::vector<Compression>& blocks, int n_log, const std::string& domain);

// A packed-MLE evaluation claim z_packed(point) = value, opened directly in
// the batched open beside the ring-switched claims (pcs.rs:57-95).
struct DirectClaim { std::vector<F128> point; F128 value; };
// Runs after the lincheck on the prover's transcript, with the packed z.
using CoreHook = std::function<std::vector<DirectClaim>(Challenger&, const std::vector<F128>&)>;
Bundle prove_with(const std::vector<Compression>& blocks, int n_log, const std::string& domain,
                  const CoreHook& after_core);
// the statement-independent prover (prover.rs:373-473 after the witness):
// commit z, zerocheck, lincheck, the batched open
Bundle prove_core(const R1cs& rc, std::vector<F128> z, const std::vector<F128>& a, const std::vector<F128>& b,
                  const std::string& domain, const CoreHook& after_core);
// Sha256HybridSetup::prove_fast (sha2.rs:1377-1408) over 2^n_log blocks
Bundle prove_sha256(const std::vector<sha::Compression>& blocks, int n_log, const std::string& domain);
// KeccakSetup::prove_fast (keccak.rs:956-978); padding: keccak_f(0)
Bundle prove_keccak(const keccak::Layout& L, const std::vector<keccak::State>& states, int n_log,
                    const std::string& domain);
// sum_j bc[j] * z[j] == target (the batched open's claim)
bool open_identity(const std::vector<F128>& z, const std::vector<F128>& bc, F128 target);
// that identity, as checked by the last prove_with with a hook on this thread
bool& last_open_identity_ok();

// Degree-4 zerocheck round 1 (zerocheck/univariate_skip_deg4.rs:77-165,
// round1_deg4_naive): five bit vectors of 2^m bits as 2^(m-6) u64 rows (bit s
// of row x is index 64 x + s), r of length m; p_abcd and p_z get the 192
// evaluations on Lambda4 = {64..255}.
void round1_deg4(const uint64_t* a, const uint64_t* b, const uint64_t* c, const uint64_t* d, const uint64_t* z,
                 int m, const std::vector<F128>& r, std::vector<F128>& p_abcd, std::vector<F128>& p_z);

// ---------------------------------------------------------------------------
// BLAKE3 hash chain.  crates/flock-prover/src/chain.rs (shift argument),
// r1cs_hashes/chain_common.rs (region fold, claim point, generic prover),
// r1cs_hashes/blake3.rs:5150-5240 (CHAIN_LAYOUT, prove_chain),
// bin/flock_chain.rs:178-193, 236-260 (the CLI's chain inputs).
// ---------------------------------------------------------------------------
struct ShiftProof { std::vector<std::pair<F128, F128>> rounds; F128 g_at_point; };
struct ChainClaims { std::vector<F128> instance_point; F128 sel0; F128 value; };
struct ChainBundle {
  Bundle core;
  ShiftProof shift;
  // the public endpoints in the region's physical bit order (one 0/1 byte per bit)
  std::vector<uint8_t> phys0, phys_last;
  uint32_t kind = 0;  // HashKind of the bundle (proof_io.rs:51-58): 0 Blake3, 1 Sha2, 2 Keccak
};
// out_lo of a compression: words 0..7 of the output state
void compress_cv(const Compression& c, uint32_t out[8]);
// the CLI's honest chain: cv_{i+1} = out_lo(compress(cv_i, m_i, 0, 64, 0)),
// m_i = 16 SplitMix64 draws (low 32 bits) from `seed`
std::vector<Compression> chain_blocks(uint64_t seed, const uint32_t initial_cv[8], size_t steps);
F128 shift_mle(const std::vector<F128>& a, const std::vector<F128>& b);
F128 eq_eval(const std::vector<F128>& a, const std::vector<F128>& b);
ShiftProof shift_prove(const std::vector<F128>& in, const std::vector<F128>& out, Challenger& ch,
                       ChainClaims& claims);
// false on a malformed proof or a failed final check
bool shift_verify(const ShiftProof& pf, F128 x0_r, F128 xlast_r, size_t n, Challenger& ch, ChainClaims& claims);
// tau_pos-MLE of a public 256-bit chaining value over its two packed positions
F128 fold_public_cv(const uint32_t cv[8], F128 tau_pos);
// prove_chain; when `check` is non-null it receives the prover-side checks:
// the shift argument verified from the public endpoints on a copy of the
// transcript, and the batched open's claim identity.  `claimed_cv_last`, when
// given, is the public output endpoint put in the bundle and checked against
// (by default the output of the last compression).
ChainBundle prove_chain(const std::vector<Compression>& blocks, int n_log, const std::string& domain,
                        bool* check = nullptr, const uint32_t* claimed_cv_last = nullptr);
std::vector<uint8_t> serialize_chain(const ChainBundle& cb);
// SHA-256 chains (sha2.rs:1557-1589): H_in of step i + 1 = sha256_compress of
// step i; the CLI's honest chain (bin/flock_chain.rs:279-316)
std::vector<sha::Compression> sha256_chain_blocks(uint64_t seed, const uint32_t initial[8], size_t steps);
ChainBundle prove_sha256_chain(const std::vector<sha::Compression>& blocks, int n_log, const std::string& domain,
                               bool* check = nullptr, const uint32_t* claimed_cv_last = nullptr);
// Keccak chains (KeccakSetup::prove_chain, keccak.rs:1000-1022, CHAIN_LAYOUT
// :839-846): state_0 of instance i + 1 = keccak_f(state_0 of instance i);
// 2048-bit slots, so tau_pos has 4 coordinates; endpoints state_to_phys_bits
// (:850-857).  claimed_last (25 lanes), when given, replaces the public end.
ChainBundle prove_keccak_chain(const std::vector<keccak::State>& states, int n_log, const std::string& domain,
                               bool* check = nullptr, const uint64_t* claimed_last = nullptr);

// ---------------------------------------------------------------------------
// SHA-256 Merkle paths.  crates/flock-prover/src/merkle_path.rs (shift
// sumcheck with a bit selector), r1cs_hashes/merkle_path_common.rs (slot
// folds, claim point, generic prover), r1cs_hashes/sha2.rs:1634-1845
// (MERKLE_LAYOUT, prove/verify_merkle_paths_ligerito).
// ---------------------------------------------------------------------------
struct MerkleShiftProof { std::vector<std::array<F128, 3>> rounds; F128 g_at_point; };
struct MerkleClaims { std::vector<F128> instance_point; F128 sel_slot, side, value; };
struct MerklePathInputs {
  std::vector<sha::Compression> blocks;   // path-id major, 2^n_log of them
  std::vector<uint8_t> b_bits;            // one per block
  std::vector<std::array<uint32_t, 8>> leaves;  // one per path
  std::array<uint32_t, 8> root{};
};
struct MerkleBundle { Bundle core; MerkleShiftProof shift; };
// slot vectors slot[0..4) (H_in, H_out, M_lo, M_hi), each 2^n values
MerkleShiftProof mp_shift_prove(int path_log, const std::vector<F128> slot[4], const std::vector<uint8_t>& b_bits,
                                Challenger& ch, MerkleClaims& claims);
bool mp_shift_verify(int path_log, const MerkleShiftProof& pf, const std::vector<F128>& leaf_evals, F128 root_r,
                     const std::vector<uint8_t>& b_bits, int n, Challenger& ch, MerkleClaims& claims);
// 2^path_log copies of one honest path of 2^(n_log - path_log) hashes
// (benches/sha2_merkle_proof.rs:49-76; sha2.rs:2475-2497)
MerklePathInputs sha256_merkle_paths(int n_log, int path_log, uint64_t seed);
// prove_merkle_paths_ligerito; `check` receives the shift argument verified
// from the public leaves and root on a copy of the transcript and the
// batched open's claim identity
MerkleBundle prove_sha256_merkle(const MerklePathInputs& in, int n_log, int path_log, const std::string& domain,
                                 bool* check = nullptr);
// bincode of (Commitment, MerklePathProofLigerito { zerocheck, lincheck,
// shift { rounds: Vec<RoundMsg { q_1, q_omega, q_omega_plus_1 }>,
// g_at_point }, pcs_open }) -- what the reference's own tests serialise
// (sha2.rs:2519-2526); there is no FLOCK header for this proof
std::vector<uint8_t> serialize_merkle(const MerkleBundle& mb);

}  // namespace flockref
