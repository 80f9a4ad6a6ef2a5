// One prover setup per (device, size): device buffers sized for 2^log2
// compressions, the statement (CSC matrices on the device), constant tables
// and the proof entry point.
#pragma once
#include <functional>
#include <string>
#include <vector>
#include "host.hpp"
#include "kernels.cuh"

namespace flock {

void scatter(f128* dst, const uint64_t* pos, const f128* vals, size_t n, cudaStream_t s);
class Setup;
// Fused witness + commit of several seeded proofs (one graph of batched
// launches on st); each setup's stream waits for it.  batch_commit waits for
// the commit; batch_commit_async only queues it and returns the resources to
// release (batch_commit_release) once st has finished.
struct BatchCommit {
  BatchJob* jobs = nullptr;  // device job table (stream-ordered on st)
  cudaStream_t st = nullptr;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t done = nullptr;
};
BatchCommit batch_commit_async(const std::vector<Setup*>& setups, const std::vector<uint64_t>& seeds,
                               cudaStream_t st);
void batch_commit_release(BatchCommit& h);
void batch_commit(const std::vector<Setup*>& setups, const std::vector<uint64_t>& seeds, cudaStream_t st);

// A Merkle-path proof over a SHA-256 setup (prove_merkle_paths_ligerito,
// r1cs_hashes/sha2.rs:1740-1783): 2^path_log paths of 2^(n_log - path_log)
// hashes each, path-id major; b_bits (host, one byte per slot) selects which
// half of each hash's message is the previous hash's output.
struct MerkleArgs {
  int path_log = 0;
  const uint8_t* b_bits = nullptr;
};
// Its public inputs on the verifier side: the leaf of every path and the
// shared root (8 u32 each) and the bit vector.
struct MerklePublic {
  int path_log = 0;
  std::vector<uint8_t> b_bits;
  std::vector<std::array<uint32_t, 8>> leaves;
  std::array<uint32_t, 8> root{};
};

// Public endpoints of a hash chain: the input cv of the first compression and
// the output cv (out_lo) of the last.
// a chain's public endpoints in the region's physical bit order (bit i = bit
// i % 64 of word i / 64; a 256-bit cv is its 8 u32 words little endian)
struct ChainEnds {
  uint64_t in[32] = {}, out[32] = {};
};

// What the verifier needs of a statement: its size, digest, and the
// lincheck's matrix combination alpha A^T eq + B^T eq (+ beta at the constant
// column) for eq = L(z_skip) (x) eq(x_inner) (lincheck.rs:5940-5960).
struct VerifyStatement {
  int m = 0, k_log = kKLog;
  int hash = kHashBlake3;                // the statement (a chain bundle names it)
  int fs_fn = kFnBlake3;                 // the transcript's hash
  const MerklePublic* merkle = nullptr;  // a Merkle-path proof's public inputs
  std::array<uint8_t, 32> digest{};
  std::function<std::vector<f128>(f128 z_skip, const std::vector<f128>& x_inner, f128 alpha, f128 beta)> comb;
  // optional: BLAKE3 leaf chaining values of rows packed back to back, group
  // k holding counts[k] rows of sizes[k] bytes; empty result = hash on the host
  std::function<std::vector<H32>(const uint8_t* data, const std::vector<size_t>& sizes,
                                 const std::vector<size_t>& counts, int merkle_fn)>
      leaf_cvs;
};
// "" when the bundle verifies, otherwise the name of the failed check
std::string verify_bundle(const uint8_t* bytes, size_t len, const std::string& domain, const VerifyStatement& V);

// A verifier with its own device scratch (about 2 MiB) and stream, for any
// statement size; the block matrices' device copy is shared per device.  One
// thread at a time per Verifier.
class Verifier {
 public:
  explicit Verifier(int device);
  ~Verifier();
  Verifier(const Verifier&) = delete;
  Verifier& operator=(const Verifier&) = delete;
  // "" when the bundle verifies, otherwise the name of the failed check;
  // hash: the statement the bundle is for (the R1CS bundle does not say)
  // fs_fn: the transcript's hash (the bundle does not say; its Merkle hash
  // it does)
  std::string verify(const uint8_t* bytes, size_t len, const std::string& domain, int hash = kHashBlake3,
                     const MerklePublic* merkle = nullptr, int fs_fn = kFnBlake3);

 private:
  static constexpr size_t kRowsCap = (size_t)1 << 20, kCvsCap = (size_t)1 << 19;
  int device_ = 0;
  cudaStream_t st_ = nullptr;
  f128 *eqx_ = nullptr, *eqi_ = nullptr, *comb_ = nullptr, *kcw_ = nullptr;
  uint8_t* rows_ = nullptr;
  uint32_t* cvs_ = nullptr;
};

struct Level {
  int lanes = 0, log_msg_pos = 0, rate = 0;
  size_t positions = 0;
  f128* cw = nullptr;
  uint32_t* tree = nullptr;
};

class Setup {
 public:
  static constexpr int kPhases = 9;  // witness, RS encode, Merkle commit, round1, zc rounds, lincheck,
                                     // ring switch, L0 folds, levels
  // stream_priority: the CUDA priority of the setup's stream (0: default;
  // lower numbers are served first when streams compete for the SMs).
  // hash: the statement (kHashBlake3: 2^log2 BLAKE3 compressions in 2^14-bit
  // blocks; kHashSha256: SHA-256 compressions in 2^15-bit blocks).
  // merkle_fn: the hash of the PCS Merkle trees (PcsParams::merkle_hash;
  // kFnBlake3, the benchmark's, or kFnSha256, the reference's default)
  Setup(int device, uint32_t log2, int stream_priority = 0, int hash = kHashBlake3, int merkle_fn = kFnBlake3);
  ~Setup();
  Setup(const Setup&) = delete;
  Setup& operator=(const Setup&) = delete;

  // seed != nullptr: inputs generated on the device from the benchmark
  // generator; otherwise blocks_dev holds n_blocks x 25 u32 on the device.
  // committed: the witness, codeword and tree were filled by batch_commit.
  // chain != nullptr: a hash-chain proof (Blake3Setup::prove_chain,
  // blake3.rs:5195-5215) whose bundle carries these endpoints; blocks_dev
  // then holds 2^log2 records of 28 u32 (cv, m, counter u64, block_len, flags).
  // full_records: blocks_dev holds n_blocks such 28-u32 records for a
  // compression proof; the slots from n_blocks on hold the all-zero
  // compression, as in the reference's padded prove_fast.
  // A SHA-256 setup takes records of 24 u32 (h_in, m) in blocks_dev, or the
  // benchmark generator's seed; its padding slots hold the compression of
  // the all-zero (h_in, m) (Sha256HybridSetup::prove_fast, sha2.rs:1185-1209).
  std::vector<uint8_t> prove(const uint64_t* seed, const uint32_t* blocks_dev, size_t n_blocks,
                             const std::string& domain, bool committed = false, const ChainEnds* chain = nullptr,
                             bool full_records = false, const MerkleArgs* merkle = nullptr);
  // Replays and checks a FLOCK v4 bundle of this statement size (compression
  // or hash chain; a chain's public endpoints are the bundle's); "" when it
  // verifies, otherwise the name of the failed check.  Uses this setup's
  // device statement and stream.
  std::string verify(const uint8_t* bytes, size_t len, const std::string& domain,
                     const MerklePublic* merkle = nullptr);
  void phase_times(double* ms) const;
  // device bytes a setup for 2^log2 compressions holds (an upper estimate,
  // used for admission before allocating)
  static size_t estimate_bytes(uint32_t log2, int hash = kHashBlake3);
  size_t device_bytes = 0;  // allocated by the constructor

  friend BatchCommit batch_commit_async(const std::vector<Setup*>& setups, const std::vector<uint64_t>& seeds,
                                        cudaStream_t st);
  uint32_t log2 = 0;
  int hash = kHashBlake3, k_log = kKLog;
  int merkle_fn = kFnBlake3;
  // the Fiat-Shamir transcript's hash (FsChallenger::with_hash); settable
  // between proofs
  int fs_fn = kFnBlake3;
  int n_log = 0, m = 0, sms = 0;
  // SMs the grid-stride kernels of this setup spread over (0: all).  The
  // serving queue lowers it for large proofs so that their long persistent
  // kernels leave some SMs to small proofs' kernels.
  int grid_sms = 0;
  size_t n_words = 0, n_leaves0 = 0;
  cudaStream_t st = nullptr;
  uint32_t* blocks_buf = nullptr;  // device staging for caller-provided compressions
  uint32_t* records_buf = nullptr;  // device staging for a hash chain's compression records

 private:
  void build_round1_tables();
  void eq_table(const std::vector<f128>& r, f128* dev);
  void fetch(const f128* dev, size_t n, f128* host);
  uint64_t grind(Transcript& tr, uint32_t bits);
  std::vector<size_t> sample_queries(Transcript& tr, size_t block_len, size_t count);
  // queues the opening's gathers and its copy into the pinned staging area;
  // `o` is filled by finish_openings once the stream has finished
  void open(Opening& o, const f128* cw, const uint32_t* tree, size_t n_leaves, int lanes, const std::vector<size_t>& q);
  void finish_openings();
  struct PendingOpen {
    Opening* o;
    size_t off, nq, lanes, ns;
  };
  static constexpr size_t kStageBytes = (size_t)1 << 21;
  std::vector<PendingOpen> pending_;
  size_t stage_off_ = 0;
  H32 root_of(const uint32_t* tree, size_t n_leaves);
  void mark(int phase);
  f128* scratch_eq() { return eqbuf[0]; }

  uint8_t lde_m[64][64] = {};  // GF(2^8) extension S -> Lambda (Lagrange basis)
  const Ladder* lad = nullptr;
  std::array<uint8_t, 32> digest{};
  f128 *z = nullptr, *a = nullptr, *b = nullptr, *cw0 = nullptr;
  uint32_t* tree0 = nullptr;
  f128* pp[4] = {nullptr, nullptr, nullptr, nullptr};
  f128* eqbuf[2] = {nullptr, nullptr};
  std::vector<Level> levels;
  f128 *induce_buf = nullptr, *out = nullptr, *lag = nullptr, *elo = nullptr, *ehi = nullptr;
  f128 *comb = nullptr, *zv = nullptr, *zv_pre = nullptr, *eq_inner = nullptr, *bc_tabs = nullptr, *gather = nullptr;
  std::vector<f128> s_hat_v_c;  // c-claim ring-switch statistic, captured by zerocheck round 1
  uint8_t* tabs_r1 = nullptr;
  uint64_t* idx = nullptr;
  unsigned long long* d_found = nullptr;
  unsigned long long* h_found = nullptr;
  f128* h_out = nullptr;
  uint8_t* h_stage = nullptr;
  uint32_t *at_ptr = nullptr, *bt_ptr = nullptr;
  uint16_t *at_row = nullptr, *bt_row = nullptr;
  f128* kc_w = nullptr;                // Keccak statement: the walker's W rows
  const uint64_t* kc_masks = nullptr;  // Keccak statement: round-constant masks (per device)
  cudaEvent_t ev[kPhases + 1] = {};
  // The commitment's RS encode (z -> cw0) and Merkle tree (cw0 -> tree0) on
  // fixed buffers, each captured once as a CUDA graph (after the NTT plans
  // are tuned) and replayed by every proof.
  cudaGraphExec_t commit_graph[2] = {nullptr, nullptr};
  uint64_t commit_launches[2] = {0, 0};
  void tune_ntt_plans();
  void capture_commit();
};

}  // namespace flock
