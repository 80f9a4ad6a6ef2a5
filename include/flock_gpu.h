/* C ABI of the B200 Flock prover (libflockgpu.so).
 *
 * The library is the drop-in replacement for the reference's proving entry
 * point; a Rust (or any FFI) host binds these symbols.  All functions return
 * 0 on success and a nonzero status otherwise (never unwind across the ABI);
 * flock_last_error() describes the last failure of a context.  Output buffers
 * are caller-owned.  One context per device; a setup is used by one thread at
 * a time.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *  - flock_setup_create  <- Blake3Setup::new(n_blocks) + pcs_params.merkle_hash
 *                           = Blake3 (crates/flock-prover/src/r1cs_hashes/
 *                           blake3.rs:4706-4780, benchmark-tools/worker/src/
 *                           main.rs:24-25)
 *  - flock_prove_seed    <- generate_compressions(log2, seed) + prove_fast +
 *                           R1csProofBundleLigerito::to_bytes
 *                           (benchmark-tools/worker/src/main.rs:42-47,
 *                           blake3.rs:4846, proof_io.rs:165)
 *  - flock_prove_blocks  <- Blake3Setup::prove_fast(&blocks, &mut FsChallenger)
 *                           + to_bytes (blake3.rs:4846-4990)
 *  - flock_pcs_commit, flock_prover_data_*
 *                        <- pcs::commit -> (Commitment, ProverData) and the
 *                           openings read from it (crates/flock-core/src/pcs/
 *                           commit.rs:143-230, merkle.rs:1020-1072)
 *  - flock_challenger_*  <- FsChallenger and the Challenger trait
 *                           (crates/flock-core/src/challenger.rs:34-100,
 *                           170-600)
 *  - flock_setup_create_blocks, flock_prove_compressions
 *                        <- Blake3Setup::new(n_blocks) (any n) + prove_fast
 *                           over full Compression tuples (blake3.rs:1854-1861,
 *                           4706, 4846)
 *  - flock_prove_chain   <- Blake3Setup::prove_chain(&blocks, &mut FsChallenger)
 *                           + ChainProofBundleLigerito::to_bytes (blake3.rs:
 *                           5195-5215, r1cs_hashes/chain_common.rs:287-350,
 *                           proof_io.rs:144-157, 943-950)
 *  - flock_verify, flock_verify_bundle
 *                        <- Blake3Setup::verify / verify_chain on a decoded
 *                           bundle (blake3.rs:5129-5145, 5217-5240;
 *                           crates/flock-core/src/verifier.rs:95-232)
 *  - flock_chain_blocks  <- the flock_chain CLI's honest BLAKE3 chain
 *                           (crates/flock-prover/src/bin/flock_chain.rs:178-193,
 *                           236-260)
 *  - flock_ntt_rs_encode <- AdditiveNttF128::standard(d) + rs_encode_interleaved
 *                           (crates/flock-core/src/ntt/additive_ntt_f128.rs:
 *                           2661-2670, 2785)
 *  - flock_merkle_tree   <- merkle::merkle_tree (crates/flock-core/src/merkle.rs:753)
 *  - flock_sumcheck_round<- ligerito round_msg_lsb (crates/flock-core/src/pcs/
 *                           ligerito.rs:4958) and zerocheck round_pair_naive
 *                           (zerocheck/multilinear.rs:616)
 *  - flock_witness       <- generate_witness_with_ab_packed_and_lincheck
 *                           (blake3.rs:4617) for the inputs of
 *                           generate_compressions (benchmark-tools/common/src/lib.rs:25)
 *  - flock_pow           <- FsChallenger::grind_pow (crates/flock-core/src/challenger.rs:384)
 *  - flock_f128_mul      <- F128 * F128 (crates/flock-core/src/field/gf2_128.rs:140-165)
 *  - flock_keccak_*      <- KeccakSetup::{new, prove_fast, verify}, keccak_f
 *                           (crates/flock-prover/src/r1cs_hashes/keccak.rs:
 *                           423-428, 863-998)
 *  - flock_keccak3_*     <- keccak3::KeccakSetup (crates/flock-prover/src/
 *                           r1cs_hashes/keccak3.rs:491-580)
 *  - flock_zerocheck_round1_deg4
 *                        <- round1_deg4_naive (crates/flock-core/src/zerocheck/
 *                           univariate_skip_deg4.rs:77-165)
 */
#ifndef FLOCK_GPU_H
#define FLOCK_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct flock_ctx flock_ctx;
typedef struct flock_setup flock_setup;

enum {
  FLOCK_OK = 0,
  FLOCK_ERR_ARG = 1,
  FLOCK_ERR_CUDA = 2,
  FLOCK_ERR_CAPACITY = 3,
  FLOCK_ERR_INTERNAL = 4,
  FLOCK_ERR_TIMEOUT = 5,
  FLOCK_ERR_VERIFY = 6
};
/* The hash behind the PCS Merkle trees and the Fiat-Shamir transcript
 * (HashKind, crates/flock-core/src/hash.rs:20-30, with its serde
 * discriminants).  SHA-256 is the reference's default (FsChallenger::new,
 * PcsParams::default); the benchmark uses BLAKE3 for both
 * (benchmark-tools/worker/src/main.rs:23-29). */
enum { FLOCK_HASH_SHA256 = 0, FLOCK_HASH_BLAKE3 = 1 };
enum { FLOCK_PROFILE_FAST = 0 };

int flock_ctx_create(int device, uint64_t hbm_budget_bytes, flock_ctx** out);
void flock_ctx_destroy(flock_ctx* ctx);
const char* flock_last_error(flock_ctx* ctx);

/* One BLAKE3 compression input, the reference's Compression tuple
 * ([u32; 8], [u32; 16], u64, u32, u32) = (cv, m, counter, block_len, flags)
 * (crates/flock-prover/src/r1cs_hashes/blake3.rs:1861) as a C struct of 28
 * u32 (112 bytes; the counter little endian). */
typedef struct flock_compression {
  uint32_t cv[8];
  uint32_t m[16];
  uint64_t counter;
  uint32_t block_len;
  uint32_t flags;
} flock_compression;

/* Untimed setup for 2^log2_n compressions (8 <= log2_n <= 20).  hash: the
 * PCS Merkle hash (pcs_params.merkle_hash; the commitment records it).  The
 * setup's transcript hash is BLAKE3 until flock_setup_set_transcript. */
int flock_setup_create(flock_ctx* ctx, uint32_t log2_n, int hash, int profile, flock_setup** out);
/* Untimed setup for n_blocks compressions, any count (Blake3Setup::new(n_blocks),
 * blake3.rs:4706-4780): the statement has 2^max(3, ceil(log2 n_blocks)) slots
 * (min_n_blocks_log, blake3.rs:1854-1858).  Supported: 129 <= n_blocks <= 2^20
 * (the fast profile's Ligerito ladders cover m = 22..34; the reference panics
 * below that, FLOCK_ERR_ARG here). */
int flock_setup_create_blocks(flock_ctx* ctx, size_t n_blocks, int hash, int profile, flock_setup** out);
void flock_setup_destroy(flock_setup* s);
/* The transcript of this setup's proofs and of flock_verify on it:
 * FsChallenger::with_hash(domain, hash) (challenger.rs:227-250; SHA-256:
 * squeezes SHA256(state || ctr), PoW SHA256(digest || nonce)). */
int flock_setup_set_transcript(flock_setup* s, int hash);
/* The transcript hash of the context's verify-bundle entry points (the
 * bundle records its Merkle hash but not its transcript's). */
int flock_ctx_set_transcript(flock_ctx* ctx, int hash);

/* One proof; inputs generated on the GPU from `seed` exactly as the
 * benchmark generator does.  Writes the FLOCK v4 bundle bytes. */
int flock_prove_seed(flock_setup* s, uint64_t seed, const uint8_t* domain, size_t dlen, uint8_t* out, size_t cap,
                     size_t* out_len);
/* One proof over caller compressions: n x 25 u32 (cv[8], m[16], counter),
 * block_len 64, flags 11, n == 2^log2_n. */
int flock_prove_blocks(flock_setup* s, const uint32_t* blocks, size_t n, const uint8_t* domain, size_t dlen,
                       uint8_t* out, size_t cap, size_t* out_len);
/* One proof over caller compressions with every field free (u64 counter,
 * block_len, flags): Blake3Setup::prove_fast(&blocks, &mut FsChallenger) +
 * to_bytes (blake3.rs:4846-4990).  n must equal the setup's n_blocks
 * (2^log2_n for flock_setup_create), as prove_fast asserts; the slots from n
 * on hold the all-zero compression, the reference's padding
 * (blake3.rs:2527, seed_pipe.rs:210-226). */
int flock_prove_compressions(flock_setup* s, const flock_compression* blocks, size_t n, const uint8_t* domain,
                             size_t dlen, uint8_t* out, size_t cap, size_t* out_len);
/* One hash-chain proof: the 2^log2_n compressions form a chain
 * x_{i+1} = out_lo(compress(x_i)) with public endpoints.  records: n x 28
 * u32, each cv[8], m[16], counter (u64, little endian), block_len, flags
 * (Compression, blake3.rs:1861); n == 2^log2_n (a chain fills every slot).
 * The bundle (FLOCK v4, flavor 3) carries the endpoints records[0].cv and
 * out_lo(compress(records[n - 1])).  The prover does not check the links: a
 * broken chain gives a proof that the reference's verify_chain rejects. */
int flock_prove_chain(flock_setup* s, const uint32_t* records, size_t n, const uint8_t* domain, size_t dlen,
                      uint8_t* out, size_t cap, size_t* out_len);
/* The PCS layer: pcs::commit (crates/flock-core/src/pcs/commit.rs:187-230)
 * under PcsParams {m, log_inv_rate 1, log_batch_size 6, Fast, Blake3}.  The
 * packed polynomial z_packed (2^(m-7) F128 as {lo, hi} u64 pairs, host
 * memory; 22 <= m <= 34) is RS-encoded as 64 interleaved lanes at rate 1/2
 * and Merkle-hashed over its 2^(m-12) positions (1 KiB leaves, BLAKE3).
 * Writes Commitment.root; the handle holds the ProverData (codeword and
 * tree, commit.rs:143-185) on the context's device until it is destroyed. */
typedef struct flock_prover_data flock_prover_data;
int flock_pcs_commit(flock_ctx* ctx, const uint64_t* z_packed, uint32_t m, uint8_t* root32, flock_prover_data** out);
/* The opening of sorted distinct positions that the Ligerito prover reads
 * from ProverData (ligerito.rs:9721 merkle_multi_proof_for): their rows
 * (n x 64 F128 into rows_out) and the Merkle multi-proof's sibling hashes
 * (merkle.rs:1020-1072; *proof_count of 32 bytes into proof_out, or
 * FLOCK_ERR_CAPACITY with *proof_count set when proof_cap is too small). */
int flock_prover_data_open(flock_prover_data* pd, const uint64_t* positions, size_t n, uint64_t* rows_out,
                           uint8_t* proof_out, size_t proof_cap, size_t* proof_count);
void flock_prover_data_destroy(flock_prover_data* pd);

/* The transcript layer: FsChallenger::with_hash(domain, Blake3) and the
 * Challenger trait (crates/flock-core/src/challenger.rs:34-100, 170-600).
 * observe_f128 absorbs one value and observe_f128_slice a framed slice;
 * sample_f128 / sample_f128_vec squeeze one value / a framed vector
 * ({lo, hi} u64 pairs).  grind_pow finds the smallest nonce whose BLAKE3
 * hash of (state digest || nonce LE || 0^24) has `bits` leading zero bits and
 * absorbs it (grind_pow, challenger.rs:384-475): on the context's GPU, or on
 * the calling thread for at most 6 bits (ctx may then be NULL);
 * verify_pow checks a nonce and absorbs it (FLOCK_ERR_VERIFY when it fails,
 * challenger.rs:502-545).  A challenger is used by one thread at a time. */
typedef struct flock_challenger flock_challenger;
int flock_challenger_create(const uint8_t* domain, size_t dlen, flock_challenger** out);
/* FsChallenger::with_hash(domain, hash); flock_challenger_create is BLAKE3. */
int flock_challenger_create_hash(const uint8_t* domain, size_t dlen, int hash, flock_challenger** out);
void flock_challenger_destroy(flock_challenger* ch);
int flock_challenger_observe_label(flock_challenger* ch, const uint8_t* label, size_t len);
int flock_challenger_observe_bytes(flock_challenger* ch, const uint8_t* bytes, size_t len);
int flock_challenger_observe_f128(flock_challenger* ch, const uint64_t* value);
int flock_challenger_observe_f128_slice(flock_challenger* ch, const uint64_t* values, size_t n);
int flock_challenger_sample_f128(flock_challenger* ch, uint64_t* out);
int flock_challenger_sample_f128_vec(flock_challenger* ch, size_t n, uint64_t* out);
int flock_challenger_grind_pow(flock_challenger* ch, flock_ctx* ctx, uint32_t bits, uint64_t* nonce);
int flock_challenger_verify_pow(flock_challenger* ch, uint64_t nonce, uint32_t bits);
int flock_challenger_state_digest(flock_challenger* ch, uint8_t* out32);

/* ---- SHA-256 compressions (crates/flock-prover/src/r1cs_hashes/sha2.rs) ----
 * The same prover (witness -> RS encode + Merkle commit -> zerocheck ->
 * lincheck -> ring switch -> Ligerito) over the hybrid SHA-256 R1CS: one
 * compression per 2^15-bit block (H_in, H_out, M, Ch/Maj AND rows, carry
 * rows of every 32-bit ADD, materialised W[16..63], T1, E_NEW, A_NEW), the
 * constant wire at bit 31400 pinned to 1 in every block. */
/* One input, the reference's ([u32; 8], [u32; 16]) = (h_in, m) (sha2.rs:1377). */
typedef struct flock_sha256_compression {
  uint32_t h[8];
  uint32_t m[16];
} flock_sha256_compression;
/* Sha256HybridSetup::new(n_compressions) (sha2.rs:1252-1330): the statement
 * has 2^max(3, ceil(log2 n)) slots (min_n_blocks_log, sha2.rs:1217-1221).
 * Supported: 65 <= n <= 2^19 (m = 15 + n_log in 22..34, the fast profile's
 * Ligerito ladders).  hash / profile as for flock_setup_create.  The setup
 * also serves flock_prove_seed (the sha2_proof bench generator:
 * benches/sha2_proof.rs:56-71, one SplitMix64 stream from the seed, h then m
 * per compression, n_compressions of them) and flock_verify. */
int flock_sha256_setup_create(flock_ctx* ctx, size_t n_compressions, int hash, int profile, flock_setup** out);
/* Sha256HybridSetup::prove_fast(&compressions, &mut FsChallenger) + to_bytes
 * (sha2.rs:1377-1408): n must equal the setup's n_compressions; the slots
 * from n on hold the compression of the all-zero (h_in, m) (sha2.rs:1195). */
int flock_sha256_prove(flock_setup* s, const flock_sha256_compression* comps, size_t n, const uint8_t* domain,
                       size_t dlen, uint8_t* out, size_t cap, size_t* out_len);
/* Sha256HybridSetup::verify (sha2.rs:1441-1486) without a prover setup, for
 * any supported size (read from the bundle); the context's verifier, as in
 * flock_verify_bundle.  The R1CS bundle does not name its hash, so the
 * statement is chosen by the entry point. */
int flock_sha256_verify_bundle(flock_ctx* ctx, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen);
/* Sha256HybridSetup::prove_chain (sha2.rs:1557-1589) + ChainProofBundleLigerito
 * (hash_kind Sha2) bytes: the n compressions (n = the setup's
 * n_compressions, a power of two: a chain fills every slot) form a chain
 * h_in[i + 1] = sha256_compress(h_in[i], m[i]); the public endpoints are
 * h_in[0] and the last output, the CHAIN_LAYOUT of sha2.rs:1476-1483 (H_in at
 * byte 0, H_out at byte 32, the BLAKE3 chain's slots).  Verified by
 * flock_verify on the setup or flock_sha256_verify_bundle. */
int flock_sha256_prove_chain(flock_setup* s, const flock_sha256_compression* comps, size_t n, const uint8_t* domain,
                             size_t dlen, uint8_t* out, size_t cap, size_t* out_len);
/* The flock_chain CLI's honest SHA-256 chain of `steps` compressions
 * (bin/flock_chain.rs:279-316): h_0 = initial_h or the SHA-256 IV, m_i = 16
 * SplitMix64(seed) draws (low 32 bits), h_(i+1) = sha256_compress(h_i, m_i). */
int flock_sha256_chain_blocks(uint64_t seed, const uint32_t* initial_h, size_t steps, flock_sha256_compression* out);
/* Merkle paths over SHA-256 compressions: Sha256HybridSetup::
 * prove_merkle_paths_ligerito (sha2.rs:1740-1783; path_log = 0 is
 * prove_merkle_path_ligerito, :1662-1697).  2^path_log paths of
 * 2^(n_log - path_log) hashes each fill the setup's n = 2^n_log slots, path-id
 * major; b_bits[i] (one byte each) says which half of hash i's message is the
 * previous hash's output (the first hash of every path takes its leaf in the
 * left half whatever its bit).  The setup must hold a power of two.  Output:
 * bincode of (Commitment, MerklePathProofLigerito) -- the reference has no
 * FLOCK bundle type for this proof; its tests serialise the two this way
 * (sha2.rs:2519-2526). */
int flock_sha256_merkle_prove(flock_setup* s, const flock_sha256_compression* comps, size_t n, const uint8_t* b_bits,
                              uint32_t path_log, const uint8_t* domain, size_t dlen, uint8_t* out, size_t cap,
                              size_t* out_len);
/* verify_merkle_paths_ligerito (sha2.rs:1785-1843): the public leaves (8 u32
 * per path), the shared root and the n bits. */
int flock_sha256_merkle_verify(flock_ctx* ctx, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen,
                               uint32_t path_log, const uint8_t* b_bits, size_t n, const uint32_t* leaves,
                               const uint32_t* root);
/* Honest inputs (host): the path of benches/sha2_merkle_proof.rs:49-76
 * (every H_in the SHA-256 IV; leaf, bits and siblings from one SplitMix64
 * stream, low 32 bits) of 2^(n_log - path_log) hashes, repeated for each of
 * the 2^path_log paths (sha2.rs:2475-2497).  comps: 2^n_log, b_bits: 2^n_log,
 * leaves: 8 u32 per path, root: 8 u32. */
int flock_sha256_merkle_inputs(uint32_t n_log, uint32_t path_log, uint64_t seed, flock_sha256_compression* comps,
                               uint8_t* b_bits, uint32_t* leaves, uint32_t* root);
/* sha256_compress (sha2.rs:1502-1546) on the host: out = h_in + rounds(h_in, m). */
void flock_sha256_compress(const uint32_t* h_in, const uint32_t* m, uint32_t* out);
/* BlockR1cs::statement_digest of the SHA-256 statement of size m. */
int flock_sha256_statement_digest(uint32_t m, uint8_t* out32);
/* Debug/test: the packed row witness z, a = A_0 z, b = B_0 z of n
 * compressions over 2^n_log blocks (2^(n_log + 8) u64 pairs each). */
int flock_sha256_witness(flock_ctx* ctx, const flock_sha256_compression* comps, size_t n, uint32_t n_log, uint64_t* z,
                         uint64_t* a, uint64_t* b);

/* ---- Keccak-f[1600] permutations (crates/flock-prover/src/r1cs_hashes/keccak.rs) ----
 * The same prover over the monolithic Keccak R1CS at K_LOG = 16
 * (keccak.rs:430-660): one permutation per 2^16-bit block holding state_0,
 * state_24, the constant wire (bit 4096) and the 24 x 1600 chi AND rows t_r.
 * The block matrices are implicit (the statement digest binds the empty stub
 * of common.rs:120-138); the lincheck applies them by the transposed
 * recurrence of KeccakLincheckCircuit (keccak.rs:681-848) on the GPU. */
/* One input: the reference's State = [bool; 1600] (keccak.rs:124), as 25
 * lanes: bit z of lanes[x + 5y] is state bit x + 5y + 25z. */
typedef struct flock_keccak_state {
  uint64_t lanes[25];
} flock_keccak_state;
/* KeccakSetup::new(n_keccaks) (keccak.rs:870-912): 2^max(3, ceil(log2 n))
 * slots (min_n_keccaks_log, keccak.rs:513-518).  Supported: 33 <= n <= 2^18
 * (m = 16 + n_log in 22..34, the fast profile's Ligerito ladders).  hash /
 * profile as for flock_setup_create (the reference's default Merkle hash is
 * SHA-256).  The setup also serves flock_prove_seed (the keccak3_proof bench
 * generator: benches/keccak3_proof.rs:66-93, one SplitMix64 stream from the
 * seed, 25 draws per state) and flock_verify. */
int flock_keccak_setup_create(flock_ctx* ctx, size_t n_keccaks, int hash, int profile, flock_setup** out);
/* KeccakSetup::prove_fast(&states, &mut FsChallenger) + to_bytes
 * (keccak.rs:956-978): n must equal the setup's n_keccaks; the slots from n on
 * hold keccak_f of the zero state (keccak.rs:646-660). */
int flock_keccak_prove(flock_setup* s, const flock_keccak_state* states, size_t n, const uint8_t* domain, size_t dlen,
                       uint8_t* out, size_t cap, size_t* out_len);
/* KeccakSetup::verify (keccak.rs:979-998) without a prover setup, for any
 * supported size (read from the bundle); the context's verifier, as in
 * flock_verify_bundle. */
int flock_keccak_verify_bundle(flock_ctx* ctx, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen);
/* keccak_f (keccak.rs:423-428; FIPS 202 Keccak-f[1600]) on the host, in place. */
void flock_keccak_f(uint64_t* lanes25);
/* The keccak3_proof bench's states (benches/keccak3_proof.rs:66-93) on the host. */
int flock_keccak_bench_inputs(size_t n, uint64_t seed, flock_keccak_state* out);
/* BlockR1cs::statement_digest of the Keccak statement of size m. */
int flock_keccak_statement_digest(uint32_t m, uint8_t* out32);
/* Debug/test: the packed row witness z, a, b of n permutations over 2^n_log
 * blocks (2^(n_log + 9) u64 pairs each). */
int flock_keccak_witness(flock_ctx* ctx, const flock_keccak_state* states, size_t n, uint32_t n_log, uint64_t* z,
                         uint64_t* a, uint64_t* b);
/* Debug/test: the lincheck's column combination alpha A^T e + B^T e + beta
 * [const] over the 2^16 rows of a block, on the GPU (e, comb: 2^16 F128 as
 * lo, hi u64 pairs; alpha, beta: one F128). */
int flock_keccak_comb(flock_ctx* ctx, const uint64_t* e, const uint64_t* alpha, const uint64_t* beta, uint64_t* comb);
/* KeccakSetup::prove_chain (keccak.rs:1000-1022) + ChainProofBundleLigerito
 * (hash_kind Keccak) bytes: the n states (n = the setup's n_keccaks, a power
 * of two: a chain fills every slot) form a chain state[i + 1] =
 * keccak_f(state[i]); the public endpoints are state[0] and keccak_f of the
 * last, 1600 bits each in the slot's physical order (state_to_phys_bits,
 * :850-857).  The chain geometry is CHAIN_LAYOUT (:839-846): state_0 and
 * state_24 in 2048-bit slots.  Verified by flock_verify on the setup or
 * flock_keccak_verify_bundle. */
int flock_keccak_prove_chain(flock_setup* s, const flock_keccak_state* states, size_t n, const uint8_t* domain,
                             size_t dlen, uint8_t* out, size_t cap, size_t* out_len);
/* The flock_chain CLI's Keccak chain (bin/flock_chain.rs:319-346): `steps`
 * successive states from `initial` (25 lanes; NULL: the zero state). */
int flock_keccak_chain_states(const uint64_t* initial, size_t steps, flock_keccak_state* out);
/* The 3-wide encoder (crates/flock-prover/src/r1cs_hashes/keccak3.rs): three
 * independent permutations per 2^17-bit block (sub-keccak i: state_0 in slot
 * 2i, state_24 in slot 2i + 1, t[i, r] tight from bit 12352 in the order
 * i * 24 + r; one shared constant wire at bit 12288).
 * keccak3::KeccakSetup::new(n_keccaks) (keccak3.rs:498-540): 2^max(3, ceil(
 * log2 ceil(n / 3))) blocks (min_n_blocks_log, :144-150); supported 49 <= n
 * <= 3 * 2^17 (m = 17 + n_log in 22..34).  Proofs through flock_keccak_prove
 * (n = the setup's n_keccaks; missing permutations of the last block and
 * padding blocks are keccak_f of the zero state, keccak3.rs:254-286) and
 * flock_prove_seed. */
int flock_keccak3_setup_create(flock_ctx* ctx, size_t n_keccaks, int hash, int profile, flock_setup** out);
/* keccak3::KeccakSetup::verify (keccak3.rs:560-580) without a prover setup. */
int flock_keccak3_verify_bundle(flock_ctx* ctx, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen);
/* BlockR1cs::statement_digest of the 3-wide statement of size m. */
int flock_keccak3_statement_digest(uint32_t m, uint8_t* out32);
/* Debug/test: the 3-wide packed witness (2^(n_log + 10) u64 pairs each) and
 * the walker's column combination over 2^17 rows. */
int flock_keccak3_witness(flock_ctx* ctx, const flock_keccak_state* states, size_t n, uint32_t n_log, uint64_t* z,
                          uint64_t* a, uint64_t* b);
int flock_keccak3_comb(flock_ctx* ctx, const uint64_t* e, const uint64_t* alpha, const uint64_t* beta, uint64_t* comb);

/* ---- Degree-4 zerocheck round 1 (crates/flock-core/src/zerocheck/univariate_skip_deg4.rs) ----
 * round1_deg4_naive(a, b, c, d, z, m, r) (univariate_skip_deg4.rs:77-165)
 * on the GPU: the round-1 message of the constraint a b c d + z = 0 over 2^m
 * rows, each factor extended from S = {0..63} to Lambda4 = {64..255} of
 * GF(2^8).  The bit vectors are packed, 2^(m-6) u64 each (bit s of word x is
 * index 64 x + s); r: m F128 (lo, hi); p_abcd, p_z: 192 F128 each, the
 * evaluations at lambda = 64 + i.  6 <= m <= 30. */
int flock_zerocheck_round1_deg4(flock_ctx* ctx, const uint64_t* a, const uint64_t* b, const uint64_t* c,
                                const uint64_t* d, const uint64_t* z, uint32_t m, const uint64_t* r, uint64_t* p_abcd,
                                uint64_t* p_z);
/* Microbenchmark (benches/round1_deg4.rs): device-resident inputs, five
 * vectors of words SplitMix64(seed) (word i of the concatenation a|b|c|d|z is
 * the draw at state seed + (i + 1) gamma) and r from SplitMix64(seed ^ 1)
 * (lo then hi); *ms = mean device time of one message (eq table + kernel)
 * over `iters` after a warm-up; the last message into p_abcd / p_z when both
 * are non-null. */
int flock_bench_round1_deg4(flock_ctx* ctx, uint32_t m, uint64_t seed, int iters, double* ms, uint64_t* p_abcd,
                            uint64_t* p_z);

/* The flock_chain CLI's honest chain of `steps` records: record i has
 * cv = x_i (x_0 = initial_cv, or the BLAKE3 IV when NULL), 16 message words
 * from SplitMix64(seed) (low 32 bits of each draw), counter 0, block_len 64,
 * flags 0; x_{i+1} = out_lo(compress(record i)).  Runs on the host (each link
 * needs the previous output). */
int flock_chain_blocks(uint64_t seed, const uint32_t* initial_cv, size_t steps, uint32_t* records);
/* Verify a FLOCK v4 bundle of this setup's size: a compression proof
 * (flavor 2) or a hash-chain proof (flavor 3, whose public endpoints are the
 * ones the bundle carries), under the transcript domain it was proved with.
 * Returns FLOCK_OK, or FLOCK_ERR_VERIFY with flock_last_error() naming the
 * failed check.  The lincheck's matrix combination runs on the GPU; the rest
 * (transcript replay, Merkle openings, proof of work, residual basis) on the
 * calling thread. */
int flock_verify(flock_setup* s, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen);
/* The same verification without a prover setup, for any supported size
 * (2^8..2^20 compressions, read from the bundle): a verifier held by the
 * context and created on first use, with about 2 MiB of device scratch, plus
 * one device copy of the block matrices per device (about 45 MB, kept until
 * the process exits).  Calls on one context are serialised. */
int flock_verify_bundle(flock_ctx* ctx, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen);
/* Self-checking serving: with on != 0, every proof served by flock_submit /
 * flock_prove_batch is verified on its setup before it is returned, and one
 * that fails gets status FLOCK_ERR_VERIFY.  Call after flock_serve_start. */
int flock_serve_verify(flock_ctx* ctx, int on);
/* Page-locked host memory for inputs and outputs: flock_prove_blocks copies
 * compressions from such a buffer at the full host-to-device rate (a
 * pageable buffer is staged by the CUDA runtime first).  No counterpart in
 * the reference, whose prover reads host memory directly. */
int flock_host_alloc(size_t bytes, void** out);
void flock_host_free(void* p);
/* Device milliseconds of the last proof's phases (witness, RS encode, Merkle
 * commit, zerocheck round 1, zerocheck rounds, lincheck, ring switch +
 * combine, Ligerito L0 folds, Ligerito levels).  Returns the number written. */
int flock_setup_phase_ms(flock_setup* s, double* ms, int n);

/* Kernel-level entry points (host buffers). */
int flock_witness(flock_ctx* ctx, uint32_t log2, uint64_t seed, uint64_t* z, uint64_t* a, uint64_t* b);
int flock_ntt_rs_encode(flock_ctx* ctx, const uint64_t* msg, uint32_t log_msg_pos, uint32_t lanes,
                        uint32_t log_inv_rate, uint64_t* out);
int flock_merkle_tree(flock_ctx* ctx, const uint8_t* data, size_t n_leaves, size_t leaf_size, uint8_t* tree_out);
/* The same with the Merkle hash chosen (FLOCK_HASH_SHA256: leaf SHA256(bytes),
 * parent SHA256(left || right); merkle.rs:205-230). */
int flock_merkle_tree_hash(flock_ctx* ctx, const uint8_t* data, size_t n_leaves, size_t leaf_size, int hash,
                           uint8_t* tree_out);
/* NTT pass plans.  A plan splits the butterfly layers into passes over
 * shared-memory tiles (layers per pass, lanes per tile, threads per CTA);
 * flock_ntt_autotune times the candidate plans of a shape on this device and
 * keeps the fastest for every later encode of that shape in this process
 * (setups tune their own shapes when created).  desc receives a short
 * description of the chosen plan.  flock_ntt_rs_encode_plan runs candidate
 * plan `plan_index` (FLOCK_ERR_ARG past the last one); every plan gives the
 * same codeword.  No counterpart in the reference, whose CPU NTT has a fixed
 * schedule (crates/flock-core/src/ntt/additive_ntt_f128.rs:2785-2940). */
int flock_ntt_autotune(flock_ctx* ctx, uint32_t log_msg_pos, uint32_t lanes, uint32_t log_inv_rate, double* best_ms,
                       char* desc, size_t desc_cap);
int flock_ntt_rs_encode_plan(flock_ctx* ctx, const uint64_t* msg, uint32_t log_msg_pos, uint32_t lanes,
                             uint32_t log_inv_rate, uint32_t plan_index, uint64_t* out);
/* The description of candidate plan plan_index (host only; FLOCK_ERR_ARG past
 * the last one), and its device time on seeded resident inputs. */
int flock_ntt_plan_desc(uint32_t log_msg_pos, uint32_t lanes, uint32_t log_inv_rate, uint32_t plan_index, char* desc,
                        size_t desc_cap);
int flock_bench_ntt_plan(flock_ctx* ctx, uint32_t log_msg_pos, uint32_t lanes, uint32_t log_inv_rate,
                         uint32_t plan_index, int iters, double* ms);

int flock_sumcheck_round(flock_ctx* ctx, const uint64_t* f, const uint64_t* b, size_t n, uint64_t* msg_out);
/* Degree-3 (zerocheck-style) round over plain F128 vectors: msg_out =
 * (G(1), G(inf)) with G(1) = sum_j e[j] a[2j+1] b[2j+1] and
 * G(inf) = sum_j e[j] (a[2j] + a[2j+1]) (b[2j] + b[2j+1]).  With rho != NULL
 * a and b (n values each) are first folded at rho into a_out, b_out (n/2
 * values: x'[j] = x[2j] + rho (x[2j] + x[2j+1])) and the message is taken
 * over the folded pairs (e: n/4 values); otherwise e has n/2 values.
 * Replaces round_pair_naive + fold_in_place_pair (crates/flock-core/src/
 * zerocheck/multilinear.rs:616-657, 3194-3219). */
int flock_sumcheck_round3(flock_ctx* ctx, const uint64_t* e, const uint64_t* a, const uint64_t* b, size_t n,
                          const uint64_t* rho, uint64_t* a_out, uint64_t* b_out, uint64_t* msg_out);
int flock_pow(flock_ctx* ctx, const uint8_t* digest32, uint32_t bits, uint64_t* nonce);
int flock_f128_mul(flock_ctx* ctx, const uint64_t* a, const uint64_t* b, size_t n, uint64_t* out);
/* BLAKE3 digest of the R1CS statement for m = 14 + log2 (host only; replaces
 * BlockR1cs::statement_digest, crates/flock-core/src/r1cs.rs:334). */
int flock_statement_digest(uint32_t m, uint8_t* out32);

/* Device-resident timing of kernel microbenchmarks (inputs generated on the
 * device, CUDA events on the launching stream; milliseconds per launch). */
int flock_bench_ntt(flock_ctx* ctx, uint32_t log_msg_pos, uint32_t lanes, uint32_t log_inv_rate, int iters,
                    double* ms);
int flock_bench_merkle(flock_ctx* ctx, size_t n_leaves, size_t leaf_size, int iters, double* ms);
/* GF(2^128) products per second by a warp-uniform constant on all SMs (a
 * register loop, `iters` x 4 products per thread): variant 0 the integer
 * product (bit classes + Karatsuba), 1 the 4-bit window table in shared
 * memory, 2 half of the products each way, 3 a CTA-wide 8-bit window table
 * (64 KiB, 16 lookups of 16 bytes per product). */
int flock_bench_f128_product(flock_ctx* ctx, int variant, int iters, double* products_per_s);
/* Number of this library's kernel launches issued by the process so far
 * (lets a profiler skip a setup's autotuning launches). */
uint64_t flock_launch_count(void);
int flock_bench_sumcheck(flock_ctx* ctx, size_t n, int iters, double* ms);
/* fused fold + degree-3 message of flock_sumcheck_round3 over n values */
int flock_bench_sumcheck3(flock_ctx* ctx, size_t n, int iters, double* ms);
/* `steps` back-to-back proofs (seeds seed0, seed0+1, ...) timed with CUDA
 * events on the setup's stream; also the mean per-phase device times and the
 * number of this library's kernel launches inside the timed region. */
int flock_bench_prove(flock_setup* s, uint64_t seed0, int steps, double* total_ms, double* phase_ms,
                      uint64_t* launches);

/* Serving: continuous batching of proof jobs of different sizes on the
 * context's device.  Jobs run as proof slots and device memory free up,
 * shortest expected proof first (aged by waiting time, with a quarter of the
 * slots kept for jobs of at most 2^16 compressions); the kernels of up to
 * `slots` proofs overlap on the GPU.  Per-size setups are cached and reused
 * within the HBM budget given to flock_ctx_create (0: the free device memory
 * less 4 GiB), evicting idle setups (the largest first) when a new setup
 * needs room.  The result of a job is
 * byte-identical to flock_prove_seed / flock_prove_blocks of the same inputs.
 * No counterpart in the reference, which proves one request at a time
 * (benchmark-tools/worker/src/main.rs); this is the served form of the same
 * prove entry point. */
typedef struct flock_job {
  uint32_t log2_n;         /* 8..20 */
  uint64_t seed;           /* inputs from the benchmark generator when blocks == NULL */
  const uint32_t* blocks;  /* or 2^log2_n x 25 u32 compressions (copied at submit) */
  const uint8_t* domain;
  size_t dlen;
} flock_job;
typedef struct flock_result {
  uint8_t* out;       /* caller buffer for the proof bytes */
  size_t cap;
  size_t out_len;     /* proof length (also set when the buffer is too small) */
  int status;         /* status of the proof itself */
  double queue_ms;    /* submit -> start */
  double run_ms;      /* start -> proof bytes ready */
  double latency_ms;  /* submit -> proof bytes ready */
} flock_result;
/* Start serving with `slots` proofs in flight (optional: the first submit
 * starts it with 4). */
int flock_serve_start(flock_ctx* ctx, int slots);
int flock_submit(flock_ctx* ctx, const flock_job* job, uint64_t* ticket);
/* Builds setups for 2^log2_n compressions until `count` are cached idle (as
 * many as fit the free HBM budget: prewarming evicts no cached setup);
 * *cached receives how many are.  A setup
 * takes tens of milliseconds to build (device buffers, statement tables,
 * tuned NTT plans, captured commit graphs), which a job that finds none
 * waits for; a server that expects bursts of a size builds them first.  No
 * counterpart in the reference. */
int flock_serve_prewarm(flock_ctx* ctx, uint32_t log2_n, int count, int* cached);
/* FLOCK_OK once the job finished (then res->status is the proof's status),
 * FLOCK_ERR_TIMEOUT if it did not finish within timeout_ms (< 0: wait), or
 * FLOCK_ERR_CAPACITY with res->out_len set when res->cap is too small (the
 * result is kept for a retry). */
int flock_poll(flock_ctx* ctx, uint64_t ticket, flock_result* res, int timeout_ms);

/* Batched form of the same prove entry point: proves jobs[0..n) together and
 * returns when all are done (results[i] as flock_poll fills it; the call
 * returns FLOCK_ERR_CAPACITY if an output buffer was too small, otherwise
 * FLOCK_OK with each proof's own status in results[i].status).  Jobs are
 * admitted in order, in waves of as many as fit the context's HBM budget.
 * The witnesses, RS encodes and Merkle trees of a wave's seeded jobs run in
 * groups of 8 jobs, each group as one CUDA graph of fused launches over its
 * jobs (one persistent NTT pass kernel over the tiles of every job, one tree
 * level of every job per launch); the remaining phases of each proof run
 * concurrently on `threads` host threads, one CUDA stream each, starting as
 * soon as the proof's group is queued.  Every result is
 * byte-identical to flock_prove_seed / flock_prove_blocks of the same job.
 * No counterpart in the reference, which proves one job per worker process
 * (benchmark-tools/worker/src/main.rs). */
int flock_prove_batch(flock_ctx* ctx, const flock_job* jobs, size_t n, flock_result* results, int threads);

/* Merkle root of leaves already in device memory, for callers that may not
 * allocate device memory when they need the root (hosts whose device memory
 * is all reserved up front, plugins whose buffers are all owned by an outer
 * framework).  No counterpart in the reference: it exists only for such
 * callers.  `leaves` (n_leaves x leaf_size bytes) and `root_out` (32 bytes)
 * are device pointers; the work is queued on `stream` (a cudaStream_t, NULL
 * for the default stream) and the call returns without waiting.  The tree is
 * built in one fixed device array that holds at most 2^15 leaves (2 MiB, kept
 * by every GPU that loads the library until exit); more leaves return
 * FLOCK_ERR_CAPACITY.  Same leaf rules and same root as flock_merkle_tree.
 * The first call on a device looks the array's address up; make it before
 * any stream capture begins.  Calls share the array, so calls whose work
 * overlaps on the GPU race: serialise them.  The address is kept for the
 * process's lifetime: resetting the device after its first call is not
 * supported.  A CUDA error already pending on the calling thread is left for
 * its owner and the call returns FLOCK_ERR_CUDA without queuing work. */
int flock_merkle_root_noalloc(const void* leaves, size_t n_leaves, size_t leaf_size, void* root_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
