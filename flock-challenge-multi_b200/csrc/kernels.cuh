// Launch wrappers of the prover's device kernels (K0..K9).
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include "gf128.cuh"
#include "blake3.cuh"


// Number of this library's kernel launches issued by this process (reported
// by the benchmark; every launch wrapper adds its launches here).
std::atomic<uint64_t>& kernel_launch_counter();
// Launches issued by the calling thread (a graph capture counts the kernel
// nodes it records from this).
inline uint64_t& thread_launch_counter() {
  static thread_local uint64_t n = 0;
  return n;
}
inline void count_launch(uint64_t n = 1) {
  kernel_launch_counter().fetch_add(n, std::memory_order_relaxed);
  thread_launch_counter() += n;
}

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};
#define CK(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess)                                                                      \
      throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_) + " @" + __FILE__ + ":" + \
                      std::to_string(__LINE__));                                                \
  } while (0)

// Grid of a grid-stride kernel that runs as exactly one wave on `sms` SMs:
// the CTAs of `threads` threads and `smem` bytes of dynamic shared memory
// that fit one SM at once (registers, shared memory, threads), times `sms`.
// A grid of 4 CTAs per SM for a kernel that fits 3 leaves a second wave of
// one CTA per SM, which runs with the SM mostly idle.  The occupancy query
// runs once per (kernel, block shape) and process.
int resident_grid(const void* kernel, int threads, size_t smem, int sms);

// Makes `device` current for a scope and restores the caller's device after
// it, so that a library call leaves the calling thread's device as it was.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != device) CK(cudaSetDevice(device));
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;
};

// XOR-reduce v over the CTA and add the sum into *out (atomically): every
// thread of the CTA must call it.
__device__ __forceinline__ void block_xor_out(f128 v, f128* out) {
  __shared__ f128 red[32];
  v = warp_xor(v);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    int nw = (blockDim.x + 31) >> 5;
    f128 x = l < nw ? red[l] : mk(0, 0);
    x = warp_xor(x);
    if (l == 0) atomic_xor128(out, x);
  }
  __syncthreads();
}

// Merkle-path shift sumcheck (SHA-256 statement): the seven tables of a
// y-round (ta, te, tb, gz, gxl, gxr, g_other) and the claim's eight word
// coefficients
struct MpTables {
  f128* t[7];
};
struct MpCoeffs {
  f128 c[8];
};

// K0
void launch_witness_seed(uint64_t seed, uint32_t log2, uint32_t n_blocks, uint32_t n_slots, f128* z, f128* a,
                         f128* b, cudaStream_t s);
// records: 28 u32 per compression (cv, m, counter u64, block_len, flags);
// otherwise 25 (cv, m, counter_lo of the benchmark generator)
void launch_witness_blocks(const uint32_t* blocks, uint32_t n_blocks, uint32_t n_slots, f128* z, f128* a, f128* b,
                           cudaStream_t s, bool records = false);
// SHA-256 compressions, 2^15-bit blocks: records of 24 u32 (h_in, m), or
// records == nullptr for the benchmark generator from `seed`
void launch_witness_sha(const uint32_t* records, uint64_t seed, uint32_t n_blocks, uint32_t n_slots, f128* z, f128* a,
                        f128* b, cudaStream_t s);
// Keccak-f[1600] permutations: states of 25 u64 lanes, or states == nullptr
// for the benchmark generator from `seed`; width 1: one permutation per
// 2^16-bit block (keccak.rs), 3: three per 2^17-bit block (keccak3.rs)
void launch_witness_keccak(const uint64_t* states, uint64_t seed, uint32_t n_perm, uint32_t n_slots, f128* z, f128* a,
                           f128* b, cudaStream_t s, int width = 1);
// K6 of the Keccak statements: comb = alpha A^T e + B^T e + beta [const] over
// the rows of a block (e and comb: 2^16 or 2^17 values); W:
// keccak_comb_scratch(width) values; masks: keccak_masks(device), the round
// constants' share
const uint64_t* keccak_masks(int device);
size_t keccak_comb_scratch(int width = 1);
void keccak_comb(const f128* e, f128 alpha, f128 beta, const uint64_t* masks, f128* W, f128* comb, cudaStream_t s,
                 int width = 1);
// Degree-4 zerocheck round 1 (zerocheck/univariate_skip_deg4.rs): device
// sums H[8 l + k] (eq over the rows whose a b c d at lambda 64 + l has bit k)
// and Zs[s] (eq over the rows whose z bit s is set), XOR-ed into H (1536
// values) and Zs (64 values); round1_deg4_finish turns them into the two
// 192-value messages on the host.  tables: deg4_tables_bytes() on the device,
// filled by deg4_build_tables on the host.
size_t deg4_tables_bytes();
void deg4_build_tables(uint8_t* host);
void round1_deg4(const uint64_t* a, const uint64_t* b, const uint64_t* c, const uint64_t* d, const uint64_t* z,
                 const f128* eq, size_t n_rows, const uint8_t* tables, f128* H, f128* Zs, int grid, cudaStream_t s);
void round1_deg4_finish(const f128* H, const f128* Zs, f128* p_abcd, f128* p_z);
// K1
// NTT pass plans: the passes (first layer l0, layer count R, 2^lgs lanes per
// tile, threads per CTA) that cover layers layer_begin..log_d-1.
struct NttPass {
  int l0, R, lgs, threads;
  // 0: a thread owns a position pair and its lanes, products by integer
  // multiplies; 1: a warp owns a position pair's 64 lanes (lgs = 6) and
  // multiplies through a 4-bit window table of the warp-uniform twiddle;
  // 2: as 1, with half of the lanes through the integer product
  int kind = 0;
};
using NttPlan = std::vector<NttPass>;
// Times the candidate plans of a shape on `scratch` (lanes << log_d values,
// overwritten), keeps the fastest for this device and returns it; later
// encodes of the shape use it (untuned shapes use the default split).
NttPlan ntt_autotune(f128* scratch, int log_d, int lanes, int layer_begin, cudaStream_t s, double* best_ms = nullptr);
NttPlan ntt_plan(int log_d, int lanes, int layer_begin);
const f128* ntt_evals(int log_d);  // device table of the per-layer basis values
std::string ntt_plan_desc(const NttPlan& plan);
// every candidate plan of a shape, for parity tests of the tiling
size_t ntt_plan_count(int log_d, int lanes, int layer_begin);
// the description of candidate plan `index` ("" past the last one)
std::string ntt_plan_desc_at(int log_d, int lanes, int layer_begin, size_t index);
void ntt_rs_encode_plan(const f128* msg, f128* cw, int log_msg_pos, int lanes, int log_inv_rate, size_t plan_idx,
                        cudaStream_t s);
void ntt_rs_encode(const f128* msg, f128* cw, int log_msg_pos, int lanes, int log_inv_rate, cudaStream_t s);
void ntt_forward(f128* data, int log_d, int lanes, int start_layer, cudaStream_t s);
void ntt_transposed_encode(f128* e, f128* out, int log_msg, int log_inv_rate, cudaStream_t s);
// Fused multi-proof commit (serving / batching): one entry per proof of a
// device-resident job table; every launch of the commit covers all jobs, a
// thread block finding its job by binary search over the per-launch first
// indices (jobs that take no part in a launch have an empty range).
struct BatchJob {
  uint64_t seed;  // witness inputs from the benchmark generator
  uint32_t log2, n_blocks, n_slots;
  f128 *z, *a, *b;
  uint64_t wcta0;  // first CTA of this job in the witness launch
  f128* cw;        // RS codeword: 64 lanes, rate 1/2, 2^log_d positions
  const f128* ev;  // per-layer basis values of the NTT of dimension log_d
  int log_d;
  uint64_t msg_len, rep0;  // message values; first element in the replicate launch
  int n_pass;
  NttPass pass[4];
  uint64_t tile0[4];  // first tile of this job in the launch of pass p
  uint32_t* tree;     // Merkle tree over 2^log_d leaves of 1 KiB
  uint64_t n_leaves, leaf0;
  uint64_t par0[24];  // first node of this job in the launch of parent level k
  uint64_t top_start, top_len;  // the level the per-job top kernel starts from
};
uint32_t witness_ctas(uint32_t n_slots);
void launch_witness_seed_batch(const BatchJob* jobs, int n_jobs, uint32_t total_ctas, cudaStream_t s);
void ntt_replicate_batch(const BatchJob* jobs, int n_jobs, uint64_t total, cudaStream_t s);
size_t ntt_pass_batch_smem(const NttPass& p);
void ntt_pass_batch(const BatchJob* jobs, int n_jobs, int pass, uint64_t total_tiles, size_t smem, int grid,
                    cudaStream_t s);
void merkle_leaves_batch(const BatchJob* jobs, int n_jobs, uint64_t total, cudaStream_t s);
void merkle_parents_batch(const BatchJob* jobs, int n_jobs, int level, uint64_t total, cudaStream_t s);
void merkle_top_batch(const BatchJob* jobs, int n_jobs, cudaStream_t s);

// K2 / K9
void merkle_build(const void* data, size_t n_leaves, size_t leaf_size, uint32_t* tree, cudaStream_t s);
void merkle_leaves(const void* data, size_t n_leaves, size_t leaf_size, uint32_t* out, cudaStream_t s);
// the same over the Merkle hash fn (0 SHA-256: leaf SHA256(bytes), parent
// SHA256(l || r), leaf sizes multiples of 4 bytes; 1 BLAKE3: the above)
void merkle_build(const void* data, size_t n_leaves, size_t leaf_size, uint32_t* tree, int fn, cudaStream_t s);
void merkle_leaves(const void* data, size_t n_leaves, size_t leaf_size, uint32_t* out, int fn, cudaStream_t s);
__global__ void k_gather_nodes(const uint32_t* tree, const uint64_t* idx, size_t n, uint32_t* out);
// The sorted distinct leaf positions q followed by the flat-tree indices of
// their Merkle multi-proof's sibling nodes, in the order the proof lists them
// (merkle.rs:1020-1072: per level, the sibling of every position whose
// sibling is not itself opened).
std::vector<uint64_t> multiproof_ids(const std::vector<size_t>& q, size_t n_leaves);
__global__ void k_gather_rows(const f128* cw, const uint64_t* pos, size_t n, int lanes, f128* out);
// fn: the PoW hash (0 SHA-256, 1 BLAKE3; HashKind)
uint64_t pow_search(const uint8_t digest[32], uint32_t bits, cudaStream_t s, unsigned long long* d_found,
                    unsigned long long* h_found, int fn = 1);
// K3..K8
void eq_split(const f128* lo, const f128* hi, int s_bits, size_t n, f128* out, cudaStream_t s);
void axpy(f128* out, const f128* x, f128 beta, size_t n, cudaStream_t s);
void eq_build(const f128* r, int n, f128 scale, f128* out, cudaStream_t s);
void outer64(const f128* L, const f128* e, size_t n_e, f128* out, cudaStream_t s);
void inner(const f128* f, const f128* g, size_t n, f128* out, int grid, cudaStream_t s);
size_t round1_tables_size();
void build_round1_tables_host(const uint8_t M[64][64], const f128* phi8, void* dst);
void zc_round1(const f128* a, const f128* b, const f128* c, const void* tabs, const f128* eqc, size_t n_blocks,
               f128* out, int grid, cudaStream_t s);
void zc_round(int mode, const f128* a_in, const f128* b_in, f128* a_out, f128* b_out, const f128* lag, f128 rho,
              size_t n_pairs, int ns, int nm, int msh, const f128* etab, f128* out, int sms, cudaStream_t s,
              f128* halve_out = nullptr, size_t halve_n = 0);
void fold_pair_final(const f128* a_in, const f128* b_in, f128 rho, f128* out, cudaStream_t s);
// k: columns of the block matrices (2^k_log)
void lc_comb(const uint32_t* at_ptr, const uint16_t* at_row, const uint32_t* bt_ptr, const uint16_t* bt_row,
             const f128* eq, f128 alpha, f128 beta, int pin, int k, f128* comb, cudaStream_t s);
void lc_zvec(const f128* z, const f128* eqo, size_t n_outer, int k_log, f128* zv, int sms, cudaStream_t s);
void lc_round(f128* comb, f128* zv, int len, bool fold, f128 r, bool emit, f128* out, cudaStream_t s);
// s_hat_v of the ab claim from the block-folded z (2^k_log values)
void ring_shat_ab(const f128* zv_pre, const f128* eqt, int k_log, f128* out, cudaStream_t s);
// f, msg (optional): also XOR the first Ligerito message over (f, b_combined)
// into msg[0..2) (zeroed), the values k_lig_msg gives for the same pairs
void ring_bcombined_ct(const f128* elo0, const f128* ehi0, const f128* elo1, const f128* ehi1, const f128* L0,
                       const f128* L1, int lo_bits, size_t n_chunks, f128* out, int sms, cudaStream_t s,
                       const f128* f = nullptr, f128* msg = nullptr);
// sms: the SMs a launch may fill (one wave of resident CTAs on them)
void lig_msg(const f128* f, const f128* b, size_t n_pairs, f128* out, int sms, cudaStream_t s);
void lig_fold_msg(const f128* f, const f128* b, f128* fo, f128* bo, f128 r, size_t n_pairs_out, bool emit, f128* out,
                  int sms, cudaStream_t s);
// hash chain: region fold of every instance's cv / out_lo words (g = [In | Out],
// 2 n_inst values) and the packed-direct claim's scatter into b_combined;
// per: packed words per block (2^(k_log - 7))
// e: the R (<= 16) region weights eq(tau_pos, .); the output region at word out_word
void chain_fold(const f128* z, size_t n_inst, size_t per, const f128* e, int R, int out_word, f128* g,
                cudaStream_t s);
// c: the W (<= 32) word coefficients of the claim
void chain_scatter(f128* bc, const f128* eq_inst, size_t n_inst, size_t per, const f128* c, int W, cudaStream_t s);
// Merkle path (2^15-bit blocks): the four slot folds (out: 4 x n_inst), the
// weight tables ta, tb, one y-round, and the claim's scatter into b_combined
void mp_fold(const f128* z, size_t n_inst, f128 e0, f128 e1, f128* out, cudaStream_t s);
void mp_tables(const f128* eq_q, const f128* eq_p, f128 alpha, int pos_log, size_t n, const uint8_t* b, f128* ta,
               f128* tb, cudaStream_t s);
void mp_round(const MpTables& T, int len, bool fold, f128 r, bool emit, f128* out, cudaStream_t s);
void mp_scatter(f128* bc, const f128* eq_inst, size_t n_inst, const MpCoeffs& c, cudaStream_t s);
void sc3_round(const f128* a, const f128* b, const f128* e, f128* ao, f128* bo, const f128* rho, size_t n_pairs,
               f128* out, int grid, cudaStream_t s);
