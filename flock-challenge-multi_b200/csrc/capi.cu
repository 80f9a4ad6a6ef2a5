// extern "C" boundary of libflockgpu.so (declared in include/flock_gpu.h).
// Status codes, never exceptions across the ABI; caller-owned buffers.
#include "../../include/flock_gpu.h"
#include "prover.hpp"
#include "serve.hpp"
#include <atomic>
#include <algorithm>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>

struct flock_ctx {
  int device = 0;
  int sms = 1;  // the device's SM count
  uint64_t budget = 0;
  cudaStream_t st = nullptr;
  std::string err;
  std::mutex mu;
  std::unique_ptr<flock::Server> server;
  int fs_fn = flock::kFnBlake3;  // the transcript hash of the verify-bundle entry points
  std::mutex vmu;  // one verification at a time on the context's verifier
  std::unique_ptr<flock::Verifier> verifier;
};
struct flock_setup {
  flock_ctx* ctx = nullptr;
  std::unique_ptr<flock::Setup> s;
  size_t n_blocks = 0;  // compressions per proof (Blake3Setup::new(n_blocks))
};
static_assert(sizeof(flock_compression) == 28 * sizeof(uint32_t), "flock_compression is 28 u32");
// pcs::commit's retained prover state (commit.rs:143-185): the codeword and
// the Merkle tree, resident on the context's device.
struct flock_prover_data {
  flock_ctx* ctx = nullptr;
  uint32_t m = 0;
  size_t n_leaves = 0;
  f128* cw = nullptr;       // [pos * 64 + lane], 2^(m-12) positions
  uint32_t* tree = nullptr;  // flat tree, 2 * n_leaves - 1 nodes of 32 B
  ~flock_prover_data() {
    if (cw) cudaFree(cw);
    if (tree) cudaFree(tree);
  }
};
// FsChallenger (challenger.rs:170-600) with the BLAKE3 hash.
struct flock_challenger {
  flock::Transcript tr;
  flock_challenger(const std::string& domain, int fn) : tr(domain, fn) {}
};

std::atomic<uint64_t>& kernel_launch_counter() {
  static std::atomic<uint64_t> n{0};
  return n;
}

int resident_grid(const void* kernel, int threads, size_t smem, int sms) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, size_t, int>, int> per_sm;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  const auto key = std::make_tuple(kernel, threads, smem, dev);
  int b = 0;
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = per_sm.find(key);
    if (it != per_sm.end()) b = it->second;
  }
  if (!b) {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem));
    b = std::max(b, 1);
    std::lock_guard<std::mutex> g(mu);
    per_sm[key] = b;
  }
  return b * std::max(sms, 1);
}

namespace {
template <class F>
int guard(flock_ctx* c, F&& f) {
  try {
    return f();
  } catch (const CudaError& e) {
    if (c) c->err = e.what();
    return FLOCK_ERR_CUDA;
  } catch (const std::exception& e) {
    if (c) c->err = e.what();
    return FLOCK_ERR_INTERNAL;
  }
}
template <class T>
struct DevBuf {
  T* p = nullptr;
  explicit DevBuf(size_t n) { CK(cudaMalloc(&p, n * sizeof(T) + 16)); }
  ~DevBuf() { if (p) cudaFree(p); }
};
__global__ void k_fill(uint64_t* p, size_t n, uint64_t seed) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  p[i] = z ^ (z >> 31);
}
// GF(2^128) product rate: every thread multiplies four running values by its
// warp's constant `iters` times.  V = 0: the integer product (bit classes +
// Karatsuba, the constant's classes split once); 1: the 4-bit window table of
// the constant in shared memory; 2: two values each way; 3: the CTA-wide
// 8-bit window table (MulTab8) of one constant per CTA.
template <int V>
__global__ void __launch_bounds__(256) k_bench_product(const f128* tw, f128* out, int iters) {
  extern __shared__ __align__(16) uint8_t bsm[];
  Tab4* tabs = reinterpret_cast<Tab4*>(bsm);
  MulTab8* t8 = reinterpret_cast<MulTab8*>(bsm);
  const int warp = threadIdx.x >> 5;
  const f128 t = tw[(blockIdx.x * 8 + (V == 3 ? 0 : warp)) & 1023];
  const MulConst M = mulconst(t);
  if (V == 1 || V == 2) {
    tab4_build(&tabs[warp], t, threadIdx.x & 31);
    __syncwarp();
  }
  if (V == 3) multab_build(t8, t);
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  f128 x[4] = {mk(g * 0x9E3779B97F4A7C15ull, ~g), mk(g ^ 0x1234, g * 7), mk(g + 99, g * 13), mk(g * 31, g ^ 0xFFFF)};
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const bool table = V == 1 || (V == 2 && k >= 2);
      x[k] = fx(V == 3 ? multab_mul(t8, x[k]) : table ? tab4_mul(&tabs[warp], x[k]) : fmul_c(x[k], M), mk(1, 0));
    }
  }
  st(out + g, fx(fx(x[0], x[1]), fx(x[2], x[3])));
}
__global__ void k_mul(const f128* a, const f128* b, size_t n, f128* out) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) st(out + i, fmul(ld(a + i), ld(b + i)));
}
}  // namespace

extern "C" {

int flock_ctx_create(int device, uint64_t hbm_budget_bytes, flock_ctx** out) {
  if (!out) return FLOCK_ERR_ARG;
  auto* c = new flock_ctx();
  c->device = device;
  c->budget = hbm_budget_bytes;
  int rc = guard(c, [&] {
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) throw std::runtime_error("no such CUDA device");
    CK(cudaSetDevice(device));
    CK(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device));
    CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    return FLOCK_OK;
  });
  if (rc) {
    *out = nullptr;
    delete c;
    return rc;
  }
  *out = c;
  return FLOCK_OK;
}

void flock_ctx_destroy(flock_ctx* c) {
  if (!c) return;
  c->server.reset();  // joins the serving threads, frees their setups
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

const char* flock_last_error(flock_ctx* c) { return c ? c->err.c_str() : "null context"; }

int flock_setup_create(flock_ctx* c, uint32_t log2_n, int hash, int profile, flock_setup** out) {
  if (!c || !out) return FLOCK_ERR_ARG;
  if (log2_n < 8 || log2_n > 20 || (hash != FLOCK_HASH_BLAKE3 && hash != FLOCK_HASH_SHA256) ||
      profile != FLOCK_PROFILE_FAST) {
    c->err = "unsupported setup (log2 in 8..=20, BLAKE3 or SHA-256 Merkle hash, fast profile)";
    return FLOCK_ERR_ARG;
  }
  return guard(c, [&] {
    auto* s = new flock_setup();
    s->ctx = c;
    s->s.reset(new flock::Setup(c->device, log2_n, 0, flock::kHashBlake3, hash));
    s->n_blocks = (size_t)1 << log2_n;
    *out = s;
    return FLOCK_OK;
  });
}

int flock_setup_create_blocks(flock_ctx* c, size_t n_blocks, int hash, int profile, flock_setup** out) {
  if (!c || !out) return FLOCK_ERR_ARG;
  if (n_blocks == 0) {
    c->err = "n_blocks must be at least 1";
    return FLOCK_ERR_ARG;
  }
  // min_n_blocks_log (blake3.rs:1854-1858): 2^max(3, ceil(log2 n)) slots
  uint32_t n_log = 3;
  while (((size_t)1 << n_log) < n_blocks) n_log++;
  if (n_log < 8 || n_log > 20) {
    c->err = "unsupported n_blocks (129..=2^20: the Ligerito fast profile has ladders for m = 22..34)";
    return FLOCK_ERR_ARG;
  }
  const int rc = flock_setup_create(c, n_log, hash, profile, out);
  if (rc == FLOCK_OK) (*out)->n_blocks = n_blocks;
  return rc;
}

void flock_setup_destroy(flock_setup* s) { delete s; }

int flock_setup_set_transcript(flock_setup* s, int hash) {
  if (!s || (hash != FLOCK_HASH_SHA256 && hash != FLOCK_HASH_BLAKE3)) return FLOCK_ERR_ARG;
  s->s->fs_fn = hash;
  return FLOCK_OK;
}

int flock_ctx_set_transcript(flock_ctx* c, int hash) {
  if (!c || (hash != FLOCK_HASH_SHA256 && hash != FLOCK_HASH_BLAKE3)) return FLOCK_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->vmu);
  c->fs_fn = hash;
  return FLOCK_OK;
}

static int emit(flock_ctx* c, const std::vector<uint8_t>& bytes, uint8_t* out, size_t cap, size_t* out_len) {
  if (out_len) *out_len = bytes.size();
  if (bytes.size() > cap || !out) {
    c->err = "output buffer too small";
    return FLOCK_ERR_CAPACITY;
  }
  memcpy(out, bytes.data(), bytes.size());
  return FLOCK_OK;
}

int flock_prove_seed(flock_setup* s, uint64_t seed, const uint8_t* domain, size_t dlen, uint8_t* out, size_t cap,
                     size_t* out_len) {
  if (!s || (!domain && dlen)) return FLOCK_ERR_ARG;
  return guard(s->ctx, [&] {
    std::string d((const char*)domain, dlen);
    // a SHA-256 / Keccak setup generates its n_blocks inputs; a BLAKE3 one 2^log2
    const size_t n = s->s->hash != flock::kHashBlake3 ? s->n_blocks : 0;
    return emit(s->ctx, s->s->prove(&seed, nullptr, n, d), out, cap, out_len);
  });
}

static bool is_blake3(flock_setup* s) {
  if (s->s->hash == flock::kHashBlake3) return true;
  s->ctx->err = std::string("this entry point proves BLAKE3 compressions; the setup is a ") +
                (flock::is_keccak(s->s->hash) ? "Keccak" : "SHA-256") + " statement";
  return false;
}

int flock_prove_blocks(flock_setup* s, const uint32_t* blocks, size_t n, const uint8_t* domain, size_t dlen,
                       uint8_t* out, size_t cap, size_t* out_len) {
  if (!s || !blocks || (!domain && dlen)) return FLOCK_ERR_ARG;
  if (!is_blake3(s)) return FLOCK_ERR_ARG;
  if (n != ((size_t)1 << s->s->log2)) {
    s->ctx->err = "expected exactly 2^log2 compressions";
    return FLOCK_ERR_ARG;
  }
  return guard(s->ctx, [&] {
    if (!s->s->blocks_buf)
      CK(cudaMallocAsync(reinterpret_cast<void**>(&s->s->blocks_buf), n * 25 * sizeof(uint32_t), s->s->st));
    CK(cudaMemcpyAsync(s->s->blocks_buf, blocks, n * 25 * sizeof(uint32_t), cudaMemcpyHostToDevice, s->s->st));
    std::string d((const char*)domain, dlen);
    return emit(s->ctx, s->s->prove(nullptr, s->s->blocks_buf, n, d), out, cap, out_len);
  });
}

int flock_prove_compressions(flock_setup* s, const flock_compression* blocks, size_t n, const uint8_t* domain,
                             size_t dlen, uint8_t* out, size_t cap, size_t* out_len) {
  if (!s || !blocks || (!domain && dlen)) return FLOCK_ERR_ARG;
  if (!is_blake3(s)) return FLOCK_ERR_ARG;
  if (n != s->n_blocks) {
    s->ctx->err = "expected exactly the setup's n_blocks compressions";
    return FLOCK_ERR_ARG;
  }
  return guard(s->ctx, [&] {
    const size_t slots = (size_t)1 << s->s->log2;
    if (!s->s->records_buf)
      CK(cudaMallocAsync(reinterpret_cast<void**>(&s->s->records_buf), slots * 28 * sizeof(uint32_t), s->s->st));
    CK(cudaMemcpyAsync(s->s->records_buf, blocks, n * sizeof(flock_compression), cudaMemcpyHostToDevice, s->s->st));
    std::string d((const char*)domain, dlen);
    return emit(s->ctx, s->s->prove(nullptr, s->s->records_buf, n, d, false, nullptr, true), out, cap, out_len);
  });
}

// ---- SHA-256 compressions (r1cs_hashes/sha2.rs)
int flock_sha256_setup_create(flock_ctx* c, size_t n_compressions, int hash, int profile, flock_setup** out) {
  if (!c || !out) return FLOCK_ERR_ARG;
  // min_n_blocks_log (sha2.rs:1217-1221): 2^max(3, ceil(log2 n)) slots
  uint32_t n_log = 3;
  while (n_compressions && ((size_t)1 << n_log) < n_compressions) n_log++;
  if (n_compressions == 0 || n_log < 7 || n_log > 19 || (hash != FLOCK_HASH_BLAKE3 && hash != FLOCK_HASH_SHA256) ||
      profile != FLOCK_PROFILE_FAST) {
    c->err = "unsupported SHA-256 setup (65..=2^19 compressions: the fast profile's Ligerito ladders cover "
             "m = 22..34; BLAKE3 or SHA-256 Merkle hash, fast profile)";
    return FLOCK_ERR_ARG;
  }
  return guard(c, [&] {
    auto* s = new flock_setup();
    s->ctx = c;
    s->s.reset(new flock::Setup(c->device, n_log, 0, flock::kHashSha256, hash));
    s->n_blocks = n_compressions;
    *out = s;
    return FLOCK_OK;
  });
}

int flock_sha256_prove(flock_setup* s, const flock_sha256_compression* comps, size_t n, const uint8_t* domain,
                       size_t dlen, uint8_t* out, size_t cap, size_t* out_len) {
  if (!s || !comps || (!domain && dlen)) return FLOCK_ERR_ARG;
  if (s->s->hash != flock::kHashSha256) {
    s->ctx->err = "not a SHA-256 setup";
    return FLOCK_ERR_ARG;
  }
  if (n != s->n_blocks) {
    s->ctx->err = "expected exactly the setup's n_compressions compressions";
    return FLOCK_ERR_ARG;
  }
  return guard(s->ctx, [&] {
    if (!s->s->records_buf)
      CK(cudaMallocAsync(reinterpret_cast<void**>(&s->s->records_buf), n * sizeof(flock_sha256_compression),
                         s->s->st));
    CK(cudaMemcpyAsync(s->s->records_buf, comps, n * sizeof(flock_sha256_compression), cudaMemcpyHostToDevice,
                       s->s->st));
    std::string d((const char*)domain, dlen);
    return emit(s->ctx, s->s->prove(nullptr, s->s->records_buf, n, d), out, cap, out_len);
  });
}

int flock_sha256_merkle_prove(flock_setup* s, const flock_sha256_compression* comps, size_t n, const uint8_t* b_bits,
                              uint32_t path_log, const uint8_t* domain, size_t dlen, uint8_t* out, size_t cap,
                              size_t* out_len) {
  if (!s || !comps || !b_bits || (!domain && dlen)) return FLOCK_ERR_ARG;
  if (s->s->hash != flock::kHashSha256 || n != s->n_blocks || n != ((size_t)1 << s->s->n_log) ||
      path_log > (uint32_t)s->s->n_log) {
    s->ctx->err = "a Merkle-path proof needs a SHA-256 setup whose n_compressions (a power of two) it fills, "
                  "and path_log <= log2(n)";
    return FLOCK_ERR_ARG;
  }
  return guard(s->ctx, [&] {
    if (!s->s->records_buf)
      CK(cudaMallocAsync(reinterpret_cast<void**>(&s->s->records_buf), n * sizeof(flock_sha256_compression),
                         s->s->st));
    CK(cudaMemcpyAsync(s->s->records_buf, comps, n * sizeof(flock_sha256_compression), cudaMemcpyHostToDevice,
                       s->s->st));
    flock::MerkleArgs ma;
    ma.path_log = (int)path_log;
    ma.b_bits = b_bits;
    std::string d((const char*)domain, dlen);
    return emit(s->ctx, s->s->prove(nullptr, s->s->records_buf, n, d, false, nullptr, false, &ma), out, cap,
                out_len);
  });
}

int flock_sha256_merkle_verify(flock_ctx* c, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen,
                               uint32_t path_log, const uint8_t* b_bits, size_t n, const uint32_t* leaves,
                               const uint32_t* root) {
  if (!c || !bytes || !b_bits || !leaves || !root || (!domain && dlen) || path_log > 30 || n == 0 ||
      (n & (n - 1)) || ((size_t)1 << path_log) > n)
    return FLOCK_ERR_ARG;
  return guard(c, [&] {
    flock::MerklePublic mp;
    mp.path_log = (int)path_log;
    mp.b_bits.assign(b_bits, b_bits + n);
    mp.leaves.resize((size_t)1 << path_log);
    for (size_t p = 0; p < mp.leaves.size(); p++) memcpy(mp.leaves[p].data(), leaves + 8 * p, 32);
    memcpy(mp.root.data(), root, 32);
    std::lock_guard<std::mutex> lk(c->vmu);
    if (!c->verifier) c->verifier.reset(new flock::Verifier(c->device));
    const std::string why =
        c->verifier->verify(bytes, len, std::string((const char*)domain, dlen), flock::kHashSha256, &mp, c->fs_fn);
    if (why.empty()) return (int)FLOCK_OK;
    c->err = "verify: " + why;
    return (int)FLOCK_ERR_VERIFY;
  });
}

int flock_sha256_merkle_inputs(uint32_t n_log, uint32_t path_log, uint64_t seed, flock_sha256_compression* comps,
                               uint8_t* b_bits, uint32_t* leaves, uint32_t* root) {
  if (!comps || !b_bits || !leaves || !root || n_log > 24 || path_log > n_log) return FLOCK_ERR_ARG;
  static const uint32_t kIv[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                  0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  uint64_t st = seed;
  auto nx = [&]() {
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return (uint32_t)(z ^ (z >> 31));
  };
  const size_t L = (size_t)1 << (n_log - path_log), P = (size_t)1 << path_log;
  uint32_t cur[8];
  for (int k = 0; k < 8; k++) cur[k] = nx();
  for (size_t p = 0; p < P; p++) memcpy(leaves + 8 * p, cur, 32);
  b_bits[0] = 0;
  for (size_t i = 1; i < L; i++) b_bits[i] = nx() & 1;
  for (size_t i = 0; i < L; i++) {
    uint32_t sib[8];
    for (int k = 0; k < 8; k++) sib[k] = nx();
    flock_sha256_compression& cp = comps[i];
    memcpy(cp.h, kIv, 32);
    memcpy(cp.m + (b_bits[i] ? 8 : 0), cur, 32);
    memcpy(cp.m + (b_bits[i] ? 0 : 8), sib, 32);
    flock::sha256_compress(cp.h, cp.m, cur);
  }
  memcpy(root, cur, 32);
  for (size_t p = 1; p < P; p++) {
    memcpy(comps + p * L, comps, L * sizeof(flock_sha256_compression));
    memcpy(b_bits + p * L, b_bits, L);
  }
  return FLOCK_OK;
}

void flock_sha256_compress(const uint32_t* h_in, const uint32_t* m, uint32_t* out) {
  if (h_in && m && out) flock::sha256_compress(h_in, m, out);
}

int flock_sha256_verify_bundle(flock_ctx* c, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen) {
  if (!c || !bytes || (!domain && dlen)) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    std::lock_guard<std::mutex> lk(c->vmu);
    if (!c->verifier) c->verifier.reset(new flock::Verifier(c->device));
    const std::string why =
        c->verifier->verify(bytes, len, std::string((const char*)domain, dlen), flock::kHashSha256, nullptr, c->fs_fn);
    if (why.empty()) return (int)FLOCK_OK;
    c->err = "verify: " + why;
    return (int)FLOCK_ERR_VERIFY;
  });
}

int flock_sha256_statement_digest(uint32_t m, uint8_t* out32) {
  if (!out32 || m < 18 || m > 40) return FLOCK_ERR_ARG;
  try {
    auto d = flock::statement_digest(flock::kHashSha256, (int)m);
    memcpy(out32, d.data(), 32);
    return FLOCK_OK;
  } catch (...) {
    return FLOCK_ERR_INTERNAL;
  }
}

int flock_sha256_witness(flock_ctx* c, const flock_sha256_compression* comps, size_t n, uint32_t n_log, uint64_t* z,
                         uint64_t* a, uint64_t* b) {
  if (!c || !z || !a || !b || n_log < 3 || n_log > 20 || n > ((size_t)1 << n_log) || (n && !comps))
    return FLOCK_ERR_ARG;
  return guard(c, [&] {
    const size_t slots = (size_t)1 << n_log, words = slots * 256;
    DevBuf<f128> dz(words), da(words), db(words);
    DevBuf<uint32_t> dr(n ? n * 24 : 1);
    if (n) CK(cudaMemcpyAsync(dr.p, comps, n * 96, cudaMemcpyHostToDevice, c->st));
    launch_witness_sha(dr.p, 0, (uint32_t)n, (uint32_t)slots, dz.p, da.p, db.p, c->st);
    CK(cudaMemcpyAsync(z, dz.p, words * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(a, da.p, words * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(b, db.p, words * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return FLOCK_OK;
  });
}

// ---- Keccak-f[1600] permutations (r1cs_hashes/keccak.rs)
static_assert(sizeof(flock_keccak_state) == 200, "flock_keccak_state is 25 u64");
namespace {
// width 1: KeccakSetup of keccak.rs; 3: the 3-wide one of keccak3.rs
int keccak_hash_of(int width) { return width == 3 ? flock::kHashKeccak3 : flock::kHashKeccak; }
int keccak_setup(flock_ctx* c, size_t n_keccaks, int width, int hash, int profile, flock_setup** out) {
  if (!c || !out) return FLOCK_ERR_ARG;
  // min_n_keccaks_log (keccak.rs:513-518) / min_n_blocks_log (keccak3.rs:144-150):
  // 2^max(3, ceil(log2 ceil(n / width))) blocks
  const size_t blocks = (n_keccaks + width - 1) / width;
  uint32_t n_log = 3;
  while (((size_t)1 << n_log) < blocks) n_log++;
  const int k_log = flock::hash_k_log(keccak_hash_of(width));
  if (n_keccaks == 0 || (int)n_log + k_log < 22 || (int)n_log + k_log > 34 ||
      (hash != FLOCK_HASH_BLAKE3 && hash != FLOCK_HASH_SHA256) || profile != FLOCK_PROFILE_FAST) {
    c->err = width == 3 ? "unsupported 3-wide Keccak setup (49..=3 * 2^17 permutations: the fast profile's Ligerito "
                          "ladders cover m = 22..34; BLAKE3 or SHA-256 Merkle hash, fast profile)"
                        : "unsupported Keccak setup (33..=2^18 permutations: the fast profile's Ligerito ladders cover "
                          "m = 22..34; BLAKE3 or SHA-256 Merkle hash, fast profile)";
    return FLOCK_ERR_ARG;
  }
  return guard(c, [&] {
    auto* s = new flock_setup();
    s->ctx = c;
    s->s.reset(new flock::Setup(c->device, n_log, 0, keccak_hash_of(width), hash));
    s->n_blocks = n_keccaks;
    *out = s;
    return FLOCK_OK;
  });
}
int keccak_verify(flock_ctx* c, int width, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen) {
  if (!c || !bytes || (!domain && dlen)) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    std::lock_guard<std::mutex> lk(c->vmu);
    if (!c->verifier) c->verifier.reset(new flock::Verifier(c->device));
    const std::string why = c->verifier->verify(bytes, len, std::string((const char*)domain, dlen),
                                                keccak_hash_of(width), nullptr, c->fs_fn);
    if (why.empty()) return (int)FLOCK_OK;
    c->err = "verify: " + why;
    return (int)FLOCK_ERR_VERIFY;
  });
}
int keccak_digest(int width, uint32_t m, uint8_t* out32) {
  if (!out32 || m < 19 || m > 40) return FLOCK_ERR_ARG;
  try {
    auto d = flock::statement_digest(keccak_hash_of(width), (int)m);
    memcpy(out32, d.data(), 32);
    return FLOCK_OK;
  } catch (...) {
    return FLOCK_ERR_INTERNAL;
  }
}
int keccak_witness(flock_ctx* c, int width, const flock_keccak_state* states, size_t n, uint32_t n_log, uint64_t* z,
                   uint64_t* a, uint64_t* b) {
  if (!c || !z || !a || !b || n_log < 3 || n_log > 18 || n > ((size_t)width << n_log) || (n && !states))
    return FLOCK_ERR_ARG;
  return guard(c, [&] {
    const size_t slots = (size_t)1 << n_log;
    const size_t words = slots << (flock::hash_k_log(keccak_hash_of(width)) - 7);  // F128 per vector
    DevBuf<f128> dz(words), da(words), db(words);
    DevBuf<flock_keccak_state> ds(n ? n : 1);
    if (n) CK(cudaMemcpyAsync(ds.p, states, n * sizeof(flock_keccak_state), cudaMemcpyHostToDevice, c->st));
    launch_witness_keccak(reinterpret_cast<const uint64_t*>(ds.p), 0, (uint32_t)n, (uint32_t)slots, dz.p, da.p, db.p,
                          c->st, width);
    CK(cudaMemcpyAsync(z, dz.p, words * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(a, da.p, words * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(b, db.p, words * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return FLOCK_OK;
  });
}
int keccak_comb_call(flock_ctx* c, int width, const uint64_t* e, const uint64_t* alpha, const uint64_t* beta,
                     uint64_t* comb) {
  if (!c || !e || !alpha || !beta || !comb) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    const size_t kk = (size_t)1 << flock::hash_k_log(keccak_hash_of(width));
    DevBuf<f128> de(kk), dc(kk), dw(keccak_comb_scratch(width));
    CK(cudaMemcpyAsync(de.p, e, kk * 16, cudaMemcpyHostToDevice, c->st));
    keccak_comb(de.p, mk(alpha[0], alpha[1]), mk(beta[0], beta[1]), keccak_masks(c->device), dw.p, dc.p, c->st,
                width);
    CK(cudaMemcpyAsync(comb, dc.p, kk * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return FLOCK_OK;
  });
}
}  // namespace

int flock_keccak_setup_create(flock_ctx* c, size_t n_keccaks, int hash, int profile, flock_setup** out) {
  return keccak_setup(c, n_keccaks, 1, hash, profile, out);
}
int flock_keccak3_setup_create(flock_ctx* c, size_t n_keccaks, int hash, int profile, flock_setup** out) {
  return keccak_setup(c, n_keccaks, 3, hash, profile, out);
}

int flock_keccak_prove(flock_setup* s, const flock_keccak_state* states, size_t n, const uint8_t* domain, size_t dlen,
                       uint8_t* out, size_t cap, size_t* out_len) {
  if (!s || !states || (!domain && dlen)) return FLOCK_ERR_ARG;
  if (!flock::is_keccak(s->s->hash)) {
    s->ctx->err = "not a Keccak setup";
    return FLOCK_ERR_ARG;
  }
  if (n != s->n_blocks) {
    s->ctx->err = "expected exactly the setup's n_keccaks states";
    return FLOCK_ERR_ARG;
  }
  return guard(s->ctx, [&] {
    if (!s->s->records_buf)
      CK(cudaMallocAsync(reinterpret_cast<void**>(&s->s->records_buf), n * sizeof(flock_keccak_state), s->s->st));
    CK(cudaMemcpyAsync(s->s->records_buf, states, n * sizeof(flock_keccak_state), cudaMemcpyHostToDevice, s->s->st));
    std::string d((const char*)domain, dlen);
    return emit(s->ctx, s->s->prove(nullptr, s->s->records_buf, n, d), out, cap, out_len);
  });
}

int flock_keccak_verify_bundle(flock_ctx* c, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen) {
  return keccak_verify(c, 1, bytes, len, domain, dlen);
}
int flock_keccak3_verify_bundle(flock_ctx* c, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen) {
  return keccak_verify(c, 3, bytes, len, domain, dlen);
}

void flock_keccak_f(uint64_t* lanes25) {
  if (lanes25) flock::keccak_f(lanes25);
}

int flock_keccak_bench_inputs(size_t n, uint64_t seed, flock_keccak_state* out) {
  if (!out && n) return FLOCK_ERR_ARG;
  uint64_t st = seed;
  for (size_t k = 0; k < n; k++) {
    uint64_t d[25];
    for (int w = 0; w < 25; w++) {
      st += 0x9E3779B97F4A7C15ull;
      uint64_t z = st;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      d[w] = z ^ (z >> 31);
    }
    for (int l = 0; l < 25; l++) {
      uint64_t v = 0;
      for (int z = 0; z < 64; z++) {
        const int i = l + 25 * z;  // state bit (x, y, z), l = x + 5y
        v |= ((d[i / 64] >> (i % 64)) & 1ull) << z;
      }
      out[k].lanes[l] = v;
    }
  }
  return FLOCK_OK;
}

int flock_keccak_statement_digest(uint32_t m, uint8_t* out32) { return keccak_digest(1, m, out32); }
int flock_keccak3_statement_digest(uint32_t m, uint8_t* out32) { return keccak_digest(3, m, out32); }

int flock_keccak_witness(flock_ctx* c, const flock_keccak_state* states, size_t n, uint32_t n_log, uint64_t* z,
                         uint64_t* a, uint64_t* b) {
  return keccak_witness(c, 1, states, n, n_log, z, a, b);
}
int flock_keccak3_witness(flock_ctx* c, const flock_keccak_state* states, size_t n, uint32_t n_log, uint64_t* z,
                          uint64_t* a, uint64_t* b) {
  return keccak_witness(c, 3, states, n, n_log, z, a, b);
}

int flock_keccak_comb(flock_ctx* c, const uint64_t* e, const uint64_t* alpha, const uint64_t* beta, uint64_t* comb) {
  return keccak_comb_call(c, 1, e, alpha, beta, comb);
}
int flock_keccak3_comb(flock_ctx* c, const uint64_t* e, const uint64_t* alpha, const uint64_t* beta, uint64_t* comb) {
  return keccak_comb_call(c, 3, e, alpha, beta, comb);
}

int flock_pcs_commit(flock_ctx* c, const uint64_t* z_packed, uint32_t m, uint8_t* root32, flock_prover_data** out) {
  if (!c || !z_packed || !root32 || !out) return FLOCK_ERR_ARG;
  if (m < 22 || m > 34) {
    c->err = "pcs_commit: m must be in 22..=34 (log_batch_size 6, rate 1/2)";
    return FLOCK_ERR_ARG;
  }
  *out = nullptr;
  return guard(c, [&] {
    std::unique_ptr<flock_prover_data> pd(new flock_prover_data());
    pd->ctx = c;
    pd->m = m;
    const size_t n_msg = (size_t)1 << (m - 7);  // packed F128 values = 2^(m-13) positions x 64 lanes
    pd->n_leaves = (size_t)1 << (m - 12);
    CK(cudaMalloc(&pd->cw, 2 * n_msg * sizeof(f128)));
    CK(cudaMalloc(&pd->tree, (2 * pd->n_leaves - 1) * 32));
    DevBuf<f128> z(n_msg);
    CK(cudaMemcpyAsync(z.p, z_packed, n_msg * sizeof(f128), cudaMemcpyHostToDevice, c->st));
    ntt_rs_encode(z.p, pd->cw, (int)m - 13, 64, 1, c->st);
    merkle_build(pd->cw, pd->n_leaves, 64 * sizeof(f128), pd->tree, c->st);
    CK(cudaMemcpyAsync(root32, pd->tree + 8 * (2 * pd->n_leaves - 2), 32, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    *out = pd.release();
    return FLOCK_OK;
  });
}

int flock_prover_data_open(flock_prover_data* pd, const uint64_t* positions, size_t n, uint64_t* rows_out,
                           uint8_t* proof_out, size_t proof_cap, size_t* proof_count) {
  if (!pd || (!positions && n) || (!rows_out && n) || !proof_count) return FLOCK_ERR_ARG;
  flock_ctx* c = pd->ctx;
  for (size_t i = 0; i < n; i++)
    if (positions[i] >= pd->n_leaves || (i && positions[i] <= positions[i - 1])) {
      c->err = "prover_data_open: positions must be sorted, distinct and below the leaf count";
      return FLOCK_ERR_ARG;
    }
  return guard(c, [&] {
    const std::vector<size_t> q(positions, positions + n);
    const std::vector<uint64_t> ids = multiproof_ids(q, pd->n_leaves);
    const size_t ns = ids.size() - n;
    *proof_count = ns;
    if (ns > proof_cap || (ns && !proof_out)) {
      c->err = "prover_data_open: proof buffer too small";
      return (int)FLOCK_ERR_CAPACITY;
    }
    DevBuf<uint64_t> idx(ids.size());
    DevBuf<f128> rows(n * 64 + 2 * ns);
    CK(cudaMemcpyAsync(idx.p, ids.data(), ids.size() * 8, cudaMemcpyHostToDevice, c->st));
    if (n) {
      count_launch();
      k_gather_rows<<<(unsigned)((n * 64 + 255) / 256), 256, 0, c->st>>>(pd->cw, idx.p, n, 64, rows.p);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(rows_out, rows.p, n * 64 * sizeof(f128), cudaMemcpyDeviceToHost, c->st));
    }
    if (ns) {
      uint32_t* nodes = reinterpret_cast<uint32_t*>(rows.p + n * 64);
      count_launch();
      k_gather_nodes<<<(unsigned)((ns + 127) / 128), 128, 0, c->st>>>(pd->tree, idx.p + n, ns, nodes);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(proof_out, nodes, ns * 32, cudaMemcpyDeviceToHost, c->st));
    }
    CK(cudaStreamSynchronize(c->st));
    return (int)FLOCK_OK;
  });
}

void flock_prover_data_destroy(flock_prover_data* pd) { delete pd; }

int flock_challenger_create(const uint8_t* domain, size_t dlen, flock_challenger** out) {
  if (!out || (!domain && dlen)) return FLOCK_ERR_ARG;
  try {
    *out = new flock_challenger(std::string((const char*)domain, dlen), flock::kFnBlake3);
  } catch (...) {
    return FLOCK_ERR_INTERNAL;
  }
  return FLOCK_OK;
}

int flock_challenger_create_hash(const uint8_t* domain, size_t dlen, int hash, flock_challenger** out) {
  if (!out || (!domain && dlen) || (hash != FLOCK_HASH_SHA256 && hash != FLOCK_HASH_BLAKE3)) return FLOCK_ERR_ARG;
  try {
    *out = new flock_challenger(std::string((const char*)domain, dlen), hash);
  } catch (...) {
    return FLOCK_ERR_INTERNAL;
  }
  return FLOCK_OK;
}
void flock_challenger_destroy(flock_challenger* ch) { delete ch; }
int flock_challenger_observe_label(flock_challenger* ch, const uint8_t* label, size_t len) {
  if (!ch || (!label && len)) return FLOCK_ERR_ARG;
  ch->tr.label_bytes(label, len);
  return FLOCK_OK;
}
int flock_challenger_observe_bytes(flock_challenger* ch, const uint8_t* bytes, size_t len) {
  if (!ch || (!bytes && len)) return FLOCK_ERR_ARG;
  ch->tr.bytes(bytes, len);
  return FLOCK_OK;
}
int flock_challenger_observe_f128(flock_challenger* ch, const uint64_t* value) {
  if (!ch || !value) return FLOCK_ERR_ARG;
  ch->tr.f128v(mk(value[0], value[1]));
  return FLOCK_OK;
}
int flock_challenger_observe_f128_slice(flock_challenger* ch, const uint64_t* values, size_t n) {
  if (!ch || (!values && n)) return FLOCK_ERR_ARG;
  std::vector<f128> v(n);
  for (size_t i = 0; i < n; i++) v[i] = mk(values[2 * i], values[2 * i + 1]);
  ch->tr.f128s(v.data(), n);
  return FLOCK_OK;
}
int flock_challenger_sample_f128(flock_challenger* ch, uint64_t* out) {
  if (!ch || !out) return FLOCK_ERR_ARG;
  const f128 v = ch->tr.sample();
  out[0] = v.lo;
  out[1] = v.hi;
  return FLOCK_OK;
}
int flock_challenger_sample_f128_vec(flock_challenger* ch, size_t n, uint64_t* out) {
  if (!ch || (!out && n)) return FLOCK_ERR_ARG;
  const std::vector<f128> v = ch->tr.sample_vec(n);
  for (size_t i = 0; i < n; i++) { out[2 * i] = v[i].lo; out[2 * i + 1] = v[i].hi; }
  return FLOCK_OK;
}
int flock_challenger_grind_pow(flock_challenger* ch, flock_ctx* c, uint32_t bits, uint64_t* nonce) {
  if (!ch || !nonce || bits > 40 || (!c && bits > flock::kHostPowBits)) return FLOCK_ERR_ARG;
  if (bits <= flock::kHostPowBits) {  // a few dozen hashes: on the calling thread
    uint8_t d[32];
    ch->tr.state_digest(d);
    *nonce = bits ? flock::pow_search_host(d, bits, ch->tr.fn()) : 0;
    ch->tr.nonce(*nonce);
    return FLOCK_OK;
  }
  return guard(c, [&] {
    uint64_t n = 0;
    if (bits) {
      uint8_t d[32];
      ch->tr.state_digest(d);
      DevBuf<unsigned long long> found(1);
      unsigned long long* h = nullptr;
      CK(cudaMallocHost(&h, 8));
      try {
        n = pow_search(d, bits, c->st, found.p, h, ch->tr.fn());
      } catch (...) {
        cudaFreeHost(h);
        throw;
      }
      cudaFreeHost(h);
    }
    ch->tr.nonce(n);
    *nonce = n;
    return (int)FLOCK_OK;
  });
}
int flock_challenger_verify_pow(flock_challenger* ch, uint64_t nonce, uint32_t bits) {
  if (!ch) return FLOCK_ERR_ARG;
  return ch->tr.verify_pow(nonce, bits) ? FLOCK_OK : FLOCK_ERR_VERIFY;
}
int flock_challenger_state_digest(flock_challenger* ch, uint8_t* out32) {
  if (!ch || !out32) return FLOCK_ERR_ARG;
  ch->tr.state_digest(out32);
  return FLOCK_OK;
}

int flock_prove_chain(flock_setup* s, const uint32_t* records, size_t n, const uint8_t* domain, size_t dlen,
                      uint8_t* out, size_t cap, size_t* out_len) {
  if (!s || !records || (!domain && dlen)) return FLOCK_ERR_ARG;
  if (!is_blake3(s)) return FLOCK_ERR_ARG;
  if (n != ((size_t)1 << s->s->log2)) {
    s->ctx->err = "a chain fills every slot: expected exactly 2^log2 compressions";
    return FLOCK_ERR_ARG;
  }
  return guard(s->ctx, [&] {
    flock::ChainEnds ends;
    memcpy(ends.in, records, 32);  // 8 u32 words, little endian
    const uint32_t* last = records + 28 * (n - 1);
    uint32_t st16[16];
    flock::b3_compress(last, last + 8, (uint64_t)last[24] | (uint64_t)last[25] << 32, last[26], last[27], st16);
    memcpy(ends.out, st16, 32);
    if (!s->s->records_buf)
      CK(cudaMallocAsync(reinterpret_cast<void**>(&s->s->records_buf), n * 28 * sizeof(uint32_t), s->s->st));
    CK(cudaMemcpyAsync(s->s->records_buf, records, n * 28 * sizeof(uint32_t), cudaMemcpyHostToDevice, s->s->st));
    std::string d((const char*)domain, dlen);
    return emit(s->ctx, s->s->prove(nullptr, s->s->records_buf, n, d, false, &ends), out, cap, out_len);
  });
}

int flock_sha256_prove_chain(flock_setup* s, const flock_sha256_compression* comps, size_t n, const uint8_t* domain,
                             size_t dlen, uint8_t* out, size_t cap, size_t* out_len) {
  if (!s || !comps || (!domain && dlen)) return FLOCK_ERR_ARG;
  if (s->s->hash != flock::kHashSha256) {
    s->ctx->err = "not a SHA-256 setup";
    return FLOCK_ERR_ARG;
  }
  if (n != s->n_blocks || n != ((size_t)1 << s->s->n_log)) {
    s->ctx->err = "a chain fills every slot: expected the setup's n_compressions, a power of two";
    return FLOCK_ERR_ARG;
  }
  return guard(s->ctx, [&] {
    flock::ChainEnds ends;
    memcpy(ends.in, comps[0].h, 32);
    uint32_t h_last[8];
    flock::sha256_compress(comps[n - 1].h, comps[n - 1].m, h_last);
    memcpy(ends.out, h_last, 32);
    if (!s->s->records_buf)
      CK(cudaMallocAsync(reinterpret_cast<void**>(&s->s->records_buf), n * sizeof(flock_sha256_compression),
                         s->s->st));
    CK(cudaMemcpyAsync(s->s->records_buf, comps, n * sizeof(flock_sha256_compression), cudaMemcpyHostToDevice,
                       s->s->st));
    std::string d((const char*)domain, dlen);
    return emit(s->ctx, s->s->prove(nullptr, s->s->records_buf, n, d, false, &ends), out, cap, out_len);
  });
}

int flock_keccak_prove_chain(flock_setup* s, const flock_keccak_state* states, size_t n, const uint8_t* domain,
                             size_t dlen, uint8_t* out, size_t cap, size_t* out_len) {
  if (!s || !states || (!domain && dlen)) return FLOCK_ERR_ARG;
  if (s->s->hash != flock::kHashKeccak) {
    s->ctx->err = "not a Keccak setup (the 3-wide statement has no chains)";
    return FLOCK_ERR_ARG;
  }
  if (n != s->n_blocks || n != ((size_t)1 << s->s->n_log)) {
    s->ctx->err = "a chain fills every slot: expected the setup's n_keccaks, a power of two";
    return FLOCK_ERR_ARG;
  }
  return guard(s->ctx, [&] {
    // endpoints in the slot's physical order: bit z of lane l at 64 l + z
    // (state_to_phys_bits, keccak.rs:850-857), i.e. the 25 lanes as words
    flock::ChainEnds ends;
    memcpy(ends.in, states[0].lanes, 200);
    uint64_t last[25];
    memcpy(last, states[n - 1].lanes, 200);
    flock::keccak_f(last);
    memcpy(ends.out, last, 200);
    if (!s->s->records_buf)
      CK(cudaMallocAsync(reinterpret_cast<void**>(&s->s->records_buf), n * sizeof(flock_keccak_state), s->s->st));
    CK(cudaMemcpyAsync(s->s->records_buf, states, n * sizeof(flock_keccak_state), cudaMemcpyHostToDevice, s->s->st));
    std::string d((const char*)domain, dlen);
    return emit(s->ctx, s->s->prove(nullptr, s->s->records_buf, n, d, false, &ends), out, cap, out_len);
  });
}

int flock_keccak_chain_states(const uint64_t* initial, size_t steps, flock_keccak_state* out) {
  if (!out && steps) return FLOCK_ERR_ARG;
  uint64_t cur[25] = {};
  if (initial) memcpy(cur, initial, sizeof(cur));
  for (size_t i = 0; i < steps; i++) {
    memcpy(out[i].lanes, cur, sizeof(cur));
    flock::keccak_f(cur);
  }
  return FLOCK_OK;
}

int flock_sha256_chain_blocks(uint64_t seed, const uint32_t* initial_h, size_t steps, flock_sha256_compression* out) {
  if (!out && steps) return FLOCK_ERR_ARG;
  static const uint32_t iv[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  uint32_t h[8];
  memcpy(h, initial_h ? initial_h : iv, sizeof(h));
  uint64_t x = seed;
  for (size_t i = 0; i < steps; i++) {
    memcpy(out[i].h, h, 32);
    for (int w = 0; w < 16; w++) {
      x += 0x9E3779B97F4A7C15ull;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      out[i].m[w] = (uint32_t)(z ^ (z >> 31));
    }
    flock::sha256_compress(out[i].h, out[i].m, h);
  }
  return FLOCK_OK;
}

int flock_verify(flock_setup* s, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen) {
  if (!s || !bytes || (!domain && dlen)) return FLOCK_ERR_ARG;
  return guard(s->ctx, [&] {
    const std::string why = s->s->verify(bytes, len, std::string((const char*)domain, dlen));
    if (why.empty()) return (int)FLOCK_OK;
    s->ctx->err = "verify: " + why;
    return (int)FLOCK_ERR_VERIFY;
  });
}

int flock_verify_bundle(flock_ctx* c, const uint8_t* bytes, size_t len, const uint8_t* domain, size_t dlen) {
  if (!c || !bytes || (!domain && dlen)) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    std::lock_guard<std::mutex> lk(c->vmu);
    if (!c->verifier) c->verifier.reset(new flock::Verifier(c->device));
    const std::string why = c->verifier->verify(bytes, len, std::string((const char*)domain, dlen), flock::kHashBlake3,
                                                nullptr, c->fs_fn);
    if (why.empty()) return (int)FLOCK_OK;
    c->err = "verify: " + why;
    return (int)FLOCK_ERR_VERIFY;
  });
}

int flock_serve_verify(flock_ctx* c, int on) {
  if (!c) return FLOCK_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  if (!c->server) {
    c->err = "serving not started";
    return FLOCK_ERR_ARG;
  }
  c->server->set_verify(on != 0);
  return FLOCK_OK;
}

int flock_chain_blocks(uint64_t seed, const uint32_t* initial_cv, size_t steps, uint32_t* records) {
  if (!records && steps) return FLOCK_ERR_ARG;
  uint32_t cv[8];
  memcpy(cv, initial_cv ? initial_cv : flock::kB3IV, sizeof(cv));
  uint64_t x = seed;
  for (size_t i = 0; i < steps; i++) {
    uint32_t* r = records + 28 * i;
    memcpy(r, cv, 32);
    for (int w = 0; w < 16; w++) {
      x += 0x9E3779B97F4A7C15ull;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      r[8 + w] = (uint32_t)(z ^ (z >> 31));
    }
    r[24] = r[25] = 0;  // counter
    r[26] = 64;         // block_len
    r[27] = 0;          // flags
    uint32_t st16[16];
    flock::b3_compress(r, r + 8, 0, 64, 0, st16);
    memcpy(cv, st16, 32);
  }
  return FLOCK_OK;
}

int flock_host_alloc(size_t bytes, void** out) {
  if (!out || bytes == 0) return FLOCK_ERR_ARG;
  *out = nullptr;
  return cudaMallocHost(out, bytes) == cudaSuccess ? FLOCK_OK : FLOCK_ERR_CUDA;
}
void flock_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

int flock_serve_prewarm(flock_ctx* c, uint32_t log2_n, int count, int* cached) {
  if (!c || log2_n < 8 || log2_n > 20 || count < 0) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->server) {
      c->err = "serving not started";
      return (int)FLOCK_ERR_ARG;
    }
    const int n = c->server->prewarm(log2_n, count);
    if (cached) *cached = n;
    return (int)FLOCK_OK;
  });
}

int flock_serve_start(flock_ctx* c, int slots) {
  if (!c || slots < 1 || slots > 64) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->server) {
      c->err = "serving already started";
      return FLOCK_ERR_ARG;
    }
    uint64_t budget = c->budget;
    if (!budget) {  // default: the device's free memory less 4 GiB of headroom
      size_t free_b = 0, total_b = 0;
      CK(cudaSetDevice(c->device));
      CK(cudaMemGetInfo(&free_b, &total_b));
      budget = free_b > ((size_t)4 << 30) ? free_b - ((size_t)4 << 30) : free_b / 2;
    }
    c->server.reset(new flock::Server(c->device, budget, slots));
    return FLOCK_OK;
  });
}

int flock_submit(flock_ctx* c, const flock_job* job, uint64_t* ticket) {
  if (!c || !job || !ticket || (!job->domain && job->dlen)) return FLOCK_ERR_ARG;
  if (job->log2_n < 8 || job->log2_n > 20) {
    c->err = "unsupported job size (log2 in 8..=20)";
    return FLOCK_ERR_ARG;
  }
  if (!c->server) {
    int rc = flock_serve_start(c, 4);
    if (rc && !c->server) return rc;
  }
  return guard(c, [&] {
    std::string d((const char*)job->domain, job->dlen);
    *ticket = c->server->submit(job->log2_n, job->seed, job->blocks, d);
    return FLOCK_OK;
  });
}

int flock_poll(flock_ctx* c, uint64_t ticket, flock_result* res, int timeout_ms) {
  if (!c || !res) return FLOCK_ERR_ARG;
  if (!c->server) {
    c->err = "serving not started";
    return FLOCK_ERR_ARG;
  }
  return guard(c, [&] {
    const size_t len = c->server->peek_len(ticket);
    if (len && (len > res->cap || !res->out)) {  // keep the result: the caller retries with room
      res->out_len = len;
      c->err = "output buffer too small";
      return FLOCK_ERR_CAPACITY;
    }
    flock::JobResult r;
    if (!c->server->wait(ticket, timeout_ms, &r)) return FLOCK_ERR_TIMEOUT;
    res->status = r.status;
    res->queue_ms = r.queue_ms;
    res->run_ms = r.run_ms;
    res->latency_ms = r.latency_ms;
    res->out_len = r.bytes.size();
    if (r.status != FLOCK_OK) {
      c->err = r.error;
      return FLOCK_OK;
    }
    if (r.bytes.size() > res->cap || !res->out) {
      c->err = "output buffer too small (the proof was dropped)";
      return FLOCK_ERR_CAPACITY;
    }
    memcpy(res->out, r.bytes.data(), r.bytes.size());
    return FLOCK_OK;
  });
}

int flock_prove_batch(flock_ctx* c, const flock_job* jobs, size_t n, flock_result* results, int threads) {
  if (!c || (n && (!jobs || !results)) || threads < 1 || threads > 64) return FLOCK_ERR_ARG;
  for (size_t i = 0; i < n; i++)
    if (jobs[i].log2_n < 8 || jobs[i].log2_n > 20 || (!jobs[i].domain && jobs[i].dlen)) {
      c->err = "unsupported job (log2 in 8..=20)";
      return FLOCK_ERR_ARG;
    }
  if (!c->server) {
    int rc = flock_serve_start(c, 4);
    if (rc && !c->server) return rc;
  }
  return guard(c, [&] {
    std::vector<flock::Server::BatchItem> items(n);
    for (size_t i = 0; i < n; i++) {
      items[i].log2 = jobs[i].log2_n;
      items[i].seed = jobs[i].seed;
      items[i].blocks = jobs[i].blocks;
      items[i].domain.assign((const char*)jobs[i].domain, jobs[i].dlen);
    }
    std::vector<flock::JobResult> rs = c->server->prove_batch(items, threads);
    int rc = FLOCK_OK;
    for (size_t i = 0; i < n; i++) {
      flock_result& o = results[i];
      const flock::JobResult& r = rs[i];
      o.status = r.status;
      o.queue_ms = r.queue_ms;
      o.run_ms = r.run_ms;
      o.latency_ms = r.latency_ms;
      o.out_len = r.bytes.size();
      if (r.status != FLOCK_OK) {
        c->err = r.error;
        continue;
      }
      if (r.bytes.size() > o.cap || !o.out) {
        o.status = FLOCK_ERR_CAPACITY;
        c->err = "output buffer too small";
        rc = FLOCK_ERR_CAPACITY;
        continue;
      }
      memcpy(o.out, r.bytes.data(), r.bytes.size());
    }
    return rc;
  });
}

int flock_statement_digest(uint32_t m, uint8_t* out32) {
  if (!out32 || m < 17 || m > 40) return FLOCK_ERR_ARG;
  try {
    auto d = flock::statement_digest((int)m);
    memcpy(out32, d.data(), 32);
    return FLOCK_OK;
  } catch (...) {
    return FLOCK_ERR_INTERNAL;
  }
}

int flock_setup_phase_ms(flock_setup* s, double* ms, int n) {
  if (!s || !ms) return 0;
  double t[flock::Setup::kPhases];
  s->s->phase_times(t);
  int k = n < flock::Setup::kPhases ? n : flock::Setup::kPhases;
  for (int i = 0; i < k; i++) ms[i] = t[i];
  return k;
}

int flock_witness(flock_ctx* c, uint32_t log2, uint64_t seed, uint64_t* z, uint64_t* a, uint64_t* b) {
  if (!c || !z || !a || !b || log2 > 24) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    uint32_t slots = 1u << (log2 < 3 ? 3 : log2);
    size_t words = (size_t)slots * 128;
    DevBuf<f128> dz(words), da(words), db(words);
    launch_witness_seed(seed, log2, 1u << log2, slots, dz.p, da.p, db.p, c->st);
    CK(cudaMemcpyAsync(z, dz.p, words * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(a, da.p, words * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(b, db.p, words * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return FLOCK_OK;
  });
}

int flock_ntt_rs_encode(flock_ctx* c, const uint64_t* msg, uint32_t log_msg_pos, uint32_t lanes, uint32_t rate,
                        uint64_t* out) {
  if (!c || !msg || !out || lanes == 0 || (lanes & (lanes - 1)) || log_msg_pos + rate > 30 || rate < 1)
    return FLOCK_ERR_ARG;
  return guard(c, [&] {
    size_t n = ((size_t)lanes) << log_msg_pos, nc = n << rate;
    DevBuf<f128> dm(n), dc(nc);
    CK(cudaMemcpyAsync(dm.p, msg, n * 16, cudaMemcpyHostToDevice, c->st));
    ntt_rs_encode(dm.p, dc.p, (int)log_msg_pos, (int)lanes, (int)rate, c->st);
    CK(cudaMemcpyAsync(out, dc.p, nc * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return FLOCK_OK;
  });
}

int flock_ntt_rs_encode_plan(flock_ctx* c, const uint64_t* msg, uint32_t log_msg_pos, uint32_t lanes,
                             uint32_t rate, uint32_t plan_index, uint64_t* out) {
  if (!c || !msg || !out || lanes == 0 || (lanes & (lanes - 1)) || log_msg_pos + rate > 30 || rate < 1)
    return FLOCK_ERR_ARG;
  if (plan_index >= ntt_plan_count((int)(log_msg_pos + rate), (int)lanes, (int)rate)) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    size_t n = ((size_t)lanes) << log_msg_pos, nc = n << rate;
    DevBuf<f128> dm(n), dc(nc);
    CK(cudaMemcpyAsync(dm.p, msg, n * 16, cudaMemcpyHostToDevice, c->st));
    ntt_rs_encode_plan(dm.p, dc.p, (int)log_msg_pos, (int)lanes, (int)rate, plan_index, c->st);
    CK(cudaMemcpyAsync(out, dc.p, nc * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return FLOCK_OK;
  });
}

int flock_ntt_autotune(flock_ctx* c, uint32_t log_msg_pos, uint32_t lanes, uint32_t rate, double* best_ms,
                       char* desc, size_t desc_cap) {
  if (!c || lanes == 0 || (lanes & (lanes - 1)) || log_msg_pos + rate > 30 || rate < 1) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    const int log_d = (int)(log_msg_pos + rate);
    NttPlan plan = ntt_plan(log_d, (int)lanes, (int)rate);
    double ms = -1;
    {
      DevBuf<f128> dc(((size_t)lanes) << log_d);
      plan = ntt_autotune(dc.p, log_d, (int)lanes, (int)rate, c->st, &ms);
    }
    if (best_ms) *best_ms = ms;
    if (desc && desc_cap) {
      std::string d = ntt_plan_desc(plan);
      std::snprintf(desc, desc_cap, "%s", d.c_str());
    }
    return FLOCK_OK;
  });
}

int flock_merkle_tree(flock_ctx* c, const uint8_t* data, size_t n_leaves, size_t leaf_size, uint8_t* tree_out) {
  return flock_merkle_tree_hash(c, data, n_leaves, leaf_size, FLOCK_HASH_BLAKE3, tree_out);
}

int flock_merkle_tree_hash(flock_ctx* c, const uint8_t* data, size_t n_leaves, size_t leaf_size, int hash,
                           uint8_t* tree_out) {
  if (!c || !data || !tree_out || n_leaves == 0 || (n_leaves & (n_leaves - 1)) || leaf_size == 0 ||
      leaf_size > 1024 || (leaf_size % 16) || (hash != FLOCK_HASH_SHA256 && hash != FLOCK_HASH_BLAKE3))
    return FLOCK_ERR_ARG;
  return guard(c, [&] {
    DevBuf<uint8_t> dd(n_leaves * leaf_size);
    DevBuf<uint32_t> dt(8 * (2 * n_leaves - 1));
    CK(cudaMemcpyAsync(dd.p, data, n_leaves * leaf_size, cudaMemcpyHostToDevice, c->st));
    merkle_build(dd.p, n_leaves, leaf_size, dt.p, hash, c->st);
    CK(cudaMemcpyAsync(tree_out, dt.p, (2 * n_leaves - 1) * 32, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return FLOCK_OK;
  });
}

int flock_sumcheck_round(flock_ctx* c, const uint64_t* f, const uint64_t* b, size_t n, uint64_t* msg_out) {
  if (!c || !f || !b || !msg_out || n < 2 || (n & (n - 1))) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    DevBuf<f128> df(n), db(n), dout(2);
    CK(cudaMemcpyAsync(df.p, f, n * 16, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(db.p, b, n * 16, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemsetAsync(dout.p, 0, 32, c->st));
    lig_msg(df.p, db.p, n / 2, dout.p, c->sms, c->st);
    CK(cudaMemcpyAsync(msg_out, dout.p, 32, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return FLOCK_OK;
  });
}

int flock_sumcheck_round3(flock_ctx* c, const uint64_t* e, const uint64_t* a, const uint64_t* b, size_t n,
                          const uint64_t* rho, uint64_t* a_out, uint64_t* b_out, uint64_t* msg_out) {
  const size_t min_n = rho ? 4 : 2;
  if (!c || !e || !a || !b || !msg_out || n < min_n || (n & (n - 1)) || (rho && (!a_out || !b_out)))
    return FLOCK_ERR_ARG;
  return guard(c, [&] {
    const size_t n_pairs = rho ? n / 4 : n / 2;
    DevBuf<f128> da(n), db(n), de(n_pairs), dao(n / 2), dbo(n / 2), dout(2);
    CK(cudaMemcpyAsync(da.p, a, n * 16, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(db.p, b, n * 16, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(de.p, e, n_pairs * 16, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemsetAsync(dout.p, 0, 32, c->st));
    f128 r = rho ? mk(rho[0], rho[1]) : mk(0, 0);
    sc3_round(da.p, db.p, de.p, dao.p, dbo.p, rho ? &r : nullptr, n_pairs, dout.p, 148 * 4, c->st);
    CK(cudaMemcpyAsync(msg_out, dout.p, 32, cudaMemcpyDeviceToHost, c->st));
    if (rho) {
      CK(cudaMemcpyAsync(a_out, dao.p, n / 2 * 16, cudaMemcpyDeviceToHost, c->st));
      CK(cudaMemcpyAsync(b_out, dbo.p, n / 2 * 16, cudaMemcpyDeviceToHost, c->st));
    }
    CK(cudaStreamSynchronize(c->st));
    return FLOCK_OK;
  });
}

int flock_pow(flock_ctx* c, const uint8_t* digest32, uint32_t bits, uint64_t* nonce) {
  if (!c || !digest32 || !nonce || bits > 40) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    DevBuf<unsigned long long> d(1);
    unsigned long long* h = nullptr;
    CK(cudaMallocHost(&h, 8));
    *nonce = pow_search(digest32, bits, c->st, d.p, h);
    cudaFreeHost(h);
    return FLOCK_OK;
  });
}

int flock_f128_mul(flock_ctx* c, const uint64_t* a, const uint64_t* b, size_t n, uint64_t* out) {
  if (!c || !a || !b || !out) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    DevBuf<f128> da(n), db(n), dout(n);
    CK(cudaMemcpyAsync(da.p, a, n * 16, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(db.p, b, n * 16, cudaMemcpyHostToDevice, c->st));
    k_mul<<<(unsigned)((n + 255) / 256), 256, 0, c->st>>>(da.p, db.p, n, dout.p);
    CK(cudaMemcpyAsync(out, dout.p, n * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return FLOCK_OK;
  });
}

}  // extern "C"

template <class F>
static double time_launches(cudaStream_t st, int iters, F&& f) {
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  f();
  CK(cudaStreamSynchronize(st));
  CK(cudaEventRecord(e0, st));
  for (int i = 0; i < iters; i++) f();
  CK(cudaEventRecord(e1, st));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms / iters;
}

extern "C" {

int flock_bench_ntt(flock_ctx* c, uint32_t log_msg_pos, uint32_t lanes, uint32_t rate, int iters, double* ms) {
  if (!c || !ms || iters < 1 || lanes == 0 || rate < 1) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    size_t n = ((size_t)lanes) << log_msg_pos, nc = n << rate;
    DevBuf<f128> dm(n), dc(nc);
    ntt_autotune(dc.p, (int)(log_msg_pos + rate), (int)lanes, (int)rate, c->st);
    k_fill<<<(unsigned)((2 * n + 255) / 256), 256, 0, c->st>>>((uint64_t*)dm.p, 2 * n, 1);
    *ms = time_launches(c->st, iters, [&] { ntt_rs_encode(dm.p, dc.p, (int)log_msg_pos, (int)lanes, (int)rate, c->st); });
    return FLOCK_OK;
  });
}

int flock_ntt_plan_desc(uint32_t log_msg_pos, uint32_t lanes, uint32_t rate, uint32_t plan_index, char* desc,
                        size_t desc_cap) {
  if (!desc || !desc_cap || lanes == 0 || (lanes & (lanes - 1)) || log_msg_pos + rate > 30 || rate < 1)
    return FLOCK_ERR_ARG;
  try {
    const std::string d = ntt_plan_desc_at((int)(log_msg_pos + rate), (int)lanes, (int)rate, plan_index);
    if (d.empty()) return FLOCK_ERR_ARG;
    std::snprintf(desc, desc_cap, "%s", d.c_str());
  } catch (...) {
    return FLOCK_ERR_INTERNAL;
  }
  return FLOCK_OK;
}

int flock_bench_ntt_plan(flock_ctx* c, uint32_t log_msg_pos, uint32_t lanes, uint32_t rate, uint32_t plan_index,
                         int iters, double* ms) {
  if (!c || !ms || iters < 1 || lanes == 0 || (lanes & (lanes - 1)) || rate < 1 || log_msg_pos + rate > 30)
    return FLOCK_ERR_ARG;
  if (plan_index >= ntt_plan_count((int)(log_msg_pos + rate), (int)lanes, (int)rate)) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    size_t n = ((size_t)lanes) << log_msg_pos, nc = n << rate;
    DevBuf<f128> dm(n), dc(nc);
    k_fill<<<(unsigned)((2 * n + 255) / 256), 256, 0, c->st>>>((uint64_t*)dm.p, 2 * n, 1);
    *ms = time_launches(c->st, iters, [&] {
      ntt_rs_encode_plan(dm.p, dc.p, (int)log_msg_pos, (int)lanes, (int)rate, plan_index, c->st);
    });
    return FLOCK_OK;
  });
}

uint64_t flock_launch_count(void) { return kernel_launch_counter().load(); }

int flock_bench_f128_product(flock_ctx* c, int variant, int iters, double* products_per_s) {
  if (!c || !products_per_s || variant < 0 || variant > 3 || iters < 1) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const unsigned blocks = (unsigned)sms * 8;
    const size_t smem = variant == 3 ? sizeof(MulTab8) : 8 * kTab4Bytes;
    DevBuf<f128> tw(1024), out((size_t)blocks * 256);
    k_fill<<<8, 256, 0, c->st>>>((uint64_t*)tw.p, 2048, 3);
    auto kern = variant == 0   ? k_bench_product<0>
                : variant == 1 ? k_bench_product<1>
                : variant == 2 ? k_bench_product<2>
                               : k_bench_product<3>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const double ms = time_launches(c->st, 3, [&] {
      count_launch();
      kern<<<blocks, 256, smem, c->st>>>(tw.p, out.p, iters);
    });
    *products_per_s = (double)blocks * 256 * 4 * iters / (ms * 1e-3);
    return FLOCK_OK;
  });
}

int flock_bench_merkle(flock_ctx* c, size_t n_leaves, size_t leaf_size, int iters, double* ms) {
  if (!c || !ms || iters < 1 || leaf_size % 16 || leaf_size > 1024) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    DevBuf<uint8_t> dd(n_leaves * leaf_size);
    DevBuf<uint32_t> dt(8 * (2 * n_leaves - 1));
    size_t words = n_leaves * leaf_size / 8;
    k_fill<<<(unsigned)((words + 255) / 256), 256, 0, c->st>>>((uint64_t*)dd.p, words, 2);
    *ms = time_launches(c->st, iters, [&] { merkle_build(dd.p, n_leaves, leaf_size, dt.p, c->st); });
    return FLOCK_OK;
  });
}

int flock_bench_prove(flock_setup* s, uint64_t seed0, int steps, double* total_ms, double* phase_ms,
                      uint64_t* launches) {
  if (!s || steps < 1 || !total_ms) return FLOCK_ERR_ARG;
  return guard(s->ctx, [&] {
    flock::Setup& S = *s->s;
    double acc[flock::Setup::kPhases] = {0};
    uint64_t l0 = kernel_launch_counter();
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaStreamSynchronize(S.st));
    CK(cudaEventRecord(e0, S.st));
    for (int i = 0; i < steps; i++) {
      S.prove(&seed0, nullptr, 0, "flock-bench-v0");
      seed0++;
      double t[flock::Setup::kPhases];
      S.phase_times(t);
      for (int k = 0; k < flock::Setup::kPhases; k++) acc[k] += t[k];
    }
    CK(cudaEventRecord(e1, S.st));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *total_ms = ms;
    if (phase_ms)
      for (int k = 0; k < flock::Setup::kPhases; k++) phase_ms[k] = acc[k] / steps;
    if (launches) *launches = kernel_launch_counter() - l0;
    return FLOCK_OK;
  });
}

int flock_bench_sumcheck(flock_ctx* c, size_t n, int iters, double* ms) {
  if (!c || !ms || iters < 1 || n < 4) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    DevBuf<f128> df(n), db(n), fo(n / 2), bo(n / 2), dout(2);
    k_fill<<<(unsigned)((2 * n + 255) / 256), 256, 0, c->st>>>((uint64_t*)df.p, 2 * n, 3);
    k_fill<<<(unsigned)((2 * n + 255) / 256), 256, 0, c->st>>>((uint64_t*)db.p, 2 * n, 4);
    f128 r = mk(0x1234567890abcdefull, 0x0fedcba987654321ull);
    *ms = time_launches(c->st, iters, [&] {
      lig_fold_msg(df.p, db.p, fo.p, bo.p, r, n / 4, true, dout.p, c->sms, c->st);
    });
    return FLOCK_OK;
  });
}

int flock_bench_sumcheck3(flock_ctx* c, size_t n, int iters, double* ms) {
  if (!c || !ms || iters < 1 || n < 4 || (n & (n - 1))) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    DevBuf<f128> da(n), db(n), de(n / 4), dao(n / 2), dbo(n / 2), dout(2);
    k_fill<<<(unsigned)((2 * n + 255) / 256), 256, 0, c->st>>>((uint64_t*)da.p, 2 * n, 5);
    k_fill<<<(unsigned)((2 * n + 255) / 256), 256, 0, c->st>>>((uint64_t*)db.p, 2 * n, 6);
    k_fill<<<(unsigned)((n / 2 + 255) / 256), 256, 0, c->st>>>((uint64_t*)de.p, n / 2, 7);
    f128 r = mk(0x1234567890abcdefull, 0x0fedcba987654321ull);
    *ms = time_launches(c->st, iters, [&] { sc3_round(da.p, db.p, de.p, dao.p, dbo.p, &r, n / 4, dout.p, 148 * 4, c->st); });
    return FLOCK_OK;
  });
}

// ---- degree-4 zerocheck round 1 (zerocheck/univariate_skip_deg4.rs)
namespace {
// eq(r, .) over n <= 30 variables on the device, low variables first
void eq_device(const f128* r, int n, f128* lo, f128* hi, f128* out, cudaStream_t st) {
  const int s = std::min(n, 12);
  eq_build(r, s, flock::hone(), lo, st);
  eq_build(r + s, n - s, flock::hone(), hi, st);
  eq_split(lo, hi, s, (size_t)1 << n, out, st);
}
struct Deg4Bufs {
  size_t rows;
  DevBuf<uint64_t> v;  // a, b, c, d, z rows
  DevBuf<f128> eq, lo, hi, sums;  // sums: H (1536) then Zs (64)
  DevBuf<uint8_t> tab;
  explicit Deg4Bufs(uint32_t m)
      : rows((size_t)1 << (m - 6)), v(5 * rows), eq(rows), lo(1 << 12), hi(std::max<size_t>(1, rows >> 12)),
        sums(1600), tab(deg4_tables_bytes()) {}
  void run(const std::vector<f128>& r, int m, int sms, cudaStream_t st) {
    eq_device(r.data() + 6, m - 6, lo.p, hi.p, eq.p, st);
    CK(cudaMemsetAsync(sums.p, 0, 1600 * sizeof(f128), st));
    round1_deg4(v.p, v.p + rows, v.p + 2 * rows, v.p + 3 * rows, v.p + 4 * rows, eq.p, rows, tab.p, sums.p,
                sums.p + 1536, 2 * sms, st);
  }
  void finish(uint64_t* p_abcd, uint64_t* p_z, cudaStream_t st) {
    std::vector<f128> h(1600);
    CK(cudaMemcpyAsync(h.data(), sums.p, 1600 * sizeof(f128), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    round1_deg4_finish(h.data(), h.data() + 1536, reinterpret_cast<f128*>(p_abcd), reinterpret_cast<f128*>(p_z));
  }
};
int sm_count(int device) {
  int n = 0;
  CK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device));
  return n;
}
std::vector<uint8_t> deg4_host_tables() {
  std::vector<uint8_t> t(deg4_tables_bytes());
  deg4_build_tables(t.data());
  return t;
}
}  // namespace

int flock_zerocheck_round1_deg4(flock_ctx* c, const uint64_t* a, const uint64_t* b, const uint64_t* cc,
                                const uint64_t* d, const uint64_t* z, uint32_t m, const uint64_t* r, uint64_t* p_abcd,
                                uint64_t* p_z) {
  if (!c || !a || !b || !cc || !d || !z || !r || !p_abcd || !p_z) return FLOCK_ERR_ARG;
  if (m < 6 || m > 30) {
    c->err = "round1_deg4: m must be in 6..=30";
    return FLOCK_ERR_ARG;
  }
  return guard(c, [&] {
    DeviceScope on(c->device);
    Deg4Bufs B(m);
    const uint64_t* in[5] = {a, b, cc, d, z};
    for (int f = 0; f < 5; f++)
      CK(cudaMemcpyAsync(B.v.p + f * B.rows, in[f], B.rows * 8, cudaMemcpyHostToDevice, c->st));
    static const std::vector<uint8_t> tabs = deg4_host_tables();
    CK(cudaMemcpyAsync(B.tab.p, tabs.data(), tabs.size(), cudaMemcpyHostToDevice, c->st));
    std::vector<f128> rv(m);
    memcpy(rv.data(), r, m * sizeof(f128));
    B.run(rv, (int)m, sm_count(c->device), c->st);
    B.finish(p_abcd, p_z, c->st);
    return FLOCK_OK;
  });
}

int flock_bench_round1_deg4(flock_ctx* c, uint32_t m, uint64_t seed, int iters, double* ms, uint64_t* p_abcd,
                            uint64_t* p_z) {
  if (!c || !ms || iters < 1 || m < 6 || m > 30) return FLOCK_ERR_ARG;
  return guard(c, [&] {
    DeviceScope on(c->device);
    Deg4Bufs B(m);
    k_fill<<<(unsigned)((5 * B.rows + 255) / 256), 256, 0, c->st>>>(B.v.p, 5 * B.rows, seed);
    static const std::vector<uint8_t> tabs = deg4_host_tables();
    CK(cudaMemcpyAsync(B.tab.p, tabs.data(), tabs.size(), cudaMemcpyHostToDevice, c->st));
    // r: SplitMix64 from seed ^ 1, lo then hi per value
    std::vector<f128> rv(m);
    uint64_t st = seed ^ 1;
    auto nx = [&] {
      st += 0x9E3779B97F4A7C15ull;
      uint64_t x = st;
      x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
      x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
      return x ^ (x >> 31);
    };
    for (auto& v : rv) {
      v.lo = nx();
      v.hi = nx();
    }
    const int sms = sm_count(c->device);
    *ms = time_launches(c->st, iters, [&] { B.run(rv, (int)m, sms, c->st); });
    if (p_abcd && p_z) B.finish(p_abcd, p_z, c->st);
    return FLOCK_OK;
  });
}

}  // extern "C"
