// K2: BLAKE3 Merkle trees (leaves, parent levels, multi-proof gathers) and
// K9: proof-of-work nonce search.
//
// Tree semantics: crates/flock-core/src/merkle.rs — flat 2n-1 layout
// (:16-21), leaf = non-root BLAKE3 chaining value of the leaf bytes (one
// chunk: blocks chained from the IV, CHUNK_START on the first, CHUNK_END on
// the last, counter 0, no ROOT; :192-197), parent = compress(IV, l||r,
// counter 0, 64, PARENT) (:199-203).  PoW: crates/flock-core/src/
// challenger.rs:384-475,549-600 — the smallest nonce n such that the root
// BLAKE3 hash of (state_digest || n_le || 0^24) has `bits` leading zero bits.
#include "kernels.cuh"
#include "sha256.cuh"
#include "host.hpp"

namespace {
// non-root chaining value of one leaf of leaf_size <= 1024 bytes (a single
// BLAKE3 chunk) into out (8 words)
__device__ __forceinline__ void leaf_cv(const uint8_t* __restrict__ p, size_t leaf_size, uint32_t* __restrict__ out) {
  uint32_t cv[8];
#pragma unroll
  for (int k = 0; k < 8; k++) cv[k] = b3d::kIV[k];
  size_t nblk = leaf_size == 0 ? 1 : (leaf_size + 63) / 64;
  for (size_t blk = 0; blk < nblk; blk++) {
    uint32_t m[16];
    size_t off = blk * 64, len = leaf_size - off < 64 ? leaf_size - off : 64;
    if (len == 64 && (((uintptr_t)(p + off)) & 15) == 0) {
      const uint4* q = reinterpret_cast<const uint4*>(p + off);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        uint4 v = q[k];
        m[4 * k] = v.x; m[4 * k + 1] = v.y; m[4 * k + 2] = v.z; m[4 * k + 3] = v.w;
      }
    } else {
      uint8_t b[64];
      for (int k = 0; k < 64; k++) b[k] = (size_t)k < len ? p[off + k] : 0;
      for (int k = 0; k < 16; k++)
        m[k] = (uint32_t)b[4 * k] | (uint32_t)b[4 * k + 1] << 8 | (uint32_t)b[4 * k + 2] << 16 | (uint32_t)b[4 * k + 3] << 24;
    }
    uint32_t flags = (blk == 0 ? b3d::CHUNK_START : 0) | (blk + 1 == nblk ? b3d::CHUNK_END : 0);
    b3d::compress(cv, m, 0, (uint32_t)len, flags, cv);
  }
  uint4* o = reinterpret_cast<uint4*>(out);
  o[0] = make_uint4(cv[0], cv[1], cv[2], cv[3]);
  o[1] = make_uint4(cv[4], cv[5], cv[6], cv[7]);
}

// parent CV of the two child CVs at in (16 words) into out (8 words)
__device__ __forceinline__ void parent_cv(const uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
  const uint4* q = reinterpret_cast<const uint4*>(in);
  uint32_t m[16];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint4 v = q[k];
    m[4 * k] = v.x; m[4 * k + 1] = v.y; m[4 * k + 2] = v.z; m[4 * k + 3] = v.w;
  }
  uint32_t cv[8];
  b3d::compress(b3d::kIV, m, 0, 64, b3d::PARENT, cv);
  uint4* o = reinterpret_cast<uint4*>(out);
  o[0] = make_uint4(cv[0], cv[1], cv[2], cv[3]);
  o[1] = make_uint4(cv[4], cv[5], cv[6], cv[7]);
}

// upper levels of one tree inside one CTA (levels of at most 1024 nodes);
// each level is read back from global memory after the barrier that
// published it
__device__ __forceinline__ void tree_top(uint32_t* tree, size_t level_start, size_t level_len) {
  int t = threadIdx.x;
  size_t len = level_len, start = level_start;
  while (len > 1) {
    size_t n = len >> 1;
    for (size_t i = t; i < n; i += blockDim.x) {
      uint32_t m[16], cv[8];
      for (int k = 0; k < 16; k++) m[k] = tree[(start + 2 * i) * 8 + k];
      b3d::compress(b3d::kIV, m, 0, 64, b3d::PARENT, cv);
      for (int k = 0; k < 8; k++) tree[(start + len + i) * 8 + k] = cv[k];
    }
    __syncthreads();
    start += len;
    len = n;
  }
}

// the job of global index i of a batched launch: the last job whose first
// index (at member offset `field`) is <= i
template <class F>
__device__ __forceinline__ int find_job(const BatchJob* __restrict__ jobs, int n_jobs, uint64_t i, F first) {
  int lo = 0, hi = n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first(jobs[mid]) <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
}  // namespace

// one thread per leaf
__global__ void k_merkle_leaves(const uint8_t* __restrict__ data, size_t leaf_size, size_t n_leaves,
                                uint32_t* __restrict__ tree) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_leaves) return;
  leaf_cv(data + i * leaf_size, leaf_size, tree + 8 * i);
}

// leaf chaining values only (no tree): out[8 i..8 i + 8) for leaf i
void merkle_leaves(const void* data, size_t n_leaves, size_t leaf_size, uint32_t* out, cudaStream_t s) {
  count_launch();
  k_merkle_leaves<<<(unsigned)((n_leaves + 127) / 128), 128, 0, s>>>((const uint8_t*)data, leaf_size, n_leaves, out);
}

// the 1 KiB-leaf trees of every job of a batch (leaves, then one parent
// level for all jobs per launch, then one CTA per job for its top levels)
__global__ void k_merkle_leaves_batch(const BatchJob* __restrict__ jobs, int n_jobs, uint64_t total) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const BatchJob& J = jobs[find_job(jobs, n_jobs, i, [](const BatchJob& b) { return b.leaf0; })];
  const uint64_t k = i - J.leaf0;
  leaf_cv(reinterpret_cast<const uint8_t*>(J.cw) + k * 1024, 1024, J.tree + 8 * k);
}
__global__ void k_merkle_parents_batch(const BatchJob* __restrict__ jobs, int n_jobs, int level, uint64_t total) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const BatchJob& J = jobs[find_job(jobs, n_jobs, i, [level](const BatchJob& b) { return b.par0[level]; })];
  const uint64_t k = i - J.par0[level];
  // level `level` starts after the leaves and the levels below it
  uint64_t start = 0, len = J.n_leaves;
  for (int l = 1; l < level; l++) { start += len; len >>= 1; }
  parent_cv(J.tree + 8 * (start + 2 * k), J.tree + 8 * (start + len + k));
}
__global__ void k_merkle_top_batch(const BatchJob* __restrict__ jobs) {
  const BatchJob& J = jobs[blockIdx.x];
  tree_top(J.tree, J.top_start, J.top_len);
}

__global__ void k_merkle_parents(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, size_t n_out) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_out) return;
  parent_cv(in + 16 * i, out + 8 * i);
}

__global__ void k_merkle_top(uint32_t* tree, size_t level_start, size_t level_len) {
  tree_top(tree, level_start, level_len);
}

void merkle_leaves_batch(const BatchJob* jobs, int n_jobs, uint64_t total, cudaStream_t s) {
  count_launch();
  k_merkle_leaves_batch<<<(unsigned)((total + 127) / 128), 128, 0, s>>>(jobs, n_jobs, total);
}
void merkle_parents_batch(const BatchJob* jobs, int n_jobs, int level, uint64_t total, cudaStream_t s) {
  count_launch();
  k_merkle_parents_batch<<<(unsigned)((total + 127) / 128), 128, 0, s>>>(jobs, n_jobs, level, total);
}
void merkle_top_batch(const BatchJob* jobs, int n_jobs, cudaStream_t s) {
  count_launch();
  k_merkle_top_batch<<<n_jobs, 512, 0, s>>>(jobs);
}

// ---- SHA-256 trees (merkle.rs:205-230): leaf = SHA256(leaf bytes),
// parent = SHA256(left || right); digests stored as their 32 bytes
// (big-endian words).  Leaf sizes are multiples of 4 bytes.
__global__ void k_merkle_leaves_sha(const uint8_t* __restrict__ data, size_t leaf_size, size_t n_leaves,
                                    uint32_t* __restrict__ tree) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_leaves) return;
  const uint32_t* d = reinterpret_cast<const uint32_t*>(data + i * leaf_size);
  uint32_t st[8], w[16];
#pragma unroll
  for (int k = 0; k < 8; k++) st[k] = sha_d::kIV[k];
  const size_t full = leaf_size / 64, rem_words = (leaf_size % 64) / 4;
  for (size_t b = 0; b < full; b++) {
#pragma unroll
    for (int k = 0; k < 16; k++) w[k] = sha_d::bswap(__ldg(d + 16 * b + k));
    sha_d::compress(st, w);
  }
#pragma unroll
  for (int k = 0; k < 16; k++) w[k] = (size_t)k < rem_words ? sha_d::bswap(__ldg(d + 16 * full + k)) : 0u;
  w[rem_words] = 0x80000000u;
  const uint64_t bits = (uint64_t)leaf_size * 8;
  if (rem_words >= 14) {
    sha_d::compress(st, w);
#pragma unroll
    for (int k = 0; k < 16; k++) w[k] = 0;
  }
  w[14] = (uint32_t)(bits >> 32);
  w[15] = (uint32_t)bits;
  sha_d::compress(st, w);
#pragma unroll
  for (int k = 0; k < 8; k++) tree[8 * i + k] = sha_d::bswap(st[k]);
}

__global__ void k_merkle_parents_sha(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, size_t n_out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_out) return;
  uint32_t st[8], w[16];
#pragma unroll
  for (int k = 0; k < 8; k++) st[k] = sha_d::kIV[k];
#pragma unroll
  for (int k = 0; k < 16; k++) w[k] = sha_d::bswap(in[16 * i + k]);
  sha_d::compress(st, w);
#pragma unroll
  for (int k = 0; k < 16; k++) w[k] = 0;
  w[0] = 0x80000000u;
  w[15] = 512;
  sha_d::compress(st, w);
#pragma unroll
  for (int k = 0; k < 8; k++) out[8 * i + k] = sha_d::bswap(st[k]);
}

void merkle_leaves(const void* data, size_t n_leaves, size_t leaf_size, uint32_t* out, int fn, cudaStream_t s) {
  if (fn != flock::kFnSha256) return merkle_leaves(data, n_leaves, leaf_size, out, s);
  count_launch();
  k_merkle_leaves_sha<<<(unsigned)((n_leaves + 127) / 128), 128, 0, s>>>((const uint8_t*)data, leaf_size, n_leaves,
                                                                         out);
}

void merkle_build(const void* data, size_t n_leaves, size_t leaf_size, uint32_t* tree, int fn, cudaStream_t s) {
  if (fn != flock::kFnSha256) return merkle_build(data, n_leaves, leaf_size, tree, s);
  merkle_leaves(data, n_leaves, leaf_size, tree, fn, s);
  for (size_t start = 0, len = n_leaves; len > 1; start += len, len >>= 1) {
    const size_t n = len >> 1;
    count_launch();
    k_merkle_parents_sha<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(tree + 8 * start, tree + 8 * (start + len), n);
  }
}

void merkle_build(const void* data, size_t n_leaves, size_t leaf_size, uint32_t* tree, cudaStream_t s) {
  count_launch(); k_merkle_leaves<<<(unsigned)((n_leaves + 127) / 128), 128, 0, s>>>((const uint8_t*)data, leaf_size, n_leaves, tree);
  size_t start = 0, len = n_leaves;
  while (len > 1024) {
    size_t n = len >> 1;
    count_launch(); k_merkle_parents<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(tree + 8 * start, tree + 8 * (start + len), n);
    start += len;
    len = n;
  }
  if (len > 1) count_launch(), k_merkle_top<<<1, 512, 0, s>>>(tree, start, len);
}

std::vector<uint64_t> multiproof_ids(const std::vector<size_t>& q, size_t n_leaves) {
  std::vector<uint64_t> ids(q.begin(), q.end());
  std::vector<size_t> act(q);
  size_t ls = 0, ll = n_leaves;  // first index and width of the current level
  while (ll > 1) {
    size_t w = 0, i = 0;
    while (i < act.size()) {
      const size_t p = act[i];
      if (i + 1 < act.size() && act[i + 1] == (p ^ 1)) i += 2;
      else { ids.push_back(ls + (p ^ 1)); i += 1; }
      act[w++] = p >> 1;
    }
    act.resize(w);
    ls += ll;
    ll >>= 1;
  }
  return ids;
}

__global__ void k_gather_nodes(const uint32_t* __restrict__ tree, const uint64_t* __restrict__ idx, size_t n,
                               uint32_t* __restrict__ out) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = 0; k < 8; k++) out[8 * i + k] = tree[idx[i] * 8 + k];
}

__global__ void k_gather_rows(const f128* __restrict__ cw, const uint64_t* __restrict__ pos, size_t n, int lanes,
                              f128* __restrict__ out) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * lanes) return;
  size_t q = i / lanes, l = i % lanes;
  st(out + i, ld(cw + pos[q] * lanes + l));
}

__global__ void k_scatter(f128* __restrict__ dst, const uint64_t* __restrict__ pos, const f128* __restrict__ vals,
                          size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) st(dst + pos[i], ld(vals + i));
}
namespace flock {
void scatter(f128* dst, const uint64_t* pos, const f128* vals, size_t n, cudaStream_t s) {
  if (n) count_launch(), k_scatter<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(dst, pos, vals, n);
}
}  // namespace flock

// ---------------------------------------------------------------- PoW --
__global__ void k_pow(uint4 d0, uint4 d1, uint32_t bits, uint64_t start, uint64_t count,
                      unsigned long long* __restrict__ found) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint64_t n = start + i;
  if (n >= *found) return;
  uint32_t m[16] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w, (uint32_t)n, (uint32_t)(n >> 32), 0, 0, 0, 0, 0, 0};
  uint32_t h[8];
  b3d::compress(b3d::kIV, m, 0, 64, b3d::CHUNK_START | b3d::CHUNK_END | b3d::ROOT, h);
  // leading zero bits of the 32-byte hash (byte order = LE words)
  uint32_t full = bits >> 3, extra = bits & 7;
  bool ok = true;
  for (uint32_t k = 0; k < full && ok; k++) ok = ((h[k >> 2] >> (8 * (k & 3))) & 0xFF) == 0;
  if (ok && extra) ok = ((((h[full >> 2] >> (8 * (full & 3))) & 0xFF) >> (8 - extra)) == 0);
  if (ok) atomicMin(found, (unsigned long long)n);
}

// SHA256(digest || nonce LE), one padded block (challenger.rs:589-595)
__global__ void k_pow_sha(uint4 d0, uint4 d1, uint32_t bits, uint64_t start, uint64_t count,
                          unsigned long long* __restrict__ found) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint64_t n = start + i;
  if (n >= *found) return;
  uint32_t w[16] = {sha_d::bswap(d0.x), sha_d::bswap(d0.y), sha_d::bswap(d0.z), sha_d::bswap(d0.w),
                    sha_d::bswap(d1.x), sha_d::bswap(d1.y), sha_d::bswap(d1.z), sha_d::bswap(d1.w),
                    sha_d::bswap((uint32_t)n), sha_d::bswap((uint32_t)(n >> 32)), 0x80000000u, 0, 0, 0, 0, 320};
  uint32_t st[8];
#pragma unroll
  for (int k = 0; k < 8; k++) st[k] = sha_d::kIV[k];
  sha_d::compress(st, w);
  // leading zero bits of the digest bytes (big-endian words)
  uint32_t full = bits >> 3, extra = bits & 7;
  bool ok = true;
  for (uint32_t k = 0; k < full && ok; k++) ok = ((st[k >> 2] >> (24 - 8 * (k & 3))) & 0xFF) == 0;
  if (ok && extra) ok = ((((st[full >> 2] >> (24 - 8 * (full & 3))) & 0xFF) >> (8 - extra)) == 0);
  if (ok) atomicMin(found, (unsigned long long)n);
}

uint64_t pow_search(const uint8_t digest[32], uint32_t bits, cudaStream_t s, unsigned long long* d_found,
                    unsigned long long* h_found, int fn) {
  if (bits == 0) return 0;
  uint4 d0, d1;
  memcpy(&d0, digest, 16);
  memcpy(&d1, digest + 16, 16);
  // the smallest valid nonce is expected near 2^bits: scan ranges of twice
  // that (at least 2^16, at most 2^22) in increasing order
  const uint64_t chunk = 1ull << (bits + 1 < 16 ? 16 : bits + 1 > 22 ? 22 : bits + 1);
  for (uint64_t start = 0;; start += chunk) {
    *h_found = ~0ull;
    CK(cudaMemcpyAsync(d_found, h_found, 8, cudaMemcpyHostToDevice, s));
    count_launch();
    if (fn == flock::kFnSha256) k_pow_sha<<<(unsigned)(chunk / 256), 256, 0, s>>>(d0, d1, bits, start, chunk, d_found);
    else k_pow<<<(unsigned)(chunk / 256), 256, 0, s>>>(d0, d1, bits, start, chunk, d_found);
    CK(cudaMemcpyAsync(h_found, d_found, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (*h_found != ~0ull) return *h_found;
  }
}
