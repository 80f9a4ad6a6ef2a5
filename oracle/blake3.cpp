// BLAKE3 restated from the published specification (test infrastructure;
// see flockref.hpp).  The reference uses the `blake3` crate 1.8.6
// (Cargo.lock:27-30): root hashes / XOF for the Fiat-Shamir transcript
// (crates/flock-core/src/challenger.rs:189-307), `finalize_non_root` for
// Merkle leaves and `merge_subtrees_non_root` for parents
// (crates/flock-core/src/merkle.rs:192-203).  Root-mode outputs are pinned
// against the Python `blake3` module in tests.
#include "flockref.hpp"

namespace flockref {
namespace b3 {

const uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                        0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
static const int PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};

static inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
static inline void g(uint32_t* s, int a, int b, int c, int d, uint32_t mx, uint32_t my) {
  s[a] = s[a] + s[b] + mx; s[d] = rotr(s[d] ^ s[a], 16);
  s[c] = s[c] + s[d];      s[b] = rotr(s[b] ^ s[c], 12);
  s[a] = s[a] + s[b] + my; s[d] = rotr(s[d] ^ s[a], 8);
  s[c] = s[c] + s[d];      s[b] = rotr(s[b] ^ s[c], 7);
}

void compress_words(const uint32_t cv[8], const uint32_t m_in[16], uint64_t counter,
                    uint32_t block_len, uint32_t flags, uint32_t out[16]) {
  uint32_t s[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                    IV[0], IV[1], IV[2], IV[3], (uint32_t)counter, (uint32_t)(counter >> 32),
                    block_len, flags};
  uint32_t m[16];
  memcpy(m, m_in, sizeof(m));
  for (int r = 0; r < 7; r++) {
    g(s, 0, 4, 8, 12, m[0], m[1]);
    g(s, 1, 5, 9, 13, m[2], m[3]);
    g(s, 2, 6, 10, 14, m[4], m[5]);
    g(s, 3, 7, 11, 15, m[6], m[7]);
    g(s, 0, 5, 10, 15, m[8], m[9]);
    g(s, 1, 6, 11, 12, m[10], m[11]);
    g(s, 2, 7, 8, 13, m[12], m[13]);
    g(s, 3, 4, 9, 14, m[14], m[15]);
    if (r < 6) {
      uint32_t p[16];
      for (int i = 0; i < 16; i++) p[i] = m[PERM[i]];
      memcpy(m, p, sizeof(m));
    }
  }
  for (int i = 0; i < 8; i++) {
    out[i] = s[i] ^ s[i + 8];
    out[i + 8] = s[i + 8] ^ cv[i];
  }
}

void compress(const uint32_t cv[8], const uint8_t block[64], uint64_t counter,
              uint32_t block_len, uint32_t flags, uint32_t out[16]) {
  uint32_t m[16];
  for (int i = 0; i < 16; i++)
    m[i] = (uint32_t)block[4 * i] | ((uint32_t)block[4 * i + 1] << 8) |
           ((uint32_t)block[4 * i + 2] << 16) | ((uint32_t)block[4 * i + 3] << 24);
  compress_words(cv, m, counter, block_len, flags, out);
}

static void words_to_bytes(const uint32_t* w, int n, uint8_t* out) {
  for (int i = 0; i < n; i++) {
    out[4 * i] = (uint8_t)w[i];
    out[4 * i + 1] = (uint8_t)(w[i] >> 8);
    out[4 * i + 2] = (uint8_t)(w[i] >> 16);
    out[4 * i + 3] = (uint8_t)(w[i] >> 24);
  }
}

Hasher::Hasher() { memcpy(chunk_cv_, IV, sizeof(chunk_cv_)); }

void Hasher::push_cv(const uint32_t cv_in[8], uint64_t total_chunks) {
  std::array<uint32_t, 8> cv;
  memcpy(cv.data(), cv_in, 32);
  while ((total_chunks & 1) == 0) {
    std::array<uint32_t, 8> left = stack_.back();
    stack_.pop_back();
    uint32_t block[16], out[16];
    memcpy(block, left.data(), 32);
    memcpy(block + 8, cv.data(), 32);
    compress_words(IV, block, 0, 64, PARENT, out);
    memcpy(cv.data(), out, 32);
    total_chunks >>= 1;
  }
  stack_.push_back(cv);
}

void Hasher::update(const void* data, size_t len) {
  const uint8_t* p = (const uint8_t*)data;
  while (len > 0) {
    // chunk full (1024 bytes consumed: 15 compressed blocks + a full buffer)
    if (blocks_compressed_ == 15 && buf_len_ == 64) {
      uint32_t out[16];
      compress(chunk_cv_, buf_, chunk_counter_, 64, CHUNK_END, out);
      uint64_t total = chunk_counter_ + 1;
      push_cv(out, total);
      chunk_counter_ = total;
      memcpy(chunk_cv_, IV, sizeof(chunk_cv_));
      blocks_compressed_ = 0;
      buf_len_ = 0;
    }
    if (buf_len_ == 64) {
      uint32_t out[16];
      compress(chunk_cv_, buf_, chunk_counter_, 64, blocks_compressed_ == 0 ? CHUNK_START : 0, out);
      memcpy(chunk_cv_, out, 32);
      blocks_compressed_++;
      buf_len_ = 0;
    }
    size_t take = 64 - buf_len_;
    if (take > len) take = len;
    memcpy(buf_ + buf_len_, p, take);
    buf_len_ += take;
    p += take;
    len -= take;
  }
}

Hasher::Output Hasher::final_output() const {
  Output o;
  memcpy(o.cv, chunk_cv_, 32);
  memset(o.block, 0, 64);
  memcpy(o.block, buf_, buf_len_);
  o.block_len = (uint32_t)buf_len_;
  o.counter = chunk_counter_;
  o.flags = CHUNK_END | (blocks_compressed_ == 0 ? CHUNK_START : 0);
  for (size_t i = stack_.size(); i-- > 0;) {
    uint32_t out[16];
    compress(o.cv, o.block, o.counter, o.block_len, o.flags, out);
    uint32_t block[16];
    memcpy(block, stack_[i].data(), 32);
    memcpy(block + 8, out, 32);
    memcpy(o.cv, IV, 32);
    words_to_bytes(block, 16, o.block);
    o.block_len = 64;
    o.counter = 0;
    o.flags = PARENT;
  }
  return o;
}

void Hasher::finalize_xof(uint8_t* out, size_t len) const {
  Output o = final_output();
  uint64_t ctr = 0;
  while (len > 0) {
    uint32_t w[16];
    compress(o.cv, o.block, ctr, o.block_len, o.flags | ROOT, w);
    uint8_t bytes[64];
    words_to_bytes(w, 16, bytes);
    size_t take = len < 64 ? len : 64;
    memcpy(out, bytes, take);
    out += take;
    len -= take;
    ctr++;
  }
}

void Hasher::finalize(uint8_t out32[32]) const { finalize_xof(out32, 32); }

void Hasher::finalize_non_root(uint8_t out32[32]) const {
  Output o = final_output();
  uint32_t w[16];
  compress(o.cv, o.block, o.counter, o.block_len, o.flags, w);
  words_to_bytes(w, 8, out32);
}

void hash(const void* data, size_t len, uint8_t out32[32]) {
  Hasher h;
  h.update(data, len);
  h.finalize(out32);
}

void leaf_cv(const void* data, size_t len, uint8_t out32[32]) {
  Hasher h;
  h.update(data, len);
  h.finalize_non_root(out32);
}

void parent_cv(const uint8_t l[32], const uint8_t r[32], uint8_t out32[32]) {
  uint8_t block[64];
  memcpy(block, l, 32);
  memcpy(block + 32, r, 32);
  uint32_t w[16];
  compress(IV, block, 0, 64, PARENT, w);
  words_to_bytes(w, 8, out32);
}

}  // namespace b3
}  // namespace flockref
