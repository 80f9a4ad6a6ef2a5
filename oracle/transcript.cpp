// Fiat-Shamir transcript + PoW grinding of the oracle (test infrastructure;
// see flockref.hpp).  Restates crates/flock-core/src/challenger.rs:
// op/kind tags :170-177, with_hash :237-250, absorb_f128 (lo LE, hi LE) :274,
// BLAKE3 XOF squeeze :286-307, observe/sample :327-380, grind_pow (smallest
// satisfying nonce) :384-475, verify_pow :502-545, PoW pre-image
// `digest || nonce_le || 0^24` :549-556, leading-zero predicate :558-600.
// Input generator: benchmark-tools/common/src/lib.rs:1-37.
#include "flockref.hpp"

namespace flockref {

enum : uint8_t { OP_DOMAIN = 1, OP_LABEL = 2, OP_OBSERVE = 3, OP_SQUEEZE = 4, OP_BYTES = 5 };
enum : uint8_t { KIND_SCALAR = 1, KIND_SLICE = 2 };

static void le64(uint64_t v, uint8_t out[8]) {
  for (int i = 0; i < 8; i++) out[i] = (uint8_t)(v >> (8 * i));
}

Challenger::Challenger(const std::string& domain, int kind) : kind_(kind) {
  uint8_t op = OP_DOMAIN, len[8];
  le64(domain.size(), len);
  absorb(&op, 1);
  absorb(len, 8);
  absorb(domain.data(), domain.size());
}

void Challenger::observe_label(const std::string& label) {
  uint8_t op = OP_LABEL, len[8];
  le64(label.size(), len);
  absorb(&op, 1);
  absorb(len, 8);
  absorb(label.data(), label.size());
}

void Challenger::observe_f128(F128 v) {
  uint8_t tag[2] = {OP_OBSERVE, KIND_SCALAR}, b[16];
  le64(v.lo, b);
  le64(v.hi, b + 8);
  absorb(tag, 2);
  absorb(b, 16);
}

void Challenger::observe_f128_slice(const std::vector<F128>& v) {
  uint8_t tag[2] = {OP_OBSERVE, KIND_SLICE}, len[8];
  le64(v.size(), len);
  absorb(tag, 2);
  absorb(len, 8);
  for (const F128& x : v) {
    uint8_t b[16];
    le64(x.lo, b);
    le64(x.hi, b + 8);
    absorb(b, 16);
  }
}

void Challenger::observe_bytes(const void* data, size_t n) {
  uint8_t op = OP_BYTES, len[8];
  le64(n, len);
  absorb(&op, 1);
  absorb(len, 8);
  absorb(data, n);
}

static F128 f128_from_le(const uint8_t* b) {
  uint64_t lo = 0, hi = 0;
  for (int i = 0; i < 8; i++) {
    lo |= (uint64_t)b[i] << (8 * i);
    hi |= (uint64_t)b[8 + i] << (8 * i);
  }
  return F128(lo, hi);
}

F128 Challenger::sample_f128() {
  uint8_t tag[2] = {OP_SQUEEZE, KIND_SCALAR}, buf[16];
  absorb(tag, 2);
  squeeze(buf, 16);
  absorb(buf, 16);
  return f128_from_le(buf);
}

std::vector<F128> Challenger::sample_f128_vec(size_t n) {
  uint8_t tag[2] = {OP_SQUEEZE, KIND_SLICE}, len[8];
  le64(n, len);
  absorb(tag, 2);
  absorb(len, 8);
  std::vector<uint8_t> buf(n * 16);
  if (n) squeeze(buf.data(), buf.size());
  absorb(buf.data(), buf.size());
  std::vector<F128> out(n);
  for (size_t i = 0; i < n; i++) out[i] = f128_from_le(&buf[16 * i]);
  return out;
}

void Challenger::state_digest(uint8_t out[32]) const {
  if (kind_ == SHA256) s_.finalize(out);
  else h_.finalize(out);
}

// BLAKE3: the XOF of the state; SHA-256: SHA256(state || ctr LE), 32 bytes
// per counter value
void Challenger::squeeze(uint8_t* out, size_t n) const {
  if (kind_ != SHA256) {
    h_.finalize_xof(out, n);
    return;
  }
  for (uint64_t ctr = 0; 32 * ctr < n; ctr++) {
    sha::Hasher s = s_;
    uint8_t c[8], blk[32];
    le64(ctr, c);
    s.update(c, 8);
    s.finalize(blk);
    memcpy(out + 32 * ctr, blk, std::min<size_t>(32, n - 32 * ctr));
  }
}

bool pow_ok(const uint8_t digest[32], uint64_t nonce, uint32_t bits, int kind) {
  uint8_t pre[64] = {0};
  memcpy(pre, digest, 32);
  le64(nonce, pre + 32);
  uint8_t h[32];
  if (kind == SHA256) sha::hash(pre, 40, h);  // digest || nonce, no padding
  else b3::hash(pre, 64, h);
  uint32_t full = bits / 8, extra = bits % 8;
  for (uint32_t i = 0; i < full; i++)
    if (h[i] != 0) return false;
  if (extra > 0 && (h[full] >> (8 - extra)) != 0) return false;
  return true;
}

uint64_t Challenger::grind_pow(uint32_t bits) {
  uint64_t nonce = 0;
  if (bits != 0) {
    uint8_t d[32];
    state_digest(d);
    while (!pow_ok(d, nonce, bits, kind_)) nonce++;
  }
  uint8_t b[8];
  le64(nonce, b);
  observe_bytes(b, 8);
  return nonce;
}

bool Challenger::verify_pow(uint64_t nonce, uint32_t bits) {
  uint8_t d[32];
  state_digest(d);
  bool ok = bits == 0 ? nonce == 0 : pow_ok(d, nonce, bits, kind_);
  uint8_t b[8];
  le64(nonce, b);
  observe_bytes(b, 8);
  return ok;
}

std::vector<Compression> generate_compressions(uint32_t log2, uint64_t seed) {
  size_t count = (size_t)1 << log2;
  uint64_t rot = ((uint64_t)log2 << 29) | ((uint64_t)log2 >> 35);
  uint64_t state = seed ^ rot;
  auto next = [&]() -> uint32_t {
    state += 0x9E3779B97F4A7C15ull;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return (uint32_t)(z ^ (z >> 31));
  };
  std::vector<Compression> out(count);
  for (size_t i = 0; i < count; i++) {
    Compression& c = out[i];
    for (int w = 0; w < 8; w++) c.cv[w] = next();
    for (int w = 0; w < 16; w++) c.m[w] = next();
    c.counter = next();
    c.block_len = 64;
    c.flags = 11;
  }
  return out;
}

}  // namespace flockref
