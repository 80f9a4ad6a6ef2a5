// Host-side support of the B200 prover (see host.hpp).
//  * GF(2^128)/GF(2^8): crates/flock-core/src/field/gf2_128.rs:22-265,
//    gf2_8.rs:20-140, phi8.rs:18-1050 (carried as the images of the eight
//    basis bytes and expanded by linearity).
//  * BLAKE3: published specification (the reference uses the blake3 crate
//    1.8.6 for its transcript, challenger.rs:189-307).
//  * Transcript framing: challenger.rs:170-380 (op/kind tags, LE lengths,
//    lo||hi F128 encoding, XOF squeeze re-absorbed).
//  * R1CS: crates/flock-prover/src/r1cs_hashes/blake3.rs:198-262 (layout),
//    :456-640 (build_matrices, Option-D cascade) and
//    crates/flock-core/src/r1cs.rs:334-385 (statement digest).
//  * Wire format: crates/flock-prover/src/proof_io.rs:40-215 (bincode 1.3
//    fixint; enum = u32 variant index; Vec = u64 length).
#include "host.hpp"
#include <algorithm>
#include <set>
#include <map>
#include <memory>
#include <mutex>
#include <wmmintrin.h>
#include <emmintrin.h>
#include <smmintrin.h>
#include <tmmintrin.h>

namespace flock {

// ---------------------------------------------------------------- field --
static inline void hclmul(uint64_t a, uint64_t b, uint64_t& lo, uint64_t& hi) {
  __m128i r = _mm_clmulepi64_si128(_mm_set_epi64x(0, (long long)a), _mm_set_epi64x(0, (long long)b), 0);
  lo = (uint64_t)_mm_cvtsi128_si64(r);
  hi = (uint64_t)_mm_cvtsi128_si64(_mm_unpackhi_epi64(r, r));
}

f128 hmul(f128 a, f128 b) {
  uint64_t l0, l1, h0, h1, m0, m1;
  hclmul(a.lo, b.lo, l0, l1);
  hclmul(a.hi, b.hi, h0, h1);
  hclmul(a.lo ^ a.hi, b.lo ^ b.hi, m0, m1);
  m0 ^= l0 ^ h0;
  m1 ^= l1 ^ h1;
  return reduce256(l0, l1 ^ m0, h0 ^ m1, h1);
}

f128 hinv(f128 a) {  // a^(2^128 - 2)
  f128 r = hone(), s = hmul(a, a);
  for (int i = 1; i < 128; i++) {
    r = hmul(r, s);
    s = hmul(s, s);
  }
  return r;
}

static const f128 kPhiBasis[8] = {
    {0x0000000000000001ull, 0x0000000000000000ull}, {0x6b8330483c2e9849ull, 0x0dcb364640a222feull},
    {0x7573da4a5f7710edull, 0x3d5bd35c94646a24ull}, {0x41a12db1f974f3acull, 0x6d58c4e181f9199full},
    {0x5e2f716f4ede412full, 0xa72ec17764d7ced5ull}, {0x5cb10fbabcf00118ull, 0x4d52354a3a3d8c86ull},
    {0x95ed1f57f3632d4dull, 0x553e92e8bc0ae9a7ull}, {0x512625b1f09fa87eull, 0x93252331bf042b11ull}};

static std::array<f128, 256> phi_expand() {
  std::array<f128, 256> t;
  for (int v = 0; v < 256; v++) {
    f128 acc = mk(0, 0);
    for (int b = 0; b < 8; b++)
      if (v & (1 << b)) acc = fx(acc, kPhiBasis[b]);
    t[v] = acc;
  }
  return t;
}
static const std::array<f128, 256> kPhiArr = phi_expand();
const f128* phi8_table() { return kPhiArr.data(); }

std::vector<f128> heq(const std::vector<f128>& r) {
  std::vector<f128> t((size_t)1 << r.size());
  t[0] = hone();
  for (size_t i = 0; i < r.size(); i++) {
    size_t len = (size_t)1 << i;
    for (size_t x = 0; x < len; x++) {
      f128 h = hmul(t[x], r[i]);
      t[x + len] = h;
      t[x] = fx(t[x], h);
    }
  }
  return t;
}

std::vector<f128> hlagrange(f128 z, int base) {
  // L_i(z) = prod_{j != i} (z + s_j) / (s_i + s_j),  s_j = phi8(base + j).
  // The denominators depend only on the nodes (one table per base, 0 or 64,
  // built once); the numerators come from prefix and suffix products of
  // (z + s_j), so a call costs 256 products and no inversion.
  const auto& P = kPhiArr;
  static std::once_flag once[2];
  static std::array<f128, 64> inv_den[2];
  const int t = base ? 1 : 0;
  std::call_once(once[t], [&P, base, t] {
    for (int i = 0; i < 64; i++) {
      f128 den = hone();
      for (int j = 0; j < 64; j++)
        if (j != i) den = hmul(den, fx(P[base + i], P[base + j]));
      inv_den[t][i] = hinv(den);
    }
  });
  f128 suf[65];
  suf[64] = hone();
  for (int j = 63; j >= 0; j--) suf[j] = hmul(suf[j + 1], fx(z, P[base + j]));
  std::vector<f128> w(64);
  f128 pre = hone();
  for (int i = 0; i < 64; i++) {
    w[i] = hmul(hmul(pre, suf[i + 1]), inv_den[t][i]);
    pre = hmul(pre, fx(z, P[base + i]));
  }
  return w;
}

uint8_t hgf8_mul(uint8_t a, uint8_t b) { return gf8_mul_slow(a, b); }

// six rounds of swapping the off-diagonal j x j blocks inside every 2j x 2j block
void transpose64(uint64_t a[64]) {
  static const uint64_t M[6] = {0x00000000FFFFFFFFull, 0x0000FFFF0000FFFFull, 0x00FF00FF00FF00FFull,
                                0x0F0F0F0F0F0F0F0Full, 0x3333333333333333ull, 0x5555555555555555ull};
  for (int k = 0, j = 32; j; k++, j >>= 1)
    for (int r = 0; r < 64; r++)
      if (!(r & j)) {
        const uint64_t t = ((a[r] >> j) ^ a[r | j]) & M[k];
        a[r | j] ^= t;
        a[r] ^= t << j;
      }
}

std::vector<f128> transpose128(const std::vector<f128>& rows) {
  uint64_t A[64], B[64], C[64], D[64];  // [rows 0..63 | 64..127] x [bits 0..63 | 64..127]
  for (int i = 0; i < 64; i++) {
    A[i] = rows[i].lo;
    B[i] = rows[i].hi;
    C[i] = rows[64 + i].lo;
    D[i] = rows[64 + i].hi;
  }
  transpose64(A);
  transpose64(B);
  transpose64(C);
  transpose64(D);
  std::vector<f128> out(128);
  for (int j = 0; j < 64; j++) {
    out[j] = mk(A[j], C[j]);
    out[64 + j] = mk(B[j], D[j]);
  }
  return out;
}

void subset_sums8(const f128* v8, f128* out) {
  out[0] = mk(0, 0);
  for (int v = 1; v < 256; v++) out[v] = fx(out[v & (v - 1)], v8[__builtin_ctz(v)]);
}

// --------------------------------------------------------------- BLAKE3 --
const uint32_t kB3IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};

// One BLAKE3 compression with the 4x4 state held as four SSE rows: the four
// column G functions run lane-parallel, the rows are rotated so the four
// diagonal G functions do too, and rotated back (the row-parallel form of the
// BLAKE3 specification's compression function).  The message schedule of
// round r is the permutation (2,6,3,10,7,0,4,13,1,11,12,5,9,14,15,8) applied r
// times.
namespace {
struct B3Sched {
  uint8_t s[7][16];
  B3Sched() {
    static const uint8_t P[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
    for (int i = 0; i < 16; i++) s[0][i] = (uint8_t)i;
    for (int r = 1; r < 7; r++)
      for (int i = 0; i < 16; i++) s[r][i] = s[r - 1][P[i]];
  }
};
const B3Sched kB3Sched;
inline __m128i rotr16(__m128i x) {
  return _mm_shuffle_epi8(x, _mm_set_epi8(13, 12, 15, 14, 9, 8, 11, 10, 5, 4, 7, 6, 1, 0, 3, 2));
}
inline __m128i rotr8(__m128i x) {
  return _mm_shuffle_epi8(x, _mm_set_epi8(12, 15, 14, 13, 8, 11, 10, 9, 4, 7, 6, 5, 0, 3, 2, 1));
}
inline __m128i rotr12(__m128i x) { return _mm_or_si128(_mm_srli_epi32(x, 12), _mm_slli_epi32(x, 20)); }
inline __m128i rotr7(__m128i x) { return _mm_or_si128(_mm_srli_epi32(x, 7), _mm_slli_epi32(x, 25)); }
inline void b3_g(__m128i& r0, __m128i& r1, __m128i& r2, __m128i& r3, __m128i mx, __m128i my) {
  r0 = _mm_add_epi32(_mm_add_epi32(r0, r1), mx);
  r3 = rotr16(_mm_xor_si128(r3, r0));
  r2 = _mm_add_epi32(r2, r3);
  r1 = rotr12(_mm_xor_si128(r1, r2));
  r0 = _mm_add_epi32(_mm_add_epi32(r0, r1), my);
  r3 = rotr8(_mm_xor_si128(r3, r0));
  r2 = _mm_add_epi32(r2, r3);
  r1 = rotr7(_mm_xor_si128(r1, r2));
}
}  // namespace

void b3_compress(const uint32_t cv[8], const uint32_t m[16], uint64_t ctr, uint32_t blen, uint32_t flags,
                 uint32_t out[16]) {
  const __m128i c0 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(cv));
  const __m128i c1 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(cv + 4));
  __m128i r0 = c0, r1 = c1;
  __m128i r2 = _mm_loadu_si128(reinterpret_cast<const __m128i*>(kB3IV));
  __m128i r3 = _mm_set_epi32((int)flags, (int)blen, (int)(uint32_t)(ctr >> 32), (int)(uint32_t)ctr);
  for (int r = 0; r < 7; r++) {
    const uint8_t* s = kB3Sched.s[r];
    // columns: G_g for g = 0..3 takes message words 2g, 2g + 1
    b3_g(r0, r1, r2, r3, _mm_set_epi32((int)m[s[6]], (int)m[s[4]], (int)m[s[2]], (int)m[s[0]]),
         _mm_set_epi32((int)m[s[7]], (int)m[s[5]], (int)m[s[3]], (int)m[s[1]]));
    // diagonals: rotate rows 1, 2, 3 left by 1, 2, 3 lanes
    r1 = _mm_shuffle_epi32(r1, _MM_SHUFFLE(0, 3, 2, 1));
    r2 = _mm_shuffle_epi32(r2, _MM_SHUFFLE(1, 0, 3, 2));
    r3 = _mm_shuffle_epi32(r3, _MM_SHUFFLE(2, 1, 0, 3));
    b3_g(r0, r1, r2, r3, _mm_set_epi32((int)m[s[14]], (int)m[s[12]], (int)m[s[10]], (int)m[s[8]]),
         _mm_set_epi32((int)m[s[15]], (int)m[s[13]], (int)m[s[11]], (int)m[s[9]]));
    r1 = _mm_shuffle_epi32(r1, _MM_SHUFFLE(2, 1, 0, 3));
    r2 = _mm_shuffle_epi32(r2, _MM_SHUFFLE(1, 0, 3, 2));
    r3 = _mm_shuffle_epi32(r3, _MM_SHUFFLE(0, 3, 2, 1));
  }
  _mm_storeu_si128(reinterpret_cast<__m128i*>(out), _mm_xor_si128(r0, r2));
  _mm_storeu_si128(reinterpret_cast<__m128i*>(out + 4), _mm_xor_si128(r1, r3));
  _mm_storeu_si128(reinterpret_cast<__m128i*>(out + 8), _mm_xor_si128(r2, c0));
  _mm_storeu_si128(reinterpret_cast<__m128i*>(out + 12), _mm_xor_si128(r3, c1));
}

// the host is little endian (x86-64), so a block's words are its bytes
static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "little-endian host");
static void le_words(const uint8_t* b, uint32_t w[16]) { memcpy(w, b, 64); }

B3::B3() { memcpy(cv_, kB3IV, 32); }

void B3::chunk_done() {
  uint32_t w[16], out[16];
  le_words(buf_, w);
  b3_compress(cv_, w, chunk_, 64, 2 /*CHUNK_END*/, out);
  std::array<uint32_t, 8> cv;
  memcpy(cv.data(), out, 32);
  uint64_t total = ++chunk_;
  while (!(total & 1)) {
    uint32_t blk[16];
    memcpy(blk, stack_.back().data(), 32);
    memcpy(blk + 8, cv.data(), 32);
    stack_.pop_back();
    b3_compress(kB3IV, blk, 0, 64, 4 /*PARENT*/, out);
    memcpy(cv.data(), out, 32);
    total >>= 1;
  }
  stack_.push_back(cv);
  memcpy(cv_, kB3IV, 32);
  nblk_ = 0;
  blen_ = 0;
}

void B3::update(const void* p, size_t n) {
  const uint8_t* d = (const uint8_t*)p;
  while (n) {
    if (blen_ == 64) {
      if (nblk_ == 15) {
        chunk_done();
      } else {
        uint32_t w[16], out[16];
        le_words(buf_, w);
        b3_compress(cv_, w, chunk_, 64, nblk_ == 0 ? 1u : 0u, out);
        memcpy(cv_, out, 32);
        nblk_++;
        blen_ = 0;
      }
    }
    size_t take = std::min(n, 64 - blen_);
    memcpy(buf_ + blen_, d, take);
    blen_ += take;
    d += take;
    n -= take;
  }
}

void B3::xof(uint8_t* out, size_t n) const {
  uint32_t cv[8], w[16], o[16];
  uint8_t blk[64] = {0};
  memcpy(cv, cv_, 32);
  memcpy(blk, buf_, blen_);
  uint32_t blen = (uint32_t)blen_, flags = 2u | (nblk_ == 0 ? 1u : 0u);
  uint64_t ctr = chunk_;
  for (size_t i = stack_.size(); i-- > 0;) {
    le_words(blk, w);
    b3_compress(cv, w, ctr, blen, flags, o);
    uint32_t pw[16];
    memcpy(pw, stack_[i].data(), 32);
    memcpy(pw + 8, o, 32);
    memcpy(blk, pw, 64);
    memcpy(cv, kB3IV, 32);
    blen = 64;
    ctr = 0;
    flags = 4;
  }
  le_words(blk, w);
  for (uint64_t c = 0; n; c++) {
    b3_compress(cv, w, c, blen, flags | 8u /*ROOT*/, o);
    size_t take = std::min<size_t>(n, 64);
    memcpy(out, o, take);
    out += take;
    n -= take;
  }
}

// ----------------------------------------------------------- transcript --
static void le64(uint64_t v, uint8_t* b) { for (int i = 0; i < 8; i++) b[i] = (uint8_t)(v >> (8 * i)); }

S256::S256() { memcpy(h_, kB3IV, 32); }
void S256::update(const void* p, size_t n) {
  const uint8_t* b = static_cast<const uint8_t*>(p);
  total_ += n;
  while (n) {
    const size_t k = std::min(n, 64 - blen_);
    memcpy(buf_ + blen_, b, k);
    blen_ += k;
    b += k;
    n -= k;
    if (blen_ == 64) {
      uint32_t m[16];
      for (int i = 0; i < 16; i++)
        m[i] = (uint32_t)buf_[4 * i] << 24 | (uint32_t)buf_[4 * i + 1] << 16 | (uint32_t)buf_[4 * i + 2] << 8 |
               buf_[4 * i + 3];
      sha256_compress(h_, m, h_);
      blen_ = 0;
    }
  }
}
void S256::digest(uint8_t out[32]) const {
  S256 s = *this;
  const uint64_t bits = total_ * 8;
  uint8_t pad[72] = {0x80};
  const size_t padn = (blen_ < 56 ? 56 - blen_ : 120 - blen_);
  for (int i = 0; i < 8; i++) pad[padn + i] = (uint8_t)(bits >> (56 - 8 * i));
  s.update(pad, padn + 8);
  for (int i = 0; i < 8; i++)
    for (int k = 0; k < 4; k++) out[4 * i + k] = (uint8_t)(s.h_[i] >> (24 - 8 * k));
}
void sha256_bytes(const void* p, size_t n, uint8_t out[32]) {
  S256 s;
  s.update(p, n);
  s.digest(out);
}

Transcript::Transcript(const std::string& domain, int fn) : fn_(fn) {
  uint8_t op = 1, n[8];
  le64(domain.size(), n);
  put(&op, 1);
  put(n, 8);
  put(domain.data(), domain.size());
}
void Transcript::label(const char* s) {
  uint8_t op = 2, n[8];
  size_t len = strlen(s);
  le64(len, n);
  put(&op, 1);
  put(n, 8);
  put(s, len);
}
void Transcript::label_bytes(const void* p, size_t len) {
  uint8_t op = 2, n[8];
  le64(len, n);
  put(&op, 1);
  put(n, 8);
  put(p, len);
}
bool pow_hash_ok(const uint8_t digest[32], uint64_t nonce, uint32_t bits, int fn) {
  uint8_t pre[64] = {0}, h[32];
  memcpy(pre, digest, 32);
  for (int i = 0; i < 8; i++) pre[32 + i] = (uint8_t)(nonce >> (8 * i));
  if (fn == kFnSha256) {
    sha256_bytes(pre, 40, h);
  } else {
    B3 b;
    b.update(pre, 64);
    b.digest(h);
  }
  bool ok = true;
  for (uint32_t k = 0; k < bits && ok; k++) ok = ((h[k / 8] >> (7 - k % 8)) & 1) == 0;
  return ok;
}
uint64_t pow_search_host(const uint8_t digest[32], uint32_t bits, int fn) {
  for (uint64_t n = 0;; n++)
    if (pow_hash_ok(digest, n, bits, fn)) return n;
}
bool Transcript::verify_pow(uint64_t nonce, uint32_t bits) {
  bool ok = true;
  if (bits == 0) {
    ok = nonce == 0;
  } else {
    uint8_t d[32];
    state_digest(d);
    ok = pow_hash_ok(d, nonce, bits, fn_);
  }
  this->nonce(nonce);
  return ok;
}
void Transcript::squeeze(uint8_t* out, size_t n) const {
  if (fn_ != kFnSha256) {
    h_.xof(out, n);
    return;
  }
  for (uint64_t ctr = 0, off = 0; off < n; ctr++, off += 32) {
    S256 s = s_;
    uint8_t c[8], blk[32];
    le64(ctr, c);
    s.update(c, 8);
    s.digest(blk);
    memcpy(out + off, blk, std::min<size_t>(32, n - off));
  }
}
void Transcript::f128v(f128 v) {
  uint8_t b[18] = {3, 1};
  le64(v.lo, b + 2);
  le64(v.hi, b + 10);
  put(b, 18);
}
void Transcript::f128s(const f128* v, size_t n) {
  std::vector<uint8_t> b(10 + 16 * n);
  b[0] = 3;
  b[1] = 2;
  le64(n, &b[2]);
  for (size_t i = 0; i < n; i++) {
    le64(v[i].lo, &b[10 + 16 * i]);
    le64(v[i].hi, &b[18 + 16 * i]);
  }
  put(b.data(), b.size());
}
void Transcript::bytes(const void* p, size_t n) {
  uint8_t h[9] = {5};
  le64(n, h + 1);
  put(h, 9);
  put(p, n);
}
static f128 from_le(const uint8_t* b) {
  uint64_t lo = 0, hi = 0;
  for (int i = 0; i < 8; i++) { lo |= (uint64_t)b[i] << (8 * i); hi |= (uint64_t)b[8 + i] << (8 * i); }
  return mk(lo, hi);
}
f128 Transcript::sample() {
  uint8_t t[2] = {4, 1}, buf[16];
  put(t, 2);
  squeeze(buf, 16);
  put(buf, 16);
  return from_le(buf);
}
std::vector<f128> Transcript::sample_vec(size_t n) {
  uint8_t t[10] = {4, 2};
  le64(n, t + 2);
  put(t, 10);
  std::vector<uint8_t> buf(16 * n);
  if (n) squeeze(buf.data(), buf.size());
  put(buf.data(), buf.size());
  std::vector<f128> v(n);
  for (size_t i = 0; i < n; i++) v[i] = from_le(&buf[16 * i]);
  return v;
}

// ------------------------------------------------------------------ R1CS --
namespace {
using Set = std::vector<uint16_t>;  // sorted, square-free slot set
Set sdiff(const Set& a, const Set& b) {
  Set out;
  out.reserve(a.size() + b.size());
  std::set_symmetric_difference(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(out));
  return out;
}
Set prefix(int base, int n) {  // {base, ..., base + n - 1}
  Set s(n);
  for (int j = 0; j < n; j++) s[j] = (uint16_t)(base + j);
  return s;
}
struct SymWord {
  std::array<Set, 32> b;
  static SymWord slots(int base) { SymWord w; for (int i = 0; i < 32; i++) w.b[i] = {(uint16_t)(base + i)}; return w; }
  static SymWord konst(uint32_t v, int pin = kZConst) { SymWord w; for (int i = 0; i < 32; i++) if (v >> i & 1) w.b[i] = {(uint16_t)pin}; return w; }
  SymWord operator^(const SymWord& o) const { SymWord w; for (int i = 0; i < 32; i++) w.b[i] = sdiff(b[i], o.b[i]); return w; }
  SymWord rotr(int n) const { SymWord w; for (int i = 0; i < 32; i++) w.b[i] = b[(i + n) & 31]; return w; }
};
const int kLanes[8][4] = {{0, 4, 8, 12}, {1, 5, 9, 13}, {2, 6, 10, 14}, {3, 7, 11, 15},
                          {0, 5, 10, 15}, {1, 6, 11, 12}, {2, 7, 8, 13}, {3, 4, 9, 14}};
const int kPerm[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
constexpr int CV0 = 0, OUTLO = 256, MSG = 513, TLO = 1025, THI = 1057, BLEN = 1089, FLG = 1121, GS = 1153, OUTHI = 15153;

// one 32-bit ADD: rows for its 31 carry slots; returns the sum word
SymWord add(std::vector<Set>& A, std::vector<Set>& B, const SymWord& x, const SymWord& y, int cb) {
  SymWord s;
  for (int i = 0; i < 32; i++) {
    Set cin = prefix(cb, i);
    if (i < 31) {
      A[cb + i] = sdiff(x.b[i], cin);
      B[cb + i] = sdiff(y.b[i], cin);
    }
    s.b[i] = sdiff(sdiff(x.b[i], y.b[i]), cin);
  }
  return s;
}

void to_csr(const std::vector<Set>& rows, std::vector<uint32_t>& ptr, std::vector<uint16_t>& col) {
  ptr.assign(rows.size() + 1, 0);
  for (size_t r = 0; r < rows.size(); r++) ptr[r + 1] = ptr[r] + (uint32_t)rows[r].size();
  col.resize(ptr.back());
  for (size_t r = 0; r < rows.size(); r++) std::copy(rows[r].begin(), rows[r].end(), col.begin() + ptr[r]);
}
void to_csc(const std::vector<uint32_t>& ptr, const std::vector<uint16_t>& col,
            std::vector<uint32_t>& cptr, std::vector<uint16_t>& crow) {
  const int k = (int)ptr.size() - 1;
  cptr.assign(k + 1, 0);
  for (uint16_t c : col) cptr[c + 1]++;
  for (int c = 0; c < k; c++) cptr[c + 1] += cptr[c];
  crow.resize(col.size());
  std::vector<uint32_t> fill(cptr.begin(), cptr.end() - 1);
  for (int r = 0; r < k; r++)
    for (uint32_t j = ptr[r]; j < ptr[r + 1]; j++) crow[fill[col[j]]++] = (uint16_t)r;
}

Statement build() {
  std::vector<Set> A(kK), B(kK);
  const Set one = {(uint16_t)kZConst};
  A[kZConst] = one;
  B[kZConst] = one;
  auto ident_rows = [&](int base, int n) {
    for (int j = 0; j < n; j++) { A[base + j] = {(uint16_t)(base + j)}; B[base + j] = one; }
  };
  ident_rows(CV0, 256);
  ident_rows(MSG, 512);
  ident_rows(TLO, 128);  // counter lo/hi, block_len, flags are contiguous
  std::array<SymWord, 16> st;
  for (int w = 0; w < 8; w++) st[w] = SymWord::slots(CV0 + 32 * w);
  for (int i = 0; i < 4; i++) st[8 + i] = SymWord::konst(kB3IV[i]);
  st[12] = SymWord::slots(TLO);
  st[13] = SymWord::slots(THI);
  st[14] = SymWord::slots(BLEN);
  st[15] = SymWord::slots(FLG);
  int perm[16];
  for (int i = 0; i < 16; i++) perm[i] = i;
  for (int r = 0; r < 7; r++) {
    for (int gi = 0; gi < 8; gi++) {
      int g = 8 * r + gi, base = GS + 250 * g;
      const int* L = kLanes[gi];
      SymWord mx = SymWord::slots(MSG + 32 * perm[2 * gi]), my = SymWord::slots(MSG + 32 * perm[2 * gi + 1]);
      SymWord a1 = add(A, B, add(A, B, st[L[0]], st[L[1]], base), mx, base + 31);
      SymWord d1 = (st[L[3]] ^ a1).rotr(16);
      SymWord c1 = add(A, B, st[L[2]], d1, base + 62);
      SymWord b1 = (st[L[1]] ^ c1).rotr(12);
      SymWord a2 = add(A, B, add(A, B, a1, b1, base + 93), my, base + 124);
      SymWord d2 = (d1 ^ a2).rotr(8);
      SymWord c2 = add(A, B, c1, d2, base + 155);
      SymWord bn = (b1 ^ c2).rotr(7);
      for (int i = 0; i < 32; i++) {
        A[base + 186 + i] = bn.b[i];
        B[base + 186 + i] = one;
        A[base + 218 + i] = d2.b[i];
        B[base + 218 + i] = one;
      }
      st[L[0]] = a2;
      st[L[1]] = SymWord::slots(base + 186);
      st[L[2]] = c2;
      st[L[3]] = SymWord::slots(base + 218);
    }
    int next[16];
    for (int i = 0; i < 16; i++) next[i] = perm[kPerm[i]];
    memcpy(perm, next, sizeof(perm));
  }
  for (int w = 0; w < 8; w++) {
    SymWord lo = st[w] ^ st[w + 8], hi = st[w + 8] ^ SymWord::slots(CV0 + 32 * w);
    for (int i = 0; i < 32; i++) {
      A[OUTLO + 32 * w + i] = lo.b[i];
      B[OUTLO + 32 * w + i] = one;
      A[OUTHI + 32 * w + i] = hi.b[i];
      B[OUTHI + 32 * w + i] = one;
    }
  }
  Statement s;
  to_csr(A, s.a_ptr, s.a_col);
  to_csr(B, s.b_ptr, s.b_col);
  to_csc(s.a_ptr, s.a_col, s.at_ptr, s.at_row);
  to_csc(s.b_ptr, s.b_col, s.bt_ptr, s.bt_row);
  return s;
}

const uint32_t kShaRc[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

// SHA-256 compression (r1cs_hashes/sha2.rs:332-520): one 32-bit ADD of
// x + y is 31 carry rows (x_i ^ cin_i)(y_i ^ cin_i) at cb..cb+30 (the `add`
// above), its sum inlined into the consumer or materialised as 32 rows
// (sum bits) * 1; Ch and Maj are one AND row per bit, e (f ^ g) and
// (a ^ b)(a ^ c).  Layout: H_in 0, H_out 256, M 512, ch 1024, maj 3072,
// round carries 5120 (7 adds x 31 per round), W[16..63] 19008, schedule
// carries 20544 (3 x 31 per word), T1 25008, E_NEW 27056, A_NEW 29104,
// output carries 31152, constant 31400.
Statement build_sha256() {
  constexpr int HB = 0, HOUT = 256, MB = 512, CH = 1024, MAJ = 3072, RC = 5120, WB = 19008, SC = 20544,
                T1 = 25008, EN = 27056, AN = 29104, OC = 31152;
  const int K = 1 << kShaKLog;
  std::vector<Set> A(K), B(K);
  const Set one = {(uint16_t)kShaZConst};
  A[kShaZConst] = one;
  B[kShaZConst] = one;
  for (int j = 0; j < 256; j++) { A[HB + j] = {(uint16_t)(HB + j)}; B[HB + j] = one; }
  for (int j = 0; j < 512; j++) { A[MB + j] = {(uint16_t)(MB + j)}; B[MB + j] = one; }
  auto shr = [](const SymWord& x, int n) { SymWord w; for (int i = 0; i + n < 32; i++) w.b[i] = x.b[i + n]; return w; };
  auto mat = [&](const SymWord& raw, int base) {
    for (int i = 0; i < 32; i++) { A[base + i] = raw.b[i]; B[base + i] = one; }
    return SymWord::slots(base);
  };
  std::array<SymWord, 64> W;
  for (int t = 0; t < 16; t++) W[t] = SymWord::slots(MB + 32 * t);
  for (int t = 16; t < 64; t++) {
    const SymWord s1 = W[t - 2].rotr(17) ^ W[t - 2].rotr(19) ^ shr(W[t - 2], 10);
    const SymWord s0 = W[t - 15].rotr(7) ^ W[t - 15].rotr(18) ^ shr(W[t - 15], 3);
    const int cb = SC + (t - 16) * 93;
    W[t] = mat(add(A, B, add(A, B, add(A, B, s1, W[t - 7], cb), s0, cb + 31), W[t - 16], cb + 62), WB + 32 * (t - 16));
  }
  std::array<SymWord, 8> h_in, s;
  for (int w = 0; w < 8; w++) s[w] = h_in[w] = SymWord::slots(HB + 32 * w);
  for (int r = 0; r < 64; r++) {
    for (int i = 0; i < 32; i++) {
      A[CH + 32 * r + i] = s[4].b[i];
      B[CH + 32 * r + i] = sdiff(s[5].b[i], s[6].b[i]);
      A[MAJ + 32 * r + i] = sdiff(s[0].b[i], s[1].b[i]);
      B[MAJ + 32 * r + i] = sdiff(s[0].b[i], s[2].b[i]);
    }
    const SymWord ch = SymWord::slots(CH + 32 * r) ^ s[6], maj = SymWord::slots(MAJ + 32 * r) ^ s[0];
    const SymWord S1 = s[4].rotr(6) ^ s[4].rotr(11) ^ s[4].rotr(25);
    const SymWord S0 = s[0].rotr(2) ^ s[0].rotr(13) ^ s[0].rotr(22);
    const int cb = RC + 217 * r;
    const SymWord t12 = add(A, B, add(A, B, add(A, B, s[7], S1, cb), ch, cb + 31), SymWord::konst(kShaRc[r], kShaZConst),
                            cb + 62);
    const SymWord t1 = mat(add(A, B, t12, W[r], cb + 93), T1 + 32 * r);
    const SymWord t2 = add(A, B, S0, maj, cb + 124);
    const SymWord e_new = mat(add(A, B, s[3], t1, cb + 155), EN + 32 * r);
    const SymWord a_new = mat(add(A, B, t1, t2, cb + 186), AN + 32 * r);
    s = {a_new, s[0], s[1], s[2], e_new, s[4], s[5], s[6]};
  }
  for (int w = 0; w < 8; w++) mat(add(A, B, s[w], h_in[w], OC + 31 * w), HOUT + 32 * w);
  Statement st;
  st.k_log = kShaKLog;
  st.z_const = kShaZConst;
  st.useful = kShaUseful;
  to_csr(A, st.a_ptr, st.a_col);
  to_csr(B, st.b_ptr, st.b_col);
  to_csc(st.a_ptr, st.a_col, st.at_ptr, st.at_row);
  to_csc(st.b_ptr, st.b_col, st.bt_ptr, st.bt_row);
  return st;
}

// KeccakSetup's BlockR1cs (keccak.rs:558-560, keccak3.rs:151-153,
// common.rs:120-138): A_0 and
// B_0 without entries, so the digest binds the sizes and C = I only; the
// lincheck applies the real matrices through keccak_comb
Statement build_keccak(bool wide) {
  const int k_log = wide ? kKeccak3KLog : kKeccakKLog, K = 1 << k_log;
  Statement st;
  st.k_log = k_log;
  st.z_const = wide ? kKeccak3ZConst : kKeccakZConst;
  st.useful = wide ? kKeccak3Useful : kKeccakUseful;
  st.implicit = true;
  st.a_ptr.assign(K + 1, 0);
  st.b_ptr.assign(K + 1, 0);
  st.at_ptr.assign(K + 1, 0);
  st.bt_ptr.assign(K + 1, 0);
  return st;
}

void put_u64(B3& h, uint64_t v) { uint8_t b[8]; le64(v, b); h.update(b, 8); }
void put_matrix(B3& h, int kk, const std::vector<uint32_t>* ptr, const std::vector<uint16_t>* col) {
  put_u64(h, kk);
  put_u64(h, kk);
  std::vector<uint8_t> buf;
  for (int r = 0; r < kk; r++) {
    uint32_t s = ptr ? (*ptr)[r] : (uint32_t)r, e = ptr ? (*ptr)[r + 1] : (uint32_t)r + 1;
    buf.assign(8 * (e - s + 1), 0);
    le64(e - s, buf.data());
    for (uint32_t j = s; j < e; j++) le64(ptr ? (*col)[j] : (uint64_t)r, &buf[8 * (1 + j - s)]);
    h.update(buf.data(), buf.size());
  }
}
}  // namespace

void sha256_compress(const uint32_t h_in[8], const uint32_t m[16], uint32_t out[8]) {
  auto rr = [](uint32_t x, int n) { return (x >> n) | (x << (32 - n)); };
  uint32_t w[64];
  for (int t = 0; t < 16; t++) w[t] = m[t];
  for (int t = 16; t < 64; t++)
    w[t] = (rr(w[t - 2], 17) ^ rr(w[t - 2], 19) ^ (w[t - 2] >> 10)) + w[t - 7] +
           (rr(w[t - 15], 7) ^ rr(w[t - 15], 18) ^ (w[t - 15] >> 3)) + w[t - 16];
  uint32_t s[8];
  for (int i = 0; i < 8; i++) s[i] = h_in[i];
  for (int r = 0; r < 64; r++) {
    const uint32_t e = s[4], a = s[0];
    const uint32_t t1 = s[7] + (rr(e, 6) ^ rr(e, 11) ^ rr(e, 25)) + ((e & (s[5] ^ s[6])) ^ s[6]) + kShaRc[r] + w[r];
    const uint32_t t2 = (rr(a, 2) ^ rr(a, 13) ^ rr(a, 22)) + (((a ^ s[1]) & (a ^ s[2])) ^ a);
    for (int i = 7; i > 0; i--) s[i] = s[i - 1];
    s[4] += t1;
    s[0] = t1 + t2;
  }
  for (int i = 0; i < 8; i++) out[i] = h_in[i] + s[i];
}

void keccak_f(uint64_t s[25]) {
  static const int rho[25] = {0,  36, 3,  41, 18, 1,  44, 10, 45, 2,  62, 6, 43,
                              15, 61, 28, 55, 25, 21, 56, 27, 20, 39, 8,  14};  // r[x][y] at 5x + y
  static const uint64_t rc[24] = {
      0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808Aull, 0x8000000080008000ull,
      0x000000000000808Bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
      0x000000000000008Aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000Aull,
      0x000000008000808Bull, 0x800000000000008Bull, 0x8000000000008089ull, 0x8000000000008003ull,
      0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800Aull, 0x800000008000000Aull,
      0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};
  auto rotl = [](uint64_t v, int n) { return n ? (v << n) | (v >> (64 - n)) : v; };
  for (int r = 0; r < 24; r++) {
    uint64_t c[5], b[25];
    for (int x = 0; x < 5; x++) c[x] = s[x] ^ s[x + 5] ^ s[x + 10] ^ s[x + 15] ^ s[x + 20];
    for (int l = 0; l < 25; l++) s[l] ^= c[(l % 5 + 4) % 5] ^ rotl(c[(l % 5 + 1) % 5], 1);
    for (int x = 0; x < 5; x++)  // rho, then pi: lane (x, y) moves to (y, 2x + 3y)
      for (int y = 0; y < 5; y++) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl(s[x + 5 * y], rho[5 * x + y]);
    for (int y = 0; y < 5; y++)
      for (int x = 0; x < 5; x++) s[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
    s[0] ^= rc[r];
  }
}

const Statement& statement(int hash) {
  static std::once_flag once[4];
  static std::unique_ptr<Statement> s[4];
  const int k = known_hash(hash) ? hash : 0;
  std::call_once(once[k], [k] {
    s[k].reset(new Statement(k == kHashSha256 ? build_sha256() : is_keccak(k) ? build_keccak(k == kHashKeccak3) : build()));
  });
  return *s[k];
}

std::array<uint8_t, 32> statement_digest(int hash, int m) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::array<uint8_t, 32>> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find({hash, m});
  if (it != cache.end()) return it->second;
  const Statement& st = statement(hash);
  const int kk = 1 << st.k_log;
  B3 h;
  h.update("flock-r1cs-stmt-v1", 18);
  put_u64(h, (uint64_t)m);
  put_u64(h, (uint64_t)st.k_log);
  put_u64(h, kKSkip);
  uint8_t row_major = 0;
  h.update(&row_major, 1);
  put_matrix(h, kk, &st.a_ptr, &st.a_col);
  put_matrix(h, kk, &st.b_ptr, &st.b_col);
  put_matrix(h, kk, nullptr, nullptr);  // C = I
  std::array<uint8_t, 32> d;
  h.digest(d.data());
  cache[{hash, m}] = d;
  return d;
}

// ----------------------------------------------------------------- ladder --
namespace {
struct Row { int rate, k, q, g, fg, ood; };
struct Levels {
  std::vector<Row> rows;
  int yr;
};
struct Entry {
  int m;
  Levels lv;
};
const std::vector<Entry>& entries() {
  static const std::vector<Entry> e = {
#include "ligerito_configs.inc"
  };
  return e;
}
}  // namespace

const Ladder* ladder_for(int m) {
  static std::mutex mu;
  static std::map<int, Ladder> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(m);
  if (it != cache.end()) return &it->second;
  for (const Entry& e : entries()) {
    if (e.m != m) continue;
    Ladder l;
    const std::vector<Row>& rows = e.lv.rows;
    l.initial_k = rows[0].k;
    l.yr_log_n = e.lv.yr;
    for (size_t i = 0; i < rows.size(); i++) {
      l.rate.push_back(rows[i].rate);
      if (i) l.ks.push_back(rows[i].k);
      l.queries.push_back(rows[i].q);
      l.grind.push_back(rows[i].g);
      l.fold_grind.push_back(rows[i].fg);
      l.ood.push_back(rows[i].ood);
    }
    return &(cache[m] = l);
  }
  return nullptr;
}

std::vector<size_t> sample_distinct_queries(Transcript& tr, size_t block_len, size_t count) {
  std::vector<size_t> q;
  std::set<size_t> seen;
  while (q.size() < count) {
    size_t v = (size_t)(tr.sample().lo % block_len);
    if (seen.insert(v).second) q.push_back(v);
  }
  std::sort(q.begin(), q.end());
  return q;
}

size_t ceil_log2(size_t n) {
  if (n <= 1) return 0;
  size_t v = n - 1, l = 0;
  while (v) { l++; v >>= 1; }
  return l;
}

std::vector<f128> small_consts() {
  const f128* P = phi8_table();
  return {P[0xF7], P[0x53], P[0xB5]};
}

std::vector<f128> medium_consts() {
  std::vector<f128> v;
  for (int sh : {1, 2, 4, 8}) {
    f128 g = mk(1ull << sh, 0);
    v.push_back(hmul(g, hinv(fx(hone(), g))));
  }
  return v;
}

// ---------------------------------------------------------------- encode --
namespace {
struct Enc {
  std::vector<uint8_t> o;
  void u32(uint32_t v) { for (int i = 0; i < 4; i++) o.push_back((uint8_t)(v >> (8 * i))); }
  void u64(uint64_t v) { for (int i = 0; i < 8; i++) o.push_back((uint8_t)(v >> (8 * i))); }
  void f(f128 v) { u64(v.lo); u64(v.hi); }
  void h(const H32& v) { o.insert(o.end(), v.begin(), v.end()); }
  void fs(const std::vector<f128>& v) { u64(v.size()); for (auto& x : v) f(x); }
  void hs(const std::vector<H32>& v) { u64(v.size()); for (auto& x : v) h(x); }
  void pairs(const std::vector<std::pair<f128, f128>>& v) { u64(v.size()); for (auto& x : v) { f(x.first); f(x.second); } }
  void open(const Opening& p) { u64(p.rows.size()); for (auto& r : p.rows) fs(r); hs(p.proof); }
};
}  // namespace

std::vector<uint8_t> encode(const Proof& p) {
  Enc e;
  e.o.reserve(512 * 1024);
  // R1csProofBundleLigerito (flavor 2) or ChainProofBundleLigerito (flavor 3:
  // hash_kind first, the shift proof after the lincheck, the endpoints last;
  // proof_io.rs:144-157, chain_common.rs:247-253).  A Merkle-path proof has
  // no bundle type in the reference: its bytes are bincode of (Commitment,
  // MerklePathProofLigerito { zerocheck, lincheck, shift, pcs_open }), as the
  // reference's tests serialise them (r1cs_hashes/sha2.rs:2519-2526).
  if (!p.merkle) {
    for (char c : std::string("FLOCK")) e.o.push_back((uint8_t)c);
    e.o.push_back(4);
    e.o.push_back(p.chain ? 3 : 2);
  }
  if (p.chain) e.u32(p.chain_kind);  // HashKind: Blake3 = 0, Sha2 = 1
  e.h(p.root);
  e.u64(p.m);
  e.u64(1);  // log_inv_rate
  e.u64(6);  // log_batch_size
  e.u32(0);  // profile Fast
  e.u32((uint32_t)p.merkle_fn);  // merkle hash: 0 Sha256, 1 Blake3
  e.fs(p.r1_ab);
  e.fs(p.r1_c);
  e.pairs(p.zc_rounds);
  e.f(p.fa);
  e.f(p.fb);
  e.f(p.fc);
  e.pairs(p.lc_rounds);
  e.fs(p.z_partial);
  if (p.chain) {
    e.pairs(p.shift_rounds);
    e.f(p.g_at_point);
  }
  if (p.merkle) {
    e.u64(p.mp_rounds.size());
    for (const auto& q : p.mp_rounds)
      for (const f128& v : q) e.f(v);
    e.f(p.g_at_point);
  }
  e.u64(p.s_hat_v.size());
  for (auto& s : p.s_hat_v) e.fs(s);
  e.h(p.lig_root);
  e.open(p.initial);
  e.hs(p.roots);
  e.u64(p.levels.size());
  for (auto& l : p.levels) e.open(l);
  e.fs(p.yr);
  e.open(p.final_open);
  e.pairs(p.sc_msgs);
  e.u64(p.grind_nonces.size());
  for (auto v : p.grind_nonces) e.u64(v);
  e.fs(p.ood);
  e.u64(p.fold_nonces.size());
  for (auto v : p.fold_nonces) e.u64(v);
  if (p.chain) {
    // Vec<bool>: u64 length, one byte per bit of the region's physical layout
    for (const uint64_t* end : {p.end0, p.end_last}) {
      e.u64((uint64_t)p.end_bits);
      for (int i = 0; i < p.end_bits; i++) e.o.push_back((uint8_t)((end[i / 64] >> (i % 64)) & 1));
    }
  }
  return e.o;
}

}  // namespace flock
