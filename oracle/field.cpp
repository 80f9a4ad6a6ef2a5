// Field arithmetic of the oracle (test infrastructure; see flockref.hpp).
// GF(2^128): crates/flock-core/src/field/gf2_128.rs:22-265 (mul, ghash_reduce,
// inv), gf2_128/portable.rs:1-38 (clmul64).  GF(2^8): field/gf2_8.rs:20-140.
// phi_8: field/phi8.rs:18-1050 — the table is a GF(2)-linear field
// embedding, so it is carried here as the images of the eight basis bytes
// 1,2,4,...,128 (verbatim table entries 1,2,4,...,128) and expanded by
// linearity; tests pin the expansion against all 256 reference entries.
#include "flockref.hpp"
#include <cstdlib>
#include <thread>
#if defined(__PCLMUL__)
#include <wmmintrin.h>
#include <emmintrin.h>
#endif

namespace flockref {

static inline void clmul64(uint64_t a, uint64_t b, uint64_t& lo, uint64_t& hi) {
#if defined(__PCLMUL__)
  __m128i r = _mm_clmulepi64_si128(_mm_set_epi64x(0, (long long)a), _mm_set_epi64x(0, (long long)b), 0);
  lo = (uint64_t)_mm_cvtsi128_si64(r);
  hi = (uint64_t)_mm_cvtsi128_si64(_mm_unpackhi_epi64(r, r));
#else
  lo = 0; hi = 0;
  for (int i = 0; i < 64; i++) {
    if ((a >> i) & 1) {
      lo ^= b << i;
      if (i) hi ^= b >> (64 - i);
    }
  }
#endif
}

U256 mul_unreduced(F128 a, F128 b) {
  uint64_t ll0, ll1, lh0, lh1, hl0, hl1, hh0, hh1;
  clmul64(a.lo, b.lo, ll0, ll1);
  clmul64(a.lo, b.hi, lh0, lh1);
  clmul64(a.hi, b.lo, hl0, hl1);
  clmul64(a.hi, b.hi, hh0, hh1);
  U256 u;
  u.r0 = ll0;
  u.r1 = ll1 ^ lh0 ^ hl0;
  u.r2 = hh0 ^ lh1 ^ hl1;
  u.r3 = hh1;
  return u;
}

F128 ghash_reduce(uint64_t r0, uint64_t r1, uint64_t r2, uint64_t r3) {
  uint64_t s1_lo = r2 << 1, s1_hi = (r3 << 1) | (r2 >> 63);
  uint64_t s2_lo = r2 << 2, s2_hi = (r3 << 2) | (r2 >> 62);
  uint64_t s7_lo = r2 << 7, s7_hi = (r3 << 7) | (r2 >> 57);
  uint64_t t_lo = r2 ^ s1_lo ^ s2_lo ^ s7_lo;
  uint64_t t_hi = r3 ^ s1_hi ^ s2_hi ^ s7_hi;
  uint64_t ov = (r3 >> 63) ^ (r3 >> 62) ^ (r3 >> 57);
  uint64_t corr = ov ^ (ov << 1) ^ (ov << 2) ^ (ov << 7);
  return F128(r0 ^ t_lo ^ corr, r1 ^ t_hi);
}

F128 operator*(F128 a, F128 b) {
  U256 u = mul_unreduced(a, b);
  return ghash_reduce(u.r0, u.r1, u.r2, u.r3);
}

// x^(2^128 - 2) by square-and-multiply; zero maps to zero (gf2_128.rs:84-97).
F128 f128_inv(F128 a) {
  F128 result = ONE, sq = a;
  // exponent 2^128 - 2: bits 1..127 set
  sq = sq * sq;  // a^2
  for (int i = 1; i < 128; i++) {
    result = result * sq;
    sq = sq * sq;
  }
  return result;
}

uint8_t gf8_mul(uint8_t a, uint8_t b) {
  uint16_t acc = 0;
  for (int i = 0; i < 8; i++)
    if ((a >> i) & 1) acc ^= (uint16_t)((uint16_t)b << i);
  uint16_t h = acc >> 8;
  uint16_t t = (acc & 0xff) ^ h ^ (h << 1) ^ (h << 3) ^ (h << 4);
  uint16_t h2 = t >> 8;
  return (uint8_t)((t & 0xff) ^ h2 ^ (h2 << 1) ^ (h2 << 3) ^ (h2 << 4));
}

uint8_t gf8_inv(uint8_t a) {
  uint8_t result = 1, sq = a;
  for (int i = 0; i < 8; i++) {
    if ((0xFE >> i) & 1) result = gf8_mul(result, sq);
    sq = gf8_mul(sq, sq);
  }
  return result;
}

// Images of bytes 1,2,4,...,128 under phi_8 (field/phi8.rs entries 1,2,4,..,128).
static const F128 PHI8_BASIS[8] = {
    F128(0x0000000000000001ull, 0x0000000000000000ull),
    F128(0x6b8330483c2e9849ull, 0x0dcb364640a222feull),
    F128(0x7573da4a5f7710edull, 0x3d5bd35c94646a24ull),
    F128(0x41a12db1f974f3acull, 0x6d58c4e181f9199full),
    F128(0x5e2f716f4ede412full, 0xa72ec17764d7ced5ull),
    F128(0x5cb10fbabcf00118ull, 0x4d52354a3a3d8c86ull),
    F128(0x95ed1f57f3632d4dull, 0x553e92e8bc0ae9a7ull),
    F128(0x512625b1f09fa87eull, 0x93252331bf042b11ull),
};

static std::array<F128, 256> make_phi8() {
  std::array<F128, 256> t{};
  for (int v = 0; v < 256; v++) {
    F128 acc = ZERO;
    for (int b = 0; b < 8; b++)
      if ((v >> b) & 1) acc += PHI8_BASIS[b];
    t[v] = acc;
  }
  return t;
}
static const std::array<F128, 256> PHI8 = make_phi8();

F128 phi8(uint8_t v) { return PHI8[v]; }
const F128* phi8_table() { return PHI8.data(); }


int par_threads() {
  static const int n = [] {
    const char* e = std::getenv("FLOCKREF_THREADS");
    int v = e ? std::atoi(e) : 1;
    return v < 1 ? 1 : v > 256 ? 256 : v;
  }();
  return n;
}

void par_for(size_t n, const std::function<void(size_t, size_t, int)>& f) {
  const int t = par_threads();
  if (t == 1 || n < 2) {
    f(0, n, 0);
    return;
  }
  std::vector<std::thread> th;
  for (int i = 0; i < t; i++) {
    const size_t b = n * i / t, e = n * (i + 1) / t;
    th.emplace_back([&f, b, e, i] { f(b, e, i); });
  }
  for (auto& x : th) x.join();
}

}  // namespace flockref
