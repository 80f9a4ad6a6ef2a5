// Device arithmetic in GF(2^128) (GHASH polynomial x^128 + x^7 + x^2 + x + 1,
// lo = coefficients x^0..x^63) and GF(2^8) (AES polynomial 0x11B).
//
// Field semantics follow the reference's crates/flock-core/src/field/
// gf2_128.rs:22-265 (mul, ghash_reduce) and gf2_8.rs:20-140.  The GPU has no
// carry-less multiplier, so a 32x32 carry-less product is built from four
// interleaved bit classes (bit positions i mod 4) and sixteen 32x32->64
// integer multiplies: within one class pair at most 8 partial products land
// on a bit position, so the integer carries never reach the next same-class
// position and the parity of every class position is exact.  64x64 and
// 128x128 products use Karatsuba on top of it.
#pragma once
#include <cstdint>

struct __align__(16) f128 {
  uint64_t lo, hi;
};

__host__ __device__ __forceinline__ f128 mk(uint64_t lo, uint64_t hi) { f128 r; r.lo = lo; r.hi = hi; return r; }
__host__ __device__ __forceinline__ f128 fx(f128 a, f128 b) { return mk(a.lo ^ b.lo, a.hi ^ b.hi); }
__host__ __device__ __forceinline__ bool fz(f128 a) { return (a.lo | a.hi) == 0; }

__device__ __forceinline__ uint64_t clmul32(uint32_t x, uint32_t y) {
  const uint32_t m0 = 0x11111111u, m1 = 0x22222222u, m2 = 0x44444444u, m3 = 0x88888888u;
  uint32_t x0 = x & m0, x1 = x & m1, x2 = x & m2, x3 = x & m3;
  uint32_t y0 = y & m0, y1 = y & m1, y2 = y & m2, y3 = y & m3;
  uint64_t z0 = ((uint64_t)x0 * y0) ^ ((uint64_t)x1 * y3) ^ ((uint64_t)x2 * y2) ^ ((uint64_t)x3 * y1);
  uint64_t z1 = ((uint64_t)x0 * y1) ^ ((uint64_t)x1 * y0) ^ ((uint64_t)x2 * y3) ^ ((uint64_t)x3 * y2);
  uint64_t z2 = ((uint64_t)x0 * y2) ^ ((uint64_t)x1 * y1) ^ ((uint64_t)x2 * y0) ^ ((uint64_t)x3 * y3);
  uint64_t z3 = ((uint64_t)x0 * y3) ^ ((uint64_t)x1 * y2) ^ ((uint64_t)x2 * y1) ^ ((uint64_t)x3 * y0);
  return (z0 & 0x1111111111111111ull) | (z1 & 0x2222222222222222ull) |
         (z2 & 0x4444444444444444ull) | (z3 & 0x8888888888888888ull);
}

// 64x64 -> 128 carry-less product (Karatsuba over clmul32)
__device__ __forceinline__ void clmul64(uint64_t a, uint64_t b, uint64_t& lo, uint64_t& hi) {
  uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  uint64_t l = clmul32(a0, b0), h = clmul32(a1, b1);
  uint64_t m = clmul32(a0 ^ a1, b0 ^ b1) ^ l ^ h;
  lo = l ^ (m << 32);
  hi = h ^ (m >> 32);
}

struct u256 { uint64_t r0, r1, r2, r3; };

__device__ __forceinline__ u256 mul_wide(f128 a, f128 b) {
  uint64_t l0, l1, h0, h1, m0, m1;
  clmul64(a.lo, b.lo, l0, l1);
  clmul64(a.hi, b.hi, h0, h1);
  clmul64(a.lo ^ a.hi, b.lo ^ b.hi, m0, m1);
  m0 ^= l0 ^ h0;
  m1 ^= l1 ^ h1;
  u256 u;
  u.r0 = l0;
  u.r1 = l1 ^ m0;
  u.r2 = h0 ^ m1;
  u.r3 = h1;
  return u;
}

__host__ __device__ __forceinline__ f128 reduce256(uint64_t r0, uint64_t r1, uint64_t r2, uint64_t r3) {
  uint64_t t_lo = r2 ^ (r2 << 1) ^ (r2 << 2) ^ (r2 << 7);
  uint64_t t_hi = r3 ^ ((r3 << 1) | (r2 >> 63)) ^ ((r3 << 2) | (r2 >> 62)) ^ ((r3 << 7) | (r2 >> 57));
  uint64_t ov = (r3 >> 63) ^ (r3 >> 62) ^ (r3 >> 57);
  uint64_t corr = ov ^ (ov << 1) ^ (ov << 2) ^ (ov << 7);
  return mk(r0 ^ t_lo ^ corr, r1 ^ t_hi);
}

__device__ __forceinline__ f128 reduce(u256 u) { return reduce256(u.r0, u.r1, u.r2, u.r3); }
__device__ __forceinline__ f128 fmul(f128 a, f128 b) { return reduce(mul_wide(a, b)); }
__device__ __forceinline__ void acc_wide(u256& acc, u256 v) { acc.r0 ^= v.r0; acc.r1 ^= v.r1; acc.r2 ^= v.r2; acc.r3 ^= v.r3; }
__device__ __forceinline__ u256 zero256() { u256 u; u.r0 = u.r1 = u.r2 = u.r3 = 0; return u; }

// multiply by x^k (0 <= k < 64) with reduction
__host__ __device__ __forceinline__ f128 mul_xk(f128 a, int k) {
  if (k == 0) return a;
  uint64_t r0 = a.lo << k, r1 = (a.hi << k) | (a.lo >> (64 - k)), r2 = a.hi >> (64 - k);
  return reduce256(r0, r1, r2, 0);
}

__device__ __forceinline__ f128 ld(const f128* p) {
  ulonglong2 v = *reinterpret_cast<const ulonglong2*>(p);
  return mk(v.x, v.y);
}
__device__ __forceinline__ f128 ldg(const f128* p) {
  ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p));
  return mk(v.x, v.y);
}
__device__ __forceinline__ void st(f128* p, f128 v) {
  *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(v.lo, v.hi);
}

// ---- warp / block XOR reductions ----
__device__ __forceinline__ uint64_t shfl_xor64(uint64_t v, int m) {
  return __shfl_xor_sync(0xffffffffu, v, m);
}
__device__ __forceinline__ f128 warp_xor(f128 v) {
#pragma unroll
  for (int m = 16; m; m >>= 1) { v.lo ^= shfl_xor64(v.lo, m); v.hi ^= shfl_xor64(v.hi, m); }
  return v;
}
__device__ __forceinline__ u256 warp_xor(u256 v) {
#pragma unroll
  for (int m = 16; m; m >>= 1) {
    v.r0 ^= shfl_xor64(v.r0, m); v.r1 ^= shfl_xor64(v.r1, m);
    v.r2 ^= shfl_xor64(v.r2, m); v.r3 ^= shfl_xor64(v.r3, m);
  }
  return v;
}
// XOR into a global 128-bit slot (order-independent => deterministic)
__device__ __forceinline__ void atomic_xor128(f128* p, f128 v) {
  if (v.lo) atomicXor(reinterpret_cast<unsigned long long*>(&p->lo), (unsigned long long)v.lo);
  if (v.hi) atomicXor(reinterpret_cast<unsigned long long*>(&p->hi), (unsigned long long)v.hi);
}

// ---- multiplication by a constant through an 8-bit window table ----
// T[p][v] = E * v(x) * x^(8p): E * y = XOR over the 16 bytes y_p of T[p][y_p].
// Built cooperatively by a CTA (8 doubling levels); 64 KiB of shared memory.
struct MulTab8 {
  f128 t[16][256];
};
__device__ __forceinline__ void multab_build(MulTab8* T, f128 E) {
  for (int i = threadIdx.x; i < 16 * 8; i += blockDim.x) {
    int p = i >> 3, j = i & 7;
    f128 v = E;
    for (int q = 0; q < p; q++) v = mul_xk(v, 8);
    T->t[p][1 << j] = mul_xk(v, j);
    if (j == 0) T->t[p][0] = mk(0, 0);
  }
  __syncthreads();
  for (int lvl = 1; lvl < 8; lvl++) {
    int base = 1 << lvl, cnt = base - 1;  // entries base+1 .. 2*base-1
    for (int i = threadIdx.x; i < 16 * cnt; i += blockDim.x) {
      int p = i / cnt, w = 1 + i % cnt;
      T->t[p][base + w] = fx(T->t[p][w], T->t[p][base]);
    }
    __syncthreads();
  }
}
__device__ __forceinline__ f128 multab_mul(const MulTab8* T, f128 y) {
  f128 acc = mk(0, 0);
#pragma unroll
  for (int p = 0; p < 8; p++) {
    acc = fx(acc, T->t[p][(y.lo >> (8 * p)) & 0xFF]);
    acc = fx(acc, T->t[8 + p][(y.hi >> (8 * p)) & 0xFF]);
  }
  return acc;
}

// ---- multiplication by a warp-uniform constant through a 4-bit window table ----
// Entry n of window w is t * n(x) * x^(4w); a product t * y is the XOR of 32
// lookups, one per nibble of y.  The halves of an entry sit in separate
// 8-byte arrays and window w's entries are permuted by n -> n ^ (w mod 16):
// a window's 16 entries of one half fill the 32 banks exactly once, so a
// warp's lookups into one window never conflict, whatever the nibbles, and
// the builder's stores (thread w writes window w) do not conflict either.
// 8 KiB per table; 32 lookups of 8 bytes per product on the shared-memory
// pipe and no integer multiplies.
struct Tab4 {
  uint64_t lo[32][16], hi[32][16];
};
constexpr size_t kTab4Bytes = sizeof(Tab4);  // 8 KiB

__device__ __forceinline__ f128 mul_x128(f128 a, int k) {  // a * x^k, 0 <= k < 128
  if (k >= 64) {
    a = reduce256(0, a.lo, a.hi, 0);
    k -= 64;
  }
  return mul_xk(a, k);
}
// Window w of the table of any GF(2)-linear map L from the images
// b_i = L(x^(4w + i)), i < 4 (the table of a product by t has b_i = t x^(4w+i)).
__device__ __forceinline__ void tab4_window(Tab4* T, int w, f128 b0, f128 b1, f128 b2, f128 b3) {
  f128 e[16];
  e[0] = mk(0, 0);
  e[1] = b0;
  e[2] = b1;
  e[3] = fx(b0, b1);
#pragma unroll
  for (int j = 4; j < 8; j++) e[j] = fx(e[j - 4], b2);
#pragma unroll
  for (int j = 8; j < 16; j++) e[j] = fx(e[j - 8], b3);
  const int r = w & 15;
#pragma unroll
  for (int j = 0; j < 16; j++) {
    T->lo[w][j ^ r] = e[j].lo;
    T->hi[w][j ^ r] = e[j].hi;
  }
}
// thread `lane` of the warp writes window `lane` of the table of t
__device__ __forceinline__ void tab4_build(Tab4* T, f128 t, int lane) {
  const f128 b0 = mul_x128(t, 4 * lane);
  tab4_window(T, lane, b0, mul_xk(b0, 1), mul_xk(b0, 2), mul_xk(b0, 3));
}

__device__ __forceinline__ f128 tab4_mul(const Tab4* T, f128 y) {
  uint64_t alo = 0, ahi = 0;
#pragma unroll
  for (int w = 0; w < 32; w++) {
    const uint64_t word = w < 16 ? y.lo : y.hi;
    const uint32_t n = ((uint32_t)(word >> (4 * (w & 15))) & 15u) ^ (uint32_t)(w & 15);
    alo ^= T->lo[w][n];
    ahi ^= T->hi[w][n];
  }
  return mk(alo, ahi);
}

// ---- products by a factor reused across many products ----
// The factor's side of the Karatsuba tree (its nine 32-bit operands) is
// split into the four bit classes once; each product then masks only its
// own operand.
struct ClassY {
  uint32_t c0, c1, c2, c3;
};
__device__ __forceinline__ ClassY classes_of(uint32_t y) {
  ClassY r;
  r.c0 = y & 0x11111111u;
  r.c1 = y & 0x22222222u;
  r.c2 = y & 0x44444444u;
  r.c3 = y & 0x88888888u;
  return r;
}
__device__ __forceinline__ uint64_t clmul32_c(uint32_t x, const ClassY& y) {
  const uint32_t x0 = x & 0x11111111u, x1 = x & 0x22222222u, x2 = x & 0x44444444u, x3 = x & 0x88888888u;
  uint64_t z0 = ((uint64_t)x0 * y.c0) ^ ((uint64_t)x1 * y.c3) ^ ((uint64_t)x2 * y.c2) ^ ((uint64_t)x3 * y.c1);
  uint64_t z1 = ((uint64_t)x0 * y.c1) ^ ((uint64_t)x1 * y.c0) ^ ((uint64_t)x2 * y.c3) ^ ((uint64_t)x3 * y.c2);
  uint64_t z2 = ((uint64_t)x0 * y.c2) ^ ((uint64_t)x1 * y.c1) ^ ((uint64_t)x2 * y.c0) ^ ((uint64_t)x3 * y.c3);
  uint64_t z3 = ((uint64_t)x0 * y.c3) ^ ((uint64_t)x1 * y.c2) ^ ((uint64_t)x2 * y.c1) ^ ((uint64_t)x3 * y.c0);
  return (z0 & 0x1111111111111111ull) | (z1 & 0x2222222222222222ull) | (z2 & 0x4444444444444444ull) |
         (z3 & 0x8888888888888888ull);
}
struct MulConst {
  ClassY k[9];  // (t0, t1, t0^t1), (t2, t3, t2^t3), (s0, s1, s0^s1), s = lo ^ hi
};
__device__ __forceinline__ MulConst mulconst(f128 t) {
  const uint32_t w0 = (uint32_t)t.lo, w1 = (uint32_t)(t.lo >> 32), w2 = (uint32_t)t.hi, w3 = (uint32_t)(t.hi >> 32);
  const uint32_t s0 = w0 ^ w2, s1 = w1 ^ w3;
  MulConst M;
  M.k[0] = classes_of(w0); M.k[1] = classes_of(w1); M.k[2] = classes_of(w0 ^ w1);
  M.k[3] = classes_of(w2); M.k[4] = classes_of(w3); M.k[5] = classes_of(w2 ^ w3);
  M.k[6] = classes_of(s0); M.k[7] = classes_of(s1); M.k[8] = classes_of(s0 ^ s1);
  return M;
}
__device__ __forceinline__ void clmul64_c(uint64_t a, const ClassY* y, uint64_t& lo, uint64_t& hi) {
  const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
  const uint64_t l = clmul32_c(a0, y[0]), h = clmul32_c(a1, y[1]);
  const uint64_t m = clmul32_c(a0 ^ a1, y[2]) ^ l ^ h;
  lo = l ^ (m << 32);
  hi = h ^ (m >> 32);
}
// a * t for the t that M was built from (same result as fmul(a, t))
__device__ __forceinline__ f128 fmul_c(f128 a, const MulConst& M) {
  uint64_t l0, l1, h0, h1, m0, m1;
  clmul64_c(a.lo, &M.k[0], l0, l1);
  clmul64_c(a.hi, &M.k[3], h0, h1);
  clmul64_c(a.lo ^ a.hi, &M.k[6], m0, m1);
  m0 ^= l0 ^ h0;
  m1 ^= l1 ^ h1;
  return reduce256(l0, l1 ^ m0, h0 ^ m1, h1);
}

// ---- GF(2^8) ----
__host__ __device__ __forceinline__ uint8_t gf8_mul_slow(uint8_t a, uint8_t b) {
  uint32_t acc = 0;
  for (int i = 0; i < 8; i++)
    if ((a >> i) & 1) acc ^= (uint32_t)b << i;
  for (int i = 14; i >= 8; i--)
    if ((acc >> i) & 1) acc ^= 0x11Bu << (i - 8);
  return (uint8_t)acc;
}
