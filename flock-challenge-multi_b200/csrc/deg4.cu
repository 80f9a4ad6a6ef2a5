// Degree-4 zerocheck round 1 (crates/flock-core/src/zerocheck/
// univariate_skip_deg4.rs, round1_deg4_naive) on the device.
//
// For every 64-bit row x of the bit vectors a, b, c, d, z (2^m bits, row x =
// indices 64x..64x+63) each factor is extended from S = {0..63} to the 192
// points lambda = 64..255 of GF(2^8); the message is
//   p_abcd[l] = sum_x eq(r[6..], x) phi8(a b c d at 64 + l)
//   p_z[l]    = sum_x eq(r[6..], x) phi8(z at 64 + l).
// phi8 is additive, so both reduce to sums of eq over row subsets:
//   H[l][k] = sum of eq_x over rows whose product at 64 + l has bit k set,
//   p_abcd[l] = sum_k phi8(2^k) H[l][k];
//   Zs[s] = sum of eq_x over rows whose z bit s is set,
//   p_z[l] = sum_s phi8(M[64 + l][s]) Zs[s]   (the extension is GF(2)-linear),
// finished on the host from the 1536 + 64 device sums.
//
// The extension of a row is GF(2)-linear in its 64 bits: M[lambda][s] is the
// value at lambda of the polynomial of degree < 64 that is 1 at node s and 0
// at the other nodes of S (S's novel basis is the prefix of V8's, so inv-NTT
// on S then fwd-NTT on V8 is this interpolation).  It is applied with 4-bit
// windows: Tab[w][nibble] holds the 192 extension bytes of a nibble at bits
// 4w..4w+3, packed four lambdas to a u32, so a factor's four bytes at one
// lambda quad cost 16 shared-memory loads.  The products a b c d are formed in
// the log domain (log / exp byte tables, a zero factor detected by its log).
//
// Mapping: a CTA of 8 warps takes 32 rows at a time, one row per lane; warp w
// owns the lambda quads 6w..6w+5 (24 lambdas) and the z bits 8w..8w+7.  Per
// quad the warp takes 32 ballots of the product bits (ballot t = lambda 4q +
// t / 8, bit t mod 8); lane t keeps ballot t, a mask of the 32 rows, and adds
// the eq sum of those rows from four 8-row subset-sum tables (256 entries each,
// built once per 32-row chunk by the CTA).  Every lane thus owns 6 of the
// 1536 (lambda, bit) sums in registers; they are XOR-ed into global memory
// once, at the end.
#include "kernels.cuh"
#include "host.hpp"

namespace {
constexpr int kThreads = 256;
constexpr int kQuadsPerWarp = 6;
constexpr int kRowWords = 49;  // u32 per (window, nibble) row: 48 quads + 1 pad
constexpr int kTabWords = 16 * 16 * kRowWords;
constexpr int kLogZero = 2048;  // log of 0: any sum holding it is >= 2048
constexpr size_t kSmem = (size_t)kTabWords * 4 + 256 * 2 + 1024 + 2 * 4 * 256 * sizeof(f128);

__global__ void __launch_bounds__(kThreads, 2) k_round1_deg4(const uint64_t* __restrict__ a,
                                                             const uint64_t* __restrict__ b,
                                                             const uint64_t* __restrict__ c,
                                                             const uint64_t* __restrict__ d,
                                                             const uint64_t* __restrict__ z,
                                                             const f128* __restrict__ eq, size_t n_rows,
                                                             const uint32_t* __restrict__ tab_g,
                                                             const uint16_t* __restrict__ log_g,
                                                             const uint8_t* __restrict__ exp_g,
                                                             f128* __restrict__ H, f128* __restrict__ Zs) {
  extern __shared__ __align__(16) uint8_t sm[];
  f128* T = reinterpret_cast<f128*>(sm);                                   // [2][4][256]
  uint32_t* tab = reinterpret_cast<uint32_t*>(sm + 2 * 4 * 256 * sizeof(f128));  // [16][16][kRowWords]
  uint16_t* lg = reinterpret_cast<uint16_t*>(tab + kTabWords);             // [256]
  uint8_t* ex = reinterpret_cast<uint8_t*>(lg + 256);                      // [1024]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < kTabWords; i += kThreads) tab[i] = tab_g[i];
  for (int i = tid; i < 256; i += kThreads) lg[i] = log_g[i];
  for (int i = tid; i < 1024; i += kThreads) ex[i] = exp_g[i];
  f128 acc[kQuadsPerWarp];
#pragma unroll
  for (int j = 0; j < kQuadsPerWarp; j++) acc[j] = mk(0, 0);
  f128 accz = mk(0, 0);
  const size_t n_chunks = (n_rows + 31) / 32;
  int buf = 0;
  for (size_t ch = blockIdx.x; ch < n_chunks; ch += gridDim.x, buf ^= 1) {
    // subset sums of the chunk's eq values, four groups of 8 rows
    f128* Tb = T + buf * 1024;
    for (int e = tid; e < 1024; e += kThreads) {
      const int g = e >> 8, idx = e & 255;
      f128 v = mk(0, 0);
#pragma unroll
      for (int bit = 0; bit < 8; bit++) {
        const size_t row = ch * 32 + 8 * g + bit;
        if (((idx >> bit) & 1) && row < n_rows) v = fx(v, ldg(eq + row));
      }
      Tb[e] = v;
    }
    // (Tb was last read two chunks ago, before the previous barrier)
    __syncthreads();
    const size_t row = ch * 32 + lane;
    const bool live = row < n_rows;
    const uint64_t va = live ? a[row] : 0, vb = live ? b[row] : 0, vc = live ? c[row] : 0,
                   vd = live ? d[row] : 0, vz = live ? z[row] : 0;
#pragma unroll
    for (int j = 0; j < kQuadsPerWarp; j++) {
      const int q = kQuadsPerWarp * warp + j;
      uint32_t ea = 0, eb = 0, ec = 0, ed = 0;
#pragma unroll
      for (int w = 0; w < 16; w++) {
        const uint32_t* tw = tab + w * 16 * kRowWords + q;
        ea ^= tw[((va >> (4 * w)) & 15) * kRowWords];
        eb ^= tw[((vb >> (4 * w)) & 15) * kRowWords];
        ec ^= tw[((vc >> (4 * w)) & 15) * kRowWords];
        ed ^= tw[((vd >> (4 * w)) & 15) * kRowWords];
      }
      uint32_t p4 = 0;
#pragma unroll
      for (int t = 0; t < 4; t++) {
        const int s = lg[(ea >> (8 * t)) & 255] + lg[(eb >> (8 * t)) & 255] + lg[(ec >> (8 * t)) & 255] +
                      lg[(ed >> (8 * t)) & 255];
        p4 |= (uint32_t)(s < 1024 ? ex[s] : 0) << (8 * t);
      }
      uint32_t mine = 0;
#pragma unroll
      for (int t = 0; t < 32; t++) {
        const uint32_t m = __ballot_sync(0xffffffffu, (p4 >> t) & 1);
        if (lane == t) mine = m;
      }
      acc[j] = fx(acc[j], fx(fx(Tb[mine & 255], Tb[256 + ((mine >> 8) & 255)]),
                             fx(Tb[512 + ((mine >> 16) & 255)], Tb[768 + (mine >> 24)])));
    }
    // z: warp w folds bits 8w..8w+7; lane l takes bit 8w + l / 4, row group l % 4
    uint32_t mz = 0;
#pragma unroll
    for (int t = 0; t < 8; t++) {
      const uint32_t m = __ballot_sync(0xffffffffu, (vz >> (8 * warp + t)) & 1);
      if ((lane >> 2) == t) mz = m;
    }
    const int g = lane & 3;
    accz = fx(accz, Tb[256 * g + ((mz >> (8 * g)) & 255)]);
  }
#pragma unroll
  for (int j = 0; j < kQuadsPerWarp; j++) {
    // lane t of quad q: lambda 4q + t / 8, bit t mod 8
    const int l = 4 * (kQuadsPerWarp * warp + j) + (lane >> 3);
    if (!fz(acc[j])) atomic_xor128(H + 8 * l + (lane & 7), acc[j]);
  }
  accz.lo ^= __shfl_xor_sync(0xffffffffu, accz.lo, 1);
  accz.hi ^= __shfl_xor_sync(0xffffffffu, accz.hi, 1);
  accz.lo ^= __shfl_xor_sync(0xffffffffu, accz.lo, 2);
  accz.hi ^= __shfl_xor_sync(0xffffffffu, accz.hi, 2);
  if ((lane & 3) == 0 && !fz(accz)) atomic_xor128(Zs + 8 * warp + (lane >> 2), accz);
}

uint8_t gf8_pow(uint8_t x, int e) {
  uint8_t r = 1;
  for (; e; e >>= 1, x = flock::hgf8_mul(x, x))
    if (e & 1) r = flock::hgf8_mul(r, x);
  return r;
}
}  // namespace

// M[l][s] (l < 192): the value at 64 + l of the Lagrange basis polynomial of
// node s over the nodes 0..63
const std::vector<uint8_t>& deg4_extension() {
  static const std::vector<uint8_t> M = [] {
    std::vector<uint8_t> m(192 * 64);
    for (int s = 0; s < 64; s++) {
      uint8_t den = 1;
      for (int j = 0; j < 64; j++)
        if (j != s) den = flock::hgf8_mul(den, (uint8_t)(s ^ j));
      const uint8_t inv = gf8_pow(den, 254);
      for (int l = 0; l < 192; l++) {
        uint8_t num = 1;
        for (int j = 0; j < 64; j++)
          if (j != s) num = flock::hgf8_mul(num, (uint8_t)((64 + l) ^ j));
        m[l * 64 + s] = flock::hgf8_mul(num, inv);
      }
    }
    return m;
  }();
  return M;
}

size_t deg4_tables_bytes() { return (size_t)kTabWords * 4 + 256 * 2 + 1024; }

void deg4_build_tables(uint8_t* host) {
  const std::vector<uint8_t>& M = deg4_extension();
  uint32_t* tab = reinterpret_cast<uint32_t*>(host);
  memset(host, 0, deg4_tables_bytes());
  for (int w = 0; w < 16; w++)
    for (int nib = 0; nib < 16; nib++)
      for (int q = 0; q < 48; q++) {
        uint32_t v = 0;
        for (int t = 0; t < 4; t++) {
          uint8_t e = 0;
          for (int bit = 0; bit < 4; bit++)
            if ((nib >> bit) & 1) e ^= M[(4 * q + t) * 64 + 4 * w + bit];
          v |= (uint32_t)e << (8 * t);
        }
        tab[(w * 16 + nib) * kRowWords + q] = v;
      }
  uint16_t* lg = reinterpret_cast<uint16_t*>(tab + kTabWords);
  uint8_t* ex = reinterpret_cast<uint8_t*>(lg + 256);
  lg[0] = kLogZero;
  uint8_t x = 1;  // generator 3 of GF(2^8)*
  for (int i = 0; i < 255; i++) {
    lg[x] = (uint16_t)i;
    x = flock::hgf8_mul(x, 3);
  }
  for (int i = 0; i < 1024; i++) ex[i] = gf8_pow(3, i % 255);
}

void round1_deg4(const uint64_t* a, const uint64_t* b, const uint64_t* c, const uint64_t* d, const uint64_t* z,
                 const f128* eq, size_t n_rows, const uint8_t* tables, f128* H, f128* Zs, int grid, cudaStream_t s) {
  const uint32_t* tab = reinterpret_cast<const uint32_t*>(tables);
  const uint16_t* lg = reinterpret_cast<const uint16_t*>(tab + kTabWords);
  const uint8_t* ex = reinterpret_cast<const uint8_t*>(lg + 256);
  CK(cudaFuncSetAttribute(k_round1_deg4, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
  const size_t n_chunks = (n_rows + 31) / 32;
  count_launch();
  k_round1_deg4<<<(unsigned)std::min<size_t>(n_chunks, (size_t)grid), kThreads, kSmem, s>>>(a, b, c, d, z, eq, n_rows,
                                                                                            tab, lg, ex, H, Zs);
}

void round1_deg4_finish(const f128* H, const f128* Zs, f128* p_abcd, f128* p_z) {
  const f128* phi = flock::phi8_table();
  const std::vector<uint8_t>& M = deg4_extension();
  for (int l = 0; l < 192; l++) {
    f128 pa = mk(0, 0), pz = mk(0, 0);
    for (int k = 0; k < 8; k++) pa = fx(pa, flock::hmul(phi[1 << k], H[8 * l + k]));
    for (int s = 0; s < 64; s++)
      if (M[l * 64 + s]) pz = fx(pz, flock::hmul(phi[M[l * 64 + s]], Zs[s]));
    p_abcd[l] = pa;
    p_z[l] = pz;
  }
}
