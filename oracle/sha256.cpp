// SHA-256-compression R1CS of the oracle (test infrastructure; see
// flockref.hpp).  Restates crates/flock-prover/src/r1cs_hashes/sha2.rs:
// layout constants and bit accessors :56-181 (the I/O-aligned layout: H_in
// slot 0, H_out slot 1, M at bit 512, Z_CONST after the output carries),
// the symbolic XOR-support words and inlined adders :183-329,
// build_matrices :332-520, the boolean block witness :523-606,
// sha256_compress :1502-1546, min_n_blocks_log :1217-1221, the padded
// prove_fast witness :1185-1209 (padding blocks hold the compression of the
// all-zero (h_in, m)), and the benchmark inputs of
// crates/flock-prover/benches/sha2_proof.rs:56-71 (one SplitMix64 stream,
// 8 + 16 draws per compression).
//
// Unlike the BLAKE3 restatement, a = A_0 z and b = B_0 z are computed here
// from the matrices (apply_block_diag), so the product's fused row witness is
// checked against the matrices themselves.
#include "flockref.hpp"
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>

namespace flockref {
namespace sha {

const uint32_t IV[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                        0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
const uint32_t RC[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2,
};

namespace {
constexpr int kRounds = 64, kSched = 48, kAddsRound = 7, kAddsSched = 3, kCarries = 31;
constexpr int H_BASE = 0, H_OUT_BASE = 256, M_BASE = 512;
constexpr int CH_BASE = M_BASE + 16 * 32;                               // 1024
constexpr int MAJ_BASE = CH_BASE + kRounds * 32;                        // 3072
constexpr int RCARRY_BASE = MAJ_BASE + kRounds * 32;                    // 5120
constexpr int W_BASE = RCARRY_BASE + kRounds * kAddsRound * kCarries;  // 19008
constexpr int SCARRY_BASE = W_BASE + kSched * 32;                       // 20544
constexpr int T1_BASE = SCARRY_BASE + kSched * kAddsSched * kCarries;   // 25008
constexpr int ENEW_BASE = T1_BASE + kRounds * 32;                       // 27056
constexpr int ANEW_BASE = ENEW_BASE + kRounds * 32;                     // 29104
constexpr int OCARRY_BASE = ANEW_BASE + kRounds * 32;                   // 31152
static_assert(OCARRY_BASE + 8 * kCarries == Z_CONST_POS, "layout");
static_assert(Z_CONST_POS + 1 == USEFUL_BITS, "layout");

inline int h_bit(int w, int b) { return H_BASE + 32 * w + b; }
inline int h_out_bit(int w, int b) { return H_OUT_BASE + 32 * w + b; }
inline int m_bit(int i, int b) { return M_BASE + 32 * i + b; }
inline int ch_bit(int r, int b) { return CH_BASE + 32 * r + b; }
inline int maj_bit(int r, int b) { return MAJ_BASE + 32 * r + b; }
inline int rcarry_bit(int r, int add, int b) { return RCARRY_BASE + r * kAddsRound * kCarries + add * kCarries + b; }
inline int w_bit(int t, int b) { return t < 16 ? m_bit(t, b) : W_BASE + (t - 16) * 32 + b; }
inline int scarry_bit(int t, int add, int b) { return SCARRY_BASE + (t - 16) * kAddsSched * kCarries + add * kCarries + b; }
inline int t1_bit(int r, int b) { return T1_BASE + 32 * r + b; }
inline int enew_bit(int r, int b) { return ENEW_BASE + 32 * r + b; }
inline int anew_bit(int r, int b) { return ANEW_BASE + 32 * r + b; }
inline int ocarry_bit(int w, int b) { return OCARRY_BASE + w * kCarries + b; }

inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

// ---- symbolic words: per bit, the sorted set of witness columns it XORs --
using Sup = std::vector<uint32_t>;
Sup sx(const Sup& a, const Sup& b) {  // symmetric difference of sorted sets
  Sup out;
  size_t i = 0, j = 0;
  while (i < a.size() && j < b.size()) {
    if (a[i] < b[j]) out.push_back(a[i++]);
    else if (a[i] > b[j]) out.push_back(b[j++]);
    else { i++; j++; }
  }
  out.insert(out.end(), a.begin() + i, a.end());
  out.insert(out.end(), b.begin() + j, b.end());
  return out;
}
using Word = std::vector<Sup>;  // 32 bits
Word wire(int base) { Word w(32); for (int b = 0; b < 32; b++) w[b] = {(uint32_t)(base + b)}; return w; }
Word wire_fn(int (*f)(int, int), int idx) { Word w(32); for (int b = 0; b < 32; b++) w[b] = {(uint32_t)f(idx, b)}; return w; }
Word wxor(const Word& x, const Word& y) { Word w(32); for (int b = 0; b < 32; b++) w[b] = sx(x[b], y[b]); return w; }
Word wrotr(const Word& x, int n) { Word w(32); for (int b = 0; b < 32; b++) w[b] = x[(b + n) % 32]; return w; }
Word wshr(const Word& x, int n) { Word w(32); for (int b = 0; b + n < 32; b++) w[b] = x[b + n]; return w; }
Word rot3(const Word& x, int r1, int r2, int r3) { return wxor(wxor(wrotr(x, r1), wrotr(x, r2)), wrotr(x, r3)); }
Word sig(const Word& x, int r1, int r2, int s) { return wxor(wxor(wrotr(x, r1), wrotr(x, r2)), wshr(x, s)); }

struct Rows {
  std::vector<Sup> a, b;
  Rows() : a(K_SHA), b(K_SHA) {}
  // x + y with 31 carry-aux rows at carry(i): row (x_i ^ cin_i) * (y_i ^ cin_i),
  // cin_{i+1} = cin_i ^ {carry(i)}; returns the symbolic sum
  template <class F>
  Word add_inline(const Word& x, const Word& y, F carry) {
    Word s(32);
    Sup cin;
    for (int i = 0; i < 32; i++) {
      s[i] = sx(sx(x[i], y[i]), cin);
      if (i < kCarries) {
        const int slot = carry(i);
        a[slot] = sx(x[i], cin);
        b[slot] = sx(y[i], cin);
        cin = sx(cin, Sup{(uint32_t)slot});
      }
    }
    return s;
  }
  // rows (support) * z[Z_CONST] = z[slot(b)]; returns the slot word
  template <class F>
  Word materialize(const Word& raw, F slot) {
    Word out(32);
    for (int bit = 0; bit < 32; bit++) {
      const int s = slot(bit);
      a[s] = raw[bit];
      b[s] = {(uint32_t)Z_CONST_POS};
      out[bit] = {(uint32_t)s};
    }
    return out;
  }
};

SparseRows to_csr(const std::vector<Sup>& rows) {
  SparseRows s;
  s.ptr.assign(rows.size() + 1, 0);
  for (size_t r = 0; r < rows.size(); r++) s.ptr[r + 1] = s.ptr[r] + (uint32_t)rows[r].size();
  s.col.resize(s.ptr.back());
  for (size_t r = 0; r < rows.size(); r++)
    for (size_t j = 0; j < rows[r].size(); j++) s.col[s.ptr[r] + j] = (uint16_t)rows[r][j];
  return s;
}

struct Bits {
  uint64_t* w;
  void set(int bit, bool v) { if (v) w[bit >> 6] |= 1ull << (bit & 63); }
  void word(int base, uint32_t v) { for (int i = 0; i < 32; i++) set(base + i, (v >> i) & 1); }
};
// add32_w: carry-aux bits z[cb + i] = (x_i ^ cin) & (y_i ^ cin), cin ^= aux
uint32_t add_w(uint32_t x, uint32_t y, int cb, Bits& z) {
  bool cin = false;
  for (int i = 0; i < kCarries; i++) {
    const bool xi = (x >> i) & 1, yi = (y >> i) & 1;
    const bool aux = (xi != cin) && (yi != cin);
    z.set(cb + i, aux);
    cin = cin != aux;
  }
  return x + y;
}
}  // namespace

void compress(const uint32_t h[8], const uint32_t m[16], uint32_t out[8]) {
  uint32_t w[64];
  for (int t = 0; t < 16; t++) w[t] = m[t];
  for (int t = 16; t < 64; t++) {
    const uint32_t s0 = rotr(w[t - 15], 7) ^ rotr(w[t - 15], 18) ^ (w[t - 15] >> 3);
    const uint32_t s1 = rotr(w[t - 2], 17) ^ rotr(w[t - 2], 19) ^ (w[t - 2] >> 10);
    w[t] = s1 + w[t - 7] + s0 + w[t - 16];
  }
  uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
  for (int r = 0; r < 64; r++) {
    const uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
    const uint32_t ch = (e & f) ^ (~e & g);
    const uint32_t t1 = hh + S1 + ch + RC[r] + w[r];
    const uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
    const uint32_t maj = (a & b) ^ (a & c) ^ (b & c);
    const uint32_t t2 = S0 + maj;
    hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
  }
  const uint32_t st[8] = {a, b, c, d, e, f, g, hh};
  for (int i = 0; i < 8; i++) out[i] = h[i] + st[i];
}

std::vector<Compression> bench_inputs(size_t n, uint64_t seed) {
  std::vector<Compression> v(n);
  uint64_t s = seed;
  auto next = [&]() -> uint32_t {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return (uint32_t)(z ^ (z >> 31));
  };
  for (auto& c : v) {
    for (int i = 0; i < 8; i++) c.h[i] = next();
    for (int i = 0; i < 16; i++) c.m[i] = next();
  }
  return v;
}

Hasher::Hasher() { memcpy(h_, IV, 32); }
void Hasher::update(const void* data, size_t len) {
  const uint8_t* p = static_cast<const uint8_t*>(data);
  total_ += len;
  for (size_t i = 0; i < len; i++) {
    buf_[blen_++] = p[i];
    if (blen_ == 64) {
      uint32_t m[16];
      for (int k = 0; k < 16; k++)
        m[k] = (uint32_t)buf_[4 * k] << 24 | (uint32_t)buf_[4 * k + 1] << 16 | (uint32_t)buf_[4 * k + 2] << 8 |
               (uint32_t)buf_[4 * k + 3];
      uint32_t out[8];
      compress(h_, m, out);
      memcpy(h_, out, 32);
      blen_ = 0;
    }
  }
}
void Hasher::finalize(uint8_t out32[32]) const {
  Hasher s = *this;
  const uint64_t bits = total_ * 8;
  const uint8_t one = 0x80, zero = 0;
  s.update(&one, 1);
  while (s.blen_ != 56) s.update(&zero, 1);
  for (int i = 7; i >= 0; i--) {
    const uint8_t b = (uint8_t)(bits >> (8 * i));
    s.update(&b, 1);
  }
  for (int w = 0; w < 8; w++)
    for (int k = 0; k < 4; k++) out32[4 * w + k] = (uint8_t)(s.h_[w] >> (24 - 8 * k));
}
void hash(const void* data, size_t len, uint8_t out32[32]) {
  Hasher h;
  h.update(data, len);
  h.finalize(out32);
}

int min_n_blocks_log(size_t n) {
  size_t p = 8;
  int l = 3;
  while (p < n) { p <<= 1; l++; }
  return l;
}

void build_matrices(SparseRows& A, SparseRows& B) {
  Rows R;
  R.a[Z_CONST_POS] = {(uint32_t)Z_CONST_POS};
  R.b[Z_CONST_POS] = {(uint32_t)Z_CONST_POS};
  for (int w = 0; w < 8; w++)
    for (int b = 0; b < 32; b++) { R.a[h_bit(w, b)] = {(uint32_t)h_bit(w, b)}; R.b[h_bit(w, b)] = {(uint32_t)Z_CONST_POS}; }
  for (int i = 0; i < 16; i++)
    for (int b = 0; b < 32; b++) { R.a[m_bit(i, b)] = {(uint32_t)m_bit(i, b)}; R.b[m_bit(i, b)] = {(uint32_t)Z_CONST_POS}; }
  std::vector<Word> h_in, W;
  for (int w = 0; w < 8; w++) h_in.push_back(wire(h_bit(w, 0)));
  for (int i = 0; i < 16; i++) W.push_back(wire(m_bit(i, 0)));
  for (int t = 16; t < 64; t++) {
    const Word s1 = sig(W[t - 2], 17, 19, 10), s0 = sig(W[t - 15], 7, 18, 3);
    const Word x0 = R.add_inline(s1, W[t - 7], [&](int i) { return scarry_bit(t, 0, i); });
    const Word x1 = R.add_inline(x0, s0, [&](int i) { return scarry_bit(t, 1, i); });
    const Word raw = R.add_inline(x1, W[t - 16], [&](int i) { return scarry_bit(t, 2, i); });
    W.push_back(R.materialize(raw, [&](int b) { return w_bit(t, b); }));
  }
  std::vector<Word> st = h_in;
  for (int r = 0; r < 64; r++) {
    const Word a = st[0], bb = st[1], c = st[2], d = st[3], e = st[4], f = st[5], g = st[6], h = st[7];
    Word ch(32), maj(32);
    for (int bit = 0; bit < 32; bit++) {
      const int s = ch_bit(r, bit);
      R.a[s] = e[bit];
      R.b[s] = sx(f[bit], g[bit]);
      ch[bit] = {(uint32_t)s};
      const int u = maj_bit(r, bit);
      R.a[u] = sx(a[bit], bb[bit]);
      R.b[u] = sx(a[bit], c[bit]);
      maj[bit] = {(uint32_t)u};
    }
    const Word ch_out = wxor(ch, g), maj_out = wxor(maj, a);
    Word kw(32);
    for (int i = 0; i < 32; i++)
      if ((RC[r] >> i) & 1) kw[i] = {(uint32_t)Z_CONST_POS};
    const Word t1_0 = R.add_inline(h, rot3(e, 6, 11, 25), [&](int i) { return rcarry_bit(r, 0, i); });
    const Word t1_1 = R.add_inline(t1_0, ch_out, [&](int i) { return rcarry_bit(r, 1, i); });
    const Word t1_2 = R.add_inline(t1_1, kw, [&](int i) { return rcarry_bit(r, 2, i); });
    const Word t1 = R.materialize(R.add_inline(t1_2, W[r], [&](int i) { return rcarry_bit(r, 3, i); }),
                                  [&](int b) { return t1_bit(r, b); });
    const Word t2 = R.add_inline(rot3(a, 2, 13, 22), maj_out, [&](int i) { return rcarry_bit(r, 4, i); });
    const Word e_new = R.materialize(R.add_inline(d, t1, [&](int i) { return rcarry_bit(r, 5, i); }),
                                     [&](int b) { return enew_bit(r, b); });
    const Word a_new = R.materialize(R.add_inline(t1, t2, [&](int i) { return rcarry_bit(r, 6, i); }),
                                     [&](int b) { return anew_bit(r, b); });
    st = {a_new, a, bb, c, e_new, e, f, g};
  }
  for (int w = 0; w < 8; w++)
    R.materialize(R.add_inline(st[w], h_in[w], [&](int i) { return ocarry_bit(w, i); }),
                  [&](int b) { return h_out_bit(w, b); });
  A = to_csr(R.a);
  B = to_csr(R.b);
}

void block_witness(const Compression& c, uint64_t* zw) {
  Bits z{zw};
  z.set(Z_CONST_POS, true);
  for (int w = 0; w < 8; w++) z.word(h_bit(w, 0), c.h[w]);
  for (int i = 0; i < 16; i++) z.word(m_bit(i, 0), c.m[i]);
  uint32_t W[64];
  for (int t = 0; t < 16; t++) W[t] = c.m[t];
  for (int t = 16; t < 64; t++) {
    const uint32_t s0 = rotr(W[t - 15], 7) ^ rotr(W[t - 15], 18) ^ (W[t - 15] >> 3);
    const uint32_t s1 = rotr(W[t - 2], 17) ^ rotr(W[t - 2], 19) ^ (W[t - 2] >> 10);
    const uint32_t x0 = add_w(s1, W[t - 7], scarry_bit(t, 0, 0), z);
    const uint32_t x1 = add_w(x0, s0, scarry_bit(t, 1, 0), z);
    W[t] = add_w(x1, W[t - 16], scarry_bit(t, 2, 0), z);
    z.word(w_bit(t, 0), W[t]);
  }
  uint32_t s[8];
  for (int i = 0; i < 8; i++) s[i] = c.h[i];
  for (int r = 0; r < 64; r++) {
    const uint32_t a = s[0], b = s[1], cc = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
    const uint32_t ch = e & (f ^ g), maj = (a ^ b) & (a ^ cc);
    z.word(ch_bit(r, 0), ch);
    z.word(maj_bit(r, 0), maj);
    const uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25), S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
    const uint32_t t1_0 = add_w(h, S1, rcarry_bit(r, 0, 0), z);
    const uint32_t t1_1 = add_w(t1_0, ch ^ g, rcarry_bit(r, 1, 0), z);
    const uint32_t t1_2 = add_w(t1_1, RC[r], rcarry_bit(r, 2, 0), z);
    const uint32_t t1 = add_w(t1_2, W[r], rcarry_bit(r, 3, 0), z);
    z.word(t1_bit(r, 0), t1);
    const uint32_t t2 = add_w(S0, maj ^ a, rcarry_bit(r, 4, 0), z);
    const uint32_t e_new = add_w(d, t1, rcarry_bit(r, 5, 0), z);
    z.word(enew_bit(r, 0), e_new);
    const uint32_t a_new = add_w(t1, t2, rcarry_bit(r, 6, 0), z);
    z.word(anew_bit(r, 0), a_new);
    s[7] = g; s[6] = f; s[5] = e; s[4] = e_new; s[3] = cc; s[2] = b; s[1] = a; s[0] = a_new;
  }
  for (int w = 0; w < 8; w++) z.word(h_out_bit(w, 0), add_w(s[w], c.h[w], ocarry_bit(w, 0), z));
}

}  // namespace sha

const R1cs& sha256_r1cs(int n_log) {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<R1cs>> cache;
  static std::unique_ptr<SparseRows> A, B;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(n_log);
  if (it != cache.end()) return *it->second;
  if (!A) {
    A.reset(new SparseRows());
    B.reset(new SparseRows());
    sha::build_matrices(*A, *B);
  }
  std::unique_ptr<R1cs> r(new R1cs());
  r->n_log = n_log;
  r->k_log = sha::K_LOG_SHA;
  r->z_const = sha::Z_CONST_POS;
  r->m = r->k_log + n_log;
  r->a0 = *A;
  r->b0 = *B;
  r->digest = statement_digest(r->m, r->k_log, K_SKIP, r->a0, r->b0);
  const R1cs& ref = *r;
  cache[n_log] = std::move(r);
  return ref;
}

void generate_sha256_witness(const std::vector<sha::Compression>& blocks, int n_log, std::vector<F128>& z,
                             std::vector<F128>& a, std::vector<F128>& b) {
  const R1cs& rc = sha256_r1cs(n_log);
  const size_t n_total = (size_t)1 << n_log, per = sha::K_SHA / 128;
  z.assign(n_total * per, ZERO);
  // padding blocks: the compression of the all-zero (h_in, m) (sha2.rs:1185-1209)
  const sha::Compression pad{};
  par_for(n_total, [&](size_t o0, size_t o1, int) {
    for (size_t o = o0; o < o1; o++) sha::block_witness(o < blocks.size() ? blocks[o] : pad, (uint64_t*)&z[o * per]);
  });
  apply_block_diag(rc.a0, z, (int)n_total, a);
  apply_block_diag(rc.b0, z, (int)n_total, b);
}

Bundle prove_sha256(const std::vector<sha::Compression>& blocks, int n_log, const std::string& domain) {
  std::vector<F128> z, a, b;
  generate_sha256_witness(blocks, n_log, z, a, b);
  return prove_core(sha256_r1cs(n_log), std::move(z), a, b, domain, CoreHook());
}

}  // namespace flockref
