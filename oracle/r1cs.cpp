// BLAKE3-compression R1CS of the oracle (test infrastructure; see
// flockref.hpp).  Restates crates/flock-prover/src/r1cs_hashes/blake3.rs:
// layout constants :198-222, bit accessors :224-262, symbolic Word cascade
// :350-440, build_matrices :456-640, build_block_witness :1763-1852 and the
// row-witness semantics of the fused generator (:1890-1905: constant row
// (1,1,1), input/lin-id rows (v,v,1), carry rows (c, X^cin, Y^cin)).
// Statement digest: crates/flock-core/src/r1cs.rs:334-385 (absorb_matrix).
// xor_dedup: crates/flock-prover/src/r1cs_hashes/common.rs:437-453.
#include "flockref.hpp"
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>

namespace flockref {

namespace {
constexpr int WORD_BITS = 32;
constexpr int CV_BASE = 0;
constexpr int OUT_LO_BASE = 256;
constexpr int M_BASE = 513;
constexpr int T_LO_BASE = 1025;
constexpr int T_HI_BASE = 1057;
constexpr int BLEN_BASE = 1089;
constexpr int FLAGS_BASE = 1121;
constexpr int GS_BASE = 1153;
constexpr int G_STRIDE = 250;
constexpr int N_G = 56;
constexpr int OUT_HI_BASE = GS_BASE + N_G * G_STRIDE;  // 15153
static_assert(OUT_HI_BASE + 256 == USEFUL_BITS, "layout");

const int G_LANES[8][4] = {{0, 4, 8, 12}, {1, 5, 9, 13}, {2, 6, 10, 14}, {3, 7, 11, 15},
                           {0, 5, 10, 15}, {1, 6, 11, 12}, {2, 7, 8, 13}, {3, 4, 9, 14}};
const int MSG_PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};

inline int cv_bit(int w, int b) { return CV_BASE + 32 * w + b; }
inline int m_bit(int i, int b) { return M_BASE + 32 * i + b; }
inline int carry_bit(int g, int add, int b) { return GS_BASE + G_STRIDE * g + 31 * add + b; }
inline int lin_bit(int g, int which, int b) { return GS_BASE + G_STRIDE * g + 6 * 31 + 32 * which + b; }
inline int out_lo_bit(int w, int b) { return OUT_LO_BASE + 32 * w + b; }
inline int out_hi_bit(int w, int b) { return OUT_HI_BASE + 32 * w + b; }

// msg_idx[r][g] = PERM^r applied to (2g, 2g+1)   (blake3.rs:326-346)
void per_round_msg_idx(int out[7][8][2]) {
  int perm[16];
  for (int i = 0; i < 16; i++) perm[i] = i;
  for (int r = 0; r < 7; r++) {
    for (int g = 0; g < 8; g++) {
      out[r][g][0] = perm[2 * g];
      out[r][g][1] = perm[2 * g + 1];
    }
    int next[16];
    for (int i = 0; i < 16; i++) next[i] = perm[MSG_PERM[i]];
    memcpy(perm, next, sizeof(perm));
  }
}

using Lin = std::vector<uint32_t>;
Lin xor_dedup(Lin v) {
  std::sort(v.begin(), v.end());
  Lin out;
  out.reserve(v.size());
  size_t i = 0;
  while (i < v.size()) {
    uint32_t val = v[i];
    size_t c = 0;
    while (i < v.size() && v[i] == val) { c++; i++; }
    if (c & 1) out.push_back(val);
  }
  return out;
}

struct Word {
  std::array<Lin, 32> bits;
  static Word slot(int base) {
    Word w;
    for (int i = 0; i < 32; i++) w.bits[i] = {(uint32_t)(base + i)};
    return w;
  }
  static Word konst(uint32_t v) {
    Word w;
    for (int i = 0; i < 32; i++)
      if ((v >> i) & 1) w.bits[i] = {(uint32_t)Z_CONST_POS};
    return w;
  }
  Word xor_with(const Word& o) const {
    Word w = *this;
    for (int i = 0; i < 32; i++) w.bits[i].insert(w.bits[i].end(), o.bits[i].begin(), o.bits[i].end());
    return w;
  }
  Word dedup() const {
    Word w;
    for (int i = 0; i < 32; i++) w.bits[i] = xor_dedup(bits[i]);
    return w;
  }
  Word rotr(int n) const {
    Word w;
    for (int i = 0; i < 32; i++) w.bits[i] = bits[(i + n) % 32];
    return w;
  }
};

Word add_rows(std::vector<Lin>& a_rows, std::vector<Lin>& b_rows, const Word& x, const Word& y, int cb) {
  for (int i = 0; i < 31; i++) {
    Lin a = x.bits[i], b = y.bits[i];
    for (int j = 0; j < i; j++) { a.push_back(cb + j); b.push_back(cb + j); }
    a_rows[cb + i] = xor_dedup(a);
    b_rows[cb + i] = xor_dedup(b);
  }
  Word s;
  for (int i = 0; i < 32; i++) {
    Lin v = x.bits[i];
    v.insert(v.end(), y.bits[i].begin(), y.bits[i].end());
    for (int j = 0; j < i; j++) v.push_back(cb + j);
    s.bits[i] = xor_dedup(v);
  }
  return s;
}

SparseRows to_csr(const std::vector<Lin>& rows) {
  SparseRows s;
  s.ptr.resize(rows.size() + 1);
  size_t nnz = 0;
  for (size_t r = 0; r < rows.size(); r++) { s.ptr[r] = (uint32_t)nnz; nnz += rows[r].size(); }
  s.ptr[rows.size()] = (uint32_t)nnz;
  s.col.resize(nnz);
  for (size_t r = 0; r < rows.size(); r++)
    for (size_t j = 0; j < rows[r].size(); j++) s.col[s.ptr[r] + j] = (uint16_t)rows[r][j];
  return s;
}
}  // namespace

void build_matrices(SparseRows& A, SparseRows& B) {
  std::vector<Lin> a(K), b(K);
  a[Z_CONST_POS] = {Z_CONST_POS};
  b[Z_CONST_POS] = {Z_CONST_POS};
  auto input_emit = [&](int base, int len) {
    for (int j = 0; j < len; j++) { a[base + j] = {(uint32_t)(base + j)}; b[base + j] = {Z_CONST_POS}; }
  };
  input_emit(CV_BASE, 256);
  input_emit(M_BASE, 512);
  input_emit(T_LO_BASE, 32);
  input_emit(T_HI_BASE, 32);
  input_emit(BLEN_BASE, 32);
  input_emit(FLAGS_BASE, 32);

  int msg_idx[7][8][2];
  per_round_msg_idx(msg_idx);
  std::array<Word, 16> st;
  for (int w = 0; w < 8; w++) st[w] = Word::slot(cv_bit(w, 0));
  for (int i = 0; i < 4; i++) st[8 + i] = Word::konst(b3::IV[i]);
  st[12] = Word::slot(T_LO_BASE);
  st[13] = Word::slot(T_HI_BASE);
  st[14] = Word::slot(BLEN_BASE);
  st[15] = Word::slot(FLAGS_BASE);

  for (int r = 0; r < 7; r++) {
    for (int gi = 0; gi < 8; gi++) {
      int g = r * 8 + gi;
      int la = G_LANES[gi][0], lb = G_LANES[gi][1], lc = G_LANES[gi][2], ld = G_LANES[gi][3];
      Word A0 = st[la], B0 = st[lb], C0 = st[lc], D0 = st[ld];
      Word mx = Word::slot(m_bit(msg_idx[r][gi][0], 0));
      Word my = Word::slot(m_bit(msg_idx[r][gi][1], 0));
      Word tmp0 = add_rows(a, b, A0, B0, carry_bit(g, 0, 0));
      Word a1 = add_rows(a, b, tmp0, mx, carry_bit(g, 1, 0));
      Word d1 = D0.xor_with(a1).dedup().rotr(16);
      Word c1 = add_rows(a, b, C0, d1, carry_bit(g, 2, 0));
      Word b1 = B0.xor_with(c1).dedup().rotr(12);
      Word tmp1 = add_rows(a, b, a1, b1, carry_bit(g, 3, 0));
      Word a2 = add_rows(a, b, tmp1, my, carry_bit(g, 4, 0));
      Word d2 = d1.xor_with(a2).dedup().rotr(8);
      Word c2 = add_rows(a, b, c1, d2, carry_bit(g, 5, 0));
      Word bnew = b1.xor_with(c2).dedup().rotr(7);
      for (int i = 0; i < 32; i++) {
        a[lin_bit(g, 0, i)] = bnew.bits[i];
        b[lin_bit(g, 0, i)] = {Z_CONST_POS};
        a[lin_bit(g, 1, i)] = d2.bits[i];
        b[lin_bit(g, 1, i)] = {Z_CONST_POS};
      }
      st[la] = a2;
      st[lb] = Word::slot(lin_bit(g, 0, 0));
      st[lc] = c2;
      st[ld] = Word::slot(lin_bit(g, 1, 0));
    }
  }
  for (int w = 0; w < 8; w++) {
    Word lo = st[w].xor_with(st[w + 8]).dedup();
    Word hi = st[w + 8].xor_with(Word::slot(cv_bit(w, 0))).dedup();
    for (int i = 0; i < 32; i++) {
      a[out_lo_bit(w, i)] = lo.bits[i];
      b[out_lo_bit(w, i)] = {Z_CONST_POS};
      a[out_hi_bit(w, i)] = hi.bits[i];
      b[out_hi_bit(w, i)] = {Z_CONST_POS};
    }
  }
  A = to_csr(a);
  B = to_csr(b);
}

static void absorb_u64(b3::Hasher& h, uint64_t v) {
  uint8_t b[8];
  for (int i = 0; i < 8; i++) b[i] = (uint8_t)(v >> (8 * i));
  h.update(b, 8);
}

static void absorb_matrix(b3::Hasher& h, const SparseRows& m) {
  const int rows = (int)m.ptr.size() - 1;
  absorb_u64(h, rows);
  absorb_u64(h, rows);
  std::vector<uint8_t> buf;
  for (int r = 0; r < rows; r++) {
    uint32_t s = m.ptr[r], e = m.ptr[r + 1];
    buf.resize(8 * (size_t)(e - s + 1));
    uint64_t v = e - s;
    for (int i = 0; i < 8; i++) buf[i] = (uint8_t)(v >> (8 * i));
    for (uint32_t j = s; j < e; j++) {
      uint64_t c = m.col[j];
      for (int i = 0; i < 8; i++) buf[8 * (1 + j - s) + i] = (uint8_t)(c >> (8 * i));
    }
    h.update(buf.data(), buf.size());
  }
}

// C = I of k rows, absorbed as absorb_matrix would (one entry per row); the
// column index of row r is r, which for 2^17-row blocks does not fit a u16
static void absorb_identity(b3::Hasher& h, int k) {
  absorb_u64(h, (uint64_t)k);
  absorb_u64(h, (uint64_t)k);
  for (int r = 0; r < k; r++) {
    uint8_t buf[16];
    for (int i = 0; i < 8; i++) buf[i] = (uint8_t)(i == 0);
    for (int i = 0; i < 8; i++) buf[8 + i] = (uint8_t)((uint64_t)r >> (8 * i));
    h.update(buf, 16);
  }
}

std::array<uint8_t, 32> statement_digest(int m, int k_log, int k_skip, const SparseRows& a0, const SparseRows& b0) {
  const int k = 1 << k_log;
  b3::Hasher h;
  const char* tag = "flock-r1cs-stmt-v1";
  h.update(tag, strlen(tag));
  absorb_u64(h, (uint64_t)m);
  absorb_u64(h, (uint64_t)k_log);
  absorb_u64(h, (uint64_t)k_skip);
  uint8_t layout = 0;  // RowMajor
  h.update(&layout, 1);
  absorb_matrix(h, a0);
  absorb_matrix(h, b0);
  absorb_identity(h, k);
  std::array<uint8_t, 32> d;
  h.finalize(d.data());
  return d;
}

const R1cs& blake3_r1cs(int n_log) {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<R1cs>> cache;
  static std::unique_ptr<SparseRows> A, B;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(n_log);
  if (it != cache.end()) return *it->second;
  if (!A) {
    A.reset(new SparseRows());
    B.reset(new SparseRows());
    build_matrices(*A, *B);
  }
  std::unique_ptr<R1cs> r(new R1cs());
  r->n_log = n_log;
  r->m = K_LOG + n_log;
  r->a0 = *A;
  r->b0 = *B;
  r->digest = statement_digest(r->m, K_LOG, K_SKIP, r->a0, r->b0);
  const R1cs& ref = *r;
  cache[n_log] = std::move(r);
  return ref;
}

// ---------------------------------------------------------------------------
// Witness generation (z, a = A z, b = B z), packed.
// ---------------------------------------------------------------------------
namespace {
struct BitBuf {
  uint64_t* w;
  void set(int bit, bool v) { if (v) w[bit >> 6] |= 1ull << (bit & 63); }
  void word(int base, uint32_t v, uint32_t nbits = 32) {
    for (uint32_t i = 0; i < nbits; i++) set(base + i, (v >> i) & 1);
  }
};
inline uint32_t rotr32(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

// One ADD: writes carry_aux to z, (X ^ cin) to a, (Y ^ cin) to b; bits 0..30.
uint32_t add_witness(uint32_t x, uint32_t y, BitBuf& z, BitBuf& a, BitBuf& b, int cb) {
  uint32_t sum = x + y;
  uint32_t cin = sum ^ x ^ y;
  uint32_t left = (x ^ cin) & 0x7FFFFFFFu, right = (y ^ cin) & 0x7FFFFFFFu;
  uint32_t carry = left & right;
  z.word(cb, carry, 31);
  a.word(cb, left, 31);
  b.word(cb, right, 31);
  return sum;
}

void block_witness(const Compression& c, uint64_t* zw, uint64_t* aw, uint64_t* bw) {
  BitBuf z{zw}, a{aw}, b{bw};
  auto ident = [&](int base, uint32_t v) {  // input / lin-id row: (v, v, 1)
    z.word(base, v);
    a.word(base, v);
    b.word(base, 0xFFFFFFFFu);
  };
  z.set(Z_CONST_POS, true);
  a.set(Z_CONST_POS, true);
  b.set(Z_CONST_POS, true);
  for (int w = 0; w < 8; w++) ident(cv_bit(w, 0), c.cv[w]);
  for (int i = 0; i < 16; i++) ident(m_bit(i, 0), c.m[i]);
  uint32_t tlo = (uint32_t)c.counter, thi = (uint32_t)(c.counter >> 32);
  ident(T_LO_BASE, tlo);
  ident(T_HI_BASE, thi);
  ident(BLEN_BASE, c.block_len);
  ident(FLAGS_BASE, c.flags);
  uint32_t s[16] = {c.cv[0], c.cv[1], c.cv[2], c.cv[3], c.cv[4], c.cv[5], c.cv[6], c.cv[7],
                    b3::IV[0], b3::IV[1], b3::IV[2], b3::IV[3], tlo, thi, c.block_len, c.flags};
  int msg_idx[7][8][2];
  per_round_msg_idx(msg_idx);
  for (int r = 0; r < 7; r++) {
    for (int gi = 0; gi < 8; gi++) {
      int g = r * 8 + gi;
      int la = G_LANES[gi][0], lb = G_LANES[gi][1], lc = G_LANES[gi][2], ld = G_LANES[gi][3];
      uint32_t mx = c.m[msg_idx[r][gi][0]], my = c.m[msg_idx[r][gi][1]];
      uint32_t A0 = s[la], B0 = s[lb], C0 = s[lc], D0 = s[ld];
      uint32_t t0 = add_witness(A0, B0, z, a, b, carry_bit(g, 0, 0));
      uint32_t a1 = add_witness(t0, mx, z, a, b, carry_bit(g, 1, 0));
      uint32_t d1 = rotr32(D0 ^ a1, 16);
      uint32_t c1 = add_witness(C0, d1, z, a, b, carry_bit(g, 2, 0));
      uint32_t b1 = rotr32(B0 ^ c1, 12);
      uint32_t t1 = add_witness(a1, b1, z, a, b, carry_bit(g, 3, 0));
      uint32_t a2 = add_witness(t1, my, z, a, b, carry_bit(g, 4, 0));
      uint32_t d2 = rotr32(d1 ^ a2, 8);
      uint32_t c2 = add_witness(c1, d2, z, a, b, carry_bit(g, 5, 0));
      uint32_t bnew = rotr32(b1 ^ c2, 7);
      ident(lin_bit(g, 0, 0), bnew);
      ident(lin_bit(g, 1, 0), d2);
      s[la] = a2; s[lb] = bnew; s[lc] = c2; s[ld] = d2;
    }
  }
  for (int w = 0; w < 8; w++) {
    ident(out_lo_bit(w, 0), s[w] ^ s[w + 8]);
    ident(out_hi_bit(w, 0), s[w + 8] ^ c.cv[w]);
  }
}
}  // namespace

void generate_witness(const std::vector<Compression>& blocks, int n_log,
                      std::vector<F128>& z, std::vector<F128>& a, std::vector<F128>& b) {
  size_t n_total = (size_t)1 << n_log;
  size_t per = K / 128;
  z.assign(n_total * per, ZERO);
  a.assign(n_total * per, ZERO);
  b.assign(n_total * per, ZERO);
  // padding slots hold the all-zero compression (blake3.rs:4631-4636)
  Compression pad{};
  par_for(n_total, [&](size_t o0, size_t o1, int) {
    for (size_t o = o0; o < o1; o++) {
      const Compression& c = o < blocks.size() ? blocks[o] : pad;
      block_witness(c, (uint64_t*)&z[o * per], (uint64_t*)&a[o * per], (uint64_t*)&b[o * per]);
    }
  });
}

void apply_block_diag(const SparseRows& m0, const std::vector<F128>& z, int n_blocks,
                      std::vector<F128>& out) {
  const int rows = (int)m0.ptr.size() - 1;
  const size_t per = (size_t)rows / 128;
  out.assign((size_t)n_blocks * per, ZERO);
  par_for((size_t)n_blocks, [&](size_t o0, size_t o1, int) {
  for (size_t o = o0; o < o1; o++) {
    const uint64_t* zw = (const uint64_t*)&z[o * per];
    uint64_t* ow = (uint64_t*)&out[o * per];
    for (int r = 0; r < rows; r++) {
      uint64_t acc = 0;
      for (uint32_t j = m0.ptr[r]; j < m0.ptr[r + 1]; j++) {
        int c = m0.col[j];
        acc ^= (zw[c >> 6] >> (c & 63)) & 1;
      }
      if (acc) ow[r >> 6] |= 1ull << (r & 63);
    }
  }
  });
}

}  // namespace flockref
