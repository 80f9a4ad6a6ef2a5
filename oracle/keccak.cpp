// Keccak-f[1600] R1CS of the oracle (test infrastructure; see flockref.hpp).
// Restates crates/flock-prover/src/r1cs_hashes/keccak.rs:
//  * Keccak-f[1600] over 1600 state bits (FIPS 202 3.2: theta, rho, pi,
//    chi, iota), bit index x + 5y + 25z (:78-82), RHO_OFFSETS and
//    ROUND_CONSTANTS (:39-75), theta_rho_pi_preimage (:89-117);
//  * the monolithic encoder at K_LOG = 16 (:430-560): state_0 in slot 0,
//    state_24 in slot 1 (2048-bit slots, lane-contiguous: bit j of a state at
//    64 (j mod 25) + j / 25), the constant at bit 4096, t_0..t_23 from bit
//    4160; rows: constant (1,1,1), state_0 (v, v, 1), t_r = chi AND
//    (~B[x+1], B[x+2]) with B = pi(rho(theta(state_r))), state_24 pin
//    (v, v, 1); padding blocks hold keccak_f of the zero state (:562-676);
//  * the lincheck walker KeccakLincheckCircuit::fold_alpha_batched (:681-828),
//    the column marginal alpha A^T e + B^T e of the implicit matrices;
//  * the empty-stub statement (common.rs:120-138: A_0 = B_0 empty, C_0 = I);
//  * the keccak3_proof bench inputs (benches/keccak3_proof.rs:66-93, 114-124);
//  * the 3-wide encoder of keccak3.rs at K_LOG = 17 (:1-140, 151-300, 430-490):
//    three independent permutations per block, sub-keccak i with state_0 in
//    slot 2i, state_24 in slot 2i + 1, one shared constant at bit 12288,
//    t[i, r] tight from bit 12352 in the order i * 24 + r; its walker is three
//    copies of the single recurrence into one comb (min_n_blocks_log :144-150:
//    ceil(n / 3) blocks, at least 8).
// Unlike the product, the oracle evaluates the permutation bit by bit on
// 1600-bit states.
#include "flockref.hpp"
#include <map>
#include <memory>
#include <mutex>

namespace flockref {
namespace keccak {

namespace {
const int RHO[5][5] = {{0, 36, 3, 41, 18}, {1, 44, 10, 45, 2}, {62, 6, 43, 15, 61}, {28, 55, 25, 21, 56},
                       {27, 20, 39, 8, 14}};
inline int sidx(int x, int y, int z) { return x + 5 * y + 25 * z; }
using Bits = std::vector<uint8_t>;  // 1600 state bits, 0/1

// the 11 state_in bits whose XOR is B[x, y, z], B = pi(rho(theta(A)))
std::array<int, 11> preimage(int x, int y, int z) {
  const int a = (x + 3 * y) % 5, b = x, r = RHO[a][b] % 64;
  const int c = (z + 64 - r) % 64, cp = (c + 63) % 64;
  std::array<int, 11> out;
  out[0] = sidx(a, b, c);
  for (int yp = 0; yp < 5; yp++) out[1 + yp] = sidx((a + 4) % 5, yp, c);
  for (int yp = 0; yp < 5; yp++) out[6 + yp] = sidx((a + 1) % 5, yp, cp);
  return out;
}
Bits phi(const Bits& s) {  // pi o rho o theta
  Bits o(1600, 0);
  for (int z = 0; z < 64; z++)
    for (int y = 0; y < 5; y++)
      for (int x = 0; x < 5; x++) {
        uint8_t v = 0;
        for (int k : preimage(x, y, z)) v ^= s[k];
        o[sidx(x, y, z)] = v;
      }
  return o;
}
int lane_pos(int j) { return 64 * (j % 25) + j / 25; }  // within_lane_contiguous
}  // namespace

const uint64_t RC[24] = {
    0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808Aull, 0x8000000080008000ull,
    0x000000000000808Bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
    0x000000000000008Aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000Aull,
    0x000000008000808Bull, 0x800000000000008Bull, 0x8000000000008089ull, 0x8000000000008003ull,
    0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800Aull, 0x800000008000000Aull,
    0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};

void permute(uint64_t lanes[25]) {
  Bits s(1600);
  for (int j = 0; j < 1600; j++) s[j] = (lanes[j % 25] >> (j / 25)) & 1;
  for (int r = 0; r < 24; r++) {
    const Bits b = phi(s);
    for (int z = 0; z < 64; z++)
      for (int y = 0; y < 5; y++)
        for (int x = 0; x < 5; x++)
          s[sidx(x, y, z)] = b[sidx(x, y, z)] ^ ((b[sidx((x + 1) % 5, y, z)] ^ 1) & b[sidx((x + 2) % 5, y, z)]);
    for (int z = 0; z < 64; z++) s[sidx(0, 0, z)] ^= (RC[r] >> z) & 1;
  }
  for (int l = 0; l < 25; l++) {
    lanes[l] = 0;
    for (int z = 0; z < 64; z++) lanes[l] |= (uint64_t)s[l + 25 * z] << z;
  }
}

std::vector<State> bench_inputs(size_t n, uint64_t seed) {
  uint64_t st = seed;
  auto nx = [&]() {
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  std::vector<State> out(n);
  for (auto& s : out) {
    uint64_t draws[25];
    for (int w = 0; w < 25; w++) draws[w] = nx();
    // bit i of the state (index x + 5y + 25z) is bit i mod 64 of draw i / 64
    for (int l = 0; l < 25; l++) {
      s.lanes[l] = 0;
      for (int z = 0; z < 64; z++) {
        const int i = l + 25 * z;
        s.lanes[l] |= ((draws[i / 64] >> (i % 64)) & 1) << z;
      }
    }
  }
  return out;
}

const Layout& single_layout() {
  static const Layout L{K_LOG_KECCAK, 1, Z_CONST, T_BASE};
  return L;
}
const Layout& wide_layout() {
  static const Layout L{K_LOG_KECCAK3, 3, Z_CONST3, T_BASE3};
  return L;
}

// sub-keccak i of a block: state_0 at slot 2i, state_24 at slot 2i + 1,
// t_r at t_base + 1600 (24 i + r)
static void sub_witness(const Layout& L, int i, const State& in, uint64_t* z, uint64_t* a, uint64_t* b) {
  const int s0 = 2 * i * 2048, s24 = (2 * i + 1) * 2048, tb = L.t_base + 1600 * 24 * i;
  Bits s(1600);
  for (int j = 0; j < 1600; j++) s[j] = (in.lanes[j % 25] >> (j / 25)) & 1;
  auto put = [](uint64_t* v, int pos, uint8_t bit) { if (bit) v[pos >> 6] |= 1ull << (pos & 63); };
  for (int j = 0; j < 1600; j++) {
    put(z, s0 + lane_pos(j), s[j]);
    put(a, s0 + lane_pos(j), s[j]);
    put(b, s0 + lane_pos(j), 1);
  }
  for (int r = 0; r < 24; r++) {
    const Bits bs = phi(s);
    for (int zz = 0; zz < 64; zz++)
      for (int y = 0; y < 5; y++)
        for (int x = 0; x < 5; x++) {
          const int j = sidx(x, y, zz), pos = tb + 1600 * r + lane_pos(j);
          const uint8_t l = bs[sidx((x + 1) % 5, y, zz)] ^ 1, rr = bs[sidx((x + 2) % 5, y, zz)];
          put(z, pos, l & rr);
          put(a, pos, l);
          put(b, pos, rr);
          s[j] = bs[j] ^ (l & rr);
        }
    for (int zz = 0; zz < 64; zz++) s[sidx(0, 0, zz)] ^= (RC[r] >> zz) & 1;
  }
  for (int j = 0; j < 1600; j++) {
    put(z, s24 + lane_pos(j), s[j]);
    put(a, s24 + lane_pos(j), s[j]);
    put(b, s24 + lane_pos(j), 1);
  }
}

void block_witness(const Layout& L, const State* in, uint64_t* z, uint64_t* a, uint64_t* b) {
  z[L.z_const >> 6] |= 1ull << (L.z_const & 63);
  a[L.z_const >> 6] |= 1ull << (L.z_const & 63);
  b[L.z_const >> 6] |= 1ull << (L.z_const & 63);
  for (int i = 0; i < L.n_sub; i++) sub_witness(L, i, in[i], z, a, b);
}

// sub-keccak i's rows into comb (the shared constant row excluded)
static void sub_comb(const Layout& L, int i, F128 alpha, const std::vector<F128>& e, std::vector<F128>& comb) {
  const int s0 = 2 * i * 2048, s24 = (2 * i + 1) * 2048, tb = L.t_base + 1600 * 24 * i, zc = L.z_const;
  auto t_pos = [tb](int r, int j) { return tb + 1600 * r + lane_pos(j); };
  // state_0 rows: A = [row], B = [const]
  for (int j = 0; j < 1600; j++) {
    comb[s0 + lane_pos(j)] += alpha * e[s0 + lane_pos(j)];
    comb[zc] += e[s0 + lane_pos(j)];
  }
  // state_24 pin rows: A = L_24[j] (through the recurrence below), B = [const]
  std::vector<F128> pin(1600);
  for (int j = 0; j < 1600; j++) {
    pin[j] = e[s24 + lane_pos(j)];
    comb[zc] += pin[j];
  }
  // chi rows of round r: A = 1 + B[x+1], B = B[x+2]; their marginals on state_r
  std::vector<std::vector<F128>> ca(24, std::vector<F128>(1600, ZERO)), cb = ca;
  F128 sum_t = ZERO;
  for (int r = 0; r < 24; r++)
    for (int zz = 0; zz < 64; zz++)
      for (int y = 0; y < 5; y++)
        for (int x = 0; x < 5; x++) {
          const F128 ev = e[t_pos(r, sidx(x, y, zz))];
          sum_t += ev;
          for (int k : preimage((x + 1) % 5, y, zz)) ca[r][k] += ev;
          for (int k : preimage((x + 2) % 5, y, zz)) cb[r][k] += ev;
        }
  comb[zc] += alpha * sum_t;
  // the round constants' share: state_r = phi^r state_0 + ... + RC_r
  Bits rc(1600, 0);
  F128 rca = ZERO, rcb = ZERO;
  for (int r = 0; r < 24; r++) {
    for (int k = 0; k < 1600; k++)
      if (rc[k]) { rca += ca[r][k]; rcb += cb[r][k]; }
    rc = phi(rc);
    for (int zz = 0; zz < 64; zz++) rc[sidx(0, 0, zz)] ^= (RC[r] >> zz) & 1;
  }
  F128 rcp = ZERO;
  for (int k = 0; k < 1600; k++)
    if (rc[k]) rcp += pin[k];
  comb[zc] += alpha * rca + rcb + alpha * rcp;
  // phi^T
  auto phi_t = [](const std::vector<F128>& v) {
    std::vector<F128> o(1600, ZERO);
    for (int zz = 0; zz < 64; zz++)
      for (int y = 0; y < 5; y++)
        for (int x = 0; x < 5; x++)
          for (int k : preimage(x, y, zz)) o[k] += v[sidx(x, y, zz)];
    return o;
  };
  // A side: K_24 = pin -> t_23; K_r = phi^T(K_{r+1}) + chi_A(r) -> t_{r-1}; K_0 -> state_0
  for (int j = 0; j < 1600; j++) comb[t_pos(23, j)] += alpha * pin[j];
  std::vector<F128> k = phi_t(pin);
  for (int j = 0; j < 1600; j++) k[j] += ca[23][j];
  for (int r = 23; r >= 1; r--) {
    for (int j = 0; j < 1600; j++) comb[t_pos(r - 1, j)] += alpha * k[j];
    std::vector<F128> nk = phi_t(k);
    for (int j = 0; j < 1600; j++) nk[j] += ca[r - 1][j];
    k = nk;
  }
  for (int j = 0; j < 1600; j++) comb[s0 + lane_pos(j)] += alpha * k[j];
  // B side: K_23 = chi_B(23)
  k = cb[23];
  for (int r = 23; r >= 1; r--) {
    for (int j = 0; j < 1600; j++) comb[t_pos(r - 1, j)] += k[j];
    std::vector<F128> nk = phi_t(k);
    for (int j = 0; j < 1600; j++) nk[j] += cb[r - 1][j];
    k = nk;
  }
  for (int j = 0; j < 1600; j++) comb[s0 + lane_pos(j)] += k[j];
}

std::vector<F128> lincheck_comb(const Layout& L, F128 alpha, const std::vector<F128>& e) {
  std::vector<F128> comb((size_t)1 << L.k_log, ZERO);
  // the shared constant row: A = B = [const]
  comb[L.z_const] += alpha * e[L.z_const] + e[L.z_const];
  for (int i = 0; i < L.n_sub; i++) sub_comb(L, i, alpha, e, comb);
  return comb;
}

int min_n_blocks_log(const Layout& L, size_t n) {
  size_t blocks = (n + L.n_sub - 1) / L.n_sub, p = 8;
  int l = 3;
  while (p < blocks) { p <<= 1; l++; }
  return l;
}

}  // namespace keccak

const R1cs& keccak_r1cs(const keccak::Layout& L, int n_log) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::unique_ptr<R1cs>> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find({L.n_sub, n_log});
  if (it != cache.end()) return *it->second;
  std::unique_ptr<R1cs> r(new R1cs());
  r->n_log = n_log;
  r->k_log = L.k_log;
  r->z_const = L.z_const;
  r->m = r->k_log + n_log;
  r->a0.ptr.assign(((size_t)1 << L.k_log) + 1, 0);
  r->b0.ptr.assign(((size_t)1 << L.k_log) + 1, 0);
  r->walker = true;
  r->keccak = &L;
  r->digest = statement_digest(r->m, r->k_log, K_SKIP, r->a0, r->b0);
  const R1cs& ref = *r;
  cache[{L.n_sub, n_log}] = std::move(r);
  return ref;
}

void generate_keccak_witness(const keccak::Layout& L, const std::vector<keccak::State>& states, int n_log,
                             std::vector<F128>& z, std::vector<F128>& a, std::vector<F128>& b) {
  const size_t n_total = (size_t)1 << n_log, per = ((size_t)1 << L.k_log) / 128;
  z.assign(n_total * per, ZERO);
  a.assign(n_total * per, ZERO);
  b.assign(n_total * per, ZERO);
  par_for(n_total, [&](size_t o0, size_t o1, int) {
    for (size_t o = o0; o < o1; o++) {
      // the block's permutations; states past the input (and padding blocks)
      // are the zero state
      keccak::State in[3] = {};
      for (int i = 0; i < L.n_sub; i++) {
        const size_t idx = o * L.n_sub + i;
        if (idx < states.size()) in[i] = states[idx];
      }
      keccak::block_witness(L, in, (uint64_t*)&z[o * per], (uint64_t*)&a[o * per], (uint64_t*)&b[o * per]);
    }
  });
}

Bundle prove_keccak(const keccak::Layout& L, const std::vector<keccak::State>& states, int n_log,
                    const std::string& domain) {
  std::vector<F128> z, a, b;
  generate_keccak_witness(L, states, n_log, z, a, b);
  // a hook that adds no claim, so that prove_core records the open identity
  const CoreHook none = [](Challenger&, const std::vector<F128>&) { return std::vector<DirectClaim>(); };
  return prove_core(keccak_r1cs(L, n_log), std::move(z), a, b, domain, none);
}

}  // namespace flockref
