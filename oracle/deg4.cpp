// Degree-4 zerocheck round 1 of the oracle (test infrastructure; see
// flockref.hpp).  Restates round1_deg4_naive,
// crates/flock-core/src/zerocheck/univariate_skip_deg4.rs:77-165: for every
// 64-bit row x of the five bit vectors, each factor is extended from S =
// {0..63} to V8 = GF(2^8) by the inverse additive NTT on S (k = 6) and the
// forward one on V8 (k = 8, zero coefficients above 64; ntt.rs), and
//   p_abcd[i] = sum_x eq(r[6..], x) phi8(a b c d at lambda = 64 + i)
//   p_z[i]    = sum_x eq(r[6..], x) phi8(z at lambda = 64 + i),  i < 192.
#include "flockref.hpp"

namespace flockref {

void round1_deg4(const uint64_t* a, const uint64_t* b, const uint64_t* c, const uint64_t* d, const uint64_t* z,
                 int m, const std::vector<F128>& r, std::vector<F128>& p_abcd, std::vector<F128>& p_z) {
  const size_t n_rows = (size_t)1 << (m - 6);
  const std::vector<F128> eq = build_eq(std::vector<F128>(r.begin() + 6, r.end()));
  const Gf8Ntt ns(6, 0), nv(8, 0);
  std::vector<std::vector<F128>> pa(par_threads(), std::vector<F128>(192, ZERO)), pz = pa;
  par_for(n_rows, [&](size_t x0, size_t x1, int ti) {
    uint8_t col[5][256];
    for (size_t x = x0; x < x1; x++) {
      const uint64_t w[5] = {a[x], b[x], c[x], d[x], z[x]};
      for (int f = 0; f < 5; f++) {
        memset(col[f], 0, 256);
        for (int s = 0; s < 64; s++) col[f][s] = (uint8_t)((w[f] >> s) & 1);
        ns.inverse(col[f]);
        nv.forward(col[f]);
      }
      for (int i = 0; i < 192; i++) {
        const int lam = 64 + i;
        const uint8_t abcd = gf8_mul(gf8_mul(col[0][lam], col[1][lam]), gf8_mul(col[2][lam], col[3][lam]));
        pa[ti][i] += eq[x] * phi8(abcd);
        pz[ti][i] += eq[x] * phi8(col[4][lam]);
      }
    }
  });
  p_abcd.assign(192, ZERO);
  p_z.assign(192, ZERO);
  for (size_t t = 0; t < pa.size(); t++)
    for (int i = 0; i < 192; i++) {
      p_abcd[i] += pa[t][i];
      p_z[i] += pz[t][i];
    }
}

}  // namespace flockref
