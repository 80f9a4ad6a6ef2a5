// K5: zerocheck multilinear rounds (crates/flock-core/src/zerocheck.rs:
// 1735-1795 verifier order; multilinear.rs:575-657 fold-at-z and
// round_pair_naive, :3194-3330 fused fold + message).
//
// Round k binds rest variable k (the LSB of the current vectors a^, b^) and
// sends G(1) = sum_j e(j) a^(2j+1) b^(2j+1) and
// G(inf) = sum_j e(j) (a^(2j)+a^(2j+1)) (b^(2j)+b^(2j+1)) with
// e(j) = eq(r[7+k..m], j).
//
// Inputs per round kind:
//  * round 0 reads the packed rows: a^(x) = sum_s L_s(z) a_s(x) is a lookup
//    in 8 byte-window tables of the Lagrange weights, and by linearity
//    a^(2j) + a^(2j+1) = Lag(row 2j ^ row 2j+1);
//  * round 1 folds the packed rows at rho while it reads them:
//    a'(i) = a^(2i) + rho (a^(2i) + a^(2i+1)) = Lag(row 2i) + rhoLag(row 2i ^
//    row 2i+1), with rhoLag = rho * Lag built in shared memory by each CTA;
//  * later rounds fold the previous round's vectors at rho through a
//    CTA-resident 8-bit window table of rho (16 lookups per product: the
//    shared-memory pipe takes the folds, the integer pipe the messages).
// The folded vectors are written for the next round.
//
// The eq weights exploit the fixed inner challenges of the zerocheck
// (univariate_skip_optimized.rs:136-233): the low `ns` bits js of j sit on
// phi8 subfield constants (weight phi8(g(js))) and the next `nm` bits jm on
// the medium constants (weight C * x^(jm << msh)); the rest is the random
// suffix, whose eq table etab (indexed by group) stays on the device.  A
// lane owns one js and one group (all bits above js and jm): it sums its
// 2^nm pairs with shifts, multiplies once by etab[group], and keeps the
// result per js.  The products by phi8(g(js)) and by the round's constant
// factor are left to the host: out[2 js] = T1(js), out[2 js + 1] = Tinf(js).
#include "kernels.cuh"

namespace {
struct ZcArgs {
  const f128* a_in;
  const f128* b_in;
  f128* a_out;
  f128* b_out;
  const f128* lag;  // 8 x 256 Lagrange byte table (packed input)
  f128 rho;
  size_t n_pairs;   // pairs of the message round
  int ns, nm, msh;
  const f128* etab;  // eq over the random suffix, indexed by group
  f128* out;
  f128* halve_out;   // next round's table: etab with its lowest variable summed out
  size_t halve_n;    // (0: none)
};

__device__ __forceinline__ f128 lag_lookup(const f128* lag, uint64_t row) {
  f128 s = mk(0, 0);
#pragma unroll
  for (int k = 0; k < 8; k++) s = fx(s, ld(lag + k * 256 + ((row >> (8 * k)) & 0xFF)));
  return s;
}

struct W3 {
  uint64_t w0, w1, w2;
};
__device__ __forceinline__ void acc_shl(W3& acc, f128 v, int sh) {
  if (sh == 0) {
    acc.w0 ^= v.lo;
    acc.w1 ^= v.hi;
  } else {
    acc.w0 ^= v.lo << sh;
    acc.w1 ^= (v.hi << sh) | (v.lo >> (64 - sh));
    acc.w2 ^= v.hi >> (64 - sh);
  }
}
__device__ __forceinline__ void xshfl(f128& v, int m) {
  v.lo ^= shfl_xor64(v.lo, m);
  v.hi ^= shfl_xor64(v.hi, m);
}

// MODE 0: packed message round; 1: packed fold + message; 2: fold + message
template <int MODE>
__global__ void __launch_bounds__(256, 2) k_zc_round(ZcArgs A) {
  extern __shared__ __align__(16) uint8_t smraw[];
  f128* lag = reinterpret_cast<f128*>(smraw);
  MulTab8* rt = reinterpret_cast<MulTab8*>(smraw);
  if (MODE < 2) {
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) {
      f128 v = ldg(A.lag + i);
      st(lag + i, v);
      if (MODE == 1) st(lag + 2048 + i, fmul(A.rho, v));
    }
    __syncthreads();
  } else {
    multab_build(rt, A.rho);
  }
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < A.halve_n; j += (size_t)gridDim.x * blockDim.x)
    st(A.halve_out + j, fx(ldg(A.etab + 2 * j), ldg(A.etab + 2 * j + 1)));
  const int lane = threadIdx.x & 31;
  const int ns = A.ns, nm = A.nm, gb = ns + nm;
  const int js = lane & ((1 << ns) - 1), gw = lane >> ns;
  const size_t gpw = (size_t)32 >> ns;  // groups per warp iteration
  const size_t n_groups = (A.n_pairs + ((size_t)1 << gb) - 1) >> gb;
  const size_t warp0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t n_warps = ((size_t)gridDim.x * blockDim.x) >> 5;
  f128 T1 = mk(0, 0), Ti = mk(0, 0);
  for (size_t it = warp0; it * gpw < n_groups; it += n_warps) {
    const size_t grp = it * gpw + gw;
    if (grp >= n_groups) continue;
    W3 s1 = {0, 0, 0}, si = {0, 0, 0};
    for (int jm = 0; jm < (1 << nm); jm++) {
      const size_t j = (grp << gb) | ((size_t)jm << ns) | (size_t)js;
      if (j >= A.n_pairs) continue;  // short final rounds
      f128 a1, ad, b1, bd;           // x^(2j+1) and the pair sum
      if (MODE == 0) {
        const f128 wa = ldg(A.a_in + j), wb = ldg(A.b_in + j);
        a1 = lag_lookup(lag, wa.hi);
        ad = lag_lookup(lag, wa.lo ^ wa.hi);
        b1 = lag_lookup(lag, wb.hi);
        bd = lag_lookup(lag, wb.lo ^ wb.hi);
      } else {
        f128 a0, b0;
        if (MODE == 1) {
          const f128 w0 = ldg(A.a_in + 2 * j), w1 = ldg(A.a_in + 2 * j + 1);
          const f128 v0 = ldg(A.b_in + 2 * j), v1 = ldg(A.b_in + 2 * j + 1);
          const f128* rl = lag + 2048;
          a0 = fx(lag_lookup(lag, w0.lo), lag_lookup(rl, w0.lo ^ w0.hi));
          a1 = fx(lag_lookup(lag, w1.lo), lag_lookup(rl, w1.lo ^ w1.hi));
          b0 = fx(lag_lookup(lag, v0.lo), lag_lookup(rl, v0.lo ^ v0.hi));
          b1 = fx(lag_lookup(lag, v1.lo), lag_lookup(rl, v1.lo ^ v1.hi));
        } else {
          const ulonglong2* pa = reinterpret_cast<const ulonglong2*>(A.a_in + 4 * j);
          const ulonglong2* pb = reinterpret_cast<const ulonglong2*>(A.b_in + 4 * j);
          f128 av[4], bv[4];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            ulonglong2 x = __ldg(pa + k), y = __ldg(pb + k);
            av[k] = mk(x.x, x.y);
            bv[k] = mk(y.x, y.y);
          }
          a0 = fx(av[0], multab_mul(rt, fx(av[0], av[1])));
          a1 = fx(av[2], multab_mul(rt, fx(av[2], av[3])));
          b0 = fx(bv[0], multab_mul(rt, fx(bv[0], bv[1])));
          b1 = fx(bv[2], multab_mul(rt, fx(bv[2], bv[3])));
        }
        st(A.a_out + 2 * j, a0);
        st(A.a_out + 2 * j + 1, a1);
        st(A.b_out + 2 * j, b0);
        st(A.b_out + 2 * j + 1, b1);
        ad = fx(a0, a1);
        bd = fx(b0, b1);
      }
      const int sh = jm << A.msh;
      acc_shl(s1, fmul(a1, b1), sh);
      acc_shl(si, fmul(ad, bd), sh);
    }
    const f128 e = ldg(A.etab + grp);
    T1 = fx(T1, fmul(reduce256(s1.w0, s1.w1, s1.w2, 0), e));
    Ti = fx(Ti, fmul(reduce256(si.w0, si.w1, si.w2, 0), e));
  }
  // XOR over the lanes of each js, then over the CTA's warps
  for (int m = 16; m >= (1 << ns); m >>= 1) {
    xshfl(T1, m);
    xshfl(Ti, m);
  }
  __shared__ f128 red[8][8];
  const int w = threadIdx.x >> 5;
  if (lane < (1 << ns)) {
    red[w][2 * lane] = T1;
    red[w][2 * lane + 1] = Ti;
  }
  __syncthreads();
  if ((int)threadIdx.x < (2 << ns)) {
    f128 x = mk(0, 0);
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) x = fx(x, red[k][threadIdx.x]);
    atomic_xor128(A.out + threadIdx.x, x);
  }
}
}  // namespace

// One zerocheck round launch: out[2 js + {0, 1}] ^= (T1, Tinf)(js) for js < 2^ns.
// mode 0: packed message round, 1: packed fold + message, 2: fold + message.
// halve_n > 0: also writes halve_out[j] = etab[2j] + etab[2j+1], j < halve_n,
// the next round's eq table (one launch less per round).  sms: the SMs the
// launch may fill (one wave of resident CTAs on them).
void zc_round(int mode, const f128* a_in, const f128* b_in, f128* a_out, f128* b_out, const f128* lag, f128 rho,
              size_t n_pairs, int ns, int nm, int msh, const f128* etab, f128* out, int sms, cudaStream_t s,
              f128* halve_out, size_t halve_n) {
  if (ns < 0 || ns > 2 || nm < 0 || nm > 4 || msh < 0 || (nm > 0 && (((1 << nm) - 1) << msh) >= 64))
    throw CudaError("zc_round: bad eq structure");
  ZcArgs A;
  A.a_in = a_in; A.b_in = b_in; A.a_out = a_out; A.b_out = b_out; A.lag = lag; A.rho = rho;
  A.n_pairs = n_pairs; A.ns = ns; A.nm = nm; A.msh = msh;
  A.etab = etab; A.out = out;
  A.halve_out = halve_out; A.halve_n = halve_n;
  const size_t smem = mode == 0 ? 2048 * sizeof(f128) : mode == 1 ? 4096 * sizeof(f128) : sizeof(MulTab8);
  const size_t lanes = (n_pairs + ((size_t)1 << nm) - 1) >> nm;
  const void* fn = mode == 0 ? (const void*)k_zc_round<0> : mode == 1 ? (const void*)k_zc_round<1>
                                                                      : (const void*)k_zc_round<2>;
  CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const size_t full = (size_t)resident_grid(fn, 256, smem, sms);
  const int g = (int)std::max<size_t>(1, std::min<size_t>(full, (lanes + 255) / 256));
  count_launch();
  if (mode == 0) k_zc_round<0><<<g, 256, smem, s>>>(A);
  else if (mode == 1) k_zc_round<1><<<g, 256, smem, s>>>(A);
  else k_zc_round<2><<<g, 256, smem, s>>>(A);
}
