// K1: additive NTT over GF(2^128) (LCH novel basis, neighbours-last) on the
// interleaved layout data[pos * lanes + lane], and its transpose.
//
// Semantics: crates/flock-core/src/ntt/additive_ntt_f128.rs — layer l pairs
// positions 2^(log_d - l - 1) apart inside 2^l blocks; butterfly
// u += v * t, v += u with t = twiddle(l, block) = sum over set bits j of the
// block index of W^_{d-l-1}(beta_{d-l+j}) (:2684-2693, :4766-4800).  RS
// encoding at rate 2^-r = replicate the message into 2^r sub-blocks, then
// layers r..d-1 (:2741-2760; commit.rs:1838-1877).  The transposed map (used
// to induce the Ligerito query basis; pcs/ligerito.rs:1579-1600,1987-2056)
// runs layers in reverse with s = u + v, u = s, v = t*s + v.
//
// GPU mapping: each pass covers R <= 10 consecutive layers.  A CTA owns one
// tile = 2^R positions (one per combination of the pass's pair bits, the
// other position bits fixed) x LG consecutive lanes, staged in shared
// memory (LG lanes of one position are contiguous: 16*LG-byte coalesced
// rows); LG is chosen so that two CTAs fit an SM.  The tile's 2^R - 1
// twiddles are derived once into shared memory from the per-layer basis
// values (XOR of at most d values each); block 0 of every layer has the zero
// twiddle and needs no product.
#include "kernels.cuh"
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include "host.hpp"

namespace {
constexpr int kMaxR = 10;  // layers per pass in the default split (the tuner also tries 11)

struct PassArgs {
  f128* data;
  const f128* ev;  // ev[l * 32 + j] = W^_{d-l-1}(beta_{d-l+j}), j < l
  int log_d, lanes, lg_shift, l0, R;
  // The first pass of an RS encode reads its tiles from the message instead
  // of from a replicated codeword: position p of the data holds message
  // position p & src_mask (the rate-2^-r replicate, layer 0..r-1 copies).
  const f128* src = nullptr;
  uint64_t src_mask = 0;
};
__device__ __forceinline__ const f128* tile_src(const PassArgs& p, uint64_t pos) {
  return p.src ? p.src + (pos & p.src_mask) * p.lanes : p.data + pos * p.lanes;
}

__device__ __forceinline__ f128 twiddle(const f128* ev, int l, uint64_t b) {
  f128 t = mk(0, 0);
  for (int j = 0; j < l; j++)
    if ((b >> j) & 1) t = fx(t, ldg(ev + l * 32 + j));
  return t;
}

// One tile of a pass (tile index t_id), staged through the CTA's shared memory.
template <bool TRANSPOSE>
__device__ __forceinline__ void ntt_tile(const PassArgs& p, uint64_t t_id, f128* smem) {
  const int R = p.R, LG = 1 << p.lg_shift;
  f128* tile = smem;                       // [2^R][LG]
  f128* tw = smem + ((size_t)LG << R);     // [2^R - 1] : stage s block k at (1<<s)-1+k
  const int log_d = p.log_d, l0 = p.l0;
  const int lo_bits = log_d - l0 - R;      // position bits below the pair bits
  const int groups = p.lanes >> p.lg_shift;
  const int grp = (int)(t_id % groups);
  t_id /= groups;
  const uint64_t lo = t_id & ((1ull << lo_bits) - 1);
  const uint64_t hi = t_id >> lo_bits;     // l0 bits
  const int n_el = LG << R;
  // load
  uint64_t any = 0;
  for (int e = threadIdx.x; e < n_el; e += blockDim.x) {
    uint64_t pl = (uint64_t)(e >> p.lg_shift);
    uint64_t pos = (hi << (log_d - l0)) | (pl << lo_bits) | lo;
    tile[e] = ld(tile_src(p, pos) + ((size_t)grp << p.lg_shift) + (e & (LG - 1)));
    if (TRANSPOSE) any |= tile[e].lo | tile[e].hi;
  }
  // The transposed transform (the query-basis induction) starts from a vector
  // that is zero outside the queried positions, and a pass maps a zero tile
  // to zeros in place: such tiles are left as they are.
  if (TRANSPOSE && !__syncthreads_or(any != 0)) return;
  for (int k = threadIdx.x; k < (1 << R) - 1; k += blockDim.x) {
    int s = 31 - __clz(k + 1);               // stage
    uint64_t blk = (uint64_t)(k + 1 - (1 << s));
    tw[k] = twiddle(p.ev, l0 + s, (hi << s) | blk);
  }
  __syncthreads();
  // A thread owns one position pair and `per` of its LG lanes (all of them
  // once the tile has as many position pairs as threads): the twiddle's
  // operand split is built once and reused for every lane.  Lanes are
  // visited in an order rotated by the thread index so that the 8 threads
  // of a quarter warp read 8 different 16-byte bank groups.
  const int n_pp = 1 << (R - 1);
  const int per = min(LG, max(1, (n_pp * LG) / (int)blockDim.x));
  const int tpp = LG / per;  // threads per position pair
  const int rs = 3 - p.lg_shift;  // rotate by pq >> rs: distinct bank groups per quarter warp
  for (int stg = 0; stg < R; stg++) {
    const int s = TRANSPOSE ? R - 1 - stg : stg;
    const int hb = R - 1 - s;                // local pair bit
    for (int w = threadIdx.x; w < n_pp * tpp; w += blockDim.x) {
      const int pq = w / tpp, lane0 = (w % tpp) * per;
      const int top = ((pq >> hb) << (hb + 1)) | (pq & ((1 << hb) - 1));
      const int bot = top | (1 << hb);
      const f128 tv = tw[(1 << s) - 1 + (top >> (hb + 1))];
      if (fz(tv)) {  // block 0 of every layer: the twiddle is the empty sum
        for (int k = 0; k < per; k++) {
          const int lane = lane0 + ((k + (pq >> rs)) & (per - 1));
          const int it = (top << p.lg_shift) | lane, ib = (bot << p.lg_shift) | lane;
          if (!TRANSPOSE) tile[ib] = fx(tile[ib], tile[it]);
          else tile[it] = fx(tile[it], tile[ib]);
        }
        continue;
      }
      const MulConst M = mulconst(tv);
      // lane order rotated by the position pair: lane0 + rot covers all 8
      // bank groups over 8 consecutive threads for every `per`
      auto bfly = [&](int lane) {
        f128 u = tile[(top << p.lg_shift) | lane], v = tile[(bot << p.lg_shift) | lane];
        if (!TRANSPOSE) {
          u = fx(u, fmul_c(v, M));
          v = fx(v, u);
        } else {
          u = fx(u, v);
          v = fx(v, fmul_c(u, M));
        }
        tile[(top << p.lg_shift) | lane] = u;
        tile[(bot << p.lg_shift) | lane] = v;
      };
      if (per == 1) {
        bfly(lane0);
      } else {
        for (int k = 0; k < per; k += 2) {  // two independent butterflies per step
          const int l0 = lane0 + ((k + (pq >> rs)) & (per - 1)), l1 = lane0 + ((k + 1 + (pq >> rs)) & (per - 1));
          f128 u0 = tile[(top << p.lg_shift) | l0], v0 = tile[(bot << p.lg_shift) | l0];
          f128 u1 = tile[(top << p.lg_shift) | l1], v1 = tile[(bot << p.lg_shift) | l1];
          if (!TRANSPOSE) {
            u0 = fx(u0, fmul_c(v0, M));
            u1 = fx(u1, fmul_c(v1, M));
            v0 = fx(v0, u0);
            v1 = fx(v1, u1);
          } else {
            u0 = fx(u0, v0);
            u1 = fx(u1, v1);
            v0 = fx(v0, fmul_c(u0, M));
            v1 = fx(v1, fmul_c(u1, M));
          }
          tile[(top << p.lg_shift) | l0] = u0;
          tile[(bot << p.lg_shift) | l0] = v0;
          tile[(top << p.lg_shift) | l1] = u1;
          tile[(bot << p.lg_shift) | l1] = v1;
        }
      }
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < n_el; e += blockDim.x) {
    uint64_t pl = (uint64_t)(e >> p.lg_shift);
    uint64_t pos = (hi << (log_d - l0)) | (pl << lo_bits) | lo;
    st(p.data + pos * p.lanes + ((size_t)grp << p.lg_shift) + (e & (LG - 1)), tile[e]);
  }
}

// ---- warp-per-pair passes: warp-uniform twiddles, table products ----
// A tile holds 2^R positions x 64 lanes.  A warp owns one position pair at a
// time (thread t takes lanes t and t + 32), so the pair's twiddle is uniform
// across the warp in every stage, and the warp multiplies by it through a
// 4-bit window table of the twiddle: entry n of window w is
// t * n(x) * x^(4w), and a product is the XOR of 32 lookups, one per nibble
// of the other factor.  The halves of an entry sit in separate 8-byte arrays
// and window w's entries are permuted by n -> n ^ (w mod 16), so the warp's
// lookups into one window, and the builder's stores, hit 16 distinct bank
// pairs.  A warp's consecutive pairs share the twiddle in all but the last
// stages, and the table is rebuilt only when the twiddle changes.  The
// table lookups load the shared-memory pipe instead of the integer
// multipliers; KIND 2 sends lane t + 32 through the integer product, so both
// pipes work.
size_t pass_w_smem(int R, int threads) {
  return ((size_t)64 << R) * sizeof(f128) + ((size_t)1 << R) * sizeof(f128) + (size_t)(threads / 32) * kTab4Bytes;
}

template <bool TRANSPOSE, int KIND>
__device__ __forceinline__ void ntt_tile_w(const PassArgs& p, uint64_t t_id, f128* smem) {
  const int R = p.R;
  f128* tile = smem;                         // [2^R][64]
  f128* tw = smem + ((size_t)64 << R);       // [2^R - 1], padded to 2^R
  Tab4* tabs = reinterpret_cast<Tab4*>(tw + (1 << R));
  const int log_d = p.log_d, l0 = p.l0;
  const int lo_bits = log_d - l0 - R;
  const int groups = p.lanes >> 6;
  const int grp = (int)(t_id % groups);
  t_id /= groups;
  const uint64_t lo = t_id & ((1ull << lo_bits) - 1);
  const uint64_t hi = t_id >> lo_bits;
  const int n_el = 64 << R;
  uint64_t any = 0;
  for (int e = threadIdx.x; e < n_el; e += blockDim.x) {
    const uint64_t pl = (uint64_t)(e >> 6);
    const uint64_t pos = (hi << (log_d - l0)) | (pl << lo_bits) | lo;
    tile[e] = ld(tile_src(p, pos) + ((size_t)grp << 6) + (e & 63));
    if (TRANSPOSE) any |= tile[e].lo | tile[e].hi;
  }
  if (TRANSPOSE && !__syncthreads_or(any != 0)) return;
  for (int k = threadIdx.x; k < (1 << R) - 1; k += blockDim.x) {
    const int s = 31 - __clz(k + 1);
    const uint64_t blk = (uint64_t)(k + 1 - (1 << s));
    tw[k] = twiddle(p.ev, l0 + s, (hi << s) | blk);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  Tab4* T = tabs + warp;
  const int chunk = (1 << (R - 1)) / nw;  // position pairs per warp per stage (the host keeps nw <= 2^(R-1))
  for (int stg = 0; stg < R; stg++) {
    const int s = TRANSPOSE ? R - 1 - stg : stg;
    const int hb = R - 1 - s;
    int cur = -1;
    MulConst M;  // KIND 2: the class split of the current twiddle
    for (int pq = warp * chunk; pq < (warp + 1) * chunk; pq++) {
      const int top = ((pq >> hb) << (hb + 1)) | (pq & ((1 << hb) - 1));
      const int bot = top | (1 << hb);
      const int k = (1 << s) - 1 + (top >> (hb + 1));
      const f128 tv = tw[k];
      f128* ut = tile + ((size_t)top << 6);
      f128* vt = tile + ((size_t)bot << 6);
      if (fz(tv)) {  // block 0 of every layer: the twiddle is the empty sum
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int l = lane + 32 * q;
          if (!TRANSPOSE) vt[l] = fx(vt[l], ut[l]);
          else ut[l] = fx(ut[l], vt[l]);
        }
        continue;
      }
      if (k != cur) {
        __syncwarp();  // every lane has finished with the previous table
        tab4_build(T, tv, lane);
        if (KIND == 2) M = mulconst(tv);
        __syncwarp();
        cur = k;
      }
      f128 u0 = ut[lane], v0 = vt[lane], u1 = ut[lane + 32], v1 = vt[lane + 32];
      if (!TRANSPOSE) {
        u0 = fx(u0, tab4_mul(T, v0));
        if (KIND == 1) u1 = fx(u1, tab4_mul(T, v1));
        else u1 = fx(u1, fmul_c(v1, M));
        v0 = fx(v0, u0);
        v1 = fx(v1, u1);
      } else {
        u0 = fx(u0, v0);
        u1 = fx(u1, v1);
        v0 = fx(v0, tab4_mul(T, u0));
        if (KIND == 1) v1 = fx(v1, tab4_mul(T, u1));
        else v1 = fx(v1, fmul_c(u1, M));
      }
      ut[lane] = u0;
      vt[lane] = v0;
      ut[lane + 32] = u1;
      vt[lane + 32] = v1;
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < n_el; e += blockDim.x) {
    const uint64_t pl = (uint64_t)(e >> 6);
    const uint64_t pos = (hi << (log_d - l0)) | (pl << lo_bits) | lo;
    st(p.data + pos * p.lanes + ((size_t)grp << 6) + (e & 63), tile[e]);
  }
}

template <bool TRANSPOSE, int KIND>
__global__ void __launch_bounds__(256, 1) k_ntt_pass_w(PassArgs p) {
  extern __shared__ f128 smem[];
  ntt_tile_w<TRANSPOSE, KIND>(p, blockIdx.x, smem);
}

template <bool TRANSPOSE>
__global__ void __launch_bounds__(256, 2) k_ntt_pass(PassArgs p) {
  extern __shared__ f128 smem[];
  ntt_tile<TRANSPOSE>(p, blockIdx.x, smem);
}

// Pass `pass` of every job of a batch: a persistent grid strides over the
// tiles of all jobs (each job's tiles numbered from its tile0[pass]).
__global__ void __launch_bounds__(256, 2) k_ntt_pass_batch(const BatchJob* __restrict__ jobs, int n_jobs, int pass,
                                                           uint64_t total_tiles) {
  extern __shared__ f128 smem[];
  for (uint64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].tile0[pass] <= t) lo = mid;
      else hi = mid - 1;
    }
    const BatchJob& J = jobs[lo];
    const NttPass& ps = J.pass[pass];
    PassArgs a{J.cw, J.ev, J.log_d, 64, ps.lgs, ps.l0, ps.R};
    if (pass == 0) {  // rate 1/2: the message fills both halves of the codeword
      a.src = J.z;
      a.src_mask = ((uint64_t)1 << (J.log_d - 1)) - 1;
    }
    __syncthreads();  // the previous tile's stores have read the shared tile
    if (ps.kind == 1) ntt_tile_w<false, 1>(a, t - J.tile0[pass], smem);
    else if (ps.kind == 2) ntt_tile_w<false, 2>(a, t - J.tile0[pass], smem);
    else ntt_tile<false>(a, t - J.tile0[pass], smem);
  }
}

__global__ void k_replicate_batch(const BatchJob* __restrict__ jobs, int n_jobs, uint64_t total) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  int lo = 0, hi = n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].rep0 <= i) lo = mid;
    else hi = mid - 1;
  }
  const BatchJob& J = jobs[lo];
  const uint64_t k = i - J.rep0;  // rate 1/2: the message and one copy
  const f128 v = ld(J.z + k);
  st(J.cw + k, v);
  st(J.cw + J.msg_len + k, v);
}

__global__ void k_replicate(const f128* __restrict__ msg, f128* __restrict__ cw, size_t msg_len, int copies) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= msg_len) return;
  f128 v = ld(msg + i);
  for (int c = 0; c < copies; c++) st(cw + (size_t)c * msg_len + i, v);
}

// SplitMix64 words: the tuner's scratch holds random values, so that the table
// passes' lookups meet the nibble patterns of real data (all-zero data would
// turn every lookup into a broadcast and time those passes too fast)
__global__ void k_fill_random(uint64_t* p, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t z = (i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  p[i] = z ^ (z >> 31);
}

__global__ void k_fold_copies(const f128* __restrict__ in, f128* __restrict__ out, size_t len, int copies) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  f128 acc = ld(in + i);
  for (int c = 1; c < copies; c++) acc = fx(acc, ld(in + (size_t)c * len + i));
  st(out + i, acc);
}

// Host-computed per-dimension basis table (additive_ntt_f128.rs:54-87).
const f128* device_evals(int dim) {
  static std::mutex mu;
  static std::map<int, f128*> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(dim);
  if (it != cache.end()) return it->second;
  std::vector<std::vector<f128>> evals;
  std::vector<f128> basis(dim);
  for (int i = 0; i < dim; i++) basis[i] = mk(i < 64 ? 1ull << i : 0, i < 64 ? 0 : 1ull << (i - 64));
  evals.push_back(basis);
  for (int i = 1; i < dim; i++) {
    std::vector<f128> row;
    const auto& prev = evals[i - 1];
    for (size_t k = 1; k < prev.size(); k++) row.push_back(flock::hmul(prev[k], fx(prev[k], prev[0])));
    evals.push_back(row);
  }
  for (auto& row : evals) {
    f128 inv = flock::hinv(row[0]);
    for (auto& v : row) v = flock::hmul(v, inv);
  }
  std::vector<f128> tab((size_t)32 * 32, mk(0, 0));
  for (int l = 0; l < dim; l++)
    for (int j = 0; j < l; j++) tab[l * 32 + j] = evals[dim - l - 1][1 + j];
  f128* d = nullptr;
  CK(cudaMalloc(&d, tab.size() * sizeof(f128)));
  CK(cudaMemcpy(d, tab.data(), tab.size() * sizeof(f128), cudaMemcpyHostToDevice));
  cache[dim] = d;
  return d;
}

// ---------------------------------------------------------------- plans --
// A plan is the list of passes (first layer, layer count R, lanes per tile
// 2^lgs, threads per CTA) that covers layers layer_begin..log_d-1.  The
// autotuner times candidate splits of the layers and, for each pass, the
// tile widths and CTA sizes that fit one or two CTAs per SM, and keeps the
// fastest combination per (device, log_d, lanes, layer_begin).

size_t pass_smem(int lgs, int R) { return ((size_t)(1 << lgs) << R) * sizeof(f128) + ((1 << R) - 1) * sizeof(f128); }
constexpr size_t kSmem2 = (size_t)112 << 10;  // two CTAs per SM
constexpr size_t kSmem1 = (size_t)200 << 10;  // one CTA per SM

int max_lgs(int lanes) {
  int g = 0;
  while ((1 << (g + 1)) <= lanes && g < 3) g++;
  return g;
}

std::vector<std::pair<int, int>> balanced_split(int begin, int n_layers, int n_pass) {
  std::vector<std::pair<int, int>> v;
  int l = begin;
  for (int i = 0; i < n_pass; i++) {
    int R = (n_layers - (l - begin) + (n_pass - i) - 1) / (n_pass - i);
    v.push_back({l, R});
    l += R;
  }
  return v;
}

// layer splits to try: the balanced split into the fewest passes of <= 10
// layers, its mirror, a split with one 11-layer pass, and one more pass
std::vector<std::vector<std::pair<int, int>>> candidate_splits(int begin, int n_layers) {
  std::vector<std::vector<std::pair<int, int>>> out;
  auto add = [&](std::vector<std::pair<int, int>> v) {
    for (auto& x : out)
      if (x == v) return;
    for (auto& pr : v)
      if (pr.second < 1 || pr.second > kMaxR + 1) return;
    out.push_back(v);
  };
  const int p0 = (n_layers + kMaxR - 1) / kMaxR;
  auto bal = balanced_split(begin, n_layers, p0);
  add(bal);
  if (p0 >= 2) {  // mirror: the larger passes last
    std::vector<int> Rs;
    for (auto& pr : bal) Rs.push_back(pr.second);
    std::reverse(Rs.begin(), Rs.end());
    std::vector<std::pair<int, int>> v;
    int l = begin;
    for (int R : Rs) { v.push_back({l, R}); l += R; }
    add(v);
  }
  if (n_layers == kMaxR + 1) add({{begin, n_layers}});
  if (p0 == 2 && n_layers > 11) {
    add({{begin, 11}, {begin + 11, n_layers - 11}});
    add({{begin, n_layers - 11}, {begin + n_layers - 11, 11}});
  }
  if (n_layers >= p0 + 1) add(balanced_split(begin, n_layers, p0 + 1));
  return out;
}

// splits for the warp-per-pair passes (at most kMaxRw layers: a 64-lane tile
// and the warps' tables share the CTA's shared memory)
constexpr int kMaxRw = 7;
std::vector<std::vector<std::pair<int, int>>> candidate_splits_w(int begin, int n_layers) {
  std::vector<std::vector<std::pair<int, int>>> out;
  const int p0 = (n_layers + kMaxRw - 1) / kMaxRw;
  for (int np = p0; np <= p0 + 1 && np <= n_layers; np++) {
    auto v = balanced_split(begin, n_layers, np);
    bool ok = true;
    for (auto& pr : v) ok = ok && pr.second >= 4 && pr.second <= kMaxRw;
    if (ok) out.push_back(v);
  }
  return out;
}

// per-pass launch shapes to try: (lgs, threads) of the thread-per-pair passes
std::vector<std::pair<int, int>> candidate_shapes(int lanes, int R) {
  std::vector<std::pair<int, int>> out;
  const int top = max_lgs(lanes);
  int g2 = top;
  while (g2 > 0 && pass_smem(g2, R) > kSmem2) g2--;
  int g1 = top;
  while (g1 > 0 && pass_smem(g1, R) > kSmem1) g1--;
  std::vector<int> gs = {g2};
  if (g2 > 0) gs.push_back(g2 - 1);
  if (g1 > g2) gs.push_back(g1);
  for (int g : gs) {
    if (pass_smem(g, R) > kSmem1) continue;
    const int work = ((1 << g) << R) / 2;  // butterflies per stage
    for (int t : {128, 256}) {
      if (t > std::max(32, work)) continue;
      out.push_back({g, t});
    }
    if (out.empty() || out.back().first != g) out.push_back({g, std::min(256, std::max(32, work))});
  }
  return out;
}

// the warp-per-pair shapes of a pass of R layers: (threads, kind) with the
// tile and every warp's table within one CTA's shared memory
std::vector<NttPass> candidate_shapes_w(int lanes, int l0, int R) {
  std::vector<NttPass> out;
  if (lanes % 64 || R < 4 || R > kMaxRw) return out;
  for (int kind : {1, 2})
    for (int t : {64, 128, 256}) {
      if (t / 32 > (1 << (R - 1)) || pass_w_smem(R, t) > kSmem1) continue;
      NttPass p{l0, R, 6, t};
      p.kind = kind;
      out.push_back(p);
    }
  return out;
}

template <bool TR>
void launch_pass_w(const NttPass& ps, const PassArgs& a, uint64_t tiles, cudaStream_t s) {
  auto k = ps.kind == 1 ? k_ntt_pass_w<TR, 1> : k_ntt_pass_w<TR, 2>;
  CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem1));
  count_launch();
  k<<<(unsigned)tiles, ps.threads, pass_w_smem(ps.R, ps.threads), s>>>(a);
}

void launch_pass(const NttPass& ps, f128* data, const f128* ev, int log_d, int lanes, bool transpose,
                 cudaStream_t s, const f128* src = nullptr) {
  PassArgs a{data, ev, log_d, lanes, ps.lgs, ps.l0, ps.R};
  if (src) {
    a.src = src;
    a.src_mask = ((uint64_t)1 << (log_d - ps.l0)) - 1;
  }
  const size_t smem = pass_smem(ps.lgs, ps.R);
  const uint64_t tiles = ((uint64_t)1 << (log_d - ps.R)) * (uint64_t)(lanes >> ps.lgs);
  if (ps.kind) {
    if (transpose) launch_pass_w<true>(ps, a, tiles, s);
    else launch_pass_w<false>(ps, a, tiles, s);
    return;
  }
  // The attribute is the same upper bound for every launch: it is global to
  // the kernel, so a per-launch size set by one host thread could undercut
  // another thread's launch of a larger tile.
  if (transpose) {
    CK(cudaFuncSetAttribute(k_ntt_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem1));
    count_launch(); k_ntt_pass<true><<<(unsigned)tiles, ps.threads, smem, s>>>(a);
  } else {
    CK(cudaFuncSetAttribute(k_ntt_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem1));
    count_launch(); k_ntt_pass<false><<<(unsigned)tiles, ps.threads, smem, s>>>(a);
  }
}

NttPlan default_plan(int log_d, int lanes, int layer_begin) {
  NttPlan plan;
  const int n_layers = log_d - layer_begin;
  if (n_layers <= 0) return plan;
  for (auto& pr : balanced_split(layer_begin, n_layers, (n_layers + kMaxR - 1) / kMaxR)) {
    int g = max_lgs(lanes);
    while (g > 0 && pass_smem(g, pr.second) > kSmem2) g--;
    plan.push_back({pr.first, pr.second, g, std::min(256, std::max(32, ((1 << g) << pr.second) / 2))});
  }
  return plan;
}

// every plan the tuner may pick: each candidate split with each launch shape
// applied to all of its passes (for parity tests of the tiling)
std::vector<NttPlan> all_plans(int log_d, int lanes, int layer_begin) {
  std::vector<NttPlan> out;
  const int n_layers = log_d - layer_begin;
  if (n_layers <= 0) return {NttPlan{}};
  for (auto& split : candidate_splits(layer_begin, n_layers)) {
    size_t n_shapes = 0;
    for (auto& pr : split) n_shapes = std::max(n_shapes, candidate_shapes(lanes, pr.second).size());
    for (size_t k = 0; k < n_shapes; k++) {
      NttPlan plan;
      for (auto& pr : split) {
        auto sh = candidate_shapes(lanes, pr.second);
        auto& c = sh[std::min(k, sh.size() - 1)];
        plan.push_back({pr.first, pr.second, c.first, c.second});
      }
      out.push_back(plan);
    }
  }
  for (auto& split : candidate_splits_w(layer_begin, n_layers)) {
    size_t n_shapes = 0;
    for (auto& pr : split) n_shapes = std::max(n_shapes, candidate_shapes_w(lanes, pr.first, pr.second).size());
    for (size_t k = 0; k < n_shapes; k++) {
      NttPlan plan;
      for (auto& pr : split) {
        auto sh = candidate_shapes_w(lanes, pr.first, pr.second);
        if (!sh.empty()) plan.push_back(sh[std::min(k, sh.size() - 1)]);
      }
      if (plan.size() == split.size()) out.push_back(plan);
    }
  }
  return out;
}

struct PlanKey {
  int device, log_d, lanes, begin;
  bool operator<(const PlanKey& o) const {
    return std::tie(device, log_d, lanes, begin) < std::tie(o.device, o.log_d, o.lanes, o.begin);
  }
};
std::mutex g_plan_mu;
std::map<PlanKey, NttPlan>& tuned_plans() {
  static std::map<PlanKey, NttPlan> m;
  return m;
}

NttPlan plan_for(int log_d, int lanes, int layer_begin) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = tuned_plans().find({dev, log_d, lanes, layer_begin});
  return it != tuned_plans().end() ? it->second : default_plan(log_d, lanes, layer_begin);
}

// src != nullptr (forward only): the message whose replicate the first pass
// reads in place of data
void run_plan(const NttPlan& plan, f128* data, int log_d, int lanes, bool transpose, cudaStream_t s,
              const f128* src = nullptr) {
  if (plan.empty()) return;
  const f128* ev = device_evals(log_d);
  if (transpose)
    for (auto it = plan.rbegin(); it != plan.rend(); ++it) launch_pass(*it, data, ev, log_d, lanes, true, s);
  else
    for (size_t i = 0; i < plan.size(); i++) launch_pass(plan[i], data, ev, log_d, lanes, false, s, i ? nullptr : src);
}

void run_passes(f128* data, int log_d, int lanes, int layer_begin, bool transpose, cudaStream_t s) {
  run_plan(plan_for(log_d, lanes, layer_begin), data, log_d, lanes, transpose, s);
}
}  // namespace

void ntt_replicate_batch(const BatchJob* jobs, int n_jobs, uint64_t total, cudaStream_t s) {
  count_launch();
  k_replicate_batch<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(jobs, n_jobs, total);
}
// the batched pass kernel runs 256 threads: a warp-per-pair pass holds 8 tables
size_t ntt_pass_batch_smem(const NttPass& p) { return p.kind ? pass_w_smem(p.R, 256) : pass_smem(p.lgs, p.R); }
void ntt_pass_batch(const BatchJob* jobs, int n_jobs, int pass, uint64_t total_tiles, size_t smem, int grid,
                    cudaStream_t s) {
  if (smem > kSmem1) throw CudaError("ntt_pass_batch: tile larger than the shared-memory bound");
  CK(cudaFuncSetAttribute(k_ntt_pass_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem1));
  count_launch();
  k_ntt_pass_batch<<<(unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)grid, total_tiles)), 256, smem, s>>>(
      jobs, n_jobs, pass, total_tiles);
}

NttPlan ntt_autotune(f128* scratch, int log_d, int lanes, int layer_begin, cudaStream_t s, double* best_ms) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  const PlanKey key{dev, log_d, lanes, layer_begin};
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = tuned_plans().find(key);
    if (it != tuned_plans().end()) {
      if (best_ms) *best_ms = -1;
      return it->second;
    }
  }
  const int n_layers = log_d - layer_begin;
  if (n_layers <= 0) return {};
  const f128* ev = device_evals(log_d);
  {
    const size_t words = ((size_t)lanes << log_d) * 2;
    count_launch();
    k_fill_random<<<(unsigned)((words + 255) / 256), 256, 0, s>>>(reinterpret_cast<uint64_t*>(scratch), words);
    CK(cudaGetLastError());
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  // one warm launch, then the best of two timed launches (CUDA events on
  // the launching stream), on the random scratch filled above
  auto time_pass = [&](const NttPass& ps) {
    launch_pass(ps, scratch, ev, log_d, lanes, false, s);
    float best = 1e30f;
    for (int r = 0; r < 2; r++) {
      CK(cudaEventRecord(e0, s));
      launch_pass(ps, scratch, ev, log_d, lanes, false, s);
      CK(cudaEventRecord(e1, s));
      CK(cudaEventSynchronize(e1));
      float t = 0;
      CK(cudaEventElapsedTime(&t, e0, e1));
      best = std::min(best, t);
    }
    return (double)best;
  };
  std::map<std::pair<int, int>, std::pair<NttPass, double>> best_pass;  // (l0, R) -> fastest shape
  NttPlan best_plan;
  double best_total = 1e300;
  auto splits = candidate_splits(layer_begin, n_layers);
  for (auto& sp : candidate_splits_w(layer_begin, n_layers))
    if (std::find(splits.begin(), splits.end(), sp) == splits.end()) splits.push_back(sp);
  for (auto& split : splits) {
    NttPlan plan;
    double total = 0;
    for (auto& pr : split) {
      auto it = best_pass.find(pr);
      if (it == best_pass.end()) {
        NttPass bp{};
        double bt = 1e300;
        std::vector<NttPass> shapes;
        if (pr.second <= kMaxR + 1)
          for (auto& sh : candidate_shapes(lanes, pr.second)) shapes.push_back({pr.first, pr.second, sh.first, sh.second});
        for (auto& ps : candidate_shapes_w(lanes, pr.first, pr.second)) shapes.push_back(ps);
        for (auto& ps : shapes) {
          const double t = time_pass(ps);
          if (t < bt) { bt = t; bp = ps; }
        }
        it = best_pass.emplace(pr, std::make_pair(bp, bt)).first;
      }
      plan.push_back(it->second.first);
      total += it->second.second;
    }
    if (total < best_total) { best_total = total; best_plan = plan; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> lk(g_plan_mu);
  tuned_plans()[key] = best_plan;
  if (best_ms) *best_ms = best_total;
  return best_plan;
}

NttPlan ntt_plan(int log_d, int lanes, int layer_begin) { return plan_for(log_d, lanes, layer_begin); }
const f128* ntt_evals(int log_d) { return device_evals(log_d); }

std::string ntt_plan_desc(const NttPlan& plan) {
  std::string d;
  for (auto& ps : plan) {
    if (!d.empty()) d += " + ";
    d += "R" + std::to_string(ps.R) + "@l" + std::to_string(ps.l0) + " x" + std::to_string(1 << ps.lgs) +
         " lanes/" + std::to_string(ps.threads) + "t" + (ps.kind == 1 ? "/tab" : ps.kind == 2 ? "/tab+imad" : "");
  }
  return d;
}

size_t ntt_plan_count(int log_d, int lanes, int layer_begin) { return all_plans(log_d, lanes, layer_begin).size(); }
std::string ntt_plan_desc_at(int log_d, int lanes, int layer_begin, size_t index) {
  const auto plans = all_plans(log_d, lanes, layer_begin);
  return index < plans.size() ? ntt_plan_desc(plans[index]) : std::string();
}

void ntt_rs_encode_plan(const f128* msg, f128* cw, int log_msg_pos, int lanes, int log_inv_rate, size_t plan_idx,
                        cudaStream_t s) {
  const int log_d = log_msg_pos + log_inv_rate;
  auto plans = all_plans(log_d, lanes, log_inv_rate);
  if (plan_idx >= plans.size()) throw std::out_of_range("ntt plan index");
  size_t msg_len = ((size_t)lanes) << log_msg_pos;
  if (plans[plan_idx].empty() || plans[plan_idx][0].l0 != log_inv_rate) {
    count_launch(); k_replicate<<<(unsigned)((msg_len + 255) / 256), 256, 0, s>>>(msg, cw, msg_len, 1 << log_inv_rate);
    run_plan(plans[plan_idx], cw, log_d, lanes, false, s);
  } else {
    run_plan(plans[plan_idx], cw, log_d, lanes, false, s, msg);
  }
}

void ntt_rs_encode(const f128* msg, f128* cw, int log_msg_pos, int lanes, int log_inv_rate, cudaStream_t s) {
  const int log_d = log_msg_pos + log_inv_rate;
  const NttPlan plan = plan_for(log_d, lanes, log_inv_rate);
  if (plan.empty()) {  // no butterfly layer: the codeword is the replicate
    size_t msg_len = ((size_t)lanes) << log_msg_pos;
    count_launch(); k_replicate<<<(unsigned)((msg_len + 255) / 256), 256, 0, s>>>(msg, cw, msg_len, 1 << log_inv_rate);
    return;
  }
  run_plan(plan, cw, log_d, lanes, false, s, msg);  // the first pass reads the message's replicate in place
}

void ntt_forward(f128* data, int log_d, int lanes, int start_layer, cudaStream_t s) {
  run_passes(data, log_d, lanes, start_layer, false, s);
}

// out[j] (j < 2^log_msg) = sum_q E[q] * (codeword position q of unit message j);
// e is overwritten.
void ntt_transposed_encode(f128* e, f128* out, int log_msg, int log_inv_rate, cudaStream_t s) {
  run_passes(e, log_msg + log_inv_rate, 1, log_inv_rate, true, s);
  size_t len = (size_t)1 << log_msg;
  count_launch(); k_fold_copies<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(e, out, len, 1 << log_inv_rate);
}
