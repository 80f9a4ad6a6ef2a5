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
#include <vector>
#include "host.hpp"

namespace {
constexpr int kMaxR = 10;

struct PassArgs {
  f128* data;
  const f128* ev;  // ev[l * 32 + j] = W^_{d-l-1}(beta_{d-l+j}), j < l
  int log_d, lanes, lg_shift, l0, R;
};

__device__ __forceinline__ f128 twiddle(const f128* ev, int l, uint64_t b) {
  f128 t = mk(0, 0);
  for (int j = 0; j < l; j++)
    if ((b >> j) & 1) t = fx(t, ldg(ev + l * 32 + j));
  return t;
}

template <bool TRANSPOSE>
__global__ void __launch_bounds__(256, 2) k_ntt_pass(PassArgs p) {
  extern __shared__ f128 smem[];
  const int R = p.R, LG = 1 << p.lg_shift;
  f128* tile = smem;                       // [2^R][LG]
  f128* tw = smem + ((size_t)LG << R);     // [2^R - 1] : stage s block k at (1<<s)-1+k
  const int log_d = p.log_d, l0 = p.l0;
  const int lo_bits = log_d - l0 - R;      // position bits below the pair bits
  const int groups = p.lanes >> p.lg_shift;
  uint64_t t_id = blockIdx.x;
  const int grp = (int)(t_id % groups);
  t_id /= groups;
  const uint64_t lo = t_id & ((1ull << lo_bits) - 1);
  const uint64_t hi = t_id >> lo_bits;     // l0 bits
  const int n_el = LG << R;
  // load
  for (int e = threadIdx.x; e < n_el; e += blockDim.x) {
    uint64_t pl = (uint64_t)(e >> p.lg_shift);
    uint64_t pos = (hi << (log_d - l0)) | (pl << lo_bits) | lo;
    tile[e] = ld(p.data + pos * p.lanes + ((size_t)grp << p.lg_shift) + (e & (LG - 1)));
  }
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

__global__ void k_replicate(const f128* __restrict__ msg, f128* __restrict__ cw, size_t msg_len, int copies) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= msg_len) return;
  f128 v = ld(msg + i);
  for (int c = 0; c < copies; c++) st(cw + (size_t)c * msg_len + i, v);
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

void run_passes(f128* data, int log_d, int lanes, int layer_begin, bool transpose, cudaStream_t s) {
  const f128* ev = device_evals(log_d);
  int lg_shift = 0;
  while ((1 << (lg_shift + 1)) <= lanes && lg_shift < 3) lg_shift++;
  int n_layers = log_d - layer_begin;
  if (n_layers <= 0) return;
  int n_pass = (n_layers + kMaxR - 1) / kMaxR;
  std::vector<std::pair<int, int>> passes;  // (l0, R)
  int l = layer_begin;
  for (int i = 0; i < n_pass; i++) {
    int R = (n_layers - (l - layer_begin) + (n_pass - i) - 1) / (n_pass - i);
    passes.push_back({l, R});
    l += R;
  }
  if (transpose) std::reverse(passes.begin(), passes.end());
  for (auto& pr : passes) {
    // lanes per tile: as many as fit two CTAs per SM (<= 112 KiB of tile +
    // twiddles each), so one CTA's stage barriers overlap the other's work
    int lgs = lg_shift;
    auto tile_bytes = [&](int sh) {
      return ((size_t)(1 << sh) << pr.second) * sizeof(f128) + ((1 << pr.second) - 1) * sizeof(f128);
    };
    while (lgs > 0 && tile_bytes(lgs) > ((size_t)112 << 10)) lgs--;
    PassArgs a{data, ev, log_d, lanes, lgs, pr.first, pr.second};
    int LG = 1 << lgs;
    size_t smem = tile_bytes(lgs);
    uint64_t tiles = ((uint64_t)1 << (log_d - pr.second)) * (uint64_t)(lanes >> lgs);
    int threads = std::min(256, std::max(32, (LG << pr.second) / 2));
    if (transpose) {
      CK(cudaFuncSetAttribute(k_ntt_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      count_launch(); k_ntt_pass<true><<<(unsigned)tiles, threads, smem, s>>>(a);
    } else {
      CK(cudaFuncSetAttribute(k_ntt_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      count_launch(); k_ntt_pass<false><<<(unsigned)tiles, threads, smem, s>>>(a);
    }
  }
}
}  // namespace

void ntt_rs_encode(const f128* msg, f128* cw, int log_msg_pos, int lanes, int log_inv_rate, cudaStream_t s) {
  size_t msg_len = ((size_t)lanes) << log_msg_pos;
  count_launch(); k_replicate<<<(unsigned)((msg_len + 255) / 256), 256, 0, s>>>(msg, cw, msg_len, 1 << log_inv_rate);
  run_passes(cw, log_msg_pos + log_inv_rate, lanes, log_inv_rate, false, s);
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
