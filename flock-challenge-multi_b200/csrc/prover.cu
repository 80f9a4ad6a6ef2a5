// Host orchestration of the B200 prover: one proof = witness -> commit ->
// bind -> zerocheck -> lincheck -> ring switch + combine -> Ligerito open ->
// FLOCK bytes.  All O(witness) work runs in the kernels of K0..K9 on one
// stream; the host keeps the Fiat-Shamir transcript and exchanges only
// round messages, challenges, roots and opened rows with the device.
//
// Transcript order mirrors the reference verifier, which is its
// specification: crates/flock-core/src/verifier.rs:134-232 (bind, zerocheck,
// lincheck, claims), zerocheck.rs:1642-1797, lincheck.rs:5880-6050,
// pcs.rs:1861-1990, pcs/ring_switch.rs:4783-4811 and
// pcs/ligerito.rs:11321-11834; prover-side values follow
// crates/flock-prover/src/prover.rs:373-473 and pcs/ligerito.rs:8894-9100.
#include "prover.hpp"
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>

namespace flock {

namespace {
thread_local size_t t_alloc_bytes = 0;  // device bytes allocated by this thread's setups
// Setup buffers come from the stream-ordered allocator on the setup's own
// stream and go back to it the same way: cudaFree (and cudaFreeHost) wait for
// the whole device, so a setup built or evicted while other proofs run would
// stall every one of them until the longest kernel in flight ends.
template <class T>
T* dalloc(size_t n, cudaStream_t st) {
  T* p = nullptr;
  CK(cudaMallocAsync(reinterpret_cast<void**>(&p), n * sizeof(T) + 256, st));
  t_alloc_bytes += n * sizeof(T) + 256;
  return p;
}
// Page-locked host blocks are recycled rather than freed, for the same reason.
std::mutex g_pin_mu;
std::multimap<size_t, void*> g_pin_free;
void* pinned_take(size_t bytes) {
  {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_pin_free.find(bytes);
    if (it != g_pin_free.end()) {
      void* p = it->second;
      g_pin_free.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  CK(cudaMallocHost(&p, bytes));
  return p;
}
void pinned_give(void* p, size_t bytes) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_pin_mu);
  g_pin_free.emplace(bytes, p);
}

}  // namespace

// ---------------------------------------------------------------- setup --
size_t Setup::estimate_bytes(uint32_t log2, int hash) {
  const size_t n_words = (size_t)1 << (hash_k_log(hash) + std::max<int>(3, (int)log2) - 7);
  // z, a, b, 4 fold buffers, eq scratch, the rate-1/2 codeword (2x), its tree
  // (1/16 of a word per word), the Ligero levels and query basis (< 1/8),
  // blocks staging (25 u32 per compression) and chain records (28 u32),
  // statement and small tables
  return n_words * 16 * 10 + n_words * 2 + n_words * 2 + (n_words / 128) * 212 + ((size_t)96 << 20);
}

Setup::Setup(int device, uint32_t log2_, int stream_priority, int hash_, int merkle_fn_)
    : log2(log2_), hash(hash_), merkle_fn(merkle_fn_) {
  CK(cudaSetDevice(device));
  const size_t bytes0 = t_alloc_bytes;
  if (!known_hash(hash)) throw std::runtime_error("unknown statement hash");
  if (merkle_fn != kFnBlake3 && merkle_fn != kFnSha256) throw std::runtime_error("unknown Merkle hash");
  k_log = hash_k_log(hash);
  n_log = std::max<int>(3, (int)log2);
  m = k_log + n_log;
  lad = ladder_for(m);
  if (!lad) throw std::runtime_error("no Ligerito configuration for this size (m = " + std::to_string(m) + ")");
  n_words = (size_t)1 << (m - 7);
  digest = statement_digest(hash, m);
  CK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, stream_priority));
  z = dalloc<f128>(n_words, st);
  a = dalloc<f128>(n_words, st);
  b = dalloc<f128>(n_words, st);
  cw0 = dalloc<f128>(2 * n_words, st);
  n_leaves0 = (size_t)1 << (m - 12);
  tree0 = dalloc<uint32_t>(8 * (2 * n_leaves0 - 1), st);
  for (int i = 0; i < 4; i++) pp[i] = dalloc<f128>(n_words, st);
  eqbuf[0] = dalloc<f128>(n_words, st);
  // recursive Ligero levels
  int n_cur = m - 7 - lad->initial_k;
  for (size_t i = 0; i < lad->ks.size(); i++) {
    Level L;
    L.lanes = 1 << lad->ks[i];
    L.log_msg_pos = n_cur - lad->ks[i];
    L.rate = lad->rate[i + 1];
    L.positions = (size_t)1 << (L.log_msg_pos + L.rate);
    L.cw = dalloc<f128>(L.positions * L.lanes, st);
    L.tree = dalloc<uint32_t>(8 * (2 * L.positions - 1), st);
    levels.push_back(L);
    n_cur -= lad->ks[i];
  }
  induce_buf = dalloc<f128>((size_t)1 << (m - 7 - lad->initial_k + lad->rate[0]), st);
  out = dalloc<f128>(1024, st);
  tabs_r1 = dalloc<uint8_t>(round1_tables_size(), st);
  lag = dalloc<f128>(8 * 256, st);
  elo = dalloc<f128>(1 << 13, st);
  ehi = dalloc<f128>(1 << 16, st);
  const size_t kk = (size_t)1 << k_log;
  comb = dalloc<f128>(kk, st);
  zv = dalloc<f128>(kk, st);
  zv_pre = dalloc<f128>(kk, st);
  eq_inner = dalloc<f128>(kk, st);
  if (is_keccak(hash)) {
    kc_w = dalloc<f128>(keccak_comb_scratch(keccak_width(hash)), st);
    kc_masks = keccak_masks(device);
  }
  bc_tabs = dalloc<f128>(2 * 16 * 256, st);
  idx = dalloc<uint64_t>(1 << 16, st);
  gather = dalloc<f128>(1 << 16, st);
  d_found = dalloc<unsigned long long>(1, st);
  h_found = static_cast<unsigned long long*>(pinned_take(8));
  h_out = static_cast<f128*>(pinned_take(1024 * sizeof(f128)));
  h_stage = static_cast<uint8_t*>(pinned_take(kStageBytes));
  const Statement& S = statement(hash);
  at_ptr = dalloc<uint32_t>(S.at_ptr.size(), st);
  bt_ptr = dalloc<uint32_t>(S.bt_ptr.size(), st);
  at_row = dalloc<uint16_t>(S.at_row.size(), st);
  bt_row = dalloc<uint16_t>(S.bt_row.size(), st);
  // the allocations above are ordered on st: complete them before other
  // streams (the synchronous copies below, later a batch stream) touch them
  CK(cudaStreamSynchronize(st));
  CK(cudaMemcpy(at_ptr, S.at_ptr.data(), S.at_ptr.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(bt_ptr, S.bt_ptr.data(), S.bt_ptr.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(at_row, S.at_row.data(), S.at_row.size() * 2, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(bt_row, S.bt_row.data(), S.bt_row.size() * 2, cudaMemcpyHostToDevice));
  build_round1_tables();
  int dev_sms = 0;
  CK(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device));
  sms = dev_sms;
  for (int i = 0; i < kPhases + 1; i++) CK(cudaEventCreate(&ev[i]));
  tune_ntt_plans();
  capture_commit();
  CK(cudaStreamSynchronize(st));  // the buffers exist for every stream from here on
  device_bytes = t_alloc_bytes - bytes0;
}

// Tune the pass plans of every NTT shape a proof of this size runs, on this
// setup's own buffers before they hold data: the commitment (64 lanes, rate
// 1/2), each Ligero level, and the transposed encodes of the query-basis
// induction (one lane).
void Setup::tune_ntt_plans() {
  ntt_autotune(cw0, m - 12, 64, 1, st);
  for (auto& L : levels) ntt_autotune(L.cw, L.log_msg_pos + L.rate, L.lanes, L.rate, st);
  int n = m - 7 - lad->initial_k;
  ntt_autotune(induce_buf, n + lad->rate[0], 1, lad->rate[0], st);
  for (size_t i = 0; i + 1 < lad->ks.size(); i++) {
    n -= lad->ks[i];
    ntt_autotune(induce_buf, n + levels[i].rate, 1, levels[i].rate, st);
  }
  CK(cudaStreamSynchronize(st));
}

namespace {
// Capture the launches `body` issues on `st` into an executable graph;
// returns the graph and the number of kernel launches it holds.
template <class F>
cudaGraphExec_t capture(cudaStream_t st, uint64_t* launches, F&& body) {
  const uint64_t l0 = thread_launch_counter();
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaGraph_t g = nullptr;
  try {
    body();
  } catch (...) {
    cudaStreamEndCapture(st, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  CK(cudaStreamEndCapture(st, &g));
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  CK(e);
  // the capture counted its kernel nodes; they run once per replay
  *launches = thread_launch_counter() - l0;
  kernel_launch_counter().fetch_sub(*launches, std::memory_order_relaxed);
  thread_launch_counter() = l0;
  return exec;
}
}  // namespace

// FLOCK_COMMIT_GRAPHS=0 launches the same kernels directly (for profilers
// that replay kernels one at a time: ncu's replay of these graph nodes failed
// to launch on this driver).
void Setup::capture_commit() {
  const char* env = getenv("FLOCK_COMMIT_GRAPHS");
  if (env && strcmp(env, "0") == 0) return;
  commit_graph[0] = capture(st, &commit_launches[0], [&] { ntt_rs_encode(z, cw0, m - 13, 64, 1, st); });
  commit_graph[1] =
      capture(st, &commit_launches[1], [&] { merkle_build(cw0, n_leaves0, 64 * 16, tree0, merkle_fn, st); });
}

// Fused witness + RS encode + Merkle commit of several seeded proofs: every
// stage is one launch over all jobs (persistent NTT passes over the tiles of
// every job, one parent level of every tree per launch), captured as one
// CUDA graph and launched on `st`.  The setups' streams wait for it; each
// proof then continues with Setup::prove(..., committed = true).  The call
// returns once the work is queued; release the handle after `st` finished.
BatchCommit batch_commit_async(const std::vector<Setup*>& setups, const std::vector<uint64_t>& seeds,
                               cudaStream_t st) {
  BatchCommit h;
  const int n = (int)setups.size();
  if (n == 0) return h;
  if ((int)seeds.size() != n) throw std::runtime_error("batch_commit: one seed per setup");
  std::vector<BatchJob> J(n);
  uint64_t wcta = 0, rep = 0, leaves = 0, tiles[4] = {0, 0, 0, 0}, par[24] = {0};
  size_t smem = 0;
  int max_pass = 0, max_level = 0;
  for (int i = 0; i < n; i++) {
    Setup& S = *setups[i];
    BatchJob& b = J[i];
    b = BatchJob{};
    b.seed = seeds[i];
    b.log2 = S.log2;
    b.n_blocks = 1u << S.log2;
    b.n_slots = 1u << S.n_log;
    b.z = S.z; b.a = S.a; b.b = S.b;
    b.wcta0 = wcta;
    wcta += witness_ctas(b.n_slots);
    b.cw = S.cw0;
    b.log_d = S.m - 12;
    b.ev = ntt_evals(b.log_d);
    b.msg_len = S.n_words;
    b.rep0 = rep;
    rep += b.msg_len;
    const NttPlan plan = ntt_plan(b.log_d, 64, 1);
    if (plan.size() > 4) throw std::runtime_error("batch_commit: more than four NTT passes");
    b.n_pass = (int)plan.size();
    max_pass = std::max(max_pass, b.n_pass);
    for (int p = 0; p < 4; p++) {
      b.tile0[p] = tiles[p];
      if (p < b.n_pass) {
        b.pass[p] = plan[p];
        tiles[p] += ((uint64_t)1 << (b.log_d - plan[p].R)) * (uint64_t)(64 >> plan[p].lgs);
        smem = std::max(smem, ntt_pass_batch_smem(plan[p]));
      }
    }
    b.tree = S.tree0;
    b.n_leaves = S.n_leaves0;
    b.leaf0 = leaves;
    leaves += b.n_leaves;
    uint64_t start = 0, len = b.n_leaves;
    int level = 0;
    for (int l = 0; l < 24; l++) b.par0[l] = par[l];
    while (len > 1024) {
      level++;
      if (level >= 24) throw std::runtime_error("batch_commit: tree too deep");
      b.par0[level] = par[level];
      par[level] += len >> 1;
      start += len;
      len >>= 1;
    }
    max_level = std::max(max_level, level);
    b.top_start = start;
    b.top_len = len;
  }
  // empty ranges for the jobs after the last one that takes part in a launch
  for (int i = 0; i < n; i++)
    for (int l = 0; l < 24; l++) J[i].par0[l] = std::min<uint64_t>(J[i].par0[l], par[l]);
  BatchJob* dj = nullptr;
  CK(cudaMallocAsync(reinterpret_cast<void**>(&dj), n * sizeof(BatchJob), st));
  h.jobs = dj;
  h.st = st;
  try {
    CK(cudaMemcpyAsync(dj, J.data(), n * sizeof(BatchJob), cudaMemcpyHostToDevice, st));
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint64_t launches = 0;
    cudaGraphExec_t g = capture(st, &launches, [&] {
      launch_witness_seed_batch(dj, n, (uint32_t)wcta, st);
      // pass 0 reads each job's message as its replicated codeword
      for (int p = 0; p < max_pass; p++) ntt_pass_batch(dj, n, p, tiles[p], smem, 2 * sms, st);
      merkle_leaves_batch(dj, n, leaves, st);
      for (int l = 1; l <= max_level; l++) merkle_parents_batch(dj, n, l, par[l], st);
      merkle_top_batch(dj, n, st);
    });
    h.graph = g;
    CK(cudaGraphLaunch(g, st));
    count_launch(launches);
    CK(cudaEventCreateWithFlags(&h.done, cudaEventDisableTiming));
    CK(cudaEventRecord(h.done, st));
    for (Setup* S : setups) CK(cudaStreamWaitEvent(S->st, h.done, 0));
  } catch (...) {
    cudaStreamSynchronize(st);
    batch_commit_release(h);
    throw;
  }
  return h;
}

void batch_commit_release(BatchCommit& h) {
  if (h.done) cudaEventDestroy(h.done);
  if (h.graph) cudaGraphExecDestroy(h.graph);
  if (h.jobs) cudaFreeAsync(h.jobs, h.st);
  h = BatchCommit{};
}

void batch_commit(const std::vector<Setup*>& setups, const std::vector<uint64_t>& seeds, cudaStream_t st) {
  BatchCommit h = batch_commit_async(setups, seeds, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  batch_commit_release(h);
  CK(e);
}

Setup::~Setup() {
  cudaStreamSynchronize(st);
  void* ptrs[] = {z, a, b, cw0, tree0, pp[0], pp[1], pp[2], pp[3], eqbuf[0], zv_pre, induce_buf, out, blocks_buf, records_buf,
                  tabs_r1, lag, elo, ehi, comb, zv, eq_inner, bc_tabs, idx, gather, d_found, at_ptr, bt_ptr,
                  at_row, bt_row, kc_w};
  for (void* p : ptrs)
    if (p) cudaFreeAsync(p, st);
  for (auto& L : levels) {
    if (L.cw) cudaFreeAsync(L.cw, st);
    if (L.tree) cudaFreeAsync(L.tree, st);
  }
  pinned_give(h_found, 8);
  pinned_give(h_out, 1024 * sizeof(f128));
  pinned_give(h_stage, kStageBytes);
  for (auto g : commit_graph)
    if (g) cudaGraphExecDestroy(g);
  for (int i = 0; i < kPhases + 1; i++) cudaEventDestroy(ev[i]);
  cudaStreamDestroy(st);
}

// Round-1 constant tables: the GF(2^8) S -> Lambda extension matrix (Lagrange
// basis of the nodes 0..63 evaluated at 64..127), log/exp tables, phi8 and
// the small-eq weights g(xs) with eq(r[6..9], xs) = phi8(g(xs)).
void Setup::build_round1_tables() {
  std::vector<uint8_t> host(round1_tables_size(), 0);
  uint8_t exp_[512], log_[256];
  uint8_t x = 1;  // generator 3 of GF(2^8)*
  for (int i = 0; i < 255; i++) {
    exp_[i] = x;
    log_[x] = (uint8_t)i;
    x = hgf8_mul(x, 3);
  }
  for (int i = 255; i < 512; i++) exp_[i] = exp_[i - 255];
  auto ginv = [&](uint8_t v) { return exp_[(255 - log_[v]) % 255]; };
  uint8_t(&M)[64][64] = lde_m;  // M[l][s] = L_s(64 + l) over nodes 0..63 in GF(2^8)
  for (int l = 0; l < 64; l++) {
    uint8_t pt = (uint8_t)(64 + l);
    for (int s = 0; s < 64; s++) {
      uint8_t num = 1, den = 1;
      for (int j = 0; j < 64; j++) {
        if (j == s) continue;
        num = hgf8_mul(num, pt ^ (uint8_t)j);
        den = hgf8_mul(den, (uint8_t)s ^ (uint8_t)j);
      }
      M[l][s] = hgf8_mul(num, ginv(den));
    }
  }
  build_round1_tables_host(M, phi8_table(), host.data());
  CK(cudaMemcpy(tabs_r1, host.data(), host.size(), cudaMemcpyHostToDevice));
}

// eq table of r into dev (length 2^|r|), as lo (<= 12 vars) x hi on the device
void Setup::eq_table(const std::vector<f128>& r, f128* dev) {
  size_t n = r.size();
  int s = (int)std::min<size_t>(n, 12);
  eq_build(r.data(), s, hone(), elo, st);
  eq_build(r.data() + s, (int)n - s, hone(), ehi, st);
  eq_split(elo, ehi, s, (size_t)1 << n, dev, st);
}

void Setup::fetch(const f128* dev, size_t n, f128* host) {
  CK(cudaMemcpyAsync(host, dev, n * sizeof(f128), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
}

uint64_t Setup::grind(Transcript& tr, uint32_t bits) {
  uint64_t nonce = 0;
  if (bits) {
    uint8_t d[32];
    tr.state_digest(d);
    // a few dozen hashes on the host cost less than a round trip to the GPU
    nonce = bits <= kHostPowBits ? pow_search_host(d, bits, tr.fn())
                                 : pow_search(d, bits, st, d_found, h_found, tr.fn());
  }
  tr.nonce(nonce);
  return nonce;
}

std::vector<size_t> Setup::sample_queries(Transcript& tr, size_t block_len, size_t count) {
  return sample_distinct_queries(tr, block_len, count);
}

// Opened rows + Merkle multi-proof (merkle.rs:1074-1120 index order).  The
// sibling indices depend only on the queries, so both gathers are issued
// together and read back with one synchronisation.
void Setup::open(Opening& o, const f128* cw, const uint32_t* tree, size_t n_leaves, int lanes,
                 const std::vector<size_t>& q) {
  const std::vector<uint64_t> ids = multiproof_ids(q, n_leaves);
  const size_t nq = q.size(), ns = ids.size() - nq, nr = nq * lanes;
  if (ids.size() > ((size_t)1 << 16) || nr + 2 * ns > ((size_t)1 << 16))
    throw std::runtime_error("opening larger than the gather buffers");
  CK(cudaMemcpyAsync(idx, ids.data(), ids.size() * 8, cudaMemcpyHostToDevice, st));
  count_launch(); k_gather_rows<<<(unsigned)((nr + 255) / 256), 256, 0, st>>>(cw, idx, nq, lanes, gather);
  uint32_t* nodes = reinterpret_cast<uint32_t*>(gather + nr);  // 32 B per node = 2 f128
  if (ns) {
    count_launch(); k_gather_nodes<<<(unsigned)((ns + 127) / 128), 128, 0, st>>>(tree, idx + nq, ns, nodes);
  }
  // nothing on the host reads the opening before the proof is encoded: copy
  // it into the pinned staging area and unpack it after the proof's final
  // synchronisation (finish_openings), with no wait of its own
  const size_t need = nr * sizeof(f128) + ns * 32;
  if (stage_off_ + need > kStageBytes) throw std::runtime_error("openings larger than the staging area");
  CK(cudaMemcpyAsync(h_stage + stage_off_, gather, nr * sizeof(f128), cudaMemcpyDeviceToHost, st));
  if (ns) CK(cudaMemcpyAsync(h_stage + stage_off_ + nr * sizeof(f128), nodes, ns * 32, cudaMemcpyDeviceToHost, st));
  pending_.push_back(PendingOpen{&o, stage_off_, nq, (size_t)lanes, ns});
  stage_off_ += need;
}

void Setup::finish_openings() {
  for (const PendingOpen& p : pending_) {
    const f128* rows = reinterpret_cast<const f128*>(h_stage + p.off);
    p.o->rows.clear();
    for (size_t i = 0; i < p.nq; i++) p.o->rows.emplace_back(rows + i * p.lanes, rows + (i + 1) * p.lanes);
    p.o->proof.resize(p.ns);
    if (p.ns) memcpy(p.o->proof.data(), h_stage + p.off + p.nq * p.lanes * sizeof(f128), p.ns * 32);
  }
  pending_.clear();
  stage_off_ = 0;
}

H32 Setup::root_of(const uint32_t* tree, size_t n_leaves) {
  H32 r;
  CK(cudaMemcpyAsync(r.data(), tree + 8 * (2 * n_leaves - 2), 32, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return r;
}

void Setup::mark(int phase) {
  if (phase >= 0 && phase <= kPhases) CK(cudaEventRecord(ev[phase], st));
}

// -------------------------------------------------------------- prove --
// Host buffers handed to cudaMemcpyAsync here are either pinned (h_out,
// h_found, h_stage) and read only after a synchronisation, or pageable, which
// the runtime stages before the call returns: the stream needs no
// synchronisation except where the transcript reads a device value.
std::vector<uint8_t> Setup::prove(const uint64_t* seed, const uint32_t* blocks_dev, size_t n_blocks,
                                  const std::string& domain, bool committed, const ChainEnds* chain,
                                  bool full_records, const MerkleArgs* merkle) {
  Proof P;
  P.m = (uint64_t)m;
  P.merkle_fn = merkle_fn;
  pending_.clear();  // (left over only by a proof that threw)
  stage_off_ = 0;
  const int gs = grid_sms > 0 && grid_sms < sms ? grid_sms : sms;
  const int G = gs * 4;
  const uint32_t n_slots = 1u << n_log;
  mark(0);
  if (hash != kHashBlake3 && committed) throw std::runtime_error("batched commits are BLAKE3 statements");
  if (chain && hash != kHashBlake3 && hash != kHashSha256 && hash != kHashKeccak)
    throw std::runtime_error("hash chains are BLAKE3, SHA-256 or Keccak statements");
  if (merkle && (hash != kHashSha256 || n_blocks != n_slots || !merkle->b_bits || merkle->path_log < 0 ||
                 merkle->path_log > n_log))
    throw std::runtime_error("a Merkle path is a SHA-256 statement whose paths fill every slot");
  if (!committed && is_keccak(hash)) {
    // ---- K0 witness of Keccak-f[1600] permutations (states of 25 u64)
    const uint32_t nb = n_blocks ? (uint32_t)n_blocks : 1u << log2;
    launch_witness_keccak(seed ? nullptr : reinterpret_cast<const uint64_t*>(blocks_dev), seed ? *seed : 0, nb,
                          n_slots, z, a, b, st, keccak_width(hash));
    CK(cudaGetLastError());
  } else if (!committed && hash == kHashSha256) {
    // ---- K0 witness of SHA-256 compressions
    const uint32_t nb = n_blocks ? (uint32_t)n_blocks : 1u << log2;
    launch_witness_sha(seed ? nullptr : blocks_dev, seed ? *seed : 0, nb, n_slots, z, a, b, st);
    CK(cudaGetLastError());
  } else if (!committed) {
    // ---- K0 witness
    if (seed) launch_witness_seed(*seed, log2, 1u << log2, n_slots, z, a, b, st);
    else launch_witness_blocks(blocks_dev, (uint32_t)n_blocks, n_slots, z, a, b, st, chain != nullptr || full_records);
    CK(cudaGetLastError());
  }
  mark(1);
  // ---- K1 + K2 commit: 64 interleaved lanes, rate 1/2, 1 KiB leaves (two
  // captured graphs, the phase event between them); a batch commit
  // (batch_commit) has already filled z, a, b, the codeword and the tree
  if (!committed) {
    if (commit_graph[0]) {
      CK(cudaGraphLaunch(commit_graph[0], st));
      count_launch(commit_launches[0]);
    } else {
      ntt_rs_encode(z, cw0, m - 13, 64, 1, st);
    }
  }
  mark(2);
  if (!committed) {
    if (commit_graph[1]) {
      CK(cudaGraphLaunch(commit_graph[1], st));
      count_launch(commit_launches[1]);
    } else {
      merkle_build(cw0, n_leaves0, 64 * 16, tree0, merkle_fn, st);
    }
  }
  P.root = root_of(tree0, n_leaves0);
  mark(3);

  Transcript tr(domain, fs_fn);
  tr.label("flock-r1cs-v0");
  tr.bytes(digest.data(), 32);
  tr.bytes(P.root.data(), 32);

  // ---- zerocheck
  tr.label("flock-zerocheck-v0");
  std::vector<f128> r = tr.sample_vec(6);
  std::vector<f128> r_outer = tr.sample_vec(m - 13);
  for (f128 v : small_consts()) r.push_back(v);
  std::vector<f128> med = medium_consts();
  for (f128 v : med) r.push_back(v);
  r.insert(r.end(), r_outer.begin(), r_outer.end());
  {
    f128 C = hone();
    for (f128 bm : med) C = hmul(C, fx(hone(), bm));
    std::vector<f128> rh(r.begin() + 13, r.end());
    int s = (int)std::min<size_t>(rh.size(), 12);
    eq_build(rh.data(), s, hone(), elo, st);
    eq_build(rh.data() + s, (int)rh.size() - s, C, ehi, st);
    eq_split(elo, ehi, s, (size_t)1 << rh.size(), scratch_eq(), st);
    CK(cudaMemsetAsync(out, 0, 1024 * sizeof(f128), st));
    size_t n_blocks128 = (size_t)1 << (m - 13);
    zc_round1(a, b, z, tabs_r1, scratch_eq(), n_blocks128, out, gs, st);
    fetch(out, 1024, h_out);
    // from here on `out` is a ring of 128 zeroed 8-value slots: every round
    // message accumulates into a fresh slot, so no round needs its own clear
    CK(cudaMemsetAsync(out, 0, 1024 * sizeof(f128), st));
    // P_AB(l) = sum_k phi8(e_k) H(l, k)
    const f128* phi8 = phi8_table();
    P.r1_ab.assign(64, mk(0, 0));
    for (int l = 0; l < 64; l++)
      for (int k = 0; k < 8; k++) P.r1_ab[l] = fx(P.r1_ab[l], hmul(phi8[1 << k], h_out[l * 8 + k]));
    // c-claim ring-switch statistic (suffix r[7..m]):
    // sv[s + 64 h] = sum_j phi8(g2(j)) H_C(s, h, j), g2(j) = eq(r[7..9], j)
    // over GF(2^8) with the small constants 0x53, 0xB5
    s_hat_v_c.assign(128, mk(0, 0));
    for (int j = 0; j < 4; j++) {
      uint8_t g2 = 1;
      g2 = hgf8_mul(g2, (j & 1) ? 0x53 : (uint8_t)(1 ^ 0x53));
      g2 = hgf8_mul(g2, (j & 2) ? 0xB5 : (uint8_t)(1 ^ 0xB5));
      for (int h = 0; h < 2; h++)
        for (int s = 0; s < 64; s++)
          s_hat_v_c[64 * h + s] = fx(s_hat_v_c[64 * h + s], hmul(phi8[g2], h_out[512 + s * 8 + 4 * h + j]));
    }
    // extract-c message: S_s = (1 + r6) sv[s] + r6 sv[64 + s];
    // P_C(l) = sum_s phi8(M[l][s]) S_s
    P.r1_c.assign(64, mk(0, 0));
    for (int s = 0; s < 64; s++) {
      f128 S = fx(hmul(fx(hone(), r[6]), s_hat_v_c[s]), hmul(r[6], s_hat_v_c[64 + s]));
      for (int l = 0; l < 64; l++)
        if (lde_m[l][s]) P.r1_c[l] = fx(P.r1_c[l], hmul(phi8_table()[lde_m[l][s]], S));
    }
  }
  mark(4);
  tr.f128s(P.r1_ab.data(), 64);
  tr.f128s(P.r1_c.data(), 64);
  f128 zc_z = tr.sample();
  {
    std::vector<f128> L = hlagrange(zc_z, 0);
    std::vector<f128> lagt(8 * 256);
    for (int k = 0; k < 8; k++) subset_sums8(L.data() + 8 * k, lagt.data() + k * 256);
    CK(cudaMemcpyAsync(lag, lagt.data(), lagt.size() * sizeof(f128), cudaMemcpyHostToDevice, st));
    std::vector<f128> LL = hlagrange(zc_z, 64);
    f128 ce = mk(0, 0);
    for (int i = 0; i < 64; i++) ce = fx(ce, hmul(LL[i], P.r1_c[i]));
    P.fc = ce;
  }
  int out_slot = 0;
  auto next_out = [&](int nslots) -> f128* {
    if (out_slot + nslots > 128) {
      CK(cudaMemsetAsync(out, 0, 1024 * sizeof(f128), st));
      out_slot = 0;
    }
    f128* p = out + 8 * out_slot;
    out_slot += nslots;
    return p;
  };
  const int n_mlv = m - 6;
  std::vector<f128> rhos;
  // Message of round k weights pair j by eq(r[7+k..m], j).  Its low bits sit
  // on the fixed small (phi8) and medium (x^(2^t) / (1 + x^(2^t))) challenges:
  // the kernel needs ns, nm, the medium shift, and eq over the random suffix;
  // it returns per-js sums that are weighted here by
  // K[js] = phi8(g(js)) * C_round / C_full.
  // The eq over the random suffix stays on the device: rounds 0..6 share
  // eq(r[13..m]) (the round-1 table, which carries the medium factor C of
  // all four medium bits); from round 7 on, each round's table is the
  // previous one with its lowest variable summed out.
  f128 C_full = hone();
  for (f128 bm : medium_consts()) C_full = hmul(C_full, fx(hone(), bm));
  const f128 C_inv = hinv(C_full);
  const f128* etab = scratch_eq();
  size_t etab_len = (size_t)1 << (m - 13), etab_off = etab_len;
  auto run_round = [&](int k, int mode, const f128* ain, const f128* bin, f128* aout, f128* bout, f128 rho,
                       size_t n_pairs) {
    const int st0 = 7 + k;
    const int ns = std::max(0, 9 - st0);
    const int med0 = std::max(st0, 9);
    const int nm = med0 <= 13 ? 13 - med0 : 0;
    f128 C = C_inv;
    for (int t = 0; t < nm; t++) C = hmul(C, fx(hone(), r[med0 + t]));
    const uint8_t sc[3] = {0xF7, 0x53, 0xB5};  // r[6], r[7], r[8] = phi8(sc)
    f128 K[4] = {};
    for (int js = 0; js < (1 << ns); js++) {
      uint8_t g = 1;
      for (int t = 0; t < ns; t++) {
        uint8_t s8 = sc[st0 - 6 + t];
        g = hgf8_mul(g, ((js >> t) & 1) ? s8 : (uint8_t)(1 ^ s8));
      }
      K[js] = hmul(phi8_table()[g], C);
    }
    // the next round's table drops r[st0]: this round's launch writes it
    f128* nxt = nullptr;
    size_t nxt_len = 0;
    if (st0 + 1 > 13 && k + 1 < n_mlv) {
      nxt = scratch_eq() + etab_off;
      nxt_len = etab_len / 2;
    }
    f128* o = next_out(1);
    zc_round(mode, ain, bin, aout, bout, lag, rho, n_pairs, ns, nm, med0 - 9, etab, o, gs, st, nxt, nxt_len);
    if (nxt) {
      etab = nxt;
      etab_len = nxt_len;
      etab_off += nxt_len;
    }
    fetch(o, 8, h_out);
    f128 g1 = mk(0, 0), gi = mk(0, 0);
    for (int js = 0; js < (1 << ns); js++) {
      g1 = fx(g1, hmul(K[js], h_out[2 * js]));
      gi = fx(gi, hmul(K[js], h_out[2 * js + 1]));
    }
    h_out[0] = g1;
    h_out[1] = gi;
  };
  // The last rounds' vectors are small.  Once a round has at most
  // kHostZcPairs pairs and only the random suffix weights its pairs (round 7
  // on), the remaining rounds run on the host from one copy of the vectors
  // and the eq table: the same folds and sums, without a GPU round trip per
  // round (a 512-pair round is about 4 K host products, 20 us).
  constexpr size_t kHostZcPairs = 512;
  bool host_tail = false;
  std::vector<f128> ha, hb, he;  // the vectors and eq table once on the host
  auto host_round = [&](f128 rho) {
    // fold the 4n values of a and b at rho into 2n, then the message over the
    // n folded pairs with this round's eq weights, then halve the eq table
    const size_t n = he.size();
    for (size_t j = 0; j < 2 * n; j++) {
      ha[j] = fx(ha[2 * j], hmul(rho, fx(ha[2 * j], ha[2 * j + 1])));
      hb[j] = fx(hb[2 * j], hmul(rho, fx(hb[2 * j], hb[2 * j + 1])));
    }
    ha.resize(2 * n);
    hb.resize(2 * n);
    f128 g1 = mk(0, 0), gi = mk(0, 0);
    for (size_t j = 0; j < n; j++) {
      const f128 a0 = ha[2 * j], a1 = ha[2 * j + 1], b0 = hb[2 * j], b1 = hb[2 * j + 1];
      g1 = fx(g1, hmul(he[j], hmul(a1, b1)));
      gi = fx(gi, hmul(he[j], hmul(fx(a0, a1), fx(b0, b1))));
    }
    const f128 K0 = hmul(phi8_table()[1], C_inv);  // ns = nm = 0: phi8(1) * C_round / C_full
    h_out[0] = hmul(K0, g1);
    h_out[1] = hmul(K0, gi);
    for (size_t j = 0; j < n / 2; j++) he[j] = fx(he[2 * j], he[2 * j + 1]);
    he.resize(n / 2);
  };
  run_round(0, 0, a, b, nullptr, nullptr, mk(0, 0), n_words);
  f128* av = pp[0];
  f128* bv = pp[1];
  f128* av2 = pp[2];
  f128* bv2 = pp[3];
  for (int i = 0; i < n_mlv; i++) {
    P.zc_rounds.push_back({h_out[0], h_out[1]});
    tr.f128v(h_out[0]);
    tr.f128v(h_out[1]);
    f128 rho = tr.sample();
    rhos.push_back(rho);
    if (i < n_mlv - 1) {
      size_t n_pairs_out = (size_t)1 << (n_mlv - i - 2);
      if (!host_tail && i + 1 >= 7 && n_pairs_out <= kHostZcPairs) {
        // av, bv hold the 4 n values the round folds; etab its n eq weights
        ha.resize(4 * n_pairs_out);
        hb.resize(4 * n_pairs_out);
        he.resize(n_pairs_out);
        CK(cudaMemcpyAsync(ha.data(), av, ha.size() * sizeof(f128), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hb.data(), bv, hb.size() * sizeof(f128), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(he.data(), etab, he.size() * sizeof(f128), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        host_tail = true;
      }
      if (host_tail) host_round(rho);
      else if (i == 0) run_round(1, 1, a, b, av, bv, rho, n_pairs_out);
      else {
        run_round(i + 1, 2, av, bv, av2, bv2, rho, n_pairs_out);
        std::swap(av, av2);
        std::swap(bv, bv2);
      }
    } else if (host_tail) {  // the last pair, folded at rho
      P.fa = fx(ha[0], hmul(rho, fx(ha[0], ha[1])));
      P.fb = fx(hb[0], hmul(rho, fx(hb[0], hb[1])));
    } else {
      f128* o = next_out(1);
      fold_pair_final(av, bv, rho, o, st);
      fetch(o, 2, h_out);
      P.fa = h_out[0];
      P.fb = h_out[1];
    }
  }
  tr.f128v(P.fa);
  tr.f128v(P.fb);
  mark(5);

  // ---- lincheck
  const int ir = k_log - kKSkip;
  const int kk = 1 << k_log;
  std::vector<f128> x_inner(rhos.begin(), rhos.begin() + ir), x_outer(rhos.begin() + ir, rhos.end());
  tr.label("flock-lincheck-v0");
  f128 alpha = tr.sample();
  f128 beta = tr.sample();
  {
    // eq_inner[s + 64 k] = L_s(z) eq(x_inner, k)
    std::vector<f128> L = hlagrange(zc_z, 0);
    eq_build(x_inner.data(), (int)x_inner.size(), hone(), zv_pre, st);
    outer64(L.data(), zv_pre, (size_t)1 << x_inner.size(), eq_inner, st);
    if (is_keccak(hash)) keccak_comb(eq_inner, alpha, beta, kc_masks, kc_w, comb, st, keccak_width(hash));
    else lc_comb(at_ptr, at_row, bt_ptr, bt_row, eq_inner, alpha, beta, statement(hash).z_const, kk, comb, st);
    eq_table(x_outer, scratch_eq());
    CK(cudaMemsetAsync(zv, 0, kk * sizeof(f128), st));
    lc_zvec(z, scratch_eq(), (size_t)1 << (m - k_log), k_log, zv, gs, st);
    // pre-sumcheck z_vec: the ab-claim's ring-switch statistic is read from it
    CK(cudaMemcpyAsync(zv_pre, zv, kk * sizeof(f128), cudaMemcpyDeviceToDevice, st));
  }
  std::vector<f128> rr;
  int len = kk;
  // the round kernel adds its message atomically into a fresh slot
  f128* lo_ = next_out(1);
  lc_round(comb, zv, len, false, mk(0, 0), true, lo_, st);
  for (int k = 0; k < ir; k++) {
    fetch(lo_, 2, h_out);
    P.lc_rounds.push_back({h_out[0], h_out[1]});
    tr.f128v(h_out[0]);
    tr.f128v(h_out[1]);
    f128 rk = tr.sample();
    rr.push_back(rk);
    len >>= 1;
    if (k + 1 < ir) lo_ = next_out(1);
    lc_round(comb, zv, len, true, rk, k + 1 < ir, lo_, st);
  }
  P.z_partial.resize(64);
  fetch(zv, 64, P.z_partial.data());
  tr.f128s(P.z_partial.data(), 64);
  f128 r_skip2 = tr.sample();
  std::vector<f128> r_inner_rest(rr.rbegin(), rr.rend());
  (void)r_skip2;
  mark(6);

  // ---- hash chain (chain_common.rs:318-324): tau_pos folds each instance's
  // input cv and output out_lo to one value (g = [In | Out]); the shift
  // sumcheck (chain.rs:155-236) over W(y, s0) g(y, s0), s0 the high
  // variable, runs on the lincheck's round kernel (same message and
  // top-variable fold) and leaves one packed-direct claim z(point) = value,
  // point = [tau_pos, s0*, 0^5, tau'].  pp[2], pp[3] are free until the
  // Ligerito folds.
  std::vector<f128> pd_point;
  f128 pd_value = mk(0, 0);
  if (chain) {
    const ChainGeom CG = chain_geom(hash);
    P.chain = true;
    P.chain_kind = (uint32_t)CG.kind;
    P.end_bits = CG.region_bits;
    memcpy(P.end0, chain->in, sizeof(P.end0));
    memcpy(P.end_last, chain->out, sizeof(P.end_last));
    const size_t N = n_slots;
    const std::vector<f128> tau_pos = tr.sample_vec((size_t)CG.region_log - 7);
    const std::vector<f128> et = heq(tau_pos);  // one weight per packed word of a region
    f128* g = pp[2];
    f128* w = pp[3];
    chain_fold(z, N, (size_t)1 << (k_log - 7), et.data(), (int)et.size(), CG.out_word, g, st);
    const std::vector<f128> tau = tr.sample_vec((size_t)n_log);
    const f128 alpha = tr.sample();
    // W(y, 0) = eq(tau, y - 1) for y >= 1, W(0, 0) = alpha; W(y, 1) = eq(tau, y)
    eq_table(tau, w + N);
    CK(cudaMemcpyAsync(w + 1, w + N, (N - 1) * sizeof(f128), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(w, &alpha, sizeof(f128), cudaMemcpyHostToDevice, st));
    int len = (int)(2 * N);
    f128* so = next_out(1);
    lc_round(w, g, len, false, mk(0, 0), true, so, st);
    std::vector<f128> rs;
    for (int k = 0; k <= n_log; k++) {
      // the last message is over g[0], g[1]; the final fold happens here
      if (k == n_log) CK(cudaMemcpyAsync(h_out + 2, g, 2 * sizeof(f128), cudaMemcpyDeviceToHost, st));
      fetch(so, 2, h_out);
      P.shift_rounds.push_back({h_out[0], h_out[1]});
      tr.f128v(h_out[0]);
      tr.f128v(h_out[1]);
      const f128 rk = tr.sample();
      rs.push_back(rk);
      if (k < n_log) {
        len >>= 1;
        so = next_out(1);
        lc_round(w, g, len, true, rk, true, so, st);
      } else {
        pd_value = fx(h_out[2], hmul(rk, fx(h_out[3], h_out[2])));
      }
    }
    P.g_at_point = pd_value;
    // round k bound variable n_log - k; variable n_log is s0; the point is
    // [tau_pos, s0, 0^(k_log - region_log - 1), instance] (k_log - 7 slot
    // coordinates; chain_common.rs:211-231)
    const size_t off = (size_t)k_log - 7, tl = tau_pos.size();
    pd_point.assign(off + (size_t)n_log, mk(0, 0));
    for (size_t j = 0; j < tl; j++) pd_point[j] = tau_pos[j];
    pd_point[tl] = rs[0];
    for (int k = 1; k <= n_log; k++) pd_point[off + (size_t)(n_log - k)] = rs[k];
  }

  // ---- Merkle paths (merkle_path_common.rs:314-430): tau_pos folds each
  // instance's four 256-bit slots (H_in, H_out = Z, M_lo = X_L, M_hi = X_R);
  // the shift sumcheck (merkle_path.rs:226-467) runs n degree-3 rounds over
  // seven tables on the device, binding the top instance variable, then two
  // degree-2 rounds over the slot selector on the host; it leaves one
  // packed-direct claim z(point) = g, point = [tau_pos, sel_slot, side, 0^5,
  // instance].  pp[2] holds the slot folds, pp[3] the weight tables.
  if (merkle) {
    P.merkle = true;
    const size_t N = n_slots;
    const int n = n_log, pos_log = n_log - merkle->path_log;
    const f128 tau_pos = tr.sample_vec(1)[0];
    f128* sl = pp[2];  // [H_in | H_out | M_lo | M_hi], N each
    f128 *ta = pp[3], *te = pp[3] + N, *tb = pp[3] + 2 * N, *eq_q = pp[3] + 3 * N, *eq_p = pp[3] + 4 * N;
    uint8_t* bdev = reinterpret_cast<uint8_t*>(pp[3] + 5 * N);
    mp_fold(z, N, fx(hone(), tau_pos), tau_pos, sl, st);
    const std::vector<f128> tau = tr.sample_vec((size_t)n);
    const f128 alpha = tr.sample();
    const std::vector<f128> tq(tau.begin(), tau.begin() + pos_log), tp(tau.begin() + pos_log, tau.end());
    const std::vector<f128> eqp = heq(tp);
    eq_table(tau, te);
    eq_table(tq, eq_q);
    CK(cudaMemcpyAsync(eq_p, eqp.data(), eqp.size() * sizeof(f128), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(bdev, merkle->b_bits, N, cudaMemcpyHostToDevice, st));
    mp_tables(eq_q, eq_p, alpha, pos_log, N, bdev, ta, tb, st);
    MpTables T{{ta, te, tb, sl + N, sl + 2 * N, sl + 3 * N, sl}};
    int len = (int)N;
    f128* so = next_out(1);
    mp_round(T, len, false, mk(0, 0), true, so, st);
    std::vector<f128> rs;
    f128 last[7];
    for (int k = 0; k < n; k++) {
      // the last message is over the tables' two values; they fold here
      if (k == n - 1)
        for (int t = 0; t < 7; t++)
          CK(cudaMemcpyAsync(h_out + 4 + 2 * t, T.t[t], 2 * sizeof(f128), cudaMemcpyDeviceToHost, st));
      fetch(so, 3, h_out);
      P.mp_rounds.push_back({h_out[0], h_out[1], h_out[2]});
      for (int e = 0; e < 3; e++) tr.f128v(h_out[e]);
      const f128 rk = tr.sample();
      rs.push_back(rk);
      if (k + 1 < n) {
        len >>= 1;
        so = next_out(1);
        mp_round(T, len, true, rk, true, so, st);
      } else {
        for (int t = 0; t < 7; t++) {
          const f128 lo = h_out[4 + 2 * t], hi = h_out[5 + 2 * t];
          last[t] = fx(lo, hmul(rk, fx(hi, lo)));
        }
      }
    }
    // slot rounds (sd, then ss) over W, g indexed ss | sd << 1: slot 0 H_in
    // (no weight), 1 Z, 2 X_L, 3 X_R
    f128 w[4] = {mk(0, 0), last[1], hmul(last[0], fx(hone(), last[2])), hmul(last[0], last[2])};
    f128 g[4] = {last[6], last[3], last[4], last[5]};
    const f128 om = mk(2, 0), pts[3] = {hone(), om, fx(om, hone())};
    for (int h = 2; h >= 1; h >>= 1) {
      f128 sum[3] = {mk(0, 0), mk(0, 0), mk(0, 0)};
      for (int e = 0; e < 3; e++)
        for (int i = 0; i < h; i++) {
          const f128 wx = fx(w[i], hmul(pts[e], fx(w[i + h], w[i])));
          const f128 gx = fx(g[i], hmul(pts[e], fx(g[i + h], g[i])));
          sum[e] = fx(sum[e], hmul(wx, gx));
        }
      P.mp_rounds.push_back({sum[0], sum[1], sum[2]});
      for (int e = 0; e < 3; e++) tr.f128v(sum[e]);
      const f128 rk = tr.sample();
      rs.push_back(rk);
      for (int i = 0; i < h; i++) {
        w[i] = fx(w[i], hmul(rk, fx(w[i + h], w[i])));
        g[i] = fx(g[i], hmul(rk, fx(g[i + h], g[i])));
      }
    }
    P.g_at_point = pd_value = g[0];
    pd_point.assign(8 + (size_t)n, mk(0, 0));
    pd_point[0] = tau_pos;
    pd_point[1] = rs[(size_t)n + 1];  // sel_slot
    pd_point[2] = rs[(size_t)n];      // side
    for (int j = 0; j < n; j++) pd_point[8 + j] = rs[(size_t)(n - 1 - j)];
  }

  // ---- PCS open: ring switches + combine
  tr.label("flock-pcs-open-batch-v0");
  std::vector<f128> x_ab = r_inner_rest;
  x_ab.insert(x_ab.end(), x_outer.begin(), x_outer.end());
  std::vector<f128> x_c(r.begin() + 6, r.end());
  std::vector<f128> eqdd[2];
  f128 claim[2];
  {
    std::vector<f128> eqt = heq(std::vector<f128>(r_inner_rest.begin() + 1, r_inner_rest.end()));
    CK(cudaMemcpyAsync(eq_inner, eqt.data(), eqt.size() * sizeof(f128), cudaMemcpyHostToDevice, st));
    f128* ro = next_out(16);
    ring_shat_ab(zv_pre, eq_inner, k_log, ro, st);
    std::vector<f128> sv(128);
    fetch(ro, 128, sv.data());
    P.s_hat_v.push_back(sv);
    P.s_hat_v.push_back(s_hat_v_c);
  }
  for (int k = 0; k < 2; k++) {
    tr.label("flock-ring-switch-v0");
    const std::vector<f128>& sv = P.s_hat_v[k];
    tr.f128s(sv.data(), 128);
    std::vector<f128> rdp = tr.sample_vec(7);
    eqdd[k] = heq(rdp);
    // s_hat_u[b] bit i = bit b of s_hat_v[i];  claim = sum_b s_hat_u[b] eq''[b]
    std::vector<f128> u = transpose128(sv);
    f128 c = mk(0, 0);
    for (int bb = 0; bb < 128; bb++) c = fx(c, hmul(u[bb], eqdd[k][bb]));
    claim[k] = c;
  }
  f128* first_msg = nullptr;  // the first Ligerito message, when summed with b_combined
  f128 gam[2] = {tr.sample(), tr.sample()};
  f128 target = fx(hmul(gam[0], claim[0]), hmul(gam[1], claim[1]));
  // the packed-direct claim after the ring-switched ones (pcs.rs:844-872)
  f128 gpd = mk(0, 0);
  if (chain || merkle) {
    tr.label("flock-pcs-packed-direct-v0");
    tr.f128v(pd_value);
    gpd = tr.sample();
    target = fx(target, hmul(gpd, pd_value));
  }
  {
    std::vector<f128> T(2 * 16 * 256);
    for (int k = 0; k < 2; k++) {
      std::vector<f128> sc(128);
      for (int bb = 0; bb < 128; bb++) sc[bb] = hmul(gam[k], eqdd[k][bb]);
      for (int byte = 0; byte < 16; byte++) subset_sums8(sc.data() + 8 * byte, T.data() + (size_t)k * 4096 + byte * 256);
    }
    CK(cudaMemcpyAsync(bc_tabs, T.data(), T.size() * sizeof(f128), cudaMemcpyHostToDevice, st));
    // eq(suffix_k, i) = lo_k(i mod 2^lo_bits) * hi_k(i >> lo_bits), both tables
    // on the device; chunks of up to 2^14 values (each CTA builds its two
    // product tables once per chunk), as long as the four tables fit eqbuf
    const int n_vars = (int)x_ab.size() - 1;
    int lo_bits = std::min(n_vars, 14);
    while (lo_bits > 0 && 2 * ((1ull << lo_bits) + (1ull << (n_vars - lo_bits))) > n_words) lo_bits--;
    const int hi_bits = n_vars - lo_bits;
    f128* d = eqbuf[0];  // [lo0 | hi0 | lo1 | hi1]
    const size_t nlo = (size_t)1 << lo_bits, nhi = (size_t)1 << hi_bits;
    for (int k = 0; k < 2; k++) {
      const std::vector<f128>& xf = k == 0 ? x_ab : x_c;
      f128* base = d + k * (nlo + nhi);
      eq_build(xf.data() + 1, lo_bits, hone(), base, st);
      eq_build(xf.data() + 1 + lo_bits, hi_bits, hone(), base + nlo, st);
    }
    // with no packed-direct claim, b_combined is final here: the first
    // Ligerito message (over z and b_combined) is summed in the same pass
    if (!chain && !merkle && lo_bits >= 1) first_msg = next_out(1);
    ring_bcombined_ct(d, d + nlo, d + nlo + nhi, d + 2 * nlo + nhi, bc_tabs, bc_tabs + 4096, lo_bits, nhi, pp[1],
                      gs, st, first_msg ? z : nullptr, first_msg);
  }
  if (chain) {
    // b_combined += gpd eq(point): words w < 2R of block i (R packed words
    // per region) get gpd eq(tau_pos, w mod R) eq(s0*, w / R) eq(tau', i)
    // (pcs.rs:1236-1248)
    const int tl = chain_geom(hash).region_log - 7, R = 1 << tl;
    const std::vector<f128> ep = heq(std::vector<f128>(pd_point.begin(), pd_point.begin() + tl));
    const f128 s0 = pd_point[(size_t)tl];
    const f128 es[2] = {fx(hone(), s0), s0};
    std::vector<f128> c((size_t)2 * R);
    for (int wd = 0; wd < 2 * R; wd++) c[(size_t)wd] = hmul(gpd, hmul(ep[(size_t)(wd % R)], es[wd / R]));
    eq_table(std::vector<f128>(pd_point.begin() + (k_log - 7), pd_point.end()), scratch_eq());
    chain_scatter(pp[1], scratch_eq(), n_slots, (size_t)1 << (k_log - 7), c.data(), (int)c.size(), st);
  }
  if (merkle) {
    // words w = 0..7 of block i get gpd eq(tau_pos, w & 1) eq(sel, w >> 1 & 1)
    // eq(side, w >> 2) eq(instance, i)
    MpCoeffs c;
    for (int wd = 0; wd < 8; wd++) {
      f128 v = gpd;
      for (int j = 0; j < 3; j++) v = hmul(v, (wd >> j) & 1 ? pd_point[j] : fx(hone(), pd_point[j]));
      c.c[wd] = v;
    }
    eq_table(std::vector<f128>(pd_point.begin() + 8, pd_point.end()), scratch_eq());
    mp_scatter(pp[1], scratch_eq(), n_slots, c, st);
  }
  mark(7);

  // ---- Ligerito
  const Ladder& Ld = *lad;
  tr.label("flock-ligerito-basis-v0");
  tr.f128v(target);
  tr.bytes(P.root.data(), 32);
  P.lig_root = P.root;
  f128* f = z;       // current f, b
  f128* bb = pp[1];
  f128* fo = pp[2];
  f128* bo = pp[3];
  size_t flen = n_words;
  f128* mo = nullptr;  // the slot of the pending message
  auto push_msg = [&]() {
    fetch(mo, 2, h_out);
    P.sc_msgs.push_back({h_out[0], h_out[1]});
    tr.f128v(h_out[0]);
    tr.f128v(h_out[1]);
  };
  if (first_msg) {
    mo = first_msg;  // summed with b_combined (no next_out since: the slot is intact)
  } else {
    mo = next_out(1);
    lig_msg(f, bb, flen / 2, mo, gs, st);
  }
  push_msg();
  auto fold_round = [&](int bits) -> f128 {
    if (bits > 0) P.fold_nonces.push_back(grind(tr, (uint32_t)bits));
    f128 rch = tr.sample();
    mo = next_out(1);
    lig_fold_msg(f, bb, fo, bo, rch, flen / 4, true, mo, gs, st);
    // after the first fold f lives in the ping-pong pair (pp[0], pp[2]) / (pp[1], pp[3])
    if (f == z) { f = fo; fo = pp[0]; }
    else std::swap(f, fo);
    std::swap(bb, bo);
    flen /= 2;
    push_msg();
    return rch;
  };
  auto introduce = [&](const f128* bnew) {
    mo = next_out(1);
    lig_msg(f, bnew, flen / 2, mo, gs, st);
    push_msg();
    f128 be = tr.sample();
    axpy(bb, bnew, be, flen, st);
  };
  int n_cur = m - 7;
  auto do_ood = [&](int count) {
    for (int s = 0; s < count; s++) {
      std::vector<f128> zp = tr.sample_vec((size_t)n_cur);
      f128* eqz = scratch_eq();
      eq_table(zp, eqz);
      f128* io = next_out(1);
      inner(f, eqz, flen, io, G, st);
      f128 y;
      fetch(io, 1, &y);
      P.ood.push_back(y);
      tr.f128v(y);
      introduce(eqz);
    }
  };
  // induced basis of a queried level: transposed RS encoding of the
  // alpha-weighted query indicator, restricted to the message (n_cur vars)
  auto induce = [&](const std::vector<size_t>& q, const std::vector<f128>& alpha_v, int rate) {
    std::vector<f128> eqa = heq(alpha_v);
    size_t dlen = (size_t)1 << (n_cur + rate);
    CK(cudaMemsetAsync(induce_buf, 0, dlen * sizeof(f128), st));
    std::vector<uint64_t> qp(q.begin(), q.end());
    CK(cudaMemcpyAsync(idx, qp.data(), qp.size() * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(gather, eqa.data(), q.size() * sizeof(f128), cudaMemcpyHostToDevice, st));
    scatter(induce_buf, idx, gather, q.size(), st);
    f128* bind = scratch_eq();
    ntt_transposed_encode(induce_buf, bind, n_cur, rate, st);
    introduce(bind);
  };

  std::vector<f128> lane_rs;
  for (int j = 0; j < Ld.initial_k; j++) lane_rs.push_back(fold_round(std::max(0, Ld.fold_grind[0] - j)));
  n_cur -= Ld.initial_k;
  mark(8);
  // level 1 commit
  auto commit = [&](Level& L) {
    ntt_rs_encode(f, L.cw, L.log_msg_pos, L.lanes, L.rate, st);
    merkle_build(L.cw, L.positions, (size_t)L.lanes * 16, L.tree, merkle_fn, st);
    H32 rt = root_of(L.tree, L.positions);
    P.roots.push_back(rt);
    tr.bytes(rt.data(), 32);
  };
  commit(levels[0]);
  do_ood(Ld.ood.size() > 1 ? Ld.ood[1] : 0);
  P.grind_nonces.push_back(grind(tr, (uint32_t)Ld.grind[0]));
  {
    std::vector<size_t> q0 = sample_queries(tr, n_leaves0, (size_t)Ld.queries[0]);
    std::vector<f128> al = tr.sample_vec(ceil_log2((size_t)Ld.queries[0]));
    open(P.initial, cw0, tree0, n_leaves0, 64, q0);
    induce(q0, al, Ld.rate[0]);
  }
  const int rsteps = (int)Ld.ks.size();
  P.levels.reserve((size_t)rsteps);  // pending openings point into it
  for (int i = 0; i < rsteps; i++) {
    for (int j = 0; j < Ld.ks[i]; j++) fold_round(std::max(0, Ld.fold_grind[i + 1] - j));
    n_cur -= Ld.ks[i];
    Level& prev = levels[i];
    if (i == rsteps - 1) {
      P.yr.resize(flen);
      fetch(f, flen, P.yr.data());
      for (f128 v : P.yr) tr.f128v(v);
      P.grind_nonces.push_back(grind(tr, (uint32_t)Ld.grind[i + 1]));
      std::vector<size_t> ql = sample_queries(tr, prev.positions, (size_t)Ld.queries[i + 1]);
      tr.sample_vec(ceil_log2((size_t)Ld.queries[i + 1]));
      open(P.final_open, prev.cw, prev.tree, prev.positions, prev.lanes, ql);
      tr.sample();
      break;
    }
    commit(levels[i + 1]);
    do_ood((i + 2) < (int)Ld.ood.size() ? Ld.ood[i + 2] : 0);
    P.grind_nonces.push_back(grind(tr, (uint32_t)Ld.grind[i + 1]));
    std::vector<size_t> qi = sample_queries(tr, prev.positions, (size_t)Ld.queries[i + 1]);
    std::vector<f128> al = tr.sample_vec(ceil_log2((size_t)Ld.queries[i + 1]));
    P.levels.emplace_back();
    open(P.levels.back(), prev.cw, prev.tree, prev.positions, prev.lanes, qi);
    induce(qi, al, prev.rate);
  }
  mark(9);
  CK(cudaStreamSynchronize(st));
  finish_openings();
  std::vector<uint8_t> bytes = encode(P);
  return bytes;
}

void Setup::phase_times(double* ms) const {
  for (int i = 0; i < kPhases; i++) {
    float t = 0;
    if (cudaEventElapsedTime(&t, ev[i], ev[i + 1]) != cudaSuccess) t = -1;
    ms[i] = t;
  }
}

}  // namespace flock
